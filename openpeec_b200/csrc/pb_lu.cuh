// pb_lu.cuh — batched dense complex LU (partial pivoting) and triangular solves.
#pragma once
#include "pb_common.cuh"
#include <cublas_v2.h>

// Trailing-update engine of the LU.
enum pb_gemm_kind {
    PB_GEMM_FP64 = 0,   // complex FP64 GEMM (cuBLAS ZGEMM: the plain FP64 path)
    PB_GEMM_FP32 = 1,   // complex FP32 GEMM, the library's own SIMT kernel
    PB_GEMM_TC   = 2,   // complex FP32 GEMM on the tensor cores: the library's tcgen05
                        // kernel (split-TF32, 3 products, FP32 accumulation in TMEM,
                        // pb_tcgemm.cu); the SIMT kernel for updates thinner than its tile
    PB_GEMM_TC_BLAS = 3 // comparison baseline: cuBLAS's BF16x9 FP32 emulation of the same
                        // update as one real GEMM (B expanded to 2x2 real blocks)
};

struct pb_lu_engine {
    cublasHandle_t blas = nullptr;
    cudaStream_t stream = nullptr;
    int gemm_kind = PB_GEMM_FP64;
    long launches = 0;         // kernels launched (own kernels + library calls)
    // Scratch for PB_GEMM_TC_BLAS: the k x nc complex right operand expanded to the real
    // 2k x 2nc matrix [[re, im], [-im, re]] per entry, nb of them (4*k*nc floats each).
    // Owned by the caller (the sweep sizes it at 4*n*n bytes per matrix); without it, or
    // when an update needs more, the update runs on the SIMT kernel.
    float *emb = nullptr;
    size_t emb_cap = 0;        // bytes
    int tc_disabled = 0;       // set if the library rejects the emulated compute type
    int *tc_err = nullptr;     // device flag: a pipeline wait of the tensor-core kernel timed out
    int tc_used = 0;           // the tensor-core kernel ran since the flag was last checked
    void *coop = nullptr;      // scratch of the cooperative leaf panel (barriers, candidates, rows)
    size_t coop_cap = 0;       // bytes
};

// C (m x nc) -= A (m x k) * B (k x nc), complex FP32, row-major, batched with one stride,
// on the engine's stream with the engine's kernel choice (PB_GEMM_FP32 / TC / TC_BLAS).
// lower = 1: only entries with row >= column (C-local indices) are needed; tiles that lie
// entirely above that diagonal are skipped (the others are computed in full).
int pb_cgemm_sub(pb_lu_engine *e, int m, int nc, int k, const float2 *A, int lda, const float2 *B,
                 int ldb, float2 *C, int ldc, long long stride, int nb, int lower = 0);

int pb_lu_engine_init(pb_lu_engine *e, cudaStream_t s);
void pb_lu_engine_free(pb_lu_engine *e);

// Factorise nb matrices (row-major, order n, leading dimension ld, batch stride
// `stride` elements) in place. piv: [nb*n] device, info: [nb] device (-1 = regular,
// else first zero-pivot row). T = float or double.
template <typename T>
int pb_lu_factor(pb_lu_engine *e, int n, int nb, typename cplx_t<T>::type *a, int ld,
                 long stride, int *piv, int *info);

// Complex-symmetric factorisation A = L D L^T without pivoting, FP32, for nb matrices as
// pb_lu_factor (only the lower triangle of A is read). The result is stored like an
// unpivoted LU (unit L below the diagonal, U = D L^T on and above it) and piv is the
// identity, so pb_lu_perm and the LU solves apply unchanged. Returns PB_ERR_UNSUP when the
// panel does not fit in shared memory (orders above ~28 000); info as pb_lu_factor (a
// zero diagonal). Growth is not controlled: callers refine against the FP64 matrix.
int pb_ldl_factor(pb_lu_engine *e, int n, int nb, float2 *a, int ld, long stride, int *piv, int *info);
bool pb_ldl_supported(int n);     // the panel of order n fits (pb_ldl_factor will not return UNSUP)

// Row permutation perm[b*n + i] (row i of P*b comes from row perm[i]) from pivots.
int pb_lu_perm(pb_lu_engine *e, int n, int nb, const int *piv, int *perm);

// Solve A x = r for nb matrices x nrhs right-hand sides using the factors (type TF).
// r, x: FP64 complex [nb][nrhs][n] device (may alias). Each RHS is scaled by its
// max-norm before conversion to TF and scaled back afterwards. operm = 1: the factors are
// of the symmetrically permuted P A P^T (pb_sym_order), x = P^T y (x and r must not alias).
template <typename TF>
int pb_lu_solve_batched(pb_lu_engine *e, int n, int nb, int nrhs,
                        const typename cplx_t<TF>::type *lu, int ld, long stride,
                        const int *perm, const double2 *r, double2 *x, int operm = 0);

// Explicit inverse X = A^-1 (row-major n x n, device) of one FP64 system from its factors
// (pb_lu_factor / pb_lu_perm), for a matrix whose factors serve many solves.
int pb_lu_inverse(pb_lu_engine *e, int n, const double2 *lu, int ld, const int *perm, double2 *X);
// y = X r for a row-major n x n FP64 complex X (r and y must not alias).
int pb_gemv(pb_lu_engine *e, int n, const double2 *X, const double2 *r, double2 *y);

// Same with an indirection: CTA row y solves system sys[y] (vector slot, nullptr = y)
// with the factors of matrix lu_of[system] (nullptr = the system itself).
template <typename TF>
int pb_lu_solve_mapped(pb_lu_engine *e, int n, int nb, int nrhs,
                       const typename cplx_t<TF>::type *lu, int ld, long stride,
                       const int *perm, const double2 *r, double2 *x, const int *sys,
                       const int *lu_of, int operm = 0);

// pb_residual for the nb systems sys[0..nb) of a batch of nall; the norms of the other
// systems are left at 0. wv (optional, laid out like r): (|A||x| + |b|) per row.
int pb_residual_mapped(pb_lu_engine *e, int n, int nb, int nrhs, const double2 *a, int ld, long stride,
                       const double2 *b, const double2 *x, double2 *r, double *rn, double *bn, double *xn,
                       double *an, int nall, const int *sys, double *cw = nullptr, double *wv = nullptr);

// pb_residual_mapped for one right-hand side of complex-symmetric systems of which only the
// lower triangle is read (half the bytes); deterministic. Norms as pb_residual_mapped (an,
// wv optional: then |A| row sums / (|A||x| + |b|) are formed too). scratch: device buffer
// of pb_sym_residual_scratch(n, nb) bytes.
size_t pb_sym_residual_scratch(int n, int nb);
int pb_sym_residual_mapped(pb_lu_engine *e, int n, int nb, const double2 *a, long stride, const double2 *b,
                           const double2 *x, double2 *r, double *rn, double *bn, double *xn, double *an, int nall,
                           const int *sys, double *wv, void *scratch);
// Symmetric ordering for the unpivoted L D L^T: per system perm = the unknowns by decreasing
// |A_kk| / sum_j |A_kj| (a: lower-triangle FP64 systems), and a32 (lower triangle) = the
// permuted matrix in FP32. n <= 16384 (else PB_ERR_UNSUP); scratch as pb_sym_residual.
int pb_sym_order(pb_lu_engine *e, int n, int nb, const double2 *a, long long stride, float2 *a32, int *perm,
                 void *scratch);
// Upper triangle := transposed lower triangle of nb FP64 matrices (stride in elements).
int pb_sym_mirror(pb_lu_engine *e, int n, int nb, double2 *a, long long stride);

// y = A x for the nb systems sys[0..nb) (nullptr = 0..nb), nrhs vectors each.
int pb_matvec_mapped(pb_lu_engine *e, int n, int nb, int nrhs, const double2 *a, int ld, long stride,
                     const double2 *x, double2 *y, const int *sys);

// r = b - A x for nb FP64 matrices, nrhs vectors each; also writes the infinity norms
// (max |re|,|im| component) of r, b and x per vector into rn, bn, xn [nb*nrhs] and,
// when an != nullptr, the infinity norm of each matrix (max row sum of |re|+|im|); when
// cw != nullptr, the componentwise backward error max_i |r_i| / (|A||x| + |b|)_i per vector
// (Oettli-Prager, with |z| measured as |re|+|im|).
int pb_residual(pb_lu_engine *e, int n, int nb, int nrhs, const double2 *a, int ld,
                long stride, const double2 *b, const double2 *x, double2 *r, double *rn,
                double *bn, double *xn, double *an, double *cw = nullptr);
