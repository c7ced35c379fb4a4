// pb_lu.cu — batched dense complex LU with partial pivoting, for many frequencies at
// once, plus the triangular solves and the FP64 residual used by iterative refinement.
//
// Algorithm: recursive (Toledo) right-looking LU over column halves. Leaves of up to
// 32 columns are factored by one CTA per matrix that keeps SW columns of the panel in
// shared memory (pivot search = block argmax of |re|+|im| with first-index tie-break,
// the reference's rule in src/lu.c:19-30); everything above the leaves is row swaps,
// a unit-lower triangular solve and a complex GEMM trailing update.
// Row-major storage, like the reference (a[i*n+j]).
#include <atomic>
#include "pb_lu.cuh"
#include "pb_tcgemm.cuh"
#include <climits>
#include <cuComplex.h>
#include <dlfcn.h>

template <typename T> using T2_t = typename cplx_t<T>::type;

// ---------------------------------------------------------------- block argmax
__device__ __forceinline__ void argmax_pair(double &m, int &i, double m2, int i2)
{
    if (m2 > m || (m2 == m && i2 < i)) { m = m2; i = i2; }
}

// Block-wide argmax; result broadcast to all threads. Caller must __syncthreads()
// before reusing sm/si.
__device__ void block_argmax(double &m, int &i, double *sm, int *si)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double m2 = __shfl_down_sync(0xffffffffu, m, o);
        const int i2 = __shfl_down_sync(0xffffffffu, i, o);
        argmax_pair(m, i, m2, i2);
    }
    if (lane == 0) { sm[warp] = m; si[warp] = i; }
    __syncthreads();
    if (warp == 0) {
        m = (lane < nw) ? sm[lane] : -1.0;
        i = (lane < nw) ? si[lane] : INT_MAX;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double m2 = __shfl_down_sync(0xffffffffu, m, o);
            const int i2 = __shfl_down_sync(0xffffffffu, i, o);
            argmax_pair(m, i, m2, i2);
        }
        if (lane == 0) { sm[32] = m; si[32] = i; }
    }
    __syncthreads();
    m = sm[32];
    i = si[32];
}

// 1/z with scaling so that |z|^2 cannot under/overflow in FP32.
template <typename T2> __device__ __forceinline__ T2 safe_inv(T2 z)
{
    const auto s = fmax(fabs((double)z.x), fabs((double)z.y));
    if (s <= 0) return mk2<T2>(0, 0);
    const double zr = z.x / s, zi = z.y / s;
    const double d = (zr * zr + zi * zi) * s;
    return mk2<T2>(zr / d, -zi / d);
}

// ---------------------------------------------------------------- leaf panel
// Factor columns [k0, k0+w) (w <= 32) over rows [k0, n) of matrix blockIdx.x, SW
// columns at a time in shared memory. Swaps are applied to the leaf's own columns only.
// G = true (orders whose panel column does not fit in shared memory, FP64 above ~14 000
// unknowns): the SW columns are worked on in place in global memory instead.
template <typename T, int SW, bool G>
__global__ void __launch_bounds__(1024)
k_lu_leaf(T2_t<T> *a, int n, int ld, long long stride, int k0, int w, int *piv, int *info)
{
    typedef T2_t<T> T2;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double red_m[33];
    __shared__ int red_i[33];
    const int m = n - k0;
    T2 *spm = reinterpret_cast<T2 *>(smraw);      // [m][SW] (G = false)
    T2 *urow = G ? spm : spm + (size_t)m * SW;     // [SW][32]
    const int b = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    a += (long long)b * stride;
    piv += (long long)b * n;

    for (int s0 = 0; s0 < w; s0 += SW) {
        const int sw = min(SW, w - s0), c0 = k0 + s0;
        // element (r, t) of the sub-panel: row k0 + r, column c0 + t
        auto P = [&](int r, int t) -> T2 & {
            return G ? a[(long long)(k0 + r) * ld + c0 + t] : spm[r * SW + t];
        };
        if (!G)
            for (int e = tid; e < m * sw; e += nt) {
                const int r = e / sw, t = e - r * sw;
                spm[r * SW + t] = a[(long long)(k0 + r) * ld + c0 + t];
            }
        __syncthreads();
        for (int t = 0; t < sw; t++) {
            const int c = c0 + t;
            double bm = -1.0;
            int bi = INT_MAX;
            for (int r = c + tid; r < n; r += nt) {
                const double mm = cmag1(P(r - k0, t));
                if (mm > bm) { bm = mm; bi = r; }
            }
            block_argmax(bm, bi, red_m, red_i);
            const int ip = (bi == INT_MAX) ? c : bi;
            if (tid == 0) {
                piv[c] = ip;
                if (bm < 1e-30 && info[b] < 0) info[b] = c;
            }
            if (ip != c) {
                for (int e = tid; e < w; e += nt) {
                    const int col = k0 + e;
                    if (col >= c0 && col < c0 + sw) {
                        T2 *x = &P(c - k0, col - c0), *y = &P(ip - k0, col - c0);
                        const T2 tmp = *x; *x = *y; *y = tmp;
                    } else {
                        T2 *x = &a[(long long)c * ld + col], *y = &a[(long long)ip * ld + col];
                        const T2 tmp = *x; *x = *y; *y = tmp;
                    }
                }
            }
            __syncthreads();
            const T2 pinv = safe_inv(P(c - k0, t));
            for (int r = c + 1 + tid; r < n; r += nt) {
                const T2 l = cmul(P(r - k0, t), pinv);
                P(r - k0, t) = l;
                for (int tt = t + 1; tt < sw; tt++) P(r - k0, tt) = cfms(P(r - k0, tt), l, P(c - k0, tt));
            }
            __syncthreads();
        }
        if (!G)
            for (int e = tid; e < m * sw; e += nt) {
                const int r = e / sw, t = e - r * sw;
                a[(long long)(k0 + r) * ld + c0 + t] = spm[r * SW + t];
            }
        const int c1 = c0 + sw, nr = k0 + w - c1;
        if (nr > 0) {
            // U rows of this sub-panel for the remaining leaf columns
            for (int col = c1 + tid; col < k0 + w; col += nt) {
                for (int t = 0; t < sw; t++) {
                    T2 v = a[(long long)(c0 + t) * ld + col];
                    for (int tp = 0; tp < t; tp++)
                        v = cfms(v, P(c0 + t - k0, tp), urow[tp * 32 + (col - c1)]);
                    urow[t * 32 + (col - c1)] = v;
                    a[(long long)(c0 + t) * ld + col] = v;
                }
            }
            __syncthreads();
            const long long tot = (long long)(n - c1) * nr;
            for (long long e = tid; e < tot; e += nt) {
                const int r = c1 + (int)(e / nr), col = c1 + (int)(e % nr);
                T2 v = a[(long long)r * ld + col];
#pragma unroll
                for (int t = 0; t < SW; t++)
                    if (t < sw) v = cfms(v, P(r - k0, t), urow[t * 32 + (col - c1)]);
                a[(long long)r * ld + col] = v;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- cooperative leaf panel
// Barrier among the P CTAs of one matrix (mb[0] arrivals, mb[1] generation), bounded: a
// wait longer than about a second sets *err and returns false, and the kernel returns.
__device__ __forceinline__ bool panel_bar(unsigned *mb, int P, unsigned &gen, int *err, int *ok_s)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        const unsigned g = gen;
        if (atomicAdd(&mb[0], 1u) == (unsigned)P - 1) {
            atomicExch(&mb[0], 0u);
            __threadfence();
            atomicExch(&mb[1], g + 1);
        } else {
            long long it = 0;
            while (atomicAdd(&mb[1], 0u) == g) {
                if (++it > (1LL << 23) || ((it & 1023) == 0 && atomicAdd(err, 0) != 0)) {
                    ok = 0;
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        *ok_s = ok;
    }
    __syncthreads();
    gen++;
    return *ok_s != 0;
}

// The leaf panel of k_lu_leaf for a few large matrices: the panel's rows [k0, n) are split
// over the P CTAs of a matrix (blockIdx.y), RS rows each, held in shared memory for the
// whole panel (all w <= 32 columns). Per column: every CTA's candidate (largest |re|+|im|,
// first index), one barrier, the same global choice in every CTA, the owners of the pivot
// row and of row c publish them, a second barrier, the swap and the rank-1 update of the
// CTA's own rows. The arithmetic of every entry is that of k_lu_leaf (the same cfms
// sequence), so the factors are the same; the panel's row traffic is spread over P SMs
// instead of one. Needs all P * nb CTAs resident (cooperative launch).
template <typename T>
__global__ void __launch_bounds__(256)
k_lu_leaf_coop(T2_t<T> *a, int n, int ld, long long stride, int k0, int w, int *piv, int *info, int P, int RS,
               unsigned *bar, double *part_m, int *part_i, T2_t<T> *rows, int *err)
{
    typedef T2_t<T> T2;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double red_m[33];
    __shared__ int red_i[33];
    __shared__ T2 pr[32];
    __shared__ double s_bm;
    __shared__ int s_bi, ok_s;
    T2 *S = reinterpret_cast<T2 *>(smraw);        // [RS][32]
    const int p = blockIdx.x, b = blockIdx.y, tid = threadIdx.x, nt = blockDim.x;
    a += (long long)b * stride;
    piv += (long long)b * n;
    unsigned *mb = bar + 2 * b;
    double *pm = part_m + (long long)b * P;
    int *pi = part_i + (long long)b * P;
    T2 *prow = rows + (long long)b * 64, *crow = prow + 32;
    const int r0 = k0 + p * RS, r1 = min(n, r0 + RS), nr = max(0, r1 - r0);
    for (int e = tid; e < nr * w; e += nt) {
        const int r = e / w, t = e - r * w;
        S[r * 32 + t] = a[(long long)(r0 + r) * ld + k0 + t];
    }
    __syncthreads();
    unsigned gen = 0;
    for (int t = 0; t < w; t++) {
        const int c = k0 + t;
        double bm = -1.0;
        int bi = INT_MAX;
        for (int r = max(c, r0) + tid; r < r1; r += nt) {
            const double mm = cmag1(S[(r - r0) * 32 + t]);
            if (mm > bm) { bm = mm; bi = r; }
        }
        block_argmax(bm, bi, red_m, red_i);
        if (tid == 0) { pm[p] = bm; pi[p] = bi; }
        if (!panel_bar(mb, P, gen, err, &ok_s)) return;
        if (tid < 32) {                                // the same choice in every CTA
            double m = -1.0;
            int i = INT_MAX;
            for (int q = tid; q < P; q += 32) argmax_pair(m, i, __ldcg(&pm[q]), __ldcg(&pi[q]));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double m2 = __shfl_down_sync(0xffffffffu, m, o);
                const int i2 = __shfl_down_sync(0xffffffffu, i, o);
                argmax_pair(m, i, m2, i2);
            }
            if (tid == 0) { s_bm = m; s_bi = i; }
        }
        __syncthreads();
        const int ip = (s_bi == INT_MAX) ? c : s_bi;
        if (ip >= r0 && ip < r1)
            for (int tt = tid; tt < w; tt += nt) prow[tt] = S[(ip - r0) * 32 + tt];
        if (ip != c && c >= r0 && c < r1)
            for (int tt = tid; tt < w; tt += nt) crow[tt] = S[(c - r0) * 32 + tt];
        if (!panel_bar(mb, P, gen, err, &ok_s)) return;
        for (int tt = tid; tt < w; tt += nt) pr[tt] = __ldcg(&prow[tt]);
        if (ip != c && ip >= r0 && ip < r1)
            for (int tt = tid; tt < w; tt += nt) S[(ip - r0) * 32 + tt] = __ldcg(&crow[tt]);
        __syncthreads();
        if (c >= r0 && c < r1)
            for (int tt = tid; tt < w; tt += nt) S[(c - r0) * 32 + tt] = pr[tt];
        if (p == 0 && tid == 0) {
            piv[c] = ip;
            if (s_bm < 1e-30 && info[b] < 0) info[b] = c;
        }
        __syncthreads();
        const T2 pinv = safe_inv(pr[t]);
        for (int r = max(c + 1, r0) + tid; r < r1; r += nt) {
            T2 *row = S + (r - r0) * 32;
            const T2 l = cmul(row[t], pinv);
            row[t] = l;
            for (int tt = t + 1; tt < w; tt++) row[tt] = cfms(row[tt], l, pr[tt]);
        }
        __syncthreads();
    }
    for (int e = tid; e < nr * w; e += nt) {
        const int r = e / w, t = e - r * w;
        a[(long long)(r0 + r) * ld + k0 + t] = S[r * 32 + t];
    }
}

// ---------------------------------------------------------------- row swaps
template <typename T>
__global__ void k_swap_rows(T2_t<T> *a, int ld, long long stride, const int *piv, int n,
                            int r0, int r1, int c0, int c1)
{
    typedef T2_t<T> T2;
    const int col = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= c1) return;
    const int b = blockIdx.y;
    a += (long long)b * stride;
    piv += (long long)b * n;
    for (int r = r0; r < r1; r++) {
        const int p = piv[r];
        if (p != r) {
            T2 *x = &a[(long long)r * ld + col], *y = &a[(long long)p * ld + col];
            const T2 t = *x; *x = *y; *y = t;
        }
    }
}

// ---------------------------------------------------------------- small TRSM
// X = L^-1 B, L unit lower w x w (w <= 64) at a[r0.., r0..], B = a[r0..r0+w, c0..c1).
template <typename T>
__global__ void __launch_bounds__(64)
k_trsm_small(T2_t<T> *a, int ld, long long stride, int r0, int w, int c0, int c1)
{
    typedef T2_t<T> T2;
    extern __shared__ __align__(16) unsigned char smraw[];
    T2 *L = reinterpret_cast<T2 *>(smraw);      // [w][w]
    T2 *X = L + w * w;                            // [w][64]
    const int b = blockIdx.y, tid = threadIdx.x;
    a += (long long)b * stride;
    const int cb = c0 + blockIdx.x * 64;
    for (int e = tid; e < w * w; e += 64) {
        const int r = e / w, c = e - r * w;
        L[e] = (c < r) ? a[(long long)(r0 + r) * ld + r0 + c] : mk2<T2>(0, 0);
    }
    for (int e = tid; e < w * 64; e += 64) {
        const int r = e / 64, c = e - r * 64;
        X[e] = (cb + c < c1) ? a[(long long)(r0 + r) * ld + cb + c] : mk2<T2>(0, 0);
    }
    __syncthreads();
    if (cb + tid < c1) {
        for (int r = 1; r < w; r++) {
            T2 v = X[r * 64 + tid];
            for (int c = 0; c < r; c++) v = cfms(v, L[r * w + c], X[c * 64 + tid]);
            X[r * 64 + tid] = v;
        }
        for (int r = 0; r < w; r++) a[(long long)(r0 + r) * ld + cb + tid] = X[r * 64 + tid];
    }
}

// ---------------------------------------------------------------- GEMM wrapper
// C(m x nc) -= A(m x k) * B(k x nc), row-major, batched with strides.
template <typename T>
static int gemm_sub(pb_lu_engine *e, int m, int nc, int k, const T2_t<T> *A, int lda,
                    const T2_t<T> *B, int ldb, T2_t<T> *Cm, int ldc, long long stride, int nb);

template <>
int gemm_sub<double>(pb_lu_engine *e, int m, int nc, int k, const double2 *A, int lda,
                     const double2 *B, int ldb, double2 *Cm, int ldc, long long stride, int nb)
{
    if (m <= 0 || nc <= 0 || k <= 0) return PB_OK;
    const cuDoubleComplex alpha = make_cuDoubleComplex(-1, 0), beta = make_cuDoubleComplex(1, 0);
    cublasStatus_t s = cublasZgemmStridedBatched(
        e->blas, CUBLAS_OP_N, CUBLAS_OP_N, nc, m, k, &alpha,
        (const cuDoubleComplex *)B, ldb, stride, (const cuDoubleComplex *)A, lda, stride, &beta,
        (cuDoubleComplex *)Cm, ldc, stride, nb);
    e->launches++;
    if (s != CUBLAS_STATUS_SUCCESS) { pb_set_error("cublasZgemmStridedBatched failed (%d)", (int)s); return PB_ERR_CUDA; }
    return PB_OK;
}

// Right operand B (k x nc complex, row-major, leading dimension ldb, batch stride sb)
// to the real 2k x 2nc row-major matrix with the 2x2 block [[br, bi], [-bi, br]] in
// place of each entry b = br + j bi. With A and C read as real matrices (interleaved
// re/im = 2 real columns per complex column), C_real -= A_real * B_emb is exactly the
// complex update: C[i][2j] -= sum_l ar br - ai bi, C[i][2j+1] -= sum_l ar bi + ai br.
__global__ void k_embed_right(const float2 *__restrict__ b, int k, int nc, int ldb, long long sb,
                              float *__restrict__ be)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = blockIdx.y;
    const long long z = blockIdx.z;
    if (j >= nc) return;
    const float2 v = b[z * sb + (long long)l * ldb + j];
    float2 *r0 = reinterpret_cast<float2 *>(be + z * 4LL * k * nc + (2LL * l) * (2LL * nc) + 2LL * j);
    float2 *r1 = r0 + nc;                       // next real row: 2nc floats = nc float2
    *r0 = make_float2(v.x, v.y);
    *r1 = make_float2(-v.y, v.x);
}

// Thin updates stay on the SIMT complex GEMM: below 128 in any dimension the BF16x9
// real form was measured slower on B200 (launch and split overheads dominate).
static const int kTcMinDim = 128;

// cublasSetEmulationStrategy exists from cuBLAS 12.9 on. It is looked up in the
// libcublas.so.12 this process has loaded rather than linked: a host may have loaded an
// older copy first (e.g. a Python framework's bundled cuBLAS), and the library must still
// load there. Without it the trailing updates stay on the SIMT complex GEMM.
typedef cublasStatus_t (*pb_set_emulation_fn)(cublasHandle_t, cublasEmulationStrategy_t);
static pb_set_emulation_fn set_emulation()
{
    static const pb_set_emulation_fn fn = []() -> pb_set_emulation_fn {
        void *h = dlopen("libcublas.so.12", RTLD_LAZY | RTLD_NOLOAD);
        return h ? reinterpret_cast<pb_set_emulation_fn>(dlsym(h, "cublasSetEmulationStrategy")) : nullptr;
    }();
    return fn;
}

// Complex FP32 update C -= A * B on the SIMT pipes, for updates thinner than the
// tensor-core kernel's 128 x 128 x 16 tile: 64 x 64 complex outputs per 256-thread block,
// 4 x 4 per thread, k staged in shared memory 16 at a time, FP32 fused multiply-adds.
__global__ void __launch_bounds__(256)
k_cgemm_simt(const float2 *__restrict__ A, int lda, const float2 *__restrict__ B, int ldb,
             float2 *__restrict__ C, int ldc, long long stride, int m, int nc, int k, int lower)
{
    if (lower && (int)(blockIdx.y + 1) * 64 <= (int)blockIdx.x * 64) return;   // tile above the diagonal
    __shared__ float2 As[16][65];               // [kk][row], padded against bank conflicts
    __shared__ float2 Bs[16][64];               // [kk][col]
    const long long bo = (long long)blockIdx.z * stride;
    A += bo;
    B += bo;
    C += bo;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float2 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = make_float2(0.f, 0.f);
    for (int k0 = 0; k0 < k; k0 += 16) {
        for (int e = threadIdx.x; e < 1024; e += 256) {
            const int r = e >> 4, kk = e & 15;
            As[kk][r] = (m0 + r < m && k0 + kk < k) ? A[(long long)(m0 + r) * lda + k0 + kk] : make_float2(0.f, 0.f);
            const int kb = e >> 6, c = e & 63;
            Bs[kb][c] = (k0 + kb < k && n0 + c < nc) ? B[(long long)(k0 + kb) * ldb + n0 + c] : make_float2(0.f, 0.f);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; kk++) {
            float2 a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    acc[i][j].x = fmaf(a[i].x, b[j].x, fmaf(-a[i].y, b[j].y, acc[i][j].x));
                    acc[i][j].y = fmaf(a[i].x, b[j].y, fmaf(a[i].y, b[j].x, acc[i][j].y));
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int r = m0 + ty + 16 * i;
        if (r >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int c = n0 + tx + 16 * j;
            if (c >= nc) continue;
            float2 &v = C[(long long)r * ldc + c];
            v.x -= acc[i][j].x;
            v.y -= acc[i][j].y;
        }
    }
}

// cuBLAS's BF16x9 FP32 emulation of the update as one real GEMM (comparison baseline,
// PB_GEMM_TC_BLAS). Returns PB_ERR_UNSUP when the library or the scratch cannot serve it.
static int gemm_sub_cublas_bf16x9(pb_lu_engine *e, int m, int nc, int k, const float2 *A, int lda,
                                  const float2 *B, int ldb, float2 *Cm, int ldc, long long stride, int nb)
{
    const size_t need = (size_t)nb * 4 * (size_t)k * nc * sizeof(float);
    const pb_set_emulation_fn set_emu = set_emulation();
    if (!set_emu) e->tc_disabled = 1;
    if (e->tc_disabled || !e->emb || need > e->emb_cap || m < kTcMinDim || nc < kTcMinDim || k < kTcMinDim)
        return PB_ERR_UNSUP;
    k_embed_right<<<dim3(ceil_div(nc, 128), k, nb), 128, 0, e->stream>>>(B, k, nc, ldb, stride, e->emb);
    PB_CHECK_LAUNCH();
    e->launches++;
    const float ra = -1.0f, rb = 1.0f;
    cublasSetMathMode(e->blas, CUBLAS_DEFAULT_MATH);
    set_emu(e->blas, CUBLAS_EMULATION_STRATEGY_EAGER);
    // row-major real C (m x 2nc) -= A (m x 2k) * Bemb (2k x 2nc); cuBLAS is
    // column-major, so it computes the transpose: C^T = Bemb^T A^T.
    const cublasStatus_t s = cublasGemmStridedBatchedEx(
        e->blas, CUBLAS_OP_N, CUBLAS_OP_N, 2 * nc, m, 2 * k, &ra, e->emb, CUDA_R_32F, 2 * nc,
        4LL * k * nc, A, CUDA_R_32F, 2 * lda, 2 * stride, &rb, Cm, CUDA_R_32F, 2 * ldc, 2 * stride, nb,
        CUBLAS_COMPUTE_32F_EMULATED_16BFX9, CUBLAS_GEMM_DEFAULT);
    set_emu(e->blas, CUBLAS_EMULATION_STRATEGY_DEFAULT);
    cublasSetMathMode(e->blas, CUBLAS_PEDANTIC_MATH);
    e->launches++;
    if (s == CUBLAS_STATUS_SUCCESS) return PB_OK;
    if (s != CUBLAS_STATUS_NOT_SUPPORTED) {
        pb_set_error("BF16x9 real GEMM failed (%d)", (int)s);
        return PB_ERR_CUDA;
    }
    e->tc_disabled = 1;                     // library without the emulation: SIMT from now on
    return PB_ERR_UNSUP;
}

int pb_cgemm_sub(pb_lu_engine *e, int m, int nc, int k, const float2 *A, int lda, const float2 *B,
                 int ldb, float2 *Cm, int ldc, long long stride, int nb, int lower)
{
    if (m <= 0 || nc <= 0 || k <= 0 || nb <= 0) return PB_OK;
    if (e->gemm_kind == PB_GEMM_TC && m >= 128 && nc >= 128 && k >= 16 &&
        pb_cgemm_tc_ok(A, lda, B, ldb, Cm, ldc, stride, nb)) {
        if (!e->tc_err) {
            PB_CUDA(cudaMalloc(&e->tc_err, sizeof(int)));
            PB_CUDA(cudaMemsetAsync(e->tc_err, 0, sizeof(int), e->stream));
        }
        e->launches++;
        e->tc_used = 1;
        return pb_cgemm_tc(m, nc, k, A, lda, B, ldb, Cm, ldc, stride, nb, e->tc_err, e->stream, lower);
    }
    if (e->gemm_kind == PB_GEMM_TC_BLAS) {
        const int r = gemm_sub_cublas_bf16x9(e, m, nc, k, A, lda, B, ldb, Cm, ldc, stride, nb);
        if (r != PB_ERR_UNSUP) return r;
    }
    k_cgemm_simt<<<dim3(ceil_div(nc, 64), ceil_div(m, 64), nb), 256, 0, e->stream>>>(A, lda, B, ldb, Cm, ldc,
                                                                                       stride, m, nc, k, lower);
    e->launches++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

// The tensor-core kernel reports a timed-out pipeline wait through a device flag; read it
// (one stream synchronisation) after a factorisation that used the kernel.
static int check_tc(pb_lu_engine *e)
{
    if (!e->tc_used || !e->tc_err) return PB_OK;
    e->tc_used = 0;
    int h = 0;
    PB_CUDA(cudaMemcpyAsync(&h, e->tc_err, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    PB_CUDA(cudaStreamSynchronize(e->stream));
    if (h) {
        PB_CUDA(cudaMemsetAsync(e->tc_err, 0, sizeof(int), e->stream));
        pb_set_error("factorisation: a device wait timed out (tensor-core pipeline or panel barrier); "
                     "the factors are invalid");
        return PB_ERR_CUDA;
    }
    return PB_OK;
}

template <>
int gemm_sub<float>(pb_lu_engine *e, int m, int nc, int k, const float2 *A, int lda,
                    const float2 *B, int ldb, float2 *Cm, int ldc, long long stride, int nb)
{
    return pb_cgemm_sub(e, m, nc, k, A, lda, B, ldb, Cm, ldc, stride, nb);
}

int pb_lu_engine_init(pb_lu_engine *e, cudaStream_t s)
{
    e->stream = s;
    if (cublasCreate(&e->blas) != CUBLAS_STATUS_SUCCESS) {
        pb_set_error("cublasCreate failed");
        return PB_ERR_CUDA;
    }
    cublasSetStream(e->blas, s);
    cublasSetMathMode(e->blas, CUBLAS_PEDANTIC_MATH);
    return PB_OK;
}

void pb_lu_engine_free(pb_lu_engine *e)
{
    if (e->blas) cublasDestroy(e->blas);
    e->blas = nullptr;
    if (e->tc_err) cudaFree(e->tc_err);
    e->tc_err = nullptr;
    if (e->coop) cudaFree(e->coop);
    e->coop = nullptr;
    e->coop_cap = 0;
}

// ---------------------------------------------------------------- recursion
template <typename T> static int leaf_sw(int m, size_t *smem)
{
    int dev = 0, cap = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&cap, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t avail = (size_t)cap - 1024;
    const size_t es = sizeof(T2_t<T>);
    for (int sw = 4; sw >= 1; sw >>= 1) {
        const size_t need = ((size_t)m * sw + (size_t)sw * 32) * es;
        if (need <= avail) { *smem = need; return sw; }
    }
    return 0;
}

template <typename T, int SW, bool G = false>
static int launch_leaf(pb_lu_engine *e, T2_t<T> *a, int n, int ld, long long stride, int nb,
                       int k0, int w, int *piv, int *info, size_t smem)
{
    static std::atomic<unsigned long long> attr_set{0};   // per device, before any launch relies on it
    PB_TRY(pb_smem_optin(k_lu_leaf<T, SW, G>, pb_smem_cap() - 1024, attr_set));
    // the panel has m = n - k0 rows: a CTA no wider than the panel (at least 128 threads)
    // lets several small systems share an SM (batches of small structures); the pivot
    // search and the updates do not depend on the thread count, so results are unchanged
    const int m = n - k0, nt = std::min(1024, std::max(128, (m + 31) / 32 * 32));
    k_lu_leaf<T, SW, G><<<nb, nt, smem, e->stream>>>(a, n, ld, stride, k0, w, piv, info);
    e->launches++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

// The cooperative panel for nb matrices of panel height m, if it applies: one CTA per SM
// at most, P >= 4 CTAs per matrix of at least 32 rows each, the CTA's rows within shared
// memory. launched = false: the one-CTA panel should run.
template <typename T>
static int launch_leaf_coop(pb_lu_engine *e, T2_t<T> *a, int n, int ld, long long stride, int nb, int k0, int w,
                            int *piv, int *info, bool &launched)
{
    launched = false;
    const int m = n - k0;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (m < 1024 || nb > nsm / 4) return PB_OK;
    const int P = std::min(nsm / nb, (m + 31) / 32);
    if (P < 4) return PB_OK;
    const int RS = (m + P - 1) / P;
    const size_t es = sizeof(T2_t<T>), smem = (size_t)RS * 32 * es;
    if (smem + 4096 > (size_t)pb_smem_cap()) return PB_OK;
    static std::atomic<unsigned long long> attr_set{0};   // per device
    PB_TRY(pb_smem_optin(k_lu_leaf_coop<T>, pb_smem_cap() - 1024, attr_set));
    int per_sm = 0;
    PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lu_leaf_coop<T>, 256, smem));
    if (per_sm * nsm < P * nb) return PB_OK;
    // scratch: barriers, candidates, the two published rows
    const size_t need = 16 * (size_t)nb + (8 + 4) * (size_t)P * nb + 64 * es * nb + 64;
    if (e->coop_cap < need) {
        if (e->coop) cudaFree(e->coop);
        e->coop = nullptr;
        e->coop_cap = 0;
        PB_CUDA(cudaMalloc(&e->coop, need));
        e->coop_cap = need;
    }
    if (!e->tc_err) {
        PB_CUDA(cudaMalloc(&e->tc_err, sizeof(int)));
        PB_CUDA(cudaMemsetAsync(e->tc_err, 0, sizeof(int), e->stream));
    }
    char *base = (char *)e->coop;
    unsigned *bar = (unsigned *)base;
    T2_t<T> *rows = (T2_t<T> *)(base + 16 * (size_t)nb);
    double *pm = (double *)((char *)rows + 64 * es * nb);
    int *pi = (int *)(pm + (size_t)P * nb);
    PB_CUDA(cudaMemsetAsync(bar, 0, 8 * (size_t)nb, e->stream));
    int Pv = P, RSv = RS;
    void *args[] = {&a, &n, &ld, &stride, &k0, &w, &piv, &info, &Pv, &RSv, &bar, &pm, &pi, &rows, &e->tc_err};
    PB_CUDA(cudaLaunchCooperativeKernel((void *)k_lu_leaf_coop<T>, dim3(P, nb), dim3(256), args, smem, e->stream));
    e->launches++;
    e->tc_used = 1;                     // check_tc reads the wait-timeout flag
    launched = true;
    return PB_OK;
}

template <typename T>
static int swap_rows(pb_lu_engine *e, T2_t<T> *a, int n, int ld, long long stride, int nb,
                     const int *piv, int r0, int r1, int c0, int c1)
{
    if (c1 <= c0 || r1 <= r0) return PB_OK;
    dim3 g(ceil_div(c1 - c0, 128), nb);
    k_swap_rows<T><<<g, 128, 0, e->stream>>>(a, ld, stride, piv, n, r0, r1, c0, c1);
    e->launches++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

template <typename T>
static int trsm_rec(pb_lu_engine *e, T2_t<T> *a, int ld, long long stride, int nb, int r0,
                    int w, int c0, int c1)
{
    if (c1 <= c0 || w <= 0) return PB_OK;
    if (w <= 64) {
        static std::atomic<unsigned long long> attr_set{0};   // per device
        PB_TRY(pb_smem_optin(k_trsm_small<T>, (64 * 64 + 64 * 64) * (int)sizeof(T2_t<T>), attr_set));
        const size_t smem = (size_t)(w * w + w * 64) * sizeof(T2_t<T>);
        dim3 g(ceil_div(c1 - c0, 64), nb);
        k_trsm_small<T><<<g, 64, smem, e->stream>>>(a, ld, stride, r0, w, c0, c1);
        e->launches++;
        PB_CHECK_LAUNCH();
        return PB_OK;
    }
    const int w1 = ((w / 2 + 31) / 32) * 32;
    PB_TRY(trsm_rec<T>(e, a, ld, stride, nb, r0, w1, c0, c1));
    PB_TRY(gemm_sub<T>(e, w - w1, c1 - c0, w1, a + (long long)(r0 + w1) * ld + r0, ld,
                       a + (long long)r0 * ld + c0, ld, a + (long long)(r0 + w1) * ld + c0, ld,
                       stride, nb));
    return trsm_rec<T>(e, a, ld, stride, nb, r0 + w1, w - w1, c0, c1);
}

template <typename T>
static int lu_rec(pb_lu_engine *e, T2_t<T> *a, int n, int ld, long long stride, int nb,
                  int k0, int w, int *piv, int *info, int sw, size_t smem)
{
    if (w <= 32) {
        bool co = false;
        PB_TRY(launch_leaf_coop<T>(e, a, n, ld, stride, nb, k0, w, piv, info, co));
        if (co) return PB_OK;
        if (sw == 0) {
            // orders whose panel column does not fit in shared memory: while it does not,
            // the panel is worked on in global memory, then one column at a time in shared
            size_t sm1 = 0;
            if (leaf_sw<T>(n - k0, &sm1) == 0)
                return launch_leaf<T, 1, true>(e, a, n, ld, stride, nb, k0, w, piv, info,
                                               32 * sizeof(T2_t<T>));
            return launch_leaf<T, 1>(e, a, n, ld, stride, nb, k0, w, piv, info,
                                     ((size_t)(n - k0) + 32) * sizeof(T2_t<T>));
        }
        if (sw == 4) return launch_leaf<T, 4>(e, a, n, ld, stride, nb, k0, w, piv, info, smem);
        if (sw == 2) return launch_leaf<T, 2>(e, a, n, ld, stride, nb, k0, w, piv, info, smem);
        return launch_leaf<T, 1>(e, a, n, ld, stride, nb, k0, w, piv, info, smem);
    }
    const int w1 = ((w / 2 + 31) / 32) * 32;
    PB_TRY(lu_rec<T>(e, a, n, ld, stride, nb, k0, w1, piv, info, sw, smem));
    PB_TRY(swap_rows<T>(e, a, n, ld, stride, nb, piv, k0, k0 + w1, k0 + w1, k0 + w));
    PB_TRY(trsm_rec<T>(e, a, ld, stride, nb, k0, w1, k0 + w1, k0 + w));
    PB_TRY(gemm_sub<T>(e, n - k0 - w1, w - w1, w1, a + (long long)(k0 + w1) * ld + k0, ld,
                       a + (long long)k0 * ld + k0 + w1, ld,
                       a + (long long)(k0 + w1) * ld + k0 + w1, ld, stride, nb));
    PB_TRY(lu_rec<T>(e, a, n, ld, stride, nb, k0 + w1, w - w1, piv, info, sw, smem));
    return swap_rows<T>(e, a, n, ld, stride, nb, piv, k0 + w1, k0 + w, k0, k0 + w1);
}

__global__ void k_fill_int(int *p, int v, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

template <typename T>
int pb_lu_factor(pb_lu_engine *e, int n, int nb, T2_t<T> *a, int ld, long stride, int *piv,
                 int *info)
{
    if (n <= 0 || nb <= 0) return PB_OK;
    k_fill_int<<<ceil_div(nb, 256), 256, 0, e->stream>>>(info, -1, nb);
    e->launches++;
    size_t smem = 0;
    const int sw = leaf_sw<T>(n, &smem);           // 0: the first panels go through global memory
    PB_TRY(lu_rec<T>(e, a, n, ld, stride, nb, 0, n, piv, info, sw, smem));
    return check_tc(e);
}
template int pb_lu_factor<float>(pb_lu_engine *, int, int, float2 *, int, long, int *, int *);
template int pb_lu_factor<double>(pb_lu_engine *, int, int, double2 *, int, long, int *, int *);

// ---------------------------------------------------------------- complex-symmetric LDL^T
// The reduced system jw Zb + G^T P G is complex symmetric (Lp and P are). Without
// pivoting its factorisation is A = L D L^T with U = D L^T, so the U part of an LU needs
// no triangular solve (U12 = D1 L21^T is a scaled transpose) and the trailing updates only
// their lower triangle: about half the flops of the pivoted LU, no row swaps. The factors
// are stored like an unpivoted LU (unit L below, U on and above the diagonal).

// Leaf: columns [k0, k0+w) (w <= 32) over rows [k0, n), SW columns at a time in shared
// memory. The U row of a column is read from the lower triangle (U[c][j] = A[j][c] before
// scaling), so entries above the diagonal that earlier updates skipped are never read.
template <int SW>
__global__ void __launch_bounds__(1024)
k_ldl_leaf(float2 *a, int n, int ld, long long stride, int k0, int w, int *info)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    const int m = n - k0;
    float2 *spm = reinterpret_cast<float2 *>(smraw);      // [m][SW], rows k0 + r
    float2 *urow = spm + (size_t)m * SW;                   // [SW][32]
    const int b = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    a += (long long)b * stride;
    for (int s0 = 0; s0 < w; s0 += SW) {
        const int sw = min(SW, w - s0), c0 = k0 + s0;
        for (int e = tid; e < (n - c0) * sw; e += nt) {
            const int r = c0 - k0 + e / sw, t = e - (e / sw) * sw;
            spm[r * SW + t] = a[(long long)(k0 + r) * ld + c0 + t];
        }
        __syncthreads();
        for (int t = 0; t < sw; t++) {
            const int c = c0 + t, rc = c - k0;
            const float2 d = spm[rc * SW + t];
            if (tid == 0 && cmag1(d) < 1e-30 && info[b] < 0) info[b] = c;
            const float2 dinv = safe_inv(d);
            float2 u[SW];
#pragma unroll
            for (int tt = 0; tt < SW; tt++)
                u[tt] = (tt > t && tt < sw) ? spm[(c0 + tt - k0) * SW + t] : mk2<float2>(0, 0);
            __syncthreads();
            for (int r = c + 1 + tid; r < n; r += nt) {
                const float2 l = cmul(spm[(r - k0) * SW + t], dinv);
                spm[(r - k0) * SW + t] = l;
#pragma unroll
                for (int tt = 0; tt < SW; tt++)
                    if (tt > t && tt < sw && r >= c0 + tt)
                        spm[(r - k0) * SW + tt] = cfms(spm[(r - k0) * SW + tt], l, u[tt]);
            }
            if (tid == 0)
                for (int tt = t + 1; tt < sw; tt++) spm[rc * SW + tt] = u[tt];   // U row c = d L^T
            __syncthreads();
        }
        for (int e = tid; e < (n - c0) * sw; e += nt) {
            const int r = c0 - k0 + e / sw, t = e - (e / sw) * sw;
            a[(long long)(k0 + r) * ld + c0 + t] = spm[r * SW + t];
        }
        const int c1 = c0 + sw, nr = k0 + w - c1;
        if (nr > 0) {
            // U rows of this sub-panel for the remaining leaf columns: U[c0+t][col] = d_t L[col][c0+t]
            for (int e = tid; e < sw * nr; e += nt) {
                const int t = e / nr, col = c1 + (e - t * nr);
                const float2 v = cmul(spm[(c0 + t - k0) * SW + t], spm[(col - k0) * SW + t]);
                urow[t * 32 + (col - c1)] = v;
                a[(long long)(c0 + t) * ld + col] = v;
            }
            __syncthreads();
            // trailing update of the remaining leaf columns, lower triangle only
            const long long tot = (long long)(n - c1) * nr;
            for (long long e = tid; e < tot; e += nt) {
                const int r = c1 + (int)(e / nr), col = c1 + (int)(e % nr);
                if (r < col) continue;
                float2 v = a[(long long)r * ld + col];
#pragma unroll
                for (int t = 0; t < SW; t++)
                    if (t < sw) v = cfms(v, spm[(r - k0) * SW + t], urow[t * 32 + (col - c1)]);
                a[(long long)r * ld + col] = v;
            }
        }
        __syncthreads();
    }
}

// U12 = D1 L21^T: a[c][j] = a[c][c] * a[j][c] for c in [r0, r0+w1), j in [j0, j1); 32 x 32
// tiles transposed through shared memory (coalesced reads along c, writes along j).
__global__ void __launch_bounds__(256)
k_sym_u(float2 *a, int ld, long long stride, int r0, int w1, int j0, int j1)
{
    __shared__ float2 t[32][33];
    __shared__ float2 dg[32];
    a += (long long)blockIdx.z * stride;
    const int cb = r0 + blockIdx.y * 32, jb = j0 + blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    if (ty == 0) dg[tx] = (cb + tx < r0 + w1) ? a[(long long)(cb + tx) * ld + cb + tx] : mk2<float2>(0, 0);
    for (int jj = ty; jj < 32; jj += 8) {
        const int j = jb + jj, c = cb + tx;
        t[jj][tx] = (j < j1 && c < r0 + w1) ? a[(long long)j * ld + c] : mk2<float2>(0, 0);
    }
    __syncthreads();
    for (int cc = ty; cc < 32; cc += 8) {
        const int c = cb + cc, j = jb + tx;
        if (c < r0 + w1 && j < j1) a[(long long)c * ld + j] = cmul(dg[cc], t[tx][cc]);
    }
}

static int ldl_sw(int m, size_t *smem)
{
    const size_t avail = (size_t)pb_smem_cap() - 1024;
    const int opts[5] = {8, 6, 4, 2, 1};
    for (int i = 0; i < 5; i++) {
        const size_t need = ((size_t)m * opts[i] + (size_t)opts[i] * 32) * sizeof(float2);
        if (need <= avail) { *smem = need; return opts[i]; }
    }
    return 0;
}

template <int SW>
static int launch_ldl_leaf(pb_lu_engine *e, float2 *a, int n, int ld, long long stride, int nb, int k0, int w,
                           int *info, size_t smem)
{
    static std::atomic<unsigned long long> attr_set{0};   // per device
    PB_TRY(pb_smem_optin(k_ldl_leaf<SW>, pb_smem_cap() - 1024, attr_set));
    const int m = n - k0, nt = std::min(1024, std::max(128, (m + 31) / 32 * 32));
    k_ldl_leaf<SW><<<nb, nt, smem, e->stream>>>(a, n, ld, stride, k0, w, info);
    e->launches++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

static int ldl_rec(pb_lu_engine *e, float2 *a, int n, int ld, long long stride, int nb, int k0, int w, int *info,
                   int sw, size_t smem)
{
    if (w <= 32) {
        switch (sw) {
        case 8: return launch_ldl_leaf<8>(e, a, n, ld, stride, nb, k0, w, info, smem);
        case 6: return launch_ldl_leaf<6>(e, a, n, ld, stride, nb, k0, w, info, smem);
        case 4: return launch_ldl_leaf<4>(e, a, n, ld, stride, nb, k0, w, info, smem);
        case 2: return launch_ldl_leaf<2>(e, a, n, ld, stride, nb, k0, w, info, smem);
        default: return launch_ldl_leaf<1>(e, a, n, ld, stride, nb, k0, w, info, smem);
        }
    }
    const int w1 = ((w / 2 + 31) / 32) * 32, w2 = w - w1;
    PB_TRY(ldl_rec(e, a, n, ld, stride, nb, k0, w1, info, sw, smem));
    k_sym_u<<<dim3(ceil_div(w2, 32), ceil_div(w1, 32), nb), 256, 0, e->stream>>>(a, ld, stride, k0, w1, k0 + w1,
                                                                                 k0 + w);
    e->launches++;
    PB_CHECK_LAUNCH();
    PB_TRY(pb_cgemm_sub(e, n - k0 - w1, w2, w1, a + (long long)(k0 + w1) * ld + k0, ld, a + (long long)k0 * ld + k0 + w1,
                        ld, a + (long long)(k0 + w1) * ld + k0 + w1, ld, stride, nb, 1));
    return ldl_rec(e, a, n, ld, stride, nb, k0 + w1, w2, info, sw, smem);
}

__global__ void k_iota_piv(int *piv, int n, int nb)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < (long long)n * nb) piv[i] = (int)(i % n);
}

bool pb_ldl_supported(int n)
{
    size_t smem = 0;
    return n > 0 && ldl_sw(n, &smem) > 0;
}

int pb_ldl_factor(pb_lu_engine *e, int n, int nb, float2 *a, int ld, long stride, int *piv, int *info)
{
    if (n <= 0 || nb <= 0) return PB_OK;
    size_t smem = 0;
    const int sw = ldl_sw(n, &smem);
    if (sw == 0) return PB_ERR_UNSUP;
    k_fill_int<<<ceil_div(nb, 256), 256, 0, e->stream>>>(info, -1, nb);
    k_iota_piv<<<ceil_div((long long)n * nb, 256), 256, 0, e->stream>>>(piv, n, nb);
    e->launches += 2;
    PB_CHECK_LAUNCH();
    PB_TRY(ldl_rec(e, a, n, ld, stride, nb, 0, n, info, sw, smem));
    return check_tc(e);
}

// ---------------------------------------------------------------- permutation
__global__ void k_perm(const int *piv, int *perm, int n, int nb)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const int *p = piv + (long long)b * n;
    int *q = perm + (long long)b * n;
    for (int i = 0; i < n; i++) q[i] = i;
    for (int k = 0; k < n; k++) {
        const int j = p[k];
        if (j != k) { const int t = q[k]; q[k] = q[j]; q[j] = t; }
    }
}

int pb_lu_perm(pb_lu_engine *e, int n, int nb, const int *piv, int *perm)
{
    k_perm<<<ceil_div(nb, 64), 64, 0, e->stream>>>(piv, perm, n, nb);
    e->launches++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

// ---------------------------------------------------------------- triangular solves
// One CTA (1024 threads) per (rhs, matrix). The whole vector lives in shared memory.
// Sum over c in [c0, c1) of row[c] * xs[c] (complex) by one warp; the result is valid in
// lane 0. Four independent accumulators keep several loads in flight; FP32 rows are read
// 16 bytes (two entries) at a time when row and c0 allow it. xs is in shared memory.
__device__ __forceinline__ float2 warp_cdot(const float2 *row, const float2 *xs, int c0, int c1, int lane)
{
    float ax = 0.f, ay = 0.f, bx = 0.f, by = 0.f, cx = 0.f, cy = 0.f, dx = 0.f, dy = 0.f;
    if (((c0 & 1) == 0) && ((reinterpret_cast<uintptr_t>(row) & 15) == 0)) {
        const float4 *r4 = reinterpret_cast<const float4 *>(row);
        const float4 *x4 = reinterpret_cast<const float4 *>(xs);
        const int pe = c1 >> 1;                          // pairs entirely inside [c0, c1)
        int p = (c0 >> 1) + lane;
        // four 16-byte row loads in flight per lane: the solve streams the factors from HBM
        // with one CTA per system, so the loads a warp keeps in flight set its bandwidth
        for (; p + 96 < pe; p += 128) {
            const float4 u0 = r4[p], u1 = r4[p + 32], u2 = r4[p + 64], u3 = r4[p + 96];
            const float4 v0 = x4[p], v1 = x4[p + 32], v2 = x4[p + 64], v3 = x4[p + 96];
            ax = fmaf(u0.x, v0.x, fmaf(-u0.y, v0.y, ax));
            ay = fmaf(u0.x, v0.y, fmaf(u0.y, v0.x, ay));
            bx = fmaf(u0.z, v0.z, fmaf(-u0.w, v0.w, bx));
            by = fmaf(u0.z, v0.w, fmaf(u0.w, v0.z, by));
            cx = fmaf(u1.x, v1.x, fmaf(-u1.y, v1.y, cx));
            cy = fmaf(u1.x, v1.y, fmaf(u1.y, v1.x, cy));
            dx = fmaf(u1.z, v1.z, fmaf(-u1.w, v1.w, dx));
            dy = fmaf(u1.z, v1.w, fmaf(u1.w, v1.z, dy));
            ax = fmaf(u2.x, v2.x, fmaf(-u2.y, v2.y, ax));
            ay = fmaf(u2.x, v2.y, fmaf(u2.y, v2.x, ay));
            bx = fmaf(u2.z, v2.z, fmaf(-u2.w, v2.w, bx));
            by = fmaf(u2.z, v2.w, fmaf(u2.w, v2.z, by));
            cx = fmaf(u3.x, v3.x, fmaf(-u3.y, v3.y, cx));
            cy = fmaf(u3.x, v3.y, fmaf(u3.y, v3.x, cy));
            dx = fmaf(u3.z, v3.z, fmaf(-u3.w, v3.w, dx));
            dy = fmaf(u3.z, v3.w, fmaf(u3.w, v3.z, dy));
        }
        for (; p + 32 < pe; p += 64) {
            const float4 u = r4[p], v = x4[p], u2 = r4[p + 32], v2 = x4[p + 32];
            ax = fmaf(u.x, v.x, fmaf(-u.y, v.y, ax));
            ay = fmaf(u.x, v.y, fmaf(u.y, v.x, ay));
            bx = fmaf(u.z, v.z, fmaf(-u.w, v.w, bx));
            by = fmaf(u.z, v.w, fmaf(u.w, v.z, by));
            cx = fmaf(u2.x, v2.x, fmaf(-u2.y, v2.y, cx));
            cy = fmaf(u2.x, v2.y, fmaf(u2.y, v2.x, cy));
            dx = fmaf(u2.z, v2.z, fmaf(-u2.w, v2.w, dx));
            dy = fmaf(u2.z, v2.w, fmaf(u2.w, v2.z, dy));
        }
        if (p < pe) {
            const float4 u = r4[p], v = x4[p];
            ax = fmaf(u.x, v.x, fmaf(-u.y, v.y, ax));
            ay = fmaf(u.x, v.y, fmaf(u.y, v.x, ay));
            bx = fmaf(u.z, v.z, fmaf(-u.w, v.w, bx));
            by = fmaf(u.z, v.w, fmaf(u.w, v.z, by));
        }
        const int c = 2 * pe;                            // odd c1: the last entry (if inside)
        if (c >= c0 && c < c1 && lane == 0) {
            cx = fmaf(row[c].x, xs[c].x, fmaf(-row[c].y, xs[c].y, cx));
            cy = fmaf(row[c].x, xs[c].y, fmaf(row[c].y, xs[c].x, cy));
        }
    } else {
        int c = c0 + lane;
        for (; c + 32 < c1; c += 64) {
            const float2 u = row[c], v = xs[c], u2 = row[c + 32], v2 = xs[c + 32];
            ax = fmaf(u.x, v.x, fmaf(-u.y, v.y, ax));
            ay = fmaf(u.x, v.y, fmaf(u.y, v.x, ay));
            bx = fmaf(u2.x, v2.x, fmaf(-u2.y, v2.y, bx));
            by = fmaf(u2.x, v2.y, fmaf(u2.y, v2.x, by));
        }
        if (c < c1) {
            ax = fmaf(row[c].x, xs[c].x, fmaf(-row[c].y, xs[c].y, ax));
            ay = fmaf(row[c].x, xs[c].y, fmaf(row[c].y, xs[c].x, ay));
        }
    }
    float sx = (ax + bx) + (cx + dx), sy = (ay + by) + (cy + dy);
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_down_sync(0xffffffffu, sx, o);
        sy += __shfl_down_sync(0xffffffffu, sy, o);
    }
    return make_float2(sx, sy);
}

__device__ __forceinline__ double2 warp_cdot(const double2 *row, const double2 *xs, int c0, int c1, int lane)
{
    double ax = 0, ay = 0, bx = 0, by = 0;
    int c = c0 + lane;
    for (; c + 32 < c1; c += 64) {
        const double2 u = row[c], v = xs[c], u2 = row[c + 32], v2 = xs[c + 32];
        ax = fma(u.x, v.x, fma(-u.y, v.y, ax));
        ay = fma(u.x, v.y, fma(u.y, v.x, ay));
        bx = fma(u2.x, v2.x, fma(-u2.y, v2.y, bx));
        by = fma(u2.x, v2.y, fma(u2.y, v2.x, by));
    }
    if (c < c1) {
        ax = fma(row[c].x, xs[c].x, fma(-row[c].y, xs[c].y, ax));
        ay = fma(row[c].x, xs[c].y, fma(row[c].y, xs[c].x, ay));
    }
    double sx = ax + bx, sy = ay + by;
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_down_sync(0xffffffffu, sx, o);
        sy += __shfl_down_sync(0xffffffffu, sy, o);
    }
    return make_double2(sx, sy);
}

template <typename TF, bool G>
__global__ void __launch_bounds__(1024)
k_lu_solve(const T2_t<TF> *lu, int n, int ld, long long stride, const int *perm,
           const double2 *r, double2 *x, int nrhs, const int *sys, const int *lu_of, int operm)
{
    typedef T2_t<TF> T2;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ T2 diag[32][33];
    __shared__ T2 tmp[32];
    __shared__ double red[33];
    const int rhs = blockIdx.x, tid = threadIdx.x;
    const int b = sys ? sys[blockIdx.y] : blockIdx.y;         // system (vector slot)
    const int fm = lu_of ? lu_of[b] : b;                      // its factors
    const int lane = tid & 31, warp = tid >> 5;
    lu += (long long)fm * stride;
    perm += (long long)fm * n;
    const double2 *rv = r + ((long long)b * nrhs + rhs) * n;
    double2 *xv = x + ((long long)b * nrhs + rhs) * n;
    // the working vector: shared memory, or (G: FP64 orders above ~13 000, whose vector
    // does not fit) the output vector itself
    T2 *xs = G ? reinterpret_cast<T2 *>(xv) : reinterpret_cast<T2 *>(smraw);

    // scale by max |component|
    double mx = 0;
    for (int i = tid; i < n; i += blockDim.x) mx = fmax(mx, fmax(fabs(rv[i].x), fabs(rv[i].y)));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if (lane == 0) red[warp] = mx;
    __syncthreads();
    if (tid == 0) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t = fmax(t, red[w]);
        red[32] = t;
    }
    __syncthreads();
    const double scale = red[32] > 0 ? red[32] : 1.0;
    if (G) {
        // r and x may alias: read every permuted entry before the first write
        constexpr int KMAX = 32;                  // n <= 32 * 1024 (checked by the launcher)
        double2 v[KMAX];
#pragma unroll
        for (int k = 0; k < KMAX; k++) {
            const int i = tid + k * (int)blockDim.x;
            if (i < n) v[k] = rv[perm[i]];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < KMAX; k++) {
            const int i = tid + k * (int)blockDim.x;
            if (i < n) xs[i] = mk2<T2>(v[k].x / scale, v[k].y / scale);
        }
    } else {
        for (int i = tid; i < n; i += blockDim.x) {
            const double2 v = rv[perm[i]];
            xs[i] = mk2<T2>(v.x / scale, v.y / scale);
        }
    }
    __syncthreads();

    // forward: unit lower (each warp takes rows warp, warp + nwarps, ... of a 32-row block:
    // small systems run on 256-thread CTAs, so that more of them share an SM)
    const int nwarps = (int)(blockDim.x >> 5);
    for (int r0 = 0; r0 < n; r0 += 32) {
        for (int wr = warp; wr < 32; wr += nwarps) {
            const int r = r0 + wr;
            if (r < n) {
                const T2 *row = lu + (long long)r * ld;
                const T2 acc = warp_cdot(row, xs, 0, r0, lane);
                if (lane == 0) tmp[wr] = csub(xs[r], acc);
                diag[wr][lane] = (r0 + lane < n) ? row[r0 + lane] : mk2<T2>(0, 0);
            }
        }
        __syncthreads();
        if (warp == 0) {
            const int nbk = min(32, n - r0);
            T2 xl = mk2<T2>(0, 0);               // lane l holds x[r0+l] once solved
            for (int i = 0; i < nbk; i++) {
                T2 p = (lane < i) ? cmul(diag[i][lane], xl) : mk2<T2>(0, 0);
                for (int o = 16; o > 0; o >>= 1) {
                    p.x += __shfl_xor_sync(0xffffffffu, p.x, o);
                    p.y += __shfl_xor_sync(0xffffffffu, p.y, o);
                }
                const T2 v = csub(tmp[i], p);
                if (lane == i) xl = v;
            }
            if (lane < nbk) xs[r0 + lane] = xl;
        }
        __syncthreads();
    }
    // backward: upper with diagonal
    const int nblk = (n + 31) / 32;
    for (int bk = nblk - 1; bk >= 0; bk--) {
        const int r0 = bk * 32, nbk = min(32, n - r0);
        for (int wr = warp; wr < nbk; wr += nwarps) {
            const int r = r0 + wr;
            const T2 *row = lu + (long long)r * ld;
            const T2 acc = warp_cdot(row, xs, r0 + 32, n, lane);
            if (lane == 0) tmp[wr] = csub(xs[r], acc);
            diag[wr][lane] = (lane < nbk) ? row[r0 + lane] : mk2<T2>(0, 0);
        }
        __syncthreads();
        if (warp == 0) {
            T2 xl = mk2<T2>(0, 0);
            for (int i = nbk - 1; i >= 0; i--) {
                T2 p = (lane > i && lane < nbk) ? cmul(diag[i][lane], xl) : mk2<T2>(0, 0);
                for (int o = 16; o > 0; o >>= 1) {
                    p.x += __shfl_xor_sync(0xffffffffu, p.x, o);
                    p.y += __shfl_xor_sync(0xffffffffu, p.y, o);
                }
                const T2 v = cmul(csub(tmp[i], p), safe_inv(diag[i][i]));
                if (lane == i) xl = v;
            }
            if (lane < nbk) xs[r0 + lane] = xl;
        }
        __syncthreads();
    }
    // operm: factors of a symmetrically permuted matrix P A P^T, so x = P^T y (x[perm[i]] = y_i);
    // only for the shared-memory variant (xs does not alias xv)
    for (int i = tid; i < n; i += blockDim.x)
        xv[(!G && operm) ? perm[i] : i] = make_double2((double)xs[i].x * scale, (double)xs[i].y * scale);
}

template <typename TF>
int pb_lu_solve_batched(pb_lu_engine *e, int n, int nb, int nrhs, const T2_t<TF> *lu, int ld,
                        long stride, const int *perm, const double2 *r, double2 *x, int operm)
{
    return pb_lu_solve_mapped<TF>(e, n, nb, nrhs, lu, ld, stride, perm, r, x, nullptr, nullptr, operm);
}

template <typename TF>
int pb_lu_solve_mapped(pb_lu_engine *e, int n, int nb, int nrhs, const T2_t<TF> *lu, int ld,
                       long stride, const int *perm, const double2 *r, double2 *x, const int *sys,
                       const int *lu_of, int operm)
{
    if (nb <= 0) return PB_OK;
    const size_t smem = (size_t)n * sizeof(T2_t<TF>);
    static std::atomic<unsigned long long> attr_set{0};   // per device
    dim3 g(nrhs, nb);
    if (smem > (size_t)pb_smem_cap() - 20480) {
        // the vector does not fit in shared memory: solve in place in x (FP64 only)
        if (sizeof(T2_t<TF>) != sizeof(double2) || n > 32 * 1024 || operm) {
            pb_set_error("triangular solve of order %d does not fit this build", n);
            return PB_ERR_UNSUP;
        }
        k_lu_solve<TF, true><<<g, 1024, 0, e->stream>>>(lu, n, ld, stride, perm, r, x, nrhs, sys, lu_of, 0);
    } else {
        PB_TRY(pb_smem_optin(k_lu_solve<TF, false>, pb_smem_cap() - 20480, attr_set));
        // the same rows and dot products either way (results do not depend on it)
        const int nt = n <= 512 ? 256 : 1024;
        k_lu_solve<TF, false><<<g, nt, smem, e->stream>>>(lu, n, ld, stride, perm, r, x, nrhs, sys, lu_of, operm);
    }
    e->launches++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}
template int pb_lu_solve_mapped<float>(pb_lu_engine *, int, int, int, const float2 *, int, long, const int *, const double2 *, double2 *, const int *, const int *, int);
template int pb_lu_solve_mapped<double>(pb_lu_engine *, int, int, int, const double2 *, int, long, const int *, const double2 *, double2 *, const int *, const int *, int);
template int pb_lu_solve_batched<float>(pb_lu_engine *, int, int, int, const float2 *, int, long, const int *, const double2 *, double2 *, int);
template int pb_lu_solve_batched<double>(pb_lu_engine *, int, int, int, const double2 *, int, long, const int *, const double2 *, double2 *, int);

// ---------------------------------------------------------------- explicit inverse
// For one FP64 system whose factors serve many solves (the circuit Schur complement of the
// compressed path's preconditioner) the explicit inverse turns every later solve into one
// bandwidth-bound matrix-vector product. A^-1 = U^-1 L^-1 P: X starts as P (X[i][perm[i]]
// = 1) and two cuBLAS triangular solves with n right-hand sides apply L^-1 and U^-1. The
// factors are row-major, which cuBLAS (column-major) sees transposed: L Y = P becomes
// Y^T L^T = P^T (right side, upper, unit) and U X = Y becomes X^T U^T = Y^T (right side,
// lower); the row-major buffer then holds X.
__global__ void k_inv_init(int n, const int *perm, double2 *X)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) X[(long long)i * n + perm[i]] = make_double2(1, 0);
}

int pb_lu_inverse(pb_lu_engine *e, int n, const double2 *lu, int ld, const int *perm, double2 *X)
{
    if (n <= 0) return PB_OK;
    PB_CUDA(cudaMemsetAsync(X, 0, sizeof(double2) * (size_t)n * n, e->stream));
    k_inv_init<<<ceil_div(n, 256), 256, 0, e->stream>>>(n, perm, X);
    PB_CHECK_LAUNCH();
    const cuDoubleComplex one = make_cuDoubleComplex(1, 0);
    cublasStatus_t s = cublasZtrsm(e->blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_UNIT,
                                   n, n, &one, (const cuDoubleComplex *)lu, ld, (cuDoubleComplex *)X, n);
    if (s == CUBLAS_STATUS_SUCCESS)
        s = cublasZtrsm(e->blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, n, n,
                        &one, (const cuDoubleComplex *)lu, ld, (cuDoubleComplex *)X, n);
    e->launches += 3;
    if (s != CUBLAS_STATUS_SUCCESS) { pb_set_error("triangular solve for the inverse failed (%d)", (int)s); return PB_ERR_CUDA; }
    return PB_OK;
}

// y = X r, X row-major n x n: one warp per row (coalesced row reads, r from L2)
__global__ void __launch_bounds__(256) k_gemv_rm(int n, const double2 *__restrict__ X, const double2 *__restrict__ r,
                                                 double2 *__restrict__ y)
{
    const int i = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= n) return;
    const double2 *row = X + (long long)i * n;
    double2 acc = make_double2(0, 0);
    for (int c = lane; c < n; c += 32) acc = cadd(acc, cmul(row[c], r[c]));
    for (int o = 16; o > 0; o >>= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
    }
    if (lane == 0) y[i] = acc;
}

int pb_gemv(pb_lu_engine *e, int n, const double2 *X, const double2 *r, double2 *y)
{
    if (n <= 0) return PB_OK;
    if ((const void *)r == (const void *)y) { pb_set_error("pb_gemv: r and y must differ"); return PB_ERR_ARG; }
    k_gemv_rm<<<ceil_div(n, 8), 256, 0, e->stream>>>(n, X, r, y);
    e->launches++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

// ---------------------------------------------------------------- FP64 residual
// r = b - A x ; 8 warps per block, each warp one row at a time; x staged in smem.
__device__ __forceinline__ void atomic_max_pos(double *addr, double v)
{
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

__global__ void __launch_bounds__(256)
k_residual(const double2 *a, int n, int ld, long long stride, const double2 *bv,
           const double2 *xv, double2 *rv, double *rn, double *bn, double *xn, double *an,
           int nrhs, int rows_per_block, const int *sys, double *cw, int stage, double *wv)
{
    // stage = 1: x is staged in shared memory [nrhs][n]; 0 (orders whose x does not fit,
    // above ~14 000 unknowns): x is read from global memory (L2 holds it)
    extern __shared__ __align__(16) unsigned char smraw[];
    const int b = sys ? sys[blockIdx.y] : blockIdx.y, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double2 *xs = stage ? reinterpret_cast<const double2 *>(smraw) : xv + (long long)b * nrhs * n;
    a += (long long)b * stride;
    if (stage) {
        double2 *xw = reinterpret_cast<double2 *>(smraw);
        for (int e = tid; e < nrhs * n; e += blockDim.x) xw[e] = xv[(long long)b * nrhs * n + e];
    }
    __syncthreads();
    if (blockIdx.x == 0 && xn) {
        for (int q = warp; q < nrhs; q += 8) {
            double m = 0;
            for (int c = lane; c < n; c += 32) m = fmax(m, fmax(fabs(xs[q * n + c].x), fabs(xs[q * n + c].y)));
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
            if (lane == 0) xn[b * nrhs + q] = m;
        }
    }
    const int rbeg = blockIdx.x * rows_per_block;
    const int rend = min(n, rbeg + rows_per_block);
    for (int r = rbeg + warp; r < rend; r += 8) {
        const double2 *row = a + (long long)r * ld;
        if (an) {
            double sa = 0;
            for (int c = lane; c < n; c += 32) sa += fabs(row[c].x) + fabs(row[c].y);
            for (int o = 16; o > 0; o >>= 1) sa += __shfl_down_sync(0xffffffffu, sa, o);
            if (lane == 0) atomic_max_pos(&an[b], sa);
        }
        for (int q = 0; q < nrhs; q++) {
            double sr = 0, si = 0, sa = 0;
            const double2 *x = xs + q * n;
            for (int c = lane; c < n; c += 32) {
                const double2 av = row[c], xx = x[c];
                sr += av.x * xx.x - av.y * xx.y;
                si += av.x * xx.y + av.y * xx.x;
                if (cw || wv) sa += (fabs(av.x) + fabs(av.y)) * (fabs(xx.x) + fabs(xx.y));
            }
            for (int o = 16; o > 0; o >>= 1) {
                sr += __shfl_down_sync(0xffffffffu, sr, o);
                si += __shfl_down_sync(0xffffffffu, si, o);
                if (cw || wv) sa += __shfl_down_sync(0xffffffffu, sa, o);
            }
            if (lane == 0) {
                const long long idx = ((long long)b * nrhs + q) * n + r;
                if (bv) {
                    const double2 bb = bv[idx];
                    const double2 res = make_double2(bb.x - sr, bb.y - si);
                    rv[idx] = res;
                    atomic_max_pos(&rn[b * nrhs + q], fmax(fabs(res.x), fabs(res.y)));
                    atomic_max_pos(&bn[b * nrhs + q], fmax(fabs(bb.x), fabs(bb.y)));
                    if (cw) {                                // componentwise (Oettli-Prager)
                        const double num = fabs(res.x) + fabs(res.y), den = sa + fabs(bb.x) + fabs(bb.y);
                        atomic_max_pos(&cw[b * nrhs + q], den > 0 ? num / den : (num > 0 ? 1.0 : 0.0));
                    }
                    if (wv) wv[idx] = sa + fabs(bb.x) + fabs(bb.y);   // (|A||x| + |b|)_r
                } else {
                    rv[idx] = make_double2(sr, si);          // product only: r = A x
                }
            }
        }
    }
}

// devices on which k_residual's shared-memory opt-in is set
static std::atomic<unsigned long long> g_residual_attr{0};

int pb_residual(pb_lu_engine *e, int n, int nb, int nrhs, const double2 *a, int ld, long stride,
                const double2 *b, const double2 *x, double2 *r, double *rn, double *bn, double *xn,
                double *an, double *cw)
{
    PB_CUDA(cudaMemsetAsync(rn, 0, sizeof(double) * nb * nrhs, e->stream));
    if (cw) PB_CUDA(cudaMemsetAsync(cw, 0, sizeof(double) * nb * nrhs, e->stream));
    PB_CUDA(cudaMemsetAsync(bn, 0, sizeof(double) * nb * nrhs, e->stream));
    if (an) PB_CUDA(cudaMemsetAsync(an, 0, sizeof(double) * nb, e->stream));
    const size_t xbytes = (size_t)nrhs * n * sizeof(double2);
    const int stage = xbytes <= (size_t)pb_smem_cap();
    const size_t smem = stage ? xbytes : 0;
    PB_TRY(pb_smem_optin(k_residual, pb_smem_cap(), g_residual_attr));
    const int rpb = 64;
    dim3 g(ceil_div(n, rpb), nb);
    k_residual<<<g, 256, smem, e->stream>>>(a, n, ld, stride, b, x, r, rn, bn, xn, an, nrhs, rpb, nullptr, cw, stage,
                                            nullptr);
    e->launches++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

int pb_residual_mapped(pb_lu_engine *e, int n, int nb, int nrhs, const double2 *a, int ld, long stride,
                       const double2 *b, const double2 *x, double2 *r, double *rn, double *bn, double *xn,
                       double *an, int nall, const int *sys, double *cw, double *wv)
{
    PB_CUDA(cudaMemsetAsync(rn, 0, sizeof(double) * nall * nrhs, e->stream));
    if (cw) PB_CUDA(cudaMemsetAsync(cw, 0, sizeof(double) * nall * nrhs, e->stream));
    PB_CUDA(cudaMemsetAsync(bn, 0, sizeof(double) * nall * nrhs, e->stream));
    if (an) PB_CUDA(cudaMemsetAsync(an, 0, sizeof(double) * nall, e->stream));
    if (nb <= 0) return PB_OK;
    const size_t xbytes = (size_t)nrhs * n * sizeof(double2);
    const int stage = xbytes <= (size_t)pb_smem_cap();
    const size_t smem = stage ? xbytes : 0;
    PB_TRY(pb_smem_optin(k_residual, pb_smem_cap(), g_residual_attr));
    const int rpb = 64;
    dim3 g(ceil_div(n, rpb), nb);
    k_residual<<<g, 256, smem, e->stream>>>(a, n, ld, stride, b, x, r, rn, bn, xn, an, nrhs, rpb, sys, cw, stage, wv);
    e->launches++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

// ---------------------------------------------------------------- symmetric FP64 residual
// r = b - A x for complex-symmetric A of which only the lower triangle (with the diagonal)
// is read: half the bytes of k_residual. Deterministic two-phase sum:
//  phase 1, one CTA per 32-row block R of a system: the block's rows against columns
//  c <= i (direct part, warp-reduced per row) and, transposed, the strictly lower entries
//  against the block's x (column partials, summed over the 8 warps in fixed order): those
//  of columns below the block go to the scratch part[R][c], those inside the block are
//  added to the block's own rows;
//  phase 2, per row i: y_i = yblk_i + sum over R > block(i) of part[R][i] in order of R.
// |A||x| and the |A| row sums (|re| + |im|, as k_residual) come along when asked for.
constexpr int SYM_RB = 32;          // rows per block
constexpr int SYM_CW = 128;         // columns per chunk (4 per lane)

template <bool AX, bool AS>
__global__ void __launch_bounds__(256)
k_symres_p1(const double2 *__restrict__ a, int n, long long stride, const double2 *__restrict__ xv,
            const int *sys, int nrb, double2 *yblk, double *axblk, double *asblk, double2 *py, double *pax,
            double *pas)
{
    __shared__ double2 xb[SYM_RB];
    __shared__ double2 tp[8][SYM_CW];
    __shared__ double tpa[AX ? 8 : 1][SYM_CW], tps[AS ? 8 : 1][SYM_CW];
    __shared__ double2 tin[SYM_RB], ydir[SYM_RB];
    __shared__ double tina[SYM_RB], tins[SYM_RB], ydira[SYM_RB], ydirs[SYM_RB];
    const int s = sys ? sys[blockIdx.y] : blockIdx.y;
    const int R = blockIdx.x, r0 = R * SYM_RB, r1 = min(n, r0 + SYM_RB);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    a += (long long)s * stride;
    const double2 *x = xv + (long long)s * n;
    if (tid < SYM_RB) {
        xb[tid] = (r0 + tid < n) ? x[r0 + tid] : make_double2(0, 0);
        tin[tid] = make_double2(0, 0);
        tina[tid] = tins[tid] = 0;
    }
    __syncthreads();
    double dr[4] = {0, 0, 0, 0}, di[4] = {0, 0, 0, 0}, da[4] = {0, 0, 0, 0}, ds[4] = {0, 0, 0, 0};
    for (int c0 = 0; c0 < r1; c0 += SYM_CW) {
        double2 xc[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int c = c0 + lane + 32 * k;
            xc[k] = c < r1 ? x[c] : make_double2(0, 0);
        }
        double tr[4] = {0, 0, 0, 0}, ti[4] = {0, 0, 0, 0}, ta[4] = {0, 0, 0, 0}, ts[4] = {0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int il = 4 * w + q, i = r0 + il;
            if (i >= n) continue;
            const double2 *row = a + (long long)i * n;
            const double2 xi = xb[il];
            double2 av[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int c = c0 + lane + 32 * k;
                av[k] = c <= i ? row[c] : make_double2(0, 0);
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int c = c0 + lane + 32 * k;
                const double2 v = av[k];
                dr[q] += v.x * xc[k].x - v.y * xc[k].y;
                di[q] += v.x * xc[k].y + v.y * xc[k].x;
                const double m = fabs(v.x) + fabs(v.y);
                if (AX) da[q] += m * (fabs(xc[k].x) + fabs(xc[k].y));
                if (AS) ds[q] += m;
                if (c < i) {                                   // strictly lower: transposed part
                    tr[k] += v.x * xi.x - v.y * xi.y;
                    ti[k] += v.x * xi.y + v.y * xi.x;
                    if (AX) ta[k] += m * (fabs(xi.x) + fabs(xi.y));
                    if (AS) ts[k] += m;
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            tp[w][lane + 32 * k] = make_double2(tr[k], ti[k]);
            if (AX) tpa[w][lane + 32 * k] = ta[k];
            if (AS) tps[w][lane + 32 * k] = ts[k];
        }
        __syncthreads();
        if (tid < SYM_CW) {
            const int c = c0 + tid;
            if (c < r1) {
                double sr = 0, si = 0, sa = 0, ss = 0;
#pragma unroll
                for (int v = 0; v < 8; v++) {
                    sr += tp[v][tid].x;
                    si += tp[v][tid].y;
                    if (AX) sa += tpa[v][tid];
                    if (AS) ss += tps[v][tid];
                }
                if (c < r0) {
                    const long long o = ((long long)blockIdx.y * nrb + R) * n + c;
                    py[o] = make_double2(sr, si);
                    if (AX) pax[o] = sa;
                    if (AS) pas[o] = ss;
                } else {
                    tin[c - r0] = make_double2(sr, si);
                    if (AX) tina[c - r0] = sa;
                    if (AS) tins[c - r0] = ss;
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        for (int o = 16; o > 0; o >>= 1) {
            dr[q] += __shfl_down_sync(0xffffffffu, dr[q], o);
            di[q] += __shfl_down_sync(0xffffffffu, di[q], o);
            if (AX) da[q] += __shfl_down_sync(0xffffffffu, da[q], o);
            if (AS) ds[q] += __shfl_down_sync(0xffffffffu, ds[q], o);
        }
        if (lane == 0) {
            ydir[4 * w + q] = make_double2(dr[q], di[q]);
            ydira[4 * w + q] = da[q];
            ydirs[4 * w + q] = ds[q];
        }
    }
    __syncthreads();
    if (tid < SYM_RB && r0 + tid < n) {
        const long long o = (long long)blockIdx.y * n + r0 + tid;
        yblk[o] = make_double2(ydir[tid].x + tin[tid].x, ydir[tid].y + tin[tid].y);
        if (AX) axblk[o] = ydira[tid] + tina[tid];
        if (AS) asblk[o] = ydirs[tid] + tins[tid];
    }
}

template <bool AX, bool AS>
__global__ void __launch_bounds__(256)
k_symres_p2(int n, int nrb, const int *sys, const double2 *yblk, const double *axblk, const double *asblk,
            const double2 *py, const double *pax, const double *pas, const double2 *bv, const double2 *xv,
            double2 *rv, double *rn, double *bn, double *xn, double *an, double *wv, double *rowsum)
{
    const int s = sys ? sys[blockIdx.y] : blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double mr = 0, mb = 0, mx = 0, ms = 0;
    if (i < n) {
        const long long o = (long long)blockIdx.y * n + i;
        double2 y = yblk[o];
        double sa = AX ? axblk[o] : 0, ss = AS ? asblk[o] : 0;
        for (int R = i / SYM_RB + 1; R < nrb; R++) {
            const long long p = ((long long)blockIdx.y * nrb + R) * n + i;
            const double2 t = py[p];
            y.x += t.x;
            y.y += t.y;
            if (AX) sa += pax[p];
            if (AS) ss += pas[p];
        }
        const long long g = (long long)s * n + i;
        if (rowsum) rowsum[g] = ss;
        if (bv) {
            const double2 b = bv[g], xx = xv[g];
            const double2 r = make_double2(b.x - y.x, b.y - y.y);
            rv[g] = r;
            mr = fmax(fabs(r.x), fabs(r.y));
            mb = fmax(fabs(b.x), fabs(b.y));
            mx = fmax(fabs(xx.x), fabs(xx.y));
            if (AX && wv) wv[g] = sa + fabs(b.x) + fabs(b.y);
        }
        ms = ss;
    }
    if (!bv) return;
    for (int o = 16; o > 0; o >>= 1) {
        mr = fmax(mr, __shfl_down_sync(0xffffffffu, mr, o));
        mb = fmax(mb, __shfl_down_sync(0xffffffffu, mb, o));
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        ms = fmax(ms, __shfl_down_sync(0xffffffffu, ms, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomic_max_pos(&rn[s], mr);
        atomic_max_pos(&bn[s], mb);
        if (xn) atomic_max_pos(&xn[s], mx);
        if (AS && an) atomic_max_pos(&an[s], ms);
    }
}

size_t pb_sym_residual_scratch(int n, int nb)
{
    const int nrb = (n + SYM_RB - 1) / SYM_RB;
    return (size_t)nb * ((size_t)nrb * n * 32 + (size_t)n * 32);
}

int pb_sym_residual_mapped(pb_lu_engine *e, int n, int nb, const double2 *a, long stride, const double2 *b,
                           const double2 *x, double2 *r, double *rn, double *bn, double *xn, double *an, int nall,
                           const int *sys, double *wv, void *scratch)
{
    PB_CUDA(cudaMemsetAsync(rn, 0, sizeof(double) * nall, e->stream));
    PB_CUDA(cudaMemsetAsync(bn, 0, sizeof(double) * nall, e->stream));
    if (xn) PB_CUDA(cudaMemsetAsync(xn, 0, sizeof(double) * nall, e->stream));
    if (an) PB_CUDA(cudaMemsetAsync(an, 0, sizeof(double) * nall, e->stream));
    if (nb <= 0) return PB_OK;
    const int nrb = (n + SYM_RB - 1) / SYM_RB;
    // scratch per system: part y [nrb][n] complex, part |A||x| and |A| [nrb][n] real each,
    // the block sums [n] complex + 2 real
    double2 *py = reinterpret_cast<double2 *>(scratch);
    double *pax = reinterpret_cast<double *>(py + (size_t)nb * nrb * n);
    double *pas = pax + (size_t)nb * nrb * n;
    double2 *yblk = reinterpret_cast<double2 *>(pas + (size_t)nb * nrb * n);
    double *axblk = reinterpret_cast<double *>(yblk + (size_t)nb * n);
    double *asblk = axblk + (size_t)nb * n;
    const bool ax = wv != nullptr, as = an != nullptr;
    const dim3 g1(nrb, nb), g2(ceil_div(n, 256), nb);
#define PB_SYMRES(AXV, ASV)                                                                                          \
    do {                                                                                                             \
        k_symres_p1<AXV, ASV><<<g1, 256, 0, e->stream>>>(a, n, stride, x, sys, nrb, yblk, axblk, asblk, py, pax, pas); \
        k_symres_p2<AXV, ASV><<<g2, 256, 0, e->stream>>>(n, nrb, sys, yblk, axblk, asblk, py, pax, pas, b, x, r, rn,  \
                                                         bn, xn, an, wv, nullptr);                                   \
    } while (0)
    if (ax && as) PB_SYMRES(true, true);
    else if (ax) PB_SYMRES(true, false);
    else if (as) PB_SYMRES(false, true);
    else PB_SYMRES(false, false);
#undef PB_SYMRES
    e->launches += 2;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

// Static symmetric ordering of the unpivoted L D L^T: per system the unknowns sorted by
// decreasing diagonal dominance |A_kk| / sum_j |A_kj| (|re| + |im|, both triangles), ties by
// index. On the benchmark's reduced systems this brings the FP32 factorisation's backward
// error from 2.2e-5 to 1.0e-6 (2 GHz; the pivoted LU: 4.6e-7).
//  k_sym_rowsum: the row sums, by the two-phase kernels of the symmetric residual
//  k_order_desc: one CTA per system, bitonic sort of (key, index) in shared memory
//  k_sym_permute_f32: M32[i][j] = (float) M64[max(p_i, p_j)][min(p_i, p_j)] for i >= j
__global__ void __launch_bounds__(1024)
k_order_desc(int n, int np2, const double *rowsum, const double2 *a, long long stride, int *perm)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    float *key = reinterpret_cast<float *>(smraw);
    int *idx = reinterpret_cast<int *>(key + np2);
    const int s = blockIdx.x, tid = threadIdx.x;
    const double2 *A = a + (long long)s * stride;
    for (int i = tid; i < np2; i += blockDim.x) {
        if (i < n) {
            const double2 d = A[(long long)i * n + i];
            const double rsum = rowsum[(long long)s * n + i];
            key[i] = rsum > 0 ? (float)((fabs(d.x) + fabs(d.y)) / rsum) : 0.f;
            idx[i] = i;
        } else {
            key[i] = -1.f;                       // padding sorts last
            idx[i] = INT_MAX;
        }
    }
    __syncthreads();
    // descending by key, ascending by index on ties
    for (int k = 2; k <= np2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < np2; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    const bool before = key[l] > key[i] || (key[l] == key[i] && idx[l] < idx[i]);
                    if (before == up) {
                        const float tk = key[i]; key[i] = key[l]; key[l] = tk;
                        const int ti = idx[i]; idx[i] = idx[l]; idx[l] = ti;
                    }
                }
            }
            __syncthreads();
        }
    for (int i = tid; i < n; i += blockDim.x) perm[(long long)s * n + i] = idx[i];
}

__global__ void __launch_bounds__(256)
k_sym_permute_f32(const double2 *__restrict__ a, int n, long long stride, const int *__restrict__ perm,
                  float2 *__restrict__ o)
{
    const int bx = blockIdx.x, by = blockIdx.y;     // tile column, tile row: lower tiles only
    if (bx > by) return;
    const long long s = blockIdx.z;
    a += s * stride;
    o += s * stride;
    const int *p = perm + s * n;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int j = bx * 32 + tx;
    if (j >= n) return;
    const int pj = p[j];
    for (int r = ty; r < 32; r += 8) {
        const int i = by * 32 + r;
        if (i >= n || j > i) continue;
        const int pi = p[i];
        const int hi = pi > pj ? pi : pj, lo = pi > pj ? pj : pi;
        const double2 v = a[(long long)hi * n + lo];
        o[(long long)i * n + j] = make_float2((float)v.x, (float)v.y);
    }
}

int pb_sym_order(pb_lu_engine *e, int n, int nb, const double2 *a, long long stride, float2 *a32, int *perm,
                 void *scratch)
{
    if (n <= 0 || nb <= 0) return PB_OK;
    int np2 = 1;
    while (np2 < n) np2 <<= 1;
    if (np2 > 16384) return PB_ERR_UNSUP;
    const int nrb = (n + SYM_RB - 1) / SYM_RB;
    double2 *py = reinterpret_cast<double2 *>(scratch);
    double *pax = reinterpret_cast<double *>(py + (size_t)nb * nrb * n);
    double *pas = pax + (size_t)nb * nrb * n;
    double2 *yblk = reinterpret_cast<double2 *>(pas + (size_t)nb * nrb * n);
    double *axblk = reinterpret_cast<double *>(yblk + (size_t)nb * n);
    double *asblk = axblk + (size_t)nb * n;
    double *rowsum = reinterpret_cast<double *>(pax);      // the |A||x| partials are not used here
    // x: any vector (the direct products are discarded); the system's own first row
    k_symres_p1<false, true><<<dim3(nrb, nb), 256, 0, e->stream>>>(a, n, stride, a, nullptr, nrb, yblk, axblk, asblk,
                                                                  py, pax, pas);
    k_symres_p2<false, true><<<dim3(ceil_div(n, 256), nb), 256, 0, e->stream>>>(
        n, nrb, nullptr, yblk, axblk, asblk, py, pax, pas, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
        nullptr, rowsum);
    const size_t smem = (size_t)np2 * (sizeof(float) + sizeof(int));
    static std::atomic<unsigned long long> attr_set{0};
    PB_TRY(pb_smem_optin(k_order_desc, pb_smem_cap(), attr_set));    // once per device, for every order
    k_order_desc<<<nb, 1024, smem, e->stream>>>(n, np2, rowsum, a, stride, perm);
    const int nt = (n + 31) / 32;
    k_sym_permute_f32<<<dim3(nt, nt, nb), 256, 0, e->stream>>>(a, n, stride, perm, a32);
    e->launches += 4;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

// Upper triangle := lower triangle (transpose) for nb FP64 matrices of order n (32 x 32 tiles
// through shared memory): the symmetric systems whose fill wrote only the lower triangle,
// before a pivoted factorisation that reads both.
__global__ void __launch_bounds__(256)
k_sym_mirror(double2 *a, int n, long long stride)
{
    __shared__ double2 t[32][33];
    const int bx = blockIdx.x, by = blockIdx.y;     // tile column, tile row; upper tiles only
    if (bx < by) return;
    a += (long long)blockIdx.z * stride;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    // read the lower tile (rows bx*32.., cols by*32..), write its transpose into the upper one
    for (int r = ty; r < 32; r += 8) {
        const int i = bx * 32 + r, j = by * 32 + tx;
        t[r][tx] = (i < n && j < n) ? a[(long long)i * n + j] : make_double2(0, 0);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int i = by * 32 + r, j = bx * 32 + tx;       // upper entry (i, j) = lower (j, i)
        if (i < n && j < n && j > i) a[(long long)i * n + j] = t[tx][r];
    }
}

int pb_sym_mirror(pb_lu_engine *e, int n, int nb, double2 *a, long long stride)
{
    if (n <= 0 || nb <= 0) return PB_OK;
    const int nt = (n + 31) / 32;
    k_sym_mirror<<<dim3(nt, nt, nb), 256, 0, e->stream>>>(a, n, stride);
    e->launches++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

int pb_matvec_mapped(pb_lu_engine *e, int n, int nb, int nrhs, const double2 *a, int ld, long stride,
                     const double2 *x, double2 *y, const int *sys)
{
    if (nb <= 0) return PB_OK;
    const size_t xbytes = (size_t)nrhs * n * sizeof(double2);
    const int stage = xbytes <= (size_t)pb_smem_cap();
    const size_t smem = stage ? xbytes : 0;
    PB_TRY(pb_smem_optin(k_residual, pb_smem_cap(), g_residual_attr));
    const int rpb = 64;
    dim3 g(ceil_div(n, rpb), nb);
    k_residual<<<g, 256, smem, e->stream>>>(a, n, ld, stride, nullptr, x, y, nullptr, nullptr, nullptr,
                                            nullptr, nrhs, rpb, sys, nullptr, stage, nullptr);
    e->launches++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}
