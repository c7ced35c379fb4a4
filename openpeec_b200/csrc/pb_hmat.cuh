// pb_hmat.cuh — hierarchical compression of the partial-inductance block, the leaf-block +
// circuit-Schur preconditioner and the matrix-free GMRES sweep (compression = 1).
#pragma once
#include <vector>
#include "pb_ctx.cuh"

#define PB_HM_LEAF  32      // largest leaf cluster (HM_LEAF, hmatrix.c:37)
#define PB_HM_ETA   2.0     // admissibility min(diam) <= eta dist (HM_ETA, hmatrix.c:38)
#define PB_HM_MAXIT 200     // largest ACA rank before a block is kept dense (hmatrix.c:39)
#define PB_HM_PROBE 4       // restarts from unrepresented rows (hmatrix.c:40)
#define PB_PC_MAXM  64      // largest leaf the preconditioner factorises (precond.c:41)
#define PB_SCHUR_INV 1024   // circuit Schur complements above this order are applied as an explicit inverse

// Cluster tree and block partition (built on the host: ct_build / hm_split,
// hmatrix.c:91-227) plus the per-leaf block lists of the matrix-vector product.
struct pb_htree {
    int n = 0;
    std::vector<int> perm;                      // cluster order -> cell
    std::vector<int> lo, hi, left, right;       // clusters: [lo, hi) in perm
    std::vector<double> cen, rad;
    std::vector<int> fr, fc;                    // far (admissible) blocks: cluster pairs
    std::vector<int> nr, nc;                    // near blocks
    std::vector<int> leafid;                    // leaf clusters in perm order
};

// Quadrature-level signature of a wavenumber (pb_sweep.cu): equal signatures mean equal
// static parts of the kernel blocks.
void level_signature(const pb_ctx *c, double kw, std::vector<long> &sig);
// Key of the FP32 path's choice of lower-order ribbon rules at largest wavenumber kwmax:
// the number of cells with kwmax * max(len, wid) > PB_FAR_KL. Wavenumbers with equal keys
// give every pair the same rule, hence the same sample count.
long far_rule_key(const pb_ctx *c, double kwmax);

// Builds the tree over pts[3n] and splits the (root, root) block.
void pb_htree_build(pb_htree &t, int n, const double *pts);

// Statistics of the last compressed sweep.
// Releases the compressed path's per-context state (trees, workspaces, kept static parts).
void pb_comp_state_free(pb_ctx *c);

struct pb_hstats {
    int nfar = 0, nnear = 0, ndense_far = 0, max_rank = 0;
    double mem_mb = 0, dense_mb = 0;
    long gmres_its = 0;
    int gmres_max = 0, gmres_rhs = 0;
};

// Compressed sweep (solve.c:251-294 + lin_rhs :75-100): per frequency the dense kernel
// block is filled on the device, compressed (ACA on the far blocks), the sparse part and
// the preconditioner are built, and every port excitation is solved by matrix-free
// right-preconditioned GMRES(60) to the relative residual tol.
// With sample_x / sample_t (nfreq = 1) no system is solved: the features of every current
// cell and the targets of the learned preconditioner correction are written instead.
// pw != nullptr: one plane-wave excitation per frequency instead of the port excitations
// (mna_rhs_planewave, src/mna.c:434-468): voc [nport][nfreq] open-circuit port voltages,
// segipw [nfreq][nseg] branch currents (either may be nullptr), zmat unused.
// Port excitations: segi [nfreq][nport][nseg] branch currents and cellq [nfreq][nport][ncell]
// cell charges (the charge unknowns, solve.c:344-351), either may be nullptr.
int pb_sweep_compressed(pb_ctx *c, int nfreq, const double *freq, const pb_sweep_opts &o,
                        double ctol, double gtol, double *zmat, pb_sweep_stats *stats, pb_hstats *hs,
                        float *sample_x = nullptr, float *sample_t = nullptr,
                        const pb_planewave_t *pw = nullptr, double *voc = nullptr, double *segipw = nullptr,
                        double *segi = nullptr, double *cellq = nullptr);

// Plane-wave right-hand side of the full MNA form at one frequency (freq_dev: one double in
// device memory): -EMF on the branch rows offS + k, zero elsewhere (n rows).
int pb_pw_rhs_full(const pb_ctx *c, const pb_planewave_t *pw, const double *freq_dev, int n, int offS,
                   double2 *rhs, cudaStream_t st);
