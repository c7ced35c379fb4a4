/*
 * peec_b200.h — C ABI of the B200 frequency-sweep library (libpeec_b200.so).
 *
 * The library exports one layer, the batched core ("pb_*"): plain C structs, pointers and
 * sizes. The caller hands over the discretised geometry once (current cells, charge
 * cells, nodes, ports) and then asks for partial-element matrices or a whole frequency
 * sweep. All device memory is owned by an opaque context; every call is synchronous on
 * return. A program built from the reference's host files (parser, geometry, outputs,
 * main) uses it through a small replacement of the reference's solve() that converts its
 * seg_t / chg arrays to pb_cell_t and calls pb_create + pb_sweep; that shim is written in
 * the reference's own C and is not compiled into this library.
 *
 * Return convention of the core: 0 = success, non-zero = error; pb_last_error() returns a
 * message for the calling thread's last failure. There is no host fallback: if no CUDA
 * device is usable every compute entry point fails with PB_ERR_CUDA.
 *
 * Complex numbers cross the ABI as interleaved double pairs {re, im}, matching the
 * reference's d_complex_t (include/complex.h:13).
 */
#ifndef PEEC_B200_H
#define PEEC_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define PB_OK            0
#define PB_ERR_ARG       1   /* invalid argument / size                              */
#define PB_ERR_CUDA      2   /* CUDA runtime or library failure (no device, OOM, ...) */
#define PB_ERR_SINGULAR  3   /* zero pivot in an LU factorisation                     */
#define PB_ERR_NOCONV    4   /* refinement / GMRES did not reach the tolerance        */
#define PB_ERR_UNSUP     5   /* input uses a feature this build does not implement    */

/* Cell shape codes, identical to the reference's SHAPE_* (include/peec.h:50-53). */
#define PB_SHAPE_ROUND 0
#define PB_SHAPE_BAR   1
#define PB_SHAPE_PLATE 2
#define PB_SHAPE_POLY  3

/*
 * One discretised cell (current cell or charge cell). Field meanings follow the
 * reference's seg_t (include/peec.h:108-136); the polygon vertex ring is not stored
 * inline (seg_t carries pv[3*64]) but in a shared pool addressed by pvoff/npv.
 * 256 bytes, no padding.
 */
typedef struct {
    double x1[3], x2[3];   /* axis end points [m]                                   */
    double len;            /* |x2 - x1|                                             */
    double wid;            /* ribbon width (0 = thin filament); polygons: area/len  */
    double thick;          /* thickness (volume bars, skin formula)                 */
    double wv[3];          /* in-plane transverse unit vector (ribbons, bars)       */
    double papex[3];       /* fan apex of a polygon cell                            */
    double aL, aP;         /* equivalent radius for inductance / potential          */
    double radius;         /* round-wire radius                                     */
    double area, perim;    /* cross-section area and perimeter                      */
    double sigma, res;     /* conductivity, DC resistance                           */
    double cexc, gexc, gfac, epss, epsinf, frelax; /* dielectric branch parameters  */
    int    n1, n2;         /* node ids of the two ends (current cells)              */
    int    shape;          /* PB_SHAPE_*                                            */
    int    vol;            /* 1 = volume bar (Hoer-Love pairs)                      */
    int    diel;           /* 1 = dielectric branch                                 */
    int    npv;            /* polygon vertex count (0 = not a polygon)              */
    int    pvoff;          /* first vertex of the ring in the vertex pool           */
    int    pad_;
} pb_cell_t;

typedef struct { int n1, n2; double z0; } pb_port_t;

/* Lumped element kinds (reference rc_t / ind_t / src_t, include/peec.h:40-44). */
#define PB_LUMP_R 0          /* resistor  val = ohm                     */
#define PB_LUMP_C 1          /* capacitor val = farad                   */
#define PB_LUMP_L 2          /* inductor  val = henry (branch current)  */
#define PB_LUMP_V 3          /* ideal voltage source (branch current)   */
typedef struct { int kind, n1, n2; double val; } pb_lump_t;

/* Mutual coupling between two inductors (indices into the PB_LUMP_L elements in
 * order of appearance), M = k sqrt(L1 L2) (reference mut_t, include/peec.h:42). */
typedef struct { int l1, l2; double k; } pb_mutual_t;

typedef struct {
    int nseg;  const pb_cell_t *seg;     /* current cells, reference p->seg order      */
    int nchg;  const pb_cell_t *chg;     /* charge sub-cells, reference p->chg order   */
    const int *chgnode;                  /* [nchg] node id of each charge sub-cell     */
    int npv;   const double *pv;         /* polygon vertex pool [3*npv]                */
    int maxid;                           /* largest node id in use                     */
    int nport; const pb_port_t *port;
    int nlump; const pb_lump_t *lump;
    int nmut;  const pb_mutual_t *mut;
    int capacitance, retardation, skin, gp;
    double gpz, gmin;
} pb_problem_t;

typedef struct pb_ctx pb_ctx;

/* Precision of the partial-element fill / the dense solve. */
#define PB_PREC_FP64   0     /* plain path: FP64 everywhere, static part re-evaluated   */
#define PB_PREC_MIXED  1     /* FP64 static part (cached) + FP32 retardation correction */

/* Dense factorisation used inside the sweep. */
#define PB_LU_FP64     0     /* FP64 panels + FP64 trailing updates                      */
#define PB_LU_FP32     1     /* FP32 panels + FP32 SIMT trailing updates, FP64 refinement */
#define PB_LU_TC       2     /* FP32 panels + tensor-core trailing updates, FP64 refinement;
                                the reduced (complex-symmetric) form is factored as L D L^T
                                without pivoting, every other system by the pivoted LU     */
#define PB_LU_TC_CUBLAS 3    /* comparison baseline: pivoted LU as PB_LU_TC, with cuBLAS's
                                BF16x9 FP32 emulation in place of the library's tcgen05
                                update kernel                                              */
#define PB_LU_TC_PIVOTED 4   /* as PB_LU_TC, always the pivoted LU (comparison)             */
#define PB_LU_LDLT     5     /* pb_lu_decomp_batched32_dev only: the L D L^T factorisation
                                PB_LU_TC uses for the reduced form                          */

/* MNA formulation inside the sweep. */
#define PB_FORM_AUTO    0    /* reduced when applicable, else full                       */
#define PB_FORM_FULL    1    /* the reference's dense MNA (mna.c:175-297), node block jwP^-1
                                written with explicit cell charges (mna.c:86-107), no inverse */
#define PB_FORM_REDUCED 2    /* branch-current Schur form (requires every node = a cell) */

typedef struct {
    int    fill_prec;       /* PB_PREC_*                                               */
    int    lu;              /* PB_LU_*                                                 */
    int    form;            /* PB_FORM_*                                               */
    int    batch;           /* frequencies per device batch (0 = automatic)            */
    double refine_tol;      /* unused (refinement stops at FP64 backward-error level)  */
    int    refine_maxit;    /* max refinement / GMRES iterations (0 = 30)              */
    int    verbose;
    int    corr_freqs;      /* frequencies per retardation-correction launch, 1..16
                               (0 = automatic); a tuning knob, results do not depend on it */
    int    accel;           /* LU reuse, the reference's acceleration = 1 (solve.c:47-64):
                               0 or 1 = one factorisation per frequency;
                               S >= 2 = one FP32 factorisation per S consecutive
                               frequencies of the mixed path, the others solved by FP64
                               right-preconditioned GMRES(60) with the nearest factored
                               frequency's LU (gmres_solve, iterative.c:230-252); systems
                               that do not converge are refactorised (FP64) */
    int    compress;        /* 1 = the reference's compression = 1 path (solve.c:251-294):
                               H-matrix (ACA) of the Lp block, leaf-block + circuit-Schur
                               preconditioner, matrix-free GMRES(60) per port to the relative
                               residual refine_tol (0 = 1e-10, ACCEL_TOL); full MNA form,
                               with capacitance the charge block P is compressed too */
    int    aca_dense;       /* compressed path: 0 = the Lp block's ACA rows / columns and its
                               dense blocks are evaluated on demand from the geometry (no
                               N x N fill, the reference's hmat_entry_fn route); 1 = fill the
                               whole block densely first and compress from it (same values) */
    double ctol;            /* ACA relative tolerance (0 = 1e-6, the reference's default) */
    const float *pc_mlp;    /* compressed path: weights (pb_mlp_nparam() floats) of the learned
                               correction of the preconditioner's leaf blocks, NULL = plain
                               preconditioner; the plain one is the fall back whenever the
                               corrected one fails (singular leaf, GMRES not converged) */
    int pc_coarse;          /* compressed path: >= 1 = two-level preconditioner, a coarse
                               correction over divergence-free coarse currents (one per
                               aggregate and current axis; aggregates = the leaves for 1, their
                               ancestors pc_coarse - 1 levels up otherwise) applied before the
                               plain preconditioner; 0 = the plain preconditioner alone (the
                               reference's) */
    int pc_exact_leaf;      /* compressed path, experiment: 1 = every leaf block of the Lp kernel
                               block replaced by the exact S_r = ((A_LL^-1)_rr)^-1 (the leaf
                               block that makes the block-diagonal preconditioner reproduce
                               the diagonal blocks of the inverse; dense inverse on the GPU,
                               for structures of a few thousand cells): the best any
                               correction of the leaf blocks alone can do; 0 = off */
} pb_sweep_opts;

typedef struct {
    double t_static_ms, t_corr_ms, t_assemble_ms, t_lu_ms, t_refine_ms, t_total_ms;
    double corr_samples;    /* retardation-correction quadrature samples evaluated (the
                               compressed path with on-demand entries: of P only)       */
    double lu_flops;        /* (8/3) n^3 per LU, (4/3) n^3 per L D L^T, summed       */
    double max_resid;       /* largest final normwise backward error |r|/(|A||x|+|b|) */
    int    max_iters;       /* largest refinement iteration count                    */
    int    form_used;       /* PB_FORM_FULL or PB_FORM_REDUCED                       */
    int    n_system;        /* order of the factorised system                        */
    int    static_refreshes;/* how many times the cached static part was rebuilt     */
    int    kernel_launches; /* kernels launched by the last pb_sweep call            */
    int    fp64_fallbacks;  /* frequencies whose mixed solve did not converge and were
                               re-factorised in FP64 (reported, never silent)          */
    int    fp64_direct;     /* frequencies solved directly in FP64 because a lower or
                               equal frequency of the same sweep needed the fallback   */
    double fp64_max_hz;     /* highest frequency that needed FP64                     */
    int    lu_count;        /* factorisations done (all precisions)                   */
    int    gmres_solves;    /* systems solved by preconditioned GMRES (accel >= 2)    */
    int    gmres_its_max;   /* largest GMRES iteration count of one system            */
    int    gmres_refactored;/* systems refactorised at their own frequency (FP32)     */
    double gmres_its_avg;   /* mean GMRES iterations per GMRES-solved system          */
    int    hmat_far, hmat_near;        /* compressed path: far (low-rank) and near blocks */
    int    hmat_max_rank, hmat_dense_far; /* largest ACA rank; far blocks kept dense      */
    double hmat_mb, hmat_dense_mb;     /* H-matrix storage vs the dense Lp block [MiB]  */
    int    pc_mlp_fallbacks;           /* frequencies that fell back to the plain preconditioner */
    int    pc_coarse_n;                /* coarse-space size of the two-level preconditioner */
    double t_coarse_ms;                /* its set-up time (coarse basis and matrix) [ms]   */
    int    probe_fallbacks;/* mixed path: frequencies sent to the FP64 fall back because the
                              conditioning probe found their port voltages sensitive above a
                              quarter of the 1e-6 bar to perturbations of the size of the
                              remaining backward error (counted in fp64_fallbacks too)    */
    int    pipelined;      /* 1 = batches were pipelined: the next batch filled on a second,
                              lower-priority stream while the current one was solved       */
    double probe_max;      /* largest probe sensitivity |dV_port| / |V_port| of the sweep   */
    double hmat_entries;   /* compressed path: entries of the Lp block evaluated, summed over
                              the frequencies (N^2 per frequency for the dense fill)        */
} pb_sweep_stats;

const char *pb_last_error(void);
int  pb_device_count(void);

/* Context lifetime. pb_create copies the geometry to the device. */
int  pb_create(const pb_problem_t *prob, pb_ctx **out);
void pb_destroy(pb_ctx *ctx);
int  pb_sizes(const pb_ctx *ctx, int *nseg, int *nchg, int *ncell, int *nnode, int *nunknown);

/*
 * Dense partial-inductance matrix at wavenumber kw (0 = quasi-static), both triangles,
 * row-major [nseg*nseg] complex. Entry (i,j) equals the reference's lp_entry(p,i,j,kw)
 * (src/partial.c:371-424) including the ground-plane image term.
 */
int  pb_lp_fill(pb_ctx *ctx, double kw, int prec, double *lp_host);

/*
 * Dense potential-coefficient matrix P at cell level (ncell x ncell, complex), entry
 * (i,j) equal to the reference's pot_entry(p,i,j,kw) (src/potential.c:124-150).
 */
int  pb_pot_fill(pb_ctx *ctx, double kw, int prec, double *p_host);

/*
 * Frequency sweep (reference solve(), src/solve.c:171-430, dense path): for every
 * frequency fill Lp/P (retardation) or reuse them (quasi-static), assemble, factorise,
 * solve one 1 A excitation per port. Output zmat [nfreq*nport*nport] complex with the
 * reference's ZIDX layout (include/peec.h:234). Any output pointer may be NULL.
 * segi [nfreq*nport*nseg] receives the segment currents (reference DIDX layout).
 */
int  pb_sweep(pb_ctx *ctx, int nfreq, const double *freq, const pb_sweep_opts *opts,
              double *zmat, double *segi, pb_sweep_stats *stats);

/*
 * pb_sweep with the distribution outputs of distribution = 1 (solve.c:331-362): segi as
 * pb_sweep, and cellq [nfreq*nport*ncell] complex (reference QIDX layout,
 * include/peec.h:237) the cell charges of each port excitation, q = C v on the dense path
 * (obtained without forming C = P^-1: from KCL, j w q = injection - G i, in the reduced
 * form; the charge unknowns in the full form), the charge unknowns on the compressed path.
 * Cells in the reference's order (first appearance of the node id among the charge
 * sub-cells). cellq is left untouched without capacitance. Any output may be NULL.
 */
int  pb_sweep_dist(pb_ctx *ctx, int nfreq, const double *freq, const pb_sweep_opts *opts,
                   double *zmat, double *segi, double *cellq, pb_sweep_stats *stats);

/*
 * Plane-wave incidence (the reference's planewave key, src/input_data.c:501-519):
 * arrival direction (theta, phi) in degrees (propagation is the opposite direction),
 * polarisation 1 = theta-hat, 2 = phi-hat, amplitude [V/m] and phase [deg]. Over a
 * ground plane the PEC reflection is added (mna_rhs_planewave, src/mna.c:434-468).
 */
typedef struct {
    double theta_deg, phi_deg;
    int    pol;
    int    pad_;
    double amp, phase_deg;
} pb_planewave_t;

/*
 * Plane-wave sweep (solve.c:372-389): the same fill and solve as pb_sweep with the
 * induced EMF -integral(E_inc . dl) of every current cell as the excitation and the ports
 * left open. voc [nport*nfreq] complex receives the open-circuit port voltages
 * V(n1) - V(n2) in the reference's layout (voc[i*nfreq + ifreq], include/peec.h:229);
 * segipw [nfreq*nseg] complex (may be NULL) the induced segment currents.
 */
int  pb_planewave(pb_ctx *ctx, int nfreq, const double *freq, const pb_sweep_opts *opts,
                  const pb_planewave_t *pw, double *voc, double *segipw, pb_sweep_stats *stats);

/*
 * Many structures at once (config-3 style batches of small, uneven structures; the
 * reference solves them one after another). Instance k sweeps nfreq[k] frequencies freq[k]
 * through ctx[k] exactly as pb_sweep(ctx[k], ...) would (same kernels, same order: the
 * results are bit-identical), zmat[k] as pb_sweep's zmat (may be NULL), stats [ninst] or
 * NULL. Instances run concurrently on their own streams, largest first, from a shared work
 * queue served by nthreads host threads (0 = min(16, ninst)). The contexts must be
 * distinct. Returns the first failing instance's status, with "instance k: " in front of
 * its message; the others still run.
 */
int  pb_sweep_many(int ninst, pb_ctx *const *ctx, const int *nfreq, const double *const *freq,
                   const pb_sweep_opts *opts, double *const *zmat, pb_sweep_stats *stats, int nthreads);

/*
 * Far field of the sweep's port-1 currents (output_far, src/farfield.c:42-182): for every
 * frequency and direction (theta = thmax*it/nth, it = 0..nth, thmax = pi, or pi/2 over a
 * ground plane with image currents; phi = 2 pi ip/nph) the radiation vector of the current
 * cells and r*E_theta, r*E_phi [V] (et, ep [nfreq][(nth+1)*nph] complex), the directivity
 * and gain [dBi] (d_dbi, g_dbi, same shape, -600 below 1e-30; may be NULL), the radiated
 * power (prad [nfreq]) and the input power 0.5 Re Zin (pin [nfreq]; zin NULL: 0).
 * segi: port-1 segment currents, frequency f at segi + 2*f*seg_stride (complex doubles).
 */
int  pb_farfield(pb_ctx *ctx, int nfreq, const double *freq, const double *segi, long long seg_stride,
                 const double *zin, int nth, int nph, double *et, double *ep, double *d_dbi,
                 double *g_dbi, double *prad, double *pin);

/*
 * Transient synthesis (tran_synth / output_tran, src/transient.c:73-177) of nsig frequency
 * responses h [nsig][nfreq] complex sampled at f_k = k df (f0 = df, f1 = f_max; else
 * PB_ERR_ARG as tran_check): a Gaussian pulse att_db down at f_max, x [2*nfreq] the pulse
 * itself, y [nsig][2*nfreq] the responses, at t_n = n dt, dt = 1/(2 f_max) (*dt_out).
 */
int  pb_transient(int nfreq, double f0, double f1, double att_db, int nsig, const double *h, double *x,
                  double *y, double *dt_out);

/*
 * Independent sources (reference src_t, include/peec.h:43; vsource / isource keys,
 * src/input_data.c:175-192). isvsrc = 1: voltage source amp at phase_deg; the k-th
 * voltage source is the k-th PB_LUMP_V element of the problem (its branch row, mna.c:77).
 * isvsrc = 0: current source, the current flowing inside the source from n1 to n2 (the
 * SPICE convention of mna_rhs_sources, src/mna.c:470-489).
 */
typedef struct { int n1, n2, isvsrc, pad_; double amp, phase_deg; } pb_source_t;

/*
 * The extra solve of solve.c:392-396: the right-hand side of mna_rhs_sources
 * (src/mna.c:471-489) through the dense full-form MNA at every frequency. vnode
 * [nfreq][maxid+1] complex gets the node voltages print_vnode reports
 * (src/solve.c:102-112): x[nodemap[id]], 0 for the reference node and for ids without a
 * matrix row. Not built for the compressed path (PB_ERR_UNSUP).
 */
int  pb_sources(pb_ctx *ctx, int nfreq, const double *freq, const pb_sweep_opts *opts, int nsrc,
                const pb_source_t *src, double *vnode, pb_sweep_stats *stats);

/*
 * Dense complex LU with partial pivoting on a host matrix, executed on the GPU
 * (reference lu_decomp, src/lu.c:16-66): row-major a[n*n] complex is replaced by L\U,
 * piv[k] = row swapped with row k at step k. Returns -1 on success or the 0-based row of
 * the first zero pivot (max |re|+|im| < 1e-30), exactly like the reference; returns -2
 * on a CUDA error. The complex entries are (re, im) double pairs, the layout of the
 * reference's d_complex_t; this C ABI takes double * so that it needs no reference header.
 * The reference-prototype entry point, lu_decomp(int, d_complex_t *, int *), is the
 * drop-in shim's (openpeec_b200/dropin/peec_shim.c), which casts and calls this one.
 */
int  pb_lu_decomp(int n, double *a, int *piv);
/* Forward/back substitution with the factors of pb_lu_decomp (reference lu_solve,
 * src/lu.c:68-96). b[n] complex is overwritten by the solution. Returns 0 or PB_ERR_*. */
int  pb_lu_solve(int n, const double *a, const int *piv, double *b);

/*
 * Batched variant operating on device memory: nb matrices of order n, row-major,
 * complex FP64, stride n*n, factorised in place with the same pivot rule.
 * info[b] = -1 or the zero-pivot row of matrix b. Device pointers (cudaMalloc'd).
 */
int  pb_lu_decomp_batched_dev(int n, int nb, double *a_dev, int *piv_dev, int *info_host);

/*
 * The mixed-precision factorisation of the sweep on device memory: nb matrices of order
 * n, row-major, complex FP32 (interleaved re/im), stride n*n, factorised in place with
 * the pivot rule of lu_decomp (src/lu.c:16-66); lu = PB_LU_TC (tensor-core trailing
 * updates), PB_LU_FP32 (SIMT updates) or PB_LU_TC_CUBLAS. lu = PB_LU_LDLT: the
 * complex-symmetric A = L D L^T without pivoting (only the lower triangle of A is read;
 * stored as an unpivoted LU, unit L below and U = D L^T on and above the diagonal, piv the
 * identity; PB_ERR_UNSUP above ~28 000 unknowns). info_host[b] as above.
 */
int  pb_lu_decomp_batched32_dev(int n, int nb, float *a_dev, int *piv_dev, int *info_host, int lu);

/*
 * The trailing update of the factorisation (the row update of lu_decomp, src/lu.c:54-62,
 * for a block of rows and columns at once): C[b] -= A[b] * B[b] for b < nb, complex FP32
 * (interleaved re/im), row-major, leading dimensions and batch stride in complex
 * elements, device pointers; C is m x nc, A m x k, B k x nc. kind = PB_LU_TC: the
 * library's tcgen05 kernel (split-TF32, 3 products, FP32 accumulation); it needs
 * m, nc >= 128, k >= 16, even leading dimensions and batch stride and 16-byte aligned
 * pointers, else PB_ERR_UNSUP (inside the factorisation such updates go to the SIMT
 * kernel). PB_LU_FP32: the SIMT kernel, any shape. PB_LU_TC_CUBLAS: cuBLAS's BF16x9 FP32
 * emulation. Runs on the default stream; returns 0 once the update is queued, or PB_ERR_*.
 */
int  pb_cgemm_sub_batched_dev(int m, int nc, int k, const float *a_dev, int lda, const float *b_dev,
                              int ldb, float *c_dev, int ldc, long long stride, int nb, int kind);

/*
 * Partial-inductance fill that allocates nothing. It has no counterpart in the reference
 * (whose lp_fill mallocs p->lp itself, src/partial.c:428-435); it exists for host programs
 * that own all device memory through their own pool and may not call cudaMalloc/cudaFree
 * (which may synchronise the whole device and would bypass the host's memory budget).
 * Same matrix as pb_lp_fill: seg_dev = nseg cells in device memory (no polygon cells),
 * lp_dev = caller-allocated device output [nseg*nseg] complex, both triangles.
 * Limit: nseg <= 512. The only scratch is a fixed 2 MiB array in the library that every
 * GPU loading it holds until exit. The first call on each device does a one-time set-up
 * (it looks the array's device address up with cudaGetSymbolAddress), so make that first
 * call before any stream capture.
 * Calls share that scratch and run on the legacy default stream: calls that overlap on
 * the GPU (e.g. from several host threads) race, so serialise them. The call reads seg_dev
 * and writes lp_dev on that stream and synchronises it before returning, so the output is
 * complete on return; the inputs must be complete before the call (a host that filled
 * seg_dev on a non-blocking stream of its own synchronises that stream first).
 */
int  pb_lp_fill_noalloc(int nseg, const pb_cell_t *seg_dev, int gp, double gpz, double kw,
                        int prec, double *lp_dev);

/*
 * Learned preconditioner correction (no counterpart in the reference; the plain method is
 * precond.c:138-391). A 12 -> 128 -> 128 -> 2 tanh MLP maps the features of a current cell
 * to a correction y of the diagonal of its leaf block, D_ii <- D_ii (1 + y_0 + j y_1).
 * Weights are pb_mlp_nparam() floats: W1[128][12], b1, W2[128][128], b2, W3[2][128], b3.
 *
 * pb_pc_samples: training data of one structure at one frequency: x [nseg][12] features,
 *   t [nseg][2] targets (S_r - D_r)_ii / D_ii with S_r = ((A_LL^-1)_rr)^-1, the leaf block
 *   that reproduces the diagonal blocks of the inverse of the whole Lp block (dense inverse
 *   on the GPU, for training-sized structures).
 * pb_mlp_train: full-batch Adam on the GPU (hand-written forward / backward kernels); w is
 *   the initial and final weights, loss_hist [steps] may be NULL.
 * pb_mlp_grad: mean-squared-error loss and its gradient (for gradient checks).
 */
int  pb_mlp_nparam(void);
int  pb_pc_samples(pb_ctx *ctx, double freq, const pb_sweep_opts *opts, float *x, float *t);
int  pb_mlp_train(float *w, int n, const float *x, const float *t, int steps, float lr, float *loss_hist);
int  pb_mlp_grad(const float *w, int n, const float *x, const float *t, float *grad, float *loss);
int  pb_mlp_predict(const float *w, int n, const float *x, float *y);

/* Measured FP32 FMA throughput of the current GPU in TFLOP/s (dependent FMA chains on
 * every SM): the denominator of the fill kernels' roofline. */
int  pb_fp32_peak(double *tflops);
/* cudaDeviceSynchronize on the current device (timing brackets). */
int  pb_device_sync(void);

#ifdef __cplusplus
}
#endif
#endif /* PEEC_B200_H */
