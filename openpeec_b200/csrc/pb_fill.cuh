// pb_fill.cuh — partial-element fill on the device.
#pragma once
#include "pb_common.cuh"

// Device-resident discretisation of one structure.
struct pb_dev_cells {
    int n = 0;
    pb_cell_t *cell = nullptr;      // [n]
    double4 *qpt = nullptr;         // 3-point poly-corr point sets, offsets from centre + weight
    int *qoff = nullptr;            // [n+1]
};

struct pb_fill_geom {
    pb_dev_cells seg, chg;
    double *pv = nullptr;           // shared polygon vertex pool [3*npv]
    int gp = 0;
    double gpz = 0;
    double pmax = 0;                // bound on |R - D| of any correction sample (0 = unknown)
    int any_poly = 0;
    // charge cells grouped by node (potential.c:29-114)
    int ncell = 0;
    int *csoff = nullptr, *csidx = nullptr;   // [ncell+1], [nchg]
    double *carea = nullptr;                   // [ncell]
    // reduced form: cell index of each segment's end nodes (-1 = reference node)
    int *seg_ca = nullptr, *seg_cb = nullptr;  // [nseg]
};

#define PB_FMAX 16
// FP32 path: lower-order product rules for separated ribbon pairs only where k * lmax <=
// PB_FAR_KL at every wavenumber of a launch (lmax: the pair's largest cell dimension)
#define PB_FAR_KL 0.1

// Epilogue of the Lp correction kernel.
enum { PB_EPI_STORE = 0, PB_EPI_REDUCED = 1, PB_EPI_LIST = 2 };

struct pb_epi_args {
    // STORE: out[f][i][j] (both triangles), FP64 complex, stride per frequency
    double2 *out = nullptr;
    long long out_stride = 0;
    // REDUCED: M'(f) = j w zint - w^2 Lp + G^T P G (FP64 and optional FP32 copy)
    double2 *m64 = nullptr;
    float2 *m32 = nullptr;
    long long m_stride = 0;
    const double2 *pm = nullptr;    // P(f) [f][ncell][ncell]
    long long pm_stride = 0;
    const double2 *zint = nullptr;  // [f][nseg]
    int lower = 0;                  // REDUCED: write only the lower triangle (symmetric solves)
    double omega[PB_FMAX];
    // LIST (one wavenumber): out[t] = lscale * Lp(pairs[t]) for t < *npair, the static
    // part read from st[t]; lcap bounds *npair and sizes the launch
    const int2 *pairs = nullptr;
    const int *npair = nullptr;
    long long lcap = 0;
    double lscale_re = 1, lscale_im = 0;
};

// FP64 static tables: stLp[i*n+j] (i <= j) = coef * sum_terms weight * static;
// stP[ci*nc+cj] (ci <= cj) likewise for P.
int pb_lp_static(const pb_fill_geom &g, double kw, double *stLp, cudaStream_t s, long *launches);
int pb_pot_static(const pb_fill_geom &g, double kw, double *stP, cudaStream_t s, long *launches);

// Entries of Lp at one wavenumber for an explicit list of cell pairs (the on-demand rows,
// columns and dense blocks of the compressed path): out[t] = scale * Lp(pairs[t].x,
// pairs[t].y) for t < *npair_dev (device count, at most cap), FP64 static part and the
// FP32 (use_fp32) or FP64 correction. Each entry is evaluated as its (min, max) pair of
// the dense fill (pb_lp_static + pb_lp_corr with nf = 1), so the values are the same bits.
// stl: scratch of cap doubles.
int pb_lp_entries(const pb_fill_geom &g, double kw, int use_fp32, const int2 *pairs, const int *npair_dev,
                  long long cap, double2 scale, double *stl, double2 *out, cudaStream_t s, long *launches);
// The two halves of pb_lp_entries, for callers that keep static parts between wavenumbers:
// static parts stl[t] of the listed pairs (idx != nullptr: only of t = idx[u], u < *nidx_dev,
// at most cap), then out[t] = scale * (stl[t] + correction) for t < *npair_dev.
int pb_lp_entries_static(const pb_fill_geom &g, double kw, const int2 *pairs, const int *idx, const int *nidx_dev,
                         long long cap, double *stl, cudaStream_t s, long *launches);
int pb_lp_entries_corr(const pb_fill_geom &g, double kw, int use_fp32, const int2 *pairs, const int *npair_dev,
                       long long cap, double2 scale, const double *stl, double2 *out, cudaStream_t s,
                       long *launches);

// Correction kernels for nf <= PB_FMAX wavenumbers (kw[f] > 0). use_fp32 selects the
// FP32 quadrature (mixed path) or FP64 (plain path). With kw == 0 (quasi-static) pass
// nf = 1, kw[0] = 0: only the static table is copied through the epilogue.
int pb_lp_corr(const pb_fill_geom &g, int nf, const double *kw, int use_fp32,
               const double *stLp, int epi, const pb_epi_args &ea, cudaStream_t s,
               long *launches, double *samples);
// P correction: sub-cell pair corrections go to igbuf [nf][nchg*nchg] (upper triangle,
// needed only when kw > 0) and are aggregated to cells with the static part into pout.
int pb_pot_corr(const pb_fill_geom &g, int nf, const double *kw, int use_fp32,
                const double *stP, double2 *pout, long long pstride, double2 *igbuf,
                cudaStream_t s, long *launches, double *samples);

// Exact number of correction quadrature samples of one Lp / P fill at wavenumber kw
// (used for throughput and roofline accounting); kw_far32 > 0: as the FP32 path samples
// a launch whose largest wavenumber is kw_far32 (0: the FP64 path).
int pb_count_samples(const pb_fill_geom &g, double kw, double *lp_samples, double *p_samples,
                     cudaStream_t s, unsigned long long *d_count, double kw_far32);

// Internal impedance per segment (skin.c:112-133, mna.c:128-138, mna.c:254-258).
int pb_zint(const pb_fill_geom &g, int skin, int nf, const double *freq, double2 *zint,
            cudaStream_t s, long *launches);

// Poly-corr point sets (cell_qpts(s, 1, 0), polygon.c:224-268) for a cell set.
int pb_build_qpts(pb_dev_cells &c, const pb_cell_t *host_cells, const double *pv_host,
                  const double *pv_dev, cudaStream_t s);
