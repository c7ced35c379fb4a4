// pb_ctx.cuh — the opaque context behind pb_ctx* (include/peec_b200.h).
#pragma once
#include <complex>
#include <map>
#include <vector>
#include "pb_common.cuh"
#include "pb_fill.cuh"
#include "pb_lu.cuh"

// Device storage a context keeps across sweep calls (grow-only, freed by pb_destroy), so
// repeated sweeps of one structure do not reallocate their batch buffers.
struct pb_cache_slot { void *p = nullptr; size_t cap = 0; };
#define PB_CACHE_SLOTS 56
#define PB_SLOT_COMP0  40     // slots [40, 48) hold the compressed path's dense kernel blocks
#define PB_SLOT_POST0  48     // slots [48, 56) hold the far-field buffers (pb_farfield)

// One additive contribution to an MNA entry whose value scales as val * {1, jw, -jw}.
enum { ST_CONST = 0, ST_JW = 1, ST_MJW = 2 };
struct pb_stamp { int kind; double val; };

struct pb_ctx {
    int dev = 0;
    cudaStream_t stream = nullptr;
    pb_lu_engine lu;

    // host copies of the problem
    std::vector<pb_cell_t> seg, chg;
    std::vector<int> chgnode;
    std::vector<double> pv;
    std::vector<pb_port_t> port;
    std::vector<pb_lump_t> lump;
    std::vector<pb_mutual_t> mut;
    int capacitance = 0, retardation = 0, skin = 0, gp = 0, maxid = 0;
    double gpz = 0, gmin = 0;

    // charge-cell grouping (potential.c:29-114)
    int ncell = 0;
    std::vector<int> cellid, cellof, csoff, csidx;
    std::vector<double> carea;
    std::vector<int> cell_of_node;             // [maxid+1] -> cell index or -1

    // MNA numbering (mna.c:16-113)
    std::vector<int> nodemap;
    int nnode = 0, refnode = 0, offL = 0, offV = 0, offS = 0, nunknown = 0, nind = 0, nvsrc = 0;

    // reduced (branch-current) form
    int reduced_ok = 0;
    std::vector<int> seg_ca, seg_cb;           // cell of each segment end, -1 = reference
    std::vector<int> inc_off, inc_seg;         // cell -> incident segments (signed: +k+1 / -(k+1))

    // full (augmented) form: unique entries and their contributions
    int nfull = 0;                             // order of the augmented system
    std::vector<int> fe_row, fe_col, fe_off;   // unique entries, contributions in [fe_off[e], fe_off[e+1])
    std::vector<pb_stamp> fe_st;

    // device geometry
    pb_fill_geom g;
    int *d_inc_off = nullptr, *d_inc_seg = nullptr;
    int *d_fe_row = nullptr, *d_fe_col = nullptr, *d_fe_off = nullptr;
    pb_stamp *d_fe_st = nullptr;
    int *d_cellnode = nullptr;                 // [ncell] matrix index of the cell's node (-1 = ref)
    unsigned long long *d_count = nullptr;     // [2] quadrature-sample counters (statistics)

    pb_cache_slot cache[PB_CACHE_SLOTS];
    // the dense sweep's second stream (lower priority): the next batch's fill runs on it while
    // the current batch is factorised and refined on `stream`
    cudaStream_t stream_fill = nullptr;
    // correction samples (Lp, P) per quadrature-level signature, for the statistics
    std::map<std::vector<long>, std::pair<double, double>> sample_counts;
    // compressed path: level signature whose static parts the held slots contain
    std::vector<long> comp_sig;
    bool comp_static_valid = false;
    // dense path: level signature of the FP64 static tables in cache slots 4 (Lp) and
    // 5 (P), and the slot storage they were written to (a reallocated slot is invalid)
    std::vector<long> dense_sig;
    bool dense_static_valid = false;
    const void *dense_static_ptr[2] = {nullptr, nullptr};
    // compressed path: host copy of the dense circuit Schur complement, page-locked once
    // (cudaHostRegister) so that its per-frequency upload runs at full link speed
    // compressed path: cluster trees, ACA workspaces and the kept static parts of the kernel
    // blocks, held between calls (owned by pb_hmat.cu, released by pb_comp_state_free)
    void *comp_state = nullptr;
    std::vector<std::complex<double>> comp_schur;
    void *comp_schur_reg = nullptr;

    long launches = 0;
};

// Number of sweeps that run concurrently from this host thread's pb_sweep_many: the dense
// sweep sizes its frequency batch from the free device memory divided by it.
extern thread_local int pb_mem_share;
