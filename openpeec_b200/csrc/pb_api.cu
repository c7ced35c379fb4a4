#include <atomic>
#include <thread>
// pb_api.cu — C entry points of the batched core (include/peec_b200.h).
#include <mutex>
#include "pb_ctx.cuh"
#include "pb_hmat.cuh"
#include "pb_tcgemm.cuh"
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <map>
#include <string>

static thread_local std::string g_err;

void pb_set_error(const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}

int pb_cuda_fail(cudaError_t e, const char *what, const char *file, int line)
{
    pb_set_error("CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e), cudaGetErrorString(e), what, file, line);
    return PB_ERR_CUDA;
}

int pb_sweep_impl(pb_ctx *c, int nfreq, const double *freq, const pb_sweep_opts *opts,
                  double *zmat, double *segi, pb_sweep_stats *stats,
                  const pb_planewave_t *pw, double *voc, double *segipw,
                  const double *rhs_fixed = nullptr, double *vnode = nullptr, double *cellq = nullptr);

extern "C" const char *pb_last_error(void) { return g_err.c_str(); }

extern "C" int pb_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

static int need_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        pb_set_error("no CUDA device available (%s); libpeec_b200 has no host fallback",
                     e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
        return PB_ERR_CUDA;
    }
    return PB_OK;
}

template <typename T> static int upload(T **d, const T *h, size_t n, cudaStream_t s)
{
    PB_CUDA(cudaMalloc(d, sizeof(T) * (n > 0 ? n : 1)));
    if (n > 0 && h) PB_CUDA(cudaMemcpyAsync(*d, h, sizeof(T) * n, cudaMemcpyHostToDevice, s));
    return PB_OK;
}

static int build(pb_ctx *c)
{
    const int nh = (int)c->chg.size(), ns = (int)c->seg.size();
    // potential.c:29-62 : cells in order of first appearance of the node id
    c->cellof.assign(nh, 0);
    c->cellid.clear();
    std::map<int, int> seen;
    for (int h = 0; h < nh; h++) {
        auto it = seen.find(c->chgnode[h]);
        int id;
        if (it == seen.end()) { id = (int)c->cellid.size(); seen[c->chgnode[h]] = id; c->cellid.push_back(c->chgnode[h]); }
        else id = it->second;
        c->cellof[h] = id;
    }
    c->ncell = (int)c->cellid.size();
    c->carea.assign(c->ncell, 0.0);
    for (int h = 0; h < nh; h++) c->carea[c->cellof[h]] += c->chg[h].len;
    c->csoff.assign(c->ncell + 1, 0);                    // potential.c:72-97
    for (int h = 0; h < nh; h++) c->csoff[c->cellof[h] + 1]++;
    for (int i = 0; i < c->ncell; i++) c->csoff[i + 1] += c->csoff[i];
    c->csidx.assign(nh, 0);
    {
        std::vector<int> fill(c->csoff);
        for (int h = 0; h < nh; h++) c->csidx[fill[c->cellof[h]]++] = h;
    }
    // mna.c:16-84 : numbering
    const int nid = c->maxid + 1;
    auto bad = [&](int id) { return id < 0 || id >= nid; };
    std::vector<int> used(nid, 0);
    for (auto &l : c->lump) { if (bad(l.n1) || bad(l.n2)) return PB_ERR_ARG; used[l.n1] = used[l.n2] = 1; }
    for (auto &p : c->port) { if (bad(p.n1) || bad(p.n2)) return PB_ERR_ARG; used[p.n1] = used[p.n2] = 1; }
    for (auto &s : c->seg) { if (bad(s.n1) || bad(s.n2)) return PB_ERR_ARG; used[s.n1] = used[s.n2] = 1; }
    for (int h = 0; h < nh; h++) if (bad(c->chgnode[h])) return PB_ERR_ARG;
    const int usecap = c->capacitance && c->ncell > 0;
    c->refnode = (usecap || used[0]) ? 0 : c->port[0].n2;
    c->nodemap.assign(nid, -2);
    int idx = 0;
    for (int id = 0; id < nid; id++) {
        if (id == c->refnode) c->nodemap[id] = -1;
        else if (used[id]) c->nodemap[id] = idx++;
    }
    c->nnode = idx;
    c->nind = c->nvsrc = 0;
    for (auto &l : c->lump) { c->nind += l.kind == PB_LUMP_L; c->nvsrc += l.kind == PB_LUMP_V; }
    c->offL = c->nnode;
    c->offV = c->offL + c->nind;
    c->offS = c->offV + c->nvsrc;
    c->nunknown = c->offS + ns;
    c->cell_of_node.assign(nid, -1);
    for (int i = 0; i < c->ncell; i++) c->cell_of_node[c->cellid[i]] = i;

    // reduced form applicability
    int ok = usecap && c->gmin == 0 && c->lump.empty() && c->mut.empty();
    for (int id = 0; ok && id < nid; id++)
        if (c->nodemap[id] >= 0 && c->cell_of_node[id] < 0) ok = 0;   // matrix node without a cell
    for (int i = 0; ok && i < c->ncell; i++)
        if (c->nodemap[c->cellid[i]] < 0) ok = 0;                       // cell on the reference node
    c->reduced_ok = ok;
    c->seg_ca.assign(ns, -1);
    c->seg_cb.assign(ns, -1);
    c->inc_off.assign(c->ncell + 1, 0);
    c->inc_seg.clear();
    if (ok) {
        for (int k = 0; k < ns; k++) {
            const pb_cell_t &s = c->seg[k];
            c->seg_ca[k] = c->nodemap[s.n1] >= 0 ? c->cell_of_node[s.n1] : -1;
            c->seg_cb[k] = c->nodemap[s.n2] >= 0 ? c->cell_of_node[s.n2] : -1;
        }
        std::vector<std::vector<int>> inc(c->ncell);
        for (int k = 0; k < ns; k++) {
            if (c->seg_ca[k] >= 0) inc[c->seg_ca[k]].push_back(k + 1);
            if (c->seg_cb[k] >= 0) inc[c->seg_cb[k]].push_back(-(k + 1));
        }
        for (int i = 0; i < c->ncell; i++) {
            c->inc_off[i + 1] = c->inc_off[i] + (int)inc[i].size();
            c->inc_seg.insert(c->inc_seg.end(), inc[i].begin(), inc[i].end());
        }
    }

    // full (augmented) form: contributions per unique entry, in the reference's
    // stamping order (mna.c:181-241, 248-251, 277-278)
    c->nfull = c->nunknown + (usecap ? c->ncell : 0);
    std::map<std::pair<int, int>, std::vector<pb_stamp>> ent;
    auto put = [&](int i, int j, int kind, double v) {
        if (i < 0 || j < 0) return;                      // mna.c:156
        ent[std::make_pair(i, j)].push_back(pb_stamp{kind, v});
    };
    const int *map = c->nodemap.data();
    if (c->gmin > 0) for (int i = 0; i < c->nnode; i++) put(i, i, ST_CONST, c->gmin);
    for (int pass = 0; pass < 2; pass++)
        for (auto &l : c->lump) {
            if (l.kind != (pass ? PB_LUMP_C : PB_LUMP_R)) continue;
            const int i1 = map[l.n1], i2 = map[l.n2];
            const int k = pass ? ST_JW : ST_CONST;
            const double y = pass ? l.val : 1 / l.val;
            put(i1, i1, k, y); put(i2, i2, k, y); put(i1, i2, k, -y); put(i2, i1, k, -y);
        }
    std::vector<double> lval;
    int il = 0;
    for (auto &l : c->lump) {
        if (l.kind != PB_LUMP_L) continue;
        const int i1 = map[l.n1], i2 = map[l.n2], r = c->offL + il++;
        lval.push_back(l.val);
        put(i1, r, ST_CONST, 1); put(r, i1, ST_CONST, 1); put(i2, r, ST_CONST, -1); put(r, i2, ST_CONST, -1);
        put(r, r, ST_MJW, l.val);
    }
    for (auto &m : c->mut) {
        if (m.l1 < 0 || m.l2 < 0 || m.l1 >= (int)lval.size() || m.l2 >= (int)lval.size()) return PB_ERR_ARG;
        const double mm = m.k * std::sqrt(lval[m.l1] * lval[m.l2]);
        put(c->offL + m.l1, c->offL + m.l2, ST_MJW, mm);
        put(c->offL + m.l2, c->offL + m.l1, ST_MJW, mm);
    }
    int iv = 0;
    for (auto &l : c->lump) {
        if (l.kind != PB_LUMP_V) continue;
        const int i1 = map[l.n1], i2 = map[l.n2], r = c->offV + iv++;
        put(i1, r, ST_CONST, 1); put(r, i1, ST_CONST, 1); put(i2, r, ST_CONST, -1); put(r, i2, ST_CONST, -1);
    }
    for (int k = 0; k < ns; k++) {
        const int i1 = map[c->seg[k].n1], i2 = map[c->seg[k].n2], rk = c->offS + k;
        put(i1, rk, ST_CONST, 1); put(rk, i1, ST_CONST, 1); put(i2, rk, ST_CONST, -1); put(rk, i2, ST_CONST, -1);
    }
    if (usecap)
        for (int i = 0; i < c->ncell; i++) {
            const int mi = map[c->cellid[i]], ri = c->nunknown + i;
            put(mi, ri, ST_JW, 1);
            put(ri, mi, ST_CONST, -1);
        }
    c->fe_row.clear(); c->fe_col.clear(); c->fe_off.assign(1, 0); c->fe_st.clear();
    for (auto &kv : ent) {
        c->fe_row.push_back(kv.first.first);
        c->fe_col.push_back(kv.first.second);
        c->fe_st.insert(c->fe_st.end(), kv.second.begin(), kv.second.end());
        c->fe_off.push_back((int)c->fe_st.size());
    }
    return PB_OK;
}

extern "C" {

int pb_create(const pb_problem_t *prob, pb_ctx **out)
{
    if (!prob || !out) { pb_set_error("pb_create: null argument"); return PB_ERR_ARG; }
    *out = nullptr;
    if (prob->nseg < 0 || prob->nchg < 0 || prob->npv < 0 || prob->nport <= 0 || prob->maxid < 0 ||
        (prob->nseg > 0 && !prob->seg) || (prob->nchg > 0 && (!prob->chg || !prob->chgnode)) ||
        (prob->npv > 0 && !prob->pv) || !prob->port || (prob->nlump > 0 && !prob->lump) ||
        (prob->nmut > 0 && !prob->mut)) {
        pb_set_error("pb_create: inconsistent problem description");
        return PB_ERR_ARG;
    }
    PB_TRY(need_device());
    pb_ctx *c = new pb_ctx();
    c->seg.assign(prob->seg, prob->seg + prob->nseg);
    c->chg.assign(prob->chg, prob->chg + prob->nchg);
    c->chgnode.assign(prob->chgnode, prob->chgnode + prob->nchg);
    c->pv.assign(prob->pv, prob->pv + 3 * (size_t)prob->npv);
    c->port.assign(prob->port, prob->port + prob->nport);
    c->lump.assign(prob->lump, prob->lump + prob->nlump);
    c->mut.assign(prob->mut, prob->mut + prob->nmut);
    c->capacitance = prob->capacitance; c->retardation = prob->retardation;
    c->skin = prob->skin; c->gp = prob->gp; c->gpz = prob->gpz; c->gmin = prob->gmin;
    c->maxid = prob->maxid;
    for (auto &s : c->seg)
        if (s.npv > 0 && (s.npv > PB_POLY_MAX || s.pvoff < 0 || s.pvoff + s.npv > prob->npv)) { delete c; pb_set_error("pb_create: polygon ring out of range"); return PB_ERR_ARG; }
    for (auto &s : c->chg)
        if (s.npv > 0 && (s.npv > PB_POLY_MAX || s.pvoff < 0 || s.pvoff + s.npv > prob->npv)) { delete c; pb_set_error("pb_create: polygon ring out of range"); return PB_ERR_ARG; }
    int r = build(c);
    if (r != PB_OK) { delete c; if (r == PB_ERR_ARG) pb_set_error("pb_create: node id out of range"); return r; }

    cudaGetDevice(&c->dev);
    // the solve stream at the highest priority, the fill stream at the lowest: while both
    // have work, the latency-bound factorisation and refinement kernels get SMs first and the
    // issue-bound fill takes what is left
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&c->stream_fill, cudaStreamNonBlocking, prio_lo) != cudaSuccess) {
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c; pb_set_error("cudaStreamCreate failed"); return PB_ERR_CUDA;
    }
    const cudaStream_t s = c->stream;
    auto fail = [&](int rr) { pb_destroy(c); return rr; };
    pb_fill_geom &g = c->g;
    g.gp = c->gp; g.gpz = c->gpz; g.ncell = c->ncell;
    {
        // largest cell extent -> bound on |R - D| = |p| <= extent(cell 1) + extent(cell 2)
        // of the correction samples (offsets p within the two cells of a term)
        double ext = 0;
        for (auto *v : {&c->seg, &c->chg})
            for (auto &x : *v) {
                double e = x.len + x.wid + x.thick + 2 * x.radius;
                if (x.npv > 0) {
                    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
                    for (int q = 0; q < x.npv; q++)
                        for (int d = 0; d < 3; d++) {
                            lo[d] = std::min(lo[d], c->pv[3 * (x.pvoff + q) + d]);
                            hi[d] = std::max(hi[d], c->pv[3 * (x.pvoff + q) + d]);
                        }
                    double d2 = 0;
                    for (int d = 0; d < 3; d++) d2 += (hi[d] - lo[d]) * (hi[d] - lo[d]);
                    e = std::max(e, std::sqrt(d2));
                }
                ext = std::max(ext, e);
            }
        g.pmax = 2 * ext;
    }
    g.seg.n = (int)c->seg.size();
    g.chg.n = (int)c->chg.size();
    if ((r = upload(&g.seg.cell, c->seg.data(), c->seg.size(), s))) return fail(r);
    if ((r = upload(&g.chg.cell, c->chg.data(), c->chg.size(), s))) return fail(r);
    if ((r = upload(&g.pv, c->pv.data(), c->pv.size(), s))) return fail(r);
    if ((r = upload(&g.csoff, c->csoff.data(), c->csoff.size(), s))) return fail(r);
    if ((r = upload(&g.csidx, c->csidx.data(), c->csidx.size(), s))) return fail(r);
    if ((r = upload(&g.carea, c->carea.data(), c->carea.size(), s))) return fail(r);
    if ((r = upload(&g.seg_ca, c->seg_ca.data(), c->seg_ca.size(), s))) return fail(r);
    if ((r = upload(&g.seg_cb, c->seg_cb.data(), c->seg_cb.size(), s))) return fail(r);
    if ((r = upload(&c->d_inc_off, c->inc_off.data(), c->inc_off.size(), s))) return fail(r);
    if ((r = upload(&c->d_inc_seg, c->inc_seg.data(), c->inc_seg.size(), s))) return fail(r);
    if ((r = upload(&c->d_fe_row, c->fe_row.data(), c->fe_row.size(), s))) return fail(r);
    if ((r = upload(&c->d_fe_col, c->fe_col.data(), c->fe_col.size(), s))) return fail(r);
    if ((r = upload(&c->d_fe_off, c->fe_off.data(), c->fe_off.size(), s))) return fail(r);
    if ((r = upload(&c->d_fe_st, c->fe_st.data(), c->fe_st.size(), s))) return fail(r);
    int anyp = 0;
    for (auto &x : c->seg) anyp |= x.npv > 0;
    for (auto &x : c->chg) anyp |= x.npv > 0;
    g.any_poly = anyp;
    if (anyp) {
        if ((r = pb_build_qpts(g.seg, c->seg.data(), c->pv.data(), g.pv, s))) return fail(r);
        if ((r = pb_build_qpts(g.chg, c->chg.data(), c->pv.data(), g.pv, s))) return fail(r);
    }
    {
        cudaError_t e = cudaMalloc(&c->d_count, 2 * sizeof(unsigned long long));
        if (e != cudaSuccess) { c->d_count = nullptr; return fail(pb_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__)); }
    }
    if ((r = pb_lu_engine_init(&c->lu, s))) return fail(r);
    if (cudaStreamSynchronize(s) != cudaSuccess) return fail(pb_cuda_fail(cudaGetLastError(), "upload", __FILE__, __LINE__));
    *out = c;
    return PB_OK;
}

void pb_destroy(pb_ctx *c)
{
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->stream_fill) cudaStreamSynchronize(c->stream_fill);
    void *ptrs[] = {c->g.seg.cell, c->g.seg.qpt, c->g.seg.qoff, c->g.chg.cell, c->g.chg.qpt,
                    c->g.chg.qoff, c->g.pv, c->g.csoff, c->g.csidx, c->g.carea, c->g.seg_ca,
                    c->g.seg_cb, c->d_inc_off, c->d_inc_seg, c->d_fe_row, c->d_fe_col, c->d_fe_off,
                    c->d_fe_st, c->d_cellnode, c->d_count};
    for (void *p : ptrs) if (p) cudaFree(p);
    for (auto &slot : c->cache) if (slot.p) cudaFree(slot.p);
    if (c->comp_schur_reg) cudaHostUnregister(c->comp_schur_reg);
    pb_comp_state_free(c);
    pb_lu_engine_free(&c->lu);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->stream_fill) cudaStreamDestroy(c->stream_fill);
    delete c;
}

int pb_sizes(const pb_ctx *c, int *nseg, int *nchg, int *ncell, int *nnode, int *nunknown)
{
    if (!c) return PB_ERR_ARG;
    if (nseg) *nseg = (int)c->seg.size();
    if (nchg) *nchg = (int)c->chg.size();
    if (ncell) *ncell = c->ncell;
    if (nnode) *nnode = c->nnode;
    if (nunknown) *nunknown = c->nunknown;
    return PB_OK;
}

int pb_lp_fill(pb_ctx *c, double kw, int prec, double *lp_host)
{
    if (!c || !lp_host || kw < 0) { pb_set_error("pb_lp_fill: bad argument"); return PB_ERR_ARG; }
    const int n = (int)c->seg.size();
    if (n == 0) return PB_OK;
    double *st = nullptr;
    double2 *out = nullptr;
    PB_CUDA(cudaMalloc(&st, sizeof(double) * (size_t)n * n));
    cudaError_t e = cudaMalloc(&out, sizeof(double2) * (size_t)n * n);
    if (e != cudaSuccess) { cudaFree(st); return pb_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__); }
    int r = pb_lp_static(c->g, kw, st, c->stream, &c->launches);
    pb_epi_args ea;
    ea.out = out;
    ea.out_stride = (long long)n * n;
    if (r == PB_OK) r = pb_lp_corr(c->g, 1, &kw, prec == PB_PREC_MIXED, st, PB_EPI_STORE, ea, c->stream, &c->launches, nullptr);
    if (r == PB_OK) {
        e = cudaMemcpyAsync(lp_host, out, sizeof(double2) * (size_t)n * n, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) r = pb_cuda_fail(e, "pb_lp_fill copy", __FILE__, __LINE__);
    }
    cudaFree(st);
    cudaFree(out);
    return r;
}

int pb_pot_fill(pb_ctx *c, double kw, int prec, double *p_host)
{
    if (!c || !p_host || kw < 0) { pb_set_error("pb_pot_fill: bad argument"); return PB_ERR_ARG; }
    const int n = c->ncell;
    if (n == 0) return PB_OK;
    double *st = nullptr;
    double2 *out = nullptr;
    PB_CUDA(cudaMalloc(&st, sizeof(double) * (size_t)n * n));
    cudaError_t e = cudaMalloc(&out, sizeof(double2) * (size_t)n * n);
    if (e != cudaSuccess) { cudaFree(st); return pb_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__); }
    double2 *ig = nullptr;
    if (kw > 0) {
        e = cudaMalloc(&ig, sizeof(double2) * (size_t)c->chg.size() * c->chg.size());
        if (e != cudaSuccess) { cudaFree(st); cudaFree(out); return pb_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__); }
    }
    int r = pb_pot_static(c->g, kw, st, c->stream, &c->launches);
    if (r == PB_OK) r = pb_pot_corr(c->g, 1, &kw, prec == PB_PREC_MIXED, st, out, (long long)n * n, ig, c->stream, &c->launches, nullptr);
    if (r == PB_OK) {
        e = cudaMemcpyAsync(p_host, out, sizeof(double2) * (size_t)n * n, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) r = pb_cuda_fail(e, "pb_pot_fill copy", __FILE__, __LINE__);
    }
    cudaFree(st);
    cudaFree(out);
    if (ig) cudaFree(ig);
    return r;
}

int pb_sweep(pb_ctx *c, int nfreq, const double *freq, const pb_sweep_opts *opts, double *zmat,
             double *segi, pb_sweep_stats *stats)
{
    if (!c) { pb_set_error("pb_sweep: null context"); return PB_ERR_ARG; }
    PB_CUDA(cudaSetDevice(c->dev));
    return pb_sweep_impl(c, nfreq, freq, opts, zmat, segi, stats, nullptr, nullptr, nullptr);
}

int pb_sweep_dist(pb_ctx *c, int nfreq, const double *freq, const pb_sweep_opts *opts, double *zmat,
                  double *segi, double *cellq, pb_sweep_stats *stats)
{
    if (!c) { pb_set_error("pb_sweep_dist: null context"); return PB_ERR_ARG; }
    PB_CUDA(cudaSetDevice(c->dev));
    return pb_sweep_impl(c, nfreq, freq, opts, zmat, segi, stats, nullptr, nullptr, nullptr, nullptr, nullptr,
                         cellq);
}

int pb_sweep_many(int ninst, pb_ctx *const *ctx, const int *nfreq, const double *const *freq,
                  const pb_sweep_opts *opts, double *const *zmat, pb_sweep_stats *stats, int nthreads)
{
    if (ninst <= 0 || !ctx || !nfreq || !freq) { pb_set_error("pb_sweep_many: bad argument"); return PB_ERR_ARG; }
    {
        std::vector<const pb_ctx *> seen(ctx, ctx + ninst);
        std::sort(seen.begin(), seen.end());
        for (int k = 0; k < ninst; k++)
            if (!seen[k] || (k > 0 && seen[k] == seen[k - 1])) {
                pb_set_error("pb_sweep_many: null or repeated context");
                return PB_ERR_ARG;
            }
    }
    // work queue: largest system first, so the long instances start early
    std::vector<int> order(ninst);
    for (int k = 0; k < ninst; k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (double)ctx[a]->nfull * ctx[a]->nfull * nfreq[a] > (double)ctx[b]->nfull * ctx[b]->nfull * nfreq[b];
    });
    const int nt = std::max(1, std::min(nthreads > 0 ? nthreads : 16, ninst));
    std::atomic<int> next{0};
    std::vector<int> rc(ninst, PB_OK);
    std::vector<std::string> msg(ninst);
    auto worker = [&]() {
        pb_mem_share = nt;
        for (;;) {
            const int q = next.fetch_add(1);
            if (q >= ninst) return;
            const int k = order[q];
            cudaError_t e = cudaSetDevice(ctx[k]->dev);
            int r = e == cudaSuccess ? PB_OK : pb_cuda_fail(e, "cudaSetDevice", __FILE__, __LINE__);
            if (r == PB_OK)
                r = pb_sweep_impl(ctx[k], nfreq[k], freq[k], opts, zmat ? zmat[k] : nullptr, nullptr,
                                  stats ? &stats[k] : nullptr, nullptr, nullptr, nullptr);
            rc[k] = r;
            if (r != PB_OK) msg[k] = pb_last_error();
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) th.emplace_back(worker);
    worker();
    pb_mem_share = 1;
    for (auto &x : th) x.join();
    for (int k = 0; k < ninst; k++)
        if (rc[k] != PB_OK) {
            pb_set_error("instance %d: %s", k, msg[k].c_str());
            return rc[k];
        }
    return PB_OK;
}

int pb_pc_samples(pb_ctx *c, double freq, const pb_sweep_opts *opts, float *x, float *t)
{
    if (!c || !x || !t || !(freq > 0)) { pb_set_error("pb_pc_samples: bad argument"); return PB_ERR_ARG; }
    PB_CUDA(cudaSetDevice(c->dev));
    pb_sweep_opts o;
    memset(&o, 0, sizeof(o));
    if (opts) o = *opts;
    else o.fill_prec = PB_PREC_MIXED;
    pb_hstats hs;
    return pb_sweep_compressed(c, 1, &freq, o, o.ctol > 0 ? o.ctol : 1e-6, 1e-10, nullptr, nullptr, &hs, x, t);
}

int pb_planewave(pb_ctx *c, int nfreq, const double *freq, const pb_sweep_opts *opts,
                 const pb_planewave_t *pw, double *voc, double *segipw, pb_sweep_stats *stats)
{
    if (!c) { pb_set_error("pb_planewave: null context"); return PB_ERR_ARG; }
    if (!pw) { pb_set_error("pb_planewave: null plane wave"); return PB_ERR_ARG; }
    if (!(pw->amp > 0)) { pb_set_error("pb_planewave: amplitude must be > 0"); return PB_ERR_ARG; }
    PB_CUDA(cudaSetDevice(c->dev));
    return pb_sweep_impl(c, nfreq, freq, opts, nullptr, nullptr, stats, pw, voc, segipw);
}

int pb_sources(pb_ctx *c, int nfreq, const double *freq, const pb_sweep_opts *opts, int nsrc,
               const pb_source_t *src, double *vnode, pb_sweep_stats *stats)
{
    if (!c || nsrc <= 0 || !src || !vnode) { pb_set_error("pb_sources: bad argument"); return PB_ERR_ARG; }
    PB_CUDA(cudaSetDevice(c->dev));
    pb_sweep_opts o;
    memset(&o, 0, sizeof(o));
    if (opts) o = *opts;
    else { o.fill_prec = PB_PREC_MIXED; o.lu = PB_LU_TC; }
    if (o.compress) { pb_set_error("pb_sources: not built for the compressed path"); return PB_ERR_UNSUP; }
    if (o.form == PB_FORM_REDUCED) { pb_set_error("pb_sources: node voltages need the full MNA form"); return PB_ERR_ARG; }
    o.form = PB_FORM_FULL;
    // right-hand side of mna_rhs_sources (src/mna.c:471-489), frequency independent
    std::vector<int> vl;
    for (size_t i = 0; i < c->lump.size(); i++)
        if (c->lump[i].kind == PB_LUMP_V) vl.push_back((int)i);
    std::vector<double> b(2 * (size_t)c->nfull, 0.0);
    size_t nv = 0;
    for (int k = 0; k < nsrc; k++) {
        const pb_source_t &e = src[k];
        if (e.n1 < 0 || e.n2 < 0 || e.n1 > c->maxid || e.n2 > c->maxid) {
            pb_set_error("pb_sources: source %d has a node outside 0..%d", k, c->maxid);
            return PB_ERR_ARG;
        }
        const double ph = e.phase_deg * PB_PI / 180, vr = e.amp * cos(ph), vi = e.amp * sin(ph);
        if (e.isvsrc) {
            if (nv >= vl.size() || c->lump[vl[nv]].n1 != e.n1 || c->lump[vl[nv]].n2 != e.n2) {
                pb_set_error("pb_sources: voltage source %d is not the %zu-th PB_LUMP_V element of the problem", k, nv);
                return PB_ERR_ARG;
            }
            const size_t r = (size_t)(c->offV + nv++);
            b[2 * r] = vr;
            b[2 * r + 1] = vi;
        } else {
            const int i1 = c->nodemap[e.n1], i2 = c->nodemap[e.n2];
            if (i1 >= 0) { b[2 * (size_t)i1] -= vr; b[2 * (size_t)i1 + 1] -= vi; }
            if (i2 >= 0) { b[2 * (size_t)i2] += vr; b[2 * (size_t)i2 + 1] += vi; }
        }
    }
    if (nv != vl.size()) {
        pb_set_error("pb_sources: %zu voltage sources for %zu PB_LUMP_V elements", nv, vl.size());
        return PB_ERR_ARG;
    }
    return pb_sweep_impl(c, nfreq, freq, &o, nullptr, nullptr, stats, nullptr, nullptr, nullptr, b.data(), vnode);
}

// ---------------------------------------------------------------- dense LU entry points
int pb_lu_decomp_batched_dev(int n, int nb, double *a_dev, int *piv_dev, int *info_host)
{
    if (n <= 0 || nb <= 0 || !a_dev || !piv_dev || !info_host) { pb_set_error("pb_lu_decomp_batched_dev: bad argument"); return PB_ERR_ARG; }
    PB_TRY(need_device());
    pb_lu_engine e;
    PB_TRY(pb_lu_engine_init(&e, nullptr));
    e.gemm_kind = PB_GEMM_FP64;
    int *info = nullptr;
    cudaError_t ce = cudaMalloc(&info, sizeof(int) * nb);
    if (ce != cudaSuccess) { pb_lu_engine_free(&e); return pb_cuda_fail(ce, "cudaMalloc", __FILE__, __LINE__); }
    int r = pb_lu_factor<double>(&e, n, nb, (double2 *)a_dev, n, (long)n * n, piv_dev, info);
    if (r == PB_OK) {
        ce = cudaMemcpy(info_host, info, sizeof(int) * nb, cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) r = pb_cuda_fail(ce, "cudaMemcpy", __FILE__, __LINE__);
    }
    cudaFree(info);
    pb_lu_engine_free(&e);
    return r;
}

int pb_lu_decomp_batched32_dev(int n, int nb, float *a_dev, int *piv_dev, int *info_host, int lu)
{
    if (n <= 0 || nb <= 0 || !a_dev || !piv_dev || !info_host) { pb_set_error("pb_lu_decomp_batched32_dev: bad argument"); return PB_ERR_ARG; }
    if (lu != PB_LU_TC && lu != PB_LU_FP32 && lu != PB_LU_TC_CUBLAS && lu != PB_LU_LDLT) {
        pb_set_error("pb_lu_decomp_batched32_dev: bad kind %d", lu);
        return PB_ERR_ARG;
    }
    PB_TRY(need_device());
    pb_lu_engine e;
    PB_TRY(pb_lu_engine_init(&e, nullptr));
    e.gemm_kind = (lu == PB_LU_TC || lu == PB_LU_LDLT) ? PB_GEMM_TC : lu == PB_LU_FP32 ? PB_GEMM_FP32 : PB_GEMM_TC_BLAS;
    int *info = nullptr;
    float *emb = nullptr;
    cudaError_t ce = cudaMalloc(&info, sizeof(int) * nb);
    if (ce == cudaSuccess && lu == PB_LU_TC_CUBLAS) {
        e.emb_cap = (size_t)nb * n * n * sizeof(float);      // largest embedded right operand
        ce = cudaMalloc(&emb, e.emb_cap);
        e.emb = emb;
    }
    if (ce != cudaSuccess) { cudaFree(info); pb_lu_engine_free(&e); return pb_cuda_fail(ce, "cudaMalloc", __FILE__, __LINE__); }
    int r = lu == PB_LU_LDLT ? pb_ldl_factor(&e, n, nb, (float2 *)a_dev, n, (long)n * n, piv_dev, info)
                             : pb_lu_factor<float>(&e, n, nb, (float2 *)a_dev, n, (long)n * n, piv_dev, info);
    if (r == PB_ERR_UNSUP) pb_set_error("pb_lu_decomp_batched32_dev: L D L^T panel of order %d does not fit", n);
    if (r == PB_OK) {
        ce = cudaMemcpy(info_host, info, sizeof(int) * nb, cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) r = pb_cuda_fail(ce, "cudaMemcpy", __FILE__, __LINE__);
    }
    cudaFree(info);
    cudaFree(emb);
    pb_lu_engine_free(&e);
    return r;
}

int pb_cgemm_sub_batched_dev(int m, int nc, int k, const float *a_dev, int lda, const float *b_dev, int ldb,
                             float *c_dev, int ldc, long long stride, int nb, int kind)
{
    if (m < 0 || nc < 0 || k < 0 || nb < 0 || (m && nc && k && nb && (!a_dev || !b_dev || !c_dev)) ||
        lda < k || ldb < nc || ldc < nc || (nb > 1 && stride < (long long)m * ldc)) {
        pb_set_error("pb_cgemm_sub_batched_dev: bad argument");
        return PB_ERR_ARG;
    }
    if (kind != PB_LU_TC && kind != PB_LU_FP32 && kind != PB_LU_TC_CUBLAS) { pb_set_error("pb_cgemm_sub_batched_dev: bad kind %d", kind); return PB_ERR_ARG; }
    PB_TRY(need_device());
    if (kind == PB_LU_TC && m > 0 && nc > 0 && k > 0 && nb > 0 &&
        (m < 128 || nc < 128 || k < 16 ||
         !pb_cgemm_tc_ok((const float2 *)a_dev, lda, (const float2 *)b_dev, ldb, (const float2 *)c_dev, ldc, stride, nb))) {
        pb_set_error("pb_cgemm_sub_batched_dev: the tensor-core kernel needs m, nc >= 128, k >= 16, even leading "
                     "dimensions and batch stride, and 16-byte aligned pointers");
        return PB_ERR_UNSUP;
    }
    static pb_lu_engine eng;                 // one engine per process for this entry point
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (!eng.blas) PB_TRY(pb_lu_engine_init(&eng, nullptr));
    eng.gemm_kind = kind == PB_LU_TC ? PB_GEMM_TC : kind == PB_LU_FP32 ? PB_GEMM_FP32 : PB_GEMM_TC_BLAS;
    if (kind == PB_LU_TC_CUBLAS) {
        // the comparison's embedded right operand, kept between calls (grow-only)
        static float *emb = nullptr;
        static size_t emb_cap = 0;
        const size_t need = (size_t)nb * 4 * k * nc * sizeof(float);
        if (need > emb_cap) {
            if (emb) PB_CUDA(cudaFree(emb));
            emb = nullptr;
            emb_cap = 0;
            PB_CUDA(cudaMalloc(&emb, need));
            emb_cap = need;
        }
        eng.emb = emb;
        eng.emb_cap = emb_cap;
    }
    int r = pb_cgemm_sub(&eng, m, nc, k, (const float2 *)a_dev, lda, (const float2 *)b_dev, ldb, (float2 *)c_dev,
                         ldc, stride, nb);
    if (r == PB_OK && eng.tc_used && eng.tc_err) {
        eng.tc_used = 0;
        int h = 0;
        PB_CUDA(cudaMemcpy(&h, eng.tc_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) {
            cudaMemset(eng.tc_err, 0, sizeof(int));
            pb_set_error("tensor-core update: a pipeline wait timed out");
            r = PB_ERR_CUDA;
        }
    }
    return r;
}

int pb_lu_decomp(int n, double *a, int *piv)
{
    if (n <= 0 || !a || !piv) { pb_set_error("pb_lu_decomp: bad argument"); return -2; }
    if (need_device() != PB_OK) return -2;
    double *d = nullptr;
    int *dp = nullptr, info = -1;
    if (cudaMalloc(&d, sizeof(double2) * (size_t)n * n) != cudaSuccess) { pb_set_error("cudaMalloc failed"); return -2; }
    if (cudaMalloc(&dp, sizeof(int) * n) != cudaSuccess) { cudaFree(d); pb_set_error("cudaMalloc failed"); return -2; }
    int r = PB_OK;
    if (cudaMemcpy(d, a, sizeof(double2) * (size_t)n * n, cudaMemcpyHostToDevice) != cudaSuccess) r = PB_ERR_CUDA;
    if (r == PB_OK) r = pb_lu_decomp_batched_dev(n, 1, d, dp, &info);
    if (r == PB_OK && cudaMemcpy(a, d, sizeof(double2) * (size_t)n * n, cudaMemcpyDeviceToHost) != cudaSuccess) r = PB_ERR_CUDA;
    if (r == PB_OK && cudaMemcpy(piv, dp, sizeof(int) * n, cudaMemcpyDeviceToHost) != cudaSuccess) r = PB_ERR_CUDA;
    cudaFree(d);
    cudaFree(dp);
    if (r != PB_OK) return -2;
    return info;          // -1 = regular, else first zero-pivot row (lu.c:15-30)
}

int pb_lu_solve(int n, const double *a, const int *piv, double *b)
{
    if (n <= 0 || !a || !piv || !b) { pb_set_error("pb_lu_solve: bad argument"); return PB_ERR_ARG; }
    PB_TRY(need_device());
    pb_lu_engine e;
    PB_TRY(pb_lu_engine_init(&e, nullptr));
    double2 *d = nullptr, *bv = nullptr;
    int *dp = nullptr, *perm = nullptr;
    int r = PB_OK;
    if (cudaMalloc(&d, sizeof(double2) * (size_t)n * n) != cudaSuccess || cudaMalloc(&bv, sizeof(double2) * n) != cudaSuccess ||
        cudaMalloc(&dp, sizeof(int) * n) != cudaSuccess || cudaMalloc(&perm, sizeof(int) * n) != cudaSuccess) {
        pb_set_error("cudaMalloc failed");
        r = PB_ERR_CUDA;
    }
    if (r == PB_OK && (cudaMemcpy(d, a, sizeof(double2) * (size_t)n * n, cudaMemcpyHostToDevice) != cudaSuccess ||
                       cudaMemcpy(bv, b, sizeof(double2) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
                       cudaMemcpy(dp, piv, sizeof(int) * n, cudaMemcpyHostToDevice) != cudaSuccess)) {
        pb_set_error("cudaMemcpy failed");
        r = PB_ERR_CUDA;
    }
    if (r == PB_OK) r = pb_lu_perm(&e, n, 1, dp, perm);
    if (r == PB_OK) r = pb_lu_solve_batched<double>(&e, n, 1, 1, d, n, (long)n * n, perm, bv, bv);
    if (r == PB_OK && cudaMemcpy(b, bv, sizeof(double2) * n, cudaMemcpyDeviceToHost) != cudaSuccess) { pb_set_error("cudaMemcpy failed"); r = PB_ERR_CUDA; }
    cudaFree(d); cudaFree(bv); cudaFree(dp); cudaFree(perm);
    pb_lu_engine_free(&e);
    return r;
}

}  // extern "C"

// ---------------------------------------------------------------- FP32 SIMT peak
// Dependent FMA chains, 8 independent per thread, enough warps to fill every SM: the
// measured FP32 FMA throughput of this GPU, the denominator of the fill roofline.
__global__ void __launch_bounds__(256) k_fma_peak(float *out, int iters, float a, float b)
{
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = threadIdx.x * 1e-3f + k;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = fmaf(x[k], a, b);
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == 12345.f) out[0] = s;                 // keeps the chains live
}

extern "C" int pb_fp32_peak(double *tflops)
{
    if (!tflops) return PB_ERR_ARG;
    PB_TRY(need_device());
    int dev = 0, nsm = 0;
    PB_CUDA(cudaGetDevice(&dev));
    PB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    float *out = nullptr;
    PB_CUDA(cudaMalloc(&out, sizeof(float)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = nsm * 8, iters = 1 << 16;
    k_fma_peak<<<blocks, 256>>>(out, 1024, 0.999f, 1e-3f);           // warm-up
    cudaEventRecord(e0);
    k_fma_peak<<<blocks, 256>>>(out, iters, 0.999f, 1e-3f);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return pb_cuda_fail(e, "k_fma_peak", __FILE__, __LINE__);
    *tflops = 2.0 * 8.0 * iters * (double)blocks * 256 / (ms * 1e-3) / 1e12;
    return PB_OK;
}

extern "C" int pb_device_sync(void)
{
    PB_CUDA(cudaDeviceSynchronize());
    return PB_OK;
}
