// pb_sweep.cu — the frequency sweep (reference solve(), src/solve.c:171-430, dense path)
// executed as batches of frequencies on the device.
//
// Two equivalent MNA formulations are built directly by the fill epilogues:
//  * reduced (default when every matrix node is a charge cell and there are no lumped
//    node elements): the node block j w C = j w P^-1 is eliminated exactly, leaving the
//    branch-current system  (j w Zb + G^T P G) ib = G^T P b  of order nseg, with
//    Zb = diag(zint) + j w Lp, G the node/segment incidence (mna.c:244-251). Node
//    voltages follow from v = P (b - G ib) / (j w). No inverse of P is formed.
//  * full: the reference's unknown vector [nodes | L | V | segments] (mna.c:81-84)
//    augmented with cell charges q (P q - v = 0, KCL + j w q), which is algebraically
//    identical to stamping j w P^-1 (mna.c:286-295) and is the reference's own compressed
//    formulation (mna.c:86-107, 271-284).
// Dense solve: batched LU of the whole batch; FP64 LU (plain path) or FP32 LU with
// tensor-core trailing updates + FP64 iterative refinement against the FP64 matrix.
#include "pb_ctx.cuh"
#include "pb_gmres.cuh"
#include "pb_hmat.cuh"
#include <algorithm>
#include <cmath>
#include <vector>

// ---------------------------------------------------------------- small kernels
// rhs'[f][j][k] = (P b_j)[ca_k] - (P b_j)[cb_k],  b_j = e(pc1_j) - e(pc2_j)   (cells)
__global__ void k_rhs_reduced(int nb, int np, int n, int nc, const double2 *P, long long pst,
                              const int *ca, const int *cb, const int *pc, double2 *rhs)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)nb * np * n) return;
    const int k = (int)(idx % n);
    const int j = (int)((idx / n) % np);
    const int f = (int)(idx / ((long long)n * np));
    const double2 *Pf = P + f * pst;
    const int c1 = pc[2 * j], c2 = pc[2 * j + 1];
    auto pb = [&](int c) -> double2 {
        double2 v = make_double2(0, 0);
        if (c < 0) return v;
        if (c1 >= 0) { const double2 p = Pf[(long long)c * nc + c1]; v.x += p.x; v.y += p.y; }
        if (c2 >= 0) { const double2 p = Pf[(long long)c * nc + c2]; v.x -= p.x; v.y -= p.y; }
        return v;
    };
    const double2 a = pb(ca[k]), b = pb(cb[k]);
    rhs[idx] = make_double2(a.x - b.x, a.y - b.y);
}

// Z[f][i][j] = (1/jw) sum_c (P[pc1_i][c] - P[pc2_i][c]) * (b_j - G ib_j)[c]: the voltage of
// port i for excitation j, which injects +1 A / -1 A at cells pcx[2j] / pcx[2j+1] (-1 = none).
__global__ void __launch_bounds__(256)
k_z_reduced(int np, int nx, int n, int nc, const double2 *P, long long pst, const int *inc_off,
            const int *inc_seg, const int *pc, const int *pcx, const double2 *x, const double *freq,
            double2 *z)
{
    const int f = blockIdx.z, i = blockIdx.y, j = blockIdx.x;
    const double2 *Pf = P + f * pst;
    const double2 *ib = x + ((long long)f * nx + j) * n;
    const int a1 = pc[2 * i], a2 = pc[2 * i + 1], b1 = pcx[2 * j], b2 = pcx[2 * j + 1];
    double sr = 0, si = 0;
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
        double yr = (c == b1 ? 1.0 : 0.0) - (c == b2 ? 1.0 : 0.0), yi = 0;
        for (int e = inc_off[c]; e < inc_off[c + 1]; e++) {
            const int s = inc_seg[e];
            const int k = (s > 0 ? s : -s) - 1;
            const double sg = s > 0 ? 1.0 : -1.0;
            yr -= sg * ib[k].x;
            yi -= sg * ib[k].y;
        }
        double wr = 0, wi = 0;
        if (a1 >= 0) { const double2 p = Pf[(long long)a1 * nc + c]; wr += p.x; wi += p.y; }
        if (a2 >= 0) { const double2 p = Pf[(long long)a2 * nc + c]; wr -= p.x; wi -= p.y; }
        sr += wr * yr - wi * yi;
        si += wr * yi + wi * yr;
    }
    __shared__ double rs[256], is_[256];
    rs[threadIdx.x] = sr;
    is_[threadIdx.x] = si;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) { rs[threadIdx.x] += rs[threadIdx.x + o]; is_[threadIdx.x] += is_[threadIdx.x + o]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double om = 2 * PB_PI * freq[f];
        // (sr + j si) / (j om) = (si - j sr) / om
        z[((long long)f * np + i) * nx + j] = make_double2(is_[0] / om, -rs[0] / om);
    }
}

// Plane-wave excitation (mna_rhs_planewave, src/mna.c:434-468).
struct PwArgs {
    double rh[3];        // arrival direction
    double ev[3];        // polarisation unit vector
    double2 e0;          // amplitude x e^{j phase}
};

__device__ __forceinline__ double pw_sinc(double x) { return fabs(x) < 1e-8 ? 1.0 : sin(x) / x; }

// EMF integral(E . dl) of one wave over a straight cell (pw_emf, src/mna.c:408-432):
// (E0 e.t) len e^{j k r.rc} sinc(k len (r.t)/2), times the width average for ribbons / bars.
__device__ double2 pw_emf(const pb_cell_t &s, const double *rh, const double *ev, double2 e0, double kw)
{
    double tv[3], rc[3];
    for (int q = 0; q < 3; q++) {
        tv[q] = (s.x2[q] - s.x1[q]) / s.len;
        rc[q] = 0.5 * (s.x1[q] + s.x2[q]);
    }
    const double et = ev[0] * tv[0] + ev[1] * tv[1] + ev[2] * tv[2];
    const double rt = rh[0] * tv[0] + rh[1] * tv[1] + rh[2] * tv[2];
    const double rr = rh[0] * rc[0] + rh[1] * rc[1] + rh[2] * rc[2];
    double amp = et * s.len * pw_sinc(0.5 * kw * s.len * rt);
    const double wl = sqrt(s.wv[0] * s.wv[0] + s.wv[1] * s.wv[1] + s.wv[2] * s.wv[2]);
    if (s.wid > 0 && wl > 0) {
        const double rw = (rh[0] * s.wv[0] + rh[1] * s.wv[1] + rh[2] * s.wv[2]) / wl;
        amp *= pw_sinc(0.5 * kw * s.wid * rw);
    }
    double sn, cs;
    sincos(kw * rr, &sn, &cs);
    return make_double2(amp * (e0.x * cs - e0.y * sn), amp * (e0.x * sn + e0.y * cs));
}

// Right-hand side of the plane-wave excitation. Full form: -EMF on the branch rows
// offS + k (mna.c:464). Reduced form: the branch equation Zb i = G^T v + EMF times jw,
// with no node injection: rhs = jw EMF.
__global__ void k_rhs_planewave(int nb, int n, int ns, int reduced, int offS, const pb_cell_t *seg,
                                const double *freq, int gp, double gpz, PwArgs a, double2 *rhs)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)nb * n) return;
    const int f = (int)(idx / n), r = (int)(idx % n);
    const int k = reduced ? r : r - offS;
    double2 v = make_double2(0, 0);
    if (k >= 0 && k < ns) {
        const double om = 2 * PB_PI * freq[f];
        const double kw = om / PB_C0;
        double2 emf = pw_emf(seg[k], a.rh, a.ev, a.e0, kw);
        if (gp) {       // PEC reflection: mirrored arrival, horizontal polarisation flipped
            const double rh2[3] = {a.rh[0], a.rh[1], -a.rh[2]};
            const double ev2[3] = {-a.ev[0], -a.ev[1], a.ev[2]};
            double sn, cs;
            sincos(2 * kw * a.rh[2] * gpz, &sn, &cs);
            const double2 e0r = make_double2(a.e0.x * cs - a.e0.y * sn, a.e0.x * sn + a.e0.y * cs);
            const double2 r2 = pw_emf(seg[k], rh2, ev2, e0r, kw);
            emf.x += r2.x;
            emf.y += r2.y;
        }
        v = reduced ? make_double2(-om * emf.y, om * emf.x) : make_double2(-emf.x, -emf.y);
    }
    rhs[idx] = v;
}

// Arrival direction, polarisation and complex amplitude of the wave (mna.c:441-452).
static int make_pw_args(const pb_planewave_t *pw, PwArgs &a)
{
    if (pw->pol != 1 && pw->pol != 2) { pb_set_error("pb_planewave: polarisation must be 1 or 2"); return PB_ERR_ARG; }
    const double th = pw->theta_deg * PB_PI / 180, ph = pw->phi_deg * PB_PI / 180;
    const double sth = sin(th), cth = cos(th), cph = cos(ph), sph = sin(ph);
    const double rh[3] = {sth * cph, sth * sph, cth};
    const double thh[3] = {cth * cph, cth * sph, -sth};
    const double phh[3] = {-sph, cph, 0};
    for (int q = 0; q < 3; q++) {
        a.rh[q] = rh[q];
        a.ev[q] = (pw->pol == 2) ? phh[q] : thh[q];
    }
    const double pr = pw->phase_deg * PB_PI / 180;
    a.e0 = make_double2(pw->amp * cos(pr), pw->amp * sin(pr));
    return PB_OK;
}

int pb_pw_rhs_full(const pb_ctx *c, const pb_planewave_t *pw, const double *freq_dev, int n, int offS,
                   double2 *rhs, cudaStream_t st)
{
    PwArgs a;
    PB_TRY(make_pw_args(pw, a));
    k_rhs_planewave<<<ceil_div(n, 256), 256, 0, st>>>(1, n, (int)c->seg.size(), 0, offS, c->g.seg.cell, freq_dev,
                                                      c->gp, c->gpz, a, rhs);
    PB_CHECK_LAUNCH();
    return PB_OK;
}

__global__ void k_rhs_full(int nb, int np, int n, const int *pm, double2 *rhs)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)nb * np * n) return;
    const int k = (int)(idx % n);
    const int j = (int)((idx / n) % np);
    double v = 0;
    if (pm[2 * j] == k) v += 1;        // mna.c:367-376
    if (pm[2 * j + 1] == k) v -= 1;
    rhs[idx] = make_double2(v, 0);
}

// one frequency-independent right-hand side for every system of the batch
__global__ void k_rhs_copy(int nb, int n, const double2 *b, double2 *rhs)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx < (long long)nb * n) rhs[idx] = b[idx % n];
}

__global__ void k_z_full(int nb, int np, int nx, int n, const int *pm, const double2 *x, double2 *z)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nb * np * nx) return;
    const int j = idx % nx, i = (idx / nx) % np, f = idx / (np * nx);
    const double2 *xv = x + ((long long)f * nx + j) * n;
    const int a = pm[2 * i], b = pm[2 * i + 1];
    double2 v = make_double2(0, 0);
    if (a >= 0) { v.x += xv[a].x; v.y += xv[a].y; }
    if (b >= 0) { v.x -= xv[b].x; v.y -= xv[b].y; }
    z[idx] = v;
}

// Cell charges of the port excitations (solve.c:344-361), q[f][j][c] (QIDX layout).
// Reduced form: KCL at cell c, j w q_c = b_j[c] - (G ib_j)[c] (the quantity k_z_reduced
// multiplies by P). Full form: the charge unknowns x[offQ + c] themselves.
__global__ void k_cellq(int nb, int np, int n, int nc, int reduced, int offQ, const int *inc_off,
                        const int *inc_seg, const int *pc, const double2 *x, const double *freq, double2 *q)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)nb * np * nc) return;
    const int c = (int)(idx % nc);
    const int j = (int)((idx / nc) % np);
    const int f = (int)(idx / ((long long)nc * np));
    const double2 *xv = x + ((long long)f * np + j) * n;
    if (!reduced) {
        q[idx] = xv[offQ + c];
        return;
    }
    double yr = (c == pc[2 * j] ? 1.0 : 0.0) - (c == pc[2 * j + 1] ? 1.0 : 0.0), yi = 0;
    for (int e = inc_off[c]; e < inc_off[c + 1]; e++) {
        const int s = inc_seg[e];
        const int k = (s > 0 ? s : -s) - 1;
        const double sg = s > 0 ? 1.0 : -1.0;
        yr -= sg * xv[k].x;
        yi -= sg * xv[k].y;
    }
    const double om = 2 * PB_PI * freq[f];
    q[idx] = make_double2(yi / om, -yr / om);
}

// Conditioning probe of the refined solutions: the right-hand side of a perturbation of the
// size of the remaining componentwise backward error, db_r = eta_q (|A||x| + |b|)_r with a
// fixed pseudo-random phase of +-1 +- j per row (per = vectors x rows of one system).
__global__ void k_probe_rhs(long long per, const int *sys, const double *w, const double *eta, double2 *out)
{
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= per) return;
    const long long q = sys[blockIdx.y];
    unsigned h = (unsigned)e * 2654435761u;          // integer hash of the row index
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    const double a = eta[q] * w[q * per + e] * 0.7071067811865476;
    out[q * per + e] = make_double2((h & 1u) ? a : -a, (h & 2u) ? a : -a);
}

// full form: blocks of the augmented matrix (Lp block with -zint, P block)
__global__ void k_full_blocks(int nb, int n, int ns, int nc, int offS, int offQ,
                              const double2 *lp, long long lst, const double2 *P, long long pst,
                              const double2 *zint, const double *freq, double2 *m, long long mst)
{
    const long long per = (long long)ns * ns + (long long)nc * nc;
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= per * nb) return;
    const int f = (int)(idx / per);
    long long e = idx - f * per;
    double2 *M = m + f * mst;
    const double om = 2 * PB_PI * freq[f];
    if (e < (long long)ns * ns) {
        const int k = (int)(e / ns), q = (int)(e % ns);
        const double2 l = lp[f * lst + e];
        double2 v = make_double2(om * l.y, -om * l.x);   // -j w Lp (mna.c:263)
        if (k == q) { const double2 zz = zint[(long long)f * ns + k]; v.x -= zz.x; v.y -= zz.y; }
        M[(long long)(offS + k) * n + offS + q] = v;
    } else {
        e -= (long long)ns * ns;
        const int c = (int)(e / nc), d = (int)(e % nc);
        M[(long long)(offQ + c) * n + offQ + d] = P[f * pst + e];
    }
}

__global__ void k_full_stamps(int nb, int n, int ne, const int *row, const int *col, const int *off,
                              const pb_stamp *st, const double *freq, double2 *m, long long mst)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)ne * nb) return;
    const int f = (int)(idx / ne), e = (int)(idx % ne);
    const double om = 2 * PB_PI * freq[f];
    double vr = 0, vi = 0;
    for (int q = off[e]; q < off[e + 1]; q++) {
        const pb_stamp s = st[q];
        if (s.kind == ST_CONST) vr += s.val;
        else if (s.kind == ST_JW) vi += om * s.val;
        else vi -= om * s.val;
    }
    double2 *p = &m[f * mst + (long long)row[e] * n + col[e]];
    p->x += vr;
    p->y += vi;
}

__global__ void k_to_f32(const double2 *a, float2 *b, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        b[i] = make_float2((float)a[i].x, (float)a[i].y);
}

__global__ void k_axpy(double2 *x, const double2 *d, long long n)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) { x[i].x += d[i].x; x[i].y += d[i].y; }
}

// x += d for the systems sys[blockIdx.y] (m = entries per system)
__global__ void k_axpy_sys(double2 *x, const double2 *d, long long m, const int *sys)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= m) return;
    const long long o = (long long)sys[blockIdx.y] * m + i;
    x[o].x += d[o].x;
    x[o].y += d[o].y;
}

// ---------------------------------------------------------------- helpers
// Device buffer of one sweep call; with a context slot the storage stays with the context
// for the next call (grow-only).
struct DevBuf {
    void *p = nullptr;
    pb_cache_slot *slot = nullptr;
    DevBuf() = default;
    explicit DevBuf(pb_cache_slot *s) : slot(s) {}
    ~DevBuf() { if (p && !slot) cudaFree(p); }
    int alloc(size_t bytes)
    {
        if (bytes == 0) bytes = 16;
        if (slot) {
            if (slot->cap < bytes) {
                if (slot->p) cudaFree(slot->p);
                slot->p = nullptr;
                slot->cap = 0;
                cudaError_t e = cudaMalloc(&slot->p, bytes);
                if (e != cudaSuccess) { slot->p = nullptr; return pb_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__); }
                slot->cap = bytes;
            }
            p = slot->p;
            return PB_OK;
        }
        if (p) { cudaFree(p); p = nullptr; }
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) { p = nullptr; return pb_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__); }
        return PB_OK;
    }
    template <typename T> T *as() const { return (T *)p; }
};

// Quadrature-level signature of a wavenumber: floor(kw * size) over the distinct cell
// sizes that can be a pair's lmax (partial.c:166-173, 216-227). Equal signatures mean
// every pair uses the same nsub, hence the same static part.
thread_local int pb_mem_share = 1;

long far_rule_key(const pb_ctx *c, double kwmax)
{
    long n = 0;
    for (const auto *v : {&c->seg, &c->chg})
        for (const auto &s : *v) n += kwmax * std::max(s.len, s.wid) > PB_FAR_KL;
    return n;
}

void level_signature(const pb_ctx *c, double kw, std::vector<long> &sig)
{
    sig.clear();
    sig.push_back(kw > 0 ? 1 : 0);
    if (kw <= 0) return;
    auto add = [&](const std::vector<pb_cell_t> &v) {
        for (const auto &s : v) {
            sig.push_back((long)std::floor(kw * s.len));
            sig.push_back((long)std::floor(kw * std::max(s.len, s.wid)));
        }
    };
    add(c->seg);
    add(c->chg);
    std::sort(sig.begin() + 1, sig.end());
    sig.erase(std::unique(sig.begin() + 1, sig.end()), sig.end());
}

struct PhaseTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    double acc = 0;
    PhaseTimer() { cudaEventCreate(&a); cudaEventCreate(&b); }
    ~PhaseTimer() { cudaEventDestroy(a); cudaEventDestroy(b); }
    void start(cudaStream_t s) { cudaEventRecord(a, s); }
    void stop(cudaStream_t s)
    {
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        acc += ms;
    }
};

// Phase timer of the fill stream: event pairs recorded without waiting (the host must not
// block on the fill stream while the other stream's batch is being solved), summed once
// the sweep is done.
struct AsyncTimer {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    cudaEvent_t cur = nullptr;
    double acc = 0;
    void start(cudaStream_t s)
    {
        cudaEventCreate(&cur);
        cudaEventRecord(cur, s);
    }
    void stop(cudaStream_t s)
    {
        cudaEvent_t b = nullptr;
        cudaEventCreate(&b);
        cudaEventRecord(b, s);
        ev.push_back(std::make_pair(cur, b));
        cur = nullptr;
    }
    void finish()
    {
        for (auto &e : ev) {
            cudaEventSynchronize(e.second);
            float ms = 0;
            cudaEventElapsedTime(&ms, e.first, e.second);
            acc += ms;
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        ev.clear();
    }
    ~AsyncTimer()
    {
        for (auto &e : ev) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
        if (cur) cudaEventDestroy(cur);
    }
};

int pb_sweep_impl(pb_ctx *c, int nfreq, const double *freq, const pb_sweep_opts *opts_in,
                  double *zmat, double *segi, pb_sweep_stats *stats,
                  const pb_planewave_t *pw, double *voc, double *segipw,
                  const double *rhs_fixed, double *vnode, double *cellq)
{
    pb_sweep_opts o;
    if (opts_in) o = *opts_in;
    else {
        memset(&o, 0, sizeof(o));                  // every option off, pointers null
        o.fill_prec = PB_PREC_MIXED;
        o.lu = PB_LU_TC;
        o.form = PB_FORM_AUTO;
    }
    if (o.compress) {
        if (rhs_fixed) { pb_set_error("source excitation is not built for the compressed path"); return PB_ERR_UNSUP; }
        if (nfreq <= 0 || freq == nullptr) { pb_set_error("pb_sweep: no frequencies"); return PB_ERR_ARG; }
        if (pw) {
            PwArgs chk;
            PB_TRY(make_pw_args(pw, chk));
        }
        pb_hstats hs;
        return pb_sweep_compressed(c, nfreq, freq, o, o.ctol > 0 ? o.ctol : 1e-6,
                                   o.refine_tol > 0 ? o.refine_tol : 1e-10, pw ? nullptr : zmat, stats, &hs,
                                   nullptr, nullptr, pw, voc, segipw, pw ? nullptr : segi, pw ? nullptr : cellq);
    }
    if (nfreq <= 0 || freq == nullptr) { pb_set_error("pb_sweep: no frequencies"); return PB_ERR_ARG; }
    for (int i = 0; i < nfreq; i++)
        if (!(freq[i] > 0)) { pb_set_error("pb_sweep: frequencies must be > 0"); return PB_ERR_ARG; }
    int form = o.form;
    if (form == PB_FORM_AUTO) form = c->reduced_ok ? PB_FORM_REDUCED : PB_FORM_FULL;
    if (form == PB_FORM_REDUCED && !c->reduced_ok) {
        pb_set_error("reduced formulation needs every matrix node to be a charge cell and no lumped node elements");
        return PB_ERR_UNSUP;
    }
    const int mixed = (o.lu != PB_LU_FP64);
    const int fill32 = (o.fill_prec == PB_PREC_MIXED);
    const double tol = o.refine_tol > 0 ? o.refine_tol : 1e-12;
    const int maxit = o.refine_maxit > 0 ? o.refine_maxit : 30;
    c->lu.gemm_kind = (o.lu == PB_LU_TC || o.lu == PB_LU_TC_PIVOTED) ? PB_GEMM_TC
                    : (o.lu == PB_LU_TC_CUBLAS) ? PB_GEMM_TC_BLAS
                    : (o.lu == PB_LU_FP32) ? PB_GEMM_FP32 : PB_GEMM_FP64;
    const long launches0 = c->launches + c->lu.launches;

    const int ns = (int)c->seg.size(), nc = c->ncell, np = (int)c->port.size();
    if (rhs_fixed && form != PB_FORM_FULL) { pb_set_error("source excitation needs the full MNA form"); return PB_ERR_ARG; }
    const int nr = (pw || rhs_fixed) ? 1 : np;   // right-hand sides per frequency
    const int n = (form == PB_FORM_REDUCED) ? ns : c->nfull;
    const cudaStream_t st = c->stream;
    if (n <= 0) { pb_set_error("pb_sweep: empty system"); return PB_ERR_ARG; }
    // FP32 factorisation of the mixed path: the reduced system is complex symmetric, so
    // PB_LU_TC factors it as L D L^T without pivoting (half the flops, no swaps; refinement
    // against the FP64 matrix and the FP64 fall back cover the missing pivoting); every
    // other case takes the pivoted LU
    const bool sym32 = (form == PB_FORM_REDUCED && o.lu == PB_LU_TC);
    auto factor32 = [&](int nm, float2 *a32, long long strd, int *piv, int *info) -> int {
        if (sym32) {
            const int r = pb_ldl_factor(&c->lu, n, nm, a32, n, strd, piv, info);
            if (r != PB_ERR_UNSUP) return r;
        }
        return pb_lu_factor<float>(&c->lu, n, nm, a32, n, strd, piv, info);
    };
    auto flops32 = [&](int nm) { return (sym32 ? 4.0 : 8.0) / 3.0 * (double)n * n * n * nm; };
    // symmetric storage: with one right-hand side and no LU reuse the fill writes only the
    // lower triangle of the FP64 and FP32 systems, the refinement residual reads only that
    // (pb_sym_residual_mapped), and the few FP64 factorisations mirror it first
    const bool lower = sym32 && pb_ldl_supported(n) && !rhs_fixed && o.accel < 2 && (pw || np == 1);
    // and the unpivoted factorisation runs on a static symmetric ordering of each system
    // (decreasing diagonal dominance, pb_sym_order), formed from the FP64 lower triangle
    const bool reorder = lower && n <= 16384;

    // batch size from free memory
    size_t fr = 0, tot = 0;
    PB_CUDA(cudaMemGetInfo(&fr, &tot));
    const double n2 = (double)n * n;
    const int tc = (o.lu == PB_LU_TC_CUBLAS);     // the library comparison needs the embedding scratch
    // per frequency: the filled systems (one set per batch in flight) and the solve's storage
    const double perf_set = n2 * 16 + (mixed ? n2 * 8 : 0) + (double)nc * nc * 16 + (double)ns * 16 + 8.0
                          + (form == PB_FORM_FULL ? (double)ns * ns * 16 : 0);
    const double perf_solve = (tc ? n2 * 4 : 0) + 4.0 * nr * n * 16 + 8.0 * n;
    const double fixed = (double)ns * ns * 8 + (double)nc * nc * 8 +
                         (c->retardation ? (double)PB_FMAX * c->chg.size() * c->chg.size() * 16 : 0.0);
    double cached = 0;                           // storage this context already holds
    for (int q = 0; q < PB_SLOT_COMP0; q++) cached += (double)c->cache[q].cap;
    // concurrent instances (pb_sweep_many) share the free memory
    const double avail = 0.80 * ((double)fr + cached) / pb_mem_share - fixed - 256e6;
    int B = o.batch;
    if (B <= 0) {
        B = (int)std::max(1.0, std::floor(avail / (perf_set + perf_solve)));
        B = std::min(B, 256);
    }
    B = std::max(1, std::min(B, nfreq));
    // Pipelined batches: with more than one batch, the next batch is filled (on the context's
    // low-priority fill stream) while the current one is factorised and refined, which needs
    // a second set of filled systems. Taken when both sets fit with batches of >= 32
    // frequencies (smaller batches lose more in the batched kernels than the overlap gains).
    bool pipe = false;
    if (nfreq > B && !rhs_fixed) {
        int Bp = o.batch > 0 ? B : (int)std::min(256.0, std::floor(avail / (2 * perf_set + perf_solve)));
        if ((o.batch > 0 || Bp >= 32) && (double)Bp * (2 * perf_set + perf_solve) <= avail) {
            pipe = true;
            B = std::max(1, std::min(Bp, nfreq));
        }
    }

    pb_cache_slot *cs = c->cache;
    DevBuf bM64a(cs + 0), bM32a(cs + 1), bPa(cs + 2), bLpa(cs + 3), bStLp(cs + 4), bStP(cs + 5), bZinta(cs + 6), bPiv(cs + 7), bPerm(cs + 8), bInfo(cs + 9), bRhs(cs + 10), bX(cs + 11), bR(cs + 12), bD(cs + 13), bRn(cs + 14), bBn(cs + 15), bFreqa(cs + 16), bZ(cs + 17), bPC(cs + 18);
    // the second set of filled systems (pipelined batches)
    DevBuf bM64b(cs + 31), bM32b(cs + 32), bPb(cs + 33), bLpb(cs + 34), bZintb(cs + 35), bFreqb(cs + 36);
    for (int set = 0; set < (pipe ? 2 : 1); set++) {
        DevBuf &m64 = set ? bM64b : bM64a, &m32 = set ? bM32b : bM32a, &pm = set ? bPb : bPa;
        DevBuf &lpb = set ? bLpb : bLpa, &zb = set ? bZintb : bZinta, &fq = set ? bFreqb : bFreqa;
        PB_TRY(m64.alloc((size_t)B * n2 * 16));
        // the FP32 factors; the FP64 fall-back later reuses this storage for up to B/2 FP64
        // matrices, so it holds at least one (B = 1)
        if (mixed) PB_TRY(m32.alloc((size_t)std::max(B, 2) * n2 * 8));
        PB_TRY(pm.alloc((size_t)B * nc * nc * 16 + 16));
        if (form == PB_FORM_FULL) PB_TRY(lpb.alloc((size_t)B * ns * ns * 16 + 16));
        PB_TRY(zb.alloc((size_t)B * ns * 16 + 16));
        PB_TRY(fq.alloc((size_t)B * 8));
    }
    // real-embedded right operands of the tensor-core trailing updates: the largest is
    // k x nc complex with k + nc = n, i.e. at most n^2/4 entries -> 4 * n^2/4 floats
    DevBuf bEmb(cs + 19);
    struct EmbGuard {
        pb_lu_engine *e;
        ~EmbGuard() { e->emb = nullptr; e->emb_cap = 0; }
    } emb_guard{&c->lu};
    if (tc) {
        PB_TRY(bEmb.alloc((size_t)B * n2 * 4));
        c->lu.emb = bEmb.as<float>();
        c->lu.emb_cap = (size_t)B * n2 * 4;
    }
    DevBuf bIg(cs + 20);                                  // sub-cell P corrections of one fill chunk
    if (c->capacitance && nc > 0 && c->retardation)
        PB_TRY(bIg.alloc((size_t)PB_FMAX * c->chg.size() * c->chg.size() * 16));
    PB_TRY(bStLp.alloc((size_t)ns * ns * 8 + 16));
    PB_TRY(bStP.alloc((size_t)nc * nc * 8 + 16));
    PB_TRY(bPiv.alloc((size_t)B * n * 4));
    PB_TRY(bPerm.alloc((size_t)B * n * 4));
    PB_TRY(bInfo.alloc((size_t)B * 4));
    const size_t vb = (size_t)B * nr * n * 16;
    PB_TRY(bRhs.alloc(vb));
    PB_TRY(bX.alloc(vb));
    PB_TRY(bR.alloc(vb));
    PB_TRY(bD.alloc(vb));
    DevBuf bXn(cs + 21), bAn(cs + 22);
    PB_TRY(bXn.alloc((size_t)B * nr * 8));
    PB_TRY(bAn.alloc((size_t)B * 8));
    PB_TRY(bRn.alloc((size_t)B * nr * 8));
    PB_TRY(bBn.alloc((size_t)B * nr * 8));
    DevBuf bCw(cs + 23);                          // componentwise backward errors (full form)
    PB_TRY(bCw.alloc((size_t)B * nr * 8));
    DevBuf bSys(cs + 24);                         // systems still refining
    PB_TRY(bSys.alloc((size_t)B * sizeof(int)));
    PB_TRY(bZ.alloc((size_t)B * np * nr * 16 + 16));
    PB_TRY(bPC.alloc((size_t)2 * (np + 1) * 4));
    DevBuf bW(cs + 26), bEta(cs + 27), bZp(cs + 28); // conditioning probe: row weights, eta, port voltages
    if (mixed && !rhs_fixed) {
        PB_TRY(bW.alloc((size_t)B * nr * n * 8));
        PB_TRY(bEta.alloc((size_t)B * 8));
        PB_TRY(bZp.alloc((size_t)2 * B * np * nr * 16 + 16));
    }
    DevBuf bSymScr(cs + 29), bOrd(cs + 30);       // partial sums of the symmetric residual; orderings
    if (lower) PB_TRY(bSymScr.alloc(pb_sym_residual_scratch(n, B)));
    if (reorder) PB_TRY(bOrd.alloc((size_t)B * n * sizeof(int)));
    DevBuf bQ(cs + 25);                           // cell charges of one batch (distribution)
    if (cellq && !pw && !rhs_fixed && c->capacitance && nc > 0) PB_TRY(bQ.alloc((size_t)B * np * nc * 16));

    // port endpoints: cells (reduced) or matrix indices (full)
    std::vector<int> pc(2 * np);
    for (int j = 0; j < np; j++) {
        if (form == PB_FORM_REDUCED) {
            const int m1 = c->nodemap[c->port[j].n1], m2 = c->nodemap[c->port[j].n2];
            pc[2 * j] = m1 >= 0 ? c->cell_of_node[c->port[j].n1] : -1;
            pc[2 * j + 1] = m2 >= 0 ? c->cell_of_node[c->port[j].n2] : -1;
        } else {
            pc[2 * j] = c->nodemap[c->port[j].n1];
            pc[2 * j + 1] = c->nodemap[c->port[j].n2];
        }
    }
    pc.push_back(-1);                            // plane wave: no current injection
    pc.push_back(-1);
    PB_CUDA(cudaMemcpyAsync(bPC.p, pc.data(), sizeof(int) * 2 * (np + 1), cudaMemcpyHostToDevice, st));
    DevBuf bFix;                                  // the source right-hand side (pb_sources)
    if (rhs_fixed) {
        PB_TRY(bFix.alloc(sizeof(double2) * (size_t)n));
        PB_CUDA(cudaMemcpyAsync(bFix.p, rhs_fixed, sizeof(double2) * (size_t)n, cudaMemcpyHostToDevice, st));
    }
    PwArgs pwa;
    if (pw) PB_TRY(make_pw_args(pw, pwa));

    PhaseTimer tLu, tRef, tAll;
    AsyncTimer tStatic, tCorr, tAsm;                // fill phases (possibly on the fill stream)
    double samples = 0, luflops = 0, maxres = 0, probe_max = 0;
    int maxits = 0, refreshes = 0, probe_fb = 0;
    // the static tables stay with the context between calls (cache slots 4 and 5): valid
    // while the quadrature-level signature is unchanged and the slots kept their storage
    std::vector<long> cur_sig, sig;
    bool static_valid = c->dense_static_valid && c->dense_static_ptr[0] == bStLp.p && c->dense_static_ptr[1] == bStP.p;
    if (static_valid) cur_sig = c->dense_sig;
    std::vector<double2> zh((size_t)B * np * np);
    std::vector<double> rnh(B * nr), bnh(B * nr), xnh(B * nr), anh(B);
    int fallbacks = 0, fp64_direct = 0, lu_count = 0, gm_solves = 0, gm_max = 0, refactored = 0;
    long gm_its = 0;
    double fp64_hz = 0;                          // frequencies <= this are solved in FP64
    double lp_samp = 0, p_samp = 0;
    std::vector<int> infoh(B);
    tAll.start(st);

    // Fill of one batch (frequencies fb0 .. fb0 + nb - 1) into buffer set `set` on stream fs:
    // internal impedances, the static tables when the quadrature levels change, the
    // correction kernels with the reduced-form epilogue, or the full-form assembly.
    auto fill_batch = [&](int fb0, int nb, int set, cudaStream_t fs) -> int {
        DevBuf &bM64 = set ? bM64b : bM64a, &bM32 = set ? bM32b : bM32a, &bP = set ? bPb : bPa;
        DevBuf &bLp = set ? bLpb : bLpa, &bZint = set ? bZintb : bZinta, &bFreq = set ? bFreqb : bFreqa;
        const double *fb = freq + fb0;
        PB_CUDA(cudaMemcpyAsync(bFreq.p, fb, sizeof(double) * nb, cudaMemcpyHostToDevice, fs));
        tAsm.start(fs);
        PB_TRY(pb_zint(c->g, c->skin, nb, bFreq.as<double>(), bZint.as<double2>(), fs, &c->launches));
        tAsm.stop(fs);
        // fill in chunks of <= 32 frequencies with one quadrature-level signature
        int f = 0;
        while (f < nb) {
            const double kw0 = c->retardation ? 2 * PB_PI * fb[f] / PB_C0 : 0.0;
            level_signature(c, kw0, sig);
            int e = f + 1;
            // plain path: one frequency at a time (static part re-evaluated each time)
            const int chunk_max = !fill32 ? 1 : (o.corr_freqs > 0 ? std::min(o.corr_freqs, PB_FMAX) : PB_FMAX);
            if (c->retardation) {
                std::vector<long> s2;
                while (e < nb && e - f < chunk_max) {
                    level_signature(c, 2 * PB_PI * fb[e] / PB_C0, s2);
                    if (s2 != sig) break;
                    e++;
                }
            } else {
                e = std::min(nb, f + chunk_max);
            }
            const int nf = e - f;
            // the static part depends on the frequency only through the quadrature levels:
            // both paths re-evaluate it when the level signature changes, and reuse it
            // (bit-identical) while it does not
            if (!static_valid || sig != cur_sig) {
                c->dense_static_valid = false;
                tStatic.start(fs);
                if (c->capacitance && nc > 0) PB_TRY(pb_pot_static(c->g, kw0, bStP.as<double>(), fs, &c->launches));
                PB_TRY(pb_lp_static(c->g, kw0, bStLp.as<double>(), fs, &c->launches));
                tStatic.stop(fs);
                cur_sig = sig;
                static_valid = true;
                c->dense_sig = sig;
                c->dense_static_valid = true;
                c->dense_static_ptr[0] = bStLp.p;
                c->dense_static_ptr[1] = bStP.p;
                refreshes++;
            }
            double kw[PB_FMAX], kwmax = 0;
            for (int q = 0; q < nf; q++) {
                kw[q] = c->retardation ? 2 * PB_PI * fb[f + q] / PB_C0 : 0.0;
                kwmax = std::max(kwmax, kw[q]);
            }
            if (kw0 > 0) {
                // exact quadrature-sample count of this chunk (statistics only): it depends on
                // the geometry, the level signature and, on the FP32 path (fewer samples for
                // separated ribbons), which cells the chunk's largest wavenumber admits to
                // the lower-order rules; the context keeps it per key
                std::vector<long> skey(sig);
                skey.push_back(fill32 ? far_rule_key(c, kwmax) : -1);
                auto it = c->sample_counts.find(skey);
                if (it == c->sample_counts.end()) {
                    PB_TRY(pb_count_samples(c->g, kw0, &lp_samp, &p_samp, fs, c->d_count, fill32 ? kwmax : 0.0));
                    c->sample_counts[skey] = std::make_pair(lp_samp, p_samp);
                } else {
                    lp_samp = it->second.first;
                    p_samp = it->second.second;
                }
            } else {
                lp_samp = p_samp = 0;
            }
            tCorr.start(fs);
            if (c->capacitance && nc > 0)
                PB_TRY(pb_pot_corr(c->g, nf, kw, fill32, bStP.as<double>(), bP.as<double2>() + (long long)f * nc * nc,
                                   (long long)nc * nc, bIg.as<double2>(), fs, &c->launches, &samples));
            pb_epi_args ea;
            for (int q = 0; q < nf; q++) ea.omega[q] = 2 * PB_PI * fb[f + q];
            if (form == PB_FORM_REDUCED) {
                ea.m64 = bM64.as<double2>() + (long long)f * n * n;
                ea.m32 = (mixed && !reorder) ? bM32.as<float2>() + (long long)f * n * n : nullptr;
                ea.m_stride = (long long)n * n;
                ea.pm = bP.as<double2>() + (long long)f * nc * nc;
                ea.pm_stride = (long long)nc * nc;
                ea.zint = bZint.as<double2>() + (long long)f * ns;
                ea.lower = lower ? 1 : 0;
                PB_TRY(pb_lp_corr(c->g, nf, kw, fill32, bStLp.as<double>(), PB_EPI_REDUCED, ea, fs,
                                  &c->launches, &samples));
            } else {
                ea.out = bLp.as<double2>() + (long long)f * ns * ns;
                ea.out_stride = (long long)ns * ns;
                PB_TRY(pb_lp_corr(c->g, nf, kw, fill32, bStLp.as<double>(), PB_EPI_STORE, ea, fs,
                                  &c->launches, &samples));
            }
            tCorr.stop(fs);
            samples += (lp_samp + (c->capacitance ? p_samp : 0)) * nf;
            f = e;
        }
        if (form == PB_FORM_FULL) {
            tAsm.start(fs);
            PB_CUDA(cudaMemsetAsync(bM64.p, 0, (size_t)nb * n2 * 16, fs));
            const int offQ = c->nunknown;
            const long long per = (long long)ns * ns + (c->capacitance ? (long long)nc * nc : 0);
            if (per > 0) k_full_blocks<<<ceil_div(per * nb, 256), 256, 0, fs>>>(
                nb, n, ns, c->capacitance ? nc : 0, c->offS, offQ, bLp.as<double2>(), (long long)ns * ns,
                bP.as<double2>(), (long long)nc * nc, bZint.as<double2>(), bFreq.as<double>(),
                bM64.as<double2>(), (long long)n * n);
            if (per > 0) c->launches++;
            PB_CHECK_LAUNCH();
            const int ne = (int)c->fe_row.size();
            if (ne > 0) {
                k_full_stamps<<<ceil_div((long long)ne * nb, 256), 256, 0, fs>>>(
                    nb, n, ne, c->d_fe_row, c->d_fe_col, c->d_fe_off, c->d_fe_st, bFreq.as<double>(),
                    bM64.as<double2>(), (long long)n * n);
                c->launches++;
                PB_CHECK_LAUNCH();
            }
            if (mixed) {
                k_to_f32<<<1184, 256, 0, fs>>>(bM64.as<double2>(), bM32.as<float2>(), (long long)nb * n * n);
                c->launches++;
                PB_CHECK_LAUNCH();
            }
            tAsm.stop(fs);
        }
        return PB_OK;
    };
    // Pipelined: the next batch's fill is queued on the fill stream before this batch is
    // solved on `st`, which waits for its own batch's fill event. Both streams only touch
    // their own buffer set; a set is refilled only after the batch that used it has been
    // solved (the solve ends with a host synchronisation of `st`).
    const cudaStream_t sf = pipe ? c->stream_fill : st;
    struct EvPair {
        cudaEvent_t e[2] = {nullptr, nullptr};
        ~EvPair() { for (auto x : e) if (x) cudaEventDestroy(x); }
    } evFill;
    if (pipe) {
        for (int q = 0; q < 2; q++) PB_CUDA(cudaEventCreateWithFlags(&evFill.e[q], cudaEventDisableTiming));
        PB_TRY(fill_batch(0, std::min(B, nfreq), 0, sf));
        PB_CUDA(cudaEventRecord(evFill.e[0], sf));
    }
    for (int b0 = 0, set = 0; b0 < nfreq; b0 += B, set ^= 1) {
        const int nb = std::min(B, nfreq - b0);
        const double *fb = freq + b0;
        if (pipe) {
            if (b0 + B < nfreq) {
                PB_TRY(fill_batch(b0 + B, std::min(B, nfreq - b0 - B), set ^ 1, sf));
                PB_CUDA(cudaEventRecord(evFill.e[set ^ 1], sf));
            }
            PB_CUDA(cudaStreamWaitEvent(st, evFill.e[set], 0));
        } else {
            PB_TRY(fill_batch(b0, nb, 0, st));
        }
        DevBuf &bM64 = set ? bM64b : bM64a, &bM32 = set ? bM32b : bM32a, &bP = set ? bPb : bPa;
        DevBuf &bFreq = set ? bFreqb : bFreqa;
        // Precision per frequency. Frequencies at or below fp64_hz (the highest frequency
        // whose mixed solve stalled earlier in this sweep) go straight to an FP64 LU; they
        // form a prefix of the ascending batch. The rest are factorised in FP32 and refined.
        int nd = 0;
        if (mixed) while (nd < nb && fb[nd] <= fp64_hz) nd++;
        else nd = nb;
        const long long nn = (long long)n * n;
        // LU reuse (accel >= 2): factor every S-th frequency of the mixed part (the anchors,
        // centred in their groups); the others are solved by GMRES preconditioned with the
        // nearest anchor's factors.
        const int mb = nb - nd;
        const int S = (mixed && o.accel >= 2 && mb >= 2) ? o.accel : 0;
        const int aoff = S ? std::min(S / 2, mb - 1) : 0;
        const int nanch = S ? (mb - 1 - aoff) / S + 1 : mb;
        std::vector<int> lu_of(std::max(mb, 1));
        for (int q = 0; q < mb; q++)
            lu_of[q] = S ? std::min(nanch - 1, std::max(0, (int)std::floor((q - aoff) / (double)S + 0.5))) : q;
        tLu.start(st);
        if (reorder && mb > 0)
            PB_TRY(pb_sym_order(&c->lu, n, mb, bM64.as<double2>() + nd * nn, nn, bM32.as<float2>() + nd * nn,
                                bOrd.as<int>() + (long long)nd * n, bSymScr.p));
        if (nd > 0 && lower) PB_TRY(pb_sym_mirror(&c->lu, n, nd, bM64.as<double2>(), nn));
        if (nd > 0) PB_TRY(pb_lu_factor<double>(&c->lu, n, nd, bM64.as<double2>(), n, nn, bPiv.as<int>(), bInfo.as<int>()));
        if (mb > 0)
            PB_TRY(factor32(nanch, bM32.as<float2>() + (nd + aoff) * nn, S ? S * nn : nn,
                            bPiv.as<int>() + (long long)nd * n, bInfo.as<int>() + nd));
        PB_TRY(pb_lu_perm(&c->lu, n, nd + (mb > 0 ? nanch : 0), bPiv.as<int>(), bPerm.as<int>()));
        if (reorder && mb > 0)
            PB_CUDA(cudaMemcpyAsync(bPerm.as<int>() + (long long)nd * n, bOrd.as<int>() + (long long)nd * n,
                                    sizeof(int) * (size_t)mb * n, cudaMemcpyDeviceToDevice, st));
        tLu.stop(st);
        luflops += 8.0 / 3.0 * (double)n * n * n * nd + (mb > 0 ? flops32(nanch) : 0.0);
        lu_count += nd + (mb > 0 ? nanch : 0);
        PB_CUDA(cudaMemcpyAsync(infoh.data(), bInfo.p, sizeof(int) * nb, cudaMemcpyDeviceToHost, st));
        PB_CUDA(cudaStreamSynchronize(st));
        for (int q = 0; q < nd; q++)
            if (infoh[q] >= 0) {
                pb_set_error("singular matrix at f = %.5e Hz (row %d : floating node or ideal voltage source loop?)",
                             fb[q], infoh[q]);
                return PB_ERR_SINGULAR;
            }
        // right-hand sides
        tRef.start(st);
        const long long nv = (long long)nb * nr * n;
        if (rhs_fixed) {
            k_rhs_copy<<<ceil_div(nv, 256), 256, 0, st>>>(nb, n, bFix.as<double2>(), bRhs.as<double2>());
        } else if (pw) {
            k_rhs_planewave<<<ceil_div(nv, 256), 256, 0, st>>>(nb, n, ns, form == PB_FORM_REDUCED, c->offS,
                                                               c->g.seg.cell, bFreq.as<double>(), c->gp, c->gpz,
                                                               pwa, bRhs.as<double2>());
        } else if (form == PB_FORM_REDUCED) {
            k_rhs_reduced<<<ceil_div(nv, 256), 256, 0, st>>>(nb, nr, n, nc, bP.as<double2>(), (long long)nc * nc,
                                                             c->g.seg_ca, c->g.seg_cb, bPC.as<int>(), bRhs.as<double2>());
        } else {
            k_rhs_full<<<ceil_div(nv, 256), 256, 0, st>>>(nb, nr, n, bPC.as<int>(), bRhs.as<double2>());
        }
        c->launches++;
        PB_CHECK_LAUNCH();
        if (nd > 0)
            PB_TRY(pb_lu_solve_batched<double>(&c->lu, n, nd, nr, bM64.as<double2>(), n, nn,
                                               bPerm.as<int>(), bRhs.as<double2>(), bX.as<double2>()));
        std::vector<int> state(nb, 1);            // 0 active, 1 converged / direct, 2 failed
        if (nb > nd && S) {
            // GMRES with the anchors' FP32 factors (anchors themselves converge in a few
            // steps, like the refinement below)
            const long long vo = (long long)nd * nr * n;
            std::vector<int> gst(mb, 0);
            for (int q = 0; q < mb; q++)
                if (infoh[nd + lu_of[q]] >= 0) gst[q] = 2;            // zero FP32 pivot: go FP64
            pb_gmres_args ga;
            ga.eng = &c->lu;
            ga.n = n;
            ga.nsys = mb;
            ga.nrhs = nr;
            ga.A = bM64.as<double2>() + nd * nn;
            ga.A_stride = nn;
            ga.lu = bM32.as<float2>() + (nd + aoff) * nn;
            ga.lu_stride = S * nn;
            ga.perm = bPerm.as<int>() + (long long)nd * n;
            ga.lu_of = lu_of.data();
            ga.b = bRhs.as<double2>() + vo;
            ga.x = bX.as<double2>() + vo;
            ga.eta = std::max(1e-14, 8.0 * std::sqrt((double)n) * 1.1e-16);
            ga.m = PB_GMRES_MAXM;
            ga.max_cycles = 2;
            pb_gmres_result gr;
            PB_TRY(pb_gmres_batched(ga, gst, &gr));
            gm_solves += gr.solved;
            gm_its += gr.iters_total;
            gm_max = std::max(gm_max, gr.iters_max);
            maxits = std::max(maxits, gr.iters_max);
            // Systems the stale factors could not bring to the target are refactorised at
            // their own frequency (accel_rhs, solve.c:52-60), in FP32, and solved again. Their
            // FP32 copies are intact (only the anchors were factorised in place); they are
            // compacted to the front of the FP32 storage, whose anchor factors are no longer
            // needed, and factorised together.
            std::vector<int> redo;
            for (int q = 0; q < mb; q++)
                if (gst[q] == 2 && infoh[nd + lu_of[q]] < 0) redo.push_back(q);
            if (!redo.empty()) {
                const int nr = (int)redo.size();
                float2 *m32 = bM32.as<float2>() + nd * nn;
                for (int t = 0; t < nr; t++)
                    if (redo[t] != t)
                        PB_CUDA(cudaMemcpyAsync(m32 + t * nn, m32 + redo[t] * nn, sizeof(float2) * nn,
                                                cudaMemcpyDeviceToDevice, st));
                tLu.start(st);
                PB_TRY(factor32(nr, m32, nn, bPiv.as<int>() + (long long)nd * n, bInfo.as<int>() + nd));
                PB_TRY(pb_lu_perm(&c->lu, n, nr, bPiv.as<int>() + (long long)nd * n, bPerm.as<int>() + (long long)nd * n));
                tLu.stop(st);
                luflops += flops32(nr);
                lu_count += nr;
                std::vector<int> rinfo(nr);
                PB_CUDA(cudaMemcpyAsync(rinfo.data(), bInfo.as<int>() + nd, sizeof(int) * nr, cudaMemcpyDeviceToHost, st));
                PB_CUDA(cudaStreamSynchronize(st));
                std::vector<int> gst2(mb, 1);
                for (int t = 0; t < nr; t++) {
                    lu_of[redo[t]] = t;
                    gst2[redo[t]] = rinfo[t] >= 0 ? 2 : 0;
                }
                ga.lu = m32;
                ga.lu_stride = nn;
                PB_TRY(pb_gmres_batched(ga, gst2, &gr));
                for (int q = 0; q < mb; q++) if (gst[q] == 2) gst[q] = gst2[q];
                gm_its += gr.iters_total;
                gm_max = std::max(gm_max, gr.iters_max);
                refactored += nr;
            }
            for (int q = 0; q < mb; q++) state[nd + q] = gst[q];
        } else if (nb > nd) {
            // Iterative refinement in FP64 against the FP64 matrix:
            //   x_0 = LU^-1 b,  r = b - A x,  x += LU^-1 r,
            // until the normwise backward error eta = |r| / (|A| |x| + |b|) (infinity norms)
            // reaches the level of an FP64 factorisation. The full form mixes rows of very
            // different scale (charge rows with P ~ 1e10, KCL rows with entries 1), where a
            // small normwise error leaves the small rows inaccurate: there the componentwise
            // error max_i |r_i| / (|A||x| + |b|)_i must reach that level too. A frequency
            // whose iteration stalls above it is re-solved with an FP64 LU
            // (stats->fp64_fallbacks).
            const int mb = nb - nd;
            const long long vo = (long long)nd * nr * n;
            double2 *m64 = bM64.as<double2>() + nd * nn;
            float2 *m32 = bM32.as<float2>() + nd * nn;
            int *perm = bPerm.as<int>() + (long long)nd * n;
            for (int q = 0; q < mb; q++)
                if (infoh[nd + q] >= 0) state[nd + q] = 2;          // zero FP32 pivot: go FP64
            PB_TRY(pb_lu_solve_batched<float>(&c->lu, n, mb, nr, m32, n, nn, perm, bRhs.as<double2>() + vo,
                                              bX.as<double2>() + vo, reorder ? 1 : 0));
            const double eta_tol = std::max(1e-14, 8.0 * std::sqrt((double)n) * 1.1e-16);
            const bool cwise = (form == PB_FORM_FULL);
            const bool probe = !rhs_fixed;
            std::vector<double> prev(nb, 1e300), cwh((size_t)mb * nr, 0.0), etah(mb, 0.0);
            for (int q = nd; q < nb; q++) if (state[q] == 1) state[q] = 0;
            // only the systems still refining are touched after the first pass (the
            // stragglers near the FP64 fallback take up to a dozen steps, most need 2-3)
            std::vector<int> act;
            int it = 0;
            for (it = 1; it <= maxit + 1; it++) {
                act.clear();
                for (int q = 0; q < mb; q++) if (state[nd + q] == 0) act.push_back(q);
                if (act.empty()) break;
                PB_CUDA(cudaMemcpyAsync(bSys.p, act.data(), sizeof(int) * act.size(), cudaMemcpyHostToDevice, st));
                if (lower)
                    PB_TRY(pb_sym_residual_mapped(&c->lu, n, (int)act.size(), m64, nn, bRhs.as<double2>() + vo,
                                                  bX.as<double2>() + vo, bR.as<double2>() + vo, bRn.as<double>(),
                                                  bBn.as<double>(), bXn.as<double>(),
                                                  it == 1 ? bAn.as<double>() : nullptr, mb, bSys.as<int>(),
                                                  probe ? bW.as<double>() : nullptr, bSymScr.p));
                else
                    PB_TRY(pb_residual_mapped(&c->lu, n, (int)act.size(), nr, m64, n, nn, bRhs.as<double2>() + vo,
                                              bX.as<double2>() + vo, bR.as<double2>() + vo, bRn.as<double>(),
                                              bBn.as<double>(), bXn.as<double>(), it == 1 ? bAn.as<double>() : nullptr,
                                              mb, bSys.as<int>(), cwise ? bCw.as<double>() : nullptr,
                                              probe ? bW.as<double>() : nullptr));
                PB_CUDA(cudaMemcpyAsync(rnh.data(), bRn.p, sizeof(double) * mb * nr, cudaMemcpyDeviceToHost, st));
                PB_CUDA(cudaMemcpyAsync(bnh.data(), bBn.p, sizeof(double) * mb * nr, cudaMemcpyDeviceToHost, st));
                PB_CUDA(cudaMemcpyAsync(xnh.data(), bXn.p, sizeof(double) * mb * nr, cudaMemcpyDeviceToHost, st));
                if (it == 1) PB_CUDA(cudaMemcpyAsync(anh.data(), bAn.p, sizeof(double) * mb, cudaMemcpyDeviceToHost, st));
                if (cwise) PB_CUDA(cudaMemcpyAsync(cwh.data(), bCw.p, sizeof(double) * mb * nr, cudaMemcpyDeviceToHost, st));
                PB_CUDA(cudaStreamSynchronize(st));
                int active = 0;
                for (int q = 0; q < mb; q++) {
                    if (state[nd + q] != 0) continue;
                    double eta = 0;
                    for (int j = 0; j < nr; j++) {
                        const int v = q * nr + j;
                        const double den = anh[q] * xnh[v] + bnh[v];
                        eta = std::max(eta, den > 0 ? rnh[v] / den : 0.0);
                        if (cwise) eta = std::max(eta, cwh[v]);
                    }
                    if (eta <= eta_tol) { state[nd + q] = 1; maxres = std::max(maxres, eta); etah[q] = eta; }
                    else if (eta > 0.5 * prev[nd + q] || it > maxit) state[nd + q] = 2;
                    else { prev[nd + q] = eta; active++; }
                }
                if (active == 0) break;
                act.clear();
                for (int q = 0; q < mb; q++) if (state[nd + q] == 0) act.push_back(q);
                PB_CUDA(cudaMemcpyAsync(bSys.p, act.data(), sizeof(int) * act.size(), cudaMemcpyHostToDevice, st));
                PB_TRY(pb_lu_solve_mapped<float>(&c->lu, n, (int)act.size(), nr, m32, n, nn, perm,
                                                 bR.as<double2>() + vo, bD.as<double2>() + vo, bSys.as<int>(), nullptr,
                                                 reorder ? 1 : 0));
                const long long mv = (long long)nr * n;
                k_axpy_sys<<<dim3(ceil_div(mv, 256), (unsigned)act.size()), 256, 0, st>>>(
                    bX.as<double2>() + vo, bD.as<double2>() + vo, mv, bSys.as<int>());
                c->launches++;
                PB_CHECK_LAUNCH();
            }
            maxits = std::max(maxits, it);
            // Conditioning probe. A backward error at FP64 level does not bound the forward
            // error of an ill-conditioned system (e.g. an inductive structure whose port
            // resistance is 1e-5 of |Z| behind 1e-9 ohm bus resistors: cond ~ 1e13), and
            // there only the reference's own elimination order reproduces its digits. Each
            // converged system is perturbed by its remaining backward error (k_probe_rhs,
            // solved with its FP32 factors); where the port voltages move by more than a
            // quarter of the 1e-6 parity bar relative to the largest, the frequency takes
            // the FP64 fall back (stats->probe_fallbacks).
            std::vector<int> conv;
            for (int q = 0; q < mb; q++) if (state[nd + q] == 1) conv.push_back(q);
            if (probe && !conv.empty()) {
                for (int q = 0; q < mb; q++) etah[q] = std::max(etah[q], 4.0 * 1.1e-16);
                PB_CUDA(cudaMemcpyAsync(bEta.p, etah.data(), sizeof(double) * mb, cudaMemcpyHostToDevice, st));
                PB_CUDA(cudaMemcpyAsync(bSys.p, conv.data(), sizeof(int) * conv.size(), cudaMemcpyHostToDevice, st));
                const long long per = (long long)nr * n;
                k_probe_rhs<<<dim3(ceil_div(per, 256), (unsigned)conv.size()), 256, 0, st>>>(
                    per, bSys.as<int>(), bW.as<double>(), bEta.as<double>(), bR.as<double2>() + vo);
                c->launches++;
                PB_CHECK_LAUNCH();
                PB_TRY(pb_lu_solve_mapped<float>(&c->lu, n, (int)conv.size(), nr, m32, n, nn, perm,
                                                 bR.as<double2>() + vo, bD.as<double2>() + vo, bSys.as<int>(), nullptr,
                                                 reorder ? 1 : 0));
                // port voltages of x (with the port injections) and of the probe solution
                // (linear part only) for systems nd .. nb
                const int *pnone = bPC.as<int>() + 2 * np;
                const int *pcx0 = pw ? pnone : bPC.as<int>();
                double2 *zx = bZp.as<double2>(), *zy = zx + (long long)mb * np * nr;
                for (int pass = 0; pass < 2; pass++) {
                    const double2 *xv = (pass ? bD.as<double2>() : bX.as<double2>()) + vo;
                    if (form == PB_FORM_REDUCED) {
                        k_z_reduced<<<dim3(nr, np, mb), 256, 0, st>>>(np, nr, n, nc, bP.as<double2>() + (long long)nd * nc * nc,
                                                                     (long long)nc * nc, c->d_inc_off, c->d_inc_seg,
                                                                     bPC.as<int>(), pass ? pnone : pcx0, xv,
                                                                     bFreq.as<double>() + nd, pass ? zy : zx);
                    } else {
                        k_z_full<<<ceil_div(mb * np * nr, 128), 128, 0, st>>>(mb, np, nr, n, bPC.as<int>(), xv,
                                                                              pass ? zy : zx);
                    }
                    c->launches++;
                    PB_CHECK_LAUNCH();
                }
                std::vector<double2> zph((size_t)2 * mb * np * nr);
                PB_CUDA(cudaMemcpyAsync(zph.data(), zx, sizeof(double2) * zph.size(), cudaMemcpyDeviceToHost, st));
                PB_CUDA(cudaStreamSynchronize(st));
                const size_t per_z = (size_t)np * nr;
                for (int q : conv) {
                    double ax = 0, ay = 0;
                    for (size_t t = 0; t < per_z; t++) {
                        const double2 a = zph[(size_t)q * per_z + t], b = zph[(size_t)(mb + q) * per_z + t];
                        ax = std::max(ax, std::hypot(a.x, a.y));
                        ay = std::max(ay, std::hypot(b.x, b.y));
                    }
                    const double sens = ax > 0 ? ay / ax : 0.0;
                    probe_max = std::max(probe_max, sens);
                    if (sens > 2.5e-7) { state[nd + q] = 2; probe_fb++; }
                }
            }
        }
        if (nb > nd) {
            // FP64 fallback, batched: copy the stalled frequencies' FP64 matrices into the
            // (no longer needed) FP32 factor storage, factorise and solve them together.
            std::vector<int> failed;
            for (int q = nd; q < nb; q++) if (state[q] == 2) failed.push_back(q);
            const int cap = std::max(1, B / 2);
            for (size_t g0 = 0; g0 < failed.size(); g0 += cap) {
                const int ng = (int)std::min<size_t>(cap, failed.size() - g0);
                double2 *scr = reinterpret_cast<double2 *>(bM32.p);
                for (int t = 0; t < ng; t++) {
                    const int q = failed[g0 + t];
                    PB_CUDA(cudaMemcpyAsync(scr + t * nn, bM64.as<double2>() + q * nn, sizeof(double2) * nn,
                                            cudaMemcpyDeviceToDevice, st));
                    PB_CUDA(cudaMemcpyAsync(bR.as<double2>() + (long long)t * nr * n,
                                            bRhs.as<double2>() + (long long)q * nr * n, sizeof(double2) * nr * n,
                                            cudaMemcpyDeviceToDevice, st));
                }
                if (lower) PB_TRY(pb_sym_mirror(&c->lu, n, ng, scr, nn));
                PB_TRY(pb_lu_factor<double>(&c->lu, n, ng, scr, n, nn, bPiv.as<int>(), bInfo.as<int>()));
                lu_count += ng;
                PB_TRY(pb_lu_perm(&c->lu, n, ng, bPiv.as<int>(), bPerm.as<int>()));
                PB_TRY(pb_lu_solve_batched<double>(&c->lu, n, ng, nr, scr, n, nn, bPerm.as<int>(), bR.as<double2>(),
                                                   bD.as<double2>()));
                PB_CUDA(cudaMemcpyAsync(infoh.data(), bInfo.p, sizeof(int) * ng, cudaMemcpyDeviceToHost, st));
                for (int t = 0; t < ng; t++) {
                    const int q = failed[g0 + t];
                    PB_CUDA(cudaMemcpyAsync(bX.as<double2>() + (long long)q * nr * n, bD.as<double2>() + (long long)t * nr * n,
                                            sizeof(double2) * nr * n, cudaMemcpyDeviceToDevice, st));
                }
                PB_CUDA(cudaStreamSynchronize(st));
                for (int t = 0; t < ng; t++)
                    if (infoh[t] >= 0) {
                        pb_set_error("singular matrix at f = %.5e Hz (row %d : floating node or ideal voltage source loop?)",
                                     fb[failed[g0 + t]], infoh[t]);
                        return PB_ERR_SINGULAR;
                    }
                fallbacks += ng;
                fp64_hz = std::max(fp64_hz, fb[failed[g0 + ng - 1]]);
                if (o.verbose)
                    for (int t = 0; t < ng; t++) fprintf(stderr, "pb_sweep: FP64 fallback at f = %.6e Hz\n", fb[failed[g0 + t]]);
            }
        }
        fp64_direct += nd;
        // port voltages -> Z
        // port voltages per excitation: Z columns (1 A at port j) or the open-circuit
        // voltages of the plane-wave excitation (no injection: excitation cells -1)
        const int *pcx = pw ? bPC.as<int>() + 2 * np : bPC.as<int>();
        if (rhs_fixed) {
            // node voltages of the source excitation (print_vnode, solve.c:102-112)
            std::vector<double2> xh((size_t)nb * n);
            PB_CUDA(cudaMemcpyAsync(xh.data(), bX.p, sizeof(double2) * xh.size(), cudaMemcpyDeviceToHost, st));
            PB_CUDA(cudaStreamSynchronize(st));
            const int nid = c->maxid + 1;
            for (int q = 0; q < nb; q++)
                for (int id = 0; id < nid; id++) {
                    const int m = c->nodemap[id];
                    const double2 v = m >= 0 ? xh[(size_t)q * n + m] : make_double2(0, 0);
                    vnode[2 * ((size_t)(b0 + q) * nid + id)] = v.x;
                    vnode[2 * ((size_t)(b0 + q) * nid + id) + 1] = v.y;
                }
        } else if (form == PB_FORM_REDUCED) {
            dim3 g(nr, np, nb);
            k_z_reduced<<<g, 256, 0, st>>>(np, nr, n, nc, bP.as<double2>(), (long long)nc * nc, c->d_inc_off,
                                           c->d_inc_seg, bPC.as<int>(), pcx, bX.as<double2>(), bFreq.as<double>(),
                                           bZ.as<double2>());
        } else {
            k_z_full<<<ceil_div(nb * np * nr, 128), 128, 0, st>>>(nb, np, nr, n, bPC.as<int>(), bX.as<double2>(),
                                                                  bZ.as<double2>());
        }
        c->launches++;
        PB_CHECK_LAUNCH();
        tRef.stop(st);
        if (zmat && !pw) PB_CUDA(cudaMemcpyAsync(zmat + 2 * (size_t)b0 * np * np, bZ.p, sizeof(double2) * nb * np * np,
                                                 cudaMemcpyDeviceToHost, st));
        if (voc && pw) {
            PB_CUDA(cudaMemcpyAsync(zh.data(), bZ.p, sizeof(double2) * nb * np, cudaMemcpyDeviceToHost, st));
            PB_CUDA(cudaStreamSynchronize(st));
            for (int q = 0; q < nb; q++)
                for (int i = 0; i < np; i++) {
                    voc[2 * ((size_t)i * nfreq + b0 + q)] = zh[(size_t)q * np + i].x;
                    voc[2 * ((size_t)i * nfreq + b0 + q) + 1] = zh[(size_t)q * np + i].y;
                }
        }
        if (segipw && pw) {
            const int off = (form == PB_FORM_REDUCED) ? 0 : c->offS;
            for (int q = 0; q < nb; q++)
                PB_CUDA(cudaMemcpyAsync(segipw + 2 * ((size_t)(b0 + q) * ns), bX.as<double2>() + (long long)q * n + off,
                                        sizeof(double2) * ns, cudaMemcpyDeviceToHost, st));
        }
        if (cellq && !pw && !rhs_fixed && c->capacitance && nc > 0) {
            k_cellq<<<(int)ceil_div((long long)nb * np * nc, 256), 256, 0, st>>>(
                nb, np, n, nc, form == PB_FORM_REDUCED, c->nunknown, c->d_inc_off, c->d_inc_seg, bPC.as<int>(),
                bX.as<double2>(), bFreq.as<double>(), bQ.as<double2>());
            c->launches++;
            PB_CHECK_LAUNCH();
            PB_CUDA(cudaMemcpyAsync(cellq + 2 * (size_t)b0 * np * nc, bQ.p, sizeof(double2) * nb * np * nc,
                                    cudaMemcpyDeviceToHost, st));
        }
        if (segi && !pw) {
            const int off = (form == PB_FORM_REDUCED) ? 0 : c->offS;
            for (int q = 0; q < nb; q++)
                for (int j = 0; j < np; j++)
                    PB_CUDA(cudaMemcpyAsync(segi + 2 * (((size_t)(b0 + q) * np + j) * ns),
                                            bX.as<double2>() + ((long long)q * np + j) * n + off,
                                            sizeof(double2) * ns, cudaMemcpyDeviceToHost, st));
        }
        PB_CUDA(cudaStreamSynchronize(st));
    }
    tAll.stop(st);
    tStatic.finish();
    tCorr.finish();
    tAsm.finish();
    if (stats) {
        stats->t_static_ms = tStatic.acc;
        stats->t_corr_ms = tCorr.acc;
        stats->t_assemble_ms = tAsm.acc;
        stats->t_lu_ms = tLu.acc;
        stats->t_refine_ms = tRef.acc;
        stats->t_total_ms = tAll.acc;
        stats->corr_samples = samples;
        stats->lu_flops = luflops;
        stats->max_resid = maxres;
        stats->max_iters = maxits;
        stats->form_used = form;
        stats->n_system = n;
        stats->static_refreshes = refreshes;
        stats->kernel_launches = (int)(c->launches + c->lu.launches - launches0);
        stats->fp64_fallbacks = fallbacks;
        stats->fp64_direct = fp64_direct;
        stats->fp64_max_hz = fp64_hz;
        stats->lu_count = lu_count;
        stats->gmres_solves = gm_solves;
        stats->gmres_its_max = gm_max;
        stats->gmres_refactored = refactored;
        stats->gmres_its_avg = gm_solves > 0 ? (double)gm_its / gm_solves : 0.0;
        stats->probe_fallbacks = probe_fb;
        stats->pipelined = pipe ? 1 : 0;
        stats->probe_max = probe_max;
    }
    return PB_OK;
}
