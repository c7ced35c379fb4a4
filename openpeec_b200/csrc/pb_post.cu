// pb_post.cu — post-processing of the sweep on the GPU: far-field radiation vector and
// pattern (output_far, src/farfield.c:42-182) and transient synthesis (tran_synth /
// output_tran, src/transient.c:73-177). Both are sums over the whole sweep that the
// reference runs serially per output sample; here one thread owns one output sample
// (direction or time step) and the summed operands are staged in shared memory tiles.
#include <cmath>
#include <vector>
#include "pb_ctx.cuh"

namespace {

struct Dev1 {
    void *p = nullptr;
    ~Dev1() { if (p) cudaFree(p); }
    int alloc(size_t b)
    {
        cudaError_t e = cudaMalloc(&p, b ? b : 16);
        if (e != cudaSuccess) { p = nullptr; return pb_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__); }
        return PB_OK;
    }
    template <typename T> T *as() const { return (T *)p; }
};

// A buffer held by the context between calls (grown when too small, freed by pb_destroy):
// no cudaMalloc / cudaFree, which synchronises the device, on repeated calls.
struct Held1 {
    pb_cache_slot *s;
    void *p = nullptr;
    explicit Held1(pb_cache_slot *slot) : s(slot) {}
    int alloc(size_t b)
    {
        if (b == 0) b = 16;
        if (s->cap < b) {
            if (s->p) cudaFree(s->p);
            s->p = nullptr;
            s->cap = 0;
            cudaError_t e = cudaMalloc(&s->p, b);
            if (e != cudaSuccess) { s->p = nullptr; return pb_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__); }
            s->cap = b;
        }
        p = s->p;
        return PB_OK;
    }
    template <typename T> T *as() const { return (T *)p; }
};

__device__ __forceinline__ double sinc_d(double x)                 // farfield.c:37-40
{
    return fabs(x) < 1e-8 ? 1.0 : sin(x) / x;
}

#define FF_T 128            // directions per CTA and segments per shared-memory tile

// Radiation vector N(r^) = sum_m I_m len_m t_m sinc(k len_m (r^.t_m)/2) exp(+j k r^.r_cm)
// (plus the image cells with -I over a ground plane) and the transverse far field
// r E = -j (omega mu0 / 4 pi) [N - (N.r^) r^] per direction (farfield.c:85-140).
// geo: [nseg][8] = t (3), centre (3), len, pad. cur: [nfreq] rows of stride cstride.
__global__ void __launch_bounds__(FF_T)
k_farfield(int nseg, const double *geo, const double2 *cur, long long cstride, const double *freq, int nth, int nph,
           double thmax, int gp, double gpz, double2 *et, double2 *ep, double *uu)
{
    __shared__ double sg[FF_T][8];
    __shared__ double2 si[FF_T];
    const int f = blockIdx.y, ndir = (nth + 1) * nph;
    const int id = blockIdx.x * FF_T + threadIdx.x;
    const double kw = 2 * PB_PI * freq[f] / PB_C0;
    const double coef = 2 * PB_PI * freq[f] * PB_MU0 / (4 * PB_PI);
    const int it = id / nph, ip = id - it * nph;
    const double th = thmax * it / nth, phv = 2 * PB_PI * ip / nph;
    double st, ct, sp, cp;
    sincos(th, &st, &ct);
    sincos(phv, &sp, &cp);
    const double rh[3] = {st * cp, st * sp, ct};
    double nr[3] = {0, 0, 0}, ni[3] = {0, 0, 0};
    const double2 *cf = cur + (long long)f * cstride;
    const int npass = gp ? 2 : 1;
    for (int pass = 0; pass < npass; pass++) {
        for (int m0 = 0; m0 < nseg; m0 += FF_T) {
            const int nt = min(FF_T, nseg - m0);
            __syncthreads();
            if (threadIdx.x < nt) {
                for (int q = 0; q < 8; q++) sg[threadIdx.x][q] = geo[(long long)(m0 + threadIdx.x) * 8 + q];
                si[threadIdx.x] = cf[m0 + threadIdx.x];
            }
            __syncthreads();
            if (id >= ndir) continue;
            for (int m = 0; m < nt; m++) {
                double tv[3] = {sg[m][0], sg[m][1], sg[m][2]}, rc[3] = {sg[m][3], sg[m][4], sg[m][5]};
                double sgn = 1;
                if (pass == 1) {                         // image: t' = (tx, ty, -tz), -I (farfield.c:103-108)
                    tv[2] = -tv[2];
                    rc[2] = 2 * gpz - rc[2];
                    sgn = -1;
                }
                const double rt = rh[0] * tv[0] + rh[1] * tv[1] + rh[2] * tv[2];
                const double rr = rh[0] * rc[0] + rh[1] * rc[1] + rh[2] * rc[2];
                const double amp = sgn * sg[m][6] * sinc_d(0.5 * kw * sg[m][6] * rt);
                double s, c;
                sincos(kw * rr, &s, &c);
                const double2 I = si[m];
                const double wr = amp * (I.x * c - I.y * s), wi = amp * (I.x * s + I.y * c);
                for (int q = 0; q < 3; q++) { nr[q] += tv[q] * wr; ni[q] += tv[q] * wi; }
            }
        }
    }
    if (id >= ndir) return;
    const double thh[3] = {ct * cp, ct * sp, -st}, phh[3] = {-sp, cp, 0};
    double ntr = 0, nti = 0, npr = 0, npi = 0;
    for (int q = 0; q < 3; q++) {
        ntr += thh[q] * nr[q]; nti += thh[q] * ni[q];
        npr += phh[q] * nr[q]; npi += phh[q] * ni[q];
    }
    const long long o = (long long)f * ndir + id;
    const double2 e1 = make_double2(coef * nti, -coef * ntr), e2 = make_double2(coef * npi, -coef * npr);
    et[o] = e1;
    ep[o] = e2;
    uu[o] = (e1.x * e1.x + e1.y * e1.y + e2.x * e2.x + e2.y * e2.y) / (2 * PB_MU0 * PB_C0);
}

#define TR_T 256            // time samples per CTA and frequencies per tile

// y[s][n] = df (g0 + 2 sum_k Re(g_k e^{j 2 pi f_k t_n})), t_n = n dt, g_k = H_k X_k
// (tran_synth, transient.c:73-95); signal 0 is the excitation pulse itself (H = 1).
__global__ void __launch_bounds__(TR_T)
k_transient(int nf, double f0, double f1, const double2 *g, const double *g0, double df, double dt, int m, double *y)
{
    __shared__ double2 gs[TR_T];
    __shared__ double fs[TR_T];
    const int sig = blockIdx.y, n = blockIdx.x * TR_T + threadIdx.x;
    const double t = n * dt;
    double sum = g0[sig];
    for (int k0 = 0; k0 < nf; k0 += TR_T) {
        const int nt = min(TR_T, nf - k0);
        __syncthreads();
        if (threadIdx.x < nt) {
            const int k = k0 + threadIdx.x;
            gs[threadIdx.x] = g[(long long)sig * nf + k];
            fs[threadIdx.x] = nf > 1 ? f0 + (f1 - f0) * k / (nf - 1) : f0;      // freq_at (peec.h:241-248)
        }
        __syncthreads();
        if (n < m)
            for (int k = 0; k < nt; k++) {
                double s, c;
                sincos(2 * PB_PI * fs[k] * t, &s, &c);
                sum += 2 * (gs[k].x * c - gs[k].y * s);
            }
    }
    if (n < m) y[(long long)sig * m + n] = df * sum;
}

}  // namespace

extern "C" int pb_farfield(pb_ctx *c, int nfreq, const double *freq, const double *segi, long long seg_stride,
                           const double *zin, int nth, int nph, double *et, double *ep, double *d_dbi, double *g_dbi,
                           double *prad, double *pin)
{
    if (!c || nfreq <= 0 || !freq || !segi || nth < 2 || nph < 2 || !et || !ep) {
        pb_set_error("pb_farfield: bad argument (nth, nph >= 2 as farfield.c requires)");
        return PB_ERR_ARG;
    }
    const int ns = (int)c->seg.size();
    if (ns <= 0) { pb_set_error("pb_farfield: no current cells"); return PB_ERR_ARG; }
    if (seg_stride < ns) { pb_set_error("pb_farfield: seg_stride below the cell count"); return PB_ERR_ARG; }
    PB_CUDA(cudaSetDevice(c->dev));
    const cudaStream_t st = c->stream;
    const int ndir = (nth + 1) * nph;
    std::vector<double> geo((size_t)ns * 8, 0.0);
    for (int m = 0; m < ns; m++) {
        const pb_cell_t &s = c->seg[m];
        for (int q = 0; q < 3; q++) {
            geo[(size_t)m * 8 + q] = (s.x2[q] - s.x1[q]) / s.len;
            geo[(size_t)m * 8 + 3 + q] = 0.5 * (s.x1[q] + s.x2[q]);
        }
        geo[(size_t)m * 8 + 6] = s.len;
    }
    pb_cache_slot *cs = c->cache + PB_SLOT_POST0;
    Held1 dgeo(cs + 0), dcur(cs + 1), dfreq(cs + 2), det(cs + 3), dep(cs + 4), duu(cs + 5);
    PB_TRY(dgeo.alloc(sizeof(double) * geo.size()));
    PB_TRY(dcur.alloc(sizeof(double2) * (size_t)nfreq * ns));
    PB_TRY(dfreq.alloc(sizeof(double) * nfreq));
    PB_TRY(det.alloc(sizeof(double2) * (size_t)nfreq * ndir));
    PB_TRY(dep.alloc(sizeof(double2) * (size_t)nfreq * ndir));
    PB_TRY(duu.alloc(sizeof(double) * (size_t)nfreq * ndir));
    PB_CUDA(cudaMemcpyAsync(dgeo.p, geo.data(), sizeof(double) * geo.size(), cudaMemcpyHostToDevice, st));
    for (int f = 0; f < nfreq; f++)
        PB_CUDA(cudaMemcpyAsync(dcur.as<double2>() + (size_t)f * ns, segi + 2 * (size_t)f * seg_stride,
                                sizeof(double2) * ns, cudaMemcpyHostToDevice, st));
    PB_CUDA(cudaMemcpyAsync(dfreq.p, freq, sizeof(double) * nfreq, cudaMemcpyHostToDevice, st));
    const double thmax = c->gp ? PB_PI / 2 : PB_PI;
    dim3 g(ceil_div(ndir, FF_T), nfreq);
    k_farfield<<<g, FF_T, 0, st>>>(ns, dgeo.as<double>(), dcur.as<double2>(), ns, dfreq.as<double>(), nth, nph, thmax,
                                   c->gp, c->gpz, det.as<double2>(), dep.as<double2>(), duu.as<double>());
    c->launches++;
    PB_CHECK_LAUNCH();
    std::vector<double> uu((size_t)nfreq * ndir);
    PB_CUDA(cudaMemcpyAsync(et, det.p, sizeof(double2) * (size_t)nfreq * ndir, cudaMemcpyDeviceToHost, st));
    PB_CUDA(cudaMemcpyAsync(ep, dep.p, sizeof(double2) * (size_t)nfreq * ndir, cudaMemcpyDeviceToHost, st));
    PB_CUDA(cudaMemcpyAsync(uu.data(), duu.p, sizeof(double) * uu.size(), cudaMemcpyDeviceToHost, st));
    PB_CUDA(cudaStreamSynchronize(st));
    // radiated power (theta trapezoid, phi periodic rectangle), input power of 1 A at
    // port 1, directivity and gain (farfield.c:143-175)
    for (int f = 0; f < nfreq; f++) {
        const double *u = &uu[(size_t)f * ndir];
        double pr = 0;
        for (int it = 0; it <= nth; it++) {
            const double wt = (it == 0 || it == nth) ? 0.5 : 1;
            const double stv = sin(thmax * it / nth);
            double row = 0;
            for (int ip = 0; ip < nph; ip++) row += u[it * nph + ip];
            pr += wt * stv * row;
        }
        pr *= (thmax / nth) * (2 * PB_PI / nph);
        const double pi_ = zin ? 0.5 * zin[2 * f] : 0.0;
        if (prad) prad[f] = pr;
        if (pin) pin[f] = pi_;
        for (int id = 0; id < ndir; id++) {
            const double d = pr > 0 ? 4 * PB_PI * u[id] / pr : 0;
            const double gg = pi_ > 0 ? 4 * PB_PI * u[id] / pi_ : 0;
            if (d_dbi) d_dbi[(size_t)f * ndir + id] = d > 1e-30 ? 10 * log10(d) : -600;
            if (g_dbi) g_dbi[(size_t)f * ndir + id] = gg > 1e-30 ? 10 * log10(gg) : -600;
        }
    }
    return PB_OK;
}

extern "C" int pb_transient(int nfreq, double f0, double f1, double att_db, int nsig, const double *h, double *x,
                            double *y, double *dt_out)
{
    if (nfreq < 3) { pb_set_error("transient : at least 3 frequency points are required"); return PB_ERR_ARG; }
    const double df = (f1 - f0) / (nfreq - 1);
    if (!(df > 0) || fabs(f0 - df) > 1e-6 * df) {              // tran_check (transient.c:40-66)
        pb_set_error("transient : sweep must be f_k = k df (start = spacing); f0 = %.6e, df = %.6e", f0, df);
        return PB_ERR_ARG;
    }
    if (!(att_db > 0) || nsig < 0 || (nsig > 0 && (!h || !y)) || !x) { pb_set_error("pb_transient: bad argument"); return PB_ERR_ARG; }
    int nd = 0;
    if (cudaGetDeviceCount(&nd) != cudaSuccess || nd <= 0) { cudaGetLastError(); pb_set_error("no CUDA device"); return PB_ERR_CUDA; }
    const int m = 2 * nfreq;
    const double dt = 1 / (2 * f1);
    // Gaussian pulse, att dB down at f_max (transient.c:110-124)
    const double sigma = sqrt(att_db * log(10.0) / (20 * 2 * PB_PI * PB_PI)) / f1, t0 = 4 * sigma;
    const double x0 = sigma * sqrt(2 * PB_PI);
    std::vector<double2> g((size_t)(nsig + 1) * nfreq);
    std::vector<double> g0(nsig + 1);
    for (int k = 0; k < nfreq; k++) {
        const double f = f0 + (f1 - f0) * k / (nfreq - 1);
        const double a = x0 * exp(-2 * PB_PI * PB_PI * sigma * sigma * f * f), ph = -2 * PB_PI * f * t0;
        g[k] = make_double2(a * cos(ph), a * sin(ph));
    }
    g0[0] = x0;                                                  // H = 1
    for (int s = 0; s < nsig; s++) {
        const double *hs = h + 2 * (size_t)s * nfreq;
        for (int k = 0; k < nfreq; k++) {
            const double2 xs = g[k];
            g[(size_t)(s + 1) * nfreq + k] = make_double2(hs[2 * k] * xs.x - hs[2 * k + 1] * xs.y,
                                                         hs[2 * k] * xs.y + hs[2 * k + 1] * xs.x);
        }
        g0[s + 1] = (2 * hs[0] - hs[2]) * x0;                   // DC extrapolated from f_1, f_2 (transient.c:78-80)
    }
    Dev1 dg, dg0, dy;
    PB_TRY(dg.alloc(sizeof(double2) * g.size()));
    PB_TRY(dg0.alloc(sizeof(double) * g0.size()));
    PB_TRY(dy.alloc(sizeof(double) * (size_t)(nsig + 1) * m));
    PB_CUDA(cudaMemcpy(dg.p, g.data(), sizeof(double2) * g.size(), cudaMemcpyHostToDevice));
    PB_CUDA(cudaMemcpy(dg0.p, g0.data(), sizeof(double) * g0.size(), cudaMemcpyHostToDevice));
    dim3 grid(ceil_div(m, TR_T), nsig + 1);
    k_transient<<<grid, TR_T>>>(nfreq, f0, f1, dg.as<double2>(), dg0.as<double>(), df, dt, m, dy.as<double>());
    PB_CHECK_LAUNCH();
    PB_CUDA(cudaMemcpy(x, dy.p, sizeof(double) * m, cudaMemcpyDeviceToHost));
    if (nsig > 0) PB_CUDA(cudaMemcpy(y, dy.as<double>() + m, sizeof(double) * (size_t)nsig * m, cudaMemcpyDeviceToHost));
    if (dt_out) *dt_out = dt;
    return PB_OK;
}
