// pb_gmres.cu — batched right-preconditioned GMRES(m) in FP64 for many frequencies at
// once: the reference's gmres_cycle / gmres_solve (src/iterative.c:83-252) as used by
// acceleration = 1 (src/solve.c:47-64), where a stale LU factorisation serves as the
// preconditioner of the following frequencies.
//
// Every (frequency, port) pair is one GMRES instance with its own Krylov basis; the
// instances advance together, so each Arnoldi step is one batched preconditioner solve
// (FP32 LU of the system's anchor frequency), one batched FP64 matrix-vector product and
// a classical Gram-Schmidt pass repeated twice (CGS2, as stable as the reference's
// modified Gram-Schmidt, two launches instead of j). The small Hessenberg least-squares
// problems (Givens rotations, back substitution) are solved on the host, exactly as
// gmres_cycle writes them. Instances that converge stop; systems whose instances have
// all converged leave the batched kernels.
//
// Stopping rule: the reference stops at |g_{j+1}| <= tol ||b|| (ACCEL_TOL = 1e-10). Here
// the target is the same normwise backward error as the iterative refinement of the
// fresh-LU path, |r|_2 <= eta (|A| |x| + |b|) (infinity norms on the right), checked with
// the true residual before every restart, so both solve paths give the same accuracy.
#include "pb_gmres.cuh"
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

typedef std::complex<double> zc;

// h[k][i] = V_i[k]^H w[k] for i < j1, for the instances of the active systems.
// Grid (active systems * nrhs, j1); one block reduces one dot product in fixed order.
__global__ void __launch_bounds__(256)
k_gs_dot(int n, int nrhs, const int *sys, const double2 *V, long long vstride, const double2 *w,
         double2 *h, int ldh)
{
    __shared__ double sr[8], si[8];
    const int s = sys[blockIdx.x / nrhs], q = blockIdx.x % nrhs, i = blockIdx.y;
    const long long k = (long long)s * nrhs + q;
    const double2 *v = V + (long long)i * vstride + k * n;
    const double2 *x = w + k * n;
    double ar = 0, ai = 0;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const double2 a = v[e], b = x[e];
        ar += a.x * b.x + a.y * b.y;                 // conj(a) * b
        ai += a.x * b.y - a.y * b.x;
    }
    for (int o = 16; o > 0; o >>= 1) {
        ar += __shfl_down_sync(0xffffffffu, ar, o);
        ai += __shfl_down_sync(0xffffffffu, ai, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { sr[warp] = ar; si[warp] = ai; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tr = 0, ti = 0;
        for (int t = 0; t < (int)(blockDim.x >> 5); t++) { tr += sr[t]; ti += si[t]; }
        h[k * ldh + i] = make_double2(tr, ti);
    }
}

// w[k] -= sum_{i<j1} h[k][i] V_i[k]. Grid (active systems * nrhs, ceil(n / 256)).
__global__ void k_gs_axpy(int n, int nrhs, const int *sys, const double2 *V, long long vstride,
                          const double2 *h, int ldh, int j1, double2 *w)
{
    const int s = sys[blockIdx.x / nrhs], q = blockIdx.x % nrhs;
    const long long k = (long long)s * nrhs + q;
    const int e = blockIdx.y * blockDim.x + threadIdx.x;
    if (e >= n) return;
    double2 acc = w[k * n + e];
    for (int i = 0; i < j1; i++) {
        const double2 c = h[k * ldh + i], v = V[(long long)i * vstride + k * n + e];
        acc.x -= c.x * v.x - c.y * v.y;
        acc.y -= c.x * v.y + c.y * v.x;
    }
    w[k * n + e] = acc;
}

// nrm[k] = |w[k]|_2 and out[k] = w[k] / nrm[k] (out untouched when the norm is 0).
// One block per instance of the active systems.
__global__ void __launch_bounds__(256)
k_norm_scale(int n, int nrhs, const int *sys, const double2 *w, double2 *out, double *nrm)
{
    __shared__ double sh[9];
    const int s = sys[blockIdx.x / nrhs], q = blockIdx.x % nrhs;
    const long long k = (long long)s * nrhs + q;
    double a = 0;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const double2 v = w[k * n + e];
        a += v.x * v.x + v.y * v.y;
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int u = 0; u < (int)(blockDim.x >> 5); u++) t += sh[u];
        sh[8] = sqrt(t);
        nrm[k] = sh[8];
    }
    __syncthreads();
    const double nv = sh[8];
    if (nv > 0)
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            const double2 v = w[k * n + e];
            out[k * n + e] = make_double2(v.x / nv, v.y / nv);
        }
}

// u[k] = sum_{l<m} y[k][l] V_l[k] for the instances of the active systems.
__global__ void k_combine(int n, int nrhs, const int *sys, const double2 *V, long long vstride,
                          const double2 *y, int ldy, int m, double2 *u)
{
    const int s = sys[blockIdx.x / nrhs], q = blockIdx.x % nrhs;
    const long long k = (long long)s * nrhs + q;
    const int e = blockIdx.y * blockDim.x + threadIdx.x;
    if (e >= n) return;
    double2 acc = make_double2(0, 0);
    for (int l = 0; l < m; l++) {
        const double2 c = y[k * ldy + l], v = V[(long long)l * vstride + k * n + e];
        acc.x += c.x * v.x - c.y * v.y;
        acc.y += c.x * v.y + c.y * v.x;
    }
    u[k * n + e] = acc;
}

// x[k] += d[k] for the instances of the active systems.
__global__ void k_add_sys(int n, int nrhs, const int *sys, const double2 *d, double2 *x)
{
    const int s = sys[blockIdx.x / nrhs], q = blockIdx.x % nrhs;
    const long long k = (long long)s * nrhs + q;
    const int e = blockIdx.y * blockDim.x + threadIdx.x;
    if (e >= n) return;
    x[k * n + e].x += d[k * n + e].x;
    x[k * n + e].y += d[k * n + e].y;
}

namespace {
struct Buf {
    void *p = nullptr;
    ~Buf() { if (p) cudaFree(p); }
    int alloc(size_t b)
    {
        cudaError_t e = cudaMalloc(&p, b ? b : 16);
        if (e != cudaSuccess) { p = nullptr; return pb_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__); }
        return PB_OK;
    }
    template <typename T> T *as() const { return (T *)p; }
};

// Host side of one GMRES instance within a cycle (gmres_cycle, iterative.c:83-196).
struct Inst {
    std::vector<zc> h;      // (m+1) x m Hessenberg, column major (h[i + j (m+1)])
    std::vector<zc> cs, sn, g;
    int done = 0;           // 0 iterating, 1 converged or broke down
    int k = 0;              // columns used for the least-squares solution
    double target = 0;      // absolute target for |g_{j+1}|
};
}  // namespace

int pb_gmres_batched(const pb_gmres_args &a, std::vector<int> &state, pb_gmres_result *res)
{
    const int n = a.n, ns = a.nsys, np = a.nrhs, m = std::max(1, std::min(a.m, PB_GMRES_MAXM));
    pb_lu_engine *e = a.eng;
    const cudaStream_t st = e->stream;
    const long long K = (long long)ns * np;
    const long long vstride = K * n;
    res->iters_total = 0;
    res->iters_max = 0;
    res->solved = 0;
    if (ns <= 0) return PB_OK;

    Buf bV, bW, bZ, bH1, bH2, bNrm, bY, bSys, bLuOf, bRn, bBn, bXn, bAn;
    PB_TRY(bV.alloc(sizeof(double2) * (size_t)(m + 1) * vstride));
    PB_TRY(bW.alloc(sizeof(double2) * (size_t)vstride));
    PB_TRY(bZ.alloc(sizeof(double2) * (size_t)vstride));
    PB_TRY(bH1.alloc(sizeof(double2) * (size_t)K * (m + 1)));
    PB_TRY(bH2.alloc(sizeof(double2) * (size_t)K * (m + 1)));
    PB_TRY(bNrm.alloc(sizeof(double) * (size_t)K));
    PB_TRY(bY.alloc(sizeof(double2) * (size_t)K * m));
    PB_TRY(bSys.alloc(sizeof(int) * (size_t)ns));
    PB_TRY(bLuOf.alloc(sizeof(int) * (size_t)ns));
    PB_TRY(bRn.alloc(sizeof(double) * (size_t)K));
    PB_TRY(bBn.alloc(sizeof(double) * (size_t)K));
    PB_TRY(bXn.alloc(sizeof(double) * (size_t)K));
    PB_TRY(bAn.alloc(sizeof(double) * (size_t)ns));
    PB_CUDA(cudaMemcpyAsync(bLuOf.p, a.lu_of, sizeof(int) * ns, cudaMemcpyHostToDevice, st));

    std::vector<double> rn(K), bn(K), xn(K), an(ns), nrm(K);
    std::vector<double2> h1(K * (m + 1)), h2(K * (m + 1)), yh(K * m);
    std::vector<int> act;
    std::vector<int> its(ns, 0);
    std::vector<Inst> inst(K);
    const int nthr = 256, nchunk = ceil_div(n, nthr);

    // x0 = M^-1 b (the anchor's factors)
    {
        std::vector<int> all;
        for (int s = 0; s < ns; s++) if (state[s] == 0) all.push_back(s);
        if (all.empty()) return PB_OK;
        PB_CUDA(cudaMemcpyAsync(bSys.p, all.data(), sizeof(int) * all.size(), cudaMemcpyHostToDevice, st));
        PB_TRY(pb_lu_solve_mapped<float>(e, n, (int)all.size(), np, a.lu, n, a.lu_stride, a.perm, a.b, a.x,
                                         bSys.as<int>(), bLuOf.as<int>()));
    }

    std::vector<int> todo;
    for (int cyc = 0; cyc <= a.max_cycles; cyc++) {
        // true residual r = b - A x into V_0 for the systems still being solved
        todo.clear();
        for (int s = 0; s < ns; s++) if (state[s] == 0) todo.push_back(s);
        if (todo.empty()) break;
        PB_CUDA(cudaMemcpyAsync(bSys.p, todo.data(), sizeof(int) * todo.size(), cudaMemcpyHostToDevice, st));
        PB_TRY(pb_residual_mapped(e, n, (int)todo.size(), np, a.A, n, a.A_stride, a.b, a.x, bV.as<double2>(),
                                  bRn.as<double>(), bBn.as<double>(), bXn.as<double>(),
                                  cyc == 0 ? bAn.as<double>() : nullptr, ns, bSys.as<int>()));
        PB_CUDA(cudaMemcpyAsync(rn.data(), bRn.p, sizeof(double) * K, cudaMemcpyDeviceToHost, st));
        PB_CUDA(cudaMemcpyAsync(bn.data(), bBn.p, sizeof(double) * K, cudaMemcpyDeviceToHost, st));
        PB_CUDA(cudaMemcpyAsync(xn.data(), bXn.p, sizeof(double) * K, cudaMemcpyDeviceToHost, st));
        if (cyc == 0) PB_CUDA(cudaMemcpyAsync(an.data(), bAn.p, sizeof(double) * ns, cudaMemcpyDeviceToHost, st));
        PB_CUDA(cudaStreamSynchronize(st));
        act.clear();
        for (int s = 0; s < ns; s++) {
            if (state[s] != 0) continue;
            bool ok = true;
            for (int q = 0; q < np; q++) {
                const long long k = (long long)s * np + q;
                const double den = an[s] * xn[k] + bn[k];
                if (den > 0 && rn[k] > a.eta * den) ok = false;
            }
            if (ok) {
                state[s] = 1;
                res->solved++;
                continue;
            }
            if (cyc == a.max_cycles) { state[s] = 2; continue; }
            act.push_back(s);
        }
        if (act.empty()) break;
        PB_CUDA(cudaMemcpyAsync(bSys.p, act.data(), sizeof(int) * act.size(), cudaMemcpyHostToDevice, st));
        const int na = (int)act.size();
        const int nk = na * np;
        // beta = |r|, V_0 = r / beta
        k_norm_scale<<<nk, 256, 0, st>>>(n, np, bSys.as<int>(), bV.as<double2>(), bV.as<double2>(), bNrm.as<double>());
        e->launches++;
        PB_CHECK_LAUNCH();
        PB_CUDA(cudaMemcpyAsync(nrm.data(), bNrm.p, sizeof(double) * K, cudaMemcpyDeviceToHost, st));
        PB_CUDA(cudaStreamSynchronize(st));
        for (int s : act)
            for (int q = 0; q < np; q++) {
                const long long k = (long long)s * np + q;
                Inst &I = inst[k];
                I.h.assign((size_t)(m + 1) * m, zc(0, 0));
                I.cs.assign(m, zc(0, 0));
                I.sn.assign(m, zc(0, 0));
                I.g.assign(m + 1, zc(0, 0));
                I.g[0] = zc(nrm[k], 0);
                // The bound is on |r|_inf; GMRES tracks |r|_2. Scale by this residual's own
                // inf/2-norm ratio (|r|_2 can exceed |r|_inf by up to sqrt(n)), with a factor
                // 2 margin; the true residual at the next cycle start decides convergence.
                const double ratio = nrm[k] > 0 ? rn[k] / nrm[k] : 1.0;
                I.target = 0.5 * a.eta * (an[s] * xn[k] + bn[k]) / std::max(ratio, 1e-300);
                I.done = (nrm[k] <= I.target) ? 1 : 0;
                I.k = 0;
            }
        std::vector<int> live = act;
        int j = 0;
        for (j = 0; j < m && !live.empty(); j++) {
            const int nl = (int)live.size();
            const int nlk = nl * np;
            PB_CUDA(cudaMemcpyAsync(bSys.p, live.data(), sizeof(int) * nl, cudaMemcpyHostToDevice, st));
            // w = A M^-1 v_j
            PB_TRY(pb_lu_solve_mapped<float>(e, n, nl, np, a.lu, n, a.lu_stride, a.perm,
                                             bV.as<double2>() + (long long)j * vstride, bZ.as<double2>(),
                                             bSys.as<int>(), bLuOf.as<int>()));
            PB_TRY(pb_matvec_mapped(e, n, nl, np, a.A, n, a.A_stride, bZ.as<double2>(), bW.as<double2>(),
                                    bSys.as<int>()));
            // CGS2 against V_0..V_j
            const int j1 = j + 1;
            k_gs_dot<<<dim3(nlk, j1), 256, 0, st>>>(n, np, bSys.as<int>(), bV.as<double2>(), vstride,
                                                    bW.as<double2>(), bH1.as<double2>(), m + 1);
            k_gs_axpy<<<dim3(nlk, nchunk), nthr, 0, st>>>(n, np, bSys.as<int>(), bV.as<double2>(), vstride,
                                                          bH1.as<double2>(), m + 1, j1, bW.as<double2>());
            k_gs_dot<<<dim3(nlk, j1), 256, 0, st>>>(n, np, bSys.as<int>(), bV.as<double2>(), vstride,
                                                    bW.as<double2>(), bH2.as<double2>(), m + 1);
            k_gs_axpy<<<dim3(nlk, nchunk), nthr, 0, st>>>(n, np, bSys.as<int>(), bV.as<double2>(), vstride,
                                                          bH2.as<double2>(), m + 1, j1, bW.as<double2>());
            k_norm_scale<<<nlk, 256, 0, st>>>(n, np, bSys.as<int>(), bW.as<double2>(),
                                              bV.as<double2>() + (long long)j1 * vstride, bNrm.as<double>());
            e->launches += 5;
            PB_CHECK_LAUNCH();
            PB_CUDA(cudaMemcpyAsync(h1.data(), bH1.p, sizeof(double2) * K * (m + 1), cudaMemcpyDeviceToHost, st));
            PB_CUDA(cudaMemcpyAsync(h2.data(), bH2.p, sizeof(double2) * K * (m + 1), cudaMemcpyDeviceToHost, st));
            PB_CUDA(cudaMemcpyAsync(nrm.data(), bNrm.p, sizeof(double) * K, cudaMemcpyDeviceToHost, st));
            PB_CUDA(cudaStreamSynchronize(st));
            std::vector<int> next;
            for (int s : live) {
                its[s]++;
                bool any = false;
                for (int q = 0; q < np; q++) {
                    const long long k = (long long)s * np + q;
                    Inst &I = inst[k];
                    if (I.done) continue;
                    zc *hc = &I.h[(size_t)j * (m + 1)];
                    for (int i = 0; i <= j; i++) {
                        const double2 a1 = h1[k * (m + 1) + i], a2 = h2[k * (m + 1) + i];
                        hc[i] = zc(a1.x + a2.x, a1.y + a2.y);
                    }
                    hc[j + 1] = zc(nrm[k], 0);
                    // previous rotations (iterative.c:140-150)
                    for (int i = 0; i < j; i++) {
                        const zc a1 = hc[i], a2 = hc[i + 1];
                        hc[i] = std::conj(I.cs[i]) * a1 + std::conj(I.sn[i]) * a2;
                        hc[i + 1] = I.cs[i] * a2 - I.sn[i] * a1;
                    }
                    // new rotation (iterative.c:153-163)
                    const zc a1 = hc[j], a2 = hc[j + 1];
                    const double rho = std::sqrt(std::norm(a1) + std::norm(a2));
                    if (rho <= 0) { I.done = 1; I.k = j; continue; }
                    I.cs[j] = a1 / rho;
                    I.sn[j] = a2 / rho;
                    hc[j] = zc(rho, 0);
                    hc[j + 1] = zc(0, 0);
                    I.g[j + 1] = -(I.sn[j] * I.g[j]);
                    I.g[j] = std::conj(I.cs[j]) * I.g[j];
                    I.k = j + 1;
                    if (std::abs(I.g[j + 1]) <= I.target || nrm[k] <= 0) I.done = 1;
                    else any = true;
                }
                if (any) next.push_back(s);
            }
            live.swap(next);
        }
        // least-squares solutions y = H^-1 g (iterative.c:172-182), u = V y, x += M^-1 u
        std::fill(yh.begin(), yh.end(), make_double2(0, 0));
        for (int s : act)
            for (int q = 0; q < np; q++) {
                const long long k = (long long)s * np + q;
                Inst &I = inst[k];
                std::vector<zc> y(I.k);
                for (int i = I.k - 1; i >= 0; i--) {
                    zc t = I.g[i];
                    for (int l = i + 1; l < I.k; l++) t -= I.h[i + (size_t)l * (m + 1)] * y[l];
                    y[i] = t / I.h[i + (size_t)i * (m + 1)];
                }
                for (int l = 0; l < I.k; l++) yh[k * m + l] = make_double2(y[l].real(), y[l].imag());
            }
        PB_CUDA(cudaMemcpyAsync(bSys.p, act.data(), sizeof(int) * na, cudaMemcpyHostToDevice, st));
        PB_CUDA(cudaMemcpyAsync(bY.p, yh.data(), sizeof(double2) * K * m, cudaMemcpyHostToDevice, st));
        k_combine<<<dim3(nk, nchunk), nthr, 0, st>>>(n, np, bSys.as<int>(), bV.as<double2>(), vstride,
                                                    bY.as<double2>(), m, m, bW.as<double2>());
        e->launches++;
        PB_CHECK_LAUNCH();
        PB_TRY(pb_lu_solve_mapped<float>(e, n, na, np, a.lu, n, a.lu_stride, a.perm, bW.as<double2>(),
                                         bZ.as<double2>(), bSys.as<int>(), bLuOf.as<int>()));
        k_add_sys<<<dim3(nk, nchunk), nthr, 0, st>>>(n, np, bSys.as<int>(), bZ.as<double2>(), a.x);
        e->launches++;
        PB_CHECK_LAUNCH();
    }
    for (int s = 0; s < ns; s++) {
        res->iters_total += its[s];
        res->iters_max = std::max(res->iters_max, its[s]);
    }
    return PB_OK;
}
