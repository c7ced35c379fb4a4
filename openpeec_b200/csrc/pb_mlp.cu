// pb_mlp.cu — the learned part of the preconditioner: a 12 -> 128 -> 128 -> 2 tanh MLP that
// predicts, per current cell, a correction to the diagonal of its leaf block in the
// compressed path's preconditioner (the plain one is precond.c:138-391). Forward, backward
// and Adam are hand-written FP32 kernels. One CTA of 128 threads (one per hidden unit) works
// on 32 samples; gradients are written per CTA and summed in a fixed order, so training is
// deterministic.
#include "pb_mlp.cuh"
#include <cmath>
#include <vector>

#define MLP_S 32            // samples per CTA

__global__ void __launch_bounds__(PB_MLP_H)
k_mlp_fwd(const float *__restrict__ w, int n, const float *__restrict__ x, float *__restrict__ y,
          float *__restrict__ h1g, float *__restrict__ h2g)
{
    __shared__ float xs[MLP_S][PB_MLP_IN];
    __shared__ float h1[MLP_S][PB_MLP_H + 1];
    __shared__ float h2[MLP_S][PB_MLP_H + 1];
    __shared__ float part[PB_MLP_H / 32][MLP_S][PB_MLP_OUT];
    const int s0 = blockIdx.x * MLP_S, u = threadIdx.x, lane = u & 31, warp = u >> 5;
    for (int e = u; e < MLP_S * PB_MLP_IN; e += blockDim.x) {
        const int s = e / PB_MLP_IN, k = e % PB_MLP_IN;
        xs[s][k] = (s0 + s < n) ? x[(long long)(s0 + s) * PB_MLP_IN + k] : 0.f;
    }
    __syncthreads();
    {
        float wr[PB_MLP_IN];
#pragma unroll
        for (int k = 0; k < PB_MLP_IN; k++) wr[k] = w[PB_MLP_OFF_W1 + u * PB_MLP_IN + k];
        const float b = w[PB_MLP_OFF_B1 + u];
        for (int s = 0; s < MLP_S; s++) {
            float a = b;
#pragma unroll
            for (int k = 0; k < PB_MLP_IN; k++) a = fmaf(wr[k], xs[s][k], a);
            h1[s][u] = tanhf(a);
        }
    }
    __syncthreads();
    {
        float acc[MLP_S];
        const float b = w[PB_MLP_OFF_B2 + u];
#pragma unroll
        for (int s = 0; s < MLP_S; s++) acc[s] = b;
        for (int v = 0; v < PB_MLP_H; v++) {
            const float wv = w[PB_MLP_OFF_W2 + u * PB_MLP_H + v];
#pragma unroll
            for (int s = 0; s < MLP_S; s++) acc[s] = fmaf(wv, h1[s][v], acc[s]);
        }
#pragma unroll
        for (int s = 0; s < MLP_S; s++) h2[s][u] = tanhf(acc[s]);
    }
    __syncthreads();
    for (int o = 0; o < PB_MLP_OUT; o++) {
        const float wo = w[PB_MLP_OFF_W3 + o * PB_MLP_H + u];
        for (int s = 0; s < MLP_S; s++) {
            float p = wo * h2[s][u];
            for (int off = 16; off > 0; off >>= 1) p += __shfl_down_sync(0xffffffffu, p, off);
            if (lane == 0) part[warp][s][o] = p;
        }
    }
    __syncthreads();
    if (u < MLP_S * PB_MLP_OUT) {
        const int s = u / PB_MLP_OUT, o = u % PB_MLP_OUT;
        float a = w[PB_MLP_OFF_B3 + o];
        for (int q = 0; q < PB_MLP_H / 32; q++) a += part[q][s][o];
        if (s0 + s < n) y[(long long)(s0 + s) * PB_MLP_OUT + o] = a;
    }
    if (h1g)
        for (int s = 0; s < MLP_S; s++)
            if (s0 + s < n) {
                h1g[(long long)(s0 + s) * PB_MLP_H + u] = h1[s][u];
                h2g[(long long)(s0 + s) * PB_MLP_H + u] = h2[s][u];
            }
}

// Gradient of L = mean over samples and outputs of (y - t)^2 for the CTA's 32 samples,
// written to gpart[blockIdx.x][NPARAM]; lpart[blockIdx.x] = the CTA's share of L.
__global__ void __launch_bounds__(PB_MLP_H)
k_mlp_bwd(const float *__restrict__ w, int n, const float *__restrict__ x, const float *__restrict__ t,
          const float *__restrict__ y, const float *__restrict__ h1g, const float *__restrict__ h2g,
          float *__restrict__ gpart, float *__restrict__ lpart)
{
    __shared__ float xs[MLP_S][PB_MLP_IN];
    __shared__ float h1[MLP_S][PB_MLP_H + 1];
    __shared__ float g2[MLP_S][PB_MLP_H + 1];    // layer-2 deltas, then layer-1 deltas
    __shared__ float dy[MLP_S][PB_MLP_OUT];
    const int s0 = blockIdx.x * MLP_S, u = threadIdx.x;
    float *g = gpart + (long long)blockIdx.x * PB_MLP_NPARAM;
    const float scale = 2.f / ((float)n * PB_MLP_OUT);
    for (int e = u; e < MLP_S * PB_MLP_IN; e += blockDim.x) {
        const int s = e / PB_MLP_IN, k = e % PB_MLP_IN;
        xs[s][k] = (s0 + s < n) ? x[(long long)(s0 + s) * PB_MLP_IN + k] : 0.f;
    }
    if (u < MLP_S * PB_MLP_OUT) {
        const int s = u / PB_MLP_OUT, o = u % PB_MLP_OUT;
        const bool ok = s0 + s < n;
        dy[s][o] = ok ? scale * (y[(long long)(s0 + s) * PB_MLP_OUT + o] - t[(long long)(s0 + s) * PB_MLP_OUT + o]) : 0.f;
    }
    float h2r[MLP_S];
    for (int s = 0; s < MLP_S; s++) {
        const bool ok = s0 + s < n;
        h1[s][u] = ok ? h1g[(long long)(s0 + s) * PB_MLP_H + u] : 0.f;
        h2r[s] = ok ? h2g[(long long)(s0 + s) * PB_MLP_H + u] : 0.f;
    }
    __syncthreads();
    if (u == 0) {
        float l = 0;
        for (int s = 0; s < MLP_S; s++)
            for (int o = 0; o < PB_MLP_OUT; o++) {
                const float d = dy[s][o] / scale;
                l += d * d;
            }
        lpart[blockIdx.x] = l / ((float)n * PB_MLP_OUT);
    }
    // output layer
    for (int o = 0; o < PB_MLP_OUT; o++) {
        float a = 0;
        for (int s = 0; s < MLP_S; s++) a = fmaf(dy[s][o], h2r[s], a);
        g[PB_MLP_OFF_W3 + o * PB_MLP_H + u] = a;
    }
    if (u < PB_MLP_OUT) {
        float a = 0;
        for (int s = 0; s < MLP_S; s++) a += dy[s][u];
        g[PB_MLP_OFF_B3 + u] = a;
    }
    {
        float w3[PB_MLP_OUT];
        for (int o = 0; o < PB_MLP_OUT; o++) w3[o] = w[PB_MLP_OFF_W3 + o * PB_MLP_H + u];
        for (int s = 0; s < MLP_S; s++) {
            float a = 0;
            for (int o = 0; o < PB_MLP_OUT; o++) a = fmaf(w3[o], dy[s][o], a);
            g2[s][u] = a * (1.f - h2r[s] * h2r[s]);
        }
    }
    __syncthreads();
    // second layer: dW2[u][v] = sum_s g2[s][u] h1[s][v]
    {
        float db = 0;
        for (int s = 0; s < MLP_S; s++) db += g2[s][u];
        g[PB_MLP_OFF_B2 + u] = db;
        for (int v = 0; v < PB_MLP_H; v++) {
            float a = 0;
            for (int s = 0; s < MLP_S; s++) a = fmaf(g2[s][u], h1[s][v], a);
            g[PB_MLP_OFF_W2 + u * PB_MLP_H + v] = a;
        }
    }
    // back to the first layer: thread u is hidden unit v = u of layer 1
    {
        float acc[MLP_S];
#pragma unroll
        for (int s = 0; s < MLP_S; s++) acc[s] = 0.f;
        for (int q = 0; q < PB_MLP_H; q++) {
            const float wq = w[PB_MLP_OFF_W2 + q * PB_MLP_H + u];
#pragma unroll
            for (int s = 0; s < MLP_S; s++) acc[s] = fmaf(wq, g2[s][q], acc[s]);
        }
        __syncthreads();                             // every thread is done reading g2
        for (int s = 0; s < MLP_S; s++) g2[s][u] = acc[s] * (1.f - h1[s][u] * h1[s][u]);
    }
    __syncthreads();
    {
        float db = 0;
        for (int s = 0; s < MLP_S; s++) db += g2[s][u];
        g[PB_MLP_OFF_B1 + u] = db;
        for (int k = 0; k < PB_MLP_IN; k++) {
            float a = 0;
            for (int s = 0; s < MLP_S; s++) a = fmaf(g2[s][u], xs[s][k], a);
            g[PB_MLP_OFF_W1 + u * PB_MLP_IN + k] = a;
        }
    }
}

__global__ void k_mlp_reduce(int nblk, const float *gpart, float *grad)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= PB_MLP_NPARAM) return;
    float a = 0;
    for (int b = 0; b < nblk; b++) a += gpart[(long long)b * PB_MLP_NPARAM + p];
    grad[p] = a;
}

__global__ void k_mlp_adam(float *w, const float *g, float *m, float *v, float lr, float b1t, float b2t)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= PB_MLP_NPARAM) return;
    const float b1 = 0.9f, b2 = 0.999f;
    m[p] = b1 * m[p] + (1 - b1) * g[p];
    v[p] = b2 * v[p] + (1 - b2) * g[p] * g[p];
    const float mh = m[p] / (1 - b1t), vh = v[p] / (1 - b2t);
    w[p] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

int pb_mlp_forward_dev(const float *d_w, int n, const float *d_x, float *d_y, cudaStream_t s)
{
    if (n <= 0) return PB_OK;
    k_mlp_fwd<<<ceil_div(n, MLP_S), PB_MLP_H, 0, s>>>(d_w, n, d_x, d_y, nullptr, nullptr);
    PB_CHECK_LAUNCH();
    return PB_OK;
}

namespace {
struct MBuf {
    void *p = nullptr;
    ~MBuf() { if (p) cudaFree(p); }
    int alloc(size_t b)
    {
        cudaError_t e = cudaMalloc(&p, b ? b : 16);
        if (e != cudaSuccess) { p = nullptr; return pb_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__); }
        return PB_OK;
    }
    float *f() const { return (float *)p; }
};

int need_gpu()
{
    int nd = 0;
    cudaError_t e = cudaGetDeviceCount(&nd);
    if (e != cudaSuccess || nd <= 0) { pb_set_error("no CUDA device"); return PB_ERR_CUDA; }
    return PB_OK;
}

// loss and gradient on the device for the whole set (full batch)
int grad_dev(const float *w, int n, const float *x, const float *t, float *y, float *h1, float *h2, float *gpart,
             float *lpart, float *grad, float *loss_host, cudaStream_t s)
{
    const int nb = ceil_div(n, MLP_S);
    k_mlp_fwd<<<nb, PB_MLP_H, 0, s>>>(w, n, x, y, h1, h2);
    k_mlp_bwd<<<nb, PB_MLP_H, 0, s>>>(w, n, x, t, y, h1, h2, gpart, lpart);
    k_mlp_reduce<<<ceil_div(PB_MLP_NPARAM, 256), 256, 0, s>>>(nb, gpart, grad);
    PB_CHECK_LAUNCH();
    if (loss_host) {
        std::vector<float> lp(nb);
        PB_CUDA(cudaMemcpyAsync(lp.data(), lpart, sizeof(float) * nb, cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaStreamSynchronize(s));
        double l = 0;
        for (float v : lp) l += v;
        *loss_host = (float)l;
    }
    return PB_OK;
}

struct Set {
    MBuf w, x, t, y, h1, h2, gp, lp, g, m, v;
    int init(int n, const float *wh, const float *xh, const float *th)
    {
        const int nb = ceil_div(n, MLP_S);
        PB_TRY(w.alloc(sizeof(float) * PB_MLP_NPARAM));
        PB_TRY(x.alloc(sizeof(float) * (size_t)n * PB_MLP_IN));
        PB_TRY(t.alloc(sizeof(float) * (size_t)n * PB_MLP_OUT));
        PB_TRY(y.alloc(sizeof(float) * (size_t)n * PB_MLP_OUT));
        PB_TRY(h1.alloc(sizeof(float) * (size_t)n * PB_MLP_H));
        PB_TRY(h2.alloc(sizeof(float) * (size_t)n * PB_MLP_H));
        PB_TRY(gp.alloc(sizeof(float) * (size_t)nb * PB_MLP_NPARAM));
        PB_TRY(lp.alloc(sizeof(float) * (size_t)nb));
        PB_TRY(g.alloc(sizeof(float) * PB_MLP_NPARAM));
        PB_TRY(m.alloc(sizeof(float) * PB_MLP_NPARAM));
        PB_TRY(v.alloc(sizeof(float) * PB_MLP_NPARAM));
        PB_CUDA(cudaMemcpy(w.p, wh, sizeof(float) * PB_MLP_NPARAM, cudaMemcpyHostToDevice));
        PB_CUDA(cudaMemcpy(x.p, xh, sizeof(float) * (size_t)n * PB_MLP_IN, cudaMemcpyHostToDevice));
        if (th) PB_CUDA(cudaMemcpy(t.p, th, sizeof(float) * (size_t)n * PB_MLP_OUT, cudaMemcpyHostToDevice));
        PB_CUDA(cudaMemset(m.p, 0, sizeof(float) * PB_MLP_NPARAM));
        PB_CUDA(cudaMemset(v.p, 0, sizeof(float) * PB_MLP_NPARAM));
        return PB_OK;
    }
};
}  // namespace

extern "C" int pb_mlp_nparam(void) { return PB_MLP_NPARAM; }

extern "C" int pb_mlp_predict(const float *w, int n, const float *x, float *y)
{
    if (n <= 0 || !w || !x || !y) { pb_set_error("pb_mlp_predict: bad argument"); return PB_ERR_ARG; }
    PB_TRY(need_gpu());
    Set S;
    PB_TRY(S.init(n, w, x, nullptr));
    PB_TRY(pb_mlp_forward_dev(S.w.f(), n, S.x.f(), S.y.f(), 0));
    PB_CUDA(cudaMemcpy(y, S.y.p, sizeof(float) * (size_t)n * PB_MLP_OUT, cudaMemcpyDeviceToHost));
    return PB_OK;
}

extern "C" int pb_mlp_grad(const float *w, int n, const float *x, const float *t, float *grad, float *loss)
{
    if (n <= 0 || !w || !x || !t || !grad) { pb_set_error("pb_mlp_grad: bad argument"); return PB_ERR_ARG; }
    PB_TRY(need_gpu());
    Set S;
    PB_TRY(S.init(n, w, x, t));
    float l = 0;
    PB_TRY(grad_dev(S.w.f(), n, S.x.f(), S.t.f(), S.y.f(), S.h1.f(), S.h2.f(), S.gp.f(), S.lp.f(), S.g.f(), &l, 0));
    PB_CUDA(cudaMemcpy(grad, S.g.p, sizeof(float) * PB_MLP_NPARAM, cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
    return PB_OK;
}

extern "C" int pb_mlp_train(float *w, int n, const float *x, const float *t, int steps, float lr, float *loss_hist)
{
    if (n <= 0 || steps <= 0 || !w || !x || !t) { pb_set_error("pb_mlp_train: bad argument"); return PB_ERR_ARG; }
    PB_TRY(need_gpu());
    Set S;
    PB_TRY(S.init(n, w, x, t));
    float b1t = 1, b2t = 1;
    for (int it = 0; it < steps; it++) {
        float l = 0;
        const bool rec = loss_hist != nullptr;
        PB_TRY(grad_dev(S.w.f(), n, S.x.f(), S.t.f(), S.y.f(), S.h1.f(), S.h2.f(), S.gp.f(), S.lp.f(), S.g.f(),
                        rec ? &l : nullptr, 0));
        if (rec) loss_hist[it] = l;
        b1t *= 0.9f;
        b2t *= 0.999f;
        k_mlp_adam<<<ceil_div(PB_MLP_NPARAM, 256), 256>>>(S.w.f(), S.g.f(), S.m.f(), S.v.f(), lr, b1t, b2t);
        PB_CHECK_LAUNCH();
    }
    PB_CUDA(cudaMemcpy(w, S.w.p, sizeof(float) * PB_MLP_NPARAM, cudaMemcpyDeviceToHost));
    return PB_OK;
}
