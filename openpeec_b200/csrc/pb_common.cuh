// pb_common.cuh — shared definitions of libpeec_b200 (constants, complex helpers,
// error plumbing, device-side cell frames).
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cmath>
#include "../../include/peec_b200.h"

// Physical constants defined exactly as the reference (include/peec.h:31-34):
// PI = 4 atan(1) is the correctly rounded double pi.
#define PB_PI   3.141592653589793
#define PB_C0   2.99792458e8
#define PB_MU0  (4.0 * PB_PI * 1e-7)
#define PB_EPS0 (1.0 / (PB_C0 * PB_C0 * PB_MU0))
#define PB_POLY_MAX 64

// ------------------------------------------------------------------ errors
void pb_set_error(const char *fmt, ...);
int  pb_cuda_fail(cudaError_t e, const char *what, const char *file, int line);
#define PB_CUDA(call) do { cudaError_t e_ = (call); \
    if (e_ != cudaSuccess) return pb_cuda_fail(e_, #call, __FILE__, __LINE__); } while (0)
#define PB_CHECK_LAUNCH() PB_CUDA(cudaGetLastError())
#define PB_TRY(call) do { int r_ = (call); if (r_ != PB_OK) return r_; } while (0)

// ------------------------------------------------------------------ complex
template <typename T> struct cplx_t;
template <> struct cplx_t<float>  { typedef float2  type; };
template <> struct cplx_t<double> { typedef double2 type; };

template <typename T2> __host__ __device__ __forceinline__ T2 mk2(double r, double i)
{ T2 z; z.x = r; z.y = i; return z; }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b)
{ return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b)
{ return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b)
{ return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b)
{ return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b)
{ return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b)
{ return make_double2(a.x - b.x, a.y - b.y); }
// a - l*u  (complex multiply-subtract, the LU update)
__host__ __device__ __forceinline__ float2 cfms(float2 a, float2 l, float2 u)
{ return make_float2(a.x - (l.x * u.x - l.y * u.y), a.y - (l.x * u.y + l.y * u.x)); }
__host__ __device__ __forceinline__ double2 cfms(double2 a, double2 l, double2 u)
{ return make_double2(a.x - (l.x * u.x - l.y * u.y), a.y - (l.x * u.y + l.y * u.x)); }
// 1/z, 0 for z == 0 (reference complex.h:52-57)
template <typename T2> __host__ __device__ __forceinline__ T2 cinv(T2 z)
{
    auto n2 = z.x * z.x + z.y * z.y;
    if (n2 <= 0) return mk2<T2>(0, 0);
    return mk2<T2>(z.x / n2, -z.y / n2);
}
template <typename T2> __host__ __device__ __forceinline__ double cmag1(T2 z)
{ return fabs((double)z.x) + fabs((double)z.y); }       // pivot measure, lu.c:10-13

// ------------------------------------------------------------------ kernel attributes
// cudaFuncSetAttribute acts on the current device only. A process that drives several
// devices (one context per device, e.g. pb_sweep_many over contexts on different GPUs)
// must set a kernel's shared-memory opt-in on each of them, so the flag that skips the
// repeated call is a bit mask over device indices; devices >= 64 set it on every call.
template <typename K>
static inline int pb_smem_optin(K kernel, int bytes, std::atomic<unsigned long long> &done)
{
    int dev = 0;
    PB_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return PB_OK;
    PB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if (bit) done.fetch_or(bit, std::memory_order_release);
    return PB_OK;
}

// Largest dynamic shared memory one block may opt in to on the current device.
static inline int pb_smem_cap()
{
    int dev = 0, cap = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&cap, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return cap;
}

// ------------------------------------------------------------------ misc
static inline unsigned ceil_div(long a, long b) { return (unsigned)((a + b - 1) / b); }

// Row of the upper triangle (i <= j, row-major packing of the n x n upper triangle)
// holding linear index t: S(i) = i*n - i*(i-1)/2 <= t < S(i+1).
__host__ __device__ __forceinline__ void tri_index(long long t, int n, int &i, int &j)
{
    const double b = 2.0 * n + 1.0;
    long long r = (long long)((b - sqrt(b * b - 8.0 * (double)t)) * 0.5);
    if (r < 0) r = 0;
    if (r > n - 1) r = n - 1;
    // fix rounding: ensure S(r) <= t < S(r+1)
    while (r > 0 && (r * (long long)n - r * (r - 1) / 2) > t) r--;
    while (r + 1 < n && ((r + 1) * (long long)n - (r + 1) * r / 2) <= t) r++;
    i = (int)r;
    j = (int)(t - (r * (long long)n - r * (r - 1) / 2) + r);
}
