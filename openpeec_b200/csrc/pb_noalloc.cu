// pb_noalloc.cu — partial-inductance fill for callers that cannot allocate device memory.
//
// Some hosts own all of the GPU's memory themselves: a solver or simulator that reserves
// the device memory up front in its own pool allocator and treats any further cudaMalloc
// as an error, or a real-time loop that cannot afford the device-wide synchronisation a
// cudaMalloc / cudaFree may cause. pb_lp_fill (include/peec_b200.h) allocates its FP64
// static table and its output on every call, so such hosts cannot use it.
// pb_lp_fill_noalloc computes the same matrix with the same kernels, but takes every
// input and output as caller-owned device memory and keeps its only scratch buffer (the
// FP64 static table) in the file-scope array below, which every GPU that loads this
// library holds until the process exits. The first call on each device looks the array's
// device address up (cudaGetSymbolAddress, with that device current); make that first
// call before any stream capture. Every call reuses the same array and the same input
// flag, so calls that overlap on the GPU race: serialise them.
#include <cstring>
#include <mutex>
#include "pb_ctx.cuh"

// Largest number of current cells the fixed scratch holds: nseg^2 doubles = 2 MiB.
#define PB_NOALLOC_MAX_SEG 512

static __device__ __align__(256) double g_noalloc_static[PB_NOALLOC_MAX_SEG * PB_NOALLOC_MAX_SEG];
static __device__ int g_noalloc_flag;        // set by the input check below
// largest cell extent, as the bit pattern of a non-negative double (atomicMax orders them)
static __device__ unsigned long long g_noalloc_ext;

// Device address of the scratch array, looked up once per device (in host code the
// symbol's name is only a stand-in, never a device address).
static double *g_scratch_addr[64];
static int *g_flag_addr[64];
static unsigned long long *g_ext_addr[64];
static std::mutex g_scratch_mu;

// Input check on the device: polygon cells need point sets this entry point does not
// keep, and every cell needs a positive length. Also the largest cell extent (the same
// expression pb_create evaluates on the host for non-polygon cells), whose double bounds
// the distance offsets of the correction samples: with it the FP32 correction takes the
// same launch variant (angle reduction, small-step series) as pb_lp_fill.
__global__ void k_noalloc_check(const pb_cell_t *seg, int n, int *flag, unsigned long long *ext)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (seg[i].npv > 0 || !(seg[i].len > 0)) atomicOr(flag, 1);
    const double e = seg[i].len + seg[i].wid + seg[i].thick + 2 * seg[i].radius;
    if (e > 0) atomicMax(ext, (unsigned long long)__double_as_longlong(e));
}

extern "C" int pb_lp_fill_noalloc(int nseg, const pb_cell_t *seg_dev, int gp, double gpz,
                                  double kw, int prec, double *lp_dev)
{
    if (nseg <= 0 || !seg_dev || !lp_dev || kw < 0) {
        pb_set_error("pb_lp_fill_noalloc: bad argument");
        return PB_ERR_ARG;
    }
    if (nseg > PB_NOALLOC_MAX_SEG) {
        pb_set_error("pb_lp_fill_noalloc: %d cells exceed the fixed scratch of %d cells; "
                     "use pb_lp_fill", nseg, PB_NOALLOC_MAX_SEG);
        return PB_ERR_ARG;
    }
    int dev = 0;
    PB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) { pb_set_error("pb_lp_fill_noalloc: device index %d out of range", dev); return PB_ERR_ARG; }
    {
        // once per device, with that device current
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        if (!g_scratch_addr[dev]) {
            double *p = nullptr;
            int *f = nullptr;
            unsigned long long *x = nullptr;
            PB_CUDA(cudaGetSymbolAddress((void **)&p, g_noalloc_static));
            PB_CUDA(cudaGetSymbolAddress((void **)&f, g_noalloc_flag));
            PB_CUDA(cudaGetSymbolAddress((void **)&x, g_noalloc_ext));
            g_flag_addr[dev] = f;
            g_ext_addr[dev] = x;
            g_scratch_addr[dev] = p;         // set last: marks the device as set up
        }
    }
    double *st = g_scratch_addr[dev];
    int *flag = g_flag_addr[dev];
    unsigned long long *ext = g_ext_addr[dev];
    const cudaStream_t s = 0;
    PB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
    PB_CUDA(cudaMemsetAsync(ext, 0, sizeof(unsigned long long), s));
    k_noalloc_check<<<ceil_div(nseg, 128), 128, 0, s>>>(seg_dev, nseg, flag, ext);
    PB_CHECK_LAUNCH();
    int hflag = 0;
    unsigned long long hext = 0;
    PB_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaMemcpyAsync(&hext, ext, sizeof(hext), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    if (hflag) {
        pb_set_error("pb_lp_fill_noalloc: polygon cells or zero-length cells are not accepted here; use pb_lp_fill");
        return PB_ERR_UNSUP;
    }
    pb_fill_geom g;
    g.seg.n = nseg;
    g.seg.cell = const_cast<pb_cell_t *>(seg_dev);
    g.gp = gp;
    g.gpz = gpz;
    double ext_max = 0;
    memcpy(&ext_max, &hext, sizeof(ext_max));
    g.pmax = 2 * ext_max;
    PB_TRY(pb_lp_static(g, kw, st, s, nullptr));          // static table -> scratch
    pb_epi_args ea;
    ea.out = reinterpret_cast<double2 *>(lp_dev);
    ea.out_stride = (long long)nseg * nseg;
    PB_TRY(pb_lp_corr(g, 1, &kw, prec == PB_PREC_MIXED, st, PB_EPI_STORE, ea, s, nullptr, nullptr));
    PB_CUDA(cudaStreamSynchronize(s));
    return PB_OK;
}
