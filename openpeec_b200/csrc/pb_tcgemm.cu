// pb_tcgemm.cu — complex FP32 trailing update of the batched LU on the sm_100a tensor
// cores: C[b] -= A[b] * B[b] (row-major, interleaved re/im), the O(n^3) part of the
// factorisation (the row update of the reference's lu_decomp, src/lu.c:54-62).
//
// Arithmetic. Each FP32 operand x is split into three BF16 terms, x = t0 + t1 + t2 with
// t0 = bf16(x), t1 = bf16(x - t0), t2 = bf16(x - t0 - t1) (the differences are exact in
// FP32; together the terms carry all 24 bits of x), and a*b is formed from the six
// products of significance >= 2^-16: a0b0 + a0b1 + a1b0 + a0b2 + a1b1 + a2b0, on
// tcgen05.mma kind::f16 (BF16 inputs) with FP32 accumulation in TMEM. The dropped terms
// are below 2^-24 relative, so the update is as accurate as an FP32 product. (A split
// into two TF32 terms and three products keeps only ~22 bits; at the ill-conditioned low
// frequencies of a sweep that pushed twice as many systems onto the FP64 fall-back.)
// BF16 runs at twice the TF32 rate, so the six products cost what three TF32 ones do.
//
// Accumulation. The tensor core adds each MMA's products into the FP32 accumulator with
// truncation, so a long accumulation in TMEM drifts toward zero (measured on B200: a
// relative shrink of ~6e-9 per complex k, 1.2e-5 at k = 2048, against 1e-6 of random
// error for an FP32 product). The kernel therefore accumulates in TMEM only over chunks
// of KC = 64 complex k and adds every chunk into FP32 registers with round-to-nearest,
// which leaves ~4e-7 of bias per chunk and none across chunks.
//
// Complex structure. With A = Ar + j Ai and B read as the real k x 2nc matrix Br
// (interleaved columns Re b, Im b), two real products share the B operand:
//     X = Ar * Br,  Y = Ai * Br   (each 128 x 192 real per CTA, FP32 in TMEM)
// and the chunk adds  Re P += X[2j] - Y[2j+1],  Im P += X[2j+1] + Y[2j]; at the end
// C -= P.
//
// CTA (448 threads, one per SM: ~170 KB of shared memory, 512 TMEM columns):
//   warp 0     TMA producer: raw FP32 tiles A (128 x 16 complex, 128B-swizzled) and
//              B (16 x 96 complex) per stage, cp.async.bulk.tensor from this GPU's memory
//   warp 1     TMEM allocation and the MMA issuer (one thread): 12 tcgen05.mma per stage,
//              tcgen05.commit frees the operand stage / signals a finished chunk
//   warps 2-13 workers: split the raw tiles into the BF16 term planes (K-major, 128B
//              swizzle: the UMMA canonical layout; a 128-B row holds the three 16-value
//              terms); after each chunk, the three warps of each TMEM lane quarter read
//              their 32 complex columns of X and Y (tcgen05.ld) into FP32 registers; at
//              the end they subtract the sums from C
// Every wait on an mbarrier is bounded (2 s of %globaltimer); a timeout sets *err, stops
// the CTA's pipeline, skips the C update and still frees TMEM.
#include "pb_tcgemm.cuh"
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

namespace {

constexpr int TM = 128;                      // rows of C per CTA = TMEM lanes
constexpr int TN = 96;                       // complex columns of C per CTA (192 real, MMA N = 192)
constexpr int TK = 16;                       // complex k per pipeline stage
constexpr int KCS = 4;                       // stages per TMEM accumulation chunk (KC = 64 complex k)
constexpr int RS = 2;                        // raw (TMA) stages
constexpr int CS = 2;                        // operand (MMA) stages
constexpr int RAW_A = TM * TK * 8;           // 16 KB: 128 rows x 128 B, TMA 128B swizzle
constexpr int RAW_B = TK * TN * 8;           // 12 KB: 16 rows x 768 B, unswizzled
constexpr int RAW_STAGE = RAW_A + RAW_B;     // 28 KB (a multiple of 1 KB)
constexpr int PL_A = TM * 128;               // 16 KB: Re(A) or Im(A), 128 rows x [t0 | t1 | t2 | -] (16 BF16 each)
constexpr int PL_B = 2 * TN * 128;           // 24 KB: Br as 192 rows (real columns), same row layout
constexpr int OP_STAGE = 2 * PL_A + PL_B;    // 56 KB
constexpr int OFF_RAW = 0;
constexpr int OFF_OP = RS * RAW_STAGE;
constexpr int OFF_BAR = OFF_OP + CS * OP_STAGE;
constexpr int NBAR = 2 * RS + 2 * CS + 2;    // raw full/empty, operand full/empty, chunk full/empty
constexpr int SMEM_BYTES = OFF_BAR + 128 + 1024;  // barriers, TMEM slot, fail flag + alignment slack
constexpr int NWORK = 12;                    // worker warps (3 per TMEM lane quarter)
constexpr int NTHREADS = 32 * (2 + NWORK);
constexpr int NWT = 32 * NWORK;              // worker threads
constexpr int CPW = TN / 3;                  // complex columns per worker warp in the chunk sums (32)
constexpr uint32_t TMEM_COLS = 512;          // X at columns [0, 192), Y at [256, 448)
constexpr uint32_t Y_COL = 256;
constexpr uint64_t WAIT_NS = 2000000000ull;  // bound of every pipeline wait

// Instruction descriptor (kind::f16): D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9,
// 10-12 = 1), both K-major (bits 15, 16 = 0), N = 192 (bits 17-22 = N/8), M = 128
// (bits 24-28 = M/16).
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(2 * TN >> 3) << 17) |
                           ((uint32_t)(TM >> 4) << 24);

static_assert(SMEM_BYTES <= 227 * 1024, "shared memory budget");
static_assert(RAW_STAGE % 1024 == 0 && OP_STAGE % 1024 == 0 && PL_A % 1024 == 0, "swizzle atoms stay 1 KB aligned");
static_assert(TN % 24 == 0 && 2 * TN % 16 == 0 && 2 * TN <= 256, "MMA N and the 3-way column split");

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t gtimer()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Bounded wait for the phase of the given parity. False when it timed out (the CTA's
// fail flag and *err are set) or when another role of the CTA has already failed.
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *fail, int *err)
{
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = gtimer();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 63) == 0) {
            if (*fail) return false;
            if (gtimer() - t0 > WAIT_NS) {
                *fail = 1;
                atomicExch(err, 1);
                return false;
            }
        }
    }
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *tm, int c0, int c1, int c2,
                                            uint32_t bar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
                 : "memory");
}

// Shared-memory matrix descriptor of a K-major operand in the 128B-swizzled canonical
// layout: rows of 128 B, 8-row atoms 1024 B apart (SBO), version 1, layout SWIZZLE_128B.
// The K offset inside the 128-B row is added to the start address (atoms 1024-B aligned).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr)
{
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;                  // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset
    d |= (uint64_t)1 << 46;                  // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                  // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ void umma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t acc)
{
    const uint32_t z = 0;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                 ::"r"(dtmem), "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
                 : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
                   "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// x = t0 + t1 + t2 (+ a remainder below 2^-24 |x|), each term a BF16 value rounded to
// nearest; the two differences are exact in FP32. Eight values -> three 16-byte rows of
// BF16 (value i of term j in half i of out[j]).
__device__ __forceinline__ void split8_bf16x3(const float (&x)[8], uint4 (&out)[3])
{
    // two values per conversion instruction (cvt.rn.bf16x2.f32: the conversion pipe is the
    // kernel's busiest), the BF16 -> FP32 expansion by bit operations
    uint32_t w[3][4];
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
        float r0 = x[i], r1 = x[i + 1];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const __nv_bfloat162 b = __floats2bfloat162_rn(r0, r1);     // .x = r0 (low half)
            const uint32_t u = *reinterpret_cast<const uint32_t *>(&b);
            w[j][i >> 1] = u;
            if (j < 2) {
                r0 -= __uint_as_float(u << 16);
                r1 -= __uint_as_float(u & 0xffff0000u);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 3; j++) out[j] = make_uint4(w[j][0], w[j][1], w[j][2], w[j][3]);
}

// byte offset of 16-B chunk c of row r in a 128B-swizzled tile (rows of 128 B)
__device__ __forceinline__ uint32_t swz(int r, int c) { return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4)); }

__global__ void __launch_bounds__(NTHREADS, 1)
k_cgemm_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
           float2 *__restrict__ C, int ldc, long long stride, int m, int nc, int k, int *err, int lower)
{
    // lower: a tile whose rows all lie above its columns is not needed (symmetric updates);
    // the whole CTA leaves before any barrier or TMEM allocation
    if (lower && (int)(blockIdx.y + 1) * TM <= (int)blockIdx.x * TN) return;
    extern __shared__ unsigned char smraw[];
    const uint32_t raw0 = smem_u32(smraw);
    const uint32_t sb = (raw0 + 1023u) & ~1023u;         // 1024-B aligned base (swizzle atoms)
    unsigned char *sm = smraw + (sb - raw0);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t bar = sb + OFF_BAR;
    // barriers: raw_full[RS], raw_empty[RS], op_full[CS], op_empty[CS], chunk_full, chunk_empty
    auto raw_full = [&](int s) { return bar + 8 * s; };
    auto raw_empty = [&](int s) { return bar + 8 * (RS + s); };
    auto op_full = [&](int s) { return bar + 8 * (2 * RS + s); };
    auto op_empty = [&](int s) { return bar + 8 * (2 * RS + CS + s); };
    const uint32_t chunk_full = bar + 8 * (2 * RS + 2 * CS), chunk_empty = chunk_full + 8;
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(sm + OFF_BAR + 8 * NBAR);
    volatile int *fail = reinterpret_cast<volatile int *>(sm + OFF_BAR + 8 * NBAR + 16);

    const int n0 = blockIdx.x * TN, m0 = blockIdx.y * TM, b = blockIdx.z;
    const int nk = (k + TK - 1) / TK;
    const int nchunk = (nk + KCS - 1) / KCS;

    if (threadIdx.x == 0) {
        for (int s = 0; s < RS; s++) {
            mbar_init(raw_full(s), 1);                    // producer + TMA bytes
            mbar_init(raw_empty(s), NWT);                 // every worker thread
        }
        for (int s = 0; s < CS; s++) {
            mbar_init(op_full(s), NWT);                   // every worker thread
            mbar_init(op_empty(s), 1);                    // tcgen05.commit
        }
        mbar_init(chunk_full, 1);                         // tcgen05.commit
        mbar_init(chunk_empty, NWT);                      // every worker thread
        *fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_proxy_async();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32((const void *)tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ---------------------------------------------------------------- TMA producer
        if (lane == 0) {
            int issued = 0;
            for (int kt = 0; kt < nk; ++kt) {
                const int s = kt % RS;
                if (kt >= RS && !mbar_wait(raw_empty(s), ((kt / RS) & 1) ^ 1, fail, err)) break;
                const uint32_t dst = sb + OFF_RAW + s * RAW_STAGE;
                mbar_expect_tx(raw_full(s), RAW_STAGE);
                tma_load_3d(dst, &tmA, kt * 2 * TK, m0, b, raw_full(s));
                tma_load_3d(dst + RAW_A, &tmB, 2 * n0, kt * TK, b, raw_full(s));
                issued = kt + 1;
            }
            if (*fail) {
                // let copies still in flight land before the CTA's shared memory goes away
                for (int kt = issued > RS ? issued - RS : 0; kt < issued; ++kt) {
                    const uint64_t t0 = gtimer();
                    while (!mbar_try(raw_full(kt % RS), (kt / RS) & 1) && gtimer() - t0 < WAIT_NS / 8) {
                    }
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------------------------------------------------------- MMA issuer
        if (lane == 0) {
            for (int kt = 0; kt < nk; ++kt) {
                const int cs = kt % CS, c = kt / KCS;
                const bool first = (kt % KCS) == 0;
                // a chunk starts only once the workers have read the previous one out of TMEM
                if (first && c > 0 && !mbar_wait(chunk_empty, (c - 1) & 1, fail, err)) break;
                if (!mbar_wait(op_full(cs), (kt / CS) & 1, fail, err)) break;
                tc_fence_after();
                const uint32_t pre = sb + OFF_OP + cs * OP_STAGE, pim = pre + PL_A, pbm = pre + 2 * PL_A;
                // term j of every operand row starts 32 j bytes into the row (16 BF16 = one K slice)
                const uint64_t r0 = sdesc(pre), r1 = sdesc(pre + 32), r2 = sdesc(pre + 64);
                const uint64_t i0 = sdesc(pim), i1 = sdesc(pim + 32), i2 = sdesc(pim + 64);
                const uint64_t b0 = sdesc(pbm), b1 = sdesc(pbm + 32), b2 = sdesc(pbm + 64);
                const uint32_t acc = first ? 0u : 1u;
                umma_bf16(tmem, r0, b0, acc);
                umma_bf16(tmem, r0, b1, 1u);
                umma_bf16(tmem, r1, b0, 1u);
                umma_bf16(tmem, r0, b2, 1u);
                umma_bf16(tmem, r1, b1, 1u);
                umma_bf16(tmem, r2, b0, 1u);
                umma_bf16(tmem + Y_COL, i0, b0, acc);
                umma_bf16(tmem + Y_COL, i0, b1, 1u);
                umma_bf16(tmem + Y_COL, i1, b0, 1u);
                umma_bf16(tmem + Y_COL, i0, b2, 1u);
                umma_bf16(tmem + Y_COL, i1, b1, 1u);
                umma_bf16(tmem + Y_COL, i2, b0, 1u);
                umma_commit(op_empty(cs));                        // operand stage free when done
                if ((kt % KCS) == KCS - 1 || kt == nk - 1) umma_commit(chunk_full);
            }
            if (*fail) umma_commit(chunk_full);     // let the workers' wait end
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------------- workers
        const int w = threadIdx.x - 64;                                // 0..NWT-1
        const int q = warp & 3, g = (warp - 2) >> 2;                   // TMEM lane quarter, column third
        const uint32_t tl = tmem + ((uint32_t)(32 * q) << 16) + 2 * CPW * g;
        float2 part[CPW];
#pragma unroll
        for (int j = 0; j < CPW; j++) part[j] = make_float2(0.f, 0.f);
        bool ok = true;
        // chunk sums: X, Y of this warp's lane quarter and column third into FP32 registers
        auto drain = [&](int c) {
            if (!mbar_wait(chunk_full, c & 1, fail, err)) { ok = false; return; }
            tc_fence_after();
#pragma unroll
            for (int s8 = 0; s8 < CPW / 8; s8++) {
                uint32_t x[16], y[16];
                tmem_ld16(tl + 16 * s8, x);
                tmem_ld16(tl + Y_COL + 16 * s8, y);
                tmem_wait_ld();
#pragma unroll
                for (int jj = 0; jj < 8; jj++) {
                    float2 &p = part[8 * s8 + jj];
                    p.x += __uint_as_float(x[2 * jj]) - __uint_as_float(y[2 * jj + 1]);
                    p.y += __uint_as_float(x[2 * jj + 1]) + __uint_as_float(y[2 * jj]);
                }
            }
            tc_fence_before();
            mbar_arrive(chunk_empty);
        };
        for (int kt = 0; kt < nk && ok; ++kt) {
            const int s = kt % RS, cs = kt % CS;
            if (!mbar_wait(raw_full(s), (kt / RS) & 1, fail, err)) { ok = false; break; }
            if (kt >= CS && !mbar_wait(op_empty(cs), ((kt / CS) & 1) ^ 1, fail, err)) { ok = false; break; }
            const unsigned char *ra = sm + OFF_RAW + s * RAW_STAGE;
            const float *rb = reinterpret_cast<const float *>(ra + RAW_A);
            unsigned char *pre = sm + OFF_OP + cs * OP_STAGE, *pim = pre + PL_A, *pbm = pre + 2 * PL_A;
            // items: A rows (128 rows x 2 halves of 8 complex k), then B rows (240 real
            // columns x 2 halves); term j of a half goes to 16-B chunk 2j + h of its row
            for (int it = w; it < 2 * TM + 2 * 2 * TN; it += NWT) {
                if (it < 2 * TM) {
                    const int r = it & (TM - 1), h = it / TM;
                    float re[8], im[8];
#pragma unroll
                    for (int qq = 0; qq < 4; qq++) {
                        const float4 v = *reinterpret_cast<const float4 *>(ra + swz(r, 4 * h + qq));
                        re[2 * qq] = v.x;
                        im[2 * qq] = v.y;
                        re[2 * qq + 1] = v.z;
                        im[2 * qq + 1] = v.w;
                    }
                    uint4 tr[3], ti[3];
                    split8_bf16x3(re, tr);
                    split8_bf16x3(im, ti);
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        *reinterpret_cast<uint4 *>(pre + swz(r, 2 * j + h)) = tr[j];
                        *reinterpret_cast<uint4 *>(pim + swz(r, 2 * j + h)) = ti[j];
                    }
                } else {
                    const int i2 = it - 2 * TM, jr = i2 % (2 * TN), h = i2 / (2 * TN);
                    float x[8];
#pragma unroll
                    for (int i = 0; i < 8; i++) x[i] = rb[(8 * h + i) * (2 * TN) + jr];
                    uint4 tb[3];
                    split8_bf16x3(x, tb);
#pragma unroll
                    for (int j = 0; j < 3; j++) *reinterpret_cast<uint4 *>(pbm + swz(jr, 2 * j + h)) = tb[j];
                }
            }
            fence_proxy_async();                                  // generic writes -> tensor core reads
            mbar_arrive(raw_empty(s));
            mbar_arrive(op_full(cs));
            // with the first stage of chunk c already converted, read chunk c - 1 out
            if (kt > 0 && (kt % KCS) == 0) drain(kt / KCS - 1);
        }
        if (ok) drain(nchunk - 1);
        ok = ok && !*fail;
        // C -= P for this thread's row and CPW complex columns
        const int row = m0 + 32 * q + lane, c0 = n0 + CPW * g;
        if (ok && row < m && c0 < nc) {
            float2 *crow = C + (long long)b * stride + (long long)row * ldc + c0;
            if (c0 + CPW <= nc) {
                float4 *cp = reinterpret_cast<float4 *>(crow);
#pragma unroll
                for (int h = 0; h < CPW / 2; h++) {
                    float4 v = cp[h];
                    v.x -= part[2 * h].x;
                    v.y -= part[2 * h].y;
                    v.z -= part[2 * h + 1].x;
                    v.w -= part[2 * h + 1].y;
                    cp[h] = v;
                }
            } else {
#pragma unroll
                for (int j = 0; j < CPW; j++)
                    if (c0 + j < nc) {
                        crow[j].x -= part[j].x;
                        crow[j].y -= part[j].y;
                    }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS)
                     : "memory");
    }
}

typedef CUresult (*encode_fn_t)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver this process runs on (no link-time libcuda).
encode_fn_t encode_tiled()
{
    static const encode_fn_t fn = []() -> encode_fn_t {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<encode_fn_t>(p);
    }();
    return fn;
}

// 3-D FP32 tensor map {inner floats, rows, batch} over a row-major complex matrix view.
int make_map(CUtensorMap *tm, const float2 *base, int rows, int cols, int ld, long long stride, int nb,
             uint32_t box_inner, uint32_t box_rows, CUtensorMapSwizzle swz_mode)
{
    const cuuint64_t dim[3] = {(cuuint64_t)2 * cols, (cuuint64_t)rows, (cuuint64_t)nb};
    const long long bstride = nb > 1 ? stride : (long long)ld * rows;
    const cuuint64_t gstride[2] = {(cuuint64_t)ld * 8, (cuuint64_t)bstride * 8};
    const cuuint32_t box[3] = {box_inner, box_rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode_tiled()(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float2 *>(base), dim,
                                      gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz_mode,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        pb_set_error("cuTensorMapEncodeTiled failed (%d) for a %d x %d complex operand", (int)r, rows, cols);
        return PB_ERR_CUDA;
    }
    return PB_OK;
}

std::atomic<unsigned long long> g_tc_attr{0};

}  // namespace

bool pb_cgemm_tc_ok(const float2 *A, int lda, const float2 *B, int ldb, const float2 *C, int ldc,
                    long long stride, int nb)
{
    auto al16 = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    if (!al16(A) || !al16(B) || !al16(C)) return false;
    if ((lda & 1) || (ldb & 1) || (ldc & 1)) return false;     // row strides multiples of 16 B
    if (nb > 1 && (stride & 1)) return false;                  // batch stride likewise
    return encode_tiled() != nullptr;
}

int pb_cgemm_tc(int m, int nc, int k, const float2 *A, int lda, const float2 *B, int ldb, float2 *C, int ldc,
                long long stride, int nb, int *err, cudaStream_t s, int lower)
{
    if (m <= 0 || nc <= 0 || k <= 0 || nb <= 0) return PB_OK;
    // the TMA boxes (128 rows of A, 128 complex columns of B, 16 of k) stay within the
    // operand extents; smaller updates belong to the SIMT kernel
    if (m < TM || nc < TN || k < TK || nb > 65535 || !pb_cgemm_tc_ok(A, lda, B, ldb, C, ldc, stride, nb)) {
        pb_set_error("pb_cgemm_tc: unsupported update %d x %d x %d", m, nc, k);
        return PB_ERR_UNSUP;
    }
    CUtensorMap ta, tb;
    PB_TRY(make_map(&ta, A, m, k, lda, stride, nb, 2 * TK, TM, CU_TENSOR_MAP_SWIZZLE_128B));
    PB_TRY(make_map(&tb, B, k, nc, ldb, stride, nb, 2 * TN, TK, CU_TENSOR_MAP_SWIZZLE_NONE));
    PB_TRY(pb_smem_optin(k_cgemm_tc, SMEM_BYTES, g_tc_attr));
    const dim3 grid(ceil_div(nc, TN), ceil_div(m, TM), nb);
    k_cgemm_tc<<<grid, NTHREADS, SMEM_BYTES, s>>>(ta, tb, C, ldc, stride, m, nc, k, err, lower);
    PB_CHECK_LAUNCH();
    return PB_OK;
}
