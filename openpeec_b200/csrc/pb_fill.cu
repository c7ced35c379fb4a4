// pb_fill.cu — partial-inductance (Lp) and potential-coefficient (P) fill kernels.
//
// Each matrix entry is split as the reference splits it (partial.c:256-317):
//   I = I_static + sum (e^{-jkR} - 1)/R   (singularity extraction).
// * Static part: FP64, one thread per entry (k_lp_static / k_pot_static), evaluated
//   once per quadrature level and cached across the frequency sweep.
// * Retardation correction: one warp per entry; the 32 lanes split the quadrature
//   samples; each sample's R is computed once and reused for up to 16 wavenumbers of
//   the sweep (per-lane accumulators, one per frequency). FP32 in the mixed path, FP64
//   in the plain path. The integrand is evaluated as
//       (e^{-jkR} - 1)/R = -(2 sin(kR/2)/R) * (sin(kR/2) + j cos(kR/2)),
//   which has no cancellation (the reference's cos(kR)-1, partial.c:168, would lose all
//   digits in FP32 for small kR).
// * FP32 phase: R = D + delta with D = |centre offset| of the term (FP64, once per term)
//   and delta = (R^2 - D^2) / (R + D) formed in FP32 from the small in-cell offset p, so
//   the error of delta scales with the cell size, not with the distance. sin/cos(kD/2)
//   come from FP64 once per term and frequency group; each sample only rotates them by
//   the small angle k delta / 2. The sample loop has no FP64 arithmetic.
// * Epilogue: store Lp / P, or assemble the reduced MNA matrix directly.
#include <atomic>
#include "pb_fill.cuh"
#include "pb_geom.cuh"
#include <vector>

template <typename R> __device__ __forceinline__ R XG4(int i);
template <> __device__ __forceinline__ float XG4<float>(int i) { return (float)cXG4[i]; }
template <> __device__ __forceinline__ double XG4<double>(int i) { return cXG4[i]; }
template <typename R> __device__ __forceinline__ R WG4(int i);
template <> __device__ __forceinline__ float WG4<float>(int i) { return (float)cWG4[i]; }
template <> __device__ __forceinline__ double WG4<double>(int i) { return cWG4[i]; }
template <typename R> __device__ __forceinline__ R XG8(int i);
template <> __device__ __forceinline__ float XG8<float>(int i) { return (float)cXG8[i]; }
template <> __device__ __forceinline__ double XG8<double>(int i) { return cXG8[i]; }
template <typename R> __device__ __forceinline__ R WG8(int i);
template <> __device__ __forceinline__ float WG8<float>(int i) { return (float)cWG8[i]; }
template <> __device__ __forceinline__ double WG8<double>(int i) { return cWG8[i]; }

// Wavenumbers of one launch. kh[f] = k_f / 2 (the integrand is written in kR/2).
// eq = 1 when the k_f are equally spaced (linear sweeps): then the FP32 path advances
// sin/cos(k_f R/2) from frequency to frequency by angle addition instead of evaluating
// them anew, re-seeding every 8 frequencies.
struct KArg {
    double kw[PB_FMAX];
    double kh[PB_FMAX];
    double dkh;
    double kwmax;        // largest wavenumber of the launch
    float khf[PB_FMAX];
    float dkhf;
    int nf, eq;
    int reduce;          // kh * (bound on |delta|) may exceed pi/4: reduce the FP32 angles
    int step_tiny;       // |dkh| * (bound on |delta|) < 0.01: two-term step sine/cosine
};                       // (selects the RED instance of the FP32 kernels)

// 3-point Gauss-Legendre rule (nodes 0, +-sqrt(3/5); weights 8/9, 5/9) for separated
// ribbon pairs on the FP32 path; the nodes in FP32, the weights in FP64.
__constant__ float cXG3f[3] = {-0.7745966692414834f, 0.0f, 0.7745966692414834f};
__constant__ double cWG3[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
// FP32 copies of the 4- and 8-point Gauss-Legendre nodes and weights (the FP64 tables
// cXG4/cWG4/cXG8/cWG8 rounded to nearest), for uniform loads in the FP32 sample loops.
__constant__ float cXG4f[4] = {-0.8611363115940526f, -0.3399810435848563f, 0.3399810435848563f, 0.8611363115940526f};
__constant__ float cWG4f[4] = {0.3478548451374538f, 0.6521451548625461f, 0.6521451548625461f, 0.3478548451374538f};
// cWG4 - cWG4f: the weights' FP32 rounding is the same for every sample of every term and
// would bias the quadrature (~2e-8 relative), so products carry the tail explicitly.
__constant__ float cWG4lo[4] = {-7.538937474e-09f, 7.538937474e-09f, 7.538937474e-09f, -7.538937474e-09f};

// sin and cos of an FP32 angle: optional Cody-Waite reduction by pi/2 (pi/2 split into
// an FP32 head and tail, so q * head is exact inside the FMA), then the Taylor series of
// sin to x^9 and cos to x^8 on |t| <= pi/4 (truncation below 2e-9).
template <int RED>
__device__ __forceinline__ void sincos_f32(float x, float &s, float &c)
{
    float t = x;
    int iq = 0;
    if (RED) {
        const float q = rintf(x * 0.636619772f);
        t = fmaf(-q, 1.57079637f, x);
        t = fmaf(-q, -4.37113883e-8f, t);
        iq = (int)q;
    }
    const float r2 = t * t;
    float ps = fmaf(r2, 2.75573192e-6f, -1.98412698e-4f);
    ps = fmaf(ps, r2, 8.33333333e-3f);
    ps = fmaf(ps, r2, -1.66666667e-1f);
    const float sn = fmaf(ps * r2, t, t);
    float pc = fmaf(r2, 2.48015873e-5f, -1.38888889e-3f);
    pc = fmaf(pc, r2, 4.16666667e-2f);
    pc = fmaf(pc, r2, -0.5f);
    const float cs = fmaf(pc, r2, 1.0f);
    const float ss = (iq & 1) ? cs : sn, cc = (iq & 1) ? sn : cs;
    s = (iq & 2) ? -ss : ss;
    c = ((iq + 1) & 2) ? -cc : cc;
}

// Accumulators of one lane for F wavenumbers.
// FP32 path: FP32 partial sums in registers, flushed every PB_FLUSH samples into this lane's
// FP64 totals kept in shared memory (tot[(2f + c) * 32], conflict-free across lanes), which
// bounds the FP32 summation error without holding 2F doubles in registers.
// FP64 path: FP64 sums in registers.
#define PB_FLUSH 16
template <typename R, int F> struct Acc;
template <int F> struct Acc<float, F> {
    float pr[F], pi[F];
    double *tot;
    int cnt;
    __device__ __forceinline__ void init(double *slot)
    {
        tot = slot;
#pragma unroll
        for (int f = 0; f < F; f++) { pr[f] = pi[f] = 0.f; tot[(2 * f) * 32] = 0.0; tot[(2 * f + 1) * 32] = 0.0; }
        cnt = 0;
    }
    __device__ __forceinline__ void flush()
    {
#pragma unroll
        for (int f = 0; f < F; f++) {
            tot[(2 * f) * 32] += (double)pr[f];
            tot[(2 * f + 1) * 32] += (double)pi[f];
            pr[f] = pi[f] = 0.f;
        }
        cnt = 0;
    }
    __device__ __forceinline__ double re(int f) const { return tot[(2 * f) * 32]; }
    __device__ __forceinline__ double im(int f) const { return tot[(2 * f + 1) * 32]; }
};
template <int F> struct Acc<double, F> {
    double tr[F], ti[F];
    __device__ __forceinline__ void init(double *)
    {
#pragma unroll
        for (int f = 0; f < F; f++) tr[f] = ti[f] = 0.0;
    }
    __device__ __forceinline__ void flush() {}
    __device__ __forceinline__ double re(int f) const { return tr[f]; }
    __device__ __forceinline__ double im(int f) const { return ti[f]; }
};

// Per-term phase bases of the FP32 path (shared memory of the warp): EQ launches hold
// sin/cos(kh[8g] D) for the groups g < F/8 and sin/cos(dkh D) after them; other launches
// hold sin/cos(kh[f] D) for every f < F. Each base is an FP32 head + tail pair
// (sin_hi, cos_hi, sin_lo, cos_lo): its rounding would otherwise be the same for every
// sample of the term and not average out.
template <int F, int EQ> constexpr int nbase() { return EQ ? (F + 7) / 8 + 1 : F; }

// sin/cos(A + B) from the head+tail base b = sin/cos(A) and FP32 sB, cB of a small B.
__device__ __forceinline__ void rot_base(const float4 b, float sB, float cB, float &s, float &c)
{
    s = fmaf(b.x, cB, fmaf(b.y, sB, fmaf(b.w, sB, b.z)));
    c = fmaf(b.y, cB, fmaf(-b.x, sB, fmaf(-b.z, sB, b.w)));
}

// Accumulate one FP32 sample for every wavenumber: distance R = D + dl with weight
// factor qw = -2 w (w = quadrature weight x term scale), q = qw / R:
//   (e^{-jkR}-1)/R = q sin(kR/2) (sin(kR/2) + j cos(kR/2)),  R -> 0 limit -jk.
template <int F, int EQ, int RED>
__device__ __forceinline__ void accum32(Acc<float, F> &a, const KArg &k, const float4 *base,
                                        float r2, float rinv, float dl, float qw)
{
    if (r2 > 0) {
        const float q = qw * rinv;
        if (EQ) {
            constexpr int NG = (F + 7) / 8;
            float ss, cs;
            if (k.step_tiny) {                     // |x| < 0.01: x^5/120 and x^4/24 < 1e-11
                const float x = k.dkhf * dl, x2 = x * x;
                ss = fmaf(x2 * x, -0.166666667f, x);
                cs = fmaf(x2, -0.5f, 1.f);
            } else {
                sincos_f32<RED>(k.dkhf * dl, ss, cs);
            }
            float sd, cd;
            rot_base(base[NG], ss, cs, sd, cd);
#pragma unroll
            for (int g = 0; g < NG; g++) {
                float ts, tc;
                sincos_f32<RED>(k.khf[8 * g] * dl, ts, tc);
                float s, c;
                rot_base(base[g], ts, tc, s, c);
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int f = 8 * g + u;
                    if (f < F) {
                        const float t = q * s;
                        a.pr[f] = fmaf(t, s, a.pr[f]);
                        a.pi[f] = fmaf(t, c, a.pi[f]);
                        const float s2 = fmaf(s, cd, c * sd);
                        c = fmaf(c, cd, -(s * sd));
                        s = s2;
                    }
                }
            }
        } else {
#pragma unroll
            for (int f = 0; f < F; f++) {
                float ts, tc;
                sincos_f32<RED>(k.khf[f] * dl, ts, tc);
                float s, c;
                rot_base(base[f], ts, tc, s, c);
                const float t = q * s;
                a.pr[f] = fmaf(t, s, a.pr[f]);
                a.pi[f] = fmaf(t, c, a.pi[f]);
            }
        }
    } else {
#pragma unroll
        for (int f = 0; f < F; f++) a.pi[f] = fmaf(qw, k.khf[f], a.pi[f]);
    }
    if (++a.cnt == PB_FLUSH) a.flush();
}

// A sample whose two points nearly coincide (R < D / 32: overlapping cells, e.g. the
// crossing current cells of a quad panel): the phase kh R is formed from the direct FP32
// R per frequency. Rotating the term's bases by kh dl there (dl = R - D ~ -D) leaves an
// absolute phase error ~kh D 1e-7 against a phase of only kh R, and sin(kh R) / R takes
// that error relative to R (it was 1e8 times the entry on a quad panel of config 5).
template <int F>
__device__ __forceinline__ void accum32_near(Acc<float, F> &a, const KArg &k, float r2, float ra, float qw)
{
    if (r2 > 0) {
        const float q = __fdividef(qw, ra);
#pragma unroll
        for (int f = 0; f < F; f++) {
            float s, c;
            sincos_f32<1>(k.khf[f] * ra, s, c);
            const float t = q * s;
            a.pr[f] = fmaf(t, s, a.pr[f]);
            a.pi[f] = fmaf(t, c, a.pi[f]);
        }
    } else {
#pragma unroll
        for (int f = 0; f < F; f++) a.pi[f] = fmaf(qw, k.khf[f], a.pi[f]);
    }
    if (++a.cnt == PB_FLUSH) a.flush();
}

// One sample of the FP32 path from its in-cell offset p (R = |cd + p|, plus the wire
// kernel's a^2): dl = R - D = p.(p + 2 cd) / (R + D) with R + D from R^2 in FP32
// (v = cd + p), then R = D + dl with D as FP32 head + tail, so that 1/R carries no
// rounding shared by all samples of the term. Where D + dl cancels (a sample next to
// the other cell of an adjacent pair) the direct FP32 R is taken instead, and where the
// two points nearly coincide the phase too (accum32_near).
template <int F, int EQ, int RED>
__device__ __forceinline__ void sample32(Acc<float, F> &a, const KArg &k, const float4 *base,
                                         const float *cd, float a2, float D, float Dlo, float px,
                                         float py, float pz, float qw)
{
    const float vx = cd[0] + px, vy = cd[1] + py, vz = cd[2] + pz;
    const float r2 = fmaf(vx, vx, fmaf(vy, vy, fmaf(vz, vz, a2)));
    const float e = fmaf(px, fmaf(2.f, cd[0], px), fmaf(py, fmaf(2.f, cd[1], py), pz * fmaf(2.f, cd[2], pz)));
    const float ra = r2 * rsqrtf(r2);
    if (!(ra >= 0.03125f * D)) {                  // also r2 = 0 (ra is then NaN)
        accum32_near<F>(a, k, r2, r2 > 0 ? ra : 0.f, qw);
        return;
    }
    const float dl = __fdividef(e, ra + D);
    const float rd = D + (dl + Dlo);
    const float r = rd > 0.5f * ra ? rd : ra;
    float rinv = __fdividef(1.f, r);
    rinv = fmaf(rinv, fmaf(-r, rinv, 1.f), rinv);
    accum32<F, EQ, RED>(a, k, base, r2, rinv, dl, qw);
}

template <int F, int EQ>
__device__ __forceinline__ void accum(Acc<double, F> &a, const KArg &k, double r, double rinv, double w)
{
    (void)rinv;
    if (r > 0) {
        const double q = -2 * w / r;
#pragma unroll
        for (int f = 0; f < F; f++) {
            if (f < k.nf) {
                double s, c;
                sincos(k.kh[f] * r, &s, &c);
                const double t = q * s;
                a.tr[f] = fma(t, s, a.tr[f]);
                a.ti[f] = fma(t, c, a.ti[f]);
            }
        }
    } else {
#pragma unroll
        for (int f = 0; f < F; f++)
            if (f < k.nf) a.ti[f] -= 2 * w * k.kh[f];
    }
}

// One (possibly mirrored) pair term reduced to what its sample loop needs, in the
// precision of that loop. Built from the FP64 cells just before the loop so that the
// cells are not live during it.
enum { TT_RIBBON = 0, TT_WIRE = 1, TT_POLY = 2, TT_RIBBON2 = 3, TT_RIBBON3 = 4, TT_WIRE48 = 5 };

// Separated wire pairs on the FP32 path: centre distance >= PB_WFAR_RATIO lmax and
// k lmax <= PB_WFAR_KL at every wavenumber of the launch. There the reference's rule
// (gauss_kernel mode 1: nsub = 2 + k lmax sub-intervals per segment, 8 Gauss-Legendre
// points in each, 256 samples at nsub = 2) is replaced by 4 points along the whole first
// segment and 8 along the whole second (32 samples, one per lane). On the smooth far
// integrand the difference is below 1e-9 of the entry, orders under the FP32 rounding of
// the correction (measured against the reference's rule in tests/test_far_rules.py).
#define PB_WFAR_RATIO 3.0
#define PB_WFAR_KL 0.5
__device__ __forceinline__ bool wire_far32(const Cell &s1, const Cell &s2, double kwmax)
{
    const double lmax = fmax(s1.len, s2.len);
    if (!(kwmax * lmax <= PB_WFAR_KL)) return false;
    double d2 = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const double d = 0.5 * (s2.x1[c] + s2.x2[c]) - 0.5 * (s1.x1[c] + s1.x2[c]);
        d2 += d * d;
    }
    return d2 >= (PB_WFAR_RATIO * lmax) * (PB_WFAR_RATIO * lmax);
}

// Separated ribbon pairs on the FP32 path: a single sub-square (nsub = 1) and k * lmax <=
// PB_FAR_KL at every wavenumber of the launch (lmax: the largest cell dimension). There
// the correction integrand (e^{-jkR}-1)/R is smooth over both cells, and lower-order
// Gauss-Legendre product rules than the reference's 4-point rule (256 samples) agree with
// it to far below the FP32 rounding of the correction:
//   centre distance >= PB_FAR2_RATIO lmax: 2-point rule (16 samples),
//   centre distance >= PB_FAR3_RATIO lmax: 3-point rule (81 samples).
// Measured on the benchmark plate at k lmax = 0.1 (parallel pairs, direct and image,
// relative to |static| + |correction|): 2-point <= 6.7e-8 at ratio 8-10 (remainder
// ~(k lmax)^4 / 1000); 3-point <= 2.6e-9 at ratio 3-4, 7e-10 at 4-5. Without the k lmax
// bound a coarser plate at k lmax = 0.225 erred by 2.6e-6 with the 2-point rule. The FP64
// (plain) path keeps the reference's 4-point rule everywhere.
#define PB_FAR2_RATIO 10.0
#define PB_FAR3_RATIO 3.0
// 4 (the reference's rule), 3 or 2: the product rule of a ribbon pair on the FP32 path
__device__ __forceinline__ int ribbon_rule32(const Cell &s1, const Cell &s2, int nsub, const double *c1,
                                             const double *c2, double kwmax)
{
    if (nsub != 1) return 4;
    const double lmax = fmax(fmax(s1.len, s2.len), fmax(s1.wid, s2.wid));
    if (kwmax * lmax > PB_FAR_KL) return 4;
    const double dx = c2[0] - c1[0], dy = c2[1] - c1[1], dz = c2[2] - c1[2];
    const double d2 = dx * dx + dy * dy + dz * dz;
    if (d2 >= (PB_FAR2_RATIO * lmax) * (PB_FAR2_RATIO * lmax)) return 2;
    if (d2 >= (PB_FAR3_RATIO * lmax) * (PB_FAR3_RATIO * lmax)) return 3;
    return 4;
}
// Centre offset of a term in the form its sample loop reads it.
template <typename R> struct TermOffset;
template <> struct TermOffset<double> {
    double cd[3];                 // centre (or start-point) offset
    double a2;                    // equivalent radius squared (wire kernel)
};
template <> struct TermOffset<float> {
    double D;                     // sqrt(|cd|^2 + a2), FP64: the term's phase kh * D
    float cdf[3], a2f, Df, Dlo, inv_rn;   // D = Df + Dlo
};
// bases of an FP32 term for EQ launches (sin/cos of kh[0], kh[8] and dkh times D), formed
// in the set-up by the term's own lane; an empty base for FP64 terms
#define PB_TBASE 3
template <typename R> struct TermBases {};
template <> struct TermBases<float> {
    float4 tb[PB_TBASE];
};
// 192 bytes for FP32 (a multiple of 16 without padding: three warps' groups of terms and
// totals fit five CTAs per SM)
template <typename R> struct Term : TermBases<R>, TermOffset<R> {
    int ty, nsub, n1, n2;
    double sc;                    // folded scale (term weight x quadrature Jacobian)
    R u1[3], v1[3], u2[3], v2[3];
    R L1, W1, L2, W2, zs;
    int qo1, qo2;                 // polygon point sets: offsets into the set's qpt
};
static_assert(sizeof(Term<float>) == 192, "FP32 term record layout");

// Quadrature choice and geometry of neumann_pair_k's retardation term
// (partial.c:256-317, neumann_self_k partial.c:320-328).
template <typename R>
__device__ void make_term(Term<R> &T, const Cell &s1, const Cell &s2, int same, double a1, double a2,
                          double scale, double kw0, double kwmax, const pb_dev_cells &set, int i1, int i2)
{
    int ty;
    const bool wire_self = same && s1.wid <= 0 && s1.npv <= 0;
    if (wire_self) ty = PT_WIRE;
    else ty = pair_type(s1, s2);
    double cdl[3], a2l = 0;
    if (ty == PT_POLY) {                                   // poly_corr, polygon.c:305-334
        T.ty = TT_POLY;
        T.qo1 = set.qoff[i1];
        T.n1 = set.qoff[i1 + 1] - set.qoff[i1];
        T.qo2 = set.qoff[i2];
        T.n2 = set.qoff[i2 + 1] - set.qoff[i2];
#pragma unroll
        for (int c = 0; c < 3; c++) cdl[c] = 0.5 * (s2.x1[c] + s2.x2[c]) - 0.5 * (s1.x1[c] + s1.x2[c]);
        T.zs = s2.mirror ? (R)-1 : (R)1;
        const double w1 = (s1.wid > 0) ? s1.wid : 1, w2 = (s2.wid > 0) ? s2.wid : 1;
        T.sc = scale / (w1 * w2);
        T.nsub = 1;
    } else if (ty == PT_HL || ty == PT_RIBBON) {           // ribbon_corr, surface.c:134-178
        T.ty = TT_RIBBON;
        const int nsub = ribbon_nsub(s1, s2, kw0);
        double t1d[3], w1d[3], n1d[3], c1d[3], t2d[3], w2d[3], n2d[3], c2d[3];
        frame(s1, t1d, w1d, n1d, c1d);
        frame(s2, t2d, w2d, n2d, c2d);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            T.u1[c] = (R)t1d[c]; T.v1[c] = (R)w1d[c]; T.u2[c] = (R)t2d[c]; T.v2[c] = (R)w2d[c];
            cdl[c] = c2d[c] - c1d[c];
        }
        T.L1 = (R)s1.len; T.W1 = (R)s1.wid; T.L2 = (R)s2.len; T.W2 = (R)s2.wid;
        T.sc = scale * s1.len * s2.len / (16.0 * nsub * nsub);   // any product rule: weights sum to 16
        T.nsub = nsub;
        if constexpr (sizeof(R) == 4) {
            const int rule = ribbon_rule32(s1, s2, nsub, c1d, c2d, kwmax);
            if (rule == 2) T.ty = TT_RIBBON2;
            if (rule == 3) T.ty = TT_RIBBON3;
        }
    } else {                                               // gauss_kernel mode 1, partial.c:61-99
        T.ty = TT_WIRE;
        const Cell &b = wire_self ? s1 : s2;
        const double aeff = wire_self ? a1 : 0.5 * (a1 + a2);
        const int nsub = corr_nsub(s1, b, kw0);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            T.u1[c] = (R)(s1.x2[c] - s1.x1[c]);
            T.u2[c] = (R)(b.x2[c] - b.x1[c]);
            cdl[c] = b.x1[c] - s1.x1[c];
        }
        a2l = aeff * aeff;
        T.sc = scale * s1.len * b.len * 0.25 / ((double)nsub * nsub);
        T.nsub = nsub;
        if constexpr (sizeof(R) == 4) {
            if (!wire_self && wire_far32(s1, b, kwmax)) {      // 4 x 8 points, no sub-intervals
                T.ty = TT_WIRE48;
                T.sc = scale * s1.len * b.len * 0.25;           // weights sum to 4 as well
                T.nsub = 1;
            }
        }
    }
    if constexpr (sizeof(R) == 4) {
        T.D = sqrt(cdl[0] * cdl[0] + cdl[1] * cdl[1] + cdl[2] * cdl[2] + a2l);
#pragma unroll
        for (int c = 0; c < 3; c++) T.cdf[c] = (float)cdl[c];
        T.a2f = (float)a2l;
        T.Df = (float)T.D;
        T.Dlo = (float)(T.D - (double)T.Df);
        T.inv_rn = 1.0f / (float)T.nsub;
    } else {
#pragma unroll
        for (int c = 0; c < 3; c++) T.cd[c] = cdl[c];
        T.a2 = a2l;
    }
}

// Distance of one sample of the FP64 path.
__device__ __forceinline__ double dist64(const double *cd, const double *p, double a2, double &rinv)
{
    const double dx = cd[0] + p[0], dy = cd[1] + p[1], dz = cd[2] + p[2];
    rinv = 0;
    return sqrt(dx * dx + dy * dy + dz * dz + a2);
}

template <typename R, int F, int EQ>
__device__ void run_term(const Term<R> &T, const KArg &k, Acc<R, F> &a, int lane, const double4 *qpt)
{
    const int nsub = T.nsub;
    const R rn = (R)nsub;
    if (T.ty == TT_RIBBON) {
        for (int sq = 0; sq < nsub * nsub; sq++) {
            const int ia = sq / nsub, ja = sq - ia * nsub;
            for (int s = lane; s < 256; s += 32) {
                const int q = s & 3, m = (s >> 2) & 3, j = (s >> 4) & 3, i = (s >> 6) & 3;
                const R a1 = T.L1 * ((ia + (R)0.5 * (1 + XG4<R>(i))) / rn - (R)0.5);
                const R b1 = T.W1 * ((R)0.5 * (1 + XG4<R>(j)) - (R)0.5);
                const R a2 = T.L2 * ((ja + (R)0.5 * (1 + XG4<R>(m))) / rn - (R)0.5);
                const R b2 = T.W2 * ((R)0.5 * (1 + XG4<R>(q)) - (R)0.5);
                R p[3];
#pragma unroll
                for (int c = 0; c < 3; c++) p[c] = (a2 * T.u2[c] + b2 * T.v2[c]) - (a1 * T.u1[c] + b1 * T.v1[c]);
                double ri;
                const double rd = dist64(T.cd, p, 0.0, ri);
                accum<F, EQ>(a, k, rd, ri, cWG4[i] * cWG4[j] * cWG4[m] * cWG4[q] * T.sc);
            }
        }
    } else if (T.ty == TT_WIRE) {
        for (int sq = 0; sq < nsub * nsub; sq++) {
            const int i1 = sq / nsub, i2 = sq - i1 * nsub;
            for (int s = lane; s < 64; s += 32) {
                const int j = s & 7, i = (s >> 3) & 7;
                const R u = (i1 + (R)0.5 * (1 + XG8<R>(i))) / rn;
                const R v = (i2 + (R)0.5 * (1 + XG8<R>(j))) / rn;
                R p[3];
#pragma unroll
                for (int c = 0; c < 3; c++) p[c] = T.u2[c] * v - T.u1[c] * u;
                double ri;
                const double rd = dist64(T.cd, p, T.a2, ri);
                accum<F, EQ>(a, k, rd, ri, cWG8[i] * cWG8[j] * T.sc);
            }
        }
    } else {
        const int S = T.n1 * T.n2;
        for (int s = lane; s < S; s += 32) {
            const int k1 = s / T.n2, k2 = s - k1 * T.n2;
            const double4 o1 = qpt[T.qo1 + k1], o2 = qpt[T.qo2 + k2];
            R p[3];
            p[0] = (R)o2.x - (R)o1.x;
            p[1] = (R)o2.y - (R)o1.y;
            p[2] = T.zs * (R)o2.z - (R)o1.z;
            double ri;
            const double rd = dist64(T.cd, p, 0.0, ri);
            accum<F, EQ>(a, k, rd, ri, o1.w * o2.w * T.sc);
        }
    }
}

// Samples of one term on the FP32 path. Lane l takes the same quadrature points as the
// FP64 path (sample s = l + 32 t of each sub-square), but with the lane-fixed parts of the
// point (and of its weight) hoisted out of the loops; the phase bases sin/cos(kh D) of the
// term are computed in FP64 by the first lanes into the warp's `base` slots.
template <int F, int EQ, int RED, bool HAS2>
__device__ void run_term32(const Term<float> &T, const KArg &k, Acc<float, F> &a, int lane,
                           float4 *bases, const double4 *qpt)
{
    constexpr int NB = nbase<F, EQ>();
    // EQ launches: the term's bases were formed in the set-up (T.tb); otherwise here
    const float4 *base = T.tb;
    if (!EQ) {
        __syncwarp();                               // previous term's bases no longer read
        if (lane < NB) {
            double sn, cs;
            sincos(k.kh[lane] * T.D, &sn, &cs);
            const float sh = (float)sn, ch = (float)cs;
            bases[lane] = make_float4(sh, ch, (float)(sn - (double)sh), (float)(cs - (double)ch));
        }
        __syncwarp();
        base = bases;
    }
    const float cd[3] = {T.cdf[0], T.cdf[1], T.cdf[2]};
    const float D = T.Df, Dlo = T.Dlo, irn = T.inv_rn;
    const int nsub = T.nsub;
    if (T.ty == TT_RIBBON) {                        // ribbon_corr, surface.c:134-178
        // sample s = lane + 32 t: q = lane&3, m = (lane>>2)&3, j = (lane>>4) + 2 (t&1), i = t>>1
        const int lq = lane & 3, lm = (lane >> 2) & 3, lj = lane >> 4;
        const float b2 = T.W2 * 0.5f * cXG4f[lq];
        const float hm = 0.5f * (1.f + cXG4f[lm]);
        const float b10 = T.W1 * 0.5f * cXG4f[lj], b11 = T.W1 * 0.5f * cXG4f[lj + 2];
        const double wqm = cWG4[lq] * cWG4[lm] * (-2.0 * T.sc);
        const double wl0d = cWG4[lj] * wqm, wl1d = cWG4[lj + 2] * wqm;
        const float wl0 = (float)wl0d, wl1 = (float)wl1d;             // head + tail
        const float wl0t = (float)(wl0d - (double)wl0), wl1t = (float)(wl1d - (double)wl1);
        float B2[3], B10[3], B11[3], U1[3], U2[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            B2[c] = b2 * T.v2[c];
            B10[c] = b10 * T.v1[c];
            B11[c] = b11 * T.v1[c];
            U1[c] = T.u1[c];
            U2[c] = T.u2[c];
        }
        const float L1 = T.L1, L2 = T.L2;
        for (int ja = 0; ja < nsub; ja++) {
            const float a2c = L2 * fmaf((float)ja + hm, irn, -0.5f);
            float Q0[3], Q1[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float P2 = fmaf(a2c, U2[c], B2[c]);
                Q0[c] = P2 - B10[c];
                Q1[c] = P2 - B11[c];
            }
            for (int ia = 0; ia < nsub; ia++) {
#pragma unroll 1
                for (int i = 0; i < 4; i++) {
                    const float a1 = L1 * fmaf((float)ia + 0.5f * (1.f + cXG4f[i]), irn, -0.5f);
                    const float wi = cWG4f[i], wit = cWG4lo[i];
                    // full weight W_i W_j W_m W_q (-2 sc) rounded once (head*head + cross terms)
                    const float w0 = fmaf(wl0, wi, fmaf(wl0, wit, wl0t * wi));
                    const float w1 = fmaf(wl1, wi, fmaf(wl1, wit, wl1t * wi));
                    sample32<F, EQ, RED>(a, k, base, cd, 0.f, D, Dlo, fmaf(-a1, U1[0], Q0[0]),
                                         fmaf(-a1, U1[1], Q0[1]), fmaf(-a1, U1[2], Q0[2]), w0);
                    sample32<F, EQ, RED>(a, k, base, cd, 0.f, D, Dlo, fmaf(-a1, U1[0], Q1[0]),
                                         fmaf(-a1, U1[1], Q1[1]), fmaf(-a1, U1[2], Q1[2]), w1);
                }
            }
        }
    } else if (HAS2 && T.ty == TT_RIBBON2) {        // well-separated ribbons: 2-point rule
        if (lane < 16) {
            const float g = 0.577350269189625765f;  // 1/sqrt(3), weights 1
            const float xi = (lane & 1) ? g : -g, xj = (lane & 2) ? g : -g;
            const float xm = (lane & 4) ? g : -g, xq = (lane & 8) ? g : -g;
            const float a1 = 0.5f * T.L1 * xi, b1 = 0.5f * T.W1 * xj, a2 = 0.5f * T.L2 * xm, b2 = 0.5f * T.W2 * xq;
            float p[3];
#pragma unroll
            for (int c = 0; c < 3; c++) p[c] = fmaf(a2, T.u2[c], fmaf(b2, T.v2[c], -fmaf(a1, T.u1[c], b1 * T.v1[c])));
            sample32<F, EQ, RED>(a, k, base, cd, 0.f, D, Dlo, p[0], p[1], p[2], (float)(-2.0 * T.sc));
        }
    } else if (T.ty == TT_RIBBON3) {                // separated ribbons: 3-point rule
        if (lane < 27) {                            // lane = i + 3 j + 9 m; q = 0..2 in the loop
            const int i = lane % 3, j = (lane / 3) % 3, m = lane / 9;
            const float a1 = 0.5f * T.L1 * cXG3f[i], b1 = 0.5f * T.W1 * cXG3f[j], a2 = 0.5f * T.L2 * cXG3f[m];
            const double wijm = cWG3[i] * cWG3[j] * cWG3[m] * (-2.0 * T.sc);
            float Q[3];
#pragma unroll
            for (int c = 0; c < 3; c++) Q[c] = fmaf(a2, T.u2[c], -fmaf(a1, T.u1[c], b1 * T.v1[c]));
#pragma unroll 1
            for (int q = 0; q < 3; q++) {
                const float b2 = 0.5f * T.W2 * cXG3f[q];
                sample32<F, EQ, RED>(a, k, base, cd, 0.f, D, Dlo, fmaf(b2, T.v2[0], Q[0]), fmaf(b2, T.v2[1], Q[1]),
                                     fmaf(b2, T.v2[2], Q[2]), (float)(wijm * cWG3[q]));
            }
        }
    } else if (T.ty == TT_WIRE || T.ty == TT_WIRE48) {
        // gauss_kernel mode 1 (partial.c:61-99): 8 x 8 points per sub-square, two samples
        // per lane; separated wires (TT_WIRE48): 4 x 8 points over the whole segments, one
        // per lane. One sample call site for both keeps the kernel's code (and its
        // instruction-cache footprint) the size it had with the reference's rule alone.
        const bool w48 = T.ty == TT_WIRE48;
        const int lj = lane & 7, li = lane >> 3;
        const float hj = 0.5f * (1.f + (float)cXG8[lj]);
        const float hi0 = 0.5f * (1.f + (w48 ? cXG4f[li] : (float)cXG8[li])), hi1 = 0.5f * (1.f + (float)cXG8[li + 4]);
        const double wj = cWG8[lj] * (-2.0 * T.sc);
        const float w0 = (float)((w48 ? cWG4[li] : cWG8[li]) * wj), w1 = (float)(cWG8[li + 4] * wj);
        const float a2 = T.a2f;
        float U1[3], U2[3];
#pragma unroll
        for (int c = 0; c < 3; c++) { U1[c] = T.u1[c]; U2[c] = T.u2[c]; }
        for (int i1 = 0; i1 < nsub; i1++) {
            const float ua = ((float)i1 + hi0) * irn, ub = ((float)i1 + hi1) * irn;
            for (int i2 = 0; i2 < nsub; i2++) {
                const float v = ((float)i2 + hj) * irn;
                const float P0 = U2[0] * v, P1 = U2[1] * v, P2 = U2[2] * v;
#pragma unroll 1
                for (int h = 0; h < (w48 ? 1 : 2); h++) {
                    const float uu = h ? ub : ua;
                    sample32<F, EQ, RED>(a, k, base, cd, a2, D, Dlo, fmaf(-U1[0], uu, P0), fmaf(-U1[1], uu, P1),
                                         fmaf(-U1[2], uu, P2), h ? w1 : w0);
                }
            }
        }
    } else {                                        // poly_corr, polygon.c:305-334
        const int S = T.n1 * T.n2;
        const double msc = -2.0 * T.sc;
        for (int s = lane; s < S; s += 32) {
            const int k1 = s / T.n2, k2 = s - k1 * T.n2;
            const double4 o1 = qpt[T.qo1 + k1], o2 = qpt[T.qo2 + k2];
            sample32<F, EQ, RED>(a, k, base, cd, 0.f, D, Dlo, (float)o2.x - (float)o1.x, (float)o2.y - (float)o1.y,
                            T.zs * (float)o2.z - (float)o1.z, (float)(o1.w * o2.w * msc));
        }
    }
}

// Warp sum of every frequency's accumulator; lane f receives frequency f.
// FP32 path: the per-lane FP64 totals already sit in shared memory (tot[(2f+c)*32 + lane]),
// so lane f adds up its frequency's 32 entries directly (no shuffles).
template <int F>
__device__ __forceinline__ void reduce_select(Acc<float, F> &a, int lane, double &cr, double &ci)
{
    a.flush();
    __syncwarp();
    cr = ci = 0;
    if (lane < F) {
        const double *base = a.tot - lane;            // this warp's tot array
#pragma unroll 8
        for (int l = 0; l < 32; l++) {
            cr += base[(2 * lane) * 32 + l];
            ci += base[(2 * lane + 1) * 32 + l];
        }
    }
    __syncwarp();
}
template <int F>
__device__ __forceinline__ void reduce_select(Acc<double, F> &a, int lane, double &cr, double &ci)
{
    cr = ci = 0;
#pragma unroll
    for (int f = 0; f < F; f++) {
        double x = a.re(f), y = a.im(f);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            x += __shfl_xor_sync(0xffffffffu, x, o);
            y += __shfl_xor_sync(0xffffffffu, y, o);
        }
        if (f == lane) { cr = x; ci = y; }
    }
}

// ---------------------------------------------------------------- static kernels
// Static part of Lp(i, j), i <= j (partial.c:392-423), as one entry.
__device__ __forceinline__ double lp_static_entry(const pb_fill_geom &g, int i, int j, double kw)
{
    const double coef = PB_MU0 / (4 * PB_PI);
    Cell si, sj, mj;
    load_cell(si, g.seg.cell, g.pv, i, 0, g.gpz);
    const double ai = g.seg.cell[i].aL, aj = g.seg.cell[j].aL;
    double t1[3], t2[3];
    tangent(si, t1);
    double v = 0;
    if (i == j) {                                   // partial.c:392-401
        v = static_term(si, si, 1, ai, ai, kw);
        if (g.gp) {
            load_cell(mj, g.seg.cell, g.pv, i, 1, g.gpz);
            const double tdm = t1[0] * t1[0] + t1[1] * t1[1] - t1[2] * t1[2];
            v -= tdm * static_term(si, mj, 0, ai, ai, kw);
        }
    } else {                                        // partial.c:403-423
        load_cell(sj, g.seg.cell, g.pv, j, 0, g.gpz);
        tangent(sj, t2);
        const double tdot = dot3(t1, t2);
        const double tdm = t1[0] * t2[0] + t1[1] * t2[1] - t1[2] * t2[2];
        if (tdot != 0) v = tdot * static_term(si, sj, 0, ai, aj, kw);
        if (g.gp && tdm != 0) {
            load_cell(mj, g.seg.cell, g.pv, j, 1, g.gpz);
            v -= tdm * static_term(si, mj, 0, ai, aj, kw);
        }
    }
    return coef * v;
}

__global__ void __launch_bounds__(128)
k_lp_static(pb_fill_geom g, double kw, double *st)
{
    const int n = g.seg.n;
    const long long T = (long long)n * (n + 1) / 2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < T;
         t += (long long)gridDim.x * blockDim.x) {
        int i, j;
        tri_index(t, n, i, j);
        st[(long long)i * n + j] = lp_static_entry(g, i, j, kw);
    }
}

// the static part of a pair list: stl[t] = static Lp(min, max of pairs[t]) for every t, or
// for t = idx[u] only
__global__ void __launch_bounds__(128)
k_lp_static_list(pb_fill_geom g, double kw, const int2 *pairs, const int *idx, const int *npair, double *stl)
{
    const long long T = *npair;
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < T;
         u += (long long)gridDim.x * blockDim.x) {
        const long long t = idx ? idx[u] : u;
        const int2 p = pairs[t];
        stl[t] = lp_static_entry(g, min(p.x, p.y), max(p.x, p.y), kw);
    }
}

__global__ void __launch_bounds__(128)
k_pot_static(pb_fill_geom g, double kw, double *st)
{
    const int nc = g.ncell;
    const long long T = (long long)nc * (nc + 1) / 2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < T;
         t += (long long)gridDim.x * blockDim.x) {
        int ci, cj;
        tri_index(t, nc, ci, cj);
        double v = 0;                                   // potential.c:124-150
        for (int e = g.csoff[ci]; e < g.csoff[ci + 1]; e++) {
            const int h1 = g.csidx[e];
            for (int q = g.csoff[cj]; q < g.csoff[cj + 1]; q++) {
                const int h2 = g.csidx[q];
                const int a = min(h1, h2), b = max(h1, h2);
                Cell sa, sb;
                load_cell(sa, g.chg.cell, g.pv, a, 0, g.gpz);
                const double aa = g.chg.cell[a].aP, ab = g.chg.cell[b].aP;
                double x;
                if (a == b) {
                    x = static_term(sa, sa, 1, aa, aa, kw);
                } else {
                    load_cell(sb, g.chg.cell, g.pv, b, 0, g.gpz);
                    x = static_term(sa, sb, 0, aa, ab, kw);
                }
                if (g.gp) {
                    load_cell(sb, g.chg.cell, g.pv, b, 1, g.gpz);
                    x -= static_term(sa, sb, 0, aa, ab, kw);
                }
                v += x;
            }
        }
        st[(long long)ci * nc + cj] = v / (4 * PB_PI * PB_EPS0 * g.carea[ci] * g.carea[cj]);
    }
}

// ---------------------------------------------------------------- correction kernels
// One warp owns a group of PB_GROUP = 16 consecutive upper-triangle pairs. Set-up: lane p
// builds the direct term descriptor of pair p of the group and lane 16 + p its
// ground-plane image - the FP64 dispatch, frames and quadrature choice - into shared
// memory. Then the warp sweeps the samples: pairs with a near term one after the other
// with all 32 lanes (lanes split the samples), far and term-less pairs two at a time,
// one per half-warp. The FP64 set-up so costs one lane-evaluation per term.
// FP64 kernels: 4 warps per CTA, 4 CTAs per SM; FP32 kernels: 3 warps per CTA, 5 CTAs per
// SM (128 registers either way; the FP32 CTA's terms and totals take 44 KB of shared memory)
template <typename R> constexpr int corr_warps() { return sizeof(R) == 4 ? 3 : 4; }
template <typename R> constexpr int corr_minb() { return sizeof(R) == 4 ? 5 : 4; }
#define PB_GROUP 16

enum { PB_SET_LP = 0, PB_SET_IG = 1 };

struct TaskHdr { int i, j, nterm, half; };   // half: far or term-less, runs on a half-warp

__device__ __forceinline__ void prefetch_l1(const void *p)
{
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// One term of a far pair (2-point rule) on a half-warp: lane l of half h takes sample
// (i, j, m, q) = bits 0..3 of l & 15 of the term T_h; the half's phase bases sit at
// base + h * nbase. T is null for a half whose pair has fewer terms.
template <int F, int EQ, int RED>
__device__ void run_far2(const Term<float> *T, const KArg &k, Acc<float, F> &a, int lane, float4 *bases)
{
    constexpr int NB = nbase<F, EQ>();
    const int hl = lane & 15;
    const float4 *base = T ? T->tb : nullptr;       // EQ: formed in the set-up
    if (!EQ) {
        float4 *bw = bases + (lane >> 4) * NB;
        __syncwarp();                               // previous term's bases no longer read
        if (T && hl < NB) {
            double sn, cs;
            sincos(k.kh[hl] * T->D, &sn, &cs);
            const float sh = (float)sn, ch = (float)cs;
            bw[hl] = make_float4(sh, ch, (float)(sn - (double)sh), (float)(cs - (double)ch));
        }
        __syncwarp();
        base = bw;
    }
    if (T) {
        const float g = 0.577350269189625765f;      // 1/sqrt(3), weights 1
        const float xi = (hl & 1) ? g : -g, xj = (hl & 2) ? g : -g;
        const float xm = (hl & 4) ? g : -g, xq = (hl & 8) ? g : -g;
        const float a1 = 0.5f * T->L1 * xi, b1 = 0.5f * T->W1 * xj, a2 = 0.5f * T->L2 * xm, b2 = 0.5f * T->W2 * xq;
        const float cd[3] = {T->cdf[0], T->cdf[1], T->cdf[2]};
        float p[3];
#pragma unroll
        for (int c = 0; c < 3; c++) p[c] = fmaf(a2, T->u2[c], fmaf(b2, T->v2[c], -fmaf(a1, T->u1[c], b1 * T->v1[c])));
        sample32<F, EQ, RED>(a, k, base, cd, 0.f, T->Df, T->Dlo, p[0], p[1], p[2], (float)(-2.0 * T->sc));
    }
}

// reduce_select for two pairs at once: lane f of half h sums frequency f over the 16
// lanes of half h (F <= 16).
template <int F>
__device__ __forceinline__ void reduce_halves(Acc<float, F> &a, int lane, double &cr, double &ci)
{
    a.flush();
    __syncwarp();
    cr = ci = 0;
    const int hl = lane & 15, h0 = lane & 16;
    if (hl < F) {
        const double *base = a.tot - lane + h0;
#pragma unroll 8
        for (int l = 0; l < 16; l++) {
            cr += base[(2 * hl) * 32 + l];
            ci += base[(2 * hl + 1) * 32 + l];
        }
    }
    __syncwarp();
}

template <typename R, int F, int EQ>
constexpr size_t corr_smem_bytes()
{
    return (size_t)corr_warps<R>() *
           (2 * PB_GROUP * sizeof(Term<R>) + PB_GROUP * sizeof(TaskHdr) +
            (sizeof(R) == 4 ? 2 * F * 32 * sizeof(double) + (EQ ? 0 : (PB_FMAX + 1) * sizeof(float4)) : 0));
}

template <typename R, int F, int SET, int EPI, int EQ, int RED>
__global__ void __launch_bounds__(32 * corr_warps<R>(), corr_minb<R>())
k_corr(pb_fill_geom g, KArg k, const double *st, pb_epi_args ea, double2 *ig, long long igs)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    Term<R> *terms = reinterpret_cast<Term<R> *>(smraw) + (size_t)wib * 2 * PB_GROUP;
    constexpr int PB_CORR_WARPS = corr_warps<R>();
    TaskHdr *hdr = reinterpret_cast<TaskHdr *>(smraw + (size_t)PB_CORR_WARPS * 2 * PB_GROUP * sizeof(Term<R>))
                   + wib * PB_GROUP;
    double *tot = reinterpret_cast<double *>(smraw + (size_t)PB_CORR_WARPS * (2 * PB_GROUP * sizeof(Term<R>) +
                                                                            PB_GROUP * sizeof(TaskHdr)))
                  + (size_t)wib * 2 * F * 32;
    float4 *bases = reinterpret_cast<float4 *>(smraw + (size_t)PB_CORR_WARPS * (2 * PB_GROUP * sizeof(Term<R>) +
                                                                              PB_GROUP * sizeof(TaskHdr) +
                                                                              2 * F * 32 * sizeof(double)))
                    + (size_t)wib * (PB_FMAX + 1);
    static_assert(nbase<F, 1>() <= PB_TBASE, "EQ bases per term");
    const pb_dev_cells &set = SET == PB_SET_LP ? g.seg : g.chg;
    const int n = set.n;
    const long long T = EPI == PB_EPI_LIST ? (long long)*ea.npair : (long long)n * (n + 1) / 2;
    const double coef = PB_MU0 / (4 * PB_PI);
    // far pairs two at a time: each half-warp needs its own phase bases
    constexpr bool PAIR_FAR = sizeof(R) == 4 && 2 * nbase<F, EQ>() <= PB_FMAX + 1;
    const double kw0 = k.kw[0];
    const int nf = k.nf;
    const long long stride = (long long)gridDim.x * PB_CORR_WARPS * PB_GROUP;
    for (long long g0 = ((long long)blockIdx.x * PB_CORR_WARPS + wib) * PB_GROUP; g0 < T; g0 += stride) {
        // ---- set-up: lane -> term (lane >> 4) of pair g0 + (lane & 15): the direct term on
        // the lower half-warp, the ground-plane image on the upper one
        static_assert(PB_GROUP == 16, "set-up maps two terms of 16 pairs onto the 32 lanes");
        const int pl = lane & 15, term = lane >> 4;
        const long long t = g0 + pl;
        int i = 0, j = 0, ok = 0;
        if (t < T) {
            if constexpr (EPI == PB_EPI_LIST) {
                const int2 p = ea.pairs[t];
                i = min(p.x, p.y);
                j = max(p.x, p.y);
            } else {
                tri_index(t, n, i, j);
            }
            if (kw0 > 0 && (term == 0 || g.gp)) {
                Cell si, sj;
                load_cell(si, set.cell, g.pv, i, 0, g.gpz);
                load_cell(sj, set.cell, g.pv, j, term, g.gpz);
                double wgt, a1, a2;
                if (SET == PB_SET_LP) {                     // partial.c:392-423
                    double t1[3], t2[3];
                    tangent(si, t1);
                    if (i == j) {
                        wgt = term == 0 ? 1.0 : -(t1[0] * t1[0] + t1[1] * t1[1] - t1[2] * t1[2]);
                    } else {
                        Cell u;
                        load_cell(u, set.cell, g.pv, j, 0, g.gpz);
                        tangent(u, t2);
                        wgt = term == 0 ? dot3(t1, t2) : -(t1[0] * t2[0] + t1[1] * t2[1] - t1[2] * t2[2]);
                    }
                    wgt *= coef;
                    a1 = set.cell[i].aL;
                    a2 = set.cell[j].aL;
                } else {                                    // potential.c:219-236
                    wgt = term == 0 ? 1.0 : -1.0;
                    a1 = set.cell[i].aP;
                    a2 = set.cell[j].aP;
                }
                if (wgt != 0) {
                    make_term<R>(terms[2 * pl + term], si, sj, (i == j && term == 0), a1, a2, wgt, kw0, k.kwmax,
                                 set, i, j);
                    ok = 1;
                }
            }
        }
        if constexpr (sizeof(R) == 4 && EQ) {
            // the term's phase bases, formed by its own lane (all lanes at once) rather than
            // by a few lanes while the others wait in the sample loops: sin/cos(kh[8 g] D) per
            // group of 8 frequencies, then sin/cos(dkh D)
            if (ok) {
                constexpr int NB = nbase<F, EQ>();
                const double D = terms[2 * pl + term].D;
                float4 *tb = terms[2 * pl + term].tb;
#pragma unroll 1
                for (int b = 0; b < NB; b++) {
                    double sn, cs;
                    sincos((b < NB - 1 ? k.kh[8 * b] : k.dkh) * D, &sn, &cs);
                    const float sh = (float)sn, ch = (float)cs;
                    tb[b] = make_float4(sh, ch, (float)(sn - (double)sh), (float)(cs - (double)ch));
                }
            }
        }
        const int ok_img = __shfl_down_sync(0xffffffffu, ok, 16);
        __syncwarp();                                       // both halves' terms written
        if (lane < PB_GROUP && t < T) {
            if (!ok && ok_img) terms[2 * pl] = terms[2 * pl + 1];   // image only: to slot 0
            const int nt = ok + ok_img;
            int far = nt > 0;
            for (int q = 0; q < nt; q++) far &= terms[2 * lane + q].ty == TT_RIBBON2;
            if (!far)                       // a pair that mixes rules takes the 3-point rule for its
                for (int q = 0; q < nt; q++)    // far terms: one sample loop less in the near path
                    if (terms[2 * lane + q].ty == TT_RIBBON2) terms[2 * lane + q].ty = TT_RIBBON3;
            // term-less pairs (e.g. perpendicular Lp cells) run with the far pairs, two at a
            // time: they need only the epilogue, which then serves two pairs per pass
            hdr[lane] = TaskHdr{i, j, nt, far || nt == 0};
        }
        __syncwarp();
        // the epilogue's scattered P(f) reads: start them into L1 before the samples, so that
        // they arrive while the samples run instead of stalling the warp afterwards
        auto prefetch_p = [&](const TaskHdr &h, int f) {
            if (EPI == PB_EPI_REDUCED && SET == PB_SET_LP && f < nf) {
                const int ca = g.seg_ca[h.i], cb = g.seg_cb[h.i], da = g.seg_ca[h.j], db = g.seg_cb[h.j];
                const double2 *P = ea.pm + f * ea.pm_stride;
                const int nc = g.ncell;
                if (ca >= 0 && da >= 0) prefetch_l1(P + (long long)ca * nc + da);
                if (ca >= 0 && db >= 0) prefetch_l1(P + (long long)ca * nc + db);
                if (cb >= 0 && da >= 0) prefetch_l1(P + (long long)cb * nc + da);
                if (cb >= 0 && db >= 0) prefetch_l1(P + (long long)cb * nc + db);
            }
        };
        // one entry (pair i, j) at frequency f from its correction cr + j cim
        auto emit = [&](int i, int j, int f, double cr, double cim, long long t) {
            if constexpr (EPI == PB_EPI_LIST) {     // one wavenumber; static part per entry
                const double lr = st[t] + cr;
                ea.out[t] = make_double2(ea.lscale_re * lr - ea.lscale_im * cim, ea.lscale_re * cim + ea.lscale_im * lr);
                return;
            }
            if (SET == PB_SET_IG) {
                ig[f * igs + (long long)i * n + j] = make_double2(cr, cim);
                return;
            }
            const double lr = st[(long long)i * n + j] + cr, li = cim;
            if (EPI == PB_EPI_STORE) {
                double2 *o = ea.out + f * ea.out_stride;
                o[(long long)i * n + j] = make_double2(lr, li);
                o[(long long)j * n + i] = make_double2(lr, li);
            } else {
                const double om = ea.omega[f];
                double vr = -om * om * lr, vi = -om * om * li;
                if (i == j) {
                    const double2 z = ea.zint[f * (long long)n + i];
                    vr -= om * z.y;
                    vi += om * z.x;
                }
                const int nc = g.ncell;
                const double2 *P = ea.pm + f * ea.pm_stride;
                const int ca = g.seg_ca[i], cb = g.seg_cb[i], da = g.seg_ca[j], db = g.seg_cb[j];
                if (ca >= 0 && da >= 0) { const double2 pp = P[(long long)ca * nc + da]; vr += pp.x; vi += pp.y; }
                if (ca >= 0 && db >= 0) { const double2 pp = P[(long long)ca * nc + db]; vr -= pp.x; vi -= pp.y; }
                if (cb >= 0 && da >= 0) { const double2 pp = P[(long long)cb * nc + da]; vr -= pp.x; vi -= pp.y; }
                if (cb >= 0 && db >= 0) { const double2 pp = P[(long long)cb * nc + db]; vr += pp.x; vi += pp.y; }
                double2 *m = ea.m64 + f * ea.m_stride;
                m[(long long)j * n + i] = make_double2(vr, vi);           // lower (i <= j)
                if (!ea.lower) m[(long long)i * n + j] = make_double2(vr, vi);
                if (ea.m32) {
                    float2 *m2 = ea.m32 + f * ea.m_stride;
                    m2[(long long)j * n + i] = make_float2((float)vr, (float)vi);
                    if (!ea.lower) m2[(long long)i * n + j] = make_float2((float)vr, (float)vi);
                }
            }
        };
        // ---- samples of the 16 pairs: other pairs one after the other with the whole warp,
        // then the far pairs (2-point rule, 16 samples per term) and the term-less pairs two
        // at a time, one per half-warp, so that no lane idles and one transposed reduction
        // and one epilogue pass serve both
        const bool valid = lane < PB_GROUP && g0 + lane < T;
        unsigned far_m = PAIR_FAR ? __ballot_sync(0xffffffffu, valid && hdr[lane].half) : 0u;
        unsigned near_m = __ballot_sync(0xffffffffu, valid) & ~far_m;
        const int half = lane >> 4, hl = lane & 15;
        while (near_m | far_m) {                           // warp-uniform
            int tk, f;
            double cr = 0, cim = 0;
            if (near_m) {
                tk = __ffs(near_m) - 1;
                near_m &= near_m - 1;
                f = lane;
                const TaskHdr h = hdr[tk];
                prefetch_p(h, f);
                if (h.nterm > 0) {           // warp-uniform; e.g. perpendicular Lp pairs have none
                    Acc<R, F> acc;
                    acc.init(tot + lane);
                    for (int q = 0; q < h.nterm; q++) {
                        if constexpr (sizeof(R) == 4) {
                            run_term32<F, EQ, RED, !PAIR_FAR>(terms[2 * tk + q], k, acc, lane, bases, set.qpt);
                        } else {
                            const Term<R> tm = terms[2 * tk + q];
                            run_term<R, F, EQ>(tm, k, acc, lane, set.qpt);
                        }
                    }
                    reduce_select<F>(acc, lane, cr, cim);
                }
            } else {
                if constexpr (PAIR_FAR) {
                    const int ta = __ffs(far_m) - 1;
                    far_m &= far_m - 1;
                    int tb = -1;
                    if (far_m) { tb = __ffs(far_m) - 1; far_m &= far_m - 1; }
                    tk = half ? tb : ta;
                    f = hl;
                    const int nq = max(hdr[ta].nterm, tb >= 0 ? hdr[tb].nterm : 0);
                    const int nt = tk >= 0 ? hdr[tk].nterm : 0;
                    if (tk >= 0) prefetch_p(hdr[tk], f);
                    if (nq > 0) {                          // warp-uniform; 0: two term-less pairs
                        // at most two samples per lane (one per term): FP32 partials, no
                        // FP64 running totals (the flush never triggers); the transposed
                        // reduction adds the 16 lanes of a half in FP64
                        Acc<R, F> acc;
                        acc.tot = nullptr;
                        acc.cnt = 0;
#pragma unroll
                        for (int ff = 0; ff < F; ff++) acc.pr[ff] = acc.pi[ff] = 0.f;
                        for (int q = 0; q < nq; q++)
                            run_far2<F, EQ, RED>(q < nt ? &terms[2 * tk + q] : nullptr, k, acc, lane, bases);
                        float *fp = reinterpret_cast<float *>(tot);
                        __syncwarp();
#pragma unroll
                        for (int ff = 0; ff < F; ff++) {
                            fp[(2 * ff) * 32 + lane] = acc.pr[ff];
                            fp[(2 * ff + 1) * 32 + lane] = acc.pi[ff];
                        }
                        __syncwarp();
                        cr = cim = 0;
                        if (hl < F) {
                            const int h0 = lane & 16;
#pragma unroll 8
                            for (int l = 0; l < 16; l++) {
                                cr += (double)fp[(2 * hl) * 32 + h0 + l];
                                cim += (double)fp[(2 * hl + 1) * 32 + h0 + l];
                            }
                        }
                        __syncwarp();
                    }
                } else {
                    tk = -1;
                    f = 0;
                }
            }
            if (tk >= 0 && f < nf) emit(hdr[tk].i, hdr[tk].j, f, cr, cim, g0 + tk);
        }
        __syncwarp();
    }
}

// P(f)[ci][cj] = static + 1/(4 pi eps0 Ai Aj) * sum over sub-cell pairs of the correction
// (potential.c:124-150 ordering of the sub-pairs); thread per (f, ci <= cj).
__global__ void k_pot_aggr(pb_fill_geom g, int nf, const double *st, const double2 *ig, long long igs,
                           double2 *out, long long ostride)
{
    const int nc = g.ncell, nh = g.chg.n;
    const long long T = (long long)nc * (nc + 1) / 2;
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= T * nf) return;
    const int f = (int)(idx / T);
    int ci, cj;
    tri_index(idx - f * T, nc, ci, cj);
    double sr = 0, si = 0;
    if (ig) {
        const double2 *I = ig + f * igs;
        for (int e = g.csoff[ci]; e < g.csoff[ci + 1]; e++) {
            const int h1 = g.csidx[e];
            for (int q = g.csoff[cj]; q < g.csoff[cj + 1]; q++) {
                const int h2 = g.csidx[q];
                const double2 v = I[(long long)min(h1, h2) * nh + max(h1, h2)];
                sr += v.x;
                si += v.y;
            }
        }
    }
    const double sc = 1.0 / (4 * PB_PI * PB_EPS0 * g.carea[ci] * g.carea[cj]);
    const double2 v = make_double2(st[(long long)ci * nc + cj] + sc * sr, sc * si);
    double2 *o = out + f * ostride;
    o[(long long)ci * nc + cj] = v;
    o[(long long)cj * nc + ci] = v;
}

static int grid_for(long long work, int per_block, int blocks_per_sm = 8);
// ---------------------------------------------------------------- sample counting
// Samples of one term; r2 counts the terms on the 2-point rule (kwf > 0: the FP32 path).
__device__ __forceinline__ long long pair_samples(const Cell &s1, const Cell &s2, int same, double kw,
                                                  const pb_dev_cells &set, int i1, int i2, double kwf, int &r2)
{
    if (same && s1.wid <= 0 && s1.npv <= 0) { const int n = corr_nsub(s1, s1, kw); return 64LL * n * n; }
    const int ty = pair_type(s1, s2);
    if (ty == PT_POLY)
        return (long long)(set.qoff[i1 + 1] - set.qoff[i1]) * (set.qoff[i2 + 1] - set.qoff[i2]);
    if (ty == PT_HL || ty == PT_RIBBON) {
        const int n = ribbon_nsub(s1, s2, kw);
        if (kwf > 0) {
            double t[3], w[3], nv[3], c1[3], c2[3];
            frame(s1, t, w, nv, c1);
            frame(s2, t, w, nv, c2);
            const int rule = ribbon_rule32(s1, s2, n, c1, c2, kwf);
            if (rule == 2) { r2++; return 16; }
            if (rule == 3) return 81;
        }
        return 256LL * n * n;
    }
    const int n = corr_nsub(s1, s2, kw);
    if (kwf > 0 && !same && wire_far32(s1, s2, kwf)) return 32;      // the FP32 path's 4 x 8 rule
    return 64LL * n * n;
}

// A pair whose terms do not all take the 2-point rule runs its 2-point terms on the 3-point
// rule (the k_corr set-up does the same).
__device__ __forceinline__ long long mixed_fix(int nterm, int r2) { return r2 < nterm ? r2 * (81LL - 16) : 0; }

__global__ void k_count(pb_fill_geom g, double kw, unsigned long long *out, double kwf)
{
    unsigned long long acc_lp = 0, acc_p = 0;
    const int n = g.seg.n, nc = g.ncell;
    const long long T1 = (long long)n * (n + 1) / 2, T2 = (long long)nc * (nc + 1) / 2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < T1 + T2;
         t += (long long)gridDim.x * blockDim.x) {
        if (t < T1) {
            int i, j;
            tri_index(t, n, i, j);
            Cell si, sj;
            load_cell(si, g.seg.cell, g.pv, i, 0, g.gpz);
            double t1[3], t2[3];
            tangent(si, t1);
            int nt = 0, r2 = 0;
            if (i == j) {
                acc_lp += pair_samples(si, si, 1, kw, g.seg, i, i, kwf, r2);
                nt++;
                const double tdm = t1[0] * t1[0] + t1[1] * t1[1] - t1[2] * t1[2];
                if (g.gp && tdm != 0) {
                    load_cell(sj, g.seg.cell, g.pv, i, 1, g.gpz);
                    acc_lp += pair_samples(si, sj, 0, kw, g.seg, i, i, kwf, r2);
                    nt++;
                }
            } else {
                load_cell(sj, g.seg.cell, g.pv, j, 0, g.gpz);
                tangent(sj, t2);
                const double tdot = dot3(t1, t2), tdm = t1[0] * t2[0] + t1[1] * t2[1] - t1[2] * t2[2];
                if (tdot != 0) { acc_lp += pair_samples(si, sj, 0, kw, g.seg, i, j, kwf, r2); nt++; }
                if (g.gp && tdm != 0) {
                    load_cell(sj, g.seg.cell, g.pv, j, 1, g.gpz);
                    acc_lp += pair_samples(si, sj, 0, kw, g.seg, i, j, kwf, r2);
                    nt++;
                }
            }
            acc_lp += mixed_fix(nt, r2);
        } else {
            int ci, cj;
            tri_index(t - T1, nc, ci, cj);
            for (int e = g.csoff[ci]; e < g.csoff[ci + 1]; e++)
                for (int q = g.csoff[cj]; q < g.csoff[cj + 1]; q++) {
                    const int a = min(g.csidx[e], g.csidx[q]), b = max(g.csidx[e], g.csidx[q]);
                    Cell sa, sb;
                    load_cell(sa, g.chg.cell, g.pv, a, 0, g.gpz);
                    load_cell(sb, g.chg.cell, g.pv, b, 0, g.gpz);
                    int r2 = 0;
                    acc_p += pair_samples(sa, sb, a == b, kw, g.chg, a, b, kwf, r2);
                    if (g.gp) { load_cell(sb, g.chg.cell, g.pv, b, 1, g.gpz); acc_p += pair_samples(sa, sb, 0, kw, g.chg, a, b, kwf, r2); }
                    acc_p += mixed_fix(g.gp ? 2 : 1, r2);
                }
        }
    }
    atomicAdd(&out[0], acc_lp);
    atomicAdd(&out[1], acc_p);
}

// d_count: two counters of device memory owned by the caller (no allocation here: a
// cudaFree would synchronise the whole device under concurrent sweeps)
int pb_count_samples(const pb_fill_geom &g, double kw, double *lp_samples, double *p_samples,
                     cudaStream_t s, unsigned long long *d_count, double kw_far32)
{
    unsigned long long *d = d_count, h[2] = {0, 0};
    PB_CUDA(cudaMemsetAsync(d, 0, 16, s));
    const long long T = (long long)g.seg.n * (g.seg.n + 1) / 2 + (long long)g.ncell * (g.ncell + 1) / 2;
    if (T > 0) k_count<<<grid_for(T, 256), 256, 0, s>>>(g, kw, d, kw_far32);
    cudaError_t e = cudaMemcpyAsync(h, d, 16, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return pb_cuda_fail(e, "pb_count_samples", __FILE__, __LINE__);
    *lp_samples = (double)h[0];
    *p_samples = (double)h[1];
    return PB_OK;
}

// ---------------------------------------------------------------- internal impedance
__device__ double2 cdiv_d(double2 a, double2 b)                   // complex.h:40-45
{
    if ((fabs(b.x) <= 0) && (fabs(b.y) <= 0)) return make_double2(0, 0);
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double cabs_d(double2 z) { return sqrt(z.x * z.x + z.y * z.y); }

__device__ double2 i0_over_i1(double2 z)                          // skin.c:23-56
{
    if (cabs_d(z) < 15.0) {
        const double2 z2 = cmul(z, z);
        double2 i0 = make_double2(1, 0), t = make_double2(1, 0);
        for (int k = 1; k <= 60; k++) {
            const double2 u = cmul(t, z2);
            const double f = 1.0 / (4.0 * k * k);
            t = make_double2(f * u.x, f * u.y);
            i0 = cadd(i0, t);
            if (cabs_d(t) < 1e-17 * cabs_d(i0)) break;
        }
        double2 s = make_double2(1, 0);
        t = make_double2(1, 0);
        for (int k = 1; k <= 60; k++) {
            const double2 u = cmul(t, z2);
            const double f = 1.0 / (4.0 * k * (k + 1));
            t = make_double2(f * u.x, f * u.y);
            s = cadd(s, t);
            if (cabs_d(t) < 1e-17 * cabs_d(s)) break;
        }
        return cdiv_d(i0, cmul(make_double2(0.5 * z.x, 0.5 * z.y), s));
    }
    const double2 u = cinv(z), u2 = cmul(u, u), u3 = cmul(u2, u);
    return make_double2(1 + 0.5 * u.x + 0.375 * u2.x + 0.375 * u3.x,
                        0.5 * u.y + 0.375 * u2.y + 0.375 * u3.y);
}

__global__ void k_zint(pb_fill_geom g, int skin, int nf, const double *freq, double2 *zint)
{
    const int n = g.seg.n;
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)n * nf) return;
    const int f = (int)(idx / n), k = (int)(idx - (long long)f * n);
    const pb_cell_t *s = &g.seg.cell[k];
    const double fr = freq[f], om = 2 * PB_PI * fr;
    double2 z = make_double2(s->res, 0);
    if (s->diel) {                                     // mna.c:128-138
        if (s->frelax > 0) {
            const double2 q = cdiv_d(make_double2(s->epss - s->epsinf, 0), make_double2(1, fr / s->frelax));
            const double2 er = make_double2(s->epsinf + q.x, q.y);
            z = cinv(make_double2(om * s->gfac * (-er.y), om * s->gfac * (er.x - 1)));
        } else {
            const double2 y = cinv(make_double2(s->gexc, s->cexc));
            z = make_double2(y.x / om, y.y / om);
        }
    } else if (skin) {                                 // skin.c:112-133
        if (s->vol) {
            z = make_double2(s->res, 0);
        } else if (s->shape == PB_SHAPE_ROUND) {       // skin.c:59-77
            const double len = s->len, a = s->radius, sg = s->sigma;
            if ((sg <= 0) || (len <= 0) || (a <= 0)) z = make_double2(0, 0);
            else if (om <= 0) z = make_double2(len / (sg * PB_PI * a * a), 0);
            else {
                const double delta = sqrt(2 / (om * PB_MU0 * sg)), q = a / delta;
                const double2 ratio = i0_over_i1(make_double2(q, q));
                const double kf = 1 / (2 * PB_PI * a * delta * sg);
                const double2 zz = cmul(make_double2(kf, kf), ratio);
                z = make_double2(len * zz.x, len * zz.y);
            }
        } else {                                       // skin.c:91-109
            const double len = s->len, ar = s->area, pe = s->perim, sg = s->sigma;
            if ((sg <= 0) || (len <= 0) || (ar <= 0) || (pe <= 0)) z = make_double2(0, 0);
            else if (om <= 0) z = make_double2(len / (sg * ar), 0);
            else {
                const double rdc = len / (sg * ar);
                const double delta = sqrt(2 / (om * PB_MU0 * sg));
                const double rhf = len / (sg * delta * pe);
                const double ldc = PB_MU0 * len / (8 * PB_PI), lhf = rhf / om;
                const double r = sqrt(rdc * rdc + rhf * rhf);
                const double l = ldc * lhf / sqrt(ldc * ldc + lhf * lhf);
                z = make_double2(r, om * l);
            }
        }
    }
    zint[idx] = z;
}

// ---------------------------------------------------------------- host launchers
static int grid_for(long long work, int per_block, int blocks_per_sm)
{
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    long long want = (work + per_block - 1) / per_block;
    const long long cap = (long long)nsm * blocks_per_sm * 64;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return (int)want;
}

int pb_lp_static(const pb_fill_geom &g, double kw, double *stLp, cudaStream_t s, long *launches)
{
    const long long T = (long long)g.seg.n * (g.seg.n + 1) / 2;
    if (T == 0) return PB_OK;
    k_lp_static<<<grid_for(T, 128), 128, 0, s>>>(g, kw, stLp);
    if (launches) (*launches)++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

int pb_pot_static(const pb_fill_geom &g, double kw, double *stP, cudaStream_t s, long *launches)
{
    const long long T = (long long)g.ncell * (g.ncell + 1) / 2;
    if (T == 0) return PB_OK;
    k_pot_static<<<grid_for(T, 128), 128, 0, s>>>(g, kw, stP);
    if (launches) (*launches)++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

template <typename R, int F, int SET, int EPI, int EQ, int RED>
static int launch_corr(const pb_fill_geom &g, const KArg &k, const double *st, const pb_epi_args &ea,
                       double2 *ig, long long igs, cudaStream_t s)
{
    const int n = SET == PB_SET_LP ? g.seg.n : g.chg.n;
    const long long T = EPI == PB_EPI_LIST ? ea.lcap : (long long)n * (n + 1) / 2;
    constexpr size_t smem = corr_smem_bytes<R, F, EQ>();
    static std::atomic<unsigned long long> attr_set{0};   // per device, before any launch relies on it
    PB_TRY(pb_smem_optin(k_corr<R, F, SET, EPI, EQ, RED>, (int)smem, attr_set));
    const int grid = grid_for((T + PB_GROUP - 1) / PB_GROUP, corr_warps<R>(), corr_minb<R>());
    k_corr<R, F, SET, EPI, EQ, RED><<<grid, 32 * corr_warps<R>(), smem, s>>>(g, k, st, ea, ig, igs);
    PB_CHECK_LAUNCH();
    return PB_OK;
}

template <typename R, int F, int SET, int EPI>
static int launch_corr_eq(const pb_fill_geom &g, const KArg &k, const double *st, const pb_epi_args &ea,
                          double2 *ig, long long igs, cudaStream_t s)
{
    if (sizeof(R) == 8) return launch_corr<R, F, SET, EPI, 0, 0>(g, k, st, ea, ig, igs, s);
    if (k.eq) {
        if (k.reduce) return launch_corr<R, F, SET, EPI, 1, 1>(g, k, st, ea, ig, igs, s);
        return launch_corr<R, F, SET, EPI, 1, 0>(g, k, st, ea, ig, igs, s);
    }
    if (k.reduce) return launch_corr<R, F, SET, EPI, 0, 1>(g, k, st, ea, ig, igs, s);
    return launch_corr<R, F, SET, EPI, 0, 0>(g, k, st, ea, ig, igs, s);
}

template <int SET, int EPI>
static int launch_corr_any(const pb_fill_geom &g, const KArg &k, int use_fp32, const double *st,
                           const pb_epi_args &ea, double2 *ig, long long igs, cudaStream_t s)
{
    const int F = k.nf <= 1 ? 1 : k.nf <= 8 ? 8 : 16;
    if (use_fp32) {
        if (F == 1) return launch_corr_eq<float, 1, SET, EPI>(g, k, st, ea, ig, igs, s);
        if (F == 8) return launch_corr_eq<float, 8, SET, EPI>(g, k, st, ea, ig, igs, s);
        return launch_corr_eq<float, 16, SET, EPI>(g, k, st, ea, ig, igs, s);
    }
    if (F == 1) return launch_corr_eq<double, 1, SET, EPI>(g, k, st, ea, ig, igs, s);
    if (F == 8) return launch_corr_eq<double, 8, SET, EPI>(g, k, st, ea, ig, igs, s);
    return launch_corr_eq<double, 16, SET, EPI>(g, k, st, ea, ig, igs, s);
}

// wavenumber set of a launch; equally spaced sets (linear sweeps) use the recurrence.
// pmax bounds |R - D| of every sample (0 = unknown): angles kh * pmax below pi/4 need no
// reduction in the FP32 path.
static void make_karg(KArg &k, int nf, const double *kw, double pmax)
{
    double khmax = 0;
    for (int f = 0; f < PB_FMAX; f++) {
        k.kw[f] = f < nf ? kw[f] : 0.0;
        k.kh[f] = 0.5 * k.kw[f];
        k.khf[f] = (float)k.kh[f];
        khmax = fmax(khmax, k.kh[f]);
    }
    k.nf = nf;
    k.kwmax = 2 * khmax;
    k.dkh = nf > 1 ? 0.5 * (kw[1] - kw[0]) : 0.0;
    k.eq = nf > 1;
    for (int f = 1; f < nf && k.eq; f++)
        if (fabs(kw[f] - kw[0] - f * (kw[1] - kw[0])) > 1e-9 * fabs(kw[nf - 1])) k.eq = 0;
    if (k.dkh <= 0) k.eq = 0;
    k.dkhf = (float)k.dkh;
    k.reduce = !(pmax > 0 && khmax * pmax < 0.78);      // |dkh| <= khmax: covers the step too
    k.step_tiny = pmax > 0 && fabs(k.dkh) * pmax < 0.01;
}

int pb_lp_corr(const pb_fill_geom &g, int nf, const double *kw, int use_fp32, const double *stLp,
               int epi, const pb_epi_args &ea, cudaStream_t s, long *launches, double *samples)
{
    if (g.seg.n == 0) return PB_OK;
    if (nf < 1 || nf > PB_FMAX) { pb_set_error("pb_lp_corr: bad frequency count %d", nf); return PB_ERR_ARG; }
    KArg k;
    make_karg(k, nf, kw, g.pmax);
    const int r = epi == PB_EPI_STORE
        ? launch_corr_any<PB_SET_LP, PB_EPI_STORE>(g, k, use_fp32, stLp, ea, nullptr, 0, s)
        : launch_corr_any<PB_SET_LP, PB_EPI_REDUCED>(g, k, use_fp32, stLp, ea, nullptr, 0, s);
    if (launches) (*launches)++;
    (void)samples;
    return r;
}

int pb_lp_entries_static(const pb_fill_geom &g, double kw, const int2 *pairs, const int *idx, const int *nidx_dev,
                         long long cap, double *stl, cudaStream_t s, long *launches)
{
    if (cap <= 0 || g.seg.n == 0) return PB_OK;
    k_lp_static_list<<<grid_for(cap, 128), 128, 0, s>>>(g, kw, pairs, idx, nidx_dev, stl);
    if (launches) (*launches)++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

int pb_lp_entries_corr(const pb_fill_geom &g, double kw, int use_fp32, const int2 *pairs, const int *npair_dev,
                       long long cap, double2 scale, const double *stl, double2 *out, cudaStream_t s,
                       long *launches)
{
    if (cap <= 0 || g.seg.n == 0) return PB_OK;
    KArg k;
    make_karg(k, 1, &kw, g.pmax);
    pb_epi_args ea;
    ea.out = out;
    ea.pairs = pairs;
    ea.npair = npair_dev;
    ea.lcap = cap;
    ea.lscale_re = scale.x;
    ea.lscale_im = scale.y;
    int r;
    if (use_fp32)
        r = k.reduce ? launch_corr<float, 1, PB_SET_LP, PB_EPI_LIST, 0, 1>(g, k, stl, ea, nullptr, 0, s)
                     : launch_corr<float, 1, PB_SET_LP, PB_EPI_LIST, 0, 0>(g, k, stl, ea, nullptr, 0, s);
    else
        r = launch_corr<double, 1, PB_SET_LP, PB_EPI_LIST, 0, 0>(g, k, stl, ea, nullptr, 0, s);
    if (launches) (*launches)++;
    return r;
}

int pb_lp_entries(const pb_fill_geom &g, double kw, int use_fp32, const int2 *pairs, const int *npair_dev,
                  long long cap, double2 scale, double *stl, double2 *out, cudaStream_t s, long *launches)
{
    PB_TRY(pb_lp_entries_static(g, kw, pairs, nullptr, npair_dev, cap, stl, s, launches));
    return pb_lp_entries_corr(g, kw, use_fp32, pairs, npair_dev, cap, scale, stl, out, s, launches);
}

int pb_pot_corr(const pb_fill_geom &g, int nf, const double *kw, int use_fp32, const double *stP,
                double2 *pout, long long pstride, double2 *igbuf, cudaStream_t s, long *launches,
                double *samples)
{
    if (g.ncell == 0) return PB_OK;
    if (nf < 1 || nf > PB_FMAX) { pb_set_error("pb_pot_corr: bad frequency count %d", nf); return PB_ERR_ARG; }
    KArg k;
    make_karg(k, nf, kw, g.pmax);
    const long long igs = (long long)g.chg.n * g.chg.n;
    const bool corr = kw[0] > 0;
    if (corr) {
        if (!igbuf) { pb_set_error("pb_pot_corr: missing sub-cell buffer"); return PB_ERR_ARG; }
        pb_epi_args ea;
        const int r = launch_corr_any<PB_SET_IG, PB_EPI_STORE>(g, k, use_fp32, nullptr, ea, igbuf, igs, s);
        if (r != PB_OK) return r;
        if (launches) (*launches)++;
    }
    const long long T = (long long)g.ncell * (g.ncell + 1) / 2 * nf;
    k_pot_aggr<<<ceil_div(T, 256), 256, 0, s>>>(g, nf, stP, corr ? igbuf : nullptr, igs, pout, pstride);
    if (launches) (*launches)++;
    PB_CHECK_LAUNCH();
    (void)samples;
    return PB_OK;
}

int pb_zint(const pb_fill_geom &g, int skin, int nf, const double *freq, double2 *zint,
            cudaStream_t s, long *launches)
{
    const long long T = (long long)g.seg.n * nf;
    if (T == 0) return PB_OK;
    k_zint<<<ceil_div(T, 128), 128, 0, s>>>(g, skin, nf, freq, zint);
    if (launches) (*launches)++;
    PB_CHECK_LAUNCH();
    return PB_OK;
}

// ---------------------------------------------------------------- poly point sets
// cell_qpts(s, nsub=1, n7=0) of polygon.c:224-268 computed on the host once per
// geometry, stored as offsets from the cell centre 0.5*(x1+x2). Degenerate fan
// triangles keep their slots with zero weight (their samples contribute exactly 0).
static void host_qpts(const pb_cell_t &c, const double *pool, std::vector<double> &out)
{
    static const double XG4h[4] = {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526};
    static const double WG4h[4] = {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538};
    static const double TB3h[3][3] = {{2.0 / 3, 1.0 / 6, 1.0 / 6}, {1.0 / 6, 2.0 / 3, 1.0 / 6}, {1.0 / 6, 1.0 / 6, 2.0 / 3}};
    double cen[3];
    for (int i = 0; i < 3; i++) cen[i] = 0.5 * (c.x1[i] + c.x2[i]);
    auto push = [&](const double *p, double w) {
        out.push_back(p[0] - cen[0]); out.push_back(p[1] - cen[1]);
        out.push_back(p[2] - cen[2]); out.push_back(w);
    };
    if (c.npv > 0) {
        const double *pv = pool + 3 * (long long)c.pvoff;
        for (int k = 0; k < c.npv; k++) {
            const double *b = &pv[3 * k], *cc = &pv[3 * ((k + 1) % c.npv)], *a = c.papex;
            double u[3], v[3], w[3];
            for (int i = 0; i < 3; i++) { u[i] = b[i] - a[i]; v[i] = cc[i] - a[i]; }
            w[0] = u[1] * v[2] - u[2] * v[1];
            w[1] = u[2] * v[0] - u[0] * v[2];
            w[2] = u[0] * v[1] - u[1] * v[0];
            const double at = 0.5 * sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
            for (int q = 0; q < 3; q++) {
                double px[3];
                for (int i = 0; i < 3; i++) px[i] = TB3h[q][0] * a[i] + TB3h[q][1] * b[i] + TB3h[q][2] * cc[i];
                push(px, at > 0 ? (1.0 / 3) * at : 0.0);
            }
        }
        return;
    }
    if (c.wid <= 0) {
        for (int q = 0; q < 4; q++) {
            const double u = 0.5 * (1 + XG4h[q]);
            double px[3];
            for (int i = 0; i < 3; i++) px[i] = c.x1[i] + (c.x2[i] - c.x1[i]) * u;
            push(px, 0.5 * WG4h[q] * c.len);
        }
        return;
    }
    double t[3];
    for (int i = 0; i < 3; i++) t[i] = (c.x2[i] - c.x1[i]) / c.len;
    for (int q = 0; q < 4; q++) {
        const double a = c.len * (0.5 * (1 + XG4h[q]) - 0.5);
        for (int j = 0; j < 4; j++) {
            const double b = c.wid * (0.5 * XG4h[j]);
            double px[3];
            for (int i = 0; i < 3; i++) px[i] = cen[i] + a * t[i] + b * c.wv[i];
            push(px, 0.25 * WG4h[q] * WG4h[j] * c.len * c.wid);
        }
    }
}

int pb_build_qpts(pb_dev_cells &c, const pb_cell_t *host_cells, const double *pv_host,
                  const double *pv_dev, cudaStream_t s)
{
    (void)pv_dev;
    std::vector<double> pts;
    std::vector<int> off(c.n + 1, 0);
    for (int i = 0; i < c.n; i++) {
        host_qpts(host_cells[i], pv_host, pts);
        off[i + 1] = (int)(pts.size() / 4);
    }
    PB_CUDA(cudaMalloc(&c.qoff, sizeof(int) * (c.n + 1)));
    PB_CUDA(cudaMalloc(&c.qpt, sizeof(double4) * (pts.size() / 4 + 1)));
    PB_CUDA(cudaMemcpyAsync(c.qoff, off.data(), sizeof(int) * (c.n + 1), cudaMemcpyHostToDevice, s));
    if (!pts.empty())
        PB_CUDA(cudaMemcpyAsync(c.qpt, pts.data(), sizeof(double) * pts.size(), cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaStreamSynchronize(s));
    return PB_OK;
}
