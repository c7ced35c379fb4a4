// pb_geom.cuh — device-side geometry of partial elements: FP64 static integrals
// (closed forms and outer quadratures) and the pair dispatch.
//
// Every function restates the reference routine named in its comment (file:line within
// the OpenPEEC project). These run in FP64 on the device: they hold the cancellation-
// prone closed forms (asinh / atan sums, Hoer-Love's 64-term alternating sum).
#pragma once
#include "pb_common.cuh"

// Gauss-Legendre nodes/weights on [-1,1] (partial.c:113-122, surface.c:26-37) and the
// 7-/3-point triangle rules (polygon.c:134-152). Same published constants as the
// reference, so the static integrals are evaluated with identical rules.
__constant__ double cXG8[8] = {
    -0.9602898564975363, -0.7966664774136267, -0.5255324099163290, -0.1834346424956498,
     0.1834346424956498,  0.5255324099163290,  0.7966664774136267,  0.9602898564975363};
__constant__ double cWG8[8] = {
     0.1012285362903763,  0.2223810344533745,  0.3137066458778873,  0.3626837833783620,
     0.3626837833783620,  0.3137066458778873,  0.2223810344533745,  0.1012285362903763};
__constant__ double cXG4[4] = {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526};
__constant__ double cWG4[4] = {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538};
__constant__ double cXG2[2] = {-0.5773502691896257, 0.5773502691896257};
__constant__ double cWG2[2] = {1.0, 1.0};
__constant__ double cTW7[7] = {0.225, 0.1323941527885062, 0.1323941527885062, 0.1323941527885062,
                               0.1259391805448271, 0.1259391805448271, 0.1259391805448271};
__constant__ double cTB7[7][3] = {
    {1.0 / 3, 1.0 / 3, 1.0 / 3},
    {0.0597158717897698, 0.4701420641051151, 0.4701420641051151},
    {0.4701420641051151, 0.0597158717897698, 0.4701420641051151},
    {0.4701420641051151, 0.4701420641051151, 0.0597158717897698},
    {0.7974269853530873, 0.1012865073234563, 0.1012865073234563},
    {0.1012865073234563, 0.7974269853530873, 0.1012865073234563},
    {0.1012865073234563, 0.1012865073234563, 0.7974269853530873}};
__constant__ double cTW3[3] = {1.0 / 3, 1.0 / 3, 1.0 / 3};
__constant__ double cTB3[3][3] = {{2.0 / 3, 1.0 / 6, 1.0 / 6}, {1.0 / 6, 2.0 / 3, 1.0 / 6}, {1.0 / 6, 1.0 / 6, 2.0 / 3}};
// sub-triangle barycentric corners of the 4-way split (polygon.c:189-193)
__constant__ double cSUB[4][3][3] = {
    {{1, 0, 0}, {0.5, 0.5, 0}, {0.5, 0, 0.5}},
    {{0.5, 0.5, 0}, {0, 1, 0}, {0, 0.5, 0.5}},
    {{0.5, 0, 0.5}, {0, 0.5, 0.5}, {0, 0, 1}},
    {{0.5, 0.5, 0}, {0, 0.5, 0.5}, {0.5, 0, 0.5}}};

// A cell as the kernels see it: geometry of pb_cell_t, optionally the ground-plane image
// (z -> 2 gpz - z for the axis, apex and ring, wv.z -> -wv.z : partial.c:352-362).
struct Cell {
    double x1[3], x2[3], wv[3], papex[3];
    double len, wid, thick;
    int vol, npv;
    const double *pv;   // ring in the vertex pool (not mirrored)
    int mirror;
    double gpz;
    __device__ __forceinline__ double pvx(int k, int c) const
    {
        const double v = pv[3 * k + c];
        return (mirror && c == 2) ? (2 * gpz - v) : v;
    }
};

__device__ __forceinline__ void load_cell(Cell &s, const pb_cell_t *cells, const double *pool,
                                          int i, int mirror, double gpz)
{
    const pb_cell_t *c = &cells[i];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        s.x1[k] = c->x1[k]; s.x2[k] = c->x2[k]; s.wv[k] = c->wv[k]; s.papex[k] = c->papex[k];
    }
    s.len = c->len; s.wid = c->wid; s.thick = c->thick; s.vol = c->vol; s.npv = c->npv;
    s.pv = pool + 3 * (long long)c->pvoff;
    s.mirror = mirror; s.gpz = gpz;
    if (mirror) {
        s.x1[2] = 2 * gpz - s.x1[2];
        s.x2[2] = 2 * gpz - s.x2[2];
        s.wv[2] = -s.wv[2];
        s.papex[2] = 2 * gpz - s.papex[2];
    }
}

__device__ __forceinline__ double dot3(const double *a, const double *b)
{ return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ void cross3(const double *a, const double *b, double *c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ void tangent(const Cell &s, double *t)
{
#pragma unroll
    for (int c = 0; c < 3; c++) t[c] = (s.x2[c] - s.x1[c]) / s.len;
}
__device__ __forceinline__ double center_dist(const Cell &a, const Cell &b)
{
    double d[3];
#pragma unroll
    for (int i = 0; i < 3; i++) d[i] = 0.5 * (b.x1[i] + b.x2[i]) - 0.5 * (a.x1[i] + a.x2[i]);
    return sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
}
__device__ __forceinline__ double lmax_len(const Cell &a, const Cell &b)
{ return (a.len > b.len) ? a.len : b.len; }
__device__ __forceinline__ double lmax_all(const Cell &a, const Cell &b)
{
    double l = lmax_len(a, b);
    if (a.wid > l) l = a.wid;
    if (b.wid > l) l = b.wid;
    return l;
}
__device__ __forceinline__ void frame(const Cell &s, double *t, double *w, double *nv, double *c)
{
#pragma unroll
    for (int i = 0; i < 3; i++) {
        t[i] = (s.x2[i] - s.x1[i]) / s.len;
        w[i] = s.wv[i];
        c[i] = 0.5 * (s.x1[i] + s.x2[i]);
    }
    cross3(t, w, nv);
}

// ------------------------------------------------------------ pair classes
enum { PT_WIRE = 0, PT_RIBBON = 1, PT_HL = 2, PT_POLY = 3 };

__device__ __forceinline__ int is_parallel(const Cell &s1, const Cell &s2)
{
    double t1[3], t2[3], c[3];
    tangent(s1, t1);
    tangent(s2, t2);
    cross3(t1, t2, c);
    return sqrt(dot3(c, c)) < 1e-9;                       // partial.c:176-188
}

// volume.c:92-110 (HL_RFAR = 8)
__device__ int bar_use_hl(const Cell &s1, const Cell &s2)
{
    double t1[3], w1[3], n1[3], c1[3], t2[3], w2[3], n2[3], c2[3];
    frame(s1, t1, w1, n1, c1);
    frame(s2, t2, w2, n2, c2);
    if (fabs(dot3(t1, t2)) < 1 - 1e-9) return 0;
    if (fabs(dot3(w1, w2)) < 1 - 1e-9) return 0;
    return center_dist(s1, s2) <= 8.0 * lmax_all(s1, s2);
}

// dispatch order of partial.c:256-317
__device__ __forceinline__ int pair_type(const Cell &s1, const Cell &s2)
{
    if (s1.npv > 0 || s2.npv > 0) return PT_POLY;
    if (s1.vol && s2.vol && bar_use_hl(s1, s2)) return PT_HL;
    if (s1.wid > 0 || s2.wid > 0) return PT_RIBBON;
    return PT_WIRE;
}

// partial.c:166-173
__device__ __forceinline__ int corr_nsub(const Cell &s1, const Cell &s2, double kw)
{
    const int n = 2 + (int)(kw * lmax_len(s1, s2));
    return n > 8 ? 8 : n;
}
// partial.c:197-213
__device__ __forceinline__ double ribbon_ratio(const Cell &s1, const Cell &s2)
{
    const double l = lmax_all(s1, s2);
    return (l > 0) ? center_dist(s1, s2) / l : 0;
}
// partial.c:216-227
__device__ __forceinline__ int ribbon_nsub(const Cell &s1, const Cell &s2, double kw)
{
    int n = (ribbon_ratio(s1, s2) > 2) ? 1 : 2;
    n += (int)(kw * lmax_all(s1, s2));
    return n > 4 ? 4 : n;
}
// partial.c:244-249
__device__ __forceinline__ int ribbon_nq(const Cell &s1, const Cell &s2)
{
    const double r = ribbon_ratio(s1, s2);
    return (r <= 2.5) ? 8 : (r <= 10) ? 4 : 2;
}

// ------------------------------------------------------------ thin wires
__device__ __forceinline__ double fpar(double x, double d)          // partial.c:49-52
{ return x * asinh(x / d) - sqrt(x * x + d * d); }
__device__ __forceinline__ double neumann_self(double l, double a)  // partial.c:55-58
{ return 2 * (l * asinh(l / a) - sqrt(l * l + a * a) + a); }

// static 1/R composite Gauss (partial.c:61-99, mode 0)
__device__ double gauss_static(const Cell &s1, const Cell &s2, double aeff, int nsub)
{
    const double a2 = aeff * aeff;
    double sr = 0;
    for (int i1 = 0; i1 < nsub; i1++)
        for (int i2 = 0; i2 < nsub; i2++)
            for (int i = 0; i < 8; i++) {
                const double u = (i1 + 0.5 * (1 + cXG8[i])) / nsub;
                double q1[3];
#pragma unroll
                for (int c = 0; c < 3; c++) q1[c] = s1.x1[c] + (s1.x2[c] - s1.x1[c]) * u;
                for (int j = 0; j < 8; j++) {
                    const double v = (i2 + 0.5 * (1 + cXG8[j])) / nsub;
                    const double dx = s2.x1[0] + (s2.x2[0] - s2.x1[0]) * v - q1[0];
                    const double dy = s2.x1[1] + (s2.x2[1] - s2.x1[1]) * v - q1[1];
                    const double dz = s2.x1[2] + (s2.x2[2] - s2.x1[2]) * v - q1[2];
                    const double r = sqrt(dx * dx + dy * dy + dz * dz + a2);
                    sr += cWG8[i] * cWG8[j] / r;
                }
            }
    return s1.len * s2.len * 0.25 / ((double)nsub * nsub) * sr;
}

// partial.c:102-163
__device__ double neumann_pair(const Cell &s1, const Cell &s2, double a1, double a2)
{
    const double aeff = 0.5 * (a1 + a2);
    double t1[3];
    tangent(s1, t1);
    const double lmax = lmax_len(s1, s2);
    if (is_parallel(s1, s2)) {
        const double p1 = 0, p2 = s1.len;
        double r1[3], r2[3], perp[3];
#pragma unroll
        for (int c = 0; c < 3; c++) { r1[c] = s2.x1[c] - s1.x1[c]; r2[c] = s2.x2[c] - s1.x1[c]; }
        double b1 = dot3(r1, t1), b2 = dot3(r2, t1);
        if (b1 > b2) { const double t = b1; b1 = b2; b2 = t; }
        const double d1 = dot3(r1, t1);
#pragma unroll
        for (int c = 0; c < 3; c++) perp[c] = r1[c] - d1 * t1[c];
        const double d = sqrt(dot3(perp, perp) + aeff * aeff);
        return fpar(p2 - b1, d) - fpar(p2 - b2, d) - fpar(p1 - b1, d) + fpar(p1 - b2, d);
    }
    const double rc = center_dist(s1, s2);
    if (rc > 20 * lmax) return s1.len * s2.len / rc;
    return gauss_static(s1, s2, aeff, (rc > 2 * lmax) ? 1 : 4);
}

// ------------------------------------------------------------ ribbons
__device__ __forceinline__ double phi_rect(double u, double v, double z)   // surface.c:48-60
{
    const double az = fabs(z), uz = u * u + z * z, vz = v * v + z * z;
    double t = 0;
    if (uz > 0) t += u * asinh(v / sqrt(uz));
    if (vz > 0) t += v * asinh(u / sqrt(vz));
    if (az > 0) t -= az * atan2(u * v, az * sqrt(uz + v * v));
    return t;
}

// rectangle potential with a precomputed frame of s (surface.c:76-91)
struct RectFrame { double t[3], w[3], nv[3], c[3], hl, hw; };
__device__ __forceinline__ void rect_frame(const Cell &s, RectFrame &f)
{
    frame(s, f.t, f.w, f.nv, f.c);
    f.hl = 0.5 * s.len;
    f.hw = 0.5 * s.wid;
}
__device__ __forceinline__ double rect_potential(const RectFrame &f, const double *pt)
{
    double d[3];
#pragma unroll
    for (int i = 0; i < 3; i++) d[i] = pt[i] - f.c[i];
    const double u = dot3(d, f.t), v = dot3(d, f.w), z = dot3(d, f.nv);
    return phi_rect(u + f.hl, v + f.hw, z) - phi_rect(u - f.hl, v + f.hw, z)
         - phi_rect(u + f.hl, v - f.hw, z) + phi_rect(u - f.hl, v - f.hw, z);
}

// surface.c:102-131
__device__ double ribbon_static(const Cell &s1, const Cell &s2, int nsub, int nq)
{
    const double *xg = (nq >= 8) ? cXG8 : (nq >= 4) ? cXG4 : cXG2;
    const double *wg = (nq >= 8) ? cWG8 : (nq >= 4) ? cWG4 : cWG2;
    const int n = (nq >= 8) ? 8 : (nq >= 4) ? 4 : 2;
    double t1[3], w1[3], n1[3], c1[3];
    frame(s1, t1, w1, n1, c1);
    RectFrame f2;
    rect_frame(s2, f2);
    double sum = 0;
    for (int ia = 0; ia < nsub; ia++)
        for (int ib = 0; ib < nsub; ib++)
            for (int i = 0; i < n; i++) {
                const double a = s1.len * ((ia + 0.5 * (1 + xg[i])) / nsub - 0.5);
                for (int j = 0; j < n; j++) {
                    const double b = s1.wid * ((ib + 0.5 * (1 + xg[j])) / nsub - 0.5);
                    double pt[3];
#pragma unroll
                    for (int k = 0; k < 3; k++) pt[k] = c1[k] + a * t1[k] + b * w1[k];
                    sum += wg[i] * wg[j] * rect_potential(f2, pt);
                }
            }
    return s1.len * sum / (4 * s2.wid * (double)nsub * nsub);
}

// ------------------------------------------------------------ volume bars
__device__ double hl_F(double x, double y, double z)                     // volume.c:44-71
{
    const double x2 = x * x, y2 = y * y, z2 = z * z;
    const double R = sqrt(x2 + y2 + z2);
    const double yz = y2 + z2, xz = x2 + z2, xy = x2 + y2;
    double t = 0;
    if ((x != 0) && (yz > 0)) t += (y2 * z2 / 4 - y2 * y2 / 24 - z2 * z2 / 24) * x * asinh(x / sqrt(yz));
    if ((y != 0) && (xz > 0)) t += (x2 * z2 / 4 - x2 * x2 / 24 - z2 * z2 / 24) * y * asinh(y / sqrt(xz));
    if ((z != 0) && (xy > 0)) t += (x2 * y2 / 4 - x2 * x2 / 24 - y2 * y2 / 24) * z * asinh(z / sqrt(xy));
    t += (x2 * x2 + y2 * y2 + z2 * z2 - 3 * (x2 * y2 + y2 * z2 + z2 * x2)) * R / 60;
    if (z != 0) t -= (x * y * z * z2 / 6) * atan((x * y) / (z * R));
    if (y != 0) t -= (x * y * y2 * z / 6) * atan((x * z) / (y * R));
    if (x != 0) t -= (x * x2 * y * z / 6) * atan((y * z) / (x * R));
    return t;
}

__device__ double bar_pair(const Cell &s1, const Cell &s2)               // volume.c:114-155
{
    double t1[3], w1[3], n1[3], c1[3], t2[3], w2[3], n2[3], c2[3];
    frame(s1, t1, w1, n1, c1);
    frame(s2, t2, w2, n2, c2);
    const double a = s1.thick, b = s1.wid, c = s1.len, d = s2.thick, e = s2.wid, f = s2.len;
    double rc[3];
#pragma unroll
    for (int i = 0; i < 3; i++) rc[i] = c2[i] - c1[i];
    const double E = dot3(rc, n1) + (a - d) / 2;
    const double P = dot3(rc, w1) + (b - e) / 2;
    const double L3 = dot3(rc, t1) + (c - f) / 2;
    const double q[4] = {E - a, E + d - a, E + d, E};
    const double r[4] = {P - b, P + e - b, P + e, P};
    const double s[4] = {L3 - c, L3 + f - c, L3 + f, L3};
    double sum = 0;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 4; k++) {
                const double sgn = (((i + j + k) % 2) == 0) ? 1.0 : -1.0;
                sum += sgn * hl_F(q[i], r[j], s[k]);
            }
    return sum / (a * b * d * e);
}

// ------------------------------------------------------------ polygons
// Newell normal (|n| = 2 area), polygon.c:46-58
__device__ void poly_normal2(const Cell &s, double *nv)
{
    nv[0] = nv[1] = nv[2] = 0;
    for (int k = 0; k < s.npv; k++) {
        const int k2 = (k + 1) % s.npv;
        const double a[3] = {s.pvx(k, 0), s.pvx(k, 1), s.pvx(k, 2)};
        const double b[3] = {s.pvx(k2, 0), s.pvx(k2, 1), s.pvx(k2, 2)};
        double c[3];
        cross3(a, b, c);
        nv[0] += c[0]; nv[1] += c[1]; nv[2] += c[2];
    }
}

// polygon.c:68-131 with the unit normal precomputed (poly_normal2 of the same ring)
__device__ double poly_potential(const Cell &s, const double *nh, const double *pt)
{
    double d0[3], rho[3];
#pragma unroll
    for (int i = 0; i < 3; i++) d0[i] = pt[i] - s.pvx(0, i);
    const double z = dot3(d0, nh), az = fabs(z);
#pragma unroll
    for (int i = 0; i < 3; i++) rho[i] = pt[i] - z * nh[i];
    double sum = 0;
    for (int k = 0; k < s.npv; k++) {
        const int k2 = (k + 1) % s.npv;
        double a[3], b[3], e[3], ra[3], rb[3], mh[3];
#pragma unroll
        for (int i = 0; i < 3; i++) { a[i] = s.pvx(k, i); b[i] = s.pvx(k2, i); e[i] = b[i] - a[i]; }
        const double el = sqrt(dot3(e, e));
        if (el <= 0) continue;
        const double sh[3] = {e[0] / el, e[1] / el, e[2] / el};
        cross3(sh, nh, mh);
#pragma unroll
        for (int i = 0; i < 3; i++) { ra[i] = a[i] - rho[i]; rb[i] = b[i] - rho[i]; }
        const double lm = dot3(ra, sh), lp = dot3(rb, sh), t0 = dot3(ra, mh);
        const double r02 = t0 * t0 + z * z;
        const double rm = sqrt(lm * lm + r02), rp = sqrt(lp * lp + r02);
        if (r02 <= 0) continue;
        const double sp = (lp >= 0) ? (rp + lp) : (r02 / (rp - lp));
        const double sm = (lm >= 0) ? (rm + lm) : (r02 / (rm - lm));
        sum += t0 * log(sp / sm);
        if (az > 0) sum -= az * (atan((t0 * lp) / (r02 + az * rp)) - atan((t0 * lm) / (r02 + az * rm)));
    }
    return fabs(sum);
}

__device__ __forceinline__ double tri_area(const double *a, const double *b, const double *c)
{
    double u[3], v[3], w[3];
#pragma unroll
    for (int i = 0; i < 3; i++) { u[i] = b[i] - a[i]; v[i] = c[i] - a[i]; }
    cross3(u, v, w);
    return 0.5 * sqrt(dot3(w, w));
}

// inner analytic potential of s2 at pt (polygon.c:271-274)
struct Inner {
    const Cell *s;
    double nh[3];
    int poly;
    RectFrame rf;
    double n2;
};
__device__ __forceinline__ void inner_setup(Inner &in, const Cell &s)
{
    in.s = &s;
    in.poly = s.npv > 0;
    if (in.poly) {
        double nv[3];
        poly_normal2(s, nv);
        in.n2 = sqrt(dot3(nv, nv));
        const double d = in.n2 > 0 ? in.n2 : 1;
        in.nh[0] = nv[0] / d; in.nh[1] = nv[1] / d; in.nh[2] = nv[2] / d;
    } else {
        rect_frame(s, in.rf);
    }
}
__device__ __forceinline__ double inner_potential(const Inner &in, const double *pt)
{
    if (in.poly) return (in.n2 <= 0) ? 0.0 : poly_potential(*in.s, in.nh, pt);
    return rect_potential(in.rf, pt);
}

// outer quadrature of s1 (polygon.c:170-268) summed against the inner potential of s2
__device__ double outer_sum(const Cell &s1, int nsub, int n7, const Inner &in)
{
    double sum = 0;
    if (s1.npv > 0) {
        const int nq = n7 ? 7 : 3;
        const int ns = (nsub >= 2) ? 4 : 1;
        for (int k = 0; k < s1.npv; k++) {
            const int k2 = (k + 1) % s1.npv;
            const double b[3] = {s1.pvx(k, 0), s1.pvx(k, 1), s1.pvx(k, 2)};
            const double c[3] = {s1.pvx(k2, 0), s1.pvx(k2, 1), s1.pvx(k2, 2)};
            const double *a = s1.papex;
            const double at = tri_area(a, b, c);
            if (at <= 0) continue;
            for (int t = 0; t < ns; t++) {
                double v0[3], v1[3], v2[3];
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    double b0[3] = {1, 0, 0}, b1[3] = {0, 1, 0}, b2[3] = {0, 0, 1};
                    if (ns == 4)
                        for (int j = 0; j < 3; j++) { b0[j] = cSUB[t][0][j]; b1[j] = cSUB[t][1][j]; b2[j] = cSUB[t][2][j]; }
                    v0[i] = b0[0] * a[i] + b0[1] * b[i] + b0[2] * c[i];
                    v1[i] = b1[0] * a[i] + b1[1] * b[i] + b1[2] * c[i];
                    v2[i] = b2[0] * a[i] + b2[1] * b[i] + b2[2] * c[i];
                }
                const double sat = at / ns;
                for (int q = 0; q < nq; q++) {
                    const double *tb = n7 ? cTB7[q] : cTB3[q];
                    const double tw = n7 ? cTW7[q] : cTW3[q];
                    double px[3];
#pragma unroll
                    for (int i = 0; i < 3; i++) px[i] = tb[0] * v0[i] + tb[1] * v1[i] + tb[2] * v2[i];
                    sum += (tw * sat) * inner_potential(in, px);
                }
            }
        }
        return sum;
    }
    if (s1.wid <= 0) {
        for (int is = 0; is < nsub; is++)
            for (int q = 0; q < 4; q++) {
                const double u = (is + 0.5 * (1 + cXG4[q])) / nsub;
                double px[3];
#pragma unroll
                for (int i = 0; i < 3; i++) px[i] = s1.x1[i] + (s1.x2[i] - s1.x1[i]) * u;
                sum += (0.5 * cWG4[q] * s1.len / nsub) * inner_potential(in, px);
            }
        return sum;
    }
    double t[3], c[3];
#pragma unroll
    for (int i = 0; i < 3; i++) { t[i] = (s1.x2[i] - s1.x1[i]) / s1.len; c[i] = 0.5 * (s1.x1[i] + s1.x2[i]); }
    for (int is = 0; is < nsub; is++)
        for (int q = 0; q < 4; q++) {
            const double a = s1.len * ((is + 0.5 * (1 + cXG4[q])) / nsub - 0.5);
            for (int j = 0; j < 4; j++) {
                const double bb = s1.wid * (0.5 * cXG4[j]);
                double px[3];
#pragma unroll
                for (int i = 0; i < 3; i++) px[i] = c[i] + a * t[i] + bb * s1.wv[i];
                sum += (0.25 * cWG4[q] * cWG4[j] * s1.len * s1.wid / nsub) * inner_potential(in, px);
            }
        }
    return sum;
}

// polygon.c:283-302
__device__ double poly_static(const Cell &s1, const Cell &s2, int nsub, int n7)
{
    const Cell *o = &s1, *i = &s2;
    if ((s2.npv <= 0) && (s2.wid <= 0)) {
        if ((s1.npv <= 0) && (s1.wid <= 0)) return 0;
        o = &s2; i = &s1;
    }
    Inner in;
    inner_setup(in, *i);
    const double sum = outer_sum(*o, nsub, n7, in);
    const double w1 = (o->wid > 0) ? o->wid : 1, w2 = (i->wid > 0) ? i->wid : 1;
    return sum / (w1 * w2);
}

// ------------------------------------------------------------ static part of pair_k
// Static (k-independent for a fixed nsub level) part of neumann_pair_k
// (partial.c:256-317) / neumann_self_k (partial.c:320-328). `same` reproduces the
// pointer identity test of partial.c:276 (self term).
__device__ double static_term(const Cell &s1, const Cell &s2, int same, double a1, double a2, double kw)
{
    if (same && s1.wid <= 0 && s1.npv <= 0) return neumann_self(s1.len, a1);
    const int ty = pair_type(s1, s2);
    if (ty == PT_POLY) {
        const double rc = center_dist(s1, s2), lmax = lmax_all(s1, s2);
        if ((rc > 20 * lmax) && !same) return s1.len * s2.len / rc;
        return poly_static(s1, s2, (rc < 2 * lmax) ? 2 : 1, (rc <= 5.0 * lmax) ? 1 : 0);
    }
    if (ty == PT_HL) return bar_pair(s1, s2);
    if (ty == PT_RIBBON) return ribbon_static(s1, s2, ribbon_nsub(s1, s2, kw), ribbon_nq(s1, s2));
    if (kw <= 0) return neumann_pair(s1, s2, a1, a2);
    const double aeff = 0.5 * (a1 + a2);
    return is_parallel(s1, s2) ? neumann_pair(s1, s2, a1, a2)
                               : gauss_static(s1, s2, aeff, corr_nsub(s1, s2, kw));
}
