/*
 * peec_oracle.c — CPU restatement of the reference's frequency-sweep hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see peec_oracle.h). Plain FP64 C, written from the
 * reference's algorithms; every function names the reference file:line it follows.
 * Loop orders follow the reference so that sums are formed in the same order.
 *
 * Reference files (paths within the OpenPEEC project):
 *   src/partial.c  thin-wire Neumann integrals, dispatch, images, Lp entries
 *   src/surface.c  ribbon cells (rectangle potential closed form + Gauss)
 *   src/volume.c   Hoer-Love closed form for aligned bars
 *   src/polygon.c  Wilton polygon potential + triangle Gauss rules
 *   src/potential.c charge-cell grouping and P entries
 *   src/skin.c, src/mna.c, src/lu.c, src/solve.c
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "peec_oracle.h"

/* Physical constants defined exactly as the reference (include/peec.h:31-34). */
#define O_PI   (4.0 * atan(1.0))
#define O_C0   (2.99792458e8)
#define O_MU0  (4.0 * O_PI * 1e-7)
#define O_EPS0 (1.0 / (O_C0 * O_C0 * O_MU0))
#define O_PMAX 64                       /* polygon ring limit (include/peec.h:56) */

typedef struct { double r, i; } cx;
static cx cmk(double r, double i) { cx z = {r, i}; return z; }
static cx cadd(cx a, cx b) { return cmk(a.r + b.r, a.i + b.i); }
static cx csub(cx a, cx b) { return cmk(a.r - b.r, a.i - b.i); }
static cx cmul(cx a, cx b) { return cmk(a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r); }
static cx crmul(double s, cx a) { return cmk(s * a.r, s * a.i); }
static double cabs_(cx z) { return sqrt(z.r * z.r + z.i * z.i); }
/* complex.h:40-57 : division / inverse returning 0 for a zero divisor */
static cx cdiv(cx a, cx b)
{
    if ((fabs(b.r) <= 0) && (fabs(b.i) <= 0)) return cmk(0, 0);
    const double d = b.r * b.r + b.i * b.i;
    return cmk((a.r * b.r + a.i * b.i) / d, (a.i * b.r - a.r * b.i) / d);
}
static cx cinv(cx z)
{
    const double n2 = z.r * z.r + z.i * z.i;
    if (n2 <= 0) return cmk(0, 0);
    return cmk(z.r / n2, -z.i / n2);
}

/* A cell as seen by the kernels: record + its polygon ring. Mirrored cells own a copy. */
typedef struct {
    pb_cell_t c;
    const double *pv;
    double ring[3 * O_PMAX];
} ocell;

struct or_prob {
    int nseg, nchg, ncell, npv;
    pb_cell_t *seg, *chg;
    double *pv;
    int *chgnode;
    int capacitance, retardation, skin, gp;
    double gpz, gmin;
    int nport; pb_port_t *port;
    int nlump; pb_lump_t *lump;
    int nmut; pb_mutual_t *mut;
    int maxid;
    /* potential.c:29-114 */
    int *cellid, *cellof, *csoff, *csidx;
    double *carea;
    /* mna.c:16-113 */
    int *nodemap, nnode, refnode, offL, offV, offS, nunknown, nind, nvsrc;
};

static void view(const or_prob *o, const pb_cell_t *c, ocell *v)
{
    v->c = *c;
    v->pv = (c->npv > 0) ? &o->pv[3 * c->pvoff] : NULL;
}

/* ---------------------------------------------------------------- quadrature tables */
/* 8/4/2-point Gauss-Legendre on [-1,1] (partial.c:113-122, surface.c:26-37). */
static const double XG8[8] = {
    -0.9602898564975363, -0.7966664774136267, -0.5255324099163290, -0.1834346424956498,
     0.1834346424956498,  0.5255324099163290,  0.7966664774136267,  0.9602898564975363};
static const double WG8[8] = {
     0.1012285362903763,  0.2223810344533745,  0.3137066458778873,  0.3626837833783620,
     0.3626837833783620,  0.3137066458778873,  0.2223810344533745,  0.1012285362903763};
static const double XG4[4] = {
    -0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526};
static const double WG4[4] = {
     0.3478548451374538,  0.6521451548625461, 0.6521451548625461, 0.3478548451374538};
static const double XG2[2] = {-0.5773502691896257, 0.5773502691896257};
static const double WG2[2] = {1.0, 1.0};
/* Triangle rules: 7-point degree 5 and 3-point degree 2 (polygon.c:134-152). */
static const double TW7[7] = {0.225, 0.1323941527885062, 0.1323941527885062,
    0.1323941527885062, 0.1259391805448271, 0.1259391805448271, 0.1259391805448271};
static const double TB7[7][3] = {
    {1.0 / 3, 1.0 / 3, 1.0 / 3},
    {0.0597158717897698, 0.4701420641051151, 0.4701420641051151},
    {0.4701420641051151, 0.0597158717897698, 0.4701420641051151},
    {0.4701420641051151, 0.4701420641051151, 0.0597158717897698},
    {0.7974269853530873, 0.1012865073234563, 0.1012865073234563},
    {0.1012865073234563, 0.7974269853530873, 0.1012865073234563},
    {0.1012865073234563, 0.1012865073234563, 0.7974269853530873}};
static const double TW3[3] = {1.0 / 3, 1.0 / 3, 1.0 / 3};
static const double TB3[3][3] = {
    {2.0 / 3, 1.0 / 6, 1.0 / 6}, {1.0 / 6, 2.0 / 3, 1.0 / 6}, {1.0 / 6, 1.0 / 6, 2.0 / 3}};

static double dot3(const double *a, const double *b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static void cross3(const double *a, const double *b, double *c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static void tangent(const pb_cell_t *s, double *t)
{
    for (int c = 0; c < 3; c++) t[c] = (s->x2[c] - s->x1[c]) / s->len;
}
static double center_dist(const pb_cell_t *a, const pb_cell_t *b)
{
    double d[3];
    for (int i = 0; i < 3; i++) d[i] = 0.5 * (b->x1[i] + b->x2[i]) - 0.5 * (a->x1[i] + a->x2[i]);
    return sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
}
/* largest of the two lengths and (optionally) the two widths */
static double cell_lmax(const pb_cell_t *a, const pb_cell_t *b, int with_wid)
{
    double l = (a->len > b->len) ? a->len : b->len;
    if (with_wid) {
        if (a->wid > l) l = a->wid;
        if (b->wid > l) l = b->wid;
    }
    return l;
}

/* --------------------------------------------------------------------- thin wires */
/* partial.c:49-52 */
static double fpar(double x, double d) { return x * asinh(x / d) - sqrt(x * x + d * d); }

/* partial.c:55-58 */
static double o_neumann_self(double l, double a)
{
    return 2 * (l * asinh(l / a) - sqrt(l * l + a * a) + a);
}

/* partial.c:61-99 : composite 8x8 Gauss over nsub x nsub sub-squares; mode 0 = 1/R,
 * mode 1 = (cos kR - 1 - j sin kR)/R */
static cx gauss_kernel(const pb_cell_t *s1, const pb_cell_t *s2, double aeff, double kw,
                       int nsub, int mode)
{
    const double a2 = aeff * aeff;
    double sr = 0, si = 0;
    for (int i1 = 0; i1 < nsub; i1++)
        for (int i2 = 0; i2 < nsub; i2++)
            for (int i = 0; i < 8; i++) {
                const double u = (i1 + 0.5 * (1 + XG8[i])) / nsub;
                double q1[3];
                for (int c = 0; c < 3; c++) q1[c] = s1->x1[c] + (s1->x2[c] - s1->x1[c]) * u;
                for (int j = 0; j < 8; j++) {
                    const double v = (i2 + 0.5 * (1 + XG8[j])) / nsub;
                    const double dx = s2->x1[0] + (s2->x2[0] - s2->x1[0]) * v - q1[0];
                    const double dy = s2->x1[1] + (s2->x2[1] - s2->x1[1]) * v - q1[1];
                    const double dz = s2->x1[2] + (s2->x2[2] - s2->x1[2]) * v - q1[2];
                    const double r = sqrt(dx * dx + dy * dy + dz * dz + a2);
                    const double w = WG8[i] * WG8[j];
                    if (mode == 0) {
                        sr += w / r;
                    } else {
                        sr += w * (cos(kw * r) - 1) / r;
                        si -= w * sin(kw * r) / r;
                    }
                }
            }
    const double fac = s1->len * s2->len * 0.25 / ((double)nsub * nsub);
    return cmk(fac * sr, fac * si);
}

static int parallel_axes(const pb_cell_t *s1, const pb_cell_t *s2)
{
    double t1[3], t2[3], c[3];
    tangent(s1, t1);
    tangent(s2, t2);
    cross3(t1, t2, c);
    return sqrt(dot3(c, c)) < 1e-9;            /* partial.c:176-188, :118-119 */
}

/* partial.c:102-163 : static pair (parallel closed form / far midpoint / Gauss) */
static double o_neumann_pair(const pb_cell_t *s1, const pb_cell_t *s2, double a1, double a2)
{
    const double aeff = 0.5 * (a1 + a2);
    double t1[3];
    tangent(s1, t1);
    const double lmax = cell_lmax(s1, s2, 0);
    if (parallel_axes(s1, s2)) {
        const double p1 = 0, p2 = s1->len;
        double r1[3], r2[3], perp[3];
        for (int c = 0; c < 3; c++) {
            r1[c] = s2->x1[c] - s1->x1[c];
            r2[c] = s2->x2[c] - s1->x1[c];
        }
        double b1 = dot3(r1, t1), b2 = dot3(r2, t1);
        if (b1 > b2) { const double t = b1; b1 = b2; b2 = t; }
        for (int c = 0; c < 3; c++) perp[c] = r1[c] - dot3(r1, t1) * t1[c];
        const double d = sqrt(dot3(perp, perp) + aeff * aeff);
        return fpar(p2 - b1, d) - fpar(p2 - b2, d) - fpar(p1 - b1, d) + fpar(p1 - b2, d);
    }
    const double rc = center_dist(s1, s2);
    if (rc > 20 * lmax) return s1->len * s2->len / rc;
    return gauss_kernel(s1, s2, aeff, 0, (rc > 2 * lmax) ? 1 : 4, 0).r;
}

/* partial.c:166-173 */
static int corr_nsub(const pb_cell_t *s1, const pb_cell_t *s2, double kw)
{
    int n = 2 + (int)(kw * cell_lmax(s1, s2, 0));
    return n > 8 ? 8 : n;
}
/* partial.c:197-213 */
static double ribbon_ratio(const pb_cell_t *s1, const pb_cell_t *s2)
{
    const double l = cell_lmax(s1, s2, 1);
    return (l > 0) ? center_dist(s1, s2) / l : 0;
}
/* partial.c:216-227 */
static int ribbon_nsub(const pb_cell_t *s1, const pb_cell_t *s2, double kw)
{
    int n = (ribbon_ratio(s1, s2) > 2) ? 1 : 2;
    n += (int)(kw * cell_lmax(s1, s2, 1));
    return n > 4 ? 4 : n;
}
/* partial.c:244-249 */
static int ribbon_nq(const pb_cell_t *s1, const pb_cell_t *s2)
{
    const double r = ribbon_ratio(s1, s2);
    return (r <= 2.5) ? 8 : (r <= 10) ? 4 : 2;
}

/* ------------------------------------------------------------------------ ribbons */
/* surface.c:48-60 */
static double phi_rect(double u, double v, double z)
{
    const double az = fabs(z), uz = u * u + z * z, vz = v * v + z * z;
    double t = 0;
    if (uz > 0) t += u * asinh(v / sqrt(uz));
    if (vz > 0) t += v * asinh(u / sqrt(vz));
    if (az > 0) t -= az * atan2(u * v, az * sqrt(uz + v * v));
    return t;
}
/* surface.c:63-73 (and volume.c:79-89) */
static void local_frame(const pb_cell_t *s, double *t, double *w, double *nv, double *c)
{
    for (int i = 0; i < 3; i++) {
        t[i] = (s->x2[i] - s->x1[i]) / s->len;
        w[i] = s->wv[i];
        c[i] = 0.5 * (s->x1[i] + s->x2[i]);
    }
    cross3(t, w, nv);
}
/* surface.c:76-91 */
static double rect_potential(const pb_cell_t *s, const double *pt)
{
    double t[3], w[3], nv[3], c[3], d[3];
    local_frame(s, t, w, nv, c);
    for (int i = 0; i < 3; i++) d[i] = pt[i] - c[i];
    const double u = dot3(d, t), v = dot3(d, w), z = dot3(d, nv);
    const double hl = 0.5 * s->len, hw = 0.5 * s->wid;
    return phi_rect(u + hl, v + hw, z) - phi_rect(u - hl, v + hw, z)
         - phi_rect(u + hl, v - hw, z) + phi_rect(u - hl, v - hw, z);
}
/* surface.c:102-131 */
static double ribbon_static(const pb_cell_t *s1, const pb_cell_t *s2, int nsub, int nq)
{
    const double *xg = (nq >= 8) ? XG8 : (nq >= 4) ? XG4 : XG2;
    const double *wg = (nq >= 8) ? WG8 : (nq >= 4) ? WG4 : WG2;
    const int n = (nq >= 8) ? 8 : (nq >= 4) ? 4 : 2;
    double t1[3], w1[3], n1[3], c1[3];
    local_frame(s1, t1, w1, n1, c1);
    double sum = 0;
    for (int ia = 0; ia < nsub; ia++)
        for (int ib = 0; ib < nsub; ib++)
            for (int i = 0; i < n; i++) {
                const double a = s1->len * ((ia + 0.5 * (1 + xg[i])) / nsub - 0.5);
                for (int j = 0; j < n; j++) {
                    const double b = s1->wid * ((ib + 0.5 * (1 + xg[j])) / nsub - 0.5);
                    double pt[3];
                    for (int k = 0; k < 3; k++) pt[k] = c1[k] + a * t1[k] + b * w1[k];
                    sum += wg[i] * wg[j] * rect_potential(s2, pt);
                }
            }
    return s1->len * sum / (4 * s2->wid * (double)nsub * nsub);
}
/* surface.c:134-178 */
static cx ribbon_corr(const pb_cell_t *s1, const pb_cell_t *s2, double kw, int nsub)
{
    double t1[3], w1[3], n1[3], c1[3], t2[3], w2[3], n2[3], c2[3];
    local_frame(s1, t1, w1, n1, c1);
    local_frame(s2, t2, w2, n2, c2);
    double sr = 0, si = 0;
    for (int ia = 0; ia < nsub; ia++)
        for (int ja = 0; ja < nsub; ja++)
            for (int i = 0; i < 4; i++) {
                const double a1 = s1->len * ((ia + 0.5 * (1 + XG4[i])) / nsub - 0.5);
                for (int j = 0; j < 4; j++) {
                    const double b1 = s1->wid * (0.5 * (1 + XG4[j]) - 0.5);
                    double pt[3];
                    for (int k = 0; k < 3; k++) pt[k] = c1[k] + a1 * t1[k] + b1 * w1[k];
                    for (int m = 0; m < 4; m++) {
                        const double a2 = s2->len * ((ja + 0.5 * (1 + XG4[m])) / nsub - 0.5);
                        for (int q = 0; q < 4; q++) {
                            const double b2 = s2->wid * (0.5 * (1 + XG4[q]) - 0.5);
                            const double dx = c2[0] + a2 * t2[0] + b2 * w2[0] - pt[0];
                            const double dy = c2[1] + a2 * t2[1] + b2 * w2[1] - pt[1];
                            const double dz = c2[2] + a2 * t2[2] + b2 * w2[2] - pt[2];
                            const double r = sqrt(dx * dx + dy * dy + dz * dz);
                            const double w = WG4[i] * WG4[j] * WG4[m] * WG4[q];
                            if (r > 1e-300) {
                                sr += w * (cos(kw * r) - 1) / r;
                                si -= w * sin(kw * r) / r;
                            } else {
                                si -= w * kw;
                            }
                        }
                    }
                }
            }
    const double fac = s1->len * s2->len / (16 * (double)nsub * nsub);
    return cmk(fac * sr, fac * si);
}

/* -------------------------------------------------------------------- volume bars */
/* volume.c:44-71 */
static double hl_F(double x, double y, double z)
{
    const double x2 = x * x, y2 = y * y, z2 = z * z;
    const double R = sqrt(x2 + y2 + z2);
    const double yz = y2 + z2, xz = x2 + z2, xy = x2 + y2;
    double t = 0;
    if ((x != 0) && (yz > 0))
        t += (y2 * z2 / 4 - y2 * y2 / 24 - z2 * z2 / 24) * x * asinh(x / sqrt(yz));
    if ((y != 0) && (xz > 0))
        t += (x2 * z2 / 4 - x2 * x2 / 24 - z2 * z2 / 24) * y * asinh(y / sqrt(xz));
    if ((z != 0) && (xy > 0))
        t += (x2 * y2 / 4 - x2 * x2 / 24 - y2 * y2 / 24) * z * asinh(z / sqrt(xy));
    t += (x2 * x2 + y2 * y2 + z2 * z2 - 3 * (x2 * y2 + y2 * z2 + z2 * x2)) * R / 60;
    if (z != 0) t -= (x * y * z * z2 / 6) * atan((x * y) / (z * R));
    if (y != 0) t -= (x * y * y2 * z / 6) * atan((x * z) / (y * R));
    if (x != 0) t -= (x * x2 * y * z / 6) * atan((y * z) / (x * R));
    return t;
}
/* volume.c:92-110 (HL_RFAR = 8, volume.c:41) */
static int bar_use_hl(const pb_cell_t *s1, const pb_cell_t *s2)
{
    double t1[3], w1[3], n1[3], c1[3], t2[3], w2[3], n2[3], c2[3];
    local_frame(s1, t1, w1, n1, c1);
    local_frame(s2, t2, w2, n2, c2);
    if (fabs(dot3(t1, t2)) < 1 - 1e-9) return 0;
    if (fabs(dot3(w1, w2)) < 1 - 1e-9) return 0;
    return center_dist(s1, s2) <= 8.0 * cell_lmax(s1, s2, 1);
}
/* volume.c:114-155 */
static double bar_pair(const pb_cell_t *s1, const pb_cell_t *s2)
{
    double t1[3], w1[3], n1[3], c1[3], t2[3], w2[3], n2[3], c2[3];
    local_frame(s1, t1, w1, n1, c1);
    local_frame(s2, t2, w2, n2, c2);
    const double a = s1->thick, b = s1->wid, c = s1->len;
    const double d = s2->thick, e = s2->wid, f = s2->len;
    double rc[3];
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

/* ----------------------------------------------------------------------- polygons */
/* polygon.c:46-58 (Newell normal, |n| = 2 area) */
static void poly_normal2(const ocell *s, double *nv)
{
    nv[0] = nv[1] = nv[2] = 0;
    for (int k = 0; k < s->c.npv; k++) {
        double c[3];
        cross3(&s->pv[3 * k], &s->pv[3 * ((k + 1) % s->c.npv)], c);
        for (int i = 0; i < 3; i++) nv[i] += c[i];
    }
}
/* polygon.c:68-131 */
static double poly_potential(const ocell *s, const double *pt)
{
    double nv[3];
    poly_normal2(s, nv);
    const double n2 = sqrt(dot3(nv, nv));
    if (n2 <= 0) return 0;
    const double nh[3] = {nv[0] / n2, nv[1] / n2, nv[2] / n2};
    double d0[3], rho[3];
    for (int i = 0; i < 3; i++) d0[i] = pt[i] - s->pv[i];
    const double z = dot3(d0, nh), az = fabs(z);
    for (int i = 0; i < 3; i++) rho[i] = pt[i] - z * nh[i];
    double sum = 0;
    for (int k = 0; k < s->c.npv; k++) {
        const double *a = &s->pv[3 * k];
        const double *b = &s->pv[3 * ((k + 1) % s->c.npv)];
        double e[3], ra[3], rb[3], mh[3];
        for (int i = 0; i < 3; i++) e[i] = b[i] - a[i];
        const double el = sqrt(dot3(e, e));
        if (el <= 0) continue;
        const double sh[3] = {e[0] / el, e[1] / el, e[2] / el};
        cross3(sh, nh, mh);
        for (int i = 0; i < 3; i++) { ra[i] = a[i] - rho[i]; rb[i] = b[i] - rho[i]; }
        const double lm = dot3(ra, sh), lp = dot3(rb, sh), t0 = dot3(ra, mh);
        const double r02 = t0 * t0 + z * z;
        const double rm = sqrt(lm * lm + r02), rp = sqrt(lp * lp + r02);
        if (r02 <= 0) continue;
        const double sp = (lp >= 0) ? (rp + lp) : (r02 / (rp - lp));
        const double sm = (lm >= 0) ? (rm + lm) : (r02 / (rm - lm));
        sum += t0 * log(sp / sm);
        if (az > 0)
            sum -= az * (atan((t0 * lp) / (r02 + az * rp)) - atan((t0 * lm) / (r02 + az * rm)));
    }
    return fabs(sum);
}
static double tri_area(const double *a, const double *b, const double *c)
{
    double u[3], v[3], w[3];
    for (int i = 0; i < 3; i++) { u[i] = b[i] - a[i]; v[i] = c[i] - a[i]; }
    cross3(u, v, w);
    return 0.5 * sqrt(dot3(w, w));
}
#define O_NQMAX (O_PMAX * 4 * 7)
/* polygon.c:170-221 : fan triangulation from papex, optional 4-way split, 7/3-pt rule */
static int poly_qpts(const ocell *s, int nsub, int n7, double *px, double *wt)
{
    static const double SUB[4][3][3] = {
        {{1, 0, 0}, {0.5, 0.5, 0}, {0.5, 0, 0.5}},
        {{0.5, 0.5, 0}, {0, 1, 0}, {0, 0.5, 0.5}},
        {{0.5, 0, 0.5}, {0, 0.5, 0.5}, {0, 0, 1}},
        {{0.5, 0.5, 0}, {0, 0.5, 0.5}, {0.5, 0, 0.5}}};
    const int nq = n7 ? 7 : 3;
    const double (*tb)[3] = n7 ? TB7 : TB3;
    const double *tw = n7 ? TW7 : TW3;
    int np = 0;
    for (int k = 0; k < s->c.npv; k++) {
        const double *b = &s->pv[3 * k];
        const double *c = &s->pv[3 * ((k + 1) % s->c.npv)];
        const double *a = s->c.papex;
        const double at = tri_area(a, b, c);
        if (at <= 0) continue;
        const int ns = (nsub >= 2) ? 4 : 1;
        for (int t = 0; t < ns; t++) {
            double v0[3], v1[3], v2[3];
            for (int i = 0; i < 3; i++) {
                double b0[3] = {1, 0, 0}, b1[3] = {0, 1, 0}, b2[3] = {0, 0, 1};
                if (ns == 4)
                    for (int j = 0; j < 3; j++) {
                        b0[j] = SUB[t][0][j]; b1[j] = SUB[t][1][j]; b2[j] = SUB[t][2][j];
                    }
                v0[i] = b0[0] * a[i] + b0[1] * b[i] + b0[2] * c[i];
                v1[i] = b1[0] * a[i] + b1[1] * b[i] + b1[2] * c[i];
                v2[i] = b2[0] * a[i] + b2[1] * b[i] + b2[2] * c[i];
            }
            const double sat = at / ns;
            for (int q = 0; q < nq; q++) {
                for (int i = 0; i < 3; i++)
                    px[3 * np + i] = tb[q][0] * v0[i] + tb[q][1] * v1[i] + tb[q][2] * v2[i];
                wt[np] = tw[q] * sat;
                np++;
            }
        }
    }
    return np;
}
/* polygon.c:224-268 */
static int cell_qpts(const ocell *s, int nsub, int n7, double *px, double *wt)
{
    if (s->c.npv > 0) return poly_qpts(s, nsub, n7, px, wt);
    int np = 0;
    if (s->c.wid <= 0) {
        for (int is = 0; is < nsub; is++)
            for (int q = 0; q < 4; q++) {
                const double u = (is + 0.5 * (1 + XG4[q])) / nsub;
                for (int i = 0; i < 3; i++)
                    px[3 * np + i] = s->c.x1[i] + (s->c.x2[i] - s->c.x1[i]) * u;
                wt[np] = 0.5 * WG4[q] * s->c.len / nsub;
                np++;
            }
        return np;
    }
    double t[3], c[3];
    for (int i = 0; i < 3; i++) {
        t[i] = (s->c.x2[i] - s->c.x1[i]) / s->c.len;
        c[i] = 0.5 * (s->c.x1[i] + s->c.x2[i]);
    }
    for (int is = 0; is < nsub; is++)
        for (int q = 0; q < 4; q++) {
            const double a = s->c.len * ((is + 0.5 * (1 + XG4[q])) / nsub - 0.5);
            for (int j = 0; j < 4; j++) {
                const double b = s->c.wid * (0.5 * XG4[j]);
                for (int i = 0; i < 3; i++) px[3 * np + i] = c[i] + a * t[i] + b * s->c.wv[i];
                wt[np] = 0.25 * WG4[q] * WG4[j] * s->c.len * s->c.wid / nsub;
                np++;
            }
        }
    return np;
}
/* polygon.c:283-302 */
static double poly_static(const ocell *s1, const ocell *s2, int nsub, int n7)
{
    if ((s2->c.npv <= 0) && (s2->c.wid <= 0)) {
        if ((s1->c.npv <= 0) && (s1->c.wid <= 0)) return 0;
        return poly_static(s2, s1, nsub, n7);
    }
    double *px = (double *)malloc(sizeof(double) * O_NQMAX * 3);
    double *wt = (double *)malloc(sizeof(double) * O_NQMAX);
    const int np = cell_qpts(s1, nsub, n7, px, wt);
    double sum = 0;
    for (int q = 0; q < np; q++)
        sum += wt[q] * ((s2->c.npv > 0) ? poly_potential(s2, &px[3 * q])
                                        : rect_potential(&s2->c, &px[3 * q]));
    free(px);
    free(wt);
    const double w1 = (s1->c.wid > 0) ? s1->c.wid : 1;
    const double w2 = (s2->c.wid > 0) ? s2->c.wid : 1;
    return sum / (w1 * w2);
}
/* polygon.c:305-334 */
static cx poly_corr(const ocell *s1, const ocell *s2, double kw)
{
    double *px1 = (double *)malloc(sizeof(double) * O_NQMAX * 3);
    double *wt1 = (double *)malloc(sizeof(double) * O_NQMAX);
    double *px2 = (double *)malloc(sizeof(double) * O_NQMAX * 3);
    double *wt2 = (double *)malloc(sizeof(double) * O_NQMAX);
    const int n1 = cell_qpts(s1, 1, 0, px1, wt1);
    const int n2 = cell_qpts(s2, 1, 0, px2, wt2);
    double sr = 0, si = 0;
    for (int i = 0; i < n1; i++)
        for (int j = 0; j < n2; j++) {
            const double dx = px2[3 * j] - px1[3 * i];
            const double dy = px2[3 * j + 1] - px1[3 * i + 1];
            const double dz = px2[3 * j + 2] - px1[3 * i + 2];
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            const double w = wt1[i] * wt2[j];
            if (r > 1e-300) {
                sr += w * (cos(kw * r) - 1) / r;
                si -= w * sin(kw * r) / r;
            } else {
                si -= w * kw;
            }
        }
    free(px1); free(wt1); free(px2); free(wt2);
    const double w1 = (s1->c.wid > 0) ? s1->c.wid : 1;
    const double w2 = (s2->c.wid > 0) ? s2->c.wid : 1;
    return cmk(sr / (w1 * w2), si / (w1 * w2));
}

/* ------------------------------------------------------------------ dispatch */
/* partial.c:256-317 ; `same` reproduces the pointer test s1 != s2 at :276 */
static cx pair_k(const ocell *s1, const ocell *s2, int same, double a1, double a2, double kw)
{
    const pb_cell_t *c1 = &s1->c, *c2 = &s2->c;
    if ((c1->npv > 0) || (c2->npv > 0)) {
        const double rc = center_dist(c1, c2), lmax = cell_lmax(c1, c2, 1);
        cx is;
        if ((rc > 20 * lmax) && !same) is = cmk(c1->len * c2->len / rc, 0);
        else is = cmk(poly_static(s1, s2, (rc < 2 * lmax) ? 2 : 1, (rc <= 5.0 * lmax) ? 1 : 0), 0);
        if (kw <= 0) return is;
        return cadd(is, poly_corr(s1, s2, kw));
    }
    if (c1->vol && c2->vol && bar_use_hl(c1, c2)) {
        const cx is = cmk(bar_pair(c1, c2), 0);
        if (kw <= 0) return is;
        return cadd(is, ribbon_corr(c1, c2, kw, ribbon_nsub(c1, c2, kw)));
    }
    if ((c1->wid > 0) || (c2->wid > 0)) {
        const int nsub = ribbon_nsub(c1, c2, kw);
        const cx is = cmk(ribbon_static(c1, c2, nsub, ribbon_nq(c1, c2)), 0);
        if (kw <= 0) return is;
        return cadd(is, ribbon_corr(c1, c2, kw, nsub));
    }
    if (kw <= 0) return cmk(o_neumann_pair(c1, c2, a1, a2), 0);
    const double aeff = 0.5 * (a1 + a2);
    const int nsub = corr_nsub(c1, c2, kw);
    const double is = parallel_axes(c1, c2) ? o_neumann_pair(c1, c2, a1, a2)
                                            : gauss_kernel(c1, c2, aeff, 0, nsub, 0).r;
    return cadd(cmk(is, 0), gauss_kernel(c1, c2, aeff, kw, nsub, 1));
}
/* partial.c:320-328 */
static cx self_k(const ocell *s, double a, double kw)
{
    if (s->c.wid > 0) return pair_k(s, s, 1, a, a, kw);
    const cx is = cmk(o_neumann_self(s->c.len, a), 0);
    if (kw <= 0) return is;
    return cadd(is, gauss_kernel(&s->c, &s->c, a, kw, corr_nsub(&s->c, &s->c, kw), 1));
}
/* partial.c:352-362 : z -> 2 gpz - z image of a cell (axis, wv, apex, ring) */
static void mirror(const ocell *s, double gpz, ocell *out)
{
    out->c = s->c;
    out->c.x1[2] = 2 * gpz - s->c.x1[2];
    out->c.x2[2] = 2 * gpz - s->c.x2[2];
    out->c.wv[2] = -s->c.wv[2];
    out->c.papex[2] = 2 * gpz - s->c.papex[2];
    out->pv = NULL;
    if (s->c.npv > 0) {
        for (int k = 0; k < 3 * s->c.npv; k++) out->ring[k] = s->pv[k];
        for (int k = 0; k < s->c.npv; k++) out->ring[3 * k + 2] = 2 * gpz - s->pv[3 * k + 2];
        out->pv = out->ring;
    }
}

/* partial.c:371-424 */
void or_lp_entry(const or_prob *o, int i, int j, double kw, double *out)
{
    const double coef = O_MU0 / (4 * O_PI);
    if (i > j) { const int t = i; i = j; j = t; }
    ocell *si = (ocell *)malloc(sizeof(ocell)), *sj = (ocell *)malloc(sizeof(ocell));
    ocell *mj = (ocell *)malloc(sizeof(ocell));
    view(o, &o->seg[i], si);
    view(o, &o->seg[j], sj);
    double t1[3], t2[3];
    tangent(&si->c, t1);
    cx v;
    if (i == j) {
        v = self_k(si, si->c.aL, kw);
        if (o->gp) {
            mirror(si, o->gpz, mj);
            const double tdm = t1[0] * t1[0] + t1[1] * t1[1] - t1[2] * t1[2];
            v = csub(v, crmul(tdm, pair_k(si, mj, 0, si->c.aL, si->c.aL, kw)));
        }
    } else {
        tangent(&sj->c, t2);
        const double tdot = dot3(t1, t2);
        const double tdm = t1[0] * t2[0] + t1[1] * t2[1] - t1[2] * t2[2];
        v = cmk(0, 0);
        if (tdot != 0) v = crmul(tdot, pair_k(si, sj, 0, si->c.aL, sj->c.aL, kw));
        if (o->gp && (tdm != 0)) {
            mirror(sj, o->gpz, mj);
            v = csub(v, crmul(tdm, pair_k(si, mj, 0, si->c.aL, sj->c.aL, kw)));
        }
    }
    free(si); free(sj); free(mj);
    out[0] = coef * v.r;
    out[1] = coef * v.i;
}

void or_pair_k(const or_prob *o, int i, int j, int mirror_j, double kw, double *out)
{
    ocell *si = (ocell *)malloc(sizeof(ocell)), *sj = (ocell *)malloc(sizeof(ocell));
    ocell *mj = (ocell *)malloc(sizeof(ocell));
    view(o, &o->seg[i], si);
    view(o, &o->seg[j], sj);
    cx v;
    if (mirror_j) {
        mirror(sj, o->gpz, mj);
        v = pair_k(si, mj, 0, si->c.aL, sj->c.aL, kw);
    } else if (i == j) {
        v = self_k(si, si->c.aL, kw);
    } else {
        v = pair_k(si, sj, 0, si->c.aL, sj->c.aL, kw);
    }
    free(si); free(sj); free(mj);
    out[0] = v.r;
    out[1] = v.i;
}

/* potential.c:124-150 */
void or_pot_entry(const or_prob *o, int i, int j, double kw, double *out)
{
    cx s = cmk(0, 0);
    ocell *a = (ocell *)malloc(sizeof(ocell)), *b = (ocell *)malloc(sizeof(ocell));
    ocell *m = (ocell *)malloc(sizeof(ocell));
    for (int e = o->csoff[i]; e < o->csoff[i + 1]; e++) {
        const int h1 = o->csidx[e];
        for (int g = o->csoff[j]; g < o->csoff[j + 1]; g++) {
            const int h2 = o->csidx[g];
            const int ia = (h1 <= h2) ? h1 : h2, ib = (h1 <= h2) ? h2 : h1;
            view(o, &o->chg[ia], a);
            view(o, &o->chg[ib], b);
            cx v = (ia == ib) ? self_k(a, a->c.aP, kw)
                              : pair_k(a, b, 0, a->c.aP, b->c.aP, kw);
            if (o->gp) {
                mirror(b, o->gpz, m);
                v = csub(v, pair_k(a, m, 0, a->c.aP, b->c.aP, kw));
            }
            s = cadd(s, v);
        }
    }
    free(a); free(b); free(m);
    const double sc = 1 / (4 * O_PI * O_EPS0 * o->carea[i] * o->carea[j]);
    out[0] = sc * s.r;
    out[1] = sc * s.i;
}

void or_lp_fill(const or_prob *o, double kw, double *lp)
{
    const int n = o->nseg;
    int i;
#pragma omp parallel for schedule(dynamic)
    for (i = 0; i < n; i++)
        for (int j = i; j < n; j++) or_lp_entry(o, i, j, kw, &lp[2 * ((size_t)i * n + j)]);
    for (i = 0; i < n; i++)
        for (int j = 0; j < i; j++) {
            lp[2 * ((size_t)i * n + j)] = lp[2 * ((size_t)j * n + i)];
            lp[2 * ((size_t)i * n + j) + 1] = lp[2 * ((size_t)j * n + i) + 1];
        }
}

void or_pot_fill(const or_prob *o, double kw, double *pm)
{
    const int n = o->ncell;
    int i;
#pragma omp parallel for schedule(dynamic)
    for (i = 0; i < n; i++)
        for (int j = 0; j < n; j++) or_pot_entry(o, i, j, kw, &pm[2 * ((size_t)i * n + j)]);
}

/* --------------------------------------------------------------- skin / zint */
/* skin.c:23-56 */
static cx i0_over_i1(cx z)
{
    if (cabs_(z) < 15.0) {
        const cx z2 = cmul(z, z);
        cx i0 = cmk(1, 0), t = cmk(1, 0);
        for (int k = 1; k <= 60; k++) {
            t = crmul(1.0 / (4.0 * k * k), cmul(t, z2));
            i0 = cadd(i0, t);
            if (cabs_(t) < 1e-17 * cabs_(i0)) break;
        }
        cx s = cmk(1, 0);
        t = cmk(1, 0);
        for (int k = 1; k <= 60; k++) {
            t = crmul(1.0 / (4.0 * k * (k + 1)), cmul(t, z2));
            s = cadd(s, t);
            if (cabs_(t) < 1e-17 * cabs_(s)) break;
        }
        return cdiv(i0, cmul(crmul(0.5, z), s));
    }
    const cx u = cinv(z), u2 = cmul(u, u), u3 = cmul(u2, u);
    return cadd(cadd(cmk(1, 0), crmul(0.5, u)), cadd(crmul(0.375, u2), crmul(0.375, u3)));
}
/* skin.c:59-77 */
static cx zint_round(double len, double a, double sigma, double f)
{
    if ((sigma <= 0) || (len <= 0) || (a <= 0)) return cmk(0, 0);
    const double rdc = len / (sigma * O_PI * a * a), om = 2 * O_PI * f;
    if (om <= 0) return cmk(rdc, 0);
    const double delta = sqrt(2 / (om * O_MU0 * sigma)), q = a / delta;
    const cx ratio = i0_over_i1(cmk(q, q));
    const double kf = 1 / (2 * O_PI * a * delta * sigma);
    return crmul(len, cmul(cmk(kf, kf), ratio));
}
/* skin.c:91-109 */
static cx zint_bar(double len, double area, double perim, double sigma, double f)
{
    if ((sigma <= 0) || (len <= 0) || (area <= 0) || (perim <= 0)) return cmk(0, 0);
    const double rdc = len / (sigma * area), om = 2 * O_PI * f;
    if (om <= 0) return cmk(rdc, 0);
    const double delta = sqrt(2 / (om * O_MU0 * sigma));
    const double rhf = len / (sigma * delta * perim);
    const double ldc = O_MU0 * len / (8 * O_PI), lhf = rhf / om;
    const double r = sqrt(rdc * rdc + rhf * rhf);
    const double l = ldc * lhf / sqrt(ldc * ldc + lhf * lhf);
    return cmk(r, om * l);
}
/* skin.c:112-133 */
static cx zint_seg(const pb_cell_t *s, double f)
{
    if (s->diel) return cmk(0, 0);
    if (s->vol) return cmk(s->res, 0);
    return (s->shape == PB_SHAPE_ROUND) ? zint_round(s->len, s->radius, s->sigma, f)
                                        : zint_bar(s->len, s->area, s->perim, s->sigma, f);
}
/* mna.c:128-138 */
static cx zint_diel(const pb_cell_t *s, double om, double f)
{
    if (s->frelax > 0) {
        const cx er = cadd(cmk(s->epsinf, 0), cdiv(cmk(s->epss - s->epsinf, 0), cmk(1, f / s->frelax)));
        return cinv(cmk(om * s->gfac * (-er.i), om * s->gfac * (er.r - 1)));
    }
    return crmul(1 / om, cinv(cmk(s->gexc, s->cexc)));
}
/* mna.c:254-258 */
void or_zint(const or_prob *o, int k, double f, double *out)
{
    const pb_cell_t *s = &o->seg[k];
    const cx z = s->diel ? zint_diel(s, 2 * O_PI * f, f) : o->skin ? zint_seg(s, f)
                                                                  : cmk(s->res, 0);
    out[0] = z.r;
    out[1] = z.i;
}

/* ------------------------------------------------------------------- setup */
or_prob *or_create(const pb_problem_t *pb)
{
    or_prob *o = (or_prob *)calloc(1, sizeof(or_prob));
    o->nseg = pb->nseg; o->nchg = pb->nchg; o->npv = pb->npv;
    o->seg = (pb_cell_t *)malloc(sizeof(pb_cell_t) * (pb->nseg > 0 ? pb->nseg : 1));
    o->chg = (pb_cell_t *)malloc(sizeof(pb_cell_t) * (pb->nchg > 0 ? pb->nchg : 1));
    o->chgnode = (int *)malloc(sizeof(int) * (pb->nchg > 0 ? pb->nchg : 1));
    o->pv = (double *)malloc(sizeof(double) * 3 * (pb->npv > 0 ? pb->npv : 1));
    if (pb->nseg) memcpy(o->seg, pb->seg, sizeof(pb_cell_t) * pb->nseg);
    if (pb->nchg) {
        memcpy(o->chg, pb->chg, sizeof(pb_cell_t) * pb->nchg);
        memcpy(o->chgnode, pb->chgnode, sizeof(int) * pb->nchg);
    }
    if (pb->npv) memcpy(o->pv, pb->pv, sizeof(double) * 3 * pb->npv);
    o->capacitance = pb->capacitance; o->retardation = pb->retardation;
    o->skin = pb->skin; o->gp = pb->gp; o->gpz = pb->gpz; o->gmin = pb->gmin;
    o->nport = pb->nport;
    o->port = (pb_port_t *)malloc(sizeof(pb_port_t) * (pb->nport > 0 ? pb->nport : 1));
    if (pb->nport) memcpy(o->port, pb->port, sizeof(pb_port_t) * pb->nport);
    o->nlump = pb->nlump;
    o->lump = (pb_lump_t *)malloc(sizeof(pb_lump_t) * (pb->nlump > 0 ? pb->nlump : 1));
    if (pb->nlump) memcpy(o->lump, pb->lump, sizeof(pb_lump_t) * pb->nlump);
    o->nmut = pb->nmut;
    o->mut = (pb_mutual_t *)malloc(sizeof(pb_mutual_t) * (pb->nmut > 0 ? pb->nmut : 1));
    if (pb->nmut) memcpy(o->mut, pb->mut, sizeof(pb_mutual_t) * pb->nmut);
    o->maxid = pb->maxid;

    /* potential.c:29-62 : cells in order of first appearance of the node id */
    const int nh = o->nchg;
    o->cellid = (int *)malloc(sizeof(int) * (nh > 0 ? nh : 1));
    o->cellof = (int *)malloc(sizeof(int) * (nh > 0 ? nh : 1));
    o->ncell = 0;
    for (int h = 0; h < nh; h++) {
        int found = -1;
        for (int i = 0; i < o->ncell; i++)
            if (o->cellid[i] == o->chgnode[h]) { found = i; break; }
        if (found < 0) { found = o->ncell; o->cellid[o->ncell++] = o->chgnode[h]; }
        o->cellof[h] = found;
    }
    o->carea = (double *)calloc(o->ncell > 0 ? o->ncell : 1, sizeof(double));
    for (int h = 0; h < nh; h++) o->carea[o->cellof[h]] += o->chg[h].len;
    /* potential.c:72-97 : cell -> sub-cell CSR */
    o->csoff = (int *)calloc(o->ncell + 1, sizeof(int));
    o->csidx = (int *)malloc(sizeof(int) * (nh > 0 ? nh : 1));
    for (int h = 0; h < nh; h++) o->csoff[o->cellof[h] + 1]++;
    for (int i = 0; i < o->ncell; i++) o->csoff[i + 1] += o->csoff[i];
    {
        int *fill = (int *)malloc(sizeof(int) * (o->ncell + 1));
        memcpy(fill, o->csoff, sizeof(int) * (o->ncell + 1));
        for (int h = 0; h < nh; h++) o->csidx[fill[o->cellof[h]]++] = h;
        free(fill);
    }

    /* mna.c:16-84 : node numbering */
    const int nid = o->maxid + 1;
    int *used = (int *)calloc(nid, sizeof(int));
    for (int i = 0; i < o->nlump; i++) { used[o->lump[i].n1] = 1; used[o->lump[i].n2] = 1; }
    for (int i = 0; i < o->nport; i++) { used[o->port[i].n1] = 1; used[o->port[i].n2] = 1; }
    for (int i = 0; i < o->nseg; i++) { used[o->seg[i].n1] = 1; used[o->seg[i].n2] = 1; }
    const int usecap = o->capacitance && (o->ncell > 0);
    o->refnode = (usecap || used[0]) ? 0 : o->port[0].n2;
    o->nodemap = (int *)malloc(sizeof(int) * nid);
    int idx = 0;
    for (int id = 0; id < nid; id++) {
        if (id == o->refnode) o->nodemap[id] = -1;
        else if (!used[id]) o->nodemap[id] = -2;
        else o->nodemap[id] = idx++;
    }
    free(used);
    o->nnode = idx;
    o->nind = o->nvsrc = 0;
    for (int i = 0; i < o->nlump; i++) {
        if (o->lump[i].kind == PB_LUMP_L) o->nind++;
        if (o->lump[i].kind == PB_LUMP_V) o->nvsrc++;
    }
    o->offL = o->nnode;
    o->offV = o->offL + o->nind;
    o->offS = o->offV + o->nvsrc;
    o->nunknown = o->offS + o->nseg;
    return o;
}

void or_destroy(or_prob *o)
{
    if (!o) return;
    free(o->seg); free(o->chg); free(o->chgnode); free(o->pv); free(o->port);
    free(o->lump); free(o->mut); free(o->cellid); free(o->cellof); free(o->carea);
    free(o->csoff); free(o->csidx); free(o->nodemap);
    free(o);
}

void or_sizes(const or_prob *o, int *out)
{
    out[0] = o->nseg; out[1] = o->nchg; out[2] = o->ncell; out[3] = o->nnode;
    out[4] = o->nunknown; out[5] = o->offS; out[6] = o->refnode; out[7] = o->offL;
    out[8] = o->offV;
}

void or_cellmap(const or_prob *o, int *cellid, int *cellof, double *carea)
{
    for (int i = 0; i < o->ncell; i++) { cellid[i] = o->cellid[i]; carea[i] = o->carea[i]; }
    for (int h = 0; h < o->nchg; h++) cellof[h] = o->cellof[h];
}

/* ---------------------------------------------------------------------- MNA */
static void stamp(double *a, int n, int i, int j, cx v)
{
    if (i < 0 || j < 0) return;                 /* mna.c:154-159 */
    a[2 * ((size_t)i * n + j)] += v.r;
    a[2 * ((size_t)i * n + j) + 1] += v.i;
}

/* mna.c:175-308 (dense, skiplp = 0) */
void or_mna_assemble(const or_prob *o, double f, const double *lp, const double *cmat,
                     double *a)
{
    const int n = o->nunknown;
    const double om = 2 * O_PI * f;
    const int *map = o->nodemap;
    memset(a, 0, sizeof(double) * 2 * (size_t)n * n);
    if (o->gmin > 0)
        for (int i = 0; i < o->nnode; i++) stamp(a, n, i, i, cmk(o->gmin, 0));
    for (int pass = 0; pass < 2; pass++)        /* resistors then capacitors */
        for (int e = 0; e < o->nlump; e++) {
            const pb_lump_t *l = &o->lump[e];
            if (l->kind != (pass ? PB_LUMP_C : PB_LUMP_R)) continue;
            const int i1 = map[l->n1], i2 = map[l->n2];
            const cx y = pass ? cmk(0, om * l->val) : cmk(1 / l->val, 0);
            stamp(a, n, i1, i1, y); stamp(a, n, i2, i2, y);
            stamp(a, n, i1, i2, crmul(-1, y)); stamp(a, n, i2, i1, crmul(-1, y));
        }
    int il = 0;
    double *lval = (double *)malloc(sizeof(double) * (o->nind > 0 ? o->nind : 1));
    for (int e = 0; e < o->nlump; e++) {
        const pb_lump_t *l = &o->lump[e];
        if (l->kind != PB_LUMP_L) continue;
        const int i1 = map[l->n1], i2 = map[l->n2], r = o->offL + il;
        lval[il] = l->val;
        stamp(a, n, i1, r, cmk(1, 0)); stamp(a, n, r, i1, cmk(1, 0));
        stamp(a, n, i2, r, cmk(-1, 0)); stamp(a, n, r, i2, cmk(-1, 0));
        stamp(a, n, r, r, cmk(0, -om * l->val));
        il++;
    }
    for (int e = 0; e < o->nmut; e++) {
        const int r1 = o->offL + o->mut[e].l1, r2 = o->offL + o->mut[e].l2;
        const double m = o->mut[e].k * sqrt(lval[o->mut[e].l1] * lval[o->mut[e].l2]);
        stamp(a, n, r1, r2, cmk(0, -om * m)); stamp(a, n, r2, r1, cmk(0, -om * m));
    }
    free(lval);
    int iv = 0;
    for (int e = 0; e < o->nlump; e++) {
        const pb_lump_t *l = &o->lump[e];
        if (l->kind != PB_LUMP_V) continue;
        const int i1 = map[l->n1], i2 = map[l->n2], r = o->offV + iv;
        stamp(a, n, i1, r, cmk(1, 0)); stamp(a, n, r, i1, cmk(1, 0));
        stamp(a, n, i2, r, cmk(-1, 0)); stamp(a, n, r, i2, cmk(-1, 0));
        iv++;
    }
    for (int k = 0; k < o->nseg; k++) {          /* mna.c:244-266 */
        const int i1 = map[o->seg[k].n1], i2 = map[o->seg[k].n2], rk = o->offS + k;
        stamp(a, n, i1, rk, cmk(1, 0)); stamp(a, n, rk, i1, cmk(1, 0));
        stamp(a, n, i2, rk, cmk(-1, 0)); stamp(a, n, rk, i2, cmk(-1, 0));
        double z[2];
        or_zint(o, k, f, z);
        stamp(a, n, rk, rk, cmk(-z[0], -z[1]));
        for (int m = 0; m < o->nseg; m++) {
            const double *l = &lp[2 * ((size_t)k * o->nseg + m)];
            stamp(a, n, rk, o->offS + m, cmul(cmk(0, -om), cmk(l[0], l[1])));
        }
    }
    if (o->capacitance && (o->ncell > 0) && cmat != NULL) {  /* mna.c:286-295 */
        for (int i = 0; i < o->ncell; i++) {
            const int mi = map[o->cellid[i]];
            for (int j = 0; j < o->ncell; j++) {
                const int mj = map[o->cellid[j]];
                const double *c = &cmat[2 * ((size_t)i * o->ncell + j)];
                stamp(a, n, mi, mj, cmul(cmk(0, om), cmk(c[0], c[1])));
            }
        }
    }
}

/* ----------------------------------------------------------------------- LU */
static double mag(const double *z) { return fabs(z[0]) + fabs(z[1]); }

/* lu.c:16-66 */
int or_lu_decomp(int n, double *a, int *piv)
{
    for (int k = 0; k < n; k++) {
        int ip = k;
        double amax = mag(&a[2 * ((size_t)k * n + k)]);
        for (int i = k + 1; i < n; i++) {
            const double m = mag(&a[2 * ((size_t)i * n + k)]);
            if (m > amax) { amax = m; ip = i; }
        }
        piv[k] = ip;
        if (amax < 1e-30) return k;
        if (ip != k)
            for (int j = 0; j < 2 * n; j++) {
                const double t = a[2 * (size_t)k * n + j];
                a[2 * (size_t)k * n + j] = a[2 * (size_t)ip * n + j];
                a[2 * (size_t)ip * n + j] = t;
            }
        const cx pinv = cinv(cmk(a[2 * ((size_t)k * n + k)], a[2 * ((size_t)k * n + k) + 1]));
        int i;
#pragma omp parallel for if ((n - k) > 64)
        for (i = k + 1; i < n; i++) {
            double *ri = &a[2 * (size_t)i * n];
            const double *rk = &a[2 * (size_t)k * n];
            const cx lik = cmul(cmk(ri[2 * k], ri[2 * k + 1]), pinv);
            ri[2 * k] = lik.r;
            ri[2 * k + 1] = lik.i;
            for (int j = k + 1; j < n; j++) {
                const cx u = cmul(lik, cmk(rk[2 * j], rk[2 * j + 1]));
                ri[2 * j] -= u.r;
                ri[2 * j + 1] -= u.i;
            }
        }
    }
    return -1;
}

/* lu.c:68-96 */
void or_lu_solve(int n, const double *a, const int *piv, double *b)
{
    for (int k = 0; k < n; k++)
        if (piv[k] != k) {
            double t = b[2 * k]; b[2 * k] = b[2 * piv[k]]; b[2 * piv[k]] = t;
            t = b[2 * k + 1]; b[2 * k + 1] = b[2 * piv[k] + 1]; b[2 * piv[k] + 1] = t;
        }
    for (int i = 1; i < n; i++) {
        cx s = cmk(b[2 * i], b[2 * i + 1]);
        for (int j = 0; j < i; j++)
            s = csub(s, cmul(cmk(a[2 * ((size_t)i * n + j)], a[2 * ((size_t)i * n + j) + 1]),
                             cmk(b[2 * j], b[2 * j + 1])));
        b[2 * i] = s.r; b[2 * i + 1] = s.i;
    }
    for (int i = n - 1; i >= 0; i--) {
        cx s = cmk(b[2 * i], b[2 * i + 1]);
        for (int j = i + 1; j < n; j++)
            s = csub(s, cmul(cmk(a[2 * ((size_t)i * n + j)], a[2 * ((size_t)i * n + j) + 1]),
                             cmk(b[2 * j], b[2 * j + 1])));
        s = cmul(s, cinv(cmk(a[2 * ((size_t)i * n + i)], a[2 * ((size_t)i * n + i) + 1])));
        b[2 * i] = s.r; b[2 * i + 1] = s.i;
    }
}

/* -------------------------------------------------------------------- sweep */
/* solve.c:239-370 (dense path): per frequency fill (retarded) -> C = P^-1 ->
 * assemble -> LU -> one 1 A port excitation per port (mna.c:367-376) -> Z column. */
int or_sweep(const or_prob *o, int nfreq, const double *freq, double *zmat, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    const int n = o->nunknown, ns = o->nseg, nc = o->ncell, np = o->nport;
    double *lp = (double *)malloc(sizeof(double) * 2 * (size_t)(ns > 0 ? ns : 1) * (ns > 0 ? ns : 1));
    double *pm = (double *)malloc(sizeof(double) * 2 * (size_t)(nc > 0 ? nc : 1) * (nc > 0 ? nc : 1));
    double *cm = (double *)malloc(sizeof(double) * 2 * (size_t)(nc > 0 ? nc : 1) * (nc > 0 ? nc : 1));
    double *a = (double *)malloc(sizeof(double) * 2 * (size_t)n * n);
    double *b = (double *)malloc(sizeof(double) * 2 * (size_t)(n > nc ? n : nc));
    int *piv = (int *)malloc(sizeof(int) * (size_t)(n > nc ? n : nc));
    const int usecap = o->capacitance && nc > 0;
    int ret = 0;
    for (int ifr = 0; ifr < nfreq; ifr++) {
        const double f = freq[ifr];
        const double kw = o->retardation ? 2 * O_PI * f / O_C0 : 0;
        if (ifr == 0 || o->retardation) {
            or_lp_fill(o, kw, lp);
            if (usecap) {                            /* potential.c:258-281 */
                or_pot_fill(o, kw, pm);
                if (or_lu_decomp(nc, pm, piv) >= 0) { ret = PB_ERR_SINGULAR; break; }
                for (int j = 0; j < nc; j++) {
                    memset(b, 0, sizeof(double) * 2 * nc);
                    b[2 * j] = 1;
                    or_lu_solve(nc, pm, piv, b);
                    for (int i = 0; i < nc; i++) {
                        cm[2 * ((size_t)i * nc + j)] = b[2 * i];
                        cm[2 * ((size_t)i * nc + j) + 1] = b[2 * i + 1];
                    }
                }
            }
        }
        or_mna_assemble(o, f, lp, usecap ? cm : NULL, a);
        if (or_lu_decomp(n, a, piv) >= 0) { ret = PB_ERR_SINGULAR; break; }
        for (int j = 0; j < np; j++) {
            memset(b, 0, sizeof(double) * 2 * n);
            const int i1 = o->nodemap[o->port[j].n1], i2 = o->nodemap[o->port[j].n2];
            if (i1 >= 0) b[2 * i1] += 1;
            if (i2 >= 0) b[2 * i2] -= 1;
            or_lu_solve(n, a, piv, b);
            for (int i = 0; i < np; i++) {
                const int k1 = o->nodemap[o->port[i].n1], k2 = o->nodemap[o->port[i].n2];
                const double vr = (k1 < 0 ? 0 : b[2 * k1]) - (k2 < 0 ? 0 : b[2 * k2]);
                const double vi = (k1 < 0 ? 0 : b[2 * k1 + 1]) - (k2 < 0 ? 0 : b[2 * k2 + 1]);
                const size_t z = ((size_t)ifr * np + i) * np + j;
                zmat[2 * z] = vr;
                zmat[2 * z + 1] = vi;
            }
        }
    }
    free(lp); free(pm); free(cm); free(a); free(b); free(piv);
    return ret;
}

/* ------------------------------------------------------------------ plane wave
 * mna_rhs_planewave / pw_emf (src/mna.c:408-468) and the plane-wave branch of solve()
 * (src/solve.c:372-389), on the same dense MNA system as or_sweep. */
static double pw_sinc(double x) { return (fabs(x) < 1e-8) ? 1.0 : (sin(x) / x); }

static void pw_emf(const pb_cell_t *s, const double *rh, const double *ev, const double *e0,
                   double kw, double *out)
{
    double tv[3], rc[3];
    for (int c = 0; c < 3; c++) {
        tv[c] = (s->x2[c] - s->x1[c]) / s->len;
        rc[c] = 0.5 * (s->x1[c] + s->x2[c]);
    }
    const double et = ev[0] * tv[0] + ev[1] * tv[1] + ev[2] * tv[2];
    const double rt = rh[0] * tv[0] + rh[1] * tv[1] + rh[2] * tv[2];
    const double rr = rh[0] * rc[0] + rh[1] * rc[1] + rh[2] * rc[2];
    double amp = et * s->len * pw_sinc(0.5 * kw * s->len * rt);
    const double wl = sqrt(s->wv[0] * s->wv[0] + s->wv[1] * s->wv[1] + s->wv[2] * s->wv[2]);
    if (s->wid > 0 && wl > 0) {
        const double rw = (rh[0] * s->wv[0] + rh[1] * s->wv[1] + rh[2] * s->wv[2]) / wl;
        amp *= pw_sinc(0.5 * kw * s->wid * rw);
    }
    const double c = cos(kw * rr), sn = sin(kw * rr);
    out[0] = amp * (e0[0] * c - e0[1] * sn);
    out[1] = amp * (e0[0] * sn + e0[1] * c);
}

/* pwp = {theta_deg, phi_deg, pol, amp, phase_deg}; voc [2*nport*nfreq] (voc[i*nfreq+f]);
 * segipw [2*nfreq*nseg] or NULL. */
int or_planewave(const or_prob *o, int nfreq, const double *freq, const double *pwp,
                 double *voc, double *segipw)
{
    const int n = o->nunknown, ns = o->nseg, nc = o->ncell, np = o->nport;
    double *lp = (double *)malloc(sizeof(double) * 2 * (size_t)(ns > 0 ? ns : 1) * (ns > 0 ? ns : 1));
    double *pm = (double *)malloc(sizeof(double) * 2 * (size_t)(nc > 0 ? nc : 1) * (nc > 0 ? nc : 1));
    double *cm = (double *)malloc(sizeof(double) * 2 * (size_t)(nc > 0 ? nc : 1) * (nc > 0 ? nc : 1));
    double *a = (double *)malloc(sizeof(double) * 2 * (size_t)n * n);
    double *b = (double *)malloc(sizeof(double) * 2 * (size_t)(n > nc ? n : nc));
    int *piv = (int *)malloc(sizeof(int) * (size_t)(n > nc ? n : nc));
    const int usecap = o->capacitance && nc > 0;
    const double th = pwp[0] * O_PI / 180, ph = pwp[1] * O_PI / 180;
    const double st = sin(th), ct = cos(th), cp = cos(ph), sp = sin(ph);
    const double rh[3] = {st * cp, st * sp, ct};
    const double thh[3] = {ct * cp, ct * sp, -st};
    const double phh[3] = {-sp, cp, 0};
    double ev[3];
    for (int c = 0; c < 3; c++) ev[c] = ((int)pwp[2] == 2) ? phh[c] : thh[c];
    const double e0[2] = {pwp[3] * cos(pwp[4] * O_PI / 180), pwp[3] * sin(pwp[4] * O_PI / 180)};
    const double rh2[3] = {rh[0], rh[1], -rh[2]};
    const double ev2[3] = {-ev[0], -ev[1], ev[2]};
    int ret = 0;
    for (int ifr = 0; ifr < nfreq; ifr++) {
        const double f = freq[ifr];
        const double kw = o->retardation ? 2 * O_PI * f / O_C0 : 0;
        const double kwp = 2 * O_PI * f / O_C0;          /* the wave's own k (mna.c:437) */
        if (ifr == 0 || o->retardation) {
            or_lp_fill(o, kw, lp);
            if (usecap) {
                or_pot_fill(o, kw, pm);
                if (or_lu_decomp(nc, pm, piv) >= 0) { ret = PB_ERR_SINGULAR; break; }
                for (int j = 0; j < nc; j++) {
                    memset(b, 0, sizeof(double) * 2 * nc);
                    b[2 * j] = 1;
                    or_lu_solve(nc, pm, piv, b);
                    for (int i = 0; i < nc; i++) {
                        cm[2 * ((size_t)i * nc + j)] = b[2 * i];
                        cm[2 * ((size_t)i * nc + j) + 1] = b[2 * i + 1];
                    }
                }
            }
        }
        or_mna_assemble(o, f, lp, usecap ? cm : NULL, a);
        if (or_lu_decomp(n, a, piv) >= 0) { ret = PB_ERR_SINGULAR; break; }
        memset(b, 0, sizeof(double) * 2 * n);
        const double psi = 2 * kwp * rh[2] * o->gpz;
        const double e0r[2] = {e0[0] * cos(psi) - e0[1] * sin(psi), e0[0] * sin(psi) + e0[1] * cos(psi)};
        for (int k = 0; k < ns; k++) {
            double emf[2], r2[2];
            pw_emf(&o->seg[k], rh, ev, e0, kwp, emf);
            if (o->gp) {
                pw_emf(&o->seg[k], rh2, ev2, e0r, kwp, r2);
                emf[0] += r2[0];
                emf[1] += r2[1];
            }
            b[2 * (o->offS + k)] = -emf[0];
            b[2 * (o->offS + k) + 1] = -emf[1];
        }
        or_lu_solve(n, a, piv, b);
        for (int i = 0; i < np; i++) {
            const int k1 = o->nodemap[o->port[i].n1], k2 = o->nodemap[o->port[i].n2];
            voc[2 * ((size_t)i * nfreq + ifr)] = (k1 < 0 ? 0 : b[2 * k1]) - (k2 < 0 ? 0 : b[2 * k2]);
            voc[2 * ((size_t)i * nfreq + ifr) + 1] = (k1 < 0 ? 0 : b[2 * k1 + 1]) - (k2 < 0 ? 0 : b[2 * k2 + 1]);
        }
        if (segipw)
            for (int m = 0; m < ns; m++) {
                segipw[2 * ((size_t)ifr * ns + m)] = b[2 * (o->offS + m)];
                segipw[2 * ((size_t)ifr * ns + m) + 1] = b[2 * (o->offS + m) + 1];
            }
    }
    free(lp); free(pm); free(cm); free(a); free(b); free(piv);
    return ret;
}

/* ------------------------------------------------------------------ CPU timing
 * Same bounded samples as the reference harness, on the restatement (used as the CPU
 * baseline when the reference build is not available). */
#include <time.h>
static double or_now(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + 1e-9 * t.tv_nsec;
}

double or_time_entries(const or_prob *o, int which, int n, const int *ij, double kw)
{
    double sink = 0;
    const double t0 = or_now();
    int e;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : sink)
    for (e = 0; e < n; e++) {
        double v[2];
        if (which) or_pot_entry(o, ij[2 * e], ij[2 * e + 1], kw, v);
        else or_lp_entry(o, ij[2 * e], ij[2 * e + 1], kw, v);
        sink += v[0];
    }
    return (or_now() - t0) + 0 * sink;
}

double or_time_lu(int n, unsigned seed)
{
    double *a = (double *)malloc(sizeof(double) * 2 * (size_t)n * n);
    int *piv = (int *)malloc(sizeof(int) * (size_t)n);
    unsigned s = seed;
    for (size_t i = 0; i < 2 * (size_t)n * n; i++) {
        s = s * 1103515245u + 12345u;
        a[i] = ((s >> 8) & 0xffff) / 65536.0 - 0.5;
    }
    const double t0 = or_now();
    or_lu_decomp(n, a, piv);
    const double t1 = or_now();
    free(a);
    free(piv);
    return t1 - t0;
}

double or_time_solves(int n, int ncol)
{
    double *a = (double *)calloc(2 * (size_t)n * n, sizeof(double));
    double *b = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    int *piv = (int *)malloc(sizeof(int) * (size_t)n);
    for (size_t i = 0; i < (size_t)n * n; i++) a[2 * i] = (i % (n + 1)) == 0 ? n : 0.5 / (1 + i % 7);
    for (int i = 0; i < n; i++) piv[i] = i;
    const double t0 = or_now();
    for (int j = 0; j < ncol; j++) {
        memset(b, 0, sizeof(double) * 2 * n);
        b[2 * (j % n)] = 1;
        or_lu_solve(n, a, piv, b);
    }
    const double t1 = or_now();
    free(a); free(b); free(piv);
    return t1 - t0;
}

int or_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}
