/*
 * peec_shim.c — the reference solver's hot-path C entry points implemented on
 * libpeec_b200, so that the reference's own CLI (main.c), parser (input_data.c),
 * geometry builder (wire.c), output writers (output.c, farfield.c, transient.c) and skin
 * model (skin.c), compiled unchanged, run their sweep on the GPU. Linked with those files
 * it replaces partial.c, potential.c, mna.c, solve.c, lu.c, polygon.c, surface.c,
 * volume.c, hmatrix.c, iterative.c and precond.c: the kept files need exactly the
 * symbols below (include/peec.h prototypes).
 *
 *   lp_fill        partial.c:428-473   Lp at frequency f into p->lp (pb_lp_fill, FP64)
 *   pot_fill       potential.c:177-303 charge-cell grouping (potential.c:29-114) and the
 *                                      total-capacitance log line; P is filled on the GPU
 *   mna_numbering  mna.c:16-113        unknown numbering (the writers read nodemap)
 *   solve          solve.c:171-430     the sweep: pb_sweep (Z per port, segment currents),
 *                                      Kurokawa S, pb_planewave (Voc), pb_sources (node
 *                                      voltages), on the dense or the compressed path
 *   poly_area      polygon.c:60-65     polygon cell area (wire.c sizes panel cells with it)
 *   hmat_free      hmatrix.c           peec_free() releases p->hlp: never set here
 *
 *   lu_decomp      lu.c:16-66          dense complex LU on the GPU (pb_lu_decomp)
 *   lu_solve       lu.c:68-96          its substitutions (pb_lu_solve)
 *
 * One CLI run drives one peec_t; its GPU context is created on first use and lives until
 * exit. Errors print the reference's style of message ("*** ...") to stdout and the log
 * and return 1, as solve.c does; a missing GPU is such an error (no CPU fall back).
 * The cell charges of distribution = 1 (p->cellq) come from pb_sweep_dist, which never
 * forms C = P^-1; pot_fill therefore leaves p->cmat NULL (no kept file reads it).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "peec.h"
#include "../../include/peec_b200.h"

static struct {
    const peec_t *owner;
    pb_ctx *ctx;
} g_shim;

static void shim_release(void)
{
    if (g_shim.ctx) pb_destroy(g_shim.ctx);
    g_shim.ctx = NULL;
}

static void fail_msg(FILE *fp_log, const char *what, int code)
{
    printf("*** %s (GPU library error %d: %s)\n", what, code, pb_last_error());
    if (fp_log) fprintf(fp_log, "*** %s (GPU library error %d: %s)\n", what, code, pb_last_error());
}

/* seg_t -> pb_cell_t: the fields the hot path reads; the polygon ring goes to the pool. */
static void to_cell(const seg_t *s, pb_cell_t *c, int pvoff)
{
    memset(c, 0, sizeof(*c));
    for (int k = 0; k < 3; k++) {
        c->x1[k] = s->x1[k];
        c->x2[k] = s->x2[k];
        c->wv[k] = s->wv[k];
        c->papex[k] = s->papex[k];
    }
    c->len = s->len;
    c->wid = s->wid;
    c->thick = s->thick;
    c->aL = s->aL;
    c->aP = s->aP;
    c->radius = s->radius;
    c->area = s->area;
    c->perim = s->perim;
    c->sigma = s->sigma;
    c->res = s->res;
    c->cexc = s->cexc;
    c->gexc = s->gexc;
    c->gfac = s->gfac;
    c->epss = s->epss;
    c->epsinf = s->epsinf;
    c->frelax = s->frelax;
    c->n1 = s->n1;
    c->n2 = s->n2;
    c->shape = s->shape;
    c->vol = s->vol;
    c->diel = s->diel;
    c->npv = s->npv;
    c->pvoff = s->npv > 0 ? pvoff : 0;
}

/* The library context of p, built from the discretisation wire_build produced. */
static pb_ctx *shim_ctx(peec_t *p, FILE *fp_log)
{
    if (g_shim.ctx && g_shim.owner == p) return g_shim.ctx;
    shim_release();
    int npv = 0;
    for (int i = 0; i < p->nseg; i++) npv += p->seg[i].npv;
    for (int i = 0; i < p->nchg; i++) npv += p->chg[i].npv;
    pb_cell_t *seg = (pb_cell_t *)calloc((size_t)(p->nseg > 0 ? p->nseg : 1), sizeof(pb_cell_t));
    pb_cell_t *chg = (pb_cell_t *)calloc((size_t)(p->nchg > 0 ? p->nchg : 1), sizeof(pb_cell_t));
    double *pv = (double *)calloc((size_t)(3 * npv + 3), sizeof(double));
    pb_port_t *port = (pb_port_t *)calloc((size_t)(p->nport + 1), sizeof(pb_port_t));
    pb_lump_t *lump = (pb_lump_t *)calloc((size_t)(p->nres + p->ncap + p->nind + p->nsrc + 1), sizeof(pb_lump_t));
    pb_mutual_t *mut = (pb_mutual_t *)calloc((size_t)(p->nmut + 1), sizeof(pb_mutual_t));
    if (!seg || !chg || !pv || !port || !lump || !mut) {
        printf("%s\n", "*** memory allocation error (GPU problem)");
        free(seg); free(chg); free(pv); free(port); free(lump); free(mut);
        return NULL;
    }
    int off = 0;
    for (int i = 0; i < p->nseg; i++) {
        to_cell(&p->seg[i], &seg[i], off);
        memcpy(pv + 3 * off, p->seg[i].pv, sizeof(double) * 3 * (size_t)p->seg[i].npv);
        off += p->seg[i].npv;
    }
    for (int i = 0; i < p->nchg; i++) {
        to_cell(&p->chg[i], &chg[i], off);
        memcpy(pv + 3 * off, p->chg[i].pv, sizeof(double) * 3 * (size_t)p->chg[i].npv);
        off += p->chg[i].npv;
    }
    for (int i = 0; i < p->nport; i++) {
        port[i].n1 = p->port[i].n1;
        port[i].n2 = p->port[i].n2;
        port[i].z0 = p->port[i].z0;
    }
    /* lumped elements in the reference's stamping order R, C, L, V (mna.c:188-241) */
    int nl = 0;
    for (int i = 0; i < p->nres; i++, nl++) {
        lump[nl].kind = PB_LUMP_R; lump[nl].n1 = p->res[i].n1; lump[nl].n2 = p->res[i].n2; lump[nl].val = p->res[i].val;
    }
    for (int i = 0; i < p->ncap; i++, nl++) {
        lump[nl].kind = PB_LUMP_C; lump[nl].n1 = p->cap[i].n1; lump[nl].n2 = p->cap[i].n2; lump[nl].val = p->cap[i].val;
    }
    for (int i = 0; i < p->nind; i++, nl++) {
        lump[nl].kind = PB_LUMP_L; lump[nl].n1 = p->ind[i].n1; lump[nl].n2 = p->ind[i].n2; lump[nl].val = p->ind[i].val;
    }
    for (int i = 0; i < p->nsrc; i++) {
        if (!p->src[i].isvsrc) continue;
        lump[nl].kind = PB_LUMP_V; lump[nl].n1 = p->src[i].n1; lump[nl].n2 = p->src[i].n2; lump[nl].val = p->src[i].amp;
        nl++;
    }
    for (int i = 0; i < p->nmut; i++) {
        mut[i].l1 = p->mut[i].l1;
        mut[i].l2 = p->mut[i].l2;
        mut[i].k = p->mut[i].k;
    }
    pb_problem_t pr;
    memset(&pr, 0, sizeof(pr));
    pr.nseg = p->nseg; pr.seg = seg;
    pr.nchg = p->nchg; pr.chg = chg; pr.chgnode = p->chgnode;
    pr.npv = npv; pr.pv = pv;
    pr.maxid = p->maxid;
    pr.nport = p->nport; pr.port = port;
    pr.nlump = nl; pr.lump = lump;
    pr.nmut = p->nmut; pr.mut = mut;
    pr.capacitance = p->capacitance; pr.retardation = p->retardation; pr.skin = p->skin; pr.gp = p->gp;
    pr.gpz = p->gpz; pr.gmin = p->gmin;
    pb_ctx *c = NULL;
    const int r = pb_create(&pr, &c);
    free(seg); free(chg); free(pv); free(port); free(lump); free(mut);
    if (r != PB_OK) {
        fail_msg(fp_log, "GPU context", r);
        return NULL;
    }
    g_shim.ctx = c;
    g_shim.owner = p;
    atexit(shim_release);
    return c;
}

static double kw_of(const peec_t *p, double f)
{
    return p->retardation ? 2 * PI * f / C0 : 0.0;          /* partial.c:436 */
}

/* ------------------------------------------------------------------ partial inductance */
void lp_fill(peec_t *p, double f, FILE *fp_log)
{
    if (p->nseg <= 0) return;
    pb_ctx *c = shim_ctx(p, fp_log);
    if (!c) return;
    if (p->lp == NULL) {
        p->lp = (d_complex_t *)calloc((size_t)p->nseg * p->nseg, sizeof(d_complex_t));
        if (p->lp == NULL) {
            printf("%s\n", "*** memory allocation error (partial inductance)");
            return;
        }
    }
    const int r = pb_lp_fill(c, kw_of(p, f), PB_PREC_FP64, (double *)p->lp);
    if (r != PB_OK) fail_msg(fp_log, "partial inductance fill", r);
}

/* ------------------------------------------------------------------ dense LU */
/* lu_decomp: -1 on success, else the zero-pivot row (lu.c:16-66). A GPU failure is
 * reported on stdout and returned as row 0, a failure in the reference's convention. */
int lu_decomp(int n, d_complex_t *a, int *piv)
{
    const int r = pb_lu_decomp(n, (double *)a, piv);
    if (r < -1) {
        printf("*** GPU LU error: %s\n", pb_last_error());
        return 0;
    }
    return r;
}

void lu_solve(int n, const d_complex_t *a, const int *piv, d_complex_t *b)
{
    const int r = pb_lu_solve(n, (const double *)a, piv, (double *)b);
    if (r != PB_OK) printf("*** GPU LU solve error %d: %s\n", r, pb_last_error());
}

/* ------------------------------------------------------------------ charge cells */
/* Node cells in first-appearance order of the charge sub-cells, their summed lengths,
 * the cell -> sub-cell index and the length-weighted sub-cell centroids
 * (potential.c:29-114; the same grouping, so the writers' p->cellof agrees). */
static int cells(peec_t *p)
{
    if (p->cellof != NULL) return 0;
    const int nh = p->nchg;
    p->cellof = (int *)malloc((size_t)(nh > 0 ? nh : 1) * sizeof(int));
    p->cellid = (int *)malloc((size_t)(nh > 0 ? nh : 1) * sizeof(int));
    if (!p->cellof || !p->cellid) return 1;
    p->ncell = 0;
    for (int h = 0; h < nh; h++) {
        int found = -1;
        for (int i = 0; i < p->ncell && found < 0; i++)
            if (p->cellid[i] == p->chgnode[h]) found = i;
        if (found < 0) {
            found = p->ncell;
            p->cellid[p->ncell++] = p->chgnode[h];
        }
        p->cellof[h] = found;
    }
    const int nc = p->ncell;
    p->carea = (double *)calloc((size_t)(nc > 0 ? nc : 1), sizeof(double));
    p->csoff = (int *)calloc((size_t)(nc + 1), sizeof(int));
    p->csidx = (int *)malloc((size_t)(nh > 0 ? nh : 1) * sizeof(int));
    p->cpt = (double *)calloc((size_t)(nc > 0 ? nc : 1) * 3, sizeof(double));
    int *fill = (int *)malloc((size_t)(nc + 1) * sizeof(int));
    if (!p->carea || !p->csoff || !p->csidx || !p->cpt || !fill) {
        free(fill);
        return 1;
    }
    for (int h = 0; h < nh; h++) {
        p->carea[p->cellof[h]] += p->chg[h].len;
        p->csoff[p->cellof[h] + 1]++;
    }
    for (int i = 0; i < nc; i++) p->csoff[i + 1] += p->csoff[i];
    memcpy(fill, p->csoff, (size_t)(nc + 1) * sizeof(int));
    for (int h = 0; h < nh; h++) p->csidx[fill[p->cellof[h]]++] = h;
    free(fill);
    for (int i = 0; i < nc; i++) {
        double w = 0, x[3] = {0, 0, 0};
        for (int e = p->csoff[i]; e < p->csoff[i + 1]; e++) {
            const seg_t *s = &p->chg[p->csidx[e]];
            for (int q = 0; q < 3; q++) x[q] += s->len * 0.5 * (s->x1[q] + s->x2[q]);
            w += s->len;
        }
        for (int q = 0; q < 3; q++) p->cpt[3 * i + q] = (w > 0) ? (x[q] / w) : 0;
    }
    return 0;
}

/* ------------------------------------------------------------------ potential coefficients */
int pot_fill(peec_t *p, double f, FILE *fp_log)
{
    if (!p->capacitance || p->nchg <= 0) return 0;
    if (cells(p)) {
        printf("%s\n", "*** memory allocation error (potential)");
        return 1;
    }
    if (p->compress) {
        if (!p->clogged) {
            p->clogged = 1;
            printf("PEEC: capacitive cells = %d (compressed : charge unknowns)\n", p->ncell);
            fprintf(fp_log, "PEEC: capacitive cells = %d (compressed : charge unknowns)\n", p->ncell);
            fflush(fp_log);
        }
        return 0;
    }
    if (p->clogged) return 0;          /* the sweep fills P on the GPU; only the log line */
    pb_ctx *c = shim_ctx(p, fp_log);
    if (!c) return 1;
    const int nc = p->ncell;
    double *pm = (double *)malloc(sizeof(double) * 2 * (size_t)nc * nc);
    double *one = (double *)calloc(2 * (size_t)nc, sizeof(double));
    int *piv = (int *)malloc(sizeof(int) * (size_t)nc);
    if (!pm || !one || !piv) {
        free(pm); free(one); free(piv);
        printf("%s\n", "*** memory allocation error (potential)");
        return 1;
    }
    int r = pb_pot_fill(c, kw_of(p, f), PB_PREC_FP64, pm);
    int ising = -1;
    if (r == PB_OK) {
        ising = pb_lu_decomp(nc, pm, piv);
        if (ising < -1) r = PB_ERR_CUDA;
    }
    if (r == PB_OK && ising < 0) {
        /* total capacitance 1^T P^-1 1 (the sum of the entries of C = P^-1): one solve */
        for (int i = 0; i < nc; i++) one[2 * i] = 1.0;
        r = pb_lu_solve(nc, pm, piv, one);
    }
    if (r != PB_OK) {
        fail_msg(fp_log, "potential coefficients", r);
        free(pm); free(one); free(piv);
        return 1;
    }
    if (ising >= 0) {
        printf("*** singular potential coefficient matrix (row %d)\n", ising);
        fprintf(fp_log, "*** singular potential coefficient matrix (row %d)\n", ising);
        free(pm); free(one); free(piv);
        return 1;
    }
    double ctotal = 0;
    for (int i = 0; i < nc; i++) ctotal += one[2 * i];
    p->clogged = 1;
    printf("PEEC: capacitive cells = %d, total capacitance = %.6e F\n", nc, ctotal);
    fprintf(fp_log, "PEEC: capacitive cells = %d, total capacitance = %.6e F\n", nc, ctotal);
    fflush(fp_log);
    free(pm); free(one); free(piv);
    return 0;
}

/* ------------------------------------------------------------------ MNA numbering */
/* The reference's numbering (mna.c:16-113): node rows in id order without the reference
 * node, then inductor branches, voltage-source branches, segment branches (and cell
 * charges on the compressed path with capacitance). */
int mna_numbering(peec_t *p, FILE *fp_log)
{
    const int nid = p->maxid + 1;
    int *used = (int *)calloc((size_t)nid, sizeof(int));
    if (!used) return 1;
#define MARK(x) do { if ((x) >= 0 && (x) < nid) used[(x)] = 1; } while (0)
    for (int i = 0; i < p->nres; i++) { MARK(p->res[i].n1); MARK(p->res[i].n2); }
    for (int i = 0; i < p->ncap; i++) { MARK(p->cap[i].n1); MARK(p->cap[i].n2); }
    for (int i = 0; i < p->nind; i++) { MARK(p->ind[i].n1); MARK(p->ind[i].n2); }
    for (int i = 0; i < p->nsrc; i++) { MARK(p->src[i].n1); MARK(p->src[i].n2); }
    for (int i = 0; i < p->nport; i++) { MARK(p->port[i].n1); MARK(p->port[i].n2); }
    for (int i = 0; i < p->nseg; i++) { MARK(p->seg[i].n1); MARK(p->seg[i].n2); }
#undef MARK
    const int usecap = (p->capacitance && p->ncell > 0);
    p->refnode = (usecap || used[0]) ? 0 : p->port[0].n2;
    p->nodemap = (int *)malloc((size_t)nid * sizeof(int));
    if (!p->nodemap) { free(used); return 1; }
    int idx = 0;
    for (int id = 0; id < nid; id++)
        p->nodemap[id] = (id == p->refnode) ? -1 : (!used[id] ? -2 : idx++);
    p->nnode = idx;
    free(used);
    int nvsrc = 0;
    for (int i = 0; i < p->nsrc; i++)
        if (p->src[i].isvsrc) p->src[i].ibr = nvsrc++;
    p->offL = p->nnode;
    p->offV = p->offL + p->nind;
    p->offS = p->offV + nvsrc;
    p->nunknown = p->offS + p->nseg;
    p->offQ = p->nunknown;
    if (p->compress && p->capacitance && p->nchg > 0) {
        if (cells(p)) {
            printf("%s\n", "*** memory allocation error (potential cells)");
            return 1;
        }
        p->nunknown = p->offQ + p->ncell;
    }
    fprintf(fp_log, "MNA : %d nodes (reference = node %d), %d unknowns\n", p->nnode + 1, p->refnode, p->nunknown);
    return 0;
}

/* ------------------------------------------------------------------ polygon area */
/* Half the length of the polygon's Newell normal (the same evaluation order as
 * polygon.c:45-65, so that wire.c sizes every panel cell bit for bit as the reference). */
double poly_area(const seg_t *s)
{
    double nv[3] = {0, 0, 0};
    for (int k = 0; k < s->npv; k++) {
        const double *a = &s->pv[3 * k];
        const double *b = &s->pv[3 * ((k + 1) % s->npv)];
        nv[0] += (a[1] * b[2]) - (a[2] * b[1]);
        nv[1] += (a[2] * b[0]) - (a[0] * b[2]);
        nv[2] += (a[0] * b[1]) - (a[1] * b[0]);
    }
    return 0.5 * sqrt((nv[0] * nv[0]) + (nv[1] * nv[1]) + (nv[2] * nv[2]));
}

void hmat_free(struct hmat_t *h)
{
    (void)h;                           /* the shim never builds one: p->hlp stays NULL */
}

/* ------------------------------------------------------------------ the sweep */
/* Z -> S with per-port real reference resistances (power waves, Kurokawa):
 * S = sqrt(z0_j / z0_i) [(Z - Z0)(Z + Z0)^-1]_ij. Small dense complex Gauss-Jordan on the
 * host (np is the port count). Returns 1 when Z + Z0 is singular. */
static int z_to_s(peec_t *p, int ifreq)
{
    const int np = p->nport;
    double *m = (double *)malloc(sizeof(double) * 2 * np * 2 * np);   /* [np][2np] augmented */
    if (!m) return 1;
    const int w = 2 * np;
    for (int i = 0; i < np; i++)
        for (int j = 0; j < w; j++) {
            double re = 0, im = 0;
            if (j < np) {
                const d_complex_t z = p->zmat[ZIDX(p, ifreq, i, j)];
                re = z.r + (i == j ? p->port[i].z0 : 0);
                im = z.i;
            } else if (j - np == i) {
                re = 1;
            }
            m[2 * (i * w + j)] = re;
            m[2 * (i * w + j) + 1] = im;
        }
    for (int c = 0; c < np; c++) {
        int pr = c;
        double best = -1;
        for (int i = c; i < np; i++) {
            const double a = fabs(m[2 * (i * w + c)]) + fabs(m[2 * (i * w + c) + 1]);
            if (a > best) { best = a; pr = i; }
        }
        if (!(best > 0)) { free(m); return 1; }
        if (pr != c)
            for (int j = 0; j < w; j++)
                for (int q = 0; q < 2; q++) {
                    const double t = m[2 * (c * w + j) + q];
                    m[2 * (c * w + j) + q] = m[2 * (pr * w + j) + q];
                    m[2 * (pr * w + j) + q] = t;
                }
        const double ar = m[2 * (c * w + c)], ai = m[2 * (c * w + c) + 1], d = ar * ar + ai * ai;
        const double ir = ar / d, ii = -ai / d;
        for (int j = 0; j < w; j++) {
            const double xr = m[2 * (c * w + j)], xi = m[2 * (c * w + j) + 1];
            m[2 * (c * w + j)] = xr * ir - xi * ii;
            m[2 * (c * w + j) + 1] = xr * ii + xi * ir;
        }
        for (int i = 0; i < np; i++) {
            if (i == c) continue;
            const double fr = m[2 * (i * w + c)], fi = m[2 * (i * w + c) + 1];
            for (int j = 0; j < w; j++) {
                const double xr = m[2 * (c * w + j)], xi = m[2 * (c * w + j) + 1];
                m[2 * (i * w + j)] -= fr * xr - fi * xi;
                m[2 * (i * w + j) + 1] -= fr * xi + fi * xr;
            }
        }
    }
    for (int i = 0; i < np; i++)
        for (int j = 0; j < np; j++) {
            double sr = 0, si = 0;
            for (int k = 0; k < np; k++) {
                d_complex_t n = p->zmat[ZIDX(p, ifreq, i, k)];
                if (i == k) n.r -= p->port[i].z0;
                const double vr = m[2 * (k * w + np + j)], vi = m[2 * (k * w + np + j) + 1];
                sr += n.r * vr - n.i * vi;
                si += n.r * vi + n.i * vr;
            }
            const double fct = sqrt(p->port[j].z0 / p->port[i].z0);
            p->smat[ZIDX(p, ifreq, i, j)].r = fct * sr;
            p->smat[ZIDX(p, ifreq, i, j)].i = fct * si;
        }
    free(m);
    return 0;
}

int solve(peec_t *p, FILE *fp_log)
{
    const int nf = p->nfreq, np = p->nport;
    pb_ctx *c = shim_ctx(p, fp_log);
    if (!c) return 1;
    double *freq = (double *)malloc(sizeof(double) * (size_t)(nf > 0 ? nf : 1));
    const size_t nmat = (size_t)nf * np * np;
    p->zin = (d_complex_t *)calloc((size_t)np * nf + 1, sizeof(d_complex_t));
    p->zmat = (d_complex_t *)calloc(nmat + 1, sizeof(d_complex_t));
    p->smat = (d_complex_t *)calloc(nmat + 1, sizeof(d_complex_t));
    if (!freq || !p->zin || !p->zmat || !p->smat) {
        free(freq);
        printf("%s\n", "*** memory allocation error (matrix)");
        return 1;
    }
    for (int i = 0; i < nf; i++) freq[i] = freq_at(p, i);
    if ((p->dist || p->ffnth > 0) && p->nseg > 0)
        p->segi = (d_complex_t *)calloc((size_t)nf * np * p->nseg, sizeof(d_complex_t));
    if (p->dist && p->capacitance && p->ncell > 0)
        p->cellq = (d_complex_t *)calloc((size_t)nf * np * p->ncell, sizeof(d_complex_t));

    pb_sweep_opts o;
    memset(&o, 0, sizeof(o));
    o.fill_prec = PB_PREC_MIXED;
    o.lu = PB_LU_TC;
    o.form = PB_FORM_AUTO;
    o.accel = p->accel ? 8 : 0;         /* one FP32 factorisation per 8 frequencies + GMRES */
    o.compress = p->compress;
    o.ctol = p->ctol;
    pb_sweep_stats st;
    memset(&st, 0, sizeof(st));
    int r = pb_sweep_dist(c, nf, freq, &o, (double *)p->zmat, p->segi ? (double *)p->segi : NULL,
                          p->cellq ? (double *)p->cellq : NULL, &st);
    if (r != PB_OK) {
        if (r == PB_ERR_SINGULAR)
            fail_msg(fp_log, "singular matrix (floating node or ideal voltage source loop?)", r);
        else if (r == PB_ERR_NOCONV && p->compress)
            fail_msg(fp_log, "compression : GMRES did not converge", r);
        else
            fail_msg(fp_log, "sweep", r);
        free(freq);
        return 1;
    }
    for (int ifr = 0; ifr < nf; ifr++) {
        for (int j = 0; j < np; j++) p->zin[(size_t)j * nf + ifr] = p->zmat[ZIDX(p, ifr, j, j)];
        if (z_to_s(p, ifr)) {
            printf("*** singular (Z + Z0) at f = %.5e Hz\n", freq[ifr]);
            fprintf(fp_log, "*** singular (Z + Z0) at f = %.5e Hz\n", freq[ifr]);
            free(freq);
            return 1;
        }
    }
    if (p->compress) {
        fprintf(fp_log, "compression Lp : %d cells, %d far blocks + %d near blocks, tol = %.1e, %.2f MB (dense %.2f MB, %.1fx)\n",
                p->nseg, st.hmat_far, st.hmat_near, p->ctol > 0 ? p->ctol : 1e-6, st.hmat_mb, st.hmat_dense_mb,
                st.hmat_mb > 0 ? st.hmat_dense_mb / st.hmat_mb : 0.0);
        fprintf(fp_log, "compression : %d GMRES solves (avg %.1f iterations)\n", st.gmres_solves, st.gmres_its_avg);
    }
    if (p->accel)
        fprintf(fp_log, "acceleration : %d LU for %d frequencies, %d GMRES solves (avg %.1f iterations)\n",
                st.lu_count, nf, st.gmres_solves, st.gmres_its_avg);

    if (p->pw && np > 0) {
        p->voc = (d_complex_t *)calloc((size_t)np * nf, sizeof(d_complex_t));
        if (p->dist && p->nseg > 0) p->segipw = (d_complex_t *)calloc((size_t)nf * p->nseg, sizeof(d_complex_t));
        pb_planewave_t w;
        memset(&w, 0, sizeof(w));
        w.theta_deg = p->pwth;
        w.phi_deg = p->pwph;
        w.pol = p->pwpol;
        w.amp = p->pwamp;
        w.phase_deg = p->pwphase;
        r = pb_planewave(c, nf, freq, &o, &w, (double *)p->voc, p->segipw ? (double *)p->segipw : NULL, NULL);
        if (r != PB_OK) {
            fail_msg(fp_log, "plane-wave excitation", r);
            free(freq);
            return 1;
        }
    }

    if (p->nsrc > 0) {
        pb_source_t *src = (pb_source_t *)calloc((size_t)p->nsrc, sizeof(pb_source_t));
        double *vn = (double *)calloc(2 * (size_t)nf * (p->maxid + 1), sizeof(double));
        if (!src || !vn) {
            free(src); free(vn); free(freq);
            printf("%s\n", "*** memory allocation error (sources)");
            return 1;
        }
        for (int i = 0; i < p->nsrc; i++) {
            src[i].n1 = p->src[i].n1;
            src[i].n2 = p->src[i].n2;
            src[i].isvsrc = p->src[i].isvsrc;
            src[i].amp = p->src[i].amp;
            src[i].phase_deg = p->src[i].phase;
        }
        pb_sweep_opts os = o;
        os.compress = 0;
        os.accel = 0;
        r = pb_sources(c, nf, freq, &os, p->nsrc, src, vn, NULL);
        if (r != PB_OK) {
            fail_msg(fp_log, "source excitation", r);
            free(src); free(vn); free(freq);
            return 1;
        }
        /* print_vnode (solve.c:102-112) */
        for (int ifr = 0; ifr < nf; ifr++) {
            fprintf(fp_log, "=== node voltage === (f = %.5e Hz)\n", freq[ifr]);
            fprintf(fp_log, "  %s\n", "node      real[V]      imag[V]       |V|[V]");
            for (int id = 0; id <= p->maxid; id++) {
                if (p->nodemap[id] == -2) continue;
                const double vr = vn[2 * ((size_t)ifr * (p->maxid + 1) + id)];
                const double vi = vn[2 * ((size_t)ifr * (p->maxid + 1) + id) + 1];
                fprintf(fp_log, "%6d %12.4e %12.4e %12.4e\n", id, vr, vi, sqrt(vr * vr + vi * vi));
            }
        }
        free(src);
        free(vn);
    }
    free(freq);
    return 0;
}
