/*
 * ref_harness.c — test-only bridge to the reference implementation.
 *
 * This file is part of the checker, not of the product. It is compiled together with
 * the reference's unmodified sources (the Makefile in this directory reads them from
 * the reference checkout) into oracle/_ref/libpeecref.so, and gives ctypes access to:
 *   - the reference's own parser and geometry builder (input_data, wire_build), so the
 *     discretised cells can be exported in the pb_cell_t layout of include/peec_b200.h;
 *   - the reference's entry-level kernels (lp_entry, pot_entry) and fills (lp_fill,
 *     pot_fill), MNA assembly, dense LU and the full sweep (solve),
 * so that tests/golden/make_golden.py can write golden vectors and the oracle
 * restatement (oracle/peec_oracle.c) can be pinned against the reference.
 *
 * Call order mirrors the reference's main (src/main.c:62-103).
 */
#include "peec.h"
#include "../include/peec_b200.h"

typedef struct {
    peec_t p;
    FILE  *log;
} rh_t;

static FILE *open_log(void)
{
    FILE *f = fopen("/dev/null", "w");
    return f ? f : stderr;
}

void *rh_load(const char *path)
{
    FILE *fp = fopen(path, "r");
    if (fp == NULL) return NULL;
    rh_t *h = (rh_t *)calloc(1, sizeof(rh_t));
    h->log = open_log();
    if (input_data(fp, &h->p)) {
        fclose(fp);
        free(h);
        return NULL;
    }
    fclose(fp);
    if (wire_build(&h->p, h->log)) return NULL;
    /* main.c:86-98 : static fill (needed for the cell count), then MNA numbering */
    if (!h->p.compress) lp_fill(&h->p, 0, h->log);
    if (pot_fill(&h->p, 0, h->log)) return NULL;
    if (mna_numbering(&h->p, h->log)) return NULL;
    return h;
}

/* Same as rh_load without the static setup fill (for timing samples): geometry,
 * charge-cell grouping and MNA numbering only. */
void *rh_load_light(const char *path)
{
    FILE *fp = fopen(path, "r");
    if (fp == NULL) return NULL;
    rh_t *h = (rh_t *)calloc(1, sizeof(rh_t));
    h->log = open_log();
    if (input_data(fp, &h->p)) {
        fclose(fp);
        free(h);
        return NULL;
    }
    fclose(fp);
    if (wire_build(&h->p, h->log)) return NULL;
    if (h->p.capacitance && h->p.nchg > 0 && pot_cells(&h->p)) return NULL;
    if (mna_numbering(&h->p, h->log)) return NULL;
    return h;
}

void rh_free(void *hv)
{
    rh_t *h = (rh_t *)hv;
    if (h == NULL) return;
    peec_free(&h->p);
    if (h->log && h->log != stderr) fclose(h->log);
    free(h);
}

/* out[0..19] : integer facts about the loaded problem */
void rh_info(void *hv, int *out)
{
    const peec_t *p = &((rh_t *)hv)->p;
    int nl = 0;
    for (int i = 0; i < p->nsrc; i++) nl += p->src[i].isvsrc;
    out[0] = p->nseg;   out[1] = p->nchg;  out[2] = p->ncell;  out[3] = p->nnode;
    out[4] = p->nunknown; out[5] = p->offS; out[6] = p->refnode; out[7] = p->maxid;
    out[8] = p->nport;  out[9] = p->nfreq; out[10] = p->capacitance;
    out[11] = p->retardation; out[12] = p->skin; out[13] = p->gp; out[14] = p->compress;
    out[15] = p->flog; out[16] = p->nres + p->ncap + p->nind + nl; out[17] = p->nmut;
    out[18] = p->offL; out[19] = p->offV;
}

/* out[0..3] : gpz, f0, f1, gmin */
void rh_infod(void *hv, double *out)
{
    const peec_t *p = &((rh_t *)hv)->p;
    out[0] = p->gpz; out[1] = p->f0; out[2] = p->f1; out[3] = p->gmin;
}

double rh_freq(void *hv, int ifreq)
{
    return freq_at(&((rh_t *)hv)->p, ifreq);
}

static void to_cell(const seg_t *s, pb_cell_t *c, int pvoff)
{
    memset(c, 0, sizeof(*c));
    for (int k = 0; k < 3; k++) {
        c->x1[k] = s->x1[k]; c->x2[k] = s->x2[k];
        c->wv[k] = s->wv[k]; c->papex[k] = s->papex[k];
    }
    c->len = s->len; c->wid = s->wid; c->thick = s->thick;
    c->aL = s->aL; c->aP = s->aP; c->radius = s->radius;
    c->area = s->area; c->perim = s->perim; c->sigma = s->sigma; c->res = s->res;
    c->cexc = s->cexc; c->gexc = s->gexc; c->gfac = s->gfac;
    c->epss = s->epss; c->epsinf = s->epsinf; c->frelax = s->frelax;
    c->n1 = s->n1; c->n2 = s->n2; c->shape = s->shape; c->vol = s->vol;
    c->diel = s->diel; c->npv = s->npv; c->pvoff = s->npv > 0 ? pvoff : 0;
}

/* Number of polygon vertices over current cells (which=0) or charge cells (which=1). */
int rh_npv(void *hv, int which)
{
    const peec_t *p = &((rh_t *)hv)->p;
    const int n = which ? p->nchg : p->nseg;
    const seg_t *s = which ? p->chg : p->seg;
    int t = 0;
    for (int i = 0; i < n; i++) t += s[i].npv;
    return t;
}

/* Export cells; pv receives the vertex pool (offsets start at pvbase). */
int rh_cells(void *hv, int which, pb_cell_t *out, double *pv, int pvbase, int *chgnode)
{
    const peec_t *p = &((rh_t *)hv)->p;
    const int n = which ? p->nchg : p->nseg;
    const seg_t *s = which ? p->chg : p->seg;
    int off = 0;
    for (int i = 0; i < n; i++) {
        to_cell(&s[i], &out[i], pvbase + off);
        if (pv != NULL) {
            for (int k = 0; k < 3 * s[i].npv; k++) pv[3 * off + k] = s[i].pv[k];
        }
        off += s[i].npv;
        if (which && chgnode != NULL) chgnode[i] = p->chgnode[i];
    }
    return n;
}

int rh_ports(void *hv, pb_port_t *out)
{
    const peec_t *p = &((rh_t *)hv)->p;
    for (int i = 0; i < p->nport; i++) {
        out[i].n1 = p->port[i].n1; out[i].n2 = p->port[i].n2; out[i].z0 = p->port[i].z0;
    }
    return p->nport;
}

/* Lumped elements in the reference's stamping order: R, C, L, V (mna.c:188-241). */
int rh_lumps(void *hv, pb_lump_t *out, pb_mutual_t *mut)
{
    const peec_t *p = &((rh_t *)hv)->p;
    int n = 0;
    for (int i = 0; i < p->nres; i++, n++) {
        out[n].kind = PB_LUMP_R; out[n].n1 = p->res[i].n1; out[n].n2 = p->res[i].n2;
        out[n].val = p->res[i].val;
    }
    for (int i = 0; i < p->ncap; i++, n++) {
        out[n].kind = PB_LUMP_C; out[n].n1 = p->cap[i].n1; out[n].n2 = p->cap[i].n2;
        out[n].val = p->cap[i].val;
    }
    for (int i = 0; i < p->nind; i++, n++) {
        out[n].kind = PB_LUMP_L; out[n].n1 = p->ind[i].n1; out[n].n2 = p->ind[i].n2;
        out[n].val = p->ind[i].val;
    }
    for (int i = 0; i < p->nsrc; i++) {
        if (!p->src[i].isvsrc) continue;
        out[n].kind = PB_LUMP_V; out[n].n1 = p->src[i].n1; out[n].n2 = p->src[i].n2;
        out[n].val = p->src[i].amp;
        n++;
    }
    for (int i = 0; i < p->nmut && mut != NULL; i++) {
        mut[i].l1 = p->mut[i].l1; mut[i].l2 = p->mut[i].l2; mut[i].k = p->mut[i].k;
    }
    return n;
}

void rh_lp_entry(void *hv, int i, int j, double kw, double *out)
{
    const d_complex_t v = lp_entry(&((rh_t *)hv)->p, i, j, kw);
    out[0] = v.r; out[1] = v.i;
}

void rh_pot_entry(void *hv, int i, int j, double kw, double *out)
{
    const d_complex_t v = pot_entry(&((rh_t *)hv)->p, i, j, kw);
    out[0] = v.r; out[1] = v.i;
}

/* Full Lp through the reference's lp_fill at frequency f; out [2*nseg*nseg]. */
void rh_lp_fill(void *hv, double f, double *out)
{
    rh_t *h = (rh_t *)hv;
    lp_fill(&h->p, f, h->log);
    memcpy(out, h->p.lp, (size_t)h->p.nseg * h->p.nseg * sizeof(d_complex_t));
}

/* C = P^-1 through the reference's pot_fill at frequency f; out [2*ncell*ncell]. */
int rh_pot_fill(void *hv, double f, double *out)
{
    rh_t *h = (rh_t *)hv;
    if (pot_fill(&h->p, f, h->log)) return 1;
    if (h->p.cmat != NULL && out != NULL)
        memcpy(out, h->p.cmat, (size_t)h->p.ncell * h->p.ncell * sizeof(d_complex_t));
    return 0;
}

/* Cell-level grouping built by pot_cells: cellid[ncell], cellof[nchg], carea[ncell]. */
void rh_cellmap(void *hv, int *cellid, int *cellof, double *carea)
{
    const peec_t *p = &((rh_t *)hv)->p;
    for (int i = 0; i < p->ncell; i++) { cellid[i] = p->cellid[i]; carea[i] = p->carea[i]; }
    for (int h = 0; h < p->nchg; h++) cellof[h] = p->cellof[h];
}

void rh_nodemap(void *hv, int *nodemap)
{
    const peec_t *p = &((rh_t *)hv)->p;
    for (int i = 0; i <= p->maxid; i++) nodemap[i] = p->nodemap[i];
}

/* Dense MNA at f after lp_fill/pot_fill at the same f (mna.c:300-308). */
void rh_mna_assemble(void *hv, double f, double *out)
{
    const peec_t *p = &((rh_t *)hv)->p;
    mna_assemble(p, f, (d_complex_t *)out);
}

/* Whole reference sweep; zmat [2*nfreq*nport*nport]. Returns solve()'s status. */
int rh_solve(void *hv, double *zmat)
{
    rh_t *h = (rh_t *)hv;
    const int r = solve(&h->p, h->log);
    if (r == 0 && zmat != NULL)
        memcpy(zmat, h->p.zmat,
               (size_t)h->p.nfreq * h->p.nport * h->p.nport * sizeof(d_complex_t));
    return r;
}

/* Plane-wave results of the last rh_solve: voc [2*nport*nfreq] (voc[i*nfreq+f]), segipw
 * [2*nfreq*nseg] (when distribution = 1), and the wave's parameters pwp[5]. Returns 0 when
 * the input has no plane wave. */
int rh_voc(void *hv, double *voc, double *segipw, double *pwp)
{
    const peec_t *p = &((rh_t *)hv)->p;
    if (!p->pw || p->voc == NULL) return 0;
    if (voc) memcpy(voc, p->voc, (size_t)p->nport * p->nfreq * sizeof(d_complex_t));
    if (segipw && p->segipw) memcpy(segipw, p->segipw, (size_t)p->nfreq * p->nseg * sizeof(d_complex_t));
    if (pwp) {
        pwp[0] = p->pwth; pwp[1] = p->pwph; pwp[2] = p->pwpol; pwp[3] = p->pwamp; pwp[4] = p->pwphase;
    }
    return 1 + (p->segipw != NULL);
}

/* Node voltages of the independent-source excitation at f, computed the way the dense
 * path of solve() does it (solve.c:243-248, 296-299, 392-396): lp_fill / pot_fill at f,
 * mna_assemble, mna_rhs_sources, lu_decomp / lu_solve. out [2*(maxid+1)] = x[nodemap[id]],
 * 0 where nodemap < 0, as print_vnode (solve.c:102-112) reports them. Returns -2 without
 * sources, -3 on allocation failure, else lu_decomp's status (-1 = regular). */
int rh_vnode(void *hv, double f, double *out)
{
    rh_t *h = (rh_t *)hv;
    peec_t *p = &h->p;
    if (p->nsrc <= 0) return -2;
    lp_fill(p, f, h->log);
    if (pot_fill(p, f, h->log)) return -3;
    const int n = p->nunknown;
    d_complex_t *a = (d_complex_t *)malloc((size_t)n * n * sizeof(d_complex_t));
    d_complex_t *b = (d_complex_t *)malloc((size_t)n * sizeof(d_complex_t));
    int *piv = (int *)malloc((size_t)n * sizeof(int));
    if (!a || !b || !piv) { free(a); free(b); free(piv); return -3; }
    mna_assemble(p, f, a);
    mna_rhs_sources(p, b);
    const int r = lu_decomp(n, a, piv);
    if (r < 0) {
        lu_solve(n, a, piv, b);
        for (int id = 0; id <= p->maxid; id++) {
            const int m = p->nodemap[id];
            out[2 * id] = m >= 0 ? b[m].r : 0;
            out[2 * id + 1] = m >= 0 ? b[m].i : 0;
        }
    }
    free(a); free(b); free(piv);
    return r;
}

/* Results of the last rh_solve that the post-processing reads: zin [2*nport*nfreq]
 * (zin[j*nfreq+f]), segi [2*nfreq*nport*nseg] (DIDX order; when distribution or farfield
 * is set), smat [2*nfreq*nport*nport] (ZIDX order). Returns 1 + (segi present). */
int rh_results(void *hv, double *zin, double *segi, double *smat)
{
    const peec_t *p = &((rh_t *)hv)->p;
    if (p->zin == NULL) return 0;
    if (zin) memcpy(zin, p->zin, (size_t)p->nport * p->nfreq * sizeof(d_complex_t));
    if (smat && p->smat) memcpy(smat, p->smat, (size_t)p->nfreq * p->nport * p->nport * sizeof(d_complex_t));
    if (segi && p->segi) memcpy(segi, p->segi, (size_t)p->nfreq * p->nport * p->nseg * sizeof(d_complex_t));
    return 1 + (p->segi != NULL);
}

/* The reference's own post-processing writers on the last rh_solve's results:
 * output_far (farfield.c:42) and output_tran (transient.c:97) into the CSV file fn. */
int rh_output_far(void *hv, const char *fn)
{
    rh_t *h = (rh_t *)hv;
    return output_far(&h->p, fn, h->log);
}

int rh_output_tran(void *hv, const char *fn)
{
    rh_t *h = (rh_t *)hv;
    return output_tran(&h->p, fn, h->log);
}

/* Restrict the sweep to [ifreq0, ifreq0+count) of the parsed list (for timing samples). */
void rh_set_freqs(void *hv, double f0, double f1, int nfreq, int flog)
{
    peec_t *p = &((rh_t *)hv)->p;
    p->f0 = f0; p->f1 = f1; p->nfreq = nfreq; p->flog = flog;
    free(p->zin); free(p->zmat); free(p->smat); free(p->segi); free(p->cellq);
    free(p->voc); free(p->segipw);
    p->zin = p->zmat = p->smat = p->segi = p->cellq = p->voc = p->segipw = NULL;
}

int rh_lu_decomp(int n, double *a, int *piv)
{
    return lu_decomp(n, (d_complex_t *)a, piv);
}

void rh_lu_solve(int n, const double *a, const int *piv, double *b)
{
    lu_solve(n, (const d_complex_t *)a, piv, (d_complex_t *)b);
}

int rh_set_threads(int n)
{
#ifdef _OPENMP
    extern void omp_set_num_threads(int);
    extern int omp_get_max_threads(void);
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* ------------------------------------------------------------------ CPU timing
 * Bounded samples of the reference's per-frequency work, timed with all OpenMP
 * threads: seconds to evaluate the listed Lp (which=0) or P (which=1) entries. */
#include <time.h>
static double rh_now(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + 1e-9 * t.tv_nsec;
}

double rh_time_entries(void *hv, int which, int n, const int *ij, double kw)
{
    const peec_t *p = &((rh_t *)hv)->p;
    double sink = 0;
    const double t0 = rh_now();
    int e;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : sink)
    for (e = 0; e < n; e++) {
        const d_complex_t v = which ? pot_entry(p, ij[2 * e], ij[2 * e + 1], kw)
                                    : lp_entry(p, ij[2 * e], ij[2 * e + 1], kw);
        sink += v.r;
    }
    const double t1 = rh_now();
    return (t1 - t0) + 0 * sink;
}

/* Seconds of the reference's lu_decomp on a random diagonally weighted complex matrix. */
double rh_time_lu(int n, unsigned seed)
{
    d_complex_t *a = (d_complex_t *)malloc((size_t)n * n * sizeof(d_complex_t));
    int *piv = (int *)malloc((size_t)n * sizeof(int));
    unsigned s = seed;
    for (size_t i = 0; i < (size_t)n * n; i++) {
        s = s * 1103515245u + 12345u;
        a[i].r = ((s >> 8) & 0xffff) / 65536.0 - 0.5;
        s = s * 1103515245u + 12345u;
        a[i].i = ((s >> 8) & 0xffff) / 65536.0 - 0.5;
    }
    const double t0 = rh_now();
    lu_decomp(n, a, piv);
    const double t1 = rh_now();
    free(a);
    free(piv);
    return t1 - t0;
}

/* Seconds of `ncol` of the reference's column solves of C = P^-1 (potential.c:274-281),
 * on the already factorised order-n random matrix of rh_time_lu's kind. */
double rh_time_solves(int n, int ncol)
{
    d_complex_t *a = (d_complex_t *)malloc((size_t)n * n * sizeof(d_complex_t));
    d_complex_t *b = (d_complex_t *)malloc((size_t)n * sizeof(d_complex_t));
    int *piv = (int *)malloc((size_t)n * sizeof(int));
    for (size_t i = 0; i < (size_t)n * n; i++) { a[i].r = (i % (n + 1)) == 0 ? n : 0.5 / (1 + i % 7); a[i].i = 0; }
    for (int i = 0; i < n; i++) piv[i] = i;
    const double t0 = rh_now();
    for (int j = 0; j < ncol; j++) {
        memset(b, 0, (size_t)n * sizeof(d_complex_t));
        b[j % n] = d_complex(1, 0);
        lu_solve(n, a, piv, b);
    }
    const double t1 = rh_now();
    free(a); free(b); free(piv);
    return t1 - t0;
}
