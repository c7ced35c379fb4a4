/*
 * peec_oracle.h — CPU restatement of the reference's frequency-sweep hot path.
 *
 * TEST INFRASTRUCTURE ONLY. The product (libpeec_b200.so) never links, loads or calls
 * this code; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
 * it, as the checker. It restates, in plain FP64 C, the algorithms of the reference's
 * src/partial.c, surface.c, volume.c, polygon.c, potential.c, skin.c, mna.c, lu.c and
 * the dense path of solve.c, on the pb_cell_t input of include/peec_b200.h.
 * It is pinned against the reference itself by tests/test_oracle_pin.py (golden
 * vectors written by tests/golden/make_golden.py from the reference's own code).
 */
#ifndef PEEC_ORACLE_H
#define PEEC_ORACLE_H
#include "../include/peec_b200.h"

typedef struct or_prob or_prob;

or_prob *or_create(const pb_problem_t *pb);
void     or_destroy(or_prob *o);
/* out: nseg, nchg, ncell, nnode, nunknown, offS, refnode, offL, offV */
void     or_sizes(const or_prob *o, int *out);
void     or_cellmap(const or_prob *o, int *cellid, int *cellof, double *carea);

void or_lp_entry(const or_prob *o, int i, int j, double kw, double *out);
void or_pot_entry(const or_prob *o, int i, int j, double kw, double *out);
/* Dense fills, both triangles, row-major complex: Lp [nseg^2], P [ncell^2]. */
void or_lp_fill(const or_prob *o, double kw, double *lp);
void or_pot_fill(const or_prob *o, double kw, double *pm);
/* Dense MNA of the reference (mna.c:300) from given Lp and C = P^-1 matrices. */
void or_mna_assemble(const or_prob *o, double f, const double *lp, const double *cmat,
                     double *a);
/* Reference lu_decomp / lu_solve (lu.c:16-96). */
int  or_lu_decomp(int n, double *a, int *piv);
void or_lu_solve(int n, const double *a, const int *piv, double *b);
/* Dense sweep of the reference solve() (solve.c:239-370); zmat [nfreq*nport*nport]. */
int  or_sweep(const or_prob *o, int nfreq, const double *freq, double *zmat, int nthreads);
/* plane-wave sweep: pwp = {theta_deg, phi_deg, pol, amp, phase_deg}; voc[i*nfreq+f] */
int  or_planewave(const or_prob *o, int nfreq, const double *freq, const double *pwp,
                  double *voc, double *segipw);
/* Internal impedance of current cell k at f (skin.c:112-133 / mna.c:128-138). */
void or_zint(const or_prob *o, int k, double f, double *out);
/* Single-pair geometric integral (partial.c:256-317) between current cells. */
void or_pair_k(const or_prob *o, int i, int j, int mirror_j, double kw, double *out);



/* CPU-baseline timing helpers (bounded samples, all OpenMP threads). */
double or_time_entries(const or_prob *o, int which, int n, const int *ij, double kw);
double or_time_lu(int n, unsigned seed);
double or_time_solves(int n, int ncol);
int    or_set_threads(int n);
#endif
