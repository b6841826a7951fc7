/* CPU oracle for the smoldyn_b200 parity tests.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline use it, as the checker.
 *
 * The oracle restates, in plain FP64 C, the reference algorithms that the
 * GPU engine replaces.  Parity is pinned two ways:
 *   - the reference itself, compiled from its own sources by oracle/Makefile
 *     (oracle/_ref/smoldyn, libsmoldyn_ref.a, librxnparam_ref.so), reproduces
 *     the reference's golden regression outputs byte for byte
 *     (examples/S95_regression/output_275, tests/test_oracle_pin.py);
 *   - this restatement is checked against that compiled reference
 *     (tests/test_oracle_rxnparam.py) and against fixtures recorded from it
 *     (tests/golden/, made by oracle/make_golden.py).
 */
#ifndef SMOLDYN_ORACLE_H
#define SMOLDYN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* rxnparam.c:57-158, 161-518, 558-584, 587-681, 690-716 */
double ora_numrxnrate(double step, double a, double b);
double ora_numrxnrateprob(double step, double a, double b, double prob);
double ora_bindingradius(double rate, double dt, double difc, double b, int rel);
double ora_bindingradiusprob(double rate, double dt, double difc, double b, int rel, double chi,
                             double *probptr);
double ora_unbindingradius(double pgem, double dt, double difc, double a);

/* rxnparam.c:719-1114: the radial-distribution-function solver that produced
 * the tables above; see rdf_oracle.c. */
double ora_erfc_nr(double x);
double ora_rdf_absorb(const double *r, double *rdf, int n, double bindrad, double prob);
void ora_rdf_diffuse(const double *r, const double *rdfa, double *rdfd, int n, double step);
void ora_rdf_reverse(const double *r, double *rdf, int n, double step, double b, double flux);
double ora_rdf_steady(const double *r, double *rdfa, double *rdfd, int n, double step, double a, double b,
                      double eps, double prob, int *iters);
int ora_rdf_grid(int mode, int n, double b, double *r);
int ora_rdf_rows(int mode, double *bvals);
int ora_rdf_steps(int dir, double *svals);
int ora_rdf_table(int mode, int n, double eps, int dir, int nprob, const double *probs, double *flux,
                  int *iters, double *rbuf, double *rdfa, double *rdfd);

/* One deterministic time step in the reference's operator order
 * (smolsim.cpp:2607-2692) with injected displacements; see engine_oracle.c. */
#define ORA_MAXSP 32
#define ORA_MAXRXN 16
#define ORA_MAXPRD 4
typedef struct {
  int dim;
  double lo[3], hi[3];
  char wall[3][2]; /* 'r' 'p' 'a' 't' */
  int nsp;
  double difc[ORA_MAXSP];
  int nr1;
  int r1_rct[ORA_MAXRXN];
  int r1_nprod[ORA_MAXRXN];
  int r1_prd[ORA_MAXRXN][ORA_MAXPRD];
  double r1_prdpos[ORA_MAXRXN][ORA_MAXPRD][3];
  int nr2;
  int r2_rct[ORA_MAXRXN][2];
  double r2_bind2[ORA_MAXRXN];
  int r2_nprod[ORA_MAXRXN];
  int r2_prd[ORA_MAXRXN][ORA_MAXPRD];
  double r2_prdpos[ORA_MAXRXN][ORA_MAXPRD][3];
} ora_net;

/* Inputs: n molecules (pos[3n], sp[n], serno[n]); disp[3n] displacement of
 * this step; force1[n] = index of the first-order reaction the molecule
 * undergoes this step or -1.
 * Outputs: survivors then products in (opos, osp, oserno, oparent), *on
 * total; product serno = 0 and oparent = serno of the first reactant.
 * fate[n]: 0 survived, 1 wall, 2 first-order, 3 second-order; partner[n] =
 * serno of the second-order partner.  *nambig counts molecules that had more
 * than one in-radius partner (the reference's first-come order decides those).
 * Returns 0, or -1 when an output capacity is exceeded. */
int ora_step(const ora_net *net, int n, const double *pos, const int *sp, const uint64_t *serno,
             const double *disp, const int *force1, int cap, double *opos, int *osp, uint64_t *oserno,
             uint64_t *oparent, int *on, int *fate, uint64_t *partner, int *nambig);

#ifdef __cplusplus
}
#endif
#endif
