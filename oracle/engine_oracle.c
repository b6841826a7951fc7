/* Oracle restatement of one Smoldyn time step with injected displacements.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Operator order of simulatetimestep (smolsim.cpp:2607-2692):
 *   diffuse       smolmolec.c:3115-3168  pos += displacement (injected here)
 *   checkwalls    smolwall.c:368-427     walls in the order x-low, x-high, y-low, ...
 *   unireact      smolreact.c:2997-3056  first-order reactions (injected choice)
 *   bireact       smolreact.c:3201-3298  pairs within the binding radius; a molecule
 *                                        reacts at most once, first come first served
 *   doreact       smolreact.c:2662-2902  products at x*p1+(1-x)*p2, x=D2/(D1+D2),
 *                                        plus the reaction's product offsets
 *   checkwalls on the new molecules      smolsim.cpp:2656-2664
 * FP64 throughout.  Periodic pair distances use the minimum image, which is
 * what the reference's wrap-coded neighbour boxes give when a box is wider
 * than the binding radius (smolwall.c:100-117, smolreact.c:3141-3153).
 * Product offsets are applied without the random rotation (the deterministic
 * comparison uses offset-free products or compares distances only).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

static int apply_walls(const ora_net *net, double *p) {
  for (int d = 0; d < net->dim; ++d) {
    const double lo = net->lo[d], hi = net->hi[d], L = hi - lo;
    /* low wall */
    switch (net->wall[d][0]) {
      case 'r': if (p[d] < lo) p[d] = 2 * lo - p[d]; break;
      case 'p': if (p[d] < lo) p[d] += L; break;
      case 'a': if (p[d] < lo) return 1; break;
      default: break;
    }
    /* high wall */
    switch (net->wall[d][1]) {
      case 'r': if (p[d] > hi) p[d] = 2 * hi - p[d]; break;
      case 'p': if (p[d] > hi) p[d] -= L; break;
      case 'a': if (p[d] > hi) return 1; break;
      default: break;
    }
  }
  return 0;
}

/* vector from a to b with the minimum image in periodic dimensions */
static double pair_vec(const ora_net *net, const double *a, const double *b, double *v) {
  double d2 = 0;
  for (int d = 0; d < net->dim; ++d) {
    double x = b[d] - a[d];
    if (net->wall[d][0] == 'p') {
      const double L = net->hi[d] - net->lo[d];
      if (x > 0.5 * L) x -= L;
      else if (x < -0.5 * L) x += L;
    }
    v[d] = x;
    d2 += x * x;
  }
  return d2;
}

static int pair_rxn(const ora_net *net, int sa, int sb, double d2) {
  for (int r = 0; r < net->nr2; ++r) {
    const int a = net->r2_rct[r][0], b = net->r2_rct[r][1];
    if (((a == sa && b == sb) || (a == sb && b == sa)) && d2 <= net->r2_bind2[r]) return r;
  }
  return -1;
}

int ora_step(const ora_net *net, int n, const double *pos, const int *sp, const uint64_t *serno,
             const double *disp, const int *force1, int cap, double *opos, int *osp, uint64_t *oserno,
             uint64_t *oparent, int *on, int *fate, uint64_t *partner, int *nambig) {
  const int dim = net->dim;
  double *p = (double *)malloc(sizeof(double) * 3 * (n > 0 ? n : 1));
  int *alive = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  int nout = 0, rc = 0;
  /* product staging: site + offsets, parent serno */
  double *ppos = (double *)malloc(sizeof(double) * 3 * (4 * n + 4));
  int *psp = (int *)malloc(sizeof(int) * (4 * n + 4));
  uint64_t *ppar = (uint64_t *)malloc(sizeof(uint64_t) * (4 * n + 4));
  int np = 0;

  for (int i = 0; i < n; ++i) {
    for (int d = 0; d < 3; ++d) p[3 * i + d] = pos[3 * i + d] + (d < dim ? disp[3 * i + d] : 0);
    fate[i] = 0;
    partner[i] = 0;
    alive[i] = 1;
    if (apply_walls(net, p + 3 * i)) { alive[i] = 0; fate[i] = 1; }
  }
  /* first order */
  for (int i = 0; i < n; ++i) {
    if (!alive[i] || force1[i] < 0) continue;
    const int r = force1[i];
    alive[i] = 0;
    fate[i] = 2;
    for (int q = 0; q < net->r1_nprod[r]; ++q) {
      for (int d = 0; d < 3; ++d) ppos[3 * np + d] = p[3 * i + d] + (d < dim ? net->r1_prdpos[r][q][d] : 0);
      psp[np] = net->r1_prd[r][q];
      ppar[np] = serno[i];
      np++;
    }
  }
  /* ambiguity count: molecules with more than one in-radius partner */
  *nambig = 0;
  for (int i = 0; i < n; ++i) {
    if (!alive[i]) continue;
    int c = 0;
    for (int j = 0; j < n && c < 2; ++j) {
      if (j == i || !alive[j]) continue;
      double v[3];
      const double d2 = pair_vec(net, p + 3 * i, p + 3 * j, v);
      if (pair_rxn(net, sp[i], sp[j], d2) >= 0) c++;
    }
    if (c > 1) (*nambig)++;
  }
  /* second order, first come first served in input order */
  for (int i = 0; i < n; ++i) {
    if (!alive[i]) continue;
    for (int j = 0; j < n; ++j) {
      if (j == i || !alive[j]) continue;
      double v[3];
      const double d2 = pair_vec(net, p + 3 * i, p + 3 * j, v);
      const int r = pair_rxn(net, sp[i], sp[j], d2);
      if (r < 0) continue;
      /* reactant 1 is the molecule of the reaction's first species */
      const int a = (sp[i] == net->r2_rct[r][0]) ? i : j, b = (a == i) ? j : i;
      double vab[3];
      pair_vec(net, p + 3 * a, p + 3 * b, vab);
      const double D1 = net->difc[sp[a]], D2 = net->difc[sp[b]];
      const double x = (D1 == 0 && D2 == 0) ? 0.5 : D2 / (D1 + D2);
      double site[3] = {0, 0, 0};
      for (int d = 0; d < dim; ++d) {
        site[d] = p[3 * a + d] + (1.0 - x) * vab[d];
        if (net->wall[d][0] == 'p') {
          const double L = net->hi[d] - net->lo[d];
          if (site[d] < net->lo[d]) site[d] += L;
          else if (site[d] > net->hi[d]) site[d] -= L;
        }
      }
      for (int q = 0; q < net->r2_nprod[r]; ++q) {
        for (int d = 0; d < 3; ++d) ppos[3 * np + d] = site[d] + (d < dim ? net->r2_prdpos[r][q][d] : 0);
        psp[np] = net->r2_prd[r][q];
        ppar[np] = serno[a];
        np++;
      }
      alive[i] = alive[j] = 0;
      fate[i] = fate[j] = 3;
      partner[i] = serno[j];
      partner[j] = serno[i];
      break;
    }
  }
  for (int i = 0; i < n; ++i) {
    if (!alive[i]) continue;
    if (nout >= cap) { rc = -1; break; }
    memcpy(opos + 3 * nout, p + 3 * i, 3 * sizeof(double));
    osp[nout] = sp[i];
    oserno[nout] = serno[i];
    oparent[nout] = 0;
    nout++;
  }
  for (int k = 0; k < np && rc == 0; ++k) {
    if (apply_walls(net, ppos + 3 * k)) continue;
    if (nout >= cap) { rc = -1; break; }
    memcpy(opos + 3 * nout, ppos + 3 * k, 3 * sizeof(double));
    osp[nout] = psp[k];
    oserno[nout] = 0;
    oparent[nout] = ppar[k];
    nout++;
  }
  *on = nout;
  free(p);
  free(alive);
  free(ppos);
  free(psp);
  free(ppar);
  return rc;
}
