/* Oracle restatement of the reference's radial-distribution-function solver,
 * the numerical method behind the rxnparam lookup tables.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Follows source/libSteve/rxnparam.c:784-1114 function by function (line
 * numbers cited per function): spherical trapezoid integration of the
 * absorbed flux, the radial diffusion Green's function convolution with a
 * 1+a2/r tail, the analytic reverse-reaction source, the alternating
 * steady-state iteration and the table sweeps over step length, unbinding
 * radius and reaction probability.  Plain C, FP64, sequential sums in the
 * reference's order.
 */
#include <math.h>
#include <stddef.h>

#include "oracle.h"

#define R_PI 3.14159265358979323846
#define R_SQRT2PI 2.50662827462 /* the reference's literal (math2.h:14) */

/* Complementary error function by the Chebyshev fit of Numerical Recipes in C
 * (2nd ed., section 6.2, "erfcc"; fractional error below 1.2e-7), the form the
 * reference uses (rxnparam.c:719-724). */
double ora_erfc_nr(double x) {
  double z = fabs(x), t = 1.0 / (1.0 + 0.5 * z);
  static const double c[10] = {-1.26551223, 1.00002368, 0.37409196, 0.09678418, -0.18628806,
                               0.27886807, -1.13520398, 1.48851587, -0.82215223, 0.17087277};
  double poly = c[9];
  for (int k = 8; k >= 1; --k) poly = c[k] + t * poly;
  double v = t * exp(-z * z + c[0] + t * poly);
  return x >= 0.0 ? v : 2.0 - v;
}

/* 4 pi r^2 integral of the linear interpolant between (r0,f0) and (r1,f1)
 * (rxnparam.c:771-776) */
static double shell(double r0, double r1, double f0, double f1) {
  return R_PI * (f1 - f0) * (r1 + r0) * (r1 * r1 + r0 * r0) +
         4.0 * R_PI / 3.0 * (r1 * f0 - r0 * f1) * (r1 * r1 + r1 * r0 + r0 * r0);
}

/* rxnparam.c:784-802: integrate rdf over r < bindrad (the last shell ends at
 * the first grid point past bindrad, minus its upper-left triangle), scale
 * the absorbed points by 1-prob, return prob times the integral. */
double ora_rdf_absorb(const double *r, double *rdf, int n, double bindrad, double prob) {
  double r0 = 0, r1 = 0, f0, f1 = rdf[0], sum = 0;
  int j = r[0] == 0 ? 1 : 0;
  while (r1 < bindrad && j < n) {
    r0 = r1;
    f0 = f1;
    r1 = r[j];
    f1 = rdf[j];
    sum += shell(r0, r1, f0, f1);
    ++j;
  }
  sum -= shell(r0, r1, 0.0, f1);
  sum *= prob;
  for (int k = j - 2; k >= 0; --k) rdf[k] *= 1.0 - prob;
  return sum;
}

/* rxnparam.c:819-857: one diffusion step of rms length `step` applied to a
 * radially symmetric rdf with unit density at infinity.  The top 10% of the
 * points fix the 1 + a2/r tail used beyond the grid. */
void ora_rdf_diffuse(const double *r, const double *rdfa, double *rdfd, int n, double step) {
  double alpha = 0, beta = 0;
  for (int i = (int)(0.9 * n); i < n; ++i) {
    alpha += 1.0 / r[i] / r[i];
    beta += (rdfa[i] - 1.0) / r[i];
  }
  const double a2 = beta / alpha / step;
  const double g0 = 2.0 * R_PI * R_SQRT2PI, g1 = 4.0 * R_PI * R_SQRT2PI;
  int i = 0;
  if (r[0] == 0) {
    double r0, r1 = 0, f0, f1 = 0, grn = 0, sum = 0;
    for (int j = 1; j < n; ++j) {
      r0 = r1;
      f0 = f1;
      r1 = r[j] / step;
      grn = exp(-r1 * r1 / 2.0) / g0;
      f1 = (rdfa[j] - rdfa[0]) * grn;
      sum += shell(r0, r1, f0, f1);
    }
    sum += (1.0 - rdfa[0]) * (4.0 * R_PI * r1 * grn + ora_erfc_nr(r1 / sqrt(2.0)));
    rdfd[0] = sum + rdfa[0];
    i = 1;
  }
  for (; i < n; ++i) {
    const double rr = r[i] / step;
    double r0, r1 = 0, f0, grn = exp(-rr * rr / 2.0) / g0, f1 = (rdfa[0] - rdfa[i]) * grn, sum = 0;
    for (int j = r[0] == 0 ? 1 : 0; j < n; ++j) {
      r0 = r1;
      f0 = f1;
      r1 = r[j] / step;
      grn = 1.0 / rr / r1 * (exp(-(rr - r1) * (rr - r1) / 2.0) - exp(-(rr + r1) * (rr + r1) / 2.0)) / g1;
      f1 = (rdfa[j] - rdfa[i]) * grn;
      sum += shell(r0, r1, f0, f1);
    }
    const double ed = ora_erfc_nr((r1 - rr) / sqrt(2.0)), es = ora_erfc_nr((r1 + rr) / sqrt(2.0));
    sum += (1.0 - rdfa[i]) * (4.0 * R_PI * r1 * grn + 1.0 / 2.0 * (ed + es)) + a2 / 2.0 / rr * (ed - es);
    rdfd[i] = sum + rdfa[i];
  }
}

/* rxnparam.c:869-882: add the diffused image of a delta source of area flux
 * placed at radius b (b = 0: at the origin). */
void ora_rdf_reverse(const double *r, double *rdf, int n, double step, double b, double flux) {
  const double k = 1.0 / (4.0 * R_PI * R_SQRT2PI * step * step * step);
  if (b == 0) {
    for (int i = 0; i < n; ++i) {
      double rr = r[i] / step;
      rdf[i] += flux * k * 2.0 * exp(-rr * rr / 2.0);
    }
    return;
  }
  b /= step;
  int i = 0;
  if (r[0] == 0) rdf[i++] += flux * k * 2.0 * exp(-b * b / 2.0);
  for (; i < n; ++i) {
    double rr = r[i] / step;
    rdf[i] += flux * k / rr / b * (exp(-(rr - b) * (rr - b) / 2.0) - exp(-(rr + b) * (rr + b) / 2.0));
  }
}

/* rxnparam.c:898-912: alternate diffusion (plus the reverse-reaction source
 * when b >= 0) and absorption until the flux changes by less than eps
 * (relative), at least 30 and at most 100000 times; -1 when it does not
 * converge or the flux exceeds 1e7. */
double ora_rdf_steady(const double *r, double *rdfa, double *rdfd, int n, double step, double a, double b,
                      double eps, double prob, int *iters) {
  const int maxit = 100000;
  const double maxflux = 1e7;
  ora_rdf_diffuse(r, rdfa, rdfd, n, step);
  double flux = ora_rdf_absorb(r, rdfd, n, a, prob), fluxold = flux;
  int it = 0;
  while (it < 30 || (it < maxit && flux < maxflux && fabs((flux - fluxold) / (fluxold + 1e-20)) > eps)) {
    fluxold = flux;
    ora_rdf_diffuse(r, rdfa, rdfd, n, step);
    if (b >= 0) ora_rdf_reverse(r, rdfd, n, step, b, flux);
    for (int i = 0; i < n; ++i) rdfa[i] = rdfd[i];
    flux = ora_rdf_absorb(r, rdfa, n, a, prob);
    ++it;
  }
  if (iters) *iters = it;
  if (it >= maxit || flux >= maxflux) flux = -1;
  return flux;
}

/* rxnparam.c:965-971: radial grid from 0 in steps of dr with the point at 1
 * replaced by the pair 0.9999, 1.0001.  rmax is 10 (mode 'i'), b+3 ('r') or
 * 5 ('b').  Returns -1 when n is too small to reach r = 1. */
int ora_rdf_grid(int mode, int n, double b, double *r) {
  double dr = mode == 'i' ? 10.0 / n : mode == 'r' ? (b + 3.0) / n : 5.0 / n;
  int i = 1;
  r[0] = 0;
  while (r[i - 1] < 1 && i < n) {
    r[i] = r[i - 1] + dr;
    ++i;
  }
  if (r[i - 1] < 1 || i >= n) return -1;
  r[i - 1] = 0.9999;
  r[i++] = 1.0001;
  for (; i < n; ++i) r[i] = r[i - 1] + dr;
  return 0;
}

/* Row values of the sweeps (rxnparam.c:921-923, 954-961, 1000-1006):
 * mode 'i' one row (b = -1); 'r' b = 1, e^0.2, ... up to e^3 (16 rows);
 * 'b' b = 0, 0.1, ... 1 (11 rows).  Returns the row count. */
int ora_rdf_rows(int mode, double *bvals) {
  int nb = 0;
  if (mode == 'i') {
    bvals[nb++] = -1;
  } else if (mode == 'r') {
    const double bincr = exp(0.2), bhi = exp(3.0);
    for (double b = exp(0.0); !(b > bhi * sqrt(bincr)); b *= bincr) bvals[nb++] = b;
  } else {
    for (double b = 0; !(b > 1.0 + 0.1 / 2.0); b += 0.1) bvals[nb++] = b;
  }
  return nb;
}

/* Step lengths of a sweep in order (rxnparam.c:921, 948-951, 987):
 * e^-3 .. e^3 by e^0.2 upward (dir 'u') or downward ('d').  Returns 31. */
int ora_rdf_steps(int dir, double *svals) {
  double slo = exp(-3.0), shi = exp(3.0), sinc = exp(0.2), s;
  int ns = 0;
  if (dir == 'd') {
    s = slo;
    slo = shi;
    shi = s;
    sinc = 1.0 / sinc;
  }
  for (s = slo; slo < shi ? s < shi * sqrt(sinc) : s > shi * sqrt(sinc); s *= sinc) svals[ns++] = s;
  return ns;
}

/* rdfmaketable (rxnparam.c:920-1005) and rdfmaketableprob (1008-1114)
 * without the terminal dialogue: for each row of `mode` and each reaction
 * probability, build the grid, set the trial rdf (the Smoluchowski form when
 * sweeping upward in modes 'i' and 'r', else a step at 1) and sweep the step
 * length, each steady state starting from the previous one; after a failed
 * solve the rest of the sweep stays -1.  probs == NULL means a single
 * probability of 1 (rdfmaketable).  flux[(row*nprob + p)*31 + k]; iters
 * (optional) receives the iteration counts in the same layout. */
int ora_rdf_table(int mode, int n, double eps, int dir, int nprob, const double *probs, double *flux,
                  int *iters, double *rbuf, double *rdfa, double *rdfd) {
  double bvals[32], svals[40];
  const int nb = ora_rdf_rows(mode, bvals), ns = ora_rdf_steps(dir, svals);
  const double one = 1.0;
  if (!probs) {
    probs = &one;
    nprob = 1;
  }
  for (int row = 0; row < nb; ++row) {
    const double b = bvals[row];
    if (ora_rdf_grid(mode, n, b, rbuf)) return -1;
    for (int p = 0; p < nprob; ++p) {
      int i = 0;
      for (; i < n && rbuf[i] < 1; ++i) rdfa[i] = 0;
      if (dir == 'u' && mode == 'i')
        for (; i < n; ++i) rdfa[i] = 1.0 - 1.0 / rbuf[i];
      else if (dir == 'u' && mode == 'r')
        for (; i < n && rbuf[i] < b; ++i) rdfa[i] = 1.0 - (b - rbuf[i]) / rbuf[i] / (b - 1.0);
      for (; i < n; ++i) rdfa[i] = 1.0;
      double f = 0;
      for (int k = 0; k < ns; ++k) {
        int it = 0;
        if (probs[p] == 0)
          f = 0;
        else if (f >= 0)
          f = ora_rdf_steady(rbuf, rdfa, rdfd, n, svals[k], 1, b, eps, probs[p], &it);
        flux[((size_t)row * nprob + p) * ns + k] = f;
        if (iters) iters[((size_t)row * nprob + p) * ns + k] = it;
      }
    }
  }
  return nb;
}
