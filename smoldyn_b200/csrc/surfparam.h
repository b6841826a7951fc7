// Surface interaction probabilities from rate constants, restating the parts
// of SurfaceParam.c that srfcalcprob (smolsurface.c:3070-3146) uses: the
// per-step probability of adsorption, desorption, flipping and transmission
// (surfaceprob, SurfaceParam.c:66-200) and the desorption distance
// (desorbdist, :202-220).  The adsorption probabilities are read from the
// reference's published lookup tables (lookupirrevadsorb :504-523,
// lookuprevads :566-666) with the same 4-point Lagrange interpolation on the
// tabulated grid (interpolate1D :452-467, interpolate2D :470-501); the table
// values are generated into _gen/srftables.h from the public-domain source.
#pragma once

#include <math.h>

#include "_gen/srftables.h"

namespace smolb {

// Algorithms of SurfParamAlgo that the surface parameter derivation uses
// (SurfaceParam.h:11, same meaning).
enum SrfAlgo { kSrfIrrTrans, kSrfIrrAds, kSrfRevAds, kSrfIrrDes, kSrfRevDes, kSrfIrrFlip, kSrfRevFlip };

// Cubic Lagrange weights of v on the four grid points x[0..3].
inline void lagrange4(const double *x, double v, double w[4]) {
  for (int a = 0; a < 4; ++a) {
    double num = 1, den = 1;
    for (int b = 0; b < 4; ++b) {
      if (b == a) continue;
      num *= v - x[b];
      den *= x[a] - x[b];
    }
    w[a] = num / den;
  }
}

// First grid index of the 4-point stencil for v: the first entry not below v,
// less two, held inside the grid (interpolate1D's stencil choice).
inline int stencil4(const double *x, int n, double v) {
  int i = 0;
  while (i < n && x[i] < v) ++i;
  if (i < 2) i = 2;
  else if (i > n - 2) i = n - 2;
  return i - 2;
}

inline double interp_1d(const double *x, const double *y, int n, double v) {
  const int s = stencil4(x, n, v);
  double w[4];
  lagrange4(x + s, v, w);
  return w[0] * y[s] + w[1] * y[s + 1] + w[2] * y[s + 2] + w[3] * y[s + 3];
}

// z[i * ny + j] at (x[i], y[j]); y is the fast index.
inline double interp_2d(const double *x, const double *y, const double *z, int nx, int ny, double u, double v) {
  const int si = stencil4(x, nx, u), sj = stencil4(y, ny, v);
  double wx[4], wy[4];
  lagrange4(x + si, u, wx);
  lagrange4(y + sj, v, wy);
  double ans = 0;
  for (int b = 0; b < 4; ++b) {
    double col = 0;
    for (int a = 0; a < 4; ++a) col += wx[a] * z[(si + a) * ny + sj + b];
    ans += wy[b] * col;
  }
  return ans;
}

// Adsorption probability per collision of an irreversibly adsorbing surface
// with reduced adsorption coefficient kapp = kappa*dt/step.
inline double irrev_ads_prob(double kapp) {
  static const double pon[] = SMOLB_SRF_PON_INIT;
  static const double kap[] = SMOLB_SRF_KAPPA_INIT;
  const int n = SMOLB_SRF_PON_LEN;
  if (kapp <= 0) return 0;
  if (kapp >= kap[n - 1]) return 1.0;
  return interp_1d(kap, pon, n, kapp);
}

// Reversible adsorption: adsorption probability per collision from the
// reduced adsorption (kapp) and desorption (kp = kd*dt) coefficients, and in
// *pdes the matching desorption probability per step.
inline double rev_ads_prob(double kapp, double kp, double *pdes) {
  static const double x[] = SMOLB_SRF_REVX_INIT;
  static const double tab[] = SMOLB_SRF_REVADS_INIT;
  const int n = SMOLB_SRF_REVX_LEN;
  if (kapp < 0) kapp = 0;
  if (kp < 0) kp = 0;
  double p = interp_2d(x, x, tab, n, n, kapp / (1.0 + kapp), kp / (1.0 + kp));
  if (p < 0) p = 0;
  else if (p > 1) p = 1;
  if (pdes) *pdes = p * kp / kapp / 2.50662827462;  // sqrt(2 pi) as in the reference's SQRT2PI
  return p;
}

// erfc(x) by the Chebyshev fit of Press et al. (Numerical Recipes, "erfcc",
// fractional error below 1.2e-7), the form the reference's math2.c
// evaluates, so that transmission probabilities agree with it closely.
inline double erfc_fit(double x) {
  const double z = fabs(x), t = 1.0 / (1.0 + 0.5 * z);
  const double c[10] = {-1.26551223, 1.00002368, 0.37409196, 0.09678418, -0.18628806,
                        0.27886807, -1.13520398, 1.48851587, -0.82215223, 0.17087277};
  double poly = c[9];
  for (int k = 8; k >= 0; --k) poly = c[k] + t * poly;
  const double ans = t * exp(-z * z + poly);
  return x >= 0 ? ans : 2.0 - ans;
}

// exp(x^2) erfc(x) - 1: the Taylor series near 0, exp(x^2) erfc(x) from the
// fit for moderate x and its asymptotic series for |x| >= 20.
inline double exp_erfc_m1(double x) {
  const double sp = 1.7724538509;  // sqrt(pi) as in the reference's SQRTPI
  if (fabs(x) <= 0.05)
    return x * (-2.0 / sp + x * (1.0 + x * (-4.0 / 3.0 / sp + x * (0.5 + x * (-8.0 / 15.0 / sp +
               x * (1.0 / 6.0 + x * (-16.0 / 105.0 / sp + x * (1.0 / 24.0))))))));
  double e;
  if (fabs(x) < 20) {
    e = exp(x * x) * erfc_fit(x);
  } else {
    const double q = 1.0 / (x * x);
    e = (1.0 + q * (-0.5 + q * (0.75 + q * (-15.0 / 8.0 + q * (105.0 / 16.0 + q * (-945.0 / 32.0)))))) / (x * sp);
    if (x < 0) e += 2.0 * exp(x * x);
  }
  return e - 1.0;
}

// Partial transmission through a membrane with forward and backward
// transmission coefficients k1, k2 (surfacetransmit, SurfaceParam.c:297-446,
// after Andrews 2009, Phys. Biol. 6:046015): probabilities p1, p2 of
// crossing per collision for the given diffusion coefficients.  A rate of
// -1 ("always") fixes that side's probability at 1 and the other side's
// coefficient is found by solving for it (bisection; the reference searches
// with a random walk to 0.1%).  Returns 0, or 1 for unusable inputs.
inline void transmit_closed(double k1, double k2, double d1, double d2, double dt, double *p1, double *p2) {
  const double pi = 3.14159265358979323846;
  const double c = sqrt(dt) * (k1 / sqrt(d1) + k2 / sqrt(d2));
  const double ct = (2.0 * c / sqrt(pi) + exp_erfc_m1(c)) / (c * c);
  *p1 = k1 * sqrt(pi * dt) / sqrt(d1) * ct;
  *p2 = k2 * sqrt(pi * dt) / sqrt(d2) * ct;
}

inline int surface_transmit(double k1, double k2, double d1, double d2, double dt, double *p1, double *p2) {
  if (d1 <= 0 || d2 <= 0 || dt <= 0) return 1;
  if (k1 == 0 && k2 == 0) { *p1 = *p2 = 0; return 0; }
  if (k1 == 0 && k2 == -1) { *p1 = 0; *p2 = 1; return 0; }
  if (k1 == -1 && k2 == 0) { *p1 = 1; *p2 = 0; return 0; }
  if (k1 == -1 && k2 == -1) {
    if (d1 <= d2) { *p1 = 1; *p2 = sqrt(d1 / d2); }
    else { *p1 = sqrt(d2 / d1); *p2 = 1; }
    return 0;
  }
  if (k1 == -1 || k2 == -1) {
    // the "always" side crosses with probability 1: find its coefficient
    const bool first = k1 == -1;
    const double kf = first ? k2 : k1;
    double lo = -40, hi = 40;  // natural log of the unknown coefficient
    for (int it = 0; it < 200; ++it) {
      const double mid = 0.5 * (lo + hi), k = exp(mid);
      double a, b;
      if (first) transmit_closed(k, kf, d1, d2, dt, &a, &b);
      else transmit_closed(kf, k, d1, d2, dt, &a, &b);
      if ((first ? a : b) < 1.0) lo = mid;
      else hi = mid;
    }
    const double k = exp(0.5 * (lo + hi));
    double a, b;
    if (first) transmit_closed(k, kf, d1, d2, dt, &a, &b);
    else transmit_closed(kf, k, d1, d2, dt, &a, &b);
    if (first) { *p1 = 1; *p2 = b > 1 ? 1 : b; }
    else { *p2 = 1; *p1 = a > 1 ? 1 : a; }
    return 0;
  }
  double a, b;
  transmit_closed(k1, k2, d1, d2, dt, &a, &b);
  if (a > 1) { a = 1; b = k2 / k1 * sqrt(d1 / d2); }
  if (b > 1) { b = 1; a = k1 / k2 * sqrt(d2 / d1); }
  *p1 = a;
  *p2 = b;
  return 0;
}

// surfaceprob (SurfaceParam.c:66-200) for the algorithms above.  k1 is the
// rate of the action, k2 the rate of its reverse (or, for irreversible
// desorption and flips, the sum of the state's leaving rates); a rate of -1
// means "every time".  *p2 gets the reverse probability where one is computed.
inline double surface_prob(double k1, double k2, double dt, double difc, double *p2, SrfAlgo algo) {
  const double step = sqrt(2.0 * difc * dt);
  double a = 0, b = 0;
  switch (algo) {
    case kSrfIrrTrans:
    case kSrfIrrAds:
      a = (k1 == -1) ? 1.0 : irrev_ads_prob(k1 * dt / step);
      break;
    case kSrfRevAds:
      if (k1 == -1 && k2 == -1) a = b = 1;
      else if (k1 == -1) { a = 1; b = 1.0 - exp(-k2 * dt); }
      else if (k2 == -1) { b = 1; a = irrev_ads_prob(k1 * dt / step); }
      else a = rev_ads_prob(k1 * dt / step, k2 * dt, &b);
      break;
    case kSrfIrrDes:
    case kSrfIrrFlip:
      if (k1 == -1) a = 1;
      else {
        if (k2 <= 0) k2 = k1;
        a = k1 / k2 * (1.0 - exp(-k2 * dt));
      }
      break;
    case kSrfRevDes:
      if (k1 == -1 && k2 == -1) a = b = 1;
      else if (k1 == -1) { a = 1; b = irrev_ads_prob(k2 * dt / step); }
      else if (k2 == -1) { a = 1.0 - exp(-k2 * dt); b = 1; }  // as the reference computes it
      else b = surface_prob(k2, k1, dt, difc, &a, kSrfRevAds);
      break;
    case kSrfRevFlip:
      if (k1 == -1 && k2 == -1) a = b = 1;
      else if (k1 == -1) { a = 1; b = 1.0 - exp(-k2 * dt); }
      else if (k2 == -1) { a = 1.0 - exp(-k1 * dt); b = 1; }
      else {
        const double f = 1.0 - exp(-(k1 + k2) * dt);
        a = k1 / (k1 + k2) * f;
        b = k2 / (k1 + k2) * f;
      }
      break;
  }
  if (p2) *p2 = b;
  return a;
}

}  // namespace smolb
