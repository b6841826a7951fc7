// Binding / unbinding radius solver (FP64), usable from host and device code.
//
// Restates the algorithm of Smoldyn's source/libSteve/rxnparam.c:
//   numrxnrate        rxnparam.c:57-158   tabulated per-step rate, cubic (Lagrange)
//                                          interpolation in ln(s/a) and in b/a or ln(b/a)
//   numrxnrateprob    rxnparam.c:161-518  same with reaction probability p<1,
//                                          trilinear over (ln s, p, b) + lambda-rho theory
//   bindingradius     rxnparam.c:558-584  doubling + 15 halvings on numrxnrate
//   bindingradiusprob rxnparam.c:587-681  p- or chi-constrained multiplicative search
//   unbindingradius   rxnparam.c:690-716  doubling + 15 halvings on 1-ki/k(b)
// The table data (rxnparam.c:58-391) comes from the generated header; the
// interpolation weights keep the reference's arithmetic order so that the
// bisections take the same branches (results match to ~1e-15 relative).
//
// On the device the tables live in global memory (they total 62.5 KB, too
// close to the 64 KB constant bank to share it with the engine's constants).
#pragma once

#include <math.h>
#include "_gen/rxntables.h"

#ifdef __CUDACC__
#define SMOLB_HD __host__ __device__
#else
#define SMOLB_HD
#endif

namespace smolb {
namespace rxnp {

#ifdef __CUDACC__
// one translation unit (engine.cu) compiles device code, so the device copies
// are defined here
static __device__ const double d_yi[SMOLB_TAB_YI_LEN] = SMOLB_TAB_YI_INIT;
static __device__ const double d_yr[SMOLB_TAB_YR_LEN] = SMOLB_TAB_YR_INIT;
static __device__ const double d_yb[SMOLB_TAB_YB_LEN] = SMOLB_TAB_YB_INIT;
static __device__ const double d_kirr[SMOLB_TAB_KIRR_LEN] = SMOLB_TAB_KIRR_INIT;
static __device__ const double d_krev[SMOLB_TAB_KREV_LEN] = SMOLB_TAB_KREV_INIT;
static __device__ const double d_kb[SMOLB_TAB_KB_LEN] = SMOLB_TAB_KB_INIT;
#endif
extern const double h_yi[SMOLB_TAB_YI_LEN];
extern const double h_yr[SMOLB_TAB_YR_LEN];
extern const double h_yb[SMOLB_TAB_YB_LEN];
extern const double h_kirr[SMOLB_TAB_KIRR_LEN];
extern const double h_krev[SMOLB_TAB_KREV_LEN];
extern const double h_kb[SMOLB_TAB_KB_LEN];

struct Tables {
  const double *yi, *yr, *yb, *kirr, *krev, *kb;
};

SMOLB_HD inline Tables tables() {
#if defined(__CUDA_ARCH__)
  return Tables{d_yi, d_yr, d_yb, d_kirr, d_krev, d_kb};
#else
  return Tables{h_yi, h_yr, h_yb, h_kirr, h_krev, h_kb};
#endif
}

constexpr double kPi = 3.14159265358979323846;

// floor(q) as an int, with q clamped to +-1e6 first so that non-finite or huge
// arguments (e.g. a binding radius that diverged to infinity) cannot overflow
// the conversion; finite table lookups never come near the clamp.
SMOLB_HD inline int ifloor_clamped(double q) {
  if (!(q > -1e6)) q = -1e6;
  if (q > 1e6) q = 1e6;
  return (int)floor(q);
}

// Weights of the cubic Lagrange interpolant through nodes x0..x3 spaced by
// `inc`, evaluated at t (rxnparam.c:94-97 form).
SMOLB_HD inline void lagrange4(double t, const double x[4], double inc, double w[4]) {
  w[0] = (t - x[1]) * (t - x[2]) * (t - x[3]) / (-6.0 * inc * inc * inc);
  w[1] = (t - x[0]) * (t - x[2]) * (t - x[3]) / (2.0 * inc * inc * inc);
  w[2] = (t - x[0]) * (t - x[1]) * (t - x[3]) / (-2.0 * inc * inc * inc);
  w[3] = (t - x[0]) * (t - x[1]) * (t - x[2]) / (6.0 * inc * inc * inc);
}

// Reaction rate times dt (units of length^3) for rms step `step`, binding
// radius a and unbinding radius b (b<0: irreversible).  rxnparam.c:57-158.
SMOLB_HD inline double numrxnrate(double step, double a, double b) {
  const Tables T = tables();
  const double slo = 3, sinc = -0.2;       // ln(s/a) grid, decreasing
  const double blor = 0, bincr = 0.2;      // ln(b/a) grid for b>=a
  const double blob = 0, bincb = 0.1;      // b/a grid for b<a
  const int snum = 31, bnumr = 16, bnumb = 11;
  double x[4], w[4], y[4];

  if (step < 0 || a < 0) return -1;
  if (step == 0 && b >= 0 && b < 1) return -1;
  if (step == 0) return 0;
  const double ls = log(step / a);
  b /= a;

  int si = ifloor_clamped((ls - slo) / sinc);
  for (int i = 0; i < 4; i++) x[i] = slo + (si - 1 + i) * sinc;
  lagrange4(ls, x, sinc, w);

  double ans = 0;
  if (b < 0) {
    for (int i = 0; i < 4; i++) {
      const int k = si - 1 + i;
      if (k >= snum) ans += w[i] * 2.0 * kPi * exp(2.0 * x[i]);
      else if (k < 0) ans += w[i] * 4.0 * kPi / 3.0;
      else ans += w[i] * T.yi[k];
    }
  } else if (b < 1.0) {
    int bi = ifloor_clamped((b - blob) / bincb);
    if (bi < 1) bi = 1;
    else if (bi + 2 >= bnumb) bi = bnumb - 3;
    // step back along s until the 4 columns used hold valid data
    while (si + 3 >= snum || (si > 0 && T.yb[(bi - 1) * snum + si + 3] < 0)) si--;
    for (int i = 0; i < 4; i++) x[i] = slo + (si - 1 + i) * sinc;
    lagrange4(ls, x, sinc, w);
    for (int j = 0; j < 4; j++) {
      y[j] = 0;
      for (int i = 0; i < 4; i++) {
        const int k = si - 1 + i;
        if (k >= snum) y[j] += w[i] * T.yb[(bi - 1 + j) * snum];
        else if (k < 0) y[j] += w[i] * 4.0 * kPi / 3.0;
        else y[j] += w[i] * T.yb[(bi - 1 + j) * snum + k];
      }
    }
    for (int j = 0; j < 4; j++) x[j] = blob + (bi - 1 + j) * bincb;
    lagrange4(b, x, bincb, w);
    ans = w[0] * y[0] + w[1] * y[1] + w[2] * y[2] + w[3] * y[3];
  } else {
    const double lb = log(b);
    int bi = ifloor_clamped((lb - blor) / bincr);
    if (bi < 1) bi = 1;
    else if (bi + 2 >= bnumr) bi = bnumr - 3;
    for (int j = 0; j < 4; j++) {
      y[j] = 0;
      for (int i = 0; i < 4; i++) {
        const int k = si - 1 + i;
        if (k >= snum && lb == 0) y[j] += w[i] * 2.0 * kPi * exp(x[i]) * (1.0 + exp(x[i]));
        else if (k >= snum) y[j] += w[i] * 2.0 * kPi * exp(2.0 * x[i]) * exp(lb) / (exp(lb) - 1.0);
        else if (k < 0) y[j] += w[i] * 4.0 * kPi / 3.0;
        else y[j] += w[i] * T.yr[(bi - 1 + j) * snum + k];
      }
    }
    for (int j = 0; j < 4; j++) x[j] = blor + (bi - 1 + j) * bincr;
    lagrange4(lb, x, bincr, w);
    ans = w[0] * y[0] + w[1] * y[1] + w[2] * y[2] + w[3] * y[3];
  }
  return ans * a * a * a;
}

// Trilinear interpolation helper over a (b, p, s) cube of table values.
SMOLB_HD inline double tri_interp(const double *tab, int snum, int pnum, int bi, int pi, int si,
                                  double wb0, double wb1, double wp0, double wp1, double ws0,
                                  double ws1, double denom) {
  const int o00 = bi * snum * pnum + pi * snum + si;
  const int o01 = bi * snum * pnum + (pi + 1) * snum + si;
  const int o10 = (bi + 1) * snum * pnum + pi * snum + si;
  const int o11 = (bi + 1) * snum * pnum + (pi + 1) * snum + si;
  const double numlll = wb0 * wp0 * ws0, numllh = wb0 * wp0 * ws1;
  const double numlhl = wb0 * wp1 * ws0, numlhh = wb0 * wp1 * ws1;
  const double numhll = wb1 * wp0 * ws0, numhlh = wb1 * wp0 * ws1;
  const double numhhl = wb1 * wp1 * ws0, numhhh = wb1 * wp1 * ws1;
  return (numlll * tab[o00] + numllh * tab[o00 + 1] + numlhl * tab[o01] + numlhh * tab[o01 + 1] +
          numhll * tab[o10] + numhlh * tab[o10 + 1] + numhhl * tab[o11] + numhhh * tab[o11 + 1]) /
         denom;
}

// Per-step rate for reaction probability p (0<p<1).  rxnparam.c:161-518.
SMOLB_HD inline double numrxnrateprob(double step, double a, double b, double prob) {
  const Tables T = tables();
  const double slo = -3, sinc = 0.2, shi = 3;
  const double blor = 0, bincr = 0.2;
  const double blob = 0, bincb = 0.1;
  const double pvect[8] = {0, 0.01, 0.02, 0.05, 0.1, 0.2, 0.5, 1.0};
  const int snum = 31, bnumr = 16, bnumb = 11, pnum = 8;

  if (prob == 1) return numrxnrate(step, a, b);
  if (step < 0 || a < 0) return -1;
  if (prob < 0 || prob > 1) return -1;
  if (prob == 0) return 0;
  if (a == 0) return 0;
  if (step == 0 && b >= 0 && b < a) return -1;
  if (step == 0) return 0;

  const double ansp1 = numrxnrate(step, a, b);
  step /= a;
  const double logstep = log(step);
  b /= a;

  int si, sflag = 0;
  double steplo, stephi;
  if (b < 0 || b >= 1.0) {
    si = ifloor_clamped((logstep - slo) / sinc);
    if (si < 0) { si = 0; sflag = -1; }
    else if (si > snum - 2) si = snum - 2;
    else sflag = 0;
    steplo = slo + si * sinc;
    stephi = slo + (si + 1) * sinc;
  } else {
    si = ifloor_clamped((shi - logstep) / sinc);
    if (si < 0) { si = 0; sflag = -1; }
    else if (si > snum - 2) si = snum - 2;
    else sflag = 0;
    steplo = shi - si * sinc;
    stephi = shi - (si + 1) * sinc;
  }
  int pi = 0;
  while (pi < pnum - 2 && prob > pvect[pi + 1]) pi++;
  const double problo = pvect[pi], probhi = pvect[pi + 1];

  double ans;
  if (b < 0) {
    const double denom = (probhi - problo) * (stephi - steplo);
    const double numll = (probhi - prob) * (stephi - logstep);
    const double numlh = (probhi - prob) * (logstep - steplo);
    const double numhl = (prob - problo) * (stephi - logstep);
    const double numhh = (prob - problo) * (logstep - steplo);
    ans = (numll * T.kirr[pi * snum + si] + numlh * T.kirr[pi * snum + si + 1] +
           numhl * T.kirr[(pi + 1) * snum + si] + numhh * T.kirr[(pi + 1) * snum + si + 1]) /
          denom;
    if (si == 0) {
      const double lambdap = sqrt(2 * prob) / step;
      const double theory = 2 * kPi * step * step * (1 - tanh(lambdap) / lambdap);
      if (sflag == -1) ans = theory;
      else {
        const double step0 = exp(steplo), step1 = exp(steplo + sinc);
        ans = ((step - step0) * ans + (step1 - step) * theory) / (step1 - step0);
      }
    } else if (ans > 4.0 * kPi / 3.0 * prob) {
      ans = 4.0 * kPi / 3.0 * prob;
    }
  } else if (b >= 1.0) {
    const double logb = log(b);
    int bi = ifloor_clamped((logb - blor) / bincr);
    if (bi < 0) bi = 0;
    else if (bi > bnumr - 2) bi = bnumr - 2;
    const double blo = blor + bi * bincr, bhi = blor + (bi + 1) * bincr;
    const double denom = (bhi - blo) * (probhi - problo) * (stephi - steplo);
    ans = tri_interp(T.krev, snum, pnum, bi, pi, si, bhi - logb, logb - blo, probhi - prob,
                     prob - problo, stephi - logstep, logstep - steplo, denom);
    if (si == 0) {
      const double lambdap = sqrt(2 * prob) / step;
      double theory;
      if (lambdap < 10)
        theory = 2 * kPi * step * step * b * (lambdap * cosh(lambdap) - sinh(lambdap)) /
                 (lambdap * (b - 1) * cosh(lambdap) + sinh(lambdap));
      else
        theory = 2 * kPi * step * step * b * (lambdap - 1) / (lambdap * (b - 1) + 1);
      if (sflag == -1) ans = theory;
      else {
        const double step0 = exp(steplo), step1 = exp(steplo + sinc);
        ans = ((step - step0) * ans + (step1 - step) * theory) / (step1 - step0);
      }
    } else if (ans > 4.0 * kPi / 3.0 * prob) {
      ans = 4.0 * kPi / 3.0 * prob;
    }
  } else {
    int bi = ifloor_clamped((b - blob) / bincb);
    if (bi < 0) bi = 0;
    else if (bi > bnumb - 2) bi = bnumb - 2;
    const double blo = blob + bi * bincb, bhi = blob + (bi + 1) * bincb;
    while (T.kb[bi * snum * pnum + (pi + 1) * snum + si + 1] == -1) si--;
    steplo = shi - si * sinc;
    stephi = shi - (si + 1) * sinc;
    const double denom = (bhi - blo) * (probhi - problo) * (stephi - steplo);
    ans = tri_interp(T.kb, snum, pnum, bi, pi, si, bhi - b, b - blo, probhi - prob, prob - problo,
                     stephi - logstep, logstep - steplo, denom);
  }
  ans *= a * a * a;
  if (ans > ansp1) ans = ansp1;
  return ans;
}

// Binding radius for rate constant `rate` (not reduced), time step dt and
// mutual diffusion coefficient difc.  b<0: irreversible; b>=0 & rel=0: b is the
// unbinding radius; rel=1: b is the ratio b/a.  rxnparam.c:558-584.
SMOLB_HD inline double bindingradius(double rate, double dt, double difc, double b, int rel) {
  if (rate < 0 || dt < 0 || difc <= 0) return -1;
  if (rate == 0) return 0;
  if (dt == 0) {
    if (b < 0) return rate / (4 * kPi * difc);
    if (rel && b > 1) return rate * (1 - 1 / b) / (4 * kPi * difc);
    if (rel && b <= 1) return -1;
    if (b > 0) return rate / (4 * kPi * difc + rate / b);
    return -1;
  }
  const double step = sqrt(2.0 * difc * dt);
  const double target = rate * dt;
  double lo = 0, a = step;
  while (numrxnrate(step, a, rel ? b * a : b) < target) {
    lo = a;
    a *= 2.0;
    if (!(a < 1e300)) return INFINITY;  // rate unreachable (e.g. ratio < 1)
  }
  double dif = a - lo;
  for (int n = 0; n < 15; n++) {
    dif *= 0.5;
    a = lo + dif;
    if (numrxnrate(step, a, rel ? b * a : b) < target) lo = a;
  }
  return lo + 0.5 * dif;
}

SMOLB_HD inline double chi_of(double rate, double difc, double a, double ub) {
  return (ub >= 0) ? rate / (4 * kPi * difc * a * ub / (ub - a)) : rate / (4 * kPi * difc * a);
}

// rxnparam.c:587-681.  probptr in/out as in the reference.
SMOLB_HD inline double bindingradiusprob(double rate, double dt, double difc, double b, int rel,
                                         double chi, double *probptr) {
  if (rate < 0 || dt < 0 || difc <= 0 || chi > 1) return -1;
  if (chi < 0 && (!probptr || *probptr == 1)) return bindingradius(rate, dt, difc, b, rel);
  if (chi < 0 && probptr && *probptr == 0) return 0;
  if (rate == 0) {
    if (probptr && *probptr < 0) *probptr = 0;
    return 0;
  }
  double abest, pbest;
  if (dt == 0) {
    double a;
    if (chi < 0) return -1;
    else if (b < 0) a = rate / (4 * kPi * difc * chi);
    else if (rel && b > 1) a = rate * (1 - 1 / b) / (4 * kPi * difc * chi);
    else if (rel && b <= 1) return -1;
    else if (b > 0) a = rate * b / (rate + 4 * kPi * difc * b * chi);
    else return -1;
    const double lambdap =
        (3.18243 * chi - 3.40864 * chi * chi + 0.984385 * chi * chi * chi) / pow(1 - chi, 2.08761);
    const double lambda = difc * lambdap / a * lambdap / a;
    if (probptr) *probptr = lambda;
    return a;
  }
  const double step = sqrt(2 * difc * dt);
  if (chi < 0) {  // known reaction probability, search the binding radius
    const double prob = *probptr;
    pbest = prob;
    double xa = step, xmult = 0.1;
    abest = xa;
    double ub = (b >= 0) ? (rel ? b * xa : b) : -1;
    double ratetry = numrxnrateprob(step, xa, ub, prob) / dt;
    double errtry = (ratetry / rate - 1.0) * (ratetry / rate - 1.0), errbest = errtry;
    for (int it = 0; it < 200 && errtry > 1.0e-6; it++) {
      const double errold = errtry;
      xa = xa * (1.0 + xmult);
      if (xa < 1.0e-15) xa = 1.0e-15;
      else if (xa > 1.0e15) xa = 1.0e15;
      ub = (b >= 0) ? (rel ? b * xa : b) : -1;
      ratetry = numrxnrateprob(step, xa, ub, prob) / dt;
      errtry = (ratetry / rate - 1.0) * (ratetry / rate - 1.0);
      if (errtry < errold) xmult *= 1.1;
      else xmult *= -0.5;
      if (errtry < errbest) {
        errbest = errtry;
        abest = xa;
      }
    }
  } else {  // known chi: 2-D search over (a, p)
    double x[2], xmult[2], xlo[2], xhi[2];
    x[0] = abest = bindingradius(rate, dt, difc, b, rel);
    x[1] = pbest = 1;
    double ub = (b >= 0) ? (rel ? b * x[0] : b) : -1;
    double chitry = chi_of(rate, difc, x[0], ub);
    if (chitry > chi) {
      xmult[0] = xmult[1] = 0.1;
      xlo[0] = xlo[1] = 1.0e-15;
      xhi[0] = 1.0e15;
      xhi[1] = 1.0;
      x[0] = abest = step;
      x[1] = pbest = 0.5;
      double ratetry = numrxnrateprob(step, x[0], rel ? b * x[0] : b, x[1]) / dt;
      ub = (b >= 0) ? (rel ? b * x[0] : b) : -1;
      chitry = chi_of(rate, difc, x[0], ub);
      double errtry = (ratetry / rate - 1.0) * (ratetry / rate - 1.0) +
                      (chitry / chi - 1.0) * (chitry / chi - 1.0);
      double errbest = errtry;
      for (int it = 0; it < 300 && errtry > 1.0e-6; it++) {
        for (int k = 0; k < 2; k++) {
          const double errold = errtry;
          x[k] = x[k] * (1.0 + xmult[k]);
          if (x[k] < xlo[k]) x[k] = xlo[k];
          else if (x[k] > xhi[k]) x[k] = xhi[k];
          ratetry = numrxnrateprob(step, x[0], rel ? b * x[0] : b, x[1]) / dt;
          ub = (b >= 0) ? (rel ? b * x[0] : b) : -1;
          chitry = chi_of(rate, difc, x[0], ub);
          errtry = (ratetry / rate - 1.0) * (ratetry / rate - 1.0) +
                   (chitry / chi - 1.0) * (chitry / chi - 1.0);
          if (errtry < errold) xmult[k] *= 1.1;
          else xmult[k] *= -0.5;
          if (errtry < errbest) {
            errbest = errtry;
            abest = x[0];
            pbest = x[1];
          }
        }
      }
    }
  }
  if (chi >= 0 && probptr) *probptr = pbest;
  return abest;
}

// Unbinding radius for geminate rebinding probability pgem; returns -2 on bad
// input and -(max achievable pgem) when pgem is unreachable.  rxnparam.c:690-716.
SMOLB_HD inline double unbindingradius(double pgem, double dt, double difc, double a) {
  if (pgem <= 0 || pgem >= 1 || difc <= 0 || a <= 0 || dt < 0) return -2;
  if (!(a < INFINITY)) return -2;
  if (dt == 0) return a / pgem;
  const double step = sqrt(2.0 * difc * dt);
  const double ki = numrxnrate(step, a, -1);
  const double kmax = numrxnrate(step, a, 0);
  if (1.0 - ki / kmax < pgem) return ki / kmax - 1.0;
  double lo = 0, b = a;
  while (1.0 - ki / numrxnrate(step, a, b) > pgem) {
    lo = b;
    b *= 2.0;
    if (!(b < 1e300)) return -2;
  }
  double dif = b - lo;
  for (int n = 0; n < 15; n++) {
    dif *= 0.5;
    b = lo + dif;
    if (1.0 - ki / numrxnrate(step, a, b) > pgem) lo = b;
  }
  return lo + 0.5 * dif;
}

}  // namespace rxnp
}  // namespace smolb

namespace smolb {
namespace rxnp {

// RevParam codes used below (smoldyn.h:358)
enum : int { kRPnone = 0, kRPirrev = 1, kRPpgem = 4, kRPpgemmax = 5, kRPpgemmaxw = 6, kRPratio = 7,
             kRPunbindrad = 8 };

struct PairRadii {
  double bindrad;    // binding radius of A + B -> C
  double unbindrad;  // unbinding radius of the reverse C -> A + B (0 if none)
  int err;           // 0 ok, 1 illegal input, 2 requested pgem unreachable
};

// Binding radius of a bimolecular reaction with rate constant kf and, when
// it has a direct reverse (rev != 0), the unbinding radius of that reverse for
// its product placement (rparamt, rparam).  Restates the order-2 branch of
// rxnsetrate (smolreact.c:1364-1414, probability 1, no chi) followed by
// rxnsetproduct for the reverse reaction (smolreact.c:1519-1571); like species
// double the rate (smolreact.c:1374).  dsum = D_A + D_B.
SMOLB_HD inline PairRadii pair_radii(double kf, int same_species, double dsum, double dt, int rev, int rparamt,
                                     double rparam) {
  PairRadii o{0, 0, 0};
  double rate3 = same_species ? 2 * kf : kf;
  if (rev && rparamt == kRPnone) {
    rparamt = kRPpgemmaxw;
    rparam = 0.2;
  }
  if (!rev) rparamt = kRPnone;
  if (rate3 <= 0) return o;
  if (dsum <= 0) { o.err = 1; return o; }
  double a;
  if (rparamt == kRPunbindrad) a = bindingradius(rate3, dt, dsum, rparam, 0);
  else if (rparamt == kRPratio) a = bindingradius(rate3, dt, dsum, rparam, 1);
  else if (rparamt == kRPpgem) a = bindingradius(rate3 * (1.0 - rparam), dt, dsum, -1, 0);
  else if (rparamt == kRPpgemmax || rparamt == kRPpgemmaxw) {
    a = bindingradius(rate3, dt, dsum, 0, 0);
    const double ub = unbindingradius(rparam, dt, dsum, a);
    if (ub > 0) a = bindingradius(rate3 * (1.0 - rparam), dt, dsum, -1, 0);
  } else {
    a = bindingradius(rate3, dt, dsum, -1, 0);
  }
  o.bindrad = a;
  if (!rev || a <= 0) return o;
  if (rparamt == kRPunbindrad) o.unbindrad = rparam;
  else if (rparamt == kRPratio) o.unbindrad = rparam * a;
  else if (rparamt == kRPpgem) {
    const double r = unbindingradius(rparam, dt, dsum, a);
    if (r == -2) o.err = 1;
    else if (r < 0) o.err = 2;
    else o.unbindrad = r;
  } else if (rparamt == kRPpgemmax || rparamt == kRPpgemmaxw) {
    const double r = unbindingradius(rparam, dt, dsum, a);
    if (r == -2) o.err = 1;
    else o.unbindrad = r > 0 ? r : 0;
  }
  return o;
}

}  // namespace rxnp
}  // namespace smolb
