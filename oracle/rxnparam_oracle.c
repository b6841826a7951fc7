/* Oracle restatement of the reference's binding/unbinding radius solver.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Follows source/libSteve/rxnparam.c function by function (line numbers
 * cited per function); the lookup tables come from the header generated from
 * that file (smoldyn_b200/csrc/gen_rxntables.py).  Plain C, FP64, no shared
 * code with the product library.
 */
#include <math.h>

#include "oracle.h"
#include "rxntables.h"

static const double T_yi[] = SMOLB_TAB_YI_INIT;
static const double T_yr[] = SMOLB_TAB_YR_INIT;
static const double T_yb[] = SMOLB_TAB_YB_INIT;
static const double T_kirr[] = SMOLB_TAB_KIRR_INIT;
static const double T_krev[] = SMOLB_TAB_KREV_INIT;
static const double T_kb[] = SMOLB_TAB_KB_INIT;

#define O_PI 3.14159265358979323846

/* cubic Lagrange weights on 4 equally spaced nodes (rxnparam.c:94-97) */
static void weights4(double t, const double *x, double h, double *z) {
  z[0] = (t - x[1]) * (t - x[2]) * (t - x[3]) / (-6.0 * h * h * h);
  z[1] = (t - x[0]) * (t - x[2]) * (t - x[3]) / (2.0 * h * h * h);
  z[2] = (t - x[0]) * (t - x[1]) * (t - x[3]) / (-2.0 * h * h * h);
  z[3] = (t - x[0]) * (t - x[1]) * (t - x[2]) / (6.0 * h * h * h);
}

/* rxnparam.c:57-158 */
double ora_numrxnrate(double step, double a, double b) {
  const double slo = 3, sinc = -0.2, blor = 0, bincr = 0.2, blob = 0, bincb = 0.1;
  const int snum = 31, bnumr = 16, bnumb = 11;
  double x[4], y[4], z[4], ans, s;
  int si, bi, i, j;

  if (step < 0 || a < 0) return -1;
  if (step == 0 && b >= 0 && b < 1) return -1;
  if (step == 0) return 0;
  s = log(step / a);
  b /= a;
  si = (int)floor((s - slo) / sinc);
  for (i = 0; i < 4; i++) x[i] = slo + (si - 1 + i) * sinc;
  weights4(s, x, sinc, z);
  if (b < 0) {
    ans = 0;
    for (i = 0; i < 4; i++) {
      int k = si - 1 + i;
      ans += (k >= snum) ? z[i] * 2.0 * O_PI * exp(2.0 * x[i])
                         : (k < 0) ? z[i] * 4.0 * O_PI / 3.0 : z[i] * T_yi[k];
    }
  } else if (b < 1.0) {
    bi = (int)floor((b - blob) / bincb);
    if (bi < 1) bi = 1;
    else if (bi + 2 >= bnumb) bi = bnumb - 3;
    while (si + 3 >= snum || (si > 0 && T_yb[(bi - 1) * snum + si + 3] < 0)) si--;
    for (i = 0; i < 4; i++) x[i] = slo + (si - 1 + i) * sinc;
    weights4(s, x, sinc, z);
    for (j = 0; j < 4; j++) {
      y[j] = 0;
      for (i = 0; i < 4; i++) {
        int k = si - 1 + i;
        y[j] += (k >= snum) ? z[i] * T_yb[(bi - 1 + j) * snum]
                            : (k < 0) ? z[i] * 4.0 * O_PI / 3.0 : z[i] * T_yb[(bi - 1 + j) * snum + k];
      }
    }
    for (j = 0; j < 4; j++) x[j] = blob + (bi - 1 + j) * bincb;
    weights4(b, x, bincb, z);
    ans = z[0] * y[0] + z[1] * y[1] + z[2] * y[2] + z[3] * y[3];
  } else {
    b = log(b);
    bi = (int)floor((b - blor) / bincr);
    if (bi < 1) bi = 1;
    else if (bi + 2 >= bnumr) bi = bnumr - 3;
    for (j = 0; j < 4; j++) {
      y[j] = 0;
      for (i = 0; i < 4; i++) {
        int k = si - 1 + i;
        if (k >= snum && b == 0) y[j] += z[i] * 2.0 * O_PI * exp(x[i]) * (1.0 + exp(x[i]));
        else if (k >= snum) y[j] += z[i] * 2.0 * O_PI * exp(2.0 * x[i]) * exp(b) / (exp(b) - 1.0);
        else if (k < 0) y[j] += z[i] * 4.0 * O_PI / 3.0;
        else y[j] += z[i] * T_yr[(bi - 1 + j) * snum + k];
      }
    }
    for (j = 0; j < 4; j++) x[j] = blor + (bi - 1 + j) * bincr;
    weights4(b, x, bincr, z);
    ans = z[0] * y[0] + z[1] * y[1] + z[2] * y[2] + z[3] * y[3];
  }
  return ans * a * a * a;
}

/* trilinear blend of a table cube (rxnparam.c:449-466 form) */
static double cube8(const double *t, int snum, int pnum, int bi, int pi, int si, double b0, double b1,
                    double p0, double p1, double s0, double s1) {
  const int g = snum * pnum;
  return b0 * p0 * s0 * t[bi * g + pi * snum + si] + b0 * p0 * s1 * t[bi * g + pi * snum + si + 1] +
         b0 * p1 * s0 * t[bi * g + (pi + 1) * snum + si] + b0 * p1 * s1 * t[bi * g + (pi + 1) * snum + si + 1] +
         b1 * p0 * s0 * t[(bi + 1) * g + pi * snum + si] + b1 * p0 * s1 * t[(bi + 1) * g + pi * snum + si + 1] +
         b1 * p1 * s0 * t[(bi + 1) * g + (pi + 1) * snum + si] +
         b1 * p1 * s1 * t[(bi + 1) * g + (pi + 1) * snum + si + 1];
}

/* rxnparam.c:161-518 */
double ora_numrxnrateprob(double step, double a, double b, double prob) {
  const double slo = -3, sinc = 0.2, shi = 3, blor = 0, bincr = 0.2, blob = 0, bincb = 0.1;
  static const double pv[8] = {0, 0.01, 0.02, 0.05, 0.1, 0.2, 0.5, 1.0};
  const int snum = 31, bnumr = 16, bnumb = 11, pnum = 8;
  double ls, slo_, shi_, plo, phi, ans, ansp1, theory, lam, blo, bhi, lb, den;
  int si, sflag = 0, pi, bi;

  if (prob == 1) return ora_numrxnrate(step, a, b);
  if (step < 0 || a < 0) return -1;
  if (prob < 0 || prob > 1) return -1;
  if (prob == 0) return 0;
  if (a == 0) return 0;
  if (step == 0 && b >= 0 && b < a) return -1;
  if (step == 0) return 0;
  ansp1 = ora_numrxnrate(step, a, b);
  step /= a;
  ls = log(step);
  b /= a;
  if (b < 0 || b >= 1.0) {
    si = (int)floor((ls - slo) / sinc);
    if (si < 0) { si = 0; sflag = -1; }
    else if (si > snum - 2) si = snum - 2;
    slo_ = slo + si * sinc;
    shi_ = slo + (si + 1) * sinc;
  } else {
    si = (int)floor((shi - ls) / sinc);
    if (si < 0) { si = 0; sflag = -1; }
    else if (si > snum - 2) si = snum - 2;
    slo_ = shi - si * sinc;
    shi_ = shi - (si + 1) * sinc;
  }
  for (pi = 0; pi < pnum - 2 && prob > pv[pi + 1]; pi++) ;
  plo = pv[pi];
  phi = pv[pi + 1];
  if (b < 0) {
    den = (phi - plo) * (shi_ - slo_);
    ans = ((phi - prob) * (shi_ - ls) * T_kirr[pi * snum + si] + (phi - prob) * (ls - slo_) * T_kirr[pi * snum + si + 1] +
           (prob - plo) * (shi_ - ls) * T_kirr[(pi + 1) * snum + si] +
           (prob - plo) * (ls - slo_) * T_kirr[(pi + 1) * snum + si + 1]) / den;
    if (si == 0) {
      lam = sqrt(2 * prob) / step;
      theory = 2 * O_PI * step * step * (1 - tanh(lam) / lam);
      if (sflag == -1) ans = theory;
      else {
        double s0 = exp(slo_), s1 = exp(slo_ + sinc);
        ans = ((step - s0) * ans + (s1 - step) * theory) / (s1 - s0);
      }
    } else if (ans > 4.0 * O_PI / 3.0 * prob) ans = 4.0 * O_PI / 3.0 * prob;
  } else if (b >= 1.0) {
    lb = log(b);
    bi = (int)floor((lb - blor) / bincr);
    if (bi < 0) bi = 0;
    else if (bi > bnumr - 2) bi = bnumr - 2;
    blo = blor + bi * bincr;
    bhi = blor + (bi + 1) * bincr;
    den = (bhi - blo) * (phi - plo) * (shi_ - slo_);
    ans = cube8(T_krev, snum, pnum, bi, pi, si, bhi - lb, lb - blo, phi - prob, prob - plo, shi_ - ls, ls - slo_) / den;
    if (si == 0) {
      lam = sqrt(2 * prob) / step;
      if (lam < 10)
        theory = 2 * O_PI * step * step * b * (lam * cosh(lam) - sinh(lam)) / (lam * (b - 1) * cosh(lam) + sinh(lam));
      else theory = 2 * O_PI * step * step * b * (lam - 1) / (lam * (b - 1) + 1);
      if (sflag == -1) ans = theory;
      else {
        double s0 = exp(slo_), s1 = exp(slo_ + sinc);
        ans = ((step - s0) * ans + (s1 - step) * theory) / (s1 - s0);
      }
    } else if (ans > 4.0 * O_PI / 3.0 * prob) ans = 4.0 * O_PI / 3.0 * prob;
  } else {
    bi = (int)floor((b - blob) / bincb);
    if (bi < 0) bi = 0;
    else if (bi > bnumb - 2) bi = bnumb - 2;
    blo = blob + bi * bincb;
    bhi = blob + (bi + 1) * bincb;
    while (T_kb[bi * snum * pnum + (pi + 1) * snum + si + 1] == -1) si--;
    slo_ = shi - si * sinc;
    shi_ = shi - (si + 1) * sinc;
    den = (bhi - blo) * (phi - plo) * (shi_ - slo_);
    ans = cube8(T_kb, snum, pnum, bi, pi, si, bhi - b, b - blo, phi - prob, prob - plo, shi_ - ls, ls - slo_) / den;
  }
  ans *= a * a * a;
  return ans > ansp1 ? ansp1 : ans;
}

/* rxnparam.c:558-584 */
double ora_bindingradius(double rate, double dt, double difc, double b, int rel) {
  double a, lo, dif, step;
  int n;
  if (rate < 0 || dt < 0 || difc <= 0) return -1;
  if (rate == 0) return 0;
  if (dt == 0) {
    if (b < 0) return rate / (4 * O_PI * difc);
    if (rel && b > 1) return rate * (1 - 1 / b) / (4 * O_PI * difc);
    if (rel && b <= 1) return -1;
    if (b > 0) return rate / (4 * O_PI * difc + rate / b);
    return -1;
  }
  step = sqrt(2.0 * difc * dt);
  lo = 0;
  a = step;
  while (ora_numrxnrate(step, a, rel ? b * a : b) < rate * dt) { lo = a; a *= 2.0; }
  dif = a - lo;
  for (n = 0; n < 15; n++) {
    dif *= 0.5;
    a = lo + dif;
    if (ora_numrxnrate(step, a, rel ? b * a : b) < rate * dt) lo = a;
  }
  return lo + 0.5 * dif;
}

/* rxnparam.c:587-681 (the known-probability and known-chi searches) */
double ora_bindingradiusprob(double rate, double dt, double difc, double b, int rel, double chi, double *probptr) {
  double step, xa, xp, mult[2], err, errold, errbest, abest, pbest, rt, ub, ch;
  int it, k;
  if (rate < 0 || dt < 0 || difc <= 0 || chi > 1) return -1;
  if (chi < 0 && (!probptr || *probptr == 1)) return ora_bindingradius(rate, dt, difc, b, rel);
  if (chi < 0 && probptr && *probptr == 0) return 0;
  if (rate == 0) { if (probptr && *probptr < 0) *probptr = 0; return 0; }
  if (dt == 0) {
    double a, lp;
    if (chi < 0) return -1;
    if (b < 0) a = rate / (4 * O_PI * difc * chi);
    else if (rel && b > 1) a = rate * (1 - 1 / b) / (4 * O_PI * difc * chi);
    else if (rel && b <= 1) return -1;
    else if (b > 0) a = rate * b / (rate + 4 * O_PI * difc * b * chi);
    else return -1;
    lp = (3.18243 * chi - 3.40864 * chi * chi + 0.984385 * chi * chi * chi) / pow(1 - chi, 2.08761);
    if (probptr) *probptr = difc * lp / a * lp / a;
    return a;
  }
  step = sqrt(2 * difc * dt);
  if (chi < 0) {
    double p = *probptr;
    pbest = p;
    xa = abest = step;
    mult[0] = 0.1;
    ub = (b >= 0) ? (rel ? b * xa : b) : -1;
    rt = ora_numrxnrateprob(step, xa, ub, p) / dt;
    err = errbest = (rt / rate - 1.0) * (rt / rate - 1.0);
    for (it = 0; it < 200 && err > 1.0e-6; it++) {
      errold = err;
      xa *= 1.0 + mult[0];
      if (xa < 1.0e-15) xa = 1.0e-15;
      else if (xa > 1.0e15) xa = 1.0e15;
      ub = (b >= 0) ? (rel ? b * xa : b) : -1;
      rt = ora_numrxnrateprob(step, xa, ub, p) / dt;
      err = (rt / rate - 1.0) * (rt / rate - 1.0);
      mult[0] *= (err < errold) ? 1.1 : -0.5;
      if (err < errbest) { errbest = err; abest = xa; }
    }
  } else {
    double x[2], lo[2] = {1.0e-15, 1.0e-15}, hi[2] = {1.0e15, 1.0};
    x[0] = abest = ora_bindingradius(rate, dt, difc, b, rel);
    x[1] = pbest = 1;
    ub = (b >= 0) ? (rel ? b * x[0] : b) : -1;
    ch = (ub >= 0) ? rate / (4 * O_PI * difc * x[0] * ub / (ub - x[0])) : rate / (4 * O_PI * difc * x[0]);
    if (ch > chi) {
      mult[0] = mult[1] = 0.1;
      x[0] = abest = step;
      x[1] = pbest = 0.5;
      rt = ora_numrxnrateprob(step, x[0], rel ? b * x[0] : b, x[1]) / dt;
      ub = (b >= 0) ? (rel ? b * x[0] : b) : -1;
      ch = (ub >= 0) ? rate / (4 * O_PI * difc * x[0] * ub / (ub - x[0])) : rate / (4 * O_PI * difc * x[0]);
      err = errbest = (rt / rate - 1.0) * (rt / rate - 1.0) + (ch / chi - 1.0) * (ch / chi - 1.0);
      for (it = 0; it < 300 && err > 1.0e-6; it++)
        for (k = 0; k < 2; k++) {
          errold = err;
          x[k] *= 1.0 + mult[k];
          if (x[k] < lo[k]) x[k] = lo[k];
          else if (x[k] > hi[k]) x[k] = hi[k];
          rt = ora_numrxnrateprob(step, x[0], rel ? b * x[0] : b, x[1]) / dt;
          ub = (b >= 0) ? (rel ? b * x[0] : b) : -1;
          ch = (ub >= 0) ? rate / (4 * O_PI * difc * x[0] * ub / (ub - x[0])) : rate / (4 * O_PI * difc * x[0]);
          err = (rt / rate - 1.0) * (rt / rate - 1.0) + (ch / chi - 1.0) * (ch / chi - 1.0);
          mult[k] *= (err < errold) ? 1.1 : -0.5;
          if (err < errbest) { errbest = err; abest = x[0]; pbest = x[1]; }
        }
    }
  }
  xp = pbest;
  if (chi >= 0 && probptr) *probptr = xp;
  return abest;
}

/* rxnparam.c:690-716 */
double ora_unbindingradius(double pgem, double dt, double difc, double a) {
  double b, lo, dif, step, ki, kmax;
  int n;
  if (pgem <= 0 || pgem >= 1 || difc <= 0 || a <= 0 || dt < 0) return -2;
  if (dt == 0) return a / pgem;
  step = sqrt(2.0 * difc * dt);
  ki = ora_numrxnrate(step, a, -1);
  kmax = ora_numrxnrate(step, a, 0);
  if (1.0 - ki / kmax < pgem) return ki / kmax - 1.0;
  lo = 0;
  b = a;
  while (1.0 - ki / ora_numrxnrate(step, a, b) > pgem) { lo = b; b *= 2.0; }
  dif = b - lo;
  for (n = 0; n < 15; n++) {
    dif *= 0.5;
    b = lo + dif;
    if (1.0 - ki / ora_numrxnrate(step, a, b) > pgem) lo = b;
  }
  return lo + 0.5 * dif;
}
