// Host-side parameter derivation and text configuration reader.
#include "sim.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "rxnparam.cuh"
#include "panelgeom.cuh"

namespace smolb {

// host copies of the radius tables (generated from the reference's rxnparam.c)
namespace rxnp {
const double h_yi[SMOLB_TAB_YI_LEN] = SMOLB_TAB_YI_INIT;
const double h_yr[SMOLB_TAB_YR_LEN] = SMOLB_TAB_YR_INIT;
const double h_yb[SMOLB_TAB_YB_LEN] = SMOLB_TAB_YB_INIT;
const double h_kirr[SMOLB_TAB_KIRR_LEN] = SMOLB_TAB_KIRR_INIT;
const double h_krev[SMOLB_TAB_KREV_LEN] = SMOLB_TAB_KREV_INIT;
const double h_kb[SMOLB_TAB_KB_LEN] = SMOLB_TAB_KB_INIT;
}  // namespace rxnp

// RevParam values (smoldyn.h:358)
enum {
  RP_none, RP_irrev, RP_confspread, RP_bounce, RP_pgem, RP_pgemmax, RP_pgemmaxw, RP_ratio,
  RP_unbindrad, RP_pgem2, RP_pgemmax2, RP_ratio2, RP_offset, RP_fixed
};

Sim::Sim() {
  species.push_back(SpeciesDef{"empty"});
}

int Sim::species_index(const std::string &name) const {
  for (size_t i = 1; i < species.size(); ++i)
    if (species[i].name == name) return (int)i;
  return -1;
}

int Sim::compartment_index(const std::string &name) const {
  for (size_t c = 0; c < cmpts.size(); ++c)
    if (cmpts[c].name == name) return (int)c;
  return -1;
}

int Sim::reaction_index(const std::string &name, int *order) const {
  for (int o = 0; o < 3; ++o)
    for (size_t r = 0; r < rxn[o].size(); ++r)
      if (rxn[o][r].name == name) {
        if (order) *order = o;
        return (int)r;
      }
  return -1;
}

// The placement stream starts at a hash of the seed: a start proportional to
// the seed would make seed k+1's stream seed k's shifted by one number, so
// neighbouring seeds would place molecules almost identically.
void Sim::set_seed(long long s) {
  seed = s;
  uint64_t z = (uint64_t)s + 0x2545F4914F6CDD1Dull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  host_rng = z ^ (z >> 31);
}

double Sim::rand_u01() {
  // SplitMix64 stream for host-side placement of initial molecules
  uint64_t z = (host_rng += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (z >> 11) * (1.0 / 9007199254740992.0);
}

static bool same_set2(int a0, int a1, int b0, int b1) {
  return (a0 == b0 && a1 == b1) || (a0 == b1 && a1 == b0);
}

// findreverserxn (smolreact.c:345-381): rev=1 when a reaction of order nprod
// consumes exactly this reaction's products (species and states: the
// reaction's permit for the product states) and makes its reactants; rev=2
// when the products only react onward.
static bool same_set_st(int a1, int s1, int a2, int s2, int b1, int t1, int b2, int t2) {
  return (a1 == b1 && s1 == t1 && a2 == b2 && s2 == t2) || (a1 == b2 && s1 == t2 && a2 == b1 && s2 == t1);
}
static int find_reverse(const Sim &s, int order, int r, int *o2, int *r2) {
  const RxnDef &x = s.rxn[order][r];
  *o2 = 0;
  *r2 = 0;
  if (order == 0 || x.nprod == 0 || x.nprod >= 3) return 0;
  const int orr = x.nprod;
  if (s.rxn[orr].empty()) return 0;
  *o2 = orr;
  int rev = 0;
  for (size_t k = 0; k < s.rxn[orr].size(); ++k) {
    const RxnDef &y = s.rxn[orr][k];
    const bool rct_match =
        (orr == 1) ? (y.rct[0] == x.prd[0] && y.rstate[0] == x.pstate[0])
                   : same_set_st(y.rct[0], y.rstate[0], y.rct[1], y.rstate[1], x.prd[0], x.pstate[0], x.prd[1],
                                 x.pstate[1]);
    if (!rct_match) continue;
    if (rev != 1 && y.nprod == order) {
      const bool back =
          (order == 1) ? (y.prd[0] == x.rct[0] && y.pstate[0] == x.rstate[0])
                       : same_set_st(y.prd[0], y.pstate[0], y.prd[1], y.pstate[1], x.rct[0], x.rstate[0], x.rct[1],
                                     x.rstate[1]);
      if (back) {
        rev = 1;
        *r2 = (int)k;
      }
    }
    if (!rev) {
      rev = 2;
      *r2 = (int)k;
    }
  }
  return rev;
}

static double system_volume(const Sim &s) {
  double v = 1;
  for (int d = 0; d < s.dim; ++d) v *= s.hi[d] - s.lo[d];
  return v;
}

// rxnsetrate (smolreact.c:1307-1414) for every reaction, then rxnsetproduct
// (smolreact.c:1431-1577), in the reference's order.
int derive_reaction_params(Sim &sim, std::string *err) {
  const double dt = sim.dt;
  // order 0
  for (RxnDef &x : sim.rxn[0]) {
    if (x.disabled) { x.prob = 0; continue; }
    if (x.rate < 0) { if (err) *err = "reaction " + x.name + " rate is undefined"; return -8; }
    // births per step: rate x dt x the compartment's volume, the surface's
    // area or the system's volume (smolreact.c:1325-1330)
    x.prob = x.rate * dt * (x.cmpt >= 0 ? compartment_volume(sim, x.cmpt)
                            : x.srf >= 0 ? surface_area(sim, x.srf) : system_volume(sim));
  }
  // order 1
  for (size_t r = 0; r < sim.rxn[1].size(); ++r) {
    RxnDef &x = sim.rxn[1][r];
    if (x.disabled) { x.prob = 0; }
    else if (x.rate < 0) { if (err) *err = "reaction " + x.name + " rate is undefined"; return -8; }
    else if (x.rate == 0) x.prob = 0;
    else {
      // the reactions of the same reactant species and state compete
      const int i = x.rct[0], st = x.rstate[0];
      double sum = 0;
      for (const RxnDef &y : sim.rxn[1])
        if (y.rct[0] == i && y.rstate[0] == st && y.rate > 0) sum += y.rate;
      x.prob = x.rate / sum * (1.0 - std::exp(-sum * dt));
      double product = 1.0;
      for (size_t k = 0; k < r; ++k) {
        const RxnDef &y = sim.rxn[1][k];
        if (y.rct[0] != i || y.rstate[0] != st) continue;
        const double pr = y.prob * product;
        product *= 1.0 - pr;
      }
      x.prob /= product;
      if (!(x.prob >= 0 && x.prob <= 1)) {
        if (err) *err = "reaction " + x.name + " probability out of range";
        return -8;
      }
    }
    int o2, r2;
    const int rev = find_reverse(sim, 1, (int)r, &o2, &r2);
    if (rev > 0 && o2 == 2 && x.rparamt == RP_none) {
      x.rparamt = RP_pgemmaxw;
      x.rparam = 0.2;
    }
  }
  // order 2
  for (size_t r = 0; r < sim.rxn[2].size(); ++r) {
    RxnDef &x = sim.rxn[2][r];
    const int i1 = x.rct[0], i2 = x.rct[1];
    if (x.disabled) { x.prob = 0; x.bindrad2 = 0; continue; }
    if (x.rparamt == RP_confspread) {  // smolreact.c:1321-1323: probability from the rate, radius as given
      if (x.rate < 0) { if (err) *err = "reaction " + x.name + " rate is undefined"; return -8; }
      x.prob = 1.0 - std::exp(-dt * x.rate);
      x.bindrad2 = x.bindrad_user >= 0 ? x.bindrad_user * x.bindrad_user : -1;
      continue;
    }
    if (x.rate < 0) {
      // rate undefined: a user binding radius (binding_radius statement) stands
      if (x.prob_user >= 0) x.prob = x.prob_user;
      else x.prob = 1;
      if (x.bindrad_user >= 0) { x.bindrad2 = x.bindrad_user * x.bindrad_user; continue; }
      if (err) *err = "reaction rate " + x.name + " is undefined";
      return -8;
    }
    // a bound reactant: the rate doubles (one surface, one solution reactant)
    // and its state's diffusion coefficient counts (smolreact.c:1371-1374)
    const int s1 = x.rstate[0], s2 = x.rstate[1];
    double rate3 = x.rate;
    if (i1 == i2) rate3 *= 2;
    if ((s1 == 0) != (s2 == 0)) rate3 *= 2;
    const double dsum = (s1 ? sim.species[i1].difc_bound[s1 - 1] : sim.species[i1].difc) +
                        (s2 ? sim.species[i2].difc_bound[s2 - 1] : sim.species[i2].difc);
    int o2 = 0, r2 = 0;
    const int rev = find_reverse(sim, 2, (int)r, &o2, &r2);
    if (rev > 0 && o2 == 2 && x.rparamt == RP_none) {
      x.rparamt = RP_pgemmaxw;
      x.rparam = 0.2;
    }
    int rpt = RP_none;
    double rpar = 0;
    if (rev == 1) {
      RxnDef &rv = sim.rxn[o2][r2];
      if (rv.rparamt == RP_none) {
        rv.rparamt = RP_pgemmaxw;
        rv.rparam = 0.2;
      }
      rpt = rv.rparamt;
      rpar = rv.rparam;
    }
    double prob = (x.prob_user >= 0) ? x.prob_user : -1;
    if (prob < 0) prob = 1;
    double a;
    if (rate3 <= 0) a = 0;
    else if (dsum <= 0) { if (err) *err = "Both diffusion coefficients are 0"; return -8; }
    else if (rpt == RP_unbindrad) a = rxnp::bindingradiusprob(rate3, dt, dsum, rpar, 0, x.chi, &prob);
    else if (rpt == RP_ratio) a = rxnp::bindingradiusprob(rate3, dt, dsum, rpar, 1, x.chi, &prob);
    else if (rpt == RP_pgem) a = rxnp::bindingradiusprob(rate3 * (1.0 - rpar), dt, dsum, -1, 0, x.chi, &prob);
    else if (rpt == RP_pgemmax || rpt == RP_pgemmaxw) {
      a = rxnp::bindingradiusprob(rate3, dt, dsum, 0, 0, x.chi, &prob);
      const double ub = rxnp::unbindingradius(rpar, dt, dsum, a);
      if (ub > 0) a = rxnp::bindingradiusprob(rate3 * (1.0 - rpar), dt, dsum, -1, 0, x.chi, &prob);
    } else {
      a = rxnp::bindingradiusprob(rate3, dt, dsum, -1, 0, x.chi, &prob);
    }
    x.prob = prob;
    if (x.bindrad_user >= 0) a = x.bindrad_user;
    x.bindrad2 = a * a;
  }
  // products
  for (int order = 0; order < 3; ++order)
    for (size_t r = 0; r < sim.rxn[order].size(); ++r) {
      RxnDef &x = sim.rxn[order][r];
      const int dim = sim.dim;
      for (int q = 0; q < kMaxProd; ++q)
        for (int d = 0; d < 3; ++d) x.prdpos[q][d] = 0;
      const int np = x.nprod;
      const int rpt = x.rparamt;
      double rpar = x.rparam;
      if (np == 0) {
        if (rpt == RP_none || rpt == RP_irrev || rpt == RP_confspread) x.unbindrad = 0;
        else { if (err) *err = "Illegal product parameter because reaction has no products"; return -8; }
      } else if (rpt == RP_offset || rpt == RP_fixed) {
        for (int q = 0; q < np; ++q)
          for (int d = 0; d < dim; ++d) x.prdpos[q][d] = x.user_prdpos[q][d];
        double dist = 0;
        if (np == 1) for (int d = 0; d < dim; ++d) dist = x.prdpos[0][d];
        else for (int d = 0; d < dim; ++d) dist += x.prdpos[0][d] - x.prdpos[1][d];
        x.unbindrad = std::sqrt(dist);
      } else if (np == 1) {
        if (rpt == RP_none || rpt == RP_irrev || rpt == RP_confspread) x.unbindrad = 0;
        else { if (err) *err = "Illegal product parameter because reaction only has one product"; return -8; }
      } else if (rpt == RP_bounce) {  // smolreact.c rxnsetproduct, bounce: split by the reactants' D
        if (order != 2) { if (err) *err = "bounce product placement needs a bimolecular reaction"; return -8; }
        if (rpar == -2) {
          if (err) *err = "bounce with ballistic reflection (parameter -2) is not supported by the GPU engine";
          return -8;
        }
        double dc1 = sim.species[x.rct[0]].difc, dc2 = sim.species[x.rct[1]].difc;
        const double dsum = dc1 + dc2;
        if (dsum == 0) dc1 = dc2 = 0.5;
        else { dc1 /= dsum; dc2 /= dsum; }
        const double len = rpar >= 0 ? rpar : (x.bindrad2 > 0 ? std::sqrt(x.bindrad2) : 0.0);
        x.unbindrad = rpar;
        x.prdpos[0][0] = len * dc1;
        x.prdpos[1][0] = len * dc2;
      } else {
        // the products' diffusion coefficients in their states (MolCalcDifcSum;
        // bsoln counts as solution)
        auto pdifc = [&](int q) {
          const int st = x.pstate[q];
          return (st == 1 || st == 2) ? sim.species[x.prd[q]].difc_bound[st - 1] : sim.species[x.prd[q]].difc;
        };
        double dc1 = pdifc(0), dc2 = pdifc(1);
        const double dsum = dc1 + dc2;
        if (dsum == 0) dc1 = dc2 = 0.5;
        else { dc1 /= dsum; dc2 /= dsum; }
        int o2, r2;
        const int rev = find_reverse(sim, order, (int)r, &o2, &r2);
        if (rpt == RP_irrev || rpt == RP_confspread) {
          x.unbindrad = 0;
        } else if (rev == 0) {
          if (rpt == RP_pgem || rpt == RP_pgemmax || rpt == RP_pgemmaxw || rpt == RP_ratio ||
              rpt == RP_pgem2 || rpt == RP_pgemmax2 || rpt == RP_ratio2) {
            if (err) *err = "Illegal product parameter because products don't react";
            return -8;
          } else if (rpt == RP_unbindrad) {
            x.unbindrad = rpar;
            x.prdpos[0][0] = rpar * dc1;
            x.prdpos[1][0] = -rpar * dc2;
          } else {
            x.unbindrad = 0;
          }
        } else {
          const RxnDef &rv = sim.rxn[o2][r2];
          const double bindradr = (rv.bindrad2 >= 0) ? std::sqrt(rv.bindrad2) : -1;
          if (rpt == RP_none) { if (err) *err = "Undefined product placement for reversible reaction"; return -8; }
          else if (rpt == RP_unbindrad) {
            x.unbindrad = rpar;
            x.prdpos[0][0] = rpar * dc1;
            x.prdpos[1][0] = -rpar * dc2;
          } else if (rv.bindrad2 < 0) {
            if (err) *err = "Binding radius of reaction products is undefined";
            return -8;
          } else if (rv.bindrad2 == 0) {
            x.unbindrad = 0;
          } else if (rpt == RP_ratio || rpt == RP_ratio2) {
            x.unbindrad = rpar * bindradr;
            x.prdpos[0][0] = rpar * bindradr * dc1;
            x.prdpos[1][0] = -rpar * bindradr * dc2;
          } else if (dsum <= 0) {
            if (err) *err = "Cannot set unbinding distance because sum of product diffusion constants is 0";
            return -8;
          } else if (rpt == RP_pgem || rpt == RP_pgem2) {
            rpar = rxnp::unbindingradius(rpar, sim.dt, dsum, bindradr);
            if (rpar == -2) { if (err) *err = "Cannot create an unbinding radius due to illegal input values"; return -8; }
            if (rpar < 0) {
              char buf[128];
              snprintf(buf, sizeof buf, "Maximum possible geminate binding probability is %g", -rpar);
              if (err) *err = buf;
              return -8;
            }
            x.unbindrad = rpar;
            x.prdpos[0][0] = rpar * dc1;
            x.prdpos[1][0] = -rpar * dc2;
          } else if (rpt == RP_pgemmax || rpt == RP_pgemmaxw || rpt == RP_pgemmax2) {
            rpar = rxnp::unbindingradius(rpar, sim.dt, dsum, bindradr);
            if (rpar == -2) { if (err) *err = "Illegal input values"; return -8; }
            if (rpar <= 0) x.unbindrad = 0;
            else {
              x.unbindrad = rpar;
              x.prdpos[0][0] = rpar * dc1;
              x.prdpos[1][0] = -rpar * dc2;
            }
          }
        }
      }
    }
  return 0;
}

// Virtual-box grid: side = ceil(L * (N/molperbox/V)^(1/dim)) (smolboxes.c:717-749),
// widened where needed so that a box is at least one binding radius wide (the
// pair search looks one box deep) and capped at 1023 boxes per dimension.
static void choose_grid(const Sim &s, long long nmol, int ncell[3]) {
  double mpbox = s.molperbox, boxsize = s.boxsize;
  if (mpbox <= 0 && boxsize <= 0) mpbox = s.auto_molperbox > 0 ? s.auto_molperbox : 4;
  double f;
  if (mpbox > 0) f = std::pow((double)nmol / mpbox / system_volume(s), 1.0 / s.dim);
  else f = 1.0 / boxsize;
  double maxrad = 0;
  for (const RxnDef &x : s.rxn[2])
    if (x.bindrad2 > 0) maxrad = std::max(maxrad, std::sqrt(x.bindrad2));
  for (int d = 0; d < 3; ++d) {
    if (d >= s.dim) { ncell[d] = 1; continue; }
    const double L = s.hi[d] - s.lo[d];
    int n = (int)std::ceil(L * f);
    if (n < 1) n = 1;
    if (maxrad > 0 && L / n < maxrad) n = std::max(1, (int)std::floor(L / maxrad));
    if (n > 1023) n = 1023;
    ncell[d] = n;
  }
}

// Effective rate constant implied by the derived parameters (rxncalcrate,
// smolreact.c:1592-1680): order 0 from the
// births per step, order 1 from the per-step probabilities of the species'
// list (undoing the correction for earlier reactions), order 2 from the
// tabulated per-step rate at the binding radius (with the reverse products'
// separation when the reverse reaction places them apart).  *pgem, when not
// null, gets the geminate recombination probability of a reaction with two
// products and a reverse (1 - ki/kr at the unbinding separation), else -1.
double calc_rate(const Sim &sim, int order, int r, double *pgem) {
  if (order < 0 || order > 2 || r < 0 || r >= (int)sim.rxn[order].size()) return -1;
  const RxnDef &x = sim.rxn[order][r];
  const double dt = sim.dt;
  double ans = 0;
  if (order == 0) {
    const double vol = x.cmpt >= 0 ? (x.cmpt < (int)sim.cmpts.size() ? sim.cmpts[x.cmpt].volume : 0)
                       : x.srf >= 0 ? surface_area(sim, x.srf) : system_volume(sim);
    ans = x.prob < 0 || !(vol > 0) ? 0 : x.prob / dt / vol;
  } else if (order == 1) {
    if (x.prob > 0) {
      const int i1 = x.rct[0];
      double probthis = 0, product = 1.0, sum = 0;
      for (const RxnDef &y : sim.rxn[1]) {  // the reactions of this species in this state
        if (y.rct[0] != i1 || y.rstate[0] != x.rstate[0] || !(y.prob > 0)) continue;
        const double pr = y.prob * product;
        if (&y == &x) probthis = pr;
        sum += pr;
        product *= 1.0 - pr;
      }
      ans = -std::log(1.0 - sum) / dt * probthis / sum;
    }
  } else {
    if (x.bindrad2 < 0 || x.prob < 0) {
      ans = 0;
    } else if (x.rparamt == RP_confspread) {
      ans = -std::log(1.0 - x.prob) / dt;
    } else {
      const int i1 = x.rct[0], i2 = x.rct[1];
      const int s1 = x.rstate[0], s2 = x.rstate[1];
      const double dsum = (s1 ? sim.species[i1].difc_bound[s1 - 1] : sim.species[i1].difc) +
                          (s2 ? sim.species[i2].difc_bound[s2 - 1] : sim.species[i2].difc);
      const double step = std::sqrt(2.0 * dsum * dt);
      const double a = std::sqrt(x.bindrad2);
      int o2 = 0, r2 = 0;
      const int rev = find_reverse(sim, 2, r, &o2, &r2);
      const int rpt = rev == 1 ? sim.rxn[o2][r2].rparamt : RP_none;
      if (rpt == RP_pgem || rpt == RP_pgemmax || rpt == RP_pgemmaxw || rpt == RP_ratio || rpt == RP_unbindrad) {
        const RxnDef &rv = sim.rxn[o2][r2];
        double b2 = 0;
        for (int d = 0; d < sim.dim; ++d) {
          const double v = rv.prdpos[0][d] - rv.prdpos[1][d];
          b2 += v * v;
        }
        ans = rxnp::numrxnrateprob(step, a, std::sqrt(b2), x.prob) / dt;
      } else {
        ans = rxnp::numrxnrateprob(step, a, -1, x.prob) / dt;
      }
      if (i1 == i2) ans /= 2.0;
      if (s1 != 0 || s2 != 0) ans /= 2.0;  // one surface-bound reactant
    }
  }
  if (pgem) {
    int o2 = 0, r2 = 0;
    if (x.nprod != 2 || find_reverse(sim, order, r, &o2, &r2) == 0) {
      *pgem = -1;
    } else {
      auto pdifc = [&](int q) {
        const int st = x.pstate[q];
        return (st == 1 || st == 2) ? sim.species[x.prd[q]].difc_bound[st - 1] : sim.species[x.prd[q]].difc;
      };
      const double step = std::sqrt(2.0 * (pdifc(0) + pdifc(1)) * dt);
      double b2 = 0;
      for (int d = 0; d < sim.dim; ++d) {
        const double v = x.prdpos[0][d] - x.prdpos[1][d];
        b2 += v * v;
      }
      const RxnDef &rv = sim.rxn[o2][r2];
      const double a = std::sqrt(rv.bindrad2);
      *pgem = 1.0 - rxnp::numrxnrateprob(step, a, -1, rv.prob) / rxnp::numrxnrateprob(step, a, std::sqrt(b2), rv.prob);
    }
  }
  return ans;
}

void set_species_difm(Sim &sim, int sp, const double *m) {
  SpeciesDef &x = sim.species[sp];
  const int dim = sim.dim;
  x.has_difm = true;
  for (int k = 0; k < 9; ++k) x.difm[k] = 0;
  for (int r = 0; r < dim; ++r)
    for (int c = 0; c < dim; ++c) x.difm[3 * r + c] = m[dim * r + c];
  double tr = 0;  // trace(M*M), as molsetdifm computes it
  for (int r = 0; r < dim; ++r)
    for (int c = 0; c < dim; ++c) tr += x.difm[3 * r + c] * x.difm[3 * c + r];
  x.difc = tr / dim;
}

// ---- compartments ----------------------------------------------------------
namespace {
// Index of each surface's first panel in the engine's panel list (surfaces in
// order, their panels in order).
std::vector<int> surface_panel_base(const Sim &sim) {
  std::vector<int> first(sim.surfaces.size());
  int n = 0;
  for (size_t k = 0; k < sim.surfaces.size(); ++k) {
    first[k] = n;
    n += (int)sim.surfaces[k].panels.size();
  }
  return first;
}

CmptSpec cmpt_spec(const Sim &sim, const CompartDef &c, const std::vector<int> &first) {
  CmptSpec cs;
  cs.pts = c.pts;
  for (int sidx : c.surfaces)
    for (size_t q = 0; q < sim.surfaces[sidx].panels.size(); ++q) {
      const int pi = first[sidx] + (int)q;
      if (pi < 32) cs.panel_mask |= 1u << pi;
    }
  cs.logic = c.logic;
  return cs;
}

// Panels and compartments in device form for host-side membership tests.
struct CmptTester {
  std::vector<DevPanel> panels;
  std::vector<DevCmpt> cmpts;
  double lo[3] = {0, 0, 0};
  explicit CmptTester(const Sim &sim) {
    for (int d = 0; d < 3; ++d) lo[d] = d < sim.dim ? sim.lo[d] : 0.0;
    for (const SurfaceDef &sf : sim.surfaces)
      for (const PanelSpec &ps : sf.panels) panels.push_back(make_dev_panel(ps, lo));
    panels.resize(std::max<size_t>(panels.size(), 1));
    const std::vector<int> first = surface_panel_base(sim);
    for (const CompartDef &c : sim.cmpts) cmpts.push_back(make_dev_cmpt(cmpt_spec(sim, c, first), lo));
  }
  bool inside(int c, const double xa[3]) const {
    const double x[3] = {xa[0] - lo[0], xa[1] - lo[1], xa[2] - lo[2]};
    return pos_in_cmpt(cmpts.data(), c, panels.data(), x);
  }
};

double sys_volume(const Sim &s) {
  double v = 1;
  for (int d = 0; d < s.dim; ++d) v *= s.hi[d] - s.lo[d];
  return v;
}
}  // namespace

bool pos_in_compartment(const Sim &sim, int c, const double x[3]) {
  if (c < 0 || c >= (int)sim.cmpts.size()) return false;
  return CmptTester(sim).inside(c, x);
}

void invalidate_compartments(Sim &sim) {
  for (CompartDef &c : sim.cmpts) c.volume = -1;
}

// The reference estimates the volume from 100 random points per box
// (compartupdatebox, smolcomparts.c:700-760); here 2^18 uniform points over
// the whole system, from a fixed-seed generator so that the derived rates do
// not depend on the simulation's random stream.
double compartment_volume(Sim &sim, int c) {
  if (c < 0 || c >= (int)sim.cmpts.size()) return 0;
  CompartDef &cd = sim.cmpts[c];
  if (cd.volume >= 0) return cd.volume;
  const CmptTester t(sim);
  uint64_t st = 0x9E3779B97F4A7C15ull ^ (uint64_t)(c + 1) * 0xD1B54A32D192ED03ull;
  auto next = [&st]() {  // splitmix64
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  const int n = 1 << 18;
  int in = 0;
  for (int k = 0; k < n; ++k) {
    double x[3] = {0, 0, 0};
    for (int d = 0; d < sim.dim; ++d)
      x[d] = sim.lo[d] + ((double)(next() >> 11) + 0.5) * (1.0 / 9007199254740992.0) * (sim.hi[d] - sim.lo[d]);
    if (t.inside(c, x)) ++in;
  }
  cd.volume = sys_volume(sim) * (double)in / (double)n;
  return cd.volume;
}

namespace {
void random_pos_with(Sim &sim, const CmptTester &t, int c, double x[3]) {
  for (int k = 0; k < 10000; ++k) {
    for (int d = 0; d < 3; ++d) x[d] = d < sim.dim ? sim.lo[d] + sim.rand_u01() * (sim.hi[d] - sim.lo[d]) : 0.0;
    if (t.inside(c, x)) return;
  }
  const CompartDef &cd = sim.cmpts[c];
  if (cd.pts.empty()) return;
  const size_t k = std::min(cd.pts.size() - 1, (size_t)(sim.rand_u01() * cd.pts.size()));
  for (int d = 0; d < 3; ++d) x[d] = d < (int)cd.pts[k].size() ? cd.pts[k][d] : 0.0;
}
}  // namespace

void compartment_random_pos(Sim &sim, int c, double x[3]) { random_pos_with(sim, CmptTester(sim), c, x); }

void compartment_random_positions(Sim &sim, int c, long long n, std::vector<double> *out) {
  const CmptTester t(sim);  // built once for all n positions
  for (long long k = 0; k < n; ++k) {
    double x[3];
    random_pos_with(sim, t, c, x);
    for (int d = 0; d < 3; ++d) out->push_back(x[d]);
  }
}

int build_engine_specs(Sim &sim, NetSpec *net, RepSpec *rep, std::string *err) {
  *net = NetSpec();
  *rep = RepSpec();
  if ((int)sim.species.size() > kMaxSpecies) { if (err) *err = "too many species (max 31)"; return -6; }
  net->nspecies = (int)sim.species.size();
  net->gauss_table_size = sim.gauss_table_size;
  for (int o = 0; o < 3; ++o) {
    if ((int)sim.rxn[o].size() > kMaxRxn) { if (err) *err = "too many reactions of one order (max 16)"; return -6; }
    net->nrxn[o] = (int)sim.rxn[o].size();
    for (size_t r = 0; r < sim.rxn[o].size(); ++r) {
      const RxnDef &x = sim.rxn[o][r];
      net->rct[o][r][0] = x.rct[0];
      net->rct[o][r][1] = x.rct[1];
      net->nprod[o][r] = x.nprod;
      for (int q = 0; q < x.nprod; ++q) net->prd[o][r][q] = x.prd[q];
      net->fixed_placement[o][r] = (x.rparamt == RP_fixed) ? 1 : 0;
      if (o == 0)
        for (int q = 0; q < kMaxProd; ++q) net->pstate0[r][q] = q < x.nprod ? x.pstate[q] : 0;
      if (o == 1) {
        net->rstate1[r] = x.rstate[0];
        for (int q = 0; q < 2; ++q) net->pstate1[r][q] = q < x.nprod ? x.pstate[q] : 0;
        if (x.rstate[0] && (x.rparamt == RP_confspread || x.rparamt == RP_bounce || x.rparamt == RP_fixed ||
                            x.rparamt == RP_offset)) {
          if (err) *err = "reaction " + x.name + ": confspread, bounce, offset and fixed are not built for surface-bound reactants";
          return -7;
        }
      }
      if (o == 2) {
        net->rstate2[r][0] = x.rstate[0];
        net->rstate2[r][1] = x.rstate[1];
        net->pstate2[r] = x.nprod ? x.pstate[0] : 0;
        if ((x.rstate[0] || x.rstate[1]) && (x.rparamt == RP_confspread || x.rparamt == RP_bounce ||
                                              x.rparamt == RP_fixed || x.rparamt == RP_offset)) {
          if (err) *err = "reaction " + x.name + ": confspread, bounce, offset and fixed are not built for surface-bound reactants";
          return -7;
        }
      }
      if (o == 2) {
        net->placement2[r] = x.rparamt == RP_confspread ? 1 : x.rparamt == RP_bounce ? 2 : 0;
        net->bounce_k[r] = x.rparam >= 0 ? 1.0 : 2.0;
      }
      for (int q = 0; q < x.nprod; ++q)
        for (int d = 0; d < 3; ++d) rep->prdpos[o][r][q][d] = x.prdpos[q][d];
      net->cmpt[o][r] = x.cmpt >= 0 ? x.cmpt + 1 : 0;
      net->rsrf[o][r] = x.srf >= 0 ? x.srf + 1 : 0;
      if (o == 0) rep->birth_mean[r] = x.prob;
      if (o == 1) rep->uni_prob[r] = x.prob;
      if (o == 2) {
        rep->bind2[r] = std::max(0.0, x.bindrad2);
        rep->pair_prob[r] = x.prob;
      }
    }
  }
  rep->dim = sim.dim;
  const bool surfaces = !sim.surfaces.empty();
  for (int d = 0; d < 3; ++d) {
    rep->lo[d] = (d < sim.dim) ? sim.lo[d] : 0;
    rep->hi[d] = (d < sim.dim) ? sim.hi[d] : 1;
    for (int side = 0; side < 2; ++side) {
      const char t = sim.btype[d][side];
      uint8_t k = kWallTransparent;
      if (!surfaces) {  // walls are transparent once surfaces exist (smolwall.c:328, 374)
        if (t == 'r') k = kWallReflect;
        else if (t == 'p') k = kWallPeriodic;
        else if (t == 'a') k = kWallAbsorb;
      }
      rep->wall[2 * d + side] = (d < sim.dim) ? k : kWallTransparent;
    }
  }
  for (size_t i = 0; i < sim.species.size(); ++i) {
    rep->difc[i] = sim.species[i].difc;
    rep->has_difm[i] = sim.species[i].has_difm;
    for (int k = 0; k < 9; ++k) rep->difm[i][k] = sim.species[i].difm[k];
    for (int d = 0; d < 3; ++d) rep->drift[i][d] = (d < sim.dim) ? sim.species[i].drift[d] : 0;
  }
  choose_grid(sim, (long long)sim.pend_sp.size(), rep->ncell);
  const std::vector<int> base = surface_panel_base(sim);
  for (size_t si = 0; si < sim.surfaces.size(); ++si) {
    const SurfaceDef &sf = sim.surfaces[si];
    for (size_t q = 0; q < sf.panels.size(); ++q) {
      PanelSpec ps = sf.panels[q];
      ps.jump_front_mask = sf.jump_front;
      ps.jump_back_mask = sf.jump_back;
      for (int f = 0; f < 2; ++f) ps.jump_pnl[f] = ps.jump_face[f] = -1;
      for (const std::array<int, 4> &j : sf.jumps)
        if (j[0] == (int)q) {
          ps.jump_pnl[j[1]] = base[si] + j[2];
          ps.jump_face[j[1]] = j[3];
        }
      ps.action_front = sf.act_front;
      ps.action_back = sf.act_back;
      ps.absorb_front_mask = sf.absorb_front;
      ps.absorb_back_mask = sf.absorb_back;
      ps.trans_front_mask = sf.trans_front;
      ps.trans_back_mask = sf.trans_back;
      ps.refl_front_mask = sf.refl_front;
      ps.refl_back_mask = sf.refl_back;
      if (net->panels.size() < (size_t)kMaxPanels) net->panel_area[net->panels.size()] = panel_area_dim(ps, sim.dim);
      net->panels.push_back(ps);
    }
  }
  const std::vector<int> first = surface_panel_base(sim);
  for (const CompartDef &c : sim.cmpts) net->cmpts.push_back(cmpt_spec(sim, c, first));
  int rc = derive_surface_params(sim, err);
  if (!rc) rc = build_surface_rules(sim, net, err);
  return rc;
}

// ---------------------------------------------------------------------------
// Text configuration reader (subset of smolsim.cpp:626-2270 simreadstring).

static std::vector<std::string> split_ws(const std::string &s) {
  std::vector<std::string> out;
  std::istringstream is(s);
  std::string w;
  while (is >> w) out.push_back(w);
  return out;
}

static bool parse_double(const std::string &s, double *v) {
  char *end = nullptr;
  *v = strtod(s.c_str(), &end);
  return end && *end == '\0' && end != s.c_str();
}

static int species_arg(Sim &sim, const std::string &w, std::vector<int> *out) {
  out->clear();
  std::string name = w;
  const size_t paren = name.find('(');
  if (paren != std::string::npos) name = name.substr(0, paren);  // state suffix: soln only
  if (name == "all") {
    for (size_t i = 1; i < sim.species.size(); ++i) out->push_back((int)i);
    return 0;
  }
  const int i = sim.species_index(name);
  if (i < 0) return -3;
  out->push_back(i);
  return 0;
}

// Restrict reaction x to surface sf (rxn->srf: it fires only where a reactant
// is bound to that surface, smolreact.c:3048, :3093, :3116).  Built for
// reactions of a surface-bound reactant; elsewhere refused.
int set_reaction_surface(Sim &sim, RxnDef &x, int sf, std::string *err) {
  (void)sim;
  bool bound = false, bprod = false;
  for (int q = 0; q < x.order; ++q) bound = bound || x.rstate[q] != 0;
  for (int q = 0; q < x.nprod; ++q) bprod = bprod || x.pstate[q] != 0;
  if (sf < 0) {
    if (x.order == 0 && bprod) {
      if (err) *err = "enter a surface for order 0 reactions with surface-bound products";
      return -7;
    }
    x.srf = -1;
    return 0;
  }
  if (!bound && x.order != 0) {
    if (err) *err = "reaction " + x.name + ": a surface restriction is built for order 0 reactions and reactions "
                    "of surface-bound reactants";
    return -7;
  }
  x.srf = sf;
  return 0;
}

// Append a reaction after checking its reactant and product states: solution
// reactions, a first-order reaction of a bound reactant with at most two
// products, or a second-order one with one or two bound reactants and at most
// one product (the reactant and product states of doreact,
// smolreact.c:2662-2902, that the engine builds).
int add_reaction_def(Sim &sim, const RxnDef &x, std::string *err) {
  int nbound = 0;
  for (int q = 0; q < x.order; ++q) {
    if (x.rstate[q] < 0 || x.rstate[q] > 2) { if (err) *err = "reactant state not supported by the GPU engine"; return -7; }
    nbound += x.rstate[q] != 0;
  }
  const bool bound = nbound > 0;
  bool bprod = false;
  for (int q = 0; q < x.nprod; ++q) {
    const int st = x.pstate[q];
    if (st < 0 || (st > 2 && st != 5)) { if (err) *err = "product state not supported by the GPU engine"; return -7; }
    bprod = bprod || st != 0;
  }
  if (bound && (x.order == 0 || x.nprod > (x.order == 1 ? 2 : 1))) {
    if (err) *err = "reactions of surface-bound molecules are supported as first order with at most two products, "
                    "or second order with at most one product";
    return -7;
  }
  if (!bound && bprod && !(x.order == 0 && x.srf >= 0)) {
    if (err) *err = "products in surface states need a surface-bound reactant, or a surface for order 0 reactions";
    return -7;
  }
  if ((int)sim.rxn[x.order].size() >= kMaxRxn) { if (err) *err = "too many reactions"; return -6; }
  sim.rxn[x.order].push_back(x);
  return 0;
}

static int add_reaction_from_words(Sim &sim, const std::vector<std::string> &w, std::string *err, int srf = -1) {
  // reaction [name] r1 [+ r2] -> p1 [+ p2 ...] [rate]
  if (w.size() < 3) { if (err) *err = "reaction: too few words"; return -7; }
  size_t k = 0;
  std::string name = w[0];
  size_t arrow = std::find(w.begin(), w.end(), "->") - w.begin();
  bool reversible = false;
  if (arrow == w.size()) {
    arrow = std::find(w.begin(), w.end(), "<->") - w.begin();
    reversible = arrow != w.size();
  }
  if (arrow == w.size()) { if (err) *err = "reaction: missing ->"; return -7; }
  k = 1;
  std::vector<std::string> rct, prd;
  for (size_t j = k; j < arrow; ++j)
    if (w[j] != "+") rct.push_back(w[j]);
  // products run up to the trailing numeric rate(s); a lone "0" means none
  std::vector<double> rates;
  size_t end = w.size();
  while (end > arrow + 1) {
    double v;
    if (!parse_double(w[end - 1], &v) || sim.species_index(w[end - 1]) >= 0 || w[end - 1].find('(') != std::string::npos)
      break;
    if (end - 1 == arrow + 1 && w[end - 1] == "0") break;  // "-> 0" with no rate
    rates.insert(rates.begin(), v);
    --end;
  }
  for (size_t j = arrow + 1; j < end; ++j)
    if (w[j] != "+") prd.push_back(w[j]);
  if (rct.size() == 1 && rct[0] == "0") rct.clear();
  if (prd.size() == 1 && prd[0] == "0") prd.clear();
  if (rct.size() > 2 || prd.size() > (size_t)kMaxProd) { if (err) *err = "reaction: too many reactants or products"; return -7; }
  // species[(state)]: solution unless a state is given (molstring2index1)
  auto split = [&](const std::string &w, int *st) -> int {
    std::string nm = w, sn;
    *st = 0;
    const size_t paren = w.find('(');
    if (paren != std::string::npos) {
      nm = w.substr(0, paren);
      sn = w.substr(paren + 1, w.find(')', paren) - paren - 1);
      if (sn == "front") *st = 1;
      else if (sn == "back") *st = 2;
      else if (sn == "bsoln") *st = 5;
      else if (!(sn == "soln" || sn == "solution" || sn == "fsoln" || sn == "aq")) *st = -1;
    }
    return sim.species_index(nm);
  };
  auto mk = [&](const std::string &nm, const std::vector<std::string> &r, const std::vector<std::string> &p,
                double rate) -> int {
    RxnDef x;
    x.name = nm;
    x.order = (int)r.size();
    for (size_t q = 0; q < r.size(); ++q) {
      int st = 0;
      const int i = split(r[q], &st);
      if (i < 0) { if (err) *err = "unknown species " + r[q]; return -3; }
      if (st < 0 || st == 5) { if (err) *err = "reactant state not supported by the GPU engine: " + r[q]; return -7; }
      x.rct[q] = i;
      x.rstate[q] = st;
    }
    x.nprod = (int)p.size();
    for (size_t q = 0; q < p.size(); ++q) {
      int st = 0;
      const int i = split(p[q], &st);
      if (i < 0) { if (err) *err = "unknown species " + p[q]; return -3; }
      if (st < 0) { if (err) *err = "product state not supported by the GPU engine: " + p[q]; return -7; }
      x.prd[q] = i;
      x.pstate[q] = st;
    }
    x.rate = rate;
    x.srf = srf;
    return add_reaction_def(sim, x, err);
  };
  int rc = mk(reversible ? name + "fwd" : name, rct, prd, rates.empty() ? -1 : rates[0]);
  if (rc) return rc;
  if (reversible) rc = mk(name + "rev", prd, rct, rates.size() > 1 ? rates[1] : -1);
  sim.need_update = sim.need_rebuild = true;
  return rc;
}

static int rp_from_string(const std::string &s) {
  static const char *names[] = {"none", "irrev", "confspread", "bounce", "pgem", "pgemmax", "pgemmaxw",
                                "ratio", "unbindrad", "pgem2", "pgemmax2", "ratio2", "offset", "fixed"};
  static const char *abbr[] = {"", "i", "a", "", "p", "x", "", "r", "b", "q", "y", "s", "o", "f"};
  for (int k = 0; k < 14; ++k)
    if (s == names[k] || (abbr[k][0] && s == abbr[k])) return k;
  return -1;
}

int read_config_statement(Sim &sim, const std::string &word, const std::string &rest, std::string *err) {
  const std::vector<std::string> w = split_ws(rest);
  auto need = [&](size_t n) -> bool {
    if (w.size() < n) { if (err) *err = word + ": missing parameters"; return false; }
    return true;
  };
  double v;
  if (word == "dim") {
    if (!need(1)) return -7;
    sim.dim = atoi(w[0].c_str());
    if (sim.dim < 1 || sim.dim > 3) { if (err) *err = "dim must be 1..3"; return -6; }
  } else if (word == "species" || word == "names") {
    for (const std::string &s : w)
      if (sim.species_index(s) < 0) sim.species.push_back(SpeciesDef{s});
    sim.need_rebuild = true;
  } else if (word == "difc") {
    if (!need(2)) return -7;
    std::vector<int> ids;
    if (species_arg(sim, w[0], &ids)) { if (err) *err = "difc: unknown species " + w[0]; return -3; }
    if (!parse_double(w[1], &v)) { if (err) *err = "difc: bad value"; return -7; }
    if (v < 0) { if (err) *err = "diffusion coefficient needs to be >=0"; return -6; }
    // species[(state)]: the solution state unless one is given (molsetdifc)
    std::string st;
    const size_t paren = w[0].find('(');
    if (paren != std::string::npos) st = w[0].substr(paren + 1, w[0].find(')', paren) - paren - 1);
    const bool soln = st.empty() || st == "solution" || st == "soln" || st == "fsoln" || st == "aq" || st == "all";
    const bool front = st == "front" || st == "all", back = st == "back" || st == "all";
    if (!soln && !front && !back) { if (err) *err = "difc: state not supported by the GPU engine: " + st; return -7; }
    for (int i : ids) {
      if (soln) sim.species[i].difc = v;
      if (front) sim.species[i].difc_bound[0] = v;
      if (back) sim.species[i].difc_bound[1] = v;
    }
    sim.need_update = sim.need_rebuild = true;
  } else if (word == "difm") {  // smolsim.cpp:863: species then dim*dim values
    if (!need(1 + (size_t)sim.dim * sim.dim)) return -7;
    std::vector<int> ids;
    if (species_arg(sim, w[0], &ids)) { if (err) *err = "difm: unknown species " + w[0]; return -3; }
    double m[9];
    for (int k = 0; k < sim.dim * sim.dim; ++k)
      if (!parse_double(w[1 + k], &m[k])) { if (err) *err = "difm: bad value"; return -7; }
    for (int i : ids) set_species_difm(sim, i, m);
    sim.need_update = true;
  } else if (word == "drift") {
    if (!need(1 + (size_t)sim.dim)) return -7;
    std::vector<int> ids;
    if (species_arg(sim, w[0], &ids)) { if (err) *err = "drift: unknown species " + w[0]; return -3; }
    for (int i : ids)
      for (int d = 0; d < sim.dim; ++d) sim.species[i].drift[d] = atof(w[1 + d].c_str());
    sim.need_update = true;
  } else if (word == "boundaries") {
    if (!need(3)) return -7;
    const int d = atoi(w[0].c_str());
    if (d < 0 || d >= 3) { if (err) *err = "boundaries: bad dimension"; return -6; }
    sim.lo[d] = atof(w[1].c_str());
    sim.hi[d] = atof(w[2].c_str());
    const char t = (w.size() > 3) ? w[3][0] : 'r';
    sim.btype[d][0] = sim.btype[d][1] = t;
    sim.need_rebuild = true;
  } else if (word == "low_wall" || word == "high_wall") {
    if (!need(3)) return -7;
    const int d = atoi(w[0].c_str());
    const int side = (word == "high_wall") ? 1 : 0;
    (side ? sim.hi : sim.lo)[d] = atof(w[1].c_str());
    sim.btype[d][side] = w[2][0];
    sim.need_rebuild = true;
  } else if (word == "time_start") {
    if (!need(1)) return -7;
    sim.tstart = sim.time = atof(w[0].c_str());
  } else if (word == "time_stop") {
    if (!need(1)) return -7;
    sim.tstop = atof(w[0].c_str());
  } else if (word == "time_step") {
    if (!need(1)) return -7;
    sim.dt = atof(w[0].c_str());
    sim.need_update = sim.need_rebuild = true;
  } else if (word == "time_now") {
    if (!need(1)) return -7;
    sim.time = atof(w[0].c_str());
  } else if (word == "random_seed") {
    if (!need(1)) return -7;
    sim.set_seed(atoll(w[0].c_str()));
    sim.need_rebuild = true;
  } else if (word == "molperbox") {
    if (!need(1)) return -7;
    sim.molperbox = atof(w[0].c_str());
    sim.boxsize = -1;
    sim.need_rebuild = true;
  } else if (word == "boxsize") {
    if (!need(1)) return -7;
    sim.boxsize = atof(w[0].c_str());
    sim.molperbox = -1;
    sim.need_rebuild = true;
  } else if (word == "accuracy") {
    if (!need(1)) return -7;
    sim.accuracy = atoi(w[0].c_str());
  } else if (word == "gauss_table_size") {
    if (!need(1)) return -7;
    sim.gauss_table_size = atoi(w[0].c_str());
    sim.need_rebuild = true;
  } else if (word == "max_mol") {
    if (!need(1)) return -7;
    sim.max_mol = atoll(w[0].c_str());
    sim.need_rebuild = true;
  } else if (word == "mol" || word == "molecule") {
    if (!need(2)) return -7;
    const long long n = atoll(w[0].c_str());
    const int i = sim.species_index(w[1]);
    if (i < 0) { if (err) *err = "mol: unknown species " + w[1]; return -3; }
    for (long long k = 0; k < n; ++k) {
      for (int d = 0; d < 3; ++d) {
        double x = 0;
        if (d < sim.dim) {
          const std::string &t = (2 + (size_t)d < w.size()) ? w[2 + d] : std::string("u");
          if (t == "u") x = sim.lo[d] + sim.rand_u01() * (sim.hi[d] - sim.lo[d]);
          else {
            const size_t dash = t.find('-', 1);
            if (dash != std::string::npos) {
              const double a = atof(t.substr(0, dash).c_str()), b = atof(t.substr(dash + 1).c_str());
              x = a + sim.rand_u01() * (b - a);
            } else x = atof(t.c_str());
          }
        }
        sim.pend_pos.push_back(x);
      }
      sim.pend_sp.push_back(i);
    }
    sim.need_rebuild = true;
  } else if (word == "surface_mol") {  // smolsim.cpp:1027
    const int rc = read_surface_mol(sim, w, err);
    if (rc) return rc;
  } else if (word == "epsilon" || word == "margin" || word == "neighbor_dist" || word == "neighbour_dist") {
    // surface simulation parameters (smolsurface.c:2060-2093)
    if (!need(1) || !parse_double(w[0], &v)) { if (err) *err = word + ": bad value"; return -7; }
    if (v < 0) { if (err) *err = word + " needs to be >= 0"; return -6; }
    (word == "epsilon" ? sim.srf_epsilon : word == "margin" ? sim.srf_margin : sim.srf_neighdist) = v;
    sim.need_rebuild = true;
  } else if (word == "compartment_mol") {  // smolsim.cpp:1072
    if (!need(3)) return -7;
    const long long n = atoll(w[0].c_str());
    const int i = sim.species_index(w[1]);
    if (i <= 0) { if (err) *err = "compartment_mol: unknown species " + w[1]; return -3; }
    const int c = sim.compartment_index(w[2]);
    if (c < 0) { if (err) *err = "compartment_mol: unknown compartment " + w[2]; return -3; }
    compartment_random_positions(sim, c, n, &sim.pend_pos);
    for (long long k = 0; k < n; ++k) sim.pend_sp.push_back(i);
    sim.need_rebuild = true;
  } else if (word == "reaction" || word == "reaction_cmpt" || word == "reaction_surface") {
    // reaction_cmpt cname ... / reaction_surface sname ... (deprecated forms)
    // or reaction cmpt=cname ... / reaction srf=sname ... (smolreact.c:2436-2490)
    std::vector<std::string> ww = w;
    int c = -1, sf = -1;
    auto surface_index = [&](const std::string &nm) {
      for (size_t k = 0; k < sim.surfaces.size(); ++k)
        if (sim.surfaces[k].name == nm) return (int)k;
      return -1;
    };
    if (word == "reaction_cmpt") {
      if (ww.empty()) { if (err) *err = "reaction_cmpt: missing compartment"; return -7; }
      c = sim.compartment_index(ww[0]);
      if (c < 0) { if (err) *err = "compartment name not recognized"; return -3; }
      ww.erase(ww.begin());
    } else if (word == "reaction_surface") {
      if (ww.empty()) { if (err) *err = "reaction_surface: missing surface"; return -7; }
      sf = surface_index(ww[0]);
      if (sf < 0) { if (err) *err = "surface " + ww[0] + " not recognized"; return -3; }
      ww.erase(ww.begin());
    }
    while (!ww.empty() && ww[0].find('=') != std::string::npos) {
      const std::string key = ww[0].substr(0, ww[0].find('=')), val = ww[0].substr(ww[0].find('=') + 1);
      if (key == "cmpt" || key == "compartment") {
        c = sim.compartment_index(val);
        if (c < 0) { if (err) *err = "compartment name not recognized"; return -3; }
      } else if (key == "srf" || key == "surface") {
        sf = surface_index(val);
        if (sf < 0) { if (err) *err = "surface " + val + " not recognized"; return -3; }
      } else {
        if (err) *err = "reaction restriction not supported by the GPU engine: " + ww[0];
        return -7;
      }
      ww.erase(ww.begin());
    }
    size_t before[3] = {sim.rxn[0].size(), sim.rxn[1].size(), sim.rxn[2].size()};
    const int rc = add_reaction_from_words(sim, ww, err, sf);
    if (rc) return rc;
    for (int o = 0; o < 3; ++o)
      for (size_t r = before[o]; r < sim.rxn[o].size(); ++r) {
        RxnDef &x = sim.rxn[o][r];
        x.cmpt = c;
        if (sf >= 0) {
          if (const int e = set_reaction_surface(sim, x, sf, err)) return e;
        }
      }
    return 0;
  } else if (word == "reaction_rate") {
    if (!need(2)) return -7;
    int o;
    const int r = sim.reaction_index(w[0], &o);
    if (r < 0) { if (err) *err = "reaction_rate: unknown reaction"; return -3; }
    sim.rxn[o][r].rate = atof(w[1].c_str());
    sim.need_update = true;
  } else if (word == "reaction_probability") {
    if (!need(2)) return -7;
    int o;
    const int r = sim.reaction_index(w[0], &o);
    if (r < 0) { if (err) *err = "reaction_probability: unknown reaction"; return -3; }
    const double v = atof(w[1].c_str());
    if (v < 0 || v > 1) { if (err) *err = "probability value must be between 0 and 1"; return -6; }
    sim.rxn[o][r].prob_user = v;
    sim.need_update = true;
  } else if (word == "reaction_chi") {  // smolsim.cpp:1799-1821: order 2 only, 0 < chi < 1 or -1
    if (!need(2)) return -7;
    int o;
    const int r = sim.reaction_index(w[0], &o);
    if (r < 0) { if (err) *err = "reaction_chi: unknown reaction"; return -3; }
    if (o != 2) { if (err) *err = "reaction chi value is only allowed for order 2 reactions"; return -6; }
    const double v = atof(w[1].c_str());
    if (!(v != 0 && v < 1)) { if (err) *err = "reaction chi value must be between 0 and 1 (or -1 to disable)"; return -6; }
    sim.rxn[2][r].chi = v;
    sim.need_update = true;
  } else if (word == "confspread_radius") {  // smolsim.cpp:1736, smolreact.c:1762
    if (!need(2)) return -7;
    int o;
    const int r = sim.reaction_index(w[0], &o);
    if (r < 0 || o != 2) { if (err) *err = "confspread_radius: unknown bimolecular reaction"; return -3; }
    const double v = atof(w[1].c_str());
    if (v < 0) { if (err) *err = "confspread radius value must be non-negative"; return -6; }
    sim.rxn[2][r].rparamt = RP_confspread;
    sim.rxn[2][r].bindrad_user = v;
    sim.need_update = true;
  } else if (word == "binding_radius") {
    if (!need(2)) return -7;
    int o;
    const int r = sim.reaction_index(w[0], &o);
    if (r < 0 || o != 2) { if (err) *err = "binding_radius: unknown bimolecular reaction"; return -3; }
    sim.rxn[2][r].bindrad_user = atof(w[1].c_str());
    sim.need_update = true;
  } else if (word == "product_placement") {
    if (!need(2)) return -7;
    int o;
    const int r = sim.reaction_index(w[0], &o);
    if (r < 0) { if (err) *err = "product_placement: unknown reaction"; return -3; }
    const int rp = rp_from_string(w[1]);
    if (rp < 0) { if (err) *err = "product_placement: unknown type " + w[1]; return -7; }
    RxnDef &x = sim.rxn[o][r];
    if ((x.rstate[0] != 0 || (o == 2 && x.rstate[1] != 0)) &&
        (rp == RP_confspread || rp == RP_bounce || rp == RP_offset || rp == RP_fixed)) {
      if (err) *err = "product_placement: confspread, bounce, offset and fixed are not built for surface-bound reactants";
      return -7;
    }
    x.rparamt = rp;
    x.rparam = (w.size() > 2) ? atof(w[2].c_str()) : 0;
    if ((rp == RP_offset || rp == RP_fixed) && w.size() >= 3 + 1 + (size_t)sim.dim) {
      const int q = sim.species_index(w[2]);
      int slot = -1;
      for (int k = 0; k < x.nprod; ++k)
        if (x.prd[k] == q) { slot = k; break; }
      if (slot >= 0)
        for (int d = 0; d < sim.dim; ++d) x.user_prdpos[slot][d] = atof(w[3 + d].c_str());
    }
    sim.need_update = true;
  } else if (word == "start_surface" || word == "new_surface") {
    SurfaceDef s;
    s.name = w.empty() ? "surf" + std::to_string(sim.surfaces.size()) : w[0];
    bool exists = false;  // a known name continues that surface (surfaddsurface)
    for (const SurfaceDef &x : sim.surfaces) exists = exists || x.name == s.name;
    if (!exists) sim.surfaces.push_back(s);
    sim.need_rebuild = true;
  } else if (word == "output_files") {
    for (const std::string &s : w) sim.outfiles.push_back(s);
  } else if (word == "cmd") {
    if (!need(2)) return -7;
    Command c;
    c.type = w[0][0];
    size_t k = 1;
    if (c.type == 'N' || c.type == 'n') { c.every = atoll(w[1].c_str()); k = 2; }
    else if (c.type == 'i') {
      if (!need(5)) return -7;
      c.on = atof(w[1].c_str()); c.off = atof(w[2].c_str()); c.dt = atof(w[3].c_str());
      k = 4;
    }
    for (; k < w.size(); ++k) c.text += (c.text.empty() ? "" : " ") + w[k];
    sim.cmds.push_back(c);
  } else if (word == "graphics" || word == "graphic_iter" || word == "graphic_delay" || word == "color" ||
             word == "display_size" || word == "text_display" || word == "frame_thickness" ||
             word == "frame_color" || word == "grid_thickness" || word == "background_color" ||
             word == "tiff_name" || word == "tiff_iter" || word == "light" || word == "text_color" ||
             word == "molecule_lists" || word == "mol_list" || word == "quit_at_end" ||
             word == "output_root" || word == "output_format" || word == "output_precision") {
    // display, list-layout and output formatting statements: no effect on the engine
  } else {
    if (err) *err = "unsupported statement: " + word;
    return -7;
  }
  return 0;
}

// surfaddpanel (smolsurface.c:2432-2640): a panel from its shape's
// parameters.  rect: axis "+0".."-2" and corner + extents (dim values, then
// dim-1 extents); sph: centre (dim) and radius (negative: front inside); in 3-D
// also tri: 3 vertices (front by the right-hand rule, Geo_TriNormal); cyl: the
// two axis end points and radius (negative: front inside); hemi: centre,
// radius (sign as sph) and a vector out of the open side; disk: centre, radius
// and front normal.  Trailing drawing parameters (slices, stacks) are ignored.
int make_panel(int dim, int shape, const std::string &axis, const double *prm, int np, PanelSpec *out,
               std::string *err) {
  PanelSpec p{};
  p.shape = shape;
  p.front_sign = 1;
  auto need = [&](int n, const char *what) {
    if (np >= n) return true;
    if (err) *err = std::string("panel ") + what + ": missing parameters";
    return false;
  };
  auto unit = [](double v[3]) {
    const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (!(l > 0)) return false;
    for (int d = 0; d < 3; ++d) v[d] /= l;
    return true;
  };
  if (shape != 0 && shape != 2 && dim != 3) {
    if (err) *err = "panel: tri, cyl, hemi and disk panels need dim 3";
    return -6;
  }
  if (shape == 0) {
    if (axis.size() < 2 || (axis[0] != '+' && axis[0] != '-')) { if (err) *err = "panel rect: bad axis"; return -7; }
    p.front_sign = axis[0] == '-' ? -1 : 1;
    const char ac = axis.back();
    p.axis = (ac >= '0' && ac <= '2') ? ac - '0' : ac - 'x';
    if (p.axis < 0 || p.axis >= dim) { if (err) *err = "panel rect: bad axis"; return -7; }
    if (!need(dim + dim - 1, "rect")) return -7;
    double corner[3] = {0, 0, 0};
    for (int d = 0; d < dim; ++d) corner[d] = prm[d];
    p.pos = corner[p.axis];
    int k = dim;
    for (int d = 0; d < 3; ++d) {
      if (d == p.axis || d >= dim) { p.lo[d] = p.hi[d] = corner[d]; continue; }
      const double ext = prm[k++];
      p.lo[d] = std::min(corner[d], corner[d] + ext);
      p.hi[d] = std::max(corner[d], corner[d] + ext);
    }
  } else if (shape == 2) {
    if (!need(dim + 1, "sph")) return -7;
    for (int d = 0; d < dim; ++d) p.center[d] = prm[d];
    p.radius = prm[dim];
    if (p.radius < 0) { p.radius = -p.radius; p.front_sign = -1; }
  } else if (shape == 1) {
    if (!need(9, "tri")) return -7;
    for (int k = 0; k < 3; ++k)
      for (int d = 0; d < 3; ++d) p.pt[k][d] = prm[3 * k + d];
    const double e1[3] = {p.pt[1][0] - p.pt[0][0], p.pt[1][1] - p.pt[0][1], p.pt[1][2] - p.pt[0][2]};
    const double e2[3] = {p.pt[2][0] - p.pt[1][0], p.pt[2][1] - p.pt[1][1], p.pt[2][2] - p.pt[1][2]};
    p.normal[0] = e1[1] * e2[2] - e1[2] * e2[1];
    p.normal[1] = e1[2] * e2[0] - e1[0] * e2[2];
    p.normal[2] = e1[0] * e2[1] - e1[1] * e2[0];
    if (!unit(p.normal)) { if (err) *err = "panel tri: degenerate triangle"; return -6; }
  } else if (shape == 3) {
    if (!need(7, "cyl")) return -7;
    for (int k = 0; k < 2; ++k)
      for (int d = 0; d < 3; ++d) p.pt[k][d] = prm[3 * k + d];
    p.radius = prm[6];
    if (p.radius < 0) { p.radius = -p.radius; p.front_sign = -1; }
    for (int d = 0; d < 3; ++d) p.normal[d] = p.pt[1][d] - p.pt[0][d];
    if (!unit(p.normal)) { if (err) *err = "panel cyl: the end points coincide"; return -6; }
  } else if (shape == 4) {
    if (!need(7, "hemi")) return -7;
    for (int d = 0; d < 3; ++d) p.center[d] = prm[d];
    p.radius = prm[3];
    if (p.radius < 0) { p.radius = -p.radius; p.front_sign = -1; }
    for (int d = 0; d < 3; ++d) p.normal[d] = prm[4 + d];
    if (!unit(p.normal)) { if (err) *err = "panel hemi: zero outward vector"; return -6; }
  } else if (shape == 5) {
    if (!need(7, "disk")) return -7;
    for (int d = 0; d < 3; ++d) p.center[d] = prm[d];
    p.radius = prm[3];
    if (!(p.radius > 0)) { if (err) *err = "panel disk: radius must be > 0"; return -6; }
    for (int d = 0; d < 3; ++d) p.normal[d] = prm[4 + d];
    if (!unit(p.normal)) { if (err) *err = "panel disk: zero normal"; return -6; }
  } else {
    if (err) *err = "panel shape not supported";
    return -7;
  }
  *out = p;
  return 0;
}

// compartment block statements (smolcomparts.c:880-930 cmptreadstring)
static int read_compartment_statement(Sim &sim, int c, const std::string &word, const std::vector<std::string> &w,
                                      std::string *err) {
  CompartDef &cd = sim.cmpts[c];
  if (word == "surface") {
    if (w.empty()) { if (err) *err = "compartment surface: missing name"; return -7; }
    int sidx = -1;
    for (size_t k = 0; k < sim.surfaces.size(); ++k)
      if (sim.surfaces[k].name == w[0]) sidx = (int)k;
    if (sidx < 0) { if (err) *err = "compartment surface '" + w[0] + "' not recognized"; return -3; }
    if (std::find(cd.surfaces.begin(), cd.surfaces.end(), sidx) != cd.surfaces.end()) {
      if (err) *err = "cannot add surface to compartment more than once";
      return -7;
    }
    cd.surfaces.push_back(sidx);
  } else if (word == "point") {
    if ((int)w.size() < sim.dim) { if (err) *err = "compartment point: missing values"; return -7; }
    if ((int)cd.pts.size() >= kMaxCmptPts) { if (err) *err = "too many compartment points"; return -6; }
    std::vector<double> p(3, 0.0);
    for (int d = 0; d < sim.dim; ++d) p[d] = atof(w[d].c_str());
    cd.pts.push_back(p);
  } else if (word == "compartment") {
    if (w.size() < 2) { if (err) *err = "compartment format: symbol name"; return -7; }
    static const char *syms[] = {"equal", "equalnot", "and", "or", "xor", "andnot", "ornot"};
    int sym = -1;
    for (int k = 0; k < 7; ++k)
      if (w[0] == syms[k]) sym = k;
    if (sym < 0) { if (err) *err = "unrecognized logic symbol " + w[0]; return -7; }
    const int other = sim.compartment_index(w[1]);
    if (other < 0) { if (err) *err = "compartment name not recognized"; return -3; }
    if (other == c) { if (err) *err = "cannot add a compartment to itself"; return -7; }
    if ((int)cd.logic.size() >= kMaxCmptLogic) { if (err) *err = "too many compartment logic terms"; return -6; }
    cd.logic.push_back({sym, other});
  } else {
    if (err) *err = "syntax error within compartment block: statement not recognized: " + word;
    return -7;
  }
  invalidate_compartments(sim);
  sim.need_update = sim.need_rebuild = true;
  return 0;
}

int read_compartment_words(Sim &sim, int c, const std::string &word, const std::vector<std::string> &w,
                           std::string *err) {
  return read_compartment_statement(sim, c, word, w, err);
}

// surface block statements (smolsurface.c surfreadstring subset)
static int read_surface_statement(Sim &sim, SurfaceDef &sf, const std::string &word,
                                  const std::vector<std::string> &w, std::string *err) {
  auto act_of = [](const std::string &s) -> int {
    if (s == "reflect" || s == "r") return 0;
    if (s == "transmit" || s == "t") return 1;
    if (s == "absorb" || s == "a") return 2;
    return -1;
  };
  const int sidx = (int)(&sf - sim.surfaces.data());
  const int rr = read_surface_rule_statement(sim, sidx, word, w, err);
  if (rr != 1) return rr;
  if (word == "name") {
    if (!w.empty()) sf.name = w[0];
  } else if (word == "panel") {
    if (w.empty()) { if (err) *err = "panel: missing shape"; return -7; }
    const std::string &sh = w[0];
    const int shape = (sh == "rect" || sh == "r") ? 0 : (sh == "tri" || sh == "t") ? 1
                      : (sh == "sph" || sh == "sphere" || sh == "s") ? 2 : (sh == "cyl" || sh == "c") ? 3
                      : (sh == "hemi" || sh == "h") ? 4 : (sh == "disk" || sh == "d") ? 5 : -1;
    if (shape < 0) { if (err) *err = "panel shape not supported by the GPU engine: " + sh; return -7; }
    std::string axis;
    size_t k = 1;
    if (shape == 0) {
      if (w.size() < 2) { if (err) *err = "panel rect: missing axis"; return -7; }
      axis = w[1];
      k = 2;
    }
    std::vector<double> prm;
    for (; k < w.size(); ++k) {
      char *end = nullptr;
      const double v = strtod(w[k].c_str(), &end);
      if (!end || *end) break;  // a trailing panel name
      prm.push_back(v);
    }
    PanelSpec p{};
    const int rc = make_panel(sim.dim, shape, axis, prm.data(), (int)prm.size(), &p, err);
    if (rc) return rc;
    const std::string name = new_panel_name(sf, shape, k < w.size() ? w[k] : std::string());
    // a name used before replaces that panel (surfaddpanel, smolsurface.c:2642-2651)
    int same = -1;
    for (size_t q = 0; q < sf.pnames.size(); ++q)
      if (sf.pnames[q] == name) same = (int)q;
    if (same >= 0) {
      if (sf.panels[same].shape != shape) { if (err) *err = "panel name was used before for a different shape"; return -6; }
      sf.panels[same] = p;
    } else {
      if ((int)sf.panels.size() >= kMaxPanels) { if (err) *err = "too many panels"; return -6; }
      sf.panels.push_back(p);
      sf.pnames.push_back(name);
    }
    invalidate_compartments(sim);
  } else if (word == "color" || word == "thickness" || word == "polygon" || word == "stipple" ||
             word == "shininess") {
  } else {
    if (err) *err = "unsupported surface statement: " + word;
    return -7;
  }
  return 0;
}

int load_config_file(Sim &sim, const std::string &path, const std::string &name, std::string *err) {
  std::string full = path.empty() ? name : (path + "/" + name);
  std::ifstream in(full);
  if (!in) { if (err) *err = "cannot open " + full; return -3; }
  sim.filepath = path;
  std::string line;
  std::vector<int> skip;  // ifdefine nesting: 1 = skipping
  SurfaceDef *cur_srf = nullptr;
  int cur_cmpt = -1;
  int lineno = 0;
  while (std::getline(in, line)) {
    ++lineno;
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    for (auto &kv : sim.defines) {  // textual substitution of defined names
      size_t pos = 0;
      while ((pos = line.find(kv.first, pos)) != std::string::npos) {
        const bool lb = pos == 0 || isspace((unsigned char)line[pos - 1]);
        const size_t e = pos + kv.first.size();
        const bool rb = e >= line.size() || isspace((unsigned char)line[e]);
        if (lb && rb) { line.replace(pos, kv.first.size(), kv.second); pos += kv.second.size(); }
        else pos = e;
      }
    }
    std::istringstream is(line);
    std::string word;
    if (!(is >> word)) continue;
    std::string rest;
    std::getline(is, rest);
    const bool skipping = !skip.empty() && skip.back();
    if (word == "ifdefine" || word == "ifundefine") {
      std::string nm;
      std::istringstream(rest) >> nm;
      bool def = sim.defines.count(nm) > 0;
      bool take = (word == "ifdefine") ? def : !def;
      skip.push_back(skipping || !take);
      continue;
    }
    if (word == "else") {
      if (!skip.empty()) {
        const bool outer = skip.size() > 1 && skip[skip.size() - 2];
        skip.back() = outer || !skip.back();
      }
      continue;
    }
    if (word == "endif") {
      if (!skip.empty()) skip.pop_back();
      continue;
    }
    if (skipping) continue;
    if (word == "end_file") break;
    if (word == "define") {
      std::istringstream rs(rest);
      std::string k, vv;
      rs >> k;
      std::getline(rs, vv);
      const size_t b = vv.find_first_not_of(" \t");
      sim.defines[k] = (b == std::string::npos) ? "" : vv.substr(b);
      continue;
    }
    if (word == "start_surface") {
      std::string nm;
      std::istringstream(rest) >> nm;
      SurfaceDef s;
      s.name = nm.empty() ? "surf" + std::to_string(sim.surfaces.size()) : nm;
      cur_srf = nullptr;  // a known name continues that surface (surfaddsurface)
      for (SurfaceDef &x : sim.surfaces)
        if (x.name == s.name) cur_srf = &x;
      if (!cur_srf) {
        sim.surfaces.push_back(s);
        cur_srf = &sim.surfaces.back();
      }
      sim.need_rebuild = true;
      continue;
    }
    if (word == "end_surface") {
      cur_srf = nullptr;
      continue;
    }
    if (word == "start_compartment") {
      std::string nm;
      std::istringstream(rest) >> nm;
      if (nm.empty() || sim.compartment_index(nm) >= 0) {
        if (err) *err = full + ":" + std::to_string(lineno) + ": start_compartment: missing or repeated name";
        return -7;
      }
      if ((int)sim.cmpts.size() >= kMaxCmpt) {
        if (err) *err = full + ":" + std::to_string(lineno) + ": too many compartments";
        return -6;
      }
      CompartDef c;
      c.name = nm;
      sim.cmpts.push_back(c);
      cur_cmpt = (int)sim.cmpts.size() - 1;
      sim.need_rebuild = true;
      continue;
    }
    if (word == "end_compartment") {
      cur_cmpt = -1;
      continue;
    }
    int rc;
    if (cur_srf) rc = read_surface_statement(sim, *cur_srf, word, split_ws(rest), err);
    else if (cur_cmpt >= 0) rc = read_compartment_statement(sim, cur_cmpt, word, split_ws(rest), err);
    else rc = read_config_statement(sim, word, rest, err);
    if (rc) {
      if (err) *err = full + ":" + std::to_string(lineno) + ": " + *err;
      return rc;
    }
  }
  return 0;
}

}  // namespace smolb

namespace smolb {
int find_reverse_rxn(const Sim &s, int order, int r, int *o2, int *r2) { return find_reverse(s, order, r, o2, r2); }
}  // namespace smolb
