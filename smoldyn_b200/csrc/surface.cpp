// Surface-bound states on the host: the surface statements that set them up
// (surfreadstring's action, rate, rate_internal, neighbors and
// neighbor_action, smolsurface.c:3265-3626; surface_mol, smolsim.cpp:1027),
// the derivation of interaction probabilities from rates (surfupdateparams
// :3735-3800 with srfcalcprob :3070-3146), placement of molecules on panels
// (addsurfmol, smolmolec.c:2744) and the device rule table.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "boundgeom.cuh"
#include "sim.h"
#include "surfparam.h"

namespace smolb {

namespace {

enum { SAreflect = 0, SAtrans = 1, SAabsorb = 2, SAjump = 3, SAport = 4, SAmult = 5, SAno = 6, SAnone = 7,
       SAadsorb = 8, SArevdes = 9, SAirrevdes = 10, SAflip = 11 };
enum { MSsoln = 0, MSfront = 1, MSback = 2, MSup = 3, MSdown = 4, MSbsoln = 5, MSall = 6, MSnone = 7 };
enum { PFfront = 0, PFback = 1, PFnone = 2, PFboth = 3 };

int detail_key(int sp, int ms, int face) { return (sp * kSrfStates + ms) * 3 + face; }

// molstring2ms (smolmolec.c:75)
int parse_ms(const std::string &s) {
  if (s == "solution" || s == "fsoln" || s == "soln" || s == "aq") return MSsoln;
  if (s == "front") return MSfront;
  if (s == "back") return MSback;
  if (s == "up") return MSup;
  if (s == "down") return MSdown;
  if (s == "bsoln") return MSbsoln;
  if (s == "all") return MSall;
  return MSnone;
}

// surfstring2face
int parse_face(const std::string &s) {
  if (s == "front" || s == "f") return PFfront;
  if (s == "back" || s == "b") return PFback;
  if (s == "both" || s == "all") return PFboth;
  return PFnone;
}

// "name" or "name(state)": species indices ("all": every species) and state
// (solution when none is given).  Returns 0, or -3 for an unknown name.
int species_state(const Sim &sim, const std::string &w, std::vector<int> *ids, int *ms) {
  ids->clear();
  std::string name = w;
  *ms = MSsoln;
  const size_t paren = w.find('(');
  if (paren != std::string::npos) {
    const size_t close = w.find(')', paren);
    if (close == std::string::npos) return -7;
    *ms = parse_ms(w.substr(paren + 1, close - paren - 1));
    name = w.substr(0, paren);
  }
  if (name == "all") {
    for (size_t i = 1; i < sim.species.size(); ++i) ids->push_back((int)i);
    return 0;
  }
  const int i = sim.species_index(name);
  if (i <= 0) return -3;
  ids->push_back(i);
  return 0;
}

const char *shape_name(int shape) {
  static const char *n[] = {"rect", "tri", "sph", "cyl", "hemi", "disk"};
  return (shape >= 0 && shape < 6) ? n[shape] : "";
}

int parse_shape(const std::string &s) {
  if (s == "rect" || s == "r") return 0;
  if (s == "tri" || s == "t") return 1;
  if (s == "sph" || s == "sphere" || s == "s") return 2;
  if (s == "cyl" || s == "c") return 3;
  if (s == "hemi" || s == "h") return 4;
  if (s == "disk" || s == "d") return 5;
  if (s == "all") return 6;
  return -1;
}

// The action in force for (species, state, face) of a surface: a statement's
// setting, else the default (solution at a face: the per-species masks or
// the surface-wide action; bound states: transmit at faces, no action with
// no face).  States 0..2 only.
int eff_act(const SurfaceDef &sf, int i, int ms, int face) {
  if (ms == MSbsoln) ms = MSsoln;
  if (ms > MSback || face > PFnone) return SAno;
  const int a = sf.act[i][ms][face];
  if (a >= 0) return a;
  if (face == PFnone) return SAno;
  if (ms != MSsoln) return SAtrans;
  const uint32_t bit = 1u << i;
  if (face == PFfront) {
    if (sf.absorb_front & bit) return SAabsorb;
    if (sf.trans_front & bit) return SAtrans;
    if (sf.refl_front & bit) return SAreflect;
    return sf.act_front;
  }
  if (sf.absorb_back & bit) return SAabsorb;
  if (sf.trans_back & bit) return SAtrans;
  if (sf.refl_back & bit) return SAreflect;
  return sf.act_back;
}

const SrfDetail *find_detail(const SurfaceDef &sf, int i, int ms, int face) {
  if (ms == MSbsoln) ms = MSsoln;
  if (ms > MSback || face > PFnone) return nullptr;
  auto it = sf.det.find(detail_key(i, ms, face));
  return it == sf.det.end() ? nullptr : &it->second;
}

SrfDetail &get_detail(SurfaceDef &sf, int i, int ms, int face) {
  auto it = sf.det.find(detail_key(i, ms, face));
  if (it != sf.det.end()) return it->second;
  SrfDetail d;
  for (int k = 0; k < 6; ++k) d.newspec[k] = i;  // surfaceactionalloc: the same species by default
  return sf.det.emplace(detail_key(i, ms, face), d).first->second;
}

// srfsamestate (smolsurface.c:638): whether destination ms2 leaves the
// molecule where it was, and in *ms3 the destination that means "stay".
bool same_state(int ms1, int face1, int ms2, int *ms3) {
  const bool same = (face1 == PFfront && ms2 == MSsoln) || (face1 == PFback && ms2 == MSbsoln) ||
                    (face1 == PFnone && ms1 == ms2);
  if (ms3) *ms3 = face1 == PFfront ? MSsoln : face1 == PFback ? MSbsoln : (ms1 == MSsoln ? MSnone : ms1);
  return same;
}

// srfreverseaction (smolsurface.c:661): the interaction that undoes
// (ms1, face1) -> ms2, as (ms3, face2) -> ms4 with the action it would be.
void reverse_action(int ms1, int face1, int ms2, int *ms3, int *face2, int *ms4, int *act) {
  const bool to_soln = ms2 == MSsoln || ms2 == MSbsoln;
  if (ms1 == MSsoln && face1 == PFnone) {
    *ms3 = *ms4 = MSnone; *face2 = PFnone; *act = SAnone;
  } else if (ms1 == MSsoln) {
    if (to_soln) {
      *ms3 = MSsoln;
      *face2 = ms2 == MSsoln ? PFfront : PFback;
      *act = face1 == *face2 ? SAreflect : SAtrans;
    } else {
      *ms3 = ms2; *face2 = PFnone; *act = SAadsorb;
    }
    *ms4 = face1 == PFfront ? MSsoln : MSbsoln;
  } else if (face1 == PFnone) {
    if (to_soln) {
      *ms3 = MSsoln; *face2 = ms2 == MSsoln ? PFfront : PFback; *act = SArevdes;
    } else {
      *ms3 = ms2; *face2 = PFnone; *act = SAflip;
    }
    *ms4 = ms1;
  } else {
    if (to_soln) {
      *ms3 = ms1;
      *face2 = ms2 == MSsoln ? PFfront : PFback;
      *ms4 = face1 == PFfront ? MSsoln : MSbsoln;
      *act = face1 == *face2 ? SAreflect : SAtrans;
    } else {
      *ms3 = ms2; *face2 = PFboth; *ms4 = ms1; *act = SAno;
    }
  }
}

}  // namespace

namespace {

// srfcalcprob (smolsurface.c:3070-3146): probability of (ms1, face) -> ms2
// for species i of surface s from the requested rates.  *err is set (and
// -3 returned) when a transmission probability cannot be computed.
double calc_prob(const Sim &sim, const SurfaceDef &sf, int i, int ms1, int face, int ms2, std::string *err) {
  if (ms1 == MSsoln && face == PFnone) return 0;
  if (eff_act(sf, i, ms1, face) != SAmult) return -1;
  const SrfDetail *d = find_detail(sf, i, ms1, face);
  if (!d) return -1;
  if (d->datasrc[ms2] == 2) return d->prob_req[ms2];
  if (d->datasrc[ms2] != 1) return 0;
  const double rate = d->rate[ms2];
  if (rate < 0 && rate != -1) return -2;
  if (rate == 0) return 0;
  int ms3, face2, ms4, actrev;
  reverse_action(ms1, face, ms2, &ms3, &face2, &ms4, &actrev);
  const int i2 = d->newspec[ms2];
  double raterev = 0;
  if (!i2 || actrev == SAno || face2 > PFnone || ms3 > MSback) {
    raterev = 0;
  } else if (eff_act(sf, i2, ms3, face2) == SAmult) {
    const SrfDetail *dr = find_detail(sf, i2, ms3, face2);
    raterev = (dr && dr->datasrc[ms4] == 1) ? dr->rate[ms4] : 0;
  } else if (eff_act(sf, i2, ms3, face2) == actrev) {
    raterev = -1;
  }
  if (raterev < 0 && raterev != -1) raterev = 0;
  const double dt = sim.dt, difc = sim.species[i].difc;
  double sum = 0;
  if (ms1 != MSsoln && face == PFnone)
    for (int k = 0; k < 6; ++k)
      if (k != ms1 && d->datasrc[k] == 1 && d->rate[k] >= 0) sum += d->rate[k];
  const bool to_soln = ms2 == MSsoln || ms2 == MSbsoln;
  const bool reflect_self = (face == PFfront && ms2 == MSsoln) || (face == PFback && ms2 == MSbsoln);
  // transmission with a reverse rate: surfacetransmit with both coefficients
  auto no_revtrans = [&]() {
    const double difcrev = sim.species[i2].difc;
    double p1 = 0, p2 = 0;
    if (surface_transmit(rate, raterev, difc, difcrev, dt, &p1, &p2)) {
      if (err) *err = "transmission rates need positive diffusion coefficients and time step";
      return -3.0;
    }
    return p1;
  };
  if (ms1 == MSsoln) {
    if (reflect_self) return 0;
    if (to_soln) return raterev == 0 ? surface_prob(rate, 0, dt, difc, nullptr, kSrfIrrTrans) : no_revtrans();
    return raterev == 0 ? surface_prob(rate, 0, dt, difc, nullptr, kSrfIrrAds)
                        : surface_prob(rate, raterev, dt, difc, nullptr, kSrfRevAds);
  }
  if (face == PFnone) {
    if (to_soln)
      return raterev == 0 ? surface_prob(rate, sum, dt, difc, nullptr, kSrfIrrDes)
                          : surface_prob(rate, raterev, dt, difc, nullptr, kSrfRevDes);
    if (ms1 == ms2) return 0;
    return raterev == 0 ? surface_prob(rate, sum, dt, difc, nullptr, kSrfIrrFlip)
                        : surface_prob(rate, raterev, dt, difc, nullptr, kSrfRevFlip);
  }
  if (reflect_self) return 0;
  if (to_soln) return raterev == 0 ? surface_prob(rate, 0, dt, difc, nullptr, kSrfIrrTrans) : no_revtrans();
  return surface_prob(rate, 0, dt, difc, nullptr, kSrfIrrAds);
}

}  // namespace

int derive_surface_params(Sim &sim, std::string *err) {
  const int ns = (int)sim.species.size();
  for (SurfaceDef &sf : sim.surfaces) {
    // probabilities of each outcome
    for (auto &kv : sf.det) {
      const int key = kv.first, face = key % 3, ms1 = (key / 3) % kSrfStates, i = key / 3 / kSrfStates;
      if (i >= ns || eff_act(sf, i, ms1, face) != SAmult) continue;
      for (int ms2 = 0; ms2 < 6; ++ms2) {
        std::string e;
        const double pr = calc_prob(sim, sf, i, ms1, face, ms2, &e);
        if (pr == -3.0 && !e.empty()) { if (err) *err = e; return -6; }
        kv.second.prob[ms2] = pr;
      }
    }
    // staying put takes what the others leave; more than 1 in total is scaled down
    for (auto &kv : sf.det) {
      const int key = kv.first, face = key % 3, ms1 = (key / 3) % kSrfStates, i = key / 3 / kSrfStates;
      if (i >= ns || eff_act(sf, i, ms1, face) != SAmult) continue;
      SrfDetail &d = kv.second;
      double sum = 0;
      for (int ms2 = 0; ms2 < 6; ++ms2)
        if (!same_state(ms1, face, ms2, nullptr)) sum += d.prob[ms2];
      if (sum > 1.0) {
        d.prob[ms1] = 0;
        for (int ms2 = 0; ms2 < 6; ++ms2) d.prob[ms2] /= sum;
      } else {
        int ms3;
        same_state(ms1, face, MSsoln, &ms3);
        if (ms3 >= 0 && ms3 < 6) d.prob[ms3] = 1.0 - sum;
      }
      double c = 0;
      for (int ms2 = 0; ms2 < 6; ++ms2) {
        c += d.prob[ms2];
        d.cum[ms2] = c;
      }
    }
    // probabilities of the reverse interactions
    for (auto &kv : sf.det) {
      const int key = kv.first, face = key % 3, ms1 = (key / 3) % kSrfStates, i = key / 3 / kSrfStates;
      if (i >= ns || eff_act(sf, i, ms1, face) != SAmult) continue;
      SrfDetail &d = kv.second;
      for (int ms2 = 0; ms2 < 6; ++ms2) {
        int ms3, face2, ms4, act;
        reverse_action(ms1, face, ms2, &ms3, &face2, &ms4, &act);
        d.rev[ms2] = 0;
        if (face2 == PFboth || face2 > PFnone || ms3 > MSback || ms3 < 0) continue;
        if (!find_detail(sf, i, ms3, face2)) continue;
        const SrfDetail *dr = find_detail(sf, d.newspec[ms2], ms3, face2);
        if (dr && ms4 >= 0 && ms4 < 6) d.rev[ms2] = dr->prob[ms4];
      }
    }
  }
  return 0;
}

bool surface_bound_mode(const Sim &sim) {
  if (!sim.pend_bound.empty()) return true;
  for (int o = 0; o < 3; ++o)  // reactions of bound reactants or with bound products
    for (const RxnDef &x : sim.rxn[o]) {
      for (int q = 0; q < x.order; ++q)
        if (x.rstate[q] != 0) return true;
      for (int q = 0; q < x.nprod; ++q)
        if (x.pstate[q] == MSfront || x.pstate[q] == MSback) return true;
    }
  for (const SurfaceDef &sf : sim.surfaces)
    for (size_t i = 1; i < sim.species.size() && i < (size_t)kMaxSpecies; ++i)
      for (int ms = 0; ms < kSrfStates; ++ms)
        for (int f = 0; f < 3; ++f) {
          const int a = sf.act[i][ms][f];
          if (a == SAmult || a == SAadsorb || (ms != MSsoln && a >= 0)) return true;
        }
  return false;
}

int find_panel(const Sim &sim, int s, const std::string &name, int *srf_out) {
  std::string pn = name;
  const size_t colon = name.find(':');
  if (colon != std::string::npos) {
    s = -1;
    for (size_t k = 0; k < sim.surfaces.size(); ++k)
      if (sim.surfaces[k].name == name.substr(0, colon)) s = (int)k;
    pn = name.substr(colon + 1);
  }
  if (s < 0 || s >= (int)sim.surfaces.size()) return -1;
  const SurfaceDef &sf = sim.surfaces[s];
  for (size_t q = 0; q < sf.pnames.size(); ++q)
    if (sf.pnames[q] == pn) {
      if (srf_out) *srf_out = s;
      return (int)q;
    }
  return -1;
}

// Surface statements of surface-bound states (surfreadstring subset):
// returns 1 when `word` is not one of them.
int read_surface_rule_statement(Sim &sim, int sidx, const std::string &word, const std::vector<std::string> &w,
                                std::string *err) {
  SurfaceDef &sf = sim.surfaces[sidx];
  if (word == "action") {
    // species[(state)] face action [new_species], or the older face species action
    if (w.size() < 3) { if (err) *err = "action format: species[(state)] face action"; return -7; }
    std::vector<int> ids;
    int ms = MSsoln;
    int face = parse_face(w[1]);
    int rc = species_state(sim, w[0], &ids, &ms);
    if (face == PFnone || rc) {
      face = parse_face(w[0]);
      rc = species_state(sim, w[1], &ids, &ms);
    }
    if (face == PFnone) { if (err) *err = "in action, face name needs to be 'front', 'back', or 'both'"; return -7; }
    if (rc) { if (err) *err = "in action, molecule name not recognized"; return -3; }
    const std::string &an = w[2];
    int a = -1;
    if (an == "reflect" || an == "r") a = SAreflect;
    else if (an == "transmit" || an == "t") a = SAtrans;
    else if (an == "absorb" || an == "a") a = SAabsorb;
    else if (an == "jump" || an == "j" || an == "periodic") a = SAjump;  // solution molecules only (dosurfinteract)
    if (a < 0) { if (err) *err = "surface action not supported by the GPU engine: " + an; return -7; }
    if (a == SAjump && ms != MSsoln && ms != MSall) {
      if (err) *err = "the jump action applies to solution molecules";
      return -7;
    }
    if (ms == MSup || ms == MSdown || ms == MSbsoln || ms == MSnone) {
      if (err) *err = "surface action state not supported by the GPU engine";
      return -7;
    }
    int newsp = 0;
    if (w.size() > 3) {
      newsp = sim.species_index(w[3]);
      if (newsp <= 0) { if (err) *err = "final word of line is not an individual species name"; return -3; }
    }
    const int lo = ms == MSall ? 0 : ms, hi = (ms == MSall && a != SAjump) ? kSrfStates - 1 : lo;
    for (int i : ids)
      for (int m = lo; m <= hi; ++m)
        for (int f = 0; f < 2; ++f) {
          if (!(face == PFboth || face == f)) continue;
          sf.act[i][m][f] = a;
          if (m == MSsoln) {  // the per-species masks of the solution state
            const uint32_t bit = 1u << i;
            uint32_t &ab = f ? sf.absorb_back : sf.absorb_front, &tr = f ? sf.trans_back : sf.trans_front,
                     &rf = f ? sf.refl_back : sf.refl_front, &jp = f ? sf.jump_back : sf.jump_front;
            ab &= ~bit; tr &= ~bit; rf &= ~bit; jp &= ~bit;
            (a == SAabsorb ? ab : a == SAtrans ? tr : a == SAjump ? jp : rf) |= bit;
          }
          if (newsp) {
            SrfDetail &d = get_detail(sf, i, m, f);
            d.datasrc[m] = 3;
            d.newspec[m] = newsp;
          }
        }
    return 0;
  }
  if (word == "jump") {
    // jump panel1 face1 -> panel2 face2, or <-> for both directions
    // (smolsurface.c:3574-3600): panels of this surface with the same shape
    if (w.size() != 5) { if (err) *err = "format for jump: panel1 face1 -> panel2 face2"; return -7; }
    int q[2] = {-1, -1}, f[2];
    const std::string pn[2] = {w[0], w[3]}, fn[2] = {w[1], w[4]};
    for (int k = 0; k < 2; ++k) {
      for (size_t j = 0; j < sf.pnames.size(); ++j)
        if (sf.pnames[j] == pn[k]) q[k] = (int)j;
      if (q[k] < 0) { if (err) *err = "panel name listed in jump is not recognized"; return -3; }
      f[k] = fn[k] == "front" ? 0 : fn[k] == "back" ? 1 : -1;
      if (f[k] < 0) { if (err) *err = "face listed in jump needs to be 'front' or 'back'"; return -7; }
    }
    if (sf.panels[q[0]].shape != sf.panels[q[1]].shape) {
      if (err) *err = "second panel name listed in jump is not recognized, or not same shape as first panel";
      return -3;
    }
    if (q[0] == q[1]) { if (err) *err = "two different panels need to be listed in a jump statement"; return -7; }
    if (w[2] != "->" && w[2] != "<->") { if (err) *err = "jump operator needs to be -> or <->"; return -7; }
    sf.jumps.push_back({q[0], f[0], q[1], f[1]});
    if (w[2] == "<->") sf.jumps.push_back({q[1], f[1], q[0], f[0]});
    return 0;
  }
  if (word == "rate" || word == "rate_internal") {
    // species[(state)] state1 state2 value [new_species] (smolsurface.c:3329-3414)
    if (w.size() < 4) { if (err) *err = "format: species[(state)] state1 state2 value [new_species]"; return -7; }
    std::vector<int> ids;
    int ms = MSsoln;
    if (species_state(sim, w[0], &ids, &ms)) { if (err) *err = "molecule name not recognized"; return -3; }
    if (ms >= MSbsoln) { if (err) *err = "state is not recognized or not permitted"; return -7; }
    const int ms1 = parse_ms(w[1]), ms2 = parse_ms(w[2]);
    if (ms1 > MSbsoln) { if (err) *err = "state1 is not recognized or not permitted"; return -7; }
    if (ms2 > MSbsoln) { if (err) *err = "state2 is not recognized or not permitted"; return -7; }
    if (ms == MSsoln && ms1 == ms2) { if (err) *err = "it is not permitted for state1 to equal state2"; return -7; }
    if (ms != MSsoln && !(ms1 == ms || ms1 == MSsoln || ms1 == MSbsoln)) {
      if (err) *err = "state1 does not make sense";
      return -7;
    }
    char *end = nullptr;
    const double v = strtod(w[3].c_str(), &end);
    if (!end || *end) { if (err) *err = "surface rate value cannot be read"; return -7; }
    if (!(v >= 0 || (word == "rate" && v == -1))) {
      if (err) *err = "surface rate values must be non-negative, or -1 to indicate maximum";
      return -6;
    }
    if (word == "rate_internal" && v > 1) { if (err) *err = "surface interaction probabilities cannot be greater than 1"; return -6; }
    int newsp = -5;
    if (w.size() > 4) {
      newsp = sim.species_index(w[4]);
      if (newsp < 0) { if (err) *err = "new species name not recognized"; return -3; }
      if (w.size() > 5) { if (err) *err = "unexpected text at end of line"; return -7; }
    }
    // srftristate2index (smolsurface.c:713): table state, face and destination
    const int m0 = ms == MSnone ? MSsoln : ms;
    int ms3 = (m0 == MSsoln) ? ((ms1 == MSsoln || ms1 == MSbsoln) ? MSsoln : ms1) : m0;
    int face = ms1 == MSsoln ? PFfront : ms1 == MSbsoln ? PFback : PFnone;
    const int ms4 = ms2;
    if (ms3 == MSup || ms3 == MSdown || ms4 == MSup || ms4 == MSdown) {
      if (err) *err = "the up and down surface states are not supported by the GPU engine";
      return -7;
    }
    for (int i : ids) {
      SrfDetail &d = get_detail(sf, i, ms3, face);
      sf.act[i][ms3][face] = SAmult;
      if (word == "rate") { d.rate[ms4] = v; d.datasrc[ms4] = 1; }
      else { d.prob_req[ms4] = v; d.datasrc[ms4] = 2; }
      d.newspec[ms4] = newsp == -5 ? i : newsp;
    }
    return 0;
  }
  if (word == "neighbors" || word == "neighbours") {
    if (w.size() < 2) { if (err) *err = "format for neighbors: panel neigh1 neigh2 ..."; return -7; }
    int s0 = sidx;
    const int p0 = find_panel(sim, sidx, w[0], &s0);
    if (p0 < 0) { if (err) *err = "first panel name listed in neighbors, '" + w[0] + "', not recognized"; return -3; }
    SurfaceDef &own = sim.surfaces[s0];
    if (own.neigh.size() < own.panels.size()) own.neigh.resize(own.panels.size());
    for (size_t k = 1; k < w.size(); ++k) {
      int s1 = sidx;
      const int p1 = find_panel(sim, sidx, w[k], &s1);
      if (p1 < 0) { if (err) *err = "neighbor panel name '" + w[k] + "' not recognized"; return -3; }
      auto &lst = own.neigh[p0];
      if (std::find(lst.begin(), lst.end(), std::make_pair(s1, p1)) == lst.end()) lst.push_back({s1, p1});
      if ((int)lst.size() > kMaxNeigh) { if (err) *err = "too many neighbouring panels (max 8)"; return -6; }
    }
    return 0;
  }
  if (word == "neighbor_action" || word == "neighbour_action") {
    if (w.size() != 1 || (w[0] != "hop" && w[0] != "stay")) {
      if (err) *err = "format for neighbor_action: 'hop' or 'stay'";
      return -7;
    }
    sf.neighhop = w[0] == "hop" ? 1 : 0;
    return 0;
  }
  return 1;
}

// Name of a new panel of `shape` in surface sf: the given name, or the
// shape's name with the panel's index among the surface's panels of that
// shape (panelsalloc, smolsurface.c:866).
std::string new_panel_name(const SurfaceDef &sf, int shape, const std::string &given) {
  if (!given.empty()) return given;
  int k = 0;
  for (const PanelSpec &p : sf.panels) k += p.shape == shape;
  return std::string(shape_name(shape)) + std::to_string(k);
}

namespace {

// panelarea: area in 3-D, length in 2-D (a rectangle is a segment, a
// sphere a circle), 1 in 1-D
double panel_area(const PanelSpec &p, int dim) {
  const double pi = 3.14159265358979323846;
  if (dim == 1) return 1.0;
  if (dim == 2) return p.shape == 2 ? 2 * pi * p.radius : std::fabs(p.hi[1 - p.axis] - p.lo[1 - p.axis]);
  switch (p.shape) {
    case 0: {
      double a = 1;
      for (int d = 0; d < 3; ++d)
        if (d != p.axis) a *= p.hi[d] - p.lo[d];
      return std::fabs(a);
    }
    case 1: {
      double e1[3], e2[3];
      for (int d = 0; d < 3; ++d) { e1[d] = p.pt[1][d] - p.pt[0][d]; e2[d] = p.pt[2][d] - p.pt[0][d]; }
      const double c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
      return 0.5 * std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    }
    case 2: return 4 * pi * p.radius * p.radius;
    case 3: {
      double l2 = 0;
      for (int d = 0; d < 3; ++d) l2 += (p.pt[1][d] - p.pt[0][d]) * (p.pt[1][d] - p.pt[0][d]);
      return 2 * pi * p.radius * std::sqrt(l2);
    }
    case 4: return 2 * pi * p.radius * p.radius;
    default: return pi * p.radius * p.radius;
  }
}

// two unit vectors perpendicular to unit vector n and to each other
void perp_basis(const double n[3], double e1[3], double e2[3]) {
  const double a[3] = {std::fabs(n[0]) < 0.9 ? 1.0 : 0.0, std::fabs(n[0]) < 0.9 ? 0.0 : 1.0, 0.0};
  e1[0] = a[1] * n[2] - a[2] * n[1];
  e1[1] = a[2] * n[0] - a[0] * n[2];
  e1[2] = a[0] * n[1] - a[1] * n[0];
  const double l = std::sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
  for (int d = 0; d < 3; ++d) e1[d] /= l;
  e2[0] = n[1] * e1[2] - n[2] * e1[1];
  e2[1] = n[2] * e1[0] - n[0] * e1[2];
  e2[2] = n[0] * e1[1] - n[1] * e1[0];
}

// panelrandpos: a uniformly random point of the panel (absolute coordinates)
void panel_rand_pos(Sim &sim, const PanelSpec &p, double x[3]) {
  const double pi = 3.14159265358979323846;
  switch (p.shape) {
    case 0:
      for (int d = 0; d < 3; ++d) x[d] = d == p.axis ? p.pos : p.lo[d] + sim.rand_u01() * (p.hi[d] - p.lo[d]);
      return;
    case 1: {
      const double r1 = std::sqrt(sim.rand_u01()), r2 = sim.rand_u01();
      for (int d = 0; d < 3; ++d)
        x[d] = (1 - r1) * p.pt[0][d] + r1 * (1 - r2) * p.pt[1][d] + r1 * r2 * p.pt[2][d];
      return;
    }
    case 2:
    case 4: {
      if (sim.dim == 2) {  // a circle in the plane
        const double ph = 2 * pi * sim.rand_u01();
        x[0] = p.center[0] + p.radius * std::cos(ph);
        x[1] = p.center[1] + p.radius * std::sin(ph);
        x[2] = 0;
        return;
      }
      const double z = 2 * sim.rand_u01() - 1, ph = 2 * pi * sim.rand_u01(), s = std::sqrt(std::max(0.0, 1 - z * z));
      double u[3] = {s * std::cos(ph), s * std::sin(ph), z};
      if (p.shape == 4 && u[0] * p.normal[0] + u[1] * p.normal[1] + u[2] * p.normal[2] > 0)
        for (int d = 0; d < 3; ++d) u[d] = -u[d];
      for (int d = 0; d < 3; ++d) x[d] = p.center[d] + p.radius * u[d];
      return;
    }
    case 3: {
      double e1[3], e2[3];
      perp_basis(p.normal, e1, e2);
      const double t = sim.rand_u01(), ph = 2 * pi * sim.rand_u01();
      for (int d = 0; d < 3; ++d)
        x[d] = p.pt[0][d] + t * (p.pt[1][d] - p.pt[0][d]) + p.radius * (std::cos(ph) * e1[d] + std::sin(ph) * e2[d]);
      return;
    }
    default: {
      double e1[3], e2[3];
      perp_basis(p.normal, e1, e2);
      const double r = p.radius * std::sqrt(sim.rand_u01()), ph = 2 * pi * sim.rand_u01();
      for (int d = 0; d < 3; ++d) x[d] = p.center[d] + r * (std::cos(ph) * e1[d] + std::sin(ph) * e2[d]);
      return;
    }
  }
}

}  // namespace

double panel_area_dim(const PanelSpec &p, int dim) { return panel_area(p, dim); }

double surface_area(const Sim &sim, int s) {
  double a = 0;
  if (s < 0 || s >= (int)sim.surfaces.size()) return 0;
  for (const PanelSpec &p : sim.surfaces[s].panels) a += panel_area(p, sim.dim);
  return a;
}

int add_surface_molecules(Sim &sim, long long n, int sp, int ms, int srf, int shape, int pnl, const double *pos,
                          std::string *err) {
  if (ms != MSfront && ms != MSback) { if (err) *err = "surface molecules must be in the front or back state"; return -6; }
  if (sp <= 0 || sp >= (int)sim.species.size()) { if (err) *err = "species not recognized"; return -3; }
  std::vector<std::pair<int, int>> cand;
  std::vector<double> area;
  for (int s = 0; s < (int)sim.surfaces.size(); ++s) {
    if (srf >= 0 && s != srf) continue;
    const SurfaceDef &sf = sim.surfaces[s];
    for (int q = 0; q < (int)sf.panels.size(); ++q) {
      if (pnl >= 0 && q != pnl) continue;
      if (shape >= 0 && shape < 6 && sf.panels[q].shape != shape) continue;
      cand.push_back({s, q});
      area.push_back(panel_area(sf.panels[q], sim.dim));
    }
  }
  if (cand.empty()) { if (err) *err = "in surface_mol, no panels match the given description"; return -3; }
  if (pos && cand.size() != 1) { if (err) *err = "in surface_mol, use of coordinates requires that a specific panel be specified"; return -6; }
  double total = 0;
  for (double a : area) total += a;
  const double lo[3] = {sim.lo[0], sim.lo[1], sim.lo[2]};
  for (long long k = 0; k < n; ++k) {
    size_t c = 0;
    if (cand.size() > 1) {  // by area (intrandpD over the area table)
      double u = sim.rand_u01() * total;
      while (c + 1 < cand.size() && u >= area[c]) { u -= area[c]; ++c; }
    }
    const PanelSpec &ps = sim.surfaces[cand[c].first].panels[cand[c].second];
    PendBound b;
    if (pos) for (int d = 0; d < 3; ++d) b.pos[d] = pos[d];
    else panel_rand_pos(sim, ps, b.pos);
    // onto the state's face, as fixpt2panel with no margin
    const DevPanel dp = make_dev_panel(ps, lo);
    double x[3] = {b.pos[0] - lo[0], b.pos[1] - lo[1], b.pos[2] - lo[2]};
    fix_to_panel(dp, x, ms == MSfront ? kFaceFront : kFaceBack, 0.0);
    for (int d = 0; d < 3; ++d) b.pos[d] = x[d] + lo[d];
    b.species = sp;
    b.state = ms;
    b.surface = cand[c].first;
    b.panel = cand[c].second;
    sim.pend_bound.push_back(b);
  }
  sim.need_rebuild = true;
  return 0;
}

// surface_mol nmol species(state) surface panel_shape panel_name [position]
int read_surface_mol(Sim &sim, const std::vector<std::string> &w, std::string *err) {
  if (w.size() < 5) { if (err) *err = "surface_mol format: nmol species(state) surface panel_shape panel_name [position]"; return -7; }
  const long long n = atoll(w[0].c_str());
  if (n < 0) { if (err) *err = "in surface_mol, the number of molecules needs to be at least 0"; return -6; }
  std::vector<int> ids;
  int ms = MSsoln;
  if (species_state(sim, w[1], &ids, &ms) || ids.size() != 1) { if (err) *err = "molecule name not recognized"; return -3; }
  if (ms == MSsoln || ms >= MSbsoln) { if (err) *err = "state needs to be front, back, up, or down"; return -7; }
  int s = -1;
  if (w[2] != "all") {
    for (size_t k = 0; k < sim.surfaces.size(); ++k)
      if (sim.surfaces[k].name == w[2]) s = (int)k;
    if (s < 0) { if (err) *err = "surface name in surface_mol is not recognized"; return -3; }
  }
  const int shape = parse_shape(w[3]);
  if (shape < 0) { if (err) *err = "in surface_mol, panel shape name not recognized"; return -3; }
  int q = -1;
  if (w[4] != "all") {
    if (s < 0) { if (err) *err = "in surface_mol, a named panel needs a named surface"; return -3; }
    q = find_panel(sim, s, w[4], nullptr);
    if (q < 0) { if (err) *err = "in surface_mol, panel name not recognized"; return -3; }
  }
  if (w.size() > 5) {
    if (w.size() < 5 + (size_t)sim.dim) { if (err) *err = "surface_mol: incomplete position"; return -7; }
    double x[3] = {0, 0, 0};
    for (int d = 0; d < sim.dim; ++d) x[d] = atof(w[5 + d].c_str());
    return add_surface_molecules(sim, n, ids[0], ms, s, shape == 6 ? -1 : shape, q, x, err);
  }
  return add_surface_molecules(sim, n, ids[0], ms, s, shape == 6 ? -1 : shape, q, nullptr, err);
}

int surface_rule_info(Sim &sim, int s, int i, int ms, int face, int *act, double *prob, double *cum, double *rev,
                      std::string *err) {
  if (s < 0 || s >= (int)sim.surfaces.size()) { if (err) *err = "surface index out of range"; return -6; }
  if (i <= 0 || i >= (int)sim.species.size() || i >= kMaxSpecies) { if (err) *err = "species out of range"; return -6; }
  if (ms < 0 || ms >= kSrfStates || face < 0 || face > PFnone) { if (err) *err = "state or face out of range"; return -6; }
  const int rc = derive_surface_params(sim, err);
  if (rc) return rc;
  const SurfaceDef &sf = sim.surfaces[s];
  *act = eff_act(sf, i, ms, face);
  const SrfDetail *d = find_detail(sf, i, ms, face);
  for (int k = 0; k < 6; ++k) {
    prob[k] = d ? d->prob[k] : 0;
    cum[k] = d ? d->cum[k] : 0;
    rev[k] = d ? d->rev[k] : 0;
  }
  return 0;
}

// Device rule table and the panels' surface, neighbour and hop data.
int build_surface_rules(const Sim &sim, NetSpec *net, std::string *err) {
  net->bound = surface_bound_mode(sim) ? 1 : 0;
  if (!net->bound) return 0;
  const int ns = (int)sim.species.size(), nsrf = (int)sim.surfaces.size();
  net->nsrf = nsrf;
  net->srf_rules.assign((size_t)std::max(1, nsrf) * kMaxSpecies * 9, SrfRule{});
  for (int s = 0; s < nsrf; ++s) {
    const SurfaceDef &sf = sim.surfaces[s];
    for (int i = 0; i < ns && i < kMaxSpecies; ++i)
      for (int ms = 0; ms < kSrfStates; ++ms)
        for (int f = 0; f < 3; ++f) {
          SrfRule &r = net->srf_rules[((size_t)(s * kMaxSpecies + i) * 3 + ms) * 3 + f];
          r.act = (int8_t)eff_act(sf, i, ms, f);
          if (r.act == SAport) { if (err) *err = "port surface actions are not supported by the GPU engine"; return -6; }
          if (r.act == SAjump && ms != MSsoln) { if (err) *err = "the jump action applies to solution molecules"; return -6; }
          const SrfDetail *d = find_detail(sf, i, ms, f);
          r.rev = 0;
          for (int k = 0; k < 6; ++k) {
            r.newspec[k] = (int8_t)(d ? d->newspec[k] : i);
            r.cum[k] = d ? d->cum[k] : 0.0;
            if (d && d->rev[k] > 0) r.rev |= (uint8_t)(1u << k);
          }
        }
  }
  for (int i = 0; i < ns && i < kMaxSpecies; ++i)
    for (int k = 0; k < 2; ++k) net->difc_bound[i][k] = sim.species[i].difc_bound[k];

  net->srf_eps = sim.srf_epsilon;
  net->srf_margin = sim.srf_margin;
  net->srf_neighdist = sim.srf_neighdist;
  std::vector<int> first(nsrf);
  for (int s = 0, k = 0; s < nsrf; ++s) { first[s] = k; k += (int)sim.surfaces[s].panels.size(); }
  for (int s = 0, k = 0; s < nsrf; ++s) {
    const SurfaceDef &sf = sim.surfaces[s];
    for (size_t q = 0; q < sf.panels.size(); ++q, ++k) {
      PanelSpec &ps = net->panels[k];
      ps.srf = s;
      ps.neighhop = sf.neighhop;
      ps.nneigh = 0;
      if (q < sf.neigh.size())
        for (const auto &nb : sf.neigh[q])
          if (ps.nneigh < kMaxNeigh) ps.neigh[ps.nneigh++] = first[nb.first] + nb.second;
    }
  }
  return 0;
}

}  // namespace smolb
