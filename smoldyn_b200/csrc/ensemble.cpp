// Ensembles: many independent replicates of one reaction network in a single
// engine (one launch sequence, one CUDA graph, for all replicates).
//
// The template simulation fixes species, reactions, product placement, walls,
// dt and seed.  Each replicate may override its box and the rate constants;
// rate-derived parameters are recomputed per replicate with the same
// derivation as a single simulation (smolreact.c:1307-1577), either on the
// host, on the device (exact FP64, one thread per replicate), or by the MLP
// surrogate with exact fallback.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/smoldyn_b200.h"
#include "autotune.h"
#include "engine.h"
#include "rxnparam.cuh"
#include "sim.h"
#include "surrogate.h"

struct smolb_sim {
  smolb::Sim s;
};

struct smolb_ens {
  smolb::Sim templ;
  int nrep = 0;
  std::vector<std::array<double, 3>> lo, hi;
  std::map<std::string, std::vector<double>> rates;   // per-replicate rate overrides
  std::vector<std::vector<int>> counts;               // [species][rep]
  std::unique_ptr<smolb::Engine> eng;
  std::vector<smolb::RepSpec> reps;
  smolb::NetSpec net;
  int radius_mode = 1;  // 0 host exact, 1 device exact, 2 surrogate with exact fallback
  bool need_update = true, need_rebuild = true;
  long long rng_steps = 0;  // steps run by earlier engines of this ensemble (random streams continue past them)
  // per-replicate derived pair parameters, [r2][rep]
  std::vector<std::vector<double>> bindrad, unbindrad;
  long long surrogate_fallbacks = 0;
  std::unique_ptr<smolb::Surrogate> sur;
  smolb::LaunchTuning tuning;  // kernel launch shape (autotuner)
  int engine_mode = 0;         // 0 automatic (the step pipeline, measured faster), 1 step pipeline, 2 persistent kernel
};

// process-global error record of the C API (api.cpp)
ErrorCode smolb_record_error(const char *, ErrorCode, const std::string &);
smolb::Surrogate *smolb_surrogate_clone(surptr);

namespace {
ErrorCode ens_error(const char *func, ErrorCode code, const std::string &msg) {
  return smolb_record_error(func, code, msg);
}

#define ECHECK(cond, code, msg)                             \
  do {                                                      \
    if (!(cond)) return ens_error(__func__, code, msg);     \
  } while (0)

// rate of reaction (order, r) for replicate k
double rate_of(const smolb_ens &e, int order, int r, int k) {
  const smolb::RxnDef &x = e.templ.rxn[order][r];
  auto it = e.rates.find(x.name);
  if (it != e.rates.end()) return it->second[k];
  return x.rate;
}

// Virtual boxes per replicate (smolboxes.c:717-749 rule, one binding radius
// wide at least), from the molecule count and the box-size setting (the
// autotuner's choice when the template sets neither molperbox nor boxsize).
void assign_boxes(smolb_ens &e) {
  const smolb::Sim &T = e.templ;
  const int R = e.nrep;
  for (int k = 0; k < R; ++k) {
    smolb::RepSpec &s = e.reps[k];
    long long n = 0;
    for (size_t sp = 1; sp < e.counts.size(); ++sp) n += e.counts[sp][k];
    double mpbox = T.molperbox, boxsize = T.boxsize;
    if (mpbox <= 0 && boxsize <= 0) mpbox = T.auto_molperbox > 0 ? T.auto_molperbox : 4;
    double vol = 1;
    for (int d = 0; d < T.dim; ++d) vol *= s.hi[d] - s.lo[d];
    const double f = (mpbox > 0) ? std::pow((double)std::max<long long>(n, 1) / mpbox / vol, 1.0 / T.dim) : 1.0 / boxsize;
    double maxrad = 0;
    for (size_t r = 0; r < T.rxn[2].size(); ++r) maxrad = std::max(maxrad, std::sqrt(s.bind2[r]));
    for (int d = 0; d < 3; ++d) {
      if (d >= T.dim) { s.ncell[d] = 1; continue; }
      const double L = s.hi[d] - s.lo[d];
      int nn = std::max(1, (int)std::ceil(L * f));
      if (maxrad > 0 && L / nn < maxrad) nn = std::max(1, (int)std::floor(L / maxrad));
      s.ncell[d] = std::min(nn, 1023);
    }
  }
}

// Derive every replicate's parameters (rates, radii, boxes) into e.reps.
int derive(smolb_ens &e, std::string *err) {
  smolb::Sim &T = e.templ;
  if (T.dt <= 0) { *err = "time step must be > 0"; return -8; }
  if (smolb::derive_reaction_params(T, err)) return -8;  // placement defaults, rate-free parts
  smolb::RepSpec base;
  if (smolb::build_engine_specs(T, &e.net, &base, err)) return -6;
  const int R = e.nrep;
  // A rate update of a built ensemble keeps each replicate's rate-free fields
  // and rewrites the rate-dependent ones below; copying the template's whole
  // parameter set into every replicate dominated the update time of large
  // ensembles.
  if (e.need_rebuild || !e.eng || (int)e.reps.size() != R) e.reps.assign(R, base);
  const double dt = T.dt;
  // zeroth and first order, per replicate (same formulas as derive_reaction_params)
  for (int k = 0; k < R; ++k) {
    smolb::RepSpec &s = e.reps[k];
    double vol = 1;
    for (int d = 0; d < 3; ++d) {
      s.lo[d] = (d < T.dim) ? e.lo[k][d] : 0;
      s.hi[d] = (d < T.dim) ? e.hi[k][d] : 1;
      if (d < T.dim) vol *= s.hi[d] - s.lo[d];
    }
    for (size_t r = 0; r < T.rxn[0].size(); ++r) s.birth_mean[r] = rate_of(e, 0, (int)r, k) * dt * vol;
    for (size_t r = 0; r < T.rxn[1].size(); ++r) {
      const int i = T.rxn[1][r].rct[0];
      const double rt = rate_of(e, 1, (int)r, k);
      if (rt <= 0) { s.uni_prob[r] = 0; continue; }
      double sum = 0;
      for (size_t q = 0; q < T.rxn[1].size(); ++q)
        if (T.rxn[1][q].rct[0] == i && rate_of(e, 1, (int)q, k) > 0) sum += rate_of(e, 1, (int)q, k);
      double pr = rt / sum * (1.0 - std::exp(-sum * dt)), product = 1.0;
      for (size_t q = 0; q < r; ++q) {
        if (T.rxn[1][q].rct[0] != i) continue;
        const double pq = s.uni_prob[q] * product;
        product *= 1.0 - pq;
      }
      s.uni_prob[r] = pr / product;
    }
  }
  // second order: binding radii and reverse unbinding radii
  e.bindrad.assign(T.rxn[2].size(), std::vector<double>(R, 0));
  e.unbindrad.assign(T.rxn[2].size(), std::vector<double>(R, 0));
  e.surrogate_fallbacks = 0;
  for (size_t r = 0; r < T.rxn[2].size(); ++r) {
    const smolb::RxnDef &x = T.rxn[2][r];
    int o2 = 0, r2 = 0;
    const int rev = smolb::find_reverse_rxn(T, 2, (int)r, &o2, &r2);
    const bool direct = (rev == 1 && o2 == 1);
    const int rpt = direct ? T.rxn[1][r2].rparamt : 0;
    const double rpar = direct ? T.rxn[1][r2].rparam : 0;
    const double dsum = T.species[x.rct[0]].difc + T.species[x.rct[1]].difc;
    const int same = x.rct[0] == x.rct[1];
    std::vector<double> kf(R), ds(R, dsum), b(R), u(R);
    std::vector<int> ev(R, 0);
    for (int k = 0; k < R; ++k) kf[k] = rate_of(e, 2, (int)r, k);
    if (x.bindrad_user >= 0) {
      std::fill(b.begin(), b.end(), x.bindrad_user);
    } else if (e.radius_mode == 0) {
      for (int k = 0; k < R; ++k) {
        const smolb::rxnp::PairRadii pr = smolb::rxnp::pair_radii(kf[k], same, dsum, dt, direct, rpt, rpar);
        b[k] = pr.bindrad;
        u[k] = pr.unbindrad;
        ev[k] = pr.err;
      }
    } else if (e.radius_mode == 1) {
      if (smolb::solve_pair_radii_device(R, kf.data(), ds.data(), dt, same, direct, rpt, rpar, b.data(), u.data(),
                                         ev.data(), err))
        return -8;
    } else {
      if (!e.sur || !e.sur->trained()) { *err = "surrogate not trained (smolgpuSurrogateTrain)"; return -8; }
      long long nfb = 0;
      if (e.sur->pair_radii(R, kf.data(), ds.data(), dt, same, direct, rpt, rpar, b.data(), u.data(), &nfb, err))
        return -8;
      e.surrogate_fallbacks += nfb;
    }
    for (int k = 0; k < R; ++k) {
      if (ev[k] == 2) { *err = "reaction " + x.name + ": requested geminate probability unreachable"; return -8; }
      if (ev[k]) { *err = "reaction " + x.name + ": illegal radius inputs"; return -8; }
      e.reps[k].bind2[r] = b[k] * b[k];
      e.bindrad[r][k] = b[k];
      e.unbindrad[r][k] = u[k];
      if (direct) {
        // products of the reverse split by D (smolreact.c:1545-1548)
        const smolb::RxnDef &y = T.rxn[1][r2];
        double dc1 = T.species[y.prd[0]].difc, dc2 = T.species[y.prd[1]].difc;
        const double dd = dc1 + dc2;
        if (dd == 0) dc1 = dc2 = 0.5;
        else { dc1 /= dd; dc2 /= dd; }
        for (int q = 0; q < smolb::kMaxProd; ++q)
          for (int d = 0; d < 3; ++d) e.reps[k].prdpos[1][r2][q][d] = 0;
        e.reps[k].prdpos[1][r2][0][0] = u[k] * dc1;
        e.reps[k].prdpos[1][r2][1][0] = -u[k] * dc2;
      }
    }
  }
  assign_boxes(e);
  return 0;
}

int build(smolb_ens &e, std::string *err) {
  int rc = derive(e, err);
  if (rc) return rc;
  const smolb::Sim &T = e.templ;
  if (!e.need_rebuild && e.eng) return e.eng->update_reps(e.reps, err);
  long long total = 0;
  for (size_t sp = 1; sp < e.counts.size(); ++sp)
    for (int k = 0; k < e.nrep; ++k) total += e.counts[sp][k];
  const long long cap = T.max_mol > 0 ? T.max_mol : std::max<long long>(2 * total + 4096, total + (1 << 20));
  if (e.eng) e.rng_steps += e.eng->steps_done();
  e.eng.reset(new smolb::Engine());
  rc = e.eng->init(e.net, e.reps, T.dt, (uint64_t)T.seed, cap, err);
  if (!rc) rc = e.eng->set_tuning(e.tuning, err);
  if (!rc) rc = e.eng->set_persistent(e.engine_mode == 2 ? 1 : 0, err);
  if (rc) return rc;
  if (e.engine_mode == 2 && !e.eng->persistent_active()) {
    *err = "the persistent kernel does not cover surfaces, compartments or injected displacements";
    return -6;
  }
  std::vector<double> pos;
  std::vector<int> sp, rep;
  pos.reserve(3 * total);
  sp.reserve(total);
  rep.reserve(total);
  smolb::Sim &M = e.templ;
  for (int k = 0; k < e.nrep; ++k)
    for (size_t s = 1; s < e.counts.size(); ++s)
      for (int m = 0; m < e.counts[s][k]; ++m) {
        for (int d = 0; d < 3; ++d)
          pos.push_back(d < M.dim ? e.lo[k][d] + M.rand_u01() * (e.hi[k][d] - e.lo[k][d]) : 0.0);
        sp.push_back((int)s);
        rep.push_back(k);
      }
  rc = e.eng->set_molecules((long long)sp.size(), pos.data(), sp.data(), rep.data(), nullptr, err);
  if (!rc && e.rng_steps > 0) rc = e.eng->set_rng_step((uint64_t)e.rng_steps, err);
  if (rc) return rc;
  e.need_rebuild = false;
  return 0;
}
}  // namespace

extern "C" {

ensptr smolgpuNewEnsemble(simptr templ, int nrep) {
  if (!templ) { ens_error(__func__, ECmissing, "missing template sim"); return nullptr; }
  if (nrep < 1 || nrep > 65536) { ens_error(__func__, ECbounds, "nrep must be 1..65536"); return nullptr; }
  ensptr e = new smolb_ens();
  const smolb::Sim &S = templ->s;
  // copy the definition, not the engine or molecules
  smolb::Sim &T = e->templ;
  T.dim = S.dim;
  for (int d = 0; d < 3; ++d) { T.lo[d] = S.lo[d]; T.hi[d] = S.hi[d]; T.btype[d][0] = S.btype[d][0]; T.btype[d][1] = S.btype[d][1]; }
  T.species = S.species;
  for (int o = 0; o < 3; ++o) T.rxn[o] = S.rxn[o];
  T.surfaces = S.surfaces;
  T.cmpts = S.cmpts;
  T.tstart = S.tstart; T.tstop = S.tstop; T.dt = S.dt; T.time = S.time;
  T.seed = S.seed;
  T.host_rng = S.host_rng;
  T.molperbox = S.molperbox; T.boxsize = S.boxsize;
  T.gauss_table_size = S.gauss_table_size;
  T.max_mol = S.max_mol;
  e->nrep = nrep;
  e->lo.assign(nrep, {S.lo[0], S.lo[1], S.lo[2]});
  e->hi.assign(nrep, {S.hi[0], S.hi[1], S.hi[2]});
  e->counts.assign(S.species.size(), std::vector<int>(nrep, 0));
  return e;
}

enum ErrorCode smolgpuEnsembleSetBoxes(ensptr ens, const double *low, const double *high) {
  ECHECK(ens && low && high, ECmissing, "missing argument");
  const int dim = ens->templ.dim;
  for (int k = 0; k < ens->nrep; ++k)
    for (int d = 0; d < dim; ++d) {
      ECHECK(low[k * dim + d] < high[k * dim + d], ECbounds, "low must be < high");
      ens->lo[k][d] = low[k * dim + d];
      ens->hi[k][d] = high[k * dim + d];
    }
  ens->need_rebuild = true;
  return ECok;
}

enum ErrorCode smolgpuEnsembleSetRates(ensptr ens, const char *reaction, const double *rates) {
  ECHECK(ens && reaction && rates, ECmissing, "missing argument");
  ECHECK(ens->templ.reaction_index(reaction, nullptr) >= 0, ECnonexist, "reaction not found");
  for (int k = 0; k < ens->nrep; ++k) ECHECK(rates[k] >= 0, ECbounds, "rates must be >= 0");
  ens->rates[reaction].assign(rates, rates + ens->nrep);
  ens->need_update = true;
  return ECok;
}

enum ErrorCode smolgpuEnsembleAddMolecules(ensptr ens, const char *species, const int *counts) {
  ECHECK(ens && species && counts, ECmissing, "missing argument");
  const int i = ens->templ.species_index(species);
  ECHECK(i > 0, ECnonexist, "species not found");
  for (int k = 0; k < ens->nrep; ++k) {
    ECHECK(counts[k] >= 0, ECbounds, "counts must be >= 0");
    ens->counts[i][k] += counts[k];
  }
  ens->need_rebuild = true;
  return ECok;
}

enum ErrorCode smolgpuEnsembleSetRadiusMode(ensptr ens, int mode) {
  ECHECK(ens, ECmissing, "missing ensemble");
  ECHECK(mode >= 0 && mode <= 2, ECbounds, "mode must be 0, 1 or 2");
  ens->radius_mode = mode;
  ens->need_update = true;
  return ECok;
}

enum ErrorCode smolgpuEnsembleSetEngine(ensptr ens, int mode) {
  ECHECK(ens, ECmissing, "missing ensemble");
  ECHECK(mode >= 0 && mode <= 2, ECbounds, "mode must be 0, 1 or 2");
  ens->engine_mode = mode;
  if (ens->eng) {
    std::string err;
    if (ens->eng->set_persistent(mode == 2 ? 1 : 0, &err)) return ens_error(__func__, ECerror, err);
    ECHECK(mode != 2 || ens->eng->persistent_active(), ECerror,
           "the persistent kernel does not cover surfaces, compartments or injected displacements");
  }
  return ECok;
}

int smolgpuEnsembleGetEngine(ensptr ens) {
  if (!ens) return (int)ens_error(__func__, ECmissing, "missing ensemble");
  if (!ens->eng) return ens->engine_mode == 2 ? 2 : 1;
  return ens->eng->persistent_active() ? 2 : 1;
}

enum ErrorCode smolgpuEnsembleUpdate(ensptr ens) {
  ECHECK(ens, ECmissing, "missing ensemble");
  std::string err;
  if (build(*ens, &err)) return ens_error(__func__, ECerror, err);
  ens->need_update = false;
  return ECok;
}

enum ErrorCode smolgpuEnsembleRunSteps(ensptr ens, long long nsteps) {
  ECHECK(ens, ECmissing, "missing ensemble");
  std::string err;
  if (ens->need_update || ens->need_rebuild || !ens->eng) {
    if (build(*ens, &err)) return ens_error(__func__, ECerror, err);
    ens->need_update = false;
  }
  if (ens->eng->run(nsteps, &err)) return ens_error(__func__, ECerror, err);
  return ECok;
}

enum ErrorCode smolgpuEnsembleGetCounts(ensptr ens, long long *counts) {
  ECHECK(ens && counts, ECmissing, "missing argument");
  ECHECK(ens->eng, ECerror, "ensemble not built");
  std::vector<long long> c;
  std::string err;
  if (ens->eng->species_counts(&c, &err)) return ens_error(__func__, ECerror, err);
  memcpy(counts, c.data(), c.size() * sizeof(long long));
  return ECok;
}

enum ErrorCode smolgpuEnsembleGetEventCounts(ensptr ens, long long counts[8]) {
  ECHECK(ens && counts, ECmissing, "missing argument");
  for (int k = 0; k < 8; ++k) counts[k] = 0;
  if (!ens->eng) return ECok;
  smolb::EngineStats st;
  std::string err;
  if (ens->eng->stats(&st, &err)) return ens_error(__func__, ECerror, err);
  counts[0] = st.wall; counts[1] = st.rxn0; counts[2] = st.rxn1; counts[3] = st.rxn2;
  counts[4] = st.unresolved; counts[5] = st.multicand; counts[6] = st.overflow;
  return ECok;
}

enum ErrorCode smolgpuEnsembleGetMolecules(ensptr ens, long long *n, double *pos, int *species, int *rep,
                                           uint64_t *serno) {
  ECHECK(ens && n, ECmissing, "missing argument");
  ECHECK(ens->eng, ECerror, "ensemble not built");
  std::vector<double> p;
  std::vector<int> sp, rp;
  std::vector<uint64_t> sn;
  std::string err;
  if (ens->eng->get_molecules(&p, &sp, &rp, &sn, &err)) return ens_error(__func__, ECerror, err);
  const long long cnt = (long long)sp.size();
  ECHECK(*n >= cnt || (!pos && !species && !rep && !serno), ECbounds, "buffer too small");
  *n = cnt;
  if (pos) memcpy(pos, p.data(), p.size() * sizeof(double));
  if (species) memcpy(species, sp.data(), sp.size() * sizeof(int));
  if (rep) memcpy(rep, rp.data(), rp.size() * sizeof(int));
  if (serno) memcpy(serno, sn.data(), sn.size() * sizeof(uint64_t));
  return ECok;
}

enum ErrorCode smolgpuEnsembleGetReactionParams(ensptr ens, const char *reaction, double *bindrad,
                                                double *unbindrad) {
  ECHECK(ens && reaction, ECmissing, "missing argument");
  int o;
  const int r = ens->templ.reaction_index(reaction, &o);
  ECHECK(r >= 0 && o == 2, ECnonexist, "bimolecular reaction not found");
  if (ens->need_update || ens->bindrad.empty()) {
    std::string err;
    if (derive(*ens, &err)) return ens_error(__func__, ECerror, err);
  }
  for (int k = 0; k < ens->nrep; ++k) {
    if (bindrad) bindrad[k] = ens->bindrad[r][k];
    if (unbindrad) unbindrad[k] = ens->unbindrad[r][k];
  }
  return ECok;
}

long long smolgpuEnsembleGetFallbackCount(ensptr ens) { return ens ? ens->surrogate_fallbacks : -1; }

enum ErrorCode smolgpuEnsembleSetStream(ensptr ens, void *stream) {
  ECHECK(ens, ECmissing, "missing ensemble");
  std::string err;
  if (!ens->eng) {
    if (build(*ens, &err)) return ens_error(__func__, ECerror, err);
    ens->need_update = false;
  }
  ens->eng->set_stream(stream);
  return ECok;
}

enum ErrorCode smolgpuEnsembleAutotune(ensptr ens, int trial_steps, double *ms_per_step) {
  ECHECK(ens, ECmissing, "missing ensemble");
  ECHECK(trial_steps >= 2 && trial_steps <= 100000, ECbounds, "trial_steps must be 2..100000");
  std::string err;
  if (build(*ens, &err)) return ens_error(__func__, ECerror, err);
  ECHECK(ens->eng->steps_done() == 0, ECerror, "autotune runs before the first time step");
  std::vector<double> pos;
  std::vector<int> sp, rep;
  std::vector<uint64_t> serno;
  if (ens->eng->get_molecules(&pos, &sp, &rep, &serno, &err)) return ens_error(__func__, ECerror, err);
  smolb::Sim &T = ens->templ;
  const bool box_free = T.molperbox <= 0 && T.boxsize <= 0;
  smolb::TuneSetup ts;
  if (box_free) ts.box_candidates = {1, 2, 4, 8};
  ts.box_default = T.auto_molperbox > 0 ? T.auto_molperbox : 4;
  ts.engine = [&]() { return ens->eng.get(); };
  ts.rebuild = [&](double mpb, std::string *e) -> int {
    if (box_free) T.auto_molperbox = mpb;
    assign_boxes(*ens);
    const long long n = (long long)sp.size();
    const long long cap = T.max_mol > 0 ? T.max_mol : std::max<long long>(2 * n + 4096, n + (1 << 20));
    const smolb::LaunchTuning keep = ens->eng->tuning();
    int rc = ens->eng->init(ens->net, ens->reps, T.dt, (uint64_t)T.seed, cap, e);
    if (!rc) rc = ens->eng->set_tuning(keep, e);
    if (!rc) rc = ens->eng->set_molecules(n, pos.data(), sp.data(), rep.data(), serno.data(), e);
    return rc;
  };
  smolb::TuneResult tr;
  if (smolb::autotune(ts, trial_steps, &tr, &err)) return ens_error(__func__, ECerror, err);
  ens->tuning = tr.launch;
  if (box_free) T.auto_molperbox = tr.molperbox;
  if (ms_per_step) *ms_per_step = tr.ms_per_step;
  return ECok;
}

enum ErrorCode smolgpuEnsembleGetTuning(ensptr ens, double *molperbox, int *pair_tile, int *tile_blocks_per_sm,
                                        int *mol_blocks_per_sm) {
  ECHECK(ens, ECmissing, "missing ensemble");
  const smolb::Sim &T = ens->templ;
  if (molperbox)
    *molperbox = T.molperbox > 0 ? T.molperbox : (T.boxsize > 0 ? -1 : (T.auto_molperbox > 0 ? T.auto_molperbox : 4));
  if (pair_tile) *pair_tile = ens->tuning.pair_tile;
  if (tile_blocks_per_sm) *tile_blocks_per_sm = ens->tuning.tile_blocks_per_sm;
  if (mol_blocks_per_sm) *mol_blocks_per_sm = ens->tuning.mol_blocks_per_sm;
  return ECok;
}

long long smolgpuEnsembleGetLaunchCount(ensptr ens) { return (ens && ens->eng) ? ens->eng->launches() : 0; }

enum ErrorCode smolgpuEnsembleSynchronize(ensptr ens) {
  ECHECK(ens, ECmissing, "missing ensemble");
  if (!ens->eng) return ECok;
  std::string err;
  if (ens->eng->synchronize(&err)) return ens_error(__func__, ECerror, err);
  return ECok;
}

enum ErrorCode smolgpuEnsembleAttachSurrogate(ensptr ens, surptr sur) {
  ECHECK(ens && sur, ECmissing, "missing argument");
  ens->sur.reset(smolb_surrogate_clone(sur));
  ens->need_update = true;
  return ECok;
}

enum ErrorCode smolgpuEnsembleFree(ensptr ens) {
  delete ens;
  return ECok;
}

}  // extern "C"
