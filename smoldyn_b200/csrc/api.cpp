// libsmoldyn-compatible C API (source/Smoldyn/libsmoldyn.h subset) over the
// B200 engine, plus the smolgpu* extensions.  Error reporting follows
// libsmoldyn.cpp:23-37: every failing call records (function, code, message)
// in process-global state read by smolGetError.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/smoldyn_b200.h"
#include "autotune.h"
#include "engine.h"
#include "rxnparam.cuh"
#include "sim.h"

struct smolb_sim {
  smolb::Sim s;
};

using smolb::Sim;

namespace {
std::mutex g_err_mu;
ErrorCode g_errcode = ECok;
std::string g_errfunc, g_errstr;
int g_debug = 0;

ErrorCode set_error(const char *func, ErrorCode code, const std::string &msg) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_errcode = code;
  g_errfunc = func;
  g_errstr = msg;
  if (g_debug && code < ECwarning) fprintf(stderr, "libsmoldyn_b200 %s: %s\n", func, msg.c_str());
  return code;
}

ErrorCode from_rc(int rc) {
  if (rc >= 0) return ECok;
  if (rc < ECwildcard) return ECerror;
  return (ErrorCode)rc;
}

#define LCHECK(cond, code, msg)                    \
  do {                                             \
    if (!(cond)) return set_error(__func__, code, msg); \
  } while (0)

long long total_pending(const Sim &s) { return (long long)s.pend_sp.size(); }

// Bring every registered meansqrdisp tracker up to date and copy its last
// unwrapped positions to the host, before the engine is re-initialised.
int msd_save(Sim &s, std::string *err) {
  if (!s.eng) return 0;
  for (auto &kv : s.msd) {
    smolb::MsdState &m = kv.second;
    if (m.handle < 0) continue;
    int rc = s.eng->msd_update(m.handle, -1, nullptr, nullptr, nullptr, err);
    if (!rc) rc = s.eng->msd_last(m.handle, &m.last, err);
    if (rc) return rc;
    m.handle = -1;
    m.since = 0;
  }
  return 0;
}

// Download molecules from the engine into the pending lists (before a
// rebuild); serial numbers are kept, as the reference keeps them.
int pull_molecules(Sim &s, std::string *err) {
  if (!s.eng || !s.started) return 0;
  int rc = msd_save(s, err);
  if (rc) return rc;
  std::vector<double> pos;
  std::vector<int> sp, rep;
  std::vector<uint64_t> serno;
  rc = s.eng->get_molecules(&pos, &sp, &rep, &serno, err);
  if (rc) return rc;
  s.pend_pos = pos;
  s.pend_sp = sp;
  s.pend_serno = serno;
  // surface-bound molecules: engine panel index back to (surface, panel)
  std::vector<double> bpos;
  std::vector<int> bsp, bst, bpn;
  std::vector<uint64_t> bsn;
  rc = s.eng->get_bound(&bpos, &bsp, &bst, &bpn, &bsn, err);
  if (rc) return rc;
  s.pend_bound.clear();
  for (size_t k = 0; k < bsp.size(); ++k) {
    smolb::PendBound b;
    for (int d = 0; d < 3; ++d) b.pos[d] = bpos[3 * k + d];
    b.species = bsp[k];
    b.state = bst[k];
    b.serno = bsn[k];
    int g = bpn[k];
    for (size_t q = 0; q < s.surfaces.size(); ++q) {
      if (g < (int)s.surfaces[q].panels.size()) { b.surface = (int)q; b.panel = g; break; }
      g -= (int)s.surfaces[q].panels.size();
    }
    s.pend_bound.push_back(b);
  }
  s.started = false;
  return 0;
}

// Upload the pending surface-bound molecules into a freshly built engine;
// molecules without a serial number get ones after every solution molecule's.
int push_bound(Sim &s, long long nsol, std::string *err) {
  uint64_t base = (uint64_t)nsol + 1;
  for (uint64_t v : s.pend_serno) base = std::max<uint64_t>(base, v + 1);
  for (const smolb::PendBound &b : s.pend_bound) base = std::max<uint64_t>(base, b.serno + 1);
  std::vector<double> pos;
  std::vector<int> sp, st, pn;
  std::vector<uint64_t> sn;
  std::vector<int> first(s.surfaces.size());
  for (size_t q = 0, k = 0; q < s.surfaces.size(); ++q) { first[q] = (int)k; k += s.surfaces[q].panels.size(); }
  for (const smolb::PendBound &b : s.pend_bound) {
    for (int d = 0; d < 3; ++d) pos.push_back(b.pos[d]);
    sp.push_back(b.species);
    st.push_back(b.state);
    pn.push_back(first[b.surface] + b.panel);
    sn.push_back(b.serno ? b.serno : base++);
  }
  const int rc = s.eng->set_bound((long long)sp.size(), pos.data(), sp.data(), st.data(), pn.data(), sn.data(), err);
  if (!rc) s.pend_bound.clear();
  return rc;
}

// simupdate equivalent: derive parameters, (re)build the engine, upload molecules.
ErrorCode update_sim(Sim &s, const char *func) {
  std::string err;
  if (!s.need_update && !s.need_rebuild && s.eng) return ECok;
  if (s.dt <= 0) return set_error(func, ECerror, "time step must be > 0");
  if (s.need_rebuild && s.eng && s.started) {
    if (pull_molecules(s, &err)) return set_error(func, ECerror, err);
  }
  int rc = smolb::derive_reaction_params(s, &err);
  if (rc) return set_error(func, ECerror, err);
  smolb::NetSpec net;
  smolb::RepSpec rep;
  rc = smolb::build_engine_specs(s, &net, &rep, &err);
  if (rc) return set_error(func, from_rc(rc), err);
  if (s.need_rebuild || !s.eng) {
    long long n = total_pending(s);
    long long cap = s.max_mol > 0 ? s.max_mol : std::max<long long>(2 * n + 4096, n + (1 << 20));
    if (!s.eng) s.eng.reset(new smolb::Engine());
    rc = s.eng->init(net, {rep}, s.dt, (uint64_t)s.seed, cap, &err);
    if (!rc) rc = s.eng->set_tuning(s.tuning, &err);
    if (rc) { s.eng.reset(); return set_error(func, from_rc(rc), err); }
    std::vector<uint64_t> sn;
    if (!s.pend_serno.empty()) {  // serials kept from a pull; molecules added since get new ones
      sn.assign((size_t)n, 0);
      for (size_t k = 0; k < s.pend_serno.size() && k < sn.size(); ++k) sn[k] = s.pend_serno[k];
    }
    rc = s.eng->set_molecules(n, s.pend_pos.data(), s.pend_sp.data(), nullptr, sn.empty() ? nullptr : sn.data(), &err);
    if (!rc && (!s.pend_bound.empty() || net.bound)) rc = push_bound(s, n, &err);
    // a rebuild mid-run continues the random streams where they were
    if (!rc && s.steps > 0) rc = s.eng->set_rng_step((uint64_t)s.steps, &err);
    if (rc) { s.eng.reset(); return set_error(func, from_rc(rc), err); }
    s.pend_pos.clear();
    s.pend_sp.clear();
    s.pend_serno.clear();
    s.started = true;
  } else {
    rc = s.eng->update_reps({rep}, &err);
    if (rc) return set_error(func, from_rc(rc), err);
  }
  s.need_update = s.need_rebuild = false;
  return ECok;
}

void record_molcount(Sim &s, const std::string &dataname) {
  std::vector<long long> counts;
  std::string err;
  std::vector<double> row;
  row.push_back(s.time);
  if (s.eng && s.started && !s.eng->species_counts(&counts, &err)) {
    for (size_t i = 1; i < s.species.size(); ++i) row.push_back((double)counts[i]);
  } else {
    std::vector<long long> c(s.species.size(), 0);
    for (int sp : s.pend_sp) c[sp]++;
    for (size_t i = 1; i < s.species.size(); ++i) row.push_back((double)c[i]);
  }
  s.outdata[dataname].push_back(row);
}

// Steps over which a molecule of species sp stays within half a period of
// every periodic axis with overwhelming probability: 10 standard deviations
// of its diffusion plus its drift must stay below L/2.  0 when no axis wraps.
long long msd_interval(const Sim &s, int sp) {
  long long best = 0;
  const smolb::SpeciesDef &S = s.species[sp];
  for (int d = 0; d < s.dim; ++d) {
    if (s.btype[d][0] != 'p' || s.btype[d][1] != 'p') continue;
    double var = 2.0 * S.difc * s.dt;  // per-step variance along d
    if (S.has_difm) {
      var = 0;
      for (int k = 0; k < 3; ++k) var += 2.0 * s.dt * S.difm[3 * d + k] * S.difm[3 * d + k];
    }
    const double a = std::fabs(S.drift[d]) * s.dt, b = 10.0 * std::sqrt(var), c = (s.hi[d] - s.lo[d]) / 2.0;
    double rk;
    if (a > 0)
      rk = (-b + std::sqrt(b * b + 4 * a * c)) / (2 * a);
    else if (b > 0)
      rk = c / b;
    else
      continue;
    const long long k = std::max<long long>(1, (long long)std::floor(rk * rk));
    best = best ? std::min(best, k) : k;
  }
  return best;
}

// Register a tracker with the current engine if it has none yet.
int msd_register(Sim &s, smolb::MsdState &m, std::string *err) {
  if (m.handle >= 0) return 0;
  const int h = s.eng->msd_track(m.species, (long long)m.keys.size(), m.keys.data(), m.start.data(), m.last.data(), err);
  if (h < 0) return h;
  m.handle = h;
  m.since = 0;
  return 0;
}

// meansqrdisp species dim data (cmdmeansqrdisp, smolcmd.c:2505-2606): on the
// first run record the molecules of the species; on every run append
// (time, <r^2>, <r^4>) over those still present, r measured from the
// recorded positions with periodic wraps undone.
void record_meansqrdisp(Sim &s, const smolb::Command &c) {
  smolb::MsdState &m = s.msd[c.text];
  if (m.failed || !s.eng) return;
  std::string err;
  if (!m.started) {
    char name[256] = {0}, spn[256] = {0}, dimstr[256] = {0}, data[256] = {0};
    const int nw = sscanf(c.text.c_str(), "%255s %255s %255s %255s", name, spn, dimstr, data);
    std::string spname(spn);
    const size_t paren = spname.find('(');
    if (paren != std::string::npos) spname = spname.substr(0, paren);  // solution state only
    m.species = s.species_index(spname);
    const std::string ds(dimstr);
    m.msddim = ds == "all" ? -1 : (ds == "0" || ds == "x") ? 0 : (ds == "1" || ds == "y") ? 1 : (ds == "2" || ds == "z") ? 2 : 3;
    m.dataname = nw >= 4 ? data : "meansqrdisp";
    if (nw < 3 || m.species <= 0 || m.msddim >= s.dim) { m.failed = true; return; }
    std::vector<double> pos;
    std::vector<int> sp, rep;
    std::vector<uint64_t> sn;
    if (s.eng->get_molecules(&pos, &sp, &rep, &sn, &err)) { m.failed = true; return; }
    for (size_t i = 0; i < sp.size(); ++i) {
      if (sp[i] != m.species) continue;
      m.keys.push_back(((uint64_t)rep[i] << 42) | sn[i]);
      for (int d = 0; d < 3; ++d) m.start.push_back(pos[3 * i + d]);
    }
    if (m.keys.empty()) { m.failed = true; return; }  // "no molecules to track"
    m.last = m.start;
    m.every = msd_interval(s, m.species);
    m.started = true;
  }
  if (msd_register(s, m, &err)) { m.failed = true; return; }
  double s2 = 0, s4 = 0;
  long long cnt = 0;
  if (s.eng->msd_update(m.handle, m.msddim, &s2, &s4, &cnt, &err)) { m.failed = true; return; }
  m.since = 0;
  s.outdata[m.dataname].push_back({s.time, s2 / (double)cnt, s4 / (double)cnt});
}

// Advance n steps, in chunks short enough that every meansqrdisp tracker
// gets an unwrapping pass before its molecules can cross half a period.
int advance_steps(Sim &s, long long n, std::string *err) {
  while (n > 0) {
    long long k = n;
    for (auto &kv : s.msd) {
      const smolb::MsdState &m = kv.second;
      if (m.started && !m.failed && m.every > 0) k = std::min(k, std::max<long long>(1, m.every - m.since));
    }
    if (s.eng->run(k, err)) return -1;
    for (long long j = 0; j < k; ++j) s.time += s.dt;
    s.steps += k;
    n -= k;
    for (auto &kv : s.msd) {
      smolb::MsdState &m = kv.second;
      if (!m.started || m.failed || m.every <= 0) continue;
      m.since += k;
      if (m.since < m.every) continue;
      if (msd_register(s, m, err) || s.eng->msd_update(m.handle, -1, nullptr, nullptr, nullptr, err)) return -1;
      m.since = 0;
    }
  }
  return 0;
}

// Molecules of species idx (-1: all) in a state (MSall / MSsome: any state),
// solution molecules from the species counts less the bound ones; -1 on error.
long long species_state_count(Sim &s, int idx, int state, std::string *err) {
  long long n = 0, nb[3] = {0, 0, 0};  // all states, then bound molecules by state
  if (s.eng && s.started && !s.need_rebuild) {
    std::vector<long long> c;
    if (s.eng->species_counts(&c, err)) return -1;
    for (size_t i = 1; i < s.species.size(); ++i)
      if (idx < 0 || (int)i == idx) n += c[i];
    if (state != MSall && state != MSsome) {
      std::vector<double> bpos;
      std::vector<int> bsp, bst, bpn;
      std::vector<uint64_t> bsn;
      if (s.eng->get_bound(&bpos, &bsp, &bst, &bpn, &bsn, err)) return -1;
      for (size_t k = 0; k < bsp.size(); ++k)
        if ((idx < 0 || bsp[k] == idx) && bst[k] >= 1 && bst[k] <= 2) nb[bst[k]]++;
    }
  } else {
    for (int sp : s.pend_sp)
      if (idx < 0 || sp == idx) n++;
    for (const smolb::PendBound &b : s.pend_bound)
      if (idx < 0 || b.species == idx) { n++; nb[b.state]++; }
  }
  if (state == MSsoln) n -= nb[1] + nb[2];
  else if (state == MSfront) n = nb[1];
  else if (state == MSback) n = nb[2];
  return n;
}

// molcountincmpt compartment data (smolcmd.c:1054-1100): (time, count of
// each species in the compartment)
void record_molcountincmpt(Sim &s, const smolb::Command &c) {
  char name[256] = {0}, cm[256] = {0}, data[256] = {0};
  const int nw = sscanf(c.text.c_str(), "%255s %255s %255s", name, cm, data);
  const int ci = s.compartment_index(cm);
  if (nw < 2 || ci < 0 || !s.eng) return;
  std::vector<long long> counts;
  std::string err;
  if (s.eng->cmpt_counts(ci, &counts, &err)) return;
  std::vector<double> row;
  row.push_back(s.time);
  for (size_t i = 1; i < s.species.size(); ++i) row.push_back(i < counts.size() ? (double)counts[i] : 0.0);
  s.outdata[nw >= 3 ? data : "molcountincmpt"].push_back(row);
}

// molcountonsurf surface data (smolcmd.c:1236-1285): (time, count of each
// species bound to the surface's panels)
void record_molcountonsurf(Sim &s, const smolb::Command &c) {
  char name[256] = {0}, sn[256] = {0}, data[256] = {0};
  const int nw = sscanf(c.text.c_str(), "%255s %255s %255s", name, sn, data);
  if (nw < 2 || !s.eng) return;
  int si = -1;
  for (size_t k = 0; k < s.surfaces.size(); ++k)
    if (s.surfaces[k].name == sn) si = (int)k;
  if (si < 0) return;
  int first = 0;
  for (int k = 0; k < si; ++k) first += (int)s.surfaces[k].panels.size();
  const int last = first + (int)s.surfaces[si].panels.size();
  std::vector<double> bpos;
  std::vector<int> bsp, bst, bpn;
  std::vector<uint64_t> bsn;
  std::string err;
  if (s.eng->get_bound(&bpos, &bsp, &bst, &bpn, &bsn, &err)) return;
  std::vector<double> row(s.species.size(), 0.0);
  row[0] = s.time;
  for (size_t k = 0; k < bsp.size(); ++k)
    if (bpn[k] >= first && bpn[k] < last && bsp[k] > 0 && bsp[k] < (int)row.size()) row[bsp[k]] += 1;
  s.outdata[nw >= 3 ? data : "molcountonsurf"].push_back(row);
}

// molcountspecies species[(state)] data (smolcmd.c:1972-1992): (time, count
// of the species in that state; all states for "all")
void record_molcountspecies(Sim &s, const smolb::Command &c) {
  char name[256] = {0}, spn[256] = {0}, data[256] = {0};
  const int nw = sscanf(c.text.c_str(), "%255s %255s %255s", name, spn, data);
  if (nw < 2 || !s.eng) return;
  std::string nm = spn, st = "solution";
  const size_t paren = nm.find('(');
  if (paren != std::string::npos) {
    st = nm.substr(paren + 1, nm.find(')', paren) - paren - 1);
    nm = nm.substr(0, paren);
  }
  int ms = MSsoln;
  if (st == "front") ms = MSfront;
  else if (st == "back") ms = MSback;
  else if (st == "all") ms = MSall;
  else if (!(st == "solution" || st == "soln" || st == "fsoln" || st == "aq")) return;
  const int idx = nm == "all" ? -1 : s.species_index(nm);
  if (idx == 0 || (idx < 0 && nm != "all")) return;
  std::string err;
  const long long n = species_state_count(s, idx, ms, &err);
  s.outdata[nw >= 3 ? data : "molcountspecies"].push_back({s.time, (double)std::max(0ll, n)});
}

void run_command(Sim &s, const smolb::Command &c) {
  char name[256] = {0}, arg[256] = {0};
  if (sscanf(c.text.c_str(), "%255s %255s", name, arg) < 1) return;
  if (!strcmp(name, "molcount")) record_molcount(s, arg[0] ? arg : "molcount");
  else if (!strcmp(name, "meansqrdisp")) record_meansqrdisp(s, c);
  else if (!strcmp(name, "molcountincmpt")) record_molcountincmpt(s, c);
  else if (!strcmp(name, "molcountonsurf")) record_molcountonsurf(s, c);
  else if (!strcmp(name, "molcountspecies")) record_molcountspecies(s, c);
}

// runtime commands (smolcmd.c docommand subset: molcount, molcountincmpt,
// molcountonsurf, meansqrdisp)
void do_commands(Sim &s, bool at_start) {
  for (smolb::Command &c : s.cmds) {
    bool run = false;
    if (c.type == 'b') run = at_start;
    else if (c.type == 'a' || c.type == 'e') run = false;
    else if (c.type == 'E') run = true;
    else if (c.type == 'N' || c.type == 'n') run = (s.steps % std::max<long long>(1, c.every)) == 0;
    else if (c.type == 'i') {
      if (s.time + 1e-12 >= c.next && s.time <= c.off + 1e-12 && s.time + 1e-12 >= c.on) {
        run = true;
        c.next = std::max(c.next, c.on) + c.dt;
      }
    }
    if (!run) continue;
    run_command(s, c);
  }
}

void do_end_commands(Sim &s) {
  for (smolb::Command &c : s.cmds) {
    if (c.type != 'a' && c.type != 'e') continue;
    run_command(s, c);
  }
}

bool has_step_commands(const Sim &s) {
  for (const smolb::Command &c : s.cmds)
    if (c.type == 'E' || c.type == 'N' || c.type == 'n' || c.type == 'i') return true;
  return false;
}

// Run steps until time >= stop (smolsimulate loop, smolsim.cpp:2747-2760).
ErrorCode run_until(Sim &s, double stop, const char *func, bool one_step) {
  ErrorCode ec = update_sim(s, func);
  if (ec != ECok) return ec;
  std::string err;
  if (s.steps == 0 && !one_step) do_commands(s, true);
  if (s.steps == 0 && one_step && s.time == s.tstart) do_commands(s, true);
  const bool percmd = has_step_commands(s);
  long long n = 0;
  double t = s.time;
  if (one_step) n = 1;
  else
    while (t < stop) { t += s.dt; ++n; }
  if (!percmd) {
    if (n > 0 && advance_steps(s, n, &err)) return set_error(func, ECerror, err);
  } else {
    for (long long k = 0; k < n; ++k) {
      if (advance_steps(s, 1, &err)) return set_error(func, ECerror, err);
      do_commands(s, false);
    }
  }
  // a single step checks the previous step's status (no wait for this one);
  // longer runs and the end of the simulation check the current one
  const bool last = s.time >= s.tstop;
  const int st = (one_step && !last) ? s.eng->status_flags_lagged() : s.eng->status_flags();
  if (st) return set_error(func, ECerror, "engine capacity exceeded (status flags " + std::to_string(st) + ")");
  if (last) {
    do_end_commands(s);
    return set_error(func, ECnotify, "Simulation complete");
  }
  return ECok;
}
}  // namespace

extern "C" {

double smolGetVersion(void) { return 2.76; }

enum ErrorCode smolGetError(char *errorfunction, char *errorstring, int clearerror) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  const ErrorCode c = g_errcode;
  if (errorfunction) { strncpy(errorfunction, g_errfunc.c_str(), 255); errorfunction[255] = 0; }
  if (errorstring) { strncpy(errorstring, g_errstr.c_str(), 255); errorstring[255] = 0; }
  if (clearerror) { g_errcode = ECok; g_errfunc.clear(); g_errstr.clear(); }
  return c;
}

void smolClearError(void) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_errcode = ECok;
  g_errfunc.clear();
  g_errstr.clear();
}

void smolSetDebugMode(int debugmode) { g_debug = debugmode; }

char *smolErrorCodeToString(enum ErrorCode erc, char *string) {
  static const char *names[] = {"ok", "notify", "warning", "nonexistant", "all", "missing", "bounds",
                                "syntax", "error", "memory", "bug", "same", "wildcard"};
  const int k = -(int)erc;
  strcpy(string, (k >= 0 && k <= 12) ? names[k] : "unknown");
  return string;
}

simptr smolNewSim(int dim, double *lowbounds, double *highbounds) {
  if (dim < 1 || dim > 3) { set_error(__func__, ECbounds, "dim must be 1..3"); return nullptr; }
  if (!lowbounds || !highbounds) { set_error(__func__, ECmissing, "missing bounds"); return nullptr; }
  for (int d = 0; d < dim; ++d)
    if (!(lowbounds[d] < highbounds[d])) { set_error(__func__, ECbounds, "lowbounds must be < highbounds"); return nullptr; }
  simptr sim = new smolb_sim();
  sim->s.dim = dim;
  for (int d = 0; d < dim; ++d) {
    sim->s.lo[d] = lowbounds[d];
    sim->s.hi[d] = highbounds[d];
  }
  return sim;
}

enum ErrorCode smolUpdateSim(simptr sim) {
  LCHECK(sim, ECmissing, "missing sim");
  return update_sim(sim->s, __func__);
}

enum ErrorCode smolRunTimeStep(simptr sim) {
  LCHECK(sim, ECmissing, "missing sim");
  return run_until(sim->s, sim->s.time + sim->s.dt / 2, __func__, true);
}

enum ErrorCode smolRunSim(simptr sim) {
  LCHECK(sim, ECmissing, "missing sim");
  ErrorCode e = run_until(sim->s, sim->s.tstop, __func__, false);
  return e == ECnotify ? ECok : e;
}

enum ErrorCode smolRunSimUntil(simptr sim, double breaktime) {
  LCHECK(sim, ECmissing, "missing sim");
  ErrorCode e = run_until(sim->s, std::min(breaktime, sim->s.tstop), __func__, false);
  return e == ECnotify ? ECok : e;
}

enum ErrorCode smolFreeSim(simptr sim) {
  delete sim;
  return ECok;
}

simptr smolPrepareSimFromFile(const char *filepath, const char *filename, const char *flags) {
  simptr sim = nullptr;
  if (smolLoadSimFromFile(filepath, filename, &sim, flags) != ECok) return nullptr;
  if (smolUpdateSim(sim) != ECok) { delete sim; return nullptr; }
  return sim;
}

enum ErrorCode smolLoadSimFromFile(const char *filepath, const char *filename, simptr *simpointer,
                                   const char *flags) {
  LCHECK(filename && simpointer, ECmissing, "missing filename or sim pointer");
  bool fresh = (*simpointer == nullptr);
  if (fresh) *simpointer = new smolb_sim();
  Sim &s = (*simpointer)->s;
  if (flags) s.flags = flags;
  std::string err;
  int rc = smolb::load_config_file(s, filepath ? filepath : "", filename, &err);
  if (rc) {
    if (fresh) { delete *simpointer; *simpointer = nullptr; }
    return set_error(__func__, from_rc(rc), err);
  }
  return ECok;
}

enum ErrorCode smolReadConfigString(simptr sim, const char *statement, char *parameters) {
  LCHECK(sim && statement, ECmissing, "missing sim or statement");
  std::string err;
  int rc = smolb::read_config_statement(sim->s, statement, parameters ? parameters : "", &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  return ECok;
}

enum ErrorCode smolSetSimTimes(simptr sim, double timestart, double timestop, double timestep) {
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(timestep > 0, ECbounds, "timestep must be > 0");
  sim->s.tstart = sim->s.time = timestart;
  sim->s.tstop = timestop;
  if (sim->s.dt != timestep) sim->s.need_update = sim->s.need_rebuild = true;
  sim->s.dt = timestep;
  return ECok;
}
enum ErrorCode smolSetTimeStart(simptr sim, double t) { LCHECK(sim, ECmissing, "missing sim"); sim->s.tstart = t; return ECok; }
enum ErrorCode smolSetTimeStop(simptr sim, double t) { LCHECK(sim, ECmissing, "missing sim"); sim->s.tstop = t; return ECok; }
enum ErrorCode smolSetTimeNow(simptr sim, double t) { LCHECK(sim, ECmissing, "missing sim"); sim->s.time = t; return ECok; }
enum ErrorCode smolSetTimeStep(simptr sim, double t) {
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(t > 0, ECbounds, "timestep must be > 0");
  sim->s.dt = t;
  sim->s.need_update = sim->s.need_rebuild = true;
  return ECok;
}
enum ErrorCode smolSetRandomSeed(simptr sim, long int seed) {
  LCHECK(sim, ECmissing, "missing sim");
  sim->s.set_seed(seed);
  sim->s.need_rebuild = true;
  return ECok;
}
enum ErrorCode smolSetPartitions(simptr sim, const char *method, double value) {
  LCHECK(sim && method, ECmissing, "missing sim or method");
  if (!strcmp(method, "molperbox")) { sim->s.molperbox = value; sim->s.boxsize = -1; }
  else if (!strcmp(method, "boxsize")) { sim->s.boxsize = value; sim->s.molperbox = -1; }
  else return set_error(__func__, ECsyntax, "method must be molperbox or boxsize");
  sim->s.need_rebuild = true;
  return ECok;
}

enum ErrorCode smolAddOutputData(simptr sim, char *dataname) {
  LCHECK(sim && dataname, ECmissing, "missing sim or name");
  sim->s.outdata[dataname];
  return ECok;
}

enum ErrorCode smolAddCommandFromString(simptr sim, char *string) {
  LCHECK(sim && string, ECmissing, "missing sim or string");
  std::string err;
  int rc = smolb::read_config_statement(sim->s, "cmd", string, &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  return ECok;
}

enum ErrorCode smolGetOutputData(simptr sim, char *dataname, int *nrow, int *ncol, double **array, int erase) {
  LCHECK(sim && dataname && nrow && ncol && array, ECmissing, "missing argument");
  auto it = sim->s.outdata.find(dataname);
  LCHECK(it != sim->s.outdata.end(), ECnonexist, "no such output data");
  const auto &rows = it->second;
  *nrow = (int)rows.size();
  *ncol = rows.empty() ? 0 : (int)rows[0].size();
  double *a = (double *)calloc((size_t)(*nrow) * (*ncol) + 1, sizeof(double));
  LCHECK(a, ECmemory, "out of memory");
  for (int r = 0; r < *nrow; ++r)
    for (int c = 0; c < *ncol && c < (int)rows[r].size(); ++c) a[r * (*ncol) + c] = rows[r][c];
  *array = a;
  if (erase) it->second.clear();
  return ECok;
}

enum ErrorCode smolAddSpecies(simptr sim, const char *species, const char *mollist) {
  LCHECK(sim && species, ECmissing, "missing sim or species");
  if (mollist && mollist[0])  // libsmoldyn.cpp:811-814: the list must exist
    LCHECK(std::find(sim->s.mollists.begin(), sim->s.mollists.end(), mollist) != sim->s.mollists.end(), ECsame,
           "molecule list not recognized");
  LCHECK(sim->s.species_index(species) < 0, ECsame, "species already exists");
  LCHECK((int)sim->s.species.size() < smolb::kMaxSpecies, ECbounds, "too many species (max 31)");
  sim->s.species.push_back(smolb::SpeciesDef{species});
  sim->s.need_update = sim->s.need_rebuild = true;
  return ECok;
}

int smolGetSpeciesIndex(simptr sim, const char *species) {
  const int i = smolGetSpeciesIndexNT(sim, species);
  if (i < 0) set_error(__func__, ECnonexist, "species not found");
  return i;
}

int smolGetSpeciesIndexNT(simptr sim, const char *species) {
  if (!sim || !species) return (int)ECmissing;
  if (!strcmp(species, "all")) return (int)ECall;
  const int i = sim->s.species_index(species);
  return i < 0 ? (int)ECnonexist : i;
}

// ---- molecule lists (libsmoldyn.cpp:954-1035): names only ----
enum ErrorCode smolAddMolList(simptr sim, const char *mollist) {
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(mollist, ECmissing, "missing mollist");
  std::vector<std::string> &L = sim->s.mollists;
  if (std::find(L.begin(), L.end(), mollist) != L.end())
    return set_error(__func__, ECwarning, "molecule list name has already been used");
  L.push_back(mollist);
  return ECok;
}

int smolGetMolListIndexNT(simptr sim, const char *mollist) {
  if (!sim || !mollist) return (int)ECmissing;
  if (sim->s.mollists.empty()) return (int)ECnonexist;
  if (!strcmp(mollist, "all")) return (int)ECall;
  const std::vector<std::string> &L = sim->s.mollists;
  const auto it = std::find(L.begin(), L.end(), mollist);
  return it == L.end() ? (int)ECnonexist : (int)(it - L.begin());
}

int smolGetMolListIndex(simptr sim, const char *mollist) {
  const int ll = smolGetMolListIndexNT(sim, mollist);
  if (ll == (int)ECmissing) set_error(__func__, ECmissing, "missing sim or mollist");
  else if (ll == (int)ECall) set_error(__func__, ECall, "molecule list is 'all'");
  else if (ll < 0) set_error(__func__, ECnonexist, "list name not recognized");
  return ll;
}

char *smolGetMolListName(simptr sim, int mollistindex, char *mollist) {
  if (!sim || !mollist) { set_error(__func__, ECmissing, "missing sim or mollist"); return nullptr; }
  if (mollistindex < 0) { set_error(__func__, ECbounds, "mollistindex < 0"); return nullptr; }
  if (mollistindex >= (int)sim->s.mollists.size()) {
    set_error(__func__, ECnonexist, "molecule list doesn't exist");
    return nullptr;
  }
  strcpy(mollist, sim->s.mollists[mollistindex].c_str());
  return mollist;
}

// species "all" or one species; ECsame otherwise (libsmoldyn.cpp:1155-1161 pattern)
static bool species_or_all(simptr sim, const char *species) {
  if (!species) return false;
  if (!strcmp(species, "all")) return true;
  return sim->s.species_index(species) > 0;
}

enum ErrorCode smolSetMolList(simptr sim, const char *species, enum MolecState state, const char *mollist) {
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(species_or_all(sim, species), ECsame, "species not recognized");
  LCHECK((state >= MSsoln && state <= MSbsoln) || state == MSall, ECsyntax, "invalid state");
  LCHECK(smolGetMolListIndexNT(sim, mollist) >= 0, ECsame, "molecule list not recognized");
  return ECok;
}

// ---- display (libsmoldyn.cpp:295, 485, 1147-1216): checked, then ignored ----
enum ErrorCode smolSetGraphicsParams(simptr sim, const char *method, int timesteps, int delay) {
  (void)timesteps;
  (void)delay;
  LCHECK(sim, ECmissing, "missing sim");
  if (method)
    LCHECK(!strcmp(method, "none") || !strcmp(method, "opengl") || !strcmp(method, "opengl_good") ||
               !strcmp(method, "opengl_better"),
           ECsyntax, "graphics method not recognized");
  return ECok;
}

enum ErrorCode smolSetMoleculeColor(simptr sim, const char *species, enum MolecState state, double *color) {
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(species_or_all(sim, species), ECsame, "species not recognized");
  LCHECK((state >= MSsoln && state <= MSbsoln) || state == MSall, ECsyntax, "invalid state");
  LCHECK(color, ECmissing, "missing color");
  for (int c = 0; c < 3; ++c) LCHECK(color[c] >= 0 && color[c] <= 1, ECbounds, "color value out of bounds");
  return ECok;
}

enum ErrorCode smolSetMoleculeSize(simptr sim, const char *species, enum MolecState state, double size) {
  (void)size;
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(species_or_all(sim, species), ECsame, "species not recognized");
  LCHECK((state >= MSsoln && state <= MSbsoln) || state == MSall, ECsyntax, "invalid state");
  return ECok;
}

enum ErrorCode smolSetMoleculeStyle(simptr sim, const char *species, enum MolecState state, double size,
                                    double *color) {
  (void)size;
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(species_or_all(sim, species), ECsame, "species not recognized");
  LCHECK((state >= MSsoln && state <= MSbsoln) || state == MSall, ECsyntax, "invalid state");
  if (color)
    for (int c = 0; c < 3; ++c) LCHECK(color[c] >= 0 && color[c] <= 1, ECbounds, "color value out of bounds");
  return ECok;
}

enum ErrorCode smolDisplaySim(simptr sim) {
  LCHECK(sim, ECmissing, "missing sim");
  const Sim &s = sim->s;
  printf("libsmoldyn_b200 simulation: %d dimension(s), time %g to %g step %g\n", s.dim, s.tstart, s.tstop, s.dt);
  for (int d = 0; d < s.dim; ++d)
    printf("  axis %d: %g to %g, walls %c %c\n", d, s.lo[d], s.hi[d], s.btype[d][0], s.btype[d][1]);
  for (size_t i = 1; i < s.species.size(); ++i)
    printf("  species %s: difc %g\n", s.species[i].name.c_str(), s.species[i].difc);
  for (int o = 0; o < 3; ++o)
    for (const smolb::RxnDef &r : s.rxn[o]) printf("  reaction %s: order %d, rate %g\n", r.name.c_str(), o, r.rate);
  printf("  surfaces %d, compartments %d\n", (int)s.surfaces.size(), (int)s.cmpts.size());
  return ECok;
}

void smolGetSpeciesName(simptr sim, int speciesindex, char *species) {
  if (!sim || !species) return;
  if (speciesindex < 0 || speciesindex >= (int)sim->s.species.size()) { species[0] = 0; return; }
  strcpy(species, sim->s.species[speciesindex].name.c_str());
}

enum ErrorCode smolSetSpeciesMobility(simptr sim, const char *species, enum MolecState state, double difc,
                                      double *drift, double *difmatrix) {
  LCHECK(sim && species, ECmissing, "missing sim or species");
  LCHECK(state == MSsoln || state == MSall || state == MSfront || state == MSback, ECbounds,
         "the up, down and bsoln states are not supported");
  LCHECK(difc >= 0 || difmatrix, ECbounds, "difc must be >= 0");
  if (state == MSfront || state == MSback) {  // surface-bound states: isotropic diffusion only
    LCHECK(!drift && !difmatrix, ECbounds, "drift and diffusion matrices of surface-bound states are not supported");
    std::vector<int> ids;
    if (!strcmp(species, "all")) for (size_t i = 1; i < sim->s.species.size(); ++i) ids.push_back((int)i);
    else {
      const int i = sim->s.species_index(species);
      LCHECK(i > 0, ECnonexist, "species not found");
      ids.push_back(i);
    }
    for (int i : ids) sim->s.species[i].difc_bound[state == MSfront ? 0 : 1] = difc;
    sim->s.need_update = sim->s.need_rebuild = true;
    return ECok;
  }
  std::vector<int> ids;
  if (!strcmp(species, "all")) for (size_t i = 1; i < sim->s.species.size(); ++i) ids.push_back((int)i);
  else {
    const int i = sim->s.species_index(species);
    LCHECK(i > 0, ECnonexist, "species not found");
    ids.push_back(i);
  }
  for (int i : ids) {  // libsmoldyn.cpp:917: difc, then drift, then the matrix (which resets difc)
    if (difc >= 0) sim->s.species[i].difc = difc;
    if (difc >= 0 && state == MSall) sim->s.species[i].difc_bound[0] = sim->s.species[i].difc_bound[1] = difc;
    if (drift) for (int d = 0; d < sim->s.dim; ++d) sim->s.species[i].drift[d] = drift[d];
    if (difmatrix) smolb::set_species_difm(sim->s, i, difmatrix);
  }
  sim->s.need_update = true;
  return ECok;
}

enum ErrorCode smolSetMaxMolecules(simptr sim, int maxmolecules) {
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(maxmolecules > 0, ECbounds, "maxmolecules must be > 0");
  sim->s.max_mol = maxmolecules;
  sim->s.need_rebuild = true;
  return ECok;
}

enum ErrorCode smolAddSolutionMolecules(simptr sim, const char *species, int number, double *lowposition,
                                        double *highposition) {
  LCHECK(sim && species, ECmissing, "missing sim or species");
  LCHECK(number >= 0, ECbounds, "number must be >= 0");
  Sim &s = sim->s;
  const int i = s.species_index(species);
  LCHECK(i > 0, ECnonexist, "species not found");
  std::string err;
  if (s.eng && s.started) {
    if (pull_molecules(s, &err)) return set_error(__func__, ECerror, err);
  }
  for (int k = 0; k < number; ++k) {
    for (int d = 0; d < 3; ++d) {
      double x = 0;
      if (d < s.dim) {
        const double lo = lowposition ? lowposition[d] : s.lo[d];
        const double hi = highposition ? highposition[d] : s.hi[d];
        x = (lo == hi) ? lo : lo + s.rand_u01() * (hi - lo);
      }
      s.pend_pos.push_back(x);
    }
    s.pend_sp.push_back(i);
  }
  s.need_rebuild = true;
  return ECok;
}

int smolGetMoleculeCount(simptr sim, const char *species, enum MolecState state) {
  if (!sim || !species) return (int)set_error(__func__, ECmissing, "missing sim or species");
  if (state != MSall && state != MSsoln && state != MSfront && state != MSback && state != MSsome)
    return (int)set_error(__func__, ECbounds, "state not supported");
  Sim &s = sim->s;
  int idx = -1;
  if (strcmp(species, "all")) {
    idx = s.species_index(species);
    if (idx < 0) return (int)set_error(__func__, ECnonexist, "species not found");
  }
  std::string err;
  const long long n = species_state_count(s, idx, (int)state, &err);
  if (n < 0) return (int)set_error(__func__, ECerror, err);
  return (int)n;
}

enum ErrorCode smolSetBoundaryType(simptr sim, int dimension, int highside, char type) {
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(dimension >= -1 && dimension < sim->s.dim, ECbounds, "dimension out of range");
  LCHECK(highside >= -1 && highside <= 1, ECbounds, "highside must be -1, 0 or 1");
  LCHECK(type == 'r' || type == 'p' || type == 'a' || type == 't', ECsyntax, "type must be r, p, a or t");
  for (int d = 0; d < sim->s.dim && d < 3; ++d) {
    if (dimension >= 0 && d != dimension) continue;
    for (int side = 0; side < 2; ++side)
      if (highside < 0 || side == highside) sim->s.btype[d][side] = type;
  }
  sim->s.need_rebuild = true;
  return ECok;
}

enum ErrorCode smolAddSurface(simptr sim, const char *surface) {
  LCHECK(sim && surface, ECmissing, "missing sim or surface");
  for (const smolb::SurfaceDef &sf : sim->s.surfaces) LCHECK(sf.name != surface, ECsame, "surface exists");
  smolb::SurfaceDef sf;
  sf.name = surface;
  sim->s.surfaces.push_back(sf);
  sim->s.need_rebuild = true;
  return ECok;
}

namespace {
const char *ms_word(int ms) {
  static const char *w[] = {"soln", "front", "back", "up", "down", "bsoln", "all"};
  return (ms >= 0 && ms <= 6) ? w[ms] : "none";
}

int surface_index(const Sim &s, const char *name) {
  for (size_t k = 0; k < s.surfaces.size(); ++k)
    if (s.surfaces[k].name == name) return (int)k;
  return -1;
}
}  // namespace

enum ErrorCode smolSetSurfaceAction(simptr sim, const char *surface, enum PanelFace face, const char *species,
                                    enum MolecState state, enum SrfAction action, const char *newspecies) {
  LCHECK(sim && surface && species, ECmissing, "missing argument");
  const int sidx = surface_index(sim->s, surface);
  LCHECK(sidx >= 0, ECnonexist, "surface not found");
  LCHECK(face == PFfront || face == PFback || face == PFboth, ECbounds, "face must be front, back or both");
  const char *an = action == SAreflect ? "reflect" : action == SAtrans ? "transmit" : action == SAabsorb ? "absorb" : nullptr;
  LCHECK(an, ECbounds, "surface action not supported by the GPU engine");
  std::vector<std::string> w = {std::string(species) + "(" + ms_word(state) + ")",
                                face == PFfront ? "front" : face == PFback ? "back" : "both", an};
  if (newspecies && newspecies[0]) w.push_back(newspecies);
  std::string err;
  const int rc = smolb::read_surface_rule_statement(sim->s, sidx, "action", w, &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  sim->s.need_update = sim->s.need_rebuild = true;
  return ECok;
}

enum ErrorCode smolSetSurfaceRate(simptr sim, const char *surface, const char *species, enum MolecState state,
                                  enum MolecState state1, enum MolecState state2, double rate, const char *newspecies,
                                  int isinternal) {
  LCHECK(sim && surface && species, ECmissing, "missing argument");
  const int sidx = surface_index(sim->s, surface);
  LCHECK(sidx >= 0, ECnonexist, "surface not found");
  std::vector<std::string> w = {std::string(species) + "(" + ms_word(state) + ")", ms_word(state1), ms_word(state2)};
  char buf[64];
  snprintf(buf, sizeof(buf), "%.17g", rate);
  w.push_back(buf);
  if (newspecies && newspecies[0]) w.push_back(newspecies);
  std::string err;
  const int rc = smolb::read_surface_rule_statement(sim->s, sidx, isinternal ? "rate_internal" : "rate", w, &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  sim->s.need_update = sim->s.need_rebuild = true;
  return ECok;
}

enum ErrorCode smolAddPanelNeighbor(simptr sim, const char *surface1, const char *panel1, const char *surface2,
                                    const char *panel2, int reciprocal) {
  LCHECK(sim && surface1 && panel1 && surface2 && panel2, ECmissing, "missing argument");
  const int s1 = surface_index(sim->s, surface1), s2 = surface_index(sim->s, surface2);
  LCHECK(s1 >= 0 && s2 >= 0, ECnonexist, "surface not found");
  std::string err;
  int rc = smolb::read_surface_rule_statement(sim->s, s1, "neighbors",
                                              {panel1, std::string(surface2) + ":" + panel2}, &err);
  if (!rc && reciprocal)
    rc = smolb::read_surface_rule_statement(sim->s, s2, "neighbors", {panel2, std::string(surface1) + ":" + panel1}, &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  sim->s.need_rebuild = true;
  return ECok;
}

enum ErrorCode smolgpuGetSurfaceRule(simptr sim, const char *surface, const char *species, enum MolecState state,
                                     enum PanelFace face, int *action, double *prob, double *cumprob,
                                     double *revprob) {
  LCHECK(sim && surface && species && action && prob && cumprob && revprob, ECmissing, "missing argument");
  const int sidx = surface_index(sim->s, surface);
  LCHECK(sidx >= 0, ECnonexist, "surface not found");
  const int i = sim->s.species_index(species);
  LCHECK(i > 0, ECnonexist, "species not found");
  std::string err;
  const int rc = smolb::surface_rule_info(sim->s, sidx, i, (int)state, (int)face, action, prob, cumprob, revprob, &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  return ECok;
}

enum ErrorCode smolSetSurfaceSimParams(simptr sim, const char *parameter, double value) {
  LCHECK(sim && parameter, ECmissing, "missing argument");
  LCHECK(value >= 0, ECbounds, "value must be >= 0");
  if (!strcmp(parameter, "epsilon")) sim->s.srf_epsilon = value;
  else if (!strcmp(parameter, "margin")) sim->s.srf_margin = value;
  else if (!strcmp(parameter, "neighbordist")) sim->s.srf_neighdist = value;
  else return set_error(__func__, ECsyntax, "parameter not recognized");
  sim->s.need_rebuild = true;
  return ECok;
}

enum ErrorCode smolAddSurfaceMolecules(simptr sim, const char *species, enum MolecState state, int number,
                                       const char *surface, enum PanelShape panelshape, const char *panel,
                                       double *position) {
  LCHECK(sim && species && surface, ECmissing, "missing argument");
  LCHECK(number >= 0, ECbounds, "number must be >= 0");
  LCHECK(state == MSfront || state == MSback, ECbounds, "state must be front or back");
  Sim &s = sim->s;
  const int sp = s.species_index(species);
  LCHECK(sp > 0, ECnonexist, "species not found");
  int sidx = -1;
  if (strcmp(surface, "all")) {
    sidx = surface_index(s, surface);
    LCHECK(sidx >= 0, ECnonexist, "surface not found");
  }
  int q = -1;
  if (panel && strcmp(panel, "all")) {
    LCHECK(sidx >= 0, ECbounds, "a named panel needs a named surface");
    q = smolb::find_panel(s, sidx, panel, nullptr);
    LCHECK(q >= 0, ECnonexist, "panel not found");
  }
  std::string err;
  if (s.eng && s.started)
    if (pull_molecules(s, &err)) return set_error(__func__, ECerror, err);
  const int shape = (panelshape == PSall || panelshape == PSnone) ? -1 : (int)panelshape;
  const int rc = smolb::add_surface_molecules(s, number, sp, (int)state, sidx, shape, q, position, &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  return ECok;
}

enum ErrorCode smolAddPanel(simptr sim, const char *surface, enum PanelShape panelshape, const char *panel,
                            const char *axisstring, double *params) {
  LCHECK(sim && surface && params, ECmissing, "missing argument");
  smolb::SurfaceDef *sf = nullptr;
  for (smolb::SurfaceDef &x : sim->s.surfaces)
    if (x.name == surface) sf = &x;
  LCHECK(sf, ECnonexist, "surface not found");
  LCHECK((int)sf->panels.size() < smolb::kMaxPanels, ECbounds, "too many panels");
  const int dim = sim->s.dim;
  int np = 0;
  switch (panelshape) {
    case PSrect: np = 2 * dim - 1; break;
    case PSsph: np = dim + 1; break;
    case PStri: np = 9; break;
    case PScyl: case PShemi: case PSdisk: np = 7; break;
    default: return set_error(__func__, ECbounds, "panel shape not supported");
  }
  LCHECK(panelshape != PSrect || axisstring, ECmissing, "missing axis string");
  smolb::PanelSpec p{};
  std::string err;
  const int rc = smolb::make_panel(dim, (int)panelshape, axisstring ? axisstring : "", params, np, &p, &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  sf->pnames.push_back(smolb::new_panel_name(*sf, (int)panelshape, panel ? panel : ""));
  sf->panels.push_back(p);
  smolb::invalidate_compartments(sim->s);
  sim->s.need_rebuild = true;
  return ECok;
}

enum ErrorCode smolAddCompartment(simptr sim, const char *compartment) {
  LCHECK(sim && compartment, ECmissing, "missing argument");
  Sim &s = sim->s;
  LCHECK(s.compartment_index(compartment) < 0, ECsame, "compartment already exists");
  LCHECK((int)s.cmpts.size() < smolb::kMaxCmpt, ECbounds, "too many compartments");
  smolb::CompartDef c;
  c.name = compartment;
  s.cmpts.push_back(c);
  s.need_update = s.need_rebuild = true;
  return ECok;
}

int smolGetCompartmentIndexNT(simptr sim, const char *compartment) {
  if (!sim || !compartment) return (int)ECmissing;
  const int c = sim->s.compartment_index(compartment);
  return c >= 0 ? c : (int)ECnonexist;
}

int smolGetCompartmentIndex(simptr sim, const char *compartment) {
  const int c = smolGetCompartmentIndexNT(sim, compartment);
  if (c < 0) return (int)set_error(__func__, (ErrorCode)c, "compartment not found");
  return c;
}

char *smolGetCompartmentName(simptr sim, int compartmentindex, char *compartment) {
  if (!sim || !compartment) { set_error(__func__, ECmissing, "missing argument"); return nullptr; }
  if (compartmentindex < 0 || compartmentindex >= (int)sim->s.cmpts.size()) {
    set_error(__func__, ECbounds, "compartment index out of range");
    return nullptr;
  }
  strcpy(compartment, sim->s.cmpts[compartmentindex].name.c_str());
  return compartment;
}

enum ErrorCode smolAddCompartmentSurface(simptr sim, const char *compartment, const char *surface) {
  LCHECK(sim && compartment && surface, ECmissing, "missing argument");
  std::string err;
  const int c = sim->s.compartment_index(compartment);
  LCHECK(c >= 0, ECnonexist, "compartment not found");
  const int rc = smolb::read_compartment_words(sim->s, c, "surface", {surface}, &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  return ECok;
}

enum ErrorCode smolAddCompartmentPoint(simptr sim, const char *compartment, double *point) {
  LCHECK(sim && compartment && point, ECmissing, "missing argument");
  std::string err;
  const int c = sim->s.compartment_index(compartment);
  LCHECK(c >= 0, ECnonexist, "compartment not found");
  std::vector<std::string> w;
  char buf[64];
  for (int d = 0; d < sim->s.dim; ++d) {
    snprintf(buf, sizeof buf, "%.17g", point[d]);
    w.push_back(buf);
  }
  const int rc = smolb::read_compartment_words(sim->s, c, "point", w, &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  return ECok;
}

enum ErrorCode smolAddCompartmentLogic(simptr sim, const char *compartment, enum CmptLogic logic,
                                       const char *compartment2) {
  LCHECK(sim && compartment && compartment2, ECmissing, "missing argument");
  static const char *syms[] = {"equal", "equalnot", "and", "or", "xor", "andnot", "ornot"};
  LCHECK(logic >= CLequal && logic <= CLornot, ECbounds, "unrecognized logic symbol");
  std::string err;
  const int c = sim->s.compartment_index(compartment);
  LCHECK(c >= 0, ECnonexist, "compartment not found");
  const int rc = smolb::read_compartment_words(sim->s, c, "compartment", {syms[logic], compartment2}, &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  return ECok;
}

enum ErrorCode smolAddCompartmentMolecules(simptr sim, const char *species, int number, const char *compartment) {
  LCHECK(sim && species && compartment, ECmissing, "missing argument");
  LCHECK(number >= 0, ECbounds, "number must be >= 0");
  Sim &s = sim->s;
  LCHECK(s.species_index(species) > 0, ECnonexist, "species not found");
  LCHECK(s.compartment_index(compartment) >= 0, ECnonexist, "compartment not found");
  std::string err;
  if (s.eng && s.started)
    if (pull_molecules(s, &err)) return set_error(__func__, ECerror, err);
  const int rc = smolb::read_config_statement(s, "compartment_mol",
                                              std::to_string(number) + " " + species + " " + compartment, &err);
  if (rc) return set_error(__func__, from_rc(rc), err);
  return ECok;
}

enum ErrorCode smolSetReactionRegion(simptr sim, const char *reaction, const char *compartment, const char *surface) {
  LCHECK(sim && reaction, ECmissing, "missing argument");
  Sim &s = sim->s;
  int o = 0;
  const int r = s.reaction_index(reaction, &o);
  LCHECK(r >= 0, ECnonexist, "reaction not found");
  int c = -1;
  if (compartment) {
    c = s.compartment_index(compartment);
    LCHECK(c >= 0, ECnonexist, "compartment not found");
  }
  int sf = -1;
  if (surface) {
    for (size_t k = 0; k < s.surfaces.size(); ++k)
      if (s.surfaces[k].name == surface) sf = (int)k;
    LCHECK(sf >= 0, ECnonexist, "surface not found");
  }
  std::string err;
  if (smolb::set_reaction_surface(s, s.rxn[o][r], sf, &err)) return set_error(__func__, ECbounds, err);
  s.rxn[o][r].cmpt = c;
  s.need_update = s.need_rebuild = true;
  return ECok;
}

enum ErrorCode smolAddReaction(simptr sim, const char *reaction, const char *reactant1, enum MolecState rstate1,
                               const char *reactant2, enum MolecState rstate2, int nproduct,
                               const char **productspecies, enum MolecState *productstates, double rate) {
  LCHECK(sim && reaction, ECmissing, "missing sim or reaction name");
  Sim &s = sim->s;
  LCHECK(s.reaction_index(reaction, nullptr) < 0, ECsame, "reaction already exists");
  LCHECK(nproduct >= 0 && nproduct <= smolb::kMaxProd, ECbounds, "0..4 products supported");
  smolb::RxnDef x;
  x.name = reaction;
  int order = 0;
  const char *rr[2] = {reactant1, reactant2};
  const enum MolecState rs[2] = {rstate1, rstate2};
  for (int k = 0; k < 2; ++k) {
    if (rr[k] && rr[k][0]) {
      const int i = s.species_index(rr[k]);
      LCHECK(i > 0, ECnonexist, "reactant species not found");
      LCHECK(rs[k] >= MSsoln && rs[k] <= MSsome, ECbounds, "invalid reactant state");
      x.rct[order] = i;
      // MSall, MSnone and MSsome name the solution state here: surface-bound
      // reactants are given by their state
      x.rstate[order] = (rs[k] == MSall || rs[k] == MSnone || rs[k] == MSsome) ? MSsoln : (int)rs[k];
      order++;
    }
  }
  x.order = order;
  x.nprod = nproduct;
  LCHECK(nproduct == 0 || productspecies, ECmissing, "missing product species");
  for (int q = 0; q < nproduct; ++q) {
    const int i = s.species_index(productspecies[q]);
    LCHECK(i > 0, ECnonexist, "product species not found");
    x.prd[q] = i;
    // product states default to solution when the caller gives none
    x.pstate[q] = productstates ? (int)productstates[q] : MSsoln;
  }
  x.rate = rate;
  std::string err;
  if (smolb::add_reaction_def(s, x, &err))
    return set_error(__func__, err.find("too many") != std::string::npos ? ECbounds : ECsyntax, err);
  s.need_update = s.need_rebuild = true;
  return ECok;
}

enum ErrorCode smolAddBimolecularReaction(simptr sim, const char *reaction, const char *reactant1,
                                          const char *reactant2, int nproduct, const char **productspecies,
                                          double rate) {
  LCHECK(reactant1 && reactant2 && reactant1[0] && reactant2[0], ECmissing, "two reactants required");
  return smolAddReaction(sim, reaction, reactant1, MSsoln, reactant2, MSsoln, nproduct, productspecies, nullptr, rate);
}

int smolGetReactionIndex(simptr sim, int *orderptr, const char *reaction) {
  if (!sim || !reaction) return (int)set_error(__func__, ECmissing, "missing argument");
  const int r = sim->s.reaction_index(reaction, orderptr);
  if (r < 0) return (int)set_error(__func__, ECnonexist, "reaction not found");
  return r;
}

enum ErrorCode smolSetReactionRate(simptr sim, const char *reaction, double rate, int type) {
  (void)type;
  LCHECK(sim && reaction, ECmissing, "missing argument");
  int o;
  const int r = sim->s.reaction_index(reaction, &o);
  LCHECK(r >= 0, ECnonexist, "reaction not found");
  sim->s.rxn[o][r].rate = rate;
  sim->s.need_update = true;
  return ECok;
}

enum ErrorCode smolSetReactionProducts(simptr sim, const char *reaction, enum RevParam method, double parameter,
                                       const char *product, double *position) {
  LCHECK(sim && reaction, ECmissing, "missing argument");
  int o;
  const int r = sim->s.reaction_index(reaction, &o);
  LCHECK(r >= 0, ECnonexist, "reaction not found");
  smolb::RxnDef &x = sim->s.rxn[o][r];
  x.rparamt = (int)method;
  x.rparam = parameter;
  if ((method == RPoffset || method == RPfixed) && product && position) {
    const int q = sim->s.species_index(product);
    for (int k = 0; k < x.nprod; ++k)
      if (x.prd[k] == q) {
        for (int d = 0; d < sim->s.dim; ++d) x.user_prdpos[k][d] = position[d];
        break;
      }
  }
  sim->s.need_update = true;
  return ECok;
}

// ---- smolgpu extensions ----------------------------------------------------

enum ErrorCode smolgpuGetReactionParams(simptr sim, const char *reaction, double *bindrad, double *unbindrad,
                                        double *prob) {
  LCHECK(sim && reaction, ECmissing, "missing argument");
  LCHECK(sim->s.dt > 0, ECerror, "time step must be > 0");
  // parameter derivation only (host FP64); no engine is built here
  std::string err;
  if (smolb::derive_reaction_params(sim->s, &err)) return set_error(__func__, ECerror, err);
  int o;
  const int r = sim->s.reaction_index(reaction, &o);
  LCHECK(r >= 0, ECnonexist, "reaction not found");
  smolb::RxnDef &x = sim->s.rxn[o][r];
  if (bindrad) *bindrad = x.bindrad2 >= 0 ? std::sqrt(x.bindrad2) : -1;
  if (unbindrad) *unbindrad = x.unbindrad;
  if (prob) *prob = x.prob;
  return ECok;
}

enum ErrorCode smolgpuGetEffectiveRate(simptr sim, const char *reaction, double *rate, double *pgem) {
  LCHECK(sim && reaction && rate, ECmissing, "missing argument");
  LCHECK(sim->s.dt > 0, ECerror, "time step must be > 0");
  std::string err;
  if (smolb::derive_reaction_params(sim->s, &err)) return set_error(__func__, ECerror, err);
  int o;
  const int r = sim->s.reaction_index(reaction, &o);
  LCHECK(r >= 0, ECnonexist, "reaction not found");
  *rate = smolb::calc_rate(sim->s, o, r, pgem);
  return ECok;
}

double smolgpuGetTime(simptr sim) { return sim ? sim->s.time : 0; }
long long smolgpuGetStepCount(simptr sim) { return sim ? sim->s.steps : 0; }

long long smolgpuGetTotalMolecules(simptr sim) {
  if (!sim) return -1;
  if (sim->s.eng && sim->s.started && !sim->s.need_rebuild) return sim->s.eng->total_molecules();
  return (long long)sim->s.pend_sp.size();
}

enum ErrorCode smolgpuGetMolecules(simptr sim, long long *n, double *pos, int *species, uint64_t *serno) {
  LCHECK(sim && n, ECmissing, "missing argument");
  Sim &s = sim->s;
  std::string err;
  std::vector<double> p;
  std::vector<int> sp;
  std::vector<uint64_t> sn;
  if (s.eng && s.started && !s.need_rebuild) {
    if (s.eng->get_molecules(&p, &sp, nullptr, &sn, &err)) return set_error(__func__, ECerror, err);
  } else {
    p = s.pend_pos;
    sp = s.pend_sp;
    sn.resize(sp.size());
    uint64_t next = 1;
    for (uint64_t v : s.pend_serno) next = std::max<uint64_t>(next, v + 1);
    for (size_t i = 0; i < sp.size(); ++i) sn[i] = i < s.pend_serno.size() ? s.pend_serno[i] : next++;
  }
  const long long cnt = (long long)sp.size();
  LCHECK(*n >= cnt || (!pos && !species && !serno), ECbounds, "buffer too small");
  *n = cnt;
  if (pos) memcpy(pos, p.data(), p.size() * sizeof(double));
  if (species) memcpy(species, sp.data(), sp.size() * sizeof(int));
  if (serno) memcpy(serno, sn.data(), sn.size() * sizeof(uint64_t));
  return ECok;
}

enum ErrorCode smolgpuGetSurfaceMolecules(simptr sim, long long *n, double *pos, int *species, int *state,
                                          int *surface, int *panel, uint64_t *serno) {
  LCHECK(sim && n, ECmissing, "missing argument");
  Sim &s = sim->s;
  std::string err;
  std::vector<smolb::PendBound> b;
  if (s.eng && s.started && !s.need_rebuild) {
    std::vector<double> bpos;
    std::vector<int> bsp, bst, bpn;
    std::vector<uint64_t> bsn;
    if (s.eng->get_bound(&bpos, &bsp, &bst, &bpn, &bsn, &err)) return set_error(__func__, ECerror, err);
    for (size_t k = 0; k < bsp.size(); ++k) {
      smolb::PendBound x;
      for (int d = 0; d < 3; ++d) x.pos[d] = bpos[3 * k + d];
      x.species = bsp[k];
      x.state = bst[k];
      x.serno = bsn[k];
      int g = bpn[k];
      for (size_t q = 0; q < s.surfaces.size(); ++q) {
        if (g < (int)s.surfaces[q].panels.size()) { x.surface = (int)q; x.panel = g; break; }
        g -= (int)s.surfaces[q].panels.size();
      }
      b.push_back(x);
    }
  } else {
    b = s.pend_bound;
  }
  const long long cnt = (long long)b.size();
  LCHECK(*n >= cnt || (!pos && !species && !state && !surface && !panel && !serno), ECbounds, "buffer too small");
  *n = cnt;
  for (long long k = 0; k < cnt; ++k) {
    if (pos) for (int d = 0; d < 3; ++d) pos[3 * k + d] = b[k].pos[d];
    if (species) species[k] = b[k].species;
    if (state) state[k] = b[k].state;
    if (surface) surface[k] = b[k].surface;
    if (panel) panel[k] = b[k].panel;
    if (serno) serno[k] = b[k].serno;
  }
  return ECok;
}

enum ErrorCode smolgpuSetMolecules(simptr sim, long long n, const double *pos, const int *species,
                                   const uint64_t *serno) {
  LCHECK(sim && (n == 0 || (pos && species)), ECmissing, "missing argument");
  Sim &s = sim->s;
  for (long long i = 0; i < n; ++i)
    LCHECK(species[i] > 0 && species[i] < (int)s.species.size(), ECbounds, "species index out of range");
  if (!s.eng || s.need_rebuild) {  // the engine is (re)built around these molecules
    s.pend_pos.assign(pos, pos + 3 * n);
    s.pend_sp.assign(species, species + n);
    if (serno) s.pend_serno.assign(serno, serno + n);
    else s.pend_serno.clear();
    return update_sim(s, __func__);
  }
  // a current engine takes the caller's arrays directly, without a host copy
  ErrorCode ec = update_sim(s, __func__);
  if (ec != ECok) return ec;
  std::string err;
  if (s.eng->set_molecules(n, pos, species, nullptr, serno, &err)) return set_error(__func__, ECerror, err);
  s.pend_pos.clear();
  s.pend_sp.clear();
  s.pend_serno.clear();
  s.started = true;
  return ECok;
}

enum ErrorCode smolgpuGetEventCounts(simptr sim, long long counts[8]) {
  LCHECK(sim && counts, ECmissing, "missing argument");
  for (int k = 0; k < 8; ++k) counts[k] = 0;
  if (!sim->s.eng) return ECok;
  smolb::EngineStats st;
  std::string err;
  if (sim->s.eng->stats(&st, &err)) return set_error(__func__, ECerror, err);
  counts[0] = st.wall; counts[1] = st.rxn0; counts[2] = st.rxn1; counts[3] = st.rxn2;
  counts[4] = st.unresolved; counts[5] = st.multicand; counts[6] = st.overflow;
  return ECok;
}

enum ErrorCode smolgpuSetInjectedDisplacements(simptr sim, long long n, const uint64_t *sernos, const double *disp) {
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(n == 0 || (sernos && disp), ECmissing, "missing arrays");
  ErrorCode ec = update_sim(sim->s, __func__);
  if (ec != ECok) return ec;
  std::string err;
  if (sim->s.eng->set_injection(n, sernos, disp, 0, &err)) return set_error(__func__, ECerror, err);
  return ECok;
}

enum ErrorCode smolgpuSetStream(simptr sim, void *stream) {
  LCHECK(sim, ECmissing, "missing sim");
  ErrorCode ec = update_sim(sim->s, __func__);
  if (ec != ECok) return ec;
  sim->s.eng->set_stream(stream);
  return ECok;
}

enum ErrorCode smolgpuAutotune(simptr sim, int trial_steps, double *ms_per_step) {
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(trial_steps >= 2 && trial_steps <= 100000, ECbounds, "trial_steps must be 2..100000");
  Sim &s = sim->s;
  ErrorCode ec = update_sim(s, __func__);
  if (ec != ECok) return ec;
  LCHECK(s.steps == 0 && s.eng->steps_done() == 0, ECerror, "autotune runs before the first time step");
  std::string err;
  std::vector<double> pos;
  std::vector<int> sp, rep;
  std::vector<uint64_t> serno;
  if (s.eng->get_molecules(&pos, &sp, &rep, &serno, &err)) return set_error(__func__, ECerror, err);
  const bool box_free = s.molperbox <= 0 && s.boxsize <= 0;
  smolb::TuneSetup ts;
  if (box_free) ts.box_candidates = {1, 2, 4, 8};
  ts.box_default = s.auto_molperbox > 0 ? s.auto_molperbox : 4;
  ts.engine = [&]() { return s.eng.get(); };
  ts.rebuild = [&](double mpb, std::string *e) -> int {
    if (box_free) s.auto_molperbox = mpb;
    smolb::NetSpec net;
    smolb::RepSpec rs;
    s.pend_sp = sp;  // the box grid follows the molecule count
    int rc = smolb::build_engine_specs(s, &net, &rs, e);
    s.pend_sp.clear();
    if (rc) return rc;
    const long long n = (long long)sp.size();
    const long long cap = s.max_mol > 0 ? s.max_mol : std::max<long long>(2 * n + 4096, n + (1 << 20));
    const smolb::LaunchTuning keep = s.eng->tuning();
    rc = msd_save(s, e);
    if (rc) return rc;
    rc = s.eng->init(net, {rs}, s.dt, (uint64_t)s.seed, cap, e);
    if (!rc) rc = s.eng->set_tuning(keep, e);
    if (!rc) rc = s.eng->set_molecules(n, pos.data(), sp.data(), nullptr, serno.data(), e);
    return rc;
  };
  smolb::TuneResult tr;
  if (smolb::autotune(ts, trial_steps, &tr, &err)) return set_error(__func__, ECerror, err);
  s.tuning = tr.launch;
  if (box_free) s.auto_molperbox = tr.molperbox;
  if (g_debug) fprintf(stderr, "smolgpuAutotune trials (molperbox tile tileblocks molblocks ms):\n%s", tr.log.c_str());
  if (ms_per_step) *ms_per_step = tr.ms_per_step;
  return ECok;
}

enum ErrorCode smolgpuGetTuning(simptr sim, double *molperbox, int *pair_tile, int *tile_blocks_per_sm,
                                int *mol_blocks_per_sm) {
  LCHECK(sim, ECmissing, "missing sim");
  const Sim &s = sim->s;
  if (molperbox) *molperbox = s.molperbox > 0 ? s.molperbox : (s.boxsize > 0 ? -1 : (s.auto_molperbox > 0 ? s.auto_molperbox : 4));
  if (pair_tile) *pair_tile = s.tuning.pair_tile;
  if (tile_blocks_per_sm) *tile_blocks_per_sm = s.tuning.tile_blocks_per_sm;
  if (mol_blocks_per_sm) *mol_blocks_per_sm = s.tuning.mol_blocks_per_sm;
  return ECok;
}

long long smolgpuGetLaunchCount(simptr sim) { return (sim && sim->s.eng) ? sim->s.eng->launches() : 0; }

enum ErrorCode smolgpuRunSteps(simptr sim, long long nsteps) {
  LCHECK(sim, ECmissing, "missing sim");
  LCHECK(nsteps >= 0, ECbounds, "nsteps must be >= 0");
  Sim &s = sim->s;
  ErrorCode ec = update_sim(s, __func__);
  if (ec != ECok) return ec;
  std::string err;
  if (advance_steps(s, nsteps, &err)) return set_error(__func__, ECerror, err);
  return ECok;
}

enum ErrorCode smolgpuProfileSteps(simptr sim, long long nsteps, int *nkernels, char *names, double *ms,
                                   long long *launches) {
  LCHECK(sim && nkernels, ECmissing, "missing argument");
  Sim &s = sim->s;
  ErrorCode ec = update_sim(s, __func__);
  if (ec != ECok) return ec;
  std::vector<std::string> nm;
  std::vector<double> t;
  std::vector<long long> l;
  std::string err;
  if (s.eng->profile(nsteps, &nm, &t, &l, &err)) return set_error(__func__, ECerror, err);
  for (long long k = 0; k < nsteps; ++k) s.time += s.dt;
  s.steps += nsteps;
  const int cap = *nkernels;
  *nkernels = (int)nm.size();
  for (int k = 0; k < (int)nm.size() && k < cap; ++k) {
    if (names) { strncpy(names + 32 * k, nm[k].c_str(), 31); names[32 * k + 31] = 0; }
    if (ms) ms[k] = t[k];
    if (launches) launches[k] = l[k];
  }
  return ECok;
}

enum ErrorCode smolgpuSynchronize(simptr sim) {
  LCHECK(sim, ECmissing, "missing sim");
  if (!sim->s.eng) return ECok;
  std::string err;
  if (sim->s.eng->synchronize(&err)) return set_error(__func__, ECerror, err);
  return ECok;
}

enum ErrorCode smolgpuSolveRadii(int mode, long long n, const double *rate, double dt, const double *difc,
                                 const double *b, int rel, double *out) {
  LCHECK(n >= 0, ECbounds, "n must be >= 0");
  LCHECK(n == 0 || (rate && difc && b && out), ECmissing, "missing arrays");
  LCHECK(mode == 0 || mode == 1, ECbounds, "mode must be 0 or 1");
  std::string err;
  if (smolb::solve_radii_device(mode, n, rate, dt, difc, b, rel, out, &err)) return set_error(__func__, ECerror, err);
  return ECok;
}

double smolgpuBindingRadiusHost(double rate, double dt, double difc, double b, int rel) {
  return smolb::rxnp::bindingradius(rate, dt, difc, b, rel);
}

double smolgpuNumRxnRateProbHost(double step, double a, double b, double prob) {
  return smolb::rxnp::numrxnrateprob(step, a, b, prob);
}

double smolgpuBindingRadiusProbHost(double rate, double dt, double difc, double b, int rel, double chi,
                                    double *prob) {
  return smolb::rxnp::bindingradiusprob(rate, dt, difc, b, rel, chi, prob);
}

enum ErrorCode smolgpuSolveRadiiProb(long long n, const double *rate, double dt, const double *difc,
                                     const double *b, int rel, const double *chi, double *prob, double *out) {
  LCHECK(n >= 0, ECbounds, "n must be >= 0");
  LCHECK(n == 0 || (rate && difc && b && chi && prob && out), ECmissing, "missing arrays");
  std::string err;
  if (smolb::solve_radii_prob_device(n, rate, dt, difc, b, rel, chi, prob, out, &err))
    return set_error(__func__, ECerror, err);
  return ECok;
}

double smolgpuUnbindingRadiusHost(double pgem, double dt, double difc, double a) {
  return smolb::rxnp::unbindingradius(pgem, dt, difc, a);
}

int smolgpuRxnTable(const char *name, double *out, int cap) {
  using namespace smolb::rxnp;
  if (!name) return -1;
  const std::string nm(name);
  const double *t = nullptr;
  int len = 0;
  if (nm == "yi") t = h_yi, len = SMOLB_TAB_YI_LEN;
  else if (nm == "yr") t = h_yr, len = SMOLB_TAB_YR_LEN;
  else if (nm == "yb") t = h_yb, len = SMOLB_TAB_YB_LEN;
  else if (nm == "kirr") t = h_kirr, len = SMOLB_TAB_KIRR_LEN;
  else if (nm == "krev") t = h_krev, len = SMOLB_TAB_KREV_LEN;
  else if (nm == "kb") t = h_kb, len = SMOLB_TAB_KB_LEN;
  else return -1;
  if (out)
    for (int i = 0; i < len && i < cap; ++i) out[i] = t[i];
  return len;
}

}  // extern "C"

// Shared with ensemble.cpp and surrogate.cu: record an error in the
// process-global slot read by smolGetError.
ErrorCode smolb_record_error(const char *func, ErrorCode code, const std::string &msg) {
  return set_error(func, code, msg);
}
