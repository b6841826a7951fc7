// Autotuner (see autotune.h).
#include "autotune.h"

#include <chrono>
#include <cstdio>
#include <limits>

namespace smolb {

namespace {

int time_steps(Engine *e, int steps, double *ms, std::string *err) {
  int rc = e->run(2, err);
  if (!rc) rc = e->synchronize(err);
  if (rc) return rc;
  const auto t0 = std::chrono::steady_clock::now();
  rc = e->run(steps, err);
  if (!rc) rc = e->synchronize(err);
  if (rc) return rc;
  *ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / steps;
  return 0;
}

}  // namespace

int autotune(const TuneSetup &setup, int trial_steps, TuneResult *res, std::string *err) {
  if (trial_steps < 2) trial_steps = 2;
  // an even count keeps every trial on whole two-step graph replays
  trial_steps += trial_steps & 1;
  char line[160];
  std::string log;
  auto trial = [&](double mpb, const LaunchTuning &lt, double *ms) -> int {
    int rc = setup.engine()->set_tuning(lt, err);
    if (!rc) rc = time_steps(setup.engine(), trial_steps, ms, err);
    if (rc) return rc;
    snprintf(line, sizeof(line), "%g %d %d %d %.5f\n", mpb, lt.pair_tile, lt.tile_blocks_per_sm,
             lt.mol_blocks_per_sm, *ms);
    log += line;
    return 0;
  };

  LaunchTuning best = setup.engine()->tuning();
  double best_mpb = setup.box_default;
  double best_ms = std::numeric_limits<double>::infinity();
  double ms = 0;
  // 1. box width at the current launch shape
  if (!setup.box_candidates.empty()) {
    for (double mpb : setup.box_candidates) {
      int rc = setup.rebuild(mpb, err);
      if (!rc) rc = trial(mpb, best, &ms);
      if (rc) return rc;
      if (ms < best_ms) { best_ms = ms; best_mpb = mpb; }
    }
    int rc = setup.rebuild(best_mpb, err);
    if (rc) return rc;
  } else {
    int rc = trial(best_mpb, best, &best_ms);
    if (rc) return rc;
  }
  // 2. pair tile: size x blocks per SM
  LaunchTuning base = best;
  for (int tile : {128, 256})
    for (int tb : {2, 4, 8}) {
      LaunchTuning t = base;
      t.pair_tile = tile;
      t.tile_blocks_per_sm = tile == 128 ? 2 * tb : tb;
      if (t.pair_tile == base.pair_tile && t.tile_blocks_per_sm == base.tile_blocks_per_sm) continue;
      int rc = trial(best_mpb, t, &ms);
      if (rc) return rc;
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
  // 3. streaming kernels' blocks per SM
  base = best;
  for (int mb : {4, 8, 16}) {
    if (mb == base.mol_blocks_per_sm) continue;
    LaunchTuning t = base;
    t.mol_blocks_per_sm = mb;
    int rc = trial(best_mpb, t, &ms);
    if (rc) return rc;
    if (ms < best_ms) { best_ms = ms; best = t; }
  }
  // leave the engine at the start state with the winner
  int rc = setup.rebuild(best_mpb, err);
  if (!rc) rc = setup.engine()->set_tuning(best, err);
  if (rc) return rc;
  res->molperbox = setup.box_candidates.empty() ? -1 : best_mpb;
  res->launch = best;
  res->ms_per_step = best_ms;
  res->log = log;
  return 0;
}

}  // namespace smolb
