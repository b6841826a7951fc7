// Autotuner for the per-step kernels: box width (molecules per virtual box),
// k_pairs_tile tile size and blocks per SM, and blocks per SM of the
// streaming kernels.  Trials run real steps on the workload at hand from a
// saved start state, which is restored afterwards, so tuning does not change
// the simulation's trajectory beyond FP32 rounding of box-local coordinates.
#pragma once

#include <functional>
#include <string>
#include <vector>

#include "engine.h"

namespace smolb {

struct TuneSetup {
  // Put the engine back at the saved start state with virtual boxes of
  // `molperbox` molecules on average (ignored when box_candidates is empty).
  std::function<int(double molperbox, std::string *err)> rebuild;
  std::function<Engine *()> engine;
  std::vector<double> box_candidates;
  double box_default = 4;
};

struct TuneResult {
  double molperbox = -1;
  LaunchTuning launch;
  double ms_per_step = 0;
  std::string log;  // one line per trial: "mpb tile tileblocks molblocks ms"
};

// Coordinate search: box width first (default launch shape), then the pair
// tile (size x blocks per SM), then the streaming kernels' blocks per SM.
// Each trial: 2 warm-up steps, then `trial_steps` timed steps.  Leaves the
// engine rebuilt at the start state with the best settings.
int autotune(const TuneSetup &setup, int trial_steps, TuneResult *res, std::string *err);

}  // namespace smolb
