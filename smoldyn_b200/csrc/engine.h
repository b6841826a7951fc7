// Host-side interface of the B200 particle engine (no CUDA types here).
//
// The engine replaces the body of Smoldyn's simulatetimestep
// (source/Smoldyn/smolsim.cpp:2607-2692): diffuse (smolmolec.c:3115),
// checkwalls (smolwall.c:368), reassignmolecs/molsort (smolboxes.c:896,
// smolmolec.c:2943), zeroreact/unireact/bireact (smolreact.c:2905/2997/3201)
// and doreact product placement (smolreact.c:2662).  One engine holds an
// ensemble of R >= 1 independent replicates that share the reaction network
// but have their own box, walls, rates and radii; a plain simulation is R=1.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace smolb {

constexpr int kMaxSpecies = 32;   // species indices 0..31 (0 = "empty" as in the reference)
constexpr int kMaxRxn = 16;       // reactions per order
constexpr int kMaxProd = 4;       // products per reaction
constexpr int kMaxUniPerSpecies = 8;
constexpr int kMaxPairRxn = 4;    // reactions per reactant species pair
constexpr int kMaxPanels = 16;
constexpr int kMaxCmpt = 8;         // compartments
constexpr int kMaxCmptPts = 8;      // interior-defining points per compartment
constexpr int kMaxCmptLogic = 4;    // logic terms per compartment
constexpr int kMaxNeigh = 8;        // neighbouring panels per panel (surface-bound molecules)

enum WallKind : uint8_t { kWallReflect = 0, kWallPeriodic = 1, kWallAbsorb = 2, kWallTransparent = 3 };

// Surface panel with one action for all species on each face
// (smolsurface.c:4930 dosurfinteract subset).  Shapes follow the reference's
// PanelShape numbering (smoldyn.h:492): 0 rect, 1 tri, 2 sph, 3 cyl, 4 hemi,
// 5 disk; faces as in panelside (smolsurface.c:3930).
struct PanelSpec {
  int shape;
  int axis;             // rect: perpendicular axis 0..2; front face toward +axis if front_sign>0
  int front_sign;       // rect: +1 / -1; sph, cyl, hemi: +1 = front outward, -1 = front inward; tri, disk: +1
  double pos;           // rect: coordinate of the plane along axis
  double lo[3], hi[3];  // rect: extent in the two in-plane axes (lo/hi per axis)
  double center[3];     // sph, hemi, disk
  double radius;        // sph, cyl, hemi, disk
  double pt[3][3];      // tri: vertices; cyl: axis end points pt[0], pt[1]
  double normal[3];     // tri, disk: unit front normal; hemi: unit vector out of the open side; cyl: unit axis
  int action_front;     // 0 reflect, 1 transmit, 2 absorb (per species below overrides)
  int action_back;
  uint32_t absorb_front_mask;   // species bitmask overriding to absorb on front
  uint32_t absorb_back_mask;
  uint32_t trans_front_mask;    // species bitmask overriding to transmit on front
  uint32_t trans_back_mask;
  uint32_t refl_front_mask;     // species bitmask overriding to reflect on front
  uint32_t refl_back_mask;
  uint32_t jump_front_mask;     // species bitmask overriding to jump on front
  uint32_t jump_back_mask;
  int jump_pnl[2];              // per face: the engine panel a jump leads to (-1 none), and its face
  int jump_face[2];
  int srf;                      // index of the panel's surface
  int nneigh;                   // neighbouring panels (engine panel indices) for surface-bound molecules
  int neigh[kMaxNeigh];
  int neighhop;                 // the surface's neighbor_action: 1 hop, 0 stay
};

// One (surface, species, state, face) interaction in device form
// (surfaction, smolsurface.c:4330): the SrfAction, and for rate-based
// actions (SAmult) the cumulative probabilities of the destination states
// (MolecState order soln, front, back, up, down, bsoln), the species after
// each outcome (0: removed), and whether the reverse of each outcome has a
// nonzero probability (reversible desorption places the molecule
// differently).
struct SrfRule {
  double cum[6];
  int8_t act;
  int8_t newspec[6];
  uint8_t rev;
};

// Compartment: interior points, bounding panels (indices into NetSpec::panels)
// and logic terms on earlier compartments (see DevCmpt).
struct CmptSpec {
  std::vector<std::vector<double>> pts;       // 3 coordinates each
  uint32_t panel_mask = 0;
  std::vector<std::pair<int, int>> logic;     // (symbol, compartment)
};

// Reaction network shared by every replicate.
struct NetSpec {
  int nspecies = 1;                          // including index 0
  int nrxn[3] = {0, 0, 0};
  int rct[3][kMaxRxn][2] = {};               // reactant species (order 1: [0]; order 2: both)
  int nprod[3][kMaxRxn] = {};
  int prd[3][kMaxRxn][kMaxProd] = {};
  int fixed_placement[3][kMaxRxn] = {};      // 1: product offsets not rotated (RPfixed)
  int placement2[kMaxRxn] = {};              // order 2: 1 confspread, 2 bounce, else 0
  double bounce_k[kMaxRxn] = {};             // bounce: 1 (unbinding radius given) or 2 (from binding radius)
  int gauss_table_size = 4096;               // power of two (smolmolec.c:781)
  std::vector<PanelSpec> panels;
  std::vector<CmptSpec> cmpts;
  int cmpt[3][kMaxRxn] = {};                 // compartment of each reaction + 1 (0: none)
  int rsrf[3][kMaxRxn] = {};                 // surface of each reaction + 1 (0: none)
  int pstate0[kMaxRxn][kMaxProd] = {};       // product states of order-0 reactions (surface births)
  double panel_area[kMaxPanels] = {};        // area (2-D: length) of each engine panel
  // first-order reactions of surface-bound reactants: reactant state (0 soln,
  // 1 front, 2 back) and product state (0 soln, 1 front, 2 back, 5 bsoln)
  int rstate1[kMaxRxn] = {};
  int pstate1[kMaxRxn][2] = {};
  // second-order reactions with one surface-bound reactant: reactant states
  // and the product's state
  int rstate2[kMaxRxn][2] = {};
  int pstate2[kMaxRxn] = {};  // (both reactants bound: bound-bound reactions, same panel only)
  // surface-bound states (single simulations only): rules by
  // ((surface * kMaxSpecies + species) * 3 + state) * 3 + face, state 0..2 =
  // soln, front, back and face 0..2 = front, back, none
  int bound = 0;
  int nsrf = 0;
  std::vector<SrfRule> srf_rules;
  double difc_bound[kMaxSpecies][2] = {};    // diffusion coefficients of the front and back states
  double srf_eps = 0, srf_margin = 0, srf_neighdist = 0;  // surfacessstruct epsilon, margin, neighdist
};

// One replicate's geometry and rate-derived parameters.
struct RepSpec {
  double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  int ncell[3] = {1, 1, 1};
  uint8_t wall[6] = {0, 0, 0, 0, 0, 0};      // [2*d+side]
  int dim = 3;
  double difc[kMaxSpecies] = {};
  double drift[kMaxSpecies][3] = {};
  bool has_difm[kMaxSpecies] = {};           // anisotropic diffusion matrix present
  double difm[kMaxSpecies][9] = {};          // 3x3 row-major M (step = M * sqrt(2 dt) * gaussian)
  double uni_prob[kMaxRxn] = {};             // rxn->prob for order 1 (smolreact.c:1333-1357)
  double bind2[kMaxRxn] = {};                // rxn->bindrad2 for order 2
  double pair_prob[kMaxRxn] = {};            // rxn->prob for order 2 (1 unless set)
  double birth_mean[kMaxRxn] = {};           // rxn->prob for order 0 (expected births/step)
  double prdpos[3][kMaxRxn][kMaxProd][3] = {};
};

// Launch shape of the per-step kernels; the autotuner picks it per workload.
struct LaunchTuning {
  int mol_blocks_per_sm = 8;    // k_move, k_scatter, k_pairs_faces: 256-thread blocks per SM
  int tile_blocks_per_sm = 4;   // k_pairs_tile blocks per SM
  int pair_tile = 256;          // threads per k_pairs_tile block (warp tiles): 128 or 256
};

struct EngineStats {
  long long wall = 0, rxn0 = 0, rxn1 = 0, rxn2 = 0, unresolved = 0, multicand = 0, overflow = 0;
};

class EngineImpl;

class Engine {
 public:
  Engine();
  ~Engine();
  Engine(const Engine &) = delete;
  Engine &operator=(const Engine &) = delete;

  // Allocates device memory for `capacity` molecules in total.  Returns 0 or
  // an ErrorCode-style negative value with *err set.
  int init(const NetSpec &net, const std::vector<RepSpec> &reps, double dt, uint64_t seed,
           long long capacity, std::string *err);
  // Replace all molecules.  pos: 3*n absolute coordinates; rep may be null (all 0);
  // serno: null or 0 entries -> assigned 1,2,... per replicate in input order.
  int set_molecules(long long n, const double *pos, const int *species, const int *rep,
                    const uint64_t *serno, std::string *err);
  // Advance `nsteps` time steps (asynchronous unless sync is requested).
  int run(long long nsteps, std::string *err);
  // Surface-bound molecules (single simulations): replace them, or copy them
  // back sorted by serial number.  state: 1 front, 2 back; panel: engine
  // panel index; serno 0 entries get serial numbers after every molecule's.
  int set_bound(long long n, const double *pos, const int *species, const int *state, const int *panel,
                const uint64_t *serno, std::string *err);
  int get_bound(std::vector<double> *pos, std::vector<int> *species, std::vector<int> *state,
                std::vector<int> *panel, std::vector<uint64_t> *serno, std::string *err);
  // Copy molecules back (absolute coordinates, sorted by (rep, serno)).
  int get_molecules(std::vector<double> *pos, std::vector<int> *species, std::vector<int> *rep,
                    std::vector<uint64_t> *serno, std::string *err);
  // Live molecule count per (rep, species): out[rep*nspecies + sp].
  int species_counts(std::vector<long long> *out, std::string *err);
  long long total_molecules();
  int stats(EngineStats *s, std::string *err);
  int status_flags();
  // Status of the previous call's step, without waiting for the current one:
  // copies the status word asynchronously and returns the copy made by the
  // previous call (0 on the first call).
  int status_flags_lagged();
  // Update rate-derived parameters of every replicate (no reallocation).
  int update_reps(const std::vector<RepSpec> &reps, std::string *err);
  // Deterministic mode: per-serno displacements for the next step only.
  int set_injection(long long n, const uint64_t *sernos, const double *disp, int rep,
                    std::string *err);
  void set_stream(void *stream);
  void *stream() const;
  int synchronize(std::string *err);
  long long launches() const;
  long long steps_done() const;
  // Step index of the random streams (Philox counter; the next step uses
  // step + 1).  A simulation that rebuilds its engine mid-run sets it to the
  // steps already taken, so that no molecule replays earlier random numbers.
  int set_rng_step(uint64_t step, std::string *err);
  // Persistent ensemble kernel (mode 1): replicates are stepped by one CTA
  // each for blocks of up to 100 steps per launch, when the configuration
  // has no surfaces, compartments or injected displacements; mode 0 keeps
  // the step pipeline.  persistent_active() tells which one run() uses.
  int set_persistent(int mode, std::string *err);
  bool persistent_active() const;
  // Capture the 2-step kernel sequence in a CUDA graph and replay it (on by default).
  void set_use_graph(bool on);
  // Launch shape (kept across init); a change re-captures the step graph.
  int set_tuning(const LaunchTuning &t, std::string *err);
  LaunchTuning tuning() const;
  // Run n steps timing every kernel launch with CUDA events.
  int profile(long long nsteps, std::vector<std::string> *names, std::vector<double> *ms,
              std::vector<long long> *launches, std::string *err);

  // Mean square displacement trackers (cmdmeansqrdisp, smolcmd.c:2505-2606).
  // A tracker follows the molecules of `species` whose keys
  // ((rep << 42) | serial, ascending) it is given, from unwrapped start
  // positions `start` and last unwrapped positions `last` (3 per key).
  // msd_track returns a handle >= 0 or a negative code.
  int msd_track(int species, long long m, const uint64_t *keys, const double *start, const double *last,
                std::string *err);
  // Brings the tracker's unwrapped positions up to the current step: each
  // tracked molecule still present moves from its last unwrapped position by
  // its displacement, with periodic axes taken to the nearest image, so the
  // caller must call it before any molecule can travel half a period.  With
  // sums non-null, also returns the sum over tracked molecules present of r^2
  // (msddim < 0: all axes, else that axis) and of r^4, and their count.
  int msd_update(int handle, int msddim, double *sum2, double *sum4, long long *count, std::string *err);
  // Last unwrapped positions (3 per key), e.g. to carry a tracker across a rebuild.
  int msd_last(int handle, std::vector<double> *last, std::string *err);
  int msd_count() const;
  // Molecules of each species inside compartment c: out[sp] (cmdmolcountincmpt).
  int cmpt_counts(int c, std::vector<long long> *out, std::string *err);

 private:
  EngineImpl *impl_;
};

// Batched FP64 radius solver on the device (mode 0: binding, 1: unbinding).
int solve_radii_device(int mode, long long n, const double *rate, double dt, const double *difc,
                       const double *b, int rel, double *out, std::string *err);
// Batched bindingradiusprob on the device (prob in/out per problem).
int solve_radii_prob_device(long long n, const double *rate, double dt, const double *difc, const double *b,
                            int rel, const double *chi, double *prob, double *out, std::string *err);

}  // namespace smolb

namespace smolb {
// Batched pair_radii (binding radius of A+B->C with rate kf[i], mutual
// diffusion dsum[i], and the reverse's unbinding radius) on the device.
int solve_pair_radii_device(long long n, const double *kf, const double *dsum, double dt, int same, int rev,
                            int rparamt, double rparam, double *bind, double *unbind, int *errs, std::string *err);
}  // namespace smolb
