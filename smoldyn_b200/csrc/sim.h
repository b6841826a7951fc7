// Host-side simulation description behind the libsmoldyn-compatible C API.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <array>
#include <vector>

#include "engine.h"

namespace smolb {

struct SpeciesDef {
  std::string name;
  double difc = 0;
  double difc_bound[2] = {0, 0};  // difc[i][MSfront], difc[i][MSback] (0 unless set)
  double drift[3] = {0, 0, 0};
  bool has_difm = false;   // anisotropic diffusion (difm statement, smolmolec.c:833)
  double difm[9] = {};     // matrix M, row-major in a 3x3 layout: step = M * sqrt(2 dt) * gaussian
};


// One reaction (smoldyn.h:389 rxnstruct subset).
struct RxnDef {
  std::string name;
  int order = 0;
  int rct[2] = {0, 0};
  int rstate[2] = {0, 0};   // reactant states (MolecState: 0 soln, 1 front, 2 back)
  int nprod = 0;
  int prd[kMaxProd] = {0, 0, 0, 0};
  int pstate[kMaxProd] = {0, 0, 0, 0};  // product states (0 soln, 1 front, 2 back, 5 bsoln)
  double rate = -1;         // requested rate constant; <0 undefined
  int cmpt = -1;            // compartment the reaction is restricted to (rxn->cmpt), -1 none
  int srf = -1;             // surface the reaction is restricted to (rxn->srf), -1 none
  int rparamt = 0;          // RevParam
  double rparam = 0;
  double user_prdpos[kMaxProd][3] = {};  // for offset / fixed placement
  double prob_user = -1;    // reaction_probability (order 2)
  double bindrad_user = -1; // binding_radius (order 2)
  double chi = -1;
  bool disabled = false;
  // derived by update (smolreact.c:1307-1577)
  double prob = 0;
  double bindrad2 = -1;
  double unbindrad = 0;
  double prdpos[kMaxProd][3] = {};
};

// Rate-based surface interaction of one (species, state, face)
// (surfactionstruct, smoldyn.h:540-548): requested rates or probabilities by
// destination state (MolecState order, soln..bsoln), their source (1 rate,
// 2 probability, 3 only a new species), the species after the action, and
// the probabilities derived from them (surfupdateparams,
// smolsurface.c:3735-3800).
struct SrfDetail {
  double rate[6] = {0, 0, 0, 0, 0, 0};
  double prob_req[6] = {0, 0, 0, 0, 0, 0};
  int datasrc[6] = {0, 0, 0, 0, 0, 0};
  int newspec[6] = {0, 0, 0, 0, 0, 0};
  double prob[6] = {0, 0, 0, 0, 0, 0};
  double cum[6] = {0, 0, 0, 0, 0, 0};
  double rev[6] = {0, 0, 0, 0, 0, 0};
};

// Molecule states a surface's action table covers: solution, front, back
// (MolecState 0..2); up and down are not supported.
constexpr int kSrfStates = 3;

struct SurfaceDef {
  std::string name;
  // action per face for all species unless overridden: 0 reflect 1 transmit 2 absorb
  int act_front = 1, act_back = 1;
  uint32_t absorb_front = 0, absorb_back = 0, trans_front = 0, trans_back = 0, refl_front = 0,
           refl_back = 0, jump_front = 0, jump_back = 0;
  // jump statements: (panel, face, partner panel, partner face), panel
  // indices within this surface, faces 0 front 1 back
  std::vector<std::array<int, 4>> jumps;
  std::vector<PanelSpec> panels;
  std::vector<std::string> pnames;   // panel names (default: shape name + index within the shape)
  // SrfAction by [species][state][face] (face 0 front, 1 back, 2 none) set
  // by action or rate statements; -1 leaves the default (solution: the masks
  // above; bound states: transmit at faces, no action otherwise)
  int act[kMaxSpecies][kSrfStates][3];
  std::map<int, SrfDetail> det;      // by (species * kSrfStates + state) * 3 + face
  std::vector<std::vector<std::pair<int, int>>> neigh;  // per panel: (surface, panel) neighbours
  int neighhop = 0;                  // neighbor_action: 0 stay, 1 hop
  SurfaceDef() {
    for (int i = 0; i < kMaxSpecies; ++i)
      for (int m = 0; m < kSrfStates; ++m)
        for (int f = 0; f < 3; ++f) act[i][m][f] = -1;
  }
};

// A molecule bound to a panel, waiting to be uploaded (absolute position).
struct PendBound {
  double pos[3] = {0, 0, 0};
  int species = 0, state = 1, surface = 0, panel = 0;
  uint64_t serno = 0;
};

struct Command {
  char type = 'E';        // 'E' every step, 'N' every n steps, 'i' interval
  double on = 0, off = 1e300, dt = 0;
  long long every = 1;
  std::string text;       // e.g. "molcount out"
  double next = 0;
};

// Compartment (smolcomparts.c compartstruct subset): a position is inside when
// the segment to one of the interior points crosses no panel of the bounding
// surfaces, combined with logic terms on earlier compartments.
struct CompartDef {
  std::string name;
  std::vector<int> surfaces;               // indices into Sim::surfaces
  std::vector<std::vector<double>> pts;    // interior-defining points
  std::vector<std::pair<int, int>> logic;  // (CmptLogic symbol, earlier compartment)
  double volume = -1;                      // Monte Carlo estimate; < 0 when not yet computed
};

// One meansqrdisp command's tracker (cmdmeansqrdisp, smolcmd.c:2505-2606):
// the molecules of `species` present on the command's first run, by
// (rep << 42) | serial, with their unwrapped start and last positions.
struct MsdState {
  bool started = false, failed = false;
  int species = 0, msddim = -1;      // msddim -1: all axes
  std::string dataname;
  std::vector<uint64_t> keys;
  std::vector<double> start, last;   // host copies; last is refreshed before an engine rebuild
  int handle = -1;                   // tracker in the current engine, -1 when it must be registered
  long long every = 0;               // steps between unwrapping passes (0: none needed)
  long long since = 0;               // steps since the last pass
};

struct Sim {
  int dim = 3;
  double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  char btype[3][2] = {{'t', 't'}, {'t', 't'}, {'t', 't'}};
  std::vector<SpeciesDef> species;   // [0] = "empty"
  std::vector<RxnDef> rxn[3];
  std::vector<SurfaceDef> surfaces;
  std::vector<CompartDef> cmpts;
  std::vector<std::string> mollists; // molecule list names (recorded only; one box-sorted array holds all)
  double tstart = 0, tstop = 0, dt = 0, time = 0;
  bool time_set = false;
  long long seed = 0;
  double molperbox = -1, boxsize = -1;
  double auto_molperbox = -1;   // box width picked by the autotuner when neither is set
  LaunchTuning tuning;          // kernel launch shape (autotuner)
  int gauss_table_size = 4096;
  long long max_mol = -1;
  int accuracy = 10;
  // molecules waiting to be uploaded (absolute positions)
  std::vector<double> pend_pos;
  std::vector<int> pend_sp;
  std::vector<uint64_t> pend_serno;   // serial numbers of the first pend_serno.size() pending molecules
  std::vector<PendBound> pend_bound;  // surface-bound molecules waiting to be uploaded
  // surface simulation parameters (surfacessalloc, smolsurface.c:1235-1237)
  double srf_epsilon = 100 * 2.220446049250313e-16, srf_margin = 100 * 2.220446049250313e-16,
         srf_neighdist = 10 * 2.220446049250313e-16;
  std::map<std::string, MsdState> msd; // meansqrdisp trackers by command text
  uint64_t host_rng = 0x853C49E6748FEA9Bull;
  // runtime commands and output data tables
  std::vector<Command> cmds;
  std::map<std::string, std::vector<std::vector<double>>> outdata;
  std::vector<std::string> outfiles;
  std::map<std::string, std::string> defines;
  std::string filepath;
  // engine state
  std::unique_ptr<Engine> eng;
  bool need_update = true;     // parameters or structure changed
  bool need_rebuild = true;    // engine must be (re)created
  long long steps = 0;
  bool started = false;
  std::string flags;

  Sim();
  int species_index(const std::string &name) const;
  int compartment_index(const std::string &name) const;
  int reaction_index(const std::string &name, int *order) const;
  double rand_u01();
  void set_seed(long long s);  // random_seed: engine key and host placement stream
};

// molsetdifm (smolmolec.c:833-867): set the diffusion matrix of a species;
// its difc becomes trace(M*M)/dim.  m is dim x dim, row-major.
void set_species_difm(Sim &sim, int sp, const double *m);
// posincompart (smolcomparts.c:119) on the host, absolute coordinates.
bool pos_in_compartment(const Sim &sim, int c, const double x[3]);
// Compartment volume (Monte Carlo over the system, fixed seed), cached.
double compartment_volume(Sim &sim, int c);
// compartrandpos (smolcomparts.c:194): a uniform position in compartment c.
void compartment_random_pos(Sim &sim, int c, double x[3]);
// n such positions appended to out (3 coordinates each).
void compartment_random_positions(Sim &sim, int c, long long n, std::vector<double> *out);
// One statement of a compartment block (surface, point, compartment logic).
int read_compartment_words(Sim &sim, int c, const std::string &word, const std::vector<std::string> &w,
                           std::string *err);
// Forget cached compartment volumes (surfaces or compartments changed).
void invalidate_compartments(Sim &sim);
// surfaddpanel (smolsurface.c:2432): a panel from its shape's parameters.
int make_panel(int dim, int shape, const std::string &axis, const double *prm, int np, PanelSpec *out,
               std::string *err);
// Restatements of the reference's parameter derivation.
int derive_reaction_params(Sim &sim, std::string *err);
// Append reaction x (order, reactants, products and their states set) after
// checking the states the engine builds; 0 or an error code with *err set.
int add_reaction_def(Sim &sim, const RxnDef &x, std::string *err);
// Restrict reaction x to surface sf (-1 lifts it); built for reactions of
// surface-bound reactants.
int set_reaction_surface(Sim &sim, RxnDef &x, int sf, std::string *err);
// Area of surface s (length in 2-D; surfacearea).
double surface_area(const Sim &sim, int s);
double panel_area_dim(const PanelSpec &p, int dim);
// rxncalcrate (smolreact.c:1592-1680): effective rate from derived parameters.
double calc_rate(const Sim &sim, int order, int r, double *pgem);
// surfupdateparams (smolsurface.c:3735-3800): derived probabilities of every
// rate-based surface interaction.
int derive_surface_params(Sim &sim, std::string *err);
// Whether any surface action can make or hold surface-bound molecules.
bool surface_bound_mode(const Sim &sim);
// Index (surface, panel) of a panel named `name` ("panel" in surface s, or
// "surface:panel"); -1 when not found.
int find_panel(const Sim &sim, int s, const std::string &name, int *srf_out);
// addsurfmol (smolmolec.c:2744): n molecules of species sp in state ms
// (1 front, 2 back) on the panels matching surface srf, shape and panel pnl
// (-1: any), chosen by area and placed uniformly on the panel, or all at pos
// when given (one panel must match).
int add_surface_molecules(Sim &sim, long long n, int sp, int ms, int srf, int shape, int pnl, const double *pos,
                          std::string *err);
// The surface_mol statement (smolsim.cpp:1027-1070).
int read_surface_mol(Sim &sim, const std::vector<std::string> &w, std::string *err);
// Surface statements for surface-bound states (action with states, rate,
// rate_internal, neighbors, neighbor_action) of surface sidx; returns 1 when
// `word` is not one of them.
int read_surface_rule_statement(Sim &sim, int sidx, const std::string &word, const std::vector<std::string> &w,
                                std::string *err);
// Name of a new panel (the given one, else shape name + index in shape).
std::string new_panel_name(const SurfaceDef &sf, int shape, const std::string &given);
// The action of (surface s, species i, state ms 0..2, face 0..2) and, for a
// rate-based one, its derived probabilities (6 destination states each).
int surface_rule_info(Sim &sim, int s, int i, int ms, int face, int *act, double *prob, double *cum, double *rev,
                      std::string *err);
// Surface rule table, bound diffusion and panel neighbours for the engine.
int build_surface_rules(const Sim &sim, NetSpec *net, std::string *err);
// Build engine inputs for a single-replicate simulation.
int build_engine_specs(Sim &sim, NetSpec *net, RepSpec *rep, std::string *err);
// Text configuration reader (statement subset of smolsim.cpp:626 simreadstring).
int read_config_statement(Sim &sim, const std::string &word, const std::string &rest, std::string *err);
int load_config_file(Sim &sim, const std::string &path, const std::string &name, std::string *err);
// findreverserxn (smolreact.c:345): 0 none, 1 direct reverse, 2 continuation.
int find_reverse_rxn(const Sim &s, int order, int r, int *o2, int *r2);

}  // namespace smolb
