/* smoldyn_b200.h -- C ABI of libsmoldyn_b200.so.
 *
 * Part 1 is a drop-in subset of Smoldyn's public C API
 * (source/Smoldyn/libsmoldyn.h): a program written against libsmoldyn that
 * uses only these calls links against libsmoldyn_b200.so unchanged and runs
 * Smoldyn's per-timestep particle engine (diffusion, walls, surfaces of all six
 * panel shapes, compartments, virtual-box binning, zeroth/first/second-order
 * reactions and product placement) on one NVIDIA B200.  Enum values equal the reference's
 * (smoldyn.h:251-512, libsmoldyn.h:13-26).  simptr is opaque here: callers that
 * read simstruct fields directly are not supported.
 *
 * Part 2 (smolgpu*) holds entry points with no libsmoldyn counterpart:
 * ensembles of independent replicates in one engine, state transfer, the
 * deterministic (injected-displacement) mode, the FP64 radius solver on the
 * device, the surrogate network, and timing hooks.
 *
 * Every function returns (or records) a status in the reference's ErrorCode
 * convention: 0 = ok, negative = notify/warning/error; the last error is kept
 * per process and read with smolGetError (libsmoldyn.cpp:23-37 behaviour).
 */
#ifndef SMOLDYN_B200_H
#define SMOLDYN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- enums (values as in the reference) ---------------------------------- */
enum ErrorCode { /* libsmoldyn.h:13-26 */
  ECok = 0, ECnotify = -1, ECwarning = -2, ECnonexist = -3, ECall = -4, ECmissing = -5,
  ECbounds = -6, ECsyntax = -7, ECerror = -8, ECmemory = -9, ECbug = -10, ECsame = -11,
  ECwildcard = -12
};
enum MolecState { /* smoldyn.h:251 */
  MSsoln, MSfront, MSback, MSup, MSdown, MSbsoln, MSall, MSnone, MSsome
};
enum RevParam { /* smoldyn.h:358 */
  RPnone, RPirrev, RPconfspread, RPbounce, RPpgem, RPpgemmax, RPpgemmaxw, RPratio, RPunbindrad,
  RPpgem2, RPpgemmax2, RPratio2, RPoffset, RPfixed
};
enum PanelFace { PFfront, PFback, PFnone, PFboth };                         /* smoldyn.h:484 */
enum PanelShape { PSrect, PStri, PSsph, PScyl, PShemi, PSdisk, PSall, PSnone }; /* smoldyn.h:491 */
enum CmptLogic { CLequal, CLequalnot, CLand, CLor, CLxor, CLandnot, CLornot, CLnone }; /* smoldyn.h:659 */
enum SrfAction {                                                             /* smoldyn.h:503 */
  SAreflect, SAtrans, SAabsorb, SAjump, SAport, SAmult, SAno, SAnone, SAadsorb, SArevdes,
  SAirrevdes, SAflip
};

typedef struct smolb_sim *simptr; /* opaque; replaces struct simstruct* (smoldyn.h:1027) */

/* ==== Part 1: libsmoldyn subset ========================================== */

/* libsmoldyn.h:37 */
double smolGetVersion(void);
/* libsmoldyn.h:44-46: last error, process-global as in the reference */
enum ErrorCode smolGetError(char *errorfunction, char *errorstring, int clearerror);
void smolClearError(void);
void smolSetDebugMode(int debugmode);
char *smolErrorCodeToString(enum ErrorCode erc, char *string);

/* libsmoldyn.h:49-55 */
simptr smolNewSim(int dim, double *lowbounds, double *highbounds);
enum ErrorCode smolUpdateSim(simptr sim);
enum ErrorCode smolRunTimeStep(simptr sim);
enum ErrorCode smolRunSim(simptr sim);
enum ErrorCode smolRunSimUntil(simptr sim, double breaktime);
enum ErrorCode smolFreeSim(simptr sim);

/* libsmoldyn.h:59-61: text configuration (statement subset, see the reader) */
simptr smolPrepareSimFromFile(const char *filepath, const char *filename, const char *flags);
enum ErrorCode smolLoadSimFromFile(const char *filepath, const char *filename, simptr *simpointer,
                                   const char *flags);
enum ErrorCode smolReadConfigString(simptr sim, const char *statement, char *parameters);

/* libsmoldyn.h:65-72 */
enum ErrorCode smolSetSimTimes(simptr sim, double timestart, double timestop, double timestep);
enum ErrorCode smolSetTimeStart(simptr sim, double timestart);
enum ErrorCode smolSetTimeStop(simptr sim, double timestop);
enum ErrorCode smolSetTimeNow(simptr sim, double timenow);
enum ErrorCode smolSetTimeStep(simptr sim, double timestep);
enum ErrorCode smolSetRandomSeed(simptr sim, long int seed);
/* method "molperbox" or "boxsize" (libsmoldyn.h:72) */
enum ErrorCode smolSetPartitions(simptr sim, const char *method, double value);

/* libsmoldyn.h:94: output data tables filled by runtime commands */
enum ErrorCode smolAddOutputData(simptr sim, char *dataname);
enum ErrorCode smolAddCommandFromString(simptr sim, char *string);
enum ErrorCode smolGetOutputData(simptr sim, char *dataname, int *nrow, int *ncol, double **array,
                                 int erase);

/* libsmoldyn.h:99-117 */
enum ErrorCode smolAddSpecies(simptr sim, const char *species, const char *mollist);
int smolGetSpeciesIndex(simptr sim, const char *species);
int smolGetSpeciesIndexNT(simptr sim, const char *species);
void smolGetSpeciesName(simptr sim, int speciesindex, char *species);
enum ErrorCode smolSetSpeciesMobility(simptr sim, const char *species, enum MolecState state,
                                      double difc, double *drift, double *difmatrix);
enum ErrorCode smolSetMaxMolecules(simptr sim, int maxmolecules);
enum ErrorCode smolAddSolutionMolecules(simptr sim, const char *species, int number,
                                        double *lowposition, double *highposition);
int smolGetMoleculeCount(simptr sim, const char *species, enum MolecState state);

/* Molecule lists (libsmoldyn.h:108-112, libsmoldyn.cpp:954-1035).  The
 * reference's live lists are a CPU data-structure choice; the engine keeps
 * one box-sorted array for all species, so list names are recorded and
 * validated as the reference does (ECwarning for a repeated name, ECsame for
 * an unknown one in smolAddSpecies/smolSetMolList) and have no other effect. */
enum ErrorCode smolAddMolList(simptr sim, const char *mollist);
int smolGetMolListIndex(simptr sim, const char *mollist);
int smolGetMolListIndexNT(simptr sim, const char *mollist);
char *smolGetMolListName(simptr sim, int mollistindex, char *mollist);
enum ErrorCode smolSetMolList(simptr sim, const char *species, enum MolecState state, const char *mollist);

/* Display (libsmoldyn.h:55, :76, :104-105, :118).  No graphics stack is
 * driven: the arguments are checked as in the reference (libsmoldyn.cpp:
 * 295, 485, 1147-1216) and otherwise ignored; smolDisplaySim prints a short
 * text summary of the simulation to stdout (the reference prints its full
 * parameter listing, simsystemoutput). */
enum ErrorCode smolDisplaySim(simptr sim);
enum ErrorCode smolSetGraphicsParams(simptr sim, const char *method, int timesteps, int delay);
enum ErrorCode smolSetMoleculeColor(simptr sim, const char *species, enum MolecState state, double *color);
enum ErrorCode smolSetMoleculeSize(simptr sim, const char *species, enum MolecState state, double size);
enum ErrorCode smolSetMoleculeStyle(simptr sim, const char *species, enum MolecState state, double size,
                                    double *color);

/* libsmoldyn.h:122-130: walls and surfaces.  Actions reflect, transmit and
 * absorb, for the solution, front and back states, optionally changing the
 * species (jump and port are not supported). */
enum ErrorCode smolSetBoundaryType(simptr sim, int dimension, int highside, char type);
enum ErrorCode smolAddSurface(simptr sim, const char *surface);
enum ErrorCode smolSetSurfaceAction(simptr sim, const char *surface, enum PanelFace face,
                                    const char *species, enum MolecState state,
                                    enum SrfAction action, const char *newspecies);
enum ErrorCode smolAddPanel(simptr sim, const char *surface, enum PanelShape panelshape,
                            const char *panel, const char *axisstring, double *params);

/* Surface-bound states (libsmoldyn.h:116, :129, :136-137; smolsurface.c
 * surfsetrate :2278, surfsetneighbors :3150, addsurfmol smolmolec.c:2744).
 * Single simulations only.  States soln, front, back and bsoln; rates of
 * adsorption, desorption, flips between faces and one-way transmission
 * (isinternal: the value is a probability per event); molecules bound to a
 * panel diffuse on it (any panel shape) and continue onto
 * neighbouring panels; first-order reactions of bound molecules with at
 * most one product.  The up and down states, surface drift and bimolecular
 * reactions of bound molecules are not supported. */
enum ErrorCode smolSetSurfaceRate(simptr sim, const char *surface, const char *species, enum MolecState state,
                                  enum MolecState state1, enum MolecState state2, double rate,
                                  const char *newspecies, int isinternal);
enum ErrorCode smolAddSurfaceMolecules(simptr sim, const char *species, enum MolecState state, int number,
                                       const char *surface, enum PanelShape panelshape, const char *panel,
                                       double *position);
enum ErrorCode smolAddPanelNeighbor(simptr sim, const char *surface1, const char *panel1, const char *surface2,
                                    const char *panel2, int reciprocal);
enum ErrorCode smolSetSurfaceSimParams(simptr sim, const char *parameter, double value);
/* The action of (surface, species, state soln/front/back, face front/back/
 * none) and, for a rate-based action, the probabilities derived from its
 * rates (surfupdateparams, smolsurface.c:3735-3800): prob, cumprob and
 * revprob, 6 destination states each (MolecState order soln..bsoln). */
enum ErrorCode smolgpuGetSurfaceRule(simptr sim, const char *surface, const char *species, enum MolecState state,
                                     enum PanelFace face, int *action, double *prob, double *cumprob,
                                     double *revprob);

/* Compartments (libsmoldyn.h:115, :142-148, :157): interior-defining points,
 * bounding surfaces and logic on earlier compartments; molecules placed
 * uniformly inside; reactions restricted to a compartment (zeroth order:
 * births inside at rate x compartment volume; first order: the molecule must
 * be inside; second order: both reactants).  At most 8 compartments, 8 points
 * and 4 logic terms each. */
enum ErrorCode smolAddCompartment(simptr sim, const char *compartment);
int smolGetCompartmentIndex(simptr sim, const char *compartment);
int smolGetCompartmentIndexNT(simptr sim, const char *compartment);
char *smolGetCompartmentName(simptr sim, int compartmentindex, char *compartment);
enum ErrorCode smolAddCompartmentSurface(simptr sim, const char *compartment, const char *surface);
enum ErrorCode smolAddCompartmentPoint(simptr sim, const char *compartment, double *point);
enum ErrorCode smolAddCompartmentLogic(simptr sim, const char *compartment, enum CmptLogic logic,
                                       const char *compartment2);
enum ErrorCode smolAddCompartmentMolecules(simptr sim, const char *species, int number, const char *compartment);
/* A surface restriction applies to reactions of surface-bound reactants
 * (they fire only for molecules bound to that surface); for other reactions
 * it is refused. */
enum ErrorCode smolSetReactionRegion(simptr sim, const char *reaction, const char *compartment, const char *surface);

/* libsmoldyn.h:152-158 */
enum ErrorCode smolAddReaction(simptr sim, const char *reaction, const char *reactant1,
                               enum MolecState rstate1, const char *reactant2,
                               enum MolecState rstate2, int nproduct, const char **productspecies,
                               enum MolecState *productstates, double rate);
int smolGetReactionIndex(simptr sim, int *orderptr, const char *reaction);
enum ErrorCode smolSetReactionRate(simptr sim, const char *reaction, double rate, int type);
enum ErrorCode smolSetReactionProducts(simptr sim, const char *reaction, enum RevParam method,
                                       double parameter, const char *product, double *position);
/* Alias: smolAddReaction with a non-empty reactant2 (no separate entry exists
 * in the reference; provided because callers look for this name). */
enum ErrorCode smolAddBimolecularReaction(simptr sim, const char *reaction, const char *reactant1,
                                          const char *reactant2, int nproduct,
                                          const char **productspecies, double rate);

/* ==== Part 2: smolgpu extensions ========================================= */

/* Derived reaction parameters after smolUpdateSim (reference fields
 * rxn->bindrad2, rxn->unbindrad, rxn->prob; smolreact.c:1307-1577). */
enum ErrorCode smolgpuGetReactionParams(simptr sim, const char *reaction, double *bindrad,
                                        double *unbindrad, double *prob);
/* Effective rate constant implied by the derived parameters (rxncalcrate,
 * smolreact.c:1592-1680; the reference computes it for its "measured vs
 * requested" rate report).  *pgem (optional): geminate recombination
 * probability for a reaction with two products and a reverse, else -1.
 * Host FP64 only; no engine is built. */
enum ErrorCode smolgpuGetEffectiveRate(simptr sim, const char *reaction, double *rate, double *pgem);
/* Simulated time and step counter. */
double smolgpuGetTime(simptr sim);
long long smolgpuGetStepCount(simptr sim);
/* Number of live molecules (all species). */
long long smolgpuGetTotalMolecules(simptr sim);
/* Copy the solution-phase molecules to host arrays (pos: 3*n doubles,
 * absolute coordinates; species: n ints; serno: n uint64).  *n is in:
 * capacity, out: count. */
enum ErrorCode smolgpuGetMolecules(simptr sim, long long *n, double *pos, int *species,
                                   uint64_t *serno);
/* The same for surface-bound molecules, with their state (MSfront, MSback),
 * surface index and panel index within the surface; sorted by serial number. */
enum ErrorCode smolgpuGetSurfaceMolecules(simptr sim, long long *n, double *pos, int *species, int *state,
                                          int *surface, int *panel, uint64_t *serno);
/* Replace the molecule set (absolute coordinates; serno 0 = assign). */
enum ErrorCode smolgpuSetMolecules(simptr sim, long long n, const double *pos, const int *species,
                                   const uint64_t *serno);
/* Event counters since start: [0]=wall [1]=rxn0 [2]=rxn1 [3]=rxn2 [4]=unresolved
 * pair conflicts [5]=multi-candidate molecules [6]=capacity overflows. */
enum ErrorCode smolgpuGetEventCounts(simptr sim, long long counts[8]);

/* Deterministic mode: while set, the next smolRunTimeStep uses displacement
 * (dx,dy,dz) = disp[3*k..3*k+2] for the molecule whose serno equals sernos[k]
 * instead of drawing Gaussian steps (molecules not listed do not move), and
 * every first-order / pair coin uses 0 (always fires when allowed).  n=0 clears. */
enum ErrorCode smolgpuSetInjectedDisplacements(simptr sim, long long n, const uint64_t *sernos,
                                               const double *disp);

/* Device stream the engine launches on (a cudaStream_t passed as void*); NULL
 * = the engine's own stream.  Lets a caller time launches with its own events. */
enum ErrorCode smolgpuSetStream(simptr sim, void *stream);
/* Number of engine kernel launches issued since the sim was created. */
long long smolgpuGetLaunchCount(simptr sim);
/* Advance n time steps with no runtime commands (the hot loop of smolRunSim,
 * smolsim.cpp:2755, as one replayed CUDA graph of two steps per launch). */
enum ErrorCode smolgpuRunSteps(simptr sim, long long nsteps);
/* Advance n steps launching kernels one by one and timing each with CUDA
 * events.  On return names[k*32..] holds kernel k's name, ms[k] its summed
 * device time and launches[k] its launch count, for k < *nkernels (in: array
 * capacity, out: number of kernels). */
enum ErrorCode smolgpuProfileSteps(simptr sim, long long nsteps, int *nkernels, char *names, double *ms,
                                   long long *launches);
/* Synchronise the engine's stream. */
enum ErrorCode smolgpuSynchronize(simptr sim);
/* Autotuner (no reference counterpart: the reference's box size comes from
 * molperbox/boxsize, smolboxes.c:717-749).  Runs timed trial steps from the
 * current state over box widths (1, 2, 4, 8 molecules per box, only when the
 * configuration sets neither molperbox nor boxsize), pair-search tile size and
 * blocks per SM, and streaming-kernel blocks per SM; keeps the fastest and
 * restores the molecules and step counter, so the trajectory is the untuned
 * one up to FP32 rounding of box-local coordinates.  Call after smolUpdateSim
 * and before the first time step.  *ms_per_step (optional) = best trial. */
enum ErrorCode smolgpuAutotune(simptr sim, int trial_steps, double *ms_per_step);
/* The current choice (molperbox -1 when boxsize is set). */
enum ErrorCode smolgpuGetTuning(simptr sim, double *molperbox, int *pair_tile, int *tile_blocks_per_sm,
                                int *mol_blocks_per_sm);

/* FP64 radius solver, batched on the device (rxnparam.c:558-716 on the GPU).
 * mode 0: bindingradius(rate[i], dt, difc[i], b[i], rel) -> out[i]
 * mode 1: unbindingradius(pgem=rate[i], dt, difc[i], a=b[i]) -> out[i]
 * Host arrays of length n. */
enum ErrorCode smolgpuSolveRadii(int mode, long long n, const double *rate, double dt,
                                 const double *difc, const double *b, int rel, double *out);
/* smolgpuSolveRadii without device allocation; no counterpart in the
 * reference.  Inputs and outputs pass through a fixed 2 MiB scratch in static
 * device memory, so callers that cannot allocate (a radius update issued
 * while an ensemble steps on another stream, where cudaMalloc/cudaFree could
 * synchronise the device; a process whose HBM is already full) can still
 * solve.  At most 65536 problems per call (ECbounds above that).  The
 * scratch is shared per device and keeps the last call's contents: calls
 * that overlap on the GPU race and must be serialised by the caller.  The
 * first call on a device sets up the scratch address (cudaGetSymbolAddress);
 * under CUDA's lazy module loading that can load the library's device code,
 * which places the scratch in device memory and may synchronise, so make the
 * first call at set-up time, before HBM is filled and before any stream
 * capture.  The address is cached per device: after cudaDeviceReset the
 * library must be reloaded.  Copies are synchronous cudaMemcpy and the kernel
 * runs on the legacy default stream, which waits for every blocking stream of
 * the process: the call overlaps only work on streams created with
 * cudaStreamNonBlocking (the engine's own streams are). */
enum ErrorCode smolgpuSolveRadiiNoAlloc(int mode, long long n, const double *rate, double dt,
                                        const double *difc, const double *b, int rel, double *out);
/* Same solver on the host CPU (product path used by parameter updates). */
double smolgpuBindingRadiusHost(double rate, double dt, double difc, double b, int rel);
/* Reaction probability p < 1 on the host, the product path of every
 * second-order reaction's parameter derivation: numrxnrateprob
 * (rxnparam.c:161-518) and bindingradiusprob (rxnparam.c:587-681, prob in/out
 * as in the reference: with chi < 0 *prob is the given probability, with
 * chi >= 0 it receives the probability found by the 2-D search). */
double smolgpuNumRxnRateProbHost(double step, double a, double b, double prob);
double smolgpuBindingRadiusProbHost(double rate, double dt, double difc, double b, int rel, double chi,
                                    double *prob);
/* bindingradiusprob batched on the device, one problem per element:
 * out[i] = bindingradiusprob(rate[i], dt, difc[i], b[i], rel, chi[i], &prob[i]).
 * Host arrays of length n; prob is read and written. */
enum ErrorCode smolgpuSolveRadiiProb(long long n, const double *rate, double dt, const double *difc,
                                     const double *b, int rel, const double *chi, double *prob, double *out);
double smolgpuUnbindingRadiusHost(double pgem, double dt, double difc, double a);

/* Radial-distribution-function solver on the device: the numerical method
 * behind the rxnparam tables (rxnparam.c:784-1114), in reduced units
 * (binding radius 1 for the sweeps).
 *
 * smolgpuRdfTable replaces rdfmaketable (rxnparam.c:920) and, with probs,
 * rdfmaketableprob (rxnparam.c:1008), without their terminal dialogue:
 *   mode 'i' irreversible (1 row), 'r' reversible with unbinding radius
 *   b = 1 .. e^3 (16 rows), 'b' reversible with b = 0 .. 1 (11 rows);
 *   n radial points (10..4000), eps the relative flux tolerance;
 *   dir 'u' step lengths e^-3 .. e^3 increasing, 'd' decreasing, or 'a' both
 *   sweeps averaged and listed in decreasing order (the form of the tables in
 *   numrxnrate, rxnparam.c:58-76);
 *   probs: nprob reaction probabilities (NULL: one probability of 1).
 * flux[(row*nprob + p)*31 + k] receives the steady-state flux (the reduced
 * rate; -1 where rdfsteadystate gives up, and for the rest of that sweep as in
 * the reference), iters (optional) the iteration counts, *nrows (optional)
 * the row count.  flux must hold rows*nprob*31 doubles. */
enum ErrorCode smolgpuRdfTable(char mode, int n, double eps, char dir, int nprob, const double *probs,
                               double *flux, int *iters, int *nrows);
/* Batched rdfsteadystate (rxnparam.c:898): nsolve independent solves on n-point
 * grids r (nsolve*n; r[0] >= 0, the others > 0) from trial profiles rdfa
 * (in/out, nsolve*n; out: after the last absorption) with step[i], binding
 * radius a[i], unbinding radius b[i] (< 0: irreversible) and probability
 * prob[i].  rdfd (optional, nsolve*n) receives the profile after the last
 * diffusion step, flux[i] the steady-state flux or -1, iters (optional) the
 * iteration counts. */
enum ErrorCode smolgpuRdfSteadyState(int nsolve, int n, const double *r, double *rdfa, double *rdfd,
                                     const double *step, const double *a, const double *b, const double *prob,
                                     double eps, double *flux, int *iters);
/* The rate tables compiled into this library (numrxnrate, numrxnrateprob;
 * rxnparam.c:58-76, 172-490): name "yi", "yr", "yb", "kirr", "krev" or "kb".
 * Copies min(cap, length) values to out (out may be NULL) and returns the
 * table length, or -1 for an unknown name. */
int smolgpuRxnTable(const char *name, double *out, int cap);

/* ==== Part 2b: ensembles of independent replicates ====================== */
/* One engine runs nrep independent copies of a template simulation (its
 * species, reactions, product placement, walls, dt and seed), each with its
 * own box and rate constants, in one launch sequence.  Arrays are per
 * replicate (boxes: nrep*dim values; counts out: nrep*nspecies with species
 * index 0 = "empty").  Rate-derived parameters follow smolreact.c:1307-1577 per
 * replicate; radius mode 0 = exact FP64 on the host, 1 = exact FP64 on the
 * device (default), 2 = MLP surrogate with exact fallback. */
typedef struct smolb_ens *ensptr;
typedef struct smolb_surrogate *surptr;
ensptr smolgpuNewEnsemble(simptr templ, int nrep);
enum ErrorCode smolgpuEnsembleSetBoxes(ensptr ens, const double *low, const double *high);
enum ErrorCode smolgpuEnsembleSetRates(ensptr ens, const char *reaction, const double *rates);
enum ErrorCode smolgpuEnsembleAddMolecules(ensptr ens, const char *species, const int *counts);
enum ErrorCode smolgpuEnsembleSetRadiusMode(ensptr ens, int mode);
enum ErrorCode smolgpuEnsembleAttachSurrogate(ensptr ens, surptr sur);
/* Which engine steps the ensemble: mode 0 (default) automatic, currently the
 * step pipeline, which measures faster on B200; 1 the step pipeline (the
 * device-wide launch sequence of a single simulation, all replicates in each
 * launch); 2 the persistent kernel (ECerror when the configuration has
 * surfaces, compartments or injected displacements).  The persistent kernel
 * gives each replicate to one thread block, which runs up to 100 whole time
 * steps of it per launch (move, box sort, pair search, conflict rounds,
 * products), one captured graph per launch, from an L2-resident working set;
 * it uses the step pipeline's per-molecule code and random streams, so both
 * engines give the same trajectories up to the ranking of equidistant
 * candidates.  smolgpuEnsembleGetEngine returns 1 or 2, the engine the next
 * step uses. */
enum ErrorCode smolgpuEnsembleSetEngine(ensptr ens, int mode);
int smolgpuEnsembleGetEngine(ensptr ens);
enum ErrorCode smolgpuEnsembleUpdate(ensptr ens);
enum ErrorCode smolgpuEnsembleRunSteps(ensptr ens, long long nsteps);
enum ErrorCode smolgpuEnsembleGetCounts(ensptr ens, long long *counts);
/* Event counters summed over the ensemble since it was built, as
 * smolgpuGetEventCounts: wall hits, zeroth-, first- and second-order events,
 * unresolved conflicts, extra candidates, status word. */
enum ErrorCode smolgpuEnsembleGetEventCounts(ensptr ens, long long counts[8]);
/* All molecules of all replicates, sorted by (replicate, serial number):
 * pos 3*n doubles (absolute coordinates of the replicate's box), species,
 * replicate index and serial number per molecule; *n is in: capacity, out:
 * count (NULL arrays: count only). */
enum ErrorCode smolgpuEnsembleGetMolecules(ensptr ens, long long *n, double *pos, int *species, int *rep,
                                           uint64_t *serno);
enum ErrorCode smolgpuEnsembleGetReactionParams(ensptr ens, const char *reaction, double *bindrad,
                                                double *unbindrad);
long long smolgpuEnsembleGetFallbackCount(ensptr ens);
enum ErrorCode smolgpuEnsembleSetStream(ensptr ens, void *stream);
long long smolgpuEnsembleGetLaunchCount(ensptr ens);
enum ErrorCode smolgpuEnsembleSynchronize(ensptr ens);
/* Autotuner for an ensemble (same search as smolgpuAutotune; box width per
 * replicate from its own molecule count). */
enum ErrorCode smolgpuEnsembleAutotune(ensptr ens, int trial_steps, double *ms_per_step);
enum ErrorCode smolgpuEnsembleGetTuning(ensptr ens, double *molperbox, int *pair_tile, int *tile_blocks_per_sm,
                                        int *mol_blocks_per_sm);
enum ErrorCode smolgpuEnsembleFree(ensptr ens);

/* ==== Part 2c: MLP surrogate of the radius solve ========================= */
/* 3->64->64->2 tanh network on x = (log10 k/(D*s), unbinding ratio, reversible
 * flag) -> y = (log10 a/s, b/s), s = sqrt(2*D*dt); trained on the device from
 * samples of the exact FP64 solver (x: n*3, y: n*2 doubles).  Inference uses
 * BF16 weights with FP32 accumulation and falls back to the exact solver when
 * one numrxnrate evaluation shows a relative rate error above the tolerance
 * (default 1e-3). */
surptr smolgpuSurrogateNew(void);
enum ErrorCode smolgpuSurrogateFree(surptr sur);
enum ErrorCode smolgpuSurrogateTrain(surptr sur, long long nsamples, int epochs, int batch, double lr,
                                     unsigned long long seed, double *final_loss, double *seconds);
enum ErrorCode smolgpuSurrogateSamples(surptr sur, long long n, unsigned long long seed, double *x, double *y);
enum ErrorCode smolgpuSurrogateForward(surptr sur, long long n, const double *x, double *y);
enum ErrorCode smolgpuSurrogateLossGrad(surptr sur, long long n, const double *x, const double *y, double *loss,
                                        float *grad);
int smolgpuSurrogateParamCount(void);
enum ErrorCode smolgpuSurrogateGetParams(surptr sur, float *params);
enum ErrorCode smolgpuSurrogateSetParams(surptr sur, const float *params);
enum ErrorCode smolgpuSurrogateSetTolerance(surptr sur, double tol);
enum ErrorCode smolgpuSurrogatePairRadii(surptr sur, long long n, const double *kf, const double *dsum, double dt,
                                         int same, int rev, int rparamt, double rparam, double *bind,
                                         double *unbind, long long *nfallback);

#ifdef __cplusplus
}
#endif
#endif /* SMOLDYN_B200_H */
