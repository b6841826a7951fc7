/* Reference harness: runs ONE time step of the reference engine on a config
 * file and dumps what the deterministic parity mode needs.
 *
 * TEST INFRASTRUCTURE ONLY.  Links the reference's own engine
 * (oracle/_ref/libsmoldyn_ref.a, built from the reference sources by
 * oracle/Makefile) and wraps two of its per-step function pointers
 * (simstruct diffusefn / unimolreactfn, smoldyn.h:1070-1077) without
 * changing what they compute:
 *   - after the reference diffuse() (smolmolec.c:3115-3168) every live
 *     molecule's displacement pos - posx is recorded: posx is its position
 *     at the start of the step;
 *   - after the reference unireact() (smolreact.c:2997-3056) every molecule
 *     it killed (ident set to 0 by molkill, smolmolec.c:2676) is recorded as a
 *     forced first-order event.
 * After the step (smolRunTimeStep, libsmoldyn.cpp:217) every live molecule is
 * dumped.  Output lines (whitespace separated, %.17g):
 *   B <rxn> <bindrad2>                 second-order reactions' squared binding radius
 *   D <serno> <ident> <x0> <y0> <z0> <dx> <dy> <dz>
 *   U <serno>                          killed by a first-order reaction
 *   F <serno> <ident> <x> <y> <z>      state after the step
 *   R <order> <rxn> <rate> <pgem>      rxncalcrate (smolreact.c:1592) after update
 *   A <surface> <species> <state> <face> <action>
 *   S <surface> <species> <state> <face> <prob x6> <cumprob x6> <revprob x6>
 *                                      surface actions and, for rate-based ones,
 *                                      the probabilities surfupdateparams
 *                                      (smolsurface.c:3735) derived
 * Usage: ref_harness <dir/> <file.txt> <out.txt> [rates|surfprobs]
 * With "rates" only the R lines are written, with "surfprobs" only the A and
 * S lines (no step is run).
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "libsmoldyn.h"
#include "smoldyn.h"

/* smolreact.c:60 declares it file-locally; it has external C linkage */
extern "C" double rxncalcrate(simptr sim, int order, int r, double *pgemptr);

static FILE *g_out = NULL;
static diffusefnptr g_diffuse = NULL;
static unimolreactfnptr g_unireact = NULL;

static int wrap_diffuse(simptr sim) {
  int er = (*g_diffuse)(sim);
  if (er) return er;
  molssptr mols = sim->mols;
  for (int ll = 0; ll < mols->nlist; ll++)
    for (int m = 0; m < mols->nl[ll]; m++) {
      moleculeptr mp = mols->live[ll][m];
      if (mp->ident <= 0) continue;
      fprintf(g_out, "D %llu %d", (unsigned long long)mp->serno, mp->ident);
      for (int d = 0; d < 3; d++) fprintf(g_out, " %.17g", mp->posx[d]);
      for (int d = 0; d < 3; d++) fprintf(g_out, " %.17g", mp->pos[d] - mp->posx[d]);
      fprintf(g_out, "\n");
    }
  return 0;
}

static int wrap_unireact(simptr sim) {
  molssptr mols = sim->mols;
  /* remember which live molecules exist before the first-order reactions */
  int total = 0;
  for (int ll = 0; ll < mols->nlist; ll++) total += mols->nl[ll];
  moleculeptr *before = (moleculeptr *)calloc(total > 0 ? total : 1, sizeof(moleculeptr));
  int k = 0;
  for (int ll = 0; ll < mols->nlist; ll++)
    for (int m = 0; m < mols->nl[ll]; m++)
      if (mols->live[ll][m]->ident > 0) before[k++] = mols->live[ll][m];
  int er = (*g_unireact)(sim);
  for (int i = 0; i < k; i++)
    if (before[i]->ident == 0) fprintf(g_out, "U %llu\n", (unsigned long long)before[i]->serno);
  free(before);
  return er;
}

int main(int argc, char **argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: ref_harness <dir/> <file> <out>\n");
    return 2;
  }
  g_out = fopen(argv[3], "w");
  if (!g_out) return 2;
  simptr sim = smolPrepareSimFromFile(argv[1], argv[2], "q");
  if (!sim) {
    fprintf(stderr, "could not load %s%s\n", argv[1], argv[2]);
    return 1;
  }
  if (smolUpdateSim(sim) != ECok) return 1;
  if (argc > 4 && !strcmp(argv[4], "rates")) {
    for (int order = 0; order < 3; order++)
      if (sim->rxnss[order])
        for (int r = 0; r < sim->rxnss[order]->totrxn; r++) {
          double pgem = -1;  /* left as is when rxncalcrate returns early */
          const double rate = rxncalcrate(sim, order, r, &pgem);
          fprintf(g_out, "R %d %d %.17g %.17g\n", order, r, rate, pgem);
        }
    /* second-order parameters as rxnsetrate left them: bindrad2 and prob */
    if (sim->rxnss[2])
      for (int r = 0; r < sim->rxnss[2]->totrxn; r++)
        fprintf(g_out, "P %d %.17g %.17g\n", r, sim->rxnss[2]->rxn[r]->bindrad2, sim->rxnss[2]->rxn[r]->prob);
    fclose(g_out);
    smolFreeSim(sim);
    return 0;
  }
  if (argc > 4 && !strcmp(argv[4], "surfprobs")) {
    if (sim->srfss)
      for (int s = 0; s < sim->srfss->nsrf; s++) {
        surfaceptr srf = sim->srfss->srflist[s];
        for (int i = 1; i < sim->mols->nspecies; i++)
          for (int ms = 0; ms < 3; ms++)
            for (int face = 0; face < 3; face++) {
              const int act = (int)srf->action[i][ms][face];
              fprintf(g_out, "A %d %d %d %d %d\n", s, i, ms, face, act);
              surfactionptr ad = srf->actdetails[i][ms][face];
              if (act != (int)SAmult || !ad) continue;
              fprintf(g_out, "S %d %d %d %d", s, i, ms, face);
              for (int k = 0; k < 6; k++) fprintf(g_out, " %.17g", ad->srfprob[k]);
              for (int k = 0; k < 6; k++) fprintf(g_out, " %.17g", ad->srfcumprob[k]);
              for (int k = 0; k < 6; k++) fprintf(g_out, " %.17g", ad->srfrevprob[k]);
              fprintf(g_out, "\n");
            }
      }
    fclose(g_out);
    smolFreeSim(sim);
    return 0;
  }
  if (sim->rxnss[2])
    for (int r = 0; r < sim->rxnss[2]->totrxn; r++)
      fprintf(g_out, "B %d %.17g\n", r, sim->rxnss[2]->rxn[r]->bindrad2);
  g_diffuse = sim->diffusefn;
  g_unireact = sim->unimolreactfn;
  sim->diffusefn = wrap_diffuse;
  sim->unimolreactfn = wrap_unireact;
  enum ErrorCode ec = smolRunTimeStep(sim);
  if (ec != ECok && ec != ECnotify) return 1;
  molssptr mols = sim->mols;
  for (int ll = 0; ll < mols->nlist; ll++)
    for (int m = 0; m < mols->nl[ll]; m++) {
      moleculeptr mp = mols->live[ll][m];
      if (mp->ident <= 0) continue;
      fprintf(g_out, "F %llu %d %.17g %.17g %.17g\n", (unsigned long long)mp->serno, mp->ident, mp->pos[0],
              mp->pos[1], mp->pos[2]);
    }
  fclose(g_out);
  smolFreeSim(sim);
  return 0;
}
