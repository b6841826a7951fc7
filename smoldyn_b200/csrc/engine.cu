// B200 particle engine: kernels and host driver.
//
// One time step (Smoldyn smolsim.cpp:2607-2692 order) is the launch sequence
//   k_begin          step counter, per-step counters
//   k_move           diffuse + walls + first-order decisions for every molecule
//                    (moved position to tmp, events for the ones that leave),
//                    histogram of destination virtual boxes (one atomic each),
//                    then zeroth-order births (Poisson per replicate and reaction)
//   k_scan           single-pass exclusive scan of box counts -> box starts
//   k_scatter        permutation of the moved molecules into box order
//   k_pairs_tile     same-box pairs from a shared-memory tile of sorted
//                    molecules; molecules near a box face are queued
//   k_pairs_faces    cross-box pairs of the queued molecules
//   k_commit / k_research (rounds) mutual-closest pairs react, losers retry
//   k_products       product placement (site, unbinding offsets under one random
//                    rotation per event), walls for the new molecules
// Molecules live in two ping-pong box-sorted SoA buffers (float4 position in
// box-local FP32 coordinates with the box index packed in .w, plus a 64-bit
// identity word) and two ping-pong product buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <utility>
#include <vector>

#include "devcommon.cuh"
#include "engine.h"
#include "rxnparam.cuh"
#include "panelgeom.cuh"
#include "boundgeom.cuh"

namespace smolb {

__constant__ DevNet c_net;
__constant__ DevPanel c_panels[kMaxPanels];
__constant__ DevCmpt c_cmpt[kMaxCmpt];
__constant__ DevGeo c_geo0;  // geometry of replicate 0 (used when the engine holds one replicate)

struct KParams {
  const DevGeo *geo;
  const float *difstep;    // [rep*nsp + sp]  sqrt(2 D dt)
  const float *driftdt;    // [(rep*nsp + sp)*3] drift*dt or null
  const float *difm;       // [(rep*nsp + sp)*9] sqrt(2 dt) * diffusion matrix (species in difm_any)
  const uint32_t *unithr;  // [(rep*nsp + sp)*kMaxUniPerSpecies] cumulative thresholds
  const float *bind2;      // [rep*nr2 + r]
  const float *pairprob;   // [rep*nr2 + r]
  const float *rsearch;    // [rep*nsp + sp] stencil radius of the pair search
  const uint16_t *boxmask; // [global box] panels that a short move starting in the box can reach
  const double *births;    // [rep*nr0 + r]
  const float *prdpos;     // [((rep*nrx + k)*kMaxProd + p)*3]
  const float *gtab;       // gaussian table
  // molecules: a = sorted input, p = product input, b = sorted output, q = product output
  const float4 *a_pc;
  ull *a_id;
  const int *a_n;
  const float4 *p_pc;
  const ull *p_id;
  const int *p_n;
  float4 *b_pc;
  ull *b_id;
  int *b_n;
  float4 *q_pc;
  ull *q_id;
  int *q_n;
  float4 *tmp;   // moved positions of the step's inputs (sorted input, then products)
  int cap, pcap;
  int *cnt;
  int *start;
  int ncell;
  Event *ev;
  int *nev;
  int evcap;
  int *cand;
  int *ncand;
  int candcap;
  ull *best;
  int *face;                     // molecules near a box face (cross-box pair search)
  unsigned long long *counters;  // [0]=wall [1]=rxn0 [2]=rxn1 [3]=rxn2 [4]=unresolved [5]=multicand
  long long *spcount;            // [rep*nsp + sp]
  int *status;
  uint32_t *step;
  // deterministic mode
  const ull *inj_key;            // sorted stream keys
  const float4 *inj_val;         // dx, dy, dz, forced order-1 reaction (or -1)
  int inj_n;
  // surface-bound molecules (single simulations with surface-bound states)
  const SrfRule *srfrule;        // [((surface*kMaxSpecies + sp)*3 + state)*3 + face]
  const BoundMol *bd_in;
  const int *bd_in_n;
  BoundMol *bd_out;
  int *bd_out_n;
  int bcap;
  // bound-solution pair reactions: per sorted molecule the best claim of a
  // bound molecule (all ones when unclaimed), per bound molecule its
  // candidate (partner, reaction, squared distance bits, state)
  ull *bclaim;
  int4 *bcand;
  // bound-bound pair reactions: hash-grid heads, per bound molecule the next
  // entry of its bucket, its box, and its best partner (priority << 32 | index)
  int *bbhead;
  int *bbnext;
  ull *bbcell;
  ull *bbbest;
};

constexpr uint32_t kTmpGone = 0xFFFFFFFFu;  // tmp[i].w of a molecule that left
// Set in the packed box word of a product-list entry that has already been
// moved this step (a molecule that desorbed from a surface): the move pass
// only re-bins it and draws its first-order reactions.
constexpr uint32_t kMovedBit = 1u << 30;

enum StatusBits { kStMolCap = 1, kStEvCap = 2, kStProdCap = 4, kStCandCap = 8, kStScanWait = 16, kStUpload = 32,
                  kStBoundCap = 64 };

// Programmatic dependent launch: the step's kernels are launched so that the
// next kernel can be scheduled while the current one runs.  Each kernel lets
// its dependent launch as soon as all of its blocks have started, and waits
// for its predecessor to complete (with memory visible) before it touches
// anything the predecessor wrote.  Both instructions are no-ops when the
// kernel was launched without the attribute.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Arithmetic helpers of the move path (plain IEEE single precision; the
// compiler may contract a multiply and an add into one FMA).
__device__ __forceinline__ float fadd(float a, float b) { return a + b; }
__device__ __forceinline__ float fsub(float a, float b) { return a - b; }
__device__ __forceinline__ float fmul(float a, float b) { return a * b; }

// Bring local coordinate w (relative to the origin of cell j, j maybe out of
// range) into cell form.
__device__ __forceinline__ void renorm(float &w, int &j, float h, float inv_h) {
  if (w >= 0.f && w < h) return;
  // one box over: the common case when a step crosses a face
  if (w < 0.f && w >= -h) {
    j -= 1;
    w = fadd(w, h);
    if (w < h) return;
    w = fsub(w, h);  // rounding put it on the face: stay in the original box
    j += 1;
    return;
  }
  if (w >= h && w < fadd(h, h)) {
    j += 1;
    w = fsub(w, h);
    if (w >= 0.f) return;
    w = fadd(w, h);
    j -= 1;
    return;
  }
  const int k = (int)floorf(fmul(w, inv_h));
  j += k;
  w = fsub(w, fmul((float)k, h));
  if (w < 0.f) { j -= 1; w = fadd(w, h); }
  else if (w >= h) { j += 1; w = fsub(w, h); }
}

// Apply the low and high wall of one dimension to (w, j) (smolwall.c:368-427,
// low wall first).  Returns 1 if the molecule crossed an absorbing wall.
__device__ __forceinline__ int walls_dim(float &w, int &j, const DevGeo &g, int d, int &hits) {
  const float h = g.h[d], inv_h = g.inv_h[d], whi = g.whi[d];
  const int n = g.n[d];
  if (j < 0) {  // beyond the low wall (position j*h + w < 0)
    const int kind = g.wall[2 * d];
    hits++;
    if (kind == kWallReflect) {
      const float q = -fadd(fmul((float)j, h), w);
      j = 0;
      w = q;
      renorm(w, j, h, inv_h);
    } else if (kind == kWallPeriodic) {
      j += n;
      w = fadd(w, fsub(whi, h));
      renorm(w, j, h, inv_h);
    } else if (kind == kWallAbsorb) {
      return 1;
    } else {
      w = fadd(fmul((float)j, h), w);
      j = 0;
    }
  }
  if (j >= n - 1) {
    // signed distance beyond the high wall
    const float e = fsub(fadd(fmul((float)(j - (n - 1)), h), w), whi);
    if (e > 0.f) {
      const int kind = g.wall[2 * d + 1];
      hits++;
      if (kind == kWallReflect) {
        j = n - 1;
        w = fsub(whi, e);
        renorm(w, j, h, inv_h);
        if (j < 0) {  // reflected past the low wall too (step longer than the box)
          if (g.wall[2 * d] == kWallReflect) {
            w = -fadd(fmul((float)j, h), w);
            j = 0;
            renorm(w, j, h, inv_h);
          } else {
            w = fadd(fmul((float)j, h), w);
            j = 0;
          }
        }
      } else if (kind == kWallPeriodic) {
        j -= n;
        w = fadd(w, fsub(h, whi));
        renorm(w, j, h, inv_h);
      } else if (kind == kWallAbsorb) {
        return 1;
      } else {
        w = fadd(e, whi);
        j = n - 1;
      }
    } else if (j > n - 1) {  // inside the box but past the nominal last cell
      w = fadd(e, whi);
      j = n - 1;
    }
  }
  return 0;
}

// Last line of defence for the box index: a displacement of several box
// lengths in one step (huge D*dt) or a non-finite position must still give an
// in-range box, so the index is clamped and the local offset kept relative to
// that box.  Only pathological inputs reach the clamp.
__device__ __forceinline__ void clamp_cell(float &w, int &j, const DevGeo &g, int d) {
  if (!(w == w)) w = 0.f;  // NaN
  const int n = g.n[d];
  if (j < 0) {
    if (g.wall[2 * d] == kWallPeriodic && j > -(1 << 20)) {
      const int k = (-j + n - 1) / n;
      j += k * n;
    } else {
      w = fadd(w, fmul((float)j, g.h[d]));
      j = 0;
    }
  }
  if (j > n - 1) {
    if (g.wall[2 * d + 1] == kWallPeriodic && j < (1 << 20)) {
      const int k = j / n;
      j -= k * n;
    } else {
      w = fadd(w, fmul((float)(j - (n - 1)), g.h[d]));
      j = n - 1;
    }
  }
  if (j < 0) j = 0;
  if (j > n - 1) j = n - 1;
}

// Distance of a (cell, local) coordinate from the low / high wall.
__device__ __forceinline__ float dist_low(int j, float w, float h) { return fadd(fmul((float)j, h), w); }
__device__ __forceinline__ float dist_high(int j, float w, const DevGeo &g, int d) {
  return fsub(fadd(fmul((float)(g.n[d] - 1 - j), g.h[d]), g.whi[d]), w);
}

__device__ __forceinline__ int find_injection(const KParams &p, ull key) {
  int lo = 0, hi = p.inj_n - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const ull k = p.inj_key[mid];
    if (k == key) return mid;
    if (k < key) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

// Geometry of a replicate: from constant memory when the engine holds one
// replicate (a plain simulation), else from the per-replicate table.
template <bool SINGLE>
__device__ __forceinline__ const DevGeo &geo_of(const KParams &p, int rep) {
  if (SINGLE) return c_geo0;
  return p.geo[rep];
}

// ---- surfaces ---------------------------------------------------------------
// Solution-phase molecules against sphere and axis-aligned rectangle panels,
// restating checksurfaces (smolsurface.c:5114-5182): walk the segment from the
// previous position to the new one, take the nearest panel crossing, apply
// the face's action (dosurfinteract :4930 - reflect about the tangent plane
// at the crossing point (surfacereflect :4821), transmit, or absorb), restart
// from the crossing point nudged to the proper side (fixpt2panel :4460), and
// stop after 100 rounds by returning the molecule to its prior position.
// FP64 throughout: the positions come from exact conversions of the FP32
// box-local coordinates.

// action of panel pn on species sp arriving at face (0 front, 1 back)
__device__ __forceinline__ int panel_action(const DevPanel &pn, int face, int sp) {
  const uint32_t bit = 1u << sp;
  if (face == 0) {
    if (pn.jp_front & bit) return 3;
    if (pn.abs_front & bit) return 2;
    if (pn.tr_front & bit) return 1;
    if (pn.rf_front & bit) return 0;
    return pn.act_front;
  }
  if (pn.jp_back & bit) return 3;
  if (pn.abs_back & bit) return 2;
  if (pn.tr_back & bit) return 1;
  if (pn.rf_back & bit) return 0;
  return pn.act_back;
}

// Jump (surfacejump, smolsurface.c:4873-4927): a solution molecule that
// crosses `face` of panel pn at x moves to the partner panel by the shape's
// offset (rectangle, triangle, disk: between the panels' centres; sphere,
// hemisphere, cylinder: the crossing point scaled between the two radii),
// with the rest of its path; the crossing point is put on the partner's face,
// and the path is reflected there when the two faces point the same way.
// Returns false when the face leads nowhere (the molecule then transmits);
// else x is the new crossing point (on the partner's face), out the unit
// normal pointing to that face's side, and p1 the path's end.
template <bool GEN>
__device__ __noinline__ bool panel_jump(const DevPanel &pn, int face, double x[3], double p1[3], double out[3]) {
  const int k2 = pn.jump_pnl[face];
  if (k2 < 0) return false;
  const DevPanel &pn2 = c_panels[k2];
  const int face2 = pn.jump_face[face];
  double delta[3];
  int dir = 1;
  if (pn.shape == 0) {
    for (int d = 0; d < 3; ++d) {
      const double c1 = d == pn.axis ? pn.pos : 0.5 * (pn.lo[d] + pn.hi[d]);
      const double c2 = d == pn2.axis ? pn2.pos : 0.5 * (pn2.lo[d] + pn2.hi[d]);
      delta[d] = c2 - c1;
    }
    dir = pn.front_sign == pn2.front_sign ? 1 : -1;
  } else if (pn.shape == 1 || pn.shape == 5) {
    for (int d = 0; d < 3; ++d)
      delta[d] = pn.shape == 1 ? ((pn2.pt[0][d] + pn2.pt[1][d] + pn2.pt[2][d]) - (pn.pt[0][d] + pn.pt[1][d] + pn.pt[2][d])) / 3.0
                               : pn2.center[d] - pn.center[d];
    dir = dot3(pn.nrm, pn2.nrm) > 0 ? 1 : -1;
  } else {
    const double *o1 = pn.shape == 3 ? pn.pt[0] : pn.center, *o2 = pn2.shape == 3 ? pn2.pt[0] : pn2.center;
    const double f = pn.radius > 0 ? pn2.radius / pn.radius : 1.0;
    for (int d = 0; d < 3; ++d) delta[d] = (x[d] - o1[d]) * f + o2[d] - x[d];
    dir = pn.front_sign == pn2.front_sign ? 1 : -1;
  }
  for (int d = 0; d < 3; ++d) {
    x[d] += delta[d];
    p1[d] += delta[d];
  }
  fix_to_panel(pn2, x, face2 == 0 ? kFaceFront : kFaceBack, 0.0);
  if (face == face2) dir = -dir;
  if (dir == -1) {  // the path would leave on the wrong side: it turns back at the partner (surfacereflect)
    double n[3];
    panel_normal<GEN>(pn2, x, n);
    double dt = 0;
    for (int d = 0; d < 3; ++d) dt += (p1[d] - x[d]) * n[d];
    for (int d = 0; d < 3; ++d) p1[d] -= 2.0 * dt * n[d];
  }
  panel_normal<GEN>(pn2, x, out);
  if (face2 != 0)
    for (int d = 0; d < 3; ++d) out[d] = -out[d];
  return true;
}

// Returns 1 if the molecule is absorbed; p1 is updated in place.
// FP32 screen for the surface walk: false when the move a0 -> a1 (absolute
// coordinates) stays more than the margin away from every panel, so no
// crossing and no eps adjustment can occur.  Conservative: flat panels are
// tested as their whole plane; spheres and hemispheres through the distances
// of the end points from the centre, cylinders from the infinite axis (the
// distance is 1-Lipschitz along the move, so a segment that starts farther
// than its length outside cannot reach the surface).
template <bool GEN>
__device__ __forceinline__ bool surface_near(const float a0[3], const float a1[3], const uint16_t *boxmask,
                                             int box0) {
  const float tol = c_net.surf_tol;
  const float sx = a1[0] - a0[0], sy = a1[1] - a0[1], sz = a1[2] - a0[2];
  const float seg = sqrtf(sx * sx + sy * sy + sz * sz);
  // a short move can only reach the panels listed for its start box
  uint32_t mask = 0xFFFFFFFFu;
  if (boxmask && seg <= c_net.mask_len) {
    mask = boxmask[box0];
    if (!mask) return false;
  }
  for (int k = 0; k < c_net.npanel; ++k) {
    if (!((mask >> k) & 1u)) continue;
    const DevPanel &pn = c_panels[k];
    if (pn.shape == 0) {  // axis-aligned rectangle: its plane along one axis
      const float q0 = a0[pn.axis] - pn.posf, q1 = a1[pn.axis] - pn.posf;
      if ((q0 > tol && q1 > tol) || (q0 < -tol && q1 < -tol)) continue;
      return true;
    }
    // other shapes: offsets from the panel's reference point; for tri, disk
    // and cyl also their components along the panel's unit vector
    float w0[3], w1[3];
    for (int d = 0; d < 3; ++d) {
      w0[d] = a0[d] - pn.p0f[d];
      w1[d] = a1[d] - pn.p0f[d];
    }
    float q0 = w0[0] * w0[0] + w0[1] * w0[1] + w0[2] * w0[2];
    float q1 = w1[0] * w1[0] + w1[1] * w1[1] + w1[2] * w1[2];
    if (GEN && (pn.shape == 1 || pn.shape == 3 || pn.shape == 5)) {
      const float s0 = w0[0] * pn.nrmf[0] + w0[1] * pn.nrmf[1] + w0[2] * pn.nrmf[2];
      const float s1 = w1[0] * pn.nrmf[0] + w1[1] * pn.nrmf[1] + w1[2] * pn.nrmf[2];
      if (!pn.curved) {  // tri, disk: the whole plane
        if ((s0 > tol && s1 > tol) || (s0 < -tol && s1 < -tol)) continue;
        return true;
      }
      q0 -= s0 * s0;  // cyl: distance from the infinite axis
      q1 -= s1 * s1;
    }
    // curved: distance from the centre (sph, hemi) or the axis (cyl)
    const float r = pn.radiusf;
    const float d0 = sqrtf(fmaxf(q0, 0.f)), d1 = sqrtf(fmaxf(q1, 0.f));
    if (d0 - seg > r + tol) continue;              // the whole move stays outside
    if (fmaxf(d0, d1) < r - tol) continue;         // the whole move stays inside
    return true;
  }
  return false;
}

template <bool GEN>
__device__ int surface_interact(int sp, const double p0_in[3], double p1[3], double eps, int &hits) {
  const int np = c_net.npanel;
  double p0[3] = {p0_in[0], p0_in[1], p0_in[2]};
  for (int it = 0; it < 100; ++it) {
    double tmin = 2.0;
    int kmin = -1, fmin = 0;
    for (int k = 0; k < np; ++k) {
      int f = 0;
      const double t = panel_cross<GEN>(c_panels[k], p0, p1, f);
      if (t < tmin) { tmin = t; kmin = k; fmin = f; }
    }
    if (kmin < 0) {
      // keep the final position at least eps off every panel, on its side
      for (int k = 0; k < np; ++k) {
        const double sd = panel_sdist<GEN>(c_panels[k], p1);
        if (fabs(sd) < eps) {
          double n[3];
          panel_normal<GEN>(c_panels[k], p1, n);
          const double side = (sd > 0 || (sd == 0 && panel_sdist<GEN>(c_panels[k], p0) > 0)) ? 1.0 : -1.0;
          for (int d = 0; d < 3; ++d) p1[d] += (side * eps - sd) * n[d];
        }
      }
      return 0;
    }
    hits++;
    const DevPanel &pn = c_panels[kmin];
    const int act = panel_action(pn, fmin, sp);
    if (act == 2) return 1;
    double x[3], n[3];
    for (int d = 0; d < 3; ++d) x[d] = p0[d] + tmin * (p1[d] - p0[d]);
    if (GEN && act == 3 && panel_jump<GEN>(pn, fmin, x, p1, n)) {  // on from just off the partner's face (general form)
      for (int d = 0; d < 3; ++d) p0[d] = x[d] + eps * n[d];
      continue;
    }
    panel_normal<GEN>(pn, x, n);
    const double side = (fmin == 0) ? 1.0 : -1.0;  // incoming side along n
    if (act == 0) {
      double dot = 0;
      for (int d = 0; d < 3; ++d) dot += (p1[d] - x[d]) * n[d];
      for (int d = 0; d < 3; ++d) p1[d] -= 2.0 * dot * n[d];
      for (int d = 0; d < 3; ++d) p0[d] = x[d] + side * eps * n[d];
    } else {
      for (int d = 0; d < 3; ++d) p0[d] = x[d] - side * eps * n[d];
    }
  }
  for (int d = 0; d < 3; ++d) p1[d] = p0_in[d];  // gave up: prior position
  return 0;
}

// absolute position (relative to the low corner) of a box-local coordinate
__device__ __forceinline__ void to_abs(const DevGeo &g, const int ix[3], const float u[3], double x[3]) {
  for (int d = 0; d < 3; ++d) x[d] = (double)ix[d] * (double)g.h[d] + (double)u[d];
}

// back to box-local form (walls are transparent once surfaces exist)
__device__ __forceinline__ void from_abs(const DevGeo &g, const double x[3], int ix[3], float u[3]) {
  for (int d = 0; d < 3; ++d) {
    const double h = (double)g.h[d];
    int j = (int)floor(x[d] / h);
    if (j < 0) j = 0;
    if (j > g.n[d] - 1) j = g.n[d] - 1;
    ix[d] = j;
    u[d] = (float)(x[d] - (double)j * h);
  }
}

// True when the segment between two molecules crosses a surface panel: such
// pairs do not react (rxnXsurface, used by bireact smolreact.c:3238).
template <bool GEN>
__device__ __forceinline__ bool pair_crosses_surface(const DevGeo &g, float4 pc, float vx, float vy, float vz) {
  int ix[3];
  unpack_cell(__float_as_uint(pc.w), ix[0], ix[1], ix[2]);
  const float u[3] = {pc.x, pc.y, pc.z};
  double a[3], b[3];
  to_abs(g, ix, u, a);
  b[0] = a[0] + vx;
  b[1] = a[1] + vy;
  b[2] = a[2] + vz;
  for (int k = 0; k < c_net.npanel; ++k) {
    int f;
    if (panel_cross<GEN>(c_panels[k], a, b, f) <= 1.0) return true;
  }
  return false;
}

// the same test as a call, for kernels whose hot loop should not carry the
// panel arithmetic's registers
template <bool GEN>
__device__ __noinline__ bool pair_crosses_surface_call(const DevGeo &g, float4 pc, float vx, float vy, float vz) {
  return pair_crosses_surface<GEN>(g, pc, vx, vy, vz);
}

// ---- surface-bound states --------------------------------------------------
// Adsorption, desorption, flips and surface-bound diffusion (dosurfinteract
// smolsurface.c:4930, surfaction :4330, checksurfacebound :5184,
// movemol2closepanel :4726), for single simulations.  Solution molecules meet
// panels in the move pass and may adsorb; bound molecules live in their own
// list (FP64 absolute positions, panel and state) that k_bound steps before
// the move pass: diffusion projected onto the panel, crossings of other
// panels, then the per-step desorption / flip coin.  A molecule that desorbs
// joins the product list already moved (kMovedBit), so the move pass only
// bins it and draws its first-order reactions, as the reference lets a
// desorbed molecule react in the step it desorbs.

enum SrfActs { kSAreflect = 0, kSAtrans = 1, kSAabsorb = 2, kSAjump = 3, kSAport = 4, kSAmult = 5, kSAno = 6,
               kSAnone = 7, kSAadsorb = 8, kSArevdes = 9, kSAirrevdes = 10, kSAflip = 11 };
enum MolStates { kMSsoln = 0, kMSfront = 1, kMSback = 2, kMSbsoln = 5 };

// random word streams of a molecule (Philox counter word 3) for the surface paths
constexpr uint32_t kCtrSrfWalk = 0x100u;   // + iteration: collision coins of a solution molecule
constexpr uint32_t kCtrSrfWalk2 = 0x200u;  // + iteration: the same for the placement walk after desorption
constexpr uint32_t kCtrSrfBound = 0x300u;  // desorption / flip coin and desorption distance
constexpr uint32_t kCtrSrfDiff = 0x301u;   // diffusion of a bound molecule
constexpr uint32_t kCtrSrfRxn = 0x302u;    // first-order reaction coin of a bound molecule
constexpr uint32_t kCtrSrfRot = 0x303u;    // rotation of that reaction's product offsets
constexpr uint32_t kCtrSrfBWalk = 0x400u;  // + iteration: collision coins of a bound molecule
constexpr uint32_t kCtrSrfEdge = 0x1000u;  // + 64 * iteration (+ 1 + neighbour): panel-edge choices

__device__ __forceinline__ uint4 srf_draw(ull skey, uint32_t step, uint32_t word) {
  const uint2 key = make_uint2(c_net.key0 ^ 0x68E31DA4u, c_net.key1 ^ 0xB5297A4Du);
  return philox(make_uint4((uint32_t)skey, (uint32_t)(skey >> 32), step, word), key);
}
// [0,1) with 32-bit resolution (randCOD), and [0,1] (randCCD)
__device__ __forceinline__ double u01co(uint32_t x) { return (double)x * (1.0 / 4294967296.0); }
__device__ __forceinline__ double u01cc(uint32_t x) { return (double)x * (1.0 / 4294967295.0); }

__device__ __forceinline__ const SrfRule &srf_rule(const KParams &p, int srf, int sp, int ms, int face) {
  return p.srfrule[((srf * kMaxSpecies + sp) * 3 + (ms == kMSbsoln ? 0 : ms)) * 3 + face];
}

// surfaction (smolsurface.c:4330-4385): the action for species sp in state ms
// meeting `face` of a panel of surface srf (kFaceNone: the per-step coin of
// a bound molecule), with the species and state it ends in.
__device__ int srf_action(const KParams &p, int srf, int sp, int ms, int face, uint32_t coin, int &sp2, int &ms2) {
  const SrfRule &r = srf_rule(p, srf, sp, ms, face);
  int act = r.act;
  if (act != kSAmult) {
    ms2 = ms == kMSbsoln ? kMSsoln : ms;
    sp2 = r.newspec[ms2];
    return act;
  }
  const double u = u01co(coin);
  int k = 0;
  while (k < 5 && !(u < r.cum[k])) ++k;
  ms2 = k;
  sp2 = r.newspec[k];
  const bool to_soln = k == kMSsoln || k == kMSbsoln;
  if (k != kMSsoln && k != kMSfront && k != kMSback && k != kMSbsoln) {  // up / down: never built
    ms2 = ms;
    sp2 = sp;
    return face == kFaceNone ? kSAno : kSAtrans;
  }
  if (sp2 == 0) return kSAabsorb;
  if (ms != kMSsoln && face == kFaceNone) {
    if (k == ms) return kSAno;
    if (to_soln) return ((r.rev >> k) & 1u) ? kSArevdes : kSAirrevdes;
    return kSAflip;
  }
  if (face == kFaceFront) return k == kMSsoln ? kSAreflect : k == kMSbsoln ? kSAtrans : kSAadsorb;
  return k == kMSsoln ? kSAtrans : k == kMSbsoln ? kSAreflect : kSAadsorb;
}

// desorbdist (SurfaceParam.c:202-220): distance from the surface at which a
// desorbing molecule is placed, from a uniform y in [0,1]; rational fits for
// irreversible and for reversible desorption.
__device__ __forceinline__ double desorb_dist(double step, bool reversible, double y) {
  const double y2 = y * y;
  if (reversible) return step * (0.729614 * y - 0.70252 * y2) / (1.0 - 1.47494 * y + 0.484371 * y2);
  return step * (0.571825 * y - 0.552246 * y2) / (1.0 - 1.53908 * y + 0.546424 * y2);
}

__device__ __forceinline__ int ms_face(int ms) { return ms == kMSback ? kFaceBack : kFaceFront; }

// movemol2closepanel (smolsurface.c:4726-4818): bring a bound molecule that
// diffused from posx (on panel pnl) to pos back onto the surface.  The move
// is projected onto the panel; if it leaves the panel's outline it continues
// on a neighbouring panel that shares the exit point (picked uniformly among
// those that do), rotated about the shared edge into that panel's plane, or
// bounces off the edge when there is none.
__device__ void move_to_close_panel(double pos[3], const double posx[3], int &pnl, int ms, ull skey, uint32_t step) {
  const int face = ms_face(ms);
  const double eps = c_net.beps, margin = c_net.bmargin, nd = c_net.bneighdist;
  int cur = pnl;
  fix_to_panel(c_panels[cur], pos, face, eps);
  if (pt_in_panel(c_panels[cur], pos)) return;
  double via[3];
  if (pt_in_panel(c_panels[cur], posx))
    for (int d = 0; d < 3; ++d) via[d] = posx[d];
  else
    closest_panel_pt(c_panels[cur], pos, via, 0.0);
  for (int iter = 1;; ++iter) {
    const DevPanel &pc = c_panels[cur];
    double edge[3];
    int exitside = 1;
    const int er = line_exit_panel(pc, via, pos, edge, &exitside);
    if (er || iter > 50) {
      move_into_panel(pc, pos, margin);
      fix_to_panel(pc, pos, face, eps);
      break;
    }
    const uint4 rr = srf_draw(skey, step, kCtrSrfEdge + 64u * (uint32_t)iter);
    int nn = 0, newp = -1, newedge = 0;
    double newpt[3] = {0, 0, 0};
    for (int q = 0; q < pc.nneigh; ++q) {  // a random neighbour meeting this edge point
      double pt[3];
      const int en = closest_panel_pt(c_panels[pc.neigh[q]], edge, pt, 1000.0 * nd);
      double d2 = 0;
      for (int d = 0; d < 3; ++d) d2 += (pt[d] - edge[d]) * (pt[d] - edge[d]);
      if (d2 < nd) {
        ++nn;
        if (nn == 1 || u01co(srf_draw(skey, step, kCtrSrfEdge + 64u * (uint32_t)iter + 1u + (uint32_t)q).x) < 1.0 / nn) {
          newp = pc.neigh[q];
          newedge = en;
          for (int d = 0; d < 3; ++d) newpt[d] = pt[d];
        }
      }
    }
    if (nn) {
      for (int d = 0; d < 3; ++d) pos[d] += newpt[d] - edge[d];  // close any gap between the edges
      const DevPanel &pn = c_panels[newp];
      double nnew[3];
      face_normal(pn, newpt, face, nnew);
      if (newedge) {  // the path crosses onto the new panel through its edge
        double nold[3], en[3], np[3];
        face_normal(pc, edge, face, nold);
        panel_edge_normal(pn, newpt, newedge, en);
        double dt = 0;
        for (int d = 0; d < 3; ++d) dt += (pos[d] - newpt[d]) * en[d];
        const int ts = dt > 0 ? -1 : 1;
        rotate_with_normals(newpt, pos, np, nold, nnew, ts);
        if (fabs(dt) < 0.01) {  // check the side when in doubt
          double d2 = 0;
          for (int d = 0; d < 3; ++d) d2 += (np[d] - newpt[d]) * en[d];
          if (d2 > 0) rotate_with_normals(newpt, pos, np, nold, nnew, -ts);
        }
        for (int d = 0; d < 3; ++d) pos[d] = np[d];
      } else {  // enters mid-panel: the reference rotates from a random direction
        const double ro[3] = {2.0 * u01cc(rr.x) - 1.0, 2.0 * u01cc(rr.y) - 1.0, 2.0 * u01cc(rr.z) - 1.0};
        double np[3];
        rotate_with_normals(newpt, pos, np, ro, nnew, 0);
        for (int d = 0; d < 3; ++d) pos[d] = np[d];
      }
      cur = newp;
    } else {  // no neighbour: bounce off the edge
      double en[3];
      panel_edge_normal(pc, edge, exitside, en);
      double dt = 0;
      for (int d = 0; d < 3; ++d) dt += (pos[d] - edge[d]) * en[d];
      for (int d = 0; d < 3; ++d) pos[d] -= 2.0 * en[d] * dt;
      for (int d = 0; d < 3; ++d) newpt[d] = edge[d];
    }
    fix_to_panel(c_panels[cur], pos, face, eps);
    for (int d = 0; d < 3; ++d) via[d] = newpt[d];
    if (pt_in_panel(c_panels[cur], pos)) break;
  }
  pnl = cur;
}

// checksurfaces (smolsurface.c:5114-5182) for a solution molecule moving
// p0 -> p1 when surface rules are in use: each crossing applies the rule of
// the panel's surface for (species, solution, face).  Returns 0 in solution
// at p1 (species sp possibly changed), 1 removed, 2 adsorbed: p1 is then its
// place on panel *pnl_out in state *ms_out.  Solution molecules are kept
// surf_eps off panels, as in surface_interact.
__device__ int walk_soln_rules(const KParams &p, int &sp, const double p0_in[3], double p1[3], int &hits, ull skey,
                               uint32_t step, uint32_t ctr, int &pnl_out, int &ms_out) {
  const int np = c_net.npanel;
  const double eps = c_net.surf_eps;
  double p0[3] = {p0_in[0], p0_in[1], p0_in[2]};
  for (int it = 0; it < 100; ++it) {
    double tmin = 2.0;
    int kmin = -1, fmin = 0;
    for (int k = 0; k < np; ++k) {
      int f = 0;
      const double t = panel_cross<true>(c_panels[k], p0, p1, f);
      if (t < tmin) { tmin = t; kmin = k; fmin = f; }
    }
    if (kmin < 0) {
      for (int k = 0; k < np; ++k) {
        const double sd = panel_sdist<true>(c_panels[k], p1);
        if (fabs(sd) < eps) {
          double n[3];
          panel_normal<true>(c_panels[k], p1, n);
          const double side = (sd > 0 || (sd == 0 && panel_sdist<true>(c_panels[k], p0) > 0)) ? 1.0 : -1.0;
          for (int d = 0; d < 3; ++d) p1[d] += (side * eps - sd) * n[d];
        }
      }
      return 0;
    }
    hits++;
    const DevPanel &pn = c_panels[kmin];
    int sp2, ms2;
    const int act = srf_action(p, pn.srf, sp, kMSsoln, fmin, srf_draw(skey, step, ctr + (uint32_t)it).x, sp2, ms2);
    if (act == kSAabsorb) return 1;
    double x[3], n[3];
    for (int d = 0; d < 3; ++d) x[d] = p0[d] + tmin * (p1[d] - p0[d]);
    if (act == kSAjump && panel_jump<true>(pn, fmin, x, p1, n)) {  // on from just off the partner's face
      for (int d = 0; d < 3; ++d) p0[d] = x[d] + eps * n[d];
      continue;
    }
    if (act == kSAadsorb) {
      for (int d = 0; d < 3; ++d) p1[d] = x[d];
      if (!pt_in_panel(pn, p1)) move_into_panel(pn, p1, c_net.bmargin);
      fix_to_panel(pn, p1, ms_face(ms2), c_net.beps);
      sp = sp2;
      pnl_out = kmin;
      ms_out = ms2;
      return 2;
    }
    panel_normal<true>(pn, x, n);
    const double side = (fmin == 0) ? 1.0 : -1.0;
    if (act == kSAreflect) {
      double dot = 0;
      for (int d = 0; d < 3; ++d) dot += (p1[d] - x[d]) * n[d];
      for (int d = 0; d < 3; ++d) p1[d] -= 2.0 * dot * n[d];
      for (int d = 0; d < 3; ++d) p0[d] = x[d] + side * eps * n[d];
    } else {
      for (int d = 0; d < 3; ++d) p0[d] = x[d] - side * eps * n[d];
    }
    if (sp2 != sp) {  // molchangeident: the rest of the step at the new species' diffusion
      const double f = c_net.sstep[sp] > 0 ? c_net.sstep[sp2] / c_net.sstep[sp] : 1.0;
      for (int d = 0; d < 3; ++d) p1[d] = x[d] + f * (p1[d] - x[d]);
      sp = sp2;
    }
  }
  for (int d = 0; d < 3; ++d) p1[d] = p0_in[d];
  return 0;
}

// The per-step coin of a bound molecule (checksurfacebound :5184 through
// dosurfinteract with no face, :5022-5052): returns 0 still bound (a flip
// changes state and species in place), 1 removed, 2 desorbed - x0 is then
// the point on the panel it leaves from, x1 its place in solution
// (desorbdist along the face's normal) and sp its species.
__device__ int bound_coin(const KParams &p, BoundMol &m, int &sp, ull skey, uint32_t step, double x0[3], double x1[3]) {
  const DevPanel &pn = c_panels[m.pnl];
  const uint4 r = srf_draw(skey, step, kCtrSrfBound);
  int sp2, ms2;
  const int act = srf_action(p, pn.srf, sp, m.ms, kFaceNone, r.x, sp2, ms2);
  if (act == kSAabsorb) return 1;
  if (act == kSArevdes || act == kSAirrevdes) {
    const int f = ms2 == kMSsoln ? kFaceFront : kFaceBack;
    for (int d = 0; d < 3; ++d) x0[d] = m.x[d];
    fix_to_panel(pn, x0, f, c_net.beps);
    const double dist = desorb_dist(c_net.sstep[sp2], act == kSArevdes, u01cc(r.y));
    double n[3];
    face_normal(pn, x0, f, n);
    for (int d = 0; d < 3; ++d) x1[d] = x0[d] + dist * n[d];
    sp = sp2;
    return 2;
  }
  if (act == kSAflip) {
    m.ms = ms2;
    sp = sp2;
    fix_to_panel(pn, m.x, ms_face(ms2), c_net.beps);
  }
  return 0;
}

__device__ __forceinline__ void random_orientation(uint4 r, int dim, float m[9]);
__device__ __forceinline__ void push_bound(const KParams &p, const BoundMol &m);

// Place product q of first-order reaction r of bound molecule m (doreact,
// smolreact.c:2806-2880): the reactant's place, kept on the product state's
// side of its panel (fixpt2panel), displaced by the product's offset under
// the reaction's random rotation R, and brought back onto the surface
// (movemol2closepanel; a solution product takes the front or back state for
// that, as the reference does, so its offset off the panel is dropped).
__device__ void bound_product_place(const KParams &p, const BoundMol &m, int r, int q, int pst, const float R[9],
                                    bool rot, ull skey, uint32_t step, double x[3], int &pnl) {
  const int f = (pst == kMSback || pst == kMSbsoln) ? kFaceBack : kFaceFront;
  double x0[3] = {m.x[0], m.x[1], m.x[2]};
  fix_to_panel(c_panels[m.pnl], x0, f, c_net.beps);
  for (int d = 0; d < 3; ++d) x[d] = x0[d];
  if (rot) {
    const float *pp = p.prdpos + ((size_t)(c_net.rxn_base[1] + r) * kMaxProd + q) * 3;  // single simulation
    for (int d = 0; d < 3; ++d)
      x[d] += (double)R[3 * d] * pp[0] + (double)R[3 * d + 1] * pp[1] + (double)R[3 * d + 2] * pp[2];
  }
  pnl = m.pnl;
  const ull k2 = mix64(skey ^ (0xB0A1ull + (ull)q)) & ((1ull << kSpShift) - 1);  // its own edge choices
  move_to_close_panel(x, x0, pnl, f == kFaceBack ? kMSback : kMSfront, k2, step);
}

// First-order reactions of a bound molecule (unireact on the bound state,
// smolreact.c:2997-3056, after the surface actions as in the reference's step
// order), with the sequential-coin thresholds of its species and state.
// Products (doreact, smolreact.c:2662-2902) start from the reactant's place:
// bound ones on its panel on their state's side, solution ones just off the
// panel's front (soln) or back (bsoln) side in the output product list, so
// that, like the reference's products, they first move in the next step;
// with two products, their offsets (unbinding radius split by diffusion
// coefficients) turn under one random rotation.  The first bound product, or
// else the first product, takes over the reactant's entry and count; another
// product is counted here.  Returns 0 no reaction, 1 reacted without product,
// 2 the reactant's entry became a bound product (m, sp updated), 3 it became
// a solution product in the product list (sp updated).
__device__ int bound_first_order(const KParams &p, BoundMol &m, int &sp, ull skey, uint32_t step) {
  const int st = m.ms - 1;
  const int nr = c_net.buni_n[sp][st];
  if (!nr) return 0;
  const uint32_t u = srf_draw(skey, step, kCtrSrfRxn).x;
  const uint32_t *thr = c_net.bthr[sp][st];
  int k = 0;
  while (k < nr && !(u < thr[k])) ++k;
  // A reaction restricted to a surface or a compartment fires only on that
  // surface or inside it (unireact smolreact.c:3040-3050); otherwise the
  // decision passes to the reactions after it in the list, each with its own
  // coin: with a fresh uniform, the first k' > k with
  // u' < 1 - (1 - cum_k') / (1 - cum_k), as for solution molecules.
  for (int round = 0; k < nr; ++round) {
    const int rk = c_net.buni_list[sp][st][k];
    const int rs = c_net.rsrf[1][rk], cm = c_net.cmpt[1][rk];
    if ((!rs || c_panels[m.pnl].srf == rs - 1) && (!cm || pos_in_cmpt(c_cmpt, cm - 1, c_panels, m.x))) break;
    const double uu = ((double)srf_draw(skey, step, kCtrSrfRxn + 0x10u + (uint32_t)round).x + 0.5) * (1.0 / 4294967296.0);
    const double rest = 1.0 - (double)thr[k] * (1.0 / 4294967296.0);
    int next = nr;
    for (int k2 = k + 1; k2 < nr; ++k2)
      if (rest > 0 && uu < 1.0 - (1.0 - (double)thr[k2] * (1.0 / 4294967296.0)) / rest) { next = k2; break; }
    k = next;
  }
  if (k >= nr) return 0;
  const int r = c_net.buni_list[sp][st][k];
  atomicAdd(&p.counters[2], 1ull);
  const int np = min((int)c_net.nprod[1][r], 2);
  if (np == 0) return 1;
  float R[9];
  const bool rot = c_net.has_offset[1][r] != 0;
  if (rot) random_orientation(srf_draw(skey, step, kCtrSrfRot), c_geo0.dim, R);
  int q0 = 0;  // the product that takes over the reactant's entry
  for (int q = np - 1; q >= 0; --q)
    if (c_net.pstate1[r][q] == kMSfront || c_net.pstate1[r][q] == kMSback) q0 = q;
  const BoundMol m0 = m;
  int ret = 0;
  for (int q = 0; q < np; ++q) {
    const int psp = c_net.prd[1][r][q], pst = c_net.pstate1[r][q];
    double x[3];
    int pnl;
    bound_product_place(p, m0, r, q, pst, R, rot, skey, step, x, pnl);
    const ull sn = q == q0 ? id_serno(m0.id)
                           : kProductSernoBit | (mix64(skey ^ ((ull)step << 20) ^ ((ull)(q + 1) << 50) ^ 0x51D0ull) &
                                                 (kProductSernoBit - 1));
    if (pst == kMSfront || pst == kMSback) {
      BoundMol b;
      for (int d = 0; d < 3; ++d) b.x[d] = x[d];
      b.pnl = pnl;
      b.ms = pst;
      b.id = make_id(psp, 0, sn);
      b.born = step;  // products react from the next step on, as the reference's join its lists then
      if (q == q0) {
        m = b;
        sp = psp;
        ret = 2;
      } else {
        push_bound(p, b);
        atomicAdd((unsigned long long *)&p.spcount[psp], 1ull);
      }
      continue;
    }
    const int f = pst == kMSbsoln ? kFaceBack : kFaceFront;
    const DevPanel &pn = c_panels[pnl];
    double n[3];
    face_normal(pn, x, f, n);
    const double sd = fabs(panel_sdist<true>(pn, x));
    if (sd < c_net.surf_eps)  // kept surf_eps off the panel, as solution molecules are
      for (int d = 0; d < 3; ++d) x[d] += (c_net.surf_eps - sd) * n[d];
    int ix[3];
    float w[3];
    from_abs(c_geo0, x, ix, w);
    const int slot = atomicAdd(p.q_n, 1);
    if (slot < p.pcap) {
      p.q_pc[slot] = make_float4(w[0], w[1], w[2], __uint_as_float(pack_cell(ix[0], ix[1], ix[2])));
      p.q_id[slot] = make_id(psp, 0, sn);
    } else {
      atomicOr(p.status, kStProdCap);
    }
    if (q == q0) {
      sp = psp;
      ret = 3;
    } else {
      atomicAdd((unsigned long long *)&p.spcount[psp], 1ull);
    }
  }
  return ret;
}

// Crossings of other panels by a bound molecule's move from posx (on panel
// pnlx) to m.x (checksurfaces on a surface-bound molecule, dosurfinteract
// :4930-5020): a neighbouring panel is crossed (transmit) or, with
// neighbor_action hop, hopped onto with probability 1/2; other panels apply
// their surface's rule for the molecule's state.  Returns 0 still bound, 1
// removed.
__device__ int walk_bound(const KParams &p, BoundMol &m, int &sp, const double posx[3], int pnlx, int &hits, ull skey,
                          uint32_t step) {
  const int np = c_net.npanel;
  const double eps = c_net.beps;
  double via[3] = {posx[0], posx[1], posx[2]};
  for (int it = 0; it < 100; ++it) {
    double tmin = 2.0;
    int kmin = -1, fmin = 0;
    for (int k = 0; k < np; ++k) {
      if (k == m.pnl) continue;
      int f = 0;
      const double t = panel_cross<true>(c_panels[k], via, m.x, f);
      if (t < tmin) { tmin = t; kmin = k; fmin = f; }
    }
    if (kmin < 0) return 0;
    hits++;
    double x[3];
    for (int d = 0; d < 3; ++d) x[d] = via[d] + tmin * (m.x[d] - via[d]);
    const DevPanel &pk = c_panels[kmin];
    const DevPanel &pm = c_panels[m.pnl];
    bool neigh = false;
    for (int q = 0; q < pm.nneigh; ++q) neigh = neigh || pm.neigh[q] == kmin;
    const uint4 r = srf_draw(skey, step, kCtrSrfBWalk + (uint32_t)it);
    int act, sp2 = sp, ms2 = m.ms;
    if (neigh) act = (pm.neighhop && u01co(r.y) < 0.5) ? kSAadsorb : kSAtrans;
    else act = srf_action(p, pk.srf, sp, m.ms, fmin, r.x, sp2, ms2);
    if (act == kSAabsorb) return 1;
    if (act == kSAadsorb) {  // onto panel kmin
      const int old = m.pnl, oldms = m.ms;
      for (int d = 0; d < 3; ++d) m.x[d] = x[d];
      if (!pt_in_panel(pk, m.x)) move_into_panel(pk, m.x, c_net.bmargin);
      fix_to_panel(c_panels[old], m.x, ms_face(oldms), eps);
      fix_to_panel(pk, m.x, ms_face(ms2), eps);
      m.pnl = kmin;
      m.ms = ms2;
      sp = sp2;
      return 0;
    }
    if (act == kSAreflect) {  // reflection within the plane of the starting panel (surfacereflect :4852-4868)
      double n[3], n2[3];
      face_normal(pk, x, fmin, n);
      face_normal(c_panels[pnlx], x, kFaceFront, n2);
      const double c = dot3(n, n2);
      for (int d = 0; d < 3; ++d) n[d] -= c * n2[d];
      double l = sqrt(dot3(n, n));
      if (l == 0) l = 1;
      for (int d = 0; d < 3; ++d) n[d] /= l;
      double a = 0, b = 0;
      for (int d = 0; d < 3; ++d) a += (m.x[d] - x[d]) * n2[d];
      for (int d = 0; d < 3; ++d) m.x[d] -= n2[d] * a;
      for (int d = 0; d < 3; ++d) b += (m.x[d] - x[d]) * n[d];
      for (int d = 0; d < 3; ++d) m.x[d] -= 2.0 * n[d] * b;
      fix_to_panel(pk, x, fmin, eps);
      m.pnl = pnlx;
      move_to_close_panel(m.x, posx, m.pnl, m.ms, skey, step);
      if (panel_side(pk, m.x, nullptr) != fmin) {  // went to the wrong side: back to the prior place
        for (int d = 0; d < 3; ++d) m.x[d] = posx[d];
        m.pnl = pnlx;
        return 0;
      }
    } else {  // transmit (and no action)
      fix_to_panel(pk, x, fmin == kFaceFront ? kFaceBack : kFaceFront, eps);
    }
    if (sp2 != sp) {
      const double f = c_net.bstep[sp][m.ms - 1] > 0 ? c_net.bstep[sp2][m.ms - 1] / c_net.bstep[sp][m.ms - 1] : 1.0;
      for (int d = 0; d < 3; ++d) m.x[d] = x[d] + f * (m.x[d] - x[d]);
      sp = sp2;
    }
    for (int d = 0; d < 3; ++d) via[d] = x[d];
  }
  for (int d = 0; d < 3; ++d) m.x[d] = posx[d];
  m.pnl = pnlx;
  return 0;
}

__device__ __forceinline__ void push_bound(const KParams &p, const BoundMol &m) {
  const int k = atomicAdd(p.bd_out_n, 1);
  if (k < p.bcap) {
    p.bd_out[k] = m;
  } else {
    atomicSub(p.bd_out_n, 1);
    atomicOr(p.status, kStBoundCap);
  }
}

// species count moves with a species change (single simulations: replicate 0)
__device__ __forceinline__ void move_count(const KParams &p, int from, int to) {
  if (from == to) return;
  atomicAdd((unsigned long long *)&p.spcount[from], (unsigned long long)(-1ll));
  atomicAdd((unsigned long long *)&p.spcount[to], 1ull);
}

// The move pass's surface step for a solution molecule when surface rules are
// in use.  Returns 1 when the molecule is removed, 3 when it was bound
// (appended to the output bound list after its per-step coin and first-order
// reactions, or turned by one into a product in the product list), else 0 with
// the molecule in solution at x1 (a molecule that adsorbs and desorbs again
// within the step stays in solution at its desorbed place); species changes
// update *id and the species counts.
__device__ __noinline__ int soln_surface_bound(const KParams &p, ull &id, const double x0[3], double x1[3], int &hits,
                                               uint32_t step) {
  const ull skey = id_stream(id);
  const int sp0 = id_species(id);
  int sp = sp0, pnl = 0, ms = 0;
  const int w = walk_soln_rules(p, sp, x0, x1, hits, skey, step, kCtrSrfWalk, pnl, ms);
  if (w == 1) return 1;
  if (w == 2) {
    BoundMol m;
    for (int d = 0; d < 3; ++d) m.x[d] = x1[d];
    m.pnl = pnl;
    m.ms = ms;
    m.id = make_id(sp, 0, id_serno(id));
    m.born = kBornNever;
    double y0[3], y1[3];
    const int c = bound_coin(p, m, sp, skey, step, y0, y1);
    if (c == 1) return 1;
    if (c == 0) {  // still bound: its first-order reactions this step
      const int r = bound_first_order(p, m, sp, skey, step);
      if (r == 1) return 1;
      if (r == 3) {  // a solution product, in the output product list
        move_count(p, sp0, sp);
        return 3;
      }
    }
    bool bound = true;
    if (c == 2) {
      int pnl2 = 0, ms2 = 0;
      const int w2 = walk_soln_rules(p, sp, y0, y1, hits, skey, step, kCtrSrfWalk2, pnl2, ms2);
      if (w2 == 1) return 1;
      if (w2 == 0) {
        bound = false;
        for (int d = 0; d < 3; ++d) x1[d] = y1[d];
      } else {
        for (int d = 0; d < 3; ++d) m.x[d] = y1[d];
        m.pnl = pnl2;
        m.ms = ms2;
      }
    }
    if (bound) {
      m.id = make_id(sp, 0, id_serno(id));
      push_bound(p, m);
      move_count(p, sp0, sp);
      return 3;
    }
  }
  if (sp != sp0) {
    move_count(p, sp0, sp);
    id = make_id(sp, 0, id_serno(id));
  }
  return 0;
}

// First-order decision when the reaction whose coin succeeded (list slot m)
// is restricted to a compartment (unireact, smolreact.c:3040-3050): it fires
// only if the molecule's new position lies in the compartment; otherwise the
// decision passes to the reactions after it in the species' list, each with
// its own coin.  thr holds the cumulative probabilities of the list as
// fractions of 2^32, so with a fresh uniform u the first of the remaining
// reactions to fire is the first k > m with u < 1 - (1 - cum_k) / (1 - cum_m).
// Returns 2 + reaction, or 0 when none fires.
__device__ __noinline__ int uni_in_cmpt(const uint32_t *thr, int nuni, int sp, int m, float4 pc, const DevGeo &g,
                                        ull skey, uint32_t step) {
  int ix[3];
  unpack_cell(__float_as_uint(pc.w), ix[0], ix[1], ix[2]);
  const float u[3] = {pc.x, pc.y, pc.z};
  double x[3];
  to_abs(g, ix, u, x);
  const uint2 key = make_uint2(c_net.key0 ^ 0x2545F491u, c_net.key1 ^ 0x4F6CDD1Du);
  const double inv32 = 1.0 / 4294967296.0;
  for (int round = 0; round < kMaxUniPerSpecies && m < nuni; ++round) {
    const int rx = c_net.uni_list[sp][m];
    const int c = c_net.cmpt[1][rx];
    if (!c || pos_in_cmpt(c_cmpt, c - 1, c_panels, x)) return 2 + rx;
    const uint4 rr = philox(make_uint4((uint32_t)skey, (uint32_t)(skey >> 32), step, 16u + (uint32_t)round), key);
    const double uu = ((double)rr.x + 0.5) * inv32;
    const double rest_m = 1.0 - (double)thr[m] * inv32;
    int next = nuni;
    for (int k = m + 1; k < nuni; ++k)
      if (rest_m > 0 && uu < 1.0 - (1.0 - (double)thr[k] * inv32) / rest_m) {
        next = k;
        break;
      }
    m = next;
  }
  return 0;
}

// advance_one's result for a molecule that became surface-bound
constexpr int kFateBound = -2;

// Move one molecule by one step (diffuse smolmolec.c:3115, checkwalls
// smolwall.c:368, unireact decision smolreact.c:2997): returns 0 alive,
// 1 removed by a wall, 2+r first-order reaction r fired (position is the
// post-move position).
template <bool SINGLE, int SURF>
__device__ __forceinline__ int advance_one(float4 &pc, ull &id, uint32_t step, const KParams &p,
                                           const float *gtab, int rebin_only, int &hits) {
  int sp = id_species(id);
  const int rep = SINGLE ? 0 : id_rep(id);
  const DevGeo &g = geo_of<SINGLE>(p, rep);
  int ix[3];
  unpack_cell(__float_as_uint(pc.w), ix[0], ix[1], ix[2]);
  float u[3] = {pc.x, pc.y, pc.z};
  if (rebin_only) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      renorm(u[d], ix[d], g.h[d], g.inv_h[d]);
      clamp_cell(u[d], ix[d], g, d);
    }
    pc = make_float4(u[0], u[1], u[2], __uint_as_float(pack_cell(ix[0], ix[1], ix[2])));
    return 0;
  }
  const ull skey = id_stream(id);
  const uint2 key = make_uint2(c_net.key0, c_net.key1);
  const uint4 r = philox_ks(make_uint4((uint32_t)skey, (uint32_t)(skey >> 32), step, 0u), c_net.move_ks);
  float dsp[3];
  int forced = -1;
  if (c_net.inject) {
    const int k = find_injection(p, skey);
    if (k >= 0) {
      const float4 v = p.inj_val[k];
      dsp[0] = v.x; dsp[1] = v.y; dsp[2] = v.z;
      forced = (int)v.w;
    } else {
      dsp[0] = dsp[1] = dsp[2] = 0.f;
    }
  } else {
    const uint32_t gm = c_net.gmask;
    const float g0 = gtab[r.x & gm], g1 = gtab[r.y & gm], g2 = gtab[r.z & gm];
    if ((c_net.difm_any >> sp) & 1u) {  // anisotropic (smolmolec.c:3158-3162)
      const float *M = p.difm + (size_t)(rep * c_net.nsp + sp) * 9;
      dsp[0] = M[0] * g0 + M[1] * g1 + M[2] * g2;
      dsp[1] = M[3] * g0 + M[4] * g1 + M[5] * g2;
      dsp[2] = M[6] * g0 + M[7] * g1 + M[8] * g2;
    } else {
      const float ds = p.difstep[rep * c_net.nsp + sp];
      dsp[0] = fmul(ds, g0);
      dsp[1] = fmul(ds, g1);
      dsp[2] = fmul(ds, g2);
    }
    if (c_net.any_drift) {
      const float *dr = p.driftdt + (size_t)(rep * c_net.nsp + sp) * 3;
      dsp[0] = fadd(dsp[0], dr[0]);
      dsp[1] = fadd(dsp[1], dr[1]);
      dsp[2] = fadd(dsp[2], dr[2]);
    }
  }
  // a molecule that desorbed this step was placed already: only binned here
  const bool moved = SURF == 3 && (__float_as_uint(pc.w) & kMovedBit);
  if (!moved) {
    const int ix0[3] = {ix[0], ix[1], ix[2]};
    const float u0[3] = {u[0], u[1], u[2]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (d >= g.dim) continue;
      float w = fadd(u[d], dsp[d]);
      int j = ix[d];
      renorm(w, j, g.h[d], g.inv_h[d]);
      if (j <= 0 || j >= g.n[d] - 1) {
        if (walls_dim(w, j, g, d, hits)) return 1;
        clamp_cell(w, j, g, d);
      }
      u[d] = w;
      ix[d] = j;
    }
    if (SURF) {
      float a0[3], a1[3];
      for (int d = 0; d < 3; ++d) {
        a0[d] = (float)ix0[d] * g.h[d] + u0[d];
        a1[d] = (float)ix[d] * g.h[d] + u[d];
      }
      if (surface_near<(SURF >= 2)>(a0, a1, p.boxmask, g.cell0 + (ix0[2] * g.n[1] + ix0[1]) * g.n[0] + ix0[0])) {
        double x0[3], x1[3];
        to_abs(g, ix0, u0, x0);
        to_abs(g, ix, u, x1);
        if (SURF == 3) {
          const int r = soln_surface_bound(p, id, x0, x1, hits, step);
          if (r == 1) return 1;
          if (r == 3) return kFateBound;
          sp = id_species(id);
        } else if (surface_interact<(SURF >= 2)>(sp, x0, x1, c_net.surf_eps, hits)) {
          return 1;
        }
        from_abs(g, x1, ix, u);
      }
    }
    if (c_net.any_absorb && !c_net.inject) {
      // Absorbing walls also remove molecules that stayed inside with probability
      // exp(-2*dold*dnew/step^2) (smolwall.c:417-420); the reference applies that
      // test in both wall passes of a step (smolsim.cpp:2625 and :2662), so the
      // survival probability is (1-p)^2.
      const float ds = p.difstep[rep * c_net.nsp + sp];
      const float inv2 = (ds > 0.f) ? __frcp_rn(fmul(ds, ds)) : 0.f;
      uint4 r2 = make_uint4(0, 0, 0, 0);
      int have = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (d >= g.dim) continue;
#pragma unroll
        for (int side = 0; side < 2; ++side) {
          if (g.wall[2 * d + side] != kWallAbsorb || ds <= 0.f) continue;
          float dn, dold;
          if (side == 0) { dn = dist_low(ix[d], u[d], g.h[d]); dold = dist_low(ix0[d], u0[d], g.h[d]); }
          else { dn = dist_high(ix[d], u[d], g, d); dold = dist_high(ix0[d], u0[d], g, d); }
          const float x = fmul(fmul(2.f, fmul(dn, dold)), inv2);
          if (x > 80.f) continue;
          const float pr = __expf(-x);
          const float pe = fmul(pr, fsub(2.f, pr));  // 1-(1-p)^2
          if (!have) { r2 = philox(make_uint4((uint32_t)skey, (uint32_t)(skey >> 32), step, 1u), key); have = 1; }
          const uint32_t bits = (d == 0) ? (side ? r2.y : r2.x) : (d == 1) ? (side ? r2.w : r2.z)
                                          : (side ? (r2.x ^ r2.w) : (r2.y ^ r2.z));
          if (u01f_open(bits) < pe) { hits++; return 1; }
        }
      }
    }
  }
  pc = make_float4(u[0], u[1], u[2], __uint_as_float(pack_cell(ix[0], ix[1], ix[2])));
  // the uniform bit mask first: the per-species table is read only by lanes
  // whose species has first-order reactions
  const int nuni = ((c_net.uni_any >> sp) & 1u) ? c_net.uni_n[sp] : 0;
  if (nuni) {
    if (c_net.inject) {
      if (forced >= 0) return 2 + forced;
    } else {
      const uint32_t *thr = p.unithr + (size_t)(rep * c_net.nsp + sp) * kMaxUniPerSpecies;
      for (int m = 0; m < nuni; ++m)
        if (r.w < thr[m]) {
          const int rx = c_net.uni_list[sp][m];
          if (SURF >= 2 && c_net.cmpt[1][rx]) return uni_in_cmpt(thr, nuni, sp, m, pc, g, skey, step);
          return 2 + rx;
        }
    }
  }
  return 0;
}

__device__ __forceinline__ int global_cell(const DevGeo &g, uint32_t w) {
  int ix, iy, iz;
  unpack_cell(w, ix, iy, iz);
  return g.cell0 + (iz * g.n[1] + iy) * g.n[0] + ix;
}

__device__ __forceinline__ void push_event(const KParams &p, const Event &e) {
  const int k = atomicAdd(p.nev, 1);
  if (k < p.evcap) p.ev[k] = e;
  else atomicOr(p.status, kStEvCap);
}

// ---------------------------------------------------------------------------
// Start of a step: step counter, per-step counters, and the clamp of the
// previous step's product count (an overflow there is already flagged).
__global__ void k_begin(KParams p, int bump_step) {
  pdl_launch_dependents();
  pdl_wait();
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    if (bump_step) *p.step += 1;
    int *pn = const_cast<int *>(p.p_n);
    if (*pn > p.pcap) *pn = p.pcap;
    *p.nev = 0;
    *p.ncand = 0;
    *p.q_n = 0;
    if (bump_step && p.bd_out_n) *p.bd_out_n = 0;  // a re-binning pass leaves the bound list alone
  }
}

// Stage the Gaussian quantile table in shared memory (16 KB at the default
// 4096 levels); larger tables are read from global memory.
__device__ __forceinline__ const float *stage_gtab(const KParams &p, float *s_gtab) {
  const int gsize = (int)c_net.gmask + 1;
  if (gsize > 8192) return p.gtab;
  for (int k = threadIdx.x; k < gsize; k += blockDim.x) s_gtab[k] = p.gtab[k];
  __syncthreads();
  return s_gtab;
}

// Runs of consecutive lanes that hold live molecules of the same box.  The
// lanes process box-sorted molecules, so most of a warp falls into a few runs
// and one slot atomic per run serves the whole run (k_scatter).
struct BoxRun {
  int head;   // first lane of this lane's run
  int count;  // live lanes in the run
  int rank;   // live lanes of the run before this lane
};

__device__ __forceinline__ BoxRun box_run(bool alive, int cell) {
  const int lane = threadIdx.x & 31;
  const unsigned live = __ballot_sync(0xffffffffu, alive);
  const int c = alive ? cell : -1;
  const int prev = __shfl_up_sync(0xffffffffu, c, 1);
  const bool head = alive && (lane == 0 || prev != c);
  const unsigned heads = __ballot_sync(0xffffffffu, head);
  const unsigned le = lanemask_lt() | (1u << lane);
  BoxRun r;
  r.head = max(0, 31 - __clz(heads & le));  // only meaningful for live lanes
  const unsigned after = heads & ~le;
  const int next = after ? __ffs(after) - 1 : 32;
  const unsigned run_mask = (next == 32 ? 0xffffffffu : ((1u << next) - 1u)) & ~((1u << r.head) - 1u);
  r.count = __popc(live & run_mask);
  r.rank = __popc(live & run_mask & lanemask_lt());
  return r;
}

// Increment of the box histogram for every lane with `alive` set.  One
// fire-and-forget atomic per molecule: measured faster here than aggregating
// runs of same-box lanes first (the L2 atomic units absorb the repeats).
template <bool SINGLE>
__device__ __forceinline__ void count_box(const KParams &p, bool alive, float4 pc, ull id) {
  int cell = -1;
  if (alive) {
    const DevGeo &g = geo_of<SINGLE>(p, SINGLE ? 0 : id_rep(id));
    cell = global_cell(g, __float_as_uint(pc.w));
  }
  if (alive) atomicAdd(&p.cnt[cell], 1);
}

__device__ void births(const KParams &p, uint32_t step);

// Move pass (one per step): diffuse + walls + first-order decisions for every
// molecule of the sorted input and of the product list, events for removed or
// reacting molecules, the moved position into tmp (w = kTmpGone when the
// molecule leaves the system), and the histogram of destination boxes.
// rebin_only: no motion and no reactions (used after uploads).
// resident 256-thread blocks per SM the register allocation must allow for
// the surface variant (the plain variant fits 64 registers at 4 blocks)
#ifndef SMOLB_SURF_MOVE_BLOCKS
#define SMOLB_SURF_MOVE_BLOCKS 4
#endif
#ifndef SMOLB_MOVE_BLOCKS
#define SMOLB_MOVE_BLOCKS 4
#endif
template <bool SINGLE, int SURF>
__global__ void __launch_bounds__(256, SURF ? SMOLB_SURF_MOVE_BLOCKS : SMOLB_MOVE_BLOCKS) k_move(KParams p, int rebin_only) {
  extern __shared__ float s_gtab[];
  pdl_launch_dependents();
  const float *gtab = rebin_only ? p.gtab : stage_gtab(p, s_gtab);  // constant data: before the wait
  pdl_wait();
  const int na = *p.a_n, np = *p.p_n;
  const int total = na + np;
  const uint32_t step = *p.step;
  int hits_acc = 0;
  // The next molecule's position and id are loaded before this one is moved,
  // so the load of one grid stride overlaps the arithmetic of the previous
  // (measured 8% faster than loading at the top of each iteration).
  const int stride = gridDim.x * blockDim.x;
  float4 npc = make_float4(0.f, 0.f, 0.f, 0.f);
  ull nid = 0;
  {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < total) {
      if (i < na) { npc = __ldg(&p.a_pc[i]); nid = __ldg(&p.a_id[i]); }
      else { npc = __ldg(&p.p_pc[i - na]); nid = __ldg(&p.p_id[i - na]); }
    }
  }
  for (int base = blockIdx.x * blockDim.x; base < total; base += stride) {
    const int i = base + threadIdx.x;
    float4 pc = npc;
    ull id = nid;
    const bool valid = (i < total) && id_species(id) != kDeadSpecies;
    {
      const int j = i + stride;
      if (j < total) {
        if (j < na) { npc = __ldg(&p.a_pc[j]); nid = __ldg(&p.a_id[j]); }
        else { npc = __ldg(&p.p_pc[j - na]); nid = __ldg(&p.p_id[j - na]); }
      }
    }
    int fate = -1;
    int hits = 0;
    const ull id_in = id;
    if (valid) fate = advance_one<SINGLE, SURF>(pc, id, step, p, gtab, rebin_only, hits);
    if (SURF == 3 && id != id_in && fate != kFateBound) {  // species changed at a surface
      if (i < na) p.a_id[i] = id;
      else const_cast<ull *>(p.p_id)[i - na] = id;
    }
    const bool alive = (fate == 0);
    if (i < total) p.tmp[i] = alive ? pc : make_float4(0.f, 0.f, 0.f, __uint_as_float(kTmpGone));
    count_box<SINGLE>(p, alive, pc, id);
    if (valid && !alive && fate != kFateBound) {
      if (fate == 1) {
        atomicAdd((unsigned long long *)&p.spcount[id_rep(id) * c_net.nsp + id_species(id)],
                  (unsigned long long)(-1ll));
      } else {
        Event e;
        e.site = pc;
        e.key = id_stream(id);
        e.rxn = (1u << 8) | (uint32_t)(fate - 2);
        e.rep = (uint32_t)id_rep(id);
        e.ia = e.ib = -1;
        push_event(p, e);
      }
    }
    hits_acc += hits;
  }
  if (hits_acc) atomicAdd(&p.counters[0], (unsigned long long)hits_acc);
  if (!rebin_only) births(p, step);
}

// Step of the surface-bound molecules, launched before the move pass: a
// mobile bound state diffuses with the move's Gaussian table and is brought
// back onto the surface (movemol2closepanel), its path is checked against
// the other panels, then the per-step desorption / flip coin is drawn
// (diffuse smolmolec.c:3164-3168, checksurfaces, checksurfacebound).
// Molecules still bound go to the output bound list; desorbed ones, after
// their placement walk, to the product list with kMovedBit set.
__global__ void __launch_bounds__(256) k_bound(KParams p) {
  pdl_launch_dependents();
  pdl_wait();
  const int n = *p.bd_in_n;
  const uint32_t step = *p.step;
  int hits_acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    BoundMol m = p.bd_in[i];
    const int sp0 = id_species(m.id);
    if (sp0 == kDeadSpecies) continue;  // reacted with a solution molecule
    int sp = sp0;
    const ull skey = id_stream(m.id);
    const double posx[3] = {m.x[0], m.x[1], m.x[2]};
    const int pnlx = m.pnl;
    int hits = 0;
    bool dead = false, bound = true;
    const double ds = c_net.bstep[sp][m.ms - 1];
    if (ds > 0) {
      const uint4 r = srf_draw(skey, step, kCtrSrfDiff);
      const uint32_t gm = c_net.gmask;
      const int dim = c_geo0.dim;  // in 2-D the panels are lines and circles in the plane
      m.x[0] += ds * (double)p.gtab[r.x & gm];
      if (dim > 1) m.x[1] += ds * (double)p.gtab[r.y & gm];
      if (dim > 2) m.x[2] += ds * (double)p.gtab[r.z & gm];
      move_to_close_panel(m.x, posx, m.pnl, m.ms, skey, step);
      dead = walk_bound(p, m, sp, posx, pnlx, hits, skey, step) == 1;
    }
    if (!dead) {
      double x0[3], x1[3];
      const int c = bound_coin(p, m, sp, skey, step, x0, x1);
      if (c == 0) {  // still bound: its first-order reactions
        const int r = bound_first_order(p, m, sp, skey, step);
        if (r == 1) dead = true;
        else if (r == 3) bound = false;
      }
      if (c == 1) {
        dead = true;
      } else if (c == 2) {
        int pnl2 = 0, ms2 = 0;
        const int w = walk_soln_rules(p, sp, x0, x1, hits, skey, step, kCtrSrfWalk2, pnl2, ms2);
        if (w == 1) {
          dead = true;
        } else if (w == 2) {
          for (int d = 0; d < 3; ++d) m.x[d] = x1[d];
          m.pnl = pnl2;
          m.ms = ms2;
        } else {  // into the product list, already moved
          bound = false;
          int ix[3];
          float u[3];
          from_abs(c_geo0, x1, ix, u);
          const float4 pc = make_float4(u[0], u[1], u[2], __uint_as_float(pack_cell(ix[0], ix[1], ix[2]) | kMovedBit));
          int *pn = const_cast<int *>(p.p_n);
          const int k = atomicAdd(pn, 1);
          if (k < p.pcap) {
            const_cast<float4 *>(p.p_pc)[k] = pc;
            const_cast<ull *>(p.p_id)[k] = make_id(sp, 0, id_serno(m.id));
          } else {
            atomicSub(pn, 1);
            atomicOr(p.status, kStProdCap);
            dead = true;
          }
        }
      }
    }
    if (dead) {
      atomicAdd((unsigned long long *)&p.spcount[sp0], (unsigned long long)(-1ll));
    } else {
      move_count(p, sp0, sp);
      if (bound) {
        m.id = make_id(sp, 0, id_serno(m.id));
        push_bound(p, m);
      }
    }
    hits_acc += hits;
  }
  if (hits_acc) atomicAdd(&p.counters[0], (unsigned long long)hits_acc);
}

// Species counts of an uploaded bound list (added to the solution counts).
__global__ void k_bound_species_count(const BoundMol *m, const int *n, long long *spcount) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < *n; i += gridDim.x * blockDim.x)
    if (id_species(m[i].id) != kDeadSpecies) atomicAdd((unsigned long long *)&spcount[id_species(m[i].id)], 1ull);
}

// ---- bound-solution pair reactions -------------------------------------------
// Second-order reactions of a surface-bound and a solution reactant (bireact
// smolreact.c:3201-3300, morebireact :3109-3157), after the solution pairs of
// the step as in the reference's list order.  A pair reacts when the solution
// molecule lies within the binding radius of the bound one, on the front side
// of the bound one's panel (a solution reactant's state is read from the
// side of that panel, :3134-3137), inside the reaction's compartment if it
// has one, on its surface if it is restricted to one, and the reaction's coin
// passes; of a pair's reactions the first in
// list order that passes is taken.  The reference takes pairs in the order of
// its molecule lists, which has nothing to do with geometry; here every pair
// gets a random priority (a hash of both identities and the step) and the
// pairs react as if taken in priority order: each bound molecule claims its
// partner of lowest priority value (an atomic minimum of priority and
// bound-list index on the partner's claim word), the claim holding the
// minimum reacts, and bound molecules whose partner went to another claim
// again, for kBPairRounds rounds in all.
constexpr uint32_t kCtrBPair = 0x500u;  // + list entry: coin of a bound-solution pair
constexpr int kBPairRounds = 4;
constexpr uint32_t kCtrBProd = 0x5A5A5A5Au;  // stream offset of a product's placement

// absolute position of a sorted molecule's entry q, as the
// displacement-nearest image of x0 in periodic dimensions
__device__ __forceinline__ void bpair_partner_xyz(const float4 q, const double x0[3], double xs[3]) {
  const DevGeo &g = c_geo0;
  int jx[3];
  unpack_cell(__float_as_uint(q.w), jx[0], jx[1], jx[2]);
  const float u[3] = {q.x, q.y, q.z};
  to_abs(g, jx, u, xs);
  for (int d = 0; d < g.dim; ++d)
    if (g.wall[2 * d] == kWallPeriodic) {
      const double L = (double)(g.n[d] - 1) * g.h[d] + g.whi[d];
      const double v = xs[d] - x0[d];
      if (v > 0.5 * L) xs[d] -= L;
      else if (v < -0.5 * L) xs[d] += L;
    }
}

// One warp per bound molecule: lanes 0..26 take the neighbour boxes that the
// largest binding radius of these reactions reaches from the molecule's place
// in its box, a warp prefix sum numbers their molecules, and the lanes test
// them 32 at a time; a warp minimum picks the claim.
__global__ void __launch_bounds__(256, 3) k_bpair_claim(KParams p, int round) {
  pdl_launch_dependents();
  pdl_wait();
  const int nb = min(*p.bd_out_n, p.bcap);
  const int n = *p.b_n;
  const uint32_t step = *p.step;
  const DevGeo &g = c_geo0;
  const uint2 key = make_uint2(c_net.key0 ^ 0x7F4A7C15u, c_net.key1 ^ 0x94D049BBu);
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const float rmax = c_net.bpair_rmax;
  // each warp takes 32 bound molecules at a time, one per lane, and searches
  // for those that need it one after the other: in the first round the live
  // ones with such a reaction, later the ones that lost their partner
  for (int k0 = gw * 32; k0 < nb; k0 += nw * 32) {
    bool need = false;
    if (k0 + lane < nb) {
      const int kl = k0 + lane;
      if (round == 0) {
        const BoundMol &ml = p.bd_out[kl];
        const int spl = id_species(ml.id);
        // a product of this step reacts from the next step on
        need = spl != kDeadSpecies && ml.born != step && c_net.bpair_mask[spl][ml.ms - 1] != 0u;
        if (!need) p.bcand[kl] = make_int4(-1, 0, 0, 0);
      } else {
        const int4 cl = p.bcand[kl];
        need = cl.x >= 0 && cl.w == 0;
      }
    }
    unsigned todo = __ballot_sync(full, need);
    while (todo) {
      const int k = k0 + __ffs(todo) - 1;
      todo &= todo - 1;
      const BoundMol m = p.bd_out[k];
      const int sp = id_species(m.id);
      const uint32_t mask = c_net.bpair_mask[sp][m.ms - 1];
      ull best = ~0ull;  // (priority << 32 | lane) of this lane's best partner
      int bj = -1, be = 0;
      if (mask) {
        const DevPanel &pn = c_panels[m.pnl];
        const ull kb = id_stream(m.id);
        int ix[3];
        float u[3];
        from_abs(g, m.x, ix, u);
        int s0 = 0, cnt = 0;
        if (lane < 27) {
          const int off[3] = {lane % 3 - 1, (lane / 3) % 3 - 1, lane / 9 - 1};
          int cc[3];
          bool ok = true;
          for (int d = 0; d < 3; ++d) {
            if (d >= g.dim && off[d] != 0) ok = false;
            const float ub = (ix[d] == g.n[d] - 1) ? g.whi[d] : g.h[d];
            if (off[d] < 0 && !(u[d] < rmax)) ok = false;
            if (off[d] > 0 && !(u[d] > ub - rmax)) ok = false;
            cc[d] = ix[d] + off[d];
            if (cc[d] < 0 || cc[d] >= g.n[d]) {
              if (g.wall[2 * d] != kWallPeriodic || g.n[d] < 3) ok = false;
              cc[d] = cc[d] < 0 ? cc[d] + g.n[d] : cc[d] - g.n[d];
            }
          }
          if (ok) {
            const int cell = g.cell0 + (cc[2] * g.n[1] + cc[1]) * g.n[0] + cc[0];
            s0 = p.start[cell];
            cnt = max(0, min(p.start[cell + 1], n) - s0);
          }
        }
        int incl = cnt;
  #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(full, incl, o);
          if (lane >= o) incl += y;
        }
        const int excl = incl - cnt;
        const int total = __shfl_sync(full, incl, 31);
        for (int t0 = 0; t0 < total; t0 += 32) {
          const int t = t0 + lane;
          int o = 0;  // the last lane whose first number is <= t
  #pragma unroll
          for (int st = 16; st > 0; st >>= 1)
            if (__shfl_sync(full, excl, o + st) <= t) o += st;
          const int j = __shfl_sync(full, s0, o) + (t - __shfl_sync(full, excl, o));
          if (t >= total) continue;
          const ull idj = p.b_id[j];
          const float4 qj = p.b_pc[j];  // loaded with the identity, not after it
          const int sj = id_species(idj);
          if (sj == kDeadSpecies || !((mask >> sj) & 1u)) continue;
          double xs[3];
          bpair_partner_xyz(qj, m.x, xs);
          const double d2 = (xs[0] - m.x[0]) * (xs[0] - m.x[0]) + (xs[1] - m.x[1]) * (xs[1] - m.x[1]) +
                            (xs[2] - m.x[2]) * (xs[2] - m.x[2]);
          const ull pk = mix64((kb * 0x9E3779B97F4A7C15ull ^ id_stream(idj)) + (ull)step * 0xD1B54A32D192ED03ull);
          const uint32_t prio = (uint32_t)(pk >> 32);
          const ull pkey = ((ull)prio << 32) | (uint32_t)lane;
          if (pkey >= best) continue;
          int side = -1;  // the panel side, read once a reaction is in range
          for (int e = 0; e < c_net.bpair_n; ++e) {
            if (c_net.bpair_bsp[e] != sp || c_net.bpair_bst[e] != m.ms || c_net.bpair_ssp[e] != sj) continue;
            const int r = c_net.bpair_rxn[e];
            if (d2 > (double)p.bind2[r]) continue;
            const float prob = p.pairprob[r];
            if (prob < 1.f) {
              const ull kk = mix64(kb * 0x9E3779B97F4A7C15ull ^ id_stream(idj));
              const uint4 rr = philox(make_uint4((uint32_t)kk, (uint32_t)(kk >> 32), step, kCtrBPair + (uint32_t)e), key);
              if (!(u01co(rr.x) < (double)prob)) continue;
            }
            if (side < 0) side = panel_side(pn, xs, nullptr) == kFaceBack ? 0 : 1;
            if (!side) break;  // behind the panel: the solution state is bsoln, which no reaction takes
            const int cm = c_net.cmpt[2][r];
            if (cm && !(pos_in_cmpt(c_cmpt, cm - 1, c_panels, xs) && pos_in_cmpt(c_cmpt, cm - 1, c_panels, m.x)))
              continue;
            const int rs = c_net.rsrf[2][r];
            if (rs && pn.srf != rs - 1) continue;  // restricted to another surface (morebireact :3116)
            best = pkey;
            bj = j;
            be = e;
            break;
          }
        }
      }
      // warp minimum: the lowest priority (ties to the lower lane)
      ull wmin = best;
  #pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const ull y = __shfl_xor_sync(full, wmin, o);
        wmin = y < wmin ? y : wmin;
      }
      if (wmin != ~0ull && best == wmin) {  // the winning lane
        p.bcand[k] = make_int4(bj, be, (int)(uint32_t)(wmin >> 32), 0);
        atomicMin(&p.bclaim[bj], (wmin & 0xFFFFFFFF00000000ull) | (ull)(uint32_t)k);
      } else if (wmin == ~0ull && lane == 0) {
        p.bcand[k] = make_int4(-1, 0, 0, 0);
      }
    }
  }
}

// The claims holding their partner's minimum react (doreact smolreact.c:2662-
// 2902 for one product): both reactants are removed and the product is placed
// at the diffusion-weighted reaction position, on the bound reactant's panel
// when the position projects inside it, else on the nearest panel of its
// surface; a bound product is brought onto that panel on its state's side
// (fixpt2panel, movemol2closepanel) and takes the bound reactant's entry, a
// solution product is put just off the front (soln) or back (bsoln) side into
// the output product list, so that both first move in the next step.
__global__ void __launch_bounds__(256) k_bpair_resolve(KParams p) {
  pdl_launch_dependents();
  pdl_wait();
  const int nb = min(*p.bd_out_n, p.bcap);
  const uint32_t step = *p.step;
  int done = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
    const int4 c = p.bcand[k];
    if (c.x < 0 || c.w != 0) continue;
    const int j = c.x;
    if (p.bclaim[j] != (((ull)(uint32_t)c.z << 32) | (ull)(uint32_t)k)) continue;  // another claim comes first
    p.bclaim[j] = ~0ull;  // the winner clears the word; losers compare against their own key only
    p.bcand[k].w = 1;
    done++;
    BoundMol m = p.bd_out[k];
    const int spb = id_species(m.id);
    const ull ids = p.b_id[j];
    const int sps = id_species(ids);
    p.b_id[j] = id_mark_dead(ids);
    atomicAdd((unsigned long long *)&p.spcount[sps], (unsigned long long)(-1ll));
    atomicAdd((unsigned long long *)&p.spcount[spb], (unsigned long long)(-1ll));
    const int e = c.y, r = c_net.bpair_rxn[e];
    if (c_net.nprod[2][r] == 0) {
      p.bd_out[k].id = id_mark_dead(m.id);
      continue;
    }
    const int psp = c_net.prd[2][r][0], pst = c_net.bpair_pst[e];
    double xs[3];
    bpair_partner_xyz(p.b_pc[j], m.x, xs);
    const double sb = c_net.bstep[spb][m.ms - 1], ss = c_net.sstep[sps];
    const double db = sb * sb, ds = ss * ss;  // proportional to the diffusion coefficients
    const double f = (db == 0 && ds == 0) ? 0.5 : ds / (db + ds);  // weight of the bound reactant
    double x[3];
    for (int d = 0; d < 3; ++d) x[d] = f * m.x[d] + (1.0 - f) * xs[d];
    int pnl = m.pnl;
    if (!pt_in_panel(c_panels[pnl], x)) {  // closestsurfacept over the bound reactant's surface
      const int srf = c_panels[m.pnl].srf;
      double bestd = 1e300;
      for (int q = 0; q < c_net.npanel; ++q) {
        if (c_panels[q].srf != srf) continue;
        double pt[3];
        closest_panel_pt(c_panels[q], x, pt, 0.0);
        const double dd = (pt[0] - x[0]) * (pt[0] - x[0]) + (pt[1] - x[1]) * (pt[1] - x[1]) + (pt[2] - x[2]) * (pt[2] - x[2]);
        if (dd < bestd) { bestd = dd; pnl = q; }
      }
    }
    const ull skey = mix64(id_stream(m.id) ^ kCtrBProd) & ((1ull << kSpShift) - 1);
    atomicAdd((unsigned long long *)&p.spcount[psp], 1ull);
    if (pst == kMSfront || pst == kMSback) {
      fix_to_panel(c_panels[pnl], x, ms_face(pst), c_net.beps);
      const double x0[3] = {x[0], x[1], x[2]};
      move_to_close_panel(x, x0, pnl, pst, skey, step);
      for (int d = 0; d < 3; ++d) m.x[d] = x[d];
      m.pnl = pnl;
      m.ms = pst;
      m.id = make_id(psp, 0, id_serno(m.id));
      m.born = step;
      p.bd_out[k] = m;
      continue;
    }
    p.bd_out[k].id = id_mark_dead(m.id);
    const int face = pst == kMSbsoln ? kFaceBack : kFaceFront;
    fix_to_panel(c_panels[pnl], x, face, c_net.beps);
    const double x0[3] = {x[0], x[1], x[2]};
    move_to_close_panel(x, x0, pnl, face == kFaceBack ? kMSback : kMSfront, skey, step);
    const DevPanel &pn = c_panels[pnl];
    double nrm[3];
    face_normal(pn, x, face, nrm);
    const double sd = fabs(panel_sdist<true>(pn, x));
    if (sd < c_net.surf_eps)  // kept surf_eps off the panel, as solution molecules are
      for (int d = 0; d < 3; ++d) x[d] += (c_net.surf_eps - sd) * nrm[d];
    int ix[3];
    float w[3];
    from_abs(c_geo0, x, ix, w);
    const int slot = atomicAdd(p.q_n, 1);
    if (slot < p.pcap) {
      p.q_pc[slot] = make_float4(w[0], w[1], w[2], __uint_as_float(pack_cell(ix[0], ix[1], ix[2])));
      p.q_id[slot] = make_id(psp, 0, id_serno(m.id));
    } else {
      atomicOr(p.status, kStProdCap);
    }
  }
  if (done) atomicAdd(&p.counters[3], (unsigned long long)done);
}

// ---- bound-bound pair reactions ----------------------------------------------
// Second-order reactions of two surface-bound reactants (bireact with both
// molecules in a bound state, morebireact smolreact.c:3109-3157: molecules on
// different panels do not react, the product takes the diffusion-weighted
// place on their panel, doreact :2690-2706).  The bound molecules with such a
// reaction go into a hash grid of their boxes (a bucket head per hashed box,
// linked through the molecules); each round every molecule finds, in the
// boxes its largest binding radius reaches, its partner of lowest random
// priority (a symmetric hash of both identities and the step) among those on
// its panel within the binding radius whose coin passes; mutual choices react
// (the lower index carries the reaction out), and the others look again, for
// kBPairRounds rounds.  A kernel at the end empties the buckets it used.
constexpr int kBBHashBits = 20;
constexpr ull kBBReacted = ~0ull - 1;  // bbbest of a molecule that reacted this step

__device__ __forceinline__ int bb_bucket(ull cell) { return (int)(mix64(cell) >> (64 - kBBHashBits)); }
constexpr ull kBBNone = ~0ull;  // bbcell of a molecule not in the grid

// Cell of the bound-bound grid: cubes of the largest binding radius of these
// reactions (bound molecules crowd on surfaces, so the solution boxes would
// hold far too many of them), coordinates offset to stay positive and packed
// 21 bits each.
__device__ __forceinline__ void bb_cell_coords(const double x[3], int c[3]) {
  const double inv = c_net.bb_inv_cs;
  for (int d = 0; d < 3; ++d) c[d] = (int)floor(x[d] * inv) + (1 << 20);
}
__device__ __forceinline__ ull bb_cell_key(const int c[3]) {
  return ((ull)(c[0] & 0x1FFFFF)) | ((ull)(c[1] & 0x1FFFFF) << 21) | ((ull)(c[2] & 0x1FFFFF) << 42);
}

__device__ __forceinline__ bool bb_candidate(const KParams &p, int k, uint32_t step) {
  const BoundMol &m = p.bd_out[k];
  const int sp = id_species(m.id);
  if (sp == kDeadSpecies || !c_net.bb_mask[sp][m.ms - 1]) return false;
  if (m.born == step) return false;  // a product of this step reacts from the next step on
  // an entry that reacted with a solution molecule this step holds a product
  if (c_net.bpair_n && p.bcand[k].x >= 0 && p.bcand[k].w == 1) return false;
  return true;
}

__global__ void __launch_bounds__(256) k_bb_insert(KParams p) {
  pdl_launch_dependents();
  pdl_wait();
  const int nb = min(*p.bd_out_n, p.bcap);
  const uint32_t step = *p.step;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
    p.bbbest[k] = ~0ull;
    if (!bb_candidate(p, k, step)) {
      p.bbcell[k] = kBBNone;
      continue;
    }
    int c[3];
    bb_cell_coords(p.bd_out[k].x, c);
    const ull cell = bb_cell_key(c);
    p.bbcell[k] = cell;
    p.bbnext[k] = atomicExch(&p.bbhead[bb_bucket(cell)], k);
  }
}

__global__ void __launch_bounds__(256) k_bb_best(KParams p) {
  pdl_launch_dependents();
  pdl_wait();
  const int nb = min(*p.bd_out_n, p.bcap);
  const uint32_t step = *p.step;
  const DevGeo &g = c_geo0;
  const uint2 key = make_uint2(c_net.key0 ^ 0x2F8A6B1Du, c_net.key1 ^ 0x5C4E9A37u);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
    if (p.bbcell[k] == kBBNone || p.bbbest[k] == kBBReacted) continue;
    const BoundMol m = p.bd_out[k];
    const int sp = id_species(m.id);
    const uint32_t mask = c_net.bb_mask[sp][m.ms - 1];
    const ull kk = id_stream(m.id);
    int ix[3];
    bb_cell_coords(m.x, ix);
    ull best = ~0ull;
    for (int q = 0; q < 27; ++q) {  // cells are one binding radius wide: the 27 around cover every partner
      const int off[3] = {q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1};
      if ((g.dim < 3 && off[2] != 0) || (g.dim < 2 && off[1] != 0)) continue;
      const int cc[3] = {ix[0] + off[0], ix[1] + off[1], ix[2] + off[2]};
      const ull cell = bb_cell_key(cc);
      for (int j = p.bbhead[bb_bucket(cell)]; j >= 0; j = p.bbnext[j]) {
        if (j == k || p.bbcell[j] != cell || p.bbbest[j] == kBBReacted) continue;
        const BoundMol mj = p.bd_out[j];
        const int sj = id_species(mj.id);
        if (mj.pnl != m.pnl || !((mask >> sj) & 1u)) continue;
        const double d2 = (mj.x[0] - m.x[0]) * (mj.x[0] - m.x[0]) + (mj.x[1] - m.x[1]) * (mj.x[1] - m.x[1]) +
                          (mj.x[2] - m.x[2]) * (mj.x[2] - m.x[2]);
        const ull kj = id_stream(mj.id);
        const ull lo = kk < kj ? kk : kj, hi = kk < kj ? kj : kk;  // symmetric in the pair
        const ull pk = mix64((lo * 0x9E3779B97F4A7C15ull ^ hi) + (ull)step * 0xD1B54A32D192ED03ull);
        const ull key2 = (pk & 0xFFFFFFFF00000000ull) | (uint32_t)j;
        if (key2 >= best) continue;
        for (int e = 0; e < c_net.bb_n; ++e) {
          const bool fw = c_net.bb_sp[e][0] == sp && c_net.bb_st[e][0] == m.ms && c_net.bb_sp[e][1] == sj &&
                          c_net.bb_st[e][1] == mj.ms;
          const bool bw = c_net.bb_sp[e][1] == sp && c_net.bb_st[e][1] == m.ms && c_net.bb_sp[e][0] == sj &&
                          c_net.bb_st[e][0] == mj.ms;
          if (!fw && !bw) continue;
          const int r = c_net.bb_rxn[e];
          if (d2 > (double)p.bind2[r]) continue;
          const float prob = p.pairprob[r];
          if (prob < 1.f) {
            const ull h = mix64(lo * 0x9E3779B97F4A7C15ull ^ hi);
            const uint4 rr = philox(make_uint4((uint32_t)h, (uint32_t)(h >> 32), step, (uint32_t)e), key);
            if (!(u01co(rr.x) < (double)prob)) continue;
          }
          const int cm = c_net.cmpt[2][r], rs = c_net.rsrf[2][r];
          if (cm && !(pos_in_cmpt(c_cmpt, cm - 1, c_panels, m.x) && pos_in_cmpt(c_cmpt, cm - 1, c_panels, mj.x)))
            continue;
          if (rs && c_panels[m.pnl].srf != rs - 1) continue;
          best = key2;
          break;
        }
      }
    }
    p.bbbest[k] = best;
  }
}

// The reaction of one mutual pair (k the lower index): its first reaction in
// list order that passed, found again from the pair's species and states.
__global__ void __launch_bounds__(256) k_bb_resolve(KParams p) {
  pdl_launch_dependents();
  pdl_wait();
  const int nb = min(*p.bd_out_n, p.bcap);
  const uint32_t step = *p.step;
  int done = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
    if (p.bbcell[k] == kBBNone) continue;
    const ull bk = p.bbbest[k];
    if (bk == ~0ull || bk == kBBReacted) continue;
    const int j = (int)(uint32_t)bk;
    if (j <= k) continue;
    const ull bj = p.bbbest[j];
    if (bj == kBBReacted || (int)(uint32_t)bj != k) continue;
    // mutual: k reacts with j
    BoundMol m = p.bd_out[k];
    const BoundMol mj = p.bd_out[j];
    const int sp = id_species(m.id), sj = id_species(mj.id);
    const double d2 = (mj.x[0] - m.x[0]) * (mj.x[0] - m.x[0]) + (mj.x[1] - m.x[1]) * (mj.x[1] - m.x[1]) +
                      (mj.x[2] - m.x[2]) * (mj.x[2] - m.x[2]);
    const ull kk = id_stream(m.id), kj = id_stream(mj.id);
    const ull lo = kk < kj ? kk : kj, hi = kk < kj ? kj : kk;
    const uint2 key = make_uint2(c_net.key0 ^ 0x2F8A6B1Du, c_net.key1 ^ 0x5C4E9A37u);
    int e = 0;
    for (; e < c_net.bb_n; ++e) {  // the same tests as the search, in the same order
      const bool fw = c_net.bb_sp[e][0] == sp && c_net.bb_st[e][0] == m.ms && c_net.bb_sp[e][1] == sj &&
                      c_net.bb_st[e][1] == mj.ms;
      const bool bw = c_net.bb_sp[e][1] == sp && c_net.bb_st[e][1] == m.ms && c_net.bb_sp[e][0] == sj &&
                      c_net.bb_st[e][0] == mj.ms;
      if (!fw && !bw) continue;
      const int r = c_net.bb_rxn[e];
      if (d2 > (double)p.bind2[r]) continue;
      const float prob = p.pairprob[r];
      if (prob < 1.f) {
        const ull h = mix64(lo * 0x9E3779B97F4A7C15ull ^ hi);
        const uint4 rr = philox(make_uint4((uint32_t)h, (uint32_t)(h >> 32), step, (uint32_t)e), key);
        if (!(u01co(rr.x) < (double)prob)) continue;
      }
      const int cm = c_net.cmpt[2][r], rs = c_net.rsrf[2][r];
      if (cm && !(pos_in_cmpt(c_cmpt, cm - 1, c_panels, m.x) && pos_in_cmpt(c_cmpt, cm - 1, c_panels, mj.x)))
        continue;
      if (rs && c_panels[m.pnl].srf != rs - 1) continue;
      break;
    }
    if (e >= c_net.bb_n) continue;  // cannot happen: the search found this pair
    p.bbbest[k] = kBBReacted;
    p.bbbest[j] = kBBReacted;
    done++;
    atomicAdd((unsigned long long *)&p.spcount[sp], (unsigned long long)(-1ll));
    atomicAdd((unsigned long long *)&p.spcount[sj], (unsigned long long)(-1ll));
    p.bd_out[j].id = id_mark_dead(mj.id);
    const int r = c_net.bb_rxn[e];
    if (c_net.nprod[2][r] == 0) {
      p.bd_out[k].id = id_mark_dead(m.id);
      continue;
    }
    const int psp = c_net.prd[2][r][0], pst = c_net.bb_pst[e];
    const double sa = c_net.bstep[sp][m.ms - 1], sb = c_net.bstep[sj][mj.ms - 1];
    const double da = sa * sa, db = sb * sb;  // proportional to the diffusion coefficients
    const double f = (da == 0 && db == 0) ? 0.5 : db / (da + db);  // weight of molecule k
    double x[3];
    for (int d = 0; d < 3; ++d) x[d] = f * m.x[d] + (1.0 - f) * mj.x[d];
    int pnl = m.pnl;
    const ull skey = mix64(kk ^ kCtrBProd) & ((1ull << kSpShift) - 1);
    atomicAdd((unsigned long long *)&p.spcount[psp], 1ull);
    if (pst == kMSfront || pst == kMSback) {
      fix_to_panel(c_panels[pnl], x, ms_face(pst), c_net.beps);
      const double x0[3] = {x[0], x[1], x[2]};
      move_to_close_panel(x, x0, pnl, pst, skey, step);
      for (int d = 0; d < 3; ++d) m.x[d] = x[d];
      m.pnl = pnl;
      m.ms = pst;
      m.id = make_id(psp, 0, id_serno(m.id));
      m.born = step;
      p.bd_out[k] = m;
      continue;
    }
    p.bd_out[k].id = id_mark_dead(m.id);
    const int face = pst == kMSbsoln ? kFaceBack : kFaceFront;
    fix_to_panel(c_panels[pnl], x, face, c_net.beps);
    const double x0[3] = {x[0], x[1], x[2]};
    move_to_close_panel(x, x0, pnl, face == kFaceBack ? kMSback : kMSfront, skey, step);
    const DevPanel &pn = c_panels[pnl];
    double nrm[3];
    face_normal(pn, x, face, nrm);
    const double sd = fabs(panel_sdist<true>(pn, x));
    if (sd < c_net.surf_eps)
      for (int d = 0; d < 3; ++d) x[d] += (c_net.surf_eps - sd) * nrm[d];
    int ix[3];
    float w[3];
    from_abs(c_geo0, x, ix, w);
    const int slot = atomicAdd(p.q_n, 1);
    if (slot < p.pcap) {
      p.q_pc[slot] = make_float4(w[0], w[1], w[2], __uint_as_float(pack_cell(ix[0], ix[1], ix[2])));
      p.q_id[slot] = make_id(psp, 0, id_serno(m.id));
    } else {
      atomicOr(p.status, kStProdCap);
    }
  }
  if (done) atomicAdd(&p.counters[3], (unsigned long long)done);
}

// Empty the hash-grid buckets used this step (all ones between steps).
__global__ void __launch_bounds__(256) k_bb_clear(KParams p) {
  pdl_launch_dependents();
  pdl_wait();
  const int nb = min(*p.bd_out_n, p.bcap);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x)
    if (p.bbcell[k] != kBBNone) p.bbhead[bb_bucket(p.bbcell[k])] = -1;
}

// Scatter pass: a pure permutation of the moved molecules into box order.
// Each warp takes its slots from a box's count with one atomic per run of
// same-box lanes.  The pass is latency-bound (load, atomic, box start,
// store), so every thread handles two molecules per iteration with their
// chains interleaved.
struct ScatterItem {
  float4 pc;
  ull id;
  bool alive;
  int cell;
};

template <bool SINGLE>
__device__ __forceinline__ ScatterItem scatter_load(const KParams &p, int i, int na, int total) {
  ScatterItem it;
  it.pc = make_float4(0.f, 0.f, 0.f, __uint_as_float(kTmpGone));
  it.id = 0;
  if (i < total) {
    it.pc = p.tmp[i];
    it.id = (i < na) ? p.a_id[i] : p.p_id[i - na];
  }
  it.alive = __float_as_uint(it.pc.w) != kTmpGone;
  it.cell = -1;
  if (it.alive) {
    const DevGeo &g = geo_of<SINGLE>(p, SINGLE ? 0 : id_rep(it.id));
    it.cell = global_cell(g, __float_as_uint(it.pc.w));
  }
  return it;
}

__device__ __forceinline__ void scatter_store(const KParams &p, const ScatterItem &it, int slot) {
  if (!it.alive) return;
  if (slot >= 0 && slot < p.cap) {
    p.b_pc[slot] = it.pc;
    p.b_id[slot] = it.id;
  } else {
    atomicOr(p.status, kStMolCap);
  }
}

// molecules per thread per iteration of the scatter pass (2 or 4)
#ifndef SMOLB_SCATTER_ITEMS
#define SMOLB_SCATTER_ITEMS 2
#endif
template <bool SINGLE>
__global__ void __launch_bounds__(256) k_scatter(KParams p) {
  constexpr int NI = SMOLB_SCATTER_ITEMS;
  pdl_launch_dependents();
  pdl_wait();
  const int na = *p.a_n, np = *p.p_n;
  const int total = na + np;
  const int lane = threadIdx.x & 31;
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < total; base += NI * stride) {
    ScatterItem it[NI];
    BoxRun run[NI];
    int old[NI], st[NI];
#pragma unroll
    for (int k = 0; k < NI; ++k) it[k] = scatter_load<SINGLE>(p, base + k * stride + threadIdx.x, na, total);
#pragma unroll
    for (int k = 0; k < NI; ++k) run[k] = box_run(it[k].alive, it[k].cell);
    // the run's first live lane takes `count` slots from the top of the box
#pragma unroll
    for (int k = 0; k < NI; ++k) {
      old[k] = 0;
      if (it[k].alive && run[k].rank == 0) old[k] = atomicSub(&p.cnt[it[k].cell], run[k].count);
    }
#pragma unroll
    for (int k = 0; k < NI; ++k) st[k] = it[k].alive ? p.start[it[k].cell] : 0;
#pragma unroll
    for (int k = 0; k < NI; ++k) {
      old[k] = __shfl_sync(0xffffffffu, old[k], it[k].alive ? run[k].head : lane);
      scatter_store(p, it[k], st[k] + old[k] - run[k].count + run[k].rank);
    }
  }
}

// ---- exclusive scan of the box histogram ------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int *s_warp, int &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    int w = (lane < nw) ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) s_warp[lane] = w;
  }
  __syncthreads();
  const int warp_excl = (warp > 0) ? s_warp[warp - 1] : 0;
  total = s_warp[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_excl + x - v;
}

// Single-pass exclusive scan of the box counts (decoupled look-back, Merrill &
// Garland 2016).  Tiles take ids from a 64-bit ticket counter in launch order,
// so a tile only waits for tiles that are already running.  Each tile
// publishes one 64-bit status word: epoch (30 bits) | kind (2 bits: 1 = tile
// total, 2 = inclusive prefix) | value (32 bits).  The epoch is the launch
// number, so words left by earlier launches read as "not yet published" and
// the status array never needs clearing.  Every wait is bounded: after
// kScanSpinLimit polls the tile records kStScanWait and proceeds.
constexpr long long kScanSpinLimit = 1ll << 22;

__device__ __forceinline__ ull scan_word(ull tag, int kind, int v) {
  return tag | ((ull)kind << 32) | (uint32_t)v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_lookback(const int *cnt, int n, int nb, ull *ticket,
                                                                 ull *tile_status, int *start, int *n_out, int cap,
                                                                 int *status) {
  __shared__ int s_warp[32];
  __shared__ ull s_ticket;
  __shared__ int s_prefix;
  pdl_launch_dependents();
  pdl_wait();
  if (threadIdx.x == 0) s_ticket = atomicAdd(ticket, 1ull);
  __syncthreads();
  const ull T = s_ticket;
  const int tile = (int)(T % (ull)nb);
  const ull tag = (((T / (ull)nb) + 1ull) & 0x3FFFFFFFull) << 34;
  const int base = tile * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < n) ? cnt[base + k] : 0;
    sum += v[k];
  }
  int total;
  const int ex = block_exclusive_scan(sum, s_warp, total);
  if (threadIdx.x == 0) {
    if (tile == 0) {
      atomicExch(&tile_status[0], scan_word(tag, 2, total));
      s_prefix = 0;
    } else {
      atomicExch(&tile_status[tile], scan_word(tag, 1, total));
    }
  }
  if (tile > 0 && threadIdx.x < 32) {
    const int lane = threadIdx.x;
    int excl = 0;
    int look = tile - 1;
    while (true) {
      const int idx = look - lane;
      ull w = scan_word(tag, 2, 0);  // before tile 0: an empty prefix
      if (idx >= 0) {
        long long spins = 0;
        w = *(volatile ull *)&tile_status[idx];
        while ((w >> 34) != (tag >> 34)) {
          if (++spins > kScanSpinLimit) {
            atomicOr(status, kStScanWait);
            w = scan_word(tag, 2, 0);
            break;
          }
          w = *(volatile ull *)&tile_status[idx];
        }
      }
      const int kind = (int)((w >> 32) & 3u);
      const int val = (int)(uint32_t)w;
      const unsigned pm = __ballot_sync(0xffffffffu, kind == 2);
      const int stop = pm ? __ffs(pm) - 1 : 31;
      int part = lane <= stop ? val : 0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      excl += part;
      if (pm) break;
      look -= 32;
    }
    if (lane == 0) {
      atomicExch(&tile_status[tile], scan_word(tag, 2, excl + total));
      s_prefix = excl;
    }
  }
  __syncthreads();
  int run = s_prefix + ex;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) start[base + k] = run;
    run += v[k];
  }
  if (tile == nb - 1 && threadIdx.x == 0) {
    const int tot = s_prefix + total;
    start[n] = tot;
    *n_out = tot < cap ? tot : cap;
  }
}

// ---- zeroth-order births ---------------------------------------------------
__device__ int poisson_sample(double mean, uint2 key, uint4 ctr) {
  if (mean <= 0) return 0;
  uint32_t it = 0;
  if (mean < 12.0) {  // product of uniforms (Knuth)
    const double g = exp(-mean);
    int n = 0;
    uint4 r = philox(ctr, key);
    double t = u01d(r.x) + 1.1641532182693481e-10;
    int used = 1;
    while (t > g && n < 100000) {
      if (used == 4) { ctr.w = ++it; r = philox(ctr, key); used = 0; }
      const uint32_t b = (used == 0) ? r.x : (used == 1) ? r.y : (used == 2) ? r.z : r.w;
      used++;
      t *= u01d(b) + 1.1641532182693481e-10;
      n++;
    }
    return n;
  }
  // transformed rejection with squeeze, PTRS (W. Hormann, Insurance: Math. Econ. 12, 1993)
  const double smu = sqrt(mean);
  const double b = 0.931 + 2.53 * smu;
  const double a = -0.059 + 0.02483 * b;
  const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
  const double vr = 0.9277 - 3.6224 / (b - 2.0);
  const double lmu = log(mean);
  for (int guard = 0; guard < 1000; ++guard) {
    ctr.w = ++it;
    const uint4 r = philox(ctr, key);
    const double U = u01d(r.x) - 0.5 + 1.1641532182693481e-10;
    const double V = u01d(r.y) + 1.1641532182693481e-10;
    const double us = 0.5 - fabs(U);
    const double k = floor((2.0 * a / us + b) * U + mean + 0.43);
    if (us >= 0.07 && V <= vr) return (int)k;
    if (k < 0 || (us < 0.013 && V > us)) continue;
    if (log(V) + log(inv_alpha) - log(a / (us * us) + b) <= -mean + k * lmu - lgamma(k + 1.0))
      return (int)k;
  }
  return (int)floor(mean + 0.5);
}

// One block per (replicate, reaction): thread 0 draws the Poisson number of
// births and reserves event slots, then the block writes the events.
// Zeroth-order births (smolreact.c:2905-2995): one Poisson draw per
// (replicate, reaction) by the first thread of a block, then one event per
// birth; products are placed by k_products.  Run by k_move's blocks after
// their molecules (all threads of the block call it).
__device__ void births(const KParams &p, uint32_t step) {
  const int nr0 = c_net.nr[0];
  if (nr0 == 0) return;
  __shared__ int s_base, s_n;
  const uint2 key = make_uint2(c_net.key0 ^ 0x5bd1e995u, c_net.key1);
  const int total = c_net.nrep * nr0;
  for (int t = blockIdx.x; t < total; t += gridDim.x) {
    const int rep = t / nr0, r = t % nr0;
    __syncthreads();
    if (threadIdx.x == 0) {
      const int nb = poisson_sample(p.births[t], key, make_uint4((uint32_t)rep, (uint32_t)r, step, 0u));
      int base = 0;
      if (nb > 0) {
        base = atomicAdd(p.nev, nb);
        atomicAdd(&p.counters[1], (unsigned long long)nb);
        if (base + nb > p.evcap) atomicOr(p.status, kStEvCap);
      }
      s_base = base;
      s_n = nb;
    }
    __syncthreads();
    const int base = s_base, nb = s_n;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
      if (base + k >= p.evcap) break;
      Event e;
      e.site = make_float4(0.f, 0.f, 0.f, 0.f);
      e.key = mix64(((ull)rep << 40) ^ ((ull)r << 32) ^ ((ull)step << 8) ^ 0xB17Aull ^
                    mix64((ull)k + 0x9E37ull * (ull)step)) & ((1ull << kSpShift) - 1);
      e.rxn = (0u << 8) | (uint32_t)r;
      e.rep = (uint32_t)rep;
      e.ia = e.ib = -1;
      p.ev[base + k] = e;
    }
  }
}

// ---- bimolecular neighbour search ------------------------------------------
// Deterministic per-pair coin for reactions with probability < 1.
__device__ __forceinline__ bool pair_coin(ull ka, ull kb, int r, uint32_t step, float prob) {
  if (prob >= 1.f) return true;
  const ull lo = ka < kb ? ka : kb, hi = ka < kb ? kb : ka;
  const uint4 x = philox(make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32)),
                         make_uint2(c_net.key0 ^ step, c_net.key1 ^ (0x7F4A7C15u + (uint32_t)r)));
  return u01d(x.x) < (double)prob;
}

// First reaction (in list order) that fires for this pair, or -1.
// Whether both molecules of a pair (sorted indices ia, ib) lie in compartment
// c: the compartment test of a restricted bimolecular reaction
// (morebireact, smolreact.c:3115).
__device__ __noinline__ bool pair_in_cmpt(const KParams &p, int c, int ia, int ib) {
  for (int k = 0; k < 2; ++k) {
    const int idx = k ? ib : ia;
    const float4 q = p.b_pc[idx];
    const DevGeo &g = p.geo[id_rep(p.b_id[idx])];
    int ix[3];
    unpack_cell(__float_as_uint(q.w), ix[0], ix[1], ix[2]);
    const float u[3] = {q.x, q.y, q.z};
    double x[3];
    to_abs(g, ix, u, x);
    if (!pos_in_cmpt(c_cmpt, c, c_panels, x)) return false;
  }
  return true;
}

// The reaction a pair at squared distance d2 undergoes this step, or -1: the
// first of the pair's reactions whose binding radius, coin and (CMPT)
// compartment test pass (bireact, smolreact.c:3201-3298).
template <bool CMPT>
__device__ __forceinline__ int pair_reaction(const KParams &p, int rep, int spa, int spb, float d2,
                                             ull ka, ull kb, uint32_t step, int ia, int ib) {
  const int nl = c_net.pair_n[spa][spb];
  const int nr2 = c_net.nr[2];
  for (int m = 0; m < nl; ++m) {
    const int r = c_net.pair_list[spa][spb][m];
    if (d2 <= p.bind2[rep * nr2 + r] && pair_coin(ka, kb, r, step, p.pairprob[rep * nr2 + r])) {
      if (CMPT && c_net.cmpt[2][r] && !pair_in_cmpt(p, c_net.cmpt[2][r] - 1, ia, ib)) continue;
      return r;
    }
  }
  return -1;
}

// Closest live partner of molecule i within its pair binding radii.
// Returns packed (dist2 bits << 32 | index) or ~0 when none; *ncand counts candidates.
// The box starts are read from st[c - base] for global box c: the step
// pipeline passes its start array (base 0), the persistent kernel a
// replicate's own table.
template <int SURF>
__device__ ull search_partner_in(const KParams &p, int i, float4 pc, ull id, uint32_t step, int &ncand,
                                 const int *st, int base) {
  const int nsorted = *p.b_n;
  const int sp = id_species(id);
  const int rep = id_rep(id);
  const DevGeo g = p.geo[rep];
  const uint32_t mask = c_net.pair_mask[sp];
  int ix, iy, iz;
  unpack_cell(__float_as_uint(pc.w), ix, iy, iz);
  const bool px = g.wall[0] == kWallPeriodic, py = g.wall[2] == kWallPeriodic, pz = g.wall[4] == kWallPeriodic;
  const ull ka = id_stream(id);
  ull best = ~0ull;
  ncand = 0;
  // Only boxes that the sphere of the largest binding radius of this species
  // can reach are scanned: the own box, plus a neighbour along an axis when
  // the molecule lies within that radius of the shared face.  Boxes are at
  // least one binding radius wide, so this covers every partner the full
  // 27-box neighbourhood would (smolreact.c:3248-3298 scans all 26 neighbours).
  const float rs = p.rsearch[rep * c_net.nsp + sp];
  const float ub0 = (ix == g.n[0] - 1) ? g.whi[0] : g.h[0];
  const float ub1 = (iy == g.n[1] - 1) ? g.whi[1] : g.h[1];
  const float ub2 = (iz == g.n[2] - 1) ? g.whi[2] : g.h[2];
  const int xlo = pc.x < rs ? -1 : 0, xhi = pc.x > ub0 - rs ? 1 : 0;
  const int ylo = pc.y < rs ? -1 : 0, yhi = pc.y > ub1 - rs ? 1 : 0;
  const int zlo = pc.z < rs ? -1 : 0, zhi = pc.z > ub2 - rs ? 1 : 0;
  for (int dz = zlo; dz <= zhi; ++dz) {
    int z = iz + dz;
    if (z < 0 || z >= g.n[2]) {
      if (!pz) continue;
      z = (z < 0) ? z + g.n[2] : z - g.n[2];
    }
    for (int dy = ylo; dy <= yhi; ++dy) {
      int y = iy + dy;
      if (y < 0 || y >= g.n[1]) {
        if (!py) continue;
        y = (y < 0) ? y + g.n[1] : y - g.n[1];
      }
      const int rowbase = g.cell0 + (z * g.n[1] + y) * g.n[0];
      for (int dx = xlo; dx <= xhi; ++dx) {
        int x = ix + dx;
        if (x < 0 || x >= g.n[0]) {
          if (!px) continue;
          x = (x < 0) ? x + g.n[0] : x - g.n[0];
        }
        const int c = rowbase + x - base;
        const int s = st[c], e = min(st[c + 1], nsorted);
        for (int j = s; j < e; ++j) {
          if (j == i) continue;
          const ull jd = p.b_id[j];
          const int spj = id_species(jd);
          if (spj == kDeadSpecies || !((mask >> spj) & 1u)) continue;
          const float4 q = p.b_pc[j];
          // antisymmetric differences keep dist2 identical from both sides
          const float vx = (q.x - pc.x) + (float)dx * g.h[0];
          const float vy = (q.y - pc.y) + (float)dy * g.h[1];
          const float vz = (q.z - pc.z) + (float)dz * g.h[2];
          const float d2 = vx * vx + vy * vy + vz * vz;
          if (pair_reaction<(SURF >= 2)>(p, rep, sp, spj, d2, ka, id_stream(jd), step, i, j) < 0) continue;
          if (SURF && pair_crosses_surface_call<(SURF >= 2)>(g, pc, vx, vy, vz)) continue;
          ncand++;
          const ull k = ((ull)__float_as_uint(d2) << 32) | (uint32_t)j;
          if (k < best) best = k;
        }
      }
    }
  }
  return best;
}

template <int SURF>
__device__ __forceinline__ ull search_partner(const KParams &p, int i, float4 pc, ull id, uint32_t step,
                                              int &ncand) {
  return search_partner_in<SURF>(p, i, pc, id, step, ncand, p.start, 0);
}

// Record candidate key k in best[x]; the first registration of x appends it
// to the candidate list.  Returns 1 if x already had a candidate.
__device__ __forceinline__ int register_candidate(const KParams &p, int x, ull k) {
  const ull old = atomicMin(&p.best[x], k);
  if (old == ~0ull) {
    const int t = atomicAdd(p.ncand, 1);
    if (t < p.candcap) p.cand[t] = x;
    else atomicOr(p.status, kStCandCap);
    return 0;
  }
  return 1;
}

// Pair test shared by the staged and the neighbour-box paths: if i and j react
// this step, fold the key into i's running best and register i on j.
template <int SURF>
__device__ __forceinline__ void try_pair(const KParams &p, int i, ull idi, int sp, int rep, float d2, int j, ull jd,
                                         float rs2, uint32_t step, ull &best, int &extra, float4 pc, float vx,
                                         float vy, float vz) {
  if (d2 > rs2) return;
  const int spj = id_species(jd);
  if (spj == kDeadSpecies || !((c_net.pair_mask[sp] >> spj) & 1u)) return;
  if (SURF && pair_crosses_surface_call<(SURF >= 2)>(p.geo[rep], pc, vx, vy, vz)) return;
  if (pair_reaction<(SURF >= 2)>(p, rep, sp, spj, d2, id_stream(idi), id_stream(jd), step, i, j) < 0) return;
  const uint32_t db = __float_as_uint(d2);
  const ull k = ((ull)db << 32) | (uint32_t)j;
  if (best != ~0ull) extra++;
  if (k < best) best = k;
  extra += register_candidate(p, j, ((ull)db << 32) | (uint32_t)i);
}


// Register an in-radius reacting pair on both molecules.
__device__ __forceinline__ int register_pair(const KParams &p, int i, int j, float d2) {
  const ull db = (ull)__float_as_uint(d2) << 32;
  return register_candidate(p, i, db | (uint32_t)j) + register_candidate(p, j, db | (uint32_t)i);
}

// Round-1 pair search, one warp per 32-molecule tile with no block-level
// synchronisation.  Each warp stages a 65-entry window of box-sorted molecules
// (its 32 plus the next 33) in its own slice of shared memory, loading the
// next window into registers while it processes the current one.  Pairs inside
// a box are tested by the lower-indexed molecule (boxes are contiguous runs of
// the sorted array, so partners sit at i+1, i+2, ...).  The warp's same-box
// pairs are enumerated flat: each lane counts its forward partners inside the
// window from two ballots of box boundaries, a warp prefix sum numbers the
// pairs, and the lanes take pair numbers 32 at a time (owner found by a
// 5-step search over the prefix), so the trip count is (pairs in the warp)/32
// instead of the longest box run.  A molecule within the stencil radius of a
// box face sets its bit in the face bitmask (one 32-bit word per tile, written
// without atomics); k_pairs_faces tests its cross-box pairs from the lower-
// numbered box.  Every in-radius pair is thus tested exactly once and
// registered on both molecules (smolreact.c:3201-3298 tests each pair once).
constexpr int kPairWin = 65;

template <bool SINGLE, int SURF, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) k_pairs_tile(KParams p) {
  constexpr int NW = BLOCK / 32;
  __shared__ float4 s_pc[NW][kPairWin];
  __shared__ ull s_id[NW][kPairWin];
  __shared__ int s_cell[NW][kPairWin];
  __shared__ float s_rsv[kMaxSpecies];  // stencil radius per species (one replicate)
  pdl_launch_dependents();
  pdl_wait();
  if (SINGLE) {
    for (int k = threadIdx.x; k < c_net.nsp; k += blockDim.x) s_rsv[k] = p.rsearch[k];
    __syncthreads();
  }
  const int n = *p.b_n;
  const uint32_t step = *p.step;
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int nwarps = gridDim.x * NW;
  float4 *wpc = s_pc[w];
  ull *wid = s_id[w];
  int *wcell = s_cell[w];
  uint32_t *facebits = reinterpret_cast<uint32_t *>(p.face);
  int extra = 0;
  // registers for the next window: entries wb+lane, wb+32+lane, and (lane 0) wb+64
  float4 pa = make_float4(0.f, 0.f, 0.f, 0.f), pb = pa, pc64 = pa;
  ull ia = 0, ib = 0, i64 = 0;
  auto prefetch = [&](int wb) {
    if (wb + lane < n) { pa = p.b_pc[wb + lane]; ia = p.b_id[wb + lane]; }
    if (wb + 32 + lane < n) { pb = p.b_pc[wb + 32 + lane]; ib = p.b_id[wb + 32 + lane]; }
    if (lane == 0 && wb + 64 < n) { pc64 = p.b_pc[wb + 64]; i64 = p.b_id[wb + 64]; }
  };
  auto stage = [&](int slot, int g, float4 q, ull qd) {
    if (g < n) {
      wpc[slot] = q;
      wid[slot] = qd;
      // box key: with one replicate the packed box coordinates identify the
      // box; across replicates the global box index does
      if (SINGLE) {
        wcell[slot] = (int)__float_as_uint(q.w);
      } else {
        const DevGeo &gg = geo_of<SINGLE>(p, id_rep(qd));
        wcell[slot] = global_cell(gg, __float_as_uint(q.w));
      }
    } else {
      wcell[slot] = -1;
      wid[slot] = make_id(kDeadSpecies, 0, 0);
    }
  };
  const int first = (blockIdx.x * NW + w) * 32;
  if (first < n) prefetch(first);
  for (int wb = first; wb < n; wb += nwarps * 32) {
    __syncwarp();
    stage(lane, wb + lane, pa, ia);
    stage(32 + lane, wb + 32 + lane, pb, ib);
    if (lane == 0) stage(64, wb + 64, pc64, i64);
    __syncwarp();
    if (wb + nwarps * 32 < n) prefetch(wb + nwarps * 32);
    const int i = wb + lane;
    const ull idi = wid[lane];
    const int sp = id_species(idi);
    const bool act = i < n && sp != kDeadSpecies && ((c_net.pair_any >> sp) & 1u);
    const int rep = SINGLE ? 0 : id_rep(idi);
    const float rs = act ? (SINGLE ? s_rsv[sp] : p.rsearch[rep * c_net.nsp + sp]) : 0.f;
    const float rs2 = rs * rs;
    const float4 pc = wpc[lane];
    const int cell = wcell[lane];
    // box boundaries in the window: bit b set when entry b is the last of its box
    const unsigned b_lo = __ballot_sync(0xffffffffu, wcell[lane] != wcell[lane + 1]);
    const unsigned b_hi = __ballot_sync(0xffffffffu, wcell[lane + 32] != wcell[lane + 33]);
    const unsigned long long ahead = (((unsigned long long)b_hi << 32) | b_lo) >> lane;
    int c = 0;            // same-box partners after this molecule inside the window
    bool spill = false;   // the box continues past the window
    if (act) {
      if (ahead) c = __ffsll((long long)ahead) - 1;
      else { c = 63 - lane; spill = true; }
    }
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int excl = incl - c;
    const int npairs = __shfl_sync(0xffffffffu, incl, 31);
    for (int q0 = 0; q0 < npairs; q0 += 32) {
      const int q = q0 + lane;
      // owner: the last lane whose first pair number is <= q
      int o = 0;
#pragma unroll
      for (int st = 16; st > 0; st >>= 1)
        if (__shfl_sync(0xffffffffu, excl, o + st) <= q) o += st;
      const int off = q - __shfl_sync(0xffffffffu, excl, o);
      const float rs2o = __shfl_sync(0xffffffffu, rs2, o);
      if (q < npairs) {
        const int tj = o + 1 + off;
        const float4 a = wpc[o], b = wpc[tj];
        const float vx = b.x - a.x, vy = b.y - a.y, vz = b.z - a.z;
        const float d2 = vx * vx + vy * vy + vz * vz;
        if (d2 <= rs2o) {
          const ull ida = wid[o], idb = wid[tj];
          const int spa = id_species(ida), spb = id_species(idb);
          const int repa = SINGLE ? 0 : id_rep(ida);
          // the reaction test draws from a stateless stream, so it can go
          // before the (rarely needed) surface test
          if (spb != kDeadSpecies && ((c_net.pair_mask[spa] >> spb) & 1u) &&
              pair_reaction<(SURF >= 2)>(p, repa, spa, spb, d2, id_stream(ida), id_stream(idb), step, wb + o, wb + tj) >= 0 &&
              !(SURF && pair_crosses_surface<(SURF >= 2)>(p.geo[repa], a, vx, vy, vz)))
            extra += register_pair(p, wb + o, wb + tj, d2);
        }
      }
    }
    // a box longer than the window continues in global memory
    if (spill) {
      const int gcell = SINGLE ? global_cell(geo_of<SINGLE>(p, 0), __float_as_uint(pc.w)) : cell;
      const int e = min(p.start[gcell + 1], n);
      for (int j = wb + 64; j < e; ++j) {
        const float4 b = p.b_pc[j];
        const float vx = b.x - pc.x, vy = b.y - pc.y, vz = b.z - pc.z;
        const float d2 = vx * vx + vy * vy + vz * vz;
        if (d2 > rs2) continue;
        const ull idb = p.b_id[j];
        const int spb = id_species(idb);
        if (spb != kDeadSpecies && ((c_net.pair_mask[sp] >> spb) & 1u) &&
            pair_reaction<(SURF >= 2)>(p, rep, sp, spb, d2, id_stream(idi), id_stream(idb), step, i, j) >= 0 &&
            !(SURF && pair_crosses_surface<(SURF >= 2)>(p.geo[rep], pc, vx, vy, vz)))
          extra += register_pair(p, i, j, d2);
      }
    }
    // Molecules near a box face also need the neighbouring boxes.  Cross-box
    // pairs are tested from the lower-numbered box, so only molecules whose
    // stencil reaches a higher-numbered box are flagged: those near a high
    // face, or near a low face that wraps (periodic) to the far end.
    bool face = false;
    if (act) {
      const DevGeo &g = geo_of<SINGLE>(p, rep);
      int ix, iy, iz;
      unpack_cell(__float_as_uint(pc.w), ix, iy, iz);
      const float ub0 = (ix == g.n[0] - 1) ? g.whi[0] : g.h[0];
      const float ub1 = (iy == g.n[1] - 1) ? g.whi[1] : g.h[1];
      const float ub2 = (iz == g.n[2] - 1) ? g.whi[2] : g.h[2];
      face = pc.x > ub0 - rs || pc.y > ub1 - rs || pc.z > ub2 - rs ||
             (pc.x < rs && ix == 0 && g.wall[0] == kWallPeriodic) ||
             (pc.y < rs && iy == 0 && g.wall[2] == kWallPeriodic) ||
             (pc.z < rs && iz == 0 && g.wall[4] == kWallPeriodic);
    }
    const unsigned fm = __ballot_sync(0xffffffffu, face);
    if (lane == 0) facebits[wb >> 5] = fm;
  }
  if (extra) atomicAdd(&p.counters[5], (unsigned long long)extra);
}

// Position of the k-th (from 0) set bit of m; k < popc(m).
__device__ __forceinline__ int nth_set_bit(uint32_t m, int k) {
  int pos = 0;
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    const uint32_t low = m & ((1u << w) - 1u);
    const int c = __popc(low);
    if (k >= c) {
      k -= c;
      m >>= w;
      pos += w;
    } else {
      m = low;
    }
  }
  return pos;
}

// Upward neighbour boxes of molecule i that its stencil reaches: bit
// (dz+1)*9 + (dy+1)*3 + (dx+1) is set for each offset whose box (after the
// periodic wrap) has a higher global number than i's own box, the boxes
// face_walk visits.
template <bool SINGLE>
__device__ __forceinline__ uint32_t face_boxes(const KParams &p, float4 pc, ull idi) {
  const int sp = id_species(idi);
  const int rep = SINGLE ? 0 : id_rep(idi);
  const DevGeo &g = geo_of<SINGLE>(p, rep);
  const float rs = p.rsearch[rep * c_net.nsp + sp];
  int ix, iy, iz;
  unpack_cell(__float_as_uint(pc.w), ix, iy, iz);
  const int cell = global_cell(g, __float_as_uint(pc.w));
  const float ub0 = (ix == g.n[0] - 1) ? g.whi[0] : g.h[0];
  const float ub1 = (iy == g.n[1] - 1) ? g.whi[1] : g.h[1];
  const float ub2 = (iz == g.n[2] - 1) ? g.whi[2] : g.h[2];
  const int xlo = pc.x < rs ? -1 : 0, xhi = pc.x > ub0 - rs ? 1 : 0;
  const int ylo = pc.y < rs ? -1 : 0, yhi = pc.y > ub1 - rs ? 1 : 0;
  const int zlo = pc.z < rs ? -1 : 0, zhi = pc.z > ub2 - rs ? 1 : 0;
  const bool px = g.wall[0] == kWallPeriodic, py = g.wall[2] == kWallPeriodic, pz = g.wall[4] == kWallPeriodic;
  uint32_t m = 0;
  for (int dz = zlo; dz <= zhi; ++dz) {
    int z = iz + dz;
    if (z < 0 || z >= g.n[2]) {
      if (!pz) continue;
      z = (z < 0) ? z + g.n[2] : z - g.n[2];
    }
    for (int dy = ylo; dy <= yhi; ++dy) {
      int y = iy + dy;
      if (y < 0 || y >= g.n[1]) {
        if (!py) continue;
        y = (y < 0) ? y + g.n[1] : y - g.n[1];
      }
      const int rowbase = g.cell0 + (z * g.n[1] + y) * g.n[0];
      for (int dx = xlo; dx <= xhi; ++dx) {
        if (dx == 0 && dy == 0 && dz == 0) continue;
        int x = ix + dx;
        if (x < 0 || x >= g.n[0]) {
          if (!px) continue;
          x = (x < 0) ? x + g.n[0] : x - g.n[0];
        }
        if (rowbase + x <= cell) continue;
        m |= 1u << ((dz + 1) * 9 + (dy + 1) * 3 + (dx + 1));
      }
    }
  }
  return m;
}

// Cross-box pairs of molecule i with the molecules of one upward neighbour
// box (offset code k of face_boxes); the closest reacting partner found is
// registered on i, every reacting pair on the partner.
template <bool SINGLE, int SURF>
__device__ __forceinline__ void face_box_walk(const KParams &p, int i, float4 pc, ull idi, int k, int n,
                                              uint32_t step, int &extra) {
  const int sp = id_species(idi);
  const int rep = SINGLE ? 0 : id_rep(idi);
  const DevGeo &g = geo_of<SINGLE>(p, rep);
  const float rs = p.rsearch[rep * c_net.nsp + sp];
  const float rs2 = rs * rs;
  const int dz = k / 9 - 1, dy = (k / 3) % 3 - 1, dx = k % 3 - 1;
  int ix, iy, iz;
  unpack_cell(__float_as_uint(pc.w), ix, iy, iz);
  int x = ix + dx, y = iy + dy, z = iz + dz;
  if (x < 0) x += g.n[0]; else if (x >= g.n[0]) x -= g.n[0];
  if (y < 0) y += g.n[1]; else if (y >= g.n[1]) y -= g.n[1];
  if (z < 0) z += g.n[2]; else if (z >= g.n[2]) z -= g.n[2];
  const int c = g.cell0 + (z * g.n[1] + y) * g.n[0] + x;
  const int s0 = p.start[c], e0 = min(p.start[c + 1], n);
  ull best = ~0ull;
  for (int j = s0; j < e0; ++j) {
    const float4 q = p.b_pc[j];
    const float vx = (q.x - pc.x) + (float)dx * g.h[0];
    const float vy = (q.y - pc.y) + (float)dy * g.h[1];
    const float vz = (q.z - pc.z) + (float)dz * g.h[2];
    const float d2 = vx * vx + vy * vy + vz * vz;
    if (d2 <= rs2)  // the partner's identity is read only for in-radius pairs
      try_pair<SURF>(p, i, idi, sp, rep, d2, j, p.b_id[j], rs2, step, best, extra, pc, vx, vy, vz);
  }
  if (best != ~0ull) extra += register_candidate(p, i, best);
}

// Cross-box pairs for the molecules flagged in the face bitmask by
// k_pairs_tile.  Each warp reads up to 32 bitmask words (1024 molecules; fewer
// when the system is too small to give every warp 32) at once, numbers their
// set bits with a warp prefix sum and takes the flagged
// molecules 32 at a time, one per lane; each such molecule lists the upward
// neighbour boxes its stencil reaches, and a second prefix sum hands the
// (molecule, neighbour box) items out 32 at a time, so a molecule reaching
// several boxes spreads over several lanes.
template <bool SINGLE, int SURF>
__global__ void __launch_bounds__(256) k_pairs_faces(KParams p) {
  pdl_launch_dependents();
  pdl_wait();
  const int n = *p.b_n;
  const int nwords = (n + 31) >> 5;
  const uint32_t step = *p.step;
  const uint32_t *facebits = reinterpret_cast<const uint32_t *>(p.face);
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  // words per warp: 32 (most words are sparse, and a group's fixed cost is
  // paid once for 32 of them) unless the system is so small that fewer than
  // one warp in eight would get a group; then fewer (a power of two, >= 1)
  int wpw = 32;
  while (wpw > 1 && 8ll * nwords < (long long)nw * wpw) wpw >>= 1;
  int extra = 0;
  for (int base = gw * wpw; base < nwords; base += nw * wpw) {
    const uint32_t bits = (lane < wpw && base + lane < nwords) ? facebits[base + lane] : 0u;
    const int cnt = __popc(bits);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int excl = incl - cnt;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    for (int q0 = 0; q0 < total; q0 += 32) {
      const int q = q0 + lane;
      int o = 0;
#pragma unroll
      for (int st = 16; st > 0; st >>= 1)
        if (__shfl_sync(0xffffffffu, excl, o + st) <= q) o += st;
      const uint32_t m = __shfl_sync(0xffffffffu, bits, o);
      const int r = q - __shfl_sync(0xffffffffu, excl, o);
      int i = 0;
      float4 pc = make_float4(0.f, 0.f, 0.f, 0.f);
      ull idi = 0;
      uint32_t boxes = 0;
      if (q < total) {
        i = ((base + o) << 5) + nth_set_bit(m, r);
        pc = p.b_pc[i];
        idi = p.b_id[i];
        boxes = face_boxes<SINGLE>(p, pc, idi);
      }
      // second level: the (molecule, neighbour box) items of these molecules
      const int c2 = __popc(boxes);
      int incl2 = c2;
#pragma unroll
      for (int u = 1; u < 32; u <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl2, u);
        if (lane >= u) incl2 += y;
      }
      const int excl2 = incl2 - c2;
      const int total2 = __shfl_sync(0xffffffffu, incl2, 31);
      for (int q1 = 0; q1 < total2; q1 += 32) {
        const int qq = q1 + lane;
        int oo = 0;
#pragma unroll
        for (int st = 16; st > 0; st >>= 1)
          if (__shfl_sync(0xffffffffu, excl2, oo + st) <= qq) oo += st;
        const int rr = qq - __shfl_sync(0xffffffffu, excl2, oo);
        const int io = __shfl_sync(0xffffffffu, i, oo);
        const uint32_t bo = __shfl_sync(0xffffffffu, boxes, oo);
        float4 po;
        po.x = __shfl_sync(0xffffffffu, pc.x, oo);
        po.y = __shfl_sync(0xffffffffu, pc.y, oo);
        po.z = __shfl_sync(0xffffffffu, pc.z, oo);
        po.w = __shfl_sync(0xffffffffu, pc.w, oo);
        const ull ido = __shfl_sync(0xffffffffu, idi, oo);
        if (qq < total2) face_box_walk<SINGLE, SURF>(p, io, po, ido, nth_set_bit(bo, rr), n, step, extra);
      }
    }
  }
  if (extra) atomicAdd(&p.counters[5], (unsigned long long)extra);
}

// Re-search for candidates still alive (conflict-resolution rounds >= 2).
template <int SURF>
__device__ __forceinline__ void research_body(const KParams &p, uint32_t step) {
  const int nc = min(*p.ncand, p.candcap);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nc; t += gridDim.x * blockDim.x) {
    const int i = p.cand[t];
    const ull id = p.b_id[i];
    if (id_species(id) == kDeadSpecies) continue;
    int ncd;
    p.best[i] = search_partner<SURF>(p, i, p.b_pc[i], id, step, ncd);
  }
}

template <int SURF>
__global__ void k_research(KParams p) {
  pdl_launch_dependents();
  pdl_wait();
  research_body<SURF>(p, *p.step);
}

// Site of a bimolecular reaction, in the local frame of molecule i
// (x = D2/(D1+D2) weighting, smolreact.c:2693-2697).
__device__ __forceinline__ float4 pair_site(const KParams &p, int i, int j, int r, int rep) {
  const float4 a = p.b_pc[i], b = p.b_pc[j];
  const DevGeo g = p.geo[rep];
  int ia[3], ib[3];
  unpack_cell(__float_as_uint(a.w), ia[0], ia[1], ia[2]);
  unpack_cell(__float_as_uint(b.w), ib[0], ib[1], ib[2]);
  const float ua[3] = {a.x, a.y, a.z}, ub[3] = {b.x, b.y, b.z};
  const int spa = id_species(p.b_id[i]);
  const int r1 = c_net.rct[2][r][0];
  const int spb = id_species(p.b_id[j]);
  const float da = p.difstep[rep * c_net.nsp + spa], db = p.difstep[rep * c_net.nsp + spb];
  // difstep^2 is proportional to D, so the weights follow from difstep^2
  const float Da = da * da, Db = db * db;
  float fa;  // fraction of the way from a toward b
  if (Da == 0.f && Db == 0.f) fa = 0.5f;
  else fa = Da / (Da + Db);
  (void)r1;
  (void)spb;
  int cell[3];
  float w[3];
  for (int d = 0; d < 3; ++d) {
    int dc = ib[d] - ia[d];
    if (dc > 1) dc -= g.n[d];
    else if (dc < -1) dc += g.n[d];
    const float v = (ub[d] - ua[d]) + (float)dc * g.h[d];
    w[d] = ua[d] + fa * v;
    cell[d] = ia[d];
    renorm(w[d], cell[d], g.h[d], g.inv_h[d]);
    int hits = 0;
    if (cell[d] < 0 || cell[d] > g.n[d] - 1 || (cell[d] == g.n[d] - 1 && w[d] > g.whi[d]))
      walls_dim(w[d], cell[d], g, d, hits);
    clamp_cell(w[d], cell[d], g, d);
  }
  return make_float4(w[0], w[1], w[2], __uint_as_float(pack_cell(cell[0], cell[1], cell[2])));
}

template <int SURF>
__device__ __forceinline__ void commit_body(const KParams &p, uint32_t step) {
  const int nc = min(*p.ncand, p.candcap);
  int done = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nc; t += gridDim.x * blockDim.x) {
    const int i = p.cand[t];
    const ull bi = p.best[i];
    if (bi == ~0ull) continue;
    const int j = (int)(uint32_t)bi;
    if (j <= i) continue;
    const ull bj = p.best[j];
    if ((int)(uint32_t)bj != i) continue;
    const ull idi = p.b_id[i], idj = p.b_id[j];
    const int spi = id_species(idi), spj = id_species(idj);
    if (spi == kDeadSpecies || spj == kDeadSpecies) continue;
    const int rep = id_rep(idi);
    const float d2 = __uint_as_float((uint32_t)(bi >> 32));
    const int r = pair_reaction<(SURF >= 2)>(p, rep, spi, spj, d2, id_stream(idi), id_stream(idj), step, i, j);
    if (r < 0) continue;
    // reactant 1 of reaction r is molecule a
    const bool i_first = (c_net.rct[2][r][0] == spi);
    const int a = i_first ? i : j, b = i_first ? j : i;
    Event e;
    e.site = pair_site(p, a, b, r, rep);
    const ull ka = id_stream(p.b_id[a]), kb = id_stream(p.b_id[b]);
    e.key = mix64(ka * 0x9E3779B97F4A7C15ull ^ kb) & ((1ull << kSpShift) - 1);
    e.rxn = (2u << 8) | (uint32_t)r;
    e.rep = (uint32_t)rep;
    e.ia = a;
    e.ib = b;
    push_event(p, e);
    p.b_id[i] = id_mark_dead(idi);
    p.b_id[j] = id_mark_dead(idj);
    atomicAdd((unsigned long long *)&p.spcount[rep * c_net.nsp + spi], (unsigned long long)(-1ll));
    atomicAdd((unsigned long long *)&p.spcount[rep * c_net.nsp + spj], (unsigned long long)(-1ll));
    done++;
  }
  if (done) atomicAdd(&p.counters[3], (unsigned long long)done);
}

template <int SURF>
__global__ void k_commit(KParams p) {
  pdl_launch_dependents();
  pdl_wait();
  commit_body<SURF>(p, *p.step);
}

// ---- product placement -----------------------------------------------------
// Uniformly random rotation matrix from a random unit quaternion (Shoemake,
// Graphics Gems III, 1992).
__device__ __forceinline__ void random_rotation(uint4 r, float m[9]) {
  const float u1 = u01f_open(r.x), u2 = u01f_open(r.y) * 6.28318530718f, u3 = u01f_open(r.z) * 6.28318530718f;
  const float s1 = sqrtf(1.f - u1), s2 = sqrtf(u1);
  float sn2, cs2, sn3, cs3;
  __sincosf(u2, &sn2, &cs2);
  __sincosf(u3, &sn3, &cs3);
  const float qx = s1 * sn2, qy = s1 * cs2, qz = s2 * sn3, qw = s2 * cs3;
  m[0] = 1.f - 2.f * (qy * qy + qz * qz); m[1] = 2.f * (qx * qy - qz * qw); m[2] = 2.f * (qx * qz + qy * qw);
  m[3] = 2.f * (qx * qy + qz * qw); m[4] = 1.f - 2.f * (qx * qx + qz * qz); m[5] = 2.f * (qy * qz - qx * qw);
  m[6] = 2.f * (qx * qz - qy * qw); m[7] = 2.f * (qy * qz + qx * qw); m[8] = 1.f - 2.f * (qx * qx + qy * qy);
}

// The random orientation of a reaction's product offsets in the system's
// dimension (doreact smolreact.c:2840-2851): a uniformly random rotation in
// 3-D, a rotation by a uniform angle in the plane in 2-D (DirCosM2D), and a
// random sign in 1-D, so the offsets keep their length.
__device__ __forceinline__ void random_orientation(uint4 r, int dim, float m[9]) {
  if (dim >= 3) {
    random_rotation(r, m);
    return;
  }
  for (int k = 0; k < 9; ++k) m[k] = (k % 4 == 0) ? 1.f : 0.f;
  if (dim == 2) {
    float sn, cs;
    __sincosf(u01f_open(r.x) * 6.28318530718f, &sn, &cs);
    m[0] = cs; m[1] = -sn;
    m[3] = sn; m[4] = cs;
  } else {
    m[0] = (r.x & 1u) ? 1.f : -1.f;
  }
}

// Birth position in compartment c (compartrandpos, smolcomparts.c:194-220):
// uniform points in the system until one lies in the compartment, at most
// 10000 tries, then one of its interior points.  site/cell hold the first
// (uniform) try on entry.
__device__ __noinline__ void birth_in_cmpt(int c, const DevGeo &g, ull ekey, uint32_t step, float site[3],
                                           int cell[3]) {
  const uint2 key = make_uint2(c_net.key0 ^ 0x1B873593u, c_net.key1 ^ 0xCC9E2D51u);
  for (int t = 0; t < 10000; ++t) {
    double x[3];
    to_abs(g, cell, site, x);
    if (pos_in_cmpt(c_cmpt, c, c_panels, x)) return;
    const uint4 rr = philox(make_uint4((uint32_t)ekey, (uint32_t)(ekey >> 32), step, 32u + (uint32_t)t), key);
    const uint32_t bits[3] = {rr.x, rr.y, rr.z};
    for (int d = 0; d < 3; ++d) {
      if (d >= g.dim) continue;
      const float L = (float)(g.n[d] - 1) * g.h[d] + g.whi[d];
      float w = u01f_open(bits[d]) * L;
      int j = 0;
      renorm(w, j, g.h[d], g.inv_h[d]);
      if (j > g.n[d] - 1) { w += (float)(j - (g.n[d] - 1)) * g.h[d]; j = g.n[d] - 1; }
      clamp_cell(w, j, g, d);
      site[d] = w;
      cell[d] = j;
    }
  }
  const DevCmpt &q = c_cmpt[c];
  if (q.npts <= 0) return;
  double x[3];
  for (int d = 0; d < 3; ++d) x[d] = q.pts[(int)(ekey % (ull)q.npts)][d];
  int ix[3];
  float u[3];
  from_abs(g, x, ix, u);
  for (int d = 0; d < 3; ++d) {
    site[d] = u[d];
    cell[d] = ix[d];
  }
}

// Products of one event (doreact, smolreact.c:2662-2902; births: zeroreact,
// smolreact.c:2905-2995): positions from the event site, the unbinding
// offsets under one random rotation per event (or the confspread / bounce
// placements), walls and surfaces for the new molecules, serial numbers.
template <int SURF, class Emit>
__device__ void surface_birth(const KParams &p, const Event &e, int r, int rep, uint32_t step, Emit emit);

// emit(position, identity) stores one new molecule.  uni counts the
// first-order events.
template <int SURF, class Emit>
__device__ __forceinline__ void place_event(const KParams &p, const Event &e, uint32_t step, int &uni, Emit emit) {
  const uint2 key = make_uint2(c_net.key0 ^ 0x68E31DA4u, c_net.key1 ^ 0xB5297A4Du);
  const int order = (int)(e.rxn >> 8), r = (int)(e.rxn & 0xFF), rep = (int)e.rep;
  const DevGeo g = p.geo[rep];
  const uint4 rr = philox(make_uint4((uint32_t)e.key, (uint32_t)(e.key >> 32), step, 7u), key);
  float site[3];
  int cell[3];
  if (SURF && order == 0 && c_net.rsrf[0][r] && !c_net.cmpt[0][r]) {  // births on a surface (a compartment wins)
    surface_birth<SURF>(p, e, r, rep, step, emit);
    return;
  }
  if (order == 0) {  // uniform position in the system (smolwall.c:42)
    const uint32_t bits[3] = {rr.x, rr.y, rr.z};
    for (int d = 0; d < 3; ++d) {
      if (d >= g.dim) { site[d] = 0.f; cell[d] = 0; continue; }
      const float L = (float)(g.n[d] - 1) * g.h[d] + g.whi[d];
      float w = u01f_open(bits[d]) * L;
      int j = 0;
      renorm(w, j, g.h[d], g.inv_h[d]);
      if (j > g.n[d] - 1) { w += (float)(j - (g.n[d] - 1)) * g.h[d]; j = g.n[d] - 1; }
      clamp_cell(w, j, g, d);
      site[d] = w;
      cell[d] = j;
    }
    if (SURF >= 2 && c_net.cmpt[0][r]) birth_in_cmpt(c_net.cmpt[0][r] - 1, g, e.key, step, site, cell);
  } else {
    site[0] = e.site.x; site[1] = e.site.y; site[2] = e.site.z;
    unpack_cell(__float_as_uint(e.site.w), cell[0], cell[1], cell[2]);
    if (order == 1) {
      uni++;
      atomicAdd((unsigned long long *)&p.spcount[rep * c_net.nsp + c_net.rct[1][r][0]],
                (unsigned long long)(-1ll));
    }
  }
  const int np = c_net.nprod[order][r];
  // confspread / bounce (doreact, smolreact.c:2736-2805): products 1 and 2
  // take (confspread) or are pushed apart from (bounce) the reactants'
  // places, keep the reactants' serial numbers, and the rest sit at the site
  const int place = order == 2 ? c_net.placement2[r] : 0;
  float cust[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
  ull keep_sn[2] = {0, 0};
  if (place) {
    float va[3], vb[3];
    int cs[3];
    unpack_cell(__float_as_uint(e.site.w), cs[0], cs[1], cs[2]);
    const float us[3] = {e.site.x, e.site.y, e.site.z};
    for (int k = 0; k < 2; ++k) {
      const int idx = k == 0 ? e.ia : e.ib;
      const float4 q = p.b_pc[idx];
      keep_sn[k] = id_serno(p.b_id[idx]);
      int cq[3];
      unpack_cell(__float_as_uint(q.w), cq[0], cq[1], cq[2]);
      const float uq[3] = {q.x, q.y, q.z};
      float *v = k == 0 ? va : vb;
      for (int d = 0; d < 3; ++d) {  // site -> reactant, nearest periodic image
        int dc = cq[d] - cs[d];
        if (dc > 1) dc -= g.n[d];
        else if (dc < -1) dc += g.n[d];
        v[d] = d < g.dim ? (uq[d] - us[d]) + (float)dc * g.h[d] : 0.f;
      }
    }
    if (place == 1) {
      for (int d = 0; d < 3; ++d) { cust[0][d] = va[d]; cust[1][d] = vb[d]; }
    } else {
      float v[3] = {vb[0] - va[0], vb[1] - va[1], vb[2] - va[2]};
      float dist = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      if (dist == 0.f) {
        dist = sqrtf(p.bind2[rep * c_net.nr[2] + r]);
        v[0] = dist;
      }
      const int kx2 = c_net.rxn_base[2] + r;
      const float *pp = p.prdpos + (size_t)(rep * c_net.nrx_total + kx2) * kMaxProd * 3;
      const float p0 = pp[0], p1 = pp[3];
      const float x = c_net.bounce_k[r] * (1.f / dist - 1.f / (p0 + p1));
      for (int d = 0; d < 3; ++d) {
        cust[0][d] = va[d] - x * p0 * v[d];
        cust[1][d] = vb[d] + x * p1 * v[d];
      }
    }
  }
  float m[9];
  bool rot = false;
  if (!place && c_net.has_offset[order][r] && !c_net.fixed[order][r] && !c_net.inject) {
    random_orientation(philox(make_uint4((uint32_t)e.key, (uint32_t)(e.key >> 32), step, 8u), key), g.dim, m);
    rot = true;
  }
  const int kx = c_net.rxn_base[order] + r;
  for (int q = 0; q < np; ++q) {
    const int psp = c_net.prd[order][r][q];
    float off[3] = {0.f, 0.f, 0.f};
    if (place) {
      if (q < 2) { off[0] = cust[q][0]; off[1] = cust[q][1]; off[2] = cust[q][2]; }
    } else if (c_net.has_offset[order][r]) {
      const float *pp = p.prdpos + ((size_t)(rep * c_net.nrx_total + kx) * kMaxProd + q) * 3;
      if (rot) {
        off[0] = m[0] * pp[0] + m[1] * pp[1] + m[2] * pp[2];
        off[1] = m[3] * pp[0] + m[4] * pp[1] + m[5] * pp[2];
        off[2] = m[6] * pp[0] + m[7] * pp[1] + m[8] * pp[2];
      } else {
        off[0] = pp[0]; off[1] = pp[1]; off[2] = pp[2];
      }
    }
    float w[3];
    int c[3];
    bool dead = false;
    int hits = 0;
    for (int d = 0; d < 3; ++d) {
      w[d] = site[d] + (d < g.dim ? off[d] : 0.f);
      c[d] = cell[d];
      renorm(w[d], c[d], g.h[d], g.inv_h[d]);
      if (d < g.dim && (c[d] <= 0 || c[d] >= g.n[d] - 1))
        if (walls_dim(w[d], c[d], g, d, hits)) dead = true;
      clamp_cell(w[d], c[d], g, d);
    }
    const ull serno = (place && q < 2) ? keep_sn[q]
                                       : kProductSernoBit |
                                             (mix64(e.key ^ ((ull)q << 50) ^ ((ull)step << 20) ^ (ull)(order * 97 + r)) &
                                              (kProductSernoBit - 1));
    int fsp = psp;
    if (SURF && !dead) {
      // new molecules are checked against surfaces from the reaction site
      // (smolsim.cpp:2656-2660, reborn pass of checksurfaces)
      double x0[3], x1[3];
      to_abs(g, cell, site, x0);
      to_abs(g, c, w, x1);
      if (SURF == 3) {
        int pnl = 0, ms = 0;
        const int res = walk_soln_rules(p, fsp, x0, x1, hits, id_stream(make_id(psp, rep, serno)), step, kCtrSrfWalk,
                                        pnl, ms);
        if (res == 1) {
          dead = true;
        } else if (res == 2) {  // adsorbed on placement: into the bound list
          BoundMol bm;
          for (int d = 0; d < 3; ++d) bm.x[d] = x1[d];
          bm.id = make_id(fsp, 0, serno);
          bm.pnl = pnl;
          bm.ms = ms;
          bm.born = step;
          push_bound(p, bm);
          atomicAdd((unsigned long long *)&p.spcount[fsp], 1ull);
          dead = true;
        } else {
          from_abs(g, x1, c, w);
        }
      } else if (surface_interact<(SURF >= 2)>(psp, x0, x1, c_net.surf_eps, hits)) {
        dead = true;
      } else {
        from_abs(g, x1, c, w);
      }
    }
    if (hits) atomicAdd(&p.counters[0], (unsigned long long)hits);
    if (dead) continue;
    emit(make_float4(w[0], w[1], w[2], __uint_as_float(pack_cell(c[0], c[1], c[2]))), make_id(fsp, rep, serno));
  }
}

// A uniformly random point of a panel (panelrandpos, smolsurface.c), from
// three uniforms: a rectangle's extent, a triangle by the square-root rule, a
// sphere's surface (a circle in 2-D), a cylinder's side, the closed side of
// a hemisphere, a disk by the square-root rule.
__device__ void panel_random_point(const DevPanel &pn, int dim, uint32_t a, uint32_t b, uint32_t c, double x[3]) {
  const double u1 = u01co(a), u2 = u01co(b), u3 = u01co(c), tau = 6.283185307179586;
  auto basis = [&](const double n[3], double e1[3], double e2[3]) {  // two unit vectors perpendicular to n
    const double t[3] = {fabs(n[0]) < 0.9 ? 1.0 : 0.0, fabs(n[0]) < 0.9 ? 0.0 : 1.0, 0.0};
    e1[0] = t[1] * n[2] - t[2] * n[1];
    e1[1] = t[2] * n[0] - t[0] * n[2];
    e1[2] = t[0] * n[1] - t[1] * n[0];
    const double l = sqrt(dot3(e1, e1));
    for (int d = 0; d < 3; ++d) e1[d] /= l;
    e2[0] = n[1] * e1[2] - n[2] * e1[1];
    e2[1] = n[2] * e1[0] - n[0] * e1[2];
    e2[2] = n[0] * e1[1] - n[1] * e1[0];
  };
  switch (pn.shape) {
    case 0: {
      const double us[3] = {u1, u2, u3};
      for (int d = 0; d < 3; ++d) x[d] = d == pn.axis ? pn.pos : pn.lo[d] + us[d] * (pn.hi[d] - pn.lo[d]);
      return;
    }
    case 1: {
      const double r1 = sqrt(u1);
      for (int d = 0; d < 3; ++d) x[d] = (1 - r1) * pn.pt[0][d] + r1 * (1 - u2) * pn.pt[1][d] + r1 * u2 * pn.pt[2][d];
      return;
    }
    case 2:
    case 4: {
      if (dim == 2) {
        x[0] = pn.center[0] + pn.radius * cos(tau * u1);
        x[1] = pn.center[1] + pn.radius * sin(tau * u1);
        x[2] = 0;
        return;
      }
      const double z = 2 * u1 - 1, s = sqrt(fmax(0.0, 1 - z * z));
      double v[3] = {s * cos(tau * u2), s * sin(tau * u2), z};
      if (pn.shape == 4 && dot3(v, pn.nrm) > 0)
        for (int d = 0; d < 3; ++d) v[d] = -v[d];
      for (int d = 0; d < 3; ++d) x[d] = pn.center[d] + pn.radius * v[d];
      return;
    }
    case 3: {
      double e1[3], e2[3];
      basis(pn.nrm, e1, e2);
      for (int d = 0; d < 3; ++d)
        x[d] = pn.pt[0][d] + u1 * (pn.pt[1][d] - pn.pt[0][d]) +
               pn.radius * (cos(tau * u2) * e1[d] + sin(tau * u2) * e2[d]);
      return;
    }
    default: {
      double e1[3], e2[3];
      basis(pn.nrm, e1, e2);
      const double rr = pn.radius * sqrt(u1);
      for (int d = 0; d < 3; ++d) x[d] = pn.center[d] + rr * (cos(tau * u2) * e1[d] + sin(tau * u2) * e2[d]);
      return;
    }
  }
}

// Births of an order-0 reaction restricted to a surface (zeroreact,
// smolreact.c:2949-2992, surfrandpos): a panel of the surface chosen by area,
// a uniform point of it, and the products there (doreact with the panel):
// bound products on the panel on their state's side (into the output bound
// list), solution products just off its front (soln) or back (bsoln) side.
template <int SURF, class Emit>
__device__ void surface_birth(const KParams &p, const Event &e, int r, int rep, uint32_t step, Emit emit) {
  const DevGeo g = p.geo[rep];
  const int s = c_net.rsrf[0][r] - 1;
  const uint2 key = make_uint2(c_net.key0 ^ 0x3C6EF372u, c_net.key1 ^ 0xA54FF53Au);
  const uint4 rr = philox(make_uint4((uint32_t)e.key, (uint32_t)(e.key >> 32), step, 9u), key);
  double total = 0;
  for (int q = 0; q < c_net.npanel; ++q)
    if (c_panels[q].srf == s) total += c_net.parea[q];
  double u = u01co(rr.x) * total;
  int pk = -1;
  for (int q = 0; q < c_net.npanel; ++q) {
    if (c_panels[q].srf != s) continue;
    pk = q;
    if (u < c_net.parea[q]) break;
    u -= c_net.parea[q];
  }
  if (pk < 0) return;
  const DevPanel &pn = c_panels[pk];
  double x0[3];
  panel_random_point(pn, g.dim, rr.y, rr.z, rr.w, x0);
  const int np = c_net.nprod[0][r];
  for (int q = 0; q < np; ++q) {
    const int psp = c_net.prd[0][r][q], pst = c_net.pstate0[r][q];
    const ull serno = kProductSernoBit |
                      (mix64(e.key ^ ((ull)q << 50) ^ ((ull)step << 20) ^ (ull)r) & (kProductSernoBit - 1));
    double x[3] = {x0[0], x0[1], x0[2]};
    if (pst == kMSfront || pst == kMSback) {
      if (SURF == 3) {
        fix_to_panel(pn, x, ms_face(pst), c_net.beps);
        BoundMol bm;
        for (int d = 0; d < 3; ++d) bm.x[d] = x[d];
        bm.id = make_id(psp, 0, serno);
        bm.pnl = pk;
        bm.ms = pst;
        bm.born = step;
        push_bound(p, bm);
        atomicAdd((unsigned long long *)&p.spcount[psp], 1ull);
      }
      continue;
    }
    const int f = pst == kMSbsoln ? kFaceBack : kFaceFront;
    fix_to_panel(pn, x, f, c_net.beps);
    double n[3];
    face_normal(pn, x, f, n);
    const double sd = fabs(panel_sdist<true>(pn, x));
    if (sd < c_net.surf_eps)  // kept surf_eps off the panel, as solution molecules are
      for (int d = 0; d < 3; ++d) x[d] += (c_net.surf_eps - sd) * n[d];
    int c[3];
    float w[3];
    from_abs(g, x, c, w);
    emit(make_float4(w[0], w[1], w[2], __uint_as_float(pack_cell(c[0], c[1], c[2]))), make_id(psp, rep, serno));
  }
}

template <int SURF>
__device__ __forceinline__ void products_body(const KParams &p, uint32_t step) {
  const int ne = min(*p.nev, p.evcap);
  int uni = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ne; t += gridDim.x * blockDim.x) {
    place_event<SURF>(p, p.ev[t], step, uni, [&](float4 npc, ull nid) {
      const int slot = atomicAdd(p.q_n, 1);
      if (slot < p.pcap) {
        p.q_pc[slot] = npc;
        p.q_id[slot] = nid;
        atomicAdd((unsigned long long *)&p.spcount[id_rep(nid) * c_net.nsp + id_species(nid)], 1ull);
      } else {
        atomicOr(p.status, kStProdCap);
      }
    });
  }
  if (uni) atomicAdd(&p.counters[2], (unsigned long long)uni);
  // clear the candidate keys of this step
  const int nc = min(*p.ncand, p.candcap);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nc; t += gridDim.x * blockDim.x)
    p.best[p.cand[t]] = ~0ull;
}

template <int SURF>
__global__ void k_products(KParams p) {
  pdl_launch_dependents();
  pdl_wait();
  products_body<SURF>(p, *p.step);
}

// ===========================================================================
// Persistent ensemble engine
// ===========================================================================
// Replicates of an ensemble are independent, so they need none of the
// device-wide synchronisation of the step pipeline above.  One CTA takes a
// replicate from a work counter (largest replicates first) and runs a whole
// block of steps on it - move, box sort, pair search, conflict rounds,
// products - with block barriers between the phases, then takes the next
// replicate.  Each replicate owns a region of the persistent buffers with
// room to grow, and its boxes are numbered after the previous replicate's
// with one spare entry, so its box counts and starts (including the end of
// its last box) are private to it: a replicate's working set stays in L2
// while its CTA steps it.  The per-molecule functions are the step
// pipeline's own (advance_one, search_partner, pair_reaction, pair_site,
// place_event), keyed by the same serial numbers and step counters, so a
// replicate follows the trajectory it follows in the step pipeline up to the
// order in which equidistant candidates are ranked.
struct PersistArgs {
  const int *order;  // replicate processing order (largest first)
  const int *roff;   // region offset of each replicate
  const int *rcap;   // region capacity of each replicate
  int *rn;           // entries (live or dead) of each replicate in the current buffer
  int *queue;        // work counter, zeroed before each launch
  Event *ev;         // event lists, evslice per CTA
  int evslice;
  int *cand;         // pair-candidate lists, candslice per CTA
  int candslice;
  int nrep;
  int nsteps;
};

constexpr int kPersistThreads = 256;
// Replicates with at most this many boxes keep their box counts and starts
// in shared memory (32 KB); larger ones use their slice of the global arrays.
constexpr int kPersistSmemBoxes = 4095;
#ifndef SMOLB_PERSIST_BLOCKS
#define SMOLB_PERSIST_BLOCKS 3
#endif

// Shared state of one CTA's step: event, candidate and product counters and
// the replicate's sorted count.
struct PersistShared {
  int nev, nc, np, ns;
  int warp[32];
};

template <int SURF>
__device__ __forceinline__ void persist_commit(const KParams &p, int rep, const int *cand, int nc, uint32_t step,
                                               Event *ev, int evcap, PersistShared &sh, int &done) {
  for (int t = threadIdx.x; t < nc; t += blockDim.x) {
    const int i = cand[t];
    const ull bi = p.best[i];
    if (bi == ~0ull) continue;
    const int j = (int)(uint32_t)bi;
    if (j <= i) continue;
    const ull bj = p.best[j];
    if ((int)(uint32_t)bj != i) continue;
    const ull idi = p.b_id[i], idj = p.b_id[j];
    const int spi = id_species(idi), spj = id_species(idj);
    if (spi == kDeadSpecies || spj == kDeadSpecies) continue;
    const float d2 = __uint_as_float((uint32_t)(bi >> 32));
    const int r = pair_reaction<(SURF >= 2)>(p, rep, spi, spj, d2, id_stream(idi), id_stream(idj), step, i, j);
    if (r < 0) continue;
    const bool i_first = (c_net.rct[2][r][0] == spi);
    const int a = i_first ? i : j, b = i_first ? j : i;
    Event e;
    e.site = pair_site(p, a, b, r, rep);
    const ull ka = id_stream(p.b_id[a]), kb = id_stream(p.b_id[b]);
    e.key = mix64(ka * 0x9E3779B97F4A7C15ull ^ kb) & ((1ull << kSpShift) - 1);
    e.rxn = (2u << 8) | (uint32_t)r;
    e.rep = (uint32_t)rep;
    e.ia = a;
    e.ib = b;
    const int k = atomicAdd(&sh.nev, 1);
    if (k < evcap) ev[k] = e;
    else atomicOr(p.status, kStEvCap);
    p.b_id[i] = id_mark_dead(idi);
    p.b_id[j] = id_mark_dead(idj);
    atomicAdd((unsigned long long *)&p.spcount[rep * c_net.nsp + spi], (unsigned long long)(-1ll));
    atomicAdd((unsigned long long *)&p.spcount[rep * c_net.nsp + spj], (unsigned long long)(-1ll));
    done++;
  }
}

// One time step of replicate `rep` (entries [off, off+n) of p.a_*): returns
// the entry count of its next state in p.b_*.  All threads of the block call
// it; it begins and ends at a block barrier.
// Box index of a packed cell within its replicate.
__device__ __forceinline__ int local_cell(const DevGeo &g, uint32_t w) {
  int ix, iy, iz;
  unpack_cell(w, ix, iy, iz);
  return (iz * g.n[1] + iy) * g.n[0] + ix;
}

// cnt / st: the replicate's box counts and starts, indexed by local box
// (shared memory for small replicates); cnt is zero on entry and on exit.
template <int SURF>
__device__ __forceinline__ int persist_step(const KParams &p, int rep, int off, int cap, int n, uint32_t step,
                                            const float *gtab, Event *ev, int evcap, int *cand, int candcap,
                                            PersistShared &sh, unsigned long long *acc, int *cnt, int *st) {
  const DevGeo &g = p.geo[rep];
  const int T = blockDim.x, tid = threadIdx.x;
  const int nb = g.n[0] * g.n[1] * g.n[2];
  const int c0 = g.cell0;
  if (tid == 0) { sh.nev = 0; sh.nc = 0; sh.np = 0; }
  __syncthreads();
  // ---- move (diffuse, walls, first-order decisions) and box histogram
  int hits = 0;
  for (int i = tid; i < n; i += T) {
    const int idx = off + i;
    float4 pc = p.a_pc[idx];
    ull id = p.a_id[idx];  // the persistent kernel runs without surfaces: id is not changed
    int fate = -1;
    if (id_species(id) != kDeadSpecies) fate = advance_one<false, SURF>(pc, id, step, p, gtab, 0, hits);
    if (fate == 0) {
      p.tmp[idx] = pc;
      atomicAdd(&cnt[local_cell(g, __float_as_uint(pc.w))], 1);
    } else {
      p.tmp[idx] = make_float4(0.f, 0.f, 0.f, __uint_as_float(kTmpGone));
      if (fate == 1) {
        atomicAdd((unsigned long long *)&p.spcount[rep * c_net.nsp + id_species(id)], (unsigned long long)(-1ll));
      } else if (fate >= 2) {
        Event e;
        e.site = pc;
        e.key = id_stream(id);
        e.rxn = (1u << 8) | (uint32_t)(fate - 2);
        e.rep = (uint32_t)rep;
        e.ia = e.ib = -1;
        const int k = atomicAdd(&sh.nev, 1);
        if (k < evcap) ev[k] = e;
        else atomicOr(p.status, kStEvCap);
      }
    }
  }
  acc[0] += (unsigned long long)hits;
  // zeroth-order births (the keys of births(): one Poisson draw per reaction)
  if (tid < c_net.nr[0]) {
    const int r = tid, nr0 = c_net.nr[0];
    const uint2 key = make_uint2(c_net.key0 ^ 0x5bd1e995u, c_net.key1);
    const int nbirth = poisson_sample(p.births[rep * nr0 + r], key, make_uint4((uint32_t)rep, (uint32_t)r, step, 0u));
    if (nbirth > 0) {
      const int base = atomicAdd(&sh.nev, nbirth);
      acc[1] += (unsigned long long)nbirth;
      for (int k = 0; k < nbirth; ++k) {
        if (base + k >= evcap) { atomicOr(p.status, kStEvCap); break; }
        Event e;
        e.site = make_float4(0.f, 0.f, 0.f, 0.f);
        e.key = mix64(((ull)rep << 40) ^ ((ull)r << 32) ^ ((ull)step << 8) ^ 0xB17Aull ^
                      mix64((ull)k + 0x9E37ull * (ull)step)) & ((1ull << kSpShift) - 1);
        e.rxn = (0u << 8) | (uint32_t)r;
        e.rep = (uint32_t)rep;
        e.ia = e.ib = -1;
        ev[base + k] = e;
      }
    }
  }
  __syncthreads();
  // ---- exclusive scan of the box counts into box starts (region offset off)
  {
    const int per = (nb + T - 1) / T;
    const int lo = min(nb, tid * per), hi = min(nb, lo + per);
    int sum = 0;
    for (int c = lo; c < hi; ++c) sum += cnt[c];
    int total;
    int run = off + block_exclusive_scan(sum, sh.warp, total);
    for (int c = lo; c < hi; ++c) {
      st[c] = run;
      run += cnt[c];
    }
    if (tid == 0) {
      st[nb] = off + total;
      sh.ns = total;
    }
  }
  __syncthreads();
  const int ns = sh.ns;
  if (ns > cap) {  // cannot happen: every counted molecule came from the region
    if (tid == 0) atomicOr(p.status, kStMolCap);
    return 0;
  }
  // ---- scatter into box order (one slot atomic per run of same-box lanes)
  for (int base = 0; base < n; base += T) {
    const int i = base + tid;
    float4 pc = make_float4(0.f, 0.f, 0.f, __uint_as_float(kTmpGone));
    if (i < n) pc = p.tmp[off + i];
    const bool alive = __float_as_uint(pc.w) != kTmpGone;
    const int cell = alive ? local_cell(g, __float_as_uint(pc.w)) : -1;
    const BoxRun run = box_run(alive, cell);
    int old = 0;
    if (alive && run.rank == 0) old = atomicSub(&cnt[cell], run.count);
    const int s0 = alive ? st[cell] : 0;
    old = __shfl_sync(0xffffffffu, old, alive ? run.head : (tid & 31));
    if (alive) {
      const int slot = s0 + old - run.count + run.rank;
      p.b_pc[slot] = pc;
      p.b_id[slot] = p.a_id[off + i];
    }
  }
  __syncthreads();
  // ---- pair search, round 1: every molecule with pair reactions finds its
  // closest reacting partner (search_partner, the step pipeline's re-search)
  int multi = 0;
  for (int j = tid; j < ns; j += T) {
    const int idx = off + j;
    const ull id = p.b_id[idx];
    const int sp = id_species(id);
    if (!((c_net.pair_any >> sp) & 1u)) continue;
    int ncd = 0;
    const ull best = search_partner_in<SURF>(p, idx, p.b_pc[idx], id, step, ncd, st, c0);
    if (ncd > 1) multi += ncd - 1;
    if (best != ~0ull) {
      p.best[idx] = best;
      const int k = atomicAdd(&sh.nc, 1);
      if (k < candcap) cand[k] = idx;
      else atomicOr(p.status, kStCandCap);
    }
  }
  acc[5] += (unsigned long long)multi;
  __syncthreads();
  const int nc = min(sh.nc, candcap);
  int done = 0;
  if (nc > 0) {
    persist_commit<SURF>(p, rep, cand, nc, step, ev, evcap, sh, done);
    for (int round = 1; round < c_net.rounds; ++round) {
      __syncthreads();
      for (int t = tid; t < nc; t += T) {  // losers search again among the molecules still present
        const int i = cand[t];
        const ull id = p.b_id[i];
        if (id_species(id) == kDeadSpecies) continue;
        int ncd;
        p.best[i] = search_partner_in<SURF>(p, i, p.b_pc[i], id, step, ncd, st, c0);
      }
      __syncthreads();
      persist_commit<SURF>(p, rep, cand, nc, step, ev, evcap, sh, done);
    }
  }
  acc[3] += (unsigned long long)done;
  __syncthreads();
  // ---- products (appended after the sorted molecules) and candidate reset
  const int ne = min(sh.nev, evcap);
  int uni = 0;
  for (int t = tid; t < ne; t += T) {
    place_event<SURF>(p, ev[t], step, uni, [&](float4 npc, ull nid) {
      const int k = ns + atomicAdd(&sh.np, 1);
      if (k < cap) {
        p.b_pc[off + k] = npc;
        p.b_id[off + k] = nid;
        atomicAdd((unsigned long long *)&p.spcount[rep * c_net.nsp + id_species(nid)], 1ull);
      } else {
        atomicOr(p.status, kStMolCap);
      }
    });
  }
  acc[2] += (unsigned long long)uni;
  for (int t = tid; t < nc; t += T) p.best[cand[t]] = ~0ull;
  __syncthreads();
  return min(ns + sh.np, cap);
}

// pA: inputs in buffer P, outputs in the other; pB the reverse.  Step k of
// the launch uses pA for even k.
template <int SURF>
__global__ void __launch_bounds__(kPersistThreads, SMOLB_PERSIST_BLOCKS) k_persist(KParams pA, KParams pB,
                                                                                    PersistArgs q) {
  extern __shared__ float s_gtab[];  // gaussian table, then the box tables of small replicates
  __shared__ PersistShared sh;
  __shared__ int s_rep;
  const float *gtab = stage_gtab(pA, s_gtab);
  const int gsize = (int)c_net.gmask + 1;
  int *s_cnt = reinterpret_cast<int *>(s_gtab + (gsize <= 8192 ? gsize : 0));
  int *s_st = s_cnt + kPersistSmemBoxes + 1;
  for (int k = threadIdx.x; k <= kPersistSmemBoxes; k += blockDim.x) s_cnt[k] = 0;
  const uint32_t step0 = *pA.step;
  Event *ev = q.ev + (size_t)blockIdx.x * q.evslice;
  int *cand = q.cand + (size_t)blockIdx.x * q.candslice;
  unsigned long long acc[6] = {0, 0, 0, 0, 0, 0};
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_rep = atomicAdd(q.queue, 1);
    __syncthreads();
    const int t = s_rep;
    if (t >= q.nrep) break;
    const int rep = q.order[t];
    const int off = q.roff[rep], cap = q.rcap[rep];
    int n = q.rn[rep];
    const DevGeo &g = pA.geo[rep];
    const int nb = g.n[0] * g.n[1] * g.n[2];
    const bool small = nb <= kPersistSmemBoxes;
    int *cnt = small ? s_cnt : pA.cnt + g.cell0;
    int *st = small ? s_st : pA.start + g.cell0;
    for (int k = 0; k < q.nsteps; k += 2) {
      n = persist_step<SURF>(pA, rep, off, cap, n, step0 + 1 + k, gtab, ev, q.evslice, cand, q.candslice, sh, acc,
                             cnt, st);
      if (k + 1 < q.nsteps)
        n = persist_step<SURF>(pB, rep, off, cap, n, step0 + 2 + k, gtab, ev, q.evslice, cand, q.candslice, sh,
                               acc, cnt, st);
    }
    if (threadIdx.x == 0) q.rn[rep] = n;
  }
  for (int k = 0; k < 6; ++k)
    if (acc[k]) atomicAdd(&pA.counters[k], acc[k]);
}

__global__ void k_bump_step(uint32_t *step, int by) { *step += (uint32_t)by; }

// First entry of every replicate's molecules in the box-sorted buffer
// (lo[r] = start of its first box; lo[R] = total).
__global__ void k_rep_ranges(const int *start, const DevGeo *geo, int R, int ncell, int *lo) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r <= R; r += gridDim.x * blockDim.x)
    lo[r] = (r < R) ? start[geo[r].cell0] : start[ncell];
}

// Copy replicate ranges between layouts: n[r] entries from src + soff[r] to
// dst + doff[r] (one block per replicate, grid-stride over replicates).
__global__ void k_copy_ranges(const float4 *spc, const ull *sid, const int *soff, const int *n, const int *doff,
                              int R, float4 *dpc, ull *did) {
  for (int r = blockIdx.x; r < R; r += gridDim.x) {
    const int a = soff[r], b = doff[r], m = n[r];
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      dpc[b + i] = spc[a + i];
      did[b + i] = sid[a + i];
    }
  }
}

// Upload conversion for one replicate: absolute FP64 positions to box-local
// FP32 coordinates with the packed box index, and identity words (serial
// number i+1 unless given).  A species index out of range sets kStUpload.
struct UploadGeo {
  double lo[3], h[3];
  int n[3];
  int dim;
};

__global__ void k_upload(long long n, const double *pos, const int *species, const ull *serno, UploadGeo ug,
                         int nspecies, float4 *pc, ull *id, int *status) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int sp = species[i];
    if (sp <= 0 || sp >= nspecies) {
      atomicOr(status, kStUpload);
      pc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      id[i] = make_id(kDeadSpecies, 0, 0);
      continue;
    }
    int ix[3];
    float w[3];
    for (int d = 0; d < 3; ++d) {
      if (d >= ug.dim) { ix[d] = 0; w[d] = 0.f; continue; }
      const double x = pos[3 * i + d] - ug.lo[d];
      int j = (int)floor(x / ug.h[d]);
      if (j < 0) j = 0;
      if (j > ug.n[d] - 1) j = ug.n[d] - 1;
      ix[d] = j;
      w[d] = (float)(x - j * ug.h[d]);
    }
    pc[i] = make_float4(w[0], w[1], w[2], __uint_as_float(pack_cell(ix[0], ix[1], ix[2])));
    id[i] = make_id(sp, 0, serno ? serno[i] : (ull)(i + 1));
  }
}

// Count live molecules per (rep, species) from scratch (used after uploads);
// per-block shared-memory tallies when the table is small, so that millions
// of molecules of a few species do not serialise on a handful of addresses.
__global__ void k_species_count(const ull *id, const int *n, long long *spcount, int nsp, int ntab) {
  __shared__ unsigned int s_cnt[1024];
  const bool local = ntab <= 1024;
  if (local)
    for (int k = threadIdx.x; k < ntab; k += blockDim.x) s_cnt[k] = 0;
  __syncthreads();
  const int nn = *n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    const ull x = id[i];
    const int sp = id_species(x);
    if (sp == kDeadSpecies) continue;
    const int k = id_rep(x) * nsp + sp;
    if (local) atomicAdd(&s_cnt[k], 1u);
    else atomicAdd((unsigned long long *)&spcount[k], 1ull);
  }
  __syncthreads();
  if (local)
    for (int k = threadIdx.x; k < ntab; k += blockDim.x)
      if (s_cnt[k]) atomicAdd((unsigned long long *)&spcount[k], (unsigned long long)s_cnt[k]);
}

// Mean square displacement of tracked molecules (cmdmeansqrdisp,
// smolcmd.c:2505-2606).  The reference keeps each molecule's periodic image
// offset (posoffset) and measures pos + posoffset against the value recorded
// on the first call.  Here the tracker keeps, per tracked molecule (keys
// sorted by (rep, serial)), the start and the last unwrapped position; a pass
// moves each present molecule from its last unwrapped position by its
// displacement, periodic axes taken to the nearest image.  That is exact
// while no molecule travels half a period between passes, which the host
// guarantees by spacing the passes; the step kernels carry nothing extra.
struct MsdGeo {
  double lo[3], h[3], len[3];
  int dim, periodic;  // periodic: bit d set when both walls of axis d wrap
};

constexpr int kMsdBlocks = 296, kMsdThreads = 256;

__global__ void __launch_bounds__(kMsdThreads) k_msd(const float4 *a_pc, const ull *a_id, const int *a_n,
                                                     const float4 *p_pc, const ull *p_id, const int *p_n, int pcap,
                                                     const MsdGeo *geo, int nrep, int species, const ull *keys,
                                                     long long m, const double *start, double *last, int msddim,
                                                     double *part) {
  const int na = *a_n, np = min(*p_n, pcap);
  double s2 = 0.0, s4 = 0.0, cnt = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)na + np;
       i += (long long)gridDim.x * blockDim.x) {
    const bool prod = i >= na;
    const ull x = prod ? p_id[i - na] : a_id[i];
    if (id_species(x) != species) continue;
    const int rp = id_rep(x);
    if (rp >= nrep) continue;
    const ull key = id_stream(x);
    long long lo = 0, hi = m;  // first key >= key
    while (lo < hi) {
      const long long mid = (lo + hi) >> 1;
      if (keys[mid] < key) lo = mid + 1;
      else hi = mid;
    }
    if (lo >= m || keys[lo] != key) continue;
    const float4 c = prod ? p_pc[i - na] : a_pc[i];
    const MsdGeo &g = geo[rp];
    int ix[3];
    unpack_cell(__float_as_uint(c.w), ix[0], ix[1], ix[2]);
    const float u[3] = {c.x, c.y, c.z};
    double r2 = 0.0;
    for (int d = 0; d < g.dim; ++d) {
      const double xa = g.lo[d] + ix[d] * g.h[d] + (double)u[d];
      double delta = xa - last[3 * lo + d];
      if ((g.periodic >> d) & 1) delta -= g.len[d] * rint(delta / g.len[d]);
      const double xu = last[3 * lo + d] + delta;
      last[3 * lo + d] = xu;
      const double df = xu - start[3 * lo + d];
      if (msddim < 0 || msddim == d) r2 += df * df;
    }
    s2 += r2;
    s4 += r2 * r2;
    cnt += 1.0;
  }
  __shared__ double red[3][kMsdThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    s4 += __shfl_xor_sync(0xffffffffu, s4, o);
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = s2;
    red[1][warp] = s4;
    red[2][warp] = cnt;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int w = 0; w < kMsdThreads / 32; ++w) v += red[threadIdx.x][w];
    part[3 * blockIdx.x + threadIdx.x] = v;
  }
}

// Molecules of each species inside compartment c (cmdmolcountincmpt,
// smolcmd.c:1054-1100): every live molecule of the sorted and product lists,
// membership by posincompart, per-block shared-memory tallies.
__global__ void __launch_bounds__(256) k_cmpt_count(const float4 *a_pc, const ull *a_id, const int *a_n,
                                                    const float4 *p_pc, const ull *p_id, const int *p_n, int pcap,
                                                    const DevGeo *geo, int nrep, int c, int nsp,
                                                    unsigned long long *out) {
  __shared__ unsigned int s_cnt[kMaxSpecies];
  for (int k = threadIdx.x; k < kMaxSpecies; k += blockDim.x) s_cnt[k] = 0;
  __syncthreads();
  const int na = *a_n, np = min(*p_n, pcap);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)na + np;
       i += (long long)gridDim.x * blockDim.x) {
    const bool prod = i >= na;
    const ull x = prod ? p_id[i - na] : a_id[i];
    const int sp = id_species(x);
    if (sp == kDeadSpecies || sp >= nsp) continue;
    const int rp = id_rep(x);
    if (rp >= nrep) continue;
    const float4 q = prod ? p_pc[i - na] : a_pc[i];
    int ix[3];
    unpack_cell(__float_as_uint(q.w), ix[0], ix[1], ix[2]);
    const float u[3] = {q.x, q.y, q.z};
    double xa[3];
    to_abs(geo[rp], ix, u, xa);
    if (pos_in_cmpt(c_cmpt, c, c_panels, xa)) atomicAdd(&s_cnt[sp], 1u);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nsp; k += blockDim.x)
    if (s_cnt[k]) atomicAdd(&out[k], (unsigned long long)s_cnt[k]);
}

// Batched pair-radius derivation (binding radius + reverse unbinding radius),
// one thread per replicate: the exact FP64 path for ensembles.
__global__ void k_pair_radii(long long n, const double *kf, const double *dsum, double dt, int same, int rev,
                             int rparamt, double rparam, double *bind, double *unbind, int *err) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const rxnp::PairRadii r = rxnp::pair_radii(kf[i], same, dsum[i], dt, rev, rparamt, rparam);
    bind[i] = r.bindrad;
    unbind[i] = r.unbindrad;
    err[i] = r.err;
  }
}

// Batched FP64 radius solve (one thread per problem).
__global__ void k_solve_radii(int mode, long long n, const double *rate, double dt, const double *difc,
                              const double *b, int rel, double *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (mode == 0) out[i] = rxnp::bindingradius(rate[i], dt, difc[i], b[i], rel);
    else out[i] = rxnp::unbindingradius(rate[i], dt, difc[i], b[i]);
  }
}

// Batched bindingradiusprob (rxnparam.c:587-681), one thread per problem:
// with chi[i] < 0 the reaction probability prob[i] is given and the binding
// radius is searched; with chi[i] >= 0 both are searched and prob[i] receives
// the probability found.
__global__ void k_solve_radii_prob(long long n, const double *rate, double dt, const double *difc, const double *b,
                                   int rel, const double *chi, double *prob, double *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double p = prob[i];
    out[i] = rxnp::bindingradiusprob(rate[i], dt, difc[i], b[i], rel, chi[i], &p);
    prob[i] = p;
  }
}

// ===========================================================================
// Host driver
// ===========================================================================
#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      if (err) *err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
      return -8;                                                                        \
    }                                                                                   \
  } while (0)

static int g_sm_count = 0;

static int sm_count() {
  if (!g_sm_count) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count <= 0) g_sm_count = 148;
  }
  return g_sm_count;
}

class EngineImpl {
 public:
  NetSpec net;
  std::vector<RepSpec> reps;
  DevNet dnet{};
  std::vector<DevGeo> geo;
  std::vector<DevPanel> panels;
  std::vector<DevCmpt> cmpts;
  double dt = 0;
  uint64_t seed = 0;
  long long cap = 0, pcap = 0, evcap = 0, candcap = 0;
  int ncell = 0, nscanblocks = 0;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  bool use_graph = true;
  cudaGraphExec_t graph2 = nullptr;  // two steps (even + odd parity)
  cudaGraphExec_t graph1[2] = {nullptr, nullptr};  // one step of each parity
  long long nlaunch = 0;
  long long nsteps = 0;
  int parity = 0;  // 0: A/P are inputs; 1: B/Q are inputs

  // device memory
  DevGeo *d_geo = nullptr;
  float *d_rsearch = nullptr;
  uint16_t *d_boxmask = nullptr;
  float *d_difm = nullptr;
  float *d_difstep = nullptr, *d_driftdt = nullptr, *d_bind2 = nullptr, *d_pairprob = nullptr,
        *d_prdpos = nullptr, *d_gtab = nullptr;
  uint32_t *d_unithr = nullptr;
  double *d_births = nullptr;
  float4 *d_pc[2] = {nullptr, nullptr}, *d_ppc[2] = {nullptr, nullptr};
  ull *d_id[2] = {nullptr, nullptr}, *d_pid[2] = {nullptr, nullptr};
  int *d_counts = nullptr;  // [0]=n sorted A [1]=n sorted B [2]=n prod P [3]=n prod Q [4]=nev [5]=ncand [6]=status
  uint32_t *d_step = nullptr;
  int *d_cnt = nullptr, *d_start = nullptr;
  ull *d_scan_ticket = nullptr, *d_scan_status = nullptr;
  Event *d_ev = nullptr;
  int *d_cand = nullptr;
  ull *d_best = nullptr;
  int *d_face = nullptr;
  float4 *d_tmp = nullptr;
  unsigned long long *d_counters = nullptr;
  long long *d_spcount = nullptr;
  ull *d_injkey = nullptr;
  float4 *d_injval = nullptr;
  int inj_n = 0;
  bool inj_pending = false;
  // surface-bound molecules: lists by parity (as the sorted buffers), rules
  BoundMol *d_bd[2] = {nullptr, nullptr};
  long long bcap = 0;
  ull *d_bclaim = nullptr;  // bound-solution pair reactions: claim word per sorted molecule
  int4 *d_bcand = nullptr;  // and candidate per bound molecule
  int *d_bbhead = nullptr, *d_bbnext = nullptr;  // bound-bound reactions: hash grid
  ull *d_bbcell = nullptr, *d_bbbest = nullptr;
  SrfRule *d_srfrule = nullptr;

  // persistent ensemble engine (k_persist): its own molecule layout, one
  // region per replicate; the step pipeline's buffers are refilled from it
  // (leave_persist) before anything else reads molecules
  int persist_mode = 0;       // 0: step pipeline only; 1: persistent kernel when the configuration allows
  bool in_persist = false;    // molecules currently held in the persistent layout
  int ppar = 0;               // persistent buffer holding the current state
  long long qtotal = 0;       // entries allocated in each persistent buffer
  int qcells = 0;             // box entries allocated (cells + one spare per replicate)
  float4 *d_qpc[2] = {nullptr, nullptr}, *d_qtmp = nullptr;
  ull *d_qid[2] = {nullptr, nullptr}, *d_qbest = nullptr;
  int *d_qcnt = nullptr, *d_qstart = nullptr;
  DevGeo *d_qgeo = nullptr;
  int *d_qint = nullptr;      // order[R] | off[R] | cap[R] | n[R] | queue | big
  Event *d_qev = nullptr;
  int *d_qcand = nullptr;
  int qgrid = 0, qevslice = 0, qcandslice = 0, qmaxcap = 0;
  std::vector<int> h_qoff, h_qcap, h_qn;
  cudaGraphExec_t qgraph[2] = {nullptr, nullptr};  // one launch block of qgraph_steps steps, per start parity
  int qgraph_steps = 0;

  ~EngineImpl() {
    release();
    for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
    for (int k = 0; k < 2; ++k)
      if (st_ev[k]) cudaEventDestroy(st_ev[k]);
    if (h_status) cudaFreeHost(h_status);
  }

  // status word read one call late (see Engine::status_flags_lagged)
  int *h_status = nullptr;
  cudaEvent_t st_ev[2] = {nullptr, nullptr};
  bool st_pending[2] = {false, false};
  int st_slot = 0;
  // species counts of the current state (valid while the step count and the
  // upload generation are unchanged)
  std::vector<long long> counts_cache;
  long long counts_step = -1, counts_gen = -1, upload_gen = 0;
  // Single-step graphs also copy their step's status word and species counts
  // into pinned host memory (slot = the step's parity), so that a caller
  // stepping one step at a time and reading counts after each queues no
  // separate copies between steps.
  int *h_tail_status = nullptr;        // [2]
  long long *h_tail_counts = nullptr;  // [2][tail_ntab], null when the table is large
  size_t tail_ntab = 0;
  cudaEvent_t tail_ev[2] = {nullptr, nullptr};
  int tail_slot = -1;                  // slot of the last single-step launch, -1 if the last run ended otherwise
  char *d_upload = nullptr;            // device staging of uploads (FP64 positions, species, serials)
  size_t upload_cap = 0;
  long long tail_step = -1, tail_gen = -1;
  int tail_prev_slot = -1;             // lagged status: slot of the previous call's step
  void tail_free() {  // the graphs that copy into these buffers must be gone already
    if (h_tail_status && stream) cudaStreamSynchronize(stream);  // no launched copy may still be in flight
    for (int k = 0; k < 2; ++k) {
      if (tail_ev[k]) cudaEventDestroy(tail_ev[k]);
      tail_ev[k] = nullptr;
    }
    if (h_tail_status) cudaFreeHost(h_tail_status);
    if (h_tail_counts) cudaFreeHost(h_tail_counts);
    h_tail_status = nullptr;
    h_tail_counts = nullptr;
    tail_ntab = 0;
    tail_slot = tail_prev_slot = -1;
    tail_step = tail_gen = -1;
  }
  int tail_setup() {
    if (h_tail_status) return 0;
    if (cudaMallocHost(&h_tail_status, 2 * sizeof(int)) != cudaSuccess) { h_tail_status = nullptr; return -1; }
    for (int k = 0; k < 2; ++k) cudaEventCreateWithFlags(&tail_ev[k], cudaEventDisableTiming);
    const size_t ntab = reps.size() * (size_t)net.nspecies;
    if (ntab * sizeof(long long) <= (1u << 20) &&
        cudaMallocHost(&h_tail_counts, 2 * ntab * sizeof(long long)) == cudaSuccess)
      tail_ntab = ntab;
    else
      h_tail_counts = nullptr;
    return 0;
  }
  // mean square displacement trackers (dropped with the molecules on init)
  struct MsdTrack {
    int species = 0;
    long long m = 0;
    ull *keys = nullptr;
    double *start = nullptr, *last = nullptr;
  };
  std::vector<MsdTrack> msd;
  MsdGeo *d_msdgeo = nullptr;
  double *d_msdpart = nullptr;
  void msd_free() {
    for (MsdTrack &t : msd) {
      if (t.keys) cudaFree(t.keys);
      if (t.start) cudaFree(t.start);
      if (t.last) cudaFree(t.last);
    }
    msd.clear();
    if (d_msdgeo) cudaFree(d_msdgeo);
    if (d_msdpart) cudaFree(d_msdpart);
    d_msdgeo = nullptr;
    d_msdpart = nullptr;
  }

  void persist_free() {
    for (int k = 0; k < 2; ++k) {
      if (qgraph[k]) cudaGraphExecDestroy(qgraph[k]);
      qgraph[k] = nullptr;
    }
    void *ptrs[] = {d_qpc[0], d_qpc[1], d_qtmp, d_qid[0], d_qid[1], d_qbest, d_qcnt, d_qstart, d_qgeo, d_qint,
                    d_qev, d_qcand};
    for (void *q : ptrs)
      if (q) cudaFree(q);
    d_qpc[0] = d_qpc[1] = d_qtmp = nullptr;
    d_qid[0] = d_qid[1] = d_qbest = nullptr;
    d_qcnt = d_qstart = d_qint = d_qcand = nullptr;
    d_qgeo = nullptr;
    d_qev = nullptr;
    qtotal = 0;
    qcells = 0;
    qgrid = 0;
    qmaxcap = 0;
    in_persist = false;
  }

  void release() {
    invalidate_graph();
    persist_free();
    msd_free();
    tail_free();
    if (d_upload) cudaFree(d_upload);
    d_upload = nullptr;
    upload_cap = 0;
    void *ptrs[] = {d_boxmask, d_difm, d_rsearch, d_geo, d_difstep, d_driftdt, d_bind2, d_pairprob, d_prdpos, d_gtab, d_unithr,
                    d_births, d_pc[0], d_pc[1], d_ppc[0], d_ppc[1], d_id[0], d_id[1], d_pid[0],
                    d_pid[1], d_face, d_tmp, d_counts, d_step, d_cnt, d_start, d_scan_ticket, d_scan_status, d_ev, d_cand, d_best,
                    d_counters, d_spcount, d_injkey, d_injval, d_bd[0], d_bd[1], d_srfrule, d_bclaim, d_bcand, d_bbhead, d_bbnext, d_bbcell, d_bbbest};
    for (void *q : ptrs)
      if (q) cudaFree(q);
    d_bd[0] = d_bd[1] = nullptr;
    d_bclaim = nullptr;
    d_bcand = nullptr;
    d_bbhead = d_bbnext = nullptr;
    d_bbcell = d_bbbest = nullptr;
    d_srfrule = nullptr;
    bcap = 0;
    d_rsearch = nullptr;
    d_boxmask = nullptr;
    d_geo = nullptr; d_difstep = d_driftdt = d_bind2 = d_pairprob = d_prdpos = d_gtab = nullptr;
    d_difm = nullptr;
    d_unithr = nullptr; d_births = nullptr;
    d_pc[0] = d_pc[1] = d_ppc[0] = d_ppc[1] = nullptr;
    d_id[0] = d_id[1] = d_pid[0] = d_pid[1] = nullptr;
    d_counts = nullptr; d_step = nullptr; d_cnt = d_start = nullptr; d_scan_ticket = d_scan_status = nullptr; d_ev = nullptr;
    d_cand = nullptr; d_best = nullptr; d_face = nullptr; d_tmp = nullptr; d_counters = nullptr; d_spcount = nullptr;
    d_injkey = nullptr; d_injval = nullptr;
    if (own_stream) {
      if (stream == own_stream) stream = nullptr;  // a later init creates a new one
      cudaStreamDestroy(own_stream);
    }
    own_stream = nullptr;
  }

  KParams params(int par) const {
    KParams p{};
    p.geo = d_geo;
    p.difstep = d_difstep;
    p.driftdt = d_driftdt;
    p.difm = d_difm;
    p.unithr = d_unithr;
    p.bind2 = d_bind2;
    p.pairprob = d_pairprob;
    p.rsearch = d_rsearch;
    p.boxmask = d_boxmask;
    p.births = d_births;
    p.prdpos = d_prdpos;
    p.gtab = d_gtab;
    const int in = par, out = 1 - par;
    p.a_pc = d_pc[in]; p.a_id = d_id[in]; p.a_n = d_counts + in;
    p.p_pc = d_ppc[in]; p.p_id = d_pid[in]; p.p_n = d_counts + 2 + in;
    p.b_pc = d_pc[out]; p.b_id = d_id[out]; p.b_n = d_counts + out;
    p.q_pc = d_ppc[out]; p.q_id = d_pid[out]; p.q_n = d_counts + 2 + out;
    p.tmp = d_tmp;
    p.cap = (int)cap;
    p.pcap = (int)pcap;
    p.cnt = d_cnt;
    p.start = d_start;
    p.ncell = ncell;
    p.ev = d_ev;
    p.nev = d_counts + 4;
    p.evcap = (int)evcap;
    p.cand = d_cand;
    p.ncand = d_counts + 5;
    p.candcap = (int)candcap;
    p.best = d_best;
    p.face = d_face;
    p.counters = d_counters;
    p.spcount = d_spcount;
    p.status = d_counts + 6;
    p.step = d_step;
    p.inj_key = d_injkey;
    p.inj_val = d_injval;
    p.inj_n = inj_n;
    if (dnet.bound) {
      p.srfrule = d_srfrule;
      p.bd_in = d_bd[in];
      p.bd_in_n = d_counts + 8 + in;
      p.bd_out = d_bd[out];
      p.bd_out_n = d_counts + 8 + out;
      p.bcap = (int)bcap;
      p.bclaim = d_bclaim;
      p.bcand = d_bcand;
      p.bbhead = d_bbhead;
      p.bbnext = d_bbnext;
      p.bbcell = d_bbcell;
      p.bbbest = d_bbbest;
    }
    return p;
  }

  LaunchTuning tune;  // kept across init
  int grid_mol() const { return sm_count() * tune.mol_blocks_per_sm; }
  int grid_tiles() const { return sm_count() * tune.tile_blocks_per_sm; }
  int grid_small() const { return sm_count(); }

  size_t adv_smem() const {
    const int gsize = (int)dnet.gmask + 1;
    return gsize <= 8192 ? (size_t)gsize * sizeof(float) : 0;
  }

  // per-kernel timing (profiling mode only)
  bool prof = false;
  std::vector<std::pair<const char *, cudaEvent_t>> marks;
  std::vector<cudaEvent_t> event_pool;
  size_t pool_used = 0;

  void mark(const char *name) {
    ++nlaunch;
    if (!prof) return;
    if (pool_used == event_pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      event_pool.push_back(e);
    }
    cudaEvent_t e = event_pool[pool_used++];
    cudaEventRecord(e, stream);
    marks.push_back({name, e});
  }

  // Upload of one replicate's molecules with the conversion on the device:
  // raw FP64 positions, species and optional serial numbers are copied into a
  // temporary buffer and k_upload writes the staging product buffer.
  int upload_device(long long n, const double *pos, const int *species, const uint64_t *serno, std::string *err) {
    const RepSpec &s = reps[0];
    UploadGeo ug;
    for (int d = 0; d < 3; ++d) {
      ug.lo[d] = s.lo[d];
      ug.h[d] = (s.hi[d] - s.lo[d]) / geo[0].n[d];
      ug.n[d] = geo[0].n[d];
    }
    ug.dim = s.dim;
    const size_t bpos = (size_t)n * 3 * sizeof(double), bsp = (size_t)n * sizeof(int),
                 bsn = serno ? (size_t)n * sizeof(ull) : 0;
    const size_t need = bpos + bsp + bsn + 32;
    if (need > upload_cap) {  // staging kept between uploads (grow only)
      if (d_upload) cudaFree(d_upload);
      d_upload = nullptr;
      upload_cap = 0;
      CK(cudaMalloc(&d_upload, need));
      upload_cap = need;
    }
    char *d = d_upload;
    double *dpos = reinterpret_cast<double *>(d);
    int *dsp = reinterpret_cast<int *>(d + bpos);
    ull *dsn = serno ? reinterpret_cast<ull *>(d + ((bpos + bsp + 15) & ~(size_t)15)) : nullptr;
    int zero[8] = {0};  // [8], [9]: bound-list counts, carried by finish_upload
    cudaError_t e = cudaMemcpyAsync(d_counts, zero, sizeof(zero), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dpos, pos, bpos, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dsp, species, bsp, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && serno) e = cudaMemcpyAsync(dsn, serno, bsn, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
      k_upload<<<sm_count() * 8, 256, 0, stream>>>(n, dpos, dsp, dsn, ug, net.nspecies, d_ppc[0], d_pid[0],
                                                   d_counts + 6);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
      if (err) *err = std::string("upload: ") + cudaGetErrorString(e);
      return -8;
    }
    int st = 0;
    CK(cudaMemcpy(&st, d_counts + 6, sizeof(int), cudaMemcpyDeviceToHost));
    if (st & kStUpload) { if (err) *err = "species index out of range"; return -6; }
    return finish_upload(n, err);
  }

  // Rebin the staged molecules (product buffer 0) into the sorted buffer and
  // count species.
  int finish_upload(long long n, std::string *err) {
    ++upload_gen;
    int staged = (int)n;
    if (dnet.bound && parity != 1) {  // the bound list follows the sorted buffers to parity 1
      int nb = 0;
      CK(cudaMemcpyAsync(&nb, d_counts + 8 + parity, sizeof(int), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      if (nb > 0) CK(cudaMemcpyAsync(d_bd[1], d_bd[parity], (size_t)nb * sizeof(BoundMol), cudaMemcpyDeviceToDevice, stream));
      CK(cudaMemcpyAsync(d_counts + 9, &nb, sizeof(int), cudaMemcpyHostToDevice, stream));
    }
    parity = 0;
    CK(cudaMemcpyAsync(d_counts + 2, &staged, sizeof(int), cudaMemcpyHostToDevice, stream));
    CK(cudaMemsetAsync(d_cnt, 0, ((size_t)ncell + 1) * sizeof(int), stream));
    enqueue_step(0, true);  // rebin only: P[0] -> sorted B (index 1)
    // sorted array now in buffer 1; make it the input of the next step
    parity = 1;
    CK(cudaMemsetAsync(d_counts + 2, 0, 2 * sizeof(int), stream));
    CK(cudaMemsetAsync(d_spcount, 0, reps.size() * net.nspecies * sizeof(long long), stream));
    k_species_count<<<grid_mol(), 256, 0, stream>>>(d_id[1], d_counts + 1, d_spcount, net.nspecies,
                                                    (int)reps.size() * net.nspecies);
    nlaunch++;
    if (dnet.bound) {
      k_bound_species_count<<<grid_small(), 256, 0, stream>>>(d_bd[1], d_counts + 9, d_spcount);
      nlaunch++;
    }
    CK(cudaStreamSynchronize(stream));
    CK(cudaGetLastError());
    int st = 0;
    CK(cudaMemcpy(&st, d_counts + 6, sizeof(int), cudaMemcpyDeviceToHost));
    if (st) { if (err) *err = "capacity overflow during upload"; return -9; }
    return 0;
  }

  // Launch with programmatic stream serialisation (see pdl_wait) when on.
  bool use_pdl = true;
  template <typename... Args, typename... Act>
  void launch(void (*k)(Args...), int grid, int block, size_t smem, Act &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = use_pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k, std::forward<Act>(args)...);
  }

  bool single_rep() const { return reps.size() == 1; }

  // Whether a panel can come within r of the box [lo, hi] (coordinates in
  // the panels' frame).  Conservative: false only when no point of the panel
  // lies within r of the box.
  static bool panel_near_box(const DevPanel &pn, const double lo[3], const double hi[3], double r) {
    auto dmin = [&](const double c[3]) {  // distance from c to the box
      double q = 0;
      for (int d = 0; d < 3; ++d) {
        const double v = c[d] < lo[d] ? lo[d] - c[d] : c[d] > hi[d] ? c[d] - hi[d] : 0.0;
        q += v * v;
      }
      return std::sqrt(q);
    };
    auto dmax = [&](const double c[3]) {  // distance from c to the farthest corner
      double q = 0;
      for (int d = 0; d < 3; ++d) {
        const double v = std::max(std::fabs(c[d] - lo[d]), std::fabs(c[d] - hi[d]));
        q += v * v;
      }
      return std::sqrt(q);
    };
    auto plane_apart = [&](const double o[3], const double n[3]) {  // every corner farther than r on one side
      int above = 0, below = 0;
      for (int c = 0; c < 8; ++c) {
        const double x[3] = {(c & 1) ? hi[0] : lo[0], (c & 2) ? hi[1] : lo[1], (c & 4) ? hi[2] : lo[2]};
        const double sd = (x[0] - o[0]) * n[0] + (x[1] - o[1]) * n[1] + (x[2] - o[2]) * n[2];
        if (sd > r) ++above;
        else if (sd < -r) ++below;
      }
      return above == 8 || below == 8;
    };
    if (pn.shape == 0) {  // rectangle: distance between the two boxes
      double q = 0;
      for (int d = 0; d < 3; ++d) {
        const double plo = d == pn.axis ? pn.pos : pn.lo[d], phi = d == pn.axis ? pn.pos : pn.hi[d];
        const double gap = std::max(0.0, std::max(plo - hi[d], lo[d] - phi));
        q += gap * gap;
      }
      return std::sqrt(q) <= r;
    }
    if (pn.shape == 2 || pn.shape == 4)  // the shell at the radius must meet the widened box
      return dmin(pn.center) <= pn.radius + r && dmax(pn.center) >= pn.radius - r;
    if (pn.shape == 3) {
      double c[3];
      for (int d = 0; d < 3; ++d) c[d] = 0.5 * (pn.pt[0][d] + pn.pt[1][d]);
      if (dmin(c) > std::sqrt(0.25 * pn.axlen * pn.axlen + pn.radius * pn.radius) + r) return false;
      double far = 0;  // radial distance to the axis is convex: its maximum over the box is at a corner
      for (int k = 0; k < 8; ++k) {
        const double x[3] = {(k & 1) ? hi[0] : lo[0], (k & 2) ? hi[1] : lo[1], (k & 4) ? hi[2] : lo[2]};
        double rr[3];
        cyl_radial(pn, x, rr);
        far = std::max(far, std::sqrt(dot3(rr, rr)));
      }
      return far >= pn.radius - r;
    }
    const double *o = pn.shape == 1 ? pn.pt[0] : pn.center;
    double c[3], rb = pn.radius;
    if (pn.shape == 1) {
      for (int d = 0; d < 3; ++d) c[d] = (pn.pt[0][d] + pn.pt[1][d] + pn.pt[2][d]) / 3.0;
      rb = 0;
      for (int k = 0; k < 3; ++k) {
        double q = 0;
        for (int d = 0; d < 3; ++d) q += (pn.pt[k][d] - c[d]) * (pn.pt[k][d] - c[d]);
        rb = std::max(rb, std::sqrt(q));
      }
    } else {
      for (int d = 0; d < 3; ++d) c[d] = pn.center[d];
    }
    if (dmin(c) > rb + r) return false;
    return !plane_apart(o, pn.nrm);
  }

  // Per-box panel masks for the FP32 surface screen: the panels that a move
  // no longer than mask_len, starting in the box, can come within the screen's
  // margin of.  mask_len covers 10 standard deviations per axis of the fastest
  // species' step plus its drift; longer moves screen every panel.
  int build_box_masks(std::string *err) {
    dnet.mask_len = 0;
    if (panels.empty() || panels.size() > 16 || ncell <= 0) return 0;
    double sig = 0, drift = 0, ext = 0;
    for (const RepSpec &s : reps) {
      for (int sp = 1; sp < net.nspecies; ++sp) {
        double var = 2.0 * s.difc[sp] * dt;
        if (s.has_difm[sp]) {
          double f = 0;
          for (int k = 0; k < 9; ++k) f += s.difm[sp][k] * s.difm[sp][k];
          var = 2.0 * dt * f;
        }
        sig = std::max(sig, std::sqrt(std::max(var, 0.0)));
        double v = 0;
        for (int d = 0; d < 3; ++d) v += s.drift[sp][d] * s.drift[sp][d];
        drift = std::max(drift, std::sqrt(v) * dt);
      }
      for (int d = 0; d < 3; ++d) ext = std::max(ext, s.hi[d] - s.lo[d]);
    }
    const double len = 10.0 * sig * std::sqrt(3.0) + drift;
    const double r = len + (double)dnet.surf_tol + 1e-6 * ext;
    std::vector<uint16_t> mask((size_t)ncell, 0);
    for (const DevGeo &g : geo)
      for (int iz = 0; iz < g.n[2]; ++iz)
        for (int iy = 0; iy < g.n[1]; ++iy)
          for (int ix = 0; ix < g.n[0]; ++ix) {
            const int ic[3] = {ix, iy, iz};
            double lo[3], hi[3];
            for (int d = 0; d < 3; ++d) {
              lo[d] = (double)ic[d] * g.h[d];
              hi[d] = ic[d] == g.n[d] - 1 ? (double)ic[d] * g.h[d] + g.whi[d] : lo[d] + g.h[d];
            }
            uint16_t m = 0;
            for (size_t k = 0; k < panels.size(); ++k)
              if (panel_near_box(panels[k], lo, hi, r)) m |= (uint16_t)(1u << k);
            mask[(size_t)g.cell0 + ((size_t)iz * g.n[1] + iy) * g.n[0] + ix] = m;
          }
    CK(cudaMalloc(&d_boxmask, mask.size() * sizeof(uint16_t)));
    CK(cudaMemcpy(d_boxmask, mask.data(), mask.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
    dnet.mask_len = (float)len;
    return 0;
  }
  template <bool SINGLE, int SURF>
  void enqueue_step_t(int par, bool rebin_only) {
    KParams p = params(par);
    launch(k_begin, 1, 32, 0, p, rebin_only ? 0 : 1);
    mark("k_begin");
    if (dnet.bound && !rebin_only) {
      launch(k_bound, grid_mol(), 256, 0, p);  // latency-bound FP64 work: many blocks in flight
      mark("k_bound");
    }
    launch(k_move<SINGLE, SURF>, grid_mol(), 256, rebin_only ? 0 : adv_smem(), p, rebin_only ? 1 : 0);
    mark("k_move");
    launch(k_scan_lookback, nscanblocks, kScanThreads, 0, (const int *)d_cnt, ncell, nscanblocks, d_scan_ticket,
           d_scan_status, d_start, p.b_n, (int)cap, p.status);
    mark("k_scan");
    launch(k_scatter<SINGLE>, grid_mol(), 256, 0, p);
    mark("k_scatter");
    if (rebin_only) return;
    if (tune.pair_tile == 128) launch(k_pairs_tile<SINGLE, SURF, 128>, grid_tiles(), 128, 0, p);
    else launch(k_pairs_tile<SINGLE, SURF, 256>, grid_tiles(), 256, 0, p);
    mark("k_pairs");
    launch(k_pairs_faces<SINGLE, SURF>, grid_mol(), 256, 0, p);
    mark("k_pairs_faces");
    launch(k_commit<SURF>, grid_small(), 128, 0, p);
    mark("k_commit");
    for (int round = 1; round < dnet.rounds; ++round) {
      launch(k_research<SURF>, grid_small(), 128, 0, p);
      mark("k_research");
      launch(k_commit<SURF>, grid_small(), 128, 0, p);
      mark("k_commit");
    }
    if (SURF == 3 && dnet.bpair_n) {
      for (int round = 0; round < kBPairRounds; ++round) {
        launch(k_bpair_claim, grid_mol(), 256, 0, p, round);
        mark("k_bpair_claim");
        launch(k_bpair_resolve, grid_small(), 256, 0, p);
        mark("k_bpair_resolve");
      }
    }
    if (SURF == 3 && dnet.bb_n) {
      launch(k_bb_insert, grid_small(), 256, 0, p);
      mark("k_bb_insert");
      for (int round = 0; round < kBPairRounds; ++round) {
        launch(k_bb_best, grid_mol(), 256, 0, p);
        mark("k_bb_best");
        launch(k_bb_resolve, grid_small(), 256, 0, p);
        mark("k_bb_resolve");
      }
      launch(k_bb_clear, grid_small(), 256, 0, p);
      mark("k_bb_clear");
    }
    launch(k_products<SURF>, grid_small(), 128, 0, p);
    mark("k_products");
  }


  // Enqueue one step with the given parity (inputs A/P = buffers `par`).
  void enqueue_step(int par, bool rebin_only) {
    // surface form: 0 none, 1 rect and sphere panels only, 2 any shape,
    // jumps or compartments (whose tests need panels to mean anything), 3 as
    // 2 with surface-bound states
    int surf = dnet.npanel > 0 ? 1 : 0;
    for (const DevPanel &pn : panels)
      if ((pn.shape != 0 && pn.shape != 2) || pn.jp_front || pn.jp_back) surf = 2;  // jumps: the general form
    if (surf && (dnet.ncmpt > 0 || dnet.bound)) surf = 2;
    if (dnet.bound) surf = 3;  // 3: any shape plus surface-bound states (single simulations)
    if (single_rep()) {
      if (surf == 0) enqueue_step_t<true, 0>(par, rebin_only);
      else if (surf == 1) enqueue_step_t<true, 1>(par, rebin_only);
      else if (surf == 2) enqueue_step_t<true, 2>(par, rebin_only);
      else enqueue_step_t<true, 3>(par, rebin_only);
    } else {
      if (surf == 0) enqueue_step_t<false, 0>(par, rebin_only);
      else if (surf == 1) enqueue_step_t<false, 1>(par, rebin_only);
      else enqueue_step_t<false, 2>(par, rebin_only);
    }
  }

  int launches_per_step() const {
    return 8 + 2 * (dnet.rounds - 1) + (dnet.bound ? 1 : 0) + (dnet.bound && dnet.bpair_n ? 2 * kBPairRounds : 0) +
           (dnet.bound && dnet.bb_n ? 2 + 2 * kBPairRounds : 0);
  }

  int upload_const(std::string *err) {
    CK(cudaMemcpyToSymbolAsync(c_net, &dnet, sizeof(DevNet), 0, cudaMemcpyHostToDevice, stream));
    if (!geo.empty())
      CK(cudaMemcpyToSymbolAsync(c_geo0, geo.data(), sizeof(DevGeo), 0, cudaMemcpyHostToDevice, stream));
    if (!panels.empty())
      CK(cudaMemcpyToSymbolAsync(c_panels, panels.data(), panels.size() * sizeof(DevPanel), 0,
                                 cudaMemcpyHostToDevice, stream));
    if (!cmpts.empty())
      CK(cudaMemcpyToSymbolAsync(c_cmpt, cmpts.data(), cmpts.size() * sizeof(DevCmpt), 0,
                                 cudaMemcpyHostToDevice, stream));
    return 0;
  }

  int build_rep_tables(std::string *err) {
    const int R = (int)reps.size(), nsp = net.nspecies;
    std::vector<float> difstep((size_t)R * nsp), driftdt((size_t)R * nsp * 3), difm((size_t)R * nsp * 9, 0.f);
    uint32_t difm_any = 0;
    std::vector<uint32_t> unithr((size_t)R * nsp * kMaxUniPerSpecies, 0);
    const int nr2 = std::max(1, net.nrxn[2]), nr0 = std::max(1, net.nrxn[0]);
    std::vector<float> bind2((size_t)R * nr2, 0.f), pairprob((size_t)R * nr2, 1.f);
    std::vector<float> rsearch((size_t)R * nsp, 0.f);
    float bpair_rmax = 0.f, bb_rmax = 0.f;
    std::vector<double> births((size_t)R * nr0, 0.0);
    const int nrx = std::max(1, dnet.nrx_total);
    std::vector<float> prdpos((size_t)R * nrx * kMaxProd * 3, 0.f);
    bool any_drift = false;
    for (int rp = 0; rp < R; ++rp) {
      const RepSpec &s = reps[rp];
      for (int sp = 0; sp < nsp; ++sp) {
        difstep[(size_t)rp * nsp + sp] = (float)std::sqrt(2.0 * s.difc[sp] * dt);
        if (s.has_difm[sp]) {  // anisotropic: step = M * sqrt(2 dt) * g (smolmolec.c:3158-3162)
          difm_any |= 1u << sp;
          for (int k = 0; k < 9; ++k)
            difm[((size_t)rp * nsp + sp) * 9 + k] = (float)(s.difm[sp][k] * std::sqrt(2.0 * dt));
        }
        for (int d = 0; d < 3; ++d) {
          driftdt[((size_t)rp * nsp + sp) * 3 + d] = (float)(s.drift[sp][d] * dt);
          if (s.drift[sp][d] != 0) any_drift = true;
        }
        // cumulative thresholds: reaction k of the species fires with probability
        // prob_k * prod_{m<k}(1-prob_m) (sequential coins of smolreact.c:3036-3055)
        double surv = 1.0, cum = 0.0;
        for (int m = 0; m < dnet.uni_n[sp]; ++m) {
          const int r = dnet.uni_list[sp][m];
          const double pr = std::min(1.0, std::max(0.0, s.uni_prob[r]));
          cum += pr * surv;
          surv *= (1.0 - pr);
          const double t = std::min(4294967295.0, std::floor(cum * 4294967296.0));
          unithr[((size_t)rp * nsp + sp) * kMaxUniPerSpecies + m] = (uint32_t)t;
        }
        if (rp == 0)  // the same thresholds for the bound states' reactions (single simulations)
          for (int st = 0; st < 2; ++st) {
            double bsurv = 1.0, bcum = 0.0;
            for (int m = 0; m < dnet.buni_n[sp][st]; ++m) {
              const double pr = std::min(1.0, std::max(0.0, s.uni_prob[dnet.buni_list[sp][st][m]]));
              bcum += pr * bsurv;
              bsurv *= (1.0 - pr);
              dnet.bthr[sp][st][m] = (uint32_t)std::min(4294967295.0, std::floor(bcum * 4294967296.0));
            }
          }
      }
      for (int r = 0; r < net.nrxn[2]; ++r) {
        bind2[(size_t)rp * nr2 + r] = (float)s.bind2[r];
        pairprob[(size_t)rp * nr2 + r] = (float)s.pair_prob[r];
        if (net.rstate2[r][0] != 0 || net.rstate2[r][1] != 0) {  // searched from the bound list
          const double hmin0 = std::min(geo[rp].h[0], std::min(geo[rp].h[1], geo[rp].h[2]));
          const double rb = std::sqrt(std::max(0.0, s.bind2[r])) * (1.0 + 1e-4) + 1e-6 * hmin0;
          if (rp == 0) {
            if (net.rstate2[r][0] != 0 && net.rstate2[r][1] != 0) bb_rmax = std::max(bb_rmax, (float)rb);
            else bpair_rmax = std::max(bpair_rmax, (float)rb);
          }
          continue;
        }
        // stencil radius: largest binding radius of the species' pair reactions,
        // padded so FP32 rounding of a distance at the radius cannot fall outside
        const double hmin = std::min(geo[rp].h[0], std::min(geo[rp].h[1], geo[rp].h[2]));
        const double rr = std::sqrt(std::max(0.0, s.bind2[r])) * (1.0 + 1e-4) + 1e-6 * hmin;
        for (int k = 0; k < 2; ++k) {
          float &v = rsearch[(size_t)rp * nsp + net.rct[2][r][k]];
          v = std::max(v, (float)rr);
        }
      }
      for (int r = 0; r < net.nrxn[0]; ++r) births[(size_t)rp * nr0 + r] = s.birth_mean[r];
      for (int o = 0; o < 3; ++o)
        for (int r = 0; r < net.nrxn[o]; ++r)
          for (int q = 0; q < kMaxProd; ++q)
            for (int d = 0; d < 3; ++d)
              prdpos[(((size_t)rp * nrx + dnet.rxn_base[o] + r) * kMaxProd + q) * 3 + d] =
                  (float)s.prdpos[o][r][q][d];
    }
    dnet.any_drift = any_drift ? 1 : 0;
    dnet.difm_any = difm_any;
    dnet.bpair_rmax = bpair_rmax;
    dnet.bb_rmax = bb_rmax;
    dnet.bb_inv_cs = bb_rmax > 0 ? 1.0 / (double)bb_rmax : 1.0;
    auto put = [&](void **dst, const void *src, size_t bytes) -> int {
      if (!*dst) CK(cudaMalloc(dst, bytes));
      CK(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, stream));
      return 0;
    };
    if (put((void **)&d_difstep, difstep.data(), difstep.size() * 4)) return -8;
    if (put((void **)&d_difm, difm.data(), difm.size() * 4)) return -8;
    if (put((void **)&d_driftdt, driftdt.data(), driftdt.size() * 4)) return -8;
    if (put((void **)&d_unithr, unithr.data(), unithr.size() * 4)) return -8;
    if (put((void **)&d_bind2, bind2.data(), bind2.size() * 4)) return -8;
    if (put((void **)&d_rsearch, rsearch.data(), rsearch.size() * 4)) return -8;
    if (put((void **)&d_pairprob, pairprob.data(), pairprob.size() * 4)) return -8;
    if (put((void **)&d_births, births.data(), births.size() * 8)) return -8;
    if (put((void **)&d_prdpos, prdpos.data(), prdpos.size() * 4)) return -8;
    // the host copies are staged; wait before the vectors go out of scope
    CK(cudaStreamSynchronize(stream));
    return upload_const(err);
  }

  void invalidate_graph() {
    if (graph2) cudaGraphExecDestroy(graph2);
    graph2 = nullptr;
    for (int k = 0; k < 2; ++k) {
      if (graph1[k]) cudaGraphExecDestroy(graph1[k]);
      graph1[k] = nullptr;
    }
  }

  // Capture the steps of parities first..last (one or two steps), `reps`
  // times over, into *out.
  int capture_steps(int first, int last, cudaGraphExec_t *out, std::string *err, int reps = 1) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    const long long before = nlaunch;
    const bool was = prof;
    prof = false;
    for (int k = 0; k < reps; ++k)
      for (int par = first; par <= last; ++par) enqueue_step(par, false);
    if (first == last && h_tail_status) {
      cudaMemcpyAsync(h_tail_status + first, d_counts + 6, sizeof(int), cudaMemcpyDeviceToHost, stream);
      if (h_tail_counts)
        cudaMemcpyAsync(h_tail_counts + (size_t)first * tail_ntab, d_spcount, tail_ntab * sizeof(long long),
                        cudaMemcpyDeviceToHost, stream);
    }
    prof = was;
    nlaunch = before;
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    if (e == cudaSuccess) {
      e = cudaGraphInstantiate(out, g, 0);
      cudaGraphDestroy(g);
    }
    if (e != cudaSuccess) {
      *out = nullptr;
      if (use_pdl) {  // capture without programmatic edges instead
        cudaGetLastError();
        invalidate_graph();
        use_pdl = false;
        return capture_steps(first, last, out, err, reps);
      }
      if (err) *err = std::string("step graph: ") + cudaGetErrorString(e);
      return -8;
    }
    return 0;
  }

  int build_graph(std::string *err) {
    if (graph2) cudaGraphExecDestroy(graph2);
    graph2 = nullptr;
    return capture_steps(0, 1, &graph2, err);
  }


  size_t persist_smem() const { return adv_smem() + 2 * (kPersistSmemBoxes + 1) * sizeof(int); }

  // The persistent kernel covers ensembles without surfaces, compartments or
  // injected displacements (the general surface form stays on the pipeline).
  bool persist_eligible() const {
    return persist_mode != 0 && dnet.npanel == 0 && dnet.ncmpt == 0 && !dnet.inject && msd.empty();
  }

  // Persistent-kernel params: a = buffer `in`, b = the other.
  KParams persist_params(int in) const {
    KParams p = params(0);
    p.geo = d_qgeo;
    p.a_pc = d_qpc[in];
    p.a_id = d_qid[in];
    p.b_pc = d_qpc[1 - in];
    p.b_id = d_qid[1 - in];
    p.b_n = d_qint + 4 * reps.size() + 1;  // a large count: box starts bound the searches
    p.tmp = d_qtmp;
    p.cnt = d_qcnt;
    p.start = d_qstart;
    p.best = d_qbest;
    return p;
  }

  // Move the state into the persistent layout: one rebin pass merges the
  // pending products and sorts every replicate into a contiguous range, then
  // each range is copied into its replicate's region (regions hold twice the
  // replicate's molecules plus 256, processing order largest first).
  // Room for zeroth-order births over one launch (100 steps): twice the
  // expected count plus 64.
  long long birth_headroom(int r) const {
    double m = 0;
    for (int k = 0; k < net.nrxn[0]; ++k) m += reps[r].birth_mean[k];
    return m > 0 ? (long long)std::ceil(2.0 * m * 100.0) + 64 : 0;
  }
  // Whether any reaction makes more molecules than it consumes.
  bool can_grow() const {
    if (net.nrxn[0] > 0) return true;
    for (int o = 1; o < 3; ++o)
      for (int r = 0; r < net.nrxn[o]; ++r)
        if (net.nprod[o][r] > o) return true;
    return false;
  }

  int enter_persist(std::string *err, const std::vector<long long> *extra = nullptr) {
    const int R = (int)reps.size();
    CK(cudaMemsetAsync(d_cnt, 0, ((size_t)ncell + 1) * sizeof(int), stream));
    enqueue_step(parity, true);
    parity ^= 1;
    int *d_lo = nullptr;
    CK(cudaMalloc(&d_lo, (size_t)(R + 1) * sizeof(int)));
    k_rep_ranges<<<(R + 256) / 256, 256, 0, stream>>>(d_start, d_geo, R, ncell, d_lo);
    std::vector<int> lo((size_t)R + 1);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(lo.data(), d_lo, lo.size() * sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
      cudaFree(d_lo);
      if (err) *err = std::string("persistent layout: ") + cudaGetErrorString(e);
      return -8;
    }
    std::vector<int> n((size_t)R), order((size_t)R);
    h_qoff.assign(R, 0);
    h_qcap.assign(R, 0);
    long long total = 0;
    int maxcap = 0;
    for (int r = 0; r < R; ++r) {
      n[r] = lo[r + 1] - lo[r];
      const long long c = 2ll * n[r] + 256 + std::max(birth_headroom(r), extra ? (*extra)[r] : 0ll);
      h_qoff[r] = (int)total;
      h_qcap[r] = (int)c;
      total += c;
      maxcap = std::max(maxcap, (int)c);
    }
    if (total > (1ll << 31) - 2) { cudaFree(d_lo); if (err) *err = "persistent layout too large"; return -9; }
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[a] > n[b]; });
    // buffers (grow only)
    const int cells = ncell + R + 1;
    if (total > qtotal || cells > qcells || maxcap > qmaxcap || !d_qgeo) {
      persist_free();
      for (int k = 0; k < 2; ++k) {
        CK(cudaMalloc(&d_qpc[k], (size_t)total * sizeof(float4)));
        CK(cudaMalloc(&d_qid[k], (size_t)total * sizeof(ull)));
      }
      CK(cudaMalloc(&d_qtmp, (size_t)total * sizeof(float4)));
      CK(cudaMalloc(&d_qbest, (size_t)total * sizeof(ull)));
      CK(cudaMemsetAsync(d_qbest, 0xFF, (size_t)total * sizeof(ull), stream));
      CK(cudaMalloc(&d_qcnt, (size_t)cells * sizeof(int)));
      CK(cudaMalloc(&d_qstart, (size_t)cells * sizeof(int)));
      CK(cudaMalloc(&d_qgeo, (size_t)R * sizeof(DevGeo)));
      CK(cudaMalloc(&d_qint, (4 * (size_t)R + 2) * sizeof(int)));
      qtotal = total;
      qcells = cells;
      qmaxcap = maxcap;
      // CTAs: as many as stay resident (one wave), at most one per replicate
      int per_sm = 0;
      CK(cudaFuncSetAttribute(k_persist<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)persist_smem()));
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persist<0>, kPersistThreads, persist_smem());
      qgrid = std::max(1, std::min(R, sm_count() * std::max(1, per_sm)));
      qevslice = std::max(1024, maxcap / 8);
      qcandslice = std::max(1024, maxcap / 4);
      CK(cudaMalloc(&d_qev, (size_t)qgrid * qevslice * sizeof(Event)));
      CK(cudaMalloc(&d_qcand, (size_t)qgrid * qcandslice * sizeof(int)));
    }
    CK(cudaMemsetAsync(d_qcnt, 0, (size_t)qcells * sizeof(int), stream));
    std::vector<DevGeo> g2 = geo;
    for (int r = 0; r < R; ++r) g2[r].cell0 += r;  // one spare box entry per replicate
    std::vector<int> ints(4 * (size_t)R + 2);
    for (int r = 0; r < R; ++r) {
      ints[r] = order[r];
      ints[R + r] = h_qoff[r];
      ints[2 * R + r] = h_qcap[r];
      ints[3 * R + r] = n[r];
    }
    ints[4 * R] = 0;
    ints[4 * R + 1] = 0x7FFFFFFF;
    CK(cudaMemcpyAsync(d_qgeo, g2.data(), g2.size() * sizeof(DevGeo), cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(d_qint, ints.data(), ints.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    k_copy_ranges<<<std::min(R, sm_count() * 8), 256, 0, stream>>>(d_pc[parity], d_id[parity], d_lo, d_qint + 3 * R,
                                                                   d_qint + R, R, d_qpc[0], d_qid[0]);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d_lo);
    if (e != cudaSuccess) { if (err) *err = std::string("persistent layout: ") + cudaGetErrorString(e); return -8; }
    nlaunch += 2;
    ppar = 0;
    in_persist = true;
    h_qn = n;
    return 0;
  }

  // After a launch: the replicates' entry counts and the status word.  A
  // replicate whose free room is below three times its growth in the last
  // launch (or its birth headroom) gets a new layout with more room before
  // the next launch; a capacity overflow is an error.
  int persist_check(bool relayout, std::string *err) {
    const int R = (int)reps.size();
    std::vector<int> n((size_t)R);
    int st = 0;
    CK(cudaMemcpyAsync(n.data(), d_qint + 3 * R, (size_t)R * sizeof(int), cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(&st, d_counts + 6, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    if (st & (kStMolCap | kStEvCap | kStCandCap)) {
      if (err)
        *err = std::string("persistent kernel: ") +
               ((st & kStMolCap) ? "replicate region" : (st & kStEvCap) ? "event list" : "candidate list") +
               " overflow";
      return -9;
    }
    if (!relayout) { h_qn = n; return 0; }
    bool need = false;
    std::vector<long long> extra((size_t)R, 0);
    for (int r = 0; r < R; ++r) {
      const long long grow = std::max(0, n[r] - (r < (int)h_qn.size() ? h_qn[r] : n[r]));
      extra[r] = 3 * grow + birth_headroom(r);
      if ((long long)h_qcap[r] - n[r] < std::max(256ll, extra[r])) need = true;
    }
    h_qn = n;
    if (!need) return 0;
    int rc = leave_persist(err);
    if (!rc) rc = enter_persist(err, &extra);
    return rc;
  }

  // Back to the step pipeline's layout: every replicate's entries are
  // gathered into the staging buffer and rebinned (dead entries drop out).
  int leave_persist(std::string *err) {
    if (!in_persist) return 0;
    const int R = (int)reps.size();
    std::vector<int> n((size_t)R);
    CK(cudaMemcpyAsync(n.data(), d_qint + 3 * R, (size_t)R * sizeof(int), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    std::vector<int> soff((size_t)R);
    long long total = 0;
    for (int r = 0; r < R; ++r) {
      soff[r] = (int)total;
      total += n[r];
    }
    if (total > cap) { if (err) *err = "more molecules than the engine capacity"; return -9; }
    if (total > pcap) {  // the staging (product) buffers take the gathered molecules
      for (int k = 0; k < 2; ++k) {
        cudaFree(d_ppc[k]);
        cudaFree(d_pid[k]);
        d_ppc[k] = nullptr;
        d_pid[k] = nullptr;
      }
      pcap = total;
      for (int k = 0; k < 2; ++k) {
        CK(cudaMalloc(&d_ppc[k], pcap * sizeof(float4)));
        CK(cudaMalloc(&d_pid[k], pcap * sizeof(ull)));
      }
      cudaFree(d_tmp);
      d_tmp = nullptr;
      CK(cudaMalloc(&d_tmp, (cap + pcap) * sizeof(float4)));
      invalidate_graph();
    }
    int *d_soff = nullptr;
    CK(cudaMalloc(&d_soff, (size_t)R * sizeof(int)));
    CK(cudaMemcpyAsync(d_soff, soff.data(), soff.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    k_copy_ranges<<<std::min(R, sm_count() * 8), 256, 0, stream>>>(d_qpc[ppar], d_qid[ppar], d_qint + R,
                                                                   d_qint + 3 * R, d_soff, R, d_ppc[0], d_pid[0]);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d_soff);
    if (e != cudaSuccess) { if (err) *err = std::string("persistent layout: ") + cudaGetErrorString(e); return -8; }
    ++nlaunch;
    in_persist = false;
    // the sorted and product counts of the pipeline's buffers are stale
    CK(cudaMemsetAsync(d_counts, 0, 4 * sizeof(int), stream));
    // finish_upload recounts species from scratch, which equals the kept counts
    const long long keep_gen = upload_gen;
    const int rc = finish_upload(total, err);
    upload_gen = keep_gen;
    return rc;
  }

  // nsteps steps of every replicate through k_persist, in launches of at
  // most 100 steps; each launch (work-counter reset, kernel, step-counter
  // bump) is one replay of a captured graph.
  int run_persist(long long nsteps, std::string *err) {
    if (!in_persist) {
      int rc = enter_persist(err);
      if (rc) return rc;
    }
    const int R = (int)reps.size();
    const bool grow = can_grow();
    long long left = nsteps;
    while (left > 0) {
      const int K = (int)std::min<long long>(left, 100);
      auto enqueue = [&](int in) {
        PersistArgs q;
        q.order = d_qint;
        q.roff = d_qint + R;
        q.rcap = d_qint + 2 * R;
        q.rn = d_qint + 3 * R;
        q.queue = d_qint + 4 * R;
        q.ev = d_qev;
        q.evslice = qevslice;
        q.cand = d_qcand;
        q.candslice = qcandslice;
        q.nrep = R;
        q.nsteps = K;
        cudaMemsetAsync(q.queue, 0, sizeof(int), stream);
        k_persist<0><<<qgrid, kPersistThreads, persist_smem(), stream>>>(persist_params(in), persist_params(1 - in),
                                                                         q);
        k_bump_step<<<1, 1, 0, stream>>>(d_step, K);
      };
      if (use_graph) {
        if (K != qgraph_steps) {
          for (int k = 0; k < 2; ++k) {
            if (qgraph[k]) cudaGraphExecDestroy(qgraph[k]);
            qgraph[k] = nullptr;
          }
          qgraph_steps = K;
        }
        if (!qgraph[ppar]) {
          cudaGraph_t g = nullptr;
          CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
          enqueue(ppar);
          CK(cudaStreamEndCapture(stream, &g));
          cudaError_t e = cudaGraphInstantiate(&qgraph[ppar], g, 0);
          cudaGraphDestroy(g);
          if (e != cudaSuccess) { qgraph[ppar] = nullptr; if (err) *err = std::string("persistent graph: ") + cudaGetErrorString(e); return -8; }
        }
        CK(cudaGraphLaunch(qgraph[ppar], stream));
      } else {
        enqueue(ppar);
      }
      nlaunch += 2;
      ppar ^= (K & 1);
      left -= K;
      if (grow) {
        int rc = persist_check(true, err);
        if (rc) return rc;
      }
    }
    CK(cudaGetLastError());
    if (!grow) return persist_check(false, err);
    return 0;
  }

  // One step of the current parity through its single-step graph.
  int run_one(std::string *err) {
    if (!graph1[parity]) {
      if (!h_tail_status && tail_setup() == 0) invalidate_graph();  // capture with the copies from now on
      int rc = capture_steps(parity, parity, &graph1[parity], err);
      if (rc) return rc;
    }
    CK(cudaGraphLaunch(graph1[parity], stream));
    nlaunch += launches_per_step();
    if (h_tail_status) {
      CK(cudaEventRecord(tail_ev[parity], stream));
      tail_slot = parity;
    }
    parity ^= 1;
    return 0;
  }
};

Engine::Engine() : impl_(new EngineImpl) {}
Engine::~Engine() { delete impl_; }

static float f_of(double x) { return (float)x; }

int Engine::init(const NetSpec &net, const std::vector<RepSpec> &reps, double dt, uint64_t seed,
                 long long capacity, std::string *err) {
  EngineImpl &E = *impl_;
  E.release();
  E.net = net;
  E.reps = reps;
  E.dt = dt;
  E.seed = seed;
  if (reps.empty() || reps.size() > 65536) { if (err) *err = "replicate count must be 1..65536"; return -6; }
  if (net.nspecies > kMaxSpecies) { if (err) *err = "too many species for the GPU engine (max 31)"; return -6; }
  for (int o = 0; o < 3; ++o)
    if (net.nrxn[o] > kMaxRxn) { if (err) *err = "too many reactions of one order (max 16)"; return -6; }
  int gs = net.gauss_table_size;
  if (gs < 2 || gs > 65536 || (gs & (gs - 1))) { if (err) *err = "gauss table size must be a power of 2 <= 65536"; return -6; }
  if (!E.own_stream) CK(cudaStreamCreateWithFlags(&E.own_stream, cudaStreamNonBlocking));
  if (!E.stream) E.stream = E.own_stream;

  // ---- network constants
  DevNet &D = E.dnet;
  memset(&D, 0, sizeof(D));
  D.nsp = net.nspecies;
  D.nrep = (int)reps.size();
  for (int o = 0; o < 3; ++o) D.nr[o] = net.nrxn[o];
  D.rxn_base[0] = 0;
  D.rxn_base[1] = net.nrxn[0];
  D.rxn_base[2] = net.nrxn[0] + net.nrxn[1];
  D.nrx_total = net.nrxn[0] + net.nrxn[1] + net.nrxn[2];
  D.gmask = (uint32_t)(gs - 1);
  D.key0 = (uint32_t)seed ^ 0xA511E9B3u;
  D.key1 = (uint32_t)(seed >> 32) ^ 0x63D83595u;
  for (int r = 0; r < 10; ++r) {  // Philox round keys (bumped by the Weyl constants)
    D.move_ks[2 * r] = D.key0 + (uint32_t)r * 0x9E3779B9u;
    D.move_ks[2 * r + 1] = D.key1 + (uint32_t)r * 0xBB67AE85u;
  }
  D.rounds = 3;
  D.npanel = (int)net.panels.size();
  D.surf_eps = 0;
  for (int r = 0; r < net.nrxn[1]; ++r) {
    const int sp = net.rct[1][r][0];
    D.rct[1][r][0] = (uint8_t)sp;
    for (int q = 0; q < 2; ++q) D.pstate1[r][q] = (uint8_t)net.pstate1[r][q];
    const int st = net.rstate1[r];
    if (st == 1 || st == 2) {  // a surface-bound reactant: the bound list's own table
      uint8_t &nb = D.buni_n[sp][st - 1];
      if (nb >= kMaxUniPerSpecies) { if (err) *err = "too many first-order reactions for one species"; return -6; }
      D.buni_list[sp][st - 1][nb++] = (uint8_t)r;
      continue;
    }
    if (D.uni_n[sp] >= kMaxUniPerSpecies) { if (err) *err = "too many first-order reactions for one species"; return -6; }
    D.uni_list[sp][D.uni_n[sp]++] = (uint8_t)r;
    D.uni_any |= 1u << sp;
  }
  for (int r = 0; r < net.nrxn[2]; ++r) {
    const int a = net.rct[2][r][0], b = net.rct[2][r][1];
    D.rct[2][r][0] = (uint8_t)a;
    D.rct[2][r][1] = (uint8_t)b;
    const int sa = net.rstate2[r][0], sb = net.rstate2[r][1];
    if (sa != 0 && sb != 0) {  // two bound reactants: the bound list's own pair pass
      if (!net.bound) { if (err) *err = "reactions of surface-bound molecules need surface rules with bound states"; return -6; }
      const int k = D.bb_n++;
      D.bb_rxn[k] = (uint8_t)r;
      D.bb_sp[k][0] = (uint8_t)a;
      D.bb_sp[k][1] = (uint8_t)b;
      D.bb_st[k][0] = (uint8_t)sa;
      D.bb_st[k][1] = (uint8_t)sb;
      D.bb_pst[k] = (uint8_t)net.pstate2[r];
      D.bb_mask[a][sa - 1] |= 1u << b;
      D.bb_mask[b][sb - 1] |= 1u << a;
      continue;
    }
    if (sa != 0 || sb != 0) {  // one bound reactant: the bound list's pair pass
      if (!net.bound) { if (err) *err = "reactions of surface-bound molecules need surface rules with bound states"; return -6; }
      const int k = D.bpair_n++;
      const bool first = sa != 0;
      D.bpair_rxn[k] = (uint8_t)r;
      D.bpair_bsp[k] = (uint8_t)(first ? a : b);
      D.bpair_bst[k] = (uint8_t)(first ? sa : sb);
      D.bpair_ssp[k] = (uint8_t)(first ? b : a);
      D.bpair_pst[k] = (uint8_t)net.pstate2[r];
      D.bpair_mask[D.bpair_bsp[k]][D.bpair_bst[k] - 1] |= 1u << D.bpair_ssp[k];
      continue;
    }
    for (int pass = 0; pass < (a == b ? 1 : 2); ++pass) {
      const int x = pass ? b : a, y = pass ? a : b;
      if (D.pair_n[x][y] >= kMaxPairRxn) { if (err) *err = "too many reactions for one reactant pair"; return -6; }
      D.pair_list[x][y][D.pair_n[x][y]++] = (uint8_t)r;
      D.pair_mask[x] |= 1u << y;
      D.pair_any |= 1u << x;
      if (x <= y) D.search_mask[x] |= 1u << y;  // the lower species index searches
    }
  }
  for (int o = 0; o < 3; ++o)
    for (int r = 0; r < net.nrxn[o]; ++r) {
      D.nprod[o][r] = (uint8_t)net.nprod[o][r];
      D.fixed[o][r] = (uint8_t)net.fixed_placement[o][r];
      if (o == 2) {
        D.placement2[r] = (uint8_t)net.placement2[r];
        D.bounce_k[r] = (float)net.bounce_k[r];
      }
      for (int q = 0; q < net.nprod[o][r]; ++q) D.prd[o][r][q] = (uint8_t)net.prd[o][r][q];
      bool off = false;
      for (const RepSpec &s : reps)
        for (int q = 0; q < net.nprod[o][r]; ++q)
          for (int d = 0; d < 3; ++d)
            if (s.prdpos[o][r][q][d] != 0) off = true;
      D.has_offset[o][r] = off ? 1 : 0;
    }

  // ---- replicate geometry
  E.geo.resize(reps.size());
  long long cells = 0;
  bool any_absorb = false;
  for (size_t k = 0; k < reps.size(); ++k) {
    const RepSpec &s = reps[k];
    DevGeo &g = E.geo[k];
    memset(&g, 0, sizeof(g));
    g.dim = s.dim;
    for (int d = 0; d < 3; ++d) {
      int n = std::max(1, s.ncell[d]);
      const double L = s.hi[d] - s.lo[d];
      if (d < s.dim && (s.wall[2 * d] == kWallPeriodic || s.wall[2 * d + 1] == kWallPeriodic) && n < 3) n = 3;
      if (n > 1023) n = 1023;
      const double h = (d < s.dim) ? L / n : 1.0;
      g.n[d] = n;
      g.h[d] = f_of(h);
      g.inv_h[d] = 1.0f / g.h[d];
      g.whi[d] = (d < s.dim) ? f_of(L - (n - 1) * h) : f_of(h);
      g.wall[2 * d] = (d < s.dim) ? s.wall[2 * d] : kWallTransparent;
      g.wall[2 * d + 1] = (d < s.dim) ? s.wall[2 * d + 1] : kWallTransparent;
      if (g.wall[2 * d] == kWallAbsorb || g.wall[2 * d + 1] == kWallAbsorb) any_absorb = true;
    }
    g.vol = (float)((s.hi[0] - s.lo[0]) * (s.dim > 1 ? s.hi[1] - s.lo[1] : 1) * (s.dim > 2 ? s.hi[2] - s.lo[2] : 1));
    g.cell0 = (int)cells;
    cells += (long long)g.n[0] * g.n[1] * g.n[2];
    if (cells > (1ll << 30)) { if (err) *err = "too many virtual boxes"; return -6; }
  }
  D.any_absorb = any_absorb ? 1 : 0;
  E.ncell = (int)cells;
  E.nscanblocks = (E.ncell + kScanTile - 1) / kScanTile;
  {
    // molecules are kept this far from panels after a surface interaction, so
    // that rounding to FP32 box-local coordinates cannot move them across
    float hmin = 1e30f;
    for (const DevGeo &g : E.geo)
      for (int d = 0; d < 3; ++d) hmin = std::min(hmin, g.h[d]);
    D.surf_eps = 1e-5 * (double)hmin;
    // FP32 screening before the FP64 surface walk: absolute positions up to the
    // largest extent carry about 2^-24 relative error; 64 ulp of margin plus eps
    double lmax = 0;
    for (const DevGeo &g : E.geo)
      for (int d = 0; d < 3; ++d) lmax = std::max(lmax, (double)g.n[d] * g.h[d] + g.whi[d]);
    D.surf_tol = (float)(D.surf_eps + 64.0 * lmax / 16777216.0);
  }

  // ---- capacities
  E.cap = std::max<long long>(capacity, 1024);
  E.pcap = std::max<long long>(E.cap / 4, 65536);
  E.evcap = std::max<long long>(E.cap / 8, 32768);
  E.candcap = std::max<long long>(E.cap / 8, 32768);
  if (E.cap > (1ll << 31) - 2) { if (err) *err = "molecule capacity too large"; return -6; }

  CK(cudaMalloc(&E.d_geo, E.geo.size() * sizeof(DevGeo)));
  CK(cudaMemcpyAsync(E.d_geo, E.geo.data(), E.geo.size() * sizeof(DevGeo), cudaMemcpyHostToDevice, E.stream));
  for (int k = 0; k < 2; ++k) {
    CK(cudaMalloc(&E.d_pc[k], E.cap * sizeof(float4)));
    CK(cudaMalloc(&E.d_id[k], E.cap * sizeof(ull)));
    CK(cudaMalloc(&E.d_ppc[k], E.pcap * sizeof(float4)));
    CK(cudaMalloc(&E.d_pid[k], E.pcap * sizeof(ull)));
  }
  CK(cudaMalloc(&E.d_counts, 16 * sizeof(int)));
  CK(cudaMemsetAsync(E.d_counts, 0, 16 * sizeof(int), E.stream));
  CK(cudaMalloc(&E.d_step, sizeof(uint32_t)));
  CK(cudaMemsetAsync(E.d_step, 0, sizeof(uint32_t), E.stream));
  CK(cudaMalloc(&E.d_cnt, ((size_t)E.ncell + 1) * sizeof(int)));
  CK(cudaMemsetAsync(E.d_cnt, 0, ((size_t)E.ncell + 1) * sizeof(int), E.stream));
  CK(cudaMalloc(&E.d_start, ((size_t)E.ncell + 1) * sizeof(int)));
  CK(cudaMemsetAsync(E.d_start, 0, ((size_t)E.ncell + 1) * sizeof(int), E.stream));
  CK(cudaMalloc(&E.d_scan_ticket, sizeof(ull)));
  CK(cudaMemsetAsync(E.d_scan_ticket, 0, sizeof(ull), E.stream));
  CK(cudaMalloc(&E.d_scan_status, (size_t)E.nscanblocks * sizeof(ull)));
  CK(cudaMemsetAsync(E.d_scan_status, 0, (size_t)E.nscanblocks * sizeof(ull), E.stream));
  CK(cudaMalloc(&E.d_ev, E.evcap * sizeof(Event)));
  CK(cudaMalloc(&E.d_cand, E.candcap * sizeof(int)));
  CK(cudaMalloc(&E.d_best, E.cap * sizeof(ull)));
  CK(cudaMalloc(&E.d_face, E.cap * sizeof(int)));
  CK(cudaMalloc(&E.d_tmp, (E.cap + E.pcap) * sizeof(float4)));
  CK(cudaMemsetAsync(E.d_best, 0xFF, E.cap * sizeof(ull), E.stream));
  CK(cudaMalloc(&E.d_counters, 8 * sizeof(unsigned long long)));
  CK(cudaMemsetAsync(E.d_counters, 0, 8 * sizeof(unsigned long long), E.stream));
  CK(cudaMalloc(&E.d_spcount, (size_t)reps.size() * net.nspecies * sizeof(long long)));
  CK(cudaMemsetAsync(E.d_spcount, 0, (size_t)reps.size() * net.nspecies * sizeof(long long), E.stream));

  // gaussian quantile table: sqrt(2)*erfinv((i+1/2)*2/n - 1) (random2.c:339-352);
  // the reference shuffles it, which does not matter for counter-based indices
  {
    std::vector<float> gt(gs);
    for (int i = 0; i < gs / 2; ++i) {
      const double pq = (i + 0.5) / gs;  // lower-tail probability
      double lo = -40, hi = 0;           // solve 0.5*erfc(-x/sqrt2) = pq by bisection
      for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (0.5 * std::erfc(-mid / std::sqrt(2.0)) < pq) lo = mid;
        else hi = mid;
      }
      gt[i] = (float)(0.5 * (lo + hi));
      gt[gs - 1 - i] = -gt[i];
    }
    CK(cudaMalloc(&E.d_gtab, gs * sizeof(float)));
    CK(cudaMemcpyAsync(E.d_gtab, gt.data(), gs * sizeof(float), cudaMemcpyHostToDevice, E.stream));
    CK(cudaStreamSynchronize(E.stream));
  }
  if (!E.net.panels.empty()) {
    if ((int)E.net.panels.size() > kMaxPanels) { if (err) *err = "too many panels (max 16)"; return -6; }
    E.panels.clear();
    for (const PanelSpec &ps : E.net.panels) {
      const DevPanel dp = make_dev_panel(ps, reps[0].lo);
      E.panels.push_back(dp);
    }
  }
  if (net.bound) {
    // surface-bound states: single simulations through the step pipeline
    if (reps.size() != 1) { if (err) *err = "surface-bound states need a single simulation"; return -6; }
    if (net.panels.empty()) { if (err) *err = "surface-bound states need surfaces"; return -6; }
    const size_t nrule = (size_t)std::max(1, net.nsrf) * kMaxSpecies * 9;
    if (net.srf_rules.size() != nrule) { if (err) *err = "surface rule table has the wrong size"; return -6; }
    D.bound = 1;
    D.beps = net.srf_eps;
    D.bmargin = net.srf_margin;
    D.bneighdist = net.srf_neighdist;
    for (int i = 0; i < net.nspecies; ++i) {
      D.sstep[i] = std::sqrt(2.0 * reps[0].difc[i] * dt);
      for (int k = 0; k < 2; ++k) D.bstep[i][k] = std::sqrt(2.0 * net.difc_bound[i][k] * dt);
    }
    E.bcap = E.cap;
    for (int k = 0; k < 2; ++k) CK(cudaMalloc(&E.d_bd[k], E.bcap * sizeof(BoundMol)));
    if (D.bpair_n) {
      CK(cudaMalloc(&E.d_bclaim, E.cap * sizeof(ull)));
      CK(cudaMemsetAsync(E.d_bclaim, 0xFF, E.cap * sizeof(ull), E.stream));
      CK(cudaMalloc(&E.d_bcand, E.bcap * sizeof(int4)));
      CK(cudaMemsetAsync(E.d_bcand, 0xFF, E.bcap * sizeof(int4), E.stream));
    }
    if (D.bb_n) {
      CK(cudaMalloc(&E.d_bbhead, ((size_t)1 << kBBHashBits) * sizeof(int)));
      CK(cudaMemsetAsync(E.d_bbhead, 0xFF, ((size_t)1 << kBBHashBits) * sizeof(int), E.stream));
      CK(cudaMalloc(&E.d_bbnext, E.bcap * sizeof(int)));
      CK(cudaMalloc(&E.d_bbcell, E.bcap * sizeof(ull)));
      CK(cudaMalloc(&E.d_bbbest, E.bcap * sizeof(ull)));
    }
    CK(cudaMalloc(&E.d_srfrule, nrule * sizeof(SrfRule)));
    CK(cudaMemcpyAsync(E.d_srfrule, net.srf_rules.data(), nrule * sizeof(SrfRule), cudaMemcpyHostToDevice, E.stream));
    CK(cudaStreamSynchronize(E.stream));
  }
  E.cmpts.clear();
  if ((int)E.net.cmpts.size() > kMaxCmpt) { if (err) *err = "too many compartments (max 8)"; return -6; }
  for (const CmptSpec &cs : E.net.cmpts) E.cmpts.push_back(make_dev_cmpt(cs, reps[0].lo));
  E.dnet.ncmpt = (int)E.cmpts.size();
  for (int o = 0; o < 3; ++o)
    for (int r = 0; r < kMaxRxn; ++r) {
      E.dnet.cmpt[o][r] = (uint8_t)E.net.cmpt[o][r];
      E.dnet.rsrf[o][r] = (uint8_t)E.net.rsrf[o][r];
      if (o == 0)
        for (int q = 0; q < kMaxProd; ++q) E.dnet.pstate0[r][q] = (uint8_t)E.net.pstate0[r][q];
    }
  for (int k = 0; k < kMaxPanels; ++k) E.dnet.parea[k] = E.net.panel_area[k];
  int rc = E.build_box_masks(err);
  if (rc) return rc;
  rc = E.build_rep_tables(err);
  if (rc) return rc;
  E.nsteps = 0;
  E.parity = 0;
  return 0;
}

int Engine::update_reps(const std::vector<RepSpec> &reps, std::string *err) {
  EngineImpl &E = *impl_;
  if (reps.size() != E.reps.size()) { if (err) *err = "replicate count changed"; return -6; }
  // the virtual boxes stay; the pair search looks one box deep, so a new
  // binding radius must still fit in a box
  for (size_t k = 0; k < reps.size(); ++k)
    for (int r = 0; r < E.net.nrxn[2]; ++r) {
      const double a = std::sqrt(std::max(0.0, reps[k].bind2[r]));
      for (int d = 0; d < reps[k].dim; ++d)
        if (a > E.geo[k].h[d]) {
          if (err) *err = "binding radius exceeds the virtual box size; rebuild the simulation";
          return -6;
        }
    }
  E.reps = reps;
  return E.build_rep_tables(err);
}

int Engine::set_molecules(long long n, const double *pos, const int *species, const int *rep,
                          const uint64_t *serno, std::string *err) {
  EngineImpl &E = *impl_;
  E.in_persist = false;  // replaced wholesale
  if (n > E.pcap) {
    // grow the product buffers so the upload fits (they are the upload staging area)
    for (int k = 0; k < 2; ++k) {
      cudaFree(E.d_ppc[k]);
      cudaFree(E.d_pid[k]);
      E.d_ppc[k] = nullptr;
      E.d_pid[k] = nullptr;
    }
    E.pcap = n;
    for (int k = 0; k < 2; ++k) {
      CK(cudaMalloc(&E.d_ppc[k], E.pcap * sizeof(float4)));
      CK(cudaMalloc(&E.d_pid[k], E.pcap * sizeof(ull)));
    }
    cudaFree(E.d_tmp);
    E.d_tmp = nullptr;
    CK(cudaMalloc(&E.d_tmp, (E.cap + E.pcap) * sizeof(float4)));
    E.invalidate_graph();
  }
  if (n > E.cap) { if (err) *err = "more molecules than the engine capacity"; return -9; }
  bool device_path = rep == nullptr && n > 0;
  if (device_path && serno)
    for (long long i = 0; i < n && device_path; ++i) device_path = serno[i] != 0;
  if (device_path) return E.upload_device(n, pos, species, serno, err);
  std::vector<float4> pc((size_t)n);
  std::vector<ull> id((size_t)n);
  std::vector<ull> next_serno(E.reps.size(), 1);
  if (serno)
    for (long long i = 0; i < n; ++i) {
      const int rp = rep ? rep[i] : 0;
      if (rp >= 0 && rp < (int)E.reps.size()) next_serno[rp] = std::max<ull>(next_serno[rp], (ull)serno[i] + 1);
    }
  for (long long i = 0; i < n; ++i) {
    const int rp = rep ? rep[i] : 0;
    if (rp < 0 || rp >= (int)E.reps.size()) { if (err) *err = "replicate index out of range"; return -6; }
    const int sp = species[i];
    if (sp <= 0 || sp >= E.net.nspecies) { if (err) *err = "species index out of range"; return -6; }
    const RepSpec &s = E.reps[rp];
    const DevGeo &g = E.geo[rp];
    int ix[3];
    float w[3];
    for (int d = 0; d < 3; ++d) {
      if (d >= s.dim) { ix[d] = 0; w[d] = 0.f; continue; }
      const double L = s.hi[d] - s.lo[d];
      const double h = L / g.n[d];
      const double x = pos[3 * i + d] - s.lo[d];
      int j = (int)std::floor(x / h);
      if (j < 0) j = 0;
      if (j > g.n[d] - 1) j = g.n[d] - 1;
      ix[d] = j;
      w[d] = (float)(x - j * h);
    }
    pc[i] = make_float4(w[0], w[1], w[2], 0.f);
    uint32_t packed = pack_cell(ix[0], ix[1], ix[2]);
    memcpy(&pc[i].w, &packed, 4);
    ull sn = (serno && serno[i]) ? (ull)serno[i] : next_serno[rp]++;
    id[i] = make_id(sp, rp, sn);
  }
  int zero[8] = {0};  // [8], [9]: bound-list counts, carried by finish_upload
  CK(cudaMemcpyAsync(E.d_counts, zero, sizeof(zero), cudaMemcpyHostToDevice, E.stream));
  CK(cudaMemcpyAsync(E.d_ppc[0], pc.data(), n * sizeof(float4), cudaMemcpyHostToDevice, E.stream));
  CK(cudaMemcpyAsync(E.d_pid[0], id.data(), n * sizeof(ull), cudaMemcpyHostToDevice, E.stream));
  return E.finish_upload(n, err);
}

int Engine::run(long long nsteps, std::string *err) {
  EngineImpl &E = *impl_;
  if (nsteps <= 0) return 0;
  if (E.persist_eligible()) {
    E.tail_slot = -1;
    int rc = E.run_persist(nsteps, err);
    if (rc) return rc;
    E.nsteps += nsteps;
    E.tail_step = E.nsteps;
    E.tail_gen = E.upload_gen;
    return 0;
  }
  if (E.in_persist) {
    int rc = E.leave_persist(err);
    if (rc) return rc;
  }
  const bool inj = E.dnet.inject != 0;
  if (inj) {
    if (nsteps != 1) { if (err) *err = "injected displacements apply to one step"; return -6; }
  }
  long long done = 0;
  E.tail_slot = -1;
  if (E.use_graph && !inj) {
    // two-step replays start at parity 0
    if (E.parity == 1) {
      int rc = E.run_one(err);
      if (rc) return rc;
      done++;
    }
    if (nsteps - done >= 2 && !E.graph2) {
      int rc = E.build_graph(err);
      if (rc) return rc;
    }
    while (nsteps - done >= 2) {
      CK(cudaGraphLaunch(E.graph2, E.stream));
      E.nlaunch += 2 * E.launches_per_step();
      done += 2;
      E.tail_slot = -1;
    }
    if (done < nsteps) {
      int rc = E.run_one(err);
      if (rc) return rc;
      done++;
    }
  }
  while (done < nsteps) {
    E.enqueue_step(E.parity, false);
    E.parity ^= 1;
    done++;
    E.tail_slot = -1;
  }
  E.nsteps += nsteps;
  E.tail_step = E.nsteps;
  E.tail_gen = E.upload_gen;
  CK(cudaGetLastError());
  if (inj) {
    E.dnet.inject = 0;
    CK(cudaMemcpyToSymbolAsync(c_net, &E.dnet, sizeof(DevNet), 0, cudaMemcpyHostToDevice, E.stream));
    CK(cudaStreamSynchronize(E.stream));
  }
  return 0;
}

int Engine::synchronize(std::string *err) {
  CK(cudaStreamSynchronize(impl_->stream));
  return 0;
}

int Engine::status_flags() {
  int st = 0;
  cudaStreamSynchronize(impl_->stream);
  cudaMemcpy(&st, impl_->d_counts + 6, sizeof(int), cudaMemcpyDeviceToHost);
  return st;
}

long long Engine::total_molecules() {
  EngineImpl &E = *impl_;
  int c[4] = {0, 0, 0, 0};
  cudaStreamSynchronize(E.stream);
  cudaMemcpy(c, E.d_counts, sizeof(c), cudaMemcpyDeviceToHost);
  std::vector<long long> sc;
  std::string err;
  if (species_counts(&sc, &err)) return -1;
  long long t = 0;
  for (long long v : sc) t += v;
  return t;
}

int Engine::species_counts(std::vector<long long> *out, std::string *err) {
  EngineImpl &E = *impl_;
  if (E.counts_step == E.nsteps && E.counts_gen == E.upload_gen &&
      E.counts_cache.size() == E.reps.size() * E.net.nspecies) {  // nothing ran since the last read
    *out = E.counts_cache;
    return 0;
  }
  out->assign(E.reps.size() * E.net.nspecies, 0);
  if (E.tail_slot >= 0 && E.tail_step == E.nsteps && E.tail_gen == E.upload_gen && E.h_tail_counts &&
      E.tail_ntab == out->size()) {  // copied by the step's own graph
    CK(cudaEventSynchronize(E.tail_ev[E.tail_slot]));
    memcpy(out->data(), E.h_tail_counts + (size_t)E.tail_slot * E.tail_ntab, out->size() * sizeof(long long));
  } else {
    CK(cudaMemcpyAsync(out->data(), E.d_spcount, out->size() * sizeof(long long), cudaMemcpyDeviceToHost,
                       E.stream));
    CK(cudaStreamSynchronize(E.stream));
  }
  E.counts_cache = *out;
  E.counts_step = E.nsteps;
  E.counts_gen = E.upload_gen;
  return 0;
}

int Engine::status_flags_lagged() {
  EngineImpl &E = *impl_;
  if (E.tail_slot >= 0 && E.tail_step == E.nsteps) {
    // the step's graph copies its status into its slot; report the previous step's
    int st = 0;
    if (E.tail_prev_slot >= 0) {
      cudaEventSynchronize(E.tail_ev[E.tail_prev_slot]);
      st = E.h_tail_status[E.tail_prev_slot];
    }
    E.tail_prev_slot = E.tail_slot;
    return st;
  }
  E.tail_prev_slot = -1;
  if (!E.h_status) {
    if (cudaMallocHost(&E.h_status, 2 * sizeof(int)) != cudaSuccess) { E.h_status = nullptr; return status_flags(); }
    for (int k = 0; k < 2; ++k) cudaEventCreateWithFlags(&E.st_ev[k], cudaEventDisableTiming);
  }
  const int prev = E.st_slot ^ 1;
  int st = 0;
  if (E.st_pending[prev]) {
    cudaEventSynchronize(E.st_ev[prev]);
    st = E.h_status[prev];
    E.st_pending[prev] = false;
  }
  cudaMemcpyAsync(&E.h_status[E.st_slot], E.d_counts + 6, sizeof(int), cudaMemcpyDeviceToHost, E.stream);
  cudaEventRecord(E.st_ev[E.st_slot], E.stream);
  E.st_pending[E.st_slot] = true;
  E.st_slot ^= 1;
  return st;
}

int Engine::stats(EngineStats *s, std::string *err) {
  EngineImpl &E = *impl_;
  unsigned long long c[8];
  CK(cudaMemcpyAsync(c, E.d_counters, sizeof(c), cudaMemcpyDeviceToHost, E.stream));
  int st = 0;
  CK(cudaMemcpyAsync(&st, E.d_counts + 6, sizeof(int), cudaMemcpyDeviceToHost, E.stream));
  CK(cudaStreamSynchronize(E.stream));
  s->wall = (long long)c[0];
  s->rxn0 = (long long)c[1];
  s->rxn1 = (long long)c[2];
  s->rxn2 = (long long)c[3];
  s->unresolved = (long long)c[4];
  s->multicand = (long long)c[5];
  s->overflow = st;
  return 0;
}

int Engine::set_bound(long long n, const double *pos, const int *species, const int *state, const int *panel,
                      const uint64_t *serno, std::string *err) {
  EngineImpl &E = *impl_;
  if (!E.dnet.bound) {
    if (n == 0) return 0;
    if (err) *err = "surface-bound molecules need surface rules with bound states";
    return -6;
  }
  if (n > E.bcap) { if (err) *err = "more surface-bound molecules than the engine capacity"; return -9; }
  std::vector<BoundMol> m((size_t)n);
  for (long long i = 0; i < n; ++i) {
    const int sp = species[i];
    if (sp <= 0 || sp >= E.net.nspecies) { if (err) *err = "species index out of range"; return -6; }
    if (state[i] != 1 && state[i] != 2) { if (err) *err = "bound state must be front or back"; return -6; }
    if (panel[i] < 0 || panel[i] >= (int)E.panels.size()) { if (err) *err = "panel index out of range"; return -6; }
    for (int d = 0; d < 3; ++d) m[i].x[d] = pos[3 * i + d] - E.reps[0].lo[d];
    m[i].pnl = panel[i];
    m[i].ms = state[i];
    m[i].born = kBornNever;
    m[i].pad = 0;
    const ull sn = (serno && serno[i]) ? (ull)serno[i] : ((1ull << 40) + (ull)i);
    m[i].id = make_id(sp, 0, sn);
  }
  const int in = E.parity;
  const int nn = (int)n;
  CK(cudaStreamSynchronize(E.stream));
  if (n) CK(cudaMemcpy(E.d_bd[in], m.data(), (size_t)n * sizeof(BoundMol), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(E.d_counts + 8 + in, &nn, sizeof(int), cudaMemcpyHostToDevice));
  // species counts: solution (sorted and product lists) plus the new bound
  // list; a product count past the capacity (an overflow already flagged)
  // is clamped first, as the next step would
  int pn = 0;
  CK(cudaMemcpy(&pn, E.d_counts + 2 + in, sizeof(int), cudaMemcpyDeviceToHost));
  if (pn > (int)E.pcap) {
    pn = (int)E.pcap;
    CK(cudaMemcpy(E.d_counts + 2 + in, &pn, sizeof(int), cudaMemcpyHostToDevice));
  }
  const size_t nt = E.reps.size() * E.net.nspecies;
  CK(cudaMemsetAsync(E.d_spcount, 0, nt * sizeof(long long), E.stream));
  k_species_count<<<E.grid_mol(), 256, 0, E.stream>>>(E.d_id[in], E.d_counts + in, E.d_spcount, E.net.nspecies, (int)nt);
  k_species_count<<<E.grid_mol(), 256, 0, E.stream>>>(E.d_pid[in], E.d_counts + 2 + in, E.d_spcount, E.net.nspecies,
                                                      (int)nt);
  k_bound_species_count<<<E.grid_small(), 256, 0, E.stream>>>(E.d_bd[in], E.d_counts + 8 + in, E.d_spcount);
  E.nlaunch += 3;
  CK(cudaStreamSynchronize(E.stream));
  CK(cudaGetLastError());
  ++E.upload_gen;
  return 0;
}

int Engine::get_bound(std::vector<double> *pos, std::vector<int> *species, std::vector<int> *state,
                      std::vector<int> *panel, std::vector<uint64_t> *serno, std::string *err) {
  EngineImpl &E = *impl_;
  pos->clear(); species->clear(); state->clear(); panel->clear(); serno->clear();
  if (!E.dnet.bound) return 0;
  const int in = E.parity;
  int nb = 0;
  CK(cudaStreamSynchronize(E.stream));
  CK(cudaMemcpy(&nb, E.d_counts + 8 + in, sizeof(int), cudaMemcpyDeviceToHost));
  nb = std::max(0, std::min<int>(nb, (int)E.bcap));
  std::vector<BoundMol> m((size_t)nb);
  if (nb) CK(cudaMemcpy(m.data(), E.d_bd[in], (size_t)nb * sizeof(BoundMol), cudaMemcpyDeviceToHost));
  std::sort(m.begin(), m.end(), [](const BoundMol &a, const BoundMol &b) { return id_serno(a.id) < id_serno(b.id); });
  for (const BoundMol &b : m) {
    if (id_species(b.id) == kDeadSpecies) continue;
    for (int d = 0; d < 3; ++d) pos->push_back(b.x[d] + E.reps[0].lo[d]);
    species->push_back(id_species(b.id));
    state->push_back(b.ms);
    panel->push_back(b.pnl);
    serno->push_back(id_serno(b.id));
  }
  return 0;
}

int Engine::get_molecules(std::vector<double> *pos, std::vector<int> *species, std::vector<int> *rep,
                          std::vector<uint64_t> *serno, std::string *err) {
  EngineImpl &E = *impl_;
  if (int rc = E.leave_persist(err)) return rc;
  int c[4];
  CK(cudaStreamSynchronize(E.stream));
  CK(cudaMemcpy(c, E.d_counts, sizeof(c), cudaMemcpyDeviceToHost));
  const int in = E.parity;
  const int na = c[in], np = std::min<int>(c[2 + in], (int)E.pcap);
  std::vector<float4> pc((size_t)na + np);
  std::vector<ull> id((size_t)na + np);
  if (na) {
    CK(cudaMemcpy(pc.data(), E.d_pc[in], (size_t)na * sizeof(float4), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(id.data(), E.d_id[in], (size_t)na * sizeof(ull), cudaMemcpyDeviceToHost));
  }
  if (np) {
    CK(cudaMemcpy(pc.data() + na, E.d_ppc[in], (size_t)np * sizeof(float4), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(id.data() + na, E.d_pid[in], (size_t)np * sizeof(ull), cudaMemcpyDeviceToHost));
  }
  std::vector<size_t> idx;
  idx.reserve(pc.size());
  for (size_t i = 0; i < pc.size(); ++i)
    if (id_species(id[i]) != kDeadSpecies) idx.push_back(i);
  std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
    const int ra = id_rep(id[a]), rb = id_rep(id[b]);
    if (ra != rb) return ra < rb;
    return id_serno(id[a]) < id_serno(id[b]);
  });
  pos->resize(idx.size() * 3);
  species->resize(idx.size());
  if (rep) rep->resize(idx.size());
  serno->resize(idx.size());
  for (size_t k = 0; k < idx.size(); ++k) {
    const size_t i = idx[k];
    const int rp = id_rep(id[i]);
    const RepSpec &s = E.reps[rp];
    const DevGeo &g = E.geo[rp];
    uint32_t w;
    memcpy(&w, &pc[i].w, 4);
    int ix[3];
    unpack_cell(w, ix[0], ix[1], ix[2]);
    const float u[3] = {pc[i].x, pc[i].y, pc[i].z};
    for (int d = 0; d < 3; ++d) {
      if (d >= s.dim) { (*pos)[3 * k + d] = 0; continue; }
      const double h = (s.hi[d] - s.lo[d]) / g.n[d];
      (*pos)[3 * k + d] = s.lo[d] + ix[d] * h + (double)u[d];
    }
    (*species)[k] = id_species(id[i]);
    if (rep) (*rep)[k] = rp;
    (*serno)[k] = id_serno(id[i]);
  }
  return 0;
}

int Engine::set_injection(long long n, const uint64_t *sernos, const double *disp, int rep,
                          std::string *err) {
  EngineImpl &E = *impl_;
  if (int rc = E.leave_persist(err)) return rc;
  if (E.d_injkey) { cudaFree(E.d_injkey); E.d_injkey = nullptr; }
  if (E.d_injval) { cudaFree(E.d_injval); E.d_injval = nullptr; }
  E.inj_n = 0;
  if (n <= 0) {
    E.dnet.inject = 0;
    return E.upload_const(err);
  }
  std::vector<std::pair<ull, float4>> v((size_t)n);
  for (long long i = 0; i < n; ++i) {
    const ull key = id_stream(make_id(0, rep, sernos[i]));
    v[i] = {key, make_float4((float)disp[4 * i], (float)disp[4 * i + 1], (float)disp[4 * i + 2],
                             (float)disp[4 * i + 3])};
  }
  std::sort(v.begin(), v.end(), [](const std::pair<ull, float4> &a, const std::pair<ull, float4> &b) {
    return a.first < b.first;
  });
  std::vector<ull> keys((size_t)n);
  std::vector<float4> vals((size_t)n);
  for (long long i = 0; i < n; ++i) { keys[i] = v[i].first; vals[i] = v[i].second; }
  CK(cudaMalloc(&E.d_injkey, n * sizeof(ull)));
  CK(cudaMalloc(&E.d_injval, n * sizeof(float4)));
  CK(cudaMemcpy(E.d_injkey, keys.data(), n * sizeof(ull), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(E.d_injval, vals.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
  E.inj_n = (int)n;
  E.dnet.inject = 1;
  E.invalidate_graph();
  return E.upload_const(err);
}

int Engine::set_rng_step(uint64_t step, std::string *err) {
  EngineImpl &E = *impl_;
  const uint32_t v = (uint32_t)step;
  CK(cudaStreamSynchronize(E.stream));
  CK(cudaMemcpy(E.d_step, &v, sizeof(v), cudaMemcpyHostToDevice));
  return 0;
}

int Engine::msd_track(int species, long long m, const uint64_t *keys, const double *start, const double *last,
                      std::string *err) {
  EngineImpl &E = *impl_;
  if (int rc = E.leave_persist(err)) return rc;
  if (species <= 0 || species >= E.net.nspecies) {
    if (err) *err = "species index out of range";
    return -6;
  }
  for (long long k = 1; k < m; ++k)
    if (keys[k] <= keys[k - 1]) {
      if (err) *err = "tracker keys must be strictly increasing";
      return -6;
    }
  if (!E.d_msdgeo) {
    std::vector<MsdGeo> g(E.reps.size());
    for (size_t r = 0; r < E.reps.size(); ++r) {
      const RepSpec &s = E.reps[r];
      MsdGeo &q = g[r];
      q.dim = s.dim;
      q.periodic = 0;
      for (int d = 0; d < 3; ++d) {
        q.lo[d] = s.lo[d];
        q.len[d] = s.hi[d] - s.lo[d];
        q.h[d] = d < s.dim ? q.len[d] / E.geo[r].n[d] : 0.0;
        if (d < s.dim && s.wall[2 * d] == kWallPeriodic && s.wall[2 * d + 1] == kWallPeriodic) q.periodic |= 1 << d;
      }
    }
    CK(cudaMalloc(&E.d_msdgeo, g.size() * sizeof(MsdGeo)));
    CK(cudaMemcpy(E.d_msdgeo, g.data(), g.size() * sizeof(MsdGeo), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&E.d_msdpart, 3 * kMsdBlocks * sizeof(double)));
  }
  EngineImpl::MsdTrack t;
  t.species = species;
  t.m = m;
  const size_t mm = (size_t)std::max<long long>(m, 1);
  CK(cudaMalloc(&t.keys, mm * sizeof(ull)));
  CK(cudaMalloc(&t.start, 3 * mm * sizeof(double)));
  CK(cudaMalloc(&t.last, 3 * mm * sizeof(double)));
  if (m > 0) {
    CK(cudaMemcpy(t.keys, keys, (size_t)m * sizeof(ull), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(t.start, start, 3 * (size_t)m * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(t.last, last, 3 * (size_t)m * sizeof(double), cudaMemcpyHostToDevice));
  }
  E.msd.push_back(t);
  return (int)E.msd.size() - 1;
}

int Engine::msd_update(int handle, int msddim, double *sum2, double *sum4, long long *count, std::string *err) {
  EngineImpl &E = *impl_;
  if (int rc = E.leave_persist(err)) return rc;
  if (handle < 0 || handle >= (int)E.msd.size()) {
    if (err) *err = "no such tracker";
    return -6;
  }
  const EngineImpl::MsdTrack &t = E.msd[handle];
  const int in = E.parity;
  k_msd<<<kMsdBlocks, kMsdThreads, 0, E.stream>>>(E.d_pc[in], E.d_id[in], E.d_counts + in, E.d_ppc[in], E.d_pid[in],
                                                  E.d_counts + 2 + in, (int)E.pcap, E.d_msdgeo, (int)E.reps.size(),
                                                  t.species, t.keys, t.m, t.start, t.last, msddim, E.d_msdpart);
  CK(cudaGetLastError());
  ++E.nlaunch;
  if (!sum2 && !sum4 && !count) return 0;
  std::vector<double> part(3 * kMsdBlocks);
  CK(cudaMemcpyAsync(part.data(), E.d_msdpart, part.size() * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
  CK(cudaStreamSynchronize(E.stream));
  double a = 0, b = 0, c = 0;
  for (int k = 0; k < kMsdBlocks; ++k) {
    a += part[3 * k];
    b += part[3 * k + 1];
    c += part[3 * k + 2];
  }
  if (sum2) *sum2 = a;
  if (sum4) *sum4 = b;
  if (count) *count = (long long)c;
  return 0;
}

int Engine::msd_last(int handle, std::vector<double> *last, std::string *err) {
  EngineImpl &E = *impl_;
  if (handle < 0 || handle >= (int)E.msd.size()) {
    if (err) *err = "no such tracker";
    return -6;
  }
  const EngineImpl::MsdTrack &t = E.msd[handle];
  last->resize(3 * (size_t)t.m);
  CK(cudaStreamSynchronize(E.stream));
  if (t.m > 0) CK(cudaMemcpy(last->data(), t.last, last->size() * sizeof(double), cudaMemcpyDeviceToHost));
  return 0;
}

int Engine::msd_count() const { return (int)impl_->msd.size(); }

int Engine::cmpt_counts(int c, std::vector<long long> *out, std::string *err) {
  EngineImpl &E = *impl_;
  if (int rc = E.leave_persist(err)) return rc;
  if (c < 0 || c >= (int)E.cmpts.size()) {
    if (err) *err = "no such compartment";
    return -6;
  }
  const int nsp = E.net.nspecies;
  unsigned long long *d = nullptr;
  CK(cudaMalloc(&d, kMaxSpecies * sizeof(unsigned long long)));
  cudaError_t e = cudaMemsetAsync(d, 0, kMaxSpecies * sizeof(unsigned long long), E.stream);
  const int in = E.parity;
  if (e == cudaSuccess) {
    k_cmpt_count<<<sm_count() * 4, 256, 0, E.stream>>>(E.d_pc[in], E.d_id[in], E.d_counts + in, E.d_ppc[in],
                                                         E.d_pid[in], E.d_counts + 2 + in, (int)E.pcap, E.d_geo,
                                                         (int)E.reps.size(), c, nsp, d);
    e = cudaGetLastError();
  }
  std::vector<unsigned long long> h(kMaxSpecies, 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                            E.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
  cudaFree(d);
  if (e != cudaSuccess) {
    if (err) *err = std::string("compartment count: ") + cudaGetErrorString(e);
    return -8;
  }
  ++E.nlaunch;
  out->assign(nsp, 0);
  for (int k = 0; k < nsp; ++k) (*out)[k] = (long long)h[k];
  return 0;
}

int Engine::profile(long long nsteps, std::vector<std::string> *names, std::vector<double> *ms,
                    std::vector<long long> *launches, std::string *err) {
  EngineImpl &E = *impl_;
  if (int rc = E.leave_persist(err)) return rc;
  names->clear();
  ms->clear();
  launches->clear();
  E.prof = true;
  E.marks.clear();
  E.pool_used = 0;
  E.mark("start");
  E.nlaunch--;
  for (long long k = 0; k < nsteps; ++k) {
    E.enqueue_step(E.parity, false);
    E.parity ^= 1;
  }
  E.nsteps += nsteps;
  E.prof = false;
  CK(cudaStreamSynchronize(E.stream));
  CK(cudaGetLastError());
  for (size_t k = 1; k < E.marks.size(); ++k) {
    float t = 0;
    CK(cudaEventElapsedTime(&t, E.marks[k - 1].second, E.marks[k].second));
    const std::string nm = E.marks[k].first;
    size_t j = 0;
    while (j < names->size() && (*names)[j] != nm) ++j;
    if (j == names->size()) {
      names->push_back(nm);
      ms->push_back(0);
      launches->push_back(0);
    }
    (*ms)[j] += t;
    (*launches)[j] += 1;
  }
  E.marks.clear();
  return 0;
}

void Engine::set_stream(void *stream) {
  impl_->invalidate_graph();
  impl_->stream = stream ? (cudaStream_t)stream : impl_->own_stream;
}
void *Engine::stream() const { return (void *)impl_->stream; }
long long Engine::launches() const { return impl_->nlaunch; }
long long Engine::steps_done() const { return impl_->nsteps; }
int Engine::set_persistent(int mode, std::string *err) {
  EngineImpl &E = *impl_;
  if (mode < 0 || mode > 1) { if (err) *err = "persistent mode must be 0 or 1"; return -6; }
  if (!mode && E.in_persist) {
    if (int rc = E.leave_persist(err)) return rc;
  }
  E.persist_mode = mode;
  return 0;
}
bool Engine::persistent_active() const { return impl_->persist_eligible(); }
void Engine::set_use_graph(bool on) {
  impl_->use_graph = on;
  if (!on) impl_->invalidate_graph();
}

int Engine::set_tuning(const LaunchTuning &t, std::string *err) {
  if (t.pair_tile != 128 && t.pair_tile != 256) { if (err) *err = "pair tile must be 128 or 256"; return -6; }
  if (t.mol_blocks_per_sm < 1 || t.mol_blocks_per_sm > 32 || t.tile_blocks_per_sm < 1 || t.tile_blocks_per_sm > 32) {
    if (err) *err = "blocks per SM must be 1..32";
    return -6;
  }
  impl_->tune = t;
  impl_->invalidate_graph();
  return 0;
}

LaunchTuning Engine::tuning() const { return impl_->tune; }

int solve_radii_device(int mode, long long n, const double *rate, double dt, const double *difc,
                       const double *b, int rel, double *out, std::string *err) {
  if (n <= 0) return 0;
  double *d = nullptr;
  CK(cudaMalloc(&d, (size_t)n * 4 * sizeof(double)));
  CK(cudaMemcpy(d, rate, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + n, difc, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + 2 * n, b, n * sizeof(double), cudaMemcpyHostToDevice));
  k_solve_radii<<<sm_count() * 2, 128>>>(mode, n, d, dt, d + n, d + 2 * n, rel, d + 3 * n);
  CK(cudaGetLastError());
  CK(cudaMemcpy(out, d + 3 * n, n * sizeof(double), cudaMemcpyDeviceToHost));
  cudaFree(d);
  return 0;
}

int solve_radii_prob_device(long long n, const double *rate, double dt, const double *difc, const double *b,
                            int rel, const double *chi, double *prob, double *out, std::string *err) {
  if (n <= 0) return 0;
  double *d = nullptr;
  CK(cudaMalloc(&d, (size_t)n * 6 * sizeof(double)));
  CK(cudaMemcpy(d, rate, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + n, difc, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + 2 * n, b, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + 3 * n, chi, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + 4 * n, prob, n * sizeof(double), cudaMemcpyHostToDevice));
  k_solve_radii_prob<<<sm_count() * 2, 128>>>(n, d, dt, d + n, d + 2 * n, rel, d + 3 * n, d + 4 * n, d + 5 * n);
  CK(cudaGetLastError());
  CK(cudaMemcpy(prob, d + 4 * n, n * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(out, d + 5 * n, n * sizeof(double), cudaMemcpyDeviceToHost));
  cudaFree(d);
  return 0;
}

}  // namespace smolb


namespace smolb {
int solve_pair_radii_device(long long n, const double *kf, const double *dsum, double dt, int same, int rev,
                            int rparamt, double rparam, double *bind, double *unbind, int *errs, std::string *err) {
  if (n <= 0) return 0;
  double *d = nullptr;
  int *de = nullptr;
  CK(cudaMalloc(&d, (size_t)n * 4 * sizeof(double)));
  CK(cudaMalloc(&de, (size_t)n * sizeof(int)));
  CK(cudaMemcpy(d, kf, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + n, dsum, n * sizeof(double), cudaMemcpyHostToDevice));
  k_pair_radii<<<sm_count() * 2, 128>>>(n, d, d + n, dt, same, rev, rparamt, rparam, d + 2 * n, d + 3 * n, de);
  CK(cudaGetLastError());
  CK(cudaMemcpy(bind, d + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(unbind, d + 3 * n, n * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(errs, de, n * sizeof(int), cudaMemcpyDeviceToHost));
  cudaFree(d);
  cudaFree(de);
  return 0;
}
}  // namespace smolb
