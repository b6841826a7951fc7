// Device-side building blocks shared by the engine kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "engine.h"

namespace smolb {

typedef unsigned long long ull;

// ---- molecule identity word ------------------------------------------------
// bits 63..58 species (63 = dead), 57..42 replicate, 41..0 serial number.
constexpr int kSpShift = 58;
constexpr int kRepShift = 42;
constexpr ull kSernoMask = (1ull << 42) - 1;
constexpr ull kRepMask = 0xFFFFull;
constexpr int kDeadSpecies = 63;
constexpr ull kProductSernoBit = 1ull << 41;  // product serial numbers have this bit set

__host__ __device__ __forceinline__ int id_species(ull id) { return (int)(id >> kSpShift); }
__host__ __device__ __forceinline__ int id_rep(ull id) { return (int)((id >> kRepShift) & kRepMask); }
__host__ __device__ __forceinline__ ull id_serno(ull id) { return id & kSernoMask; }
__host__ __device__ __forceinline__ ull make_id(int sp, int rep, ull serno) {
  return ((ull)sp << kSpShift) | ((ull)rep << kRepShift) | (serno & kSernoMask);
}
__host__ __device__ __forceinline__ ull id_mark_dead(ull id) {
  return (id & ~(63ull << kSpShift)) | ((ull)kDeadSpecies << kSpShift);
}
// identity without the species field (stable RNG stream key of a molecule)
__host__ __device__ __forceinline__ ull id_stream(ull id) { return id & ((1ull << kSpShift) - 1); }

// ---- cell coordinates packed into the w lane of the position float4 --------
__host__ __device__ __forceinline__ uint32_t pack_cell(int ix, int iy, int iz) {
  return (uint32_t)ix | ((uint32_t)iy << 10) | ((uint32_t)iz << 20);
}
__host__ __device__ __forceinline__ void unpack_cell(uint32_t w, int &ix, int &iy, int &iz) {
  ix = (int)(w & 1023u);
  iy = (int)((w >> 10) & 1023u);
  iz = (int)((w >> 20) & 1023u);
}

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw; SC'11) ----------------------
__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

__host__ __device__ __forceinline__ uint4 philox(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = mulhi32(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = mulhi32(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// Same generator with the 10 round keys precomputed (ks[2r], ks[2r+1]); used
// with a key schedule held in constant memory so no per-thread key arithmetic
// is issued.  Produces exactly philox(c, {ks[0], ks[1]}).
__host__ __device__ __forceinline__ uint4 philox_ks(uint4 c, const uint32_t *ks) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = mulhi32(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = mulhi32(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ ks[2 * r], lo1, hi0 ^ c.w ^ ks[2 * r + 1], lo0);
  }
  return c;
}

// uniform in [0,1) with 32-bit resolution (matches randCOD's granularity)
__host__ __device__ __forceinline__ double u01d(uint32_t x) { return x * 2.3283064365386963e-10; }
// uniform in (0,1) as float with 24-bit resolution
__host__ __device__ __forceinline__ float u01f_open(uint32_t x) {
  return ((x >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

// SplitMix64 finaliser, used to derive product serial numbers and birth keys.
__host__ __device__ __forceinline__ ull mix64(ull z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// ---- engine constants (one copy per library, set before each launch batch) --
struct DevNet {
  int nsp, nrep;
  int nr[3];
  int rxn_base[3];     // order o reaction r -> index rxn_base[o]+r in per-rep product tables
  int nrx_total;
  uint32_t gmask;      // gaussian table size - 1
  uint32_t key0, key1; // Philox key (seed)
  uint32_t move_ks[20]; // round keys of the move generator (key0, key1 scheduled)
  int any_drift;
  uint32_t difm_any;   // species with an anisotropic diffusion matrix
  int any_absorb;
  int inject;          // deterministic mode active
  int npanel;
  double surf_eps;     // distance kept between a molecule and a panel after an interaction
  float surf_tol;      // FP32 screening margin: eps plus the FP32 rounding of absolute positions
  float mask_len;      // moves up to this length screen only their start box's panels (0: no box masks)
  int rounds;          // pair conflict-resolution rounds
  uint32_t uni_any;    // species with at least one first-order reaction (bit per species)
  uint32_t pair_any;   // species with at least one second-order reaction
  int uni_n[kMaxSpecies];
  uint8_t uni_list[kMaxSpecies][kMaxUniPerSpecies];
  uint32_t pair_mask[kMaxSpecies];    // partner species of a pair reaction
  uint32_t search_mask[kMaxSpecies];  // partners searched in round 1: each pair once
  uint8_t pair_n[kMaxSpecies][kMaxSpecies];
  uint8_t pair_list[kMaxSpecies][kMaxSpecies][kMaxPairRxn];
  uint8_t rct[3][kMaxRxn][2];
  uint8_t nprod[3][kMaxRxn];
  uint8_t prd[3][kMaxRxn][kMaxProd];
  uint8_t fixed[3][kMaxRxn];
  uint8_t has_offset[3][kMaxRxn];
  // order-2 product placement: 0 = at the site (with offsets), 1 = confspread
  // (products take the reactants' places), 2 = bounce (reactants pushed apart)
  uint8_t placement2[kMaxRxn];
  float bounce_k[kMaxRxn];   // bounce scaling: 1 (given unbinding radius) or 2 (from the binding radius)
  int ncmpt;
  uint8_t cmpt[3][kMaxRxn];  // compartment of each reaction + 1 (0: anywhere)
  uint8_t rsrf[3][kMaxRxn];  // surface of each reaction + 1 (0: any): births on it (order 0), or bound reactants
  uint8_t pstate0[kMaxRxn][kMaxProd];  // product states of order-0 reactions (births on a surface)
  double parea[kMaxPanels];  // area of each panel (length in 2-D), for births on a surface
  // surface-bound states (single simulations)
  int bound;                       // 1: surface rules and bound molecules in use
  double beps, bmargin, bneighdist; // surfacessstruct epsilon, margin, neighdist for bound molecules
  double bstep[kMaxSpecies][2];    // sqrt(2 D dt) of the front and back states
  double sstep[kMaxSpecies];       // sqrt(2 D dt) of the solution state, FP64 (desorption distance)
  // first-order reactions of bound molecules by (species, front/back): the
  // reactions in list order and their cumulative thresholds (fractions of 2^32)
  uint8_t buni_n[kMaxSpecies][2];
  uint8_t buni_list[kMaxSpecies][2][kMaxUniPerSpecies];
  uint32_t bthr[kMaxSpecies][2][kMaxUniPerSpecies];
  uint8_t pstate1[kMaxRxn][2];     // product states of each first-order reaction (first two products)
  // second-order reactions of a bound and a solution reactant, in list
  // order: the reaction, the bound reactant's species and state (1 front,
  // 2 back), the solution reactant's species and the product's state; per
  // bound (species, front/back) the solution species it reacts with
  int bpair_n;
  uint8_t bpair_rxn[kMaxRxn], bpair_bsp[kMaxRxn], bpair_bst[kMaxRxn], bpair_ssp[kMaxRxn], bpair_pst[kMaxRxn];
  uint32_t bpair_mask[kMaxSpecies][2];
  float bpair_rmax;  // largest binding radius of these reactions, padded as the stencil radii are
  // second-order reactions of two bound reactants (same panel), in list
  // order: the reaction, both reactants' species and states, the product's
  // state; per bound (species, front/back) the bound species it reacts with
  int bb_n;
  uint8_t bb_rxn[kMaxRxn], bb_sp[kMaxRxn][2], bb_st[kMaxRxn][2], bb_pst[kMaxRxn];
  uint32_t bb_mask[kMaxSpecies][2];
  float bb_rmax;
  double bb_inv_cs;  // 1 / cell side of the bound-bound grid (the largest binding radius)
};

// A molecule bound to a panel: absolute position (relative to the system's
// low corner), id as for solution molecules, engine panel index and state
// (1 front, 2 back; MolecState numbering).
struct BoundMol {
  double x[3];
  ull id;
  int pnl;
  int ms;
  uint32_t born;  // step in which a reaction made it (it reacts again from the next step), else all ones
  uint32_t pad;
};
constexpr uint32_t kBornNever = 0xFFFFFFFFu;

// Per-replicate geometry.  Cells are cubes of size h; the last cell in each
// dimension extends to the high wall, which sits at local coordinate whi.
struct DevGeo {
  float h[3], inv_h[3], whi[3];
  int n[3];
  int cell0;   // first global cell index of this replicate
  int dim;
  uint8_t wall[6];
  uint8_t pad[2];
  float vol;
};

// Surface panel (shared by all replicates; coordinates relative to the low
// corner of the system, FP64 because crossing tests near a panel need it).
struct DevPanel {
  int shape;        // 0 rect, 1 tri, 2 sph, 3 cyl, 4 hemi, 5 disk (PanelSpec)
  int axis;         // rect: perpendicular axis
  int front_sign;   // +1: front face toward +axis (rect) / outward (sph, cyl, hemi); tri, disk: +1
  int pad;
  double pos;       // rect plane coordinate
  double lo[3], hi[3];
  double center[3]; // sph, hemi, disk centre
  double radius;
  double pt[3][3];  // tri vertices; cyl axis end points
  double nrm[3];    // tri, disk: unit front normal; hemi: unit open-side vector; cyl: unit axis
  double axlen;     // cyl: axis length
  int act_front, act_back;   // default action per face: 0 reflect 1 transmit 2 absorb
  uint32_t abs_front, abs_back, tr_front, tr_back, rf_front, rf_back;  // per-species overrides
  uint32_t jp_front, jp_back;        // species that jump at the front / back face
  int jump_pnl[2], jump_face[2];     // per face: the panel a jump leads to (-1 none) and its face
  float posf, radiusf, centerf[3];   // FP32 copies for the screening test
  float p0f[3], nrmf[3];             // screen reference point and unit vector (zero for sph, hemi)
  int curved;                        // screen: 1 sph, cyl, hemi (radial test); 0 flat (plane test)
  int srf;                           // surface index (rule table)
  int nneigh, neighhop;              // neighbouring panels for surface-bound molecules; 1: hop
  int neigh[kMaxNeigh];
};

// Compartment (smolcomparts.c compartstruct subset): interior points, the
// panels of its bounding surfaces (bit per panel index) and logic terms on
// earlier compartments (symbol 0 equal, 1 equalnot, 2 and, 3 or, 4 xor,
// 5 andnot, 6 ornot).  Positions relative to the system's low corner.
struct DevCmpt {
  int npts, ncl;
  uint32_t panels;
  int pad;
  double pts[kMaxCmptPts][3];
  int clsym[kMaxCmptLogic], clcmpt[kMaxCmptLogic];
};

struct Event {      // one reaction or birth; products are placed by k_products
  float4 site;      // reaction site: local coordinates + packed cell (orders 1, 2)
  ull key;          // parent identity (stream key) used for product RNG and serial numbers
  uint32_t rxn;     // order << 8 | reaction index
  uint32_t rep;
  int ia, ib;       // order 2: sorted indices of reactants 1 and 2 (else -1)
};

}  // namespace smolb
