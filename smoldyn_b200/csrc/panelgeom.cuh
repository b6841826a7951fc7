// Panel geometry shared by the engine kernels and the host (placement and
// volume of compartments): crossings of a segment with a panel, the panel's
// front normal and signed distance, and the compartment membership test.
// Coordinates are relative to the system's low corner.
#pragma once

#include <math.h>

#include "devcommon.cuh"
#include "rxnparam.cuh"

#ifdef __CUDACC__
#define SMOLB_HDI __host__ __device__ __forceinline__
#else
#define SMOLB_HDI inline
#endif

namespace smolb {

SMOLB_HDI double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// component of x - pt[0] normal to a cylinder's axis
SMOLB_HDI void cyl_radial(const DevPanel &pn, const double x[3], double r[3]) {
  double w[3];
  for (int d = 0; d < 3; ++d) w[d] = x[d] - pn.pt[0][d];
  const double s = dot3(w, pn.nrm);
  for (int d = 0; d < 3; ++d) r[d] = w[d] - s * pn.nrm[d];
}

// unit normal toward the front face at point x of the panel (panelnormal,
// smolsurface.c:3967)
template <bool GEN>
SMOLB_HDI void panel_normal(const DevPanel &pn, const double x[3], double n[3]) {
  if (pn.shape == 2 || (GEN && (pn.shape == 4 || pn.shape == 3))) {  // sph, hemi: from the centre; cyl: from the axis
    if (GEN && pn.shape == 3) {
      cyl_radial(pn, x, n);
    } else {
      for (int d = 0; d < 3; ++d) n[d] = x[d] - pn.center[d];
    }
    const double l2 = dot3(n, n);
    const double l = (l2 > 0) ? pn.front_sign / sqrt(l2) : 0.0;
    for (int d = 0; d < 3; ++d) n[d] *= l;
  } else if (GEN && (pn.shape == 1 || pn.shape == 5)) {  // tri, disk: the front normal
    for (int d = 0; d < 3; ++d) n[d] = pn.nrm[d];
  } else {
    n[0] = n[1] = n[2] = 0.0;
    n[pn.axis] = (double)pn.front_sign;
  }
}

// signed distance from the panel's surface, positive on the front side
// (panelside, smolsurface.c:3930)
template <bool GEN>
SMOLB_HDI double panel_sdist(const DevPanel &pn, const double x[3]) {
  if (pn.shape == 2 || (GEN && pn.shape == 4)) {
    double r2 = 0;
    for (int d = 0; d < 3; ++d) r2 += (x[d] - pn.center[d]) * (x[d] - pn.center[d]);
    return pn.front_sign * (sqrt(r2) - pn.radius);
  }
  if (GEN && pn.shape == 3) {
    double r[3];
    cyl_radial(pn, x, r);
    return pn.front_sign * (sqrt(dot3(r, r)) - pn.radius);
  }
  if (GEN && (pn.shape == 1 || pn.shape == 5)) {
    const double *o = pn.shape == 1 ? pn.pt[0] : pn.center;
    double w[3];
    for (int d = 0; d < 3; ++d) w[d] = x[d] - o[d];
    return dot3(w, pn.nrm);
  }
  return pn.front_sign * (x[pn.axis] - pn.pos);
}

// whether a point on a curved panel's full surface lies on the panel: the
// closed half of a hemisphere away from its open side; a cylinder between
// its end planes (smolsurface.c:4060-4065, Geo_PtInSlab)
SMOLB_HDI bool on_curved_part(const DevPanel &pn, const double x[3]) {
  double w[3];
  if (pn.shape == 4) {
    for (int d = 0; d < 3; ++d) w[d] = x[d] - pn.center[d];
    return dot3(w, pn.nrm) <= 0;
  }
  if (pn.shape == 3) {
    for (int d = 0; d < 3; ++d) w[d] = x[d] - pn.pt[0][d];
    const double s = dot3(w, pn.nrm);
    return s >= 0 && s <= pn.axlen;
  }
  return true;
}

// Crossings with the shapes other than rect and sphere.  Kernels are compiled
// in two surface forms: rect and sphere panels only (GEN false, the common
// case, whose registers the other shapes would otherwise raise), and every
// shape (GEN true).
// quadric with an open part: cyl (radial parts only) and hemi
SMOLB_HDI double cross_cyl_hemi(const DevPanel &pn, const double a[3], const double b[3], int &face) {
  double v[3], w[3], vq[3];
  for (int d = 0; d < 3; ++d) v[d] = b[d] - a[d];
  if (pn.shape == 3) {
    cyl_radial(pn, a, w);
    const double s = dot3(v, pn.nrm);
    for (int d = 0; d < 3; ++d) vq[d] = v[d] - s * pn.nrm[d];
  } else {
    for (int d = 0; d < 3; ++d) {
      w[d] = a[d] - pn.center[d];
      vq[d] = v[d];
    }
  }
  const double vv = dot3(vq, vq), wv = dot3(w, vq), ww = dot3(w, w);
  if (vv <= 0) return 2.0;
  const double c = ww - pn.radius * pn.radius;
  const double disc = wv * wv - vv * c;
  if (disc < 0) return 2.0;
  const double sq = sqrt(disc);
  const bool inside = c < 0;
  // the inside face is the back one when the front faces out
  const int face_in = pn.front_sign > 0 ? 1 : 0, face_out = 1 - face_in;
  const double t2 = (-wv + sq) / vv;  // exit from the full quadric
  double x[3];
  if (!inside) {
    const double t1 = (-wv - sq) / vv;  // entry
    if (!(t1 > 0 && t1 <= 1)) return 2.0;
    for (int d = 0; d < 3; ++d) x[d] = a[d] + t1 * v[d];
    if (on_curved_part(pn, x)) {
      face = face_out;
      return t1;
    }
    // entered through the open part: the exit may still hit the panel from
    // inside (smolsurface.c:4062-4069)
    if (!(t2 > 0 && t2 <= 1)) return 2.0;
    for (int d = 0; d < 3; ++d) x[d] = a[d] + t2 * v[d];
    if (!on_curved_part(pn, x)) return 2.0;
    face = face_in;
    return t2;
  }
  if (!(t2 > 0 && t2 <= 1)) return 2.0;
  for (int d = 0; d < 3; ++d) x[d] = a[d] + t2 * v[d];
  if (!on_curved_part(pn, x)) return 2.0;
  face = face_in;
  return t2;
}

// flat: tri and disk in the plane of their front normal
SMOLB_HDI double cross_tri_disk(const DevPanel &pn, const double a[3], const double b[3], int &face) {
  const double *o = pn.shape == 1 ? pn.pt[0] : pn.center;
  double w0[3], w1[3];
  for (int d = 0; d < 3; ++d) {
    w0[d] = a[d] - o[d];
    w1[d] = b[d] - o[d];
  }
  const double d0 = dot3(w0, pn.nrm), d1 = dot3(w1, pn.nrm);
  if (d0 == 0 || (d0 > 0) == (d1 > 0)) return 2.0;
  const double t = d0 / (d0 - d1);
  if (!(t > 0 && t <= 1)) return 2.0;
  double x[3];
  for (int d = 0; d < 3; ++d) x[d] = a[d] + t * (b[d] - a[d]);
  if (pn.shape == 5) {
    double r2 = 0;
    for (int d = 0; d < 3; ++d) r2 += (x[d] - pn.center[d]) * (x[d] - pn.center[d]);
    if (r2 > pn.radius * pn.radius) return 2.0;
  } else {
    // inside when on the inner side of all three edges (Geo_PtInTriangle2)
    for (int k = 0; k < 3; ++k) {
      const double *p = pn.pt[k], *q = pn.pt[(k + 1) % 3];
      const double e[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
      const double f[3] = {x[0] - p[0], x[1] - p[1], x[2] - p[2]};
      const double cr[3] = {e[1] * f[2] - e[2] * f[1], e[2] * f[0] - e[0] * f[2], e[0] * f[1] - e[1] * f[0]};
      if (dot3(cr, pn.nrm) < 0) return 2.0;
    }
  }
  face = d0 > 0 ? 0 : 1;
  return t;
}

// Crossing of segment a->b with a panel: t in (0,1] and the face hit, or
// t = 2 when the segment does not cross (smolsurface.c:4000 lineXpanel).
template <bool GEN>
SMOLB_HDI double panel_cross(const DevPanel &pn, const double a[3], const double b[3], int &face) {
  if (GEN && (pn.shape == 1 || pn.shape == 5)) return cross_tri_disk(pn, a, b, face);
  if (GEN && (pn.shape == 3 || pn.shape == 4)) return cross_cyl_hemi(pn, a, b, face);
  double v[3];
  for (int d = 0; d < 3; ++d) v[d] = b[d] - a[d];
  if (pn.shape == 2) {
    double w[3], vv = 0, wv = 0, ww = 0;
    for (int d = 0; d < 3; ++d) {
      w[d] = a[d] - pn.center[d];
      vv += v[d] * v[d];
      wv += w[d] * v[d];
      ww += w[d] * w[d];
    }
    if (vv <= 0) return 2.0;
    const double c = ww - pn.radius * pn.radius;
    const double disc = wv * wv - vv * c;
    if (disc < 0) return 2.0;
    const double sq = sqrt(disc);
    const bool inside = c < 0;
    const double t = inside ? (-wv + sq) / vv : (-wv - sq) / vv;
    if (!(t > 0 && t <= 1)) return 2.0;
    // arriving from inside: the inside face is the back one when front faces out
    face = (inside == (pn.front_sign > 0)) ? 1 : 0;
    return t;
  }
  const int ax = pn.axis;
  const double d0 = a[ax] - pn.pos, d1 = b[ax] - pn.pos;
  if (d0 == 0 || (d0 > 0) == (d1 > 0)) return 2.0;
  const double t = d0 / (d0 - d1);
  if (!(t > 0 && t <= 1)) return 2.0;
  for (int d = 0; d < 3; ++d) {
    if (d == ax) continue;
    const double x = a[d] + t * v[d];
    if (x < pn.lo[d] || x > pn.hi[d]) return 2.0;
  }
  face = ((d0 > 0) == (pn.front_sign > 0)) ? 0 : 1;
  return t;
}


// Device form of a panel from its definition (positions shifted by the
// system's low corner lo).
inline DevPanel make_dev_panel(const PanelSpec &ps, const double lo[3]) {
  DevPanel dp{};
  dp.shape = ps.shape;
  dp.axis = ps.axis;
  dp.front_sign = ps.front_sign;
  dp.pos = ps.pos - lo[ps.axis];
  for (int d = 0; d < 3; ++d) {
    dp.lo[d] = ps.lo[d] - lo[d];
    dp.hi[d] = ps.hi[d] - lo[d];
    dp.center[d] = ps.center[d] - lo[d];
  }
  dp.radius = ps.radius;
  for (int k = 0; k < 3; ++k)
    for (int d = 0; d < 3; ++d) dp.pt[k][d] = ps.pt[k][d] - lo[d];
  for (int d = 0; d < 3; ++d) dp.nrm[d] = ps.normal[d];
  dp.axlen = 0;
  if (ps.shape == 3)
    for (int d = 0; d < 3; ++d) dp.axlen += (dp.pt[1][d] - dp.pt[0][d]) * dp.nrm[d];
  dp.posf = (float)dp.pos;
  dp.radiusf = (float)dp.radius;
  dp.curved = (ps.shape == 2 || ps.shape == 3 || ps.shape == 4) ? 1 : 0;
  for (int d = 0; d < 3; ++d) {
    dp.centerf[d] = (float)dp.center[d];
    // screen reference point and unit vector: rect plane point and axis; tri
    // vertex and normal; disk centre and normal; sph / hemi centre and no
    // vector; cyl axis start and axis
    double p0 = 0, n0 = 0;
    if (ps.shape == 0) { p0 = d == ps.axis ? dp.pos : 0.0; n0 = d == ps.axis ? 1.0 : 0.0; }
    else if (ps.shape == 1 || ps.shape == 3) { p0 = dp.pt[0][d]; n0 = dp.nrm[d]; }
    else if (ps.shape == 5) { p0 = dp.center[d]; n0 = dp.nrm[d]; }
    else { p0 = dp.center[d]; n0 = 0.0; }
    dp.p0f[d] = (float)p0;
    dp.nrmf[d] = (float)n0;
  }
  dp.act_front = ps.action_front;
  dp.act_back = ps.action_back;
  dp.abs_front = ps.absorb_front_mask;
  dp.abs_back = ps.absorb_back_mask;
  dp.tr_front = ps.trans_front_mask;
  dp.tr_back = ps.trans_back_mask;
  dp.rf_front = ps.refl_front_mask;
  dp.rf_back = ps.refl_back_mask;
  dp.jp_front = ps.jump_front_mask;
  dp.jp_back = ps.jump_back_mask;
  for (int f = 0; f < 2; ++f) {
    dp.jump_pnl[f] = ps.jump_pnl[f];
    dp.jump_face[f] = ps.jump_face[f];
  }
  dp.srf = ps.srf;
  dp.nneigh = ps.nneigh < kMaxNeigh ? ps.nneigh : kMaxNeigh;
  for (int k = 0; k < dp.nneigh; ++k) dp.neigh[k] = ps.neigh[k];
  dp.neighhop = ps.neighhop;
  return dp;
}

// Device form of a compartment (points shifted by the system's low corner).
inline DevCmpt make_dev_cmpt(const CmptSpec &cs, const double lo[3]) {
  DevCmpt c{};
  c.npts = (int)cs.pts.size() < kMaxCmptPts ? (int)cs.pts.size() : kMaxCmptPts;
  for (int k = 0; k < c.npts; ++k)
    for (int d = 0; d < 3; ++d) c.pts[k][d] = (d < (int)cs.pts[k].size() ? cs.pts[k][d] : 0.0) - lo[d];
  c.panels = cs.panel_mask;
  c.ncl = (int)cs.logic.size() < kMaxCmptLogic ? (int)cs.logic.size() : kMaxCmptLogic;
  for (int l = 0; l < c.ncl; ++l) {
    c.clsym[l] = cs.logic[l].first;
    c.clcmpt[l] = cs.logic[l].second;
  }
  return c;
}

// posincompart (smolcomparts.c:119-190): x is in compartment `target` when
// the segment from x to one of its interior points crosses no panel of its
// surfaces, combined in order with its logic terms, each of which names an
// earlier compartment.  All compartments up to the target are evaluated in
// index order, so no recursion is needed.
SMOLB_HDI bool pos_in_cmpt(const DevCmpt *cm, int target, const DevPanel *panels, const double x[3]) {
  uint32_t in_mask = 0;
  for (int c = 0; c <= target; ++c) {
    const DevCmpt &q = cm[c];
    bool in = false;
    for (int k = 0; k < q.npts && !in; ++k) {
      bool cross = false;
      for (int pi = 0; pi < kMaxPanels && !cross; ++pi) {
        int f = 0;
        if (((q.panels >> pi) & 1u) && panel_cross<true>(panels[pi], x, q.pts[k], f) <= 1.0) cross = true;
      }
      if (!cross) in = true;
    }
    for (int l = 0; l < q.ncl; ++l) {
      const bool o = (in_mask >> q.clcmpt[l]) & 1u;
      switch (q.clsym[l]) {
        case 0: in = o; break;           // equal
        case 1: in = !o; break;          // equalnot
        case 2: in = in && o; break;     // and
        case 3: in = in || o; break;     // or
        case 4: in = in != o; break;     // xor
        case 5: in = in && !o; break;    // andnot
        default: in = in || !o; break;   // ornot
      }
    }
    if (in) in_mask |= 1u << c;
  }
  return (in_mask >> target) & 1u;
}

}  // namespace smolb
