// Panel geometry for surface-bound molecules: keeping a point on a panel's
// chosen side (fixpt2panel, smolsurface.c:4460), whether a point lies within
// a panel's outline (ptinpanel :4276), pulling it inside (movept2panel :4516),
// where a path leaves the panel (lineexitpanel :4105), the nearest point of a
// panel (closestpanelpt :4572), the outward normal of a panel edge
// (paneledgenormal :4166), the normal facing a given side (panelnormal
// :3967), and the rotation that carries a path across an edge onto a
// neighbouring panel (Sph_RotateVectWithNormals3D, Sphere.c:618).
//
// Shapes use the engine's panel form (DevPanel).  Rectangle edges are coded
// 1 / 2 for the low / high side along the first in-plane axis and 3 / 4
// along the second; triangle edges 1, 2, 3 run v0->v1, v1->v2, v2->v0; a
// disk and a hemisphere have the single edge 1 (the rim), a cylinder the
// edges 1 and 2 (the rims at its first and second axis end).  Edge code 0
// means "inside".
// Coordinates are relative to the system's low corner, FP64 throughout.
#pragma once

#include <float.h>
#include <math.h>

#include "panelgeom.cuh"

namespace smolb {

// Faces as in PanelFace (smoldyn.h:484).
constexpr int kFaceFront = 0, kFaceBack = 1, kFaceNone = 2;

// the two in-plane axes of a rectangle, ascending
SMOLB_HDI void rect_axes(const DevPanel &pn, int &u0, int &u1) {
  u0 = pn.axis == 0 ? 1 : 0;
  u1 = pn.axis == 2 ? 1 : 2;
}

// side of the panel a point is on, strict: front (dist > 0), back (< 0), or
// none exactly on it (panelside with strict set)
SMOLB_HDI int panel_side(const DevPanel &pn, const double x[3], double *dist) {
  const double s = panel_sdist<true>(pn, x);
  if (dist) *dist = s;
  return s > 0 ? kFaceFront : s < 0 ? kFaceBack : kFaceNone;
}

// normal at x toward `face` (front unless face is back)
SMOLB_HDI void face_normal(const DevPanel &pn, const double x[3], int face, double n[3]) {
  panel_normal<true>(pn, x, n);
  if (face == kFaceBack)
    for (int d = 0; d < 3; ++d) n[d] = -n[d];
}

// Move x onto the panel's surface and then just onto side `face` (none: on
// the surface), unless it is already on that side within eps.
SMOLB_HDI void fix_to_panel(const DevPanel &pn, double x[3], int face, double eps) {
  double dist;
  const int at = panel_side(pn, x, &dist);
  if ((at == face || face == kFaceNone) && fabs(dist) <= eps) return;
  double n[3];
  panel_normal<true>(pn, x, n);
  for (int d = 0; d < 3; ++d) x[d] -= dist * n[d];
  if (face == kFaceNone) return;
  const double sgn = face == kFaceFront ? 1.0 : -1.0;
  double f = 1.0;
  for (int k = 0; k < 64 && panel_side(pn, x, nullptr) != face; ++k, f *= 2.0)
    for (int d = 0; d < 3; ++d) x[d] += sgn * f * DBL_EPSILON * n[d];
}

// outward unit normal of triangle edge k (in the panel's plane)
SMOLB_HDI void tri_edge_out(const DevPanel &pn, int k, double o[3]) {
  const double *a = pn.pt[k], *b = pn.pt[(k + 1) % 3], *c = pn.pt[(k + 2) % 3];
  const double e[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  o[0] = e[1] * pn.nrm[2] - e[2] * pn.nrm[1];
  o[1] = e[2] * pn.nrm[0] - e[0] * pn.nrm[2];
  o[2] = e[0] * pn.nrm[1] - e[1] * pn.nrm[0];
  const double w[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  const double l = sqrt(dot3(o, o));
  const double s = (dot3(o, w) > 0 ? -1.0 : 1.0) / (l > 0 ? l : 1.0);
  for (int d = 0; d < 3; ++d) o[d] *= s;
}

SMOLB_HDI bool pt_in_panel(const DevPanel &pn, const double x[3]) {
  switch (pn.shape) {
    case 0: {
      int u0, u1;
      rect_axes(pn, u0, u1);
      return pn.lo[u0] <= x[u0] && x[u0] <= pn.hi[u0] && pn.lo[u1] <= x[u1] && x[u1] <= pn.hi[u1];
    }
    case 1:
      for (int k = 0; k < 3; ++k) {
        double o[3];
        tri_edge_out(pn, k, o);
        const double w[3] = {x[0] - pn.pt[k][0], x[1] - pn.pt[k][1], x[2] - pn.pt[k][2]};
        if (dot3(w, o) > 0) return false;
      }
      return true;
    case 2: return true;
    case 5: {
      double w[3];
      for (int d = 0; d < 3; ++d) w[d] = x[d] - pn.center[d];
      double l2 = dot3(w, w);
      if (l2 <= pn.radius * pn.radius) return true;
      const double s = dot3(w, pn.nrm);
      l2 -= s * s;
      return l2 <= pn.radius * pn.radius;
    }
    default: return on_curved_part(pn, x);  // cyl, hemi
  }
}

// nearest point of segment a-b to x (clamped), for the triangle outline
SMOLB_HDI void seg_nearest(const double a[3], const double b[3], const double x[3], double out[3], int *corner) {
  const double e[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const double w[3] = {x[0] - a[0], x[1] - a[1], x[2] - a[2]};
  const double l2 = dot3(e, e), t = dot3(e, w);
  *corner = 0;
  if (t <= 0) { for (int d = 0; d < 3; ++d) out[d] = a[d]; *corner = 1; return; }
  if (t >= l2) { for (int d = 0; d < 3; ++d) out[d] = b[d]; *corner = 2; return; }
  for (int d = 0; d < 3; ++d) out[d] = a[d] + t / l2 * e[d];
}

// Nearest point of a panel to x, and the edge it lies on (0: interior, or a
// shape without edges); points within `margin` of an edge count as on it.
SMOLB_HDI int closest_panel_pt(const DevPanel &pn, const double x[3], double out[3], double margin) {
  int edge = 0;
  switch (pn.shape) {
    case 0: {
      int u[2];
      rect_axes(pn, u[0], u[1]);
      for (int d = 0; d < 3; ++d) out[d] = x[d];
      out[pn.axis] = pn.pos;
      for (int q = 0; q < 2; ++q) {  // the second axis's edge wins at a corner
        const int a = u[q];
        if (pn.lo[a] + margin < x[a] && x[a] < pn.hi[a] - margin) continue;
        if (fabs(x[a] - pn.lo[a]) < fabs(x[a] - pn.hi[a])) { out[a] = pn.lo[a]; edge = 2 * q + 1; }
        else { out[a] = pn.hi[a]; edge = 2 * q + 2; }
      }
      return edge;
    }
    case 1: {
      double dots[3];
      for (int k = 0; k < 3; ++k) {
        double o[3];
        tri_edge_out(pn, k, o);
        const double w[3] = {x[0] - pn.pt[k][0], x[1] - pn.pt[k][1], x[2] - pn.pt[k][2]};
        dots[k] = dot3(w, o);
      }
      if (dots[0] <= 0 && dots[1] <= 0 && dots[2] <= 0) {
        const double w[3] = {x[0] - pn.pt[0][0], x[1] - pn.pt[0][1], x[2] - pn.pt[0][2]};
        const double s = dot3(w, pn.nrm);
        for (int d = 0; d < 3; ++d) out[d] = x[d] - s * pn.nrm[d];
        for (int k = 0; k < 3; ++k)
          if (dots[k] > -margin) return k + 1;
        return 0;
      }
      for (int k = 0; k < 3; ++k) {
        if (dots[k] <= 0) continue;
        int corner;
        seg_nearest(pn.pt[k], pn.pt[(k + 1) % 3], x, out, &corner);
        // a corner belongs to the edge that starts there (the reference's numbering)
        return corner == 2 ? (k + 1) % 3 + 1 : k + 1;
      }
      return 0;
    }
    case 2: {
      double w[3];
      for (int d = 0; d < 3; ++d) w[d] = x[d] - pn.center[d];
      const double l = sqrt(dot3(w, w));
      for (int d = 0; d < 3; ++d) out[d] = pn.center[d] + (l > 0 ? pn.radius / l : 0.0) * w[d];
      return 0;
    }
    case 5: {
      double w[3];
      for (int d = 0; d < 3; ++d) w[d] = x[d] - pn.center[d];
      const double s = dot3(w, pn.nrm);
      for (int d = 0; d < 3; ++d) w[d] -= s * pn.nrm[d];
      const double l = sqrt(dot3(w, w));
      double f = 1.0;
      if (l >= pn.radius - margin) { f = pn.radius / l; edge = 1; }
      for (int d = 0; d < 3; ++d) out[d] = pn.center[d] + f * w[d];
      return edge;
    }
    case 3: {  // cylinder: the nearest point of its side, an end rim within margin (Geo_NearestCylinderPt)
      double w[3];
      for (int d = 0; d < 3; ++d) w[d] = x[d] - pn.pt[0][d];
      double s = dot3(w, pn.nrm) / pn.axlen;  // axial fraction
      const double m = margin / pn.axlen;
      if (s <= m) { s = 0; edge = 1; }
      else if (s >= 1 - m) { s = 1; edge = 2; }
      double rad[3];
      cyl_radial(pn, x, rad);
      const double l = sqrt(dot3(rad, rad));
      for (int d = 0; d < 3; ++d) out[d] = pn.pt[0][d] + s * pn.axlen * pn.nrm[d] + (l > 0 ? pn.radius / l : 0.0) * rad[d];
      return edge;
    }
    case 4: {  // hemisphere: the sphere's nearest point, or the rim's (Geo_NearestRingPt)
      double w[3];
      for (int d = 0; d < 3; ++d) w[d] = x[d] - pn.center[d];
      const double s = dot3(w, pn.nrm);
      if (s < -margin) {
        const double l = sqrt(dot3(w, w));
        for (int d = 0; d < 3; ++d) out[d] = pn.center[d] + (l > 0 ? pn.radius / l : 0.0) * w[d];
        return 0;
      }
      for (int d = 0; d < 3; ++d) w[d] -= s * pn.nrm[d];
      const double l = sqrt(dot3(w, w));
      for (int d = 0; d < 3; ++d) out[d] = pn.center[d] + (l > 0 ? pn.radius / l : 0.0) * w[d];
      return 1;
    }
    default:
      for (int d = 0; d < 3; ++d) out[d] = x[d];
      return 0;
  }
}

// Pull x inside the panel's outline by at least `margin` (movept2panel).
SMOLB_HDI void move_into_panel(const DevPanel &pn, double x[3], double margin) {
  if (pn.shape == 0) {
    int u[2];
    rect_axes(pn, u[0], u[1]);
    for (int q = 0; q < 2; ++q) {
      const int a = u[q];
      const double lo = pn.lo[a] + margin, hi = pn.hi[a] - margin;
      if (x[a] < lo) x[a] = lo;
      else if (x[a] > hi) x[a] = hi;
    }
  } else if (pn.shape == 1) {
    // nearest point of the triangle shrunk toward its centroid by margin
    if (pt_in_panel(pn, x)) return;
    double c[3], v[3][3];
    for (int d = 0; d < 3; ++d) c[d] = (pn.pt[0][d] + pn.pt[1][d] + pn.pt[2][d]) / 3.0;
    for (int k = 0; k < 3; ++k) {
      double w[3];
      for (int d = 0; d < 3; ++d) w[d] = c[d] - pn.pt[k][d];
      const double l = sqrt(dot3(w, w));
      for (int d = 0; d < 3; ++d) v[k][d] = pn.pt[k][d] + (l > 0 ? margin / l : 0.0) * w[d];
    }
    DevPanel sh = pn;
    for (int k = 0; k < 3; ++k)
      for (int d = 0; d < 3; ++d) sh.pt[k][d] = v[k][d];
    double out[3];
    closest_panel_pt(sh, x, out, 0.0);
    const double w[3] = {x[0] - out[0], x[1] - out[1], x[2] - out[2]};
    const double s = dot3(w, pn.nrm);  // keep the distance from the plane
    for (int d = 0; d < 3; ++d) x[d] = out[d] + s * pn.nrm[d];
  } else if (pn.shape == 5) {
    double w[3];
    for (int d = 0; d < 3; ++d) w[d] = x[d] - pn.center[d];
    const double s = dot3(w, pn.nrm);
    for (int d = 0; d < 3; ++d) w[d] -= s * pn.nrm[d];
    const double l = sqrt(dot3(w, w)), r = pn.radius - margin;
    if (l > r && l > 0)
      for (int d = 0; d < 3; ++d) x[d] -= (1.0 - r / l) * w[d];
  } else if (pn.shape == 4) {
    double w[3];
    for (int d = 0; d < 3; ++d) w[d] = x[d] - pn.center[d];
    const double s = dot3(w, pn.nrm);
    if (s > 0)
      for (int d = 0; d < 3; ++d) x[d] -= s * pn.nrm[d] + margin;
  } else if (pn.shape == 3) {  // between the end planes, margin inside (Geo_NearestSlabPt)
    double w[3];
    for (int d = 0; d < 3; ++d) w[d] = x[d] - pn.pt[0][d];
    const double s = dot3(w, pn.nrm);
    const double lo = margin, hi = pn.axlen - margin;
    const double t = s < lo ? lo : s > hi ? hi : s;
    for (int d = 0; d < 3; ++d) x[d] += (t - s) * pn.nrm[d];
  }
}

// Where the path a->b (a inside the outline) leaves the panel, and through
// which edge.  Returns 1 (nothing computed) when a == b.
SMOLB_HDI int line_exit_panel(const DevPanel &pn, const double a[3], const double b[3], double out[3], int *edge) {
  if (a[0] == b[0] && a[1] == b[1] && a[2] == b[2]) return 1;
  *edge = 1;
  double t = 0;
  if (pn.shape == 0) {
    int u[2];
    rect_axes(pn, u[0], u[1]);
    double tq[2];
    int eq[2];
    for (int q = 0; q < 2; ++q) {
      const int ax = u[q];
      const double dx = b[ax] - a[ax];
      if (dx == 0) { tq[q] = INFINITY; eq[q] = 2 * q + 2; continue; }
      const double tl = (pn.lo[ax] - a[ax]) / dx, th = (pn.hi[ax] - a[ax]) / dx;
      if (th > tl) { tq[q] = th; eq[q] = 2 * q + 2; }
      else { tq[q] = tl; eq[q] = 2 * q + 1; }
    }
    const int q = (tq[1] < tq[0] && b[u[1]] != a[u[1]]) || b[u[0]] == a[u[0]] ? 1 : 0;
    t = tq[q];
    *edge = eq[q];
  } else if (pn.shape == 1) {
    const double v[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    double tk[3];
    for (int k = 0; k < 3; ++k) {
      double o[3];
      tri_edge_out(pn, k, o);
      const double dv = dot3(o, v);
      const double w[3] = {pn.pt[k][0] - a[0], pn.pt[k][1] - a[1], pn.pt[k][2] - a[2]};
      tk[k] = dv > 0 ? dot3(w, o) / dv : INFINITY;
    }
    // ties go to the second edge over the first, and to either over the third
    int k = tk[0] < tk[1] ? 0 : 1;
    if (tk[2] < tk[k]) k = 2;
    t = tk[k];
    *edge = k + 1;
  } else if (pn.shape == 3) {
    // cylinder: through the end the path heads for, where it meets that end's
    // plane, taken to the rim (Geo_LineExitCylinder)
    const double v[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double dv = dot3(v, pn.nrm);
    const int end = dv > 0 ? 2 : 1;
    double c[3];
    for (int d = 0; d < 3; ++d) c[d] = pn.pt[end - 1][d];
    const double w[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    t = dv != 0 ? dot3(w, pn.nrm) / dv : 0.0;
    double q[3];
    for (int d = 0; d < 3; ++d) q[d] = a[d] + t * v[d];
    double rad[3];  // out to that end's rim
    cyl_radial(pn, q, rad);
    const double l = sqrt(dot3(rad, rad));
    for (int d = 0; d < 3; ++d) out[d] = c[d] + (l > 0 ? pn.radius / l : 0.0) * rad[d];
    *edge = end;
    return 0;
  } else if (pn.shape == 4) {
    // hemisphere: where the path meets the rim's plane, out to the rim
    // (Geo_LineExitHemisphere)
    const double v[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double w[3] = {pn.center[0] - a[0], pn.center[1] - a[1], pn.center[2] - a[2]};
    const double dv = dot3(v, pn.nrm);
    t = dv != 0 ? dot3(w, pn.nrm) / dv : 0.0;
    double q[3];
    for (int d = 0; d < 3; ++d) q[d] = a[d] + t * v[d] - pn.center[d];
    const double l = sqrt(dot3(q, q));
    for (int d = 0; d < 3; ++d) out[d] = pn.center[d] + (l > 0 ? pn.radius / l : 0.0) * q[d];
    *edge = 1;
    return 0;
  } else {  // disk (rim as a sphere of the disk's radius)
    double v[3], w[3];
    for (int d = 0; d < 3; ++d) { v[d] = b[d] - a[d]; w[d] = pn.center[d] - a[d]; }
    const double qa = dot3(v, v), qb = -2.0 * dot3(w, v), qc = dot3(w, w) - pn.radius * pn.radius;
    double disc = qb * qb - 4 * qa * qc;
    disc = disc <= 0 ? 0 : sqrt(disc);
    t = (-qb + disc) / (2 * qa);
  }
  for (int d = 0; d < 3; ++d) out[d] = a[d] + t * (b[d] - a[d]);
  return 0;
}

// outward in-plane unit normal of a panel edge at edge point e
SMOLB_HDI void panel_edge_normal(const DevPanel &pn, const double e[3], int edge, double n[3]) {
  if (edge == 0) edge = 1;
  n[0] = n[1] = n[2] = 0;
  if (pn.shape == 0) {
    int u[2];
    rect_axes(pn, u[0], u[1]);
    n[u[(edge - 1) / 2]] = (edge % 2) ? -1.0 : 1.0;
  } else if (pn.shape == 1) {
    tri_edge_out(pn, (edge - 1) % 3, n);
  } else if (pn.shape == 3) {  // cylinder ends: along the axis, outward
    for (int d = 0; d < 3; ++d) n[d] = (edge == 2 ? 1.0 : -1.0) * pn.nrm[d];
  } else if (pn.shape == 4) {  // hemisphere rim: out of the open side
    for (int d = 0; d < 3; ++d) n[d] = pn.nrm[d];
  } else {
    for (int d = 0; d < 3; ++d) n[d] = e[d] - pn.center[d];
    if (pn.shape == 5) {
      const double s = dot3(n, pn.nrm);
      for (int d = 0; d < 3; ++d) n[d] -= s * pn.nrm[d];
    }
    const double l = sqrt(dot3(n, n));
    for (int d = 0; d < 3; ++d) n[d] = l > 0 ? n[d] / l : 0.0;
  }
}

// Rotate p2 about p1 by the rotation that takes unit normal `oldn` to `newn`
// (axis oldn x newn).  sign +1 / -1 selects the rotation whose cosine is
// positive / negative (the supplementary one otherwise), 0 the direct one.
SMOLB_HDI void rotate_with_normals(const double p1[3], const double p2[3], double out[3], const double oldn[3],
                                   const double newn[3], int sign) {
  double c = dot3(oldn, newn);
  double ss = 1.0;
  if ((sign == 1 && c < 0) || (sign == -1 && c >= 0)) { c = -c; ss = -1.0; }
  const double eps = 1e-14;
  const double x[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
  if (c > -1 + eps && c < 1 - eps) {
    double ax[3] = {oldn[1] * newn[2] - oldn[2] * newn[1], oldn[2] * newn[0] - oldn[0] * newn[2],
                    oldn[0] * newn[1] - oldn[1] * newn[0]};
    double s = sqrt(dot3(ax, ax));
    if (s >= eps) {
      for (int d = 0; d < 3; ++d) ax[d] /= s;
      s *= ss;
      // Rodrigues: R x = c x + s (ax cross x) + (1 - c)(ax . x) ax
      const double cr[3] = {ax[1] * x[2] - ax[2] * x[1], ax[2] * x[0] - ax[0] * x[2], ax[0] * x[1] - ax[1] * x[0]};
      const double ad = dot3(ax, x);
      for (int d = 0; d < 3; ++d) out[d] = p1[d] + c * x[d] + s * cr[d] + (1.0 - c) * ad * ax[d];
      return;
    }
  }
  if (c > 0)
    for (int d = 0; d < 3; ++d) out[d] = p2[d];
  else
    for (int d = 0; d < 3; ++d) out[d] = p1[d] - x[d];
}

}  // namespace smolb
