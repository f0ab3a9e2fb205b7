// gdem_contact_common.cuh -- narrow-phase geometry and the HODC force law in
// FP64, shared by the FP64-mode contact kernels (and by the wall contacts of
// the FP32-split mode).  Every expression keeps the operation order of the
// reference functions cited beside it.
#pragma once
#include "gdem_device.cuh"
#include "gdem_gjk.cuh"

namespace gdem {

struct Contact64 {
  d3 point, overlap;
  double dist;
  bool contact;
  bool error;
  int gjk_iters = 0;     // GJK iterations spent on this pair (0: no GJK call)
};

// GJK work of one thread of a force kernel (convex systems): calls,
// iterations and the most iterations of one call; flushed once per warp.
struct GjkTally {
  int calls = 0, iters = 0, maxit = 0;
  __device__ __forceinline__ void add(int it) {
    if (it > 0) { ++calls; iters += it; maxit = max(maxit, it); }
  }
  // every lane of the warp calls this
  __device__ __forceinline__ void flush(unsigned long long* out) const {
    const unsigned full = 0xffffffffu;
    const int c = __reduce_add_sync(full, calls), i = __reduce_add_sync(full, iters);
    const int m = __reduce_max_sync(full, (unsigned)maxit);
    if ((threadIdx.x & 31) == 0 && c) {
      atomicAdd(out, (unsigned long long)c);
      atomicAdd(out + 1, (unsigned long long)i);
      atomicMax(out + 2, (unsigned long long)m);
    }
  }
};

// Overlap statistics of one thread's contacts (AppCollision::
// addToContactsFeatures, Base/src/AppCollision.cpp:159-179), flushed once
// per warp into the system's ContactStats.
struct StatsTally {
  double sum = 0., mx = 0.;
  int count = 0;
  __device__ __forceinline__ void add(double dist) {
    const double o = -dist;
    sum += o;
    mx = fmax(mx, o);
    ++count;
  }
  // every lane of the warp calls this
  __device__ __forceinline__ void flush(ContactStats* cs, int epoch) const {
    const unsigned full = 0xffffffffu;
    const int c = __reduce_add_sync(full, count);
    if (!c || !cs) return;
    double s = sum, m = mx;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_down_sync(full, s, o);
      m = fmax(m, __shfl_down_sync(full, m, o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&cs->sum, s);
      atomicAdd(&cs->count, (unsigned long long)c);
      const unsigned long long bits = (unsigned long long)__double_as_longlong(m);
      // the first evaluation at which the largest overlap was reached: later
      // evaluations only write when they exceed it
      if (atomicMax(&cs->max_bits, bits) < bits) cs->max_epoch = epoch;
    }
  }
};

// ClosestPointSPHERESPHERE (Geometry/src/RigidBodyWithCrust.cpp:596-639).
// On overlap >= crustA + crustB the reference retries with a 10x crust
// shrink (ClosestPoint_ErreurHandling, :534-588): for spheres the imposed
// overlap is crustA + crustB along the centre line, the contact point the
// midpoint of the shrunk spheres' closest points.
__device__ __forceinline__ Contact64 sphereSphere64(d3 xa, double ra, double ca, d3 xb,
                                                    double rb, double cb) {
  Contact64 c;
  c.error = false;
  d3 AB = xb - xa;
  double distance = norm(AB) - (ra + rb);
  c.dist = distance;
  if (distance > 0.) { c.contact = false; return c; }
  c.contact = true;
  double nAB = norm(AB);
  if (-distance >= ca + cb) {
    c.error = true;
    double sa = (ra - 10. * ca) / ra, sb = (rb - 10. * cb) / rb;
    double ras = ra * (sa > 0.5 ? sa : 0.5), rbs = rb * (sb > 0.5 ? sb : 0.5);
    d3 u = AB / nAB;
    d3 pA = xa + ras * u, pB = xb - rbs * u;
    d3 ba = pA - pB;
    ba = ba / norm(ba);
    double imp = 1. * (ca + cb);
    c.point = pA / 2.0 + pB / 2.0;
    c.overlap = imp * ba;
    c.dist = -imp;
    return c;
  }
  c.point = xa + ((ra + 0.5 * distance) * AB) / nAB;
  c.overlap = distance * (AB / nAB);
  return c;
}

// Box corners in Box's numbering (Geometry/src/Box.cpp constructor).
__device__ __forceinline__ d3 boxCorner(d3 e, int n) {
  double sx = (n == 1 || n == 2 || n == 5 || n == 6) ? 1. : -1.;
  double sy = (n >= 4) ? 1. : -1.;
  double sz = (n == 2 || n == 3 || n == 6 || n == 7) ? 1. : -1.;
  return mk(sx * e.x, sy * e.y, sz * e.z);
}
__device__ __forceinline__ double comp(d3 a, int d) { return d == 0 ? a.x : (d == 1 ? a.y : a.z); }
__device__ __forceinline__ void setc(d3& a, int d, double v) { if (d == 0) a.x = v; else if (d == 1) a.y = v; else a.z = v; }

// Box::ContactCornerSPHERE / ContactEdgeSPHERE (Box.cpp:690-742)
__device__ __forceinline__ d3 contactCorner(d3 e, d3 c, double r, int n, double& ov) {
  d3 cp = mk(0., 0., 0.);
  d3 dist = c - boxCorner(e, n);
  double nd = norm(dist);
  if (nd < r) { ov = nd - r; cp = c - (1. + 0.5 * ov / nd) * dist; }
  return cp;
}
__device__ __forceinline__ d3 contactEdge(d3 e, d3 c, double r, int n, int dir, double& ov) {
  d3 cp = mk(0., 0., 0.), proj = c;
  d3 cn = boxCorner(e, n);
  setc(proj, dir, comp(cn, dir));
  d3 dist = proj - cn;
  double nd = norm(dist);
  if (nd < r) { ov = nd - r; cp = c - (1. + 0.5 * ov / nd) * dist; }
  return cp;
}

// Box::IntersectionPointSPHERE (Box.cpp:466-676) in the box frame.
__device__ inline d3 boxSphere(d3 e, d3 c, double r, double& ov) {
  d3 cp = mk(0., 0., 0.);
  double gx = c.x, gy = c.y, gz = c.z;
  ov = 1.;
  if (gx > e.x) {
    if (gy > e.y) {
      if (gz > e.z) cp = contactCorner(e, c, r, 6, ov);
      else if (gz < -e.z) cp = contactCorner(e, c, r, 5, ov);
      else cp = contactEdge(e, c, r, 5, 2, ov);
    } else if (gy < -e.y) {
      if (gz > e.z) cp = contactCorner(e, c, r, 2, ov);
      else if (gz < -e.z) cp = contactCorner(e, c, r, 1, ov);
      else cp = contactEdge(e, c, r, 1, 2, ov);
    } else {
      if (gz > e.z) cp = contactEdge(e, c, r, 6, 1, ov);
      else if (gz < -e.z) cp = contactEdge(e, c, r, 1, 1, ov);
      else { double nd = gx - e.x; if (nd < r) { ov = nd - r; cp = mk(e.x + 0.5 * ov, c.y, c.z); } }
    }
  } else if (gx < -e.x) {
    if (gy > e.y) {
      if (gz > e.z) cp = contactCorner(e, c, r, 7, ov);
      else if (gz < -e.z) cp = contactCorner(e, c, r, 4, ov);
      else cp = contactEdge(e, c, r, 4, 2, ov);
    } else if (gy < -e.y) {
      if (gz > e.z) cp = contactCorner(e, c, r, 3, ov);
      else if (gz < -e.z) cp = contactCorner(e, c, r, 0, ov);
      else cp = contactEdge(e, c, r, 0, 2, ov);
    } else {
      if (gz > e.z) cp = contactEdge(e, c, r, 3, 1, ov);
      else if (gz < -e.z) cp = contactEdge(e, c, r, 0, 1, ov);
      else { double nd = -e.x - gx; if (nd < r) { ov = nd - r; cp = mk(-e.x - 0.5 * ov, c.y, c.z); } }
    }
  } else {
    if (gy > e.y) {
      if (gz > e.z) cp = contactEdge(e, c, r, 6, 0, ov);
      else if (gz < -e.z) cp = contactEdge(e, c, r, 4, 0, ov);
      else { double nd = gy - e.y; if (nd < r) { ov = nd - r; cp = mk(c.x, e.y + 0.5 * ov, c.z); } }
    } else if (gy < -e.y) {
      if (gz > e.z) cp = contactEdge(e, c, r, 3, 0, ov);
      else if (gz < -e.z) cp = contactEdge(e, c, r, 0, 0, ov);
      else { double nd = -e.y - gy; if (nd < r) { ov = nd - r; cp = mk(c.x, -e.y - 0.5 * ov, c.z); } }
    } else {
      if (gz > e.z) { double nd = gz - e.z; if (nd < r) { ov = nd - r; cp = mk(c.x, c.y, e.z + 0.5 * ov); } }
      else if (gz < -e.z) { double nd = -e.z - gz; if (nd < r) { ov = nd - r; cp = mk(c.x, c.y, -e.z - 0.5 * ov); } }
      else ov = -10000.;
    }
  }
  return cp;
}

// ClosestPointSPHEREBOX with the sphere first (RigidBodyWithCrust.cpp:
// 647-689), for an axis-aligned wall: w2b(p) = p - centre, b2w(p) = p + centre.
__device__ __forceinline__ Contact64 sphereWall64(d3 xa, double ra, double ca, WallDesc const& w) {
  Contact64 c;
  c.contact = false;
  c.error = false;
  d3 local = xa - mk(w.centre[0], w.centre[1], w.centre[2]);
  double ov = 0.;
  d3 cpl = boxSphere(mk(w.extent[0], w.extent[1], w.extent[2]), local, ra, ov);
  c.dist = ov;
  if (ov < 0.) {
    if (-ov >= ca + w.crust) { c.error = true; return c; }
    d3 contact = cpl + mk(w.centre[0], w.centre[1], w.centre[2]);
    d3 AB = contact - xa;
    c.point = contact;
    c.overlap = (ov / norm(AB)) * AB;
    c.contact = true;
  }
  return c;
}

// RigidBodyWithCrust::ClosestPoint, general branch (RigidBodyWithCrust.cpp:
// 277-351): bounding-sphere test on the circumscribed radii, GJK between the
// crust-shrunk bodies, overlap = distance - crustA - crustB along the
// witness direction, contact at the witness midpoint.  A GJK distance below
// 1e-10 is the reference's ContactError (it then retries with a 10x crust
// shrink); here it raises the overlap status and no force is applied.
// curA, curB: the bodies' current polyhedron vertices (updated by the GJK).
// early: the closest-point search stops once the shrunk bodies are known to
// be farther apart than the sum of the crusts (no contact: the same decision,
// without the witness points and with the polyhedron vertices the shortened
// search reached).
__device__ inline Contact64 convexContact64(ConvexRef const& a, XForm64 const& a2w, double Ra,
                                            double ca, ConvexRef const& b, XForm64 const& b2w,
                                            double Rb, double cb, int& curA, int& curB,
                                            bool early = false) {
  Contact64 c;
  c.contact = false;
  c.error = false;
  c.dist = 1.;
  d3 gg = a2w.o - b2w.o;
  if (!(norm(gg) < Ra + Rb)) return c;
  d3 pA, pB;
  int it = 0;
  bool separated = false;
  // a relative margin far above the rounding of the bound
  const double sep = early ? (ca + cb) * (1. + 1.e-9) : 0.;
  double distance = closestPoints64(a, a2w, b, b2w, pA, pB, &it, curA, curB, sep, &separated);
  c.gjk_iters = it;
  if (separated) return c;
  if (distance < 1.0e-10) { c.error = true; return c; }
  d3 ba = pA - pB;
  d3 contact = pA / 2.0 + pB / 2.0;
  d3 ov = ba / distance;
  ov.x = fabs(ov.x) < 1.0e-10 ? 0. : ov.x;
  ov.y = fabs(ov.y) < 1.0e-10 ? 0. : ov.y;
  ov.z = fabs(ov.z) < 1.0e-10 ? 0. : ov.z;
  ov = ov * (ca + cb - distance);
  distance = distance - (ca + cb);
  c.point = contact;
  c.overlap = ov;
  c.dist = distance;
  c.contact = true;
  return c;
}

__device__ __forceinline__ ConvexRef convexOf(TypeDesc const& t, const double* verts,
                                              const int* adj_off, const int* adj) {
  ConvexRef r;
  r.kind = t.shape;
  r.radius = t.radius;
  r.extent = mk(t.extent[0], t.extent[1], t.extent[2]);
  r.verts = verts ? verts + 3 * t.poly_begin : nullptr;
  r.nverts = t.poly_count;
  r.adj_off = adj_off ? adj_off + t.poly_begin : nullptr;
  r.adj = adj;
  return r;
}
__device__ __forceinline__ ConvexRef convexOf(TypeDesc const& t, DevState const& S) {
  return convexOf(t, S.poly_verts, S.poly_adj_off, S.poly_adj);
}
__device__ __forceinline__ ConvexRef convexOf(WallDesc const& w) {
  ConvexRef r;
  r.kind = 1;
  r.radius = w.radius;
  r.extent = mk(w.extent[0], w.extent[1], w.extent[2]);
  r.verts = nullptr;
  r.nverts = 0;
  r.adj_off = nullptr;
  r.adj = nullptr;
  return r;
}

// Which partner the reference takes as p0 (the body whose InterAction runs)
// for a pair t, u (t the lower ID) without a periodic image shift: its force
// loop (LinkedCell::ComputeForces, Base/src/LinkedCell.cpp:1019-1103) takes
// each particle with the later particles of its own cell and the particles of
// the 13 cells of its contact neighbourhood (setCellContactNeighborhood,
// :958-984), which are exactly the adjacent cells with a larger cell number
// (j nbk nbi + k nbi + i); within a cell the earlier particle of the cell's
// list, which is the lower ID after a reload.  Returns true when u is p0.
// The contact law is evaluated with the reference's p0 so that its FP64
// result has the reference's rounding.
__device__ __forceinline__ int referenceCellNumber(GridDesc const& g, d3 x) {
  const int i = (int)floor((x.x - g.lc_origin[0]) / g.edge[0]);
  const int j = (int)floor((x.y - g.lc_origin[1]) / g.edge[1]);
  const int k = (int)floor((x.z - g.lc_origin[2]) / g.edge[2]);
  return j * g.nb[2] * g.nb[0] + k * g.nb[0] + i;
}
__device__ __forceinline__ bool referenceFlip(GridDesc const& g, d3 xt, d3 xu, const int* sh) {
  // across a periodic boundary the reference pairs a particle with the other's
  // clone in its ghost cells; there the lower ID stays p0
  if (sh[0] | sh[1] | sh[2]) return false;
  return referenceCellNumber(g, xu) < referenceCellNumber(g, xt);
}

// The current polyhedron vertex of the particle in slot s at the start of
// this evaluation (Polyhedron::m_curr_vertex), and the record of the one a
// GJK call left: of all the calls of an evaluation on one particle, the one
// of its last row entry (priority = entry + 1, below kWallPriority) or of its
// walls (after every entry) is kept, so the choice does not depend on the
// order in which the calls run; the leapfrog kernel makes it the current
// vertex.
__device__ __forceinline__ int startVertex(DevState const& S, TypeDesc const& t, int s) {
  return t.shape == 2 ? S.curv[s] : 0;
}
constexpr int kWallPriority = 0x7FFF;
__device__ __forceinline__ void recordVertex(DevState const& S, TypeDesc const& t, int s,
                                             int priority, int vertex) {
  if (t.shape == 2)
    atomicMax(&S.curv_next[s], (priority << 16) | (vertex & 0xFFFF));
}

// HookeMemoryContactForceModel::computeTangentialVector (:54-65)
__device__ __forceinline__ d3 tangent64(ModelDesc const& m, double n_t, d3 ut, d3 kd) {
  if (norm(ut) > 0.001) return (-ut) / norm(ut);
  d3 s = kd + n_t * ut;
  if ((norm(kd) > m.epst || norm(n_t * ut) > m.epst) && norm(s) > m.epst) return (-s) / norm(s);
  return mk(0., 0., 0.);
}

// HookeMemoryContactForceModel::performForcesCalculus (:72-193) seen from p0.
// kd/pn/sp hold the stored memory on entry (valid when existed) and the
// updated memory on exit.  f is the force on p0 (p1 receives -f), mr the
// rolling torque on p0.
__device__ inline void hodc64(ModelDesc const& m, double dt, d3 pcp, d3 pen,
                              d3 x0, d3 v0, d3 w0, double m0, double rad0,
                              d3 x1, d3 v1, d3 w1, double m1, double rad1,
                              bool existed, d3& kd, d3& pn, d3& sp, d3& f, d3& mr) {
  d3 normal = pen;
  normal = normal / norm(normal);
  normal.x = fabs(normal.x) < 1.0e-10 ? 0. : normal.x;     // Group3::round
  normal.y = fabs(normal.y) < 1.0e-10 ? 0. : normal.y;
  normal.z = fabs(normal.z) < 1.0e-10 ? 0. : normal.z;
  d3 va = v0 + cross(w0, pcp - x0);
  d3 vb = v1 + cross(w1, pcp - x1);
  d3 tmpV = va - vb;
  d3 v_n = normal * dot(tmpV, normal);
  d3 v_t = tmpV - v_n;
  d3 delFN = m.kn * pen;
  double avmass = 1. / (1. / m0 + 1. / m1);
  double gamman = -2. * m.beta * sqrt(avmass * m.kn);
  delFN = delFN - gamman * v_n;
  double normFN = norm(delFN);
  double etat = m.etat == -1. ? -m.beta * sqrt(m.kn / avmass) : m.etat;
  double gammat = 2. * etat * avmass;
  d3 viscousFT = -gammat * v_t;
  dq qrot = qmk(mk(0., 0., 0.), 0.);
  if (!existed) { kd = mk(0., 0., 0.); sp = mk(0., 0., 0.); }
  else {
    qrot = rotFromTwoVectors(pn, normal);
    kd = rotateVector(qrot, kd);
  }
  kd = kd + (dt * m.kt) * v_t;
  pn = normal;
  d3 tij = tangent64(m, gammat, v_t, kd);
  double normFT = norm(-kd + viscousFT);
  d3 delFT;
  if (normFT <= m.muc * normFN) delFT = norm(-kd + viscousFT) * tij;
  else {
    if (m.kt != 0.) kd = ((-m.muc * normFN) * tij + viscousFT) / m.kt;
    delFT = (m.muc * normFN) * tij;
  }
  mr = mk(0., 0., 0.);
  if (m.rolling) {
    double Req = 1. / (1. / rad0 + 1. / rad1);
    double kr = 3. * m.kn * m.mur * m.mur * Req * Req;
    double etar = 3. * gamman * m.mur * m.mur * Req * Req;
    double maxM = m.mur * Req * normFN;
    d3 wrel = w0 - w1;
    if (existed) sp = rotateVector(qrot, sp);
    sp = sp - (kr * dt) * wrel;
    double nM = norm(sp);
    if (nM > maxM) sp = sp * (maxM / nM);
    mr = sp - (m.etarpf * etar) * wrel;
  }
  f = 1. * (delFN + delFT);
}

// HookeContactForceModel::performForcesCalculus (HookeContactForceModel.cpp:
// 44-121): the normal law of hodc64 without tangential memory; the viscous
// tangential force is capped at muc |Fn|; with kr != 0 a rolling-resistance
// moment -kr Req |Fn| |w0 x (x0 - pc) - w1 x (x1 - pc)| / |w0 - w1| (w0 - w1).
__device__ inline void hooke64(ModelDesc const& m, d3 pcp, d3 pen, d3 x0, d3 v0, d3 w0,
                               double m0, double rad0, d3 x1, d3 v1, d3 w1, double m1,
                               double rad1, d3& f, d3& mr) {
  d3 normal = pen;
  normal = normal / norm(normal);
  normal.x = fabs(normal.x) < 1.0e-10 ? 0. : normal.x;     // Group3::round
  normal.y = fabs(normal.y) < 1.0e-10 ? 0. : normal.y;
  normal.z = fabs(normal.z) < 1.0e-10 ? 0. : normal.z;
  d3 va = v0 + cross(w0, pcp - x0);
  d3 vb = v1 + cross(w1, pcp - x1);
  d3 tmpV = va - vb;
  d3 v_n = normal * dot(tmpV, normal);
  d3 v_t = tmpV - v_n;
  d3 delFN = m.kn * pen;
  double avmass = 1. / (1. / m0 + 1. / m1);
  double gamman = -2. * m.beta * sqrt(avmass * m.kn);
  delFN = delFN - gamman * v_n;
  double normFN = norm(delFN);
  double etat = m.etat == -1. ? -m.beta * sqrt(m.kn / avmass) : m.etat;
  double gammat = 2. * etat * avmass;
  d3 delFT = -gammat * v_t;
  double fn = m.muc * normFN;
  double ft = norm(delFT);
  if (fn < ft) {
    double normv_t = norm(v_t);
    d3 tangent = mk(0., 0., 0.);
    if (normv_t > 1.0e-10) tangent = (-v_t) / normv_t;
    delFT = tangent * fn;
  }
  mr = mk(0., 0., 0.);
  if (m.kr != 0.) {
    d3 wrel = w0 - w1;
    double normwrel = norm(wrel);
    double normwtrel = norm(cross(w0, x0 - pcp) - cross(w1, x1 - pcp));
    if (normwrel > 1.0e-10) {
      double Req = 1. / (1. / rad0 + 1. / rad1);
      mr = -(m.kr * Req * normFN * normwtrel / normwrel) * wrel;
    }
  }
  f = 1. * (delFN + delFT);
}

}  // namespace gdem
