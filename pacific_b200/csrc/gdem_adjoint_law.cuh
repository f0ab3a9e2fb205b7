// gdem_adjoint_law.cuh -- the sphere contact geometry and the Hooke /
// HookeMemory force law written for a generic scalar (double or Dual<N>), so
// that the adjoint engine can differentiate it.  The expressions are those of
// the production FP64 path (gdem_contact_common.cuh) and of the reference:
//   ClosestPointSPHERESPHERE   (Geometry/src/RigidBodyWithCrust.cpp:596-639)
//   ClosestPointSPHEREBOX and Box::IntersectionPointSPHERE
//                              (RigidBodyWithCrust.cpp:647-689, Box.cpp:466-742)
//   HookeMemoryContactForceModel::performForcesCalculus (:72-193),
//   computeTangentialVector (:54-65)
//   HookeContactForceModel::performForcesCalculus (HookeContactForceModel.cpp:44-121)
//   Quaternion::setRotFromTwoVectors / rotateVector (Quaternion.cpp:263-299)
// Rolling resistance is not part of the differentiated law.
#pragma once
#include "gdem_dual.cuh"
#include "gdem_types.h"

namespace gdem {

template <typename T>
__host__ __device__ __forceinline__ V3<T> vscale(V3<T> a, T s) { return s * a; }
template <typename T>
__host__ __device__ __forceinline__ V3<T> vconst(double x, double y, double z) {
  return v3(Scal<T>::make(x), Scal<T>::make(y), Scal<T>::make(z));
}

// Group3::round: components below 1e-10 in magnitude are set to zero.
template <typename T>
__host__ __device__ __forceinline__ V3<T> roundSmall(V3<T> a) {
  const T z = Scal<T>::make(0.);
  if (dfabs(val(a.x)) < 1.0e-10) a.x = z;
  if (dfabs(val(a.y)) < 1.0e-10) a.y = z;
  if (dfabs(val(a.z)) < 1.0e-10) a.z = z;
  return a;
}

// Rotation taking u to v as (vector, scalar) quaternion, then applied to x.
template <typename T>
__host__ __device__ __forceinline__ V3<T> rotateFromTo(V3<T> u, V3<T> v, V3<T> x) {
  T nn = dsqrt(vdot(u, u) * vdot(v, v));
  T real = nn + vdot(u, v);
  V3<T> vect;
  if (val(real) < 1.e-6 * val(nn)) {
    real = Scal<T>::make(0.);
    vect = dfabs(val(u.x)) > dfabs(val(u.z)) ? v3(-u.y, u.x, Scal<T>::make(0.))
                                             : v3(Scal<T>::make(0.), -u.z, u.y);
  } else {
    vect = vcross(u, v);
  }
  T nq = dsqrt(vect.x * vect.x + vect.y * vect.y + vect.z * vect.z + real * real);
  T s = Scal<T>::make(1.) / nq;
  V3<T> qv = vscale(vect, s);
  T qw = real * s;
  T nv = vnorm(qv);
  return (vscale(x, qw * qw - nv * nv) + vscale(qv, Scal<T>::make(2.) * vdot(x, qv))) +
         vscale(vcross(qv, x), Scal<T>::make(2.) * qw);
}

template <typename T>
struct LawOut {
  V3<T> f;    // force on body 0
  V3<T> kd;   // updated tangential spring
  V3<T> pn;   // contact normal (the next step's previous normal)
};

// Force on body 0 from body 1 at contact point pcp with overlap vector pen.
template <typename T>
__host__ __device__ __forceinline__ LawOut<T> contactLaw(ModelDesc const& m, double dt, T kn, T en,
                                                         T muc, V3<T> pcp, V3<T> pen, V3<T> x0,
                                                         V3<T> v0, V3<T> w0, double m0, V3<T> x1,
                                                         V3<T> v1, V3<T> w1, double m1,
                                                         bool existed, V3<T> kd, V3<T> pn) {
  const double PI = 3.14159265358979323846;
  V3<T> normal = pen / vnorm(pen);
  normal = roundSmall(normal);
  V3<T> va = v0 + vcross(w0, pcp - x0);
  V3<T> vb = v1 + vcross(w1, pcp - x1);
  V3<T> tmpV = va - vb;
  V3<T> v_n = vscale(normal, vdot(tmpV, normal));
  V3<T> v_t = tmpV - v_n;
  T len = dlog(en);
  T beta = len / dsqrt(PI * PI + len * len);
  V3<T> delFN = vscale(pen, kn);
  double avmass = 1. / (1. / m0 + 1. / m1);
  T gamman = (-2. * beta) * dsqrt(kn * avmass);
  delFN = delFN - vscale(v_n, gamman);
  T normFN = vnorm(delFN);
  T etat = m.etat == -1. ? -beta * dsqrt(kn / avmass) : Scal<T>::make(m.etat);
  T gammat = (2. * etat) * avmass;
  V3<T> viscousFT = vscale(v_t, -gammat);
  LawOut<T> o;
  o.pn = normal;
  if (!m.memory) {
    // Hooke: viscous tangential force capped at muc |Fn|
    V3<T> delFT = viscousFT;
    T fn = muc * normFN;
    if (val(fn) < val(vnorm(delFT))) {
      T nvt = vnorm(v_t);
      V3<T> tangent = vconst<T>(0., 0., 0.);
      if (val(nvt) > 1.0e-10) tangent = vscale(-v_t, Scal<T>::make(1.) / nvt);
      delFT = vscale(tangent, fn);
    }
    o.f = delFN + delFT;
    o.kd = vconst<T>(0., 0., 0.);
    return o;
  }
  if (!existed) kd = vconst<T>(0., 0., 0.);
  else kd = rotateFromTo(pn, normal, kd);
  kd = kd + vscale(v_t, Scal<T>::make(dt * m.kt));
  // computeTangentialVector
  V3<T> tij;
  T nut = vnorm(v_t);
  if (val(nut) > 0.001) {
    tij = vscale(-v_t, Scal<T>::make(1.) / nut);
  } else {
    V3<T> s = kd + vscale(v_t, gammat);
    T ns = vnorm(s);
    if ((val(vnorm(kd)) > m.epst || val(vnorm(vscale(v_t, gammat))) > m.epst) && val(ns) > m.epst)
      tij = vscale(-s, Scal<T>::make(1.) / ns);
    else
      tij = vconst<T>(0., 0., 0.);
  }
  V3<T> trial = -kd + viscousFT;
  T normFT = vnorm(trial);
  V3<T> delFT;
  if (val(normFT) <= val(muc * normFN)) {
    delFT = vscale(tij, normFT);
  } else {
    if (m.kt != 0.) kd = vscale(vscale(tij, -muc * normFN) + viscousFT, Scal<T>::make(1. / m.kt));
    delFT = vscale(tij, muc * normFN);
  }
  o.f = delFN + delFT;
  o.kd = kd;
  return o;
}

// ClosestPointSPHERESPHERE with body a first: contact point and overlap
// vector (from b to a when in contact).
template <typename T>
__host__ __device__ __forceinline__ bool sphereSphereG(V3<T> xa, double ra, V3<T> xb, double rb,
                                                       V3<T>& pc, V3<T>& pen) {
  V3<T> AB = xb - xa;
  T nAB = vnorm(AB);
  T distance = nAB - (ra + rb);
  if (!(val(distance) < 0.)) return false;
  pc = xa + vscale(AB, (distance * 0.5 + ra) / nAB);
  pen = vscale(AB / nAB, distance);
  return true;
}

// Box::IntersectionPointSPHERE in the box frame (half extents e) for the
// sphere centre c of radius r: contact point and overlap (< 0 in contact).
template <typename T>
__host__ __device__ __forceinline__ V3<T> cornerG(const double* e, int n) {
  const double sx = (n == 1 || n == 2 || n == 5 || n == 6) ? 1. : -1.;
  const double sy = (n >= 4) ? 1. : -1.;
  const double sz = (n == 2 || n == 3 || n == 6 || n == 7) ? 1. : -1.;
  return vconst<T>(sx * e[0], sy * e[1], sz * e[2]);
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> contactCornerG(const double* e, V3<T> c, double r,
                                                         int n, T& ov, bool& hit) {
  V3<T> dist = c - cornerG<T>(e, n);
  T nd = vnorm(dist);
  if (val(nd) < r) {
    hit = true;
    ov = nd - r;
    return c - vscale(dist, (ov * 0.5) / nd + 1.);
  }
  return c;
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> contactEdgeG(const double* e, V3<T> c, double r, int n,
                                                       int dir, T& ov, bool& hit) {
  V3<T> cn = cornerG<T>(e, n);
  V3<T> proj = c;
  if (dir == 0) proj.x = cn.x;
  else if (dir == 1) proj.y = cn.y;
  else proj.z = cn.z;
  V3<T> dist = proj - cn;
  T nd = vnorm(dist);
  if (val(nd) < r) {
    hit = true;
    ov = nd - r;
    return c - vscale(dist, (ov * 0.5) / nd + 1.);
  }
  return c;
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> boxSphereG(const double* e, V3<T> c, double r, T& ov,
                                                     bool& hit) {
  hit = false;
  const double gx = val(c.x), gy = val(c.y), gz = val(c.z);
  V3<T> cp = c;
  auto face = [&](T nd, int d, double sign) {
    if (val(nd) < r) {
      hit = true;
      ov = nd - r;
      cp = c;
      T wall = Scal<T>::make(sign * e[d]) + ov * (0.5 * sign);
      if (d == 0) cp.x = wall;
      else if (d == 1) cp.y = wall;
      else cp.z = wall;
    }
  };
  if (gx > e[0]) {
    if (gy > e[1]) {
      if (gz > e[2]) cp = contactCornerG(e, c, r, 6, ov, hit);
      else if (gz < -e[2]) cp = contactCornerG(e, c, r, 5, ov, hit);
      else cp = contactEdgeG(e, c, r, 5, 2, ov, hit);
    } else if (gy < -e[1]) {
      if (gz > e[2]) cp = contactCornerG(e, c, r, 2, ov, hit);
      else if (gz < -e[2]) cp = contactCornerG(e, c, r, 1, ov, hit);
      else cp = contactEdgeG(e, c, r, 1, 2, ov, hit);
    } else {
      if (gz > e[2]) cp = contactEdgeG(e, c, r, 6, 1, ov, hit);
      else if (gz < -e[2]) cp = contactEdgeG(e, c, r, 1, 1, ov, hit);
      else face(c.x - e[0], 0, 1.);
    }
  } else if (gx < -e[0]) {
    if (gy > e[1]) {
      if (gz > e[2]) cp = contactCornerG(e, c, r, 7, ov, hit);
      else if (gz < -e[2]) cp = contactCornerG(e, c, r, 4, ov, hit);
      else cp = contactEdgeG(e, c, r, 4, 2, ov, hit);
    } else if (gy < -e[1]) {
      if (gz > e[2]) cp = contactCornerG(e, c, r, 3, ov, hit);
      else if (gz < -e[2]) cp = contactCornerG(e, c, r, 0, ov, hit);
      else cp = contactEdgeG(e, c, r, 0, 2, ov, hit);
    } else {
      if (gz > e[2]) cp = contactEdgeG(e, c, r, 3, 1, ov, hit);
      else if (gz < -e[2]) cp = contactEdgeG(e, c, r, 0, 1, ov, hit);
      else face(-c.x - e[0], 0, -1.);
    }
  } else {
    if (gy > e[1]) {
      if (gz > e[2]) cp = contactEdgeG(e, c, r, 6, 0, ov, hit);
      else if (gz < -e[2]) cp = contactEdgeG(e, c, r, 4, 0, ov, hit);
      else face(c.y - e[1], 1, 1.);
    } else if (gy < -e[1]) {
      if (gz > e[2]) cp = contactEdgeG(e, c, r, 3, 0, ov, hit);
      else if (gz < -e[2]) cp = contactEdgeG(e, c, r, 0, 0, ov, hit);
      else face(-c.y - e[1], 1, -1.);
    } else {
      if (gz > e[2]) face(c.z - e[2], 2, 1.);
      else if (gz < -e[2]) face(-c.z - e[2], 2, -1.);
    }
  }
  return cp;
}

// ClosestPointSPHEREBOX for an axis-aligned wall: contact point and overlap
// vector (from the wall to the sphere).
template <typename T>
__host__ __device__ __forceinline__ bool sphereWallG(V3<T> x, double r, WallDesc const& w,
                                                     V3<T>& pc, V3<T>& pen) {
  V3<T> local = x - vconst<T>(w.centre[0], w.centre[1], w.centre[2]);
  T ov = Scal<T>::make(1.);
  bool hit = false;
  V3<T> cpl = boxSphereG(w.extent, local, r, ov, hit);
  if (!hit || !(val(ov) < 0.)) return false;
  pc = cpl + vconst<T>(w.centre[0], w.centre[1], w.centre[2]);
  V3<T> AB = pc - x;
  pen = vscale(AB, ov / vnorm(AB));
  return true;
}

}  // namespace gdem
