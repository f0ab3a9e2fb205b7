// gdem_gjk.cuh -- closest points between convex bodies on the device (FP64).
//
// Johnson's distance sub-algorithm of the GJK method (the SOLID formulation
// the reference uses: Geometry/src/Convex.cpp:219-430 for the sub-algorithm,
// :536-627 for closest_points), with the reference's default settings:
// relative tolerance 1e-10, absolute 1e-14, no acceleration, at most 1000
// iterations.  Bodies are shrunk by their crust thickness
// (RigidBodyWithCrust::getTransformWithCrust, RigidBodyWithCrust.cpp:
// 749-760): the local-to-world map is  x = basis * diag(scaling) * p + origin.
// Support functions: Sphere.cpp:99-108, Box.cpp:307-316, Cylinder.cpp:
// 112-133, and for polyhedra Polyhedron::support (Polyhedron.cpp:265-293):
// a climb over the vertex graph from the body's current vertex, moving to the
// first neighbour whose projection gains at least 1e-16, so that among tied
// vertices (a face or an edge facing the direction) the search stays where it
// is.  Each body's current vertex is carried from call to call (its
// m_curr_vertex); the caller passes it in and gets the final one back.
#pragma once
#include "gdem_device.cuh"

namespace gdem {

struct ConvexRef {
  int kind;              // 0 sphere, 1 box, 2 polyhedron, 3 cylinder
  double radius;         // sphere radius
  d3 extent;             // box half lengths
  const double* verts;   // polyhedron vertices (x, y, z), local frame
  int nverts;
  // polyhedron vertex graph (Polyhedron::m_cobound, built from the faces by
  // Polyhedron::BuildPolyhedron): the neighbours of vertex v are
  // adj[adj_off[v] .. adj_off[v + 1]), in the reference's order
  const int* adj_off;
  const int* adj;
};

struct XForm64 { double M[9]; d3 o; };   // row-major M = basis * diag(scaling)

__device__ __forceinline__ XForm64 crustXForm(const double* basis, int stride, int s,
                                              const double* scaling, d3 o) {
  XForm64 t;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) t.M[3 * r + c] = basis[(3 * r + c) * stride + s] * scaling[c];
  t.o = o;
  return t;
}
__device__ __forceinline__ XForm64 identityXForm(const double* scaling, d3 o) {
  XForm64 t;
#pragma unroll
  for (int k = 0; k < 9; ++k) t.M[k] = 0.;
  t.M[0] = scaling[0]; t.M[4] = scaling[1]; t.M[8] = scaling[2];
  t.o = o;
  return t;
}
// Transform::operator() (Transform.cpp:312-317)
__device__ __forceinline__ d3 apply(XForm64 const& t, d3 p) {
  return mk((t.M[0] * p.x + t.M[1] * p.y + t.M[2] * p.z) + t.o.x,
            (t.M[3] * p.x + t.M[4] * p.y + t.M[5] * p.z) + t.o.y,
            (t.M[6] * p.x + t.M[7] * p.y + t.M[8] * p.z) + t.o.z);
}
// Vector3 * Matrix (Matrix.cpp:238-241, 527-530)
__device__ __forceinline__ d3 tmul(d3 v, XForm64 const& t) {
  return mk(t.M[0] * v.x + t.M[3] * v.y + t.M[6] * v.z, t.M[1] * v.x + t.M[4] * v.y + t.M[7] * v.z,
            t.M[2] * v.x + t.M[5] * v.y + t.M[8] * v.z);
}

__device__ __forceinline__ d3 vertexOf(ConvexRef const& s, int i) {
  return mk(s.verts[3 * i], s.verts[3 * i + 1], s.verts[3 * i + 2]);
}
__device__ __forceinline__ double projection(ConvexRef const& s, int i, d3 v) {
  return s.verts[3 * i] * v.x + s.verts[3 * i + 1] * v.y + s.verts[3 * i + 2] * v.z;
}

// cur: the body's current polyhedron vertex (ignored for other shapes)
__device__ __forceinline__ d3 support(ConvexRef const& s, d3 v, int& cur) {
  if (s.kind == 0) {
    double n = norm(v);
    if (n > 1.0e-10) { double r = s.radius / n; return mk(v.x * r, v.y * r, v.z * r); }
    return mk(0., 0., 0.);
  }
  if (s.kind == 3) {
    // Cylinder::support (Geometry/src/Cylinder.cpp:112-133): axis along local
    // Y, extent = (radius, half height, radius)
    if (!(norm(v) > 1.0e-10)) return mk(0., 0., 0.);
    const double sxz = sqrt(v.x * v.x + v.z * v.z);
    const double hh = v.y < 0. ? -s.extent.y : s.extent.y;
    if (sxz > 1.0e-10) {
      const double d = s.extent.x / sxz;
      return mk(v.x * d, fabs(v.y) < 1.0e-10 ? 0. : hh, v.z * d);
    }
    return mk(0., hh, 0.);
  }
  if (s.kind == 1) {
    if (norm(v) < 1.0e-10) return mk(0., 0., 0.);
    return mk(v.x < 0. ? -s.extent.x : s.extent.x, v.y < 0. ? -s.extent.y : s.extent.y,
              v.z < 0. ? -s.extent.z : s.extent.z);
  }
  if (!(norm(v) > 1.0e-10)) return mk(0., 0., 0.);
  if (cur < 0 || cur >= s.nverts) cur = 0;
  int last = -1;
  double h = projection(s, cur, v);
  // each move gains at least 1e-16, so the climb ends; the bound also covers
  // a direction with a NaN component
  for (int moves = 0; moves < s.nverts * s.nverts; ++moves) {
    const int b = s.adj_off[cur], e = s.adj_off[cur + 1];
    int i = b;
    double d = 0.;
    for (; i < e; ++i) {
      if (s.adj[i] == last) continue;
      d = projection(s, s.adj[i], v);
      if (!(d - h < 1.e-16)) break;
    }
    if (i == e) break;
    last = cur;
    cur = s.adj[i];
    h = d;
  }
  return vertexOf(s, cur);
}

struct Simplex64 {
  d3 y[4], p[4], q[4];
  double det[16][4];
  double dp[4][4];
};

__device__ inline void computeDet(Simplex64& S, unsigned bits, unsigned last, unsigned last_bit,
                                  unsigned all_bits) {
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if (bits & bit) S.dp[i][last] = S.dp[last][i] = dot(S.y[i], S.y[last]);
  S.dp[last][last] = dot(S.y[last], S.y[last]);
  S.det[last_bit][last] = 1.;
  for (unsigned j = 0, sj = 1; j < 4; ++j, sj <<= 1) {
    if (bits & sj) {
      unsigned s2 = sj | last_bit;
      S.det[s2][j] = S.dp[last][last] - S.dp[last][j];
      S.det[s2][last] = S.dp[j][j] - S.dp[j][last];
      for (unsigned k = 0, sk = 1; k < j; ++k, sk <<= 1) {
        if (bits & sk) {
          unsigned s3 = sk | s2;
          S.det[s3][k] = S.det[s2][j] * (S.dp[j][j] - S.dp[j][k]) +
                         S.det[s2][last] * (S.dp[last][j] - S.dp[last][k]);
          S.det[s3][j] = S.det[sk | last_bit][k] * (S.dp[k][k] - S.dp[k][j]) +
                         S.det[sk | last_bit][last] * (S.dp[last][k] - S.dp[last][j]);
          S.det[s3][last] = S.det[sk | sj][k] * (S.dp[k][k] - S.dp[k][last]) +
                            S.det[sk | sj][j] * (S.dp[j][k] - S.dp[j][last]);
        }
      }
    }
  }
  if (all_bits == 15) {
    S.det[15][0] = S.det[14][1] * (S.dp[1][1] - S.dp[1][0]) + S.det[14][2] * (S.dp[2][1] - S.dp[2][0]) +
                   S.det[14][3] * (S.dp[3][1] - S.dp[3][0]);
    S.det[15][1] = S.det[13][0] * (S.dp[0][0] - S.dp[0][1]) + S.det[13][2] * (S.dp[2][0] - S.dp[2][1]) +
                   S.det[13][3] * (S.dp[3][0] - S.dp[3][1]);
    S.det[15][2] = S.det[11][0] * (S.dp[0][0] - S.dp[0][2]) + S.det[11][1] * (S.dp[1][0] - S.dp[1][2]) +
                   S.det[11][3] * (S.dp[3][0] - S.dp[3][2]);
    S.det[15][3] = S.det[7][0] * (S.dp[0][0] - S.dp[0][3]) + S.det[7][1] * (S.dp[1][0] - S.dp[1][3]) +
                   S.det[7][2] * (S.dp[2][0] - S.dp[2][3]);
  }
}

__device__ __forceinline__ bool validSet(Simplex64 const& S, unsigned s, unsigned all_bits) {
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1) {
    if (all_bits & bit) {
      if (s & bit) { if (S.det[s][i] <= 1.0e-20) return false; }
      else if (S.det[s | bit][i] > 0) return false;
    }
  }
  return true;
}

__device__ __forceinline__ d3 computeVector(Simplex64 const& S, unsigned bits) {
  double sum = 0.;
  d3 v = mk(0., 0., 0.);
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if (bits & bit) { sum += S.det[bits][i]; v = v + S.det[bits][i] * S.y[i]; }
  return v * (1. / sum);
}

__device__ __forceinline__ bool properSet(Simplex64 const& S, unsigned s) {
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if ((s & bit) && S.det[s][i] <= 1.0e-20) return false;
  return true;
}

__device__ inline bool closestSub(Simplex64& S, unsigned& bits, unsigned last, unsigned last_bit,
                                  unsigned all_bits, d3& v) {
  computeDet(S, bits, last, last_bit, all_bits);
  for (unsigned s = bits; s; --s) {
    if ((s & bits) == s && validSet(S, s | last_bit, all_bits)) {
      bits = s | last_bit;
      v = computeVector(S, bits);
      return true;
    }
  }
  if (validSet(S, last_bit, all_bits)) {
    bits = last_bit;
    v = S.y[last];
    return true;
  }
  double min_dist2 = __longlong_as_double(0x7ff0000000000000ll);
  for (unsigned s = all_bits; s; --s) {
    if ((s & all_bits) == s && properSet(S, s)) {
      d3 u = computeVector(S, s);
      double d2 = u.x * u.x + u.y * u.y + u.z * u.z;
      if (d2 < min_dist2) { min_dist2 = d2; bits = s; v = u; }
    }
  }
  return false;
}

// closest_points: distance between the two shrunk bodies and the witness
// points in world coordinates; *iters receives the iteration count.
// curA, curB: the bodies' current polyhedron vertices, updated.
// sep > 0: the search stops as soon as the distance is known to exceed sep
// -- the lower bound v.w / |v| that each support point gives (w the support
// point of A - B in direction -v) is above it -- and returns that bound
// with *separated set; pa, pb are then not computed.  The bound is a lower
// bound of the distance the full search would return, so a caller that only
// needs "distance > sep" decides the same.
__device__ inline double closestPoints64(ConvexRef const& a, XForm64 const& a2w,
                                         ConvexRef const& b, XForm64 const& b2w, d3& pa, d3& pb,
                                         int* iters, int& curA, int& curB, double sep = 0.,
                                         bool* separated = nullptr) {
  unsigned bits = 0, last = 0, last_bit = 0, all_bits = 0;
  Simplex64 S;
  // the simplex starts zeroed; that is done just before its first use, so a
  // search that ends at its first separation test never touches it
  bool ready = false;
  auto clear = [&S]() {
#pragma unroll
    for (int i = 0; i < 16; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) S.det[i][j] = 0.;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      S.y[i] = S.p[i] = S.q[i] = mk(0., 0., 0.);
#pragma unroll
      for (int j = 0; j < 4; ++j) S.dp[i][j] = 0.;
    }
  };
  int numIterations = 0;
  const double relError = 1.e-10, absError = 1.e-4 * relError;
  d3 v = apply(a2w, support(a, mk(0., 0., 0.), curA)) - apply(b2w, support(b, mk(0., 0., 0.), curB));
  d3 w = v;
  double dist = norm(v);
  while (bits < 15 && dist > 1.0e-15 && numIterations < 1000) {
    ++numIterations;
    last = 0;
    last_bit = 1;
    while (bits & last_bit) { ++last; last_bit <<= 1; }
    d3 d = v;
    const d3 pl = support(a, tmul(-d, a2w), curA);
    const d3 ql = support(b, tmul(d, b2w), curB);
    w = apply(a2w, pl) - apply(b2w, ql);
    if (sep > 0. && dot(v, w) > sep * dist) {
      *iters = numIterations;
      *separated = true;
      return dot(v, w) / dist;
    }
    if (!ready) { clear(); ready = true; }
    S.p[last] = pl;
    S.q[last] = ql;
    double mu = dist - dot(v, w) / dist;
    if (mu < dist * relError || mu < absError) break;
    bool degen = false;
    for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
      if ((all_bits & bit) && S.y[i].x == w.x && S.y[i].y == w.y && S.y[i].z == w.z) degen = true;
    if (degen) break;
    S.y[last] = w;
    all_bits = bits | last_bit;
    if (!closestSub(S, bits, last, last_bit, all_bits, v)) break;
    dist = norm(v);
  }
  if (!ready) clear();
  // computePoints: barycentric witnesses in the local frames, then to world
  double sum = 0.;
  d3 p1 = mk(0., 0., 0.), p2 = mk(0., 0., 0.);
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if (bits & bit) {
      sum += S.det[bits][i];
      p1 = p1 + S.det[bits][i] * S.p[i];
      p2 = p2 + S.det[bits][i] * S.q[i];
    }
  double sc = 1. / sum;
  pa = apply(a2w, p1 * sc);
  pb = apply(b2w, p2 * sc);
  *iters = numIterations;
  return dist;
}

// The first iteration of closestPoints64 alone (its start from the
// supports in direction 0, then the supports in direction -v and v): true
// when their lower bound v.w/|v| on the distance of the bodies already
// exceeds sep, the test that ends the full search there; curA, curB as that
// search leaves them.  False when it does not, or when the start points
// coincide (the full search decides those).
__device__ inline bool separatedAtFirst(ConvexRef const& a, XForm64 const& a2w, ConvexRef const& b,
                                        XForm64 const& b2w, int& curA, int& curB, double sep) {
  const d3 v = apply(a2w, support(a, mk(0., 0., 0.), curA)) -
               apply(b2w, support(b, mk(0., 0., 0.), curB));
  const double dist = norm(v);
  if (!(dist > 1.0e-15)) return false;
  const d3 pl = support(a, tmul(-v, a2w), curA);
  const d3 ql = support(b, tmul(v, b2w), curB);
  const d3 w = apply(a2w, pl) - apply(b2w, ql);
  return dot(v, w) > sep * dist;
}

}  // namespace gdem
