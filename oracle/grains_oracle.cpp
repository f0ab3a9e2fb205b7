// grains_oracle.cpp -- CPU FP64 restatement of the Grains3D DEM time step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
// compared against; the product library never links, loads or calls it.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
//
// It restates, in plain scalar C++ with the reference's own operation order
// (compiled with -ffp-contract=off so no FMA is introduced), the serial
// Type="Standard" leapfrog step of Grains3D (GRAINS_V1/Grains):
//   * Grains::Simulation leapfrog branch        Base/src/Grains.cpp:344-364
//   * Grains::computeParticlesForceAndTorque    Base/src/Grains.cpp:459-482
//   * LinkedCell::set (grid sizing)             Base/src/LinkedCell.cpp:47-160
//   * Cell::GetCell                             Base/src/Cell.cpp:172-184
//   * Cell::add (push_front)                    Base/src/Cell.cpp:90-93
//   * LinkedCell::LinkUpdateActiveParticle      Base/src/LinkedCell.cpp:1502-1547
//   * LinkedCell::setCellContactNeighborhood    Base/src/LinkedCell.cpp:958-984
//   * LinkedCell::ComputeForces                 Base/src/LinkedCell.cpp:1019-1103
//   * Particle::InterAction                     Component/src/Particle.cpp:477-545
//   * SimpleObstacle::InterAction               Component/src/SimpleObstacle.cpp:222-271
//   * ClosestPointSPHERESPHERE / SPHEREBOX      Geometry/src/RigidBodyWithCrust.cpp:596-721
//   * Box::IntersectionPointSPHERE & helpers    Geometry/src/Box.cpp:466-800
//   * HookeMemoryContactForceModel              Component/src/HookeMemoryContactForceModel.cpp:12-249
//   * Component contact memory map              Component/src/Component.cpp:570-689
//   * Torsor::addForce                          Component/src/Torsor.cpp:184-189
//   * SecondOrderLeapFrog::Move/advanceVelocity TimeIntegration/src/SecondOrderLeapFrog.cpp:44-94
//   * ParticleKinematics::Move/advanceVelocity  Component/src/ParticleKinematics.cpp:62-128
//   * ParticleKinematicsSphere angular accel    Component/src/ParticleKinematicsSphere.cpp:47-55
//   * Quaternion ops                            Geometry/src/Quaternion.cpp:74-299,442-472
//   * Transform::composeLeftByRotation          Geometry/src/Transform.cpp:140-159
//
// Periodic boundaries: the reference keeps periodic "clones" (same ID as the
// master, LinkedCell.cpp:2008-2400) in two extra cell layers; this
// restatement uses the equivalent minimum-image convention on the same grid
// (cell indices are reported in the reference's numbering, i.e. with the
// extra layer, so inner cells are 1..n).  A master that leaves the inner
// domain is replaced by its clone at x +/- L, which is what the wrap below
// does.  Forces agree with the clone formulation up to the rounding of the
// periodic translation.
//
// Scope: spheres + axis-aligned box walls (the obstacle type of the north-star
// configurations), HookeMemory (with rolling-friction memory), fluid-free
// (coupling factor 1).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <list>
#include <map>
#include <tuple>
#include <vector>
#include <algorithm>

namespace {

const double PI = 3.14159265358979323846;   // Basic.hh:22
const double EPSILON = 1.0e-10;              // Basic.hh:26

// ---------------------------------------------------------------- vectors --
struct V3 {
  double c[3];
  V3() { c[0] = c[1] = c[2] = 0.; }
  V3(double x, double y, double z) { c[0] = x; c[1] = y; c[2] = z; }
  double& operator[](int i) { return c[i]; }
  double operator[](int i) const { return c[i]; }
};
inline V3 operator+(V3 const& a, V3 const& b) { return V3(a[0]+b[0], a[1]+b[1], a[2]+b[2]); }
inline V3 operator-(V3 const& a, V3 const& b) { return V3(a[0]-b[0], a[1]-b[1], a[2]-b[2]); }
inline V3 operator-(V3 const& a) { return V3(-a[0], -a[1], -a[2]); }
inline V3 operator*(V3 const& a, double d) { return V3(a[0]*d, a[1]*d, a[2]*d); }
inline V3 operator*(double d, V3 const& a) { return V3(a[0]*d, a[1]*d, a[2]*d); }
inline V3 operator/(V3 const& a, double d) { return V3(a[0]/d, a[1]/d, a[2]/d); }
inline double dot(V3 const& a, V3 const& b) { return a[0]*b[0] + a[1]*b[1] + a[2]*b[2]; }
// Vector3::operator^ (Geometry/src/Vector3.cpp:114-119)
inline V3 cross(V3 const& a, V3 const& b) {
  return V3(a[1]*b[2] - a[2]*b[1], - a[0]*b[2] + a[2]*b[0], a[0]*b[1] - a[1]*b[0]);
}
inline double norm(V3 const& a) { return std::sqrt(a[0]*a[0] + a[1]*a[1] + a[2]*a[2]); }
// Group3::round (Geometry/src/Group3.cpp:390-395), default tol EPSILON
inline void round3(V3& a) {
  for (int i = 0; i < 3; ++i) a[i] = std::fabs(a[i]) < EPSILON ? 0. : a[i];
}
inline V3& operator+=(V3& a, V3 const& b) { a[0] += b[0]; a[1] += b[1]; a[2] += b[2]; return a; }
inline V3& operator-=(V3& a, V3 const& b) { a[0] -= b[0]; a[1] -= b[1]; a[2] -= b[2]; return a; }

// ------------------------------------------------------------ quaternions --
struct Q { V3 v; double w; };   // [w, v]
inline Q qmake(V3 const& v, double w) { Q q; q.v = v; q.w = w; return q; }
inline Q conj(Q const& q) { return qmake(-q.v, q.w); }
// Quaternion::operator* (Quaternion.cpp:442-448)
inline Q qmul(Q const& a, Q const& b) {
  double tmp = (a.w * b.w) - dot(a.v, b.v);
  V3 vt = (cross(a.v, b.v) + (a.w * b.v)) + (b.w * a.v);
  return qmake(vt, tmp);
}
// operator,(Vector3 lhs, Quaternion q) -> q.multLeftVec(lhs) (Quaternion.cpp:93-98,468-472)
inline Q vecq(V3 const& lhs, Q const& q) {
  double tmp = dot(-lhs, q.v);
  V3 vt = cross(lhs, q.v) + (lhs * q.w);
  return qmake(vt, tmp);
}
// Quaternion::multToVector3 (Quaternion.cpp:108-113)
inline V3 multToVector3(Q const& a, Q const& rhs) {
  return (cross(a.v, rhs.v) + (a.w * rhs.v)) + (rhs.w * a.v);
}
inline double qnorm(Q const& q) {
  return std::sqrt(q.v[0]*q.v[0] + q.v[1]*q.v[1] + q.v[2]*q.v[2] + q.w*q.w);
}
// Quaternion::setRotFromTwoVectors (Quaternion.cpp:263-288)
inline Q rotFromTwoVectors(V3 const& u, V3 const& v) {
  double nn = std::sqrt(dot(u, u) * dot(v, v));
  double real = nn + dot(u, v);
  V3 vect;
  if (real < 1.e-6 * nn) {
    real = 0.;
    vect = std::fabs(u[0]) > std::fabs(u[2]) ? V3(-u[1], u[0], 0.) : V3(0., -u[2], u[1]);
  } else {
    vect = cross(u, v);
  }
  Q qq = qmake(vect, real);
  double s = 1. / qnorm(qq);
  return qmake(qq.v * s, qq.w * s);
}
// Quaternion::rotateVector (Quaternion.cpp:293-299)
inline V3 rotateVector(Q const& q, V3 const& v) {
  double nv = norm(q.v);
  return ((q.w * q.w - nv * nv) * v + (2. * dot(v, q.v)) * q.v) + (2. * q.w) * cross(q.v, v);
}

// ---------------------------------------------------------------- system ---
struct Hist {                 // tuple<bool, kdelta, prev_normal, cumulSpringTorque>
  bool active;
  V3 kdelta, prevn, spring;
};
typedef std::tuple<int, int, int> Key;

struct Model {
  double kn, en, etat, muc, kt, mur, etarpf, epst;
  double kr;       // Hooke rolling coefficient
  double beta;
  bool memory;     // HookeMemory (true) or Hooke (false)
  bool rolling;    // HookeMemory: mur != 0; Hooke: kr != 0
};

// Convex shape of a particle class or a wall.
struct Shape {
  int kind = 0;                      // 0 sphere, 1 box, 2 polyhedron, 3 cylinder
  double radius = 0.;                // circumscribed radius
  V3 extent;                         // box half lengths; cylinder (radius, half height, radius)
  std::vector<V3> verts;             // polyhedron vertices (local frame)
  std::vector<std::vector<int>> cob; // vertex neighbours (Polyhedron::BuildPolyhedron)
  V3 scaling;                        // crust shrink factors (RigidBodyWithCrust ctor)
  double volume = 0.;
  double inertia[6] = {0, 0, 0, 0, 0, 0};
};

struct Particle {
  int id, type;
  double radius, crust, mass, inertia, density, eqrad;
  double I[3] = {0, 0, 0};           // body-frame principal inertia (inertia[0], [3], [5])
  const Shape* shape = nullptr;
  int curv = 0;                      // Polyhedron::m_curr_vertex of this particle's clone
  int matbit;
  V3 weight;
  V3 x, v, w, wbf;
  Q q;
  double basis[9];
  V3 F, T, ref;
  int cell[3];
  int cellnum;
  std::map<Key, Hist> cmap;
};

struct Wall {
  int id;
  Shape shape;          // box with the wall's crust scaling
  V3 centre, extent;    // half lengths
  double crust;
  int matbit;
};

struct ContactRec {
  int id0, id1;          // id1 < 0 : wall k as -(k+2)
  double delta;
  V3 point, overlap, force;
};

}  // namespace

extern "C" {

// Configuration passed by the test harness.  Field meanings follow the
// Grains3D XML (Construction/LinkedCell, Origin, Periodicity, Particles,
// Obstacles, ContactForceModels, Forces/Gravity, Simulation/TimeStep).
typedef struct {
  double origin[3];
  double maxc[3];
  int periodic[3];
  double cell_size_factor;
  double gravity[3];
  double dt;
  int n_types;
  const double* type_radius;
  const double* type_crust;
  const double* type_density;
  const int* type_matbit;
  int n_walls;
  const double* wall_centre;   // 3 per wall
  const double* wall_extent;   // 3 per wall (half lengths)
  const double* wall_crust;
  const int* wall_matbit;
  int n_models;
  const int* model_mask;
  const double* model_params;  // kn en etat muc kt mur etarpf epst kr memory (10 per model)
  // convex particle classes (NULL: all spheres)
  const int* type_shape;       // 0 sphere, 1 box, 2 polyhedron
  const double* type_extent;   // box half lengths, 3 per class
  const int* type_poly;        // 4 per class: first vertex, vertex count, first face int, face ints
  const double* poly_verts;    // 3 per vertex
  const int* poly_faces;       // per face: size, then vertex indices
} or_config;

enum { OR_OK = 0, OR_ERR_CONTACT = 1, OR_ERR_MOTION = 2, OR_ERR_OUT_OF_GRID = 4 };

}  // extern "C"

namespace {

struct System {
  // grid
  double dom_origin[3], dom_size[3];
  int periodic[3];
  int nb[3];
  double edge[3];
  double lc_origin[3];
  std::vector<std::list<int>> cells;
  std::vector<int> nbr_order;      // the 13 half-stencil offsets, in list order
  double gravity[3], dt;
  std::vector<Particle> parts;     // active list order == insertion order
  std::vector<Wall> walls;
  std::map<int, Model> models;
  std::vector<double> type_radius, type_crust, type_density;
  std::vector<Shape> shapes;       // per particle class
  std::vector<int> type_matbit;
  std::vector<ContactRec> contacts;
  int err = 0;
  double time = 0.;

  int cellnum(int i, int j, int k) const { return j * nb[2] * nb[0] + k * nb[0] + i; }
  bool valid(int i, int j, int k) const {
    return -1 < i && i < nb[0] && -1 < j && j < nb[1] && -1 < k && k < nb[2];
  }
  void getCell(V3 const& p, int* id) const {   // Cell::GetCell
    for (int d = 0; d < 3; ++d) id[d] = int(std::floor((p[d] - lc_origin[d]) / edge[d]));
  }
  Model const& model(int ma, int mb) const {
    auto it = models.find(ma | mb);
    return it->second;
  }
};

const int STENCIL[3][13] = {{-1,  0, +1, +1, -1,  0, +1, -1,  0, +1, -1,  0, +1},
                            { 0,  0,  0,  0, +1, +1, +1, +1, +1, +1, +1, +1, +1},
                            {+1, +1, +1,  0, +1, +1, +1,  0,  0,  0, -1, -1, -1}};

// LinkedCell::set (LinkedCell.cpp:47-160) with cellsize = 2 * factor * maxR
// (Grains.cpp:1005-1022, 2522-2526)
void setGrid(System& s, double cellsize) {
  for (int d = 0; d < 3; ++d) {
    int n = (int)((s.dom_size[d] + EPSILON) / cellsize);
    if (!n) n = 1;
    s.nb[d] = n;
    s.edge[d] = s.dom_size[d] / n;
    s.lc_origin[d] = s.dom_origin[d];
  }
  for (int d = 0; d < 3; ++d)
    if (s.periodic[d]) {
      s.lc_origin[d] += -s.edge[d];      // Point3::Move( -edge ) : += (-edge)
      s.nb[d] += 2;
    }
  s.cells.assign((size_t)s.nb[0] * s.nb[1] * s.nb[2], std::list<int>());
  // m_neighborsContact is filled with push_front: reverse order of STENCIL
  s.nbr_order.clear();
  for (int j = 12; j >= 0; --j) s.nbr_order.push_back(j);
}

// Periodic wrap: inner cells are 1..n-2 in a periodic direction.
void wrapPeriodic(System& s, Particle& p) {
  for (int d = 0; d < 3; ++d) {
    if (!s.periodic[d]) continue;
    int id[3];
    s.getCell(p.x, id);
    if (id[d] < 1) p.x[d] = p.x[d] + s.dom_size[d];
    else if (id[d] > s.nb[d] - 2) p.x[d] = p.x[d] + (-s.dom_size[d]);
  }
}

// Cell index of a (possibly periodic) neighbour cell; returns -1 when absent.
// In a periodic direction the clone layer (0 or n-1) maps to the inner cell
// holding the master, and the returned shift is the image translation.
int neighbourCell(System const& s, int i, int j, int k, int* shift) {
  int c[3] = {i, j, k};
  for (int d = 0; d < 3; ++d) {
    shift[d] = 0;
    if (s.periodic[d]) {
      int nin = s.nb[d] - 2;
      if (c[d] < 1) { c[d] += nin; shift[d] = -1; }
      else if (c[d] > nin) { c[d] -= nin; shift[d] = +1; }
    }
  }
  if (!s.valid(c[0], c[1], c[2])) return -1;
  return s.cellnum(c[0], c[1], c[2]);
}

// -------------------------------------------------------------- kinematics --
// ParticleKinematicsSphere / ParticleKinematics3D::computeAngularAccelerationBodyFixed
// (ParticleKinematicsSphere.cpp:47-55, ParticleKinematics3D.cpp:56-77; the
// predictor-mode gyroscopic term is on, Grains.cpp:18)
inline V3 dOmega(Particle const& p, V3 const& tbf, V3 const& om) {
  double c = 1.;
  const double* I = p.I;
  if (!p.shape || p.shape->kind == 0)
    return V3(tbf[0] / (c * I[0]), tbf[1] / (c * I[1]), tbf[2] / (c * I[2]));
  return V3(tbf[0] / (c * I[0]) + om[1] * om[2] * (I[1] - I[2]) / I[0],
            tbf[1] / (c * I[1]) + om[2] * om[0] * (I[2] - I[0]) / I[1],
            tbf[2] / (c * I[2]) + om[0] * om[1] * (I[0] - I[1]) / I[2]);
}

// SSP-RK3 of SecondOrderLeapFrog::Move / advanceVelocity (:53-62, :83-92)
inline V3 rk3(Particle const& p, V3 const& tbf, V3 const& wbf, double h) {
  V3 K1 = dOmega(p, tbf, wbf); K1 = K1 * h;
  V3 K2 = dOmega(p, tbf, wbf + K1); K2 = K2 * h;
  V3 K3 = dOmega(p, tbf, wbf + 0.25 * (K1 + K2)); K3 = K3 * h;
  return wbf + ((K1 + K2) + 4. * K3) / 6.;
}

// ParticleKinematics::Move (ParticleKinematics.cpp:62-104); returns |dx|
double moveParticle(Particle& p, double h, double dt) {
  Q pc = conj(p.q);
  V3 tbf = multToVector3(pc, vecq(p.T, p.q));
  double c = 1.;
  p.v += (p.F / (p.mass * c)) * h;
  V3 dx = p.v * dt;
  p.wbf = rk3(p, tbf, p.wbf, h);
  V3 meanw = p.wbf;
  p.w = multToVector3(p.q, vecq(p.wbf, pc));
  meanw = multToVector3(p.q, vecq(meanw, pc));
  p.x += dx;                                      // composeLeftByTranslation
  double nOmega = norm(meanw);
  Q qdt;
  if (nOmega > EPSILON) {
    double cc = std::cos(nOmega * dt / 2.);
    double ss = std::sin(nOmega * dt / 2.);
    V3 t = (ss * 1. / nOmega) * meanw;
    qdt = qmake(t, cc);
  } else {
    qdt = qmake(V3(0., 0., 0.), 1.);
  }
  p.q = qmul(qdt, p.q);
  // Transform::composeLeftByRotation (Transform.cpp:140-159)
  double* mm = p.basis;
  double qx = qdt.v[0], qy = qdt.v[1], qz = qdt.v[2], qw = qdt.w;
  double out[9];
  for (int i = 0; i < 3; ++i) {
    double px = qy * mm[6 + i] - qz * mm[3 + i] + qw * mm[0 + i];
    double py = qz * mm[0 + i] - qx * mm[6 + i] + qw * mm[3 + i];
    double pz = qx * mm[3 + i] - qy * mm[0 + i] + qw * mm[6 + i];
    double pw = - qx * mm[0 + i] - qy * mm[3 + i] - qz * mm[6 + i];
    out[0 + i] = qy * pz - qz * py - pw * qx + qw * px;
    out[3 + i] = qz * px - qx * pz - pw * qy + qw * py;
    out[6 + i] = qx * py - qy * px - pw * qz + qw * pz;
  }
  std::memcpy(p.basis, out, sizeof(out));
  return norm(dx);
}

// ParticleKinematics::advanceVelocity (ParticleKinematics.cpp:110-128)
void advanceVelocity(Particle& p, double h) {
  Q pc = conj(p.q);
  V3 tbf = multToVector3(pc, vecq(p.T, p.q));
  double c = 1.;
  p.v += (p.F / (p.mass * c)) * h;
  p.wbf = rk3(p, tbf, p.wbf, h);
  p.w = multToVector3(p.q, vecq(p.wbf, pc));
}

// ------------------------------------------------------------ narrow phase --
struct PointContact {
  V3 point, overlap;
  double dist;
  bool contact;
};

// ClosestPointSPHERESPHERE (RigidBodyWithCrust.cpp:596-639).  xb is the
// image position of B.  Sets *err when -distance >= crustA + crustB; the
// reference then retries with a 10x crust shrink (RigidBodyWithCrust.cpp:
// 534-588), which for spheres imposes an overlap of crustA + crustB along the
// centre line and places the contact at the midpoint of the shrunk spheres'
// witness points.
PointContact sphereSphere(Particle const& a, V3 const& xb, Particle const& b, int* err) {
  PointContact pc;
  V3 AB = xb - a.x;
  double rA = a.radius, rB = b.radius;
  double distance = norm(AB) - (rA + rB);
  if (distance > 0.) { pc.contact = false; pc.dist = distance; return pc; }
  if (-distance >= a.crust + b.crust) {
    *err |= OR_ERR_CONTACT;
    auto shrunk = [](double r, double crust) {
      double s = (r - 10. * crust) / r;   // getTransformWithCrust(factor, 0.5)
      return r * (s > 0.5 ? s : 0.5);
    };
    double ra = shrunk(rA, a.crust), rb = shrunk(rB, b.crust);
    double nAB = norm(AB);
    V3 u = AB / nAB;
    V3 pA = a.x + ra * u, pB = xb - rb * u;
    V3 ba = pA - pB;
    ba = ba / norm(ba);
    double imp = 1. * (a.crust + b.crust);
    pc.point = pA / 2.0 + pB / 2.0;
    pc.overlap = imp * ba;
    pc.dist = -imp;
    pc.contact = true;
    return pc;
  }
  double nAB = norm(AB);
  pc.point = a.x + ((rA + 0.5 * distance) * AB) / nAB;
  pc.overlap = distance * (AB / nAB);
  pc.dist = distance;
  pc.contact = true;
  return pc;
}

// Box::ContactCornerSPHERE / ContactEdgeSPHERE (Box.cpp)
V3 cornerOf(V3 const& e, int n) {
  // m_corners numbering of Box (Box.cpp constructor): 0:(-,-,-) 1:(+,-,-)
  // 2:(+,-,+) 3:(-,-,+) 4:(-,+,-) 5:(+,+,-) 6:(+,+,+) 7:(-,+,+)
  static const int sg[8][3] = {{-1,-1,-1},{1,-1,-1},{1,-1,1},{-1,-1,1},
                               {-1,1,-1},{1,1,-1},{1,1,1},{-1,1,1}};
  return V3(sg[n][0] * e[0], sg[n][1] * e[1], sg[n][2] * e[2]);
}
V3 contactCorner(V3 const& e, V3 const& c, double r, int n, double& ov) {
  V3 cp;
  V3 dist = c - cornerOf(e, n);
  double nd = norm(dist);
  if (nd < r) { ov = nd - r; cp = c - (1. + 0.5 * ov / nd) * dist; }
  return cp;
}
V3 contactEdge(V3 const& e, V3 const& c, double r, int n, int dir, double& ov) {
  V3 cp, proj = c;
  V3 cn = cornerOf(e, n);
  proj[dir] = cn[dir];
  V3 dist = proj - cn;
  double nd = norm(dist);
  if (nd < r) { ov = nd - r; cp = c - (1. + 0.5 * ov / nd) * dist; }
  return cp;
}
// Box::IntersectionPointSPHERE (Box.cpp:466-676); e = half extents
V3 boxSphere(V3 const& e, V3 const& c, double r, double& ov) {
  V3 cp;
  double gx = c[0], gy = c[1], gz = c[2];
  ov = 1.;
  const int X = 0, Y = 1, Z = 2;
  if (gx > e[X]) {
    if (gy > e[Y]) {
      if (gz > e[Z]) cp = contactCorner(e, c, r, 6, ov);
      else if (gz < -e[Z]) cp = contactCorner(e, c, r, 5, ov);
      else cp = contactEdge(e, c, r, 5, Z, ov);
    } else if (gy < -e[Y]) {
      if (gz > e[Z]) cp = contactCorner(e, c, r, 2, ov);
      else if (gz < -e[Z]) cp = contactCorner(e, c, r, 1, ov);
      else cp = contactEdge(e, c, r, 1, Z, ov);
    } else {
      if (gz > e[Z]) cp = contactEdge(e, c, r, 6, Y, ov);
      else if (gz < -e[Z]) cp = contactEdge(e, c, r, 1, Y, ov);
      else {
        double nd = gx - e[X];
        if (nd < r) { ov = nd - r; cp = V3(e[X] + 0.5 * ov, c[Y], c[Z]); }
      }
    }
  } else if (gx < -e[X]) {
    if (gy > e[Y]) {
      if (gz > e[Z]) cp = contactCorner(e, c, r, 7, ov);
      else if (gz < -e[Z]) cp = contactCorner(e, c, r, 4, ov);
      else cp = contactEdge(e, c, r, 4, Z, ov);
    } else if (gy < -e[Y]) {
      if (gz > e[Z]) cp = contactCorner(e, c, r, 3, ov);
      else if (gz < -e[Z]) cp = contactCorner(e, c, r, 0, ov);
      else cp = contactEdge(e, c, r, 0, Z, ov);
    } else {
      if (gz > e[Z]) cp = contactEdge(e, c, r, 3, Y, ov);
      else if (gz < -e[Z]) cp = contactEdge(e, c, r, 0, Y, ov);
      else {
        double nd = -e[X] - gx;
        if (nd < r) { ov = nd - r; cp = V3(-e[X] - 0.5 * ov, c[Y], c[Z]); }
      }
    }
  } else {
    if (gy > e[Y]) {
      if (gz > e[Z]) cp = contactEdge(e, c, r, 6, X, ov);
      else if (gz < -e[Z]) cp = contactEdge(e, c, r, 4, X, ov);
      else {
        double nd = gy - e[Y];
        if (nd < r) { ov = nd - r; cp = V3(c[X], e[Y] + 0.5 * ov, c[Z]); }
      }
    } else if (gy < -e[Y]) {
      if (gz > e[Z]) cp = contactEdge(e, c, r, 3, X, ov);
      else if (gz < -e[Z]) cp = contactEdge(e, c, r, 0, X, ov);
      else {
        double nd = -e[Y] - gy;
        if (nd < r) { ov = nd - r; cp = V3(c[X], -e[Y] - 0.5 * ov, c[Z]); }
      }
    } else {
      if (gz > e[Z]) {
        double nd = gz - e[Z];
        if (nd < r) { ov = nd - r; cp = V3(c[X], c[Y], e[Z] + 0.5 * ov); }
      } else if (gz < -e[Z]) {
        double nd = -e[Z] - gz;
        if (nd < r) { ov = nd - r; cp = V3(c[X], c[Y], -e[Z] - 0.5 * ov); }
      } else {
        ov = -10000.;
      }
    }
  }
  return cp;
}

// ClosestPointSPHEREBOX, sphere first (RigidBodyWithCrust.cpp:647-689).
// Walls are axis aligned: the inverse transform is p - centre and the direct
// transform is p + centre (Transform.cpp:71-77, 312-317 with identity basis).
PointContact sphereWall(Particle const& a, Wall const& w, int* err) {
  PointContact pc;
  pc.contact = false;
  V3 local = a.x - w.centre;
  double ov = 0.;
  V3 cpl = boxSphere(w.extent, local, a.radius, ov);
  pc.dist = ov;
  if (ov < 0.) {
    if (-ov >= a.crust + w.crust) {
      *err |= OR_ERR_CONTACT;
      return pc;   // the reference falls back to GJK on shrunk bodies
    }
    V3 contact = cpl + w.centre;
    V3 AB = contact - a.x;
    pc.point = contact;
    pc.overlap = (ov / norm(AB)) * AB;
    pc.contact = true;
  }
  return pc;
}

// -------------------------------------------------------------------- GJK --
// Transform with the crust shrink (RigidBodyWithCrust::getTransformWithCrust,
// RigidBodyWithCrust.cpp:749-760): M = basis * diag(scaling) (Matrix::
// multiplyByScalingMatrix scales columns), origin = centre.  Row-major M.
struct XForm { double M[9]; V3 o; };

XForm crustTransform(const double* basis, V3 const& s, V3 const& o) {
  XForm t;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) t.M[3 * r + c] = basis[3 * r + c] * s[c];
  t.o = o;
  return t;
}
// Transform::operator() (Transform.cpp:312-317): m_basis[i] * p + m_origin[i]
inline V3 apply(XForm const& t, V3 const& p) {
  return V3((t.M[0] * p[0] + t.M[1] * p[1] + t.M[2] * p[2]) + t.o[0],
            (t.M[3] * p[0] + t.M[4] * p[1] + t.M[5] * p[2]) + t.o[1],
            (t.M[6] * p[0] + t.M[7] * p[1] + t.M[8] * p[2]) + t.o[2]);
}
// Vector3 * Matrix = (tdot(X, v), tdot(Y, v), tdot(Z, v)) (Matrix.cpp:238-241, 527-530)
inline V3 tmul(V3 const& v, XForm const& t) {
  return V3(t.M[0] * v[0] + t.M[3] * v[1] + t.M[6] * v[2],
            t.M[1] * v[0] + t.M[4] * v[1] + t.M[7] * v[2],
            t.M[2] * v[0] + t.M[5] * v[1] + t.M[8] * v[2]);
}

// Support functions in the shape's frame: Sphere.cpp:99-108, Box.cpp:307-316,
// Polyhedron.cpp:265-293 (hill climbing over the vertex neighbours from the
// clone's current vertex, moving only on a gain of at least 1e-16).
V3 support(Shape const& s, int* curv, V3 const& v) {
  if (s.kind == 0) {
    double n = norm(v);
    if (n > EPSILON) { double r = s.radius / n; return V3(v[0] * r, v[1] * r, v[2] * r); }
    return V3();
  }
  if (s.kind == 3) {   // Cylinder::support (Cylinder.cpp:112-133), axis along local Y
    if (!(norm(v) > EPSILON)) return V3();
    double r = s.extent[0], hh = s.extent[1];
    double sxz = std::sqrt(v[0] * v[0] + v[2] * v[2]);
    if (sxz > EPSILON) {
      double d = r / sxz;
      if (std::fabs(v[1]) < EPSILON) return V3(v[0] * d, 0., v[2] * d);
      return V3(v[0] * d, v[1] < 0. ? -hh : hh, v[2] * d);
    }
    return V3(0., v[1] < 0. ? -hh : hh, 0.);
  }
  if (s.kind == 1) {
    if (norm(v) < EPSILON) return V3();
    return V3(v[0] < 0. ? -s.extent[0] : s.extent[0], v[1] < 0. ? -s.extent[1] : s.extent[1],
              v[2] < 0. ? -s.extent[2] : s.extent[2]);
  }
  if (!(norm(v) > EPSILON)) return V3();
  int last = -1;
  double h = dot(s.verts[*curv], v), d = 0.;
  for (;;) {
    std::vector<int> const& cb = s.cob[*curv];
    size_t i = 0, n = cb.size();
    while (i != n && (cb[i] == last || (d = dot(s.verts[cb[i]], v)) - h < 1.e-16)) ++i;
    if (i == n) break;
    last = *curv;
    *curv = cb[i];
    h = d;
  }
  return s.verts[*curv];
}

// Johnson's distance sub-algorithm as in Convex.cpp:219-430 (SOLID).
struct Simplex {
  V3 y[4], p[4], q[4];
  double det[16][4];
  double dp[4][4];
  Simplex() {
    for (auto& r : det) for (double& x : r) x = 0.;
    for (auto& r : dp) for (double& x : r) x = 0.;
  }
};

void computeDet(Simplex& S, unsigned bits, unsigned last, unsigned last_bit, unsigned all_bits) {
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

bool validSet(Simplex const& S, unsigned s, unsigned all_bits) {
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1) {
    if (all_bits & bit) {
      if (s & bit) { if (S.det[s][i] <= 1.0e-20) return false; }
      else if (S.det[s | bit][i] > 0) return false;
    }
  }
  return true;
}

V3 computeVector(Simplex const& S, unsigned bits) {
  double sum = 0.;
  V3 v(0., 0., 0.);
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if (bits & bit) { sum += S.det[bits][i]; v += S.det[bits][i] * S.y[i]; }
  return v * (1. / sum);
}

void computePoints(Simplex const& S, unsigned bits, V3& p1, V3& p2) {
  double sum = 0.;
  p1 = V3(0., 0., 0.);
  p2 = V3(0., 0., 0.);
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if (bits & bit) {
      sum += S.det[bits][i];
      p1 += S.det[bits][i] * S.p[i];
      p2 += S.det[bits][i] * S.q[i];
    }
  double s = 1. / sum;
  p1 = p1 * s;
  p2 = p2 * s;
}

bool properSet(Simplex const& S, unsigned s) {
  for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    if ((s & bit) && S.det[s][i] <= 1.0e-20) return false;
  return true;
}

bool closestSub(Simplex& S, unsigned& bits, unsigned last, unsigned last_bit, unsigned all_bits,
                V3& v) {
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
  double min_dist2 = INFINITY;
  for (unsigned s = all_bits; s; --s) {
    if ((s & all_bits) == s && properSet(S, s)) {
      V3 u = computeVector(S, s);
      double d2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
      if (d2 < min_dist2) { min_dist2 = d2; bits = s; v = u; }
    }
  }
  return false;
}

// closest_points (Convex.cpp:536-627), default settings: tolerance 1e-10,
// no acceleration.  pa/pb are in the shapes' own frames.
double closestPoints(Shape const& a, int* ca, XForm const& a2w, Shape const& b, int* cb,
                     XForm const& b2w, V3& pa, V3& pb, int& nIter) {
  unsigned bits = 0, last = 0, last_bit = 0, all_bits = 0;
  Simplex S;
  double mu = 0.;
  int numIterations = 0;
  const double relError = 1.e-10, absError = 1.e-4 * relError;
  V3 v = apply(a2w, support(a, ca, V3())) - apply(b2w, support(b, cb, V3()));
  V3 w = v;
  double dist = norm(v);
  while (bits < 15 && dist > 1.0e-15 && numIterations < 1000) {
    ++numIterations;
    last = 0;
    last_bit = 1;
    while (bits & last_bit) { ++last; last_bit <<= 1; }
    V3 d = v;
    S.p[last] = support(a, ca, tmul(-d, a2w));
    S.q[last] = support(b, cb, tmul(d, b2w));
    w = apply(a2w, S.p[last]) - apply(b2w, S.q[last]);
    mu = dist - dot(v, w) / dist;
    if (mu < dist * relError || mu < absError) break;
    bool degen = false;
    for (unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
      if ((all_bits & bit) && S.y[i][0] == w[0] && S.y[i][1] == w[1] && S.y[i][2] == w[2]) degen = true;
    if (degen) break;
    S.y[last] = w;
    all_bits = bits | last_bit;
    if (!closestSub(S, bits, last, last_bit, all_bits, v)) break;
    dist = norm(v);
  }
  computePoints(S, bits, pa, pb);
  nIter = numIterations;
  return dist;
}

// RigidBodyWithCrust::ClosestPoint, general branch (RigidBodyWithCrust.cpp:
// 277-351): bounding-sphere test, GJK between the crust-shrunk bodies,
// overlap = distance - crustA - crustB, contact at the witness midpoint.
PointContact convexContact(Shape const& a, int* ca, const double* basisA, V3 const& xa,
                           double crustA, Shape const& b, int* cb, const double* basisB,
                           V3 const& xb, double crustB, int* err) {
  PointContact pc;
  pc.contact = false;
  V3 gg = xa - xb;
  if (!(norm(gg) < a.radius + b.radius)) { pc.dist = 1.; return pc; }
  XForm a2w = crustTransform(basisA, a.scaling, xa);
  XForm b2w = crustTransform(basisB, b.scaling, xb);
  V3 pA, pB;
  int it = 0;
  double distance = closestPoints(a, ca, a2w, b, cb, b2w, pA, pB, it);
  if (distance < EPSILON) {
    // ContactError: the reference retries with a 10x crust shrink
    *err |= OR_ERR_CONTACT;
    pc.dist = 1.;
    return pc;
  }
  pA = apply(a2w, pA);
  pB = apply(b2w, pB);
  V3 ba = pA - pB;
  V3 contact = pA / 2.0 + pB / 2.0;
  V3 ov = ba / distance;
  round3(ov);
  ov = ov * (crustA + crustB - distance);
  distance -= crustA + crustB;
  pc.point = contact;
  pc.overlap = ov;
  pc.dist = distance;
  pc.contact = true;
  return pc;
}

// ------------------------------------------------------------ force model --
// HookeMemoryContactForceModel::computeTangentialVector (:54-65)
V3 tangentVector(Model const& m, double n_t, V3 const& ut, V3 const& kdelta) {
  if (norm(ut) > 0.001) return (-ut) / norm(ut);
  V3 s = kdelta + n_t * ut;
  if ((norm(kdelta) > m.epst || norm(n_t * ut) > m.epst) && norm(s) > m.epst)
    return (-s) / norm(s);
  return V3(0., 0., 0.);
}

struct Body {      // view of p0 / p1 as the force model sees them
  V3 x, v, w;
  double mass, rad;
  std::map<Key, Hist>* cmap;
  int id;
};

// performForcesCalculus (:72-193) + computeForces (:200-249)
void hookeMemory(Model const& m, Body& p0, Body& p1, double dt, PointContact const& ci,
                 V3& fOn0, V3& mOn0) {
  V3 pcp = ci.point;
  V3 pen = ci.overlap;
  Key id0 = std::make_tuple(1, p1.id, 1);
  Key id1 = std::make_tuple(1, p0.id, 1);
  V3 normal = pen;
  normal = normal / norm(normal);
  round3(normal);
  V3 v0 = p0.v + cross(p0.w, pcp - p0.x);
  V3 v1 = p1.v + cross(p1.w, pcp - p1.x);
  V3 tmpV = v0 - v1;
  V3 v_n = normal * dot(tmpV, normal);
  V3 v_t = tmpV - v_n;
  V3 delFN = m.kn * pen;
  double avmass = 1. / (1. / p0.mass + 1. / p1.mass);
  double gamman = -2. * m.beta * std::sqrt(avmass * m.kn);
  delFN -= gamman * v_n;
  double normFN = norm(delFN);
  double etat = m.etat == -1. ? -m.beta * std::sqrt(m.kn / avmass) : m.etat;
  double gammat = 2. * etat * avmass;
  V3 viscousFT = -gammat * v_t;
  // Component::getContactMemory (Component.cpp:634-670)
  bool existed;
  auto it = p0.cmap->find(id0);
  if (it != p0.cmap->end()) { existed = true; it->second.active = true; }
  else {
    existed = false;
    Hist h; h.active = true;
    it = p0.cmap->insert(std::make_pair(id0, h)).first;
  }
  Hist& H = it->second;
  Q qrot = qmake(V3(0., 0., 0.), 0.);
  if (existed) {
    qrot = rotFromTwoVectors(H.prevn, normal);
    H.kdelta = rotateVector(qrot, H.kdelta);
  }
  H.kdelta += (dt * m.kt) * v_t;
  H.prevn = normal;
  V3 tij = tangentVector(m, gammat, v_t, H.kdelta);
  double normFT = norm(-H.kdelta + viscousFT);
  V3 delFT;
  if (normFT <= m.muc * normFN) delFT = norm(-H.kdelta + viscousFT) * tij;
  else {
    if (m.kt) H.kdelta = ((-m.muc * normFN) * tij + viscousFT) / m.kt;
    delFT = (m.muc * normFN) * tij;
  }
  V3 delM;
  if (m.rolling) {
    double Req = 1. / (1. / p0.rad + 1. / p1.rad);
    double kr = 3. * m.kn * m.mur * m.mur * Req * Req;
    double etar = 3. * gamman * m.mur * m.mur * Req * Req;
    double maxM = m.mur * Req * normFN;
    V3 wrel = p0.w - p1.w;
    if (existed) H.spring = rotateVector(qrot, H.spring);
    H.spring -= (kr * dt) * wrel;
    double nM = norm(H.spring);
    if (nM > maxM) H.spring = H.spring * (maxM / nM);
    delM = H.spring - (m.etarpf * etar) * wrel;
  }
  // Component::addDeplContactInMap on p1 (Component.cpp:677-689)
  if (p1.cmap) {
    Hist& H1 = (*p1.cmap)[id1];
    H1.active = true;
    H1.kdelta = -H.kdelta;
    H1.prevn = -normal;
    H1.spring = -H.spring;
  }
  fOn0 = 1. * (delFN + delFT);
  mOn0 = delM;
}

// HookeContactForceModel::performForcesCalculus (HookeContactForceModel.cpp:
// 44-121): the same normal law without tangential memory; the viscous
// tangential force is capped at muc |Fn|, and the optional rolling moment is
// kr Req |Fn| |w x r|_rel / |w_rel| against w_rel.
void hooke(Model const& m, Body const& p0, Body const& p1, PointContact const& ci, V3& fOn0,
           V3& mOn0) {
  V3 pcp = ci.point;
  V3 pen = ci.overlap;
  V3 normal = pen;
  normal = normal / norm(normal);
  round3(normal);
  V3 v0 = p0.v + cross(p0.w, pcp - p0.x);
  V3 v1 = p1.v + cross(p1.w, pcp - p1.x);
  V3 tmpV = v0 - v1;
  V3 v_n = normal * dot(tmpV, normal);
  V3 v_t = tmpV - v_n;
  V3 delFN = m.kn * pen;
  double avmass = 1. / (1. / p0.mass + 1. / p1.mass);
  double gamman = -2. * m.beta * std::sqrt(avmass * m.kn);
  delFN -= gamman * v_n;
  double normFN = norm(delFN);
  double etat = m.etat == -1. ? -m.beta * std::sqrt(m.kn / avmass) : m.etat;
  double gammat = 2. * etat * avmass;
  V3 delFT = -gammat * v_t;
  double fn = m.muc * normFN;
  double ft = norm(delFT);
  if (fn < ft) {
    double normv_t = norm(v_t);
    V3 tangent(0., 0., 0.);
    if (normv_t > EPSILON) tangent = (-v_t) / normv_t;
    delFT = tangent * fn;
  }
  V3 delM(0., 0., 0.);
  if (m.kr != 0.) {
    V3 wrel = p0.w - p1.w;
    double normwrel = norm(wrel);
    double normwtrel = norm(cross(p0.w, p0.x - pcp) - cross(p1.w, p1.x - pcp));
    if (normwrel > EPSILON) {
      double Req = 1. / (1. / p0.rad + 1. / p1.rad);
      delM = -(m.kr * Req * normFN * normwtrel / normwrel) * wrel;
    }
  }
  fOn0 = 1. * (delFN + delFT);
  mOn0 = delM * 1.;
}

void contactLaw(Model const& m, Body& b0, Body& b1, double dt, PointContact const& pc, V3& f,
                V3& mm) {
  if (m.memory) hookeMemory(m, b0, b1, dt, pc, f, mm);
  else hooke(m, b0, b1, pc, f, mm);
}

void addForce(Particle& p, V3 const& point, V3 const& f) {   // Torsor::addForce
  p.F += f;
  V3 a = point - p.ref;
  p.T += cross(a, f);
}

// Particle::InterAction + HookeMemory::computeForces for a particle pair
void interactPP(System& s, Particle& p0, Particle& p1, V3 const& shift) {
  V3 xb = p1.x + shift;
  PointContact pc;
  if (p0.shape->kind == 0 && p1.shape->kind == 0) pc = sphereSphere(p0, xb, p1, &s.err);
  else
    pc = convexContact(*p0.shape, &p0.curv, p0.basis, p0.x, p0.crust, *p1.shape, &p1.curv,
                       p1.basis, xb, p1.crust, &s.err);
  if (!pc.contact || !(pc.dist < 0.)) return;
  Model const& m = s.model(p0.matbit, p1.matbit);
  Body b0{p0.x, p0.v, p0.w, p0.mass, p0.eqrad, &p0.cmap, p0.id};
  Body b1{xb, p1.v, p1.w, p1.mass, p1.eqrad, &p1.cmap, p1.id};
  V3 f, mm;
  contactLaw(m, b0, b1, s.dt, pc, f, mm);
  addForce(p0, pc.point, f);
  if (m.rolling) p0.T += mm;
  // p1 torque lever arm uses its own (image) reference point
  V3 fm = (-f);
  p1.F += fm;
  V3 arm = pc.point - (p1.ref + shift);
  p1.T += cross(arm, fm);
  if (m.rolling) p1.T += (-mm);
  ContactRec r{p0.id, p1.id, pc.dist, pc.point, pc.overlap, f};
  s.contacts.push_back(r);
}

// SimpleObstacle::InterAction: the particle is p0, the wall p1
void interactPW(System& s, Particle& p, Wall& w, int k) {
  static const double I3[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  PointContact pc;
  if (p.shape->kind == 0) {
    pc = sphereWall(p, w, &s.err);
  } else {
    // SimpleObstacle::InterAction: bounding-box zone test, then the particle
    // is A and the wall B of RigidBodyWithCrust::ClosestPoint
    int wc = 0;
    pc = convexContact(*p.shape, &p.curv, p.basis, p.x, p.crust, w.shape, &wc, I3, w.centre,
                       w.crust, &s.err);
  }
  if (!pc.contact || !(pc.dist < 0.)) return;
  Model const& m = s.model(p.matbit, w.matbit);
  Body b0{p.x, p.v, p.w, p.mass, p.eqrad, &p.cmap, p.id};
  Body b1{V3(), V3(), V3(), 1.e20, 0., nullptr, w.id};   // Component::m_massObstacle
  // Component::getEquivalentSphereRadius (Component.cpp:205-208) of the box
  b1.x = w.centre;
  b1.rad = std::pow((0.75 / PI) * (8. * w.extent[0] * w.extent[1] * w.extent[2]), 1. / 3.);
  V3 f, mm;
  contactLaw(m, b0, b1, s.dt, pc, f, mm);
  addForce(p, pc.point, f);
  if (m.rolling) p.T += mm;
  ContactRec r{p.id, w.id, pc.dist, pc.point, pc.overlap, f};
  s.contacts.push_back(r);
}

// Grains::computeParticlesForceAndTorque + LinkedCell::ComputeForces
void computeForces(System& s) {
  s.contacts.clear();
  for (auto& p : s.parts)
    for (auto& kv : p.cmap) kv.second.active = false;    // setContactMapToFalse
  for (auto& p : s.parts) {                              // InitializeForce
    p.F = p.weight;
    p.T = V3(0., 0., 0.);
    p.ref = p.x;
  }
  std::vector<int> nbrs;
  std::vector<V3> shifts;
  for (size_t ip = 0; ip < s.parts.size(); ++ip) {
    Particle& p = s.parts[ip];
    int id[3];
    s.getCell(p.x, id);
    int cn = s.cellnum(id[0], id[1], id[2]);
    nbrs.clear(); shifts.clear();
    std::list<int>& own = s.cells[cn];
    auto it = std::find(own.begin(), own.end(), p.id);
    for (++it; it != own.end(); ++it) { nbrs.push_back(*it); shifts.push_back(V3()); }
    for (int jn : s.nbr_order) {
      int sh[3];
      int c = neighbourCell(s, id[0] + STENCIL[0][jn], id[1] + STENCIL[1][jn],
                            id[2] + STENCIL[2][jn], sh);
      if (c < 0) continue;
      V3 shift(sh[0] * s.dom_size[0], sh[1] * s.dom_size[1], sh[2] * s.dom_size[2]);
      for (int q : s.cells[c]) { nbrs.push_back(q); shifts.push_back(shift); }
    }
    for (size_t n = 0; n < nbrs.size(); ++n)
      if (nbrs[n] != p.id) interactPP(s, p, s.parts[nbrs[n]], shifts[n]);
    for (size_t k = 0; k < s.walls.size(); ++k) interactPW(s, p, s.walls[k], (int)k);
  }
  for (auto& p : s.parts) {                              // updateContactMap
    for (auto it = p.cmap.begin(); it != p.cmap.end();) {
      if (!it->second.active) it = p.cmap.erase(it); else ++it;
    }
  }
}

// LinkedCell::LinkUpdateActiveParticle
void linkUpdate(System& s) {
  for (auto& p : s.parts) {
    int id[3];
    s.getCell(p.x, id);
    if (!s.valid(id[0], id[1], id[2])) { s.err |= OR_ERR_OUT_OF_GRID; continue; }
    int cn = s.cellnum(id[0], id[1], id[2]);
    if (cn != p.cellnum) {
      s.cells[cn].push_front(p.id);
      s.cells[p.cellnum].remove(p.id);
      p.cellnum = cn;
    }
    p.cell[0] = id[0]; p.cell[1] = id[1]; p.cell[2] = id[2];
  }
}

void step(System& s) {
  double dt = s.dt;
  s.time += dt;
  for (auto& p : s.parts) {
    double depl = moveParticle(p, 0.5 * dt, dt);
    if (depl > p.crust) s.err |= OR_ERR_MOTION;
    wrapPeriodic(s, p);
  }
  linkUpdate(s);
  computeForces(s);
  for (auto& p : s.parts) advanceVelocity(p, 0.5 * dt);
}

}  // namespace

extern "C" {

// GrainsExec::computeVolumeInertiaContrib (Base/src/GrainsExec.cpp:746-797):
// volume and inertia of the tetrahedron (origin, A2, A3, A4), Tonon (2004).
void tetContrib(V3 const& A2, V3 const& A3, V3 const& A4, double& vol, double* I) {
  double x1 = 0., x2 = A2[0], x3 = A3[0], x4 = A4[0];
  double y1 = 0., y2 = A2[1], y3 = A3[1], y4 = A4[1];
  double z1 = 0., z2 = A2[2], z3 = A3[2], z4 = A4[2];
  double det = std::fabs((x2 - x1) * (y3 - y1) * (z4 - z1) + (y2 - y1) * (z3 - z1) * (x4 - x1) +
                         (z2 - z1) * (x3 - x1) * (y4 - y1) - (z2 - z1) * (y3 - y1) * (x4 - x1) -
                         (x2 - x1) * (z3 - z1) * (y4 - y1) - (y2 - y1) * (x3 - x1) * (z4 - z1));
  vol += det / 6.;
  I[0] += det * (y1 * y1 + y1 * y2 + y2 * y2 + y1 * y3 + y2 * y3 + y3 * y3 + y1 * y4 + y2 * y4 +
                 y3 * y4 + y4 * y4 + z1 * z1 + z1 * z2 + z2 * z2 + z1 * z3 + z2 * z3 + z3 * z3 +
                 z1 * z4 + z2 * z4 + z3 * z4 + z4 * z4) / 60.;
  I[3] += det * (x1 * x1 + x1 * x2 + x2 * x2 + x1 * x3 + x2 * x3 + x3 * x3 + x1 * x4 + x2 * x4 +
                 x3 * x4 + x4 * x4 + z1 * z1 + z1 * z2 + z2 * z2 + z1 * z3 + z2 * z3 + z3 * z3 +
                 z1 * z4 + z2 * z4 + z3 * z4 + z4 * z4) / 60.;
  I[5] += det * (x1 * x1 + x1 * x2 + x2 * x2 + x1 * x3 + x2 * x3 + x3 * x3 + x1 * x4 + x2 * x4 +
                 x3 * x4 + x4 * x4 + y1 * y1 + y1 * y2 + y2 * y2 + y1 * y3 + y2 * y3 + y3 * y3 +
                 y1 * y4 + y2 * y4 + y3 * y4 + y4 * y4) / 60.;
}

// Shape of particle class t: geometry, volume, inertia (Sphere / Box /
// Polyhedron BuildInertia, getVolume, computeCircumscribedRadius) and the
// crust scaling from the identity-frame bounding box (RigidBodyWithCrust ctor,
// RigidBodyWithCrust.cpp:58-78; Convex::bbox, Convex.cpp:29-41).
Shape makeShape(or_config const* c, int t) {
  Shape sh;
  sh.kind = c->type_shape ? c->type_shape[t] : 0;
  double crust = c->type_crust[t];
  if (sh.kind == 0) {
    double r = c->type_radius[t];
    sh.radius = r;
    sh.volume = 4.0 * PI * std::pow(r, 3.) / 3.0;
    double I = 8.0 * PI * std::pow(r, 5.) / 15.0;
    sh.inertia[0] = sh.inertia[3] = sh.inertia[5] = I;
    sh.extent = V3(r, r, r);
  } else if (sh.kind == 1) {
    V3 e(c->type_extent[3 * t], c->type_extent[3 * t + 1], c->type_extent[3 * t + 2]);
    sh.extent = e;
    sh.radius = norm(e);
    sh.volume = 8.0 * e[0] * e[1] * e[2];
    sh.inertia[0] = 8.0 * e[0] * e[1] * e[2] * (e[1] * e[1] + e[2] * e[2]) / 3.0;
    sh.inertia[3] = 8.0 * e[0] * e[1] * e[2] * (e[0] * e[0] + e[2] * e[2]) / 3.0;
    sh.inertia[5] = 8.0 * e[0] * e[1] * e[2] * (e[0] * e[0] + e[1] * e[1]) / 3.0;
  } else if (sh.kind == 3) {
    // Cylinder (Geometry/src/Cylinder.cpp): radius r, half height hh; the
    // class extent holds (r, hh, r)
    double r = c->type_extent[3 * t], hh = c->type_extent[3 * t + 1];
    sh.extent = V3(r, hh, r);
    sh.radius = std::sqrt(r * r + hh * hh);                    // computeCircumscribedRadius
    sh.volume = 2 * hh * PI * r * r;                           // getVolume
    double constant = 0.5 * hh * r * r * PI;                   // BuildInertia
    sh.inertia[0] = sh.inertia[5] = constant * (4.0 * hh * hh / 3.0 + r * r);
    sh.inertia[3] = 2.0 * constant * r * r;
  } else {
    const int* P = c->type_poly + 4 * t;
    for (int k = 0; k < P[1]; ++k) {
      const double* v = c->poly_verts + 3 * (P[0] + k);
      sh.verts.push_back(V3(v[0], v[1], v[2]));
    }
    sh.cob.assign(sh.verts.size(), std::vector<int>());
    const int* f = c->poly_faces + P[2];
    const int* fend = f + P[3];
    double vol = 0.;
    double I[6] = {0, 0, 0, 0, 0, 0};
    while (f < fend) {
      int nf = *f++;
      for (int j = 0, k = nf - 1; j < nf; k = j++) sh.cob[f[k]].push_back(f[j]);
      if (nf == 3) {
        tetContrib(sh.verts[f[0]], sh.verts[f[1]], sh.verts[f[2]], vol, I);
      } else {
        V3 G;
        for (int j = 0; j < nf; ++j) G += sh.verts[f[j]];
        G = G / double(nf);
        for (int j = 0, k = nf - 1; j < nf; k = j++) tetContrib(G, sh.verts[f[k]], sh.verts[f[j]], vol, I);
      }
      f += nf;
    }
    sh.volume = vol;
    for (int k = 0; k < 6; ++k) sh.inertia[k] = I[k];
    double ray = dot(sh.verts[0], sh.verts[0]);
    for (size_t k = 1; k < sh.verts.size(); ++k) {
      double d = dot(sh.verts[k], sh.verts[k]);
      if (d > ray) ray = d;
    }
    sh.radius = std::sqrt(ray);
    int cv = 0;
    V3 mn, mx;
    for (int d = 0; d < 3; ++d) {
      V3 e; e[d] = 1.;
      mn[d] = support(sh, &cv, -e)[d];
      mx[d] = support(sh, &cv, e)[d];
    }
    sh.extent = (mx - mn) / 2.;
  }
  for (int d = 0; d < 3; ++d)
    sh.scaling[d] = sh.extent[d] < EPSILON ? 1. : (sh.extent[d] - crust) / sh.extent[d];
  return sh;
}

void* or_create(or_config const* c) {
  System* s = new System();
  for (int d = 0; d < 3; ++d) {
    s->dom_origin[d] = c->origin[d];
    s->dom_size[d] = c->maxc[d] - c->origin[d];   // App::set_dimensions
    s->periodic[d] = c->periodic[d] ? 1 : 0;
    s->gravity[d] = c->gravity[d];
  }
  s->dt = c->dt;
  for (int t = 0; t < c->n_types; ++t) {
    s->shapes.push_back(makeShape(c, t));
    s->type_radius.push_back(s->shapes.back().radius);
    s->type_crust.push_back(c->type_crust[t]);
    s->type_density.push_back(c->type_density[t]);
    s->type_matbit.push_back(c->type_matbit[t]);
  }
  for (int k = 0; k < c->n_walls; ++k) {
    Wall w;
    w.id = -(k + 2);
    w.centre = V3(c->wall_centre[3*k], c->wall_centre[3*k+1], c->wall_centre[3*k+2]);
    w.extent = V3(c->wall_extent[3*k], c->wall_extent[3*k+1], c->wall_extent[3*k+2]);
    w.crust = c->wall_crust[k];
    w.matbit = c->wall_matbit[k];
    w.shape.kind = 1;
    w.shape.extent = w.extent;
    w.shape.radius = norm(w.extent);
    for (int d = 0; d < 3; ++d)
      w.shape.scaling[d] = w.extent[d] < EPSILON ? 1. : (w.extent[d] - w.crust) / w.extent[d];
    s->walls.push_back(w);
  }
  for (int k = 0; k < c->n_models; ++k) {
    const double* q = c->model_params + 10 * k;
    Model m;
    m.kn = q[0]; m.en = q[1]; m.etat = q[2]; m.muc = q[3];
    m.kt = q[4]; m.mur = q[5]; m.etarpf = q[6]; m.epst = q[7];
    m.kr = q[8];
    m.memory = q[9] != 0.;
    m.rolling = m.memory ? m.mur != 0. : m.kr != 0.;
    m.beta = std::log(m.en) / std::sqrt(PI * PI + std::log(m.en) * std::log(m.en));
    s->models[c->model_mask[k]] = m;
  }
  double maxR = 0.;
  for (double r : s->type_radius) maxR = std::max(maxR, r);
  double coef = c->cell_size_factor < 1. ? 1. : c->cell_size_factor;
  setGrid(*s, 2. * (coef * maxR));
  return s;
}

void or_destroy(void* h) { delete static_cast<System*>(h); }

// Particles are inserted in index order (ID = index) and linked to their
// cell with push_front, as LinkedCell::Link does at insertion.
int or_set_particles(void* h, int n, const int* type, const double* x, const double* v,
                     const double* w, const double* q, const double* basis) {
  System& s = *static_cast<System*>(h);
  s.parts.clear();
  for (auto& c : s.cells) c.clear();
  s.parts.resize(n);
  for (int i = 0; i < n; ++i) {
    Particle& p = s.parts[i];
    int t = type[i];
    p.id = i; p.type = t;
    p.shape = &s.shapes[t];
    p.radius = s.type_radius[t];
    p.crust = s.type_crust[t];
    p.density = s.type_density[t];
    p.matbit = s.type_matbit[t];
    double vol = p.shape->volume;
    p.mass = p.density * vol;                                       // Particle.cpp:150
    p.eqrad = std::pow((0.75 / PI) * vol, 1. / 3.);
    p.I[0] = p.shape->inertia[0] * p.density;                       // Particle.cpp:152-157
    p.I[1] = p.shape->inertia[3] * p.density;
    p.I[2] = p.shape->inertia[5] * p.density;
    p.inertia = p.I[0];
    p.weight = V3(s.gravity[0], s.gravity[1], s.gravity[2]) * (p.mass * (1. - 0. / p.density));
    p.x = V3(x[3*i], x[3*i+1], x[3*i+2]);
    p.v = V3(v[3*i], v[3*i+1], v[3*i+2]);
    p.w = V3(w[3*i], w[3*i+1], w[3*i+2]);
    p.q = qmake(V3(q[4*i], q[4*i+1], q[4*i+2]), q[4*i+3]);
    // angular velocity in body frame: q* (w, q) (ParticleKinematics.cpp:220-221)
    p.wbf = multToVector3(conj(p.q), vecq(p.w, p.q));
    for (int k = 0; k < 9; ++k) p.basis[k] = basis ? basis[9 * i + k] : ((k % 4 == 0) ? 1. : 0.);
    p.F = V3(); p.T = V3();
    int id[3];
    s.getCell(p.x, id);
    if (!s.valid(id[0], id[1], id[2])) return OR_ERR_OUT_OF_GRID;
    p.cellnum = s.cellnum(id[0], id[1], id[2]);
    p.cell[0] = id[0]; p.cell[1] = id[1]; p.cell[2] = id[2];
    s.cells[p.cellnum].push_front(i);
  }
  return OR_OK;
}

// Leapfrog start (Grains.cpp:168-173): forces at t0, then zero the
// cumulative tangential and rolling memories.
int or_init(void* h) {
  System& s = *static_cast<System*>(h);
  s.err = 0;
  computeForces(s);
  for (auto& p : s.parts)
    for (auto& kv : p.cmap) { kv.second.kdelta = V3(); kv.second.spring = V3(); }
  return s.err;
}

int or_step(void* h, int nsteps) {
  System& s = *static_cast<System*>(h);
  s.err = 0;
  for (int k = 0; k < nsteps; ++k) step(s);
  return s.err;
}

// State arrays are indexed by particle ID.  w is the space-fixed angular
// velocity, wbf the body-fixed one.
void or_get_state(void* h, double* x, double* v, double* w, double* wbf, double* q,
                  double* F, double* T) {
  System& s = *static_cast<System*>(h);
  for (size_t i = 0; i < s.parts.size(); ++i) {
    Particle& p = s.parts[i];
    for (int d = 0; d < 3; ++d) {
      if (x) x[3*i+d] = p.x[d];
      if (v) v[3*i+d] = p.v[d];
      if (w) w[3*i+d] = p.w[d];
      if (wbf) wbf[3*i+d] = p.wbf[d];
      if (F) F[3*i+d] = p.F[d];
      if (T) T[3*i+d] = p.T[d];
    }
    if (q) { q[4*i] = p.q.v[0]; q[4*i+1] = p.q.v[1]; q[4*i+2] = p.q.v[2]; q[4*i+3] = p.q.w; }
  }
}

void or_get_basis(void* h, double* basis) {
  System& s = *static_cast<System*>(h);
  for (size_t i = 0; i < s.parts.size(); ++i)
    for (int k = 0; k < 9; ++k) basis[9 * i + k] = s.parts[i].basis[k];
}

// Polyhedron::m_curr_vertex of every particle (0 for other shapes).
void or_get_curv(void* h, int* out) {
  System& s = *static_cast<System*>(h);
  for (size_t i = 0; i < s.parts.size(); ++i) out[i] = s.parts[i].curv;
}

void or_get_cells(void* h, int* ijk) {
  System& s = *static_cast<System*>(h);
  for (size_t i = 0; i < s.parts.size(); ++i)
    for (int d = 0; d < 3; ++d) ijk[3*i+d] = s.parts[i].cell[d];
}

void or_get_grid(void* h, int* nb, double* edge, double* lc_origin) {
  System& s = *static_cast<System*>(h);
  for (int d = 0; d < 3; ++d) { nb[d] = s.nb[d]; edge[d] = s.edge[d]; lc_origin[d] = s.lc_origin[d]; }
}

int or_num_contacts(void* h) { return (int)static_cast<System*>(h)->contacts.size(); }

// Contacts of the last force evaluation, in evaluation order.  id1 < 0 is a
// wall k as -(k+2).  f is the force on id0.
void or_get_contacts(void* h, int* id0, int* id1, double* delta, double* point, double* f) {
  System& s = *static_cast<System*>(h);
  for (size_t k = 0; k < s.contacts.size(); ++k) {
    ContactRec& r = s.contacts[k];
    id0[k] = r.id0; id1[k] = r.id1; delta[k] = r.delta;
    for (int d = 0; d < 3; ++d) { point[3*k+d] = r.point[d]; f[3*k+d] = r.force[d]; }
  }
}

int or_num_history(void* h) {
  System& s = *static_cast<System*>(h);
  int n = 0;
  for (auto& p : s.parts) n += (int)p.cmap.size();
  return n;
}

// Contact memory entries: owner ID, partner ID (wall: -(k+2)), kdelta,
// previous normal, spring torque.
void or_get_history(void* h, int* owner, int* partner, double* kdelta, double* prevn,
                    double* spring) {
  System& s = *static_cast<System*>(h);
  int n = 0;
  for (auto& p : s.parts)
    for (auto& kv : p.cmap) {
      owner[n] = p.id; partner[n] = std::get<1>(kv.first);
      for (int d = 0; d < 3; ++d) {
        kdelta[3*n+d] = kv.second.kdelta[d];
        prevn[3*n+d] = kv.second.prevn[d];
        spring[3*n+d] = kv.second.spring[d];
      }
      ++n;
    }
}

}  // extern "C"
