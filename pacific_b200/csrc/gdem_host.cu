// gdem_host.cu -- host runtime behind the C ABI of include/grains_b200.h.
//
// Builds the device descriptors from Grains3D XML input (same element and
// attribute names as Grains::Construction, Base/src/Grains.cpp:535-1030, and
// the contact-model factory, Component/src/ContactBuilderFactory.cpp:88-169),
// owns every device buffer, and sequences the kernels of one leapfrog step
// (Grains::Simulation, Grains.cpp:344-364).  A gdem_step call is:
//
//   k_move (opening kick dt/2 + drift dt with the stored F, T), then per step
//   k_decide -> [pair-list rebuild, when some particle moved half the skin:
//                k_bin, scan, k_place, k_cellsort, k_permute, k_copyback,
//                k_pairs_count, row scan, k_pairs_fill, k_link]
//   -> k_filter (kept pairs, particles near a wall)
//   -> k_pairlaw (narrow phase, contact law, history; shares into the rows)
//   -> k_move (sums of the shares; closing kick, next opening kick + drift)
//
// Each step is one captured CUDA graph (the rebuild inside a conditional
// node); two graphs alternate with the contact-history tables.
#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/grains_b200.h"
#include "gdem_kernels.cuh"
#include "gdem_setup.h"
#include "xml_reader.hpp"

namespace gdem {

namespace {

thread_local std::string g_last_error;
const double PI = 3.14159265358979323846;
// steps between two checks of the pair list's allocation within a call
constexpr int kCapacityCheck = 512;

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_));           \
  } while (0)

template <typename T>
T* dalloc(size_t count) {
  void* p = nullptr;
  if (count == 0) count = 1;
  CK(cudaMalloc(&p, count * sizeof(T)));
  return static_cast<T*>(p);
}

int nextPow2Log(size_t n) {
  int l = 10;
  while ((size_t(1) << l) < n) ++l;
  return l;
}

// ----------------------------------------------------------- XML import --
struct InstanceDesc {
  GridDesc grid;        // the reference linked-cell grid
  GridDesc bgrid;       // the pair-list grid: cells of at least 2 rmax f + skin
  std::vector<TypeDesc> types;
  std::vector<WallDesc> walls;
  std::vector<double> poly_verts;   // polyhedron vertices of this instance (x, y, z)
  // each polyhedron vertex's neighbours (Polyhedron::m_cobound), aligned with
  // poly_verts: indices within the vertex's polyhedron
  std::vector<std::vector<int>> poly_cob;
  // per class, a polyhedron's faces as its file lists them (empty otherwise)
  std::vector<std::vector<std::vector<int>>> class_faces;
  ModelDesc models[kMaxMat * kMaxMat];
  double gravity[3];
  double dt;
  // coupled runs (GrainsCoupledWithFluid::AdditionalFeatures,
  // Fluid/src/GrainsCoupledWithFluid.cpp:510-530): TimeStep mindt, maxdt,
  // ndt; a plain run's dt is all three
  double min_dt, max_dt;
  int ndt;
  std::string reload_file;   // Construction/Reload Filename, if any
  bool reload_reset = false; // Reload Velocity="Reset": kinematics zeroed on reading
  std::string rawdata_root;  // Simulation/PostProcessing/Writers/RawData Name, if any
  bool rawdata_binary = false;
  int nmat;
  std::vector<std::string> mat_names;   // material name of each index
  // what the pair-list grid is made from (it is remade when the skin changes)
  double box_org[3], box_max[3];
  int box_per[3];
  double cellsize;      // 2 rmax f: the reference cell size
  double max_radius;    // largest circumscribed radius
  double xml_skin;      // LinkedCell Skin attribute, or < 0 when absent
};

// Pair-list grid of one instance for a skin (a length).  The list holds the
// pairs whose bounding spheres are closer than the skin and stays valid while
// no particle has moved more than skin / 2, so its cells must be at least
// 2 rmax f + skin wide; the skin shrinks when a periodic direction would get
// fewer than 3 cells.  Only the cell layout and the skin change; the fields
// shared with the reference grid (safe bands, periods, filter margin) stay.
void makePairGrid(InstanceDesc& I, double skin) {
  if (!(skin >= 0.)) throw std::runtime_error("LinkedCell Skin must be >= 0");
  for (int d = 0; d < 3; ++d)
    if (I.box_per[d])
      skin = std::min(skin, std::max(0., (I.box_max[d] - I.box_org[d]) / 3. - I.cellsize) * 0.999999);
  GridDesc& b = I.bgrid;
  for (int d = 0; d < 3; ++d) {
    double size = I.box_max[d] - I.box_org[d];
    int n = (int)((size + 1.0e-10) / (I.cellsize + skin));
    if (!n) n = 1;
    if (I.box_per[d] && n < 3) n = 3;
    b.nb[d] = n;
    b.edge[d] = size / n;
    b.lc_origin[d] = I.box_org[d];
    if (I.box_per[d]) {
      b.lc_origin[d] += -b.edge[d];
      b.nb[d] += 2;
    }
    b.edge_f[d] = (float)b.edge[d];
  }
  b.skin = skin;
  b.skin_f = (float)skin;
}

int materialIndex(std::map<std::string, int>& mats, std::vector<std::string>& order,
                  std::string const& name) {
  auto it = mats.find(name);
  if (it != mats.end()) return it->second;
  int idx = (int)order.size();
  if (idx >= kMaxMat) throw std::runtime_error("more than 8 materials");
  mats[name] = idx;
  order.push_back(name);
  return idx;
}

double childD(XmlNode const* n, const char* name, bool required, double dflt) {
  XmlNode const* c = n->child(name);
  if (!c) {
    if (required) throw std::runtime_error(std::string("missing <") + name + ">");
    return dflt;
  }
  return c->valueD();
}

// HookeMemoryContactForceModel::defineParameters (:256-310) and
// HookeContactForceModel::defineParameters (HookeContactForceModel.cpp:
// 170-200, where <kr> is required).  A missing <epst> leaves epst at zero in
// the reference (the default is stored under the key "eps").
ModelDesc readModel(XmlNode const* law, std::string const& kind) {
  ModelDesc m{};
  m.kn = childD(law, "kn", true, 0.);
  m.muc = childD(law, "muc", true, 0.);
  m.en = childD(law, "en", true, 0.);
  m.etat = childD(law, "etat", false, -1.);
  m.mur = childD(law, "mur", false, 0.);
  m.etarpf = childD(law, "etarpf", false, 0.);
  m.kt = childD(law, "kt", kind == "HookeMemory", 0.);
  m.epst = childD(law, "epst", false, 0.);
  m.kr = childD(law, "kr", kind == "Hooke", 0.);
  m.memory = kind == "HookeMemory" ? 1 : 0;
  m.rolling = (m.memory ? m.mur != 0. : m.kr != 0.) ? 1 : 0;
  m.beta = std::log(m.en) / std::sqrt(PI * PI + std::log(m.en) * std::log(m.en));
  m.valid = 1;
  return m;
}

void collectObstacles(XmlNode const* n, std::vector<XmlNode const*>& out) {
  for (auto const& c : n->children) {
    if (c->name == "Obstacle") out.push_back(c.get());
    else if (c->name == "Composite") collectObstacles(c.get(), out);
  }
}

// Polyhedron description file (Polyhedron::create and Polyhedron::readface,
// Geometry/src/Polyhedron.cpp:143-180, 580-620): "<token> <nb_vertices>", one
// vertex per line, "<nb_faces>", then one line of vertex indices per face.
struct PolyFile {
  std::vector<std::array<double, 3>> verts;
  std::vector<std::vector<int>> faces;
};

PolyFile readPolyFile(std::string const& path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open polyhedron file " + path);
  PolyFile P;
  int tok = 0, nv = 0, nf = 0;
  if (!(in >> tok >> nv) || nv < 4) throw std::runtime_error("bad polyhedron header in " + path);
  P.verts.resize(nv);
  for (auto& v : P.verts)
    if (!(in >> v[0] >> v[1] >> v[2])) throw std::runtime_error("bad polyhedron vertex in " + path);
  if (!(in >> nf) || nf < 4) throw std::runtime_error("bad polyhedron face count in " + path);
  std::string line;
  std::getline(in, line);
  for (int f = 0; f < nf; ++f) {
    if (!std::getline(in, line)) throw std::runtime_error("missing polyhedron face in " + path);
    std::istringstream ls(line);
    std::vector<int> face;
    int k;
    while (ls >> k) {
      if (k < 0 || k >= nv) throw std::runtime_error("polyhedron face index out of range in " + path);
      face.push_back(k);
    }
    if (face.size() < 3) throw std::runtime_error("polyhedron face with fewer than 3 vertices in " + path);
    P.faces.push_back(face);
  }
  return P;
}

// Volume and principal inertia (unit density) of the tetrahedron (origin, a,
// b, c), by Tonon's closed form (F. Tonon, J. Math. Stat. 1 (2004) 8-11), as
// used by GrainsExec::computeVolumeInertiaContrib (Base/src/GrainsExec.cpp:
// 746-797).  The sums run in the same order as there so that the masses agree
// to the last bit.
void tetMass(std::array<double, 3> const& a, std::array<double, 3> const& b,
             std::array<double, 3> const& c, double& vol, double* I) {
  const double o = 0.;
  double x2 = a[0], x3 = b[0], x4 = c[0], y2 = a[1], y3 = b[1], y4 = c[1];
  double z2 = a[2], z3 = b[2], z4 = c[2];
  double det = std::fabs((x2 - o) * (y3 - o) * (z4 - o) + (y2 - o) * (z3 - o) * (x4 - o) +
                         (z2 - o) * (x3 - o) * (y4 - o) - (z2 - o) * (y3 - o) * (x4 - o) -
                         (x2 - o) * (z3 - o) * (y4 - o) - (y2 - o) * (x3 - o) * (z4 - o));
  vol += det / 6.;
  // sum over i <= j of u_i u_j for the four vertices (u_1 = 0), continued
  auto chain = [](double s, double u2, double u3, double u4) {
    const double u1 = 0.;
    s = s + u1 * u1; s = s + u1 * u2; s = s + u2 * u2; s = s + u1 * u3; s = s + u2 * u3;
    s = s + u3 * u3; s = s + u1 * u4; s = s + u2 * u4; s = s + u3 * u4; s = s + u4 * u4;
    return s;
  };
  I[0] += det * chain(chain(0., y2, y3, y4), z2, z3, z4) / 60.;
  I[1] += det * chain(chain(0., x2, x3, x4), z2, z3, z4) / 60.;
  I[2] += det * chain(chain(0., x2, x3, x4), y2, y3, y4) / 60.;
}

// Polyhedron volume and inertia: triangles form tetrahedra with the origin,
// larger faces are fanned around their vertex centroid (Polyhedron::
// BuildInertia / computeVolumeInertia, Geometry/src/Polyhedron.cpp).
void polyMassProperties(PolyFile const& P, double& vol, double* Iv) {
  vol = 0.;
  Iv[0] = Iv[1] = Iv[2] = 0.;
  for (auto const& f : P.faces) {
    int nf = (int)f.size();
    if (nf == 3) {
      tetMass(P.verts[f[0]], P.verts[f[1]], P.verts[f[2]], vol, Iv);
    } else {
      std::array<double, 3> G = {0., 0., 0.};
      for (int j = 0; j < nf; ++j)
        for (int d = 0; d < 3; ++d) G[d] += P.verts[f[j]][d];
      for (int d = 0; d < 3; ++d) G[d] = G[d] / double(nf);
      for (int j = 0, k = nf - 1; j < nf; k = j++) tetMass(G, P.verts[f[k]], P.verts[f[j]], vol, Iv);
    }
  }
}

InstanceDesc readInstance(std::string const& path) {
  auto doc = parseXmlFile(path);
  XmlNode const* root = doc.get();
  XmlNode const* cons = root->find("Construction");
  if (!cons) throw std::runtime_error("no <Construction> in " + path);
  InstanceDesc I{};
  std::memset(&I.grid, 0, sizeof(I.grid));
  XmlNode const* lc = cons->child("LinkedCell");
  if (!lc) throw std::runtime_error("no <LinkedCell>");
  double maxc[3] = {lc->attrD("MX"), lc->attrD("MY"), lc->attrD("MZ")};
  double org[3] = {0., 0., 0.};
  if (XmlNode const* o = cons->child("Origin")) {
    org[0] = o->attrD("OX"); org[1] = o->attrD("OY"); org[2] = o->attrD("OZ");
  }
  int per[3] = {0, 0, 0};
  if (XmlNode const* p = cons->child("Periodicity")) {
    per[0] = p->attrI("PX") == 1; per[1] = p->attrI("PY") == 1; per[2] = p->attrI("PZ") == 1;
  }
  double lcf = lc->has("CellSizeFactor") ? lc->attrD("CellSizeFactor") : 1.;
  if (lcf < 1.) lcf = 1.;

  std::map<std::string, int> mats;
  std::vector<std::string> morder;
  // particle classes (Particle::Particle(DOMNode*), Component/src/Particle.cpp:120-160)
  double maxR = 0.;
  for (XmlNode const* pn : [&] {
         std::vector<XmlNode const*> v;
         if (XmlNode const* ps = cons->child("Particles")) v = ps->childrenNamed("Particle");
         return v;
       }()) {
    TypeDesc t{};
    std::vector<std::vector<int>> class_faces_of_this;
    double density = pn->attrD("Density");
    XmlNode const* cv = pn->child("Convex");
    if (!cv) throw std::runtime_error("<Particle> without <Convex>");
    t.crust = cv->attrD("CrustThickness");
    if (!(t.crust > 0.)) throw std::runtime_error("crust thickness must be > 0");
    double vol = 0., Iv[3] = {0., 0., 0.};
    if (XmlNode const* sp = cv->child("Sphere")) {
      double r = sp->attrD("Radius");
      t.shape = 0;
      t.radius = r;
      vol = 4.0 * PI * std::pow(r, 3.) / 3.0;                         // Sphere::getVolume
      double I0 = 8.0 * PI * std::pow(r, 5.) / 15.0;                  // Sphere::BuildInertia
      Iv[0] = Iv[1] = Iv[2] = I0;
      t.extent[0] = t.extent[1] = t.extent[2] = r;
    } else if (XmlNode const* bx = cv->child("Box")) {
      // Box::getVolume, Box::BuildInertia, Box::computeCircumscribedRadius
      // (Geometry/src/Box.cpp); the XML gives full lengths
      t.shape = 1;
      double e[3] = {0.5 * bx->attrD("LX"), 0.5 * bx->attrD("LY"), 0.5 * bx->attrD("LZ")};
      for (int d = 0; d < 3; ++d) t.extent[d] = e[d];
      t.radius = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
      vol = 8.0 * e[0] * e[1] * e[2];
      Iv[0] = 8.0 * e[0] * e[1] * e[2] * (e[1] * e[1] + e[2] * e[2]) / 3.0;
      Iv[1] = 8.0 * e[0] * e[1] * e[2] * (e[0] * e[0] + e[2] * e[2]) / 3.0;
      Iv[2] = 8.0 * e[0] * e[1] * e[2] * (e[0] * e[0] + e[1] * e[1]) / 3.0;
    } else if (XmlNode const* cy = cv->child("Cylinder")) {
      // Cylinder::getVolume, BuildInertia, computeCircumscribedRadius
      // (Geometry/src/Cylinder.cpp:32-106); axis along the local Y
      t.shape = 3;
      double r = cy->attrD("Radius"), hh = cy->attrD("Height") / 2.;
      t.extent[0] = r; t.extent[1] = hh; t.extent[2] = r;
      t.radius = std::sqrt(r * r + hh * hh);
      vol = 2 * hh * PI * r * r;
      double constant = 0.5 * hh * r * r * PI;
      Iv[0] = Iv[2] = constant * (4.0 * hh * hh / 3.0 + r * r);
      Iv[1] = 2.0 * constant * r * r;
    } else if (XmlNode const* ph = cv->child("Polyhedron")) {
      t.shape = 2;
      PolyFile P = readPolyFile(ph->attr("Name"));
      class_faces_of_this = P.faces;
      polyMassProperties(P, vol, Iv);
      double ray = 0.;
      for (auto const& v : P.verts) ray = std::max(ray, v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      t.radius = std::sqrt(ray);                 // Polyhedron::computeCircumscribedRadius
      // identity-frame bounding box (Convex::bbox, Convex.cpp:29-41)
      for (int d = 0; d < 3; ++d) {
        double lo = P.verts[0][d], hi = P.verts[0][d];
        for (auto const& v : P.verts) { lo = std::min(lo, v[d]); hi = std::max(hi, v[d]); }
        t.extent[d] = (hi - lo) / 2.;
      }
      t.poly_begin = (int)I.poly_verts.size() / 3;
      t.poly_count = (int)P.verts.size();
      for (auto const& v : P.verts)
        for (int d = 0; d < 3; ++d) I.poly_verts.push_back(v[d]);
      // the vertex graph as Polyhedron::BuildPolyhedron builds it
      // (Geometry/src/Polyhedron.cpp:322-365): along each face, vertex k gets
      // its successor j; a new particle's search starts at the first vertex
      // with a neighbour
      std::vector<std::vector<int>> cob(P.verts.size());
      for (auto const& f : P.faces) {
        const int nf = (int)f.size();
        for (int j = 0, k = nf - 1; j < nf; k = j++) cob[f[k]].push_back(f[j]);
      }
      t.poly_start = 0;
      while (t.poly_start < (int)cob.size() && cob[t.poly_start].empty()) ++t.poly_start;
      if (t.poly_start == (int)cob.size()) throw std::runtime_error("polyhedron without faces");
      for (auto& c : cob) I.poly_cob.push_back(std::move(c));
    } else {
      throw std::runtime_error("unsupported particle shape in <Convex>");
    }
    t.mass = density * vol;
    for (int d = 0; d < 3; ++d) t.inertia[d] = Iv[d] * density;
    t.density = density;
    t.coupling = 1.;
    t.inv_mass = 1. / t.mass;
    for (int d = 0; d < 3; ++d) {
      t.inv_inertia[d] = 1. / t.inertia[d];
      t.inv_inertia_c[d] = t.inv_inertia[d];
    }
    t.eqrad = std::pow((0.75 / PI) * vol, 1. / 3.);                   // getEquivalentSphereRadius
    // crust shrink factors (RigidBodyWithCrust ctor, RigidBodyWithCrust.cpp:58-78)
    for (int d = 0; d < 3; ++d)
      t.scaling[d] = t.extent[d] < 1.e-10 ? 1. : (t.extent[d] - t.crust) / t.extent[d];
    XmlNode const* mat = pn->child("Material");
    if (!mat) throw std::runtime_error("<Particle> without <Material>");
    t.mat = materialIndex(mats, morder, mat->valueS());
    t.r_f = (float)t.radius;
    maxR = std::max(maxR, t.radius);
    I.types.push_back(t);
    I.class_faces.push_back(class_faces_of_this);
  }
  if (I.types.empty()) throw std::runtime_error("no <Particle> class");
  // obstacles: boxes with identity orientation
  if (XmlNode const* obs = cons->child("Obstacles")) {
    std::vector<XmlNode const*> list;
    collectObstacles(obs, list);
    for (XmlNode const* on : list) {
      WallDesc w{};
      XmlNode const* cv = on->child("Convex");
      if (!cv) throw std::runtime_error("<Obstacle> without <Convex>");
      w.crust = cv->attrD("CrustThickness");
      XmlNode const* bx = cv->child("Box");
      if (!bx) throw std::runtime_error("only <Box> obstacles are supported");
      w.extent[0] = 0.5 * bx->attrD("LX");
      w.extent[1] = 0.5 * bx->attrD("LY");
      w.extent[2] = 0.5 * bx->attrD("LZ");
      XmlNode const* ce = on->child("Centre");
      if (!ce) throw std::runtime_error("<Obstacle> without <Centre>");
      w.centre[0] = ce->attrD("X"); w.centre[1] = ce->attrD("Y"); w.centre[2] = ce->attrD("Z");
      if (XmlNode const* ap = on->child("AngularPosition"))
        if (ap->has("Type") && ap->attr("Type") != "Identity")
          throw std::runtime_error("only Identity obstacle orientation is supported");
      XmlNode const* mat = on->child("Material");
      if (!mat) throw std::runtime_error("<Obstacle> without <Material>");
      w.mat = materialIndex(mats, morder, mat->valueS());
      double vol = 8. * w.extent[0] * w.extent[1] * w.extent[2];
      w.eqrad = std::pow((0.75 / PI) * vol, 1. / 3.);
      w.radius = std::sqrt(w.extent[0] * w.extent[0] + w.extent[1] * w.extent[1] +
                           w.extent[2] * w.extent[2]);
      for (int d = 0; d < 3; ++d)
        w.scaling[d] = w.extent[d] < 1.e-10 ? 1. : (w.extent[d] - w.crust) / w.extent[d];
      w.id = (int)I.walls.size();
      I.walls.push_back(w);
    }
  }
  I.nmat = (int)morder.size();
  // contact force models keyed by the material pair
  std::map<int, ModelDesc> bymask;
  if (XmlNode const* cfm = cons->child("ContactForceModels")) {
    for (auto const& c : cfm->children) {
      int mask = 0;
      if (c->name != "Default") {
        XmlNode const* m = c->child("Material");
        if (!m) throw std::runtime_error("<ContactForceModel> without <Material>");
        int a = materialIndex(mats, morder, m->attr("materialA"));
        int b = materialIndex(mats, morder, m->attr("materialB"));
        mask = (1 << a) | (1 << b);
      }
      bool found = false;
      for (auto const& law : c->children) {
        if (law->name == "HookeMemory" || law->name == "Hooke") {
          bymask[mask] = readModel(law.get(), law->name);
          found = true;
        } else if (law->name == "Hertz" || law->name == "HertzMemory") {
          throw std::runtime_error("Hertz contact models are not supported");
        }
      }
      if (!found) throw std::runtime_error("<ContactForceModel> without a known law");
    }
  }
  I.nmat = (int)morder.size();
  I.mat_names = morder;
  for (int a = 0; a < kMaxMat; ++a)
    for (int b = 0; b < kMaxMat; ++b) {
      ModelDesc m{};
      if (a < I.nmat && b < I.nmat) {
        auto it = bymask.find((1 << a) | (1 << b));
        if (it != bymask.end()) m = it->second;
      }
      I.models[a * kMaxMat + b] = m;
    }
  for (auto const& t : I.types) {
    for (auto const& t2 : I.types)
      if (!I.models[t.mat * kMaxMat + t2.mat].valid)
        throw std::runtime_error("no contact force model for a particle material pair");
    for (auto const& w : I.walls)
      if (!I.models[t.mat * kMaxMat + w.mat].valid)
        throw std::runtime_error("no contact force model for a particle/obstacle material pair");
  }
  // gravity and time step
  I.gravity[0] = I.gravity[1] = I.gravity[2] = 0.;
  if (XmlNode const* fo = root->find("Forces"))
    if (XmlNode const* g = fo->child("Gravity")) {
      I.gravity[0] = g->attrD("GX"); I.gravity[1] = g->attrD("GY"); I.gravity[2] = g->attrD("GZ");
    }
  XmlNode const* ts = root->find("TimeStep");
  if (!ts) throw std::runtime_error("no <TimeStep>");
  if (ts->has("dt")) I.dt = ts->attrD("dt");
  else if (ts->has("mindt")) I.dt = ts->attrD("mindt");   // the coupled run's start
  else throw std::runtime_error("<TimeStep> needs dt (or mindt, maxdt, ndt)");
  I.min_dt = ts->has("mindt") ? ts->attrD("mindt") : I.dt;
  I.max_dt = ts->has("maxdt") ? ts->attrD("maxdt") : I.dt;
  I.ndt = ts->has("ndt") ? ts->attrI("ndt") : 1;
  I.reload_file.clear();
  I.reload_reset = false;
  if (XmlNode const* rl = root->find("Reload")) {
    if (rl->has("Filename")) I.reload_file = rl->attr("Filename");
    // Grains::Construction (Base/src/Grains.cpp:842-843) then
    // AllComponents::resetKinematics (Component/src/AllComponents.cpp:762-771)
    I.reload_reset = rl->has("Velocity") && rl->attr("Velocity") == "Reset";
  }
  // a RawData post-processing writer (PostProcessingWriterBuilderFactory,
  // PostProcessing/src/PostProcessingWriterBuilderFactory.cpp:19-20;
  // RawDataPostProcessingWriter ctor: Name, WritingMode="Binary")
  I.rawdata_root.clear();
  I.rawdata_binary = false;
  if (XmlNode const* rd = root->find("RawData"))
    if (rd->has("Name")) {
      I.rawdata_root = rd->attr("Name");
      I.rawdata_binary = rd->has("WritingMode") && rd->attr("WritingMode") == "Binary";
    }
  for (auto& t : I.types)
    for (int d = 0; d < 3; ++d) t.weight[d] = I.gravity[d] * (t.mass * (1. - 0. / 1.));
  // linked cell grid (LinkedCell::set, Base/src/LinkedCell.cpp:47-160)
  double cellsize = 2. * (lcf * maxR);
  GridDesc& g = I.grid;
  for (int d = 0; d < 3; ++d) {
    double size = maxc[d] - org[d];
    int n = (int)((size + 1.0e-10) / cellsize);
    if (!n) n = 1;
    g.nb[d] = n;
    g.edge[d] = size / n;
    g.lc_origin[d] = org[d];
    g.L[d] = size;
    g.periodic[d] = per[d];
    if (per[d]) {
      if (n < 3) throw std::runtime_error("a periodic direction needs at least 3 cells");
      g.lc_origin[d] += -g.edge[d];
      g.nb[d] += 2;
    }
    g.edge_f[d] = (float)g.edge[d];
  }
  // Pair-list grid.  The skin defaults to a quarter of the largest
  // circumscribed radius (the LinkedCell attribute Skin, a length, overrides
  // it; 0 rebuilds the list every step).
  for (int d = 0; d < 3; ++d) {
    I.box_org[d] = org[d];
    I.box_max[d] = maxc[d];
    I.box_per[d] = per[d];
  }
  I.cellsize = cellsize;
  I.max_radius = maxR;
  I.xml_skin = lc->has("Skin") ? lc->attrD("Skin") : -1.;
  GridDesc& b = I.bgrid;
  b = g;
  makePairGrid(I, I.xml_skin >= 0. ? I.xml_skin : 0.25 * maxR);
  // FP32 contact filter: positions rounded to float carry at most half an ulp
  // of the largest coordinate each (2^-24 relative); 5e-7 of it bounds the
  // error of a difference plus an image shift with room to spare
  double maxabs = 0.;
  for (int d = 0; d < 3; ++d) {
    maxabs = std::max(maxabs, std::fabs(org[d]) + (maxc[d] - org[d]));
    b.Lf[d] = (float)(maxc[d] - org[d]);
    g.Lf[d] = b.Lf[d];
  }
  // (the filter's positions are continuous since the last rebuild, so they
  // may leave the box by less than a period: the margin allows a period more)
  double maxL = 0.;
  for (int d = 0; d < 3; ++d) maxL = std::max(maxL, maxc[d] - org[d]);
  b.filt_margin = (float)(5.e-7 * (maxabs + maxL));
  g.filt_margin = b.filt_margin;
  // band in which a particle stays in the reference grid's inner cells
  // (periodic: cells 1 .. nb-2; otherwise 0 .. nb-1), with a relative margin
  // of 1e-6 of a cell that dwarfs the rounding of the cell computation
  for (int d = 0; d < 3; ++d) {
    const double lo_cell = per[d] ? 1. : 0., hi_cell = per[d] ? g.nb[d] - 1. : (double)g.nb[d];
    g.safe_lo[d] = g.lc_origin[d] + (lo_cell + 1.e-6) * g.edge[d];
    g.safe_hi[d] = g.lc_origin[d] + (hi_cell - 1.e-6) * g.edge[d];
    b.safe_lo[d] = g.safe_lo[d];
    b.safe_hi[d] = g.safe_hi[d];
  }
  return I;
}

// ---------------------------------------------------------------- system --
struct System {
  int precision = GDEM_FP64;
  std::vector<InstanceDesc> inst;
  std::vector<std::string> xml_paths;
  std::vector<GridDesc> h_bgrids;  // host copy of the pair-list grids
  std::vector<TypeDesc> h_types;   // host copy of the particle classes (all instances)
  std::vector<int> h_type, h_inst; // uploaded classes (instance-local) and instances, by ID
  std::vector<int> ref_ids;        // reload particle IDs by particle index (empty: index + 1)
  double tune_skin = -1.;          // skin as a multiple of rmax (< 0: the XML's or 0.25)
  int tune_bps = 0;                // force-kernel blocks per multiprocessor (0: 4)
  std::vector<int> type_base;     // first global type of each instance
  std::vector<int> id_base;       // first particle ID of each instance
  std::vector<int> inst_n;
  int reserve_extra = 0;           // room for particles inserted after the upload
  int* d_hit = nullptr;            // insertion overlap flag
  DevState S{};
  GridDesc* d_grids = nullptr; TypeDesc* d_types = nullptr; ModelDesc* d_models = nullptr;
  WallDesc* d_walls = nullptr;
  double* d_poly = nullptr;        // polyhedron vertex table of all instances
  int* d_poly_adj_off = nullptr;   // polyhedron vertex graphs
  int* d_poly_adj = nullptr;
  GridDesc* d_bgrids = nullptr;    // pair-list grids
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool have_state = false, started = false, diag = false, use_graphs = true;
  // contact memory of ended contacts dropped each evaluation (the plain
  // step) or carried (the coupled step); the tables are four times larger
  // when it is carried, since the entries of every pair that ever touched
  // stay
  bool prune_memory = true;
  // the last force evaluation: 0 none since the state was set, 1 recorded by
  // the diagnostics, 2 run without them
  int evaluated = 0;
  bool id_order = false;           // state arrays are in particle-ID order (not yet binned)
  double last_ms = 0.;
  int status_host = 0;
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  long parity = 0;                 // force evaluations so far (state and history swap together)
  long epoch = 0;                  // host copy of the evaluation counter (history tags)
  long epoch_t0 = 0;               // evaluation counter at the leapfrog's t0 (contact features)
  bool graph_conditional = false;  // the graphs rebuild through a conditional node
  std::vector<void*> allocs;
  double* d_stage = nullptr;       // AoS staging, ID order (x v w wbf q F T: 22 doubles/particle)
  int* d_type_id = nullptr;        // particle class by ID
  int* d_inst_id = nullptr;        // instance by ID
  double* d_vstats = nullptr;      // velocity statistics: partials + result
  // per-kernel CUDA-event timing
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evpool;
  size_t evused = 0;
  std::vector<std::pair<int, size_t>> pending;
  std::vector<std::string> knames;
  std::vector<double> ktotal;
  std::vector<long> kcount;

  ~System() { release(); }
  void release() {
    for (auto& row : graph)
      for (auto& gx : row) if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
    for (void* p : allocs) cudaFree(p);
    allocs.clear();
    if (d_grids) cudaFree(d_grids);
    if (d_types) cudaFree(d_types);
    if (d_models) cudaFree(d_models);
    if (d_walls) cudaFree(d_walls);
    if (d_poly) cudaFree(d_poly);
    if (d_poly_adj_off) cudaFree(d_poly_adj_off);
    if (d_poly_adj) cudaFree(d_poly_adj);
    d_poly_adj_off = d_poly_adj = nullptr;
    if (d_bgrids) cudaFree(d_bgrids);
    d_bgrids = nullptr;
    d_grids = nullptr; d_types = nullptr; d_models = nullptr; d_walls = nullptr; d_poly = nullptr;
    for (auto& e : evpool) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    evpool.clear();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    ev0 = ev1 = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
  }
  template <typename T>
  T* alloc(size_t n) {
    T* p = dalloc<T>(n);
    allocs.push_back(p);
    return p;
  }
  void invalidateGraphs() {
    for (auto& row : graph)
      for (auto& gx : row) if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
  }
  void freeAlloc(void* p) {
    for (auto& a : allocs)
      if (a == p) { CK(cudaFree(a)); a = allocs.back(); allocs.pop_back(); return; }
  }

  // Pair-list skin (a multiple of each instance's largest circumscribed
  // radius; < 0 restores the XML's) and the force kernels' blocks per
  // multiprocessor (<= 0: the default).  Neither changes a result: the
  // contact set is exact for any skin and the sums run in partner-ID order.
  void applyTuning(double skin_factor, int bps) {
    if (started) throw std::runtime_error("tuning is set before gdem_init");
    tune_skin = skin_factor;
    tune_bps = bps > 0 ? bps : 0;
    int offset = 0;
    for (size_t k = 0; k < inst.size(); ++k) {
      InstanceDesc& I = inst[k];
      makePairGrid(I, skin_factor >= 0. ? skin_factor * I.max_radius
                                        : (I.xml_skin >= 0. ? I.xml_skin : 0.25 * I.max_radius));
      GridDesc b = I.bgrid;
      b.cell_offset = offset;
      b.wall_begin = h_bgrids[k].wall_begin;
      b.wall_count = h_bgrids[k].wall_count;
      b.model_base = h_bgrids[k].model_base;
      offset += b.nb[0] * b.nb[1] * b.nb[2];
      h_bgrids[k] = b;
    }
    CK(cudaMemcpy(d_bgrids, h_bgrids.data(), h_bgrids.size() * sizeof(GridDesc), cudaMemcpyHostToDevice));
    S.forces_bps = tune_bps;
    if (S.cell_count && offset != S.ncells) {
      freeAlloc(S.cell_count); freeAlloc(S.cell_start); freeAlloc(S.scan_tmp);
      S.ncells = offset;
      S.cell_count = alloc<int>(S.ncells); S.cell_start = alloc<int>(S.ncells + 1);
      S.scan_tmp = alloc<int>((S.ncells + 1023) / 1024 + 1);
      CK(cudaMemset(S.cell_count, 0, (size_t)S.ncells * sizeof(int)));
    }
    S.ncells = offset;
    invalidateGraphs();
  }

  // Runs f between two events when profiling (plain launches only).
  template <typename Fn>
  void timed(const char* name, Fn&& f) {
    if (!profiling) { f(); return; }
    if (evused == evpool.size()) {
      cudaEvent_t a, b;
      CK(cudaEventCreate(&a));
      CK(cudaEventCreate(&b));
      evpool.push_back({a, b});
    }
    size_t e = evused++;
    int k = 0;
    while (k < (int)knames.size() && knames[k] != name) ++k;
    if (k == (int)knames.size()) { knames.push_back(name); ktotal.push_back(0.); kcount.push_back(0); }
    CK(cudaEventRecord(evpool[e].first, stream));
    f();
    CK(cudaEventRecord(evpool[e].second, stream));
    pending.push_back({k, e});
  }
  void collectTimes() {
    if (pending.empty()) return;
    CK(cudaStreamSynchronize(stream));
    for (auto& p : pending) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, evpool[p.second].first, evpool[p.second].second));
      ktotal[p.first] += ms;
      kcount[p.first] += 1;
    }
    pending.clear();
    evused = 0;
  }

  // The instances' contact-force-model tables to the device (read by the
  // kernels when they run: captured graphs stay valid).
  void uploadModels() {
    std::vector<ModelDesc> models;
    for (auto const& I : inst)
      for (int k = 0; k < kMaxMat * kMaxMat; ++k) models.push_back(I.models[k]);
    CK(cudaMemcpy(d_models, models.data(), models.size() * sizeof(ModelDesc),
                  cudaMemcpyHostToDevice));
  }

  void setupTables() {
    std::vector<GridDesc> grids;
    std::vector<TypeDesc> types;
    std::vector<ModelDesc> models;
    std::vector<WallDesc> walls;
    std::vector<double> poly;
    std::vector<int> adj_off, adj;   // polyhedron vertex graphs (CSR over all vertices)
    int cell_offset = 0, max_walls = 1;
    S.any_convex = 0;
    std::vector<GridDesc> bgrids;
    int ref_cells = 0;
    for (auto& I : inst) {
      GridDesc g = I.grid;
      g.cell_offset = ref_cells;
      ref_cells += g.nb[0] * g.nb[1] * g.nb[2];
      g.wall_begin = (int)walls.size();
      g.wall_count = (int)I.walls.size();
      g.model_base = (int)models.size();
      GridDesc b = I.bgrid;
      b.cell_offset = cell_offset;
      cell_offset += b.nb[0] * b.nb[1] * b.nb[2];
      b.wall_begin = g.wall_begin;
      b.wall_count = g.wall_count;
      b.model_base = g.model_base;
      bgrids.push_back(b);
      type_base.push_back((int)types.size());
      const int vbase = (int)poly.size() / 3;
      for (auto const& t : I.types) {
        types.push_back(t);
        if (t.shape == 2) types.back().poly_begin += vbase;
        if (t.shape != 0) S.any_convex = 1;
      }
      poly.insert(poly.end(), I.poly_verts.begin(), I.poly_verts.end());
      for (auto const& c : I.poly_cob) {
        adj_off.push_back((int)adj.size());
        adj.insert(adj.end(), c.begin(), c.end());
      }
      for (auto const& w : I.walls) walls.push_back(w);
      for (int k = 0; k < kMaxMat * kMaxMat; ++k) models.push_back(I.models[k]);
      max_walls = std::max(max_walls, (int)I.walls.size());
      grids.push_back(g);
    }
    S.ncells = cell_offset;
    S.ninst = (int)inst.size();
    S.max_walls = max_walls;
    S.any_walls = 0;
    S.filt_margin_max = 0.f;
    for (auto const& b : bgrids) {
      if (b.wall_count) S.any_walls = 1;
      S.filt_margin_max = std::max(S.filt_margin_max, b.filt_margin);
    }
    S.dt = inst[0].dt;
    for (auto& I : inst)
      if (I.dt != S.dt) throw std::runtime_error("all instances of a batch must share dt");
    auto up = [&](auto*& dst, auto const& vec) {
      using T = typename std::remove_reference<decltype(vec)>::type::value_type;
      CK(cudaMalloc(reinterpret_cast<void**>(&dst), std::max<size_t>(1, vec.size()) * sizeof(T)));
      if (!vec.empty()) CK(cudaMemcpy(dst, vec.data(), vec.size() * sizeof(T), cudaMemcpyHostToDevice));
    };
    adj_off.push_back((int)adj.size());
    S.any_poly = 0;
    for (auto const& t : types) if (t.shape == 2) S.any_poly = 1;
    up(d_grids, grids); up(d_types, types); up(d_models, models); up(d_walls, walls);
    up(d_poly, poly); up(d_bgrids, bgrids); up(d_poly_adj_off, adj_off); up(d_poly_adj, adj);
    S.poly_adj_off = d_poly_adj_off;
    S.poly_adj = d_poly_adj;
    h_bgrids = bgrids;
    h_types = types;
    S.grids = d_grids; S.types = d_types; S.models = d_models; S.walls = d_walls;
    S.bgrids = d_bgrids;
    S.poly_verts = d_poly;
  }

  void allocateParticles(int n) {
    S.n = n;
    S.cap = std::max(n + reserve_extra, 1);
    size_t c = (size_t)S.cap;
    S.id = alloc<int>(c); S.type = alloc<int>(c); S.inst = alloc<int>(c);
    S.id2 = alloc<int>(c); S.type2 = alloc<int>(c); S.inst2 = alloc<int>(c);
    S.x = alloc<double>(3 * c); S.v = alloc<double>(3 * c); S.w = alloc<double>(3 * c);
    S.wbf = alloc<double>(3 * c); S.q = alloc<double>(4 * c);
    S.x2 = alloc<double>(3 * c); S.v2 = alloc<double>(3 * c); S.w2 = alloc<double>(3 * c);
    S.wbf2 = alloc<double>(3 * c); S.q2 = alloc<double>(4 * c);
    S.F = alloc<double>(3 * c); S.T = alloc<double>(3 * c);
    S.F2 = alloc<double>(3 * c); S.T2 = alloc<double>(3 * c);
    S.posf0 = alloc<float4>(c); S.wrap = alloc<int>(c); S.wrap2 = alloc<int>(c);
    S.ctl = alloc<int>(kCtlWords);
    CK(cudaMemset(S.ctl, 0, kCtlWords * sizeof(int)));
    epoch = 0;
    // orientation matrices, SoA (9 x cap), only when some class is not a sphere
    S.basis = S.any_convex ? alloc<double>(9 * c) : nullptr;
    S.basis2 = S.any_convex ? alloc<double>(9 * c) : nullptr;
    if (S.any_poly) {
      S.curv = alloc<int>(c); S.curv2 = alloc<int>(c); S.curv_next = alloc<int>(c);
      CK(cudaMemset(S.curv, 0, c * sizeof(int)));
      CK(cudaMemset(S.curv_next, 0, c * sizeof(int)));
    } else {
      S.curv = S.curv2 = S.curv_next = nullptr;
    }
    S.skey = alloc<int>(c); S.rank = alloc<int>(c); S.order = alloc<int>(c);
    S.cell_count = alloc<int>(S.ncells); S.cell_start = alloc<int>(S.ncells + 1);
    S.scan_tmp = alloc<int>((S.ncells + 1023) / 1024 + 1);
    S.cellc = alloc<int4>(c);
    S.wbf_state = (precision == GDEM_FP64 || S.any_convex) ? 1 : 0;
    if (precision == GDEM_FP64) {
      S.pos64 = alloc<double4>(c);
      S.offh = nullptr;
    } else {
      S.offh = alloc<float4>(c);
      S.pos64 = nullptr;
    }
    S.npairs = alloc<int>(c);
    S.pair_off = alloc<int>(c + 1);
    S.pair_scan_tmp = alloc<int>((c + 1023) / 1024 + 1);
    CK(cudaMemset(S.npairs, 0, c * sizeof(int)));
    CK(cudaMemset(S.pair_off, 0, (c + 1) * sizeof(int)));
    S.pairs = nullptr; S.upairs = nullptr; S.epos = nullptr; S.kept = nullptr; S.kept2 = nullptr;
    S.share = nullptr;
    S.pair_cap = 0;
    S.pair_delta = nullptr; S.wall_delta = nullptr; S.diag = 0;
    S.pair_force = nullptr; S.wall_force = nullptr;
    allocatePairs((long long)16 * (long long)c + 4096);
    S.wshare = alloc<char>(c * (precision == GDEM_FP64 ? 48 : 32));
    S.nact = alloc<int>(2 * c);
    CK(cudaMemset(S.nact, 0, 2 * c * sizeof(int)));
    S.work = alloc<int>(c);
    S.cstats = alloc<ContactStats>(1);
    CK(cudaMemset(S.cstats, 0, sizeof(ContactStats)));
    {
      int dev = 0;
      CK(cudaGetDevice(&dev));
      CK(cudaDeviceGetAttribute(&S.nsm, cudaDevAttrMultiProcessorCount, dev));
    }
    S.posf = alloc<float4>(c);
    int l2 = nextPow2Log((size_t)8 * c + 64) + (prune_memory ? 0 : 2);
    size_t hc = size_t(1) << l2;
    size_t vsz = precision == GDEM_FP64 ? sizeof(double) : sizeof(float);
    for (HistTable* t : {&S.hist_old, &S.hist_new}) {
      t->log2cap = l2;
      t->keys = alloc<unsigned long long>(hc);
      t->vals = alloc<char>(hc * 9 * vsz);
      // all-ones keys: tag 1023, which the first 512 uses of a table never carry
      CK(cudaMemset(t->keys, 0xFF, hc * sizeof(unsigned long long)));
    }
    S.status = alloc<int>(1);
    CK(cudaMemset(S.status, 0, sizeof(int)));
    S.law_counts = alloc<unsigned long long>(2);
    CK(cudaMemset(S.law_counts, 0, 2 * sizeof(unsigned long long)));
    S.gjk_counts = alloc<unsigned long long>(3);
    CK(cudaMemset(S.gjk_counts, 0, 3 * sizeof(unsigned long long)));
    CK(cudaMemset(S.cell_count, 0, (size_t)S.ncells * sizeof(int)));
    CK(cudaMemset(S.F, 0, 3 * c * sizeof(double)));
    CK(cudaMemset(S.T, 0, 3 * c * sizeof(double)));
    d_stage = alloc<double>(22 * c);
    d_type_id = alloc<int>(c);
    d_inst_id = alloc<int>(c);
    d_vstats = alloc<double>(2 * ((c + 255) / 256) + 2);
    // the memsets above ran on the legacy default stream
    CK(cudaDeviceSynchronize());
  }

  // The arrays sized by the pair list's entries: the rows, the compact pair
  // list with the pairs' positions in their rows, the contact filter's kept
  // list, the shares (tag words all ones: no evaluation's tag) and, when on,
  // the diagnostics records.  The rows are rebuilt before the next
  // evaluation (the contents are not carried over).
  void allocatePairs(long long entries) {
    if (entries > (long long)INT_MAX - 64)
      throw std::runtime_error("pair list too large for 32-bit row offsets");
    for (void* p : {(void*)S.pairs, (void*)S.upairs, (void*)S.epos, (void*)S.kept, (void*)S.kept2, S.share,
                    (void*)S.pair_delta, (void*)S.pair_force})
      if (p) freeAlloc(p);
    const size_t e = (size_t)entries, pc = e / 2 + 1;
    S.pair_cap = (int)entries;
    S.pairs = alloc<int>(e);
    S.upairs = alloc<int2>(pc);
    S.epos = alloc<int>(pc);
    S.kept = alloc<int>(pc);
    // the cold pairs' first pass (FP32-split, non-spherical classes)
    S.kept2 = (precision == GDEM_FP32_SPLIT && S.any_convex) ? alloc<int>(pc) : nullptr;
    const size_t sb = precision == GDEM_FP64 ? 64 : 32;
    S.share = alloc<char>(e * sb);
    // (on the library's stream, which does not synchronise with the legacy
    // default stream)
    CK(cudaMemsetAsync(S.share, 0xFF, e * sb, stream));
    if (S.wall_delta) {
      S.pair_delta = alloc<double>(e);
      S.pair_force = alloc<double>(3 * e);
    } else {
      S.pair_delta = nullptr;
      S.pair_force = nullptr;
    }
    static const int one = 1;
    if (S.ctl) CK(cudaMemcpyAsync(S.ctl + kCtlNeed, &one, sizeof(int), cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    invalidateGraphs();
  }
  // Grows the pair list when the most entries a rebuild needed since the
  // last check exceed 80 % of the allocation (to 1.5 times that need);
  // the next evaluation rebuilds.  Synchronises the stream.  Returns whether
  // it grew.
  bool checkPairCapacity() {
    int hwm = 0;
    CK(cudaStreamSynchronize(stream));
    CK(cudaMemcpy(&hwm, S.ctl + kCtlEntriesMax, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemsetAsync(S.ctl + kCtlEntriesMax, 0, sizeof(int), stream));
    CK(cudaStreamSynchronize(stream));
    if ((double)hwm <= 0.8 * (double)S.pair_cap) return false;
    allocatePairs(std::max((long long)(1.5 * (double)hwm) + 4096, (long long)S.pair_cap));
    return true;
  }
  // Sizes the pair list for the current state before the leapfrog start: the
  // rebuild up to the scan of the row lengths (it only reorders the state),
  // then the allocation check.
  void sizePairList() {
    static const int one = 1;
    CK(cudaMemcpyAsync(S.ctl + kCtlActive, &one, sizeof(int), cudaMemcpyHostToDevice, stream));
    const int* gate = S.ctl + kCtlActive;
    launch_bin(S, gate, stream);
    launch_scan(S, gate, stream);
    launch_place(S, gate, stream);
    launch_cellsort(S, gate, stream);
    launch_permute(S, gate, stream);
    launch_copyback(S, gate, stream);
    if (precision == GDEM_FP64) launch_pairs64(S, gate, 0, stream);
    else launch_pairs32(S, gate, 0, stream);
    launch_row_scan(S, gate, stream);
    CK(cudaGetLastError());
    id_order = false;
    checkPairCapacity();
  }

  // Host AoS arrays (by ID) -> staging -> SoA state in ID order.
  void loadState(const double* x, const double* v, const double* w, const double* wbf,
                 const double* q, const double* F, const double* T) {
    size_t n = (size_t)S.n;
    double* st = d_stage;
    double *dx = st, *dv = st + 3 * n, *dw = st + 6 * n, *dwb = st + 9 * n, *dq = st + 12 * n,
           *dF = st + 16 * n, *dT = st + 19 * n;
    auto cp = [&](double* d, const double* h, size_t k) {
      if (h) CK(cudaMemcpyAsync(d, h, k * n * sizeof(double), cudaMemcpyHostToDevice, stream));
    };
    cp(dx, x, 3); cp(dv, v, 3); cp(dw, w, 3); cp(dwb, wbf, 3); cp(dq, q, 4); cp(dF, F, 3); cp(dT, T, 3);
    launch_load_state(S, dx, dv, dw, wbf ? dwb : nullptr, dq, F ? dF : nullptr, T ? dT : nullptr,
                      d_type_id, d_inst_id, stream);
    CK(cudaGetLastError());
    // the pair list no longer describes this state: rebuild before the next
    // force evaluation
    const int one = 1;
    CK(cudaMemcpyAsync(S.ctl + kCtlNeed, &one, sizeof(int), cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    id_order = true;
  }

  // The contact-history tables alternate with every force evaluation.
  void swapHist() { std::swap(S.hist_old, S.hist_new); }

  // The table that evaluation e (1-based) writes is refilled every 512 of its
  // uses with the tag e - 1, which none of its next 512 uses carries.
  void maybeClearHistory(long e) {
    if ((e % 512) >= 2) return;
    size_t hc = size_t(1) << S.hist_new.log2cap;
    unsigned long long v = tagged((1ull << kTagShift) - 1, (unsigned)(e - 1));
    timed("hist_fill", [&] { launch_fill64(S.hist_new.keys, hc, v, stream); });
  }

  // Pair-list rebuild: cells, counting sort, permutation into cell order,
  // pair search.  gate: the control word that tells gated kernels whether
  // this step rebuilds (plain launches), or null inside the graph's
  // conditional node.
  void rebuild(const int* gate) {
    id_order = false;
    timed("bin", [&] { launch_bin(S, gate, stream); });
    timed("scan", [&] { launch_scan(S, gate, stream); });
    timed("place", [&] { launch_place(S, gate, stream); });
    timed("cellsort", [&] { launch_cellsort(S, gate, stream); });
    timed("permute", [&] { launch_permute(S, gate, stream); });
    timed("copyback", [&] { launch_copyback(S, gate, stream); });
    if (precision == GDEM_FP64) {
      timed("pairs_count64", [&] { launch_pairs64(S, gate, 0, stream); });
      timed("row_scan", [&] { launch_row_scan(S, gate, stream); });
      timed("pairs_fill64", [&] { launch_pairs64(S, gate, 1, stream); });
    } else {
      timed("pairs_count32", [&] { launch_pairs32(S, gate, 0, stream); });
      timed("row_scan", [&] { launch_row_scan(S, gate, stream); });
      timed("pairs_fill32", [&] { launch_pairs32(S, gate, 1, stream); });
    }
    timed("link", [&] { launch_link(S, gate, stream); });
  }
  // Contact filter, pair kernel (contacts and walls), then the leapfrog
  // kernel: the sums of the shares and the leapfrog parts in flags (at the
  // leapfrog start only the sums, stored as F, T).
  void forcesAndMove(int flags) {
    if (diag) timed("diag_prefill", [&] { launch_diag_prefill(S, stream); });
    timed("filter", [&] { launch_filter(S, stream); });
    if (precision == GDEM_FP64) timed("pairlaw64", [&] { launch_pairlaw64(S, stream); });
    else {
      if (S.any_convex) timed("pairsep32", [&] { launch_pairsep32(S, stream); });
      timed("pairlaw32", [&] { launch_pairlaw32(S, stream); });
    }
    timed("move", [&] { launch_move(S, flags | kStepSum, precision == GDEM_FP32_SPLIT, stream); });
    if (!prune_memory)
      timed("hist_carry", [&] { launch_hist_carry(S, precision == GDEM_FP64, stream); });
  }
  // One force evaluation with plain launches: decide, gated rebuild, filter,
  // forces, move.
  void evaluate(int flags) {
    maybeClearHistory(epoch + 1);
    timed("decide", [&] { launch_decide(S, cudaGraphConditionalHandle(), 0, stream); });
    rebuild(S.ctl + kCtlActive);
    forcesAndMove(flags);
    ++epoch;
    swapHist();
  }

  // The same evaluation as one graph: decide -> conditional node holding the
  // rebuild -> step kernel.  If the conditional node cannot be built, the
  // graph holds the gated rebuild instead.
  cudaGraphExec_t captureEvaluation(int flags) {
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    bool conditional = true;
    cudaGraphConditionalHandle h{};
    if (cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) {
      cudaGetLastError();
      conditional = false;
    }
    CK(cudaStreamBeginCaptureToGraph(stream, g, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    launch_decide(S, h, conditional ? 1 : 0, stream);
    CK(cudaStreamEndCapture(stream, &g));
    cudaGraphNode_t decide_node = nullptr;
    size_t nn = 1;
    CK(cudaGraphGetNodes(g, &decide_node, &nn));
    cudaGraphNode_t tail = decide_node;
    if (conditional) {
      cudaGraphNodeParams cp{};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeIf;
      cp.conditional.size = 1;
      cudaGraphNode_t cond = nullptr;
      if (cudaGraphAddNode(&cond, g, &decide_node, 1, &cp) == cudaSuccess) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal));
        rebuild(nullptr);
        CK(cudaStreamEndCapture(stream, &body));
        tail = cond;
      } else {
        cudaGetLastError();
        conditional = false;
      }
    }
    CK(cudaStreamBeginCaptureToGraph(stream, g, &tail, nullptr, 1,
                                     cudaStreamCaptureModeThreadLocal));
    if (!conditional) rebuild(S.ctl + kCtlActive);
    forcesAndMove(flags);
    CK(cudaStreamEndCapture(stream, &g));
    cudaGraphExec_t ex = nullptr;
    CK(cudaGraphInstantiate(&ex, g, 0));
    CK(cudaGraphDestroy(g));
    graph_conditional = conditional;
    return ex;
  }
  // Graph of evaluation kind k (0: inside a call, 1: last of a call) for the
  // current history-table parity; built on first use.
  void launchEvaluation(int k, int flags) {
    maybeClearHistory(epoch + 1);
    const int par = (int)(parity & 1);
    if (!graph[k][par]) graph[k][par] = captureEvaluation(flags);
    CK(cudaGraphLaunch(graph[k][par], stream));
    ++epoch;
    ++parity;
    swapHist();
  }

  void init() {
    sizePairList();
    epoch_t0 = epoch + 1;   // the evaluation at t0 is the next one
    evaluate(kStepStoreFT);
    ++parity;
    launch_hist_zero_cumulative(S.hist_old, S.ctl, precision == GDEM_FP64, stream);
    CK(cudaStreamSynchronize(stream));
    // size the contact filter's grid for the pair list just built: one block
    // per 2,048 pairs (kFilterPairsPerBlock) and a quarter more for growth
    // (the kernel loops over any excess)
    int np = 0;
    CK(cudaMemcpy(&np, S.ctl + kCtlPairs, sizeof(int), cudaMemcpyDeviceToHost));
    S.filter_qblocks = std::max(1, (int)((1.25 * np + 2047.) / 2048.));
    invalidateGraphs();
    collectTimes();
    started = true;
    evaluated = diag ? 1 : 2;
  }
  // nsteps leapfrog steps: the opening kick and drift of the first (with the
  // stored forces), then per step a force evaluation followed by the closing
  // kick and -- except after the last -- the next opening kick and drift.
  void step(int nsteps) {
    if (nsteps <= 0) return;
    id_order = false;
    CK(cudaEventRecord(ev0, stream));
    timed("move", [&] { launch_move(S, kStepMove, precision == GDEM_FP32_SPLIT, stream); });
    const int mid = kStepClose | kStepMove;
    const int last = kStepClose | kStepStoreFT;
    for (int k = 0; k < nsteps; ++k) {
      const bool is_last = k == nsteps - 1;
      // the pair list's allocation is checked every kCapacityCheck steps
      // within a call (and at its end); it grows before it can run short
      if (k > 0 && k % kCapacityCheck == 0) checkPairCapacity();
      const bool graphs = use_graphs && !diag && !profiling;
      if (graphs) {
        launchEvaluation(is_last ? 1 : 0, is_last ? last : mid);
      } else {
        evaluate(is_last ? last : mid);
        ++parity;
      }
    }
    CK(cudaEventRecord(ev1, stream));
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    last_ms = ms;
    collectTimes();
    evaluated = diag ? 1 : 2;
    checkPairCapacity();
  }
  int readStatus() {
    int st = 0;
    CK(cudaMemcpy(&st, S.status, sizeof(int), cudaMemcpyDeviceToHost));
    status_host |= st;
    return status_host;
  }
};

System* sys(gdem_handle h) { return reinterpret_cast<System*>(h); }

template <typename F>
int guarded(F&& f) {
  try {
    return f();
  } catch (CudaError const& e) {
    g_last_error = e.what();
    return GDEM_ERR_CUDA;
  } catch (std::exception const& e) {
    g_last_error = e.what();
    return GDEM_ERR_INVALID;
  }
}

}  // namespace

void setLastError(std::string const& msg) { g_last_error = msg; }

void readAdjointSetup(std::string const& path, AdjointSetup& out) {
  InstanceDesc I = readInstance(path);
  out.types = I.types;
  out.walls = I.walls;
  for (int k = 0; k < kMaxMat * kMaxMat; ++k) out.models[k] = I.models[k];
  out.dt = I.dt;
  for (int d = 0; d < 3; ++d) {
    out.periodic[d] = I.grid.periodic[d];
    out.origin[d] = I.box_org[d];
    out.maxc[d] = I.box_max[d];
  }
}

}  // namespace gdem

using namespace gdem;

extern "C" {

const char* gdem_last_error(void) { return g_last_error.c_str(); }

int gdem_create_batch(int n, const char* const* xml_paths, int precision, gdem_handle* out) {
  return guarded([&] {
    if (!out || n <= 0 || !xml_paths) throw std::runtime_error("invalid arguments");
    if (precision != GDEM_FP64 && precision != GDEM_FP32_SPLIT)
      throw std::runtime_error("unknown precision mode");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw CudaError("no CUDA device: the Grains3D B200 step has no CPU fallback");
    auto s = std::make_unique<System>();
    s->precision = precision;
    for (int k = 0; k < n; ++k) {
      s->inst.push_back(readInstance(xml_paths[k]));
      s->xml_paths.push_back(xml_paths[k]);
    }
    s->setupTables();
    CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&s->ev0));
    CK(cudaEventCreate(&s->ev1));
    *out = reinterpret_cast<gdem_handle>(s.release());
    return GDEM_OK;
  });
}

int gdem_create(const char* xml_path, int precision, gdem_handle* out) {
  const char* paths[1] = {xml_path};
  return gdem_create_batch(1, paths, precision, out);
}

int gdem_upload_state(gdem_handle h, int64_t n, const int* inst, const int* type,
                      const double* x, const double* v, const double* w, const double* wbf,
                      const double* q) {
  return guarded([&] {
    System* s = sys(h);
    // (an empty system only when particles are to be inserted into it)
    if (!s || n < 0 || (n == 0 && s->reserve_extra == 0) || !type || !x || !v || !w || !q)
      throw std::runtime_error("invalid arguments");
    if (n + s->reserve_extra > (int64_t(1) << kMaxIdBits) - 64)
      throw std::runtime_error("too many particles for the 27-bit particle IDs of the contact keys");
    if (s->have_state) throw std::runtime_error("state already uploaded");
    int N = (int)n;
    std::vector<int> hinst(N, 0), htype(N), hid(N);
    s->inst_n.assign(s->inst.size(), 0);
    for (int i = 0; i < N; ++i) {
      int k = inst ? inst[i] : 0;
      if (k < 0 || k >= (int)s->inst.size()) throw std::runtime_error("instance index out of range");
      if (type[i] < 0 || type[i] >= (int)s->inst[k].types.size())
        throw std::runtime_error("particle type out of range");
      if (i > 0 && k < hinst[i - 1]) throw std::runtime_error("particles must be grouped by instance");
      hinst[i] = k;
      htype[i] = s->type_base[k] + type[i];
      hid[i] = i;
      s->inst_n[k]++;
    }
    s->h_inst = hinst;
    s->h_type.assign(type, type + N);
    s->id_base.assign(s->inst.size(), 0);
    for (size_t k = 1; k < s->inst.size(); ++k) s->id_base[k] = s->id_base[k - 1] + s->inst_n[k - 1];
    s->allocateParticles(N);
    DevState& S = s->S;
    (void)hid;
    CK(cudaMemcpy(s->d_type_id, htype.data(), N * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->d_inst_id, hinst.data(), N * sizeof(int), cudaMemcpyHostToDevice));
    (void)S;
    s->loadState(x, v, w, wbf, q, nullptr, nullptr);
    s->have_state = true;
    s->evaluated = 0;
    return GDEM_OK;
  });
}

int gdem_reserve(gdem_handle h, int64_t extra) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || extra < 0 || extra > (int64_t(1) << kMaxIdBits)) throw std::runtime_error("invalid arguments");
    if (s->have_state) throw std::runtime_error("reserve before the state is uploaded");
    s->reserve_extra = (int)extra;
    return GDEM_OK;
  });
}

int gdem_insert_particle(gdem_handle h, int type, const double* x, const double* v,
                         const double* w, const double* q, const double* basis, int force,
                         int bv_only, int ref_id, int* inserted, int* id) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !x || !v || !w || !q || !inserted) throw std::runtime_error("invalid arguments");
    if (!s->have_state) throw std::runtime_error("upload the state first");
    if (s->inst.size() != 1) throw std::runtime_error("insertion is for single systems");
    if (type < 0 || type >= (int)s->inst[0].types.size())
      throw std::runtime_error("particle type out of range");
    DevState& S = s->S;
    if (S.n >= S.cap) throw std::runtime_error("no room for another particle (gdem_reserve)");
    NewParticle p{};
    p.type = s->type_base[0] + type;
    p.id = S.n;
    p.slot = S.n;
    p.has_basis = basis ? 1 : 0;
    for (int d = 0; d < 3; ++d) { p.x[d] = x[d]; p.v[d] = v[d]; p.w[d] = w[d]; }
    for (int k = 0; k < 4; ++k) p.q[k] = q[k];
    if (basis) {
      for (int k = 0; k < 9; ++k) p.basis[k] = basis[k];
    } else {
      // Matrix::setRotation (Geometry/src/Matrix.cpp:114-127), for the test
      const double qx = q[0], qy = q[1], qz = q[2], qw = q[3];
      const double sc = 2.0 / (qx * qx + qy * qy + qz * qz + qw * qw);
      const double xs = qx * sc, ys = qy * sc, zs = qz * sc;
      const double wx = qw * xs, wy = qw * ys, wz = qw * zs;
      const double xx = qx * xs, xy = qx * ys, xz = qx * zs, yy = qy * ys, yz = qy * zs,
                   zz = qz * zs;
      const double m[9] = {1.0 - (yy + zz), xy - wz, xz + wy, xy + wz, 1.0 - (xx + zz),
                           yz - wx, xz - wy, yz + wx, 1.0 - (xx + yy)};
      for (int k = 0; k < 9; ++k) p.basis[k] = m[k];
    }
    *inserted = 0;
    if (!force) {
      if (!s->d_hit) s->d_hit = s->alloc<int>(1);
      CK(cudaMemsetAsync(s->d_hit, 0, sizeof(int), s->stream));
      launch_insert_test(S, p, bv_only, s->d_hit, s->stream);
      CK(cudaGetLastError());
      int hit = 0;
      CK(cudaMemcpyAsync(&hit, s->d_hit, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
      CK(cudaStreamSynchronize(s->stream));
      if (hit) return GDEM_OK;
    }
    launch_append_particle(S, p, s->stream);
    CK(cudaGetLastError());
    S.n += 1;
    s->h_type.push_back(type);
    s->h_inst.push_back(0);
    s->inst_n[0] += 1;
    if (!s->ref_ids.empty()) s->ref_ids.push_back(ref_id > 0 ? ref_id : S.n);
    // the pair list does not hold the new particle: rebuild before the next
    // force evaluation; the graphs hold the old particle count
    static const int one = 1;
    CK(cudaMemcpyAsync(S.ctl + kCtlNeed, &one, sizeof(int), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    // the contact filter's grid, for about 4 pairs per particle (its kernel
    // loops over any excess)
    S.filter_qblocks = std::max(S.filter_qblocks, (4 * S.n + 2047) / 2048);
    s->invalidateGraphs();
    *inserted = 1;
    if (id) *id = p.id;
    return GDEM_OK;
  });
}

int gdem_upload_forces(gdem_handle h, const double* F, const double* T) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || !F || !T) throw std::runtime_error("upload the state first");
    if (s->started) throw std::runtime_error("forces can only be set before the first step");
    // the state is still in ID order: copy F and T through the staging area
    DevState& S = s->S;
    size_t n = (size_t)S.n, c = (size_t)S.cap;
    std::vector<double> hF(3 * c), hT(3 * c);
    for (int d = 0; d < 3; ++d)
      for (size_t i = 0; i < n; ++i) { hF[d * c + i] = F[3 * i + d]; hT[d * c + i] = T[3 * i + d]; }
    CK(cudaMemcpy(S.F, hF.data(), 3 * c * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(S.T, hT.data(), 3 * c * sizeof(double), cudaMemcpyHostToDevice));
    s->started = true;
    s->epoch_t0 = s->epoch;   // the forces are those of t0; the next evaluation is t0 + dt
    return GDEM_OK;
  });
}

int gdem_set_state(gdem_handle h, const double* x, const double* v, const double* w,
                   const double* wbf, const double* q, const double* F, const double* T) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || !x || !v || !w || !q)
      throw std::runtime_error("gdem_set_state needs an uploaded system and x, v, w, q");
    if ((F == nullptr) != (T == nullptr)) throw std::runtime_error("give both F and T, or neither");
    s->loadState(x, v, w, wbf, q, F, T);
    s->started = F != nullptr;
    if (F) s->epoch_t0 = s->epoch;
    return GDEM_OK;
  });
}

int gdem_velocity_stats(gdem_handle h, double* vmax, double* vmean) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state) throw std::runtime_error("no state");
    DevState& S = s->S;
    int nb = (S.n + 255) / 256;
    double* out = s->d_vstats + 2 * nb;
    launch_vstats(S, s->d_vstats, out, s->stream);
    double r[2];
    CK(cudaMemcpyAsync(r, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (vmax) *vmax = r[0];
    if (vmean) *vmean = r[1];
    return GDEM_OK;
  });
}

int gdem_pair_counts(gdem_handle h, int64_t* entries, int64_t* contacts) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->started) throw std::runtime_error("no force evaluation yet");
    unsigned long long* d = reinterpret_cast<unsigned long long*>(s->d_vstats);
    launch_pair_counts(s->S, d, s->stream);
    unsigned long long r[2];
    CK(cudaMemcpyAsync(r, d, sizeof(r), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (entries) *entries = (int64_t)r[0];
    if (contacts) *contacts = (int64_t)r[1];
    return GDEM_OK;
  });
}

int gdem_step_counts(gdem_handle h, int64_t* evaluations, int64_t* rebuilds) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state) throw std::runtime_error("no state");
    int r[kCtlWords];
    CK(cudaStreamSynchronize(s->stream));
    CK(cudaMemcpy(r, s->S.ctl, sizeof(r), cudaMemcpyDeviceToHost));
    if (evaluations) *evaluations = r[kCtlEpoch];
    if (rebuilds) *rebuilds = r[kCtlRebuilds];
    return GDEM_OK;
  });
}

int gdem_law_counts(gdem_handle h, int64_t* evaluated, int64_t* reevaluated, int reset) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state) throw std::runtime_error("no state");
    unsigned long long r[2];
    CK(cudaStreamSynchronize(s->stream));
    CK(cudaMemcpy(r, s->S.law_counts, sizeof(r), cudaMemcpyDeviceToHost));
    if (reset) CK(cudaMemset(s->S.law_counts, 0, sizeof(r)));
    if (evaluated) *evaluated = (int64_t)r[0];
    if (reevaluated) *reevaluated = (int64_t)r[1];
    return GDEM_OK;
  });
}

int gdem_gjk_counts(gdem_handle h, int64_t* calls, int64_t* iterations, int64_t* max_iterations,
                    int reset) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state) throw std::runtime_error("no state");
    unsigned long long r[3];
    CK(cudaStreamSynchronize(s->stream));
    CK(cudaMemcpy(r, s->S.gjk_counts, sizeof(r), cudaMemcpyDeviceToHost));
    if (reset) CK(cudaMemset(s->S.gjk_counts, 0, sizeof(r)));
    if (calls) *calls = (int64_t)r[0];
    if (iterations) *iterations = (int64_t)r[1];
    if (max_iterations) *max_iterations = (int64_t)r[2];
    return GDEM_OK;
  });
}

int gdem_contact_features(gdem_handle h, double* overlap_max, double* overlap_mean,
                          int64_t* evaluation_of_max, double* gjk_iterations_mean, int reset) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state) throw std::runtime_error("upload the state first");
    ContactStats cs{};
    CK(cudaStreamSynchronize(s->stream));
    CK(cudaMemcpy(&cs, s->S.cstats, sizeof(ContactStats), cudaMemcpyDeviceToHost));
    unsigned long long g[3] = {0, 0, 0};
    CK(cudaMemcpy(g, s->S.gjk_counts, sizeof(g), cudaMemcpyDeviceToHost));
    double mx = 0.;
    std::memcpy(&mx, &cs.max_bits, sizeof(double));
    if (overlap_max) *overlap_max = cs.count ? mx : 0.;
    if (overlap_mean) *overlap_mean = cs.count ? cs.sum / (double)cs.count : 0.;
    if (evaluation_of_max) *evaluation_of_max = cs.count ? (int64_t)(cs.max_epoch - s->epoch_t0) : -1;
    if (gjk_iterations_mean) *gjk_iterations_mean = g[0] ? (double)g[1] / (double)g[0] : 0.;
    if (reset) {
      CK(cudaMemsetAsync(s->S.cstats, 0, sizeof(ContactStats), s->stream));
      CK(cudaStreamSynchronize(s->stream));
    }
    return GDEM_OK;
  });
}

int gdem_set_profiling(gdem_handle h, int on) {
  return guarded([&] {
    System* s = sys(h);
    if (!s) throw std::runtime_error("invalid handle");
    s->profiling = on != 0;
    s->knames.clear(); s->ktotal.clear(); s->kcount.clear();
    return GDEM_OK;
  });
}

int gdem_kernel_times(gdem_handle h, int capacity, int* count, char* names, double* total_ms,
                      int64_t* launches) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !count) throw std::runtime_error("invalid arguments");
    *count = (int)s->knames.size();
    for (int k = 0; k < *count && k < capacity; ++k) {
      if (names) {
        std::memset(names + 32 * k, 0, 32);
        std::strncpy(names + 32 * k, s->knames[k].c_str(), 31);
      }
      if (total_ms) total_ms[k] = s->ktotal[k];
      if (launches) launches[k] = s->kcount[k];
    }
    return GDEM_OK;
  });
}

int gdem_upload_history(gdem_handle h, int64_t n, const int* owner, const int* partner,
                        const double* kdelta, const double* prevn, const double* spring) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || n < 0) throw std::runtime_error("upload the state first");
    DevState& S = s->S;
    HistTable& t = S.hist_old;   // read by the next force evaluation
    size_t hc = size_t(1) << t.log2cap;
    // the next evaluation (epoch + 1) looks up tag epoch; the free slots get
    // tag epoch - 1, which this table's next uses (tags epoch + 2, + 4, ...)
    // never carry
    const unsigned tag = (unsigned)s->epoch;
    const unsigned long long empty = tagged((1ull << kTagShift) - 1, tag - 1u);
    std::vector<unsigned long long> keys(hc, empty);
    bool fp64 = s->precision == GDEM_FP64;
    std::vector<double> vd(fp64 ? 9 * hc : 0);
    std::vector<float> vf(fp64 ? 0 : 9 * hc);
    for (int64_t e = 0; e < n; ++e) {
      int a = owner[e], b = partner[e];
      unsigned long long key;
      if (b >= 0) {
        if (!(a < b)) continue;   // the lower ID's view is stored
        key = pairKey(a, b);
      } else {
        key = wallKey(a, -b - 2);
      }
      uint32_t slot = hashSlot(key, t.log2cap);
      while (keys[slot] != empty) slot = (slot + 1) & (uint32_t)(hc - 1);
      keys[slot] = tagged(key, tag);
      double vals[9] = {kdelta[3 * e], kdelta[3 * e + 1], kdelta[3 * e + 2],
                        prevn[3 * e], prevn[3 * e + 1], prevn[3 * e + 2],
                        spring ? spring[3 * e] : 0., spring ? spring[3 * e + 1] : 0.,
                        spring ? spring[3 * e + 2] : 0.};
      for (int k = 0; k < 9; ++k) {
        if (fp64) vd[9 * slot + k] = vals[k];
        else vf[9 * slot + k] = (float)vals[k];
      }
    }
    CK(cudaMemcpy(t.keys, keys.data(), hc * sizeof(unsigned long long), cudaMemcpyHostToDevice));
    if (fp64) CK(cudaMemcpy(t.vals, vd.data(), vd.size() * sizeof(double), cudaMemcpyHostToDevice));
    else CK(cudaMemcpy(t.vals, vf.data(), vf.size() * sizeof(float), cudaMemcpyHostToDevice));
    return GDEM_OK;
  });
}

int gdem_download_history(gdem_handle h, int64_t capacity, int64_t* count, int* owner,
                          int* partner, double* kdelta, double* prevn, double* spring) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || !count) throw std::runtime_error("invalid arguments");
    DevState& S = s->S;
    CK(cudaStreamSynchronize(s->stream));
    HistTable& t = S.hist_old;   // written by the last force evaluation
    const size_t hc = size_t(1) << t.log2cap;
    std::vector<unsigned long long> keys(hc);
    CK(cudaMemcpy(keys.data(), t.keys, hc * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    const bool fp64 = s->precision == GDEM_FP64;
    std::vector<double> vd(fp64 ? 9 * hc : 0);
    std::vector<float> vf(fp64 ? 0 : 9 * hc);
    if (fp64) CK(cudaMemcpy(vd.data(), t.vals, vd.size() * sizeof(double), cudaMemcpyDeviceToHost));
    else CK(cudaMemcpy(vf.data(), t.vals, vf.size() * sizeof(float), cudaMemcpyDeviceToHost));
    struct Rec { int a, b; double v[9]; };
    std::vector<Rec> recs;
    const unsigned tag = (unsigned)s->epoch & kTagMask;
    const unsigned idmask = (1u << kMaxIdBits) - 1u;
    const unsigned n = (unsigned)S.n;
    for (size_t k = 0; k < hc; ++k) {
      if (tagOf(keys[k]) != tag) continue;
      const unsigned hi = (unsigned)((keys[k] >> kMaxIdBits) & idmask);
      const unsigned lo = (unsigned)(keys[k] & idmask);
      if (hi >= n) continue;
      Rec r;
      for (int c = 0; c < 9; ++c) r.v[c] = fp64 ? vd[9 * k + c] : (double)vf[9 * k + c];
      r.a = (int)hi;
      if (lo < n) {
        r.b = (int)lo;
        recs.push_back(r);
        Rec q{(int)lo, (int)hi, {}};   // the other body's view is the negation
        for (int c = 0; c < 9; ++c) q.v[c] = -r.v[c];
        recs.push_back(q);
      } else {
        r.b = -((int)(idmask - lo) + 2);
        recs.push_back(r);
      }
    }
    std::sort(recs.begin(), recs.end(),
              [](Rec const& x, Rec const& y) { return x.a != y.a ? x.a < y.a : x.b < y.b; });
    *count = (int64_t)recs.size();
    if (capacity >= *count && owner && partner) {
      for (size_t e = 0; e < recs.size(); ++e) {
        owner[e] = recs[e].a;
        partner[e] = recs[e].b;
        for (int d = 0; d < 3; ++d) {
          if (kdelta) kdelta[3 * e + d] = recs[e].v[d];
          if (prevn) prevn[3 * e + d] = recs[e].v[3 + d];
          if (spring) spring[3 * e + d] = recs[e].v[6 + d];
        }
      }
    }
    return GDEM_OK;
  });
}

int gdem_init(gdem_handle h) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state) throw std::runtime_error("upload the state first");
    s->invalidateGraphs();
    s->init();
    s->readStatus();
    return GDEM_OK;
  });
}

int gdem_set_tuning(gdem_handle h, double skin_factor, int blocks_per_sm) {
  return guarded([&] {
    System* s = sys(h);
    if (!s) throw std::runtime_error("invalid handle");
    if (!(skin_factor < 0.) && !(skin_factor <= 4.)) throw std::runtime_error("skin factor out of range");
    if (blocks_per_sm > 64) throw std::runtime_error("blocks per multiprocessor out of range");
    s->applyTuning(skin_factor, blocks_per_sm);
    return GDEM_OK;
  });
}

// Autotuner: times trial_steps steps (after 3 warm-up steps) of a copy of
// the uploaded system for each candidate skin (as a multiple of rmax: it sets
// the pair-list cell size and how often the list is rebuilt), then for each
// candidate number of force-kernel blocks per multiprocessor at the best
// skin, and keeps the fastest pair.  The copies start from the same state, so
// the choice reflects this workload; the results of the system do not depend
// on it.
int gdem_autotune(gdem_handle h, int trial_steps, double* skin_factor, int* blocks_per_sm,
                  double* ms_per_step) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state) throw std::runtime_error("upload the state first");
    if (s->started) throw std::runtime_error("gdem_autotune runs before gdem_init");
    if (trial_steps < 1) throw std::runtime_error("trial_steps must be >= 1");
    const int n = s->S.n;
    std::vector<double> x(3 * (size_t)n), v(3 * (size_t)n), w(3 * (size_t)n),
        wb(3 * (size_t)n), q(4 * (size_t)n), basis;
    auto rc = [](int code) {
      if (code != GDEM_OK) throw std::runtime_error("autotune trial: " + g_last_error);
    };
    rc(gdem_download_state(h, x.data(), v.data(), w.data(), wb.data(), q.data(), nullptr, nullptr));
    if (s->S.basis) {
      basis.resize(9 * (size_t)n);
      rc(gdem_download_basis(h, basis.data()));
    }
    std::vector<const char*> paths;
    for (auto const& p : s->xml_paths) paths.push_back(p.c_str());
    auto trial = [&](double sf, int bps) {
      gdem_handle c = nullptr;
      rc(gdem_create_batch((int)paths.size(), paths.data(), s->precision, &c));
      std::unique_ptr<System> guard(sys(c));
      rc(gdem_set_tuning(c, sf, bps));
      rc(gdem_upload_state(c, n, s->h_inst.data(), s->h_type.data(), x.data(), v.data(),
                           w.data(), wb.data(), q.data()));
      if (!basis.empty()) rc(gdem_upload_basis(c, basis.data()));
      rc(gdem_init(c));
      rc(gdem_step(c, 3));
      rc(gdem_step(c, trial_steps));
      if (guard->status_host) return 1.e300;   // a failing candidate is never chosen
      return guard->last_ms / trial_steps;
    };
    const double skins[] = {0.1, 0.175, 0.25, 0.4, 0.6};
    const int bpss[] = {2, 4, 8};
    double best = 1.e300, best_sf = 0.25;
    int best_bps = 4;
    for (double sf : skins) {
      const double ms = trial(sf, 4);
      if (ms < best) { best = ms; best_sf = sf; }
    }
    for (int bps : bpss) {
      if (bps == 4) continue;
      const double ms = trial(best_sf, bps);
      if (ms < best) { best = ms; best_bps = bps; }
    }
    s->applyTuning(best_sf, best_bps);
    if (skin_factor) *skin_factor = best_sf;
    if (blocks_per_sm) *blocks_per_sm = best_bps;
    if (ms_per_step) *ms_per_step = best;
    return GDEM_OK;
  });
}

// ----------------------------------------------------- fluid coupling --
int gdem_set_fluid(gdem_handle h, double fluid_density, int corrected_acceleration) {
  return guarded([&] {
    System* s = sys(h);
    if (!s) throw std::runtime_error("invalid handle");
    if (!(fluid_density >= 0.)) throw std::runtime_error("fluid density must be >= 0");
    size_t k = 0;
    for (auto const& I : s->inst)
      for (size_t c = 0; c < I.types.size(); ++c, ++k) {
        TypeDesc& t = s->h_types[k];
        if (!(fluid_density < t.density)) throw std::runtime_error("fluid denser than a particle class");
        // Particle::computeWeight (Particle.cpp:413-418) and
        // ParticleKinematics::setCouplingFactor (ParticleKinematics.cpp:483-488)
        for (int d = 0; d < 3; ++d)
          t.weight[d] = I.gravity[d] * (t.mass * (1. - fluid_density / t.density));
        t.coupling = 1.;
        if (corrected_acceleration) t.coupling -= fluid_density / t.density;
        t.inv_mass = 1. / (t.mass * t.coupling);
        for (int d = 0; d < 3; ++d) t.inv_inertia_c[d] = 1. / (t.coupling * t.inertia[d]);
      }
    // the kernels read the class table when they run: no graph to recapture
    CK(cudaMemcpy(s->d_types, s->h_types.data(), s->h_types.size() * sizeof(TypeDesc),
                  cudaMemcpyHostToDevice));
    return GDEM_OK;
  });
}

int gdem_set_time_step(gdem_handle h, double dt) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !(dt > 0.)) throw std::runtime_error("invalid time step");
    if (dt != s->S.dt) {
      s->S.dt = dt;
      for (auto& I : s->inst) I.dt = dt;
      s->invalidateGraphs();   // the kernels take dt by value
    }
    return GDEM_OK;
  });
}

int gdem_time_step_bounds(gdem_handle h, double* min_dt, double* max_dt, int* ndt) {
  return guarded([&] {
    System* s = sys(h);
    if (!s) throw std::runtime_error("invalid handle");
    InstanceDesc const& I = s->inst[0];
    if (min_dt) *min_dt = I.min_dt;
    if (max_dt) *max_dt = I.max_dt;
    if (ndt) *ndt = I.ndt;
    return GDEM_OK;
  });
}

int gdem_reload_filename(gdem_handle h, char* buf, int capacity) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !buf || capacity <= 0) throw std::runtime_error("invalid arguments");
    std::string const& f = s->inst[0].reload_file;
    if ((int)f.size() >= capacity) throw std::runtime_error("buffer too small");
    std::memcpy(buf, f.c_str(), f.size() + 1);
    return GDEM_OK;
  });
}

int gdem_rawdata_spec(gdem_handle h, char* root, int capacity, int* binary) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !root || capacity <= 0) throw std::runtime_error("invalid arguments");
    std::string const& r = s->inst[0].rawdata_root;
    if ((int)r.size() >= capacity) throw std::runtime_error("buffer too small");
    std::memcpy(root, r.c_str(), r.size() + 1);
    if (binary) *binary = s->inst[0].rawdata_binary ? 1 : 0;
    return GDEM_OK;
  });
}

int gdem_particle_class(gdem_handle h, int cls, double* props, int* shape) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || cls < 0 || cls >= (int)s->inst[0].types.size()) throw std::runtime_error("no such class");
    TypeDesc const& t = s->h_types[cls];
    if (props) {
      props[0] = t.mass; props[1] = t.density;
      props[2] = t.inertia[0]; props[3] = t.inertia[1]; props[4] = t.inertia[2];
      props[5] = t.radius; props[6] = t.crust;
    }
    if (shape) *shape = t.shape;
    return GDEM_OK;
  });
}

int gdem_set_velocities(gdem_handle h, const double* v, const double* w) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || !v || !w) throw std::runtime_error("invalid arguments");
    DevState& S = s->S;
    const size_t n = (size_t)S.n;
    double* dv = s->d_stage;
    double* dw = s->d_stage + 3 * n;
    CK(cudaMemcpyAsync(dv, v, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(dw, w, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    launch_set_velocities(S, dv, dw, s->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    return GDEM_OK;
  });
}

int gdem_set_hydro_forces(gdem_handle h, const double* F, const double* T) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state) throw std::runtime_error("upload the state first");
    DevState& S = s->S;
    const size_t n = (size_t)S.n;
    if (!F && !T) {
      if (S.hydro) { CK(cudaMemset(S.hydro, 0, 6 * n * sizeof(double))); }
      return GDEM_OK;
    }
    if (!F || !T) throw std::runtime_error("give both F and T, or neither");
    if (!S.hydro) {
      S.hydro = s->alloc<double>(6 * (size_t)S.cap);
      s->invalidateGraphs();   // the move kernel now adds them
    }
    std::vector<double> hv(6 * n);
    for (size_t i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) { hv[6 * i + d] = F[3 * i + d]; hv[6 * i + 3 + d] = T[3 * i + d]; }
    CK(cudaMemcpy(S.hydro, hv.data(), hv.size() * sizeof(double), cudaMemcpyHostToDevice));
    return GDEM_OK;
  });
}

int gdem_step(gdem_handle h, int nsteps) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state) throw std::runtime_error("upload the state first");
    if (!s->started) throw std::runtime_error("call gdem_init (or gdem_upload_forces) before stepping");
    s->step(nsteps);
    s->readStatus();
    return GDEM_OK;
  });
}

int gdem_download_state(gdem_handle h, double* x, double* v, double* w, double* wbf, double* q,
                        double* F, double* T) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state) throw std::runtime_error("no state");
    DevState& S = s->S;
    size_t n = (size_t)S.n;
    double* st = s->d_stage;
    double* dx = st; double* dv = st + 3 * n; double* dw = st + 6 * n; double* dwb = st + 9 * n;
    double* dq = st + 12 * n; double* dF = st + 16 * n; double* dT = st + 19 * n;
    launch_scatter_by_id(S, x ? dx : nullptr, v ? dv : nullptr, w ? dw : nullptr,
                         wbf ? dwb : nullptr, q ? dq : nullptr, F ? dF : nullptr,
                         T ? dT : nullptr, 0, s->stream);
    CK(cudaGetLastError());
    struct { double* h; double* d; size_t k; } items[] = {
        {x, dx, 3}, {v, dv, 3}, {w, dw, 3}, {wbf, dwb, 3}, {q, dq, 4}, {F, dF, 3}, {T, dT, 3}};
    for (auto& it : items)
      if (it.h) CK(cudaMemcpyAsync(it.h, it.d, it.k * n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return GDEM_OK;
  });
}

int gdem_upload_basis(gdem_handle h, const double* basis) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || !basis) throw std::runtime_error("upload the state first");
    if (!s->id_order)
      throw std::runtime_error("orientations can only be set right after gdem_upload_state or gdem_set_state");
    DevState& S = s->S;
    if (!S.basis) return GDEM_OK;   // spheres only: orientation matrices are not used
    size_t n = (size_t)S.n, c = (size_t)S.cap;
    std::vector<double> hb(9 * c, 0.);
    for (size_t i = 0; i < n; ++i)
      for (int k = 0; k < 9; ++k) hb[k * c + i] = basis[9 * i + k];
    CK(cudaMemcpy(S.basis, hb.data(), hb.size() * sizeof(double), cudaMemcpyHostToDevice));
    return GDEM_OK;
  });
}

int gdem_download_basis(gdem_handle h, double* basis) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || !basis) throw std::runtime_error("no state");
    DevState& S = s->S;
    size_t n = (size_t)S.n;
    if (!S.basis) {
      // spheres carry no orientation matrix: report the identity
      for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 9; ++k) basis[9 * i + k] = (k % 4 == 0) ? 1. : 0.;
      return GDEM_OK;
    }
    double* d = s->d_stage;   // 22 doubles per particle: room for 9
    launch_basis_by_id(S, d, 0, s->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(basis, d, 9 * n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return GDEM_OK;
  });
}

// ------------------------------------------------------ Format2024 reload --
// The particle file of a Format2024 reload (the "<reload>_Particles" text
// file that AllComponents::write and AllComponents::read_particles exchange,
// Component/src/AllComponents.cpp:1299-1420, 1136-1290), one line per
// particle (Particle::write2014, Particle.cpp:1167-1176):
//   class ID tag active | origin(3) basis(9, by rows) transform-type |
//   v(3) q(w, x, y, z) w(3) | F(3) T(3) (SecondOrderLeapFrog.cpp:102-109) |
//   n, then n x (1 partner-ID 1 active kdelta(3) normal(3) spring(3)): the
//   key's elementary IDs are 1 for simple bodies (HookeMemoryContactForce
//   Model.cpp:218-221), (Component::writeContactMemory2014, Component.cpp:
//   776-801).
// Numbers as GrainsExec::doubleToString(ios::scientific, 16 digits) (d16).
// Particle IDs are the reference's (1-based insertion numbers, Particle.cpp:
// 45-50); an obstacle partner is -(k + 1) for wall k (obstacle IDs count
// down from -1, Obstacle.cpp:28-32).  Both partners of a pair carry it, the
// higher ID with the signs reversed (HookeMemoryContactForceModel.cpp:
// 191-192).  The transform type is written 3 (translation | rotation), what
// the reference's particles carry after their first step.
namespace {

// GrainsExec::doubleToString(ios::scientific, 16, v) (Base/src/GrainsExec.cpp:
// 212-224): an exact zero in the stream's default format
std::string d16(double v) {
  if (v == 0.) return std::signbit(v) ? "-0" : "0";
  char buf[40];
  std::snprintf(buf, sizeof(buf), "%.16e", v);
  return buf;
}

// Matrix::setRotation (Geometry/src/Matrix.cpp:114-127) of q = (x, y, z, w).
void rotationOf(const double* q, double* m) {
  const double x = q[0], y = q[1], z = q[2], w = q[3];
  const double s = 2.0 / (x * x + y * y + z * z + w * w);
  const double xs = x * s, ys = y * s, zs = z * s;
  const double wx = w * xs, wy = w * ys, wz = w * zs;
  const double xx = x * xs, xy = x * ys, xz = x * zs, yy = y * ys, yz = y * zs, zz = z * zs;
  const double r[9] = {1.0 - (yy + zz), xy - wz, xz + wy, xy + wz, 1.0 - (xx + zz), yz - wx,
                       xz - wy, yz + wx, 1.0 - (xx + yy)};
  for (int k = 0; k < 9; ++k) m[k] = r[k];
}

struct MapEntry {
  int partner;          // reload ID
  double v[9];          // kdelta, normal, spring
};

}  // namespace

}  // extern "C"

namespace {

// Binary record helpers of the Hybrid reload format (raw host-order bytes,
// as std::ostream::write of the reference's fields).
template <typename V>
void putRaw(std::string& out, V const& v) {
  out.append(reinterpret_cast<const char*>(&v), sizeof(V));
}
template <typename V>
V getRaw(const char*& p, const char* end) {
  if (end - p < (std::ptrdiff_t)sizeof(V)) throw std::runtime_error("truncated particle record");
  V v;
  std::memcpy(&v, p, sizeof(V));
  p += sizeof(V);
  return v;
}

}  // namespace

extern "C" {

// The particle file of a Format2024 reload from the device state: text
// (Particle::write2014, Component/src/Particle.cpp:1167-1176) or, hybrid,
// binary records each preceded by its byte count (AllComponents::write,
// AllComponents.cpp:1387-1404; Particle::write2014_binary,
// Particle.cpp:1183-1193, get_numberOfBytes :1201-1208).
static int writeReloadParticles(gdem_handle h, const char* path, bool hybrid) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->started || !path) throw std::runtime_error("no stepped state to write");
    if (s->inst.size() != 1) throw std::runtime_error("a reload file holds one system, not a batch");
    DevState& S = s->S;
    const size_t n = (size_t)S.n;
    std::vector<double> x(3 * n), v(3 * n), w(3 * n), q(4 * n), F(3 * n), T(3 * n), B(9 * n);
    CK(cudaStreamSynchronize(s->stream));
    int rc = gdem_download_state(h, x.data(), v.data(), w.data(), nullptr, q.data(), F.data(),
                                 T.data());
    if (rc != GDEM_OK) throw std::runtime_error(g_last_error);
    if (S.basis) {
      rc = gdem_download_basis(h, B.data());
      if (rc != GDEM_OK) throw std::runtime_error(g_last_error);
    } else {
      for (size_t i = 0; i < n; ++i) rotationOf(&q[4 * i], &B[9 * i]);
    }
    auto refId = [&](size_t i) { return s->ref_ids.empty() ? (int)i + 1 : s->ref_ids[i]; };
    // contact memory of the last evaluation: the table the next one reads
    HistTable const& t = S.hist_old;
    const size_t hc = size_t(1) << t.log2cap;
    std::vector<unsigned long long> keys(hc);
    CK(cudaMemcpy(keys.data(), t.keys, hc * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    const bool fp64 = s->precision == GDEM_FP64;
    std::vector<double> vd(fp64 ? 9 * hc : 0);
    std::vector<float> vf(fp64 ? 0 : 9 * hc);
    if (fp64) CK(cudaMemcpy(vd.data(), t.vals, vd.size() * sizeof(double), cudaMemcpyDeviceToHost));
    else CK(cudaMemcpy(vf.data(), t.vals, vf.size() * sizeof(float), cudaMemcpyDeviceToHost));
    std::vector<std::vector<MapEntry>> maps(n);
    const unsigned tag = (unsigned)s->epoch & kTagMask;
    const unsigned idmask = (1u << kMaxIdBits) - 1u;
    for (size_t k = 0; k < hc; ++k) {
      if (tagOf(keys[k]) != tag) continue;
      const unsigned base_hi = (unsigned)((keys[k] >> kMaxIdBits) & idmask);
      const unsigned base_lo = (unsigned)(keys[k] & idmask);
      double val[9];
      for (int c = 0; c < 9; ++c) val[c] = fp64 ? vd[9 * k + c] : (double)vf[9 * k + c];
      const size_t a = base_hi;
      if (a >= n) continue;
      if (base_lo < n) {
        const size_t b = base_lo;
        MapEntry ea{refId(b), {}}, eb{refId(a), {}};
        for (int c = 0; c < 9; ++c) { ea.v[c] = val[c]; eb.v[c] = -val[c]; }
        maps[a].push_back(ea);
        maps[b].push_back(eb);
      } else {
        const int wall = (int)(idmask - base_lo);
        MapEntry ea{-(wall + 1), {}};
        for (int c = 0; c < 9; ++c) ea.v[c] = val[c];
        maps[a].push_back(ea);
      }
    }
    if (hybrid) {
      std::ofstream out(path, std::ios::out | std::ios::binary);
      if (!out) throw std::runtime_error(std::string("cannot write ") + path);
      std::string rec;
      for (size_t i = 0; i < n; ++i) {
        auto& m = maps[i];
        std::sort(m.begin(), m.end(), [](MapEntry const& p, MapEntry const& r) { return p.partner < r.partner; });
        // class, ID, tag, activity | origin, basis, transform type | v, q
        // (w first), omega, F, T | map size, entries (key triple, active,
        // 9 doubles)
        const size_t nb = 3 * sizeof(int) + sizeof(unsigned) + 12 * sizeof(double) +
                          sizeof(unsigned) + 16 * sizeof(double) + sizeof(int) +
                          m.size() * (4 * sizeof(int) + 9 * sizeof(double));
        rec.clear();
        putRaw(rec, nb);
        putRaw(rec, s->h_type[i]);
        putRaw(rec, refId(i));
        putRaw(rec, 0);
        putRaw(rec, 1u);
        for (int d = 0; d < 3; ++d) putRaw(rec, x[3 * i + d]);
        for (int k = 0; k < 9; ++k) putRaw(rec, B[9 * i + k]);
        putRaw(rec, 3u);
        for (int d = 0; d < 3; ++d) putRaw(rec, v[3 * i + d]);
        putRaw(rec, q[4 * i + 3]);
        for (int d = 0; d < 3; ++d) putRaw(rec, q[4 * i + d]);
        for (int d = 0; d < 3; ++d) putRaw(rec, w[3 * i + d]);
        for (int d = 0; d < 3; ++d) putRaw(rec, F[3 * i + d]);
        for (int d = 0; d < 3; ++d) putRaw(rec, T[3 * i + d]);
        putRaw(rec, (int)m.size());
        for (auto const& e : m) {
          putRaw(rec, 1);
          putRaw(rec, e.partner);
          putRaw(rec, 1);
          putRaw(rec, 1);
          for (int c = 0; c < 9; ++c) putRaw(rec, e.v[c]);
        }
        out.write(rec.data(), (std::streamsize)rec.size());
      }
      if (!out) throw std::runtime_error(std::string("write failed: ") + path);
      return GDEM_OK;
    }
    std::ofstream out(path);
    if (!out) throw std::runtime_error(std::string("cannot write ") + path);
    for (size_t i = 0; i < n; ++i) {
      auto& m = maps[i];
      std::sort(m.begin(), m.end(), [](MapEntry const& p, MapEntry const& r) { return p.partner < r.partner; });
      const double* b = &B[9 * i];
      out << s->h_type[i] << " " << refId(i) << " 0 1 ";
      out << d16(x[3 * i]) << " " << d16(x[3 * i + 1]) << " " << d16(x[3 * i + 2]);
      for (int k = 0; k < 9; ++k) out << " " << d16(b[k]);
      out << " 3 ";
      out << d16(v[3 * i]) << " " << d16(v[3 * i + 1]) << " " << d16(v[3 * i + 2]) << " ";
      out << d16(q[4 * i + 3]) << " " << d16(q[4 * i]) << " " << d16(q[4 * i + 1]) << " "
          << d16(q[4 * i + 2]) << " ";
      out << d16(w[3 * i]) << " " << d16(w[3 * i + 1]) << " " << d16(w[3 * i + 2]) << " ";
      out << d16(F[3 * i]) << " " << d16(F[3 * i + 1]) << " " << d16(F[3 * i + 2]) << " ";
      out << d16(T[3 * i]) << " " << d16(T[3 * i + 1]) << " " << d16(T[3 * i + 2]);
      out << " " << m.size();
      for (auto const& e : m) {
        out << " 1 " << e.partner << " 1 1";
        for (int c = 0; c < 9; ++c) out << " " << d16(e.v[c]);
      }
      out << "\n";
    }
    if (!out) throw std::runtime_error(std::string("write failed: ") + path);
    return GDEM_OK;
  });
}

int gdem_write_reload_particles(gdem_handle h, const char* path) {
  return writeReloadParticles(h, path, false);
}
int gdem_write_reload_particles_hybrid(gdem_handle h, const char* path) {
  return writeReloadParticles(h, path, true);
}

// A Format2024 reload's particle file into a fresh system: text
// (Particle::read2014, Component/src/Particle.cpp:972-1024) or hybrid binary
// records (AllComponents::read_particles, AllComponents.cpp:1163-1256;
// Particle::read2014_binary, Particle.cpp:1032-1080).
static int readReloadParticles(gdem_handle h, const char* path, bool hybrid) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !path) throw std::runtime_error("invalid arguments");
    if (s->have_state) throw std::runtime_error("the system already has particles");
    if (s->inst.size() != 1) throw std::runtime_error("a reload file holds one system, not a batch");
    std::ifstream in(path, hybrid ? std::ios::in | std::ios::binary : std::ios::in);
    if (!in) throw std::runtime_error(std::string("cannot read ") + path);
    struct Rec {
      int cls, id;
      double x[3], B[9], v[3], q[4], w[3], F[3], T[3];
      std::vector<MapEntry> map;
    };
    std::vector<Rec> recs;
    auto keep = [&](Rec&& r, int tag, unsigned active) {
      if (tag > 1 || !active) return;   // periodic clones and waiting particles
      if (r.cls < 0 || r.cls >= (int)s->inst[0].types.size())
        throw std::runtime_error("particle class out of range in " + std::string(path));
      recs.push_back(std::move(r));
    };
    std::string line;
    while (hybrid) {
      size_t nb = 0;
      if (!in.read(reinterpret_cast<char*>(&nb), sizeof nb)) break;
      if (nb > (size_t(1) << 24)) throw std::runtime_error("malformed particle record in " + std::string(path));
      std::string buf(nb, '\0');
      if (!in.read(&buf[0], (std::streamsize)nb)) throw std::runtime_error("truncated particle record in " + std::string(path));
      const char* p = buf.data();
      const char* end = p + nb;
      Rec r;
      r.cls = getRaw<int>(p, end);
      r.id = getRaw<int>(p, end);
      const int tag = getRaw<int>(p, end);
      const unsigned active = getRaw<unsigned>(p, end);
      for (double& d : r.x) d = getRaw<double>(p, end);
      for (double& d : r.B) d = getRaw<double>(p, end);
      (void)getRaw<unsigned>(p, end);
      for (double& d : r.v) d = getRaw<double>(p, end);
      r.q[3] = getRaw<double>(p, end);
      for (int d = 0; d < 3; ++d) r.q[d] = getRaw<double>(p, end);
      for (double& d : r.w) d = getRaw<double>(p, end);
      for (double& d : r.F) d = getRaw<double>(p, end);
      for (double& d : r.T) d = getRaw<double>(p, end);
      const int nm = getRaw<int>(p, end);
      for (int k = 0; k < nm; ++k) {
        MapEntry e;
        (void)getRaw<int>(p, end);
        e.partner = getRaw<int>(p, end);
        (void)getRaw<int>(p, end);
        const int act = getRaw<int>(p, end);
        for (double& d : e.v) d = getRaw<double>(p, end);
        if (act) r.map.push_back(e);
      }
      if (p != end) throw std::runtime_error("particle record size mismatch in " + std::string(path));
      keep(std::move(r), tag, active);
    }
    while (!hybrid && std::getline(in, line)) {
      std::istringstream is(line);
      Rec r;
      int tag = 0, ttype = 0;
      unsigned active = 0;
      if (!(is >> r.cls >> r.id >> tag >> active)) continue;   // blank line
      for (double& d : r.x) is >> d;
      for (double& d : r.B) is >> d;
      is >> ttype;
      for (double& d : r.v) is >> d;
      is >> r.q[3] >> r.q[0] >> r.q[1] >> r.q[2];
      for (double& d : r.w) is >> d;
      for (double& d : r.F) is >> d;
      for (double& d : r.T) is >> d;
      int nm = 0;
      is >> nm;
      for (int k = 0; k < nm; ++k) {
        int e0 = 0, e1 = 0;
        unsigned act = 0;
        MapEntry e;
        is >> e0 >> e.partner >> e1 >> act;
        for (double& d : e.v) is >> d;
        if (act) r.map.push_back(e);
      }
      if (!is) throw std::runtime_error("malformed particle line in " + std::string(path));
      keep(std::move(r), tag, active);
    }
    if (recs.empty()) throw std::runtime_error(std::string("no particle in ") + path);
    std::sort(recs.begin(), recs.end(), [](Rec const& a, Rec const& b) { return a.id < b.id; });
    const size_t n = recs.size();
    std::map<int, int> index;
    std::vector<int> type(n), ids(n);
    std::vector<double> x(3 * n), v(3 * n), w(3 * n), q(4 * n), F(3 * n), T(3 * n), B(9 * n);
    for (size_t i = 0; i < n; ++i) {
      Rec const& r = recs[i];
      if (!index.emplace(r.id, (int)i).second) throw std::runtime_error("duplicate particle ID");
      type[i] = r.cls;
      ids[i] = r.id;
      for (int d = 0; d < 3; ++d) {
        x[3 * i + d] = r.x[d]; v[3 * i + d] = r.v[d]; w[3 * i + d] = r.w[d];
        F[3 * i + d] = r.F[d]; T[3 * i + d] = r.T[d];
      }
      for (int d = 0; d < 4; ++d) q[4 * i + d] = r.q[d];
      for (int k = 0; k < 9; ++k) B[9 * i + k] = r.B[k];
      if (s->inst[0].reload_reset) {
        // ParticleKinematics::reset (Component/src/ParticleKinematics.cpp:
        // 165-170): both velocities and the kinematics quaternion; the
        // orientation of the transform (the basis) is kept
        for (int d = 0; d < 3; ++d) v[3 * i + d] = w[3 * i + d] = 0.;
        q[4 * i] = q[4 * i + 1] = q[4 * i + 2] = 0.;
        q[4 * i + 3] = 1.;
      }
    }
    auto check = [](int code) {
      if (code != GDEM_OK) throw std::runtime_error(g_last_error);
    };
    check(gdem_upload_state(h, (int64_t)n, nullptr, type.data(), x.data(), v.data(), w.data(),
                            nullptr, q.data()));
    check(gdem_upload_basis(h, B.data()));
    s->ref_ids = ids;
    // contact memory: owner index, partner index (walls -(k+2))
    std::vector<int> owner, partner;
    std::vector<double> kd, pn, sp;
    for (size_t i = 0; i < n; ++i)
      for (auto const& e : recs[i].map) {
        int p;
        if (e.partner >= 0) {
          auto it = index.find(e.partner);
          if (it == index.end()) continue;   // a partner not in the file
          p = it->second;
        } else {
          p = e.partner - 1;   // obstacle -(k + 1) is wall k, -(k + 2) here
        }
        owner.push_back((int)i);
        partner.push_back(p);
        for (int c = 0; c < 3; ++c) {
          kd.push_back(e.v[c]); pn.push_back(e.v[3 + c]); sp.push_back(e.v[6 + c]);
        }
      }
    check(gdem_upload_forces(h, F.data(), T.data()));
    check(gdem_upload_history(h, (int64_t)owner.size(), owner.data(), partner.data(), kd.data(),
                              pn.data(), sp.data()));
    return GDEM_OK;
  });
}

int gdem_read_reload_particles(gdem_handle h, const char* path) {
  return readReloadParticles(h, path, false);
}
int gdem_read_reload_particles_hybrid(gdem_handle h, const char* path) {
  return readReloadParticles(h, path, true);
}

int gdem_download_cells(gdem_handle h, int* ijk) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->started || !ijk) throw std::runtime_error("no binned state");
    DevState& S = s->S;
    int* d = reinterpret_cast<int*>(s->d_stage);
    launch_cells_by_id(S, d, 0, s->stream);
    CK(cudaMemcpyAsync(ijk, d, 3 * (size_t)S.n * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return GDEM_OK;
  });
}

int gdem_set_diagnostics(gdem_handle h, int on) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state) throw std::runtime_error("upload the state first");
    DevState& S = s->S;
    if (on && !S.pair_delta) {
      S.pair_delta = s->alloc<double>((size_t)S.pair_cap);
      S.wall_delta = s->alloc<double>((size_t)S.cap * S.max_walls);
      S.pair_force = s->alloc<double>((size_t)S.pair_cap * 3);
      S.wall_force = s->alloc<double>((size_t)S.cap * S.max_walls * 3);
    }
    // the graphs hold the evaluation without diagnostics (an evaluation with
    // them runs as plain launches), so they stay valid either way
    S.diag = on ? 1 : 0;
    s->diag = on != 0;
    return GDEM_OK;
  });
}

int gdem_download_contacts(gdem_handle h, int64_t capacity, int64_t* count, int* id0, int* id1,
                           double* delta, double* force) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->started || !count) throw std::runtime_error("invalid arguments");
    DevState& S = s->S;
    if (!S.pair_delta) throw std::runtime_error("enable diagnostics before the step");
    size_t n = (size_t)S.n;
    std::vector<int> ids(n), np(n), off(n + 1);
    CK(cudaMemcpy(ids.data(), S.id, n * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(np.data(), S.npairs, n * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(off.data(), S.pair_off, (n + 1) * sizeof(int), cudaMemcpyDeviceToHost));
    size_t ne = 0;
    for (size_t t = 0; t < n; ++t) ne = std::max(ne, (size_t)off[t] + (size_t)np[t]);
    std::vector<int> pairs(ne);
    std::vector<double> pd(ne), pf(3 * ne);
    std::vector<double> wd(n * S.max_walls), wf(3 * n * S.max_walls);
    std::vector<int4> cells(n);
    CK(cudaMemcpy(pairs.data(), S.pairs, ne * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(pd.data(), S.pair_delta, pd.size() * sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(wd.data(), S.wall_delta, wd.size() * sizeof(double), cudaMemcpyDeviceToHost));
    if (force) {
      CK(cudaMemcpy(pf.data(), S.pair_force, pf.size() * sizeof(double), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(wf.data(), S.wall_force, wf.size() * sizeof(double), cudaMemcpyDeviceToHost));
    }
    CK(cudaMemcpy(cells.data(), S.cellc, n * sizeof(int4), cudaMemcpyDeviceToHost));
    int64_t c = 0;
    for (size_t t = 0; t < n; ++t) {
      for (int e = 0; e < np[t]; ++e) {
        size_t slot = (size_t)off[t] + e;
        int u = pairs[slot] & ((1 << 27) - 1);   // pair-list entries
        double dl = pd[slot];
        if (!(dl < 0.) || !(ids[t] < ids[u])) continue;
        if (c < capacity && id0) {
          id0[c] = ids[t]; id1[c] = ids[u]; delta[c] = dl;
          if (force) for (int d = 0; d < 3; ++d) force[3 * c + d] = pf[3 * slot + d];
        }
        ++c;
      }
      int nw = s->inst[cells[t].w].walls.size();
      for (int k = 0; k < nw; ++k) {
        size_t slot = t * S.max_walls + k;
        double dl = wd[slot];
        if (!(dl < 0.)) continue;
        if (c < capacity && id0) {
          id0[c] = ids[t]; id1[c] = -(k + 2); delta[c] = dl;
          if (force) for (int d = 0; d < 3; ++d) force[3 * c + d] = wf[3 * slot + d];
        }
        ++c;
      }
    }
    *count = c;
    return GDEM_OK;
  });
}

int gdem_download_coordination(gdem_handle h, int* coord) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || !coord) throw std::runtime_error("invalid arguments");
    DevState& S = s->S;
    const size_t n = (size_t)S.n;
    if (s->evaluated == 0) {
      // no force evaluation since the state was set: the reference's
      // particles enter with none (Particle::InitializeForce)
      std::fill(coord, coord + n, 0);
      return GDEM_OK;
    }
    if (s->evaluated != 1 || !S.pair_delta)
      throw std::runtime_error("the last force evaluation ran without diagnostics");
    int* d = reinterpret_cast<int*>(s->d_stage);
    launch_coordination_by_id(S, d, 0, s->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(coord, d, n * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return GDEM_OK;
  });
}

int gdem_upload_support_vertices(gdem_handle h, const int* vertex) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || !vertex) throw std::runtime_error("invalid arguments");
    DevState& S = s->S;
    if (!S.curv) return GDEM_OK;   // no polyhedron class
    const size_t n = (size_t)S.n;
    std::vector<int> ids(n), slot(n);
    CK(cudaStreamSynchronize(s->stream));
    CK(cudaMemcpy(ids.data(), S.id, n * sizeof(int), cudaMemcpyDeviceToHost));
    for (size_t t = 0; t < n; ++t) {
      const int i = ids[t];
      TypeDesc const& tp = s->h_types[s->type_base[s->h_inst[i]] + s->h_type[i]];
      const int v = vertex[i];
      if (tp.shape == 2 && (v < 0 || v >= tp.poly_count))
        throw std::runtime_error("support vertex out of range for particle " + std::to_string(i));
      slot[t] = tp.shape == 2 ? v : 0;
    }
    CK(cudaMemcpyAsync(S.curv, slot.data(), n * sizeof(int), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return GDEM_OK;
  });
}

int gdem_download_support_vertices(gdem_handle h, int* vertex) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || !vertex) throw std::runtime_error("invalid arguments");
    DevState& S = s->S;
    const size_t n = (size_t)S.n;
    if (!S.curv) {
      std::fill(vertex, vertex + n, 0);
      return GDEM_OK;
    }
    std::vector<int> ids(n), cur(n);
    CK(cudaStreamSynchronize(s->stream));
    CK(cudaMemcpy(ids.data(), S.id, n * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(cur.data(), S.curv, n * sizeof(int), cudaMemcpyDeviceToHost));
    for (size_t t = 0; t < n; ++t) vertex[ids[t]] = cur[t];
    return GDEM_OK;
  });
}

int gdem_download_ids(gdem_handle h, int* ids) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || !ids) throw std::runtime_error("invalid arguments");
    const size_t n = s->h_type.size();
    for (size_t i = 0; i < n; ++i) ids[i] = s->ref_ids.empty() ? (int)i + 1 : s->ref_ids[i];
    return GDEM_OK;
  });
}

int gdem_download_classes(gdem_handle h, int* cls) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !s->have_state || !cls) throw std::runtime_error("invalid arguments");
    std::copy(s->h_type.begin(), s->h_type.end(), cls);
    return GDEM_OK;
  });
}

int gdem_status(gdem_handle h, int* bits, int reset) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !bits) throw std::runtime_error("invalid arguments");
    if (s->have_state) s->readStatus();
    *bits = s->status_host;
    if (reset) {
      s->status_host = 0;
      if (s->have_state) CK(cudaMemset(s->S.status, 0, sizeof(int)));
    }
    return GDEM_OK;
  });
}

int gdem_grid(gdem_handle h, int k, int* nb, double* edge, double* origin) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || k < 0 || k >= (int)s->inst.size()) throw std::runtime_error("invalid arguments");
    GridDesc const& g = s->inst[k].grid;
    for (int d = 0; d < 3; ++d) {
      if (nb) nb[d] = g.nb[d];
      if (edge) edge[d] = g.edge[d];
      if (origin) origin[d] = g.lc_origin[d];
    }
    return GDEM_OK;
  });
}

int gdem_num_instances(gdem_handle h) {
  System* s = sys(h);
  if (!s) {
    setLastError("invalid handle");
    return GDEM_ERR_INVALID;
  }
  return (int)s->inst.size();
}

int64_t gdem_num_particles(gdem_handle h) {
  System* s = sys(h);
  return s && s->have_state ? s->S.n : 0;
}

double gdem_last_step_ms(gdem_handle h) {
  System* s = sys(h);
  return s ? s->last_ms : 0.;
}

int gdem_class_envelope(gdem_handle h, int cls, int* code, int point_capacity, int* npoints,
                        double* points, int word_capacity, int* nwords, int* nfaces, int* faces) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !code || !npoints || !nwords || !nfaces) throw std::runtime_error("invalid arguments");
    InstanceDesc const& I = s->inst[0];
    if (cls < 0 || cls >= (int)I.types.size()) throw std::runtime_error("class out of range");
    TypeDesc const& t = I.types[cls];
    std::vector<double> P;
    std::vector<int> W;
    int nf = 0;
    const double ex = t.extent[0], ey = t.extent[1], ez = t.extent[2];
    if (t.shape == 0) {
      // Sphere::getEnvelope (Geometry/src/Sphere.cpp:116-123): the centre
      *code = 1;
      P = {0., 0., 0.};
    } else if (t.shape == 1) {
      // Box::getNbCorners 666; Box::setCornersFaces (Geometry/src/Box.cpp:
      // 91-147): the eight corners and the six faces in its order
      *code = 666;
      P = {-ex, -ey, -ez, ex, -ey, -ez, ex, -ey, ez, -ex, -ey, ez,
           -ex, ey, -ez, ex, ey, -ez, ex, ey, ez, -ex, ey, ez};
      const int F[6][4] = {{4, 5, 6, 7}, {5, 1, 2, 6}, {1, 0, 3, 2},
                           {0, 4, 7, 3}, {4, 0, 1, 5}, {3, 7, 6, 2}};
      for (auto const& f : F) {
        W.push_back(4);
        W.insert(W.end(), f, f + 4);
      }
      nf = 6;
    } else if (t.shape == 3) {
      // Cylinder::getNbCorners 777; getEnvelope (Geometry/src/Cylinder.cpp:
      // 142-151): the bottom centre, a bottom rim point, the top centre
      *code = 777;
      P = {0., -ey, 0., ex, -ey, 0., 0., ey, 0.};
    } else {
      // Polytope::getNbCorners / getEnvelope (Geometry/src/Polytope.cpp:
      // 76-95): the vertices in file order; the faces as the file lists them
      *code = t.poly_count;
      P.assign(I.poly_verts.begin() + 3 * (size_t)t.poly_begin,
               I.poly_verts.begin() + 3 * (size_t)(t.poly_begin + t.poly_count));
      for (auto const& f : I.class_faces[cls]) {
        W.push_back((int)f.size());
        W.insert(W.end(), f.begin(), f.end());
      }
      nf = (int)I.class_faces[cls].size();
    }
    *npoints = (int)P.size() / 3;
    *nwords = (int)W.size();
    *nfaces = nf;
    if (points && point_capacity >= *npoints) std::copy(P.begin(), P.end(), points);
    if (faces && word_capacity >= *nwords) std::copy(W.begin(), W.end(), faces);
    return GDEM_OK;
  });
}

int gdem_read_reload_contact_models(gdem_handle h, const char* header) {
  return guarded([&] {
    System* s = sys(h);
    if (!s || !header) throw std::runtime_error("invalid arguments");
    if (s->inst.size() != 1) throw std::runtime_error("a reload holds one system, not a batch");
    // the header's "<ContactForceModels> <file> </ContactForceModels>" line
    // (ContactBuilderFactory::save); the file is looked for in the header's
    // directory (ContactBuilderFactory::reload, Component/src/
    // ContactBuilderFactory.cpp:199-212)
    std::ifstream in(header);
    if (!in) throw std::runtime_error(std::string("cannot read ") + header);
    std::string tok, file;
    while (in >> tok)
      if (tok == "<ContactForceModels>") { in >> file; break; }
    if (file.empty()) throw std::runtime_error(std::string("no contact force models named in ") + header);
    const std::string hp(header);
    const size_t cut = hp.find_last_of('/');
    const std::string dir = cut == std::string::npos ? std::string(".") : hp.substr(0, cut);
    const size_t fcut = file.find_last_of('/');
    const std::string name = fcut == std::string::npos ? file : file.substr(fcut + 1);
    auto root = parseXmlFile(dir + "/" + name);
    // material values (powers of two) by name; a model's key is the OR of
    // its two materials' values (ContactBuilderFactory::contactForceModel)
    std::map<std::string, int> matval;
    if (XmlNode const* mats = root->name == "Materials" ? root.get() : root->find("Materials"))
      for (auto const& c : mats->children)
        if (c->name == "Material") matval[c->valueS()] = (int)c->attrD("value");
    std::map<int, ModelDesc> bykey;
    if (XmlNode const* cms = root->find("ContactForceModels"))
      for (auto const& c : cms->children) {
        if (c->name != "ContactForceModel") continue;
        const int type = (int)c->attrD("type"), key = (int)c->attrD("value");
        // the models' constructors from a parameter map (Hooke[Memory]
        // ContactForceModel.cpp:11-25): a parameter absent from the file is 0
        std::map<std::string, double> P;
        if (XmlNode const* ps = c->child("Parameters"))
          for (auto const& q : ps->children)
            if (q->name == "Parameter") P[q->attr("name")] = q->valueD();
        auto get = [&P](const char* k) { auto it = P.find(k); return it == P.end() ? 0. : it->second; };
        ModelDesc m{};
        m.kn = get("kn"); m.en = get("en"); m.etat = get("etat"); m.muc = get("muc");
        if (type == 1) {          // HookeMemory
          m.kt = get("kt"); m.mur = get("mur"); m.etarpf = get("etarpf"); m.epst = get("epst");
          m.memory = 1;
          m.rolling = m.mur != 0. ? 1 : 0;
        } else if (type == 0) {   // Hooke
          m.kr = get("kr");
          m.memory = 0;
          m.rolling = m.kr != 0. ? 1 : 0;
        } else {
          throw std::runtime_error("Hertz contact models are not supported");
        }
        m.beta = std::log(m.en) / std::sqrt(PI * PI + std::log(m.en) * std::log(m.en));
        m.valid = 1;
        bykey[key] = m;
      }
    InstanceDesc& I = s->inst[0];
    for (int a = 0; a < I.nmat; ++a)
      for (int b = 0; b < I.nmat; ++b) {
        auto ia = matval.find(I.mat_names[a]), ib = matval.find(I.mat_names[b]);
        if (ia == matval.end() || ib == matval.end()) continue;
        auto it = bykey.find(ia->second | ib->second);
        if (it != bykey.end()) I.models[a * kMaxMat + b] = it->second;
      }
    s->uploadModels();
    return GDEM_OK;
  });
}

int gdem_set_contact_memory_pruning(gdem_handle h, int prune) {
  return guarded([&] {
    System* s = sys(h);
    if (!s) throw std::runtime_error("invalid handle");
    if (s->have_state) throw std::runtime_error("set the contact-memory pruning before the particles");
    s->prune_memory = prune != 0;
    s->invalidateGraphs();
    return GDEM_OK;
  });
}

int gdem_use_graphs(gdem_handle h, int on) {
  return guarded([&] {
    System* s = sys(h);
    if (!s) throw std::runtime_error("invalid handle");
    s->use_graphs = on != 0;
    s->invalidateGraphs();
    return GDEM_OK;
  });
}

void gdem_destroy(gdem_handle h) {
  if (!h) return;
  gdem_rawdata_end(h);   // closes the system's RawData files, if open
  delete sys(h);
}

}  // extern "C"
