// gdem_basilisk.cpp -- the Basilisk coupling C ABI of Grains3D
// (GRAINS_V1/Grains/InterfaceCBasilisk/include/InterfaceGrains3DBasilisk.h,
// src/InterfaceGrains3DBasilisk.cpp) on the B200 DEM step.  Built as
// libgrains_b200_basilisk.so over libgrains_b200.so; it exports the same
// symbols with the same signatures, so a Basilisk DLMFD build links it in
// place of the reference's interface library.
//
// Like the reference (InterfaceGrains3DBasilisk.cpp:15) it keeps one system
// in a file-static handle, has no error returns (errors are printed and
// recorded, and later calls then do nothing) and is meant for one process.
// What each entry does:
//   Init_Grains       the XML's system (FP64; GRAINS_B200_PRECISION=fp32split
//                     selects the FP32-split mode) with the particles of its
//                     Construction/Reload file (the "<stem>_Particles.result"
//                     file of the Format2024 reload, or
//                     "<stem>_Particles.result.bin" when the reload's reading
//                     mode is Hybrid, AllComponents::read and read_particles),
//                     the contact force models of the reload's
//                     material-contact file (GrainsCoupledWithFluid::
//                     Construction reads them there, not in the XML), the
//                     fluid density in the weight; the coupling factor
//                     stays 1, as for the reference's reloaded particles
//                     whatever b_fluidcorrectedacc is (see Init_Grains).
//                     The particle classes and obstacles come from the XML,
//                     which must describe the system the reload was written
//                     from (the reference takes them from the reload header).
//   Simu_Grains       sub-steps over the fluid step as
//                     GrainsCoupledWithFluid::Simulation (:123-133): ndt from
//                     the XML's TimeStep, dt = dt_fluid / ndt within
//                     [mindt, maxdt].
//   GrainsToBasilisk  the rigid-body stream of GrainsCoupledWithFluid::
//                     GrainsToFluid (:912-1120), tokens separated by one
//                     space (InterfaceGrains3DBasilisk.cpp:62-82), for every
//                     class: corner code, envelope points through the
//                     particle's transform, faces (gdem_class_envelope).
//   UpdateVelocityGrains  velocities from the fluid (updateParticlesVelocity).
//   SaveResults_Grains  the XML's RawData writer, if any (started at the first
//                     call, an output time at each later one; the last
//                     sub-step of Simu_Grains then records its contacts for
//                     the coordination numbers), and a Format2024 particle
//                     file "grains_b200_<cycle>_Particles".
// Contact memory: the reference's coupled step never prunes a contact map
// entry whose contact has ended (it skips Grains::computeParticlesForceAnd
// Torque's setContactMapToFalse / updateContactMap), so a pair that touches
// again resumes its old tangential spring; the same here
// (gdem_set_contact_memory_pruning(h, 0)).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/grains_b200.h"

namespace {

gdem_handle g_sys = nullptr;
bool g_error = false;
double g_time = 0.;
int g_cycle = 0;
int g_ndt = 1;
double g_min_dt = 0., g_max_dt = 0.;
int64_t g_n = 0;
std::vector<int> g_class;      // particle class by particle index
std::vector<int> g_ids;        // reload IDs by particle index
bool g_restart = false;
std::string g_raw_root;        // the XML's RawData writer ("" if none)
int g_raw_binary = 0;
bool g_raw_started = false;

void fail(const char* where) {
  std::fprintf(stderr, "Grains3D B200 coupling: %s: %s\n", where, gdem_last_error());
  g_error = true;
}

// GrainsExec::doubleToString(ios::scientific, 16, v)
std::string d16(double v) {
  if (v == 0.) return std::signbit(v) ? "-0" : "0";
  char buf[40];
  std::snprintf(buf, sizeof(buf), "%.16e", v);
  return buf;
}

// The reading mode of a Format2024 reload file: the word after the
// "NbFiles <n>" line, "Hybrid" or "Text" (AllComponents::write, Component/
// src/AllComponents.cpp:1370-1374; AllComponents::read, :1114-1126).  Returns
// false when the file cannot be read or has no such line.  The header is
// the reload name with ".result" appended (Grains::Construction, Base/src/
// Grains.cpp:811, GrainsExec::fullResultFileName); the name as written is
// tried when that file does not exist.
bool readReloadMode(const std::string& reload, bool& hybrid) {
  FILE* f = std::fopen((reload + ".result").c_str(), "r");
  if (!f) f = std::fopen(reload.c_str(), "r");
  if (!f) return false;
  char tok[4096];
  bool found = false;
  while (std::fscanf(f, "%4095s", tok) == 1) {
    if (std::strcmp(tok, "NbFiles") != 0) continue;
    long nfiles = 0;
    if (std::fscanf(f, "%ld %4095s", &nfiles, tok) == 2) {
      hybrid = std::strcmp(tok, "Hybrid") == 0;
      found = true;
    }
    break;
  }
  std::fclose(f);
  return found;
}

// The reload header (the reload name with ".result" appended, else the
// name as written) when it names a material-contact file, else "".
std::string headerWithContactModels(const std::string& reload) {
  for (const std::string& path : {reload + ".result", reload}) {
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) continue;
    char tok[4096];
    bool named = false;
    while (!named && std::fscanf(f, "%4095s", tok) == 1)
      named = std::strcmp(tok, "<ContactForceModels>") == 0;
    std::fclose(f);
    return named ? path : std::string();
  }
  return std::string();
}

// Particle IDs (1-based) and classes, by particle index, from the handle.
bool readIds() {
  g_ids.assign((size_t)g_n, 0);
  g_class.assign((size_t)g_n, 0);
  return g_n == 0 || (gdem_download_ids(g_sys, g_ids.data()) == GDEM_OK &&
                      gdem_download_classes(g_sys, g_class.data()) == GDEM_OK);
}

// Matrix::setRotation (Geometry/src/Matrix.cpp:114-127) of q = (x, y, z, w):
// a sphere's orientation, which the reference carries in its transform.
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

// Row-major 3x3 product as Matrix::operator* (Geometry/src/Matrix.cpp).
void matmul(const double* a, const double* b, double* c) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      c[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}

}  // namespace

extern "C" {

void Init_Grains(char const* inputfile, double fluid_rho, const bool b_restart,
                 const bool b_fluidcorrectedacc) {
  // the particles always come from the XML's reload file; b_restart makes
  // the RawData writer append (a reload of type "same")
  g_restart = b_restart;
  if (g_sys) { gdem_destroy(g_sys); g_sys = nullptr; }
  g_error = false;
  g_raw_started = false;
  const char* prec = std::getenv("GRAINS_B200_PRECISION");
  const int mode = (prec && std::strcmp(prec, "fp32split") == 0) ? GDEM_FP32_SPLIT : GDEM_FP64;
  if (gdem_create(inputfile, mode, &g_sys) != GDEM_OK) { fail("Init_Grains"); return; }
  // the coupled step keeps the memory of ended contacts
  // (GrainsCoupledWithFluid::Simulation never prunes it)
  if (gdem_set_contact_memory_pruning(g_sys, 0) != GDEM_OK) { fail("Init_Grains"); return; }
  char reload[4096];
  if (gdem_reload_filename(g_sys, reload, sizeof(reload)) != GDEM_OK) { fail("Init_Grains"); return; }
  if (!reload[0]) {
    std::fprintf(stderr, "Grains3D B200 coupling: Init_Grains: the XML has no Construction/Reload"
                         " file (particle insertion is not part of this library)\n");
    g_error = true;
    return;
  }
  // AllComponents::read_particles (:1152-1164): the reload name up to its
  // first '.', then "_Particles" and ".result" (GrainsExec::
  // fullResultFileName, Base/src/GrainsExec.cpp:708-716), with ".bin" after
  // it in the Hybrid reading mode
  std::string pfile(reload);
  const size_t dot = pfile.find_first_of('.');
  if (dot != std::string::npos) pfile.erase(dot);
  pfile += "_Particles.result";
  // GrainsCoupledWithFluid::Construction (Fluid/src/GrainsCoupledWithFluid.
  // cpp:238-420) takes the contact force models from the reload, as printed
  // in its material-contact file, and never reads the XML's
  // <ContactForceModels>
  // (a particle file without such a header, as this library's
  // gdem_write_reload_particles writes, keeps the XML's models)
  const std::string header = headerWithContactModels(reload);
  if (!header.empty() && gdem_read_reload_contact_models(g_sys, header.c_str()) != GDEM_OK) {
    fail("Init_Grains");
    return;
  }
  bool hybrid = false;
  if (!readReloadMode(reload, hybrid)) {
    // no reload header beside the particle file: the binary particle file
    // alone means the Hybrid mode
    FILE* ft = std::fopen(pfile.c_str(), "r");
    FILE* fb = ft ? nullptr : std::fopen((pfile + ".bin").c_str(), "rb");
    hybrid = fb != nullptr;
    if (ft) std::fclose(ft);
    if (fb) std::fclose(fb);
  }
  const int rc = hybrid ? gdem_read_reload_particles_hybrid(g_sys, (pfile + ".bin").c_str())
                        : gdem_read_reload_particles(g_sys, pfile.c_str());
  if (rc != GDEM_OK) { fail("Init_Grains"); return; }
  g_n = gdem_num_particles(g_sys);
  if (!readIds()) { fail("Init_Grains"); return; }
  // The reference's particles of a reload keep a coupling factor of 1 with
  // either value of b_fluidcorrectedacc: Particle::read2014 (Component/src/
  // Particle.cpp:984-1023) gives them a new kinematics object (factor 1) and
  // the buoyant weight, and Init_Grains resets the factors
  // (GrainsCoupledWithFluid::setFluidCorrectedAcceleration,
  // setParticlesCouplingFactor) only when b_fluidcorrectedacc is false.  The
  // particles here all come from the reload, so they get the same: the
  // buoyant weight, no corrected acceleration.
  (void)b_fluidcorrectedacc;
  if (gdem_set_fluid(g_sys, fluid_rho, 0) != GDEM_OK) {
    fail("Init_Grains");
    return;
  }
  if (gdem_time_step_bounds(g_sys, &g_min_dt, &g_max_dt, &g_ndt) != GDEM_OK) {
    fail("Init_Grains");
    return;
  }
  char raw[4096];
  if (gdem_rawdata_spec(g_sys, raw, sizeof(raw), &g_raw_binary) != GDEM_OK) {
    fail("Init_Grains");
    return;
  }
  g_raw_root = raw;
  std::printf("Construction of Grains completed\n");
}

void Simu_Grains(const double dt_fluid) {
  if (!g_sys || g_error) return;
  // GrainsCoupledWithFluid::Simulation (:127-132)
  const double dteff = std::max(std::min(g_max_dt, dt_fluid / double(g_ndt)), g_min_dt);
  g_ndt = (int)(size_t)(dt_fluid / dteff);
  if (g_ndt < 1) g_ndt = 1;
  const double dt = dt_fluid / double(g_ndt);
  if (gdem_set_time_step(g_sys, dt) != GDEM_OK) {
    fail("Simu_Grains");
    return;
  }
  // with a RawData writer, the last sub-step records its contacts so that
  // SaveResults_Grains can write the coordination numbers
  const bool record = !g_raw_root.empty();
  if (gdem_step(g_sys, record ? g_ndt - 1 : g_ndt) != GDEM_OK ||
      (record && (gdem_set_diagnostics(g_sys, 1) != GDEM_OK || gdem_step(g_sys, 1) != GDEM_OK ||
                  gdem_set_diagnostics(g_sys, 0) != GDEM_OK))) {
    fail("Simu_Grains");
    return;
  }
  g_time += dt_fluid;
  int bits = 0;
  gdem_status(g_sys, &bits, 0);
  if (bits) {
    std::fprintf(stderr, "Grains3D B200 coupling: Simu_Grains: simulation status %#x\n", bits);
    g_error = true;
  }
}

char* GrainsToBasilisk(int* pstrsize) {
  // the stream is built with snprintf: tokens joined by one space, as the
  // reference's interface re-joins them (InterfaceGrains3DBasilisk.cpp:62-82)
  std::string out;
  auto tok = [&](const std::string& t) { out += t; out += ' '; };
  char buf[64];
  const int64_t n = g_sys && !g_error ? g_n : 0;
  std::vector<double> x(3 * n), v(3 * n), w(3 * n), q(4 * n), B(9 * n);
  // the classes' envelopes (Convex::getNbCorners / getEnvelope / getFaces)
  struct Env { int code = 0; std::vector<double> pts; std::vector<int> faces; int nfaces = 0; };
  std::vector<Env> env;
  bool all_spheres = true;
  for (int c = 0; n && !g_error; ++c) {
    Env e;
    int np = 0, nw = 0;
    if (gdem_class_envelope(g_sys, c, &e.code, 0, &np, nullptr, 0, &nw, &e.nfaces, nullptr) != GDEM_OK)
      break;   // past the last class
    e.pts.resize(3 * (size_t)np);
    e.faces.resize((size_t)nw);
    if (gdem_class_envelope(g_sys, c, &e.code, np, &np, e.pts.data(), nw, &nw, &e.nfaces,
                            e.faces.data()) != GDEM_OK) {
      fail("GrainsToBasilisk");
      break;
    }
    if (e.code != 1) all_spheres = false;
    env.push_back(std::move(e));
  }
  if (n && !g_error) {
    if (gdem_download_state(g_sys, x.data(), v.data(), w.data(), nullptr, q.data(), nullptr,
                            nullptr) != GDEM_OK)
      fail("GrainsToBasilisk");
    // the transform's basis: integrated with the rotation (the reference's
    // composeLeftByRotation) where the system keeps orientation matrices,
    // else the matrix of the quaternion
    if (!all_spheres) {
      if (gdem_download_basis(g_sys, B.data()) != GDEM_OK) fail("GrainsToBasilisk");
    } else {
      for (int64_t i = 0; i < n; ++i) rotationOf(&q[4 * i], &B[9 * i]);
    }
  }
  std::snprintf(buf, sizeof(buf), "%lld", (long long)n);
  tok(buf);
  for (int64_t i = 0; i < n && !g_error; ++i) {
    double props[7];
    int shape = 0;
    if (gdem_particle_class(g_sys, g_class[i], props, &shape) != GDEM_OK) { fail("GrainsToBasilisk"); break; }
    if (g_class[i] < 0 || g_class[i] >= (int)env.size()) { fail("GrainsToBasilisk"); break; }
    Env const& e = env[g_class[i]];
    const double* mr = &B[9 * i];
    // Particle::computeInertiaTensorSpaceFixed (Particle.cpp:1797-1821):
    // Mr (I_body Mr^t), I_body diagonal in the body frame
    const double ib[9] = {props[2], 0., 0., 0., props[3], 0., 0., 0., props[4]};
    const double mrt[9] = {mr[0], mr[3], mr[6], mr[1], mr[4], mr[7], mr[2], mr[5], mr[8]};
    double tmp[9], is[9];
    matmul(ib, mrt, tmp);
    matmul(mr, tmp, is);
    const double inertia[6] = {is[0], is[1], is[2], is[4], is[5], is[8]};
    // GrainsToFluid (:950-1030): ID - 1, corners (1 for a sphere), "P",
    // v, w, density, mass, space-fixed inertia, orientation, centre
    std::snprintf(buf, sizeof(buf), "%d", g_ids[i] - 1);
    tok(buf);
    std::snprintf(buf, sizeof(buf), "%d", e.code);
    tok(buf);
    tok("P");
    for (int d = 0; d < 3; ++d) tok(d16(v[3 * i + d]));
    for (int d = 0; d < 3; ++d) tok(d16(w[3 * i + d]));
    tok(d16(props[1]));
    tok(d16(props[0]));
    for (double c : inertia) tok(d16(c));
    for (int k = 0; k < 9; ++k) tok(d16(mr[k]));
    for (int d = 0; d < 3; ++d) tok(d16(x[3 * i + d]));
    // radius in the stream's default format (%g), then RigidBody::
    // writePositionInFluid (RigidBody.cpp:445-500): the envelope points
    // through the particle's transform (Transform::operator(), Transform.cpp:
    // 309-314: basis row . p + origin), then the faces (count, indices) or 0
    std::snprintf(buf, sizeof(buf), "%g", props[5]);
    tok(buf);
    const int np = (int)e.pts.size() / 3;
    std::snprintf(buf, sizeof(buf), "%d", np);
    tok(buf);
    for (int k = 0; k < np; ++k) {
      const double* pt = &e.pts[3 * (size_t)k];
      for (int d = 0; d < 3; ++d)
        tok(d16(mr[3 * d] * pt[0] + mr[3 * d + 1] * pt[1] + mr[3 * d + 2] * pt[2] + x[3 * i + d]));
    }
    std::snprintf(buf, sizeof(buf), "%d", e.nfaces);
    tok(buf);
    for (int w = 0; w < (int)e.faces.size(); ++w) {
      std::snprintf(buf, sizeof(buf), "%d", e.faces[w]);
      tok(buf);
    }
  }
  *pstrsize = (int)out.size() + 1;
  char* res = new char[*pstrsize];
  std::memcpy(res, out.c_str(), out.size() + 1);
  return res;
}

void SetInitialTime(double tinit) { g_time = tinit; }

void SaveResults_Grains() {
  // GrainsCoupledWithFluid::InitialPostProcessing at the first call,
  // doPostProcessing after (:870-893): the XML's RawData writer, if any, and
  // a Format2024 particle file of the current state
  if (!g_sys || g_error) return;
  if (!g_raw_root.empty()) {
    const int rc = g_raw_started ? gdem_rawdata_write(g_sys, g_time)
                                 : gdem_rawdata_start(g_sys, g_raw_root.c_str(), g_raw_binary,
                                                      g_restart ? 1 : 0, g_time);
    if (rc != GDEM_OK) { fail("SaveResults_Grains"); return; }
    g_raw_started = true;
  }
  char name[64];
  std::snprintf(name, sizeof(name), "grains_b200_%06d_Particles", g_cycle++);
  if (gdem_write_reload_particles(g_sys, name) != GDEM_OK) fail("SaveResults_Grains");
}

void checkParaviewPostProcessing_Grains(char* solid_resDir) { (void)solid_resDir; }

void UpdateVelocityGrains(double** arrayv, const int m) {
  if (!g_sys || g_error) return;
  if (m != g_n) {
    std::fprintf(stderr, "WARNING: numbers of particles in Grains and in the fluid solver are "
                         "different in UpdateVelocityGrains\n");
    if (m < g_n) return;
  }
  // the particles' current velocities: a particle whose row is missing keeps
  // its own
  std::vector<double> v(3 * g_n), w(3 * g_n);
  if (gdem_download_state(g_sys, nullptr, v.data(), w.data(), nullptr, nullptr, nullptr,
                          nullptr) != GDEM_OK) {
    fail("UpdateVelocityGrains");
    return;
  }
  int64_t missing = 0;
  for (int64_t i = 0; i < g_n; ++i) {
    // row i belongs to the particle of ID i + 1 (GrainsCoupledWithFluid.cpp:1150);
    // an ID beyond the m rows the fluid sent has no row
    const int row_index = g_ids[i] - 1;
    if (row_index < 0 || row_index >= m) { ++missing; continue; }
    const double* row = arrayv[row_index];
    for (int d = 0; d < 3; ++d) { v[3 * i + d] = row[d]; w[3 * i + d] = row[3 + d]; }
  }
  if (missing)
    std::fprintf(stderr, "WARNING: UpdateVelocityGrains: %lld particles have an ID beyond the %d "
                         "rows of the fluid solver and keep their velocities\n",
                 (long long)missing, m);
  if (gdem_set_velocities(g_sys, v.data(), w.data()) != GDEM_OK) fail("UpdateVelocityGrains");
}

void SetInitialCycleNumber(int cycle0) { g_cycle = cycle0; }

void NumberOfRigidBodiesInBasilisk(size_t* nparticles, size_t* nobstacles) {
  *nparticles = (size_t)(g_sys && !g_error ? g_n : 0);
  *nobstacles = 0;   // no obstacle of these XMLs is sent to the fluid
}

}  // extern "C"
