// ref_harness.cpp -- drives the unmodified Grains3D reference (serial,
// Type="Standard") from a given particle state, one leapfrog step at a time.
// TEST INFRASTRUCTURE ONLY: it is built into oracle/_ref/ by
// oracle/build_ref.sh, from the reference sources and the MPI / Xerces
// stand-ins under oracle/shim/, and is used to pin the CPU restatement
// (grains_oracle.cpp) and to produce the golden vectors in tests/golden/.
//
// The sequence below is the one of Grains::do_before_time_stepping and
// Grains::Simulation (Base/src/Grains.cpp:95-173, 286-364), minus file
// output: Construction + Forces read the XML; particles are inserted with
// the calls Grains::insertParticle makes (Grains.cpp:2070-2130:
// getParticleToInsert, setPosition, setTranslationalVelocity,
// setAngularVelocity, setQuaternionRotation, insertParticleSerial,
// WaitToActive, InitializeForce); the leapfrog start is
// computeParticlesForceAndTorque + setAllContactMapCumulativeFeaturesToZero;
// a step is moveParticlesAndObstacles(dt/2, dt, dt),
// computeParticlesForceAndTorque, advanceParticlesVelocity(dt/2).
#include <cstdio>
#include <exception>
#include <fstream>
#include <map>
#include <vector>

#include "Cell.hh"
#include "ContactBuilderFactory.hh"
#include "Error.hh"
#include "Grains.hh"
#include "GrainsBuilderFactory.hh"
#include "GrainsExec.hh"
#include "LinkedCell.hh"
#include "Obstacle.hh"
#include "Particle.hh"
#include "RawDataPostProcessingWriter.hh"
#include "ReaderXML.hh"
#include "SimpleObstacle.hh"

namespace {

class RefGrains : public Grains {
 public:
  std::map<int, int> id_to_index;     // reference component ID -> caller index
  std::map<int, int> obstacle_index;  // obstacle ID -> wall index (XML order)
  std::vector<Particle*> by_index;

  void setup(DOMElement* root) {
    Construction(root);
    Forces(root);
    DOMNode* simu = ReaderXML::getNode(root, "Simulation");
    DOMNode* ts = ReaderXML::getNode(simu, "TimeStep");
    m_dt = ReaderXML::getNodeAttr_Double(ts, "dt");
    m_time = 0.;
    // phase timers that the step functions start and stop (Grains.cpp:277-282)
    SCT_insert_app("ParticlesInsertion");
    SCT_insert_app("ComputeForces");
    SCT_insert_app("Move");
    SCT_insert_app("UpdateParticleActivity");
    SCT_insert_app("LinkUpdate");
    SCT_insert_app("OutputResults");
    std::list<SimpleObstacle*> obs = m_allcomponents.getObstacles()->getObstacles();
    int k = 0;
    for (SimpleObstacle* o : obs) obstacle_index[o->getID()] = k++;
  }

  int insert(int n, const int* type, const double* x, const double* v, const double* w,
             const double* q) {
    by_index.assign(n, nullptr);
    for (int i = 0; i < n; ++i) {
      Particle* p = m_allcomponents.getParticleToInsert(type[i]);
      p->setPosition(Point3(x[3 * i], x[3 * i + 1], x[3 * i + 2]));
      // orientation as Grains::insertParticle applies a random rotation:
      // basis = basis o R(q), then the quaternion is rebuilt from the basis
      Quaternion qq(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]);
      if (!(q[4 * i] == 0. && q[4 * i + 1] == 0. && q[4 * i + 2] == 0.)) {
        Matrix R;
        R.setRotation(qq);
        Transform trot;
        trot.setBasis(R);
        p->composePositionRightByTransform(trot);
        qq.setQuaternion(p->getRigidBody()->getTransform()->getBasis());
      }
      p->setTranslationalVelocity(Vector3(v[3 * i], v[3 * i + 1], v[3 * i + 2]));
      p->setQuaternionRotation(qq);
      p->setAngularVelocity(Vector3(w[3 * i], w[3 * i + 1], w[3 * i + 2]));
      p->initialize_transformWithCrust_to_notComputed();
      bool ok = m_collision->insertParticleSerial(p, m_allcomponents.getActiveParticles(),
                                                  m_allcomponents.getPeriodicCloneParticles(),
                                                  m_allcomponents.getReferenceParticles(),
                                                  m_periodic, true);
      if (!ok) return 1;
      m_allcomponents.WaitToActive();
      p->InitializeForce(true);
      id_to_index[p->getID()] = i;
      by_index[i] = p;
    }
    m_allcomponents.computeNumberParticles(m_wrapper);
    return 0;
  }

  int init() {
    try {
      computeParticlesForceAndTorque();
      m_allcomponents.setAllContactMapCumulativeFeaturesToZero();
    } catch (ContactError&) { return 1; }
    catch (MotionError&) { return 2; }
    catch (SimulationError&) { return 4; }
    return 0;
  }

  int step(int nsteps) {
    try {
      for (int k = 0; k < nsteps; ++k) {
        m_time += m_dt;
        GrainsExec::m_time_counter++;
        moveParticlesAndObstacles(0.5 * m_dt, m_dt, m_dt);
        computeParticlesForceAndTorque();
        m_allcomponents.advanceParticlesVelocity(m_time, 0.5 * m_dt);
      }
    } catch (ContactError&) { return 1; }
    catch (MotionError&) { return 2; }
    catch (SimulationError&) { return 4; }
    return 0;
  }

  // The master of each ID (periodic clones carry their master's ID and tag 2).
  std::vector<Particle*> masters() {
    std::vector<Particle*> out(by_index.size(), nullptr);
    for (Particle* p : *m_allcomponents.getActiveParticles()) {
      if (p->getTag() == 2) continue;
      auto it = id_to_index.find(p->getID());
      if (it != id_to_index.end()) out[it->second] = p;
    }
    return out;
  }

  // A particle state read from a Format2024 particle file with the
  // reference's own reload path (Grains::Construction, Grains.cpp:1024-1026:
  // AllComponents::read_particles; Grains::InsertCreateNewParticles,
  // :1970-1976: AllComponents::Link and, when periodic, checkClonesReload).
  // The particles keep the forces and contact memory of the file, so the
  // next step continues the leapfrog from there (a reload: no force
  // initialisation).  Particle ID i + 1 is caller index i.
  int load(const char* stem, int npart) {
    m_allcomponents.read_particles(stem, (size_t)npart, m_collision, 0, 1, nullptr);
    m_allcomponents.Link(*m_collision);
    if (m_periodic) checkClonesReload();
    m_allcomponents.computeNumberParticles(m_wrapper);
    by_index.assign(npart, nullptr);
    for (Particle* p : *m_allcomponents.getActiveParticles()) {
      if (p->getTag() == 2) continue;
      const int i = p->getID() - 1;
      if (i < 0 || i >= npart) return 1;
      id_to_index[p->getID()] = i;
      by_index[i] = p;
    }
    for (Particle* p : by_index)
      if (!p) return 1;
    return 0;
  }

  void addRawData(PostProcessingWriter* w) { m_allcomponents.addPostProcessingWriter(w); }
  void postProcessing(double time, bool start) {
    if (start)
      m_allcomponents.PostProcessing_start(time, m_dt, m_collision, m_insertion_windows);
    else
      m_allcomponents.PostProcessing(time, m_dt, m_collision, m_insertion_windows);
  }
  void postProcessingEnd() { m_allcomponents.PostProcessing_end(); }
  void maxMeanVelocity(double& vmax, double& vmean) {
    m_allcomponents.ComputeMaxMeanVelocity(vmax, vmean, nullptr);
  }
  // the contact features Grains::do_after_time_stepping prints
  // (Base/src/Grains.cpp:228-244)
  void contactFeatures(double* out) {
    out[0] = m_collision->getOverlapMax();
    out[1] = m_collision->getOverlapMean();
    out[2] = m_collision->getTimeOverlapMax();
    out[3] = m_collision->getNbIterGJKMean();
  }

  int partnerIndex(int id) {
    auto it = id_to_index.find(id);
    if (it != id_to_index.end()) return it->second;
    auto jt = obstacle_index.find(id);
    if (jt != obstacle_index.end()) return -(jt->second + 2);
    return -1000000;
  }
};

}  // namespace

extern "C" {

void* ref_create(const char* xml_path) {
  static bool initialized = false;
  if (!initialized) {
    ReaderXML::initialize();
    initialized = true;
  }
  DOMElement* root = ReaderXML::getRoot(xml_path);
  if (!root) return nullptr;
  delete GrainsBuilderFactory::create(root);   // sets the 3D context
  RefGrains* g = new RefGrains();
  g->setup(root);
  return g;
}

int ref_set_particles(void* h, int n, const int* type, const double* x, const double* v,
                      const double* w, const double* q) {
  return static_cast<RefGrains*>(h)->insert(n, type, x, v, w, q);
}

int ref_init(void* h) { return static_cast<RefGrains*>(h)->init(); }
// Reads "<stem>_Particles.result" for a reload name "<stem>.<ext>" (the
// reference cuts the name at its first '.', so stem holds none), a particle
// file in the Format2024 layout.
int ref_load_particles(void* h, const char* stem, int npart) {
  try {
    return static_cast<RefGrains*>(h)->load(stem, npart);
  } catch (std::exception const& e) {
    std::fprintf(stderr, "ref_load_particles: %s\n", e.what());
    return 2;
  } catch (...) {
    std::fprintf(stderr, "ref_load_particles: exception from the reference\n");
    return 2;
  }
}
int ref_step(void* h, int nsteps) { return static_cast<RefGrains*>(h)->step(nsteps); }

void ref_get_state(void* h, double* x, double* v, double* w, double* q, double* F, double* T) {
  RefGrains* g = static_cast<RefGrains*>(h);
  std::vector<Particle*> m = g->masters();
  for (size_t i = 0; i < m.size(); ++i) {
    Particle* p = m[i];
    if (!p) continue;
    Point3 const* P = p->getPosition();
    Vector3 const* V = p->getTranslationalVelocity();
    Vector3 const* W = p->getAngularVelocity();
    Vector3 const* f = p->getForce();
    Vector3 const* t = p->getTorque();
    Quaternion const* Q = p->getQuaternionRotation();
    for (int d = 0; d < 3; ++d) {
      if (x) x[3 * i + d] = (*P)[d];
      if (v) v[3 * i + d] = (*V)[d];
      if (w) w[3 * i + d] = (*W)[d];
      if (F) F[3 * i + d] = (*f)[d];
      if (T) T[3 * i + d] = (*t)[d];
    }
    if (q) {
      Vector3 const* vq = Q->getVector3();
      q[4 * i] = (*vq)[0]; q[4 * i + 1] = (*vq)[1]; q[4 * i + 2] = (*vq)[2];
      q[4 * i + 3] = Q->getdouble();
    }
  }
}

// Rotation part of each master's transform, row-major 3x3.
void ref_get_basis(void* h, double* basis) {
  RefGrains* g = static_cast<RefGrains*>(h);
  std::vector<Particle*> m = g->masters();
  for (size_t i = 0; i < m.size(); ++i) {
    if (!m[i]) continue;
    Matrix const& B = m[i]->getRigidBody()->getTransform()->getBasis();
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) basis[9 * i + 3 * r + c] = B[r][c];
  }
}

void ref_get_cells(void* h, int* ijk) {
  RefGrains* g = static_cast<RefGrains*>(h);
  std::vector<Particle*> m = g->masters();
  for (size_t i = 0; i < m.size(); ++i)
    for (int d = 0; d < 3; ++d) ijk[3 * i + d] = m[i] ? (*m[i]->getCell())[d] : -1;
}

int ref_num_history(void* h) {
  RefGrains* g = static_cast<RefGrains*>(h);
  int n = 0;
  for (Particle* p : g->masters())
    if (p) n += (int)p->getContactMap()->size();
  return n;
}

// Contact memory of the masters: owner index, partner index (walls as
// -(k+2)), kdelta, previous normal, spring torque.
void ref_get_history(void* h, int* owner, int* partner, double* kdelta, double* prevn,
                     double* spring) {
  RefGrains* g = static_cast<RefGrains*>(h);
  std::vector<Particle*> m = g->masters();
  int n = 0;
  for (size_t i = 0; i < m.size(); ++i) {
    if (!m[i]) continue;
    for (auto const& kv : *m[i]->getContactMap()) {
      owner[n] = (int)i;
      partner[n] = g->partnerIndex(std::get<1>(kv.first));
      Vector3 const& kd = std::get<1>(kv.second);
      Vector3 const& pn = std::get<2>(kv.second);
      Vector3 const& sp = std::get<3>(kv.second);
      for (int d = 0; d < 3; ++d) {
        kdelta[3 * n + d] = kd[d]; prevn[3 * n + d] = pn[d]; spring[3 * n + d] = sp[d];
      }
      ++n;
    }
  }
}

// The particle file of a Format2024 reload, written by the reference's own
// Particle::write2014 (Component/src/Particle.cpp:1167-1176) for every
// master in particle-index order.
int ref_write_particles(void* h, const char* path) {
  RefGrains* g = static_cast<RefGrains*>(h);
  std::ofstream out(path);
  if (!out) return 1;
  for (Particle* p : g->masters())
    if (p) p->write2014(out);
  return out ? 0 : 1;
}

// The same file in the hybrid (binary) form: each master's byte count, then
// its Particle::write2014_binary record (AllComponents.cpp:1387-1404).
int ref_write_particles_hybrid(void* h, const char* path) {
  RefGrains* g = static_cast<RefGrains*>(h);
  std::ofstream out(path, std::ios::out | std::ios::binary);
  if (!out) return 1;
  for (Particle* p : g->masters())
    if (p) {
      size_t nb = p->get_numberOfBytes();
      out.write(reinterpret_cast<char*>(&nb), sizeof(size_t));
      p->write2014_binary(out);
    }
  return out ? 0 : 1;
}

// RawData output of the reference's own RawDataPostProcessingWriter
// (PostProcessing/src/RawDataPostProcessingWriter.cpp), registered as the
// one post-processing writer and driven as Grains::do_before_time_stepping
// (PostProcessing_start, Grains.cpp:131-132), Grains::Simulation
// (PostProcessing, Grains.cpp:417-418) and Grains::do_after_time_stepping
// (PostProcessing_end) drive it.  writer_xml holds one <RawData Name=...
// WritingMode=.../> element.  The reload type is set to "same" so that the
// writer appends to (creates) its files instead of running the reference's
// clearing script.
int ref_rawdata_start(void* h, const char* writer_xml, double time) {
  RefGrains* g = static_cast<RefGrains*>(h);
  DOMElement* node = ReaderXML::getRoot(writer_xml);
  if (!node) return 1;
  GrainsExec::m_ReloadType = "same";
  g->addRawData(new RawDataPostProcessingWriter(node, 0, 1, false));
  g->postProcessing(time, true);
  return 0;
}
int ref_rawdata_write(void* h, double time) {
  static_cast<RefGrains*>(h)->postProcessing(time, false);
  return 0;
}
void ref_rawdata_end(void* h) { static_cast<RefGrains*>(h)->postProcessingEnd(); }

// AllComponents::ComputeMaxMeanVelocity (Component/src/AllComponents.cpp:1781-1821),
// the figures of the _VelocityMaxMean.dat lines.
void ref_velocity_max_mean(void* h, double* vmax, double* vmean) {
  static_cast<RefGrains*>(h)->maxMeanVelocity(*vmax, *vmean);
}

// AppCollision's contact features (Base/src/AppCollision.cpp:159-179):
// maximum overlap, mean overlap, time of the maximum, mean GJK iterations;
// accumulated over every evaluation of the process (the reference keeps the
// counters in function statics).
void ref_contact_features(void* h, double* out) {
  static_cast<RefGrains*>(h)->contactFeatures(out);
}

void ref_destroy(void* h) { delete static_cast<RefGrains*>(h); }

}  // extern "C"
