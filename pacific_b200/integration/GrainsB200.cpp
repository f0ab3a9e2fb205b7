// GrainsB200.cpp -- see GrainsB200.hh.  Compiled against the Grains3D
// headers (GRAINS_V1/Grains/*/include) and linked with libgrains_b200.so.
#include "GrainsB200.hh"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <tuple>

#include "GrainsExec.hh"
#include "Obstacle.hh"
#include "Particle.hh"
#include "SimpleObstacle.hh"

using namespace std;

namespace {

void fail(char const* where) {
  cerr << "GrainsB200: " << where << ": " << gdem_last_error() << endl;
}

}  // namespace

GrainsB200::GrainsB200() : Grains(), m_dev(nullptr), m_convex(false), m_insert_counter(0) {}

GrainsB200::~GrainsB200() {
  if (m_dev) gdem_destroy(m_dev);
}

// Grains::do_before_time_stepping (Base/src/Grains.cpp:95-173) builds the
// system and inserts the particles on the host; they then go to the device,
// in particle-ID order, where the leapfrog starts (gdem_init: forces at t0,
// cumulative contact memory zeroed, as the reference's start).
void GrainsB200::do_before_time_stepping(DOMElement* rootElement) {
  Grains::do_before_time_stepping(rootElement);
  if (!m_processorIsActive || m_nprocs != 1) {
    cerr << "GrainsB200: one process only" << endl;
    m_error_occured = true;
    return;
  }
  char const* prec = getenv("GRAINS_B200_PRECISION");
  const int mode = (prec && strcmp(prec, "fp32split") == 0) ? GDEM_FP32_SPLIT : GDEM_FP64;
  if (gdem_create(GrainsExec::m_inputFile.c_str(), mode, &m_dev) != GDEM_OK) {
    fail("gdem_create");
    m_dev = nullptr;
    m_error_occured = true;
    return;
  }
  // the particles (periodic clones stay on the host: the device uses the
  // minimum image)
  map<int, Particle*> byId;
  for (Particle* p : *m_allcomponents.getActiveParticles())
    if (p->getTag() != 2) byId[p->getID()] = p;
  m_byIndex.clear();
  for (auto const& e : byId) m_byIndex.push_back(e.second);
  const size_t n = m_byIndex.size();
  // (arrays of at least one entry: an over-time insertion may start empty)
  vector<int> type(max<size_t>(n, 1));
  vector<double> x(3 * max<size_t>(n, 1)), v(x.size()), w(x.size()), q(4 * max<size_t>(n, 1)),
      basis(9 * max<size_t>(n, 1));
  m_convex = false;
  for (Particle const* r : *m_allcomponents.getReferenceParticles())
    if (r->getRigidBody()->getConvex()->getConvexType() != SPHERE) m_convex = true;
  for (size_t i = 0; i < n; ++i) {
    Particle* p = m_byIndex[i];
    type[i] = p->getGeometricType();
    Point3 const* c = p->getPosition();
    Vector3 const* vt = p->getTranslationalVelocity();
    Vector3 const* om = p->getAngularVelocity();
    Quaternion const* qr = p->getQuaternionRotation();
    Matrix const& b = p->getRigidBody()->getTransform()->getBasis();
    for (int d = 0; d < 3; ++d) {
      x[3 * i + d] = (*c)[d];
      v[3 * i + d] = (*vt)[d];
      w[3 * i + d] = (*om)[d];
      for (int k = 0; k < 3; ++k) basis[9 * i + 3 * d + k] = b[d][k];
    }
    q[4 * i] = (*qr)[X];
    q[4 * i + 1] = (*qr)[Y];
    q[4 * i + 2] = (*qr)[Z];
    q[4 * i + 3] = (*qr)[W];
    if (p->getRigidBody()->getConvex()->getConvexType() != SPHERE) m_convex = true;
  }
  const size_t waiting =
      m_insertion_mode == IM_OVERTIME ? m_allcomponents.getNumberPhysicalParticlesToInsert() : 0;
  if ((waiting && gdem_reserve(m_dev, (int64_t)waiting) != GDEM_OK) ||
      gdem_upload_state(m_dev, (int64_t)n, nullptr, type.data(), x.data(), v.data(), w.data(),
                        nullptr, q.data()) != GDEM_OK ||
      (m_convex && gdem_upload_basis(m_dev, basis.data()) != GDEM_OK) ||
      gdem_set_time_step(m_dev, m_dt) != GDEM_OK || gdem_init(m_dev) != GDEM_OK) {
    fail("device set-up");
    m_error_occured = true;
  }
}

// Grains::insertParticle (Base/src/Grains.cpp:2063-2139) during the run: the
// particle to insert, its position (the list of positions, else a random
// point of a random window), its angular position and its velocities come
// from the reference's own members in the reference's order (so the random
// draws are the same); LinkedCell::insertParticleSerial's overlap test and
// the insertion are gdem_insert_particle.  The attempt counter and the
// bookkeeping of the position lists are the reference's.
bool GrainsB200::insertParticle(PullMode const& mode) {
  if (!m_dev) return Grains::insertParticle(mode);
  bool insert = true;
  const size_t npositions = m_insertion_position->size();
  const size_t nangpositions = m_insertion_angular_position->size();
  if (m_insert_counter == 0) {
    Particle* particle = m_allcomponents.getParticleToInsert(mode);
    if (particle) {
      particle->setPosition(getInsertionPoint());
      if (m_init_angpos != IAP_FIXED) {
        Transform trot;
        if (m_init_angpos == IAP_RANDOM) {
          trot.setBasis(GrainsExec::RandomRotationMatrix(m_dimension));
        } else {
          m_il_sap = m_insertion_angular_position->begin();
          trot.setBasis(*m_il_sap);
        }
        particle->composePositionRightByTransform(trot);
      }
      Vector3 vtrans, vrot;
      computeInitVit(vtrans, vrot);
      particle->setTranslationalVelocity(vtrans);
      particle->setAngularVelocity(vrot);
      particle->initialize_transformWithCrust_to_notComputed();
      Quaternion qrot;
      qrot.setQuaternion(particle->getRigidBody()->getTransform()->getBasis());
      particle->setQuaternionRotation(qrot);
      double x[3], v[3], w[3], q[4] = {qrot[X], qrot[Y], qrot[Z], qrot[W]}, basis[9];
      Matrix const& b = particle->getRigidBody()->getTransform()->getBasis();
      for (int d = 0; d < 3; ++d) {
        x[d] = (*particle->getPosition())[d];
        v[d] = vtrans[d];
        w[d] = vrot[d];
        for (int k = 0; k < 3; ++k) basis[3 * d + k] = b[d][k];
      }
      int inserted = 0, id = -1;
      if (gdem_insert_particle(m_dev, particle->getGeometricType(), x, v, w, q, basis,
                               m_force_insertion ? 1 : 0,
                               GrainsExec::m_InsertionWithBVonly ? 1 : 0, particle->getID(),
                               &inserted, &id) != GDEM_OK) {
        fail("gdem_insert_particle");
        m_error_occured = true;
        inserted = 0;
      }
      insert = inserted != 0;
      if (insert) {
        m_allcomponents.WaitToActive();
        particle->InitializeForce(true);
        m_byIndex.push_back(particle);   // device particle index id
        if (npositions) {
          if (m_insertion_order == PM_RANDOM)
            (*m_insertion_position)[m_i_sp] = m_insertion_position->back();
          m_insertion_position->pop_back();
          if (m_insertion_position->size() < size_t(0.5 * double(m_insertion_position->capacity())))
            m_insertion_position->shrink_to_fit();
        }
        if (nangpositions) m_insertion_angular_position->erase(m_il_sap);
      }
    }
  }
  ++m_insert_counter;
  if (m_insert_counter == m_insertion_frequency) m_insert_counter = 0;
  return insert || m_force_insertion;
}

bool GrainsB200::checkStatus() {
  int bits = 0;
  if (gdem_status(m_dev, &bits, 0) != GDEM_OK) {
    fail("gdem_status");
    return true;
  }
  if (!bits) return false;
  cout << endl << "GrainsB200: the device step stopped: "
       << ((bits & GDEM_ST_CONTACT_OVERLAP) ? "ContactError (max overlap exceeded) " : "")
       << ((bits & GDEM_ST_MOTION) ? "MotionError (motion over one step exceeds the crust) " : "")
       << ((bits & GDEM_ST_OUT_OF_GRID) ? "SimulationError (particle out of the linked cell) " : "")
       << ((bits & ~(GDEM_ST_CONTACT_OVERLAP | GDEM_ST_MOTION | GDEM_ST_OUT_OF_GRID))
               ? "status bits " + to_string(bits)
               : string())
       << endl;
  return true;
}

void GrainsB200::downloadToParticles(bool contacts) {
  const size_t n = m_byIndex.size();
  vector<double> x(3 * n), v(3 * n), w(3 * n), q(4 * n), F(3 * n), T(3 * n), basis(9 * n);
  if (gdem_download_state(m_dev, x.data(), v.data(), w.data(), nullptr, q.data(), F.data(),
                          T.data()) != GDEM_OK ||
      (m_convex && gdem_download_basis(m_dev, basis.data()) != GDEM_OK)) {
    fail("gdem_download_state");
    return;
  }
  for (size_t i = 0; i < n; ++i) {
    Particle* p = m_byIndex[i];
    if (m_convex) {
      double m[12];
      for (int k = 0; k < 9; ++k) m[k] = basis[9 * i + k];
      for (int d = 0; d < 3; ++d) m[9 + d] = x[3 * i + d];
      p->setTransform(Transform(m));
    } else {
      p->setPosition(Point3(x[3 * i], x[3 * i + 1], x[3 * i + 2]));
    }
    p->setTranslationalVelocity(Vector3(v[3 * i], v[3 * i + 1], v[3 * i + 2]));
    p->setAngularVelocity(Vector3(w[3 * i], w[3 * i + 1], w[3 * i + 2]));
    p->setQuaternionRotation(Quaternion(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]));
  }
  if (contacts) {
    // the contacting components of the last evaluation (Particle::
    // addContactingComponentID, as Particle::InterAction records them)
    vector<int> obstacleId;
    for (SimpleObstacle* o : m_allcomponents.getObstacles()->getObstacles())
      obstacleId.push_back(o->getID());
    for (size_t i = 0; i < n; ++i) m_byIndex[i]->InitializeForce(false);
    int64_t cnt = 0;
    if (gdem_download_contacts(m_dev, 0, &cnt, nullptr, nullptr, nullptr, nullptr) == GDEM_OK) {
      vector<int> id0(cnt), id1(cnt);
      vector<double> dl(cnt);
      if (gdem_download_contacts(m_dev, cnt, &cnt, id0.data(), id1.data(), dl.data(), nullptr) ==
          GDEM_OK) {
        for (int64_t c = 0; c < cnt; ++c) {
          Particle* a = m_byIndex[id0[c]];
          if (id1[c] >= 0) {
            Particle* b = m_byIndex[id1[c]];
            a->addContactingComponentID(b->getID());
            b->addContactingComponentID(a->getID());
          } else {
            const int k = -id1[c] - 2;
            if (k < (int)obstacleId.size()) a->addContactingComponentID(obstacleId[k]);
          }
        }
      }
    }
    // contact memory (Component::m_contactMap: key (1, partner ID, 1) for
    // simple particles, obstacles by their negative IDs)
    int64_t nh = 0;
    if (gdem_download_history(m_dev, 0, &nh, nullptr, nullptr, nullptr, nullptr, nullptr) ==
        GDEM_OK) {
      vector<int> own(nh), par(nh);
      vector<double> kd(3 * nh), pn(3 * nh), sp(3 * nh);
      if (gdem_download_history(m_dev, nh, &nh, own.data(), par.data(), kd.data(), pn.data(),
                                sp.data()) == GDEM_OK) {
        vector<map<tuple<int, int, int>, tuple<bool, Vector3, Vector3, Vector3>>> maps(n);
        for (int64_t e = 0; e < nh; ++e) {
          const int partner = par[e] >= 0 ? m_byIndex[par[e]]->getID()
                                          : (-par[e] - 2 < (int)obstacleId.size()
                                                 ? obstacleId[-par[e] - 2]
                                                 : par[e]);
          maps[own[e]][make_tuple(1, partner, 1)] = make_tuple(
              true, Vector3(kd[3 * e], kd[3 * e + 1], kd[3 * e + 2]),
              Vector3(pn[3 * e], pn[3 * e + 1], pn[3 * e + 2]),
              Vector3(sp[3 * e], sp[3 * e + 1], sp[3 * e + 2]));
        }
        // Component::setContactMap (Component/src/Component.cpp:1017) merges;
        // the pairs that separated since the last download are dropped first
        // by flagging every entry false and erasing the false ones
        // (Component.cpp:567-593), the reference's own per-step pruning.
        for (size_t i = 0; i < n; ++i) {
          m_byIndex[i]->setContactMapToFalse();
          m_byIndex[i]->updateContactMap();
          m_byIndex[i]->setContactMap(maps[i]);
        }
      }
    }
  }
  // the force and torque of the last evaluation (after InitializeForce)
  for (size_t i = 0; i < n; ++i) {
    m_byIndex[i]->setForce(Vector3(F[3 * i], F[3 * i + 1], F[3 * i + 2]));
    m_byIndex[i]->setTorque(Vector3(T[3 * i], T[3 * i + 1], T[3 * i + 2]));
  }
}

// The time loop of Grains::Simulation (Base/src/Grains.cpp:286-451) with the
// steps between two output times on the device: the same time counter and
// output schedule, the steps up to an output time (or the end) in one
// gdem_step call, the last of them recording its contacts; at an output time
// the reference's outputs from the downloaded state.  Over-time insertion
// runs at the start of a step, before its move, as in the reference: the
// steps before an insertion attempt are run first.
void GrainsB200::Simulation(double) {
  if (!m_dev || m_error_occured) return;
  double vmax = 0., vmean = 0.;
  int pending = 0;
  while (m_tend - m_time > 0.01 * m_dt) {
    m_time += m_dt;
    GrainsExec::m_time_counter++;
    bool output = false;
    if (m_timeSave != m_save.end() && *m_timeSave - m_time < 0.01 * m_dt) {
      output = true;
      m_timeSave++;
    }
    m_insertion_windows.Move(m_time, m_dt);
    if (m_insertion_mode == IM_OVERTIME) {
      if (m_insert_counter == 0 && m_allcomponents.getNumberPhysicalParticlesToInsert() &&
          pending) {
        if (gdem_step(m_dev, pending) != GDEM_OK) {
          fail("gdem_step");
          m_error_occured = true;
          break;
        }
        pending = 0;
        if (checkStatus()) {
          m_error_occured = true;
          break;
        }
      }
      insertParticle(m_insertion_order);
      m_allcomponents.computeNumberParticles(m_wrapper);
      if (m_error_occured) break;
    }
    ++pending;
    if (!output && m_tend - m_time > 0.01 * m_dt) continue;
    int rc = GDEM_OK;
    if (output) {
      if (pending > 1) rc = gdem_step(m_dev, pending - 1);
      if (rc == GDEM_OK) rc = gdem_set_diagnostics(m_dev, 1);
      if (rc == GDEM_OK) rc = gdem_step(m_dev, 1);
      if (rc == GDEM_OK) rc = gdem_set_diagnostics(m_dev, 0);
    } else {
      rc = gdem_step(m_dev, pending);
    }
    pending = 0;
    if (rc != GDEM_OK) {
      fail("gdem_step");
      m_error_occured = true;
      break;
    }
    if (checkStatus()) {
      m_error_occured = true;
      break;
    }
    if (!output) continue;
    cout << '\r' << m_time << "  \t" << m_tend << flush;
    GrainsExec::m_output_data_at_this_time = true;
    downloadToParticles(true);
    m_allcomponents.ComputeMaxMeanVelocity(vmax, vmean, m_wrapper);
    cout << endl << "Component velocity : max = " << vmax << " average = " << vmean << endl;
    fVitMax << GrainsExec::doubleToString(ios::scientific, 6, m_time) << "\t"
            << GrainsExec::doubleToString(ios::scientific, 6, vmax) << "\t"
            << GrainsExec::doubleToString(ios::scientific, 6, vmean) << endl;
    saveReload(m_time);
    m_allcomponents.PostProcessing(m_time, m_dt, m_collision, m_insertion_windows);
    GrainsExec::m_output_data_at_this_time = false;
  }
}

void GrainsB200::do_after_time_stepping() {
  if (m_dev) downloadToParticles(false);
  Grains::do_after_time_stepping();
}
