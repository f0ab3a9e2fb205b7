// GrainsB200.hh -- a Grains3D application whose DEM time loop runs on a B200
// through libgrains_b200 (include/grains_b200.h).
//
// The class is the drop-in a Grains3D build adds: an input file with
// <Grains3D Type="B200"> runs the reference's own driver (GRAINS_V1/Main/src/
// main.cpp: GrainsBuilderFactory::create, do_before_time_stepping,
// Simulation, do_after_time_stepping) with this application in place of the
// serial Grains one.  Construction, insertion, the output schedule and every
// writer stay the reference's; only the steps between two output times run on
// the device:
//
//   do_before_time_stepping  Grains::do_before_time_stepping (XML, insertion
//                            at the initial time, first post-processing
//                            output), then the particles go to the device
//                            (gdem_create on the same input file, gdem_reserve
//                            for the particles still waiting, gdem_upload_state,
//                            gdem_upload_basis) and the leapfrog starts there
//                            (gdem_init);
//   Simulation               the reference's output schedule (m_save): the steps
//                            up to the next output time (or insertion attempt)
//                            in one gdem_step call, the last one with the
//                            contact diagnostics on; at an output time the
//                            device state, forces and contacts come back into
//                            the particles and the reference's own outputs run
//                            (velocity max/mean line, reload, post-processing
//                            writers);
//   insertParticle           insertion over time (Grains::insertParticle): the
//                            reference picks the particle, its position,
//                            orientation and velocities as usual; the overlap
//                            test and the insertion run on the device
//                            (gdem_insert_particle);
//   do_after_time_stepping   the final state back into the particles, then
//                            Grains::do_after_time_stepping.
//
// Precision: FP64 unless the environment sets GRAINS_B200_PRECISION=fp32split.
// Not covered: moving obstacles, MPI.  An inserted
// polyhedron's overlap test starts its GJK searches from the current support
// vertices without moving them (the reference's moves them).
#ifndef _GRAINSB200_HH_
#define _GRAINSB200_HH_

#include <vector>

#include "Grains.hh"
#include "grains_b200.h"

class GrainsB200 : public Grains {
 public:
  GrainsB200();
  ~GrainsB200();

  void do_before_time_stepping(DOMElement* rootElement);
  void Simulation(double time_interval = 0.);
  void do_after_time_stepping();

 protected:
  // One insertion attempt every m_insertion_frequency calls, as the
  // reference's; before the device is set up (insertion at the initial
  // time), the reference's own.
  bool insertParticle(PullMode const& mode);
  // The device's status bits as the reference's exceptions would have ended
  // the run (ContactError, MotionError, SimulationError); true on an error.
  bool checkStatus();
  // Device state (positions and orientations, velocities, angular velocities,
  // quaternions, forces, torques) back into the particles; with contacts, the
  // contacting-component sets of the last evaluation (coordination numbers).
  void downloadToParticles(bool contacts);

  gdem_handle m_dev;
  std::vector<Particle*> m_byIndex;   // device particle index -> particle
  bool m_convex;
  size_t m_insert_counter;            // Grains::insertParticle's attempt counter
};

#endif
