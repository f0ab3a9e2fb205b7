/* grains_b200.h -- C ABI of the B200-native Grains3D DEM time step.
 *
 * The reference (PacIFiC / Grains3D, GRAINS_V1/Grains) exposes its DEM step
 * through C++ virtuals and one C ABI for the Basilisk coupling.  The entry
 * points below replace, for the DEM step only:
 *   - Grains::Construction / do_before_time_stepping
 *       (Base/src/Grains.cpp:95-173, 535-1030)            -> gdem_create
 *   - Grains reload of particle state (Format2024 reload:
 *       Grains.cpp:784-845, AllComponents.cpp:1024-1290)  -> gdem_upload_*
 *   - the leapfrog initial force evaluation
 *       (Grains.cpp:168-173)                              -> gdem_init
 *   - Grains::Simulation time loop, leapfrog branch
 *       (Grains.cpp:271-452, 344-364)                     -> gdem_step
 *   - particle state / contact output (Particle::write2014, Particle.cpp:
 *       1167-1176; RawDataPostProcessingWriter)            -> gdem_download_*
 *   - ContactError / MotionError / SimulationError exceptions
 *       (Base/include/Error.hh:19-151)                    -> status bits
 * Ownership: device memory belongs to the handle; host arrays belong to the
 * caller and are not retained.  One host thread per handle.  Every call
 * returns GDEM_OK (0) or a negative error; gdem_last_error() describes it.
 */
#ifndef GRAINS_B200_H
#define GRAINS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gdem_system* gdem_handle;

/* precision modes */
#define GDEM_FP64 0        /* all contact arithmetic in FP64 (reference order) */
#define GDEM_FP32_SPLIT 1  /* FP32 cell-relative pair search, FP64 contact geometry,
                              FP32 force law (FP64 when ill-conditioned), FP64 leapfrog */

/* return codes */
#define GDEM_OK 0
#define GDEM_ERR_INVALID (-1)   /* bad argument or XML */
#define GDEM_ERR_CUDA (-2)      /* CUDA runtime error */
#define GDEM_ERR_STATE (-3)     /* call out of sequence */

/* simulation status bits (gdem_status): the reference's exceptions */
#define GDEM_ST_CONTACT_OVERLAP 0x01  /* overlap >= crustA + crustB (ContactError) */
#define GDEM_ST_MOTION 0x02           /* |dx| > crust in one step (MotionError) */
#define GDEM_ST_OUT_OF_GRID 0x04      /* particle left the linked cell (SimulationError) */
#define GDEM_ST_HASH_FULL 0x08        /* contact-history table full */
#define GDEM_ST_GJK_MAXITER 0x10      /* GJK iteration cap reached */
#define GDEM_ST_TIMEOUT 0x20          /* a bounded device wait gave up */
#define GDEM_ST_PAIRS_FULL 0x40       /* the pair list's allocation was too small at a rebuild (rows emptied; grown before the next call) */

/* Builds a system from a Grains3D XML input (Construction: LinkedCell,
 * Origin, Periodicity, Particles, Obstacles, ContactForceModels; Forces:
 * Gravity; Simulation: TimeStep).  Replaces Grains::Construction
 * (Base/src/Grains.cpp:535-1030) for the DEM step. */
int gdem_create(const char* xml_path, int precision, gdem_handle* out);

/* Same, for n independent instances stepped together (one XML each).
 * Particle IDs are global: instance k owns IDs [base_k, base_k + n_k). */
int gdem_create_batch(int n, const char* const* xml_paths, int precision, gdem_handle* out);

/* Sets the particles (replaces the insertion / reload of particle state,
 * Grains.cpp:784-845).  Arrays are indexed by particle ID (0..n-1); inst
 * may be NULL for a single instance; type is the index of the <Particle>
 * class within its instance.  x, v, w (space-fixed angular velocity) are
 * 3 per particle, q is (qx, qy, qz, qw).  wbf (body-fixed angular velocity)
 * may be NULL: it is then derived as q* w q (ParticleKinematics.cpp:220). */
int gdem_upload_state(gdem_handle h, int64_t n, const int* inst, const int* type,
                      const double* x, const double* v, const double* w,
                      const double* wbf, const double* q);

/* Force and torque of the last evaluation (the Format2024 reload carries
 * them, SecondOrderLeapFrog.cpp:102-109); marks the leapfrog as started. */
int gdem_upload_forces(gdem_handle h, const double* F, const double* T);

/* Room for `extra` particles inserted after the upload (gdem_insert_particle):
 * the particle buffers are sized for n + extra when the state is uploaded.
 * Call before gdem_upload_state.  Replaces the reference's waiting particles
 * (AllComponents::m_WaitParticles, activated by Grains::insertParticle,
 * Base/src/Grains.cpp:2063-2139). */
int gdem_reserve(gdem_handle h, int64_t extra);

/* One insertion attempt (Grains::insertParticle with
 * LinkedCell::insertParticleSerial, Base/src/LinkedCell.cpp:1765-1840): a
 * particle of class `type` at position x, velocity v, space-fixed angular
 * velocity w, quaternion q (qx, qy, qz, qw) and, when basis is not NULL, that
 * orientation matrix (row-major; otherwise the matrix of q).  Unless force,
 * it is inserted only when it touches no particle (at its periodic images
 * within one period where the domain is periodic) and no wall, as
 * RigidBodyWithCrust::isContact (Geometry/src/RigidBodyWithCrust.cpp:
 * 840-958) decides: two spheres when their centres are closer than the sum
 * of their radii, a sphere and a box when the sphere overlaps the box,
 * other shapes when their circumscribed spheres overlap and -- unless bv_only
 * (GeometricOverlap Value="BV") -- the GJK distance of the shrunk bodies is
 * below the sum of the crusts minus 1e-10.  On insertion *inserted = 1 and
 * *id (may be NULL) = its particle ID (the particle count before the call);
 * its force is its weight and its torque zero (Particle::InitializeForce),
 * and the next gdem_step starts its leapfrog with the others'.  ref_id: its
 * ID in reload files written later (<= 0: its particle ID + 1).  Single
 * systems, between gdem_step calls; needs room from gdem_reserve.  A
 * polyhedron's GJK search starts from the particle's and the candidate's
 * current vertices and moves neither. */
int gdem_insert_particle(gdem_handle h, int type, const double* x, const double* v,
                         const double* w, const double* q, const double* basis, int force,
                         int bv_only, int ref_id, int* inserted, int* id);

/* Replaces the whole particle state of an uploaded system (same particle
 * count) without allocating: x, v, w, q (and optionally wbf) by particle ID
 * from caller memory (pinned memory gives full-speed copies).  With F and T
 * the leapfrog continues from them (a reload, Grains.cpp:784-845); without
 * them gdem_init must run before the next step.  Contact memory is kept. */
int gdem_set_state(gdem_handle h, const double* x, const double* v, const double* w,
                   const double* wbf, const double* q, const double* F, const double* T);

/* Orientation matrices of non-spherical particles (the basis of
 * RigidBody::m_transform, Geometry/src/Transform.cpp; Particle::
 * setAngularPosition), row-major, 9 per particle, by particle ID.  Without
 * this call they are built from q as Matrix::setRotation does
 * (Geometry/src/Matrix.cpp:114-127); gdem_set_state rebuilds them the same
 * way.  Allowed only right after gdem_upload_state or gdem_set_state.  For a
 * spheres-only system it does nothing. */
int gdem_upload_basis(gdem_handle h, const double* basis);

/* Current orientation matrices by particle ID (9 each, row-major); the
 * identity for a spheres-only system. */
int gdem_download_basis(gdem_handle h, double* basis);

/* The polyhedron support search's current vertex of every particle, by
 * particle ID (Polyhedron::m_curr_vertex, Geometry/src/Polyhedron.cpp:
 * 265-293: the search climbs the vertex graph from it and, among vertices
 * tied within 1e-16, stays where it is, so it decides the witness points of
 * face contacts).  A particle's vertex after an evaluation is the one its
 * last GJK call in row order left (its wall calls come last).  A new or
 * reloaded particle starts at the first vertex with a neighbour, as the
 * reference's does; 0 for other shapes.  Upload after gdem_upload_state. */
int gdem_upload_support_vertices(gdem_handle h, const int* vertex);
int gdem_download_support_vertices(gdem_handle h, int* vertex);

/* Maximum and mean translational speed over the particles
 * (AllComponents::ComputeMaxMeanVelocity, Component/src/AllComponents.cpp:
 * 1781-1811), the quantity Grains3D writes to *_VelocityMaxMean.dat. */
int gdem_velocity_stats(gdem_handle h, double* vmax, double* vmean);

/* Force evaluations and pair-list rebuilds since the state was created.
 * The pair list holds every pair whose bounding spheres are closer than the
 * skin; it is rebuilt (counting sort into cell order + 27-cell search) only
 * before an evaluation at which some particle has moved more than half the
 * skin since the last rebuild. */
int gdem_step_counts(gdem_handle h, int64_t* evaluations, int64_t* rebuilds);

/* FP32-split mode: contact-law evaluations since the last reset (each pair
 * in contact once per force evaluation, walls once per particle), and how
 * many of them were re-evaluated in FP64 because the FP32 force was
 * ill-conditioned (a small difference of large terms).  Zero in FP64 mode. */
int gdem_law_counts(gdem_handle h, int64_t* evaluated, int64_t* reevaluated, int reset);

/* Systems with convex bodies: GJK closest-point calls of the force kernels
 * since the last reset (each pair and each particle-wall pair whose bounding
 * spheres overlap, once per force evaluation), their
 * iterations, and the most iterations of one call (the reference stops at
 * 1000, Convex.cpp:536-627).  No counterpart in the reference. */
int gdem_gjk_counts(gdem_handle h, int64_t* calls, int64_t* iterations, int64_t* max_iterations,
                    int reset);

/* Contact features over the evaluations since the state was created (or the
 * last reset), as Grains3D prints them at the end of a run (Grains.cpp:
 * 228-244, AppCollision::addToContactsFeatures, Base/src/AppCollision.cpp:
 * 159-179): the largest and the mean |overlap| over the contacts (each pair
 * and each particle-wall contact once per force evaluation), the evaluation
 * at which the largest was first reached (0 is the leapfrog start at t0,
 * k the evaluation at t0 + k dt; -1 without contact) and the mean GJK
 * iterations per GJK call (0 for spheres only).  Accumulated on the device;
 * the mean's last bits depend on the order of the warps' additions.  Any
 * pointer may be NULL. */
int gdem_contact_features(gdem_handle h, double* overlap_max, double* overlap_mean,
                          int64_t* evaluation_of_max, double* gjk_iterations_mean, int reset);

/* Per-kernel device timing with CUDA events (replaces the SCT_* phase timers,
 * Base/include/solvercomputingtime.hh:46-75).  While on, gdem_step uses plain
 * launches instead of graph replay.  gdem_kernel_times returns, per timed
 * phase, its name (32 chars each), total milliseconds and launch count. */
int gdem_set_profiling(gdem_handle h, int on);
int gdem_kernel_times(gdem_handle h, int capacity, int* count, char* names, double* total_ms,
                      int64_t* launches);

/* Contact memory entries (Component::m_contactMap, Component.cpp:776-801):
 * owner particle ID, partner ID (>= 0 particle, -(k+2) wall k of the
 * owner's instance), kdelta, previous normal, spring torque (3 each). */
int gdem_upload_history(gdem_handle h, int64_t n, const int* owner, const int* partner,
                        const double* kdelta, const double* prevn, const double* spring);
/* The contact memory of the last force evaluation in the same layout, both
 * views of a pair (the second body's is the negation), ordered by owner then
 * partner: *count receives the entry count; the arrays are filled when
 * capacity >= *count (spring may be NULL). */
int gdem_download_history(gdem_handle h, int64_t capacity, int64_t* count, int* owner,
                          int* partner, double* kdelta, double* prevn, double* spring);

/* Launch tuning, before gdem_init.  No counterpart in the reference (its
 * LinkedCell has a cell size only, Grains.cpp:1005-1022).  skin_factor is
 * the pair-list skin as a multiple of each instance's largest circumscribed
 * radius (it sets the pair-list cell size, 2 rmax f + skin, and how often the
 * list is rebuilt; < 0 restores the LinkedCell Skin attribute or 0.25);
 * blocks_per_sm is the force kernels' persistent grid, in blocks per
 * multiprocessor (<= 0: 4).  Results do not depend on either. */
int gdem_set_tuning(gdem_handle h, double skin_factor, int blocks_per_sm);

/* Autotuner, before gdem_init: steps copies of the uploaded system for
 * trial_steps steps per candidate (skin factors 0.1, 0.175, 0.25, 0.4, 0.6,
 * then 2, 4 or 8 blocks per multiprocessor at the best skin), applies the
 * fastest with gdem_set_tuning and returns it with its device time per step.
 * Needs device memory for one more copy of the system. */
int gdem_autotune(gdem_handle h, int trial_steps, double* skin_factor, int* blocks_per_sm,
                  double* ms_per_step);

/* Leapfrog start (Grains.cpp:168-173): forces at t0, then zero the
 * cumulative tangential and rolling memories. */
int gdem_init(gdem_handle h);

/* ---- fluid coupling (GrainsCoupledWithFluid, Fluid/src/
 * GrainsCoupledWithFluid.cpp; the Basilisk C ABI of
 * libgrains_b200_basilisk.so is built on these) ---- */

/* Fluid density: the weight becomes m (1 - rho_f / rho) g
 * (Particle::computeWeight, Particle.cpp:413-418) and, with
 * corrected_acceleration, the kicks divide by m c and c I with the coupling
 * factor c = 1 - rho_f / rho (ParticleKinematics::setCouplingFactor,
 * ParticleKinematics.cpp:483-488). */
int gdem_set_fluid(gdem_handle h, double fluid_density, int corrected_acceleration);

/* Time step of the next steps (the coupled run's sub-step,
 * GrainsCoupledWithFluid::Simulation, :123-133). */
int gdem_set_time_step(gdem_handle h, double dt);

/* TimeStep mindt, maxdt, ndt of a coupled run's XML (a plain run's dt for
 * both bounds and 1). */
int gdem_time_step_bounds(gdem_handle h, double* min_dt, double* max_dt, int* ndt);

/* The Construction/Reload Filename attribute ("" without one). */
int gdem_reload_filename(gdem_handle h, char* buf, int capacity);

/* Class cls (of the first instance): props = mass, density, principal
 * inertia (3), circumscribed radius, crust thickness; shape 0 sphere, 1 box,
 * 2 polyhedron, 3 cylinder. */
int gdem_particle_class(gdem_handle h, int cls, double* props, int* shape);

/* The envelope of class cls (of the first instance) as GrainsCoupledWithFluid::
 * GrainsToFluid writes it (Fluid/src/GrainsCoupledWithFluid.cpp:912-1120,
 * RigidBody::writePositionInFluid, Geometry/src/RigidBody.cpp:445-500):
 * *code = Convex::getNbCorners (1 sphere, 666 box, 777 cylinder, a
 * polyhedron's vertex count); *npoints body-frame points of the shape without
 * its crust shrink (Convex::getEnvelope: the sphere's centre, the box's eight
 * corners in Box::setCornersFaces's order, the cylinder's bottom centre,
 * bottom rim point and top centre, the polyhedron's vertices in file order),
 * 3 doubles each in points; the faces (Convex::getFaces; none for a sphere or
 * a cylinder): *nfaces runs of (vertex count, vertex indices) in faces,
 * *nwords ints in all.  points / faces are filled when their capacities
 * (points, ints) suffice; the sizes are always returned. */
int gdem_class_envelope(gdem_handle h, int cls, int* code, int point_capacity, int* npoints,
                        double* points, int word_capacity, int* nwords, int* nfaces, int* faces);

/* Velocities and space-frame angular velocities from the fluid solver, by
 * particle ID, 3 each (GrainsCoupledWithFluid::updateParticlesVelocity,
 * :1126-1180; the body-frame angular velocity follows as q* w q). */
int gdem_set_velocities(gdem_handle h, const double* v, const double* w);

/* Hydrodynamic force and torque by particle ID (3 each), added to every
 * particle's force and torque at each step until replaced (the PRSHydroFT
 * application, GrainsCoupledWithFluid::updateParticlesHydroFT, :1187-1193);
 * both NULL clears them. */
int gdem_set_hydro_forces(gdem_handle h, const double* F, const double* T);

/* Advances nsteps kick-drift-kick leapfrog steps of size dt (from the XML).
 * Equivalent to the loop body of Grains::Simulation (Grains.cpp:286-364).
 * Per step: a contact filter over the pair list, the force kernel over the
 * particles in contact, and the leapfrog kernel (closing kick, next opening
 * kick and drift); the pair list is rebuilt only when needed
 * (gdem_step_counts), inside a CUDA-graph conditional node. */
int gdem_step(gdem_handle h, int nsteps);

/* State by particle ID; any pointer may be NULL. */
int gdem_download_state(gdem_handle h, double* x, double* v, double* w, double* wbf,
                        double* q, double* F, double* T);

/* Format2024 reload, particle file: the "<reload>_Particles" text file that
 * AllComponents::write writes and AllComponents::read_particles reads
 * (Component/src/AllComponents.cpp:1299-1420, 1136-1290), one line per
 * particle as Particle::write2014 (Particle.cpp:1167-1176): class, ID, tag,
 * activity, position and orientation matrix (Transform::writeTransform2014),
 * velocity, quaternion (w, x, y, z), angular velocity, force, torque
 * (SecondOrderLeapFrog.cpp:102-109) and the contact memory
 * (Component::writeContactMemory2014, Component.cpp:776-801).  IDs are the
 * reference's (1-based); an obstacle partner is -(k + 1) for wall k.  One
 * system (not a batch).  gdem_write_reload_particles writes the state after
 * the last step (tags written 0, activity 1); gdem_read_reload_particles
 * loads such a file into a created system without particles (it replaces
 * gdem_upload_state + gdem_upload_basis + gdem_upload_forces +
 * gdem_upload_history: the leapfrog continues from the stored forces,
 * without gdem_init); periodic clones (tag 2) and inactive particles are
 * skipped.  When the XML's Construction/Reload has Velocity="Reset", the
 * loaded velocities are zero and the quaternions the identity
 * (AllComponents::resetKinematics, AllComponents.cpp:762-771). */
int gdem_write_reload_particles(gdem_handle h, const char* path);
int gdem_read_reload_particles(gdem_handle h, const char* path);
/* The same particle file in the hybrid (binary) form of a Format2024 reload
 * (the "<reload>_Particles.bin" file: per particle its record's byte count
 * as a size_t, then the Particle::write2014_binary record, Component/src/
 * Particle.cpp:1183-1193, in host byte order; AllComponents::write :1387-1404
 * and read_particles :1163-1256). */
int gdem_write_reload_particles_hybrid(gdem_handle h, const char* path);
int gdem_read_reload_particles_hybrid(gdem_handle h, const char* path);

/* Cell (i, j, k) of every particle, in Cell::GetCell numbering
 * (Base/src/Cell.cpp:172-184), by particle ID. */
int gdem_download_cells(gdem_handle h, int* ijk);

/* Records overlaps during force evaluation (needed by gdem_download_contacts). */
int gdem_set_diagnostics(gdem_handle h, int on);

/* Contacts (overlap < 0) of the last force evaluation: *count receives the
 * number of contacts; when capacity >= *count the arrays are filled with
 * (id0 < id1) pairs, their overlap distance and (force may be NULL) the
 * contact force exerted on id0, 3 per contact (the per-contact record of
 * AppCollision / PostProcessingWriter force output); walls appear as
 * id1 = -(k+2), with the force on the particle. */
int gdem_download_contacts(gdem_handle h, int64_t capacity, int64_t* count, int* id0,
                           int* id1, double* delta, double* force);

/* Coordination number of every particle, by ID: the partners and walls it
 * touched (negative overlap) in the last force evaluation, counted on the
 * device from that evaluation's diagnostics records (Particle::
 * getCoordinationNumber, Component/src/Particle.cpp:1398-1401, set by
 * addContactingComponentID, :1702-1706).  All zero before the first
 * evaluation after a state upload; an error when the last evaluation ran
 * without diagnostics.  gdem_download_classes gives each particle's class
 * (Particle::getGeometricType, Particle.cpp:1651-1654). */
int gdem_download_coordination(gdem_handle h, int* coord);
int gdem_download_classes(gdem_handle h, int* cls);
/* Reference particle IDs (Component::getID, 1-based) by particle index: the
 * IDs of the Format2024 particle file the state was read from, else
 * index + 1. */
int gdem_download_ids(gdem_handle h, int* ids);

/* RawData post-processing output of a system
 * (PostProcessing/src/RawDataPostProcessingWriter.cpp): per output time, a
 * line (text) or record (binary) in <root>_position_{x,y,z}.dat,
 * _translational_velocity_{x,y,z}.dat, _angular_velocity_{x,y,z}.dat and
 * _coordinationNumber.dat, and <root>_particleType.dat rewritten, particle
 * ID i in column i + 1 (reference IDs 1..n).  gdem_rawdata_start opens the
 * files (append = 0 truncates them, as a "new" run; 1 appends, as a reload
 * of type "same") and writes the first output time (PostProcessing_start,
 * :55-78); gdem_rawdata_write adds one (one_output_Standard, :374-600);
 * gdem_rawdata_end closes them (PostProcessing_end, :123-141).  The
 * coordination numbers are gdem_download_coordination's, so the step before
 * an output time runs with diagnostics on (a start before gdem_init writes
 * zeros, as the reference's PostProcessing_start does).  The reference's
 * file quirks are kept: the coordination file carries no time in text mode,
 * and in binary mode _angular_velocity_z.dat receives the time twice. */
int gdem_rawdata_start(gdem_handle h, const char* root, int binary, int append, double time);
int gdem_rawdata_write(gdem_handle h, double time);
int gdem_rawdata_end(gdem_handle h);

/* One line "time<TAB>vmax<TAB>vmean" of <root>_VelocityMaxMean.dat
 * (Grains::Simulation, Base/src/Grains.cpp:401-408), from the device
 * reduction of gdem_velocity_stats; append = 0 truncates the file first
 * (Grains::do_before_time_stepping opens it anew, Grains.cpp:137-145). */
int gdem_write_velocity_max_mean(gdem_handle h, const char* path, int append, double time);

/* The XML's RawData writer (<Simulation><PostProcessing><Writers><RawData
 * Name=".." WritingMode="Text|Binary"/>, PostProcessingWriterBuilderFactory.cpp
 * :19-20): its root name ("" when the XML has none) and binary flag. */
int gdem_rawdata_spec(gdem_handle h, char* root, int capacity, int* binary);

/* OR of the status bits raised since creation (or the last reset). */
int gdem_status(gdem_handle h, int* bits, int reset);

/* Linked-cell grid of instance k: cells per direction, edge, origin. */
int gdem_grid(gdem_handle h, int k, int* nb, double* edge, double* origin);

/* Sizes of the last force evaluation: directed pair-list entries (each
 * candidate pair appears once per partner) and live contact-memory entries
 * (active contacts, particle-particle and particle-wall). */
int gdem_pair_counts(gdem_handle h, int64_t* entries, int64_t* contacts);

/* Instances of a system (1 unless made by gdem_create_batch), or
 * GDEM_ERR_INVALID for a null handle. */
int gdem_num_instances(gdem_handle h);

/* Particle count and device time of the last gdem_step in ms. */
int64_t gdem_num_particles(gdem_handle h);
double gdem_last_step_ms(gdem_handle h);

/* Runs gdem_step's loop as captured CUDA graphs (1) or plain launches (0). */
int gdem_use_graphs(gdem_handle h, int on);

/* Contact memory of contacts that have ended: dropped at the next force
 * evaluation (prune = 1, the default: Grains::computeParticlesForceAndTorque,
 * Base/src/Grains.cpp:459-482, with Component::setContactMapToFalse /
 * updateContactMap) or kept, so that a pair that touches again resumes its
 * tangential spring (prune = 0: GrainsCoupledWithFluid::Simulation,
 * Fluid/src/GrainsCoupledWithFluid.cpp:123-228, which never prunes).  Set it
 * before the particles are uploaded or read; with prune = 0 the history
 * tables are four times larger, and a run that fills them raises
 * GDEM_ST_HASH_FULL. */
int gdem_set_contact_memory_pruning(gdem_handle h, int prune);

/* The contact force models of a Format2024 reload, in place of the XML's:
 * header is the reload file ("<name>.result"), whose "<ContactForceModels>
 * <file> </ContactForceModels>" line names the material-contact file that
 * ContactBuilderFactory::save wrote beside it; that file (looked for in the
 * header's directory) gives each material pair's model and parameters as
 * printed there (ContactBuilderFactory::reload, Component/src/
 * ContactBuilderFactory.cpp:199-262).  GrainsCoupledWithFluid::Construction
 * (Fluid/src/GrainsCoupledWithFluid.cpp:238-420) takes its models from there
 * only, so a coupled run reloads them this way.  One system (not a batch). */
int gdem_read_reload_contact_models(gdem_handle h, const char* header);

const char* gdem_last_error(void);
void gdem_destroy(gdem_handle h);

/* ---------------------------------------------------------------- adjoint
 * Calibration gradients (the reference has no differentiation).  The
 * adjoint engine integrates spheres in a walled box with the same leapfrog
 * and Hooke / HookeMemory law as gdem_step (FP64, no rolling resistance, no
 * periodic directions) and differentiates the loss
 *     L = sum_i |x_i(nsteps) - target_x_i|^2 + |v_i(nsteps) - target_v_i|^2
 * with respect to params = (kn, en, muc) (replacing those of every contact
 * model of the XML) and the initial velocities, by a reverse sweep over the
 * steps with the transposed leapfrog and contact-force Jacobians, recomputing
 * states from checkpoints taken every checkpoint_every steps. */
typedef struct gdem_adjoint* gdem_adjoint_handle;
int gdem_adjoint_create(const char* xml_path, gdem_adjoint_handle* out);
/* Particles by index: class, x0, v0 (3 each), w0 (3 each; NULL: zero). */
int gdem_adjoint_set_particles(gdem_adjoint_handle h, int64_t n, const int* type,
                               const double* x0, const double* v0, const double* w0);
/* Forward run, loss and gradients; every output pointer may be NULL (no
 * gradient pointer: forward only; no target: no loss). */
int gdem_adjoint_run(gdem_adjoint_handle h, int nsteps, int checkpoint_every,
                     const double* params, const double* target_x, const double* target_v,
                     double* loss, double* x_out, double* v_out, double* dL_dparams,
                     double* dL_dv0);
/* The same loss differentiated in forward mode, to check the adjoint: with
 * seed_particle < 0 the dual numbers are seeded on (kn, en, muc) and
 * dL_dseed receives 3 values; otherwise on the initial velocity component
 * (seed_particle, seed_component) and dL_dseed receives 1 value. */
int gdem_adjoint_forward_dual(gdem_adjoint_handle h, int nsteps, const double* params,
                              const double* target_x, const double* target_v,
                              int seed_particle, int seed_component, double* loss,
                              double* dL_dseed);
void gdem_adjoint_destroy(gdem_adjoint_handle h);

/* No counterpart in the reference.  Maximum and mean |v| (as
 * gdem_velocity_stats, AllComponents::ComputeMaxMeanVelocity) of n particle
 * velocities v (device memory, 3 doubles per particle), written to out
 * (device memory, 2 doubles: max, mean) in stream order on stream (a
 * cudaStream_t; NULL for the default stream).  Needs no handle and allocates
 * nothing: the reduction's scratch is a fixed device array of the library,
 * so n is limited to 1,048,576 (larger n returns GDEM_ERR_INVALID).  Calls
 * that overlap in time on one device race on that scratch.  The first call on
 * a device sets up the scratch address and should come before any stream
 * capture; the set-up is repeated when the device's context has changed
 * since (after a cudaDeviceReset). */
int gdem_speed_stats_static(const double* v, int64_t n, double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GRAINS_B200_H */
