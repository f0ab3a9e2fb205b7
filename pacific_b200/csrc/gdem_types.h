// gdem_types.h -- plain-old-data descriptors shared by the host runtime and
// the sm_100a kernels of the Grains3D DEM step.
#pragma once
#include <stdint.h>

namespace gdem {

// Most entries of one particle's row of the pair list (an entry's position
// in its row is kept in 16 bits).
constexpr int kRowMax = 65535;
// Material indices per instance (materials are bits in the reference,
// ContactBuilderFactory.cpp:176-192; here they are indices 0..kMaxMat-1).
constexpr int kMaxMat = 8;

// Error bits reported through the device status word.  They replace the
// reference's C++ exceptions (Base/include/Error.hh): ContactError,
// MotionError, SimulationError; plus the capacity checks of this runtime.
enum StatusBits : int {
  kErrContactOverlap = 1 << 0,   // overlap >= sum of crusts (ContactError)
  kErrMotion = 1 << 1,           // |dx| > crust over one step (MotionError)
  kErrOutOfGrid = 1 << 2,        // particle outside the linked-cell grid (SimulationError)
  kErrHashFull = 1 << 3,         // contact-history table has no free slot
  kErrGjkMaxIter = 1 << 4,       // GJK hit its iteration cap
  kErrTimeout = 1 << 5,          // a bounded device wait gave up
  kErrPairsFull = 1 << 6,        // the pair list outgrew its allocation (or a row kRowMax)
};

// Words of the device control block (DevState::ctl).
enum CtlWords : int {
  kCtlNeed = 0,     // set by the step kernels: a particle moved more than skin / 2
  kCtlActive = 1,   // this step rebuilds the pair list (set by k_decide)
  kCtlEpoch = 2,    // force evaluations so far (tags the contact-history keys)
  kCtlRebuilds = 3, // pair-list rebuilds so far
  kCtlWork = 4,     // particles near a wall this evaluation (contact filter)
  kCtlPairs = 5,    // pairs of the compact pair list (set by the rebuild)
  kCtlKept = 6,     // pairs kept by this evaluation's contact filter
  kCtlEntries = 7,  // pair-list entries of the last rebuild
  kCtlEntriesMax = 8,  // most entries any rebuild needed since the last allocation check
  kCtlKeptCold = 9,  // kept pairs not in contact at the last evaluation (listed from the back)
  kCtlKept2 = 10,    // of those, the pairs the first search iteration left undecided (kept2)
  kCtlWords = 16
};

// One independent simulation ("instance").  A single Grains3D system is a
// batch of one.  Cell numbering follows LinkedCell::getCellNumber
// (Base/src/LinkedCell.cpp:1165-1168): j * nbk * nbi + k * nbi + i.
struct GridDesc {
  double lc_origin[3];   // linked-cell origin (shifted by one cell where periodic)
  double edge[3];        // cell edge lengths
  double L[3];           // domain size: the periodic translation vector
  int nb[3];             // cells per direction (incl. the 2 periodic layers)
  int periodic[3];
  int cell_offset;       // first global cell key of this instance
  int wall_begin, wall_count;
  int model_base;        // first entry of this instance in the model table
  int pad0;
  float edge_f[3];       // edge in FP32 (FP32-split broad phase)
  float skin_f;          // pair-list skin in FP32
  float filt_margin;     // absolute margin of the FP32 contact filter (covers rounding)
  float Lf[3];           // domain size in FP32
  float pad_f;
  double skin;           // pair-list skin: pairs closer than the sum of radii + skin are listed
  double safe_lo[3], safe_hi[3];  // coordinates strictly inside these need no wrap or grid check
};

// Particle class (a <Particle> node of the XML input).
struct TypeDesc {
  double radius;         // circumscribed radius
  double crust;          // crust thickness
  double mass;
  double inertia[3];     // body-fixed principal inertia (inertia[0], [3], [5] of the reference)
  double eqrad;          // Component::getEquivalentSphereRadius
  double weight[3];      // m (1 - rho_f / rho) g
  int mat;               // material index
  int shape;             // 0 sphere, 1 box, 2 polyhedron, 3 cylinder
  float r_f;             // radius in FP32 (FP32-split broad phase)
  int pad_r;
  double extent[3];      // box half lengths / bounding-box half extent;
                         // cylinder (radius, half height, radius)
  double scaling[3];     // crust shrink factors (extent - crust) / extent
  int poly_begin;        // first vertex of a polyhedron in the vertex table
  int poly_count;        // its vertex count
  int poly_start;        // the current vertex of a new particle (Polyhedron::BuildPolyhedron:
                         // the first vertex with a neighbour)
  int pad_p;
  double inv_mass;       // 1 / (mass c) and 1 / inertia (FP32-split leapfrog)
  double inv_inertia[3];
  double density;
  // coupling factor c (ParticleKinematics::setCouplingFactor,
  // ParticleKinematics.cpp:483-488): 1 - rho_f / rho in a coupled run with
  // fluid-corrected acceleration, else 1; the kicks divide by m c and c I
  double coupling;
  double inv_inertia_c[3];   // 1 / (c inertia) (FP32-split leapfrog)
};

// HookeMemory / Hooke parameters (HookeMemoryContactForceModel.cpp:12-27).
struct ModelDesc {
  double kn, en, etat, muc, kt, mur, etarpf, epst;
  double beta;           // ln(en) / sqrt(pi^2 + ln^2(en))
  double kr;             // Hooke rolling-resistance coefficient
  int rolling;           // HookeMemory: mur != 0; Hooke: kr != 0
  int memory;            // 1 HookeMemory, 0 Hooke (no tangential history)
  int valid;
  int pad;
};

// Axis-aligned box obstacle (SimpleObstacle with a Box convex).
struct WallDesc {
  double centre[3];
  double extent[3];      // half lengths
  double crust;
  double eqrad;
  double radius;         // circumscribed radius |extent|
  double scaling[3];     // crust shrink factors
  int mat;
  int id;                // obstacle index within its instance
};

}  // namespace gdem
