// gdem_device.cuh -- device-side state and helpers for the Grains3D DEM step.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "gdem_types.h"

namespace gdem {

// Contact-history table: open addressing with linear probing, keyed on the
// unordered particle pair or on (particle, wall).  Values are stored as seen
// from the lower-ID body (or the particle, for a wall); the other body's view
// is the negation, as in the reference where p1 holds (-kdelta, -normal,
// -spring) (HookeMemoryContactForceModel.cpp:191-192).  Two tables
// alternate: the one written by force evaluation e is read by evaluation
// e + 1, so entries not touched in a step disappear, which is what
// Component::updateContactMap (Component.cpp:583-595) does.
//
// Key layout: bits 54-63 the evaluation tag (e mod 1024), bits 27-53 the
// lower particle ID, bits 0-26 the higher particle ID or, for a wall,
// 2^27 - 1 - wall index.  A slot whose tag is not the current evaluation's is
// free, so a table needs no clearing between uses; the host clears each
// table once every 512 of its uses, before a tag value can come round again.
constexpr int kTagShift = 54;
constexpr unsigned kTagMask = 1023u;
constexpr int kMaxIdBits = 27;
constexpr unsigned long long kEmptyKey = 0xFFFFFFFFFFFFFFFFull;

struct HistTable {
  unsigned long long* keys;
  void* vals;            // 9 values per slot (kdelta, prev normal, spring torque)
  int log2cap;
};

__host__ __device__ inline unsigned long long pairKey(int ida, int idb) {
  return ((unsigned long long)(uint32_t)ida << kMaxIdBits) | (uint32_t)idb;
}
__host__ __device__ inline unsigned long long wallKey(int id, int wall) {
  return ((unsigned long long)(uint32_t)id << kMaxIdBits) |
         (uint32_t)((1 << kMaxIdBits) - 1 - wall);
}
__host__ __device__ inline unsigned long long tagged(unsigned long long base, unsigned tag) {
  return ((unsigned long long)(tag & kTagMask) << kTagShift) | base;
}
__host__ __device__ inline unsigned tagOf(unsigned long long key) {
  return (unsigned)(key >> kTagShift);
}
__host__ __device__ inline uint32_t hashSlot(unsigned long long k, int log2cap) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return (uint32_t)(k & ((1ull << log2cap) - 1));
}
// Slot holding base with tag, or -1.
__device__ inline int histFind(HistTable const& t, unsigned long long base, unsigned tag) {
  const uint32_t mask = (1u << t.log2cap) - 1;
  const unsigned long long key = tagged(base, tag);
  uint32_t s = hashSlot(base, t.log2cap);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const unsigned long long k = t.keys[s];
    if (k == key) return (int)s;
    if (tagOf(k) != (tag & kTagMask)) return -1;
    s = (s + 1) & mask;
  }
  return -1;
}
// histFind after its first probe (slot first, key k0 read there) matched
// neither the key nor an empty slot: the lookup from the next slot on.
__device__ inline int histFindAfter(HistTable const& t, unsigned long long base, unsigned tag,
                                    uint32_t first) {
  const uint32_t mask = (1u << t.log2cap) - 1;
  const unsigned long long key = tagged(base, tag);
  uint32_t s = (first + 1) & mask;
  for (uint32_t probe = 1; probe <= mask; ++probe) {
    const unsigned long long k = t.keys[s];
    if (k == key) return (int)s;
    if (tagOf(k) != (tag & kTagMask)) return -1;
    s = (s + 1) & mask;
  }
  return -1;
}
// Claims a slot for base with tag (one writer per key and evaluation); -1
// when every slot carries the tag already (table full).
__device__ inline int histInsert(HistTable const& t, unsigned long long base, unsigned tag) {
  const uint32_t mask = (1u << t.log2cap) - 1;
  const unsigned long long key = tagged(base, tag);
  uint32_t s = hashSlot(base, t.log2cap);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    unsigned long long cur = t.keys[s];
    for (;;) {
      if (tagOf(cur) == (tag & kTagMask)) {
        if (cur == key) return (int)s;
        break;                                   // taken this evaluation
      }
      const unsigned long long prev = atomicCAS(&t.keys[s], cur, key);
      if (prev == cur) return (int)s;
      cur = prev;                                // raced: look again
    }
    s = (s + 1) & mask;
  }
  return -1;
}

// Overlap statistics of the contacts over the evaluations since the last
// reset (AppCollision::addToContactsFeatures, Base/src/AppCollision.cpp:
// 159-179): the sum and the count of |overlap| over the contacts (pairs and
// walls, each once per evaluation), the largest |overlap| (its FP64 bits:
// non-negative doubles order like their bit patterns) and the evaluation
// counter at which it was first reached.
struct ContactStats {
  double sum;
  unsigned long long count;
  unsigned long long max_bits;
  long long max_epoch;
};

// Whole device state of one batch of instances.  Per-particle arrays are in
// the current sorted (cell) order; component d of particle s of an n-vector
// field lives at [d * cap + s] (structure of arrays).
struct DevState {
  int n;                  // particles
  int cap;                // allocated particles (component stride)
  int ncells;             // total cell keys of all instances (pair-list grids)
  int ninst;
  double dt;
  int* id; int* type; int* inst;
  double* x; double* v; double* w; double* wbf; double* q; double* F; double* T;
  // wbf_state: w_bf is integrated (FP64 mode, or convex bodies present);
  // otherwise (FP32-split, spheres only) w is the angular state and w_bf is
  // derived on output as q* w q
  int wbf_state;
  double* basis;          // 9 per particle, non-spherical shapes only
  // second buffers: a step reads x, v, w, w_bf, q, basis and writes x2 ...;
  // a pair-list rebuild permutes everything into them and copies back
  int* id2; int* type2; int* inst2;
  double* x2; double* v2; double* w2; double* wbf2; double* q2; double* basis2;
  double* F2; double* T2;
  // pair-list validity: the FP32 position at the last rebuild (the posf
  // value written then; displacement = posf - posf0) and the periodic wraps
  // since then (signed bytes x, y, z)
  float4* posf0; int* wrap; int* wrap2;
  int* ctl;               // control words (CtlWords)
  // binning
  int* skey;              // cell key in the old order
  int* rank;              // arrival rank within the cell
  int* cell_count; int* cell_start; int* order;
  int* scan_tmp;
  // compact copies for the contact kernels (sorted order)
  double4* pos64;         // x, y, z, radius
  double4* vel64;         // v, mass
  double4* omg64;         // w (space frame), equivalent radius
  float4* offh;           // FP32 cell-relative offset; FP32 radius
  int4* cellc;            // pair-list cell i, j, k and instance at the last rebuild
  // skin pair list, compressed rows: the entries of slot t are
  // pairs[pair_off[t] .. pair_off[t] + npairs[t]), pair_off the exclusive
  // scan of npairs; pair_cap entries are allocated (kCtlEntries holds the
  // total of the last rebuild)
  int* pairs; int* npairs; int* pair_off;
  int pair_cap;
  int* pair_scan_tmp;     // tile sums of the pair-count scan
  double* hydro;          // coupled runs: hydrodynamic force and torque by particle ID (6 each), or null
  int2* upairs;           // compact pair list: (slot, entry) of every upper entry, ctl[kCtlPairs] of them
  int* epos;              // per compact pair: position of the pair in its two rows, e_t | e_u << 16
  // compact-list indices of the pairs kept by the filter: ctl[kCtlKept] from
  // the front and, in FP32-split with non-spherical classes, the pairs not in
  // contact at the last evaluation, ctl[kCtlKeptCold], from slot pair_cap / 2
  // downwards
  int* kept;
  int* kept2;             // the cold pairs k_pairsep32 left undecided, ctl[kCtlKept2]
  // per list entry: this evaluation's force and torque on the row's particle
  // from that pair (written by the pair kernel for a contact, tagged with the
  // evaluation counter), summed in row order by the leapfrog kernel
  void* share;
  void* wshare;           // per particle: the sum of its wall contacts (this evaluation)
  int* nact;              // flag words, two buffers of cap (contactFlags)
  float4* posf;           // FP32 continuous position since the last rebuild + circumscribed radius
  int* work;              // particles near a wall (this evaluation), ctl[kCtlWork]
  int nsm;                // multiprocessors of the device (persistent grids)
  int forces_bps;         // blocks per multiprocessor of the pair kernel's persistent grid (0: 4)
  double* pair_delta;     // diagnostics: overlap of each entry (+inf: no contact)
  double* wall_delta;     // diagnostics: overlap with each wall slot
  double* pair_force;     // diagnostics: contact force on the lower ID (3 per entry)
  unsigned long long* gjk_counts;   // convex: GJK calls, iterations, most iterations of a call
  unsigned long long* law_counts;   // FP32-split: contacts evaluated, re-evaluated in FP64
  ContactStats* cstats;   // overlap statistics over all evaluations
  double* wall_force;     // diagnostics: wall contact force on the particle (3 per slot)
  int diag;
  HistTable hist_old, hist_new;
  int* status;
  GridDesc const* grids;  // reference linked-cell grids (cell reports, periodic wrap)
  GridDesc const* bgrids; // pair-list grids: cells at least 2 rmax + skin wide
  TypeDesc const* types; ModelDesc const* models;
  WallDesc const* walls;
  const double* poly_verts;   // polyhedron vertices of all classes (x, y, z)
  const int* poly_adj_off;    // vertex graph of the polyhedra: per global vertex, its first neighbour
  const int* poly_adj;        // neighbours (vertex indices within their polyhedron)
  // current polyhedron vertex of each particle (Polyhedron::m_curr_vertex),
  // its permutation buffer, and the record this evaluation's GJK calls leave
  // (0: none; else priority << 16 | vertex, see recordVertex)
  int* curv; int* curv2; int* curv_next;
  int max_walls;          // walls of the largest instance
  int any_convex;         // some class is not a sphere (GJK narrow phase)
  int any_poly;           // some class is a polyhedron (carried support vertices)
  int any_walls;          // some instance has walls
  float filt_margin_max;  // largest contact-filter margin of the instances
  int filter_qblocks;     // contact filter: blocks for the pairs (0: from the particle count)
};

// ----------------------------------------------------------- FP64 helpers --
struct d3 { double x, y, z; };
__device__ __forceinline__ d3 mk(double a, double b, double c) { d3 r; r.x = a; r.y = b; r.z = c; return r; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ d3 operator-(d3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ d3 operator*(d3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ d3 operator*(double s, d3 a) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ d3 operator/(d3 a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// Vector3::operator^ (Geometry/src/Vector3.cpp:114-119)
__device__ __forceinline__ d3 cross(d3 a, d3 b) {
  return mk(a.y * b.z - a.z * b.y, -a.x * b.z + a.z * b.x, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double norm(d3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ d3 ld3(const double* p, int cap, int s) {
  return mk(p[s], p[cap + s], p[2 * cap + s]);
}
__device__ __forceinline__ void st3(double* p, int cap, int s, d3 a) {
  p[s] = a.x; p[cap + s] = a.y; p[2 * cap + s] = a.z;
}

struct dq { d3 v; double w; };
__device__ __forceinline__ dq qmk(d3 v, double w) { dq q; q.v = v; q.w = w; return q; }
__device__ __forceinline__ dq conj(dq q) { return qmk(-q.v, q.w); }
// Quaternion::operator* (Geometry/src/Quaternion.cpp:442-448)
__device__ __forceinline__ dq qmul(dq a, dq b) {
  double t = (a.w * b.w) - dot(a.v, b.v);
  d3 vt = (cross(a.v, b.v) + (a.w * b.v)) + (b.w * a.v);
  return qmk(vt, t);
}
// operator,(Vector3, Quaternion) = q.multLeftVec(lhs) (Quaternion.cpp:93-98)
__device__ __forceinline__ dq vecq(d3 l, dq q) {
  double t = dot(-l, q.v);
  d3 vt = cross(l, q.v) + (l * q.w);
  return qmk(vt, t);
}
// Quaternion::multToVector3 (Quaternion.cpp:108-113)
__device__ __forceinline__ d3 multToVector3(dq a, dq r) {
  return (cross(a.v, r.v) + (a.w * r.v)) + (r.w * a.v);
}
// Quaternion::setRotFromTwoVectors (Quaternion.cpp:263-288)
__device__ __forceinline__ dq rotFromTwoVectors(d3 u, d3 v) {
  double nn = sqrt(dot(u, u) * dot(v, v));
  double real = nn + dot(u, v);
  d3 vect;
  if (real < 1.e-6 * nn) {
    real = 0.;
    vect = fabs(u.x) > fabs(u.z) ? mk(-u.y, u.x, 0.) : mk(0., -u.z, u.y);
  } else {
    vect = cross(u, v);
  }
  double nq = sqrt(vect.x * vect.x + vect.y * vect.y + vect.z * vect.z + real * real);
  double s = 1. / nq;
  return qmk(vect * s, real * s);
}
// Quaternion::rotateVector (Quaternion.cpp:293-299)
__device__ __forceinline__ d3 rotateVector(dq q, d3 v) {
  double nv = norm(q.v);
  return ((q.w * q.w - nv * nv) * v + (2. * dot(v, q.v)) * q.v) + (2. * q.w) * cross(q.v, v);
}

__device__ __forceinline__ void raise(int* status, int bits) { atomicOr(status, bits); }

// Cell of a neighbour offset (di, dj, dk) around (i, j, k) of grid g, with
// the periodic minimum-image wrap.  Returns the global cell key or -1, and the
// image shift (in units of the period) of the particles found there.
__device__ __forceinline__ int neighbourKey(GridDesc const& g, int i, int j, int k,
                                            int di, int dj, int dk, int* sh) {
  int c[3] = {i + di, j + dj, k + dk};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    sh[d] = 0;
    if (g.periodic[d]) {
      int nin = g.nb[d] - 2;
      if (c[d] < 1) { c[d] += nin; sh[d] = -1; }
      else if (c[d] > nin) { c[d] -= nin; sh[d] = 1; }
    } else if (c[d] < 0 || c[d] >= g.nb[d]) {
      return -1;
    }
  }
  return g.cell_offset + c[1] * g.nb[2] * g.nb[0] + c[2] * g.nb[0] + c[0];
}

// Enumerates the particles of the 27 cells around cell cc (i, j, k, inst),
// row by row: for each of the 9 (dj, dk) rows the cells i-1, i, i+1 are
// consecutive in the cell numbering, so their particles are one contiguous
// slot range [cell_start[i-1], cell_start[i+2]); the cell of a candidate
// within the row follows from two boundaries.  In a periodic x direction the
// two extra layers are empty and the wrapped neighbour cell is visited
// separately.  fn(u, dcx, dj, dk, shx, shy, shz) receives the candidate slot,
// its cell offset and the periodic image shift (in periods); the centre
// particle itself is included.
template <typename Fn>
__device__ __forceinline__ void forEachCandidate(const int* __restrict__ cs, GridDesc const& g,
                                                 int4 cc, Fn&& fn) {
  const int nbx = g.nb[0];
  for (int dj = -1; dj <= 1; ++dj) {
    int jj = cc.y + dj, shy = 0;
    if (g.periodic[1]) {
      int nin = g.nb[1] - 2;
      if (jj < 1) { jj += nin; shy = -1; } else if (jj > nin) { jj -= nin; shy = 1; }
    } else if (jj < 0 || jj >= g.nb[1]) {
      continue;
    }
    for (int dk = -1; dk <= 1; ++dk) {
      int kk = cc.z + dk, shz = 0;
      if (g.periodic[2]) {
        int nin = g.nb[2] - 2;
        if (kk < 1) { kk += nin; shz = -1; } else if (kk > nin) { kk -= nin; shz = 1; }
      } else if (kk < 0 || kk >= g.nb[2]) {
        continue;
      }
      const int row = g.cell_offset + jj * g.nb[2] * nbx + kk * nbx;
      int ilo = cc.x - 1, ihi = cc.x + 1;
      if (!g.periodic[0]) { ilo = max(ilo, 0); ihi = min(ihi, nbx - 1); }
      const int b0 = cs[row + ilo], b1 = cs[row + cc.x], b2 = cs[row + cc.x + 1],
                b3 = cs[row + ihi + 1];
      for (int u = b0; u < b3; ++u) fn(u, u < b1 ? -1 : (u < b2 ? 0 : 1), dj, dk, 0, shy, shz);
      if (g.periodic[0]) {
        const int nin = nbx - 2;
        if (cc.x == 1) {
          const int e0 = cs[row + nin], e1 = cs[row + nin + 1];
          for (int u = e0; u < e1; ++u) fn(u, -1, dj, dk, -1, shy, shz);
        }
        if (cc.x == nin) {
          const int e0 = cs[row + 1], e1 = cs[row + 2];
          for (int u = e0; u < e1; ++u) fn(u, 1, dj, dk, 1, shy, shz);
        }
      }
    }
  }
}

// Orders a particle's list entries by partner ID, the partners with a
// higher ID than the particle's own (idt) first, and returns how many those
// are.  The reduction order of its forces then does not depend on the cells
// at the last rebuild (nor on when the list was rebuilt), and the contact
// filter tests each pair once, from the lower ID's "upper" entries.
__device__ __forceinline__ int sortEntriesUpperFirst(int* seg, int cnt, const int* id, int idt) {
  auto key = [&](int e) {
    const int idu = id[e & ((1 << 27) - 1)];
    return idu > idt ? idu : (1 << 30) | idu;
  };
  int nup = 0;
  for (int i = 0; i < cnt; ++i) {
    const int e = seg[i];
    const int ke = key(e);
    if (ke < (1 << 30)) ++nup;
    int j = i - 1;
    while (j >= 0 && key(seg[j]) > ke) {
      seg[j + 1] = seg[j];
      --j;
    }
    seg[j + 1] = e;
  }
  return nup;
}

// Row length of a particle with cnt candidates: at most kRowMax (an entry's
// position in its row is kept in 16 bits); more raises kErrPairsFull.
__device__ __forceinline__ int rowLength(DevState const& S, int cnt) {
  if (cnt > kRowMax) {
    raise(S.status, kErrPairsFull);
    return kRowMax;
  }
  return cnt;
}
// Whether slot t's row, placed by the scan of the row lengths, lies inside
// the allocation of the pair list; a row that does not is emptied (its
// particle then sees no partner) and kErrPairsFull raised -- the host grows
// the allocation before the next call.
__device__ __forceinline__ bool rowFits(DevState const& S, int t) {
  const int off = S.pair_off[t];   // negative when the scan's total overflowed
  if (off >= 0 && (long long)off + S.npairs[t] <= (long long)S.pair_cap) return true;
  S.npairs[t] = 0;
  raise(S.status, kErrPairsFull);
  return false;
}

// Appends the first nu entries of slot t's row (seg) to the compact pair
// list (one atomic per warp), with each entry's position in the row.  Every
// lane of the warp calls it; valid lanes only contribute.
__device__ __forceinline__ void appendUpperPairs(DevState const& S, int t, const int* seg, int nu,
                                                 int* status) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int incl = nu;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(full, incl, o);
    if (lane >= o) incl += y;
  }
  const int total = __shfl_sync(full, incl, 31);
  if (!total) return;
  int base = 0;
  if (lane == 31) base = atomicAdd(&S.ctl[kCtlPairs], total);
  base = __shfl_sync(full, base, 31);
  const long long cap = (long long)S.pair_cap / 2 + 1;
  if (base + (long long)total > cap) {
    if (lane == 0) raise(status, kErrPairsFull);
    return;
  }
  const int first = base + incl - nu;
  for (int e = 0; e < nu; ++e) {
    S.upairs[first + e] = make_int2(t, seg[e]);
    S.epos[first + e] = e;
  }
}

// Programmatic dependent launch (sm_90 and later): a kernel launched with
// the programmatic-serialization attribute (launchAfterPrevious) may start
// while the previous kernel of its stream still runs.  pdlWait() returns once
// that kernel has completed and its writes are visible (at once for a kernel
// launched without the attribute); pdlTrigger() lets the next kernel start
// early.  Everything a kernel reads that its predecessor writes, and all its
// writes, come after its pdlWait().
__device__ __forceinline__ void pdlWait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdlTrigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Contact-filter flags of the current force evaluation: two buffers used
// alternately, the filter of one evaluation clearing the other's, so that no
// kernel needs to clear flags that other warps may still be setting.
__device__ __forceinline__ int* contactFlags(DevState const& S, int which = 0) {
  return S.nact + (size_t)(((unsigned)S.ctl[kCtlEpoch] + (unsigned)which) & 1u) * S.cap;
}

// Code of a periodic image shift (in periods, each -1, 0 or 1) in 0..26.
__device__ __forceinline__ int shiftCode(int sx, int sy, int sz) {
  return (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1);
}

// Code of a stencil offset in 0..26 and back.
__device__ __forceinline__ int offCode(int di, int dj, int dk) { return (di + 1) + 3 * (dk + 1) + 9 * (dj + 1); }
__device__ __forceinline__ void offDecode(int c, int* di, int* dj, int* dk) {
  *di = c % 3 - 1; *dk = (c / 3) % 3 - 1; *dj = c / 9 - 1;
}

}  // namespace gdem
