// gdem_contact64.cu -- FP64 mode: pair-list search and the fused force +
// leapfrog step.  Compiled with -fmad=false so that every FP64 expression
// rounds like the reference's scalar CPU code.
//
//   k_pairs64   27-cell stencil enumeration over the pair-list grid (the
//               reference uses the 13-cell half stencil of LinkedCell::
//               setCellContactNeighborhood, Base/src/LinkedCell.cpp:958-984;
//               here each particle lists all its partners so that its forces
//               can be reduced without atomics).  A candidate is listed when
//               its bounding spheres are closer than the skin, evaluated with
//               the lower-ID body first so both directions of a pair agree.
//   k_forces64  for each particle: narrow phase on every entry that the
//               contact filter kept (ClosestPointSPHERESPHERE or GJK), Hooke /
//               HookeMemory force with the tangential history in the hashed
//               pair table, the deterministic reduction of its force and
//               torque over those entries in list (partner-ID) order, then its
//               wall contacts (SimpleObstacle::InterAction, Component/src/
//               SimpleObstacle.cpp:222-271).
#include <algorithm>

#include "gdem_contact_common.cuh"
#include "gdem_kernels.cuh"
#include "gdem_motion.cuh"

namespace gdem {

namespace {

// Lists a candidate when its bounding spheres are closer than the skin (with
// a relative margin of 1e-12, for periodic images whose two orientations
// round the image translation differently); k_forces64 then decides contact
// exactly (distance < 0) in lower-ID-first orientation.
// The list of slot t; returns its number of upper entries.
__device__ __forceinline__ int listPairs64(DevState const& S, int t) {
  const int4 cc = S.cellc[t];
  GridDesc const& g = S.bgrids[cc.w];
  const double4 pa = S.pos64[t];
  int* out = S.pairs + (size_t)t * kPairCap;
  int cnt = 0;
  const double4* __restrict__ pos = S.pos64;
  forEachCandidate(S.cell_start, g, cc, [&](int u, int dcx, int dj, int dk, int sx, int sy, int sz) {
    if (u == t) return;
    const double4 pb = pos[u];
    d3 shift = mk(sx * g.L[0], sy * g.L[1], sz * g.L[2]);
    d3 d = u > t ? (mk(pb.x, pb.y, pb.z) + shift) - mk(pa.x, pa.y, pa.z)
                 : (mk(pa.x, pa.y, pa.z) + (-shift)) - mk(pb.x, pb.y, pb.z);
    double R = pa.w + pb.w;
    if (norm(d) - R > g.skin + 1.0e-12 * R) return;
    if (cnt < kPairCap) out[cnt] = u | (shiftCode(sx, sy, sz) << 27);
    ++cnt;
  });
  if (cnt > kPairCap) { raise(S.status, kErrPairsFull); cnt = kPairCap; }
  const int nu = sortEntriesUpperFirst(out, cnt, S.id, S.id[t]);
  S.npairs[t] = cnt;
  return nu;
}

__global__ void __launch_bounds__(256) k_pairs64(DevState S, const int* gate) {
  if (gate && !*gate) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = t < S.n;
  const int nu = valid ? listPairs64(S, t) : 0;
  // each pair once, from its lower ID, into the compact list of the filter
  appendUpperPairs(S, t, valid ? S.pairs + (size_t)t * kPairCap : S.pairs, nu, S.status);
}

__device__ __forceinline__ void loadHist(HistTable const& t, int slot, d3& kd, d3& pn, d3& sp) {
  const double* v = static_cast<const double*>(t.vals) + 9 * (size_t)slot;
  kd = mk(v[0], v[1], v[2]); pn = mk(v[3], v[4], v[5]); sp = mk(v[6], v[7], v[8]);
}
__device__ __forceinline__ void storeHist(HistTable const& t, int slot, d3 kd, d3 pn, d3 sp) {
  double* v = static_cast<double*>(t.vals) + 9 * (size_t)slot;
  v[0] = kd.x; v[1] = kd.y; v[2] = kd.z; v[3] = pn.x; v[4] = pn.y; v[5] = pn.z;
  v[6] = sp.x; v[7] = sp.y; v[8] = sp.z;
}

// One pair in the canonical orientation -- p0 (slot s0, the lower ID) at its
// own position, p1 at its periodic image seen from p0 -- with the
// reference's expressions (closest points, Hooke / HookeMemory) and the
// contact history (the new entry written when insert).  Returns true for a
// contact, with the force f on p0, the torques c0 = (point - x0) x f and
// c1m = (point - x1) x (-f) of p0 and p1, and the rolling torque mr
// (rolling: the model has rolling resistance); delta gets the distance
// (+inf without contact).  kConvex: some class is not a sphere, so the GJK
// narrow phase is compiled in.
template <bool kConvex>
__device__ __forceinline__ bool evalPair64(DevState const& S, GridDesc const& g, int s0, int s1,
                                           int id0, int id1, TypeDesc const& tp0,
                                           TypeDesc const& tp1, d3 x0, d3 x1, d3 v0, d3 v1,
                                           d3 w0, d3 w1, bool insert, GjkTally& gjk,
                                           double& delta, d3& f, d3& c0, d3& c1m, d3& mr,
                                           bool& rolling) {
  const int cap = S.cap;
  const unsigned tag = (unsigned)S.ctl[kCtlEpoch], tag_old = tag - 1u;
  Contact64 ct;
  if (!kConvex || (tp0.shape == 0 && tp1.shape == 0)) {
    ct = sphereSphere64(x0, tp0.radius, tp0.crust, x1, tp1.radius, tp1.crust);
  } else {
    ct = convexContact64(convexOf(tp0, S.poly_verts), crustXForm(S.basis, cap, s0, tp0.scaling, x0),
                         tp0.radius, tp0.crust, convexOf(tp1, S.poly_verts),
                         crustXForm(S.basis, cap, s1, tp1.scaling, x1), tp1.radius, tp1.crust);
    if (insert) gjk.add(ct.gjk_iters);   // each pair counted once
  }
  delta = ct.contact ? ct.dist : __longlong_as_double(0x7ff0000000000000ll);
  if (!ct.contact || !(ct.dist < 0.)) return false;
  if (ct.error) raise(S.status, kErrContactOverlap);
  ModelDesc const& m = S.models[g.model_base + tp0.mat * kMaxMat + tp1.mat];
  if (m.memory) {
    const unsigned long long key = pairKey(id0, id1);
    int old = histFind(S.hist_old, key, tag_old);
    d3 kd, pn, sp;
    if (old >= 0) loadHist(S.hist_old, old, kd, pn, sp);
    hodc64(m, S.dt, ct.point, ct.overlap, x0, v0, w0, tp0.mass, tp0.eqrad, x1, v1, w1, tp1.mass,
           tp1.eqrad, old >= 0, kd, pn, sp, f, mr);
    if (insert) {
      int slot = histInsert(S.hist_new, key, tag);
      if (slot < 0) raise(S.status, kErrHashFull);
      else storeHist(S.hist_new, slot, kd, pn, sp);
    }
  } else {
    hooke64(m, ct.point, ct.overlap, x0, v0, w0, tp0.mass, tp0.eqrad, x1, v1, w1, tp1.mass,
            tp1.eqrad, f, mr);
  }
  c0 = cross(ct.point - x0, f);
  c1m = cross(ct.point - x1, -f);
  rolling = m.rolling != 0;
  if (!rolling) mr = mk(0., 0., 0.);
  return true;
}

// Position in slot t's list of the entry whose partner is slot u.
__device__ __forceinline__ int findEntry(DevState const& S, int t, int u) {
  const int n = S.npairs[t];
  const int* seg = S.pairs + (size_t)t * kPairCap;
  for (int e = 0; e < n; ++e)
    if ((int)((unsigned)seg[e] & ((1u << 27) - 1u)) == u) return e;
  return -1;
}

// One side's share of a pair (two-phase path): force and torque terms in the
// order the per-particle sum adds them.
struct PairShare64 { double f[3], c[3], mr[3]; };

// Forces and torques on particle t.  kSums (two-phase path, systems with
// convex bodies): the pairs were evaluated once each by k_pairforces64, and
// each kept entry's share is read back; otherwise both partners of a pair
// evaluate it, with identical operands, and the lower ID writes the history.
// Either way the shares are added in list order, then the walls.
template <bool kConvex, bool kSums>
__device__ __forceinline__ void forcesOn64(DevState const& S, int t, int na, int sparse,
                                           GjkTally& gjk) {
  const int cap = S.cap;
  const int4 cc = S.cellc[t];
  GridDesc const& g = S.grids[cc.w];
  const int ida = S.id[t];
  TypeDesc const& ta = S.types[S.type[t]];
  const d3 xt = ld3(S.x, cap, t), vt = ld3(S.v, cap, t), wt = ld3(S.w, cap, t);
  d3 F = mk(ta.weight[0], ta.weight[1], ta.weight[2]);
  d3 T = mk(0., 0., 0.);
  const double dt = S.dt;
  const unsigned tag = (unsigned)S.ctl[kCtlEpoch], tag_old = tag - 1u;
  // the pair-list entries that pass the contact filter's test
  const int np = (!sparse || (na & kHasPair)) ? S.npairs[t] : 0;
  const int* seg = S.pairs + (size_t)t * kPairCap;
  GridDesc const& bg = S.bgrids[cc.w];
  const float4 pt = S.posf[t];
  for (int e0 = 0; e0 < np; e0 += kProbe) {
    unsigned keep = probeEntries(S, bg, pt, seg, e0, np);
    if (S.diag)
      for (int e = e0; e < min(e0 + kProbe, np); ++e)
        if (!(keep >> (e - e0) & 1u))
          S.pair_delta[(size_t)t * kPairCap + e] = __longlong_as_double(0x7ff0000000000000ll);
    // the kept entries in list order; lane by lane the k-th kept entries run
    // together, as the warp's lanes hold different particles
    while (keep) {
      const int e = e0 + __ffs(keep) - 1;
      keep &= keep - 1u;
      if constexpr (kSums) {
        const PairShare64 r = static_cast<const PairShare64*>(S.pshare)[S.eslot[(size_t)t * kPairCap + e]];
        F = F + mk(r.f[0], r.f[1], r.f[2]);
        T = T + mk(r.c[0], r.c[1], r.c[2]);
        T = T + mk(r.mr[0], r.mr[1], r.mr[2]);
        continue;
      }
      const uint32_t ent = (uint32_t)seg[e];
      const int u = (int)(ent & ((1u << 27) - 1));
      int sh[3];
      entryShift(S, ent, t, u, sh);
      d3 shift = mk(sh[0] * g.L[0], sh[1] * g.L[1], sh[2] * g.L[2]);
      const int idb = S.id[u];
      TypeDesc const& tb = S.types[S.type[u]];
      const d3 xu = ld3(S.x, cap, u), vu = ld3(S.v, cap, u), wu = ld3(S.w, cap, u);
      const bool t0 = ida < idb;
      // canonical bodies: p0 = lower ID at its own position, p1 at its image
      d3 f, c0, c1m, mr;
      double dl;
      bool rolling;
      const bool hit = evalPair64<kConvex>(
          S, g, t0 ? t : u, t0 ? u : t, t0 ? ida : idb, t0 ? idb : ida, t0 ? ta : tb,
          t0 ? tb : ta, t0 ? xt : xu, t0 ? xu + shift : xt + (-shift), t0 ? vt : vu,
          t0 ? vu : vt, t0 ? wt : wu, t0 ? wu : wt, t0, gjk, dl, f, c0, c1m, mr, rolling);
      if (S.diag) {
        S.pair_delta[(size_t)t * kPairCap + e] = dl;
        if (hit) {
          double* fd = S.pair_force + 3 * ((size_t)t * kPairCap + e);
          fd[0] = f.x; fd[1] = f.y; fd[2] = f.z;
        }
      }
      if (!hit) continue;
      if (t0) {
        F = F + f;
        T = T + c0;
        if (rolling) T = T + mr;
      } else {
        F = F + (-f);
        T = T + c1m;
        if (rolling) T = T + (-mr);
      }
    }
  }
  // walls: the particle is p0, the obstacle p1 (mass Component::m_massObstacle)
  const int nwalls = (!sparse || (na & kNearWall)) ? g.wall_count : 0;
  for (int k = 0; k < nwalls; ++k) {
    WallDesc const& wd = S.walls[g.wall_begin + k];
    Contact64 ct = (!kConvex || ta.shape == 0)
        ? sphereWall64(xt, ta.radius, ta.crust, wd)
        : convexContact64(convexOf(ta, S.poly_verts), crustXForm(S.basis, cap, t, ta.scaling, xt),
                          ta.radius, ta.crust, convexOf(wd),
                          identityXForm(wd.scaling, mk(wd.centre[0], wd.centre[1], wd.centre[2])),
                          wd.radius, wd.crust);
    if (kConvex) gjk.add(ct.gjk_iters);
    if (S.diag) S.wall_delta[(size_t)t * S.max_walls + k] = ct.contact ? ct.dist : __longlong_as_double(0x7ff0000000000000ll);
    if (ct.error) raise(S.status, kErrContactOverlap);
    if (!ct.contact || !(ct.dist < 0.)) continue;
    ModelDesc const& m = S.models[g.model_base + ta.mat * kMaxMat + wd.mat];
    d3 f, mr;
    const d3 zero = mk(0., 0., 0.);
    const d3 wc = mk(wd.centre[0], wd.centre[1], wd.centre[2]);
    if (m.memory) {
      const unsigned long long key = wallKey(ida, k);
      int old = histFind(S.hist_old, key, tag_old);
      d3 kd, pn, sp;
      if (old >= 0) loadHist(S.hist_old, old, kd, pn, sp);
      hodc64(m, dt, ct.point, ct.overlap, xt, vt, wt, ta.mass, ta.eqrad, wc, zero, zero, 1.e20,
             wd.eqrad, old >= 0, kd, pn, sp, f, mr);
      int slot = histInsert(S.hist_new, key, tag);
      if (slot < 0) raise(S.status, kErrHashFull);
      else storeHist(S.hist_new, slot, kd, pn, sp);
    } else {
      hooke64(m, ct.point, ct.overlap, xt, vt, wt, ta.mass, ta.eqrad, wc, zero, zero, 1.e20,
              wd.eqrad, f, mr);
    }
    if (S.diag) {
      double* fd = S.wall_force + 3 * ((size_t)t * S.max_walls + k);
      fd[0] = f.x; fd[1] = f.y; fd[2] = f.z;
    }
    F = F + f;
    T = T + cross(ct.point - xt, f);
    if (m.rolling) T = T + mr;
  }
  st3(S.F, cap, t, F);
  st3(S.T, cap, t, T);
}

// Persistent grid.  sparse: only the particles of the work list (those with
// a listed contact or near a wall); the others keep their weight, which
// k_move applies without reading F, T.  Otherwise every particle.
template <bool kConvex, bool kSums>
__global__ void __launch_bounds__(256) k_forces64(DevState S, int sparse) {
  const int stride = gridDim.x * blockDim.x;
  pdlWait();      // the contact filter's work list and flags
  pdlTrigger();   // the move kernel may be scheduled; it waits for this one
  const int nw = sparse ? S.ctl[kCtlWork] : S.n;
  const int* flags = contactFlags(S);
  GjkTally gjk;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += stride) {
    const int t = sparse ? S.work[i] : i;
    forcesOn64<kConvex, kSums>(S, t, flags[t], sparse, gjk);
  }
  // (every lane of the warp reaches this point: no thread leaves the loop early)
  if constexpr (kConvex) gjk.flush(S.gjk_counts);
}

// First phase of the two-phase force path (systems with convex bodies):
// each pair kept by the contact filter is evaluated once, by one thread, and
// its two shares are written for the partners' sums (forcesOn64 with
// kSums).  The pair is seen from its lower ID (an upper entry), which writes
// the history, as in the one-phase path, so both paths give the same forces.
template <bool kConvex>
__global__ void __launch_bounds__(128) k_pairforces64(DevState S) {
  pdlWait();      // the contact filter's kept pairs
  pdlTrigger();   // the force sums may be scheduled; they wait for this kernel
  const int nk = S.ctl[kCtlKept];
  const int stride = gridDim.x * blockDim.x;
  const int cap = S.cap;
  GjkTally gjk;
  PairShare64* share = static_cast<PairShare64*>(S.pshare);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += stride) {
    const int2 pr = S.upairs[S.kept[k]];
    const int t = pr.x;
    const unsigned ent = (unsigned)pr.y;
    const int u = (int)(ent & ((1u << 27) - 1u));
    const int et = findEntry(S, t, u), eu = findEntry(S, u, t);
    GridDesc const& g = S.grids[S.inst[t]];
    int sh[3];
    entryShift(S, ent, t, u, sh);
    const d3 shift = mk(sh[0] * g.L[0], sh[1] * g.L[1], sh[2] * g.L[2]);
    const d3 xt = ld3(S.x, cap, t), xu = ld3(S.x, cap, u);
    d3 f, c0, c1m, mr;
    double dl;
    bool rolling;
    const bool hit = evalPair64<kConvex>(
        S, g, t, u, S.id[t], S.id[u], S.types[S.type[t]], S.types[S.type[u]], xt, xu + shift,
        ld3(S.v, cap, t), ld3(S.v, cap, u), ld3(S.w, cap, t), ld3(S.w, cap, u), true, gjk, dl,
        f, c0, c1m, mr, rolling);
    const d3 zero = mk(0., 0., 0.);
    const d3 fa = hit ? f : zero, ca = hit ? c0 : zero, ma = hit ? mr : zero;
    const d3 fb = hit ? -f : zero, cb = hit ? c1m : zero, mb = hit ? -mr : zero;
    PairShare64 a, b;
    a.f[0] = fa.x; a.f[1] = fa.y; a.f[2] = fa.z; a.c[0] = ca.x; a.c[1] = ca.y; a.c[2] = ca.z;
    a.mr[0] = ma.x; a.mr[1] = ma.y; a.mr[2] = ma.z;
    b.f[0] = fb.x; b.f[1] = fb.y; b.f[2] = fb.z; b.c[0] = cb.x; b.c[1] = cb.y; b.c[2] = cb.z;
    b.mr[0] = mb.x; b.mr[1] = mb.y; b.mr[2] = mb.z;
    share[2 * k] = a;
    share[2 * k + 1] = b;
    if (et >= 0) S.eslot[(size_t)t * kPairCap + et] = 2 * k;
    if (eu >= 0) S.eslot[(size_t)u * kPairCap + eu] = 2 * k + 1;
    if (S.diag) {
      for (int side = 0; side < 2; ++side) {
        const int s = side ? u : t, e = side ? eu : et;
        if (e < 0) continue;
        S.pair_delta[(size_t)s * kPairCap + e] = dl;
        if (hit) {
          double* fd = S.pair_force + 3 * ((size_t)s * kPairCap + e);
          fd[0] = f.x; fd[1] = f.y; fd[2] = f.z;
        }
      }
    }
  }
  // (every lane of the warp reaches this point)
  if constexpr (kConvex) gjk.flush(S.gjk_counts);
}

}  // namespace

void launch_pairs64(DevState const& S, const int* gate, cudaStream_t st) {
  if (S.n) k_pairs64<<<(S.n + 255) / 256, 256, 0, st>>>(S, gate);
}
void launch_forces64(DevState const& S, int sparse, cudaStream_t st) {
  if (!S.n) return;
  const int grid = std::min((S.n + 255) / 256, (S.forces_bps > 0 ? S.forces_bps : 4) * S.nsm);
  if (S.any_convex) {
    // two phases: each kept pair once, then the sums
    launchAfterPrevious(k_pairforces64<true>, 4 * S.nsm, 128, st, S);
    launchAfterPrevious(k_forces64<true, true>, grid, 256, st, S, sparse);
  } else {
    launchAfterPrevious(k_forces64<false, false>, grid, 256, st, S, sparse);
  }
}

}  // namespace gdem
