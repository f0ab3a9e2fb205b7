// gdem_contact64.cu -- FP64 mode: pair-list search and the fused force +
// leapfrog step.  Compiled with -fmad=false so that every FP64 expression
// rounds like the reference's scalar CPU code.
//
//   k_pairs_count64 / k_pairs_fill64
//               27-cell stencil enumeration over the pair-list grid (the
//               reference uses the 13-cell half stencil of LinkedCell::
//               setCellContactNeighborhood, Base/src/LinkedCell.cpp:958-984;
//               here each particle lists all its partners so that its forces
//               can be reduced without atomics), first counted, then written
//               into the rows the scan of the counts placed.  A candidate is
//               listed when its bounding spheres are closer than the skin,
//               evaluated with the lower-ID body first so both directions of
//               a pair agree.
//   k_pairlaw64 one thread per pair the contact filter kept: narrow phase
//               (ClosestPointSPHERESPHERE or GJK), Hooke / HookeMemory force
//               with the tangential history in the hashed pair table, and the
//               pair's two shares written into both partners' rows; then one
//               thread per particle near a wall for its wall contacts
//               (SimpleObstacle::InterAction, Component/src/
//               SimpleObstacle.cpp:222-271).  The leapfrog kernel adds the
//               shares of each particle in row (partner-ID) order.
#include <algorithm>

#include "gdem_contact_common.cuh"
#include "gdem_kernels.cuh"
#include "gdem_motion.cuh"

namespace gdem {

namespace {

// Lists a candidate when its bounding spheres are closer than the skin (with
// a relative margin of 1e-12, for periodic images whose two orientations
// round the image translation differently); the pair kernel then decides
// contact exactly (distance < 0) in lower-ID-first orientation.
// kFill = false: returns the row length of slot t.  kFill = true: writes the
// row (its length known from the counting pass), orders it and returns its
// number of upper entries.
template <bool kFill>
__device__ __forceinline__ int listPairs64(DevState const& S, int t) {
  const int4 cc = S.cellc[t];
  GridDesc const& g = S.bgrids[cc.w];
  const double4 pa = S.pos64[t];
  int* out = kFill ? S.pairs + S.pair_off[t] : nullptr;
  const int room = kFill ? S.npairs[t] : 0;
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
    if (kFill && cnt < room) out[cnt] = u | (shiftCode(sx, sy, sz) << 27);
    ++cnt;
  });
  if (!kFill) return cnt;
  return sortEntriesUpperFirst(out, min(cnt, room), S.id, S.id[t]);
}

__global__ void __launch_bounds__(256) k_pairs_count64(DevState S, const int* gate) {
  if (gate && !*gate) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  S.npairs[t] = rowLength(S, listPairs64<false>(S, t));
}

__global__ void __launch_bounds__(256) k_pairs_fill64(DevState S, const int* gate) {
  if (gate && !*gate) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = t < S.n && rowFits(S, t);
  const int nu = valid ? listPairs64<true>(S, t) : 0;
  // each pair once, from its lower ID, into the compact list of the filter
  appendUpperPairs(S, t, valid ? S.pairs + S.pair_off[t] : S.pairs, nu, S.status);
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
                                           int prio0, int prio1, int id0, int id1,
                                           TypeDesc const& tp0,
                                           TypeDesc const& tp1, d3 x0, d3 x1, d3 v0, d3 v1,
                                           d3 w0, d3 w1, bool insert, GjkTally& gjk,
                                           double& delta, d3& f, d3& c0, d3& c1m, d3& mr,
                                           bool& rolling) {
  const int cap = S.cap;
  const unsigned tag = (unsigned)S.ctl[kCtlEpoch], tag_old = tag - 1u;
  // spheres: the history lookup's first probe (key and values) is read
  // before the narrow phase -- the key depends on the two IDs only -- so its
  // loads overlap the narrow phase
  const unsigned long long hkey = pairKey(min(id0, id1), max(id0, id1));
  uint32_t hslot = 0;
  unsigned long long hfirst = 0;
  double hv[9];
  if constexpr (!kConvex) {
    hslot = hashSlot(hkey, S.hist_old.log2cap);
    hfirst = S.hist_old.keys[hslot];
    const double* p = static_cast<const double*>(S.hist_old.vals) + 9 * (size_t)hslot;
#pragma unroll
    for (int k = 0; k < 9; ++k) hv[k] = p[k];
  }
  Contact64 ct;
  if (!kConvex || (tp0.shape == 0 && tp1.shape == 0)) {
    ct = sphereSphere64(x0, tp0.radius, tp0.crust, x1, tp1.radius, tp1.crust);
  } else {
    int c0v = startVertex(S, tp0, s0), c1v = startVertex(S, tp1, s1);
    ct = convexContact64(convexOf(tp0, S), crustXForm(S.basis, cap, s0, tp0.scaling, x0),
                         tp0.radius, tp0.crust, convexOf(tp1, S),
                         crustXForm(S.basis, cap, s1, tp1.scaling, x1), tp1.radius, tp1.crust,
                         c0v, c1v);
    if (ct.gjk_iters > 0) {
      recordVertex(S, tp0, s0, prio0, c0v);
      recordVertex(S, tp1, s1, prio1, c1v);
    }
    if (insert) gjk.add(ct.gjk_iters);   // each pair counted once
  }
  delta = ct.contact ? ct.dist : __longlong_as_double(0x7ff0000000000000ll);
  if (!ct.contact || !(ct.dist < 0.)) return false;
  if (ct.error) raise(S.status, kErrContactOverlap);
  ModelDesc const& m = S.models[g.model_base + tp0.mat * kMaxMat + tp1.mat];
  if (m.memory) {
    // the table holds the lower ID's view; p0 may be the higher ID (the
    // reference's pair orientation), whose view is the negation
    const bool flip = id0 > id1;
    const unsigned long long key = hkey;
    int old;
    if constexpr (!kConvex) {
      if (hfirst == tagged(key, tag_old)) old = (int)hslot;
      else if (tagOf(hfirst) != (tag_old & kTagMask)) old = -1;
      else old = histFindAfter(S.hist_old, key, tag_old, hslot);
    } else {
      old = histFind(S.hist_old, key, tag_old);
    }
    d3 kd, pn, sp;
    if (old >= 0) {
      if (!kConvex && old == (int)hslot) {
        kd = mk(hv[0], hv[1], hv[2]); pn = mk(hv[3], hv[4], hv[5]); sp = mk(hv[6], hv[7], hv[8]);
      } else {
        loadHist(S.hist_old, old, kd, pn, sp);
      }
      if (flip) { kd = -kd; pn = -pn; sp = -sp; }
    }
    hodc64(m, S.dt, ct.point, ct.overlap, x0, v0, w0, tp0.mass, tp0.eqrad, x1, v1, w1, tp1.mass,
           tp1.eqrad, old >= 0, kd, pn, sp, f, mr);
    if (insert) {
      int slot = histInsert(S.hist_new, key, tag);
      if (slot < 0) raise(S.status, kErrHashFull);
      else if (flip) storeHist(S.hist_new, slot, -kd, -pn, -sp);
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

// One side of a pair in contact, as the leapfrog kernel adds it: the
// evaluation tag, the force on the row's particle and its torque (lever arm
// x force, plus the rolling torque); 64 bytes, four 16-byte words.
__device__ __forceinline__ void storeShare64(DevState const& S, int64_t entry, int tag, d3 f,
                                             d3 c) {
  double2* sh = static_cast<double2*>(S.share) + 4 * entry;
  sh[0] = make_double2(__longlong_as_double((long long)tag), f.x);
  sh[1] = make_double2(f.y, f.z);
  sh[2] = make_double2(c.x, c.y);
  sh[3] = make_double2(c.z, 0.);
}

// The wall contacts of particle t (near a wall per the contact filter): the
// particle is p0, the obstacle p1 (mass Component::m_massObstacle); their
// sum is the particle's wall share.
template <bool kConvex>
__device__ __forceinline__ void wallsOf64(DevState const& S, int t, int tag, GjkTally& gjk,
                                          StatsTally& st) {
  const int cap = S.cap;
  GridDesc const& g = S.grids[S.inst[t]];
  const int ida = S.id[t];
  TypeDesc const& ta = S.types[S.type[t]];
  const d3 xt = ld3(S.x, cap, t), vt = ld3(S.v, cap, t), wt = ld3(S.w, cap, t);
  const double dt = S.dt;
  const unsigned utag = (unsigned)tag, tag_old = utag - 1u;
  d3 Fw = mk(0., 0., 0.), Tw = mk(0., 0., 0.);
  bool any = false;
  // the particle's polyhedron vertex runs through its wall calls in order
  int curw = kConvex ? startVertex(S, ta, t) : 0;
  bool walls_gjk = false;
  for (int k = 0; k < g.wall_count; ++k) {
    WallDesc const& wd = S.walls[g.wall_begin + k];
    int cw = 0;
    Contact64 ct = (!kConvex || ta.shape == 0)
        ? sphereWall64(xt, ta.radius, ta.crust, wd)
        : convexContact64(convexOf(ta, S), crustXForm(S.basis, cap, t, ta.scaling, xt),
                          ta.radius, ta.crust, convexOf(wd),
                          identityXForm(wd.scaling, mk(wd.centre[0], wd.centre[1], wd.centre[2])),
                          wd.radius, wd.crust, curw, cw);
    if (kConvex) gjk.add(ct.gjk_iters);
    if (kConvex && ct.gjk_iters > 0) walls_gjk = true;
    if (S.diag) S.wall_delta[(size_t)t * S.max_walls + k] = ct.contact ? ct.dist : __longlong_as_double(0x7ff0000000000000ll);
    if (ct.error) raise(S.status, kErrContactOverlap);
    if (!ct.contact || !(ct.dist < 0.)) continue;
    st.add(ct.dist);
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
      int slot = histInsert(S.hist_new, key, utag);
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
    Fw = Fw + f;
    Tw = Tw + cross(ct.point - xt, f);
    if (m.rolling) Tw = Tw + mr;
    any = true;
  }
  if (walls_gjk) recordVertex(S, ta, t, kWallPriority, curw);
  if (!any) return;
  double2* ws = static_cast<double2*>(S.wshare) + 3 * (size_t)t;
  ws[0] = make_double2(Fw.x, Fw.y);
  ws[1] = make_double2(Fw.z, Tw.x);
  ws[2] = make_double2(Tw.y, Tw.z);
  atomicOr(reinterpret_cast<unsigned*>(&contactFlags(S)[t]), kNearWall);
}

// One pair kept by the contact filter (compact pair c), seen from its lower
// ID, which writes the history: exact narrow phase, force law, and for a
// contact its two shares written into the rows of both partners and their
// entry bits set.  The leapfrog kernel adds each particle's shares in row
// order, so the sums are deterministic and need no float atomics.
template <bool kConvex>
__device__ __forceinline__ void pairItem64(DevState const& S, int c, int tag, GjkTally& gjk,
                                           StatsTally& st) {
  const int cap = S.cap;
  const int2 pr = S.upairs[c];
  const int ep = S.epos[c];
  const int t = pr.x;
  const unsigned ent = (unsigned)pr.y;
  const int u = (int)(ent & ((1u << 27) - 1u));
  const int et = ep & 0xFFFF, eu = (int)((unsigned)ep >> 16);
  GridDesc const& g = S.grids[S.inst[t]];
  int sh[3];
  entryShift(S, ent, t, u, sh);
  const d3 shift = mk(sh[0] * g.L[0], sh[1] * g.L[1], sh[2] * g.L[2]);
  const d3 xt = ld3(S.x, cap, t), xu = ld3(S.x, cap, u);
  const int idt = S.id[t], idu = S.id[u];
  // the rest of both particles' inputs and their row offsets load with the
  // positions (the stores of the history update would otherwise hold the
  // later loads back); a pair of non-spherical bodies loads its velocities
  // after the closest-point search, which keeps them out of its registers
  const int tyt = S.type[t], tyu = S.type[u];
  const int offt = S.pair_off[t], offu = S.pair_off[u];
  d3 vt, vu, wt, wu;
  if constexpr (!kConvex) {
    vt = ld3(S.v, cap, t); vu = ld3(S.v, cap, u);
    wt = ld3(S.w, cap, t); wu = ld3(S.w, cap, u);
  }
  // p0 as in the reference (flip: u is p0, at its own position)
  const bool flip = referenceFlip(g, xt, xu, sh);
  const int a = flip ? u : t, b = flip ? t : u;
  if constexpr (kConvex) {
    vt = ld3(S.v, cap, a); vu = ld3(S.v, cap, b);
    wt = ld3(S.w, cap, a); wu = ld3(S.w, cap, b);
  } else if (flip) {
    const d3 sv = vt, sw = wt;
    vt = vu; vu = sv; wt = wu; wu = sw;
  }
  const int pa = min((flip ? eu : et) + 1, kWallPriority - 1),
            pb = min((flip ? et : eu) + 1, kWallPriority - 1);
  d3 f, c0, c1m, mr;
  double dl;
  bool rolling;
  const bool hit = evalPair64<kConvex>(
      S, g, a, b, pa, pb, flip ? idu : idt, flip ? idt : idu, S.types[flip ? tyu : tyt], S.types[flip ? tyt : tyu],
      flip ? xu : xt, flip ? xt + (-shift) : xu + shift, vt, vu, wt, wu, true, gjk, dl, f, c0, c1m, mr, rolling);
  const int64_t rt = (int64_t)offt + et, ru = (int64_t)offu + eu;
  // p0's share (f, its torque) and p1's (-f, its torque), given to t and u
  const d3 t0 = rolling ? c0 + mr : c0, t1 = rolling ? c1m + (-mr) : c1m;
  const d3 ft = flip ? -f : f;
  if (S.diag) {
    S.pair_delta[rt] = dl;
    if (eu != 0xFFFF) S.pair_delta[ru] = dl;
    if (hit) {
      double* fd = S.pair_force + 3 * rt;
      fd[0] = ft.x; fd[1] = ft.y; fd[2] = ft.z;
      if (eu != 0xFFFF) {
        fd = S.pair_force + 3 * ru;
        fd[0] = ft.x; fd[1] = ft.y; fd[2] = ft.z;
      }
    }
  }
  if (!hit) return;
  st.add(dl);
  int* flags = contactFlags(S);
  storeShare64(S, rt, tag, ft, flip ? t1 : t0);
  atomicOr(reinterpret_cast<unsigned*>(&flags[t]), entryBit(et));
  if (eu != 0xFFFF) {
    storeShare64(S, ru, tag, -ft, flip ? t0 : t1);
    atomicOr(reinterpret_cast<unsigned*>(&flags[u]), entryBit(eu));
  }
}

// The pair kernel of an evaluation, one thread per item over a persistent
// grid: first the pairs the contact filter kept, then the particles near a
// wall.  Its trigger comes after its wait, so the leapfrog kernel, which
// starts at the trigger, sees the filter's candidate marks complete.
template <bool kConvex>
__global__ void __launch_bounds__(128) k_pairlaw64(DevState S) {
  pdlWait();      // the contact filter's lists
  pdlTrigger();   // the leapfrog kernel may start; its candidates wait for this kernel
  const int nk = S.ctl[kCtlKept], nw = S.ctl[kCtlWork];
  const int tag = S.ctl[kCtlEpoch];
  const int stride = gridDim.x * blockDim.x;
  GjkTally gjk;
  StatsTally st;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nk + nw; i += stride) {
    if (i < nk) pairItem64<kConvex>(S, S.kept[i], tag, gjk, st);
    else wallsOf64<kConvex>(S, S.work[i - nk], tag, gjk, st);
  }
  // (every lane of the warp reaches this point: no thread leaves the loop early)
  if constexpr (kConvex) gjk.flush(S.gjk_counts);
  st.flush(S.cstats, tag);
}


// ------------------------------------------------------------- insertion --
// The overlap test of one insertion attempt (LinkedCell::isContactWithCrust,
// Base/src/LinkedCell.cpp:1211-1240, through Cell::isContactWithCrust,
// Base/src/Cell.cpp:250-290): the candidate against every particle (at its
// periodic images within one period where the domain is periodic, as the
// reference tests the candidate and its clones against the cells' particles
// and clones) and every wall.  The test of two bodies is
// RigidBodyWithCrust::isContact (Geometry/src/RigidBodyWithCrust.cpp:
// 840-958): two spheres touch when their centres are closer than the sum of
// the radii (isContactSPHERESPHERE), a sphere and a box when the sphere
// overlaps the box (isContactSPHEREBOX, the box's own frame: a wall's is its
// centre); otherwise when the circumscribed spheres overlap and -- unless
// bv_only (GeometricOverlap Value="BV") -- the GJK distance of the shrunk
// bodies is below the sum of the crusts minus 1e-10.  A polyhedron's search
// starts from the particle's current vertex and from the candidate's first
// vertex with a neighbour, and moves neither.
__device__ bool insertTouch(DevState const& S, TypeDesc const& ta, XForm64 const& a2w,
                            const double* basis_a, int stride_a, int slot_a, int cur_a,
                            TypeDesc const& tb, d3 xb, const double* basis_b, int bv_only) {
  const d3 xa = a2w.o;
  if (ta.shape == 0 && tb.shape == 0) return norm(xb - xa) - (ta.radius + tb.radius) < 0.;
  if ((ta.shape == 0 && tb.shape == 1) || (ta.shape == 1 && tb.shape == 0)) {
    // the sphere's centre in the box's frame: R^T (p - o)
    const bool a_sphere = ta.shape == 0;
    TypeDesc const& box = a_sphere ? tb : ta;
    const d3 p = (a_sphere ? xa : xb) - (a_sphere ? xb : xa);
    double R[9];
    if (a_sphere) {
      for (int k = 0; k < 9; ++k) R[k] = basis_b[k];
    } else {
      for (int k = 0; k < 9; ++k) R[k] = basis_a[k * stride_a + slot_a];
    }
    const d3 local = mk(R[0] * p.x + R[3] * p.y + R[6] * p.z, R[1] * p.x + R[4] * p.y + R[7] * p.z,
                        R[2] * p.x + R[5] * p.y + R[8] * p.z);
    double ov = 1.;
    boxSphere(mk(box.extent[0], box.extent[1], box.extent[2]), local,
              a_sphere ? ta.radius : tb.radius, ov);
    return ov < 0.;
  }
  if (!(norm(xa - xb) < ta.radius + tb.radius)) return false;
  if (bv_only) return true;
  const XForm64 b2w = crustXForm(basis_b, 1, 0, tb.scaling, xb);
  d3 pA, pB;
  int it = 0, ca = cur_a, cb = tb.poly_start;
  const double d = closestPoints64(convexOf(ta, S), a2w, convexOf(tb, S), b2w, pA, pB, &it, ca, cb);
  return d < ta.crust + tb.crust - 1.0e-10;
}

__global__ void k_insert_test(DevState S, NewParticle p, int bv_only, int* hit) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  GridDesc const& g = S.grids[0];
  TypeDesc const& tc = S.types[p.type];
  const d3 xc = mk(p.x[0], p.x[1], p.x[2]);
  bool touch = false;
  if (i < S.n) {
    TypeDesc const& tu = S.types[S.type[i]];
    const d3 xu = ld3(S.x, S.cap, i);
    const int cur = S.curv ? S.curv[i] : 0;
    for (int sx = g.periodic[0] ? -1 : 0; sx <= (g.periodic[0] ? 1 : 0) && !touch; ++sx)
      for (int sy = g.periodic[1] ? -1 : 0; sy <= (g.periodic[1] ? 1 : 0) && !touch; ++sy)
        for (int sz = g.periodic[2] ? -1 : 0; sz <= (g.periodic[2] ? 1 : 0) && !touch; ++sz) {
          const d3 xi = xu + mk(sx * g.L[0], sy * g.L[1], sz * g.L[2]);
          const XForm64 a2w = (tu.shape == 0 || !S.basis)
                                  ? identityXForm(tu.scaling, xi)
                                  : crustXForm(S.basis, S.cap, i, tu.scaling, xi);
          touch = insertTouch(S, tu, a2w, S.basis, S.cap, i, cur, tc, xc, p.basis, bv_only);
        }
  } else if (i < S.n + g.wall_count) {
    WallDesc const& wd = S.walls[g.wall_begin + (i - S.n)];
    const d3 o = mk(wd.centre[0], wd.centre[1], wd.centre[2]);
    if (tc.shape == 0) {
      double ov = 1.;
      boxSphere(mk(wd.extent[0], wd.extent[1], wd.extent[2]), xc - o, tc.radius, ov);
      touch = ov < 0.;
    } else if (norm(xc - o) < wd.radius + tc.radius) {
      touch = true;
      if (!bv_only) {
        d3 pA, pB;
        int it = 0, cw = 0, cb = tc.poly_start;
        const double d = closestPoints64(convexOf(wd), identityXForm(wd.scaling, o), convexOf(tc, S),
                                         crustXForm(p.basis, 1, 0, tc.scaling, xc), pA, pB, &it, cw, cb);
        touch = d < wd.crust + tc.crust - 1.0e-10;
      }
    }
  }
  if (touch) atomicOr(hit, 1);
}
}  // namespace

void launch_pairs64(DevState const& S, const int* gate, int fill, cudaStream_t st) {
  if (!S.n) return;
  if (fill) k_pairs_fill64<<<(S.n + 255) / 256, 256, 0, st>>>(S, gate);
  else k_pairs_count64<<<(S.n + 255) / 256, 256, 0, st>>>(S, gate);
}
void launch_pairlaw64(DevState const& S, cudaStream_t st) {
  if (!S.n) return;
  const int grid = (S.forces_bps > 0 ? S.forces_bps : 4) * S.nsm;
  if (S.any_convex) launchAfterPrevious(k_pairlaw64<true>, grid, 128, st, S);
  else launchAfterPrevious(k_pairlaw64<false>, grid, 128, st, S);
}
void launch_insert_test(DevState const& S, NewParticle const& p, int bv_only, int* hit,
                        cudaStream_t st) {
  const int n = S.n + S.max_walls;
  k_insert_test<<<(n + 127) / 128, 128, 0, st>>>(S, p, bv_only, hit);
}

}  // namespace gdem
