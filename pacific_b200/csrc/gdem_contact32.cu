// gdem_contact32.cu -- FP32-split mode contact kernels.
//
// Broad phase: positions enter as the particle's cell (integer) plus its FP32
// offset from the cell's lower corner, so the vector between two particles in
// neighbouring cells,  d = dc * edge + (off_b - off_a)  with dc in {-1, 0, 1},
// is formed from small FP32 numbers whatever the domain size; candidates are
// kept with a relative margin of 4e-6 on the sum of radii.
//
// Narrow phase: each kept candidate (a near contact: a few per particle) is
// decided on the FP64 master positions with the reference's expressions, so
// contact sets equal the FP64 mode's and the overlap keeps FP64 accuracy even
// for a contact that has only just formed (an FP32 or float-float overlap
// would carry a relative error of 1e-5 when the overlap is 1e-11 m).  The
// relative velocity at the contact point and its normal/tangential split are
// formed in FP64 too (differences of nearly equal quantities).  The Hooke /
// HookeMemory force law, the tangential history, the torque lever arms and
// the per-particle reduction are FP32.  Results are written to the FP64
// force/torque arrays that the FP64 leapfrog consumes.
//
// Reference functions restated: ClosestPointSPHERESPHERE
// (Geometry/src/RigidBodyWithCrust.cpp:596-639), HookeMemoryContactForceModel
// (Component/src/HookeMemoryContactForceModel.cpp:54-249), Torsor::addForce
// (Component/src/Torsor.cpp:184-189).
#include <algorithm>

#include "gdem_contact_common.cuh"
#include "gdem_kernels.cuh"
#include "gdem_motion.cuh"

namespace gdem {

namespace {

// ------------------------------------------------------------ float3 ops --
__device__ __forceinline__ float3 f3(float a, float b, float c) { return make_float3(a, b, c); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dotf(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 crossf(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float normf3(float3 a) { return sqrtf(dotf(a, a)); }

// Quaternion::setRotFromTwoVectors (the rotation taking u to v) in FP32.
struct rot32 { float3 v; float w; };
__device__ __forceinline__ rot32 rotFromTo(float3 u, float3 v) {
  float nn = sqrtf(dotf(u, u) * dotf(v, v));
  float real = nn + dotf(u, v);
  float3 vect;
  if (real < 1.e-6f * nn) {
    real = 0.f;
    vect = fabsf(u.x) > fabsf(u.z) ? f3(-u.y, u.x, 0.f) : f3(0.f, -u.z, u.y);
  } else {
    vect = crossf(u, v);
  }
  float nq = sqrtf(dotf(vect, vect) + real * real);
  rot32 r;
  if (!(nq > 0.f)) { r.v = f3(0.f, 0.f, 0.f); r.w = 1.f; return r; }
  float s = 1.f / nq;
  r.v = vect * s;
  r.w = real * s;
  return r;
}
// Quaternion::rotateVector in FP32
__device__ __forceinline__ float3 rotate(rot32 const& q, float3 x) {
  float nv2 = dotf(q.v, q.v);
  return ((q.w * q.w - nv2) * x + (2.f * dotf(x, q.v)) * q.v) + (2.f * q.w) * crossf(q.v, x);
}

// Normal and tangential parts of the relative contact velocity.  Both come
// from FP64 inputs: the velocity difference cancels when two bodies move
// together, and the tangential part cancels when the motion is mostly normal,
// where a normal rounded to FP32 would tilt it by 6e-8 rad.
struct RelVel { float3 normal, vn, vt; };
__device__ __forceinline__ RelVel splitRelVel(d3 nD, d3 tmpV) {
  d3 vn = nD * dot(tmpV, nD);
  d3 vt = tmpV - vn;
  RelVel r;
  r.normal = f3((float)nD.x, (float)nD.y, (float)nD.z);
  r.vn = f3((float)vn.x, (float)vn.y, (float)vn.z);
  r.vt = f3((float)vt.x, (float)vt.y, (float)vt.z);
  return r;
}

// HookeMemory force in FP32, seen from p0 (same structure as hodc64); rv is
// the decomposed relative velocity of p0 with respect to p1 at the contact
// point and wrel = w0 - w1.
__device__ __forceinline__ void hodc32(ModelDesc const& m, float kn, float beta, float dt,
                                       float3 pen, RelVel const& rv, float3 wrel, float m0, float rad0,
                                       float m1, float rad1, bool existed, float3& kd,
                                       float3& pn, float3& sp, float3& f, float3& mr,
                                       float& cond) {
  const float3 normal = rv.normal;
  const float3 v_n = rv.vn;
  const float3 v_t = rv.vt;
  float avmass = 1.f / (1.f / m0 + 1.f / m1);
  float gamman = -2.f * beta * sqrtf(avmass * kn);
  float3 delFN = kn * pen - gamman * v_n;
  float normFN = normf3(delFN);
  float etat = m.etat == -1. ? -beta * sqrtf(kn / avmass) : (float)m.etat;
  float gammat = 2.f * etat * avmass;
  float3 viscousFT = -gammat * v_t;
  rot32 qrot;
  if (!existed) { kd = f3(0.f, 0.f, 0.f); sp = f3(0.f, 0.f, 0.f); }
  else {
    qrot = rotFromTo(pn, normal);
    kd = rotate(qrot, kd);
  }
  float kt = (float)m.kt;
  kd = kd + (dt * kt) * v_t;
  pn = normal;
  // computeTangentialVector
  float3 tij;
  float nut = normf3(v_t);
  float epst = (float)m.epst;
  if (nut > 0.001f) tij = (-1.f / nut) * v_t;
  else {
    float3 s = kd + gammat * v_t;
    float ns = normf3(s);
    if ((normf3(kd) > epst || normf3(gammat * v_t) > epst) && ns > epst) tij = (-1.f / ns) * s;
    else tij = f3(0.f, 0.f, 0.f);
  }
  float3 trial = -kd + viscousFT;
  float normFT = normf3(trial);
  float muc = (float)m.muc;
  float3 delFT;
  if (normFT <= muc * normFN) delFT = normFT * tij;
  else {
    if (kt != 0.f) kd = ((-muc * normFN) * tij + viscousFT) * (1.f / kt);
    delFT = (muc * normFN) * tij;
  }
  mr = f3(0.f, 0.f, 0.f);
  if (m.rolling) {
    float mur = (float)m.mur;
    float Req = 1.f / (1.f / rad0 + 1.f / rad1);
    float kr = 3.f * kn * mur * mur * Req * Req;
    float etar = 3.f * gamman * mur * mur * Req * Req;
    float maxM = mur * Req * normFN;
    if (existed) sp = rotate(qrot, sp);
    sp = sp - (kr * dt) * wrel;
    float nM = normf3(sp);
    if (nM > maxM) sp = sp * (maxM / nM);
    mr = sp - ((float)m.etarpf * etar) * wrel;
  }
  f = delFN + delFT;
  // size of the terms against the result: FP32 rounding of the terms is
  // amplified by this factor in f
  cond = (kn * normf3(pen) + fabsf(gamman) * normf3(v_n) + normf3(kd) + normf3(viscousFT)) /
         normf3(f);
}

__device__ __forceinline__ float3 tof(d3 a) { return f3((float)a.x, (float)a.y, (float)a.z); }

__device__ __forceinline__ void loadHistF(HistTable const& t, int slot, float3& kd, float3& pn, float3& sp) {
  const float* v = static_cast<const float*>(t.vals) + 9 * (size_t)slot;
  kd = f3(v[0], v[1], v[2]); pn = f3(v[3], v[4], v[5]); sp = f3(v[6], v[7], v[8]);
}
__device__ __forceinline__ void storeHistF(HistTable const& t, int slot, float3 kd, float3 pn, float3 sp) {
  float* v = static_cast<float*>(t.vals) + 9 * (size_t)slot;
  v[0] = kd.x; v[1] = kd.y; v[2] = kd.z; v[3] = pn.x; v[4] = pn.y; v[5] = pn.z;
  v[6] = sp.x; v[7] = sp.y; v[8] = sp.z;
}

// Hooke law (no tangential memory) in FP32, seen from p0 (same structure as
// hooke64).  lev0 / lev1 are the contact point relative to p0 / p1; w0, w1
// the space-fixed angular velocities.
__device__ __forceinline__ void hooke32(ModelDesc const& m, float kn, float beta, float3 pen,
                                        RelVel const& rv, float3 w0, float3 w1, float3 lev0,
                                        float3 lev1, float m0, float rad0, float m1, float rad1,
                                        float3& f, float3& mr, float& cond) {
  const float3 v_n = rv.vn;
  const float3 v_t = rv.vt;
  float avmass = 1.f / (1.f / m0 + 1.f / m1);
  float gamman = -2.f * beta * sqrtf(avmass * kn);
  float3 delFN = kn * pen - gamman * v_n;
  float normFN = normf3(delFN);
  float etat = m.etat == -1. ? -beta * sqrtf(kn / avmass) : (float)m.etat;
  float gammat = 2.f * etat * avmass;
  float3 delFT = -gammat * v_t;
  float fn = (float)m.muc * normFN;
  if (fn < normf3(delFT)) {
    float nvt = normf3(v_t);
    delFT = nvt > 1.e-10f ? (-fn / nvt) * v_t : f3(0.f, 0.f, 0.f);
  }
  mr = f3(0.f, 0.f, 0.f);
  if (m.kr != 0.) {
    float3 wrel = w0 - w1;
    float nwr = normf3(wrel);
    // w0 x (x0 - pc) - w1 x (x1 - pc) = w1 x lev1 - w0 x lev0
    float nwt = normf3(crossf(w1, lev1) - crossf(w0, lev0));
    if (nwr > 1.e-10f) {
      float Req = 1.f / (1.f / rad0 + 1.f / rad1);
      mr = (-((float)m.kr * Req * normFN * nwt / nwr)) * wrel;
    }
  }
  f = delFN + delFT;
  cond = (kn * normf3(pen) + fabsf(gamman) * normf3(v_n) + fabsf(gammat) * normf3(v_t)) /
         normf3(f);
}

// A contact whose FP32 force carries more than this amplification of FP32
// rounding (about 6e-8 times it, relative to |f|) is re-evaluated in FP64:
// the result then stays within ~1e-6 of the FP64 force per contact.
constexpr float kReevalCond = 16.f;

struct Body64 { d3 x, v, w; double m, rad; };
__device__ __forceinline__ float3 tof3(d3 a) { return make_float3((float)a.x, (float)a.y, (float)a.z); }
__device__ __forceinline__ d3 tod3(float3 a) { return mk((double)a.x, (double)a.y, (double)a.z); }

// FP64 evaluation of one contact from the loaded FP32 history (kd0, pn0,
// sp0).
__device__ __forceinline__ void contactLaw64(ModelDesc const& m, double dt, Contact64 const& ct,
                                          Body64 const& b0, Body64 const& b1, bool existed,
                                          float3 kd0, float3 pn0, float3 sp0, float3& kd,
                                          float3& pn, float3& sp, float3& f, float3& mr) {
  d3 f64, mr64;
  if (m.memory) {
    d3 kdd = tod3(kd0), pnd = tod3(pn0), spd = tod3(sp0);
    hodc64(m, dt, ct.point, ct.overlap, b0.x, b0.v, b0.w, b0.m, b0.rad, b1.x, b1.v, b1.w, b1.m,
           b1.rad, existed, kdd, pnd, spd, f64, mr64);
    kd = tof3(kdd); pn = tof3(pnd); sp = tof3(spd);
  } else {
    hooke64(m, ct.point, ct.overlap, b0.x, b0.v, b0.w, b0.m, b0.rad, b1.x, b1.v, b1.w, b1.m,
            b1.rad, f64, mr64);
  }
  f = tof3(f64);
  mr = tof3(mr64);
}

// One contact's force law seen from b0 (force on b0 returned in f, rolling
// moment in mr), evaluated in FP32 from FP64 geometry and velocities, and
// again in FP64 from the same inputs when the FP32 result is ill-conditioned
// (a force that is a small difference of large terms: a contact that is
// about to open, a rebound).  kd/pn/sp hold the loaded history on entry and
// the updated history on exit.
__device__ __forceinline__ void contactLaw32(ModelDesc const& m, double dt, Contact64 const& ct,
                                             Body64 const& b0, Body64 const& b1, bool existed,
                                             float3& kd, float3& pn, float3& sp, float3& f,
                                             float3& mr, int& reeval) {
  const d3 lev0 = ct.point - b0.x, lev1 = ct.point - b1.x;
  const d3 nD = ct.overlap / norm(ct.overlap);
  // relative velocity at the contact point (Particle::getVelocityAtPoint)
  const d3 tmpV = (b0.v + cross(b0.w, lev0)) - (b1.v + cross(b1.w, lev1));
  const RelVel rv = splitRelVel(nD, tmpV);
  const float3 pen = tof3(ct.overlap);
  const float3 kd0 = kd, pn0 = pn, sp0 = sp;
  float cond;
  if (m.memory)
    hodc32(m, (float)m.kn, (float)m.beta, (float)dt, pen, rv, tof3(b0.w - b1.w), (float)b0.m,
           (float)b0.rad, (float)b1.m, (float)b1.rad, existed, kd, pn, sp, f, mr, cond);
  else
    hooke32(m, (float)m.kn, (float)m.beta, pen, rv, tof3(b0.w), tof3(b1.w), tof3(lev0),
            tof3(lev1), (float)b0.m, (float)b0.rad, (float)b1.m, (float)b1.rad, f, mr, cond);
  reeval = 0;
  if (!(cond <= kReevalCond)) {
    contactLaw64(m, dt, ct, b0, b1, existed, kd0, pn0, sp0, kd, pn, sp, f, mr);
    reeval = 1;
  }
}

// Lists a candidate when its bounding spheres are closer than the skin, with
// a relative margin of 4e-6 that covers the FP32 rounding of the test.
// kFill = false: returns the row length of slot t.  kFill = true: writes the
// row (its length known from the counting pass), orders it and returns its
// number of upper entries.
template <bool kFill>
__device__ __forceinline__ int listPairs32(DevState const& S, int t) {
  const int4 cc = S.cellc[t];
  GridDesc const& g = S.bgrids[cc.w];
  const float4 ha = S.offh[t];
  int* out = kFill ? S.pairs + S.pair_off[t] : nullptr;
  const int room = kFill ? S.npairs[t] : 0;
  int cnt = 0;
  const float4* __restrict__ offh = S.offh;
  const float ex = g.edge_f[0], ey = g.edge_f[1], ez = g.edge_f[2];
  forEachCandidate(S.cell_start, g, cc, [&](int u, int dcx, int dj, int dk, int sx, int sy, int sz) {
    if (u == t) return;
    const float4 hb = offh[u];
    // lower slot first, so both directions of a pair evaluate the same
    // expression and agree on the (conservative) decision
    const bool lo = t < u;
    const float4 h0 = lo ? ha : hb, h1 = lo ? hb : ha;
    const float s = lo ? 1.f : -1.f;
    float dx = fmaf(s * (float)dcx, ex, h1.x - h0.x);
    float dy = fmaf(s * (float)dj, ey, h1.y - h0.y);
    float dz = fmaf(s * (float)dk, ez, h1.z - h0.z);
    float R = (h0.w + h1.w + g.skin_f) * (1.f + 4.e-6f);
    if (dx * dx + dy * dy + dz * dz > R * R) return;
    if (kFill && cnt < room) out[cnt] = u | (shiftCode(sx, sy, sz) << 27);
    ++cnt;
  });
  if (!kFill) return cnt;
  return sortEntriesUpperFirst(out, min(cnt, room), S.id, S.id[t]);
}

__global__ void __launch_bounds__(256) k_pairs_count32(DevState S, const int* gate) {
  if (gate && !*gate) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  S.npairs[t] = rowLength(S, listPairs32<false>(S, t));
}

__global__ void __launch_bounds__(256) k_pairs_fill32(DevState S, const int* gate) {
  if (gate && !*gate) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = t < S.n && rowFits(S, t);
  const int nu = valid ? listPairs32<true>(S, t) : 0;
  // each pair once, from its lower ID, into the compact list of the filter
  appendUpperPairs(S, t, valid ? S.pairs + S.pair_off[t] : S.pairs, nu, S.status);
}

// One pair in the canonical orientation -- p0 (slot s0, the lower ID) at its
// own position, p1 at its periodic image seen from p0 -- with the exact
// narrow phase on the FP64 master positions, the FP32 law (FP64 when
// ill-conditioned) and the contact history (the new entry written when
// insert).  Returns true for a contact, with the force f on p0, the torques
// c0 = lev0 x f and c1 = lev1 x f of the lever arms from p0 and p1, and the
// rolling torque mr (rolling: the model has rolling resistance); delta gets
// the overlap (+inf without contact).  kConvex: some class is not a sphere,
// so the GJK narrow phase is compiled in (it is kept out of the sphere-only
// kernel, whose registers it would triple).
template <bool kConvex>
__device__ __forceinline__ bool evalPair32(DevState const& S, GridDesc const& g, int s0, int s1,
                                           int prio0, int prio1, int id0, int id1,
                                           TypeDesc const& tp0,
                                           TypeDesc const& tp1, d3 x0, d3 x1, d3 v0, d3 v1,
                                           d3 w0, d3 w1, bool insert, int& nlaw, int& nre,
                                           GjkTally& gjk, double& delta, float3& f, float3& c0,
                                           float3& c1, float3& mr, bool& rolling) {
  const int cap = S.cap;
  const unsigned tag = (unsigned)S.ctl[kCtlEpoch], tag_old = tag - 1u;
  // spheres: the history lookup's first probe (key and values) is read
  // before the narrow phase -- the key depends on the two IDs only -- so its
  // loads overlap the narrow phase
  const unsigned long long hkey = pairKey(min(id0, id1), max(id0, id1));
  uint32_t hslot = 0;
  unsigned long long hfirst = 0;
  float hv[9];
  if constexpr (!kConvex) {
    hslot = hashSlot(hkey, S.hist_old.log2cap);
    hfirst = S.hist_old.keys[hslot];
    const float* p = static_cast<const float*>(S.hist_old.vals) + 9 * (size_t)hslot;
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
                         c0v, c1v, true);
    if (ct.gjk_iters > 0) {
      recordVertex(S, tp0, s0, prio0, c0v);
      recordVertex(S, tp1, s1, prio1, c1v);
    }
    if (insert) gjk.add(ct.gjk_iters);   // each pair counted once
  }
  delta = ct.contact && ct.dist < 0. ? ct.dist : __longlong_as_double(0x7ff0000000000000ll);
  if (!ct.contact || !(ct.dist < 0.)) return false;
  if (ct.error) raise(S.status, kErrContactOverlap);
  // the force law from here on is FP32 (FP64 when ill-conditioned)
  const float3 lev0 = tof(ct.point - x0);
  const float3 lev1 = tof(ct.point - x1);
  ModelDesc const& m = S.models[g.model_base + tp0.mat * kMaxMat + tp1.mat];
  const Body64 b0{x0, v0, w0, tp0.mass, tp0.eqrad};
  const Body64 b1{x1, v1, w1, tp1.mass, tp1.eqrad};
  float3 kd = f3(0.f, 0.f, 0.f), pn = kd, sp = kd;
  int re;
  if (insert) ++nlaw;   // each pair counted once, by its lower ID
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
    if (old >= 0) {
      if (!kConvex && old == (int)hslot) {
        kd = f3(hv[0], hv[1], hv[2]); pn = f3(hv[3], hv[4], hv[5]); sp = f3(hv[6], hv[7], hv[8]);
      } else {
        loadHistF(S.hist_old, old, kd, pn, sp);
      }
      if (flip) { kd = -kd; pn = -pn; sp = -sp; }
    }
    contactLaw32(m, S.dt, ct, b0, b1, old >= 0, kd, pn, sp, f, mr, re);
    if (insert) {
      int slot = histInsert(S.hist_new, key, tag);
      if (slot < 0) raise(S.status, kErrHashFull);
      else if (flip) storeHistF(S.hist_new, slot, -kd, -pn, -sp);
      else storeHistF(S.hist_new, slot, kd, pn, sp);
    }
  } else {
    contactLaw32(m, S.dt, ct, b0, b1, false, kd, pn, sp, f, mr, re);
  }
  if (insert) nre += re;
  c0 = crossf(lev0, f);
  c1 = crossf(lev1, f);
  rolling = m.rolling != 0;
  if (!rolling) mr = f3(0.f, 0.f, 0.f);
  return true;
}

// One side of a pair in contact, as the leapfrog kernel adds it: the force
// on the row's particle with the evaluation tag in its fourth word, then the
// torque (lever arm x force, plus the rolling torque).
__device__ __forceinline__ void storeShare32(DevState const& S, int64_t entry, int tag, float3 f,
                                             float3 c) {
  float4* sh = static_cast<float4*>(S.share) + 2 * entry;
  sh[0] = make_float4(f.x, f.y, f.z, __int_as_float(tag));
  sh[1] = make_float4(c.x, c.y, c.z, 0.f);
}

// The wall contacts of particle t (near a wall per the contact filter): the
// geometry from the FP64 position, the force law in FP32 (FP64 when
// ill-conditioned); their sum is the particle's wall share.
template <bool kConvex>
__device__ __forceinline__ void wallsOf32(DevState const& S, int t, int tag, int& nlaw, int& nre,
                                          GjkTally& gjk, StatsTally& st) {
  const int cap = S.cap;
  const int inst = S.inst[t];
  GridDesc const& g = S.grids[inst];
  const unsigned utag = (unsigned)tag, tag_old = utag - 1u;
  const int ida = S.id[t];
  TypeDesc const& ta = S.types[S.type[t]];
  const d3 xt = ld3(S.x, cap, t), vt = ld3(S.v, cap, t), wt = ld3(S.w, cap, t);
  float3 Fw = f3(0.f, 0.f, 0.f), Tw = f3(0.f, 0.f, 0.f);
  bool any = false;
  // the particle's polyhedron vertex runs through its wall calls in order
  int curw = kConvex ? startVertex(S, ta, t) : 0;
  bool walls_gjk = false;
  for (int k = 0; k < g.wall_count; ++k) {
    WallDesc const& wd = S.walls[g.wall_begin + k];
    if (kConvex && ta.shape != 0) {
      // the shrunk body lies inside its circumscribed sphere and the shrunk
      // wall inside the wall's box: when the sphere is farther from the box
      // than the two crusts (with a margin far above the rounding), the
      // closest-point search would decide "no contact"; skip it
      double d2 = 0.;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double c = d == 0 ? xt.x : (d == 1 ? xt.y : xt.z);
        const double e = fabs(c - wd.centre[d]) - wd.extent[d];
        if (e > 0.) d2 += e * e;
      }
      const double lim = (ta.radius + ta.crust + wd.crust) * (1. + 1.e-9);
      if (d2 > lim * lim) {
        if (S.diag) S.wall_delta[(size_t)t * S.max_walls + k] = __longlong_as_double(0x7ff0000000000000ll);
        continue;
      }
    }
    int cw = 0;
    Contact64 ct = (!kConvex || ta.shape == 0)
        ? sphereWall64(xt, ta.radius, ta.crust, wd)
        : convexContact64(convexOf(ta, S), crustXForm(S.basis, cap, t, ta.scaling, xt),
                          ta.radius, ta.crust, convexOf(wd),
                          identityXForm(wd.scaling, mk(wd.centre[0], wd.centre[1], wd.centre[2])),
                          wd.radius, wd.crust, curw, cw, true);
    if (kConvex) gjk.add(ct.gjk_iters);
    if (kConvex && ct.gjk_iters > 0) walls_gjk = true;
    if (S.diag) S.wall_delta[(size_t)t * S.max_walls + k] = ct.contact ? ct.dist : __longlong_as_double(0x7ff0000000000000ll);
    if (ct.error) raise(S.status, kErrContactOverlap);
    if (!ct.contact || !(ct.dist < 0.)) continue;
    st.add(ct.dist);
    ModelDesc const& m = S.models[g.model_base + ta.mat * kMaxMat + wd.mat];
    const float3 lev0 = tof(ct.point - xt);
    const d3 zero = mk(0., 0., 0.);
    const Body64 b0{xt, vt, wt, ta.mass, ta.eqrad};
    const Body64 b1{mk(wd.centre[0], wd.centre[1], wd.centre[2]), zero, zero, 1.e20, wd.eqrad};
    float3 f, mr, kd = f3(0.f, 0.f, 0.f), pn = kd, sp = kd;
    int re;
    ++nlaw;
    if (m.memory) {
      const unsigned long long key = wallKey(ida, k);
      int old = histFind(S.hist_old, key, tag_old);
      if (old >= 0) loadHistF(S.hist_old, old, kd, pn, sp);
      contactLaw32(m, S.dt, ct, b0, b1, old >= 0, kd, pn, sp, f, mr, re);
      int slot = histInsert(S.hist_new, key, utag);
      if (slot < 0) raise(S.status, kErrHashFull);
      else storeHistF(S.hist_new, slot, kd, pn, sp);
    } else {
      contactLaw32(m, S.dt, ct, b0, b1, false, kd, pn, sp, f, mr, re);
    }
    nre += re;
    if (S.diag) {
      double* fd = S.wall_force + 3 * ((size_t)t * S.max_walls + k);
      fd[0] = f.x; fd[1] = f.y; fd[2] = f.z;
    }
    Fw = Fw + f;
    Tw = Tw + crossf(lev0, f);
    if (m.rolling) Tw = Tw + mr;
    any = true;
  }
  if (walls_gjk) recordVertex(S, ta, t, kWallPriority, curw);
  if (!any) return;
  float4* ws = static_cast<float4*>(S.wshare) + 2 * (size_t)t;
  ws[0] = make_float4(Fw.x, Fw.y, Fw.z, 0.f);
  ws[1] = make_float4(Tw.x, Tw.y, Tw.z, 0.f);
  atomicOr(reinterpret_cast<unsigned*>(&contactFlags(S)[t]), kNearWall);
}

// One pair kept by the contact filter (compact pair c), seen from its lower
// ID, which writes the history: exact narrow phase, force law, and for a
// contact its two shares written into the rows of both partners and their
// entry bits set.  The leapfrog kernel adds each particle's shares in row
// order, so the sums are deterministic and need no float atomics.
template <bool kConvex>
__device__ __forceinline__ void pairItem32(DevState const& S, int c, int tag, int& nlaw, int& nre,
                                           GjkTally& gjk, StatsTally& st) {
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
  float3 f, c0, c1, mr;
  double dl;
  bool rolling;
  const bool hit = evalPair32<kConvex>(
      S, g, a, b, pa, pb, flip ? idu : idt, flip ? idt : idu, S.types[flip ? tyu : tyt], S.types[flip ? tyt : tyu],
      flip ? xu : xt, flip ? xt + (-shift) : xu + shift, vt, vu, wt, wu, true, nlaw, nre, gjk, dl, f, c0, c1, mr, rolling);
  const int64_t rt = (int64_t)offt + et, ru = (int64_t)offu + eu;
  // force on t (the lower ID) and the two torques
  const float3 mt = rolling ? mr : f3(0.f, 0.f, 0.f);
  const float3 ft = flip ? -f : f;
  const float3 tt = flip ? -(c1 + mt) : c0 + mt, tu = flip ? c0 + mt : -(c1 + mt);
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
  storeShare32(S, rt, tag, ft, tt);
  atomicOr(reinterpret_cast<unsigned*>(&flags[t]), entryBit(et));
  if (eu != 0xFFFF) {
    storeShare32(S, ru, tag, -ft, tu);
    atomicOr(reinterpret_cast<unsigned*>(&flags[u]), entryBit(eu));
  }
}

// First pass over the kept pairs that were not in contact at the last
// evaluation (FP32-split with non-spherical classes: the back of the kept
// list): the bounding-sphere test and the first iteration of the
// closest-point search (separatedAtFirst), in a kernel without the
// search's simplex and the force law.  A pair they prove apart ends here
// with what the pair kernel would have recorded for it -- no contact, its
// GJK call and the polyhedron vertices its search reached (recordVertex) --
// and the others are listed in kept2 for the pair kernel, which then runs
// their full searches in warps of their own instead of beside searches that
// stop at once.  Pairs of two spheres go to the pair kernel as they are.
__device__ __forceinline__ bool apartAtFirst(DevState const& S, int c, GjkTally& gjk) {
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
  // the orientation and priorities of pairItem32
  const bool flip = referenceFlip(g, xt, xu, sh);
  const int a = flip ? u : t, b = flip ? t : u;
  const int pa = min((flip ? eu : et) + 1, kWallPriority - 1),
            pb = min((flip ? et : eu) + 1, kWallPriority - 1);
  TypeDesc const& tp0 = S.types[S.type[a]];
  TypeDesc const& tp1 = S.types[S.type[b]];
  if (tp0.shape == 0 && tp1.shape == 0) return false;
  const d3 x0 = flip ? xu : xt, x1 = flip ? xt + (-shift) : xu + shift;
  const XForm64 a2w = crustXForm(S.basis, cap, a, tp0.scaling, x0);
  const XForm64 b2w = crustXForm(S.basis, cap, b, tp1.scaling, x1);
  // convexContact64's bounding-sphere test, then its search's first
  // iteration with the same separation margin
  if (norm(a2w.o - b2w.o) < tp0.radius + tp1.radius) {
    int c0v = startVertex(S, tp0, a), c1v = startVertex(S, tp1, b);
    const double sep = (tp0.crust + tp1.crust) * (1. + 1.e-9);
    if (!separatedAtFirst(convexOf(tp0, S), a2w, convexOf(tp1, S), b2w, c0v, c1v, sep))
      return false;
    recordVertex(S, tp0, a, pa, c0v);
    recordVertex(S, tp1, b, pb, c1v);
    gjk.add(1);
  }
  if (S.diag) {
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    S.pair_delta[(int64_t)S.pair_off[t] + et] = inf;
    if (eu != 0xFFFF) S.pair_delta[(int64_t)S.pair_off[u] + eu] = inf;
  }
  return true;
}

__global__ void __launch_bounds__(128) k_pairsep32(DevState S) {
  pdlWait();      // the contact filter's lists
  pdlTrigger();   // the pair kernel may be scheduled; it waits for this one
  const int nc = S.ctl[kCtlKeptCold];
  const int* cold = S.kept + S.pair_cap / 2;   // listed downwards
  const int lane = threadIdx.x & 31;
  GjkTally gjk;
  for (int j0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); j0 < nc;
       j0 += gridDim.x * blockDim.x) {   // warp-uniform
    const int j = j0 + lane;
    int c = 0;
    bool open = false;
    if (j < nc) {
      c = cold[-j];
      open = !apartAtFirst(S, c, gjk);
    }
    const unsigned m = __ballot_sync(0xffffffffu, open);
    if (m) {
      int base = 0;
      if (lane == 0) base = atomicAdd(S.ctl + kCtlKept2, __popc(m));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (open) S.kept2[base + __popc(m & ((1u << lane) - 1u))] = c;
    }
  }
  gjk.flush(S.gjk_counts);
}

// The pair kernel of an evaluation, one thread per item over a persistent
// grid: first the pairs the contact filter kept, then the particles near a
// wall.  Its trigger comes after its wait, so the leapfrog kernel, which
// starts at the trigger, sees the filter's candidate marks complete.
template <bool kConvex>
__global__ void __launch_bounds__(128) k_pairlaw32(DevState S) {
  pdlWait();      // the contact filter's lists
  pdlTrigger();   // the leapfrog kernel may start; its candidates wait for this kernel
  // the pairs in contact at the last evaluation (all kept pairs, without
  // non-spherical classes), then those k_pairsep32 left undecided, then the
  // particles near a wall
  const int nh = S.ctl[kCtlKept], n2 = kConvex ? S.ctl[kCtlKept2] : 0, nw = S.ctl[kCtlWork];
  const int nk = nh + n2;
  const int tag = S.ctl[kCtlEpoch];
  const int stride = gridDim.x * blockDim.x;
  int nlaw = 0, nre = 0;   // contacts evaluated / re-evaluated in FP64
  GjkTally gjk;
  StatsTally st;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nk + nw; i += stride) {
    if (i < nh) pairItem32<kConvex>(S, S.kept[i], tag, nlaw, nre, gjk, st);
    else if (i < nk) pairItem32<kConvex>(S, S.kept2[i - nh], tag, nlaw, nre, gjk, st);
    else wallsOf32<kConvex>(S, S.work[i - nk], tag, nlaw, nre, gjk, st);
  }
  // warp-aggregated counters (every lane of the warp reaches this point)
  const int wl = __reduce_add_sync(0xffffffffu, nlaw), wr = __reduce_add_sync(0xffffffffu, nre);
  if ((threadIdx.x & 31) == 0 && wl) {
    atomicAdd(S.law_counts, (unsigned long long)wl);
    if (wr) atomicAdd(S.law_counts + 1, (unsigned long long)wr);
  }
  if constexpr (kConvex) gjk.flush(S.gjk_counts);
  st.flush(S.cstats, tag);
}

}  // namespace

void launch_pairs32(DevState const& S, const int* gate, int fill, cudaStream_t st) {
  if (!S.n) return;
  if (fill) k_pairs_fill32<<<(S.n + 255) / 256, 256, 0, st>>>(S, gate);
  else k_pairs_count32<<<(S.n + 255) / 256, 256, 0, st>>>(S, gate);
}
void launch_pairsep32(DevState const& S, cudaStream_t st) {
  if (!S.n || !S.any_convex) return;
  // one wave: three blocks per multiprocessor fit (140 registers); measured
  // on the convex pour, 8 per multiprocessor took 59.6 us a step and an
  // empty launch cost the pour at rest 1.7 us more, 2 took 70.5 us
  launchAfterPrevious(k_pairsep32, 3 * S.nsm, 128, st, S);
}
void launch_pairlaw32(DevState const& S, cudaStream_t st) {
  if (!S.n) return;
  const int grid = (S.forces_bps > 0 ? S.forces_bps : 4) * S.nsm;
  if (S.any_convex) launchAfterPrevious(k_pairlaw32<true>, grid, 128, st, S);
  else launchAfterPrevious(k_pairlaw32<false>, grid, 128, st, S);
}

}  // namespace gdem
