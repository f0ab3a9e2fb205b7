// gdem_adjoint.cu -- gradients of a trajectory loss for calibration: a
// hand-written adjoint of the DEM step for spheres in a walled box.
//
// Forward model (one step, spheres, h = dt / 2; the production FP64 step in
// exact arithmetic: for a sphere the body-frame SSP-RK3 update rotated back
// to the space frame is w + T h / I):
//   vh = v_n + F_n h / m,  wh = w_n + T_n h / I,  x_{n+1} = x_n + vh dt,
//   (F, T, history)_{n+1} = Phi(x_{n+1}, vh, wh, history_n; kn, en, muc),
//   v_{n+1} = vh + F_{n+1} h / m,  w_{n+1} = wh + T_{n+1} h / I,
// with Phi the sphere-sphere and sphere-wall contact geometry and the Hooke /
// HookeMemory law of gdem_adjoint_law.cuh (tangential spring carried from
// step to step), and (F, T)_0 = Phi(x_0, v_0, w_0) with the cumulative spring
// then zeroed (Grains.cpp:168-173).
//
// Loss: L = sum_i |x_i(N) - x*_i|^2 + |v_i(N) - v*_i|^2.
//
// Reverse sweep: the transposed leapfrog per particle, and per contact the
// transposed Jacobian of Phi applied to the adjoints of its outputs.  Each
// Jacobian column is one evaluation of the contact law on Dual<1> numbers
// seeded on that input (its own position, half-step velocities, the
// tangential history and, once per contact, kn, en, muc).  States are
// recomputed from checkpoints taken every K steps.  A forward run on
// Dual<3> numbers seeded on (kn, en, muc) gives the forward-mode gradient
// that checks the parameter part of the adjoint.
//
// Pair search: a linked-cell grid over the domain box (cells at least the
// largest contact distance wide, coordinates outside the box clamped into the
// edge cells) is rebuilt at every force evaluation; each particle collects
// the partners of its 27 cells whose centres pass the contact-distance test
// and takes them in ascending index, the order of an all-pairs loop, so the
// sums and lists do not depend on the grid.
//
// Scope: spheres (any number of classes), box walls, Hooke / HookeMemory
// without rolling resistance, non-periodic domains.  kt and the other law
// parameters come from the XML; kn, en and muc of every contact model are
// replaced by the calibrated values.  MotionError and grid checks are not
// made here (the forward model of a calibration is the step's own).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/grains_b200.h"
#include "gdem_adjoint_law.cuh"
#include "gdem_setup.h"

namespace gdem {
namespace {

constexpr int kAdjCap = 32;      // contacts per particle
constexpr int kAdjWalls = 8;     // walls

struct AdjCheck : std::runtime_error {
  using std::runtime_error::runtime_error;
};
#define ACK(call)                                                                    \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) throw AdjCheck(std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Per-class and per-wall constants on the device.
struct AdjTables {
  const TypeDesc* types;
  const WallDesc* walls;
  const ModelDesc* models;
  int nwalls;
  double dt;
};

template <typename T>
__device__ __forceinline__ V3<T> ldv(const T* p, size_t i) {
  return v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}
template <typename T>
__device__ __forceinline__ void stv(T* p, size_t i, V3<T> a) {
  p[3 * i] = a.x; p[3 * i + 1] = a.y; p[3 * i + 2] = a.z;
}
__device__ __forceinline__ V3<double> ldd(const double* p, size_t i) {
  return v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}
template <typename T>
__device__ __forceinline__ V3<T> promote(V3<double> a) {
  return v3(Scal<T>::make(a.x), Scal<T>::make(a.y), Scal<T>::make(a.z));
}

__device__ __forceinline__ ModelDesc const& modelOf(AdjTables const& A, int ma, int mb) {
  return A.models[ma * kMaxMat + mb];
}

// Slot of partner u in particle t's list (of the previous step), or -1.
template <typename L>
__device__ __forceinline__ int findSlotT(L const& lists, int t, int u) {
  const int np = lists.npart[t];
  for (int k = 0; k < np; ++k)
    if (lists.partner[(size_t)t * kAdjCap + k] == u) return k;
  return -1;
}

// Outputs of one pair contact (a = lower index, b = higher index): the force
// and torque it adds to a and to b, the new spring and normal.
template <typename T>
struct PairY {
  V3<T> fa, ta, fb, tb, kd, pn;
  bool contact;
};
template <typename T>
struct PairIn {
  V3<T> xa, xb, va, vb, wa, wb, kd, pn;
  T kn, en, muc;
};

template <typename T>
__device__ __forceinline__ PairY<T> pairContact(AdjTables const& A, PairIn<T> const& in,
                                                TypeDesc const& ta, TypeDesc const& tb,
                                                bool existed) {
  PairY<T> y;
  V3<T> pc, pen;
  y.contact = sphereSphereG(in.xa, ta.radius, in.xb, tb.radius, pc, pen);
  if (!y.contact) return y;
  ModelDesc const& m = modelOf(A, ta.mat, tb.mat);
  LawOut<T> o = contactLaw(m, A.dt, in.kn, in.en, in.muc, pc, pen, in.xa, in.va, in.wa, ta.mass,
                           in.xb, in.vb, in.wb, tb.mass, existed, in.kd, in.pn);
  y.fa = o.f;
  y.ta = vcross(pc - in.xa, o.f);
  y.fb = -o.f;
  y.tb = vcross(pc - in.xb, -o.f);
  y.kd = o.kd;
  y.pn = o.pn;
  return y;
}

template <typename T>
struct WallY {
  V3<T> f, t, kd, pn;
  bool contact;
};
template <typename T>
struct WallIn {
  V3<T> x, v, w, kd, pn;
  T kn, en, muc;
};

template <typename T>
__device__ __forceinline__ WallY<T> wallContact(AdjTables const& A, WallIn<T> const& in,
                                                TypeDesc const& tp, WallDesc const& wd,
                                                bool existed) {
  WallY<T> y;
  V3<T> pc, pen;
  y.contact = sphereWallG(in.x, tp.radius, wd, pc, pen);
  if (!y.contact) return y;
  ModelDesc const& m = modelOf(A, tp.mat, wd.mat);
  const V3<T> zero = vconst<T>(0., 0., 0.);
  LawOut<T> o = contactLaw(m, A.dt, in.kn, in.en, in.muc, pc, pen, in.x, in.v, in.w, tp.mass,
                           vconst<T>(wd.centre[0], wd.centre[1], wd.centre[2]), zero, zero, 1.e20,
                           existed, in.kd, in.pn);
  y.f = o.f;
  y.t = vcross(pc - in.x, o.f);
  y.kd = o.kd;
  y.pn = o.pn;
  return y;
}

template <typename T>
struct ListsT {
  int* partner;
  int* npart;
  T* kd;
  T* pn;
  int* wflag;
  T* wkd;
  T* wpn;
};

// ---------------------------------------------------------- pair search --
// The linked-cell grid of the forward model: cell (i, j, k) has key
// (k nb1 + j) nb0 + i; start[c] .. start[c + 1] index its particles in items.
struct AdjGrid {
  double org[3], inv_edge[3];
  int nb[3];
  int ncells;
  const int* cell;    // cell key of each particle
  const int* start;   // ncells + 1 offsets
  const int* items;   // particles in cell order
};

__device__ __forceinline__ int adjCellIndex(AdjGrid const& g, int d, double x) {
  const double f = floor((x - g.org[d]) * g.inv_edge[d]);
  return f < 0. ? 0 : (f >= (double)g.nb[d] ? g.nb[d] - 1 : (int)f);
}

template <typename T>
__global__ void k_adj_bin(int n, AdjGrid g, const T* x, int* cell, int* count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = adjCellIndex(g, 0, val(x[3 * t]));
  const int j = adjCellIndex(g, 1, val(x[3 * t + 1]));
  const int k = adjCellIndex(g, 2, val(x[3 * t + 2]));
  const int c = (k * g.nb[1] + j) * g.nb[0] + i;
  cell[t] = c;
  atomicAdd(&count[c], 1);
}

// Exclusive scan of the cell counts by one block of 1024 threads, chunk by
// chunk; start[ncells] receives the total.
__global__ void __launch_bounds__(1024) k_adj_scan(int ncells, const int* count, int* start) {
  __shared__ int warp_sum[32];
  __shared__ int carry_s;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (int base = 0; base < ncells; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < ncells ? count[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int y = warp_sum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int z = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= o) y += z;
      }
      warp_sum[lane] = y;
    }
    __syncthreads();
    const int carry = carry_s;
    const int before = wid > 0 ? warp_sum[wid - 1] : 0;
    if (i < ncells) start[i] = carry + before + x - v;
    __syncthreads();
    if (threadIdx.x == 0) carry_s = carry + warp_sum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) start[ncells] = carry_s;
}

__global__ void k_adj_place(int n, const int* cell, const int* start, int* fill, int* items) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int c = cell[t];
  items[start[c] + atomicAdd(&fill[c], 1)] = t;
}

// ------------------------------------------------------------- forward --
// Contact forces and the new contact lists at one step.  vel/omg are the
// velocities the law sees (half-step ones, or the initial ones at the
// leapfrog start).  zero_spring: the leapfrog start zeroes the cumulative
// spring after the evaluation.
template <typename T>
__global__ void k_fwd_forces(int n, AdjTables A, AdjGrid G, const int* type, const T* x,
                             const T* vel, const T* omg, ListsT<T> prev, int has_prev,
                             ListsT<T> cur, T* F, T* Tq, T kn, T en, T muc, int zero_spring,
                             int* overflow) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  TypeDesc const& tp = A.types[type[t]];
  const V3<T> xt = ldv(x, t);
  V3<T> Ft = vconst<T>(tp.weight[0], tp.weight[1], tp.weight[2]);
  V3<T> Tt = vconst<T>(0., 0., 0.);
  const V3<T> zero = vconst<T>(0., 0., 0.);
  // partners whose centres pass the contact-distance test, from the 27
  // cells around t's, in ascending index
  int cand[kAdjCap];
  int nc = 0;
  {
    const int c = G.cell[t];
    const int ci = c % G.nb[0], cj = (c / G.nb[0]) % G.nb[1], ck = c / (G.nb[0] * G.nb[1]);
    for (int k3 = max(ck - 1, 0); k3 <= min(ck + 1, G.nb[2] - 1); ++k3)
      for (int j3 = max(cj - 1, 0); j3 <= min(cj + 1, G.nb[1] - 1); ++j3)
        for (int i3 = max(ci - 1, 0); i3 <= min(ci + 1, G.nb[0] - 1); ++i3) {
          const int cc = (k3 * G.nb[1] + j3) * G.nb[0] + i3;
          for (int e = G.start[cc]; e < G.start[cc + 1]; ++e) {
            const int u = G.items[e];
            if (u == t) continue;
            TypeDesc const& tu = A.types[type[u]];
            const V3<T> xu = ldv(x, u);
            const double dx = val(xu.x) - val(xt.x), dy = val(xu.y) - val(xt.y),
                         dz = val(xu.z) - val(xt.z);
            const double R = (tp.radius + tu.radius) * (1. + 1.e-9);
            if (dx * dx + dy * dy + dz * dz >= R * R) continue;
            if (nc < kAdjCap) cand[nc++] = u;
            else atomicOr(overflow, 1);
          }
        }
    for (int i = 1; i < nc; ++i) {
      const int u = cand[i];
      int j = i - 1;
      while (j >= 0 && cand[j] > u) {
        cand[j + 1] = cand[j];
        --j;
      }
      cand[j + 1] = u;
    }
  }
  int k = 0;
  for (int q = 0; q < nc; ++q) {
    const int u = cand[q];
    const int a = t < u ? t : u, b = t < u ? u : t;
    TypeDesc const& ta = A.types[type[a]];
    TypeDesc const& tb = A.types[type[b]];
    const int j = has_prev ? findSlotT(prev, t, u) : -1;
    const bool existed = j >= 0;
    PairIn<T> in;
    in.xa = ldv(x, a); in.xb = ldv(x, b);
    in.va = ldv(vel, a); in.vb = ldv(vel, b);
    in.wa = ldv(omg, a); in.wb = ldv(omg, b);
    in.kd = existed ? ldv(prev.kd, (size_t)t * kAdjCap + j) : zero;
    in.pn = existed ? ldv(prev.pn, (size_t)t * kAdjCap + j) : zero;
    in.kn = kn; in.en = en; in.muc = muc;
    PairY<T> y = pairContact(A, in, ta, tb, existed);
    if (!y.contact) continue;
    if (t == a) { Ft = Ft + y.fa; Tt = Tt + y.ta; }
    else { Ft = Ft + y.fb; Tt = Tt + y.tb; }
    if (k < kAdjCap) {
      const size_t sl = (size_t)t * kAdjCap + k;
      cur.partner[sl] = u;
      stv(cur.kd, sl, zero_spring ? zero : y.kd);
      stv(cur.pn, sl, y.pn);
      ++k;
    } else {
      atomicOr(overflow, 1);
    }
  }
  cur.npart[t] = k;
  for (int w = 0; w < A.nwalls; ++w) {
    WallDesc const& wd = A.walls[w];
    const size_t sl = (size_t)t * kAdjWalls + w;
    const bool existed = has_prev && prev.wflag[sl];
    WallIn<T> in;
    in.x = xt; in.v = ldv(vel, t); in.w = ldv(omg, t);
    in.kd = existed ? ldv(prev.wkd, sl) : zero;
    in.pn = existed ? ldv(prev.wpn, sl) : zero;
    in.kn = kn; in.en = en; in.muc = muc;
    WallY<T> y = wallContact(A, in, tp, wd, existed);
    cur.wflag[sl] = y.contact ? 1 : 0;
    if (!y.contact) continue;
    Ft = Ft + y.f;
    Tt = Tt + y.t;
    stv(cur.wkd, sl, zero_spring ? zero : y.kd);
    stv(cur.wpn, sl, y.pn);
  }
  stv(F, t, Ft);
  stv(Tq, t, Tt);
}

// Opening kick + drift: vh = v + F h / m, wh = w + T h / I, x' = x + vh dt.
template <typename T>
__global__ void k_fwd_move(int n, AdjTables A, const int* type, const T* x, const T* v,
                           const T* w, const T* F, const T* Tq, T* xo, T* vh, T* wh) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  TypeDesc const& tp = A.types[type[t]];
  const double h = 0.5 * A.dt;
  const V3<T> vv = ldv(v, t) + vscale(ldv(F, t), Scal<T>::make(h / tp.mass));
  const V3<T> ww = ldv(w, t) + vscale(ldv(Tq, t), Scal<T>::make(h / tp.inertia[0]));
  stv(vh, t, vv);
  stv(wh, t, ww);
  stv(xo, t, ldv(x, t) + vscale(vv, Scal<T>::make(A.dt)));
}

// Closing kick: v = vh + F h / m, w = wh + T h / I.
template <typename T>
__global__ void k_fwd_close(int n, AdjTables A, const int* type, const T* vh, const T* wh,
                            const T* F, const T* Tq, T* v, T* w) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  TypeDesc const& tp = A.types[type[t]];
  const double h = 0.5 * A.dt;
  stv(v, t, ldv(vh, t) + vscale(ldv(F, t), Scal<T>::make(h / tp.mass)));
  stv(w, t, ldv(wh, t) + vscale(ldv(Tq, t), Scal<T>::make(h / tp.inertia[0])));
}

// Per-particle squared error of positions and velocities.
template <typename T>
__global__ void k_fwd_loss(int n, const T* x, const T* v, const double* tx, const double* tv,
                           T* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const V3<T> dx = ldv(x, t) - promote<T>(ldd(tx, t));
  const V3<T> dv = ldv(v, t) - promote<T>(ldd(tv, t));
  out[t] = vdot(dx, dx) + vdot(dv, dv);
}

// ------------------------------------------------------------- reverse --
// Closing kick of step s, transposed: lvh = lv, lF += lv h / m, and the same
// for the rotation.
__global__ void k_bwd_close(int n, AdjTables A, const int* type, const double* lv,
                            const double* lw, double* lF, double* lT, double* lvh, double* lwh) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  TypeDesc const& tp = A.types[type[t]];
  const double h = 0.5 * A.dt;
  for (int d = 0; d < 3; ++d) {
    lvh[3 * t + d] = lv[3 * t + d];
    lF[3 * t + d] += lv[3 * t + d] * (h / tp.mass);
    lwh[3 * t + d] = lw[3 * t + d];
    lT[3 * t + d] += lw[3 * t + d] * (h / tp.inertia[0]);
  }
}

// Opening kick + drift of step s (from s - 1), transposed: the adjoints of
// x, v, w, F, T at s - 1 from those of x_s, vh, wh.
__global__ void k_bwd_move(int n, AdjTables A, const int* type, const double* lx,
                           const double* lvh, const double* lwh, double* lv, double* lw,
                           double* lF, double* lT) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  TypeDesc const& tp = A.types[type[t]];
  const double h = 0.5 * A.dt;
  for (int d = 0; d < 3; ++d) {
    const double g = lvh[3 * t + d] + lx[3 * t + d] * A.dt;
    lv[3 * t + d] = g;
    lF[3 * t + d] = g * (h / tp.mass);
    lw[3 * t + d] = lwh[3 * t + d];
    lT[3 * t + d] = lwh[3 * t + d] * (h / tp.inertia[0]);
  }
}

__device__ __forceinline__ double dotY(V3<double> l, V3<Dual<1>> y) {
  return l.x * y.x.d[0] + l.y * y.y.d[0] + l.z * y.z.d[0];
}
__device__ __forceinline__ void seedVec(V3<Dual<1>>& v, int c) {
  if (c == 0) v.x.d[0] = 1.;
  else if (c == 1) v.y.d[0] = 1.;
  else v.z.d[0] = 1.;
}
__device__ __forceinline__ V3<Dual<1>> lift(V3<double> a) { return promote<Dual<1>>(a); }

// Contact forces of step s, transposed.  For every contact of particle t the
// law is re-evaluated on Dual<1> numbers once per input of t's (position,
// velocity, angular velocity; the history it carried in; kn, en, muc once
// per contact, by its lower index), and the derivative of every output is
// contracted with that output's adjoint.  The history adjoints go to the
// slots of step s - 1 that supplied the history.
__global__ void k_bwd_forces(int n, AdjTables A, const int* type, const double* x,
                             const double* vel, const double* omg, ListsT<double> prev,
                             int has_prev, ListsT<double> cur, const double* lF, const double* lT,
                             const double* lkd, const double* lpn, const double* lwkd,
                             const double* lwpn, int spring_zeroed, double* lx, double* lvh,
                             double* lwh, double* lkd_prev, double* lpn_prev, double* lwkd_prev,
                             double* lwpn_prev, double* lp, double kn, double en, double muc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  TypeDesc const& tp = A.types[type[t]];
  double gx[3] = {0., 0., 0.}, gv[3] = {0., 0., 0.}, gw[3] = {0., 0., 0.};
  double gp[3] = {0., 0., 0.};
  const V3<double> zero = v3(0., 0., 0.);
  const int np = cur.npart[t];
  for (int k = 0; k < np; ++k) {
    const size_t sl = (size_t)t * kAdjCap + k;
    const int u = cur.partner[sl];
    const int a = t < u ? t : u, b = t < u ? u : t;
    TypeDesc const& ta = A.types[type[a]];
    TypeDesc const& tb = A.types[type[b]];
    const int j = has_prev ? findSlotT(prev, t, u) : -1;
    const bool existed = j >= 0;
    const size_t pj = (size_t)t * kAdjCap + (j >= 0 ? j : 0);
    PairIn<double> in;
    in.xa = ldd(x, a); in.xb = ldd(x, b);
    in.va = ldd(vel, a); in.vb = ldd(vel, b);
    in.wa = ldd(omg, a); in.wb = ldd(omg, b);
    in.kd = existed ? ldd(prev.kd, pj) : zero;
    in.pn = existed ? ldd(prev.pn, pj) : zero;
    const V3<double> lFa = ldd(lF, a), lTa = ldd(lT, a), lFb = ldd(lF, b), lTb = ldd(lT, b);
    const V3<double> lk = spring_zeroed ? zero : ldd(lkd, sl), ln = ldd(lpn, sl);
    const bool mine_a = t == a;
    const bool memory = modelOf(A, ta.mat, tb.mat).memory != 0;
    // inputs seeded by t: 0-8 own x, v, w; 9-14 history (when carried in);
    // 15-17 kn, en, muc (lower index only)
    const int nseed = 9 + ((existed && memory) ? 6 : 0) + (mine_a ? 3 : 0);
    double ghist[6] = {0., 0., 0., 0., 0., 0.};
    for (int s = 0; s < nseed; ++s) {
      int slot = s;
      if (s >= 9 && !(existed && memory)) slot = s + 6;
      PairIn<Dual<1>> din;
      din.xa = lift(in.xa); din.xb = lift(in.xb);
      din.va = lift(in.va); din.vb = lift(in.vb);
      din.wa = lift(in.wa); din.wb = lift(in.wb);
      din.kd = lift(in.kd); din.pn = lift(in.pn);
      din.kn = dconst<1>(kn); din.en = dconst<1>(en); din.muc = dconst<1>(muc);
      if (slot < 3) seedVec(mine_a ? din.xa : din.xb, slot);
      else if (slot < 6) seedVec(mine_a ? din.va : din.vb, slot - 3);
      else if (slot < 9) seedVec(mine_a ? din.wa : din.wb, slot - 6);
      else if (slot < 12) seedVec(din.kd, slot - 9);
      else if (slot < 15) seedVec(din.pn, slot - 12);
      else if (slot == 15) din.kn.d[0] = 1.;
      else if (slot == 16) din.en.d[0] = 1.;
      else din.muc.d[0] = 1.;
      PairY<Dual<1>> y = pairContact(A, din, ta, tb, existed);
      if (!y.contact) continue;
      const double g = dotY(lFa, y.fa) + dotY(lTa, y.ta) + dotY(lFb, y.fb) + dotY(lTb, y.tb) +
                       dotY(lk, y.kd) + dotY(ln, y.pn);
      if (slot < 3) gx[slot] += g;
      else if (slot < 6) gv[slot - 3] += g;
      else if (slot < 9) gw[slot - 6] += g;
      else if (slot < 15) ghist[slot - 9] += g;
      else gp[slot - 15] += g;
    }
    if (existed && memory) {
      for (int d = 0; d < 3; ++d) {
        lkd_prev[3 * pj + d] = ghist[d];
        lpn_prev[3 * pj + d] = ghist[3 + d];
      }
    }
  }
  for (int w = 0; w < A.nwalls; ++w) {
    const size_t sl = (size_t)t * kAdjWalls + w;
    if (!cur.wflag[sl]) continue;
    WallDesc const& wd = A.walls[w];
    const bool existed = has_prev && prev.wflag[sl];
    const bool memory = modelOf(A, tp.mat, wd.mat).memory != 0;
    WallIn<double> in;
    in.x = ldd(x, t); in.v = ldd(vel, t); in.w = ldd(omg, t);
    in.kd = existed ? ldd(prev.wkd, sl) : zero;
    in.pn = existed ? ldd(prev.wpn, sl) : zero;
    const V3<double> lFt = ldd(lF, t), lTt = ldd(lT, t);
    const V3<double> lk = spring_zeroed ? zero : ldd(lwkd, sl), ln = ldd(lwpn, sl);
    const int nseed = 9 + ((existed && memory) ? 6 : 0) + 3;
    double ghist[6] = {0., 0., 0., 0., 0., 0.};
    for (int s = 0; s < nseed; ++s) {
      int slot = s;
      if (s >= 9 && !(existed && memory)) slot = s + 6;
      WallIn<Dual<1>> din;
      din.x = lift(in.x); din.v = lift(in.v); din.w = lift(in.w);
      din.kd = lift(in.kd); din.pn = lift(in.pn);
      din.kn = dconst<1>(kn); din.en = dconst<1>(en); din.muc = dconst<1>(muc);
      if (slot < 3) seedVec(din.x, slot);
      else if (slot < 6) seedVec(din.v, slot - 3);
      else if (slot < 9) seedVec(din.w, slot - 6);
      else if (slot < 12) seedVec(din.kd, slot - 9);
      else if (slot < 15) seedVec(din.pn, slot - 12);
      else if (slot == 15) din.kn.d[0] = 1.;
      else if (slot == 16) din.en.d[0] = 1.;
      else din.muc.d[0] = 1.;
      WallY<Dual<1>> y = wallContact(A, din, tp, wd, existed);
      if (!y.contact) continue;
      const double g = dotY(lFt, y.f) + dotY(lTt, y.t) + dotY(lk, y.kd) + dotY(ln, y.pn);
      if (slot < 3) gx[slot] += g;
      else if (slot < 6) gv[slot - 3] += g;
      else if (slot < 9) gw[slot - 6] += g;
      else if (slot < 15) ghist[slot - 9] += g;
      else gp[slot - 15] += g;
    }
    if (existed && memory) {
      for (int d = 0; d < 3; ++d) {
        lwkd_prev[3 * sl + d] = ghist[d];
        lwpn_prev[3 * sl + d] = ghist[3 + d];
      }
    }
  }
  for (int d = 0; d < 3; ++d) {
    lx[3 * t + d] += gx[d];
    lvh[3 * t + d] += gv[d];
    lwh[3 * t + d] += gw[d];
    lp[3 * t + d] += gp[d];
  }
}

__global__ void k_bwd_seed(int n, const double* x, const double* v, const double* tx,
                           const double* tv, double* lx, double* lv) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  for (int d = 0; d < 3; ++d) {
    lx[3 * t + d] = 2. * (x[3 * t + d] - tx[3 * t + d]);
    lv[3 * t + d] = 2. * (v[3 * t + d] - tv[3 * t + d]);
  }
}

}  // namespace
}  // namespace gdem

// ------------------------------------------------------------------ host --
namespace gdem {
namespace {

template <typename T>
__global__ void k_promote(int n3, const double* a, T* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) out[i] = Scal<T>::make(a[i]);
}

inline int nblk(int n) { return (n + 127) / 128; }

// Sets the first derivative slot of one element to 1 (forward-mode seed).
template <typename T>
__global__ void k_seed(T* a, int i) {
  a[i].d[0] = 1.;
}
template <>
__global__ void k_seed<double>(double*, int) {}

struct AdjointSystem {
  AdjointSetup setup;
  AdjTables A{};
  int n = 0;
  int* d_type = nullptr;
  double *d_x0 = nullptr, *d_v0 = nullptr, *d_w0 = nullptr;
  int* d_overflow = nullptr;
  AdjGrid G{};
  int *d_cell = nullptr, *d_count = nullptr, *d_fill = nullptr, *d_start = nullptr,
      *d_items = nullptr;
  std::vector<void*> allocs;
  cudaStream_t st = nullptr;

  ~AdjointSystem() {
    for (void* p : allocs) cudaFree(p);
    if (st) cudaStreamDestroy(st);
  }
  template <typename T>
  T* alloc(size_t count) {
    void* p = nullptr;
    ACK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    allocs.push_back(p);
    return static_cast<T*>(p);
  }
  template <typename T>
  ListsT<T> allocLists() {
    ListsT<T> L;
    L.partner = alloc<int>((size_t)n * kAdjCap);
    L.npart = alloc<int>(n);
    L.kd = alloc<T>((size_t)n * kAdjCap * 3);
    L.pn = alloc<T>((size_t)n * kAdjCap * 3);
    L.wflag = alloc<int>((size_t)n * kAdjWalls);
    L.wkd = alloc<T>((size_t)n * kAdjWalls * 3);
    L.wpn = alloc<T>((size_t)n * kAdjWalls * 3);
    ACK(cudaMemsetAsync(L.npart, 0, n * sizeof(int), st));
    ACK(cudaMemsetAsync(L.wflag, 0, (size_t)n * kAdjWalls * sizeof(int), st));
    return L;
  }
  template <typename T>
  void copyLists(ListsT<T> const& dst, ListsT<T> const& src) {
    auto cp = [&](void* d, const void* s, size_t bytes) {
      ACK(cudaMemcpyAsync(d, s, bytes, cudaMemcpyDeviceToDevice, st));
    };
    cp(dst.partner, src.partner, (size_t)n * kAdjCap * sizeof(int));
    cp(dst.npart, src.npart, (size_t)n * sizeof(int));
    cp(dst.kd, src.kd, (size_t)n * kAdjCap * 3 * sizeof(T));
    cp(dst.pn, src.pn, (size_t)n * kAdjCap * 3 * sizeof(T));
    cp(dst.wflag, src.wflag, (size_t)n * kAdjWalls * sizeof(int));
    cp(dst.wkd, src.wkd, (size_t)n * kAdjWalls * 3 * sizeof(T));
    cp(dst.wpn, src.wpn, (size_t)n * kAdjWalls * 3 * sizeof(T));
  }

  void create(std::string const& xml) {
    readAdjointSetup(xml, setup);
    for (auto const& t : setup.types)
      if (t.shape != 0) throw std::runtime_error("the adjoint handles spheres only");
    for (int d = 0; d < 3; ++d)
      if (setup.periodic[d]) throw std::runtime_error("the adjoint handles non-periodic domains only");
    if ((int)setup.walls.size() > kAdjWalls) throw std::runtime_error("the adjoint handles at most 8 walls");
    for (auto const& m : setup.models)
      if (m.valid && m.rolling) throw std::runtime_error("the adjoint has no rolling resistance");
    ACK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    TypeDesc* dt = alloc<TypeDesc>(setup.types.size());
    WallDesc* dw = alloc<WallDesc>(setup.walls.size());
    ModelDesc* dm = alloc<ModelDesc>(kMaxMat * kMaxMat);
    ACK(cudaMemcpy(dt, setup.types.data(), setup.types.size() * sizeof(TypeDesc), cudaMemcpyHostToDevice));
    if (!setup.walls.empty())
      ACK(cudaMemcpy(dw, setup.walls.data(), setup.walls.size() * sizeof(WallDesc), cudaMemcpyHostToDevice));
    ACK(cudaMemcpy(dm, setup.models, sizeof(setup.models), cudaMemcpyHostToDevice));
    A.types = dt; A.walls = dw; A.models = dm;
    A.nwalls = (int)setup.walls.size();
    A.dt = setup.dt;
    d_overflow = alloc<int>(1);
    // pair-search grid: cells at least the largest contact distance wide,
    // at most 2^22 of them
    double rmax = 0.;
    for (auto const& t : setup.types) rmax = std::max(rmax, t.radius);
    const double emin = 2. * rmax * (1. + 1.e-6);
    for (int d = 0; d < 3; ++d) {
      const double L = setup.maxc[d] - setup.origin[d];
      G.nb[d] = (L > 0. && emin > 0.) ? std::max(1, (int)std::min(std::floor(L / emin), 1.e6)) : 1;
      G.org[d] = setup.origin[d];
    }
    while ((long long)G.nb[0] * G.nb[1] * G.nb[2] > (1ll << 22)) {
      int dm = 0;
      for (int d = 1; d < 3; ++d)
        if (G.nb[d] > G.nb[dm]) dm = d;
      G.nb[dm] = (G.nb[dm] + 1) / 2;
    }
    for (int d = 0; d < 3; ++d) {
      const double L = setup.maxc[d] - setup.origin[d];
      G.inv_edge[d] = L > 0. ? G.nb[d] / L : 0.;
    }
    G.ncells = G.nb[0] * G.nb[1] * G.nb[2];
    d_count = alloc<int>(G.ncells);
    d_fill = alloc<int>(G.ncells);
    d_start = alloc<int>((size_t)G.ncells + 1);
    G.start = d_start;
  }

  void setParticles(int64_t nn, const int* type, const double* x0, const double* v0,
                    const double* w0) {
    if (nn <= 0 || nn > (1 << 24)) throw std::runtime_error("particle count out of range");
    if (d_type) throw std::runtime_error("particles already set");
    n = (int)nn;
    for (int64_t i = 0; i < nn; ++i)
      if (type[i] < 0 || type[i] >= (int)setup.types.size())
        throw std::runtime_error("particle type out of range");
    d_type = alloc<int>(n);
    d_x0 = alloc<double>(3 * (size_t)n);
    d_v0 = alloc<double>(3 * (size_t)n);
    d_w0 = alloc<double>(3 * (size_t)n);
    d_cell = alloc<int>(n);
    d_items = alloc<int>(n);
    G.cell = d_cell;
    G.items = d_items;
    ACK(cudaMemcpy(d_type, type, n * sizeof(int), cudaMemcpyHostToDevice));
    ACK(cudaMemcpy(d_x0, x0, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    ACK(cudaMemcpy(d_v0, v0, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    if (w0) ACK(cudaMemcpy(d_w0, w0, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    else ACK(cudaMemset(d_w0, 0, 3 * (size_t)n * sizeof(double)));
  }

  // Frees the buffers allocated after a mark (one run's working memory).
  struct Scope {
    AdjointSystem* sys;
    size_t mark;
    explicit Scope(AdjointSystem* s) : sys(s), mark(s->allocs.size()) {}
    ~Scope() {
      if (sys->st) cudaStreamSynchronize(sys->st);
      for (size_t k = mark; k < sys->allocs.size(); ++k) cudaFree(sys->allocs[k]);
      sys->allocs.resize(mark);
    }
  };

  void checkOverflow() {
    int ov = 0;
    ACK(cudaMemcpyAsync(&ov, d_overflow, sizeof(int), cudaMemcpyDeviceToHost, st));
    ACK(cudaStreamSynchronize(st));
    if (ov) throw std::runtime_error("a particle has more than 32 contacts");
  }

  // State of one step of the forward model.
  template <typename T>
  struct State {
    T *x, *v, *w, *F, *Tq;
  };
  template <typename T>
  State<T> allocState() {
    State<T> S;
    S.x = alloc<T>(3 * (size_t)n); S.v = alloc<T>(3 * (size_t)n); S.w = alloc<T>(3 * (size_t)n);
    S.F = alloc<T>(3 * (size_t)n); S.Tq = alloc<T>(3 * (size_t)n);
    return S;
  }
  template <typename T>
  void copyState(State<T> const& d, State<T> const& s) {
    const size_t b = 3 * (size_t)n * sizeof(T);
    for (auto pr : {std::make_pair(d.x, s.x), std::make_pair(d.v, s.v), std::make_pair(d.w, s.w),
                    std::make_pair(d.F, s.F), std::make_pair(d.Tq, s.Tq)})
      ACK(cudaMemcpyAsync(pr.first, pr.second, b, cudaMemcpyDeviceToDevice, st));
  }

  // Contact forces at positions x (the grid is rebuilt from them first).
  template <typename T>
  void forces(const T* x, const T* vel, const T* omg, ListsT<T> const& prev, int has_prev,
              ListsT<T> const& cur, T* F, T* Tq, T kn, T en, T muc, int zero_spring) {
    ACK(cudaMemsetAsync(d_count, 0, (size_t)G.ncells * sizeof(int), st));
    ACK(cudaMemsetAsync(d_fill, 0, (size_t)G.ncells * sizeof(int), st));
    k_adj_bin<T><<<nblk(n), 128, 0, st>>>(n, G, x, d_cell, d_count);
    k_adj_scan<<<1, 1024, 0, st>>>(G.ncells, d_count, d_start);
    k_adj_place<<<nblk(n), 128, 0, st>>>(n, d_cell, d_start, d_fill, d_items);
    k_fwd_forces<T><<<nblk(n), 128, 0, st>>>(n, A, G, d_type, x, vel, omg, prev, has_prev, cur,
                                             F, Tq, kn, en, muc, zero_spring, d_overflow);
  }

  // Leapfrog start: forces at (x0, v0, w0) with no history, spring zeroed.
  template <typename T>
  void start(State<T>& S, ListsT<T>& L, T kn, T en, T muc, int seed_v0 = -1) {
    const int n3 = 3 * n;
    k_promote<T><<<nblk(n3), 128, 0, st>>>(n3, d_x0, S.x);
    k_promote<T><<<nblk(n3), 128, 0, st>>>(n3, d_v0, S.v);
    if (seed_v0 >= 0) k_seed<T><<<1, 1, 0, st>>>(S.v, seed_v0);
    k_promote<T><<<nblk(n3), 128, 0, st>>>(n3, d_w0, S.w);
    forces<T>(S.x, S.v, S.w, L, 0, L, S.F, S.Tq, kn, en, muc, 1);
    ACK(cudaGetLastError());
  }
  // One step: move into (xs, vh, wh), forces with history prev -> cur,
  // closing kick; S.x becomes xs.
  template <typename T>
  void advance(State<T>& S, T* xs, T* vh, T* wh, ListsT<T> const& prev, ListsT<T> const& cur,
               T kn, T en, T muc) {
    k_fwd_move<T><<<nblk(n), 128, 0, st>>>(n, A, d_type, S.x, S.v, S.w, S.F, S.Tq, xs, vh, wh);
    forces<T>(xs, vh, wh, prev, 1, cur, S.F, S.Tq, kn, en, muc, 0);
    k_fwd_close<T><<<nblk(n), 128, 0, st>>>(n, A, d_type, vh, wh, S.F, S.Tq, S.v, S.w);
    ACK(cudaMemcpyAsync(S.x, xs, 3 * (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, st));
    ACK(cudaGetLastError());
  }
  template <typename T>
  void lossOf(State<T> const& S, const double* tx, const double* tv, std::vector<T>& per) {
    double* dtx = alloc<double>(3 * (size_t)n);
    double* dtv = alloc<double>(3 * (size_t)n);
    T* out = alloc<T>(n);
    ACK(cudaMemcpyAsync(dtx, tx, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
    ACK(cudaMemcpyAsync(dtv, tv, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
    k_fwd_loss<T><<<nblk(n), 128, 0, st>>>(n, S.x, S.v, dtx, dtv, out);
    per.resize(n);
    ACK(cudaMemcpyAsync(per.data(), out, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    ACK(cudaStreamSynchronize(st));
  }

  // Forward run (and, with gradients requested, the reverse sweep) in FP64.
  void run(int nsteps, int K, const double* p, const double* tx, const double* tv, double* loss,
           double* x_out, double* v_out, double* dLdp, double* dLdv0) {
    if (nsteps < 1 || K < 1) throw std::runtime_error("nsteps and the checkpoint interval must be >= 1");
    if (!d_type) throw std::runtime_error("set the particles first");
    Scope scope(this);
    const bool grads = dLdp || dLdv0;
    if ((grads || loss) && (!tx || !tv)) throw std::runtime_error("the loss needs target x and v");
    const double kn = p[0], en = p[1], muc = p[2];
    const size_t n3 = 3 * (size_t)n;
    ACK(cudaMemsetAsync(d_overflow, 0, sizeof(int), st));
    State<double> S = allocState<double>();
    double* xs = alloc<double>(n3);
    double* vh = alloc<double>(n3);
    double* wh = alloc<double>(n3);
    ListsT<double> L[2] = {allocLists<double>(), allocLists<double>()};
    const int nseg = (nsteps + K - 1) / K;
    std::vector<State<double>> ck;
    std::vector<ListsT<double>> ckL;
    start(S, L[0], kn, en, muc);
    if (grads) {
      ck.push_back(allocState<double>()); ckL.push_back(allocLists<double>());
      copyState(ck[0], S); copyLists(ckL[0], L[0]);
    }
    for (int s = 1; s <= nsteps; ++s) {
      advance(S, xs, vh, wh, L[(s - 1) & 1], L[s & 1], kn, en, muc);
      if (grads && s % K == 0 && s < nsteps) {
        ck.push_back(allocState<double>()); ckL.push_back(allocLists<double>());
        copyState(ck.back(), S); copyLists(ckL.back(), L[s & 1]);
      }
    }
    checkOverflow();
    if (x_out) ACK(cudaMemcpy(x_out, S.x, n3 * sizeof(double), cudaMemcpyDeviceToHost));
    if (v_out) ACK(cudaMemcpy(v_out, S.v, n3 * sizeof(double), cudaMemcpyDeviceToHost));
    if (tx && tv) {
      std::vector<double> per;
      lossOf(S, tx, tv, per);
      double Ls = 0.;
      for (double a : per) Ls += a;
      if (loss) *loss = Ls;
    }
    if (!grads) return;
    // ------------------------------------------------------ reverse sweep
    double *lx = alloc<double>(n3), *lv = alloc<double>(n3), *lw = alloc<double>(n3);
    double *lF = alloc<double>(n3), *lT = alloc<double>(n3);
    double *lvh = alloc<double>(n3), *lwh = alloc<double>(n3), *lp = alloc<double>(n3);
    const size_t nh = (size_t)n * kAdjCap * 3, nwh = (size_t)n * kAdjWalls * 3;
    double *lkd[2], *lpn[2], *lwkd[2], *lwpn[2];
    for (int k = 0; k < 2; ++k) {
      lkd[k] = alloc<double>(nh); lpn[k] = alloc<double>(nh);
      lwkd[k] = alloc<double>(nwh); lwpn[k] = alloc<double>(nwh);
      ACK(cudaMemsetAsync(lkd[k], 0, nh * sizeof(double), st));
      ACK(cudaMemsetAsync(lpn[k], 0, nh * sizeof(double), st));
      ACK(cudaMemsetAsync(lwkd[k], 0, nwh * sizeof(double), st));
      ACK(cudaMemsetAsync(lwpn[k], 0, nwh * sizeof(double), st));
    }
    double* dtx = alloc<double>(n3);
    double* dtv = alloc<double>(n3);
    ACK(cudaMemcpyAsync(dtx, tx, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
    ACK(cudaMemcpyAsync(dtv, tv, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
    k_bwd_seed<<<nblk(n), 128, 0, st>>>(n, S.x, S.v, dtx, dtv, lx, lv);
    for (double* z : {lw, lF, lT, lp}) ACK(cudaMemsetAsync(z, 0, n3 * sizeof(double), st));
    // per-step storage of one segment
    std::vector<double*> Xs(K + 1), Vh(K + 1), Wh(K + 1);
    std::vector<ListsT<double>> Ls(K + 1);
    for (int k = 0; k <= K; ++k) {
      Xs[k] = alloc<double>(n3); Vh[k] = alloc<double>(n3); Wh[k] = alloc<double>(n3);
      Ls[k] = allocLists<double>();
    }
    State<double> R = allocState<double>();
    int cur = 0;
    for (int seg = nseg - 1; seg >= 0; --seg) {
      const int c = seg * K, e = std::min(c + K, nsteps);
      copyState(R, ck[seg]);
      copyLists(Ls[0], ckL[seg]);
      for (int s = c + 1; s <= e; ++s)
        advance(R, Xs[s - c], Vh[s - c], Wh[s - c], Ls[s - c - 1], Ls[s - c], kn, en, muc);
      for (int s = e; s >= c + 1; --s) {
        const int prv = cur ^ 1;
        k_bwd_close<<<nblk(n), 128, 0, st>>>(n, A, d_type, lv, lw, lF, lT, lvh, lwh);
        ACK(cudaMemsetAsync(lkd[prv], 0, nh * sizeof(double), st));
        ACK(cudaMemsetAsync(lpn[prv], 0, nh * sizeof(double), st));
        ACK(cudaMemsetAsync(lwkd[prv], 0, nwh * sizeof(double), st));
        ACK(cudaMemsetAsync(lwpn[prv], 0, nwh * sizeof(double), st));
        k_bwd_forces<<<nblk(n), 128, 0, st>>>(
            n, A, d_type, Xs[s - c], Vh[s - c], Wh[s - c], Ls[s - c - 1], 1, Ls[s - c], lF, lT,
            lkd[cur], lpn[cur], lwkd[cur], lwpn[cur], 0, lx, lvh, lwh, lkd[prv], lpn[prv],
            lwkd[prv], lwpn[prv], lp, kn, en, muc);
        k_bwd_move<<<nblk(n), 128, 0, st>>>(n, A, d_type, lx, lvh, lwh, lv, lw, lF, lT);
        ACK(cudaGetLastError());
        cur = prv;
      }
    }
    // leapfrog start: forces at (x0, v0, w0), the spring it leaves is zeroed
    ACK(cudaMemsetAsync(lvh, 0, n3 * sizeof(double), st));
    ACK(cudaMemsetAsync(lwh, 0, n3 * sizeof(double), st));
    {
      const int prv = cur ^ 1;
      k_bwd_forces<<<nblk(n), 128, 0, st>>>(
          n, A, d_type, d_x0, d_v0, d_w0, ckL[0], 0, ckL[0], lF, lT, lkd[cur], lpn[cur],
          lwkd[cur], lwpn[cur], 1, lx, lvh, lwh, lkd[prv], lpn[prv], lwkd[prv], lwpn[prv], lp,
          kn, en, muc);
      ACK(cudaGetLastError());
    }
    std::vector<double> hv(n3), hvh(n3), hp(n3);
    ACK(cudaMemcpyAsync(hv.data(), lv, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    ACK(cudaMemcpyAsync(hvh.data(), lvh, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    ACK(cudaMemcpyAsync(hp.data(), lp, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    ACK(cudaStreamSynchronize(st));
    checkOverflow();
    if (dLdv0)
      for (size_t i = 0; i < n3; ++i) dLdv0[i] = hv[i] + hvh[i];
    if (dLdp) {
      dLdp[0] = dLdp[1] = dLdp[2] = 0.;
      for (int t = 0; t < n; ++t)
        for (int d = 0; d < 3; ++d) dLdp[d] += hp[3 * (size_t)t + d];
    }
  }

  // Forward-mode derivative of the loss: the whole forward run on Dual<3>
  // numbers seeded on (kn, en, muc), or, with seed_particle >= 0, on the one
  // initial velocity component (seed_particle, seed_component) in slot 0.
  void forwardDual(int nsteps, const double* p, const double* tx, const double* tv,
                   double* loss, double* dLdp, int seed_particle, int seed_component) {
    using D = Dual<3>;
    if (nsteps < 1) throw std::runtime_error("nsteps must be >= 1");
    if (!tx || !tv) throw std::runtime_error("the loss needs target x and v");
    if (!d_type) throw std::runtime_error("set the particles first");
    Scope scope(this);
    ACK(cudaMemsetAsync(d_overflow, 0, sizeof(int), st));
    D kn = dconst<3>(p[0]), en = dconst<3>(p[1]), muc = dconst<3>(p[2]);
    const bool seed_v = seed_particle >= 0;
    if (seed_v && (seed_particle >= n || seed_component < 0 || seed_component > 2))
      throw std::runtime_error("seed out of range");
    if (!seed_v) { kn.d[0] = 1.; en.d[1] = 1.; muc.d[2] = 1.; }
    const size_t n3 = 3 * (size_t)n;
    State<D> S = allocState<D>();
    D* xs = alloc<D>(n3);
    D* vh = alloc<D>(n3);
    D* wh = alloc<D>(n3);
    ListsT<D> L[2] = {allocLists<D>(), allocLists<D>()};
    start(S, L[0], kn, en, muc, seed_v ? 3 * seed_particle + seed_component : -1);
    for (int s = 1; s <= nsteps; ++s) advance(S, xs, vh, wh, L[(s - 1) & 1], L[s & 1], kn, en, muc);
    checkOverflow();
    std::vector<D> per;
    lossOf(S, tx, tv, per);
    double Lv = 0., g[3] = {0., 0., 0.};
    for (auto const& a : per) {
      Lv += a.v;
      for (int d = 0; d < 3; ++d) g[d] += a.d[d];
    }
    if (loss) *loss = Lv;
    if (dLdp) {
      if (seed_v) dLdp[0] = g[0];
      else for (int d = 0; d < 3; ++d) dLdp[d] = g[d];
    }
  }
};

}  // namespace
}  // namespace gdem

// ----------------------------------------------------------------- C ABI --
using namespace gdem;

namespace {
template <typename F>
int adjGuarded(F&& f) {
  try {
    f();
    return GDEM_OK;
  } catch (AdjCheck const& e) {
    setLastError(e.what());
    return GDEM_ERR_CUDA;
  } catch (std::exception const& e) {
    setLastError(e.what());
    return GDEM_ERR_INVALID;
  }
}
AdjointSystem* adj(gdem_adjoint_handle h) { return reinterpret_cast<AdjointSystem*>(h); }
}  // namespace

extern "C" {

int gdem_adjoint_create(const char* xml_path, gdem_adjoint_handle* out) {
  return adjGuarded([&] {
    if (!xml_path || !out) throw std::runtime_error("invalid arguments");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw AdjCheck("no CUDA device: the adjoint has no CPU fallback");
    auto s = std::make_unique<AdjointSystem>();
    s->create(xml_path);
    *out = reinterpret_cast<gdem_adjoint_handle>(s.release());
  });
}

int gdem_adjoint_set_particles(gdem_adjoint_handle h, int64_t n, const int* type,
                               const double* x0, const double* v0, const double* w0) {
  return adjGuarded([&] {
    if (!h || !type || !x0 || !v0) throw std::runtime_error("invalid arguments");
    adj(h)->setParticles(n, type, x0, v0, w0);
  });
}

int gdem_adjoint_run(gdem_adjoint_handle h, int nsteps, int checkpoint_every,
                     const double* params, const double* target_x, const double* target_v,
                     double* loss, double* x_out, double* v_out, double* dL_dparams,
                     double* dL_dv0) {
  return adjGuarded([&] {
    if (!h || !params) throw std::runtime_error("invalid arguments");
    adj(h)->run(nsteps, checkpoint_every, params, target_x, target_v, loss, x_out, v_out,
                dL_dparams, dL_dv0);
  });
}

int gdem_adjoint_forward_dual(gdem_adjoint_handle h, int nsteps, const double* params,
                              const double* target_x, const double* target_v,
                              int seed_particle, int seed_component, double* loss,
                              double* dL_dseed) {
  return adjGuarded([&] {
    if (!h || !params) throw std::runtime_error("invalid arguments");
    adj(h)->forwardDual(nsteps, params, target_x, target_v, loss, dL_dseed, seed_particle,
                        seed_component);
  });
}

void gdem_adjoint_destroy(gdem_adjoint_handle h) { delete adj(h); }

}  // extern "C"
