// gdem_motion.cuh -- second-order leapfrog of one particle, shared by the
// move-only kernel and the fused force + move step kernels.
//
// The expressions follow the reference operation by operation (the files
// that include this header are compiled with -fmad=false):
//   SecondOrderLeapFrog::Move / advanceVelocity
//     (TimeIntegration/src/SecondOrderLeapFrog.cpp:44-94),
//   ParticleKinematics::Move (Component/src/ParticleKinematics.cpp:62-128),
//   ParticleKinematicsSphere / ParticleKinematics3D angular acceleration
//     (ParticleKinematicsSphere.cpp:47-55, ParticleKinematics3D.cpp:56-77),
//   Transform::composeLeftByRotation (Geometry/src/Transform.cpp:140-159),
//   MotionError (Component/src/Particle.cpp:446-456),
//   Cell::GetCell and the periodic master/clone swap
//     (Base/src/Cell.cpp:172-184, Base/src/LinkedCell.cpp:1502-1547).
#pragma once
#include "gdem_device.cuh"

namespace gdem {

// Angular acceleration in the body frame; the gyroscopic term for
// non-spherical classes (predictor mode).
__device__ __forceinline__ d3 dOmega(TypeDesc const& t, d3 tbf, d3 om) {
  const double c = t.coupling;
  if (t.shape == 0)
    return mk(tbf.x / (c * t.inertia[0]), tbf.y / (c * t.inertia[1]), tbf.z / (c * t.inertia[2]));
  const double* I = t.inertia;
  return mk(tbf.x / (c * I[0]) + om.y * om.z * (I[1] - I[2]) / I[0],
            tbf.y / (c * I[1]) + om.z * om.x * (I[2] - I[0]) / I[1],
            tbf.z / (c * I[2]) + om.x * om.y * (I[0] - I[1]) / I[2]);
}

// SSP-RK3 update of the body-fixed angular velocity over h.  For a sphere
// the acceleration does not depend on omega, so K1 = K2 = K3 and one
// evaluation gives the same bits as three.
__device__ __forceinline__ d3 rk3(TypeDesc const& t, d3 tbf, d3 wbf, double h) {
  if (t.shape == 0) {
    d3 K = dOmega(t, tbf, wbf);
    K = K * h;
    return wbf + ((K + K) + 4. * K) / 6.;
  }
  d3 K1 = dOmega(t, tbf, wbf);
  K1 = K1 * h;
  d3 K2 = dOmega(t, tbf, wbf + K1);
  K2 = K2 * h;
  d3 K3 = dOmega(t, tbf, wbf + 0.25 * (K1 + K2));
  K3 = K3 * h;
  return wbf + ((K1 + K2) + 4. * K3) / 6.;
}

// advanceVelocity: v, w_bf (and the space-frame w) over h.
__device__ __forceinline__ void kick(TypeDesc const& tp, d3 F, d3 T, d3& v, d3& wbf, d3& w,
                                     dq q, double h) {
  dq pc = conj(q);
  d3 tbf = multToVector3(pc, vecq(T, q));
  const double c = tp.coupling;
  v = v + (F / (tp.mass * c)) * h;
  wbf = rk3(tp, tbf, wbf, h);
  w = multToVector3(q, vecq(wbf, pc));
}

// Signed periodic wrap counts, one byte per axis.
__device__ __forceinline__ int wrapGet(int w, int d) {
  return (int)(signed char)((unsigned)w >> (8 * d) & 0xFFu);
}
__device__ __forceinline__ int wrapSet(int w, int d, int val) {
  const unsigned m = 0xFFu << (8 * d);
  return (int)(((unsigned)w & ~m) | (((unsigned)val & 0xFFu) << (8 * d)));
}

// Cell of x in the reference grid after the periodic wrap (a particle that
// left the inner cells is replaced by its image; x is updated).  wrapd[d]
// counts the wrap: the continuous position is x + wrapd * L.  Out-of-grid
// particles raise kErrOutOfGrid.
__device__ __forceinline__ void wrapToGrid(GridDesc const& g, d3& x, int* wrapd, int* status) {
  double xs[3] = {x.x, x.y, x.z};
  bool outside = false;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    wrapd[d] = 0;
    // well inside the inner cells: the cell test below cannot trigger
    if (xs[d] > g.safe_lo[d] && xs[d] < g.safe_hi[d]) continue;
    int id = (int)floor((xs[d] - g.lc_origin[d]) / g.edge[d]);
    if (g.periodic[d]) {
      if (id < 1) { xs[d] = xs[d] + g.L[d]; wrapd[d] = -1; }
      else if (id > g.nb[d] - 2) { xs[d] = xs[d] + (-g.L[d]); wrapd[d] = 1; }
      id = (int)floor((xs[d] - g.lc_origin[d]) / g.edge[d]);
    }
    outside |= id < 0 || id >= g.nb[d];
  }
  if (outside) raise(status, kErrOutOfGrid);
  x = mk(xs[0], xs[1], xs[2]);
}

// ------------------------------------------------- FP32-split leapfrog --
// The same integration with the FP64 arithmetic reorganised: products by
// precomputed reciprocals instead of divisions, the sphere's SSP-RK3 taken as
// the single evaluation it equals in exact arithmetic, the sine and cosine of
// the small rotation angle from their series.  Every quantity stays FP64;
// the results differ from the reference's operation order by a few ulps per
// step, far below the FP32 force law of this mode.
__device__ __forceinline__ d3 dOmegaFast(TypeDesc const& t, d3 tbf, d3 om) {
  const double* iIc = t.inv_inertia_c;
  if (t.shape == 0) return mk(tbf.x * iIc[0], tbf.y * iIc[1], tbf.z * iIc[2]);
  const double* I = t.inertia;
  const double* iI = t.inv_inertia;
  return mk(tbf.x * iIc[0] + om.y * om.z * (I[1] - I[2]) * iI[0],
            tbf.y * iIc[1] + om.z * om.x * (I[2] - I[0]) * iI[1],
            tbf.z * iIc[2] + om.x * om.y * (I[0] - I[1]) * iI[2]);
}
__device__ __forceinline__ d3 rk3Fast(TypeDesc const& t, d3 tbf, d3 wbf, double h) {
  if (t.shape == 0) return wbf + dOmegaFast(t, tbf, wbf) * h;
  const double sixth = 1. / 6.;
  d3 K1 = dOmegaFast(t, tbf, wbf) * h;
  d3 K2 = dOmegaFast(t, tbf, wbf + K1) * h;
  d3 K3 = dOmegaFast(t, tbf, wbf + 0.25 * (K1 + K2)) * h;
  return wbf + ((K1 + K2) + 4. * K3) * sixth;
}
__device__ __forceinline__ void kickFast(TypeDesc const& tp, d3 F, d3 T, d3& v, d3& wbf, d3& w,
                                         dq q, double h) {
  dq pc = conj(q);
  d3 tbf = multToVector3(pc, vecq(T, q));
  v = v + F * (h * tp.inv_mass);
  wbf = rk3Fast(tp, tbf, wbf, h);
  w = multToVector3(q, vecq(wbf, pc));
}
// sin and cos of the small rotation angle of the FP64 leapfrog, rounded as
// the reference's host library rounds them: below 1e-3 the Taylor tails
// t = sin a - a and u = cos a - 1 (through a^9 and a^8) are summed in
// double, where their own rounding is far below half an ulp of the result,
// and added to a and 1 with one final rounding, which gives the correctly
// rounded value except in a vanishing fraction of cases; compared with the
// x86-64 glibc sin / cos over 6e7 arguments in [1e-12, 1e-3] the two never
// differed (about 1 in 1e5 do above 1e-3, where the CUDA functions are used
// instead).  Rounding the same way as the reference keeps the quaternion and
// orientation matrix of an FP64 step bit-identical to the reference's, which
// matters for curved bodies (cylinders), whose closest-point search stops
// at a tolerance and so amplifies an ulp of orientation.
__device__ __forceinline__ void sinCosRef(double a, double* s, double* c) {
  if (fabs(a) < 1.e-3) {
    const double a2 = a * a;
    const double ts = a * (a2 * (-1. / 6. + a2 * (1. / 120. + a2 * (-1. / 5040. + a2 * (1. / 362880.)))));
    const double tc = a2 * (-0.5 + a2 * (1. / 24. + a2 * (-1. / 720. + a2 * (1. / 40320.))));
    *s = a + ts;
    *c = 1. + tc;
  } else {
    sincos(a, s, c);
  }
}
// sin and cos of a; series below 1e-2 (truncation below 1e-19 relative)
__device__ __forceinline__ void sinCosSmall(double a, double* s, double* c) {
  if (fabs(a) < 1.e-2) {
    const double a2 = a * a;
    *s = a * (1. - a2 * (1. / 6. - a2 * (1. / 120. - a2 * (1. / 5040.))));
    *c = 1. - a2 * (0.5 - a2 * (1. / 24. - a2 * (1. / 720.)));
  } else {
    sincos(a, s, c);
  }
}

// FP32-split leapfrog of a sphere in a spheres-only system.  With an
// isotropic inertia the body-frame kick followed by the rotation back to the
// space frame (kick: w = q (w_bf + q* T q / I h) q*) equals the space-frame
// kick w + T / I h in exact arithmetic, and the drift's rotation about w
// leaves w unchanged, so the space-frame angular velocity is the state and
// the body-frame one is derived on output (q* w q).  Same leapfrog otherwise.
__device__ __forceinline__ void leapfrogSphere(TypeDesc const& tp, d3 F, d3 T, bool close,
                                               double hc, bool move, double h, double dt,
                                               d3& x, d3& v, d3& w, dq& q, d3& dx, int* status) {
  const double iI = tp.inv_inertia_c[0];
  if (close) {
    v = v + F * (hc * tp.inv_mass);
    w = w + T * (hc * iI);
  }
  dx = mk(0., 0., 0.);
  if (!move) return;
  v = v + F * (h * tp.inv_mass);
  w = w + T * (h * iI);
  dx = v * dt;
  x = x + dx;
  const double nOm = norm(w);
  dq qdt;
  if (nOm > 1.0e-10) {
    double cc, ss;
    sinCosSmall(nOm * dt * 0.5, &ss, &cc);
    qdt = qmk((ss / nOm) * w, cc);
  } else {
    qdt = qmk(mk(0., 0., 0.), 1.);
  }
  q = qmul(qdt, q);
  if (dot(dx, dx) > tp.crust * tp.crust) raise(status, kErrMotion);
}

// One particle's leapfrog: optionally the closing kick of the previous step
// (with this step's F, T over hc), then optionally the opening kick over h
// and the drift over dt with the quaternion and orientation update.
// basis: 9 entries (row-major) or null.  dx receives the translation.
template <bool kFast>
__device__ __forceinline__ void leapfrog(TypeDesc const& tp, d3 F, d3 T, bool close, double hc,
                                         bool move, double h, double dt, d3& x, d3& v,
                                         d3& wbf, d3& w, dq& q, double* basis, d3& dx,
                                         int* status) {
  if (close) {
    if (kFast) kickFast(tp, F, T, v, wbf, w, q, hc);
    else kick(tp, F, T, v, wbf, w, q, hc);
  }
  dx = mk(0., 0., 0.);
  if (!move) return;
  dq pc = conj(q);
  d3 tbf = multToVector3(pc, vecq(T, q));
  const double c = tp.coupling;
  if (kFast) {
    v = v + F * (h * tp.inv_mass);
    wbf = rk3Fast(tp, tbf, wbf, h);
  } else {
    v = v + (F / (tp.mass * c)) * h;
  }
  dx = v * dt;
  if (!kFast) wbf = rk3(tp, tbf, wbf, h);
  w = multToVector3(q, vecq(wbf, pc));
  const d3 meanw = w;     // same expression as w (ParticleKinematics.cpp:79-82)
  x = x + dx;
  double nOm = norm(meanw);
  dq qdt;
  if (nOm > 1.0e-10) {
    double cc, ss;
    if (kFast) {
      sinCosSmall(nOm * dt * 0.5, &ss, &cc);
      qdt = qmk((ss / nOm) * meanw, cc);
    } else {
      sinCosRef(nOm * dt / 2., &ss, &cc);
      qdt = qmk((ss * 1. / nOm) * meanw, cc);
    }
  } else {
    qdt = qmk(mk(0., 0., 0.), 1.);
  }
  q = qmul(qdt, q);
  if (basis) {
    double out[9];
    const double qx = qdt.v.x, qy = qdt.v.y, qz = qdt.v.z, qw = qdt.w;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double px = qy * basis[6 + i] - qz * basis[3 + i] + qw * basis[0 + i];
      double py = qz * basis[0 + i] - qx * basis[6 + i] + qw * basis[3 + i];
      double pz = qx * basis[3 + i] - qy * basis[0 + i] + qw * basis[6 + i];
      double pw = -qx * basis[0 + i] - qy * basis[3 + i] - qz * basis[6 + i];
      out[0 + i] = qy * pz - qz * py - pw * qx + qw * px;
      out[3 + i] = qz * px - qx * pz - pw * qy + qw * py;
      out[6 + i] = qx * py - qy * px - pw * qz + qw * pz;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) basis[k] = out[k];
  }
  if (kFast ? dot(dx, dx) > tp.crust * tp.crust : norm(dx) > tp.crust) raise(status, kErrMotion);
}

// The state of particle t that the leapfrog reads besides F and T; loaded
// before the move kernel waits for the force kernel (nothing between them
// writes it).
struct MoveIn {
  d3 x, v, w, wbf;
  dq q;
  double bas[9];
  int wrap;
  float4 p0;   // FP32 position at the last rebuild
};
template <bool kFast, bool kBasis>
__device__ __forceinline__ void loadMoveIn(DevState const& S, int t, MoveIn& m) {
  const int cap = S.cap;
  // FP32-split, spheres only: w is the angular state (leapfrogSphere)
  constexpr bool kSphereW = kFast && !kBasis;
  m.x = ld3(S.x, cap, t); m.v = ld3(S.v, cap, t); m.w = ld3(S.w, cap, t);
  m.wbf = kSphereW ? mk(0., 0., 0.) : ld3(S.wbf, cap, t);
  m.q = qmk(mk(S.q[t], S.q[cap + t], S.q[2 * cap + t]), S.q[3 * cap + t]);
  // FP32-split: the basis array exists only in the instantiation for
  // systems that carry one (convex bodies), a compile-time choice that keeps
  // it in registers.  FP64: one instantiation tests for it at run time, in
  // advanceParticle (the faster of the two on B200 for that path, measured).
  if constexpr (kFast && kBasis) {
#pragma unroll
    for (int k = 0; k < 9; ++k) m.bas[k] = S.basis[k * cap + t];
  }
  m.wrap = S.wrap[t];
  m.p0 = S.posf0[t];
}

// Moves particle t (state m, F, T as given) and writes the result to the
// second buffers; updates the wraps and the FP32 position and flags a
// pair-list rebuild when the particle has moved half the skin or more.  close/move
// select the kicks as in leapfrog().
template <bool kFast, bool kBasis>
__device__ __forceinline__ void advanceParticle(DevState const& S, int t, TypeDesc const& tp,
                                                d3 F, d3 T, bool close, bool move, MoveIn& m) {
  const int cap = S.cap;
  const double dt = S.dt;
  GridDesc const& g = S.grids[S.inst[t]];
  constexpr bool kSphereW = kFast && !kBasis;
  d3 x = m.x, v = m.v, w = m.w, wbf = m.wbf;
  dq q = m.q;
  double* bas = m.bas;
  double* bp = nullptr;
  if constexpr (kFast) {
    if constexpr (kBasis) bp = bas;
  } else if (S.basis) {
#pragma unroll
    for (int k = 0; k < 9; ++k) bas[k] = S.basis[k * cap + t];
    bp = bas;
  }
  d3 dx;
  if constexpr (kSphereW)
    leapfrogSphere(tp, F, T, close, 0.5 * dt, move, 0.5 * dt, dt, x, v, w, q, dx, S.status);
  else
    leapfrog<kFast>(tp, F, T, close, 0.5 * dt, move, 0.5 * dt, dt, x, v, wbf, w, q, bp, dx, S.status);
  int wr = m.wrap;
  if (move) {
    int wd[3];
    wrapToGrid(g, x, wd, S.status);
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (wd[d]) wr = wrapSet(wr, d, wrapGet(wr, d) + wd[d]);
  }
  st3(S.x2, cap, t, x); st3(S.v2, cap, t, v); st3(S.w2, cap, t, w);
  if (!kSphereW) st3(S.wbf2, cap, t, wbf);
  S.q2[t] = q.v.x; S.q2[cap + t] = q.v.y; S.q2[2 * cap + t] = q.v.z; S.q2[3 * cap + t] = q.w;
  if (bp) {
#pragma unroll
    for (int k = 0; k < 9; ++k) S.basis2[k * cap + t] = bas[k];
  }
  S.wrap2[t] = wr;
  // FP32 copy for the contact filter: the continuous position since the
  // last rebuild (the wrapped one plus the wraps), so that the image shift
  // recorded in a list entry at the rebuild stays valid
  // (in FP32: its rounding is covered by the filter's margin)
  GridDesc const& bg = S.bgrids[S.inst[t]];
  const float4 pf = make_float4((float)x.x + (float)wrapGet(wr, 0) * bg.Lf[0],
                                (float)x.y + (float)wrapGet(wr, 1) * bg.Lf[1],
                                (float)x.z + (float)wrapGet(wr, 2) * bg.Lf[2], (float)tp.radius);
  S.posf[t] = pf;
  if (move) {
    // displacement since the rebuild as the difference of the two FP32
    // positions; each coordinate of either carries at most three roundings
    // of its own magnitude (the conversion, the wrap product, the sum), so
    // half the skin less 2.4e-7 times the summed magnitudes still bounds
    // the exact FP64 displacement
    const float ex = pf.x - m.p0.x, ey = pf.y - m.p0.y, ez = pf.z - m.p0.z;
    const float tol = 2.4e-7f * (fabsf(pf.x) + fabsf(pf.y) + fabsf(pf.z) + fabsf(m.p0.x) +
                                 fabsf(m.p0.y) + fabsf(m.p0.z));
    const float half = fmaxf(0.5f * bg.skin_f - tol, 0.f);
    if (ex * ex + ey * ey + ez * ez >= half * half) S.ctl[kCtlNeed] = 1;
  }
}

// Image shift (in periods) of list entry ent (partner u) of slot t: the
// shift recorded at the rebuild (bits 27-31 of the entry, shiftCode),
// corrected by the wraps of both particles since the rebuild.
__device__ __forceinline__ void entryShift(DevState const& S, unsigned ent, int t, int u,
                                           int* sh) {
  const int c = (int)(ent >> 27);
  sh[0] = c % 3 - 1; sh[1] = (c / 3) % 3 - 1; sh[2] = c / 9 - 1;
  const int wt = S.wrap[t], wu = S.wrap[u];
  if (wt | wu) {
#pragma unroll
    for (int d = 0; d < 3; ++d) sh[d] += wrapGet(wu, d) - wrapGet(wt, d);
  }
}

}  // namespace gdem
