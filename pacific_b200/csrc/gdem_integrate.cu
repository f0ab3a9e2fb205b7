// gdem_integrate.cu -- leapfrog kick/drift and linked-cell binning kernels.
//
// Compiled with -fmad=false: positions, velocities and cell indices are FP64
// and follow the reference's expression order, so cell assignments are
// bit-identical to Cell::GetCell on the same state.
//
//   k_key       post-move cell of each particle (Cell::GetCell, Base/src/
//               Cell.cpp:172-184; SimulationError when outside the grid,
//               Base/src/LinkedCell.cpp:1506-1531) and the cell histogram of
//               the counting-sort binning.
//   scan/place/cellsort
//               counting sort of particles on their cell key: a one-digit
//               radix sort whose digit is the cell key, made stable by
//               ordering each cell's entries by particle ID; it yields the
//               cell start/end tables.
//   k_move_gather
//               SecondOrderLeapFrog::Move + ParticleKinematics::Move
//               (TimeIntegration/src/SecondOrderLeapFrog.cpp:44-67,
//                Component/src/ParticleKinematics.cpp:62-104) and MotionError
//               (Component/src/Particle.cpp:446-456), applied while the state
//               is permuted into cell order, so the state is read and written
//               once per step.
//   k_kick      advanceVelocity (SecondOrderLeapFrog.cpp:74-94,
//               ParticleKinematics.cpp:110-128).
#include "gdem_kernels.cuh"

namespace gdem {

namespace {

// ParticleKinematicsSphere / ParticleKinematics3D angular acceleration
// (ParticleKinematicsSphere.cpp:47-55, ParticleKinematics3D.cpp:56-77, with
// the predictor-mode gyroscopic term).
__device__ __forceinline__ d3 dOmega(TypeDesc const& t, d3 tbf, d3 om) {
  const double c = 1.;
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

__device__ __forceinline__ void kick(TypeDesc const& tp, d3 F, d3 T, d3& v, d3& wbf, d3& w,
                                     dq q, double h) {
  dq pc = conj(q);
  d3 tbf = multToVector3(pc, vecq(T, q));
  const double c = 1.;
  v = v + (F / (tp.mass * c)) * h;
  wbf = rk3(tp, tbf, wbf, h);
  w = multToVector3(q, vecq(wbf, pc));
}

// Cell of a position after the periodic wrap: a master leaving the inner
// cells is replaced by its image (x is updated).  Cell::GetCell.
__device__ __forceinline__ void cellOf(GridDesc const& g, d3& x, int* id) {
  double xs[3] = {x.x, x.y, x.z};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    id[d] = (int)floor((xs[d] - g.lc_origin[d]) / g.edge[d]);
    if (g.periodic[d]) {
      if (id[d] < 1) xs[d] = xs[d] + g.L[d];
      else if (id[d] > g.nb[d] - 2) xs[d] = xs[d] + (-g.L[d]);
      id[d] = (int)floor((xs[d] - g.lc_origin[d]) / g.edge[d]);
    }
  }
  x = mk(xs[0], xs[1], xs[2]);
}

__device__ __forceinline__ int keyOf(GridDesc const& g, int* id, int* status) {
  bool valid = id[0] >= 0 && id[0] < g.nb[0] && id[1] >= 0 && id[1] < g.nb[1] &&
               id[2] >= 0 && id[2] < g.nb[2];
  if (!valid) {
    raise(status, kErrOutOfGrid);
    id[0] = min(max(id[0], 0), g.nb[0] - 1);
    id[1] = min(max(id[1], 0), g.nb[1] - 1);
    id[2] = min(max(id[2], 0), g.nb[2] - 1);
  }
  return g.cell_offset + id[1] * g.nb[2] * g.nb[0] + id[2] * g.nb[0] + id[0];
}

// First binning pass: the cell each particle will occupy after this step's
// kick + drift.  Evaluates exactly the translational part of k_move_gather
// (same expressions, same order), so both passes agree bit for bit.
__global__ void k_key(DevState S, double h, double dt, int pre_kick, double pre_h) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n) return;
  const int cap = S.cap;
  const double mass = S.types[S.type[s]].mass;
  GridDesc const& g = S.grids[S.inst[s]];
  const d3 F = ld3(S.F, cap, s);
  d3 v = ld3(S.v, cap, s), x = ld3(S.x, cap, s);
  const double c = 1.;
  if (pre_kick) v = v + (F / (mass * c)) * pre_h;
  v = v + (F / (mass * c)) * h;
  x = x + v * dt;
  int id[3];
  cellOf(g, x, id);
  int key = keyOf(g, id, S.status);
  S.skey[s] = key;
  S.rank[s] = atomicAdd(&S.cell_count[key], 1);
}

// Binning without motion (initial linking, LinkedCell::Link).
__global__ void k_bin(DevState S) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n) return;
  GridDesc const& g = S.grids[S.inst[s]];
  int id[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) id[d] = (int)floor((S.x[d * S.cap + s] - g.lc_origin[d]) / g.edge[d]);
  int key = keyOf(g, id, S.status);
  S.skey[s] = key;
  S.rank[s] = atomicAdd(&S.cell_count[key], 1);
}

__global__ void k_kick(DevState S, double h) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n) return;
  const int cap = S.cap;
  TypeDesc const tp = S.types[S.type[s]];
  d3 F = ld3(S.F, cap, s), T = ld3(S.T, cap, s);
  d3 v = ld3(S.v, cap, s), wbf = ld3(S.wbf, cap, s), w;
  dq q = qmk(mk(S.q[s], S.q[cap + s], S.q[2 * cap + s]), S.q[3 * cap + s]);
  kick(tp, F, T, v, wbf, w, q, h);
  st3(S.v, cap, s, v); st3(S.wbf, cap, s, wbf); st3(S.w, cap, s, w);
}

// ------------------------------------------------------------------ scan --
// Exclusive scan of cell counts, three phases over 1024-element tiles.
constexpr int kScanTile = 1024;

__device__ __forceinline__ int blockExclusiveScan(int v, int* smem, int& total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    int y = lane < nw ? smem[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int z = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += z;
    }
    smem[lane] = y;
  }
  __syncthreads();
  int before = wid > 0 ? smem[wid - 1] : 0;
  total = smem[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void k_scan_tiles(const int* in, int* out, int* tile_sums, int n) {
  __shared__ int smem[32];
  int i = blockIdx.x * kScanTile + threadIdx.x;
  int v = i < n ? in[i] : 0;
  int total;
  int ex = blockExclusiveScan(v, smem, total);
  if (i < n) out[i] = ex;
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Scans the tile sums in place with one block, looping over chunks.
__global__ void k_scan_sums(int* sums, int ntiles) {
  __shared__ int smem[32];
  int carry = 0;
  for (int base = 0; base < ntiles; base += kScanTile) {
    int i = base + threadIdx.x;
    int v = i < ntiles ? sums[i] : 0;
    int total;
    int ex = blockExclusiveScan(v, smem, total);
    if (i < ntiles) sums[i] = ex + carry;
    carry += total;
    __syncthreads();
  }
}

// Adds the tile offsets; out[n] receives the total so that cell c spans
// [out[c], out[c + 1]).
__global__ void k_scan_add(int* out, const int* tile_sums, const int* in, int n) {
  int i = blockIdx.x * kScanTile + threadIdx.x;
  if (i < n) {
    int v = out[i] + tile_sums[blockIdx.x];
    out[i] = v;
    if (i == n - 1) out[n] = v + in[i];
  }
}

__global__ void k_place(DevState S) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n) return;
  S.order[S.cell_start[S.skey[s]] + S.rank[s]] = s;
}

// Orders each cell's entries by particle ID, so the permutation does not
// depend on the arrival order of the atomic histogram.
// It also resets the cell histogram for the next binning (every count has
// been consumed by the scan at this point).
__global__ void k_cellsort(DevState S) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= S.ncells) return;
  int b = S.cell_start[c];
  int cnt = S.cell_start[c + 1] - b;
  S.cell_count[c] = 0;
  if (cnt < 2) return;
  for (int i = 1; i < cnt; ++i) {
    int e = S.order[b + i];
    int ide = S.id[e];
    int j = i - 1;
    while (j >= 0 && S.id[S.order[b + j]] > ide) {
      S.order[b + j + 1] = S.order[b + j];
      --j;
    }
    S.order[b + j + 1] = e;
  }
}

// Second binning pass: permutes the state into cell order and, when moving,
// applies the step's kick + drift on the way (ParticleKinematics::Move,
// ParticleKinematics.cpp:62-104, with SecondOrderLeapFrog::Move,
// SecondOrderLeapFrog.cpp:44-67), then builds the compact contact arrays.
__global__ void k_move_gather(DevState S, int moving, double h, double dt, int pre_kick,
                              double pre_h) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  const int cap = S.cap;
  const int s = S.order[t];
  const int idv = S.id[s], ty = S.type[s], in = S.inst[s];
  const int key = S.skey[s];
  TypeDesc const& tp = S.types[ty];
  GridDesc const& g = S.grids[in];
  d3 x = ld3(S.x, cap, s), v = ld3(S.v, cap, s), wbf = ld3(S.wbf, cap, s), w;
  dq q = qmk(mk(S.q[s], S.q[cap + s], S.q[2 * cap + s]), S.q[3 * cap + s]);
  if (moving) {
    const d3 F = ld3(S.F, cap, s), T = ld3(S.T, cap, s);
    if (pre_kick) kick(tp, F, T, v, wbf, w, q, pre_h);
    dq pc = conj(q);
    d3 tbf = multToVector3(pc, vecq(T, q));
    const double c = 1.;
    v = v + (F / (tp.mass * c)) * h;
    d3 dx = v * dt;
    wbf = rk3(tp, tbf, wbf, h);
    w = multToVector3(q, vecq(wbf, pc));
    const d3 meanw = w;     // same expression as w (ParticleKinematics.cpp:79-82)
    x = x + dx;
    double nOm = norm(meanw);
    dq qdt;
    if (nOm > 1.0e-10) {
      double cc, ss;
      sincos(nOm * dt / 2., &ss, &cc);
      qdt = qmk((ss * 1. / nOm) * meanw, cc);
    } else {
      qdt = qmk(mk(0., 0., 0.), 1.);
    }
    q = qmul(qdt, q);
    if (S.basis) {
      // Transform::composeLeftByRotation (Geometry/src/Transform.cpp:140-159)
      double mm[9], out[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) mm[k] = S.basis[k * cap + s];
      double qx = qdt.v.x, qy = qdt.v.y, qz = qdt.v.z, qw = qdt.w;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double px = qy * mm[6 + i] - qz * mm[3 + i] + qw * mm[0 + i];
        double py = qz * mm[0 + i] - qx * mm[6 + i] + qw * mm[3 + i];
        double pz = qx * mm[3 + i] - qy * mm[0 + i] + qw * mm[6 + i];
        double pw = -qx * mm[0 + i] - qy * mm[3 + i] - qz * mm[6 + i];
        out[0 + i] = qy * pz - qz * py - pw * qx + qw * px;
        out[3 + i] = qz * px - qx * pz - pw * qy + qw * py;
        out[6 + i] = qx * py - qy * px - pw * qz + qw * pz;
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) S.basis2[k * cap + t] = out[k];
    }
    if (norm(dx) > tp.crust) raise(S.status, kErrMotion);   // Particle.cpp:446-456
    int id[3];
    cellOf(g, x, id);
  } else {
    w = ld3(S.w, cap, s);
    if (S.basis) {
#pragma unroll
      for (int k = 0; k < 9; ++k) S.basis2[k * cap + t] = S.basis[k * cap + s];
    }
  }
  S.id2[t] = idv; S.type2[t] = ty; S.inst2[t] = in;
  S.key[t] = key;
  st3(S.x2, cap, t, x); st3(S.v2, cap, t, v); st3(S.w2, cap, t, w); st3(S.wbf2, cap, t, wbf);
  S.q2[t] = q.v.x; S.q2[cap + t] = q.v.y; S.q2[2 * cap + t] = q.v.z; S.q2[3 * cap + t] = q.w;
  int c = key - g.cell_offset;
  int ci = c % g.nb[0];
  int ck = (c / g.nb[0]) % g.nb[2];
  int cj = c / (g.nb[0] * g.nb[2]);
  S.cellc[t] = make_int4(ci, cj, ck, in);
  if (S.pos64) {
    S.pos64[t] = make_double4(x.x, x.y, x.z, tp.radius);
    S.vel64[t] = make_double4(v.x, v.y, v.z, tp.mass);
    S.omg64[t] = make_double4(w.x, w.y, w.z, tp.eqrad);
  }
  if (S.offh) {
    // FP32 offset from the cell's lower corner (broad phase of FP32-split)
    S.offh[t] = make_float4((float)(x.x - (g.lc_origin[0] + ci * g.edge[0])),
                            (float)(x.y - (g.lc_origin[1] + cj * g.edge[1])),
                            (float)(x.z - (g.lc_origin[2] + ck * g.edge[2])), tp.r_f);
  }
}

// Scatter of sorted-order state into ID order (for download).
__global__ void k_scatter_by_id(DevState S, double* out_x, double* out_v, double* out_w,
                                double* out_wbf, double* out_q, double* out_F, double* out_T,
                                int id_base) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  const int cap = S.cap, n = S.n;
  int i = S.id[t] - id_base;
  if (i < 0 || i >= n) return;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (out_x) out_x[3 * i + d] = S.x[d * cap + t];
    if (out_v) out_v[3 * i + d] = S.v[d * cap + t];
    if (out_w) out_w[3 * i + d] = S.w[d * cap + t];
    if (out_wbf) out_wbf[3 * i + d] = S.wbf[d * cap + t];
    if (out_F) out_F[3 * i + d] = S.F[d * cap + t];
    if (out_T) out_T[3 * i + d] = S.T[d * cap + t];
  }
  if (out_q) {
#pragma unroll
    for (int k = 0; k < 4; ++k) out_q[4 * i + k] = S.q[k * cap + t];
  }
}

// Orientation matrices (row-major, 9 per particle) into ID order.
__global__ void k_basis_by_id(DevState S, double* out, int id_base) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  int i = S.id[t] - id_base;
  if (i < 0 || i >= S.n) return;
#pragma unroll
  for (int k = 0; k < 9; ++k) out[9 * (size_t)i + k] = S.basis[k * S.cap + t];
}

__global__ void k_cells_by_id(DevState S, int* ijk, int id_base) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  int i = S.id[t] - id_base;
  if (i < 0 || i >= S.n) return;
  int4 c = S.cellc[t];
  ijk[3 * i] = c.x; ijk[3 * i + 1] = c.y; ijk[3 * i + 2] = c.z;
}

// Zeroes the cumulative tangential and rolling memories of every live entry
// (Component::setContactMapCumulativeFeaturesToZero, Component.cpp:842-851).
template <typename V>
__global__ void k_hist_zero_cumulative(HistTable t) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= (1 << t.log2cap)) return;
  if (t.keys[s] == kEmptyKey) return;
  V* v = static_cast<V*>(t.vals) + 9 * (size_t)s;
  v[0] = v[1] = v[2] = 0;
  v[6] = v[7] = v[8] = 0;
}

// Loads host-layout state (AoS, by particle ID, staged in device memory)
// into the SoA arrays, in ID order.
__global__ void k_load_state(DevState S, const double* x, const double* v, const double* w,
                             const double* wbf, const double* q, const double* F,
                             const double* T, const int* type_by_id, const int* inst_by_id) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n) return;
  const int cap = S.cap;
  S.id[i] = i;
  S.type[i] = type_by_id[i];
  S.inst[i] = inst_by_id[i];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    S.x[d * cap + i] = x[3 * i + d];
    S.v[d * cap + i] = v[3 * i + d];
    S.w[d * cap + i] = w[3 * i + d];
    if (wbf) S.wbf[d * cap + i] = wbf[3 * i + d];
    if (F) S.F[d * cap + i] = F[3 * i + d];
    if (T) S.T[d * cap + i] = T[3 * i + d];
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) S.q[k * cap + i] = q[4 * i + k];
  if (S.basis) {
    // orientation matrix of q with the expression order of Matrix::setRotation
    // (Geometry/src/Matrix.cpp:114-127); gdem_upload_basis may replace it
    double x = q[4 * i], y = q[4 * i + 1], z = q[4 * i + 2], w4 = q[4 * i + 3];
    double s = 2.0 / (x * x + y * y + z * z + w4 * w4);
    double xs = x * s, ys = y * s, zs = z * s;
    double wx = w4 * xs, wy = w4 * ys, wz = w4 * zs;
    double xx = x * xs, xy = x * ys, xz = x * zs, yy = y * ys, yz = y * zs, zz = z * zs;
    double m[9] = {1.0 - (yy + zz), xy - wz, xz + wy, xy + wz, 1.0 - (xx + zz), yz - wx,
                   xz - wy, yz + wx, 1.0 - (xx + yy)};
#pragma unroll
    for (int k = 0; k < 9; ++k) S.basis[k * cap + i] = m[k];
  }
  if (!wbf) {
    // q* (w, q) (ParticleKinematics.cpp:220-221)
    dq qq = qmk(mk(q[4 * i], q[4 * i + 1], q[4 * i + 2]), q[4 * i + 3]);
    d3 wb = multToVector3(conj(qq), vecq(mk(w[3 * i], w[3 * i + 1], w[3 * i + 2]), qq));
    st3(S.wbf, cap, i, wb);
  }
}

// AllComponents::ComputeMaxMeanVelocity (Component/src/AllComponents.cpp:
// 1781-1811): block partial max and sum of |v|, reduced in a fixed order.
__global__ void k_vstats_partial(DevState S, double* part) {
  __shared__ double smax[256], ssum[256];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double vit = 0.;
  if (i < S.n) vit = norm(ld3(S.v, S.cap, i));
  smax[threadIdx.x] = vit;
  ssum[threadIdx.x] = vit;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + o]);
      ssum[threadIdx.x] += ssum[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = smax[0]; part[2 * blockIdx.x + 1] = ssum[0]; }
}
__global__ void k_vstats_final(const double* part, int nparts, int n, double* out) {
  __shared__ double smax[256], ssum[256];
  double m = 0., s = 0.;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) { m = fmax(m, part[2 * k]); s += part[2 * k + 1]; }
  smax[threadIdx.x] = m;
  ssum[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + o]);
      ssum[threadIdx.x] += ssum[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) { out[0] = smax[0]; out[1] = n > 0 ? ssum[0] / n : 0.; }
}

// Sum of the pair-list segment lengths and count of live history keys.
__global__ void k_pair_counts(DevState S, unsigned long long* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long e = 0, c = 0;
  if (i < S.n) e = (unsigned long long)S.npairs[i];
  int cap = 1 << S.hist_old.log2cap;
  for (int k = i; k < cap; k += gridDim.x * blockDim.x) c += S.hist_old.keys[k] != kEmptyKey;
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, o);
    c += __shfl_down_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) { atomicAdd(&out[0], e); atomicAdd(&out[1], c); }
}

}  // namespace

inline int blocks(int n, int b) { return (n + b - 1) / b; }

void launch_pair_counts(DevState const& S, unsigned long long* out, cudaStream_t st) {
  cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), st);
  k_pair_counts<<<blocks(std::max(S.n, 1), 256), 256, 0, st>>>(S, out);
}

void launch_load_state(DevState const& S, const double* x, const double* v, const double* w,
                       const double* wbf, const double* q, const double* F, const double* T,
                       const int* type_by_id, const int* inst_by_id, cudaStream_t st) {
  if (S.n) k_load_state<<<blocks(S.n, 256), 256, 0, st>>>(S, x, v, w, wbf, q, F, T, type_by_id, inst_by_id);
}
void launch_vstats(DevState const& S, double* part, double* out, cudaStream_t st) {
  int nb = blocks(S.n, 256);
  k_vstats_partial<<<nb, 256, 0, st>>>(S, part);
  k_vstats_final<<<1, 256, 0, st>>>(part, nb, S.n, out);
}

void launch_key(DevState const& S, double h, double dt, int pre_kick, double pre_h, cudaStream_t st) {
  if (S.n) k_key<<<blocks(S.n, 256), 256, 0, st>>>(S, h, dt, pre_kick, pre_h);
}
void launch_bin(DevState const& S, cudaStream_t st) {
  if (S.n) k_bin<<<blocks(S.n, 256), 256, 0, st>>>(S);
}
void launch_kick(DevState const& S, double h, cudaStream_t st) {
  if (S.n) k_kick<<<blocks(S.n, 256), 256, 0, st>>>(S, h);
}
void launch_scan(DevState const& S, cudaStream_t st) {
  int ntiles = blocks(S.ncells, kScanTile);
  k_scan_tiles<<<ntiles, kScanTile, 0, st>>>(S.cell_count, S.cell_start, S.scan_tmp, S.ncells);
  k_scan_sums<<<1, kScanTile, 0, st>>>(S.scan_tmp, ntiles);
  k_scan_add<<<ntiles, kScanTile, 0, st>>>(S.cell_start, S.scan_tmp, S.cell_count, S.ncells);
}
void launch_place(DevState const& S, cudaStream_t st) {
  if (S.n) k_place<<<blocks(S.n, 256), 256, 0, st>>>(S);
}
void launch_cellsort(DevState const& S, cudaStream_t st) {
  k_cellsort<<<blocks(S.ncells, 256), 256, 0, st>>>(S);
}
void launch_move_gather(DevState const& S, int moving, double h, double dt, int pre_kick,
                        double pre_h, cudaStream_t st) {
  if (S.n) k_move_gather<<<blocks(S.n, 256), 256, 0, st>>>(S, moving, h, dt, pre_kick, pre_h);
}
void launch_scatter_by_id(DevState const& S, double* x, double* v, double* w, double* wbf,
                          double* q, double* F, double* T, int id_base, cudaStream_t st) {
  if (S.n) k_scatter_by_id<<<blocks(S.n, 256), 256, 0, st>>>(S, x, v, w, wbf, q, F, T, id_base);
}
void launch_basis_by_id(DevState const& S, double* out, int id_base, cudaStream_t st) {
  if (S.n && S.basis) k_basis_by_id<<<blocks(S.n, 256), 256, 0, st>>>(S, out, id_base);
}
void launch_cells_by_id(DevState const& S, int* ijk, int id_base, cudaStream_t st) {
  if (S.n) k_cells_by_id<<<blocks(S.n, 256), 256, 0, st>>>(S, ijk, id_base);
}
void launch_hist_zero_cumulative(HistTable const& t, int fp64, cudaStream_t st) {
  int cap = 1 << t.log2cap;
  if (fp64) k_hist_zero_cumulative<double><<<blocks(cap, 256), 256, 0, st>>>(t);
  else k_hist_zero_cumulative<float><<<blocks(cap, 256), 256, 0, st>>>(t);
}

}  // namespace gdem
