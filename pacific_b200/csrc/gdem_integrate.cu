// gdem_integrate.cu -- leapfrog move and pair-list rebuild kernels.
//
// Compiled with -fmad=false: positions, velocities and cell indices are FP64
// and follow the reference's expression order, so cell assignments are
// bit-identical to Cell::GetCell on the same state.
//
// A step is (host side, gdem_host.cu): k_decide, then -- only when some
// particle has moved more than half the pair-list skin since the last
// rebuild -- the rebuild below, then k_filter, the force kernel
// (gdem_contact64.cu / gdem_contact32.cu) and k_move.
//
//   k_decide    turns the rebuild request of the previous step into this
//               step's decision (and the CUDA-graph condition), and counts
//               the force evaluation (contact-history tag).
//   k_bin       pair-list cell of each particle and the cell histogram.
//   scan/place/cellsort
//               counting sort of particles on their cell key: a one-digit
//               radix sort whose digit is the cell key, made stable by
//               ordering each cell's entries by particle ID; it yields the
//               cell start/end tables.
//   k_permute / k_copyback
//               the whole state into cell order (through the second
//               buffers), with the compact copies the pair search reads.
//   k_pairs_*   (gdem_contact64/32.cu) the rows of the skin pair list:
//               counted, placed by a scan of the counts, written; k_link
//               then records where each pair of the compact list sits in
//               its partner's row.
//   k_filter    lists the pairs of the skin list whose bounding spheres
//               overlap now, and the particles near a wall, and marks them
//               as candidates; the pair kernel (gdem_contact64/32.cu)
//               evaluates them exactly and writes each contact's two shares
//               into the partners' rows.
//   k_move      the leapfrog of each particle in place: its force and torque
//               as the weight plus its shares in row order, then the closing
//               kick of the step that ends and the opening kick + drift of
//               the next (SecondOrderLeapFrog::Move / advanceVelocity,
//               ParticleKinematics::Move).
// Rebuild kernels take a gate: with a non-null gate they return at once
// unless this step rebuilds (plain launches); inside the graph's conditional
// node they run ungated.
#include <algorithm>

#include "gdem_kernels.cuh"
#include "gdem_motion.cuh"

namespace gdem {

namespace {

__device__ __forceinline__ bool gatedOff(const int* gate) { return gate && !*gate; }

__global__ void k_decide(DevState S, cudaGraphConditionalHandle h, int use_handle) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int need = S.ctl[kCtlNeed];
  S.ctl[kCtlActive] = need;
  S.ctl[kCtlNeed] = 0;
  S.ctl[kCtlEpoch] += 1;
  S.ctl[kCtlWork] = 0;
  S.ctl[kCtlKept] = 0;
  S.ctl[kCtlKeptCold] = 0;
  S.ctl[kCtlKept2] = 0;
  S.ctl[kCtlRebuilds] += need ? 1 : 0;
  if (need) S.ctl[kCtlPairs] = 0;
  if (use_handle) cudaGraphSetConditional(h, need ? 1u : 0u);
}

// Pair-list cell key of x (clamped into the grid; outside it raises
// kErrOutOfGrid like the reference's SimulationError).
__device__ __forceinline__ int buildKey(GridDesc const& bg, d3 x, int* status) {
  const double xs[3] = {x.x, x.y, x.z};
  int id[3];
  bool valid = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    id[d] = (int)floor((xs[d] - bg.lc_origin[d]) / bg.edge[d]);
    if (id[d] < 0 || id[d] >= bg.nb[d]) {
      valid = false;
      id[d] = min(max(id[d], 0), bg.nb[d] - 1);
    }
  }
  if (!valid) raise(status, kErrOutOfGrid);
  return bg.cell_offset + id[1] * bg.nb[2] * bg.nb[0] + id[2] * bg.nb[0] + id[0];
}

__global__ void k_bin(DevState S, const int* gate) {
  if (gatedOff(gate)) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n) return;
  const int key = buildKey(S.bgrids[S.inst[s]], ld3(S.x, S.cap, s), S.status);
  S.skey[s] = key;
  S.rank[s] = atomicAdd(&S.cell_count[key], 1);
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

__global__ void k_scan_tiles(const int* in, int* out, int* tile_sums, int n, const int* gate) {
  if (gatedOff(gate)) return;
  __shared__ int smem[32];
  int i = blockIdx.x * kScanTile + threadIdx.x;
  int v = i < n ? in[i] : 0;
  int total;
  int ex = blockExclusiveScan(v, smem, total);
  if (i < n) out[i] = ex;
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Scans the tile sums in place with one block, looping over chunks.
__global__ void k_scan_sums(int* sums, int ntiles, const int* gate) {
  if (gatedOff(gate)) return;
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
__global__ void k_scan_add(int* out, const int* tile_sums, const int* in, int n,
                           const int* gate, int* ctl) {
  if (gatedOff(gate)) return;
  int i = blockIdx.x * kScanTile + threadIdx.x;
  if (i < n) {
    int v = out[i] + tile_sums[blockIdx.x];
    out[i] = v;
    if (i == n - 1) {
      // (a total beyond 2^31 - 1 wraps negative: the rows then do not fit)
      const int total = v + in[i];
      out[n] = total;
      if (ctl) {
        ctl[kCtlEntries] = total;
        atomicMax(&ctl[kCtlEntriesMax], total < 0 ? INT_MAX : total);
      }
    }
  }
}

__global__ void k_place(DevState S, const int* gate) {
  if (gatedOff(gate)) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n) return;
  S.order[S.cell_start[S.skey[s]] + S.rank[s]] = s;
}

// Orders each cell's entries by particle ID, so the permutation does not
// depend on the arrival order of the atomic histogram.  It also resets the
// cell histogram for the next rebuild (every count has been consumed by the
// scan at this point).
__global__ void k_cellsort(DevState S, const int* gate) {
  if (gatedOff(gate)) return;
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

// Gathers the state into cell order (second buffers) and writes the compact
// arrays of the pair search: the cell, the FP64 position + radius (FP64
// mode) or the FP32 offset from the cell's lower corner + radius (FP32-split).
__global__ void k_permute(DevState S, const int* gate) {
  if (gatedOff(gate)) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  const int cap = S.cap;
  const int s = S.order[t];
  const int ty = S.type[s], in = S.inst[s];
  S.id2[t] = S.id[s]; S.type2[t] = ty; S.inst2[t] = in;
  const d3 x = ld3(S.x, cap, s);
  st3(S.x2, cap, t, x);
  st3(S.v2, cap, t, ld3(S.v, cap, s));
  st3(S.w2, cap, t, ld3(S.w, cap, s));
  if (S.wbf_state) st3(S.wbf2, cap, t, ld3(S.wbf, cap, s));
  st3(S.F2, cap, t, ld3(S.F, cap, s));
  st3(S.T2, cap, t, ld3(S.T, cap, s));
#pragma unroll
  for (int k = 0; k < 4; ++k) S.q2[k * cap + t] = S.q[k * cap + s];
  if (S.basis) {
#pragma unroll
    for (int k = 0; k < 9; ++k) S.basis2[k * cap + t] = S.basis[k * cap + s];
  }
  if (S.curv) S.curv2[t] = S.curv[s];
  GridDesc const& bg = S.bgrids[in];
  const int c = S.skey[s] - bg.cell_offset;
  const int ci = c % bg.nb[0];
  const int ck = (c / bg.nb[0]) % bg.nb[2];
  const int cj = c / (bg.nb[0] * bg.nb[2]);
  S.cellc[t] = make_int4(ci, cj, ck, in);
  TypeDesc const& tp = S.types[ty];
  if (S.pos64) S.pos64[t] = make_double4(x.x, x.y, x.z, tp.radius);
  if (S.offh) {
    S.offh[t] = make_float4((float)(x.x - (bg.lc_origin[0] + ci * bg.edge[0])),
                            (float)(x.y - (bg.lc_origin[1] + cj * bg.edge[1])),
                            (float)(x.z - (bg.lc_origin[2] + ck * bg.edge[2])), tp.r_f);
  }
}

// Second buffers back into the current ones; the wraps since the rebuild
// start again from zero and the FP32 position becomes the rebuild's.
__global__ void k_copyback(DevState S, const int* gate) {
  if (gatedOff(gate)) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  const int cap = S.cap;
  S.id[t] = S.id2[t]; S.type[t] = S.type2[t]; S.inst[t] = S.inst2[t];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const size_t k = (size_t)d * cap + t;
    S.x[k] = S.x2[k]; S.v[k] = S.v2[k]; S.w[k] = S.w2[k];
    if (S.wbf_state) S.wbf[k] = S.wbf2[k];
    S.F[k] = S.F2[k]; S.T[k] = S.T2[k];
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) S.q[k * cap + t] = S.q2[k * cap + t];
  if (S.basis) {
#pragma unroll
    for (int k = 0; k < 9; ++k) S.basis[k * cap + t] = S.basis2[k * cap + t];
  }
  if (S.curv) S.curv[t] = S.curv2[t];
  S.wrap[t] = 0;
  const d3 x = ld3(S.x, cap, t);
  const float4 p = make_float4((float)x.x, (float)x.y, (float)x.z,
                               (float)S.types[S.type[t]].radius);
  S.posf[t] = p;
  S.posf0[t] = p;
}

// Force and torque of particle t in this evaluation: its weight plus the
// shares the pair kernel wrote into its row, in row order, then its wall
// share.  The entry bits of the flag word name the shares of the first
// kMaskEntries entries, so their loads are issued together, two at a time
// (a particle rarely has more contacts, and larger batches spill);
// entries beyond (kFarEntry) are found by their evaluation tags.  FP32-split
// (kFast): FP32 shares summed in FP32; FP64: FP64 shares summed in FP64 onto
// the weight.
template <bool kFast>
__device__ __forceinline__ void sumShares(DevState const& S, int t, TypeDesc const& tp,
                                          unsigned na, int off, int tag, d3& F, d3& T) {
  constexpr int kBatch = 2;
  if constexpr (kFast) {
    float fx = 0.f, fy = 0.f, fz = 0.f, tx = 0.f, ty = 0.f, tz = 0.f;
    const float4* sh = static_cast<const float4*>(S.share) + 2 * (size_t)off;
    unsigned m = na & kEntryBits;
    while (m) {
      float4 a[kBatch], b[kBatch];
      int cnt = 0;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        if (m) {
          const int e = __ffs(m) - 1;
          m &= m - 1u;
          a[j] = sh[2 * e];
          b[j] = sh[2 * e + 1];
          cnt = j + 1;
        }
      }
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        if (j < cnt) {
          fx += a[j].x; fy += a[j].y; fz += a[j].z;
          tx += b[j].x; ty += b[j].y; tz += b[j].z;
        }
      }
    }
    if (na & kFarEntry) {
      const int np = S.npairs[t];
      for (int e = kMaskEntries; e < np; ++e) {
        const float4 a = sh[2 * e];
        if (__float_as_int(a.w) != tag) continue;
        const float4 b = sh[2 * e + 1];
        fx += a.x; fy += a.y; fz += a.z;
        tx += b.x; ty += b.y; tz += b.z;
      }
    }
    if (na & kNearWall) {
      const float4* ws = static_cast<const float4*>(S.wshare) + 2 * (size_t)t;
      const float4 a = ws[0], b = ws[1];
      fx += a.x; fy += a.y; fz += a.z;
      tx += b.x; ty += b.y; tz += b.z;
    }
    F = mk(tp.weight[0] + (double)fx, tp.weight[1] + (double)fy, tp.weight[2] + (double)fz);
    T = mk((double)tx, (double)ty, (double)tz);
  } else {
    F = mk(tp.weight[0], tp.weight[1], tp.weight[2]);
    T = mk(0., 0., 0.);
    const double2* sh = static_cast<const double2*>(S.share) + 4 * (size_t)off;
    unsigned m = na & kEntryBits;
    while (m) {
      double2 a[kBatch], b[kBatch], c[kBatch], d[kBatch];
      int cnt = 0;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        if (m) {
          const int e = __ffs(m) - 1;
          m &= m - 1u;
          a[j] = sh[4 * e]; b[j] = sh[4 * e + 1]; c[j] = sh[4 * e + 2]; d[j] = sh[4 * e + 3];
          cnt = j + 1;
        }
      }
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        if (j < cnt) {
          F = F + mk(a[j].y, b[j].x, b[j].y);
          T = T + mk(c[j].x, c[j].y, d[j].x);
        }
      }
    }
    if (na & kFarEntry) {
      const int np = S.npairs[t];
      for (int e = kMaskEntries; e < np; ++e) {
        const double2 a = sh[4 * e];
        if ((int)__double_as_longlong(a.x) != tag) continue;
        const double2 b = sh[4 * e + 1], c = sh[4 * e + 2], d = sh[4 * e + 3];
        F = F + mk(a.y, b.x, b.y);
        T = T + mk(c.x, c.y, d.x);
      }
    }
    if (na & kNearWall) {
      const double2* ws = static_cast<const double2*>(S.wshare) + 3 * (size_t)t;
      const double2 a = ws[0], b = ws[1], c = ws[2];
      F = F + mk(a.x, a.y, b.x);
      T = T + mk(b.y, c.x, c.y);
    }
  }
}

// Threads per block of k_move.
template <bool kFast, bool kBasis>
constexpr int kMoveBlock() { return kBasis ? 256 : 128; }

// Leapfrog of each particle (128-thread blocks: FP32-split spheres eight per
// multiprocessor at 64 registers, FP64 six at 80; both measured faster at 1M
// than 256-thread blocks -- three, four or five per multiprocessor for
// FP32-split, three or four for FP64; the kernel is bound by the latency of
// its loads).  FP32-split with an orientation matrix: two 256-thread blocks.  With kStepSum the force and torque of this
// evaluation: the weight for a particle the contact filter did not mark as a
// candidate, else the weight plus its shares (sumShares); without it, the
// stored F, T (the opening kick of a call continues from the last evaluation
// of the previous one).  Then the closing kick of the step that ends
// (flags & kStepClose) and the opening kick + drift of the next
// (flags & kStepMove); kStepStoreFT writes F, T back (the last evaluation of
// a call, and the leapfrog start, which only stores them).  Per particle
// only, so it runs in place (the launcher aliases the second buffers to the
// current ones).
//
// The kernel starts while the pair kernel still runs (programmatic launch:
// the pair kernel triggers after its own wait, so the filter has completed
// and its candidate marks are final).  A particle that is not a candidate
// takes no share and is not read by the pair kernel, so its leapfrog runs at
// once; a candidate waits for the pair kernel before it reads its shares.
template <bool kFast, bool kBasis>
__global__ void __launch_bounds__(kMoveBlock<kFast, kBasis>(), (kFast && kBasis) ? 2 : (kFast ? 8 : 6))
    k_move(DevState S, int flags) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  TypeDesc const& tp = S.types[S.type[t]];
  MoveIn m;
  loadMoveIn<kFast, kBasis>(S, t, m);   // nothing the contact kernels write
  const bool sum = (flags & kStepSum) != 0;
  d3 F, T;
  bool candidate = false;
  if (sum) {
    int* fl = contactFlags(S);
    candidate = ((unsigned)fl[t] & kCandidate) != 0u;
    if (!candidate) {
      F = mk(tp.weight[0], tp.weight[1], tp.weight[2]);
      T = mk(0., 0., 0.);
    } else {
      // the row of t (written by the last rebuild, before the filter)
      const int off = S.pair_off[t];
      pdlWait();
      sumShares<kFast>(S, t, tp, (unsigned)fl[t], off, S.ctl[kCtlEpoch], F, T);
    }
    if (flags & kStepStoreFT) { st3(S.F, S.cap, t, F); st3(S.T, S.cap, t, T); }
  } else {
    pdlWait();
    F = ld3(S.F, S.cap, t);
    T = ld3(S.T, S.cap, t);
  }
  if (S.hydro) {
    // coupled run: the fluid's force and torque, added after the contacts as
    // the PRSHydroFT application does (it runs after the collision one)
    const double* hy = S.hydro + 6 * (size_t)S.id[t];
    F = F + mk(hy[0], hy[1], hy[2]);
    T = T + mk(hy[3], hy[4], hy[5]);
  }
  if (flags & (kStepClose | kStepMove))
    advanceParticle<kFast, kBasis>(S, t, tp, F, T, (flags & kStepClose) != 0,
                                   (flags & kStepMove) != 0, m);
  // the next evaluation's flag words start clear (no other kernel touches
  // that buffer until the next contact filter)
  contactFlags(S, 1)[t] = 0;
  if (candidate && S.curv_next) {
    // the polyhedron vertex this evaluation's GJK calls left (recordVertex;
    // only candidates take part in GJK calls)
    const int r = S.curv_next[t];
    if (r) {
      S.curv[t] = r & 0xFFFF;
      S.curv_next[t] = 0;
    }
  }
}

// Contact filter.  One lane per pair of the compact pair list (each pair
// once, from its lower ID): the FP32 bounding-sphere test, a superset of the
// contacts; the kept pairs are listed for the pair kernel, which decides each
// exactly, and both partners marked as candidates.  With walls, the first
// pblocks blocks take one particle per thread and list (and mark) those near
// a wall.  The pairs are taken in chunks of kFilterUnroll rounds of 32 per
// warp with their loads issued together, in a grid-stride loop over chunks
// (the count is known on the device only) on a grid of one block per 2,048
// pairs at the leapfrog start (kFilterPairsPerBlock; the host resizes it
// then).  Measured at 1M spheres: one round per chunk and that grid take
// 21.3 us, four rounds on a grid of one block per 1,024 pairs 27.0 us (the
// kernel is bound by the latency of its gathers: fewer registers, more warps).
constexpr int kFilterUnroll = 1;
constexpr int kFilterPairsPerBlock = 2048;

// Appends idx to list (length *count) for every lane whose pred holds (one
// atomic per warp); every lane of the warp calls it.
__device__ __forceinline__ void appendList(int* list, int* count, bool pred, int idx) {
  const unsigned m = __ballot_sync(0xffffffffu, pred);
  if (!m) return;
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == 0) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (pred) list[base + __popc(m & ((1u << lane) - 1u))] = idx;
}

// Appends idx below list[0] (list[-1], list[-2], ...: a list growing
// downwards from its last slot), for every lane whose pred holds; every lane
// of the warp calls it.
__device__ __forceinline__ void appendListBack(int* list, int* count, bool pred, int idx) {
  const unsigned m = __ballot_sync(0xffffffffu, pred);
  if (!m) return;
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == 0) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (pred) list[-(base + __popc(m & ((1u << lane) - 1u)))] = idx;
}

// Whether particle t (posf: its FP32 continuous position) comes within the
// margin of a wall box of its instance: the wall contacts can only come
// from such particles.
__device__ __forceinline__ bool nearWall(DevState const& S, int t) {
  const int inst = S.inst[t];
  GridDesc const& g = S.grids[inst];
  if (!g.wall_count) return false;
  // the centre wrapped back into the box, against the bounding radius
  GridDesc const& bg = S.bgrids[inst];
  const float4 pt = S.posf[t];
  const int wt = S.wrap[t];
  const float q[3] = {pt.x - (float)wrapGet(wt, 0) * bg.Lf[0],
                      pt.y - (float)wrapGet(wt, 1) * bg.Lf[1],
                      pt.z - (float)wrapGet(wt, 2) * bg.Lf[2]};
  for (int w = 0; w < g.wall_count; ++w) {
    WallDesc const& wd = S.walls[g.wall_begin + w];
    float d2 = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float o = fabsf(q[d] - (float)wd.centre[d]) - (float)wd.extent[d];
      if (o > 0.f) d2 += o * o;
    }
    const float R = pt.w + bg.filt_margin;
    if (d2 <= R * R) return true;
  }
  return false;
}

__global__ void __launch_bounds__(256) k_filter(DevState S, int pblocks) {
  pdlTrigger();   // the pair kernel may be scheduled; it waits for this one
  const int lane = threadIdx.x & 31;
  unsigned* flags = reinterpret_cast<unsigned*>(contactFlags(S));
  if ((int)blockIdx.x < pblocks) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool near = t < S.n && nearWall(S, t);
    if (near) atomicOr(&flags[t], kCandidate);
    appendList(S.work, S.ctl + kCtlWork, near, t);
    return;
  }
  const int np = S.ctl[kCtlPairs];
  constexpr int chunk = 32 * kFilterUnroll;
  const long long wq = ((long long)((int)blockIdx.x - pblocks) * blockDim.x + threadIdx.x) >> 5;
  const long long nwq = ((long long)(gridDim.x - pblocks) * blockDim.x) >> 5;
  for (long long c0l = wq * chunk; c0l < np; c0l += nwq * chunk) {   // warp-uniform
    const int c0 = (int)c0l;
    int2 pr[kFilterUnroll];
    float4 pa[kFilterUnroll], pb[kFilterUnroll];
#pragma unroll
    for (int j = 0; j < kFilterUnroll; ++j) {
      const int i = c0 + 32 * j + lane;
      pr[j] = i < np ? S.upairs[i] : make_int2(0, 0);
    }
#pragma unroll
    for (int j = 0; j < kFilterUnroll; ++j) {
      pa[j] = pb[j] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (c0 + 32 * j + lane < np) {
        pa[j] = S.posf[pr[j].x];
        pb[j] = S.posf[(unsigned)pr[j].y & ((1u << 27) - 1u)];
      }
    }
#pragma unroll
    for (int j = 0; j < kFilterUnroll; ++j) {
      const int t = pr[j].x, u = (int)((unsigned)pr[j].y & ((1u << 27) - 1u));
      bool keep = false;
      if (c0 + 32 * j + lane < np) {
        // the largest margin of the instances (a superset of the contacts);
        // the period only for an entry with an image shift (code 13 is
        // none), which needs the instance's grid
        const unsigned code = (unsigned)pr[j].y >> 27;
        float sx = 0.f, sy = 0.f, sz = 0.f;
        if (code != 13u) {
          GridDesc const& bg = S.bgrids[S.inst[t]];
          sx = (float)((int)(code % 3u) - 1) * bg.Lf[0];
          sy = (float)((int)((code / 3u) % 3u) - 1) * bg.Lf[1];
          sz = (float)((int)(code / 9u) - 1) * bg.Lf[2];
        }
        const float dx = (pb[j].x - pa[j].x) + sx;
        const float dy = (pb[j].y - pa[j].y) + sy;
        const float dz = (pb[j].z - pa[j].z) + sz;
        const float R = pa[j].w + pb[j].w + S.filt_margin_max;
        keep = dx * dx + dy * dy + dz * dz <= R * R;
      }
      if (keep) {
        atomicOr(&flags[t], kCandidate);
        atomicOr(&flags[u], kCandidate);
      }
      if (S.any_convex && !S.pos64) {
        // FP32-split with non-spherical classes: a pair in contact at the
        // last evaluation (its share on t's side carries that evaluation's
        // tag) goes to the front of the list, the others to the back, so the
        // pair kernel runs the full closest-point searches and laws of the
        // likely contacts in warps of their own and the searches that stop
        // early in others (measured: 3 % off the convex pour's FP32-split
        // step; the FP64 step, whose searches all run to their end, was 1 %
        // slower with it).  A guess that a rebuild made stale only reorders.
        bool hot = false;
        if (keep) {
          const int c = c0 + 32 * j + lane;
          const long long e = (long long)S.pair_off[t] + (S.epos[c] & 0xFFFF);
          hot = __float_as_int(static_cast<const float4*>(S.share)[2 * e].w) ==
                S.ctl[kCtlEpoch] - 1;
        }
        appendList(S.kept, S.ctl + kCtlKept, keep && hot, c0 + 32 * j + lane);
        appendListBack(S.kept + (S.pair_cap / 2), S.ctl + kCtlKeptCold, keep && !hot,
                       c0 + 32 * j + lane);
      } else {
        appendList(S.kept, S.ctl + kCtlKept, keep, c0 + 32 * j + lane);
      }
    }
  }
}

// Where each pair of the compact list sits in its partner's row: the entry of
// the lower-ID slot t in the row of u (rows are symmetric: the pair search
// decides both directions with the same expression).  0xFFFF when absent (a
// row emptied for lack of room).  Grid-stride over the pairs, whose count is
// known on the device only.
__global__ void __launch_bounds__(256) k_link(DevState S, const int* gate) {
  if (gatedOff(gate)) return;
  const int np = S.ctl[kCtlPairs];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
    const int2 pr = S.upairs[k];
    const int t = pr.x;
    const int u = (int)((unsigned)pr.y & ((1u << 27) - 1u));
    const int nu = S.npairs[u];
    const int* row = S.pairs + S.pair_off[u];
    int eu = 0xFFFF;
    for (int e = 0; e < nu; ++e)
      if ((int)((unsigned)row[e] & ((1u << 27) - 1u)) == t) { eu = e; break; }
    S.epos[k] = (S.epos[k] & 0xFFFF) | (eu << 16);
  }
}

// Diagnostics: every entry and wall slot starts at +inf (no contact); the
// pair kernel records the pairs it evaluates.
__global__ void k_diag_prefill(DevState S) {
  const double inf = __longlong_as_double(0x7ff0000000000000ll);
  const long long ne = S.ctl[kCtlEntries] < 0 ? 0 : min(S.ctl[kCtlEntries], S.pair_cap);
  const long long nw = (long long)S.n * S.max_walls;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ne + nw; i += stride) {
    if (i < ne) S.pair_delta[i] = inf;
    else S.wall_delta[i - ne] = inf;
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
  if (out_wbf && !S.wbf_state) {
    // q* w q (ParticleKinematics.cpp:220-221), the body-frame image of the state w
    const dq qq = qmk(mk(S.q[t], S.q[cap + t], S.q[2 * cap + t]), S.q[3 * cap + t]);
    const d3 wb = multToVector3(conj(qq), vecq(ld3(S.w, cap, t), qq));
    out_wbf[3 * i] = wb.x; out_wbf[3 * i + 1] = wb.y; out_wbf[3 * i + 2] = wb.z;
    out_wbf = nullptr;
  }
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

// Reference-grid cell (Cell::GetCell) of each particle, by ID.
__global__ void k_cells_by_id(DevState S, int* ijk, int id_base) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  int i = S.id[t] - id_base;
  if (i < 0 || i >= S.n) return;
  GridDesc const& g = S.grids[S.inst[t]];
  const d3 x = ld3(S.x, S.cap, t);
  const double xs[3] = {x.x, x.y, x.z};
#pragma unroll
  for (int d = 0; d < 3; ++d) ijk[3 * i + d] = (int)floor((xs[d] - g.lc_origin[d]) / g.edge[d]);
}

// Coordination number of each particle at the last force evaluation, by ID:
// the listed partners and the walls whose overlap recorded by that
// evaluation is negative.  The reference counts the distinct components a
// particle touched in its force computation (Particle::
// addContactingComponentID, Component/src/Particle.cpp:1702-1706, called by
// Particle::InterAction and SimpleObstacle::InterAction for each contact of
// negative overlap, Particle.cpp:530-543, SimpleObstacle.cpp:262-270); the
// pair list holds each partner once and each wall has one slot.
__global__ void k_coordination_by_id(DevState S, int* out, int id_base) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  int i = S.id[t] - id_base;
  if (i < 0 || i >= S.n) return;
  const int np = S.npairs[t];
  const double* pd = S.pair_delta + S.pair_off[t];
  int c = 0;
  for (int e = 0; e < np; ++e) c += pd[e] < 0. ? 1 : 0;
  const int nw = S.grids[S.inst[t]].wall_count;
  const double* wd = S.wall_delta + (size_t)t * S.max_walls;
  for (int k = 0; k < nw; ++k) c += wd[k] < 0. ? 1 : 0;
  out[i] = c;
}

// Zeroes the cumulative tangential and rolling memories of every entry of
// the given evaluation (Component::setContactMapCumulativeFeaturesToZero,
// Component.cpp:842-851).
template <typename V>
__global__ void k_hist_zero_cumulative(HistTable t, const int* ctl) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= (1 << t.log2cap)) return;
  if (tagOf(t.keys[s]) != ((unsigned)ctl[kCtlEpoch] & kTagMask)) return;
  V* v = static_cast<V*>(t.vals) + 9 * (size_t)s;
  v[0] = v[1] = v[2] = 0;
  v[6] = v[7] = v[8] = 0;
}

__global__ void k_fill64(unsigned long long* p, size_t n, unsigned long long value) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = value;
}

// Orientation matrix of the quaternion q (x, y, z, w) with the expression
// order of Matrix::setRotation (Geometry/src/Matrix.cpp:114-127).
__device__ __forceinline__ void basisOfQuaternion(const double* q, double* m) {
  const double x = q[0], y = q[1], z = q[2], w4 = q[3];
  const double s = 2.0 / (x * x + y * y + z * z + w4 * w4);
  const double xs = x * s, ys = y * s, zs = z * s;
  const double wx = w4 * xs, wy = w4 * ys, wz = w4 * zs;
  const double xx = x * xs, xy = x * ys, xz = x * zs, yy = y * ys, yz = y * zs, zz = z * zs;
  m[0] = 1.0 - (yy + zz); m[1] = xy - wz; m[2] = xz + wy;
  m[3] = xy + wz; m[4] = 1.0 - (xx + zz); m[5] = yz - wx;
  m[6] = xz - wy; m[7] = yz + wx; m[8] = 1.0 - (xx + yy);
}

// An inserted particle (Grains::insertParticle, Base/src/Grains.cpp:
// 2063-2139) written into slot p.slot, after the others: position,
// velocities, quaternion and its orientation matrix (or the given one), the
// body-frame angular velocity q* w q, its weight as force and a zero torque
// (Particle::InitializeForce(true)), the start vertex of a new polyhedron,
// no displacement, wraps or contact marks.  The host asks for a pair-list
// rebuild before the next force evaluation.
__global__ void k_append_particle(DevState S, NewParticle p) {
  if (threadIdx.x || blockIdx.x) return;
  const int cap = S.cap, i = p.slot;
  TypeDesc const& tp = S.types[p.type];
  S.id[i] = p.id;
  S.type[i] = p.type;
  S.inst[i] = 0;
  const d3 x = mk(p.x[0], p.x[1], p.x[2]), w = mk(p.w[0], p.w[1], p.w[2]);
  st3(S.x, cap, i, x);
  st3(S.v, cap, i, mk(p.v[0], p.v[1], p.v[2]));
  st3(S.w, cap, i, w);
#pragma unroll
  for (int k = 0; k < 4; ++k) S.q[k * cap + i] = p.q[k];
  if (S.basis) {
    double m[9];
    if (p.has_basis) {
      for (int k = 0; k < 9; ++k) m[k] = p.basis[k];
    } else {
      basisOfQuaternion(p.q, m);
    }
    for (int k = 0; k < 9; ++k) S.basis[k * cap + i] = m[k];
  }
  const dq qq = qmk(mk(p.q[0], p.q[1], p.q[2]), p.q[3]);
  st3(S.wbf, cap, i, multToVector3(conj(qq), vecq(w, qq)));
  st3(S.F, cap, i, mk(tp.weight[0], tp.weight[1], tp.weight[2]));
  st3(S.T, cap, i, mk(0., 0., 0.));
  S.wrap[i] = 0;
  if (S.curv) {
    S.curv[i] = tp.poly_start;
    S.curv_next[i] = 0;
  }
  S.nact[i] = 0;
  S.nact[cap + i] = 0;
  const float4 pf = make_float4((float)x.x, (float)x.y, (float)x.z, (float)tp.radius);
  S.posf[i] = pf;
  S.posf0[i] = pf;
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
    // gdem_upload_basis may replace it
    double m[9];
    basisOfQuaternion(q + 4 * i, m);
#pragma unroll
    for (int k = 0; k < 9; ++k) S.basis[k * cap + i] = m[k];
  }
  // the host requests a pair-list rebuild after a load, which sets posf and
  // posf0 from these positions
  S.wrap[i] = 0;
  // a new (or reloaded) polyhedron starts its support search where
  // Polyhedron::BuildPolyhedron leaves it
  if (S.curv) S.curv[i] = S.types[type_by_id[i]].poly_start;
  if (!wbf) {
    // q* (w, q) (ParticleKinematics.cpp:220-221)
    dq qq = qmk(mk(q[4 * i], q[4 * i + 1], q[4 * i + 2]), q[4 * i + 3]);
    d3 wb = multToVector3(conj(qq), vecq(mk(w[3 * i], w[3 * i + 1], w[3 * i + 2]), qq));
    st3(S.wbf, cap, i, wb);
  }
}

// GrainsCoupledWithFluid::updateParticlesVelocity (Fluid/src/
// GrainsCoupledWithFluid.cpp:1126-1180): velocities and space-frame angular
// velocities by particle ID (AoS), the body-frame one rebuilt as q* w q.
__global__ void k_set_velocities(DevState S, const double* v, const double* w) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.n) return;
  const int cap = S.cap, i = S.id[t];
  const d3 vi = mk(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
  const d3 wi = mk(w[3 * i], w[3 * i + 1], w[3 * i + 2]);
  st3(S.v, cap, t, vi);
  st3(S.w, cap, t, wi);
  if (S.wbf_state) {
    const dq qq = qmk(mk(S.q[t], S.q[cap + t], S.q[2 * cap + t]), S.q[3 * cap + t]);
    st3(S.wbf, cap, t, multToVector3(conj(qq), vecq(wi, qq)));
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

// Sum of the pair-list segment lengths and count of the history keys of
// the last force evaluation.
__global__ void k_pair_counts(DevState S, unsigned long long* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long e = 0, c = 0;
  if (i < S.n) e = (unsigned long long)S.npairs[i];
  const unsigned tag = (unsigned)S.ctl[kCtlEpoch] & kTagMask;
  int cap = 1 << S.hist_old.log2cap;
  for (int k = i; k < cap; k += gridDim.x * blockDim.x) c += tagOf(S.hist_old.keys[k]) == tag;
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, o);
    c += __shfl_down_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) { atomicAdd(&out[0], e); atomicAdd(&out[1], c); }
}

}  // namespace

inline int blocks(int n, int b) { return (n + b - 1) / b; }

void launch_decide(DevState const& S, cudaGraphConditionalHandle h, int use_handle,
                   cudaStream_t st) {
  k_decide<<<1, 32, 0, st>>>(S, h, use_handle);
}
void launch_bin(DevState const& S, const int* gate, cudaStream_t st) {
  if (S.n) k_bin<<<blocks(S.n, 256), 256, 0, st>>>(S, gate);
}
void launch_scan(DevState const& S, const int* gate, cudaStream_t st) {
  int ntiles = blocks(S.ncells, kScanTile);
  k_scan_tiles<<<ntiles, kScanTile, 0, st>>>(S.cell_count, S.cell_start, S.scan_tmp, S.ncells, gate);
  k_scan_sums<<<1, kScanTile, 0, st>>>(S.scan_tmp, ntiles, gate);
  k_scan_add<<<ntiles, kScanTile, 0, st>>>(S.cell_start, S.scan_tmp, S.cell_count, S.ncells, gate,
                                           nullptr);
}
void launch_row_scan(DevState const& S, const int* gate, cudaStream_t st) {
  if (!S.n) return;
  int ntiles = blocks(S.n, kScanTile);
  k_scan_tiles<<<ntiles, kScanTile, 0, st>>>(S.npairs, S.pair_off, S.pair_scan_tmp, S.n, gate);
  k_scan_sums<<<1, kScanTile, 0, st>>>(S.pair_scan_tmp, ntiles, gate);
  k_scan_add<<<ntiles, kScanTile, 0, st>>>(S.pair_off, S.pair_scan_tmp, S.npairs, S.n, gate, S.ctl);
}
void launch_filter(DevState const& S, cudaStream_t st) {
  if (!S.n) return;
  const int pblocks = S.any_walls ? blocks(S.n, 256) : 0;
  // about 4 pairs per particle until the leapfrog start has counted them
  const int qblocks = S.filter_qblocks > 0
                          ? S.filter_qblocks
                          : (4 * S.n + kFilterPairsPerBlock - 1) / kFilterPairsPerBlock;
  k_filter<<<pblocks + qblocks, 256, 0, st>>>(S, pblocks);
}
void launch_link(DevState const& S, const int* gate, cudaStream_t st) {
  if (S.n) k_link<<<4 * S.nsm, 256, 0, st>>>(S, gate);
}
void launch_diag_prefill(DevState const& S, cudaStream_t st) {
  if (S.n && S.pair_delta) k_diag_prefill<<<8 * S.nsm, 256, 0, st>>>(S);
}
void launch_place(DevState const& S, const int* gate, cudaStream_t st) {
  if (S.n) k_place<<<blocks(S.n, 256), 256, 0, st>>>(S, gate);
}
void launch_cellsort(DevState const& S, const int* gate, cudaStream_t st) {
  k_cellsort<<<blocks(S.ncells, 256), 256, 0, st>>>(S, gate);
}
void launch_permute(DevState const& S, const int* gate, cudaStream_t st) {
  if (S.n) k_permute<<<blocks(S.n, 256), 256, 0, st>>>(S, gate);
}
void launch_copyback(DevState const& S, const int* gate, cudaStream_t st) {
  if (S.n) k_copyback<<<blocks(S.n, 256), 256, 0, st>>>(S, gate);
}
void launch_move(DevState const& S, int flags, int fast, cudaStream_t st) {
  if (!S.n) return;
  DevState M = S;   // in place: the "next" buffers are the current ones
  M.x2 = S.x; M.v2 = S.v; M.w2 = S.w; M.wbf2 = S.wbf; M.q2 = S.q; M.basis2 = S.basis;
  M.wrap2 = S.wrap;
  const int nb = blocks(S.n, 256);
  if (!fast) launchAfterPrevious(k_move<false, false>, blocks(S.n, kMoveBlock<false, false>()), kMoveBlock<false, false>(), st, M, flags);   // basis tested at run time
  else if (S.basis) launchAfterPrevious(k_move<true, true>, nb, 256, st, M, flags);
  else launchAfterPrevious(k_move<true, false>, blocks(S.n, kMoveBlock<true, false>()), kMoveBlock<true, false>(), st, M, flags);
}
void launch_append_particle(DevState const& S, NewParticle const& p, cudaStream_t st) {
  k_append_particle<<<1, 32, 0, st>>>(S, p);
}
void launch_fill64(unsigned long long* p, size_t n, unsigned long long value, cudaStream_t st) {
  if (n) k_fill64<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, n, value);
}
void launch_pair_counts(DevState const& S, unsigned long long* out, cudaStream_t st) {
  cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), st);
  k_pair_counts<<<blocks(std::max(S.n, 1), 256), 256, 0, st>>>(S, out);
}
void launch_load_state(DevState const& S, const double* x, const double* v, const double* w,
                       const double* wbf, const double* q, const double* F, const double* T,
                       const int* type_by_id, const int* inst_by_id, cudaStream_t st) {
  if (S.n) k_load_state<<<blocks(S.n, 256), 256, 0, st>>>(S, x, v, w, wbf, q, F, T, type_by_id, inst_by_id);
}
void launch_set_velocities(DevState const& S, const double* v, const double* w, cudaStream_t st) {
  if (S.n) k_set_velocities<<<blocks(S.n, 256), 256, 0, st>>>(S, v, w);
}
void launch_vstats(DevState const& S, double* part, double* out, cudaStream_t st) {
  int nb = blocks(S.n, 256);
  if (nb) k_vstats_partial<<<nb, 256, 0, st>>>(S, part);   // (none: an empty system)
  k_vstats_final<<<1, 256, 0, st>>>(part, nb, S.n, out);
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
void launch_coordination_by_id(DevState const& S, int* out, int id_base, cudaStream_t st) {
  if (S.n) k_coordination_by_id<<<blocks(S.n, 256), 256, 0, st>>>(S, out, id_base);
}
// Contact memory of a step that does not prune it (GrainsCoupledWithFluid::
// Simulation, Fluid/src/GrainsCoupledWithFluid.cpp:135-205, runs the
// collision application without Grains::computeParticlesForceAndTorque's
// setContactMapToFalse / updateContactMap, Component/src/Component.cpp:
// 567-593): every entry of the previous evaluation's table that this
// evaluation did not rewrite -- a contact that has ended -- is carried into
// this evaluation's table unchanged, so that the pair, if it touches again,
// resumes its tangential spring.  Runs after the pair kernel.
template <typename T>
__global__ void k_hist_carry(HistTable old_t, HistTable new_t, const int* ctl, int* status) {
  const unsigned tag = (unsigned)ctl[kCtlEpoch], tag_old = tag - 1u;
  const size_t cap = size_t(1) << old_t.log2cap;
  const T* src = static_cast<const T*>(old_t.vals);
  T* dst = static_cast<T*>(new_t.vals);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap;
       i += (size_t)gridDim.x * blockDim.x) {
    const unsigned long long k = old_t.keys[i];
    if (tagOf(k) != (tag_old & kTagMask)) continue;
    const unsigned long long base = k & ((1ull << kTagShift) - 1ull);
    if (histFind(new_t, base, tag) >= 0) continue;   // rewritten this evaluation
    const int s = histInsert(new_t, base, tag);
    if (s < 0) { raise(status, kErrHashFull); continue; }
#pragma unroll
    for (int j = 0; j < 9; ++j) dst[(size_t)s * 9 + j] = src[i * 9 + j];
  }
}
void launch_hist_carry(DevState const& S, int fp64, cudaStream_t st) {
  if (fp64) k_hist_carry<double><<<4 * S.nsm, 256, 0, st>>>(S.hist_old, S.hist_new, S.ctl, S.status);
  else k_hist_carry<float><<<4 * S.nsm, 256, 0, st>>>(S.hist_old, S.hist_new, S.ctl, S.status);
}

void launch_hist_zero_cumulative(HistTable const& t, const int* ctl, int fp64, cudaStream_t st) {
  int cap = 1 << t.log2cap;
  if (fp64) k_hist_zero_cumulative<double><<<blocks(cap, 256), 256, 0, st>>>(t, ctl);
  else k_hist_zero_cumulative<float><<<blocks(cap, 256), 256, 0, st>>>(t, ctl);
}

}  // namespace gdem
