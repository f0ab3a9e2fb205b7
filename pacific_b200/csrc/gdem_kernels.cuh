// gdem_kernels.cuh -- launcher declarations of the DEM step kernels.
#pragma once
#include "gdem_device.cuh"

namespace gdem {

// Launches kernel k so that it may start while the previous kernel of the
// stream still runs (programmatic stream serialization; k calls pdlWait()
// before it touches that kernel's results).
template <typename... KArgs, typename... Args>
inline void launchAfterPrevious(void (*k)(KArgs...), unsigned grid, unsigned block,
                                cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  (void)cudaLaunchKernelEx(&cfg, k, args...);   // a failure shows in cudaGetLastError
}

// Parts of the leapfrog applied by k_move.
enum StepFlags : int {
  kStepClose = 2,     // closing kick of the step that ends here (dt / 2)
  kStepMove = 4,      // opening kick (dt / 2) and drift (dt) of the next step
  kStepStoreFT = 8,   // write F, T back (last evaluation of a call, leapfrog start)
  kStepSum = 16,      // F, T of this evaluation from the pair kernel's shares
};
// nact[t], the particle's flag word for this evaluation, cleared by k_move:
// kCandidate, set by the contact filter, when the particle is a partner of a
// pair the filter kept or near a wall (only then can it receive a share);
// then, set by the pair kernel (atomically: both partners of a pair in
// contact set theirs), bit e (e < kMaskEntries) when entry e of its row holds
// a share of this evaluation, kFarEntry when an entry at or beyond
// kMaskEntries does (those are found by their tags), kNearWall when its wall
// share is set.  A particle without kCandidate carries its weight only.
constexpr int kMaskEntries = 29;
constexpr unsigned kEntryBits = (1u << kMaskEntries) - 1u;
constexpr unsigned kCandidate = 1u << 29;
constexpr unsigned kFarEntry = 1u << 30;
constexpr unsigned kNearWall = 1u << 31;
__device__ __forceinline__ unsigned entryBit(int e) {
  return e < kMaskEntries ? (1u << e) : kFarEntry;
}

// gdem_integrate.cu
void launch_decide(DevState const& S, cudaGraphConditionalHandle h, int use_handle,
                   cudaStream_t st);
void launch_bin(DevState const& S, const int* gate, cudaStream_t st);
void launch_scan(DevState const& S, const int* gate, cudaStream_t st);
// exclusive scan of the row lengths into pair_off (total into kCtlEntries)
void launch_row_scan(DevState const& S, const int* gate, cudaStream_t st);
void launch_filter(DevState const& S, cudaStream_t st);
void launch_link(DevState const& S, const int* gate, cudaStream_t st);
void launch_diag_prefill(DevState const& S, cudaStream_t st);
void launch_place(DevState const& S, const int* gate, cudaStream_t st);
void launch_cellsort(DevState const& S, const int* gate, cudaStream_t st);
void launch_permute(DevState const& S, const int* gate, cudaStream_t st);
void launch_copyback(DevState const& S, const int* gate, cudaStream_t st);
// fast: the FP32-split leapfrog (reciprocals, series; not the reference's
// operation order)
void launch_move(DevState const& S, int flags, int fast, cudaStream_t st);
void launch_fill64(unsigned long long* p, size_t n, unsigned long long value, cudaStream_t st);
void launch_scatter_by_id(DevState const& S, double* x, double* v, double* w, double* wbf,
                          double* q, double* F, double* T, int id_base, cudaStream_t st);
void launch_basis_by_id(DevState const& S, double* out, int id_base, cudaStream_t st);
void launch_cells_by_id(DevState const& S, int* ijk, int id_base, cudaStream_t st);
// needs the diagnostics records (pair_delta, wall_delta) of the last evaluation
void launch_coordination_by_id(DevState const& S, int* out, int id_base, cudaStream_t st);
void launch_hist_zero_cumulative(HistTable const& t, const int* ctl, int fp64, cudaStream_t st);
void launch_hist_carry(DevState const& S, int fp64, cudaStream_t st);
void launch_load_state(DevState const& S, const double* x, const double* v, const double* w,
                       const double* wbf, const double* q, const double* F, const double* T,
                       const int* type_by_id, const int* inst_by_id, cudaStream_t st);
void launch_vstats(DevState const& S, double* part, double* out, cudaStream_t st);
void launch_set_velocities(DevState const& S, const double* v, const double* w, cudaStream_t st);
void launch_pair_counts(DevState const& S, unsigned long long* out, cudaStream_t st);

// gdem_contact64.cu (FP64 mode); fill = 0 counts the rows, 1 writes them
void launch_pairs64(DevState const& S, const int* gate, int fill, cudaStream_t st);
void launch_pairlaw64(DevState const& S, cudaStream_t st);

// A particle inserted during the run (gdem_insert_particle): its class
// (global index), device ID and slot, position, velocity, space-frame
// angular velocity, quaternion (x, y, z, w) and, when has_basis, its
// orientation matrix (row-major; otherwise the matrix of q).
struct NewParticle {
  int type, id, slot, has_basis;
  double x[3], v[3], w[3], q[4], basis[9];
};
// Sets *hit when the particle p would touch a particle or a wall
// (LinkedCell::insertParticleSerial's test); FP64.
void launch_insert_test(DevState const& S, NewParticle const& p, int bv_only, int* hit,
                        cudaStream_t st);
// Writes p into slot p.slot with its weight as force (Particle::InitializeForce).
void launch_append_particle(DevState const& S, NewParticle const& p, cudaStream_t st);

// gdem_contact32.cu (FP32-split mode)
void launch_pairs32(DevState const& S, const int* gate, int fill, cudaStream_t st);
void launch_pairlaw32(DevState const& S, cudaStream_t st);
// First pass over the cold kept pairs (FP32-split, non-spherical classes).
void launch_pairsep32(DevState const& S, cudaStream_t st);

}  // namespace gdem
