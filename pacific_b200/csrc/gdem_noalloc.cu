// gdem_noalloc.cu -- speed statistics over caller-owned device velocities,
// with the reduction's scratch in a fixed device array of this library.
//
// gdem_speed_stats_static computes what gdem_velocity_stats computes (the
// maximum and the mean of |v| over the particles, AllComponents::
// ComputeMaxMeanVelocity, Component/src/AllComponents.cpp:1781-1811) for a
// velocity array that the caller holds in device memory, without a handle
// and without allocating: the block partials of the two-pass reduction live
// in g_speed_scratch below.
//
//   * Capacity: at most kSpeedMaxBlocks blocks of 256 particles, i.e.
//     n <= 1,048,576 particles; larger n is rejected with GDEM_ERR_INVALID.
//   * Nothing in the scratch has to start at zero: every call writes each
//     partial it later reads.
//   * The scratch is shared by every call in the process on a given device:
//     two calls that overlap in time (other host threads, or other streams
//     whose work is not ordered with this one) race on it.  Callers order
//     them, e.g. by issuing them on one stream from one thread.
//   * The first call on a device looks up the scratch address with
//     cudaGetSymbolAddress while that device is current; it should come
//     before any stream capture.  Later calls only launch two kernels.
//   * The address belongs to the device's context.  Each call compares the
//     current context's ID (cuCtxGetId, reached through the runtime's driver
//     entry point, so this library needs no link to libcuda) with the one the
//     address was looked up in, and looks it up again after a change, e.g.
//     after cudaDeviceReset ended the previous context.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/grains_b200.h"

namespace gdem {
namespace {

constexpr int kSpeedThreads = 256;
constexpr int kSpeedMaxBlocks = 4096;
constexpr int64_t kSpeedMaxN = (int64_t)kSpeedMaxBlocks * kSpeedThreads;
constexpr int kMaxDevices = 64;

// block partials: (max |v|, sum |v|) per block
static __device__ __align__(256) double g_speed_scratch[2 * kSpeedMaxBlocks];

std::mutex g_addr_mutex;
double* g_addr[kMaxDevices] = {nullptr};
// ID of the context each cached address was looked up in (0: none)
unsigned long long g_ctx_id[kMaxDevices] = {0};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// ID of the calling thread's current context, 0 when there is none (or the
// driver cannot tell).  Caller holds g_addr_mutex.
unsigned long long currentContextId() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    looked_up = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  unsigned long long id = 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// |v| of particle i from AoS velocities (3 per particle)
__device__ __forceinline__ double speed(const double* v, int i) {
  const double x = v[3 * (size_t)i], y = v[3 * (size_t)i + 1], z = v[3 * (size_t)i + 2];
  return sqrt(x * x + y * y + z * z);
}

__global__ void __launch_bounds__(kSpeedThreads) k_speed_partial(const double* v, int n,
                                                                 double* part) {
  __shared__ double smax[kSpeedThreads], ssum[kSpeedThreads];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double s = i < n ? speed(v, i) : 0.;
  smax[threadIdx.x] = s;
  ssum[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + o]);
      ssum[threadIdx.x] += ssum[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = smax[0];
    part[2 * blockIdx.x + 1] = ssum[0];
  }
}

__global__ void __launch_bounds__(kSpeedThreads) k_speed_final(const double* part, int nparts,
                                                               int n, double* out) {
  __shared__ double smax[kSpeedThreads], ssum[kSpeedThreads];
  double m = 0., s = 0.;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) {
    m = fmax(m, part[2 * k]);
    s += part[2 * k + 1];
  }
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
  if (threadIdx.x == 0) {
    out[0] = smax[0];
    out[1] = n > 0 ? ssum[0] / n : 0.;
  }
}

}  // namespace

// gdem_host.cu: the message gdem_last_error() returns
void setLastError(std::string const& msg);

namespace {
int fail(int code, std::string const& msg) {
  setLastError(msg);
  return code;
}
}  // namespace
}  // namespace gdem

using namespace gdem;

extern "C" {

int gdem_speed_stats_static(const double* v, int64_t n, double* out, void* stream) {
  if (!v || !out || n < 0)
    return fail(GDEM_ERR_INVALID, "gdem_speed_stats_static: null pointer or negative n");
  if (n > kSpeedMaxN)
    return fail(GDEM_ERR_INVALID,
                "gdem_speed_stats_static: n = " + std::to_string(n) +
                    " exceeds the fixed scratch capacity of " + std::to_string(kSpeedMaxN) +
                    " particles; use gdem_velocity_stats on a handle instead");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(GDEM_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return fail(GDEM_ERR_INVALID, "gdem_speed_stats_static: device index out of range");
  double* part;
  {
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    // the cached address is valid while the context it was looked up in is
    // still the current one (a context ID is never reused)
    const unsigned long long ctx = currentContextId();
    if (!g_addr[dev] || ctx == 0 || ctx != g_ctx_id[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_speed_scratch);
      if (e != cudaSuccess) return fail(GDEM_ERR_CUDA, cudaGetErrorString(e));
      g_addr[dev] = static_cast<double*>(p);
      // the lookup has made the device's context current on this thread
      g_ctx_id[dev] = currentContextId();
    }
    part = g_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nn = (int)n;
  const int nb = nn > 0 ? (nn + kSpeedThreads - 1) / kSpeedThreads : 0;
  if (nb > 0) k_speed_partial<<<nb, kSpeedThreads, 0, st>>>(v, nn, part);
  k_speed_final<<<1, kSpeedThreads, 0, st>>>(part, nb, nn, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(GDEM_ERR_CUDA, cudaGetErrorString(e));
  return GDEM_OK;
}

}  // extern "C"
