// stats_static.cu -- simulation statistics that allocate nothing.
//
// Some callers cannot allocate device memory when they need the statistics: an in-situ
// analysis hook inside a host application that owns the whole device memory budget and forbids
// allocation after start-up, or a loop that must not pay cudaMalloc's implicit device-wide
// synchronisation while other streams run.  hlbm_simulation_state_static() serves them: the
// caller passes the FP64 populations, the flag bytes and a 3-double output, all already in
// device memory, and the per-block partial sums live in the fixed array below instead of in
// allocated scratch.
//
// The array is a file-scope __device__ object, so every GPU that loads this library holds it
// (HLBM_STATIC_PARTIALS slots of 3 doubles, 384 KiB) until the process exits.  Host code
// cannot use its name as a device address: the first call on each device, with that device
// current, looks the address up with cudaGetSymbolAddress and caches it.  The address belongs
// to the device's current CUDA context, so the cache also records that context's unique id and
// looks the address up again when a call finds another context current (after a
// cudaDeviceReset, or when a driver-API caller made its own context current).  Make the first
// call on a device, and the first call after such a change, before any stream capture.  Each
// block writes its own slot before the second pass reads it, so nothing needs clearing between
// calls, but every call shares the one array: calls that overlap on the GPU (on different
// streams, say) race on it.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "hippolbm.h"
#include "lbm_step.cuh"

namespace {

constexpr int kBlock = 256;
constexpr int kNodesPerThread = 64;
constexpr int64_t kNodesPerBlock = int64_t(kBlock) * kNodesPerThread;  // 16,384 nodes per partial
constexpr int kMaxPartials = HLBM_STATIC_PARTIALS;

static __device__ __align__(256) double g_stats_partials[3 * kMaxPartials];

constexpr int kMaxDevices = 64;
double* g_partials_addr[kMaxDevices] = {nullptr};
unsigned long long g_partials_ctx[kMaxDevices] = {0};  // unique id of the context the address is of
std::mutex g_setup_mutex;

// The unique id of the calling thread's current CUDA context (cuCtxGetId, reached through the
// runtime's driver entry points so that the library needs no link against the driver library);
// 0 when it cannot be read, in which case the cached address is kept.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void* a = nullptr;
    void* b = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, nullptr) == cudaSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, nullptr) == cudaSuccess) {
      get_current = reinterpret_cast<GetCurrent>(a);
      get_id = reinterpret_cast<GetId>(b);
    }
    looked_up = true;
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Per-block sum of rho and extrema of |u| over one fixed range of kNodesPerBlock nodes (the
// node ranges do not depend on the GPU, so the sum order is reproducible).  rho and u follow
// macro_variables (macro_variables.hpp:48-79); walls contribute rho = 0 and |u| = 0.
__global__ void __launch_bounds__(kBlock) k_static_partials(const double* __restrict__ f, int64_t stride,
                                                            const int8_t* __restrict__ flags, int64_t ncell,
                                                            double* __restrict__ partials) {
  double s = 0.0, vmin = 1.79769313486231570815e+308, vmax = -1.79769313486231570815e+308;
  const int64_t base = int64_t(blockIdx.x) * kNodesPerBlock;
  for (int k = 0; k < kNodesPerThread; k++) {
    const int64_t idx = base + int64_t(k) * kBlock + threadIdx.x;
    if (idx >= ncell) break;
    double rho = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
    if (flags[idx] >= hlbm::FLAG_FLUID) {
      double v[hlbm::Q];
#pragma unroll
      for (int i = 0; i < hlbm::Q; i++) v[i] = f[i * stride + idx];
      hlbm::macro<double, true>(v, rho, ux, uy, uz);
    }
    s += rho;
    const double n = sqrt(ux * ux + uy * uy + uz * uz);
    vmin = n < vmin ? n : vmin;
    vmax = n > vmax ? n : vmax;
  }
  for (int off = 16; off > 0; off >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, off);
    const double a = __shfl_down_sync(0xffffffffu, vmin, off);
    const double b = __shfl_down_sync(0xffffffffu, vmax, off);
    vmin = a < vmin ? a : vmin;
    vmax = b > vmax ? b : vmax;
  }
  __shared__ double sh[3][kBlock / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sh[0][warp] = s;
    sh[1][warp] = vmin;
    sh[2][warp] = vmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = sh[0][0], b = sh[1][0], c = sh[2][0];
    for (int w = 1; w < kBlock / 32; w++) {
      a += sh[0][w];
      b = sh[1][w] < b ? sh[1][w] : b;
      c = sh[2][w] > c ? sh[2][w] : c;
    }
    partials[3 * blockIdx.x + 0] = a;
    partials[3 * blockIdx.x + 1] = b;
    partials[3 * blockIdx.x + 2] = c;
  }
}

// One block folds the partials in a fixed order and writes {sum rho, min |u|, max |u|}.
__global__ void __launch_bounds__(kBlock) k_static_fold(const double* __restrict__ partials, int nparts,
                                                        double* __restrict__ out) {
  __shared__ double sh[3][kBlock];
  double s = 0.0, vmin = 1.79769313486231570815e+308, vmax = -1.79769313486231570815e+308;
  for (int i = threadIdx.x; i < nparts; i += kBlock) {
    s += partials[3 * i];
    vmin = partials[3 * i + 1] < vmin ? partials[3 * i + 1] : vmin;
    vmax = partials[3 * i + 2] > vmax ? partials[3 * i + 2] : vmax;
  }
  sh[0][threadIdx.x] = s;
  sh[1][threadIdx.x] = vmin;
  sh[2][threadIdx.x] = vmax;
  __syncthreads();
  for (int h = kBlock / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + h];
      sh[1][threadIdx.x] = sh[1][threadIdx.x + h] < sh[1][threadIdx.x] ? sh[1][threadIdx.x + h] : sh[1][threadIdx.x];
      sh[2][threadIdx.x] = sh[2][threadIdx.x + h] > sh[2][threadIdx.x] ? sh[2][threadIdx.x + h] : sh[2][threadIdx.x];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sh[0][0];
    out[1] = sh[1][0];
    out[2] = sh[2][0];
  }
}

}  // namespace

namespace hlbm {
int record_error(int code, const std::string& msg);  // capi.cu: feeds hlbm_last_error()
}
using hlbm::record_error;

extern "C" int hlbm_simulation_state_static(const double* f, int64_t stride, const int8_t* flags,
                                            const int32_t n[3], double* out3, void* stream) {
  if (!f || !flags || !n || !out3)
    return record_error(HLBM_EINVAL, "hlbm_simulation_state_static: NULL argument");
  if (n[0] < 1 || n[1] < 1 || n[2] < 1)
    return record_error(HLBM_EINVAL, "hlbm_simulation_state_static: node counts must be >= 1");
  const int64_t ncell = int64_t(n[0]) * n[1] * n[2];
  if (stride < ncell) return record_error(HLBM_EINVAL, "hlbm_simulation_state_static: stride < node count");
  if (ncell > HLBM_STATIC_MAX_NODES)
    return record_error(HLBM_EINVAL, "hlbm_simulation_state_static: " + std::to_string(ncell) +
                                        " nodes exceed the static scratch limit of " +
                                        std::to_string((long long)HLBM_STATIC_MAX_NODES) + " nodes");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return record_error(HLBM_ECUDA, "hlbm_simulation_state_static: no current CUDA device");
  double* partials = nullptr;
  {
    // set-up, once per device (and again when another context is current on it), with that
    // device current: the host-side name of the array is not a device address, so fetch the
    // real one
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long ctx = current_context_id();
    if (!g_partials_addr[dev] || (ctx != 0 && ctx != g_partials_ctx[dev])) {
      void* addr = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&addr, g_stats_partials);
      if (e != cudaSuccess)
        return record_error(HLBM_ECUDA, std::string("hlbm_simulation_state_static: cudaGetSymbolAddress: ") +
                                           cudaGetErrorString(e));
      g_partials_addr[dev] = static_cast<double*>(addr);
      g_partials_ctx[dev] = current_context_id();  // the lookup makes the primary context current
    }
    partials = g_partials_addr[dev];
  }
  const int nparts = int((ncell + kNodesPerBlock - 1) / kNodesPerBlock);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_static_partials<<<nparts, kBlock, 0, s>>>(f, stride, flags, ncell, partials);
  k_static_fold<<<1, kBlock, 0, s>>>(partials, nparts, out3);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return record_error(HLBM_ECUDA, std::string("hlbm_simulation_state_static: ") + cudaGetErrorString(e));
  return HLBM_OK;
}
