// raycastFirst for callers that cannot allocate device memory.
//
// Who needs this: code that runs under a fixed device-memory budget owned by someone else (a
// renderer or simulation whose allocator must not be bypassed), code on a latency-critical thread
// where a cudaMalloc could block for milliseconds or fail under memory pressure, and hosts that
// pre-allocate everything at start-up and forbid allocation afterwards.  The other query entry
// points may grow staging buffers with cudaMalloc on the first large host-memory call; this one
// never allocates.  Its scratch -- the persistent kernel's work counter and, for host-memory
// buffers, the device staging of rays and hits -- is the file-scope array below, which every GPU
// that loads the library holds (3.6 MB) until the process exits.
//
// Limits and sharing:
//   * host-memory calls take at most kStaticMaxRays (65,536) rays; larger requests are rejected
//     with BVHC_ERR_SCRATCH_LIMIT before any work is enqueued (device-memory calls stage nothing
//     and are not limited);
//   * every call on a device shares the one array, which keeps the previous call's contents; the
//     work counter is reset at the start of each call and the staging areas are fully overwritten,
//     so no stale value is read -- but two calls that overlap on the GPU (different streams, or
//     different host threads) race on the array and must not be issued;
//   * the first call on each device looks up the array's device address (cudaGetSymbolAddress) with
//     that device current; make that first call before any stream capture.  The address belongs to
//     the device's context: a cudaDeviceReset ends it (and every mesh made on that device before),
//     so each call compares the current context's id with the one the address was looked up in and
//     looks it up again in a new context.  The first call after a reset is then a set-up call too.
#include <cuda.h>  // driver types only: the two context queries are fetched at run time
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "bvhcuda.h"
#include "kernels.cuh"

namespace {

constexpr uint64_t kStaticMaxRays = 65536;
constexpr size_t kCounterBytes = 256;  // work counter, padded to keep the staging areas aligned
constexpr size_t kRaysBytes = kStaticMaxRays * 24;
constexpr size_t kHitsBytes = kStaticMaxRays * sizeof(bvhc_hit);
constexpr size_t kScratchBytes = kCounterBytes + kRaysBytes + kHitsBytes;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // id of the context the address belongs to

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Id of the current context (unique within the process; a device reset makes a new context and
// so a new id); 0 when there is no current context yet or the driver cannot tell.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

// Device address of g_noalloc_scratch on `device` (which must be current).  In host code the
// array's name is only a stand-in for the symbol, so the address is looked up once per device and
// context, and again after the device's context was replaced (cudaDeviceReset).
cudaError_t scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  unsigned long long ctx = current_context_id();
  if (!g_scratch_addr[device] || (ctx != 0 && ctx != g_scratch_ctx[device])) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = static_cast<unsigned char*>(p);
    g_scratch_ctx[device] = current_context_id();   // the look-up made the context current if it was not
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

bvhc_status status_of(cudaError_t e) {
  if (e == cudaSuccess) return BVHC_OK;
  if (e == cudaErrorMemoryAllocation) return BVHC_ERR_OUT_OF_MEMORY;
  return BVHC_ERR_CUDA;
}

}  // namespace

extern "C" bvhc_status bvhc_raycast_first_noalloc(bvhc_mesh* mesh, const float* rays, uint64_t n, int side,
                                                  float near_dist, float far_dist, bvhc_hit* out, int mem,
                                                  void* stream) {
  using namespace bvhc;
  MeshDev view;
  TraversalConfig cfg;
  int device = 0;
  if (!mesh_launch_info(mesh, &view, &cfg, &device) || side < BVHC_FRONT_SIDE || side > BVHC_DOUBLE_SIDE ||
      (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE))
    return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!rays || !out) return BVHC_ERR_INVALID_ARGUMENT;
  if (mem == BVHC_MEM_HOST && n > kStaticMaxRays) return BVHC_ERR_SCRATCH_LIMIT;
  if (mem == BVHC_MEM_DEVICE &&
      (reinterpret_cast<uintptr_t>(rays) % 8 != 0 || reinterpret_cast<uintptr_t>(out) % 16 != 0))
    return BVHC_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return status_of(e);
  unsigned char* scratch = nullptr;
  e = scratch_address(device, &scratch);
  if (e != cudaSuccess) return status_of(e);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto* work = reinterpret_cast<unsigned long long*>(scratch);
  SideTable one_side{};
  TraversalConfig persistent = cfg;
  persistent.persistent = 1;
  if (mem == BVHC_MEM_DEVICE)
    return status_of(launch_raycast_first_persistent(view, nullptr, rays, n, side, one_side, near_dist, far_dist, out,
                                                     work, persistent, s));
  auto* d_rays = reinterpret_cast<float*>(scratch + kCounterBytes);
  auto* d_hits = reinterpret_cast<bvhc_hit*>(scratch + kCounterBytes + kRaysBytes);
  e = cudaMemcpyAsync(d_rays, rays, n * 24, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = launch_raycast_first_persistent(view, nullptr, d_rays, n, side, one_side, near_dist, far_dist, d_hits, work,
                                        persistent, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_hits, n * sizeof(bvhc_hit), cudaMemcpyDeviceToHost, s);
  unsigned int err_word = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&err_word, view.err, sizeof err_word, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return status_of(e);
  if (err_word == 0) return BVHC_OK;
  e = cudaMemsetAsync(view.err, 0, sizeof err_word, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? BVHC_ERR_DEVICE : status_of(e);
}
