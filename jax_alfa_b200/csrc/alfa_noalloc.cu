// alfa_PlanarMean_noalloc: the plane mean of alfa_PlanarMean for callers
// that may not allocate device memory.
//
// Who needs it: code that runs inside another runtime's memory management.
// A JAX/XLA custom call is the case closest to this project: XLA reserves
// most of the GPU's memory for its own allocator when it starts and hands a
// custom call only the buffers it owns, so a cudaMalloc inside the call can
// fail, or take memory XLA has already promised to other buffers.  The same
// holds for applications that fix their device-memory budget at start-up.
// Such callers cannot create an alfa_ctx (its set-up allocates the
// workspace), so this entry point needs no context.
//
// The two-level reduction keeps one partial sum per (block, level); here
// those partials live in a fixed array in the library's device image, so
// nothing is allocated at call time.  Every device that loads the library
// holds its own copy of the array until the process exits.
#include <cuda.h>

#include <mutex>

#include "alfa.h"
#include "alfa_internal.cuh"

#include "alfa_physics.cuh"

namespace {

constexpr int kBlocks = alfa::NOALLOC_RED_BLOCKS;  // partial sums per level (the launch's blocks)
constexpr int kMaxLevels = 2048;                   // largest nz accepted
// 256 x 2048 doubles = 4 MiB per device
static __device__ __align__(256) double g_partials[kBlocks * kMaxLevels];

// Driver entry points that identify the current context, fetched through the
// runtime (no link against the driver library).  Either may stay null on a
// driver without it; the cache below is then bypassed.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
std::once_flag g_entry_once;

// Id of the context current on this thread, 0 when none is current or the
// id cannot be read.  Ids are unique within the process, so a device whose
// primary context was destroyed (cudaDeviceReset) and re-created reports a
// new one.
unsigned long long current_context_id() {
  std::call_once(g_entry_once, [] {
    cudaDriverEntryPointQueryResult q;
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  });
  if (!g_ctx_current || !g_ctx_id) return 0;
  CUcontext c = nullptr;
  if (g_ctx_current(&c) != CUDA_SUCCESS || c == nullptr) return 0;
  unsigned long long id = 0;
  if (g_ctx_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

std::mutex g_mu;
constexpr int kMaxDevices = 256;
struct Cached {
  unsigned long long ctx = 0;  // context the address belongs to
  double* addr = nullptr;
};
Cached g_addr[kMaxDevices];

// Device address of g_partials on the current device, looked up with that
// device current the first time and again whenever the device's context has
// changed since (the old address died with the old context).  In host code
// the name g_partials is a host-side stand-in, not a device address, so it is
// never passed as is.
int partials_on_current_device(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return ALFA_E_CUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  Cached& slot = g_addr[dev];
  const unsigned long long ctx = current_context_id();
  if (slot.addr == nullptr || ctx == 0 || slot.ctx != ctx) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_partials) != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return ALFA_E_CUDA;
    }
    slot.addr = static_cast<double*>(p);
    slot.ctx = current_context_id();  // the lookup made the device's context current
  }
  *out = slot.addr;
  return ALFA_OK;
}

}  // namespace

extern "C" int alfa_PlanarMean_noalloc(const double* F, int nx, int ny, int nz, double* mean_nz,
                                       void* cuda_stream) {
  if (!F || !mean_nz || nx < 1 || ny < 1 || nz < 1) return ALFA_E_SHAPE;
  if (nz > kMaxLevels) return ALFA_E_NOALLOC_LIMIT;
  double* partials = nullptr;
  const int st = partials_on_current_device(&partials);
  if (st != ALFA_OK) return st;
  // Every partial read by the final sum is written by this call's first
  // kernel, so the array needs no clearing; it keeps the last call's values.
  alfa::f64::plane_mean_with_scratch(F, (size_t)nx * (size_t)ny, nz, partials, mean_nz,
                                static_cast<cudaStream_t>(cuda_stream));
  return cudaGetLastError() == cudaSuccess ? ALFA_OK : ALFA_E_CUDA;
}
