// noalloc.cu - COMPRESS_16 snapshot encoding for callers that cannot allocate
// GPU memory.
//
// Some callers of this library cannot call cudaMalloc: a host program that
// runs the propagation inside its own fixed GPU memory budget (the whole HBM
// carved up up-front by its pool allocator), or a service thread that must
// not block on the allocator.  rtm_c16_compress() stages its buffers with
// cudaMalloc; the entry point below takes device buffers from the caller and
// keeps its only scratch (one float per y slab: the slab's max |w|) in a fixed
// array of this file.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/rtm_b200.h"
#include "kernel_api.h"

namespace {

// Per-slab max |w| of the last call.  Lives in every GPU that loads this
// library until the process exits; shared by all calls on that GPU.
constexpr int kMaxSlabs = RTM_NOALLOC_MAX_SLABS;
static __device__ __align__(256) float g_slab_scratch[kMaxSlabs];

// A module's __device__ arrays belong to a CUDA context, not to a device: a
// caller may run under a context of its own (cuCtxCreate) or after
// cudaDeviceReset made a new primary context.  So the device address of
// g_slab_scratch is cached per context, keyed by the context's process-unique
// id (cuCtxGetId; a context handle value can be reused after a destroy).  The
// driver calls come through cudaGetDriverEntryPoint, so the library does not
// link libcuda.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

struct DriverFns {
  CtxGetCurrentFn get_current = nullptr;
  CtxGetIdFn get_id = nullptr;
};

const DriverFns &driver_fns() {
  static const DriverFns fns = [] {
    DriverFns f;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      f.get_current = (CtxGetCurrentFn)p;
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      f.get_id = (CtxGetIdFn)p;
    cudaGetLastError();
    return f;
  }();
  return fns;
}

struct ScratchEntry {
  unsigned long long ctx_id;
  float *ptr;
};
constexpr int kMaxContexts = 64;
std::mutex g_cache_mu;
ScratchEntry g_cache[kMaxContexts] = {};
int g_cache_used = 0, g_cache_next = 0;

// Id of the context current on this thread, or 0 when none is current yet.
int current_context_id(unsigned long long *id) {
  const DriverFns &f = driver_fns();
  if (!f.get_current || !f.get_id) return RTM_ERR_CUDA;
  CUcontext ctx = nullptr;
  if (f.get_current(&ctx) != CUDA_SUCCESS) return RTM_ERR_CUDA;
  *id = 0;
  if (ctx && f.get_id(ctx, id) != CUDA_SUCCESS) return RTM_ERR_CUDA;
  return RTM_OK;
}

// Device address of g_slab_scratch in the current context.  The first call in
// a context looks it up with cudaGetSymbolAddress (which also makes the
// runtime's primary context current when no context is).
int scratch_address(float **out) {
  unsigned long long id = 0;
  if (current_context_id(&id) != RTM_OK) return RTM_ERR_CUDA;
  if (id != 0) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (int i = 0; i < g_cache_used; ++i)
      if (g_cache[i].ctx_id == id) {
        *out = g_cache[i].ptr;
        return RTM_OK;
      }
  }
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_slab_scratch) != cudaSuccess || !p) {
    cudaGetLastError();
    return RTM_ERR_CUDA;
  }
  if (current_context_id(&id) != RTM_OK || id == 0) return RTM_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_cache_mu);
  int slot = g_cache_used < kMaxContexts ? g_cache_used++ : (g_cache_next++ % kMaxContexts);
  g_cache[slot] = ScratchEntry{id, (float *)p};
  *out = (float *)p;
  return RTM_OK;
}

}  // namespace

extern "C" int rtm_c16_compress_noalloc(const float *d_in, unsigned short *d_out, int nx, int ny, int nz,
                                        void *stream) {
  if (!d_in || !d_out || nx < 1 || ny < 1 || nz < 1) return RTM_ERR_ARG;
  if (ny > kMaxSlabs) return RTM_ERR_ARG;  // more y slabs than the fixed scratch (and a grid's y extent) holds
  float *scratch = nullptr;
  if (scratch_address(&scratch) != RTM_OK) return RTM_ERR_CUDA;
  // the per-slab maxima are written (not accumulated) by the first kernel, so
  // the scratch needs no clearing between calls
  rtm::launch_c16_compress(d_in, (uint16_t *)d_out, scratch, nx, ny, nz, (cudaStream_t)stream);
  if (cudaGetLastError() != cudaSuccess) return RTM_ERR_CUDA;
  return RTM_OK;
}
