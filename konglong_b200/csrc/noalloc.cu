// noalloc.cu - COMPRESS_16 snapshot encoding for callers that cannot allocate
// GPU memory.
//
// Some callers of this library cannot call cudaMalloc: a host program that
// runs the propagation inside its own fixed GPU memory budget (the whole HBM
// carved up up-front by its pool allocator), code that records work into a
// CUDA graph it builds itself, or a service thread that must not block on the
// allocator.  rtm_c16_compress() stages its buffers with cudaMalloc; the entry
// point below takes device buffers from the caller and keeps its only scratch
// (one float per y slab: the slab's max |w|) in a fixed array of this file.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/rtm_b200.h"
#include "kernel_api.h"

namespace {

// Per-slab max |w| of the last call.  Lives in every GPU that loads this
// library until the process exits; shared by all calls on that GPU.
constexpr int kMaxSlabs = RTM_NOALLOC_MAX_SLABS;
static __device__ __align__(256) float g_slab_scratch[kMaxSlabs];

// Device address of g_slab_scratch per device, looked up once (with that
// device current) the first time the entry point runs on it.
constexpr int kMaxDevices = 64;
static float *g_scratch_ptr[kMaxDevices] = {};

}  // namespace

extern "C" int rtm_c16_compress_noalloc(const float *d_in, unsigned short *d_out, int nx, int ny, int nz,
                                        void *stream) {
  if (!d_in || !d_out || nx < 1 || ny < 1 || nz < 1) return RTM_ERR_ARG;
  if (ny > kMaxSlabs) return RTM_ERR_ARG;  // more y slabs than the fixed scratch holds
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return RTM_ERR_CUDA;
  }
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_slab_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return RTM_ERR_CUDA;
    }
    g_scratch_ptr[dev] = (float *)p;
  }
  // the per-slab maxima are written (not accumulated) by the first kernel, so
  // the scratch needs no clearing between calls
  rtm::launch_c16_compress(d_in, (uint16_t *)d_out, g_scratch_ptr[dev], nx, ny, nz, (cudaStream_t)stream);
  if (cudaGetLastError() != cudaSuccess) return RTM_ERR_CUDA;
  return RTM_OK;
}
