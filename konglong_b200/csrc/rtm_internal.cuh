// rtm_internal.cuh - device-side data structures shared by the kernels of the
// B200 RTM engine.  Volumes are z-fastest FP32, element (ix,iy,iz) at
// ((iy*nx + ix)*nz + iz), exactly the reference's layout, so host buffers map
// onto device buffers with one copy.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace rtm {

enum { DX = 0, DY = 1, DZ = 2 };
enum { SIDE_LO = 0, SIDE_HI = 1 };

// One PML layer stack (one face of the grid).  Memory per round r and
// component c is [plane][w] (z faces) or [plane][nz] (x / y faces) with the
// reference's indexing (bgprtm/FdEngine.cpp:324-389).  co[L*6 + k] holds, per
// layer L counted from the outer edge, the recursion constants of
// bgprtm/PML.cpp:126-134 for damping g (k = 0..2: (1-g)/(1+g), 2g/(1-g^2),
// 1/(1-g)) and for g * pml3d_scaler (k = 3..5), built in FP64.
struct PmlFace {
  int w;            // layer count, 0 = no PML on this face
  const float *co;  // [w][6]
  float *q[2][3];   // [round][component]
};

struct PmlDev {
  PmlFace f[3][2];  // [dim][side]
};

// Separable spread kernels of traces whose z kernels are identical (one
// group), or the trace list of an ungrouped set.
struct TraceDev {
  int ntr, lx, ly, lz, nt;
  const int *ids;     // optional subset of trace ids handled by a launch
  int nids;
  const int *off;     // [ntr][3]
  const int *len;     // [ntr][3]
  const float *kx, *ky, *kz;  // [ntr][lx], [ntr][ly], [ntr][lz]
  const float *traces;        // [ntr][nt] (injection only)
  float scaler;
};

// Receiver / source groups sharing one z kernel (same first index, length
// and coefficients): the xy part is gathered per cell of an xy tile.
struct GroupDev {
  int ntr;               // members
  const int *members;    // trace ids
  int offz, lz;
  const float *kz;       // [lz]
  // xy tiles covered by the group and, per tile, the member list (CSR)
  int ntiles, tile;      // tile edge (cells)
  const int *tile_xy;    // [ntiles][2] tile origin (ix0, iy0)
  const int *tile_ptr;   // [ntiles+1]
  const int *tile_list;  // member trace ids
};

// Snapshot / imaging-condition access fused into the stencil kernels.
struct SnapDev {
  int fmt;              // 0 fp32, 1 c16 (reference COMPRESS_16), 2 fp16 with slab scale
  void *base;           // slot storage
  const float *slab;    // per-y-slab vmax (c16) / scale (fp16s), [ny]
};

struct FusedIo {
  // store the centre value (the previous step's final wavefield) into a snapshot slot
  int store;
  SnapDev st;
  // image += T(src slot) * T(centre)
  int ic;
  SnapDev src;
  float *image, *comp;
  int use_t;                // 1: time taper tscale (slot < ntaper_t), 0: depth taper
  float tscale;
  const float *taper_z;     // [nz] depth taper (1 below), used when tscale == 0
  const float *ex, *ey, *ez;  // decode edge tapers per axis (1 inside)
  float *illum;               // source illumination sum of s^2 (calIllum), null when off
};

struct QDev {
  int order;
  float cqsum;
  float cq[8], wq[8];
  const float *invq;
  float *d0, *d1;  // [order][n] halves selected by iq0/iq1 (FP32, or BF16 when bf16)
  int bf16;        // memory variables stored as bfloat16 (the update arithmetic stays FP32)
};

}  // namespace rtm

#define RTM_CUDA_OK(call)                                          \
  do {                                                             \
    cudaError_t e__ = (call);                                      \
    if (e__ != cudaSuccess) return rtm::cuda_fail(e__, #call, h);  \
  } while (0)

namespace rtm {
struct Engine;
int cuda_fail(cudaError_t e, const char *what, Engine *h);
}
