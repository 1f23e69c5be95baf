// kernels_tma.cu - FD8 time-step kernels with a TMA plane pipeline (sm_100a).
//
// A CTA owns a 32 (z) x 8 (x) column tile and marches along y.  One thread is
// the producer: it issues cp.async.bulk.tensor loads of future planes into
// shared-memory rings, each plane's stage tracked by an mbarrier with its
// transaction byte count.  Ring A holds the stencil input with its 4-cell x/z
// halo (40 x 16 floats) for the whole +-4 y window plus P planes of
// prefetch; ring B holds the unhaloed per-cell inputs (w0, (v dt)^2, ...)
// P planes ahead.  Out-of-grid parts of a box are zero-filled by the TMA unit,
// which is exactly the reference's stencil truncation at the grid edge
// (bgprtm/FdEngine_fd.cpp:228-236, 266-274).  Consumers never wait on DRAM:
// every operand of a plane is in shared memory before its compute starts.
// The innermost TMA coordinate is z and always a multiple of 4 (tile origin
// 32*k - 4), so every copy starts on a 16-byte boundary; the path requires
// nz % 4 == 0 (row strides in multiples of 16 bytes).
//
//  iso_fd8_tma   KernelCPU::ISO + laplacian_irreg + pml2_bnd + update2nd,
//                with the snapshot store / imaging condition of the previous step
//                (bgprtm/KernelCPU.cpp:125-140, bgprtm/FdEngine_fd.cpp:204-325,
//                bgprtm/Propagator.cpp:1767-1818)
#include "kernel_api.h"
#include "rtm_device.cuh"
#include "tma.cuh"

namespace rtm {

namespace {

constexpr int TZ = 32, R = 4;
constexpr int HZ = TZ + 2 * R;  // haloed tile height (z)

// Shared-memory rings of one CTA: TX = tile width (x), P = prefetch depth.
template <int TX, int P>
struct __align__(128) IsoSmem {
  static constexpr int HX = TX + 2 * R;
  static constexpr int SA = 2 * R + 1 + P;  // ring A stages (the +-4 window + prefetch)
  static constexpr int SB = P + 1;          // ring B stages
  float a[SA][HX][HZ];    // w1 tiles with halo
  float w0[SB][TX][TZ];   // w0 tiles
  float vel[SB][TX][TZ];  // (v dt)^2 tiles
  uint64_t bar_a[SA];
  uint64_t bar_b[SB];
};

template <int TX, int P, int MODE, bool PML3D>
__global__ void __launch_bounds__(TZ *TX) iso_fd8_tma(IsoArgs a, const __grid_constant__ CUtensorMap map_w1,
                                                      const __grid_constant__ CUtensorMap map_w0,
                                                      const __grid_constant__ CUtensorMap map_vel, int *err) {
  using Smem = IsoSmem<TX, P>;
  constexpr int HX = Smem::HX, SA = Smem::SA, SB = Smem::SB;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem &s = *reinterpret_cast<Smem *>(smem_raw);
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  const int tz = threadIdx.x, tx = threadIdx.y;
  const int iz0 = blockIdx.x * TZ, ix0 = blockIdx.y * TX;
  const int iz = iz0 + tz, ix = ix0 + tx;
  const int y0 = blockIdx.z * a.yseg;
  const int y1 = min(a.ny, y0 + a.yseg);
  const bool act = iz < a.nz && ix < a.nx;
  const bool producer = tz == 0 && tx == 0;
  const long long col = (long long)ix * a.nz + iz;
  const bool do_y = a.ny > 2;
  constexpr uint32_t BYTES_A = HZ * HX * 4, BYTES_B = 2 * TZ * TX * 4;

  auto stage_a = [&](int p) { return (p - (y0 - R)) % SA; };
  auto par_a = [&](int p) { return (uint32_t)(((p - (y0 - R)) / SA) & 1); };
  auto stage_b = [&](int p) { return (p - y0) % SB; };
  auto par_b = [&](int p) { return (uint32_t)(((p - y0) / SB) & 1); };
  auto issue_a = [&](int p) {
    const int st = stage_a(p);
    if (p < 0 || p >= a.ny) {  // planes outside the grid: zeros written here, no copy
      float *d = &s.a[st][0][0];
      for (int k = 0; k < HX * HZ; k++) d[k] = 0.f;
      mbar_arrive(&s.bar_a[st]);
      return;
    }
    mbar_expect_tx(&s.bar_a[st], BYTES_A);
    tma_load_3d(&s.a[st][0][0], &map_w1, &s.bar_a[st], iz0 - R, ix0 - R, p);
  };
  auto issue_b = [&](int p) {
    const int st = stage_b(p);
    mbar_expect_tx(&s.bar_b[st], BYTES_B);
    tma_load_3d(&s.w0[st][0][0], &map_w0, &s.bar_b[st], iz0, ix0, p);
    tma_load_3d(&s.vel[st][0][0], &map_vel, &s.bar_b[st], iz0, ix0, p);
  };

  if (producer) {
    for (int k = 0; k < SA; k++) mbar_init(&s.bar_a[k], 1);
    for (int k = 0; k < SB; k++) mbar_init(&s.bar_b[k], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (producer) {
    for (int p = y0 - R; p < min(y0 + R + P, y1 + R); p++) issue_a(p);
    for (int p = y0; p < min(y0 + P, y1); p++) issue_b(p);
  }
  bool ok = true;
  for (int p = y0 - R; p < y0 + R && ok; p++) ok = mbar_wait(&s.bar_a[stage_a(p)], par_a(p), err);
  // ring-A stages of the y window iy-R .. iy+R, rotated once per plane
  int win[2 * R + 1];
#pragma unroll
  for (int k = 0; k <= 2 * R; k++) win[k] = stage_a(y0 - R + k);

  for (int iy = y0; iy < y1; iy++) {
    if (producer) {
      if (iy + R + P < y1 + R) issue_a(iy + R + P);
      if (iy + P < y1) issue_b(iy + P);
    }
    ok = ok && mbar_wait(&s.bar_a[stage_a(iy + R)], par_a(iy + R), err);
    ok = ok && mbar_wait(&s.bar_b[stage_b(iy)], par_b(iy), err);
    if (act && ok) {
      const float(*T)[HZ] = s.a[win[R]];
      const float u = T[tx + R][tz + R];
      float lz = a.c2z[0] * u, lx = a.c2x[0] * u, ly = 0.0f;
#pragma unroll
      for (int m = 1; m <= R; m++) {
        lz += a.c2z[m] * (T[tx + R][tz + R - m] + T[tx + R][tz + R + m]);
        lx += a.c2x[m] * (T[tx + R - m][tz + R] + T[tx + R + m][tz + R]);
      }
      if (do_y) {
        ly = a.c2y[0] * u;
#pragma unroll
        for (int m = 1; m <= R; m++) ly += a.c2y[m] * (s.a[win[R - m]][tx + R][tz + R] + s.a[win[R + m]][tx + R][tz + R]);
      }
      float v;
      const bool edge = in_pml(a.pml, g, ix, iy, iz);
      if (PML3D) {
        v = lz + lx + ly;
        if (edge) {
          pml2_dim(a.pml, g, DZ, v, ix, iy, iz);
          pml2_dim(a.pml, g, DX, v, ix, iy, iz);
          pml2_dim(a.pml, g, DY, v, ix, iy, iz);
        }
      } else {
        if (edge) {
          pml2_dim(a.pml, g, DZ, lz, ix, iy, iz);
          pml2_dim(a.pml, g, DX, lx, ix, iy, iz);
          if (do_y) pml2_dim(a.pml, g, DY, ly, ix, iy, iz);
        }
        v = lz + lx + ly;
      }
      const long long i = (long long)iy * g.nxz + col;
      if (a.io.store | a.io.ic) fused_io(a.io, g, i, ix, iy, iz, col, u);
      const int sb = stage_b(iy);
      const float t = s.w0[sb][tx][tz] - v * s.vel[sb][tx][tz];
      float out;
      if (MODE == 0) out = t;
      else if (MODE == 1) out = (u + u) - t;
      else out = q_update(a.q, i, (long long)a.ny * g.nxz, t, u);
      a.w0[i] = out;
    }
    __syncthreads();  // every thread is done with the stages the producer refills next
#pragma unroll
    for (int k = 0; k < 2 * R; k++) win[k] = win[k + 1];
    win[2 * R] = win[2 * R - 1] + 1 == SA ? 0 : win[2 * R - 1] + 1;
  }
}

}  // namespace

// ---- host side: tensor maps ----------------------------------------------------

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
    cudaGetLastError();
  }
  return fn;
}

// A wait that nothing completes: one thread initialises an mbarrier for one
// arrival that never comes and waits on it; the bounded wait gives up and
// raises *err.  Issues no copy, so returning early leaves nothing in flight.
__global__ void selftest_wait_k(int *err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) (void)mbar_wait(&bar, 0, err);
}

void launch_selftest_wait(int *err, cudaStream_t st) { selftest_wait_k<<<1, 32, 0, st>>>(err); }

bool tma_supported(int nz) { return nz % 4 == 0 && encode_fn() != nullptr; }

// fp32 volume [ny][nx][nz] with a box of (bz, bx, 1) cells
bool make_tmap(CUtensorMap *m, const void *base, int nx, int ny, int nz, int bz, int bx, int by) {
  EncodeTiledFn fn = encode_fn();
  if (!fn || nz % 4 != 0 || ((uintptr_t)base & 15)) return false;
  cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)nx, (cuuint64_t)ny};
  cuuint64_t strides[2] = {(cuuint64_t)nz * 4, (cuuint64_t)nz * nx * 4};
  cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)bx, (cuuint32_t)by};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void *>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Q memory variables [L][ny][nx][nz] (FP32 or BF16) as one 4-D tensor with a
// box of (bz, bx, 1, L): every order of a column tile in one copy.  The row,
// plane and order strides must be multiples of 16 bytes (nz % 4 == 0 for
// FP32, nz % 8 == 0 for BF16).
bool make_tmap_q(CUtensorMap *m, const void *base, int nx, int ny, int nz, int L, bool bf16, int bz, int bx) {
  EncodeTiledFn fn = encode_fn();
  const int es = bf16 ? 2 : 4;
  if (!fn || L < 1 || L > 8 || (nz * es) % 16 != 0 || ((uintptr_t)base & 15)) return false;
  cuuint64_t dims[4] = {(cuuint64_t)nz, (cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)L};
  cuuint64_t strides[3] = {(cuuint64_t)nz * es, (cuuint64_t)nz * nx * es, (cuuint64_t)nz * nx * ny * es};
  cuuint32_t box[4] = {(cuuint32_t)bz, (cuuint32_t)bx, 1, (cuuint32_t)L};
  cuuint32_t est[4] = {1, 1, 1, 1};
  CUresult r = fn(m, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                  const_cast<void *>(base), dims, strides, box, est, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int TX, int P>
static void iso_tma_shape(const IsoArgs &a, const CUtensorMap &w1, const CUtensorMap &w0, const CUtensorMap &vel,
                          int *err, int mode, int pml3d, cudaStream_t st) {
  dim3 grid((a.nz + TZ - 1) / TZ, (a.nx + TX - 1) / TX, (a.ny + a.yseg - 1) / a.yseg), block(TZ, TX);
  const size_t smem = sizeof(IsoSmem<TX, P>);
#define L_(M, P3) iso_fd8_tma<TX, P, M, P3><<<grid, block, smem, st>>>(a, w1, w0, vel, err)
  if (pml3d) {
    if (mode == 0) L_(0, true);
    else if (mode == 1) L_(1, true);
    else L_(2, true);
  } else {
    if (mode == 0) L_(0, false);
    else if (mode == 1) L_(1, false);
    else L_(2, false);
  }
#undef L_
}

template <int TX, int P>
static bool iso_tma_attr() {
  const int smem = (int)sizeof(IsoSmem<TX, P>);
  bool ok = true;
  ok &= cudaFuncSetAttribute(iso_fd8_tma<TX, P, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == 0;
  ok &= cudaFuncSetAttribute(iso_fd8_tma<TX, P, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == 0;
  ok &= cudaFuncSetAttribute(iso_fd8_tma<TX, P, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == 0;
  ok &= cudaFuncSetAttribute(iso_fd8_tma<TX, P, 0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == 0;
  ok &= cudaFuncSetAttribute(iso_fd8_tma<TX, P, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == 0;
  ok &= cudaFuncSetAttribute(iso_fd8_tma<TX, P, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == 0;
  return ok;
}

// (tile width, prefetch depth) shapes the autotuner chooses from
const TmaShape kIsoTmaShapes[] = {{8, 3}, {8, 6}, {8, 10}, {16, 4}, {16, 8}};
const int kIsoTmaNShapes = sizeof(kIsoTmaShapes) / sizeof(kIsoTmaShapes[0]);

bool iso_tma_init() {
  return iso_tma_attr<8, 3>() && iso_tma_attr<8, 6>() && iso_tma_attr<8, 10>() && iso_tma_attr<16, 4>() &&
         iso_tma_attr<16, 8>();
}

void launch_iso_fd8_tma(const IsoArgs &a, const CUtensorMap &w1, const CUtensorMap &w0, const CUtensorMap &vel,
                        int *err, int mode, int pml3d, int shape, cudaStream_t st) {
  switch (shape) {
    case 0: iso_tma_shape<8, 3>(a, w1, w0, vel, err, mode, pml3d, st); break;
    case 1: iso_tma_shape<8, 6>(a, w1, w0, vel, err, mode, pml3d, st); break;
    case 2: iso_tma_shape<8, 10>(a, w1, w0, vel, err, mode, pml3d, st); break;
    case 3: iso_tma_shape<16, 4>(a, w1, w0, vel, err, mode, pml3d, st); break;
    default: iso_tma_shape<16, 8>(a, w1, w0, vel, err, mode, pml3d, st); break;
  }
}

}  // namespace rtm
