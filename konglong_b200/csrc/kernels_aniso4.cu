// kernels_aniso4.cu - FD8 VTI / TTI two-pass step with 4 z cells per thread and TMA rings.
//
// KernelCPU::TTI (bgprtm/KernelCPU.cpp:93-119): pass 1 takes the first derivatives of w1 with
// PML round 1 and the ScalarVTI / ScalarTTI scaling (bgprtm/KernelCPU.cpp:176-297), pass 2 the
// divergence with PML round 2, the accumulation into w0 and update2nd (+Q,
// bgprtm/Propagator.cpp:1767-1818).  Same arithmetic in the same order as grad_fd8 / div_fd8
// (bitwise-equal results), in the structure of iso_fd8_tma4: a thread owns 4 consecutive z
// cells (128-bit accesses), a CTA of 8 x TX threads marches a 32 (z) x TX (x) column tile along
// y, one producer thread fills shared-memory rings with cp.async.bulk.tensor on mbarriers
// (every wait bounded), the +-4 y neighbours come from a register queue fed from a ring, and
// PML-free interior tiles and PML tiles are separate launches over the tile table.  PML tiles
// keep the x / z face memory of their 4 cells (pointers advancing by a constant stride per
// plane) and load every memory value of a plane before its recursion.
// Requires nz % 4 == 0.
#include <type_traits>

#include "kernel_api.h"
#include "rtm_device.cuh"
#include "tma.cuh"

namespace rtm {
namespace {

constexpr int R4 = 4;  // stencil radius

__device__ __forceinline__ float cmp4(const float4 &v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ void set4(float4 &v, int c, float x) {
  if (c == 0) v.x = x;
  else if (c == 1) v.y = x;
  else if (c == 2) v.z = x;
  else v.w = x;
}
__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }

// Round-R memory of one PML face for the thread's 4 cells: the arrays of the z, x
// and y derivative components (pml1's component index per face dimension) at the
// current plane, the per-plane stride, and the face's recursion constants with the
// layer of the first cell and its step along z (z faces: one layer per cell).
struct Face1 {
  float *zc, *xc, *yc;
  long long stride;
  const float *co;
  int L, dl;
};

template <int R>
__device__ __forceinline__ Face1 face1(const PmlFace &F, int d, long long idx, long long stride, int L, int dl) {
  const int cz = d == DZ ? 0 : 1, cx = d == DX ? 0 : d == DZ ? 1 : 2, cy = d == DY ? 0 : 2;
  return Face1{F.q[R][cz] + idx, F.q[R][cx] + idx, F.q[R][cy] + idx, stride, F.co, L, dl};
}

// PML round R (pml1 for the z, x, y components in turn: own dimension unscaled, then
// the cross dimensions scaled; pml1_all's order) of the thread's 4 cells; hz / hx / hy
// say which faces hold them.  Loads first, then the recursions, then the stores.
template <int R>
__device__ __forceinline__ void pml1_4(const Face1 &fz, const Face1 &fx, const Face1 &fy, bool hz, bool hx, bool hy,
                                       bool cross, bool ycross, bool do_y, float (&pz)[4], float (&px)[4],
                                       float (&py)[4]) {
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 zz = z4, zx = z4, zy = z4, xz = z4, xx = z4, xy = z4, yz = z4, yx = z4, yy = z4;  // [face][component]
  const bool zyc = do_y && ycross;
  if (hz) {
    zz = ld4(fz.zc);
    if (cross) zx = ld4(fz.xc);
    if (zyc) zy = ld4(fz.yc);
  }
  if (hx) {
    xx = ld4(fx.xc);
    if (cross) xz = ld4(fx.zc);
    if (zyc) xy = ld4(fx.yc);
  }
  if (hy) {
    if (do_y) yy = ld4(fy.yc);
    if (cross) yz = ld4(fy.zc), yx = ld4(fy.xc);
  }
  const float *cox = fx.co + fx.L * 6, *coy = fy.co + fy.L * 6;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const float *coz = fz.co + (fz.L + c * fz.dl) * 6;
    float m;
    if (hz) m = cmp4(zz, c), pml_round(coz, pz[c], &m), set4(zz, c, m);
    if (cross) {
      if (hx) m = cmp4(xz, c), pml_round(cox + 3, pz[c], &m), set4(xz, c, m);
      if (hy) m = cmp4(yz, c), pml_round(coy + 3, pz[c], &m), set4(yz, c, m);
    }
    if (hx) m = cmp4(xx, c), pml_round(cox, px[c], &m), set4(xx, c, m);
    if (cross) {
      if (hz) m = cmp4(zx, c), pml_round(coz + 3, px[c], &m), set4(zx, c, m);
      if (hy) m = cmp4(yx, c), pml_round(coy + 3, px[c], &m), set4(yx, c, m);
    }
    if (do_y) {
      if (hy) m = cmp4(yy, c), pml_round(coy, py[c], &m), set4(yy, c, m);
      if (ycross) {
        if (hz) m = cmp4(zy, c), pml_round(coz + 3, py[c], &m), set4(zy, c, m);
        if (hx) m = cmp4(xy, c), pml_round(cox + 3, py[c], &m), set4(xy, c, m);
      }
    }
  }
  if (hz) {
    st4(fz.zc, zz);
    if (cross) st4(fz.xc, zx);
    if (zyc) st4(fz.yc, zy);
  }
  if (hx) {
    st4(fx.xc, xx);
    if (cross) st4(fx.zc, xz);
    if (zyc) st4(fx.yc, xy);
  }
  if (hy) {
    if (do_y) st4(fy.yc, yy);
    if (cross) st4(fy.zc, yz), st4(fy.xc, yx);
  }
}

// Per-thread PML state of a tile marching y from y0: the x and z faces of the thread's
// cells (fixed over the planes; z faces a multiple of 4 cells wide) and the y face of a
// plane.
template <int R>
struct TilePml {
  Face1 fx{}, fz{};
  bool hx = false, hz = false;
  __device__ __forceinline__ void init(const PmlDev &P, const Grid3 &g, int ix, int iz4, int y0, bool act) {
    const int nx = g.nx, nz = g.nz;
    if (act && (ix < P.f[DX][0].w || ix >= nx - P.f[DX][1].w)) {
      const int s = ix < P.f[DX][0].w ? 0 : 1;
      const PmlFace &F = P.f[DX][s];
      const int w = F.w;
      const long long idx = ((long long)y0 * w + (s ? ix - (nx - w) : ix)) * nz + iz4;
      fx = face1<R>(F, DX, idx, (long long)w * nz, s ? nx - 1 - ix : ix, 0);
      hx = true;
    }
    if (act && (iz4 < P.f[DZ][0].w || iz4 >= nz - P.f[DZ][1].w)) {
      const int s = iz4 < P.f[DZ][0].w ? 0 : 1;
      const PmlFace &F = P.f[DZ][s];
      const int w = F.w;
      const long long idx = ((long long)y0 * nx + ix) * w + (s ? iz4 - (nz - w) : iz4);
      fz = face1<R>(F, DZ, idx, (long long)nx * w, s ? nz - 1 - iz4 : iz4, s ? -1 : 1);
      hz = true;
    }
  }
  // the y face holding plane iy (hy = false when none)
  __device__ __forceinline__ Face1 yface(const PmlDev &P, const Grid3 &g, int ix, int iz4, int iy, bool &hy) const {
    hy = iy < P.f[DY][0].w || iy >= g.ny - P.f[DY][1].w;
    if (!hy) return Face1{};
    const int s = iy < P.f[DY][0].w ? 0 : 1;
    const PmlFace &F = P.f[DY][s];
    const long long idx = ((long long)(s ? iy - (g.ny - F.w) : iy) * g.nx + ix) * g.nz + iz4;
    return face1<R>(F, DY, idx, 0, s ? g.ny - 1 - iy : iy, 0);
  }
  __device__ __forceinline__ void advance() {
    if (hx) fx.zc += fx.stride, fx.xc += fx.stride, fx.yc += fx.stride;
    if (hz) fz.zc += fz.stride, fz.xc += fz.stride, fz.yc += fz.stride;
  }
  // L1 prefetch of the x / z face memory k planes ahead and of the y face of plane y
  __device__ __forceinline__ void prefetch(const PmlDev &P, const Grid3 &g, int ix, int iz4, int y, int k,
                                           bool cross, bool yc) const {
    auto pf = [](const float *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(__cvta_generic_to_global(p))); };
    if (hx) {
      pf(fx.xc + k * fx.stride);
      if (cross) pf(fx.zc + k * fx.stride);
      if (yc) pf(fx.yc + k * fx.stride);
    }
    if (hz) {
      pf(fz.zc + k * fz.stride);
      if (cross) pf(fz.xc + k * fz.stride);
      if (yc) pf(fz.yc + k * fz.stride);
    }
    bool hy;
    const Face1 fy = yface(P, g, ix, iz4, y, hy);
    if (hy) {
      pf(fy.yc);
      if (cross) pf(fy.zc), pf(fy.xc);
    }
  }
};

// ---- pass 1: gradient -----------------------------------------------------------
template <int TX, int P, int NM>
struct __align__(128) Grad4Smem {
  static constexpr int HX = TX + 2 * R4;
  static constexpr int SA = 5 + P;  // planes iy .. iy+4+P of the haloed w1 tile
  static constexpr int SB = P + 1;  // planes iy .. iy+P of the anisotropy parameters
  float4 a[SA][HX][10];
  float4 m[SB][NM][TX][8];
  uint64_t bar_a[SA];
  uint64_t bar_b[SB];
};

template <int TX, int P, int MODEL, bool EDGE>
__global__ void __launch_bounds__(8 * TX, EDGE ? 384 / (8 * TX) : 0)
    grad4_k(const __grid_constant__ GradArgs a, const Tile4 *__restrict__ tiles, const __grid_constant__ Grad4Maps mp,
            int *err) {
  constexpr int NM = MODEL == 3 ? 4 : MODEL == 2 ? 2 : 1;
  using S = Grad4Smem<TX, P, NM>;
  constexpr int SA = S::SA, SB = S::SB, HX = S::HX;
  constexpr uint32_t BYTES_A = HX * 160, BYTES_B = (MODEL >= 2 ? NM : 0) * TX * 128;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S &s = *reinterpret_cast<S *>(smem_raw);
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const Grid3 g{nx, ny, nz, (long long)nx * nz};
  const int tzq = threadIdx.x, tx = threadIdx.y;
  const Tile4 tile = tiles[blockIdx.x];
  const int iz0 = tile.bz * 32, ix0 = tile.bx * TX, iz4 = iz0 + 4 * tzq, ix = ix0 + tx;
  const int y0 = tile.y0, y1 = tile.y1;
  const bool act = iz4 < nz && ix < nx;
  const bool producer = tzq == 0 && tx == 0;
  const long long col = (long long)ix * nz + iz4;
  const bool do_y = ny > 1;
  const bool cross = a.pml3d != 0, ycross = a.pml3d != 0 && ny > 1;
  const int zl = a.pml.f[DZ][0].w, zh = a.pml.f[DZ][1].w;
  const bool z4ok = zl % 4 == 0 && zh % 4 == 0;
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);

  auto issue_a = [&](int p) {
    const int st = (p - y0) % SA;
    if (p >= ny) {  // beyond the grid: zeros written here, no copy
      for (int k = 0; k < HX * 10; k++) (&s.a[st][0][0])[k] = zero4;
      mbar_arrive(&s.bar_a[st]);
      return;
    }
    mbar_expect_tx(&s.bar_a[st], BYTES_A);
    tma_load_3d(&s.a[st][0][0], &mp.w1, &s.bar_a[st], iz0 - R4, ix0 - R4, p);
  };
  auto issue_b = [&](int p) {
    const int st = (p - y0) % SB;
    if (MODEL < 2) {
      mbar_arrive(&s.bar_b[st]);
      return;
    }
    mbar_expect_tx(&s.bar_b[st], BYTES_B);
#pragma unroll
    for (int k = 0; k < NM; k++) tma_load_3d(&s.m[st][k][0][0], &mp.m[k], &s.bar_b[st], iz0, ix0, p);
  };
  if (producer) {
    for (int k = 0; k < SA; k++) mbar_init(&s.bar_a[k], 1);
    for (int k = 0; k < SB; k++) mbar_init(&s.bar_b[k], 1);
    mbar_fence_init();
  }
  __syncthreads();
  int last_a = y0 - 1, last_b = y0 - 1;  // last planes the producer issued
  if (producer) {
    for (int p = y0; p < min(y0 + R4 + P, y1 + R4); p++) issue_a(p), last_a = p;
    for (int p = y0; p < min(y0 + P, y1); p++) issue_b(p), last_b = p;
  }
  const float4 *__restrict__ w1g = reinterpret_cast<const float4 *>(a.w1);
  const long long nxz4 = g.nxz / 4, col4 = col / 4;
  float4 q[2 * R4 + 1];
#pragma unroll
  for (int k = 0; k < 2 * R4; k++) {
    const int y = y0 - R4 + k;
    q[k] = act && y >= 0 && y < ny ? __ldg(w1g + y * nxz4 + col4) : zero4;
  }
  TilePml<0> pm;
  if constexpr (EDGE) {
    if (z4ok) {
      pm.init(a.pml, g, ix, iz4, y0, act);
      if (act)
        for (int y = y0; y < min(y0 + 2, y1); y++) pm.prefetch(a.pml, g, ix, iz4, y, y - y0, cross, do_y && ycross);
    }
  }
  bool ok = true;
#pragma unroll 1
  for (int iy = y0; iy < y1; iy++) {
    if (producer && ok) {  // after a failed wait nothing more is issued
      if (iy + R4 + P < y1 + R4) issue_a(iy + R4 + P), last_a = iy + R4 + P;
      if (iy + P < y1) issue_b(iy + P), last_b = iy + P;
    }
    if constexpr (EDGE) {
      if (z4ok && act && iy + 2 < y1) pm.prefetch(a.pml, g, ix, iz4, iy + 2, 2, cross, do_y && ycross);
    }
    const int r0 = iy - y0, sa0 = r0 % SA, sa4 = (r0 + R4) % SA, sb = r0 % SB;
    if (r0 < R4) ok = ok && mbar_wait(&s.bar_a[sa0], (uint32_t)((r0 / SA) & 1), err);
    ok = ok && mbar_wait(&s.bar_a[sa4], (uint32_t)(((r0 + R4) / SA) & 1), err);
    ok = ok && mbar_wait(&s.bar_b[sb], (uint32_t)((r0 / SB) & 1), err);
    q[2 * R4] = s.a[sa4][tx + R4][tzq + 1];
    if (act && ok) {
      const float4 zL = s.a[sa0][tx + R4][tzq], zR = s.a[sa0][tx + R4][tzq + 2];
      const float4 u4 = q[R4];
      const float zw[12] = {zL.x, zL.y, zL.z, zL.w, u4.x, u4.y, u4.z, u4.w, zR.x, zR.y, zR.z, zR.w};
      float gz[4] = {0.f, 0.f, 0.f, 0.f}, gx[4] = {0.f, 0.f, 0.f, 0.f}, gy[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int m = 1; m <= R4; m++) {
        const float4 xm = s.a[sa0][tx + R4 - m][tzq + 1], xp = s.a[sa0][tx + R4 + m][tzq + 1];
#pragma unroll
        for (int c = 0; c < 4; c++) {
          gz[c] = d1_acc(gz[c], a.c1z[m], zw[4 + c + m], zw[4 + c - m]);
          gx[c] = d1_acc(gx[c], a.c1x[m], cmp4(xp, c), cmp4(xm, c));
          if (do_y) gy[c] = d1_acc(gy[c], a.c1y[m], cmp4(q[R4 + m], c), cmp4(q[R4 - m], c));
        }
      }
      const long long i0 = (long long)iy * g.nxz + col;
      if (a.io.store | a.io.ic) fused_io4(a.io, g, i0, ix, iy, iz4, col, u4);
      if constexpr (EDGE) {
        if (z4ok) {
          bool hy;
          const Face1 fy = pm.yface(a.pml, g, ix, iz4, iy, hy);
          if (pm.hx || pm.hz || hy) pml1_4<0>(pm.fz, pm.fx, fy, pm.hz, pm.hx, hy, cross, ycross, do_y, gz, gx, gy);
        } else {
#pragma unroll
          for (int c = 0; c < 4; c++)
            if (in_pml(a.pml, g, ix, iy, iz4 + c))
              pml1_all<0>(a.pml, g, a.pml3d, do_y, ix, iy, iz4 + c, gz[c], gx[c], gy[c]);
        }
      }
      if (MODEL == 2 || MODEL == 3) {
        float4 mv[4];
#pragma unroll
        for (int k = 0; k < NM; k++) mv[k] = s.m[sb][k][tx][tzq];
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const float4 cm = make_float4(cmp4(mv[0], c), NM > 1 ? cmp4(mv[1], c) : 0.f, NM > 2 ? cmp4(mv[2], c) : 0.f,
                                        NM > 3 && do_y ? cmp4(mv[3], c) : 0.f);
          aniso_scale<MODEL>(cm, gx[c], gy[c], gz[c]);
        }
      }
      st4(a.px + i0, make_float4(gx[0], gx[1], gx[2], gx[3]));
      st4(a.pz + i0, make_float4(gz[0], gz[1], gz[2], gz[3]));
      if (do_y) st4(a.py + i0, make_float4(gy[0], gy[1], gy[2], gy[3]));
    }
    if constexpr (EDGE) pm.advance();
    __syncthreads();  // every thread is done with the stages the producer refills next
#pragma unroll
    for (int k = 0; k < 2 * R4; k++) q[k] = q[k + 1];
  }
  // After the producer's own wait gave up, its last copies (at most one per stage)
  // may still be in flight: it waits for them, bounded, before the CTA leaves.
  if (producer && !ok) {
    for (int p = max(y0, last_a - SA + 1); p <= last_a; p++) mbar_drain(&s.bar_a[(p - y0) % SA], ((p - y0) / SA) & 1);
    for (int p = max(y0, last_b - SB + 1); p <= last_b; p++) mbar_drain(&s.bar_b[(p - y0) % SB], ((p - y0) / SB) & 1);
  }
}

// ---- pass 2: divergence ---------------------------------------------------------
template <int TX, int P>
struct __align__(128) Div4Smem {
  // ring A feeds the y queue: plane p (>= y0 + 4) is issued at step p-4-P and read at step p-4
  static constexpr int SA = P + 2;
  static constexpr int SB = P + 1;  // planes iy .. iy+P of px (x halo), pz (z halo), w0, vel, w1
  float4 py[SA][TX][8];
  float4 px[SB][TX + 2 * R4][8];
  float4 pz[SB][TX][10];
  float4 w[SB][3][TX][8];  // w0, (v dt)^2, w1
  uint64_t bar_a[SA];
  uint64_t bar_b[SB];
};

// The visco-acoustic operands of ring B's planes (after Div4Smem in shared
// memory): the d0 / d1 halves of the Q memory, orders [0, kDiv4QMax), and 1/Q.
template <int TX, int SB, typename QT>
struct __align__(128) Div4QRing {
  QT qa[SB][kDiv4QMax][TX][32];
  QT qb[SB][kDiv4QMax][TX][32];
  float iq[SB][TX][32];
};

template <int QR>
using QType = typename std::conditional<QR == 2, __nv_bfloat16, float>::type;

template <int TX, int P, int QR>
constexpr size_t div4_smem() {
  return sizeof(Div4Smem<TX, P>) + (QR ? sizeof(Div4QRing<TX, Div4Smem<TX, P>::SB, QType<QR>>) : 0);
}

// QR: 0 the Q update loads its own operands; 1 / 2 ring B also carries the Q
// memory (FP32 / BF16) and 1/Q of its planes (MODE 2, order <= kDiv4QMax)
template <int TX, int P, int MODE, bool EDGE, int QR>
__global__ void __launch_bounds__(8 * TX, EDGE && MODE != 2 ? 384 / (8 * TX) : 0)
    div4_k(const __grid_constant__ DivArgs a, const Tile4 *__restrict__ tiles, const __grid_constant__ Div4Maps mp,
           int *err) {
  using S = Div4Smem<TX, P>;
  constexpr int SA = S::SA, SB = S::SB;
  using QT = QType<QR>;
  using QRing = Div4QRing<TX, SB, QT>;
  constexpr uint32_t BYTES_A = TX * 128, BYTES_B = (TX + 2 * R4) * 128 + TX * 160 + 3 * TX * 128;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S &s = *reinterpret_cast<S *>(smem_raw);
  QRing &qr = *reinterpret_cast<QRing *>(smem_raw + sizeof(S));
  const uint32_t bytes_q = QR ? (uint32_t)(2 * a.q.order * TX * 32 * sizeof(QT) + TX * 32 * 4) : 0u;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const Grid3 g{nx, ny, nz, (long long)nx * nz};
  const int tzq = threadIdx.x, tx = threadIdx.y;
  const Tile4 tile = tiles[blockIdx.x];
  const int iz0 = tile.bz * 32, ix0 = tile.bx * TX, iz4 = iz0 + 4 * tzq, ix = ix0 + tx;
  const int y0 = tile.y0, y1 = tile.y1;
  const bool act = iz4 < nz && ix < nx;
  const bool producer = tzq == 0 && tx == 0;
  const long long col = (long long)ix * nz + iz4;
  const bool do_y = ny > 1;
  const bool cross = a.pml3d != 0, ycross = a.pml3d != 0 && ny > 1;
  const int zl = a.pml.f[DZ][0].w, zh = a.pml.f[DZ][1].w;
  const bool z4ok = zl % 4 == 0 && zh % 4 == 0;
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);

  // ring-A plane p (>= y0 + 4) lives in stage (p - y0 - 4) % SA, phase ((p - y0 - 4) / SA) & 1
  auto issue_a = [&](int p) {
    const int st = (p - y0 - R4) % SA;
    if (p >= ny || !do_y) {  // beyond the grid (or no y derivative): zeros, no copy
      for (int k = 0; k < TX * 8; k++) (&s.py[st][0][0])[k] = zero4;
      mbar_arrive(&s.bar_a[st]);
      return;
    }
    mbar_expect_tx(&s.bar_a[st], BYTES_A);
    tma_load_3d(&s.py[st][0][0], &mp.py, &s.bar_a[st], iz0, ix0, p);
  };
  auto issue_b = [&](int p) {
    const int st = (p - y0) % SB;
    mbar_expect_tx(&s.bar_b[st], BYTES_B + bytes_q);
    tma_load_3d(&s.px[st][0][0], &mp.px, &s.bar_b[st], iz0, ix0 - R4, p);
    tma_load_3d(&s.pz[st][0][0], &mp.pz, &s.bar_b[st], iz0 - R4, ix0, p);
    tma_load_3d(&s.w[st][0][0][0], &mp.w0, &s.bar_b[st], iz0, ix0, p);
    tma_load_3d(&s.w[st][1][0][0], &mp.vel, &s.bar_b[st], iz0, ix0, p);
    tma_load_3d(&s.w[st][2][0][0], &mp.w1, &s.bar_b[st], iz0, ix0, p);
    if constexpr (QR != 0) {
      tma_load_4d(&qr.qa[st][0][0][0], &mp.qa, &s.bar_b[st], iz0, ix0, p, 0);
      tma_load_4d(&qr.qb[st][0][0][0], &mp.qb, &s.bar_b[st], iz0, ix0, p, 0);
      tma_load_3d(&qr.iq[st][0][0], &mp.iq, &s.bar_b[st], iz0, ix0, p);
    }
  };
  if (producer) {
    for (int k = 0; k < SA; k++) mbar_init(&s.bar_a[k], 1);
    for (int k = 0; k < SB; k++) mbar_init(&s.bar_b[k], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // ring A carries planes y0+4 .. y1+3 only (the queue starts with planes
  // y0-4 .. y0+3 read from global memory), so every copy it gets is waited for
  int last_a = y0 + R4 - 1, last_b = y0 - 1;
  if (producer) {
    for (int p = y0 + R4; p < min(y0 + R4 + P, y1 + R4); p++) issue_a(p), last_a = p;
    for (int p = y0; p < min(y0 + P, y1); p++) issue_b(p), last_b = p;
  }
  const float4 *__restrict__ pyg = reinterpret_cast<const float4 *>(a.py);
  const long long nxz4 = g.nxz / 4, col4 = col / 4;
  float4 q[2 * R4 + 1];
#pragma unroll
  for (int k = 0; k < 2 * R4; k++) {
    const int y = y0 - R4 + k;
    q[k] = do_y && act && y >= 0 && y < ny ? __ldg(pyg + y * nxz4 + col4) : zero4;
  }
  TilePml<1> pm;
  if constexpr (EDGE) {
    if (z4ok) {
      pm.init(a.pml, g, ix, iz4, y0, act);
      if (act)
        for (int y = y0; y < min(y0 + 2, y1); y++) pm.prefetch(a.pml, g, ix, iz4, y, y - y0, cross, do_y && ycross);
    }
  }
  bool ok = true;
#pragma unroll 1
  for (int iy = y0; iy < y1; iy++) {
    if (producer && ok) {
      if (iy + R4 + P < y1 + R4) issue_a(iy + R4 + P), last_a = iy + R4 + P;
      if (iy + P < y1) issue_b(iy + P), last_b = iy + P;
    }
    if constexpr (EDGE) {
      if (z4ok && act && iy + 2 < y1) pm.prefetch(a.pml, g, ix, iz4, iy + 2, 2, cross, do_y && ycross);
    }
    const int r0 = iy - y0, sa4 = r0 % SA, sb = r0 % SB;
    ok = ok && mbar_wait(&s.bar_a[sa4], (uint32_t)((r0 / SA) & 1), err);
    ok = ok && mbar_wait(&s.bar_b[sb], (uint32_t)((r0 / SB) & 1), err);
    q[2 * R4] = s.py[sa4][tx][tzq];
    if (act && ok) {
      const float4 zL = s.pz[sb][tx][tzq], zc = s.pz[sb][tx][tzq + 1], zR = s.pz[sb][tx][tzq + 2];
      const float zw[12] = {zL.x, zL.y, zL.z, zL.w, zc.x, zc.y, zc.z, zc.w, zR.x, zR.y, zR.z, zR.w};
      float dx[4] = {0.f, 0.f, 0.f, 0.f}, dz[4] = {0.f, 0.f, 0.f, 0.f}, dy[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int m = 1; m <= R4; m++) {
        const float4 xm = s.px[sb][tx + R4 - m][tzq], xp = s.px[sb][tx + R4 + m][tzq];
#pragma unroll
        for (int c = 0; c < 4; c++) {
          dx[c] = d1_acc(dx[c], a.c1x[m], cmp4(xp, c), cmp4(xm, c));
          dz[c] = d1_acc(dz[c], a.c1z[m], zw[4 + c + m], zw[4 + c - m]);
          if (do_y) dy[c] = d1_acc(dy[c], a.c1y[m], cmp4(q[R4 + m], c), cmp4(q[R4 - m], c));
        }
      }
      const long long i0 = (long long)iy * g.nxz + col;
      if constexpr (EDGE) {
        if (z4ok) {
          bool hy;
          const Face1 fy = pm.yface(a.pml, g, ix, iz4, iy, hy);
          if (pm.hx || pm.hz || hy) pml1_4<1>(pm.fz, pm.fx, fy, pm.hz, pm.hx, hy, cross, ycross, do_y, dz, dx, dy);
        } else {
#pragma unroll
          for (int c = 0; c < 4; c++)
            if (in_pml(a.pml, g, ix, iy, iz4 + c))
              pml1_all<1>(a.pml, g, a.pml3d, do_y, ix, iy, iz4 + c, dz[c], dx[c], dy[c]);
        }
      }
      const float4 cw0 = s.w[sb][0][tx][tzq], cvel = s.w[sb][1][tx][tzq], cw1 = s.w[sb][2][tx][tzq];
      float4 t4, out4;
#pragma unroll
      for (int c = 0; c < 4; c++) set4(t4, c, div_accumulate(cmp4(cw0, c), cmp4(cvel, c), dx[c], dz[c], dy[c]));
      if (MODE == 0) {
        out4 = t4;
      } else if (MODE == 1) {
#pragma unroll
        for (int c = 0; c < 4; c++) set4(out4, c, __fsub_rn(__fadd_rn(cmp4(cw1, c), cmp4(cw1, c)), cmp4(t4, c)));
      } else if constexpr (QR != 0) {
        const float4 iq4 = *reinterpret_cast<const float4 *>(&qr.iq[sb][tx][4 * tzq]);
        out4 = q_update4_ring<QT>(a.q, i0, (long long)ny * g.nxz, t4, cw1, &qr.qa[sb][0][tx][4 * tzq],
                                  &qr.qb[sb][0][tx][4 * tzq], TX * 32, iq4);
      } else {
        out4 = q_update4(a.q, i0, (long long)ny * g.nxz, t4, cw1);
      }
      st4(a.w0 + i0, out4);
    }
    if constexpr (EDGE) pm.advance();
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 2 * R4; k++) q[k] = q[k + 1];
  }
  if (producer && !ok) {
    for (int p = max(y0 + R4, last_a - SA + 1); p <= last_a; p++)
      mbar_drain(&s.bar_a[(p - y0 - R4) % SA], ((p - y0 - R4) / SA) & 1);
    for (int p = max(y0, last_b - SB + 1); p <= last_b; p++) mbar_drain(&s.bar_b[(p - y0) % SB], ((p - y0) / SB) & 1);
  }
}

// ---- host side -------------------------------------------------------------------
template <int TX, int P, int MODEL>
size_t grad4_smem() {
  return sizeof(Grad4Smem<TX, P, MODEL == 3 ? 4 : MODEL == 2 ? 2 : 1>);
}

template <int TX, int P, int MODEL, bool EDGE>
bool grad4_attr1() {
  return cudaFuncSetAttribute(grad4_k<TX, P, MODEL, EDGE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)grad4_smem<TX, P, MODEL>()) == cudaSuccess;
}
template <int TX, int P, int MODE, bool EDGE, int QR = 0>
bool div4_attr1() {
  return cudaFuncSetAttribute(div4_k<TX, P, MODE, EDGE, QR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)div4_smem<TX, P, QR>()) == cudaSuccess;
}

constexpr int kTX = kAniso4TX, kP = 2;

}  // namespace

bool aniso4_init() {
  bool ok = true;
  ok &= grad4_attr1<kTX, kP, 2, false>() && grad4_attr1<kTX, kP, 2, true>();
  ok &= grad4_attr1<kTX, kP, 3, false>() && grad4_attr1<kTX, kP, 3, true>();
  ok &= div4_attr1<kTX, kP, 0, false>() && div4_attr1<kTX, kP, 0, true>();
  ok &= div4_attr1<kTX, kP, 1, false>() && div4_attr1<kTX, kP, 1, true>();
  ok &= div4_attr1<kTX, kP, 2, false>() && div4_attr1<kTX, kP, 2, true>();
  ok &= div4_attr1<kTX, kP, 2, false, 1>() && div4_attr1<kTX, kP, 2, true, 1>();
  ok &= div4_attr1<kTX, kP, 2, false, 2>() && div4_attr1<kTX, kP, 2, true, 2>();
  return ok;
}

int aniso4_ctas_per_sm() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, div4_k<kTX, kP, 1, false, 0>, 8 * kTX, div4_smem<kTX, kP, 0>());
  return n > 0 ? n : 1;
}

void launch_grad4(const GradArgs &a, const Tile4 *tiles, int ntiles, bool edge, int model, const Grad4Maps &m,
                  int *err, cudaStream_t st) {
  if (ntiles <= 0) return;
  const dim3 block(8, kTX);
#define G_(MD, E) grad4_k<kTX, kP, MD, E><<<ntiles, block, grad4_smem<kTX, kP, MD>(), st>>>(a, tiles, m, err)
  if (model == 3) {
    if (edge) G_(3, true);
    else G_(3, false);
  } else {
    if (edge) G_(2, true);
    else G_(2, false);
  }
#undef G_
}

void launch_div4(const DivArgs &a, const Tile4 *tiles, int ntiles, bool edge, int mode, const Div4Maps &m, int *err,
                 cudaStream_t st) {
  if (ntiles <= 0) return;
  const dim3 block(8, kTX);
#define D_(MD, E, QR) div4_k<kTX, kP, MD, E, QR><<<ntiles, block, div4_smem<kTX, kP, QR>(), st>>>(a, tiles, m, err)
  if (mode == 0) {
    if (edge) D_(0, true, 0);
    else D_(0, false, 0);
  } else if (mode == 1) {
    if (edge) D_(1, true, 0);
    else D_(1, false, 0);
  } else if (m.qring == 1) {
    if (edge) D_(2, true, 1);
    else D_(2, false, 1);
  } else if (m.qring == 2) {
    if (edge) D_(2, true, 2);
    else D_(2, false, 2);
  } else {
    if (edge) D_(2, true, 0);
    else D_(2, false, 0);
  }
#undef D_
}

}  // namespace rtm
