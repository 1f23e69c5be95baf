// kernels_fd8.cu - 8th-order finite-difference time-step kernels for sm_100a.
//
// Tiling: a CTA owns a 32 (z) x TX (x) column tile and marches along y, the
// slowest axis.  Each thread keeps its column's +-4 y neighbours in a
// register queue; the current y plane of the tile plus a 4-cell x/z halo is
// staged in shared memory, so every wavefield value is fetched from L2 about
// once per plane and from HBM about once per step.  Warps run along z, the
// contiguous axis: all global accesses are 128-byte coalesced rows.
//
//  iso_fd8_step   KernelCPU::ISO + FdEngine_fd::laplacian_irreg + pml2_bnd
//                 (bgprtm/KernelCPU.cpp:125-140, bgprtm/FdEngine_fd.cpp:204-325)
//                 fused with update2nd (bgprtm/Propagator.cpp:1767-1818), the
//                 snapshot store / imaging condition of the previous step.
//  grad_fd8       first pass of KernelCPU::TTI (bgprtm/KernelCPU.cpp:93-119):
//                 gradient with PML round 1 and the VTI/TTI scaling
//                 (bgprtm/KernelCPU.cpp:176-297).
//  div_fd8        second pass: divergence with PML round 2, accumulated into
//                 w0, fused with update2nd.
#include <algorithm>

#include "kernel_api.h"
#include "rtm_device.cuh"

namespace rtm {

namespace {

constexpr int TZ = 32;
constexpr int R = 4;  // stencil radius (order 8)

__device__ __forceinline__ float ld_or0(const float *__restrict__ p, long long i, bool ok) {
  return ok ? __ldg(p + i) : 0.0f;
}

// Halo values a thread stages into the plane tile: two z-halo cells (threads
// tz < R) and two x-halo cells (threads tx < R).  Fetched two planes ahead so
// the loads overlap the compute of the current plane.
struct Halo {
  float zl, zh, xl, xh;
};

template <int TX>
__device__ __forceinline__ Halo fetch_halo(const float *__restrict__ f, int iy, int ny, int ix, int iz, int nx, int nz,
                                           long long nxz, int tx, int tz) {
  Halo h{0.f, 0.f, 0.f, 0.f};
  if (iy < 0 || iy >= ny) return h;
  const long long plane = (long long)iy * nxz;
  if (tz < R) {
    const int izl = iz - R, izh = iz + TZ;
    h.zl = ld_or0(f, plane + (long long)ix * nz + izl, ix < nx && izl >= 0);
    h.zh = ld_or0(f, plane + (long long)ix * nz + izh, ix < nx && izh < nz);
  }
  if (tx < R) {
    const int ixl = ix - R, ixh = ix + TX;
    h.xl = ld_or0(f, plane + (long long)ixl * nz + iz, iz < nz && ixl >= 0);
    h.xh = ld_or0(f, plane + (long long)ixh * nz + iz, iz < nz && ixh < nx);
  }
  return h;
}

// fetch_halo with an accessor v(i, iy) for the wavefield (FP16 state)
template <int TX, typename V>
__device__ __forceinline__ Halo fetch_halo_v(V v, int iy, int ny, int ix, int iz, int nx, int nz, long long nxz, int tx,
                                             int tz) {
  Halo h{0.f, 0.f, 0.f, 0.f};
  if (iy < 0 || iy >= ny) return h;
  const long long plane = (long long)iy * nxz;
  if (tz < R) {
    const int izl = iz - R, izh = iz + TZ;
    if (ix < nx && izl >= 0) h.zl = v(plane + (long long)ix * nz + izl, iy);
    if (ix < nx && izh < nz) h.zh = v(plane + (long long)ix * nz + izh, iy);
  }
  if (tx < R) {
    const int ixl = ix - R, ixh = ix + TX;
    if (iz < nz && ixl >= 0) h.xl = v(plane + (long long)ixl * nz + iz, iy);
    if (iz < nz && ixh < nx) h.xh = v(plane + (long long)ixh * nz + iz, iy);
  }
  return h;
}

// FP16 state value: half * per-slab scale
__device__ __forceinline__ float f16v(const __half *h, const float *s, long long i, int iy) {
  return __half2float(h[i]) * __ldg(s + iy);
}

template <int TX>
__device__ __forceinline__ void put_tile(float (*tile)[TZ + 2 * R], const Halo &h, float c, int tx, int tz) {
  tile[tx + R][tz + R] = c;
  if (tz < R) tile[tx + R][tz] = h.zl, tile[tx + R][tz + TZ + R] = h.zh;
  if (tx < R) tile[tx][tz + R] = h.xl, tile[tx + TX + R][tz + R] = h.xh;
}

// One 32 (z) x TX (x) column tile of an ISO step, marching y over segment
// bz (planes bz*yseg .. ), tile (bx, by); w1 / w0 are the wavefields of this
// step (the batched kernel passes a shot's buffers of the current parity).
// The coefficients and the PML widths are read once into registers.
template <int TX, int MODE, bool PML3D>
__device__ __forceinline__ void iso_tile(const IsoArgs &a, const float *__restrict__ w1, float *__restrict__ w0, int bx,
                                         int by, int bz, float (*tile)[TZ + 2 * R]) {
  const int nx = a.nx, ny = a.ny, nz = a.nz, yseg = a.yseg;
  const Grid3 g{nx, ny, nz, (long long)nx * nz};
  float c2x[R + 1], c2y[R + 1], c2z[R + 1];
#pragma unroll
  for (int m = 0; m <= R; m++) c2x[m] = a.c2x[m], c2y[m] = a.c2y[m], c2z[m] = a.c2z[m];
  const int zl = a.pml.f[DZ][0].w, zh = a.pml.f[DZ][1].w, xl = a.pml.f[DX][0].w, xh = a.pml.f[DX][1].w,
            yl = a.pml.f[DY][0].w, yh = a.pml.f[DY][1].w;
  const float *__restrict__ vel = a.vel;
  const int tz = threadIdx.x, tx = threadIdx.y;
  const int iz = bx * TZ + tz;
  const int ix = by * TX + tx;
  const int y0 = bz * yseg;
  const int y1 = min(ny, y0 + yseg);
  const bool act = iz < nz && ix < nx;
  const long long col = (long long)ix * nz + iz;
  const bool do_y = ny > 2;
  const bool xz_edge = iz < zl || iz >= nz - zh || ix < xl || ix >= nx - xh;

  float q[2 * R + 1];
#pragma unroll
  for (int k = 0; k < 2 * R; k++) {
    const int y = y0 - R + k;
    q[k] = ld_or0(w1, (long long)y * g.nxz + col, act && y >= 0 && y < ny);
  }
  Halo h0 = fetch_halo<TX>(w1, y0, ny, ix, iz, nx, nz, g.nxz, tx, tz);
  Halo h1 = fetch_halo<TX>(w1, y0 + 1, ny, ix, iz, nx, nz, g.nxz, tx, tz);
  // per-cell inputs of the next plane
  float nw0 = act ? w0[(long long)y0 * g.nxz + col] : 0.f;
  float nvel = act ? __ldg(vel + (long long)y0 * g.nxz + col) : 0.f;
  for (int iy = y0; iy < y1; iy++) {
    q[2 * R] = ld_or0(w1, (long long)(iy + R) * g.nxz + col, act && iy + R < ny);
    const long long plane = (long long)iy * g.nxz;
    put_tile<TX>(tile, h0, q[R], tx, tz);
    h0 = h1;
    h1 = fetch_halo<TX>(w1, iy + 2 < y1 ? iy + 2 : ny, ny, ix, iz, nx, nz, g.nxz, tx, tz);
    const float cw0 = nw0, cvel = nvel;
    if (act && iy + 1 < y1) {
      nw0 = w0[plane + g.nxz + col];
      nvel = __ldg(vel + plane + g.nxz + col);
    }
    __syncthreads();
    if (act) {
      const float u = q[R];
      float lz = c2z[0] * u, lx = c2x[0] * u, ly = 0.0f;
#pragma unroll
      for (int m = 1; m <= R; m++) {
        lz += c2z[m] * (tile[tx + R][tz + R - m] + tile[tx + R][tz + R + m]);
        lx += c2x[m] * (tile[tx + R - m][tz + R] + tile[tx + R + m][tz + R]);
      }
      if (do_y) {
        ly = c2y[0] * u;
#pragma unroll
        for (int m = 1; m <= R; m++) ly += c2y[m] * (q[R - m] + q[R + m]);
      }
      float v;
      const bool edge = xz_edge || iy < yl || iy >= ny - yh;
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
      const long long i = plane + col;
      if (a.io.store | a.io.ic) fused_io(a.io, g, i, ix, iy, iz, col, u);
      const float t = cw0 - v * cvel;
      float out;
      if (MODE == 0) out = t;                         // KernelCPU seam: w0 -= vel * L[w1]
      else if (MODE == 1) out = (u + u) - t;          // + update2nd (leapfrog)
      else out = q_update(a.q, i, (long long)ny * g.nxz, t, u);  // + Q
      w0[i] = out;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 2 * R; k++) q[k] = q[k + 1];
  }
}

template <int TX, int MODE, bool PML3D>
__global__ void __launch_bounds__(TZ *TX) iso_fd8_step(IsoArgs a) {
  __shared__ float tile[TX + 2 * R][TZ + 2 * R];
  iso_tile<TX, MODE, PML3D>(a, a.w1, a.w0, blockIdx.x, blockIdx.y, blockIdx.z, tile);
}

// Many shots in one persistent launch: the work items are the column tiles of
// the active shots (a prefix of the step-count-sorted batch), laid end to end
// (start[s] = first item of shot s); each CTA strides over them.  Shot s
// steps its buffers wa / wb in lockstep with the others: at step `it` w1 is wa
// on even steps and wb on odd ones.  Leapfrog update (MODE 1), no snapshot I/O.
template <int TX, bool PML3D>
__global__ void __launch_bounds__(TZ *TX) iso_fd8_batch(const IsoBatchShot *__restrict__ shots,
                                                         const int *__restrict__ start, int nactive, int total, int it) {
  __shared__ float tile[TX + 2 * R][TZ + 2 * R];
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    int lo = 0, hi = nactive - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(start + mid) <= w) lo = mid;
      else hi = mid - 1;
    }
    const IsoBatchShot &S = shots[lo];
    const int l = w - __ldg(start + lo);
    const int bx = l % S.tiles_z, by = (l / S.tiles_z) % S.tiles_x, bz = l / (S.tiles_z * S.tiles_x);
    const float *w1 = (it & 1) ? S.wb : S.wa;
    float *w0 = (it & 1) ? S.wa : S.wb;
    iso_tile<TX, 1, PML3D>(S.a, w1, w0, bx, by, bz, tile);
  }
}

// ---- anisotropic two-pass ----------------------------------------------------
// One CTA per tile of the table; EDGE = false tiles hold no PML cell and are
// compiled without the PML code (fewer registers, more resident warps).
// The gradient pass of one column tile (z tile bz, x tile bx, planes [y0, y1))
// reading the field w1; every thread of the CTA calls it.
template <int TX, int MODEL, bool F16, bool EDGE>
__device__ __forceinline__ void grad_tile(const GradArgs &a, const float *__restrict__ w1, int bz, int bx, int y0,
                                          int y1, float (&tile)[TX + 2 * R][TZ + 2 * R]) {
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  const int tz = threadIdx.x, tx = threadIdx.y;
  const int iz = bz * TZ + tz;
  const int ix = bx * TX + tx;
  const bool act = iz < a.nz && ix < a.nx;
  const long long col = (long long)ix * a.nz + iz;
  const bool do_y = a.ny > 1;
  auto v1 = [&](long long i, int iy) -> float { return F16 ? f16v(a.h.w1, a.h.s1, i, iy) : __ldg(w1 + i); };

  float q[2 * R + 1];
#pragma unroll
  for (int k = 0; k < 2 * R; k++) {
    const int y = y0 - R + k;
    q[k] = act && y >= 0 && y < a.ny ? v1((long long)y * g.nxz + col, y) : 0.f;
  }
  Halo h0 = fetch_halo_v<TX>(v1, y0, a.ny, ix, iz, a.nx, a.nz, g.nxz, tx, tz);
  Halo h1 = fetch_halo_v<TX>(v1, y0 + 1, a.ny, ix, iz, a.nx, a.nz, g.nxz, tx, tz);
  // anisotropy parameters of the next plane
  float4 nm = make_float4(0.f, 0.f, 0.f, 0.f);
  auto fetch_model = [&](long long i) {
    float4 m = make_float4(0.f, 0.f, 0.f, 0.f);
    if (MODEL >= 2) m.x = __ldg(a.eps + i), m.y = __ldg(a.del + i);
    if (MODEL == 3) m.z = __ldg(a.pjx + i), m.w = do_y ? __ldg(a.pjy + i) : 0.f;
    return m;
  };
  if (act) nm = fetch_model((long long)y0 * g.nxz + col);
  for (int iy = y0; iy < y1; iy++) {
    q[2 * R] = act && iy + R < a.ny ? v1((long long)(iy + R) * g.nxz + col, iy + R) : 0.f;
    const long long plane = (long long)iy * g.nxz;
    put_tile<TX>(tile, h0, q[R], tx, tz);
    h0 = h1;
    h1 = fetch_halo_v<TX>(v1, iy + 2 < y1 ? iy + 2 : a.ny, a.ny, ix, iz, a.nx, a.nz, g.nxz, tx, tz);
    const float4 cm = nm;
    if (act && iy + 1 < y1) nm = fetch_model(plane + g.nxz + col);
    __syncthreads();
    if (act) {
      const long long i = plane + col;
      float gz = 0.f, gx = 0.f, gy = 0.f;
#pragma unroll
      for (int m = 1; m <= R; m++) {
        gz = d1_acc(gz, a.c1z[m], tile[tx + R][tz + R + m], tile[tx + R][tz + R - m]);
        gx = d1_acc(gx, a.c1x[m], tile[tx + R + m][tz + R], tile[tx + R - m][tz + R]);
        if (do_y) gy = d1_acc(gy, a.c1y[m], q[R + m], q[R - m]);
      }
      if (a.io.store | a.io.ic) fused_io(a.io, g, i, ix, iy, iz, col, q[R]);
      if (EDGE && in_pml(a.pml, g, ix, iy, iz)) pml1_all<0>(a.pml, g, a.pml3d, do_y, ix, iy, iz, gz, gx, gy);
      if (a.rho) divide_rho(__ldg(a.rho + i), do_y, gx, gy, gz);
      if (MODEL == 2 || MODEL == 3) aniso_scale<MODEL>(cm, gx, gy, gz);
      a.px[i] = gx;
      a.pz[i] = gz;
      if (do_y) a.py[i] = gy;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 2 * R; k++) q[k] = q[k + 1];
  }
}

template <int TX, int MODEL, bool F16, bool EDGE>
__global__ void __launch_bounds__(TZ *TX) grad_fd8(GradArgs a, const Tile4 *__restrict__ tiles) {
  __shared__ float tile[TX + 2 * R][TZ + 2 * R];
  const Tile4 tl = tiles[blockIdx.x];
  grad_tile<TX, MODEL, F16, EDGE>(a, a.w1, tl.bz, tl.bx, tl.y0, tl.y1, tile);
}

struct DivPlane {
  float pxc, pzc, zl, zh, xl, xh;
};

template <int TX>
__device__ __forceinline__ DivPlane fetch_div(const DivArgs &a, int iy, int ix, int iz, long long nxz, int tx, int tz,
                                              bool act) {
  DivPlane d{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (iy < 0 || iy >= a.ny) return d;
  const long long plane = (long long)iy * nxz, col = (long long)ix * a.nz + iz;
  d.pxc = ld_or0(a.px, plane + col, act);
  d.pzc = ld_or0(a.pz, plane + col, act);
  if (tz < R) {
    const int izl = iz - R, izh = iz + TZ;
    d.zl = ld_or0(a.pz, plane + (long long)ix * a.nz + izl, ix < a.nx && izl >= 0);
    d.zh = ld_or0(a.pz, plane + (long long)ix * a.nz + izh, ix < a.nx && izh < a.nz);
  }
  if (tx < R) {
    const int ixl = ix - R, ixh = ix + TX;
    d.xl = ld_or0(a.px, plane + (long long)ixl * a.nz + iz, iz < a.nz && ixl >= 0);
    d.xh = ld_or0(a.px, plane + (long long)ixh * a.nz + iz, iz < a.nz && ixh < a.nx);
  }
  return d;
}

// The divergence pass of one column tile reading w1 and the previous field w0,
// which it overwrites with the new one; every thread of the CTA calls it.
template <int TX, int MODE, bool F16, bool EDGE>
__device__ __forceinline__ void div_tile(const DivArgs &a, const float *__restrict__ w1, float *w0, int bz, int bx,
                                         int y0, int y1, float (&tpx)[TX + 2 * R][TZ], float (&tpz)[TX][TZ + 2 * R]) {
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  const int tz = threadIdx.x, tx = threadIdx.y;
  const int iz = bz * TZ + tz;
  const int ix = bx * TX + tx;
  const bool act = iz < a.nz && ix < a.nx;
  const long long col = (long long)ix * a.nz + iz;
  const bool do_y = a.ny > 1;

  float q[2 * R + 1];
#pragma unroll
  for (int k = 0; k < 2 * R; k++) {
    const int y = y0 - R + k;
    q[k] = do_y ? ld_or0(a.py, (long long)y * g.nxz + col, act && y >= 0 && y < a.ny) : 0.f;
  }
  DivPlane d0 = fetch_div<TX>(a, y0, ix, iz, g.nxz, tx, tz, act);
  DivPlane d1 = fetch_div<TX>(a, y0 + 1 < y1 ? y0 + 1 : a.ny, ix, iz, g.nxz, tx, tz, act);
  auto v0 = [&](long long i, int iy) -> float { return F16 ? f16v(a.h.w0, a.h.s0, i, iy) : w0[i]; };
  auto v1 = [&](long long i, int iy) -> float { return F16 ? f16v(a.h.w1, a.h.s1, i, iy) : __ldg(w1 + i); };
  float nw0 = act ? v0((long long)y0 * g.nxz + col, y0) : 0.f;
  float nvel = act ? __ldg(a.vel + (long long)y0 * g.nxz + col) : 0.f;
  float nw1 = act && MODE != 0 ? v1((long long)y0 * g.nxz + col, y0) : 0.f;
  float amax = 0.f;
  for (int iy = y0; iy < y1; iy++) {
    if (do_y) q[2 * R] = ld_or0(a.py, (long long)(iy + R) * g.nxz + col, act && iy + R < a.ny);
    const long long plane = (long long)iy * g.nxz;
    tpx[tx + R][tz] = d0.pxc;
    tpz[tx][tz + R] = d0.pzc;
    if (tz < R) tpz[tx][tz] = d0.zl, tpz[tx][tz + TZ + R] = d0.zh;
    if (tx < R) tpx[tx][tz] = d0.xl, tpx[tx + TX + R][tz] = d0.xh;
    d0 = d1;
    d1 = fetch_div<TX>(a, iy + 2 < y1 ? iy + 2 : a.ny, ix, iz, g.nxz, tx, tz, act);
    const float cw0 = nw0, cvel = nvel, cw1 = nw1;
    if (act && iy + 1 < y1) {
      nw0 = v0(plane + g.nxz + col, iy + 1);
      nvel = __ldg(a.vel + plane + g.nxz + col);
      if (MODE != 0) nw1 = v1(plane + g.nxz + col, iy + 1);
    }
    __syncthreads();
    if (act) {
      const long long i = plane + col;
      float dxv = 0.f, dzv = 0.f, dyv = 0.f;
#pragma unroll
      for (int m = 1; m <= R; m++) {
        dxv = d1_acc(dxv, a.c1x[m], tpx[tx + R + m][tz], tpx[tx + R - m][tz]);
        dzv = d1_acc(dzv, a.c1z[m], tpz[tx][tz + R + m], tpz[tx][tz + R - m]);
        if (do_y) dyv = d1_acc(dyv, a.c1y[m], q[R + m], q[R - m]);
      }
      if (EDGE && in_pml(a.pml, g, ix, iy, iz)) pml1_all<1>(a.pml, g, a.pml3d, do_y, ix, iy, iz, dzv, dxv, dyv);
      const float t = a.rho ? div_accumulate_rho<-1>(cw0, cvel, __ldg(a.rho + i), dxv, dzv, dyv)
                            : div_accumulate(cw0, cvel, dxv, dzv, dyv);
      float out;
      if (MODE == 0) out = t;
      else out = MODE == 1 ? __fsub_rn(__fadd_rn(cw1, cw1), t) : q_update(a.q, i, (long long)a.ny * g.nxz, t, cw1);
      if (F16) {
        const float sc = __ldg(a.h.sn + iy);
        float hv = out / sc;
        if (fabsf(hv) > 65504.f) hv = copysignf(65504.f, hv);  // saturate; a NaN stays a NaN
        a.h.w0[i] = __float2half_rn(hv);
        amax = fabsf(out);
      } else {
        w0[i] = out;
      }
    }
    if (F16) {  // slab max of the new field (all lanes of a warp are on plane iy)
      for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
      if ((threadIdx.x & 31) == 0 && amax > 0.f) atomicMax(a.h.m0 + iy, __float_as_uint(amax));
      amax = 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 2 * R; k++) q[k] = q[k + 1];
  }
}

template <int TX, int MODE, bool F16, bool EDGE>
__global__ void __launch_bounds__(TZ *TX) div_fd8(DivArgs a, const Tile4 *__restrict__ tiles) {
  __shared__ float tpx[TX + 2 * R][TZ];
  __shared__ float tpz[TX][TZ + 2 * R];
  const Tile4 tl = tiles[blockIdx.x];
  div_tile<TX, MODE, F16, EDGE>(a, a.w1, a.w0, tl.bz, tl.bx, tl.y0, tl.y1, tpx, tpz);
}

// Many VTI / TTI shots in two persistent launches per step (gradient pass
// over every active shot's column tiles, then the divergence pass), the work
// items laid out as in iso_fd8_batch; every tile takes the PML code path;
// leapfrog update (MODE 1), FP32 state.
template <int TX, int MODEL>
__global__ void __launch_bounds__(TZ *TX) grad_fd8_batch(const AnisoBatchShot *__restrict__ shots,
                                                          const int *__restrict__ start, int nactive, int total,
                                                          int it) {
  __shared__ float tile[TX + 2 * R][TZ + 2 * R];
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    int lo = 0, hi = nactive - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(start + mid) <= w) lo = mid;
      else hi = mid - 1;
    }
    const AnisoBatchShot &S = shots[lo];
    const int l = w - __ldg(start + lo);
    const int bz = l % S.tiles_z, bx = (l / S.tiles_z) % S.tiles_x, by = l / (S.tiles_z * S.tiles_x);
    const int y0 = by * S.yseg, y1 = min(S.g.ny, y0 + S.yseg);
    grad_tile<TX, MODEL, false, true>(S.g, (it & 1) ? S.wb : S.wa, bz, bx, y0, y1, tile);
  }
}

template <int TX>
__global__ void __launch_bounds__(TZ *TX) div_fd8_batch(const AnisoBatchShot *__restrict__ shots,
                                                         const int *__restrict__ start, int nactive, int total, int it) {
  __shared__ float tpx[TX + 2 * R][TZ];
  __shared__ float tpz[TX][TZ + 2 * R];
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    int lo = 0, hi = nactive - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(start + mid) <= w) lo = mid;
      else hi = mid - 1;
    }
    const AnisoBatchShot &S = shots[lo];
    const int l = w - __ldg(start + lo);
    const int bz = l % S.tiles_z, bx = (l / S.tiles_z) % S.tiles_x, by = l / (S.tiles_z * S.tiles_x);
    const int y0 = by * S.yseg, y1 = min(S.d.ny, y0 + S.yseg);
    div_tile<TX, 1, false, true>(S.d, (it & 1) ? S.wb : S.wa, (it & 1) ? S.wa : S.wb, bz, bx, y0, y1, tpx, tpz);
  }
}

}  // namespace

static dim3 fd_grid(int nx, int ny, int nz, int tx, int yseg) {
  return dim3((nz + TZ - 1) / TZ, (nx + tx - 1) / tx, (ny + yseg - 1) / yseg);
}

template <int TX>
static void iso_launch_tx(const IsoArgs &a, int mode, int pml3d, cudaStream_t st) {
  dim3 grid = fd_grid(a.nx, a.ny, a.nz, TX, a.yseg), block(TZ, TX);
#define ISO_L(M, P) iso_fd8_step<TX, M, P><<<grid, block, 0, st>>>(a)
  if (pml3d) {
    if (mode == 0) ISO_L(0, true);
    else if (mode == 1) ISO_L(1, true);
    else ISO_L(2, true);
  } else {
    if (mode == 0) ISO_L(0, false);
    else if (mode == 1) ISO_L(1, false);
    else ISO_L(2, false);
  }
#undef ISO_L
}

void launch_iso_fd8(const IsoArgs &a, int mode, int pml3d, int tx, cudaStream_t st) {
  if (tx == 4) iso_launch_tx<4>(a, mode, pml3d, st);
  else if (tx == 16) iso_launch_tx<16>(a, mode, pml3d, st);
  else iso_launch_tx<8>(a, mode, pml3d, st);
}

template <int TX>
static void iso_batch_tx(const IsoBatchShot *shots, const int *start, int nactive, int total, int it, int pml3d,
                         int ctas, cudaStream_t st) {
  const unsigned grid = (unsigned)std::max(1, std::min(total, ctas));
  if (pml3d) iso_fd8_batch<TX, true><<<grid, dim3(TZ, TX), 0, st>>>(shots, start, nactive, total, it);
  else iso_fd8_batch<TX, false><<<grid, dim3(TZ, TX), 0, st>>>(shots, start, nactive, total, it);
}

void launch_iso_fd8_batch(const IsoBatchShot *shots, const int *start, int nactive, int total, int it, int pml3d,
                          int tx, int ctas, cudaStream_t st) {
  if (total <= 0 || nactive <= 0) return;
  if (tx == 16) iso_batch_tx<16>(shots, start, nactive, total, it, pml3d, ctas, st);
  else iso_batch_tx<8>(shots, start, nactive, total, it, pml3d, ctas, st);
}

int iso_batch_ctas_per_sm(int tx, int pml3d) {
  int n = 0;
  if (tx == 16) {
    if (pml3d) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, iso_fd8_batch<16, true>, TZ * 16, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, iso_fd8_batch<16, false>, TZ * 16, 0);
  } else {
    if (pml3d) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, iso_fd8_batch<8, true>, TZ * 8, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, iso_fd8_batch<8, false>, TZ * 8, 0);
  }
  return std::max(1, n);
}

void launch_aniso_fd8_batch(const AnisoBatchShot *shots, const int *start, int nactive, int total, int it, int model,
                            int ctas, cudaStream_t st) {
  if (total <= 0 || nactive <= 0) return;
  const unsigned grid = (unsigned)std::max(1, std::min(total, ctas));
  const dim3 block(TZ, kAnisoBatchTX);
  if (model == 3) grad_fd8_batch<kAnisoBatchTX, 3><<<grid, block, 0, st>>>(shots, start, nactive, total, it);
  else grad_fd8_batch<kAnisoBatchTX, 2><<<grid, block, 0, st>>>(shots, start, nactive, total, it);
  div_fd8_batch<kAnisoBatchTX><<<grid, block, 0, st>>>(shots, start, nactive, total, it);
}

int aniso_batch_ctas_per_sm() {
  int a = 0, b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, grad_fd8_batch<kAnisoBatchTX, 3>, TZ * kAnisoBatchTX, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, div_fd8_batch<kAnisoBatchTX>, TZ * kAnisoBatchTX, 0);
  return std::max(1, std::min(a, b));
}

template <int TX, bool F16, bool EDGE>
static void grad_launch_tx(const GradArgs &a, const Tile4 *tiles, int n, int model, cudaStream_t st) {
  const dim3 block(TZ, TX);
  if (model == 3) grad_fd8<TX, 3, F16, EDGE><<<n, block, 0, st>>>(a, tiles);
  else if (model == 2) grad_fd8<TX, 2, F16, EDGE><<<n, block, 0, st>>>(a, tiles);
  else grad_fd8<TX, 1, F16, EDGE><<<n, block, 0, st>>>(a, tiles);
}

template <bool F16, bool EDGE>
static void grad_launch(const GradArgs &a, const Tile4 *tiles, int n, int model, int tx, cudaStream_t st) {
  if (tx == 4) grad_launch_tx<4, F16, EDGE>(a, tiles, n, model, st);
  else if (tx == 16) grad_launch_tx<16, F16, EDGE>(a, tiles, n, model, st);
  else grad_launch_tx<8, F16, EDGE>(a, tiles, n, model, st);
}

void launch_grad_fd8(const GradArgs &a, const Tile4 *tiles, int ntiles, bool edge, int model, int tx,
                     cudaStream_t st, bool f16) {
  if (ntiles <= 0) return;
  if (f16) {
    if (edge) grad_launch<true, true>(a, tiles, ntiles, model, tx, st);
    else grad_launch<true, false>(a, tiles, ntiles, model, tx, st);
  } else {
    if (edge) grad_launch<false, true>(a, tiles, ntiles, model, tx, st);
    else grad_launch<false, false>(a, tiles, ntiles, model, tx, st);
  }
}

template <int TX, bool F16, bool EDGE>
static void div_launch_tx(const DivArgs &a, const Tile4 *tiles, int n, int mode, cudaStream_t st) {
  const dim3 block(TZ, TX);
  if (mode == 0) div_fd8<TX, 0, F16, EDGE><<<n, block, 0, st>>>(a, tiles);
  else if (mode == 1) div_fd8<TX, 1, F16, EDGE><<<n, block, 0, st>>>(a, tiles);
  else div_fd8<TX, 2, F16, EDGE><<<n, block, 0, st>>>(a, tiles);
}

template <bool F16, bool EDGE>
static void div_launch(const DivArgs &a, const Tile4 *tiles, int n, int mode, int tx, cudaStream_t st) {
  if (tx == 4) div_launch_tx<4, F16, EDGE>(a, tiles, n, mode, st);
  else if (tx == 16) div_launch_tx<16, F16, EDGE>(a, tiles, n, mode, st);
  else div_launch_tx<8, F16, EDGE>(a, tiles, n, mode, st);
}

void launch_div_fd8(const DivArgs &a, const Tile4 *tiles, int ntiles, bool edge, int mode, int tx, cudaStream_t st,
                    bool f16) {
  if (ntiles <= 0) return;
  if (f16) {
    if (edge) div_launch<true, true>(a, tiles, ntiles, mode, tx, st);
    else div_launch<true, false>(a, tiles, ntiles, mode, tx, st);
  } else {
    if (edge) div_launch<false, true>(a, tiles, ntiles, mode, tx, st);
    else div_launch<false, false>(a, tiles, ntiles, mode, tx, st);
  }
}

}  // namespace rtm
