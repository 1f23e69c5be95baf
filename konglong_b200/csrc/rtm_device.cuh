// rtm_device.cuh - inline device helpers shared by the kernel files: PML
// recursion, fused snapshot / imaging-condition access, the COMPRESS_16 code,
// the FP16 slab codec and the visco-acoustic update.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "rtm_internal.cuh"

namespace rtm {

struct Grid3 {
  int nx, ny, nz;
  long long nxz;
};

// One recursion round of the split-field PML on value p with memory q
// (bgprtm/PML.cpp:126-134): q' = (1-g)/(1+g) q - 2g/(1-g^2) p ; p' = q' + p/(1-g).
// The roundings are written out (fused multiply-adds in a fixed form) so that
// every kernel computing this recursion gives the same bits.
__device__ __forceinline__ void pml_round(const float *co, float &p, float *q) {
  const float qn = __fmaf_rn(co[0], *q, -__fmul_rn(co[1], p));
  *q = qn;
  p = __fmaf_rn(co[2], p, qn);
}

// Memory cell and constants of face (d, s) for grid cell (ix,iy,iz), or null
// outside the face's layers.  Indexing follows bgprtm/FdEngine.cpp:324-389.
__device__ __forceinline__ float *pml_at(const PmlDev &P, const Grid3 &g, int d, int s, int r, int c, int ix, int iy,
                                         int iz, const float *&co) {
  const PmlFace &F = P.f[d][s];
  const int w = F.w;
  if (!w) return nullptr;
  long long idx;
  int L;
  if (d == DZ) {
    if (s == SIDE_LO) {
      if (iz >= w) return nullptr;
      L = iz;
      idx = ((long long)iy * g.nx + ix) * w + iz;
    } else {
      if (iz < g.nz - w) return nullptr;
      L = g.nz - 1 - iz;
      idx = ((long long)iy * g.nx + ix) * w + (iz - (g.nz - w));
    }
  } else if (d == DX) {
    if (s == SIDE_LO) {
      if (ix >= w) return nullptr;
      L = ix;
      idx = ((long long)iy * w + ix) * g.nz + iz;
    } else {
      if (ix < g.nx - w) return nullptr;
      L = g.nx - 1 - ix;
      idx = ((long long)iy * w + ix - (g.nx - w)) * g.nz + iz;
    }
  } else {
    if (s == SIDE_LO) {
      if (iy >= w) return nullptr;
      L = iy;
      idx = ((long long)iy * g.nx + ix) * g.nz + iz;
    } else {
      if (iy < g.ny - w) return nullptr;
      L = g.ny - 1 - iy;
      idx = ((long long)(iy - (g.ny - w)) * g.nx + ix) * g.nz + iz;
    }
  }
  co = F.co + L * 6;
  return F.q[r][c] + idx;
}

// True when (ix,iy,iz) lies in any PML layer; interior cells skip the PML code.
__device__ __forceinline__ bool in_pml(const PmlDev &P, const Grid3 &g, int ix, int iy, int iz) {
  const int zl = P.f[DZ][0].w, zh = P.f[DZ][1].w, xl = P.f[DX][0].w, xh = P.f[DX][1].w, yl = P.f[DY][0].w,
            yh = P.f[DY][1].w;
  return iz < zl || iz >= g.nz - zh || ix < xl || ix >= g.nx - xh || iy < yl || iy >= g.ny - yh;
}

// Two rounds along dim d on the summed 2nd-derivative operator
// (pml2_{z,x,y}bnd, bgprtm/FdEngine.cpp:352-389).
__device__ __forceinline__ void pml2_dim(const PmlDev &P, const Grid3 &g, int d, float &p, int ix, int iy, int iz) {
#pragma unroll
  for (int s = 0; s < 2; s++) {
    const float *co;
    float *q1 = pml_at(P, g, d, s, 0, 0, ix, iy, iz, co);
    if (!q1) continue;
    const float *co2;
    float *q2 = pml_at(P, g, d, s, 1, 0, ix, iy, iz, co2);
    pml_round(co, p, q1);
    pml_round(co, p, q2);
  }
}

// One round (round r) on a first derivative along `axis`, own direction
// unscaled then the other two scaled (pml1_{z,x,y}bnd, bgprtm/FdEngine.cpp:301-350).
__device__ __forceinline__ void pml1_dim(const PmlDev &P, const Grid3 &g, int d, int c, int scaled, int r, float &p,
                                         int ix, int iy, int iz) {
#pragma unroll
  for (int s = 0; s < 2; s++) {
    const float *co;
    float *q = pml_at(P, g, d, s, r, c, ix, iy, iz, co);
    if (!q) continue;
    pml_round(co + 3 * scaled, p, q);
  }
}
__device__ __forceinline__ void pml1(const PmlDev &P, const Grid3 &g, int pml3d, int axis, int r, float &p, int ix,
                                     int iy, int iz) {
  if (axis == DZ) {
    pml1_dim(P, g, DZ, 0, 0, r, p, ix, iy, iz);
    if (pml3d) pml1_dim(P, g, DX, 1, 1, r, p, ix, iy, iz), pml1_dim(P, g, DY, 1, 1, r, p, ix, iy, iz);
  } else if (axis == DX) {
    pml1_dim(P, g, DX, 0, 0, r, p, ix, iy, iz);
    if (pml3d) pml1_dim(P, g, DZ, 1, 1, r, p, ix, iy, iz), pml1_dim(P, g, DY, 2, 1, r, p, ix, iy, iz);
  } else {
    pml1_dim(P, g, DY, 0, 0, r, p, ix, iy, iz);
    if (pml3d && g.ny > 1) pml1_dim(P, g, DZ, 2, 1, r, p, ix, iy, iz), pml1_dim(P, g, DX, 2, 1, r, p, ix, iy, iz);
  }
}

// Index of cell (ix, iy, iz) in the memory arrays of the face of dimension d
// that holds it, with its side in bit 30 (the two sides of a dimension never
// overlap), or -1 outside both; *layer = its distance from the outer edge.
// Same indexing as pml_at; every face array has fewer than 2^30 cells.
__device__ __forceinline__ int pml_face_index(const PmlDev &P, const Grid3 &g, int d, int ix, int iy, int iz,
                                              int &layer) {
  const int wl = P.f[d][SIDE_LO].w, wh = P.f[d][SIDE_HI].w;
  if (d == DZ) {
    if (iz < wl) return layer = iz, (int)(((long long)iy * g.nx + ix) * wl + iz);
    if (wh && iz >= g.nz - wh)
      return layer = g.nz - 1 - iz, (1 << 30) | (int)(((long long)iy * g.nx + ix) * wh + (iz - (g.nz - wh)));
  } else if (d == DX) {
    if (ix < wl) return layer = ix, (int)(((long long)iy * wl + ix) * g.nz + iz);
    if (wh && ix >= g.nx - wh)
      return layer = g.nx - 1 - ix, (1 << 30) | (int)(((long long)iy * wh + ix - (g.nx - wh)) * g.nz + iz);
  } else {
    if (iy < wl) return layer = iy, (int)(((long long)iy * g.nx + ix) * g.nz + iz);
    if (wh && iy >= g.ny - wh)
      return layer = g.ny - 1 - iy, (1 << 30) | (int)(((long long)(iy - (g.ny - wh)) * g.nx + ix) * g.nz + iz);
  }
  return -1;
}

// First-derivative PML round R on component AXIS of U cells at once (pml1's
// arithmetic and order per cell: own dimension unscaled, then the two cross
// dimensions scaled when pml3d).  dm[u]: bit d set when dimension d's layers
// may hold cell u (the caller knows which coordinates are fixed for it); 0
// skips the cell.  Every memory value of the U cells is loaded before the
// first recursion, so the batch costs one memory round trip instead of one
// per face and cell.
template <int AXIS, int R, int U>
__device__ __forceinline__ void pml1_batch(const PmlDev &P, const Grid3 &g, int pml3d, float (&v)[U], const int (&ix)[U],
                                           const int (&iy)[U], const int (&iz)[U], const int (&dm)[U]) {
  // dimensions in pml1's order for this component and the memory component
  // each keeps for it (bgprtm/FdEngine.cpp:301-350)
  constexpr int D1 = AXIS == DZ ? DX : DZ, D2 = AXIS == DY ? DX : DY;
  constexpr int C1 = AXIS == DY ? 2 : 1, C2 = AXIS == DZ ? 1 : 2;
  const bool cross = pml3d != 0 && (AXIS != DY || g.ny > 1);
  int enc[U][3], lay[U][3];
  float q[U][3];
#pragma unroll
  for (int u = 0; u < U; u++)
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int d = k == 0 ? AXIS : k == 1 ? D1 : D2, c = k == 0 ? 0 : k == 1 ? C1 : C2;
      enc[u][k] = ((dm[u] >> d) & 1) && (k == 0 || cross) ? pml_face_index(P, g, d, ix[u], iy[u], iz[u], lay[u][k])
                                                            : -1;
      if (enc[u][k] >= 0) q[u][k] = P.f[d][enc[u][k] >> 30].q[R][c][enc[u][k] & 0x3fffffff];
    }
#pragma unroll
  for (int u = 0; u < U; u++)
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int d = k == 0 ? AXIS : k == 1 ? D1 : D2;
      if (enc[u][k] >= 0) pml_round(P.f[d][enc[u][k] >> 30].co + lay[u][k] * 6 + (k ? 3 : 0), v[u], &q[u][k]);
    }
#pragma unroll
  for (int u = 0; u < U; u++)
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int d = k == 0 ? AXIS : k == 1 ? D1 : D2, c = k == 0 ? 0 : k == 1 ? C1 : C2;
      if (enc[u][k] >= 0) P.f[d][enc[u][k] >> 30].q[R][c][enc[u][k] & 0x3fffffff] = q[u][k];
    }
}

// Where a cell sits in the split-field PML faces: for each dimension d and
// side s (lo, hi) the layer L (-1 outside the face) and the cell's index in
// the face arrays.  Same indexing as pml_at.
struct PmlCell {
  int layer[3][2];
  long long idx[3][2];
};

// MASK: faces to consider, bit 2*d + s (the others are known not to hold the cell)
template <int MASK = 63>
__device__ __forceinline__ void pml_locate(const PmlDev &P, const Grid3 &g, int ix, int iy, int iz, PmlCell &c) {
#pragma unroll
  for (int d = 0; d < 3; d++)
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const int w = (MASK >> (2 * d + s)) & 1 ? P.f[d][s].w : 0;
      int L = -1;
      long long idx = 0;
      if (d == DZ) {
        if (s == SIDE_LO && iz < w) L = iz, idx = ((long long)iy * g.nx + ix) * w + iz;
        if (s == SIDE_HI && w && iz >= g.nz - w)
          L = g.nz - 1 - iz, idx = ((long long)iy * g.nx + ix) * w + (iz - (g.nz - w));
      } else if (d == DX) {
        if (s == SIDE_LO && ix < w) L = ix, idx = ((long long)iy * w + ix) * g.nz + iz;
        if (s == SIDE_HI && w && ix >= g.nx - w)
          L = g.nx - 1 - ix, idx = ((long long)iy * w + ix - (g.nx - w)) * g.nz + iz;
      } else {
        if (s == SIDE_LO && iy < w) L = iy, idx = ((long long)iy * g.nx + ix) * g.nz + iz;
        if (s == SIDE_HI && w && iy >= g.ny - w)
          L = g.ny - 1 - iy, idx = ((long long)(iy - (g.ny - w)) * g.nx + ix) * g.nz + iz;
      }
      c.layer[d][s] = L, c.idx[d][s] = idx;
    }
}

// Round R of the first-derivative PML on all three components of one cell
// (pml1 for axes z, x, y in turn: own dimension unscaled, then the two cross
// dimensions scaled when pml3d; each dimension lo face before hi face;
// bgprtm/FdEngine.cpp:301-350).  The work is grouped by face (d, s) behind
// one branch each, so a cell pays only for the faces that hold it; every
// memory value is loaded before the first recursion (one memory round trip),
// and the recursion order is that of pml1.
template <int R, int MASK = 63>
__device__ __forceinline__ void pml1_all(const PmlDev &P, const Grid3 &g, int pml3d, bool do_y, int ix, int iy, int iz,
                                         float &pz, float &px, float &py) {
  PmlCell c;
  pml_locate<MASK>(P, g, ix, iy, iz, c);
  // cross terms only when pml3d (for the y component only when ny > 1)
  const bool cross = pml3d != 0, ycross = pml3d != 0 && g.ny > 1;
  // q values per face and component (k: 0 z, 1 x, 2 y)
  float qz[3][2], qx[3][2], qy[3][2];
  // memory component index of component k in face dim d
  auto cz = [](int d) { return d == DZ ? 0 : 1; };           // z component: own DZ(0), cross DX(1), DY(1)
  auto cx = [](int d) { return d == DX ? 0 : d == DZ ? 1 : 2; };  // x component: own DX(0), DZ(1), DY(2)
  auto cy = [](int d) { return d == DY ? 0 : 2; };           // y component: own DY(0), DZ(2), DX(2)
#pragma unroll
  for (int d = 0; d < 3; d++)
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (c.layer[d][s] >= 0) {
        const long long i = c.idx[d][s];
        if (d == DZ || cross) qz[d][s] = P.f[d][s].q[R][cz(d)][i];
        if (d == DX || cross) qx[d][s] = P.f[d][s].q[R][cx(d)][i];
        if (do_y && (d == DY || ycross)) qy[d][s] = P.f[d][s].q[R][cy(d)][i];
      }
  auto round = [&](float &p, float &q, int d, int s, int scaled) {
    pml_round(P.f[d][s].co + c.layer[d][s] * 6 + 3 * scaled, p, &q);
  };
  // component z: DZ, then DX, DY scaled
#pragma unroll
  for (int s = 0; s < 2; s++)
    if (c.layer[DZ][s] >= 0) round(pz, qz[DZ][s], DZ, s, 0);
  if (cross) {
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (c.layer[DX][s] >= 0) round(pz, qz[DX][s], DX, s, 1);
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (c.layer[DY][s] >= 0) round(pz, qz[DY][s], DY, s, 1);
  }
  // component x: DX, then DZ, DY scaled
#pragma unroll
  for (int s = 0; s < 2; s++)
    if (c.layer[DX][s] >= 0) round(px, qx[DX][s], DX, s, 0);
  if (cross) {
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (c.layer[DZ][s] >= 0) round(px, qx[DZ][s], DZ, s, 1);
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (c.layer[DY][s] >= 0) round(px, qx[DY][s], DY, s, 1);
  }
  // component y: DY, then DZ, DX scaled
  if (do_y) {
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (c.layer[DY][s] >= 0) round(py, qy[DY][s], DY, s, 0);
    if (ycross) {
#pragma unroll
      for (int s = 0; s < 2; s++)
        if (c.layer[DZ][s] >= 0) round(py, qy[DZ][s], DZ, s, 1);
#pragma unroll
      for (int s = 0; s < 2; s++)
        if (c.layer[DX][s] >= 0) round(py, qy[DX][s], DX, s, 1);
    }
  }
#pragma unroll
  for (int d = 0; d < 3; d++)
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (c.layer[d][s] >= 0) {
        const long long i = c.idx[d][s];
        if (d == DZ || cross) P.f[d][s].q[R][cz(d)][i] = qz[d][s];
        if (d == DX || cross) P.f[d][s].q[R][cx(d)][i] = qx[d][s];
        if (do_y && (d == DY || ycross)) P.f[d][s].q[R][cy(d)][i] = qy[d][s];
      }
}

// --- FD8 two-pass pieces shared by the one-cell and the 4-cell kernels ---------
// (roundings written out so that both give the same bits)

// one tap pair of a first derivative: acc + c (a - b)
__device__ __forceinline__ float d1_acc(float acc, float c, float a, float b) {
  return __fmaf_rn(c, __fsub_rn(a, b), acc);
}

// accumulation order of KernelCPU::TTI: w0 - vel dx, then - vel dz, then - vel dy
__device__ __forceinline__ float div_accumulate(float w0, float vel, float dx, float dz, float dy) {
  float t = __fmaf_rn(-dx, vel, w0);
  t = __fmaf_rn(-dz, vel, t);
  return __fmaf_rn(-dy, vel, t);
}

// The same with a density model, in each engine's association of d vel rho:
// FdEngine_fd (d vel) rho on every axis (bgprtm/FdEngine_fd.cpp:411, 437,
// 463); FORM 0 FdEngine_cfd: (d vel) rho on x and z, d (vel rho) on y
// (bgprtm/FdEngine_cfd.cpp:42, 64-67, 91); FORM 1 FdEngine_r2c / _r2r: vel
// (rho d) on x and y (Util::transposeAndAdd, bgprtm/Util.cpp:155-175), (d vel)
// rho on z; FORM 2 the Derivative path: ((dz + dx) + dy) rho, then vel
// (getDiverge0, multiplyRho, applyVel; bgprtm/Derivative.cpp:92-112,
// bgprtm/Propagator.cpp:1722-1746).  FORM -1: the FD form.
template <int FORM>
__device__ __forceinline__ float div_accumulate_rho(float w0, float vel, float rho, float dx, float dz, float dy) {
  if (FORM == 2) return __fmaf_rn(-__fmul_rn(__fadd_rn(__fadd_rn(dz, dx), dy), rho), vel, w0);
  float t;
  if (FORM == 1) t = __fmaf_rn(-vel, __fmul_rn(rho, dx), w0);
  else t = __fmaf_rn(-__fmul_rn(dx, vel), rho, w0);
  t = __fmaf_rn(-__fmul_rn(dz, vel), rho, t);
  if (FORM == 0) return __fmaf_rn(-dy, __fmul_rn(vel, rho), t);
  if (FORM == 1) return __fmaf_rn(-vel, __fmul_rn(rho, dy), t);
  return __fmaf_rn(-__fmul_rn(dy, vel), rho, t);
}

// KernelCPU::divideRho (bgprtm/KernelCPU.cpp:340-348)
__device__ __forceinline__ void divide_rho(float rho, bool do_y, float &gx, float &gy, float &gz) {
  gx = __fdiv_rn(gx, rho);
  if (do_y) gy = __fdiv_rn(gy, rho);
  gz = __fdiv_rn(gz, rho);
}

// pseudo-acoustic scaling of the gradient (ScalarVTI / ScalarTTI,
// bgprtm/KernelCPU.cpp:176-297); m = (eps, delta, pjx, pjy)
template <int MODEL>
__device__ __forceinline__ void aniso_scale(const float4 &m, float &gx, float &gy, float &gz) {
  float e = m.x;
  const float dl = __fsub_rn(e, m.y);
  e = __fmaf_rn(2.0f, e, 1.0f);
  if (MODEL == 3) {
    const float ax = m.z, ay = m.w;
    const float az = sqrtf(__fsub_rn(1.0f, __fmaf_rn(ax, ax, __fmul_rn(ay, ay))));
    const float v2 = __fmaf_rn(gz, gz, __fmaf_rn(gy, gy, __fmul_rn(gx, gx)));
    const float vzz = __fmaf_rn(gz, az, __fmaf_rn(gy, ay, __fmul_rn(gx, ax)));
    const float vz2 = __fmul_rn(vzz, vzz);
    const float vh2 = __fsub_rn(v2, vz2);
    const float ecl = __fmaf_rn(e, vh2, vz2);
    const float parts =
        sqrtf(__fsub_rn(1.0f, __fmul_rn(__fmul_rn(8.0f, __fmul_rn(dl, __fmul_rn(vh2, vz2))),
                                        __frcp_rn(__fmaf_rn(ecl, ecl, 1e-32f)))));
    const float sc = fminf(__fmul_rn(0.5f, __fadd_rn(1.0f, parts)), 1.0f);
    const float bx = __fmul_rn(vzz, ax), by = __fmul_rn(vzz, ay), bz = __fmul_rn(vzz, az);
    gx = __fmul_rn(__fmaf_rn(__fsub_rn(gx, bx), e, bx), sc);
    gy = __fmul_rn(__fmaf_rn(__fsub_rn(gy, by), e, by), sc);
    gz = __fmul_rn(__fmaf_rn(__fsub_rn(gz, bz), e, bz), sc);
  } else {
    const float vx2 = __fmaf_rn(gy, gy, __fmul_rn(gx, gx)), vz2 = __fmul_rn(gz, gz);
    const float ecl = __fmaf_rn(e, vx2, vz2);
    const float parts =
        sqrtf(__fsub_rn(1.0f, __fmul_rn(__fmul_rn(8.0f, __fmul_rn(dl, __fmul_rn(vx2, vz2))),
                                        __frcp_rn(__fmaf_rn(ecl, ecl, 1e-32f)))));
    const float sc2 = __fmul_rn(e, fminf(__fmul_rn(0.5f, __fadd_rn(1.0f, parts)), 1.0f));
    gx = __fmul_rn(gx, sc2);
    gy = __fmul_rn(gy, sc2);
  }
}

// --- COMPRESS_16 code (bgprtm/WaveFieldCompress.cpp:107-133) ----------------
__device__ __forceinline__ uint16_t c16_encode(float v) {
  const int idat = __float_as_int(v);
  const uint16_t sgn = (uint16_t)(((unsigned)idat & 0x80000000u) >> 16);
  int e = ((idat & 0x7f800000) >> 23) - 127;
  if (e > 0) return 0x8000;
  if (e == 0) return sgn | 0x1;
  if (e > -5) return sgn | (uint16_t)((((idat & 0x7fffff) | 0x800000)) >> (9 - e));
  if (e > -21) return sgn | 0x4000 | (uint16_t)((e + 20) << 10) | (uint16_t)((idat & 0x7fffff) >> 13);
  if (e > -30) return sgn | (uint16_t)((((idat & 0x7fffff) | 0x800000)) >> (-7 - e));
  return 0;
}
// Value of the decode table entry (bgprtm/WaveFieldCompress.cpp:52-86),
// rebuilt arithmetically: every entry is an exact power-of-two multiple.
__device__ __forceinline__ float c16_table(uint16_t c) {
  const int m = c & 0x7fff;
  float v;
  if (m == 0) return (c & 0x8000) ? __int_as_float(0x7fffffff) : 0.0f;
  if (m == 1) v = 1.0f;
  else if (m < 1024) v = (float)m * 9.31322574615478515625e-10f;  // 2^-30
  else if (m < 16384) v = (float)m * 6.103515625e-05f;          // 2^-14
  else {
    const int j = (m - 16384) >> 10, i = m & 1023;
    v = __int_as_float((127 - 20 + j) << 23) * (1.0f + (float)i * 9.765625e-4f);
  }
  return (c & 0x8000) ? -v : v;
}

// FP16 with a per-y-slab scale: stored h = fp16(v * (1/s)), value = h * s
__device__ __forceinline__ float slab16_decode(__half h, float s) { return __half2float(h) * s; }
__device__ __forceinline__ __half slab16_encode(float v, float s) { return __float2half_rn(s > 0.f ? v / s : 0.f); }

// Raw decoded value of a snapshot cell (no tapers).
__device__ __forceinline__ float snap_read(const SnapDev &S, const Grid3 &g, long long i, int iy, long long inslab) {
  if (S.fmt == 0) return ((const float *)S.base)[i];
  if (S.fmt == 1) {
    const uint16_t c = ((const uint16_t *)S.base)[(long long)iy * (g.nxz + 2) + 2 + inslab];
    return S.slab[iy] * c16_table(c);
  }
  return slab16_decode(((const __half *)S.base)[i], S.slab[iy]);
}
__device__ __forceinline__ void snap_write(const SnapDev &S, const Grid3 &g, long long i, int iy, long long inslab,
                                           float v) {
  if (S.fmt == 0) {
    ((float *)S.base)[i] = v;
  } else if (S.fmt == 1) {
    const float vmax = S.slab[iy];
    uint16_t c = 0;
    if (vmax > 1e-25f) c = c16_encode(v * __frcp_rn(vmax));
    ((uint16_t *)S.base)[(long long)iy * (g.nxz + 2) + 2 + inslab] = c;
  } else {
    ((__half *)S.base)[i] = slab16_encode(v, S.slab[iy]);
  }
}

// Fused snapshot store / zero-lag imaging of the centre value u (the final
// wavefield of the previous step) at cell (ix,iy,iz).
__device__ __forceinline__ void fused_io(const FusedIo &io, const Grid3 &g, long long i, int ix, int iy, int iz,
                                         long long inslab, float u) {
  if (io.store) snap_write(io.st, g, i, iy, inslab, u);
  if (io.ic) {
    float s = snap_read(io.src, g, i, iy, inslab);
    // decode tapers (y, x, z order as bgprtm/WaveFieldCompress.cpp:189-200),
    // then the source time / depth taper (bgprtm/ImagingCondition.cpp:207-225)
    s = s * io.ey[iy];
    s = s * io.ex[ix];
    s = s * io.ez[iz];
    if (io.use_t) s = s * io.tscale;
    else s = s * io.taper_z[iz];
    // source illumination (ImagingCondition::calIllum, bgprtm/ImagingCondition.cpp:143-149)
    if (io.illum) io.illum[i] = __fmaf_rn(s, s, io.illum[i]);
    float r = u * io.ey[iy];
    r = r * io.ex[ix];
    r = r * io.ez[iz];
    // Kahan-compensated accumulation (image, comp)
    const float prod = s * r;
    const float img = io.image[i];
    const float y = prod - io.comp[i];
    const float t = img + y;
    io.comp[i] = (t - img) - y;
    io.image[i] = t;
  }
}

__device__ __forceinline__ float io4_get(const float4 &v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ void io4_set(float4 &v, int c, float x) {
  if (c == 0) v.x = x;
  else if (c == 1) v.y = x;
  else if (c == 2) v.z = x;
  else v.w = x;
}

// Fused snapshot store / imaging condition (fused_io) of the thread's 4 cells
// with one vector access per array: FP32 slots and the image / compensation
// pair as float4, FP16 slots as 8 bytes, COMPRESS_16 codes as two 4-byte
// words (a slab's codes start 4 bytes into it).  Same arithmetic per cell.
__device__ __forceinline__ void fused_io4(const FusedIo &io, const Grid3 &g, long long i0, int ix, int iy, int iz4,
                                         long long col, float4 u4) {
  const float uv[4] = {u4.x, u4.y, u4.z, u4.w};
  if (io.store) {
    const SnapDev &S = io.st;
    if (S.fmt == 0) {
      *reinterpret_cast<float4 *>((float *)S.base + i0) = u4;
    } else if (S.fmt == 1) {
      const float vmax = S.slab[iy];
      uint16_t c[4] = {0, 0, 0, 0};
      if (vmax > 1e-25f)
#pragma unroll
        for (int k = 0; k < 4; k++) c[k] = c16_encode(uv[k] * __frcp_rn(vmax));
      uint32_t *w = reinterpret_cast<uint32_t *>((uint16_t *)S.base + (long long)iy * (g.nxz + 2) + 2 + col);
      w[0] = (uint32_t)c[0] | ((uint32_t)c[1] << 16);
      w[1] = (uint32_t)c[2] | ((uint32_t)c[3] << 16);
    } else {
      const float sc = S.slab[iy];
      __half2 h[2] = {__halves2half2(slab16_encode(uv[0], sc), slab16_encode(uv[1], sc)),
                      __halves2half2(slab16_encode(uv[2], sc), slab16_encode(uv[3], sc))};
      *reinterpret_cast<uint2 *>((__half *)S.base + i0) = *reinterpret_cast<uint2 *>(h);
    }
  }
  if (io.ic) {
    const SnapDev &S = io.src;
    float sv[4];
    if (S.fmt == 0) {
      const float4 v = *reinterpret_cast<const float4 *>((const float *)S.base + i0);
      sv[0] = v.x, sv[1] = v.y, sv[2] = v.z, sv[3] = v.w;
    } else if (S.fmt == 1) {
      const uint32_t *w = reinterpret_cast<const uint32_t *>((const uint16_t *)S.base + (long long)iy * (g.nxz + 2) + 2 + col);
      const uint32_t a = w[0], b = w[1];
      const float sl = S.slab[iy];
      sv[0] = sl * c16_table((uint16_t)(a & 0xffff)), sv[1] = sl * c16_table((uint16_t)(a >> 16));
      sv[2] = sl * c16_table((uint16_t)(b & 0xffff)), sv[3] = sl * c16_table((uint16_t)(b >> 16));
    } else {
      const uint2 hv = *reinterpret_cast<const uint2 *>((const __half *)S.base + i0);
      const __half2 h0 = *reinterpret_cast<const __half2 *>(&hv.x), h1 = *reinterpret_cast<const __half2 *>(&hv.y);
      const float sl = S.slab[iy];
      sv[0] = slab16_decode(__low2half(h0), sl), sv[1] = slab16_decode(__high2half(h0), sl);
      sv[2] = slab16_decode(__low2half(h1), sl), sv[3] = slab16_decode(__high2half(h1), sl);
    }
    float4 img = *reinterpret_cast<const float4 *>(io.image + i0), cmp = *reinterpret_cast<const float4 *>(io.comp + i0);
    float4 ill = io.illum ? *reinterpret_cast<const float4 *>(io.illum + i0) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float ey = io.ey[iy], ex = io.ex[ix];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int iz = iz4 + k;
      float s = sv[k] * ey;
      s = s * ex;
      s = s * io.ez[iz];
      if (io.use_t) s = s * io.tscale;
      else s = s * io.taper_z[iz];
      io4_set(ill, k, __fmaf_rn(s, s, io4_get(ill, k)));
      float r = uv[k] * ey;
      r = r * ex;
      r = r * io.ez[iz];
      const float prod = s * r;
      const float im = io4_get(img, k);
      const float y = prod - io4_get(cmp, k);
      const float t = im + y;
      io4_set(cmp, k, (t - im) - y);
      io4_set(img, k, t);
    }
    *reinterpret_cast<float4 *>(io.comp + i0) = cmp;
    *reinterpret_cast<float4 *>(io.image + i0) = img;
    if (io.illum) *reinterpret_cast<float4 *>(io.illum + i0) = ill;
  }
}

// Visco-acoustic update (bgprtm/Propagator.cpp:1789-1816) for one cell:
// t = w0 - vel*L[w1] on entry, u = w1.
// Steps of the update with every rounding written out (fused multiply-adds
// in a fixed form), so that the one-cell and the 4-cell kernels compute
// identical bits whatever the compiler would otherwise contract:
//   v   = u (2 + iq cqsum) - t
//   v  += iq ((1 + w_l) d0_l - 2 d1_l)
//   d0' = cq_l u + w_l d0_l
__device__ __forceinline__ float q_init(float u, float iq, float cqsum, float t) {
  return __fmaf_rn(u, __fmaf_rn(iq, cqsum, 2.0f), -t);
}
__device__ __forceinline__ float q_acc(float v, float iq, float el, float d0, float d1) {
  return __fmaf_rn(iq, __fmaf_rn(__fadd_rn(1.0f, el), d0, -2.0f * d1), v);
}
__device__ __forceinline__ float q_next(float cq, float u, float el, float d0) {
  return __fmaf_rn(el, d0, __fmul_rn(cq, u));
}

// Memory variable element j of a Q half, FP32 or BF16 storage.
__device__ __forceinline__ float q_ld(const QDev &Q, const float *h, long long j) {
  return Q.bf16 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(h)[j]) : h[j];
}
__device__ __forceinline__ void q_st(const QDev &Q, float *h, long long j, float v) {
  if (Q.bf16) reinterpret_cast<__nv_bfloat16 *>(h)[j] = __float2bfloat16_rn(v);
  else h[j] = v;
}
// four consecutive elements (j a multiple of 4)
__device__ __forceinline__ float4 q_ld4(const QDev &Q, const float *h, long long j) {
  if (!Q.bf16) return *reinterpret_cast<const float4 *>(h + j);
  const uint2 r = *reinterpret_cast<const uint2 *>(reinterpret_cast<const __nv_bfloat16 *>(h) + j);
  const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&r.x));
  const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&r.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void q_st4(const QDev &Q, float *h, long long j, float4 v) {
  if (!Q.bf16) {
    *reinterpret_cast<float4 *>(h + j) = v;
    return;
  }
  const __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
  uint2 r;
  r.x = *reinterpret_cast<const unsigned *>(&a);
  r.y = *reinterpret_cast<const unsigned *>(&b);
  *reinterpret_cast<uint2 *>(reinterpret_cast<__nv_bfloat16 *>(h) + j) = r;
}

// The memory variables of up to 4 orders are loaded before any is updated, so
// a cell waits for one load round trip per 4 orders (order <= 8, QDev::cq).
__device__ __forceinline__ float q_update(const QDev &Q, long long i, long long n, float t, float u) {
  const float iq = Q.invq[i];
  float v = q_init(u, iq, Q.cqsum, t);
#pragma unroll
  for (int l0 = 0; l0 < 8; l0 += 4) {
    if (l0 >= Q.order) break;
    float d0[4], d1[4];
#pragma unroll
    for (int l = 0; l < 4; l++)
      if (l0 + l < Q.order) d0[l] = q_ld(Q, Q.d0, (long long)(l0 + l) * n + i), d1[l] = q_ld(Q, Q.d1, (long long)(l0 + l) * n + i);
#pragma unroll
    for (int l = 0; l < 4; l++)
      if (l0 + l < Q.order) {
        const float el = Q.wq[l0 + l];
        v = q_acc(v, iq, el, d0[l], d1[l]);
        q_st(Q, Q.d0, (long long)(l0 + l) * n + i, q_next(Q.cq[l0 + l], u, el, d0[l]));
      }
  }
  return v;
}

// Visco-acoustic update (q_update) of the thread's 4 cells: the memory
// variables of up to 4 orders are loaded before any is computed or written.
static __device__ __noinline__ float4 q_update4(const QDev &Q, long long i, long long n, float4 t, float4 u) {
  const float4 iq = *reinterpret_cast<const float4 *>(Q.invq + i);
  const float uv[4] = {u.x, u.y, u.z, u.w}, iv[4] = {iq.x, iq.y, iq.z, iq.w};
  float v[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
  for (int c = 0; c < 4; c++) v[c] = q_init(uv[c], iv[c], Q.cqsum, v[c]);
  for (int l0 = 0; l0 < Q.order; l0 += 4) {
    float4 d0[4], d1[4];
#pragma unroll
    for (int l = 0; l < 4; l++)
      if (l0 + l < Q.order) {
        d0[l] = q_ld4(Q, Q.d0, (long long)(l0 + l) * n + i);
        d1[l] = q_ld4(Q, Q.d1, (long long)(l0 + l) * n + i);
      }
#pragma unroll
    for (int c = 0; c < 4; c++)
#pragma unroll
      for (int l = 0; l < 4; l++)
        if (l0 + l < Q.order) {
          const float e0 = io4_get(d0[l], c), e1 = io4_get(d1[l], c);
          const float el = Q.wq[l0 + l];
          v[c] = q_acc(v[c], iv[c], el, e0, e1);
          io4_set(d0[l], c, q_next(Q.cq[l0 + l], uv[c], el, e0));
        }
#pragma unroll
    for (int l = 0; l < 4; l++)
      if (l0 + l < Q.order) q_st4(Q, Q.d0, (long long)(l0 + l) * n + i, d0[l]);
  }
  return make_float4(v[0], v[1], v[2], v[3]);
}

// four consecutive memory-variable values staged in shared memory
__device__ __forceinline__ float4 q_sm4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float4 q_sm4(const __nv_bfloat16 *p) {
  const uint2 r = *reinterpret_cast<const uint2 *>(p);
  const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&r.x));
  const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&r.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
// four consecutive memory-variable values to global memory (j a multiple of 4)
__device__ __forceinline__ void q_gst4(float *h, long long j, float4 v) { *reinterpret_cast<float4 *>(h + j) = v; }
__device__ __forceinline__ void q_gst4(__nv_bfloat16 *h, long long j, float4 v) {
  const __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
  uint2 r;
  r.x = *reinterpret_cast<const unsigned *>(&a);
  r.y = *reinterpret_cast<const unsigned *>(&b);
  *reinterpret_cast<uint2 *>(h + j) = r;
}

// q_update4 with its operands already in shared memory (staged by a TMA ring
// ahead of the step that needs them): qa / qb point at order 0 of the d0 / d1
// halves for the thread's 4 cells, order l at + l * ostride elements, iq is
// 1/Q of the cells; order <= 4.  The new d0 values go to global memory.  The
// arithmetic and its order are q_update4's, so the results are bitwise equal.
template <typename QT>
__device__ __forceinline__ float4 q_update4_ring(const QDev &Q, long long i, long long n, float4 t, float4 u,
                                                 const QT *qa, const QT *qb, int ostride, float4 iq) {
  const float uv[4] = {u.x, u.y, u.z, u.w}, iv[4] = {iq.x, iq.y, iq.z, iq.w};
  float v[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
  for (int c = 0; c < 4; c++) v[c] = q_init(uv[c], iv[c], Q.cqsum, v[c]);
  float4 d0[4], d1[4];
#pragma unroll
  for (int l = 0; l < 4; l++)
    if (l < Q.order) d0[l] = q_sm4(qa + l * ostride), d1[l] = q_sm4(qb + l * ostride);
#pragma unroll
  for (int c = 0; c < 4; c++)
#pragma unroll
    for (int l = 0; l < 4; l++)
      if (l < Q.order) {
        const float e0 = io4_get(d0[l], c), e1 = io4_get(d1[l], c);
        const float el = Q.wq[l];
        v[c] = q_acc(v[c], iv[c], el, e0, e1);
        io4_set(d0[l], c, q_next(Q.cq[l], uv[c], el, e0));
      }
  QT *gd = reinterpret_cast<QT *>(Q.d0);
#pragma unroll
  for (int l = 0; l < 4; l++)
    if (l < Q.order) q_gst4(gd, (long long)l * n + i, d0[l]);
  return make_float4(v[0], v[1], v[2], v[3]);
}

}  // namespace rtm
