// kernels_iso4.cu - ISO FD8 time step with register blocking along z.
//
// KernelCPU::ISO + FdEngine_fd::laplacian_irreg + pml2_bnd (bgprtm/KernelCPU.cpp:125-140,
// bgprtm/FdEngine_fd.cpp:204-325) fused with update2nd (bgprtm/Propagator.cpp:1767-1818) and
// the snapshot store / imaging condition of the previous step, as iso_fd8_step, with the same
// arithmetic in the same order (bitwise-equal results).  Each thread owns 4 consecutive z
// cells (one float4): every global and shared access is 128 bits wide.  A CTA is 8 x TX
// threads = a 32 (z) x TX (x) column tile marching a y segment:
//   - the thread's +-4 y neighbours live in a register queue of 10 float4 (the 10th holds the
//     plane loaded one step ahead); the y loop is unrolled by 10 so the queue slot of every
//     plane is a compile-time index (no moves);
//   - the centre plane and its 4-cell x / z halo sit in a double-buffered shared tile
//     (one barrier per plane); halos and the next plane's w0 / vel are fetched a plane ahead;
//   - the PML recursion and the Q update are out-of-line calls that load every memory value
//     of the thread's 4 cells before writing any; the snapshot / imaging terms are vector
//     accesses of the 4 cells.
// Requires nz % 4 == 0 (16-byte rows).
#include <type_traits>

#include "kernel_api.h"
#include "rtm_device.cuh"
#include "tma.cuh"

namespace rtm {
namespace {

constexpr int R4 = 4;  // stencil radius

// PML rounds of one cell and the Laplacian sum (iso_fd8_step's order)
template <bool PML3D>
__device__ __noinline__ float iso4_pml_cell(const PmlDev &P, Grid3 g, float lz, float lx, float ly, bool do_y, int ix,
                                            int iy, int iz) {
  if (PML3D) {
    float v = lz + lx + ly;
    pml2_dim(P, g, DZ, v, ix, iy, iz);
    pml2_dim(P, g, DX, v, ix, iy, iz);
    pml2_dim(P, g, DY, v, ix, iy, iz);
    return v;
  }
  pml2_dim(P, g, DZ, lz, ix, iy, iz);
  pml2_dim(P, g, DX, lx, ix, iy, iz);
  if (do_y) pml2_dim(P, g, DY, ly, ix, iy, iz);
  return lz + lx + ly;
}

__device__ __forceinline__ float comp(const float4 &v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ void setc(float4 &v, int c, float x) {
  if (c == 0) v.x = x;
  else if (c == 1) v.y = x;
  else if (c == 2) v.z = x;
  else v.w = x;
}

// The split-field PML memory of the face of dimension d that covers the
// thread's 4 z cells (null when none does) and the layer of its first cell;
// every face array keeps z fastest, so the 4 cells are one aligned float4.
// Requires the z faces to be a multiple of 4 cells wide.
struct Face4 {
  float *q1, *q2;
  const float *co;
  int L;
};

__device__ __forceinline__ Face4 face4(const PmlDev &P, const Grid3 &g, int d, int ix, int iy, int iz4) {
  Face4 f{nullptr, nullptr, nullptr, 0};
  long long idx = 0;
  int s = -1;
  if (d == DZ) {
    const int wl = P.f[DZ][0].w, wh = P.f[DZ][1].w;
    if (iz4 < wl) s = 0, f.L = iz4, idx = ((long long)iy * g.nx + ix) * wl + iz4;
    else if (iz4 >= g.nz - wh) s = 1, f.L = g.nz - 1 - iz4, idx = ((long long)iy * g.nx + ix) * wh + iz4 - (g.nz - wh);
  } else if (d == DX) {
    const int wl = P.f[DX][0].w, wh = P.f[DX][1].w;
    if (ix < wl) s = 0, f.L = ix, idx = ((long long)iy * wl + ix) * g.nz + iz4;
    else if (ix >= g.nx - wh) s = 1, f.L = g.nx - 1 - ix, idx = ((long long)iy * wh + ix - (g.nx - wh)) * g.nz + iz4;
  } else {
    const int wl = P.f[DY][0].w, wh = P.f[DY][1].w;
    if (iy < wl) s = 0, f.L = iy, idx = ((long long)iy * g.nx + ix) * g.nz + iz4;
    else if (iy >= g.ny - wh) s = 1, f.L = g.ny - 1 - iy, idx = ((long long)(iy - (g.ny - wh)) * g.nx + ix) * g.nz + iz4;
  }
  if (s < 0) return f;
  const PmlFace &F = P.f[d][s];
  f.q1 = F.q[0][0] + idx, f.q2 = F.q[1][0] + idx, f.co = F.co;
  return f;
}

// Two PML rounds (pml2_dim) of the 4 cells on values p with the face memory
// m1 / m2; z faces have one layer per cell (layer L, L+1, ... on the low side,
// L, L-1, ... on the high side), x / y faces one layer for all 4.
__device__ __forceinline__ void rounds4(const Face4 &f, int d, float4 &p, float4 &m1, float4 &m2, int dl) {
  float pv[4] = {p.x, p.y, p.z, p.w}, a[4] = {m1.x, m1.y, m1.z, m1.w}, b[4] = {m2.x, m2.y, m2.z, m2.w};
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const float *co = f.co + (f.L + (d == DZ ? c * dl : 0)) * 6;
    pml_round(co, pv[c], &a[c]);
    pml_round(co, pv[c], &b[c]);
  }
  p = make_float4(pv[0], pv[1], pv[2], pv[3]);
  m1 = make_float4(a[0], a[1], a[2], a[3]);
  m2 = make_float4(b[0], b[1], b[2], b[3]);
}

// PML of the thread's 4 cells (all in some face: x or y edge, or a z face of
// a width that is a multiple of 4) and the Laplacian sums, in pml2_dim's
// order per cell.  Every memory value is loaded before any is written, so a
// step waits for one load round trip rather than one per round and cell.
template <bool PML3D>
__device__ __noinline__ float4 iso4_pml4(const PmlDev &P, Grid3 g, float4 lz, float4 lx, float4 ly, bool do_y, int ix,
                                         int iy, int iz4) {
  const Face4 fz = face4(P, g, DZ, ix, iy, iz4), fx = face4(P, g, DX, ix, iy, iz4);
  const Face4 fy = (PML3D || do_y) ? face4(P, g, DY, ix, iy, iz4) : Face4{nullptr, nullptr, nullptr, 0};
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 z1 = fz.q1 ? *reinterpret_cast<float4 *>(fz.q1) : z4, z2 = fz.q2 ? *reinterpret_cast<float4 *>(fz.q2) : z4;
  float4 x1 = fx.q1 ? *reinterpret_cast<float4 *>(fx.q1) : z4, x2 = fx.q2 ? *reinterpret_cast<float4 *>(fx.q2) : z4;
  float4 y1 = fy.q1 ? *reinterpret_cast<float4 *>(fy.q1) : z4, y2 = fy.q2 ? *reinterpret_cast<float4 *>(fy.q2) : z4;
  const int dl = fz.q1 && iz4 >= P.f[DZ][0].w ? -1 : 1;  // layer step along z: down on the high face
  float4 v;
  if (PML3D) {
    v = make_float4(lz.x + lx.x + ly.x, lz.y + lx.y + ly.y, lz.z + lx.z + ly.z, lz.w + lx.w + ly.w);
    if (fz.q1) rounds4(fz, DZ, v, z1, z2, dl);
    if (fx.q1) rounds4(fx, DX, v, x1, x2, 0);
    if (fy.q1) rounds4(fy, DY, v, y1, y2, 0);
  } else {
    if (fz.q1) rounds4(fz, DZ, lz, z1, z2, dl);
    if (fx.q1) rounds4(fx, DX, lx, x1, x2, 0);
    if (fy.q1) rounds4(fy, DY, ly, y1, y2, 0);
    v = make_float4(lz.x + lx.x + ly.x, lz.y + lx.y + ly.y, lz.z + lx.z + ly.z, lz.w + lx.w + ly.w);
  }
  if (fz.q1) *reinterpret_cast<float4 *>(fz.q1) = z1, *reinterpret_cast<float4 *>(fz.q2) = z2;
  if (fx.q1) *reinterpret_cast<float4 *>(fx.q1) = x1, *reinterpret_cast<float4 *>(fx.q2) = x2;
  if (fy.q1) *reinterpret_cast<float4 *>(fy.q1) = y1, *reinterpret_cast<float4 *>(fy.q2) = y2;
  return v;
}


template <int TX, int MODE, bool PML3D>
__global__ void __launch_bounds__(8 * TX) iso_fd8_v4(const __grid_constant__ IsoArgs a) {
  __shared__ float4 tile[2][TX + 2 * R4][10];  // [buffer][x + halo][z float4 + one halo float4 each side]
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const Grid3 g{nx, ny, nz, (long long)nx * nz};
  const int tzq = threadIdx.x, tx = threadIdx.y;
  const int z0 = blockIdx.x * 32, iz4 = z0 + 4 * tzq;
  const int ix = blockIdx.y * TX + tx;
  const int y0 = blockIdx.z * a.yseg, y1 = min(ny, y0 + a.yseg);
  const bool act = iz4 < nz && ix < nx;
  const long long col = (long long)ix * nz + iz4;
  const bool do_y = ny > 2;
  float c2x[R4 + 1], c2y[R4 + 1], c2z[R4 + 1];
#pragma unroll
  for (int m = 0; m <= R4; m++) c2x[m] = a.c2x[m], c2y[m] = a.c2y[m], c2z[m] = a.c2z[m];
  const int zl = a.pml.f[DZ][0].w, zh = a.pml.f[DZ][1].w, xl = a.pml.f[DX][0].w, xh = a.pml.f[DX][1].w,
            yl = a.pml.f[DY][0].w, yh = a.pml.f[DY][1].w;
  const bool x_edge = ix < xl || ix >= nx - xh;
  const bool z4ok = zl % 4 == 0 && zh % 4 == 0;  // z faces hold whole float4s
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 *__restrict__ w1 = reinterpret_cast<const float4 *>(a.w1);
  const float4 *__restrict__ vel = reinterpret_cast<const float4 *>(a.vel);
  float4 *__restrict__ w0 = reinterpret_cast<float4 *>(a.w0);
  const long long nxz4 = g.nxz / 4, col4 = col / 4;
  auto ld1 = [&](int y) -> float4 { return (act && y >= 0 && y < ny) ? __ldg(w1 + y * nxz4 + col4) : zero4; };
  // halo float4s of plane y: x side (tx < 4: ix - 4; tx >= TX - 4: ix + 4), z side
  // (tzq == 0: z0 - 4; tzq == 7: z0 + 32)
  const bool hx_lo = tx < R4, hx_hi = tx >= TX - R4, hz_lo = tzq == 0, hz_hi = tzq == 7;
  auto ld_hx = [&](int y) -> float4 {
    if (y < 0 || y >= ny || iz4 >= nz) return zero4;
    const int xx = hx_lo ? ix - R4 : ix + R4;
    if ((!hx_lo && !hx_hi) || xx < 0 || xx >= nx) return zero4;
    return __ldg(w1 + y * nxz4 + ((long long)xx * nz + iz4) / 4);
  };
  auto ld_hz = [&](int y) -> float4 {
    if (y < 0 || y >= ny || ix >= nx) return zero4;
    const int zz = hz_lo ? z0 - 4 : z0 + 32;
    if ((!hz_lo && !hz_hi) || zz < 0 || zz >= nz) return zero4;
    return __ldg(w1 + y * nxz4 + ((long long)ix * nz + zz) / 4);
  };

  constexpr int NQ = 2 * R4 + 2;
  float4 q[NQ];
#pragma unroll
  for (int k = 0; k < NQ - 1; k++) q[k] = ld1(y0 - R4 + k);
  float4 hx = ld_hx(y0), hz = ld_hz(y0);
  float4 nw0 = act ? w0[y0 * nxz4 + col4] : zero4;
  float4 nvel = act ? __ldg(vel + y0 * nxz4 + col4) : zero4;

  auto step = [&](auto kk, int iy) {
    constexpr int k = decltype(kk)::value;
    auto slot = [](int d) { return (k + R4 + d + NQ) % NQ; };  // queue slot of plane iy + d
    if (iy + 1 < y1) q[slot(R4 + 1)] = ld1(iy + R4 + 1);
    const int b = (iy - y0) & 1;
    tile[b][tx + R4][tzq + 1] = q[slot(0)];
    if (hx_lo) tile[b][tx][tzq + 1] = hx;
    if (hx_hi) tile[b][tx + 2 * R4][tzq + 1] = hx;
    if (hz_lo) tile[b][tx + R4][0] = hz;
    if (hz_hi) tile[b][tx + R4][9] = hz;
    if (iy + 1 < y1) hx = ld_hx(iy + 1), hz = ld_hz(iy + 1);
    const float4 cw0 = nw0, cvel = nvel;
    const long long plane4 = iy * nxz4;
    if (act && iy + 1 < y1) {
      nw0 = w0[plane4 + nxz4 + col4];
      nvel = __ldg(vel + plane4 + nxz4 + col4);
    }
    __syncthreads();
    if (act) {
      const float4 zL = tile[b][tx + R4][tzq], zR = tile[b][tx + R4][tzq + 2];
      const float4 u4 = q[slot(0)];
      float zw[12];
      zw[0] = zL.x, zw[1] = zL.y, zw[2] = zL.z, zw[3] = zL.w;
      zw[4] = u4.x, zw[5] = u4.y, zw[6] = u4.z, zw[7] = u4.w;
      zw[8] = zR.x, zw[9] = zR.y, zw[10] = zR.z, zw[11] = zR.w;
      float4 xm[R4], xp[R4];
#pragma unroll
      for (int m = 1; m <= R4; m++) xm[m - 1] = tile[b][tx + R4 - m][tzq + 1], xp[m - 1] = tile[b][tx + R4 + m][tzq + 1];
      const bool y_edge = iy < yl || iy >= ny - yh;
      float lzv[4], lxv[4], lyv[4];
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const float u = zw[4 + c];
        float lz = c2z[0] * u, lx = c2x[0] * u, ly = 0.0f;
#pragma unroll
        for (int m = 1; m <= R4; m++) {
          lz += c2z[m] * (zw[4 + c - m] + zw[4 + c + m]);
          lx += c2x[m] * (comp(xm[m - 1], c) + comp(xp[m - 1], c));
        }
        if (do_y) {
          ly = c2y[0] * u;
#pragma unroll
          for (int m = 1; m <= R4; m++) ly += c2y[m] * (comp(q[slot(-m)], c) + comp(q[slot(m)], c));
        }
        lzv[c] = lz, lxv[c] = lx, lyv[c] = ly;
      }
      float v[4];
      if (x_edge || y_edge || iz4 < zl || iz4 + 3 >= nz - zh) {
        if (z4ok) {
          const float4 r = iso4_pml4<PML3D>(a.pml, g, make_float4(lzv[0], lzv[1], lzv[2], lzv[3]),
                                            make_float4(lxv[0], lxv[1], lxv[2], lxv[3]),
                                            make_float4(lyv[0], lyv[1], lyv[2], lyv[3]), do_y, ix, iy, iz4);
          v[0] = r.x, v[1] = r.y, v[2] = r.z, v[3] = r.w;
        } else {
#pragma unroll
          for (int c = 0; c < 4; c++) {
            const int iz = iz4 + c;
            if (x_edge || y_edge || iz < zl || iz >= nz - zh)
              v[c] = iso4_pml_cell<PML3D>(a.pml, g, lzv[c], lxv[c], lyv[c], do_y, ix, iy, iz);
            else v[c] = lzv[c] + lxv[c] + lyv[c];
          }
        }
      } else {
#pragma unroll
        for (int c = 0; c < 4; c++) v[c] = lzv[c] + lxv[c] + lyv[c];
      }
      const long long i0 = (long long)iy * g.nxz + col;
      if (a.io.store | a.io.ic) fused_io4(a.io, g, i0, ix, iy, iz4, col, u4);
      float4 t4, out4;
#pragma unroll
      for (int c = 0; c < 4; c++) setc(t4, c, comp(cw0, c) - v[c] * comp(cvel, c));
      if (MODE == 0) out4 = t4;  // KernelCPU seam: w0 -= vel * L[w1]
      else if (MODE == 1)        // + update2nd (leapfrog)
        out4 = make_float4((u4.x + u4.x) - t4.x, (u4.y + u4.y) - t4.y, (u4.z + u4.z) - t4.z, (u4.w + u4.w) - t4.w);
      else out4 = q_update4(a.q, i0, (long long)ny * g.nxz, t4, u4);  // + Q
      w0[plane4 + col4] = out4;
    }
  };
  for (int r0 = y0; r0 < y1; r0 += NQ) {
#define ISO4_STEP(K) \
  if (r0 + K < y1) step(std::integral_constant<int, K>{}, r0 + K)
    ISO4_STEP(0);
    ISO4_STEP(1);
    ISO4_STEP(2);
    ISO4_STEP(3);
    ISO4_STEP(4);
    ISO4_STEP(5);
    ISO4_STEP(6);
    ISO4_STEP(7);
    ISO4_STEP(8);
    ISO4_STEP(9);
#undef ISO4_STEP
  }
}

template <int TX, bool PML3D>
void iso4_launch(const IsoArgs &a, int mode, cudaStream_t st) {
  const dim3 grid((a.nz + 31) / 32, (a.nx + TX - 1) / TX, (a.ny + a.yseg - 1) / a.yseg), block(8, TX);
  if (mode == 0) iso_fd8_v4<TX, 0, PML3D><<<grid, block, 0, st>>>(a);
  else if (mode == 1) iso_fd8_v4<TX, 1, PML3D><<<grid, block, 0, st>>>(a);
  else iso_fd8_v4<TX, 2, PML3D><<<grid, block, 0, st>>>(a);
}

// ---- TMA rings ---------------------------------------------------------------
// The same step with the streamed inputs in shared-memory rings filled by TMA:
// ring A holds w1 plane tiles with their 4-cell x / z halo (40 x (TX+8)
// floats), ring B the w0 and (v dt)^2 tiles; one producer thread issues plane
// iy+4+P of ring A and plane iy+P of ring B at step iy, so every operand is
// resident P planes before it is needed and no register holds a load in
// flight.  The +-4 y neighbours stay in a register queue fed from ring A (the
// own column of plane iy+4).  The memory of the PML faces, the Q variables and
// the imaging operands of plane iy+2 are prefetched into L1 at step iy.
// Out-of-grid parts of a box are zero-filled by the TMA unit (the stencil's
// truncation at the grid edge); planes beyond the grid are zeroed here.
template <int TX, int P>
struct __align__(128) Iso4Smem {
  static constexpr int HX = TX + 2 * R4;
  // the producer refills a stage at the start of a step, after the barrier that
  // ends the previous one: ring A holds planes iy .. iy+4+P, ring B iy .. iy+P
  static constexpr int SA = 5 + P;
  static constexpr int SB = P + 1;
  float4 a[SA][HX][10];
  float4 w0[SB][TX][8];
  float4 vel[SB][TX][8];
  uint64_t bar_a[SA];
  uint64_t bar_b[SB];
};

__device__ __forceinline__ void prefetch_l1(const void *p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(__cvta_generic_to_global(p)));
}

// L1 prefetch of the per-cell operands besides the stencil input that the
// thread's 4 cells of plane iy read: PML face memory, Q variables, imaging
// condition (image, compensation, source snapshot)
template <int MODE>
__device__ __forceinline__ void iso4_prefetch(const IsoArgs &a, const Grid3 &g, bool pml, int ix, int iy, int iz4,
                                              long long col) {
  if (pml)
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const Face4 f = face4(a.pml, g, d, ix, iy, iz4);
      if (f.q1) prefetch_l1(f.q1), prefetch_l1(f.q2);
    }
  const long long i = (long long)iy * g.nxz + col;
  if (MODE == 2) {
    const long long n = (long long)g.ny * g.nxz;
    prefetch_l1(a.q.invq + i);
    const long long es = a.q.bf16 ? 2 : 4;  // bytes per memory variable
    for (int l = 0; l < a.q.order; l++)
      prefetch_l1((const char *)a.q.d0 + (l * n + i) * es), prefetch_l1((const char *)a.q.d1 + (l * n + i) * es);
  }
  if (a.io.ic) {
    prefetch_l1(a.io.image + i), prefetch_l1(a.io.comp + i);
    const SnapDev &S = a.io.src;
    if (S.fmt == 0) prefetch_l1((const float *)S.base + i);
    else if (S.fmt == 1) prefetch_l1((const uint16_t *)S.base + (long long)iy * (g.nxz + 2) + 2 + col);
    else prefetch_l1((const __half *)S.base + i);
  }
}

// PML tiles without the Q update: at most 128 registers per thread (512 threads per SM)
template <int TX, int P, int MODE, bool PML3D, bool EDGE>
__global__ void __launch_bounds__(8 * TX, EDGE && MODE != 2 ? 512 / (8 * TX) : 0) iso_fd8_tma4(const __grid_constant__ IsoArgs a,
                                                       const Tile4 *__restrict__ tiles,
                                                       const __grid_constant__ CUtensorMap map_w1,
                                                       const __grid_constant__ CUtensorMap map_w0,
                                                       const __grid_constant__ CUtensorMap map_vel, int *err) {
  using S = Iso4Smem<TX, P>;
  constexpr int SA = S::SA, SB = S::SB, HX = S::HX;
  constexpr uint32_t BYTES_A = HX * 160, BYTES_B = 2 * TX * 128;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S &s = *reinterpret_cast<S *>(smem_raw);
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const Grid3 g{nx, ny, nz, (long long)nx * nz};
  const int tzq = threadIdx.x, tx = threadIdx.y;
  const Tile4 tile = tiles[blockIdx.x];
  const int iz0 = tile.bz * 32, ix0 = tile.bx * TX;
  const int iz4 = iz0 + 4 * tzq, ix = ix0 + tx;
  const int y0 = tile.y0, y1 = tile.y1;
  const bool act = iz4 < nz && ix < nx;
  const bool producer = tzq == 0 && tx == 0;
  const long long col = (long long)ix * nz + iz4;
  const bool do_y = ny > 2;
  const int zl = a.pml.f[DZ][0].w, zh = a.pml.f[DZ][1].w, xl = a.pml.f[DX][0].w, xh = a.pml.f[DX][1].w,
            yl = a.pml.f[DY][0].w, yh = a.pml.f[DY][1].w;
  // interior tiles hold no PML cell (the tile table guarantees it)
  const bool x_edge = EDGE && (ix < xl || ix >= nx - xh);
  const bool z_edge = EDGE && (iz4 < zl || iz4 + 3 >= nz - zh);
  const bool z4ok = zl % 4 == 0 && zh % 4 == 0;
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  auto y_edge_at = [&](int y) { return EDGE && (y < yl || y >= ny - yh); };
  // PML tiles with z faces a multiple of 4 cells wide: the x and z faces of
  // the thread's 4 cells are fixed over the tile's planes; their round-0 /
  // round-1 memory (one float4 per array, z fastest) advances by a constant
  // stride per plane and their recursion constants stay in registers
  const bool vpml = EDGE && z4ok;
  float *qx1 = nullptr, *qx2 = nullptr, *qz1 = nullptr, *qz2 = nullptr;
  long long stx = 0, stz = 0;
  float cx[3] = {0.f, 0.f, 0.f}, cz[4][3] = {};
  if (vpml && act && x_edge) {
    const int sd = ix < xl ? 0 : 1;
    const PmlFace &F = a.pml.f[DX][sd];
    const int w = F.w, L = sd ? nx - 1 - ix : ix;
    const long long idx = ((long long)y0 * w + (sd ? ix - (nx - w) : ix)) * nz + iz4;
    qx1 = F.q[0][0] + idx, qx2 = F.q[1][0] + idx, stx = (long long)w * nz;
#pragma unroll
    for (int k = 0; k < 3; k++) cx[k] = F.co[L * 6 + k];
  }
  if (vpml && act && z_edge) {
    const int sd = iz4 < zl ? 0 : 1;
    const PmlFace &F = a.pml.f[DZ][sd];
    const int w = F.w;
    const long long idx = ((long long)y0 * nx + ix) * w + (sd ? iz4 - (nz - w) : iz4);
    qz1 = F.q[0][0] + idx, qz2 = F.q[1][0] + idx, stz = (long long)nx * w;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int L = sd ? nz - 1 - (iz4 + c) : iz4 + c;
#pragma unroll
      for (int k = 0; k < 3; k++) cz[c][k] = F.co[L * 6 + k];
    }
  }
  // the y face of plane y (memory of the thread's cells, recursion constants)
  auto yface = [&](int y, float *&q1, float *&q2, const float *&co) {
    const int sd = y < yl ? 0 : 1;
    const PmlFace &F = a.pml.f[DY][sd];
    const long long idx = ((long long)(sd ? y - (ny - F.w) : y) * nx + ix) * nz + iz4;
    q1 = F.q[0][0] + idx, q2 = F.q[1][0] + idx, co = F.co + (sd ? ny - 1 - y : y) * 6;
  };
  // L1 prefetch of the face memory of plane y, k planes beyond the one the
  // x / z pointers are at
  auto pml_prefetch = [&](int y, int k) {
    if (qx1) prefetch_l1(qx1 + k * stx), prefetch_l1(qx2 + k * stx);
    if (qz1) prefetch_l1(qz1 + k * stz), prefetch_l1(qz2 + k * stz);
    if ((PML3D || do_y) && y_edge_at(y)) {
      float *q1, *q2;
      const float *co;
      yface(y, q1, q2, co);
      prefetch_l1(q1), prefetch_l1(q2);
    }
  };

  // plane p (y0 <= p) lives in stage (p - y0) % S of its ring, phase ((p - y0) / S) & 1
  auto issue_a = [&](int p) {
    const int st = (p - y0) % SA;
    if (p >= ny) {  // beyond the grid: zeros written here, no copy
      for (int k = 0; k < HX * 10; k++) (&s.a[st][0][0])[k] = zero4;
      mbar_arrive(&s.bar_a[st]);
      return;
    }
    mbar_expect_tx(&s.bar_a[st], BYTES_A);
    tma_load_3d(&s.a[st][0][0], &map_w1, &s.bar_a[st], iz0 - R4, ix0 - R4, p);
  };
  auto issue_b = [&](int p) {
    const int st = (p - y0) % SB;
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
  int last_a = y0 - 1, last_b = y0 - 1;  // last planes the producer issued
  if (producer) {
    for (int p = y0; p < min(y0 + R4 + P, y1 + R4); p++) issue_a(p), last_a = p;
    for (int p = y0; p < min(y0 + P, y1); p++) issue_b(p), last_b = p;
  }
  // the queue's first 8 planes (y0-4 .. y0+3) of the own column from global memory
  const float4 *__restrict__ w1g = reinterpret_cast<const float4 *>(a.w1);
  const long long nxz4 = g.nxz / 4, col4 = col / 4;
  float4 q[2 * R4 + 1];
#pragma unroll
  for (int k = 0; k < 2 * R4; k++) {
    const int y = y0 - R4 + k;
    q[k] = act && y >= 0 && y < ny ? __ldg(w1g + y * nxz4 + col4) : zero4;
  }
  if (act)
    for (int y = y0; y < min(y0 + 2, y1); y++) {
      iso4_prefetch<MODE>(a, g, !vpml && (x_edge || z_edge || y_edge_at(y)), ix, y, iz4, col);
      if (vpml) pml_prefetch(y, y - y0);
    }
  bool ok = true;
#pragma unroll 1
  for (int iy = y0; iy < y1; iy++) {
    if (producer && ok) {  // after a failed wait nothing more is issued
      if (iy + R4 + P < y1 + R4) issue_a(iy + R4 + P), last_a = iy + R4 + P;
      if (iy + P < y1) issue_b(iy + P), last_b = iy + P;
    }
    if (act && iy + 2 < y1) {
      iso4_prefetch<MODE>(a, g, !vpml && (x_edge || z_edge || y_edge_at(iy + 2)), ix, iy + 2, iz4, col);
      if (vpml) pml_prefetch(iy + 2, 2);
    }
    // PML face memory of this plane, loaded before the waits and the stencil
    // so that its latency overlaps them (PML tiles only)
    const bool yf = (PML3D || do_y) && y_edge_at(iy);
    float4 z1, z2, x1, x2, y1, y2;
    float *qy1 = nullptr, *qy2 = nullptr;
    float cy[3] = {0.f, 0.f, 0.f};
    if constexpr (EDGE) {
      if (vpml && act) {
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        z1 = z2 = x1 = x2 = y1 = y2 = z4;
        if (qz1) z1 = *reinterpret_cast<const float4 *>(qz1), z2 = *reinterpret_cast<const float4 *>(qz2);
        if (qx1) x1 = *reinterpret_cast<const float4 *>(qx1), x2 = *reinterpret_cast<const float4 *>(qx2);
        if (yf) {
          const float *cyp;
          yface(iy, qy1, qy2, cyp);
          y1 = *reinterpret_cast<const float4 *>(qy1), y2 = *reinterpret_cast<const float4 *>(qy2);
          cy[0] = cyp[0], cy[1] = cyp[1], cy[2] = cyp[2];
        }
      }
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
      float lzv[4], lxv[4], lyv[4];
#pragma unroll
      for (int c = 0; c < 4; c++) lzv[c] = a.c2z[0] * zw[4 + c], lxv[c] = a.c2x[0] * zw[4 + c];
#pragma unroll
      for (int m = 1; m <= R4; m++) {
        const float4 xm = s.a[sa0][tx + R4 - m][tzq + 1], xp = s.a[sa0][tx + R4 + m][tzq + 1];
#pragma unroll
        for (int c = 0; c < 4; c++) {
          lzv[c] += a.c2z[m] * (zw[4 + c - m] + zw[4 + c + m]);
          lxv[c] += a.c2x[m] * (comp(xm, c) + comp(xp, c));
        }
      }
#pragma unroll
      for (int c = 0; c < 4; c++) {
        float ly = 0.0f;
        if (do_y) {
          ly = a.c2y[0] * zw[4 + c];
#pragma unroll
          for (int m = 1; m <= R4; m++) ly += a.c2y[m] * (comp(q[R4 - m], c) + comp(q[R4 + m], c));
        }
        lyv[c] = ly;
      }
      float v[4];
      const bool y_edge = y_edge_at(iy);
      bool pml_done = false;
      if constexpr (EDGE) {
        if (vpml && (qx1 || qz1 || yf)) {
          // pml2_dim's rounds per cell in the order z, x, y
          pml_done = true;
#pragma unroll
          for (int c = 0; c < 4; c++) {
            float pz = PML3D ? lzv[c] + lxv[c] + lyv[c] : lzv[c], px = lxv[c], py = lyv[c];
            float m;
            if (qz1) {
              m = comp(z1, c), pml_round(cz[c], pz, &m), setc(z1, c, m);
              m = comp(z2, c), pml_round(cz[c], pz, &m), setc(z2, c, m);
            }
            float &pxr = PML3D ? pz : px;
            if (qx1) {
              m = comp(x1, c), pml_round(cx, pxr, &m), setc(x1, c, m);
              m = comp(x2, c), pml_round(cx, pxr, &m), setc(x2, c, m);
            }
            float &pyr = PML3D ? pz : py;
            if (yf) {
              m = comp(y1, c), pml_round(cy, pyr, &m), setc(y1, c, m);
              m = comp(y2, c), pml_round(cy, pyr, &m), setc(y2, c, m);
            }
            v[c] = PML3D ? pz : pz + px + py;
          }
          if (qz1) *reinterpret_cast<float4 *>(qz1) = z1, *reinterpret_cast<float4 *>(qz2) = z2;
          if (qx1) *reinterpret_cast<float4 *>(qx1) = x1, *reinterpret_cast<float4 *>(qx2) = x2;
          if (yf) *reinterpret_cast<float4 *>(qy1) = y1, *reinterpret_cast<float4 *>(qy2) = y2;
        } else if (!z4ok && (x_edge || y_edge || z_edge)) {
          pml_done = true;
#pragma unroll
          for (int c = 0; c < 4; c++) {
            const int iz = iz4 + c;
            if (x_edge || y_edge || iz < zl || iz >= nz - zh)
              v[c] = iso4_pml_cell<PML3D>(a.pml, g, lzv[c], lxv[c], lyv[c], do_y, ix, iy, iz);
            else v[c] = lzv[c] + lxv[c] + lyv[c];
          }
        }
      }
      if (!pml_done)
#pragma unroll
        for (int c = 0; c < 4; c++) v[c] = lzv[c] + lxv[c] + lyv[c];
      const long long i0 = (long long)iy * g.nxz + col;
      if (a.io.store | a.io.ic) fused_io4(a.io, g, i0, ix, iy, iz4, col, u4);
      const float4 cw0 = s.w0[sb][tx][tzq], cvel = s.vel[sb][tx][tzq];
      float4 t4, out4;
#pragma unroll
      for (int c = 0; c < 4; c++) setc(t4, c, comp(cw0, c) - v[c] * comp(cvel, c));
      if (MODE == 0) out4 = t4;
      else if (MODE == 1)
        out4 = make_float4((u4.x + u4.x) - t4.x, (u4.y + u4.y) - t4.y, (u4.z + u4.z) - t4.z, (u4.w + u4.w) - t4.w);
      else out4 = q_update4(a.q, i0, (long long)ny * g.nxz, t4, u4);
      reinterpret_cast<float4 *>(a.w0)[i0 / 4] = out4;
    }
    if (qx1) qx1 += stx, qx2 += stx;
    if (qz1) qz1 += stz, qz2 += stz;
    __syncthreads();  // every thread is done with the stages the producer refills next
#pragma unroll
    for (int k = 0; k < 2 * R4; k++) q[k] = q[k + 1];
  }
  // After the producer's own wait gave up, its last copies (at most one per
  // stage) may still be in flight: it waits for them, bounded, before the CTA
  // leaves.  Otherwise it has waited for every plane it issued.
  if (producer && !ok) {
    for (int p = max(y0, last_a - SA + 1); p <= last_a; p++) mbar_drain(&s.bar_a[(p - y0) % SA], ((p - y0) / SA) & 1);
    for (int p = max(y0, last_b - SB + 1); p <= last_b; p++) mbar_drain(&s.bar_b[(p - y0) % SB], ((p - y0) / SB) & 1);
  }
}

template <int TX, int P, bool EDGE>
void tma4_launch(const IsoArgs &a, const Tile4 *tiles, int ntiles, const CUtensorMap &w1, const CUtensorMap &w0,
                 const CUtensorMap &vel, int *err, int mode, int pml3d, cudaStream_t st) {
  const size_t smem = sizeof(Iso4Smem<TX, P>);
#define L_(M, P3) iso_fd8_tma4<TX, P, M, P3, EDGE><<<ntiles, dim3(8, TX), smem, st>>>(a, tiles, w1, w0, vel, err)
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
void tma4_shape(const IsoArgs &a, const Tile4 *tiles, int ntiles, bool edge, const CUtensorMap &w1,
                const CUtensorMap &w0, const CUtensorMap &vel, int *err, int mode, int pml3d, cudaStream_t st) {
  if (ntiles <= 0) return;
  if (edge) tma4_launch<TX, P, true>(a, tiles, ntiles, w1, w0, vel, err, mode, pml3d, st);
  else tma4_launch<TX, P, false>(a, tiles, ntiles, w1, w0, vel, err, mode, pml3d, st);
}

template <int TX, int P, bool EDGE>
bool tma4_attr_e(int smem) {
  bool ok = true;
#define A_(M, P3) \
  ok &= cudaFuncSetAttribute(iso_fd8_tma4<TX, P, M, P3, EDGE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == 0
  A_(0, true);
  A_(1, true);
  A_(2, true);
  A_(0, false);
  A_(1, false);
  A_(2, false);
#undef A_
  return ok;
}

template <int TX, int P>
bool tma4_attr() {
  const int smem = (int)sizeof(Iso4Smem<TX, P>);
  return tma4_attr_e<TX, P, true>(smem) && tma4_attr_e<TX, P, false>(smem);
}

// resident CTAs per SM of the interior (PML-free) kernel, leapfrog mode
template <int TX, int P>
int tma4_occupancy(int pml3d) {
  int n = 0;
  const size_t smem = sizeof(Iso4Smem<TX, P>);
  if (pml3d) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, iso_fd8_tma4<TX, P, 1, true, false>, 8 * TX, smem);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, iso_fd8_tma4<TX, P, 1, false, false>, 8 * TX, smem);
  return n;
}

template <int TX, bool PML3D>
int iso4_occupancy() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, iso_fd8_v4<TX, 1, PML3D>, 8 * TX, 0);
  return n;
}

}  // namespace

int iso_v4_ctas_per_sm(int tx, int pml3d) {
  int n = tx == 32 ? (pml3d ? iso4_occupancy<32, true>() : iso4_occupancy<32, false>())
          : tx == 8 ? (pml3d ? iso4_occupancy<8, true>() : iso4_occupancy<8, false>())
                    : (pml3d ? iso4_occupancy<16, true>() : iso4_occupancy<16, false>());
  return n > 0 ? n : 1;
}

void launch_iso_fd8_v4(const IsoArgs &a, int mode, int pml3d, int tx, cudaStream_t st) {
  if (tx == 32) {
    if (pml3d) iso4_launch<32, true>(a, mode, st);
    else iso4_launch<32, false>(a, mode, st);
  } else if (tx == 8) {
    if (pml3d) iso4_launch<8, true>(a, mode, st);
    else iso4_launch<8, false>(a, mode, st);
  } else {
    if (pml3d) iso4_launch<16, true>(a, mode, st);
    else iso4_launch<16, false>(a, mode, st);
  }
}

// (tile width, prefetch planes) of the TMA-ring kernel
const TmaShape kIso4TmaShapes[] = {{16, 2}, {16, 4}, {32, 2}};
const int kIso4TmaNShapes = sizeof(kIso4TmaShapes) / sizeof(kIso4TmaShapes[0]);

bool iso_tma4_init() { return tma4_attr<16, 2>() && tma4_attr<16, 4>() && tma4_attr<32, 2>(); }

int iso_tma4_ctas_per_sm(int shape, int pml3d) {
  const int n = shape == 0 ? tma4_occupancy<16, 2>(pml3d) : shape == 1 ? tma4_occupancy<16, 4>(pml3d)
                                                                       : tma4_occupancy<32, 2>(pml3d);
  return n > 0 ? n : 1;
}

void launch_iso_fd8_tma4(const IsoArgs &a, const Tile4 *tiles, int ntiles, bool edge, const CUtensorMap &w1,
                         const CUtensorMap &w0, const CUtensorMap &vel, int *err, int mode, int pml3d, int shape,
                         cudaStream_t st) {
  if (shape == 0) tma4_shape<16, 2>(a, tiles, ntiles, edge, w1, w0, vel, err, mode, pml3d, st);
  else if (shape == 1) tma4_shape<16, 4>(a, tiles, ntiles, edge, w1, w0, vel, err, mode, pml3d, st);
  else tma4_shape<32, 2>(a, tiles, ntiles, edge, w1, w0, vel, err, mode, pml3d, st);
}

}  // namespace rtm
