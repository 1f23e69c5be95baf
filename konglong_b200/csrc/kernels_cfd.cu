// kernels_cfd.cu - compact finite differences (FdEngine_cfd + Cfd_plan) on
// sm_100a.  A derivative along one axis solves B f' = A f for every grid line:
// the 11-point right-hand side (banmul_*, bgprtm/FdEngine_cfd.cpp:164-201,
// 304-327), the forward elimination of the band LU and the back substitution
// (banbks_*, bgprtm/FdEngine_cfd.cpp:203-302, 328-356).  A CTA stages 32 lines
// in shared memory (one HBM read and one write per cell):
//   phase 1  all four warps form the right-hand sides of a quarter of every
//            line each, in place (embarrassingly parallel along the line);
//   phase 2  one warp (lane = line) runs the two sequential recurrences in
//            register chunks of 8 points: the chunk's operands are loaded
//            together and the next chunk is prefetched, so the dependency
//            chain is one FMA per point in elimination, FMA + multiply in
//            back substitution.
// The PML / scaling / accumulation steps of FdEngine_cfd::d{x,y,z}1_2D and
// KernelCPU::TTI run as pointwise epilogues afterwards.
#include "kernel_api.h"
#include "rtm_device.cuh"

namespace rtm {

namespace {

constexpr int kChunk = 8;  // points per register chunk (both phases)

// Phase 1: right-hand sides of positions [p0, p1) of one line (element i at
// L[i * S]), in place, C outputs per chunk from a window of C + 10 inputs
// carried in registers.  The first and the last five outputs of the range
// are parked in head / tail and written after a barrier, because the
// neighbouring warps read those inputs as their window ends.  Rows within 5
// of a line end use the one-sided rows of A (banmul_dev_z_c,
// bgprtm/FdEngine_cfd.cpp:304-327).  Requires p1 - p0 to be a multiple of C
// unless p1 == n.
template <int S, int C>
__device__ __forceinline__ void cfd_rhs_range(const float *__restrict__ a, float *L, int n, int p0, int p1,
                                              float (&head)[5], float (&tail)[5]) {
  const float a55 = __ldg(a + 55), a56 = __ldg(a + 56), a57 = __ldg(a + 57), a58 = __ldg(a + 58),
              a59 = __ldg(a + 59);
  float w[C + 10];
#pragma unroll
  for (int k = 0; k < 10; k++) {
    const int j = p0 - 5 + k;
    w[k] = (j >= 0 && j < n) ? L[j * S] : 0.f;
  }
  for (int i0 = p0; i0 < p1; i0 += C) {
#pragma unroll
    for (int k = 10; k < C + 10; k++) {
      const int j = i0 - 5 + k;
      w[k] = j < n ? L[j * S] : 0.f;
    }
    float r[C];
    if (i0 >= 5 && i0 + C <= n - 5) {
#pragma unroll
      for (int k = 0; k < C; k++)
        r[k] = a55 * (w[k + 6] - w[k + 4]) + a56 * (w[k + 7] - w[k + 3]) + a57 * (w[k + 8] - w[k + 2]) +
               a58 * (w[k + 9] - w[k + 1]) + a59 * (w[k + 10] - w[k]);
    } else {
#pragma unroll
      for (int k = 0; k < C; k++) {
        const int i = i0 + k;
        float v = 0.f;
        if (i < 5) {
#pragma unroll
          for (int j = 0; j < 11; j++)
            if (j >= 5 - i) v = v + __ldg(a + j * 5 + i) * w[k + j];
        } else if (i >= n - 5) {
          const int t = n - i;
#pragma unroll
          for (int j = 0; j < 11; j++)
            if (j < t + 5) v = v - __ldg(a + t + 49 - 5 * j) * w[k + j];
        } else {
          v = a55 * (w[k + 6] - w[k + 4]) + a56 * (w[k + 7] - w[k + 3]) + a57 * (w[k + 8] - w[k + 2]) +
              a58 * (w[k + 9] - w[k + 1]) + a59 * (w[k + 10] - w[k]);
        }
        r[k] = v;
      }
    }
#pragma unroll
    for (int k = 0; k < C; k++) {
      const int i = i0 + k;
      if (i < p1) {
        const bool h = i0 == p0 && k < 5, t = i0 + C == p1 && k >= C - 5;
        if (h) head[k < 5 ? k : 0] = r[k];
        if (t) tail[k >= C - 5 ? k - (C - 5) : 0] = r[k];
        if (!h && !t) L[i * S] = r[k];
      }
    }
#pragma unroll
    for (int k = 0; k < 10; k++) w[k] = w[k + C];
  }
}

// Phase 2, forward: y_i = rhs_i - l[i-4][3] y_{i-4} - l[i-3][2] y_{i-3}
// - l[i-2][1] y_{i-2} - l[i-1][0] y_{i-1}, oldest pivot first, with the
// row-packed multipliers lm[i] = (l[i-1][0], l[i-2][1], l[i-3][2], l[i-4][3]).
template <int S, int C>
__device__ __forceinline__ void cfd_forward(const float4 *__restrict__ lm, float *L, int n) {
  float y1 = 0.f, y2 = 0.f, y3 = 0.f, y4 = 0.f;
  float rv[C];
  float4 m[C];
#pragma unroll
  for (int k = 0; k < C; k++) {
    const int i = min(k, n - 1);
    rv[k] = L[i * S];
    m[k] = __ldg(lm + i);
  }
  for (int i0 = 0; i0 < n; i0 += C) {
    float nrv[C];
    float4 nm[C];
#pragma unroll
    for (int k = 0; k < C; k++) {
      const int i = min(i0 + C + k, n - 1);
      nrv[k] = L[i * S];
      nm[k] = __ldg(lm + i);
    }
#pragma unroll
    for (int k = 0; k < C; k++) {
      float r = rv[k];
      r = r - m[k].w * y4;
      r = r - m[k].z * y3;
      r = r - m[k].y * y2;
      r = r - m[k].x * y1;
      y4 = y3, y3 = y2, y2 = y1, y1 = r;
      rv[k] = r;
    }
#pragma unroll
    for (int k = 0; k < C; k++)
      if (i0 + k < n) L[(i0 + k) * S] = rv[k];
#pragma unroll
    for (int k = 0; k < C; k++) rv[k] = nrv[k], m[k] = nm[k];
  }
}

// Phase 2, backward: f_i = (y_i - u3 f_{i+4} - u2 f_{i+3} - u1 f_{i+2}
// - u0 f_{i+1}) * (1 / pivot_i), the reciprocal pivots from the FP64 plan
// set-up.  Upper-factor entries beyond the line end are zero.
template <int S, int C>
__device__ __forceinline__ void cfd_backward(const float4 *__restrict__ bu4, const float *__restrict__ rd, float *L,
                                             int n) {
  float z1 = 0.f, z2 = 0.f, z3 = 0.f, z4 = 0.f;
  float yv[C], rv[C];
  float4 u[C];
#pragma unroll
  for (int k = 0; k < C; k++) {
    const int i = max(n - 1 - k, 0);
    yv[k] = L[i * S];
    u[k] = __ldg(bu4 + i);
    rv[k] = __ldg(rd + i);
  }
  for (int i0 = n - 1; i0 >= 0; i0 -= C) {
    float nyv[C], nrv[C];
    float4 nu[C];
#pragma unroll
    for (int k = 0; k < C; k++) {
      const int i = max(i0 - C - k, 0);
      nyv[k] = L[i * S];
      nu[k] = __ldg(bu4 + i);
      nrv[k] = __ldg(rd + i);
    }
#pragma unroll
    for (int k = 0; k < C; k++) {
      float v = yv[k];
      v = v - u[k].w * z4;
      v = v - u[k].z * z3;
      v = v - u[k].y * z2;
      v = v - u[k].x * z1;
      v = v * rv[k];
      z4 = z3, z3 = z2, z2 = z1, z1 = v;
      yv[k] = v;
    }
#pragma unroll
    for (int k = 0; k < C; k++)
      if (i0 - k >= 0) L[(i0 - k) * S] = yv[k];
#pragma unroll
    for (int k = 0; k < C; k++) yv[k] = nyv[k], u[k] = nu[k], rv[k] = nrv[k];
  }
}

// 32 lines per CTA staged through shared memory; warp 0 walks the lines
// (lane = line), all warps move data.  x / y lines (STRIDED): element i of
// line l at base + l + i*es, smem [i][32]; z lines: line l at base + l*n + i,
// smem [l][n+1].  One HBM read and one write per cell.
template <bool STRIDED>
__global__ void __launch_bounds__(128) cfd_lines_k(CfdPlanDev p, const float *__restrict__ in, float *__restrict__ out,
                                                   int nz, long long es, long long other_stride, int n_other,
                                                   long long nlines) {
  extern __shared__ float sm[];
  const int n = p.n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  constexpr int U = 16;  // independent loads in flight per thread during staging
  long long base;
  int nl;
  if (STRIDED) {
    const int izc = blockIdx.x, o = blockIdx.y;
    const int iz0 = izc * 32;
    nl = min(32, nz - iz0);
    base = (long long)o * other_stride + iz0;
    // rows i of 32 lines: warp w stages rows w*U .. w*U+U-1, then every nw*U rows
    for (int i0 = warp * U; i0 < n; i0 += nw * U) {
      float v[U];
#pragma unroll
      for (int k = 0; k < U; k++) {
        const int i = i0 + k;
        v[k] = (i < n && lane < nl) ? __ldcg(in + base + lane + (long long)i * es) : 0.f;
      }
#pragma unroll
      for (int k = 0; k < U; k++)
        if (i0 + k < n) sm[(i0 + k) * 32 + lane] = v[k];
    }
  } else {
    const long long l0 = (long long)blockIdx.x * 32;
    nl = (int)min(32LL, nlines - l0);
    base = l0 * n;
    const int per_line = (n + 31) / 32;  // 32-float chunks per line
    const int chunks = nl * per_line;
    for (int c0 = warp * U; c0 < chunks; c0 += nw * U) {
      float v[U];
#pragma unroll
      for (int k = 0; k < U; k++) {
        const int c = c0 + k, l = c / per_line, i = (c - l * per_line) * 32 + lane;
        v[k] = (c < chunks && i < n) ? __ldcg(in + base + (long long)l * n + i) : 0.f;
      }
#pragma unroll
      for (int k = 0; k < U; k++) {
        const int c = c0 + k, l = c / per_line, i = (c - l * per_line) * 32 + lane;
        if (c < chunks && i < n) sm[l * (n + 1) + i] = v[k];
      }
    }
  }
  // phase 1: right-hand sides, each warp a run of whole chunks of every line
  constexpr int S = STRIDED ? 32 : 1;
  float *L = STRIDED ? sm + lane : sm + lane * (n + 1);
  const int run = (((n + nw - 1) / nw) + kChunk - 1) / kChunk * kChunk;
  const int p0 = min(n, warp * run), p1 = min(n, p0 + run);
  float head[5], tail[5];
  __syncthreads();
  if (lane < nl && p0 < p1) cfd_rhs_range<S, kChunk>(p.am, L, n, p0, p1, head, tail);
  __syncthreads();
  if (lane < nl && p0 < p1) {
#pragma unroll
    for (int k = 0; k < 5; k++)
      if (p0 + k < p1) L[(p0 + k) * S] = head[k];
    if ((p1 - p0) % kChunk == 0) {
#pragma unroll
      for (int k = 0; k < 5; k++) L[(p1 - 5 + k) * S] = tail[k];
    }
  }
  __syncthreads();
  // phase 2: the two sequential recurrences, one warp
  if (warp == 0 && lane < nl) {
    cfd_forward<S, kChunk>(reinterpret_cast<const float4 *>(p.lm), L, n);
    cfd_backward<S, kChunk>(reinterpret_cast<const float4 *>(p.bu), p.rdiag, L, n);
  }
  __syncthreads();
  if (STRIDED) {
    for (int i = warp; i < n; i += nw)
      if (lane < nl) __stcg(out + base + lane + (long long)i * es, sm[i * 32 + lane]);
  } else {
    for (int l = warp; l < nl; l += nw)
      for (int i = lane; i < n; i += 32) __stcg(out + base + (long long)l * n + i, sm[l * (n + 1) + i]);
  }
}

// pointwise epilogues: block (32 z, 8 x), grid (z tiles, x tiles, ny)
__global__ void __launch_bounds__(256) cfd_grad_epi_k(CfdGradEpiArgs a) {
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  const int iz = blockIdx.x * 32 + threadIdx.x, ix = blockIdx.y * 8 + threadIdx.y, iy = blockIdx.z;
  if (iz >= a.nz || ix >= a.nx) return;
  const bool do_y = a.ny > 1;
  const long long i = (long long)iy * g.nxz + (long long)ix * a.nz + iz;
  {
    float gz = a.gz[i], gx = a.gx[i], gy = do_y ? a.gy[i] : 0.f;
    if (in_pml(a.pml, g, ix, iy, iz)) {
      pml1(a.pml, g, a.pml3d, DZ, 0, gz, ix, iy, iz);
      pml1(a.pml, g, a.pml3d, DX, 0, gx, ix, iy, iz);
      if (do_y) pml1(a.pml, g, a.pml3d, DY, 0, gy, ix, iy, iz);
    }
    if (a.model >= 2) {
      float e = __ldg(a.eps + i);
      const float dl = e - __ldg(a.del + i);
      e = 1.0f + 2.0f * e;
      if (a.model == 3) {
        const float ax = __ldg(a.pjx + i), ay = do_y ? __ldg(a.pjy + i) : 0.f;
        const float az = sqrtf(1.0f - (ax * ax + ay * ay));
        const float v2 = gx * gx + gy * gy + gz * gz;
        const float vzz = gx * ax + gy * ay + gz * az;
        const float vz2 = vzz * vzz, vh2 = v2 - vz2;
        const float ecl = e * vh2 + vz2;
        const float parts = sqrtf(1.0f - 8.0f * (dl * (vh2 * vz2)) * __frcp_rn(ecl * ecl + 1e-32f));
        const float sc = fminf(0.5f * (1.0f + parts), 1.0f);
        const float bx = vzz * ax, by = vzz * ay, bz = vzz * az;
        gx = (bx + (gx - bx) * e) * sc;
        gy = (by + (gy - by) * e) * sc;
        gz = (bz + (gz - bz) * e) * sc;
      } else {
        const float vx2 = gx * gx + gy * gy, vz2 = gz * gz;
        const float ecl = e * vx2 + vz2;
        const float parts = sqrtf(1.0f - 8.0f * (dl * (vx2 * vz2)) * __frcp_rn(ecl * ecl + 1e-32f));
        const float sc2 = e * fminf(0.5f * (1.0f + parts), 1.0f);
        gx *= sc2;
        gy *= sc2;
      }
    }
    a.gz[i] = gz;
    a.gx[i] = gx;
    if (do_y) a.gy[i] = gy;
  }
}

__global__ void __launch_bounds__(256) cfd_div_epi_k(CfdDivEpiArgs a) {
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  const int iz = blockIdx.x * 32 + threadIdx.x, ix = blockIdx.y * 8 + threadIdx.y, iy = blockIdx.z;
  if (iz >= a.nz || ix >= a.nx) return;
  const bool do_y = a.ny > 1 && a.dy;
  const long long i = (long long)iy * g.nxz + (long long)ix * a.nz + iz;
  float dxv = a.dx[i], dzv = a.dz[i], dyv = do_y ? a.dy[i] : 0.f;
  if (in_pml(a.pml, g, ix, iy, iz)) {
    pml1(a.pml, g, a.pml3d, DX, 1, dxv, ix, iy, iz);
    pml1(a.pml, g, a.pml3d, DZ, 1, dzv, ix, iy, iz);
    if (do_y) pml1(a.pml, g, a.pml3d, DY, 1, dyv, ix, iy, iz);
  }
  const float vel = __ldg(a.vel + i);
  float t = a.w0[i] - dxv * vel;
  t = t - dzv * vel;
  t = t - dyv * vel;
  float out;
  if (a.mode == 0) out = t;
  else {
    const float u = __ldg(a.w1 + i);
    out = a.mode == 1 ? (u + u) - t : q_update(a.q, i, g.nxz * a.ny, t, u);
  }
  a.w0[i] = out;
}

}  // namespace

void launch_cfd_deriv(int axis, const CfdPlanDev &p, const float *in, float *out, float *scratch, int nx, int ny,
                      int nz, cudaStream_t st) {
  (void)scratch;
  const long long nxz = (long long)nx * nz;
  if (axis == DZ) {
    const long long nlines = (long long)nx * ny;
    const size_t smem = (size_t)32 * (nz + 1) * sizeof(float);
    cfd_lines_k<false><<<(unsigned)((nlines + 31) / 32), 128, smem, st>>>(p, in, out, nz, 1, 0, 0, nlines);
  } else {
    const int n = axis == DX ? nx : ny;
    const size_t smem = (size_t)32 * n * sizeof(float);
    dim3 grid((nz + 31) / 32, axis == DX ? ny : nx);
    if (axis == DX) cfd_lines_k<true><<<grid, 128, smem, st>>>(p, in, out, nz, nz, nxz, ny, 0);
    else cfd_lines_k<true><<<grid, 128, smem, st>>>(p, in, out, nz, nxz, nz, nx, 0);
  }
}

int cfd_init() {
  const int mx = 227 * 1024;
  bool ok = cudaFuncSetAttribute(cfd_lines_k<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute(cfd_lines_k<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  return ok ? 0 : -1;
}

void launch_cfd_grad_epilogue(const CfdGradEpiArgs &a, cudaStream_t st) {
  cfd_grad_epi_k<<<dim3((a.nz + 31) / 32, (a.nx + 7) / 8, a.ny), dim3(32, 8), 0, st>>>(a);
}

void launch_cfd_div_epilogue(const CfdDivEpiArgs &a, cudaStream_t st) {
  cfd_div_epi_k<<<dim3((a.nz + 31) / 32, (a.nx + 7) / 8, a.ny), dim3(32, 8), 0, st>>>(a);
}

}  // namespace rtm
