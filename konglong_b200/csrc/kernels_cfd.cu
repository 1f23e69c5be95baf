// kernels_cfd.cu - compact finite differences (FdEngine_cfd + Cfd_plan) on
// sm_100a.  A derivative along one axis solves B f' = A f for every grid line:
// the 11-point right-hand side (banmul_*, bgprtm/FdEngine_cfd.cpp:164-201,
// 304-327) is fused with the forward elimination of the band LU, then the back
// substitution (banbks_*, bgprtm/FdEngine_cfd.cpp:203-302, 328-356) runs from
// the far end.  The recurrences are sequential along a line, so parallelism
// comes from the batch of lines:
//   x / y lines: one thread per (z, other) line, the walk along the line is a
//     z-coalesced sweep; the forward results are parked in the output array
//     and read back by the backward sweep (same thread, same addresses).
//   z lines (contiguous): a CTA stages 32 lines in shared memory (stride nz+1,
//     bank-conflict free), one thread walks one line, the result is written
//     back through shared memory with coalesced stores.
// The PML / scaling / accumulation steps of FdEngine_cfd::d{x,y,z}1_2D and
// KernelCPU::TTI run as pointwise epilogues afterwards.
#include "kernel_api.h"
#include "rtm_device.cuh"

namespace rtm {

namespace {

// Line solve on an accessor A(i) -> float& into shared memory, in place.
// Forward: rhs_i = (A x)_i, then y_i = rhs_i - sum_j al[(i-j)*4+j-1] y_{i-j};
// backward: f_i = (y_i - sum_k bm[i*5+k] f_{i+k}) * (1 / bm[i*5]).  The
// newest recurrence term is applied last, so one FMA sits on the dependency
// chain per point; the pivots' reciprocals come from the FP64 plan set-up.
template <typename Acc>
__device__ __forceinline__ void cfd_solve_line(const CfdPlanDev &p, Acc A) {
  const int n = p.n;
  const float *__restrict__ a = p.am;
  const float4 *__restrict__ bu4 = reinterpret_cast<const float4 *>(p.bu);
  const float4 *__restrict__ al4 = reinterpret_cast<const float4 *>(p.bl);
  const float *__restrict__ rd = p.rdiag;
  const float a55 = __ldg(a + 55), a56 = __ldg(a + 56), a57 = __ldg(a + 57), a58 = __ldg(a + 58),
              a59 = __ldg(a + 59);
  float xw[11];  // x[i-5 .. i+5]
#pragma unroll
  for (int k = 0; k < 11; k++) xw[k] = (k >= 5 && k - 5 < n) ? A(k - 5) : 0.f;
  float y1 = 0.f, y2 = 0.f, y3 = 0.f, y4 = 0.f;
  // multipliers applied to row i: al[i-1].x, al[i-2].y, al[i-3].z, al[i-4].w
  float4 m1 = make_float4(0.f, 0.f, 0.f, 0.f), m2 = m1, m3 = m1, m4 = m1;  // rows i-1 .. i-4
  // rows 0..4: one-sided boundary rows of A
#pragma unroll
  for (int i = 0; i < 5; i++) {
    float r = 0.f;
#pragma unroll
    for (int j = 5 - i; j < 11; j++) r = r + __ldg(a + j * 5 + i) * xw[j];
    r = r - m4.w * y4;
    r = r - m3.z * y3;
    r = r - m2.y * y2;
    r = r - m1.x * y1;
#pragma unroll
    for (int k = 0; k < 10; k++) xw[k] = xw[k + 1];
    xw[10] = (i + 6 < n) ? A(i + 6) : 0.f;
    A(i) = r;
    y4 = y3, y3 = y2, y2 = y1, y1 = r;
    m4 = m3, m3 = m2, m2 = m1, m1 = __ldg(al4 + i);
  }
  // interior rows: antisymmetric 11-point stencil; the next row's multipliers
  // are fetched one step ahead so no load sits on the recurrence
  float4 nxt = __ldg(al4 + 5);
#pragma unroll 2
  for (int i = 5; i < n - 5; i++) {
    const float x_ahead = (i + 6 < n) ? A(i + 6) : 0.f;
    float r = a55 * (xw[6] - xw[4]) + a56 * (xw[7] - xw[3]) + a57 * (xw[8] - xw[2]) + a58 * (xw[9] - xw[1]) +
              a59 * (xw[10] - xw[0]);
    r = r - m4.w * y4;
    r = r - m3.z * y3;
    r = r - m2.y * y2;
    r = r - m1.x * y1;
#pragma unroll
    for (int k = 0; k < 10; k++) xw[k] = xw[k + 1];
    xw[10] = x_ahead;
    A(i) = r;
    y4 = y3, y3 = y2, y2 = y1, y1 = r;
    m4 = m3, m3 = m2, m2 = m1, m1 = nxt;
    nxt = __ldg(al4 + min(i + 1, n - 1));
  }
  // rows n-5 .. n-1: the mirrored boundary rows
#pragma unroll
  for (int t = 5; t >= 1; t--) {
    const int i = n - t;
    float r = 0.f;
#pragma unroll
    for (int j = 0; j < 11; j++)
      if (j < t + 5) r = r - __ldg(a + t + 49 - 5 * j) * xw[j];
    r = r - m4.w * y4;
    r = r - m3.z * y3;
    r = r - m2.y * y2;
    r = r - m1.x * y1;
#pragma unroll
    for (int k = 0; k < 10; k++) xw[k] = xw[k + 1];
    xw[10] = 0.f;
    A(i) = r;
    y4 = y3, y3 = y2, y2 = y1, y1 = r;
    m4 = m3, m3 = m2, m2 = m1, m1 = __ldg(al4 + i);
  }
  // backward substitution: f_i = (y_i - u3 f_{i+4} - u2 f_{i+3} - u1 f_{i+2} - u0 f_{i+1}) / pivot_i
  float z1 = 0.f, z2 = 0.f, z3 = 0.f, z4 = 0.f;
#pragma unroll
  for (int t = 1; t <= 4; t++) {
    const int i = n - t;
    const float4 u = __ldg(bu4 + i);
    float v = A(i);
    if (t >= 4) v = v - u.z * z3;
    if (t >= 3) v = v - u.y * z2;
    if (t >= 2) v = v - u.x * z1;
    v = v * __ldg(rd + i);
    A(i) = v;
    z4 = z3, z3 = z2, z2 = z1, z1 = v;
  }
  float4 u = __ldg(bu4 + n - 5);
  float rdi = __ldg(rd + n - 5);
  float yv = A(n - 5);
#pragma unroll 2
  for (int i = n - 5; i >= 0; i--) {
    const int j = max(i - 1, 0);
    const float4 un = __ldg(bu4 + j);
    const float rdn = __ldg(rd + j);
    const float yn = A(j);
    float v = yv;
    v = v - u.w * z4;
    v = v - u.z * z3;
    v = v - u.y * z2;
    v = v - u.x * z1;
    v = v * rdi;
    A(i) = v;
    z4 = z3, z3 = z2, z2 = z1, z1 = v;
    u = un, rdi = rdn, yv = yn;
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
  __syncthreads();
  if (warp == 0 && lane < nl) {
    if (STRIDED) cfd_solve_line(p, [&](int i) -> float & { return sm[i * 32 + lane]; });
    else cfd_solve_line(p, [&](int i) -> float & { return sm[lane * (n + 1) + i]; });
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
