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

// Line solve on an abstract accessor: X(i) reads the input, Y(i) / SET(i, v)
// read / write the in-place result.  in and out may be the same storage.
template <typename Ld, typename St, typename LdOut>
__device__ __forceinline__ void cfd_solve_line(const CfdPlanDev &p, Ld X, St SET, LdOut Y) {
  const int n = p.n;
  const float *__restrict__ a = p.am;
  const float *__restrict__ bm = p.bm;
  const float *__restrict__ al = p.bl;
  // --- forward: rhs_i then y_i = rhs_i - sum_j al[(i-j)*4 + j-1] * y_{i-j}
  float xw[11];  // x[i-5 .. i+5]
#pragma unroll
  for (int k = 0; k < 11; k++) xw[k] = (k >= 5 && k - 5 < n) ? X(k - 5) : 0.f;
  float y1 = 0.f, y2 = 0.f, y3 = 0.f, y4 = 0.f;  // y_{i-1} .. y_{i-4}
  for (int i = 0; i < n; i++) {
    float r;
    if (i < 5) {
      r = 0.f;
      for (int j = 5 - i; j < 11; j++) r = r + a[j * 5 + i] * xw[j];
    } else if (i < n - 5) {
      r = a[55] * (xw[6] - xw[4]) + a[56] * (xw[7] - xw[3]) + a[57] * (xw[8] - xw[2]) + a[58] * (xw[9] - xw[1]) +
          a[59] * (xw[10] - xw[0]);
    } else {
      r = 0.f;
      const int jmax = min(11, n - (i - 5));
      for (int j = 0; j < jmax; j++) r = r - a[n - i + 49 - 5 * j] * xw[j];
    }
    // subtract the elimination terms in the reference's order (oldest pivot first)
    if (i >= 4) r = r - al[(i - 4) * 4 + 3] * y4;
    if (i >= 3) r = r - al[(i - 3) * 4 + 2] * y3;
    if (i >= 2) r = r - al[(i - 2) * 4 + 1] * y2;
    if (i >= 1) r = r - al[(i - 1) * 4 + 0] * y1;
    // slide the input window before the in-place store overwrites x_i
#pragma unroll
    for (int k = 0; k < 10; k++) xw[k] = xw[k + 1];
    xw[10] = (i + 6 < n) ? X(i + 6) : 0.f;
    SET(i, r);
    y4 = y3, y3 = y2, y2 = y1, y1 = r;
  }
  // --- backward substitution with the 5-band upper factor
  float z1 = 0.f, z2 = 0.f, z3 = 0.f, z4 = 0.f;  // f_{i+1} .. f_{i+4}
  for (int i = n - 1; i >= 0; i--) {
    const float *u = bm + i * 5;
    float v = Y(i);
    if (i >= n - 4) {
      const int l = n - 1 - i;  // terms available
      if (l >= 1) v += -u[1] * z1;
      if (l >= 2) v += -u[2] * z2;
      if (l >= 3) v += -u[3] * z3;
      v = v / u[0];
    } else {
      v = (v - u[1] * z1 - u[2] * z2 - u[3] * z3 - u[4] * z4) / u[0];
    }
    SET(i, v);
    z4 = z3, z3 = z2, z2 = z1, z1 = v;
  }
}

// x or y lines: thread per (iz, other index); stride between line points.
__global__ void cfd_strided_k(CfdPlanDev p, const float *__restrict__ in, float *out, int nz, long long stride,
                              long long other_stride, int n_other) {
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  const int o = blockIdx.y;
  if (iz >= nz || o >= n_other) return;
  const long long base = (long long)o * other_stride + iz;
  const float *src = in + base;
  float *dst = out + base;
  cfd_solve_line(
      p, [&](int i) { return __ldg(src + (long long)i * stride); }, [&](int i, float v) { dst[(long long)i * stride] = v; },
      [&](int i) { return dst[(long long)i * stride]; });
}

// z lines: 32 lines per CTA through shared memory
__global__ void cfd_z_k(CfdPlanDev p, const float *__restrict__ in, float *out, long long nlines) {
  extern __shared__ float sm[];
  const int n = p.n, ld = n + 1;
  const long long l0 = (long long)blockIdx.x * 32;
  const int nl = (int)min(32LL, nlines - l0);
  // coalesced stage-in: warp w copies lines w, w+nw, ...
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int l = warp; l < nl; l += nw)
    for (int i = lane; i < n; i += 32) sm[l * ld + i] = __ldg(in + (l0 + l) * n + i);
  __syncthreads();
  if (threadIdx.x < nl) {
    float *line = sm + threadIdx.x * ld;
    cfd_solve_line(
        p, [&](int i) { return line[i]; }, [&](int i, float v) { line[i] = v; }, [&](int i) { return line[i]; });
  }
  __syncthreads();
  for (int l = warp; l < nl; l += nw)
    for (int i = lane; i < n; i += 32) out[(l0 + l) * n + i] = sm[l * ld + i];
}

__global__ void cfd_grad_epi_k(CfdGradEpiArgs a) {
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  const long long n = g.nxz * a.ny;
  const bool do_y = a.ny > 1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int iy = (int)(i / g.nxz);
    const long long in = i - (long long)iy * g.nxz;
    const int ix = (int)(in / a.nz), iz = (int)(in - (long long)ix * a.nz);
    float gz = a.gz[i], gx = a.gx[i], gy = do_y ? a.gy[i] : 0.f;
    pml1(a.pml, g, a.pml3d, DZ, 0, gz, ix, iy, iz);
    pml1(a.pml, g, a.pml3d, DX, 0, gx, ix, iy, iz);
    if (do_y) pml1(a.pml, g, a.pml3d, DY, 0, gy, ix, iy, iz);
    if (a.model >= 2) {
      float e = a.eps[i];
      const float dl = e - a.del[i];
      e = 1.0f + 2.0f * e;
      if (a.model == 3) {
        const float ax = a.pjx[i], ay = do_y ? a.pjy[i] : 0.f;
        const float az = sqrtf(1.0f - (ax * ax + ay * ay));
        const float v2 = gx * gx + gy * gy + gz * gz;
        const float vzz = gx * ax + gy * ay + gz * az;
        const float vz2 = vzz * vzz, vh2 = v2 - vz2;
        const float ecl = e * vh2 + vz2;
        const float parts = sqrtf(1.0f - 8.0f * (dl * (vh2 * vz2)) / (ecl * ecl + 1e-32f));
        const float sc = fminf(0.5f * (1.0f + parts), 1.0f);
        const float bx = vzz * ax, by = vzz * ay, bz = vzz * az;
        gx = (bx + (gx - bx) * e) * sc;
        gy = (by + (gy - by) * e) * sc;
        gz = (bz + (gz - bz) * e) * sc;
      } else {
        const float vx2 = gx * gx + gy * gy, vz2 = gz * gz;
        const float ecl = e * vx2 + vz2;
        const float parts = sqrtf(1.0f - 8.0f * (dl * (vx2 * vz2)) / (ecl * ecl + 1e-32f));
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

__global__ void cfd_div_epi_k(CfdDivEpiArgs a) {
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  const long long n = g.nxz * a.ny;
  const bool do_y = a.ny > 1 && a.dy;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int iy = (int)(i / g.nxz);
    const long long in = i - (long long)iy * g.nxz;
    const int ix = (int)(in / a.nz), iz = (int)(in - (long long)ix * a.nz);
    float dxv = a.dx[i], dzv = a.dz[i], dyv = do_y ? a.dy[i] : 0.f;
    pml1(a.pml, g, a.pml3d, DX, 1, dxv, ix, iy, iz);
    pml1(a.pml, g, a.pml3d, DZ, 1, dzv, ix, iy, iz);
    if (do_y) pml1(a.pml, g, a.pml3d, DY, 1, dyv, ix, iy, iz);
    const float vel = a.vel[i];
    float t = a.w0[i] - dxv * vel;
    t = t - dzv * vel;
    t = t - dyv * vel;
    float out;
    if (a.mode == 0) out = t;
    else {
      const float u = a.w1[i];
      out = a.mode == 1 ? (u + u) - t : q_update(a.q, i, n, t, u);
    }
    a.w0[i] = out;
  }
}

int grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  return (int)(b < 148LL * 16 ? b : 148LL * 16);
}

}  // namespace

void launch_cfd_deriv(int axis, const CfdPlanDev &p, const float *in, float *out, float *scratch, int nx, int ny,
                      int nz, cudaStream_t st) {
  (void)scratch;
  const long long nxz = (long long)nx * nz;
  if (axis == DZ) {
    const long long nlines = (long long)nx * ny;
    const size_t smem = (size_t)32 * (nz + 1) * sizeof(float);
    cfd_z_k<<<(unsigned)((nlines + 31) / 32), 128, smem, st>>>(p, in, out, nlines);
  } else if (axis == DX) {
    dim3 grid((nz + 127) / 128, ny);
    cfd_strided_k<<<grid, 128, 0, st>>>(p, in, out, nz, nz, nxz, ny);
  } else {
    dim3 grid((nz + 127) / 128, nx);
    cfd_strided_k<<<grid, 128, 0, st>>>(p, in, out, nz, nxz, nz, nx);
  }
}

int cfd_init() {
  return cudaFuncSetAttribute(cfd_z_k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) == cudaSuccess ? 0 : -1;
}

void launch_cfd_grad_epilogue(const CfdGradEpiArgs &a, cudaStream_t st) {
  cfd_grad_epi_k<<<grid_for((long long)a.nx * a.ny * a.nz, 256), 256, 0, st>>>(a);
}

void launch_cfd_div_epilogue(const CfdDivEpiArgs &a, cudaStream_t st) {
  cfd_div_epi_k<<<grid_for((long long)a.nx * a.ny * a.nz, 256), 256, 0, st>>>(a);
}

}  // namespace rtm
