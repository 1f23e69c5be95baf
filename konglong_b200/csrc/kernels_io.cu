// kernels_io.cu - the non-stencil kernels of a time step: leapfrog update,
// source / receiver injection (Receiver::apply), receiver extraction
// (ExtractReceiverData::extract), snapshot codecs (WaveFieldCompress) and the
// standalone imaging condition.  All are HBM- or latency-bound elementwise /
// gather work: no tensor cores, coalesced along z.
#include <cuda_fp16.h>

#include <algorithm>

#include "kernel_api.h"
#include "rtm_device.cuh"

namespace rtm {

namespace {

__global__ void update2nd_k(float *__restrict__ w0, const float *__restrict__ w1, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float u = w1[i];
    w0[i] = (u + u) - w0[i];
  }
}

__global__ void update2nd_q_k(float *__restrict__ w0, const float *__restrict__ w1, QDev q, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    w0[i] = q_update(q, i, n, w0[i], w1[i]);
}

// one CTA per (trace, y tap), threads over the x-z taps (z fastest)
__global__ void inject_scatter_k(TraceDev t, int it, float *__restrict__ w0, const float *__restrict__ vel, int nx,
                                 int nz) {
  const int r = t.ids ? t.ids[blockIdx.x] : blockIdx.x;
  const int *o = t.off + 3 * r, *l = t.len + 3 * r;
  const int lx = l[0], lz = l[2];
  const int iy = blockIdx.y;
  if (iy >= l[1]) return;
  const float val = t.traces[(long long)r * t.nt + it] * t.scaler;
  const int ntap = lx * lz;
  for (int k = threadIdx.x; k < ntap; k += blockDim.x) {
    const int iz = k % lz, ix = k / lz;
    const float cy = val * t.ky[(long long)r * t.ly + iy];
    const float cx = cy * t.kx[(long long)r * t.lx + ix];
    const long long c = ((long long)(iy + o[1]) * nx + ix + o[0]) * nz + o[2] + iz;
    atomicAdd(w0 + c, cx * t.kz[(long long)r * t.lz + iz] * vel[c]);
  }
}

// Grouped injection: one CTA per xy tile; every cell of the tile sums the xy
// weight of the group members whose kernel box covers it, then the tile's
// columns receive that sum times the common z kernel.
__global__ void inject_group_k(GroupDev g, TraceDev t, int it, float *__restrict__ w0, const float *__restrict__ vel,
                               int nx, int ny, int nz) {
  extern __shared__ float s_xy[];
  const int T = g.tile;
  const int tile = blockIdx.x;
  const int x0 = g.tile_xy[2 * tile], y0 = g.tile_xy[2 * tile + 1];
  const int b = g.tile_ptr[tile], e = g.tile_ptr[tile + 1];
  for (int c = threadIdx.x; c < T * T; c += blockDim.x) {
    const int ix = x0 + c % T, iy = y0 + c / T;
    float acc = 0.f;
    for (int k = b; k < e; k++) {
      const int r = g.tile_list[k];
      const int *o = t.off + 3 * r, *l = t.len + 3 * r;
      const int jx = ix - o[0], jy = iy - o[1];
      if (jx < 0 || jx >= l[0] || jy < 0 || jy >= l[1]) continue;
      const float val = t.traces[(long long)r * t.nt + it] * t.scaler;
      acc += val * t.ky[(long long)r * t.ly + jy] * t.kx[(long long)r * t.lx + jx];
    }
    s_xy[c] = acc;
  }
  __syncthreads();
  const int lz = g.lz;
  for (int k = threadIdx.x; k < T * T * lz; k += blockDim.x) {
    const int iz = k % lz, c = k / lz;
    const int ix = x0 + c % T, iy = y0 + c / T;
    const float s = s_xy[c];
    if (ix >= nx || iy >= ny || s == 0.f) continue;
    const long long i = ((long long)iy * nx + ix) * nz + g.offz + iz;
    w0[i] += s * g.kz[iz] * vel[i];
  }
}

// one warp per receiver over its kernel box
__global__ void extract_direct_k(TraceDev t, const float *__restrict__ w0, float *__restrict__ out, int jt, int nt_out,
                                 int nx, int nz) {
  const int k0 = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (k0 >= (t.ids ? t.nids : t.ntr)) return;
  const int r = t.ids ? t.ids[k0] : k0;
  const int *o = t.off + 3 * r, *l = t.len + 3 * r;
  const int lx = l[0], ly = l[1], lz = l[2];
  float acc = 0.f;
  for (int k = lane; k < lx * ly * lz; k += 32) {
    const int iz = k % lz, ix = (k / lz) % lx, iy = k / (lz * lx);
    const float cx = t.ky[(long long)r * t.ly + iy] * t.kx[(long long)r * t.lx + ix];
    acc += cx * t.kz[(long long)r * t.lz + iz] * w0[((long long)(iy + o[1]) * nx + ix + o[0]) * nz + o[2] + iz];
  }
#pragma unroll
  for (int s = 16; s; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
  if (lane == 0) out[(long long)r * nt_out + jt] = acc;
}

// z reduction of a group's band on its tiles: plane[iy*nx+ix] = sum kz * w0
__global__ void extract_zplane_k(GroupDev g, const float *__restrict__ w0, float *__restrict__ plane, int nx, int ny,
                                 int nz) {
  const int T = g.tile;
  const int tile = blockIdx.x;
  const int x0 = g.tile_xy[2 * tile], y0 = g.tile_xy[2 * tile + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x / 32, nw = blockDim.x / 32;
  for (int c = warp; c < T * T; c += nw) {
    const int ix = x0 + c % T, iy = y0 + c / T;
    if (ix >= nx || iy >= ny) continue;
    const long long base = ((long long)iy * nx + ix) * nz + g.offz;
    float acc = 0.f;
    for (int iz = lane; iz < g.lz; iz += 32) acc += g.kz[iz] * w0[base + iz];
#pragma unroll
    for (int s = 16; s; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
    if (lane == 0) plane[(long long)iy * nx + ix] = acc;
  }
}

__global__ void extract_xy_k(GroupDev g, TraceDev t, const float *__restrict__ plane, float *__restrict__ out, int jt,
                             int nt_out, int nx) {
  const int m = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (m >= g.ntr) return;
  const int r = g.members[m];
  const int *o = t.off + 3 * r, *l = t.len + 3 * r;
  float acc = 0.f;
  for (int k = lane; k < l[0] * l[1]; k += 32) {
    const int ix = k % l[0], iy = k / l[0];
    acc += t.ky[(long long)r * t.ly + iy] * t.kx[(long long)r * t.lx + ix] *
           plane[(long long)(iy + o[1]) * nx + ix + o[0]];
  }
#pragma unroll
  for (int s = 16; s; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
  if (lane == 0) out[(long long)r * nt_out + jt] = acc;
}

// per-slab max |w| (one CTA per y slab)
__global__ void slab_max_k(const float *__restrict__ w, float *__restrict__ slab, uint16_t *c16, int fmt, long long nxz) {
  const int iy = blockIdx.x;
  const float *p = w + (long long)iy * nxz;
  float m = 0.f;
  for (long long i = threadIdx.x; i < nxz; i += blockDim.x) m = fmaxf(m, fabsf(p[i]));
#pragma unroll
  for (int s = 16; s; s >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, s));
  __shared__ float red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.f;
#pragma unroll
    for (int s = 16; s; s >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, s));
    if (threadIdx.x == 0) {
      if (fmt == 1) {
        const float hdr = m > 1e-25f ? m : 0.f;  // compress16 zeroes silent slabs
        slab[iy] = hdr;
        if (c16) {
          const unsigned bits = __float_as_uint(hdr);
          uint16_t *h = c16 + (long long)iy * (nxz + 2);
          h[0] = (uint16_t)(bits & 0xffffu);
          h[1] = (uint16_t)(bits >> 16);
        }
      } else {
        slab[iy] = m * 6.103515625e-05f;  // fp16 slab scale: max maps to 2^14
      }
    }
  }
}

// elementwise kernels: block (32 z, 8 x), grid (z tiles, x tiles, ny)
__global__ void __launch_bounds__(256) fused_io_k(FusedIo io, const float *__restrict__ u, int nx, int ny, int nz) {
  const Grid3 g{nx, ny, nz, (long long)nx * nz};
  const int iz = blockIdx.x * 32 + threadIdx.x, ix = blockIdx.y * 8 + threadIdx.y, iy = blockIdx.z;
  if (iz >= nz || ix >= nx) return;
  const long long in = (long long)ix * nz + iz, i = (long long)iy * g.nxz + in;
  fused_io(io, g, i, ix, iy, iz, in, u[i]);
}

__global__ void __launch_bounds__(256) snap_decode_k(SnapDev s, float *__restrict__ out, const float *ex,
                                                     const float *ey, const float *ez, int nx, int ny, int nz) {
  const Grid3 g{nx, ny, nz, (long long)nx * nz};
  const int iz = blockIdx.x * 32 + threadIdx.x, ix = blockIdx.y * 8 + threadIdx.y, iy = blockIdx.z;
  if (iz >= nz || ix >= nx) return;
  const long long in = (long long)ix * nz + iz, i = (long long)iy * g.nxz + in;
  float v = snap_read(s, g, i, iy, in);
  if (ex) {
    v = v * ey[iy];
    v = v * ex[ix];
    v = v * ez[iz];
  }
  out[i] = v;
}

__global__ void c16_encode_k(const float *__restrict__ in, uint16_t *__restrict__ out, const float *__restrict__ slab,
                             long long nxz) {
  const int iy = blockIdx.y;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nxz; k += (long long)gridDim.x * blockDim.x) {
    const float vmax = slab[iy];
    out[(long long)iy * (nxz + 2) + 2 + k] =
        vmax > 1e-25f ? c16_encode(in[(long long)iy * nxz + k] * __frcp_rn(vmax)) : (uint16_t)0;
  }
}

__global__ void c16_slab_hdr_k(const uint16_t *__restrict__ c, float *__restrict__ slab, int ny, long long nxz) {
  const int iy = blockIdx.x * blockDim.x + threadIdx.x;
  if (iy >= ny) return;
  const uint16_t *h = c + (long long)iy * (nxz + 2);
  slab[iy] = __uint_as_float((unsigned)h[0] | ((unsigned)h[1] << 16));
}

__global__ void nonfinite_k(const float *__restrict__ w, long long n, int *flag) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!isfinite(w[i])) {
      *flag = 1;
      return;
    }
}

// Propagator::Vel2 (bgprtm/Propagator.cpp:711-742): v -> (v dt)^2, Q-corrected
__global__ void vel2_k(float *__restrict__ vel, float *__restrict__ invq, long long n, float dt2, float cq0, int use_q) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float v = vel[i];
    if (!use_q) {
      vel[i] = (v * v) * dt2;
    } else {
      const float q = invq[i], q2 = q * q;
      const float corr = 1.0f / (1.0f - cq0 * q);
      vel[i] = v * v * dt2 * (1.0f - 0.25f * q2 + q2 * q2 / 48.0f) * corr;
      invq[i] = q * corr;
    }
  }
}

int grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  return (int)(b < 148LL * 16 ? b : 148LL * 16);
}

}  // namespace

void launch_update2nd(float *w0, const float *w1, const QDev *q, long long n, cudaStream_t st) {
  if (q) update2nd_q_k<<<grid_for(n, 256), 256, 0, st>>>(w0, w1, *q, n);
  else update2nd_k<<<grid_for(n, 256), 256, 0, st>>>(w0, w1, n);
}

void launch_inject_scatter(const TraceDev &t, int it, float *w0, const float *vel, int nx, int ny, int nz,
                           cudaStream_t st) {
  (void)ny;
  const int cnt = t.ids ? t.nids : t.ntr;
  if (cnt <= 0 || it < 0 || it >= t.nt) return;
  inject_scatter_k<<<dim3(cnt, t.ly), 256, 0, st>>>(t, it, w0, vel, nx, nz);
}

// Batched injection: block (trace, y row of its kernel, shot); the same
// scatter as inject_scatter_k into the step output of each shot.
__global__ void batch_inject_k(const IsoBatchShot *__restrict__ shots, int it_src, int it) {
  const IsoBatchShot &S = shots[blockIdx.z];
  const TraceDev &t = S.inj;
  const int r = blockIdx.x;
  if (r >= t.ntr || it_src < 0 || it_src >= t.nt) return;
  const int *o = t.off + 3 * r, *l = t.len + 3 * r;
  const int lx = l[0], lz = l[2];
  const int iy = blockIdx.y;
  if (iy >= l[1]) return;
  float *w0 = (it & 1) ? S.wa : S.wb;
  const float *vel = S.a.vel;
  const int nx = S.a.nx, nz = S.a.nz;
  const float val = t.traces[(long long)r * t.nt + it_src] * t.scaler;
  const int ntap = lx * lz;
  for (int k = threadIdx.x; k < ntap; k += blockDim.x) {
    const int iz = k % lz, ix = k / lz;
    const float cy = val * t.ky[(long long)r * t.ly + iy];
    const float cx = cy * t.kx[(long long)r * t.lx + ix];
    const long long c = ((long long)(iy + o[1]) * nx + ix + o[0]) * nz + o[2] + iz;
    atomicAdd(w0 + c, cx * t.kz[(long long)r * t.lz + iz] * vel[c]);
  }
}

// Batched extraction: a warp per receiver (extract_direct_k), blockIdx.y = shot.
__global__ void batch_extract_k(const IsoBatchShot *__restrict__ shots, int jt, int it) {
  const IsoBatchShot &S = shots[blockIdx.y];
  const TraceDev &t = S.ext;
  const int r = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (r >= t.ntr || jt < 0 || jt >= t.nt) return;
  const float *w0 = (it & 1) ? S.wa : S.wb;
  const int nx = S.a.nx, nz = S.a.nz;
  const int *o = t.off + 3 * r, *l = t.len + 3 * r;
  const int lx = l[0], ly = l[1], lz = l[2];
  float acc = 0.f;
  for (int k = lane; k < lx * ly * lz; k += 32) {
    const int iz = k % lz, ix = (k / lz) % lx, iy = k / (lz * lx);
    const float cx = t.ky[(long long)r * t.ly + iy] * t.kx[(long long)r * t.lx + ix];
    acc += cx * t.kz[(long long)r * t.lz + iz] * w0[((long long)(iy + o[1]) * nx + ix + o[0]) * nz + o[2] + iz];
  }
#pragma unroll
  for (int s = 16; s; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
  if (lane == 0) S.ext_out[(long long)r * t.nt + jt] = acc;
}

void launch_batch_inject(const IsoBatchShot *shots, int nactive, int max_ntr, int max_ly, int it_src, int it,
                         cudaStream_t st) {
  if (nactive <= 0 || max_ntr <= 0 || max_ly <= 0) return;
  batch_inject_k<<<dim3(max_ntr, max_ly, nactive), 256, 0, st>>>(shots, it_src, it);
}

void launch_batch_extract(const IsoBatchShot *shots, int nactive, int max_ntr, int jt, int it, cudaStream_t st) {
  if (nactive <= 0 || max_ntr <= 0) return;
  batch_extract_k<<<dim3((max_ntr + 7) / 8, nactive), 256, 0, st>>>(shots, jt, it);
}

// ---- FP16 wavefield state ----------------------------------------------------
// new-field scales: the largest slab max within +-4 slabs of either field
// (the stencil radius bounds how far the wave moves in one step), at least
// `floor`, with 16x headroom (2^-12 of the FP16 range 65504 ~ 2^16)
__global__ void f16_scales_k(const unsigned *__restrict__ m0, const unsigned *__restrict__ m1, float *sn, int ny,
                             float floor) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= ny) return;
  float m = floor;
  for (int d = -4; d <= 4; d++) {
    const int k = y + d;
    if (k < 0 || k >= ny) continue;
    m = fmaxf(m, fmaxf(__uint_as_float(m0[k]), __uint_as_float(m1[k])));
  }
  sn[y] = m * (1.0f / 4096.0f);
}

// snapshot slab headers (COMPRESS_16 vmax / FP16 slab scale, as slab_max_k
// writes them) from the tracked slab maxima of the FP16 state
__global__ void f16_slab_hdr_k(const unsigned *__restrict__ m, float *slab, uint16_t *c16, int fmt, long long nxz,
                               int ny) {
  const int iy = blockIdx.x * blockDim.x + threadIdx.x;
  if (iy >= ny) return;
  const float mx = __uint_as_float(m[iy]);
  if (fmt == 1) {
    const float hdr = mx > 1e-25f ? mx : 0.f;
    slab[iy] = hdr;
    if (c16) {
      const unsigned bits = __float_as_uint(hdr);
      uint16_t *h = c16 + (long long)iy * (nxz + 2);
      h[0] = (uint16_t)(bits & 0xffffu);
      h[1] = (uint16_t)(bits >> 16);
    }
  } else {
    slab[iy] = mx * 6.103515625e-05f;
  }
}

__global__ void f16_to_f32_k(const __half *__restrict__ h, const float *__restrict__ s, float *__restrict__ out,
                             long long nxz, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = __half2float(h[i]) * s[i / nxz];
}

// one block per y slab: max, scale, conversion
__global__ void f32_to_f16_k(const float *__restrict__ in, __half *__restrict__ h, float *s, unsigned *m, long long nxz,
                             float floor) {
  __shared__ float red[32];
  const long long base = (long long)blockIdx.x * nxz;
  float a = 0.f;
  for (long long i = threadIdx.x; i < nxz; i += blockDim.x) a = fmaxf(a, fabsf(in[base + i]));
  for (int o = 16; o; o >>= 1) a = fmaxf(a, __shfl_xor_sync(0xffffffffu, a, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x < 32) {
    a = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
    for (int o = 16; o; o >>= 1) a = fmaxf(a, __shfl_xor_sync(0xffffffffu, a, o));
    if (threadIdx.x == 0) red[0] = a;
  }
  __syncthreads();
  const float mx = red[0], sc = fmaxf(mx, floor) * (1.0f / 4096.0f);
  if (threadIdx.x == 0) s[blockIdx.x] = sc, m[blockIdx.x] = __float_as_uint(mx);
  const float r = 1.0f / sc;
  for (long long i = threadIdx.x; i < nxz; i += blockDim.x) h[base + i] = __float2half_rn(in[base + i] * r);
}

// Receiver::apply_src into FP16 state: value / scale added with a 16-bit atomic
__global__ void inject_scatter_f16_k(TraceDev t, int it, __half *__restrict__ h, const float *__restrict__ s,
                                     unsigned *m, const float *__restrict__ vel, int nx, int nz) {
  const int r = blockIdx.x;
  const int *o = t.off + 3 * r, *l = t.len + 3 * r;
  const int lx = l[0], lz = l[2];
  const int iy = blockIdx.y;
  if (iy >= l[1]) return;
  const int gy = iy + o[1];
  const float val = t.traces[(long long)r * t.nt + it] * t.scaler;
  const float rs = 1.0f / s[gy];
  float amax = 0.f;
  for (int k = threadIdx.x; k < lx * lz; k += blockDim.x) {
    const int iz = k % lz, ix = k / lz;
    const float cy = val * t.ky[(long long)r * t.ly + iy];
    const float cx = cy * t.kx[(long long)r * t.lx + ix];
    const long long c = ((long long)gy * nx + ix + o[0]) * nz + o[2] + iz;
    const float add = cx * t.kz[(long long)r * t.lz + iz] * vel[c];
    const __half old = atomicAdd(h + c, __float2half_rn(add * rs));
    amax = fmaxf(amax, fabsf(__half2float(old) + add * rs) * s[gy]);
  }
  for (int o2 = 16; o2; o2 >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o2));
  if ((threadIdx.x & 31) == 0 && amax > 0.f) atomicMax(m + gy, __float_as_uint(amax));
}

__global__ void extract_direct_f16_k(TraceDev t, const __half *__restrict__ h, const float *__restrict__ s,
                                     float *__restrict__ out, int jt, int nt_out, int nx, int nz) {
  const int r = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (r >= t.ntr) return;
  const int *o = t.off + 3 * r, *l = t.len + 3 * r;
  const int lx = l[0], ly = l[1], lz = l[2];
  float acc = 0.f;
  for (int k = lane; k < lx * ly * lz; k += 32) {
    const int iz = k % lz, ix = (k / lz) % lx, iy = k / (lz * lx);
    const float cx = t.ky[(long long)r * t.ly + iy] * t.kx[(long long)r * t.lx + ix];
    const long long c = ((long long)(iy + o[1]) * nx + ix + o[0]) * nz + o[2] + iz;
    acc += cx * t.kz[(long long)r * t.lz + iz] * (__half2float(h[c]) * s[iy + o[1]]);
  }
  for (int o2 = 16; o2; o2 >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o2);
  if (lane == 0) out[(long long)r * nt_out + jt] = acc;
}

void launch_f16_scales(const unsigned *m0, const unsigned *m1, float *sn, int ny, float floor, cudaStream_t st) {
  f16_scales_k<<<(ny + 127) / 128, 128, 0, st>>>(m0, m1, sn, ny, floor);
}
void launch_f16_slab_hdr(const unsigned *m, float *slab, uint16_t *c16, int fmt, int nx, int ny, int nz,
                         cudaStream_t st) {
  f16_slab_hdr_k<<<(ny + 127) / 128, 128, 0, st>>>(m, slab, c16, fmt, (long long)nx * nz, ny);
}
void launch_f16_to_f32(const __half *h, const float *s, float *out, int ny, long long nxz, cudaStream_t st) {
  const long long n = nxz * ny;
  f16_to_f32_k<<<(int)std::min<long long>((n + 255) / 256, 148 * 16), 256, 0, st>>>(h, s, out, nxz, n);
}
void launch_f32_to_f16(const float *in, __half *h, float *s, unsigned *m, int ny, long long nxz, float floor,
                       cudaStream_t st) {
  f32_to_f16_k<<<ny, 512, 0, st>>>(in, h, s, m, nxz, floor);
}
void launch_inject_scatter_f16(const TraceDev &t, int it, __half *h, const float *s, unsigned *m, const float *vel,
                               int nx, int ny, int nz, cudaStream_t st) {
  (void)ny;
  if (t.ntr <= 0 || it < 0 || it >= t.nt) return;
  inject_scatter_f16_k<<<dim3(t.ntr, t.ly), 256, 0, st>>>(t, it, h, s, m, vel, nx, nz);
}
void launch_extract_direct_f16(const TraceDev &t, const __half *h, const float *s, float *out, int jt, int nt_out,
                               int nx, int ny, int nz, cudaStream_t st) {
  (void)ny;
  if (t.ntr <= 0 || jt < 0 || jt >= nt_out) return;
  extract_direct_f16_k<<<(t.ntr + 7) / 8, 256, 0, st>>>(t, h, s, out, jt, nt_out, nx, nz);
}

void launch_inject_group(const GroupDev &gr, const TraceDev &t, int it, float *plane, float *w0, const float *vel,
                         int nx, int ny, int nz, cudaStream_t st) {
  (void)plane;
  if (gr.ntiles <= 0 || it < 0 || it >= t.nt) return;
  inject_group_k<<<gr.ntiles, 256, gr.tile * gr.tile * sizeof(float), st>>>(gr, t, it, w0, vel, nx, ny, nz);
}

void launch_extract_direct(const TraceDev &t, const float *w0, float *out, int jt, int nt_out, int nx, int ny, int nz,
                           cudaStream_t st) {
  (void)ny;
  const int cnt = t.ids ? t.nids : t.ntr;
  if (cnt <= 0 || jt < 0 || jt >= nt_out) return;
  extract_direct_k<<<(cnt + 7) / 8, 256, 0, st>>>(t, w0, out, jt, nt_out, nx, nz);
}

void launch_extract_group(const GroupDev &gr, const TraceDev &t, const float *w0, float *plane, float *out, int jt,
                          int nt_out, int nx, int ny, int nz, cudaStream_t st) {
  if (gr.ntiles <= 0 || jt < 0 || jt >= nt_out) return;
  extract_zplane_k<<<gr.ntiles, 256, 0, st>>>(gr, w0, plane, nx, ny, nz);
  extract_xy_k<<<(gr.ntr + 7) / 8, 256, 0, st>>>(gr, t, plane, out, jt, nt_out, nx);
}

void launch_slab_max(const float *w, float *slab, uint16_t *c16_base, int fmt, int nx, int ny, int nz, cudaStream_t st) {
  slab_max_k<<<ny, 1024, 0, st>>>(w, slab, c16_base, fmt, (long long)nx * nz);
}

void launch_fused_io(const FusedIo &io, const float *u, int nx, int ny, int nz, cudaStream_t st) {
  fused_io_k<<<dim3((nz + 31) / 32, (nx + 7) / 8, ny), dim3(32, 8), 0, st>>>(io, u, nx, ny, nz);
}

void launch_snap_decode(const SnapDev &s, float *out, const float *ex, const float *ey, const float *ez, int nx, int ny,
                        int nz, cudaStream_t st) {
  snap_decode_k<<<dim3((nz + 31) / 32, (nx + 7) / 8, ny), dim3(32, 8), 0, st>>>(s, out, ex, ey, ez, nx, ny, nz);
}

void launch_c16_compress(const float *in, uint16_t *out, float *slab, int nx, int ny, int nz, cudaStream_t st) {
  const long long nxz = (long long)nx * nz;
  slab_max_k<<<ny, 1024, 0, st>>>(in, slab, out, 1, nxz);
  c16_encode_k<<<dim3((unsigned)std::min<long long>((nxz + 255) / 256, 64), ny), 256, 0, st>>>(in, out, slab, nxz);
}

void launch_c16_uncompress(const uint16_t *in, float *out, float *slab, const float *ex, const float *ey,
                           const float *ez, int nx, int ny, int nz, cudaStream_t st) {
  // the header of each slab is its scale; then the generic decode path
  const long long nxz = (long long)nx * nz;
  c16_slab_hdr_k<<<(ny + 255) / 256, 256, 0, st>>>(in, slab, ny, nxz);
  SnapDev s{1, (void *)in, slab};
  launch_snap_decode(s, out, ex, ey, ez, nx, ny, nz, st);
}

void launch_vel2(float *vel, float *invq, long long n, float dt2, float cq0, int use_q, cudaStream_t st) {
  vel2_k<<<grid_for(n, 256), 256, 0, st>>>(vel, invq, n, dt2, cq0, use_q);
}

void launch_nonfinite_scan(const float *w, long long n, int *flag, cudaStream_t st) {
  nonfinite_k<<<grid_for(n, 256), 256, 0, st>>>(w, n, flag);
}

// ---- shot illumination compensation (ImagingCondition::computeDamping /
// applyDamping, bgprtm/ImagingCondition.cpp:600-677; avgVolume3D / avgVolume1D,
// bgprtm/volumefilter.cpp:59-135) --------------------------------------------

namespace {

// Running box average of half width h along one axis of every line (one thread
// per line, the reference's order: edge value counted h+1 times, then one add
// and one subtract per step).  Line t: axis 0 = y (lines over x, z), 1 = x
// (lines over y, z), 2 = z (lines over y, x).
__global__ void box_avg_k(const float *__restrict__ a, float *__restrict__ b, int axis, int nx, int ny, int nz, int h) {
  const long long nxz = (long long)nx * nz;
  const long long nl = axis == 0 ? nxz : axis == 1 ? (long long)ny * nz : (long long)ny * nx;
  const float scaler = 1.0f / (2.0f * h + 1.0f);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nl; t += (long long)gridDim.x * blockDim.x) {
    long long base, stride;
    int n1;
    if (axis == 0) base = t, stride = nxz, n1 = ny;
    else if (axis == 1) base = (t / nz) * nxz + t % nz, stride = nz, n1 = nx;
    else base = t * nz, stride = 1, n1 = nz;
    float m = __fmul_rn((float)h + 1.0f, a[base]);
    for (int j = 1; j <= h; j++) m = __fadd_rn(m, a[base + (long long)min(j, n1 - 1) * stride]);
    b[base] = __fmul_rn(m, scaler);
    for (int k = 1; k < n1; k++) {
      const int k1 = max(0, k - h - 1), k2 = min(n1 - 1, k + h);
      m = __fadd_rn(m, __fsub_rn(a[base + (long long)k2 * stride], a[base + (long long)k1 * stride]));
      b[base + (long long)k * stride] = __fmul_rn(m, scaler);
    }
  }
}

__global__ void sum_k(const float *__restrict__ a, long long n, double *out) {
  double v = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v += a[i];
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) atomicAdd(out, v);
  }
}

// damping factor 1 / (avg (a + w e^-a)), a = illum / avg, x / y edge tapers,
// then image *= factor; the factor stays in illum
__global__ void damping_k(float *__restrict__ illum, float *__restrict__ image, const double *sum, double count,
                          float amp_damping, float damp_weight, int nx, int ny, int nz) {
  const long long nxz = (long long)nx * nz, n = nxz * ny;
  const double average = pow(*sum / count, (double)amp_damping), o_average = 1.0 / average;
  const int ntaper = 10;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int iy = (int)(i / nxz), ix = (int)((i % nxz) / nz);
    const float aa = (float)(illum[i] * o_average);
    const float bb = expf(-aa);
    float f = (float)(1.0 / (average * (double)__fadd_rn(aa, __fmul_rn(damp_weight, bb))));
    auto wt = [&](int k) { return 0.5f * (1.0f - cosf((float)M_PI * float(k) / float(ntaper))); };
    if (iy < ntaper && ny > 1) f *= wt(iy);
    if (iy > ny - ntaper - 1 && ny > 1) f *= wt(ny - iy - 1);
    if (ix < ntaper) f *= wt(ix);
    if (ix > nx - ntaper - 1) f *= wt(nx - ix - 1);
    illum[i] = f;
    if (image) image[i] *= f;
  }
}

}  // namespace

void launch_illum_compensate(float *illum, float *tmp, float *image, double *dsum, int nx, int ny, int nz, int smooth,
                             int hxy, int hz, float amp_damping, float damp_weight, cudaStream_t st) {
  const long long nxz = (long long)nx * nz, n = nxz * ny;
  auto lines = [&](int axis) { return axis == 0 ? nxz : axis == 1 ? (long long)ny * nz : (long long)ny * nx; };
  if (smooth) {  // avgVolume3D for ny > 1 (y, x, z), avgVolume2D otherwise (x, z)
    if (ny > 1) {
      box_avg_k<<<grid_for(lines(0), 256), 256, 0, st>>>(illum, tmp, 0, nx, ny, nz, hxy);
      box_avg_k<<<grid_for(lines(1), 256), 256, 0, st>>>(tmp, illum, 1, nx, ny, nz, hxy);
    } else {
      box_avg_k<<<grid_for(lines(1), 256), 256, 0, st>>>(illum, tmp, 1, nx, ny, nz, hxy);
      cudaMemcpyAsync(illum, tmp, 4 * (size_t)n, cudaMemcpyDeviceToDevice, st);
    }
    box_avg_k<<<grid_for(lines(2), 256), 256, 0, st>>>(illum, tmp, 2, nx, ny, nz, hz);
    cudaMemcpyAsync(illum, tmp, 4 * (size_t)n, cudaMemcpyDeviceToDevice, st);
  }
  cudaMemsetAsync(dsum, 0, sizeof(double), st);
  sum_k<<<1184, 256, 0, st>>>(illum, n, dsum);
  damping_k<<<grid_for(n, 256), 256, 0, st>>>(illum, image, dsum, (double)n, amp_damping, damp_weight, nx, ny, nz);
}

}  // namespace rtm
