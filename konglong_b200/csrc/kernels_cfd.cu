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
#include <type_traits>

#include <algorithm>

#include "kernel_api.h"
#include "rtm_device.cuh"
#include "tma.cuh"

namespace rtm {

namespace {

constexpr int kChunk = 8;  // points per register chunk (both phases)
// prefetch depth (chunks) of the streamed x / y kernel with 32- / 64-bit line
// offsets: the deepest that fits 128 registers without spilling
constexpr int kStreamD = 3, kStreamDWide = 2;

// One right-hand-side row of the 11-band A with every rounding explicit, so
// that each line kernel (staged, streamed, pipelined) gives the same bits:
// interior rows sum_d a[54 + d] (x[i + d] - x[i - d]), d = 1 .. 5, and the
// one-sided rows within 5 of a line end (banmul_dev_z_c,
// bgprtm/FdEngine_cfd.cpp:304-327) accumulated in the reference order.
struct RhsCoef {
  float c1, c2, c3, c4, c5;
};
__device__ __forceinline__ float rhs_interior(const RhsCoef &c, float m5, float m4, float m3, float m2, float m1,
                                              float p1, float p2, float p3, float p4, float p5) {
  float t = __fmul_rn(c.c1, __fsub_rn(p1, m1));
  t = __fmaf_rn(c.c2, __fsub_rn(p2, m2), t);
  t = __fmaf_rn(c.c3, __fsub_rn(p3, m3), t);
  t = __fmaf_rn(c.c4, __fsub_rn(p4, m4), t);
  return __fmaf_rn(c.c5, __fsub_rn(p5, m5), t);
}
// row i < 5 from x[i - 5 + j], j = 0 .. 10 (x[j] here)
__device__ __forceinline__ float rhs_low(const float (&a)[60], int i, const float *x) {
  float v = 0.f;
#pragma unroll
  for (int j = 0; j < 11; j++)
    if (j >= 5 - i) v = __fmaf_rn(a[j * 5 + i], x[j], v);
  return v;
}
// row i = n - t, t = 1 .. 5, from x[i - 5 + j], j = 0 .. 10
__device__ __forceinline__ float rhs_high(const float (&a)[60], int t, const float *x) {
  float v = 0.f;
#pragma unroll
  for (int j = 0; j < 11; j++)
    if (j < t + 5) v = __fmaf_rn(-a[t + 49 - 5 * j], x[j], v);
  return v;
}

// Phase 1: right-hand sides of positions [p0, p1) of one line (element i at
// L[i * S]), in place, C outputs per chunk from a window of C + 10 inputs
// carried in registers.  The first and the last five outputs of the range
// are parked in head / tail and written after a barrier, because the
// neighbouring warps read those inputs as their window ends.  Rows within 5
// of a line end use the one-sided rows of A (banmul_dev_z_c,
// bgprtm/FdEngine_cfd.cpp:304-327); A is the plan's copy in the
// kernel-parameter bank (uniform, runtime-indexed reads).  Requires p1 - p0
// to be a multiple of C unless p1 == n.
template <int S, int C>
__device__ __forceinline__ void cfd_rhs_range(const float (&a)[60], float *L, int n, int p0, int p1, float (&head)[5],
                                              float (&tail)[5]) {
  const RhsCoef rc{a[55], a[56], a[57], a[58], a[59]};
  float w[C + 10];
#pragma unroll
  for (int k = 0; k < 10; k++) {
    const int j = p0 - 5 + k;
    w[k] = (j >= 0 && j < n) ? L[j * S] : 0.f;
  }
  for (int i0 = p0; i0 < p1; i0 += C) {
    if (i0 + C + 5 <= n) {
#pragma unroll
      for (int k = 10; k < C + 10; k++) w[k] = L[(i0 - 5 + k) * S];
    } else {
#pragma unroll
      for (int k = 10; k < C + 10; k++) {
        const int j = i0 - 5 + k;
        w[k] = j < n ? L[j * S] : 0.f;
      }
    }
    float r[C];
    if (i0 >= 5 && i0 + C <= n - 5) {
#pragma unroll
      for (int k = 0; k < C; k++)
        r[k] = rhs_interior(rc, w[k], w[k + 1], w[k + 2], w[k + 3], w[k + 4], w[k + 6], w[k + 7], w[k + 8],
                            w[k + 9], w[k + 10]);
    } else {
#pragma unroll
      for (int k = 0; k < C; k++) {
        const int i = i0 + k;
        float v;
        if (i < 5) v = rhs_low(a, i, w + k);
        else if (i >= n - 5) v = rhs_high(a, n - i, w + k);
        else
          v = rhs_interior(rc, w[k], w[k + 1], w[k + 2], w[k + 3], w[k + 4], w[k + 6], w[k + 7], w[k + 8],
                           w[k + 9], w[k + 10]);
        r[k] = v;
      }
    }
    if (i0 != p0 && i0 + C < p1) {  // an inner chunk: no parked rows
#pragma unroll
      for (int k = 0; k < C; k++) L[(i0 + k) * S] = r[k];
    } else {
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
    }
#pragma unroll
    for (int k = 0; k < 10; k++) w[k] = w[k + C];
  }
}

// Phase 2, forward: y_i = rhs_i - l[i-4][3] y_{i-4} - l[i-3][2] y_{i-3}
// - l[i-2][1] y_{i-2} - l[i-1][0] y_{i-1}, oldest pivot first, with the
// row-packed multipliers lm[i] = (l[i-1][0], l[i-2][1], l[i-3][2], l[i-4][3]).
// Rows [b, e) in chunks of C from b, the next chunk prefetched; CST: the
// multipliers are the register constant mc; PART: the last chunk may run
// past e (= n), otherwise e - b is a multiple of C.
struct Chain {
  float y1, y2, y3, y4;
};

template <int S, int C, bool CST, bool PART>
__device__ __forceinline__ void fwd_region(const float4 *__restrict__ lm, float4 mc, float *L, int b, int e, int n,
                                           Chain &y) {
  if (b >= e) return;
  float rv[C];
  float4 m[C];
#pragma unroll
  for (int k = 0; k < C; k++) {
    const int i = PART ? min(b + k, n - 1) : b + k;
    rv[k] = L[i * S];
    if (!CST) m[k] = __ldg(lm + i);
  }
  for (int i0 = b; i0 < e; i0 += C) {
    const bool more = i0 + C < e;
    float nrv[C];
    float4 nm[C];
    if (more) {
#pragma unroll
      for (int k = 0; k < C; k++) {
        const int i = PART ? min(i0 + C + k, n - 1) : i0 + C + k;
        nrv[k] = L[i * S];
        if (!CST) nm[k] = __ldg(lm + i);
      }
    }
#pragma unroll
    for (int k = 0; k < C; k++) {
      const float4 c = CST ? mc : m[k];
      float r = rv[k];
      r = r - c.w * y.y4;
      r = r - c.z * y.y3;
      r = r - c.y * y.y2;
      r = r - c.x * y.y1;
      y.y4 = y.y3, y.y3 = y.y2, y.y2 = y.y1, y.y1 = r;
      rv[k] = r;
    }
    if (!PART || i0 + C <= e) {
#pragma unroll
      for (int k = 0; k < C; k++) L[(i0 + k) * S] = rv[k];
    } else {
#pragma unroll
      for (int k = 0; k < C; k++)
        if (i0 + k < e) L[(i0 + k) * S] = rv[k];
    }
    if (more) {
#pragma unroll
      for (int k = 0; k < C; k++) {
        rv[k] = nrv[k];
        if (!CST) m[k] = nm[k];
      }
    }
  }
}

// Phase 2, backward: f_i = (y_i - u3 f_{i+4} - u2 f_{i+3} - u1 f_{i+2}
// - u0 f_{i+1}) * (1 / pivot_i), the reciprocal pivots from the FP64 plan
// set-up; upper-factor entries beyond the line end are zero.  Rows hi down
// to lo in chunks of C; PART: the last chunk may run below lo (= 0).
template <int S, int C, bool CST, bool PART>
__device__ __forceinline__ void bwd_region(const float4 *__restrict__ bu4, const float *__restrict__ rd, float4 uc,
                                           float rc, float *L, int hi, int lo, Chain &z) {
  if (hi < lo) return;
  float yv[C], rv[C];
  float4 u[C];
#pragma unroll
  for (int k = 0; k < C; k++) {
    const int i = PART ? max(hi - k, 0) : hi - k;
    yv[k] = L[i * S];
    if (!CST) u[k] = __ldg(bu4 + i), rv[k] = __ldg(rd + i);
  }
  for (int t = hi; t >= lo; t -= C) {
    const bool more = t - C >= lo;
    float nyv[C], nrv[C];
    float4 nu[C];
    if (more) {
#pragma unroll
      for (int k = 0; k < C; k++) {
        const int i = PART ? max(t - C - k, 0) : t - C - k;
        nyv[k] = L[i * S];
        if (!CST) nu[k] = __ldg(bu4 + i), nrv[k] = __ldg(rd + i);
      }
    }
#pragma unroll
    for (int k = 0; k < C; k++) {
      const float4 c = CST ? uc : u[k];
      float v = yv[k];
      v = v - c.w * z.y4;
      v = v - c.z * z.y3;
      v = v - c.y * z.y2;
      v = v - c.x * z.y1;
      v = v * (CST ? rc : rv[k]);
      z.y4 = z.y3, z.y3 = z.y2, z.y2 = z.y1, z.y1 = v;
      yv[k] = v;
    }
    if (!PART || t - C + 1 >= lo) {
#pragma unroll
      for (int k = 0; k < C; k++) L[(t - k) * S] = yv[k];
    } else {
#pragma unroll
      for (int k = 0; k < C; k++)
        if (t - k >= lo) L[(t - k) * S] = yv[k];
    }
    if (more) {
#pragma unroll
      for (int k = 0; k < C; k++) {
        yv[k] = nyv[k];
        if (!CST) u[k] = nu[k], rv[k] = nrv[k];
      }
    }
  }
}

// Both recurrences of one line: table rows, the constant interior run
// [c0, c1] from registers, table rows again.
template <int S, int C>
__device__ __forceinline__ void cfd_solve(const CfdPlanDev &p, float *L, int n) {
  const float4 *__restrict__ lm = reinterpret_cast<const float4 *>(p.lm);
  const float4 *__restrict__ bu4 = reinterpret_cast<const float4 *>(p.bu);
  const float4 mc = make_float4(p.lmc[0], p.lmc[1], p.lmc[2], p.lmc[3]);
  const float4 uc = make_float4(p.buc[0], p.buc[1], p.buc[2], p.buc[3]);
  // forward chunks j cover [jC, jC + C - 1]; constant for ka <= j < kb
  int ka = (p.c0 + C - 1) / C, kb = (p.c1 + 1) / C;
  if (p.c0 > p.c1 || ka >= kb) ka = kb = 0;
  Chain y{0.f, 0.f, 0.f, 0.f};
  fwd_region<S, C, false, false>(lm, mc, L, 0, ka * C, n, y);
  fwd_region<S, C, true, false>(lm, mc, L, ka * C, kb * C, n, y);
  fwd_region<S, C, false, true>(lm, mc, L, kb * C, n, n, y);
  // backward chunks j cover [n - (j+1)C, n - 1 - jC]; constant for ja <= j < jb
  int ja = (n - 1 - p.c1 + C - 1) / C, jb = (n - p.c0) / C;
  if (p.c0 > p.c1 || ja >= jb) ja = jb = 0;
  Chain z{0.f, 0.f, 0.f, 0.f};
  bwd_region<S, C, false, false>(bu4, p.rdiag, uc, p.rdc, L, n - 1, n - ja * C, z);
  bwd_region<S, C, true, false>(bu4, p.rdiag, uc, p.rdc, L, n - 1 - ja * C, n - jb * C, z);
  bwd_region<S, C, false, true>(bu4, p.rdiag, uc, p.rdc, L, n - 1 - jb * C, 0, z);
}

// Phases 1 and 2 on a staged tile (element i of this lane's line at L[i*S]);
// entered after a barrier that follows the staging, leaves the tile final
// for this warp only (callers barrier before storing).
template <int S>
__device__ __forceinline__ void cfd_tile_compute(const CfdPlanDev &p, float *L, int n, int nl, int lane, int warp,
                                                 int nw) {
  // phase 1: right-hand sides, each warp a run of whole chunks of every line
  const int run = (((n + nw - 1) / nw) + kChunk - 1) / kChunk * kChunk;
  const int p0 = min(n, warp * run), p1 = min(n, p0 + run);
  float head[5], tail[5];
  if (lane < nl && p0 < p1) cfd_rhs_range<S, kChunk>(p.a, L, n, p0, p1, head, tail);
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
  if (warp == 0 && lane < nl) cfd_solve<S, kChunk>(p, L, n);
}

// 32 lines per CTA staged through shared memory; warp 0 walks the lines
// (lane = line), all warps move data.  x / y lines (STRIDED): element i of
// line l at base + l + i*es, smem [i][32]; z lines: line l at base + l*n + i,
// smem [l][n+1] (bank-conflict free), filled by asynchronous 4-byte copies.
// One HBM read and one write per cell.
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
    for (int l = warp; l < nl; l += nw) {
      const float *src = in + base + (long long)l * n;
      float *dst = sm + l * (n + 1);
#pragma unroll 4
      for (int i = lane; i < n; i += 32) cp_async4(dst + i, src + i);
    }
    cp_async_wait_all();
  }
  constexpr int S = STRIDED ? 32 : 1;
  __syncthreads();
  cfd_tile_compute<S>(p, STRIDED ? sm + lane : sm + lane * (n + 1), n, nl, lane, warp, nw);
  __syncthreads();
  if (STRIDED) {
    for (int i = warp; i < n; i += nw)
      if (lane < nl) __stcg(out + base + lane + (long long)i * es, sm[i * 32 + lane]);
  } else {
    for (int l = warp; l < nl; l += nw)
      for (int i = lane; i < n; i += 32) __stcg(out + base + (long long)l * n + i, sm[l * (n + 1) + i]);
  }
}

// x / y lines streamed through registers, no shared memory: lane = z line,
// one warp per 32 z of one line set (element i of a line at X[i * es]).
// Forward: the 11-point right-hand side (one-sided rows at both ends) fused
// with the elimination.  x arrives in chunks of C rows into a ring of R =
// D + 2 register slots (chunk c in slot c % R, prefetched D + 1 chunks
// ahead); the chunk loop is unrolled by R so every window read is a static
// register.  y is parked in `out` (L2-resident until read back).  Backward:
// y read back in reverse through a ring of D + 1 slots and overwritten by f'.
// Lanes past nz read a valid column and store nothing.  Arithmetic and its
// order are those of the staged kernels: the results are bitwise equal.
template <int D, typename Off>
__global__ void __launch_bounds__(128, 4) cfd_stream_k(const CfdPlanDev p, const float *__restrict__ in, float *out,
                                                       int nz, long long es, long long other_stride, long long ntask) {
  constexpr int C = kChunk, R = D + 2, RB = D + 1;
  const int lane = threadIdx.x & 31;
  const long long task = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (task >= ntask) return;
  const int nzc = (nz + 31) >> 5;
  const int izc = (int)(task % nzc);
  const long long o = task / nzc;
  const int iz = izc * 32 + lane;
  const bool act = iz < nz;
  const long long off = o * other_stride + min(iz, nz - 1);
  const float *X = in + off;
  float *Y = out + off;
  const Off e = (Off)es;
  const int n = p.n;
  const int nch = (n + C - 1) / C;
  const RhsCoef rhc{p.a[55], p.a[56], p.a[57], p.a[58], p.a[59]};

  // ---- right-hand sides of the one-sided end rows
  float rbf[5], rbb[5];
  {
    float xf[11], xb[11];
#pragma unroll
    for (int m = 0; m < 11; m++) xf[m] = __ldcs(X + (Off)m * e), xb[m] = __ldcs(X + (Off)(n - 11 + m) * e);
#pragma unroll
    for (int i = 0; i < 5; i++) {
      float v = 0.f;
#pragma unroll
      for (int j = 5 - i; j < 11; j++) v = __fmaf_rn(p.a[j * 5 + i], xf[i - 5 + j], v);
      rbf[i] = v;
    }
#pragma unroll
    for (int t = 5; t >= 1; t--) {
      float v = 0.f;
#pragma unroll
      for (int j = 0; j < t + 5; j++) v = __fmaf_rn(-p.a[t + 49 - 5 * j], xb[6 - t + j], v);
      rbb[5 - t] = v;
    }
  }

  // ---- forward: fused right-hand side + elimination
  const float4 *__restrict__ lm = reinterpret_cast<const float4 *>(p.lm);
  const float4 mc = make_float4(p.lmc[0], p.lmc[1], p.lmc[2], p.lmc[3]);
  int ka = (p.c0 + C - 1) / C, kb = (p.c1 + 1) / C;
  if (p.c0 > p.c1 || ka >= kb) ka = kb = 0;
  float xr[R][C];
  auto load_chunk = [&](float(&dst)[C], int c) {
#pragma unroll
    for (int k = 0; k < C; k++) {
      const int i = c * C + k;
      dst[k] = i < n ? __ldcs(X + (Off)i * e) : 0.f;
    }
  };
#pragma unroll
  for (int k = 0; k < C; k++) xr[R - 1][k] = 0.f;  // chunk -1
#pragma unroll
  for (int d = 0; d <= D; d++) load_chunk(xr[d], d);
  float y1 = 0.f, y2 = 0.f, y3 = 0.f, y4 = 0.f;
  for (int c0 = 0; c0 < nch; c0 += R) {
#pragma unroll
    for (int s = 0; s < R; s++) {
      const int c = c0 + s;
      if (c < nch) {
        const int sp = (s + R - 1) % R, sn = (s + 1) % R;
        // x at chunk-relative row q in [-5, C + 5)
        auto xa = [&](int q) -> float { return q < 0 ? xr[sp][C + q] : q < C ? xr[s][q] : xr[sn][q - C]; };
        const int i0 = c * C;
        const bool cst = c >= ka && c < kb;
        float4 m[C];
        if (!cst) {
#pragma unroll
          for (int k = 0; k < C; k++) m[k] = __ldg(lm + min(i0 + k, n - 1));
        }
        float r[C];
#pragma unroll
        for (int k = 0; k < C; k++)
          r[k] = rhs_interior(rhc, xa(k - 5), xa(k - 4), xa(k - 3), xa(k - 2), xa(k - 1), xa(k + 1), xa(k + 2),
                              xa(k + 3), xa(k + 4), xa(k + 5));
        if (i0 < 5 || i0 + C > n - 5) {
#pragma unroll
          for (int k = 0; k < C; k++) {
            const int i = i0 + k;
#pragma unroll
            for (int q = 0; q < 5; q++) {
              if (i == q) r[k] = rbf[q];
              if (i == n - 5 + q) r[k] = rbb[q];
            }
          }
        }
        // slot sp (chunk c - 1) is free now: chunk c + D + 1 goes there
        load_chunk(xr[sp], c + D + 1);
        if (cst) {
#pragma unroll
          for (int k = 0; k < C; k++) {
            float v = r[k];
            v = v - mc.w * y4;
            v = v - mc.z * y3;
            v = v - mc.y * y2;
            v = v - mc.x * y1;
            y4 = y3, y3 = y2, y2 = y1, y1 = v;
            r[k] = v;
          }
        } else {
#pragma unroll
          for (int k = 0; k < C; k++) {
            float v = r[k];
            v = v - m[k].w * y4;
            v = v - m[k].z * y3;
            v = v - m[k].y * y2;
            v = v - m[k].x * y1;
            y4 = y3, y3 = y2, y2 = y1, y1 = v;
            r[k] = v;
          }
        }
        if (act) {
#pragma unroll
          for (int k = 0; k < C; k++)
            if (i0 + k < n) __stcg(Y + (Off)(i0 + k) * e, r[k]);
        }
      }
    }
  }

  // ---- backward: chunks j cover rows n-1-jC down to n-(j+1)C
  const float4 *__restrict__ bu4 = reinterpret_cast<const float4 *>(p.bu);
  const float *__restrict__ rd = p.rdiag;
  const float4 uc = make_float4(p.buc[0], p.buc[1], p.buc[2], p.buc[3]);
  const float rc = p.rdc;
  int ja = (n - 1 - p.c1 + C - 1) / C, jb = (n - p.c0) / C;
  if (p.c0 > p.c1 || ja >= jb) ja = jb = 0;
  float yr[RB][C];
  auto load_back = [&](float(&dst)[C], int j) {
#pragma unroll
    for (int k = 0; k < C; k++) {
      const int i = n - 1 - j * C - k;
      dst[k] = i >= 0 ? __ldcg(Y + (Off)i * e) : 0.f;
    }
  };
#pragma unroll
  for (int d = 0; d < RB; d++) load_back(yr[d], d);
  float z1 = 0.f, z2 = 0.f, z3 = 0.f, z4 = 0.f;
  for (int j0 = 0; j0 < nch; j0 += RB) {
#pragma unroll
    for (int s = 0; s < RB; s++) {
      const int j = j0 + s;
      if (j < nch) {
        const int t = n - 1 - j * C;
        const bool cst = j >= ja && j < jb;
        float v[C];
#pragma unroll
        for (int k = 0; k < C; k++) v[k] = yr[s][k];
        load_back(yr[s], j + RB);
        if (cst) {
#pragma unroll
          for (int k = 0; k < C; k++) {
            float w = v[k];
            w = w - uc.w * z4;
            w = w - uc.z * z3;
            w = w - uc.y * z2;
            w = w - uc.x * z1;
            w = w * rc;
            z4 = z3, z3 = z2, z2 = z1, z1 = w;
            v[k] = w;
          }
        } else {
#pragma unroll
          for (int k = 0; k < C; k++) {
            const int i = max(t - k, 0);
            const float4 u = __ldg(bu4 + i);
            const float rr = __ldg(rd + i);
            float w = v[k];
            w = w - u.w * z4;
            w = w - u.z * z3;
            w = w - u.y * z2;
            w = w - u.x * z1;
            w = w * rr;
            z4 = z3, z3 = z2, z2 = z1, z1 = w;
            v[k] = w;
          }
        }
        if (act) {
#pragma unroll
          for (int k = 0; k < C; k++)
            if (t - k >= 0) __stcg(Y + (Off)(t - k) * e, v[k]);
        }
      }
    }
  }
}

// x / y lines with TMA tile moves: the 32 (z) x n tile arrives as nb boxes of
// R rows on one mbarrier and leaves as nb bulk tensor stores.  Rows past n in
// the last box and z >= nz are zero-filled on load and clipped on store.
// Shared memory: 128 B for the barrier, then the tile [nb*R][32].
template <int AXIS>
__global__ void __launch_bounds__(128) cfd_lines_tma_k(CfdPlanDev p, const __grid_constant__ CUtensorMap tin,
                                                       const __grid_constant__ CUtensorMap tout, int nz, int R, int nb,
                                                       int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smraw);
  float *sm = reinterpret_cast<float *>(smraw + 128);
  const int n = p.n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int iz0 = blockIdx.x * 32, o = blockIdx.y;
  const int nl = min(32, nz - iz0);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect_tx(bar, (uint32_t)nb * (uint32_t)R * 32u * 4u);
    for (int b = 0; b < nb; b++) {
      if (AXIS == DX) tma_load_3d(sm + (size_t)b * R * 32, &tin, bar, iz0, b * R, o);
      else tma_load_3d(sm + (size_t)b * R * 32, &tin, bar, iz0, o, b * R);
    }
  }
  const bool ok = __syncthreads_and(mbar_wait(bar, 0, err));
  if (!ok) return;
  cfd_tile_compute<32>(p, sm + lane, n, nl, lane, warp, nw);
  fence_proxy_async();
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int b = 0; b < nb; b++) {
      if (AXIS == DX) tma_store_3d(&tout, sm + (size_t)b * R * 32, iz0, b * R, o);
      else tma_store_3d(&tout, sm + (size_t)b * R * 32, iz0, o, b * R);
    }
    bulk_commit();
    bulk_wait_read();
  }
}

// Forward elimination with the right-hand side formed on the fly (one warp,
// lane = line, element i of the lane's line at L[i * S]): rows [b, e) in
// chunks of C; w carries the inputs x[b - 5 .. b + 4] in and x[e - 5 .. e + 4]
// out.  The inputs ahead of the elimination are still in place (row i + 5 is
// read before row i + 5 is overwritten), so no separate right-hand-side pass
// or barrier is needed; the rows are those of cfd_rhs_range and fwd_region
// (same roundings, same bits).  CST / PART as in fwd_region.
template <int S, int C, bool CST, bool PART>
__device__ __forceinline__ void fwd_rhs_region(const CfdPlanDev &p, const RhsCoef &rc, const float4 *__restrict__ lm,
                                               float4 mc, float *L, int b, int e, int n, float (&w)[10], Chain &y) {
  for (int i0 = b; i0 < e; i0 += C) {
    float x[C + 10];
#pragma unroll
    for (int k = 0; k < 10; k++) x[k] = w[k];
#pragma unroll
    for (int k = 10; k < C + 10; k++) {
      const int j = i0 - 5 + k;
      x[k] = j < n ? L[j * S] : 0.f;
    }
    float4 m[C];
    if (!CST) {
#pragma unroll
      for (int k = 0; k < C; k++) m[k] = __ldg(lm + min(i0 + k, n - 1));
    }
    float r[C];
#pragma unroll
    for (int k = 0; k < C; k++)
      r[k] = rhs_interior(rc, x[k], x[k + 1], x[k + 2], x[k + 3], x[k + 4], x[k + 6], x[k + 7], x[k + 8], x[k + 9],
                          x[k + 10]);
    if (i0 < 5 || i0 + C > n - 5) {
#pragma unroll
      for (int k = 0; k < C; k++) {
        const int i = i0 + k;
        if (i < 5) r[k] = rhs_low(p.a, i, x + k);
        else if (i >= n - 5 && i < n) r[k] = rhs_high(p.a, n - i, x + k);
      }
    }
#pragma unroll
    for (int k = 0; k < C; k++) {
      const float4 c = CST ? mc : m[k];
      float v = r[k];
      v = v - c.w * y.y4;
      v = v - c.z * y.y3;
      v = v - c.y * y.y2;
      v = v - c.x * y.y1;
      y.y4 = y.y3, y.y3 = y.y2, y.y2 = y.y1, y.y1 = v;
      r[k] = v;
    }
    if (!PART || i0 + C <= e) {
#pragma unroll
      for (int k = 0; k < C; k++) L[(i0 + k) * S] = r[k];
    } else {
#pragma unroll
      for (int k = 0; k < C; k++)
        if (i0 + k < e) L[(i0 + k) * S] = r[k];
    }
#pragma unroll
    for (int k = 0; k < 10; k++) w[k] = x[k + C];
  }
}

// Both recurrences of one line with the right-hand side fused into the
// forward pass (cfd_solve's regions and backward pass)
template <int S, int C>
__device__ __forceinline__ void cfd_solve_fused(const CfdPlanDev &p, float *L, int n) {
  const float4 *__restrict__ lm = reinterpret_cast<const float4 *>(p.lm);
  const float4 *__restrict__ bu4 = reinterpret_cast<const float4 *>(p.bu);
  const float4 mc = make_float4(p.lmc[0], p.lmc[1], p.lmc[2], p.lmc[3]);
  const float4 uc = make_float4(p.buc[0], p.buc[1], p.buc[2], p.buc[3]);
  const RhsCoef rc{p.a[55], p.a[56], p.a[57], p.a[58], p.a[59]};
  int ka = (p.c0 + C - 1) / C, kb = (p.c1 + 1) / C;
  if (p.c0 > p.c1 || ka >= kb) ka = kb = 0;
  float w[10];
#pragma unroll
  for (int k = 0; k < 10; k++) w[k] = (k >= 5 && k - 5 < n) ? L[(k - 5) * S] : 0.f;
  Chain y{0.f, 0.f, 0.f, 0.f};
  fwd_rhs_region<S, C, false, false>(p, rc, lm, mc, L, 0, ka * C, n, w, y);
  fwd_rhs_region<S, C, true, false>(p, rc, lm, mc, L, ka * C, kb * C, n, w, y);
  fwd_rhs_region<S, C, false, true>(p, rc, lm, mc, L, kb * C, n, n, w, y);
  int ja = (n - 1 - p.c1 + C - 1) / C, jb = (n - p.c0) / C;
  if (p.c0 > p.c1 || ja >= jb) ja = jb = 0;
  Chain z{0.f, 0.f, 0.f, 0.f};
  bwd_region<S, C, false, false>(bu4, p.rdiag, uc, p.rdc, L, n - 1, n - ja * C, z);
  bwd_region<S, C, true, false>(bu4, p.rdiag, uc, p.rdc, L, n - 1 - ja * C, n - jb * C, z);
  bwd_region<S, C, false, true>(bu4, p.rdiag, uc, p.rdc, L, n - 1 - jb * C, 0, z);
}

// Pipelined persistent x / y line solves.  One CTA per SM walks the tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... (tile = 32 z lines of one y (x
// lines) or x (y lines) column) through a ring of nbuf shared-memory tile
// buffers.  Warp nbuf - 1 is the producer: its lane 0 loads tile j into
// buffer j % nbuf by TMA, and once the worker of tile j - nbuf has released
// that buffer stores its result by TMA and loads the next tile into it.
// Warps 0 .. nbuf - 2 are workers: worker w takes tiles w, w + nbuf - 1, ...
// and runs both recurrences with the right-hand side fused into the forward
// pass, so a worker goes from one loaded tile to the next without waiting on
// a load or a store.  Barriers full[b] (TMA bytes landed) and done[b] (the
// worker's writes fenced to the async proxy) alternate parity per reuse of
// buffer b; every wait is bounded and raises *err.
template <int AXIS>
__global__ void __launch_bounds__(256, 1) cfd_pipe_k(CfdPlanDev p, const __grid_constant__ CUtensorMap tin,
                                                     const __grid_constant__ CUtensorMap tout, int nz, int nzt,
                                                     long long ntiles, int R, int nb, int nbuf, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smraw);
  uint64_t *done = full + 8;
  float *buf = reinterpret_cast<float *>(smraw + 128);
  const int n = p.n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwork = nbuf - 1;
  const size_t tile = (size_t)nb * R * 32;
  const long long G = gridDim.x;
  const int J = (int)((ntiles - blockIdx.x + G - 1) / G);
  if (threadIdx.x == 0) {
    for (int b = 0; b < nbuf; b++) mbar_init(full + b, 1), mbar_init(done + b, 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto coords = [&](int j, int &iz0, int &o) {
    const long long t = blockIdx.x + (long long)j * G;
    iz0 = (int)(t % nzt) * 32;
    o = (int)(t / nzt);
  };
  if (warp == nwork) {
    if (lane != 0) return;
    int loaded = 0;  // tiles whose loads were issued
    bool ok = true;
    for (int j = 0; j < J + nbuf && ok; j++) {
      const int b = j % nbuf;
      float *sb = buf + (size_t)b * tile;
      if (j >= nbuf) {
        const int jd = j - nbuf;
        if (jd >= J) continue;
        ok = mbar_wait(done + b, (uint32_t)(jd / nbuf) & 1u, err);
        if (!ok) break;
        int iz0, o;
        coords(jd, iz0, o);
        for (int q = 0; q < nb; q++) {
          if (AXIS == DX) tma_store_3d(&tout, sb + (size_t)q * R * 32, iz0, q * R, o);
          else tma_store_3d(&tout, sb + (size_t)q * R * 32, iz0, o, q * R);
        }
        bulk_commit();
        bulk_wait_read();
      }
      if (j < J) {
        int iz0, o;
        coords(j, iz0, o);
        mbar_expect_tx(full + b, (uint32_t)tile * 4u);
        for (int q = 0; q < nb; q++) {
          if (AXIS == DX) tma_load_3d(sb + (size_t)q * R * 32, &tin, full + b, iz0, q * R, o);
          else tma_load_3d(sb + (size_t)q * R * 32, &tin, full + b, iz0, o, q * R);
        }
        loaded = j + 1;
      }
    }
    if (!ok) {
      // loads issued for tiles no worker consumed must land before exit
      for (int j = max(0, loaded - nbuf); j < loaded; j++) mbar_drain(full + j % nbuf, (uint32_t)(j / nbuf) & 1u);
    }
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    return;
  }
  for (int j = warp; j < J; j += nwork) {
    const int b = j % nbuf;
    if (!mbar_wait(full + b, (uint32_t)(j / nbuf) & 1u, err)) break;
    int iz0, o;
    coords(j, iz0, o);
    const int nl = min(32, nz - iz0);
    if (lane < nl) cfd_solve_fused<32, kChunk>(p, buf + (size_t)b * tile + lane, n);
    fence_proxy_async();
    __syncwarp();
    if (lane == 0) mbar_arrive(done + b);
  }
}

// Cell regions of the pointwise epilogues.  The PML cells form six disjoint
// boxes (y bands over the whole xz plane, x bands inside the y interior, z
// bands inside both); the rest is the interior box.  Each box is one launch
// of a 3-D grid: interior cells run without PML code, PML cells gather every
// PML memory value of the cell first (pml1_all).
struct EpiBox {
  int z0, z1, x0, x1, y0, y1;
};

// density division and VTI / TTI scaling of one cell's gradients after PML
// round 1 (KernelCPU::ScalarVTI / ScalarTTI), every rounding explicit so that
// each kernel inlining it gives the same bits
__device__ __forceinline__ void grad_finish(const CfdGradEpiArgs &a, bool do_y, float &gx, float &gy, float &gz,
                                            float ep, float dl, float ax, float ay, float r) {
  if (a.rho) divide_rho(r, do_y, gx, gy, gz);
  if (a.model == 3) aniso_scale<3>(make_float4(ep, dl, ax, ay), gx, gy, gz);
  else if (a.model == 2) aniso_scale<2>(make_float4(ep, dl, 0.f, 0.f), gx, gy, gz);
}

// PML round 1 + VTI / TTI scaling of the raw gradients of one cell, in place
// (pml1 on each component, then grad_finish)
template <bool PML, int MASK>
__device__ __forceinline__ void grad_cell(const CfdGradEpiArgs &a, const Grid3 &g, int ix, int iy, int iz) {
  const bool do_y = a.ny > 1;
  const long long i = (long long)iy * g.nxz + (long long)ix * a.nz + iz;
  float gx = a.gx[i], gy = do_y ? a.gy[i] : 0.f, gz = a.gz[i];
  float ep = 0.f, dl = 0.f, ax = 0.f, ay = 0.f;
  if (a.model >= 2) ep = __ldg(a.eps + i), dl = __ldg(a.del + i);
  if (a.model == 3) ax = __ldg(a.pjx + i), ay = do_y ? __ldg(a.pjy + i) : 0.f;
  if (PML) pml1_all<0, MASK>(a.pml, g, a.pml3d, do_y, ix, iy, iz, gz, gx, gy);
  grad_finish(a, do_y, gx, gy, gz, ep, dl, ax, ay, a.rho ? __ldg(a.rho + i) : 0.f);
  a.gz[i] = gz;
  a.gx[i] = gx;
  if (do_y) a.gy[i] = gy;
}

// accumulation w0 - vel (dx + dz + dy) (with density in the engine's form)
// and the update of MODE 0 (none) or 1 (leapfrog)
template <int MODE>
__device__ __forceinline__ float div_finish(const CfdDivEpiArgs &a, float dxv, float dyv, float dzv, float vel,
                                            float w0, float w1, float r) {
  float t;
  if (a.rho) {
    t = a.rho_form == 2   ? div_accumulate_rho<2>(w0, vel, r, dxv, dzv, dyv)
        : a.rho_form == 1 ? div_accumulate_rho<1>(w0, vel, r, dxv, dzv, dyv)
                          : div_accumulate_rho<0>(w0, vel, r, dxv, dzv, dyv);
  } else {
    t = __fmaf_rn(-dxv, vel, w0);
    t = __fmaf_rn(-dzv, vel, t);
    t = __fmaf_rn(-dyv, vel, t);
  }
  return MODE == 1 ? __fsub_rn(__fadd_rn(w1, w1), t) : t;
}

// PML round 2 on the raw divergence parts of one cell, then
// w0 = w0 - vel (dx + dz + dy) followed by the leapfrog / Q update of MODE
// (KernelCPU::applyVel_minus + Propagator::update2nd).
template <bool PML, int MASK, int MODE>
__device__ __forceinline__ void div_cell(const CfdDivEpiArgs &a, const Grid3 &g, int ix, int iy, int iz) {
  const bool do_y = a.ny > 1 && a.dy;
  const long long i = (long long)iy * g.nxz + (long long)ix * a.nz + iz;
  float dxv = a.dx[i], dyv = do_y ? a.dy[i] : 0.f, dzv = a.dz[i];
  const float vel = __ldg(a.vel + i);
  const float w0 = a.w0[i];
  const float w1 = MODE != 0 ? __ldg(a.w1 + i) : 0.f;
  if (PML) pml1_all<1, MASK>(a.pml, g, a.pml3d, do_y, ix, iy, iz, dzv, dxv, dyv);
  const float r = a.rho ? __ldg(a.rho + i) : 0.f;
  float out;
  if (MODE == 2) out = q_update(a.q, i, g.nxz * a.ny, div_finish<0>(a, dxv, dyv, dzv, vel, w0, w1, r), w1);
  else out = div_finish<MODE>(a, dxv, dyv, dzv, vel, w0, w1, r);
  a.w0[i] = out;
}

// 32 z lines of `in` (line l at l * n) staged through shared memory [l][n + 1]
// and solved in place (cfd_lines_k's z path); returns the lines in the tile
__device__ __forceinline__ int zlines_solve(const CfdPlanDev &p, const float *__restrict__ in, float *sm,
                                            long long nlines) {
  const int n = p.n, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const long long l0 = (long long)blockIdx.x * 32;
  const int nl = (int)min(32LL, nlines - l0);
  for (int l = warp; l < nl; l += nw) {
    const float *src = in + (l0 + l) * n;
    float *dst = sm + l * (n + 1);
#pragma unroll 4
    for (int i = lane; i < n; i += 32) cp_async4(dst + i, src + i);
  }
  cp_async_wait_all();
  __syncthreads();
  cfd_tile_compute<1>(p, sm + lane * (n + 1), n, nl, lane, warp, nw);
  __syncthreads();
  return nl;
}

constexpr int kZfU = 4;  // cells per lane whose loads are in flight together

// The z line solve of the gradient pass fused with the gradient epilogue of
// the interior box (no PML cell): the raw z gradient of the tile's 32 lines
// stays in shared memory while every interior cell of those lines takes the
// density division and the VTI / TTI scaling with the raw x / y gradients of
// the earlier line solves (grad_cell's arithmetic: the same bits as the
// separate z solve and epilogue launches).  PML cells get their raw z
// gradient stored for the six PML face-box launches that follow.  A warp
// takes whole lines; each lane kZfU cells 32 apart, all loads issued before
// any store.
__global__ void __launch_bounds__(128) cfd_zgrad_k(CfdPlanDev p, const float *__restrict__ in, CfdGradEpiArgs a,
                                                   EpiBox ib, long long nlines) {
  extern __shared__ float sm[];
  const int nl = zlines_solve(p, in, sm, nlines);
  const int n = p.n, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const bool do_y = a.ny > 1;
  for (int l = warp; l < nl; l += nw) {
    const long long line = (long long)blockIdx.x * 32 + l;
    const int ix = (int)(line % a.nx), iy = (int)(line / a.nx);
    const bool xy_in = ix >= ib.x0 && ix < ib.x1 && iy >= ib.y0 && iy < ib.y1;
    const long long base = line * n;
    const float *zs = sm + l * (n + 1);
    for (int iz0 = lane; iz0 < n; iz0 += 32 * kZfU) {
      float gx[kZfU], gy[kZfU], ep[kZfU], dl[kZfU], ax[kZfU], ay[kZfU], r[kZfU];
#pragma unroll
      for (int u = 0; u < kZfU; u++) {
        const int iz = iz0 + 32 * u;
        const long long i = base + iz;
        gx[u] = gy[u] = ep[u] = dl[u] = ax[u] = ay[u] = r[u] = 0.f;
        if (iz < n && xy_in && iz >= ib.z0 && iz < ib.z1) {
          gx[u] = a.gx[i];
          if (do_y) gy[u] = a.gy[i];
          if (a.model >= 2) ep[u] = __ldg(a.eps + i), dl[u] = __ldg(a.del + i);
          if (a.model == 3) ax[u] = __ldg(a.pjx + i), ay[u] = do_y ? __ldg(a.pjy + i) : 0.f;
          if (a.rho) r[u] = __ldg(a.rho + i);
        }
      }
#pragma unroll
      for (int u = 0; u < kZfU; u++) {
        const int iz = iz0 + 32 * u;
        if (iz >= n) continue;
        const long long i = base + iz;
        float gz = zs[iz];
        if (xy_in && iz >= ib.z0 && iz < ib.z1) {
          grad_finish(a, do_y, gx[u], gy[u], gz, ep[u], dl[u], ax[u], ay[u], r[u]);
          a.gx[i] = gx[u];
          if (do_y) a.gy[i] = gy[u];
        }
        a.gz[i] = gz;
      }
    }
  }
}

// The z line solve of the divergence pass fused with the divergence epilogue
// of the interior box (accumulation and update of MODE 0 / 1; div_cell's
// arithmetic).  PML cells get their raw z part stored in a.dz for the PML
// face-box launches.
template <int MODE>
__global__ void __launch_bounds__(128) cfd_zdiv_k(CfdPlanDev p, const float *__restrict__ in, CfdDivEpiArgs a,
                                                  EpiBox ib, long long nlines) {
  extern __shared__ float sm[];
  const int nl = zlines_solve(p, in, sm, nlines);
  const int n = p.n, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const bool do_y = a.ny > 1 && a.dy;
  float *dz_raw = const_cast<float *>(a.dz);
  for (int l = warp; l < nl; l += nw) {
    const long long line = (long long)blockIdx.x * 32 + l;
    const int ix = (int)(line % a.nx), iy = (int)(line / a.nx);
    const bool xy_in = ix >= ib.x0 && ix < ib.x1 && iy >= ib.y0 && iy < ib.y1;
    const long long base = line * n;
    const float *zs = sm + l * (n + 1);
    for (int iz0 = lane; iz0 < n; iz0 += 32 * kZfU) {
      float dxv[kZfU], dyv[kZfU], vel[kZfU], w0[kZfU], w1[kZfU], r[kZfU];
#pragma unroll
      for (int u = 0; u < kZfU; u++) {
        const int iz = iz0 + 32 * u;
        const long long i = base + iz;
        dxv[u] = dyv[u] = vel[u] = w0[u] = w1[u] = r[u] = 0.f;
        if (iz < n && xy_in && iz >= ib.z0 && iz < ib.z1) {
          dxv[u] = a.dx[i];
          if (do_y) dyv[u] = a.dy[i];
          vel[u] = __ldg(a.vel + i);
          w0[u] = a.w0[i];
          if (MODE != 0) w1[u] = __ldg(a.w1 + i);
          if (a.rho) r[u] = __ldg(a.rho + i);
        }
      }
#pragma unroll
      for (int u = 0; u < kZfU; u++) {
        const int iz = iz0 + 32 * u;
        if (iz >= n) continue;
        const long long i = base + iz;
        if (xy_in && iz >= ib.z0 && iz < ib.z1) a.w0[i] = div_finish<MODE>(a, dxv[u], dyv[u], zs[iz], vel[u], w0[u], w1[u], r[u]);
        else dz_raw[i] = zs[iz];
      }
    }
  }
}

// one box: block (32 z, 8 x), grid (z tiles, x tiles, y count) from (z0, x0, y0);
// MASK (bit 2*d + s) lists the PML faces that can hold the box's cells
template <bool PML, int MASK>
__global__ void __launch_bounds__(256) cfd_grad_box_k(CfdGradEpiArgs a, EpiBox b) {
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  const int iz = b.z0 + blockIdx.x * 32 + threadIdx.x, ix = b.x0 + blockIdx.y * 8 + threadIdx.y, iy = b.y0 + blockIdx.z;
  if (iz < b.z1 && ix < b.x1) grad_cell<PML, MASK>(a, g, ix, iy, iz);
}
template <bool PML, int MASK, int MODE>
__global__ void __launch_bounds__(256) cfd_div_box_k(CfdDivEpiArgs a, EpiBox b) {
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  const int iz = b.z0 + blockIdx.x * 32 + threadIdx.x, ix = b.x0 + blockIdx.y * 8 + threadIdx.y, iy = b.y0 + blockIdx.z;
  if (iz < b.z1 && ix < b.x1) div_cell<PML, MASK, MODE>(a, g, ix, iy, iz);
}

// face masks of the PML boxes: y band (its y face, any x / z face), x band
// (its x face, any z face), z band (its z face)
constexpr int kZL = 1 << (2 * DZ), kZH = 2 << (2 * DZ), kXL = 1 << (2 * DX), kXH = 2 << (2 * DX),
              kYL = 1 << (2 * DY), kYH = 2 << (2 * DY);
constexpr int kBoxMask[7] = {0, kYL | kXL | kXH | kZL | kZH, kYH | kXL | kXH | kZL | kZH, kXL | kZL | kZH,
                             kXH | kZL | kZH, kZL, kZH};

// interior box [0] and the six PML boxes [1..6] (kBoxMask order; empty boxes
// have z1 <= z0)
void epi_boxes(const PmlDev &P, int nx, int ny, int nz, EpiBox *out) {
  const int zl = min(P.f[DZ][0].w, nz), zh = min(P.f[DZ][1].w, nz - zl);
  const int xl = min(P.f[DX][0].w, nx), xh = min(P.f[DX][1].w, nx - xl);
  const int yl = min(P.f[DY][0].w, ny), yh = min(P.f[DY][1].w, ny - yl);
  out[0] = EpiBox{zl, nz - zh, xl, nx - xh, yl, ny - yh};
  out[1] = EpiBox{0, nz, 0, nx, 0, yl};
  out[2] = EpiBox{0, nz, 0, nx, ny - yh, ny};
  out[3] = EpiBox{0, nz, 0, xl, yl, ny - yh};
  out[4] = EpiBox{0, nz, nx - xh, nx, yl, ny - yh};
  out[5] = EpiBox{0, zl, xl, nx - xh, yl, ny - yh};
  out[6] = EpiBox{nz - zh, nz, xl, nx - xh, yl, ny - yh};
}

dim3 box_grid(const EpiBox &b) { return dim3((b.z1 - b.z0 + 31) / 32, (b.x1 - b.x0 + 7) / 8, b.y1 - b.y0); }
bool box_empty(const EpiBox &b) { return b.z1 <= b.z0 || b.x1 <= b.x0 || b.y1 <= b.y0; }

}  // namespace

void cfd_tma_box(int n, int *R, int *nb) {
  *nb = (n + 255) / 256;
  *R = (n + *nb - 1) / *nb;
}

void launch_cfd_deriv(int axis, const CfdPlanDev &p, const float *in, float *out, int nx, int ny, int nz,
                      const CUtensorMap *tin, const CUtensorMap *tout, int *err, cudaStream_t st) {
  const long long nxz = (long long)nx * nz;
  if (axis == DZ) {
    const long long nlines = (long long)nx * ny;
    const size_t smem = (size_t)32 * (nz + 1) * sizeof(float);
    cfd_lines_k<false><<<(unsigned)((nlines + 31) / 32), 128, smem, st>>>(p, in, out, nz, 1, 0, 0, nlines);
    return;
  }
  const int n = axis == DX ? nx : ny;
  dim3 grid((nz + 31) / 32, axis == DX ? ny : nx);
  if (tin && tout) {
    int R, nb;
    cfd_tma_box(n, &R, &nb);
    const size_t smem = 128 + (size_t)nb * R * 32 * sizeof(float);
    if (axis == DX) cfd_lines_tma_k<DX><<<grid, 128, smem, st>>>(p, *tin, *tout, nz, R, nb, err);
    else cfd_lines_tma_k<DY><<<grid, 128, smem, st>>>(p, *tin, *tout, nz, R, nb, err);
    return;
  }
  const size_t smem = (size_t)32 * n * sizeof(float);
  if (axis == DX) cfd_lines_k<true><<<grid, 128, smem, st>>>(p, in, out, nz, nz, nxz, ny, 0);
  else cfd_lines_k<true><<<grid, 128, smem, st>>>(p, in, out, nz, nxz, nz, nx, 0);
}

static int g_cfd_sms = 0;  // SM count of the device cfd_init ran on

bool launch_cfd_deriv_pipe(int axis, const CfdPlanDev &p, int nx, int ny, int nz, const CUtensorMap *tin,
                           const CUtensorMap *tout, int *err, cudaStream_t st) {
  const int n = axis == DX ? nx : ny;
  int R, nb;
  cfd_tma_box(n, &R, &nb);
  const size_t tile = (size_t)nb * R * 32 * sizeof(float);
  const int nbuf = (int)std::min<size_t>(8, (227 * 1024 - 128) / tile);
  if (nbuf < 3 || g_cfd_sms <= 0) return false;
  const int nzt = (nz + 31) / 32;
  const long long ntiles = (long long)nzt * (axis == DX ? ny : nx);
  const unsigned grid = (unsigned)std::min<long long>(ntiles, g_cfd_sms);
  const size_t smem = 128 + (size_t)nbuf * tile;
  if (axis == DX) cfd_pipe_k<DX><<<grid, nbuf * 32, smem, st>>>(p, *tin, *tout, nz, nzt, ntiles, R, nb, nbuf, err);
  else cfd_pipe_k<DY><<<grid, nbuf * 32, smem, st>>>(p, *tin, *tout, nz, nzt, ntiles, R, nb, nbuf, err);
  return true;
}

void launch_cfd_deriv_stream(int axis, const CfdPlanDev &p, const float *in, float *out, int nx, int ny, int nz,
                             cudaStream_t st) {
  const long long nxz = (long long)nx * nz;
  const long long ntask = (long long)((nz + 31) / 32) * (axis == DX ? ny : nx);
  const unsigned blocks = (unsigned)((ntask + 3) / 4);
  const long long es = axis == DX ? nz : nxz, other = axis == DX ? nxz : nz;
  // 32-bit element offsets along a line when they cannot overflow
  if ((long long)p.n * es < (1LL << 31)) cfd_stream_k<kStreamD, int><<<blocks, 128, 0, st>>>(p, in, out, nz, es, other, ntask);
  else cfd_stream_k<kStreamDWide, long long><<<blocks, 128, 0, st>>>(p, in, out, nz, es, other, ntask);
}

int cfd_init() {
  const int mx = 227 * 1024;
  bool ok = cudaFuncSetAttribute(cfd_lines_k<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute(cfd_lines_k<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute(cfd_lines_tma_k<DX>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute(cfd_lines_tma_k<DY>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute(cfd_pipe_k<DX>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute(cfd_pipe_k<DY>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute(cfd_zgrad_k, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute(cfd_zdiv_k<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute(cfd_zdiv_k<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  int dev = 0;
  ok = ok && cudaGetDevice(&dev) == cudaSuccess &&
       cudaDeviceGetAttribute(&g_cfd_sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess;
  return ok ? 0 : -1;
}

template <int K, typename F>
static void each_box(const EpiBox *bx, F &&f) {
  if constexpr (K < 7) {
    if (!box_empty(bx[K])) f(std::integral_constant<int, K>{});
    each_box<K + 1>(bx, f);
  }
}

// lo and hi layers of one dimension overlap (small grids): a cell of a band
// box can then also lie in the opposite face, so every box takes all faces
static bool pml_overlap(const PmlDev &P, int nx, int ny, int nz) {
  return P.f[DZ][0].w + P.f[DZ][1].w > nz || P.f[DX][0].w + P.f[DX][1].w > nx || P.f[DY][0].w + P.f[DY][1].w > ny;
}

void launch_cfd_grad_epilogue(const CfdGradEpiArgs &a, cudaStream_t st, bool pml_only) {
  EpiBox bx[7];
  epi_boxes(a.pml, a.nx, a.ny, a.nz, bx);
  if (pml_only) bx[0].z1 = bx[0].z0;
  const bool all = pml_overlap(a.pml, a.nx, a.ny, a.nz);
  each_box<0>(bx, [&](auto k) {
    constexpr int K = decltype(k)::value;
    const dim3 g = box_grid(bx[K]), block(32, 8);
    if (K > 0 && all) cfd_grad_box_k<true, 63><<<g, block, 0, st>>>(a, bx[K]);
    else cfd_grad_box_k<(K > 0), kBoxMask[K]><<<g, block, 0, st>>>(a, bx[K]);
  });
}

template <int K, int MODE>
static void div_box(const CfdDivEpiArgs &a, const EpiBox &b, bool all, cudaStream_t st) {
  const dim3 g = box_grid(b), block(32, 8);
  if (K > 0 && all) cfd_div_box_k<true, 63, MODE><<<g, block, 0, st>>>(a, b);
  else cfd_div_box_k<(K > 0), kBoxMask[K], MODE><<<g, block, 0, st>>>(a, b);
}

void launch_cfd_div_epilogue(const CfdDivEpiArgs &a, cudaStream_t st, bool pml_only) {
  EpiBox bx[7];
  epi_boxes(a.pml, a.nx, a.ny, a.nz, bx);
  if (pml_only) bx[0].z1 = bx[0].z0;
  const bool all = pml_overlap(a.pml, a.nx, a.ny, a.nz);
  each_box<0>(bx, [&](auto k) {
    constexpr int K = decltype(k)::value;
    if (a.mode == 0) div_box<K, 0>(a, bx[K], all, st);
    else if (a.mode == 1) div_box<K, 1>(a, bx[K], all, st);
    else div_box<K, 2>(a, bx[K], all, st);
  });
}

void launch_cfd_zgrad(const CfdPlanDev &p, const float *in, const CfdGradEpiArgs &a, cudaStream_t st) {
  const long long nlines = (long long)a.nx * a.ny;
  EpiBox bx[7];
  epi_boxes(a.pml, a.nx, a.ny, a.nz, bx);
  if (pml_overlap(a.pml, a.nx, a.ny, a.nz)) bx[0].z1 = bx[0].z0;  // every cell goes through the PML boxes
  cfd_zgrad_k<<<(unsigned)((nlines + 31) / 32), 128, (size_t)32 * (a.nz + 1) * sizeof(float), st>>>(p, in, a, bx[0],
                                                                                                     nlines);
  launch_cfd_grad_epilogue(a, st, true);
}

void launch_cfd_zdiv(const CfdPlanDev &p, const float *in, const CfdDivEpiArgs &a, cudaStream_t st) {
  const long long nlines = (long long)a.nx * a.ny;
  const unsigned grid = (unsigned)((nlines + 31) / 32);
  const size_t smem = (size_t)32 * (a.nz + 1) * sizeof(float);
  EpiBox bx[7];
  epi_boxes(a.pml, a.nx, a.ny, a.nz, bx);
  if (pml_overlap(a.pml, a.nx, a.ny, a.nz)) bx[0].z1 = bx[0].z0;
  if (a.mode == 0) cfd_zdiv_k<0><<<grid, 128, smem, st>>>(p, in, a, bx[0], nlines);
  else cfd_zdiv_k<1><<<grid, 128, smem, st>>>(p, in, a, bx[0], nlines);
  launch_cfd_div_epilogue(a, st, true);
}


// ============================================================================
// Segment-parallel line solves and the fused compact-FD step.
//
// A tile of 32 lines (lane = line) is cut along the line into nseg segments
// of seglen rows, one warp each.  Both recurrences are linear, so every warp
// runs both passes over its segment from zero incoming states (the particular
// solutions yp, then fp = the segment-local back substitution of yp), and the
// true values follow from the four values carried across each boundary:
//   S_j = (y_{b-1}, y_{b-2}, y_{b-3}, y_{b-4})   forward state entering segment j
//   T_j = (f_e, f_{e+1}, f_{e+2}, f_{e+3})       backward state entering it
//   f_i = fp_i + gb[i] . S_j + hb[i] . T_j
// hf[i] is the response of the forward recurrence to unit entering states,
// gb[i] the segment-local back substitution of those responses and hb[i] the
// response of the back substitution to unit entering states; all three are
// built once per axis on the host in FP64 from the device's FP32 factors
// (every line of an axis shares them).  The states follow from the segments'
// end values by two scans over the segments (one 4x4 step per segment):
//   S_{k+1}[m] = yp_{e_k-1-m} + hf[e_k-1-m] . S_k
//   T_{k-1}[m] = fp_{b_k+m} + gb[b_k+m] . S_k + hb[b_k+m] . T_k
// In exact arithmetic this is the sequential solve; in FP32 it differs from it
// by rounding only (the interior recurrences decay with ratios <= 0.9, so the
// corrections never amplify).  The right-hand sides are formed in place
// first (cfd_rhs_range, ends parked until the neighbours have read them).
// ============================================================================
namespace {

constexpr int kSegMax = 8;  // segments (warps) per tile

struct SegSmem {
  float endf[kSegMax][4][32];  // yp_{e-1} .. yp_{e-4} per segment and line
  float endb[kSegMax][4][32];  // fp_b .. fp_{b+3}
  float sin[kSegMax][4][32];   // S_j
};
constexpr size_t kSegHdr = 128 + sizeof(SegSmem);  // mbarrier slot + SegSmem, then the tile

__device__ __forceinline__ void seg_range(const CfdPlanDev &p, int j, int &b, int &e) {
  b = j * p.seglen;
  e = j == p.nseg - 1 ? p.n : b + p.seglen;
}

// Forward elimination over rows [b, e) from a zero incoming state, in place
// (b a multiple of the chunk).  On return (y1 .. y4) = (y_{e-1} .. y_{e-4}).
template <int S>
__device__ __forceinline__ void seg_fwd(const CfdPlanDev &p, float *L, int b, int e, Chain &y) {
  constexpr int C = kChunk;
  const float4 *__restrict__ lm = reinterpret_cast<const float4 *>(p.lm);
  const float4 mc = make_float4(p.lmc[0], p.lmc[1], p.lmc[2], p.lmc[3]);
  y = Chain{0.f, 0.f, 0.f, 0.f};
  float rv[C];
#pragma unroll
  for (int k = 0; k < C; k++) rv[k] = L[min(b + k, e - 1) * S];
  for (int i0 = b; i0 < e; i0 += C) {
    const bool more = i0 + C < e;
    float nrv[C];
    if (more) {
#pragma unroll
      for (int k = 0; k < C; k++) nrv[k] = L[min(i0 + C + k, e - 1) * S];
    }
    if (i0 >= p.c0 && i0 + C - 1 <= p.c1) {  // constant chunks are full (c1 < n)
#pragma unroll
      for (int k = 0; k < C; k++) {
        float v = rv[k];
        v = v - mc.w * y.y4;
        v = v - mc.z * y.y3;
        v = v - mc.y * y.y2;
        v = v - mc.x * y.y1;
        y.y4 = y.y3, y.y3 = y.y2, y.y2 = y.y1, y.y1 = v;
        rv[k] = v;
      }
    } else {
      float4 m[C];
#pragma unroll
      for (int k = 0; k < C; k++) m[k] = __ldg(lm + min(i0 + k, e - 1));
#pragma unroll
      for (int k = 0; k < C; k++) {
        if (i0 + k < e) {
          float v = rv[k];
          v = v - m[k].w * y.y4;
          v = v - m[k].z * y.y3;
          v = v - m[k].y * y.y2;
          v = v - m[k].x * y.y1;
          y.y4 = y.y3, y.y3 = y.y2, y.y2 = y.y1, y.y1 = v;
          rv[k] = v;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < C; k++)
      if (i0 + k < e) L[(i0 + k) * S] = rv[k];
    if (more) {
#pragma unroll
      for (int k = 0; k < C; k++) rv[k] = nrv[k];
    }
  }
}

// Back substitution over rows e-1 down to b from a zero incoming state, in
// place.  On return (z1 .. z4) = (f_b .. f_{b+3}).
template <int S>
__device__ __forceinline__ void seg_bwd(const CfdPlanDev &p, float *L, int b, int e, Chain &z) {
  constexpr int C = kChunk;
  const float4 *__restrict__ bu4 = reinterpret_cast<const float4 *>(p.bu);
  const float *__restrict__ rd = p.rdiag;
  const float4 uc = make_float4(p.buc[0], p.buc[1], p.buc[2], p.buc[3]);
  const float rc = p.rdc;
  z = Chain{0.f, 0.f, 0.f, 0.f};
  float yv[C];
#pragma unroll
  for (int k = 0; k < C; k++) yv[k] = L[max(e - 1 - k, b) * S];
  for (int t = e - 1; t >= b; t -= C) {
    const int tn = t - C;
    const bool more = tn >= b;
    float nyv[C];
    if (more) {
#pragma unroll
      for (int k = 0; k < C; k++) nyv[k] = L[max(tn - k, b) * S];
    }
    if (t - C + 1 >= b && t - C + 1 >= p.c0 && t <= p.c1) {
#pragma unroll
      for (int k = 0; k < C; k++) {
        float w = yv[k];
        w = w - uc.w * z.y4;
        w = w - uc.z * z.y3;
        w = w - uc.y * z.y2;
        w = w - uc.x * z.y1;
        w = w * rc;
        z.y4 = z.y3, z.y3 = z.y2, z.y2 = z.y1, z.y1 = w;
        yv[k] = w;
      }
    } else {
      float4 u[C];
      float rr[C];
#pragma unroll
      for (int k = 0; k < C; k++) {
        const int i = max(t - k, b);
        u[k] = __ldg(bu4 + i), rr[k] = __ldg(rd + i);
      }
#pragma unroll
      for (int k = 0; k < C; k++) {
        if (t - k >= b) {
          float w = yv[k];
          w = w - u[k].w * z.y4;
          w = w - u[k].z * z.y3;
          w = w - u[k].y * z.y2;
          w = w - u[k].x * z.y1;
          w = w * rr[k];
          z.y4 = z.y3, z.y3 = z.y2, z.y2 = z.y1, z.y1 = w;
          yv[k] = w;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < C; k++)
      if (t - k >= b) L[(t - k) * S] = yv[k];
    if (more) {
#pragma unroll
      for (int k = 0; k < C; k++) yv[k] = nyv[k];
    }
  }
}

__device__ __forceinline__ float dot4_acc(float v, const float4 &h, const float (&s)[4]) {
  v = v + h.x * s[0];
  v = v + h.y * s[1];
  v = v + h.z * s[2];
  v = v + h.w * s[3];
  return v;
}

// Right-hand sides and both particular recurrences of this warp's segment
// (warp < p.nseg; every thread of the CTA calls it), then the two scans:
// leaves fp in the tile and this segment's entering states in sv / tv.  The
// final value of row i is seg_final.
template <int S>
__device__ __forceinline__ void seg_solve(const CfdPlanDev &p, float *L, int lane, int warp, SegSmem &ss,
                                          float (&sv)[4], float (&tv)[4]) {
  int b, e;
  seg_range(p, warp, b, e);
  {
    float head[5], tail[5];
    cfd_rhs_range<S, kChunk>(p.a, L, p.n, b, e, head, tail);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 5; k++) L[(b + k) * S] = head[k];
    if ((e - b) % kChunk == 0) {
#pragma unroll
      for (int k = 0; k < 5; k++) L[(e - 5 + k) * S] = tail[k];
    }
  }
  {
    Chain y;
    seg_fwd<S>(p, L, b, e, y);
    ss.endf[warp][0][lane] = y.y1, ss.endf[warp][1][lane] = y.y2;
    ss.endf[warp][2][lane] = y.y3, ss.endf[warp][3][lane] = y.y4;
  }
  {
    Chain z;
    seg_bwd<S>(p, L, b, e, z);
    ss.endb[warp][0][lane] = z.y1, ss.endb[warp][1][lane] = z.y2;
    ss.endb[warp][2][lane] = z.y3, ss.endb[warp][3][lane] = z.y4;
  }
  __syncthreads();
  // forward scan up to this segment
  const float4 *__restrict__ hf = reinterpret_cast<const float4 *>(p.hf);
  sv[0] = sv[1] = sv[2] = sv[3] = 0.f;
  for (int k = 0; k < warp; k++) {
    const int ek = (k + 1) * p.seglen;
    float ns[4];
#pragma unroll
    for (int m = 0; m < 4; m++) ns[m] = dot4_acc(ss.endf[k][m][lane], __ldg(hf + ek - 1 - m), sv);
#pragma unroll
    for (int m = 0; m < 4; m++) sv[m] = ns[m];
  }
#pragma unroll
  for (int m = 0; m < 4; m++) ss.sin[warp][m][lane] = sv[m];
  __syncthreads();
  // backward scan down to this segment
  const float4 *__restrict__ gb = reinterpret_cast<const float4 *>(p.gb);
  const float4 *__restrict__ hb = reinterpret_cast<const float4 *>(p.hb);
  tv[0] = tv[1] = tv[2] = tv[3] = 0.f;
  for (int k = p.nseg - 1; k > warp; k--) {
    const int bk = k * p.seglen;
    float sk[4], nt[4];
#pragma unroll
    for (int m = 0; m < 4; m++) sk[m] = ss.sin[k][m][lane];
#pragma unroll
    for (int m = 0; m < 4; m++)
      nt[m] = dot4_acc(dot4_acc(ss.endb[k][m][lane], __ldg(gb + bk + m), sk), __ldg(hb + bk + m), tv);
#pragma unroll
    for (int m = 0; m < 4; m++) tv[m] = nt[m];
  }
}

// f_i = fp_i + gb[i] . S_j + hb[i] . T_j (the tables are zero where a
// segment has no entering state)
__device__ __forceinline__ float seg_final(const CfdPlanDev &p, int i, float fp, const float (&sv)[4],
                                           const float (&tv)[4]) {
  const float4 g = __ldg(reinterpret_cast<const float4 *>(p.gb) + i);
  const float4 h = __ldg(reinterpret_cast<const float4 *>(p.hb) + i);
  return dot4_acc(dot4_acc(fp, g, sv), h, tv);
}

// cells handled together by the epilogues (their PML memory in one round trip)
constexpr int kSegU = 4;

// Interior of the grid (cells in no PML layer): [lo, hi) per dimension.
struct PmlInterior {
  int x0, x1, y0, y1, z0, z1;
};
__device__ __forceinline__ PmlInterior pml_interior(const PmlDev &P, const Grid3 &g) {
  return PmlInterior{P.f[DX][0].w, g.nx - P.f[DX][1].w, P.f[DY][0].w, g.ny - P.f[DY][1].w,
                     P.f[DZ][0].w, g.nz - P.f[DZ][1].w};
}
// bit d set when coordinate c of dimension d lies in one of its PML layers
__device__ __forceinline__ int pml_bit(int d, int c, int lo, int hi) { return (c < lo || c >= hi) << d; }
__device__ __forceinline__ int pml_bits(const PmlInterior &in, int ix, int iy, int iz) {
  return pml_bit(DX, ix, in.x0, in.x1) | pml_bit(DY, iy, in.y0, in.y1) | pml_bit(DZ, iz, in.z0, in.z1);
}

// First-derivative PML round `round` on component AXIS of a batch of cells
// (dm: the layers that hold each cell, 0 = none); skipped when no cell of
// the thread's batch lies in a layer.
template <int AXIS, int U>
__device__ __forceinline__ void seg_pml(const CfdSegArgs &a, const Grid3 &g, int round, float (&v)[U],
                                        const int (&ix)[U], const int (&iy)[U], const int (&iz)[U],
                                        const int (&dm)[U]) {
  int any = 0;
#pragma unroll
  for (int u = 0; u < U; u++) any |= dm[u];
  if (!any) return;
  if (round) pml1_batch<AXIS, 1, U>(a.pml, g, a.pml3d, v, ix, iy, iz, dm);
  else pml1_batch<AXIS, 0, U>(a.pml, g, a.pml3d, v, ix, iy, iz, dm);
}

// Strided tile (x or y lines of 32 z columns, rows [0, n) at sm[i * 32 + lane])
// loaded by TMA boxes (R rows each, zero fill past the tensor) or by plain
// loads; false when the bounded wait gave up (the CTA then returns).
template <int AXIS, bool TMA>
__device__ __forceinline__ bool seg_load_strided(unsigned char *smraw, float *sm, const CUtensorMap *tin,
                                                 const float *in, long long base, long long es, int n, int nl, int iz0,
                                                 int o, int R, int nb, int *err) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (TMA) {
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw);
    if (threadIdx.x == 0) {
      mbar_init(bar, 1);
      mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      mbar_expect_tx(bar, (uint32_t)nb * (uint32_t)R * 32u * 4u);
      for (int b = 0; b < nb; b++) {
        if (AXIS == DX) tma_load_3d(sm + (size_t)b * R * 32, tin, bar, iz0, b * R, o);
        else tma_load_3d(sm + (size_t)b * R * 32, tin, bar, iz0, o, b * R);
      }
    }
    const bool ok = __syncthreads_and(mbar_wait(bar, 0, err));
    if (!ok && threadIdx.x == 0) mbar_drain(bar, 0);  // its own copies land before the CTA leaves
    return ok;
  }
  constexpr int U = 16;
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
  __syncthreads();
  return true;
}

// Z or X (or Y) line derivative with the first-derivative PML round `round` of
// that component: out = PML(D in).
template <int AXIS, bool TMA>
__global__ void __launch_bounds__(256, 2) cfd_seg_line_k(const CfdPlanDev p, const float *__restrict__ in,
                                                         float *__restrict__ out, const CfdSegArgs a,
                                                         const __grid_constant__ CUtensorMap tin, int round, int R,
                                                         int nb, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  SegSmem &ss = *reinterpret_cast<SegSmem *>(smraw + 128);
  float *sm = reinterpret_cast<float *>(smraw + kSegHdr);
  const int n = p.n, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  float sv[4], tv[4];
  int b, e;
  seg_range(p, warp, b, e);
  if (AXIS == DZ) {
    const long long nlines = (long long)a.nx * a.ny, l0 = (long long)blockIdx.x * 32;
    const int nl = (int)min(32LL, nlines - l0);
    const int st = n + 1;
    for (int l = warp; l < nl; l += nw) {
      const float *src = in + (l0 + l) * n;
      float *dst = sm + l * st;
#pragma unroll 4
      for (int i = lane; i < n; i += 32) cp_async4(dst + i, src + i);
    }
    cp_async_wait_all();
    __syncthreads();
    float *L = sm + lane * st;
    seg_solve<1>(p, L, lane, warp, ss, sv, tv);
    for (int i = b; i < e; i++) L[i] = seg_final(p, i, L[i], sv, tv);
    __syncthreads();
    constexpr int U = kSegU;
    const PmlInterior in = pml_interior(a.pml, g);
    for (int l = warp; l < nl; l += nw) {
      const long long line = l0 + l;
      const int ix = (int)(line % a.nx), iy = (int)(line / a.nx);
      const int fixed = pml_bit(DX, ix, in.x0, in.x1) | pml_bit(DY, iy, in.y0, in.y1);
      const float *row = sm + l * st;
      float *dst = out + line * n;
      for (int i0 = lane; i0 < n; i0 += 32 * U) {
        float v[U];
        int xs[U], ys[U], zs[U], dm[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const int i = i0 + 32 * u;
          v[u] = i < n ? row[i] : 0.f;
          xs[u] = ix, ys[u] = iy, zs[u] = min(i, n - 1);
          dm[u] = i < n ? fixed | pml_bit(DZ, i, in.z0, in.z1) : 0;
        }
        seg_pml<DZ, U>(a, g, round, v, xs, ys, zs, dm);
#pragma unroll
        for (int u = 0; u < U; u++)
          if (i0 + 32 * u < n) __stcg(dst + i0 + 32 * u, v[u]);
      }
    }
    return;
  }
  const int iz0 = blockIdx.x * 32, o = blockIdx.y;
  const int nl = min(32, a.nz - iz0);
  const long long es = AXIS == DX ? (long long)a.nz : g.nxz;
  const long long base = AXIS == DX ? (long long)o * g.nxz + iz0 : (long long)o * a.nz + iz0;
  if (!seg_load_strided<AXIS, TMA>(smraw, sm, &tin, in, base, es, n, nl, iz0, o, R, nb, err)) return;
  float *L = sm + lane;
  seg_solve<32>(p, L, lane, warp, ss, sv, tv);
  if (lane < nl) {
    constexpr int U = kSegU;
    const PmlInterior in = pml_interior(a.pml, g);
    // PML cells of the tile: all rows when its fixed coordinate or its z columns
    // reach a layer, else the rows in the layers of the line's own dimension
    const int iz = iz0 + lane;
    // layers holding the thread's fixed coordinates (the tile's y or x, its z)
    const int fixed = (AXIS == DX ? pml_bit(DY, o, in.y0, in.y1) : pml_bit(DX, o, in.x0, in.x1)) |
                      pml_bit(DZ, iz, in.z0, in.z1);
    const int r0 = AXIS == DX ? in.x0 : in.y0, r1 = AXIS == DX ? in.x1 : in.y1;
    for (int i0 = b; i0 < e; i0 += U) {
      float v[U];
      int xs[U], ys[U], zs[U], dm[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = min(i0 + u, e - 1);
        v[u] = seg_final(p, i, L[i * 32], sv, tv);
        xs[u] = AXIS == DX ? i : o, ys[u] = AXIS == DX ? o : i, zs[u] = iz;
        dm[u] = i0 + u < e ? fixed | pml_bit(AXIS, i, r0, r1) : 0;
      }
      seg_pml<AXIS, U>(a, g, round, v, xs, ys, zs, dm);
#pragma unroll
      for (int u = 0; u < U; u++)
        if (i0 + u < e) __stcg(out + base + lane + (long long)(i0 + u) * es, v[u]);
    }
  }
}

// The fused y kernel: y lines of w1 (x = o, 32 z columns).  Gradient pass:
// gy = Dy w1 with PML round 1; with the x / z gradients (already through
// their PML) each cell is divided by rho (KernelCPU::divideRho) and scaled
// (ScalarVTI / ScalarTTI); px, pz go back to global memory, py stays in the
// tile.  Divergence pass along y: dy = Dy py with PML round 2.
template <int MODEL, bool RHO, bool TMA>
__global__ void __launch_bounds__(256, 2) cfd_seg_yf_k(const CfdPlanDev pg, const CfdPlanDev pd, const CfdSegArgs a,
                                                       const __grid_constant__ CUtensorMap tin, int R, int nb,
                                                       int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  SegSmem &ss = *reinterpret_cast<SegSmem *>(smraw + 128);
  float *sm = reinterpret_cast<float *>(smraw + kSegHdr);
  const int n = pg.n, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  const int iz0 = blockIdx.x * 32, o = blockIdx.y;
  const int nl = min(32, a.nz - iz0);
  const long long es = g.nxz, base = (long long)o * a.nz + iz0;
  if (!seg_load_strided<DY, TMA>(smraw, sm, &tin, a.w1, base, es, n, nl, iz0, o, R, nb, err)) return;
  float *L = sm + lane;
  float sv[4], tv[4];
  seg_solve<32>(pg, L, lane, warp, ss, sv, tv);
  int b, e;
  seg_range(pg, warp, b, e);
  const int iz = iz0 + lane;
  constexpr int U = kSegU;
  const PmlInterior in = pml_interior(a.pml, g);
  const int fixed = pml_bit(DX, o, in.x0, in.x1) | pml_bit(DZ, iz, in.z0, in.z1);
  if (lane < nl) {
    for (int i0 = b; i0 < e; i0 += U) {
      float gx[U], gz[U], gy[U], r[U];
      float4 m[U];
      int xs[U], ys[U], zs[U], dm[U];
      bool act[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = min(i0 + u, e - 1);
        const long long c = base + lane + (long long)i * es;
        gx[u] = a.gx[c], gz[u] = a.gz[c];
        if (RHO) r[u] = __ldg(a.rho + c);
        if (MODEL >= 2) m[u].x = __ldg(a.eps + c), m[u].y = __ldg(a.del + c);
        if (MODEL == 3) m[u].z = __ldg(a.pjx + c), m[u].w = __ldg(a.pjy + c);
        gy[u] = seg_final(pg, i, L[i * 32], sv, tv);
        act[u] = i0 + u < e;
        xs[u] = o, ys[u] = i, zs[u] = iz;
        dm[u] = act[u] ? fixed | pml_bit(DY, i, in.y0, in.y1) : 0;
      }
      seg_pml<DY, U>(a, g, 0, gy, xs, ys, zs, dm);
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u;
        if (act[u]) {
          const long long c = base + lane + (long long)i * es;
          float x = gx[u], y = gy[u], z = gz[u];
          if (RHO) divide_rho(r[u], true, x, y, z);
          if (MODEL >= 2) aniso_scale<MODEL>(m[u], x, y, z);
          a.gx[c] = x, a.gz[c] = z;
          L[i * 32] = y;
        }
      }
    }
  }
  __syncthreads();
  seg_solve<32>(pd, L, lane, warp, ss, sv, tv);
  if (lane < nl) {
    for (int i0 = b; i0 < e; i0 += U) {
      float v[U];
      int xs[U], ys[U], zs[U], dm[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = min(i0 + u, e - 1);
        v[u] = seg_final(pd, i, L[i * 32], sv, tv);
        xs[u] = o, ys[u] = i, zs[u] = iz;
        dm[u] = i0 + u < e ? fixed | pml_bit(DY, i, in.y0, in.y1) : 0;
      }
      seg_pml<DY, U>(a, g, 1, v, xs, ys, zs, dm);
#pragma unroll
      for (int u = 0; u < U; u++)
        if (i0 + u < e) __stcg(a.dy + base + lane + (long long)(i0 + u) * es, v[u]);
    }
  }
}

// The fused x kernel: x lines of px (y = o, 32 z columns).  dx = Dx px with
// PML round 2; then w0 - vel dx, - vel dz, - vel dy (with rho: (d vel) rho for
// x and z, d (vel rho) for y, FdEngine_cfd::d{x,z,y}1_2D's forms) and the
// leapfrog / Q update of MODE.
template <int MODE, bool RHO, bool TMA>
__global__ void __launch_bounds__(256, 2) cfd_seg_xf_k(const CfdPlanDev p, const CfdSegArgs a,
                                                       const __grid_constant__ CUtensorMap tin, int R, int nb,
                                                       int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  SegSmem &ss = *reinterpret_cast<SegSmem *>(smraw + 128);
  float *sm = reinterpret_cast<float *>(smraw + kSegHdr);
  const int n = p.n, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const Grid3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.nz};
  const int iz0 = blockIdx.x * 32, o = blockIdx.y;
  const int nl = min(32, a.nz - iz0);
  const long long es = a.nz, base = (long long)o * g.nxz + iz0;
  if (!seg_load_strided<DX, TMA>(smraw, sm, &tin, a.gx, base, es, n, nl, iz0, o, R, nb, err)) return;
  float *L = sm + lane;
  float sv[4], tv[4];
  seg_solve<32>(p, L, lane, warp, ss, sv, tv);
  int b, e;
  seg_range(p, warp, b, e);
  const int iz = iz0 + lane;
  const long long ntot = g.nxz * a.ny;
  const PmlInterior in = pml_interior(a.pml, g);
  const int fixed = pml_bit(DY, o, in.y0, in.y1) | pml_bit(DZ, iz, in.z0, in.z1);
  if (lane < nl) {
    constexpr int U = kSegU;
    for (int i0 = b; i0 < e; i0 += U) {
      float dz[U], dy[U], vel[U], w0[U], w1[U], r[U], dxs[U];
      int xs[U], ys[U], zs[U], dm[U];
      bool act[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = min(i0 + u, e - 1);
        const long long c = base + lane + (long long)i * es;
        dz[u] = __ldcs(a.dz + c), dy[u] = __ldcs(a.dy + c);
        vel[u] = __ldg(a.vel + c), w0[u] = a.w0[c];
        if (MODE != 0) w1[u] = __ldg(a.w1 + c);
        if (RHO) r[u] = __ldg(a.rho + c);
        dxs[u] = seg_final(p, i, L[i * 32], sv, tv);
        act[u] = i0 + u < e;
        xs[u] = i, ys[u] = o, zs[u] = iz;
        dm[u] = act[u] ? fixed | pml_bit(DX, i, in.x0, in.x1) : 0;
      }
      seg_pml<DX, U>(a, g, 1, dxs, xs, ys, zs, dm);
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u;
        if (act[u]) {
          const long long c = base + lane + (long long)i * es;
          const float dx = dxs[u];
          float t;
          if (RHO) {
            t = div_accumulate_rho<0>(w0[u], vel[u], r[u], dx, dz[u], dy[u]);
          } else {
            t = div_accumulate(w0[u], vel[u], dx, dz[u], dy[u]);
          }
          float out;
          if (MODE == 0) out = t;
          else if (MODE == 1) out = (w1[u] + w1[u]) - t;
          else out = q_update(a.q, c, ntot, t, w1[u]);
          a.w0[c] = out;
        }
      }
    }
  }
}

size_t seg_smem_strided(int n, bool tma) {
  int R = n, nb = 1;
  if (tma) cfd_tma_box(n, &R, &nb);
  return kSegHdr + (size_t)nb * R * 32 * sizeof(float);
}
size_t seg_smem_z(int n) { return kSegHdr + (size_t)32 * (n + 1) * sizeof(float); }

}  // namespace

int cfd_seg_max_n(int axis) {
  const size_t cap = 227 * 1024;
  int n = 16;
  while (n < 8192 && (axis == DZ ? seg_smem_z(n + 1) : seg_smem_strided(n + 1, true)) <= cap &&
         (axis == DZ || seg_smem_strided(n + 1, false) <= cap))
    n++;
  return n;
}

int cfd_seg_init() {
  const int mx = 227 * 1024;
  bool ok = true;
  auto set = [&](const void *f) {
    ok = ok && cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  };
  set((const void *)cfd_seg_line_k<DZ, false>);
  set((const void *)cfd_seg_line_k<DX, false>);
  set((const void *)cfd_seg_line_k<DX, true>);
  set((const void *)cfd_seg_line_k<DY, false>);
  set((const void *)cfd_seg_line_k<DY, true>);
  set((const void *)cfd_seg_yf_k<1, false, false>), set((const void *)cfd_seg_yf_k<1, false, true>);
  set((const void *)cfd_seg_yf_k<1, true, false>), set((const void *)cfd_seg_yf_k<1, true, true>);
  set((const void *)cfd_seg_yf_k<2, false, false>), set((const void *)cfd_seg_yf_k<2, false, true>);
  set((const void *)cfd_seg_yf_k<2, true, false>), set((const void *)cfd_seg_yf_k<2, true, true>);
  set((const void *)cfd_seg_yf_k<3, false, false>), set((const void *)cfd_seg_yf_k<3, false, true>);
  set((const void *)cfd_seg_yf_k<3, true, false>), set((const void *)cfd_seg_yf_k<3, true, true>);
  set((const void *)cfd_seg_xf_k<0, false, false>), set((const void *)cfd_seg_xf_k<0, false, true>);
  set((const void *)cfd_seg_xf_k<0, true, false>), set((const void *)cfd_seg_xf_k<0, true, true>);
  set((const void *)cfd_seg_xf_k<1, false, false>), set((const void *)cfd_seg_xf_k<1, false, true>);
  set((const void *)cfd_seg_xf_k<1, true, false>), set((const void *)cfd_seg_xf_k<1, true, true>);
  set((const void *)cfd_seg_xf_k<2, false, false>), set((const void *)cfd_seg_xf_k<2, false, true>);
  set((const void *)cfd_seg_xf_k<2, true, false>), set((const void *)cfd_seg_xf_k<2, true, true>);
  return ok ? 0 : -1;
}

void launch_cfd_seg_line(int axis, int round, const CfdPlanDev &p, const float *in, float *out, const CfdSegArgs &a,
                         const CUtensorMap *tin, int *err, cudaStream_t st) {
  const dim3 block(32 * p.nseg);
  CUtensorMap none{};
  if (axis == DZ) {
    const long long nlines = (long long)a.nx * a.ny;
    cfd_seg_line_k<DZ, false><<<(unsigned)((nlines + 31) / 32), block, seg_smem_z(p.n), st>>>(p, in, out, a, none,
                                                                                               round, 0, 0, err);
    return;
  }
  const dim3 grid((a.nz + 31) / 32, axis == DX ? a.ny : a.nx);
  int R = p.n, nb = 1;
  if (tin) cfd_tma_box(p.n, &R, &nb);
  const size_t smem = seg_smem_strided(p.n, tin != nullptr);
  if (axis == DX) {
    if (tin) cfd_seg_line_k<DX, true><<<grid, block, smem, st>>>(p, in, out, a, *tin, round, R, nb, err);
    else cfd_seg_line_k<DX, false><<<grid, block, smem, st>>>(p, in, out, a, none, round, R, nb, err);
  } else {
    if (tin) cfd_seg_line_k<DY, true><<<grid, block, smem, st>>>(p, in, out, a, *tin, round, R, nb, err);
    else cfd_seg_line_k<DY, false><<<grid, block, smem, st>>>(p, in, out, a, none, round, R, nb, err);
  }
}

template <int MODEL, bool RHO>
static void yf_launch(const CfdPlanDev &pg, const CfdPlanDev &pd, const CfdSegArgs &a, const CUtensorMap *tin,
                      int *err, cudaStream_t st) {
  const dim3 grid((a.nz + 31) / 32, a.nx), block(32 * pg.nseg);
  int R = pg.n, nb = 1;
  if (tin) cfd_tma_box(pg.n, &R, &nb);
  const size_t smem = seg_smem_strided(pg.n, tin != nullptr);
  CUtensorMap none{};
  if (tin) cfd_seg_yf_k<MODEL, RHO, true><<<grid, block, smem, st>>>(pg, pd, a, *tin, R, nb, err);
  else cfd_seg_yf_k<MODEL, RHO, false><<<grid, block, smem, st>>>(pg, pd, a, none, R, nb, err);
}

void launch_cfd_seg_yfused(const CfdPlanDev &pg, const CfdPlanDev &pd, const CfdSegArgs &a, const CUtensorMap *tin,
                           int *err, cudaStream_t st) {
  const bool rho = a.rho != nullptr;
  if (a.model == 3) rho ? yf_launch<3, true>(pg, pd, a, tin, err, st) : yf_launch<3, false>(pg, pd, a, tin, err, st);
  else if (a.model == 2) rho ? yf_launch<2, true>(pg, pd, a, tin, err, st) : yf_launch<2, false>(pg, pd, a, tin, err, st);
  else rho ? yf_launch<1, true>(pg, pd, a, tin, err, st) : yf_launch<1, false>(pg, pd, a, tin, err, st);
}

template <int MODE, bool RHO>
static void xf_launch(const CfdPlanDev &p, const CfdSegArgs &a, const CUtensorMap *tin, int *err, cudaStream_t st) {
  const dim3 grid((a.nz + 31) / 32, a.ny), block(32 * p.nseg);
  int R = p.n, nb = 1;
  if (tin) cfd_tma_box(p.n, &R, &nb);
  const size_t smem = seg_smem_strided(p.n, tin != nullptr);
  CUtensorMap none{};
  if (tin) cfd_seg_xf_k<MODE, RHO, true><<<grid, block, smem, st>>>(p, a, *tin, R, nb, err);
  else cfd_seg_xf_k<MODE, RHO, false><<<grid, block, smem, st>>>(p, a, none, R, nb, err);
}

void launch_cfd_seg_xfused(const CfdPlanDev &p, const CfdSegArgs &a, const CUtensorMap *tin, int *err,
                           cudaStream_t st) {
  const bool rho = a.rho != nullptr;
  if (a.mode == 0) rho ? xf_launch<0, true>(p, a, tin, err, st) : xf_launch<0, false>(p, a, tin, err, st);
  else if (a.mode == 1) rho ? xf_launch<1, true>(p, a, tin, err, st) : xf_launch<1, false>(p, a, tin, err, st);
  else rho ? xf_launch<2, true>(p, a, tin, err, st) : xf_launch<2, false>(p, a, tin, err, st);
}

}  // namespace rtm
