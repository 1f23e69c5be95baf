// kernels_r2r_tc.cu - FFTWR2R line operators on the 5th-generation tensor
// cores (tcgen05, sm_100a).
//
// The FFTWR2R derivative of every z line is one fixed n x n matrix D applied
// to the line (FdEngine_r2r's transform, bin product and inverse transform,
// bgprtm/FdEngine_r2r.cpp; the matrix is built on the host in FP64):
//   out[l][j] = sum_k D[j][k] in[l][k],   l over the nx ny lines.
// As a GEMM, A = in ([lines][n], K-major), B = D ([n][n], K-major), and the
// accumulator tile [128 lines][n] lives in tensor memory (n <= 512 columns).
// FP32 accuracy comes from split TF32: x = x_hi + x_lo with x_hi the TF32
// rounding of x and x_lo the TF32 rounding of x - x_hi, and
//   A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi
// (three kind::tf32 MMAs into one FP32 accumulator; the dropped A_lo B_lo term
// is below 2^-22 of the product).  D is split once when the plans are made;
// the lines are split while they are staged.
//
// Per CTA: 128 lines; K in blocks of 16 through two shared-memory stages.  All
// 128 threads load a block (float4 loads, rows contiguous), split it and store
// hi / lo into the canonical no-swizzle K-major layout (8-row x 16-byte core
// matrices: rows of a core matrix 16 B apart, its two K halves of one MMA
// k-step 128 B apart (LBO), 8-row groups 256 B apart (SBO)); one thread issues
// the MMAs of the block and commits them to the stage's mbarrier, which the
// threads wait on before they refill that stage.  After the last block every
// warp reads its 32 accumulator lanes (tcgen05.ld 32x32b) and stores its lines.
// Every wait is bounded (2^16 polls, error flag); a CTA that gives up waits for
// its committed MMAs and frees its tensor memory before it returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "kernel_api.h"
#include "rtm_b200.h"
#include "tma.cuh"

namespace rtm {
namespace {

constexpr int kTcM = 128;   // lines per CTA (MMA M)
constexpr int kTcBK = 16;   // K per stage (two MMA k-steps of 8)
constexpr int kTcThreads = 128;

__device__ __forceinline__ uint32_t tf32_round(float x) {
  uint32_t r;
  asm("cvt.rn.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// shared-memory matrix descriptor, no swizzle, K-major (start, LBO, SBO in
// 16-byte units; descriptor version 1)
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor: D F32, A / B TF32, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t tf32_idesc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// byte offset of (row r, 4-float chunk q) of a [rows][16] block in the
// canonical layout: k-step q / 2 at (q / 2) rows 32 B, then 8-row groups
// (256 B), the k-step's two halves (128 B) and the row in the group (16 B)
__device__ __forceinline__ uint32_t kblock_off(int r, int q, int rows) {
  return (uint32_t)((q >> 1) * rows * 32 + (r >> 3) * 256 + (q & 1) * 128 + (r & 7) * 16);
}

}  // namespace

// out[l][j] = sum_k D[j][k] in[l][k] for the lines of this CTA; D given as its
// TF32 parts Dh, Dl ([n][n]); npad = n rounded up to 16
__global__ void __launch_bounds__(kTcThreads, 1)
    r2r_tc_z_k(const float *__restrict__ in, float *__restrict__ out, const float *__restrict__ Dh,
               const float *__restrict__ Dl, int n, int npad, long long M, int *err) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smraw);            // [2] stage MMA commits
  uint32_t *tslot = reinterpret_cast<uint32_t *>(smraw + 64);      // tensor-memory base
  unsigned char *ops = smraw + 1024;
  const uint32_t a_bytes = kTcM * kTcBK * 4, b_bytes = (uint32_t)npad * kTcBK * 4;
  const uint32_t stage_bytes = 2 * a_bytes + 2 * b_bytes;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long m0 = (long long)blockIdx.x * kTcM;
  const uint32_t ncols = npad <= 32 ? 32 : npad <= 64 ? 64 : npad <= 128 ? 128 : npad <= 256 ? 256 : 512;

  if (tid == 0) {
    mbar_init(bar, 1), mbar_init(bar + 1, 1);
    mbar_fence_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;

  const int nkb = (n + kTcBK - 1) / kTcBK;
  bool ok = true;
  int issued = 0;  // K blocks committed
  for (int kb = 0; kb < nkb && ok; kb++) {
    const int s = kb & 1;
    unsigned char *st = ops + (size_t)s * stage_bytes;
    // the MMAs of block kb - 2 read this stage
    if (kb >= 2) ok = __syncthreads_and(mbar_wait(bar + s, (uint32_t)((kb - 2) >> 1) & 1u, err));
    if (!ok) break;
    const int k0 = kb * kTcBK;
    // A: 128 rows x 4 chunks of 4 floats
    for (int idx = tid; idx < kTcM * 4; idx += kTcThreads) {
      const int r = idx >> 2, q = idx & 3, k = k0 + 4 * q;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (m0 + r < M && k < n) v = __ldcs(reinterpret_cast<const float4 *>(in + (m0 + r) * n + k));
      uint4 hi, lo;
      hi.x = tf32_round(v.x), hi.y = tf32_round(v.y), hi.z = tf32_round(v.z), hi.w = tf32_round(v.w);
      lo.x = tf32_round(v.x - __uint_as_float(hi.x)), lo.y = tf32_round(v.y - __uint_as_float(hi.y));
      lo.z = tf32_round(v.z - __uint_as_float(hi.z)), lo.w = tf32_round(v.w - __uint_as_float(hi.w));
      const uint32_t o = kblock_off(r, q, kTcM);
      *reinterpret_cast<uint4 *>(st + o) = hi;
      *reinterpret_cast<uint4 *>(st + a_bytes + o) = lo;
    }
    // B: npad rows of D x 4 chunks (rows >= n zero)
    for (int idx = tid; idx < npad * 4; idx += kTcThreads) {
      const int r = idx >> 2, q = idx & 3, k = k0 + 4 * q;
      float4 h = make_float4(0.f, 0.f, 0.f, 0.f), l = h;
      if (r < n && k < n) {
        h = __ldg(reinterpret_cast<const float4 *>(Dh + (long long)r * n + k));
        l = __ldg(reinterpret_cast<const float4 *>(Dl + (long long)r * n + k));
      }
      const uint32_t o = kblock_off(r, q, npad);
      *reinterpret_cast<float4 *>(st + 2 * a_bytes + o) = h;
      *reinterpret_cast<float4 *>(st + 2 * a_bytes + b_bytes + o) = l;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t sa = smem_u32(st);
      for (int ks = 0; ks < kTcBK / 8; ks++) {
        const uint32_t ah = sa + ks * kTcM * 32, al = ah + a_bytes;
        for (int h0 = 0; h0 < npad; h0 += 256) {
          const int nh = min(256, npad - h0);
          const uint32_t bh = sa + 2 * a_bytes + ks * npad * 32 + (h0 >> 3) * 256, bl = bh + b_bytes;
          const uint32_t idesc = tf32_idesc(nh), d = tbase + (uint32_t)h0;
          const uint32_t first = (kb == 0 && ks == 0) ? 0u : 1u;
          mma_tf32(d, kmajor_desc(ah, 128, 256), kmajor_desc(bh, 128, 256), idesc, first);
          mma_tf32(d, kmajor_desc(ah, 128, 256), kmajor_desc(bl, 128, 256), idesc, 1u);
          mma_tf32(d, kmajor_desc(al, 128, 256), kmajor_desc(bh, 128, 256), idesc, 1u);
        }
      }
      mma_commit(bar + s);
    }
    issued = kb + 1;
  }
  // every committed block done (the last commit covers all earlier MMAs)
  if (issued > 0) {
    const int kl = issued - 1;
    if (ok) ok = __syncthreads_and(mbar_wait(bar + (kl & 1), (uint32_t)(kl >> 1) & 1u, err));
    else mbar_drain(bar + (kl & 1), (uint32_t)(kl >> 1) & 1u);
  }
  tc_fence_after();
  if (ok) {
    const long long row = m0 + warp * 32 + lane;
    const uint32_t taddr = tbase + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < npad; c0 += 8) {
      uint32_t v[8];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                   : "r"(taddr + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
        float *o = out + row * n + c0;
        if (c0 + 4 <= n)
          __stcs(reinterpret_cast<float4 *>(o),
                 make_float4(__uint_as_float(v[0]), __uint_as_float(v[1]), __uint_as_float(v[2]), __uint_as_float(v[3])));
        if (c0 + 8 <= n)
          __stcs(reinterpret_cast<float4 *>(o + 4),
                 make_float4(__uint_as_float(v[4]), __uint_as_float(v[5]), __uint_as_float(v[6]), __uint_as_float(v[7])));
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(ncols) : "memory");
  }
}

namespace {
__global__ void tf32_split_k(const float *__restrict__ D, float *Dh, float *Dl, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float x = D[i];
    const uint32_t h = tf32_round(x);
    Dh[i] = __uint_as_float(h);
    Dl[i] = __uint_as_float(tf32_round(x - __uint_as_float(h)));
  }
}
}  // namespace

size_t r2r_tc_smem(int n) {
  const int npad = (n + 15) / 16 * 16;
  return 1024 + 2 * (2 * (size_t)kTcM * kTcBK * 4 + 2 * (size_t)npad * kTcBK * 4);
}

bool r2r_tc_supported(int n) { return n % 4 == 0 && n >= 16 && n <= 512 && r2r_tc_smem(n) <= 227 * 1024; }

int r2r_tc_init() {
  return cudaFuncSetAttribute(r2r_tc_z_k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) == cudaSuccess
             ? 0
             : -1;
}

void launch_tf32_split(const float *D, float *Dh, float *Dl, long long count, cudaStream_t st) {
  tf32_split_k<<<(unsigned)std::min<long long>((count + 255) / 256, 148LL * 8), 256, 0, st>>>(D, Dh, Dl, count);
}

void launch_r2r_tc_z(const float *in, float *out, const float *Dh, const float *Dl, int n, long long lines, int *err,
                     cudaStream_t st) {
  const int npad = (n + 15) / 16 * 16;
  const unsigned grid = (unsigned)((lines + kTcM - 1) / kTcM);
  r2r_tc_z_k<<<grid, kTcThreads, r2r_tc_smem(n), st>>>(in, out, Dh, Dl, n, npad, lines, err);
}

}  // namespace rtm
