// kernels_r2r_tc.cu - FFTWR2R line operators on the 5th-generation tensor
// cores (tcgen05, sm_100a).
//
// The FFTWR2R derivative along an axis is one fixed n x n matrix D applied to
// every line (FdEngine_r2r's transform, bin product and inverse transform,
// bgprtm/FdEngine_r2r.cpp; the matrix is built on the host in FP64):
//   z lines:  out[l][j] = sum_k D[j][k] in[l][k],  l over the nx ny lines
//   y lines:  out[j][c] = sum_k D[j][k] in[k][c],  c over the nx nz columns
//   x lines:  the y form per y plane, c over nz.
// As a GEMM D_acc[m][j] = sum_k A[m][k] B[j][k] with B = D (K-major) and
// A[m][k] the input: for z lines m is the line (k contiguous), for x / y
// lines m is the column c (m contiguous: each 16-byte copy brings 4 m of one
// k, and the split pass transposes them into the K-major layout).  The
// accumulator tile [128 m][n] lives in tensor memory (n <= 512 columns).
// FP32 accuracy comes from split TF32: x = x_hi + x_lo with x_hi the TF32
// rounding of x and x_lo the TF32 rounding of x - x_hi, and
//   A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi
// (three kind::tf32 MMAs into one FP32 accumulator; the dropped A_lo B_lo term
// is below 2^-22 of the product).  D is split once when the plans are made;
// the lines are split while they are staged.
//
// Per CTA: 128 m and all n output columns (at most 512 accumulator columns);
// K in blocks of 8 (one MMA k-step) through 2 to 6 shared-memory stages,
// each holding the raw A block, its hi / lo parts and
// the B block's hi / lo rows of the CTA's columns.  Operands sit in the
// canonical no-swizzle K-major layout (8-row x 16-byte core matrices: rows of
// a core matrix 16 B apart, the two K halves of one MMA k-step 128 B apart
// (LBO), 8-row groups 256 B apart (SBO)).  Warp roles, handing off through
// mbarriers only: warp 0 copies the raw A block by 16-byte cp.async
// (zero-filled past the grid; completion counted on the stage barrier) and
// the B rows by bulk copies from D's TF32 parts, pre-arranged in global
// memory in that layout; warps 1-2 split A into hi / lo; one thread of warp 3
// issues the MMAs and commits each stage back to the producer.  After the
// last block all four warps read their 32 accumulator lanes (tcgen05.ld
// 32x32b, 32 columns per load) and store.  Every wait is bounded (2^16
// polls, error flag); a CTA that gives up drains its committed MMAs and
// issued copies and frees its tensor memory before it returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "kernel_api.h"
#include "rtm_b200.h"
#include "tma.cuh"

namespace rtm {
namespace {

constexpr int kTcM = 128;   // lines per CTA (MMA M)
constexpr int kTcBK = 8;    // K per stage (one MMA k-step)
constexpr int kTcCh = kTcBK / 4;  // 16-byte chunks per row of a stage
static_assert(kTcM / 4 == 32, "an x / y tile's 4-m chunks map one to one onto a warp's lanes");
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

// 32 consecutive accumulator columns of the warp's 32 lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}

// byte offset of (row r, 4-float chunk q) of a [rows][16] block in the
// canonical layout: k-step q / 2 at (q / 2) rows 32 B, then 8-row groups
// (256 B), the k-step's two halves (128 B) and the row in the group (16 B)
__device__ __forceinline__ uint32_t kblock_off(int r, int q, int rows) {
  return (uint32_t)((q >> 1) * rows * 32 + (r >> 3) * 256 + (q & 1) * 128 + (r & 7) * 16);
}

}  // namespace

// geometry of one launch: MODE 0 `lines` lines along K; MODE 1 `total_m`
// values of m, element (m, k) at (m / group_m) group_stride + k ldk +
// m % group_m (x lines: groups = y planes of nz m; y lines: one group of nx nz
// m); group_m % 4 == 0, so a 16-byte run of 4 m never crosses a group
struct TcGeom {
  long long lines;
  long long ldk, group_stride, group_m, total_m;
};

// 16-byte asynchronous copy, zero-filled when src_bytes is 0
__device__ __forceinline__ void cp_async16(void *dst, const void *src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(__cvta_generic_to_global(src)),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// D_acc[m][j] = sum_k A[m][k] D[j][k] for the 128 m of this CTA (MODE 0: z
// lines, MODE 1: x / y columns).  Bg holds D's TF32 parts pre-arranged per K
// block exactly as a stage's B region (hi then lo, canonical layout, rows
// n .. npad-1 and columns past n zero), so a stage's B arrives by bulk copies;
// A arrives raw by 16-byte asynchronous copies and is split into hi / lo in
// shared memory.  Stage s: raw A | A hi | A lo | B hi | B lo; S stages.
template <int MODE, int S>
__global__ void __launch_bounds__(kTcThreads, 1)
    r2r_tc_k(const float *__restrict__ in, float *__restrict__ out, const unsigned char *__restrict__ Bg, int n, int npad,
             TcGeom geo, int *err) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  uint64_t *rawf = reinterpret_cast<uint64_t *>(smraw);  // [S] raw A copies and B bytes landed
  uint64_t *conv = rawf + 8;                              // [S] hi / lo written
  uint64_t *empty = rawf + 16;                            // [S] the block's MMAs finished reading the stage
  uint64_t *accf = rawf + 24;                             // every MMA finished
  uint32_t *tslot = reinterpret_cast<uint32_t *>(smraw + 256);
  unsigned char *ops = smraw + 1024;
  // this CTA's output columns [c_lo, c_lo + nw) (all npad of them: one column block per line tile)
  const int c_lo = 0, nw = npad;
  const uint32_t a_bytes = kTcM * kTcBK * 4, b_bytes = (uint32_t)nw * kTcBK * 4;
  const size_t bfull = (size_t)npad * kTcBK * 4;  // one part of a K block of Bg
  const uint32_t stage_bytes = 3 * a_bytes + 2 * b_bytes;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // MODE 0: lines m0 .. m0 + 127 of length n, element (m, k) at in[m n + k];
  // MODE 1: m0 .. m0 + 127 of total_m, element (m, k) at mn_off(m) + k ldk
  const long long m0 = (long long)blockIdx.x * kTcM;
  const long long M = MODE == 0 ? geo.lines : geo.total_m;
  auto mn_off = [&](long long m) { return (m / geo.group_m) * geo.group_stride + m % geo.group_m; };
  // MODE 1 producer: lane = the tile's 4-m chunk (kTcM / 4 == 32), located once
  const bool lane_m_ok = MODE == 1 && m0 + 4 * lane < M;
  const long long lane_off = lane_m_ok ? mn_off(m0 + 4 * lane) : 0;
  const uint32_t ncols = nw <= 32 ? 32 : nw <= 64 ? 64 : nw <= 128 ? 128 : nw <= 256 ? 256 : 512;
  const int nkb = (n + kTcBK - 1) / kTcBK;

  if (tid == 0) {
    for (int i = 0; i < S; i++) mbar_init(rawf + i, 33), mbar_init(conv + i, 64), mbar_init(empty + i, 1);
    mbar_init(accf, 1);
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

  // Warp roles over the K blocks (stage s = kb % S, use u = kb / S):
  //  warp 0     producer: after empty[s] of use u - 1, the raw A block by 16-byte
  //             copies (every lane: cp.async.mbarrier.arrive.noinc on rawf[s])
  //             and the B block by one bulk copy (lane 0: expect_tx on rawf[s])
  //  warps 1-2  split: after rawf[s], hi / lo (MODE 1: transposed), then conv[s]
  //  warp 3     lane 0 issues the block's MMAs after conv[s] and commits them to
  //             empty[s]; after the last block a commit to accf
  bool ok = true;
  int kb_last = -1;  // producer: last block whose copies were issued
  if (warp == 0) {
    for (int kb = 0; kb < nkb; kb++) {
      const int s = kb % S, u = kb / S;
      if (u > 0 && !mbar_wait(empty + s, (uint32_t)(u - 1) & 1u, err)) {
        ok = false;
        break;
      }
      unsigned char *raw = ops + (size_t)s * stage_bytes;
      const int k0 = kb * kTcBK;
      if (MODE == 0) {
        for (int idx = lane; idx < kTcM * kTcCh; idx += 32) {
          const int r = idx / kTcCh, q = idx % kTcCh, k = k0 + 4 * q;
          const bool v = m0 + r < M && k < n;
          cp_async16(raw + kblock_off(r, q, kTcM), v ? in + (m0 + r) * n + k : in, v ? 16u : 0u);
        }
      } else {  // raw chunk (m group g, k row kr) at g * 128 + kr * 16: 4 consecutive m of one k
        for (int kr = 0; kr < kTcBK; kr++) {  // one k row per copy
          const int k = k0 + kr;
          const bool v = k < n && lane_m_ok;
          cp_async16(raw + lane * 128 + kr * 16, v ? in + lane_off + (long long)k * geo.ldk : in, v ? 16u : 0u);
        }
      }
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(rawf + s)) : "memory");
      if (lane == 0) {  // rows [c_lo, c_lo + nw) of the block's hi and lo parts (8-row groups of 256 B)
        const unsigned char *blk = Bg + (size_t)kb * 2 * bfull + (size_t)c_lo * 32;
        mbar_expect_tx(rawf + s, 2 * b_bytes);
        bulk_load(raw + 3 * a_bytes, blk, b_bytes, rawf + s);
        bulk_load(raw + 3 * a_bytes + b_bytes, blk + bfull, b_bytes, rawf + s);
      }
      kb_last = kb;
    }
    cp_async_wait<0>();
  } else if (warp <= 2) {
    const int ct = tid - 32;
    for (int kb = 0; kb < nkb; kb++) {
      const int s = kb % S;
      if (!mbar_wait(rawf + s, (uint32_t)(kb / S) & 1u, err)) {
        ok = false;
        break;
      }
      unsigned char *st = ops + (size_t)s * stage_bytes;
      for (int c = ct; c < kTcM * kTcBK / 4; c += 64) {
        const float4 v = *reinterpret_cast<const float4 *>(st + 16 * c);
        uint4 hi, lo;
        hi.x = tf32_round(v.x), hi.y = tf32_round(v.y), hi.z = tf32_round(v.z), hi.w = tf32_round(v.w);
        lo.x = tf32_round(v.x - __uint_as_float(hi.x)), lo.y = tf32_round(v.y - __uint_as_float(hi.y));
        lo.z = tf32_round(v.z - __uint_as_float(hi.z)), lo.w = tf32_round(v.w - __uint_as_float(hi.w));
        if (MODE == 0) {
          *reinterpret_cast<uint4 *>(st + a_bytes + 16 * c) = hi;
          *reinterpret_cast<uint4 *>(st + 2 * a_bytes + 16 * c) = lo;
        } else {
          const int g = c >> 3, kr = c & 7;
          const uint32_t h4[4] = {hi.x, hi.y, hi.z, hi.w}, l4[4] = {lo.x, lo.y, lo.z, lo.w};
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const uint32_t o = kblock_off(4 * g + e, kr >> 2, kTcM) + (kr & 3) * 4;
            *reinterpret_cast<uint32_t *>(st + a_bytes + o) = h4[e];
            *reinterpret_cast<uint32_t *>(st + 2 * a_bytes + o) = l4[e];
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(conv + s);
    }
  } else if (lane == 0) {
    int issued = 0;
    for (int kb = 0; kb < nkb; kb++) {
      const int s = kb % S;
      if (!mbar_wait(conv + s, (uint32_t)(kb / S) & 1u, err)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t sa = smem_u32(ops + (size_t)s * stage_bytes);
      const uint32_t ah = sa + a_bytes, al = ah + a_bytes;
      for (int h0 = 0; h0 < nw; h0 += 256) {  // N of at most 256 per MMA
        const int nh = min(256, nw - h0);
        const uint32_t bh = sa + 3 * a_bytes + (h0 >> 3) * 256, bl = bh + b_bytes;
        const uint32_t idesc = tf32_idesc(nh), d = tbase + (uint32_t)h0;
        const uint64_t dah = kmajor_desc(ah, 128, 256), dal = kmajor_desc(al, 128, 256);
        mma_tf32(d, dah, kmajor_desc(bh, 128, 256), idesc, kb == 0 ? 0u : 1u);
        mma_tf32(d, dah, kmajor_desc(bl, 128, 256), idesc, 1u);
        mma_tf32(d, dal, kmajor_desc(bh, 128, 256), idesc, 1u);
      }
      mma_commit(empty + s);
      issued = kb + 1;
    }
    (void)issued;
    mma_commit(accf);  // completes once every MMA issued above has finished
  }
  ok = __syncthreads_and(ok);
  if (ok) {
    ok = __syncthreads_and(mbar_wait(accf, 0u, err));
  } else {
    // MMAs issued before the failure, and bulk copies issued but not consumed,
    // finish before the shared and tensor memory are released
    mbar_drain(accf, 0u);
    if (tid == 0)
      for (int i = 0; i < S && i <= kb_last; i++) {
        const int kb = kb_last - ((kb_last - i) % S);  // the last block issued into stage i
        mbar_drain(rawf + i, (uint32_t)(kb / S) & 1u);
      }
  }
  __syncthreads();
  tc_fence_after();
  if (ok && MODE == 1) {  // lane = m: for each column j the warp writes 32 consecutive floats
    const long long m = m0 + warp * 32 + lane;
    const long long mo = m < M ? mn_off(m) : 0;
    const uint32_t taddr = tbase + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < nw; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(taddr + (uint32_t)c0, v);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < M) {
        float *o = out + mo + (long long)(c_lo + c0) * geo.ldk;
#pragma unroll
        for (int j = 0; j < 32; j++)
          if (c_lo + c0 + j < n) __stcs(o + (long long)j * geo.ldk, __uint_as_float(v[j]));
      }
    }
  }
  if (ok && MODE == 0) {
    const long long row = m0 + warp * 32 + lane;
    const uint32_t taddr = tbase + ((uint32_t)(warp * 32) << 16);
    // 32 accumulator columns per load (nw is a multiple of 16: the last
    // load may read 16 columns past nw, inside the allocation)
    for (int c0 = 0; c0 < nw; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(taddr + (uint32_t)c0, v);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
        float *o = out + row * n + c_lo + c0;
#pragma unroll
        for (int j = 0; j < 32; j += 4)
          if (c_lo + c0 + j + 4 <= n)
            __stcs(reinterpret_cast<float4 *>(o + j), make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]),
                                                                  __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3])));
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
// D's TF32 parts in the per-K-block stage layout of B (hi then lo)
__global__ void tf32_arrange_k(const float *__restrict__ D, unsigned char *Bg, int n, int npad) {
  const int nkb = (n + kTcBK - 1) / kTcBK;
  const long long total = (long long)nkb * npad * kTcCh;
  const uint32_t b_bytes = (uint32_t)npad * kTcBK * 4;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(t % kTcCh), r = (int)((t / kTcCh) % npad), kb = (int)(t / ((long long)kTcCh * npad));
    const int k = kb * kTcBK + 4 * q;
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    if (r < n)
      for (int e = 0; e < 4; e++)
        if (k + e < n) v[e] = D[(long long)r * n + k + e];
    uint32_t h[4], l[4];
    for (int e = 0; e < 4; e++) {
      h[e] = tf32_round(v[e]);
      l[e] = tf32_round(v[e] - __uint_as_float(h[e]));
    }
    unsigned char *blk = Bg + (size_t)kb * 2 * b_bytes;
    const uint32_t o = kblock_off(r, q, npad);
    *reinterpret_cast<uint4 *>(blk + o) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4 *>(blk + b_bytes + o) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}
}  // namespace

// stages: lines of up to 256 points keep a CTA within half the shared memory
// (two CTAs of at most 256 accumulator columns share an SM; 2-4 stages);
// longer lines take one CTA per SM with a 512-column accumulator (up to 6)
static int tc_stages(int npad) {
  const size_t stage = 3 * (size_t)kTcM * kTcBK * 4 + 2 * (size_t)npad * kTcBK * 4;
  if (npad <= 256) return (int)std::min<size_t>(4, (113 * 1024 - 2048) / stage);  // two CTAs (1 KB reserved each)
  return (int)std::min<size_t>(6, (227 * 1024 - 1024) / stage);                  // one CTA, 512 columns
}

size_t r2r_tc_smem(int n) {
  const int npad = (n + 15) / 16 * 16;
  return 1024 + (size_t)tc_stages(npad) * (3 * (size_t)kTcM * kTcBK * 4 + 2 * (size_t)npad * kTcBK * 4);
}

// axis 2 reads its lines as float4 runs (n % 4 == 0); every axis needs nz % 4 == 0
// (16-byte copies along z) and a line matrix of at most 512 rows
bool r2r_tc_supported(int axis, int nx, int ny, int nz) {
  const int n = axis == 0 ? nx : axis == 1 ? ny : nz;
  return nz % 4 == 0 && n >= 2 && n <= 512 && tc_stages((n + 15) / 16 * 16) >= 2 && r2r_tc_smem(n) <= 227 * 1024;
}

size_t r2r_tc_bytes(int n) {
  const int npad = (n + 15) / 16 * 16;
  return (size_t)((n + kTcBK - 1) / kTcBK) * 2 * npad * kTcBK * 4;
}

#define RTM_TC_ALL(X) X(0, 2) X(0, 3) X(0, 4) X(0, 5) X(0, 6) X(1, 2) X(1, 3) X(1, 4) X(1, 5) X(1, 6)

int r2r_tc_init() {
  const int mx = 227 * 1024;
  bool ok = true;
#define RTM_TC_ATTR(MODE, S) \
  ok = ok && cudaFuncSetAttribute(r2r_tc_k<MODE, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) == cudaSuccess;
  RTM_TC_ALL(RTM_TC_ATTR)
#undef RTM_TC_ATTR
  return ok ? 0 : -1;
}

void launch_tf32_arrange(const float *D, unsigned char *Bg, int n, cudaStream_t st) {
  const int npad = (n + 15) / 16 * 16;
  const long long total = (long long)((n + kTcBK - 1) / kTcBK) * npad * kTcCh;
  tf32_arrange_k<<<(unsigned)std::min<long long>((total + 255) / 256, 148LL * 8), 256, 0, st>>>(D, Bg, n, npad);
}

// axis 2 (z): out[l][j] = sum_k D[j][k] in[l][k]; axis 1 (y): out[j][c] = sum_k D[j][k] in[k][c] over
// c < nx nz; axis 0 (x): per y plane out[j][z] = sum_k D[j][k] in[k][z]
void launch_r2r_tc(int axis, const float *in, float *out, const unsigned char *Bg, int nx, int ny, int nz,
                   int *err, cudaStream_t st) {
  const int n = axis == 0 ? nx : axis == 1 ? ny : nz;
  const int npad = (n + 15) / 16 * 16;
  const long long nxz = (long long)nx * nz;
  TcGeom geo{};
  long long tiles;
  if (axis == 2) {
    geo.lines = (long long)nx * ny;
    tiles = (geo.lines + kTcM - 1) / kTcM;
  } else if (axis == 1) {
    geo.ldk = nxz, geo.group_stride = 0, geo.group_m = nxz, geo.total_m = nxz;
    tiles = (geo.total_m + kTcM - 1) / kTcM;
  } else {  // x lines: m over (y, z) pairs, so no tile is cut short at a y plane's end
    geo.ldk = nz, geo.group_stride = nxz, geo.group_m = nz, geo.total_m = (long long)ny * nz;
    tiles = (geo.total_m + kTcM - 1) / kTcM;
  }
  const size_t sm = r2r_tc_smem(n);
  const int S = tc_stages(npad), mode = axis == 2 ? 0 : 1;
#define RTM_TC_LAUNCH(MODE, SS) \
  if (mode == MODE && S == SS)                                                                               \
    r2r_tc_k<MODE, SS><<<(unsigned)tiles, kTcThreads, sm, st>>>(in, out, Bg, n, npad, geo, err);
  RTM_TC_ALL(RTM_TC_LAUNCH)
#undef RTM_TC_LAUNCH
}

}  // namespace rtm
