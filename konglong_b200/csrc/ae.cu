// ae.cu - learned snapshot compressor: a small 3-D convolutional autoencoder
// on 8^3-cell blocks, trained and run with hand-written tensor-core kernels.
//
// A block's cells are kept in Morton order (bit triples z y x from the least
// significant end), so the 8 children of every 2^3 cube are consecutive.
// With that layout every layer is one row-major GEMM on the previous layer's
// output memory, no reshaping:
//   E1  2^3 patch conv, stride 2   1 -> 16 ch   rows/block 64  K   8 N  16  leaky ReLU
//   E2  2^3 patch conv, stride 2  16 -> 16 ch              8   K 128 N  16  leaky ReLU
//   E3  pointwise                 16 -> 16 ch              8   K  16 N  16  leaky ReLU
//   E4  2^3 patch conv, stride 2  16 -> 64 ch (latent)     1   K 128 N  64  linear
//   D1  transposed 2^3, stride 2  64 -> 16 ch              1   K  64 N 128  leaky ReLU
//   D2  pointwise                 16 -> 16 ch              8   K  16 N  16  leaky ReLU
//   D3  transposed 2^3, stride 2  16 -> 16 ch              8   K  16 N 128  leaky ReLU
//   D4  transposed 2^3, stride 2  16 ->  1 ch              64  K  16 N   8  linear
// 512 cells -> 64 latent values stored as BF16 (the decoder's first GEMM rounds
// its operand to BF16, so BF16 storage keeps everything the decoder can use:
// 64 values in the bytes of 32 floats, 15.5:1 with the block's max |value|
// scale).
// GEMMs: mma.sync m16n8k16, BF16 operands (rounded from the FP32 activations
// and FP32 master weights), FP32 accumulation.  Training: MSE loss on the
// scale-normalised block, backward GEMMs, Adam on the FP32 master weights.
#include <cuda_bf16.h>
#include <stdint.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_fp16.h>

#include "kernel_api.h"
#include "rtm_b200.h"

namespace rtm {
namespace {

constexpr int kLayers = 8;
constexpr int kL_K[kLayers] = {8, 128, 16, 128, 64, 16, 16, 16};
constexpr int kL_N[kLayers] = {16, 16, 16, 64, 128, 16, 128, 8};
constexpr int kL_R[kLayers] = {64, 8, 8, 1, 1, 8, 8, 64};  // rows per block
constexpr int kL_ACT[kLayers] = {1, 1, 1, 0, 1, 1, 1, 0};
constexpr float kSlope = 0.1f;  // leaky ReLU
constexpr int kLatent = 64;
constexpr int kBlock = 512;

constexpr int w_off(int l) {
  int o = 0;
  for (int k = 0; k < l; k++) o += kL_K[k] * kL_N[k] + kL_N[k];
  return o;
}
constexpr int kNParams = w_off(kLayers);

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// C(m, n) [+]= sum_k A(m, k) B(k, n) over k in this block's split of [0, K),
// A(m, k) = A[m*sam + k*sak], B(k, n) = B[k*sbk + n*sbn]; operands rounded to
// BF16.  Epilogue: + bias[n], optional pre-activation copy, leaky ReLU; or an
// atomic add into C (split-K reductions, bias / activation not allowed).
struct Gemm {
  int M, N, K, ksplit;
  const float *A;
  long long sam, sak;
  const float *B;
  long long sbk, sbn;
  float *C;
  long long ldc;
  const float *bias;
  float *pre;
  int act, atomic;
};

// block: 4 warps, each a 16 x 32 tile; grid (M / 64, N / 32, ksplit)
__global__ void __launch_bounds__(128) gemm_bf16_k(Gemm g) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gr = lane >> 2, t = lane & 3;
  const int m0 = blockIdx.x * 64 + warp * 16, n0 = blockIdx.y * 32;
  const int kc = ((g.K + g.ksplit - 1) / g.ksplit + 15) / 16 * 16;
  const int kb = blockIdx.z * kc, ke = min(g.K, kb + kc);
  float acc[4][4] = {};
  auto a_at = [&](int m, int k) -> float { return (m < g.M && k < ke) ? g.A[m * g.sam + k * g.sak] : 0.f; };
  auto b_at = [&](int k, int n) -> float { return (n < g.N && k < ke) ? g.B[k * g.sbk + n * g.sbn] : 0.f; };
  for (int k0 = kb; k0 < ke; k0 += 16) {
    uint32_t a[4];
    const int r0 = m0 + gr, r1 = m0 + gr + 8, c0 = k0 + 2 * t, c1 = k0 + 2 * t + 8;
    a[0] = pack_bf16(a_at(r0, c0), a_at(r0, c0 + 1));
    a[1] = pack_bf16(a_at(r1, c0), a_at(r1, c0 + 1));
    a[2] = pack_bf16(a_at(r0, c1), a_at(r0, c1 + 1));
    a[3] = pack_bf16(a_at(r1, c1), a_at(r1, c1 + 1));
#pragma unroll
    for (int nt = 0; nt < 4; nt++) {
      const int n = n0 + nt * 8 + gr;
      const uint32_t b0 = pack_bf16(b_at(c0, n), b_at(c0 + 1, n));
      const uint32_t b1 = pack_bf16(b_at(c1, n), b_at(c1 + 1, n));
      mma_bf16(acc[nt], a, b0, b1);
    }
  }
#pragma unroll
  for (int nt = 0; nt < 4; nt++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int m = m0 + gr + (q >= 2 ? 8 : 0), n = n0 + nt * 8 + 2 * t + (q & 1);
      if (m >= g.M || n >= g.N) continue;
      float v = acc[nt][q];
      float *c = g.C + m * g.ldc + n;
      if (g.atomic) {
        atomicAdd(c, v);
        continue;
      }
      if (g.bias) v += g.bias[n];
      if (g.pre) g.pre[m * g.ldc + n] = v;
      if (g.act) v = v > 0.f ? v : kSlope * v;
      *c = v;
    }
}

void gemm(const Gemm &g0, cudaStream_t st) {
  Gemm g = g0;
  if (g.M <= 0 || g.N <= 0) return;
  if (!g.atomic) g.ksplit = 1;
  const dim3 grid((g.M + 63) / 64, (g.N + 31) / 32, std::max(1, g.ksplit));
  gemm_bf16_k<<<grid, 128, 0, st>>>(g);
}

// dP = dY * act'(pre) in place (leaky ReLU), for n elements
__global__ void act_back_k(float *dy, const float *pre, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (pre[i] <= 0.f) dy[i] *= kSlope;
}

// column sums of an R x N matrix into out[n] (atomic across row chunks)
__global__ void colsum_k(const float *dy, int R, int N, float *out) {
  const int n = blockIdx.y * 32 + (threadIdx.x & 31);
  if (n >= N) return;
  float s = 0.f;
  for (int r = blockIdx.x * 8 + (threadIdx.x >> 5); r < R; r += gridDim.x * 8) s += dy[(long long)r * N + n];
  atomicAdd(out + n, s);
}

// MSE loss on n values: loss += sum (y - x)^2 / n; dy = 2 (y - x) / n
__global__ void mse_k(const float *y, const float *x, long long n, float *dy, float *loss) {
  float s = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float d = y[i] - x[i];
    s += d * d;
    dy[i] = 2.f * d / (float)n;
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s / (float)n);
}

// Adam (bias-corrected) on the FP32 master parameters
__global__ void adam_k(float *p, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi, v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Morton index of cell (x, y, z) of an 8^3 block: bits z0 y0 x0 z1 y1 x1 z2 y2 x2
__host__ __device__ __forceinline__ int morton8(int x, int y, int z) {
  int m = 0;
#pragma unroll
  for (int b = 0; b < 3; b++) m |= (((z >> b) & 1) << (3 * b)) | (((y >> b) & 1) << (3 * b + 1)) | (((x >> b) & 1) << (3 * b + 2));
  return m;
}

}  // namespace
}  // namespace rtm

// ---- the compressor object ---------------------------------------------------
struct rtm_ae {
  int device = 0;
  cudaStream_t st = nullptr;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // params, grads, Adam moments
  float *loss = nullptr;
  int step = 0;
  // workspace for `cap` blocks: normalised input, per-layer outputs; training
  // also keeps pre-activations and gradients
  int cap = 0, cap_train = 0;
  float *x0 = nullptr, *y[8] = {}, *pre[8] = {}, *dy[8] = {}, *dx0 = nullptr, *sc = nullptr;
  std::string err;
};

namespace rtm {
namespace {

void ae_free_ws(rtm_ae *a) {
  auto fr = [](float *&q) {
    cudaFree(q);
    q = nullptr;
  };
  fr(a->x0), fr(a->dx0), fr(a->sc);
  for (int l = 0; l < kLayers; l++) fr(a->y[l]), fr(a->pre[l]), fr(a->dy[l]);
  a->cap = a->cap_train = 0;
}

// workspace for n blocks (train: also pre-activations and gradients)
int ae_reserve(rtm_ae *a, int n, bool train) {
  if (n <= a->cap && (!train || n <= a->cap_train)) return RTM_OK;
  const int cap = std::max(n, a->cap);
  const bool tr = train || a->cap_train > 0;
  ae_free_ws(a);
  bool ok = cudaMalloc(&a->x0, (size_t)cap * kBlock * 4) == cudaSuccess &&
            cudaMalloc(&a->sc, (size_t)cap * 4) == cudaSuccess;
  if (tr) ok = ok && cudaMalloc(&a->dx0, (size_t)cap * kBlock * 4) == cudaSuccess;
  for (int l = 0; l < kLayers && ok; l++) {
    const size_t e = (size_t)cap * kL_R[l] * kL_N[l] * 4;
    ok = cudaMalloc(&a->y[l], e) == cudaSuccess;
    if (tr) ok = ok && cudaMalloc(&a->pre[l], e) == cudaSuccess && cudaMalloc(&a->dy[l], e) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    ae_free_ws(a);
    a->err = "compressor workspace allocation failed";
    return RTM_ERR_NOMEM;
  }
  a->cap = cap, a->cap_train = tr ? cap : 0;
  return RTM_OK;
}

// forward of layers [l0, l1) for n blocks, input of layer l0 at `in`
void ae_forward(rtm_ae *a, int n, const float *in, int l0, int l1, bool keep_pre, cudaStream_t st) {
  const float *x = in;
  for (int l = l0; l < l1; l++) {
    Gemm g{};
    g.M = n * kL_R[l], g.N = kL_N[l], g.K = kL_K[l], g.ksplit = 1;
    g.A = x, g.sam = kL_K[l], g.sak = 1;
    g.B = a->p + w_off(l), g.sbk = kL_N[l], g.sbn = 1;
    g.C = a->y[l], g.ldc = kL_N[l];
    g.bias = a->p + w_off(l) + kL_K[l] * kL_N[l];
    g.pre = keep_pre ? a->pre[l] : nullptr;
    g.act = kL_ACT[l];
    gemm(g, st);
    x = a->y[l];
  }
}

// loss and parameter gradients (into a->g) of n normalised blocks at a->x0
void ae_loss_grad(rtm_ae *a, int n) {
  cudaStream_t st = a->st;
  ae_forward(a, n, a->x0, 0, kLayers, true, st);
  cudaMemsetAsync(a->loss, 0, 4, st);
  cudaMemsetAsync(a->g, 0, (size_t)kNParams * 4, st);
  const long long tot = (long long)n * kBlock;
  mse_k<<<(int)std::min<long long>((tot + 255) / 256, 1024), 256, 0, st>>>(a->y[kLayers - 1], a->x0, tot,
                                                                            a->dy[kLayers - 1], a->loss);
  for (int l = kLayers - 1; l >= 0; l--) {
    const int R = n * kL_R[l], K = kL_K[l], N = kL_N[l];
    const long long e = (long long)R * N;
    if (kL_ACT[l])
      act_back_k<<<(int)std::min<long long>((e + 255) / 256, 2048), 256, 0, st>>>(a->dy[l], a->pre[l], e);
    const float *xin = l == 0 ? a->x0 : a->y[l - 1];
    Gemm gw{};  // dW = X^T dP (K x N), reduction over the R rows, split-K
    gw.M = K, gw.N = N, gw.K = R, gw.ksplit = std::max(1, std::min(128, R / 256));
    gw.A = xin, gw.sam = 1, gw.sak = K;
    gw.B = a->dy[l], gw.sbk = N, gw.sbn = 1;
    gw.C = a->g + w_off(l), gw.ldc = N, gw.atomic = 1;
    gemm(gw, st);
    colsum_k<<<dim3(std::min(64, (R + 7) / 8), (N + 31) / 32), 256, 0, st>>>(a->dy[l], R, N,
                                                                            a->g + w_off(l) + K * N);
    Gemm gx{};  // dX = dP W^T (R x K)
    gx.M = R, gx.N = K, gx.K = N, gx.ksplit = 1;
    gx.A = a->dy[l], gx.sam = N, gx.sak = 1;
    gx.B = a->p + w_off(l), gx.sbk = 1, gx.sbn = N;
    gx.C = l == 0 ? a->dx0 : a->dy[l - 1], gx.ldc = K;
    gemm(gx, st);
  }
}

constexpr int kChunkBlocks = 8192;  // blocks per encode / decode pass over a volume

// ---- fused inference over a volume -------------------------------------------
// One warp per 8^3 block, a CTA of 4 warps per 4 blocks consecutive in z (32 z
// cells of each x / y row: 128-byte rows in and out).  The CTA stages the
// encoder (or decoder) weights once as BF16 in shared memory; each warp runs
// its block through the four layers with the layer outputs in shared memory
// (BF16: the next layer's operand rounding) and writes only the latent and the
// scale (or the decoded cells).  Each output element is the same mma.sync
// chain over k in steps of 16 as in gemm_bf16_k, with the same operand
// roundings, bias and activation, so the results equal the layer-by-layer
// path bit for bit.  Rows of a layer beyond its M (8 or 1 per block) and
// columns beyond K (8 in E1) enter the MMA as zeros.
constexpr int kFusedWarps = 4;

// Row strides (bf16 elements) of the operands in shared memory: K + 8 for a
// layer's transposed weights and its input rows, so that the 32-bit loads of
// a fragment's column pairs fall in distinct banks (a row of K + 8 bf16 moves
// the bank by 4 words: the 8 row groups x 4 column pairs of a fragment cover
// the 32 banks once).  Rows of E1's input (K = 8) stay unpadded (4 words).
constexpr int kpad(int k) { return k == 8 ? 8 : k + 8; }

// out(m, n, v) for m < M, n < N: v = act(bias[n] + sum_k A[m][k] W[k][n]),
// A bf16 [M][LDA] and the weights transposed, Wt bf16 [N][kpad(K)], in shared
// memory.  Each pair of adjacent columns is one 32-bit load.
template <int M, int K, int N, int LDA, bool ACT, typename Out>
__device__ __forceinline__ void warp_layer(const __nv_bfloat16 *A, const __nv_bfloat16 *Wt, const float *bias,
                                           Out out) {
  constexpr int LDW = kpad(K);
  const int lane = threadIdx.x & 31, gr = lane >> 2, t = lane & 3;
  auto a2 = [&](int m, int k) -> uint32_t {
    return (m < M && k < K) ? *reinterpret_cast<const uint32_t *>(A + m * LDA + k) : 0u;
  };
  auto b2 = [&](int k, int n) -> uint32_t {
    return k < K ? *reinterpret_cast<const uint32_t *>(Wt + n * LDW + k) : 0u;
  };
#pragma unroll 1
  for (int m0 = 0; m0 < M; m0 += 16) {
#pragma unroll 1
    for (int n0 = 0; n0 < N; n0 += 8) {
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int k0 = 0; k0 < K; k0 += 16) {
        const int r0 = m0 + gr, r1 = r0 + 8, c0 = k0 + 2 * t, c1 = c0 + 8, n = n0 + gr;
        uint32_t a[4];
        a[0] = a2(r0, c0);
        a[1] = a2(r1, c0);
        a[2] = a2(r0, c1);
        a[3] = a2(r1, c1);
        mma_bf16(acc, a, b2(c0, n), b2(c1, n));
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int m = m0 + gr + (q >= 2 ? 8 : 0), n = n0 + 2 * t + (q & 1);
        if (m >= M) continue;
        float v = acc[q] + bias[n];
        if (ACT) v = v > 0.f ? v : kSlope * v;
        out(m, n, v);
      }
    }
  }
}

// transposed, padded weights of a layer and of four consecutive layers
template <int L> constexpr int wt_size() { return kL_N[L] * kpad(kL_K[L]); }
template <int L0> constexpr int half_wt() { return wt_size<L0>() + wt_size<L0 + 1>() + wt_size<L0 + 2>() + wt_size<L0 + 3>(); }
constexpr int half_b(int l0) { return kL_N[l0] + kL_N[l0 + 1] + kL_N[l0 + 2] + kL_N[l0 + 3]; }

// layer L's weights W[k][n] (FP32 master) into Wt[n][kpad(K)] as bf16, its biases as FP32
template <int L>
__device__ __forceinline__ void stage_layer(const float *__restrict__ p, __nv_bfloat16 *wt, float *b) {
  constexpr int K = kL_K[L], N = kL_N[L], wo = w_off(L);
  for (int i = threadIdx.x; i < K * N; i += blockDim.x) {
    const int k = i / N, n = i % N;
    wt[n * kpad(K) + k] = __float2bfloat16_rn(p[wo + i]);
  }
  for (int i = threadIdx.x; i < N; i += blockDim.x) b[i] = p[wo + K * N + i];
}
template <int L0>
__device__ __forceinline__ void stage_weights(const float *__restrict__ p, __nv_bfloat16 *w, float *b) {
  constexpr int w1 = wt_size<L0>(), w2 = w1 + wt_size<L0 + 1>(), w3 = w2 + wt_size<L0 + 2>();
  constexpr int b1 = kL_N[L0], b2 = b1 + kL_N[L0 + 1], b3 = b2 + kL_N[L0 + 2];
  stage_layer<L0>(p, w, b);
  stage_layer<L0 + 1>(p, w + w1, b + b1);
  stage_layer<L0 + 2>(p, w + w2, b + b2);
  stage_layer<L0 + 3>(p, w + w3, b + b3);
}

// input row strides: E2 reads E1's output as [8][128], E3 E2's as [8][16],
// D2 D1's as [8][16], D3 D2's as [8][16], D4 D3's as [64][16]
constexpr int kLdE2 = kpad(128), kLdE3 = kpad(16), kLdD2 = kpad(16), kLdD3 = kpad(16), kLdD4 = kpad(16);

struct __align__(16) AeEncSmem {
  __nv_bfloat16 w[half_wt<0>()];
  float b[half_b(0)];
  float raw[kFusedWarps][kBlock];           // the blocks' cells, Morton order
  __nv_bfloat16 x[kFusedWarps][kBlock];     // E1 input [64][8]
  __nv_bfloat16 h1[kFusedWarps][8 * kLdE2]; // E1 output = E2 input [8][128]
  __nv_bfloat16 h2[kFusedWarps][8 * kLdE3]; // E2 output = E3 input [8][16]
  __nv_bfloat16 h3[kFusedWarps][8 * 16];    // E3 output = E4 input [1][128]
};

// Persistent: each CTA stages the weights once, then takes groups of 4
// blocks consecutive in z (group g: z group g % nbzg, then x, then y; block
// bz = 4 (g % nbzg) + warp) until none is left.
__global__ void __launch_bounds__(32 * kFusedWarps) ae_encode_k(const float *__restrict__ p,
                                                               const float *__restrict__ vol, int nx, int ny, int nz,
                                                               __nv_bfloat16 *__restrict__ latent,
                                                               float *__restrict__ scales) {
  extern __shared__ __align__(16) unsigned char smem_ae[];
  AeEncSmem &s = *reinterpret_cast<AeEncSmem *>(smem_ae);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nbz = (nz + 7) / 8, nbx = (nx + 7) / 8, nby = (ny + 7) / 8, nbzg = (nbz + kFusedWarps - 1) / kFusedWarps;
  const long long ngroups = (long long)nbzg * nbx * nby;
  stage_weights<0>(p, s.w, s.b);
  for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
  const int bx = (int)((grp / nbzg) % nbx), by = (int)(grp / ((long long)nbzg * nbx)), z0 = (int)(grp % nbzg) * 32;
  // 32 z x 8 x x 8 y cells: thread -> (z quad, x, y) rows of 128 bytes
  for (int i = threadIdx.x; i < 8 * 8 * 8; i += blockDim.x) {
    const int zq = i & 7, xi = (i >> 3) & 7, yj = i >> 6;
    const int x = bx * 8 + xi, y = by * 8 + yj;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int zl = zq * 4 + c, z = z0 + zl;
      const float v = (x < nx && y < ny && z < nz) ? vol[((long long)y * nx + x) * nz + z] : 0.f;
      s.raw[zl >> 3][morton8(xi, yj, zl & 7)] = v;
    }
  }
  __syncthreads();
  const int bz = (int)(grp % nbzg) * kFusedWarps + warp;
  if (bz < nbz) {
    float a = 0.f;
    for (int i = lane; i < kBlock; i += 32) a = fmaxf(a, fabsf(s.raw[warp][i]));
    for (int o = 16; o; o >>= 1) a = fmaxf(a, __shfl_xor_sync(0xffffffffu, a, o));
    const float sc = a;
    for (int i = lane; i < kBlock; i += 32)
      s.x[warp][i] = __float2bfloat16_rn(sc > 0.f ? s.raw[warp][i] / sc : 0.f);
    __syncwarp();
    const __nv_bfloat16 *w = s.w;
    const float *b = s.b;
    __nv_bfloat16 *h1 = s.h1[warp], *h2 = s.h2[warp], *h3 = s.h3[warp];
    warp_layer<64, 8, 16, 8, true>(s.x[warp], w, b, [&](int m, int n, float v) {
      h1[(m >> 3) * kLdE2 + (m & 7) * 16 + n] = __float2bfloat16_rn(v);
    });
    __syncwarp();
    w += wt_size<0>(), b += 16;
    warp_layer<8, 128, 16, kLdE2, true>(h1, w, b, [&](int m, int n, float v) {
      h2[m * kLdE3 + n] = __float2bfloat16_rn(v);
    });
    __syncwarp();
    w += wt_size<1>(), b += 16;
    warp_layer<8, 16, 16, kLdE3, true>(h2, w, b, [&](int m, int n, float v) { h3[m * 16 + n] = __float2bfloat16_rn(v); });
    __syncwarp();
    w += wt_size<2>(), b += 16;
    const long long blk = ((long long)by * nbx + bx) * nbz + bz;
    __nv_bfloat16 *lat = latent + blk * kLatent;
    warp_layer<1, 128, kLatent, 128, false>(h3, w, b, [&](int, int n, float v) { lat[n] = __float2bfloat16_rn(v); });
    if (lane == 0) scales[blk] = sc;
  }
  __syncthreads();  // the next group overwrites raw
  }
}

struct __align__(16) AeDecSmem {
  __nv_bfloat16 w[half_wt<4>()];
  float b[half_b(4)];
  __nv_bfloat16 l[kFusedWarps][kLatent];     // D1 input [1][kLatent]
  __nv_bfloat16 g1[kFusedWarps][8 * kLdD2];  // D1 output = D2 input [8][16]
  __nv_bfloat16 g2[kFusedWarps][8 * kLdD3];  // D2 output = D3 input [8][16]
  __nv_bfloat16 g3[kFusedWarps][64 * kLdD4]; // D3 output = D4 input [64][16]
  float out[kFusedWarps][kBlock];            // D4 output x scale, Morton order
};

__global__ void __launch_bounds__(32 * kFusedWarps) ae_decode_k(const float *__restrict__ p,
                                                               const __nv_bfloat16 *__restrict__ latent,
                                                               const float *__restrict__ scales, int nx, int ny, int nz,
                                                               float *__restrict__ vol) {
  extern __shared__ __align__(16) unsigned char smem_ae[];
  AeDecSmem &s = *reinterpret_cast<AeDecSmem *>(smem_ae);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nbz = (nz + 7) / 8, nbx = (nx + 7) / 8, nby = (ny + 7) / 8, nbzg = (nbz + kFusedWarps - 1) / kFusedWarps;
  const long long ngroups = (long long)nbzg * nbx * nby;
  stage_weights<4>(p, s.w, s.b);
  __syncthreads();
  for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
  const int bx = (int)((grp / nbzg) % nbx), by = (int)(grp / ((long long)nbzg * nbx)), z0 = (int)(grp % nbzg) * 32;
  const int bz = (int)(grp % nbzg) * kFusedWarps + warp;
  if (bz < nbz) {
    const long long blk = ((long long)by * nbx + bx) * nbz + bz;
    for (int k = lane; k < kLatent; k += 32) s.l[warp][k] = latent[blk * kLatent + k];
    const float sc = scales[blk];
    __syncwarp();
    const __nv_bfloat16 *w = s.w;
    const float *b = s.b;
    __nv_bfloat16 *g1 = s.g1[warp], *g2 = s.g2[warp], *g3 = s.g3[warp];
    float *o = s.out[warp];
    warp_layer<1, kLatent, 128, kLatent, true>(s.l[warp], w, b, [&](int, int n, float v) {
      g1[(n >> 4) * kLdD2 + (n & 15)] = __float2bfloat16_rn(v);
    });
    __syncwarp();
    w += wt_size<4>(), b += 128;
    warp_layer<8, 16, 16, kLdD2, true>(g1, w, b, [&](int m, int n, float v) {
      g2[m * kLdD3 + n] = __float2bfloat16_rn(v);
    });
    __syncwarp();
    w += wt_size<5>(), b += 16;
    warp_layer<8, 16, 128, kLdD3, true>(g2, w, b, [&](int m, int n, float v) {
      g3[(m * 8 + (n >> 4)) * kLdD4 + (n & 15)] = __float2bfloat16_rn(v);
    });
    __syncwarp();
    w += wt_size<6>(), b += 128;
    warp_layer<64, 16, 8, kLdD4, false>(g3, w, b, [&](int m, int n, float v) { o[m * 8 + n] = sc * v; });
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 8 * 8 * 8; i += blockDim.x) {
    const int zq = i & 7, xi = (i >> 3) & 7, yj = i >> 6;
    const int x = bx * 8 + xi, y = by * 8 + yj;
    if (x >= nx || y >= ny) continue;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int zl = zq * 4 + c, z = z0 + zl;
      if (z < nz) vol[((long long)y * nx + x) * nz + z] = s.out[zl >> 3][morton8(xi, yj, zl & 7)];
    }
  }
  __syncthreads();  // the next group overwrites out
  }
}

}  // namespace

long long ae_volume_blocks(int nx, int ny, int nz) {
  return (long long)((nx + 7) / 8) * ((ny + 7) / 8) * ((nz + 7) / 8);
}

int ae_prepare(rtm_ae *a) { return ae_reserve(a, kChunkBlocks, false); }

// CTAs of one wave of the persistent codec kernels (set by ae_fused_init)
static int g_ae_wave = 0;

// shared-memory size of the fused encoder / decoder (beyond the 48 KB default)
// and the CTAs of one wave; called when a compressor is created (outside any
// stream capture)
static bool ae_fused_init() {
  if (cudaFuncSetAttribute(ae_encode_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(AeEncSmem)) !=
          cudaSuccess ||
      cudaFuncSetAttribute(ae_decode_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(AeDecSmem)) !=
          cudaSuccess)
    return false;
  int dev = 0, sms = 0, occ_e = 0, occ_d = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_e, ae_encode_k, 32 * kFusedWarps, sizeof(AeEncSmem));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_d, ae_decode_k, 32 * kFusedWarps, sizeof(AeDecSmem));
  g_ae_wave = std::max(1, sms) * std::max(1, std::min(occ_e, occ_d));
  return true;
}

// volume -> latents [nb][64] (bfloat16) + scales [nb] (device), on stream st
// (the fused kernel)
// CTAs of a persistent codec launch over `groups` work items: one wave
static unsigned ae_grid(long long groups) {
  return (unsigned)std::max(1LL, std::min<long long>(groups, std::max(1, g_ae_wave)));
}
static long long ae_groups(int nx, int ny, int nz) {
  return (long long)((((nz + 7) / 8) + kFusedWarps - 1) / kFusedWarps) * ((nx + 7) / 8) * ((ny + 7) / 8);
}

int ae_compress(rtm_ae *a, const float *w, int nx, int ny, int nz, void *latent, float *scales, cudaStream_t st) {
  ae_encode_k<<<ae_grid(ae_groups(nx, ny, nz)), 32 * kFusedWarps, sizeof(AeEncSmem), st>>>(
      a->p, w, nx, ny, nz, static_cast<__nv_bfloat16 *>(latent), scales);
  return cudaGetLastError() == cudaSuccess ? RTM_OK : RTM_ERR_CUDA;
}
// latents + scales -> volume (device), on stream st (the fused kernel)
int ae_decompress(rtm_ae *a, const void *latent, const float *scales, int nx, int ny, int nz, float *w,
                  cudaStream_t st) {
  ae_decode_k<<<ae_grid(ae_groups(nx, ny, nz)), 32 * kFusedWarps, sizeof(AeDecSmem), st>>>(
      a->p, static_cast<const __nv_bfloat16 *>(latent), scales, nx, ny, nz, w);
  return cudaGetLastError() == cudaSuccess ? RTM_OK : RTM_ERR_CUDA;
}


// ---- FP16 fallback of the high-energy blocks of a learned snapshot ----------
// Per slot: a header, the indices of the stored blocks, and each stored block
// as 512 FP16 values of v / scale (natural z, x, y order).  The stored blocks
// are the candidates (scale > 0 and > tau x the largest) whose scale exceeds
// the (cap+1)-th largest candidate scale, all of them when there are at most
// cap: a deterministic choice, found by a radix select over the scales' IEEE
// bit patterns (positive floats order like their bits) in three levels of
// 11, 11 and 9 bits; thr ends as the smallest bit pattern stored.
namespace {

constexpr int kFbBins = 2048;
__host__ __device__ constexpr int fb_shift(int L) { return L == 0 ? 20 : L == 1 ? 9 : 0; }
__host__ __device__ constexpr int fb_width(int L) { return L == 2 ? 9 : 11; }

struct FbHdr {
  unsigned maxbits, prefix, thr;
  int count, rem, done;
  int hist[kFbBins];
};

__global__ void fb_max_k(const float *__restrict__ scales, long long nb, FbHdr *h) {
  float m = 0.f;
  for (long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, scales[b]);
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(&h->maxbits, __float_as_uint(m));
}

// histogram of the candidates inside the current prefix, by their next bits
template <int L>
__global__ void fb_hist_k(const float *__restrict__ scales, long long nb, float tau, FbHdr *h) {
  if (h->done) return;
  constexpr int hi = fb_shift(L) + fb_width(L);
  const float mx = __uint_as_float(h->maxbits);
  const unsigned pre = h->prefix >> hi;
  for (long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (long long)gridDim.x * blockDim.x) {
    const float s = scales[b];
    const unsigned u = __float_as_uint(s);
    if (s > 0.f && s > tau * mx && (u >> hi) == pre)
      atomicAdd(&h->hist[(u >> fb_shift(L)) & ((1u << fb_width(L)) - 1)], 1);
  }
}

// the bin, from the top, where the running count passes the capacity left
template <int L>
__global__ void __launch_bounds__(256) fb_scan_k(FbHdr *h, int cap) {
  __shared__ int part[256];
  __shared__ int found;
  if (h->done) return;
  constexpr int nbin = 1 << fb_width(L), per = nbin / 256 > 0 ? nbin / 256 : 1;
  const int t = threadIdx.x;
  const int top = nbin - 1 - t * per;  // this thread's bins: top, top-1, ..., top-per+1 (t * per < nbin)
  int v[8], sum = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    v[i] = (i < per && t * per < nbin) ? h->hist[top - i] : 0;
    sum += v[i];
  }
  part[t] = sum;
  if (t == 0) found = 0;
  __syncthreads();
  for (int o = 1; o < 256; o <<= 1) {  // inclusive scan (Hillis-Steele)
    const int x = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += x;
    __syncthreads();
  }
  const int rem = L == 0 ? cap : h->rem;  // read by all before the one write below
  const int before = part[t] - sum;  // candidates in the bins above this thread's
  if (before <= rem && part[t] > rem) {  // the boundary bin is one of this thread's
    int cum = before, k = 0;
    while (cum + v[k] <= rem) cum += v[k++];
    const unsigned bin = (unsigned)(top - k);
    if (L == 2) {
      h->thr = h->prefix + (bin + 1);  // the bins above the boundary (bin + 1 may carry into the prefix)
      h->done = 1;
    } else {
      h->prefix |= bin << fb_shift(L);
      h->rem = rem - cum;
    }
    found = 1;
  }
  __syncthreads();
  if (t == 0 && !found) {  // every candidate inside the prefix fits
    h->thr = h->prefix;
    h->done = 1;
  }
  for (int i = t; i < kFbBins; i += 256) h->hist[i] = 0;  // for the next level
}

// the chosen blocks: index and FP16 copy of v / scale (one CTA of 512 per block)
__global__ void __launch_bounds__(512) fb_store_k(const float *__restrict__ w, const float *__restrict__ scales,
                                                  long long nb, float tau, int nx, int ny, int nz, FbHdr *h, int *idx,
                                                  __half *data) {
  __shared__ int slot;
  const float mx = __uint_as_float(h->maxbits);
  for (long long b = blockIdx.x; b < nb; b += gridDim.x) {
    const float s = scales[b];
    if (!(s > 0.f && s > tau * mx && __float_as_uint(s) >= h->thr)) continue;  // uniform over the CTA
    if (threadIdx.x == 0) {
      slot = atomicAdd(&h->count, 1);
      idx[slot] = (int)b;
    }
    __syncthreads();
    const int nbz = (nz + 7) / 8, nbx = (nx + 7) / 8;
    const int bz = (int)(b % nbz), bx = (int)((b / nbz) % nbx), by = (int)(b / ((long long)nbz * nbx));
    const int k = threadIdx.x & 7, i = (threadIdx.x >> 3) & 7, j = threadIdx.x >> 6;
    const int x = bx * 8 + i, y = by * 8 + j, z = bz * 8 + k;
    const float v = (x < nx && y < ny && z < nz) ? w[((long long)y * nx + x) * nz + z] : 0.f;
    data[(long long)slot * 512 + threadIdx.x] = __float2half_rn(v / s);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(512) fb_apply_k(const float *__restrict__ scales, const FbHdr *h, const int *idx,
                                                  const __half *data, int cap, int nx, int ny, int nz, float *w) {
  const int n = min(h->count, cap);  // a slot never stored holds no valid count: clamp, check each index
  const long long nb = (long long)((nx + 7) / 8) * ((ny + 7) / 8) * ((nz + 7) / 8);
  for (int t = blockIdx.x; t < n; t += gridDim.x) {
    const long long b = idx[t];
    if (b < 0 || b >= nb) continue;
    const int nbz = (nz + 7) / 8, nbx = (nx + 7) / 8;
    const int bz = (int)(b % nbz), bx = (int)((b / nbz) % nbx), by = (int)(b / ((long long)nbz * nbx));
    const int k = threadIdx.x & 7, i = (threadIdx.x >> 3) & 7, j = threadIdx.x >> 6;
    const int x = bx * 8 + i, y = by * 8 + j, z = bz * 8 + k;
    if (x < nx && y < ny && z < nz)
      w[((long long)y * nx + x) * nz + z] = __half2float(data[(long long)t * 512 + threadIdx.x]) * scales[b];
  }
}

}  // namespace

size_t ae_fallback_bytes(long long cap) { return sizeof(FbHdr) + (size_t)cap * 4 + (size_t)cap * 1024; }

void ae_fallback_store(const float *w, const float *scales, int nx, int ny, int nz, float tau, long long cap, void *fb,
                       cudaStream_t st) {
  const long long nb = ae_volume_blocks(nx, ny, nz);
  FbHdr *h = static_cast<FbHdr *>(fb);
  int *idx = reinterpret_cast<int *>(h + 1);
  __half *data = reinterpret_cast<__half *>(idx + cap);
  cudaMemsetAsync(h, 0, sizeof(FbHdr), st);
  const unsigned g = (unsigned)std::min<long long>((nb + 255) / 256, 1184);
  fb_max_k<<<g, 256, 0, st>>>(scales, nb, h);
  fb_hist_k<0><<<g, 256, 0, st>>>(scales, nb, tau, h);
  fb_scan_k<0><<<1, 256, 0, st>>>(h, (int)cap);
  fb_hist_k<1><<<g, 256, 0, st>>>(scales, nb, tau, h);
  fb_scan_k<1><<<1, 256, 0, st>>>(h, (int)cap);
  fb_hist_k<2><<<g, 256, 0, st>>>(scales, nb, tau, h);
  fb_scan_k<2><<<1, 256, 0, st>>>(h, (int)cap);
  fb_store_k<<<(unsigned)std::min<long long>(nb, 4096), 512, 0, st>>>(w, scales, nb, tau, nx, ny, nz, h, idx, data);
}

void ae_fallback_apply(const float *scales, int nx, int ny, int nz, long long cap, const void *fb, float *w,
                       cudaStream_t st) {
  const FbHdr *h = static_cast<const FbHdr *>(fb);
  const int *idx = reinterpret_cast<const int *>(h + 1);
  const __half *data = reinterpret_cast<const __half *>(idx + cap);
  fb_apply_k<<<(unsigned)std::max<long long>(1, std::min<long long>(cap, 4096)), 512, 0, st>>>(scales, h, idx, data,
                                                                                                  (int)cap, nx, ny, nz, w);
}

}  // namespace rtm

extern "C" {

int rtm_ae_nparams(void) { return rtm::kNParams; }

int rtm_ae_create(rtm_ae **out) {
  if (!out) return RTM_ERR_ARG;
  *out = nullptr;
  rtm_ae *a = new rtm_ae();
  cudaGetDevice(&a->device);
  const size_t b = (size_t)rtm::kNParams * 4;
  // a blocking stream: ordered after the parameter uploads (pageable cudaMemcpy)
  if (cudaStreamCreate(&a->st) || cudaMalloc(&a->p, b) || cudaMalloc(&a->g, b) ||
      cudaMalloc(&a->m, b) || cudaMalloc(&a->v, b) || cudaMalloc(&a->loss, 4) || cudaMemset(a->p, 0, b) ||
      cudaMemset(a->m, 0, b) || cudaMemset(a->v, 0, b)) {
    cudaGetLastError();
    rtm_ae_destroy(a);
    return RTM_ERR_NOMEM;
  }
  if (!rtm::ae_fused_init()) {
    cudaGetLastError();
    rtm_ae_destroy(a);
    return RTM_ERR_CUDA;
  }
  *out = a;
  return RTM_OK;
}

int rtm_ae_destroy(rtm_ae *a) {
  if (!a) return RTM_ERR_ARG;
  cudaSetDevice(a->device);
  if (a->st) cudaStreamSynchronize(a->st);
  rtm::ae_free_ws(a);
  cudaFree(a->p), cudaFree(a->g), cudaFree(a->m), cudaFree(a->v), cudaFree(a->loss);
  if (a->st) cudaStreamDestroy(a->st);
  delete a;
  return RTM_OK;
}

int rtm_ae_set_params(rtm_ae *a, const float *params) {
  if (!a || !params) return RTM_ERR_ARG;
  cudaSetDevice(a->device);
  if (cudaMemcpy(a->p, params, (size_t)rtm::kNParams * 4, cudaMemcpyHostToDevice)) return RTM_ERR_CUDA;
  cudaMemset(a->m, 0, (size_t)rtm::kNParams * 4), cudaMemset(a->v, 0, (size_t)rtm::kNParams * 4);
  a->step = 0;
  return RTM_OK;
}

int rtm_ae_get_params(rtm_ae *a, float *params) {
  if (!a || !params) return RTM_ERR_ARG;
  cudaSetDevice(a->device);
  cudaStreamSynchronize(a->st);
  return cudaMemcpy(params, a->p, (size_t)rtm::kNParams * 4, cudaMemcpyDeviceToHost) ? RTM_ERR_CUDA : RTM_OK;
}

int rtm_ae_loss_grad(rtm_ae *a, const float *blocks, int n, float *loss, float *grads) {
  if (!a || !blocks || n < 1 || !loss) return RTM_ERR_ARG;
  cudaSetDevice(a->device);
  if (int rc = rtm::ae_reserve(a, n, true)) return rc;
  if (cudaMemcpyAsync(a->x0, blocks, (size_t)n * rtm::kBlock * 4, cudaMemcpyHostToDevice, a->st)) return RTM_ERR_CUDA;
  rtm::ae_loss_grad(a, n);
  cudaMemcpyAsync(loss, a->loss, 4, cudaMemcpyDeviceToHost, a->st);
  if (grads) cudaMemcpyAsync(grads, a->g, (size_t)rtm::kNParams * 4, cudaMemcpyDeviceToHost, a->st);
  return cudaStreamSynchronize(a->st) == cudaSuccess ? RTM_OK : RTM_ERR_CUDA;
}

int rtm_ae_train_step(rtm_ae *a, const float *blocks, int n, float lr, float *loss) {
  if (!a || !blocks || n < 1 || !loss || !(lr > 0.f)) return RTM_ERR_ARG;
  cudaSetDevice(a->device);
  if (int rc = rtm::ae_reserve(a, n, true)) return rc;
  if (cudaMemcpyAsync(a->x0, blocks, (size_t)n * rtm::kBlock * 4, cudaMemcpyHostToDevice, a->st)) return RTM_ERR_CUDA;
  rtm::ae_loss_grad(a, n);
  a->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)a->step), c2 = 1.f - powf(b2, (float)a->step);
  rtm::adam_k<<<(rtm::kNParams + 255) / 256, 256, 0, a->st>>>(a->p, a->g, a->m, a->v, rtm::kNParams, lr, b1, b2, 1e-8f,
                                                            c1, c2);
  cudaMemcpyAsync(loss, a->loss, 4, cudaMemcpyDeviceToHost, a->st);
  return cudaStreamSynchronize(a->st) == cudaSuccess ? RTM_OK : RTM_ERR_CUDA;
}

int rtm_ae_reconstruct(rtm_ae *a, const float *blocks, int n, float *out, float *latent) {
  if (!a || !blocks || n < 1 || !out) return RTM_ERR_ARG;
  cudaSetDevice(a->device);
  if (int rc = rtm::ae_reserve(a, n, false)) return rc;
  if (cudaMemcpyAsync(a->x0, blocks, (size_t)n * rtm::kBlock * 4, cudaMemcpyHostToDevice, a->st)) return RTM_ERR_CUDA;
  rtm::ae_forward(a, n, a->x0, 0, rtm::kLayers, false, a->st);
  cudaMemcpyAsync(out, a->y[rtm::kLayers - 1], (size_t)n * rtm::kBlock * 4, cudaMemcpyDeviceToHost, a->st);
  if (latent) cudaMemcpyAsync(latent, a->y[3], (size_t)n * rtm::kLatent * 4, cudaMemcpyDeviceToHost, a->st);
  return cudaStreamSynchronize(a->st) == cudaSuccess ? RTM_OK : RTM_ERR_CUDA;
}

int rtm_ae_compress_volume(rtm_ae *a, const float *d_vol, int nx, int ny, int nz, void *d_latent, float *d_scales,
                           void *stream) {
  if (!a || !d_vol || !d_latent || !d_scales || nx < 1 || ny < 1 || nz < 1) return RTM_ERR_ARG;
  cudaSetDevice(a->device);
  return rtm::ae_compress(a, d_vol, nx, ny, nz, d_latent, d_scales, (cudaStream_t)stream);
}

int rtm_ae_decompress_volume(rtm_ae *a, const void *d_latent, const float *d_scales, int nx, int ny, int nz,
                             float *d_vol, void *stream) {
  if (!a || !d_vol || !d_latent || !d_scales || nx < 1 || ny < 1 || nz < 1) return RTM_ERR_ARG;
  cudaSetDevice(a->device);
  return rtm::ae_decompress(a, d_latent, d_scales, nx, ny, nz, d_vol, (cudaStream_t)stream);
}

}  // extern "C"
