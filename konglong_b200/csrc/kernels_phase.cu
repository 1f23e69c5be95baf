// kernels_phase.cu - time-dispersion / phase correction of traces on sm_100a:
// PhaseCorrection (bgprtm/PhaseCorrection.cpp:14-235).
//   init (:62-115): the table T[iw][it] = exp(i phs(iw, it)) * factor(iw) for
//     the band iw < nw1 (up to fmax) and it < nt_dft, built on the host in
//     float with the reference's operation order and types (row blocks on
//     host threads); on the device as
//     rows 2 iw (real parts) and 2 iw + 1 (imaginary parts) of one matrix.
//   fft_dft (:141-190): zero-padded forward transform (cuFFT R2C, conjugated:
//     libfftv's forward carries exp(+i w t)), Nyquist cleared, the band's bins
//     times c_phase * factor * scaler, bin 0 real; with the table
//     out[it] = sum_iw Re(X) Re(T) - Im(X) Im(T) (bin 0 halved), the product
//     [ntr][2 nw1] x [2 nw1][nt_dft]; without it the inverse transform (cuFFT
//     C2R of the conjugate: libfftv's backward carries exp(-i w t)) and its
//     first nt_dft samples.
//   dft_fft (:192-235): with the table X[iw] = sum_it x[it] conj(T[iw][it]),
//     the product [ntr][nt] x [nt][2 nw1], else the forward transform; then the
//     same scaling, the inverse transform and its first nt samples.
// libfftv is absent from the reference tree: the packing (Nyquist in bin 0's
// imaginary part, cleared by every reference path), the signs and the
// unnormalised inverse are inferred from these call sites.  The product
// kernel sums each output in the reference's order (over iw the real term
// then the imaginary term; over it), one FMA per term.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "rtm_b200.h"

namespace rtm {
namespace {

constexpr float kPcPi = 3.14159265358979323846f;  // FLT_PI of the reference's libCommon
constexpr int kPcBM = 64, kPcBN = 64, kPcBK = 16;

// C[m][n] = sum_k A[m][k] B(k, n), B(k, n) at B[k * sk + n * sn]; 64 x 64
// tiles, 256 threads with 4 x 4 outputs each, k in chunks of 16 through
// shared memory; the sum of each output runs over k in order.
__global__ void __launch_bounds__(256) pc_gemm_k(const float *__restrict__ A, long long lda,
                                                 const float *__restrict__ B, long long sk, long long sn,
                                                 float *__restrict__ C, long long ldc, int M, int N, int K) {
  __shared__ float As[kPcBK][kPcBM + 4];
  __shared__ float Bs[kPcBK][kPcBN + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const long long m0 = (long long)blockIdx.x * kPcBM;
  const int n0 = blockIdx.y * kPcBN;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
  for (int k0 = 0; k0 < K; k0 += kPcBK) {
    for (int e = threadIdx.x; e < kPcBM * kPcBK; e += 256) {
      const int mm = e / kPcBK, kk = e % kPcBK;
      const long long m = m0 + mm;
      const int k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? A[m * lda + k] : 0.f;
    }
    for (int e = threadIdx.x; e < kPcBK * kPcBN; e += 256) {
      int kk, nn;
      if (sn == 1) kk = e / kPcBN, nn = e % kPcBN;  // rows of B contiguous in n
      else nn = e / kPcBK, kk = e % kPcBK;          // columns contiguous in k
      const int k = k0 + kk, n = n0 + nn;
      Bs[kk][nn] = (k < K && n < N) ? B[(long long)k * sk + (long long)n * sn] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kPcBK; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = __fmaf_rn(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const long long m = m0 + ty + 16 * i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int n = n0 + tx + 16 * j;
      if (n < N) C[m * ldc + n] = acc[i][j];
    }
  }
}

struct PcSpec {
  int ntr, nw, nw1, nyq;
  int src;     // 0: cuFFT R2C spectrum [ntr][nw]; 1: product output [ntr][2 nw1] (dft_fft's table sum)
  int dst;     // 0: cuFFT C2R input [ntr][nw]; 1: product input [ntr][2 nw1] (fft_dft's table sum)
  int halve0;  // fft_dft with the table: bin 0 halved
};

// One thread per bin: the spectrum in libfftv's sign convention, the Nyquist
// bin and bin 0's imaginary part cleared, the band's bins times mul[iw]
// (c_phase * factor * scaler), bin 0 made real again (and halved), written
// where the next step reads it.  Bins above the band keep the transform's
// values (zero for the table sum), as in the reference.
__global__ void pc_spectrum_k(const float2 *__restrict__ spec, const float *__restrict__ gout,
                              const float2 *__restrict__ mul, float2 *c2r, float *gin, PcSpec s) {
  const int nb = s.dst == 1 ? s.nw1 : s.nw;
  const long long total = (long long)s.ntr * nb;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long tr = i / nb;
    const int iw = (int)(i % nb);
    float xr = 0.f, xi = 0.f;
    if (s.src == 0) {
      const float2 v = spec[tr * s.nw + iw];
      xr = v.x, xi = -v.y;
    } else if (iw < s.nw1) {
      const float *c = gout + tr * 2 * s.nw1 + 2 * iw;
      xr = c[0], xi = -c[1];  // sum x conj(T): the product gives Re and -Im
    }
    if (iw == s.nyq) xr = 0.f, xi = 0.f;
    if (iw == 0) xi = 0.f;
    if (iw < s.nw1) {
      const float2 m = mul[iw];
      const float r = __fsub_rn(__fmul_rn(xr, m.x), __fmul_rn(xi, m.y));
      const float q = __fadd_rn(__fmul_rn(xr, m.y), __fmul_rn(xi, m.x));
      xr = r, xi = q;
    }
    if (iw == 0) {
      xi = 0.f;
      if (s.halve0) xr *= 0.5f;
    }
    if (s.dst == 0) c2r[tr * s.nw + iw] = make_float2(xr, -xi);
    else {
      float *g = gin + tr * 2 * s.nw1 + 2 * iw;
      g[0] = xr, g[1] = -xi;  // Re(X) Re(T) + (-Im(X)) Im(T)
    }
  }
}

// out[tr][it] *= scaler for it < n (rows of pitch `pitch`)
__global__ void pc_scale_k(float *y, long long pitch, int ntr, int n, float scaler) {
  const long long total = (long long)ntr * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    y[(i / n) * pitch + i % n] *= scaler;
}

unsigned pc_blocks(long long n) { return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 16)); }

double dsp_acos(double x) { return acos(1 - 0.5 * x * x) - x; }  // arccos(1 - x^2 / 2) - x (:53-55)
double dsp_sin(double x) { return x - 2. * sin(x / 2.0); }         // x - 2 sin(x / 2) (:58-60)

float round_down_angle(float angle) {  // the angle less the nearest multiple of 2 pi (:45-48)
  const int n = (int)nearbyintf(angle / (2 * kPcPi));
  return angle - n * 2 * kPcPi;
}

// The constructor's and init()'s derived quantities.
struct PcPlan {
  int nt, ntfft, nw, nw1, nt_dft, tdsp;
  bool resample, do_fft_dft, identity;
  std::vector<float> table;  // [2 nw1][nt_dft]: rows of Re(T), Im(T)
  std::vector<float2> mul;   // [nw1]: c_phase * factor(w_pow) * (1 / ntfft)
};

void pc_plan(const rtm_phase_args &a, PcPlan &p) {
  const int dir = a.direction;
  const float phase = a.phase_deg * kPcPi / 180;
  const float cpr = cosf(-phase), cpi = sinf(-phase);  // c_phase = exp(-i phase) (:19)
  p.nt = a.nt, p.ntfft = a.ntfft, p.nw = a.ntfft / 2 + 1;
  const int skip = a.skip_tdsp_correction & dir;
  p.tdsp = a.do_tdsp ? a.tdsp_correction : 0;
  p.resample = a.dt_out > 0 && a.nt_out > 0;
  float t0_out = a.t0_out, t_shift, dt_dft;
  if (p.resample) p.nt_dft = a.nt_out, dt_dft = a.dt_out, t_shift = a.t0_out - a.t0;
  else p.nt_dft = a.nt, dt_dft = a.dt, t_shift = 0, t0_out = a.t0 + t_shift;
  const int it_shift = (int)(t_shift / dt_dft);
  const float t_shift_frac = t_shift - it_shift * dt_dft;
  p.identity = !p.tdsp && a.w_pow == 0 && phase == 0;
  // init (:62-115)
  p.do_fft_dft = dir == 2;
  if (a.transform == 1) p.do_fft_dft = true;
  else if (a.transform == 2) p.do_fft_dft = false;
  const bool jacobian = dir == 1 && !skip && !a.skip_jacobian;
  const float it0 = (p.do_fft_dft ? t0_out : a.t0) / dt_dft;
  const double dw = 2.0 * M_PI / (a.ntfft * a.dt);
  p.nw1 = std::min(p.nw, (int)nearbyintf((float)(2.0f * kPcPi * a.fmax / dw)) + 1);
  const int nw1 = p.nw1, nt_dft = p.nt_dft;
  const float ratio = a.tdsp_acos_ratio;
  // rows iw0 .. iw1 - 1 of the table; rows are independent, so the row
  // blocks run on host threads and the table is the same bit for bit
  auto rows = [&](int iw0, int iw1) {
    for (int iw = iw0; iw < iw1; iw++) {
      const double x = (double)iw * dw * a.Dt;
      const float factor = jacobian ? 2.0f * cosf((float)(x / 2)) : 2.0f;
      const float dsp =
          (a.Dt == 0 || skip) ? 0.f : (float)((ratio * dsp_acos(x) + (1 - ratio) * dsp_sin(x)) * dt_dft / a.Dt);
      float *tr = &p.table[(size_t)2 * iw * nt_dft], *ti = tr + nt_dft;
      for (int it = 0; it < nt_dft; it++) {
        float phs;
        if (a.dt == dt_dft) {
          const float lin = (it - it0) * dsp;
          phs = (float)(lin - (double)(((long)(it - it_shift) * iw) % a.ntfft) * dw * dt_dft + t_shift_frac * iw * dw);
        } else {
          phs = (it - it0) * dsp - (float)dw * dt_dft * it * iw + (float)dw * t_shift * iw;
          phs = round_down_angle(phs);
        }
        tr[it] = cosf(phs) * factor;
        ti[it] = sinf(phs) * factor;
      }
    }
  };
  if (p.tdsp) {
    p.table.assign((size_t)2 * nw1 * nt_dft, 0.f);
    const long long work = (long long)nw1 * nt_dft;
    const int nth = (int)std::min<long long>({(long long)std::max(1u, std::thread::hardware_concurrency()), 16LL,
                                              work / (1LL << 16) + 1, (long long)nw1});
    std::vector<std::thread> th;
    int handed = 0;  // rows given to threads
    try {
      for (int t = 0; t < nth - 1; t++) {
        const int r1 = (int)((long long)nw1 * (t + 1) / nth);
        th.emplace_back(rows, handed, r1);
        handed = r1;
      }
    } catch (...) {  // no more threads: this one takes the rest
    }
    rows(handed, nw1);
    for (auto &t : th) t.join();
  }
  // the band's spectral multipliers of fft_dft / dft_fft (:158-163, :210-214)
  const float dwf = (float)(2.0f * M_PI / (a.ntfft * a.dt)), scaler = 1.0f / a.ntfft;
  p.mul.resize(nw1);
  for (int iw = 0; iw < nw1; iw++) {
    const float f = (a.w_pow == 0) ? 1.f : (iw == 0) ? 0.f : powf(iw * dwf, a.w_pow);
    p.mul[iw] = make_float2(cpr * f * scaler, cpi * f * scaler);
  }
}

}  // namespace
}  // namespace rtm

extern "C" int rtm_phase_correct(const rtm_phase_args *a, int apply, int ntr, const float *in, float *out,
                                 float scaler) {
  using namespace rtm;
  if (!a || ntr < 0 || (ntr > 0 && (!in || !out)) || (apply != 1 && apply != 2) || a->nt < 1 || !(a->dt > 0.f) ||
      !(a->Dt >= 0.f) || !(a->fmax >= 0.f) || a->direction < 0 || a->direction > 2 || a->ntfft < a->nt ||
      a->ntfft < 2 || (a->ntfft & 1) || a->tdsp_correction < 0 || a->transform < 0 || a->transform > 2 ||
      !std::isfinite(a->t0) || !std::isfinite(a->w_pow) || !std::isfinite(a->phase_deg) ||
      !std::isfinite(a->tdsp_acos_ratio) || !std::isfinite(scaler) ||
      (a->dt_out > 0.f && a->nt_out > 0 && !std::isfinite(a->t0_out)))
    return RTM_ERR_ARG;
  if (apply == 1 && a->direction != 1) return RTM_ERR_ARG;  // applyForward asserts FWD (:117)
  if (a->dt_out > 0.f && a->nt_out > 0 && (a->nt_out + kPcBN - 1) / kPcBN > 65535) return RTM_ERR_ARG;
  if ((a->nt + kPcBN - 1) / kPcBN > 65535 || (a->ntfft / 2 + 1) > 65535 * kPcBN / 2) return RTM_ERR_ARG;
  PcPlan p;
  try {
    pc_plan(*a, p);
  } catch (...) {  // the host table
    return RTM_ERR_NOMEM;
  }
  const int nt = a->nt, N = p.ntfft, nw = p.nw, nw1 = p.nw1, nt_dft = p.nt_dft;
  if (p.identity) {  // the no-op of applyForward / applyBackward (:118, :129-132)
    if (p.resample) return RTM_ERR_ARG;
    if (ntr > 0 && out != in) std::memmove(out, in, (size_t)ntr * nt * 4);
    return RTM_OK;
  }
  if (apply == 1 && p.resample) return RTM_ERR_ARG;
  // applyForward (:116-126) / applyBackward (:128-140)
  const bool fft_dft = apply == 1 ? (p.do_fft_dft && p.tdsp == 1) : (p.do_fft_dft || p.tdsp != 1);
  if (!fft_dft && p.resample) return RTM_ERR_ARG;  // dft_fft asserts no resampling (:193)
  if (fft_dft && !p.tdsp && nt_dft > N) return RTM_ERR_ARG;
  const int nout = fft_dft ? nt_dft : nt;  // samples per output trace
  if (ntr == 0) return RTM_OK;
  float *x = nullptr, *gin = nullptr, *gout = nullptr, *tab = nullptr;
  float2 *spec = nullptr, *mul = nullptr;
  cufftHandle fwd = 0, inv = 0;
  int made = 0;
  cudaStream_t st = nullptr;
  auto done = [&](int code) {
    if (made & 1) cufftDestroy(fwd);
    if (made & 2) cufftDestroy(inv);
    for (void *q : {(void *)x, (void *)gin, (void *)gout, (void *)tab, (void *)spec, (void *)mul})
      if (q) cudaFree(q);
    if (st) cudaStreamDestroy(st);
    if (code != RTM_OK) cudaGetLastError();
    return code;
  };
  const size_t R = (size_t)ntr;
  if (cudaStreamCreate(&st) != cudaSuccess) return done(RTM_ERR_CUDA);
  if (cudaMalloc(&x, R * N * 4) != cudaSuccess || cudaMalloc(&spec, R * nw * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&mul, (size_t)nw1 * sizeof(float2)) != cudaSuccess)
    return done(RTM_ERR_NOMEM);
  if (p.tdsp && (cudaMalloc(&tab, p.table.size() * 4) != cudaSuccess ||
                 cudaMalloc(&gin, R * 2 * nw1 * 4) != cudaSuccess ||
                 cudaMalloc(&gout, R * std::max(nt_dft, 2 * nw1) * 4) != cudaSuccess))
    return done(RTM_ERR_NOMEM);
  int n1 = N;
  if (cufftPlanMany(&inv, 1, &n1, nullptr, 1, nw, nullptr, 1, N, CUFFT_C2R, ntr) != CUFFT_SUCCESS)
    return done(RTM_ERR_CUDA);
  made |= 2;
  if (cufftPlanMany(&fwd, 1, &n1, nullptr, 1, N, nullptr, 1, nw, CUFFT_R2C, ntr) != CUFFT_SUCCESS)
    return done(RTM_ERR_CUDA);
  made |= 1;
  if (cufftSetStream(inv, st) != CUFFT_SUCCESS || cufftSetStream(fwd, st) != CUFFT_SUCCESS) return done(RTM_ERR_CUDA);
  cudaMemcpyAsync(mul, p.mul.data(), (size_t)nw1 * sizeof(float2), cudaMemcpyHostToDevice, st);
  if (p.tdsp) cudaMemcpyAsync(tab, p.table.data(), p.table.size() * 4, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(x, 0, R * N * 4, st);
  cudaMemcpy2DAsync(x, (size_t)N * 4, in, (size_t)nt * 4, (size_t)nt * 4, R, cudaMemcpyHostToDevice, st);
  PcSpec s{ntr, nw, nw1, N / 2, 0, 0, 0};
  const float *res = x;  // the result rows on the device
  long long pitch = N;
  if (fft_dft) {
    if (cufftExecR2C(fwd, x, (cufftComplex *)spec) != CUFFT_SUCCESS) return done(RTM_ERR_CUDA);
    if (p.tdsp) {
      s.src = 0, s.dst = 1, s.halve0 = 1;
      pc_spectrum_k<<<pc_blocks((long long)ntr * nw1), 256, 0, st>>>(spec, nullptr, mul, nullptr, gin, s);
      const dim3 g((unsigned)((ntr + kPcBM - 1) / kPcBM), (unsigned)((nt_dft + kPcBN - 1) / kPcBN));
      pc_gemm_k<<<g, 256, 0, st>>>(gin, 2 * nw1, tab, nt_dft, 1, gout, nt_dft, ntr, nt_dft, 2 * nw1);
      res = gout, pitch = nt_dft;
    } else {
      pc_spectrum_k<<<pc_blocks((long long)ntr * nw), 256, 0, st>>>(spec, nullptr, mul, spec, nullptr, s);
      if (cufftExecC2R(inv, (cufftComplex *)spec, x) != CUFFT_SUCCESS) return done(RTM_ERR_CUDA);
    }
  } else {
    if (p.tdsp) {
      const dim3 g((unsigned)((ntr + kPcBM - 1) / kPcBM), (unsigned)((2 * nw1 + kPcBN - 1) / kPcBN));
      pc_gemm_k<<<g, 256, 0, st>>>(x, N, tab, 1, nt_dft, gout, 2 * nw1, ntr, 2 * nw1, nt);
      s.src = 1;
      pc_spectrum_k<<<pc_blocks((long long)ntr * nw), 256, 0, st>>>(nullptr, gout, mul, spec, nullptr, s);
    } else {
      if (cufftExecR2C(fwd, x, (cufftComplex *)spec) != CUFFT_SUCCESS) return done(RTM_ERR_CUDA);
      pc_spectrum_k<<<pc_blocks((long long)ntr * nw), 256, 0, st>>>(spec, nullptr, mul, spec, nullptr, s);
    }
    if (cufftExecC2R(inv, (cufftComplex *)spec, x) != CUFFT_SUCCESS) return done(RTM_ERR_CUDA);
  }
  if (apply == 2 && scaler != 1.0f && a->nt_out > 0) {  // (:138-139)
    const int ns = std::min(a->nt_out, nout);
    pc_scale_k<<<pc_blocks((long long)ntr * ns), 256, 0, st>>>(const_cast<float *>(res), pitch, ntr, ns, scaler);
  }
  if (cudaMemcpy2DAsync(out, (size_t)nout * 4, res, (size_t)pitch * 4, (size_t)nout * 4, R, cudaMemcpyDeviceToHost,
                        st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return done(RTM_ERR_CUDA);
  return done(cudaGetLastError() == cudaSuccess ? RTM_OK : RTM_ERR_CUDA);
}
