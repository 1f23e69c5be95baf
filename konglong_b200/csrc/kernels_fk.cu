// kernels_fk.cu - receiver FK true-amplitude / deghost spreading on sm_100a:
// Receiver::spread_sdomain (bgprtm/Receiver.cpp:851-1010), the space-domain
// form Receiver::spread selects by default (:1012-1041).
//   1. every trace is spread onto the (ny, nx) receiver grid with its
//      separable x / y kernels (spreadCoeffs :306-363, apply_src_coefxy
//      :509-530: wf += (trace * kx) * ky; atomic adds, receivers overlap),
//      zero-padded to ntfft samples;
//   2. forward real FFT over (y, x, t) (cuFFT, unnormalised);
//   3. one thread per bin: kx / ky of get_wavenumber (:605-617), k = iw dwv,
//      tmp = 1 - (kx^2 + ky^2) / k^2; DC and evanescent bins (tmp <= 0) are
//      zeroed; factor = (trueamp ? sqrt(tmp) : 1) * sqrt(1 / (nx ny ntfft));
//      with deghost factor *= (kzdz >= pi/2 ? 1 : sin(kzdz) <= thr ? 1/thr :
//      1/sin(kzdz)) / 2 (kzdz = k sqrt(tmp) z), the low-cut ramp, and the bin is
//      multiplied by i factor side (:957-977), otherwise by factor.  The float
//      operations are the reference's, one rounding each (no contraction).
//      With deghost the Nyquist frequency plane (even ntfft) comes out
//      anti-Hermitian in (ky, kx); an inverse real FFT reads only part of it,
//      differently from one library to another, so it is zeroed (band-limited
//      data carry nothing there);
//   4. inverse real FFT (unnormalised) and the first nt samples per column.
// The wavenumber-domain form Receiver::spread_kdomain (:641-849) replaces
// steps 1-2: each trace, scaled by sqrt(1 / (nx ny ntfft)), is transformed in
// time (batched cuFFT R2C) and summed into the (ky, kx) grid with the phase
// shifts exp(-i (kx x + ky y)) of its offset from the grid origin and the k
// tapers (get_ktaper :619-639) - a complex GEMM spectrum[k][w] = sum_r
// S[k][r] T[r][w], with S built in chunks of wavenumbers by a kernel and the
// products run by cuBLAS (pedantic FP32); step 3 omits the scalar and scales
// the ghost threshold by sin(2 pi fmax z / vsurf) when that angle is below
// pi / 2 (:792-794).  nx > 1: with nx = 1 the reference's x taper is 0 / 0.
// libfftv::padfftv (the choice of ntfft) is absent from the reference tree;
// ntfft is the caller's.
#include <cublas_v2.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "host_setup.h"
#include "rtm_b200.h"

namespace rtm {
namespace {

__global__ void fk_spread_k(const float *__restrict__ tr, int nt, const int *__restrict__ ox, const int *__restrict__ lx,
                            const float *__restrict__ kx, const int *__restrict__ oy, const int *__restrict__ ly,
                            const float *__restrict__ ky, int LX, int LY, int nx, int ntfft, float *__restrict__ g) {
  const int r = blockIdx.x, ij = blockIdx.y;
  const int i = ij % LX, j = ij / LX;
  if (i >= lx[r] || j >= ly[r]) return;
  const float cx = kx[(size_t)r * LX + i], cy = ky[(size_t)r * LY + j];
  float *col = g + ((size_t)(oy[r] + j) * nx + ox[r] + i) * ntfft;
  const float *t = tr + (size_t)r * nt;
  for (int it = threadIdx.x; it < nt; it += blockDim.x) atomicAdd(col + it, __fmul_rn(__fmul_rn(t[it], cx), cy));
}

struct FkConst {
  int nx, ny, nw, ntfft, trueamp, deghost, iw_lc, iw_lp;
  float dkx, dky, dwv, scalar, z, thr, side;
};

__device__ __forceinline__ float fk_wavenumber(int i, int n, float dk) {
  return n == 1 ? 0.f : __fmul_rn((float)(i < n / 2 + 1 ? i : i - n), dk);
}

__global__ void fk_filter_k(float2 *__restrict__ s, FkConst c) {
  const long long total = (long long)c.ny * c.nx * c.nw;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int iw = (int)(t % c.nw);
    const int ix = (int)((t / c.nw) % c.nx), iy = (int)(t / ((long long)c.nw * c.nx));
    float2 v = s[t];
    if (iw == 0 || (c.deghost && c.ntfft % 2 == 0 && iw == c.nw - 1)) {
      s[t] = make_float2(0.f, 0.f);
      continue;
    }
    const float kx = fk_wavenumber(ix, c.nx, c.dkx), ky = fk_wavenumber(iy, c.ny, c.dky);
    const float k = __fmul_rn((float)iw, c.dwv);
    const float tmp = __fsub_rn(1.0f, __fdiv_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(k, k)));
    if (!(tmp > 0.f)) {
      s[t] = make_float2(0.f, 0.f);
      continue;
    }
    const float cosv = __fsqrt_rn(tmp);
    float f = __fmul_rn(c.trueamp ? cosv : 1.0f, c.scalar);
    if (c.deghost) {
      const float kzdz = __fmul_rn(__fmul_rn(k, cosv), c.z);
      const float sinv = sinf(kzdz);
      f = __fmul_rn(f, kzdz >= 1.57079632679489661923f ? 1.0f
                       : sinv <= c.thr                 ? __fdiv_rn(1.0f, c.thr)
                                                       : __fdiv_rn(1.0f, sinv));
      f = __fmul_rn(f, 0.5f);
      if (iw <= c.iw_lc) {
        f = 0.f;
      } else if (iw <= c.iw_lp) {
        const float a = __fdiv_rn(__fmul_rn(3.14159265358979323846f, (float)(iw - c.iw_lc)), (float)(c.iw_lp - c.iw_lc + 1));
        f = __fmul_rn(f, __fmul_rn(0.5f, __fsub_rn(1.0f, cosf(a))));
      }
      const float m = __fmul_rn(f, c.side);  // times i m
      v = make_float2(-__fmul_rn(v.y, m), __fmul_rn(v.x, m));
    } else {
      v = make_float2(__fmul_rn(v.x, f), __fmul_rn(v.y, f));
    }
    s[t] = v;
  }
}

// S[k][r] for wavenumbers k0 .. k0 + nk - 1 (k = iky nx + ikx):
// ((shift_x * taper_x) * shift_y) * taper_y, shift = cos(ph) - i sin(ph)
__global__ void fk_shift_k(const float *__restrict__ xm, const float *__restrict__ ym, int nr, const float *__restrict__ kx,
                           const float *__restrict__ ky, const float *__restrict__ tx, const float *__restrict__ ty,
                           int nx, int ny, long long k0, int nk, float2 *__restrict__ S) {
  const long long total = (long long)nk * nr;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t % nr);
    const long long k = k0 + t / nr;
    const int ikx = (int)(k % nx), iky = (int)(k / nx);
    const float px = __fmul_rn(xm[r], kx[ikx]);
    float2 v = make_float2(__fmul_rn(cosf(px), tx[ikx]), __fmul_rn(-sinf(px), tx[ikx]));
    if (ny > 1) {
      const float py = __fmul_rn(ym[r], ky[iky]);
      const float c = cosf(py), sn = -sinf(py);
      v = make_float2(__fsub_rn(__fmul_rn(v.x, c), __fmul_rn(v.y, sn)), __fadd_rn(__fmul_rn(v.x, sn), __fmul_rn(v.y, c)));
      v = make_float2(__fmul_rn(v.x, ty[iky]), __fmul_rn(v.y, ty[iky]));
    }
    S[t] = v;
  }
}

// get_wavenumber and get_ktaper (Receiver.cpp:605-639) in the reference's arithmetic
void fk_wavenumbers(int n, float dk, float k1, float k2, std::vector<float> &k, std::vector<float> &taper) {
  k.assign(n, 0.f), taper.assign(n, 0.f);
  if (n > 1)
    for (int i = 0; i < n; i++) k[i] = (float)(i < n / 2 + 1 ? i : i - n) * dk;
  const float kmax = std::fabs(k[n / 2]);
  const float kmax1 = kmax * k1 * 2, kmax2 = kmax * k2 * 2;
  for (int i = 0; i < n; i++) {
    const float ak = std::fabs(k[i]);
    if (ak < kmax1) taper[i] = 1.0f;
    else if (ak > kmax2) taper[i] = 0.0f;
    else {
      const float tmp = (ak - kmax1) / (kmax2 - kmax1) * M_PI / 2.0;
      taper[i] = std::cos(tmp) * std::cos(tmp);
    }
  }
}

// a cuFFT plan over the dimensions of the grid that exceed one cell, then t
cufftResult fk_plan(cufftHandle *p, int ny, int nx, int ntfft, cufftType type) {
  int dims[3], r = 0;
  if (ny > 1) dims[r++] = ny;
  if (nx > 1) dims[r++] = nx;
  dims[r++] = ntfft;
  return cufftPlanMany(p, r, dims, nullptr, 1, 0, nullptr, 1, 0, type, 1);
}

}  // namespace
}  // namespace rtm

extern "C" int rtm_fk_spread(const rtm_fk_args *a, int nr, const float *xy, const float *traces, float *out) {
  using namespace rtm;
  if (!a || !out || nr < 0 || (nr > 0 && (!xy || !traces)) || a->nx < 1 || a->ny < 1 || a->nt < 1 ||
      a->ntfft < a->nt || !(a->dt > 0.f) || !(a->dx > 0.f) || !(a->dy > 0.f) || !(a->vsurf > 0.f) ||
      (a->side != 1 && a->side != -1) || !(a->ghost_threshold > 0.f) || !(a->khpass > 0.f) || a->khpass > a->khcut ||
      a->khcut > 0.5f || a->nlimit < 1 || (a->domain != 0 && a->domain != 1) || (a->domain == 1 && a->nx < 2) ||
      (a->domain == 1 && a->khpass == a->khcut))
    return RTM_ERR_ARG;
  const bool kdom = a->domain == 1;
  const int nx = a->nx, ny = a->ny, nt = a->nt, ntfft = a->ntfft, nw = ntfft / 2 + 1;
  const size_t ncol = (size_t)nx * ny;
  for (int r = 0; r < nr; r++) {
    const float x = xy[2 * r], y = xy[2 * r + 1];
    if (!std::isfinite(x) || !std::isfinite(y) || x < 0.f || x > (float)(nx - 1) || y < 0.f || y > (float)(ny - 1))
      return RTM_ERR_ARG;
  }
  const float dkx = nx == 1 ? 0.f : (float)(2.0f * M_PI / (double)(a->dx * (float)nx));
  const float dky = ny == 1 ? 0.f : (float)(2.0f * M_PI / (double)(a->dy * (float)ny));
  const float scalar = (float)std::sqrt(1.0 / nx / ny / ntfft);
  float *g = nullptr, *dtr = nullptr, *dkx_ = nullptr, *dky_ = nullptr, *dk = nullptr;
  int *dint = nullptr;
  float2 *spec = nullptr, *T = nullptr, *S = nullptr;
  cufftHandle fwd = 0, inv = 0;
  cublasHandle_t blas = nullptr;
  int made = 0;
  cudaStream_t st = nullptr;
  auto done = [&](int code) {
    if (made & 1) cufftDestroy(fwd);
    if (made & 2) cufftDestroy(inv);
    if (blas) cublasDestroy(blas);
    for (void *p : {(void *)g, (void *)dtr, (void *)dkx_, (void *)dky_, (void *)dk, (void *)dint, (void *)spec,
                    (void *)T, (void *)S})
      if (p) cudaFree(p);
    if (st) cudaStreamDestroy(st);
    if (code != RTM_OK) cudaGetLastError();
    return code;
  };
  if (cudaStreamCreate(&st) != cudaSuccess) return done(RTM_ERR_CUDA);  // blocking: after the legacy-stream uploads
  if (cudaMalloc(&g, ncol * ntfft * 4) != cudaSuccess || cudaMalloc(&spec, ncol * nw * sizeof(float2)) != cudaSuccess)
    return done(RTM_ERR_NOMEM);
  if (fk_plan(&inv, ny, nx, ntfft, CUFFT_C2R) != CUFFT_SUCCESS) return done(RTM_ERR_CUDA);
  made |= 2;
  if (cufftSetStream(inv, st) != CUFFT_SUCCESS) return done(RTM_ERR_CUDA);
  if (!kdom) {
    // 1-2: grid spreading (the engine's spread kernels) and the forward FFT over (y, x, t)
    const int LX = nx == 1 ? 1 : a->nlimit, LY = ny == 1 ? 1 : a->nlimit;
    std::vector<int> ints(4 * (size_t)nr);
    int *ox = ints.data(), *lx = ox + nr, *oy = lx + nr, *ly = oy + nr;
    std::vector<float> kx((size_t)nr * LX, 0.f), ky((size_t)nr * LY, 0.f);
    for (int r = 0; r < nr; r++) {
      lx[r] = LX, ly[r] = LY;
      ox[r] = spread_coeffs(nx, xy[2 * r], a->khpass, a->khcut, &lx[r], 0, nx > 1 ? 10 : 0, &kx[(size_t)r * LX]);
      oy[r] = spread_coeffs(ny, xy[2 * r + 1], a->khpass, a->khcut, &ly[r], 0, ny > 1 ? 10 : 0, &ky[(size_t)r * LY]);
    }
    if (cudaMalloc(&dtr, std::max<size_t>(1, (size_t)nr * nt) * 4) != cudaSuccess ||
        cudaMalloc(&dkx_, std::max<size_t>(1, kx.size()) * 4) != cudaSuccess ||
        cudaMalloc(&dky_, std::max<size_t>(1, ky.size()) * 4) != cudaSuccess ||
        cudaMalloc(&dint, std::max<size_t>(1, ints.size()) * 4) != cudaSuccess)
      return done(RTM_ERR_NOMEM);
    if (fk_plan(&fwd, ny, nx, ntfft, CUFFT_R2C) != CUFFT_SUCCESS) return done(RTM_ERR_CUDA);
    made |= 1;
    if (cufftSetStream(fwd, st) != CUFFT_SUCCESS) return done(RTM_ERR_CUDA);
    cudaMemsetAsync(g, 0, ncol * ntfft * 4, st);
    if (nr > 0) {
      cudaMemcpyAsync(dtr, traces, (size_t)nr * nt * 4, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(dkx_, kx.data(), kx.size() * 4, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(dky_, ky.data(), ky.size() * 4, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(dint, ints.data(), ints.size() * 4, cudaMemcpyHostToDevice, st);
      fk_spread_k<<<dim3(nr, LX * LY), 128, 0, st>>>(dtr, nt, dint, dint + nr, dkx_, dint + 2 * nr, dint + 3 * nr,
                                                     dky_, LX, LY, nx, ntfft, g);
    }
    if (cufftExecR2C(fwd, g, (cufftComplex *)spec) != CUFFT_SUCCESS) return done(RTM_ERR_CUDA);
  } else {
    // 1-2 (k domain): scaled traces to the frequency domain, then the phase-shift sums as complex GEMMs
    std::vector<float> kx, ky, tx, ty, off(2 * (size_t)nr);
    fk_wavenumbers(nx, dkx, a->khpass, a->khcut, kx, tx);
    fk_wavenumbers(ny, dky, a->khpass, a->khcut, ky, ty);
    for (int r = 0; r < nr; r++) off[r] = xy[2 * r] * a->dx, off[nr + r] = xy[2 * r + 1] * a->dy;
    std::vector<float> ts((size_t)nr * nt);
    for (size_t i = 0; i < ts.size(); i++) ts[i] = traces[i] * scalar;
    const size_t ktab = 2 * (size_t)nx + 2 * (size_t)ny + off.size();
    long long kchunk = std::max<long long>(1, std::min<long long>((long long)ncol, (256LL << 20) / 8 / std::max(1, nr)));
    if (cudaMalloc(&dtr, std::max<size_t>(1, (size_t)nr * ntfft) * 4) != cudaSuccess ||
        cudaMalloc(&T, std::max<size_t>(1, (size_t)nr * nw) * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&S, std::max<size_t>(1, (size_t)kchunk * nr) * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&dk, ktab * 4) != cudaSuccess)
      return done(RTM_ERR_NOMEM);
    float *d_kx = dk, *d_ky = d_kx + nx, *d_tx = d_ky + ny, *d_ty = d_tx + nx, *d_off = d_ty + ny;
    cudaMemcpyAsync(d_kx, kx.data(), nx * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_ky, ky.data(), ny * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_tx, tx.data(), nx * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_ty, ty.data(), ny * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(spec, 0, ncol * nw * sizeof(float2), st);
    if (nr > 0) {
      cudaMemsetAsync(dtr, 0, (size_t)nr * ntfft * 4, st);
      cudaMemcpy2DAsync(dtr, (size_t)ntfft * 4, ts.data(), (size_t)nt * 4, (size_t)nt * 4, nr, cudaMemcpyHostToDevice,
                        st);
      int n1 = ntfft;
      if (cufftPlanMany(&fwd, 1, &n1, nullptr, 1, ntfft, nullptr, 1, nw, CUFFT_R2C, nr) != CUFFT_SUCCESS)
        return done(RTM_ERR_CUDA);
      made |= 1;
      if (cufftSetStream(fwd, st) != CUFFT_SUCCESS || cufftExecR2C(fwd, dtr, (cufftComplex *)T) != CUFFT_SUCCESS)
        return done(RTM_ERR_CUDA);
      if (cublasCreate(&blas) != CUBLAS_STATUS_SUCCESS) {
        blas = nullptr;
        return done(RTM_ERR_CUDA);
      }
      if (cublasSetStream(blas, st) != CUBLAS_STATUS_SUCCESS ||
          cublasSetMathMode(blas, CUBLAS_PEDANTIC_MATH) != CUBLAS_STATUS_SUCCESS)
        return done(RTM_ERR_CUDA);
      const cuComplex one = make_cuComplex(1.f, 0.f), zero = make_cuComplex(0.f, 0.f);
      for (long long k0 = 0; k0 < (long long)ncol; k0 += kchunk) {
        const int nk = (int)std::min<long long>(kchunk, (long long)ncol - k0);
        const long long tot = (long long)nk * nr;
        fk_shift_k<<<(unsigned)std::min<long long>((tot + 255) / 256, 148LL * 16), 256, 0, st>>>(
            d_off, d_off + nr, nr, d_kx, d_ky, d_tx, d_ty, nx, ny, k0, nk, S);
        if (cublasCgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, nw, nk, nr, &one, (const cuComplex *)T, nw,
                        (const cuComplex *)S, nr, &zero, (cuComplex *)(spec + k0 * nw), nw) != CUBLAS_STATUS_SUCCESS)
          return done(RTM_ERR_CUDA);
      }
    }
  }
  // 3: the per-bin product
  FkConst c{};
  c.nx = nx, c.ny = ny, c.nw = nw, c.ntfft = ntfft, c.trueamp = a->trueamp != 0, c.deghost = a->deghost != 0;
  c.dkx = dkx, c.dky = dky;
  c.dwv = (float)(2.0f * M_PI / (double)(a->dt * (float)ntfft * a->vsurf));
  c.scalar = kdom ? 1.0f : scalar;
  c.iw_lc = (int)nearbyintf(a->flcut * a->dt * (float)ntfft);
  c.iw_lp = (int)nearbyintf(a->flpass * a->dt * (float)ntfft);
  c.z = a->z, c.thr = a->ghost_threshold, c.side = (float)a->side;
  if (kdom) {
    const float kzdzmax = a->fmax * 6.28318530717958647692f / a->vsurf * a->z;
    if (kzdzmax < 1.57079632679489661923f) c.thr *= sinf(kzdzmax);
  }
  const long long bins = (long long)ncol * nw;
  fk_filter_k<<<(unsigned)std::min<long long>((bins + 255) / 256, 148LL * 16), 256, 0, st>>>(spec, c);
  // 4: back to (y, x, t), the first nt samples of each column
  if (cufftExecC2R(inv, (cufftComplex *)spec, g) != CUFFT_SUCCESS) return done(RTM_ERR_CUDA);
  if (cudaMemcpy2DAsync(out, (size_t)nt * 4, g, (size_t)ntfft * 4, (size_t)nt * 4, ncol, cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return done(RTM_ERR_CUDA);
  return done(cudaGetLastError() == cudaSuccess ? RTM_OK : RTM_ERR_CUDA);
}
