// kernels_fft.cu - pseudo-spectral first derivative of the FFTWR2C engine
// (FdEngine_r2c, bgprtm/FdEngine_r2c.cpp) on sm_100a: every grid line along
// the axis goes through a real-to-complex FFT, bin j of the half spectrum is
// multiplied by i k_j, and a complex-to-real FFT brings it back.  The
// wavenumbers carry the 1 / n of the unnormalised inverse transform:
//   dk  = (float)(2 pi / (d n) * (1 / n))           (FdEngine_r2c.cpp:10-12)
//   k_j = -j dk for j <= n/2                        (assignW, :52-56)
//   bin j < n/2:  (re, im) -> (-k_j im, k_j re)     (fftderiv1_r2c, :222-226)
//   bin n/2:      the same times isign              (:228-231)
// For even n, bin n/2 is the Nyquist bin: the transform of a real line has no
// imaginary part there, so the product is real-free and the inverse transform
// (which reads only the real parts of the DC and Nyquist bins) drops it; the
// kernel writes zero there, and zero at DC (k_0 = 0).  For odd n, bin n/2 is
// the highest ordinary bin and keeps its isign factor.
//
// Layouts ([ny][nx][nz], z fastest): z lines are contiguous (batch nx ny,
// distance nz); y lines have stride nx nz and the batch is the nx nz
// contiguous columns (distance 1), so the half spectrum is [n/2+1][nx nz]
// and every access stays coalesced; x lines have stride nz with two batch
// strides (z and y), so each y plane is transposed to [nz][nx] through a
// shared-memory tile, transformed as contiguous lines and transposed back.
// cuFFT does the transforms; the bin products and the transposes are ours.
//
// FFTWR2R (FdEngine_r2r, bgprtm/FdEngine_r2r.cpp): the derivative of a line
// is a cosine (or sine) transform, a shifted bin product and the opposite
// inverse transform - one fixed n x n matrix per axis and pass (built on the
// host in FP64, host_setup.cpp).  Applied to every line at once it is a plain
// FP32 GEMM on the volume as it lies: z lines [nx ny][nz] x D^T, y lines
// D x [ny][nx nz], x lines D x [nx][nz] per y plane (strided batch); cuBLAS
// (pedantic FP32 math, workspace fixed for graph capture) runs them.
#include <cublas_v2.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "host_setup.h"
#include "kernel_api.h"
#include "rtm_b200.h"

namespace rtm {

namespace {

// bin products of one axis: bin j = (t / inner) % nh of the half spectrum
__global__ void fft_ik_k(float2 *__restrict__ s, const float *__restrict__ k, long long total, int nh, long long inner,
                         int n, float isign) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)((t / inner) % nh);
    const float2 v = s[t];
    float2 r;
    if (j == 0 || (j == n / 2 && n % 2 == 0)) {
      r = make_float2(0.f, 0.f);
    } else if (j == n / 2) {  // odd n: the last bin, with the isign factor
      const float kj = k[j];
      r = make_float2(__fmul_rn(__fmul_rn(-kj, v.y), isign), __fmul_rn(__fmul_rn(kj, v.x), isign));
    } else {
      const float kj = k[j];
      r = make_float2(__fmul_rn(-kj, v.y), __fmul_rn(kj, v.x));
    }
    s[t] = r;
  }
}

// Line filters of the double-grid imaging condition (libfftv's SHIFTHALF and
// HIGHTAPE filters): bin j of the half spectrum times
//   kind 0, half shift:  e^{i pi j / n} / n, so the inverse transform gives the
//          band-limited line at x + d/2 (the odd points of the doubled grid);
//          for even n the Nyquist bin is zero (its cosine vanishes at the
//          midpoints);
//   kind 1, high cut:    w(j / (n/2)) / n with w = 1 up to `high` of the
//          Nyquist wavenumber and a cosine roll-off to 0 at Nyquist.
__global__ void fft_filter_k(float2 *__restrict__ s, long long total, int nh, long long inner, int n, int kind,
                             float high) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)((t / inner) % nh);
    const float2 v = s[t];
    const float inv_n = 1.0f / float(n);
    float2 r;
    if (kind == 0) {
      if (n % 2 == 0 && j == n / 2) {
        r = make_float2(0.f, 0.f);
      } else {
        float sn, cs;
        sincospif(float(j) / float(n), &sn, &cs);
        r = make_float2((v.x * cs - v.y * sn) * inv_n, (v.x * sn + v.y * cs) * inv_n);
      }
    } else {
      const float q = float(j) / (0.5f * float(n));
      const float w = q <= high ? 1.0f : 0.5f * (1.0f + cospif(fminf((q - high) / (1.0f - high), 1.0f)));
      r = make_float2(v.x * w * inv_n, v.y * w * inv_n);
    }
    s[t] = r;
  }
}

// out[p][c][r] = in[p][r][c] for rows x cols planes (32 x 32 tiles)
__global__ void __launch_bounds__(256) transpose_k(const float *__restrict__ in, float *__restrict__ out, int rows,
                                                   int cols) {
  __shared__ float tile[32][33];
  const long long plane = (long long)blockIdx.z * rows * cols;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
#pragma unroll
  for (int k = 0; k < 32; k += 8) {
    const int r = r0 + ty + k, c = c0 + tx;
    if (r < rows && c < cols) tile[ty + k][tx] = in[plane + (long long)r * cols + c];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 32; k += 8) {
    const int c = c0 + ty + k, r = r0 + tx;
    if (r < rows && c < cols) out[plane + (long long)c * rows + r] = tile[tx][ty + k];
  }
}

unsigned grid_for(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16); }

}  // namespace

struct FftAxis {
  cufftHandle fwd = 0, inv = 0;
  int n = 0, nh = 0, made = 0;
  long long lines = 0, inner = 1;
  float *k = nullptr;  // [nh] wavenumbers (device)
};

struct FftPlans {
  FftAxis ax[3];
  // the same derivatives as circulant line matrices on the tensor cores
  // (kernels_r2r_tc.cu), per axis and isign, where that kernel applies
  unsigned char *Bg[3][2] = {};
  int tc[3] = {};
  int *err = nullptr;
  int nx = 0, ny = 0, nz = 0;
  float2 *spec = nullptr;  // half spectrum of the largest axis set
  float *tr = nullptr;     // x lines made contiguous ([ny][nz][nx])
};

// k table of FdEngine_r2c::assignW in the reference's float arithmetic
static std::vector<float> r2c_wavenumbers(int n, float d) {
  const float scale = 1.0f / float(n);
  const float dk = (float)(2.0f * M_PI / (double)(d * (float)n) * (double)scale);
  std::vector<float> k(n / 2 + 1);
  for (int j = 0; j <= n / 2; j++) k[j] = (float)(-j) * dk;
  return k;
}

void fft_plans_destroy(FftPlans *p) {
  if (!p) return;
  for (auto &a : p->Bg)
    for (unsigned char *b : a)
      if (b) cudaFree(b);
  for (FftAxis &a : p->ax) {
    if (a.made & 1) cufftDestroy(a.fwd);
    if (a.made & 2) cufftDestroy(a.inv);
    if (a.k) cudaFree(a.k);
  }
  if (p->spec) cudaFree(p->spec);
  if (p->tr) cudaFree(p->tr);
  delete p;
}

int fft_plans_create(FftPlans **out, int nx, int ny, int nz, float dx, float dy, float dz, cudaStream_t st,
                     bool tensor_cores, int *err) {
  *out = nullptr;
  FftPlans *p = new FftPlans();
  p->nx = nx, p->ny = ny, p->nz = nz, p->err = err;
  const long long nxz = (long long)nx * nz;
  const int nn[3] = {nx, ny, nz};
  const float dd[3] = {dx, dy, dz};
  long long spec = 0;
  for (int a = 0; a < 3; a++) {
    if (nn[a] < 2) continue;  // no y derivative on a 2-D grid
    FftAxis &f = p->ax[a];
    int n = nn[a];
    f.n = n, f.nh = n / 2 + 1;
    int inembed[1] = {n}, onembed[1] = {f.nh};
    int istride, idist, ostride, odist;
    if (a == 1) {  // y: stride nx nz, batch over the contiguous columns
      f.lines = nxz, f.inner = nxz;
      istride = (int)nxz, idist = 1, ostride = (int)nxz, odist = 1;
    } else {  // z, and x after the transpose: contiguous lines
      f.lines = a == 2 ? (long long)nx * ny : (long long)ny * nz;
      f.inner = 1;
      istride = 1, idist = n, ostride = 1, odist = f.nh;
    }
    if (f.lines > 0x7fffffffLL || nxz > 0x7fffffffLL) {
      fft_plans_destroy(p);
      return RTM_ERR_ARG;
    }
    if (cufftPlanMany(&f.fwd, 1, &n, inembed, istride, idist, onembed, ostride, odist, CUFFT_R2C, (int)f.lines) !=
        CUFFT_SUCCESS) {
      fft_plans_destroy(p);
      return RTM_ERR_CUDA;
    }
    f.made |= 1;
    if (cufftPlanMany(&f.inv, 1, &n, onembed, ostride, odist, inembed, istride, idist, CUFFT_C2R, (int)f.lines) !=
        CUFFT_SUCCESS) {
      fft_plans_destroy(p);
      return RTM_ERR_CUDA;
    }
    f.made |= 2;
    if (cufftSetStream(f.fwd, st) != CUFFT_SUCCESS || cufftSetStream(f.inv, st) != CUFFT_SUCCESS) {
      fft_plans_destroy(p);
      return RTM_ERR_CUDA;
    }
    const std::vector<float> k = r2c_wavenumbers(n, dd[a]);
    if (cudaMalloc(&f.k, k.size() * 4) != cudaSuccess ||
        cudaMemcpyAsync(f.k, k.data(), k.size() * 4, cudaMemcpyHostToDevice, st) != cudaSuccess) {
      cudaGetLastError();
      fft_plans_destroy(p);
      return RTM_ERR_NOMEM;
    }
    spec = std::max(spec, (long long)f.nh * f.lines);
  }
  if (cudaMalloc(&p->spec, (size_t)spec * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&p->tr, (size_t)ny * nxz * 4) != cudaSuccess) {
    cudaGetLastError();
    fft_plans_destroy(p);
    return RTM_ERR_NOMEM;
  }
  if (tensor_cores && r2r_tc_init() == 0) {
    std::vector<float> D;
    float *dD = nullptr;
    for (int a = 0; a < 3; a++) {
      if (nn[a] < 2 || !r2r_tc_supported(a, nx, ny, nz)) continue;
      for (int s = 0; s < 2; s++) {
        r2c_line_matrix(nn[a], dd[a], s == 0 ? 1 : -1, D);
        if (cudaMalloc(&p->Bg[a][s], r2r_tc_bytes(nn[a])) != cudaSuccess ||
            cudaMalloc(&dD, D.size() * 4) != cudaSuccess ||
            cudaMemcpyAsync(dD, D.data(), D.size() * 4, cudaMemcpyHostToDevice, st) != cudaSuccess) {
          cudaGetLastError();
          if (dD) cudaFree(dD);
          fft_plans_destroy(p);
          return RTM_ERR_NOMEM;
        }
        launch_tf32_arrange(dD, p->Bg[a][s], nn[a], st);
        const cudaError_t e = cudaStreamSynchronize(st);
        cudaFree(dD), dD = nullptr;
        if (e != cudaSuccess) {
          fft_plans_destroy(p);
          return RTM_ERR_CUDA;
        }
      }
      p->tc[a] = 1;
    }
  }
  cudaGetLastError();
  *out = p;
  return RTM_OK;
}

int launch_fft_deriv(FftPlans *p, int axis, int isign, const float *in, float *out, cudaStream_t st) {
  const FftAxis &f = p->ax[axis];
  if ((f.made & 3) != 3) return RTM_ERR_ARG;
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  if (p->tc[axis]) {  // the circulant line matrix on the tensor cores (split TF32)
    launch_r2r_tc(axis, in, out, p->Bg[axis][isign == 1 ? 0 : 1], nx, ny, nz, p->err, st);
    return cudaGetLastError() == cudaSuccess ? RTM_OK : RTM_ERR_CUDA;
  }
  const float *src = in;
  float *dst = out;
  if (axis == 0) {  // [ny][nx][nz] -> [ny][nz][nx]
    transpose_k<<<dim3((nz + 31) / 32, (nx + 31) / 32, ny), 256, 0, st>>>(in, p->tr, nx, nz);
    src = dst = p->tr;
  }
  if (cufftExecR2C(f.fwd, const_cast<float *>(src), (cufftComplex *)p->spec) != CUFFT_SUCCESS) return RTM_ERR_CUDA;
  const long long total = (long long)f.nh * f.lines;
  fft_ik_k<<<grid_for(total), 256, 0, st>>>(p->spec, f.k, total, f.nh, f.inner, f.n, (float)isign);
  if (cufftExecC2R(f.inv, (cufftComplex *)p->spec, dst) != CUFFT_SUCCESS) return RTM_ERR_CUDA;
  if (axis == 0)  // [ny][nz][nx] -> [ny][nx][nz]
    transpose_k<<<dim3((nx + 31) / 32, (nz + 31) / 32, ny), 256, 0, st>>>(p->tr, out, nz, nx);
  return RTM_OK;
}

struct R2rPlans {
  cublasHandle_t blas = nullptr;
  void *ws = nullptr;
  float *D[3][2] = {};  // [axis][pass: 0 isign +1, 1 isign -1], row-major n x n
  // line operators on the tensor cores: D split into its TF32 parts and laid
  // out as the kernel's B stages (kernels_r2r_tc.cu), per axis and pass
  unsigned char *Bg[3][2] = {};
  int tc[3] = {};
  int *err = nullptr;
  cudaStream_t st = nullptr;
  int nx = 0, ny = 0, nz = 0;
};

constexpr size_t kBlasWorkspace = 32u << 20;

void r2r_plans_destroy(R2rPlans *p) {
  if (!p) return;
  if (p->blas) cublasDestroy(p->blas);
  for (auto &a : p->D)
    for (float *m : a)
      if (m) cudaFree(m);
  for (auto &a : p->Bg)
    for (unsigned char *b : a)
      if (b) cudaFree(b);
  if (p->ws) cudaFree(p->ws);
  delete p;
}

int r2r_plans_create(R2rPlans **out, int nx, int ny, int nz, float dx, float dy, float dz, cudaStream_t st,
                     bool tensor_cores, int *err) {
  *out = nullptr;
  R2rPlans *p = new R2rPlans();
  p->nx = nx, p->ny = ny, p->nz = nz;
  p->st = st, p->err = err;
  if (cublasCreate(&p->blas) != CUBLAS_STATUS_SUCCESS) {
    p->blas = nullptr;
    r2r_plans_destroy(p);
    return RTM_ERR_CUDA;
  }
  if (cudaMalloc(&p->ws, kBlasWorkspace) != cudaSuccess) {
    cudaGetLastError();
    r2r_plans_destroy(p);
    return RTM_ERR_NOMEM;
  }
  if (cublasSetStream(p->blas, st) != CUBLAS_STATUS_SUCCESS ||
      cublasSetWorkspace(p->blas, p->ws, kBlasWorkspace) != CUBLAS_STATUS_SUCCESS ||
      cublasSetMathMode(p->blas, CUBLAS_PEDANTIC_MATH) != CUBLAS_STATUS_SUCCESS) {
    r2r_plans_destroy(p);
    return RTM_ERR_CUDA;
  }
  const int nn[3] = {nx, ny, nz};
  const float dd[3] = {dx, dy, dz};
  std::vector<float> D;
  for (int a = 0; a < 3; a++) {
    if (nn[a] < 2) continue;
    for (int s = 0; s < 2; s++) {
      r2r_line_matrix(nn[a], dd[a], s == 0 ? 1 : -1, D);
      if (cudaMalloc(&p->D[a][s], D.size() * 4) != cudaSuccess ||
          cudaMemcpyAsync(p->D[a][s], D.data(), D.size() * 4, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        cudaGetLastError();
        r2r_plans_destroy(p);
        return RTM_ERR_NOMEM;
      }
    }
  }
  if (tensor_cores && r2r_tc_init() == 0) {
    for (int a = 0; a < 3; a++) {
      if (!p->D[a][0] || !r2r_tc_supported(a, nx, ny, nz)) continue;
      for (int s = 0; s < 2; s++) {
        if (cudaMalloc(&p->Bg[a][s], r2r_tc_bytes(nn[a])) != cudaSuccess) {
          cudaGetLastError();
          r2r_plans_destroy(p);
          return RTM_ERR_NOMEM;
        }
        launch_tf32_arrange(p->D[a][s], p->Bg[a][s], nn[a], st);
      }
      p->tc[a] = 1;
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      cudaGetLastError();
      r2r_plans_destroy(p);
      return RTM_ERR_CUDA;
    }
  }
  cudaGetLastError();
  *out = p;
  return RTM_OK;
}

int launch_r2r_deriv(R2rPlans *p, int axis, int isign, const float *in, float *out) {
  const float *D = p->D[axis][isign == 1 ? 0 : 1];
  if (!D) return RTM_ERR_ARG;
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  const long long nxz = (long long)nx * nz, lines = (long long)nx * ny;
  if (nxz > 0x7fffffffLL || lines > 0x7fffffffLL) return RTM_ERR_ARG;
  const float one = 1.f, zero = 0.f;
  cublasStatus_t r;
  if (p->tc[axis]) {  // the same products on the tensor cores (split TF32)
    launch_r2r_tc(axis, in, out, p->Bg[axis][isign == 1 ? 0 : 1], nx, ny, nz, p->err, p->st);
    return cudaGetLastError() == cudaSuccess ? RTM_OK : RTM_ERR_CUDA;
  }
  if (axis == 2)  // out[l][t] = sum_u D[t][u] in[l][u]
    r = cublasSgemm(p->blas, CUBLAS_OP_T, CUBLAS_OP_N, nz, (int)lines, nz, &one, D, nz, in, nz, &zero, out, nz);
  else if (axis == 1)  // out[t][c] = sum_u D[t][u] in[u][c], c over nx nz
    r = cublasSgemm(p->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)nxz, ny, ny, &one, in, (int)nxz, D, ny, &zero, out,
                    (int)nxz);
  else  // per y plane: out[t][z] = sum_u D[t][u] in[u][z]
    r = cublasSgemmStridedBatched(p->blas, CUBLAS_OP_N, CUBLAS_OP_N, nz, nx, nx, &one, in, nz, nxz, D, nx, 0, &zero,
                                  out, nz, nxz, ny);
  return r == CUBLAS_STATUS_SUCCESS ? RTM_OK : RTM_ERR_CUDA;
}

}  // namespace rtm

namespace rtm {

int launch_fft_filter(FftPlans *p, int axis, int kind, float high, const float *in, float *out, cudaStream_t st) {
  const FftAxis &f = p->ax[axis];
  if ((f.made & 3) != 3 || (kind != 0 && kind != 1) || (kind == 1 && !(high >= 0.f && high < 1.f)))
    return RTM_ERR_ARG;
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  const float *src = in;
  float *dst = out;
  if (axis == 0) {  // [ny][nx][nz] -> [ny][nz][nx]
    transpose_k<<<dim3((nz + 31) / 32, (nx + 31) / 32, ny), 256, 0, st>>>(in, p->tr, nx, nz);
    src = dst = p->tr;
  }
  if (cufftExecR2C(f.fwd, const_cast<float *>(src), (cufftComplex *)p->spec) != CUFFT_SUCCESS) return RTM_ERR_CUDA;
  const long long total = (long long)f.nh * f.lines;
  fft_filter_k<<<grid_for(total), 256, 0, st>>>(p->spec, total, f.nh, f.inner, f.n, kind, high);
  if (cufftExecC2R(f.inv, (cufftComplex *)p->spec, dst) != CUFFT_SUCCESS) return RTM_ERR_CUDA;
  if (axis == 0)
    transpose_k<<<dim3((nx + 31) / 32, (nz + 31) / 32, ny), 256, 0, st>>>(p->tr, out, nz, nx);
  return RTM_OK;
}

}  // namespace rtm
