// kernels_ic.cu - INVERSION imaging condition (ImagingCorrelator::inversion1,
// bgprtm/ImagingCorrelator.cpp:374-424; derive / lapx / lapy / lapz, :195-278).
//
// image += s r - dz(s) dz(r) - dx(s) dx(r) - dy(s) dy(r), where d_a is the
// normalised k-domain derivative F^-1[ i (k_a / |k|) F[.] ] (zero at k = 0) of the
// tapered source and receiver wavefields, with the reference's wavenumber
// convention (k[i] = -i dk for i <= n/2, (n - i) dk above) and its 1/sqrt(N)
// scaling on the way into and out of the unnormalised transforms.  The
// transforms are cuFFT 3-D (2-D when ny == 1) real <-> complex plans; the terms
// are added to the Kahan-compensated image in the reference's order.
#include <cufft.h>

#include "kernel_api.h"
#include "rtm_device.cuh"

namespace rtm {
namespace {

// tapered source and receiver values of every cell (fused_io's tapers), the s r
// term into the image and the illumination
__global__ void ic_fields_k(FusedIo io, const float *__restrict__ u, float *__restrict__ S, float *__restrict__ Rv,
                            int nx, int ny, int nz) {
  const Grid3 g{nx, ny, nz, (long long)nx * nz};
  const long long n = g.nxz * ny;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int iy = (int)(i / g.nxz), ix = (int)((i % g.nxz) / nz), iz = (int)(i % nz);
    const long long inslab = i % g.nxz;
    float s = snap_read(io.src, g, i, iy, inslab);
    s = s * io.ey[iy];
    s = s * io.ex[ix];
    s = s * io.ez[iz];
    if (io.use_t) s = s * io.tscale;
    else s = s * io.taper_z[iz];
    if (io.illum) io.illum[i] = __fmaf_rn(s, s, io.illum[i]);
    float r = u[i] * io.ey[iy];
    r = r * io.ex[ix];
    r = r * io.ez[iz];
    S[i] = s, Rv[i] = r;
    const float prod = s * r;
    const float img = io.image[i];
    const float y = prod - io.comp[i];
    const float t = img + y;
    io.comp[i] = (t - img) - y;
    io.image[i] = t;
  }
}

__device__ __forceinline__ float wavenumber(int i, int n, float dk) { return i <= n / 2 ? -i * dk : (n - i) * dk; }

// out = i (k_axis / |k|) in * scale (axis 0 z, 1 x, 2 y), zero where |k| <= 1e-25
__global__ void kderiv_k(const float2 *__restrict__ in, float2 *__restrict__ out, int axis, int nx, int ny, int nz,
                         float dkx, float dky, float dkz, float scale) {
  const int nzc = nz / 2 + 1;
  const long long n = (long long)ny * nx * nzc;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(i % nzc), ix = (int)((i / nzc) % nx), iy = (int)(i / ((long long)nzc * nx));
    const float kx = wavenumber(ix, nx, dkx), ky = ny > 1 ? wavenumber(iy, ny, dky) : 0.f, kz = wavenumber(iz, nz, dkz);
    const float kk = sqrtf(kx * kx + kz * kz + ky * ky);
    float2 o = make_float2(0.f, 0.f);
    if (kk > 1.0e-25f) {
      const float ka = (axis == 0 ? kz : axis == 1 ? kx : ky) / kk;
      const float2 v = in[i];
      o = make_float2(-ka * v.y * scale, ka * v.x * scale);
    }
    out[i] = o;
  }
}

// image -= (a scale) (b scale), Kahan-compensated
__global__ void ic_sub_k(const float *__restrict__ a, const float *__restrict__ b, float *image, float *comp,
                         long long n, float scale) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float prod = -((a[i] * scale) * (b[i] * scale));
    const float img = image[i];
    const float y = prod - comp[i];
    const float t = img + y;
    comp[i] = (t - img) - y;
    image[i] = t;
  }
}

unsigned blocks_for(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16); }

}  // namespace

struct IcPlans {
  cufftHandle r2c = 0, c2r = 0;
  int ok = 0;
};

void *ic_plans_create(int nx, int ny, int nz) {
  IcPlans *p = new IcPlans();
  cufftResult a, b;
  if (ny > 1) {
    a = cufftPlan3d(&p->r2c, ny, nx, nz, CUFFT_R2C);
    b = cufftPlan3d(&p->c2r, ny, nx, nz, CUFFT_C2R);
  } else {
    a = cufftPlan2d(&p->r2c, nx, nz, CUFFT_R2C);
    b = cufftPlan2d(&p->c2r, nx, nz, CUFFT_C2R);
  }
  p->ok = a == CUFFT_SUCCESS && b == CUFFT_SUCCESS;
  if (!p->ok) {
    if (a == CUFFT_SUCCESS) cufftDestroy(p->r2c);
    if (b == CUFFT_SUCCESS) cufftDestroy(p->c2r);
    delete p;
    return nullptr;
  }
  return p;
}

void ic_plans_destroy(void *plans) {
  IcPlans *p = static_cast<IcPlans *>(plans);
  if (!p) return;
  cufftDestroy(p->r2c), cufftDestroy(p->c2r);
  delete p;
}

long long ic_spectrum_floats(int nx, int ny, int nz) { return 2LL * ny * nx * (nz / 2 + 1); }

int launch_ic_inversion(void *plans, const FusedIo &io, const float *u, float *S, float *Rv, float *Ds, float *Dr,
                        float *Sh, float *Rh, float *Th, int nx, int ny, int nz, float dx, float dy, float dz,
                        cudaStream_t st) {
  IcPlans *p = static_cast<IcPlans *>(plans);
  const long long n = (long long)nx * ny * nz, nc = (long long)ny * nx * (nz / 2 + 1);
  const float scalef = sqrtf((1.0f / float(nx)) * (1.0f / float(ny)) * (1.0f / float(nz)));
  const float dkx = 2.0f * (float)M_PI / (dx * nx), dky = 2.0f * (float)M_PI / (dy * ny),
              dkz = 2.0f * (float)M_PI / (dz * nz);
  if (cufftSetStream(p->r2c, st) != CUFFT_SUCCESS || cufftSetStream(p->c2r, st) != CUFFT_SUCCESS) return -1;
  ic_fields_k<<<blocks_for(n), 256, 0, st>>>(io, u, S, Rv, nx, ny, nz);
  if (cufftExecR2C(p->r2c, S, (cufftComplex *)Sh) != CUFFT_SUCCESS) return -1;
  if (cufftExecR2C(p->r2c, Rv, (cufftComplex *)Rh) != CUFFT_SUCCESS) return -1;
  // z, x, then y (ny > 1), as inversion1
  for (int axis = 0; axis < (ny > 1 ? 3 : 2); axis++) {
    kderiv_k<<<blocks_for(nc), 256, 0, st>>>((const float2 *)Sh, (float2 *)Th, axis, nx, ny, nz, dkx, dky, dkz, scalef);
    if (cufftExecC2R(p->c2r, (cufftComplex *)Th, Ds) != CUFFT_SUCCESS) return -1;
    kderiv_k<<<blocks_for(nc), 256, 0, st>>>((const float2 *)Rh, (float2 *)Th, axis, nx, ny, nz, dkx, dky, dkz, scalef);
    if (cufftExecC2R(p->c2r, (cufftComplex *)Th, Dr) != CUFFT_SUCCESS) return -1;
    ic_sub_k<<<blocks_for(n), 256, 0, st>>>(Ds, Dr, io.image, io.comp, n, scalef);
  }
  return 0;
}

}  // namespace rtm
