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
#include "rtm_b200.h"
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

// ---------------------------------------------------------------------------
// Double-grid IMAGE1 (ImagingCondition::stackImageInterp with ic_double_* = 2,
// bgprtm/ImagingCondition.cpp:104-141; ImagingCorrelator::imaging1 /
// interleave2d / interleave3d, bgprtm/ImagingCorrelator.cpp:363-372, 440-507;
// ImagingCondition::interpIllum, bgprtm/ImagingCondition.cpp:759-808).
// Per imaging step the tapered source and receiver fields are high-cut along
// each doubled axis, half-shifted into the 2, 4 or 8 copies of the doubled
// grid's sub-lattices (line FFTs, kernels_fft.cu), and copy i of each field is
// correlated into image cube i.  The cubes are interleaved onto the doubled
// grid when read.
namespace rtm {
namespace {

// tapered source and receiver fields (ic_fields_k's tapers), no image term
__global__ void dbl_fields_k(FusedIo io, const float *__restrict__ u, float *__restrict__ S, float *__restrict__ Rv,
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
    float r = u[i] * io.ey[iy];
    r = r * io.ex[ix];
    r = r * io.ez[iz];
    S[i] = s, Rv[i] = r;
  }
}

// illum += s^2 (calIllum on the filtered source field)
__global__ void dbl_illum_acc_k(const float *__restrict__ S, float *illum, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    illum[i] = __fmaf_rn(S[i], S[i], illum[i]);
}

// image += s r, Kahan-compensated (crossone with isign +1)
__global__ void dbl_cross_k(const float *__restrict__ S, const float *__restrict__ Rv, float *image, float *comp,
                            long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float prod = S[i] * Rv[i];
    const float img = image[i];
    const float y = prod - comp[i];
    const float t = img + y;
    comp[i] = (t - img) - y;
    image[i] = t;
  }
}

// cube `slot[c]` of every doubled-grid point class c = (y odd, x odd, z odd)
// (the sub-lattice each half-shifted copy sits on) into the doubled grid
__global__ void dbl_interleave_k(const float *__restrict__ cubes, float *out, DblMap m, int nx, int ny, int nz) {
  const long long nx2 = (long long)nx * m.dx, nz2 = (long long)nz * m.dz, ny2 = (long long)ny * m.dy;
  const long long n2 = nx2 * ny2 * nz2, n = (long long)nx * ny * nz;
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < n2; o += (long long)gridDim.x * blockDim.x) {
    const long long z2 = o % nz2, x2 = (o / nz2) % nx2, y2 = o / (nz2 * nx2);
    const int zo = (int)(z2 % m.dz), xo = (int)(x2 % m.dx), yo = (int)(y2 % m.dy);
    const long long idd = ((y2 / m.dy) * nx + x2 / m.dx) * nz + z2 / m.dz;
    out[o] = cubes[(long long)m.slot[(yo << 2) | (xo << 1) | zo] * n + idd];
  }
}

// illumination on the doubled grid, interpIllum's arithmetic per base cell:
// the eight targets (y1x1z1, y2x1z1, y1x2z1, y1x1z2, y2x1z2, y1x2z2, y2x2z1,
// y2x2z2) written in that order with neighbours clamped at the far edges; on
// an axis that is not doubled its "odd" index is the even one, so later
// targets overwrite earlier ones at the same point as in the reference
__global__ void dbl_illum_k(const float *__restrict__ in, float *out, DblMap m, int nx, int ny, int nz) {
  const long long nxy = (long long)nx * ny;
  const long long nx2 = (long long)nx * m.dx, nz2 = (long long)nz * m.dz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < nxy * nz;
       c += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(c % nz);
    const long long ixy = c / nz;
    const int ix = (int)(ixy % nx), iy = (int)(ixy / nx);
    const long long iy1 = (long long)iy * m.dy, iy2 = iy1 + (m.dy - 1), ix1 = (long long)ix * m.dx,
                    ix2 = ix1 + (m.dx - 1), iz1 = (long long)iz * m.dz, iz2 = iz1 + (m.dz - 1);
    const int iyp1 = min(iy + 1, ny - 1), ixp1 = min(ix + 1, nx - 1), izp1 = min(iz + 1, nz - 1);
    auto at = [&](int y, int x, int z) { return in[((long long)y * nx + x) * nz + z]; };
    auto o = [&](long long y, long long x, long long z) -> float & { return out[(y * nx2 + x) * nz2 + z]; };
    const float a = at(iy, ix, iz);
    o(iy1, ix1, iz1) = a;
    o(iy2, ix1, iz1) = 0.5f * (a + at(iyp1, ix, iz));
    o(iy1, ix2, iz1) = 0.5f * (a + at(iy, ixp1, iz));
    o(iy1, ix1, iz2) = 0.5f * (a + at(iy, ix, izp1));
    o(iy2, ix1, iz2) = 0.25f * (a + at(iy, ix, izp1) + at(iyp1, ix, iz) + at(iyp1, ix, izp1));
    o(iy1, ix2, iz2) = 0.25f * (a + at(iy, ix, izp1) + at(iy, ixp1, iz) + at(iy, ixp1, izp1));
    o(iy2, ix2, iz1) = 0.25f * (a + at(iyp1, ix, iz) + at(iy, ixp1, iz) + at(iyp1, ixp1, iz));
    o(iy2, ix2, iz2) = 0.125f * (a + at(iyp1, ix, iz) + at(iy, ixp1, iz) + at(iy, ix, izp1) + at(iyp1, ix, izp1) +
                                 at(iyp1, ixp1, iz) + at(iy, ixp1, izp1) + at(iyp1, ixp1, izp1));
  }
}

}  // namespace

int launch_ic_double(FftPlans *fft, const DblMap &m, const FusedIo &io, const float *u, float *const *S,
                     float *const *Rv, float *image, float *comp, float *illum, int nx, int ny, int nz, float high_z,
                     float high_xy, cudaStream_t st) {
  const long long n = (long long)nx * ny * nz;
  dbl_fields_k<<<blocks_for(n), 256, 0, st>>>(io, u, S[0], Rv[0], nx, ny, nz);
  // ImagingCondition::applyFFTV: high cut along z, x, y (the doubled axes), in place
  const int axes[3] = {DZ, DX, DY};
  const int on[3] = {m.dz > 1, m.dx > 1, m.dy > 1};
  for (int k = 0; k < 3; k++) {
    if (!on[k]) continue;
    const float hi = k == 0 ? high_z : high_xy;
    for (float *f : {S[0], Rv[0]}) {
      const int rc = launch_fft_filter(fft, axes[k], 1, hi, f, f, st);
      if (rc != RTM_OK) return rc;
    }
  }
  if (illum) dbl_illum_acc_k<<<blocks_for(n), 256, 0, st>>>(S[0], illum, n);
  // ImagingCorrelator::interp: z, x, y from copy 0, then zx, zy, xy, zxy
  const int src_of[7] = {0, 0, 0, m.iv[0], m.iv[0], m.iv[1], m.iv[3]};
  const int ax_of[7] = {DZ, DX, DY, DX, DY, DY, DY};
  for (int k = 0; k < 7; k++) {
    const int dst = m.iv[k];
    if (!dst) continue;
    for (int f = 0; f < 2; f++) {
      float *const *V = f ? Rv : S;
      const int rc = launch_fft_filter(fft, ax_of[k], 0, 0.f, V[src_of[k]], V[dst], st);
      if (rc != RTM_OK) return rc;
    }
  }
  for (int i = 0; i < m.nloop; i++)
    dbl_cross_k<<<blocks_for(n), 256, 0, st>>>(S[i], Rv[i], image + (size_t)i * n, comp + (size_t)i * n, n);
  return RTM_OK;
}

void launch_dbl_interleave(const float *cubes, float *out, const DblMap &m, int nx, int ny, int nz, cudaStream_t st) {
  const long long n2 = (long long)nx * ny * nz * m.dx * m.dy * m.dz;
  dbl_interleave_k<<<blocks_for(n2), 256, 0, st>>>(cubes, out, m, nx, ny, nz);
}

void launch_dbl_illum(const float *in, float *out, const DblMap &m, int nx, int ny, int nz, cudaStream_t st) {
  dbl_illum_k<<<blocks_for((long long)nx * ny * nz), 256, 0, st>>>(in, out, m, nx, ny, nz);
}

}  // namespace rtm
