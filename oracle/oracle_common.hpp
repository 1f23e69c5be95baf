// oracle_common.hpp - restated setup helpers of the oracle (TEST INFRASTRUCTURE
// ONLY; the product has its own implementation in konglong_b200/csrc).
//   taylor_weights : central-difference weights (the absent libCommon::Taylor)
//   spread_coeffs  : Util::CompactOrmsbySpreadCoeff + Receiver taper_kernel
//   c16_*          : WaveFieldCompress COMPRESS_16 codec
#pragma once
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {

// Weights of the order-2*ne central differences, solved from the Taylor
// moment conditions in long double: first derivative
//   f'(0) ~ sum_j c1[j] (f_j - f_-j),   c1[0] = 0
// second derivative
//   f''(0) ~ c2[0] f_0 + sum_j c2[j] (f_j + f_-j).
inline void taylor_weights(int ne, double *c1, double *c2) {
  const int N = ne;
  std::vector<long double> A(N * N), b(N);
  auto solve = [&](std::vector<long double> &M, std::vector<long double> &r) {
    for (int c = 0; c < N; c++) {
      int piv = c;
      for (int k = c + 1; k < N; k++)
        if (std::fabs((double)M[k * N + c]) > std::fabs((double)M[piv * N + c])) piv = k;
      for (int k = 0; k < N; k++) std::swap(M[c * N + k], M[piv * N + k]);
      std::swap(r[c], r[piv]);
      for (int k = c + 1; k < N; k++) {
        long double f = M[k * N + c] / M[c * N + c];
        for (int j = c; j < N; j++) M[k * N + j] -= f * M[c * N + j];
        r[k] -= f * r[c];
      }
    }
    for (int c = N - 1; c >= 0; c--) {
      long double s = r[c];
      for (int j = c + 1; j < N; j++) s -= M[c * N + j] * r[j];
      r[c] = s / M[c * N + c];
    }
  };
  // 1st derivative: sum_j c_j * 2 j^(2k+1) = [k == 0]
  for (int k = 0; k < N; k++) {
    for (int j = 1; j <= N; j++) A[k * N + j - 1] = 2.0L * std::pow((long double)j, 2 * k + 1);
    b[k] = k == 0 ? 1.0L : 0.0L;
  }
  solve(A, b);
  c1[0] = 0;
  for (int j = 1; j <= N; j++) c1[j] = (double)b[j - 1];
  // 2nd derivative: sum_j c_j * 2 j^(2k) = 2 [k == 1], k = 1..N
  for (int k = 1; k <= N; k++) {
    for (int j = 1; j <= N; j++) A[(k - 1) * N + j - 1] = 2.0L * std::pow((long double)j, 2 * k);
    b[k - 1] = k == 1 ? 2.0L : 0.0L;
  }
  solve(A, b);
  long double s = 0;
  for (int j = 1; j <= N; j++) c2[j] = (double)b[j - 1], s += b[j - 1];
  c2[0] = (double)(-2.0L * s);
}

// libCommon::sincf_unnorm / dipole_unnorm / blackman are absent from the
// reference tree; restated from their definitions (parity unpinned).
inline float sinc_unnorm(float x) { return x == 0.0f ? 1.0f : sinf(x) / x; }
inline float dipole_unnorm(float x) { return x == 0.0f ? 0.0f : (x * cosf(x) - sinf(x)) / (x * x); }
inline float blackman(float t) { return 0.42f - 0.5f * cosf(t) + 0.08f * cosf(2.0f * t); }

// Util::CompactOrmsbySpreadCoeff, nlimit form (bgprtm/Util.cpp:317-397), then
// taper_kernel with an ntaper-point cosine ramp (bgprtm/Receiver.cpp:291-303,
// 316-318).  coeff[*nlimit] is written from the returned first index.
inline int spread_coeffs(int n, float x, float k1, float k2, int *nlimit, int dipole, int ntaper, float *coeff) {
  const float kPi = 3.14159265358979323846f;
  if (n == 1 || *nlimit < 2) {
    coeff[0] = 1.0f;
    *nlimit = 1;
    return (int)nearbyintf(x);
  }
  bool use_sinc = (k1 == k2) || dipole;
  float a1 = k1 * kPi, a2 = k2 * kPi;
  if (use_sinc) a1 *= 2;
  int ix = (int)floorf(x);
  int m = std::min(ix, n - 1 - ix);
  m = std::min(m, *nlimit / 2);
  *nlimit = 2 * m;
  int ix0 = ix - m + 1;
  int ntap = m / 2;
  int i0 = ix - m + 1, i1 = ix + m;
  float halfwin = std::max(i1 - x, x - i0);
  for (int i = i0; i < i1 + 1; i++) {
    float shift = i - x;
    float b1 = shift * a1;
    float s1 = dipole ? dipole_unnorm(b1) : sinc_unnorm(b1);
    float val;
    if (!use_sinc) {
      float s2 = sinc_unnorm(shift * a2);
      val = (a2 * a2 * s2 * s2 - a1 * a1 * s1 * s1) / kPi / (a2 - a1);
      int ie = std::min(i - i0, i1 - i);
      if (ie < ntap && m > 1) val *= 0.5f * (1 - cosf(kPi * ie / ntap));
    } else {
      val = s1 * 2 * k1;
      if (m > 1) val *= blackman(kPi * (halfwin - x + i) / halfwin);
    }
    coeff[i - ix0] = val;
  }
  if (ntaper > 0 && n > ntaper * 2) {
    std::vector<float> w(ntaper);
    for (int i = 0; i < ntaper; i++) w[i] = 0.5f * (1.0f - cosf((float)(M_PI * i / ntaper)));
    int l = *nlimit, off = ix0;
    if (off < ntaper)
      for (int i = std::max(0, off); i < std::min(ntaper, l + off); i++) coeff[i - off] *= w[i];
    if (off + l > n - ntaper)
      for (int i = std::max(0, n - off - l); i < std::min(ntaper, n - off); i++) coeff[n - (off + i + 1)] *= w[i];
  }
  return ix0;
}

// WaveFieldCompress::init (bgprtm/WaveFieldCompress.cpp:52-99)
inline void c16_tables(std::vector<float> &table, std::vector<float> &w20, std::vector<float> &w10) {
  table.assign(65536, 0.0f);
  table[1] = 1.0f;
  uint32_t nanbits = 0x7fffffffu;
  std::memcpy(&table[32768], &nanbits, 4);
  float f = 1.f / ((float)(1 << 30));
  for (int i = 2; i < 1024; i++) table[i] = f * i;
  f = 1.f / ((float)(1 << 14));
  for (int i = 1024; i < 16384; i++) table[i] = f * i;
  float octave[1024];
  f = 1.f / 1024.f;
  for (int i = 0; i < 1024; i++) octave[i] = 1.f + i * f;
  for (int j = 0; j < 16; j++) {
    f = 1.f / ((float)(1 << (20 - j)));
    for (int i = 0; i < 1024; i++) table[16384 + j * 1024 + i] = f * octave[i];
  }
  for (int i = 1; i < 32768; i++) table[i + 32768] = -table[i];
  w20.resize(20), w10.resize(10);
  for (int i = 0; i < 20; i++) w20[i] = 0.5f * (1.0f - cosf((float)M_PI * float(i) / float(20)));
  for (int i = 0; i < 10; i++) w10[i] = 0.5f * (1.0f - cosf((float)M_PI * float(i) / float(10)));
}

// WaveFieldCompress::shift (bgprtm/WaveFieldCompress.cpp:107-133)
inline uint16_t c16_code(float v) {
  int32_t idat;
  std::memcpy(&idat, &v, 4);
  uint16_t sgn = (uint16_t)(((uint32_t)idat & 0x80000000u) >> 16);
  int e = ((idat & 0x7f800000) >> 23) - 127;
  int frc;
  if (e > 0) return 0x8000;
  if (e == 0) return sgn | 0x1;
  if (e > -5) {
    frc = (idat & 0x7fffff) | 0x800000;
    return sgn | (uint16_t)(frc >> (9 - e));
  }
  if (e > -21) {
    e += 20;
    frc = idat & 0x7fffff;
    return sgn | 0x4000 | (uint16_t)(e << 10) | (uint16_t)(frc >> 13);
  }
  if (e > -30) {
    frc = (idat & 0x7fffff) | 0x800000;
    return sgn | (uint16_t)(frc >> (-7 - e));
  }
  return 0;
}

// compress16 (bgprtm/WaveFieldCompress.cpp:135-168): per y slab a float vmax
// header (2 uint16) then one code per cell.
inline void c16_compress(const float *in, uint16_t *out, int nx, int ny, int nz) {
  const float eps = 1e-25f;
  size_t nxz = (size_t)nx * nz;
  for (int iy = 0; iy < ny; iy++) {
    const float *p = in + iy * nxz;
    uint16_t *o = out + iy * (nxz + 2);
    float vmax = fabsf(p[0]);
    for (size_t i = 1; i < nxz; i++) vmax = std::max(vmax, fabsf(p[i]));
    if (vmax > eps) {
      float scale = 1.0f / vmax;
      for (size_t i = 0; i < nxz; i++) o[i + 2] = c16_code(p[i] * scale);
      std::memcpy(o, &vmax, 4);
    } else {
      std::memset(o, 0, (nxz + 2) * 2);
    }
  }
}

// uncompress16 (bgprtm/WaveFieldCompress.cpp:171-207); edge = 0 skips the tapers
inline void c16_uncompress(const uint16_t *in, float *out, int nx, int ny, int nz, const float *table,
                           const float *w20, const float *w10, int edge) {
  size_t nxz = (size_t)nx * nz;
  for (int iy = 0; iy < ny; iy++) {
    const uint16_t *p = in + iy * (nxz + 2);
    float *o = out + iy * nxz;
    float scale;
    std::memcpy(&scale, p, 4);
    if (!(scale > 1e-25f)) {
      std::memset(o, 0, nxz * 4);
      continue;
    }
    for (int ix = 0; ix < nx; ix++)
      for (int iz = 0; iz < nz; iz++) {
        size_t id = (size_t)ix * nz + iz;
        float v = scale * table[p[id + 2]];
        if (edge) {
          if (ny > 40) {
            if (iy < 20) v *= w20[iy];
            if (iy > ny - 21) v *= w20[ny - iy - 1];
          }
          if (nx > 40) {
            if (ix < 20) v *= w20[ix];
            if (ix > nx - 21) v *= w20[nx - ix - 1];
          }
          if (nz > 20) {
            if (iz < 10) v *= w10[iz];
            if (iz > nz - 11) v *= w10[nz - iz - 1];
          }
        }
        o[id] = v;
      }
  }
}

}  // namespace orc
