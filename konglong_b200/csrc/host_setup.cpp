// host_setup.cpp - host-side set-up of the B200 RTM engine (tables built once
// per handle, in FP64 where the arithmetic is set-up rather than stencil):
//   fd_weights       central-difference weights (the reference reads them from
//                    libCommon::Taylor, bgprtm/FdEngine_fd.cpp:30-54, 106-127)
//   cfd_plan         compact-FD band LU (bgprtm/Cfd_plan.cpp:54-290)
//   pml_profile      PML damping (bgprtm/PML.cpp:87-100) and the per-layer
//                    recursion constants of bgprtm/PML.cpp:126-134
//   spread_coeffs    Util::CompactOrmsbySpreadCoeff (bgprtm/Util.cpp:317-397)
//                    with Receiver's taper_kernel (bgprtm/Receiver.cpp:291-303)
//   r2r_line_matrix  FdEngine_r2r's derivative (bgprtm/FdEngine_r2r.cpp:4-102)
//   r2c_line_matrix  FdEngine_r2c's derivative as a circulant (bgprtm/FdEngine_r2c.cpp:200-240)
//                    as one matrix per axis and pass
#include <algorithm>
#include <cmath>
#include <vector>

#include "host_setup.h"

namespace rtm {

void fd_weights(int ne, double *c1, double *c2) {
  // Moment conditions of the symmetric stencils, solved by Gauss elimination
  // with partial pivoting in long double:
  //   sum_j c1_j * 2 j^(2k+1) = [k == 0],        k = 0..ne-1
  //   sum_j c2_j * 2 j^(2k)   = 2 [k == 1],      k = 1..ne,  c2_0 = -2 sum c2_j
  const int N = ne;
  std::vector<long double> M(N * N), r(N);
  auto gauss = [&]() {
    for (int c = 0; c < N; c++) {
      int p = c;
      for (int k = c + 1; k < N; k++)
        if (std::fabs((double)M[k * N + c]) > std::fabs((double)M[p * N + c])) p = k;
      for (int k = 0; k < N; k++) std::swap(M[c * N + k], M[p * N + k]);
      std::swap(r[c], r[p]);
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
  for (int k = 0; k < N; k++) {
    for (int j = 1; j <= N; j++) M[k * N + j - 1] = 2.0L * powl((long double)j, 2 * k + 1);
    r[k] = k == 0 ? 1.0L : 0.0L;
  }
  gauss();
  c1[0] = 0.0;
  for (int j = 1; j <= N; j++) c1[j] = (double)r[j - 1];
  for (int k = 1; k <= N; k++) {
    for (int j = 1; j <= N; j++) M[(k - 1) * N + j - 1] = 2.0L * powl((long double)j, 2 * k);
    r[k - 1] = k == 1 ? 2.0L : 0.0L;
  }
  gauss();
  long double s = 0;
  for (int j = 1; j <= N; j++) c2[j] = (double)r[j - 1], s += r[j - 1];
  c2[0] = (double)(-2.0L * s);
}

void cfd_plan(int n, double d, int isgn, std::vector<float> &bm, std::vector<float> &bl, std::vector<float> &am,
              std::vector<float> *rdiag) {
  // Compact scheme B f' = A f, B 9-banded symmetric, A 11-point antisymmetric
  // (10th-order coefficient set of bgprtm/Cfd_plan.cpp:139-149).  Boundary
  // rows fold the stencil back onto the grid with sign -1 for B / +1 for A
  // when isgn = 1 and the opposite signs when isgn = 2.
  static const double ca5[5] = {0.861085998189822, 0.753782983214427, 0.257072513289755, 0.031326722562826,
                                0.000410456919800};
  static const double cb5[5] = {1.0, 0.753205475977546, 0.312203852849021, 0.063580085296350, 0.004597763362256};
  const double cb[9] = {cb5[4], cb5[3], cb5[2], cb5[1], cb5[0], cb5[1], cb5[2], cb5[3], cb5[4]};
  const double ca[11] = {-ca5[4], -ca5[3], -ca5[2], -ca5[1], -ca5[0], 0.0, ca5[0], ca5[1], ca5[2], ca5[3], ca5[4]};
  std::vector<double> B(9 * (size_t)n, 0.0), L(4 * (size_t)n, 0.0), A(60, 0.0);
  const double sb = isgn == 1 ? -1.0 : 1.0, sa = isgn == 1 ? 1.0 : -1.0;
  auto b = [&](int band, int row) -> double & { return B[(size_t)band * n + row]; };
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < 9; j++) {
      int col = i - 4 + j;  // column of band j in row i
      if (i >= 4 && i < n - 4) {
        b(j, i) = cb[j];
      } else if (col < 0) {
        b(4 - i - col, i) += sb * cb[j];  // reflect across the first grid point
      } else if (col > n - 1) {
        b((n + 3 - i) - (col - n + 1), i) += sb * cb[j];  // reflect across the last
      } else {
        b(j, i) += cb[j];
      }
    }
  }
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 11; j++) {
      int col = i - 5 + j;
      if (col < 0) A[(5 - i - col) * 5 + i] += sa * ca[j];
      else A[j * 5 + i] += ca[j];
    }
  for (int i = 0; i < 5; i++) A[55 + i] = ca5[i];
  for (int i = 0; i < 60; i++) A[i] = A[i] / d * 0.5;
  // banded LU without pivoting (4 sub-, 4 super-diagonals): first left-justify
  // the top rows, then eliminate; L multipliers kept per pivot row.
  const int m1 = 4, mm = 9;
  int l = m1;
  for (int i = 0; i < m1; i++) {
    for (int j = m1 - i; j < mm; j++) b(j - l, i) = b(j, i);
    l--;
    for (int j = mm - l - 1; j < mm; j++) b(j, i) = 0.0;
  }
  l = m1;
  for (int k = 0; k < n; k++) {
    if (l < n) l++;
    if (b(0, k) == 0.0) b(0, k) = 1e-20;
    for (int i = k + 1; i < l; i++) {
      double f = b(0, i) / b(0, k);
      L[(size_t)(i - k - 1) * n + k] = f;
      for (int j = 1; j < mm; j++) b(j - 1, i) = b(j, i) - f * b(j, k);
      b(mm - 1, i) = 0.0;
    }
  }
  bm.resize(5 * (size_t)n), bl.resize(4 * (size_t)n), am.resize(60);
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < 5; j++) bm[(size_t)i * 5 + j] = (float)b(j, i);
    for (int j = 0; j < 4; j++) bl[(size_t)i * 4 + j] = (float)L[(size_t)j * n + i];
  }
  for (int i = 0; i < 60; i++) am[i] = (float)A[i];
  if (rdiag) {
    rdiag->resize(n);
    for (int i = 0; i < n; i++) (*rdiag)[i] = (float)(1.0 / b(0, i));
  }
}

void pml_profile(int w, double d, double dt, double vmax, double eps, double scaler, std::vector<float> &co) {
  // damping g_L = 0.75 ((w-L)/w)^2 ln(1/eps) / (w d / (dt vmax)), L from the
  // outer edge; per layer the constants of q' = a q - b p, p' = q' + c p.
  co.resize((size_t)w * 6);
  double beta = d / (dt * vmax);
  double dg1 = std::log(1.0 / eps) / (w * beta);
  for (int L = 0; L < w; L++) {
    double t = double(w - L) / w;
    double g0 = 0.75 * t * t * dg1;
    for (int k = 0; k < 2; k++) {
      double g = k ? g0 * scaler : g0;
      co[(size_t)L * 6 + 3 * k + 0] = (float)((1.0 - g) / (1.0 + g));
      co[(size_t)L * 6 + 3 * k + 1] = (float)(2.0 * g / (1.0 - g * g));
      co[(size_t)L * 6 + 3 * k + 2] = (float)(1.0 / (1.0 - g));
    }
  }
}

// libCommon's sincf_unnorm / blackman / dipole_unnorm are not in the reference
// tree; they are restated from their definitions.
// FdEngine_r2r::fftderiv1_r2r composes three linear maps on a line of n
// points, all unnormalised FFTW real-to-real transforms:
//   isign +1: F = DCT-II (REDFT10)  F[q][u] = 2 cos(pi (u + 1/2) q / n)
//             S: bin i <- -k_i bin i+1 (i < n-1), bin n-1 <- 0
//             B = DST-III (RODFT01) B[t][j] = 2 sin(pi (j + 1) (t + 1/2) / n), j < n-1;
//                                   B[t][n-1] = (-1)^t
//   isign -1: F = DST-II (RODFT10)  F[q][u] = 2 sin(pi (u + 1/2) (q + 1) / n)
//             S: bin i <- k_{i-1} bin i-1 (i >= 1), bin 0 <- 0
//             B = DCT-III (REDFT01) B[t][0] = 1, B[t][j] = 2 cos(pi j (t + 1/2) / n)
// with k_i = -(i + 1) dk and dk = pi / (d n) / 2 / n in float (constructor
// :11-13, assignW :66-70).  D = B S F in FP64, rounded once.
// FdEngine_r2c::fftderiv1_r2c (bgprtm/FdEngine_r2c.cpp:200-240) as the n x n
// matrix it applies to a line: a real-to-complex FFT, bin j times i k_j
// (k_j = -j dk, dk = 2 pi / (d n) / n in float, assignW :52-56; the DC bin and
// an even line's Nyquist bin give 0; an odd line's last bin carries isign),
// and the unnormalised complex-to-real FFT.  For a real line that is the
// circulant D[t][u] = c[(t - u) mod n] with
//   c[m] = -2 sum_{j=1..J} s_j k_j sin(2 pi j m / n),
// J the last bin below Nyquist, s_j = isign for an odd line's last bin and 1
// otherwise; FP64, rounded once.
void r2c_line_matrix(int n, float d, int isign, std::vector<float> &D) {
  const float dk = (float)(2.0f * M_PI / (double)(d * (float)n) * (double)(1.0f / float(n)));
  const int J = n % 2 == 0 ? n / 2 - 1 : (n - 1) / 2;
  std::vector<double> c(n, 0.0);
  for (int m = 0; m < n; m++) {
    double v = 0.0;
    for (int j = 1; j <= J; j++) {
      const double kj = (double)((float)(-j) * dk), sj = (n % 2 == 1 && j == n / 2) ? (double)isign : 1.0;
      v += sj * kj * std::sin(2.0 * M_PI * (double)(((long long)j * m) % n) / n);
    }
    c[m] = -2.0 * v;
  }
  D.assign((size_t)n * n, 0.f);
  for (int t = 0; t < n; t++)
    for (int u = 0; u < n; u++) D[(size_t)t * n + u] = (float)c[(t - u + n) % n];
}

void r2r_line_matrix(int n, float d, int isign, std::vector<float> &D) {
  const float dk = (float)(M_PI / (double)(d * (float)n) * 0.5 * (double)(1.0f / float(n)));
  std::vector<double> SF((size_t)n * n, 0.0);  // S F: row i = the multiplied bin i
  for (int i = 0; i < n; i++) {
    const int q = isign == 1 ? i + 1 : i - 1;  // the bin moved into i
    if (q < 0 || q >= n) continue;
    const double ki = (double)((float)(-((isign == 1 ? i : i - 1) + 1)) * dk);
    const double m = isign == 1 ? -ki : ki;
    for (int u = 0; u < n; u++) {
      const double f = isign == 1 ? 2.0 * std::cos(M_PI * (u + 0.5) * q / n)
                                  : 2.0 * std::sin(M_PI * (u + 0.5) * (q + 1) / n);
      SF[(size_t)i * n + u] = m * f;
    }
  }
  D.assign((size_t)n * n, 0.f);
  std::vector<double> b(n);
  for (int t = 0; t < n; t++) {
    for (int j = 0; j < n; j++)
      b[j] = isign == 1 ? (j == n - 1 ? (t % 2 ? -1.0 : 1.0) : 2.0 * std::sin(M_PI * (j + 1) * (t + 0.5) / n))
                        : (j == 0 ? 1.0 : 2.0 * std::cos(M_PI * j * (t + 0.5) / n));
    for (int u = 0; u < n; u++) {
      double v = 0;
      for (int j = 0; j < n; j++) v += b[j] * SF[(size_t)j * n + u];
      D[(size_t)t * n + u] = (float)v;
    }
  }
}

static float sinc_u(float x) { return x == 0.0f ? 1.0f : sinf(x) / x; }
static float dipole_u(float x) { return x == 0.0f ? 0.0f : (x * cosf(x) - sinf(x)) / (x * x); }
static float blackman_w(float t) { return 0.42f - 0.5f * cosf(t) + 0.08f * cosf(2.0f * t); }

int spread_coeffs(int n, float x, float k1, float k2, int *nlimit, int dipole, int ntaper, float *coeff) {
  const float pi = 3.14159265358979323846f;
  if (n == 1 || *nlimit < 2) {
    coeff[0] = 1.0f;
    *nlimit = 1;
    return (int)nearbyintf(x);
  }
  const bool sinc_only = (k1 == k2) || dipole;
  float a1 = k1 * pi * (sinc_only ? 2.0f : 1.0f), a2 = k2 * pi;
  int ix = (int)floorf(x);
  int m = std::min(std::min(ix, n - 1 - ix), *nlimit / 2);
  *nlimit = 2 * m;
  const int first = ix - m + 1, last = ix + m;
  const int ramp = m / 2;
  const float halfwin = std::max(last - x, x - first);
  for (int i = first; i <= last; i++) {
    float s = i - x;
    float p1 = dipole ? dipole_u(s * a1) : sinc_u(s * a1);
    float v;
    if (sinc_only) {
      v = p1 * 2 * k1;
      if (m > 1) v *= blackman_w(pi * (halfwin - x + i) / halfwin);
    } else {
      // band-pass between k1 and k2 (difference of two squared sincs)
      float p2 = sinc_u(s * a2);
      v = (a2 * a2 * p2 * p2 - a1 * a1 * p1 * p1) / pi / (a2 - a1);
      int e = std::min(i - first, last - i);
      if (e < ramp && m > 1) v *= 0.5f * (1 - cosf(pi * e / ramp));
    }
    coeff[i - first] = v;
  }
  if (ntaper > 0 && n > 2 * ntaper) {
    // cosine ramp on kernel taps that fall within ntaper cells of either grid edge
    for (int t = 0; t < *nlimit; t++) {
      int g = first + t;
      int e = std::min(g, n - 1 - g);
      if (e < ntaper) coeff[t] *= 0.5f * (1.0f - cosf((float)(M_PI * e / ntaper)));
    }
  }
  return first;
}

}  // namespace rtm
