// ref_shim.cpp - definitions the reference's compiled CPU kernels need from
// libraries that are absent from the reference tree (libCommon, MPI printing,
// FFTW's 1-D real transforms, the engines KernelCPU's constructor can name
// but our runs never select).
// TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/libbgprtm_ref.so.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "GetPar.h"
#include "MpiPrint.h"
#include "TimeRecorder.h"
#include "FdEngine_r2c.h"
#include "FdEngine_hfd.h"
#include "Util.h"
#include "libFFTV/transpose.h"
#include "libCommon/Taylor.h"
#include "../oracle_common.hpp"

ShimStore &shim_store() {
  static ShimStore s;
  return s;
}
Node global_pars;
TimeRecorder timeRecorder;

bool getBool(const Node &n, bool defaults) { return n.as<bool>(defaults); }
bool getBool(string key, bool defaults) { return global_pars[key].as<bool>(defaults); }
bool getBool(string key) { return global_pars[key].as<bool>(); }
int init_num_threads(bool) { return 1; }

namespace MpiPrint {
int printed1 = 0, rank = 0, verbose = 0;
static int vp(const char *fmt, va_list ap) { return verbose ? vfprintf(stderr, fmt, ap) : 0; }
int print1(const char *fmt, ...) { va_list a; va_start(a, fmt); int r = vp(fmt, a); va_end(a); return r; }
int printm(const char *fmt, ...) { va_list a; va_start(a, fmt); int r = vp(fmt, a); va_end(a); return r; }
int print1m(const char *fmt, ...) { va_list a; va_start(a, fmt); int r = vp(fmt, a); va_end(a); return r; }
int print2m(const char *fmt, ...) { va_list a; va_start(a, fmt); int r = vp(fmt, a); va_end(a); return r; }
}  // namespace MpiPrint

namespace libCommon {
float Taylor::coef1[12][13];
float Taylor::coef2[12][13];
float (&Taylor::optim1)[12][13] = Taylor::coef1;
float (&Taylor::optim2)[12][13] = Taylor::coef2;
static struct TaylorInit {
  TaylorInit() {
    for (int ne = 1; ne <= 12; ne++) {
      double c1[13], c2[13];
      orc::taylor_weights(ne, c1, c2);
      for (int j = 1; j <= ne; j++) Taylor::coef1[ne - 1][j - 1] = (float)c1[j];
      for (int j = 0; j <= ne; j++) Taylor::coef2[ne - 1][j] = (float)c2[j];
    }
  }
} taylor_init;
}  // namespace libCommon

// FFTW's single-precision 1-D real transforms, by their documented
// definitions (unnormalised; forward sign -1):
//   r2c  X_j = sum_t x_t e^{-2 pi i j t / n},  j = 0 .. n/2
//   c2r  y_t = sum_{j=0}^{n-1} X_j e^{+2 pi i j t / n} with X_{n-j} = conj(X_j);
//        the imaginary parts of X_0 and (n even) X_{n/2} are not read.
// Plain DFTs in double rounded to float: FFTW's results, not its rounding.
struct fftwf_plan_s {
  int n, c2r, kind;
};
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *, fftwf_complex *, unsigned) { return new fftwf_plan_s{n, 0, -1}; }
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *, float *, unsigned) { return new fftwf_plan_s{n, 1, -1}; }
fftwf_plan fftwf_plan_r2r_1d(int n, float *, float *, fftwf_r2r_kind kind, unsigned) {
  return new fftwf_plan_s{n, 0, (int)kind};
}
// The four r2r kinds FdEngine_r2r plans (unnormalised, FFTW's definitions):
//   REDFT10  Y_k = 2 sum_j X_j cos(pi (j + 1/2) k / n)
//   REDFT01  Y_k = X_0 + 2 sum_{j>=1} X_j cos(pi j (k + 1/2) / n)
//   RODFT10  Y_k = 2 sum_j X_j sin(pi (j + 1/2) (k + 1) / n)
//   RODFT01  Y_k = (-1)^k X_{n-1} + 2 sum_{j<=n-2} X_j sin(pi (j + 1) (k + 1/2) / n)
void fftwf_execute_r2r(const fftwf_plan p, float *in, float *out) {
  const int n = p->n;
  std::vector<double> y(n);
  for (int k = 0; k < n; k++) {
    double v = 0;
    switch (p->kind) {
      case FFTW_REDFT10:
        for (int j = 0; j < n; j++) v += 2.0 * in[j] * std::cos(M_PI * (j + 0.5) * k / n);
        break;
      case FFTW_REDFT01:
        v = in[0];
        for (int j = 1; j < n; j++) v += 2.0 * in[j] * std::cos(M_PI * j * (k + 0.5) / n);
        break;
      case FFTW_RODFT10:
        for (int j = 0; j < n; j++) v += 2.0 * in[j] * std::sin(M_PI * (j + 0.5) * (k + 1) / n);
        break;
      case FFTW_RODFT01:
        v = (k % 2 ? -1.0 : 1.0) * in[n - 1];
        for (int j = 0; j < n - 1; j++) v += 2.0 * in[j] * std::sin(M_PI * (j + 1) * (k + 0.5) / n);
        break;
      default:
        assertion(false, "r2r kind not in the stand-in");
    }
    y[k] = v;
  }
  for (int k = 0; k < n; k++) out[k] = (float)y[k];
}
void fftwf_destroy_plan(fftwf_plan p) { delete p; }
void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out) {
  const int n = p->n;
  std::vector<double> re(n / 2 + 1), im(n / 2 + 1);
  for (int j = 0; j <= n / 2; j++) {
    double a = 0, b = 0;
    for (int t = 0; t < n; t++) {
      const double th = 2.0 * M_PI * (double)(((long long)j * t) % n) / n;
      a += in[t] * std::cos(th), b -= in[t] * std::sin(th);
    }
    re[j] = a, im[j] = b;
  }
  for (int j = 0; j <= n / 2; j++) out[j][0] = (float)re[j], out[j][1] = (float)im[j];
}
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out) {
  const int n = p->n, top = n % 2 == 0 ? n / 2 - 1 : n / 2;
  std::vector<double> y(n);
  for (int t = 0; t < n; t++) {
    double v = in[0][0];
    if (n % 2 == 0) v += (t % 2 ? -1.0 : 1.0) * in[n / 2][0];
    for (int j = 1; j <= top; j++) {
      const double th = 2.0 * M_PI * (double)(((long long)j * t) % n) / n;
      v += 2.0 * (in[j][0] * std::cos(th) - in[j][1] * std::sin(th));
    }
    y[t] = v;
  }
  for (int t = 0; t < n; t++) out[t] = (float)y[t];
}

// libfftv::ssetranspose, as volumefilter.cpp uses it (a plain transpose of
// n2 rows of n1 values)
namespace libfftv {
void ssetranspose(int n1, int n2, float *in, int ldin, float *out, int ldout) {
  for (int r = 0; r < n2; r++)
    for (int c = 0; c < n1; c++) out[(size_t)c * ldout + r] = in[(size_t)r * ldin + c];
}
}  // namespace libfftv

// Util::transpose (bgprtm/Util.cpp:25-76) as intended: out[ix][iy] =
// in[iy][ix] for nx x ny, row pitches dimIn / dimOut.  The reference's SSE
// body omits the store of the third transposed row (Util.cpp:51-54).
void Util::transpose(int nx, int ny, int dimIn, int dimOut, float *in, float *out) {
  for (int ix = 0; ix < nx; ix++)
    for (int iy = 0; iy < ny; iy++) out[(size_t)ix * dimOut + iy] = in[(size_t)iy * dimIn + ix];
}

// Engines KernelCPU's constructor can name (HFD); never selected here.
#define NOT_BUILT(...) assertion(false, "engine not built in the oracle harness")
FdEngine_hfd::FdEngine_hfd(int a, int b, int c, float d, float e, float f, int g) : FdEngine(a, b, c, d, e, f, g) { NOT_BUILT(); }
FdEngine_hfd::~FdEngine_hfd() {}
void FdEngine_hfd::dx1_2D(float *, float *, float *, int, int, int) {}
void FdEngine_hfd::dy1_2D(float *, float *, float *, int, int, int) {}
void FdEngine_hfd::dz1_2D(float *, float *, float *, int, int, int) {}
