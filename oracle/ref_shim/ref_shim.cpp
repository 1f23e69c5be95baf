// ref_shim.cpp - definitions the reference's compiled CPU kernels need from
// libraries that are absent from the reference tree (libCommon, MPI printing,
// the FFT engines KernelCPU's constructor can name but our runs never select).
// TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/libbgprtm_ref.so.
#include <cstdarg>
#include <cstdio>
#include <string>

#include "GetPar.h"
#include "MpiPrint.h"
#include "TimeRecorder.h"
#include "FdEngine_r2c.h"
#include "FdEngine_r2r.h"
#include "FdEngine_hfd.h"
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

// Engines KernelCPU's constructor can name (FFT / HFD); never selected here.
#define NOT_BUILT(...) assertion(false, "engine not built in the oracle harness")
FdEngine_r2c::FdEngine_r2c(int a, int b, int c, float d, float e, float f, int g) : FdEngine(a, b, c, d, e, f, g) { NOT_BUILT(); }
FdEngine_r2c::~FdEngine_r2c() {}
void FdEngine_r2c::dx1_2D(float *, float *, float *, int, int, int) {}
void FdEngine_r2c::dy1_2D(float *, float *, float *, int, int, int) {}
void FdEngine_r2c::dz1_2D(float *, float *, float *, int, int, int) {}
void FdEngine_r2c::dx1_2D(float *, float *, float *, int, int, int, float *, float *) {}
void FdEngine_r2c::dy1_2D(float *, float *, float *, int, int, int, float *, float *) {}
void FdEngine_r2c::dz1_2D(float *, float *, float *, int, int, int, float *, float *) {}
FdEngine_r2r::FdEngine_r2r(int a, int b, int c, float d, float e, float f, int g) : FdEngine(a, b, c, d, e, f, g) { NOT_BUILT(); }
FdEngine_r2r::~FdEngine_r2r() {}
void FdEngine_r2r::dx1_2D(float *, float *, float *, int, int, int) {}
void FdEngine_r2r::dy1_2D(float *, float *, float *, int, int, int) {}
void FdEngine_r2r::dz1_2D(float *, float *, float *, int, int, int) {}
void FdEngine_r2r::dx1_2D(float *, float *, float *, int, int, int, float *, float *) {}
void FdEngine_r2r::dy1_2D(float *, float *, float *, int, int, int, float *, float *) {}
void FdEngine_r2r::dz1_2D(float *, float *, float *, int, int, int, float *, float *) {}
FdEngine_hfd::FdEngine_hfd(int a, int b, int c, float d, float e, float f, int g) : FdEngine(a, b, c, d, e, f, g) { NOT_BUILT(); }
FdEngine_hfd::~FdEngine_hfd() {}
void FdEngine_hfd::dx1_2D(float *, float *, float *, int, int, int) {}
void FdEngine_hfd::dy1_2D(float *, float *, float *, int, int, int) {}
void FdEngine_hfd::dz1_2D(float *, float *, float *, int, int, int) {}
