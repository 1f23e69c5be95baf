// Stand-in for the absent libCommon/Taylor.h.  The reference reads
// Taylor::coef1[nev-1][j-1] (1st-derivative central-difference weights of
// order 2*nev) and Taylor::coef2[nev-1][0..nev] (2nd-derivative weights).
// The tables are filled from the standard Taylor-series conditions (solved
// in double in ref_shim.cpp).  The "optim" tables of the original library
// are unpublished, so optim1/optim2 alias the Taylor ones; the oracle runs
// with fd_use_taylor=1 anyway.  Test infrastructure for oracle/_ref only.
#ifndef RTM_SHIM_TAYLOR_H
#define RTM_SHIM_TAYLOR_H
namespace libCommon {
struct Taylor {
  static float coef1[12][13];
  static float coef2[12][13];
  static float (&optim1)[12][13];
  static float (&optim2)[12][13];
  static void derive1(float *, const float *, int, float, int, bool) {}
  static void derive2(float *, const float *, int, float, int, bool) {}
};
}
#endif
