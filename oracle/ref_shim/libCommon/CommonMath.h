// Stand-in for the absent libCommon/CommonMath.h (test infrastructure for oracle/_ref).
#ifndef RTM_SHIM_COMMONMATH_H
#define RTM_SHIM_COMMONMATH_H
#include <cfloat>
#include <cmath>
#include <cstddef>
#ifndef FLT_PI
#define FLT_PI 3.14159265358979323846f
#endif
#ifndef FLT_2_PI
#define FLT_2_PI 6.28318530717958647692f
#endif
namespace libCommon {
// the basis functions Util::CompactOrmsbySpreadCoeff calls, from their
// definitions: unnormalised sinc sin(x)/x, its derivative-like dipole
// (x cos x - sin x)/x^2, and the Blackman window 0.42 - 0.5 cos t + 0.08 cos 2t
inline float sincf_unnorm(float x) { return x == 0.0f ? 1.0f : sinf(x) / x; }
inline float dipole_unnorm(float x) { return x == 0.0f ? 0.0f : (x * cosf(x) - sinf(x)) / (x * x); }
inline float blackman(float t) { return 0.42f - 0.5f * cosf(t) + 0.08f * cosf(2.0f * t); }
inline float maxfabs(const float *d, size_t n1, size_t n2, int = 1) {
  float m = 0;
  for (size_t i = 0; i < n1 * n2; i++) m = std::fabs(d[i]) > m ? std::fabs(d[i]) : m;
  return m;
}
}
#endif
