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
inline float maxfabs(const float *d, size_t n1, size_t n2, int = 1) {
  float m = 0;
  for (size_t i = 0; i < n1 * n2; i++) m = std::fabs(d[i]) > m ? std::fabs(d[i]) : m;
  return m;
}
}
#endif
