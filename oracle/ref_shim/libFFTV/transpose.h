// Stand-in for libFFTV/transpose.h: the one call volumefilter.cpp makes.
// ssetranspose(n1, n2, in, ldin, out, ldout): in holds n2 rows of n1 values
// (row pitch ldin); out[c * ldout + r] = in[r * ldin + c] (ref_shim.cpp).
#ifndef RTM_SHIM_LIBFFTV_TRANSPOSE_H
#define RTM_SHIM_LIBFFTV_TRANSPOSE_H
// volumefilter.cpp gets memcpy, min and max through this header
#include <algorithm>
#include <cstring>
using std::max;
using std::min;
namespace libfftv {
void ssetranspose(int n1, int n2, float *in, int ldin, float *out, int ldout);
}
#endif
