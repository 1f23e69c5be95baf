// Stand-in for the absent jseisIO/jseisUtil.h (test infrastructure for oracle/_ref).
#ifndef RTM_SHIM_JSEISUTIL_H
#define RTM_SHIM_JSEISUTIL_H
namespace jsIO {
struct jseisUtil {
  template <typename... A> static void save_zxy(A...) {}
};
}
#endif
