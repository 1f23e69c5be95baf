// Stand-in for the absent libCommon/Utl.hpp (test infrastructure for oracle/_ref).
#ifndef RTM_SHIM_UTL_HPP
#define RTM_SHIM_UTL_HPP
#include <string>
namespace libCommon {
struct Utl {
  static std::string free_memory() { return "n/a"; }
  static int mkpath(const char *) { return 0; }
  static bool haveFile(const std::string &) { return false; }
};
}
#endif
