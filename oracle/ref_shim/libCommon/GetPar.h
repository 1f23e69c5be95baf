// Stand-in for the absent in-house libCommon/GetPar.h (a yaml-cpp based
// parameter tree).  Only what the compiled CPU kernels read is provided: a
// flat string map addressed by "a/b" paths, `as<T>(default)`, `IsDefined()`,
// truthiness and assignment.  Test infrastructure for oracle/_ref only.
#ifndef RTM_SHIM_LIBCOMMON_GETPAR_H
#define RTM_SHIM_LIBCOMMON_GETPAR_H
#include <map>
#include <string>
#include <sstream>
#include <vector>
#include <bitset>
#include <algorithm>
#include <stdexcept>
using std::string;
using std::bitset;
using std::min;
using std::max;

struct ShimStore {
  std::map<string, string> kv;
};
ShimStore &shim_store();

class Node {
public:
  Node() : path_("") {}
  explicit Node(const string &p) : path_(p) {}
  Node operator[](const string &k) const { return Node(path_.empty() ? k : path_ + "/" + k); }
  Node operator[](const char *k) const { return (*this)[string(k)]; }
  bool IsDefined() const {
    auto &kv = shim_store().kv;
    if (kv.count(path_)) return true;
    string pre = path_ + "/";
    for (auto &e : kv) if (e.first.compare(0, pre.size(), pre) == 0) return true;
    return false;
  }
  explicit operator bool() const { return IsDefined(); }
  bool operator!() const { return !IsDefined(); }
  template <typename T> T as() const {
    auto &kv = shim_store().kv;
    auto it = kv.find(path_);
    if (it == kv.end()) throw std::runtime_error("shim Node: missing key " + path_);
    return conv<T>(it->second);
  }
  template <typename T> T as(const T &def) const {
    auto &kv = shim_store().kv;
    auto it = kv.find(path_);
    if (it == kv.end()) return def;
    return conv<T>(it->second);
  }
  string as(const char *def) const { return as<string>(string(def)); }
  template <typename T> Node &operator=(const T &v) {
    std::ostringstream os;
    os.precision(17);
    os << v;
    shim_store().kv[path_] = os.str();
    return *this;
  }
  Node &operator=(const string &v) { shim_store().kv[path_] = v; return *this; }
  Node &operator=(const char *v) { shim_store().kv[path_] = v; return *this; }
  const string &path() const { return path_; }

private:
  template <typename T> static T conv(const string &s) {
    std::istringstream is(s);
    T v{};
    is >> v;
    return v;
  }
  string path_;
};
template <> inline string Node::conv<string>(const string &s) { return s; }
template <> inline bool Node::conv<bool>(const string &s) {
  string t = s;
  std::transform(t.begin(), t.end(), t.begin(), ::tolower);
  return t == "1" || t == "true" || t == "yes" || t == "on";
}

#include <cstdio>
#include <cstdlib>
#define assertion(cond, ...)                                                    \
  do {                                                                         \
    if (!(cond)) {                                                             \
      fprintf(stderr, "reference assertion failed: %s (%s:%d): ", #cond,       \
              __FILE__, __LINE__);                                             \
      fprintf(stderr, __VA_ARGS__);                                            \
      fprintf(stderr, "\n");                                                   \
      abort();                                                                 \
    }                                                                          \
  } while (0)
#define GLOBAL "global"
#define LOCAL "local"
bool getBool(const Node &n, bool defaults);
#endif
