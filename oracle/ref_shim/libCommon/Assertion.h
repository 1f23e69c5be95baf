// Stand-in for libCommon/Assertion.h: assertion() comes with the GetPar stand-in.
#ifndef RTM_SHIM_ASSERTION_H
#define RTM_SHIM_ASSERTION_H
#include "libCommon/GetPar.h"
// Util.cpp reaches std::cout and memset through this header
#include <cstring>
#include <iostream>
#endif
