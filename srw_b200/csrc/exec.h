// Host helpers shared by the entry points (capi.cpp, noalloc.cu).
#pragma once
#include <string>
#include "kernels.h"

namespace srwg {
int line_config(const LineDesc& d, LineLaunch& p);   // launch shape of a line pass (capi.cpp)
int radix_plan(int N, int* r);
void set_last_detail(const std::string& s);          // detail text for srwlUtiGetErrText
}  // namespace srwg
