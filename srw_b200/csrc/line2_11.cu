// Line pass instantiation for lines of 2^11 points (see line2.cuh).
#include "line2.cuh"

namespace srwg {
Line2Fn line2_get_11(bool cols) { return cols ? line2_kernel<11, true> : line2_kernel<11, false>; }
}  // namespace srwg
