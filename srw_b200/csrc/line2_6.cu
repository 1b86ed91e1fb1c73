// Line pass instantiation for lines of 2^6 points (see line2.cuh).
#include "line2.cuh"

namespace srwg {
Line2Fn line2_get_6(bool cols) { return cols ? line2_kernel<6, true> : line2_kernel<6, false>; }
}  // namespace srwg
