// Line pass instantiation for lines of 2^8 points (see line2.cuh).
#include "line2.cuh"

namespace srwg {
Line2Fn line2_get_8(bool cols) { return cols ? line2_kernel<8, true> : line2_kernel<8, false>; }
}  // namespace srwg
