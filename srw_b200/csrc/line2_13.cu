// Line pass instantiation for lines of 2^13 points without non-separable point-wise work (see
// line2.cuh).
#include "line2.cuh"

namespace srwg {
Line2Fn line2_get_13(bool cols) { return cols ? line2_kernel<13, true, false> : line2_kernel<13, false, false>; }
}  // namespace srwg
