// Line pass instantiation for lines of 2^10 points without non-separable point-wise work (see
// line2.cuh).
#include "line2.cuh"

namespace srwg {
Line2Fn line2_get_10(bool cols) { return cols ? line2_kernel<10, true, false> : line2_kernel<10, false, false>; }
}  // namespace srwg
