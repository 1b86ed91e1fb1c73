// Line pass instantiation for lines of 2^12 points with non-separable point-wise work (see
// line2.cuh).
#include "line2.cuh"

namespace srwg {
Line2Fn line2e_get_12(bool cols) { return cols ? line2_kernel<12, true, true> : line2_kernel<12, false, true>; }
}  // namespace srwg
