// Line pass instantiation for lines of 2^6 points with non-separable point-wise work (see
// line2.cuh).
#include "line2.cuh"

namespace srwg {
Line2Fn line2e_get_6(bool cols) { return cols ? line2_kernel<6, true, true> : line2_kernel<6, false, true>; }
}  // namespace srwg
