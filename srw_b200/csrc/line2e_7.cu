// Line pass instantiations for lines of 2^7 points with non-separable point-wise work (see
// line2.cuh).
#include "line2.cuh"

namespace srwg {
Line2Fn line2e_get_7(bool cols, int f1, int f2)
{
    return cols ? line2_select<7, true, true>(f1, f2) : line2_select<7, false, true>(f1, f2);
}
}  // namespace srwg
