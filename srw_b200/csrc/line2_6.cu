// Line pass instantiations for lines of 2^6 points without non-separable point-wise work (see
// line2.cuh).
#include "line2.cuh"

namespace srwg {
Line2Fn line2_get_6(bool cols, int f1, int f2)
{
    return cols ? line2_select<6, true, false>(f1, f2) : line2_select<6, false, false>(f1, f2);
}
}  // namespace srwg
