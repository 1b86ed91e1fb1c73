// General-length line pass instantiations with non-separable point-wise work (see lineg.cuh).
#include "lineg.cuh"

namespace srwg {
Line2Fn lineg_e_get(bool cols) { return cols ? lineg_kernel<true, true> : lineg_kernel<false, true>; }
}  // namespace srwg
