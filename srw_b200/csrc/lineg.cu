// General-length line pass instantiations without non-separable point-wise work (see lineg.cuh).
#include "lineg.cuh"

namespace srwg {
Line2Fn lineg_get(bool cols) { return cols ? lineg_kernel<true, false> : lineg_kernel<false, false>; }
}  // namespace srwg
