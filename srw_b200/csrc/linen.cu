// Specialised general-length line pass, compiled once per length: nvcc -DSRWG_LINEN=<N> (see
// linen_lengths.h for the lengths and linen.cuh for the kernel).
#include "linen.cuh"

#ifndef SRWG_LINEN
#error "compile with -DSRWG_LINEN=<line length>"
#endif
#define SRWG_CAT2(a, b) a##b
#define SRWG_CAT(a, b) SRWG_CAT2(a, b)

namespace srwg {
Line2Fn SRWG_CAT(linen_get_, SRWG_LINEN)(bool cols, bool extra, int nt, bool inten)
{
    return linen_select<SRWG_LINEN>(cols, extra, nt, inten);
}
}  // namespace srwg
