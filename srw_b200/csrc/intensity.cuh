// Intensity components of one point of the field (srTRadGenManip, cpp/src/core/srradmnp.h:367-434),
// shared by srwlCalcIntFromElecField and the intensity extraction passes of a propagation.
#pragma once
#include <cuda_runtime.h>

namespace srwg {

// FormalPhase (srradmnp.h:434): argument from atan of the FP32 ratio, the reference's quadrants
__device__ __forceinline__ double formal_phase(float re, float im)
{
    const double HalhPi = 1.5707963267949, Pi = 3.1415926535898;
    if (re != 0.f) {
        const double a = atan((double)__fdiv_rn(im, re));
        if (im <= 0.f) return re < 0.f ? a - Pi : a;
        return re < 0.f ? a + Pi : a;
    }
    if (im == 0.f) return 0.;
    return im > 0.f ? HalhPi : -HalhPi;
}

// IntensityComponent (srradmnp.h:367-425) with its FP32 / FP64 operation order (no contraction):
// what 0 intensity, 2 phase, 3 Re E, 6 Im E; pol 0..6 and the Stokes components -1..-4
__device__ __forceinline__ float int_component(float2 x, float2 z, int pol, int what)
{
    if (pol == -1)
        return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(x.x, x.x), __fmul_rn(x.y, x.y)), __fmul_rn(z.x, z.x)),
                         __fmul_rn(z.y, z.y));
    if (pol == -2)
        return __fsub_rn(__fadd_rn(__fmul_rn(x.x, x.x), __fmul_rn(x.y, x.y)),
                         __fadd_rn(__fmul_rn(z.x, z.x), __fmul_rn(z.y, z.y)));
    if (pol == -3) return (float)(2. * (double)__fadd_rn(__fmul_rn(x.x, z.x), __fmul_rn(x.y, z.y)));
    if (pol == -4) return (float)(2. * (double)__fsub_rn(__fmul_rn(x.x, z.y), __fmul_rn(x.y, z.x)));
    float a, b;
    bool half = true;
    switch (pol) {
    case 0: a = x.x; b = x.y; half = false; break;
    case 1: a = z.x; b = z.y; half = false; break;
    case 2: a = __fadd_rn(x.x, z.x); b = __fadd_rn(x.y, z.y); break;
    case 3: a = __fsub_rn(x.x, z.x); b = __fsub_rn(x.y, z.y); break;
    case 5: a = __fsub_rn(x.x, z.y); b = __fadd_rn(x.y, z.x); break;
    case 4: a = __fadd_rn(x.x, z.y); b = __fsub_rn(x.y, z.x); break;
    default:
        if (what == 0)
            return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(x.x, x.x), __fmul_rn(x.y, x.y)), __fmul_rn(z.x, z.x)),
                             __fmul_rn(z.y, z.y));
        a = x.x; b = x.y; half = false;
    }
    if (what == 0) {
        const float v = __fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b));
        return half ? (float)(0.5 * (double)v) : v;
    }
    if (what == 2) return (float)formal_phase(a, b);
    const float v = what == 3 ? a : b;
    return half ? (float)__dmul_rn(0.70710678, (double)v) : v;
}

}  // namespace srwg
