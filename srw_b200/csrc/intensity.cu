// srwlCalcIntFromElecField (cpp/src/lib/srwlib.h:748, srwlib.cpp:757) on the GPU for a wavefront at a
// single photon energy, vs x and y (srTRadGenManip::ExtractSingleElecIntensity2DvsXZ,
// cpp/src/core/srradmnp.cpp:681): single-electron intensity of a polarisation component, its phase,
// Re E or Im E, or the four Stokes components; written into, averaged into or added to the caller's
// array.  One element-wise pass over the two field components (HBM-bound: 16 B read and 4-16 B
// written per point).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/srwl_b200.h"
#include "errors.h"
#include "exec.h"

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

// mode 0: write; 1: average with weight iter (FP64, then FP32); 2: add
__global__ void __launch_bounds__(256) intensity_kernel(const float2* __restrict__ ex, const float2* __restrict__ ez,
                                                        long long n, int pol, int what, int mode, double iter,
                                                        double inv, float* outF, double* outD)
{
    const int np = pol == -5 ? 4 : 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float2 x = ex[i], z = ez[i];
        for (int k = 0; k < np; k++) {
            const float v = int_component(x, z, np == 4 ? -1 - k : pol, what);
            const long long o = i + k * n;
            if (outD) {
                const double r = (double)v;
                if (mode == 0) outD[o] = r;
                else if (mode == 1) outD[o] = __dmul_rn(__dadd_rn(__dmul_rn(outD[o], iter), r), inv);
                else outD[o] = __dadd_rn(outD[o], r);
            } else {
                if (mode == 0) outF[o] = v;
                else if (mode == 1) outF[o] = (float)__dmul_rn(__dadd_rn(__dmul_rn((double)outF[o], iter), (double)v), inv);
                else outF[o] = __fadd_rn(outF[o], v);
            }
        }
    }
}

}  // namespace srwg

using namespace srwg;

#define INT_TRY(x)                                                                      \
    do {                                                                                \
        cudaError_t e__ = (x);                                                          \
        if (e__ != cudaSuccess) {                                                       \
            set_last_detail(std::string(#x) + ": " + cudaGetErrorString(e__));          \
            return SRWG_ERR_CUDA;                                                       \
        }                                                                               \
    } while (0)

extern "C" SRWG_API int srwlCalcIntFromElecField(char* pInt, SRWLWfr* pWfr, char pol, char intType, char depType,
                                                 double e, double x, double y, double* arMeth, void* pFldTrj,
                                                 double* arParGPU)
{
    std::lock_guard<std::mutex> lk(library_mutex());
    set_last_detail("");
    (void)e; (void)x; (void)y;
    if (pWfr == nullptr || pInt == nullptr) return SRWL_INCORRECT_PARAM_FOR_INT_EXTR;
    if (pFldTrj != nullptr) {
        set_last_detail("intensity with the central electron's field or trajectory (finite energy spread)");
        return SRWG_ERR_UNSUPPORTED;
    }
    if (pWfr->mesh.ne != 1) { set_last_detail("intensity extraction for ne == 1 only"); return SRWG_ERR_UNSUPPORTED; }
    if (depType != 3) { set_last_detail("intensity extraction vs x and y (depType 3) only"); return SRWG_ERR_UNSUPPORTED; }
    int what;
    switch (intType) {           // SRWL numbering -> the reference's internal one (srwlib.cpp:792)
    case 0: what = 0; break;
    case 4: what = 2; break;
    case 5: what = 3; break;
    case 6: what = 6; break;
    default:
        set_last_detail("intensity type " + std::to_string((int)intType) + " (single-electron intensity, phase, Re E "
                        "and Im E are supported)");
        return SRWG_ERR_UNSUPPORTED;
    }
    if (pol == -5 && what != 0) { set_last_detail("all Stokes components for the intensity only"); return SRWG_ERR_UNSUPPORTED; }
    // method: [0] = 1 averages with [1] earlier iterations (0: writes, < 0: adds), [0] = 2 adds
    int mode = 0;
    double iter = 0.;
    if (arMeth != nullptr) {
        if (arMeth[0] == 1) iter = arMeth[1];
        else if (arMeth[0] == 2) iter = -1;
        mode = iter == 0. ? 0 : (iter > 0. ? 1 : 2);
    }
    int dev = 0;
    if (arParGPU != nullptr && arParGPU[0] >= 1. && arParGPU[1] >= 1.) dev = (int)arParGPU[1] - 1;
    DeviceCtx* c = nullptr;
    int r = device_ctx(dev, &c);
    if (r) return r;
    const long long n = (long long)pWfr->mesh.nx * pWfr->mesh.ny;
    if (n <= 0) return SRWL_INCORRECT_PARAM_FOR_INT_EXTR;
    const long long nOut = n * (pol == -5 ? 4 : 1);
    const size_t esz = what == 2 ? sizeof(double) : sizeof(float);
    const size_t bytes = 2 * n * sizeof(float2) + nOut * esz;
    if (c->intBuf == nullptr || c->intBytes < bytes) {
        if (c->intBuf) cudaFree(c->intBuf);
        c->intBuf = nullptr; c->intBytes = 0;
        INT_TRY(cudaMalloc(&c->intBuf, bytes));
        c->intBytes = bytes;
    }
    float2* dX = (float2*)c->intBuf;
    float2* dZ = dX + n;
    char* dOut = (char*)(dZ + n);
    cudaStream_t st = c->stream;
    if (pWfr->arEx) INT_TRY(cudaMemcpyAsync(dX, pWfr->arEx, n * sizeof(float2), cudaMemcpyHostToDevice, st));
    else INT_TRY(cudaMemsetAsync(dX, 0, n * sizeof(float2), st));
    if (pWfr->arEy) INT_TRY(cudaMemcpyAsync(dZ, pWfr->arEy, n * sizeof(float2), cudaMemcpyHostToDevice, st));
    else INT_TRY(cudaMemsetAsync(dZ, 0, n * sizeof(float2), st));
    if (mode != 0) INT_TRY(cudaMemcpyAsync(dOut, pInt, nOut * esz, cudaMemcpyHostToDevice, st));
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    intensity_kernel<<<blocks, 256, 0, st>>>(dX, dZ, n, (int)pol, what, mode, iter, 1. / (iter + 1.),
                                             what == 2 ? nullptr : (float*)dOut, what == 2 ? (double*)dOut : nullptr);
    INT_TRY(cudaGetLastError());
    INT_TRY(cudaMemcpyAsync(pInt, dOut, nOut * esz, cudaMemcpyDeviceToHost, st));
    INT_TRY(cudaStreamSynchronize(st));
    return 0;
}
