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
#include "common.cuh"
#include "exec.h"
#include "intensity.cuh"
#include "kernels.h"

namespace srwg {

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

// 1D cuts and the single point (dependences 1: vs x at y, 2: vs y at x, 0: at (x, y)) of a wavefront
// with ne == 1: ExtractSingleElecIntensity1DvsX / 1DvsZ / 1DvsE (srradmnp.cpp:224-680) reduce to
// IntensityComponentSimpleInterpol2D (srradmnp.h:353) on two lines L0, L1 of the field (rows z0, z1
// for the x cut and the point, columns x0, x1 for the y cut), with the reference's FP32 differences
// and FP64 weights; the phase takes the first corner.  k0, k1: the corners' positions along the lines
// for the point (dep 0); the cuts take position p of both lines.
__global__ void __launch_bounds__(256) cut_kernel(const float2* __restrict__ ex, const float2* __restrict__ ez,
                                                  int nLine, int nOut, int dep, int k0, int k1, double a1, double a2,
                                                  int pol, int what, float* outF, double* outD)
{
    const int np = pol == -5 ? 4 : 1;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nOut; p += gridDim.x * blockDim.x) {
        const int i0 = dep == 0 ? k0 : p, i1 = dep == 0 ? k1 : p;
        const float2 x00 = ex[i0], x10 = ex[i1], x01 = ex[nLine + i0], x11 = ex[nLine + i1];
        const float2 z00 = ez[i0], z10 = ez[i1], z01 = ez[nLine + i0], z11 = ez[nLine + i1];
        for (int k = 0; k < np; k++) {
            const int pc = np == 4 ? -1 - k : pol;
            const float I00 = int_component(x00, z00, pc, what);
            double r;
            if (what == 2) {
                r = (double)I00;
            } else {
                const float I10 = int_component(x10, z10, pc, what), I01 = int_component(x01, z01, pc, what);
                const float I11 = int_component(x11, z11, pc, what);
                const float t = __fadd_rn(__fsub_rn(__fsub_rn(I00, I01), I10), I11);
                r = __dmul_rn((double)t, __dmul_rn(a1, a2));
                r = __dadd_rn(r, __dmul_rn((double)__fsub_rn(I10, I00), a1));
                r = __dadd_rn(r, __dmul_rn((double)__fsub_rn(I01, I00), a2));
                r = (double)(float)__dadd_rn(r, (double)I00);
            }
            const long long o = p + (long long)k * nOut;
            if (outD) outD[o] = r;
            else outF[o] = (float)r;
        }
    }
}

// SetupIntCoord (srradmnp.cpp:35): the node below arg (truncation), the next one, and the relative
// distance from the first (FP64, the reference's operation order)
static void setup_int_coord(double start, double step, long long n, double arg, long long& i0, long long& i1,
                            double& rel)
{
    if (n <= 1) { i0 = i1 = 0; rel = 0.; return; }
    const double inv = 1. / step;
    i0 = (long)((arg - start) * inv);
    if (i0 < 0) { i0 = 0; i1 = i0; }
    else if (i0 >= n - 1) { i0 = n - 1; i1 = i0; }
    else i1 = i0 + 1;
    rel = inv * (arg - i0 * step - start);
}

// intensity extraction pass of a propagation (srTCompositeOptElem::ExtractPropagatedIntensity,
// cpp/src/core/sroptcnt.cpp:429, writing as srwlCalcIntFromElecField does): the field at an element
// boundary is the source buffer times the operators still pending on it (separable tables and the
// non-separable work), applied on the fly
__global__ void __launch_bounds__(256) extract_kernel(const MomDesc* __restrict__ gd, const float2* __restrict__ s0,
                                                      const float2* __restrict__ s1, const float2* __restrict__ tabs,
                                                      float* outF, double* outD)
{
    const MomDesc& d = *gd;
    const int nx = d.nx;
    const long long n = (long long)nx * d.nz;
    const long long tx = d.t.tab, tz = d.t.ltab;
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
        const int iz = (int)(o / nx), ix = (int)(o - (long long)iz * nx);
        float2 f = make_float2(1.f, 0.f);
        if (tx >= 0) f = __ldg(&tabs[tx + ix]);
        if (tz >= 0) f = cmul(f, __ldg(&tabs[tz + iz]));
        if (d.has_extra) {
            bool zero = false;
            extra_eval(d.extra, ix, iz, f, zero, tabs);
            if (zero) f = make_float2(0.f, 0.f);
        }
        const float2 x = cmul(f, __ldg(&s0[o])), z = cmul(f, __ldg(&s1[o]));
        const float v = int_component(x, z, d.ipol, d.iwhat);
        if (outD) outD[o] = (double)v;
        else outF[o] = v;
    }
}

cudaError_t launch_extract(const MomDesc& d, const MomDesc* gd, const float2* s0, const float2* s1,
                           const float2* tabs, char* out, cudaStream_t st)
{
    const long long n = (long long)d.nx * d.nz;
    if (n <= 0 || out == nullptr) return cudaErrorInvalidValue;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    extract_kernel<<<blocks, 256, 0, st>>>(gd, s0, s1, tabs, d.iwhat == 2 ? nullptr : (float*)out,
                                           d.iwhat == 2 ? (double*)out : nullptr);
    return cudaGetLastError();
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

// dependences 0, 1, 2: the two field lines the result needs go to the device (rows: contiguous;
// columns: strided copies), one kernel makes the cut, which comes back (written, as the reference's
// 1D extractions do: no averaging)
static int int_cut(DeviceCtx* c, char* pInt, const SRWLWfr* pWfr, char pol, int what, int dep, double x, double y)
{
    const long long nx = pWfr->mesh.nx, nz = pWfr->mesh.ny;
    const double xStep = nx > 1 ? (pWfr->mesh.xFin - pWfr->mesh.xStart) / (nx - 1) : 0.;
    const double zStep = nz > 1 ? (pWfr->mesh.yFin - pWfr->mesh.yStart) / (nz - 1) : 0.;
    long long x0, x1, z0, z1;
    double ax, az;
    setup_int_coord(pWfr->mesh.xStart, xStep, nx, x, x0, x1, ax);
    setup_int_coord(pWfr->mesh.yStart, zStep, nz, y, z0, z1, az);
    const bool cols = dep == 2;
    const long long nLine = cols ? nz : nx;
    const int nOut = dep == 0 ? 1 : (int)nLine;
    const int np = pol == -5 ? 4 : 1;
    const size_t esz = what == 2 ? sizeof(double) : sizeof(float);
    const size_t bytes = 4 * nLine * sizeof(float2) + (size_t)np * nOut * esz;
    if (c->intBuf == nullptr || c->intBytes < bytes) {
        if (c->intBuf) cudaFree(c->intBuf);
        c->intBuf = nullptr; c->intBytes = 0;
        INT_TRY(cudaMalloc(&c->intBuf, bytes));
        c->intBytes = bytes;
    }
    float2* dX = (float2*)c->intBuf;
    float2* dZ = dX + 2 * nLine;
    char* dOut = (char*)(dZ + 2 * nLine);
    cudaStream_t st = c->stream;
    const float2* src[2] = {(const float2*)pWfr->arEx, (const float2*)pWfr->arEy};
    float2* dst[2] = {dX, dZ};
    for (int comp = 0; comp < 2; comp++) {
        for (int l = 0; l < 2; l++) {
            float2* d = dst[comp] + l * nLine;
            if (src[comp] == nullptr) { INT_TRY(cudaMemsetAsync(d, 0, nLine * sizeof(float2), st)); continue; }
            if (cols) {
                const long long ix = l == 0 ? x0 : x1;
                INT_TRY(cudaMemcpy2DAsync(d, sizeof(float2), src[comp] + ix, nx * sizeof(float2), sizeof(float2), nz,
                                          cudaMemcpyHostToDevice, st));
            } else {
                const long long iz = l == 0 ? z0 : z1;
                INT_TRY(cudaMemcpyAsync(d, src[comp] + iz * nx, nx * sizeof(float2), cudaMemcpyHostToDevice, st));
            }
        }
    }
    const double a1 = dep == 0 ? ax : 0., a2 = dep == 0 ? az : (cols ? ax : az);
    cut_kernel<<<(nOut + 255) / 256, 256, 0, st>>>(dX, dZ, (int)nLine, nOut, dep, (int)x0, (int)x1, a1, a2, (int)pol,
                                                   what, what == 2 ? nullptr : (float*)dOut,
                                                   what == 2 ? (double*)dOut : nullptr);
    INT_TRY(cudaGetLastError());
    INT_TRY(cudaMemcpyAsync(pInt, dOut, (size_t)np * nOut * esz, cudaMemcpyDeviceToHost, st));
    INT_TRY(cudaStreamSynchronize(st));
    return 0;
}

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
    if (depType < 0 || depType > 3) {
        set_last_detail("intensity extraction vs x and y (depType 3), x (1), y (2) or at one point (0) only");
        return SRWG_ERR_UNSUPPORTED;
    }
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
    if (depType != 3) return int_cut(c, pInt, pWfr, pol, what, depType, x, y);
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
