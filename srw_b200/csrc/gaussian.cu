// srwlCalcElecFieldGaussian (cpp/src/lib/srwlib.cpp:544) on the GPU for a single photon energy:
// the electric field of a (Hermite-)Gaussian beam on the wavefront's mesh (srTGsnBeam,
// cpp/src/core/srgsnbm.cpp: constants :15-78 and :104-126, field :230-310, polarisation
// srgsnbm.h:74), the wavefront's radius, centre and 4x4 matrix (AuxSetupActionsArbSrc,
// srradstr.cpp:324-349; InitialSetupOf4x4PropMatr, srradstr.h:399) and its statistical moments
// (ComputeRadMoments: one MOM pass on the generated field).  Every point is independent: FP64
// phase, envelope and Hermite polynomials, rounded to FP32 at the store.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/srwl_b200.h"
#include "errors.h"
#include "exec.h"
#include "kernels.h"
#include "planner.h"

namespace srwg {

// per-wavefront constants of the frequency-domain field, FP64, in the reference's formulas
struct GsnParams {
    int nx, nz, mx, mz, polar;
    double xs0, zs0, xStep, zStep;        // x - x0Prop, z - z0Prop of index 0
    double xm0, zm0;                      // x - x0, z - z0 of index 0
    double x0, z0, dxds0, dzds0, L;
    double en, enMult, PropInvRx, PropInvRz, xpMult, zpMult, NuX, NuZ;
    double PropInvTwoSigXe2, PropInvTwoSigZe2, PropInvSigX, PropInvSigZ;
    int spec;                             // the average photon energy term is on
    double dPhotEn2InvTwoSig;             // dPhotEn^2 / (2 sigma_E^2)
    double amp;                           // field constant * sqrt(PropInvSigX PropInvSigZ)
};

// srTGsnBeam::HermitePolynomial (srgsnbm.cpp:97): H_n by the three-term recursion
__device__ __forceinline__ double hermite(int n, double x)
{
    if (n == 0) return 1.;
    double hm = 1., h = 2. * x;
    for (int k = 2; k <= n; k++) {
        const double hn = 2. * (x * h - (k - 1) * hm);
        hm = h;
        h = hn;
    }
    return h;
}

__global__ void __launch_bounds__(256) gaussian_kernel(const GsnParams g, float2* __restrict__ ex,
                                                       float2* __restrict__ ez)
{
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iz = blockIdx.y;
    if (ix >= g.nx) return;
    const double x = g.xs0 + ix * g.xStep, z = g.zs0 + iz * g.zStep;
    const double xmx0 = g.xm0 + ix * g.xStep, zmz0 = g.zm0 + iz * g.zStep;
    const double xx = xmx0 + g.x0, zz = zmz0 + g.z0;
    double Phase = g.en * g.enMult *
                       ((xmx0 * xmx0 + 2 * g.L * g.x0 * g.dxds0 + g.xpMult * (2 * xx - g.L * g.dxds0)) * g.PropInvRx +
                        (zmz0 * zmz0 + 2 * g.L * g.z0 * g.dzds0 + g.zpMult * (2 * zz - g.L * g.dzds0)) * g.PropInvRz) +
                   (g.mx + 0.5) * g.NuX + (g.mz + 0.5) * g.NuZ;
    const double TwoPI = 6.28318530717959, InvTwoPI = 1. / TwoPI;
    Phase -= TwoPI * (double)(long long)(Phase * InvTwoPI);
    double sn, cs;
    sincos(Phase, &sn, &cs);
    double arg = -(x * x) * g.PropInvTwoSigXe2 - (z * z) * g.PropInvTwoSigZe2;
    if (g.spec) arg -= g.dPhotEn2InvTwoSig;
    const double BufA = g.amp * exp(arg) * hermite(g.mx, x * g.PropInvSigX) * hermite(g.mz, z * g.PropInvSigZ);
    const double ReA = BufA * cs, ImA = BufA * sn;
    const double c = 0.70710678118655;
    float2 a, b;
    switch (g.polar) {
    case 1: a = make_float2((float)ReA, (float)ImA); b = make_float2(0.f, 0.f); break;
    case 2: a = make_float2(0.f, 0.f); b = make_float2((float)ReA, (float)ImA); break;
    case 3: a = make_float2((float)(c * ReA), (float)(c * ImA)); b = a; break;
    case 4: a = make_float2((float)(c * ReA), (float)(c * ImA)); b = make_float2((float)(-c * ReA), (float)(-c * ImA)); break;
    case 5: a = make_float2((float)(c * ReA), (float)(c * ImA)); b = make_float2((float)(-c * ImA), (float)(c * ReA)); break;
    default: a = make_float2((float)(c * ReA), (float)(c * ImA)); b = make_float2((float)(c * ImA), (float)(-c * ReA)); break;
    }
    const size_t o = (size_t)iz * g.nx + ix;
    ex[o] = a;
    ez[o] = b;
}

}  // namespace srwg

using namespace srwg;

#define GSN_TRY(x)                                                                      \
    do {                                                                                \
        cudaError_t e__ = (x);                                                          \
        if (e__ != cudaSuccess) {                                                       \
            set_last_detail(std::string(#x) + ": " + cudaGetErrorString(e__));          \
            return SRWG_ERR_CUDA;                                                       \
        }                                                                               \
    } while (0)

extern "C" SRWG_API int srwlCalcElecFieldGaussian(SRWLWfr* pWfr, SRWLGsnBm* pGsnBm, double* precPar)
{
    std::lock_guard<std::mutex> lk(library_mutex());
    set_last_detail("");
    if (pWfr == nullptr || pGsnBm == nullptr) return SRWL_INCORRECT_PARAM_FOR_GAUS_BEAM_COMP;
    if (precPar != nullptr && precPar[0] > 0.) {
        set_last_detail("automatic mesh sampling of the Gaussian beam (precPar[0] > 0)");
        return SRWG_ERR_UNSUPPORTED;
    }
    const SRWLRadMesh& m = pWfr->mesh;
    if (m.ne != 1 || pWfr->presFT != 0) { set_last_detail("Gaussian beam at a single photon energy only"); return SRWG_ERR_UNSUPPORTED; }
    if (m.nx < 2 || m.ny < 2) { set_last_detail("Gaussian beam on a 2D mesh only"); return SRWG_ERR_UNSUPPORTED; }
    if (pWfr->arEx == nullptr || pWfr->arEy == nullptr) return SRWL_INCORRECT_PARAM_FOR_GAUS_BEAM_COMP;
    if (m.eStart == 0.) return PHOT_EN_SHOULD_BE_POSITIVE;                // CheckInputConsistency
    const SRWLGsnBm& gb = *pGsnBm;
    // srTGsnBeam constructor (srgsnbm.cpp:15-78), spectral flux from the pulse energy
    const double Pi = 3.1415926535898, sqrt_2 = sqrt(2.);
    const double SigmaX = gb.sigX * sqrt_2, SigmaZ = gb.sigY * sqrt_2;
    const int mx = gb.mx, mz = gb.my;
    const double SigmaPhotEn = gb.sigT > 0 ? (0.5 * 6.58211889E-16 / gb.sigT) * sqrt_2 : 1.e+23;
    double PhotPerBW = -1.;
    if (gb.pulseEn > 0 && gb.sigT > 0) {
        PhotPerBW = 6.2415096E+15 * gb.pulseEn / (sqrt(Pi) * SigmaPhotEn);
        if (gb.repRate > 0) PhotPerBW *= gb.repRate;
    }
    double fact = 1.;
    for (int k = 2; k <= mx; k++) fact *= k;
    double factz = 1.;
    for (int k = 2; k <= mz; k++) factz *= k;
    const double AuxConst = double(1 << (mx + mz)) * fact * factz;
    double NormConst = sqrt(PhotPerBW / (AuxConst * ((1.E+06) * Pi)));
    if (pWfr->unitElFld == 2) NormConst *= sqrt(1.602176462e-16);
    // SetupSourceConstantsFreqDomain (srgsnbm.cpp:104-126)
    const double PhEnConv = 1.239842E-06;
    const double en = m.eStart;
    const double Robs = m.zStart - gb.z;
    double L = Robs;
    if (L == 0.) L = 0.01 * (PhEnConv / en);       // shifted off the waist to avoid the singularity
    const double InvTwoSigXe2 = 0.5 / (SigmaX * SigmaX), InvTwoSigZe2 = 0.5 / (SigmaZ * SigmaZ);
    const double InvTwoSigPhotEnE2 = 0.5 / (SigmaPhotEn * SigmaPhotEn);
    const double Buf = (Pi * 1.) / (PhEnConv * L);
    const double PropagMultX = Buf / InvTwoSigXe2, PropagMultZ = Buf / InvTwoSigZe2;
    const double x0Prop = gb.x + gb.xp * L, z0Prop = gb.y + gb.yp * L;
    GsnParams g;
    memset(&g, 0, sizeof(g));
    g.nx = (int)m.nx; g.nz = (int)m.ny; g.mx = mx; g.mz = mz; g.polar = gb.polar;
    g.xStep = (m.xFin - m.xStart) / (m.nx - 1);
    g.zStep = (m.yFin - m.yStart) / (m.ny - 1);
    g.xs0 = m.xStart - x0Prop; g.zs0 = m.yStart - z0Prop;
    g.xm0 = m.xStart - gb.x; g.zm0 = m.yStart - gb.y;
    g.x0 = gb.x; g.z0 = gb.y; g.dxds0 = gb.xp; g.dzds0 = gb.yp; g.L = L;
    g.en = en; g.enMult = 2.53384080189E+06;
    const double InvLongDist = 1. / L;
    const double PropRatX = en * PropagMultX, PropRatZ = en * PropagMultZ;
    const double InvPropRatX = 1. / PropRatX, InvPropRatZ = 1. / PropRatZ;
    const double SigMultX = 1. + InvPropRatX * InvPropRatX, SigMultZ = 1. + InvPropRatZ * InvPropRatZ;
    const double DisMultX = 1. + PropRatX * PropRatX, DisMultZ = 1. + PropRatZ * PropRatZ;
    g.PropInvTwoSigXe2 = InvTwoSigXe2 / SigMultX; g.PropInvTwoSigZe2 = InvTwoSigZe2 / SigMultZ;
    g.PropInvSigX = sqrt(2. * g.PropInvTwoSigXe2); g.PropInvSigZ = sqrt(2. * g.PropInvTwoSigZe2);
    g.PropInvRx = InvLongDist / DisMultX; g.PropInvRz = InvLongDist / DisMultZ;
    g.xpMult = (1. / g.PropInvRx - L) * gb.xp; g.zpMult = (1. / g.PropInvRz - L) * gb.yp;
    g.NuX = atan(InvPropRatX); g.NuZ = atan(InvPropRatZ);
    g.spec = gb.avgPhotEn > 0 ? 1 : 0;
    const double dPhotEn = en - gb.avgPhotEn;
    g.dPhotEn2InvTwoSig = dPhotEn * dPhotEn * InvTwoSigPhotEnE2;
    g.amp = NormConst * sqrt(g.PropInvSigX * g.PropInvSigZ);

    // the wavefront: radius and centre at the observation plane (AuxSetupActionsArbSrc)
    WfrState w;
    w.nx = (int)m.nx; w.nz = (int)m.ny; w.eStart = en;
    w.xStart = m.xStart; w.xStep = g.xStep; w.zStart = m.yStart; w.zStep = g.zStep;
    w.RobsX = w.RobsZ = Robs;
    w.RobsXAbsErr = w.RobsZAbsErr = 0.01 * ::fabs(Robs);
    w.xc = gb.x; w.zc = gb.y;
    KernelDesc kd;
    MomOp op;
    std::vector<float2> tabs;
    single_moment_pass(w, kd, op, tabs);

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    DeviceCtx* c = nullptr;
    int r = device_ctx(dev, &c);
    if (r) return r;
    const size_t n = (size_t)m.nx * m.ny;
    const size_t tabBytes = ((tabs.size() * sizeof(float2) + 255) / 256) * 256;
    const size_t scr = mom_scratch_doubles(w.nx, w.nz);
    const size_t bytes = 2 * n * sizeof(float2) + tabBytes + 256 + sizeof(KernelDesc) + (SRWG_MOM_SLOT + scr) * sizeof(double) + 256;
    if (c->genBuf == nullptr || c->genBytes < bytes) {
        if (c->genBuf) cudaFree(c->genBuf);
        c->genBuf = nullptr; c->genBytes = 0;
        GSN_TRY(cudaMalloc(&c->genBuf, bytes));
        c->genBytes = bytes;
    }
    char* base = (char*)c->genBuf;
    float2* dX = (float2*)base;
    float2* dZ = dX + n;
    float2* dTab = (float2*)(base + 2 * n * sizeof(float2));
    KernelDesc* dDesc = (KernelDesc*)((char*)dTab + tabBytes);
    double* dMom = (double*)(((uintptr_t)((char*)dDesc + sizeof(KernelDesc)) + 255) & ~(uintptr_t)255);
    cudaStream_t st = c->stream;
    if (!tabs.empty()) GSN_TRY(cudaMemcpyAsync(dTab, tabs.data(), tabs.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
    GSN_TRY(cudaMemcpyAsync(dDesc, &kd, sizeof(KernelDesc), cudaMemcpyHostToDevice, st));
    dim3 grid((unsigned)((m.nx + 255) / 256), (unsigned)m.ny);
    gaussian_kernel<<<grid, 256, 0, st>>>(g, dX, dZ);
    GSN_TRY(cudaGetLastError());
    MomLaunch ml;
    memset(&ml, 0, sizeof(ml));
    ml.d = kd.mom;
    ml.src[0] = dX; ml.src[1] = dZ;
    ml.tabs = dTab;
    ml.gd = &dDesc->mom;
    ml.scratch = dMom + SRWG_MOM_SLOT;
    ml.out = dMom;
    ml.nb = 1;
    GSN_TRY(launch_moments(ml, st));
    double S[SRWG_MOM_SLOT];
    GSN_TRY(cudaMemcpyAsync(pWfr->arEx, dX, n * sizeof(float2), cudaMemcpyDeviceToHost, st));
    GSN_TRY(cudaMemcpyAsync(pWfr->arEy, dZ, n * sizeof(float2), cudaMemcpyDeviceToHost, st));
    GSN_TRY(cudaMemcpyAsync(S, dMom, sizeof(S), cudaMemcpyDeviceToHost, st));
    GSN_TRY(cudaStreamSynchronize(st));
    // outputs as OutSRWRadPtrs writes them
    pWfr->Rx = pWfr->Ry = Robs;
    pWfr->dRx = pWfr->dRy = 0.01 * ::fabs(Robs);
    pWfr->xc = gb.x; pWfr->yc = gb.y;
    pWfr->presCA = 0;
    pWfr->avgPhotEn = en;
    double mx_[11], mz_[11];
    moments_from_sums(S, op, mx_, mz_);
    if (pWfr->arMomX) for (int i = 0; i < 11; i++) pWfr->arMomX[i] = mx_[i];
    if (pWfr->arMomY) for (int i = 0; i < 11; i++) pWfr->arMomY[i] = mz_[i];
    if (pWfr->arElecPropMatr) {          // InitialSetupOf4x4PropMatr: drift from the beam's s0
        double* p = pWfr->arElecPropMatr;
        for (int i = 0; i < 16; i++) p[i] = 0.;
        for (int i = 0; i < 4; i++) p[5 * i] = 1.;
        p[1] = p[11] = m.zStart - pWfr->partBeam.partStatMom1.z;
    }
    return 0;
}
