// Allocation-free entry point: srwgPropagElecFieldStatic.
//
// Some callers cannot call cudaMalloc at run time: applications that reserve all device memory
// up front and hand out slices themselves, processes whose memory must go through a caching
// allocator that has to see every allocation (such as PyTorch's), or codes whose memory budget is
// fixed once at start-up.  For them this entry point runs a whole propagation with no device
// allocation of its own: the caller passes the input and output fields, and the intermediate
// fields, point-wise tables, pass descriptors and FFT twiddles live in one file-scope device
// array of fixed size (below), which every GPU that loads the library holds until the process
// exits.
//
// Limits: the largest intermediate grid of the planned passes may hold at most
// SRWG_STATIC_WORK_POINTS complex points (512 x 512), and the plan's constant data at most
// SRWG_STATIC_CONST_POINTS float2 (1 MiB), and the moment passes (result slots and scratch) at
// most SRWG_STATIC_MOM_DOUBLES doubles (2 MiB); larger propagations are rejected with
// SRWG_ERR_STATIC_LIMIT and a message giving the sizes.
//
// Where the propagation recomputes the statistical moments from the field (an aperture that clips
// the beam, an obstacle) and pWfrOut has moment arrays, the call waits for the stream to finish
// and reads the passes' result slots back; otherwise it returns without waiting.
//
// All calls share the array and it keeps the last call's contents.  Nothing has to start at
// zero: every point a pass reads was written earlier in the same call (a resize that leaves the
// points outside its window unwritten is followed by a pass that treats them as zero without
// reading them).  Calls
// that overlap on the GPU (issued on different streams with no ordering between them) race on
// the array; issue them on one stream, or order them with events.
//
// The first call on a device does the set-up: it looks up the array's device address with
// cudaGetSymbolAddress, with that device current, and keeps it for the following calls on that
// device.  Make that first call before any stream capture.
//
// Every call copies the plan's tables and pass descriptors from host memory into the array (and
// may wait for the stream, above); a call whose stream is being captured is refused with
// SRWG_ERR_BAD_ARG before anything is queued.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/srwl_b200.h"
#include "errors.h"
#include "exec.h"
#include "kernels.h"
#include "planner.h"

#define SRWG_STATIC_WORK_POINTS (512 * 512)
#define SRWG_STATIC_CONST_POINTS (128 * 1024)
#define SRWG_STATIC_MOM_DOUBLES (256 * 1024)
#define SRWG_STATIC_POINTS (4 * SRWG_STATIC_WORK_POINTS + SRWG_STATIC_CONST_POINTS + SRWG_STATIC_MOM_DOUBLES)

namespace srwg {

// [ work buffer A: Ex, Ey | work buffer B: Ex, Ey | constant data | moment slots and scratch ]  (11 MiB)
static __device__ __align__(256) float2 g_static_scratch[SRWG_STATIC_POINTS];

static std::mutex g_static_mutex;
static std::map<int, float2*> g_static_addr;   // device -> address of g_static_scratch

static int static_scratch(int dev, float2** out)
{
    auto it = g_static_addr.find(dev);
    if (it != g_static_addr.end()) { *out = it->second; return 0; }
    float2* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_static_scratch);
    if (e != cudaSuccess || p == nullptr) {
        set_last_detail(std::string("cudaGetSymbolAddress of the static scratch array: ") + cudaGetErrorString(e));
        return SRWG_ERR_CUDA;
    }
    g_static_addr[dev] = p;
    *out = p;
    return 0;
}

}  // namespace srwg

using namespace srwg;

extern "C" SRWG_API int srwgPropagElecFieldStatic(const SRWLWfr* pWfr, const SRWLOptC* pOpt, const float* dExIn,
                                                  const float* dEyIn, float* dExOut, float* dEyOut,
                                                  long long outCapacity, void* stream, SRWLWfr* pWfrOut)
{
    std::lock_guard<std::mutex> lk(g_static_mutex);
    set_last_detail("");
    if (pWfr == nullptr || pOpt == nullptr || dExIn == nullptr || dEyIn == nullptr || dExOut == nullptr ||
        dEyOut == nullptr)
        return SRWG_ERR_BAD_ARG;
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        const cudaError_t ce = cudaStreamIsCapturing((cudaStream_t)stream, &cs);
        if (ce != cudaSuccess) {
            set_last_detail(std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(ce));
            return SRWG_ERR_CUDA;
        }
        if (cs != cudaStreamCaptureStatusNone) {
            set_last_detail("the stream is being captured: this entry point copies the plan's tables from host memory "
                            "on every call, which a stream capture does not take");
            return SRWG_ERR_BAD_ARG;
        }
    }
    Planner pl;
    int r = pl.plan(pWfr, pOpt);
    if (r) { set_last_detail(pl.err); return r; }
    if (pl.maxElems > SRWG_STATIC_WORK_POINTS) {
        set_last_detail("an intermediate grid of " + std::to_string(pl.maxElems) + " points exceeds the static limit of " +
                        std::to_string(SRWG_STATIC_WORK_POINTS) + " points (512 x 512)");
        return SRWG_ERR_STATIC_LIMIT;
    }
    const long long nOut = (long long)pl.w.nx * pl.w.nz;
    if (nOut > outCapacity) {
        set_last_detail("output arrays hold " + std::to_string(outCapacity) + " points, the result has " +
                        std::to_string(nOut));
        return SRWG_ERR_BAD_ARG;
    }
    // constant data: tables | (256-byte aligned) pass descriptors | twiddle tables per line length
    std::vector<float2> cst(pl.tables);
    while ((cst.size() * sizeof(float2)) % 256) cst.push_back(float2{0.f, 0.f});
    const size_t descOff = cst.size();
    const size_t descPts = (pl.kernels.size() * sizeof(KernelDesc) + sizeof(float2) - 1) / sizeof(float2);
    cst.resize(descOff + descPts);
    memcpy(&cst[descOff], pl.kernels.data(), pl.kernels.size() * sizeof(KernelDesc));
    std::map<int, size_t> twOff;
    for (const KernelDesc& k : pl.kernels) {
        if (k.kind != K_LINE) continue;
        int N = k.line.axis == 0 ? k.line.nx : k.line.nz;
        if (twOff.count(N)) continue;
        while ((cst.size() * sizeof(float2)) % 256) cst.push_back(float2{0.f, 0.f});
        twOff[N] = cst.size();
        for (int i = 0; i < N; i++) {
            double a = -2. * M_PI * (double)i / (double)N;
            cst.push_back(float2{(float)cos(a), (float)sin(a)});
        }
    }
    if (cst.size() > SRWG_STATIC_CONST_POINTS) {
        set_last_detail("the plan's tables need " + std::to_string(cst.size()) + " points, above the static limit of " +
                        std::to_string(SRWG_STATIC_CONST_POINTS));
        return SRWG_ERR_STATIC_LIMIT;
    }
    const size_t nSlotD = (size_t)pl.nMomSlots * SRWG_MOM_SLOT;
    size_t momNeed = 0;
    for (const KernelDesc& k : pl.kernels)
        if (k.kind == K_MOM) momNeed = std::max(momNeed, mom_scratch_doubles(k.mom.nx, k.mom.nz));
    if (nSlotD + momNeed > SRWG_STATIC_MOM_DOUBLES) {
        set_last_detail("the moment passes need " + std::to_string(nSlotD + momNeed) + " doubles, above the static limit of " +
                        std::to_string(SRWG_STATIC_MOM_DOUBLES));
        return SRWG_ERR_STATIC_LIMIT;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { set_last_detail("cudaGetDevice failed"); return SRWG_ERR_NO_DEVICE; }
    float2* base = nullptr;
    r = static_scratch(dev, &base);
    if (r) return r;
    cudaStream_t st = (cudaStream_t)stream;
    float2* work = base;
    float2* cdev = base + 4 * (size_t)SRWG_STATIC_WORK_POINTS;
    double* mom = (double*)(cdev + SRWG_STATIC_CONST_POINTS);     // slots | scratch
    cudaError_t e = cudaMemcpyAsync(cdev, cst.data(), cst.size() * sizeof(float2), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) { set_last_detail(std::string("constant upload: ") + cudaGetErrorString(e)); return SRWG_ERR_CUDA; }
    const KernelDesc* gk = (const KernelDesc*)(cdev + descOff);
    const float2* inX = (const float2*)dExIn;
    const float2* inY = (const float2*)dEyIn;
    float2* outX = (float2*)dExOut;
    float2* outY = (float2*)dEyOut;
    const size_t W = SRWG_STATIC_WORK_POINTS;
    float2* wb[3][2] = {{nullptr, nullptr}, {work, work + W}, {work + 2 * W, work + 3 * W}};
    const size_t nk = pl.kernels.size();
    if (nk == 0) {
        e = cudaMemcpyAsync(outX, inX, nOut * sizeof(float2), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(outY, inY, nOut * sizeof(float2), cudaMemcpyDeviceToDevice, st);
    }
    // the last pass that writes a field writes the output; moment passes after it read the output
    size_t lastField = nk;
    for (size_t i = nk; i-- > 0;)
        if (pl.kernels[i].kind != K_MOM) { lastField = i; break; }
    if (nk > 0 && lastField == nk) { set_last_detail("plan without field passes"); return SRWG_ERR_BAD_ARG; }
    for (size_t i = 0; i < nk && e == cudaSuccess; i++) {
        const KernelDesc& k = pl.kernels[i];
        const bool fromOut = k.kind == K_MOM && k.src != 0 && i > lastField && k.src == pl.kernels[lastField].dst;
        const float2* s0 = fromOut ? outX : k.src == 0 ? inX : wb[k.src][0];
        const float2* s1 = fromOut ? outY : k.src == 0 ? inY : wb[k.src][1];
        float2* d0 = (i == lastField) ? outX : wb[k.dst][0];
        float2* d1 = (i == lastField) ? outY : wb[k.dst][1];
        if (k.kind == K_MOM) {
            MomLaunch p;
            memset(&p, 0, sizeof(p));
            p.d = k.mom;
            p.src[0] = s0; p.src[1] = s1;
            p.tabs = cdev;
            p.gd = &gk[i].mom;
            p.scratch = mom + nSlotD;
            p.out = mom + (size_t)k.mom.slot * SRWG_MOM_SLOT;
            p.nb = 1;
            e = launch_moments(p, st);
        } else if (k.kind == K_LINE) {
            LineLaunch p;
            memset(&p, 0, sizeof(p));
            r = line_config(k.line, p);
            if (r) return r;
            p.tw = cdev + twOff[p.N];
            p.src[0] = s0; p.src[1] = s1; p.dst[0] = d0; p.dst[1] = d1;
            p.tabs = cdev;
            p.gd = &gk[i].line;
            e = launch_line(p, st);
        } else if (k.kind == K_RESIZE) {
            ResizeLaunch p;
            memset(&p, 0, sizeof(p));
            p.d = k.rs;
            p.src[0] = s0; p.src[1] = s1; p.dst[0] = d0; p.dst[1] = d1;
            p.xStepInvO = 1. / k.rs.xStepO;
            p.zStepInvO = 1. / k.rs.zStepO;
            p.tabs = cdev;
            p.gd = &gk[i].rs;
            e = launch_resize(p, st);
        } else {
            PwLaunch p;
            memset(&p, 0, sizeof(p));
            p.d = k.pwk;
            p.src[0] = s0; p.src[1] = s1; p.dst[0] = d0; p.dst[1] = d1;
            p.tabs = cdev;
            p.gd = &gk[i].pwk;
            e = launch_pw(p, st);
        }
    }
    if (e != cudaSuccess) { set_last_detail(std::string("launch: ") + cudaGetErrorString(e)); return SRWG_ERR_CUDA; }
    if (pWfrOut) {
        // output mesh and scalars as srwgPlanGetOutput writes them
        const WfrState& w = pl.w;
        pWfrOut->mesh.eStart = w.eStart; pWfrOut->mesh.eFin = w.eStart;
        pWfrOut->mesh.xStart = w.xStart; pWfrOut->mesh.xFin = w.xStart + w.xStep * (w.nx - 1);
        pWfrOut->mesh.yStart = w.zStart; pWfrOut->mesh.yFin = w.zStart + w.zStep * (w.nz - 1);
        pWfrOut->mesh.ne = 1; pWfrOut->mesh.nx = w.nx; pWfrOut->mesh.ny = w.nz;
        pWfrOut->Rx = w.RobsX; pWfrOut->Ry = w.RobsZ; pWfrOut->dRx = w.RobsXAbsErr; pWfrOut->dRy = w.RobsZAbsErr;
        pWfrOut->xc = w.xc; pWfrOut->yc = w.zc; pWfrOut->presCA = (char)w.Pres; pWfrOut->avgPhotEn = w.avgPhotEn;
        if (pWfrOut->arElecPropMatr != nullptr && w.havePropM)
            for (int m = 0; m < 20; m++) pWfrOut->arElecPropMatr[m] = w.propM[m];
        double mx[11], mz[11];
        for (int m = 0; m < 11; m++) { mx[m] = w.momX[m]; mz[m] = w.momZ[m]; }
        if (nSlotD && (pWfrOut->arMomX || pWfrOut->arMomY)) {
            // moments recomputed from the field: wait for the passes and read their result slots
            std::vector<double> hs(nSlotD);
            e = cudaStreamSynchronize(st);
            if (e == cudaSuccess) e = cudaMemcpy(hs.data(), mom, nSlotD * sizeof(double), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) { set_last_detail(std::string("moment read-back: ") + cudaGetErrorString(e)); return SRWG_ERR_CUDA; }
            pl.replay_moments(hs.data(), mx, mz);
        }
        if (pWfrOut->arMomX) for (int m = 0; m < 11; m++) pWfrOut->arMomX[m] = mx[m];
        if (pWfrOut->arMomY) for (int m = 0; m < 11; m++) pWfrOut->arMomY[m] = mz[m];
    }
    return 0;
}
