// Host helpers shared by the entry points (capi.cpp, noalloc.cu).
#pragma once
#include <map>
#include <mutex>
#include <string>
#include <vector>
#include "kernels.h"

namespace srwg {
// per-device state of the library (capi.cpp)
struct DeviceCtx {
    int dev = 0;
    std::map<int, float2*> tw;          // twiddle tables by FFT length
    float2* work = nullptr;             // 2 work buffers x 2 components
    size_t workElems = 0;               // per buffer per component
    float2* io = nullptr;               // input + output staging for the host-memory entry point
    size_t ioElems = 0;
    float2* tab = nullptr;              // point-wise tables of the one-shot entry point
    size_t tabElems = 0;
    double* mom = nullptr;              // moment passes of the one-shot entry point: slots | scratch
    size_t momDoubles = 0;
    float2* stg[2] = {nullptr, nullptr};  // stage outputs of a staged propagation (2 components each)
    void* intBuf = nullptr;             // intensity extraction: both components and the result
    size_t intBytes = 0;
    void* genBuf = nullptr;             // field generation: both components, tables, moment scratch
    size_t genBytes = 0;
    size_t stgElems[2] = {0, 0};
    cudaStream_t stream = nullptr;
    int* status = nullptr;              // device counter of bounded waits that gave up (kernels add to it)
};
long long wait_limit();                               // iteration limit of the kernels' bounded waits (0: default)
std::mutex& library_mutex();                          // serialises the entry points
int device_ctx(int dev, DeviceCtx** out);             // makes `dev` current, returns its state
int device_twiddles(DeviceCtx& c, int N, const float2** out);
int execute_passes(const std::vector<KernelDesc>& ks, DeviceCtx& c, int nb, const float2* inX, const float2* inY,
                   long long inStride, float2* outX, float2* outY, long long outStride, float2* work, size_t workElems,
                   const char* dconst, long long constStride, size_t descOff, cudaStream_t st, cudaEvent_t* ev,
                   const std::vector<KernelDesc>* hostMax, double* momScratch = nullptr, double* momSlots = nullptr,
                   int nSlots = 0, char* intOut = nullptr);
int line_config(const LineDesc& d, LineLaunch& p);   // launch shape of a line pass (capi.cpp)
void line_window(const LineDesc& d, LineLaunch& p);  // only the window's line blocks (zskip row passes)
void resize_window(const ResizeDesc& r, ResizeLaunch& p);   // only the window's tiles (skip_zero)
int radix_plan(int N, int* r);
void set_last_detail(const std::string& s);          // detail text for srwlUtiGetErrText
const std::string& last_detail();
}  // namespace srwg
