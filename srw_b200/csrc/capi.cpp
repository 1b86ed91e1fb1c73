// C-ABI of the library: the reference's srwlPropagElecField / srwlUtiSetWfrModifFunc /
// srwlUtiSetAllocArrayFunc / srwlUtiGetErrText (cpp/src/lib/srwlib.h:542, 549, 574, 821) and the srwgPlan* extensions, plus the
// executor that runs a plan's passes on a CUDA stream.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/srwl_b200.h"
#include "errors.h"
#include "kernels.h"
#include "exec.h"
#include "planner.h"

namespace srwg {

static std::string g_lastDetail;                          // detail text of the last error
void set_last_detail(const std::string& s) { g_lastDetail = s; }
const std::string& last_detail() { return g_lastDetail; }
static int (*g_modifFunc)(int, SRWLWfr*, char) = nullptr;  // client re-allocation callback
static char* (*g_allocArrayFunc)(char, long long) = nullptr; // client array allocation (extracted intensities)
static std::mutex g_mutex;
std::mutex& library_mutex() { return g_mutex; }

static std::map<int, DeviceCtx*> g_ctx;
static long long g_waitLimit = 0;                           // 0: the kernels' own default
long long wait_limit() { return g_waitLimit; }

#define CUDA_TRY(x)                                                                     \
    do {                                                                                \
        cudaError_t e__ = (x);                                                          \
        if (e__ != cudaSuccess) {                                                       \
            g_lastDetail = std::string(#x) + ": " + cudaGetErrorString(e__);            \
            return SRWG_ERR_CUDA;                                                       \
        }                                                                               \
    } while (0)

int device_ctx(int dev, DeviceCtx** out)
{
    auto it = g_ctx.find(dev);
    if (it != g_ctx.end()) {
        CUDA_TRY(cudaSetDevice(dev));
        *out = it->second;
        return 0;
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        g_lastDetail = "no CUDA device available";
        return SRWG_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= n) {
        g_lastDetail = "device index out of range";
        return SRWG_ERR_NO_DEVICE;
    }
    CUDA_TRY(cudaSetDevice(dev));
    DeviceCtx* c = new DeviceCtx();
    c->dev = dev;
    CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaMalloc(&c->status, sizeof(int)));
    CUDA_TRY(cudaMemset(c->status, 0, sizeof(int)));
    g_ctx[dev] = c;
    *out = c;
    return 0;
}

// exp(-2 pi i k/N) in FP64, rounded to FP32
int device_twiddles(DeviceCtx& c, int N, const float2** out)
{
    auto it = c.tw.find(N);
    if (it != c.tw.end()) { *out = it->second; return 0; }
    std::vector<float2> h(N);
    for (int k = 0; k < N; k++) {
        double a = -2. * M_PI * (double)k / (double)N;
        h[k] = make_float2((float)cos(a), (float)sin(a));
    }
    float2* d = nullptr;
    CUDA_TRY(cudaMalloc(&d, sizeof(float2) * N));
    CUDA_TRY(cudaMemcpy(d, h.data(), sizeof(float2) * N, cudaMemcpyHostToDevice));
    c.tw[N] = d;
    *out = d;
    return 0;
}

// radix schedule of an even N: power-of-two part in radix-16/8 stages (4/8-bit splits), then 3, 5, 7, 11, 13
int radix_plan(int N, int* r)
{
    int n = N, p2 = 0, ns = 0;
    while (n % 2 == 0) { n /= 2; p2++; }
    int odd[32], no = 0;
    const int primes[5] = {3, 5, 7, 11, 13};
    for (int i = 0; i < 5; i++)
        while (n % primes[i] == 0) { odd[no++] = primes[i]; n /= primes[i]; }
    if (n != 1) return -1;
    int bits[16], nb = 0;
    while (p2 >= 4 && p2 != 5) {
        if (p2 == 6) { bits[nb++] = 3; bits[nb++] = 3; p2 = 0; break; }
        bits[nb++] = 4;
        p2 -= 4;
    }
    if (p2 == 5) { bits[nb++] = 3; bits[nb++] = 2; p2 = 0; }
    else if (p2 >= 1 && p2 <= 3) { bits[nb++] = p2; p2 = 0; }
    for (int i = 0; i < nb; i++) r[ns++] = 1 << bits[i];
    for (int i = 0; i < no; i++) r[ns++] = odd[i];
    if (ns > SRWG_MAX_STAGES) return -1;
    return ns;
}

// ------------------------------------------------------------------------------------------------
// autotuned launch shapes: kernel family and lines per CTA of the compile-time-length line kernels
// per (axis, N), measured by srw_b200.tune and stored as lines "rows|cols N L [spec]" in
// models/line_tuning.txt next to the library (or the file named by SRWG_TUNING); "spec" selects the
// specialised kernel for a power of two.  srwgTuneSetLines / srwgTuneSetFamily change entries at
// run time.
// ------------------------------------------------------------------------------------------------
static std::mutex g_tuneMutex;
struct TuneEntry {
    int fam = 0;       // 0: the default family of the length
    int lines = 0;     // 0: the family's default lines per CTA
};
static std::map<std::pair<int, int>, TuneEntry> g_tune;
static bool g_tuneLoaded = false;

static int default_family(int N)
{
    return line2_supported(N) ? FAM_POW2 : linen_supported(N) ? FAM_SPEC : 0;
}

static int tune_load_file(const char* path, int* nOut)
{
    FILE* f = fopen(path, "r");
    if (!f) return -1;
    char line[256];
    int n = 0;
    while (fgets(line, sizeof(line), f)) {
        char ax[16], fam[16] = {0};
        int N = 0, L = 0;
        if (line[0] == '#') continue;
        const int got = sscanf(line, "%15s %d %d %15s", ax, &N, &L, fam);
        if (got < 3) continue;
        const int axis = strcmp(ax, "rows") == 0 ? 0 : strcmp(ax, "cols") == 0 ? 1 : -1;
        const int f = (got == 4 && strcmp(fam, "spec") == 0) ? FAM_SPEC : default_family(N);
        if (axis < 0 || !fixed_lines_valid(axis, N, L, f)) continue;
        TuneEntry e;
        e.fam = f;
        e.lines = L;
        g_tune[std::make_pair(axis, N)] = e;
        n++;
    }
    fclose(f);
    if (nOut) *nOut = n;
    return 0;
}

static void tune_ensure_loaded()
{
    if (g_tuneLoaded) return;
    g_tuneLoaded = true;
    const char* env = getenv("SRWG_TUNING");
    if (env != nullptr) {
        if (*env) tune_load_file(env, nullptr);           // SRWG_TUNING="" : defaults only
        return;
    }
    Dl_info info;
    if (dladdr((void*)&tune_load_file, &info) && info.dli_fname) {
        std::string so(info.dli_fname);
        const size_t cut = so.find_last_of('/');
        const std::string dir = cut == std::string::npos ? std::string(".") : so.substr(0, cut);
        tune_load_file((dir + "/../models/line_tuning.txt").c_str(), nullptr);
    }
}

static TuneEntry tuned(int axis, int N)
{
    std::lock_guard<std::mutex> lk(g_tuneMutex);
    tune_ensure_loaded();
    auto it = g_tune.find(std::make_pair(axis, N));
    return it != g_tune.end() ? it->second : TuneEntry();
}

int fixed_family(int axis, int N)
{
    const TuneEntry e = tuned(axis, N);
    return e.fam ? e.fam : default_family(N);
}

int fixed_lines_per_cta(int axis, int N)
{
    const int fam = fixed_family(axis, N);
    if (fam != FAM_POW2 && fam != FAM_SPEC) return 0;
    const TuneEntry e = tuned(axis, N);
    if (e.lines > 0 && fixed_lines_valid(axis, N, e.lines, fam)) return e.lines;
    return fam == FAM_POW2 ? line2_lines_per_cta(axis, N) : linen_lines_per_cta(axis, N);
}

int line_config(const LineDesc& d, LineLaunch& p)
{
    p.d = d;
    int N = d.axis == 0 ? d.nx : d.nz;
    p.N = N;
    p.nlines = d.axis == 0 ? d.nz : d.nx;
    const size_t cap = SRWG_LINE_SMEM_MAX;
    const int fam = fixed_family(d.axis, N);
    if (fam == FAM_POW2) {
        // power of two: 16 points per thread, radix-16 stages then a 16/8/4/2 stage
        p.v2 = 1;
        p.T = N / 16;
        int nb = 0;
        while ((1 << nb) < N) nb++;
        p.nst = 0;
        while (nb > 4 && nb - 4 >= 1) {
            if (nb - 4 < 1) break;
            p.radix[p.nst++] = 16;
            nb -= 4;
        }
        p.radix[p.nst++] = 1 << nb;          // 16, 8, 4 or 2
        const int L = fixed_lines_per_cta(d.axis, N);
        p.P = (int)line_pitch(N, L, d.axis == 1);
        if (p.T * L > 1024) { g_lastDetail = "line pass too large"; return SRWG_ERR_UNSUPPORTED; }
        p.L = L;
        p.G = L;
        if ((size_t)p.L * p.P * sizeof(float2) > cap) { g_lastDetail = "line too long for shared memory"; return SRWG_ERR_UNSUPPORTED; }
        return 0;
    }
    // general length (or a power of two the tuner gave it) with a specialised kernel (linen.cuh):
    // compile-time schedule, T = ceil(N/16)
    if (fam == FAM_SPEC) {
        p.v2 = 3;
        p.T = (N + 15) / 16;
        p.L = fixed_lines_per_cta(d.axis, N);
        p.P = (int)line_pitch(N, p.L, d.axis == 1);
        p.G = p.L;
        p.nst = 0;
        if (p.T * p.L > 512 || (size_t)p.L * p.P * sizeof(float2) > cap) {
            g_lastDetail = "line too long for shared memory";
            return SRWG_ERR_UNSUPPORTED;
        }
        return 0;
    }
    // general good number with radices 16/8/4/2, 3, 5, 7 and at least two stages: the fused pass of
    // lineg.cuh (T >= N/16 threads per line, rows ~256 threads, columns up to 512 threads per CTA)
    {
        int rad[SRWG_MAX_STAGES];
        const int ns = radix_plan(N, rad);
        bool gen = ns >= 2 && N <= 8192;
        for (int i = 0; i < ns && gen; i++) gen = rad[i] != 11 && rad[i] != 13;
        if (gen) {
            p.v2 = 2;
            int T = (N + 15) / 16;
            T = ((T + 31) / 32) * 32;
            p.T = T;
            int L = d.axis == 0 ? 256 / T : 512 / T;
            if (L < 1) L = 1;
            while (L > 1 && (size_t)L * line_pitch(N, L, d.axis == 1) * sizeof(float2) > cap) L--;
            p.P = (int)line_pitch(N, L, d.axis == 1);
            if (T * L > 512 || (size_t)L * p.P * sizeof(float2) > cap) {
                g_lastDetail = "line too long for shared memory";
                return SRWG_ERR_UNSUPPORTED;
            }
            p.L = L;
            p.G = L;
            p.nst = ns;
            for (int i = 0; i < ns; i++) p.radix[i] = rad[i];
            return 0;
        }
    }
    p.v2 = 0;
    // general good number: T threads per line, at most 16 points each; G = threads per CTA / T
    // groups work on the CTA's L lines in batches
    int T = (N + 15) / 16;
    T = ((T + 31) / 32) * 32;
    if (T < 32) T = 32;
    if (T > 512) { g_lastDetail = "FFT length above 8192"; return SRWG_ERR_UNSUPPORTED; }
    p.T = T;
    int L;
    if (d.axis == 0) {
        L = 256 / T > 1 ? 256 / T : 1;          // rows: ~256 threads, one batch
        p.P = N;
    } else {
        L = 512 / T > 4 ? 512 / T : 4;          // columns: >= 4 per tile (32-byte row segments)
        p.P = N + 1;
    }
    while (L > 1 && (size_t)L * p.P * sizeof(float2) > cap) L--;
    p.L = L;
    if ((size_t)p.L * p.P * sizeof(float2) > cap) { g_lastDetail = "line too long for shared memory"; return SRWG_ERR_UNSUPPORTED; }
    int G = 512 / T;
    if (G > L) G = L;
    if (G < 1) G = 1;
    p.G = G;
    p.nst = radix_plan(N, p.radix);
    if (p.nst < 0) { g_lastDetail = "FFT length is not 2^a 3^b 5^c 7^d 11^e 13^f"; return SRWG_ERR_UNSUPPORTED; }
    return 0;
}

// device copy of a plan's constant data: its point-wise tables, then (256-byte aligned) its pass
// descriptors; returns the byte offset of the descriptors
static size_t const_bytes(const Planner& pl, size_t* descOff)
{
    size_t tb = pl.tables.size() * sizeof(float2);
    size_t off = (tb + 255) & ~(size_t)255;
    *descOff = off;
    return off + pl.kernels.size() * sizeof(KernelDesc);
}

static int upload_tables(const Planner& pl, float2** buf, size_t* capElems, cudaStream_t st)
{
    size_t descOff;
    size_t bytes = const_bytes(pl, &descOff);
    size_t n = (bytes + sizeof(float2) - 1) / sizeof(float2);
    if (*capElems < n || *buf == nullptr) {
        if (*buf) cudaFree(*buf);
        *buf = nullptr;
        *capElems = 0;
        CUDA_TRY(cudaMalloc(buf, n * sizeof(float2)));
        *capElems = n;
    }
    if (!pl.tables.empty())
        CUDA_TRY(cudaMemcpyAsync(*buf, pl.tables.data(), pl.tables.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
    if (!pl.kernels.empty())
        CUDA_TRY(cudaMemcpyAsync((char*)*buf + descOff, pl.kernels.data(), pl.kernels.size() * sizeof(KernelDesc),
                                 cudaMemcpyHostToDevice, st));
    return 0;
}

// runs a pass list on nb wavefronts at once: buffer 0 = input (wavefront b at inX + b * inStride), 1/2 =
// work buffers (layout [buffer][component][wavefront][workElems]); the last pass writes the output
// (outX + b * outStride).  dconst holds per wavefront (stride constStride bytes) the tables and, at
// descOff, the pass descriptors; all wavefronts have passes of the same kinds and sizes.
// a row pass whose lines outside its window are zero and read by nothing (zskip) launches only the
// window's line blocks; `d` holds the window of the launch (for a batch: the union of its electrons')
void line_window(const LineDesc& d, LineLaunch& p)
{
    if (d.zwin && d.zskip && d.zl0 <= d.zl1 && p.L > 0) {
        const int l0 = std::max(0, d.zl0), l1 = std::min(p.nlines - 1, d.zl1);
        if (l0 <= l1) {
            p.blk0 = l0 / p.L;
            p.nblk = l1 / p.L - p.blk0 + 1;
        }
    }
}

// a tiled resize that writes only its window launches only the window's tiles
void resize_window(const ResizeDesc& r, ResizeLaunch& p)
{
    if (!r.skip_zero || r.tile_or <= 0) return;
    const long xs = std::max(0L, r.ixStart), xe = std::min((long)r.nxn - 1, r.ixEnd);
    const long zs = std::max(0L, r.izStart), ze = std::min((long)r.nzn - 1, r.izEnd);
    if (xs > xe || zs > ze) return;
    p.tx0 = (int)(xs / SRWG_RESIZE_TX);
    p.ntx = (int)(xe / SRWG_RESIZE_TX) - p.tx0 + 1;
    p.tz0 = (int)(zs / SRWG_RESIZE_TZ);
    p.ntz = (int)(ze / SRWG_RESIZE_TZ) - p.tz0 + 1;
}

int execute_passes(const std::vector<KernelDesc>& ks, DeviceCtx& c, int nb, const float2* inX, const float2* inY,
                   long long inStride, float2* outX, float2* outY, long long outStride, float2* work, size_t workElems,
                   const char* dconst, long long constStride, size_t descOff, cudaStream_t st, cudaEvent_t* ev,
                   const std::vector<KernelDesc>* hostMax, double* momScratch, double* momSlots, int nSlots,
                   char* intOut)
{
    const size_t nk = ks.size();
    const size_t W = (size_t)nb * workElems;
    float2* wb[3][2] = {{nullptr, nullptr}, {work, work + W}, {work + 2 * W, work + 3 * W}};
    const float2* tabs = (const float2*)dconst;
    const KernelDesc* gk = (const KernelDesc*)(dconst + descOff);
    const long long tabStride = constStride / (long long)sizeof(float2);
    // the last pass that writes a field writes the output; MOM passes after it read the output
    size_t lastField = nk;
    for (size_t i = nk; i-- > 0;)
        if (!reads_only(ks[i].kind)) { lastField = i; break; }

    for (size_t i = 0; i < nk; i++) {
        const KernelDesc& k = hostMax ? (*hostMax)[i] : ks[i];
        if (ev) CUDA_TRY(cudaEventRecord(ev[2 * i], st));
        const bool fromOut = reads_only(k.kind) && k.src != 0 && i > lastField && k.src == ks[lastField].dst;
        const bool fromIn = k.src == 0, toOut = i == lastField;
        const float2* s0 = fromOut ? outX : fromIn ? inX : wb[k.src][0];
        const float2* s1 = fromOut ? outY : fromIn ? inY : wb[k.src][1];
        float2* d0 = toOut ? outX : wb[k.dst][0];
        float2* d1 = toOut ? outY : wb[k.dst][1];
        const long long bSrc = fromOut ? outStride : fromIn ? inStride : (long long)workElems;
        const long long bDst = toOut ? outStride : (long long)workElems;
        cudaError_t e = cudaSuccess;
        if (k.kind == K_MOM) {
            if (momScratch == nullptr || momSlots == nullptr || k.mom.slot < 0 || k.mom.slot >= nSlots) {
                g_lastDetail = "moment pass without result buffers";
                return SRWG_ERR_BAD_ARG;
            }
            MomLaunch p;
            memset(&p, 0, sizeof(p));
            p.d = k.mom;
            p.src[0] = s0;
            p.src[1] = s1;
            p.tabs = tabs;
            p.gd = &gk[i].mom;
            p.scratch = momScratch;
            p.out = momSlots + (size_t)k.mom.slot * SRWG_MOM_SLOT;
            p.nb = nb; p.bDesc = constStride; p.bTab = tabStride;
            p.bSrc = bSrc;
            p.bOut = (long long)nSlots * SRWG_MOM_SLOT;
            e = launch_moments(p, st);
        } else if (k.kind == K_INT) {
            if (intOut == nullptr || nb != 1) {
                g_lastDetail = "intensity extraction pass without its buffer";
                return SRWG_ERR_BAD_ARG;
            }
            e = launch_extract(k.mom, &gk[i].mom, s0, s1, tabs, intOut + k.mom.ioff, st);
        } else if (k.kind == K_LINE) {
            LineLaunch p;
            memset(&p, 0, sizeof(p));
            int r = line_config(k.line, p);
            if (r) return r;
            r = device_twiddles(c, p.N, &p.tw);
            if (r) return r;
            p.src[0] = s0; p.src[1] = s1; p.dst[0] = d0; p.dst[1] = d1;
            p.tabs = tabs;
            p.gd = &gk[i].line;
            p.nb = nb; p.bDesc = constStride; p.bTab = tabStride; p.bSrc = bSrc; p.bDst = bDst;
            p.status = c.status;
            p.spin = g_waitLimit;
            line_window(k.line, p);
            e = launch_line(p, st);
        } else if (k.kind == K_RESIZE) {
            ResizeLaunch p;
            memset(&p, 0, sizeof(p));
            p.d = k.rs;
            p.src[0] = s0; p.src[1] = s1; p.dst[0] = d0; p.dst[1] = d1;
            p.xStepInvO = 1. / k.rs.xStepO;
            p.zStepInvO = 1. / k.rs.zStepO;
            resize_window(k.rs, p);
            p.tabs = tabs;
            p.gd = &gk[i].rs;
            p.nb = nb; p.bDesc = constStride; p.bTab = tabStride; p.bSrc = bSrc; p.bDst = bDst;
            e = launch_resize(p, st);
        } else {
            PwLaunch p;
            memset(&p, 0, sizeof(p));
            p.d = k.pwk;
            p.src[0] = s0; p.src[1] = s1; p.dst[0] = d0; p.dst[1] = d1;
            p.tabs = tabs;
            p.gd = &gk[i].pwk;
            p.nb = nb; p.bDesc = constStride; p.bTab = tabStride; p.bSrc = bSrc; p.bDst = bDst;
            e = launch_pw(p, st);
        }
        if (e != cudaSuccess) {
            g_lastDetail = std::string("kernel launch: ") + cudaGetErrorString(e);
            return SRWG_ERR_CUDA;
        }
        if (ev) CUDA_TRY(cudaEventRecord(ev[2 * i + 1], st));
    }
    return 0;
}

// doubles of the scratch of the plan's largest moment pass (0: no moment pass)
static size_t mom_scratch_for(const Planner& pl)
{
    size_t m = 0;
    for (const KernelDesc& k : pl.kernels)
        if (k.kind == K_MOM) m = std::max(m, mom_scratch_doubles(k.mom.nx, k.mom.nz));
    return m;
}

static int ensure_doubles(double** buf, size_t* cap, size_t n)
{
    if (*buf && *cap >= n) return 0;
    if (*buf) { cudaFree(*buf); *buf = nullptr; *cap = 0; }
    CUDA_TRY(cudaMalloc(buf, n * sizeof(double)));
    *cap = n;
    return 0;
}

// runs the plan's passes on one wavefront (or nb wavefronts with the same plan); moment passes
// write their sums to momSlots (nMomSlots * SRWG_MOM_SLOT doubles per wavefront)
static int execute(Planner& pl, DeviceCtx& c, const float2* inX, const float2* inY, float2* outX, float2* outY,
                   float2* work, size_t workElems, const float2* dtab, cudaStream_t st, cudaEvent_t* ev = nullptr,
                   int nb = 1, long long inStride = 0, long long outStride = 0, double* momSlots = nullptr,
                   double* momScratch = nullptr, char* intOut = nullptr)
{
    const size_t nOut = (size_t)pl.w.nx * pl.w.nz;
    bool anyField = false;
    for (const KernelDesc& k : pl.kernels) anyField |= !reads_only(k.kind);
    if (!anyField) {          // the output is the input (moment passes, if any, read the input)
        for (int b = 0; b < nb; b++) {
            CUDA_TRY(cudaMemcpyAsync(outX + b * outStride, inX + b * inStride, nOut * sizeof(float2),
                                     cudaMemcpyDeviceToDevice, st));
            CUDA_TRY(cudaMemcpyAsync(outY + b * outStride, inY + b * inStride, nOut * sizeof(float2),
                                     cudaMemcpyDeviceToDevice, st));
        }
        if (pl.kernels.empty()) return 0;
    }
    size_t descOff;
    const_bytes(pl, &descOff);
    return execute_passes(pl.kernels, c, nb, inX, inY, inStride, outX, outY, outStride, work, workElems,
                          (const char*)dtab, 0, descOff, st, ev, nullptr, momScratch, momSlots, pl.nMomSlots, intOut);
}

static int ensure_work(DeviceCtx& c, size_t elems)
{
    if (c.workElems >= elems && c.work) return 0;
    if (c.work) { cudaFree(c.work); c.work = nullptr; c.workElems = 0; }
    CUDA_TRY(cudaMalloc(&c.work, 4 * elems * sizeof(float2)));
    c.workElems = elems;
    return 0;
}

static int ensure_io(DeviceCtx& c, size_t elems)
{
    if (c.ioElems >= elems && c.io) return 0;
    if (c.io) { cudaFree(c.io); c.io = nullptr; c.ioElems = 0; }
    CUDA_TRY(cudaMalloc(&c.io, 4 * elems * sizeof(float2)));
    c.ioElems = elems;
    return 0;
}

static void out_wfr(const Planner& pl, SRWLWfr* p)
{   // OutSRWRadPtrs (srradstr.cpp:687): mesh and scalars
    const WfrState& w = pl.w;
    p->mesh.eStart = w.eStart;
    p->mesh.eFin = w.eStart;
    p->mesh.xStart = w.xStart;
    p->mesh.xFin = w.xStart + w.xStep * (w.nx - 1);
    p->mesh.yStart = w.zStart;
    p->mesh.yFin = w.zStart + w.zStep * (w.nz - 1);
    p->mesh.ne = 1;
    p->mesh.nx = w.nx;
    p->mesh.ny = w.nz;
    p->Rx = w.RobsX; p->Ry = w.RobsZ;
    p->dRx = w.RobsXAbsErr; p->dRy = w.RobsZAbsErr;
    p->xc = w.xc; p->yc = w.zc;
    p->presCA = (char)w.Pres;
    p->avgPhotEn = w.avgPhotEn;
    if (p->arElecPropMatr != nullptr && w.havePropM)
        for (int i = 0; i < 20; i++) p->arElecPropMatr[i] = w.propM[i];
}

// output moments: the plan-time ones, or (with moment passes) the replayed bookkeeping with the
// passes' result slots of one wavefront
static void out_moments(const Planner& pl, SRWLWfr* p, const double* slots = nullptr)
{
    double mx[11], mz[11];
    if (pl.nMomSlots > 0 && slots != nullptr) pl.replay_moments(slots, mx, mz);
    else for (int i = 0; i < 11; i++) { mx[i] = pl.w.momX[i]; mz[i] = pl.w.momZ[i]; }
    if (p->arMomX) for (int i = 0; i < 11; i++) p->arMomX[i] = mx[i];
    if (p->arMomY) for (int i = 0; i < 11; i++) p->arMomY[i] = mz[i];
}

}  // namespace srwg

using namespace srwg;

struct srwgPlan {
    Planner pl;
    int device = 0;
    DeviceCtx* ctx = nullptr;   // bound at the first execution
    float2* dtab = nullptr;     // the plan's point-wise tables on that device
    size_t dtabElems = 0;
    bool tabReady = false;
    double* dmom = nullptr;     // moment passes: result slots of every wavefront | scratch
    size_t dmomDoubles = 0;
    int lastN = 0;              // wavefronts of the last execution
    cudaEvent_t momEv = nullptr;  // recorded after the last execution
    ~srwgPlan()
    {
        if (dtab) cudaFree(dtab);
        if (dmom) cudaFree(dmom);
        if (momEv) cudaEventDestroy(momEv);
    }
};

// moment buffers of a plan for n wavefronts; slots of wavefront b at dmom + b * nMomSlots * SLOT
static int plan_moments(srwgPlan* plan, int n, double** slots, double** scratch)
{
    *slots = *scratch = nullptr;
    if (plan->pl.nMomSlots == 0) return 0;
    const size_t per = (size_t)plan->pl.nMomSlots * SRWG_MOM_SLOT;
    int r = ensure_doubles(&plan->dmom, &plan->dmomDoubles, per * (size_t)n + mom_scratch_for(plan->pl));
    if (r) return r;
    if (plan->momEv == nullptr) CUDA_TRY(cudaEventCreateWithFlags(&plan->momEv, cudaEventDisableTiming));
    *slots = plan->dmom;
    *scratch = plan->dmom + per * (size_t)n;
    return 0;
}

// result slots of wavefront b of the last execution (host copy); false when there are none
static bool plan_slots(const srwgPlan* plan, int b, std::vector<double>& hs)
{
    if (plan->pl.nMomSlots == 0 || plan->lastN <= b || plan->dmom == nullptr || plan->momEv == nullptr) return false;
    const size_t per = (size_t)plan->pl.nMomSlots * SRWG_MOM_SLOT;
    hs.resize(per);
    if (cudaSetDevice(plan->device) != cudaSuccess || cudaEventSynchronize(plan->momEv) != cudaSuccess ||
        cudaMemcpy(hs.data(), plan->dmom + per * (size_t)b, per * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return false;
    return true;
}

static int plan_bind(srwgPlan* plan, cudaStream_t st)
{
    int r = device_ctx(plan->device, &plan->ctx);
    if (r) return r;
    if (!plan->tabReady) {
        r = upload_tables(plan->pl, &plan->dtab, &plan->dtabElems, st);
        if (r) return r;
        CUDA_TRY(cudaStreamSynchronize(st));
        plan->tabReady = true;
    }
    return ensure_work(*plan->ctx, (size_t)plan->pl.maxElems);
}

extern "C" {

void srwlUtiSetWfrModifFunc(int (*pExtFunc)(int action, SRWLWfr* pWfrIn, char pol))
{
    std::lock_guard<std::mutex> lk(g_mutex);
    g_modifFunc = pExtFunc;
}

void srwlUtiSetAllocArrayFunc(char* (*pExtFunc)(char type, long long len))
{
    std::lock_guard<std::mutex> lk(g_mutex);
    g_allocArrayFunc = pExtFunc;
}

int srwlUtiGetErrText(char* t, int erNo)
{
    if (t == nullptr) return 0;
    const char* s = nullptr;
    switch (erNo) {
    case 0: s = ""; break;
    case MEMORY_ALLOCATION_FAILURE: s = "Memory allocation failure."; break;
    case UNKNOWN_OPTICAL_ELEMENT: s = "Unknown optical element or incorrect optical element definition."; break;
    case ERROR_IN_FFT: s = "Error in FFT."; break;
    case CAN_NOT_PROPAGATE_1D_RAD: s = "Propagation needs more than one point in both the horizontal and the vertical direction."; break;
    case PHOT_EN_SHOULD_BE_POSITIVE: s = "Photon energy should be positive."; break;
    case SRWL_INCORRECT_PARAM_FOR_GAUS_BEAM_COMP: s = "Incorrect or insufficient parameters for Gaussian beam calculation."; break;
    case SRWL_INCORRECT_PARAM_FOR_INT_EXTR: s = "Incorrect or insufficient parameters for intensity extraction."; break;
    case SRWL_WFR_EXT_MODIF_FAILED: s = "The wavefront modification (re-allocation) callback failed."; break;
    case SRWL_INCORRECT_PARAM_FOR_WFR_PROP: s = "Incorrect or insufficient parameters for wavefront propagation."; break;
    case SRWL_WFR_EXT_FUNC_NOT_DEFINED: s = "No wavefront modification (re-allocation) callback is registered."; break;
    case SRWL_EXT_ARRAY_ALLOC_FAILED: s = "Failed to allocate array in front-end / client environment."; break;
    case SRWG_ERR_UNSUPPORTED: s = "Not supported on the GPU propagation path"; break;
    case SRWG_ERR_CUDA: s = "CUDA error"; break;
    case SRWG_ERR_NO_DEVICE: s = "No usable CUDA device"; break;
    case SRWG_ERR_BAD_ARG: s = "Invalid argument"; break;
    case SRWG_ERR_STATIC_LIMIT: s = "Propagation too large for the allocation-free entry point"; break;
    default: s = "Unknown error or warning number."; break;
    }
    std::string txt(s);
    if ((erNo >= SRWG_ERR_UNSUPPORTED && erNo <= SRWG_ERR_STATIC_LIMIT) && !g_lastDetail.empty()) txt += ": " + g_lastDetail;
    strncpy(t, txt.c_str(), 2047);
    t[2047] = 0;
    return 0;
}

// the intensity extractions of a stage that ran: each into the caller's array (allocated through the
// registered allocation function when the caller passed none, AllocExtIntArray srradstr.cpp:799),
// with its mesh (GetIntMesh, srradstr.cpp:4140: the wavefront's x and y mesh, eStart kept)
static int deliver_extractions(const Planner& pl, const char* dev, cudaStream_t st, char** arI, SRWLRadMesh* arIM)
{
    for (const IntOut& o : pl.intOuts) {
        char*& dst = arI[o.index];
        if (dst == nullptr) {
            if (g_allocArrayFunc != nullptr) dst = (*g_allocArrayFunc)(o.arType, (long long)o.nx * o.nz);
            if (dst == nullptr) return SRWL_EXT_ARRAY_ALLOC_FAILED;
        }
        CUDA_TRY(cudaMemcpyAsync(dst, dev + o.off, (size_t)o.bytes, cudaMemcpyDeviceToHost, st));
        if (arIM != nullptr) {
            SRWLRadMesh& m = arIM[o.index];
            m.ne = 1;
            m.nx = o.nx;
            m.xStart = o.xStart;
            m.xFin = o.xStart + o.xStep * (o.nx - 1);
            m.ny = o.nz;
            m.yStart = o.zStart;
            m.yFin = o.zStart + o.zStep * (o.nz - 1);
        }
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    return 0;
}

// srwlPropagElecField for a plan with stage boundaries (an element planned on moments measured from
// the field) or intensity extractions: each stage runs from the previous stage's output into a stage
// buffer, its moment results and extractions come back to the host, and planning resumes; the last
// stage's output is the result.  pr: the planning status (SRWG_NEED_STAGE or 0 for a single stage)
static int propagate_staged(Planner& pl, SRWLWfr* pWfr, int dev, int pr, char** arI, SRWLRadMesh* arIM)
{
    DeviceCtx* c = nullptr;
    int r = device_ctx(dev, &c);
    if (r) return r;
    cudaStream_t st = c->stream;
    const size_t nIn = (size_t)pl.in.nx * pl.in.nz;
    r = ensure_io(*c, nIn);
    if (r) return r;
    if (pWfr->arEx) CUDA_TRY(cudaMemcpyAsync(c->io, pWfr->arEx, nIn * sizeof(float2), cudaMemcpyHostToDevice, st));
    else CUDA_TRY(cudaMemsetAsync(c->io, 0, nIn * sizeof(float2), st));
    if (pWfr->arEy) CUDA_TRY(cudaMemcpyAsync(c->io + c->ioElems, pWfr->arEy, nIn * sizeof(float2), cudaMemcpyHostToDevice, st));
    else CUDA_TRY(cudaMemsetAsync(c->io + c->ioElems, 0, nIn * sizeof(float2), st));
    const float2* curX = c->io;
    const float2* curY = c->io + c->ioElems;
    float2 *oX = nullptr, *oY = nullptr;
    std::vector<double> slots, tmp;
    for (int k = 0;; k++) {
        const bool last = (pr == 0);
        const size_t nSt = (size_t)pl.w.nx * pl.w.nz;
        float2*& sb = c->stg[k & 1];
        size_t& se = c->stgElems[k & 1];
        if (sb == nullptr || se < nSt) {
            if (sb) cudaFree(sb);
            sb = nullptr; se = 0;
            CUDA_TRY(cudaMalloc(&sb, 2 * nSt * sizeof(float2)));
            se = nSt;
        }
        oX = sb; oY = sb + se;
        r = ensure_work(*c, (size_t)std::max<long long>(pl.maxElems, 1));
        if (r) return r;
        r = upload_tables(pl, &c->tab, &c->tabElems, st);
        if (r) return r;
        const size_t nSlotD = (size_t)pl.nMomSlots * SRWG_MOM_SLOT;
        if (nSlotD) {
            r = ensure_doubles(&c->mom, &c->momDoubles, nSlotD + mom_scratch_for(pl));
            if (r) return r;
        }
        if (pl.intBytes > 0 && (c->genBuf == nullptr || c->genBytes < (size_t)pl.intBytes)) {
            if (c->genBuf) cudaFree(c->genBuf);
            c->genBuf = nullptr; c->genBytes = 0;
            CUDA_TRY(cudaMalloc(&c->genBuf, (size_t)pl.intBytes));
            c->genBytes = (size_t)pl.intBytes;
        }
        r = execute(pl, *c, curX, curY, oX, oY, c->work, c->workElems, c->tab, st, nullptr, 1, 0, 0,
                    nSlotD ? c->mom : nullptr, nSlotD ? c->mom + nSlotD : nullptr,
                    pl.intBytes > 0 ? (char*)c->genBuf : nullptr);
        if (r) return r;
        if (!pl.intOuts.empty()) {
            r = deliver_extractions(pl, (const char*)c->genBuf, st, arI, arIM);
            if (r) return r;
        }
        tmp.assign(nSlotD, 0.);
        if (nSlotD) CUDA_TRY(cudaMemcpyAsync(tmp.data(), c->mom, nSlotD * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        slots.resize(nSlotD, 0.);
        for (const KernelDesc& kd : pl.kernels)          // the slots this stage's passes wrote
            if (kd.kind == K_MOM)
                std::copy(tmp.begin() + (size_t)kd.mom.slot * SRWG_MOM_SLOT,
                          tmp.begin() + (size_t)(kd.mom.slot + 1) * SRWG_MOM_SLOT,
                          slots.begin() + (size_t)kd.mom.slot * SRWG_MOM_SLOT);
        if (last) break;
        pr = pl.resume(slots.data());
        if (pr && pr != SRWG_NEED_STAGE) { g_lastDetail = pl.err; return pr; }
        curX = oX; curY = oY;
    }
    const size_t nOut = (size_t)pl.w.nx * pl.w.nz;
    bool hadX = pWfr->arEx != nullptr, hadY = pWfr->arEy != nullptr;
    bool resized = (pl.w.nx != pl.in.nx) || (pl.w.nz != pl.in.nz);
    out_wfr(pl, pWfr);
    if (resized) {
        if (g_modifFunc == nullptr) return SRWL_WFR_EXT_FUNC_NOT_DEFINED;
        if ((*g_modifFunc)(2, pWfr, 0)) return SRWL_WFR_EXT_MODIF_FAILED;
        out_wfr(pl, pWfr);
    }
    if (hadX && pWfr->arEx) CUDA_TRY(cudaMemcpyAsync(pWfr->arEx, oX, nOut * sizeof(float2), cudaMemcpyDeviceToHost, st));
    if (hadY && pWfr->arEy) CUDA_TRY(cudaMemcpyAsync(pWfr->arEy, oY, nOut * sizeof(float2), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    out_moments(pl, pWfr, slots.empty() ? nullptr : slots.data());
    return 0;
}

int srwlPropagElecField(SRWLWfr* pWfr, SRWLOptC* pOpt, int nInt, char** arID, SRWLRadMesh* arIM, char** arI,
                        double* arParGPU)
{
    std::lock_guard<std::mutex> lk(g_mutex);
    g_lastDetail.clear();
    if (pWfr == nullptr || pOpt == nullptr) return SRWL_INCORRECT_PARAM_FOR_WFR_PROP;
    int dev = 0;
    if (arParGPU != nullptr && arParGPU[0] >= 1. && arParGPU[1] >= 1.) dev = (int)arParGPU[1] - 1;
    if (pWfr->arEx == nullptr && pWfr->arEy == nullptr) return SRWL_INCORRECT_PARAM_FOR_WFR_PROP;

    Planner pl;
    pl.allowStages = true;
    // intensity extractions after elements (PropagateRadiationGuided, sroptcnt.cpp:268, and
    // ExtractPropagatedIntensity :429): arID[0..4][i] = element number (1-based), polarisation,
    // intensity type, dependence, representation; negative values (and arIM[i].ne < 0) of the
    // later requests take the first request's
    const bool wantInt = nInt > 0 && arID != nullptr && arI != nullptr;
    if (wantInt) {
        for (int j = 0; j < 5; j++)
            if (arID[j] == nullptr) return SRWL_INCORRECT_PARAM_FOR_WFR_PROP;
        for (int i = 0; i < nInt; i++) {
            IntReq q;
            q.index = i;
            q.elem = (int)arID[0][i] - 1;
            q.pol = arID[1][i]; q.type = arID[2][i]; q.dep = arID[3][i]; q.pres = arID[4][i];
            if (nInt > 1 && i > 0) {
                if (q.pol < 0) q.pol = arID[1][0];
                if (q.type < 0) q.type = arID[2][0];
                if (q.dep < 0) q.dep = arID[3][0];
                if (q.pres < 0) q.pres = arID[4][0];
                if (arIM != nullptr && arIM[i].ne < 0) arIM[i] = arIM[0];
            }
            pl.intReqs.push_back(q);
        }
    }
    int r = pl.plan(pWfr, pOpt);
    if (r == SRWG_NEED_STAGE || (r == 0 && wantInt))
        return propagate_staged(pl, pWfr, dev, r, wantInt ? arI : nullptr, wantInt ? arIM : nullptr);
    if (r) { g_lastDetail = pl.err; return r; }
    DeviceCtx* c = nullptr;
    r = device_ctx(dev, &c);
    if (r) return r;
    const size_t nIn = (size_t)pl.in.nx * pl.in.nz, nOut = (size_t)pl.w.nx * pl.w.nz;
    r = ensure_io(*c, nIn > nOut ? nIn : nOut);
    if (r) return r;
    r = ensure_work(*c, (size_t)pl.maxElems);
    if (r) return r;
    float2* inX = c->io;
    float2* inY = c->io + c->ioElems;
    float2* outX = c->io + 2 * c->ioElems;
    float2* outY = c->io + 3 * c->ioElems;
    cudaStream_t st = c->stream;
    if (pWfr->arEx) CUDA_TRY(cudaMemcpyAsync(inX, pWfr->arEx, nIn * sizeof(float2), cudaMemcpyHostToDevice, st));
    else CUDA_TRY(cudaMemsetAsync(inX, 0, nIn * sizeof(float2), st));
    if (pWfr->arEy) CUDA_TRY(cudaMemcpyAsync(inY, pWfr->arEy, nIn * sizeof(float2), cudaMemcpyHostToDevice, st));
    else CUDA_TRY(cudaMemsetAsync(inY, 0, nIn * sizeof(float2), st));
    r = upload_tables(pl, &c->tab, &c->tabElems, st);
    if (r) return r;
    const size_t nSlotD = (size_t)pl.nMomSlots * SRWG_MOM_SLOT;
    if (nSlotD) {
        r = ensure_doubles(&c->mom, &c->momDoubles, nSlotD + mom_scratch_for(pl));
        if (r) return r;
    }
    r = execute(pl, *c, inX, inY, outX, outY, c->work, c->workElems, c->tab, st, nullptr, 1, 0, 0,
                nSlotD ? c->mom : nullptr, nSlotD ? c->mom + nSlotD : nullptr);
    if (r) return r;
    std::vector<double> hs(nSlotD);
    if (nSlotD) CUDA_TRY(cudaMemcpyAsync(hs.data(), c->mom, nSlotD * sizeof(double), cudaMemcpyDeviceToHost, st));
    bool hadX = pWfr->arEx != nullptr, hadY = pWfr->arEy != nullptr;
    bool resized = (pl.w.nx != pl.in.nx) || (pl.w.nz != pl.in.nz);
    out_wfr(pl, pWfr);
    if (resized) {
        CUDA_TRY(cudaStreamSynchronize(st));
        if (g_modifFunc == nullptr) return SRWL_WFR_EXT_FUNC_NOT_DEFINED;
        if ((*g_modifFunc)(2, pWfr, 0)) return SRWL_WFR_EXT_MODIF_FAILED;
        out_wfr(pl, pWfr);
    }
    if (hadX && pWfr->arEx) CUDA_TRY(cudaMemcpyAsync(pWfr->arEx, outX, nOut * sizeof(float2), cudaMemcpyDeviceToHost, st));
    if (hadY && pWfr->arEy) CUDA_TRY(cudaMemcpyAsync(pWfr->arEy, outY, nOut * sizeof(float2), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    out_moments(pl, pWfr, nSlotD ? hs.data() : nullptr);
    return 0;
}

int srwgPlanCreate(const SRWLWfr* pWfr, const SRWLOptC* pOpt, int device, srwgPlan** ppPlan)
{
    if (ppPlan == nullptr) return SRWG_ERR_BAD_ARG;
    *ppPlan = nullptr;
    // the planner is host bookkeeping without shared state: plans are made outside the library lock,
    // so that threads can plan concurrently
    srwgPlan* p = new srwgPlan();
    int r = p->pl.plan(pWfr, pOpt);
    std::lock_guard<std::mutex> lk(g_mutex);
    g_lastDetail.clear();
    if (r) { g_lastDetail = p->pl.err; delete p; return r; }
    p->device = device;
    // validate every pass configuration up front
    for (const KernelDesc& k : p->pl.kernels) {
        if (k.kind == K_LINE) {
            LineLaunch l;
            memset(&l, 0, sizeof(l));
            r = line_config(k.line, l);
            if (r) { delete p; return r; }
        }
    }
    *ppPlan = p;
    return 0;
}

int srwgPlanGetOutput(const srwgPlan* plan, SRWLWfr* pWfrOut)
{
    if (plan == nullptr || pWfrOut == nullptr) return SRWG_ERR_BAD_ARG;
    out_wfr(plan->pl, pWfrOut);
    std::vector<double> hs;
    const bool have = plan_slots(plan, 0, hs);
    out_moments(plan->pl, pWfrOut, have ? hs.data() : nullptr);
    return 0;
}

int srwgPlanGetMoments(const srwgPlan* plan, int index, double* momX, double* momY)
{
    if (plan == nullptr || index < 0) return SRWG_ERR_BAD_ARG;
    double mx[11], mz[11];
    if (plan->pl.nMomSlots == 0) {
        for (int i = 0; i < 11; i++) { mx[i] = plan->pl.w.momX[i]; mz[i] = plan->pl.w.momZ[i]; }
    } else {
        std::vector<double> hs;
        if (!plan_slots(plan, index, hs)) {
            g_lastDetail = "no executed wavefront with this index";
            return SRWG_ERR_BAD_ARG;
        }
        plan->pl.replay_moments(hs.data(), mx, mz);
    }
    if (momX) for (int i = 0; i < 11; i++) momX[i] = mx[i];
    if (momY) for (int i = 0; i < 11; i++) momY[i] = mz[i];
    return 0;
}

int srwgPlanInfo(const srwgPlan* plan, long* nxIn, long* nyIn, long* nxOut, long* nyOut, int* nKernels, long long* workBytes)
{
    if (plan == nullptr) return SRWG_ERR_BAD_ARG;
    if (nxIn) *nxIn = plan->pl.in.nx;
    if (nyIn) *nyIn = plan->pl.in.nz;
    if (nxOut) *nxOut = plan->pl.w.nx;
    if (nyOut) *nyOut = plan->pl.w.nz;
    if (nKernels) *nKernels = (int)plan->pl.kernels.size();
    if (workBytes) *workBytes = 4LL * plan->pl.maxElems * (long long)sizeof(float2);
    return 0;
}

int srwgPlanExecute(srwgPlan* plan, const float* dExIn, const float* dEyIn, float* dExOut, float* dEyOut, void* stream)
{
    return srwgPlanExecuteBatch(plan, 1, dExIn, dEyIn, 0, dExOut, dEyOut, 0, stream);
}

int srwgPlanExecuteBatch(srwgPlan* plan, int n, const float* dExIn, const float* dEyIn, long long strideIn,
                         float* dExOut, float* dEyOut, long long strideOut, void* stream)
{
    std::lock_guard<std::mutex> lk(g_mutex);
    g_lastDetail.clear();
    if (plan == nullptr || dExIn == nullptr || dEyIn == nullptr || dExOut == nullptr || dEyOut == nullptr || n < 1)
        return SRWG_ERR_BAD_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int r = plan_bind(plan, st);
    if (r) return r;
    DeviceCtx& c = *plan->ctx;
    if ((strideIn & 1) || (strideOut & 1)) return SRWG_ERR_BAD_ARG;     // whole complex points
    // one launch per pass for the whole batch (grid z = wavefront) when the work buffers hold it
    const size_t per = (size_t)plan->pl.maxElems;
    int chunk = n;
    const size_t budget = (size_t)1 << 30;                               // work elements (8 GiB)
    while (chunk > 1 && 4 * (size_t)chunk * per > budget) chunk = (chunk + 1) / 2;
    r = ensure_work(c, (size_t)chunk * per);
    if (r) return r;
    double *slots, *scratch;
    r = plan_moments(plan, n, &slots, &scratch);
    if (r) return r;
    const size_t perSlots = (size_t)plan->pl.nMomSlots * SRWG_MOM_SLOT;
    for (int b0 = 0; b0 < n; b0 += chunk) {
        const int nb = std::min(chunk, n - b0);
        r = execute(plan->pl, c, (const float2*)(dExIn + b0 * strideIn), (const float2*)(dEyIn + b0 * strideIn),
                    (float2*)(dExOut + b0 * strideOut), (float2*)(dEyOut + b0 * strideOut), c.work, per, plan->dtab,
                    st, nullptr, nb, strideIn / 2, strideOut / 2, slots ? slots + perSlots * b0 : nullptr, scratch);
        if (r) return r;
    }
    if (slots) {
        CUDA_TRY(cudaEventRecord(plan->momEv, st));
        plan->lastN = n;
    }
    return 0;
}

int srwgPlanExecuteTimed(srwgPlan* plan, const float* dExIn, const float* dEyIn, float* dExOut, float* dEyOut,
                         void* stream, float* kernelMs, int maxKernels, int* nTimed)
{
    std::lock_guard<std::mutex> lk(g_mutex);
    g_lastDetail.clear();
    if (plan == nullptr || dExIn == nullptr || dEyIn == nullptr || dExOut == nullptr || dEyOut == nullptr)
        return SRWG_ERR_BAD_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int r = plan_bind(plan, st);
    if (r) return r;
    DeviceCtx& c = *plan->ctx;
    const size_t nk = plan->pl.kernels.size();
    std::vector<cudaEvent_t> ev(2 * nk);
    for (auto& e : ev) CUDA_TRY(cudaEventCreate(&e));
    double *slots, *scratch;
    r = plan_moments(plan, 1, &slots, &scratch);
    if (r == 0)
        r = execute(plan->pl, c, (const float2*)dExIn, (const float2*)dEyIn, (float2*)dExOut, (float2*)dEyOut, c.work,
                    c.workElems, plan->dtab, st, nk ? ev.data() : nullptr, 1, 0, 0, slots, scratch);
    if (r == 0 && slots) {
        if (cudaEventRecord(plan->momEv, st) != cudaSuccess) r = SRWG_ERR_CUDA;
        else plan->lastN = 1;
    }
    if (r == 0) {
        CUDA_TRY(cudaStreamSynchronize(st));
        for (size_t i = 0; i < nk && (int)i < maxKernels; i++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
            if (kernelMs) kernelMs[i] = ms;
        }
        if (nTimed) *nTimed = (int)nk;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return r;
}

int srwgPlanDestroy(srwgPlan* plan)
{
    delete plan;
    return 0;
}

int srwgSetWaitLimit(long long iterations)
{
    std::lock_guard<std::mutex> lk(g_mutex);
    if (iterations < 0) return SRWG_ERR_BAD_ARG;
    g_waitLimit = iterations;
    return 0;
}

int srwgGetWaitStatus(int device, int* count, int reset)
{
    std::lock_guard<std::mutex> lk(g_mutex);
    if (count == nullptr) return SRWG_ERR_BAD_ARG;
    DeviceCtx* c = nullptr;
    int r = device_ctx(device, &c);
    if (r) return r;
    CUDA_TRY(cudaMemcpy(count, c->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (reset) CUDA_TRY(cudaMemset(c->status, 0, sizeof(int)));
    return 0;
}

long srwgNextFftNumber(long n)
{
    return srwg::next_correct_number_for_fft(n);
}

int srwgTuneSetFamily(int axis, int N, int family)
{
    std::lock_guard<std::mutex> lk(g_tuneMutex);
    tune_ensure_loaded();
    if ((axis != 0 && axis != 1) || !default_family(N)) return SRWG_ERR_BAD_ARG;
    const int f = family == 0 ? default_family(N) : family;
    if (!(f == FAM_POW2 && line2_supported(N)) && !(f == FAM_SPEC && (linen_supported(N) || linen_pow2(N)))) {
        g_lastDetail = "no kernel of this family for this line length";
        return SRWG_ERR_BAD_ARG;
    }
    TuneEntry& e = g_tune[std::make_pair(axis, N)];
    e.fam = f;
    if (e.lines && !fixed_lines_valid(axis, N, e.lines, f)) e.lines = 0;
    return 0;
}

int srwgTuneSetLines(int axis, int N, int lines)
{
    std::lock_guard<std::mutex> lk(g_tuneMutex);
    tune_ensure_loaded();
    if (axis != 0 && axis != 1) return SRWG_ERR_BAD_ARG;
    auto key = std::make_pair(axis, N);
    auto it = g_tune.find(key);
    const int fam = (it != g_tune.end() && it->second.fam) ? it->second.fam : default_family(N);
    if (lines == 0) {
        if (it != g_tune.end()) g_tune.erase(it);
        return 0;
    }
    if (!fixed_lines_valid(axis, N, lines, fam)) {
        g_lastDetail = "not a valid launch shape for this line length";
        return SRWG_ERR_BAD_ARG;
    }
    g_tune[key].fam = fam;
    g_tune[key].lines = lines;
    return 0;
}

int srwgTuneGetLines(int axis, int N, int* lines)
{
    if (lines == nullptr || (axis != 0 && axis != 1)) return SRWG_ERR_BAD_ARG;
    *lines = fixed_lines_per_cta(axis, N);
    return 0;
}

int srwgTuneGetFamily(int axis, int N, int* family)
{
    if (family == nullptr || (axis != 0 && axis != 1)) return SRWG_ERR_BAD_ARG;
    *family = fixed_family(axis, N);
    return 0;
}

int srwgTuneLoad(const char* path, int* nEntries)
{
    std::lock_guard<std::mutex> lk(g_tuneMutex);
    g_tuneLoaded = true;
    g_tune.clear();
    if (path == nullptr || !*path) { if (nEntries) *nEntries = 0; return 0; }
    if (tune_load_file(path, nEntries) != 0) {
        g_lastDetail = std::string("cannot read ") + path;
        return SRWG_ERR_BAD_ARG;
    }
    return 0;
}

int srwgPlanDescribe(const srwgPlan* plan, char* buf, int bufLen)
{
    if (plan == nullptr || buf == nullptr || bufLen <= 0) return SRWG_ERR_BAD_ARG;
    std::string s = plan->pl.describe();
    strncpy(buf, s.c_str(), bufLen - 1);
    buf[bufLen - 1] = 0;
    return 0;
}

}  // extern "C"
