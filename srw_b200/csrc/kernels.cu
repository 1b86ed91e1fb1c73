// sm_100a kernels for SRW's Fourier-optics propagation path.
//
// All passes are HBM-bandwidth bound (a complex FP32 point is read and written once per pass,
// ~1-4 flop/B), so they are plain SIMT kernels organised around full-line shared-memory tiles;
// no tensor cores.  Phase arguments are formed and reduced modulo 2*pi in FP64 and evaluated
// with an FP32 sincosf, as the reference forms them in double before its float CosAndSin
// (sroptelm.h:856-871).
#include <mutex>
#include <set>

#include "common.cuh"

namespace srwg {

// CUDA function attributes (here: the dynamic shared-memory limit) belong to a device's context,
// so they are set once per device and kernel group, before that group's first launch there
static bool attrs_needed(int group)
{
    static std::mutex m;
    static std::set<long long> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return true;
    std::lock_guard<std::mutex> lk(m);
    return done.insert(((long long)dev << 8) | group).second;
}

// ------------------------------------------------------------------------------------------------
// LINE pass: a CTA owns L whole rows (axis 0) or L whole columns (axis 1) in shared memory; G
// thread groups of T threads transform them in ceil(L/G) batches (T*G <= 512 threads, so each
// thread can hold its 16 in-flight points and twiddles in registers).
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(512, 1) line_kernel(const LineLaunch p)
{
    extern __shared__ float2 sm[];
    // descriptor in shared memory: point-wise code takes references to it (a reference to a
    // kernel parameter would force a copy of the whole parameter block to local memory)
    const LineDesc& d = *reinterpret_cast<const LineDesc*>(reinterpret_cast<const char*>(p.gd) + blockIdx.z * p.bDesc);
    __shared__ int radix[SRWG_MAX_STAGES];
    if (threadIdx.x < SRWG_MAX_STAGES) radix[threadIdx.x] = p.radix[threadIdx.x];
    __syncthreads();
    const int comp = blockIdx.y;
    const float2* __restrict__ src = p.src[comp] + blockIdx.z * p.bSrc;
    float2* __restrict__ dst = p.dst[comp] + blockIdx.z * p.bDst;
    const int N = p.N, T = p.T, L = p.L, P = p.P, nl = p.nlines;
    const int tid = threadIdx.x, nth = blockDim.x;
    const int G = nth / T;
    const int g = tid / T, t = tid - g * T;
    const int line0 = (blockIdx.x + p.blk0) * L;

    // ---- load the tile
    if (d.axis == 0) {
        for (int e = tid; e < N * L; e += nth) {
            int c = e / N, k = e - c * N;
            if (line0 + c < nl) sm[(size_t)c * P + k] = __ldcs(&src[(size_t)(line0 + c) * N + k]);
        }
    } else {
        for (int e = tid; e < N * L; e += nth) {
            int r = e / L, c = e - r * L;
            int col = line0 + c;
            if (col < nl) sm[(size_t)c * P + r] = __ldcs(&src[(size_t)r * nl + col]);
        }
    }
    __syncthreads();

    // chains with their along-line factors in the plan's tables (as the power-of-two kernels); the
    // per-line factors of all chains are multiplied once and applied at the store
    const float2* tabs = p.tabs + blockIdx.z * p.bTab;
    const PwOps* ex = &d.extra;
    ChainG pre, mid, fin;
    pre.rs1 = 0; pre.mir = 0; pre.rs2 = d.f1_pre.rs; pre.tab = (int)d.t_pre.tab; pre.extra = 0;
    mid.rs1 = d.f1 ? d.f1_post.rs : 0; mid.mir = d.mirror_along; mid.rs2 = d.f2 ? d.f2_pre.rs : 0;
    mid.tab = (int)d.t_mid.tab; mid.extra = d.has_extra;
    if (d.f2) {
        fin.rs1 = d.f2_post.rs; fin.mir = 0; fin.rs2 = 0; fin.tab = (int)d.t_fin.tab; fin.extra = 0;
    } else {
        fin = mid;
    }
    const bool has_lf = (d.t_pre.ltab >= 0) || (d.t_mid.ltab >= 0) || (d.t_fin.ltab >= 0);

    // ---- transforms, batch by batch (uniform trip count: every thread reaches every barrier)
    if (d.f1 || d.f2) {
        const int nb = (L + G - 1) / G;
        for (int it = 0; it < nb; it++) {
            const int c = it * G + g;
            const int line = line0 + c;
            const bool active = (g < G) && (c < L) && (line < nl);
            float2* s = sm + (size_t)(c < L ? c : 0) * P;
            if (d.f1) {
                if (!chainG_trivial(pre)) gather_pass_t(s, N, line, pre, t, T, active, tabs, ex, d.axis);
                if (d.f1 > 0) run_fft<1>(s, N, radix, p.nst, p.tw, t, T, active);
                else run_fft<-1>(s, N, radix, p.nst, p.tw, t, T, active);
            }
            if (d.f2) {
                if (!chainG_trivial(mid)) gather_pass_t(s, N, line, mid, t, T, active, tabs, ex, d.axis);
                if (d.f2 > 0) run_fft<1>(s, N, radix, p.nst, p.tw, t, T, active);
                else run_fft<-1>(s, N, radix, p.nst, p.tw, t, T, active);
            }
        }
    }
    const bool triv = chainG_trivial(fin) && !has_lf;

    // ---- store the tile
    for (int e = tid; e < N * L; e += nth) {
        int c, k;
        if (d.axis == 0) { c = e / N; k = e - c * N; }
        else { k = e / L; c = e - k * L; }
        const int line = line0 + c;
        if (line >= nl) continue;
        const float2* sc = sm + (size_t)c * P;
        float2 v;
        if (triv) {
            v = sc[k];
        } else {
            int i;
            const int sr = chainG_src(fin, k, N, i);
            v = cmul(chainG_factor(fin, k, i, line, tabs, ex, d.axis), sc[sr]);
            if (has_lf) {
                float2 lf = make_float2(1.f, 0.f);
                if (d.t_pre.ltab >= 0) lf = cmul(lf, __ldg(&tabs[d.t_pre.ltab + line]));
                if (d.t_mid.ltab >= 0) lf = cmul(lf, __ldg(&tabs[d.t_mid.ltab + line]));
                if (d.t_fin.ltab >= 0) lf = cmul(lf, __ldg(&tabs[d.t_fin.ltab + line]));
                v = cmul(lf, v);
            }
        }
        const int ol = d.mirror_lines ? (nl - 1 - line) : line;
        if (d.axis == 0) __stcs(&dst[(size_t)ol * N + k], v);
        else __stcs(&dst[(size_t)k * nl + ol], v);
    }
}

// ------------------------------------------------------------------------------------------------
// RESIZE pass (RadResizeCore, sroptelm.cpp:3038-3337; OnlyLargerRange :4231)
// ------------------------------------------------------------------------------------------------
// sqrt(FI / app), the amplitude correction of ImproveReAndIm, from two reciprocal square roots (no
// division, and FI * app cannot overflow); within a few ulp of the correctly rounded value; FI >= 0,
// app > 0
__device__ __forceinline__ float amp_ratio(float FI, float app)
{
    return FI > 0.f ? FI * rsqrtf(FI) * rsqrtf(app) : 0.f;
}

__device__ __forceinline__ void lagrange4(float t, float* w)
{
    // cubic through nodes -1, 0, 1, 2 (the reference's SetupInterpolAux02 polynomial)
    float tm1 = t - 1.f, tm2 = t - 2.f, tp1 = t + 1.f;
    w[0] = -t * tm1 * tm2 * (1.f / 6.f);
    w[1] = tp1 * tm1 * tm2 * 0.5f;
    w[2] = -tp1 * t * tm2 * 0.5f;
    w[3] = tp1 * t * tm1 * (1.f / 6.f);
}

__device__ __forceinline__ ResizeAxis load_axis(const float2* tabs, long long off, int i)
{
    ResizeAxis a;
    float4 v = __ldg(reinterpret_cast<const float4*>(tabs + off) + i);
    a.st = __float_as_int(v.x);
    a.ir = __float_as_int(v.y);
    a.rel = v.z;
    a.pad = v.w;
    return a;
}

// one new point of one component: bicubic of Re, Im and |E|^2 over the 4x4 old stencil, the
// reference's bilinear fallback when any of the 32 values is exactly zero, and the amplitude
// correction by the interpolated intensity (ImproveReAndIm)
__device__ __forceinline__ float2 pre_factor(const ResizeDesc& d, const float2* tabs, int ix, int iz);

__device__ __forceinline__ float2 resize_point(const float2* __restrict__ o, int nxo, const float* wx, const float* wz,
                                               float xr, float zr, int irx, int irz, const ResizeDesc* pre = nullptr,
                                               const float2* tabs = nullptr, int gx = 0, int gz = 0)
{
    float2 f[4][4];
    bool low = false;
#pragma unroll
    for (int dz = 0; dz < 4; dz++)
#pragma unroll
        for (int dx = 0; dx < 4; dx++) {
            float2 v = __ldg(&o[(size_t)dz * nxo + dx]);
            if (pre) v = cmul(pre_factor(*pre, tabs, gx + dx, gz + dz), v);
            f[dz][dx] = v;
            low |= (v.x == 0.f) || (v.y == 0.f);
        }
    float2 F;
    float FI;
    if (!low) {
        F = make_float2(0.f, 0.f);
        FI = 0.f;
#pragma unroll
        for (int dz = 0; dz < 4; dz++) {
            float2 rowF = make_float2(0.f, 0.f);
            float rowI = 0.f;
#pragma unroll
            for (int dx = 0; dx < 4; dx++) {
                float2 v = f[dz][dx];
                rowF.x = fmaf(wx[dx], v.x, rowF.x);
                rowF.y = fmaf(wx[dx], v.y, rowF.y);
                rowI = fmaf(wx[dx], v.x * v.x + v.y * v.y, rowI);
            }
            F.x = fmaf(wz[dz], rowF.x, F.x);
            F.y = fmaf(wz[dz], rowF.y, F.y);
            FI = fmaf(wz[dz], rowI, FI);
        }
    } else {
        // bilinear on the 2x2 sub-cell (irx, irz) evaluated at (xr, zr): CheckForLowOrderInterp
        float2 f00 = f[irz][irx], f10 = f[irz][irx + 1], f01 = f[irz + 1][irx], f11 = f[irz + 1][irx + 1];
        float xz = xr * zr;
        F.x = f00.x + (f10.x - f00.x) * xr + (f01.x - f00.x) * zr + (f00.x - f01.x - f10.x + f11.x) * xz;
        F.y = f00.y + (f10.y - f00.y) * xr + (f01.y - f00.y) * zr + (f00.y - f01.y - f10.y + f11.y) * xz;
        float i00 = f00.x * f00.x + f00.y * f00.y, i10 = f10.x * f10.x + f10.y * f10.y;
        float i01 = f01.x * f01.x + f01.y * f01.y, i11 = f11.x * f11.x + f11.y * f11.y;
        FI = i00 + (i10 - i00) * xr + (i01 - i00) * zr + (i00 - i01 - i10 + i11) * xz;
    }
    FI = FI > 0.f ? FI : 0.f;
    float app = F.x * F.x + F.y * F.y;          // ImproveReAndIm
    if (app != 0.f) {
        float fac = amp_ratio(FI, app);
        F.x *= fac; F.y *= fac;
    }
    return F;
}

// interpolation of one point from its 4x4 stencil already in registers (see resize_point)
__device__ __forceinline__ float2 interp_stencil(const float2 (&f)[4][4], const float* wx, const float* wz, float xr,
                                                 float zr, int irx, int irz)
{
    bool low = false;
#pragma unroll
    for (int dz = 0; dz < 4; dz++)
#pragma unroll
        for (int dx = 0; dx < 4; dx++) low |= (f[dz][dx].x == 0.f) || (f[dz][dx].y == 0.f);
    float2 F;
    float FI;
    if (!low) {
        F = make_float2(0.f, 0.f);
        FI = 0.f;
#pragma unroll
        for (int dz = 0; dz < 4; dz++) {
            float2 rowF = make_float2(0.f, 0.f);
            float rowI = 0.f;
#pragma unroll
            for (int dx = 0; dx < 4; dx++) {
                float2 v = f[dz][dx];
                rowF.x = fmaf(wx[dx], v.x, rowF.x);
                rowF.y = fmaf(wx[dx], v.y, rowF.y);
                rowI = fmaf(wx[dx], v.x * v.x + v.y * v.y, rowI);
            }
            F.x = fmaf(wz[dz], rowF.x, F.x);
            F.y = fmaf(wz[dz], rowF.y, F.y);
            FI = fmaf(wz[dz], rowI, FI);
        }
    } else {
        float2 f00 = f[0][0], f10 = f[0][1], f01 = f[1][0], f11 = f[1][1];
        // select the 2x2 sub-cell (irx, irz) without dynamic register indexing
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int c = 0; c < 3; c++)
                if (a == irz && c == irx) { f00 = f[a][c]; f10 = f[a][c + 1]; f01 = f[a + 1][c]; f11 = f[a + 1][c + 1]; }
        float xz = xr * zr;
        F.x = f00.x + (f10.x - f00.x) * xr + (f01.x - f00.x) * zr + (f00.x - f01.x - f10.x + f11.x) * xz;
        F.y = f00.y + (f10.y - f00.y) * xr + (f01.y - f00.y) * zr + (f00.y - f01.y - f10.y + f11.y) * xz;
        float i00 = f00.x * f00.x + f00.y * f00.y, i10 = f10.x * f10.x + f10.y * f10.y;
        float i01 = f01.x * f01.x + f01.y * f01.y, i11 = f11.x * f11.x + f11.y * f11.y;
        FI = i00 + (i10 - i00) * xr + (i01 - i00) * zr + (i00 - i01 - i10 + i11) * xz;
    }
    FI = FI > 0.f ? FI : 0.f;
    float app = F.x * F.x + F.y * F.y;          // ImproveReAndIm
    if (app != 0.f) {
        float fac = amp_ratio(FI, app);
        F.x *= fac; F.y *= fac;
    }
    return F;
}

__device__ __forceinline__ float2 pick3(const float2* c, int o, int dx)
{   // c[o + dx] for o in {0, 1, 2} with compile-time register indices
    return o == 0 ? c[dx] : (o == 1 ? c[dx + 1] : c[dx + 2]);
}

__device__ __forceinline__ float2 resize_factor(const ResizeDesc& d, const float2* tabs, int ix, int iz)
{
    float2 e = make_float2(1.f, 0.f);
    if (d.t.tab >= 0) e = __ldg(&tabs[d.t.tab + ix]);
    if (d.t.ltab >= 0) e = cmul(e, __ldg(&tabs[d.t.ltab + iz]));
    bool zero = false;
    if (d.has_extra) extra_eval(d.extra, ix, iz, e, zero, tabs);
    return zero ? make_float2(0.f, 0.f) : e;
}

// RESIZE pass (RadResizeCore, sroptelm.cpp:3038-3337; OnlyLargerRange :4231).  The index
// arithmetic is tabulated per axis by the host (exact reference formulas); this kernel gathers,
// interpolates, applies the new-mesh point-wise factors and writes every new point (zero outside
// the window).  A thread produces two horizontally adjacent points: when their stencils start at
// most one old node apart, each stencil row is read once as three aligned float4 (6 complex).
__global__ void __launch_bounds__(256) resize_kernel(const ResizeLaunch p)
{
    const ResizeDesc& d = *reinterpret_cast<const ResizeDesc*>(reinterpret_cast<const char*>(p.gd) + blockIdx.z * p.bDesc);
    const float2* S[2] = {p.src[0] + blockIdx.z * p.bSrc, p.src[1] + blockIdx.z * p.bSrc};
    float2* D[2] = {p.dst[0] + blockIdx.z * p.bDst, p.dst[1] + blockIdx.z * p.bDst};
    const float2* tabs = p.tabs + blockIdx.z * p.bTab;
    const int ix0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix0 >= d.nxn || iz >= d.nzn) return;
    const bool two = ix0 + 1 < d.nxn;
    float2 out[2][2] = {{make_float2(0.f, 0.f), make_float2(0.f, 0.f)}, {make_float2(0.f, 0.f), make_float2(0.f, 0.f)}};
    const bool zin = (iz >= d.izStart) && (iz <= d.izEnd);
    const bool in0 = zin && (ix0 >= d.ixStart) && (ix0 <= d.ixEnd);
    const bool in1 = two && zin && (ix0 + 1 >= d.ixStart) && (ix0 + 1 <= d.ixEnd);
    if (in0 || in1) {
        const ResizeAxis az = load_axis(tabs, d.axz, iz);
        const ResizeAxis a0 = load_axis(tabs, d.axx, ix0);
        const ResizeAxis a1 = two ? load_axis(tabs, d.axx, ix0 + 1) : a0;
        if (d.only_larger) {
#pragma unroll
            for (int c = 0; c < 2; c++) {
                if (in0) out[0][c] = __ldg(&S[c][(size_t)az.st * d.nxo + a0.st]);
                if (in1) out[1][c] = __ldg(&S[c][(size_t)az.st * d.nxo + a1.st]);
            }
        } else {
            float wz[4], wx0[4], wx1[4];
            lagrange4(az.rel, wz);
            lagrange4(a0.rel, wx0);
            lagrange4(a1.rel, wx1);
            const int base = a0.st & ~1;
            const int o0 = a0.st - base, o1 = a1.st - base;
            const bool vec = p.vec_ok && in0 && in1 && (o1 >= o0) && (o1 <= 2) && (base + 6 <= d.nxo) && !d.has_pre;
            if (vec) {
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    const float2* __restrict__ o = S[c] + (size_t)az.st * d.nxo + base;
                    float2 f0[4][4], f1[4][4];
#pragma unroll
                    for (int dz = 0; dz < 4; dz++) {
                        const float4* r4 = reinterpret_cast<const float4*>(o + (size_t)dz * d.nxo);
                        float4 q0 = __ldg(r4), q1 = __ldg(r4 + 1), q2 = __ldg(r4 + 2);
                        float2 cc[6] = {make_float2(q0.x, q0.y), make_float2(q0.z, q0.w), make_float2(q1.x, q1.y),
                                        make_float2(q1.z, q1.w), make_float2(q2.x, q2.y), make_float2(q2.z, q2.w)};
#pragma unroll
                        for (int dx = 0; dx < 4; dx++) {
                            f0[dz][dx] = pick3(cc, o0, dx);
                            f1[dz][dx] = pick3(cc, o1, dx);
                        }
                    }
                    out[0][c] = interp_stencil(f0, wx0, wz, a0.rel, az.rel, a0.ir, az.ir);
                    out[1][c] = interp_stencil(f1, wx1, wz, a1.rel, az.rel, a1.ir, az.ir);
                }
            } else {
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    const ResizeDesc* pre = d.has_pre ? &d : nullptr;
                    if (in0) out[0][c] = resize_point(S[c] + (size_t)az.st * d.nxo + a0.st, d.nxo, wx0, wz, a0.rel,
                                                      az.rel, a0.ir, az.ir, pre, tabs, a0.st, az.st);
                    if (in1) out[1][c] = resize_point(S[c] + (size_t)az.st * d.nxo + a1.st, d.nxo, wx1, wz, a1.rel,
                                                      az.rel, a1.ir, az.ir, pre, tabs, a1.st, az.st);
                }
            }
        }
        if (d.has_pw) {
            if (in0) {
                float2 e = resize_factor(d, tabs, ix0, iz);
                out[0][0] = cmul(out[0][0], e);
                out[0][1] = cmul(out[0][1], e);
            }
            if (in1) {
                float2 e = resize_factor(d, tabs, ix0 + 1, iz);
                out[1][0] = cmul(out[1][0], e);
                out[1][1] = cmul(out[1][1], e);
            }
        }
    }
    const size_t o = (size_t)iz * d.nxn + ix0;
#pragma unroll
    for (int c = 0; c < 2; c++) {
        if (p.vec_ok && two && ((o & 1) == 0)) {
            __stcs(reinterpret_cast<float4*>(D[c] + o), make_float4(out[0][c].x, out[0][c].y, out[1][c].x, out[1][c].y));
        } else {
            __stcs(&D[c][o], out[0][c]);
            if (two) __stcs(&D[c][o + 1], out[1][c]);
        }
    }
}

// point-wise work folded in from a preceding element-wise pass, at old index (ix, iz); the same
// operations in the same order as pw_kernel
__device__ __forceinline__ float2 pre_factor(const ResizeDesc& d, const float2* tabs, int ix, int iz)
{
    float2 e = make_float2(1.f, 0.f);
    if (d.tp.tab >= 0) e = __ldg(&tabs[d.tp.tab + ix]);
    if (d.tp.ltab >= 0) e = cmul(e, __ldg(&tabs[d.tp.ltab + iz]));
    bool zero = false;
    if (d.has_pre_extra) extra_eval(d.pre_extra, ix, iz, e, zero, tabs);
    return zero ? make_float2(0.f, 0.f) : e;
}

// Tiled RESIZE pass: a CTA makes a TZ x TX tile of new points.  The old points under the tile's
// stencils are staged once in shared memory (with the folded point-wise work applied); the 4x4
// interpolation is separable, so the x interpolation of Re, Im and |E|^2 is done once per (old
// row, new column) and each new point combines four of those rows.  The operation order per new
// point is that of resize_kernel (x first, then z; same FMAs), so both kernels give identical
// results.  Points outside the window are written as zeros.
__global__ void __launch_bounds__(256) resize2_kernel(const ResizeLaunch p)
{
    const ResizeDesc& d = *reinterpret_cast<const ResizeDesc*>(reinterpret_cast<const char*>(p.gd) + blockIdx.z * p.bDesc);
    const float2* S[2] = {p.src[0] + blockIdx.z * p.bSrc, p.src[1] + blockIdx.z * p.bSrc};
    float2* D[2] = {p.dst[0] + blockIdx.z * p.bDst, p.dst[1] + blockIdx.z * p.bDst};
    const float2* tabs = p.tabs + blockIdx.z * p.bTab;
    constexpr int TX = SRWG_RESIZE_TX, TZ = SRWG_RESIZE_TZ;
    extern __shared__ float4 rsm[];
    const int OR = d.tile_or, OC = d.tile_oc;
    float4* wxs = rsm;                    // x weights per tile column
    float4* axs = wxs + TX;               // (st, ir, rel) per tile column
    float4* wzs = axs + TX;               // z weights per tile row
    float4* azs = wzs + TZ;
    float4* H = azs + TZ;                 // [comp][old row][tile column]: (Re, Im, |E|^2, any zero)
    float2* old = reinterpret_cast<float2*>(H + 2 * OR * TX);   // [comp][old row][old column]
    __shared__ int ext[4];
    const int tid = threadIdx.x;
    const int x0 = (blockIdx.x + p.tx0) * TX, z0 = (blockIdx.y + p.tz0) * TZ;
    const int xa = max(x0, (int)d.ixStart), xb = min(min(x0 + TX, d.nxn) - 1, (int)d.ixEnd);
    const int za = max(z0, (int)d.izStart), zb = min(min(z0 + TZ, d.nzn) - 1, (int)d.izEnd);
    if (xa > xb || za > zb) {
        if (d.skip_zero) return;
        for (int e = tid; e < TZ * TX; e += 256) {
            const int gi = x0 + (e & (TX - 1)), gj = z0 + e / TX;
            if (gi < d.nxn && gj < d.nzn) {
                const size_t o = (size_t)gj * d.nxn + gi;
                __stcs(&D[0][o], make_float2(0.f, 0.f));
                __stcs(&D[1][o], make_float2(0.f, 0.f));
            }
        }
        return;
    }
    if (tid == 0) { ext[0] = 1 << 30; ext[1] = -1; ext[2] = 1 << 30; ext[3] = -1; }
    __syncthreads();
    if (tid < TX) {
        const int i = x0 + tid;
        if (i >= xa && i <= xb) {
            const ResizeAxis a = load_axis(tabs, d.axx, i);
            float w[4];
            lagrange4(a.rel, w);
            wxs[tid] = make_float4(w[0], w[1], w[2], w[3]);
            axs[tid] = make_float4(__int_as_float(a.st), __int_as_float(a.ir), a.rel, 0.f);
            atomicMin(&ext[0], a.st);
            atomicMax(&ext[1], a.st);
        }
    } else if (tid >= 128 && tid < 128 + TZ) {
        const int j = z0 + tid - 128;
        if (j >= za && j <= zb) {
            const ResizeAxis a = load_axis(tabs, d.axz, j);
            float w[4];
            lagrange4(a.rel, w);
            wzs[tid - 128] = make_float4(w[0], w[1], w[2], w[3]);
            azs[tid - 128] = make_float4(__int_as_float(a.st), __int_as_float(a.ir), a.rel, 0.f);
            atomicMin(&ext[2], a.st);
            atomicMax(&ext[3], a.st);
        }
    }
    __syncthreads();
    const int ox0 = ext[0], oz0 = ext[2];
    const int nc = ext[1] - ox0 + 4, nr = ext[3] - oz0 + 4;     // <= OC, OR (host-computed maxima)
    // old tile of both components, with the folded point-wise work
    for (int e = tid; e < nr * nc; e += 256) {
        const int r = e / nc, c = e - r * nc;
        const int gx = ox0 + c, gz = oz0 + r;
        const size_t go = (size_t)gz * d.nxo + gx;
        float2 v0 = __ldg(&S[0][go]), v1 = __ldg(&S[1][go]);
        if (d.has_pre) {
            const float2 f = pre_factor(d, tabs, gx, gz);
            v0 = cmul(f, v0);
            v1 = cmul(f, v1);
        }
        old[r * OC + c] = v0;
        old[OR * OC + r * OC + c] = v1;
    }
    __syncthreads();
    // x interpolation per (old row, tile column)
    for (int e = tid; e < 2 * nr * TX; e += 256) {
        const int comp = e >= nr * TX;
        const int e2 = e - comp * nr * TX;
        const int r = e2 / TX, i = e2 & (TX - 1);
        const int gi = x0 + i;
        if (gi < xa || gi > xb) continue;
        const float4 w4 = wxs[i];
        const float w[4] = {w4.x, w4.y, w4.z, w4.w};
        const float2* row = old + comp * OR * OC + r * OC + (__float_as_int(axs[i].x) - ox0);
        float rx = 0.f, ry = 0.f, ri = 0.f;
        bool low = false;
#pragma unroll
        for (int dx = 0; dx < 4; dx++) {
            const float2 v = row[dx];
            low |= (v.x == 0.f) || (v.y == 0.f);
            rx = fmaf(w[dx], v.x, rx);
            ry = fmaf(w[dx], v.y, ry);
            ri = fmaf(w[dx], v.x * v.x + v.y * v.y, ri);
        }
        H[comp * OR * TX + r * TX + i] = make_float4(rx, ry, ri, low ? 1.f : 0.f);
    }
    __syncthreads();
    // new points: z interpolation, low-order fallback, amplitude correction, new-mesh factors
    for (int e = tid; e < TZ * TX; e += 256) {
        const int jj = e / TX, i = e & (TX - 1);
        const int gi = x0 + i, gj = z0 + jj;
        if (gi >= d.nxn || gj >= d.nzn) continue;
        float2 out[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        const bool inw = gi >= xa && gi <= xb && gj >= za && gj <= zb;
        if (!inw && d.skip_zero) continue;
        if (inw) {
            const float4 wz4 = wzs[jj], az = azs[jj], ax = axs[i];
            const float wz[4] = {wz4.x, wz4.y, wz4.z, wz4.w};
            const int r0 = __float_as_int(az.x) - oz0;
#pragma unroll
            for (int comp = 0; comp < 2; comp++) {
                const float4* h = H + comp * OR * TX + r0 * TX + i;
                float2 F = make_float2(0.f, 0.f);
                float FI = 0.f;
                bool low = false;
#pragma unroll
                for (int dz = 0; dz < 4; dz++) {
                    const float4 q = h[dz * TX];
                    low |= q.w != 0.f;
                    F.x = fmaf(wz[dz], q.x, F.x);
                    F.y = fmaf(wz[dz], q.y, F.y);
                    FI = fmaf(wz[dz], q.z, FI);
                }
                if (low) {
                    // bilinear on the 2x2 sub-cell (ir_x, ir_z) of the stencil (CheckForLowOrderInterp)
                    const int irx = __float_as_int(ax.y), irz = __float_as_int(az.y);
                    const float xr = ax.z, zr = az.z;
                    const float2* c0 = old + comp * OR * OC + (r0 + irz) * OC + (__float_as_int(ax.x) - ox0) + irx;
                    const float2 f00 = c0[0], f10 = c0[1], f01 = c0[OC], f11 = c0[OC + 1];
                    const float xz = xr * zr;
                    F.x = f00.x + (f10.x - f00.x) * xr + (f01.x - f00.x) * zr + (f00.x - f01.x - f10.x + f11.x) * xz;
                    F.y = f00.y + (f10.y - f00.y) * xr + (f01.y - f00.y) * zr + (f00.y - f01.y - f10.y + f11.y) * xz;
                    const float i00 = f00.x * f00.x + f00.y * f00.y, i10 = f10.x * f10.x + f10.y * f10.y;
                    const float i01 = f01.x * f01.x + f01.y * f01.y, i11 = f11.x * f11.x + f11.y * f11.y;
                    FI = i00 + (i10 - i00) * xr + (i01 - i00) * zr + (i00 - i01 - i10 + i11) * xz;
                }
                FI = FI > 0.f ? FI : 0.f;
                const float app = F.x * F.x + F.y * F.y;      // ImproveReAndIm
                if (app != 0.f) {
                    const float fac = amp_ratio(FI, app);
                    F.x *= fac;
                    F.y *= fac;
                }
                out[comp] = F;
            }
            if (d.has_pw) {
                const float2 f = resize_factor(d, tabs, gi, gj);
                out[0] = cmul(out[0], f);
                out[1] = cmul(out[1], f);
            }
        }
        const size_t o = (size_t)gj * d.nxn + gi;
        __stcs(&D[0][o], out[0]);
        __stcs(&D[1][o], out[1]);
    }
}

// ------------------------------------------------------------------------------------------------
// element-wise PW pass
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) pw_kernel(const PwLaunch p)
{
    const PwDesc& d = *reinterpret_cast<const PwDesc*>(reinterpret_cast<const char*>(p.gd) + blockIdx.z * p.bDesc);
    const float2* S[2] = {p.src[0] + blockIdx.z * p.bSrc, p.src[1] + blockIdx.z * p.bSrc};
    float2* D[2] = {p.dst[0] + blockIdx.z * p.bDst, p.dst[1] + blockIdx.z * p.bDst};
    const float2* tabs = p.tabs + blockIdx.z * p.bTab;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y;
    if (ix >= d.nx) return;
    float2 e = make_float2(1.f, 0.f);
    if (d.t.tab >= 0) e = __ldg(&tabs[d.t.tab + ix]);
    if (d.t.ltab >= 0) e = cmul(e, __ldg(&tabs[d.t.ltab + iz]));
    bool zero = false;
    if (d.has_extra) extra_eval(d.extra, ix, iz, e, zero, tabs);
    if (zero) e = make_float2(0.f, 0.f);
    const int ox = d.mirror_x ? d.nx - 1 - ix : ix;
    const int oz = d.mirror_z ? d.nz - 1 - iz : iz;
    const size_t i = (size_t)iz * d.nx + ix, o = (size_t)oz * d.nx + ox;
#pragma unroll
    for (int c = 0; c < 2; c++) __stcs(&D[c][o], cmul(e, __ldcs(&S[c][i])));
}

// ------------------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------------------
Line2Fn line2_kernel_ptr(int logn, bool cols, bool extra, int f1, int f2)
{
    switch (logn) {
    case 6: return extra ? line2e_get_6(cols, f1, f2) : line2_get_6(cols, f1, f2);
    case 7: return extra ? line2e_get_7(cols, f1, f2) : line2_get_7(cols, f1, f2);
    case 8: return extra ? line2e_get_8(cols, f1, f2) : line2_get_8(cols, f1, f2);
    case 9: return extra ? line2e_get_9(cols, f1, f2) : line2_get_9(cols, f1, f2);
    case 10: return extra ? line2e_get_10(cols, f1, f2) : line2_get_10(cols, f1, f2);
    case 11: return extra ? line2e_get_11(cols, f1, f2) : line2_get_11(cols, f1, f2);
    case 12: return extra ? line2e_get_12(cols, f1, f2) : line2_get_12(cols, f1, f2);
    case 13: return extra ? line2e_get_13(cols, f1, f2) : line2_get_13(cols, f1, f2);
    case 14: return extra ? line2e_get_14(cols, f1, f2) : line2_get_14(cols, f1, f2);
    default: return nullptr;
    }
}

Line2Fn linen_kernel_ptr(int N, bool cols, bool extra, int nt, bool inten)
{
#define SRWG_LINEN_CASE(M) if (N == M) return linen_get_##M(cols, extra, nt, inten);
    SRWG_LINEN_LENGTHS(SRWG_LINEN_CASE)
    SRWG_LINEN_POW2(SRWG_LINEN_CASE)
#undef SRWG_LINEN_CASE
    return nullptr;
}

cudaError_t launch_line(const LineLaunch& pin, cudaStream_t st)
{
    LineLaunch p = pin;
    dim3 grid((p.nlines + p.L - 1) / p.L, 2, p.nb > 1 ? p.nb : 1);
    if (p.nblk > 0) {
        // only the line blocks of the window (the others would write nothing)
        if (p.blk0 < 0 || p.blk0 + p.nblk > (int)grid.x) return cudaErrorInvalidValue;
        grid.x = p.nblk;
    } else {
        p.blk0 = 0;
    }
    size_t smem = (size_t)p.L * p.P * sizeof(float2);
    if (smem > SRWG_LINE_SMEM_MAX) return cudaErrorInvalidValue;
    if (attrs_needed(0)) {
        cudaFuncSetAttribute(line_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SRWG_LINE_SMEM_MAX);
        const int dirs[8][2] = {{1, 1}, {1, -1}, {-1, 1}, {-1, -1}, {1, 0}, {-1, 0}, {0, 1}, {0, -1}};
        for (int lg = 6; lg <= 14; lg++)
            for (int e = 0; e < 4; e++)
                for (int m = 0; m < 8; m++)
                    cudaFuncSetAttribute(line2_kernel_ptr(lg, e & 1, e >> 1, dirs[m][0], dirs[m][1]),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, SRWG_LINE_SMEM_MAX);
        for (int e = 0; e < 2; e++) {
            cudaFuncSetAttribute(lineg_get(e != 0), cudaFuncAttributeMaxDynamicSharedMemorySize, SRWG_LINE_SMEM_MAX);
            cudaFuncSetAttribute(lineg_e_get(e != 0), cudaFuncAttributeMaxDynamicSharedMemorySize, SRWG_LINE_SMEM_MAX);
        }
#define SRWG_LINEN_ATTR(M)                                                                                 \
        for (int e = 0; e < 10; e++)                                                                       \
            cudaFuncSetAttribute(linen_get_##M(e & 1, (e >> 1) & 1, 1 + ((e >> 2) & 1), e >= 8),           \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, SRWG_LINE_SMEM_MAX);
        SRWG_LINEN_LENGTHS(SRWG_LINEN_ATTR)
        SRWG_LINEN_POW2(SRWG_LINEN_ATTR)
#undef SRWG_LINEN_ATTR
    }
    if (p.d.out_int && p.v2 != 3) return cudaErrorInvalidValue;    // intensity passes: specialised kernels only
    if (p.v2 == 3) {
        const bool inten = p.d.out_int != 0;
        if (inten && (p.d.has_extra || (p.d.f1 && p.d.f2))) return cudaErrorInvalidValue;
        Line2Fn f = linen_kernel_ptr(p.N, p.d.axis != 0, p.d.has_extra != 0, (p.d.f1 && p.d.f2) ? 2 : 1, inten);
        if (f == nullptr || p.T * p.L > 512) return cudaErrorInvalidValue;
        if (inten) {
            grid.y = 1;                         // one CTA transforms both components of its lines
            // the first component's intensity of every point a thread stores, in shared memory
            // after the line slots
            smem += (size_t)linen_int_floats(p.N) * p.T * p.L * sizeof(float);
            if (smem > SRWG_LINE_SMEM_MAX) return cudaErrorInvalidValue;
        }
        // input tiles by bulk async copies: 16-byte aligned sources; rows are contiguous, columns
        // only when the row pass wrote them in blocks of exactly the tile's (even) width
        LineLaunch q = p;
        const bool aligned = ((((uintptr_t)p.src[0]) | ((uintptr_t)p.src[1])) & 15) == 0 && (p.bSrc & 1) == 0;
        q.bulk = aligned && (p.d.axis == 0 || (p.d.blk_in == p.L && (p.L & 1) == 0));
        f<<<grid, p.T * p.L, smem, st>>>(q);
    } else if (p.v2 == 2) {
        Line2Fn f = p.d.has_extra ? lineg_e_get(p.d.axis != 0) : lineg_get(p.d.axis != 0);
        if (p.T * p.L > 512) return cudaErrorInvalidValue;
        f<<<grid, p.T * p.L, smem, st>>>(p);
    } else if (p.v2) {
        int lg = 0;
        while ((1 << lg) < p.N) lg++;
        Line2Fn f = line2_kernel_ptr(lg, p.d.axis != 0, p.d.has_extra != 0, p.d.f1, p.d.f2);
        if (f == nullptr) return cudaErrorInvalidValue;
        f<<<grid, p.T * p.L, smem, st>>>(p);
    } else {
        line_kernel<<<grid, p.T * p.G, smem, st>>>(p);
    }
    return cudaGetLastError();
}

cudaError_t launch_resize(const ResizeLaunch& q, cudaStream_t st)
{
    ResizeLaunch p = q;
    p.vec_ok = ((q.d.nxo & 1) == 0) && ((q.d.nxn & 1) == 0) && ((q.bSrc & 1) == 0) && ((q.bDst & 1) == 0);
    for (int c = 0; c < 2; c++)
        p.vec_ok = p.vec_ok && ((((uintptr_t)q.src[c]) & 15) == 0) && ((((uintptr_t)q.dst[c]) & 15) == 0);
    if (p.d.tile_or > 0 && p.d.tile_oc > 0 && p.d.tile_or <= SRWG_RESIZE_OR_MAX && p.d.tile_oc <= SRWG_RESIZE_OC_MAX) {
        const size_t smem = (size_t)(2 * SRWG_RESIZE_TX + 2 * SRWG_RESIZE_TZ) * sizeof(float4) +
                            (size_t)2 * p.d.tile_or * SRWG_RESIZE_TX * sizeof(float4) +
                            (size_t)2 * p.d.tile_or * p.d.tile_oc * sizeof(float2);
        if (attrs_needed(1))
            cudaFuncSetAttribute(resize2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SRWG_LINE_SMEM_MAX);
        dim3 grid((p.d.nxn + SRWG_RESIZE_TX - 1) / SRWG_RESIZE_TX, (p.d.nzn + SRWG_RESIZE_TZ - 1) / SRWG_RESIZE_TZ,
                  p.nb > 1 ? p.nb : 1);
        ResizeLaunch q = p;
        if (p.ntx > 0 && p.ntz > 0) {
            // only the tiles of the window (the others would write nothing)
            if (p.tx0 < 0 || p.tz0 < 0 || p.tx0 + p.ntx > (int)grid.x || p.tz0 + p.ntz > (int)grid.y)
                return cudaErrorInvalidValue;
            grid.x = p.ntx;
            grid.y = p.ntz;
        } else {
            q.tx0 = q.tz0 = 0;
        }
        resize2_kernel<<<grid, 256, smem, st>>>(q);
        return cudaGetLastError();
    }
    dim3 blk(64, 4);
    const int nxh = (p.d.nxn + 1) / 2;
    dim3 grid((nxh + blk.x - 1) / blk.x, (p.d.nzn + blk.y - 1) / blk.y, p.nb > 1 ? p.nb : 1);
    resize_kernel<<<grid, blk, 0, st>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_pw(const PwLaunch& p, cudaStream_t st)
{
    dim3 blk(256);
    dim3 grid((p.d.nx + 255) / 256, p.d.nz, p.nb > 1 ? p.nb : 1);
    pw_kernel<<<grid, blk, 0, st>>>(p);
    return cudaGetLastError();
}

}  // namespace srwg
