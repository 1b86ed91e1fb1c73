// Line pass for general (not power-of-two) FFT lengths N = 2^a 3^b 5^c 7^d (a >= 1), e.g. the
// 1280 .. 3584-point grids that resize factors such as 1.25 x 1.75 produce.  Same organisation as
// the power-of-two pass (line2.cuh): a CTA owns L whole lines in padded shared memory, the first
// Stockham stage reads global memory directly through the input chain, the last one writes global
// memory directly through the output chain (tables of the plan, per-line factor at the store),
// intermediate stages exchange through shared memory.  The radix schedule is the host's
// (radix_plan: 16/8/4/2 first, then 3, 5, 7) and runs at run time; every stage is a compile-time
// radix with at most ceil(16 / R) butterflies per thread (T >= N / 16 threads per line), compiled
// as a separate (not inlined) function so that each keeps its own registers.
#pragma once
#include <cstdio>
#include "common.cuh"

namespace srwg {

#define PADG(p) ((p) + ((p) >> 4))

// Every index is checked before its access; an out-of-range index is reported (printf) and the
// access skipped.  This checked form is the one validated on the GPU: an unchecked build of the same
// kernel raised an illegal-address error on its first run (96 x 80 mesh) although the checks never
// fire on any tested case, and the cause was not found.
__device__ __forceinline__ bool gok(bool cond, int code, int a, int b, int N, int NS, int R)
{
    if (!cond) printf("srwg general-length pass: index check %d failed (%d %d; N %d NS %d R %d)\n", code, a, b, N, NS, R);
    return cond;
}
#define GOK(cond, code, a, b) gok((cond), (code), (int)(a), (int)(b), N, NS, R)

struct GLine {
    int P;
    const float2* gin;
    float2* gout;
    int gstr;                // stride between the points of a line (elements)
    int line, axis;
    bool active;
    const float2* tabs;
    const PwOps* ex;
    bool has_lf;
    float2 lf;
};

// destination index of transform output q through an output chain (rotation rs1, then mirror)
__device__ __forceinline__ int chainG_dst(const ChainG& c, int q, int N)
{
    int k = q;
    if (c.rs1) { k = q + (N >> 1); if (k >= N) k -= N; }
    return c.mir ? (N - 1 - k) : k;
}

// one stage of radix R; IN: 0 shared, 1 shared through chain cin, 2 global through chain cin;
// OUT: 0 shared, 1 global through chain cout
template <int R, int DIR, int IN, int OUT, bool EXTRA>
__device__ __noinline__ void gstage(float2* s, const GLine& x, const ChainG& cin, const ChainG& cout,
                                    const float2* __restrict__ tw, int N, int NS, int t, int T)
{
    constexpr int MAXB = (16 + R - 1) / R;
    const int NR = N / R;
    const int tws = N / (NS * R);
    float2 v[MAXB][R];
    if (IN == 2) {
        // first stage from global memory: all loads issued before any dependent arithmetic
#pragma unroll
        for (int b = 0; b < MAXB; b++) {
            const int j = t + b * T;
            const bool ok = x.active && j < NR;
#pragma unroll
            for (int r = 0; r < R; r++) {
                int i;
                const int src = chainG_src(cin, j + r * NR, N, i);
                v[b][r] = (ok && GOK(src >= 0 && src < N, 1, src, j)) ? __ldcs(&x.gin[src * x.gstr])
                                                                      : make_float2(0.f, 0.f);
            }
        }
#pragma unroll
        for (int b = 0; b < MAXB; b++) {
            const int j = t + b * T;
            if (!(x.active && j < NR)) continue;
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int p = j + r * NR;
                int i;
                chainG_src(cin, p, N, i);
                v[b][r] = cmul(chainG_factor<EXTRA>(cin, p, i, x.line, x.tabs, x.ex, x.axis), v[b][r]);
            }
        }
    } else {
#pragma unroll
        for (int b = 0; b < MAXB; b++) {
            const int j = t + b * T;
            const bool ok = x.active && j < NR;
            const int k = NS > 1 ? j % NS : 0;
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int p = j + r * NR;
                float2 a = make_float2(0.f, 0.f);
                if (ok) {
                    if (IN == 0) {
                        if (GOK(PADG(p) < x.P, 2, p, j)) a = s[PADG(p)];
                    } else {
                        int i;
                        const int src = chainG_src(cin, p, N, i);
                        if (GOK(src >= 0 && PADG(src) < x.P, 3, src, j))
                            a = cmul(chainG_factor<EXTRA>(cin, p, i, x.line, x.tabs, x.ex, x.axis), s[PADG(src)]);
                    }
                    if (NS > 1 && r > 0) {
                        float2 w = GOK(k * tws * r < N, 4, k, tws) ? __ldg(&tw[k * tws * r]) : make_float2(1.f, 0.f);
                        if (DIR < 0) w.y = -w.y;
                        a = cmul(a, w);
                    }
                }
                v[b][r] = a;
            }
        }
    }
    if (OUT == 0) __syncthreads();
#pragma unroll
    for (int b = 0; b < MAXB; b++) {
        const int j = t + b * T;
        if (!(x.active && j < NR)) continue;
        dftR<R, DIR>(v[b], tw, N);
        const int k = NS > 1 ? j % NS : 0;
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int q = base + r * NS;
            if (OUT == 0) {
                if (GOK(q >= 0 && PADG(q) < x.P, 5, q, j)) s[PADG(q)] = v[b][r];
            } else {
                const int kk = chainG_dst(cout, q, N);
                if (!GOK(kk >= 0 && kk < N, 6, kk, q)) continue;
                int i;
                chainG_src(cout, kk, N, i);
                float2 o = cmul(chainG_factor<EXTRA>(cout, kk, i, x.line, x.tabs, x.ex, x.axis), v[b][r]);
                if (x.has_lf) o = cmul(x.lf, o);
                __stcs(&x.gout[kk * x.gstr], o);
            }
        }
    }
    if (OUT == 0) __syncthreads();
}

// one FFT along the line with the host's radix schedule; inMode 2: the first stage reads global
// memory through cin, 1: shared memory through cin; outMode 1: the last stage writes global memory
// through cout, 0: shared memory
template <int DIR, bool EXTRA>
__device__ __forceinline__ void gfft(float2* s, const GLine& x, const ChainG& cin, const ChainG& cout,
                                     const float2* __restrict__ tw, int N, const int* radix, int nst, int inMode,
                                     int outMode, int t, int T)
{
    // first stage: a power of two (the schedule puts them first)
    const int R0 = radix[0];
#define G_FIRST(RR)                                                                         \
    if (inMode == 2) gstage<RR, DIR, 2, 0, EXTRA>(s, x, cin, cout, tw, N, 1, t, T);         \
    else gstage<RR, DIR, 1, 0, EXTRA>(s, x, cin, cout, tw, N, 1, t, T);
    if (R0 == 16) { G_FIRST(16) } else if (R0 == 8) { G_FIRST(8) } else if (R0 == 4) { G_FIRST(4) } else { G_FIRST(2) }
#undef G_FIRST
    int NS = R0;
    for (int st = 1; st < nst; st++) {
        const int R = radix[st];
        const bool last = st == nst - 1;
#define G_STAGE(RR)                                                                         \
    if (last && outMode == 1) gstage<RR, DIR, 0, 1, EXTRA>(s, x, cin, cout, tw, N, NS, t, T); \
    else gstage<RR, DIR, 0, 0, EXTRA>(s, x, cin, cout, tw, N, NS, t, T);
        switch (R) {
        case 16: G_STAGE(16) break;
        case 8: G_STAGE(8) break;
        case 4: G_STAGE(4) break;
        case 2: G_STAGE(2) break;
        case 3: G_STAGE(3) break;
        case 5: G_STAGE(5) break;
        default: G_STAGE(7) break;
        }
#undef G_STAGE
        NS *= R;
    }
}

template <bool COLS, bool EXTRA>
__global__ void __launch_bounds__(512, 1) lineg_kernel(const LineLaunch p)
{
    extern __shared__ float2 smg[];
    const LineDesc& d = *reinterpret_cast<const LineDesc*>(reinterpret_cast<const char*>(p.gd) + blockIdx.z * p.bDesc);
    const int comp = blockIdx.y;
    const float2* __restrict__ src = p.src[comp] + blockIdx.z * p.bSrc;
    float2* __restrict__ dst = p.dst[comp] + blockIdx.z * p.bDst;
    const int N = p.N, T = p.T, L = p.L, nl = p.nlines;
    const int tid = threadIdx.x;
    const int g = COLS ? (tid % L) : (tid / T);
    const int t = COLS ? (tid / L) : (tid - g * T);
    GLine x;
    x.line = (blockIdx.x + p.blk0) * L + g;
    x.active = x.line < nl;
    x.axis = d.axis;
    float2* s = smg + (size_t)g * p.P;
    x.P = p.P;
    x.gstr = COLS ? nl : 1;
    x.gin = COLS ? (src + x.line) : (src + (size_t)x.line * N);
    const int oline = d.mirror_lines ? (nl - 1 - x.line) : x.line;
    x.gout = COLS ? (dst + oline) : (dst + (size_t)oline * N);
    x.tabs = p.tabs + blockIdx.z * p.bTab;
    x.ex = &d.extra;
    ChainG pre, mid, fin;
    pre.rs1 = 0; pre.mir = 0; pre.rs2 = d.f1_pre.rs; pre.tab = (int)d.t_pre.tab; pre.extra = 0;
    mid.rs1 = d.f1 ? d.f1_post.rs : 0; mid.mir = d.mirror_along; mid.rs2 = d.f2 ? d.f2_pre.rs : 0;
    mid.tab = (int)d.t_mid.tab; mid.extra = EXTRA ? d.has_extra : 0;
    fin.rs1 = d.f2 ? d.f2_post.rs : 0; fin.mir = 0; fin.rs2 = 0; fin.tab = (int)d.t_fin.tab; fin.extra = 0;
    x.has_lf = (d.t_pre.ltab >= 0) || (d.t_mid.ltab >= 0) || (d.t_fin.ltab >= 0);
    x.lf = make_float2(1.f, 0.f);
    if (x.has_lf && x.active) {
        if (d.t_pre.ltab >= 0) x.lf = cmul(x.lf, __ldg(&x.tabs[d.t_pre.ltab + x.line]));
        if (d.t_mid.ltab >= 0) x.lf = cmul(x.lf, __ldg(&x.tabs[d.t_mid.ltab + x.line]));
        if (d.t_fin.ltab >= 0) x.lf = cmul(x.lf, __ldg(&x.tabs[d.t_fin.ltab + x.line]));
    }
    const float2* tw = p.tw;
    if (d.f1 && d.f2) {
        if (d.f1 > 0) gfft<1, EXTRA>(s, x, pre, mid, tw, N, p.radix, p.nst, 2, 0, t, T);
        else gfft<-1, EXTRA>(s, x, pre, mid, tw, N, p.radix, p.nst, 2, 0, t, T);
        if (d.f2 > 0) gfft<1, EXTRA>(s, x, mid, fin, tw, N, p.radix, p.nst, 1, 1, t, T);
        else gfft<-1, EXTRA>(s, x, mid, fin, tw, N, p.radix, p.nst, 1, 1, t, T);
    } else if (d.f1) {
        if (d.f1 > 0) gfft<1, EXTRA>(s, x, pre, mid, tw, N, p.radix, p.nst, 2, 1, t, T);
        else gfft<-1, EXTRA>(s, x, pre, mid, tw, N, p.radix, p.nst, 2, 1, t, T);
    } else {
        if (d.f2 > 0) gfft<1, EXTRA>(s, x, mid, fin, tw, N, p.radix, p.nst, 2, 1, t, T);
        else gfft<-1, EXTRA>(s, x, mid, fin, tw, N, p.radix, p.nst, 2, 1, t, T);
    }
}

}  // namespace srwg
