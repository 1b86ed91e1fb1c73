// Power-of-two line pass templates (instantiated per line length in line2_*.cu).
#pragma once
#include "common.cuh"

namespace srwg {

// ------------------------------------------------------------------------------------------------
// LINE pass, power-of-two lines (N >= 64): every thread owns 16 points of its line.  The first
// FFT stage reads its butterfly inputs straight from global memory through the point-wise chain
// (coalesced: thread t reads t + T*m), the last stage writes straight to global memory through
// the output chain; intermediate stages exchange through shared memory padded by one point per
// 16 (conflict-free Stockham writes).  Complex adds and subtracts are packed FP32x2 instructions.  A second transform in the same pass (f1 -> f2) reads the
// first one's output from shared memory through the middle chain.
// ------------------------------------------------------------------------------------------------
#define PADI(p) ((p) + ((p) >> 4))

// IN: 0 shared, 1 shared through chain cin, 2 global through chain cin;  OUT: 0 shared, 1 global through chain cout
// N (line length), R (radix) and Ns (product of the radices already applied) are compile-time.
template <int N, int R, int NS, int DIR, int IN, int OUT, bool EXTRA>
__device__ __forceinline__ void stage16(float2* s, const float2* __restrict__ gin, float2* __restrict__ gout,
                                        int gstr, const OutMap& om, int t, int line, const Chain2& cin, const Chain2& cout,
                                        const float2* __restrict__ tw, bool active, bool has_lf, float2 lf,
                                        const float2* __restrict__ tabs, const PwOps* ex, int axis,
                                        int za0, int za1)
{
    constexpr int T = N / 16;
    constexpr int B = 16 / R;
    constexpr int NR = N / R;
    constexpr int TWS = N / (NS * R);
    float2 v[B][R];
    if (IN == 2) {
        // first stage from global memory: all 16 loads are issued before any dependent arithmetic
#pragma unroll
        for (int b = 0; b < B; b++)
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int p = t + T * b + r * NR;
                const int q = p ^ cin.xs;
                const bool in = active && q >= za0 && q <= za1;
                v[b][r] = in ? __ldcs(&gin[q * gstr]) : make_float2(0.f, 0.f);
            }
#pragma unroll
        for (int b = 0; b < B; b++)
#pragma unroll
            for (int r = 0; r < R; r++) v[b][r] = chain2_apply<EXTRA>(cin, t + T * b + r * NR, line, v[b][r], tabs, ex, axis);
        // NS == 1 for the first stage: no twiddles
    } else {
#pragma unroll
        for (int b = 0; b < B; b++) {
            const int j = t + T * b;
            const int k = j & (NS - 1);
            // twiddles W^(k r): W^k, W^2k, W^4k, W^8k from the table, the other powers as products
            float2 wp[4];
            if (NS > 1) {
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    if ((1 << e) < R) {
                        float2 w = __ldg(&tw[(k * TWS) << e]);
                        if (DIR < 0) w.y = -w.y;
                        wp[e] = w;
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int p = j + r * NR;
                float2 x = make_float2(0.f, 0.f);
                if (active) {
                    if (IN == 0) x = s[PADI(p)];
                    else x = chain2_apply<EXTRA>(cin, p, line, s[PADI(p ^ cin.xs)], tabs, ex, axis);
                }
                if (NS > 1 && r > 0) {
                    float2 w = make_float2(1.f, 0.f);
                    bool first = true;
#pragma unroll
                    for (int e = 0; e < 4; e++)
                        if (r & (1 << e)) { w = first ? wp[e] : cmul(w, wp[e]); first = false; }
                    x = cmul(x, w);
                }
                v[b][r] = x;
            }
        }
    }
    if (OUT == 0) __syncthreads();
#pragma unroll
    for (int b = 0; b < B; b++) {
        const int j = t + T * b;
        const int k = j & (NS - 1);
        dftR<R, DIR>(v[b], tw, N);
        const int base = (j / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int q = base + r * NS;
            if (active) {
                if (OUT == 0) {
                    s[PADI(q)] = v[b][r];
                } else {
                    const int i = q ^ cout.xinv;
                    float2 o = chain2_apply<EXTRA>(cout, i, line, v[b][r], tabs, ex, axis);
                    if (has_lf) o = cmul(lf, o);
                    __stcs(&gout[om.at(i)], o);
                }
            }
        }
    }
    if (OUT == 0) __syncthreads();
}

// one FFT of N = 2^LOGN points along the line: radix-16 stages, the last one of radix 2..16
template <int LOGN, int DIR, int IN, int OUT, bool EXTRA>
__device__ __forceinline__ void fftN(float2* s, const float2* __restrict__ gin, float2* __restrict__ gout,
                                     int gstr, const OutMap& om, int t, int line, const Chain2& cin, const Chain2& cout,
                                     const float2* __restrict__ tw, bool active, bool has_lf, float2 lf,
                                     const float2* __restrict__ tabs, const PwOps* ex, int axis, int za0,
                                     int za1)
{
    constexpr int N = 1 << LOGN;
    constexpr int NST = (LOGN + 3) / 4;
    constexpr int RL = 1 << (LOGN - 4 * (NST - 1));
    stage16<N, 16, 1, DIR, IN, 0, EXTRA>(s, gin, nullptr, gstr, om, t, line, cin, cout, tw, active, has_lf, lf, tabs, ex, axis, za0, za1);
    if constexpr (NST >= 3)
        stage16<N, 16, 16, DIR, 0, 0, EXTRA>(s, nullptr, nullptr, gstr, om, t, line, cin, cout, tw, active, has_lf, lf, tabs, ex, axis, za0, za1);
    if constexpr (NST >= 4)
        stage16<N, 16, 256, DIR, 0, 0, EXTRA>(s, nullptr, nullptr, gstr, om, t, line, cin, cout, tw, active, has_lf, lf, tabs, ex, axis, za0, za1);
    stage16<N, RL, (1 << (4 * (NST - 1))), DIR, 0, OUT, EXTRA>(s, nullptr, gout, gstr, om, t, line, cin, cout, tw, active,
                                                         has_lf, lf, tabs, ex, axis, za0, za1);
}

// EXTRA: the pass has non-separable point-wise work (circular masks, rectangular obstacles, the
// quartic part of the angular transfer function); a separate instantiation keeps its registers out
// of the common kernels
template <int LOGN, bool COLS, bool EXTRA, int D1, int D2>
__global__ void __launch_bounds__(1024, 1) line2_kernel(const LineLaunch p)
{
    constexpr int N = 1 << LOGN;
    constexpr int T = N / 16;
    extern __shared__ float2 sm[];
    // device-memory descriptor (read-only, cached); blockIdx.z = wavefront of a batched launch
    const LineDesc& d = *reinterpret_cast<const LineDesc*>(reinterpret_cast<const char*>(p.gd) + blockIdx.z * p.bDesc);
    const int comp = blockIdx.y;
    const float2* __restrict__ src = p.src[comp] + blockIdx.z * p.bSrc;
    float2* __restrict__ dst = p.dst[comp] + blockIdx.z * p.bDst;
    const int L = p.L, P = p.P, nl = p.nlines;
    const int tid = threadIdx.x;
    const int g = COLS ? (tid % L) : (tid / T);          // line of the tile
    const int t = COLS ? (tid / L) : (tid - g * T);      // thread within the line
    const int bx = blockIdx.x + p.blk0;                 // line block
    const int line = bx * L + g;
    bool active = line < nl;
    float2* s = sm + (size_t)g * P;
    // input: row-major, or (column pass after a row pass) blocks of blk_in columns stored together
    int gstr = COLS ? nl : 1;
    const float2* gin = COLS ? (src + line) : (src + (size_t)line * N);
    if (COLS && d.blk_in > 0) {
        gstr = d.blk_in;
        gin = src + (size_t)(line / d.blk_in) * N * d.blk_in + (line % d.blk_in);
    }
    const int oline = d.mirror_lines ? (nl - 1 - line) : line;
    float2* gout = COLS ? (dst + oline) : (dst + (size_t)oline * N);
    OutMap om;
    om.str = COLS ? nl : 1;
    om.lg = -1;
    om.bstr = 0;
    if (!COLS && d.blk_out > 0) {
        om.lg = 31 - __clz(d.blk_out);
        om.bstr = nl * d.blk_out;
        gout = dst + (size_t)oline * d.blk_out;
    }

    // input known to be zero outside lines [zl0, zl1] x points [za0, za1] (output of a resize that
    // wrote only its window): loads outside are skipped, all-zero tiles write zeros directly
    int za0 = 0, za1 = N - 1;
    if (d.zwin) {
        const int l0 = bx * L, l1 = min(l0 + L, nl) - 1;
        if (l1 < d.zl0 || l0 > d.zl1) {
            if (active && !d.zskip) {
#pragma unroll
                for (int m = 0; m < 16; m++) __stcs(&gout[om.at(t + T * m)], make_float2(0.f, 0.f));
            }
            return;
        }
        if (line < d.zl0 || line > d.zl1) {
            za0 = 1;
            za1 = 0;
            if (d.zskip) active = false;        // a zero line that nothing reads
        } else {
            za0 = d.za0;
            za1 = d.za1;
        }
    }
    const float2* tabs = p.tabs + blockIdx.z * p.bTab;
    const PwOps* ex = &d.extra;
    const int axis = d.axis;
    Chain2 pre = make_chain2(d.t_pre, 0, 0, d.f1_pre.rs, 0, N);
    Chain2 mid = make_chain2(d.t_mid, d.f1 ? d.f1_post.rs : 0, d.mirror_along, d.f2 ? d.f2_pre.rs : 0, d.has_extra, N);
    Chain2 fin = make_chain2(d.t_fin, d.f2 ? d.f2_post.rs : 0, 0, 0, 0, N);
    // product of the line factors of all chains of the pass, applied once at the store
    const bool has_lf = (d.t_pre.ltab >= 0) || (d.t_mid.ltab >= 0) || (d.t_fin.ltab >= 0);
    float2 lf = make_float2(1.f, 0.f);
    if (has_lf && active) {
        if (d.t_pre.ltab >= 0) lf = cmul(lf, __ldg(&tabs[d.t_pre.ltab + line]));
        if (d.t_mid.ltab >= 0) lf = cmul(lf, __ldg(&tabs[d.t_mid.ltab + line]));
        if (d.t_fin.ltab >= 0) lf = cmul(lf, __ldg(&tabs[d.t_fin.ltab + line]));
    }
    const float2* tw = p.tw;
    // D1, D2: directions of the first / second transform (0: none), fixed per instantiation so that
    // each kernel holds one code path (and its registers)
    if constexpr (D1 != 0 && D2 != 0) {
        fftN<LOGN, D1, 2, 0, EXTRA>(s, gin, nullptr, gstr, om, t, line, pre, mid, tw, active, has_lf, lf, tabs, ex, axis,
                                    za0, za1);
        fftN<LOGN, D2, 1, 1, EXTRA>(s, nullptr, gout, gstr, om, t, line, mid, fin, tw, active, has_lf, lf, tabs, ex,
                                    axis, za0, za1);
    } else if constexpr (D1 != 0) {
        fftN<LOGN, D1, 2, 1, EXTRA>(s, gin, gout, gstr, om, t, line, pre, mid, tw, active, has_lf, lf, tabs, ex, axis,
                                    za0, za1);
    } else {
        fftN<LOGN, D2, 2, 1, EXTRA>(s, gin, gout, gstr, om, t, line, mid, fin, tw, active, has_lf, lf, tabs, ex, axis,
                                    za0, za1);
    }
}

// kernel of a (COLS, EXTRA, f1, f2) combination
template <int LOGN, bool COLS, bool EXTRA>
Line2Fn line2_select(int f1, int f2)
{
    if (f1 > 0 && f2 > 0) return line2_kernel<LOGN, COLS, EXTRA, 1, 1>;
    if (f1 > 0 && f2 < 0) return line2_kernel<LOGN, COLS, EXTRA, 1, -1>;
    if (f1 < 0 && f2 > 0) return line2_kernel<LOGN, COLS, EXTRA, -1, 1>;
    if (f1 < 0 && f2 < 0) return line2_kernel<LOGN, COLS, EXTRA, -1, -1>;
    if (f1 > 0) return line2_kernel<LOGN, COLS, EXTRA, 1, 0>;
    if (f1 < 0) return line2_kernel<LOGN, COLS, EXTRA, -1, 0>;
    if (f2 > 0) return line2_kernel<LOGN, COLS, EXTRA, 0, 1>;
    if (f2 < 0) return line2_kernel<LOGN, COLS, EXTRA, 0, -1>;
    return nullptr;
}

}  // namespace srwg
