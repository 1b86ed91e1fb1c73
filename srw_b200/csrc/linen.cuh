// Line pass for general FFT lengths N = 2^a 3^b 5^c 7^d (a >= 1), specialised per length: the 1280 ..
// 7168-point grids that resize factors such as 1.25, 1.5 or 1.75 produce.  Same organisation as the
// power-of-two pass (line2.cuh): a CTA owns L whole lines in padded shared memory, the first
// Stockham stage reads global memory directly through the input chain, the last one writes global
// memory directly through the output chain (tables of the plan, per-line factor at the store),
// intermediate stages exchange through shared memory.  N, the radix schedule (radix-16 stages, one
// 8/4/2 stage, then 3, 5, 7), the threads per line (T = ceil(N/16)) and every index are
// compile-time; a stage of radix R gives each thread ceil(N/R / T) butterflies.  Inverse transforms
// are forward transforms of the conjugated line, conjugated back (conj(DFT(conj x)) = IDFT x), so one
// instantiation serves both directions.  The centring rotation (k + N/2 mod N) and the mirror
// (N - 1 - k) are an add and a compare.
#pragma once
#include "common.cuh"

namespace srwg {

#define PADN(p) ((p) + ((p) >> 4))

// ------------------------------------------------------------------------------------------------
// bulk async copies into shared memory, completion through an mbarrier (one per CTA, phase 0)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(uint64_t* bar, unsigned bytes)
{
    asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }" ::"r"(smem_addr(bar)),
                 "r"(bytes) : "memory");
}
// global -> shared, `bytes` a multiple of 16, both addresses 16-byte aligned
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}
// non-blocking test of the phase of parity `phase` (try_wait would suspend the thread for a
// hardware-defined time, which would make an iteration limit meaningless)
__device__ __forceinline__ bool mbar_try(uint64_t* bar, unsigned phase)
{
    unsigned ok;
    asm volatile("{ .reg .pred p; mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                 : "=r"(ok) : "r"(smem_addr(bar)), "r"(phase) : "memory");
    return ok != 0;
}
// waits for the phase of parity `phase` at most `limit` tries (32 ns apart); on giving up it counts
// the event in *status and waits (at most 2^24 more tries, about a second) for the copies still in
// flight, so that none lands after the CTA has left.
// Returns false when any thread of the CTA gave up (the CTA then skips its work as a whole).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned phase, long long limit, int* status)
{
    long long it = 0;
    bool done = mbar_try(bar, phase);
    while (!done && ++it < limit) {
        __nanosleep(32);
        done = mbar_try(bar, phase);
    }
    const bool gave_up = !done;
    if (gave_up) {
        if (status) atomicAdd(status, 1);
        long long k = 0;
        while (!mbar_try(bar, phase) && ++k < (1ll << 24)) __nanosleep(64);
    }
    return !__syncthreads_or(gave_up);
}

// compile-time radix schedule of N
struct NSched {
    int n;
    int r[SRWG_MAX_STAGES];
};
__host__ __device__ constexpr NSched nsched(int N)
{
    NSched s{0, {0}};
    int m = N, p2 = 0;
    while (m % 2 == 0) { m /= 2; p2++; }
    while (p2 >= 4) { s.r[s.n++] = 16; p2 -= 4; }
    if (p2 > 0) s.r[s.n++] = 1 << p2;
    while (m % 3 == 0) { s.r[s.n++] = 3; m /= 3; }
    while (m % 5 == 0) { s.r[s.n++] = 5; m /= 5; }
    while (m % 7 == 0) { s.r[s.n++] = 7; m /= 7; }
    if (m != 1) s.n = -1;
    return s;
}
__host__ __device__ constexpr int nsched_ns(int N, int i)
{
    NSched s = nsched(N);
    int ns = 1;
    for (int k = 0; k < i; k++) ns *= s.r[k];
    return ns;
}
template <int N> struct NPlan {
    static constexpr NSched s = nsched(N);
    static constexpr int T = (N + 15) / 16;
};
__host__ __device__ constexpr int NSched_last(int N) { return nsched(N).r[nsched(N).n - 1]; }

// (k + N/2) mod N
template <int N> __device__ __forceinline__ int rot_n(int k)
{
    const int m = k + N / 2;
    return m >= N ? m - N : m;
}
// source index of destination k through a chain (rotation rs2, mirror, rotation rs1); i: the index
// at which the non-separable work is evaluated
template <int N> __device__ __forceinline__ int chain_src_n(const ChainG& c, int k, int& i)
{
    const int m = c.rs2 ? rot_n<N>(k) : k;
    i = c.mir ? (N - 1 - m) : m;
    return c.rs1 ? rot_n<N>(i) : i;
}
// destination of transform output q through an output chain (rotation rs1, then mirror)
template <int N> __device__ __forceinline__ int chain_dst_n(const ChainG& c, int q)
{
    const int k = c.rs1 ? rot_n<N>(q) : q;
    return c.mir ? (N - 1 - k) : k;
}

// factor of the non-separable point-wise work at kernel index (i, j) (0 where it zeroes the point);
// out of line: such passes are rare, and inlining it at every point of every stage multiplies the
// kernels' code size
static __device__ __noinline__ float2 linen_extra(const PwOps* ex, int i, int j, const float2* tabs)
{
    bool zero = false;
    float2 f = make_float2(1.f, 0.f);
    extra_eval(*ex, i, j, f, zero, tabs);
    return zero ? make_float2(0.f, 0.f) : f;
}

// chain factor at destination k (evaluation index i): the along-line table and, in EXTRA kernels,
// the non-separable work
template <bool EXTRA>
__device__ __forceinline__ float2 factor_n(const ChainG& c, int k, int i, int line, const float2* tabs,
                                           const PwOps* ex, int axis)
{
    float2 f = c.tab >= 0 ? __ldg(&tabs[c.tab + k]) : make_float2(1.f, 0.f);
    if (EXTRA && c.extra) f = cmul(f, linen_extra(ex, axis == 0 ? i : line, axis == 0 ? line : i, tabs));
    return f;
}

// Per-thread view of its line: global input and output, the plan's tables, the line factor.
struct NLine {
    const float2* gin;      // input line (point k at gin[k * gstr])
    int gstr;
    float2* gout;           // output line (point k at gout[om.at(k)])
    OutMap om;
    const float2* tabs;
    const PwOps* ex;
    int line, axis;
    bool store;             // the line exists (inactive threads of the last tile compute on a copy of
                            // the last line and store nothing)
    bool has_lf;
    float2 lf;
    int za0, za1;           // input points outside [za0, za1] are zero
    const float2* sin;      // bulk-copied input tile: point k of the line at sin[k * sst]
    int sst;
    float iscale;           // intensity passes: factor of the stored intensity
};

// padded shared-memory address of point p, and its separable form for a per-thread base plus a
// compile-time step (exact when the step is a multiple of 16 and the base's low bits carry nothing)
__device__ __forceinline__ float2* spad(float2* s, int p) { return s + PADN(p); }
template <int STEP> __host__ __device__ constexpr int pstep() { return STEP + STEP / 16; }

// the evaluation index of destination k through chain c (for the non-separable work)
template <int N> __device__ __forceinline__ int chain_eval_n(const ChainG& c, int k)
{
    const int m = c.rs2 ? rot_n<N>(k) : k;
    return c.mir ? (N - 1 - m) : m;
}

// the chain's factors at destinations p = j + r NR of butterfly round b (v *= tab[p] (and the
// non-separable work)); rounds beyond the last butterfly (PART) are left alone
template <int N, int R, int NR, int T, int B, bool PART, bool EXTRA>
__device__ __forceinline__ void apply_factors(float2 (&v)[B][R], const NLine& x, const ChainG& c, int t)
{
    if (c.tab >= 0) {
        const float2* tb = x.tabs + c.tab + t;
#pragma unroll
        for (int b = 0; b < B; b++)
#pragma unroll
            for (int r = 0; r < R; r++)
                if (!PART || b < B - 1 || t + T * b < NR) v[b][r] = cmul(__ldg(&tb[T * b + r * NR]), v[b][r]);
    }
    if (EXTRA && c.extra) {
#pragma unroll
        for (int b = 0; b < B; b++)
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int p = t + T * b + r * NR;
                if (!PART || b < B - 1 || t + T * b < NR) {
                    const int i = chain_eval_n<N>(c, p);
                    v[b][r] = cmul(linen_extra(x.ex, x.axis == 0 ? i : x.line, x.axis == 0 ? x.line : i, x.tabs),
                                   v[b][r]);
                }
            }
    }
}

template <int B, int R> __device__ __forceinline__ void conj_all(float2 (&v)[B][R])
{
#pragma unroll
    for (int b = 0; b < B; b++)
#pragma unroll
        for (int r = 0; r < R; r++) v[b][r].y = -v[b][r].y;
}

// One Stockham stage of radix R (NS: product of the radices applied before it).  IN: 0 shared memory,
// 1 shared memory through chain cin (first stage of the second transform), 2 global memory through
// chain cin; OUT: 0 shared memory, 1 global memory through chain cout.  Inverse transforms (cj < 0)
// conjugate the inputs of their first stage after the chain and the outputs of their last stage
// before the chain.
// intensity of the points a thread stores in the last stage, carried from the first component's
// transform to the second one's (OUTI passes)
template <int N> struct IAcc {
    static constexpr int R = NSched_last(N);
    static constexpr int B = (N / R + NPlan<N>::T - 1) / NPlan<N>::T;
    // in shared memory (registers would halve the CTAs per SM): value (b, r) of thread tid at
    // v[(b R + r) nt + tid], nt threads per CTA (consecutive threads, consecutive words)
    float* v;
    int nt, tid;
    __device__ __forceinline__ float& at(int b, int r) const { return v[(b * R + r) * nt + tid]; }
};

template <int N, int R, int NS, int IN, int OUT, bool FIRST, bool LAST, bool EXTRA, int OUTI = 0>
__device__ __forceinline__ void nstage(float2* s, const NLine& x, const ChainG& cin, const ChainG& cout, float cj,
                                       const float2* __restrict__ tw, int t, IAcc<N>* acc = nullptr)
{
    constexpr int T = NPlan<N>::T;
    constexpr int NR = N / R;
    constexpr int B = (NR + T - 1) / T;              // butterflies per thread
    constexpr bool PART = (NR % T) != 0;             // the last round has idle threads
    constexpr int TWS = N / (NS * R);
    float2 v[B][R];
    if (IN == 2 || IN == 3) {
        // first stage from global memory (IN 2: all loads issued before any dependent arithmetic) or
        // from the bulk-copied input tile in shared memory (IN 3); the source of destination p is p,
        // p rotated by N/2 (a permutation of the radix index: R is even here), or the general map
        // with the mirror
        const bool rot = cin.rs1 != cin.rs2;
#pragma unroll
        for (int b = 0; b < B; b++) {
            const int j = t + T * b;
            const bool okj = !PART || b < B - 1 || j < NR;
#pragma unroll
            for (int r = 0; r < R; r++) {
                int q;
                if (!cin.mir) {
                    const int rr = (R % 2 == 0 && rot) ? (r + R / 2) % R : r;
                    q = j + rr * NR;
                    if (R % 2 != 0 && rot) q = rot_n<N>(q);
                } else {
                    int i;
                    q = chain_src_n<N>(cin, j + r * NR, i);
                }
                const bool in = okj && q >= x.za0 && q <= x.za1;
                if (IN == 2) v[b][r] = in ? __ldcs(&x.gin[q * x.gstr]) : make_float2(0.f, 0.f);
                else v[b][r] = in ? x.sin[q * x.sst] : make_float2(0.f, 0.f);
            }
        }
        apply_factors<N, R, NR, T, B, PART, EXTRA>(v, x, cin, t);
        if (cj < 0.f) conj_all(v);
        // NS == 1 for the first stage: no twiddles
    } else {
#pragma unroll
        for (int b = 0; b < B; b++) {
            const int j = t + T * b;
            const bool okj = !PART || b < B - 1 || j < NR;
            if (okj) {
                if (IN == 0) {
                    if constexpr (NR % 16 == 0) {
                        const float2* sj = spad(s, j);
#pragma unroll
                        for (int r = 0; r < R; r++) v[b][r] = sj[r * pstep<NR>()];
                    } else {
#pragma unroll
                        for (int r = 0; r < R; r++) v[b][r] = *spad(s, j + r * NR);
                    }
                } else {
#pragma unroll
                    for (int r = 0; r < R; r++) {
                        int i;
                        v[b][r] = *spad(s, chain_src_n<N>(cin, j + r * NR, i));
                    }
                }
            } else {
#pragma unroll
                for (int r = 0; r < R; r++) v[b][r] = make_float2(0.f, 0.f);
            }
        }
        if (IN == 1) {
            apply_factors<N, R, NR, T, B, PART, EXTRA>(v, x, cin, t);
            if (cj < 0.f) conj_all(v);
        }
        if (NS > 1) {
            // twiddles W^(k r), k = j mod NS: the table powers W^k, W^2k, W^4k, W^8k and their products
#pragma unroll
            for (int b = 0; b < B; b++) {
                const int j = t + T * b;
                const int k = j % NS;
                const bool okj = !PART || b < B - 1 || j < NR;
                float2 wp[4];
#pragma unroll
                for (int e = 0; e < 4; e++)
                    if ((1 << e) < R) wp[e] = okj ? __ldg(&tw[(k * TWS) << e]) : make_float2(1.f, 0.f);
#pragma unroll
                for (int r = 1; r < R; r++) {
                    float2 w = make_float2(1.f, 0.f);
                    bool first = true;
#pragma unroll
                    for (int e = 0; e < 4; e++)
                        if (r & (1 << e)) { w = first ? wp[e] : cmul(w, wp[e]); first = false; }
                    v[b][r] = cmul(v[b][r], w);
                }
            }
        }
    }
    if (OUT == 0) __syncthreads();
#pragma unroll
    for (int b = 0; b < B; b++) dftR<R, 1>(v[b], tw, N);
    if (LAST && cj < 0.f) conj_all(v);
    if (OUT == 0) {
#pragma unroll
        for (int b = 0; b < B; b++) {
            const int j = t + T * b;
            if (!PART || b < B - 1 || j < NR) {
                const int k = NS > 1 ? j % NS : 0;
                const int base = (j - k) * R + k;
                if constexpr (NS % 16 == 0) {
                    float2* sb = spad(s, base);
#pragma unroll
                    for (int r = 0; r < R; r++) sb[r * pstep<NS>()] = v[b][r];
                } else if constexpr (NS == 1 && R == 16) {
                    float2* sb = s + 17 * j;
#pragma unroll
                    for (int r = 0; r < R; r++) sb[r] = v[b][r];
                } else {
#pragma unroll
                    for (int r = 0; r < R; r++) *spad(s, base + r * NS) = v[b][r];
                }
            }
        }
        __syncthreads();
    } else {
        // last stage (NS R == N, so q = j + r NS): the destination is q, q rotated by N/2 (for an even
        // radix a permutation of r), or the general map with the mirror; factors and the line factor,
        // then the store
        const bool rot = cout.rs1 != 0;
#pragma unroll
        for (int b = 0; b < B; b++) {
            const int j = t + T * b;
            if (!(!PART || b < B - 1 || j < NR)) continue;
#pragma unroll
            for (int r = 0; r < R; r++) {
                int kk;
                if (!cout.mir) {
                    const int rr = (R % 2 == 0 && rot) ? (r + R / 2) % R : r;
                    kk = j + rr * NS;
                    if (R % 2 != 0 && rot) kk = rot_n<N>(kk);
                } else {
                    kk = chain_dst_n<N>(cout, j + r * NS);
                }
                float2 o = v[b][r];
                if (cout.tab >= 0) o = cmul(__ldg(&x.tabs[cout.tab + kk]), o);
                if (EXTRA && cout.extra) {
                    const int i = chain_eval_n<N>(cout, kk);
                    o = cmul(linen_extra(x.ex, x.axis == 0 ? i : x.line, x.axis == 0 ? x.line : i, x.tabs), o);
                }
                if (x.has_lf) o = cmul(x.lf, o);
                if constexpr (OUTI == 0) {
                    if (x.store) __stcs(&x.gout[x.om.at(kk)], o);
                } else if constexpr (OUTI == 1) {
                    acc->at(b, r) = o.x * o.x + o.y * o.y;           // first component
                } else {
                    const float I = (acc->at(b, r) + o.x * o.x + o.y * o.y) * x.iscale;
                    if (x.store) __stcs(reinterpret_cast<float*>(x.gout) + x.om.at(kk), I);
                }
            }
        }
    }
}

// one transform along the line with the compile-time schedule of N; INM: mode of the first stage's
// input (1 shared through cin, 2 global through cin, 3 the bulk-copied input tile through cin), OUTM:
// of the last stage's output (0 shared, 1 global through cout)
template <int N, int INM, int OUTM, bool EXTRA, int OUTI = 0>
__device__ __forceinline__ void fft_n(float2* s, const NLine& x, const ChainG& cin, const ChainG& cout, float cj,
                                      const float2* __restrict__ tw, int t, IAcc<N>* acc = nullptr)
{
    constexpr NSched S = NPlan<N>::s;
    static_assert(S.n >= 2 && S.n <= 8, "radix schedule");
#define SRWG_NSTAGE(I)                                                                                          \
    if constexpr (S.n > (I))                                                                                    \
        nstage<N, S.r[(I) < S.n ? (I) : 0], nsched_ns(N, (I)), (I) == 0 ? INM : 0, (I) == S.n - 1 ? OUTM : 0,   \
               (I) == 0, (I) == S.n - 1, EXTRA, (I) == S.n - 1 ? OUTI : 0>(s, x, cin, cout, cj, tw, t, acc);
    SRWG_NSTAGE(0) SRWG_NSTAGE(1) SRWG_NSTAGE(2) SRWG_NSTAGE(3)
    SRWG_NSTAGE(4) SRWG_NSTAGE(5) SRWG_NSTAGE(6) SRWG_NSTAGE(7)
#undef SRWG_NSTAGE
}

// NT: transforms in the pass (1 or 2); their directions come from the descriptor.  Passes with one
// transform and no non-separable work run at two 512-thread CTAs per SM (64 registers per thread,
// measured: at most a few spilled words); the others keep 128 registers (their state spills heavily
// at 64).
// The pass for one component of the CTA's lines.  OUTI 0: the component's field is written;
// 1 / 2: the first / second component of an intensity pass (the intensity of the points each thread
// stores is carried in `acc` and written after the second).  `phase`: parity of the bulk-copy
// mbarrier use.  Returns false when the CTA gave its work up (a bounded wait ran out).
template <int N, bool COLS, bool EXTRA, int NT, int OUTI>
__device__ __forceinline__ bool linen_body(const LineLaunch& p, int comp, IAcc<N>* acc, uint64_t* barp, unsigned phase)
{
    constexpr int T = NPlan<N>::T;
    extern __shared__ __align__(16) float2 smn[];
    const LineDesc& d = *reinterpret_cast<const LineDesc*>(reinterpret_cast<const char*>(p.gd) + blockIdx.z * p.bDesc);
    const float2* __restrict__ src = p.src[comp] + blockIdx.z * p.bSrc;
    // intensity passes write floats (element stride bDst in floats) through dst[0]: the output
    // offsets below are in elements of the output type
    float2* __restrict__ dst = p.dst[comp] + blockIdx.z * p.bDst;
    float* __restrict__ fdst = reinterpret_cast<float*>(p.dst[0]) + blockIdx.z * p.bDst;
    const int L = p.L, P = p.P, nl = p.nlines;
    const int tid = threadIdx.x;
    const int g = COLS ? (tid % L) : (tid / T);          // line of the tile
    const int t = COLS ? (tid / L) : (tid - g * T);      // thread within the line
    const int bx = blockIdx.x + p.blk0;                 // line block
    const int line0 = bx * L + g;
    NLine x;
    x.store = line0 < nl;
    const int line = x.store ? line0 : nl - 1;           // inactive threads work on the last line
    x.line = line;
    x.axis = d.axis;
    float2* s = smn + (size_t)g * P;
    x.gstr = COLS ? nl : 1;
    x.gin = COLS ? (src + line) : (src + (size_t)line * N);
    if (COLS && d.blk_in > 0) {
        x.gstr = d.blk_in;
        x.gin = src + (size_t)(line / d.blk_in) * N * d.blk_in + (line % d.blk_in);
    }
    const int oline = d.mirror_lines ? (nl - 1 - line) : line;
    size_t obase = COLS ? (size_t)oline : (size_t)oline * N;
    x.om.str = COLS ? nl : 1;
    x.om.lg = -1;
    x.om.bstr = 0;
    if (!COLS && d.blk_out > 0) {
        x.om.lg = 31 - __clz(d.blk_out);
        x.om.bstr = nl * d.blk_out;
        obase = (size_t)oline * d.blk_out;
    }
    if (COLS && OUTI && d.blk_out > 0) {
        // the intensity in blocks of blk_out columns: a tile of blk_out columns writes one
        // contiguous piece
        x.om.str = d.blk_out;
        obase = (size_t)(oline / d.blk_out) * N * d.blk_out + (oline % d.blk_out);
    }
    x.gout = OUTI ? reinterpret_cast<float2*>(fdst + obase) : dst + obase;
    x.za0 = 0;
    x.za1 = N - 1;
    if (d.zwin) {
        const int l0 = bx * L, l1 = min(l0 + L, nl) - 1;
        if (l1 < d.zl0 || l0 > d.zl1) {
            // the whole tile is zero: so is its transform
            if (x.store && OUTI == 0 && !d.zskip)
                for (int m = t; m < N; m += T) __stcs(&x.gout[x.om.at(m)], make_float2(0.f, 0.f));
            if (x.store && OUTI == 2)
                for (int m = t; m < N; m += T) __stcs(reinterpret_cast<float*>(x.gout) + x.om.at(m), 0.f);
            return true;
        }
        if (line < d.zl0 || line > d.zl1) {
            x.za0 = 1;
            x.za1 = 0;
            if (d.zskip && OUTI == 0) x.store = false;      // a zero line that nothing reads
        } else {
            x.za0 = d.za0;
            x.za1 = d.za1;
        }
    }
    x.tabs = p.tabs + blockIdx.z * p.bTab;
    x.ex = &d.extra;
    x.sin = nullptr;
    x.sst = 1;
    if (p.bulk) {
        // the tile's input arrives in shared memory by bulk async copies (thread 0 issues them):
        // rows: each line's nonzero window [za0, za1] (rounded out to even / odd ends: 16-byte pieces)
        // into its own slot (line g at g P); columns: the column block (the tile's L columns stored
        // together by the row pass) over the nonzero rows, as one piece (point k of column g at k L + g)
        uint64_t& bar = *barp;
        if (tid == 0) {
            if (phase == 0) mbar_init(&bar);
            unsigned bytes = 0;
            if (COLS) {
                if (x.za0 <= x.za1) bytes = (unsigned)((x.za1 - x.za0 + 1) * L * sizeof(float2));
            } else {
                for (int gg = 0; gg < L; gg++) {
                    const int ln = min(bx * L + gg, nl - 1);
                    const bool inl = !d.zwin || (ln >= d.zl0 && ln <= d.zl1);
                    const int lo = d.zwin ? (d.za0 & ~1) : 0, hi = d.zwin ? (d.za1 | 1) : N - 1;
                    if (inl && lo <= hi) bytes += (unsigned)((hi - lo + 1) * sizeof(float2));
                }
            }
            mbar_expect(&bar, bytes);
            if (COLS) {
                if (bytes) {
                    const size_t blk = (size_t)(bx * L / d.blk_in) * N * d.blk_in;
                    bulk_load(smn + (size_t)x.za0 * L, src + blk + (size_t)x.za0 * L, bytes, &bar);
                }
            } else {
                for (int gg = 0; gg < L; gg++) {
                    const int ln = min(bx * L + gg, nl - 1);
                    const bool inl = !d.zwin || (ln >= d.zl0 && ln <= d.zl1);
                    const int lo = d.zwin ? (d.za0 & ~1) : 0, hi = d.zwin ? (d.za1 | 1) : N - 1;
                    if (inl && lo <= hi)
                        bulk_load(smn + (size_t)gg * P + lo, src + (size_t)ln * N + lo,
                                  (unsigned)((hi - lo + 1) * sizeof(float2)), &bar);
                }
            }
        }
        __syncthreads();
        if (!mbar_wait_bounded(&bar, phase, p.spin > 0 ? p.spin : (1ll << 22), p.status)) return false;
        x.sin = COLS ? (smn + g) : (smn + (size_t)g * P);
        x.sst = COLS ? L : 1;
    }
    ChainG pre, mid, fin;
    pre.rs1 = 0; pre.mir = 0; pre.rs2 = d.f1_pre.rs; pre.tab = (int)d.t_pre.tab; pre.extra = 0;
    mid.rs1 = d.f1 ? d.f1_post.rs : 0; mid.mir = d.mirror_along; mid.rs2 = d.f2 ? d.f2_pre.rs : 0;
    mid.tab = (int)d.t_mid.tab; mid.extra = EXTRA ? d.has_extra : 0;
    fin.rs1 = d.f2 ? d.f2_post.rs : 0; fin.mir = 0; fin.rs2 = 0; fin.tab = (int)d.t_fin.tab; fin.extra = 0;
    x.has_lf = (d.t_pre.ltab >= 0) || (d.t_mid.ltab >= 0) || (d.t_fin.ltab >= 0);
    x.lf = make_float2(1.f, 0.f);
    x.iscale = 1.f;
    if (OUTI && d.int_flat) {
        // the output factors have one magnitude: the intensity is scaled instead (the single
        // transform's output chain is mid after f1, fin after f2)
        if (d.f1) mid.tab = -1;
        else fin.tab = -1;
        x.has_lf = false;
        x.iscale = d.int_scale;
    }
    if (x.has_lf) {
        if (d.t_pre.ltab >= 0) x.lf = cmul(x.lf, __ldg(&x.tabs[d.t_pre.ltab + line]));
        if (d.t_mid.ltab >= 0) x.lf = cmul(x.lf, __ldg(&x.tabs[d.t_mid.ltab + line]));
        if (d.t_fin.ltab >= 0) x.lf = cmul(x.lf, __ldg(&x.tabs[d.t_fin.ltab + line]));
    }
    const float2* tw = p.tw;
    if constexpr (NT == 2) {
        if (p.bulk) fft_n<N, 3, 0, EXTRA>(s, x, pre, mid, d.f1 < 0 ? -1.f : 1.f, tw, t);
        else fft_n<N, 2, 0, EXTRA>(s, x, pre, mid, d.f1 < 0 ? -1.f : 1.f, tw, t);
        fft_n<N, 1, 1, EXTRA, OUTI>(s, x, mid, fin, d.f2 < 0 ? -1.f : 1.f, tw, t, acc);
    } else {
        const bool one = d.f1 != 0;
        const float cj = (one ? d.f1 : d.f2) < 0 ? -1.f : 1.f;
        if (p.bulk) fft_n<N, 3, 1, EXTRA, OUTI>(s, x, one ? pre : mid, one ? mid : fin, cj, tw, t, acc);
        else fft_n<N, 2, 1, EXTRA, OUTI>(s, x, one ? pre : mid, one ? mid : fin, cj, tw, t, acc);
    }
    return true;
}

template <int N, bool COLS, bool EXTRA, int NT>
__global__ void __launch_bounds__(512, (EXTRA || NT == 2) ? 1 : 2) linen_kernel(const LineLaunch p)
{
    __shared__ uint64_t bar;
    linen_body<N, COLS, EXTRA, NT, 0>(p, blockIdx.y, nullptr, &bar, 0);
}

// intensity pass (the last pass of a multi-electron batch): both components of the CTA's lines one
// after the other (one transform each, no non-separable work), |Ex|^2 + |Ey|^2 written as float
template <int N, bool COLS>
__global__ void __launch_bounds__(512, 2) linen_int_kernel(const LineLaunch p)
{
    static_assert(linen_int_floats(N) == IAcc<N>::B * IAcc<N>::R, "host size of the intensity carry");
    extern __shared__ __align__(16) float2 smn[];
    __shared__ uint64_t bar;
    IAcc<N> acc;
    acc.v = reinterpret_cast<float*>(smn + (size_t)p.L * p.P);
    acc.nt = blockDim.x;
    acc.tid = threadIdx.x;
    if (!linen_body<N, COLS, false, 1, 1>(p, 0, &acc, &bar, 0)) return;
    __syncthreads();                          // the second component's copies overwrite the tile
    linen_body<N, COLS, false, 1, 2>(p, 1, &acc, &bar, 1);
}

// the kernel of a (COLS, EXTRA, transforms) combination for length N; intensity passes: `inten`
template <int N>
Line2Fn linen_select(bool cols, bool extra, int nt, bool inten = false)
{
    if (inten) return cols ? linen_int_kernel<N, true> : linen_int_kernel<N, false>;
    if (cols) {
        if (extra) return nt == 2 ? linen_kernel<N, true, true, 2> : linen_kernel<N, true, true, 1>;
        return nt == 2 ? linen_kernel<N, true, false, 2> : linen_kernel<N, true, false, 1>;
    }
    if (extra) return nt == 2 ? linen_kernel<N, false, true, 2> : linen_kernel<N, false, true, 1>;
    return nt == 2 ? linen_kernel<N, false, false, 2> : linen_kernel<N, false, false, 1>;
}

}  // namespace srwg
