// Device helpers shared by the pass kernels (included by kernels.cu and the line2_*.cu units).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "kdesc.h"
#include "kernels.h"

namespace srwg {

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// complex add / subtract as one packed FP32x2 instruction each (sm_100); b * (-1) + a is exactly a - b
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward, DIR=+1) or +i (inverse, DIR=-1)
template <int DIR> __device__ __forceinline__ float2 mul_mi(float2 a)
{
    return DIR > 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

// exp(i*ph): Cody-Waite reduction of the FP64 argument by 2*pi (two-term constant) to [-pi, pi],
// then the FP32 hardware sine/cosine (absolute error ~4e-7 on that interval, the same order as
// the reference's own polynomial CosAndSin, sroptelm.h:856).
__device__ __forceinline__ float2 expi(double ph)
{
    const double inv2pi = 0.15915494309189533577;
    const double twopi_hi = 6.283185307179586232;      // nearest double to 2*pi
    const double twopi_lo = 2.4492935982947064e-16;    // 2*pi - twopi_hi
    double k = rint(ph * inv2pi);
    double r = fma(-k, twopi_hi, ph);
    r = fma(-k, twopi_lo, r);
    float s, c;
    __sincosf((float)r, &s, &c);
    return make_float2(c, s);
}

// ------------------------------------------------------------------------------------------------
// small DFTs (DIR=+1: exp(-2 pi i nk/R) like FFTW_FORWARD; DIR=-1: exp(+...) like FFTW_BACKWARD)
// ------------------------------------------------------------------------------------------------
template <int DIR> __device__ __forceinline__ void dft2(float2* v)
{
    float2 a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
}
template <int DIR> __device__ __forceinline__ void dft4(float2& v0, float2& v1, float2& v2, float2& v3)
{
    float2 a0 = cadd(v0, v2), a1 = csub(v0, v2), a2 = cadd(v1, v3), a3 = mul_mi<DIR>(csub(v1, v3));
    v0 = cadd(a0, a2);
    v2 = csub(a0, a2);
    v1 = cadd(a1, a3);
    v3 = csub(a1, a3);
}
template <int DIR> __device__ __forceinline__ void dft4(float2* v) { dft4<DIR>(v[0], v[1], v[2], v[3]); }

template <int DIR> __device__ __forceinline__ void dft8(float2* v)
{
    const float h = 0.70710678118654752440f;
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<DIR>(e0, e1, e2, e3);
    dft4<DIR>(o0, o1, o2, o3);
    // W8^1 = (1 -/+ i)/sqrt2, W8^2 = -/+ i, W8^3 = (-1 -/+ i)/sqrt2
    float2 t1 = make_float2(h * (o1.x + (DIR > 0 ? o1.y : -o1.y)), h * (o1.y - (DIR > 0 ? o1.x : -o1.x)));
    float2 t2 = mul_mi<DIR>(o2);
    float2 t3 = make_float2(h * (-o3.x + (DIR > 0 ? o3.y : -o3.y)), h * (-o3.y - (DIR > 0 ? o3.x : -o3.x)));
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, t1); v[5] = csub(e1, t1);
    v[2] = cadd(e2, t2); v[6] = csub(e2, t2);
    v[3] = cadd(e3, t3); v[7] = csub(e3, t3);
}

template <int DIR> __device__ __forceinline__ void dft16(float2* v)
{
    // n = 4 n1 + n2, k = k1 + 4 k2
    float2 y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
        float2 a0 = v[n2], a1 = v[4 + n2], a2 = v[8 + n2], a3 = v[12 + n2];
        dft4<DIR>(a0, a1, a2, a3);
        y[n2][0] = a0; y[n2][1] = a1; y[n2][2] = a2; y[n2][3] = a3;
    }
    // twiddles W16^(n2 k1)
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f, h = 0.70710678118654752440f;
    const float sg = DIR > 0 ? -1.f : 1.f;
    const float2 w1 = make_float2(c1, sg * s1), w2 = make_float2(h, sg * h), w3 = make_float2(s1, sg * c1);
    y[1][1] = cmul(y[1][1], w1); y[1][2] = cmul(y[1][2], w2); y[1][3] = cmul(y[1][3], w3);
    y[2][1] = cmul(y[2][1], w2); y[2][2] = mul_mi<DIR>(y[2][2]);
    y[2][3] = cmul(y[2][3], make_float2(-h, sg * h));
    y[3][1] = cmul(y[3][1], w3); y[3][2] = cmul(y[3][2], make_float2(-h, sg * h));
    y[3][3] = cmul(y[3][3], make_float2(-c1, -sg * s1));
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
        float2 a0 = y[0][k1], a1 = y[1][k1], a2 = y[2][k1], a3 = y[3][k1];
        dft4<DIR>(a0, a1, a2, a3);
        v[k1] = a0; v[k1 + 4] = a1; v[k1 + 8] = a2; v[k1 + 12] = a3;
    }
}

template <int DIR> __device__ __forceinline__ void dft3(float2* v)
{
    const float s = 0.86602540378443864676f;
    float2 t1 = cadd(v[1], v[2]);
    float2 t2 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    float2 t3 = mul_mi<DIR>(cscale(csub(v[1], v[2]), s));
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
}

template <int DIR> __device__ __forceinline__ void dft5(float2* v)
{
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
    float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]), t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    float2 a1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    float2 a2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    float2 b1 = mul_mi<DIR>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
    float2 b2 = mul_mi<DIR>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, b1); v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2); v[3] = csub(a2, b2);
}

// 7-point DFT from the symmetric pairs (v_k +/- v_(7-k)): 36 real multiply-adds, no table
template <int DIR> __device__ __forceinline__ void dft7(float2* v)
{
    const float c1 = 0.62348980185873353053f, c2 = -0.22252093395631440429f, c3 = -0.90096886790241912624f;
    const float s1 = 0.78183148246802980871f, s2 = 0.97492791218182360702f, s3 = 0.43388373911755812048f;
    const float2 a1 = cadd(v[1], v[6]), a2 = cadd(v[2], v[5]), a3 = cadd(v[3], v[4]);
    const float2 b1 = csub(v[1], v[6]), b2 = csub(v[2], v[5]), b3 = csub(v[3], v[4]);
    const float2 x0 = v[0];
    auto lin = [&](float p, float q, float r, float2 u1, float2 u2, float2 u3, float2 z) {
        return make_float2(fmaf(p, u1.x, fmaf(q, u2.x, fmaf(r, u3.x, z.x))), fmaf(p, u1.y, fmaf(q, u2.y, fmaf(r, u3.y, z.y))));
    };
    const float2 z0 = make_float2(0.f, 0.f);
    const float2 A1 = lin(c1, c2, c3, a1, a2, a3, x0), B1 = mul_mi<DIR>(lin(s1, s2, s3, b1, b2, b3, z0));
    const float2 A2 = lin(c2, c3, c1, a1, a2, a3, x0), B2 = mul_mi<DIR>(lin(s2, -s3, -s1, b1, b2, b3, z0));
    const float2 A3 = lin(c3, c1, c2, a1, a2, a3, x0), B3 = mul_mi<DIR>(lin(s3, -s1, s2, b1, b2, b3, z0));
    v[0] = cadd(x0, cadd(a1, cadd(a2, a3)));
    v[1] = cadd(A1, B1); v[6] = csub(A1, B1);
    v[2] = cadd(A2, B2); v[5] = csub(A2, B2);
    v[3] = cadd(A3, B3); v[4] = csub(A3, B3);
}

// generic odd radix (7, 11, 13): direct O(R^2) DFT; W_R^m = tw[m * N / R]
template <int R, int DIR> __device__ __forceinline__ void dftg(float2* v, const float2* __restrict__ tw, int NdR)
{
    float2 o[R];
#pragma unroll
    for (int m = 0; m < R; m++) {
        float2 acc = v[0];
#pragma unroll
        for (int n = 1; n < R; n++) {
            float2 w = __ldg(&tw[((n * m) % R) * NdR]);
            if (DIR < 0) w.y = -w.y;
            acc = cadd(acc, cmul(v[n], w));
        }
        o[m] = acc;
    }
#pragma unroll
    for (int m = 0; m < R; m++) v[m] = o[m];
}

template <int R, int DIR> __device__ __forceinline__ void dftR(float2* v, const float2* __restrict__ tw, int N)
{
    if (R == 2) dft2<DIR>(v);
    else if (R == 3) dft3<DIR>(v);
    else if (R == 4) dft4<DIR>(v);
    else if (R == 5) dft5<DIR>(v);
    else if (R == 8) dft8<DIR>(v);
    else if (R == 16) dft16<DIR>(v);
    else if (R == 7) dft7<DIR>(v);
    else dftg<R, DIR>(v, tw, N / R);
}

// One Stockham autosort stage on a line of N points in shared memory.  Thread t of T owns the
// butterflies j = t, t+T, ...; all its inputs are read into registers before the barrier, so the
// stage works in place.  Ns = product of the radices already applied.
template <int R, int DIR>
__device__ __forceinline__ void stockham_stage(float2* s, int N, int Ns, const float2* __restrict__ tw, int t, int T,
                                               bool active)
{
    constexpr int MAXB = (16 + R - 1) / R;
    const int NR = N / R;
    const int tws = N / (Ns * R);
    float2 v[MAXB][R];
#pragma unroll
    for (int b = 0; b < MAXB; b++) {
        int j = t + b * T;
        if (active && j < NR) {
            int k = j % Ns;
#pragma unroll
            for (int r = 0; r < R; r++) {
                float2 x = s[j + r * NR];
                if (r > 0 && k != 0) {
                    float2 w = __ldg(&tw[k * tws * r]);
                    if (DIR < 0) w.y = -w.y;
                    x = cmul(x, w);
                }
                v[b][r] = x;
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < MAXB; b++) {
        int j = t + b * T;
        if (active && j < NR) {
            dftR<R, DIR>(v[b], tw, N);
            int k = j % Ns;
            int base = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) s[base + r * Ns] = v[b][r];
        }
    }
    __syncthreads();
}

template <int DIR>
__device__ void run_fft(float2* s, int N, const int* radix, int nst, const float2* __restrict__ tw, int t, int T,
                        bool active)
{
    int Ns = 1;
    for (int st = 0; st < nst; st++) {
        int R = radix[st];
        switch (R) {
        case 16: stockham_stage<16, DIR>(s, N, Ns, tw, t, T, active); break;
        case 8: stockham_stage<8, DIR>(s, N, Ns, tw, t, T, active); break;
        case 4: stockham_stage<4, DIR>(s, N, Ns, tw, t, T, active); break;
        case 2: stockham_stage<2, DIR>(s, N, Ns, tw, t, T, active); break;
        case 3: stockham_stage<3, DIR>(s, N, Ns, tw, t, T, active); break;
        case 5: stockham_stage<5, DIR>(s, N, Ns, tw, t, T, active); break;
        case 7: stockham_stage<7, DIR>(s, N, Ns, tw, t, T, active); break;
        case 11: stockham_stage<11, DIR>(s, N, Ns, tw, t, T, active); break;
        case 13: stockham_stage<13, DIR>(s, N, Ns, tw, t, T, active); break;
        default: break;
        }
        Ns *= R;
    }
}

// ------------------------------------------------------------------------------------------------
// point-wise operators
// ------------------------------------------------------------------------------------------------
// exact (non-contracted) FP64 coordinate arithmetic, as the reference's x87/SSE code evaluates it
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// accumulates phase, complex factor and zeroing of PwOps at kernel index (i, j)
__device__ __forceinline__ void pw_eval(const PwOps& pw, int i, int j, double& ph, float2& f, bool& zero)
{
    if (pw.has_quad) {
        double di = (double)i, dj = (double)j;
        ph += fma(fma(pw.Ai, di, pw.Bi), di, fma(fma(pw.Aj, dj, pw.Bj), dj, pw.C));
    }
    if (pw.has_ang) {
        double qx = pw.qx0 + (double)i * pw.dqx, qz = pw.qz0 + (double)j * pw.dqz;
        double q2 = qx * qx + qz * qz;
        double c1q2 = pw.c1 * q2;
        ph += pw.c0 * q2 * (1. + c1q2 + 2. * c1q2 * c1q2);
    }
    if (pw.has_scale) f = cmul(f, make_float2(pw.sre, pw.sim));
    for (int m = 0; m < pw.nmask; m++) {
        const PwMask& k = pw.mask[m];
        double x = dadd(k.x0, dmul((double)i, k.dx));
        double z = dadd(k.z0, dmul((double)j, k.dz));
        double xr = dsub(x, k.cx), zr = dsub(z, k.cz);
        bool outside;
        if (k.type == 1) outside = (xr < -k.hx) || (xr > k.hx) || (zr < -k.hz) || (zr > k.hz);
        else outside = dadd(dmul(xr, xr), dmul(zr, zr)) > k.r2;
        zero |= k.obstacle ? !outside : outside;
    }
}

// W[k] = factor(k) * V[src(k)] for the chain: [post of a previous transform] -> [point-wise] ->
// [mirror along the line] -> [pre of the next transform].
struct Chain {
    int rs1, sh1;
    double a1;
    float sc1;
    const PwOps* pw;
    int mir;
    int rs2, sh2;
    double a2;
    int axis;
};

__device__ __forceinline__ float2 chain_eval(const Chain& c, int k, int N, int line, int& src)
{
    const int half = N >> 1;
    double ph = 0.;
    bool hasph = false, zero = false;
    float sg = 1.f;
    float2 f = make_float2(1.f, 0.f);
    int m = k;
    if (c.rs2) {                      // rotate then sign: W[k] = (-1)^k M[(k+N/2)%N]
        m = k + half; if (m >= N) m -= N;
        if (k & 1) sg = -sg;
    }
    if (c.sh2) { ph += c.a2 * (double)(m - half); hasph = true; }   // shift-before (on the source index)
    int i = c.mir ? (N - 1 - m) : m;
    if (c.pw) {
        int ix = c.axis == 0 ? i : line, jz = c.axis == 0 ? line : i;
        double p0 = ph;
        pw_eval(*c.pw, ix, jz, ph, f, zero);
        hasph = hasph || (ph != p0) || c.pw->has_quad || c.pw->has_ang;
    }
    int s = i;
    if (c.rs1) {                      // sign then rotate: Z[i] = (-1)^s Y[s], s = (i+N/2)%N
        s = i + half; if (s >= N) s -= N;
        if (s & 1) sg = -sg;
    }
    if (c.sh1) { ph += c.a1 * (double)(i - half); hasph = true; }   // shift-after (on the output index)
    src = s;
    float sc = sg * c.sc1;
    float2 r = make_float2(sc * f.x, sc * f.y);
    if (hasph) r = cmul(r, expi(ph));
    if (zero) r = make_float2(0.f, 0.f);
    return r;
}

__device__ __forceinline__ bool chain_trivial(const Chain& c)
{
    return !c.rs1 && !c.sh1 && c.sc1 == 1.f && c.pw == nullptr && !c.mir && !c.rs2 && !c.sh2;
}

// register-staged in-place gather on one line: s[k] <- factor(k) s[src(k)]
__device__ __forceinline__ void gather_pass(float2* s, int N, int line, const Chain& c, int t, int T, bool active)
{
    float2 tmp[16];
#pragma unroll
    for (int v = 0; v < 16; v++) {
        int k = t + v * T;
        if (active && k < N) {
            int src;
            float2 f = chain_eval(c, k, N, line, src);
            tmp[v] = cmul(f, s[src]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 16; v++) {
        int k = t + v * T;
        if (active && k < N) s[k] = tmp[v];
    }
    __syncthreads();
}

// chain of a general (even) line length with its along-line factors in the plan's tables:
// W[k] = tab[k] * extra(i(k), line) * V[src(k)], m = rot2(k), i = mirror(m), src = rot1(i)
struct ChainG {
    int rs1, mir, rs2;
    int tab;                 // offset of the along-line factors in the plan's tables, or -1
    int extra;               // the pass's non-separable work applies to this chain
};

__device__ __forceinline__ int chainG_src(const ChainG& c, int k, int N, int& i)
{
    const int h = N >> 1;
    int m = k;
    if (c.rs2) { m = k + h; if (m >= N) m -= N; }
    i = c.mir ? (N - 1 - m) : m;
    int s = i;
    if (c.rs1) { s = i + h; if (s >= N) s -= N; }
    return s;
}

__device__ __forceinline__ bool chainG_trivial(const ChainG& c)
{
    return !c.rs1 && !c.mir && !c.rs2 && c.tab < 0 && !c.extra;
}

__device__ __forceinline__ void extra_eval(const PwOps& e, int i, int j, float2& f, bool& zero, const float2* tabs);

template <bool EXTRA = true>
__device__ __forceinline__ float2 chainG_factor(const ChainG& c, int k, int i, int line, const float2* tabs,
                                                const PwOps* ex, int axis)
{
    float2 f = c.tab >= 0 ? __ldg(&tabs[c.tab + k]) : make_float2(1.f, 0.f);
    if (EXTRA && c.extra) {
        bool zero = false;
        extra_eval(*ex, axis == 0 ? i : line, axis == 0 ? line : i, f, zero, tabs);
        if (zero) f = make_float2(0.f, 0.f);
    }
    return f;
}

// register-staged in-place gather on one line through a table chain: s[k] <- factor(k) s[src(k)]
__device__ __forceinline__ void gather_pass_t(float2* s, int N, int line, const ChainG& c, int t, int T, bool active,
                                              const float2* tabs, const PwOps* ex, int axis)
{
    float2 tmp[16];
#pragma unroll
    for (int v = 0; v < 16; v++) {
        const int k = t + v * T;
        if (active && k < N) {
            int i;
            const int src = chainG_src(c, k, N, i);
            tmp[v] = cmul(chainG_factor(c, k, i, line, tabs, ex, axis), s[src]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 16; v++) {
        const int k = t + v * T;
        if (active && k < N) s[k] = tmp[v];
    }
    __syncthreads();
}

// RadPointModifier_PropToWaistBeyondParax (sroptdrf.h:712-754): exp(i k L (sqrt(1 + X) - 1)), or with
// k L sqrt(1 + X) on the path-length option, X = -lambda^2 (qx^2 + qz^2); the square root for
// |X| > 0.01, else the reference's binomial series; FP64, then reduced by 2 pi.  Out of line: rare,
// and it keeps the passes that may evaluate it small.
static __device__ __noinline__ float2 bpx_factor(const PwOps& e, int i, int j)
{
    const double qx = e.bqx0 + (double)i * e.bdqx, qz = e.bqz0 + (double)j * e.bdqz;
    const double lx = e.blam * qx, lz = e.blam * qz;
    const double X = -(lx * lx + lz * lz);
    double r;
    if (fabs(X) > 0.01) {
        r = sqrt(1. + X);
        if (!e.btreat) r -= 1.;
    } else {
        r = X * (0.5 + X * (-0.125 + X * (0.0625 + X * (-0.0390625 + X * (0.02734375 + X * (-0.0205078125 +
                                                                                  X * 0.01611328125))))));
        if (e.btreat) r += 1.;
    }
    return expi(e.bkL * r);
}

// srTGenTransmission::RadPointModifier (sroptgtr.h:163-310), one photon energy: amplitude
// transmission and optical path difference bilinear in the table (FP64, its index rules: the
// 1e-5 step snap, clamping to the last cell), the phase 2 pi / lambda * OPD; zero outside the table
// (within 1e-3 of a step) when the element says so.  Returns false to zero the point.
static __device__ __noinline__ bool tr_factor(const PwOps& e, int i, int j, const float2* tabs, float2& f)
{
    const double xRel = dadd(e.tr_x0, dmul((double)i, e.tr_dx)), zRel = dadd(e.tr_z0, dmul((double)j, e.tr_dz));
    const int Nx = e.tr_nx, Nz = e.tr_nz;
    const double xs = e.tr_xs, zs = e.tr_zs, xst = e.tr_xstep, zst = e.tr_zstep;
    if (e.tr_outer == 1) {
        const double xEnd = xs + (Nx - 1) * xst, zEnd = zs + (Nz - 1) * zst;
        const double tx = xst * 0.001, tz = zst * 0.001;
        if ((xRel < xs - tx) || (xRel > xEnd + tx) || (zRel < zs - tz) || (zRel > zEnd + tz)) return false;
    }
    double xr = 0., zr = 0.;
    long long ix = (long long)((xRel - xs) / xst);
    if (fabs(xRel - ((ix + 1) * xst + xs)) < 1.E-05 * xst) ix++;
    if (ix < 0) ix = 0;
    else if (ix > Nx - 2) { ix = Nx - 2; xr = 1.; }
    else xr = (xRel - (ix * xst + xs)) / xst;
    long long iz = (long long)((zRel - zs) / zst);
    if (fabs(zRel - ((iz + 1) * zst + zs)) < 1.E-05 * zst) iz++;
    if (iz < 0) iz = 0;
    else if (iz > Nz - 2) { iz = Nz - 2; zr = 1.; }
    else zr = (zRel - (iz * zst + zs)) / zst;
    const double xrzr = xr * zr;
    const double* d = reinterpret_cast<const double*>(tabs + e.tr_off);
    const long long zPer = (long long)Nx << 1;
    const double* p00 = d + (iz * zPer + (ix << 1));
    const double *p10 = p00 + 2, *p01 = p00 + zPer, *p11 = p01 + 2;
    const double Axz = p00[0] - p01[0] - p10[0] + p11[0], Bxz = p00[1] - p01[1] - p10[1] + p11[1];
    const double Ax = p10[0] - p00[0], Bx = p10[1] - p00[1];
    const double Az = p01[0] - p00[0], Bz = p01[1] - p00[1];
    const double T = Axz * xrzr + Ax * xr + Az * zr + p00[0];
    const double Ph = (Bxz * xrzr + Bx * xr + Bz * zr + p00[1]) * e.tr_k;
    const float2 c = expi(Ph);
    f = cmul(f, make_float2((float)(T * c.x), (float)(T * c.y)));
    return true;
}

// non-separable point-wise work: circular masks, rectangular obstacles, the quartic remainder of
// the angular transfer function, the beyond-paraxial propagator (everything separable is in the
// plan's tables)
__device__ __forceinline__ void extra_eval(const PwOps& e, int i, int j, float2& f, bool& zero, const float2* tabs)
{
    if (e.has_ang) {
        float qx = (float)(e.qx0 + (double)i * e.dqx), qz = (float)(e.qz0 + (double)j * e.dqz);
        float q2 = qx * qx + qz * qz;
        float c1q2 = (float)e.c1 * q2;
        float ph = (float)e.c0 * q2 * c1q2 * (1.f + 2.f * c1q2);
        float sn, cs;
        __sincosf(ph, &sn, &cs);
        f = cmul(f, make_float2(cs, sn));
    }
    if (e.has_bpx) f = cmul(f, bpx_factor(e, i, j));
    if (e.has_tr && !tr_factor(e, i, j, tabs, f)) zero = true;
    for (int m = 0; m < e.nmask; m++) {
        const PwMask& k = e.mask[m];
        double x = dadd(k.x0, dmul((double)i, k.dx));
        double z = dadd(k.z0, dmul((double)j, k.dz));
        double xr = dsub(x, k.cx), zr = dsub(z, k.cz);
        bool outside;
        if (k.type == 1) outside = (xr < -k.hx) || (xr > k.hx) || (zr < -k.hz) || (zr > k.hz);
        else outside = dadd(dmul(xr, xr), dmul(zr, zr)) > k.r2;
        zero |= k.obstacle ? !outside : outside;
    }
}

// chain with its along-line factors in a table: W[k] = tab[k] * extra(k ^ xi, line) * V[k ^ xs].  For
// power-of-two lines the centring rotation and the mirror are XOR masks: (k + N/2) mod N = k ^ N/2,
// N - 1 - k = k ^ (N - 1).  The chain's per-line factor is not part of it: the line factors of all
// chains of a pass are multiplied once per line and applied at the store (a per-line constant
// commutes with the FFT along the line).
struct Chain2 {
    int xs;                  // source index mask: rotation (rs2), mirror, rotation (rs1)
    int xi;                  // evaluation index mask of the non-separable work (rs2, mirror)
    int xinv;                // output chains: destination of transform output q is q ^ xinv
    int tab;                 // offset of the along-line factors in the plan's tables, or -1
    int extra;               // the pass's non-separable work applies to this chain
};

// v <- factor(k) v; `tabs` are the plan's tables, `ex` the pass's non-separable work
template <bool EXTRA>
__device__ __forceinline__ float2 chain2_apply(const Chain2& c, int k, int line, float2 v, const float2* tabs,
                                               const PwOps* ex, int axis)
{
    if (c.tab >= 0) v = cmul(__ldg(&tabs[c.tab + k]), v);
    if (EXTRA && c.extra) {
        const int i = k ^ c.xi;
        bool zero = false;
        float2 f = make_float2(1.f, 0.f);
        extra_eval(*ex, axis == 0 ? i : line, axis == 0 ? line : i, f, zero, tabs);
        v = zero ? make_float2(0.f, 0.f) : cmul(f, v);
    }
    return v;
}

__device__ __forceinline__ Chain2 make_chain2(const ChainTab& t, int rs1, int mir, int rs2, int extra, int N)
{
    Chain2 c;
    const int h = N >> 1;
    c.xi = (rs2 ? h : 0) ^ (mir ? N - 1 : 0);
    c.xs = c.xi ^ (rs1 ? h : 0);
    c.xinv = (rs1 ? h : 0) ^ (mir ? N - 1 : 0);
    c.tab = t.tab >= 0 ? (int)t.tab : -1;
    c.extra = extra;
    return c;
}

// element i of a line pass's output line: row-major (offset i * str) or, for a row pass feeding a
// column pass, column-blocked: blocks of 2^lg columns stored contiguously per row, offset
// (i >> lg) * bstr + (i & mask)
struct OutMap {
    int str, lg, bstr;
    __device__ __forceinline__ int at(int i) const { return lg < 0 ? i * str : ((i >> lg) * bstr + (i & ((1 << lg) - 1))); }
};

}  // namespace srwg
