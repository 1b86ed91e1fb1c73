// sm_100a kernels for SRW's Fourier-optics propagation path.
//
// All passes are HBM-bandwidth bound (a complex FP32 point is read and written once per pass,
// ~1-4 flop/B), so they are plain SIMT kernels organised around full-line shared-memory tiles;
// no tensor cores.  Phase arguments are formed and reduced modulo 2*pi in FP64 and evaluated
// with an FP32 sincosf, as the reference forms them in double before its float CosAndSin
// (sroptelm.h:856-871).
#include <cuda_runtime.h>
#include <stdint.h>
#include "kdesc.h"
#include "kernels.h"

namespace srwg {

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
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
    __shared__ LineDesc d;
    __shared__ int radix[SRWG_MAX_STAGES];
    if (threadIdx.x == 0) {
        d = p.d;
        for (int i = 0; i < SRWG_MAX_STAGES; i++) radix[i] = p.radix[i];
    }
    __syncthreads();
    const int comp = blockIdx.y;
    const float2* __restrict__ src = p.src[comp];
    float2* __restrict__ dst = p.dst[comp];
    const int N = p.N, T = p.T, L = p.L, P = p.P, nl = p.nlines;
    const int tid = threadIdx.x, nth = blockDim.x;
    const int G = nth / T;
    const int g = tid / T, t = tid - g * T;
    const int line0 = blockIdx.x * L;

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

    Chain mid;
    mid.rs1 = 0; mid.sh1 = 0; mid.a1 = 0.; mid.sc1 = 1.f; mid.pw = d.has_pw ? &d.pw : nullptr;
    mid.mir = d.mirror_along; mid.rs2 = 0; mid.sh2 = 0; mid.a2 = 0.; mid.axis = d.axis;
    Chain pre;
    pre.rs1 = 0; pre.sh1 = 0; pre.a1 = 0.; pre.sc1 = 1.f; pre.pw = nullptr; pre.mir = 0;
    pre.rs2 = d.f1_pre.rs; pre.sh2 = d.f1_pre.has_shift; pre.a2 = d.f1_pre.shift_a; pre.axis = d.axis;
    if (d.f1) { mid.rs1 = d.f1_post.rs; mid.sh1 = d.f1_post.has_shift; mid.a1 = d.f1_post.shift_a; mid.sc1 = d.f1_post.scale; }
    Chain fin;
    if (d.f2) {
        mid.rs2 = d.f2_pre.rs; mid.sh2 = d.f2_pre.has_shift; mid.a2 = d.f2_pre.shift_a;
        fin.rs1 = d.f2_post.rs; fin.sh1 = d.f2_post.has_shift; fin.a1 = d.f2_post.shift_a; fin.sc1 = d.f2_post.scale;
        fin.pw = nullptr; fin.mir = 0; fin.rs2 = 0; fin.sh2 = 0; fin.a2 = 0.; fin.axis = d.axis;
    } else {
        fin = mid;
    }

    // ---- transforms, batch by batch (uniform trip count: every thread reaches every barrier)
    if (d.f1 || d.f2) {
        const int nb = (L + G - 1) / G;
        for (int it = 0; it < nb; it++) {
            const int c = it * G + g;
            const int line = line0 + c;
            const bool active = (g < G) && (c < L) && (line < nl);
            float2* s = sm + (size_t)(c < L ? c : 0) * P;
            if (d.f1) {
                if (!chain_trivial(pre)) gather_pass(s, N, line, pre, t, T, active);
                if (d.f1 > 0) run_fft<1>(s, N, radix, p.nst, p.tw, t, T, active);
                else run_fft<-1>(s, N, radix, p.nst, p.tw, t, T, active);
            }
            if (d.f2) {
                if (!chain_trivial(mid)) gather_pass(s, N, line, mid, t, T, active);
                if (d.f2 > 0) run_fft<1>(s, N, radix, p.nst, p.tw, t, T, active);
                else run_fft<-1>(s, N, radix, p.nst, p.tw, t, T, active);
            }
        }
    }
    const bool triv = chain_trivial(fin);

    // ---- store the tile
    if (d.axis == 0) {
        for (int e = tid; e < N * L; e += nth) {
            int c = e / N, k = e - c * N;
            int line = line0 + c;
            if (line < nl) {
                const float2* sc = sm + (size_t)c * P;
                float2 v;
                if (triv) v = sc[k];
                else { int sr; float2 f = chain_eval(fin, k, N, line, sr); v = cmul(f, sc[sr]); }
                int ol = d.mirror_lines ? (nl - 1 - line) : line;
                __stcs(&dst[(size_t)ol * N + k], v);
            }
        }
    } else {
        for (int e = tid; e < N * L; e += nth) {
            int r = e / L, c = e - r * L;
            int col = line0 + c;
            if (col < nl) {
                const float2* sc = sm + (size_t)c * P;
                float2 v;
                if (triv) v = sc[r];
                else { int sr; float2 f = chain_eval(fin, r, N, col, sr); v = cmul(f, sc[sr]); }
                int oc = d.mirror_lines ? (nl - 1 - col) : col;
                __stcs(&dst[(size_t)r * nl + oc], v);
            }
        }
    }
}

// ------------------------------------------------------------------------------------------------
// LINE pass, power-of-two lines (N >= 64): every thread owns 16 points of its line.  The first
// FFT stage reads its butterfly inputs straight from global memory through the point-wise chain
// (coalesced: thread t reads t + T*m), the last stage writes straight to global memory through
// the output chain; intermediate stages exchange through shared memory padded by one point per
// 16 (conflict-free Stockham writes).  A second transform in the same pass (f1 -> f2) reads the
// first one's output from shared memory through the middle chain.
// ------------------------------------------------------------------------------------------------
#define PADI(p) ((p) + ((p) >> 4))

// output index k whose source is q under a store chain (no pre-rotation): k = mir(rot(q))
__device__ __forceinline__ int chain_inv(const Chain& c, int q, int N)
{
    int i = q;
    if (c.rs1) { i = q + (N >> 1); if (i >= N) i -= N; }
    return c.mir ? (N - 1 - i) : i;
}

// IN: 0 shared, 1 shared through chain cin, 2 global through chain cin;  OUT: 0 shared, 1 global through chain cout
template <int R, int DIR, int IN, int OUT>
__device__ __forceinline__ void stage16(float2* s, const float2* __restrict__ gin, float2* __restrict__ gout,
                                        long long gstr, int N, int Ns, int t, int T, int line, const Chain& cin,
                                        const Chain& cout, const float2* __restrict__ tw, bool active)
{
    constexpr int B = 16 / R;
    const int NR = N / R;
    const int lgNs = __ffs(Ns) - 1;
    const int tws = N / (Ns * R);
    float2 v[B][R];
#pragma unroll
    for (int b = 0; b < B; b++) {
        const int j = t + T * b;
        const int k = j & (Ns - 1);
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int p = j + r * NR;
            float2 x = make_float2(0.f, 0.f);
            if (active) {
                if (IN == 0) {
                    x = s[PADI(p)];
                } else {
                    int sp;
                    float2 f = chain_eval(cin, p, N, line, sp);
                    x = (IN == 1) ? s[PADI(sp)] : __ldcs(&gin[(long long)sp * gstr]);
                    x = cmul(f, x);
                }
                if (r > 0 && k != 0) {
                    float2 w = __ldg(&tw[k * tws * r]);
                    if (DIR < 0) w.y = -w.y;
                    x = cmul(x, w);
                }
            }
            v[b][r] = x;
        }
    }
    if (OUT == 0) __syncthreads();
#pragma unroll
    for (int b = 0; b < B; b++) {
        const int j = t + T * b;
        const int k = j & (Ns - 1);
        dftR<R, DIR>(v[b], tw, N);
        const int base = ((j >> lgNs) << lgNs) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int q = base + r * Ns;
            if (active) {
                if (OUT == 0) {
                    s[PADI(q)] = v[b][r];
                } else {
                    int i = chain_inv(cout, q, N), sp;
                    float2 f = chain_eval(cout, i, N, line, sp);
                    __stcs(&gout[(long long)i * gstr], cmul(f, v[b][r]));
                }
            }
        }
    }
    if (OUT == 0) __syncthreads();
}

// last stage dispatch on its radix (16, 8, 4, 2)
template <int DIR, int OUT>
__device__ __forceinline__ void stage_last(int R, float2* s, float2* __restrict__ gout, long long gstr, int N, int Ns,
                                           int t, int T, int line, const Chain& cin, const Chain& cout,
                                           const float2* __restrict__ tw, bool active)
{
    switch (R) {
    case 16: stage16<16, DIR, 0, OUT>(s, nullptr, gout, gstr, N, Ns, t, T, line, cin, cout, tw, active); break;
    case 8: stage16<8, DIR, 0, OUT>(s, nullptr, gout, gstr, N, Ns, t, T, line, cin, cout, tw, active); break;
    case 4: stage16<4, DIR, 0, OUT>(s, nullptr, gout, gstr, N, Ns, t, T, line, cin, cout, tw, active); break;
    default: stage16<2, DIR, 0, OUT>(s, nullptr, gout, gstr, N, Ns, t, T, line, cin, cout, tw, active); break;
    }
}

// one FFT along the line: radix-16 stages then radix[nst-1]; IN mode of the first stage, OUT of the last
template <int DIR, int IN, int OUT>
__device__ __forceinline__ void fft16(float2* s, const float2* __restrict__ gin, float2* __restrict__ gout,
                                      long long gstr, int N, const int* radix, int nst, int t, int T, int line,
                                      const Chain& cin, const Chain& cout, const float2* __restrict__ tw, bool active)
{
    stage16<16, DIR, IN, 0>(s, gin, nullptr, gstr, N, 1, t, T, line, cin, cout, tw, active);
    int Ns = 16;
    for (int st = 1; st < nst - 1; st++) {
        stage16<16, DIR, 0, 0>(s, nullptr, nullptr, gstr, N, Ns, t, T, line, cin, cout, tw, active);
        Ns *= 16;
    }
    stage_last<DIR, OUT>(radix[nst - 1], s, gout, gstr, N, Ns, t, T, line, cin, cout, tw, active);
}

template <bool COLS>
__global__ void __launch_bounds__(1024, 1) line2_kernel(const LineLaunch p)
{
    extern __shared__ float2 sm[];
    __shared__ LineDesc d;
    __shared__ int radix[SRWG_MAX_STAGES];
    if (threadIdx.x == 0) {
        d = p.d;
        for (int i = 0; i < SRWG_MAX_STAGES; i++) radix[i] = p.radix[i];
    }
    __syncthreads();
    const int comp = blockIdx.y;
    const float2* __restrict__ src = p.src[comp];
    float2* __restrict__ dst = p.dst[comp];
    const int N = p.N, T = p.T, L = p.L, P = p.P, nl = p.nlines;
    const int tid = threadIdx.x;
    const int g = COLS ? (tid % L) : (tid / T);          // line of the tile
    const int t = COLS ? (tid / L) : (tid - g * T);      // thread within the line
    const int line = blockIdx.x * L + g;
    const bool active = line < nl;
    float2* s = sm + (size_t)g * P;
    const long long gstr = COLS ? (long long)nl : 1;
    const float2* gin = COLS ? (src + line) : (src + (size_t)line * N);
    const int oline = d.mirror_lines ? (nl - 1 - line) : line;
    float2* gout = COLS ? (dst + oline) : (dst + (size_t)oline * N);

    Chain pre, mid, fin;
    pre.rs1 = 0; pre.sh1 = 0; pre.a1 = 0.; pre.sc1 = 1.f; pre.pw = nullptr; pre.mir = 0;
    pre.rs2 = d.f1_pre.rs; pre.sh2 = d.f1_pre.has_shift; pre.a2 = d.f1_pre.shift_a; pre.axis = d.axis;
    mid.rs1 = 0; mid.sh1 = 0; mid.a1 = 0.; mid.sc1 = 1.f; mid.pw = d.has_pw ? &d.pw : nullptr;
    mid.mir = d.mirror_along; mid.rs2 = 0; mid.sh2 = 0; mid.a2 = 0.; mid.axis = d.axis;
    if (d.f1) { mid.rs1 = d.f1_post.rs; mid.sh1 = d.f1_post.has_shift; mid.a1 = d.f1_post.shift_a; mid.sc1 = d.f1_post.scale; }
    if (d.f2) {
        mid.rs2 = d.f2_pre.rs; mid.sh2 = d.f2_pre.has_shift; mid.a2 = d.f2_pre.shift_a;
        fin.rs1 = d.f2_post.rs; fin.sh1 = d.f2_post.has_shift; fin.a1 = d.f2_post.shift_a; fin.sc1 = d.f2_post.scale;
        fin.pw = nullptr; fin.mir = 0; fin.rs2 = 0; fin.sh2 = 0; fin.a2 = 0.; fin.axis = d.axis;
    }
    const int nst = p.nst;
    if (d.f1 && d.f2) {
        if (d.f1 > 0) fft16<1, 2, 0>(s, gin, nullptr, gstr, N, radix, nst, t, T, line, pre, mid, p.tw, active);
        else fft16<-1, 2, 0>(s, gin, nullptr, gstr, N, radix, nst, t, T, line, pre, mid, p.tw, active);
        if (d.f2 > 0) fft16<1, 1, 1>(s, nullptr, gout, gstr, N, radix, nst, t, T, line, mid, fin, p.tw, active);
        else fft16<-1, 1, 1>(s, nullptr, gout, gstr, N, radix, nst, t, T, line, mid, fin, p.tw, active);
    } else if (d.f1) {
        if (d.f1 > 0) fft16<1, 2, 1>(s, gin, gout, gstr, N, radix, nst, t, T, line, pre, mid, p.tw, active);
        else fft16<-1, 2, 1>(s, gin, gout, gstr, N, radix, nst, t, T, line, pre, mid, p.tw, active);
    } else {
        if (d.f2 > 0) fft16<1, 2, 1>(s, gin, gout, gstr, N, radix, nst, t, T, line, mid, fin, p.tw, active);
        else fft16<-1, 2, 1>(s, gin, gout, gstr, N, radix, nst, t, T, line, mid, fin, p.tw, active);
    }
}

// ------------------------------------------------------------------------------------------------
// RESIZE pass (RadResizeCore, sroptelm.cpp:3038-3337; OnlyLargerRange :4231)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void lagrange4(float t, float* w)
{
    // cubic through nodes -1, 0, 1, 2 (the reference's SetupInterpolAux02 polynomial)
    float tm1 = t - 1.f, tm2 = t - 2.f, tp1 = t + 1.f;
    w[0] = -t * tm1 * tm2 * (1.f / 6.f);
    w[1] = tp1 * tm1 * tm2 * 0.5f;
    w[2] = -tp1 * t * tm2 * 0.5f;
    w[3] = tp1 * t * tm1 * (1.f / 6.f);
}

struct AxisPos {
    int st;      // first of the 4 old nodes
    int ic;      // cell index
    double rel;  // relative coordinate in old steps, w.r.t. node st+1
};

__device__ __forceinline__ AxisPos resize_axis(int inew, double startN, double stepN, double startO, double stepO,
                                               double invO, int nO)
{
    AxisPos a;
    double absc = dadd(startN, dmul((double)inew, stepN));
    int ic = (int)dadd(dmul(dsub(absc, startO), invO), 1.E-06);
    double rel = dsub(absc, dadd(startO, dmul((double)ic, stepO)));
    int st;
    if (ic == nO - 1) { st = ic - 3; rel = dadd(rel, dmul(2., stepO)); }
    else if (ic == nO - 2) { st = ic - 2; rel = dadd(rel, stepO); }
    else if (ic == 0) { st = ic; rel = dsub(rel, stepO); }
    else st = ic - 1;
    // the reference reads outside the old grid if a new point falls outside it: clamp instead
    if (st < 0) st = 0;
    if (st > nO - 4) st = nO - 4;
    a.st = st; a.ic = ic; a.rel = dmul(rel, invO);
    return a;
}

__global__ void __launch_bounds__(256) resize_kernel(const ResizeLaunch p)
{
    __shared__ ResizeDesc d;
    if (threadIdx.x == 0 && threadIdx.y == 0) d = p.d;
    __syncthreads();
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= d.nxn || iz >= d.nzn) return;
    float2 out[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    const bool inwin = (ix >= d.ixStart) && (ix <= d.ixEnd) && (iz >= d.izStart) && (iz <= d.izEnd);
    if (inwin) {
        if (d.only_larger) {
            double xAbs = dadd(d.xStartN, dmul((double)ix, d.xStepN));
            double zAbs = dadd(d.zStartN, dmul((double)iz, d.zStepN));
            long xo = (long)dadd(dmul(dsub(xAbs, d.xStartO), p.xStepInvO), 1.E-08);
            long zo = (long)dadd(dmul(dsub(zAbs, d.zStartO), p.zStepInvO), 1.E-08);
            if (xo < 0) xo = 0;
            if (xo > d.nxo - 1) xo = d.nxo - 1;
            if (zo < 0) zo = 0;
            if (zo > d.nzo - 1) zo = d.nzo - 1;
#pragma unroll
            for (int c = 0; c < 2; c++) out[c] = p.src[c][(size_t)zo * d.nxo + xo];
        } else {
            AxisPos ax = resize_axis(ix, d.xStartN, d.xStepN, d.xStartO, d.xStepO, p.xStepInvO, d.nxo);
            AxisPos az = resize_axis(iz, d.zStartN, d.zStepN, d.zStartO, d.zStepO, p.zStepInvO, d.nzo);
            float xr = (float)ax.rel, zr = (float)az.rel;
            float wx[4], wz[4];
            lagrange4(xr, wx);
            lagrange4(zr, wz);
            int irx = ax.ic - ax.st, irz = az.ic - az.st;
            irx = irx < 0 ? 0 : (irx > 2 ? 2 : irx);
            irz = irz < 0 ? 0 : (irz > 2 ? 2 : irz);
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const float2* __restrict__ o = p.src[c] + (size_t)az.st * d.nxo + ax.st;
                float2 f[4][4];
                bool low = false;
#pragma unroll
                for (int dz = 0; dz < 4; dz++)
#pragma unroll
                    for (int dx = 0; dx < 4; dx++) {
                        float2 v = __ldg(&o[(size_t)dz * d.nxo + dx]);
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
                    float fac = sqrtf(FI / app);
                    F.x *= fac; F.y *= fac;
                }
                out[c] = F;
            }
        }
        if (d.has_pw) {
            double ph = 0.;
            float2 f = make_float2(1.f, 0.f);
            bool zero = false;
            pw_eval(d.pw, ix, iz, ph, f, zero);
            float2 e = (d.pw.has_quad || d.pw.has_ang) ? cmul(f, expi(ph)) : f;
            if (zero) e = make_float2(0.f, 0.f);
            out[0] = cmul(out[0], e);
            out[1] = cmul(out[1], e);
        }
    }
    const size_t o = (size_t)iz * d.nxn + ix;
    __stcs(&p.dst[0][o], out[0]);
    __stcs(&p.dst[1][o], out[1]);
}

// ------------------------------------------------------------------------------------------------
// element-wise PW pass
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) pw_kernel(const PwLaunch p)
{
    __shared__ PwDesc d;
    if (threadIdx.x == 0) d = p.d;
    __syncthreads();
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y;
    if (ix >= d.nx) return;
    double ph = 0.;
    float2 f = make_float2(1.f, 0.f);
    bool zero = false;
    pw_eval(d.pw, ix, iz, ph, f, zero);
    float2 e = (d.pw.has_quad || d.pw.has_ang) ? cmul(f, expi(ph)) : f;
    if (zero) e = make_float2(0.f, 0.f);
    const int ox = d.mirror_x ? d.nx - 1 - ix : ix;
    const int oz = d.mirror_z ? d.nz - 1 - iz : iz;
    const size_t i = (size_t)iz * d.nx + ix, o = (size_t)oz * d.nx + ox;
#pragma unroll
    for (int c = 0; c < 2; c++) __stcs(&p.dst[c][o], cmul(e, __ldcs(&p.src[c][i])));
}

// ------------------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------------------
cudaError_t launch_line(const LineLaunch& p, cudaStream_t st)
{
    dim3 grid((p.nlines + p.L - 1) / p.L, 2);
    size_t smem = (size_t)p.L * p.P * sizeof(float2);
    static int attr_set = 0;
    if (smem > SRWG_LINE_SMEM_MAX) return cudaErrorInvalidValue;
    if (!attr_set) {
        cudaFuncSetAttribute(line_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SRWG_LINE_SMEM_MAX);
        cudaFuncSetAttribute(line2_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SRWG_LINE_SMEM_MAX);
        cudaFuncSetAttribute(line2_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SRWG_LINE_SMEM_MAX);
        attr_set = 1;
    }
    if (p.v2) {
        if (p.d.axis == 0) line2_kernel<false><<<grid, p.T * p.L, smem, st>>>(p);
        else line2_kernel<true><<<grid, p.T * p.L, smem, st>>>(p);
    } else {
        line_kernel<<<grid, p.T * p.G, smem, st>>>(p);
    }
    return cudaGetLastError();
}

cudaError_t launch_resize(const ResizeLaunch& p, cudaStream_t st)
{
    dim3 blk(64, 4);
    dim3 grid((p.d.nxn + blk.x - 1) / blk.x, (p.d.nzn + blk.y - 1) / blk.y);
    resize_kernel<<<grid, blk, 0, st>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_pw(const PwLaunch& p, cudaStream_t st)
{
    dim3 blk(256);
    dim3 grid((p.d.nx + 255) / 256, p.d.nz);
    pw_kernel<<<grid, blk, 0, st>>>(p);
    return cudaGetLastError();
}

}  // namespace srwg
