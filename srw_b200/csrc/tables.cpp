// Separable point-wise tables.  Every point-wise factor of this path -- quadratic and linear phases
// (lens, drift passes, resize quadratic-term removal/restoration), the separable c0*q^2 part of
// the angular transfer function, FFT centring signs and shift tables, scales and rectangular
// apertures -- is a product of a function of the index along a line and a function of the line.
// They are evaluated here once per plan in FP64 (phases reduced modulo 2*pi by the C library's
// cos/sin) and stored as complex FP32 tables, so the passes apply them with table reads and
// complex multiplies.  What is not separable (circular masks, rectangular obstacles, the quartic
// remainder of the angular transfer function) stays in PwOps 'extra' for the device.
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "kernels.h"
#include "planner.h"

namespace srwg {

typedef std::complex<double> cd;

struct SepPart {
    std::vector<double> ph;   // phase per index
    std::vector<char> zero;   // index masked out
    bool any = false;         // anything non-trivial
};

// splits PwOps of a pass whose lines run along `axis` (0: along = x index, line = z index)
static void separate(const PwOps& pw, int axis, int nAlong, int nLine, SepPart& A, SepPart& Lp, cd& scale,
                     PwOps& extra, int& has_extra)
{
    A.ph.assign(nAlong, 0.); A.zero.assign(nAlong, 0); A.any = false;
    Lp.ph.assign(nLine, 0.); Lp.zero.assign(nLine, 0); Lp.any = false;
    scale = cd(1., 0.);
    memset(&extra, 0, sizeof(extra));
    has_extra = 0;
    if (pw.has_quad) {
        double Aa = axis == 0 ? pw.Ai : pw.Aj, Ba = axis == 0 ? pw.Bi : pw.Bj;
        double Al = axis == 0 ? pw.Aj : pw.Ai, Bl = axis == 0 ? pw.Bj : pw.Bi;
        for (int a = 0; a < nAlong; a++) A.ph[a] += (Aa * a + Ba) * a + pw.C;
        for (int l = 0; l < nLine; l++) Lp.ph[l] += (Al * l + Bl) * l;
        A.any = Lp.any = true;
    }
    if (pw.has_ang) {
        double qa0 = axis == 0 ? pw.qx0 : pw.qz0, dqa = axis == 0 ? pw.dqx : pw.dqz;
        double ql0 = axis == 0 ? pw.qz0 : pw.qx0, dql = axis == 0 ? pw.dqz : pw.dqx;
        for (int a = 0; a < nAlong; a++) { double q = qa0 + a * dqa; A.ph[a] += pw.c0 * q * q; }
        for (int l = 0; l < nLine; l++) { double q = ql0 + l * dql; Lp.ph[l] += pw.c0 * q * q; }
        A.any = Lp.any = true;
        extra.has_ang = 1;
        extra.ang_resid = 1;
        extra.qx0 = pw.qx0; extra.dqx = pw.dqx; extra.qz0 = pw.qz0; extra.dqz = pw.dqz;
        extra.c0 = pw.c0; extra.c1 = pw.c1;
        has_extra = 1;
    }
    if (pw.has_bpx) {       // non-separable: evaluated per point in FP64 (common.cuh extra_eval)
        extra.has_bpx = 1;
        extra.bqx0 = pw.bqx0; extra.bdqx = pw.bdqx; extra.bqz0 = pw.bqz0; extra.bdqz = pw.bdqz;
        extra.blam = pw.blam; extra.bkL = pw.bkL; extra.btreat = pw.btreat;
        has_extra = 1;
    }
    if (pw.has_tr) {        // non-separable: table interpolation per point (common.cuh extra_eval)
        extra.has_tr = 1;
        extra.tr_id = pw.tr_id; extra.tr_nx = pw.tr_nx; extra.tr_nz = pw.tr_nz; extra.tr_outer = pw.tr_outer;
        extra.tr_off = pw.tr_off;
        extra.tr_x0 = pw.tr_x0; extra.tr_dx = pw.tr_dx; extra.tr_z0 = pw.tr_z0; extra.tr_dz = pw.tr_dz;
        extra.tr_xs = pw.tr_xs; extra.tr_xstep = pw.tr_xstep; extra.tr_zs = pw.tr_zs; extra.tr_zstep = pw.tr_zstep;
        extra.tr_k = pw.tr_k;
        has_extra = 1;
    }
    if (pw.has_scale) { scale = cd(pw.sre, pw.sim); A.any = true; }
    for (int m = 0; m < pw.nmask; m++) {
        const PwMask& k = pw.mask[m];
        if (k.type == 1 && !k.obstacle) {   // rectangular aperture: zero outside in x OR outside in z
            for (int a = 0; a < nAlong; a++) {
                double c0 = axis == 0 ? k.x0 : k.z0, dc = axis == 0 ? k.dx : k.dz, cc = axis == 0 ? k.cx : k.cz;
                double h = axis == 0 ? k.hx : k.hz;
                double r = (c0 + (double)a * dc) - cc;
                if ((r < -h) || (r > h)) A.zero[a] = 1;
            }
            for (int l = 0; l < nLine; l++) {
                double c0 = axis == 0 ? k.z0 : k.x0, dc = axis == 0 ? k.dz : k.dx, cc = axis == 0 ? k.cz : k.cx;
                double h = axis == 0 ? k.hz : k.hx;
                double r = (c0 + (double)l * dc) - cc;
                if ((r < -h) || (r > h)) Lp.zero[l] = 1;
            }
            A.any = Lp.any = true;
        } else {
            extra.mask[extra.nmask++] = k;
            has_extra = 1;
        }
    }
}

// cos(ph[i]) + i sin(ph[i]), i < n.  Cody-Waite reduction (W. J. Cody and W. Waite, Software Manual
// for the Elementary Functions, 1980): r = x - k pi/2, pi/2 split into two 33-bit parts and a
// remainder (from pi to 80 digits), so that k P1 and k P2 are exact for |k| < 2^20; sin r and cos r
// on [-pi/4, pi/4] by their Taylor series to degree 15 and 16 (truncation error below 1e-16); k mod 4
// swaps and signs them.  Phases beyond 2^20 pi/2 (1.6e6 rad) and non-finite ones go to the C
// library.  The loop has no branches, so that the compiler vectorises it; the tables of a plan hold
// about ten thousand factors, and the C library's sincos was two thirds of the planning time.
// Compiled for AVX2 as well (chosen at load time where the CPU has it; the same operations, so the
// same results), with the vectoriser's full cost model (the cheap one at -O2 leaves the loop scalar:
// 9 ns per value instead of 4).  The values go to separate cosine and sine arrays first.
__attribute__((target_clones("avx2", "default"), optimize("vect-cost-model=dynamic", "fp-contract=off")))
static void cis_n(const double* ph, cd* out, int n)
{
    const double P1 = 0x1.921fb544p+0, P2 = 0x1.0b4611a6p-34, P3 = 0x1.3198a2e037073p-69;
    const double TWO_OVER_PI = 0x1.45f306dc9c883p-1;
    const double RND = 6755399441055744.0;          // 2^52 + 2^51: adding and subtracting it rounds to nearest
    const double s3 = -1. / 6., s5 = 1. / 120., s7 = -1. / 5040., s9 = 1. / 362880., s11 = -1. / 39916800.,
                 s13 = 1. / 6227020800., s15 = -1. / 1307674368000.;
    const double c2 = -0.5, c4 = 1. / 24., c6 = -1. / 720., c8 = 1. / 40320., c10 = -1. / 3628800.,
                 c12 = 1. / 479001600., c14 = -1. / 87178291200., c16 = 1. / 20922789888000.;
    thread_local std::vector<double> re, im;        // scratch of the calling planner thread
    if ((int)re.size() < n) { re.resize(n); im.resize(n); }
    double* __restrict__ pr = re.data();
    double* __restrict__ pi = im.data();
    for (int i = 0; i < n; i++) {
        const double x = ph[i];
        const double k = (x * TWO_OVER_PI + RND) - RND;
        const double r = ((x - k * P1) - k * P2) - k * P3;
        const double r2 = r * r;
        const double sn = r + r * r2 * (s3 + r2 * (s5 + r2 * (s7 + r2 * (s9 + r2 * (s11 + r2 * (s13 + r2 * s15))))));
        const double cs =
            1. + r2 * (c2 + r2 * (c4 + r2 * (c6 + r2 * (c8 + r2 * (c10 + r2 * (c12 + r2 * (c14 + r2 * c16)))))));
        const int q = (int)k & 3;
        const double a = (q & 1) ? cs : sn, b = (q & 1) ? sn : cs;     // sin x, cos x up to signs
        pi[i] = (q & 2) ? -a : a;
        pr[i] = ((q + 1) & 2) ? -b : b;
    }
    for (int i = 0; i < n; i++) {
        if (!(std::fabs(ph[i]) < 1.6e6)) {
            double sn, cs;
            ::sincos(ph[i], &sn, &cs);
            pr[i] = cs;
            pi[i] = sn;
        }
        out[i] = cd(pr[i], pi[i]);
    }
}

static long long push(std::vector<float2>& T, const std::vector<cd>& v)
{
    const long long off = (long long)T.size();
    T.resize(T.size() + v.size());
    float2* d = T.data() + off;
    for (size_t i = 0; i < v.size(); i++) { d[i].x = (float)v[i].real(); d[i].y = (float)v[i].imag(); }
    return off;
}

// table of one chain W[k] = tab[k] * ltab[line] * extra * V[src(k)]:
// [post of a previous transform: rs1 / shift1 / scale1] -> [pw] -> [mirror] -> [pre of the next: rs2 / shift2]
static ChainTab chain_table(std::vector<float2>& T, int N, int nLine, int rs1, int sh1, double a1, float sc1,
                            const SepPart* A, const SepPart* Lp, cd scale, int mir, int rs2, int sh2, double a2)
{
    ChainTab ct;
    ct.tab = -1;
    ct.ltab = -1;
    bool along = rs1 || sh1 || sc1 != 1.f || (A && A->any) || rs2 || sh2 || scale != cd(1., 0.);
    if (along) {
        std::vector<cd> v(N);
        std::vector<double> ph(N), sg(N);
        std::vector<char> z(N);
        const int half = N >> 1;
        for (int k = 0; k < N; k++) {
            double g = 1., p = 0.;
            int m = k;
            if (rs2) { m = k + half; if (m >= N) m -= N; if (k & 1) g = -g; }
            if (sh2) p += a2 * (double)(m - half);
            int i = mir ? (N - 1 - m) : m;
            z[k] = 0;
            if (A) { p += A->ph[i]; z[k] = A->zero[i]; }
            int s = i;
            if (rs1) { s = i + half; if (s >= N) s -= N; if (s & 1) g = -g; }
            if (sh1) p += a1 * (double)(i - half);
            ph[k] = p;
            sg[k] = g;
        }
        cis_n(ph.data(), v.data(), N);
        for (int k = 0; k < N; k++) {
            // (sg sc1 scale) v, the complex product written out (std::complex's operator* goes through
            // a library call that also handles infinities and NaNs: none arise here)
            const cd f = (sg[k] * (double)sc1) * scale;
            const double vr = v[k].real(), vi = v[k].imag();
            v[k] = z[k] ? cd(0., 0.) : cd(f.real() * vr - f.imag() * vi, f.real() * vi + f.imag() * vr);
        }
        ct.tab = push(T, v);
    }
    if (Lp && Lp->any) {
        std::vector<cd> v(nLine);
        cis_n(Lp->ph.data(), v.data(), nLine);
        for (int l = 0; l < nLine; l++)
            if (Lp->zero[l]) v[l] = cd(0., 0.);
        ct.ltab = push(T, v);
    }
    return ct;
}

// RadResizeCore (sroptelm.cpp:3038-3337) index arithmetic along one axis, in the reference's FP64
// operation order (this file is compiled without FP contraction): for every new index in the
// window, the 4-point stencil start, the clipped sub-cell and the relative coordinate.
static long long resize_axis_table(std::vector<float2>& T, int nNew, long iS, long iE, double startN, double stepN,
                                   double startO, double stepO, int nO, bool only_larger)
{
    if (T.size() & 1) {                      // entries are read as 16-byte float4: keep them aligned
        float2 z; z.x = z.y = 0.f;
        T.push_back(z);
    }
    long long off = (long long)T.size();
    const double inv = 1. / stepO;
    for (int i = 0; i < nNew; i++) {
        ResizeAxis a;
        a.st = 0; a.ir = 0; a.rel = 0.f; a.pad = 0.f;
        if (i >= iS && i <= iE) {
            double absc = startN + (double)i * stepN;
            if (only_larger) {
                long o = (long)((absc - startO) * inv + 1.E-08);
                if (o < 0) o = 0;
                if (o > nO - 1) o = nO - 1;
                a.st = (int)o;
            } else {
                int ic = (int)((absc - startO) * inv + 1.E-06);
                double rel = absc - (startO + (double)ic * stepO);
                int st;
                if (ic == nO - 1) { st = ic - 3; rel += 2. * stepO; }
                else if (ic == nO - 2) { st = ic - 2; rel += stepO; }
                else if (ic == 0) { st = ic; rel -= stepO; }
                else st = ic - 1;
                // a new point outside the old mesh would make the reference read outside it: clamp
                if (st < 0) st = 0;
                if (st > nO - 4) st = nO - 4;
                int ir = ic - st;
                ir = ir < 0 ? 0 : (ir > 2 ? 2 : ir);
                a.st = st; a.ir = ir; a.rel = (float)(rel * inv);
            }
        }
        float2 f0, f1;
        memcpy(&f0, &a, sizeof(float2));
        memcpy(&f1, ((const char*)&a) + sizeof(float2), sizeof(float2));
        T.push_back(f0);
        T.push_back(f1);
    }
    return off;
}

// largest (max st - min st + 4) over the in-window new indices of each tile of `tile` new indices
static int tile_extent(const std::vector<float2>& T, long long off, int nNew, long iS, long iE, int tile)
{
    int best = 0;
    for (int t0 = 0; t0 < nNew; t0 += tile) {
        int lo = 1 << 30, hi = -1;
        for (int i = t0; i < t0 + tile && i < nNew; i++) {
            if (i < iS || i > iE) continue;
            ResizeAxis a;
            memcpy(&a, &T[off + 2 * i], sizeof(a));
            if (a.st < lo) lo = a.st;
            if (a.st > hi) hi = a.st;
        }
        if (hi >= lo && hi - lo + 4 > best) best = hi - lo + 4;
    }
    return best;
}

void build_tables(std::vector<KernelDesc>& ks, std::vector<float2>& T)
{
    T.clear();
    // room for the largest tables the passes can ask for (no reallocation while they are added)
    size_t most = 0;
    for (const KernelDesc& k : ks) {
        if (k.kind == K_LINE) most += 3 * (size_t)(k.line.nx + k.line.nz);
        else if (k.kind == K_RESIZE) most += 4 * (size_t)(k.rs.nxn + k.rs.nzn) + 2 * (size_t)(k.rs.nxo + k.rs.nzo) + 2;
        else if (reads_only(k.kind)) most += (size_t)(k.mom.nx + k.mom.nz);
        else most += (size_t)(k.pwk.nx + k.pwk.nz);
    }
    T.reserve(most);
    for (KernelDesc& k : ks) {
        if (k.kind == K_LINE) {
            LineDesc& d = k.line;
            int N = d.axis == 0 ? d.nx : d.nz, nl = d.axis == 0 ? d.nz : d.nx;
            SepPart A, Lp;
            cd scale(1., 0.);
            d.has_extra = 0;
            memset(&d.extra, 0, sizeof(d.extra));
            if (d.has_pw) separate(d.pw, d.axis, N, nl, A, Lp, scale, d.extra, d.has_extra);
            const SepPart* pA = d.has_pw ? &A : nullptr;
            const SepPart* pL = d.has_pw ? &Lp : nullptr;
            d.t_pre = chain_table(T, N, nl, 0, 0, 0., 1.f, nullptr, nullptr, cd(1., 0.), 0, d.f1_pre.rs,
                                  d.f1_pre.has_shift, d.f1_pre.shift_a);
            int rs1 = 0, sh1 = 0, rs2 = 0, sh2 = 0;
            double a1 = 0., a2 = 0.;
            float sc1 = 1.f;
            if (d.f1) { rs1 = d.f1_post.rs; sh1 = d.f1_post.has_shift; a1 = d.f1_post.shift_a; sc1 = d.f1_post.scale; }
            if (d.f2) { rs2 = d.f2_pre.rs; sh2 = d.f2_pre.has_shift; a2 = d.f2_pre.shift_a; }
            d.t_mid = chain_table(T, N, nl, rs1, sh1, a1, sc1, pA, pL, scale, d.mirror_along, rs2, sh2, a2);
            d.t_fin.tab = d.t_fin.ltab = -1;
            if (d.f2)
                d.t_fin = chain_table(T, N, nl, d.f2_post.rs, d.f2_post.has_shift, d.f2_post.shift_a, d.f2_post.scale,
                                      nullptr, nullptr, cd(1., 0.), 0, 0, 0, 0.);
        } else if (k.kind == K_RESIZE) {
            ResizeDesc& r = k.rs;
            r.t.tab = r.t.ltab = -1;
            r.has_extra = 0;
            memset(&r.extra, 0, sizeof(r.extra));
            if (r.has_pw) {
                SepPart A, Lp;
                cd scale;
                separate(r.pw, 0, r.nxn, r.nzn, A, Lp, scale, r.extra, r.has_extra);
                r.t = chain_table(T, r.nxn, r.nzn, 0, 0, 0., 1.f, &A, &Lp, scale, 0, 0, 0, 0.);
            }
            r.tp.tab = r.tp.ltab = -1;
            r.has_pre_extra = 0;
            memset(&r.pre_extra, 0, sizeof(r.pre_extra));
            if (r.has_pre) {
                SepPart A, Lp;
                cd scale;
                separate(r.pre, 0, r.nxo, r.nzo, A, Lp, scale, r.pre_extra, r.has_pre_extra);
                r.tp = chain_table(T, r.nxo, r.nzo, 0, 0, 0., 1.f, &A, &Lp, scale, 0, 0, 0, 0.);
            }
            r.axx = resize_axis_table(T, r.nxn, r.ixStart, r.ixEnd, r.xStartN, r.xStepN, r.xStartO, r.xStepO, r.nxo,
                                      r.only_larger != 0);
            r.axz = resize_axis_table(T, r.nzn, r.izStart, r.izEnd, r.zStartN, r.zStepN, r.zStartO, r.zStepO, r.nzo,
                                      r.only_larger != 0);
            r.tile_or = r.tile_oc = 0;
            if (!r.only_larger) {
                // largest old extent (stencil rows / columns) over the tiles of the tiled kernel
                const int er = tile_extent(T, r.axz, r.nzn, r.izStart, r.izEnd, SRWG_RESIZE_TZ);
                const int ec = tile_extent(T, r.axx, r.nxn, r.ixStart, r.ixEnd, SRWG_RESIZE_TX);
                if (er > 0 && ec > 0 && er <= SRWG_RESIZE_OR_MAX && ec <= SRWG_RESIZE_OC_MAX) {
                    r.tile_or = er;
                    r.tile_oc = ec;
                }
            }
        } else if (reads_only(k.kind)) {
            MomDesc& m = k.mom;
            SepPart A, Lp;
            cd scale;
            m.has_extra = 0;
            memset(&m.extra, 0, sizeof(m.extra));
            separate(m.pw, 0, m.nx, m.nz, A, Lp, scale, m.extra, m.has_extra);
            m.t = chain_table(T, m.nx, m.nz, 0, 0, 0., 1.f, &A, &Lp, scale, 0, 0, 0, 0.);
        } else {
            PwDesc& p = k.pwk;
            SepPart A, Lp;
            cd scale;
            separate(p.pw, 0, p.nx, p.nz, A, Lp, scale, p.extra, p.has_extra);
            p.t = chain_table(T, p.nx, p.nz, 0, 0, 0., 1.f, &A, &Lp, scale, 0, 0, 0, 0.);
        }
    }
}

}  // namespace srwg
