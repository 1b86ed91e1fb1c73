// Host planner (see planner.h).  Every mesh / radius / centre / moment update below follows the
// reference's statement order in FP64 (compiled without FP contraction), so resized and
// transformed meshes are bit-identical to the reference's; the field work is only described
// (kdesc.h) and fused into as few GPU passes as possible by Builder.
#include "kernels.h"
#include "exec.h"
#include "planner.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "errors.h"

namespace srwg {

// ================================================================================================
// FFT good numbers (CGenMathFFT::NextCorrectNumberForFFT, cpp/src/ext/genmath/gmfft.cpp:156-228).
// The reference's table (gmfft.cpp:26) holds the even n <= 100000 of the form 2^a 3^b 5^c 7^d 11^e
// 13^f with e, f <= 1; it is generated here from that rule.
// ================================================================================================
static std::vector<long> make_good_numbers()
{
    std::vector<long> g;
    for (long n = 2; n <= 100000; n += 2) {
        long m = n;
        while (m % 2 == 0) m /= 2;
        while (m % 3 == 0) m /= 3;
        while (m % 5 == 0) m /= 5;
        while (m % 7 == 0) m /= 7;
        if (m % 11 == 0) m /= 11;
        if (m % 13 == 0) m /= 13;
        if (m == 1) g.push_back(n);
    }
    return g;
}

static const std::vector<long>& good_numbers()
{
    static const std::vector<long> g = make_good_numbers();     // initialised once, thread-safe
    return g;
}

long next_correct_number_for_fft(long n)
{
    if (n < 4) return 4;
    if (n < 100001) {
        const std::vector<long>& g = good_numbers();
        return *std::lower_bound(g.begin(), g.end(), n);
    }
    const double mults[] = {10. / 9., 9. / 8., 6. / 5., 5. / 4., 4. / 3., 3. / 2., 8. / 5., 5. / 3., 16. / 9., 15. / 8.};
    long k = 99000;
    for (int j = 0; j < 100; j++) {
        for (int m = 0; m < 10; m++) {
            double dk = k * mults[m];
            long kt = (long)dk;
            if ((dk - (double)kt) >= 0.5) kt++;
            if (n <= kt) return kt;
        }
        k <<= 1;
        if (n <= k) return k;
    }
    return n;
}

// ================================================================================================
// Builder: fuses the stream of point-wise operators, centred 2D FFTs, resizes and mirrors into
// LINE / RESIZE / PW passes.
//
//  - a 2D FFT is split into an x transform (row pass) and a z transform (column pass); the first
//    half closes the currently open line pass of the same axis (as its second transform) when
//    there is one, the second half opens a pass of the other axis whose middle section then
//    collects the following point-wise operators;
//  - point-wise operators are converted to the index space of the open pass at the time they
//    are added (so later re-labelling of the mesh or mirrors inside the pass are accounted for);
//  - a resize closes everything before it and opens a RESIZE pass that collects the operators
//    on the new mesh.
// ================================================================================================
class Builder {
public:
    std::vector<KernelDesc>& ks;
    long long& maxElems;
    int cur = 0;       // buffer with the current field (0: caller's input)
    int open = -1;     // pass collecting point-wise operators
    int fx = 0, fz = 0;
    Builder(std::vector<KernelDesc>& k, long long& me) : ks(k), maxElems(me) {}

    int next_buf() const { return cur == 1 ? 2 : 1; }
    KernelDesc& newk(int kind, int nx, int nz)
    {
        KernelDesc k;
        memset(&k, 0, sizeof(k));
        k.kind = kind;
        k.src = cur;
        k.dst = next_buf();
        cur = k.dst;
        long long e = (long long)nx * nz;
        if (e > maxElems) maxElems = e;
        ks.push_back(k);
        return ks.back();
    }
    void close() { open = -1; fx = fz = 0; }

    PwOps* open_ops()
    {
        if (open < 0) return nullptr;
        KernelDesc& k = ks[open];
        if (k.kind == K_LINE) { k.line.has_pw = 1; return &k.line.pw; }
        if (k.kind == K_RESIZE) { k.rs.has_pw = 1; return &k.rs.pw; }
        return &k.pwk.pw;
    }
    PwOps* ensure(const WfrState& w)
    {
        if (open < 0) {
            KernelDesc& k = newk(K_PW, w.nx, w.nz);
            k.pwk.nx = w.nx;
            k.pwk.nz = w.nz;
            open = (int)ks.size() - 1;
            fx = fz = 0;
        }
        return open_ops();
    }
    // affine map: kernel index -> physical coordinate of the current logical mesh
    void axis_map(const WfrState& w, double& X0, double& DX, double& Z0, double& DZ) const
    {
        if (fx) { X0 = w.xStart + (w.nx - 1) * w.xStep; DX = -w.xStep; }
        else { X0 = w.xStart; DX = w.xStep; }
        if (fz) { Z0 = w.zStart + (w.nz - 1) * w.zStep; DZ = -w.zStep; }
        else { Z0 = w.zStart; DZ = w.zStep; }
    }
    // phase += ax x^2 + bx x + az z^2 + bz z + c  (x, z physical on the current mesh)
    void quad(const WfrState& w, double ax, double bx, double az, double bz, double c)
    {
        PwOps* p = ensure(w);
        double X0, DX, Z0, DZ;
        axis_map(w, X0, DX, Z0, DZ);
        add_quad(p, X0, DX, Z0, DZ, ax, bx, az, bz, c);
    }
    static void add_quad(PwOps* p, double X0, double DX, double Z0, double DZ, double ax, double bx, double az,
                         double bz, double c)
    {
        p->has_quad = 1;
        p->Ai += ax * DX * DX;
        p->Bi += (2. * ax * X0 + bx) * DX;
        p->Aj += az * DZ * DZ;
        p->Bj += (2. * az * Z0 + bz) * DZ;
        p->C += ax * X0 * X0 + bx * X0 + az * Z0 * Z0 + bz * Z0 + c;
    }
    // read-only moment pass on the current field (index order = the logical mesh).  The operators
    // still pending in an element-wise pass are applied on the fly by the moment pass, which runs
    // just before that pass and reads its source; the element-wise pass stays open.
    MomDesc& moments(const WfrState& w, int kind = K_MOM)
    {
        KernelDesc k;
        memset(&k, 0, sizeof(k));
        k.kind = kind;
        if (open >= 0 && open == (int)ks.size() - 1 && ks[open].kind == K_PW && !fx && !fz &&
            !ks[open].pwk.mirror_x && !ks[open].pwk.mirror_z && ks[open].pwk.nx == w.nx && ks[open].pwk.nz == w.nz) {
            k.src = k.dst = ks[open].src;
            k.mom.pw = ks[open].pwk.pw;
            ks.insert(ks.begin() + open, k);
            open++;
            return ks[open - 1].mom;
        }
        close();
        k.src = k.dst = cur;
        ks.push_back(k);
        return ks.back().mom;
    }
    // transmission table on the current (coordinate) mesh
    void transm(const WfrState& w, const ElemDesc& e)
    {
        PwOps* p = ensure(w);
        if (p->has_tr) {
            close();
            p = ensure(w);
        }
        double X0, DX, Z0, DZ;
        axis_map(w, X0, DX, Z0, DZ);
        p->has_tr = 1;
        p->tr_id = e.tr; p->tr_nx = e.trNx; p->tr_nz = e.trNz;
        p->tr_outer = e.extTr + 1;        // OuterTransmIs (sroptgtr.cpp:142)
        p->tr_off = -1;
        p->tr_x0 = X0; p->tr_dx = DX; p->tr_z0 = Z0; p->tr_dz = DZ;
        p->tr_xs = e.trXs; p->tr_xstep = (e.trXf - e.trXs) / (e.trNx - 1);
        p->tr_zs = e.trZs; p->tr_zstep = (e.trZf - e.trZs) / (e.trNz - 1);
        p->tr_k = w.eStart * 5.0676816042E+06;   // 2 pi / lambda [1/m] (sroptgtr.h:287)
    }
    // exact beyond-paraxial propagator phase on the current (angular-frequency) mesh
    void bpx(const WfrState& w, double lam, double kL, int treat)
    {
        PwOps* p = ensure(w);
        if (p->has_bpx) {
            close();
            p = ensure(w);
        }
        double X0, DX, Z0, DZ;
        axis_map(w, X0, DX, Z0, DZ);
        p->has_bpx = 1;
        p->bqx0 = X0; p->bdqx = DX; p->bqz0 = Z0; p->bdqz = DZ;
        p->blam = lam; p->bkL = kL; p->btreat = treat;
    }
    void ang(const WfrState& w, double c0, double c1, double cconst)
    {
        PwOps* p = ensure(w);
        if (p->has_ang) {      // one angular transfer function per pass: materialise first
            close();
            p = ensure(w);
        }
        double X0, DX, Z0, DZ;
        axis_map(w, X0, DX, Z0, DZ);
        p->has_ang = 1;
        p->qx0 = X0; p->dqx = DX; p->qz0 = Z0; p->dqz = DZ;
        p->c0 = c0; p->c1 = c1;
        if (cconst != 0.) { p->has_quad = 1; p->C += cconst; }
    }
    void mask(const WfrState& w, int type, int obstacle, double cx, double cz, double hx, double hz, double r2)
    {
        PwOps* p = ensure(w);
        if (p->nmask >= SRWG_MAX_MASKS) {
            close();
            p = ensure(w);
        }
        PwMask& m = p->mask[p->nmask++];
        axis_map(w, m.x0, m.dx, m.z0, m.dz);
        m.type = type; m.obstacle = obstacle;
        m.cx = cx; m.cz = cz; m.hx = hx; m.hz = hz; m.r2 = r2;
    }
    void scale(const WfrState& w, float re, float im)
    {
        PwOps* p = ensure(w);
        if (!p->has_scale) { p->has_scale = 1; p->sre = re; p->sim = im; }
        else {
            float r = p->sre * re - p->sim * im, i = p->sre * im + p->sim * re;
            p->sre = r; p->sim = i;
        }
    }
    // centred 2D FFT on a (nx, nz) mesh; sides per axis
    void fft2(int nx, int nz, int dir, const FftSide& xpre, const FftSide& xpost, const FftSide& zpre,
              const FftSide& zpost)
    {
        int A = 0;
        bool reuse = (open >= 0) && ks[open].kind == K_LINE && ks[open].line.f2 == 0;
        bool upgrade = (open >= 0) && ks[open].kind == K_PW;
        if (reuse) {
            LineDesc& d = ks[open].line;
            A = d.axis;
            d.f2 = dir;
            d.f2_pre = A == 0 ? xpre : zpre;
            d.f2_post = A == 0 ? xpost : zpost;
            close();
        } else if (upgrade) {
            // a pending element-wise pass becomes the row pass of the transform: its operators
            // (and mirrors) run in shared memory just before the row FFT
            KernelDesc& k = ks[open];
            PwDesc pd = k.pwk;
            memset(&k.line, 0, sizeof(k.line));
            k.kind = K_LINE;
            k.line.axis = 0; k.line.nx = nx; k.line.nz = nz;
            k.line.has_pw = 1; k.line.pw = pd.pw;
            k.line.mirror_along = pd.mirror_x; k.line.mirror_lines = pd.mirror_z;
            k.line.f2 = dir; k.line.f2_pre = xpre; k.line.f2_post = xpost;
            A = 0;
            close();
        } else {
            close();
            KernelDesc& k = newk(K_LINE, nx, nz);
            k.line.axis = 0; k.line.nx = nx; k.line.nz = nz;
            k.line.f2 = dir; k.line.f2_pre = xpre; k.line.f2_post = xpost;
            A = 0;
        }
        int B = 1 - A;
        KernelDesc& k = newk(K_LINE, nx, nz);
        k.line.axis = B; k.line.nx = nx; k.line.nz = nz;
        k.line.f1 = dir;
        k.line.f1_pre = B == 0 ? xpre : zpre;
        k.line.f1_post = B == 0 ? xpost : zpost;
        open = (int)ks.size() - 1;
        fx = fz = 0;
    }
    void mirror(const WfrState& w, int sx, int sz)
    {
        int mx = sx < 0, mz = sz < 0;
        if (!mx && !mz) return;
        if (open >= 0 && ks[open].kind == K_LINE) {
            LineDesc& d = ks[open].line;
            if (d.axis == 0) { d.mirror_along ^= mx; d.mirror_lines ^= mz; }
            else { d.mirror_along ^= mz; d.mirror_lines ^= mx; }
        } else {
            if (open >= 0 && ks[open].kind == K_RESIZE) close();
            ensure(w);
            PwDesc& d = ks[open].pwk;
            d.mirror_x ^= mx; d.mirror_z ^= mz;
        }
        fx ^= mx;
        fz ^= mz;
    }
    void resize(const WfrState& o, const WfrState& n, int only_larger)
    {
        // a pending element-wise pass without mirrors on the old mesh is folded into the resize
        // (applied to the old points as they are gathered)
        PwOps pre;
        int has_pre = 0;
        if (!only_larger && open >= 0 && open == (int)ks.size() - 1 && ks[open].kind == K_PW &&
            !ks[open].pwk.mirror_x && !ks[open].pwk.mirror_z && ks[open].pwk.nx == o.nx && ks[open].pwk.nz == o.nz) {
            pre = ks[open].pwk.pw;
            has_pre = 1;
            cur = ks[open].src;
            ks.pop_back();
        }
        close();
        KernelDesc& k = newk(K_RESIZE, n.nx, n.nz);
        if (has_pre) { k.rs.has_pre = 1; k.rs.pre = pre; }
        ResizeDesc& r = k.rs;
        r.nxo = o.nx; r.nzo = o.nz; r.nxn = n.nx; r.nzn = n.nz;
        r.xStartO = o.xStart; r.xStepO = o.xStep; r.zStartO = o.zStart; r.zStepO = o.zStep;
        r.xStartN = n.xStart; r.xStepN = n.xStep; r.zStartN = n.zStart; r.zStepN = n.zStep;
        r.ixStart = n.AuxLong1; r.ixEnd = n.AuxLong2; r.izStart = n.AuxLong3; r.izEnd = n.AuxLong4;
        r.only_larger = only_larger;
        open = (int)ks.size() - 1;
        fx = fz = 0;
    }
};

// ================================================================================================
// SRWLOptC parsing (srTCompositeOptElem ctor, cpp/src/core/sroptcnt.cpp:87-221)
// ================================================================================================
// the propagation parameter list of entry i of a container (srTRadResize defaults when it has none)
static PropDesc prop_desc(const SRWLOptC* opt, int i)
{
    PropDesc pd;
    pd.n = 0;
    for (int k = 0; k < 17; k++) pd.pp[k] = 0;
    pd.pp[2] = 1.; pd.pp[5] = pd.pp[6] = pd.pp[7] = pd.pp[8] = 1.;
    if (i < opt->nProp && opt->arProp[i] != nullptr) {
        int n = 9;
        if (opt->arPropN != nullptr) n = opt->arPropN[i];
        if (n > 17) n = 17;
        for (int k = 0; k < n; k++) pd.pp[k] = opt->arProp[i][k];
        pd.n = n;
    } else {
        pd.n = -1;   // default instruction: no resize
    }
    return pd;
}

int Planner::flatten(const SRWLOptC* opt, std::vector<ElemDesc>& els, std::vector<PropDesc>& props, bool nested)
{
    if (opt == nullptr || opt->nElem <= 0 || opt->arOpt == nullptr || opt->arOptTypes == nullptr)
        return UNKNOWN_OPTICAL_ELEMENT;
    for (int i = 0; i <= opt->nElem; i++) {
        bool isElem = false;
        if (i < opt->nElem) {
            void* p = opt->arOpt[i];
            const char* t = opt->arOptTypes[i];
            if (p == nullptr || t == nullptr) return UNKNOWN_OPTICAL_ELEMENT;
            ElemDesc e;
            if (strcmp(t, "drift") == 0) {
                const SRWLOptD* d = (const SRWLOptD*)p;
                e.kind = E_DRIFT; e.L = d->L; e.treat = d->treat;
            } else if (strcmp(t, "aperture") == 0 || strcmp(t, "obstacle") == 0) {
                const SRWLOptA* a = (const SRWLOptA*)p;
                e.kind = E_APERTURE; e.shape = a->shape; e.Dx = a->Dx; e.Dy = a->Dy; e.x = a->x; e.y = a->y;
                if (a->ap_or_ob == 'a' || a->ap_or_ob == 'A') e.apob = 'a';
                else if (a->ap_or_ob == 'o' || a->ap_or_ob == 'O') e.apob = 'o';
                else return UNKNOWN_OPTICAL_ELEMENT;
                if (e.shape != 'r' && e.shape != 'c') { isElem = false; goto props_only; }
            } else if (strcmp(t, "lens") == 0) {
                const SRWLOptL* l = (const SRWLOptL*)p;
                e.kind = E_LENS; e.Fx = l->Fx; e.Fy = l->Fy; e.x = l->x; e.y = l->y;
            } else if (strcmp(t, "transmission") == 0) {
                // srTGenTransmission(const SRWLOptT&) (sroptgtr.cpp:139): table over the element's
                // mesh, centre = the mesh's centre, estimated focal lengths for the bookkeeping
                const SRWLOptT* tr = (const SRWLOptT*)p;
                if (tr->arTr == nullptr || tr->mesh.nx < 2 || tr->mesh.ny < 2) return UNKNOWN_OPTICAL_ELEMENT;
                if (tr->mesh.ne < 1) return UNKNOWN_OPTICAL_ELEMENT;
                e.kind = E_TRANSM;
                e.Fx = tr->Fx; e.Fy = tr->Fy;
                e.x = 0.5 * (tr->mesh.xStart + tr->mesh.xFin);
                e.y = 0.5 * (tr->mesh.yStart + tr->mesh.yFin);
                e.trNx = (int)tr->mesh.nx; e.trNz = (int)tr->mesh.ny; e.extTr = tr->extTr;
                e.trXs = tr->mesh.xStart; e.trXf = tr->mesh.xFin; e.trZs = tr->mesh.yStart; e.trZf = tr->mesh.yFin;
                e.tr = (int)trTables_.size();
                if (tr->mesh.ne == 1) {
                    trTables_.emplace_back(tr->arTr, tr->arTr + 2 * (size_t)e.trNx * e.trNz);
                } else {
                    // a table vs photon energy ([ny][nx][ne] pairs): linear in e at the wavefront's
                    // photon energy (the e part of the trilinear lookup, sroptgtr.h:275-300: cell by
                    // truncation with 1e-10, clamped to the last cell, extrapolating outside), then
                    // the (x, z) lookup of a single-energy table
                    const long long Ne = tr->mesh.ne;
                    const double eS = tr->mesh.eStart, eSt = (tr->mesh.eFin - tr->mesh.eStart) / (Ne - 1);
                    long long ie = (long long)((w.eStart - eS) / eSt + 1.e-10);
                    if (ie < 0) ie = 0;
                    else if (ie > Ne - 2) ie = Ne - 2;
                    const double er = (w.eStart - (ie * eSt + eS)) / eSt;
                    std::vector<double> t(2 * (size_t)e.trNx * e.trNz);
                    for (size_t q = 0; q < (size_t)e.trNx * e.trNz; q++)
                        for (int c2 = 0; c2 < 2; c2++) {
                            const double* p0 = tr->arTr + (q * Ne + ie) * 2 + c2;
                            t[2 * q + c2] = p0[0] * (1. - er) + p0[2] * er;
                        }
                    trTables_.push_back(std::move(t));
                }
            } else if (strcmp(t, "container") == 0) {
                // a nested container is one element of the outer chain (sroptcnt.cpp:171): the outer
                // chain's pre-resize for it comes first, then every element inside it (nested
                // containers included) propagates with the outer entry's parameters, its own lists
                // unused (srTCompositeOptElem::PropagateRadiation, sroptcnt.h:52-76)
                std::vector<ElemDesc> sub;
                std::vector<PropDesc> subp;
                int r = flatten((const SRWLOptC*)p, sub, subp, true);
                if (r) return r;
                PropDesc pd;
                const bool withProps = opt->arProp != nullptr;
                if (withProps) pd = prop_desc(opt, i);
                for (size_t j = 0; j < sub.size(); j++) {
                    sub[j].outer = i;
                    els.push_back(sub[j]);
                    if (withProps) {
                        PropDesc q = pd;           // after the first: the same treatment, no resize
                        if (j > 0) {
                            for (int k = 5; k <= 8; k++) q.pp[k] = 1.;
                            for (int k = 9; k <= 11; k++) q.pp[k] = 0.;
                        }
                        props.push_back(q);
                    }
                }
                continue;
            } else {
                err = std::string("optical element type not supported on the GPU path: ") + t;
                return SRWG_ERR_UNSUPPORTED;
            }
            e.outer = i;
            els.push_back(e);
            isElem = true;
        }
    props_only:
        if (opt->arProp != nullptr && (isElem || i == opt->nElem)) props.push_back(prop_desc(opt, i));
    }
    (void)nested;
    return 0;
}

// ================================================================================================
// wavefront bookkeeping helpers (srradstr.cpp / srradstr.h)
// ================================================================================================
void Planner::set_full_range()
{   // SetNonZeroWavefrontLimitsToFullRange (srradstr.h:339)
    w.xWfrMin = w.xStart;
    w.xWfrMax = w.xStart + w.nx * w.xStep;
    w.zWfrMin = w.zStart;
    w.zWfrMax = w.zStart + w.nz * w.zStep;
}

void Planner::srwl_roundtrip()
{   // ModifyWfrNeNxNz (srradstr.cpp:760): OutSRWRadPtrs then InSRWRadPtrs on the client struct
    double xFin = w.xStart + w.xStep * (w.nx - 1);
    double yFin = w.zStart + w.zStep * (w.nz - 1);
    double xS = w.xStart, yS = w.zStart;
    if (w.nx <= 1) { w.xStart = 0.5 * (xS + xFin); w.xStep = 0.; }
    else { w.xStart = xS; w.xStep = (xFin - xS) / (w.nx - 1); }
    if (w.nz <= 1) { w.zStart = 0.5 * (yS + yFin); w.zStep = 0.; }
    else { w.zStart = yS; w.zStep = (yFin - yS) / (w.nz - 1); }
    w.xWfrMin = xS; w.xWfrMax = xFin;
    w.zWfrMin = yS; w.zWfrMax = yFin;
}

// One centred 2D FFT (CGenMathFFT2D::Make2DFFT, gmfft.cpp:295-897): computes the transformed
// mesh (SetupLimitsTr, gmfft.h:232) and the per-axis side operations, and emits the transform.
void Planner::fft2_emit(int dir, bool use_given, double& xStepTr, double& zStepTr, double& xStartTr, double& zStartTr)
{
    const double RelShiftTol = 1.E-06;
    long Nx = w.nx, Ny = w.nz;
    long HalfNx = Nx >> 1, HalfNy = Ny >> 1;
    double xStartTr0 = -0.5 / w.xStep;
    xStepTr = -xStartTr0 / HalfNx;
    double yStartTr0 = -0.5 / w.zStep;
    zStepTr = -yStartTr0 / HalfNy;
    if (use_given) { xStartTr = w.xStartTr; zStartTr = w.zStartTr; }
    else { xStartTr = xStartTr0; zStartTr = yStartTr0; }
    double xStepNx = Nx * w.xStep, yStepNy = Ny * w.zStep;
    double x0_After = w.xStart + 0.5 * xStepNx;
    double y0_After = w.zStart + 0.5 * yStepNy;
    bool aftX = ::fabs(x0_After) > RelShiftTol * xStepNx;
    bool aftY = ::fabs(y0_After) > RelShiftTol * yStepNy;
    bool befX = false, befY = false;
    double x0_Before = 0., y0_Before = 0.;
    if (use_given) {
        x0_Before = w.xStartTr - xStartTr0;
        y0_Before = w.zStartTr - yStartTr0;
        befX = ::fabs(x0_Before) > RelShiftTol * ::fabs(xStartTr0);
        befY = ::fabs(y0_Before) > RelShiftTol * ::fabs(yStartTr0);
    }
    double sg = (dir > 0) ? -1. : 1.;
    const double twoPi = 6.283185307179586477;
    FftSide xpre{}, xpost{}, zpre{}, zpost{};
    xpre.scale = xpost.scale = zpre.scale = zpost.scale = 1.f;
    // FillArrayShift (gmfft.h:250): exp(i 2 pi t0 (k - N/2) tStep)
    if (befX) { xpre.has_shift = 1; xpre.shift_a = twoPi * (sg * x0_Before) * w.xStep; }
    if (befY) { zpre.has_shift = 1; zpre.shift_a = twoPi * (sg * y0_Before) * w.zStep; }
    if (aftX) { xpost.has_shift = 1; xpost.shift_a = twoPi * (sg * x0_After) * xStepTr; }
    if (aftY) { zpost.has_shift = 1; zpost.shift_a = twoPi * (sg * y0_After) * zStepTr; }
    if (dir > 0) { xpost.rs = 1; zpost.rs = 1; }     // RepairSign then Rotate after the forward FFT
    else { xpre.rs = 1; zpre.rs = 1; }               // Rotate then RepairSign before the backward FFT
    zpost.scale = (float)(w.xStep * w.zStep);        // NormalizeDataAfter2DFFT (x dx dy)
    b->fft2(w.nx, w.nz, dir, xpre, xpost, zpre, zpost);
}

void Planner::set_rad_repres(int to)
{   // srTGenOptElem::SetRadRepres (sroptelm.cpp:1243-1528), ne == 1; edge correction is never on
    if (w.Pres == to) return;
    int dir = (to == 0) ? -1 : 1;
    bool use_given = (w.AuxLong4 == 7777777) || ((to == 0) && w.UseStartTrToShiftAtChangingRepresToCoord);
    double xs, zs, x0, z0;
    fft2_emit(dir, use_given, xs, zs, x0, z0);
    w.xStep = xs; w.zStep = zs; w.xStart = x0; w.zStart = z0;
    w.Pres = to;
    set_full_range();
}

void Planner::mirror(int sx, int sz)
{
    b->mirror(w, sx, sz);
}

// ================================================================================================
// Drift space (cpp/src/core/sroptdrf.h, sroptdrf.cpp)
// ================================================================================================
static const double PI_D_LAMBDA_PER_EV = 2.53384080189E+06;   // sroptdrf.h:479
static const double INV_LAMBDA_PER_EV = 806546.577258;         // sroptdrf.h:481
static const double LAMBDA_EV_M = 1.239842e-06;                // sroptdrf.h:617

double Planner::diff_lim_spot(char xz, double L) const
{   // DiffractionLimitedPropagatedSpotSize (sroptdrf.h:1020)
    double lam = LAMBDA_EV_M / w.eStart;
    double dLim = (xz == 'x') ? (w.nx - 1) * w.xStep : (w.nz - 1) * w.zStep;
    double dWfr = (xz == 'x') ? (w.xWfrMax - w.xWfrMin) : (w.zWfrMax - w.zWfrMin);
    double d = ((dWfr > 0.) && (dWfr < dLim)) ? dWfr : dLim;
    return lam * L / d;
}

static void mom_apply(double* m, const double ax[2][2], const double az[2][2])
{   // MultSquareMatrByVect steps of AuxPropagateRadMoments / GenAuxPropagateRadMoments
    double bx[3][3] = {{ax[0][0] * ax[0][0], 2. * ax[0][0] * ax[0][1], ax[0][1] * ax[0][1]},
                       {ax[0][0] * ax[1][0], ax[0][1] * ax[1][0] + ax[0][0] * ax[1][1], ax[0][1] * ax[1][1]},
                       {ax[1][0] * ax[1][0], 2. * ax[1][0] * ax[1][1], ax[1][1] * ax[1][1]}};
    double bz[3][3] = {{az[0][0] * az[0][0], 2. * az[0][0] * az[0][1], az[0][1] * az[0][1]},
                       {az[0][0] * az[1][0], az[0][1] * az[1][0] + az[0][0] * az[1][1], az[0][1] * az[1][1]},
                       {az[1][0] * az[1][0], 2. * az[1][0] * az[1][1], az[1][1] * az[1][1]}};
    double v2[2], v3[3];
    v2[0] = m[1]; v2[1] = m[2];
    for (int i = 0; i < 2; i++) { double s = 0; for (int j = 0; j < 2; j++) s += ax[i][j] * v2[j]; m[1 + i] = s; }
    v2[0] = m[3]; v2[1] = m[4];
    for (int i = 0; i < 2; i++) { double s = 0; for (int j = 0; j < 2; j++) s += az[i][j] * v2[j]; m[3 + i] = s; }
    v3[0] = m[5]; v3[1] = m[6]; v3[2] = m[7];
    for (int i = 0; i < 3; i++) { double s = 0; for (int j = 0; j < 3; j++) s += bx[i][j] * v3[j]; m[5 + i] = s; }
    v3[0] = m[8]; v3[1] = m[9]; v3[2] = m[10];
    for (int i = 0; i < 3; i++) { double s = 0; for (int j = 0; j < 3; j++) s += bz[i][j] * v3[j]; m[8 + i] = s; }
}

static void apply_matrix_op(const MomOp& op, double* m)
{
    if (!op.clamp) { mom_apply(m, op.ax, op.az); return; }
    if (m[0] == 0.) return;
    mom_apply(m, op.ax, op.az);
    if (m[5] - m[1] * m[1] < op.sx * op.sx) m[5] = op.sx * op.sx + m[1] * m[1];
    if (m[8] - m[3] * m[3] < op.sz * op.sz) m[8] = op.sz * op.sz + m[3] * m[3];
}

void Planner::record_matrix(const double ax[2][2], const double az[2][2], int clamp, double sx, double sz)
{
    MomOp op;
    op.kind = MOP_MATRIX;
    memcpy(op.ax, ax, sizeof(op.ax));
    memcpy(op.az, az, sizeof(op.az));
    op.clamp = clamp; op.sx = sx; op.sz = sz;
    momOps.push_back(op);
    apply_matrix_op(op, w.momX);
    apply_matrix_op(op, w.momZ);
}

void Planner::drift_moments(double L)
{   // srTDriftSpace::PropagateRadMoments -> AuxPropagateRadMoments (sroptdrf.h:967, sroptdrf.cpp:22):
    // drift matrices, then the rms sizes floored at the diffraction-limited spot
    const double a[2][2] = {{1., L}, {0., 1.}};
    record_matrix(a, a, 1, diff_lim_spot('x', L), diff_lim_spot('z', L));
}

// CheckIfMomentsShouldBeRecomputed of the rectangular / circular apertures (sroptapt.h:206, 384) on the
// Ex and Ez moments, with the rms sizes of srTMomentsPtrs::ComputeCentralMoments (srstraux.h:357)
static bool mom_outside(const double* mx, const double* mz, const MomOp& op)
{
    auto rms = [](const double* m, double& sx, double& sz) {
        double Mxx = m[5] - m[1] * m[1], Mzz = m[8] - m[3] * m[3];
        if (Mxx < 0.1 * m[5]) Mxx = 0.1 * m[5];
        if (Mzz < 0.1 * m[8]) Mzz = 0.1 * m[8];
        sx = ::sqrt(::fabs(Mxx)); sz = ::sqrt(::fabs(Mzz));
    };
    const double* ms[2] = {mx, mz};
    for (int c = 0; c < 2; c++) {
        const double* m = ms[c];
        double sx, sz;
        rms(m, sx, sz);
        sx *= 1.7; sz *= 1.7;
        if (((m[1] - sx) < (op.cx - op.hx)) || ((m[1] + sx) > (op.cx + op.hx)) || ((m[3] - sz) < (op.cz - op.hz)) ||
            ((m[3] + sz) > (op.cz + op.hz)))
            return true;
    }
    return false;
}

// the 22 sums of a MOM pass normalised into the 11 moments of Ex and of Ez, each rounded to FP32 as
// the reference stores them (sroptelm.cpp:1937-2080, coordinate representation)
void moments_from_sums(const double* S, const MomOp& op, double* mx, double* mz)
{
    const double FourPi = 3.141592653590 * 2. * 2.;
    const double lam_d_4pi = 1.239842E-06 / (FourPi * op.eStart);
    const double lam_d_2pi = 2. * lam_d_4pi, lam_d_2pi_e2 = lam_d_2pi * lam_d_2pi;
    const double isx = 1. / op.xStep, isz = 1. / op.zStep;
    const bool scx = op.nx > 1, scz = op.nz > 1;
    auto f32 = [](double v) { return (double)(float)v; };
    double* out[2] = {mx, mz};
    for (int c = 0; c < 2; c++) {
        const double* s = S + 11 * c;
        double* m = out[c];
        if (s[0] == 0.) { for (int i = 0; i < 11; i++) m[i] = 0.; continue; }
        const double inv_n = 1. / s[0];
        const double a = inv_n * lam_d_2pi, ax = a * isx, az = a * isz;
        const double a2 = inv_n * lam_d_2pi_e2, ax2 = a2 * (isx * isx), az2 = a2 * (isz * isz);
        m[0] = f32((scx && scz) ? s[0] * (op.xStep * op.zStep * 1.E+06) : 0.);
        m[1] = f32(scx ? s[1] * inv_n : op.xStart);
        m[2] = f32(scx ? s[2] * ax : 0.);
        m[3] = f32(scz ? s[3] * inv_n : op.zStart);
        m[4] = f32(scz ? s[4] * az : 0.);
        m[5] = f32(scx ? s[5] * inv_n : op.xStart * op.xStart);
        m[6] = f32(scx ? s[6] * ax : 0.);
        m[7] = f32(scx ? s[7] * ax2 : 0.);
        m[8] = f32(scz ? s[8] * inv_n : op.zStart * op.zStart);
        m[9] = f32(scz ? s[9] * az : 0.);
        m[10] = f32(scz ? s[10] * az2 : 0.);
    }
}

// central moments as srTMomentsPtrs caches them (srstraux.h:357): usable flag, rms divergences
struct CenMom { bool ok; double sxp, szp; };
static CenMom cen_mom(const double* m)
{
    double Mxx = m[5] - m[1] * m[1], Mxpxp = m[7] - m[2] * m[2];
    double Mzz = m[8] - m[3] * m[3], Mzpzp = m[10] - m[4] * m[4];
    CenMom c;
    c.ok = !((Mxx < 0) || (Mxpxp < 0) || (Mzz < 0) || (Mzpzp < 0));
    if (Mxpxp < 0.1 * m[7]) Mxpxp = 0.1 * m[7];
    if (Mzpzp < 0.1 * m[10]) Mzpzp = 0.1 * m[10];
    c.sxp = ::sqrt(::fabs(Mxpxp)); c.szp = ::sqrt(::fabs(Mzpzp));
    return c;
}

// the moment handling of EstimateWfrRadToSub_AnalytTreatQuadPhaseTerm (sroptdrf.cpp:1156-1213): the
// moments are recomputed from the field when both norms are zero, or when the central moments of
// the stronger component, as they were cached before any recomputation, are unusable; then the rms
// divergences of that component.  S: the sums of the field (nullptr: none measured).  Returns false
// when a recomputation is needed and S is nullptr.
static bool estimate_moments(const MomOp& op, const double* S, double* mx, double* mz, double& sxp, double& szp,
                             bool* recomputed = nullptr)
{
    const CenMom cX = cen_mom(mx), cZ = cen_mom(mz);
    bool rec = false;
    if (mx[0] == 0. && mz[0] == 0.) {
        if (S == nullptr) return false;
        moments_from_sums(S, op, mx, mz);
        rec = true;
    }
    const bool useX = mx[0] >= mz[0];
    CenMom c = useX ? cX : cZ;
    if (!c.ok || c.sxp == 0. || c.szp == 0.) {
        if (S == nullptr) return false;
        moments_from_sums(S, op, mx, mz);
        c = cen_mom(useX ? mx : mz);
        rec = true;
    }
    sxp = c.sxp; szp = c.szp;
    if (recomputed) *recomputed = rec;
    return true;
}

// a MOM pass on the current field (ComputeRadMoments, sroptelm.cpp:1608) with the result slot of op;
// certain: the recomputation is known to happen (its treatment flags stay behind, as the reference's)
void Planner::emit_moment_pass(MomOp& op, bool certain)
{
    op.slot = nMomSlots++;
    MomDesc& d = b->moments(w);
    fill_moment_desc(w, d, op);
    if (certain) { w.QuadX = op.qx; w.QuadZ = op.qz; }
    else quadFlagsUncertain_ = true;
    momProvisional = true;
}

// the MOM pass descriptor of a wavefront state (adds to the point-wise work already in d.pw) and the
// mesh / flags of its bookkeeping op; op.slot must be set
void fill_moment_desc(const WfrState& w, MomDesc& d, MomOp& op)
{
    op.nx = w.nx; op.nz = w.nz; op.eStart = w.eStart;
    op.xStart = w.xStart; op.xStep = w.xStep; op.zStart = w.zStart; op.zStep = w.zStep;
    d.nx = w.nx; d.nz = w.nz;
    d.xStart = w.xStart; d.xStep = w.xStep; d.zStart = w.zStart; d.zStep = w.zStep;
    d.slot = op.slot;
    // WaveFrontTermCanBeTreated (sroptelm.cpp:4692) and TreatStronglyOscillatingTerm 'r' (:4774): the
    // quadratic phase of the wavefront radius about (xc, zc) comes off before the sums (the reference
    // adds it back after, so the field itself is unchanged)
    const bool qx = ::fabs(w.RobsXAbsErr) < 0.4 * ::fabs(w.RobsX);
    const bool qz = ::fabs(w.RobsZAbsErr) < 0.4 * ::fabs(w.RobsZ);
    op.qx = qx; op.qz = qz;
    if (qx || qz) {
        const double Const = 3.14159265358979 * 1.E+06 / 1.23984186;
        const double cx = qx ? -Const / w.RobsX * w.eStart : 0., cz = qz ? -Const / w.RobsZ * w.eStart : 0.;
        Builder::add_quad(&d.pw, w.xStart, w.xStep, w.zStart, w.zStep, cx, -2. * cx * w.xc, cz, -2. * cz * w.zc,
                          cx * w.xc * w.xc + cz * w.zc * w.zc);
    }
    // 2 pi / (lambda R) * step with the reference's constants (R = 100 lambda when 0)
    const double FourPi = 3.141592653590 * 2. * 2.;
    const double lam_d_4pi = 1.239842E-06 / (FourPi * w.eStart), lam = lam_d_4pi * FourPi;
    const double Rx = (w.RobsX != 0.) ? w.RobsX : 100. * lam, Rz = (w.RobsZ != 0.) ? w.RobsZ : 100. * lam;
    d.ax = 0.5 * (w.xStep * ((1. / lam_d_4pi) / Rx));
    d.az = 0.5 * (w.zStep * ((1. / lam_d_4pi) / Rz));
}

void single_moment_pass(const WfrState& w, KernelDesc& k, MomOp& op, std::vector<float2>& tables)
{
    std::vector<KernelDesc> ks(1);
    memset(&ks[0], 0, sizeof(KernelDesc));
    ks[0].kind = K_MOM;
    op.slot = 0;
    fill_moment_desc(w, ks[0].mom, op);
    build_tables(ks, tables);
    k = ks[0];
}

// srTCompositeOptElem::ExtractPropagatedIntensity (sroptcnt.cpp:429-475) for the requests of element
// `elem`: a read-only pass on the field as the element leaves it (the operators still pending on it
// applied on the fly) writes the intensity component into the stage's extraction buffer; the mesh is
// the wavefront's (GetIntMesh, srradstr.cpp:4140).  Vs x and y (dep 3) in the coordinate
// representation, single-electron intensity / phase / Re E / Im E (SRWL numbering 0, 4, 5, 6)
void Planner::extract_after(int elem)
{
    for (const IntReq& q : intReqs) {
        if (q.elem != elem) continue;
        if (q.dep != 3 || q.pres != 0 || w.Pres != 0) {
            err = "intensity extraction during propagation vs x and y (dep 3) in the coordinate representation only";
            throw (int)SRWG_ERR_UNSUPPORTED;
        }
        int what;
        switch (q.type) {      // arIntTypeConv (sroptcnt.cpp:446): SRWL numbering -> internal
        case 0: what = 0; break;
        case 4: what = 2; break;
        case 5: what = 3; break;
        case 6: what = 6; break;
        default:
            err = "intensity type " + std::to_string(q.type) + " during propagation (0, 4, 5 and 6 are supported)";
            throw (int)SRWG_ERR_UNSUPPORTED;
        }
        if (q.pol < -4 || q.pol > 6) {
            err = "polarisation " + std::to_string(q.pol) + " for intensity extraction during propagation";
            throw (int)SRWG_ERR_UNSUPPORTED;
        }
        MomDesc& d = b->moments(w, K_INT);
        d.nx = w.nx; d.nz = w.nz;
        d.xStart = w.xStart; d.xStep = w.xStep; d.zStart = w.zStart; d.zStep = w.zStep;
        d.slot = -1;
        d.ipol = q.pol; d.iwhat = what;
        IntOut o;
        o.index = q.index; o.nx = w.nx; o.nz = w.nz;
        o.xStart = w.xStart; o.xStep = w.xStep; o.zStart = w.zStart; o.zStep = w.zStep;
        o.arType = what == 2 ? 'd' : 'f';
        o.bytes = (long long)w.nx * w.nz * (what == 2 ? 8 : 4);
        o.off = intBytes;
        d.ioff = o.off;
        intBytes += (o.bytes + 255) & ~255LL;
        intOuts.push_back(o);
    }
}

// EstimateWfrRadToSub_AnalytTreatQuadPhaseTerm (sroptdrf.cpp:1123-1365): the radius to subtract in
// the pp[3]=1 drift, from the rms divergence.  When the moments it needs come from the field, the
// field is measured here and the plan stops at a stage boundary; the element is planned again once
// the measurement is back.
void Planner::estimate_rad(double L, double& effRx, double& effRz)
{
    MomOp op;
    op.kind = MOP_ESTIMATE;
    const double* S = nullptr;
    if (pendingEstSlot_ >= 0) {
        op = pendingEstOp_;
        S = slotVals_.data() + (size_t)op.slot * SRWG_MOM_SLOT;
    } else {
        double mx[11], mz[11], a, c;
        memcpy(mx, w.momX, sizeof(mx));
        memcpy(mz, w.momZ, sizeof(mz));
        if (momProvisional || !estimate_moments(op, nullptr, mx, mz, a, c)) {
            if (!allowStages || !numMoments || w.Pres != 0) {
                err = "drift mode pp[3]=1 needs the moments of the field while planning: only "
                      "srwlPropagElecField plans in stages";
                throw (int)SRWG_ERR_UNSUPPORTED;
            }
            emit_moment_pass(op, false);
            pendingEstSlot_ = op.slot;
            pendingEstOp_ = op;
            throw (int)SRWG_NEED_STAGE;
        }
    }
    double SigXp = 0., SigZp = 0.;
    bool rec = false;
    estimate_moments(op, S, w.momX, w.momZ, SigXp, SigZp, &rec);
    if (rec) { w.QuadX = op.qx; w.QuadZ = op.qz; }
    momOps.push_back(op);
    pendingEstSlot_ = -1;
    const double infLarge = 1E+23;
    if ((SigXp == 0) || (SigZp == 0)) {
        effRx = (w.RobsX != 0) ? w.RobsX : infLarge;
        effRz = (w.RobsZ != 0) ? w.RobsZ : infLarge;
        return;
    }
    const double coefAngRange = 0.2, fourPi = 4. * 3.14159265359;
    const double lambM = 1.239842E-06 / w.eStart;
    auto one = [&](double s1, double sig) {
        const double s2 = s1 + L;
        const double ap = coefAngRange * sig;
        const double smin = lambM / (fourPi * ap * ap);
        double Rmin = 2 * smin;
        if (::fabs(s1) < smin) {
            if (::fabs(s2) < smin) {
                if (::fabs(s1) < ::fabs(s2)) return (L > 0) ? Rmin : -Rmin;
                return (L > 0) ? (-Rmin - L) : (Rmin - L);
            }
            return (L > 0) ? Rmin : -Rmin;
        }
        double eff = s1 + smin * smin / s1;
        const double eff_p_L = eff + L;
        const double minRmin = 0.007 * (::fabs(eff));
        if (Rmin < minRmin) Rmin = minRmin;
        if (::fabs(eff_p_L) < Rmin) eff = (eff_p_L < 0) ? (-Rmin - L) : (Rmin - L);
        return eff;
    };
    effRx = one(w.RobsX, SigXp);
    effRz = one(w.RobsZ, SigZp);
}

void Planner::replay_moments(const double* slots, double* mx, double* mz, bool* quadX, bool* quadZ) const
{
    for (int i = 0; i < 11; i++) { mx[i] = in.momX[i]; mz[i] = in.momZ[i]; }
    bool qx = in.QuadX, qz = in.QuadZ;     // treatment flags left by the last recomputation
    for (const MomOp& op : momOps) {
        if (op.kind == MOP_MATRIX) {
            apply_matrix_op(op, mx);
            apply_matrix_op(op, mz);
        } else if (op.kind == MOP_ESTIMATE) {
            double a, c;
            bool rec = false;
            if (op.slot >= 0 && slots != nullptr)
                estimate_moments(op, slots + (size_t)op.slot * SRWG_MOM_SLOT, mx, mz, a, c, &rec);
            if (rec) { qx = op.qx; qz = op.qz; }
        } else if (op.slot >= 0 && slots != nullptr && (op.obstacle || mom_outside(mx, mz, op))) {
            moments_from_sums(slots + (size_t)op.slot * SRWG_MOM_SLOT, op, mx, mz);
            qx = op.qx; qz = op.qz;
        }
    }
    if (quadX) *quadX = qx;
    if (quadZ) *quadZ = qz;
}

void Planner::drift_ang(const ElemDesc& e)
{   // PropagateRadiationSimple_AngRepres (sroptdrf.h:348-411), RadPointModifier_AngRepres (:615)
    double xStartOld = w.xStart, zStartOld = w.zStart;
    w.xStart = -(w.nx >> 1) * w.xStep;
    w.zStart = -(w.nz >> 1) * w.zStep;
    double xShift = w.xStart - xStartOld, zShift = w.zStart - zStartOld;
    w.xWfrMin += xShift; w.xWfrMax += xShift;
    w.zWfrMin += zShift; w.zWfrMax += zShift;
    if (w.Pres != 1) set_rad_repres(1);
    double lam = LAMBDA_EV_M / w.eStart;
    double c0 = -3.1415926536 * e.L * lam, c1 = 0.25 * lam * lam;
    double cc = (e.treat == 1) ? (5.067730652e+06) * e.L * w.eStart : 0.;
    b->ang(w, c0, c1, cc);
    if (w.UseStartTrToShiftAtChangingRepresToCoord) { w.xStartTr += xShift; w.zStartTr += zShift; }
    set_rad_repres(0);
    w.xStart = xStartOld; w.zStart = zStartOld;
    if (w.UseStartTrToShiftAtChangingRepresToCoord) {
        w.xStart = w.xStartTr - xShift;
        w.zStart = w.zStartTr - zShift;
    }
    set_full_range();
}

void Planner::drift_to_waist(const ElemDesc& e)
{   // PropagateRadiationSimple_PropToWaist (sroptdrf.cpp:356-489), SetupPropBufVars_PropToWaist
    // (sroptdrf.h:476), RadPointModifier_PropToWaist (sroptdrf.h:649-710)
    const double L = e.L;
    set_full_range();
    double InvLength = 1. / L;
    double Pi_d_LambdaM = w.eStart * PI_D_LAMBDA_PER_EV;
    double Pi_d_LambdaM_d_Length = Pi_d_LambdaM * InvLength;
    double InvLength_d_Lambda = InvLength * w.eStart * INV_LAMBDA_PER_EV;
    double TwoPi_d_LambdaM = 2. * Pi_d_LambdaM;
    double TwoPiXc = TwoPi_d_LambdaM * w.xc / w.RobsX;
    double TwoPiZc = TwoPi_d_LambdaM * w.zc / w.RobsZ;
    if (w.Pres != 0) set_rad_repres(0);
    double cc = (e.treat == 1) ? (5.067730652e+06) * L * w.eStart : 0.;
    b->quad(w, Pi_d_LambdaM_d_Length, TwoPiXc, Pi_d_LambdaM_d_Length, TwoPiZc, cc);
    double InvLambda_m = w.eStart * INV_LAMBDA_PER_EV;
    double InvLambda_m_d_Length = InvLambda_m / L;
    double LambdaM_Length = 1. / InvLambda_m_d_Length;
    double xs, zs, x0, z0;
    fft2_emit(1, false, xs, zs, x0, z0);     // Make2DFFT forward, representation flag unchanged
    double qxCen = -w.xc * InvLambda_m / w.RobsX;
    double qzCen = -w.zc * InvLambda_m / w.RobsZ;
    w.xStart = (x0 + qxCen) * LambdaM_Length;
    w.zStart = (z0 + qzCen) * LambdaM_Length;
    w.xStep = xs * LambdaM_Length;
    w.zStep = zs * LambdaM_Length;
    b->quad(w, Pi_d_LambdaM_d_Length, 0., Pi_d_LambdaM_d_Length, 0., 0.);
    b->scale(w, 0.f, (float)(-InvLength_d_Lambda));     // x InvLength_d_Lambda, then (re,im) <- (im,-re)
    if (LambdaM_Length < 0) {
        mirror(-1, -1);
        double xEnd = w.xStart + (w.xStep) * (w.nx - 1);
        w.xStart = xEnd;
        w.xStep *= -1.;
        double zEnd = w.zStart + (w.zStep) * (w.nz - 1);
        w.zStart = zEnd;
        w.zStep *= -1.;
    }
}

void Planner::drift_from_waist(const ElemDesc& e)
{   // PropagateRadiationSimple_PropFromWaist (sroptdrf.cpp:614-724), SetupPropBufVars_PropFromWaist
    // (sroptdrf.h:522), RadPointModifier_PropFromWaist (sroptdrf.h:756-804): as to the waist without
    // the centre terms and the mirror, the path-length phase in the second pass
    const double L = e.L;
    double InvLength = 1. / L;
    double Pi_d_LambdaM = w.eStart * PI_D_LAMBDA_PER_EV;
    double Pi_d_LambdaM_d_Length = Pi_d_LambdaM * InvLength;
    double InvLength_d_Lambda = InvLength * w.eStart * INV_LAMBDA_PER_EV;
    if (w.Pres != 0) set_rad_repres(0);
    b->quad(w, Pi_d_LambdaM_d_Length, 0., Pi_d_LambdaM_d_Length, 0., 0.);
    double InvLambda_m = w.eStart * INV_LAMBDA_PER_EV;
    double InvLambda_m_d_Length = InvLambda_m / L;
    double LambdaM_Length = 1. / InvLambda_m_d_Length;
    double xs, zs, x0, z0;
    fft2_emit(1, false, xs, zs, x0, z0);     // Make2DFFT forward, representation flag unchanged
    w.xStart = x0 * LambdaM_Length;
    w.zStart = z0 * LambdaM_Length;
    w.xStep = xs * LambdaM_Length;
    w.zStep = zs * LambdaM_Length;
    double cc = (e.treat == 1) ? (5.067730652e+06) * L * w.eStart : 0.;
    b->quad(w, Pi_d_LambdaM_d_Length, 0., Pi_d_LambdaM_d_Length, 0., cc);
    b->scale(w, 0.f, (float)(-InvLength_d_Lambda));     // x InvLength_d_Lambda, then (re,im) <- (im,-re)
}

void Planner::drift_beyond_parax(const ElemDesc& e)
{   // PropagateRadiationSimple_PropToWaistBeyondParax (sroptdrf.cpp:491-612), its buffer set-up
    // (sroptdrf.h:492) and RadPointModifier_PropToWaistBeyondParax (sroptdrf.h:712-754)
    if (quadFlagsUncertain_) {
        // TreatQuadPhaseTerm below uses the treatment flags that the last moment recomputation left;
        // whether an aperture recomputed is only known once its passes ran
        if (!allowStages) {
            err = "drift mode pp[3]=5 after an aperture whose moment recomputation is decided on the "
                  "device: only srwlPropagElecField plans in stages";
            throw (int)SRWG_ERR_UNSUPPORTED;
        }
        throw (int)SRWG_NEED_STAGE;
    }
    const double L = e.L;
    set_full_range();
    const double sqrtAbsRxRz = ::sqrt(::fabs(w.RobsX * w.RobsZ));
    const int sgnRx = (w.RobsX >= 0) ? 1 : -1, sgnRz = (w.RobsZ >= 0) ? 1 : -1;
    const double dPhaseSignR = 0.7853981633974483 * (sgnRx + sgnRz);
    const double Pi_MultLambdaM = 3.141592653589793 * 1.239842e-06;
    const double Pi_MultLambdaM_Rx = Pi_MultLambdaM * w.RobsX, Pi_MultLambdaM_Rz = Pi_MultLambdaM * w.RobsZ;
    const double MultEn_TwoPi_L_d_LambdaM = 2. * 2.53384080189E+06 * L;
    if (w.Pres != 0) set_rad_repres(0);
    treat_quad('r');                     // TreatQuadPhaseTerm (srradstr.h:841), flags as they stand
    const double xcOrig = w.xc, zcOrig = w.zc;
    const double InvLambdaM = w.eStart * 806546.577258;
    const double InvLambdaM_d_Rx = InvLambdaM / w.RobsX, InvLambdaM_d_Rz = InvLambdaM / w.RobsZ;
    w.xStep *= InvLambdaM_d_Rx;
    w.zStep *= InvLambdaM_d_Rz;
    w.xStart = (w.xStart - xcOrig) * InvLambdaM_d_Rx;
    w.zStart = (w.zStart - zcOrig) * InvLambdaM_d_Rz;
    const double en = w.eStart, LambdaM = 1.239842e-06 / en;
    b->quad(w, -Pi_MultLambdaM_Rx / en, 0., -Pi_MultLambdaM_Rz / en, 0., dPhaseSignR);
    b->bpx(w, LambdaM, MultEn_TwoPi_L_d_LambdaM * en, e.treat == 1 ? 1 : 0);
    b->scale(w, (float)(LambdaM * sqrtAbsRxRz), 0.f);
    double xs, zs, x0, z0;
    fft2_emit(-1, false, xs, zs, x0, z0);
    int sx = 1, sz = 1;
    double xStartNew = x0 + xcOrig, xStepNew = xs, zStartNew = z0 + zcOrig, zStepNew = zs;
    if (xs < 0) { sx = -1; xStartNew = -x0 + xcOrig; xStepNew = -xs; }
    if (zs < 0) { sz = -1; zStartNew = -z0 + zcOrig; zStepNew = -zs; }
    if ((sx < 0) || (sz < 0)) mirror(sx, sz);
    w.xStart = xStartNew; w.zStart = zStartNew;
    w.xStep = xStepNew; w.zStep = zStepNew;
}

static double sgn(double v) { return v > 0 ? 1. : (v < 0 ? -1. : 0.); }

int Planner::drift_quad(const ElemDesc& e, int subtype)
{   // PropagateRadiationSimple_AnalytTreatQuadPhaseTerm (sroptdrf.cpp:726-887),
    // SetupPropBufVars_AnalytTreatQuadPhaseTerm (:889), EstimateWfrRadToSub2 (:1085),
    // RadPointModifier_AnalytTreatQuadPhaseTerm (sroptdrf.h:806-880)
    const double L = e.L;
    const double infLarge = 1E+23;
    double xc = w.xc, zc = w.zc;
    double invRx = 0, invRz = 0, Lx = 0, Lz = 0, invRxL = 1. / L, invRzL = 1. / L;
    double kx = infLarge, kxc = infLarge, kz = infLarge, kzc = infLarge;
    double trueRx = w.RobsX, trueRz = w.RobsZ;
    if (subtype == 2) {
        const double factRadEr = 3.;
        double minAbsEffRx = factRadEr * w.RobsXAbsErr, minAbsEffRz = factRadEr * w.RobsZAbsErr;
        double effRx_p_L = trueRx + L;
        if (::fabs(trueRx) < minAbsEffRx) trueRx = minAbsEffRx * ((trueRx >= 0) ? 1. : -1.);
        else if (::fabs(effRx_p_L) < minAbsEffRx) trueRx = minAbsEffRx * ((effRx_p_L >= 0) ? 1. : -1.) - L;
        double effRz_p_L = trueRz + L;
        if (::fabs(trueRz) < minAbsEffRz) trueRz = minAbsEffRz * ((trueRz >= 0) ? 1. : -1.);
        else if (::fabs(effRz_p_L) < minAbsEffRz) trueRz = minAbsEffRz * ((effRz_p_L >= 0) ? 1. : -1.) - L;
    } else if (subtype == 1) {
        estimate_rad(L, trueRx, trueRz);
    }
    if (trueRx != 0) {
        invRx = 1. / trueRx;
        kx = (trueRx + L) * invRx;
        kxc = L / trueRx;
        if (-L != trueRx) { Lx = L / (1. + L * invRx); invRxL = 1. / (L + trueRx); }
        else { Lx = infLarge; invRxL = infLarge; }
    }
    if (trueRz != 0) {
        invRz = 1. / trueRz;
        kz = (trueRz + L) * invRz;
        kzc = L / trueRz;
        if (-L != trueRz) { Lz = L / (1. + L * invRz); invRzL = 1. / (L + trueRz); }
        else { Lz = infLarge; invRzL = infLarge; }
    }
    double sqrt_LxLz_d_L = ::sqrt(::fabs(Lx * Lz)) / L;
    double phase_term = 0.25 * 3.141592653589793 * (2. - sgn(Lx) - sgn(Lz));

    if (w.Pres != 0) set_rad_repres(0);
    double lam = LAMBDA_EV_M / w.eStart;
    double Pi_d_Lambda_m = 3.1415926536 / lam;
    // pass 1: -pi/lambda ((x-xc)^2/Rx + (z-zc)^2/Rz)
    {
        double ax = -Pi_d_Lambda_m * invRx, az = -Pi_d_Lambda_m * invRz;
        b->quad(w, ax, -2. * ax * xc, az, -2. * az * zc, ax * xc * xc + az * zc * zc);
    }
    double xStartOld = w.xStart, zStartOld = w.zStart;
    w.xStart = -(w.nx >> 1) * w.xStep;
    w.zStart = -(w.nz >> 1) * w.zStep;
    double xShift = w.xStart - xStartOld, zShift = w.zStart - zStartOld;
    w.xWfrMin += xShift; w.xWfrMax += xShift;
    w.zWfrMin += zShift; w.zWfrMax += zShift;
    set_rad_repres(1);
    // pass 2 (angular side): -pi lambda (Lx qx^2 + Lz qz^2) + sign term, x sqrt(|Lx Lz|)/L
    {
        double Pi_Lambda_m = 3.1415926536 * lam;
        b->quad(w, -Pi_Lambda_m * Lx, 0., -Pi_Lambda_m * Lz, 0., phase_term);
        b->scale(w, (float)sqrt_LxLz_d_L, 0.f);
    }
    if (w.UseStartTrToShiftAtChangingRepresToCoord) { w.xStartTr += xShift; w.zStartTr += zShift; }
    set_rad_repres(0);
    w.xStart = xStartOld; w.zStart = zStartOld;
    if (w.UseStartTrToShiftAtChangingRepresToCoord) { w.xStart = w.xStartTr - xShift; w.zStart = w.zStartTr - zShift; }
    w.xStart = kx * (w.xStart) - kxc * (w.xc);
    w.xStep *= kx;
    w.zStart = kz * (w.zStart) - kzc * (w.zc);
    w.zStep *= kz;
    // pass 3: +pi/lambda ((x-xc)^2/(R+L) ...)
    {
        double ax = Pi_d_Lambda_m * invRxL, az = Pi_d_Lambda_m * invRzL;
        double cc = ax * xc * xc + az * zc * zc;
        if (e.treat == 1) cc += 2 * Pi_d_Lambda_m * L;
        b->quad(w, ax, -2. * ax * xc, az, -2. * az * zc, cc);
    }
    mirror((int)sgn(kx), (int)sgn(kz));
    if (kx < 0) {
        double xEnd = w.xStart + (w.nx - 1) * w.xStep;
        w.xStart = xEnd;
        w.xStep *= -1;
    }
    if (kz < 0) {
        double zEnd = w.zStart + (w.nz - 1) * w.zStep;
        w.zStart = zEnd;
        w.zStep *= -1;
    }
    set_full_range();
    return 0;
}

void Planner::drift(const ElemDesc& e, int anal)
{   // srTDriftSpace::PropagateRadiation (sroptdrf.h:116) -> PropagateRadiationSingleE_Meth_0 (:158)
    if (anal == 1 || anal == 2) {
        int r = drift_quad(e, anal);
        if (r) throw r;
    } else if (anal == 4) drift_to_waist(e);
    else if (anal == 3) drift_from_waist(e);
    else if (anal == 5) drift_beyond_parax(e);
    else if (anal == 0) drift_ang(e);
    else {
        err = "drift mode pp[3]=" + std::to_string(anal) + " is not supported on the GPU path";
        throw (int)SRWG_ERR_UNSUPPORTED;
    }
    drift_moments(e.L);
    w.RobsX += e.L;                       // PropagateWaveFrontRadius (sroptdrf.h:981)
    w.RobsZ += e.L;
    set_full_range();
    // Propagate4x4PropMatr of the drift (sroptdrf.h:1002): no vector
    const double D[16] = {1., e.L, 0., 0., 0., 1., 0., 0., 0., 0., 1., e.L, 0., 0., 0., 1.};
    const double v0[4] = {0., 0., 0., 0.};
    prop_4x4(D, v0);
}

// GenAuxPropagate4x4PropMatr (sroptelm.cpp:5594): M <- E M, V <- E V + e for the element's 4x4 matrix
// E and vector e (the wavefront's arElecPropMatr: 16 matrix entries, then the vector)
void Planner::prop_4x4(const double E[16], const double e[4])
{
    double R[16], V[4];
    for (int i = 0; i < 4; i++) {
        V[i] = 0.;
        for (int j = 0; j < 4; j++) {
            double r = 0.;
            for (int k = 0; k < 4; k++) r += E[4 * i + k] * w.propM[4 * k + j];
            R[4 * i + j] = r;
            V[i] += E[4 * i + j] * w.propM[16 + j];
        }
    }
    for (int i = 0; i < 16; i++) w.propM[i] = R[i];
    for (int i = 0; i < 4; i++) w.propM[16 + i] = V[i] + e[i];
}

// ================================================================================================
// Linear phase terms (CheckAndSubtract/ResetPhaseTermsLin, srradstr.cpp:2610-2705)
// ================================================================================================
void Planner::phase_lin_subtract(double newXc, double newZc)
{
    const double ratAllowSubtract = 0.2, minNumOptCycles = 10;
    double lambda_m = 3.1415926535898 / (w.eStart * 2.53384080189E+06);
    const double twoPi = 2. * 3.1415926535898;
    bool xOK = false;
    double dxcSubNew = newXc - w.xc;
    if (w.RobsX != 0) {
        double r = w.xStep * (w.nx - 1);
        double nc = 0.25 * r * r / (lambda_m * w.RobsX);
        xOK = (::fabs(w.RobsX) > ::fabs(w.RobsXAbsErr)) && (nc > minNumOptCycles) && (::fabs(dxcSubNew) / r > ratAllowSubtract);
    }
    if (!xOK) dxcSubNew = 0;
    bool zOK = false;
    double dzcSubNew = newZc - w.zc;
    if (w.RobsZ != 0) {
        double r = w.zStep * (w.nz - 1);
        double nc = 0.25 * r * r / (lambda_m * w.RobsZ);
        zOK = (::fabs(w.RobsZ) > ::fabs(w.RobsZAbsErr)) && (nc > minNumOptCycles) && (::fabs(dzcSubNew) / r > ratAllowSubtract);
    }
    if (!zOK) dzcSubNew = 0;
    if (!xOK && !zOK) return;
    double dxc = dxcSubNew;
    if (w.xLinOnly) {
        dxc -= w.dxcSub;
        if (::fabs(dxc) / ::fabs(w.dxcSub) < ratAllowSubtract) { dxc = 0; dxcSubNew = w.dxcSub; }
    }
    w.dxcSub = dxcSubNew;
    w.xLinOnly = (dxcSubNew != 0);
    double xMult = -twoPi * dxc / (lambda_m * w.RobsX);
    double dzc = dzcSubNew;
    if (zOK && w.zLinOnly) {
        dzc -= w.dzcSub;
        if (::fabs(dzc) / ::fabs(w.dzcSub) < ratAllowSubtract) { dzc = 0; dzcSubNew = w.dzcSub; }
    }
    w.dzcSub = dzcSubNew;
    w.zLinOnly = (dzcSubNew != 0);
    double zMult = -twoPi * dzc / (lambda_m * w.RobsZ);
    if (xMult == 0 && zMult == 0) return;
    b->quad(w, 0., xMult, 0., zMult, 0.);       // MultiplyElFieldByPhaseLin
}

void Planner::phase_lin_reset()
{
    if (!w.xLinOnly && !w.zLinOnly) return;
    double lambda_m = 3.1415926535898 / (w.eStart * 2.53384080189E+06);
    const double twoPi = 2. * 3.1415926535898;
    double xMult = 0, zMult = 0;
    if (w.xLinOnly && w.dxcSub != 0 && w.RobsX != 0) xMult = twoPi * w.dxcSub / (lambda_m * w.RobsX);
    if (w.zLinOnly && w.dzcSub != 0 && w.RobsZ != 0) zMult = twoPi * w.dzcSub / (lambda_m * w.RobsZ);
    w.xLinOnly = w.zLinOnly = false;
    w.dxcSub = w.dzcSub = 0;
    if (xMult == 0 && zMult == 0) return;
    b->quad(w, 0., xMult, 0., zMult, 0.);
}

void Planner::fix_abs_err()
{   // tail of srTGenOptElem::PropagateRadiationMeth_0 (sroptel2.cpp:151)
    if ((w.RobsX != 0) && (w.RobsXAbsErr == 0)) w.RobsXAbsErr = ::fabs(0.1 * w.RobsX);
    if ((w.RobsZ != 0) && (w.RobsZAbsErr == 0)) w.RobsZAbsErr = ::fabs(0.1 * w.RobsZ);
}

// ================================================================================================
// Thin lens (cpp/src/core/sroptfoc.h:18-276)
// ================================================================================================
void Planner::lens(const ElemDesc& e)
{
    phase_lin_subtract(e.x, e.y);
    if (w.Pres != 0) set_rad_repres(0);
    double Pi_d_Lambda_m = w.eStart * 2.533865612E+06;
    {   // -pi/lambda ((x-cx)^2/Fx + (z-cz)^2/Fz)
        double ax = -Pi_d_Lambda_m / e.Fx, az = -Pi_d_Lambda_m / e.Fy;
        b->quad(w, ax, -2. * ax * e.x, az, -2. * az * e.y, ax * e.x * e.x + az * e.y * e.y);
    }
    const double ax[2][2] = {{1., 0.}, {-1. / e.Fx, 1.}};
    const double az[2][2] = {{1., 0.}, {-1. / e.Fy, 1.}};
    record_matrix(ax, az, 0, 0., 0.);
    const double dSmall = 1E-23;
    double difX = (e.Fx == w.RobsX) ? dSmall : e.Fx - w.RobsX;
    double difZ = (e.Fy == w.RobsZ) ? dSmall : e.Fy - w.RobsZ;
    double MagnX = e.Fx / difX, MagnZ = e.Fy / difZ;
    w.RobsX *= MagnX;
    w.RobsZ *= MagnZ;
    w.RobsXAbsErr *= (MagnX * MagnX);
    w.RobsZAbsErr *= (MagnZ * MagnZ);
    w.xc = e.x - (e.x - w.xc) * MagnX;
    w.zc = e.y - (e.y - w.zc) * MagnZ;
    // Propagate4x4PropMatr of the focusing element (sroptfoc.h:101)
    const double Foc[16] = {1., 0., 0., 0., -1. / e.Fx, 1., 0., 0., 0., 0., 1., 0., 0., 0., -1. / e.Fy, 1.};
    const double fv[4] = {0., e.x / e.Fx, 0., e.y / e.Fy};
    prop_4x4(Foc, fv);
    fix_abs_err();
    phase_lin_reset();
}

// ================================================================================================
// Generic transmission (cpp/src/core/sroptgtr.h:86-140): a focusing element in the bookkeeping
// (srTFocusingElem radius / moments / 4x4 with the estimated focal lengths), the table as the
// point-wise work, linear phase terms about the table's centre subtracted before and reset after
// ================================================================================================
void Planner::transmission(const ElemDesc& e)
{
    phase_lin_subtract(e.x, e.y);
    if (w.Pres != 0) set_rad_repres(0);
    b->transm(w, e);
    const double ax[2][2] = {{1., 0.}, {-1. / e.Fx, 1.}};
    const double az[2][2] = {{1., 0.}, {-1. / e.Fy, 1.}};
    record_matrix(ax, az, 0, 0., 0.);
    const double dSmall = 1E-23;
    double difX = (e.Fx == w.RobsX) ? dSmall : e.Fx - w.RobsX;
    double difZ = (e.Fy == w.RobsZ) ? dSmall : e.Fy - w.RobsZ;
    double MagnX = e.Fx / difX, MagnZ = e.Fy / difZ;
    w.RobsX *= MagnX;
    w.RobsZ *= MagnZ;
    w.RobsXAbsErr *= (MagnX * MagnX);
    w.RobsZAbsErr *= (MagnZ * MagnZ);
    w.xc = e.x - (e.x - w.xc) * MagnX;
    w.zc = e.y - (e.y - w.zc) * MagnZ;
    const double Foc[16] = {1., 0., 0., 0., -1. / e.Fx, 1., 0., 0., 0., 0., 1., 0., 0., 0., -1. / e.Fy, 1.};
    const double fv[4] = {0., e.x / e.Fx, 0., e.y / e.Fy};
    prop_4x4(Foc, fv);
    fix_abs_err();
    phase_lin_reset();
}

// ================================================================================================
// Apertures / obstacles (cpp/src/core/sroptapt.h, sroptapt.cpp:248-350)
// ================================================================================================
void Planner::aperture(const ElemDesc& e)
{
    if (w.Pres != 0) set_rad_repres(0);
    int obstacle = (e.apob == 'o');
    if (e.shape == 'r') {
        const double SmallOffset = 1.E-10;
        b->mask(w, 1, obstacle, e.x, e.y, 0.5 * e.Dx + SmallOffset, 0.5 * e.Dy + SmallOffset, 0.);
    } else {
        double R = 0.5 * e.Dx;
        b->mask(w, 2, obstacle, e.x, e.y, 0., 0., R * R);
    }
    // srTAperture::PropagateRadMoments (sroptapt.cpp:248-350): the moments are recomputed from the
    // masked field (ComputeRadMoments) when 1.7 sigma of the beam is not inside the opening, always
    // for obstacles.  A MOM pass measures the field whenever the answer may be yes: the check itself
    // is replayed on the host after the run (earlier recomputations make plan-time moments provisional).
    {
        MomOp op;
        op.kind = MOP_APERTURE;
        op.obstacle = obstacle;
        op.cx = e.x; op.cz = e.y;
        op.hx = 0.5 * e.Dx;
        op.hz = (e.shape == 'r') ? 0.5 * e.Dy : 0.5 * e.Dx;
        const bool recompute = obstacle || mom_outside(w.momX, w.momZ, op);
        if ((recompute || momProvisional) && numMoments) emit_moment_pass(op, !momProvisional);
        momOps.push_back(op);
    }
    if (e.apob == 'a') {     // SetNewNonZeroWfrLimits of the apertures
        double hx = (e.shape == 'r') ? 0.5 * e.Dx : 0.5 * e.Dx;
        double hz = (e.shape == 'r') ? 0.5 * e.Dy : 0.5 * e.Dx;
        if (w.xWfrMin < e.x - hx) w.xWfrMin = e.x - hx;
        if (w.xWfrMax > e.x + hx) w.xWfrMax = e.x + hx;
        if (w.zWfrMin < e.y - hz) w.zWfrMin = e.y - hz;
        if (w.zWfrMax > e.y + hz) w.zWfrMax = e.y + hz;
    }
    fix_abs_err();
}

// ================================================================================================
// Resizing (RadResizeGen, sroptelm.cpp:2242-3036; RadResizeCore :3038-3337)
// ================================================================================================
void Planner::treat_quad(char add_or_rem)
{   // TreatStronglyOscillatingTerm (sroptelm.cpp:4774-5014) as a point-wise phase
    const double Const = 3.14159265358979 * 1.E+06 / 1.23984186;
    double cRx, cRz;
    if (w.Pres == 0) { cRx = w.QuadX ? Const / w.RobsX : 0.; cRz = w.QuadZ ? Const / w.RobsZ : 0.; }
    else {
        double lam = LAMBDA_EV_M / w.eStart;
        cRx = w.QuadX ? -Const * w.RobsX * lam * lam : 0.;
        cRz = w.QuadZ ? -Const * w.RobsZ * lam * lam : 0.;
    }
    if (add_or_rem == 'r') { cRx = -cRx; cRz = -cRz; }
    double ax = cRx * w.eStart, az = cRz * w.eStart;
    b->quad(w, ax, -2. * ax * w.xc, az, -2. * az * w.zc, ax * w.xc * w.xc + az * w.zc * w.zc);
}

// TuneStepToKeepInterpLimitsTheSameAtResize (cpp/src/core/sroptel3.cpp:537-623): where the new mesh
// reaches past the old one's first / last node, its step and start are tuned so that new nodes land
// on the old mesh's limits, node ic of the old mesh staying at the new centre
static void tune_step_keep_interp_limits(const WfrState& o, WfrState& n, double pm, char axis, long ic)
{
    double& nStart = axis == 'x' ? n.xStart : n.zStart;
    double& nStep = axis == 'x' ? n.xStep : n.zStep;
    const double oStart = axis == 'x' ? o.xStart : o.zStart, oStep = axis == 'x' ? o.xStep : o.zStep;
    const long nNp = axis == 'x' ? n.nx : n.nz, oNp = axis == 'x' ? o.nx : o.nz;
    const double NewEndInterp = nStart + (nNp - 1) * nStep;
    const double OldEndInterp = oStart + (oNp - 1) * oStep;
    const bool left = nStart <= oStart, right = NewEndInterp >= OldEndInterp;
    if (!(left || right)) return;
    const double cArg = oStart + ic * oStep;
    const long half = nNp >> 1;
    if (left && !right) {
        const double dist = cArg - nStart;
        const long steps = (long)(dist / nStep + 1.E-10);
        nStep = dist / double(steps);
        nStart = cArg - half * nStep;
    } else if (!left && right) {
        const double dist = OldEndInterp - cArg;
        const long steps = (long)(dist / nStep + 1.E-10);
        nStep = dist / double(steps);
        nStart = cArg - half * nStep;
    } else {
        const double OldRange = OldEndInterp - oStart;
        if (pm != 1.) {
            const long nIn = (long)(OldRange / nStep + 1.E-10);
            const long nLeft = (long)((oStart - nStart) / nStep + 1.E-10);
            nStep = OldRange / double(nIn);
            nStart = oStart - nLeft * nStep;
        } else {
            nStep = OldRange / double(nNp - 1);
            nStart = oStart;
        }
    }
}

int Planner::resize(double pxm, double pxd, double pzm, double pzd, int shift, double xcs, double zcs, bool other_side)
{
    if ((pxm == 1.) && (pxd == 1.) && (pzm == 1.) && (pzd == 1.) && (shift <= 0)) return 0;
    double RelCenPosX = 0.5, RelCenPosZ = 0.5;
    const double RelCenPosTol = 1.e-06;
    if (shift & 1) {
        double rxTot = w.xStep * (w.nx - 1), rxLeft = xcs - w.xStart;
        if ((rxLeft > 0.) && (xcs < (w.xStart + rxTot))) RelCenPosX = rxLeft / rxTot;
    }
    if (shift & 2) {
        double rzTot = w.zStep * (w.nz - 1), rzLeft = zcs - w.zStart;
        if ((rzLeft > 0.) && (zcs < (w.zStart + rzTot))) RelCenPosZ = rzLeft / rzTot;
    }
    int nxOld = w.nx, nzOld = w.nz;
    double xStartOld = w.xStart, zStartOld = w.zStart, xStepOld = w.xStep, zStepOld = w.zStep;
    double xRangeOld = xStepOld * nxOld, zRangeOld = zStepOld * nzOld;
    bool useStartTrOther = (::fabs(xStartOld + 0.5 * xRangeOld) > 0.5 * w.xStep) ||
                           (::fabs(zStartOld + 0.5 * zRangeOld) > 0.5 * w.zStep);
    double pxmIn = pxm, pxdIn = pxd, pzmIn = pzm, pzdIn = pzd;
    if (other_side) {
        int to = (w.Pres == 0) ? 1 : 0;
        if (useStartTrOther) {
            w.xStart = -(w.nx >> 1) * w.xStep;
            w.zStart = -(w.nz >> 1) * w.zStep;
            double xs = w.xStart - xStartOld, zs = w.zStart - zStartOld;
            w.xWfrMin += xs; w.xWfrMax += xs;
            w.zWfrMin += zs; w.zWfrMax += zs;
        }
        set_rad_repres(to);
        double t;
        t = pxm; pxm = pxd; pxd = t;
        t = pzm; pzm = pzd; pzd = t;
    }
    WfrState old = w;
    WfrState nw = w;
    double pxTot = pxm * pxd, pzTot = pzm * pzd;
    long NewNx = w.nx, NewNz = w.nz;
    bool changed = (pxTot != 1.) || (pzTot != 1.);
    if (changed) {
        double v = pxTot * NewNx;
        long iv = (long)v;
        NewNx = ((v - iv) >= 0.5) ? iv + 1 : iv;
        v = pzTot * NewNz;
        iv = (long)v;
        NewNz = ((v - iv) >= 0.5) ? iv + 1 : iv;
        NewNx = next_correct_number_for_fft(NewNx);
        NewNz = next_correct_number_for_fft(NewNz);
        nw.nx = (int)NewNx;
        nw.nz = (int)NewNz;
    }
    // centre of the new mesh: the old mesh's middle node, or the node nearest the requested centre
    // (IntegerOffsetCoord, sroptelm.h:995)
    auto ioc = [](double start, double step, double val) {
        long i = (long)((val - start) / step);
        if (::fabs(val - ((i + 1) * step + start)) < 1.E-05 * step) i++;
        return i;
    };
    bool centerOffset = false;
    long iXc = w.nx >> 1, iZc = w.nz >> 1;
    if (::fabs(RelCenPosX - 0.5) > RelCenPosTol) {
        iXc = ioc(w.xStart, w.xStep, w.xStart + w.nx * w.xStep * RelCenPosX);
        centerOffset = true;
    }
    if (::fabs(RelCenPosZ - 0.5) > RelCenPosTol) {
        iZc = ioc(w.zStart, w.zStep, w.zStart + w.nz * w.zStep * RelCenPosZ);
        centerOffset = true;
    }
    const double Xc = w.xStart + w.xStep * iXc, Zc = w.zStart + w.zStep * iZc;
    auto preserve = [&](char ax) {   // PreserveLogicsOfWfrLimitsAtRangeResizing (srradstr.cpp:1598)
        if (ax == 'x') {
            double tol = 0.01 * nw.xStep;
            if ((::fabs(old.xWfrMin - old.xStart) < tol) && (::fabs(old.xStart + old.nx * old.xStep - old.xWfrMax) < tol)) {
                nw.xWfrMin = nw.xStart; nw.xWfrMax = nw.xStart + nw.nx * nw.xStep;
            } else { nw.xWfrMin = old.xWfrMin; nw.xWfrMax = old.xWfrMax; }
        } else {
            double tol = 0.01 * nw.zStep;
            if ((::fabs(old.zWfrMin - old.zStart) < tol) && (::fabs(old.zStart + old.nz * old.zStep - old.zWfrMax) < tol)) {
                nw.zWfrMin = nw.zStart; nw.zWfrMax = nw.zStart + nw.nz * nw.zStep;
            } else { nw.zWfrMin = old.zWfrMin; nw.zWfrMax = old.zWfrMax; }
        }
    };
    if (centerOffset) {
        // new mesh centred on node iXc / iZc of the old one (sroptelm.cpp:2383-2433), its step tuned
        // so that the interpolation limits stay those of the old mesh
        const long NewNxLeftHalf = NewNx >> 1;
        nw.xStep = w.xStep / pxd;
        nw.xStart = Xc - NewNxLeftHalf * nw.xStep;
        const double NewNxEndInterp = nw.xStart + (NewNx - 1) * nw.xStep;
        const double OldNxEndInterp = w.xStart + (w.nx - 1) * w.xStep;
        tune_step_keep_interp_limits(w, nw, pxm, 'x', iXc);
        nw.AuxLong1 = (nw.xStart < w.xStart) ? ioc(nw.xStart, nw.xStep, w.xStart) : 0;
        nw.AuxLong2 = (NewNxEndInterp > OldNxEndInterp) ? ioc(nw.xStart, nw.xStep, OldNxEndInterp) : NewNx - 1;
        if (pxm > 1.) preserve('x');
        else {
            if (nw.xStart > nw.xWfrMin) nw.xWfrMin = nw.xStart;
            const double xEndNew = nw.xStart + nw.nx * nw.xStep;
            if (xEndNew < nw.xWfrMax) nw.xWfrMax = xEndNew;
        }
        const long NewNzLeftHalf = NewNz >> 1;
        nw.zStep = w.zStep / pzd;
        nw.zStart = Zc - NewNzLeftHalf * nw.zStep;
        tune_step_keep_interp_limits(w, nw, pzm, 'z', iZc);
        // the reference's z branch starts one node later and takes the end limit after the tuning
        nw.AuxLong3 = (nw.zStart < w.zStart) ? 1 + ioc(nw.zStart, nw.zStep, w.zStart) : 0;
        const double NewNzEndInterp = nw.zStart + (NewNz - 1) * nw.zStep;
        const double OldNzEndInterp = w.zStart + (w.nz - 1) * w.zStep;
        nw.AuxLong4 = (NewNzEndInterp > OldNzEndInterp) ? ioc(nw.zStart, nw.zStep, OldNzEndInterp) : NewNz - 1;
        if (pzm > 1.) preserve('z');
        else {
            if (nw.zStart > nw.zWfrMin) nw.zWfrMin = nw.zStart;
            const double zEndNew = nw.zStart + nw.nz * nw.zStep;
            if (zEndNew < nw.zWfrMax) nw.zWfrMax = zEndNew;
        }
    } else {
        double xMagOld = (w.nx - 1) * w.xStep;
        if (pxm > 1.) {
            long NxInner = (pxd != 1.) ? (long)(NewNx / pxm) : w.nx;
            long d = NewNx - NxInner;
            long left = d >> 1;
            if ((left << 1) != d) left++;
            nw.xStep = xMagOld / (NxInner - 1);
            nw.xStart = w.xStart - left * nw.xStep;
            nw.AuxLong1 = left;
            nw.AuxLong2 = left + NxInner - 1;
            preserve('x');
        } else {
            double xEndOld = w.xStart + (w.nx - 1) * w.xStep;
            double xMid = 0.5 * (w.xStart + xEndOld);
            double xMagNew = xMagOld * pxm;
            nw.xStep = xMagNew / (NewNx - 1);
            if (pxd == 1) { nw.xStep = w.xStep; xMagNew = (NewNx - 1) * nw.xStep; }
            nw.xStart = xMid - 0.5 * xMagNew;
            nw.AuxLong1 = 0;
            nw.AuxLong2 = NewNx - 1;
            if (nw.xStart > nw.xWfrMin) nw.xWfrMin = nw.xStart;
            if ((nw.xStart + xMagNew) < nw.xWfrMax) nw.xWfrMax = nw.xStart + xMagNew;
        }
        double zMagOld = (w.nz - 1) * w.zStep;
        if (pzm > 1.) {
            long NzInner = (pzd != 1.) ? (long)(NewNz / pzm) : w.nz;
            long d = NewNz - NzInner;
            long left = d >> 1;
            if ((left << 1) != d) left++;
            nw.zStep = zMagOld / (NzInner - 1);
            nw.zStart = w.zStart - left * nw.zStep;
            nw.AuxLong3 = left;
            nw.AuxLong4 = left + NzInner - 1;
            preserve('z');
        } else {
            double zEndOld = w.zStart + (w.nz - 1) * w.zStep;
            double zMid = 0.5 * (w.zStart + zEndOld);
            double zMagNew = zMagOld * pzm;
            nw.zStep = zMagNew / (NewNz - 1);
            if (pzd == 1) { nw.zStep = w.zStep; zMagNew = (NewNz - 1) * nw.zStep; }
            nw.zStart = zMid - 0.5 * zMagNew;
            nw.AuxLong3 = 0;
            nw.AuxLong4 = NewNz - 1;
            if (nw.zStart > nw.zWfrMin) nw.zWfrMin = nw.zStart;
            if ((nw.zStart + zMagNew) < nw.zWfrMax) nw.zWfrMax = nw.zStart + zMagNew;
        }
    }
    bool grow = (pxmIn * pxdIn * pzmIn * pzdIn) >= 1.;
    if (grow && changed) { WfrState t = w; w = nw; srwl_roundtrip(); nw = w; w = t; }

    const double RelStepTol = 1.e-05;
    bool only_larger = ((pxd == 1.) && (pzd == 1.) && (pxm >= 1.) && (pzm >= 1.)) &&
                       ((::fabs(old.xStep - nw.xStep) < RelStepTol) && (::fabs(old.zStep - nw.zStep) < RelStepTol));
    if (only_larger) {
        b->resize(old, nw, 1);
        w = nw;
    } else {
        bool origQX = old.QuadX, origQZ = old.QuadZ;
        // WaveFrontTermCanBeTreated (sroptelm.cpp:4692), checkBenefit = false
        bool qx = ::fabs(old.RobsXAbsErr) < 0.4 * ::fabs(old.RobsX);
        bool qz = ::fabs(old.RobsZAbsErr) < 0.4 * ::fabs(old.RobsZ);
        bool treated = false;
        if ((qx || qz) && old.Pres < 1) {
            w.QuadX = qx; w.QuadZ = qz;
            treat_quad('r');            // on the old mesh, before the gather
            nw.QuadX = qx; nw.QuadZ = qz;
            treated = true;
        }
        b->resize(old, nw, 0);
        w = nw;
        if (treated) treat_quad('a');   // on the new mesh
        w.QuadX = origQX; w.QuadZ = origQZ;
    }
    if (!grow && changed) srwl_roundtrip();
    if (other_side) {
        int to = (w.Pres == 0) ? 1 : 0;
        set_rad_repres(to);
        if (useStartTrOther) {
            double xcOld = xStartOld + (nxOld >> 1) * xStepOld;
            w.xStart = xcOld - (w.nx >> 1) * w.xStep;
            double zcOld = zStartOld + (nzOld >> 1) * zStepOld;
            w.zStart = zcOld - (w.nz >> 1) * w.zStep;
            set_full_range();
        }
    }
    return 0;
}

// ================================================================================================
// Container (PropagateRadiationGuided, sroptcnt.cpp:254-425)
// ================================================================================================
int Planner::plan(const SRWLWfr* pw, const SRWLOptC* opt)
{
    kernels.clear();
    tables.clear();
    maxElems = 0;
    err.clear();
    momOps.clear();
    nMomSlots = 0;
    momProvisional = false;
    intOuts.clear();
    intBytes = 0;
    nStages = 0;
    slotVals_.clear();
    pendingEstSlot_ = -1;
    elemIdx_ = 0;
    resizeDone_ = false;
    quadFlagsUncertain_ = false;
    if (pw == nullptr || opt == nullptr) return SRWL_INCORRECT_PARAM_FOR_WFR_PROP;
    // InSRWRadPtrs (srradstr.cpp:501)
    const SRWLRadMesh& m = pw->mesh;
    w = WfrState();
    w.eStart = m.eStart;
    if (m.nx <= 1) { w.xStart = 0.5 * (m.xStart + m.xFin); w.xStep = 0.; }
    else { w.xStart = m.xStart; w.xStep = (m.xFin - m.xStart) / (m.nx - 1); }
    if (m.ny <= 1) { w.zStart = 0.5 * (m.yStart + m.yFin); w.zStep = 0.; }
    else { w.zStart = m.yStart; w.zStep = (m.yFin - m.yStart) / (m.ny - 1); }
    w.nx = (int)m.nx; w.nz = (int)m.ny;
    w.yStart = m.zStart;
    w.RobsX = pw->Rx; w.RobsZ = pw->Ry; w.RobsXAbsErr = pw->dRx; w.RobsZAbsErr = pw->dRy;
    w.xc = pw->xc; w.zc = pw->yc;
    w.xWfrMin = m.xStart; w.xWfrMax = m.xFin; w.zWfrMin = m.yStart; w.zWfrMax = m.yFin;
    w.Pres = pw->presCA;
    w.avgPhotEn = pw->avgPhotEn;
    if (pw->arMomX != nullptr) { for (int i = 0; i < 11; i++) w.momX[i] = pw->arMomX[i]; w.haveMom = true; }
    if (pw->arMomY != nullptr) for (int i = 0; i < 11; i++) w.momZ[i] = pw->arMomY[i];
    if (pw->arElecPropMatr != nullptr) {
        for (int i = 0; i < 20; i++) w.propM[i] = pw->arElecPropMatr[i];
        w.havePropM = true;
    }
    if (m.ne != 1) { err = "only ne == 1 wavefronts are supported on the GPU path"; return SRWG_ERR_UNSUPPORTED; }
    if (pw->presFT != 0) { err = "time-domain wavefronts are not supported on the GPU path"; return SRWG_ERR_UNSUPPORTED; }
    if (pw->numTypeElFld != 0 && pw->numTypeElFld != 'f') { err = "only float fields are supported"; return SRWG_ERR_UNSUPPORTED; }
    in = w;
    stageIn = w;
    els_.clear();
    props_.clear();
    trTables_.clear();
    int r = flatten(opt, els_, props_, false);
    if (r) return r;
    if ((w.nx <= 1) || (w.nz <= 1)) return CAN_NOT_PROPAGATE_1D_RAD;   // CheckRadStructForPropagation
    return run();
}

int Planner::resume(const double* slots)
{
    // moments as they stand after the stage: the bookkeeping replayed with every result so far
    slotVals_.assign(slots, slots + (size_t)nMomSlots * SRWG_MOM_SLOT);
    replay_moments(slotVals_.data(), w.momX, w.momZ, &w.QuadX, &w.QuadZ);
    momProvisional = false;
    quadFlagsUncertain_ = false;
    kernels.clear();
    tables.clear();
    intOuts.clear();
    intBytes = 0;
    maxElems = 0;
    stageIn = w;
    nStages++;
    return run();
}

// plans the chain from the element reached; a stage boundary (SRWG_NEED_STAGE) leaves a complete
// pass list behind and the element to be planned again on resume (its pre-resize already done)
int Planner::run()
{
    Builder bld(kernels, maxElems);
    b = &bld;
    const double tolRes = 1.e-04;
    const std::vector<ElemDesc>& els = els_;
    const std::vector<PropDesc>& props = props_;
    try {
        if (inPhase && nStages == 0 && elemIdx_ == 0 && !resizeDone_) b->quad(w, 0., inKx, 0., inKz, inC);
        size_t numRes = props.size();
        size_t& i = elemIdx_;
        for (; i < els.size(); i++, resizeDone_ = false) {
            const ElemDesc& e = els[i];
            int anal = 0;
            if (i < numRes) {
                const PropDesc& p = props[i];
                if (p.n >= 0) {
                    if ((int)p.get(0, 0) || (int)p.get(1, 0)) {
                        err = "automatic resizing (pp[0], pp[1]) is not supported on the GPU path";
                        throw (int)SRWG_ERR_UNSUPPORTED;
                    }
                    anal = (int)p.get(3, 0);
                    double pxm = p.get(5, 1.), pxd = p.get(6, 1.), pzm = p.get(7, 1.), pzd = p.get(8, 1.);
                    int sh = (int)(char)p.get(9, 0);
                    if (!resizeDone_ && ((::fabs(pxd - 1.) > tolRes) || (::fabs(pxm - 1.) > tolRes) ||
                                         (::fabs(pzd - 1.) > tolRes) || (::fabs(pzm - 1.) > tolRes) || (sh > 0))) {
                        int rr = resize(pxm, pxd, pzm, pzd, sh, p.get(10, 0.), p.get(11, 0.), (int)p.get(4, 0) != 0);
                        if (rr) throw rr;
                    }
                    resizeDone_ = true;
                }
            }
            if (e.kind == E_DRIFT) drift(e, anal);
            else if (e.kind == E_LENS) lens(e);
            else if (e.kind == E_APERTURE) aperture(e);
            else if (e.kind == E_TRANSM) transmission(e);
            // extractions after a top-level element: after the last element of a nested container
            if (!intReqs.empty() && (i + 1 == els.size() || els[i + 1].outer != e.outer)) extract_after(e.outer);
        }
        if (i < numRes) {
            const PropDesc& p = props[i];
            if (p.n >= 0) {
                double pxm = p.get(5, 1.), pxd = p.get(6, 1.), pzm = p.get(7, 1.), pzd = p.get(8, 1.);
                if ((::fabs(pxd - 1.) > tolRes) || (::fabs(pxm - 1.) > tolRes) || (::fabs(pzd - 1.) > tolRes) ||
                    (::fabs(pzm - 1.) > tolRes)) {
                    int rr = resize(pxm, pxd, pzm, pzd, 0, 0., 0., (int)p.get(4, 0) != 0);
                    if (rr) throw rr;
                }
            }
            if (!intReqs.empty()) extract_after(els.empty() ? 0 : els.back().outer + 1);   // after the post-resize (sroptcnt.cpp:421)
        }
    } catch (int code) {
        if (code != SRWG_NEED_STAGE) {
            b = nullptr;
            return code;
        }
        bld.close();
        outBuf = bld.cur;
        b = nullptr;
        int r = finalize();
        return r ? r : SRWG_NEED_STAGE;
    }
    bld.close();
    outBuf = bld.cur;
    b = nullptr;
    return finalize();
}

// Box of old-mesh indices [i0, i1] x [j0, j1] outside which the point-wise work `pw` (indices of an
// nx x nz mesh) zeroes the field: the intersection of its apertures' (not obstacles') rectangles or
// the squares around their circles, widened by 2 indices against rounding of the coordinates.
// False when it has no aperture mask.
static bool aperture_box(const PwOps& pw, int nx, int nz, int& i0, int& i1, int& j0, int& j1)
{
    bool any = false;
    i0 = 0; i1 = nx - 1; j0 = 0; j1 = nz - 1;
    for (int m = 0; m < pw.nmask; m++) {
        const PwMask& k = pw.mask[m];
        if (k.obstacle || k.dx == 0. || k.dz == 0.) continue;
        const double hx = k.type == 1 ? k.hx : std::sqrt(k.r2), hz = k.type == 1 ? k.hz : std::sqrt(k.r2);
        auto range = [](double lo, double hi, double x0, double dx, int n, int& a, int& b) {
            double u = (lo - x0) / dx, v = (hi - x0) / dx;
            if (u > v) std::swap(u, v);
            const double fa = std::floor(u) - 2., fb = std::ceil(v) + 2.;
            a = std::max(a, (int)std::max(-1., std::min((double)n, fa)));
            b = std::min(b, (int)std::max(-1., std::min((double)n, fb)));
        };
        range(k.cx - hx, k.cx + hx, k.x0, k.dx, nx, i0, i1);
        range(k.cz - hz, k.cz + hz, k.z0, k.dz, nz, j0, j1);
        any = true;
    }
    return any;
}

// new indices in [s, e] whose gather stencil (old nodes st .. st+3, ResizeAxis at float2 offset
// `off` of the tables) meets the old indices [lo, hi]: a contiguous range (st is non-decreasing)
static void stencil_window(const std::vector<float2>& T, long long off, int lo, int hi, int& s, int& e)
{
    int a = s, b = e;
    ResizeAxis x;
    while (a <= b) {
        memcpy(&x, &T[off + 2 * a], sizeof(x));
        if (x.st + 3 >= lo) break;
        a++;
    }
    while (b >= a) {
        memcpy(&x, &T[off + 2 * b], sizeof(x));
        if (x.st <= hi) break;
        b--;
    }
    s = a;
    e = b;
}

// checks the passes of the plan (or stage), fills their tables and links neighbouring passes
int Planner::finalize()
{
    // the GPU passes need even line lengths (centring rotation) and at most 16384 points per line
    for (const KernelDesc& k : kernels) {
        if (k.kind == K_LINE) {
            int N = k.line.axis == 0 ? k.line.nx : k.line.nz;
            if ((N & 1) || N > 16384 || N < 4) {
                err = "FFT length " + std::to_string(N) + " not supported on the GPU path (even, 4..16384)";
                return SRWG_ERR_UNSUPPORTED;
            }
        }
        if (k.kind == K_RESIZE && !k.rs.only_larger && (k.rs.nxo < 4 || k.rs.nzo < 4)) {
            err = "resize of a mesh smaller than 4 points";
            return SRWG_ERR_UNSUPPORTED;
        }
    }
    build_tables(kernels, tables);
    // transmission tables after the separable ones (each double of a (T, OPD) pair in one float2
    // slot), and their offsets into every point-wise description that uses them
    if (!trTables_.empty()) {
        std::vector<long long> base(trTables_.size(), -1);
        auto patch = [&](PwOps& o) {
            if (!o.has_tr) return;
            if (base[o.tr_id] < 0) {
                base[o.tr_id] = (long long)tables.size();
                const std::vector<double>& t = trTables_[o.tr_id];
                const size_t at = tables.size();
                tables.resize(at + t.size());
                memcpy(&tables[at], t.data(), t.size() * sizeof(double));
            }
            o.tr_off = base[o.tr_id];
        };
        for (KernelDesc& k : kernels) {
            if (k.kind == K_LINE) { patch(k.line.pw); patch(k.line.extra); }
            else if (k.kind == K_RESIZE) { patch(k.rs.pw); patch(k.rs.extra); patch(k.rs.pre); patch(k.rs.pre_extra); }
            else if (reads_only(k.kind)) { patch(k.mom.pw); patch(k.mom.extra); }
            else { patch(k.pwk.pw); patch(k.pwk.extra); }
        }
    }
    // a tiled resize followed by a line pass on its output writes only its window; the line pass
    // reads zeros outside it (the buffer is overwritten before anything else reads it)
    for (size_t i = 0; i + 1 < kernels.size(); i++) {
        ResizeDesc& r = kernels[i].rs;
        KernelDesc& n = kernels[i + 1];
        if (kernels[i].kind != K_RESIZE || r.only_larger || r.tile_or == 0 || n.kind != K_LINE ||
            n.src != kernels[i].dst || n.line.nx != r.nxn || n.line.nz != r.nzn)
            continue;
        const int N = n.line.axis == 0 ? n.line.nx : n.line.nz;
        if (fixed_lines_per_cta(n.line.axis, N) == 0) continue;      // compile-time-length line kernels only
        LineDesc& d = n.line;
        int ixs = (int)std::max(0L, r.ixStart), ixe = (int)std::min((long)r.nxn - 1, r.ixEnd);
        int izs = (int)std::max(0L, r.izStart), ize = (int)std::min((long)r.nzn - 1, r.izEnd);
        // an aperture folded in before the resampling zeroes the old field outside its box: the new
        // points whose stencils miss the box are zeros, so the window (what the resize computes and
        // the line pass loads) shrinks to the new points whose stencils meet it
        int i0, i1, j0, j1;
        if (r.has_pre && ixs <= ixe && izs <= ize && aperture_box(r.pre, r.nxo, r.nzo, i0, i1, j0, j1)) {
            int a = ixs, b = ixe, c = izs, e = ize;
            stencil_window(tables, r.axx, i0, i1, a, b);
            stencil_window(tables, r.axz, j0, j1, c, e);
            if (a <= b && c <= e) {
                ixs = a; ixe = b; izs = c; ize = e;
                r.ixStart = a; r.ixEnd = b; r.izStart = c; r.izEnd = e;
            }
        }
        r.skip_zero = 1;
        d.zwin = 1;
        if (d.axis == 0) { d.zl0 = izs; d.zl1 = ize; d.za0 = ixs; d.za1 = ixe; }
        else { d.zl0 = ixs; d.zl1 = ixe; d.za0 = izs; d.za1 = ize; }
    }
    // a row pass followed by a column pass on its output writes it in blocks of as many columns as
    // a column CTA transforms, so that the column pass reads whole blocks sequentially
    for (size_t i = 0; i + 1 < kernels.size(); i++) {
        KernelDesc& a = kernels[i];
        KernelDesc& n = kernels[i + 1];
        if (a.kind != K_LINE || n.kind != K_LINE || a.line.axis != 0 || n.line.axis != 1 || n.src != a.dst ||
            a.line.nx != n.line.nx || a.line.nz != n.line.nz)
            continue;
        const int Nr = a.line.nx, Nc = n.line.nz;
        if (fixed_lines_per_cta(0, Nr) == 0 || fixed_lines_per_cta(1, Nc) == 0) continue;
        const int bw = fixed_lines_per_cta(1, Nc);
        if (bw < 2 || (bw & (bw - 1)) != 0 || n.line.nx % bw != 0) continue;
        a.line.blk_out = bw;
        n.line.blk_in = bw;
    }
    // a row pass that transforms only the rows of a resize window: the column pass on its output
    // loads only those rows of every column (the same window along its lines), so the row pass does
    // not write the other (zero) rows at all
    for (size_t i = 0; i + 1 < kernels.size(); i++) {
        KernelDesc& a = kernels[i];
        KernelDesc& n = kernels[i + 1];
        if (a.kind != K_LINE || n.kind != K_LINE || a.line.axis != 0 || n.line.axis != 1 || !a.line.zwin ||
            n.line.zwin || n.src != a.dst || a.line.nx != n.line.nx || a.line.nz != n.line.nz)
            continue;
        const int Nc = n.line.nz;
        if (fixed_lines_per_cta(1, Nc) == 0) continue;
        const int nz = a.line.nz;
        LineDesc& d = n.line;
        d.zwin = 1;
        d.zl0 = 0;
        d.zl1 = n.line.nx - 1;
        d.za0 = a.line.mirror_lines ? nz - 1 - a.line.zl1 : a.line.zl0;
        d.za1 = a.line.mirror_lines ? nz - 1 - a.line.zl0 : a.line.zl1;
        a.line.zskip = 1;
    }
    return 0;
}

std::string Planner::describe() const
{
    std::string s;
    char buf[512];
    for (size_t i = 0; i < kernels.size(); i++) {
        const KernelDesc& k = kernels[i];
        if (k.kind == K_LINE) {
            const LineDesc& d = k.line;
            // kernel family of the pass: power-of-two, specialised general length, run-time
            // scheduled general length, table-driven
            LineLaunch lp;
            memset(&lp, 0, sizeof(lp));
            const char* fam = line_config(d, lp) ? "none" : lp.v2 == 1 ? "pow2" : lp.v2 == 3 ? "spec" : lp.v2 == 2 ? "gen" : "tab";
            char win[96] = "";
            if (d.zwin) snprintf(win, sizeof(win), "  lines=%d:%d points=%d:%d", d.zl0, d.zl1, d.za0, d.za1);
            if (d.out_int)
                snprintf(win + strlen(win), sizeof(win) - strlen(win), "  intensity%s", d.int_flat ? " flat" : "");
            snprintf(buf, sizeof(buf), "%zu LINE %s %dx%d f1=%d pw=%d(q%d a%d m%d s%d) mir=%d/%d f2=%d zwin=%d blk=%d/%d  buf %d->%d  fft=%s L=%d%s\n",
                     i, d.axis == 0 ? "rows" : "cols", d.nx, d.nz, d.f1, d.has_pw, d.pw.has_quad, d.pw.has_ang, d.pw.nmask,
                     d.pw.has_scale, d.mirror_along, d.mirror_lines, d.f2, d.zwin, d.blk_in, d.blk_out, k.src, k.dst, fam, lp.L,
                     win);
        } else if (k.kind == K_RESIZE) {
            snprintf(buf, sizeof(buf), "%zu RESIZE %dx%d -> %dx%d only_larger=%d pre=%d pw=%d tile=%dx%d  buf %d->%d  window=x%ld:%ld,z%ld:%ld\n",
                     i, k.rs.nxo, k.rs.nzo, k.rs.nxn, k.rs.nzn, k.rs.only_larger, k.rs.has_pre, k.rs.has_pw, k.rs.tile_or,
                     k.rs.tile_oc, k.src, k.dst, k.rs.ixStart, k.rs.ixEnd, k.rs.izStart, k.rs.izEnd);
        } else if (k.kind == K_MOM) {
            snprintf(buf, sizeof(buf), "%zu MOM %dx%d (q%d a%d m%d s%d) slot=%d  buf %d\n", i, k.mom.nx, k.mom.nz,
                     k.mom.pw.has_quad, k.mom.pw.has_ang, k.mom.pw.nmask, k.mom.pw.has_scale, k.mom.slot, k.src);
        } else if (k.kind == K_INT) {
            snprintf(buf, sizeof(buf), "%zu INT %dx%d (q%d a%d m%d s%d) pol=%d what=%d off=%lld  buf %d\n", i, k.mom.nx,
                     k.mom.nz, k.mom.pw.has_quad, k.mom.pw.has_ang, k.mom.pw.nmask, k.mom.pw.has_scale, k.mom.ipol,
                     k.mom.iwhat, k.mom.ioff, k.src);
        } else {
            snprintf(buf, sizeof(buf), "%zu PW %dx%d (q%d a%d m%d s%d) mirror=%d/%d  buf %d->%d\n", i, k.pwk.nx, k.pwk.nz,
                     k.pwk.pw.has_quad, k.pwk.pw.has_ang, k.pwk.pw.nmask, k.pwk.pw.has_scale, k.pwk.mirror_x,
                     k.pwk.mirror_z, k.src, k.dst);
        }
        s += buf;
    }
    return s;
}

}  // namespace srwg
