// Partially coherent (multi-electron) propagation in batches.
//
// The reference averages the intensity of many macro-electron wavefronts in a Python loop
// (srwl_wfr_emit_prop_multi_e, env/python/srwpy/srwlib.py:8506): per electron a field, then
// srwlPropagElecField, srwlCalcIntFromElecField (total polarisation, intensity vs x and y) and
// avg_update_interp (srwlib.py:1116) onto a common mesh.  Here the electrons' wavefronts are made
// on the device from one base field by the source offset of SRWLWfr.sim_src_offset with
// _move_mesh=True (srwlib.py:2803): the angular kick of srTOptAngle (cpp/src/core/sroptang.h:64,
// phase 5.06773065e6 * e * (x' x + y' y) on the unshifted mesh) followed by a shift of the mesh by
// (x + x' R, y + y' R), R = (Rx + Ry)/2, and xc += x, yc += y.  Each electron is planned on the host
// (its own mesh, exact bookkeeping), the kick being a linear phase that the planner fuses into the
// first pass (no kicked copy of the field is written: every electron's first pass reads the base
// field); electrons whose passes have the same kinds and sizes run together: every pass is ONE
// launch over the batch (grid z = electron, per-electron descriptors and tables), then one kernel
// adds the batch's intensities, interpolated bilinearly onto the common mesh as avg_update_interp
// does with order 1, to an FP64 accumulator on the device.
// With `graph` set, the launch sequence of a full batch is captured once as a CUDA graph and
// replayed (only the descriptor and parameter uploads change between batches).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/srwl_b200.h"
#include "common.cuh"
#include "errors.h"
#include "exec.h"
#include "kernels.h"
#include "planner.h"
#include "workers.h"

namespace srwg {

// per-electron parameters in device memory
struct ElecParams {
    double kx, kz;                       // kick: phase kx x + kz z on the base mesh (fused by the planner)
    double dx, dz;                       // mesh shift of the electron's wavefront
    double oxStart, oxStep, ozStart, ozStep;   // output mesh (steps as (Fin - Start)/(n - 1))
    double oxInv, ozInv;                       // 1 / step: the accumulation multiplies (no FP64 divisions)
    int onx, onz;
    int pad[2];
};

// acc[p] += sum over the batch of the bilinearly interpolated total intensity at common-mesh
// point p (avg_update_interp, order 1: points outside an electron's mesh add nothing)
__global__ void __launch_bounds__(256) accum_kernel(const float2* __restrict__ ex, const float2* __restrict__ ey,
                                                    long long stride, int nb, const ElecParams* __restrict__ ep,
                                                    double* __restrict__ acc, int anx, int anz, double axStart,
                                                    double axStep, double azStart, double azStep)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= anx) return;
    const double x = axStart + (double)i * axStep, y = azStart + (double)j * azStep;
    double sum = 0.;
    for (int b = 0; b < nb; b++) {
        const ElecParams& e = ep[b];
        const int ix0 = (int)trunc((x - e.oxStart) * e.oxInv + 1.e-09);
        if (ix0 < 0 || ix0 >= e.onx - 1) continue;
        const int iy0 = (int)trunc((y - e.ozStart) * e.ozInv + 1.e-09);
        if (iy0 < 0 || iy0 >= e.onz - 1) continue;
        const double tx = (x - (e.oxStart + e.oxStep * ix0)) * e.oxInv;
        const double ty = (y - (e.ozStart + e.ozStep * iy0)) * e.ozInv;
        const float2* px = ex + (size_t)b * stride + (size_t)iy0 * e.onx + ix0;
        const float2* py = ey + (size_t)b * stride + (size_t)iy0 * e.onx + ix0;
        float I[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const size_t o = (c >> 1) * (size_t)e.onx + (c & 1);
            const float2 u = __ldg(&px[o]), v = __ldg(&py[o]);
            I[c] = u.x * u.x + u.y * u.y + v.x * v.x + v.y * v.y;     // total intensity (FP32, as the reference)
        }
        const double a00 = I[0], f10 = I[1], f01 = I[2], f11 = I[3];
        const double a10 = f10 - a00, a01 = f01 - a00, a11 = a00 - f01 - f10 + f11;
        sum += a00 + tx * (a10 + ty * a11) + ty * a01;
    }
    acc[(size_t)j * anx + i] += sum;
}

// the same with the intensities written by the last pass (an intensity pass, float per point of the
// electron's onz x onx mesh at stride `stride` floats): row-major (bw 0) or in blocks of bw columns
// (point (ix, iy) at ((ix / bw) onz + iy) bw + ix % bw)
__global__ void __launch_bounds__(256) accum_int_kernel(const float* __restrict__ in, long long stride, int nb,
                                                        const ElecParams* __restrict__ ep, double* __restrict__ acc,
                                                        int anx, int anz, double axStart, double axStep,
                                                        double azStart, double azStep, int bw)
{
    // column blocks (bw > 0): the threads of a CTA walk a common-mesh column, so that neighbouring
    // threads read neighbouring rows of one block (contiguous); row-major: they walk a row
    const int i = bw > 0 ? (int)blockIdx.y : (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = bw > 0 ? (int)(blockIdx.x * blockDim.x + threadIdx.x) : (int)blockIdx.y;
    if (i >= anx || j >= anz) return;
    const double x = axStart + (double)i * axStep, y = azStart + (double)j * azStep;
    double sum = 0.;
    for (int b = 0; b < nb; b++) {
        const ElecParams& e = ep[b];
        const int ix0 = (int)trunc((x - e.oxStart) * e.oxInv + 1.e-09);
        if (ix0 < 0 || ix0 >= e.onx - 1) continue;
        const int iy0 = (int)trunc((y - e.ozStart) * e.ozInv + 1.e-09);
        if (iy0 < 0 || iy0 >= e.onz - 1) continue;
        const double tx = (x - (e.oxStart + e.oxStep * ix0)) * e.oxInv;
        const double ty = (y - (e.ozStart + e.ozStep * iy0)) * e.ozInv;
        const float* pe = in + (size_t)b * stride;
        double a00, f10, f01, f11;
        if (bw > 0) {
            const size_t c0 = ((size_t)(ix0 / bw) * e.onz + iy0) * bw + ix0 % bw;
            const size_t c1 = ((size_t)((ix0 + 1) / bw) * e.onz + iy0) * bw + (ix0 + 1) % bw;
            a00 = __ldg(&pe[c0]); f01 = __ldg(&pe[c0 + bw]);
            f10 = __ldg(&pe[c1]); f11 = __ldg(&pe[c1 + bw]);
        } else {
            const float* pi = pe + (size_t)iy0 * e.onx + ix0;
            a00 = __ldg(&pi[0]); f10 = __ldg(&pi[1]); f01 = __ldg(&pi[e.onx]); f11 = __ldg(&pi[e.onx + 1]);
        }
        const double a10 = f10 - a00, a01 = f01 - a00, a11 = a00 - f01 - f10 + f11;
        sum += a00 + tx * (a10 + ty * a11) + ty * a01;
    }
    acc[(size_t)j * anx + i] += sum;
}

// magnitude^2 of the n complex values at float2 offset `off` of the plan's tables when all of them
// have it (relative spread within 1e-6), else -1
static double flat_mag2(const std::vector<float2>& T, long long off, int n)
{
    if (off < 0) return 1.;
    if (n <= 0 || off + n > (long long)T.size()) return -1.;
    double lo = 1e300, hi = 0.;
    for (int i = 0; i < n; i++) {
        const double a = (double)T[off + i].x * T[off + i].x + (double)T[off + i].y * T[off + i].y;
        lo = std::min(lo, a);
        hi = std::max(hi, a);
    }
    return (hi > 0. && hi - lo <= 1e-6 * hi) ? 0.5 * (lo + hi) : -1.;
}

// the last pass writes the total intensity instead of the two fields where it runs on a specialised
// kernel with one transform and no non-separable work (the accumulation then reads one float per
// sample instead of two complex values).  Where its output factors -- the output chain's table along
// the lines and every chain's line factor -- have one magnitude, |f v|^2 = |f|^2 |v|^2: the pass
// skips them and scales the intensity by that magnitude squared.
static void mark_intensity_pass(std::vector<KernelDesc>& ks, const std::vector<float2>& tables)
{
    for (size_t i = ks.size(); i-- > 0;) {
        if (reads_only(ks[i].kind)) continue;
        LineDesc& d = ks[i].line;
        if (ks[i].kind == K_LINE && !d.has_extra && !(d.f1 && d.f2)) {
            const int N = d.axis == 0 ? d.nx : d.nz, nl = d.axis == 0 ? d.nz : d.nx;
            if (fixed_family(d.axis, N) == FAM_SPEC) {
                d.out_int = 1;
                // a column pass writes the intensity in blocks of its tile's columns (contiguous
                // pieces); the accumulation reads that layout
                const int bw = fixed_lines_per_cta(1, N);
                if (d.axis == 1 && d.blk_out == 0 && bw > 1 && d.nx % bw == 0) d.blk_out = bw;
                const ChainTab& out = d.f1 ? d.t_mid : d.t_fin;
                const double a = flat_mag2(tables, out.tab, N), b = flat_mag2(tables, d.t_pre.ltab, nl),
                             c = flat_mag2(tables, d.t_mid.ltab, nl), e = flat_mag2(tables, d.t_fin.ltab, nl);
                if (a >= 0. && b >= 0. && c >= 0. && e >= 0.) {
                    d.int_flat = 1;
                    d.int_scale = (float)(a * b * c * e);
                }
            }
        }
        return;
    }
}

static bool intensity_pass(const std::vector<KernelDesc>& ks, int* bw = nullptr)
{
    for (size_t i = ks.size(); i-- > 0;)
        if (!reads_only(ks[i].kind)) {
            const bool yes = ks[i].kind == K_LINE && ks[i].line.out_int;
            if (bw) *bw = yes && ks[i].line.axis == 1 ? ks[i].line.blk_out : 0;
            return yes;
        }
    return false;
}

}  // namespace srwg

using namespace srwg;

struct srwgMultiE {
    int device = 0;
    DeviceCtx* ctx = nullptr;
    // base wavefront (host copy of its description; field on the device)
    SRWLWfr base;
    std::vector<double> momX, momY;
    const SRWLOptC* opt = nullptr;       // caller-owned beamline
    int nx = 0, nz = 0;
    double xStart = 0, xStep = 0, zStart = 0, zStep = 0, eStart = 0;
    float2* dBase = nullptr;             // [2][nIn]
    // common mesh and FP64 accumulator
    int anx = 0, anz = 0;
    double axStart = 0, axStep = 0, azStart = 0, azStep = 0;
    double* dAcc = nullptr;
    double* dSnap = nullptr;             // the accumulator as it was before the current add call
    bool ownAcc = true;                  // false: caller-provided accumulator (srwgMultiESetAccumulator)
    long long nAdded = 0;
    // batch buffers
    int maxBatch = 0;
    size_t nIn = 0, nOut = 0, perWork = 0, constStride = 0, descOff = 0;
    float2* dOut = nullptr;              // [2][B][nOut]
    float2* dWork = nullptr;             // [4][B][perWork]
    // per-electron constants (tables, descriptors) and parameters in two slots used in turn: the
    // host stages batch k+1 in pinned memory and a copy stream uploads it while batch k runs
    char* dConst[2] = {nullptr, nullptr};          // [B][constStride] per slot
    ElecParams* dParams[2] = {nullptr, nullptr};   // [B] per slot
    char* hConst[2] = {nullptr, nullptr};          // pinned staging
    ElecParams* hParams[2] = {nullptr, nullptr};
    cudaEvent_t staged[2] = {nullptr, nullptr};    // the slot's upload has completed
    cudaEvent_t used[2] = {nullptr, nullptr};      // the last batch that read the slot has completed
    cudaStream_t copy = nullptr;                   // upload stream
    int slot = 0;
    int upTo = 0;                        // electrons of the current slot already uploaded
    bool upWaited = false;               // the copy stream waits for the slot's last reader
    bool useGraph = false;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // per slot
    std::vector<KernelDesc> graphKs[2];  // host copy (launch shapes) each graph was captured with
    std::vector<cudaEvent_t> tev;        // srwgMultiEAddTimed: events around every pass and the accumulation
    long long nFlush = 0;                // batches run so far
    std::unique_ptr<WorkerPool> pool;    // host threads planning the electrons and staging their constants
    ~srwgMultiE()
    {
        pool.reset();
        for (cudaEvent_t e : tev) cudaEventDestroy(e);
        for (int i = 0; i < 2; i++)
            if (graph[i]) cudaGraphExecDestroy(graph[i]);
        if (ownAcc) cudaFree(dAcc);
        cudaFree(dSnap);
        cudaFree(dBase); cudaFree(dOut); cudaFree(dWork);
        for (int i = 0; i < 2; i++) {
            cudaFree(dConst[i]);
            cudaFree(dParams[i]);
            cudaFreeHost(hConst[i]);
            cudaFreeHost(hParams[i]);
            if (staged[i]) cudaEventDestroy(staged[i]);
            if (used[i]) cudaEventDestroy(used[i]);
        }
        if (copy) cudaStreamDestroy(copy);
    }
};

namespace srwg {

#define MTRY(x)                                                                          \
    do {                                                                                 \
        cudaError_t e__ = (x);                                                           \
        if (e__ != cudaSuccess) {                                                        \
            set_last_detail(std::string(#x) + ": " + cudaGetErrorString(e__));           \
            return SRWG_ERR_CUDA;                                                        \
        }                                                                                \
    } while (0)

// the electron's wavefront description: kicked on the base mesh, then the mesh moved
// (SRWLWfr.sim_src_offset with _move_mesh=True, srwlib.py:2803-2849; srTOptAngle moments, sroptang.h:81)
// With a fifth value (relative electron energy deviation d), the photon energy of the electron's
// wavefront is rescaled to E (1 + 2 d), the shift of an undulator harmonic with the electron energy.
static void electron_wfr(const srwgMultiE& m, const double* off, int stride, SRWLWfr& w, double* momX, double* momY,
                         ElecParams& ep)
{
    const double dx0 = off[0], dxp = off[1], dy0 = off[2], dyp = off[3];
    const double de = stride > 4 ? off[4] : 0.;
    w = m.base;
    for (int i = 0; i < 11; i++) { momX[i] = m.momX[i]; momY[i] = m.momY[i]; }
    w.arMomX = momX;
    w.arMomY = momY;
    const double E = de != 0. ? m.eStart * (1. + 2. * de) : m.eStart;
    if (de != 0.) { w.mesh.eStart = E; w.mesh.eFin = E; }
    const double twoPiDLambda = 5.06773065e+06 * E;
    ep.kx = twoPiDLambda * dxp;
    ep.kz = twoPiDLambda * dyp;
    momX[1] += dxp; momX[3] += dyp; momY[1] += dxp; momY[3] += dyp;     // srTOptAngle::PropagateRadMoments
    const double R = 0.5 * (w.Rx + w.Ry);
    const double dx = dx0 + dxp * R, dy = dy0 + dyp * R;
    ep.dx = dx;
    ep.dz = dy;
    w.mesh.xStart += dx; w.mesh.xFin += dx;
    w.mesh.yStart += dy; w.mesh.yFin += dy;
    w.xc += dx0; w.yc += dy0;
    momX[0] += dx; momX[1] += dxp; momX[2] += dy; momX[3] += dyp;
    momY[0] += dx; momY[1] += dxp; momY[2] += dy; momY[3] += dyp;
}

// passes of the same kinds, sizes, buffers and launch-relevant flags
static bool same_structure(const std::vector<KernelDesc>& a, const std::vector<KernelDesc>& b)
{
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); i++) {
        const KernelDesc &x = a[i], &y = b[i];
        if (x.kind != y.kind || x.src != y.src || x.dst != y.dst) return false;
        if (x.kind == K_LINE) {
            const LineDesc &p = x.line, &q = y.line;
            if (p.axis != q.axis || p.nx != q.nx || p.nz != q.nz || p.f1 != q.f1 || p.f2 != q.f2 ||
                p.has_extra != q.has_extra || p.zwin != q.zwin || p.blk_in != q.blk_in || p.blk_out != q.blk_out ||
                p.out_int != q.out_int || p.int_flat != q.int_flat)
                return false;
        } else if (x.kind == K_RESIZE) {
            const ResizeDesc &p = x.rs, &q = y.rs;
            if (p.nxo != q.nxo || p.nzo != q.nzo || p.nxn != q.nxn || p.nzn != q.nzn || p.only_larger != q.only_larger ||
                (p.tile_or > 0) != (q.tile_or > 0) || p.skip_zero != q.skip_zero)
                return false;
        } else {
            if (x.pwk.nx != y.pwk.nx || x.pwk.nz != y.pwk.nz) return false;
        }
    }
    return true;
}

// runs one batch: passes (the first one applies each electron's kick) -> accumulation; ks = launch
// shapes (largest resize tiles of the batch)
static int run_batch(srwgMultiE& m, int nb, const std::vector<KernelDesc>& ks, cudaStream_t st, int slot)
{
    dim3 blk(256);
    float2* outX = m.dOut;
    float2* outY = m.dOut + (size_t)m.maxBatch * m.nOut;
    if (ks.empty()) { set_last_detail("multi-electron plan without passes"); return SRWG_ERR_BAD_ARG; }
    // every electron's first pass reads the base field (input stride 0) and applies its kick
    cudaEvent_t* ev = m.tev.size() >= 2 * ks.size() + 2 ? m.tev.data() : nullptr;
    int r = execute_passes(ks, *m.ctx, nb, m.dBase, m.dBase + m.nIn, 0, outX, outY, (long long)m.nOut, m.dWork,
                           m.perWork, m.dConst[slot], (long long)m.constStride, m.descOff, st, ev, &ks);
    if (r) return r;
    dim3 ga((m.anx + 255) / 256, m.anz);
    if (ev) MTRY(cudaEventRecord(ev[2 * ks.size()], st));
    int bw = 0;
    if (intensity_pass(ks, &bw))
        accum_int_kernel<<<bw > 0 ? dim3((m.anz + 255) / 256, m.anx) : ga, blk, 0, st>>>(
            reinterpret_cast<const float*>(outX), (long long)m.nOut, nb, m.dParams[slot],
                                             m.dAcc, m.anx, m.anz, m.axStart, m.axStep, m.azStart, m.azStep, bw);
    else
        accum_kernel<<<ga, blk, 0, st>>>(outX, outY, (long long)m.nOut, nb, m.dParams[slot], m.dAcc, m.anx, m.anz,
                                         m.axStart, m.axStep, m.azStart, m.azStep);
    MTRY(cudaGetLastError());
    if (ev) MTRY(cudaEventRecord(ev[2 * ks.size() + 1], st));
    return 0;
}

// uploads the staged constants of nb electrons (copy stream, after the last batch that read the slot)
// and runs (or replays) the batch on `st` once the upload has landed; the host then stages the next
// batch in the other slot, once that slot's previous upload has completed
// uploads the staged constants of electrons upTo .. nb - 1 of the current slot (copy stream, after
// the last batch that read the slot): a batch is uploaded in pieces while its later electrons are
// still being planned
static int upload_staged(srwgMultiE& m, int nb)
{
    const int s = m.slot;
    if (nb <= m.upTo) return 0;
    if (!m.upWaited) {
        MTRY(cudaStreamWaitEvent(m.copy, m.used[s], 0));
        m.upWaited = true;
    }
    const size_t a = (size_t)m.upTo, n = (size_t)(nb - m.upTo);
    MTRY(cudaMemcpyAsync(m.dConst[s] + a * m.constStride, m.hConst[s] + a * m.constStride, n * m.constStride,
                         cudaMemcpyHostToDevice, m.copy));
    MTRY(cudaMemcpyAsync(m.dParams[s] + a, m.hParams[s] + a, n * sizeof(ElecParams), cudaMemcpyHostToDevice, m.copy));
    m.upTo = nb;
    return 0;
}

static int flush(srwgMultiE& m, int nb, std::vector<KernelDesc>& ks, cudaStream_t st)
{
    if (nb == 0) return 0;
    m.nFlush++;
    const int s = m.slot;
    int ru = upload_staged(m, nb);
    if (ru) return ru;
    MTRY(cudaEventRecord(m.staged[s], m.copy));
    MTRY(cudaStreamWaitEvent(st, m.staged[s], 0));
    int r = 0;
    if (m.useGraph && nb == m.maxBatch && m.tev.empty()) {
        // the graph holds the launch shapes; a batch whose resize tiles are larger needs a new one
        // (and launches only the windows' CTAs: a batch whose windows reach beyond them too)
        bool fits = m.graph[s] != nullptr && m.graphKs[s].size() == ks.size();
        for (size_t i = 0; fits && i < ks.size(); i++) {
            const KernelDesc &a = ks[i], &g = m.graphKs[s][i];
            if (a.kind == K_RESIZE &&
                (a.rs.tile_or > g.rs.tile_or || a.rs.tile_oc > g.rs.tile_oc || a.rs.ixStart < g.rs.ixStart ||
                 a.rs.ixEnd > g.rs.ixEnd || a.rs.izStart < g.rs.izStart || a.rs.izEnd > g.rs.izEnd))
                fits = false;
            if (a.kind == K_LINE && a.line.zwin && (a.line.zl0 < g.line.zl0 || a.line.zl1 > g.line.zl1)) fits = false;
        }
        if (!fits) {
            // the new graph's shapes cover this batch, the graph it replaces (so that the windows
            // grow to what the electrons' distribution needs in a few captures; an instantiation
            // costs milliseconds of host time) and headroom for other batches: larger tiles,
            // windows wider by a quarter of theirs (every CTA launched outside an electron's window
            // costs a little)
            std::vector<KernelDesc> cap = ks;
            if (m.graph[s] && m.graphKs[s].size() == cap.size())
                for (size_t i = 0; i < cap.size(); i++) {
                    const KernelDesc& o = m.graphKs[s][i];
                    if (cap[i].kind == K_RESIZE) {
                        ResizeDesc& r = cap[i].rs;
                        r.tile_or = std::max(r.tile_or, o.rs.tile_or);
                        r.tile_oc = std::max(r.tile_oc, o.rs.tile_oc);
                        r.ixStart = std::min(r.ixStart, o.rs.ixStart);
                        r.ixEnd = std::max(r.ixEnd, o.rs.ixEnd);
                        r.izStart = std::min(r.izStart, o.rs.izStart);
                        r.izEnd = std::max(r.izEnd, o.rs.izEnd);
                    } else if (cap[i].kind == K_LINE && cap[i].line.zwin) {
                        cap[i].line.zl0 = std::min(cap[i].line.zl0, o.line.zl0);
                        cap[i].line.zl1 = std::max(cap[i].line.zl1, o.line.zl1);
                    }
                }
            if (m.graph[s]) { cudaGraphExecDestroy(m.graph[s]); m.graph[s] = nullptr; }
            for (size_t i = 0; i < cap.size(); i++) {
                if (cap[i].kind == K_RESIZE && cap[i].rs.tile_or > 0) {
                    ResizeDesc& r = cap[i].rs;
                    r.tile_or = std::min(SRWG_RESIZE_OR_MAX, r.tile_or + 2);
                    r.tile_oc = std::min(SRWG_RESIZE_OC_MAX, r.tile_oc + 2);
                    const long mx = std::max(2L * SRWG_RESIZE_TX, (r.ixEnd - r.ixStart) / 4);
                    const long mz = std::max(2L * SRWG_RESIZE_TZ, (r.izEnd - r.izStart) / 4);
                    r.ixStart = std::max(0L, r.ixStart - mx);
                    r.ixEnd = std::min((long)r.nxn - 1, r.ixEnd + mx);
                    r.izStart = std::max(0L, r.izStart - mz);
                    r.izEnd = std::min((long)r.nzn - 1, r.izEnd + mz);
                }
                if (cap[i].kind == K_LINE && cap[i].line.zwin) {
                    LineDesc& d = cap[i].line;
                    const int nl = d.axis == 0 ? d.nz : d.nx;
                    const int ml = std::max(64, (d.zl1 - d.zl0) / 4);
                    d.zl0 = std::max(0, d.zl0 - ml);
                    d.zl1 = std::min(nl - 1, d.zl1 + ml);
                }
            }
            // this batch runs directly (which also creates every lazily made resource -- twiddle
            // tables, kernel attributes -- before the capture); the capture only records the launches
            r = run_batch(m, nb, cap, st, s);
            if (r) return r;
            cudaGraph_t g;
            MTRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            r = run_batch(m, nb, cap, st, s);
            cudaError_t e = cudaStreamEndCapture(st, &g);
            if (r) return r;
            MTRY(e);
            MTRY(cudaGraphInstantiate(&m.graph[s], g, 0));
            cudaGraphDestroy(g);
            m.graphKs[s] = cap;
        } else {
            MTRY(cudaGraphLaunch(m.graph[s], st));
        }
    } else {
        r = run_batch(m, nb, ks, st, s);
        if (r) return r;
    }
    MTRY(cudaEventRecord(m.used[s], st));
    m.nAdded += nb;
    m.slot ^= 1;
    m.upTo = 0;
    m.upWaited = false;
    MTRY(cudaEventSynchronize(m.staged[m.slot]));
    return 0;
}

}  // namespace srwg

extern "C" SRWG_API int srwgMultiECreate(const SRWLWfr* pBase, const SRWLOptC* pOpt, const SRWLRadMesh* pAccMesh,
                                         int maxBatch, int useGraph, int device, srwgMultiE** out)
{
    std::lock_guard<std::mutex> lk(library_mutex());
    set_last_detail("");
    if (!pBase || !pOpt || !pAccMesh || !out || maxBatch < 1 || !pBase->arEx || !pBase->arEy) return SRWG_ERR_BAD_ARG;
    if (pBase->mesh.ne != 1 || pBase->mesh.nx < 2 || pBase->mesh.ny < 2 || pAccMesh->nx < 2 || pAccMesh->ny < 2)
        return SRWG_ERR_BAD_ARG;
    srwgMultiE* m = new srwgMultiE();
    DeviceCtx* c = nullptr;
    int r = device_ctx(device, &c);
    if (r) { delete m; return r; }
    m->device = device;
    m->ctx = c;
    m->base = *pBase;
    m->momX.assign(11, 0.);
    m->momY.assign(11, 0.);
    if (pBase->arMomX) for (int i = 0; i < 11; i++) m->momX[i] = pBase->arMomX[i];
    if (pBase->arMomY) for (int i = 0; i < 11; i++) m->momY[i] = pBase->arMomY[i];
    m->opt = pOpt;
    m->nx = (int)pBase->mesh.nx;
    m->nz = (int)pBase->mesh.ny;
    m->xStart = pBase->mesh.xStart;
    m->xStep = (pBase->mesh.xFin - pBase->mesh.xStart) / (m->nx - 1);
    m->zStart = pBase->mesh.yStart;
    m->zStep = (pBase->mesh.yFin - pBase->mesh.yStart) / (m->nz - 1);
    m->eStart = pBase->mesh.eStart;
    m->anx = (int)pAccMesh->nx;
    m->anz = (int)pAccMesh->ny;
    m->axStart = pAccMesh->xStart;
    m->axStep = (pAccMesh->xFin - pAccMesh->xStart) / (m->anx - 1);
    m->azStart = pAccMesh->yStart;
    m->azStep = (pAccMesh->yFin - pAccMesh->yStart) / (m->anz - 1);
    m->maxBatch = maxBatch;
    m->useGraph = useGraph != 0;
    // sizes from the unshifted electron's plan
    Planner pl;
    pl.numMoments = false;               // only the intensity is kept: no moment passes
    pl.inPhase = true;                   // the electrons' kick (here zero): the same passes as theirs
    r = pl.plan(pBase, pOpt);
    if (!r) mark_intensity_pass(pl.kernels, pl.tables);
    if (r) { set_last_detail(pl.err); delete m; return r; }
    m->nIn = (size_t)m->nx * m->nz;
    m->nOut = (size_t)pl.w.nx * pl.w.nz;
    m->perWork = (size_t)std::max<long long>(pl.maxElems, 1);
    const size_t tabBytes = ((pl.tables.size() * sizeof(float2) + 255) & ~(size_t)255) + 4096;   // slack for alignment pads
    m->descOff = tabBytes;
    m->constStride = (tabBytes + pl.kernels.size() * sizeof(KernelDesc) + 255) & ~(size_t)255;
#define MALLOC(p, n)                                                                 \
    do {                                                                             \
        cudaError_t e__ = cudaMalloc(&(p), (n));                                     \
        if (e__ != cudaSuccess) {                                                    \
            set_last_detail(std::string("cudaMalloc: ") + cudaGetErrorString(e__));  \
            delete m;                                                                \
            return MEMORY_ALLOCATION_FAILURE;                                        \
        }                                                                            \
    } while (0)
    const size_t B = (size_t)maxBatch;
    MALLOC(m->dBase, 2 * m->nIn * sizeof(float2));
    MALLOC(m->dOut, 2 * B * m->nOut * sizeof(float2));
    MALLOC(m->dWork, 4 * B * m->perWork * sizeof(float2));
    for (int i = 0; i < 2; i++) {
        MALLOC(m->dConst[i], B * m->constStride);
        MALLOC(m->dParams[i], B * sizeof(ElecParams));
    }
    MALLOC(m->dAcc, (size_t)m->anx * m->anz * sizeof(double));
    MALLOC(m->dSnap, (size_t)m->anx * m->anz * sizeof(double));
#undef MALLOC
    for (int i = 0; i < 2; i++) {
        if (cudaMallocHost(&m->hConst[i], B * m->constStride) != cudaSuccess ||
            cudaMallocHost(&m->hParams[i], B * sizeof(ElecParams)) != cudaSuccess ||
            cudaEventCreateWithFlags(&m->staged[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&m->used[i], cudaEventDisableTiming) != cudaSuccess) {
            set_last_detail("pinned staging buffers could not be allocated");
            delete m;
            return MEMORY_ALLOCATION_FAILURE;
        }
        cudaEventRecord(m->staged[i], 0);
        cudaEventRecord(m->used[i], 0);
    }
    if (cudaStreamCreateWithFlags(&m->copy, cudaStreamNonBlocking) != cudaSuccess) {
        set_last_detail("upload stream could not be created");
        delete m;
        return SRWG_ERR_CUDA;
    }
    if (cudaMemcpy(m->dBase, pBase->arEx, m->nIn * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->dBase + m->nIn, pBase->arEy, m->nIn * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(m->dAcc, 0, (size_t)m->anx * m->anz * sizeof(double)) != cudaSuccess) {
        set_last_detail("base field upload failed");
        delete m;
        return SRWG_ERR_CUDA;
    }
    m->base.arEx = nullptr;           // the host arrays are not kept
    m->base.arEy = nullptr;
    *out = m;
    return 0;
}

static int add_impl(srwgMultiE* m, int n, const double* arOffsets, int stride, void* stream);

extern "C" SRWG_API int srwgMultiEAdd(srwgMultiE* m, int n, const double* arOffsets, void* stream)
{
    return add_impl(m, n, arOffsets, 4, stream);
}

extern "C" SRWG_API int srwgMultiEAddE(srwgMultiE* m, int n, const double* arOffsets, void* stream)
{
    return add_impl(m, n, arOffsets, 5, stream);
}

static int add_body(srwgMultiE* m, int n, const double* arOffsets, int stride, cudaStream_t st);

// one batch (1 <= n <= maxBatch electrons of one pass structure) added without the graph, with CUDA
// events around every pass and the accumulation; passMs[i] = the device time of pass i, the last
// value the accumulation's.  The electrons are added as by srwgMultiEAdd(E).
extern "C" SRWG_API int srwgMultiEAddTimed(srwgMultiE* m, int n, const double* arOffsets, int stride, void* stream,
                                           float* passMs, int maxPasses, int* nPasses)
{
    if (!m || n < 1 || n > m->maxBatch || !arOffsets || (stride != 4 && stride != 5) || !passMs || maxPasses < 1)
        return SRWG_ERR_BAD_ARG;
    int r = 0;
    {
        std::lock_guard<std::mutex> lk(library_mutex());
        Planner pl;
        pl.numMoments = false;
        pl.inPhase = true;
        r = pl.plan(&m->base, m->opt);
        if (r) { set_last_detail(pl.err); return r; }
        const size_t ne = 2 * pl.kernels.size() + 2;
        for (cudaEvent_t e : m->tev) cudaEventDestroy(e);
        m->tev.assign(ne, nullptr);
        for (size_t i = 0; i < ne; i++) MTRY(cudaEventCreate(&m->tev[i]));
    }
    const long long n0 = m->nAdded, f0 = m->nFlush;
    r = add_impl(m, n, arOffsets, stride, stream);
    std::lock_guard<std::mutex> lk(library_mutex());
    if (r == 0 && (m->nAdded - n0 != n || m->nFlush - f0 != 1)) {
        set_last_detail("timed add: the electrons did not run as one batch");
        r = SRWG_ERR_BAD_ARG;
    }
    const int np = (int)(m->tev.size() / 2);
    if (r == 0) {
        DeviceCtx* c = nullptr;
        r = device_ctx(m->device, &c);
        if (r == 0 && cudaStreamSynchronize(stream ? (cudaStream_t)stream : c->stream) != cudaSuccess) r = SRWG_ERR_CUDA;
        for (int i = 0; r == 0 && i < np && i < maxPasses; i++) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, m->tev[2 * i], m->tev[2 * i + 1]) != cudaSuccess) r = SRWG_ERR_CUDA;
            passMs[i] = ms;
        }
        if (nPasses) *nPasses = np;
    }
    for (cudaEvent_t e : m->tev) cudaEventDestroy(e);
    m->tev.clear();
    return r;
}

// A call either adds all its electrons or none: the accumulator is copied aside first, and on an
// error (an electron whose passes differ in size from the base wavefront's, a failed launch) the
// batches already added are taken out again by restoring that copy and the electron count.
static int add_impl(srwgMultiE* m, int n, const double* arOffsets, int stride, void* stream)
{
    std::lock_guard<std::mutex> lk(library_mutex());
    set_last_detail("");
    if (!m || n < 0 || (n > 0 && !arOffsets)) return SRWG_ERR_BAD_ARG;
    DeviceCtx* c = nullptr;
    int r = device_ctx(m->device, &c);
    if (r) return r;
    // the library's own stream when none is given (stream capture needs a non-default stream)
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    if (n == 0) return 0;
    const size_t accBytes = (size_t)m->anx * m->anz * sizeof(double);
    MTRY(cudaMemcpyAsync(m->dSnap, m->dAcc, accBytes, cudaMemcpyDeviceToDevice, st));
    const long long n0 = m->nAdded;
    r = add_body(m, n, arOffsets, stride, st);
    if (r) {
        const std::string why = last_detail();
        cudaMemcpyAsync(m->dAcc, m->dSnap, accBytes, cudaMemcpyDeviceToDevice, st);
        cudaStreamSynchronize(st);
        m->nAdded = n0;
        set_last_detail(why);
        return r;
    }
    if (!stream) MTRY(cudaStreamSynchronize(st));
    return 0;
}

static int add_body(srwgMultiE* m, int n, const double* arOffsets, int stride, cudaStream_t st)
{
    int r = 0;
    m->upTo = 0;                          // a batch abandoned by an error left nothing to keep
    m->upWaited = false;
    std::vector<KernelDesc> first, launchKs;
    int nb = 0;
    // electrons are planned on host threads a group at a time (the planner keeps no shared state);
    // the GPU runs the previous batches meanwhile
    const int group = std::max(m->maxBatch, 16);
    if (!m->pool) m->pool.reset(new WorkerPool((int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()))));
    const int nthr = m->pool->size();
    std::vector<Planner> pls(group);
    std::vector<ElecParams> eps(group);
    std::vector<int> rcs(group);
    // the electrons' tables and descriptors are copied into the pinned staging slot by the host
    // threads too (≈130 KB per electron at 1536 x 1600: one thread would take about as long as the
    // GPU takes for the batch): (electron of the group, position in the batch), copied before the
    // batch is flushed or the group is planned again
    std::vector<std::pair<int, int>> pending;
    auto copy_pending = [&]() {
        if (pending.empty()) return;
        char* base = m->hConst[m->slot];
        auto cp = [&](int t0) {
            for (size_t i = t0; i < pending.size(); i += nthr) {
                const Planner& q = pls[pending[i].first];
                char* blk = base + (size_t)pending[i].second * m->constStride;
                memcpy(blk, q.tables.data(), q.tables.size() * sizeof(float2));
                memcpy(blk + m->descOff, q.kernels.data(), q.kernels.size() * sizeof(KernelDesc));
            }
        };
        m->pool->run(std::min(nthr, (int)pending.size()), cp);
        pending.clear();
    };
    for (int e = 0; e < n; e++) {
        const int g = e % group;
        if (g == 0) {
            copy_pending();
            if (nb > 0) {
                r = upload_staged(*m, nb);
                if (r) return r;
            }
            const int cnt = std::min(group, n - e);
            auto work = [&](int t0) {
                double momX[11], momY[11];
                for (int k = t0; k < cnt; k += nthr) {
                    SRWLWfr w;
                    memset(&eps[k], 0, sizeof(ElecParams));
                    electron_wfr(*m, arOffsets + (size_t)stride * (e + k), stride, w, momX, momY, eps[k]);
                    pls[k] = Planner();
                    pls[k].numMoments = false;
                    // the kick kx (x - dx) + kz (z - dz) on the electron's (shifted) mesh
                    pls[k].inPhase = true;
                    pls[k].inKx = eps[k].kx;
                    pls[k].inKz = eps[k].kz;
                    pls[k].inC = -(eps[k].kx * eps[k].dx + eps[k].kz * eps[k].dz);
                    rcs[k] = pls[k].plan(&w, m->opt);
                    if (!rcs[k]) mark_intensity_pass(pls[k].kernels, pls[k].tables);
                }
            };
            m->pool->run(std::min(nthr, cnt), work);
        }
        Planner& pl = pls[g];
        ElecParams& ep = eps[g];
        r = rcs[g];
        if (r) { set_last_detail(pl.err); return r; }
        const size_t tb = pl.tables.size() * sizeof(float2);
        if ((size_t)pl.w.nx * pl.w.nz != m->nOut || (size_t)pl.maxElems > m->perWork || tb > m->descOff ||
            m->descOff + pl.kernels.size() * sizeof(KernelDesc) > m->constStride) {
            set_last_detail("electron " + std::to_string(e) + ": its passes differ in size from the base wavefront's");
            return SRWG_ERR_UNSUPPORTED;
        }
        if (nb > 0 && (!same_structure(first, pl.kernels) || nb == m->maxBatch)) {
            copy_pending();
            r = flush(*m, nb, launchKs, st);
            if (r) return r;
            nb = 0;
        }
        if (nb == 0) { first = pl.kernels; launchKs = pl.kernels; }
        // launch shapes of the batch: the largest resize tiles and the union of the windows (the
        // kernels read every electron's own descriptor)
        for (size_t i = 0; i < launchKs.size(); i++)
            if (launchKs[i].kind == K_RESIZE) {
                ResizeDesc &a = launchKs[i].rs;
                const ResizeDesc& b = pl.kernels[i].rs;
                a.tile_or = std::max(a.tile_or, b.tile_or);
                a.tile_oc = std::max(a.tile_oc, b.tile_oc);
                a.ixStart = std::min(a.ixStart, b.ixStart);
                a.ixEnd = std::max(a.ixEnd, b.ixEnd);
                a.izStart = std::min(a.izStart, b.izStart);
                a.izEnd = std::max(a.izEnd, b.izEnd);
            } else if (launchKs[i].kind == K_LINE && launchKs[i].line.zwin) {
                launchKs[i].line.zl0 = std::min(launchKs[i].line.zl0, pl.kernels[i].line.zl0);
                launchKs[i].line.zl1 = std::max(launchKs[i].line.zl1, pl.kernels[i].line.zl1);
            }
        pending.emplace_back(g, nb);
        // output mesh as the reference's SRWLWfr holds it, step re-derived from (Fin - Start)/(n - 1)
        const double xFin = pl.w.xStart + pl.w.xStep * (pl.w.nx - 1);
        const double zFin = pl.w.zStart + pl.w.zStep * (pl.w.nz - 1);
        ep.oxStart = pl.w.xStart;
        ep.oxStep = (xFin - pl.w.xStart) / (pl.w.nx - 1);
        ep.ozStart = pl.w.zStart;
        ep.ozStep = (zFin - pl.w.zStart) / (pl.w.nz - 1);
        ep.oxInv = 1. / ep.oxStep;
        ep.ozInv = 1. / ep.ozStep;
        ep.onx = pl.w.nx;
        ep.onz = pl.w.nz;
        m->hParams[m->slot][nb] = ep;
        nb++;
    }
    copy_pending();
    return flush(*m, nb, launchKs, st);
}

// passes of a batch, whether the last one writes the intensity instead of the two fields, and the
// planner's description of the passes (the base electron's)
extern "C" SRWG_API int srwgMultiEInfo(srwgMultiE* m, int* nPasses, int* intensityPass, char* desc, int descLen)
{
    std::lock_guard<std::mutex> lk(library_mutex());
    if (!m) return SRWG_ERR_BAD_ARG;
    Planner pl;
    pl.numMoments = false;
    pl.inPhase = true;
    int r = pl.plan(&m->base, m->opt);
    if (r) { set_last_detail(pl.err); return r; }
    mark_intensity_pass(pl.kernels, pl.tables);
    if (nPasses) *nPasses = (int)pl.kernels.size();
    if (intensityPass) *intensityPass = intensity_pass(pl.kernels) ? 1 : 0;
    if (desc && descLen > 0) {
        const std::string s = pl.describe();
        strncpy(desc, s.c_str(), descLen - 1);
        desc[descLen - 1] = 0;
    }
    return 0;
}

extern "C" SRWG_API int srwgMultiEGetMean(srwgMultiE* m, double* arMean, long long* nElec, void* stream)
{
    std::lock_guard<std::mutex> lk(library_mutex());
    if (!m) return SRWG_ERR_BAD_ARG;
    if (nElec) *nElec = m->nAdded;
    if (!arMean) return 0;
    DeviceCtx* c = nullptr;
    int r = device_ctx(m->device, &c);
    if (r) return r;
    const size_t na = (size_t)m->anx * m->anz;
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    MTRY(cudaMemcpyAsync(arMean, m->dAcc, na * sizeof(double), cudaMemcpyDeviceToHost, st));
    MTRY(cudaStreamSynchronize(st));
    if (m->nAdded > 0)
        for (size_t i = 0; i < na; i++) arMean[i] /= (double)m->nAdded;
    return 0;
}

extern "C" SRWG_API int srwgMultiEAccumulator(srwgMultiE* m, double** dAcc, long long* nElec)
{
    if (!m || !dAcc) return SRWG_ERR_BAD_ARG;
    *dAcc = m->dAcc;
    if (nElec) *nElec = m->nAdded;
    return 0;
}

extern "C" SRWG_API int srwgMultiESetAccumulator(srwgMultiE* m, double* dAcc)
{
    std::lock_guard<std::mutex> lk(library_mutex());
    if (!m || !dAcc) return SRWG_ERR_BAD_ARG;
    if (!m->ownAcc) return SRWG_ERR_BAD_ARG;
    cudaFree(m->dAcc);
    m->dAcc = dAcc;
    m->ownAcc = false;
    for (int i = 0; i < 2; i++)              // captured launches name the old accumulator
        if (m->graph[i]) {
            cudaGraphExecDestroy(m->graph[i]);
            m->graph[i] = nullptr;
            m->graphKs[i].clear();
        }
    return 0;
}

extern "C" SRWG_API int srwgMultiEReset(srwgMultiE* m, void* stream)
{
    std::lock_guard<std::mutex> lk(library_mutex());
    if (!m) return SRWG_ERR_BAD_ARG;
    DeviceCtx* c = nullptr;
    int r = device_ctx(m->device, &c);
    if (r) return r;
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    MTRY(cudaMemsetAsync(m->dAcc, 0, (size_t)m->anx * m->anz * sizeof(double), st));
    if (!stream) MTRY(cudaStreamSynchronize(st));
    m->nAdded = 0;
    return 0;
}

extern "C" SRWG_API int srwgMultiEDestroy(srwgMultiE* m)
{
    std::lock_guard<std::mutex> lk(library_mutex());
    if (m) {
        DeviceCtx* c = nullptr;
        device_ctx(m->device, &c);
        delete m;
    }
    return 0;
}
