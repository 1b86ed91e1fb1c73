// MOM passes: the statistical moments of a field, srTGenOptElem::ComputeRadMoments
// (cpp/src/core/sroptelm.cpp:1608-2092) for the coordinate representation and ne == 1, as
// bandwidth-bound reductions over the field in device memory.
//
//   1. rows:    per-row sums of the FP32 intensity (the field after the pass's point-wise work:
//               operators still pending on it, and the removal of the wavefront's quadratic phase)
//   2. limits:  the total power and the rows holding 90 % of it (FindIntensityLimitsInds,
//               srmatsta.cpp:572, with FindIntensityLimits2D :452 and FindLimit1DLeft/Right :400-450)
//   3. columns: per-column sums over those rows, in row segments, then their totals
//   4. limits:  the columns holding 90 % of the power, the reference's FP32 round trip of the
//               limits into mesh indices
//   5. sums:    the 22 weighted sums (norms, first moments, second moments inside the limits, and the
//               angular moments from finite differences along x and z), per CTA
//   6. final:   the per-CTA sums added into the result slot
// All sums are FP64 in a fixed order (no atomics): the result does not depend on scheduling.  The
// host normalises the sums into moments (planner.cpp, moments_from_sums).
#include <cuda_runtime.h>
#include <climits>

#include "common.cuh"
#include "kernels.h"

namespace srwg {

#define MOM_T 256          // threads per CTA of the row / column / sum kernels
#define MOM_R5 8           // rows per CTA of the sum kernel
#define MOM_LT 1024        // threads of the limit kernels (one CTA)

struct MomArgs {
    const MomDesc* d;
    const float2* s0;
    const float2* s1;
    const float2* tabs;
    double* sc;            // scratch: rows | column segments | per-CTA sums | limits
    double* out;           // result slot
    int S, RS;             // column segments and rows per segment
    long long offCol, offPart, offLim;
};

static int mom_segments(int nx, int nz)
{
    const int cx = (nx + MOM_T - 1) / MOM_T;
    int S = (4 * 148 + cx - 1) / cx;     // about four CTAs per SM
    if (S > 256) S = 256;
    if (S > nz) S = nz;
    return S < 1 ? 1 : S;
}

static long long up32(long long v) { return (v + 31) & ~31LL; }

static void mom_layout(int nx, int nz, long long& offCol, long long& offPart, long long& offLim, long long& total)
{
    const long long S = mom_segments(nx, nz);
    const long long n5 = (long long)((nx + MOM_T - 1) / MOM_T) * ((nz + MOM_R5 - 1) / MOM_R5);
    offCol = up32(nz);
    offPart = offCol + up32(S * nx);
    offLim = offPart + up32(n5 * 22);
    total = offLim + 32;
}

size_t mom_scratch_doubles(int nx, int nz)
{
    long long a, b, c, t;
    mom_layout(nx, nz, a, b, c, t);
    return (size_t)t;
}

// the pass's point-wise factor at (ix, iz): separable tables and masks
__device__ __forceinline__ float2 mom_factor(const MomDesc& d, const float2* tabs, long long tx, long long tz, int ix,
                                             int iz)
{
    float2 f = make_float2(1.f, 0.f);
    if (tx >= 0) f = __ldg(&tabs[tx + ix]);
    if (tz >= 0) f = cmul(f, __ldg(&tabs[tz + iz]));
    if (d.has_extra) {
        bool zero = false;
        extra_eval(d.extra, ix, iz, f, zero, tabs);
        if (zero) f = make_float2(0.f, 0.f);
    }
    return f;
}

struct MomField {
    const MomDesc* d;
    const float2* s0;
    const float2* s1;
    const float2* tabs;
    long long tx, tz;
    int nx;
    __device__ __forceinline__ void load(int ix, int iz, float2& ex, float2& ey) const
    {
        const size_t o = (size_t)iz * nx + ix;
        const float2 f = mom_factor(*d, tabs, tx, tz, ix, iz);
        ex = cmul(f, __ldg(&s0[o]));
        ey = cmul(f, __ldg(&s1[o]));
    }
};

__device__ __forceinline__ MomField mom_field(const MomArgs& a)
{
    MomField F;
    F.d = a.d; F.s0 = a.s0; F.s1 = a.s1; F.tabs = a.tabs;
    F.tx = a.d->t.tab; F.tz = a.d->t.ltab; F.nx = a.d->nx;
    return F;
}

// total intensity (polarisation 6) of one point, FP32 as the reference extracts it (srradmnp.h:372)
__device__ __forceinline__ float mom_int(float2 ex, float2 ey)
{
    const double v = (double)ex.x * ex.x + (double)ex.y * ex.y + (double)ey.x * ey.x + (double)ey.y * ey.y;
    return (float)v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// 1. per-row intensity sums, one CTA per row (warp sums, then the CTA's in warp order)
__global__ void __launch_bounds__(MOM_T) mom_rows_kernel(const MomArgs a)
{
    __shared__ double ws[MOM_T / 32];
    const MomField F = mom_field(a);
    const int iz = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double s = 0.;
    for (int ix = threadIdx.x; ix < F.nx; ix += MOM_T) {
        float2 ex, ey;
        F.load(ix, iz, ex, ey);
        s += (double)mom_int(ex, ey);
    }
    s = warp_sum(s);
    if (lane == 0) ws[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.;
        for (int w = 0; w < MOM_T / 32; w++) t += ws[w];
        a.sc[iz] = t;
    }
}

// first index where the running sum of v(0..n-1) exceeds `stop` (0 if none; `left`), or the last
// index where the running sum from the right does (n - 1 if none); one CTA of MOM_LT threads.
template <class V>
__device__ int mom_find_limit(const V& v, int n, double stop, bool left, double* sh, int* ish)
{
    const int t = threadIdx.x;
    const int C = (n + MOM_LT - 1) / MOM_LT;
    const int lo = t * C < n ? t * C : n, hi = lo + C < n ? lo + C : n;
    double cs = 0.;
    for (int i = lo; i < hi; i++) cs += v(i);
    // inclusive scan of the chunk sums (Hillis-Steele)
    sh[t] = cs;
    __syncthreads();
    for (int o = 1; o < MOM_LT; o <<= 1) {
        const double add = t >= o ? sh[t - o] : 0.;
        __syncthreads();
        sh[t] += add;
        __syncthreads();
    }
    const double incl = sh[t], total = sh[MOM_LT - 1];
    if (t == 0) *ish = left ? INT_MAX : -1;
    __syncthreads();
    int cand = left ? INT_MAX : -1;
    if (left) {
        double run = incl - cs;
        for (int i = lo; i < hi; i++) {
            run += v(i);
            if (run > stop) { cand = i; break; }
        }
        if (cand != INT_MAX) atomicMin(ish, cand);
    } else {
        double run = total - incl;
        for (int i = hi - 1; i >= lo; i--) {
            run += v(i);
            if (run > stop) { cand = i; break; }
        }
        if (cand >= 0) atomicMax(ish, cand);
    }
    __syncthreads();
    int r = *ish;
    __syncthreads();
    if (left) return r == INT_MAX ? 0 : r;
    return r < 0 ? n - 1 : r;
}

struct RowVals {
    const double* r; double step; int ok;
    __device__ double operator()(int i) const { return ok ? step * r[i] : 0.; }
};
struct ColVals {
    const double* c; double step;
    __device__ double operator()(int i) const { return step * c[i]; }
};
struct Plain {
    const double* r;
    __device__ double operator()(int i) const { return r[i]; }
};

__device__ __forceinline__ double block_sum(double v, double* sh)
{
    const int t = threadIdx.x;
    v = warp_sum(v);
    __syncthreads();
    if ((t & 31) == 0) sh[t >> 5] = v;
    __syncthreads();
    double s = 0.;
    for (int w = 0; w < MOM_LT / 32; w++) s += sh[w];
    __syncthreads();
    return s;
}

// 2. / 4. power limits (phase 0: rows, phase 1: columns and the final mesh indices)
__global__ void __launch_bounds__(MOM_LT) mom_limits_kernel(const MomArgs a, int phase)
{
    __shared__ double sh[MOM_LT];
    __shared__ int ish;
    const MomDesc& d = *a.d;
    const int nx = d.nx, nz = d.nz, t = threadIdx.x;
    double* lim = a.sc + a.offLim;
    if (phase == 0) {
        // IntegrateSimple over the whole mesh, rounded to FP32 (TotPower), and the stop level
        double s = 0.;
        for (int i = t; i < nz; i += MOM_LT) s += a.sc[i];
        s = block_sum(s, sh);
        const double tot = (double)(float)((s * d.xStep) * d.zStep);
        const double stop = (tot * (1. - 0.9)) * 0.25;
        int ok = (nx >= 2 && nz >= 2) ? 1 : 0;        // IntegrateOverX needs ixStart < ixEnd
        const RowVals rv{a.sc, d.xStep, 1};
        int iy0 = 0, iy1 = nz - 1;
        if (ok) {
            iy0 = mom_find_limit(rv, nz, stop / d.zStep, true, sh, &ish);
            iy1 = mom_find_limit(rv, nz, stop / d.zStep, false, sh, &ish);
            if (iy1 <= iy0) ok = 0;
        }
        if (t == 0) { lim[0] = iy0; lim[1] = iy1; lim[2] = ok; lim[3] = stop; }
        return;
    }
    const int ok = (int)lim[2];
    int L0 = 0, L1 = nx - 1, L2 = 0, L3 = nz - 1;
    if (ok) {
        const int iy0 = (int)lim[0], iy1 = (int)lim[1];
        const double stop = lim[3];
        const double* col = a.sc + a.offCol;       // column totals (mom_colsum_kernel)
        const ColVals cv{col, d.zStep};
        const int ix0 = mom_find_limit(cv, nx, stop / d.xStep, true, sh, &ish);
        const int ix1 = mom_find_limit(cv, nx, stop / d.xStep, false, sh, &ish);
        // the limits as FP32 coordinates, back to indices (srmatsta.cpp:610-617)
        const float f1 = (float)(d.xStart + d.xStep * ix0), f2 = (float)(d.xStart + d.xStep * ix1);
        const float f3 = (float)(d.zStart + d.zStep * iy0), f4 = (float)(d.zStart + d.zStep * iy1);
        L0 = (int)((((double)f1 - d.xStart) * 1.0000001) / d.xStep);
        if (L0 < 0) L0 = 0;
        L1 = (int)((((double)f2 - d.xStart) * 1.0000001) / d.xStep);
        if (L1 >= nx) L1 = nx - 1;
        L2 = (int)((((double)f3 - d.zStart) * 1.0000001) / d.zStep);
        if (L2 < 0) L2 = 0;
        L3 = (int)((((double)f4 - d.zStart) * 1.0000001) / d.zStep);
        if (L3 >= nz) L3 = nz - 1;
    }
    if (t == 0) {
        lim[4] = L0; lim[5] = L1; lim[6] = L2; lim[7] = L3;
        a.out[22] = L0; a.out[23] = L1; a.out[24] = L2; a.out[25] = L3;
        a.out[26] = ok;
    }
}

// 3. per-column intensity sums over the rows of the power limits, one row segment per grid row
__global__ void __launch_bounds__(MOM_T) mom_cols_kernel(const MomArgs a)
{
    const MomField F = mom_field(a);
    const int nx = F.nx, nz = a.d->nz;
    const int ix = blockIdx.x * MOM_T + threadIdx.x, s = blockIdx.y;
    if (ix >= nx) return;
    const double* lim = a.sc + a.offLim;
    double* col = a.sc + a.offCol + (size_t)s * nx;
    if (!(int)lim[2]) { col[ix] = 0.; return; }
    const int iy0 = (int)lim[0], iy1 = (int)lim[1];
    int r0 = s * a.RS, r1 = (s + 1) * a.RS - 1;
    if (r0 < iy0) r0 = iy0;
    if (r1 > iy1) r1 = iy1;
    if (r1 > nz - 1) r1 = nz - 1;
    double acc = 0.;
    for (int iz = r0; iz <= r1; iz++) {
        float2 ex, ey;
        F.load(ix, iz, ex, ey);
        acc += (double)mom_int(ex, ey);
    }
    col[ix] = acc;
}

// 3b. column totals over the row segments, in place into segment 0: one warp per column, each lane
// adding every 32nd segment, then a shuffle tree (fixed order)
__global__ void __launch_bounds__(MOM_T) mom_colsum_kernel(const MomArgs a)
{
    const int nx = a.d->nx;
    const int c = blockIdx.x * (MOM_T / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (c >= nx) return;
    double* col = a.sc + a.offCol;
    double s = 0.;
    for (int k = lane; k < a.S; k += 32) s += col[(size_t)k * nx + c];
    s = warp_sum(s);
    if (lane == 0) col[c] = s;                  // every lane of this warp has read its segments
}

// the 11 weighted terms of one component at one point (sroptelm.cpp:1770-1906): c the value, l
// its left neighbour (along x), p the one below (along z); wA the weight of all terms, wXp / wZp
// those of the angular terms along x / z
__device__ __forceinline__ void mom_terms(double* acc, float2 c, float2 l, bool hasL, float2 p, bool hasP, double x,
                                          double z, bool in, double ax, double az, double wA, double wXp, double wZp)
{
    const double re = c.x, im = c.y;
    const double n = re * re + im * im;
    const double f1 = x * n, f3 = z * n;
    acc[0] += n * wA;
    acc[1] += f1 * wA;
    acc[3] += f3 * wA;
    if (in) {
        acc[5] += (x * f1) * wA;
        acc[8] += (z * f3) * wA;
    }
    if (hasL) {
        const double dr = re - (double)l.x, di = im - (double)l.y;
        const double cr = di * re - dr * im;
        const double f2 = cr + (ax * x) * n;
        acc[2] += f2 * wXp;
        if (in) {
            acc[6] += (x * f2) * wXp;
            acc[7] += ((dr * dr + di * di) + (cr * ax) * x + (((ax * ax) * x) * x) * n) * wXp;
        }
    }
    if (hasP) {
        const double dr = re - (double)p.x, di = im - (double)p.y;
        const double cr = di * re - dr * im;
        const double f4 = cr + (az * z) * n;
        acc[4] += f4 * wZp;
        if (in) {
            acc[9] += (z * f4) * wZp;
            acc[10] += ((dr * dr + di * di) + (cr * az) * z + (((az * az) * z) * z) * n) * wZp;
        }
    }
}

// 5. the 22 sums over a tile of MOM_T columns x MOM_R5 rows; one thread per column walks the rows
__global__ void __launch_bounds__(MOM_T) mom_sums_kernel(const MomArgs a)
{
    __shared__ double red[MOM_T / 32][22];
    const MomField F = mom_field(a);
    const MomDesc& d = *a.d;
    const int nx = F.nx, nz = d.nz;
    const double xStart = d.xStart, xStep = d.xStep, zStart = d.zStart, zStep = d.zStep, ax = d.ax, az = d.az;
    const double* lim = a.sc + a.offLim;
    const int L0 = (int)lim[4], L1 = (int)lim[5], L2 = (int)lim[6], L3 = (int)lim[7];
    const int ix = blockIdx.x * MOM_T + threadIdx.x;
    const int r0 = blockIdx.y * MOM_R5;
    const int r1 = r0 + MOM_R5 < nz ? r0 + MOM_R5 : nz;
    double acc[22];
#pragma unroll
    for (int k = 0; k < 22; k++) acc[k] = 0.;
    if (ix < nx) {
        const double x = xStart + ix * xStep;
        const double wx = (ix == 0 || ix == nx - 1) ? 0.5 : 1.;
        const double wx1 = ix == 1 ? 0.5 * wx : wx;
        const bool inx = ix >= L0 && ix <= L1, hasL = ix > 0;
        float2 px = make_float2(0.f, 0.f), py = px;
        if (r0 > 0) F.load(ix, r0 - 1, px, py);
        for (int iz = r0; iz < r1; iz++) {
            float2 cx, cy, lx = make_float2(0.f, 0.f), ly = lx;
            F.load(ix, iz, cx, cy);
            if (hasL) F.load(ix - 1, iz, lx, ly);
            const double z = zStart + iz * zStep;
            const double wz = (iz == 0 || iz == nz - 1) ? 0.5 : 1.;
            const double wz1 = iz == 1 ? 0.5 * wz : wz;
            const bool in = inx && iz >= L2 && iz <= L3, hasP = iz > 0;
            mom_terms(acc, cx, lx, hasL, px, hasP, x, z, in, ax, az, wx * wz, wx1 * wz, wx * wz1);
            mom_terms(acc + 11, cy, ly, hasL, py, hasP, x, z, in, ax, az, wx * wz, wx1 * wz, wx * wz1);
            px = cx; py = cy;
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 22; k++) {
        const double v = warp_sum(acc[k]);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 22) {
        double s = 0.;
        for (int w = 0; w < MOM_T / 32; w++) s += red[w][threadIdx.x];
        a.sc[a.offPart + (size_t)(blockIdx.y * gridDim.x + blockIdx.x) * 22 + threadIdx.x] = s;
    }
}

// 6. per-CTA sums into the result slot, one warp per sum
__global__ void __launch_bounds__(22 * 32) mom_final_kernel(const MomArgs a, int n5)
{
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* part = a.sc + a.offPart;
    double s = 0.;
    for (int i = lane; i < n5; i += 32) s += part[(size_t)i * 22 + k];
    s = warp_sum(s);
    if (lane == 0) a.out[k] = s;
}

cudaError_t launch_moments(const MomLaunch& p, cudaStream_t st)
{
    const int nx = p.d.nx, nz = p.d.nz;
    if (nx < 1 || nz < 1) return cudaErrorInvalidValue;
    long long offCol, offPart, offLim, total;
    mom_layout(nx, nz, offCol, offPart, offLim, total);
    const int S = mom_segments(nx, nz);
    const int cx = (nx + MOM_T - 1) / MOM_T, cz5 = (nz + MOM_R5 - 1) / MOM_R5;
    const int nb = p.nb > 1 ? p.nb : 1;
    for (int b = 0; b < nb; b++) {
        MomArgs a;
        a.d = (const MomDesc*)((const char*)p.gd + b * p.bDesc);
        a.s0 = p.src[0] + b * p.bSrc;
        a.s1 = p.src[1] + b * p.bSrc;
        a.tabs = p.tabs + b * p.bTab;
        a.sc = p.scratch;
        a.out = p.out + b * p.bOut;
        a.S = S;
        a.RS = (nz + S - 1) / S;
        a.offCol = offCol; a.offPart = offPart; a.offLim = offLim;
        mom_rows_kernel<<<nz, MOM_T, 0, st>>>(a);
        mom_limits_kernel<<<1, MOM_LT, 0, st>>>(a, 0);
        mom_cols_kernel<<<dim3(cx, S), MOM_T, 0, st>>>(a);
        mom_colsum_kernel<<<(nx + MOM_T / 32 - 1) / (MOM_T / 32), MOM_T, 0, st>>>(a);
        mom_limits_kernel<<<1, MOM_LT, 0, st>>>(a, 1);
        mom_sums_kernel<<<dim3(cx, cz5), MOM_T, 0, st>>>(a);
        mom_final_kernel<<<1, 22 * 32, 0, st>>>(a, cx * cz5);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace srwg
