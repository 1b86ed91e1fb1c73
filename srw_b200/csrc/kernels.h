// Launch parameters of the sm_100a kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include "kdesc.h"
#include "linen_lengths.h"

namespace srwg {

// dynamic shared memory of a line pass (leaves room for the static descriptor copy)
#define SRWG_LINE_SMEM_MAX (220 * 1024)

// shared-memory pitch of a line of N points in the line passes: one pad point per 16 (conflict-free
// Stockham exchanges), then rounded up so that the lines of a column tile start 32 / L banks apart
// (a half-warp of a column pass reads 16 / L points of each of L lines, 8 bytes each: together 32
// distinct banks): P = 16 / L modulo 16 points for L = 2, 4, 8, 1 for L >= 16; rows (their lanes
// stay within one line) and L = 1: 4 modulo 16, which keeps every slot 16-byte aligned for the
// bulk copies of row tiles
inline size_t line_pitch(int N, int L = 1, bool cols = false)
{
    const size_t P = (size_t)N + N / 16;
    const size_t r = (cols && L >= 2) ? (L >= 16 ? 1 : 16 / L) : 4;
    return P + ((r + 16 - P % 16) % 16);
}

// lines per CTA of the power-of-two line pass (line2_kernel): rows ~256 threads, columns up to
// 1024 threads (at most 32 columns), within the shared-memory budget; pitch N + N/16 + 4 points.
// (Column tiles of half the width, two CTAs per SM, measured slower: the row pass then writes
// 16-byte pieces per row and column block, and the column pass's stores are half sectors.)
inline int line2_lines_per_cta(int axis, int N)
{
    const int T = N / 16;
    int L = axis == 0 ? 256 / T : 1024 / T;
    if (L < 1) L = 1;
    if (axis == 1 && L > 32) L = 32;
    while (L > 1 && (size_t)L * line_pitch(N, L, axis == 1) * 8 > SRWG_LINE_SMEM_MAX) L--;
    return L;
}

struct LineLaunch {
    LineDesc d;
    const float2* src[2];
    float2* dst[2];
    const float2* tw;        // exp(-2 pi i k / N), k < N (FP64-accurate, rounded to FP32)
    int N, nlines;           // line length, number of lines
    int T, L, P, G;          // threads per line, lines per CTA, shared-memory pitch (float2), thread groups
    int nst;
    int radix[SRWG_MAX_STAGES];
    int v2;                  // 1: power-of-two pass (line2_kernel), 2: general length (lineg_kernel),
                             // 3: specialised general length (linen_kernel)
    const float2* tabs;      // the plan's separable point-wise tables
    const LineDesc* gd;      // this pass's descriptor in device memory
    int nb;                  // wavefronts in the launch (grid z; 0 or 1: one)
    long long bDesc, bTab;   // per wavefront: descriptor stride (bytes), table stride (float2)
    long long bSrc, bDst;    // per wavefront: source / destination field stride (float2)
    int bulk;                // specialised pass: each CTA's input tile arrives by bulk async copies
    int* status;             // device counter of waits that gave up (NULL: not recorded)
    long long spin;          // iteration limit of the bulk-copy wait
    int blk0, nblk;          // the line blocks launched: blk0 .. blk0 + nblk - 1 (nblk 0: all)
};

// tiled resize: a CTA makes TZ x TX new points from an old tile of at most OR_MAX x OC_MAX points
#define SRWG_RESIZE_TX 64
#define SRWG_RESIZE_TZ 16
#define SRWG_RESIZE_OR_MAX 40
#define SRWG_RESIZE_OC_MAX 80

struct ResizeLaunch {
    ResizeDesc d;
    const float2* src[2];
    float2* dst[2];
    const float2* tabs;
    const ResizeDesc* gd;
    int vec_ok;              // even row lengths and 16-byte aligned buffers: float4 paths allowed
    double xStepInvO, zStepInvO;
    int nb;                  // wavefronts in the launch (grid z; 0 or 1: one)
    long long bDesc, bTab;   // per wavefront: descriptor stride (bytes), table stride (float2)
    long long bSrc, bDst;    // per wavefront: source / destination field stride (float2)
    int tx0, tz0, ntx, ntz;  // tiled kernel: the tiles launched (first, count per axis; ntx 0: all)
};

struct PwLaunch {
    PwDesc d;
    const float2* src[2];
    float2* dst[2];
    const float2* tabs;
    const PwDesc* gd;
    int nb;                  // wavefronts in the launch (grid z; 0 or 1: one)
    long long bDesc, bTab;   // per wavefront: descriptor stride (bytes), table stride (float2)
    long long bSrc, bDst;    // per wavefront: source / destination field stride (float2)
};

// MOM pass (moments.cu): reduction of one field into the 22 sums of ComputeRadMoments.  For nb
// wavefronts the passes run one wavefront after the other (scratch reused in stream order).
struct MomLaunch {
    MomDesc d;                 // host copy (launch shapes); the kernels read gd
    const float2* src[2];
    const float2* tabs;
    const MomDesc* gd;
    double* scratch;           // mom_scratch_doubles(nx, nz) doubles
    double* out;               // result slot of wavefront 0 (SRWG_MOM_SLOT doubles)
    int nb;
    long long bDesc, bTab;     // per wavefront: descriptor stride (bytes), table stride (float2)
    long long bSrc, bOut;      // per wavefront: field stride (float2), result stride (doubles)
};
size_t mom_scratch_doubles(int nx, int nz);
cudaError_t launch_moments(const MomLaunch& p, cudaStream_t st);

// intensity extraction from a field with the operators still pending on it (d: host copy, gd: the
// device copy the kernel reads); writes nx * nz values (float, or double for the phase) to out
cudaError_t launch_extract(const MomDesc& d, const MomDesc* gd, const float2* s0, const float2* s1,
                           const float2* tabs, char* out, cudaStream_t st);

cudaError_t launch_line(const LineLaunch& p, cudaStream_t st);

// power-of-two line pass kernels, one translation unit per line length (line2_<logn>.cu)
typedef void (*Line2Fn)(const LineLaunch);
Line2Fn line2_kernel_ptr(int logn, bool cols, bool extra, int f1, int f2);
#define SRWG_LINE2_DECL(L) Line2Fn line2_get_##L(bool cols, int f1, int f2); Line2Fn line2e_get_##L(bool cols, int f1, int f2);
SRWG_LINE2_DECL(6) SRWG_LINE2_DECL(7) SRWG_LINE2_DECL(8) SRWG_LINE2_DECL(9) SRWG_LINE2_DECL(10)
SRWG_LINE2_DECL(11) SRWG_LINE2_DECL(12) SRWG_LINE2_DECL(13) SRWG_LINE2_DECL(14)
// general-length line pass kernels (lineg.cu, lineg_e.cu)
Line2Fn lineg_get(bool cols);
Line2Fn lineg_e_get(bool cols);
// specialised general-length kernels (linen.cu, one unit per length of linen_lengths.h)
#define SRWG_LINEN_DECL(N) Line2Fn linen_get_##N(bool cols, bool extra, int nt, bool inten);
SRWG_LINEN_LENGTHS(SRWG_LINEN_DECL)
SRWG_LINEN_POW2(SRWG_LINEN_DECL)
#undef SRWG_LINEN_DECL
Line2Fn linen_kernel_ptr(int N, bool cols, bool extra, int nt, bool inten = false);
inline bool line2_supported(int N) { return N >= 64 && N <= 16384 && (N & (N - 1)) == 0; }
// general lengths of the specialised kernel
inline bool linen_supported(int N)
{
#define SRWG_LINEN_IS(M) if (N == M) return true;
    SRWG_LINEN_LENGTHS(SRWG_LINEN_IS)
#undef SRWG_LINEN_IS
    return false;
}
// powers of two that the specialised kernel is compiled for as well (the tuner's alternative)
inline bool linen_pow2(int N)
{
#define SRWG_LINEN_IS(M) if (N == M) return true;
    SRWG_LINEN_POW2(SRWG_LINEN_IS)
#undef SRWG_LINEN_IS
    return false;
}
// floats per thread that an intensity pass of the specialised kernel keeps between its two
// components: the last stage's butterflies per thread times its radix (the radix schedule of
// linen.cuh: radix-16 stages, one 8/4/2 stage, then 3, 5, 7; ceil(N/16) threads per line)
__host__ __device__ constexpr int linen_int_floats(int N)
{
    int m = N, p2 = 0;
    while (m % 2 == 0) { m /= 2; p2++; }
    const int R = m % 7 == 0 ? 7 : m % 5 == 0 ? 5 : m % 3 == 0 ? 3 : (p2 % 4 ? 1 << (p2 % 4) : 16);
    const int T = (N + 15) / 16;
    return ((N / R + T - 1) / T) * R;
}
// line-pass kernel families (LineLaunch::v2)
enum { FAM_TAB = 0, FAM_POW2 = 1, FAM_GEN = 2, FAM_SPEC = 3 };
// lines per CTA of the specialised general-length pass (at most 512 threads, 128 registers each):
// rows up to 512 threads, columns a power of two up to 512 threads / 32 columns (the column-block
// width of the row pass before it), within the shared-memory budget; T = ceil(N/16) threads per
// line, pitch N + N/16 + 4 points
inline int linen_lines_per_cta(int axis, int N)
{
    const int T = (N + 15) / 16;
    int L;
    if (axis == 0) {
        L = 512 / T;
        if (L < 1) L = 1;
    } else {
        L = 1;
        while (2 * L * T <= 512 && 2 * L <= 32) L *= 2;
    }
    while (L > 1 && (size_t)L * line_pitch(N, L, axis == 1) * 8 > SRWG_LINE_SMEM_MAX) L = axis == 0 ? L - 1 : L / 2;
    return L;
}
// whether L lines per CTA is a valid launch shape of kernel family fam for length N
inline bool fixed_lines_valid(int axis, int N, int L, int fam)
{
    if (L < 1 || (size_t)L * line_pitch(N, L, axis == 1) * 8 > SRWG_LINE_SMEM_MAX) return false;
    if (axis == 1 && (L > 32 || (L & (L - 1)) != 0)) return false;      // column blocks: a power of two
    if (fam == FAM_POW2 && line2_supported(N)) return (N / 16) * L <= 1024;
    if (fam == FAM_SPEC && (linen_supported(N) || linen_pow2(N))) return ((N + 15) / 16) * L <= 512;
    return false;
}
// kernel family and lines per CTA of the line kernels with compile-time lengths (line2 / linen; they
// skip a zero window and read / write column blocks): the autotuned choice where the tuning table has
// one (capi.cpp), else the power-of-two kernel for powers of two and the specialised one for the
// listed general lengths with the defaults above; lines 0 for other lengths
int fixed_family(int axis, int N);
int fixed_lines_per_cta(int axis, int N);
cudaError_t launch_resize(const ResizeLaunch& p, cudaStream_t st);
cudaError_t launch_pw(const PwLaunch& p, cudaStream_t st);

}  // namespace srwg
