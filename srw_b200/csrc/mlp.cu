// Kernels of the learned resize-factor predictor: a small FP32 MLP (GEMM, bias + GELU, their
// gradients, mean-squared-error loss, Adam) and the wavefront features it reads (intensity
// downsampled to 64 x 64, fitted phase-curvature radii).  The network is small (a few 10^6
// multiply-adds per wavefront), so these are plain SIMT kernels with shared-memory tiling; the
// training loop and the memory they run on are driven from the host (srw_b200/learned.py).
// Nothing here has a counterpart in the reference: it chooses the resize factors that the
// reference's users set by hand in the propagation parameters (pp[5..8]).
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "../../include/srwl_b200.h"
#include "errors.h"
#include "exec.h"

namespace srwg {

// C[M x N] = alpha * op(A) * op(B) + beta * C; op(A) is M x K (A row-major, lda; transposed when
// transA), op(B) is K x N.  64 x 64 tile per CTA, K in steps of 16, 256 threads x 4 x 4 outputs.
#define GT 64
#define GK 16
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda, int transA,
                                                   const float* __restrict__ B, int ldb, int transB, float* __restrict__ C,
                                                   int ldc, float alpha, float beta)
{
    __shared__ float As[GK][GT + 4];
    __shared__ float Bs[GK][GT + 4];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
    float acc[4][4] = {{0.f}};
    for (int k0 = 0; k0 < K; k0 += GK) {
        // 64 x 16 tile of op(A) and 16 x 64 tile of op(B): 1024 elements each, 4 per thread
        for (int e = threadIdx.x; e < GT * GK; e += 256) {
            const int mm = e / GK, kk = e % GK;                 // A tile element (m0 + mm, k0 + kk)
            const int gm = m0 + mm, gk = k0 + kk;
            float a = 0.f;
            if (gm < M && gk < K) a = transA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
            As[kk][mm] = a;
            const int kb = e / GT, nb = e % GT;                 // B tile element (k0 + kb, n0 + nb)
            const int gkb = k0 + kb, gn = n0 + nb;
            float b = 0.f;
            if (gkb < K && gn < N) b = transB ? B[(size_t)gn * ldb + gkb] : B[(size_t)gkb * ldb + gn];
            Bs[kb][nb] = b;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int gm = m0 + ty * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gn = n0 + tx * 4 + j;
            if (gn >= N) continue;
            float* c = &C[(size_t)gm * ldc + gn];
            *c = alpha * acc[i][j] + (beta != 0.f ? beta * *c : 0.f);
        }
    }
}

__device__ __forceinline__ float gelu(float z)
{   // tanh form of GELU (Hendrycks & Gimpel 2016)
    const float c = 0.7978845608028654f;
    return 0.5f * z * (1.f + tanhf(c * (z + 0.044715f * z * z * z)));
}
__device__ __forceinline__ float gelu_grad(float z)
{
    const float c = 0.7978845608028654f;
    const float u = c * (z + 0.044715f * z * z * z);
    const float t = tanhf(u);
    return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * c * (1.f + 3.f * 0.044715f * z * z);
}

// Z[M x N] += bias (row broadcast); Y = act(Z) with act 0 = identity, 1 = GELU
__global__ void bias_act_kernel(float* __restrict__ Z, const float* __restrict__ bias, float* __restrict__ Y, int M,
                                int N, int act)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)M * N) return;
    const float z = Z[i] + bias[i % N];
    Z[i] = z;
    Y[i] = act ? gelu(z) : z;
}

// dY <- dY * act'(Z)
__global__ void act_backward_kernel(const float* __restrict__ Z, float* __restrict__ dY, size_t n, int act)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !act) return;
    dY[i] *= gelu_grad(Z[i]);
}

// db[N] = sum over rows of dZ[M x N]
__global__ void colsum_kernel(const float* __restrict__ dZ, float* __restrict__ db, int M, int N)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    float s = 0.f;
    for (int i = 0; i < M; i++) s += dZ[(size_t)i * N + j];
    db[j] = s;
}

// mean squared error over M x N: loss (one value, summed in FP64 per block then atomically) and
// dOut = 2 (out - target) / (M N)
__global__ void mse_kernel(const float* __restrict__ out, const float* __restrict__ target, float* __restrict__ dout,
                           double* __restrict__ loss, int n)
{
    __shared__ double red[256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.;
    if (i < n) {
        const float d = out[i] - target[i];
        dout[i] = 2.f * d / (float)n;
        l = (double)d * d / n;
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0]);
}

// Adam (Kingma & Ba 2015) with bias correction, step t >= 1
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// features of one wavefront: total intensity averaged over 64 x 64 cells of the mesh (cell (cy, cx)
// covers rows [cy ny / 64, (cy + 1) ny / 64) and the same for columns), written to feat[64 * 64]
__global__ void downsample_kernel(const float2* __restrict__ ex, const float2* __restrict__ ey, int nx, int ny,
                                  float* __restrict__ feat)
{
    const int cx = blockIdx.x, cy = blockIdx.y;
    const int x0 = (int)((long long)cx * nx / 64), x1 = (int)((long long)(cx + 1) * nx / 64);
    const int y0 = (int)((long long)cy * ny / 64), y1 = (int)((long long)(cy + 1) * ny / 64);
    __shared__ double red[128];
    double s = 0.;
    const int w = x1 - x0, h = y1 - y0;
    for (int e = threadIdx.x; e < w * h; e += blockDim.x) {
        const int y = y0 + e / w, x = x0 + e % w;
        const float2 u = ex[(size_t)y * nx + x], v = ey[(size_t)y * nx + x];
        s += (double)u.x * u.x + (double)u.y * u.y + (double)v.x * v.x + (double)v.y * v.y;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = 64; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) feat[cy * 64 + cx] = (w * h > 0) ? (float)(red[0] / (w * h)) : 0.f;
}

// phase-curvature fit: for neighbouring points along x (and along z) the phase difference
// arg(E(p+1) conj(E(p))) ~ k x dx / R.  The known part 1/R0 (the wavefront's own radius, whose
// quadratic phase the mesh need not resolve) is taken out first, the rest wrapped to [-pi, pi];
// sums for the intensity-weighted least squares 1/R - 1/R0 = sum(w x dphi) / (k dx sum(w x^2))
// (w = |E(p)| |E(p+1)|): sums[0] = sum w x dphi, sums[1] = sum w x^2 (x), sums[2], sums[3] along z
__global__ void curvature_kernel(const float2* __restrict__ ex, int nx, int ny, double xStart, double xStep,
                                 double zStart, double zStep, double k, double invRx0, double invRz0,
                                 double* __restrict__ sums)
{
    const double twoPi = 6.283185307179586;
    __shared__ double red[4][256];
    double a0 = 0., a1 = 0., a2 = 0., a3 = 0.;
    const size_t n = (size_t)nx * ny;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / nx), x = (int)(i % nx);
        const float2 e = ex[i];
        if (x + 1 < nx) {
            const float2 f = ex[i + 1];
            const double re = (double)f.x * e.x + (double)f.y * e.y, im = (double)f.y * e.x - (double)f.x * e.y;
            const double w = sqrt(re * re + im * im);
            const double xm = xStart + (x + 0.5) * xStep;
            double d = atan2(im, re) - k * xm * xStep * invRx0;
            d -= twoPi * rint(d / twoPi);
            a0 += w * xm * d;
            a1 += w * xm * xm;
        }
        if (y + 1 < ny) {
            const float2 f = ex[i + nx];
            const double re = (double)f.x * e.x + (double)f.y * e.y, im = (double)f.y * e.x - (double)f.x * e.y;
            const double w = sqrt(re * re + im * im);
            const double zm = zStart + (y + 0.5) * zStep;
            double d = atan2(im, re) - k * zm * zStep * invRz0;
            d -= twoPi * rint(d / twoPi);
            a2 += w * zm * d;
            a3 += w * zm * zm;
        }
    }
    red[0][threadIdx.x] = a0; red[1][threadIdx.x] = a1; red[2][threadIdx.x] = a2; red[3][threadIdx.x] = a3;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k)
            for (int c = 0; c < 4; c++) red[c][threadIdx.x] += red[c][threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 4; c++) atomicAdd(&sums[c], red[c][0]);
}

}  // namespace srwg

using namespace srwg;

static int launch_status(cudaError_t e)
{
    if (e == cudaSuccess) return 0;
    set_last_detail(std::string("kernel launch: ") + cudaGetErrorString(e));
    return SRWG_ERR_CUDA;
}

extern "C" SRWG_API int srwgMlpGemm(int M, int N, int K, const float* A, int lda, int transA, const float* B, int ldb,
                                    int transB, float* C, int ldc, float alpha, float beta, void* stream)
{
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) return SRWG_ERR_BAD_ARG;
    dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT);
    gemm_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(M, N, K, A, lda, transA, B, ldb, transB, C, ldc, alpha, beta);
    return launch_status(cudaGetLastError());
}

extern "C" SRWG_API int srwgMlpBiasAct(float* Z, const float* bias, float* Y, int M, int N, int act, void* stream)
{
    if (M <= 0 || N <= 0 || !Z || !bias || !Y) return SRWG_ERR_BAD_ARG;
    const size_t n = (size_t)M * N;
    bias_act_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(Z, bias, Y, M, N, act);
    return launch_status(cudaGetLastError());
}

extern "C" SRWG_API int srwgMlpActBackward(const float* Z, float* dY, long long n, int act, void* stream)
{
    if (n <= 0 || !Z || !dY) return SRWG_ERR_BAD_ARG;
    act_backward_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(Z, dY, (size_t)n, act);
    return launch_status(cudaGetLastError());
}

extern "C" SRWG_API int srwgMlpColSum(const float* dZ, float* db, int M, int N, void* stream)
{
    if (M <= 0 || N <= 0 || !dZ || !db) return SRWG_ERR_BAD_ARG;
    colsum_kernel<<<(N + 255) / 256, 256, 0, (cudaStream_t)stream>>>(dZ, db, M, N);
    return launch_status(cudaGetLastError());
}

extern "C" SRWG_API int srwgMlpMse(const float* out, const float* target, float* dout, double* loss, int n, void* stream)
{
    if (n <= 0 || !out || !target || !dout || !loss) return SRWG_ERR_BAD_ARG;
    mse_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(out, target, dout, loss, n);
    return launch_status(cudaGetLastError());
}

extern "C" SRWG_API int srwgMlpAdam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1,
                                    float b2, float eps, int t, void* stream)
{
    if (n <= 0 || !w || !g || !m || !v || t < 1) return SRWG_ERR_BAD_ARG;
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    adam_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, (size_t)n, lr, b1, b2, eps, c1,
                                                                              c2);
    return launch_status(cudaGetLastError());
}

extern "C" SRWG_API int srwgWfrFeatures(const float* dEx, const float* dEy, int nx, int ny, double xStart, double xStep,
                                        double zStart, double zStep, double k, double invRx0, double invRz0,
                                        float* dFeat, double* dSums, void* stream)
{
    if (!dEx || !dEy || nx < 64 || ny < 64 || !dFeat || !dSums) return SRWG_ERR_BAD_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    downsample_kernel<<<dim3(64, 64), 128, 0, st>>>((const float2*)dEx, (const float2*)dEy, nx, ny, dFeat);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(dSums, 0, 4 * sizeof(double), st);
    if (e == cudaSuccess) {
        curvature_kernel<<<296, 256, 0, st>>>((const float2*)dEx, nx, ny, xStart, xStep, zStart, zStep, k, invRx0,
                                              invRz0, dSums);
        e = cudaGetLastError();
    }
    return launch_status(e);
}
