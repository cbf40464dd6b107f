// Post-processing on the GPU, on a velocity field in the vel_print layout
// [nx][ny][zd][3] held in device memory (the moments of the running state, or
// a vel file uploaded by the caller): the quadrant analysis of the
// reference's quadrant-analysis/src/qUADrantA.c and the two-point
// correlations of its 2pt-correlations program (below).
//
// Quadrants.  Per wall-normal fluid plane k = 1 .. zd-2 (one block each): the plane means
// of u, v, w over (x, y); the fluctuations u' = u - <u>, w' = w - <w>; the
// products u'w' summed over the plane and over each quadrant Q1 (u' > 0,
// w' > 0), Q2 (u' < 0, w' > 0), Q3 (u' < 0, w' < 0), Q4 (u' > 0, w' < 0),
// with the cell count of each quadrant (a zero u' or w' falls in none, as in
// the reference).  Sums are FP64 in a fixed order (per-thread strided sums,
// then the deterministic block reduction), so a result does not depend on the
// run; it differs from the reference's sequential sums by rounding only.
#include <cuda_runtime.h>

#include <algorithm>

#include "step_common.cuh"

namespace dnslbm {

constexpr int kQuadThreads = 256;

__global__ void __launch_bounds__(kQuadThreads) vel_plane_means_kernel(const double *__restrict__ vel, int nx, int ny,
                                                                       int zd, double *mean /* [zd][3] */)
{
    __shared__ double smem[32 * 3];
    const int k = blockIdx.x + 1;
    const size_t n = (size_t)nx * ny;
    double s[3] = {0.0, 0.0, 0.0};
    for (size_t c = threadIdx.x; c < n; c += blockDim.x) {  // c = x * ny + y
        const double *v = vel + (c * zd + k) * 3;
        s[0] += v[0];
        s[1] += v[1];
        s[2] += v[2];
    }
    block_sum<3>(s, smem);
    if (threadIdx.x == 0)
        for (int i = 0; i < 3; ++i) mean[k * 3 + i] = s[i] / (double)n;
}

// out[k][0..3]: u'w' summed per quadrant, [4..7]: the quadrants' cell
// counts, [8]: u'w' summed over the plane.
__global__ void __launch_bounds__(kQuadThreads) quadrant_kernel(const double *__restrict__ vel,
                                                                const double *__restrict__ mean, int nx, int ny,
                                                                int zd, double *out /* [zd][9] */)
{
    __shared__ double smem[32 * 9];
    const int k = blockIdx.x + 1;
    const size_t n = (size_t)nx * ny;
    const double mu = mean[k * 3 + 0], mw = mean[k * 3 + 2];
    double s[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) s[i] = 0.0;
    for (size_t c = threadIdx.x; c < n; c += blockDim.x) {
        const double *v = vel + (c * zd + k) * 3;
        const double up = v[0] - mu, wp = v[2] - mw, p = up * wp;
        s[8] += p;
        const int q = up > 0.0 ? (wp > 0.0 ? 0 : (wp < 0.0 ? 3 : -1)) : (up < 0.0 ? (wp > 0.0 ? 1 : (wp < 0.0 ? 2 : -1)) : -1);
#pragma unroll
        for (int a = 0; a < 4; ++a)
            if (q == a) s[a] += p, s[4 + a] += 1.0;
    }
    block_sum<9>(s, smem);
    if (threadIdx.x == 0)
        for (int i = 0; i < 9; ++i) out[(size_t)k * 9 + i] = s[i];
}

void launch_quadrant(const double *vel, int nx, int ny, int zd, double *mean, double *out, cudaStream_t s)
{
    vel_plane_means_kernel<<<zd - 2, kQuadThreads, 0, s>>>(vel, nx, ny, zd, mean);
    quadrant_kernel<<<zd - 2, kQuadThreads, 0, s>>>(vel, mean, nx, ny, zd, out);
}

// ------------------------------------------------------------------ correlations
// Two-point velocity correlations of the reference's 2pt-correlations
// program (mean_subtract.c, xcorrel.c, ycorrel.c), one velocity field:
//   ua[k]              the subtracted mean of plane k: the plane means of
//                      u, v, w over (x, y), made symmetric about the channel
//                      centre (u, v even, w odd: mean_subtract.c:178-196);
//                      0 on the wall planes, which are not shifted;
//   xcorl[k][d][c]     sum over (x, y) of u'_c(x, y, k) u'_c(x + d, y, k),
//                      d = 0 .. nx-1 periodic (xcorrel.c);
//   ycorl[k][d][c]     sum over (x, y) of u'_c(x, y, k) u'_c(x, y + d, k),
//                      d = 0 .. ny-1 periodic (ycorrel.c).
// The fluctuations go to two copies, one with x-lines contiguous and one with
// y-lines contiguous; both correlations are then the same kernel: the
// autocorrelation of every line of a (plane, component), summed over the
// lines.  A block takes a chunk of lines, one line at a time in shared memory
// (stored twice, so a lag never wraps an index), one lag per thread and
// pass; the chunks' partial sums are added in chunk order, so the result does
// not depend on the run.  FP64 throughout.

constexpr int kCorrThreads = 256;
constexpr int kCorrLagPasses = 8;  // lines up to kCorrThreads * kCorrLagPasses cells

__global__ void corr_mean_kernel(const double *__restrict__ mean, int zd, double *ua /* [zd][3] */)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= zd) return;
    if (k == 0 || k == zd - 1) {
        ua[k * 3] = ua[k * 3 + 1] = ua[k * 3 + 2] = 0.0;
        return;
    }
    const int kk = zd - 1 - k;
    ua[k * 3 + 0] = 0.5 * (mean[k * 3 + 0] + mean[kk * 3 + 0]);
    ua[k * 3 + 1] = 0.5 * (mean[k * 3 + 1] + mean[kk * 3 + 1]);
    ua[k * 3 + 2] = 0.5 * (mean[k * 3 + 2] - mean[kk * 3 + 2]);
}

// vel [nx][ny][zd][3] -> rows [zd][3][ny][nx] and cols [zd][3][nx][ny],
// minus ua on the fluid planes
__global__ void corr_fluct_kernel(const double *__restrict__ vel, const double *__restrict__ ua, int nx, int ny,
                                  int zd, double *rows, double *cols)
{
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n = (size_t)nx * ny * zd;
    if (idx >= n) return;
    const int x = (int)(idx % nx);
    const size_t t = idx / nx;
    const int y = (int)(t % ny), k = (int)(t / ny);
    const double *v = vel + (((size_t)x * ny + y) * zd + k) * 3;
    const bool fluid = k >= 1 && k <= zd - 2;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double u = v[c] - (fluid ? ua[k * 3 + c] : 0.0);
        rows[(((size_t)k * 3 + c) * ny + y) * nx + x] = u;
        cols[(((size_t)k * 3 + c) * nx + x) * ny + y] = u;
    }
}

// lines [zd][3][nlines][len]; part [chunks][zd][3][len]
__global__ void __launch_bounds__(kCorrThreads) line_corr_kernel(const double *__restrict__ lines, int len, int nlines,
                                                                 int per_chunk, int zd, double *part)
{
    extern __shared__ double ln[];  // the line twice: ln[i] == ln[i + len]
    const int chunk = blockIdx.x, c = blockIdx.y, k = blockIdx.z;
    const int m0 = chunk * per_chunk, m1 = min(m0 + per_chunk, nlines);
    const double *base = lines + ((size_t)k * 3 + c) * nlines * len;
    double acc[kCorrLagPasses];
#pragma unroll
    for (int q = 0; q < kCorrLagPasses; ++q) acc[q] = 0.0;
    for (int m = m0; m < m1; ++m) {
        __syncthreads();  // the previous line is no longer read
        for (int i = threadIdx.x; i < len; i += blockDim.x) {
            const double v = base[(size_t)m * len + i];
            ln[i] = v;
            ln[i + len] = v;
        }
        __syncthreads();
        for (int i = 0; i < len; ++i) {
            const double a = ln[i];
#pragma unroll
            for (int q = 0; q < kCorrLagPasses; ++q) {
                const int d = threadIdx.x + q * blockDim.x;
                if (d < len) acc[q] = fma(a, ln[i + d], acc[q]);
            }
        }
    }
    double *out = part + (((size_t)chunk * zd + k) * 3 + c) * len;
#pragma unroll
    for (int q = 0; q < kCorrLagPasses; ++q) {
        const int d = threadIdx.x + q * blockDim.x;
        if (d < len) out[d] = acc[q];
    }
}

// out [zd][len][3] = sum over the chunks, in chunk order
__global__ void corr_reduce_kernel(const double *__restrict__ part, int nchunks, int len, int zd, double *out)
{
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n = (size_t)zd * 3 * len;
    if (idx >= n) return;
    const int d = (int)(idx % len);
    const size_t t = idx / len;
    const int c = (int)(t % 3), k = (int)(t / 3);
    double s = 0.0;
    for (int ch = 0; ch < nchunks; ++ch) s += part[(((size_t)ch * zd + k) * 3 + c) * len + d];
    out[((size_t)k * len + d) * 3 + c] = s;
}

// Scratch of launch_correlations, in doubles.
size_t correlation_scratch(int nx, int ny, int zd, int per_chunk)
{
    const size_t cells = (size_t)nx * ny * zd;
    const size_t cx = (size_t)(ny + per_chunk - 1) / per_chunk, cy = (size_t)(nx + per_chunk - 1) / per_chunk;
    return (size_t)zd * 3 * 2 + 2 * cells * 3 + std::max(cx * nx, cy * ny) * zd * 3;
}

int correlation_max_line() { return kCorrThreads * kCorrLagPasses; }

// vel in device memory; scratch of correlation_scratch doubles; xcorl
// [zd][nx][3], ycorl [zd][ny][3], ua [zd][3] in device memory.
cudaError_t launch_correlations(const double *vel, int nx, int ny, int zd, int per_chunk, double *scratch,
                                double *xcorl, double *ycorl, double *ua, cudaStream_t s)
{
    if (nx > correlation_max_line() || ny > correlation_max_line()) return cudaErrorInvalidValue;
    const size_t cells = (size_t)nx * ny * zd;
    double *mean = scratch, *rows = scratch + (size_t)zd * 3 * 2, *cols = rows + cells * 3, *part = cols + cells * 3;
    cudaError_t e = cudaMemsetAsync(mean, 0, sizeof(double) * zd * 3, s);
    if (e != cudaSuccess) return e;
    vel_plane_means_kernel<<<zd - 2, kQuadThreads, 0, s>>>(vel, nx, ny, zd, mean);
    corr_mean_kernel<<<(zd + 127) / 128, 128, 0, s>>>(mean, zd, ua);
    corr_fluct_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(vel, ua, nx, ny, zd, rows, cols);
    const int cx = (ny + per_chunk - 1) / per_chunk, cy = (nx + per_chunk - 1) / per_chunk;
    line_corr_kernel<<<dim3(cx, 3, zd), kCorrThreads, 2 * nx * sizeof(double), s>>>(rows, nx, ny, per_chunk, zd, part);
    corr_reduce_kernel<<<(unsigned)(((size_t)zd * 3 * nx + 255) / 256), 256, 0, s>>>(part, cx, nx, zd, xcorl);
    line_corr_kernel<<<dim3(cy, 3, zd), kCorrThreads, 2 * ny * sizeof(double), s>>>(cols, ny, nx, per_chunk, zd, part);
    corr_reduce_kernel<<<(unsigned)(((size_t)zd * 3 * ny + 255) / 256), 256, 0, s>>>(part, cy, ny, zd, ycorl);
    return cudaGetLastError();
}

}  // namespace dnslbm
