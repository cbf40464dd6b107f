// Post-processing on the GPU: the quadrant analysis of the reference's
// quadrant-analysis/src/qUADrantA.c, on a velocity field in the vel_print
// layout [nx][ny][zd][3] held in device memory (the moments of the running
// state, or a vel file uploaded by the caller).
//
// Per wall-normal fluid plane k = 1 .. zd-2 (one block each): the plane means
// of u, v, w over (x, y); the fluctuations u' = u - <u>, w' = w - <w>; the
// products u'w' summed over the plane and over each quadrant Q1 (u' > 0,
// w' > 0), Q2 (u' < 0, w' > 0), Q3 (u' < 0, w' < 0), Q4 (u' > 0, w' < 0),
// with the cell count of each quadrant (a zero u' or w' falls in none, as in
// the reference).  Sums are FP64 in a fixed order (per-thread strided sums,
// then the deterministic block reduction), so a result does not depend on the
// run; it differs from the reference's sequential sums by rounding only.
#include <cuda_runtime.h>

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

}  // namespace dnslbm
