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

namespace dnslbm {

// ------------------------------------------------------------------ spectra
// One-dimensional energy spectra of the reference's e-spectra program
// (e-spectra/src/1d-spectra.c), one velocity field.  Per fluid plane k and
// component c: the 2-D real-to-complex DFT over (x, y) (FFTW's r2c_2d,
// C[i][j] = sum_{x,y} u(x, y) e^{-2 pi i (i x / nx + j y / ny)}, i < nx,
// j <= ny/2), scaled by 2 / (2 nx ny) (:131-143), the (0, 0) mode set to 0
// (:146-151), then p = 0.5 fac_j |C|^2 with fac_0 = 1, fac_j = 2 otherwise
// (:156-172), summed over j into E_x[i][k] and over i into E_y[j][k]; the
// wall planes are 0.  The DFT is evaluated directly in FP64 (two passes: the
// half spectrum along y for every x line, then the full transform along x of
// every kept y mode), with exact twiddle factors sincospi(2 m / n), m = n*index
// mod n; the sums are FP64 in a fixed order.  Output files Euux/Evvx/Ewwx
// ([nx][zd] each) and Euuy/Evvy/Ewwy ([ny/2+1][zd] each).

constexpr int kSpecThreads = 256;

// twiddles: tw[m] = (cos(2 pi m / n), -sin(2 pi m / n)), m < n
__global__ void spec_twiddle_kernel(int n, double2 *tw)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double s, c;
    sincospi(2.0 * (double)m / (double)n, &s, &c);
    tw[m] = make_double2(c, -s);
}

// pass 1: V[k][c][j][x] = sum_y u(x, y, k, c) tw_y[(j y) mod ny], j < nj
// grid (ceil(nx / lines), zd - 2, 3); one x line per warp-sized group
__global__ void __launch_bounds__(kSpecThreads) spec_y_kernel(const double *__restrict__ vel,
                                                              const double2 *__restrict__ twy, int nx, int ny,
                                                              int zd, int nj, int lines, double2 *V)
{
    extern __shared__ double sm[];  // twiddles (2 ny), then `lines` lines of ny
    double2 *tw = reinterpret_cast<double2 *>(sm);
    double *ln = sm + 2 * ny;
    const int x0 = blockIdx.x * lines, k = blockIdx.y + 1, c = blockIdx.z;
    const int nl = min(lines, nx - x0);
    for (int m = threadIdx.x; m < ny; m += blockDim.x) tw[m] = twy[m];
    for (int e = threadIdx.x; e < nl * ny; e += blockDim.x) {
        const int l = e / ny, y = e - l * ny;
        ln[e] = vel[(((size_t)(x0 + l) * ny + y) * zd + k) * 3 + c];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nl * nj; e += blockDim.x) {
        const int l = e / nj, j = e - l * nj;
        const double *u = ln + (size_t)l * ny;
        double re = 0.0, im = 0.0;
        int m = 0;
        for (int y = 0; y < ny; ++y) {
            const double2 w = tw[m];
            re = fma(u[y], w.x, re);
            im = fma(u[y], w.y, im);
            m += j;
            if (m >= ny) m -= ny;
        }
        V[(((size_t)blockIdx.y * 3 + c) * nj + j) * nx + x0 + l] = make_double2(re, im);
    }
}

// pass 2: C[i][j] = sum_x V[j][x] tw_x[(i x) mod nx] for the block's `jb` modes
// j; p = 0.5 fac_j |s C|^2 (C[0][0] = 0); ey[k][c][j] = sum_i p, and the
// block's partial sum over its j of p per i in part[chunk][k][c][i]
__global__ void __launch_bounds__(kSpecThreads) spec_x_kernel(const double2 *__restrict__ V,
                                                              const double2 *__restrict__ twx, int nx, int nj,
                                                              int zd, int jb, double scale, double *ey,
                                                              double *part)
{
    extern __shared__ double sm[];
    double2 *tw = reinterpret_cast<double2 *>(sm);  // nx twiddles, then jb columns of nx
    double2 *col = tw + nx;
    __shared__ double red[32];
    const int j0 = blockIdx.x * jb, kk = blockIdx.y, c = blockIdx.z;
    const int nb = min(jb, nj - j0);
    for (int m = threadIdx.x; m < nx; m += blockDim.x) tw[m] = twx[m];
    const double2 *src = V + (((size_t)kk * 3 + c) * nj + j0) * nx;
    for (int e = threadIdx.x; e < nb * nx; e += blockDim.x) col[e] = src[e];
    __syncthreads();
    double *pout = part + (((size_t)blockIdx.x * (zd - 2) + kk) * 3 + c) * nx;
    for (int i0 = 0; i0 < nx; i0 += blockDim.x) {
        const int i = i0 + threadIdx.x;
        double px = 0.0;
        for (int b = 0; b < nb; ++b) {
            const int j = j0 + b;
            double p = 0.0;
            if (i < nx) {
                const double2 *v = col + (size_t)b * nx;
                double re = 0.0, im = 0.0;
                int m = 0;
                for (int x = 0; x < nx; ++x) {
                    const double2 w = tw[m], a = v[x];
                    re = fma(a.x, w.x, re);
                    re = fma(-a.y, w.y, re);
                    im = fma(a.x, w.y, im);
                    im = fma(a.y, w.x, im);
                    m += i;
                    if (m >= nx) m -= nx;
                }
                re *= scale;
                im *= scale;
                if (i == 0 && j == 0) re = im = 0.0;
                p = (j == 0 ? 0.5 : 1.0) * (re * re + im * im);
                px += p;
            }
            // the block's sum over i for mode j, in a fixed order
            double s[1] = {p};
            block_sum<1>(s, red);
            if (threadIdx.x == 0) {
                double *dst = ey + (((size_t)kk * 3 + c) * nj + j);
                *dst = (i0 == 0 ? 0.0 : *dst) + s[0];
            }
            __syncthreads();
        }
        if (i < nx) pout[i] = px;
    }
}

// E_x[k][c][i] = sum over the j chunks of part, in chunk order
__global__ void spec_reduce_kernel(const double *__restrict__ part, int nchunks, int nx, int nzf, double *ex)
{
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n = (size_t)nzf * 3 * nx;
    if (idx >= n) return;
    double s = 0.0;
    for (int ch = 0; ch < nchunks; ++ch) s += part[(size_t)ch * n + idx];
    ex[idx] = s;
}

// Scratch of launch_spectra, in doubles.
size_t spectra_scratch(int nx, int ny, int zd, int jb)
{
    const int nj = ny / 2 + 1, chunks = (nj + jb - 1) / jb;
    return 2 * (size_t)(nx + ny) + 2 * (size_t)(zd - 2) * 3 * nj * nx + (size_t)chunks * (zd - 2) * 3 * nx;
}

// ex [zd-2][3][nx], ey [zd-2][3][ny/2+1] in device memory (fluid planes)
cudaError_t launch_spectra(const double *vel, int nx, int ny, int zd, int jb, double *scratch, double *ex, double *ey,
                           cudaStream_t s)
{
    const int nj = ny / 2 + 1, nzf = zd - 2, chunks = (nj + jb - 1) / jb;
    double2 *twx = reinterpret_cast<double2 *>(scratch), *twy = twx + nx;
    double2 *V = twy + ny;
    double *part = reinterpret_cast<double *>(V + (size_t)nzf * 3 * nj * nx);
    const size_t sm1_lines = 8;
    const size_t sm1 = (2 * (size_t)ny + sm1_lines * ny) * sizeof(double);
    const size_t sm2 = ((size_t)nx + (size_t)jb * nx) * sizeof(double2);
    cudaError_t e = cudaFuncSetAttribute(spec_y_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(spec_x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
    if (e != cudaSuccess) return e;
    spec_twiddle_kernel<<<(nx + 255) / 256, 256, 0, s>>>(nx, twx);
    spec_twiddle_kernel<<<(ny + 255) / 256, 256, 0, s>>>(ny, twy);
    spec_y_kernel<<<dim3((nx + (int)sm1_lines - 1) / (int)sm1_lines, nzf, 3), kSpecThreads, sm1, s>>>(
        vel, twy, nx, ny, zd, nj, (int)sm1_lines, V);
    spec_x_kernel<<<dim3(chunks, nzf, 3), kSpecThreads, sm2, s>>>(V, twx, nx, nj, zd, jb,
                                                                    2.0 * (1.0 / (2.0 * nx * ny)), ey, part);
    spec_reduce_kernel<<<(unsigned)(((size_t)nzf * 3 * nx + 255) / 256), 256, 0, s>>>(part, chunks, nx, nzf, ex);
    return cudaGetLastError();
}

}  // namespace dnslbm
