// State import/export in the reference's AoS lbf layout, per-cell moments
// (vel_print.c) and the two-pass plane statistics (statistics.c), for every
// storage precision and either AA parity.
//
// After an even step the populations sit post-collision in swapped slots; the
// natural (post-stream) value f_a of a cell is then what the odd step would
// load into f[a], so every reader here gathers through the odd address set.
#include <cuda_fp16.h>

#include "step_common.cuh"

namespace dnslbm {

template <typename T> struct Nat;
template <> struct Nat<double> {
    static __device__ __forceinline__ double ld(const double *p, int) { return *p; }
    static __device__ __forceinline__ void st(double *p, double f, int) { *p = f; }
};
template <> struct Nat<float> {
    static __device__ __forceinline__ double ld(const float *p, int a) { return wq(a) + (double)*p; }
    static __device__ __forceinline__ void st(float *p, double f, int a) { *p = (float)(f - wq(a)); }
    static __device__ __forceinline__ double wq(int a) { return a == 0 ? 1. / 3. : a <= 6 ? 1. / 18. : 1. / 36.; }
};
template <> struct Nat<__half> {
    static __device__ __forceinline__ double ld(const __half *p, int a)
    {
        return Nat<float>::wq(a) + (double)__half2float(*p) * (1. / 32768.);
    }
    static __device__ __forceinline__ void st(__half *p, double f, int a)
    {
        *p = __double2half((f - Nat<float>::wq(a)) * 32768.);
    }
};

template <typename T, int A>
__device__ __forceinline__ double gather_one(const IoArgs &p, const Nbr &n, int wall, unsigned bits)
{
    int slot, idx;
    aa_address<A, true>(n, wall, bits, slot, idx);
    return Nat<T>::ld(static_cast<const T *>(p.pop[slot]) + idx, lat_opp(A));
}

template <typename T, int A>
__device__ __forceinline__ double gather_one_links(const IoArgs &p, const Nbr &n, int wall, unsigned lk)
{
    int slot, idx;
    aa_address_links<A, true>(n, wall, lk, slot, idx);
    return Nat<T>::ld(static_cast<const T *>(p.pop[slot]) + idx, lat_opp(A));
}

// natural populations of cell (x, y, z)
template <typename T>
__device__ __forceinline__ void gather_natural(const IoArgs &p, int x, int y, int z, double (&f)[Q])
{
    const unsigned lk = p.textured == 2 ? cell_links(p.band_of, p.links, p.nx, p.ny, x, y, z) : 0u;
    if (!p.odd || (lk & 1u)) {  // a solid cell keeps its (symmetric) rest state in place
        const int c = (z * p.ny + y) * p.pitch + x;
#pragma unroll
        for (int a = 0; a < Q; ++a) f[a] = Nat<T>::ld(static_cast<const T *>(p.pop[a]) + c, a);
        return;
    }
    const Nbr n = make_nbr(x, y, z, p.nx, p.ny, p.pitch);
    const int wall = z == 0 ? -1 : (z == p.nz - 1 ? 1 : 0);
    if (p.textured == 2 && p.band_of[z] >= 0) {
#pragma unroll
        for (int a = 0; a < Q; ++a) {
            double v;
            switch (a) {
#define G1(A) case A: v = gather_one_links<T, A>(p, n, wall, lk); break;
                G1(0) G1(1) G1(2) G1(3) G1(4) G1(5) G1(6) G1(7) G1(8) G1(9)
                G1(10) G1(11) G1(12) G1(13) G1(14) G1(15) G1(16) G1(17) G1(18)
#undef G1
            }
            f[lat_opp(a)] = v;
        }
        return;
    }
    unsigned bits = 0x1fu;
    if (p.textured && wall != 0) bits = p.wallmask[(size_t)(wall > 0) * p.nx * p.ny + y * p.nx + x];
#pragma unroll
    for (int a = 0; a < Q; ++a) {
        double v;
        switch (a) {
#define G1(A) case A: v = gather_one<T, A>(p, n, wall, bits); break;
            G1(0) G1(1) G1(2) G1(3) G1(4) G1(5) G1(6) G1(7) G1(8) G1(9)
            G1(10) G1(11) G1(12) G1(13) G1(14) G1(15) G1(16) G1(17) G1(18)
#undef G1
        }
        f[lat_opp(a)] = v;
    }
}

// Tiles of kTX consecutive x by kTZ consecutive z of one y, through shared
// memory: the SoA side is read or written along x (coalesced per
// direction), the AoS side along a cell's kTZ * 19 contiguous doubles.  AoS
// index of x-slab [x0, x0+nxc): ((x-x0)*ny + y)*zd + (z+1), times 19.
constexpr int kTX = 32, kTZ = 8;

template <typename T>
__global__ void __launch_bounds__(kTX * kTZ) export_kernel(const IoArgs p, int x0, int nxc, double *aos)
{
    __shared__ double sh[kTX][kTZ * Q + 1];
    const int tx = threadIdx.x % kTX, tz = threadIdx.x / kTX;
    const int xl0 = blockIdx.x * kTX, z0 = blockIdx.y * kTZ, y = blockIdx.z;
    if (xl0 + tx < nxc && z0 + tz < p.nz) {
        double f[Q];
        gather_natural<T>(p, x0 + xl0 + tx, y, z0 + tz, f);
#pragma unroll
        for (int a = 0; a < Q; ++a) sh[tx][tz * Q + a] = f[a];
    }
    __syncthreads();
    const int per_x = min(kTZ, p.nz - z0) * Q;
    for (int i = threadIdx.x; i < kTX * per_x; i += blockDim.x) {
        const int xi = i / per_x, r = i - xi * per_x;
        if (xl0 + xi < nxc) aos[(((size_t)(xl0 + xi) * p.ny + y) * (p.nz + 2) + (z0 + 1)) * Q + r] = sh[xi][r];
    }
}

template <typename T>
__global__ void __launch_bounds__(kTX * kTZ) import_kernel(const IoArgs p, int x0, int nxc, const double *aos)
{
    __shared__ double sh[kTX][kTZ * Q + 1];
    const int tx = threadIdx.x % kTX, tz = threadIdx.x / kTX;
    const int xl0 = blockIdx.x * kTX, z0 = blockIdx.y * kTZ, y = blockIdx.z;
    const int per_x = min(kTZ, p.nz - z0) * Q;
    for (int i = threadIdx.x; i < kTX * per_x; i += blockDim.x) {
        const int xi = i / per_x, r = i - xi * per_x;
        if (xl0 + xi < nxc) sh[xi][r] = aos[(((size_t)(xl0 + xi) * p.ny + y) * (p.nz + 2) + (z0 + 1)) * Q + r];
    }
    __syncthreads();
    const int x = x0 + xl0 + tx, z = z0 + tz;
    if (xl0 + tx >= nxc || z >= p.nz) return;
    const int c = (z * p.ny + y) * p.pitch + x;
    const bool solid = p.textured == 2 && (cell_links(p.band_of, p.links, p.nx, p.ny, x, y, z) & 1u);
#pragma unroll
    for (int a = 0; a < Q; ++a)
        Nat<T>::st(static_cast<T *>(p.pop[a]) + c, solid ? Nat<float>::wq(a) : sh[tx][tz * Q + a], a);
}

// solid cells inside the flow -> rest state (after the flags change)
template <typename T>
__global__ void solid_rest_kernel(const IoArgs p)
{
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long)p.nx * p.ny * p.nz) return;
    const int x = (int)(tid % p.nx), y = (int)((tid / p.nx) % p.ny), z = (int)(tid / ((long long)p.nx * p.ny));
    if (!(cell_links(p.band_of, p.links, p.nx, p.ny, x, y, z) & 1u)) return;
    const int c = (z * p.ny + y) * p.pitch + x;
#pragma unroll
    for (int a = 0; a < Q; ++a) Nat<T>::st(static_cast<T *>(p.pop[a]) + c, Nat<float>::wq(a), a);
}

// rest state f = w (init.c:6-19); row padding included
template <typename T>
__global__ void rest_kernel(const IoArgs p)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)p.pitch * p.ny * p.nz) return;
#pragma unroll
    for (int a = 0; a < Q; ++a) Nat<T>::st(static_cast<T *>(p.pop[a]) + c, Nat<float>::wq(a), a);
}

// vel_print.c:71-96: moments in the reference's order, u = 0, rho = 0 where
// rho <= 0; wall planes are written as zeros.
template <typename T>
__global__ void moments_kernel(const IoArgs p, int x0, int nxc, double *vel, double *den)
{
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int zd = p.nz + 2;
    const long long ncell = (long long)nxc * p.ny * zd;
    if (tid >= ncell) return;
    const int k = (int)(tid % zd);
    const int y = (int)((tid / zd) % p.ny);
    const int xl = (int)(tid / ((long long)zd * p.ny));
    double ux = 0., uy = 0., uz = 0., dens = 0.;
    if (k >= 1 && k <= p.nz) {
        double f[Q];
        gather_natural<T>(p, x0 + xl, y, k - 1, f);
#pragma unroll
        for (int a = 0; a < Q; ++a) {
            if (lat_ex(a) > 0) ux = ux + f[a];
            if (lat_ex(a) < 0) ux = ux - f[a];
            if (lat_ey(a) > 0) uy = uy + f[a];
            if (lat_ey(a) < 0) uy = uy - f[a];
            if (lat_ez(a) > 0) uz = uz + f[a];
            if (lat_ez(a) < 0) uz = uz - f[a];
            dens = dens + f[a];
        }
        if (dens > 0.) {
            ux /= dens;
            uy /= dens;
            uz /= dens;
        } else {
            ux = 0.; uy = 0.; uz = 0.; dens = 0.;
        }
    }
    const size_t o = ((size_t)xl * p.ny + y) * zd + k;
    if (vel) {
        vel[o * 3 + 0] = ux;
        vel[o * 3 + 1] = uy;
        vel[o * 3 + 2] = uz;
    }
    if (den) den[o] = dens;
}

// Two-pass plane statistics (statistics.c:31-132).  pass 0: sums of
// u, v, w, rho per plane; pass 1: sums of u'^2, v'^2, w'^2, u'w', rho'^2
// about the plane means `mean` [nz][4].  Block partials [nz][bpp][5].
constexpr int NS = 5;
template <typename T>
__global__ void __launch_bounds__(128) stats_kernel(const IoArgs p, int rows, int pass, const double *mean,
                                                    double *partials)
{
    __shared__ double smem[32 * NS];
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.z;
    double acc[NS] = {0, 0, 0, 0, 0};
    if (x < p.nx) {
        const int y0 = blockIdx.y * rows, y1 = min(y0 + rows, p.ny);
        for (int y = y0; y < y1; ++y) {
            double f[Q];
            gather_natural<T>(p, x, y, z, f);
            double dens = 0., u = 0., v = 0., w = 0.;
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                dens = dens + f[a];
                if (lat_ex(a) > 0) u = u + f[a];
                if (lat_ex(a) < 0) u = u - f[a];
                if (lat_ey(a) > 0) v = v + f[a];
                if (lat_ey(a) < 0) v = v - f[a];
                if (lat_ez(a) > 0) w = w + f[a];
                if (lat_ez(a) < 0) w = w - f[a];
            }
            if (pass == 0) {
                acc[0] += u / dens;
                acc[1] += v / dens;
                acc[2] += w / dens;
                acc[3] += dens;
            } else {
                const double uf = (u / dens) - mean[z * 4 + 0], vf = (v / dens) - mean[z * 4 + 1];
                const double wf = (w / dens) - mean[z * 4 + 2], df = dens - mean[z * 4 + 3];
                acc[0] += uf * uf;
                acc[1] += vf * vf;
                acc[2] += wf * wf;
                acc[3] += uf * wf;
                acc[4] += df * df;
            }
        }
    }
    block_sum<NS>(acc, smem);
    if (threadIdx.x == 0) {
        const unsigned bpp = gridDim.x * gridDim.y;
        double *o = partials + ((size_t)z * bpp + blockIdx.y * gridDim.x + blockIdx.x) * NS;
#pragma unroll
        for (int i = 0; i < NS; ++i) o[i] = acc[i];
    }
}

// one block per plane: fixed-order sum of the plane's block partials
__global__ void plane_reduce_kernel(const double *partials, int bpp, double *out /* [nz][NS] */)
{
    __shared__ double smem[32 * NS];
    const int z = blockIdx.x;
    double s[NS] = {0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < bpp; b += blockDim.x)
#pragma unroll
        for (int i = 0; i < NS; ++i) s[i] += partials[((size_t)z * bpp + b) * NS + i];
    block_sum<NS>(s, smem);
    if (threadIdx.x == 0)
#pragma unroll
        for (int i = 0; i < NS; ++i) out[z * NS + i] = s[i];
}

// On-device time averages of the plane statistics: the plane means of a
// sample from its pass-0 sums, and the running FP64 sums of the sample's
// nine statistics rows (statistics.c order: u, v, w means, u', v', w' rms,
// <u'w'>, rho mean, rho' rms) with each rms entered as its square, which is
// how the reference's post-processing pools rms values over a time window
// (TKE-budget/postprocessing/time_stats.c:203-213).
__global__ void stats_means_kernel(const double *planes, int nz, double np, double *mean)
{
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= nz) return;
#pragma unroll
    for (int i = 0; i < 4; ++i) mean[z * 4 + i] = planes[z * NS + i] / np;
}

__global__ void stats_accumulate_kernel(const double *planes, const double *mean, int nz, double np, double *acc)
{
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= nz) return;
    const double *pl = planes + (size_t)z * NS;
    acc[0 * nz + z] += mean[z * 4 + 0];
    acc[1 * nz + z] += mean[z * 4 + 1];
    acc[2 * nz + z] += mean[z * 4 + 2];
    acc[3 * nz + z] += pl[0] / np;
    acc[4 * nz + z] += pl[1] / np;
    acc[5 * nz + z] += pl[2] / np;
    acc[6 * nz + z] += pl[3] / np;
    acc[7 * nz + z] += mean[z * 4 + 3];
    acc[8 * nz + z] += pl[4] / np;
}

// The statistics rows of one sample in the turb-fld layout [9][nz + 2]
// (statistics.c:139-147 file order; wall entries left as they are): plane
// means from pass 0 (mean[z][u v w rho]) and the pass-1 second-moment sums.
__global__ void stats_rows_kernel(const double *mean, const double *planes, int nz, double np, double *out)
{
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= nz) return;
    const int zd = nz + 2;
    const double *pl = planes + (size_t)z * NS;
    out[0 * zd + z + 1] = mean[z * 4 + 0];
    out[1 * zd + z + 1] = mean[z * 4 + 1];
    out[2 * zd + z + 1] = mean[z * 4 + 2];
    out[3 * zd + z + 1] = sqrt(pl[0] / np);
    out[4 * zd + z + 1] = sqrt(pl[1] / np);
    out[5 * zd + z + 1] = sqrt(pl[2] / np);
    out[6 * zd + z + 1] = pl[3] / np;
    out[7 * zd + z + 1] = mean[z * 4 + 3];
    out[8 * zd + z + 1] = sqrt(pl[4] / np);
}

// ---------------------------------------------------------------- launchers
template <typename T>
static void io_dispatch(int what, const IoArgs &p, int x0, int nxc, double *a, double *b, cudaStream_t s)
{
    const int bs = 256;
    if (what == 0 || what == 1) {
        const dim3 grid((nxc + kTX - 1) / kTX, (p.nz + kTZ - 1) / kTZ, p.ny);
        if (what == 0) export_kernel<T><<<grid, kTX * kTZ, 0, s>>>(p, x0, nxc, a);
        else import_kernel<T><<<grid, kTX * kTZ, 0, s>>>(p, x0, nxc, a);
    } else if (what == 2) {
        const long long n = (long long)p.pitch * p.ny * p.nz;
        rest_kernel<T><<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(p);
    } else if (what == 4) {
        const long long n = (long long)p.nx * p.ny * p.nz;
        solid_rest_kernel<T><<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(p);
    } else {
        const long long n = (long long)nxc * p.ny * (p.nz + 2);
        moments_kernel<T><<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(p, x0, nxc, a, b);
    }
}

void launch_io(int precision, int what, const IoArgs &p, int x0, int nxc, double *a, double *b, cudaStream_t s)
{
    if (precision == 64) io_dispatch<double>(what, p, x0, nxc, a, b, s);
    else if (precision == 32) io_dispatch<float>(what, p, x0, nxc, a, b, s);
    else io_dispatch<__half>(what, p, x0, nxc, a, b, s);
}

void launch_stats_sample(int nz, double np, const double *planes, double *mean, double *acc, bool accumulate,
                         cudaStream_t s)
{
    const int bs = 128, nb = (nz + bs - 1) / bs;
    if (accumulate) stats_accumulate_kernel<<<nb, bs, 0, s>>>(planes, mean, nz, np, acc);
    else stats_means_kernel<<<nb, bs, 0, s>>>(planes, nz, np, mean);
}

void launch_stats_rows(int nz, double np, const double *mean, const double *planes, double *out, cudaStream_t s)
{
    const int bs = 128;
    stats_rows_kernel<<<(nz + bs - 1) / bs, bs, 0, s>>>(mean, planes, nz, np, out);
}

void launch_stats(int precision, const IoArgs &p, dim3 grid, dim3 block, int rows, int pass, const double *mean,
                  double *partials, double *plane_out, cudaStream_t s)
{
    if (precision == 64) stats_kernel<double><<<grid, block, 0, s>>>(p, rows, pass, mean, partials);
    else if (precision == 32) stats_kernel<float><<<grid, block, 0, s>>>(p, rows, pass, mean, partials);
    else stats_kernel<__half><<<grid, block, 0, s>>>(p, rows, pass, mean, partials);
    plane_reduce_kernel<<<p.nz, 128, 0, s>>>(partials, (int)(grid.x * grid.y), plane_out);
}

}  // namespace dnslbm
