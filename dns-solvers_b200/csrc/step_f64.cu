// Plain FP64 fused step (collide + stream + wall rules + periodic wrap +
// per-step reductions), AA pattern, one launch per time step.
//
// Every floating-point operation of the collision keeps the reference's
// operand order (xcomputations.c:314-342) and this file is compiled with
// -fmad=false, so on a grid the reference can express the populations after
// any number of constant-g steps are bit-identical to the reference's.
// Zero terms of the reference's sums (E*f with E == 0) are omitted: adding a
// signed zero to a non-zero partial sum leaves it unchanged.
#include "collide_f64.cuh"
#include "step_common.cuh"
#include "step_links.cuh"

namespace dnslbm {

template <int A, bool ODD>
__device__ __forceinline__ double *f64_ptr(const StepArgs &p, const Nbr &n, int wall, unsigned bits)
{
    int slot, idx;
    aa_address<A, ODD>(n, wall, bits, slot, idx);
    return static_cast<double *>(p.pop[slot]) + idx;
}

template <bool ODD, bool CONSTQ, int TEX>
__global__ void __launch_bounds__(128, 4) step_f64_kernel(const StepArgs p)
{
    const long long step = *p.step_ctr;
    const double G = CONSTQ ? p.force[step & 1] : p.gx;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.z;
    const int wall = plane_wall(p, z);
    const double c0 = p.shift[(size_t)(step & 1) * p.nz * 3 + z * 3 + 0];
    const double c1 = p.shift[(size_t)(step & 1) * p.nz * 3 + z * 3 + 1];
    const double c2 = p.shift[(size_t)(step & 1) * p.nz * 3 + z * 3 + 2];
    double acc[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i] = 0.0;

    if (x < p.nx) {
        const int y0 = blockIdx.y * p.rows;
        const int y1 = min(y0 + p.rows, p.ny);
        for (int y = y0; y < y1; ++y) {
            const Nbr n = make_nbr(x, y, z, p.nx, p.ny, p.pitch);
            unsigned bits = 0x1fu;
            if (TEX != 0 && wall != 0) bits = p.wallmask[(size_t)(wall > 0) * p.nx * p.ny + y * p.nx + x];
            if (TEX == 2 && p.band_of[z] >= 0) {  // plane next to a solid: per-cell links
                float racc[NP] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                links_cell<double, ODD, CONSTQ>(p, n, wall, cell_links(p.band_of, p.links, p.nx, p.ny, x, y, z), nullptr, 0,
                                          G, c0, c1, c2, acc, racc);
#pragma unroll
                for (int i = 0; i < NP; ++i) acc[i] += (double)racc[i];
                continue;
            }
            double f[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                double *q;
                switch (a) {
#define PT(A) case A: q = f64_ptr<A, ODD>(p, n, wall, bits); break;
                    PT(0) PT(1) PT(2) PT(3) PT(4) PT(5) PT(6) PT(7) PT(8) PT(9)
                    PT(10) PT(11) PT(12) PT(13) PT(14) PT(15) PT(16) PT(17) PT(18)
#undef PT
                }
                f[ODD ? lat_opp(a) : a] = *q;
            }
            const F64Cell c = f64_collide(f, p.omega, G);
            acc[0] += c.dens;
            acc[1] += c.jx;
            acc[2] += c.u0;
            acc[3] += c.u1;
            acc[4] += c.u2;
            {
                const double d0 = c.u0 - c0, d1 = c.u1 - c1, d2 = c.u2 - c2;
                acc[5] += d0 * d0 + d1 * d1 + d2 * d2;
            }
            if (CONSTQ) {
                double s = 0.0, m = 0.0;
#pragma unroll
                for (int a = 0; a < Q; ++a) {
                    s += f[a];
                    if (lat_ex(a) > 0) m += f[a];
                    if (lat_ex(a) < 0) m -= f[a];
                }
                // links that bounce back arrive with e_x reversed
                if (wall != 0) {
                    const int ap = wall < 0 ? 12 : 11, am = wall < 0 ? 13 : 14;  // e_x = +1 / -1 into the wall
                    if (bits & 2u) m -= 2. * f[ap];
                    if (bits & 4u) m += 2. * f[am];
                }
                acc[6] += s;
                acc[7] += m;
            }
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                double *q;
                switch (a) {
#define PT(A) case A: q = f64_ptr<A, ODD>(p, n, wall, bits); break;
                    PT(0) PT(1) PT(2) PT(3) PT(4) PT(5) PT(6) PT(7) PT(8) PT(9)
                    PT(10) PT(11) PT(12) PT(13) PT(14) PT(15) PT(16) PT(17) PT(18)
#undef PT
                }
                *q = f[ODD ? a : lat_opp(a)];
            }
        }
    }
    block_epilogue(p, acc, step, G, 0);
}

// Reader-only reduction of the current state (after a load/init): force and
// plane means for the first step.  Reads the natural layout.
__global__ void __launch_bounds__(128) reduce_f64_kernel(const StepArgs p)
{
    const long long step = *p.step_ctr;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.z;
    double acc[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i] = 0.0;
    if (x < p.nx) {
        const int y0 = blockIdx.y * p.rows;
        const int y1 = min(y0 + p.rows, p.ny);
        for (int y = y0; y < y1; ++y) {
            const int c = (z * p.ny + y) * p.pitch + x;
            double f[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a) f[a] = static_cast<const double *>(p.pop[a])[c];
            double dens, jx, jy, jz;
            f64_moments(f, dens, jx, jy, jz);
            acc[0] += dens;
            acc[1] += jx;
            acc[2] += jx / dens;
            acc[3] += jy / dens;
            acc[4] += jz / dens;
        }
    }
    block_epilogue(p, acc, step, 0.0, 1);
}

// The same for a state left by an odd number of steps (post-collision
// values in swapped slots): each cell gathers its populations through the
// odd-step address set (periodic wrap, wall links by the wall mask), so the
// sums are those of the state the next step starts from.  Used by the
// allocation-free entry point, which has no plane means carried over from an
// earlier call.
template <int TEX>
__global__ void __launch_bounds__(128) reduce_f64_odd_kernel(const StepArgs p)
{
    const long long step = *p.step_ctr;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.z;
    const int wall = plane_wall(p, z);
    double acc[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i] = 0.0;
    if (x < p.nx) {
        const int y0 = blockIdx.y * p.rows;
        const int y1 = min(y0 + p.rows, p.ny);
        for (int y = y0; y < y1; ++y) {
            const Nbr n = make_nbr(x, y, z, p.nx, p.ny, p.pitch);
            unsigned bits = 0x1fu;
            if (TEX != 0 && wall != 0) bits = p.wallmask[(size_t)(wall > 0) * p.nx * p.ny + y * p.nx + x];
            double f[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                const double *q;
                switch (a) {
#define PT(A) case A: q = f64_ptr<A, true>(p, n, wall, bits); break;
                    PT(0) PT(1) PT(2) PT(3) PT(4) PT(5) PT(6) PT(7) PT(8) PT(9)
                    PT(10) PT(11) PT(12) PT(13) PT(14) PT(15) PT(16) PT(17) PT(18)
#undef PT
                }
                f[lat_opp(a)] = *q;
            }
            double dens, jx, jy, jz;
            f64_moments(f, dens, jx, jy, jz);
            acc[0] += dens;
            acc[1] += jx;
            acc[2] += jx / dens;
            acc[3] += jy / dens;
            acc[4] += jz / dens;
        }
    }
    block_epilogue(p, acc, step, 0.0, 1);
}

void launch_step_f64(const StepArgs &p, dim3 grid, dim3 block, bool odd, int tex, cudaStream_t s)
{
    const bool q = p.const_q != 0;
#define L(O, C, T) step_f64_kernel<O, C, T><<<grid, block, 0, s>>>(p)
#define LX(O, C) do { if (tex == 2) L(O, C, 2); else if (tex) L(O, C, 1); else L(O, C, 0); } while (0)
    if (odd) {
        if (q) LX(true, true); else LX(true, false);
    } else {
        if (q) LX(false, true); else LX(false, false);
    }
#undef LX
#undef L
}

void launch_reduce_f64(const StepArgs &p, dim3 grid, dim3 block, cudaStream_t s)
{
    reduce_f64_kernel<<<grid, block, 0, s>>>(p);
}

void launch_reduce_f64_odd(const StepArgs &p, dim3 grid, dim3 block, int tex, cudaStream_t s)
{
    if (tex) reduce_f64_odd_kernel<1><<<grid, block, 0, s>>>(p);
    else reduce_f64_odd_kernel<0><<<grid, block, 0, s>>>(p);
}

// Step tail of one wall-normal slab of a channel split over several GPUs
// (one block).  `a` describes the whole channel: nz planes, the plane sums
// of all slabs gathered in plane order, the context's copy of the whole
// channel's plane means.  The tail is the one a whole-channel step runs
// (step_tail: logs, force, plane means; identical on every slab, which all
// hold the same gathered sums); then the slab's planes [z0, z0 + nzs) of
// the new plane means go to its own shift array ([2][nzs][3]), which its
// step kernel reads.  mode 0 after a step, 1 after a state load.
__global__ void __launch_bounds__(256) slab_tail_kernel(const StepArgs a, int mode, double *slab_shift, int z0,
                                                        int nzs)
{
    __shared__ double smem[32 * NP];
    const long long step = __ldcg(a.step_ctr);
    const double force_used = __ldcg(a.force + (step & 1));
    step_tail(a, step, force_used, mode, smem, blockDim.x);
    __syncthreads();
    const int par = (int)((mode == 0 ? step + 1 : step) & 1);
    const double *src = a.shift + (size_t)par * a.nz * 3 + (size_t)z0 * 3;
    double *dst = slab_shift + (size_t)par * nzs * 3;
    for (int i = threadIdx.x; i < nzs * 3; i += blockDim.x) dst[i] = __ldcg(src + i);
}

void launch_slab_tail(const StepArgs &a, int mode, double *slab_shift, int z0, int nzs, cudaStream_t s)
{
    slab_tail_kernel<<<1, 256, 0, s>>>(a, mode, slab_shift, z0, nzs);
}

}  // namespace dnslbm
