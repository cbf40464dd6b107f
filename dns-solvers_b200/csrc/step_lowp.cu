// Reduced-precision fused step with per-thread global accesses (one thread
// per cell): populations stored as deviations f_a - w_a in FP32 or FP16
// (collide_lp.cuh), collided in FP32; the per-step reductions and the
// constant-Q force are accumulated in FP64.  Used where the row-pipelined
// kernel (step_tma.cuh) does not fit shared memory.
#include <cuda_fp16.h>

#include "collide_lp.cuh"
#include "step_common.cuh"
#include "step_links.cuh"

namespace dnslbm {

template <typename T, int A, bool ODD>
__device__ __forceinline__ T *lp_ptr(const StepArgs &p, const Nbr &n, int wall, unsigned bits)
{
    int slot, idx;
    aa_address<A, ODD>(n, wall, bits, slot, idx);
    return static_cast<T *>(p.pop[slot]) + idx;
}

template <typename T, bool ODD, bool CONSTQ, int TEX>
__global__ void __launch_bounds__(128, 4) step_lp_kernel(const StepArgs p)
{
    using S = LpStore<T>;
    constexpr float iS = S::kInv;
    const long long step = *p.step_ctr;
    const double Gd = CONSTQ ? p.force[step & 1] : p.gx;
    const float G = (float)Gd;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.z;
    const int wall = plane_wall(p, z);
    const double *sh = p.shift + (size_t)(step & 1) * p.nz * 3 + z * 3;
    const double c0 = sh[0], c1 = sh[1], c2 = sh[2];
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
                links_cell<T, ODD, CONSTQ>(p, n, wall, cell_links(p.band_of, p.links, p.nx, p.ny, x, y, z), nullptr, 0,
                                          Gd, c0, c1, c2, acc, racc);
#pragma unroll
                for (int i = 0; i < NP; ++i) acc[i] += (double)racc[i];
                continue;
            }
            float d[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                T *q;
                switch (a) {
#define PT(A) case A: q = lp_ptr<T, A, ODD>(p, n, wall, bits); break;
                    PT(0) PT(1) PT(2) PT(3) PT(4) PT(5) PT(6) PT(7) PT(8) PT(9)
                    PT(10) PT(11) PT(12) PT(13) PT(14) PT(15) PT(16) PT(17) PT(18)
#undef PT
                }
                d[ODD ? lat_opp(a) : a] = S::ld(q);
            }
            const LpCell c = lp_collide<T>(d, p.omega, G);
            acc[0] += 1.0 + (double)c.drho;
            acc[1] += (double)c.jx;
            acc[2] += (double)c.u0;
            acc[3] += (double)c.u1;
            acc[4] += (double)c.u2;
            {
                const float d0 = c.u0 - (float)c0, d1 = c.u1 - (float)c1, d2 = c.u2 - (float)c2;
                acc[5] += (double)(d0 * d0 + d1 * d1 + d2 * d2);
            }
            if (CONSTQ) {
                float s = 0.f, m = 0.f;
#pragma unroll
                for (int a = 0; a < Q; ++a) {
                    s += d[a];
                    if (lat_ex(a)) m += lat_ex(a) > 0 ? d[a] : -d[a];
                }
                s *= iS;
                m *= iS;
                if (wall != 0) {
                    const int ap = wall < 0 ? 12 : 11, am = wall < 0 ? 13 : 14;
                    // a bounced link arrives with e_x reversed; its weight
                    // part w_a contributes -2 e_x w_a too
                    if (bits & 2u) m -= 2.f * (d[ap] * iS + 1.f / 36.f);
                    if (bits & 4u) m += 2.f * (d[am] * iS + 1.f / 36.f);
                }
                acc[6] += 1.0 + (double)s;
                acc[7] += (double)m;
            }
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                T *q;
                switch (a) {
#define PT(A) case A: q = lp_ptr<T, A, ODD>(p, n, wall, bits); break;
                    PT(0) PT(1) PT(2) PT(3) PT(4) PT(5) PT(6) PT(7) PT(8) PT(9)
                    PT(10) PT(11) PT(12) PT(13) PT(14) PT(15) PT(16) PT(17) PT(18)
#undef PT
                }
                S::st(q, d[ODD ? a : lat_opp(a)]);
            }
        }
    }
    block_epilogue(p, acc, step, Gd, 0);
}

template <typename T>
__global__ void __launch_bounds__(128) reduce_lp_kernel(const StepArgs p)
{
    using S = LpStore<T>;
    constexpr float iS = S::kInv;
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
            float dr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                const float v = S::ld(static_cast<const T *>(p.pop[a]) + c) * iS;
                dr += v;
                if (lat_ex(a)) jx += lat_ex(a) > 0 ? v : -v;
                if (lat_ey(a)) jy += lat_ey(a) > 0 ? v : -v;
                if (lat_ez(a)) jz += lat_ez(a) > 0 ? v : -v;
            }
            const double rho = 1.0 + (double)dr;
            acc[0] += rho;
            acc[1] += (double)jx;
            acc[2] += (double)jx / rho;
            acc[3] += (double)jy / rho;
            acc[4] += (double)jz / rho;
        }
    }
    block_epilogue(p, acc, step, 0.0, 1);
}

template <typename T>
static void launch_lp(const StepArgs &p, dim3 grid, dim3 block, bool odd, int tex, cudaStream_t s)
{
    const bool q = p.const_q != 0;
#define L(O, C, X) step_lp_kernel<T, O, C, X><<<grid, block, 0, s>>>(p)
#define LX(O, C) do { if (tex == 2) L(O, C, 2); else if (tex) L(O, C, 1); else L(O, C, 0); } while (0)
    if (odd) {
        if (q) LX(true, true); else LX(true, false);
    } else {
        if (q) LX(false, true); else LX(false, false);
    }
#undef LX
#undef L
}

void launch_step_lp(int precision, const StepArgs &p, dim3 grid, dim3 block, bool odd, int tex, cudaStream_t s)
{
    if (precision == 32) launch_lp<float>(p, grid, block, odd, tex, s);
    else launch_lp<__half>(p, grid, block, odd, tex, s);
}

void launch_reduce_lp(int precision, const StepArgs &p, dim3 grid, dim3 block, cudaStream_t s)
{
    if (precision == 32) reduce_lp_kernel<float><<<grid, block, 0, s>>>(p);
    else reduce_lp_kernel<__half><<<grid, block, 0, s>>>(p);
}

}  // namespace dnslbm
