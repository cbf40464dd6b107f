// Cells of the planes next to solids inside the flow (boundary mode
// DNSLBM_BC_GENERAL: riblets, bars, blocks).  Such a plane carries a per-cell
// link mask (cell_links, step_common.cuh) and its cells move every
// population by a per-thread access: a bounced link's address is a slot of
// the cell's own row that the bulk row of another direction would also
// cover, so these planes are left out of the row-pipelined kernel and
// stepped by links_pass_kernel (below) right after it, or by the per-thread
// step kernels.  Solid cells are never collided: they keep the rest state,
// and their stored populations enter the plane sums as they are, so the sums
// run over every cell of the plane like the reference's encalc / wshearstr /
// statistics loops.
#pragma once

#include <type_traits>
#include <utility>

#include "collide_f64.cuh"
#include "collide_lp.cuh"
#include "step_common.cuh"

namespace dnslbm {

template <typename T>
using RegT = typename std::conditional<std::is_same<T, double>::value, double, float>::type;

template <typename T>
__device__ __forceinline__ RegT<T> ld_raw(const T *q)
{
    if constexpr (std::is_same<T, double>::value) return *q;
    else return LpStore<T>::ld(q);
}
// Global-memory load that bypasses L1 (ld.global.cg): a population that
// another SM wrote earlier in the same launch (the persistent batch kernel
// runs many steps in one launch) is read from L2, never from a stale L1 line.
template <typename T>
__device__ __forceinline__ RegT<T> ld_glb(const T *q)
{
    if constexpr (std::is_same<T, __half>::value) return __half2float(__ldcg(q));
    else return __ldcg(q);
}
template <typename T>
__device__ __forceinline__ void st_raw(T *q, RegT<T> v)
{
    if constexpr (std::is_same<T, double>::value) *q = v;
    else LpStore<T>::st(q, v);
}

// f(std::integral_constant<int, I>) for I = 0 .. N-1, unrolled at compile time
template <typename F, int... I>
__device__ __forceinline__ void static_for_impl(F &f, std::integer_sequence<int, I...>)
{
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F &&f)
{
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// Address of link A of a (fluid) cell with link mask lk: the rule of
// aa_address_links, written with compile-time slot indices only so the
// population pointers stay in registers.
template <typename T, int A>
__device__ __forceinline__ T *links_ptr(const StepArgs &p, const Nbr &n, int wall, unsigned lk)
{
    constexpr int ex = lat_ex(A), ey = lat_ey(A), ez = lat_ez(A);
    if constexpr (A == 0) {
        return static_cast<T *>(p.pop[0]) + n.c0;
    } else {
        if ((lk >> A) & 1u) return static_cast<T *>(p.pop[lat_opp(A)]) + n.c0;
        if constexpr (ez != 0)
            if (wall == ez) return static_cast<T *>(p.pop[lat_mir(A)]) + n.row[ey + 1][1] + nbr_x(n, ex);
        return static_cast<T *>(p.pop[A]) + n.row[ey + 1][ez + 1] + nbr_x(n, ex);
    }
}

// Plane sums of a solid cell from its stored (rest) populations f.
template <typename T, bool CONSTQ>
__device__ __forceinline__ void solid_sums(const RegT<T> (&f)[Q], double c0, double c1, double c2, double (&acc)[NP],
                                           float (&racc)[NP])
{
    if constexpr (std::is_same<T, double>::value) {
        double dens, jx, jy, jz;
        f64_moments(f, dens, jx, jy, jz);
        const double u0 = jx / dens, u1 = jy / dens, u2 = jz / dens;
        acc[0] += dens;
        acc[1] += jx;
        acc[2] += u0;
        acc[3] += u1;
        acc[4] += u2;
        const double d0 = u0 - c0, d1 = u1 - c1, d2 = u2 - c2;
        acc[5] += d0 * d0 + d1 * d1 + d2 * d2;
        if (CONSTQ) {
            double s = 0.0, m = 0.0;
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                s += f[a];
                if (lat_ex(a) > 0) m += f[a];
                if (lat_ex(a) < 0) m -= f[a];
            }
            acc[6] += s;
            acc[7] += m;
        }
    } else {
        constexpr float iS = LpStore<T>::kInv;
        float dr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
        for (int a = 0; a < Q; ++a) {
            dr += f[a];
            if (lat_ex(a)) jx += lat_ex(a) > 0 ? f[a] : -f[a];
            if (lat_ey(a)) jy += lat_ey(a) > 0 ? f[a] : -f[a];
            if (lat_ez(a)) jz += lat_ez(a) > 0 ? f[a] : -f[a];
        }
        const float drho = dr * iS, inv = iS / (1.f + drho);
        const float u0 = jx * inv, u1 = jy * inv, u2 = jz * inv;
        acc[0] += 1.0;
        racc[0] += drho;
        racc[1] += jx * iS;
        racc[2] += u0;
        racc[3] += u1;
        racc[4] += u2;
        const float d0 = u0 - (float)c0, d1 = u1 - (float)c1, d2 = u2 - (float)c2;
        racc[5] += d0 * d0 + d1 * d1 + d2 * d2;
        if (CONSTQ) {
            acc[6] += 1.0;
            racc[6] += drho;
            racc[7] += jx * iS;
        }
    }
}

// One cell with link mask `lk` (plane `wall` = -1 bottom, +1 top, 0
// interior).  Even step: the cell's own populations, from shared memory at
// sbx[A * dstride] when sbx is given (the bulk-copied own rows), else from
// global memory.  Odd step: global memory through the link addresses, except
// that with sbx given (the bulk-copied rows of the odd address set, element
// x at sbx, x - 1 at sbx + om, x + 1 at sbx + op) a link that neither
// bounces nor meets a wall is read from shared memory; the odd step's
// results always go to global memory.
// FP64 sums go to acc; low-precision sums go to racc (FP32, flushed by the
// caller) except the cell counts, which go to acc[0] and acc[6].
template <typename T, bool ODD, bool CONSTQ>
__device__ __forceinline__ void links_cell(const StepArgs &p, const Nbr &n, int wall, unsigned lk, T *sbx, int dstride,
                                           double G, double c0, double c1, double c2, double (&acc)[NP],
                                           float (&racc)[NP], int om = 0, int op = 0)
{
    using V = RegT<T>;
    if (lk & 1u) {
        // a solid cell holds the (symmetric) rest state in its own slots
        V f[Q];
#pragma unroll
        for (int A = 0; A < Q; ++A)
            f[A] = (!ODD && sbx) ? ld_raw<T>(sbx + A * dstride) : ld_glb<T>(static_cast<const T *>(p.pop[A]) + n.c0);
        solid_sums<T, CONSTQ>(f, c0, c1, c2, acc, racc);
        return;
    }
    V f[Q];
    static_for<Q>([&](auto ac) {
        constexpr int A = decltype(ac)::value;
        V v;
        constexpr int ex = lat_ex(A), ez = lat_ez(A);
        if (!ODD && sbx) v = ld_raw<T>(sbx + A * dstride);
        else if (!ODD) v = ld_glb<T>(static_cast<const T *>(p.pop[A]) + n.c0);
        else if (sbx && !((lk >> A) & 1u) && !(ez != 0 && wall == ez))
            v = ld_raw<T>(sbx + A * dstride + (ex > 0 ? op : (ex < 0 ? om : 0)));
        else v = ld_glb<T>(links_ptr<T, A>(p, n, wall, lk));
        f[ODD ? lat_opp(A) : A] = v;
    });
    if constexpr (std::is_same<T, double>::value) {
        const F64Cell c = f64_collide(f, p.omega, G);
        acc[0] += c.dens;
        acc[1] += c.jx;
        acc[2] += c.u0;
        acc[3] += c.u1;
        acc[4] += c.u2;
        const double d0 = c.u0 - c0, d1 = c.u1 - c1, d2 = c.u2 - c2;
        acc[5] += d0 * d0 + d1 * d1 + d2 * d2;
        if (CONSTQ) {
            double s = 0.0, m = 0.0;
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                s += f[a];
                if (lat_ex(a) > 0) m += f[a];
                if (lat_ex(a) < 0) m -= f[a];
            }
            // links that bounce back arrive with e_x reversed
#pragma unroll
            for (int a = 1; a < Q; ++a)
                if (lat_ex(a) != 0 && ((lk >> a) & 1u)) m += lat_ex(a) > 0 ? -2. * f[a] : 2. * f[a];
            acc[6] += s;
            acc[7] += m;
        }
    } else {
        constexpr float iS = LpStore<T>::kInv;
        const LpCell c = lp_collide<T>(f, (float)p.omega, (float)G);
        acc[0] += 1.0;
        racc[0] += c.drho;
        racc[1] += c.jx;
        racc[2] += c.u0;
        racc[3] += c.u1;
        racc[4] += c.u2;
        const float d0 = c.u0 - (float)c0, d1 = c.u1 - (float)c1, d2 = c.u2 - (float)c2;
        racc[5] += d0 * d0 + d1 * d1 + d2 * d2;
        if (CONSTQ) {
            float s = 0.f, m = 0.f;
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                s += f[a];
                if (lat_ex(a)) m += lat_ex(a) > 0 ? f[a] : -f[a];
            }
            s *= iS;
            m *= iS;
            // a bounced link carries -2 e_x (w + d)
#pragma unroll
            for (int a = 1; a < Q; ++a)
                if (lat_ex(a) != 0 && ((lk >> a) & 1u)) {
                    const float full = f[a] * iS + lat_wf(a);
                    m += lat_ex(a) > 0 ? -2.f * full : 2.f * full;
                }
            acc[6] += 1.0;
            racc[6] += s;
            racc[7] += m;
        }
    }
    static_for<Q>([&](auto ac) {
        constexpr int A = decltype(ac)::value;
        const V v = f[ODD ? A : lat_opp(A)];
        if (!ODD && sbx) st_raw<T>(sbx + A * dstride, v);
        else if (!ODD) st_raw<T>(static_cast<T *>(p.pop[A]) + n.c0, v);
        else st_raw<T>(links_ptr<T, A>(p, n, wall, lk), v);
    });
}

// ------------------------------------------------------------------ pass
// The planes with link masks of one or more channels, one thread per x and
// `rows` rows per block (the per-thread kernels' block shape, so a plane has
// as many contributors as there are partial-sum slots).  It runs as the
// second launch of a step, after the row-pipelined kernel has done the
// other planes; the last plane to finish runs the step tail.
struct LinksLaunch {
    StepArgs p;
    const int *planes;  // the channel's planes with link masks
    int nplanes;
    int xblocks, yblocks, rows;
    int first_block;    // first block of the channel in the launch
};

template <typename T, bool ODD, bool CONSTQ>
__device__ __forceinline__ void links_pass_body(const LinksLaunch &L, int blk)
{
    const StepArgs &p = L.p;
    const int per_plane = L.xblocks * L.yblocks;
    const int pi = blk / per_plane, r = blk - pi * per_plane;
    const int by = r / L.xblocks, bx = r - by * L.xblocks;
    const int z = L.planes[pi];
    const int wall = plane_wall(p, z);
    const long long step = *p.step_ctr;
    const double G = CONSTQ ? p.force[step & 1] : p.gx;
    const double *sh = p.shift + (size_t)(step & 1) * p.nz * 3 + z * 3;
    const double c0 = sh[0], c1 = sh[1], c2 = sh[2];
    double acc[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i] = 0.0;
    const int x = bx * blockDim.x + threadIdx.x;
    if (x < p.nx) {
        const int y0 = by * L.rows, y1 = min(y0 + L.rows, p.ny);
        for (int y = y0; y < y1; ++y) {
            float racc[NP];
#pragma unroll
            for (int i = 0; i < NP; ++i) racc[i] = 0.f;
            const Nbr n = make_nbr(x, y, z, p.nx, p.ny, p.pitch);
            links_cell<T, ODD, CONSTQ>(p, n, wall, cell_links(p.band_of, p.links, p.nx, p.ny, x, y, z), nullptr, 0,
                                       G, c0, c1, c2, acc, racc);
#pragma unroll
            for (int i = 0; i < NP; ++i) acc[i] += (double)racc[i];
        }
    }
    plane_contribute(p, acc, z, r, per_plane, step, G, 0, blockDim.x);
}

constexpr int kLinksThreads = 128;

template <typename T, bool ODD>
__global__ void __launch_bounds__(kLinksThreads) links_pass_kernel(const LinksLaunch *__restrict__ tab, int n)
{
    __shared__ LinksLaunch L;
    __shared__ int s_c;
    if (threadIdx.x == 0) {
        int c = 0;
        while (c + 1 < n && tab[c + 1].first_block <= (int)blockIdx.x) ++c;
        s_c = c;
    }
    __syncthreads();
    {
        const int *src = reinterpret_cast<const int *>(tab + s_c);
        int *dst = reinterpret_cast<int *>(&L);
        for (int i = threadIdx.x; i < (int)(sizeof(LinksLaunch) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const int blk = blockIdx.x - L.first_block;
    if (L.p.const_q) links_pass_body<T, ODD, true>(L, blk);
    else links_pass_body<T, ODD, false>(L, blk);
}

template <typename T>
void launch_links_pass(const LinksLaunch *tab, int n, int blocks, bool odd, cudaStream_t s)
{
    if (odd) links_pass_kernel<T, true><<<blocks, kLinksThreads, 0, s>>>(tab, n);
    else links_pass_kernel<T, false><<<blocks, kLinksThreads, 0, s>>>(tab, n);
}

}  // namespace dnslbm
