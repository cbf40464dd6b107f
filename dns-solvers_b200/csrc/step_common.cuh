// Shared machinery of the fused step kernels: launch arguments, the AA
// address set of a cell (with periodic wrap and wall links), the
// deterministic block/plane/grid reduction, and the per-step tail that turns
// per-plane sums into the encalc/wshearstr log record and the next force.
#pragma once

#include <cuda_runtime.h>

#include "lattice.cuh"

namespace dnslbm {

// Per-block partial sums.  Reader side (state at the start of the step):
//   0 sum rho, 1 sum jx (raw momentum), 2..4 sum u,v,w (u = j/rho),
//   5 sum |u - c(z)|^2 with c(z) the previous plane means (a shift that keeps
//     the one-pass variance free of cancellation).
// Writer side (state after the step, constant-Q only):
//   6 sum of post-collision populations, 7 their x-momentum as received
//     (bounce-back flips e_x, specular reflection keeps it).
constexpr int NP = 8;

struct StepArgs {
    void *pop[Q];            // population arrays (slot a)
    int nx, ny, nz;
    int pitch;               // row pitch in elements (>= nx)
    int rows;                // rows (y) per block (scalar kernels)
    int slots;               // partial-sum slots per plane
    const uint8_t *wallmask; // [2][ny][nx] wall-link bits (bottom, top)
    double omega, ubulk, gx;
    int const_q;
    double *force;           // [2] force of step s is force[s & 1]
    double *shift;           // [2][nz][3] plane means of the previous state
    long long *step_ctr;     // steps done (advanced by the step tail)
    double *partials;        // [nz][slots][NP]
    double *plane_sums;      // [nz][NP]
    unsigned *plane_ctr;     // [nz]
    unsigned *total_ctr;     // [1]
    double *logs;            // [log_cap][9]
    int log_cap;
    long long *status;       // [0] first NaN step + 1 (0: none), [1] a bounded wait gave up
    // solids inside the flow (general boundary mode): planes within one
    // plane of a solid cell carry a per-cell link mask, see cell_links
    const int *band_of;      // [nz] index of the plane's mask block, -1: none
    const unsigned *links;   // [nband][ny][nx]
    // bounded waits of the row-pipelined kernels: a wait gives up after
    // wait_ns of the GPU's global timer (status[1] set); withhold_stage is a
    // test switch (0 otherwise) that makes one block withhold a load
    unsigned long long wait_ns;
    int withhold_stage;
    // wall-normal slab of a channel split over several GPUs: wall_lo /
    // wall_hi say whether plane 0 / nz-1 lies next to the bottom / top wall
    // (else next to a ghost plane, z = -1 / nz, that mirrors the neighbour
    // slab); tail = 0 leaves the plane sums to the caller instead of running
    // the step tail (whole channels: 1, 1, 1)
    int wall_lo = 1, wall_hi = 1;
    int tail = 1;
};

// -1: plane z lies next to the bottom wall, +1: next to the top wall, 0:
// between fluid planes (a ghost plane of a slab included)
__device__ __forceinline__ int plane_wall(const StepArgs &p, int z)
{
    return (z == 0 && p.wall_lo) ? -1 : ((z == p.nz - 1 && p.wall_hi) ? 1 : 0);
}

// Arguments of the state readers/writers (import, export, moments, stats).
struct IoArgs {
    void *pop[Q];
    int nx, ny, nz;
    int pitch;  // row pitch in elements
    const uint8_t *wallmask;
    int textured;  // 0 smooth walls, 1 textured walls, 2 solids inside the flow
    int odd;  // 1: populations are post-collision in swapped slots
    const int *band_of;
    const unsigned *links;
};

// Link mask of a cell in a plane next to a solid inside the flow
// (boundary mode DNSLBM_BC_GENERAL): bit 0 set for a solid cell (never
// collided, holds the rest state), bit A (1..18) set when the link from the
// cell in direction A bounces back -- into a solid cell, into a no-slip wall
// cell whose own wall cell is no-slip too, or a specular reflection whose
// target cell is solid.  A clear bit of a link into a wall plane means
// specular reflection; every other clear bit is plain streaming.  Cells of
// planes without a mask block have no solid neighbour (0).
__device__ __forceinline__ unsigned cell_links(const int *band_of, const unsigned *links, int nx, int ny, int x,
                                               int y, int z)
{
    const int b = band_of[z];
    return b < 0 ? 0u : links[((size_t)b * ny + y) * nx + x];
}

// ---------------------------------------------------------------- addresses
// Neighbourhood of a cell: wrapped x and the 9 row offsets (dy, dz).
struct Nbr {
    int x, xm, xp;
    int row[3][3];  // row[dy+1][dz+1] = ((z+dz)*ny + wrap(y+dy))*pitch
    int c0;         // own cell
};

__device__ __forceinline__ Nbr make_nbr(int x, int y, int z, int nx, int ny, int pitch)
{
    Nbr n;
    n.x = x;
    n.xm = x == 0 ? nx - 1 : x - 1;
    n.xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1;
    const int yp = y == ny - 1 ? 0 : y + 1;
    const int ys[3] = {ym, y, yp};
#pragma unroll
    for (int dy = 0; dy < 3; ++dy)
#pragma unroll
        for (int dz = 0; dz < 3; ++dz) n.row[dy][dz] = ((z + dz - 1) * ny + ys[dy]) * pitch;
    n.c0 = n.row[1][1] + x;
    return n;
}

__device__ __forceinline__ int nbr_x(const Nbr &n, int ex) { return ex == 0 ? n.x : ex > 0 ? n.xp : n.xm; }

// Element index (within population array `slot`) of the A-th address of the
// cell, and the slot it lives in.
//   even: slot A at the cell; load -> f[A], store <- f*[opp A]
//   odd:  slot A at cell + e_A; load -> f[opp A], store <- f*[A]
// Odd step, wall plane, A pointing into the wall: bounce-back uses slot
// opp(A) at the cell, specular reflection slot mirror(A) at the tangential
// neighbour (cell + (ex, ey, 0)).  `wall` is -1 (bottom plane), +1 (top
// plane) or 0; `bits` are the cell's wall-link bits.
template <int A, bool ODD>
__device__ __forceinline__ void aa_address(const Nbr &n, int wall, unsigned bits, int &slot, int &idx)
{
    constexpr int ex = lat_ex(A), ey = lat_ey(A), ez = lat_ez(A);
    if (!ODD || A == 0) {
        slot = A;
        idx = n.c0;
        return;
    }
    if (ez != 0 && wall == ez) {
        if ((bits >> wall_link(A)) & 1u) {
            slot = lat_opp(A);
            idx = n.c0;
        } else {
            slot = lat_mir(A);
            idx = n.row[ey + 1][1] + nbr_x(n, ex);
        }
        return;
    }
    slot = A;
    idx = n.row[ey + 1][ez + 1] + nbr_x(n, ex);
}

// The same with a per-cell link mask (boundary mode DNSLBM_BC_GENERAL, a
// cell that is not solid): bounce-back to slot opp(A) of the cell, specular
// reflection for the other links into a wall plane, else plain streaming.
template <int A, bool ODD>
__device__ __forceinline__ void aa_address_links(const Nbr &n, int wall, unsigned links, int &slot, int &idx)
{
    constexpr int ex = lat_ex(A), ey = lat_ey(A), ez = lat_ez(A);
    if (!ODD || A == 0) {
        slot = A;
        idx = n.c0;
    } else if ((links >> A) & 1u) {
        slot = lat_opp(A);
        idx = n.c0;
    } else if (ez != 0 && wall == ez) {
        slot = lat_mir(A);
        idx = n.row[ey + 1][1] + nbr_x(n, ex);
    } else {
        slot = A;
        idx = n.row[ey + 1][ez + 1] + nbr_x(n, ex);
    }
}

// ---------------------------------------------------------------- reduction
template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV])
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] += __shfl_down_sync(0xffffffffu, v[i], off);
}

// Barrier over the first `nthreads` threads of the block (all of them when
// nthreads == blockDim.x): named barrier 1, so a producer warp outside the
// group never has to take part.
__device__ __forceinline__ void group_sync(int nthreads)
{
    if (nthreads == (int)blockDim.x) __syncthreads();
    else asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// Deterministic sum over the first `nthreads` threads (fixed shuffle tree,
// warps added in order); the result is valid in thread 0.  smem holds
// 32*NV doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem, int nthreads)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarp = (nthreads + 31) >> 5;
    warp_sum<NV>(v);
    group_sync(nthreads);
    if (lane == 0)
#pragma unroll
        for (int i = 0; i < NV; ++i) smem[warp * NV + i] = v[i];
    group_sync(nthreads);
    if (warp == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] = lane < nwarp ? smem[lane * NV + i] : 0.0;
        warp_sum<NV>(v);
    }
}

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem)
{
    block_sum<NV>(v, smem, blockDim.x);
}

// Final step tail, run by the last block of the launch: plane sums ->
// per-step log record, the plane means (next TKE shift) and, in constant-Q
// mode, the force of the next step from the writer-side totals.
// mode 0: after a step (logs, advances the step counter);
// mode 1: initial reduction of a freshly loaded state (force and shift of
//         the current step from the reader-side totals, nothing logged).
// step < 0 (mode 0): the step is read from the step counter (the tail is
// its only writer, once per step).
static __device__ __forceinline__ void step_tail(const StepArgs &a, long long step, double force_used, int mode, double *smem,
                                                 int nthreads)
{
    if (step < 0) step = __ldcg(a.step_ctr);
    const int nz = a.nz;
    const double np = (double)a.nx * (double)a.ny;
    const double *cshift = a.shift + (size_t)(step & 1) * nz * 3;
    double *nshift = a.shift + (size_t)((mode == 0 ? step + 1 : step) & 1) * nz * 3;
    double t[6] = {0, 0, 0, 0, 0, 0};  // rho, jx, sum of plane means u, K, writer rho, writer jx
    for (int z = threadIdx.x; z < nz; z += nthreads) {
        const double *ps = a.plane_sums + (size_t)z * NP;
        double s[NP];
#pragma unroll
        for (int i = 0; i < NP; ++i) s[i] = __ldcg(ps + i);
        const double um = s[2] / np, vm = s[3] / np, wm = s[4] / np;
        const double du = um - __ldcg(cshift + z * 3 + 0), dv = vm - __ldcg(cshift + z * 3 + 1),
                     dw = wm - __ldcg(cshift + z * 3 + 2);
        t[0] += s[0];
        t[1] += s[1];
        t[2] += um;
        t[3] += 0.5 * (s[5] - np * (du * du + dv * dv + dw * dw));
        t[4] += s[6];
        t[5] += s[7];
        nshift[z * 3 + 0] = um;
        nshift[z * 3 + 1] = vm;
        nshift[z * 3 + 2] = wm;
    }
    block_sum<6>(t, smem, nthreads);
    if (threadIdx.x != 0) return;
    const double N = np * (double)nz;
    const double rho = t[0] / N, momentum = t[1] / N;
    if (mode == 1) {
        a.force[step & 1] = a.const_q ? rho * a.ubulk - momentum : a.gx;
        return;
    }
    // wall shear stress, wshearstr.c:24-121 (top density from plane zd-4)
    auto umean = [&](int z) { return __ldcg(a.plane_sums + (size_t)z * NP + 2) / np; };
    const double mu = (1. / 6.) * (2. / a.omega - 1);
    const double davg_dn = __ldcg(a.plane_sums + 0 * NP + 0) / np;
    const double davg_up = __ldcg(a.plane_sums + (size_t)(nz - 3) * NP + 0) / np;
    double stdown = -2. * umean(0) + 3. * umean(1) - umean(2);
    double stup = -(2. * umean(nz - 1) - 3. * umean(nz - 2) + umean(nz - 3));
    stdown *= mu * davg_dn;
    stup *= mu * davg_up;
    const double stress = 0.5 * (stup + stdown);
    double *rec = a.logs + (size_t)(step % a.log_cap) * 9;
    rec[0] = force_used;
    rec[1] = rho;
    rec[2] = t[3] / N;
    rec[3] = (t[2] / (double)nz) * (double)(a.ny * nz);
    rec[4] = momentum * (double)(a.ny * nz);
    rec[5] = stup;
    rec[6] = stdown;
    rec[7] = stress;
    rec[8] = force_used * nz / 2.;
    if (stress != stress && __ldcg(a.status) == 0) a.status[0] = step + 1;
    // constant-Q: next force from the totals of the state this step wrote
    // (encalc.c:121 evaluated one step ahead); sum of populations = t[4]
    a.force[(step + 1) & 1] = a.const_q ? (t[4] / N) * a.ubulk - t[5] / N : a.gx;
    *a.step_ctr = step + 1;
}

// One block's contribution to plane z: block partials -> (last contributor
// of the plane) plane sums in a fixed order -> (last plane) step tail.  No
// block waits for another: the last arrival does the work, found with atomic
// tickets.  `slot` numbers the block among the `ncontrib` contributors of
// the plane; the call is block-uniform.
__device__ __forceinline__ void plane_contribute(const StepArgs &a, double (&acc)[NP], int z, int slot, int ncontrib,
                                                 long long step, double force_used, int mode, int nthreads)
{
    __shared__ double smem[32 * NP];
    __shared__ unsigned ticket;
    block_sum<NP>(acc, smem, nthreads);
    if (threadIdx.x == 0) {
        double *p = a.partials + ((size_t)z * a.slots + slot) * NP;
#pragma unroll
        for (int i = 0; i < NP; ++i) p[i] = acc[i];
        __threadfence();
        ticket = atomicAdd(a.plane_ctr + z, 1u);
    }
    group_sync(nthreads);
    if (ticket != (unsigned)ncontrib - 1) return;
    // last contributor of plane z: fixed-order plane sum
    __threadfence();
    double s[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) s[i] = 0.0;
    for (int b = threadIdx.x; b < ncontrib; b += nthreads) {
        const double *p = a.partials + ((size_t)z * a.slots + b) * NP;
#pragma unroll
        for (int i = 0; i < NP; ++i) s[i] += __ldcg(p + i);
    }
    block_sum<NP>(s, smem, nthreads);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NP; ++i) a.plane_sums[(size_t)z * NP + i] = s[i];
        a.plane_ctr[z] = 0;
        __threadfence();
        ticket = atomicAdd(a.total_ctr, 1u);
    }
    group_sync(nthreads);
    if (ticket != (unsigned)a.nz - 1) return;
    __threadfence();
    if (a.tail) step_tail(a, step, force_used, mode, smem, nthreads);
    if (threadIdx.x == 0) *a.total_ctr = 0;
    group_sync(nthreads);
}

// Epilogue of the scalar kernels: one block per (x-chunk, row-chunk) of a
// plane, blockIdx.z = plane.
__device__ __forceinline__ void block_epilogue(const StepArgs &a, double (&acc)[NP], long long step, double force_used,
                                               int mode)
{
    const int bpp = gridDim.x * gridDim.y;
    plane_contribute(a, acc, blockIdx.z, blockIdx.y * gridDim.x + blockIdx.x, bpp, step, force_used, mode, blockDim.x);
}

}  // namespace dnslbm
