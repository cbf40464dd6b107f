// Row-pipelined fused step on the Blackwell bulk-copy engine.
//
// A block owns a contiguous range of cell rows (y, z) (x runs along the
// row).  In the AA scheme the 19 addresses of a cell are, per direction A,
// one element of one population row: for the whole cell row they are 19
// complete rows of the population arrays (row (y+ey, z+ez) of slot A in an
// odd step, row (y, z) of slot A in an even step), which no other cell row
// touches.  The block is warp-specialised:
//   * the last warp is the producer: lane A moves direction A's row --
//     a cp.async.bulk load into a shared-memory stage (completing on the
//     stage's "full" mbarrier), and, once the consumers release the stage
//     (its "empty" mbarrier), the cp.async.bulk store of the updated row;
//     `stages` rows are in flight per block;
//   * the other warps are consumers: they collide every cell of the row,
//     reading direction A at x + ex (the periodic wrap in x is a
//     shared-memory index) and writing the result back to the same
//     shared-memory element, then release the stage.
// Rows are padded to a 16-byte pitch so every copy is aligned.  No consumer
// computes a global address on the interior path, and no consumer ever waits
// for the producer's copy issue or store completion.
//
// Wall rows of an odd step: with smooth walls a link into the wall bounces
// back to the cell's own slot opp(A), again a whole own row (bulk).  With a
// textured wall the five links into the wall go to rows that several cell
// rows share (bounce-back or specular per cell), so those five are moved by
// per-thread loads/stores and never by a bulk copy.  Planes next to solids
// inside the flow are not in this kernel's plane list: a second launch of
// the same step (links_pass_kernel, step_links.cuh) moves them per thread.
//
// TEX: 0 smooth walls, 1 textured walls.
//
// Every wait on an mbarrier is bounded in time (StepArgs::wait_ns of the
// GPU's global timer); a wait that runs out records status[1] and a shared
// abort flag, after which no thread of the block waits again except the
// producer for the copies it has already issued (the host reports
// DNSLBM_ERR_TIMEOUT).
#pragma once

#include <cuda_fp16.h>

#include <type_traits>

#include "collide_f64.cuh"
#include "collide_lp.cuh"
#include "step_common.cuh"
#include "step_links.cuh"

namespace dnslbm {

struct TmaArgs {
    int ngroups;          // row groups: nz * gpp
    int groups_per_block; // contiguous row groups per block
    int stages;           // row groups in flight per block
    int row_bytes;        // pitch * sizeof(storage)
    int k;                // cell rows per group (consecutive y of one plane)
    int gpp;              // groups per plane, ceil(ny / k) * nseg
    const int *planes;    // planes of the kernel's groups in order (nullptr: 0 .. nz-1)
    // x-segments (FP64 rows too long for two whole-row stages): a group is
    // one x-segment [s*seg, min((s+1)*seg, nx)) of one row (k = 1), seg even
    int nseg, seg;
    int dir_elems;        // elements between two directions' blocks of a stage
};

// Plane and first row of row group gi.
__device__ __forceinline__ void group_origin(const TmaArgs &t, int gi, int &z, int &y0)
{
    const int pi = gi / t.gpp;
    z = t.planes ? t.planes[pi] : pi;
    y0 = ((gi - pi * t.gpp) / t.nseg) * t.k;
}

// x-range of row group gi.
__device__ __forceinline__ void group_xrange(const TmaArgs &t, int gi, int nx, int &x0, int &x1)
{
    const int s = (gi % t.gpp) % t.nseg;
    x0 = s * t.seg;
    x1 = t.nseg > 1 ? min(x0 + t.seg, nx) : nx;
}

// ------------------------------------------------------------------ PTX
__device__ __forceinline__ uint32_t sm_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sm_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sm_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(sm_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     sm_addr(dst)),
                 "l"(src), "r"(bytes), "r"(sm_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void bulk_s2g(void *dst, const void *src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(sm_addr(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of an mbarrier for at most limit_ns nanoseconds of
// the GPU's global timer, or until another thread of the block has raised
// the abort flag (none when abort is null).  Returns false when the wait
// gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, unsigned long long limit_ns,
                                                  volatile int *abort)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((abort && *abort) || globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// ------------------------------------------------------------------ rows
// Row group g = cell rows y0 .. y0+k-1 of plane z.  Direction A's
// shared-memory block holds the k population rows of A's address set, in
// order of the cell rows: rows y0+j+ey (periodic in y) of plane z+ez and slot
// A in an odd step, rows y0+j of plane z and slot A in an even step, or the
// cell rows' own rows of slot opp(A) for a smooth-wall bounce-back.  In
// memory they are contiguous except where the y index wraps, so a direction
// needs one copy, or two at the wrap.  `bulk` is false for the textured wall
// links of an odd step, which move per thread.
struct GroupRows {
    int slot, zz;     // population array and plane of the rows
    int y_first;      // first source row (j = 0), before wrapping
    bool bulk;
};

template <bool ODD, int TEX>
__device__ __forceinline__ GroupRows group_rows(const StepArgs &p, int A, int y0, int z, int wall)
{
    GroupRows g;
    const int ez = lat_ez(A);
    g.bulk = true;
    if (!ODD) {
        g.slot = A; g.zz = z; g.y_first = y0;
    } else if (ez != 0 && ez == wall) {
        g.bulk = TEX == 0;
        g.slot = lat_opp(A); g.zz = z; g.y_first = y0;  // bounce-back to the cell's own rows
    } else {
        g.slot = A; g.zz = z + ez; g.y_first = y0 + lat_ey(A);
    }
    return g;
}

// Issue the copies of one direction's rows (load: to_smem, else store).
template <typename T>
__device__ __forceinline__ void copy_group(const StepArgs &p, const TmaArgs &t, const GroupRows &g, int k,
                                           unsigned char *sdir, bool to_smem, uint64_t *bar)
{
    const int ny = p.ny;
    const size_t rb = (size_t)t.row_bytes;
    auto one = [&](int ysrc, int j, int nrows) {
        T *gp = static_cast<T *>(p.pop[g.slot]) + (ptrdiff_t)(g.zz * ny + ysrc) * p.pitch;
        unsigned char *sp = sdir + (size_t)j * rb;
        if (to_smem) bulk_g2s(sp, gp, (uint32_t)(nrows * rb), bar);
        else bulk_s2g(gp, sp, (uint32_t)(nrows * rb));
    };
    const int y = g.y_first;
    if (y < 0) {                    // j = 0 wraps to the last row
        one(ny - 1, 0, 1);
        if (k > 1) one(0, 1, k - 1);
    } else if (y + k > ny) {        // the last j wraps to row 0 (y <= ny)
        if (ny - y > 0) one(y, 0, ny - y);
        one(0, ny - y, k - (ny - y));
    } else {
        one(y, 0, k);
    }
}

// The bulk copies of one direction of an x-segment group [x0, x1) (k = 1).
// Shared memory holds element x of the row at index x - x0 + 2 (a halo of
// two elements on either side keeps every copy 16-byte aligned).  The load
// brings [x0, x0 + Lp), Lp = L rounded up to even (the row padding covers
// the last segment's odd end).  A direction shifted by e_x = +1 in an odd
// step writes elements x0+1 .. x1; a 16-byte aligned store can start at
// x0+2 and covers E = (L-1) rounded down to even elements; shifted by -1 it
// writes x0-1 .. x1-2 and the store covers [x0, x0+E).  The elements outside
// (at most two per segment and direction) are written by their cells
// directly (tma_group, SEG).
template <typename T>
__device__ __forceinline__ void copy_segment(const StepArgs &p, const GroupRows &g, int x0, int x1, int shift,
                                             unsigned char *sdir, bool to_smem, uint64_t *bar)
{
    const int ny = p.ny, L = x1 - x0, Lp = (L + 1) & ~1;
    int y = g.y_first;
    y = y < 0 ? y + ny : (y >= ny ? y - ny : y);
    T *row = static_cast<T *>(p.pop[g.slot]) + (ptrdiff_t)(g.zz * ny + y) * p.pitch;
    if (to_smem) {
        bulk_g2s(sdir + 2 * sizeof(T), row + x0, (uint32_t)(Lp * sizeof(T)), bar);
        return;
    }
    const int E = (L - 1) & ~1;
    const int start = shift > 0 ? x0 + 2 : x0, cnt = shift != 0 ? E : Lp;
    if (cnt > 0) bulk_s2g(row + start, sdir + (size_t)(start - x0 + 2) * sizeof(T), (uint32_t)(cnt * sizeof(T)));
}

// ------------------------------------------------------------------ cells
// The k cell rows of a row group from the stage buffer: direction A's
// element x of row j at sb[A * dstride + j * pitch + x].  The group's k * nx
// cells are spread over the nc consumer threads as one range, so rows
// shorter than the consumer set keep every thread busy.
// WALL: 0 interior plane, -1 bottom plane, +1 top plane.
// SEG: the group is the x-segment [x0, x1) of one row (k = 1), element x at
// shared-memory index x - x0 + 2; the segment's two edge cells move their
// e_x-shifted directions of an odd step through global memory (the element
// may lie outside the segment's copies), and into shared memory too where
// the segment's bulk store will write it.
template <typename T, bool ODD, bool CONSTQ, bool TEXTURED, int WALL, bool SEG = false>
__device__ __forceinline__ void tma_group(const StepArgs &p, T *sb, int dstride, int y0, int k, int z, double G,
                                          const double *shift, double (&acc)[NP], int nc, int x0 = 0, int x1 = -1)
{
    using V = RegT<T>;
    const double c0 = shift[0], c1 = shift[1], c2 = shift[2];
    const int nx = p.nx, pitch = p.pitch;
    if (!SEG) x0 = 0, x1 = nx;
    const int sxoff = SEG ? 2 - x0 : 0;  // shared-memory index of element x: x + sxoff
    // low precision: the thread's cells of the group are summed in FP32 (the
    // cell count too), then added to the FP64 accumulators
    float racc[NP], ncell = 0.f;
#pragma unroll
    for (int i = 0; i < NP; ++i) racc[i] = 0.f;
    // one cell (row j of the group, column x)
    auto cell = [&](int j, int x) {
        const int y = y0 + j;
        T *sbj = sb + (size_t)j * pitch + sxoff;
        const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
        const bool edge = SEG && ODD && (x == x0 || x == x1 - 1);
        // global element of an e_x-shifted direction A of an odd step (edge cells)
        auto shifted_ptr = [&](int A, int xs) {
            int yy = y + lat_ey(A);
            yy = yy < 0 ? yy + p.ny : (yy >= p.ny ? yy - p.ny : yy);
            return static_cast<T *>(p.pop[A]) + ((ptrdiff_t)(z + lat_ez(A)) * p.ny + yy) * pitch + xs;
        };
        unsigned bits = 0x1fu;
        if (TEXTURED && WALL != 0) bits = p.wallmask[(size_t)(WALL > 0) * nx * p.ny + (size_t)y * nx + x];
        Nbr n;
        if (TEXTURED && ODD && WALL != 0) n = make_nbr(x, y, z, nx, p.ny, pitch);
        V f[Q];
#pragma unroll
        for (int A = 0; A < Q; ++A) {
            constexpr bool kOdd = ODD;
            const bool wdir = kOdd && lat_ez(A) != 0 && lat_ez(A) == WALL;
            V v;
            if (TEXTURED && wdir) {
                int slot, idx;
                switch (A) {
#define AD(K) case K: aa_address<K, true>(n, WALL, bits, slot, idx); break;
                    AD(0) AD(1) AD(2) AD(3) AD(4) AD(5) AD(6) AD(7) AD(8) AD(9)
                    AD(10) AD(11) AD(12) AD(13) AD(14) AD(15) AD(16) AD(17) AD(18)
#undef AD
                }
                v = ld_glb<T>(static_cast<const T *>(p.pop[slot]) + idx);
            } else {
                const int xs = (ODD && !wdir) ? (lat_ex(A) > 0 ? xp : (lat_ex(A) < 0 ? xm : x)) : x;
                if (SEG && edge && !wdir && lat_ex(A) != 0) v = ld_glb<T>(shifted_ptr(A, xs));
                else v = ld_raw<T>(sbj + A * dstride + xs);
            }
            f[ODD ? lat_opp(A) : A] = v;
        }
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
                if (WALL != 0) {  // bounced links arrive with e_x reversed
                    const int ap = WALL < 0 ? 12 : 11, am = WALL < 0 ? 13 : 14;
                    if (bits & 2u) m -= 2. * f[ap];
                    if (bits & 4u) m += 2. * f[am];
                }
                acc[6] += s;
                acc[7] += m;
            }
        } else {
            constexpr float iS = LpStore<T>::kInv;
            const LpCell c = lp_collide<T>(f, (float)p.omega, (float)G);
            ncell += 1.f;
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
                if (WALL != 0) {  // a bounced link carries -2 e_x (w + d)
                    const int ap = WALL < 0 ? 12 : 11, am = WALL < 0 ? 13 : 14;
                    if (bits & 2u) m -= 2.f * (f[ap] * iS + 1.f / 36.f);
                    if (bits & 4u) m += 2.f * (f[am] * iS + 1.f / 36.f);
                }
                racc[6] += s;
                racc[7] += m;
            }
        }
#pragma unroll
        for (int A = 0; A < Q; ++A) {
            constexpr bool kOdd = ODD;
            const bool wdir = kOdd && lat_ez(A) != 0 && lat_ez(A) == WALL;
            const V v = f[ODD ? A : lat_opp(A)];
            if (TEXTURED && wdir) {
                int slot, idx;
                switch (A) {
#define AD(K) case K: aa_address<K, true>(n, WALL, bits, slot, idx); break;
                    AD(0) AD(1) AD(2) AD(3) AD(4) AD(5) AD(6) AD(7) AD(8) AD(9)
                    AD(10) AD(11) AD(12) AD(13) AD(14) AD(15) AD(16) AD(17) AD(18)
#undef AD
                }
                st_raw<T>(static_cast<T *>(p.pop[slot]) + idx, v);
            } else {
                const int xs = (ODD && !wdir) ? (lat_ex(A) > 0 ? xp : (lat_ex(A) < 0 ? xm : x)) : x;
                if (SEG && edge && !wdir && lat_ex(A) != 0) {
                    st_raw<T>(shifted_ptr(A, xs), v);
                    if ((unsigned)(xs + sxoff) < (unsigned)dstride) st_raw<T>(sbj + A * dstride + xs, v);
                } else {
                    st_raw<T>(sbj + A * dstride + xs, v);
                }
            }
        }
    };
    if (SEG) {
        for (int x = x0 + threadIdx.x; x < x1; x += nc) cell(0, x);
    } else if (nx >= nc) {  // rows at least as long as the consumer set: row by row
        for (int j = 0; j < k; ++j)
            for (int x = threadIdx.x; x < nx; x += nc) cell(j, x);
    } else {  // shorter rows: the group's k * nx cells as one range
        int j = 0, x = threadIdx.x;
        while (x >= nx && j < k) x -= nx, ++j;
        for (; j < k; x += nc) {
            while (x >= nx) x -= nx, ++j;
            if (j >= k) break;
            cell(j, x);
        }
    }
    // low precision: the FP32 sums of the thread's cells of the group go to
    // the FP64 accumulators once (slots 0 and 6 sum 1 + deviation per cell)
    if constexpr (!std::is_same<T, double>::value) {
#pragma unroll
        for (int i = 0; i < NP; ++i) {
            if (i == 0 || (CONSTQ && i == 6)) acc[i] += (double)ncell;
            acc[i] += (double)racc[i];
        }
    }
}

// ------------------------------------------------------------------ cell pairs
// FP32 / FP16 storage: two neighbouring cells (x, x+1), x even, per thread
// and iteration, collided together on the packed FP32 pipe (float2 values,
// fma/add/mul .f32x2) -- half the arithmetic instructions per cell of the
// one-cell form, with bit-identical populations (collide_lp.cuh).  A
// direction whose source column is x itself (every direction of an even
// step; e_x = 0 and the smooth-wall bounce-back of an odd step) moves both
// cells' values with one 4-byte (FP16) or 8-byte (FP32) shared-memory
// access; a direction shifted by e_x = +-1 in an odd step moves them one by
// one.  For an odd nx the last pair has one cell: its second lane computes on
// the row padding and is neither stored nor summed.  Textured wall planes use
// the one-cell form (tma_group), whose wall links move per thread.
template <typename T> struct PairIO;
template <> struct PairIO<float> {
    static __device__ __forceinline__ float2 ld2(const float *q) { return *reinterpret_cast<const float2 *>(q); }
    static __device__ __forceinline__ void st2(float *q, float2 v) { *reinterpret_cast<float2 *>(q) = v; }
    static __device__ __forceinline__ float ld1(const float *q) { return *q; }
    static __device__ __forceinline__ void st1(float *q, float v) { *q = v; }
};
template <> struct PairIO<__half> {
    static __device__ __forceinline__ float2 ld2(const __half *q)
    {
        return __half22float2(*reinterpret_cast<const __half2 *>(q));
    }
    static __device__ __forceinline__ void st2(__half *q, float2 v)
    {
        *reinterpret_cast<__half2 *>(q) = __floats2half2_rn(v.x, v.y);
    }
    static __device__ __forceinline__ float ld1(const __half *q) { return __half2float(*q); }
    static __device__ __forceinline__ void st1(__half *q, float v) { *q = __float2half_rn(v); }
};

// WALL: 0 interior plane, -1 bottom plane, +1 top plane (smooth walls).
template <typename T, bool ODD, bool CONSTQ, int WALL>
__device__ __forceinline__ void tma_group2(const StepArgs &p, const LpParams &lk, T *sb, int dstride, int k,
                                           const double *shift, double (&acc)[NP], int nc)
{
    using IO = PairIO<T>;
    constexpr float iS = LpStore<T>::kInv;
    const int nx = p.nx, pitch = p.pitch, npair = (nx + 1) >> 1;
    const float2 c0 = vsplat<float2>((float)shift[0]), c1 = vsplat<float2>((float)shift[1]),
                 c2 = vsplat<float2>((float)shift[2]);
    float2 racc[NP];
    float ncell = 0.f;
#pragma unroll
    for (int i = 0; i < NP; ++i) racc[i] = make_float2(0.f, 0.f);
    auto pair = [&](int j, int x) {
        T *sbj = sb + (size_t)j * pitch;
        const bool two = x + 1 < nx;
        int xm0 = x, xp0 = x, xp1 = x;
        if (ODD) {
            xm0 = x == 0 ? nx - 1 : x - 1;
            xp0 = x + 1 < nx ? x + 1 : 0;
            xp1 = x + 2 < nx ? x + 2 : x + 2 - nx;
        }
        float2 f[Q];
#pragma unroll
        for (int A = 0; A < Q; ++A) {
            const bool wdir = ODD && lat_ez(A) != 0 && lat_ez(A) == WALL;
            const T *row = sbj + A * dstride;
            float2 v;
            if (!ODD || wdir || lat_ex(A) == 0) v = IO::ld2(row + x);
            else if (lat_ex(A) > 0) v = make_float2(IO::ld1(row + xp0), IO::ld1(row + xp1));
            else v = make_float2(IO::ld1(row + xm0), IO::ld1(row + x));
            f[ODD ? lat_opp(A) : A] = v;
        }
        // the post-collision value of population a goes to direction A = a
        // (odd step) or opp(a) (even step) at once, with the writer-side sums
        float2 s = make_float2(0.f, 0.f), m = make_float2(0.f, 0.f);
        auto emit = [&](int a) {
            const int A = ODD ? a : lat_opp(a);
            const bool wdir = ODD && lat_ez(A) != 0 && lat_ez(A) == WALL;
            T *row = sbj + A * dstride;
            const float2 v = f[a];
            if (!ODD || wdir || lat_ex(A) == 0) {
                IO::st2(row + x, v);  // for a one-cell pair the second lane lands in the row padding
            } else if (lat_ex(A) > 0) {
                IO::st1(row + xp0, v.x);
                if (two) IO::st1(row + xp1, v.y);
            } else {
                IO::st1(row + xm0, v.x);
                if (two) IO::st1(row + x, v.y);
            }
            if (CONSTQ) {
                s = vadd(s, v);
                if (lat_ex(a) > 0) m = vadd(m, v);
                if (lat_ex(a) < 0) m = vsub(m, v);
            }
        };
        const LpCellV<float2> c = lp_collide_v<T, float2>(f, lk, emit);
        if (CONSTQ) {
            s = vmul(s, vsplat<float2>(iS));
            m = vmul(m, vsplat<float2>(iS));
            if (WALL != 0) {  // smooth walls: every link into the wall bounces back, -2 e_x (w + d)
                const int ap = WALL < 0 ? 12 : 11, am = WALL < 0 ? 13 : 14;
                const float2 w36 = vsplat<float2>(1.f / 36.f), two_ = vsplat<float2>(2.f);
                m = vsub(m, vmul(two_, vfma(f[ap], vsplat<float2>(iS), w36)));
                m = vadd(m, vmul(two_, vfma(f[am], vsplat<float2>(iS), w36)));
            }
        }
        const float2 d0 = vsub(c.u0, c0), d1 = vsub(c.u1, c1), d2 = vsub(c.u2, c2);
        const float2 var = vfma(d2, d2, vfma(d1, d1, vmul(d0, d0)));
        if (two) {
            ncell += 2.f;
            racc[0] = vadd(racc[0], c.drho);
            racc[1] = vadd(racc[1], c.jx);
            racc[2] = vadd(racc[2], c.u0);
            racc[3] = vadd(racc[3], c.u1);
            racc[4] = vadd(racc[4], c.u2);
            racc[5] = vadd(racc[5], var);
            if (CONSTQ) {
                racc[6] = vadd(racc[6], s);
                racc[7] = vadd(racc[7], m);
            }
        } else {
            ncell += 1.f;
            racc[0].x += c.drho.x;
            racc[1].x += c.jx.x;
            racc[2].x += c.u0.x;
            racc[3].x += c.u1.x;
            racc[4].x += c.u2.x;
            racc[5].x += var.x;
            if (CONSTQ) {
                racc[6].x += s.x;
                racc[7].x += m.x;
            }
        }
    };
    // the group's k * npair pairs as one range over the consumer threads
    int j = 0, pr = threadIdx.x;
    while (pr >= npair && j < k) pr -= npair, ++j;
    for (; j < k; pr += nc) {
        while (pr >= npair) pr -= npair, ++j;
        if (j >= k) break;
        pair(j, 2 * pr);
    }
    // the thread's FP32 partial sums over its k * nx / nc cells of the group
    // go to the FP64 accumulators once; slots 0 and 6 sum 1 + deviation per
    // cell
#pragma unroll
    for (int i = 0; i < NP; ++i) {
        if (i >= 6 && !CONSTQ) continue;
        if (i == 0 || i == 6) acc[i] += (double)ncell;
        acc[i] += (double)racc[i].x + (double)racc[i].y;
    }
}

// ------------------------------------------------------------------ kernel
// Producer warp: lane A < 19 moves direction A's rows of every row group of
// the block; lane 0 also arms the stage's full barrier with the byte count.
// When a wait of the block gives up (the abort flag), the producer issues no
// further copy and, before it returns, waits for every load it has issued
// and every store it has committed, so no bulk copy into or out of the
// block's shared memory outlives the block.
// p.withhold_stage (a test switch, 0 in every normal launch) makes block 0
// neither arm nor load its first row group: its consumers' first wait then
// runs out after p.wait_ns with no copy in flight on that stage.
template <typename T, bool ODD, int TEX>
__device__ __forceinline__ void tma_producer(const StepArgs &p, const TmaArgs &t, int g0, int n, int lane,
                                             unsigned char *smem, uint64_t *full, uint64_t *empty, volatile int *abort)
{
    const int S = t.stages;
    const size_t dir_bytes = (size_t)t.dir_elems * sizeof(T), stage_bytes = (size_t)Q * dir_bytes;
    const bool withhold = p.withhold_stage != 0 && g0 == 0;
    // e_x shift of direction `lane`'s elements in an odd step (0: the cell's own column)
    auto shift_of = [&](int wall) {
        const int ez = lat_ez(lane < Q ? lane : 0);
        return (ODD && !(ez != 0 && ez == wall) && lane < Q) ? lat_ex(lane) : 0;
    };
    unsigned loaded = 0;  // bit s: a load into stage s was issued (its phase is the last one armed)
    unsigned phase = 0;   // bit s: parity of that phase
    for (int i = 0; i < n + S; ++i) {
        const int st = i % S;
        unsigned char *stage = smem + (size_t)st * stage_bytes;
        if (i >= S) {  // store group i - S once the consumers have released its stage
            if (!*abort && !mbar_wait_bounded(empty + st, (uint32_t)((i / S - 1) & 1), p.wait_ns, abort)) {
                *abort = 1;
                atomicExch(reinterpret_cast<unsigned long long *>(p.status + 1), 1ull);
            }
            const int gi = g0 + i - S;
            int z, y0;
            group_origin(t, gi, z, y0);
            const int k = min(t.k, p.ny - y0);
            const int wall = plane_wall(p, z);
            if (lane < Q && !*abort) {
                const GroupRows g = group_rows<ODD, TEX>(p, lane, y0, z, wall);
                if (g.bulk) {
                    if (t.nseg > 1) {
                        int x0, x1;
                        group_xrange(t, gi, p.nx, x0, x1);
                        copy_segment<T>(p, g, x0, x1, shift_of(wall), stage + (size_t)lane * dir_bytes, false, nullptr);
                    } else {
                        copy_group<T>(p, t, g, k, stage + (size_t)lane * dir_bytes, false, nullptr);
                    }
                }
                bulk_commit();
            }
        }
        if (i < n) {  // load group i into the stage
            const int gi = g0 + i;
            int z, y0;
            group_origin(t, gi, z, y0);
            const int k = min(t.k, p.ny - y0);
            const int wall = plane_wall(p, z);
            GroupRows g{};
            if (lane < Q) g = group_rows<ODD, TEX>(p, lane, y0, z, wall);
            const unsigned vote = __ballot_sync(0xffffffffu, lane < Q && g.bulk);
            if (lane < Q) bulk_wait_read_all();  // this lane's store of the stage has read it
            __syncwarp();
            // one decision for the whole warp: lane 0's reading of the flag
            const bool issue = __shfl_sync(0xffffffffu, *abort, 0) == 0 && !(withhold && i == 0);
            if (issue) {
                int x0 = 0, x1 = p.nx;
                if (t.nseg > 1) group_xrange(t, gi, p.nx, x0, x1);
                const size_t bytes = t.nseg > 1 ? (size_t)((x1 - x0 + 1) & ~1) * sizeof(T) : (size_t)k * t.row_bytes;
                if (lane == 0) mbar_expect_tx(full + st, (uint32_t)(__popc(vote) * bytes));
                __syncwarp();
                if (lane < Q && g.bulk) {
                    if (t.nseg > 1)
                        copy_segment<T>(p, g, x0, x1, shift_of(wall), stage + (size_t)lane * dir_bytes, true, full + st);
                    else
                        copy_group<T>(p, t, g, k, stage + (size_t)lane * dir_bytes, true, full + st);
                }
                loaded |= 1u << st;
                phase = (phase & ~(1u << st)) | ((unsigned)((i / S) & 1) << st);
            }
        }
    }
    if (lane < Q) bulk_wait_all();
    if (*abort) {
        // loads still landing in shared memory: wait for the last phase armed
        // on each stage (bounded; a load that was issued does complete)
        for (int st = 0; st < S; ++st)
            if ((loaded >> st) & 1u) mbar_wait_bounded(full + st, (phase >> st) & 1u, p.wait_ns, nullptr);
    }
}

constexpr int kTmaMaxThreads = 384;  // up to 11 consumer warps + the producer warp

// Launch bounds of the row-pipelined kernels.  Every step is compiled
// "wide": up to 384 threads (11 consumer warps), one block per SM, up to 168
// registers (a sub-partition's 16K registers shared by three warps).  The
// low-precision steps also have a "dense" form: the FP32 constant-force step
// for up to 256 threads and two blocks per SM (128 registers, no spills:
// more warps in flight where the stages are small enough for two blocks);
// the FP16 steps for up to 256 threads and one block per SM, up to 255
// registers (their cell pairs need 180-200: no spills; registers are
// allocated per sub-partition, so 288-320 threads, three warps on some
// sub-partitions, would be held to 168 like the wide form).  A launch of
// more threads than the dense form's takes the wide form.
template <typename T, bool CONSTQ>
struct TmaBounds {
    // blocks per SM of the dense form (0: not compiled)
    static constexpr int dense_blocks =
        std::is_same<T, double>::value ? 0 : (std::is_same<T, __half>::value ? 1 : (CONSTQ ? 0 : 2));
    static constexpr bool has_dense = dense_blocks > 0;
    static constexpr int dense_threads = 256;
    static constexpr int threads = has_dense ? dense_threads : kTmaMaxThreads;  // the dense form, when there is one
    static constexpr int min_blocks = has_dense ? dense_blocks : 1;
};

// The consumers' work on one row group in a stage: FP64 one cell per thread
// and iteration in the reference's operand order; FP32/FP16 cell pairs on
// the packed FP32 pipe, except the planes next to a textured wall.
template <typename T, bool ODD, bool CONSTQ, bool TXT>
__device__ __forceinline__ void consume_group(const StepArgs &p, const LpParams &lk, T *sb, int dstride, int y0, int k,
                                              int z, double G, const double *sh, double (&acc)[NP], int nc)
{
    const int wall = plane_wall(p, z);
    if constexpr (std::is_same<T, double>::value) {
        if (wall < 0) tma_group<T, ODD, CONSTQ, TXT, -1>(p, sb, dstride, y0, k, z, G, sh, acc, nc);
        else if (wall > 0) tma_group<T, ODD, CONSTQ, TXT, 1>(p, sb, dstride, y0, k, z, G, sh, acc, nc);
        else tma_group<T, ODD, CONSTQ, TXT, 0>(p, sb, dstride, y0, k, z, G, sh, acc, nc);
    } else {
        if (wall < 0) {
            if (TXT) tma_group<T, ODD, CONSTQ, true, -1>(p, sb, dstride, y0, k, z, G, sh, acc, nc);
            else tma_group2<T, ODD, CONSTQ, -1>(p, lk, sb, dstride, k, sh, acc, nc);
        } else if (wall > 0) {
            if (TXT) tma_group<T, ODD, CONSTQ, true, 1>(p, sb, dstride, y0, k, z, G, sh, acc, nc);
            else tma_group2<T, ODD, CONSTQ, 1>(p, lk, sb, dstride, k, sh, acc, nc);
        } else {
            tma_group2<T, ODD, CONSTQ, 0>(p, lk, sb, dstride, k, sh, acc, nc);
        }
    }
}

// The step of one channel by one block: `blk` numbers the block among the
// channel's blocks, `tma_smem` is the block's dynamic shared memory.
template <typename T, bool ODD, bool CONSTQ, int TEX>
__device__ __forceinline__ void tma_step_body(const StepArgs &p, const TmaArgs &t, int blk, unsigned char *tma_smem)
{
    __shared__ int s_abort;
    const int G_ = t.groups_per_block, S = t.stages;
    const int g0 = blk * G_;
    const int n = min(g0 + G_, t.ngroups) - g0;
    if (n <= 0) return;  // block-uniform; empty blocks contribute to no plane
    const int nc = blockDim.x - 32;  // consumer threads; the last warp produces
    const size_t dir_bytes = (size_t)t.dir_elems * sizeof(T), stage_bytes = (size_t)Q * dir_bytes;
    uint64_t *full = reinterpret_cast<uint64_t *>(tma_smem + (size_t)S * stage_bytes);
    uint64_t *empty = full + S;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, nc / 32);
        }
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();
    if (threadIdx.x >= nc) {
        tma_producer<T, ODD, TEX>(p, t, g0, n, threadIdx.x - nc, tma_smem, full, empty, &s_abort);
        return;
    }

    const long long step = *p.step_ctr;
    const double G = CONSTQ ? p.force[step & 1] : p.gx;
    const double *shift_now = p.shift + (size_t)(step & 1) * p.nz * 3;
    const int dstride = t.dir_elems;
    [[maybe_unused]] const LpParams lk = lp_params<typename std::conditional<std::is_same<T, double>::value, float, T>::type>(
        (float)p.omega, (float)G);
    double acc[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i] = 0.0;
    for (int i = 0; i < n; ++i) {
        const int st = i % S, gi = g0 + i;
        int z, y0;
        group_origin(t, gi, z, y0);
        const int k = min(t.k, p.ny - y0);
        if (!*(volatile int *)&s_abort &&
            !mbar_wait_bounded(full + st, (uint32_t)((i / S) & 1), p.wait_ns, (volatile int *)&s_abort)) {
            s_abort = 1;
            atomicExch(reinterpret_cast<unsigned long long *>(p.status + 1), 1ull);
        }
        T *sb = reinterpret_cast<T *>(tma_smem + (size_t)st * stage_bytes);
        if constexpr (std::is_same<T, double>::value) {
            if (t.nseg > 1) {  // an x-segment of one row
                int x0, x1;
                group_xrange(t, gi, p.nx, x0, x1);
                constexpr bool TXT = TEX != 0;
                const double *sh = shift_now + z * 3;
                const int wall = plane_wall(p, z);
                if (wall < 0) tma_group<T, ODD, CONSTQ, TXT, -1, true>(p, sb, dstride, y0, 1, z, G, sh, acc, nc, x0, x1);
                else if (wall > 0)
                    tma_group<T, ODD, CONSTQ, TXT, 1, true>(p, sb, dstride, y0, 1, z, G, sh, acc, nc, x0, x1);
                else tma_group<T, ODD, CONSTQ, TXT, 0, true>(p, sb, dstride, y0, 1, z, G, sh, acc, nc, x0, x1);
            } else {
                consume_group<T, ODD, CONSTQ, TEX != 0>(p, lk, sb, dstride, y0, k, z, G, shift_now + z * 3, acc, nc);
            }
        } else {
            consume_group<T, ODD, CONSTQ, TEX != 0>(p, lk, sb, dstride, y0, k, z, G, shift_now + z * 3, acc, nc);
        }
        fence_async_smem();  // this thread's shared-memory writes -> visible to the bulk stores
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(empty + st);
        if (i + 1 == n || (gi + 1) % t.gpp == 0) {  // this block's last group of plane z
            const int pi = gi / t.gpp;  // position of plane z in the kernel's plane list
            const int bfirst = (pi * t.gpp) / G_;
            const int blast = min(((pi + 1) * t.gpp - 1) / G_, (t.ngroups - 1) / G_);
            plane_contribute(p, acc, z, blk - bfirst, blast - bfirst + 1, step, G, 0, nc);
#pragma unroll
            for (int q = 0; q < NP; ++q) acc[q] = 0.0;
        }
    }
}

template <typename T, bool ODD, bool CONSTQ, int TEX, bool WIDE>
__global__ void __launch_bounds__(WIDE ? kTmaMaxThreads : TmaBounds<T, CONSTQ>::threads, WIDE ? 1 : TmaBounds<T, CONSTQ>::min_blocks)
    step_tma_kernel(const StepArgs p, const TmaArgs t)
{
    extern __shared__ __align__(128) unsigned char tma_smem[];
    // Launched with programmatic stream serialization (launch_tma): a block
    // may start on an SM that the previous step's grid has left while that
    // grid still runs.  Before anything else it waits for the previous grid
    // to complete with its memory visible; then it lets the next step's grid
    // be scheduled, whose blocks wait here in turn.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if constexpr (WIDE || TmaBounds<T, CONSTQ>::has_dense) tma_step_body<T, ODD, CONSTQ, TEX>(p, t, blockIdx.x, tma_smem);
}

// the form of step_tma_kernel a launch of `threads` threads takes
template <typename T, bool CONSTQ>
__host__ __forceinline__ bool tma_wide(int threads)
{
    return !TmaBounds<T, CONSTQ>::has_dense || threads > TmaBounds<T, CONSTQ>::threads;
}

// Many independent channels in one launch: block b belongs to the channel c
// with first[c] <= b < first[c+1] and runs that channel's step, reading its
// arguments from the read-only table (through a restrict pointer, so they
// stay in registers across the block's shared-memory stores).
struct ChannelLaunch {
    StepArgs p;
    TmaArgs t;
    int first_block;
    int textured;  // TEX of the channel (0 smooth, else textured walls)
};

template <typename T, bool ODD>
__global__ void __launch_bounds__(kTmaMaxThreads, 1) step_tma_batch_kernel(const ChannelLaunch *__restrict__ chans,
                                                                           int nchan)
{
    extern __shared__ __align__(128) unsigned char tma_smem[];
    int c = 0;
    while (c + 1 < nchan && chans[c + 1].first_block <= (int)blockIdx.x) ++c;
    const ChannelLaunch &L = chans[c];
    const int blk = blockIdx.x - L.first_block;
    const bool q = L.p.const_q != 0;
    if (q) {
        if (L.textured) tma_step_body<T, ODD, true, 1>(L.p, L.t, blk, tma_smem);
        else tma_step_body<T, ODD, true, 0>(L.p, L.t, blk, tma_smem);
    } else {
        if (L.textured) tma_step_body<T, ODD, false, 1>(L.p, L.t, blk, tma_smem);
        else tma_step_body<T, ODD, false, 0>(L.p, L.t, blk, tma_smem);
    }
}

template <typename T>
int tma_set_smem_attr(size_t bytes)
{
    const void *ks[] = {
        (const void *)step_tma_kernel<T, false, false, 0, true>, (const void *)step_tma_kernel<T, false, false, 1, true>,
        (const void *)step_tma_kernel<T, false, true, 0, true>,  (const void *)step_tma_kernel<T, false, true, 1, true>,
        (const void *)step_tma_kernel<T, true, false, 0, true>,  (const void *)step_tma_kernel<T, true, false, 1, true>,
        (const void *)step_tma_kernel<T, true, true, 0, true>,   (const void *)step_tma_kernel<T, true, true, 1, true>,
        (const void *)step_tma_kernel<T, false, false, 0, false>, (const void *)step_tma_kernel<T, false, false, 1, false>,
        (const void *)step_tma_kernel<T, true, false, 0, false>,  (const void *)step_tma_kernel<T, true, false, 1, false>,
        (const void *)step_tma_kernel<T, false, true, 0, false>,  (const void *)step_tma_kernel<T, false, true, 1, false>,
        (const void *)step_tma_kernel<T, true, true, 0, false>,   (const void *)step_tma_kernel<T, true, true, 1, false>};
    for (int i = 0; i < 16; ++i)
        if (cudaFuncSetAttribute(ks[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
            return -1;
    return 0;
}

template <typename T>
int tma_occupancy(int threads, size_t smem, bool const_q)
{
    int n = 0;
    if (threads > kTmaMaxThreads) return 0;
    cudaError_t e;
    if (const_q && tma_wide<T, true>(threads))
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, step_tma_kernel<T, true, true, 0, true>, threads, smem);
    else if (const_q)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, step_tma_kernel<T, true, true, 0, false>, threads, smem);
    else if (tma_wide<T, false>(threads))
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, step_tma_kernel<T, true, false, 0, true>, threads, smem);
    else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, step_tma_kernel<T, true, false, 0, false>, threads, smem);
    return e == cudaSuccess ? n : 0;
}

template <typename T>
void launch_tma(const StepArgs &p, const TmaArgs &t, int grid, int threads, size_t smem, bool odd, int tex,
                cudaStream_t s)
{
    const bool q = p.const_q != 0;
    const bool wide = q ? tma_wide<T, true>(threads) : tma_wide<T, false>(threads);
    // programmatic stream serialization: the launch and the blocks' start
    // overlap the end of the previous step (the kernel orders itself after
    // it with griddepcontrol.wait); the grid is never larger than what is
    // resident at once, so a waiting block never keeps one of the previous
    // grid's blocks from running
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
#define L(O, C, X)                                                                            \
    do {                                                                                      \
        if (wide || !TmaBounds<T, C>::has_dense) cudaLaunchKernelEx(&cfg, step_tma_kernel<T, O, C, X, true>, p, t); \
        else cudaLaunchKernelEx(&cfg, step_tma_kernel<T, O, C, X, false>, p, t);             \
    } while (0)
#define LX(O, C) do { if (tex) L(O, C, 1); else L(O, C, 0); } while (0)
    if (odd) {
        if (q) LX(true, true); else LX(true, false);
    } else {
        if (q) LX(false, true); else LX(false, false);
    }
#undef LX
#undef L
}

template <typename T>
int tma_batch_set_smem_attr(size_t bytes)
{
    const void *ks[] = {(const void *)step_tma_batch_kernel<T, false>, (const void *)step_tma_batch_kernel<T, true>};
    for (const void *k : ks)
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) return -1;
    return 0;
}

template <typename T>
int tma_batch_occupancy(int threads, size_t smem)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, step_tma_batch_kernel<T, true>, threads, smem) !=
        cudaSuccess)
        return 0;
    return n;
}

template <typename T>
void launch_tma_batch(const ChannelLaunch *chans, int nchan, int grid, int threads, size_t smem, bool odd,
                      cudaStream_t s)
{
    if (odd) step_tma_batch_kernel<T, true><<<grid, threads, smem, s>>>(chans, nchan);
    else step_tma_batch_kernel<T, false><<<grid, threads, smem, s>>>(chans, nchan);
}

}  // namespace dnslbm
