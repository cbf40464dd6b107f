// Batched channels in one persistent launch.
//
// One cooperative launch (every block resident at once) advances all
// channels of a batch through nsteps time steps.  Within a step the work is
// a table of items, largest first, each a run of row groups of one plane of
// one channel moved through the block's shared-memory stages by the
// bulk-copy engine and collided by the consumer warps:
//   kind 0  a plane without link masks: the row-pipelined step of
//           step_tma.cuh (rows in, rows out);
//   kind 1  a plane with per-cell link masks (solids inside the flow), one
//           cell per thread (links_cell).  An even step touches only the
//           cells' own rows, which go in and out as for kind 0.  An odd step
//           brings in the rows of the regular address set; a link that
//           bounces back or meets a wall reads its own address from global
//           memory, and every result goes to global memory: a bounced link's
//           address lies in a row of another cell row's set (that of the
//           solid neighbour, which is never collided), so the rows are not
//           stored back.  Every address is still read and written by one
//           cell only.
// A block's producer warp takes the next item from the step's counter
// (atomicAdd), so blocks that drew small items take more: no block waits
// for a channel it owns.  Each item sums its cells into its own partial-sum
// slot of its plane (the item's index within the plane), so the plane sums,
// the logs and the next force do not depend on which block took which item.
// The last item of a channel's step runs that channel's step tail.  Steps
// are separated by a grid-wide barrier.
//
// Every wait is bounded by the GPU's global timer: the stage waits (as in
// step_tma.cuh) and the grid barrier.  A wait that runs out raises the
// launch's abort flag: the block's consumers leave the step together (one
// barrier-reduction per stage makes that decision uniform), its producer
// waits for the copies it has issued, every block still arrives at the
// grid barrier, and no block starts another step.
//
// Memory written by other SMs earlier in the launch is read through L2:
// bulk copies always are; the per-thread loads use ld.global.cg, and the
// per-channel force, plane means and step counter are read with __ldcg.
#pragma once

#include "step_tma.cuh"

namespace dnslbm {

struct BatchItem {
    int chan;            // index into the channel table
    int kind;            // 0: row groups through the stages, 1: cells of a plane with link masks
    int first, count;    // row groups first .. first+count-1 (the channel's group numbering)
    int plane;           // the plane z
    int slot, ncontrib;  // partial-sum slot of the item in its plane, items of that plane
};

struct PersistArgs {
    const ChannelLaunch *chans;
    const BatchItem *items;
    int nitems, nsteps, first_odd, stages;
    unsigned stage_bytes;          // bytes of one stage (the largest channel's)
    unsigned *counters;            // [nsteps] items taken in each step (zero at launch)
    unsigned *arrivals;            // grid-barrier arrivals (zero at launch)
    int *abort;                    // a bounded wait gave up: the launch stops
    unsigned long long wait_ns;    // limit of every bounded wait
    int withhold;                  // test switch (0 otherwise): the first item's first load is withheld
};

// Per-stage header, written by the producer before it arms the stage: the
// item and row group of the stage.  The channel's arguments stay in the
// read-only global table (a restrict pointer lets the compiler keep them in
// registers across the consumers' shared-memory stores; a copy in shared
// memory would be reloaded after each of them).
struct StageHeader {
    BatchItem it;
    int item;   // index of the item; -1 ends the step
    int group;  // row group within the item
    int z, y0;  // plane and first row of the group
};

// Shared memory after the stages: full[S], empty[S] (8 bytes each), then
// the stage headers.
__host__ __device__ constexpr size_t persist_smem(int stages, size_t stage_bytes)
{
    return (size_t)stages * stage_bytes + 16 * (size_t)stages + sizeof(StageHeader) * (size_t)stages;
}

// OR of v over the first nthreads threads (named barrier 2): every one of
// them gets the same answer at the same point.
__device__ __forceinline__ bool consumers_any(int v, int nthreads)
{
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.s32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 2, %2, q;\n\t"
        "selp.s32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"(v), "r"(nthreads)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

__device__ __forceinline__ void persist_raise(const PersistArgs &a, volatile int *s_abort)
{
    *s_abort = 1;
    atomicExch(a.abort, 1);
}

template <typename T, bool ODD>
__device__ __forceinline__ void persist_producer(const PersistArgs &a, int s, int lane, unsigned char *smem,
                                                 uint64_t *full, uint64_t *empty, StageHeader *hdr,
                                                 volatile int *s_abort)
{
    const int S = a.stages;
    const ChannelLaunch *__restrict__ chans = a.chans;
    int i = 0;            // stage sequence number within the step
    // test switch: the block that takes the first item of the first step
    // neither arms nor loads its first row group, so its consumers' wait runs
    // out with no copy in flight
    const bool withhold_step = a.withhold != 0 && s == 0;
    unsigned loaded = 0;  // bit st: a load into stage st was issued (its phase is the last one armed)
    unsigned phase = 0;   // bit st: parity of that phase
    // once the consumers have released sequence seq, store the row group it held
    auto store_seq = [&](int seq) {
        const int st = seq % S;
        if (!*s_abort && !mbar_wait_bounded(empty + st, (uint32_t)((seq / S) & 1), a.wait_ns, s_abort))
            persist_raise(a, s_abort);
        const StageHeader &H = hdr[st];
        // a kind-1 item's odd-step results went to global memory
        if (*s_abort || H.item < 0 || (ODD && H.it.kind == 1) || lane >= Q) return;
        const ChannelLaunch &L = chans[H.it.chan];
        const int k = min(L.t.k, L.p.ny - H.y0);
        const int wall = plane_wall(L.p, H.z);
        const GroupRows gr = L.textured ? group_rows<ODD, 1>(L.p, lane, H.y0, H.z, wall)
                                        : group_rows<ODD, 0>(L.p, lane, H.y0, H.z, wall);
        const size_t dir_bytes = (size_t)L.t.dir_elems * sizeof(T);
        if (gr.bulk) copy_group<T>(L.p, L.t, gr, k, smem + (size_t)st * a.stage_bytes + lane * dir_bytes, false, nullptr);
        bulk_commit();
    };
    // the stage of sequence i, free for new contents
    auto next_stage = [&]() {
        if (i >= S) store_seq(i - S);
        if (lane < Q) bulk_wait_read_all();  // this lane's store of the stage has read it
        __syncwarp();
        return i % S;
    };
    // the header of a stage: the item and the row group it holds
    auto fill = [&](int st, int h, const BatchItem &it, int g, int z, int y0) {
        if (lane == 0) {
            StageHeader &H = hdr[st];
            H.it = it;
            H.item = h;
            H.group = g;
            H.z = z;
            H.y0 = y0;
        }
        __syncwarp();
    };
    auto take = [&]() { return lane == 0 ? (*s_abort ? a.nitems : (int)atomicAdd(a.counters + s, 1u)) : 0; };
    int h = __shfl_sync(0xffffffffu, take(), 0);
    while (h < a.nitems) {
        const BatchItem it = a.items[h];
        const int hn = take();  // the next item, fetched while this one is issued
        {
            const ChannelLaunch &L = chans[it.chan];
            // kind 1: the regular rows only (the wall links of an odd step
            // read their own addresses, as for a textured wall)
            const bool tex = L.textured || it.kind == 1;
            const size_t dir_bytes = (size_t)L.t.dir_elems * sizeof(T);
            for (int g = 0; g < it.count; ++g) {
                const int st = next_stage();
                int z, y0;
                group_origin(L.t, it.first + g, z, y0);
                const int k = min(L.t.k, L.p.ny - y0);
                const int wall = plane_wall(L.p, z);
                GroupRows gr{};
                if (lane < Q)
                    gr = tex ? group_rows<ODD, 1>(L.p, lane, y0, z, wall) : group_rows<ODD, 0>(L.p, lane, y0, z, wall);
                const unsigned vote = __ballot_sync(0xffffffffu, lane < Q && gr.bulk);
                const bool issue = __shfl_sync(0xffffffffu, *s_abort, 0) == 0 && !(withhold_step && h == 0 && g == 0);
                if (issue) {
                    fill(st, h, it, g, z, y0);
                    if (lane == 0) mbar_expect_tx(full + st, (uint32_t)((size_t)__popc(vote) * k * L.t.row_bytes));
                    __syncwarp();
                    if (lane < Q && gr.bulk)
                        copy_group<T>(L.p, L.t, gr, k, smem + (size_t)st * a.stage_bytes + lane * dir_bytes, true,
                                      full + st);
                    loaded |= 1u << st;
                    phase = (phase & ~(1u << st)) | ((unsigned)((i / S) & 1) << st);
                }
                ++i;
            }
        }
        h = __shfl_sync(0xffffffffu, hn, 0);
        if (__shfl_sync(0xffffffffu, *s_abort, 0)) break;
    }
    {  // end of the step
        const int st = next_stage();
        if (lane == 0) {
            hdr[st].item = -1;
            mbar_arrive(full + st);
        }
        __syncwarp();
        ++i;
    }
    for (int seq = max(0, i - S); seq < i - 1; ++seq) store_seq(seq);
    if (lane < Q) bulk_wait_all();
    if (*s_abort)  // loads still landing in shared memory (bounded; an issued load completes)
        for (int st = 0; st < S; ++st)
            if ((loaded >> st) & 1u) mbar_wait_bounded(full + st, (phase >> st) & 1u, a.wait_ns, nullptr);
}

// A row group of a kind-1 item from the stage: rows y0 .. y0+k-1 of plane z,
// one cell per thread (links_cell; the odd step's shifted elements at x-1
// and x+1 wrap around the row).
template <typename T, bool ODD, bool CONSTQ>
__device__ __forceinline__ void persist_links(const StepArgs &p, T *sb, int dstride, int y0, int k, int z, double G,
                                              const double (&sh)[3], double (&acc)[NP], int nc)
{
    const int nx = p.nx;
    const int wall = plane_wall(p, z);
    for (int c = threadIdx.x; c < k * nx; c += nc) {
        const int j = c / nx, x = c - j * nx, y = y0 + j;
        float racc[NP];
#pragma unroll
        for (int q = 0; q < NP; ++q) racc[q] = 0.f;
        const Nbr n = make_nbr(x, y, z, nx, p.ny, p.pitch);
        const int om = x == 0 ? nx - 1 : -1, op = x == nx - 1 ? 1 - nx : 1;
        links_cell<T, ODD, CONSTQ>(p, n, wall, cell_links(p.band_of, p.links, nx, p.ny, x, y, z),
                                   sb + (size_t)j * p.pitch + x, dstride, G, sh[0], sh[1], sh[2], acc, racc, om, op);
#pragma unroll
        for (int q = 0; q < NP; ++q) acc[q] += (double)racc[q];
    }
}

template <typename T, bool ODD, bool ANYQ>
__device__ __forceinline__ void persist_consumers(const PersistArgs &a, int s, unsigned char *smem, uint64_t *full,
                                                  uint64_t *empty, const StageHeader *hdr, int nc,
                                                  volatile int *s_abort)
{
    using LpT = typename std::conditional<std::is_same<T, double>::value, float, T>::type;
    const int S = a.stages;
    const ChannelLaunch *__restrict__ chans = a.chans;
    // parity of the step counter (every channel of a batch is at the same
    // step, and a loaded state starts at step 0 with the even AA step)
    const int sp = (a.first_odd + s) & 1;
    double acc[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) acc[q] = 0.0;
    // per item: the force of the step and the plane's shift (the previous
    // plane means), read once at the item's first stage
    double G = 0.0, sh[3] = {0.0, 0.0, 0.0};
    for (int i = 0;; ++i) {
        const int st = i % S;
        int bad = 0;
        if (!*s_abort && !mbar_wait_bounded(full + st, (uint32_t)((i / S) & 1), a.wait_ns, s_abort)) bad = 1;
        if (consumers_any(bad | *s_abort, nc)) {  // every consumer leaves the step here together
            if (threadIdx.x == 0) persist_raise(a, s_abort);
            return;
        }
        const StageHeader &H = hdr[st];
        if (H.item < 0) return;  // end of the step (the same header for every consumer)
        const ChannelLaunch &L = chans[H.it.chan];
        const StepArgs &p = L.p;
        const bool q = ANYQ && p.const_q != 0;  // a batch without constant-Q channels compiles no such path
        const int z = H.z;
        if (H.group == 0) {  // an item's first stage
            G = q ? __ldcg(p.force + sp) : p.gx;
            const double *shp = p.shift + (size_t)sp * p.nz * 3 + z * 3;
            sh[0] = __ldcg(shp);
            sh[1] = __ldcg(shp + 1);
            sh[2] = __ldcg(shp + 2);
        }
        const int k = min(L.t.k, p.ny - H.y0);
        const int dstride = L.t.dir_elems;
        T *sb = reinterpret_cast<T *>(smem + (size_t)st * a.stage_bytes);
        if (H.it.kind == 1) {
            if (q) persist_links<T, ODD, true>(p, sb, dstride, H.y0, k, z, G, sh, acc, nc);
            else persist_links<T, ODD, false>(p, sb, dstride, H.y0, k, z, G, sh, acc, nc);
            fence_async_smem();  // the even step's rows go back by bulk store
        } else {
            [[maybe_unused]] const LpParams lk = lp_params<LpT>((float)p.omega, (float)G);
            if (q) {
                if (L.textured) consume_group<T, ODD, true, true>(p, lk, sb, dstride, H.y0, k, z, G, sh, acc, nc);
                else consume_group<T, ODD, true, false>(p, lk, sb, dstride, H.y0, k, z, G, sh, acc, nc);
            } else {
                if (L.textured) consume_group<T, ODD, false, true>(p, lk, sb, dstride, H.y0, k, z, G, sh, acc, nc);
                else consume_group<T, ODD, false, false>(p, lk, sb, dstride, H.y0, k, z, G, sh, acc, nc);
            }
            fence_async_smem();  // this thread's shared-memory writes -> visible to the bulk stores
        }
        const bool done = H.group == H.it.count - 1;
        if (done) {  // the item is done: its plane contribution (the stage is released after it)
            // step -1: the channel's step tail reads its own step counter
            plane_contribute(p, acc, z, H.it.slot, H.it.ncontrib, -1, G, 0, nc);
#pragma unroll
            for (int r = 0; r < NP; ++r) acc[r] = 0.0;
        }
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(empty + st);
    }
}

template <typename T, bool ODD, bool ANYQ>
__device__ __forceinline__ void persist_step(const PersistArgs &a, int s, unsigned char *smem, volatile int *s_abort)
{
    const int S = a.stages, nc = blockDim.x - 32;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + (size_t)S * a.stage_bytes);
    uint64_t *empty = full + S;
    StageHeader *hdr = reinterpret_cast<StageHeader *>(empty + S);
    if (threadIdx.x == 0) {
        for (int st = 0; st < S; ++st) {
            mbar_init(full + st, 1);
            mbar_init(empty + st, nc / 32);
        }
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x >= nc) persist_producer<T, ODD>(a, s, threadIdx.x - nc, smem, full, empty, hdr, s_abort);
    else persist_consumers<T, ODD, ANYQ>(a, s, smem, full, empty, hdr, nc, s_abort);
}

// Grid-wide barrier between steps (all blocks are resident: cooperative
// launch).  Bounded: gives up after wait_ns, raising the abort flag.
// Returns false when the launch is to stop.
__device__ __forceinline__ bool persist_grid_barrier(const PersistArgs &a, unsigned target)
{
    __shared__ int s_go;
    __syncthreads();
    if (threadIdx.x == 0) {
        fence_async_global();  // this block's bulk stores before its arrival
        __threadfence();
        atomicAdd(a.arrivals, 1u);
        int go = !*(volatile int *)a.abort;
        const unsigned long long t0 = globaltimer_ns();
        while (go && *(volatile unsigned *)a.arrivals < target) {
            if (*(volatile int *)a.abort) go = 0;
            else if (globaltimer_ns() - t0 > a.wait_ns) {
                atomicExch(a.abort, 1);
                go = 0;
            } else {
                __nanosleep(100);
            }
        }
        __threadfence();
        fence_async_global();  // the other blocks' stores before this block's next loads
        s_go = go && !*(volatile int *)a.abort;
    }
    __syncthreads();
    return s_go != 0;
}

// ANYQ: some channel runs with a constant flow rate.  The launch bounds are
// those of the dense step form where the precision has one (FP32 without
// ANYQ: 256 threads, two blocks per SM; FP16: 256 threads, one block).
template <typename T, bool ANYQ>
__global__ void __launch_bounds__(TmaBounds<T, ANYQ>::threads, TmaBounds<T, ANYQ>::min_blocks)
    persist_batch_kernel(const PersistArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_abort;
    for (int s = 0; s < a.nsteps; ++s) {
        if (threadIdx.x == 0) s_abort = 0;
        if ((a.first_odd + s) & 1) persist_step<T, true, ANYQ>(a, s, smem, &s_abort);
        else persist_step<T, false, ANYQ>(a, s, smem, &s_abort);
        if (!persist_grid_barrier(a, (unsigned)(s + 1) * gridDim.x)) break;
    }
}

template <typename T>
int persist_set_smem_attr(size_t bytes)
{
    const bool ok = cudaFuncSetAttribute(persist_batch_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)bytes) == cudaSuccess &&
                    cudaFuncSetAttribute(persist_batch_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)bytes) == cudaSuccess;
    return ok ? 0 : -1;
}

template <typename T>
int persist_occupancy(int threads, size_t smem, bool any_q)
{
    int n = 0;
    if (threads > (any_q ? TmaBounds<T, true>::threads : TmaBounds<T, false>::threads)) return 0;
    const cudaError_t e =
        any_q ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, persist_batch_kernel<T, true>, threads, smem)
              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, persist_batch_kernel<T, false>, threads, smem);
    return e == cudaSuccess ? n : 0;
}

// Cooperative launch: fails (instead of deadlocking) when the grid cannot
// be resident at once.
template <typename T>
cudaError_t launch_persist(const PersistArgs &a, int grid, int threads, size_t smem, bool any_q, cudaStream_t s)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return any_q ? cudaLaunchKernelEx(&cfg, persist_batch_kernel<T, true>, a)
                 : cudaLaunchKernelEx(&cfg, persist_batch_kernel<T, false>, a);
}

}  // namespace dnslbm
