// C-ABI implementation: device context, flags, state I/O and the step driver.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dnslbm.h"
#include "step_common.cuh"
#include "step_persist.cuh"

namespace dnslbm {
void launch_step_f64(const StepArgs &p, dim3 grid, dim3 block, bool odd, int tex, cudaStream_t s);
void launch_reduce_f64(const StepArgs &p, dim3 grid, dim3 block, cudaStream_t s);
void launch_step_lp(int precision, const StepArgs &p, dim3 grid, dim3 block, bool odd, int tex, cudaStream_t s);
void launch_reduce_lp(int precision, const StepArgs &p, dim3 grid, dim3 block, cudaStream_t s);
void launch_io(int precision, int what, const IoArgs &p, int x0, int nxc, double *a, double *b, cudaStream_t s);
void launch_stats(int precision, const IoArgs &p, dim3 grid, dim3 block, int rows, int pass, const double *mean,
                  double *partials, double *plane_out, cudaStream_t s);
void launch_stats_sample(int nz, double np, const double *planes, double *mean, double *acc, bool accumulate,
                         cudaStream_t s);
void launch_stats_rows(int nz, double np, const double *mean, const double *planes, double *out, cudaStream_t s);
void launch_quadrant(const double *vel, int nx, int ny, int zd, double *mean, double *out, cudaStream_t s);
size_t correlation_scratch(int nx, int ny, int zd, int per_chunk);
int correlation_max_line();
cudaError_t launch_correlations(const double *vel, int nx, int ny, int zd, int per_chunk, double *scratch,
                                double *xcorl, double *ycorl, double *ua, cudaStream_t s);
size_t spectra_scratch(int nx, int ny, int zd, int jb);
cudaError_t launch_spectra(const double *vel, int nx, int ny, int zd, int jb, double *scratch, double *ex, double *ey,
                           cudaStream_t s);
int persist_prepare_f64(size_t smem);
int persist_occupancy_f64(int threads, size_t smem, bool any_q);
cudaError_t launch_persist_f64(const PersistArgs &a, int grid, int threads, size_t smem, bool any_q, cudaStream_t s);
int persist_prepare_lp(int precision, size_t smem);
int persist_occupancy_lp(int precision, int threads, size_t smem, bool any_q);
cudaError_t launch_persist_lp(int precision, const PersistArgs &a, int grid, int threads, size_t smem, bool any_q,
                              cudaStream_t s);
static int persist_prepare(int precision, size_t smem)
{
    return precision == 64 ? persist_prepare_f64(smem) : persist_prepare_lp(precision, smem);
}
static int persist_occupancy_of(int precision, int threads, size_t smem, bool any_q)
{
    return precision == 64 ? persist_occupancy_f64(threads, smem, any_q)
                           : persist_occupancy_lp(precision, threads, smem, any_q);
}
static cudaError_t launch_persist_batch(int precision, const PersistArgs &a, int grid, int threads, size_t smem,
                                        bool any_q, cudaStream_t s)
{
    return precision == 64 ? launch_persist_f64(a, grid, threads, smem, any_q, s)
                           : launch_persist_lp(precision, a, grid, threads, smem, any_q, s);
}
int tma_prepare_f64(size_t smem);
int tma_occupancy_f64(int threads, size_t smem, bool const_q);
void launch_tma_f64(const StepArgs &p, const TmaArgs &t, int grid, int threads, size_t smem, bool odd, int tex,
                    cudaStream_t s);
int tma_prepare_lp(int precision, size_t smem);
int tma_occupancy_lp(int precision, int threads, size_t smem, bool const_q);
void launch_tma_lp(int precision, const StepArgs &p, const TmaArgs &t, int grid, int threads, size_t smem, bool odd,
                   int tex, cudaStream_t s);
int tma_batch_prepare_f64(size_t smem);
int tma_batch_occupancy_f64(int threads, size_t smem);
void launch_tma_batch_f64(const ChannelLaunch *chans, int nchan, int grid, int threads, size_t smem, bool odd,
                          cudaStream_t s);
int tma_batch_prepare_lp(int precision, size_t smem);
int tma_batch_occupancy_lp(int precision, int threads, size_t smem);
void launch_tma_batch_lp(int precision, const ChannelLaunch *chans, int nchan, int grid, int threads, size_t smem,
                         bool odd, cudaStream_t s);
void launch_links_f64(const LinksLaunch *tab, int n, int blocks, bool odd, cudaStream_t s);
void launch_links_lp(int precision, const LinksLaunch *tab, int n, int blocks, bool odd, cudaStream_t s);
void launch_slab_tail(const StepArgs &a, int mode, double *slab_shift, int z0, int nzs, cudaStream_t s);
}  // namespace dnslbm

using namespace dnslbm;

struct dnslbm_ctx {
    dnslbm_deck deck;
    int nx, ny, nz;
    int pitch;  // row pitch in elements: rows padded to 16 bytes for bulk copies
    size_t ncell, pstride, esize;
    void *popmem = nullptr;
    uint8_t *wallmask = nullptr;
    int textured = 0;        // 0 smooth walls, 1 textured walls, 2 solids inside the flow
    int walls_textured = 0;  // wall planes with slip cells (the row-pipelined kernel's TEX)
    int *band_of = nullptr;      // [nz] mask block of a plane next to a solid, -1: none
    unsigned *links = nullptr;   // [nband][ny][nx] per-cell link masks
    size_t links_bytes = 0;
    int nband = 0;
    // planes of the row-pipelined kernel (nclean, ascending) followed by the
    // planes with link masks (ndirty), which a second launch steps per cell
    int *plane_list = nullptr;
    std::vector<int> plane_host;  // host copy of plane_list
    int nclean = 0, ndirty = 0;
    LinksLaunch *d_llaunch = nullptr;  // the second launch's table (one entry)
    int tma_target = 0;                // resident blocks of the row-pipelined kernel
    double *force = nullptr, *shift = nullptr, *partials = nullptr, *plane_sums = nullptr, *logs = nullptr;
    long long *step_ctr = nullptr, *status = nullptr;
    unsigned *plane_ctr = nullptr, *total_ctr = nullptr;
    double *staging = nullptr;  // device AoS staging for I/O
    size_t staging_bytes = 0;
    double *stat_partials = nullptr, *stat_planes = nullptr, *stat_mean = nullptr;
    double *stat_acc = nullptr;  // [9][nz] running sums of the time average
    long stat_samples = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;                // the per-cell pass runs here beside the bulk kernel
    cudaEvent_t fj[2] = {nullptr, nullptr};     // fork / join of the side stream
    // asynchronous output (dnslbm_output_begin): device buffers of one
    // snapshot, the stream their copies to the host run on, and the events
    // that order them (ready: kernels done; done: copies landed)
    double *out_lbf = nullptr, *out_vel = nullptr, *out_den = nullptr, *out_stats = nullptr;
    cudaStream_t out_stream = nullptr;
    cudaEvent_t out_ev[2] = {nullptr, nullptr};
    int out_pending = 0;
    double *quad_buf = nullptr;  // quadrant analysis: plane means [zd][3], plane sums [zd][9]
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::vector<cudaEvent_t> tev;  // per-launch timing events
    dim3 grid, block;
    int rows = 8;
    int slots = 1;  // partial-sum slots per plane
    // row-pipelined (bulk-copy) step; with odd_split the odd steps use their
    // own launch shape (odd_*), chosen by the autotuner
    int use_tma = 0, tma_threads = 0, tma_grid = 0;
    int odd_split = 0, odd_threads = 0, odd_grid = 0, odd_target = 0;
    size_t odd_smem = 0;
    TmaArgs odd_tma{};
    char kernel_desc[512] = {0};
    size_t tma_smem = 0;
    TmaArgs tma{};
    int have_state = 0;
    unsigned long long wait_ns = 1000000000ull;  // limit of a bounded device wait (1 s)
    int withhold = 0;                            // test hook: the next bulk-copy launch withholds a load
    int odd = 0;  // parity of the next step (1: populations are post-collision, swapped)
    long long done = 0;
    int slab_next = 0;  // next x of a state loaded in slabs
    // wall-normal slab of a channel split over several GPUs
    // (dnslbm_create_slab): the context holds fluid planes [z0, z0 + nz) of a
    // channel of nz_all planes, each population array with one ghost plane
    // on either side (pop_off elements from the array's start to plane 0)
    int slab = 0, z0 = 0, nz_all = 0;
    int wall_lo = 1, wall_hi = 1;
    size_t pop_off = 0;
    double *shift_all = nullptr;  // [2][nz_all][3] the channel's plane means (slab tail)
    int tail_owed = -1;           // the slab tail the caller owes: 1 after a load, 0 after a step, -1 none
    char err[512] = {0};
};

static thread_local char g_create_err[512];

static int fail(dnslbm_ctx *c, int code, const char *fmt, ...)
{
    char *dst = c ? c->err : g_create_err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(dst, 512, fmt, ap);
    va_end(ap);
    return code;
}

#define CK(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return fail(c, DNSLBM_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

static StepArgs step_args(const dnslbm_ctx *c)
{
    StepArgs p;
    for (int a = 0; a < Q; ++a) p.pop[a] = (char *)c->popmem + ((size_t)a * c->pstride + c->pop_off) * c->esize;
    p.nx = c->nx;
    p.ny = c->ny;
    p.nz = c->nz;
    p.pitch = c->pitch;
    p.rows = c->rows;
    p.slots = c->slots;
    p.wallmask = c->wallmask;
    p.omega = c->deck.omega;
    p.ubulk = c->deck.ubulk;
    p.gx = c->deck.gx;
    p.const_q = c->deck.force_mode == DNSLBM_FORCE_CONST_Q;
    p.force = c->force;
    p.shift = c->shift;
    p.step_ctr = c->step_ctr;
    p.partials = c->partials;
    p.plane_sums = c->plane_sums;
    p.plane_ctr = c->plane_ctr;
    p.total_ctr = c->total_ctr;
    p.logs = c->logs;
    p.log_cap = c->deck.log_capacity;
    p.status = c->status;
    p.band_of = c->band_of;
    p.links = c->links;
    p.wait_ns = c->wait_ns;
    p.withhold_stage = 0;
    p.wall_lo = c->wall_lo;
    p.wall_hi = c->wall_hi;
    p.tail = c->slab ? 0 : 1;
    return p;
}

static IoArgs io_args(const dnslbm_ctx *c)
{
    IoArgs p;
    for (int a = 0; a < Q; ++a) p.pop[a] = (char *)c->popmem + ((size_t)a * c->pstride + c->pop_off) * c->esize;
    p.nx = c->nx;
    p.ny = c->ny;
    p.nz = c->nz;
    p.pitch = c->pitch;
    p.wallmask = c->wallmask;
    p.textured = c->textured;
    p.odd = c->odd;
    p.band_of = c->band_of;
    p.links = c->links;
    return p;
}

static void free_all(dnslbm_ctx *c)
{
    void *ptrs[] = {c->popmem,     c->wallmask,   c->force,         c->shift,       c->partials,
                    c->plane_sums, c->logs,       c->step_ctr,      c->status,      c->plane_ctr,
                    c->total_ctr,  c->staging,    c->stat_partials, c->stat_planes, c->stat_mean,
                    c->band_of,    c->links,      c->plane_list,    c->d_llaunch,   c->stat_acc,
                    c->out_lbf,    c->out_vel,    c->out_den,       c->out_stats,   c->quad_buf,
                    c->shift_all};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (auto &e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : c->tev)
        if (e) cudaEventDestroy(e);
    for (auto &e : c->fj)
        if (e) cudaEventDestroy(e);
    for (auto &e : c->out_ev)
        if (e) cudaEventDestroy(e);
    if (c->out_stream) cudaStreamDestroy(c->out_stream);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->stream) cudaStreamDestroy(c->stream);
}

extern "C" const char *dnslbm_last_error(const dnslbm_ctx *c) { return c ? c->err : g_create_err; }

// Configure the row-pipelined step with k rows per stage group, `stages`
// groups in flight and `consumers` compute threads (+ one producer warp);
// bps > 0 caps the blocks per SM.  Returns 0 when the configuration runs on
// this device (and selects it), -1 otherwise (the previous choice stays).
// Dynamic shared memory the step kernels may be given: the device's opt-in
// maximum less this reserve for their static shared memory (about 2.5 KB).
constexpr size_t kStaticSmemReserve = 4096;

// Row groups of the row-pipelined kernel over its planes (all planes, or the
// planes without link masks) shared among tma_target blocks.
static void tma_layout_of(dnslbm_ctx *c, TmaArgs &t, int target, int &grid)
{
    const int ngroups = t.gpp * c->nclean;
    target = std::max(1, target);
    const int GB = std::max(1, (ngroups + target - 1) / target);
    t.ngroups = ngroups;
    t.groups_per_block = GB;
    t.planes = c->nclean < c->nz ? c->plane_list : nullptr;
    grid = (ngroups + GB - 1) / GB;
}

static void tma_layout(dnslbm_ctx *c)
{
    tma_layout_of(c, c->tma, c->tma_target, c->tma_grid);
    if (c->odd_split) tma_layout_of(c, c->odd_tma, c->odd_target, c->odd_grid);
}

// seg > 0 (FP64 only): groups are x-segments of seg elements (even) of one
// row, for rows too long for two whole-row stages.
constexpr int kMaxSegments = 4;
static int tma_configure(dnslbm_ctx *c, int k, int stages, int consumers, int bps, int seg = 0)
{
    const int row_bytes = c->pitch * (int)c->esize;
    k = std::max(1, std::min(k, c->ny));
    consumers = std::max(32, std::min(352, consumers / 32 * 32));
    if (seg > 0 && (c->deck.precision != 64 || seg % 2 || seg >= c->nx)) return -1;
    if (seg > 0) k = 1;
    const int nseg = seg > 0 ? (c->nx + seg - 1) / seg : 1;
    if (nseg > kMaxSegments) return -1;  // more groups per plane than partial-sum slots
    const int dir_elems = seg > 0 ? seg + 4 : k * c->pitch;  // a segment keeps a halo of 2 elements a side
    const size_t smem_stage = (size_t)Q * dir_elems * c->esize;
    int maxsmem = 0, nsm = 0;
    cudaDeviceGetAttribute(&maxsmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->deck.device);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->deck.device);
    const size_t smem = (size_t)stages * smem_stage + 16 * (size_t)stages;  // + full/empty mbarriers
    const size_t cap = (size_t)maxsmem - kStaticSmemReserve;  // room for the kernels' static shared memory
    if (stages < 2 || smem > cap || nsm <= 0) return -1;
    const int threads = consumers + 32;
    const bool const_q = c->deck.force_mode == DNSLBM_FORCE_CONST_Q;
    // the kernels may use up to the device's opt-in shared memory (a batch can
    // give a channel a larger stage than its own shape)
    const int prep = c->deck.precision == 64 ? tma_prepare_f64(cap) : tma_prepare_lp(c->deck.precision, cap);
    int occ = prep ? 0
                   : (c->deck.precision == 64 ? tma_occupancy_f64(threads, smem, const_q)
                                              : tma_occupancy_lp(c->deck.precision, threads, smem, const_q));
    cudaGetLastError();  // a failed query only rules the configuration out
    if (bps > 0) occ = std::min(occ, bps);
    if (occ < 1) return -1;
    const int gpp = (c->ny + k - 1) / k * nseg;
    c->use_tma = 1;
    c->odd_split = 0;
    c->tma_threads = threads;
    c->tma_smem = smem;
    c->tma_target = occ * nsm;
    c->tma = TmaArgs{0, 1, stages, row_bytes, k, gpp, nullptr, nseg, seg > 0 ? seg : c->nx, dir_elems};
    tma_layout(c);
    return 0;
}

// x-segment length (even) that splits rows of nx into nseg near-equal parts.
static int segment_for(int nx, int nseg) { return ((nx + nseg - 1) / nseg + 1) & ~1; }

static void describe_kernel(dnslbm_ctx *c)
{
    if (c->use_tma) {
        int m = snprintf(c->kernel_desc, sizeof c->kernel_desc,
                         "step_tma_kernel<fp%d> row-pipelined bulk-copy: %d blocks x %d threads, %d groups of %d "
                         "rows/block, %d stages, %zu B smem",
                         c->deck.precision, c->tma_grid, c->tma_threads, c->tma.groups_per_block, c->tma.k,
                         c->tma.stages, c->tma_smem);
        if (c->tma.nseg > 1 && m > 0 && m < (int)sizeof c->kernel_desc)
            m += snprintf(c->kernel_desc + m, sizeof c->kernel_desc - m, ", rows in %d x-segments of %d", c->tma.nseg,
                          c->tma.seg);
        if (c->odd_split && m > 0 && m < (int)sizeof c->kernel_desc)
            m += snprintf(c->kernel_desc + m, sizeof c->kernel_desc - m,
                          "; odd steps: %d blocks x %d threads, %d groups of %d rows/block, %d stages, %zu B smem",
                          c->odd_grid, c->odd_threads, c->odd_tma.groups_per_block, c->odd_tma.k, c->odd_tma.stages,
                          c->odd_smem);
        if (c->ndirty > 0 && m > 0 && m < (int)sizeof c->kernel_desc)
            snprintf(c->kernel_desc + m, sizeof c->kernel_desc - m, " + links_pass_kernel over %d planes", c->ndirty);
    } else {
        snprintf(c->kernel_desc, sizeof c->kernel_desc, "%s per-thread: grid %ux%ux%u x %u threads",
                 c->deck.precision == 64 ? "step_f64_kernel" : "step_lp_kernel", c->grid.x, c->grid.y, c->grid.z,
                 c->block.x);
    }
}

// plane_list: the planes without link masks, then those with them
static cudaError_t upload_planes(dnslbm_ctx *c, const std::vector<int> *band = nullptr)
{
    std::vector<int> pl;
    for (int z = 0; z < c->nz; ++z)
        if (!band || (*band)[z] < 0) pl.push_back(z);
    c->nclean = (int)pl.size();
    for (int z = 0; z < c->nz; ++z)
        if (band && (*band)[z] >= 0) pl.push_back(z);
    c->ndirty = c->nz - c->nclean;
    c->plane_host = pl;
    return cudaMemcpy(c->plane_list, pl.data(), pl.size() * sizeof(int), cudaMemcpyHostToDevice);
}

// A whole channel (slab = 0) or the wall-normal slab [z0, z0 + nzs) of one
// (slab = 1, dnslbm_create_slab).
static int create_ctx(const dnslbm_deck *deck, int slab, int z0, int nzs, dnslbm_ctx **out)
{
    dnslbm_ctx *c = nullptr;
    if (!deck || !out) return fail(c, DNSLBM_ERR_ARG, "null deck or output pointer");
    *out = nullptr;
    if (slab) {
        if (z0 < 0 || nzs < 2 || (long long)z0 + nzs > deck->zdv)
            return fail(c, DNSLBM_ERR_ARG, "slab of planes [%d, %d) is not a range of at least 2 of the %d planes", z0,
                        z0 + nzs, deck->zdv);
        if (deck->bc_mode != DNSLBM_BC_REFERENCE)
            return fail(c, DNSLBM_ERR_ARG, "slabs take the reference boundary mode (no solids inside the flow)");
    }
    if (deck->xdv < 2 || deck->ydv < 2 || deck->zdv < 3)
        return fail(c, DNSLBM_ERR_ARG, "grid %dx%dx%d too small (need xdv,ydv >= 2, zdv >= 3)", deck->xdv, deck->ydv,
                    deck->zdv);
    if (deck->ydv > 65535)
        return fail(c, DNSLBM_ERR_ARG, "ydv %d above 65535 (one grid row of blocks per y in the state I/O)", deck->ydv);
    if ((long long)(deck->xdv + 8) * deck->ydv * deck->zdv >= (1LL << 31))
        return fail(c, DNSLBM_ERR_ARG, "grid of %lld cells exceeds 2^31", (long long)deck->xdv * deck->ydv * deck->zdv);
    if (!(deck->omega > 0.0 && deck->omega < 2.0)) return fail(c, DNSLBM_ERR_ARG, "omega %g outside (0,2)", deck->omega);
    if (deck->precision != 64 && deck->precision != 32 && deck->precision != 16)
        return fail(c, DNSLBM_ERR_ARG, "precision %d not one of 64, 32, 16", deck->precision);
    if (deck->force_mode != DNSLBM_FORCE_CONST_Q && deck->force_mode != DNSLBM_FORCE_CONST_G)
        return fail(c, DNSLBM_ERR_ARG, "unknown force mode %d", deck->force_mode);
    if (deck->bc_mode != DNSLBM_BC_REFERENCE && deck->bc_mode != DNSLBM_BC_GENERAL)
        return fail(c, DNSLBM_ERR_ARG, "unknown bc mode %d", deck->bc_mode);
    if (deck->log_capacity < 0) return fail(c, DNSLBM_ERR_ARG, "negative log capacity");

    c = new dnslbm_ctx();
    c->deck = *deck;
    if (c->deck.log_capacity == 0) c->deck.log_capacity = 4096;
    c->nx = deck->xdv;
    c->ny = deck->ydv;
    c->nz = slab ? nzs : deck->zdv;
    c->slab = slab;
    c->z0 = slab ? z0 : 0;
    c->nz_all = deck->zdv;
    c->wall_lo = c->z0 == 0;
    c->wall_hi = c->z0 + c->nz == deck->zdv;
    c->nclean = c->nz;
    c->esize = deck->precision / 8;
    {
        // rows start on `align` bytes (16 at least, for the bulk copies).
        // Measured on 628-wide rows: FP32 is faster unpadded (16 bytes: 628,
        // not 632 elements), FP16 faster on 32 bytes (640, not 632); FP64
        // rows of 628 are 32-byte multiples either way.
        int align_bytes = c->esize == 4 ? 16 : 32;
        if (const char *e = getenv("DNSLBM_ROW_ALIGN")) align_bytes = std::max(16, atoi(e));
        const int v = align_bytes / (int)c->esize;
        c->pitch = (c->nx + v - 1) / v * v;
    }
    c->ncell = (size_t)c->pitch * c->ny * c->nz;
    const size_t align = 256 / c->esize;
    if (slab) {
        // a ghost plane on either side: plane -1 just below plane 0, plane
        // nz just above plane nz-1; plane 0 starts on 256 bytes
        const size_t plane = (size_t)c->pitch * c->ny;
        c->pop_off = (plane + align - 1) / align * align;
        c->ncell = c->pop_off + (size_t)(c->nz + 1) * plane;
    }
    c->pstride = (c->ncell + align - 1) / align * align;

    int rc = DNSLBM_OK;
    auto bail = [&](int code) {
        snprintf(g_create_err, sizeof g_create_err, "%s", c->err);
        free_all(c);
        delete c;
        return code;
    };
    if (cudaSetDevice(deck->device) != cudaSuccess) {
        fail(c, DNSLBM_ERR_CUDA, "cannot select CUDA device %d", deck->device);
        return bail(DNSLBM_ERR_CUDA);
    }
    // launch shape: BX threads along x, `rows` rows of y per block, one plane per grid z
    int bx = ((c->nx + 31) / 32) * 32;
    if (bx > 128) bx = 128;
    c->block = dim3(bx, 1, 1);
    c->grid = dim3((c->nx + bx - 1) / bx, (c->ny + c->rows - 1) / c->rows, c->nz);
    // partial-sum slots per plane: enough for the per-thread kernels and for
    // any split of a plane's row groups among blocks (at most one per group,
    // plus one; x-segmented FP64 rows: kMaxSegments groups per row)
    c->slots = std::max((int)(c->grid.x * c->grid.y), (deck->precision == 64 ? kMaxSegments : 1) * c->ny + 1);
    {
        // Row-pipelined step.  A stage holds a group of k consecutive rows of
        // one plane for all 19 directions.  Defaults measured on a B200
        // (628-wide rows): two stages of about 48 KB (FP16) to 96 KB
        // (FP32/FP64) per block; consumer threads about 2 cells each for FP64
        // (at most 320), 3 for FP32 (at most 192), 5 for FP16 (at most 128, so
        // two blocks share an SM).  dnslbm_autotune replaces them by measured
        // choices; the DNSLBM_* environment variables override them.
        const char *path = getenv("DNSLBM_PATH");
        const int row_bytes = c->pitch * (int)c->esize;
        const size_t stage_target = c->deck.precision == 16 ? 49152 : 98304;
        int k = 1;
        while (k < 8 && k * 2 <= c->ny && (size_t)Q * row_bytes * k * 2 <= stage_target) k *= 2;
        if (const char *e = getenv("DNSLBM_GROUP_ROWS")) k = std::max(1, std::min(atoi(e), c->ny));
        int stages = 2;
        if (const char *e = getenv("DNSLBM_STAGES")) stages = atoi(e);
        const int cap = c->deck.precision == 64 ? 320 : (c->deck.precision == 32 ? 192 : 128);
        int consumers = std::min(cap, (c->nx + 31) / 32 * 32);
        if (const char *e = getenv("DNSLBM_THREADS")) consumers = atoi(e) / 32 * 32;
        int bps = 0;
        if (const char *e = getenv("DNSLBM_BLOCKS_PER_SM")) bps = atoi(e);
        if (!(path && !strcmp(path, "scalar"))) {
            int seg = 0;
            if (const char *e = getenv("DNSLBM_SEGMENT")) seg = atoi(e) & ~1;
            if (seg > 0 || tma_configure(c, k, stages, consumers, bps)) {
                // FP64 rows too long for two whole-row stages: x-segments
                for (int nseg = 2; seg == 0 && c->deck.precision == 64 && nseg <= kMaxSegments; ++nseg)
                    if (!tma_configure(c, 1, stages, consumers, bps, segment_for(c->nx, nseg))) break;
                if (seg > 0) tma_configure(c, 1, stages, consumers, bps, seg);
            }
        }
        describe_kernel(c);
    }
    if (slab && !c->use_tma) {
        fail(c, DNSLBM_ERR_ARG, "slab contexts step with the row-pipelined kernel, which this grid cannot take");
        return bail(DNSLBM_ERR_ARG);
    }
    const size_t nblocks = (size_t)c->nz * c->slots;

    struct Alloc { void **p; size_t bytes; };
    c->staging_bytes = std::min<size_t>((size_t)256 << 20, (size_t)c->ny * (c->nz + 2) * Q * sizeof(double) * c->nx);
    const size_t row_bytes = (size_t)c->ny * (c->nz + 2) * Q * sizeof(double);
    if (c->staging_bytes < row_bytes) c->staging_bytes = row_bytes;
    Alloc al[] = {
        {&c->popmem, (size_t)Q * c->pstride * c->esize},
        {(void **)&c->wallmask, (size_t)2 * c->nx * c->ny},
        {(void **)&c->force, 2 * sizeof(double)},
        {(void **)&c->shift, (size_t)2 * c->nz * 3 * sizeof(double)},
        {(void **)&c->partials, nblocks * NP * sizeof(double)},
        {(void **)&c->plane_sums, (size_t)c->nz * NP * sizeof(double)},
        {(void **)&c->logs, (size_t)c->deck.log_capacity * 9 * sizeof(double)},
        {(void **)&c->step_ctr, sizeof(long long)},
        {(void **)&c->status, 2 * sizeof(long long)},
        {(void **)&c->plane_ctr, (size_t)c->nz * sizeof(unsigned)},
        {(void **)&c->total_ctr, sizeof(unsigned)},
        {(void **)&c->staging, c->staging_bytes},
        {(void **)&c->stat_partials, nblocks * 5 * sizeof(double)},
        {(void **)&c->stat_planes, (size_t)c->nz * 5 * sizeof(double)},
        {(void **)&c->stat_mean, (size_t)c->nz * 4 * sizeof(double)},
        {(void **)&c->band_of, (size_t)c->nz * sizeof(int)},
        {(void **)&c->plane_list, (size_t)c->nz * sizeof(int)},
        {(void **)&c->stat_acc, (size_t)9 * c->nz * sizeof(double)},
        {(void **)&c->d_llaunch, sizeof(LinksLaunch)},
    };
    for (auto &a : al) {
        cudaError_t e = cudaMalloc(a.p, a.bytes);
        if (e != cudaSuccess) {
            fail(c, DNSLBM_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", a.bytes, cudaGetErrorString(e));
            return bail(DNSLBM_ERR_NOMEM);
        }
        cudaMemset(*a.p, 0, a.bytes);
    }
    if (slab) {
        const size_t bytes = (size_t)2 * c->nz_all * 3 * sizeof(double);
        if (cudaMalloc((void **)&c->shift_all, bytes) != cudaSuccess) {
            fail(c, DNSLBM_ERR_NOMEM, "cudaMalloc of %zu bytes failed", bytes);
            return bail(DNSLBM_ERR_NOMEM);
        }
        cudaMemset(c->shift_all, 0, bytes);
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->out_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->out_ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->out_ev[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->fj[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->fj[1], cudaEventDisableTiming) != cudaSuccess) {
        fail(c, DNSLBM_ERR_CUDA, "cannot create streams");
        return bail(DNSLBM_ERR_CUDA);
    }
    for (auto &e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            fail(c, DNSLBM_ERR_CUDA, "cannot create event");
            return bail(DNSLBM_ERR_CUDA);
        }
    // default flags: smooth no-slip walls (solid_init.c), no solid inside
    std::vector<uint8_t> m((size_t)2 * c->nx * c->ny, 0x1f);
    if (cudaMemcpy(c->wallmask, m.data(), m.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(c->band_of, 0xff, (size_t)c->nz * sizeof(int)) != cudaSuccess ||
        upload_planes(c) != cudaSuccess ||
        cudaDeviceSynchronize() != cudaSuccess) {
        fail(c, DNSLBM_ERR_CUDA, "initialisation failed: %s", cudaGetErrorString(cudaGetLastError()));
        return bail(DNSLBM_ERR_CUDA);
    }
    (void)rc;
    *out = c;
    return DNSLBM_OK;
}

extern "C" int dnslbm_create(const dnslbm_deck *deck, dnslbm_ctx **out) { return create_ctx(deck, 0, 0, 0, out); }

extern "C" int dnslbm_create_slab(const dnslbm_deck *deck, int z0, int nzs, dnslbm_ctx **out)
{
    return create_ctx(deck, 1, z0, nzs, out);
}

extern "C" void dnslbm_destroy(dnslbm_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->deck.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_all(c);
    delete c;
}

static int initial_reduce(dnslbm_ctx *c);

// wall-link bits from the wall-plane flags (xcomputations.c:368-375): the
// link from fluid cell P toward wall cell T bounces back iff s(T) == -1 and
// s(P's own wall cell) == -1; otherwise it reflects specularly.
//
// Boundary mode DNSLBM_BC_GENERAL also takes solid cells (-1) inside the
// flow.  Every plane within one plane of such a cell gets per-cell link
// masks (cell_links): a link from a fluid cell bounces back when its target
// is solid, when both wall cells of the wall rule are no-slip, or when the
// specular reflection would land on a solid cell; the remaining links into a
// wall plane reflect specularly and all others stream.  Solid cells keep the
// rest state.
// The host-side tables of a flag array: the wall-link bits of the two
// wall-adjacent planes, the planes with link masks and the masks.  Pure host
// computation; `err` receives the reason of a refusal.
struct FlagTables {
    std::vector<uint8_t> wallmask;  // [2][ny][nx]
    std::vector<int> band;          // [nz], -1: no masks
    std::vector<unsigned> links;    // [nband][ny][nx]
    int nband = 0;
    int textured = 0;  // 0 smooth walls, 1 textured walls, 2 solids inside the flow
};

static int build_flag_tables(int nx, int ny, int nz, bool general, const int8_t *fl /* [nx][ny][zd] */,
                             FlagTables &t, char *err, size_t errlen)
{
    const int zd = nz + 2;
    auto S = [&](int x, int y, int k) { return (int)fl[((size_t)x * ny + y) * zd + k]; };
    std::vector<char> has_solid(nz, 0);
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
            for (int k : {0, zd - 1}) {
                const int v = S(x, y, k);
                if (v != -1 && v != -2) {
                    snprintf(err, errlen, "wall cell (%d,%d,%d) has flag %d; wall planes must be -1 or -2", x, y, k,
                             v);
                    return DNSLBM_ERR_ARG;
                }
            }
            for (int k = 1; k < zd - 1; ++k) {
                const int v = S(x, y, k);
                if (v == -1 && general) {
                    has_solid[k - 1] = 1;
                    continue;
                }
                if (v != 0 && v != 1) {
                    snprintf(err, errlen,
                             general ? "cell (%d,%d,%d) has flag %d; inside the flow a cell is fluid (0, 1) or solid (-1)"
                                     : "cell (%d,%d,%d) has flag %d; solids inside the flow need the general boundary "
                                       "mode (DNSLBM_BC_GENERAL)",
                             x, y, k, v);
                    return DNSLBM_ERR_ARG;
                }
            }
        }
    t.wallmask.assign((size_t)2 * nx * ny, 0);
    const int off[5][2] = {{0, 0}, {1, 0}, {-1, 0}, {0, 1}, {0, -1}};
    t.textured = 0;
    for (int w = 0; w < 2; ++w) {
        const int k = w == 0 ? 0 : zd - 1;
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                unsigned bits = 0;
                for (int l = 0; l < 5; ++l) {
                    const int xt = (x + off[l][0] + nx) % nx, yt = (y + off[l][1] + ny) % ny;
                    if (S(xt, yt, k) == -1 && S(x, y, k) == -1) bits |= 1u << l;
                }
                t.wallmask[(size_t)w * nx * ny + (size_t)y * nx + x] = (uint8_t)bits;
                if (bits != 0x1f) t.textured = 1;
            }
    }
    // planes with link masks
    t.band.assign(nz, -1);
    t.nband = 0;
    for (int z = 0; z < nz; ++z)
        if (has_solid[z] || (z > 0 && has_solid[z - 1]) || (z + 1 < nz && has_solid[z + 1])) t.band[z] = t.nband++;
    t.links.assign((size_t)t.nband * ny * nx, 0u);
    for (int z = 0; z < nz; ++z) {
        if (t.band[z] < 0) continue;
        const int k = z + 1;
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                unsigned v = 0;
                if (S(x, y, k) == -1) {
                    v = 1u;
                } else {
                    for (int a = 1; a < Q; ++a) {
                        const int xt = (x + lat_ex(a) + nx) % nx, yt = (y + lat_ey(a) + ny) % ny, kt = k + lat_ez(a);
                        const int sld = S(xt, yt, kt), sld1 = S(x, y, kt);
                        bool bounce;
                        if (sld > -1) bounce = false;
                        else if (sld == -1 && sld1 == -1) bounce = true;
                        else if ((sld == -1 && sld1 == -2) || sld == -2) bounce = S(xt, yt, k) == -1;
                        else bounce = true;
                        if (bounce) v |= 1u << a;
                    }
                }
                t.links[((size_t)t.band[z] * ny + y) * nx + x] = v;
            }
    }
    if (t.nband > 0) t.textured = 2;
    return DNSLBM_OK;
}

extern "C" int dnslbm_link_masks(int xdv, int ydv, int zdv, int bc_mode, const int8_t *flags, int *band_of,
                                 unsigned *links, size_t links_capacity, int *nband)
{
    dnslbm_ctx *c = nullptr;
    if (!flags || !band_of || !nband || xdv < 1 || ydv < 1 || zdv < 1)
        return fail(c, DNSLBM_ERR_ARG, "bad grid or null argument");
    FlagTables t;
    char err[256];
    int rc = build_flag_tables(xdv, ydv, zdv, bc_mode == DNSLBM_BC_GENERAL, flags, t, err, sizeof err);
    if (rc) return fail(c, rc, "%s", err);
    *nband = t.nband;
    for (int z = 0; z < zdv; ++z) band_of[z] = t.band[z];
    if (t.links.size() > links_capacity || (!links && !t.links.empty()))
        return fail(c, DNSLBM_ERR_ARG, "link masks need %zu entries, %zu given", t.links.size(), links_capacity);
    std::copy(t.links.begin(), t.links.end(), links);
    return DNSLBM_OK;
}

static int apply_flags(dnslbm_ctx *c, const int8_t *fl /* [nx][ny][zd] */)
{
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    std::vector<int8_t> view;
    if (c->slab) {
        // the whole channel's flags -> the slab's planes k = z0 .. z0 + nz + 1,
        // a side that faces a neighbour slab reading as a no-slip wall plane
        // (its wall-link bits are never used: plane_wall is 0 there)
        const int zd_all = c->nz_all + 2, zd = nz + 2;
        view.resize((size_t)nx * ny * zd);
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y)
                for (int kk = 0; kk < zd; ++kk) {
                    const bool ghost = (kk == 0 && !c->wall_lo) || (kk == zd - 1 && !c->wall_hi);
                    view[((size_t)x * ny + y) * zd + kk] =
                        ghost ? (int8_t)-1 : fl[((size_t)x * ny + y) * zd_all + c->z0 + kk];
                }
        fl = view.data();
    }
    FlagTables t;
    char err[256];
    const int brc = build_flag_tables(nx, ny, nz, c->deck.bc_mode == DNSLBM_BC_GENERAL, fl, t, err, sizeof err);
    if (brc) return fail(c, brc, "%s", err);
    if (c->have_state && c->odd) {
        // the populations in flight were placed under the old flags
        return fail(c, DNSLBM_ERR_STATE, "flags can only change between even numbers of steps");
    }
    std::vector<uint8_t> &m = t.wallmask;
    std::vector<int> &band = t.band;
    std::vector<unsigned> &lk = t.links;
    const int nband = t.nband, textured = t.textured;
    CK(cudaSetDevice(c->deck.device));
    const size_t lbytes = lk.size() * sizeof(unsigned);
    if (lbytes > c->links_bytes) {
        if (c->links) CK(cudaFree(c->links));
        c->links = nullptr;
        c->links_bytes = 0;
        cudaError_t e = cudaMalloc(&c->links, lbytes);
        if (e != cudaSuccess) return fail(c, DNSLBM_ERR_NOMEM, "cudaMalloc of %zu bytes of link masks failed", lbytes);
        c->links_bytes = lbytes;
    }
    CK(cudaMemcpyAsync(c->wallmask, m.data(), m.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->band_of, band.data(), band.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    if (lbytes) CK(cudaMemcpyAsync(c->links, lk.data(), lbytes, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->walls_textured = 0;
    for (size_t i = 0; i < m.size() && !c->walls_textured; ++i) c->walls_textured = m[i] != 0x1f;
    c->textured = textured;
    c->nband = nband;
    CK(upload_planes(c, &band));
    {
        LinksLaunch L{};
        L.p = step_args(c);
        L.planes = c->plane_list + c->nclean;
        L.nplanes = c->ndirty;
        L.xblocks = (int)c->grid.x;
        L.yblocks = (int)c->grid.y;
        L.rows = c->rows;
        L.first_block = 0;
        CK(cudaMemcpy(c->d_llaunch, &L, sizeof L, cudaMemcpyHostToDevice));
    }
    if (c->use_tma) tma_layout(c);
    describe_kernel(c);
    if (textured == 2 && c->have_state) {
        // cells that became solid take the rest state; the sums of the
        // current step are taken again
        launch_io(c->deck.precision, 4, io_args(c), 0, 0, nullptr, nullptr, c->stream);
        CK(cudaGetLastError());
        return initial_reduce(c);
    }
    return DNSLBM_OK;
}

extern "C" int dnslbm_set_flags_periodic(dnslbm_ctx *c, const int8_t *flags)
{
    if (!c || !flags) return fail(c, DNSLBM_ERR_ARG, "null argument");
    return apply_flags(c, flags);
}

extern "C" int dnslbm_set_flags(dnslbm_ctx *c, const int *s)
{
    if (!c || !s) return fail(c, DNSLBM_ERR_ARG, "null argument");
    const int nx = c->nx, ny = c->ny, zd = (c->slab ? c->nz_all : c->nz) + 2, yd = ny + 1;
    std::vector<int8_t> fl((size_t)nx * ny * zd);
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int k = 0; k < zd; ++k) {
                int v = s[((size_t)x * yd + y) * zd + k];
                fl[((size_t)x * ny + y) * zd + k] = (int8_t)(v == 1 ? 0 : v);
            }
    return apply_flags(c, fl.data());
}

// initial reduction of a freshly set state: force and plane means of step 0
// (a slab leaves its plane sums to the caller, who owes dnslbm_slab_tail)
static int initial_reduce(dnslbm_ctx *c)
{
    StepArgs p = step_args(c);
    if (c->deck.precision == 64) launch_reduce_f64(p, c->grid, c->block, c->stream);
    else launch_reduce_lp(c->deck.precision, p, c->grid, c->block, c->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    c->tail_owed = c->slab ? 1 : -1;
    return DNSLBM_OK;
}

static int reset_counters(dnslbm_ctx *c)
{
    CK(cudaMemsetAsync(c->plane_ctr, 0, (size_t)c->nz * sizeof(unsigned), c->stream));
    CK(cudaMemsetAsync(c->total_ctr, 0, sizeof(unsigned), c->stream));
    CK(cudaMemsetAsync(c->step_ctr, 0, sizeof(long long), c->stream));
    CK(cudaMemsetAsync(c->status, 0, 2 * sizeof(long long), c->stream));
    CK(cudaMemsetAsync(c->shift, 0, (size_t)2 * c->nz * 3 * sizeof(double), c->stream));
    if (c->shift_all) CK(cudaMemsetAsync(c->shift_all, 0, (size_t)2 * c->nz_all * 3 * sizeof(double), c->stream));
    c->done = 0;
    c->odd = 0;
    c->tail_owed = -1;
    return DNSLBM_OK;
}

extern "C" int dnslbm_init_rest(dnslbm_ctx *c)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    CK(cudaSetDevice(c->deck.device));
    int rc = reset_counters(c);
    if (rc) return rc;
    IoArgs p = io_args(c);
    launch_io(c->deck.precision, 2, p, 0, 0, nullptr, nullptr, c->stream);
    CK(cudaGetLastError());
    c->have_state = 1;
    return initial_reduce(c);
}

extern "C" int dnslbm_load_state(dnslbm_ctx *c, const double *state)
{
    if (!c || !state) return fail(c, DNSLBM_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->deck.device));
    int rc = reset_counters(c);
    if (rc) return rc;
    IoArgs p = io_args(c);
    const size_t slab = (size_t)c->ny * (c->nz + 2) * Q;  // doubles per x
    const int xchunk = (int)std::max<size_t>(1, c->staging_bytes / (slab * sizeof(double)));
    for (int x0 = 0; x0 < c->nx; x0 += xchunk) {
        const int n = std::min(xchunk, c->nx - x0);
        CK(cudaMemcpyAsync(c->staging, state + (size_t)x0 * slab, (size_t)n * slab * sizeof(double),
                           cudaMemcpyHostToDevice, c->stream));
        launch_io(c->deck.precision, 1, p, x0, n, c->staging, nullptr, c->stream);
        CK(cudaGetLastError());
    }
    c->have_state = 1;
    return initial_reduce(c);
}

extern "C" int dnslbm_load_state_slab(dnslbm_ctx *c, int x0, int nxs, const double *slab)
{
    if (!c || !slab) return fail(c, DNSLBM_ERR_ARG, "null argument");
    if (nxs < 1 || x0 < 0 || x0 + nxs > c->nx)
        return fail(c, DNSLBM_ERR_ARG, "slab x in [%d, %d) is not inside [0, %d)", x0, x0 + nxs, c->nx);
    if (x0 != 0 && x0 != c->slab_next)
        return fail(c, DNSLBM_ERR_STATE, "slabs come in order of x: expected x0 = %d (or 0 to start over), got %d",
                    c->slab_next, x0);
    CK(cudaSetDevice(c->deck.device));
    if (x0 == 0) {
        int rc = reset_counters(c);
        if (rc) return rc;
        c->have_state = 0;
    }
    IoArgs p = io_args(c);
    const size_t plane = (size_t)c->ny * (c->nz + 2) * Q;  // doubles per x
    const int xchunk = (int)std::max<size_t>(1, c->staging_bytes / (plane * sizeof(double)));
    for (int i = 0; i < nxs; i += xchunk) {
        const int n = std::min(xchunk, nxs - i);
        CK(cudaMemcpyAsync(c->staging, slab + (size_t)i * plane, (size_t)n * plane * sizeof(double),
                           cudaMemcpyHostToDevice, c->stream));
        launch_io(c->deck.precision, 1, p, x0 + i, n, c->staging, nullptr, c->stream);
        CK(cudaGetLastError());
    }
    c->slab_next = x0 + nxs;
    if (c->slab_next < c->nx) {
        CK(cudaStreamSynchronize(c->stream));  // the caller may reuse its slab buffer
        return DNSLBM_OK;
    }
    c->slab_next = 0;
    c->have_state = 1;
    return initial_reduce(c);
}

// Readers of the state need one; a slab is read between even numbers of
// steps only (after an even step a reader gathers across the ghost planes,
// which mirror the neighbour slabs only around an odd step).
static int readable(dnslbm_ctx *c)
{
    if (!c->have_state) return fail(c, DNSLBM_ERR_STATE, "no state loaded");
    if (c->slab && c->odd) return fail(c, DNSLBM_ERR_STATE, "a slab is read after an even number of steps only");
    return DNSLBM_OK;
}

extern "C" int dnslbm_store_state(dnslbm_ctx *c, double *state)
{
    if (!c || !state) return fail(c, DNSLBM_ERR_ARG, "null argument");
    if (int rc_ = readable(c)) return rc_;
    CK(cudaSetDevice(c->deck.device));
    IoArgs p = io_args(c);
    const size_t slab = (size_t)c->ny * (c->nz + 2) * Q;
    const int xchunk = (int)std::max<size_t>(1, c->staging_bytes / (slab * sizeof(double)));
    for (int x0 = 0; x0 < c->nx; x0 += xchunk) {
        const int n = std::min(xchunk, c->nx - x0);
        CK(cudaMemsetAsync(c->staging, 0, (size_t)n * slab * sizeof(double), c->stream));
        launch_io(c->deck.precision, 0, p, x0, n, c->staging, nullptr, c->stream);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(state + (size_t)x0 * slab, c->staging, (size_t)n * slab * sizeof(double),
                           cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return DNSLBM_OK;
}

static int launch_steps(dnslbm_ctx *c, long n, bool timed, double *ms_even, double *ms_odd)
{
    StepArgs p = step_args(c);
    // timed: an event pair around every launch, read after one final sync
    // (no host round trip between launches)
    if (timed && c->tev.size() < (size_t)(2 * n)) {
        const size_t old = c->tev.size();
        c->tev.resize((size_t)(2 * n), nullptr);
        for (size_t i = old; i < c->tev.size(); ++i) CK(cudaEventCreate(&c->tev[i]));
    }
    const int first_parity = c->odd;
    for (long s = 0; s < n; ++s) {
        const bool odd = c->odd != 0;
        if (timed) CK(cudaEventRecord(c->tev[2 * s], c->stream));
        if (c->use_tma) {
            if (c->withhold && c->tma.ngroups > 0) {  // test hook, one launch only
                p.withhold_stage = 1;
                c->withhold = 0;
            } else {
                p.withhold_stage = 0;
            }
            // the row-pipelined kernel over its planes and, beside it on a
            // second stream, the planes with link masks per cell (disjoint
            // addresses; whichever finishes the last plane runs the step tail)
            const bool both = c->tma.ngroups > 0 && c->ndirty > 0;
            cudaStream_t ls = both ? c->side : c->stream;
            if (both) {
                CK(cudaEventRecord(c->fj[0], c->stream));
                CK(cudaStreamWaitEvent(c->side, c->fj[0], 0));
            }
            if (c->tma.ngroups > 0) {
                const bool alt = odd && c->odd_split;
                const TmaArgs &t = alt ? c->odd_tma : c->tma;
                const int grid = alt ? c->odd_grid : c->tma_grid, threads = alt ? c->odd_threads : c->tma_threads;
                const size_t smem = alt ? c->odd_smem : c->tma_smem;
                if (c->deck.precision == 64)
                    launch_tma_f64(p, t, grid, threads, smem, odd, c->walls_textured, c->stream);
                else
                    launch_tma_lp(c->deck.precision, p, t, grid, threads, smem, odd, c->walls_textured, c->stream);
            }
            if (c->ndirty > 0) {
                const int blocks = c->ndirty * (int)(c->grid.x * c->grid.y);
                if (c->deck.precision == 64) launch_links_f64(c->d_llaunch, 1, blocks, odd, ls);
                else launch_links_lp(c->deck.precision, c->d_llaunch, 1, blocks, odd, ls);
            }
            if (both) {
                CK(cudaEventRecord(c->fj[1], c->side));
                CK(cudaStreamWaitEvent(c->stream, c->fj[1], 0));
            }
        } else if (c->deck.precision == 64) {
            launch_step_f64(p, c->grid, c->block, odd, c->textured, c->stream);
        } else {
            launch_step_lp(c->deck.precision, p, c->grid, c->block, odd, c->textured, c->stream);
        }
        CK(cudaGetLastError());
        if (timed) CK(cudaEventRecord(c->tev[2 * s + 1], c->stream));
        c->odd ^= 1;
        c->done++;
    }
    if (timed) {
        CK(cudaEventSynchronize(c->tev[2 * n - 1]));
        for (long s = 0; s < n; ++s) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, c->tev[2 * s], c->tev[2 * s + 1]));
            *(((first_parity + s) & 1) ? ms_odd : ms_even) += ms;
        }
    }
    return DNSLBM_OK;
}

static int check_status(dnslbm_ctx *c)
{
    long long st[2];
    CK(cudaMemcpyAsync(st, c->status, sizeof st, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (st[1]) {
        c->have_state = 0;  // blocks that gave up left their rows unstepped
        return fail(c, DNSLBM_ERR_TIMEOUT, "a bounded wait for a bulk copy ran out; state invalid, reload it");
    }
    if (st[0]) return fail(c, DNSLBM_ERR_NAN, "NaN wall shear stress at step %lld", st[0] - 1);
    return DNSLBM_OK;
}

extern "C" int dnslbm_step(dnslbm_ctx *c, long nsteps)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (nsteps < 0) return fail(c, DNSLBM_ERR_ARG, "negative step count");
    if (c->slab) return fail(c, DNSLBM_ERR_STATE, "a slab context steps with dnslbm_slab_step and dnslbm_slab_tail");
    if (!c->have_state) return fail(c, DNSLBM_ERR_STATE, "no state: call dnslbm_init_rest or dnslbm_load_state");
    CK(cudaSetDevice(c->deck.device));
    int rc = launch_steps(c, nsteps, false, nullptr, nullptr);
    if (rc) return rc;
    return check_status(c);
}

extern "C" int dnslbm_step_timed(dnslbm_ctx *c, long nsteps, double *ms_total, double *ms_even, double *ms_odd)
{
    if (!c || !ms_total || (!ms_even) != (!ms_odd)) return fail(c, DNSLBM_ERR_ARG, "null argument");
    if (c->slab) return fail(c, DNSLBM_ERR_STATE, "a slab context steps with dnslbm_slab_step and dnslbm_slab_tail");
    if (!c->have_state) return fail(c, DNSLBM_ERR_STATE, "no state");
    CK(cudaSetDevice(c->deck.device));
    const bool per_launch = ms_even != nullptr;  // an event pair around every launch
    if (per_launch) *ms_even = *ms_odd = 0.0;
    if (nsteps <= 0) return fail(c, DNSLBM_ERR_ARG, "timed run needs at least one step");
    CK(cudaEventRecord(c->ev[0], c->stream));
    int rc = launch_steps(c, nsteps, per_launch, ms_even, ms_odd);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev[1], c->stream));
    CK(cudaEventSynchronize(c->ev[1]));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    *ms_total = ms;
    return check_status(c);
}

// ---------------------------------------------------------------- slabs
// A channel split into wall-normal slabs over several GPUs: the step kernel
// of each slab leaves its plane sums; the caller gathers every slab's sums
// in plane order and hands them to dnslbm_slab_tail, which runs the step
// tail of the whole channel on each slab.  Around an odd step the caller
// exchanges the ghost planes (dnslbm_slab_halo).
static_assert(DNSLBM_SUM_N == NP, "the slab sums are the plane sums of the step kernels");

extern "C" int dnslbm_slab_step(dnslbm_ctx *c)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (!c->slab) return fail(c, DNSLBM_ERR_STATE, "not a slab context (dnslbm_create_slab)");
    if (!c->have_state) return fail(c, DNSLBM_ERR_STATE, "no state: call dnslbm_init_rest or dnslbm_load_state");
    if (c->tail_owed >= 0)
        return fail(c, DNSLBM_ERR_STATE, "the tail of the last %s is owed first (dnslbm_slab_tail)",
                    c->tail_owed ? "load" : "step");
    CK(cudaSetDevice(c->deck.device));
    int rc = launch_steps(c, 1, false, nullptr, nullptr);
    if (rc) return rc;
    c->tail_owed = 0;
    return DNSLBM_OK;
}

extern "C" int dnslbm_slab_sums(dnslbm_ctx *c, double **sums)
{
    if (!c || !sums) return fail(c, DNSLBM_ERR_ARG, "null argument");
    if (!c->slab) return fail(c, DNSLBM_ERR_STATE, "not a slab context (dnslbm_create_slab)");
    *sums = c->plane_sums;
    return DNSLBM_OK;
}

extern "C" int dnslbm_slab_tail(dnslbm_ctx *c, const double *sums_all)
{
    if (!c || !sums_all) return fail(c, DNSLBM_ERR_ARG, "null argument");
    if (!c->slab) return fail(c, DNSLBM_ERR_STATE, "not a slab context (dnslbm_create_slab)");
    if (c->tail_owed < 0) return fail(c, DNSLBM_ERR_STATE, "no step or load of this slab awaits its tail");
    CK(cudaSetDevice(c->deck.device));
    StepArgs a = step_args(c);
    a.nz = c->nz_all;
    a.plane_sums = const_cast<double *>(sums_all);
    a.shift = c->shift_all;
    launch_slab_tail(a, c->tail_owed, c->shift, c->z0, c->nz, c->stream);
    CK(cudaGetLastError());
    c->tail_owed = -1;
    return DNSLBM_OK;
}

extern "C" int dnslbm_slab_status(dnslbm_ctx *c)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    CK(cudaSetDevice(c->deck.device));
    return check_status(c);
}

extern "C" int dnslbm_slab_halo(dnslbm_ctx *c, int side, void **ghost, void **edge, size_t *bytes)
{
    if (!c || !ghost || !edge || !bytes) return fail(c, DNSLBM_ERR_ARG, "null argument");
    if (!c->slab) return fail(c, DNSLBM_ERR_STATE, "not a slab context (dnslbm_create_slab)");
    if (side != 0 && side != 1) return fail(c, DNSLBM_ERR_ARG, "side %d is neither 0 (lower) nor 1 (upper)", side);
    if (side == 0 ? c->wall_lo : c->wall_hi)
        return fail(c, DNSLBM_ERR_ARG, "the %s face of this slab is a wall", side ? "upper" : "lower");
    // directions leaving through the lower face (e_z = -1) and the upper one
    static const int down[5] = {6, 12, 13, 16, 17}, up[5] = {5, 11, 14, 15, 18};
    const StepArgs p = step_args(c);
    const ptrdiff_t plane = (ptrdiff_t)c->ny * c->pitch;
    for (int i = 0; i < 5; ++i) {
        const int gs = side == 0 ? down[i] : up[i], es = side == 0 ? up[i] : down[i];
        ghost[i] = (char *)p.pop[gs] + (side == 0 ? -plane : (ptrdiff_t)c->nz * plane) * (ptrdiff_t)c->esize;
        edge[i] = (char *)p.pop[es] + (side == 0 ? 0 : (ptrdiff_t)(c->nz - 1) * plane) * (ptrdiff_t)c->esize;
    }
    *bytes = (size_t)plane * c->esize;
    return DNSLBM_OK;
}

extern "C" void *dnslbm_stream(const dnslbm_ctx *c) { return c ? (void *)c->stream : nullptr; }

extern "C" int dnslbm_set_wait_limit(dnslbm_ctx *c, double ms)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (!(ms > 0.0 && ms <= 600000.0)) return fail(c, DNSLBM_ERR_ARG, "wait limit %g ms outside (0, 600000]", ms);
    c->wait_ns = (unsigned long long)(ms * 1e6);
    return DNSLBM_OK;
}

extern "C" int dnslbm_test_withhold_load(dnslbm_ctx *c)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (!c->use_tma || c->tma.ngroups <= 0)
        return fail(c, DNSLBM_ERR_STATE, "the context steps with a kernel that has no bounded waits");
    c->withhold = 1;
    return DNSLBM_OK;
}

extern "C" long dnslbm_steps_done(const dnslbm_ctx *c) { return c ? (long)c->done : -1; }

extern "C" int dnslbm_logs(dnslbm_ctx *c, long first, long count, double *out)
{
    if (!c || (!out && count > 0)) return fail(c, DNSLBM_ERR_ARG, "null argument");
    const long cap = c->deck.log_capacity;
    if (first < 0 || count < 0 || first + count > c->done || first < c->done - cap)
        return fail(c, DNSLBM_ERR_ARG, "log range [%ld,%ld) not held (done %lld, capacity %ld)", first, first + count,
                    c->done, cap);
    CK(cudaSetDevice(c->deck.device));
    long s = first;
    while (s < first + count) {
        const long slot = s % cap;
        const long n = std::min(first + count - s, cap - slot);
        CK(cudaMemcpyAsync(out + (s - first) * 9, c->logs + slot * 9, (size_t)n * 9 * sizeof(double),
                           cudaMemcpyDeviceToHost, c->stream));
        s += n;
    }
    CK(cudaStreamSynchronize(c->stream));
    return DNSLBM_OK;
}

extern "C" int dnslbm_get_force(dnslbm_ctx *c, double *force)
{
    if (!c || !force) return fail(c, DNSLBM_ERR_ARG, "null argument");
    if (!c->have_state) return fail(c, DNSLBM_ERR_STATE, "no state");
    CK(cudaSetDevice(c->deck.device));
    CK(cudaMemcpyAsync(force, c->force + (c->done & 1), sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DNSLBM_OK;
}

extern "C" int dnslbm_moments(dnslbm_ctx *c, double *vel, double *den)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (int rc_ = readable(c)) return rc_;
    if (!vel && !den) return DNSLBM_OK;
    CK(cudaSetDevice(c->deck.device));
    IoArgs p = io_args(c);
    const size_t per_x = (size_t)c->ny * (c->nz + 2) * 4;  // 3 vel + 1 den doubles
    const int xchunk = (int)std::max<size_t>(1, c->staging_bytes / (per_x * sizeof(double)));
    for (int x0 = 0; x0 < c->nx; x0 += xchunk) {
        const int n = std::min(xchunk, c->nx - x0);
        double *dv = c->staging, *dd = c->staging + (size_t)n * c->ny * (c->nz + 2) * 3;
        launch_io(c->deck.precision, 3, p, x0, n, dv, dd, c->stream);
        CK(cudaGetLastError());
        const size_t cells = (size_t)n * c->ny * (c->nz + 2);
        const size_t off = (size_t)x0 * c->ny * (c->nz + 2);
        if (vel)
            CK(cudaMemcpyAsync(vel + off * 3, dv, cells * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (den) CK(cudaMemcpyAsync(den + off, dd, cells * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return DNSLBM_OK;
}

extern "C" int dnslbm_stats_accumulate(dnslbm_ctx *c)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (int rc_ = readable(c)) return rc_;
    CK(cudaSetDevice(c->deck.device));
    const double np = (double)c->nx * c->ny;
    IoArgs p = io_args(c);
    launch_stats(c->deck.precision, p, c->grid, c->block, c->rows, 0, nullptr, c->stat_partials, c->stat_planes,
                 c->stream);
    launch_stats_sample(c->nz, np, c->stat_planes, c->stat_mean, nullptr, false, c->stream);
    launch_stats(c->deck.precision, p, c->grid, c->block, c->rows, 1, c->stat_mean, c->stat_partials, c->stat_planes,
                 c->stream);
    launch_stats_sample(c->nz, np, c->stat_planes, c->stat_mean, c->stat_acc, true, c->stream);
    CK(cudaGetLastError());
    ++c->stat_samples;
    return DNSLBM_OK;
}

extern "C" int dnslbm_stats_average(dnslbm_ctx *c, double *out, long *nsamples)
{
    if (!c || !out) return fail(c, DNSLBM_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->deck.device));
    const int nz = c->nz, zd = nz + 2;
    std::vector<double> acc((size_t)9 * nz);
    CK(cudaMemcpyAsync(acc.data(), c->stat_acc, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memset(out, 0, sizeof(double) * 9 * zd);
    if (nsamples) *nsamples = c->stat_samples;
    if (c->stat_samples == 0) return DNSLBM_OK;
    const double n = (double)c->stat_samples;
    for (int r = 0; r < 9; ++r) {
        const bool rms = r == 3 || r == 4 || r == 5 || r == 8;
        for (int z = 0; z < nz; ++z) {
            const double v = acc[(size_t)r * nz + z] / n;
            out[(size_t)r * zd + z + 1] = rms ? std::sqrt(v) : v;
        }
    }
    return DNSLBM_OK;
}

extern "C" int dnslbm_stats_reset(dnslbm_ctx *c)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    CK(cudaSetDevice(c->deck.device));
    CK(cudaMemsetAsync(c->stat_acc, 0, (size_t)9 * c->nz * sizeof(double), c->stream));
    c->stat_samples = 0;
    return DNSLBM_OK;
}

extern "C" int dnslbm_statistics(dnslbm_ctx *c, double *out)
{
    if (!c || !out) return fail(c, DNSLBM_ERR_ARG, "null argument");
    if (int rc_ = readable(c)) return rc_;
    CK(cudaSetDevice(c->deck.device));
    const int nz = c->nz, zd = nz + 2;
    const double np = (double)c->nx * c->ny;
    IoArgs p = io_args(c);
    std::vector<double> pl((size_t)nz * 5), mean((size_t)nz * 4);
    // pass 1: plane means of u, v, w, rho (statistics.c:31-60)
    launch_stats(c->deck.precision, p, c->grid, c->block, c->rows, 0, nullptr, c->stat_partials, c->stat_planes,
                 c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(pl.data(), c->stat_planes, pl.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memset(out, 0, sizeof(double) * 9 * zd);
    double *UAVG = out, *VAVG = out + zd, *WAVG = out + 2 * zd, *UTIN = out + 3 * zd, *VTIN = out + 4 * zd;
    double *WTIN = out + 5 * zd, *REYS = out + 6 * zd, *DAVG = out + 7 * zd, *DTIN = out + 8 * zd;
    for (int z = 0; z < nz; ++z) {
        UAVG[z + 1] = pl[z * 5 + 0] / np;
        VAVG[z + 1] = pl[z * 5 + 1] / np;
        WAVG[z + 1] = pl[z * 5 + 2] / np;
        DAVG[z + 1] = pl[z * 5 + 3] / np;
        mean[z * 4 + 0] = UAVG[z + 1];
        mean[z * 4 + 1] = VAVG[z + 1];
        mean[z * 4 + 2] = WAVG[z + 1];
        mean[z * 4 + 3] = DAVG[z + 1];
    }
    // pass 2: second moments about the plane means (statistics.c:74-132)
    CK(cudaMemcpyAsync(c->stat_mean, mean.data(), mean.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    launch_stats(c->deck.precision, p, c->grid, c->block, c->rows, 1, c->stat_mean, c->stat_partials, c->stat_planes,
                 c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(pl.data(), c->stat_planes, pl.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int z = 0; z < nz; ++z) {
        UTIN[z + 1] = std::sqrt(pl[z * 5 + 0] / np);
        VTIN[z + 1] = std::sqrt(pl[z * 5 + 1] / np);
        WTIN[z + 1] = std::sqrt(pl[z * 5 + 2] / np);
        REYS[z + 1] = pl[z * 5 + 3] / np;
        DTIN[z + 1] = std::sqrt(pl[z * 5 + 4] / np);
    }
    return DNSLBM_OK;
}

// ---------------------------------------------------------------- output
// dnslbm_output_begin: the outputs of the current state are computed on the
// context's stream (so later steps see the state only after the kernels
// that read it) into device buffers, and copied to the caller's host
// buffers on out_stream while the steps that follow run.
static int out_alloc(dnslbm_ctx *c, double **p, size_t n)
{
    if (*p) return DNSLBM_OK;
    cudaError_t e = cudaMalloc(p, n * sizeof(double));
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(c, DNSLBM_ERR_NOMEM, "cudaMalloc of %zu bytes for an output snapshot failed: %s",
                    n * sizeof(double), cudaGetErrorString(e));
    }
    CK(cudaMemset(*p, 0, n * sizeof(double)));  // wall-plane entries stay zero
    return DNSLBM_OK;
}

extern "C" int dnslbm_output_begin(dnslbm_ctx *c, double *state, double *vel, double *den, double *stats)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (int rc_ = readable(c)) return rc_;
    CK(cudaSetDevice(c->deck.device));
    const size_t cells = (size_t)c->nx * c->ny * (c->nz + 2);
    const int zd = c->nz + 2;
    int rc;
    if (state && (rc = out_alloc(c, &c->out_lbf, cells * Q))) return rc;
    if ((vel || den) && ((rc = out_alloc(c, &c->out_vel, cells * 3)) || (rc = out_alloc(c, &c->out_den, cells))))
        return rc;
    if (stats && (rc = out_alloc(c, &c->out_stats, (size_t)9 * zd))) return rc;
    CK(cudaDeviceSynchronize());  // the allocations' zero fill
    // the previous snapshot's copies read these buffers: wait on the device
    if (c->out_pending) CK(cudaStreamWaitEvent(c->stream, c->out_ev[1], 0));
    IoArgs p = io_args(c);
    if (state) launch_io(c->deck.precision, 0, p, 0, c->nx, c->out_lbf, nullptr, c->stream);
    if (vel || den) launch_io(c->deck.precision, 3, p, 0, c->nx, c->out_vel, c->out_den, c->stream);
    if (stats) {
        const double np = (double)c->nx * c->ny;
        launch_stats(c->deck.precision, p, c->grid, c->block, c->rows, 0, nullptr, c->stat_partials, c->stat_planes,
                     c->stream);
        launch_stats_sample(c->nz, np, c->stat_planes, c->stat_mean, nullptr, false, c->stream);
        launch_stats(c->deck.precision, p, c->grid, c->block, c->rows, 1, c->stat_mean, c->stat_partials,
                     c->stat_planes, c->stream);
        launch_stats_rows(c->nz, np, c->stat_mean, c->stat_planes, c->out_stats, c->stream);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->out_ev[0], c->stream));
    CK(cudaStreamWaitEvent(c->out_stream, c->out_ev[0], 0));
    if (state)
        CK(cudaMemcpyAsync(state, c->out_lbf, cells * Q * sizeof(double), cudaMemcpyDeviceToHost, c->out_stream));
    if (vel) CK(cudaMemcpyAsync(vel, c->out_vel, cells * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->out_stream));
    if (den) CK(cudaMemcpyAsync(den, c->out_den, cells * sizeof(double), cudaMemcpyDeviceToHost, c->out_stream));
    if (stats)
        CK(cudaMemcpyAsync(stats, c->out_stats, (size_t)9 * zd * sizeof(double), cudaMemcpyDeviceToHost,
                           c->out_stream));
    CK(cudaEventRecord(c->out_ev[1], c->out_stream));
    c->out_pending = 1;
    return DNSLBM_OK;
}

// ---------------------------------------------------------------- post-processing
// Quadrant analysis (quadrant-analysis/src/qUADrantA.c:140-170): from the
// per-plane sums of quadrant_kernel to the reference's output arrays.
static void quadrant_finish(int zd, double n, const double *sums, double *quadrant, double *dquadrant, double *uw)
{
    for (int i = 0; i < 4 * zd; ++i) {
        if (quadrant) quadrant[i] = 0.0;
        if (dquadrant) dquadrant[i] = 0.0;
    }
    for (int k = 0; k < zd; ++k)
        if (uw) uw[k] = 0.0;
    for (int k = 1; k < zd - 1; ++k) {
        const double *p = sums + (size_t)k * 9;
        for (int a = 0; a < 4; ++a) {
            if (quadrant) quadrant[a * zd + k] = p[a] / p[4 + a];  // an empty quadrant gives 0/0, as the reference
            if (dquadrant) dquadrant[a * zd + k] = p[a] / n;
        }
        if (uw) uw[k] = p[8] / n;
    }
}

extern "C" int dnslbm_quadrant(dnslbm_ctx *c, double *quadrant, double *dquadrant, double *uw)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (int rc_ = readable(c)) return rc_;
    CK(cudaSetDevice(c->deck.device));
    const int zd = c->nz + 2;
    const size_t cells = (size_t)c->nx * c->ny * zd;
    int rc;
    if ((rc = out_alloc(c, &c->out_vel, cells * 3)) || (rc = out_alloc(c, &c->out_den, cells)) ||
        (rc = out_alloc(c, &c->quad_buf, (size_t)zd * 12)))
        return rc;
    CK(cudaDeviceSynchronize());
    // the velocity field in the vel layout, then the two plane passes
    if (c->out_pending) CK(cudaStreamWaitEvent(c->stream, c->out_ev[1], 0));
    launch_io(c->deck.precision, 3, io_args(c), 0, c->nx, c->out_vel, c->out_den, c->stream);
    launch_quadrant(c->out_vel, c->nx, c->ny, zd, c->quad_buf, c->quad_buf + (size_t)zd * 3, c->stream);
    CK(cudaGetLastError());
    std::vector<double> sums((size_t)zd * 9);
    CK(cudaMemcpyAsync(sums.data(), c->quad_buf + (size_t)zd * 3, sums.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    quadrant_finish(zd, (double)c->nx * c->ny, sums.data(), quadrant, dquadrant, uw);
    return DNSLBM_OK;
}

extern "C" int dnslbm_quadrant_vel(const double *vel, int xdv, int ydv, int zdv, int device, double *quadrant,
                                   double *dquadrant, double *uw)
{
    dnslbm_ctx *c = nullptr;  // errors go to dnslbm_last_error(NULL)
    if (!vel) return fail(c, DNSLBM_ERR_ARG, "null velocity field");
    if (xdv < 1 || ydv < 1 || zdv < 1) return fail(c, DNSLBM_ERR_ARG, "grid %dx%dx%d too small", xdv, ydv, zdv);
    const int zd = zdv + 2;
    const size_t n = (size_t)xdv * ydv * zd * 3;
    CK(cudaSetDevice(device));
    double *dv = nullptr, *buf = nullptr;
    cudaError_t e = cudaMalloc(&dv, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&buf, (size_t)zd * 12 * sizeof(double));
    std::vector<double> sums((size_t)zd * 9);
    if (e == cudaSuccess) e = cudaMemcpy(dv, vel, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        launch_quadrant(dv, xdv, ydv, zd, buf, buf + (size_t)zd * 3, 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(sums.data(), buf + (size_t)zd * 3, sums.size() * sizeof(double), cudaMemcpyDeviceToHost);
    if (dv) cudaFree(dv);
    if (buf) cudaFree(buf);
    if (e != cudaSuccess) return fail(c, DNSLBM_ERR_CUDA, "quadrant analysis of a velocity field: %s", cudaGetErrorString(e));
    quadrant_finish(zd, (double)xdv * ydv, sums.data(), quadrant, dquadrant, uw);
    return DNSLBM_OK;
}

// Two-point correlations (2pt-correlations/src: mean_subtract.c, xcorrel.c,
// ycorrel.c) of a velocity field already in device memory: temporary device
// memory for the fluctuations and the partial sums, results copied to the
// caller's host arrays (any may be NULL).
constexpr int kCorrLinesPerChunk = 8;

static cudaError_t correlations_of(const double *dvel, int nx, int ny, int zd, cudaStream_t s, double *xcorl,
                                   double *ycorl, double *uavg)
{
    double *scratch = nullptr, *res = nullptr;
    const size_t nres = (size_t)zd * 3 * (nx + ny + 1);
    cudaError_t e = cudaMalloc(&scratch, correlation_scratch(nx, ny, zd, kCorrLinesPerChunk) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&res, nres * sizeof(double));
    double *dx = res, *dy = res + (size_t)zd * 3 * nx, *du = dy + (size_t)zd * 3 * ny;
    if (e == cudaSuccess) e = launch_correlations(dvel, nx, ny, zd, kCorrLinesPerChunk, scratch, dx, dy, du, s);
    std::vector<double> h(nres);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), res, nres * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (scratch) cudaFree(scratch);
    if (res) cudaFree(res);
    if (e != cudaSuccess) return e;
    if (xcorl) memcpy(xcorl, h.data(), sizeof(double) * zd * 3 * nx);
    if (ycorl) memcpy(ycorl, h.data() + (size_t)zd * 3 * nx, sizeof(double) * zd * 3 * ny);
    if (uavg)
        for (int k = 0; k < zd; ++k) uavg[k] = h[(size_t)zd * 3 * (nx + ny) + (size_t)k * 3];
    return cudaSuccess;
}

extern "C" int dnslbm_correlations(dnslbm_ctx *c, double *xcorl, double *ycorl, double *uavg)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (int rc_ = readable(c)) return rc_;
    if (c->nx > correlation_max_line() || c->ny > correlation_max_line())
        return fail(c, DNSLBM_ERR_ARG, "correlation lines longer than %d cells", correlation_max_line());
    CK(cudaSetDevice(c->deck.device));
    const int zd = c->nz + 2;
    const size_t cells = (size_t)c->nx * c->ny * zd;
    int rc;
    if ((rc = out_alloc(c, &c->out_vel, cells * 3)) || (rc = out_alloc(c, &c->out_den, cells))) return rc;
    CK(cudaDeviceSynchronize());
    if (c->out_pending) CK(cudaStreamWaitEvent(c->stream, c->out_ev[1], 0));
    launch_io(c->deck.precision, 3, io_args(c), 0, c->nx, c->out_vel, c->out_den, c->stream);
    CK(cudaGetLastError());
    const cudaError_t e = correlations_of(c->out_vel, c->nx, c->ny, zd, c->stream, xcorl, ycorl, uavg);
    if (e != cudaSuccess) return fail(c, DNSLBM_ERR_CUDA, "correlations: %s", cudaGetErrorString(e));
    return DNSLBM_OK;
}

extern "C" int dnslbm_correlations_vel(const double *vel, int xdv, int ydv, int zdv, int device, double *xcorl,
                                       double *ycorl, double *uavg)
{
    dnslbm_ctx *c = nullptr;  // errors go to dnslbm_last_error(NULL)
    if (!vel) return fail(c, DNSLBM_ERR_ARG, "null velocity field");
    if (xdv < 1 || ydv < 1 || zdv < 1) return fail(c, DNSLBM_ERR_ARG, "grid %dx%dx%d too small", xdv, ydv, zdv);
    if (xdv > correlation_max_line() || ydv > correlation_max_line())
        return fail(c, DNSLBM_ERR_ARG, "correlation lines longer than %d cells", correlation_max_line());
    const int zd = zdv + 2;
    const size_t n = (size_t)xdv * ydv * zd * 3;
    CK(cudaSetDevice(device));
    double *dv = nullptr;
    cudaError_t e = cudaMalloc(&dv, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(dv, vel, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = correlations_of(dv, xdv, ydv, zd, 0, xcorl, ycorl, uavg);
    if (dv) cudaFree(dv);
    if (e != cudaSuccess) return fail(c, DNSLBM_ERR_CUDA, "correlations of a velocity field: %s", cudaGetErrorString(e));
    return DNSLBM_OK;
}

// One-dimensional energy spectra (e-spectra/src/1d-spectra.c) of a velocity
// field in device memory; results in the program's file layouts: ex
// [3][nx][zd] (Euux, Evvx, Ewwx), ey [3][ny/2+1][zd] (Euuy, Evvy, Ewwy).
static cudaError_t spectra_of(const double *dvel, int nx, int ny, int zd, cudaStream_t s, double *ex, double *ey)
{
    const int nj = ny / 2 + 1, nzf = zd - 2;
    const int jb = std::max(1, std::min(8, (int)((180 * 1024) / (16 * (size_t)nx)) - 1));
    double *scratch = nullptr, *res = nullptr;
    const size_t nres = (size_t)nzf * 3 * (nx + nj);
    cudaError_t e = cudaMalloc(&scratch, spectra_scratch(nx, ny, zd, jb) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&res, nres * sizeof(double));
    if (e == cudaSuccess) e = launch_spectra(dvel, nx, ny, zd, jb, scratch, res, res + (size_t)nzf * 3 * nx, s);
    std::vector<double> h(nres);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), res, nres * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (scratch) cudaFree(scratch);
    if (res) cudaFree(res);
    if (e != cudaSuccess) return e;
    const double *hx = h.data(), *hy = h.data() + (size_t)nzf * 3 * nx;
    for (int c = 0; c < 3; ++c) {
        if (ex)
            for (int i = 0; i < nx; ++i)
                for (int k = 0; k < zd; ++k)
                    ex[((size_t)c * nx + i) * zd + k] =
                        (k == 0 || k == zd - 1) ? 0.0 : hx[((size_t)(k - 1) * 3 + c) * nx + i];
        if (ey)
            for (int j = 0; j < nj; ++j)
                for (int k = 0; k < zd; ++k)
                    ey[((size_t)c * nj + j) * zd + k] =
                        (k == 0 || k == zd - 1) ? 0.0 : hy[((size_t)(k - 1) * 3 + c) * nj + j];
    }
    return cudaSuccess;
}

extern "C" int dnslbm_spectra(dnslbm_ctx *c, double *ex, double *ey)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (int rc_ = readable(c)) return rc_;
    CK(cudaSetDevice(c->deck.device));
    const int zd = c->nz + 2;
    const size_t cells = (size_t)c->nx * c->ny * zd;
    int rc;
    if ((rc = out_alloc(c, &c->out_vel, cells * 3)) || (rc = out_alloc(c, &c->out_den, cells))) return rc;
    CK(cudaDeviceSynchronize());
    if (c->out_pending) CK(cudaStreamWaitEvent(c->stream, c->out_ev[1], 0));
    launch_io(c->deck.precision, 3, io_args(c), 0, c->nx, c->out_vel, c->out_den, c->stream);
    CK(cudaGetLastError());
    const cudaError_t e = spectra_of(c->out_vel, c->nx, c->ny, zd, c->stream, ex, ey);
    if (e != cudaSuccess) return fail(c, DNSLBM_ERR_CUDA, "spectra: %s", cudaGetErrorString(e));
    return DNSLBM_OK;
}

extern "C" int dnslbm_spectra_vel(const double *vel, int xdv, int ydv, int zdv, int device, double *ex, double *ey)
{
    dnslbm_ctx *c = nullptr;  // errors go to dnslbm_last_error(NULL)
    if (!vel) return fail(c, DNSLBM_ERR_ARG, "null velocity field");
    if (xdv < 1 || ydv < 1 || zdv < 1) return fail(c, DNSLBM_ERR_ARG, "grid %dx%dx%d too small", xdv, ydv, zdv);
    const int zd = zdv + 2;
    const size_t n = (size_t)xdv * ydv * zd * 3;
    CK(cudaSetDevice(device));
    double *dv = nullptr;
    cudaError_t e = cudaMalloc(&dv, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(dv, vel, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = spectra_of(dv, xdv, ydv, zd, 0, ex, ey);
    if (dv) cudaFree(dv);
    if (e != cudaSuccess) return fail(c, DNSLBM_ERR_CUDA, "spectra of a velocity field: %s", cudaGetErrorString(e));
    return DNSLBM_OK;
}

extern "C" int dnslbm_output_wait(dnslbm_ctx *c)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (!c->out_pending) return DNSLBM_OK;
    CK(cudaSetDevice(c->deck.device));
    CK(cudaEventSynchronize(c->out_ev[1]));
    c->out_pending = 0;
    return DNSLBM_OK;
}

extern "C" const char *dnslbm_step_kernel(const dnslbm_ctx *c) { return c ? c->kernel_desc : ""; }

extern "C" double dnslbm_bytes_per_cell(const dnslbm_ctx *c) { return c ? 2.0 * Q * (double)c->esize : 0.0; }

extern "C" int dnslbm_sync(dnslbm_ctx *c)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    CK(cudaSetDevice(c->deck.device));
    CK(cudaStreamSynchronize(c->stream));
    return DNSLBM_OK;
}

extern "C" void *dnslbm_host_alloc(size_t bytes)
{
    void *p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
    return p;
}

extern "C" void dnslbm_host_free(void *p)
{
    if (p) cudaFreeHost(p);
}

// ---------------------------------------------------------------- autotuner
struct TmaChoice {
    int use_tma, threads, grid, target;
    size_t smem;
    TmaArgs t;
    int odd_split, odd_threads, odd_grid, odd_target;
    size_t odd_smem;
    TmaArgs odd_t;
};

static TmaChoice save_choice(const dnslbm_ctx *c)
{
    return {c->use_tma,   c->tma_threads, c->tma_grid,   c->tma_target, c->tma_smem, c->tma,
            c->odd_split, c->odd_threads, c->odd_grid,   c->odd_target, c->odd_smem, c->odd_tma};
}
static void load_choice(dnslbm_ctx *c, const TmaChoice &k)
{
    c->use_tma = k.use_tma;
    c->tma_threads = k.threads;
    c->tma_grid = k.grid;
    c->tma_target = k.target;
    c->tma_smem = k.smem;
    c->tma = k.t;
    c->odd_split = k.odd_split;
    c->odd_threads = k.odd_threads;
    c->odd_grid = k.odd_grid;
    c->odd_target = k.odd_target;
    c->odd_smem = k.odd_smem;
    c->odd_tma = k.odd_t;
}

// A choice whose even steps use shape e and odd steps shape o (both whole
// row-pipelined shapes).
static TmaChoice split_choice(const TmaChoice &e, const TmaChoice &o)
{
    TmaChoice k = e;
    k.odd_split = 1;
    k.odd_threads = o.threads;
    k.odd_grid = o.grid;
    k.odd_target = o.target;
    k.odd_smem = o.smem;
    k.odd_t = o.t;
    return k;
}

// device time per even and per odd step of the current launch shape, on a
// rest state
static int time_choice(dnslbm_ctx *c, int steps, double *ms, double *ms_even = nullptr, double *ms_odd = nullptr)
{
    int rc = reset_counters(c);
    if (rc) return rc;
    launch_io(c->deck.precision, 2, io_args(c), 0, 0, nullptr, nullptr, c->stream);
    CK(cudaGetLastError());
    if ((rc = initial_reduce(c))) return rc;
    double e = 0, o = 0;
    if ((rc = launch_steps(c, 2, true, &e, &o))) return rc;
    e = o = 0;
    if ((rc = launch_steps(c, steps, true, &e, &o))) return rc;
    if ((rc = check_status(c))) return rc;
    *ms = (e + o) / steps;
    const int ne = (steps + 1) / 2, no = steps / 2;  // the timed run starts on an even step
    if (ms_even) *ms_even = ne ? e / ne : 0.0;
    if (ms_odd) *ms_odd = no ? o / no : 0.0;
    return DNSLBM_OK;
}

extern "C" int dnslbm_autotune(dnslbm_ctx *c, int steps, char *report, size_t report_len)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (c->have_state) return fail(c, DNSLBM_ERR_STATE, "autotune runs before a state is loaded (it steps a rest state)");
    if (steps < 2) steps = 2;
    CK(cudaSetDevice(c->deck.device));
    int ncand = 0;
    double best_ms = 1e30;
    TmaChoice best = save_choice(c);
    int rc;
    // the per-thread kernel
    {
        c->use_tma = 0;
        double ms;
        if ((rc = time_choice(c, steps, &ms))) return rc;
        ++ncand;
        if (ms < best_ms) best_ms = ms, best = save_choice(c);
    }
    // row-pipelined: group rows x stages at the default consumer count, then
    // the consumer count and the blocks per SM for the best pair; the even
    // and the odd steps are timed apart and may end with different shapes
    // (their address sets differ: one row position, or three planes x three
    // rows)
    const int cap = c->deck.precision == 64 ? 320 : (c->deck.precision == 32 ? 192 : 128);
    const int cons0 = std::min(cap, (c->nx + 31) / 32 * 32);
    struct Best {
        double ms = 1e30;
        TmaChoice ch{};
        int k = -1, st = -1, seg = 0, cons = 0;
    } be, bo, bt;  // best even / odd step shape, best shape for both
    auto timed = [&](int k, int st, int seg, int cons) -> int {
        double ms, e, o;
        int r = time_choice(c, steps, &ms, &e, &o);
        if (r) return r;
        ++ncand;
        if (e < be.ms) be.ms = e, be.ch = save_choice(c), be.k = k, be.st = st, be.seg = seg, be.cons = cons;
        if (o < bo.ms) bo.ms = o, bo.ch = save_choice(c), bo.k = k, bo.st = st, bo.seg = seg, bo.cons = cons;
        if (ms < bt.ms) bt.ms = ms, bt.ch = save_choice(c), bt.k = k, bt.st = st, bt.seg = seg, bt.cons = cons;
        return DNSLBM_OK;
    };
    // the default consumer count and the widest consumer sets (a block with
    // large stages is alone on its SM and needs more warps)
    const int widest = std::min(352, (c->nx + 31) / 32 * 32 + 32);
    for (int k : {1, 2, 4, 8})
        for (int st : {2, 3, 4})
            for (int cons : {cons0, 224, widest}) {
                if ((cons != cons0 && (cons <= cons0 || (cons == 224 && widest <= 224))) || k > c->ny ||
                    tma_configure(c, k, st, cons, 0))
                    continue;
                if ((rc = timed(k, st, 0, cons))) return rc;
            }
    // FP64 rows as x-segments (the only bulk-copy form for rows too long for
    // two whole-row stages)
    if (c->deck.precision == 64 && c->nx >= 256)
        for (int nseg : {2, 3, 4})
            for (int st : {2, 3, 4}) {
                const int seg = segment_for(c->nx, nseg);
                if (tma_configure(c, 1, st, cons0, 0, seg)) continue;
                if ((rc = timed(1, st, seg, cons0))) return rc;
            }
    // consumer counts, then a cap on the blocks per SM, for each parity's best
    const Best leaders[3] = {be, bo, bt};
    for (int pass = 0; pass < 3; ++pass) {
        const Best b0 = leaders[pass];
        bool seen = false;
        for (int q = 0; q < pass; ++q)
            seen |= leaders[q].k == b0.k && leaders[q].st == b0.st && leaders[q].seg == b0.seg;
        if (b0.k < 0 || seen) continue;
        for (int cons = 64; cons <= widest; cons += 32) {
            if (cons == cons0 || cons == 224 || cons == widest || tma_configure(c, b0.k, b0.st, cons, 0, b0.seg)) continue;
            if ((rc = timed(b0.k, b0.st, b0.seg, cons))) return rc;
        }
    }
    const Best leaders2[3] = {be, bo, bt};
    for (int pass = 0; pass < 3; ++pass) {
        const Best b0 = leaders2[pass];
        if (b0.k < 0) continue;
        for (int bps : {1, 2, 3}) {
            if (tma_configure(c, b0.k, b0.st, b0.cons, bps, b0.seg)) continue;
            if ((rc = timed(b0.k, b0.st, b0.seg, b0.cons))) return rc;
        }
    }
    if (bt.k > 0 && bt.ms < best_ms) best_ms = bt.ms, best = bt.ch;  // one shape for both parities
    if (be.k > 0) {
        const bool same = be.ch.threads == bo.ch.threads && be.ch.grid == bo.ch.grid && be.ch.smem == bo.ch.smem &&
                          be.ch.t.k == bo.ch.t.k && be.ch.t.stages == bo.ch.t.stages && be.ch.t.nseg == bo.ch.t.nseg;
        if (!same) {  // the parities' own shapes, measured together (a change of shape between launches costs too)
            load_choice(c, split_choice(be.ch, bo.ch));
            double ms;
            if ((rc = time_choice(c, steps, &ms))) return rc;
            ++ncand;
            if (ms < best_ms) best_ms = ms, best = save_choice(c);
        }
    }
    load_choice(c, best);
    describe_kernel(c);
    // leave the context as created: no state, counters clear
    if ((rc = reset_counters(c))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->have_state = 0;
    if (report && report_len)
        snprintf(report, report_len, "%s: %.4f ms/step (best of %d launch shapes, %d steps each)", c->kernel_desc,
                 best_ms, ncand, steps);
    return DNSLBM_OK;
}

// ---------------------------------------------------------------- batches
struct dnslbm_batch {
    std::vector<dnslbm_ctx *> ch;
    int precision = 64, device = 0;
    cudaStream_t stream = nullptr;
    ChannelLaunch *d_launch = nullptr;
    LinksLaunch *d_links = nullptr;  // channels with planes next to solids
    int nlinks = 0, links_blocks = 0;
    int target = 0;                  // resident blocks of the row-pipelined kernel
    int grid = 0, threads = 0;
    size_t smem = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // a chunk of steps starting on an even / odd parity
    int graph_steps = 32;
    // the persistent kernel (default): one cooperative launch per chunk of
    // steps, blocks taking items of work from a per-step counter
    int persistent = 1;
    int any_q = 0;                      // some channel runs with a constant flow rate
    int pgrid = 0;                      // its blocks (all resident)
    size_t pstage = 0, psmem = 0;       // bytes of one stage, dynamic shared memory
    std::vector<BatchItem> items;       // the items of one step, largest first
    int items_per_block = 4;            // items per resident block and step the items are cut for
    std::vector<BatchItem> items_uploaded;
    BatchItem *d_items = nullptr;
    size_t d_items_cap = 0;
    unsigned *d_counters = nullptr;     // [graph_steps] items taken per step
    unsigned *d_arrivals = nullptr;     // grid-barrier arrivals
    int *d_abort = nullptr;             // a bounded wait of the launch gave up
    int graph_ok = 1;                   // 0: stream capture of the cooperative launch was refused
    int withhold = 0;                   // test hook: the next run withholds a load
    unsigned long long withhold_wait_ns = 0;
    char graph_note[160] = {0};
    size_t budget = 0;  // shared-memory budget per block the stages were sized for
    int stages = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaStream_t side = nullptr;             // the per-cell pass beside the bulk kernel
    cudaEvent_t fj[2] = {nullptr, nullptr};  // fork / join of the side stream
    char err[512] = {0};
};

static int bfail(dnslbm_batch *b, int code, const char *fmt, ...)
{
    char *dst = b ? b->err : g_create_err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(dst, 512, fmt, ap);
    va_end(ap);
    return code;
}

#define BCK(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) return bfail(b, DNSLBM_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

extern "C" const char *dnslbm_batch_last_error(const dnslbm_batch *b) { return b ? b->err : g_create_err; }

static void destroy_graphs(dnslbm_batch *b)
{
    for (auto &g : b->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

extern "C" void dnslbm_batch_destroy(dnslbm_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    destroy_graphs(b);
    for (auto &e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->d_launch) cudaFree(b->d_launch);
    if (b->d_links) cudaFree(b->d_links);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_counters) cudaFree(b->d_counters);
    if (b->d_arrivals) cudaFree(b->d_arrivals);
    if (b->d_abort) cudaFree(b->d_abort);
    for (auto &e : b->fj)
        if (e) cudaEventDestroy(e);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (auto *c : b->ch) dnslbm_destroy(c);
    delete b;
}

// Shared-memory budgets per block for one, two and three blocks per SM
// (228 KB per SM, 1 KB of it reserved per block, the static shared memory of
// the kernel on top).
constexpr size_t kBatchBudget1 = 220 * 1024, kBatchBudget2 = 108 * 1024, kBatchBudget3 = 70 * 1024;

// Row groups of every channel's planes without link masks shared among the
// resident blocks, each block taking whole row groups of one channel and
// about the same number of cells, and the block count of the per-cell pass
// over the planes with link masks.  A change of
// either grid invalidates the captured graphs.
static void persist_items(dnslbm_batch *b);

static void batch_layout(dnslbm_batch *b)
{
    // a common amount of work per block (cells of whole row groups), the
    // smallest for which the blocks fit the resident set at once
    double total = 0;
    for (auto *c : b->ch) total += (double)c->nx * c->ny * c->nclean;
    const int target = std::max(1, b->target);
    auto blocks_for = [&](double w, dnslbm_ctx *c) {
        const double cells = (double)c->nx * c->ny * c->nclean;
        if (cells <= 0) return 0;
        const int ng = c->tma.gpp * c->nclean;
        const int want = std::max(1, std::min(ng, (int)std::ceil(cells / w)));
        const int gpb = (ng + want - 1) / want;
        return (ng + gpb - 1) / gpb;
    };
    double w = std::max(1.0, total / target);
    for (int it = 0; it < 400; ++it, w *= 1.01) {
        int sum = 0;
        for (auto *c : b->ch) sum += blocks_for(w, c);
        if (sum <= target) break;
    }
    int grid = 0, lblocks = 0, nl = 0;
    for (auto *c : b->ch) {
        TmaArgs &t = c->tma;
        t.ngroups = t.gpp * c->nclean;
        t.planes = c->nclean < c->nz ? c->plane_list : nullptr;
        const int nb = blocks_for(w, c);
        t.groups_per_block = nb > 0 ? (t.ngroups + nb - 1) / nb : 1;
        c->tma_grid = nb;
        grid += c->tma_grid;
        if (c->ndirty > 0) {
            lblocks += c->ndirty * (int)(c->grid.x * c->grid.y);
            ++nl;
        }
    }
    if (grid != b->grid || lblocks != b->links_blocks) destroy_graphs(b);
    b->grid = grid;
    b->links_blocks = lblocks;
    b->nlinks = nl;
    if (b->persistent) persist_items(b);
}

// The items of one step of the persistent kernel: each plane of each
// channel cut into runs of whole row groups of about W cells, W chosen so
// that every resident block takes about items_per_block items per step (more
// and smaller items even out the blocks' ends of a step, at a cost per
// item; the batch autotuner picks the count); kind 1 for the
// planes with link masks (the channel's plane list holds them after the
// others, so the group numbering covers them).  Largest first, so the last
// items taken are the small ones.  An item's slot is its index within its
// plane, so the plane sums do not depend on which block takes it.
static void persist_items(dnslbm_batch *b)
{
    double total = 0;
    for (auto *c : b->ch) total += (double)c->nx * c->ny * c->nz;
    const double W = std::max(1.0, total / ((double)b->items_per_block * std::max(1, b->pgrid)));
    std::vector<BatchItem> it;
    std::vector<double> cells;
    for (int ci = 0; ci < (int)b->ch.size(); ++ci) {
        dnslbm_ctx *c = b->ch[ci];
        const TmaArgs &t = c->tma;
        for (int pi = 0; pi < c->nz; ++pi) {
            const double gcells = (double)t.k * c->nx;
            const int per = std::max(1, (int)(W / gcells));
            const int n = (t.gpp + per - 1) / per;
            for (int j = 0; j < n; ++j) {
                const int g0 = (int)((long long)t.gpp * j / n), g1 = (int)((long long)t.gpp * (j + 1) / n);
                BatchItem x{};
                x.chan = ci;
                x.kind = pi < c->nclean ? 0 : 1;
                x.first = pi * t.gpp + g0;
                x.count = g1 - g0;
                x.plane = c->plane_host[pi];
                x.slot = j;
                x.ncontrib = n;
                it.push_back(x);
                cells.push_back(std::min((double)(g1 - g0) * t.k, (double)c->ny) * c->nx);
            }
        }
    }
    std::vector<int> order(it.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return cells[a] > cells[c]; });
    b->items.resize(it.size());
    for (size_t i = 0; i < order.size(); ++i) b->items[i] = it[order[i]];
}

// Shape of the persistent kernel for the current stages and consumers:
// stage bytes of the largest channel, dynamic shared memory, resident grid.
static int persist_configure(dnslbm_batch *b)
{
    size_t stage = 0;
    for (auto *c : b->ch) stage = std::max(stage, (size_t)Q * c->tma.row_bytes * c->tma.k);
    const size_t smem = persist_smem(b->stages, stage);
    int maxsmem = 0, nsm = 0;
    cudaDeviceGetAttribute(&maxsmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
    const size_t cap = (size_t)maxsmem - kStaticSmemReserve;
    if (smem > cap || nsm < 1) return -1;
    b->any_q = 0;
    for (auto *c : b->ch) b->any_q |= c->deck.force_mode == DNSLBM_FORCE_CONST_Q;
    const int occ =
        persist_prepare(b->precision, cap) ? 0 : persist_occupancy_of(b->precision, b->threads, smem, b->any_q != 0);
    cudaGetLastError();
    if (occ < 1) return -1;
    b->pstage = stage;
    b->psmem = smem;
    b->pgrid = occ * nsm;
    return 0;
}

// One launch shape for all channels: per channel the most rows per stage
// group (up to 16) whose `stages` groups fit `budget` bytes, so channels of
// short rows move about as many bytes per stage as those of long rows; the
// block takes the largest of these stages.  Returns 0 and selects the shape
// when it runs on the device.
static int batch_configure(dnslbm_batch *b, size_t budget, int stages, int consumers)
{
    consumers = std::max(32, std::min(352, consumers / 32 * 32));
    size_t smem = 0;
    std::vector<int> ks(b->ch.size());
    for (size_t i = 0; i < b->ch.size(); ++i) {
        dnslbm_ctx *c = b->ch[i];
        const int row_bytes = c->pitch * (int)c->esize;
        auto need = [&](int k) { return (size_t)stages * Q * row_bytes * k + 16 * (size_t)stages; };
        if (need(1) > budget) return -1;
        int k = 1;
        while (k < 16 && k + 1 <= c->ny && need(k + 1) <= budget) ++k;
        ks[i] = k;
        smem = std::max(smem, need(k));
    }
    const int threads = consumers + 32;
    int maxsmem = 0;
    cudaDeviceGetAttribute(&maxsmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device);
    const size_t cap = (size_t)maxsmem - kStaticSmemReserve;
    if (smem > cap) return -1;
    const int prep = b->precision == 64 ? tma_batch_prepare_f64(cap) : tma_batch_prepare_lp(b->precision, cap);
    const int occ = prep ? 0
                         : (b->precision == 64 ? tma_batch_occupancy_f64(threads, smem)
                                               : tma_batch_occupancy_lp(b->precision, threads, smem));
    cudaGetLastError();  // a failed query only rules the shape out
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
    if (occ < 1 || nsm < 1) return -1;
    for (size_t i = 0; i < b->ch.size(); ++i) {
        dnslbm_ctx *c = b->ch[i];
        const int row_bytes = c->pitch * (int)c->esize;
        c->tma = TmaArgs{0, 1, stages, row_bytes, ks[i], (c->ny + ks[i] - 1) / ks[i], nullptr, 1, c->nx,
                         ks[i] * c->pitch};
        c->odd_split = 0;
        c->tma_threads = threads;
        c->tma_smem = smem;
        c->tma_target = occ * nsm;
    }
    b->target = occ * nsm;
    b->threads = threads;
    b->smem = smem;
    b->budget = budget;
    b->stages = stages;
    if (b->persistent && persist_configure(b)) return -1;
    destroy_graphs(b);
    batch_layout(b);
    return 0;
}

extern "C" int dnslbm_batch_create(const dnslbm_deck *decks, int n, dnslbm_batch **out)
{
    dnslbm_batch *b = nullptr;
    if (!decks || !out || n < 1) return bfail(b, DNSLBM_ERR_ARG, "need at least one deck and an output pointer");
    *out = nullptr;
    for (int i = 1; i < n; ++i)
        if (decks[i].precision != decks[0].precision || decks[i].device != decks[0].device)
            return bfail(b, DNSLBM_ERR_ARG, "all channels of a batch share one precision and one device");
    b = new dnslbm_batch();
    b->precision = decks[0].precision;
    b->device = decks[0].device;
    // DNSLBM_BATCH=launch: one launch of the per-step batch kernel per step
    // (the layout before the persistent kernel, kept for comparison)
    if (const char *e = getenv("DNSLBM_BATCH")) b->persistent = strcmp(e, "launch") != 0;
    for (int i = 0; i < n; ++i) {
        dnslbm_ctx *c = nullptr;
        int rc = dnslbm_create(&decks[i], &c);
        if (rc) {
            char msg[512];
            snprintf(msg, sizeof msg, "channel %d: %s", i, g_create_err);
            dnslbm_batch_destroy(b);
            snprintf(g_create_err, sizeof g_create_err, "%s", msg);
            return rc;
        }
        b->ch.push_back(c);
        if (!c->use_tma) {
            dnslbm_batch_destroy(b);
            snprintf(g_create_err, sizeof g_create_err,
                     "channel %d does not fit the row-pipelined kernel (rows too long for two stages)", i);
            return DNSLBM_ERR_ARG;
        }
    }
    auto bail = [&](int code) {
        snprintf(g_create_err, sizeof g_create_err, "%s", b->err);
        dnslbm_batch_destroy(b);
        return code;
    };
    if (cudaSetDevice(b->device) != cudaSuccess) return bail(bfail(b, DNSLBM_ERR_CUDA, "cannot select device"));
    // default launch shape: stages sized for two blocks per SM, the widest
    // consumer set any channel would use alone
    int consumers = 32;
    for (auto *c : b->ch) consumers = std::max(consumers, c->tma_threads - 32);
    if (batch_configure(b, kBatchBudget2, 2, consumers) && batch_configure(b, kBatchBudget1, 2, consumers))
        return bail(bfail(b, DNSLBM_ERR_ARG, "batched kernel does not fit the device"));
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev[0]) != cudaSuccess || cudaEventCreate(&b->ev[1]) != cudaSuccess ||
        cudaMalloc(&b->d_launch, sizeof(ChannelLaunch) * n) != cudaSuccess ||
        cudaMalloc(&b->d_links, sizeof(LinksLaunch) * n) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fj[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fj[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&b->d_counters, sizeof(unsigned) * b->graph_steps) != cudaSuccess ||
        cudaMalloc(&b->d_arrivals, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&b->d_abort, sizeof(int)) != cudaSuccess || cudaMemset(b->d_abort, 0, sizeof(int)) != cudaSuccess)
        return bail(bfail(b, DNSLBM_ERR_CUDA, "batch set-up failed: %s", cudaGetErrorString(cudaGetLastError())));
    *out = b;
    return DNSLBM_OK;
}

extern "C" int dnslbm_batch_size(const dnslbm_batch *b) { return b ? (int)b->ch.size() : 0; }
extern "C" dnslbm_ctx *dnslbm_batch_channel(dnslbm_batch *b, int i)
{
    return b && i >= 0 && i < (int)b->ch.size() ? b->ch[i] : nullptr;
}

static int batch_launch(dnslbm_batch *b, bool odd)
{
    // the bulk kernel and, beside it on a second stream, the per-cell pass
    const bool both = b->grid > 0 && b->links_blocks > 0;
    cudaStream_t ls = both ? b->side : b->stream;
    if (both) {
        BCK(cudaEventRecord(b->fj[0], b->stream));
        BCK(cudaStreamWaitEvent(b->side, b->fj[0], 0));
    }
    if (b->grid > 0) {
        if (b->precision == 64)
            launch_tma_batch_f64(b->d_launch, (int)b->ch.size(), b->grid, b->threads, b->smem, odd, b->stream);
        else
            launch_tma_batch_lp(b->precision, b->d_launch, (int)b->ch.size(), b->grid, b->threads, b->smem, odd,
                                b->stream);
    }
    if (b->links_blocks > 0) {
        if (b->precision == 64) launch_links_f64(b->d_links, b->nlinks, b->links_blocks, odd, ls);
        else launch_links_lp(b->precision, b->d_links, b->nlinks, b->links_blocks, odd, ls);
    }
    if (both) {
        BCK(cudaEventRecord(b->fj[1], b->side));
        BCK(cudaStreamWaitEvent(b->stream, b->fj[1], 0));
    }
    BCK(cudaGetLastError());
    return DNSLBM_OK;
}

// The persistent kernel's chunk of n steps from parity `odd`: counters and
// barrier arrivals cleared, then one cooperative launch.
static int persist_launch(dnslbm_batch *b, int n, int odd)
{
    PersistArgs a;
    a.chans = b->d_launch;
    a.items = b->d_items;
    a.nitems = (int)b->items.size();
    a.nsteps = n;
    a.first_odd = odd;
    a.stages = b->stages;
    a.stage_bytes = (unsigned)b->pstage;
    a.counters = b->d_counters;
    a.arrivals = b->d_arrivals;
    a.abort = b->d_abort;
    a.wait_ns = b->withhold ? b->withhold_wait_ns : b->ch[0]->wait_ns;
    a.withhold = b->withhold;
    BCK(cudaMemsetAsync(b->d_counters, 0, sizeof(unsigned) * n, b->stream));
    BCK(cudaMemsetAsync(b->d_arrivals, 0, sizeof(unsigned), b->stream));
    BCK(launch_persist_batch(b->precision, a, b->pgrid, b->threads, b->psmem, b->any_q != 0, b->stream));
    return DNSLBM_OK;
}

static int persist_run(dnslbm_batch *b, long nsteps)
{
    int odd = b->ch[0]->odd;
    long left = nsteps;
    BCK(cudaMemsetAsync(b->d_abort, 0, sizeof(int), b->stream));
    while (left > 0) {
        const int n = (int)std::min<long>(left, b->graph_steps);
        if (n == b->graph_steps && b->graph_ok && !b->withhold) {
            cudaGraphExec_t &g = b->graph[odd];
            if (!g) {
                // the time loop's chunk captured as a graph; a driver that
                // refuses to capture the cooperative launch leaves plain
                // launches (noted in the kernel description)
                cudaGraph_t graph = nullptr;
                BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
                const int rc = persist_launch(b, n, odd);
                cudaError_t ee = cudaStreamEndCapture(b->stream, &graph);
                if (rc == DNSLBM_OK && ee == cudaSuccess) ee = cudaGraphInstantiate(&g, graph, 0);
                if (graph) cudaGraphDestroy(graph);
                if (rc != DNSLBM_OK || ee != cudaSuccess) {
                    cudaGetLastError();
                    g = nullptr;
                    b->graph_ok = 0;
                    snprintf(b->graph_note, sizeof b->graph_note, " (graph capture refused: %s)",
                             ee != cudaSuccess ? cudaGetErrorString(ee) : b->err);
                    continue;
                }
            }
            BCK(cudaGraphLaunch(g, b->stream));
        } else {
            const int rc = persist_launch(b, n, odd);
            b->withhold = 0;
            if (rc) return rc;
        }
        left -= n;
        odd = (odd + n) & 1;
    }
    return DNSLBM_OK;
}

static int batch_run(dnslbm_batch *b, long nsteps, double *ms)
{
    const int n = (int)b->ch.size();
    for (int i = 0; i < n; ++i) {
        dnslbm_ctx *c = b->ch[i];
        if (!c->have_state) return bfail(b, DNSLBM_ERR_STATE, "channel %d has no state", i);
        if (c->done != b->ch[0]->done || c->odd != b->ch[0]->odd)
            return bfail(b, DNSLBM_ERR_STATE, "channel %d is at step %lld, channel 0 at %lld", i, c->done,
                         b->ch[0]->done);
        if (c->stream) BCK(cudaStreamSynchronize(c->stream));
    }
    BCK(cudaSetDevice(b->device));
    // launch tables (flags may have changed a channel's walls and planes)
    batch_layout(b);
    std::vector<ChannelLaunch> h(n);
    std::vector<LinksLaunch> hl;
    int first = 0, lfirst = 0;
    for (int i = 0; i < n; ++i) {
        dnslbm_ctx *c = b->ch[i];
        h[i].p = step_args(c);
        h[i].t = c->tma;
        h[i].first_block = first;
        h[i].textured = c->walls_textured;
        first += c->tma_grid;
        if (c->ndirty > 0) {
            LinksLaunch L{};
            L.p = h[i].p;
            L.planes = c->plane_list + c->nclean;
            L.nplanes = c->ndirty;
            L.xblocks = (int)c->grid.x;
            L.yblocks = (int)c->grid.y;
            L.rows = c->rows;
            L.first_block = lfirst;
            lfirst += c->ndirty * L.xblocks * L.yblocks;
            hl.push_back(L);
        }
    }
    BCK(cudaMemcpyAsync(b->d_launch, h.data(), sizeof(ChannelLaunch) * n, cudaMemcpyHostToDevice, b->stream));
    if (!hl.empty())
        BCK(cudaMemcpyAsync(b->d_links, hl.data(), sizeof(LinksLaunch) * hl.size(), cudaMemcpyHostToDevice,
                            b->stream));
    if (b->persistent) {
        // the item table (a new one invalidates the captured graphs, which
        // hold its address and length)
        if (b->items.size() > b->d_items_cap) {
            if (b->d_items) cudaFree(b->d_items);
            b->d_items = nullptr;
            b->d_items_cap = 0;
            BCK(cudaMalloc(&b->d_items, sizeof(BatchItem) * b->items.size()));
            b->d_items_cap = b->items.size();
            destroy_graphs(b);
        }
        if (b->items.size() != b->items_uploaded.size() ||
            memcmp(b->items.data(), b->items_uploaded.data(), sizeof(BatchItem) * b->items.size())) {
            destroy_graphs(b);
            b->items_uploaded = b->items;
        }
        BCK(cudaMemcpyAsync(b->d_items, b->items.data(), sizeof(BatchItem) * b->items.size(),
                            cudaMemcpyHostToDevice, b->stream));
    }
    int odd = b->ch[0]->odd;
    long left = nsteps;
    if (ms) BCK(cudaEventRecord(b->ev[0], b->stream));
    if (b->persistent) {
        const int rc = persist_run(b, nsteps);
        if (rc) return rc;
        left = 0;
    }
    // the time loop: chunks of graph_steps launches replayed from a CUDA graph
    while (left >= b->graph_steps) {
        cudaGraphExec_t &g = b->graph[odd];
        if (!g) {
            cudaGraph_t graph;
            BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            int rc = DNSLBM_OK;
            for (int s = 0; s < b->graph_steps && rc == DNSLBM_OK; ++s) rc = batch_launch(b, ((odd + s) & 1) != 0);
            cudaError_t ee = cudaStreamEndCapture(b->stream, &graph);
            if (rc) return rc;
            if (ee != cudaSuccess) return bfail(b, DNSLBM_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ee));
            ee = cudaGraphInstantiate(&g, graph, 0);
            cudaGraphDestroy(graph);
            if (ee != cudaSuccess) return bfail(b, DNSLBM_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ee));
        }
        BCK(cudaGraphLaunch(g, b->stream));
        left -= b->graph_steps;
        odd = (odd + b->graph_steps) & 1;
    }
    for (; left > 0; --left) {
        int rc = batch_launch(b, odd != 0);
        if (rc) return rc;
        odd ^= 1;
    }
    if (ms) BCK(cudaEventRecord(b->ev[1], b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    if (ms) {
        float f = 0.f;
        BCK(cudaEventElapsedTime(&f, b->ev[0], b->ev[1]));
        *ms = f;
    }
    for (int i = 0; i < n; ++i) {
        dnslbm_ctx *c = b->ch[i];
        c->done += nsteps;
        c->odd = (c->odd + (int)(nsteps & 1)) & 1;
    }
    if (b->persistent) {
        int ab = 0;
        BCK(cudaMemcpy(&ab, b->d_abort, sizeof ab, cudaMemcpyDeviceToHost));
        if (ab) {
            for (auto *c : b->ch) c->have_state = 0;
            return bfail(b, DNSLBM_ERR_TIMEOUT, "a bounded wait of the persistent batch kernel ran out; states "
                                                "invalid, reload them");
        }
    }
    for (int i = 0; i < n; ++i) {
        int rc = check_status(b->ch[i]);
        if (rc) return bfail(b, rc, "channel %d: %s", i, b->ch[i]->err);
    }
    return DNSLBM_OK;
}

extern "C" int dnslbm_batch_step(dnslbm_batch *b, long nsteps)
{
    if (!b || nsteps < 0) return bfail(b, DNSLBM_ERR_ARG, "bad batch or step count");
    return batch_run(b, nsteps, nullptr);
}

extern "C" int dnslbm_batch_step_timed(dnslbm_batch *b, long nsteps, double *ms)
{
    if (!b || nsteps < 1 || !ms) return bfail(b, DNSLBM_ERR_ARG, "bad batch, step count or output");
    return batch_run(b, nsteps, ms);
}

extern "C" int dnslbm_batch_test_withhold_load(dnslbm_batch *b, double wait_ms)
{
    if (!b) return bfail(b, DNSLBM_ERR_ARG, "null batch");
    if (!b->persistent) return bfail(b, DNSLBM_ERR_STATE, "the batch steps with one launch per step");
    if (!(wait_ms > 0.0 && wait_ms <= 600000.0)) return bfail(b, DNSLBM_ERR_ARG, "wait limit %g ms out of range", wait_ms);
    b->withhold = 1;
    b->withhold_wait_ns = (unsigned long long)(wait_ms * 1e6);
    return DNSLBM_OK;
}

extern "C" const char *dnslbm_batch_kernel(const dnslbm_batch *b)
{
    static thread_local char buf[384];
    if (!b) return "";
    if (b->persistent) {
        snprintf(buf, sizeof buf,
                 "persist_batch_kernel<fp%d>: %zu channels, %zu items per step, %d blocks x %d threads, %d stages, "
                 "%zu B smem; one cooperative launch per %d steps, CUDA graph%s",
                 b->precision, b->ch.size(), b->items.size(), b->pgrid, b->threads, b->stages, b->psmem,
                 b->graph_steps, b->graph_note);
        return buf;
    }
    snprintf(buf, sizeof buf, "step_tma_batch_kernel<fp%d>: %zu channels, %d blocks x %d threads, %d stages, %zu B smem"
             "%s%s; CUDA graph of %d steps", b->precision, b->ch.size(), b->grid, b->threads, b->stages, b->smem,
             b->links_blocks ? " + links_pass_kernel: " : "",
             b->links_blocks ? (std::to_string(b->links_blocks) + " blocks").c_str() : "", b->graph_steps);
    return buf;
}

extern "C" int dnslbm_batch_autotune(dnslbm_batch *b, int steps, char *report, size_t report_len)
{
    if (!b) return bfail(b, DNSLBM_ERR_ARG, "null batch");
    for (size_t i = 0; i < b->ch.size(); ++i)
        if (b->ch[i]->have_state)
            return bfail(b, DNSLBM_ERR_STATE, "autotune runs before any state is loaded (it steps rest states)");
    if (steps < 2) steps = 2;
    if (steps >= b->graph_steps) steps = b->graph_steps - 1;  // plain launches, no graph to capture
    BCK(cudaSetDevice(b->device));
    size_t bb = b->budget;
    int bs = b->stages, bc = b->threads - 32, ncand = 0;
    double best = 1e30;
    for (size_t budget : {kBatchBudget1, kBatchBudget2, kBatchBudget3})
        for (int st : {2, 3, 4})
            for (int cons : {64, 128, 192, 256, 320}) {
                if (batch_configure(b, budget, st, cons)) continue;
                int rc = DNSLBM_OK;
                for (auto *c : b->ch)
                    if ((rc = dnslbm_init_rest(c))) return bfail(b, rc, "%s", c->err);
                double ms = 0;
                if ((rc = batch_run(b, 2, nullptr)) || (rc = batch_run(b, steps, &ms))) return rc;
                ++ncand;
                if (ms < best) best = ms, bb = budget, bs = st, bc = cons;
            }
    // the persistent kernel: how finely each step's work is cut, at the best shape
    if (b->persistent) {
        int bi = b->items_per_block;
        for (int ipb : {2, 8, 16}) {
            b->items_per_block = ipb;
            if (batch_configure(b, bb, bs, bc)) continue;
            int rc = DNSLBM_OK;
            for (auto *c : b->ch)
                if ((rc = dnslbm_init_rest(c))) return bfail(b, rc, "%s", c->err);
            double ms = 0;
            if ((rc = batch_run(b, 2, nullptr)) || (rc = batch_run(b, steps, &ms))) return rc;
            ++ncand;
            if (ms < best) best = ms, bi = ipb;
        }
        b->items_per_block = bi;
    }
    // leave the channels as created: no state, counters clear
    for (auto *c : b->ch) {
        int rc = reset_counters(c);
        if (rc) return bfail(b, rc, "%s", c->err);
        c->have_state = 0;
    }
    if (batch_configure(b, bb, bs, bc)) return bfail(b, DNSLBM_ERR_CUDA, "cannot restore the chosen launch shape");
    BCK(cudaDeviceSynchronize());
    if (report && report_len)
        snprintf(report, report_len, "%s: %.4f ms/step (best of %d launch shapes, %d steps each)",
                 dnslbm_batch_kernel(b), best / steps, ncand, steps);
    return DNSLBM_OK;
}
