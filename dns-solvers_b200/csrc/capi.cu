// C-ABI implementation: device context, flags, state I/O and the step driver.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/dnslbm.h"
#include "step_common.cuh"

namespace dnslbm {
void launch_step_f64(const StepArgs &p, dim3 grid, dim3 block, bool odd, bool textured, cudaStream_t s);
void launch_reduce_f64(const StepArgs &p, dim3 grid, dim3 block, cudaStream_t s);
void launch_step_lp(int precision, const StepArgs &p, dim3 grid, dim3 block, bool odd, bool textured, cudaStream_t s);
void launch_reduce_lp(int precision, const StepArgs &p, dim3 grid, dim3 block, cudaStream_t s);
void launch_io(int precision, int what, const IoArgs &p, int x0, int nxc, double *a, double *b, cudaStream_t s);
void launch_stats(int precision, const IoArgs &p, dim3 grid, dim3 block, int rows, int pass, const double *mean,
                  double *partials, double *plane_out, cudaStream_t s);
struct TmaArgs {
    int ngroups, groups_per_block, stages, row_bytes, k, gpp;
};
int tma_prepare_f64(size_t smem);
int tma_occupancy_f64(int threads, size_t smem);
void launch_tma_f64(const StepArgs &p, const TmaArgs &t, int grid, int threads, size_t smem, bool odd, bool textured,
                    cudaStream_t s);
int tma_prepare_lp(int precision, size_t smem);
int tma_occupancy_lp(int precision, int threads, size_t smem);
void launch_tma_lp(int precision, const StepArgs &p, const TmaArgs &t, int grid, int threads, size_t smem, bool odd,
                   bool textured, cudaStream_t s);
}  // namespace dnslbm

using namespace dnslbm;

struct dnslbm_ctx {
    dnslbm_deck deck;
    int nx, ny, nz;
    int pitch;  // row pitch in elements: rows padded to 16 bytes for bulk copies
    size_t ncell, pstride, esize;
    void *popmem = nullptr;
    uint8_t *wallmask = nullptr;
    int textured = 0;
    double *force = nullptr, *shift = nullptr, *partials = nullptr, *plane_sums = nullptr, *logs = nullptr;
    long long *step_ctr = nullptr, *status = nullptr;
    unsigned *plane_ctr = nullptr, *total_ctr = nullptr;
    double *staging = nullptr;  // device AoS staging for I/O
    size_t staging_bytes = 0;
    double *stat_partials = nullptr, *stat_planes = nullptr, *stat_mean = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::vector<cudaEvent_t> tev;  // per-launch timing events
    dim3 grid, block;
    int rows = 8;
    int slots = 1;  // partial-sum slots per plane
    // row-pipelined (bulk-copy) step
    int use_tma = 0, tma_threads = 0, tma_grid = 0;
    char kernel_desc[160] = {0};
    size_t tma_smem = 0;
    TmaArgs tma{};
    int have_state = 0;
    int odd = 0;  // parity of the next step (1: populations are post-collision, swapped)
    long long done = 0;
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
    for (int a = 0; a < Q; ++a) p.pop[a] = (char *)c->popmem + (size_t)a * c->pstride * c->esize;
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
    return p;
}

static IoArgs io_args(const dnslbm_ctx *c)
{
    IoArgs p;
    for (int a = 0; a < Q; ++a) p.pop[a] = (char *)c->popmem + (size_t)a * c->pstride * c->esize;
    p.nx = c->nx;
    p.ny = c->ny;
    p.nz = c->nz;
    p.pitch = c->pitch;
    p.wallmask = c->wallmask;
    p.textured = c->textured;
    p.odd = c->odd;
    return p;
}

static void free_all(dnslbm_ctx *c)
{
    void *ptrs[] = {c->popmem, c->wallmask, c->force, c->shift, c->partials, c->plane_sums, c->logs, c->step_ctr,
                    c->status, c->plane_ctr, c->total_ctr, c->staging, c->stat_partials, c->stat_planes, c->stat_mean};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (auto &e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : c->tev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
}

extern "C" const char *dnslbm_last_error(const dnslbm_ctx *c) { return c ? c->err : g_create_err; }

// Configure the row-pipelined step with k rows per stage group, `stages`
// groups in flight and `consumers` compute threads (+ one producer warp);
// bps > 0 caps the blocks per SM.  Returns 0 when the configuration runs on
// this device (and selects it), -1 otherwise (the previous choice stays).
static int tma_configure(dnslbm_ctx *c, int k, int stages, int consumers, int bps)
{
    const int row_bytes = c->pitch * (int)c->esize;
    k = std::max(1, std::min(k, c->ny));
    consumers = std::max(32, std::min(352, consumers / 32 * 32));
    const size_t smem_stage = (size_t)Q * row_bytes * k;
    int maxsmem = 0, nsm = 0;
    cudaDeviceGetAttribute(&maxsmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->deck.device);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->deck.device);
    const size_t smem = (size_t)stages * smem_stage + 16 * (size_t)stages;  // + full/empty mbarriers
    if (stages < 2 || smem > (size_t)maxsmem || nsm <= 0) return -1;
    const int threads = consumers + 32;
    const int prep = c->deck.precision == 64 ? tma_prepare_f64(smem) : tma_prepare_lp(c->deck.precision, smem);
    int occ = prep ? 0
                   : (c->deck.precision == 64 ? tma_occupancy_f64(threads, smem)
                                              : tma_occupancy_lp(c->deck.precision, threads, smem));
    cudaGetLastError();  // a failed query only rules the configuration out
    if (bps > 0) occ = std::min(occ, bps);
    if (occ < 1) return -1;
    const int gpp = (c->ny + k - 1) / k, ngroups = gpp * c->nz;
    const int target = occ * nsm;
    const int GB = (ngroups + target - 1) / target;
    c->use_tma = 1;
    c->tma_threads = threads;
    c->tma_smem = smem;
    c->tma_grid = (ngroups + GB - 1) / GB;
    c->tma = TmaArgs{ngroups, GB, stages, row_bytes, k, gpp};
    return 0;
}

static void describe_kernel(dnslbm_ctx *c)
{
    if (c->use_tma)
        snprintf(c->kernel_desc, sizeof c->kernel_desc,
                 "step_tma_kernel<fp%d> row-pipelined bulk-copy: %d blocks x %d threads, %d groups of %d rows/block, "
                 "%d stages, %zu B smem",
                 c->deck.precision, c->tma_grid, c->tma_threads, c->tma.groups_per_block, c->tma.k, c->tma.stages,
                 c->tma_smem);
    else
        snprintf(c->kernel_desc, sizeof c->kernel_desc, "%s per-thread: grid %ux%ux%u x %u threads",
                 c->deck.precision == 64 ? "step_f64_kernel" : "step_lp_kernel", c->grid.x, c->grid.y, c->grid.z,
                 c->block.x);
}

extern "C" int dnslbm_create(const dnslbm_deck *deck, dnslbm_ctx **out)
{
    dnslbm_ctx *c = nullptr;
    if (!deck || !out) return fail(c, DNSLBM_ERR_ARG, "null deck or output pointer");
    *out = nullptr;
    if (deck->xdv < 2 || deck->ydv < 2 || deck->zdv < 3)
        return fail(c, DNSLBM_ERR_ARG, "grid %dx%dx%d too small (need xdv,ydv >= 2, zdv >= 3)", deck->xdv, deck->ydv,
                    deck->zdv);
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
    c->nz = deck->zdv;
    c->esize = deck->precision / 8;
    {
        // rows start on `align` bytes (16 at least, for the bulk copies)
        int align_bytes = 32;
        if (const char *e = getenv("DNSLBM_ROW_ALIGN")) align_bytes = std::max(16, atoi(e));
        const int v = align_bytes / (int)c->esize;
        c->pitch = (c->nx + v - 1) / v * v;
    }
    c->ncell = (size_t)c->pitch * c->ny * c->nz;
    const size_t align = 256 / c->esize;
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
    c->slots = (int)(c->grid.x * c->grid.y);
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
        if (!(path && !strcmp(path, "scalar"))) tma_configure(c, k, stages, consumers, bps);
        describe_kernel(c);
    }
    // partial-sum slots: enough for the per-thread kernels and for any row
    // group split the tuner may choose
    c->slots = std::max(c->slots, c->ny + 1);
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
    };
    for (auto &a : al) {
        cudaError_t e = cudaMalloc(a.p, a.bytes);
        if (e != cudaSuccess) {
            fail(c, DNSLBM_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", a.bytes, cudaGetErrorString(e));
            return bail(DNSLBM_ERR_NOMEM);
        }
        cudaMemset(*a.p, 0, a.bytes);
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        fail(c, DNSLBM_ERR_CUDA, "cannot create stream");
        return bail(DNSLBM_ERR_CUDA);
    }
    for (auto &e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            fail(c, DNSLBM_ERR_CUDA, "cannot create event");
            return bail(DNSLBM_ERR_CUDA);
        }
    // default flags: smooth no-slip walls (solid_init.c)
    std::vector<uint8_t> m((size_t)2 * c->nx * c->ny, 0x1f);
    if (cudaMemcpy(c->wallmask, m.data(), m.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaDeviceSynchronize() != cudaSuccess) {
        fail(c, DNSLBM_ERR_CUDA, "initialisation failed: %s", cudaGetErrorString(cudaGetLastError()));
        return bail(DNSLBM_ERR_CUDA);
    }
    (void)rc;
    *out = c;
    return DNSLBM_OK;
}

extern "C" void dnslbm_destroy(dnslbm_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->deck.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_all(c);
    delete c;
}

// wall-link bits from the wall-plane flags (xcomputations.c:368-375): the
// link from fluid cell P toward wall cell T bounces back iff s(T) == -1 and
// s(P's own wall cell) == -1; otherwise it reflects specularly.
static int apply_flags(dnslbm_ctx *c, const int8_t *fl /* [nx][ny][zd] */)
{
    const int nx = c->nx, ny = c->ny, zd = c->nz + 2;
    auto S = [&](int x, int y, int k) { return (int)fl[((size_t)x * ny + y) * zd + k]; };
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
            for (int k : {0, zd - 1}) {
                const int v = S(x, y, k);
                if (v != -1 && v != -2)
                    return fail(c, DNSLBM_ERR_ARG, "wall cell (%d,%d,%d) has flag %d; wall planes must be -1 or -2", x, y,
                                k, v);
            }
            for (int k = 1; k < zd - 1; ++k) {
                const int v = S(x, y, k);
                if (v != 0 && v != 1)
                    return fail(c, DNSLBM_ERR_ARG,
                                "cell (%d,%d,%d) has flag %d; solids inside the flow are not supported by this build", x,
                                y, k, v);
            }
        }
    std::vector<uint8_t> m((size_t)2 * nx * ny);
    const int off[5][2] = {{0, 0}, {1, 0}, {-1, 0}, {0, 1}, {0, -1}};
    int textured = 0;
    for (int w = 0; w < 2; ++w) {
        const int k = w == 0 ? 0 : zd - 1;
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                unsigned bits = 0;
                for (int l = 0; l < 5; ++l) {
                    const int xt = (x + off[l][0] + nx) % nx, yt = (y + off[l][1] + ny) % ny;
                    if (S(xt, yt, k) == -1 && S(x, y, k) == -1) bits |= 1u << l;
                }
                m[(size_t)w * nx * ny + (size_t)y * nx + x] = (uint8_t)bits;
                if (bits != 0x1f) textured = 1;
            }
    }
    if (c->have_state && c->odd) {
        // the populations in flight were placed under the old flags
        return fail(c, DNSLBM_ERR_STATE, "flags can only change between even numbers of steps");
    }
    CK(cudaSetDevice(c->deck.device));
    CK(cudaMemcpyAsync(c->wallmask, m.data(), m.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->textured = textured;
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
    const int nx = c->nx, ny = c->ny, zd = c->nz + 2, yd = ny + 1;
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
static int initial_reduce(dnslbm_ctx *c)
{
    StepArgs p = step_args(c);
    if (c->deck.precision == 64) launch_reduce_f64(p, c->grid, c->block, c->stream);
    else launch_reduce_lp(c->deck.precision, p, c->grid, c->block, c->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return DNSLBM_OK;
}

static int reset_counters(dnslbm_ctx *c)
{
    CK(cudaMemsetAsync(c->plane_ctr, 0, (size_t)c->nz * sizeof(unsigned), c->stream));
    CK(cudaMemsetAsync(c->total_ctr, 0, sizeof(unsigned), c->stream));
    CK(cudaMemsetAsync(c->step_ctr, 0, sizeof(long long), c->stream));
    CK(cudaMemsetAsync(c->status, 0, 2 * sizeof(long long), c->stream));
    CK(cudaMemsetAsync(c->shift, 0, (size_t)2 * c->nz * 3 * sizeof(double), c->stream));
    c->done = 0;
    c->odd = 0;
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

extern "C" int dnslbm_store_state(dnslbm_ctx *c, double *state)
{
    if (!c || !state) return fail(c, DNSLBM_ERR_ARG, "null argument");
    if (!c->have_state) return fail(c, DNSLBM_ERR_STATE, "no state loaded");
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
            if (c->deck.precision == 64)
                launch_tma_f64(p, c->tma, c->tma_grid, c->tma_threads, c->tma_smem, odd, c->textured != 0, c->stream);
            else
                launch_tma_lp(c->deck.precision, p, c->tma, c->tma_grid, c->tma_threads, c->tma_smem, odd,
                              c->textured != 0, c->stream);
        } else if (c->deck.precision == 64) {
            launch_step_f64(p, c->grid, c->block, odd, c->textured != 0, c->stream);
        } else {
            launch_step_lp(c->deck.precision, p, c->grid, c->block, odd, c->textured != 0, c->stream);
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
    if (st[1]) return fail(c, DNSLBM_ERR_TIMEOUT, "a bounded wait for a bulk copy ran out; state invalid, reload it");
    if (st[0]) return fail(c, DNSLBM_ERR_NAN, "NaN wall shear stress at step %lld", st[0] - 1);
    return DNSLBM_OK;
}

extern "C" int dnslbm_step(dnslbm_ctx *c, long nsteps)
{
    if (!c) return fail(c, DNSLBM_ERR_ARG, "null context");
    if (nsteps < 0) return fail(c, DNSLBM_ERR_ARG, "negative step count");
    if (!c->have_state) return fail(c, DNSLBM_ERR_STATE, "no state: call dnslbm_init_rest or dnslbm_load_state");
    CK(cudaSetDevice(c->deck.device));
    int rc = launch_steps(c, nsteps, false, nullptr, nullptr);
    if (rc) return rc;
    return check_status(c);
}

extern "C" int dnslbm_step_timed(dnslbm_ctx *c, long nsteps, double *ms_total, double *ms_even, double *ms_odd)
{
    if (!c || !ms_total || !ms_even || !ms_odd) return fail(c, DNSLBM_ERR_ARG, "null argument");
    if (!c->have_state) return fail(c, DNSLBM_ERR_STATE, "no state");
    CK(cudaSetDevice(c->deck.device));
    *ms_even = *ms_odd = 0.0;
    if (nsteps <= 0) return fail(c, DNSLBM_ERR_ARG, "timed run needs at least one step");
    CK(cudaEventRecord(c->ev[0], c->stream));
    int rc = launch_steps(c, nsteps, true, ms_even, ms_odd);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev[1], c->stream));
    CK(cudaEventSynchronize(c->ev[1]));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    *ms_total = ms;
    return check_status(c);
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
    if (!c->have_state) return fail(c, DNSLBM_ERR_STATE, "no state");
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

extern "C" int dnslbm_statistics(dnslbm_ctx *c, double *out)
{
    if (!c || !out) return fail(c, DNSLBM_ERR_ARG, "null argument");
    if (!c->have_state) return fail(c, DNSLBM_ERR_STATE, "no state");
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
    int use_tma, threads, grid;
    size_t smem;
    TmaArgs t;
};

static TmaChoice save_choice(const dnslbm_ctx *c) { return {c->use_tma, c->tma_threads, c->tma_grid, c->tma_smem, c->tma}; }
static void load_choice(dnslbm_ctx *c, const TmaChoice &k)
{
    c->use_tma = k.use_tma;
    c->tma_threads = k.threads;
    c->tma_grid = k.grid;
    c->tma_smem = k.smem;
    c->tma = k.t;
}

// device time per step of the current launch shape, on a rest state
static int time_choice(dnslbm_ctx *c, int steps, double *ms)
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
    // the consumer count for the best pair
    const int cap = c->deck.precision == 64 ? 320 : (c->deck.precision == 32 ? 192 : 128);
    const int cons0 = std::min(cap, (c->nx + 31) / 32 * 32);
    int bk = -1, bs = -1;
    for (int k : {1, 2, 4, 8})
        for (int st : {2, 3, 4}) {
            if (k > c->ny || tma_configure(c, k, st, cons0, 0)) continue;
            double ms;
            if ((rc = time_choice(c, steps, &ms))) return rc;
            ++ncand;
            if (ms < best_ms) best_ms = ms, best = save_choice(c), bk = k, bs = st;
        }
    if (bk > 0)
        for (int cons = 64; cons <= 352 && cons <= (c->nx + 31) / 32 * 32 + 32; cons += 32) {
            if (cons == cons0 || tma_configure(c, bk, bs, cons, 0)) continue;
            double ms;
            if ((rc = time_choice(c, steps, &ms))) return rc;
            ++ncand;
            if (ms < best_ms) best_ms = ms, best = save_choice(c);
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
