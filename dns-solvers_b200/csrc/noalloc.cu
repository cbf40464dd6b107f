// dnslbm_step_f64_noalloc: the FP64 fused step for callers that cannot
// allocate device memory.
//
// Some host codes own every byte of device memory through their own pool or
// arena (for example a solver that reserves the GPU up front and hands
// buffers to several libraries) and do not allow a library to call
// cudaMalloc.  Such a caller already holds the populations in device memory;
// this entry point advances them in place and writes the per-step log
// records into a device buffer the caller provides.  The step kernel's
// scratch (block partial sums, plane sums, ticket counters, the force and
// plane-mean double buffers, the step counter) lives in the file-scope
// array below instead of in allocations.
//
// The array is a fixed 1 MiB of device memory that every GPU which loads the
// library holds until the process exits.  All calls on a device share it and
// it keeps the last call's contents: each call first re-initialises the parts
// that must start from zero, on the caller's stream.  Calls whose work
// overlaps on the GPU (different streams, or different host threads, on the
// same device) race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/dnslbm.h"
#include "step_common.cuh"

namespace dnslbm {
void launch_step_f64(const StepArgs &p, dim3 grid, dim3 block, bool odd, int tex, cudaStream_t s);
void launch_reduce_f64(const StepArgs &p, dim3 grid, dim3 block, cudaStream_t s);
void launch_reduce_f64_odd(const StepArgs &p, dim3 grid, dim3 block, int tex, cudaStream_t s);
}  // namespace dnslbm

using namespace dnslbm;

namespace {

constexpr size_t kScratchDoubles = size_t(1) << 17;  // 1 MiB
static __device__ __align__(256) double g_step_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
double *g_scratch_addr[kMaxDevices];  // device address of g_step_scratch, per device

// Offsets (in doubles) of the pieces of the scratch array for one grid.
struct ScratchLayout {
    size_t force, shift, plane_sums, partials, logs, step_ctr, status, plane_ctr, total_ctr, total;
};

ScratchLayout layout(int nz, size_t nblocks)
{
    ScratchLayout L;
    size_t o = 0;
    L.force = o;       o += 2;
    L.shift = o;       o += (size_t)2 * nz * 3;
    L.plane_sums = o;  o += (size_t)nz * NP;
    L.partials = o;    o += nblocks * NP;
    L.logs = o;        o += 9;           // record slot used when the caller passes no log buffer
    L.step_ctr = o;    o += 1;           // long long
    L.status = o;      o += 2;           // long long[2]
    L.plane_ctr = o;   o += ((size_t)nz + 1) / 2;  // unsigned[nz]
    L.total_ctr = o;   o += 1;           // unsigned
    L.total = o;
    return L;
}

// Everything a call must find at zero (or at the force g) before its first
// step: counters, status, step counter, plane means, force.
__global__ void noalloc_reset_kernel(double *s, ScratchLayout L, int nz, double gx)
{
    const size_t n0 = L.shift, n1 = L.shift + (size_t)2 * nz * 3;
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n1 - n0; i += (size_t)gridDim.x * blockDim.x)
        s[n0 + i] = 0.0;
    for (size_t i = L.step_ctr + threadIdx.x + (size_t)blockIdx.x * blockDim.x; i < L.total;
         i += (size_t)gridDim.x * blockDim.x)
        s[i] = 0.0;  // step counter, status, plane and total tickets (all-zero bit patterns)
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        s[L.force] = gx;
        s[L.force + 1] = gx;
    }
}

int report(char *err, size_t len, int code, const char *msg)
{
    if (err && len) snprintf(err, len, "%s", msg);
    return code;
}

}  // namespace

extern "C" int dnslbm_step_f64_noalloc(double *pop, size_t pop_stride, int xdv, int ydv, int zdv, double omega,
                                       double gx, const uint8_t *wallmask, int parity, long nsteps, double *logs,
                                       void *stream, char *err, size_t err_len)
{
    char msg[256];
    if (!pop) return report(err, err_len, DNSLBM_ERR_ARG, "null population pointer");
    if (((uintptr_t)pop & 7u) != 0) return report(err, err_len, DNSLBM_ERR_ARG, "populations not 8-byte aligned");
    if (xdv < 2 || ydv < 2 || zdv < 3) return report(err, err_len, DNSLBM_ERR_ARG, "grid too small (xdv,ydv >= 2, zdv >= 3)");
    const long long ncell = (long long)xdv * ydv * zdv;
    if (ncell >= (1LL << 31)) return report(err, err_len, DNSLBM_ERR_ARG, "grid exceeds 2^31 cells");
    if (pop_stride < (size_t)ncell) return report(err, err_len, DNSLBM_ERR_ARG, "pop_stride smaller than the cell count");
    if (!(omega > 0.0 && omega < 2.0)) return report(err, err_len, DNSLBM_ERR_ARG, "omega outside (0,2)");
    if (parity != 0 && parity != 1) return report(err, err_len, DNSLBM_ERR_ARG, "parity must be 0 or 1");
    if (nsteps < 0) return report(err, err_len, DNSLBM_ERR_ARG, "negative step count");
    if (nsteps == 0) return DNSLBM_OK;

    // launch shape as the context path; taller blocks when the partial sums
    // would not fit the scratch array
    int bx = ((xdv + 31) / 32) * 32;
    if (bx > 128) bx = 128;
    int rows = 8;
    ScratchLayout L;
    for (;;) {
        const size_t nblocks = (size_t)((xdv + bx - 1) / bx) * ((ydv + rows - 1) / rows) * zdv;
        L = layout(zdv, nblocks);
        if (L.total <= kScratchDoubles || rows >= ydv) break;
        rows *= 2;
    }
    if (L.total > kScratchDoubles) {
        snprintf(msg, sizeof msg,
                 "grid %dx%dx%d needs %zu doubles of step scratch; the static array holds %zu (at most about %zu "
                 "wall-normal planes)",
                 xdv, ydv, zdv, L.total, kScratchDoubles, kScratchDoubles / (size_t)(6 + 2 * NP));
        return report(err, err_len, DNSLBM_ERR_ARG, msg);
    }

    // once per device, with that device current: the array's device address
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return report(err, err_len, DNSLBM_ERR_CUDA, "no usable current CUDA device");
    double *scratch;
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (!g_scratch_addr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_step_scratch);
            if (e != cudaSuccess) {
                snprintf(msg, sizeof msg, "cudaGetSymbolAddress of the step scratch failed: %s", cudaGetErrorString(e));
                return report(err, err_len, DNSLBM_ERR_CUDA, msg);
            }
            g_scratch_addr[dev] = static_cast<double *>(p);
        }
        scratch = g_scratch_addr[dev];
    }

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    StepArgs p;
    for (int a = 0; a < Q; ++a) p.pop[a] = pop + (size_t)a * pop_stride;
    p.nx = xdv;
    p.ny = ydv;
    p.nz = zdv;
    p.pitch = xdv;  // the caller's rows are unpadded
    p.rows = rows;
    p.slots = ((xdv + bx - 1) / bx) * ((ydv + rows - 1) / rows);
    p.wallmask = wallmask;
    p.band_of = nullptr;
    p.links = nullptr;
    p.omega = omega;
    p.ubulk = 0.0;
    p.gx = gx;
    p.const_q = 0;
    p.force = scratch + L.force;
    p.shift = scratch + L.shift;
    p.step_ctr = reinterpret_cast<long long *>(scratch + L.step_ctr);
    p.partials = scratch + L.partials;
    p.plane_sums = scratch + L.plane_sums;
    p.plane_ctr = reinterpret_cast<unsigned *>(scratch + L.plane_ctr);
    p.total_ctr = reinterpret_cast<unsigned *>(scratch + L.total_ctr);
    p.logs = logs ? logs : scratch + L.logs;
    p.log_cap = logs ? (int)(nsteps < 0x7fffffffL ? nsteps : 0x7fffffffL) : 1;
    p.status = reinterpret_cast<long long *>(scratch + L.status);
    p.wait_ns = 1000000000ull;  // the per-thread kernel has no bounded waits
    p.withhold_stage = 0;

    const dim3 block(bx, 1, 1), grid((xdv + bx - 1) / bx, (ydv + rows - 1) / rows, zdv);
    noalloc_reset_kernel<<<64, 256, 0, s>>>(scratch, L, zdv, gx);
    // the plane means of the state the first step starts from (the shift of
    // the one-pass energy sum), as after dnslbm_load_state; a state left by
    // an odd number of steps is read through the odd-step address set
    if (parity == 0) launch_reduce_f64(p, grid, block, s);
    else launch_reduce_f64_odd(p, grid, block, wallmask != nullptr ? 1 : 0, s);
    for (long n = 0; n < nsteps; ++n)
        launch_step_f64(p, grid, block, ((parity + n) & 1) != 0, wallmask != nullptr ? 1 : 0, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(msg, sizeof msg, "step launch failed: %s", cudaGetErrorString(e));
        return report(err, err_len, DNSLBM_ERR_CUDA, msg);
    }
    return DNSLBM_OK;
}
