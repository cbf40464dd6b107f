/*
 * dnslbm -- B200 (sm_100a) D3Q19 BGK channel-flow time step behind a C ABI.
 *
 * Drop-in for the time step of the DNS solver (DNS-solver/src): the state
 * lives in GPU memory for the whole run; the host keeps the reference's
 * parameter deck, wall-flag semantics and file formats.  Every function
 * returns an int status (DNSLBM_OK = 0) and never aborts; the message of the
 * last failure is available from dnslbm_last_error().
 *
 * Axes and sizes follow the reference: x = i streamwise (periodic),
 * y = j spanwise (periodic), z = k wall-normal; xdv, ydv, zdv count fluid
 * cells (walls excluded, definitions.h:32-34); zd = zdv + 2 includes the two
 * wall planes k = 0 and k = zd - 1.
 *
 * Host arrays use the reference's own layouts:
 *   state  double [xdv][ydv][zd][19]   the lbf/ftemp layout without ghosts
 *                                      (dns-const-q-xycut.c:405-416)
 *   flags  int    [xdv+1][ydv+1][zd]   the reference's V.s with ghost planes
 *                                      (solid_init.c:3-8: 0 fluid, 1 periodic,
 *                                      -1 no-slip, -2 slip)
 *   vel    double [xdv][ydv][zd][3], den double [xdv][ydv][zd] (vel_print.c)
 *   stats  double [9][zd]  (statistics.c:139-147 file order)
 *
 * Threading: one host thread per context; each context owns one CUDA stream.
 */
#ifndef DNSLBM_H
#define DNSLBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define DNSLBM_OK 0
#define DNSLBM_ERR_ARG 1      /* bad deck or argument                          */
#define DNSLBM_ERR_CUDA 2     /* a CUDA call failed                            */
#define DNSLBM_ERR_NAN 3      /* NaN wall shear stress (the reference aborts,  */
                              /* wshearstr.c:126-130)                          */
#define DNSLBM_ERR_TIMEOUT 4  /* a bounded device-side wait ran out            */
#define DNSLBM_ERR_NOMEM 5    /* device allocation failed                      */
#define DNSLBM_ERR_IO 6       /* file read/write failed                        */
#define DNSLBM_ERR_STATE 7    /* call out of order (e.g. step before a state)  */

/* storage precision of the populations */
#define DNSLBM_F64 64         /* plain FP64, the reference's arithmetic order  */
#define DNSLBM_F32 32         /* FP32 deviations f - w, FP32 collision         */
#define DNSLBM_F16 16         /* FP16 deviations (scaled by 2^15), FP32 collision */

/* body-force mode */
#define DNSLBM_FORCE_CONST_Q 0 /* V.force = rho_mean*ub - jx_mean every step (encalc.c:121) */
#define DNSLBM_FORCE_CONST_G 1 /* fixed body force gx                              */

/* wall rule for solids inside the flow */
#define DNSLBM_BC_REFERENCE 0 /* exactly xcomputations.c:359-400              */
#define DNSLBM_BC_GENERAL 1   /* + solids inside the flow (riblets, blocks):  */
                              /* bounce-back on every link into a solid cell  */
                              /* and where a specular reflection would land   */
                              /* on one; no counterpart in the reference      */

/* per-step log record: state at the start of each step, in this order */
#define DNSLBM_LOG_FORCE 0    /* force used by the step (V.force)               */
#define DNSLBM_LOG_RHO 1      /* mean density V.rho (encalc.c:62,79)            */
#define DNSLBM_LOG_ENERGY 2   /* K (encalc.c:106-114) -> energy.txt             */
#define DNSLBM_LOG_FLOWRATE 3 /* U*(ydv*zdv) (encalc.c:132) -> flowrate.txt     */
#define DNSLBM_LOG_MASSRATE 4 /* mean jx*(ydv*zdv) (encalc.c:136) -> massrate.txt */
#define DNSLBM_LOG_STUP 5     /* wshearstr.c:72-123 -> str-up.txt               */
#define DNSLBM_LOG_STDOWN 6   /* wshearstr.c:26-70 -> str-do.txt                */
#define DNSLBM_LOG_STRESS 7   /* wshearstr.c:125 -> w-str.txt                   */
#define DNSLBM_LOG_PGRAD 8    /* wshearstr.c:119-121 -> p-grad.txt              */
#define DNSLBM_LOG_N 9

/* The parameter deck.  Replaces the compile-time #defines of
 * definitions.h:30-59 (Rebs, ub, zdv, ydv, xdv) and the derived omega of
 * dns-const-q-xycut.c:216-217, read at run time. */
typedef struct dnslbm_deck {
    int xdv, ydv, zdv;  /* fluid cells (xdv, ydv >= 2; zdv >= 3)                 */
    double omega;       /* relaxation rate 1/tau (the reference's `tau` variable) */
    double ubulk;       /* target bulk velocity (constant-Q)                     */
    double gx;          /* body force (constant-g)                               */
    int force_mode;     /* DNSLBM_FORCE_*                                        */
    int precision;      /* DNSLBM_F64 | DNSLBM_F32 | DNSLBM_F16                  */
    int bc_mode;        /* DNSLBM_BC_*                                           */
    int log_capacity;   /* per-step records kept on the device (0 -> 4096)       */
    int device;         /* CUDA device ordinal                                   */
} dnslbm_deck;

typedef struct dnslbm_ctx dnslbm_ctx;

/* Allocate a device context for the deck.  Replaces the calloc block of
 * dns-const-q-xycut.c:239-356 and the halo request set-up of :363-376 (the
 * halo exchange is an in-kernel periodic wrap here).  Flags default to
 * solid_init (smooth no-slip walls). */
int dnslbm_create(const dnslbm_deck *deck, dnslbm_ctx **out);
void dnslbm_destroy(dnslbm_ctx *ctx);
/* message of the last failure of this context (ctx NULL: of the last failed
 * dnslbm_create on this thread) */
const char *dnslbm_last_error(const dnslbm_ctx *ctx);

/* Wall flags in the reference's V.s layout with ghost planes.  Replaces
 * solid_init.c:10-46, slip_ridges_init.c:3-43 and slip_posts_init.c:3-74 as
 * inputs to the step; the ghost planes are ignored (the grid is periodic). */
int dnslbm_set_flags(dnslbm_ctx *ctx, const int *s);
/* The same on the ghost-free periodic grid: int8 [xdv][ydv][zd].  With
 * DNSLBM_BC_GENERAL a cell inside the flow may be solid (-1); solid cells
 * hold the rest state f = w (a loaded state is overwritten there) and enter
 * the plane sums like any other cell.  Wall planes are -1 or -2 in either
 * mode; flags change only between even numbers of steps. */
int dnslbm_set_flags_periodic(dnslbm_ctx *ctx, const int8_t *flags);
/* Host only (no device is touched): the per-cell link masks that
 * dnslbm_set_flags_periodic builds from `flags` for boundary mode
 * `bc_mode`: band_of[zdv] gets each fluid plane's mask block (-1: none),
 * links[nband][ydv][xdv] the masks (bit 0 solid, bit A: link A bounces
 * back), nband the number of blocks.  A diagnostic of the wall rule; no
 * counterpart in the reference.  DNSLBM_ERR_ARG for invalid flags or a
 * links_capacity (entries) below nband * ydv * xdv. */
int dnslbm_link_masks(int xdv, int ydv, int zdv, int bc_mode, const int8_t *flags, int *band_of, unsigned *links,
                      size_t links_capacity, int *nband);

/* Initial state: rest, f = w (init.c:6-19). */
int dnslbm_init_rest(dnslbm_ctx *ctx);
/* Load / store the state in the lbf ftemp layout (dns-const-q-xycut.c:405-416
 * read, :494-497 write).  Wall-plane entries are ignored on load and written
 * as zeros on store.  Loading resets the step counter. */
int dnslbm_load_state(dnslbm_ctx *ctx, const double *state);
/* The same in x-slabs, like the reference's per-rank read of its x-range of
 * the lbf file (dns-const-q-xycut.c:405-416): `slab` holds x in [x0, x0+nxs)
 * in the lbf layout (nxs * ydv * zd * 19 doubles).  Slabs come in order of
 * x; x0 = 0 starts a new state (and resets the step counter), the slab that
 * ends at xdv completes it.  Until then the context holds no state. */
int dnslbm_load_state_slab(dnslbm_ctx *ctx, int x0, int nxs, const double *slab);
int dnslbm_store_state(dnslbm_ctx *ctx, double *state);

/* Advance nsteps time steps on the device.  Each step is the reference's loop
 * body (dns-const-q-xycut.c:487-518): the encalc/wshearstr reductions of the
 * state (logged), then collide + stream + wall rules + periodic wrap
 * (xcomputations.c:5-562).  Returns DNSLBM_ERR_NAN if any step saw a NaN wall
 * stress. */
int dnslbm_step(dnslbm_ctx *ctx, long nsteps);
/* Steps done since the last load/init. */
long dnslbm_steps_done(const dnslbm_ctx *ctx);
/* Copy the log records of steps [first, first+count) (count*DNSLBM_LOG_N
 * doubles); only the last log_capacity steps are kept. */
int dnslbm_logs(dnslbm_ctx *ctx, long first, long count, double *out);
/* Force the next step will use (V.force). */
int dnslbm_get_force(dnslbm_ctx *ctx, double *force);

/* ---- A channel split over several GPUs: wall-normal slabs ----
 * Replaces the reference's domain decomposition (the MPI cartesian grid of
 * dns-const-q-xycut.c:63-125) and its halo exchange (the persistent
 * requests of :363-376 started in xcomputations.c:222-289,435-555) for a
 * decomposition across the wall-normal planes: a slab holds whole planes,
 * which are contiguous in each population array, so its halo is five whole
 * planes per face and its plane statistics stay its own.  One context per
 * GPU (one process per GPU); the exchange is the caller's (NCCL, CUDA-aware
 * MPI, device copies) through the pointers below, on the context's stream.
 *
 * dnslbm_create_slab: fluid planes [z0, z0+nzs) (nzs >= 2) of the channel
 * `deck` describes (deck->zdv planes), the reference boundary mode only.
 * Flags (dnslbm_set_flags / _periodic) are the whole channel's; states
 * (dnslbm_load_state / dnslbm_store_state and the other readers) are the
 * slab's planes in the lbf layout with zd = nzs + 2 (planes k = z0 .. z0 +
 * nzs + 1 of the whole lbf, the first and last ignored on load), read only
 * after an even number of steps.  dnslbm_step refuses a slab; per step:
 *   1. before an odd step (dnslbm_steps_done odd): every slab fills its
 *      ghost planes from its neighbours (ghost <- neighbour's edge);
 *   2. dnslbm_slab_step: the step kernel; it leaves the slab's plane sums
 *      (nzs * DNSLBM_SUM_N doubles, dnslbm_slab_sums) on the device;
 *   3. after an odd step: every slab sends its ghost planes back
 *      (neighbour's edge <- ghost);
 *   4. the caller gathers all slabs' sums in plane order (deck->zdv *
 *      DNSLBM_SUM_N doubles in device memory) and calls dnslbm_slab_tail:
 *      logs, constant-Q force and plane means of the whole channel, the same
 *      on every slab.  A load or dnslbm_init_rest also owes one
 *      dnslbm_slab_tail (steps 2 and 4 without the step).
 * With constant g the populations are bit-identical to the whole channel
 * stepped by one context.  No call of the sequence synchronises the host;
 * dnslbm_slab_status waits for the stream and reports NaN / timeouts. */
#define DNSLBM_SUM_N 8
int dnslbm_create_slab(const dnslbm_deck *deck, int z0, int nzs, dnslbm_ctx **out);
int dnslbm_slab_step(dnslbm_ctx *ctx);
int dnslbm_slab_sums(dnslbm_ctx *ctx, double **sums);
int dnslbm_slab_tail(dnslbm_ctx *ctx, const double *sums_all);
int dnslbm_slab_status(dnslbm_ctx *ctx);
/* Device pointers of the five population planes exchanged across the lower
 * (side 0) or upper (side 1) face, in a fixed direction order: ghost[i] of
 * the ghost plane beyond the face, edge[i] of the slab's own plane at the
 * face; *bytes per plane.  Pairing: a slab's ghost on side s mirrors its
 * neighbour's edge on side 1-s, entry for entry.  DNSLBM_ERR_ARG on a face
 * next to a wall. */
int dnslbm_slab_halo(dnslbm_ctx *ctx, int side, void **ghost, void **edge, size_t *bytes);
/* The context's CUDA stream (a cudaStream_t): every call of the context is
 * ordered on it. */
void *dnslbm_stream(const dnslbm_ctx *ctx);

/* statistics.c:3-183 of the current state: out[9*zd]. */
int dnslbm_statistics(dnslbm_ctx *ctx, double *out);
/* Time averages of the plane statistics kept on the device: each
 * dnslbm_stats_accumulate adds a sample of the current state (the rows of
 * dnslbm_statistics) to FP64 running sums without a copy to the host;
 * dnslbm_stats_average returns the averages in the turb-fld layout
 * (9 * zd doubles, wall entries 0): means averaged, rms values pooled as
 * the root of the mean square, as the reference's post-processing averages
 * turb-fld files over a window (TKE-budget/postprocessing/time_stats.c).
 * dnslbm_stats_reset starts a new window (dnslbm_create starts one). */
int dnslbm_stats_accumulate(dnslbm_ctx *ctx);
int dnslbm_stats_average(dnslbm_ctx *ctx, double *out, long *nsamples);
int dnslbm_stats_reset(dnslbm_ctx *ctx);
/* vel_print.c:65-99 of the current state (either pointer may be NULL). */
int dnslbm_moments(dnslbm_ctx *ctx, double *vel, double *den);

/* Output without stopping the time loop (the output cadence of
 * dns-const-q-xycut.c:489-516).  dnslbm_output_begin queues, on the
 * context's stream ahead of any later step, the kernels that compute the
 * requested outputs of the current state into device buffers -- the state
 * as dnslbm_store_state writes it, vel/den as dnslbm_moments, the turb-fld
 * rows as dnslbm_statistics -- and their copies into the caller's host
 * buffers on a second stream, and returns at once: steps called after it
 * run while the copies drain.  Any pointer may be NULL.  Host buffers should
 * be page-locked (dnslbm_host_alloc) so that the copies overlap the steps;
 * they must not be read or reused until dnslbm_output_wait returns.  Device
 * buffers are allocated by the first call that needs them
 * (DNSLBM_ERR_NOMEM if they do not fit) and kept; a new begin waits, on the
 * device, for the previous copies. */
int dnslbm_output_begin(dnslbm_ctx *ctx, double *state, double *vel, double *den, double *stats);
/* Block until the copies of the last dnslbm_output_begin have landed. */
int dnslbm_output_wait(dnslbm_ctx *ctx);

/* Quadrant analysis of the current state, on the GPU
 * (quadrant-analysis/src/qUADrantA.c): per wall-normal plane, the
 * fluctuations u' = u - <u>, w' = w - <w> of the cell velocities (those
 * dnslbm_moments returns) split into the quadrants Q1 (u'>0, w'>0),
 * Q2 (u'<0, w'>0), Q3 (u'<0, w'<0), Q4 (u'>0, w'<0):
 *   quadrant[4][zd]   the conditional mean of u'w' in each quadrant,
 *   dquadrant[4][zd]  each quadrant's contribution (its sum / cells of the plane),
 *   uw[zd]            the plane mean of u'w',
 * wall planes 0 -- the reference's quadrant.000.TTTT file holds quadrant
 * then uw, dquadrant.000.TTTT dquadrant then uw.  Any pointer may be NULL. */
int dnslbm_quadrant(dnslbm_ctx *ctx, double *quadrant, double *dquadrant, double *uw);
/* The same for a velocity field read from a vel.NNNN file
 * ([xdv][ydv][zdv+2][3] doubles), on CUDA device `device` (temporary device
 * memory, freed before return; errors in dnslbm_last_error(NULL)). */
int dnslbm_quadrant_vel(const double *vel, int xdv, int ydv, int zdv, int device, double *quadrant, double *dquadrant,
                        double *uw);

/* Two-point velocity correlations of the current state, on the GPU
 * (2pt-correlations/src/correlations.c: mean_subtract.c, xcorrel.c,
 * ycorrel.c), from the cell velocities dnslbm_moments returns:
 *   uavg[zd]          the subtracted mean of each plane: the plane mean of u
 *                     over (x, y), made symmetric about the channel centre
 *                     (u, v even, w odd); 0 on the wall planes, which keep
 *                     their velocities (mean_subtract.c writes it to uavg.TTT);
 *   xcorl[zd][xdv][3] per plane and component, the sum over (x, y) of
 *                     u'(x, y) u'(x + d, y), d = 0 .. xdv-1 periodic
 *                     (the program's xcorl.TTTT file);
 *   ycorl[zd][ydv][3] the same along y (ycorl.TTTT).
 * The sums are unnormalised, as the program writes them.  mean_subtract.c
 * averages over the period of a stripe texture given at compile time; its
 * shipped setting (no period) cannot run, and the plane mean here is its
 * value for any period that divides the span.  Lines up to 2048 cells;
 * temporary device memory of about 2.1 times the velocity field.  Any
 * pointer may be NULL. */
int dnslbm_correlations(dnslbm_ctx *ctx, double *xcorl, double *ycorl, double *uavg);
/* The same for a velocity field read from a vel.NNNN file
 * ([xdv][ydv][zdv+2][3] doubles), on CUDA device `device`. */
int dnslbm_correlations_vel(const double *vel, int xdv, int ydv, int zdv, int device, double *xcorl, double *ycorl,
                            double *uavg);

/* One-dimensional energy spectra of the current state, on the GPU
 * (e-spectra/src/1d-spectra.c): per fluid plane, the 2-D DFT of u, v, w
 * over (x, y) scaled by 1/(xdv ydv) with the mean mode removed, and
 * 0.5 |C|^2 summed over the half spectrum in y (modes j > 0 twice) into
 *   ex[3][xdv][zd]       Euux, Evvx, Ewwx (per streamwise mode i),
 *   ey[3][ydv/2+1][zd]   Euuy, Evvy, Ewwy (per spanwise mode j),
 * the program's file layouts ([mode][zd] per component, wall planes 0).  The
 * transforms are evaluated directly in FP64 (the program calls FFTW), to
 * rounding of the DFT.  Either pointer may be NULL. */
int dnslbm_spectra(dnslbm_ctx *ctx, double *ex, double *ey);
/* The same for a velocity field read from a vel.NNNN file
 * ([xdv][ydv][zdv+2][3] doubles), on CUDA device `device`. */
int dnslbm_spectra_vel(const double *vel, int xdv, int ydv, int zdv, int device, double *ex, double *ey);

/* Timing support for benchmarks: advance nsteps like dnslbm_step and return
 * CUDA-event times on the context's stream: total, and the summed device
 * time of the two step kernels (even / odd parity launches).  With ms_even
 * and ms_odd both NULL only the total is taken (no event between launches,
 * which lets each launch overlap the end of the previous one). */
int dnslbm_step_timed(dnslbm_ctx *ctx, long nsteps, double *ms_total, double *ms_even, double *ms_odd);
/* Autotuner: choose the step kernel's launch shape (per-thread kernel, or the
 * row-pipelined kernel's rows per stage group, stages in flight and consumer
 * warps) by timing each candidate for `steps` steps on this context's own grid
 * and precision, and keep the fastest.  Call it after dnslbm_create and before
 * a state is set: it steps a rest state and leaves the context without one.
 * report (may be NULL) receives the choice and its time.  No counterpart in
 * the reference, whose loop tiling is the compile-time constant cs
 * (definitions.h:117). */
int dnslbm_autotune(dnslbm_ctx *ctx, int steps, char *report, size_t report_len);

/* Limit of each bounded device-side wait of the row-pipelined step kernel
 * (its consumers waiting for a bulk copy to land, its producer waiting for
 * them to release a stage), in milliseconds of the GPU's global timer;
 * default 1000.  A wait that runs out ends that block's part of the step
 * early (no copy left in flight) and the step call returns
 * DNSLBM_ERR_TIMEOUT; the state is then invalid until the next load.  No
 * counterpart in the reference, whose MPI waits are unbounded
 * (xcomputations.c:435-555). */
int dnslbm_set_wait_limit(dnslbm_ctx *ctx, double ms);
/* Test hook for the bounded waits (no counterpart in the reference): the
 * next launch of the row-pipelined kernel has its first block withhold the
 * load of its first row group, so that block's consumers wait for data that
 * never comes, give up after the wait limit, and the step call returns
 * DNSLBM_ERR_TIMEOUT.  Nothing faults and no copy is left in flight.
 * DNSLBM_ERR_STATE when the context steps with the per-thread kernel. */
int dnslbm_test_withhold_load(dnslbm_ctx *ctx);

/* Name of the step kernel this context launches ("row-pipelined bulk-copy"
 * or "per-thread"), with its launch shape. */
const char *dnslbm_step_kernel(const dnslbm_ctx *ctx);
/* Populations bytes moved per fluid cell per step (2*19*storage bytes). */
double dnslbm_bytes_per_cell(const dnslbm_ctx *ctx);
/* Block until all work of the context is done. */
int dnslbm_sync(dnslbm_ctx *ctx);

/* Page-locked host memory for state buffers (faster load/store); NULL on
 * failure.  Replaces nothing in the reference (its arrays are calloc'ed,
 * dns-const-q-xycut.c:248-262). */
void *dnslbm_host_alloc(size_t bytes);
void dnslbm_host_free(void *ptr);

/* Batched channels: many independent channels (own grid, walls, force,
 * state and logs) advanced together by one persistent kernel: one
 * cooperative launch runs a chunk of 32 steps (the time loop, replayed from
 * a CUDA graph), its blocks taking items of work -- runs of row groups, and
 * the cells of planes next to solids -- from a per-step counter, largest
 * first, with a bounded grid-wide barrier between steps.  All decks share
 * one precision and device.  Use dnslbm_batch_channel(b, i) with the
 * single-channel calls (flags, load/store, logs, statistics) between batch
 * steps.  The environment variable DNSLBM_BATCH=launch selects one launch
 * per step instead.  No counterpart in the reference (one channel per run). */
typedef struct dnslbm_batch dnslbm_batch;
int dnslbm_batch_create(const dnslbm_deck *decks, int n, dnslbm_batch **out);
void dnslbm_batch_destroy(dnslbm_batch *b);
const char *dnslbm_batch_last_error(const dnslbm_batch *b);
int dnslbm_batch_size(const dnslbm_batch *b);
dnslbm_ctx *dnslbm_batch_channel(dnslbm_batch *b, int i);
/* Advance every channel nsteps steps (all channels must hold a state and be
 * at the same step). */
int dnslbm_batch_step(dnslbm_batch *b, long nsteps);
/* The same, returning the device time of the whole batch in ms. */
int dnslbm_batch_step_timed(dnslbm_batch *b, long nsteps, double *ms);
/* Test hook for the persistent kernel's bounded waits (no counterpart in
 * the reference): the next dnslbm_batch_step has its first block withhold
 * its first load, with waits limited to wait_ms; the call returns
 * DNSLBM_ERR_TIMEOUT and the channels need a new state.  DNSLBM_ERR_STATE
 * when the batch steps with one launch per step. */
int dnslbm_batch_test_withhold_load(dnslbm_batch *b, double wait_ms);
/* Launch shape of the batched kernel. */
const char *dnslbm_batch_kernel(const dnslbm_batch *b);
/* Time the batched kernel's launch shapes (shared-memory budget for 1-3
 * blocks per SM x 2-4 stages x consumer threads) on rest states of all
 * channels, `steps` steps each, and keep the fastest.  Runs before any state
 * is loaded (DNSLBM_ERR_STATE otherwise); leaves the channels without state.
 * `report` (may be NULL) receives the choice. */
int dnslbm_batch_autotune(dnslbm_batch *b, int steps, char *report, size_t report_len);

/* FP64 constant-g step that allocates nothing.  No counterpart in the
 * reference: it is for callers that own all device memory through their own
 * pool or arena and do not let a library call cudaMalloc.  The caller passes
 * its populations in device memory -- 19 arrays of doubles, array a at
 * pop + a*pop_stride, each holding cell (x, y, z) at (z*ydv + y)*xdv + x,
 * z = 0..zdv-1 -- and they are advanced nsteps steps in place (the AA scheme
 * of dnslbm_step).  parity is 0 when the populations are in this natural
 * layout and 1 after an odd number of steps; it becomes (parity + nsteps) % 2.
 * wallmask (device, may be NULL for smooth no-slip walls) holds per
 * wall-adjacent cell, bottom plane then top plane, [2][ydv][xdv] bytes whose
 * bits 0..4 mark the links with in-plane offsets (0,0) (1,0) (-1,0) (0,1)
 * (0,-1) that bounce back (1) rather than reflect specularly (0).  logs
 * (device, may be NULL) receives nsteps records of DNSLBM_LOG_N doubles.
 * Work is queued on `stream` (NULL: the default stream) and the call returns
 * without waiting; a NaN wall stress shows as NaN in the log records.
 * Scratch lives in a fixed 1 MiB device array that every GPU loading the
 * library holds until exit; a grid needs about 15 + 8*ceil(xdv/128) doubles
 * of it per wall-normal plane (about 2400 planes at xdv = 628), and grids
 * whose scratch does not fit are rejected with DNSLBM_ERR_ARG.
 * All calls on a device share that array: calls that overlap on the GPU race.
 * The first call on each device (made with the device that holds pop
 * current) looks up the array's device address; make it before any stream
 * capture.  err (may be NULL) receives a message on failure. */
int dnslbm_step_f64_noalloc(double *pop, size_t pop_stride, int xdv, int ydv, int zdv, double omega, double gx,
                            const uint8_t *wallmask, int parity, long nsteps, double *logs, void *stream, char *err,
                            size_t err_len);

#ifdef __cplusplus
}
#endif
#endif
