/*
 * CPU oracle for the D3Q19 BGK channel step -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64 restatement of the reference's time step and its per-step
 * reductions, on a periodic (ghost-free) grid.  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg may load it; the product library never
 * links it.  Each function cites the reference file:line it restates.
 *
 * Grid and layout (the reference's lbf/ftemp layout without ghost planes):
 *   state[((x*ny + y)*zd + z)*19 + a],  x in [0,nx) streamwise (periodic),
 *   y in [0,ny) spanwise (periodic), z in [0,zd) wall-normal, zd = nz+2 with
 *   z=0 and z=zd-1 the wall planes.  Wall-plane entries are never read.
 *   flags[(x*ny + y)*zd + z]: 0 fluid, -1 no-slip solid, -2 slip solid
 *   (DNS-solver/src/solid_init.c:3-8 semantics; no "periodic" value 1 since
 *   there are no ghost planes).
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* per-step log record, one per time step, state at the START of the step */
enum {
    ORC_LOG_FORCE = 0,   /* body force used by this step (V.force)            */
    ORC_LOG_RHO,         /* mean density (V.rho), encalc.c:62,79              */
    ORC_LOG_ENERGY,      /* K, encalc.c:106-114 (energy.txt)                  */
    ORC_LOG_FLOWRATE,    /* U*(ny*nz), encalc.c:116-119,132 (flowrate.txt)    */
    ORC_LOG_MASSRATE,    /* momentum*(ny*nz), encalc.c:136 (massrate.txt)     */
    ORC_LOG_STUP,        /* wshearstr.c:72-123 (str-up.txt)                   */
    ORC_LOG_STDOWN,      /* wshearstr.c:26-70 (str-do.txt)                    */
    ORC_LOG_STRESS,      /* wshearstr.c:125 (w-str.txt)                       */
    ORC_LOG_PGRAD,       /* wshearstr.c:119-121 (p-grad.txt)                  */
    ORC_LOG_N
};

/* bc_mode: 0 = the reference rule exactly (a link into a no-slip cell whose
 * wall-normal neighbour is fluid writes nothing, xcomputations.c:368-375);
 * 1 = generalised: such links (solids inside the flow, e.g. riblets) bounce
 * back, and a specular reflection whose target is solid bounces back. */
int orc_step(int nx, int ny, int nz, double *state, double *scratch, const int8_t *flags,
             double omega, double force, int bc_mode);

/* nsteps steps at a fixed force without the per-step reductions (the
 * two-buffer swap of xcomputations.c:557-559); result in `state`. */
int orc_steps(int nx, int ny, int nz, double *state, double *scratch, const int8_t *flags, double omega,
              double force, int bc_mode, long nsteps);

/* encalc.c:3-146 restated; returns force = rho*ubulk - momentum and fills
 * out[ORC_LOG_RHO..ORC_LOG_MASSRATE]. */
double orc_encalc(int nx, int ny, int nz, const double *state, double ubulk, double *out);

/* wshearstr.c:3-156 restated; fills out[ORC_LOG_STUP..ORC_LOG_PGRAD].
 * Returns 1 if the stress is NaN (the reference aborts there). */
int orc_wshearstr(int nx, int ny, int nz, const double *state, double omega, double force, double *out);

/* statistics.c:31-132 restated: out[9*zd] in the turb-fld file order
 * UAVG,VAVG,WAVG,UTIN,VTIN,WTIN,REYS,DAVG,DTIN (statistics.c:139-147). */
void orc_statistics(int nx, int ny, int nz, const double *state, double *out);

/* vel_print.c:65-99 restated: vel[nx][ny][zd][3], den[nx][ny][zd]. */
void orc_moments(int nx, int ny, int nz, const double *state, double *vel, double *den);

/* The reference time loop (dns-const-q-xycut.c:485-519) without file I/O:
 * per step encalc -> wshearstr -> step.  const_g != 0 replaces the encalc
 * force by gx.  logs[nsteps][ORC_LOG_N] (may be NULL).  Returns the number of
 * steps done (stops early on a NaN wall stress). */
long orc_run(int nx, int ny, int nz, double *state, const int8_t *flags, double omega,
             double ubulk, double gx, int const_g, long nsteps, double *logs, int bc_mode);

/* Flag builders on the periodic grid (flags must be nx*ny*zd). */
void orc_flags_smooth(int nx, int ny, int nz, int8_t *flags);
/* slip_ridges_init.c:11-40 with its hard-coded gap/width as parameters:
 * streamwise stripes of `gap` slip cells, then `width` no-slip, first stripe
 * at y = width/2, on both walls. */
void orc_flags_ridges(int nx, int ny, int nz, int gap, int width, int8_t *flags);
/* the same rule rotated: spanwise stripes (transverse grooves) */
void orc_flags_transverse(int nx, int ny, int nz, int gap, int width, int8_t *flags);
/* slip_posts_init.c:14-70 parameterised: gx x gy slip squares, periods
 * gx+wx and gy+wy, first square at (1,1), both walls. */
void orc_flags_posts(int nx, int ny, int nz, int gx, int wx, int gy, int wy, int8_t *flags);

#ifdef __cplusplus
}
#endif
#endif
