/*
 * CPU oracle for the D3Q19 BGK channel step -- TEST INFRASTRUCTURE ONLY.
 * See lbm_oracle.h.  Every floating-point expression below keeps the
 * reference's operand order (and is compiled with -ffp-contract=off), so on
 * grids the reference can express this file reproduces it bit for bit.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* D3Q19 lattice, DNS-solver/src/globals.c:3-13 (same velocity numbering, so
 * that states and flags are interchangeable with the reference's). */
static const double W[19] = {1. / 3., 1. / 18., 1. / 18., 1. / 18., 1. / 18., 1. / 18., 1. / 18.,
                             1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36.,
                             1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36.};
static const int EX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, 1, -1, -1, 0, 0, 0, 0};
static const int EY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, 1, -1, -1};
static const int EZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const int OPP[19] = {0, 2, 1, 4, 3, 6, 5, 9, 10, 7, 8, 13, 14, 11, 12, 17, 18, 15, 16};
static const int MIR[19] = {0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 12, 11, 14, 13, 16, 15, 18, 17};

#define IDX(x, y, z) (((size_t)(x) * ny + (y)) * zd + (z))

/* Moments of one cell, xcomputations.c:314-326 / encalc.c:35-42 order. */
static inline void moments(const double *f, double *dens, double *ux, double *uy, double *uz)
{
    double d = 0., x = 0., y = 0., z = 0.;
    for (int a = 0; a < 19; a++) {
        x += (double)EX[a] * f[a];
        y += (double)EY[a] * f[a];
        z += (double)EZ[a] * f[a];
        d += f[a];
    }
    *dens = d; *ux = x; *uy = y; *uz = z;
}

/* BGK collision with the reference's forcing term, in place on f[19]:
 * xcomputations.c:314-342 (Fi without a rho factor and without a (1-omega/2)
 * prefactor; velocity not shifted by half the force). */
static inline void collide(double *f, double omega, double Gx)
{
    double dens, ux, uy, uz, ueq[3], v, u, feq, Fi;
    moments(f, &dens, &ux, &uy, &uz);
    ueq[0] = ux / dens;
    ueq[1] = uy / dens;
    ueq[2] = uz / dens;
    v = ueq[0] * ueq[0] + ueq[1] * ueq[1] + ueq[2] * ueq[2];
    for (int a = 0; a < 19; a++) {
        u = (double)EX[a] * ueq[0] + (double)EY[a] * ueq[1] + (double)EZ[a] * ueq[2];
        feq = W[a] * dens * (1. + 3. * u + 4.5 * u * u - 1.5 * v);
        Fi = W[a] * (3. * ((double)EX[a] - ueq[0]) + 9. * u * (double)EX[a]) * Gx;
        f[a] += (Fi - omega * (f[a] - feq));
    }
}

/* one step from `src` (collided) streamed into `dst` */
static void orc_step_ab(int nx, int ny, int nz, const double *src, double *dst, const int8_t *flags,
                        double omega, double force, int bc_mode)
{
    const int zd = nz + 2;
    /* Each fluid destination slot has exactly one writer (a permutation), so
     * the sweep over source cells is race-free when split over x. */
#pragma omp parallel for schedule(static)
    for (int x = 0; x < nx; x++) {
        double f[19];
        for (int y = 0; y < ny; y++) {
            for (int z = 1; z < zd - 1; z++) {
                if (flags[IDX(x, y, z)] != 0) continue;
                memcpy(f, src + IDX(x, y, z) * 19, sizeof f);
                collide(f, omega, force);
                /* streaming + wall rules, xcomputations.c:359-376 */
                for (int a = 0; a < 19; a++) {
                    int xt = x + EX[a], yt = y + EY[a], zt = z + EZ[a];
                    xt = xt < 0 ? nx - 1 : (xt >= nx ? 0 : xt);
                    yt = yt < 0 ? ny - 1 : (yt >= ny ? 0 : yt);
                    int sld = flags[IDX(xt, yt, zt)];
                    int sld1 = flags[IDX(x, y, zt)];
                    if (sld > -1) {
                        dst[IDX(xt, yt, zt) * 19 + a] = f[a];
                    } else if (sld == -1 && sld1 == -1) {
                        dst[IDX(x, y, z) * 19 + OPP[a]] = f[a];
                    } else if ((sld == -1 && sld1 == -2) || sld == -2) {
                        if (bc_mode == 1 && flags[IDX(xt, yt, z)] != 0)
                            dst[IDX(x, y, z) * 19 + OPP[a]] = f[a];
                        else
                            dst[IDX(xt, yt, z) * 19 + MIR[a]] = f[a];
                    } else if (bc_mode == 1) {
                        /* solid inside the flow: halfway bounce-back */
                        dst[IDX(x, y, z) * 19 + OPP[a]] = f[a];
                    }
                }
            }
        }
    }
}

int orc_step(int nx, int ny, int nz, double *state, double *scratch, const int8_t *flags,
             double omega, double force, int bc_mode)
{
    /* the reference swaps f/ftemp (xcomputations.c:557-559); copy back so the
     * caller's buffer is the new state.  `scratch` must hold the previous
     * contents of the destination (a copy of state is fine). */
    orc_step_ab(nx, ny, nz, state, scratch, flags, omega, force, bc_mode);
    memcpy(state, scratch, (size_t)nx * ny * (nz + 2) * 19 * sizeof(double));
    return 0;
}

int orc_steps(int nx, int ny, int nz, double *state, double *scratch, const int8_t *flags, double omega,
              double force, int bc_mode, long nsteps)
{
    /* alternate the two buffers (the reference's f/ftemp swap) and leave the
     * result in `state` */
    const size_t n = (size_t)nx * ny * (nz + 2) * 19;
    double *a = state, *b = scratch;
    memcpy(b, a, n * sizeof(double));
    for (long s = 0; s < nsteps; s++) {
        orc_step_ab(nx, ny, nz, a, b, flags, omega, force, bc_mode);
        double *t = a; a = b; b = t;
    }
    if (a != state) memcpy(state, a, n * sizeof(double));
    return 0;
}

double orc_encalc(int nx, int ny, int nz, const double *state, double ubulk, double *out)
{
    const int zd = nz + 2;
    double *uavg = calloc(zd, sizeof(double)), *vavg = calloc(zd, sizeof(double));
    double *wavg = calloc(zd, sizeof(double));
    double momentum = 0., denst = 0., K = 0., U = 0.;
    double dens, ux, uy, uz;
    /* first pass, encalc.c:29-53 */
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 1; k < zd - 1; k++) {
                moments(state + IDX(i, j, k) * 19, &dens, &ux, &uy, &uz);
                momentum += ux;
                ux /= dens;
                uy /= dens;
                uz /= dens;
                denst += dens;
                uavg[k] += ux;
                vavg[k] += uy;
                wavg[k] += uz;
            }
    /* encalc.c:54-62 */
    for (int k = 0; k < zd; k++) {
        uavg[k] /= ((double)(nx * ny));
        vavg[k] /= ((double)(nx * ny));
        wavg[k] /= ((double)(nx * ny));
    }
    momentum /= ((double)((long)nx * ny * (zd - 2)));
    denst /= ((double)((long)nx * ny * (zd - 2)));
    /* second pass, encalc.c:84-111 */
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 1; k < zd - 1; k++) {
                moments(state + IDX(i, j, k) * 19, &dens, &ux, &uy, &uz);
                ux /= dens;
                uy /= dens;
                uz /= dens;
                double uf = ux - uavg[k], vf = uy - vavg[k], wf = uz - wavg[k];
                K += 0.5 * (uf * uf + vf * vf + wf * wf);
            }
    K /= ((double)((long)nx * ny * (zd - 2)));
    for (int k = 0; k < zd; k++) U += uavg[k];
    U /= ((double)(zd - 2));
    double force = denst * ubulk - momentum; /* encalc.c:121 */
    if (out) {
        out[ORC_LOG_RHO] = denst;
        out[ORC_LOG_ENERGY] = K;
        out[ORC_LOG_FLOWRATE] = U * (ny * (zd - 2));
        out[ORC_LOG_MASSRATE] = momentum * ((double)(ny * (zd - 2)));
    }
    free(uavg); free(vavg); free(wavg);
    return force;
}

int orc_wshearstr(int nx, int ny, int nz, const double *state, double omega, double force, double *out)
{
    const int zd = nz + 2;
    double mu = (1. / 6.) * (2. / omega - 1); /* wshearstr.c:24 */
    double stdown = 0., stup = 0., davg = 0.;
    double dens, ux, uy, uz, ux1, ux2, ux3;
    /* bottom wall, wshearstr.c:26-59 */
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            moments(state + IDX(i, j, 1) * 19, &dens, &ux, &uy, &uz);
            ux1 = ux / dens;
            davg += dens;
            moments(state + IDX(i, j, 2) * 19, &dens, &ux, &uy, &uz);
            ux2 = ux / dens;
            moments(state + IDX(i, j, 3) * 19, &dens, &ux, &uy, &uz);
            ux3 = ux / dens;
            stdown += (-2. * ux1 + 3. * ux2 - ux3);
        }
    davg /= ((double)(nx * ny));
    stdown /= ((double)(nx * ny));
    stdown *= mu * davg;
    /* top wall, wshearstr.c:72-107; the density averaged is that of plane
     * zd-4, the last one whose moments were taken (wshearstr.c:105) */
    davg = 0.;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            moments(state + IDX(i, j, zd - 2) * 19, &dens, &ux, &uy, &uz);
            ux1 = ux / dens;
            moments(state + IDX(i, j, zd - 3) * 19, &dens, &ux, &uy, &uz);
            ux2 = ux / dens;
            moments(state + IDX(i, j, zd - 4) * 19, &dens, &ux, &uy, &uz);
            ux3 = ux / dens;
            stup += -(2. * ux1 - 3. * ux2 + ux3);
            davg += dens;
        }
    davg /= ((double)(nx * ny));
    stup /= ((double)(nx * ny));
    double pgrad = force * (zd - 2) / 2.; /* wshearstr.c:119-121 */
    stup *= mu * davg;
    double stress = 0.5 * (stup + stdown);
    if (out) {
        out[ORC_LOG_STUP] = stup;
        out[ORC_LOG_STDOWN] = stdown;
        out[ORC_LOG_STRESS] = stress;
        out[ORC_LOG_PGRAD] = pgrad;
    }
    return isnan(stress) ? 1 : 0;
}

void orc_statistics(int nx, int ny, int nz, const double *state, double *out)
{
    const int zd = nz + 2;
    double *UAVG = out, *VAVG = out + zd, *WAVG = out + 2 * zd, *UTIN = out + 3 * zd;
    double *VTIN = out + 4 * zd, *WTIN = out + 5 * zd, *REYS = out + 6 * zd, *DAVG = out + 7 * zd;
    double *DTIN = out + 8 * zd;
    double dens, u, v, w;
    memset(out, 0, sizeof(double) * 9 * zd);
    /* statistics.c:31-60 */
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 1; k < zd - 1; k++) {
                moments(state + IDX(i, j, k) * 19, &dens, &u, &v, &w);
                UAVG[k] += (u / dens);
                VAVG[k] += (v / dens);
                WAVG[k] += (w / dens);
                DAVG[k] += dens;
            }
    for (int k = 0; k < zd; k++) {
        UAVG[k] /= (double)(nx * ny);
        VAVG[k] /= (double)(nx * ny);
        WAVG[k] /= (double)(nx * ny);
        DAVG[k] /= (double)(nx * ny);
    }
    /* statistics.c:74-132 */
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 1; k < zd - 1; k++) {
                moments(state + IDX(i, j, k) * 19, &dens, &u, &v, &w);
                double UF = (u / dens) - UAVG[k], VF = (v / dens) - VAVG[k];
                double WF = (w / dens) - WAVG[k], DF = dens - DAVG[k];
                UTIN[k] += UF * UF;
                VTIN[k] += VF * VF;
                WTIN[k] += WF * WF;
                REYS[k] += UF * WF;
                DTIN[k] += DF * DF;
            }
    for (int k = 0; k < zd; k++) {
        UTIN[k] /= (double)(nx * ny);
        VTIN[k] /= (double)(ny * nx);
        WTIN[k] /= (double)(ny * nx);
        REYS[k] /= (double)(nx * ny);
        DTIN[k] /= (double)(nx * ny);
    }
    for (int k = 0; k < zd; k++) {
        UTIN[k] = sqrt(UTIN[k]);
        VTIN[k] = sqrt(VTIN[k]);
        WTIN[k] = sqrt(WTIN[k]);
        DTIN[k] = sqrt(DTIN[k]);
    }
}

void orc_moments(int nx, int ny, int nz, const double *state, double *vel, double *den)
{
    const int zd = nz + 2;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < zd; k++) {
                double dens, ux, uy, uz;
                /* vel_print.c:71-91 sums ux,uy,uz,dens in this order */
                const double *f = state + IDX(i, j, k) * 19;
                ux = 0.; uy = 0.; uz = 0.; dens = 0.;
                for (int a = 0; a < 19; a++) {
                    ux += (double)EX[a] * f[a];
                    uy += (double)EY[a] * f[a];
                    uz += (double)EZ[a] * f[a];
                    dens += f[a];
                }
                if (dens > 0.) {
                    ux /= dens; uy /= dens; uz /= dens;
                } else {
                    ux = 0.; uy = 0.; uz = 0.; dens = 0.;
                }
                size_t c = IDX(i, j, k);
                vel[c * 3 + 0] = ux;
                vel[c * 3 + 1] = uy;
                vel[c * 3 + 2] = uz;
                den[c] = dens;
            }
}

long orc_run(int nx, int ny, int nz, double *state, const int8_t *flags, double omega,
             double ubulk, double gx, int const_g, long nsteps, double *logs, int bc_mode)
{
    const int zd = nz + 2;
    double *scratch = malloc((size_t)nx * ny * zd * 19 * sizeof(double));
    if (!scratch) return -1;
    memcpy(scratch, state, (size_t)nx * ny * zd * 19 * sizeof(double));
    double rec[ORC_LOG_N];
    long s;
    for (s = 0; s < nsteps; s++) {
        double force = orc_encalc(nx, ny, nz, state, ubulk, rec);
        if (const_g) force = gx;
        rec[ORC_LOG_FORCE] = force;
        int bad = orc_wshearstr(nx, ny, nz, state, omega, force, rec);
        if (logs) memcpy(logs + s * ORC_LOG_N, rec, sizeof rec);
        if (bad) break;
        orc_step(nx, ny, nz, state, scratch, flags, omega, force, bc_mode);
    }
    free(scratch);
    return s;
}

/* ---- wall flags ------------------------------------------------------------ */
static void flags_base(int nx, int ny, int nz, int8_t *flags)
{
    const int zd = nz + 2;
    memset(flags, 0, (size_t)nx * ny * zd);
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++) {
            flags[IDX(x, y, 0)] = -1;
            flags[IDX(x, y, zd - 1)] = -1;
        }
}

void orc_flags_smooth(int nx, int ny, int nz, int8_t *flags) { flags_base(nx, ny, nz, flags); }

void orc_flags_ridges(int nx, int ny, int nz, int gap, int width, int8_t *flags)
{
    const int zd = nz + 2;
    flags_base(nx, ny, nz, flags);
    for (int j = width / 2; j < ny; j += gap + width)
        for (int a = 0; a < gap && j + a < ny; a++)
            for (int x = 0; x < nx; x++) {
                flags[IDX(x, j + a, 0)] = -2;
                flags[IDX(x, j + a, zd - 1)] = -2;
            }
}

void orc_flags_transverse(int nx, int ny, int nz, int gap, int width, int8_t *flags)
{
    const int zd = nz + 2;
    flags_base(nx, ny, nz, flags);
    for (int i = width / 2; i < nx; i += gap + width)
        for (int a = 0; a < gap && i + a < nx; a++)
            for (int y = 0; y < ny; y++) {
                flags[IDX(i + a, y, 0)] = -2;
                flags[IDX(i + a, y, zd - 1)] = -2;
            }
}

void orc_flags_posts(int nx, int ny, int nz, int gx, int wx, int gy, int wy, int8_t *flags)
{
    const int zd = nz + 2;
    flags_base(nx, ny, nz, flags);
    for (int j = 1; j < ny; j += gy + wy)
        for (int a = 0; a < gy && j + a < ny; a++)
            for (int i = 1; i < nx; i += gx + wx)
                for (int b = 0; b < gx && i + b < nx; b++) {
                    flags[IDX(i + b, j + a, 0)] = -2;
                    flags[IDX(i + b, j + a, zd - 1)] = -2;
                }
}
