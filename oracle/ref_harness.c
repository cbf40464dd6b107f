/*
 * Harness main() that drives the REFERENCE's own, unmodified step functions
 * (DNS-solver/src: xcomputations.c, encalc.c, wshearstr.c, statistics.c,
 * vel_print.c, solid_init.c, slip_ridges_init.c, slip_posts_init.c, init.c,
 * globals.c) on one rank through the single-rank MPI stand-in.
 *
 * Test infrastructure: built into oracle/_ref/dnsref from the sources where
 * they lie, never shipped.  It replaces the reference's main()
 * (DNS-solver/src/dns-const-q-xycut.c:13-576) with the parts the step needs:
 *   - allocation of the POINTER arrays and the 12 halo buffers (:239-356),
 *   - the persistent halo requests, created in the same order (:363-376),
 *   - flags: solid_init (+ slip_ridges_init | slip_posts_init) (:385-395) or
 *     an explicit flag file,
 *   - state: reference init() (rest, :395) or a state file in the lbf layout
 *     global [xdv][ydv][zd][19] doubles, ghosts filled as the periodic image
 *     the restart path's Sendrecv calls produce (:418-425),
 *   - the time loop body (:485-519): encalc -> wshearstr -> [statistics,
 *     vel_print every `stats_every` steps] -> xcomputations.
 * In constant-g mode encalc still runs (its log lines are produced) and the
 * force it computed is replaced by the fixed g before xcomputations reads it.
 *
 * Usage: dnsref key=value ...
 *   xdv= ydv= zdv=        fluid cells (x streamwise, y spanwise, z wall-normal)
 *   omega=                relaxation rate (the reference's `tau` after 1/tau)
 *   ubulk=                target bulk velocity (constant-Q mode)
 *   mode=q|g  gx=         force mode; fixed body force for mode=g
 *   texture=smooth|ridges|posts|file   flags=<file> (int32 [xd][yd][zd])
 *   in=<file>             initial state (lbf ftemp layout); default: init()
 *   out=<file>            final state (lbf ftemp layout)
 *   force_out=<file>      per-step (force used, V.rho) doubles
 *   steps=N  stats_every=U (0: never)  vel_every=U (0: never)
 *   time=1                print timing line "MLUPS_STEP <mlups> <seconds>"
 *   warmup=W              untimed steps before the timed ones (time=1)
 *   only_step=1           timed steps run xcomputations alone (V.force
 *                         fixed at its first value; for timing only)
 */
#include "definitions.h"
#include "fun_defs.h"

#include <stdint.h>
#include <time.h>

static const char *arg(int argc, char **argv, const char *key, const char *def)
{
    size_t n = strlen(key);
    for (int i = 1; i < argc; i++)
        if (!strncmp(argv[i], key, n) && argv[i][n] == '=') return argv[i] + n + 1;
    return def;
}

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int main(int argc, char **argv)
{
    int xdv_ = atoi(arg(argc, argv, "xdv", "16"));
    int ydv_ = atoi(arg(argc, argv, "ydv", "8"));
    int zdv_ = atoi(arg(argc, argv, "zdv", "6"));
    double omega = atof(arg(argc, argv, "omega", "1.5"));
    double ubulk = atof(arg(argc, argv, "ubulk", "0.05"));
    double gx = atof(arg(argc, argv, "gx", "0"));
    const char *mode = arg(argc, argv, "mode", "q");
    const char *texture = arg(argc, argv, "texture", "smooth");
    const char *in = arg(argc, argv, "in", NULL);
    const char *out = arg(argc, argv, "out", NULL);
    const char *force_out = arg(argc, argv, "force_out", NULL);
    const char *flags_file = arg(argc, argv, "flags", NULL);
    long steps = atol(arg(argc, argv, "steps", "1"));
    long stats_every = atol(arg(argc, argv, "stats_every", "0"));
    long vel_every = atol(arg(argc, argv, "vel_every", "0"));
    int timing = atoi(arg(argc, argv, "time", "0"));
    long warmup = atol(arg(argc, argv, "warmup", "0"));
    int only_step = atoi(arg(argc, argv, "only_step", "0"));
    int const_g = (mode[0] == 'g');

    int xd = xdv_ + 1, yd = ydv_ + 1, zd = zdv_ + 2;
    int tagl = 1, tagr = 2;
    PDATA pd;
    POINTER V;
    MPI_Comm cart_grid;
    int dim[2] = {1, 1}, period[2] = {1, 1};

    MPI_Init(&argc, &argv);
    PI = 4. * atan(1.);
    pd.myrank = 0;
    pd.numproc = 1;
    MPI_Cart_create(MPI_COMM_WORLD, 2, dim, period, 1, &cart_grid);
    pd.up = pd.dw = pd.right = pd.left = pd.dl = pd.ur = pd.ul = pd.dr = 0;

    size_t ncell = (size_t)xd * yd * zd;
    V.s = (int *)calloc(ncell, sizeof(int));
    V.f = (DP *)calloc(ncell * 19, sizeof(DP));
    V.ftemp = (DP *)calloc(ncell * 19, sizeof(DP));
    V.rightbufs = (DP *)calloc(5 * yd * zd, sizeof(DP));
    V.rightbufr = (DP *)calloc(5 * yd * zd, sizeof(DP));
    V.leftbufs = (DP *)calloc(5 * yd * zd, sizeof(DP));
    V.leftbufr = (DP *)calloc(5 * yd * zd, sizeof(DP));
    V.upbufs = (DP *)calloc(5 * xd * zd, sizeof(DP));
    V.upbufr = (DP *)calloc(5 * xd * zd, sizeof(DP));
    V.dwbufs = (DP *)calloc(5 * xd * zd, sizeof(DP));
    V.dwbufr = (DP *)calloc(5 * xd * zd, sizeof(DP));
    V.urbufs = (DP *)calloc(9 * zd, sizeof(DP));
    V.dlbufr = (DP *)calloc(9 * zd, sizeof(DP));
    V.dlbufs = (DP *)calloc(9 * zd, sizeof(DP));
    V.urbufr = (DP *)calloc(9 * zd, sizeof(DP));
    if (!V.s || !V.f || !V.ftemp) {
        fprintf(stderr, "dnsref: allocation failed\n");
        return 2;
    }
    V.force = 0.;
    V.rho = 0.;

    /* same creation order as dns-const-q-xycut.c:363-376 */
    MPI_Send_init(V.leftbufs, (5 * yd * zd), MPDP, pd.left, tagl, MPI_COMM_WORLD, &V.req[0]);
    MPI_Send_init(V.rightbufs, (5 * yd * zd), MPDP, pd.right, tagr, MPI_COMM_WORLD, &V.req[1]);
    MPI_Recv_init(V.leftbufr, (5 * yd * zd), MPDP, pd.left, tagr, MPI_COMM_WORLD, &V.req[2]);
    MPI_Recv_init(V.rightbufr, (5 * yd * zd), MPDP, pd.right, tagl, MPI_COMM_WORLD, &V.req[3]);
    MPI_Send_init(V.dwbufs, (5 * xd * zd), MPDP, pd.dw, tagl, MPI_COMM_WORLD, &V.req[4]);
    MPI_Send_init(V.upbufs, (5 * xd * zd), MPDP, pd.up, tagr, MPI_COMM_WORLD, &V.req[5]);
    MPI_Recv_init(V.dwbufr, (5 * xd * zd), MPDP, pd.dw, tagr, MPI_COMM_WORLD, &V.req[6]);
    MPI_Recv_init(V.upbufr, (5 * xd * zd), MPDP, pd.up, tagl, MPI_COMM_WORLD, &V.req[7]);
    MPI_Send_init(V.urbufs, 9 * zd, MPDP, pd.ur, tagl, MPI_COMM_WORLD, &V.req[8]);
    MPI_Recv_init(V.dlbufr, 9 * zd, MPDP, pd.dl, tagl, MPI_COMM_WORLD, &V.req[9]);
    MPI_Send_init(V.dlbufs, 9 * zd, MPDP, pd.dl, tagr, MPI_COMM_WORLD, &V.req[10]);
    MPI_Recv_init(V.urbufr, 9 * zd, MPDP, pd.ur, tagr, MPI_COMM_WORLD, &V.req[11]);

    /* flags */
    V = solid_init(xd, yd, zd, V);
    if (!strcmp(texture, "ridges")) {
        V = slip_ridges_init(xd, yd, zd, V, pd, cart_grid);
    } else if (!strcmp(texture, "posts")) {
        V = slip_posts_init(xd, yd, zd, V, pd);
    } else if (!strcmp(texture, "file")) {
        FILE *ff = flags_file ? fopen(flags_file, "rb") : NULL;
        if (!ff || fread(V.s, sizeof(int), ncell, ff) != ncell) {
            fprintf(stderr, "dnsref: cannot read flags file\n");
            return 2;
        }
        fclose(ff);
    } else if (strcmp(texture, "smooth")) {
        fprintf(stderr, "dnsref: unknown texture %s\n", texture);
        return 2;
    }

    /* state */
    if (in) {
        FILE *fi = fopen(in, "rb");
        if (!fi) {
            fprintf(stderr, "dnsref: cannot open %s\n", in);
            return 2;
        }
        size_t col = (size_t)zd * 19;
        for (int i = 0; i < xdv_; i++)
            for (int j = 0; j < ydv_; j++)
                if (fread(&Fb(V.ftemp, i, j, 0, 0, xd, yd, zd, 19), sizeof(DP), col, fi) != col) {
                    fprintf(stderr, "dnsref: short state file\n");
                    return 2;
                }
        fclose(fi);
        /* ghost plane i=xd-1 <- i=0, row j=yd-1 <- j=0, corner <- (0,0) */
        /* (the reference's Fb macro does not parenthesise its arguments,
         * so every index passed to it is a plain variable) */
        int ig = xd - 1, jg = yd - 1;
        for (int j = 0; j < ydv_; j++)
            memcpy(&Fb(V.ftemp, ig, j, 0, 0, xd, yd, zd, 19), &Fb(V.ftemp, 0, j, 0, 0, xd, yd, zd, 19), col * sizeof(DP));
        for (int i = 0; i < xdv_; i++)
            memcpy(&Fb(V.ftemp, i, jg, 0, 0, xd, yd, zd, 19), &Fb(V.ftemp, i, 0, 0, 0, xd, yd, zd, 19), col * sizeof(DP));
        memcpy(&Fb(V.ftemp, ig, jg, 0, 0, xd, yd, zd, 19), &Fb(V.ftemp, 0, 0, 0, 0, xd, yd, zd, 19), col * sizeof(DP));
        memcpy(V.f, V.ftemp, ncell * 19 * sizeof(DP));
    } else {
        V = init(xd, yd, zd, V);
    }

    /* initial mean density, dns-const-q-xycut.c:464-480 */
    {
        double rho = 0.;
        for (int i = 0; i < xd - 1; i++)
            for (int j = 0; j < yd - 1; j++)
                for (int k = 1; k < zd - 1; k++) {
                    double r = 0.;
                    for (int a = 0; a < 19; a++) r += Fb(V.ftemp, i, j, k, a, xd, yd, zd, 19);
                    rho += r;
                }
        V.rho = rho / ((double)((xd - 1) * (yd - 1) * (zd - 2)));
    }

    FILE *fo = force_out ? fopen(force_out, "wb") : NULL;
    int TM = 0;
    double t0 = now_s();
    for (long ss = -warmup; ss < steps; ss++) {
        if (ss == 0) t0 = now_s();
        if (!only_step || ss == -warmup) {
            V = encalc(xd, yd, zd, V, 0., TM, ss, ubulk, cart_grid);
            if (const_g) V.force = gx;
            V = wshearstr(xd, yd, zd, V, 0., omega, TM, ss, cart_grid);
        }
        if (ss >= 0 && stats_every > 0 && !(ss % stats_every)) V = statistics(xd, yd, zd, V, pd, ss / stats_every);
        if (ss >= 0 && vel_every > 0 && !(ss % vel_every)) V = vel_print(xd, yd, zd, V, ss / vel_every, cart_grid);
        if (fo && ss >= 0) {
            double rec[2] = {V.force, V.rho};
            fwrite(rec, sizeof(double), 2, fo);
        }
        V = xcomputations(xd, yd, zd, V, pd, 0., 0., 0., 1., omega, ubulk);
    }
    double t1 = now_s();
    if (fo) fclose(fo);

    if (timing) {
        double cells = (double)xdv_ * ydv_ * zdv_ * (double)steps;
        printf("MLUPS_STEP %.6f %.6f\n", cells / (t1 - t0) / 1e6, t1 - t0);
    }

    if (out) {
        FILE *fw = fopen(out, "wb");
        if (!fw) {
            fprintf(stderr, "dnsref: cannot open %s\n", out);
            return 2;
        }
        size_t col = (size_t)zd * 19;
        for (int i = 0; i < xdv_; i++)
            for (int j = 0; j < ydv_; j++)
                fwrite(&Fb(V.ftemp, i, j, 0, 0, xd, yd, zd, 19), sizeof(DP), col, fw);
        fclose(fw);
    }
    return 0;
}
