/*
 * run-dns: the channel-flow DNS driver on one B200, through the dnslbm C ABI.
 *
 * Mirrors the reference's main program (DNS-solver/src/dns-const-q-xycut.c)
 * with its deck, start modes and output files; the time step itself runs on
 * the GPU.  Usage, as the reference's (README "Usage"):
 *
 *     run-dns -s|-p [deck-file] [NAME=value ...]
 *
 *   -s  fresh start from rest (init.c), flags from the deck's texture
 *   -p  restart from lbf.TSTR (ftemp then f, [xdv][ydv][zd][19] doubles)
 *       and force.TSTR (one double), dns-const-q-xycut.c:399-454
 *
 * Deck (file lines "NAME value", or NAME=value arguments): the reference's
 * compile-time names Rebs ub zdv ydv xdv TSTR TEND CFL ITER (definitions.h:
 * 30-52) and RSLIP / PSLIP (set to 1 to select those textures with the
 * reference's constants), plus
 *   TEXTURE smooth|ridges|transverse|posts|riblets   GAP WIDTH   PGX PWX PGY PWY
 *   RIBH RIBS (riblet height and spacing; riblets select the general wall
 *   rule, DNSLBM_BC_GENERAL)
 *   PRECISION 64|32|16   FORCE q|g   GX   DEVICE   OMEGA (overrides Rebs)
 *   QUADRANT 1  also the quadrant analysis of quadrant-analysis/src/
 *               qUADrantA.c at every output event, on the GPU, from the live
 *               state: quadrant.000.TTTT and dquadrant.000.TTTT ([4][zd] then
 *               [zd] doubles)
 *   CORREL 1    also the two-point correlations of 2pt-correlations/src
 *               (mean_subtract.c, xcorrel.c, ycorrel.c) at every output
 *               event, on the GPU: xcorl.TTTT ([zd][xdv][3]), ycorl.TTTT
 *               ([zd][ydv][3]) and uavg.TTT ([zd]) doubles
 *   SPECTRA 1   also the one-dimensional energy spectra of e-spectra/src/
 *               1d-spectra.c at every output event, on the GPU: Euux.TTTT,
 *               Evvx.TTTT, Ewwx.TTTT ([xdv][zd]) and Euuy, Evvy, Ewwy
 *               ([ydv/2+1][zd]) doubles
 *   ASYNC 1|0   output without stopping the time loop (default 1): at an
 *               output step the library computes the outputs on the GPU and
 *               copies them to page-locked host buffers while the next steps
 *               run (dnslbm_output_begin), and a writer thread writes the
 *               files; 0 stores, writes and only then steps on
 *
 * Files written (formats of the reference):
 *   energy.txt flowrate.txt massrate.txt   encalc.c:125-138, every step
 *   str-up.txt str-do.txt w-str.txt p-grad.txt   wshearstr.c:133-154
 *   lbf.NNNN force.NNNN   every 10*utime steps, dns-const-q-xycut.c:491-513
 *   vel.NNNN den.NNNN     every utime steps, vel_print.c
 *   turb-fld.000.TTT uavg-temp.dat   every utime steps, statistics.c:135-165
 *   report.code           dns-const-q-xycut.c:522-540
 * The lbf file's second half (the reference's f array, whose values the next
 * step overwrites before reading) holds the state again.
 */
#include <errno.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../include/dnslbm.h"
#include "textures.h"

typedef struct {
    double Rebs, ub, CFL, GX, OMEGA;
    int zdv, ydv, xdv, TSTR, TEND, ITER, RSLIP, PSLIP;
    int PRECISION, DEVICE, GAP, WIDTH, PGX, PWX, PGY, PWY, RIBH, RIBS, ASYNC, QUADRANT, CORREL, SPECTRA;
    char TEXTURE[32], FORCE[8];
} Deck;

static void deck_defaults(Deck *d)
{
    /* the reference's shipped deck, definitions.h:30-37 */
    memset(d, 0, sizeof *d);
    d->Rebs = 100.0;
    d->ub = 0.1;
    d->zdv = 25;
    d->ydv = 8;
    d->xdv = 16;
    d->TSTR = 420;
    d->TEND = 440;
    d->CFL = 0.1;
    d->ITER = -1;
    d->PRECISION = 64;
    d->GAP = 2;
    d->WIDTH = 2;
    d->PGX = 2;
    d->PWX = 2;
    d->PGY = 2;
    d->PWY = 2;
    d->RIBH = 8;
    d->RIBS = 16;
    d->ASYNC = 1;
    strcpy(d->TEXTURE, "smooth");
    strcpy(d->FORCE, "q");
}

static int deck_set(Deck *d, const char *k, const char *v)
{
#define DBL(N) if (!strcmp(k, #N)) { d->N = atof(v); return 0; }
#define INT(N) if (!strcmp(k, #N)) { d->N = atoi(v); return 0; }
#define STR(N) if (!strcmp(k, #N)) { snprintf(d->N, sizeof d->N, "%s", v); return 0; }
    DBL(Rebs) DBL(ub) DBL(CFL) DBL(GX) DBL(OMEGA)
    INT(zdv) INT(ydv) INT(xdv) INT(TSTR) INT(TEND) INT(ITER) INT(RSLIP) INT(PSLIP)
    INT(PRECISION) INT(DEVICE) INT(GAP) INT(WIDTH) INT(PGX) INT(PWX) INT(PGY) INT(PWY) INT(RIBH) INT(RIBS) INT(ASYNC) INT(QUADRANT) INT(CORREL) INT(SPECTRA)
    STR(TEXTURE) STR(FORCE)
#undef DBL
#undef INT
#undef STR
    fprintf(stderr, "run-dns: unknown deck entry %s\n", k);
    return -1;
}

static int deck_read(Deck *d, const char *path)
{
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char line[256], k[64], v[128];
    while (fgets(line, sizeof line, f)) {
        char *h = strchr(line, '#');
        if (h) *h = 0;
        for (char *p = line; *p; p++)
            if (*p == '=') *p = ' ';
        if (sscanf(line, "%63s %127s", k, v) == 2 && deck_set(d, k, v)) {
            fclose(f);
            return -2;
        }
    }
    fclose(f);
    return 0;
}

static int die(dnslbm_ctx *c, int rc, const char *what)
{
    fprintf(stderr, "run-dns: %s failed (%d): %s\n", what, rc, dnslbm_last_error(c));
    return 1;
}

static void append(const char *fn, const char *fmt, double t, double v)
{
    FILE *f = fopen(fn, "a");
    if (!f) return;
    fprintf(f, fmt, t, v);
    fclose(f);
}

static int write_file(const char *fn, const void *p, size_t bytes, size_t copies)
{
    FILE *f = fopen(fn, "wb");
    if (!f) return -1;
    for (size_t i = 0; i < copies; i++)
        if (fwrite(p, 1, bytes, f) != bytes) {
            fclose(f);
            return -1;
        }
    return fclose(f);
}

/* One output event's files: lbf/force (checkpoints only), vel, den,
 * turb-fld and uavg-temp.dat, from host buffers. */
typedef struct {
    double *state, *vel, *den, *stats;
    double force;
    long label;
    int checkpoint;
} Snapshot;

typedef struct {
    size_t state_n, ncol;
    int zd;
} Shape;

static int write_snapshot(const Snapshot *sn, const Shape *sh)
{
    char fn[64];
    if (sn->checkpoint) {
        snprintf(fn, sizeof fn, "lbf.%.4ld", sn->label);
        if (write_file(fn, sn->state, sh->state_n * sizeof(double), 2)) return -1;
        snprintf(fn, sizeof fn, "force.%.4ld", sn->label);
        if (write_file(fn, &sn->force, sizeof sn->force, 1)) return -1;
    }
    snprintf(fn, sizeof fn, "vel.%.4d", (int)sn->label);
    if (write_file(fn, sn->vel, sh->ncol * sh->zd * 3 * sizeof(double), 1)) return -1;
    snprintf(fn, sizeof fn, "den.%.4d", (int)sn->label);
    if (write_file(fn, sn->den, sh->ncol * sh->zd * sizeof(double), 1)) return -1;
    snprintf(fn, sizeof fn, "turb-fld.%.3d.%.3ld", 0, sn->label);
    if (write_file(fn, sn->stats, 9 * sh->zd * sizeof(double), 1)) return -1;
    FILE *u = fopen("uavg-temp.dat", "w");
    if (u) {
        const int zd = sh->zd;
        for (int k = 0; k < zd; k++) {
            double z = k == 0 ? 0. : (k == zd - 1 ? zd - 2. : k - 0.5);
            fprintf(u, "%.12f %.12f\n", z / (zd - 2.), sn->stats[k]);
        }
        fclose(u);
    }
    return 0;
}

/* The writer thread: one job at a time, handed over by the time loop. */
typedef struct {
    pthread_t th;
    pthread_mutex_t mu;
    pthread_cond_t cv;
    const Snapshot *job;  /* pending job, NULL when idle */
    const Shape *shape;
    int quit, failed;
} Writer;

static void *writer_main(void *arg)
{
    Writer *w = arg;
    pthread_mutex_lock(&w->mu);
    for (;;) {
        while (!w->job && !w->quit) pthread_cond_wait(&w->cv, &w->mu);
        if (!w->job) break;
        const Snapshot *sn = w->job;
        pthread_mutex_unlock(&w->mu);
        const int bad = write_snapshot(sn, w->shape);
        pthread_mutex_lock(&w->mu);
        if (bad) w->failed = 1;
        w->job = NULL;
        pthread_cond_broadcast(&w->cv);
    }
    pthread_mutex_unlock(&w->mu);
    return NULL;
}

/* Wait until the writer is idle; returns nonzero if a write failed. */
static int writer_wait(Writer *w)
{
    pthread_mutex_lock(&w->mu);
    while (w->job) pthread_cond_wait(&w->cv, &w->mu);
    const int failed = w->failed;
    pthread_mutex_unlock(&w->mu);
    return failed;
}

static void writer_submit(Writer *w, const Snapshot *sn)
{
    pthread_mutex_lock(&w->mu);
    w->job = sn;
    pthread_cond_broadcast(&w->cv);
    pthread_mutex_unlock(&w->mu);
}

/* Page-locked when possible (the copies then overlap the steps). */
static double *host_buffer(size_t n, int *pinned)
{
    double *p = dnslbm_host_alloc(n * sizeof(double));
    *pinned = p != NULL;
    return p ? p : malloc(n * sizeof(double));
}

static void host_buffer_free(double *p, int pinned)
{
    if (pinned) dnslbm_host_free(p);
    else free(p);
}

int main(int argc, char **argv)
{
    if (argc < 2 || (strcmp(argv[1], "-s") && strcmp(argv[1], "-p"))) {
        fprintf(stderr, "usage: run-dns -s|-p [deck-file] [NAME=value ...]\n");
        return 2;
    }
    Deck D;
    deck_defaults(&D);
    int a = 2;
    if (argc > 2 && !strchr(argv[2], '=')) {
        if (deck_read(&D, argv[2])) {
            fprintf(stderr, "run-dns: cannot read deck %s\n", argv[2]);
            return 2;
        }
        a = 3;
    }
    for (; a < argc; a++) {
        char k[64];
        const char *eq = strchr(argv[a], '=');
        if (!eq || eq - argv[a] >= (long)sizeof k) return 2;
        memcpy(k, argv[a], eq - argv[a]);
        k[eq - argv[a]] = 0;
        if (deck_set(&D, k, eq + 1)) return 2;
    }
    if (D.RSLIP) strcpy(D.TEXTURE, "ridges");
    if (D.PSLIP) strcpy(D.TEXTURE, "posts");

    /* derived parameters, dns-const-q-xycut.c:55,203-237 */
    const int zd = D.zdv + 2;
    double utime_d = 0.5 * (zd - 2.) / D.CFL;
    const double dt = 1. / utime_d;
    const long utime = (long)utime_d;
    double tau = (3. / D.Rebs) * D.ub * (zd - 2.) + 0.5;
    double omega = D.OMEGA > 0 ? D.OMEGA : 1. / tau;
    long up = (long)(D.TEND - D.TSTR) * utime;
    if (D.ITER >= 0) up = D.ITER;
    if (utime < 1) {
        fprintf(stderr, "run-dns: CFL gives less than one step per time unit\n");
        return 2;
    }

    dnslbm_deck dk = {D.xdv, D.ydv, D.zdv, omega, D.ub, D.GX,
                      D.FORCE[0] == 'g' ? DNSLBM_FORCE_CONST_G : DNSLBM_FORCE_CONST_Q,
                      D.PRECISION, strcmp(D.TEXTURE, "riblets") ? DNSLBM_BC_REFERENCE : DNSLBM_BC_GENERAL, 0,
                      D.DEVICE};
    dnslbm_ctx *c = NULL;
    int rc = dnslbm_create(&dk, &c);
    if (rc) return die(NULL, rc, "dnslbm_create");

    const size_t nflag = (size_t)D.xdv * D.ydv * zd;
    int8_t *flags = malloc(nflag);
    const size_t ncol = (size_t)D.xdv * D.ydv, state_n = ncol * zd * 19;
    double *state = malloc(state_n * sizeof(double));
    if (!flags || !state) {
        fprintf(stderr, "run-dns: host allocation failed: %s\n", strerror(errno));
        return 1;
    }
    if (!strcmp(D.TEXTURE, "smooth")) tex_smooth(D.xdv, D.ydv, D.zdv, flags);
    else if (!strcmp(D.TEXTURE, "ridges")) tex_longitudinal(D.xdv, D.ydv, D.zdv, D.GAP, D.WIDTH, flags);
    else if (!strcmp(D.TEXTURE, "transverse")) tex_transverse(D.xdv, D.ydv, D.zdv, D.GAP, D.WIDTH, flags);
    else if (!strcmp(D.TEXTURE, "posts")) tex_posts(D.xdv, D.ydv, D.zdv, D.PGX, D.PWX, D.PGY, D.PWY, flags);
    else if (!strcmp(D.TEXTURE, "riblets") && D.RIBH > 0 && D.RIBS > 1)
        tex_riblets(D.xdv, D.ydv, D.zdv, D.RIBH, D.RIBS, flags);
    else {
        fprintf(stderr, "run-dns: unknown texture %s\n", D.TEXTURE);
        return 2;
    }
    if ((rc = dnslbm_set_flags_periodic(c, flags))) return die(c, rc, "dnslbm_set_flags_periodic");

    char fn[64];
    int TM;
    if (argv[1][1] == 's') {
        TM = D.TSTR;
        if ((rc = dnslbm_init_rest(c))) return die(c, rc, "dnslbm_init_rest");
    } else {
        fprintf(stderr, "TRYING TO READ DATA FROM FILES\n");
        snprintf(fn, sizeof fn, "lbf.%.4d", D.TSTR);
        FILE *f = fopen(fn, "rb");
        if (!f || fread(state, sizeof(double), state_n, f) != state_n) {
            fprintf(stderr, "run-dns: cannot read %s (need %zu doubles of ftemp)\n", fn, state_n);
            return 1;
        }
        fclose(f);
        snprintf(fn, sizeof fn, "force.%.4d", D.TSTR);
        f = fopen(fn, "rb");
        double force = 0.;
        if (f) {
            if (fread(&force, sizeof force, 1, f) != 1) force = 0.;
            fclose(f);
        }
        if ((rc = dnslbm_load_state(c, state))) return die(c, rc, "dnslbm_load_state");
        TM = D.TSTR;
        fprintf(stderr, "END OF READING DATA FROM FILES\nSTARTING FROM %d\n", TM);
    }

    /* Output buffers: one checkpoint state (checkpoints are ten output
     * events apart, so the writer is long done with it) and two sets of
     * vel/den/turb-fld, one being filled while the writer drains the other.
     * The synchronous mode uses the first set and the state array. */
    const Shape shape = {state_n, ncol, zd};
    Snapshot snap[2];
    int pin_state = 0, pin[2][3] = {{0}};
    double *ckpt = D.ASYNC ? host_buffer(state_n, &pin_state) : state;
    for (int i = 0; i < 2; i++) {
        snap[i].state = ckpt;
        snap[i].vel = host_buffer(ncol * zd * 3, &pin[i][0]);
        snap[i].den = host_buffer(ncol * zd, &pin[i][1]);
        snap[i].stats = host_buffer(9 * (size_t)zd, &pin[i][2]);
    }
    const long cap = 4096;
    double *logs = malloc(cap * DNSLBM_LOG_N * sizeof(double));
    int bad_alloc = !ckpt || !logs;
    for (int i = 0; i < 2; i++) bad_alloc |= !snap[i].vel || !snap[i].den || !snap[i].stats;
    if (bad_alloc) {
        fprintf(stderr, "run-dns: host allocation failed\n");
        return 1;
    }
    Writer W = {.job = NULL, .shape = &shape, .quit = 0, .failed = 0};
    pthread_mutex_init(&W.mu, NULL);
    pthread_cond_init(&W.cv, NULL);
    if (D.ASYNC && pthread_create(&W.th, NULL, writer_main, &W)) {
        fprintf(stderr, "run-dns: cannot start the writer thread\n");
        return 1;
    }

    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    long ss = 0, nout = 0;
    int nan_stop = 0;
    while (ss < up + 1 && !nan_stop) {
        if (!(ss % utime)) {
            Snapshot *sn = &snap[nout & 1];
            sn->label = TM + ss / utime;
            sn->checkpoint = !(ss % (10 * utime));
            if (sn->checkpoint && (rc = dnslbm_get_force(c, &sn->force))) return die(c, rc, "dnslbm_get_force");
            if (D.QUADRANT) {
                double *q = malloc(9 * (size_t)zd * sizeof(double));
                if (!q) return die(c, DNSLBM_ERR_IO, "host allocation");
                if ((rc = dnslbm_quadrant(c, q, q + 4 * zd, q + 8 * zd))) return die(c, rc, "dnslbm_quadrant");
                char qn[64];
                snprintf(qn, sizeof qn, "quadrant.%.3d.%.4d", 0, (int)sn->label);
                FILE *qf = fopen(qn, "wb");
                int bad = !qf || fwrite(q, sizeof(double), 4 * (size_t)zd, qf) != 4 * (size_t)zd ||
                          fwrite(q + 8 * zd, sizeof(double), zd, qf) != (size_t)zd;
                if (qf) bad |= fclose(qf) != 0;
                snprintf(qn, sizeof qn, "dquadrant.%.3d.%.4d", 0, (int)sn->label);
                qf = fopen(qn, "wb");
                bad |= !qf || fwrite(q + 4 * zd, sizeof(double), 4 * (size_t)zd, qf) != 4 * (size_t)zd ||
                       fwrite(q + 8 * zd, sizeof(double), zd, qf) != (size_t)zd;
                if (qf) bad |= fclose(qf) != 0;
                free(q);
                if (bad) return die(c, DNSLBM_ERR_IO, qn);
            }
            if (D.CORREL) {
                const size_t nxc = (size_t)zd * D.xdv * 3, nyc = (size_t)zd * D.ydv * 3;
                double *r = malloc((nxc + nyc + (size_t)zd) * sizeof(double));
                if (!r) return die(c, DNSLBM_ERR_IO, "host allocation");
                if ((rc = dnslbm_correlations(c, r, r + nxc, r + nxc + nyc))) return die(c, rc, "dnslbm_correlations");
                char cn[64];
                const char *fmt[3] = {"xcorl.%.4d", "ycorl.%.4d", "uavg.%.3d"};
                const size_t off[3] = {0, nxc, nxc + nyc}, len[3] = {nxc, nyc, (size_t)zd};
                int bad = 0;
                for (int f = 0; f < 3 && !bad; ++f) {
                    snprintf(cn, sizeof cn, fmt[f], (int)sn->label);
                    FILE *cf = fopen(cn, "wb");
                    bad = !cf || fwrite(r + off[f], sizeof(double), len[f], cf) != len[f];
                    if (cf) bad |= fclose(cf) != 0;
                }
                free(r);
                if (bad) return die(c, DNSLBM_ERR_IO, cn);
            }
            if (D.SPECTRA) {
                const size_t nex = (size_t)D.xdv * zd, ney = (size_t)(D.ydv / 2 + 1) * zd;
                double *r = malloc(3 * (nex + ney) * sizeof(double));
                if (!r) return die(c, DNSLBM_ERR_IO, "host allocation");
                if ((rc = dnslbm_spectra(c, r, r + 3 * nex))) return die(c, rc, "dnslbm_spectra");
                static const char *name[6] = {"Euux", "Evvx", "Ewwx", "Euuy", "Evvy", "Ewwy"};
                char sn_[64];
                int bad = 0;
                for (int f = 0; f < 6 && !bad; ++f) {
                    const double *src = f < 3 ? r + f * nex : r + 3 * nex + (f - 3) * ney;
                    const size_t len = f < 3 ? nex : ney;
                    snprintf(sn_, sizeof sn_, "%s.%.4d", name[f], (int)sn->label);
                    FILE *sf = fopen(sn_, "wb");
                    bad = !sf || fwrite(src, sizeof(double), len, sf) != len;
                    if (sf) bad |= fclose(sf) != 0;
                }
                free(r);
                if (bad) return die(c, DNSLBM_ERR_IO, sn_);
            }
            if (D.ASYNC) {
                /* the previous event's copies have landed (the steps since
                 * took longer); hand them to the writer once it is done with
                 * the event before, whose buffers this event reuses */
                if (nout > 0) {
                    if ((rc = dnslbm_output_wait(c))) return die(c, rc, "dnslbm_output_wait");
                    if (writer_wait(&W)) return die(c, DNSLBM_ERR_IO, "writing an output file");
                    writer_submit(&W, &snap[(nout - 1) & 1]);
                }
                if ((rc = dnslbm_output_begin(c, sn->checkpoint ? sn->state : NULL, sn->vel, sn->den, sn->stats)))
                    return die(c, rc, "dnslbm_output_begin");
            } else {
                if (sn->checkpoint && (rc = dnslbm_store_state(c, sn->state))) return die(c, rc, "dnslbm_store_state");
                if ((rc = dnslbm_moments(c, sn->vel, sn->den))) return die(c, rc, "dnslbm_moments");
                if ((rc = dnslbm_statistics(c, sn->stats))) return die(c, rc, "dnslbm_statistics");
                if (write_snapshot(sn, &shape)) return die(c, DNSLBM_ERR_IO, "writing an output file");
            }
            nout++;
        }
        /* steps up to the next output event, in one device batch */
        long n = utime - ss % utime;
        if (n > up + 1 - ss) n = up + 1 - ss;
        if (n > cap) n = cap;
        rc = dnslbm_step(c, n);
        long have = n;
        if (rc == DNSLBM_ERR_NAN) {
            /* logs up to the failing step, then stop as the reference's abort() */
            long first_bad = n;
            double *tmp = logs;
            dnslbm_logs(c, dnslbm_steps_done(c) - n, n, tmp);
            for (long i = 0; i < n; i++)
                if (tmp[i * DNSLBM_LOG_N + DNSLBM_LOG_STRESS] != tmp[i * DNSLBM_LOG_N + DNSLBM_LOG_STRESS]) {
                    first_bad = i;
                    break;
                }
            have = first_bad;
            nan_stop = 1;
        } else if (rc) {
            return die(c, rc, "dnslbm_step");
        } else if ((rc = dnslbm_logs(c, dnslbm_steps_done(c) - n, n, logs))) {
            return die(c, rc, "dnslbm_logs");
        }
        for (long i = 0; i < have; i++) {
            const double *r = logs + i * DNSLBM_LOG_N;
            const double t = (double)TM + dt * (ss + i);
            append("energy.txt", "%f %.14f\n", t, r[DNSLBM_LOG_ENERGY]);
            append("flowrate.txt", "%f %.12f\n", t, r[DNSLBM_LOG_FLOWRATE]);
            append("massrate.txt", "%f %.12f\n", t, r[DNSLBM_LOG_MASSRATE]);
            append("str-up.txt", "%f %.12f\n", t, r[DNSLBM_LOG_STUP]);
            append("str-do.txt", "%f %.12f\n", t, r[DNSLBM_LOG_STDOWN]);
            append("w-str.txt", "%f %.12f\n", t, r[DNSLBM_LOG_STRESS]);
            append("p-grad.txt", "%f %.12f\n", t, r[DNSLBM_LOG_PGRAD]);
        }
        if (nan_stop && have < n) {
            /* energy/flowrate/massrate of the failing step come before the
             * check in the reference (encalc runs before wshearstr) */
            const double *r = logs + have * DNSLBM_LOG_N;
            const double t = (double)TM + dt * (ss + have);
            append("energy.txt", "%f %.14f\n", t, r[DNSLBM_LOG_ENERGY]);
            append("flowrate.txt", "%f %.12f\n", t, r[DNSLBM_LOG_FLOWRATE]);
            append("massrate.txt", "%f %.12f\n", t, r[DNSLBM_LOG_MASSRATE]);
            fprintf(stderr, "Eroor: NAN, found in wall shear stress\n");
        }
        ss += n;
    }
    if (D.ASYNC) {
        if (nout > 0) {
            if ((rc = dnslbm_output_wait(c))) return die(c, rc, "dnslbm_output_wait");
            if (writer_wait(&W)) return die(c, DNSLBM_ERR_IO, "writing an output file");
            writer_submit(&W, &snap[(nout - 1) & 1]);
        }
        const int failed = writer_wait(&W);
        pthread_mutex_lock(&W.mu);
        W.quit = 1;
        pthread_cond_broadcast(&W.cv);
        pthread_mutex_unlock(&W.mu);
        pthread_join(W.th, NULL);
        if (failed) return die(c, DNSLBM_ERR_IO, "writing an output file");
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    const double secs = (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);

    FILE *tm = fopen("report.code", "w");
    if (tm) {
        fprintf(tm, "xd=%d,yd=%d,zd+2=%d,Reb=%f,tau=%f,G=%.10f,Ub=%f,CFLnumber=%f\n", D.xdv + 1, D.ydv + 1, zd,
                D.Rebs, omega, D.GX, D.ub, D.CFL);
        fprintf(tm, "number of processors: 1 GPU (device %d)\n", D.DEVICE);
        fprintf(tm, "Executed File's Name: %s\n", __FILE__);
        fprintf(tm, "Compilation Option: dnslbm fp%d\n", D.PRECISION);
        fprintf(tm, "slip option: %s\n", D.TEXTURE);
        fprintf(tm, "Total computational time is: %f s\n", secs);
        fprintf(tm, "Unit non-dimensional time is: %f iterations\n", (double)utime);
        fprintf(tm, "Starting time: %d\n", D.TSTR);
        fprintf(tm, "Current Time is: %d\n", D.TEND);
        fclose(tm);
    }
    free(flags);
    free(state);
    if (D.ASYNC) host_buffer_free(ckpt, pin_state);
    for (int i = 0; i < 2; i++) {
        host_buffer_free(snap[i].vel, pin[i][0]);
        host_buffer_free(snap[i].den, pin[i][1]);
        host_buffer_free(snap[i].stats, pin[i][2]);
    }
    free(logs);
    pthread_mutex_destroy(&W.mu);
    pthread_cond_destroy(&W.cv);
    dnslbm_destroy(c);
    return nan_stop ? 1 : 0;
}
