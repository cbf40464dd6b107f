/*
 * Harness main() that drives the REFERENCE's own, unmodified two-point
 * correlation functions (2pt-correlations/src/xcorrel.c and ycorrel.c) on one
 * rank through the single-rank MPI stand-in.  Test infrastructure: built into
 * oracle/_ref/corref from the sources where they lie, never shipped.
 *
 * It replaces the reference's main (correlations.c), its MPI-IO reader
 * (reading.c) and its mean subtraction (mean_subtract.c, which divides by
 * gplus + wplus, both 0 in the program's definitions.h, so it cannot run as
 * shipped): the input file holds the velocity fluctuations already, layout
 * [xd][yd][zd][3] doubles (vel_print.c), and the harness writes what the
 * program's main writes for one time: xcorl.TTTT ([zd][xdv][3]) and
 * ycorl.TTTT ([zd][yd][3]).  xcorrel.c sizes and wraps its lags with the
 * program's compile-time xdv, so the streamwise extent must equal it.
 *
 * Usage: corref nx ny nz fluct-file label   (fluid cells x, y, z; nx = xdv)
 */
#include "definitions.h"
#include "fun_defs.h"

int main(int argc, char **argv)
{
    if (argc != 6) {
        fprintf(stderr, "usage: corref nx ny nz fluct-file label\n");
        return 2;
    }
    const int nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]);
    const int label = atoi(argv[5]);
    if (nx != xdv) {
        fprintf(stderr, "corref: the program is compiled for %d streamwise cells, got %d\n", xdv, nx);
        return 2;
    }
    MPI_Init(&argc, &argv);
    const int xd = nx, yd = ny, zd = nz + 2;
    const size_t n = (size_t)xd * yd * zd * 3;
    POINTER V;
    V.s = (int *)calloc((size_t)xd * yd * zd, sizeof(int));
    V.vel = (DP *)calloc(n, sizeof(DP));
    V.velrecv = (DP *)calloc(n, sizeof(DP));
    V.xcorl = (DP *)calloc((size_t)xdv * zd * 3, sizeof(DP));
    V.xcorlsl = (DP *)calloc((size_t)xdv * zd * 3, sizeof(DP));
    V.xcorlnsl = (DP *)calloc((size_t)xdv * zd * 3, sizeof(DP));
    V.ycorl = (DP *)calloc((size_t)yd * zd * 3, sizeof(DP));
    FILE *f = fopen(argv[4], "rb");
    if (!f || !V.vel || !V.velrecv || fread(V.vel, sizeof(DP), n, f) != n) {
        fprintf(stderr, "corref: cannot read %s\n", argv[4]);
        return 1;
    }
    fclose(f);
    PDATA pd;
    pd.myrank = 0;
    pd.numproc = 1;
    pd.left = 0;
    pd.right = 0;
    V = ycorrel(xd, yd, zd, V, pd, label, 0.);
    V = xcorrel(xd, yd, zd, V, pd, label, 0.);
    char fn[64];
    snprintf(fn, sizeof fn, "xcorl.%.4d", label);
    FILE *o = fopen(fn, "wb");
    if (!o || fwrite(V.xcorl, sizeof(DP), (size_t)xdv * zd * 3, o) != (size_t)xdv * zd * 3) return 1;
    fclose(o);
    snprintf(fn, sizeof fn, "ycorl.%.4d", label);
    o = fopen(fn, "wb");
    if (!o || fwrite(V.ycorl, sizeof(DP), (size_t)yd * zd * 3, o) != (size_t)yd * zd * 3) return 1;
    fclose(o);
    free(V.s);
    free(V.vel);
    free(V.velrecv);
    free(V.xcorl);
    free(V.xcorlsl);
    free(V.xcorlnsl);
    free(V.ycorl);
    MPI_Finalize();
    return 0;
}
