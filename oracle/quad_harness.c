/*
 * Harness main() that drives the REFERENCE's own, unmodified quadrant
 * analysis (quadrant-analysis/src/qUADrantA.c) on one rank through the
 * single-rank MPI stand-in.  Test infrastructure: built into oracle/_ref/
 * quadref from the sources where they lie, never shipped.
 *
 * It replaces the reference's main (postproc-base-flow-quadrant.c) and its
 * MPI-IO reader (reading.c): the velocity field of one vel file, layout
 * [xdv][ydv][zd][3] doubles (vel_print.c), is placed into V.vel with the
 * reference's two leading halo planes in x (definitions.h: Fb offsets i by
 * 2), the periodic images in the halo planes as reading.c fills them, and
 * qUADrantA writes quadrant.000.TTTT and dquadrant.000.TTTT.
 *
 * Usage: quadref nx ny nz vel-file label   (fluid cells x, y, z)
 */
#include "definitions.h"
#include "fun_defs.h"

int main(int argc, char **argv)
{
    if (argc != 6) {
        fprintf(stderr, "usage: quadref nx ny nz vel-file label\n");
        return 2;
    }
    /* (the reference's definitions.h defines xdv/ydv/zdv as its own constants) */
    const int nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]);
    const long label = atol(argv[5]);
    MPI_Init(&argc, &argv);
    const int zd = nz + 2, yd = ny, xd = nx + 1;  /* one rank: xd = 1 + x-extent/numproc */
    const size_t plane = (size_t)yd * zd * 3;
    POINTER V;
    V.s = (int *)calloc((size_t)xd * yd * zd, sizeof(int));
    V.vel = (DP *)calloc((size_t)(xd + 3) * plane, sizeof(DP));
    V.den = (DP *)calloc((size_t)(xd + 3) * yd * zd, sizeof(DP));
    FILE *f = fopen(argv[4], "rb");
    if (!f || !V.vel || !V.den || fread(V.vel + 2 * plane, sizeof(DP), (size_t)nx * plane, f) != (size_t)nx * plane) {
        fprintf(stderr, "quadref: cannot read %s\n", argv[4]);
        return 1;
    }
    fclose(f);
    /* halo planes i = -2, -1 and i = nx: the periodic images */
    memcpy(V.vel, V.vel + (size_t)nx * plane, 2 * plane * sizeof(DP));
    memcpy(V.vel + (size_t)(nx + 2) * plane, V.vel + 2 * plane, plane * sizeof(DP));
    PDATA pd;
    pd.myrank = 0;
    pd.numproc = 1;
    pd.left = 0;
    pd.right = 0;
    V = qUADrantA(xd, yd, zd, V, pd, label);
    free(V.s);
    free(V.vel);
    free(V.den);
    MPI_Finalize();
    return 0;
}
