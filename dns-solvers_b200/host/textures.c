/*
 * Wall textures on the periodic grid, in the reference's flag semantics
 * (DNS-solver/src/solid_init.c:3-8: 0 fluid, -1 no-slip, -2 slip/gas).
 * flags[(x*ny + y)*zd + z], zd = nz + 2, z = 0 and zd-1 the wall planes.
 */
#include "textures.h"

#include <math.h>
#include <string.h>

#define IDX(x, y, z) (((size_t)(x) * ny + (y)) * zd + (z))

/* solid_init.c:18-45 without ghost planes: both wall planes no-slip */
void tex_smooth(int nx, int ny, int nz, int8_t *flags)
{
    const int zd = nz + 2;
    memset(flags, 0, (size_t)nx * ny * zd);
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++) {
            flags[IDX(x, y, 0)] = -1;
            flags[IDX(x, y, zd - 1)] = -1;
        }
}

static void slip_both(int nx, int ny, int nz, int8_t *flags, int x, int y)
{
    const int zd = nz + 2;
    flags[IDX(x, y, 0)] = -2;
    flags[IDX(x, y, zd - 1)] = -2;
}

/* slip_ridges_init.c:11-40 with its constants as parameters: streamwise
 * stripes of `gap` slip cells followed by `width` no-slip cells, the first
 * at y = width/2; the top wall copies the bottom. */
void tex_longitudinal(int nx, int ny, int nz, int gap, int width, int8_t *flags)
{
    tex_smooth(nx, ny, nz, flags);
    for (int j = width / 2; j < ny; j += gap + width)
        for (int a = 0; a < gap && j + a < ny; a++)
            for (int x = 0; x < nx; x++) slip_both(nx, ny, nz, flags, x, j + a);
}

/* the stripe rule across the flow: spanwise (transverse) grooves */
void tex_transverse(int nx, int ny, int nz, int gap, int width, int8_t *flags)
{
    tex_smooth(nx, ny, nz, flags);
    for (int i = width / 2; i < nx; i += gap + width)
        for (int a = 0; a < gap && i + a < nx; a++)
            for (int y = 0; y < ny; y++) slip_both(nx, ny, nz, flags, i + a, y);
}

/* slip_posts_init.c:14-70 parameterised: gx x gy slip squares, periods
 * gx+wx (x) and gy+wy (y), the first at (1,1), both walls */
void tex_posts(int nx, int ny, int nz, int gx, int wx, int gy, int wy, int8_t *flags)
{
    tex_smooth(nx, ny, nz, flags);
    for (int j = 1; j < ny; j += gy + wy)
        for (int a = 0; a < gy && j + a < ny; a++)
            for (int i = 1; i < nx; i += gx + wx)
                for (int b = 0; b < gx && i + b < nx; b++) slip_both(nx, ny, nz, flags, i + b, j + a);
}

/* Triangular streamwise riblets cut into both no-slip walls (solid cells -1
 * inside the flow; the general boundary mode): in each spanwise period of
 * `spacing` cells a triangle of the given height, h(y) = height (1 -
 * |2 y_c / spacing - 1|) with y_c = (y mod spacing) + 1/2; a cell of wall
 * distance k - 1/2 (k = 1 the first fluid plane) is solid when below it. */
void tex_riblets(int nx, int ny, int nz, int height, int spacing, int8_t *flags)
{
    const int zd = nz + 2;
    tex_smooth(nx, ny, nz, flags);
    for (int y = 0; y < ny; y++) {
        const double yc = (y % spacing) + 0.5;
        const double h = height * (1.0 - fabs(2.0 * yc / spacing - 1.0));
        int nk = (int)ceil(h + 0.5) - 1;
        if (nk > nz / 2) nk = nz / 2;
        for (int k = 1; k <= nk; k++)
            for (int x = 0; x < nx; x++) {
                flags[IDX(x, y, k)] = -1;
                flags[IDX(x, y, zd - 1 - k)] = -1;
            }
    }
}
