// D3Q19 lattice and the structure-of-arrays population layout.
//
// Velocity numbering, weights, opposite() and mirror() are those of
// DNS-solver/src/globals.c:3-13, so states, flags and per-direction results
// are interchangeable with the reference's.
//
// HBM layout (one GPU, no ghost planes): population a of fluid cell
// (x, y, z), z = 0..zdv-1 (the reference's k = z + 1), lives at
//   pop[a][(z * ny + y) * nx + x]
// with x (streamwise, periodic) contiguous.  Each population array starts on
// a 256-byte boundary.  The AA pattern keeps one copy of the populations:
//   even step: cell x reads slot a at x, writes post-collision f*_a to slot
//              opp(a) at x;
//   odd step:  cell x reads slot opp(a) at x - e_a (which holds f*_a of its
//              upstream neighbour) and writes f*_a to slot a at x + e_a.
// Both steps therefore touch, per cell, one fixed set of 19 addresses for
// both the loads and the stores, which makes the sweep in-place safe.
#pragma once

#include <cstdint>

namespace dnslbm {

constexpr int Q = 19;

__host__ __device__ __forceinline__ constexpr int lat_ex(int a)
{
    return a == 1 || a == 7 || a == 10 || a == 11 || a == 12 ? 1
         : a == 2 || a == 8 || a == 9 || a == 13 || a == 14 ? -1 : 0;
}
__host__ __device__ __forceinline__ constexpr int lat_ey(int a)
{
    return a == 3 || a == 7 || a == 8 || a == 15 || a == 16 ? 1
         : a == 4 || a == 9 || a == 10 || a == 17 || a == 18 ? -1 : 0;
}
__host__ __device__ __forceinline__ constexpr int lat_ez(int a)
{
    return a == 5 || a == 11 || a == 14 || a == 15 || a == 18 ? 1
         : a == 6 || a == 12 || a == 13 || a == 16 || a == 17 ? -1 : 0;
}
// opposite direction (globals.c:12)
__host__ __device__ __forceinline__ constexpr int lat_opp(int a)
{
    return a == 0 ? 0 : a == 1 ? 2 : a == 2 ? 1 : a == 3 ? 4 : a == 4 ? 3 : a == 5 ? 6 : a == 6 ? 5
         : a == 7 ? 9 : a == 8 ? 10 : a == 9 ? 7 : a == 10 ? 8 : a == 11 ? 13 : a == 12 ? 14
         : a == 13 ? 11 : a == 14 ? 12 : a == 15 ? 17 : a == 16 ? 18 : a == 17 ? 15 : 16;
}
// reflection of the wall-normal component (globals.c:13)
__host__ __device__ __forceinline__ constexpr int lat_mir(int a)
{
    return a == 5 ? 6 : a == 6 ? 5 : a == 11 ? 12 : a == 12 ? 11 : a == 13 ? 14 : a == 14 ? 13
         : a == 15 ? 16 : a == 16 ? 15 : a == 17 ? 18 : a == 18 ? 17 : a;
}
// weight class: 0 -> 1/3, 1 -> 1/18, 2 -> 1/36 (globals.c:3)
__host__ __device__ __forceinline__ constexpr int lat_wclass(int a) { return a == 0 ? 0 : a <= 6 ? 1 : 2; }

// Wall links.  A cell in the plane next to a wall has five directions that
// point into the wall.  Their in-plane offsets (0,0) (1,0) (-1,0) (0,1)
// (0,-1) are numbered 0..4; bit i of the per-cell wall mask is 1 when that
// link bounces back (both the wall cell it points at and the wall cell below
// the fluid cell are no-slip) and 0 when it reflects specularly
// (xcomputations.c:368-375).
__host__ __device__ __forceinline__ constexpr int wall_link(int a)
{
    // in-plane offset index of a direction with ez != 0
    return lat_ex(a) == 1 ? 1 : lat_ex(a) == -1 ? 2 : lat_ey(a) == 1 ? 3 : lat_ey(a) == -1 ? 4 : 0;
}

struct Dims {
    int nx, ny, nz;  // fluid cells
};

}  // namespace dnslbm
