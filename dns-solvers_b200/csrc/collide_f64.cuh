// FP64 collision in the reference's operand order (xcomputations.c:314-342).
// Every translation unit that calls f64_collide must be compiled with
// -fmad=false: the bit-exact parity with the reference depends on no fused
// multiply-add.  Zero terms of the reference's sums (E*f with E == 0) are
// omitted: adding a signed zero to a non-zero partial sum leaves it unchanged.
#pragma once

#include "lattice.cuh"

namespace dnslbm {

// Moments in the reference's summation order (a = 0..18).
__device__ __forceinline__ void f64_moments(const double (&f)[Q], double &dens, double &jx, double &jy, double &jz)
{
    dens = 0.0;
#pragma unroll
    for (int a = 0; a < Q; ++a) dens = dens + f[a];
    jx = 0.0;
    jy = 0.0;
    jz = 0.0;
#pragma unroll
    for (int a = 0; a < Q; ++a) {
        if (lat_ex(a) > 0) jx = jx + f[a];
        if (lat_ex(a) < 0) jx = jx - f[a];
        if (lat_ey(a) > 0) jy = jy + f[a];
        if (lat_ey(a) < 0) jy = jy - f[a];
        if (lat_ez(a) > 0) jz = jz + f[a];
        if (lat_ez(a) < 0) jz = jz - f[a];
    }
}

// e_a . u with the reference's grouping (E0*u0 + E1*u1) + E2*u2.
template <int A>
__device__ __forceinline__ double f64_eu(double u0, double u1, double u2)
{
    constexpr int ex = lat_ex(A), ey = lat_ey(A), ez = lat_ez(A);
    double s = 0.0;
    bool first = true;
    if (ex != 0) { s = ex > 0 ? u0 : -u0; first = false; }
    if (ey != 0) { s = first ? (ey > 0 ? u1 : -u1) : (ey > 0 ? s + u1 : s - u1); first = false; }
    if (ez != 0) { s = first ? (ez > 0 ? u2 : -u2) : (ez > 0 ? s + u2 : s - u2); }
    return s;
}

struct F64Cell {
    double dens, jx, u0, u1, u2;
};

// BGK collision with the reference's forcing term, in place.
__device__ __forceinline__ F64Cell f64_collide(double (&f)[Q], double omega, double G)
{
    F64Cell c;
    double jy, jz;
    f64_moments(f, c.dens, c.jx, jy, jz);
    c.u0 = c.jx / c.dens;
    c.u1 = jy / c.dens;
    c.u2 = jz / c.dens;
    const double v15 = 1.5 * (c.u0 * c.u0 + c.u1 * c.u1 + c.u2 * c.u2);
    const double wd[3] = {(1. / 3.) * c.dens, (1. / 18.) * c.dens, (1. / 36.) * c.dens};
    const double wc[3] = {1. / 3., 1. / 18., 1. / 36.};
    const double m3 = 3. * (0. - c.u0), p3 = 3. * (1. - c.u0), n3 = 3. * (-1. - c.u0);
#pragma unroll
    for (int a = 0; a < Q; ++a) {
        double u;
        switch (a) {  // unrolled: one case survives per a
#define EU(A) case A: u = f64_eu<A>(c.u0, c.u1, c.u2); break;
            EU(0) EU(1) EU(2) EU(3) EU(4) EU(5) EU(6) EU(7) EU(8) EU(9)
            EU(10) EU(11) EU(12) EU(13) EU(14) EU(15) EU(16) EU(17) EU(18)
#undef EU
        }
        const double t = ((1. + 3. * u) + (4.5 * u) * u) - v15;
        const double feq = wd[lat_wclass(a)] * t;
        const double br = lat_ex(a) == 0 ? m3 : lat_ex(a) > 0 ? p3 + 9. * u : n3 - 9. * u;
        const double Fi = (wc[lat_wclass(a)] * br) * G;
        f[a] = f[a] + (Fi - omega * (f[a] - feq));
    }
    return c;
}

}  // namespace dnslbm
