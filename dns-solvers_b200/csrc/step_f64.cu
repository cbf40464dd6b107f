// Plain FP64 fused step (collide + stream + wall rules + periodic wrap +
// per-step reductions), AA pattern, one launch per time step.
//
// Every floating-point operation of the collision keeps the reference's
// operand order (xcomputations.c:314-342) and this file is compiled with
// -fmad=false, so on a grid the reference can express the populations after
// any number of constant-g steps are bit-identical to the reference's.
// Zero terms of the reference's sums (E*f with E == 0) are omitted: adding a
// signed zero to a non-zero partial sum leaves it unchanged.
#include "step_common.cuh"

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

template <int A, bool ODD>
__device__ __forceinline__ double *f64_ptr(const StepArgs &p, const Nbr &n, int wall, unsigned bits)
{
    int slot, idx;
    aa_address<A, ODD>(n, wall, bits, slot, idx);
    return static_cast<double *>(p.pop[slot]) + idx;
}

template <bool ODD, bool CONSTQ, bool TEXTURED>
__global__ void __launch_bounds__(128, 4) step_f64_kernel(const StepArgs p)
{
    const long long step = *p.step_ctr;
    const double G = CONSTQ ? p.force[step & 1] : p.gx;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.z;
    const int wall = z == 0 ? -1 : (z == p.nz - 1 ? 1 : 0);
    const double c0 = p.shift[(size_t)(step & 1) * p.nz * 3 + z * 3 + 0];
    const double c1 = p.shift[(size_t)(step & 1) * p.nz * 3 + z * 3 + 1];
    const double c2 = p.shift[(size_t)(step & 1) * p.nz * 3 + z * 3 + 2];
    double acc[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i] = 0.0;

    if (x < p.nx) {
        const int y0 = blockIdx.y * p.rows;
        const int y1 = min(y0 + p.rows, p.ny);
        for (int y = y0; y < y1; ++y) {
            const Nbr n = make_nbr(x, y, z, p.nx, p.ny);
            unsigned bits = 0x1fu;
            if (TEXTURED && wall != 0) bits = p.wallmask[(size_t)(wall > 0) * p.nx * p.ny + y * p.nx + x];
            double f[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                double *q;
                switch (a) {
#define PT(A) case A: q = f64_ptr<A, ODD>(p, n, wall, bits); break;
                    PT(0) PT(1) PT(2) PT(3) PT(4) PT(5) PT(6) PT(7) PT(8) PT(9)
                    PT(10) PT(11) PT(12) PT(13) PT(14) PT(15) PT(16) PT(17) PT(18)
#undef PT
                }
                f[ODD ? lat_opp(a) : a] = *q;
            }
            const F64Cell c = f64_collide(f, p.omega, G);
            acc[0] += c.dens;
            acc[1] += c.jx;
            acc[2] += c.u0;
            acc[3] += c.u1;
            acc[4] += c.u2;
            {
                const double d0 = c.u0 - c0, d1 = c.u1 - c1, d2 = c.u2 - c2;
                acc[5] += d0 * d0 + d1 * d1 + d2 * d2;
            }
            if (CONSTQ) {
                double s = 0.0, m = 0.0;
#pragma unroll
                for (int a = 0; a < Q; ++a) {
                    s += f[a];
                    if (lat_ex(a) > 0) m += f[a];
                    if (lat_ex(a) < 0) m -= f[a];
                }
                // links that bounce back arrive with e_x reversed
                if (wall != 0) {
                    const int ap = wall < 0 ? 12 : 11, am = wall < 0 ? 13 : 14;  // e_x = +1 / -1 into the wall
                    if (bits & 2u) m -= 2. * f[ap];
                    if (bits & 4u) m += 2. * f[am];
                }
                acc[6] += s;
                acc[7] += m;
            }
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                double *q;
                switch (a) {
#define PT(A) case A: q = f64_ptr<A, ODD>(p, n, wall, bits); break;
                    PT(0) PT(1) PT(2) PT(3) PT(4) PT(5) PT(6) PT(7) PT(8) PT(9)
                    PT(10) PT(11) PT(12) PT(13) PT(14) PT(15) PT(16) PT(17) PT(18)
#undef PT
                }
                *q = f[ODD ? a : lat_opp(a)];
            }
        }
    }
    block_epilogue(p, acc, step, G, 0);
}

// Reader-only reduction of the current state (after a load/init): force and
// plane means for the first step.  Reads the natural layout.
__global__ void __launch_bounds__(128) reduce_f64_kernel(const StepArgs p)
{
    const long long step = *p.step_ctr;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.z;
    double acc[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i] = 0.0;
    if (x < p.nx) {
        const int y0 = blockIdx.y * p.rows;
        const int y1 = min(y0 + p.rows, p.ny);
        for (int y = y0; y < y1; ++y) {
            const int c = (z * p.ny + y) * p.nx + x;
            double f[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a) f[a] = static_cast<const double *>(p.pop[a])[c];
            double dens, jx, jy, jz;
            f64_moments(f, dens, jx, jy, jz);
            acc[0] += dens;
            acc[1] += jx;
            acc[2] += jx / dens;
            acc[3] += jy / dens;
            acc[4] += jz / dens;
        }
    }
    block_epilogue(p, acc, step, 0.0, 1);
}

void launch_step_f64(const StepArgs &p, dim3 grid, dim3 block, bool odd, bool textured, cudaStream_t s)
{
    const bool q = p.const_q != 0;
#define L(O, C, T) step_f64_kernel<O, C, T><<<grid, block, 0, s>>>(p)
    if (odd) {
        if (q) { if (textured) L(true, true, true); else L(true, true, false); }
        else   { if (textured) L(true, false, true); else L(true, false, false); }
    } else {
        if (q) { if (textured) L(false, true, true); else L(false, true, false); }
        else   { if (textured) L(false, false, true); else L(false, false, false); }
    }
#undef L
}

void launch_reduce_f64(const StepArgs &p, dim3 grid, dim3 block, cudaStream_t s)
{
    reduce_f64_kernel<<<grid, block, 0, s>>>(p);
}

}  // namespace dnslbm
