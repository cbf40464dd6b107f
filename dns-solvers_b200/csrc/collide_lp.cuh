// Collision of deviation-stored populations in FP32.
//
// Storage holds raw values r_a = S * (f_a - w_a) with S = 1 (FP32) or 2^15
// (FP16; an exact power of two keeps deviations of 1e-7..2 normal in
// binary16).  The reference's BGK + forcing (xcomputations.c:314-342) in
// these variables, with dr = sum r_a, rho = 1 + dr/S, u = j/(S rho):
//   r_a' = (1-w) r_a + omega * S (feq_a - w_a) + S Fi_a
//   S (feq_a - w_a) = w_a (dr + S rho (3 e.u + 4.5 (e.u)^2 - 1.5 u.u))
//   S Fi_a          = w_a S G (3 (e_x - u_x) + 9 (e.u) e_x)
// Opposite directions a and abar share |e.u| and e_x -> -e_x, so each pair
// is computed from one symmetric part A and one antisymmetric part B:
//   r_a' = (1-w) r_a + A + B,  r_abar' = (1-w) r_abar + A - B.
//
// Two choices keep FP32 rounding from biasing the momentum, which a body
// force of 1e-7 per step makes visible (the bulk velocity of a long run):
//  * u = j/rho as j - j*(drho/rho): a rounded 1/rho times rho is not 1 on
//    average for rho just below 1 (the binade boundary), which biased the
//    equilibrium momentum by ~3e-8 relative, ~0.6 % of the force; in this
//    form the quotient's own error enters u scaled by drho ~ 1e-3;
//  * the two momentum coefficients 3 w omega of the axis and diagonal pairs
//    taken so that b1 + 4 b2 == omega / 2 exactly (their rounded products
//    otherwise carry a fixed relative error of the same size).
#pragma once

#include <cuda_fp16.h>

#include "lattice.cuh"

namespace dnslbm {

template <typename T> struct LpStore;
template <> struct LpStore<float> {
    static constexpr float kScale = 1.f, kInv = 1.f;
    static __device__ __forceinline__ float ld(const float *p) { return *p; }
    static __device__ __forceinline__ void st(float *p, float v) { *p = v; }
};
template <> struct LpStore<__half> {
    static constexpr float kScale = 32768.f, kInv = 1.f / 32768.f;
    static __device__ __forceinline__ float ld(const __half *p) { return __half2float(*p); }
    static __device__ __forceinline__ void st(__half *p, float v) { *p = __float2half_rn(v); }
};

__host__ __device__ __forceinline__ constexpr float lat_wf(int a)
{
    return a == 0 ? 1.f / 3.f : a <= 6 ? 1.f / 18.f : 1.f / 36.f;
}

// the nine direction pairs (a, opp a) with a the member listed first in
// globals.c order
__host__ __device__ __forceinline__ constexpr int pair_dir(int k)
{
    return k == 0 ? 1 : k == 1 ? 3 : k == 2 ? 5 : k == 3 ? 7 : k == 4 ? 8 : k == 5 ? 11 : k == 6 ? 12 : k == 7 ? 15 : 16;
}

struct LpCell {
    float drho, jx, u0, u1, u2;  // drho = rho - 1, jx unscaled
};

// e_a . u with every 0/+-1 factor resolved at compile time (a multiplication
// by a constant zero is not foldable under IEEE rules).
template <int A>
__device__ __forceinline__ float lp_eu(float u0, float u1, float u2)
{
    constexpr int ex = lat_ex(A), ey = lat_ey(A), ez = lat_ez(A);
    float s = 0.f;
    bool first = true;
    if (ex != 0) { s = ex > 0 ? u0 : -u0; first = false; }
    if (ey != 0) { s = first ? (ey > 0 ? u1 : -u1) : (ey > 0 ? s + u1 : s - u1); first = false; }
    if (ez != 0) { s = first ? (ez > 0 ? u2 : -u2) : (ez > 0 ? s + u2 : s - u2); }
    return s;
}

// Per-cell constants of the pair update, per weight class (1/18, 1/36).
struct LpConst {
    float dr, Srho, usq15, om1;
    float wom[2], a0[2], b_eu[2], b_ex[2], a_eu[2];
};

// Pair (a, opp a): A = w (omega (dr + S rho t) + S G (9 e_x e.u - 3 u_x)),
// B = w (3 omega S rho e.u + 3 S G e_x), t = 4.5 (e.u)^2 - 1.5 u.u.
template <int K>
__device__ __forceinline__ void lp_pair(float (&r)[Q], const LpConst &k, float u0, float u1, float u2)
{
    constexpr int a = pair_dir(K), b = lat_opp(pair_dir(K));
    constexpr int cls = lat_wclass(a) - 1;
    constexpr int ex = lat_ex(a);
    const float eu = lp_eu<a>(u0, u1, u2);
    const float t = fmaf(4.5f * eu, eu, -k.usq15);
    const float X = fmaf(k.Srho, t, k.dr);
    float A, B;
    if (ex == 0) {
        A = fmaf(k.wom[cls], X, k.a0[cls]);
        B = k.b_eu[cls] * eu;
    } else {
        A = fmaf(k.wom[cls], X, fmaf(ex > 0 ? k.a_eu[cls] : -k.a_eu[cls], eu, k.a0[cls]));
        B = fmaf(k.b_eu[cls], eu, ex > 0 ? k.b_ex[cls] : -k.b_ex[cls]);
    }
    r[a] = fmaf(k.om1, r[a], A + B);
    r[b] = fmaf(k.om1, r[b], A - B);
}

// In place on raw values r[19] of one storage type with scale S.
template <typename T>
__device__ __forceinline__ LpCell lp_collide(float (&r)[Q], float omega, float G)
{
    constexpr float S = LpStore<T>::kScale, iS = LpStore<T>::kInv;
    float sum[9], dif[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int a = pair_dir(k), b = lat_opp(pair_dir(k));
        sum[k] = r[a] + r[b];
        dif[k] = r[a] - r[b];
    }
    float dr = r[0];
#pragma unroll
    for (int k = 0; k < 9; ++k) dr += sum[k];
    float jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int a = pair_dir(k);
        if (lat_ex(a)) jx += lat_ex(a) > 0 ? dif[k] : -dif[k];
        if (lat_ey(a)) jy += lat_ey(a) > 0 ? dif[k] : -dif[k];
        if (lat_ez(a)) jz += lat_ez(a) > 0 ? dif[k] : -dif[k];
    }
    LpCell c;
    c.drho = dr * iS;
    const float rho = 1.f + c.drho;
    // drho/rho to ~2 ulp (fast reciprocal): its error reaches u scaled by drho
    const float dl = __fdividef(c.drho, rho);
    c.jx = jx * iS;
    const float jy_ = jy * iS, jz_ = jz * iS;
    c.u0 = fmaf(-c.jx, dl, c.jx);
    c.u1 = fmaf(-jy_, dl, jy_);
    c.u2 = fmaf(-jz_, dl, jz_);
    LpConst k;
    k.dr = dr;
    k.Srho = S * rho;
    k.usq15 = 1.5f * (c.u0 * c.u0 + c.u1 * c.u1 + c.u2 * c.u2);
    k.om1 = 1.f - omega;
    const float SG = S * G;
    const float bq2 = omega * (1.f / 12.f), bq1 = fmaf(-4.f, bq2, 0.5f * omega);  // bq1 + 4 bq2 == omega / 2
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const float w = q == 0 ? 1.f / 18.f : 1.f / 36.f;
        k.wom[q] = w * omega;
        k.a0[q] = -3.f * w * SG * c.u0;
        k.a_eu[q] = 9.f * w * SG;
        k.b_eu[q] = (q == 0 ? bq1 : bq2) * k.Srho;
        k.b_ex[q] = 3.f * w * SG;
    }
    // rest direction
    r[0] = fmaf(k.om1, r[0], (1.f / 3.f) * fmaf(omega, fmaf(k.Srho, -k.usq15, dr), -3.f * SG * c.u0));
    lp_pair<0>(r, k, c.u0, c.u1, c.u2);
    lp_pair<1>(r, k, c.u0, c.u1, c.u2);
    lp_pair<2>(r, k, c.u0, c.u1, c.u2);
    lp_pair<3>(r, k, c.u0, c.u1, c.u2);
    lp_pair<4>(r, k, c.u0, c.u1, c.u2);
    lp_pair<5>(r, k, c.u0, c.u1, c.u2);
    lp_pair<6>(r, k, c.u0, c.u1, c.u2);
    lp_pair<7>(r, k, c.u0, c.u1, c.u2);
    lp_pair<8>(r, k, c.u0, c.u1, c.u2);
    return c;
}

}  // namespace dnslbm
