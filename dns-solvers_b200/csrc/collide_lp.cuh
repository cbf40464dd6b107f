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
    const float inv = iS / rho;
    c.jx = jx * iS;
    c.u0 = jx * inv;
    c.u1 = jy * inv;
    c.u2 = jz * inv;
    const float usq15 = 1.5f * (c.u0 * c.u0 + c.u1 * c.u1 + c.u2 * c.u2);
    const float Srho = S * rho, SG = S * G, om1 = 1.f - omega;
    // rest direction
    {
        constexpr float w = 1.f / 3.f;
        r[0] = fmaf(om1, r[0], w * (omega * fmaf(Srho, -usq15, dr) - 3.f * SG * c.u0));
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int a = pair_dir(k), b = lat_opp(a);
        const float w = lat_wf(a);
        const float eu = (float)lat_ex(a) * c.u0 + (float)lat_ey(a) * c.u1 + (float)lat_ez(a) * c.u2;
        const float t = fmaf(4.5f * eu, eu, -usq15);
        const float A = w * (omega * fmaf(Srho, t, dr) + SG * fmaf(9.f * (float)lat_ex(a), eu, -3.f * c.u0));
        const float B = w * (omega * 3.f * Srho * eu + 3.f * SG * (float)lat_ex(a));
        r[a] = fmaf(om1, r[a], A + B);
        r[b] = fmaf(om1, r[b], A - B);
    }
    return c;
}

}  // namespace dnslbm
