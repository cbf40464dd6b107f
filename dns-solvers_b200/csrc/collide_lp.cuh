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
//
// The collision is written once over a value type V: float (one cell) or
// float2 (two cells at once on the packed FP32 pipe of sm_100, fma/add/mul
// .f32x2).  Every operation is an explicitly rounded one (no contraction left
// to the compiler), so the two forms give bit-identical populations.
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

// ------------------------------------------------------------------ ops
__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float vsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float vmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float vneg(float a) { return -a; }
__device__ __forceinline__ float vdiv_fast(float a, float b) { return __fdividef(a, b); }

// The packed add, sub and mul are written in PTX: a product feeding a sum
// must stay two roundings (the compiler may otherwise fuse the packed
// intrinsics __fmul2_rn + __fadd2_rn into one fma, which the one-cell form,
// with __fmul_rn / __fadd_rn, never does).
#define DNSLBM_F32X2_OP(NAME, OP)                                                     \
    __device__ __forceinline__ float2 NAME(float2 a, float2 b)                        \
    {                                                                                 \
        float2 d;                                                                     \
        asm("{\n\t.reg .b64 ra, rb, rd;\n\t"                                      \
            "mov.b64 ra, {%2, %3};\n\t"                                             \
            "mov.b64 rb, {%4, %5};\n\t" OP " rd, ra, rb;\n\t"                     \
            "mov.b64 {%0, %1}, rd;\n\t}"                                            \
            : "=f"(d.x), "=f"(d.y)                                                    \
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                \
        return d;                                                                     \
    }
DNSLBM_F32X2_OP(vadd, "add.rn.f32x2")
DNSLBM_F32X2_OP(vsub, "sub.rn.f32x2")
DNSLBM_F32X2_OP(vmul, "mul.rn.f32x2")
#undef DNSLBM_F32X2_OP
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 vneg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 vdiv_fast(float2 a, float2 b)
{
    return make_float2(__fdividef(a.x, b.x), __fdividef(a.y, b.y));
}

template <typename V> __device__ __forceinline__ V vsplat(float s);
template <> __device__ __forceinline__ float vsplat<float>(float s) { return s; }
template <> __device__ __forceinline__ float2 vsplat<float2>(float s) { return make_float2(s, s); }

// ------------------------------------------------------------------ collision
// Per-launch constants (omega, the body force G and the storage scale),
// per weight class q (0: 1/18, 1: 1/36).
struct LpParams {
    float omega, om1, m3sg;  // m3sg = -3 S G
    float wom[2], a0c[2], a_eu[2], b_ex[2], bq[2];
};

template <typename T>
__device__ __forceinline__ LpParams lp_params(float omega, float G)
{
    constexpr float S = LpStore<T>::kScale;
    LpParams k;
    const float SG = __fmul_rn(S, G);
    k.omega = omega;
    k.om1 = __fsub_rn(1.f, omega);
    k.m3sg = __fmul_rn(-3.f, SG);
    const float bq2 = __fmul_rn(omega, 1.f / 12.f);
    k.bq[1] = bq2;
    k.bq[0] = __fmaf_rn(-4.f, bq2, __fmul_rn(0.5f, omega));  // bq1 + 4 bq2 == omega / 2
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const float w = q == 0 ? 1.f / 18.f : 1.f / 36.f;
        k.wom[q] = __fmul_rn(w, omega);
        k.a0c[q] = __fmul_rn(-3.f * w, SG);
        k.a_eu[q] = __fmul_rn(9.f * w, SG);
        k.b_ex[q] = __fmul_rn(3.f * w, SG);
    }
    return k;
}

template <typename V>
struct LpCellV {
    V drho, jx, u0, u1, u2;  // drho = rho - 1, jx unscaled
};
using LpCell = LpCellV<float>;

// e_a . u with every 0/+-1 factor resolved at compile time (a multiplication
// by a constant zero is not foldable under IEEE rules); round-to-nearest is
// symmetric in sign, so (-a) + b == b - a and (-a) - b == -(a + b) exactly.
template <int A, typename V>
__device__ __forceinline__ V lp_eu(V u0, V u1, V u2)
{
    constexpr int ex = lat_ex(A), ey = lat_ey(A), ez = lat_ez(A);
    V s = vsplat<V>(0.f);
    int sgn = 0;  // sign of s relative to the running sum: +1 s, -1 -s, 0 none yet
    auto add = [&](V u, int e) {
        if (e == 0) return;
        if (sgn == 0) { s = u; sgn = e; return; }
        if (sgn > 0) s = e > 0 ? vadd(s, u) : vsub(s, u);
        else if (e > 0) { s = vsub(u, s); sgn = 1; }
        else s = vadd(s, u);  // -(s + u)
    };
    add(u0, ex);
    add(u1, ey);
    add(u2, ez);
    return sgn < 0 ? vneg(s) : s;
}

// Pair (a, opp a): A = w (omega (dr + S rho t) + S G (9 e_x e.u - 3 u_x)),
// B = w (3 omega S rho e.u + 3 S G e_x), t = 4.5 (e.u)^2 - 1.5 u.u; for
// e_x = 0, A +- B is one fused multiply-add on A.
template <int K, typename V>
__device__ __forceinline__ void lp_pair(V (&r)[Q], const LpParams &k, V dr, V Srho, V nusq15, const V (&a0)[2],
                                        const V (&beu)[2], V u0, V u1, V u2)
{
    constexpr int a = pair_dir(K), b = lat_opp(pair_dir(K));
    constexpr int cls = lat_wclass(a) - 1;
    constexpr int ex = lat_ex(a);
    const V eu = lp_eu<a>(u0, u1, u2);
    const V t = vfma(vmul(vsplat<V>(4.5f), eu), eu, nusq15);
    const V X = vfma(Srho, t, dr);
    const V om1 = vsplat<V>(k.om1);
    if (ex == 0) {
        // A +- B with B = beu e.u as one fused operation each (a separate
        // product and sum is what the compiler may fuse on the packed pipe)
        const V A = vfma(vsplat<V>(k.wom[cls]), X, a0[cls]);
        r[a] = vfma(om1, r[a], vfma(beu[cls], eu, A));
        r[b] = vfma(om1, r[b], vfma(vneg(beu[cls]), eu, A));
    } else {
        const V A = vfma(vsplat<V>(k.wom[cls]), X, vfma(vsplat<V>(ex > 0 ? k.a_eu[cls] : -k.a_eu[cls]), eu, a0[cls]));
        const V B = vfma(beu[cls], eu, vsplat<V>(ex > 0 ? k.b_ex[cls] : -k.b_ex[cls]));
        r[a] = vfma(om1, r[a], vadd(A, B));
        r[b] = vfma(om1, r[b], vsub(A, B));
    }
}

// In place on raw values r[19] of one storage type with scale S.  emit(a)
// is called as soon as r[a] holds its post-collision value (so a caller can
// store it and free its registers early).
struct LpNoEmit {
    __device__ __forceinline__ void operator()(int) const {}
};

template <typename T, typename V, typename Emit = LpNoEmit>
__device__ __forceinline__ LpCellV<V> lp_collide_v(V (&r)[Q], const LpParams &k, Emit &&emit = Emit())
{
    constexpr float S = LpStore<T>::kScale, iS = LpStore<T>::kInv;
    V sum[9], dif[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int a = pair_dir(q), b = lat_opp(pair_dir(q));
        sum[q] = vadd(r[a], r[b]);
        dif[q] = vsub(r[a], r[b]);
    }
    V dr = r[0];
#pragma unroll
    for (int q = 0; q < 9; ++q) dr = vadd(dr, sum[q]);
    // momentum: the signed differences in pair order, first term taken as is
    V j[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        int sgn = 0;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const int a = pair_dir(q);
            const int e = d == 0 ? lat_ex(a) : d == 1 ? lat_ey(a) : lat_ez(a);
            if (e == 0) continue;
            if (sgn == 0) { j[d] = dif[q]; sgn = e; }
            else if (sgn > 0) j[d] = e > 0 ? vadd(j[d], dif[q]) : vsub(j[d], dif[q]);
            else if (e > 0) { j[d] = vsub(dif[q], j[d]); sgn = 1; }
            else j[d] = vadd(j[d], dif[q]);
        }
        if (sgn < 0) j[d] = vneg(j[d]);
    }
    LpCellV<V> c;
    c.drho = S == 1.f ? dr : vmul(dr, vsplat<V>(iS));
    const V rho = vadd(vsplat<V>(1.f), c.drho);
    // drho/rho to ~2 ulp (fast reciprocal): its error reaches u scaled by drho
    const V ndl = vneg(vdiv_fast(c.drho, rho));
    c.jx = S == 1.f ? j[0] : vmul(j[0], vsplat<V>(iS));
    const V jy = S == 1.f ? j[1] : vmul(j[1], vsplat<V>(iS));
    const V jz = S == 1.f ? j[2] : vmul(j[2], vsplat<V>(iS));
    c.u0 = vfma(c.jx, ndl, c.jx);
    c.u1 = vfma(jy, ndl, jy);
    c.u2 = vfma(jz, ndl, jz);
    const V Srho = S == 1.f ? rho : vmul(vsplat<V>(S), rho);
    const V usq = vfma(c.u2, c.u2, vfma(c.u1, c.u1, vmul(c.u0, c.u0)));
    const V nusq15 = vmul(vsplat<V>(-1.5f), usq);
    V a0[2], beu[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        a0[q] = vmul(vsplat<V>(k.a0c[q]), c.u0);
        beu[q] = vmul(vsplat<V>(k.bq[q]), Srho);
    }
    // rest direction
    r[0] = vfma(vsplat<V>(k.om1), r[0],
                vmul(vsplat<V>(1.f / 3.f), vfma(vsplat<V>(k.omega), vfma(Srho, nusq15, dr),
                                                vmul(vsplat<V>(k.m3sg), c.u0))));
    emit(0);
#define DNSLBM_PAIR(K)                                                 \
    lp_pair<K>(r, k, dr, Srho, nusq15, a0, beu, c.u0, c.u1, c.u2);     \
    emit(pair_dir(K));                                                 \
    emit(lat_opp(pair_dir(K)));
    DNSLBM_PAIR(0) DNSLBM_PAIR(1) DNSLBM_PAIR(2) DNSLBM_PAIR(3) DNSLBM_PAIR(4)
    DNSLBM_PAIR(5) DNSLBM_PAIR(6) DNSLBM_PAIR(7) DNSLBM_PAIR(8)
#undef DNSLBM_PAIR
    return c;
}

// One cell.
template <typename T>
__device__ __forceinline__ LpCell lp_collide(float (&r)[Q], float omega, float G)
{
    const LpParams k = lp_params<T>(omega, G);
    return lp_collide_v<T, float>(r, k);
}

}  // namespace dnslbm
