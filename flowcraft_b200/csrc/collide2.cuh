// Two-cell collision with Blackwell's packed FP32x2 arithmetic, for the
// 16-bit offset formats.
//
// The two-cell interior kernel holds an x-adjacent pair of cells; every
// value below is a float2 with cell A in .x and cell B in .y, and each add,
// multiply or fused multiply-add is one FADD2 / FMUL2 / FFMA2 instruction for
// both cells, halving the arithmetic instruction count of the collision.
// (The FP32 format keeps the scalar reference-order collision per cell: a
// packed version of it was not bit-identical on the device, although each
// packed operation matched its scalar twin and a float32 emulation of the
// rearranged order matched the reference.)
#pragma once

#include "collide.cuh"

namespace fc {

__device__ __forceinline__ float2 bc2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// True when direction i's leading non-zero component is positive. Each +-e
// pair has exactly one such member; e.u is computed for it and the other
// member takes exactly -e.u (rounding to nearest is sign-symmetric).
template <int Q>
__host__ __device__ constexpr bool lead_positive(int i) {
    using L = Lattice<Q>;
    return L::ex(i) > 0 || (L::ex(i) == 0 && (L::ey(i) > 0 || (L::ey(i) == 0 && L::ez(i) > 0)));
}

// e_i . u for a direction whose leading non-zero component is positive;
// association and zero-term dropping as edotu.
template <int Q, int I>
__device__ __forceinline__ float2 edotu2(float2 ux, float2 uy, float2 uz) {
    constexpr int X = Lattice<Q>::ex(I), Y = Lattice<Q>::ey(I), Z = Lattice<Q>::ez(I);
    static_assert(X > 0 || (X == 0 && (Y > 0 || (Y == 0 && Z > 0))), "leading component must be positive");
    float2 s;
    if constexpr (X != 0) {
        s = ux;
        if constexpr (Y > 0) s = add2(s, uy);
        if constexpr (Y < 0) s = sub2(s, uy);
    } else if constexpr (Y != 0) {
        s = uy;
    } else {
        s = uz;
    }
    if constexpr ((X != 0 || Y != 0) && Z > 0) s = add2(s, uz);
    if constexpr ((X != 0 || Y != 0) && Z < 0) s = sub2(s, uz);
    return s;
}

// Offset-space collision (collide_offsets) for two cells with FFMA2.
template <int Q>
__device__ __forceinline__ unsigned collide_offsets2(float2 (&h)[Q], float tau, float cs) {
    using L = Lattice<Q>;
    constexpr int NP = (Q - 1) / 2;
    constexpr float si = 1.0f / 256.0f;
    float2 sp[NP], dp[NP];
    static_for<0, NP>([&](auto P) {
        constexpr int k = decltype(P)::value, i = 2 * k + 1;
        sp[k] = add2(h[i], h[i + 1]);
        dp[k] = sub2(h[i], h[i + 1]);
    });
    float2 m = h[0];
    float2 jx = bc2(0.0f), jy = bc2(0.0f), jz = bc2(0.0f);
    float2 sxx = bc2(0.0f), syy = bc2(0.0f), szz = bc2(0.0f), sxy = bc2(0.0f), sxz = bc2(0.0f), syz = bc2(0.0f);
    static_for<0, NP>([&](auto P) {
        constexpr int k = decltype(P)::value, i = 2 * k + 1;
        constexpr int X = L::ex(i), Y = L::ey(i), Z = L::ez(i);
        m = add2(m, sp[k]);
        if constexpr (X > 0) jx = add2(jx, dp[k]);
        if constexpr (X < 0) jx = sub2(jx, dp[k]);
        if constexpr (Y > 0) jy = add2(jy, dp[k]);
        if constexpr (Y < 0) jy = sub2(jy, dp[k]);
        if constexpr (Z > 0) jz = add2(jz, dp[k]);
        if constexpr (Z < 0) jz = sub2(jz, dp[k]);
        if constexpr (X != 0) sxx = add2(sxx, sp[k]);
        if constexpr (Y != 0) syy = add2(syy, sp[k]);
        if constexpr (Z != 0) szz = add2(szz, sp[k]);
        if constexpr (X * Y > 0) sxy = add2(sxy, sp[k]);
        if constexpr (X * Y < 0) sxy = sub2(sxy, sp[k]);
        if constexpr (X * Z > 0) sxz = add2(sxz, sp[k]);
        if constexpr (X * Z < 0) sxz = sub2(sxz, sp[k]);
        if constexpr (Y * Z > 0) syz = add2(syz, sp[k]);
        if constexpr (Y * Z < 0) syz = sub2(syz, sp[k]);
    });
    const float2 drho = mul2(m, bc2(si));
    const float2 rho = add2(bc2(1.0f), drho);
    float2 inv;
    inv.x = rho.x > 1e-6f ? __fdividef(1.0f, rho.x) : 1.0f;
    inv.y = rho.y > 1e-6f ? __fdividef(1.0f, rho.y) : 1.0f;
    const float2 isi = mul2(inv, bc2(si));
    const float2 ux = mul2(jx, isi), uy = mul2(jy, isi), uz = mul2(jz, isi);
    const float2 u2 = fma2(ux, ux, fma2(uy, uy, mul2(uz, uz)));
    // bit 0: cell A trips the divergence test, bit 1: cell B
    const unsigned bad = (rho.x > 0.0f && rho.x < __int_as_float(0x7f800000) && u2.x <= 4.0f ? 0u : 1u) |
                         (rho.y > 0.0f && rho.y < __int_as_float(0x7f800000) && u2.y <= 4.0f ? 0u : 2u);

    // Pi_neq = 2^-8 S - drho/3 I - rho u u, with the negations folded into
    // constants so every step is one FFMA2 / FMUL2
    constexpr float third = 1.0f / 3.0f;
    const float2 nd3 = mul2(drho, bc2(-third));
    const float2 nrho = mul2(rho, bc2(-1.0f));
    const float2 nrux = mul2(nrho, ux), nruy = mul2(nrho, uy);
    const float2 pxx = fma2(nrux, ux, fma2(sxx, bc2(si), nd3));
    const float2 pyy = fma2(nruy, uy, fma2(syy, bc2(si), nd3));
    const float2 pzz = fma2(mul2(nrho, uz), uz, fma2(szz, bc2(si), nd3));
    const float2 pxy = fma2(nrux, uy, mul2(sxy, bc2(si)));
    const float2 pxz = fma2(nrux, uz, mul2(sxz, bc2(si)));
    const float2 pyz = fma2(nruy, uz, mul2(syz, bc2(si)));

    const float2 off = fma2(pxy, pxy, fma2(pxz, pxz, mul2(pyz, pyz)));
    const float2 pp = fma2(pxx, pxx, fma2(pyy, pyy, fma2(pzz, pzz, mul2(bc2(2.0f), off))));
    float2 g;
    {
        const float k0 = (18.0f * 1.41421356f) * cs * cs;
        const float tt = tau * tau;
        float pim = pp.x > 0.0f ? pp.x * rsqrtf(pp.x) : 0.0f;
        float t2 = fmaf(k0, pim * (rho.x < 1e-6f ? 1e6f : inv.x), tt);
        g.x = (1.0f - __fdividef(2.0f, tau + t2 * rsqrtf(t2))) * 4.5f;
        pim = pp.y > 0.0f ? pp.y * rsqrtf(pp.y) : 0.0f;
        t2 = fmaf(k0, pim * (rho.y < 1e-6f ? 1e6f : inv.y), tt);
        g.y = (1.0f - __fdividef(2.0f, tau + t2 * rsqrtf(t2))) * 4.5f;
    }

    const float2 ntr3 = mul2(add2(add2(pxx, pyy), pzz), bc2(-third));  // -tr/3
    const float2 a = fma2(mul2(bc2(-1.5f), rho), u2, drho);            // drho - 1.5 rho u^2
    h[0] = mul2(bc2(256.0f * L::w(0)), fma2(g, ntr3, a));
    static_for<0, NP>([&](auto P) {
        constexpr int i = 2 * decltype(P)::value + 1;
        constexpr int o = i + 1;
        static_assert(L::opp(i) == o, "direction pairs must be adjacent");
        constexpr int X = L::ex(i), Y = L::ey(i), Z = L::ez(i);
        constexpr float ws = 256.0f * L::w(i);
        constexpr bool flip = !lead_positive<Q>(i);  // then o leads positive
        const float2 eu = edotu2<Q, flip ? o : i>(ux, uy, uz);
        const float2 re = mul2(rho, eu);
        const float2 base = fma2(mul2(bc2(4.5f), re), eu, a);
        float2 qp = ntr3;
        if constexpr (X != 0) qp = add2(qp, pxx);
        if constexpr (Y != 0) qp = add2(qp, pyy);
        if constexpr (Z != 0) qp = add2(qp, pzz);
        if constexpr (X * Y != 0) qp = fma2(bc2(2.0f * (float)(X * Y)), pxy, qp);
        if constexpr (X * Z != 0) qp = fma2(bc2(2.0f * (float)(X * Z)), pxz, qp);
        if constexpr (Y * Z != 0) qp = fma2(bc2(2.0f * (float)(Y * Z)), pyz, qp);
        const float2 r = mul2(bc2(ws), fma2(g, qp, base));
        const float2 s = mul2(bc2(3.0f * ws), re);
        h[flip ? o : i] = add2(r, s);
        h[flip ? i : o] = sub2(r, s);
    });
    return bad;
}

}  // namespace fc
