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

// Moments and Pi_neq of two cells, the first half of the offset-space
// collision: everything the relaxation needs once the populations are spent.
struct Mom2 {
    float2 drho, rho, inv, ux, uy, uz, u2;
    float2 pxx, pyy, pzz, pxy, pxz, pyz, pp;  // Pi_neq and Pi:Pi
};

// Returns the two-bit divergence mask (bit 0: cell A, bit 1: cell B).
template <int Q>
__device__ __forceinline__ unsigned moments2(const float2 (&h)[Q], Mom2& mo) {
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
    mo.drho = mul2(m, bc2(si));
    mo.rho = add2(bc2(1.0f), mo.drho);
    mo.inv.x = mo.rho.x > 1e-6f ? __fdividef(1.0f, mo.rho.x) : 1.0f;
    mo.inv.y = mo.rho.y > 1e-6f ? __fdividef(1.0f, mo.rho.y) : 1.0f;
    const float2 isi = mul2(mo.inv, bc2(si));
    mo.ux = mul2(jx, isi), mo.uy = mul2(jy, isi), mo.uz = mul2(jz, isi);
    mo.u2 = fma2(mo.ux, mo.ux, fma2(mo.uy, mo.uy, mul2(mo.uz, mo.uz)));
    const float2 rho = mo.rho, u2 = mo.u2;
    // bit 0: cell A trips the divergence test, bit 1: cell B
    const unsigned bad = (rho.x > 0.0f && rho.x < __int_as_float(0x7f800000) && u2.x <= 4.0f ? 0u : 1u) |
                         (rho.y > 0.0f && rho.y < __int_as_float(0x7f800000) && u2.y <= 4.0f ? 0u : 2u);

    // Pi_neq = 2^-8 S - drho/3 I - rho u u, with the negations folded into
    // constants so every step is one FFMA2 / FMUL2
    constexpr float third = 1.0f / 3.0f;
    const float2 nd3 = mul2(mo.drho, bc2(-third));
    const float2 nrho = mul2(rho, bc2(-1.0f));
    const float2 nrux = mul2(nrho, mo.ux), nruy = mul2(nrho, mo.uy);
    mo.pxx = fma2(nrux, mo.ux, fma2(sxx, bc2(si), nd3));
    mo.pyy = fma2(nruy, mo.uy, fma2(syy, bc2(si), nd3));
    mo.pzz = fma2(mul2(nrho, mo.uz), mo.uz, fma2(szz, bc2(si), nd3));
    mo.pxy = fma2(nrux, mo.uy, mul2(sxy, bc2(si)));
    mo.pxz = fma2(nrux, mo.uz, mul2(sxz, bc2(si)));
    mo.pyz = fma2(nruy, mo.uz, mul2(syz, bc2(si)));
    const float2 off = fma2(mo.pxy, mo.pxy, fma2(mo.pxz, mo.pxz, mul2(mo.pyz, mo.pyz)));
    mo.pp = fma2(mo.pxx, mo.pxx, fma2(mo.pyy, mo.pyy, fma2(mo.pzz, mo.pzz, mul2(bc2(2.0f), off))));
    return bad;
}

// Relaxation factor g = (1 - 1/tau_eff) * 4.5 of one cell under the
// Smagorinsky closure, tau_eff = (tau + sqrt(tau^2 + 18 sqrt2 Cs^2 |Pi|/rho))/2
// (LbmReference.cpp:439-444).
__device__ __forceinline__ float smagorinsky_g(float pp, float rho, float inv, float tau, float cs) {
    const float k0 = (18.0f * 1.41421356f) * cs * cs;
    const float pim = pp > 0.0f ? pp * rsqrtf(pp) : 0.0f;
    const float t2 = fmaf(k0, pim * (rho < 1e-6f ? 1e6f : inv), tau * tau);
    return (1.0f - __fdividef(2.0f, tau + t2 * rsqrtf(t2))) * 4.5f;
}

// 3 nu_t = tau_eff - tau of one cell under the Smagorinsky closure, from the
// same operations as smagorinsky_g (the learned closure's anchor).
__device__ __forceinline__ float smagorinsky_d3(float pp, float rho, float inv, float tau, float cs) {
    const float k0 = (18.0f * 1.41421356f) * cs * cs;
    const float pim = pp > 0.0f ? pp * rsqrtf(pp) : 0.0f;
    const float t2 = fmaf(k0, pim * (rho < 1e-6f ? 1e6f : inv), tau * tau);
    return fmaf(0.5f, tau + t2 * rsqrtf(t2), -tau);
}

// Second half: post-collision offsets of both cells from their moments and
// relaxation factors g.
template <int Q>
__device__ __forceinline__ void relax2(float2 (&h)[Q], const Mom2& mo, float2 g) {
    using L = Lattice<Q>;
    constexpr int NP = (Q - 1) / 2;
    constexpr float third = 1.0f / 3.0f;
    const float2 rho = mo.rho;
    const float2 ntr3 = mul2(add2(add2(mo.pxx, mo.pyy), mo.pzz), bc2(-third));  // -tr/3
    const float2 a = fma2(mul2(bc2(-1.5f), rho), mo.u2, mo.drho);              // drho - 1.5 rho u^2
    h[0] = mul2(bc2(256.0f * L::w(0)), fma2(g, ntr3, a));
    static_for<0, NP>([&](auto P) {
        constexpr int i = 2 * decltype(P)::value + 1;
        constexpr int o = i + 1;
        static_assert(L::opp(i) == o, "direction pairs must be adjacent");
        constexpr int X = L::ex(i), Y = L::ey(i), Z = L::ez(i);
        constexpr float ws = 256.0f * L::w(i);
        constexpr bool flip = !lead_positive<Q>(i);  // then o leads positive
        const float2 eu = edotu2<Q, flip ? o : i>(mo.ux, mo.uy, mo.uz);
        const float2 re = mul2(rho, eu);
        const float2 base = fma2(mul2(bc2(4.5f), re), eu, a);
        float2 qp = ntr3;
        if constexpr (X != 0) qp = add2(qp, mo.pxx);
        if constexpr (Y != 0) qp = add2(qp, mo.pyy);
        if constexpr (Z != 0) qp = add2(qp, mo.pzz);
        if constexpr (X * Y != 0) qp = fma2(bc2(2.0f * (float)(X * Y)), mo.pxy, qp);
        if constexpr (X * Z != 0) qp = fma2(bc2(2.0f * (float)(X * Z)), mo.pxz, qp);
        if constexpr (Y * Z != 0) qp = fma2(bc2(2.0f * (float)(Y * Z)), mo.pyz, qp);
        const float2 r = mul2(bc2(ws), fma2(g, qp, base));
        const float2 s = mul2(bc2(3.0f * ws), re);
        h[flip ? o : i] = add2(r, s);
        h[flip ? i : o] = sub2(r, s);
    });
}

// Offset-space collision (collide_offsets) for two cells with FFMA2.
template <int Q>
__device__ __forceinline__ unsigned collide_offsets2(float2 (&h)[Q], float tau, float cs) {
    Mom2 mo;
    const unsigned bad = moments2<Q>(h, mo);
    const float2 g = make_float2(smagorinsky_g(mo.pp.x, mo.rho.x, mo.inv.x, tau, cs),
                                 smagorinsky_g(mo.pp.y, mo.rho.y, mo.inv.y, tau, cs));
    relax2<Q>(h, mo, g);
    return bad;
}

}  // namespace fc
