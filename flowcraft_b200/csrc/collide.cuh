// Per-cell LBM arithmetic: moments, second-order equilibrium and the
// regularized (Latt-Chopard) collision with a Smagorinsky relaxation time.
//
// Every expression keeps the operand association of FlowCraft's CPU solver
// (FlowCraft/LbmReference.cpp:9-13, :385-453) and this translation unit is
// compiled without FMA contraction, so in FP32 each rounding step matches the
// reference and the result is bit-identical. Terms whose lattice coefficient
// is zero are dropped at compile time: adding +-0 never changes an IEEE sum,
// and multiplying by +-1 is exact, so dropping them changes no bit while it
// removes most of the work the reference's generic loops do.
#pragma once

#include "lattice.cuh"

namespace fc {

// e_i . u with the reference association ((ex*ux + ey*uy) + ez*uz).
template <int Q, int I>
__device__ __forceinline__ float edotu(float ux, float uy, float uz) {
    constexpr int X = Lattice<Q>::ex(I), Y = Lattice<Q>::ey(I), Z = Lattice<Q>::ez(I);
    float s = 0.0f;
    if constexpr (X != 0) s = X > 0 ? ux : -ux;
    if constexpr (Y != 0) {
        if constexpr (X != 0)
            s = Y > 0 ? s + uy : s - uy;
        else
            s = Y > 0 ? uy : -uy;
    }
    if constexpr (Z != 0) {
        if constexpr (X != 0 || Y != 0)
            s = Z > 0 ? s + uz : s - uz;
        else
            s = Z > 0 ? uz : -uz;
    }
    return s;
}

// w*rho*(1 + 3eu + 4.5eu*eu - 1.5u2) as (w*rho)*(((1 + 3eu) + (4.5eu)eu) - 1.5u2)
// (LbmReference.cpp:9-13).
template <int Q, int I>
__device__ __forceinline__ float equilibrium(float rho, float ux, float uy, float uz, float u2) {
    constexpr float w = Lattice<Q>::w(I);
    const float eu = edotu<Q, I>(ux, uy, uz);
    return (w * rho) * (((1.0f + 3.0f * eu) + (4.5f * eu) * eu) - 1.5f * u2);
}

__device__ __forceinline__ float speed2(float ux, float uy, float uz) { return (ux * ux + uy * uy) + uz * uz; }

// Density and velocity, summing over directions in index order; velocity is
// divided by rho only when rho > 1e-6 (LbmReference.cpp:43-61, :385-396).
template <int Q>
__device__ __forceinline__ void moments(const float (&f)[Q], float& rho, float& ux, float& uy, float& uz) {
    float r = 0.0f, a = 0.0f, b = 0.0f, c = 0.0f;
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        constexpr int X = Lattice<Q>::ex(i), Y = Lattice<Q>::ey(i), Z = Lattice<Q>::ez(i);
        r = r + f[i];
        if constexpr (X > 0) a = a + f[i];
        if constexpr (X < 0) a = a - f[i];
        if constexpr (Y > 0) b = b + f[i];
        if constexpr (Y < 0) b = b - f[i];
        if constexpr (Z > 0) c = c + f[i];
        if constexpr (Z < 0) c = c - f[i];
    });
    if (r > 1e-6f) {
        a = a / r;
        b = b / r;
        c = c / r;
    }
    rho = r;
    ux = a;
    uy = b;
    uz = c;
}

// Equilibrium populations for given moments into out[].
template <int Q>
__device__ __forceinline__ void equilibrium_all(float rho, float ux, float uy, float uz, float (&out)[Q]) {
    const float u2 = speed2(ux, uy, uz);
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        out[i] = equilibrium<Q, i>(rho, ux, uy, uz, u2);
    });
}

// One regularized collision in place: f[] holds the streamed (pre-collision)
// populations on entry and the post-collision ones on exit
// (LbmReference.cpp:385-453). Returns true when the cell trips the
// reference's divergence test (non-finite, rho <= 0 or |u|^2 > 4,
// LbmReference.cpp:397-400).
template <int Q>
__device__ __forceinline__ bool collide_regularized(float (&f)[Q], float tau, float cs) {
    using L = Lattice<Q>;
    float rho, ux, uy, uz;
    moments<Q>(f, rho, ux, uy, uz);
    const float u2 = speed2(ux, uy, uz);
    const bool bad = !isfinite(rho) || !isfinite(ux) || !isfinite(uy) || !isfinite(uz) || rho <= 0.0f || u2 > 4.0f;

    float pxx = 0.0f, pyy = 0.0f, pzz = 0.0f, pxy = 0.0f, pxz = 0.0f, pyz = 0.0f;
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        constexpr int X = L::ex(i), Y = L::ey(i), Z = L::ez(i);
        const float e = equilibrium<Q, i>(rho, ux, uy, uz, u2);
        const float ne = f[i] - e;
        f[i] = e;  // keep feq; the raw value is not needed again
        if constexpr (X != 0) pxx = pxx + ne;
        if constexpr (Y != 0) pyy = pyy + ne;
        if constexpr (Z != 0) pzz = pzz + ne;
        if constexpr (X * Y > 0) pxy = pxy + ne;
        if constexpr (X * Y < 0) pxy = pxy - ne;
        if constexpr (X * Z > 0) pxz = pxz + ne;
        if constexpr (X * Z < 0) pxz = pxz - ne;
        if constexpr (Y * Z > 0) pyz = pyz + ne;
        if constexpr (Y * Z < 0) pyz = pyz - ne;
    });

    // Smagorinsky: tau_eff = (tau + sqrt(tau^2 + 18 sqrt2 Cs^2 |Pi| / rho)) / 2
    // with the reference's literal 1.41421356 and left-to-right products
    // (LbmReference.cpp:439-444).
    const float pimag =
        sqrtf(((pxx * pxx + pyy * pyy) + pzz * pzz) + 2.0f * ((pxy * pxy + pxz * pxz) + pyz * pyz));
    const float rden = (rho < 1e-6f) ? 1e-6f : rho;  // std::max(rho, 1e-6f), NaN passes through
    float t = 18.0f * 1.41421356f;
    t = t * cs;
    t = t * cs;
    t = t * pimag;
    t = t / rden;
    const float tau_eff = 0.5f * (tau + sqrtf(tau * tau + t));
    const float omega = 1.0f / tau_eff;
    const float om1 = 1.0f - omega;

    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        constexpr int X = L::ex(i), Y = L::ey(i), Z = L::ez(i);
        constexpr float cs2 = 1.0f / 3.0f;
        constexpr float qxx = (float)(X * X) - cs2;
        constexpr float qyy = (float)(Y * Y) - cs2;
        constexpr float qzz = (float)(Z * Z) - cs2;
        constexpr float w45 = L::w(i) * 4.5f;
        float s = qxx * pxx + qyy * pyy;
        s = s + qzz * pzz;
        if constexpr (X * Y != 0) s = s + (2.0f * (float)(X * Y)) * pxy;
        if constexpr (X * Z != 0) s = s + (2.0f * (float)(X * Z)) * pxz;
        if constexpr (Y * Z != 0) s = s + (2.0f * (float)(Y * Z)) * pyz;
        f[i] = f[i] + om1 * (w45 * s);
    });
    return bad;
}

}  // namespace fc

namespace fc {

// The same regularized + Smagorinsky collision, rearranged for throughput.
// Used with the 16-bit storage formats, whose accuracy is measured against the
// FP64 oracle rather than bit-for-bit; the FP32 format keeps
// collide_regularized.
//
//   * Pi_neq from raw second moments: sum_i feq_i e_a e_b = rho(c_s^2 d_ab +
//     u_a u_b) holds exactly for the second-order equilibrium on D3Q19 and
//     D3Q15 (both are fourth-order isotropic), so Pi_neq = sum_i f_i e_a e_b
//     - rho(d_ab/3 + u_a u_b) needs no equilibrium per direction;
//   * directions come in +-e pairs (i odd, opp(i) = i+1 in both tables):
//     feq_+- = w(rho(1 - 1.5u^2) + 4.5 rho eu^2 +- 3 rho eu) and both share
//     one regularized term, since Q_i = e_i e_i - I/3 is even in e;
//   * one approximate reciprocal of rho (the velocity is divided only when
//     rho > 1e-6, as in the reference, LbmReference.cpp:392-396), square
//     roots through rsqrtf, and FMA contraction written out with fmaf; the
//     relative error of these is ~1e-7, far below the 16-bit storage step.
template <int Q>
__device__ __forceinline__ bool collide_regularized_fast(float (&f)[Q], float tau, float cs) {
    using L = Lattice<Q>;
    constexpr int NP = (Q - 1) / 2;
    // Moments from +-e pair sums and differences: the pair (i, i+1) adds
    // sum = f_i + f_{i+1} to every even moment and +-(f_i - f_{i+1}) to the
    // odd ones.
    float sp[NP], dp[NP];
    static_for<0, NP>([&](auto P) {
        constexpr int k = decltype(P)::value, i = 2 * k + 1;
        sp[k] = f[i] + f[i + 1];
        dp[k] = f[i] - f[i + 1];
    });
    float rho = f[0];
    float jx = 0.0f, jy = 0.0f, jz = 0.0f;
    float sxx = 0.0f, syy = 0.0f, szz = 0.0f, sxy = 0.0f, sxz = 0.0f, syz = 0.0f;
    static_for<0, NP>([&](auto P) {
        constexpr int k = decltype(P)::value, i = 2 * k + 1;
        constexpr int X = L::ex(i), Y = L::ey(i), Z = L::ez(i);
        rho += sp[k];
        if constexpr (X > 0) jx += dp[k];
        if constexpr (X < 0) jx -= dp[k];
        if constexpr (Y > 0) jy += dp[k];
        if constexpr (Y < 0) jy -= dp[k];
        if constexpr (Z > 0) jz += dp[k];
        if constexpr (Z < 0) jz -= dp[k];
        if constexpr (X != 0) sxx += sp[k];
        if constexpr (Y != 0) syy += sp[k];
        if constexpr (Z != 0) szz += sp[k];
        if constexpr (X * Y > 0) sxy += sp[k];
        if constexpr (X * Y < 0) sxy -= sp[k];
        if constexpr (X * Z > 0) sxz += sp[k];
        if constexpr (X * Z < 0) sxz -= sp[k];
        if constexpr (Y * Z > 0) syz += sp[k];
        if constexpr (Y * Z < 0) syz -= sp[k];
    });
    const float inv = rho > 1e-6f ? __fdividef(1.0f, rho) : 1.0f;
    const float ux = jx * inv, uy = jy * inv, uz = jz * inv;
    const float u2 = fmaf(ux, ux, fmaf(uy, uy, uz * uz));
    // The reference's test (non-finite rho or u, rho <= 0, |u|^2 > 4) in three
    // comparisons: a NaN or infinite velocity makes u2 fail u2 <= 4.
    const bool bad = !(rho > 0.0f && rho < __int_as_float(0x7f800000) && u2 <= 4.0f);

    constexpr float third = 1.0f / 3.0f;
    const float rho3 = rho * third;
    const float pxx = sxx - fmaf(rho * ux, ux, rho3);
    const float pyy = syy - fmaf(rho * uy, uy, rho3);
    const float pzz = szz - fmaf(rho * uz, uz, rho3);
    const float pxy = fmaf(-rho * ux, uy, sxy);
    const float pxz = fmaf(-rho * ux, uz, sxz);
    const float pyz = fmaf(-rho * uy, uz, syz);

    const float off = fmaf(pxy, pxy, fmaf(pxz, pxz, pyz * pyz));
    const float pp = fmaf(pxx, pxx, fmaf(pyy, pyy, fmaf(pzz, pzz, 2.0f * off)));
    const float pimag = pp > 0.0f ? pp * rsqrtf(pp) : 0.0f;
    const float rden = (rho < 1e-6f) ? 1e-6f : rho;
    const float k = __fdividef((18.0f * 1.41421356f) * cs * cs * pimag, rden);
    const float t2 = fmaf(tau, tau, k);  // > 0.25
    const float omega = __fdividef(2.0f, tau + t2 * rsqrtf(t2));
    const float g = (1.0f - omega) * 4.5f;  // regularized factor before w_i

    const float tr3 = (pxx + pyy + pzz) * third;
    const float a = rho * fmaf(-1.5f, u2, 1.0f);  // rho(1 - 1.5u^2)
    f[0] = L::w(0) * fmaf(g, -tr3, a);
    static_for<0, (Q - 1) / 2>([&](auto P) {
        constexpr int i = 2 * decltype(P)::value + 1;
        constexpr int o = i + 1;
        static_assert(L::opp(i) == o, "direction pairs must be adjacent");
        constexpr int X = L::ex(i), Y = L::ey(i), Z = L::ez(i);
        constexpr float w = L::w(i);
        const float eu = edotu<Q, i>(ux, uy, uz);
        const float re = rho * eu;
        const float base = fmaf(4.5f * re, eu, a);
        const float s = 3.0f * re;
        // Q_i : Pi_neq = e e : Pi - tr/3
        float qp = -tr3;
        if constexpr (X != 0) qp += pxx;
        if constexpr (Y != 0) qp += pyy;
        if constexpr (Z != 0) qp += pzz;
        if constexpr (X * Y != 0) qp = fmaf(2.0f * (float)(X * Y), pxy, qp);
        if constexpr (X * Z != 0) qp = fmaf(2.0f * (float)(X * Z), pxz, qp);
        if constexpr (Y * Z != 0) qp = fmaf(2.0f * (float)(Y * Z), pyz, qp);
        const float r = fmaf(g, qp, base);
        f[i] = w * (r + s);
        f[o] = w * (r - s);
    });
    return bad;
}

// Storage formats choose the collision: FP32 reproduces the reference bit
// for bit, the 16-bit offset formats take the rearranged form.
template <int Q, bool Exact>
__device__ __forceinline__ bool collide(float (&f)[Q], float tau, float cs) {
    if constexpr (Exact)
        return collide_regularized<Q>(f, tau, cs);
    else
        return collide_regularized_fast<Q>(f, tau, cs);
}

}  // namespace fc

namespace fc {

// The rearranged collision carried out directly on the stored 16-bit
// representation: h_i = (f_i - w_i) * 2^8 in, the post-collision h_i out.
// With sum_i w_i = 1, sum_i w_i e_i = 0 and sum_i w_i e_a e_b = d_ab / 3:
//   drho = rho - 1 = 2^-8 sum_i h_i,   j = 2^-8 sum_i h_i e_i,
//   Pi_neq = 2^-8 sum_i h_i e_a e_b - drho d_ab / 3 - rho u_a u_b,
//   feq_i - w_i = w_i (drho + rho (3 eu + 4.5 eu^2 - 1.5 u^2)).
// The offsets are never turned into populations: loading costs one
// conversion, storing one pack, the 2^-8 scale is applied to the ten moments
// only, and drho is accumulated without the cancellation of sum f_i - 1.
template <int Q>
__device__ __forceinline__ bool collide_offsets(float (&h)[Q], float tau, float cs) {
    using L = Lattice<Q>;
    constexpr int NP = (Q - 1) / 2;
    constexpr float si = 1.0f / 256.0f;
    float sp[NP], dp[NP];
    static_for<0, NP>([&](auto P) {
        constexpr int k = decltype(P)::value, i = 2 * k + 1;
        sp[k] = h[i] + h[i + 1];
        dp[k] = h[i] - h[i + 1];
    });
    float m = h[0];
    float jx = 0.0f, jy = 0.0f, jz = 0.0f;
    float sxx = 0.0f, syy = 0.0f, szz = 0.0f, sxy = 0.0f, sxz = 0.0f, syz = 0.0f;
    static_for<0, NP>([&](auto P) {
        constexpr int k = decltype(P)::value, i = 2 * k + 1;
        constexpr int X = L::ex(i), Y = L::ey(i), Z = L::ez(i);
        m += sp[k];
        if constexpr (X > 0) jx += dp[k];
        if constexpr (X < 0) jx -= dp[k];
        if constexpr (Y > 0) jy += dp[k];
        if constexpr (Y < 0) jy -= dp[k];
        if constexpr (Z > 0) jz += dp[k];
        if constexpr (Z < 0) jz -= dp[k];
        if constexpr (X != 0) sxx += sp[k];
        if constexpr (Y != 0) syy += sp[k];
        if constexpr (Z != 0) szz += sp[k];
        if constexpr (X * Y > 0) sxy += sp[k];
        if constexpr (X * Y < 0) sxy -= sp[k];
        if constexpr (X * Z > 0) sxz += sp[k];
        if constexpr (X * Z < 0) sxz -= sp[k];
        if constexpr (Y * Z > 0) syz += sp[k];
        if constexpr (Y * Z < 0) syz -= sp[k];
    });
    const float drho = m * si;
    const float rho = 1.0f + drho;
    const float inv = rho > 1e-6f ? __fdividef(1.0f, rho) : 1.0f;
    const float ux = (jx * si) * inv, uy = (jy * si) * inv, uz = (jz * si) * inv;
    const float u2 = fmaf(ux, ux, fmaf(uy, uy, uz * uz));
    const bool bad = !(rho > 0.0f && rho < __int_as_float(0x7f800000) && u2 <= 4.0f);

    constexpr float third = 1.0f / 3.0f;
    const float d3 = drho * third;
    const float rux = rho * ux, ruy = rho * uy;
    const float pxx = fmaf(sxx, si, -fmaf(rux, ux, d3));
    const float pyy = fmaf(syy, si, -fmaf(ruy, uy, d3));
    const float pzz = fmaf(szz, si, -fmaf(rho * uz, uz, d3));
    const float pxy = fmaf(sxy, si, -rux * uy);
    const float pxz = fmaf(sxz, si, -rux * uz);
    const float pyz = fmaf(syz, si, -ruy * uz);

    const float off = fmaf(pxy, pxy, fmaf(pxz, pxz, pyz * pyz));
    const float pp = fmaf(pxx, pxx, fmaf(pyy, pyy, fmaf(pzz, pzz, 2.0f * off)));
    const float pimag = pp > 0.0f ? pp * rsqrtf(pp) : 0.0f;
    const float rden = (rho < 1e-6f) ? 1e-6f : rho;
    const float kk = __fdividef((18.0f * 1.41421356f) * cs * cs * pimag, rden);
    const float t2 = fmaf(tau, tau, kk);
    const float omega = __fdividef(2.0f, tau + t2 * rsqrtf(t2));
    const float g = (1.0f - omega) * 4.5f;

    const float tr3 = (pxx + pyy + pzz) * third;
    const float a = fmaf(-1.5f * rho, u2, drho);  // drho - 1.5 rho u^2
    h[0] = (256.0f * L::w(0)) * fmaf(g, -tr3, a);
    static_for<0, NP>([&](auto P) {
        constexpr int i = 2 * decltype(P)::value + 1;
        constexpr int o = i + 1;
        static_assert(L::opp(i) == o, "direction pairs must be adjacent");
        constexpr int X = L::ex(i), Y = L::ey(i), Z = L::ez(i);
        constexpr float ws = 256.0f * L::w(i);
        const float eu = edotu<Q, i>(ux, uy, uz);
        const float re = rho * eu;
        const float base = fmaf(4.5f * re, eu, a);
        float qp = -tr3;
        if constexpr (X != 0) qp += pxx;
        if constexpr (Y != 0) qp += pyy;
        if constexpr (Z != 0) qp += pzz;
        if constexpr (X * Y != 0) qp = fmaf(2.0f * (float)(X * Y), pxy, qp);
        if constexpr (X * Z != 0) qp = fmaf(2.0f * (float)(X * Z), pxz, qp);
        if constexpr (Y * Z != 0) qp = fmaf(2.0f * (float)(Y * Z), pyz, qp);
        const float r = ws * fmaf(g, qp, base);
        const float s = (3.0f * ws) * re;
        h[i] = r + s;
        h[o] = r - s;
    });
    return bad;
}

}  // namespace fc
