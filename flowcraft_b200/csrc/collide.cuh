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
