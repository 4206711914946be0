// Compile-time D3Q19 / D3Q15 lattices.
//
// Direction order, velocities, weights and `opposite` are those of
// FlowCraft/LatticeModel.h:20-43 (D3Q19) and :45-64 (D3Q15): parity with the
// reference depends on the order because every moment sum runs over
// directions in index order. The Y / Z reflection tables are the ones the
// reference finds by search at init (LbmReference.cpp:168-183); here they
// are resolved at compile time.
#pragma once

#include <cstdint>
#include <type_traits>

namespace fc {

template <int Q>
struct Lattice;

template <>
struct Lattice<19> {
    static constexpr int kQ = 19;
    __host__ __device__ static constexpr int ex(int i) {
        constexpr int t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
        return t[i];
    }
    __host__ __device__ static constexpr int ey(int i) {
        constexpr int t[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
        return t[i];
    }
    __host__ __device__ static constexpr int ez(int i) {
        constexpr int t[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
        return t[i];
    }
    __host__ __device__ static constexpr int opp(int i) {
        constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
        return t[i];
    }
    // Float weights computed exactly as the reference spells them
    // (1.0f / 3.0f, 1.0f / 18.0f, 1.0f / 36.0f).
    __host__ __device__ static constexpr float w(int i) {
        return i == 0 ? 1.0f / 3.0f : (i < 7 ? 1.0f / 18.0f : 1.0f / 36.0f);
    }
};

template <>
struct Lattice<15> {
    static constexpr int kQ = 15;
    __host__ __device__ static constexpr int ex(int i) {
        constexpr int t[15] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
        return t[i];
    }
    __host__ __device__ static constexpr int ey(int i) {
        constexpr int t[15] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1};
        return t[i];
    }
    __host__ __device__ static constexpr int ez(int i) {
        constexpr int t[15] = {0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1, 1, -1};
        return t[i];
    }
    __host__ __device__ static constexpr int opp(int i) {
        constexpr int t[15] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13};
        return t[i];
    }
    __host__ __device__ static constexpr float w(int i) {
        return i == 0 ? 2.0f / 9.0f : (i < 7 ? 1.0f / 9.0f : 1.0f / 72.0f);
    }
};

// Reflection of direction i across a Y-normal (mirror_y) or Z-normal
// (mirror_z) plane: the direction with the same velocity but that one
// component negated.
template <int Q>
__host__ __device__ constexpr int mirror_y(int i) {
    using L = Lattice<Q>;
    for (int j = 0; j < Q; ++j)
        if (L::ex(j) == L::ex(i) && L::ey(j) == -L::ey(i) && L::ez(j) == L::ez(i)) return j;
    return L::opp(i);
}
template <int Q>
__host__ __device__ constexpr int mirror_z(int i) {
    using L = Lattice<Q>;
    for (int j = 0; j < Q; ++j)
        if (L::ex(j) == L::ex(i) && L::ey(j) == L::ey(i) && L::ez(j) == -L::ez(i)) return j;
    return L::opp(i);
}

// Unrolled loop over I = B..E-1 with I available as a constant expression.
template <int B, int E, class F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

}  // namespace fc
