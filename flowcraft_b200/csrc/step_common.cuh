// Pieces shared by the step kernels (lbm_step.cu: ping-pong; lbm_step_aa.cu:
// one set streamed in place).
#pragma once

#include "collide.cuh"
#include "collide2.cuh"
#include "lbm_internal.h"
#include "storage.cuh"

#include <type_traits>

namespace fc {

constexpr int kBulkRows = 8;  // block = 32 x-lanes x 8 rows
constexpr int kBatchChunk = 8;  // consecutive tiles a block of the batch kernel takes at a time

template <int Q>
__device__ __forceinline__ long long link_offset(int i, const Geom& g) {
    return (long long)Lattice<Q>::ex(i) + (long long)Lattice<Q>::ey(i) * g.nx + (long long)Lattice<Q>::ez(i) * g.nxy;
}

// Source of population i for a fluid cell whose upstream neighbour is off
// the Y and/or Z edge (oy / oz): the free-slip mirror when every wall crossed
// is free-slip, else plain bounce-back (LbmReference.cpp:370-380). Returns the
// plane to read at the cell itself; every candidate has the weight of i.
template <int Q, int I>
__device__ __forceinline__ int edge_plane(bool oy, bool oz, const StepParams& p) {
    const bool mirror = (!oy || p.slip_y) && (!oz || p.slip_z);
    if (!mirror) return Lattice<Q>::opp(I);
    if (oy && oz) return mirror_z<Q>(mirror_y<Q>(I));
    return oy ? mirror_y<Q>(I) : mirror_z<Q>(I);
}

template <int Q, class S>
__device__ __forceinline__ float load_plane(const typename S::T* __restrict__ f, int plane, size_t n, size_t cell,
                                            float w) {
    return S::dec(S::ld(f + (size_t)plane * n + cell), w);
}

// Both cells of a pair through the collision the storage format uses;
// returns a two-bit divergence mask (bit 0: cell A, bit 1: cell B).
template <int Q, class S>
__device__ __forceinline__ unsigned collide_pair(float2 (&v)[Q], float tau, float cs) {
    if constexpr (S::kExact) {  // bit-exact path: the scalar reference-order collision per cell
        float a[Q], b[Q];
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            a[i] = v[i].x;
            b[i] = v[i].y;
        });
        const unsigned bad = (collide_regularized<Q>(a, tau, cs) ? 1u : 0u) | (collide_regularized<Q>(b, tau, cs) ? 2u : 0u);
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            v[i] = make_float2(a[i], b[i]);
        });
        return bad;
    } else {
        return collide_offsets2<Q>(v, tau, cs);
    }
}

// Lattice constants for a run-time direction i (lane i of a warp that
// shares one cell's populations): the weight, and each component of e_i from
// a table packed two bits per direction (component + 1).
template <int Q>
__device__ __forceinline__ float lattice_w_rt(unsigned i) {
    return i == 0 ? Lattice<Q>::w(0) : (i < 7 ? Lattice<Q>::w(1) : Lattice<Q>::w(Q - 1));
}

// Component `axis` of e_i for a run-time direction: the table packed two bits
// per direction (component + 1) into one compile-time constant.
template <int Q>
__host__ __device__ constexpr unsigned long long lattice_e_bits(int axis) {
    unsigned long long b = 0;
    for (int i = 0; i < Q; ++i) {
        const int e = axis == 0 ? Lattice<Q>::ex(i) : (axis == 1 ? Lattice<Q>::ey(i) : Lattice<Q>::ez(i));
        b |= (unsigned long long)(e + 1) << (2 * i);
    }
    return b;
}

template <int Q, int Axis>
__device__ __forceinline__ float lattice_e_rt(unsigned i) {
    constexpr unsigned long long bits = lattice_e_bits<Q>(Axis);
    return (float)((int)((bits >> (2 * i)) & 3ull) - 1);
}

// equilibrium<Q, I> for a run-time direction: e.u as ((ex ux + ey uy) + ez uz)
// with e in {-1, 0, 1}, which equals edotu's sum of the non-zero terms (a
// zero term adds +-0, and only the sign of a zero result can differ, which
// the equilibrium does not see), then the same operations.
template <int Q>
__device__ __forceinline__ float equilibrium_rt(unsigned i, float rho, float ux, float uy, float uz, float u2) {
    const float eu = (lattice_e_rt<Q, 0>(i) * ux + lattice_e_rt<Q, 1>(i) * uy) + lattice_e_rt<Q, 2>(i) * uz;
    return (lattice_w_rt<Q>(i) * rho) * (((1.0f + 3.0f * eu) + (4.5f * eu) * eu) - 1.5f * u2);
}

// Storage code of a format (0 FP32, 1 FP16 offset, 2 BF16 offset).
template <class S>
constexpr int storage_code() {
    return S::kBytes == 4 ? 0 : (std::is_same<S, StoreF16>::value ? 1 : 2);
}

}  // namespace fc
