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

// Storage code of a format (0 FP32, 1 FP16 offset, 2 BF16 offset).
template <class S>
constexpr int storage_code() {
    return S::kBytes == 4 ? 0 : (std::is_same<S, StoreF16>::value ? 1 : 2);
}

}  // namespace fc
