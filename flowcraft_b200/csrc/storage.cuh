// Population storage formats in HBM.
//
// StoreF32 keeps f_i as is (152 B per D3Q19 cell update, read + write).
// StoreF16 / StoreBF16 keep the offset (f_i - w_i) scaled by 2^8 in 16 bits
// (76 B per D3Q19 cell update): near equilibrium f_i - w_i is O(w_i * Ma),
// so the 16-bit mantissa spends its bits on the deviation rather than on the
// constant weight, and the 2^8 scale lifts that deviation out of FP16's
// subnormal range. All collision arithmetic stays FP32.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "lattice.cuh"

namespace fc {

constexpr float kOffsetScale = 256.0f;
constexpr float kOffsetScaleInv = 1.0f / 256.0f;

struct StoreF32 {
    using T = float;
    static constexpr int kBytes = 4;
    __device__ __forceinline__ static float dec(T v, float /*w*/) { return v; }
    __device__ __forceinline__ static T enc(float f, float /*w*/) { return f; }
    __device__ __forceinline__ static T ld(const T* p) { return __ldg(p); }
};

struct StoreF16 {
    using T = __half;
    static constexpr int kBytes = 2;
    __device__ __forceinline__ static float dec(T v, float w) { return w + __half2float(v) * kOffsetScaleInv; }
    __device__ __forceinline__ static T enc(float f, float w) { return __float2half_rn((f - w) * kOffsetScale); }
    __device__ __forceinline__ static T ld(const T* p) { return __ldg(p); }
};

struct StoreBF16 {
    using T = __nv_bfloat16;
    static constexpr int kBytes = 2;
    __device__ __forceinline__ static float dec(T v, float w) { return w + __bfloat162float(v) * kOffsetScaleInv; }
    __device__ __forceinline__ static T enc(float f, float w) { return __float2bfloat16_rn((f - w) * kOffsetScale); }
    __device__ __forceinline__ static T ld(const T* p) { return __ldg(p); }
};

// Population i of `cell` in an SoA plane set with plane stride n.
template <int Q, class S>
__device__ __forceinline__ float load_pop(const typename S::T* __restrict__ f, int i, size_t n, size_t cell) {
    return S::dec(S::ld(f + (size_t)i * n + cell), Lattice<Q>::w(i));
}

template <int Q, class S, int I>
__device__ __forceinline__ float load_pop_c(const typename S::T* __restrict__ f, size_t n, size_t cell) {
    return S::dec(S::ld(f + (size_t)I * n + cell), Lattice<Q>::w(I));
}

template <int Q, class S, int I>
__device__ __forceinline__ void store_pop_c(typename S::T* __restrict__ f, size_t n, size_t cell, float v) {
    f[(size_t)I * n + cell] = S::enc(v, Lattice<Q>::w(I));
}

}  // namespace fc
