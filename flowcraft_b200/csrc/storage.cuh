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
    using T2 = float2;  // two x-adjacent cells of one plane
    static constexpr int kBytes = 4;
    static constexpr bool kExact = true;  // bit-for-bit with the reference
    __device__ __forceinline__ static float dec(T v, float /*w*/) { return v; }
    __device__ __forceinline__ static T enc(float f, float /*w*/) { return f; }
    __device__ __forceinline__ static T ld(const T* p) { return __ldg(p); }
    __device__ __forceinline__ static float2 dec2(T2 v, float /*w*/) { return v; }
    __device__ __forceinline__ static T2 enc2(float a, float b, float /*w*/) { return make_float2(a, b); }
    __device__ __forceinline__ static T2 ld2(const T* p) { return __ldg(reinterpret_cast<const T2*>(p)); }
};

// The 16-bit formats also expose their stored values as plain floats (the
// scaled offsets h = (f - w) * 2^8) for kernels that collide in offset space.
struct StoreF16 {
    using T = __half;
    using T2 = __half2;
    static constexpr int kBytes = 2;
    static constexpr bool kExact = false;
    __device__ __forceinline__ static float2 dec2(T2 v, float w) {
        const float2 h = __half22float2(v);
        return make_float2(fmaf(h.x, kOffsetScaleInv, w), fmaf(h.y, kOffsetScaleInv, w));
    }
    __device__ __forceinline__ static T2 enc2(float a, float b, float w) {
        return __floats2half2_rn(fmaf(a, kOffsetScale, -w * kOffsetScale), fmaf(b, kOffsetScale, -w * kOffsetScale));
    }
    __device__ __forceinline__ static T2 ld2(const T* p) { return __ldg(reinterpret_cast<const T2*>(p)); }
    __device__ __forceinline__ static float raw(T v) { return __half2float(v); }
    __device__ __forceinline__ static float2 raw2(T2 v) { return __half22float2(v); }
    __device__ __forceinline__ static T2 pack2(float a, float b) { return __floats2half2_rn(a, b); }
    __device__ __forceinline__ static float dec(T v, float w) { return fmaf(__half2float(v), kOffsetScaleInv, w); }
    __device__ __forceinline__ static T enc(float f, float w) {
        return __float2half_rn(fmaf(f, kOffsetScale, -w * kOffsetScale));
    }
    __device__ __forceinline__ static T ld(const T* p) { return __ldg(p); }
};

struct StoreBF16 {
    using T = __nv_bfloat16;
    using T2 = __nv_bfloat162;
    static constexpr int kBytes = 2;
    static constexpr bool kExact = false;
    __device__ __forceinline__ static float2 dec2(T2 v, float w) {
        const float2 h = __bfloat1622float2(v);
        return make_float2(fmaf(h.x, kOffsetScaleInv, w), fmaf(h.y, kOffsetScaleInv, w));
    }
    __device__ __forceinline__ static T2 enc2(float a, float b, float w) {
        return __floats2bfloat162_rn(fmaf(a, kOffsetScale, -w * kOffsetScale), fmaf(b, kOffsetScale, -w * kOffsetScale));
    }
    __device__ __forceinline__ static T2 ld2(const T* p) { return __ldg(reinterpret_cast<const T2*>(p)); }
    __device__ __forceinline__ static float raw(T v) { return __bfloat162float(v); }
    __device__ __forceinline__ static float2 raw2(T2 v) { return __bfloat1622float2(v); }
    __device__ __forceinline__ static T2 pack2(float a, float b) { return __floats2bfloat162_rn(a, b); }
    __device__ __forceinline__ static float dec(T v, float w) { return fmaf(__bfloat162float(v), kOffsetScaleInv, w); }
    __device__ __forceinline__ static T enc(float f, float w) {
        return __float2bfloat16_rn(fmaf(f, kOffsetScale, -w * kOffsetScale));
    }
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

// Same with 32-bit cell indices relative to one plane's base pointer (cells
// per lattice are below 2^32, plane offsets are not).
template <int Q, class S, int I>
__device__ __forceinline__ float load_pop_i(const typename S::T* __restrict__ f, size_t n, uint32_t cell) {
    const typename S::T* plane = f + (size_t)I * n;
    return S::dec(S::ld(plane + cell), Lattice<Q>::w(I));
}

template <int Q, class S, int I>
__device__ __forceinline__ void store_pop_i(typename S::T* __restrict__ f, size_t n, uint32_t cell, float v) {
    typename S::T* plane = f + (size_t)I * n;
    plane[cell] = S::enc(v, Lattice<Q>::w(I));
}

template <int Q, class S, int I>
__device__ __forceinline__ void store_pop_c(typename S::T* __restrict__ f, size_t n, size_t cell, float v) {
    f[(size_t)I * n + cell] = S::enc(v, Lattice<Q>::w(I));
}

}  // namespace fc
