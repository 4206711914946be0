// Learned sub-grid closure fused into the collision: a per-cell MLP
// (5 inputs -> 32 -> 32 -> 1, ReLU) that predicts the eddy viscosity nu_t and
// replaces the constant-coefficient Smagorinsky closure of the regularized
// collision (LbmReference.cpp:439-444, lbm_step.comp.glsl:347-350).
//
// Inputs per cell, computed from the same moments the collision uses:
//   0  log2(|Pi_neq| / rho)            strain magnitude (Smagorinsky's input)
//   1  tr(Pi_neq) / |Pi_neq|           normalized first invariant
//   2  det(Pi_neq) / |Pi_neq|^3        normalized third invariant
//   3  wall distance in cells (1/16 cell steps, capped at 15.9)
//   4  filter width (per lattice)
// normalized by the training mean and standard deviation in FP32, then
// rounded to BF16.
//
// Inference runs on the tensor cores with the warp-level BF16 MMA
// (mma.sync m16n8k8 / m16n8k16, FP32 accumulate) over the 64 cells of a warp
// (two per lane) in four 16-cell row tiles. Each layer's FP32 accumulator
// fragment becomes the next layer's BF16 A fragment in registers (row r of
// the accumulator and of the A fragment sit in the same lanes), with the
// ReLU folded into the conversion (cvt.rn.relu.bf16x2.f32). Every
// accumulator starts at zero: the first layer's bias is the weight row of a
// constant input 1 (K slot 5), the second layer's bias one more K = 8 MMA of
// a constant-1 column, the output bias a single add, so no accumulator is
// ever filled by register copies. Weights are stored in fragment order, so
// each lane reads its own B fragments as 16-byte read-only loads that stay
// in L1 (5.6 KB shared by every warp of the SM); the only shared memory is
// per warp (the input transpose and the outputs), so no warp ever waits for
// another. The output nu_t = relu(z) (its scale folded into the last layer)
// gives tau_eff = tau + 3 nu_t. A cell whose invariants fall outside the
// training range keeps the Smagorinsky tau_eff.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "collide2.cuh"
#include "lbm_internal.h"

namespace fc {

__device__ __forceinline__ uint32_t pack_relu_bf16(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// d = A B (K = 8), accumulator from zero
__device__ __forceinline__ void mma_k8(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t b0) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%7,%7,%7,%7};"
        : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
        : "r"(a0), "r"(a1), "r"(b0), "f"(0.0f));
}

// d += A B (K = 8)
__device__ __forceinline__ void mma_k8_acc(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t b0) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(b0));
}

// d = A B (K = 16), accumulator from zero
__device__ __forceinline__ void mma_k16_z(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                          uint32_t b0, uint32_t b1) {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%10,%10,%10,%10};"
        : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1), "f"(0.0f));
}

// d += A B (K = 16)
__device__ __forceinline__ void mma_k16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                        uint32_t b0, uint32_t b1) {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Raw inputs 0-2 of one cell from its Pi_neq, |Pi|^2 (pp) and 1/rho.
// Input 0 alone; r receives 1/|Pi| for closure_x12.
__device__ __forceinline__ float closure_x0(float pp, float inv_rho, float& r) {
    r = pp > 0.0f ? rsqrtf(pp) : 0.0f;  // 1/|Pi|
    const float mag = pp * r;           // |Pi|
    return __log2f(fmaf(mag, inv_rho, 1e-12f));
}

// Inputs 1 and 2 from Pi_neq and r = 1/|Pi|.
__device__ __forceinline__ void closure_x12(float pxx, float pyy, float pzz, float pxy, float pxz, float pyz, float r,
                                            float& x1, float& x2) {
    x1 = (pxx + pyy + pzz) * r;
    const float det = pxx * fmaf(pyy, pzz, -pyz * pyz) - pxy * fmaf(pxy, pzz, -pyz * pxz) +
                      pxz * fmaf(pxy, pyz, -pyy * pxz);
    x2 = det * (r * r * r);
}

__device__ __forceinline__ void closure_invariants(float pxx, float pyy, float pzz, float pxy, float pxz, float pyz,
                                                   float pp, float inv_rho, float& x0, float& x1, float& x2) {
    float r;
    x0 = closure_x0(pp, inv_rho, r);
    closure_x12(pxx, pyy, pzz, pxy, pxz, pyz, r, x1, x2);
}

__device__ __forceinline__ bool closure_x0_in_range(const ClosureDev& cl, float x0) {
    return x0 >= cl.lo[0] && x0 <= cl.hi[0];
}

__device__ __forceinline__ bool closure_x12_in_range(const ClosureDev& cl, float x1, float x2) {
    return x1 >= cl.lo[1] && x1 <= cl.hi[1] && x2 >= cl.lo[2] && x2 <= cl.hi[2];
}

__device__ __forceinline__ bool closure_in_range(const ClosureDev& cl, float x0, float x1, float x2) {
    return closure_x0_in_range(cl, x0) && closure_x12_in_range(cl, x1, x2);
}

// The near-wall fallback: a cell whose wall-distance byte (1/16 cells) is
// below cl.wall_min keeps the Smagorinsky closure.
__device__ __forceinline__ bool closure_wall_ok(const ClosureDev& cl, unsigned wd) { return wd >= cl.wall_min; }

// True when the learned nu_t is held inside a band around the Smagorinsky
// value, so every covered cell also needs that value (smagorinsky_d3).
__device__ __forceinline__ bool closure_anchored(const ClosureDev& cl) { return cl.trust > 0.0f; }

// Relaxation factor g = (1 - 1/tau_eff) * 4.5 of a cell the MLP covers.
// Unanchored: tau_eff = tau + 3 nu. Anchored (trust factor k > 0): 3 nu is
// clamped into [ds / k, ds k], ds = 3 nu of the Smagorinsky closure, so the
// Smagorinsky value bounds how far the network may move the cell.
__device__ __forceinline__ float closure_g(const ClosureDev& cl, float nu, float tau, float ds) {
    if (cl.trust > 0.0f) {
        const float d = fminf(fmaxf(3.0f * nu, ds * cl.inv_trust), ds * cl.trust);
        return (1.0f - __fdividef(1.0f, tau + d)) * 4.5f;
    }
    return (1.0f - __fdividef(1.0f, fmaf(3.0f, nu, tau))) * 4.5f;
}

// Packs a cell's five normalized inputs and the constant 1 that carries the
// first layer's bias into the three BF16 pairs an A fragment row of K = 8
// holds per lane quarter: (x0,x1) (x2,x3) (x4,1).
__device__ __forceinline__ void closure_pack_inputs(const ClosureDev& cl, float x0, float x1, float x2, float x3,
                                                    uint32_t* out) {
    const float n0 = (x0 - cl.mean[0]) * cl.inv_std[0];
    const float n1 = (x1 - cl.mean[1]) * cl.inv_std[1];
    const float n2 = (x2 - cl.mean[2]) * cl.inv_std[2];
    const float n3 = (x3 - cl.mean[3]) * cl.inv_std[3];
    const float n4 = (cl.filter_width - cl.mean[4]) * cl.inv_std[4];
    out[0] = pack_bf16(n0, n1);
    out[1] = pack_bf16(n2, n3);
    out[2] = pack_bf16(n4, 1.0f);
    out[3] = 0u;
}

// nu_t for the 64 cells of a warp: lane L supplies the packed inputs of its
// cells A and B in s_in[L*8 + 0..3] and [L*8 + 4..7] (written, then
// __syncwarp, before the call) and receives (nu_A, nu_B). Every lane of the
// warp must call it together. Row r of row tile j is cell A (r < 8) or B
// (r >= 8) of lane 8j + (r & 7).
// `tiles`: bit j set when row tile j (the cells of lanes 8j .. 8j+7) has a
// cell that needs nu_t; cleared tiles are skipped (warp-uniform) and their
// lanes receive whatever s_out held.
__device__ __forceinline__ float2 closure_warp_mlp(const uint4* __restrict__ wt, const uint32_t* s_in,
                                                   float2* s_out, unsigned tiles = 0xfu) {
    const int lane = threadIdx.x & 31;
    const int gq = lane >> 2, tq = lane & 3;
    // the small operands stay in registers across the four row tiles; each
    // tile reads its W2 fragments (16 B per lane per n-tile) from L1
    const uint4 w1 = __ldg(wt + 0 * 32 + lane);
    const uint4 bb2 = __ldg(wt + 1 * 32 + lane);
    const uint4 w3 = __ldg(wt + 6 * 32 + lane);
    const float b3 = __uint_as_float(__ldg(reinterpret_cast<const unsigned*>(wt + 7 * 32 + lane)));
    const uint32_t w1v[4] = {w1.x, w1.y, w1.z, w1.w};
    const uint32_t b2v[4] = {bb2.x, bb2.y, bb2.z, bb2.w};
    // A fragment of a constant-1 column (K slot 0) for the bias MMA
    const uint32_t one = tq == 0 ? 0x3f80u : 0u;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!((tiles >> j) & 1u)) continue;
        const int src = 8 * j + gq;
        const uint32_t a0 = s_in[src * 8 + tq];      // cell A of lane src: row gq
        const uint32_t a1 = s_in[src * 8 + 4 + tq];  // cell B: row gq + 8
        // layer 1 (K = 8, bias in K slot 5) -> h1 as the two K = 16 A
        // fragments of layer 2
        uint32_t h1[8];
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            float d[4];
            mma_k8(d, a0, a1, w1v[n]);
            h1[2 * n] = pack_relu_bf16(d[0], d[1]);      // row gq, cols 8n + 2tq, +1
            h1[2 * n + 1] = pack_relu_bf16(d[2], d[3]);  // row gq + 8
        }
        // layer 2 -> h2 as the K = 16 A fragments of layer 3
        uint32_t h2[8];
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            const uint4 w2 = __ldg(wt + (2 + n) * 32 + lane);
            float d[4];
            mma_k16_z(d, h1[0], h1[1], h1[2], h1[3], w2.x, w2.y);  // k 0-15: n-tiles 0, 1 of h1
            mma_k16(d, h1[4], h1[5], h1[6], h1[7], w2.z, w2.w);    // k 16-31: n-tiles 2, 3
            mma_k8_acc(d, one, one, b2v[n]);                       // + b2
            h2[2 * n] = pack_relu_bf16(d[0], d[1]);
            h2[2 * n + 1] = pack_relu_bf16(d[2], d[3]);
        }
        // layer 3: output column 0
        float d[4];
        mma_k16_z(d, h2[0], h2[1], h2[2], h2[3], w3.x, w3.y);
        mma_k16(d, h2[4], h2[5], h2[6], h2[7], w3.z, w3.w);
        if (tq == 0) s_out[src] = make_float2(fmaxf(d[0] + b3, 0.0f), fmaxf(d[2] + b3, 0.0f));
    }
    __syncwarp();
    return s_out[lane];
}

}  // namespace fc
