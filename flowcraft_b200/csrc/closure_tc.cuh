// The learned closure's MLP on the 5th-generation tensor cores (tcgen05,
// sm_100a), one evaluation for the 512 cells of a block of the two-cell bulk
// kernels (8 warps x 32 lanes x 2 cells).
//
// The cells form four M = 128 row tiles: warp w, lane l, cell b (0 = the
// pair's first cell, 1 = its second) is row 32 (w % 4) + l of tile
// 2 (w / 4) + b, so each warp's rows sit in the TMEM lanes 32 (w % 4) .. +31
// that the warp may read. Per layer, one thread issues a tcgen05.mma per
// tile (kind::f16: BF16 operands from shared memory, FP32 accumulators in
// TMEM) and commits them to an mbarrier; every warp then reads its rows'
// accumulators with tcgen05.ld, applies the ReLU while rounding to BF16
// (cvt.rn.relu.bf16x2) and writes them back to shared memory as the next
// layer's A operand:
//   layer 1  A = the inputs (K = 16: inputs 0-4, the constant 1 that carries
//            b1, zeros), B = W1, N = 32           -> TMEM columns 32 t ..
//   layer 2  A = h1 (K = 32, two MMAs) + a constant-1 column times the b2
//            block, B = W2, N = 32                  -> the same columns
//   layer 3  A = h2 (K = 32), B = W3 (N = 16, row 0 = w3 * out_scale)
//                                                  -> columns 16 t ..
// and nu_t = relu(z + b3). The weights (a 5 KB image packed on the host,
// pack_closure_tc) arrive with one bulk copy (cp.async.bulk, no multicast).
// Operands use the canonical K-major layout without swizzle: 8-row x
// 16-byte core matrices, LBO = 128 bytes between the two core matrices of
// an MMA's K = 16, SBO = K * 16 bytes between 8-row groups.
//
// Every thread of the block must call closure_cta_mlp together. The block
// holds 128 TMEM columns from the allocation to the release at the end of
// the call. Every barrier wait is bounded; a wait that runs out makes the
// whole block leave the MLP (a block-wide vote), waits once more (bounded)
// for its own MMAs, frees the TMEM, flags the step (*err | 2) and returns
// zeros.
#pragma once

#include <stdint.h>

#include "closure.cuh"

namespace fc {

constexpr int kTcTiles = 4;
constexpr int kTcCols = 128;          // TMEM columns a block holds
constexpr unsigned kTcWaitLimit = 1u << 22;

struct __align__(128) TcSmem {
    uint8_t act[kTcTiles][128 * 64];  // A operands: the inputs (K = 16), then h1 and h2 (K = 32)
    uint8_t one[128 * 32];            // A of the bias MMA: a constant-1 column (K = 16)
    uint8_t w[kTcWeightBytes];        // B operands (pack_closure_tc)
    unsigned long long bar_w, bar_mma;
    uint32_t taddr;
};

__device__ __forceinline__ uint32_t tc_smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start, LBO, SBO (bytes), version 1,
// no swizzle.
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: F32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n.
__device__ __forceinline__ constexpr uint32_t tc_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ bool tc_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
    for (unsigned it = 0; it < kTcWaitLimit; ++it)
        if (tc_try_wait(bar, parity)) return true;
    return false;
}

// 16 consecutive FP32 columns of this warp's 32 TMEM lanes (one row per lane).
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ uint32_t tc_ld1(uint32_t taddr) {
    uint32_t r;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr) : "memory");
    return r;
}

__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Byte offset of row r, core-matrix column q in an act tile (K = 32).
__device__ __forceinline__ uint32_t tc_act_off(int r, int q) { return (uint32_t)((r >> 3) * 512 + q * 128 + (r & 7) * 16); }

// Reads one row's 32 accumulator columns starting at `col`, and writes
// relu(.) as BF16 into the row's four core-matrix columns of `dst`.
__device__ __forceinline__ void tc_relu_row(uint32_t taddr_row, uint32_t col, uint8_t* dst_tile, int r) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        uint32_t v[16];
        tc_ld16(taddr_row + col + 16u * h, v);
        tc_wait_ld();
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float* f = reinterpret_cast<const float*>(v) + 8 * q;
            const uint4 pk = make_uint4(pack_relu_bf16(f[0], f[1]), pack_relu_bf16(f[2], f[3]),
                                        pack_relu_bf16(f[4], f[5]), pack_relu_bf16(f[6], f[7]));
            *reinterpret_cast<uint4*>(dst_tile + tc_act_off(r, 2 * h + q)) = pk;
        }
    }
}

// nu_t of the calling lane's two cells, given their packed inputs (chunk 0 of
// the K = 16 input row, closure_pack_inputs). `live`: this warp's rows feed
// results that are used (a warp with no cell in range passes false and
// skips the per-row work; its rows still ride in the tiles).
__device__ __forceinline__ float2 closure_cta_mlp(TcSmem& sm, const ClosureDev& cl, uint4 in_a, uint4 in_b, bool live,
                                                  int* __restrict__ err) {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int warp = tid >> 5, lane = tid & 31;
    const int r = 32 * (warp & 3) + lane;                // row in the tiles
    const int ta = 2 * (warp >> 2), tb = ta + 1;         // tiles of cells A and B
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t bar_w = tc_smem_u32(&sm.bar_w), bar_mma = tc_smem_u32(&sm.bar_mma);

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_w) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_mma) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(&sm.taddr)),
                     "r"((uint32_t)kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // the constant-1 column (K slot 0) of the bias MMA's A, one 16-byte chunk per thread
    {
        const int o = 16 * tid;
        *reinterpret_cast<uint4*>(sm.one + o) = ((o >> 7) & 1) ? make_uint4(0u, 0u, 0u, 0u) : make_uint4(0x3f80u, 0u, 0u, 0u);
    }
    if (live) {
        *reinterpret_cast<uint4*>(sm.act[ta] + tc_act_off(r, 0)) = in_a;
        *reinterpret_cast<uint4*>(sm.act[ta] + tc_act_off(r, 1)) = make_uint4(0u, 0u, 0u, 0u);
        *reinterpret_cast<uint4*>(sm.act[tb] + tc_act_off(r, 0)) = in_b;
        *reinterpret_cast<uint4*>(sm.act[tb] + tc_act_off(r, 1)) = make_uint4(0u, 0u, 0u, 0u);
    }
    tc_fence_proxy();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = sm.taddr;

    const uint32_t s_act = tc_smem_u32(sm.act[0]), s_one = tc_smem_u32(sm.one), s_w = tc_smem_u32(sm.w);
    bool ok = true;
    // layer 1
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_w), "r"((uint32_t)kTcWeightBytes)
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(s_w),
                     "l"(cl.tcw), "r"((uint32_t)kTcWeightBytes), "r"(bar_w)
                     : "memory");
        ok = tc_wait(bar_w, 0);
        if (ok) {
            for (int t = 0; t < kTcTiles; ++t)
                tc_mma(taddr + 32u * t, tc_desc(s_act + 8192u * t, 128, 512), tc_desc(s_w, 128, 256), tc_idesc(32), 0u);
            tc_commit(bar_mma);
        }
    }
    ok = __syncthreads_and(ok) != 0;
    if (ok) ok = tc_wait(bar_mma, 0);
    ok = __syncthreads_and(ok) != 0;
    if (ok) {
        tc_fence_after();
        if (live) {
            tc_relu_row(taddr + lane_base, 32u * ta, sm.act[ta], r);
            tc_relu_row(taddr + lane_base, 32u * tb, sm.act[tb], r);
        }
        tc_fence_proxy();
        tc_fence_before();
        __syncthreads();
        // layer 2: D = h1 W2 + 1 b2 over the same columns
        if (tid == 0) {
            tc_fence_after();
            for (int t = 0; t < kTcTiles; ++t) {
                const uint32_t d = taddr + 32u * t, a = s_act + 8192u * t;
                tc_mma(d, tc_desc(a, 128, 512), tc_desc(s_w + 1024u, 128, 512), tc_idesc(32), 0u);
                tc_mma(d, tc_desc(a + 256u, 128, 512), tc_desc(s_w + 1024u + 256u, 128, 512), tc_idesc(32), 1u);
                tc_mma(d, tc_desc(s_one, 128, 256), tc_desc(s_w + 3072u, 128, 256), tc_idesc(32), 1u);
            }
            tc_commit(bar_mma);
        }
        ok = tc_wait(bar_mma, 1);
        ok = __syncthreads_and(ok) != 0;
    }
    if (ok) {
        tc_fence_after();
        if (live) {
            tc_relu_row(taddr + lane_base, 32u * ta, sm.act[ta], r);
            tc_relu_row(taddr + lane_base, 32u * tb, sm.act[tb], r);
        }
        tc_fence_proxy();
        tc_fence_before();
        __syncthreads();
        // layer 3: N = 16, column 0 is the output
        if (tid == 0) {
            tc_fence_after();
            for (int t = 0; t < kTcTiles; ++t) {
                const uint32_t d = taddr + 16u * t, a = s_act + 8192u * t;
                tc_mma(d, tc_desc(a, 128, 512), tc_desc(s_w + 4096u, 128, 512), tc_idesc(16), 0u);
                tc_mma(d, tc_desc(a + 256u, 128, 512), tc_desc(s_w + 4096u + 256u, 128, 512), tc_idesc(16), 1u);
            }
            tc_commit(bar_mma);
        }
        ok = tc_wait(bar_mma, 0);
        ok = __syncthreads_and(ok) != 0;
    }
    float2 nu = make_float2(0.0f, 0.0f);
    if (ok) {
        tc_fence_after();
        const float za = __uint_as_float(tc_ld1(taddr + lane_base + 16u * ta));
        const float zb = __uint_as_float(tc_ld1(taddr + lane_base + 16u * tb));
        tc_wait_ld();
        nu = make_float2(fmaxf(za + cl.b3, 0.0f), fmaxf(zb + cl.b3, 0.0f));
    } else {
        // a wait ran out: let this block's own MMAs finish (bounded) before the TMEM goes
        if (tid == 0) {
            tc_wait(bar_mma, 0);
            tc_wait(bar_mma, 1);
            atomicOr(err, 2);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"((uint32_t)kTcCols)
                     : "memory");
    }
    return nu;
}

}  // namespace fc
