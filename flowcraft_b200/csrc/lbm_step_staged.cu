// The interior of the ping-pong bulk step with the source rows staged in
// shared memory by TMA tensor copies (cp.async.bulk.tensor), for the 16-bit
// storage formats.
//
// A tile is 8 rows x 64 cells of one z layer: rows y0 .. y0+7 off the Y
// faces, one 64-cell chunk off the row ends, a layer off the Z faces (the
// interior warps of k_bulk_pairs). For direction i the tile pulls rows
// (y0 - e_y .. y0 - e_y + 7) of layer z - e_z in plane i:
//   * cells [x0, x0 + 64) as one 2D tensor copy of a 64 x 8 box, whose rows
//     start on 128-byte boundaries (whole 32-byte sectors, nothing shared
//     with the neighbouring tiles);
//   * for e_x = +1 also cell x0 - 1, and for e_x = -1 cell x0 + 64, as an
//     8 x 8 box of the same rows (16 bytes per row, the smallest tensor copy
//     that keeps x 16-byte aligned): [x0 - 8, x0) or [x0 + 64, x0 + 72),
//     both inside the row since the chunk is not the first or last.
// A D3Q19 or D3Q15 tile's sources arrive as Q main copies and 10 halo copies
// instead of Q x 8 x 2 element loads per lane pair.
//
// Each block is a pipeline of kTileStages tiles:
//   * a producer warp (its lane 0) waits until the 8 consumer warps
//     have released a stage (the "empty" barrier, 8 arrivals), arms the
//     stage's "full" barrier with the byte count, and issues the tile's
//     Q + 10 copies;
//   * consumer warp r computes row y0 + r of the tile: each lane takes the
//     cell pair (x, x+1), reads its Q values from shared memory at the e_x
//     shift, collides exactly as k_bulk_pairs does (the pair collision for
//     full pairs, the one-cell collision next to a wall), stores aligned
//     pairs to HBM, then releases the stage.
// Every barrier wait has an iteration limit; a wait that runs out marks the
// step failed (divergence flag | 2), the producer waits (bounded) for the
// copies it has in flight, and the block leaves. Tiles are handed out in
// row order, grid-stride, so neighbouring tiles' shared rows hit L2.
//
// Needs nx a multiple of 8 (16-byte aligned rows), nx > 128 (one interior
// chunk), ny, nz >= 3.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "step_common.cuh"

namespace fc {

namespace {

constexpr int kTileRows = 8;       // consumer warps per block, one row each
constexpr int kTileStages = 3;     // tiles in flight per block
constexpr int kTileThreads = 32 * (kTileRows + 1);
constexpr int kTileBlocksPerSm = 3;
constexpr unsigned kWaitLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
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

// Bounded wait on a barrier phase; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (unsigned it = 0; it < kWaitLimit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 2D tensor copy of one box into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Work decomposition of one launch: tile t -> (z, y0, chunk).
struct TilePlan {
    unsigned long long tiles;
    int zi0;      // first interior z of the range
    int chunks;   // interior chunks per row (gx - 2)
    int yblocks;  // 8-row blocks over the interior rows 1 .. ny-2
};

// e_x + 1, e_y + 1 or e_z + 1 of every direction in 2-bit fields (axis 0, 1,
// 2), for run-time indexing.
template <int Q>
__host__ __device__ constexpr unsigned long long packed_e(int axis) {
    unsigned long long v = 0;
    for (int i = 0; i < Q; ++i) {
        const int e = axis == 0 ? Lattice<Q>::ex(i) : axis == 1 ? Lattice<Q>::ey(i) : Lattice<Q>::ez(i);
        v |= (unsigned long long)(e + 1) << (2 * i);
    }
    return v;
}

// Halo slot of direction i among the directions with e_x != 0, in order.
template <int Q>
__host__ __device__ constexpr int halo_slot(int i) {
    int h = 0;
    for (int j = 0; j < i; ++j) h += Lattice<Q>::ex(j) != 0;
    return h;
}

template <int Q, class S>
struct TileStaging {
    static constexpr int kCols = 64;                 // main box width
    static constexpr int kHaloCols = 16 / S::kBytes;  // halo box width (16 bytes)
    static constexpr int kHalos = halo_slot<Q>(Q);   // directions with e_x != 0
    static constexpr int kMain = kCols * kTileRows;  // elements per main box
    static constexpr int kHalo = kHaloCols * kTileRows;
    static constexpr uint32_t kMainBytes = (uint32_t)kMain * S::kBytes;  // a multiple of 128
    static constexpr uint32_t kHaloBytes = (uint32_t)kHalo * S::kBytes;  // 128
    static constexpr uint32_t kStageBytes = Q * kMainBytes + kHalos * kHaloBytes;
    static constexpr size_t kSmem = (size_t)kTileStages * kStageBytes + 128;  // + alignment slack
};

}  // namespace

template <int Q, class S>
__global__ void __launch_bounds__(kTileThreads, kTileBlocksPerSm) k_bulk_tiles(const __grid_constant__ CUtensorMap map,
                                                                              const __grid_constant__ CUtensorMap halo,
                                                                              const uint32_t* __restrict__ bulk_bits,
                                                                              Geom g, StepParams p, PlanePtrs pp,
                                                                              TilePlan plan,
                                                                              int* __restrict__ diverged) {
    using L = Lattice<Q>;
    using T = typename S::T;
    using T2 = typename S::T2;
    using St = TileStaging<Q, S>;
    constexpr int kStage = St::kStageBytes / sizeof(T);  // elements per stage
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long full[kTileStages], empty[kTileStages];
    T* stages = reinterpret_cast<T*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kTileStages; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), kTileRows);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if ((unsigned long long)blockIdx.x >= plan.tiles) return;
    const unsigned long long count = (plan.tiles - 1 - blockIdx.x) / gridDim.x + 1;
    auto tile_of = [&](unsigned long long k, int& z, int& y0, int& cx) {
        const unsigned long long t = blockIdx.x + k * gridDim.x;
        cx = 1 + (int)(t % plan.chunks);
        const unsigned long long r = t / plan.chunks;
        y0 = 1 + kTileRows * (int)(r % plan.yblocks);
        z = plan.zi0 + (int)(r / plan.yblocks);
    };

    if (warp == kTileRows) {  // producer
        if (lane != 0) return;
        constexpr unsigned long long kEx = packed_e<Q>(0), kEy = packed_e<Q>(1), kEz = packed_e<Q>(2);
        const long long layer_rows = (long long)g.ny * g.nz;
        unsigned long long k = 0;
        for (; k < count; ++k) {
            const int s = (int)(k % kTileStages);
            if (k >= kTileStages && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((k / kTileStages - 1) & 1))) {
                atomicOr(diverged, 3);
                break;
            }
            int z, y0, cx;
            tile_of(k, z, y0, cx);
            const uint32_t bar = smem_u32(&full[s]);
            mbar_expect_tx(bar, St::kStageBytes);
            const uint32_t dst = smem_u32(stages + (size_t)s * kStage);
            const uint32_t dst_halo = dst + Q * St::kMainBytes;
            const int x0 = 64 * cx;
            int h = 0;
            for (int i = 0; i < Q; ++i) {
                const int ex = (int)((kEx >> (2 * i)) & 3ull) - 1;
                const int ey = (int)((kEy >> (2 * i)) & 3ull) - 1, ez = (int)((kEz >> (2 * i)) & 3ull) - 1;
                const int row = (int)((long long)i * layer_rows + (long long)(z - ez) * g.ny + (y0 - ey));
                tma_load_2d(dst + (uint32_t)i * St::kMainBytes, &map, x0, row, bar);
                if (ex != 0) {
                    tma_load_2d(dst_halo + (uint32_t)h * St::kHaloBytes, &halo, ex > 0 ? x0 - St::kHaloCols : x0 + 64,
                                row, bar);
                    ++h;
                }
            }
        }
        // copies still in flight land in this block's stages: wait for them (bounded)
        const unsigned long long issued = k;
        const unsigned long long from = issued > kTileStages ? issued - kTileStages : 0;
        for (unsigned long long j = from; j < issued; ++j)
            mbar_wait(smem_u32(&full[(int)(j % kTileStages)]), (uint32_t)((j / kTileStages) & 1));
        return;
    }

    // consumer warp `warp`: row y0 + warp of every tile
    const int kk = 2 * lane;
    // source of cell kk + j - e_x, j in {0, 1}, of direction i: the main box,
    // or for the row's first / last cell the halo box (its last / first column)
    auto src = [&](const T* st, auto I, int j) -> const T* {
        constexpr int i = decltype(I)::value;
        constexpr int ex = L::ex(i);
        const T* main = st + i * St::kMain + warp * St::kCols;
        if constexpr (ex == 0) {
            return main + kk + j;
        } else {
            const T* hal = st + Q * St::kMain + halo_slot<Q>(i) * St::kHalo + warp * St::kHaloCols;
            const int x = kk + j - ex;  // -1 .. 64
            if constexpr (ex > 0)
                return x < 0 ? hal + (St::kHaloCols - 1) : main + x;
            else
                return x >= 64 ? hal : main + x;
        }
    };
    for (unsigned long long k = 0; k < count; ++k) {
        const int s = (int)(k % kTileStages);
        if (!mbar_wait(smem_u32(&full[s]), (uint32_t)((k / kTileStages) & 1))) {
            if (lane == 0) atomicOr(diverged, 3);
            return;  // the producer's own waits run out and it drains its copies
        }
        int z, y0, cx;
        tile_of(k, z, y0, cx);
        const int y = y0 + warp;
        if (y <= g.ny - 2) {
            const T* st = stages + (size_t)s * kStage;
            const size_t row = (size_t)z * g.ny + y;
            const uint32_t bits = __ldg(bulk_bits + row * g.wpr + 2 * cx + (kk >> 5));
            const unsigned pair = (bits >> (kk & 31)) & 3u;
            const uint32_t c = (uint32_t)(row * g.nx + 64 * cx + kk);
            T* const fout = static_cast<T*>(pp.dst[0]);
            if (pair == 3u) {
                float2 v[Q];
                static_for<0, Q>([&](auto I) {
                    constexpr int i = decltype(I)::value;
                    if constexpr (L::ex(i) == 0) {
                        const T2 h = *reinterpret_cast<const T2*>(src(st, I, 0));
                        if constexpr (S::kExact)
                            v[i] = S::dec2(h, L::w(i));
                        else
                            v[i] = S::raw2(h);
                    } else {
                        const T a = *src(st, I, 0), b = *src(st, I, 1);
                        if constexpr (S::kExact)
                            v[i] = make_float2(S::dec(a, L::w(i)), S::dec(b, L::w(i)));
                        else
                            v[i] = make_float2(S::raw(a), S::raw(b));
                    }
                });
                if (collide_pair<Q, S>(v, p.tau, p.cs)) atomicOr(diverged, 1);
                static_for<0, Q>([&](auto I) {
                    constexpr int i = decltype(I)::value;
                    T* dst = static_cast<T*>(pp.dst[i]);
                    if constexpr (S::kExact)
                        *reinterpret_cast<T2*>(dst + c) = S::enc2(v[i].x, v[i].y, L::w(i));
                    else
                        *reinterpret_cast<T2*>(dst + c) = S::pack2(v[i].x, v[i].y);
                });
            } else if (pair) {  // one cell of the pair next to a wall: the one-cell path
                const int b = pair == 1u ? 0 : 1;
                float f[Q];
                static_for<0, Q>([&](auto I) {
                    constexpr int i = decltype(I)::value;
                    f[i] = S::dec(*src(st, I, b), L::w(i));
                });
                if (collide<Q, S::kExact>(f, p.tau, p.cs)) atomicOr(diverged, 1);
                static_for<0, Q>([&](auto I) {
                    constexpr int i = decltype(I)::value;
                    store_pop_i<Q, S, i>(fout, g.n, c + (uint32_t)b, f[i]);
                });
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&empty[s]));  // this row is done with stage s
    }
}

namespace {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

}  // namespace

template <int Q, class S>
static cudaError_t tiles_t(const void* fin, void* fout, const uint32_t* bits, const Geom& g, const StepParams& p,
                           int z0, int zc, int* dv, cudaStream_t s, int* launched) {
    *launched = 0;
    if constexpr (S::kExact) {
        return cudaErrorNotSupported;
    } else {
        using St = TileStaging<Q, S>;
        const int zi0 = z0 > 1 ? z0 : 1, zi1 = (z0 + zc) < g.nz - 1 ? (z0 + zc) : g.nz - 1;
        const int gx = (g.nx + 63) / 64;
        if (zi1 <= zi0 || gx < 3 || g.ny < 3) return cudaSuccess;
        TilePlan plan{};
        plan.zi0 = zi0;
        plan.chunks = gx - 2;
        plan.yblocks = (g.ny - 2 + kTileRows - 1) / kTileRows;
        plan.tiles = (unsigned long long)(zi1 - zi0) * plan.yblocks * plan.chunks;

        auto encode = tensor_map_encoder();
        if (!encode) return cudaErrorNotSupported;
        // the whole population set as nx columns x (Q * nz * ny) rows of 16-bit
        // elements, read as 64 x 8 main boxes and 8 x 8 (16-byte) halo boxes
        const cuuint64_t dims[2] = {(cuuint64_t)g.nx, (cuuint64_t)Q * g.nz * g.ny};
        const cuuint64_t strides[1] = {(cuuint64_t)g.nx * S::kBytes};
        const cuuint32_t estr[2] = {1, 1};
        CUtensorMap maps[2] = {};
        const cuuint32_t boxes[2][2] = {{(cuuint32_t)St::kCols, (cuuint32_t)kTileRows},
                                        {(cuuint32_t)St::kHaloCols, (cuuint32_t)kTileRows}};
        for (int m = 0; m < 2; ++m)
            if (encode(&maps[m], CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, const_cast<void*>(fin), dims, strides, boxes[m],
                       estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return cudaErrorInvalidValue;

        PlanePtrs pp{};
        for (int i = 0; i < Q; ++i) {
            pp.src[i] = nullptr;
            pp.dst[i] = (typename S::T*)fout + (size_t)i * g.n;
        }
        // per instantiation and device: the shared-memory opt-in and the grid
        constexpr int kMaxDev = 64;
        static int blocks_dev[kMaxDev] = {};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
        if (blocks_dev[dev] <= 0) {
            e = cudaFuncSetAttribute(k_bulk_tiles<Q, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)St::kSmem);
            int n = 0, sms = 0;
            if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_bulk_tiles<Q, S>, kTileThreads, St::kSmem);
            if (e != cudaSuccess) return e;
            blocks_dev[dev] = sms * (n > 0 ? n : 1);
        }
        unsigned long long blocks = (unsigned long long)blocks_dev[dev];
        if (blocks > plan.tiles) blocks = plan.tiles;
        k_bulk_tiles<Q, S><<<(unsigned)blocks, kTileThreads, St::kSmem, s>>>(
            maps[0], maps[1], bits, g, p, pp, plan, dv);
        ++*launched;
        return cudaGetLastError();
    }
}

bool staged_eligible(int storage, const Geom& g) {
    // 16-bit formats: the FP32 step is bandwidth-bound unstaged, and its
    // stages would not fit three blocks per SM
    return storage != 0 && g.nx % 8 == 0 && g.nx > 128 && g.ny >= 3 && g.nz >= 3;
}

#define FC_DISPATCH(q, storage, FN, ...)                              \
    do {                                                              \
        if ((q) == 19) {                                              \
            if ((storage) == 0) return FN<19, StoreF32>(__VA_ARGS__);  \
            if ((storage) == 1) return FN<19, StoreF16>(__VA_ARGS__);  \
            if ((storage) == 2) return FN<19, StoreBF16>(__VA_ARGS__); \
        } else if ((q) == 15) {                                       \
            if ((storage) == 0) return FN<15, StoreF32>(__VA_ARGS__);  \
            if ((storage) == 1) return FN<15, StoreF16>(__VA_ARGS__);  \
            if ((storage) == 2) return FN<15, StoreBF16>(__VA_ARGS__); \
        }                                                             \
        return cudaErrorInvalidValue;                                 \
    } while (0)

cudaError_t launch_bulk_staged(int q, int storage, const void* fin, void* fout, const uint32_t* bulk_bits,
                               const Geom& g, const StepParams& p, int z0, int zc, int* diverged, cudaStream_t s,
                               int* launched) {
    FC_DISPATCH(q, storage, tiles_t, fin, fout, bulk_bits, g, p, z0, zc, diverged, s, launched);
}

}  // namespace fc
