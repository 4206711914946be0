// The LBM step on B200: one fused pull-stream + boundary + regularized
// collision update per cell (FlowCraft/LbmReference.cpp:241-469, the GPU
// twin shaders/lbm_step.comp.glsl:98-364), split into two kernels so the
// kernel that touches >99% of the cells never branches on geometry:
//
//   k_bulk_pull      one thread per cell, warps on 32 consecutive x of one
//                    row; a warp reads one 32-bit word of the bit-packed bulk
//                    mask and every set lane gathers Q populations from its
//                    upstream neighbours (coalesced SoA loads, the +-x shifts
//                    misaligned by one element), collides, and writes Q
//                    populations. Boundary and solid lanes just exit.
//   k_boundary_pull  one thread per entry of the compacted boundary list:
//                    fluid cells with a wall, domain-edge or Bouzidi link,
//                    the x = 0 / x = nx-1 inlet/outlet planes, and the solid
//                    cells an outlet may read. Link kinds and Bouzidi
//                    coefficients were precomputed at init from the solid
//                    mask and SDF with the reference's float operations.
//
// Both kernels read one population set and write the other (ping-pong), so
// they are independent and touch disjoint cells.
#include "collide.cuh"
#include "lbm_internal.h"
#include "storage.cuh"

namespace fc {

constexpr int kBulkRows = 8;  // block = 32 x-lanes x 8 rows

template <int Q>
__device__ __forceinline__ long long link_offset(int i, const Geom& g) {
    return (long long)Lattice<Q>::ex(i) + (long long)Lattice<Q>::ey(i) * g.nx + (long long)Lattice<Q>::ez(i) * g.nxy;
}

template <int Q, class S>
__global__ void __launch_bounds__(32 * kBulkRows) k_bulk_pull(const typename S::T* __restrict__ fin,
                                                               typename S::T* __restrict__ fout,
                                                               const uint32_t* __restrict__ bulk_bits, Geom g,
                                                               StepParams p, int z0, int* __restrict__ diverged) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * kBulkRows + threadIdx.y;
    const int z = z0 + blockIdx.z;
    if (y >= g.ny) return;
    const size_t row = (size_t)z * g.ny + y;
    const uint32_t bits = __ldg(bulk_bits + row * g.wpr + blockIdx.x);
    if (!((bits >> threadIdx.x) & 1u)) return;  // bits beyond nx are zero
    const size_t c = row * g.nx + x;

    float f[Q];
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        f[i] = load_pop_c<Q, S, i>(fin, g.n, c - link_offset<Q>(i, g));
    });
    if (collide_regularized<Q>(f, p.tau, p.cs)) atomicOr(diverged, 1);
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        store_pop_c<Q, S, i>(fout, g.n, c, f[i]);
    });
}

template <int Q, class S>
__global__ void __launch_bounds__(128) k_boundary_pull(const typename S::T* __restrict__ fin,
                                                        typename S::T* __restrict__ fout, BoundaryList bl,
                                                        uint32_t begin, uint32_t end, Geom g, StepParams p,
                                                        int* __restrict__ diverged) {
    using L = Lattice<Q>;
    const uint32_t e = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= end) return;
    const uint32_t c = __ldg(bl.cells + e);
    const unsigned long long lk = __ldg(bl.links + e);
    const unsigned cls = (unsigned)(lk >> kClassShift) & 7u;
    const uint32_t z = (uint32_t)(c / (unsigned long long)g.nxy);
    const uint32_t rem = c - z * (uint32_t)g.nxy;
    const uint32_t y = rem / (uint32_t)g.nx;
    const int x = (int)(rem - y * (uint32_t)g.nx);

    float f[Q];
    if (cls == kCellSolidFill) {  // solid cell: f_i = w_i (LbmReference.cpp:264-267)
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            store_pop_c<Q, S, i>(fout, g.n, c, L::w(i));
        });
        return;
    }
    if (cls == kCellPlane) {
        if (x == p.inlet_x) {  // equilibrium at rho = 1, u = (+-U, 0, 0) (LbmReference.cpp:269-273)
            equilibrium_all<Q>(1.0f, p.inlet_ux, 0.0f, 0.0f, f);
        } else {  // zero-gradient outlet from the neighbour's fIn moments (LbmReference.cpp:275-327)
            const size_t nb = p.reverse ? (size_t)c + 1 : (size_t)c - 1;
            float g0[Q];
            static_for<0, Q>([&](auto I) {
                constexpr int i = decltype(I)::value;
                g0[i] = load_pop_c<Q, S, i>(fin, g.n, nb);
            });
            float nr, nu, nv, nw;
            moments<Q>(g0, nr, nu, nv, nw);
            const float rho = nr > 1e-6f ? 1.0f + 0.999f * (nr - 1.0f) : 1.0f;
            equilibrium_all<Q>(rho, nu, nv, nw, f);
        }
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            store_pop_c<Q, S, i>(fout, g.n, c, f[i]);
        });
        return;
    }

    // Fluid cell next to a wall, an edge, or both (LbmReference.cpp:329-383).
    uint32_t co = __ldg(bl.coef_off + e);
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        constexpr int op = L::opp(i);
        const unsigned kind = (unsigned)(lk >> (3 * i)) & 7u;
        float v;
        if (kind == kLinkStream) {
            v = load_pop_c<Q, S, i>(fin, g.n, (size_t)c - link_offset<Q>(i, g));
        } else if (kind == kLinkBounce) {
            v = load_pop_c<Q, S, op>(fin, g.n, c);
        } else if (kind == kLinkBzNear) {
            const float2 k = __ldg(bl.coef + co++);
            const float a = load_pop_c<Q, S, op>(fin, g.n, c);
            const float b = load_pop_c<Q, S, op>(fin, g.n, (size_t)c + link_offset<Q>(i, g));
            v = k.x * a + k.y * b;
        } else if (kind == kLinkBzFar) {
            const float2 k = __ldg(bl.coef + co++);
            const float a = load_pop_c<Q, S, op>(fin, g.n, c);
            const float b = load_pop_c<Q, S, i>(fin, g.n, c);
            v = k.x * a + k.y * b;
        } else {
            // Off the Y and/or Z edge: free-slip mirror if every wall crossed
            // is free-slip, else plain bounce-back (LbmReference.cpp:370-380).
            const int py = (int)y - L::ey(i), pz = (int)z - L::ez(i);
            const bool oy = py < 0 || py >= g.ny;
            const bool oz = pz < 0 || pz >= g.nz;
            const bool mirror = (oy || oz) && (!oy || p.slip_y) && (!oz || p.slip_z);
            if (!mirror)
                v = load_pop_c<Q, S, op>(fin, g.n, c);
            else if (oy && oz)
                v = load_pop_c<Q, S, mirror_z<Q>(mirror_y<Q>(i))>(fin, g.n, c);
            else if (oy)
                v = load_pop_c<Q, S, mirror_y<Q>(i)>(fin, g.n, c);
            else
                v = load_pop_c<Q, S, mirror_z<Q>(i)>(fin, g.n, c);
        }
        f[i] = v;
    });
    if (collide_regularized<Q>(f, p.tau, p.cs)) atomicOr(diverged, 1);
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        store_pop_c<Q, S, i>(fout, g.n, c, f[i]);
    });
}

template <int Q, class S>
static cudaError_t bulk_t(const void* fin, void* fout, const uint32_t* bits, const Geom& g, const StepParams& p,
                          int z0, int zc, int* dv, cudaStream_t s) {
    if (zc <= 0) return cudaSuccess;
    dim3 block(32, kBulkRows, 1);
    dim3 grid((unsigned)g.wpr, (unsigned)((g.ny + kBulkRows - 1) / kBulkRows), (unsigned)zc);
    k_bulk_pull<Q, S><<<grid, block, 0, s>>>((const typename S::T*)fin, (typename S::T*)fout, bits, g, p, z0, dv);
    return cudaGetLastError();
}

template <int Q, class S>
static cudaError_t boundary_t(const void* fin, void* fout, const BoundaryList& bl, uint32_t b, uint32_t e,
                              const Geom& g, const StepParams& p, int* dv, cudaStream_t s) {
    if (e <= b) return cudaSuccess;
    const unsigned threads = 128;
    const unsigned blocks = (e - b + threads - 1) / threads;
    k_boundary_pull<Q, S><<<blocks, threads, 0, s>>>((const typename S::T*)fin, (typename S::T*)fout, bl, b, e, g, p,
                                                     dv);
    return cudaGetLastError();
}

#define FC_DISPATCH(q, storage, FN, ...)                                              \
    do {                                                                              \
        if ((q) == 19) {                                                              \
            if ((storage) == 0) return FN<19, StoreF32>(__VA_ARGS__);                 \
            if ((storage) == 1) return FN<19, StoreF16>(__VA_ARGS__);                 \
            if ((storage) == 2) return FN<19, StoreBF16>(__VA_ARGS__);                \
        } else if ((q) == 15) {                                                       \
            if ((storage) == 0) return FN<15, StoreF32>(__VA_ARGS__);                 \
            if ((storage) == 1) return FN<15, StoreF16>(__VA_ARGS__);                 \
            if ((storage) == 2) return FN<15, StoreBF16>(__VA_ARGS__);                \
        }                                                                             \
        return cudaErrorInvalidValue;                                                 \
    } while (0)

cudaError_t launch_bulk_pull(int q, int storage, const void* fin, void* fout, const uint32_t* bulk_bits,
                             const Geom& g, const StepParams& p, int z0, int zc, int* diverged, cudaStream_t s) {
    FC_DISPATCH(q, storage, bulk_t, fin, fout, bulk_bits, g, p, z0, zc, diverged, s);
}

cudaError_t launch_boundary_pull(int q, int storage, const void* fin, void* fout, const BoundaryList& bl,
                                 uint32_t begin, uint32_t end, const Geom& g, const StepParams& p, int* diverged,
                                 cudaStream_t s) {
    FC_DISPATCH(q, storage, boundary_t, fin, fout, bl, begin, end, g, p, diverged, s);
}

}  // namespace fc
