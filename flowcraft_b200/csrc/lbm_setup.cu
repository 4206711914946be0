// Init-time geometry work, all on the device:
//   * classify every cell: bulk fluid (bit set in the bulk mask: no solid
//     neighbour, or on the inlet/outlet planes; Y/Z domain faces included)
//     or a boundary-list entry (flag byte), from the solid mask alone;
//   * compact the flagged cells into a sorted list (CUB select);
//   * per list entry, resolve each link: plain pull, halfway bounce-back,
//     Bouzidi near/far with precomputed coefficients, or domain edge. The
//     link test is LbmReference::Step's (LbmReference.cpp:331-381) and the
//     Bouzidi q and coefficients use InterpolatedBounceBack's float
//     operations (LbmReference.cpp:100-122), so the step reproduces them
//     exactly;
//   * seed populations (LbmReference::Reset / ResetFromField,
//     LbmReference.cpp:192-239).
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "aa.cuh"
#include "collide.cuh"
#include "lbm_internal.h"
#include "storage.cuh"

namespace fc {

__device__ __forceinline__ bool in_bounds(const Geom& g, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && x < g.nx && y < g.ny && z < g.nz;
}
__device__ __forceinline__ size_t cell_index(const Geom& g, int x, int y, int z) {
    return ((size_t)z * g.ny + y) * g.nx + x;
}

template <int Q>
__global__ void __launch_bounds__(256) k_classify(const uint8_t* __restrict__ solid, Geom g,
                                                   uint8_t* __restrict__ flags, uint32_t* __restrict__ bulk_bits,
                                                   unsigned long long* __restrict__ counts) {
    using L = Lattice<Q>;
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    bool bulk = false, flag = false;
    const bool live = x < g.nx && y < g.ny;
    if (live) {
        const size_t c = cell_index(g, x, y, z);
        if (solid[c]) {
            flag = (x == 1 || x == g.nx - 2);  // a possible outlet neighbour
        } else if (x == 0 || x == g.nx - 1) {
            bulk = true;  // inlet / outlet plane: handled inside the bulk kernel
        } else {
            // A solid upstream neighbour sends the cell to the list; a
            // neighbour off the Y/Z edge does not (the bulk kernel mirrors it).
            bool wall = false;
            for (int i = 1; i < Q; ++i) {
                const int px = x - L::ex(i), py = y - L::ey(i), pz = z - L::ez(i);
                if (in_bounds(g, px, py, pz) && solid[cell_index(g, px, py, pz)]) wall = true;
            }
            flag = wall;
            bulk = !wall;
        }
        flags[c] = flag ? 1 : 0;
    }
    const unsigned word = __ballot_sync(0xffffffffu, bulk);
    const unsigned fword = __ballot_sync(0xffffffffu, live && flag);
    if (threadIdx.x == 0 && y < g.ny) {
        bulk_bits[((size_t)z * g.ny + y) * g.wpr + blockIdx.x] = word;
        if (fword) atomicAdd(&counts[0], (unsigned long long)__popc(fword));
        if (word) atomicAdd(&counts[1], (unsigned long long)__popc(word));
    }
}

// Bouzidi link for fluid node (x,y,z) = cell c whose direction-i upstream
// neighbour s is solid. Returns the link kind and, for Bouzidi, (c1, c2).
template <int Q>
__device__ __forceinline__ unsigned resolve_wall_link(const uint8_t* __restrict__ solid, const float* __restrict__ sdf,
                                                      const Geom& g, int x, int y, int z, size_t c, int i, size_t s,
                                                      float2& k) {
    using L = Lattice<Q>;
    if (!sdf) return kLinkBounce;
    const float phi_f = sdf[c];
    const float phi_s = sdf[s];
    if (!isfinite(phi_f) || !isfinite(phi_s)) return kLinkBounce;
    const float denom = phi_f - phi_s;
    if (!(denom > 1e-4f)) return kLinkBounce;
    float q = phi_f / denom;
    q = (q < 0.0f) ? 0.0f : ((1.0f < q) ? 1.0f : q);  // std::clamp(q, 0, 1)
    if (q < 0.5f) {
        const int fx = x + L::ex(i), fy = y + L::ey(i), fz = z + L::ez(i);
        if (!in_bounds(g, fx, fy, fz) || solid[cell_index(g, fx, fy, fz)]) return kLinkBounce;
        k.x = 2.0f * q;
        k.y = 1.0f - 2.0f * q;
        return kLinkBzNear;
    }
    const float inv = 1.0f / (2.0f * q);
    k.x = inv;
    k.y = 1.0f - inv;
    return kLinkBzFar;
}

template <int Q>
__global__ void __launch_bounds__(128) k_links(const uint32_t* __restrict__ cells, size_t count,
                                               const uint8_t* __restrict__ solid, const float* __restrict__ sdf,
                                               Geom g, unsigned long long* __restrict__ links,
                                               uint32_t* __restrict__ nbz, const uint32_t* __restrict__ coef_off,
                                               float2* __restrict__ coef) {
    using L = Lattice<Q>;
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const uint32_t c = cells[e];
    const int z = (int)(c / (unsigned long long)g.nxy);
    const uint32_t rem = c - (uint32_t)z * (uint32_t)g.nxy;
    const int y = (int)(rem / (uint32_t)g.nx);
    const int x = (int)(rem - (uint32_t)y * (uint32_t)g.nx);
    unsigned long long word = 0;
    uint32_t nb = 0;
    if (solid[c]) {
        word = (unsigned long long)kCellSolidFill << kClassShift;
    } else {
        uint32_t co = coef ? coef_off[e] : 0;
        for (int i = 0; i < Q; ++i) {
            const int px = x - L::ex(i), py = y - L::ey(i), pz = z - L::ez(i);
            unsigned kind;
            if (!in_bounds(g, px, py, pz)) {
                kind = kLinkEdge;
            } else {
                const size_t s = cell_index(g, px, py, pz);
                if (!solid[s]) {
                    kind = kLinkStream;
                } else {
                    float2 k = make_float2(0.0f, 0.0f);
                    kind = resolve_wall_link<Q>(solid, sdf, g, x, y, z, c, i, s, k);
                    if (kind == kLinkBzNear || kind == kLinkBzFar) {
                        if (coef) coef[co++] = k;
                        ++nb;
                    }
                }
            }
            word |= (unsigned long long)kind << (3 * i);
        }
        word |= (unsigned long long)kCellFluid << kClassShift;
    }
    if (links) links[e] = word;
    if (nbz) nbz[e] = nb;
}

__global__ void k_z_offsets(const uint32_t* __restrict__ cells, size_t count, Geom g, uint32_t* __restrict__ z_begin) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z > g.nz) return;
    const unsigned long long key = (unsigned long long)z * (unsigned long long)g.nxy;
    size_t lo = 0, hi = count;  // first entry with cell >= key
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if ((unsigned long long)cells[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    z_begin[z] = (uint32_t)lo;
}

// Writes populations e[] of cell c where `layout` keeps them (aa.cuh).
template <int Q, class S>
__device__ __forceinline__ void seed_cell(typename S::T* __restrict__ f, const Geom& g, size_t c, const float (&e)[Q],
                                          int layout) {
    const int z = (int)(c / (size_t)g.nxy);
    const size_t rem = c - (size_t)z * g.nxy;
    const int y = (int)(rem / g.nx);
    const int x = (int)(rem - (size_t)y * g.nx);
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        f[pop_slot<Q, i>(c, x, y, z, g, layout)] = S::enc(e[i], Lattice<Q>::w(i));
    });
}

template <int Q, class S>
__global__ void k_seed_uniform(typename S::T* __restrict__ f, Geom g, float rho, float ux, float uy, float uz,
                               int layout) {
    float e[Q];
    equilibrium_all<Q>(rho, ux, uy, uz, e);
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < g.n; c += (size_t)gridDim.x * blockDim.x) {
        if (layout == kLayoutPlanes) {
            static_for<0, Q>([&](auto I) {
                constexpr int i = decltype(I)::value;
                store_pop_c<Q, S, i>(f, g.n, c, e[i]);
            });
        } else {
            seed_cell<Q, S>(f, g, c, e, layout);
        }
    }
}

template <int Q, class S>
__global__ void k_seed_field(typename S::T* __restrict__ f, Geom g, const float4* __restrict__ field,
                             const uint8_t* __restrict__ solid, size_t cell0, size_t cells, int layout) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cells) return;
    const size_t c = cell0 + k;
    float4 v = field[k];
    if (solid[c]) v = make_float4(1.0f, 0.0f, 0.0f, 0.0f);  // LbmReference.cpp:231-234
    float e[Q];
    equilibrium_all<Q>(v.x, v.y, v.z, v.w, e);
    seed_cell<Q, S>(f, g, c, e, layout);
}

template <int Q, class S>
static cudaError_t seed_uniform_t(void* f, const Geom& g, float rho, float ux, float uy, float uz, int layout,
                                  cudaStream_t s) {
    const unsigned blocks = 148 * 8;
    k_seed_uniform<Q, S><<<blocks, 256, 0, s>>>((typename S::T*)f, g, rho, ux, uy, uz, layout);
    return cudaGetLastError();
}

template <int Q, class S>
static cudaError_t seed_field_t(void* f, const Geom& g, const float* field, const uint8_t* solid, size_t cell0,
                                size_t cells, int layout, cudaStream_t s) {
    if (cells == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((cells + 255) / 256);
    k_seed_field<Q, S><<<blocks, 256, 0, s>>>((typename S::T*)f, g, (const float4*)field, solid, cell0, cells,
                                              layout);
    return cudaGetLastError();
}

#define FC_DISPATCH(q, storage, FN, ...)                              \
    do {                                                              \
        if ((q) == 19) {                                              \
            if ((storage) == 0) return FN<19, StoreF32>(__VA_ARGS__); \
            if ((storage) == 1) return FN<19, StoreF16>(__VA_ARGS__); \
            if ((storage) == 2) return FN<19, StoreBF16>(__VA_ARGS__); \
        } else if ((q) == 15) {                                       \
            if ((storage) == 0) return FN<15, StoreF32>(__VA_ARGS__); \
            if ((storage) == 1) return FN<15, StoreF16>(__VA_ARGS__); \
            if ((storage) == 2) return FN<15, StoreBF16>(__VA_ARGS__); \
        }                                                             \
        return cudaErrorInvalidValue;                                 \
    } while (0)

cudaError_t launch_seed_uniform(int q, int storage, void* f, const Geom& g, float rho, float ux, float uy, float uz,
                                int layout, cudaStream_t s) {
    FC_DISPATCH(q, storage, seed_uniform_t, f, g, rho, ux, uy, uz, layout, s);
}

cudaError_t launch_seed_field(int q, int storage, void* f, const Geom& g, const float* field, const uint8_t* solid,
                              size_t cell0, size_t cells, int layout, cudaStream_t s) {
    FC_DISPATCH(q, storage, seed_field_t, f, g, field, solid, cell0, cells, layout, s);
}

cudaError_t launch_classify(int q, const uint8_t* solid, const Geom& g, uint8_t* flags, uint32_t* bulk_bits,
                            unsigned long long* counts, cudaStream_t s) {
    dim3 block(32, 8, 1);
    dim3 grid((unsigned)g.wpr, (unsigned)((g.ny + 7) / 8), (unsigned)g.nz);
    if (q == 19)
        k_classify<19><<<grid, block, 0, s>>>(solid, g, flags, bulk_bits, counts);
    else if (q == 15)
        k_classify<15><<<grid, block, 0, s>>>(solid, g, flags, bulk_bits, counts);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_links(int q, const uint32_t* cells, size_t count, const uint8_t* solid, const float* sdf,
                         const Geom& g, unsigned long long* links, uint32_t* nbz, const uint32_t* coef_off,
                         float2* coef, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((count + 127) / 128);
    if (q == 19)
        k_links<19><<<blocks, 128, 0, s>>>(cells, count, solid, sdf, g, links, nbz, coef_off, coef);
    else if (q == 15)
        k_links<15><<<blocks, 128, 0, s>>>(cells, count, solid, sdf, g, links, nbz, coef_off, coef);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_z_offsets(const uint32_t* cells, size_t count, const Geom& g, uint32_t* z_begin, cudaStream_t s) {
    const unsigned blocks = (unsigned)((g.nz + 1 + 127) / 128);
    k_z_offsets<<<blocks, 128, 0, s>>>(cells, count, g, z_begin);
    return cudaGetLastError();
}

cudaError_t select_flagged_cells(void* temp, size_t& temp_bytes, const uint8_t* flags, uint32_t* out,
                                 uint32_t* count_out, size_t n, cudaStream_t s) {
    thrust::counting_iterator<uint32_t> first(0);
    return cub::DeviceSelect::Flagged(temp, temp_bytes, first, flags, out, count_out, (int64_t)n, s);
}

cudaError_t exclusive_scan_u32(void* temp, size_t& temp_bytes, const uint32_t* in, uint32_t* out, size_t n,
                               cudaStream_t s) {
    return cub::DeviceScan::ExclusiveSum(temp, temp_bytes, in, out, (int64_t)n, s);
}

}  // namespace fc
