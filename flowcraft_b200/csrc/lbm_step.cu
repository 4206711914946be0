// The LBM step on B200: one fused pull-stream + boundary + regularized
// collision update per cell (FlowCraft/LbmReference.cpp:241-469, the GPU
// twin shaders/lbm_step.comp.glsl:98-364), split into two kernels so the
// kernel that touches >99% of the cells never branches on geometry:
//
//   k_bulk_interior  one thread per cell, warps on 32 consecutive x of one
//   k_bulk_shell     row; a warp reads one 32-bit word of the bit-packed bulk
//                    mask and every set lane gathers Q populations from its
//                    upstream neighbours (coalesced SoA loads, the +-x shifts
//                    misaligned by one element), collides, and writes Q
//                    populations. Boundary and solid lanes just exit. The
//                    shell kernel covers the warps that can hold a Y/Z-face
//                    cell (mirror / bounce-back sources) or an inlet/outlet
//                    cell; the interior kernel is a pure pull.
//   k_boundary_pull  one thread per entry of the compacted boundary list:
//                    fluid cells with a solid neighbour (halfway or Bouzidi
//                    links) and the solid cells an outlet may read. Link kinds and
//                    Bouzidi coefficients were precomputed at init from the
//                    solid mask and SDF with the reference's float operations.
//
// Both kernels read one population set and write the other (ping-pong), so
// they are independent and touch disjoint cells.
#include "aa.cuh"
#include "closure.cuh"
#include "closure_tc.cuh"
#include "collide.cuh"
#include "collide2.cuh"
#include "lbm_internal.h"
#include "step_common.cuh"
#include "storage.cuh"

namespace fc {

// One bulk cell. General = false is the interior path: a pure pull from the
// 19 (15) upstream neighbours. General = true adds the Y/Z domain-face
// sources and the inlet/outlet lanes; it only runs in warps that can hold
// such cells (face rows, and the first and last warp of each row), so the
// interior never pays for the selects.
template <int Q, class S, bool General>
__device__ __forceinline__ void bulk_cell(const typename S::T* __restrict__ fin, typename S::T* __restrict__ fout,
                                          const Geom& g, const StepParams& p, int x, int y, int z, uint32_t c,
                                          int* __restrict__ diverged) {
    using L = Lattice<Q>;
    float f[Q];
    if constexpr (!General) {
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            f[i] = load_pop_i<Q, S, i>(fin, g.n, c - (uint32_t)link_offset<Q>(i, g));
        });
        if (collide<Q, S::kExact>(f, p.tau, p.cs)) atomicOr(diverged, 1);
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            store_pop_i<Q, S, i>(fout, g.n, c, f[i]);
        });
    } else {
        const bool inlet = x == p.inlet_x;
        const bool outlet = !inlet && x == p.outlet_x;
        const uint32_t nb = p.reverse ? c + 1u : c - 1u;  // outlet's upstream neighbour (LbmReference.cpp:320)
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const int py = y - L::ey(i), pz = z - L::ez(i);
            const bool oy = py < 0 || py >= g.ny;
            const bool oz = pz < 0 || pz >= g.nz;
            const bool out = (oy || oz) && !outlet;
            const int plane = out ? edge_plane<Q, i>(oy, oz, p) : i;
            // the inlet lane reads nothing; its address is kept in bounds anyway
            const uint32_t src = outlet ? nb : ((out || inlet) ? c : c - (uint32_t)link_offset<Q>(i, g));
            f[i] = inlet ? 0.0f : load_plane<Q, S>(fin, plane, g.n, src, L::w(i));
        });
        if (outlet) {
            // zero-gradient outlet: neighbour's fIn moments, rho relaxed
            // toward 1 (LbmReference.cpp:275-327)
            float nr, nu, nv, nw;
            moments<Q>(f, nr, nu, nv, nw);
            const float rho = nr > 1e-6f ? 1.0f + 0.999f * (nr - 1.0f) : 1.0f;
            equilibrium_all<Q>(rho, nu, nv, nw, f);
        } else {
            const bool bad = collide<Q, S::kExact>(f, p.tau, p.cs);
            if (bad && !inlet) atomicOr(diverged, 1);
        }
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            store_pop_i<Q, S, i>(fout, g.n, c, inlet ? p.feq_inlet[i] : f[i]);
        });
    }
}

// The bulk cells (every fluid cell without a solid neighbour, plus the fluid
// cells of the x = 0 and x = nx-1 planes) are split by warp position into a
// disjoint interior and shell, each its own kernel so each gets its own
// register allocation:
//   interior  rows with 1 <= y <= ny-2 and 1 <= z <= nz-2, 32-cell chunks
//             1 .. wpr-2 of the row: no face, inlet or outlet cell can occur;
//   shell     Y-face rows (all chunks), Z-face rows (all chunks), and the
//             first and last chunk of every other row.
// Folding the inlet/outlet planes into warps makes their accesses part of
// coalesced requests instead of one element per 32-byte sector.
template <int Q, class S>
__global__ void __launch_bounds__(32 * kBulkRows) k_bulk_interior(const typename S::T* __restrict__ fin,
                                                                   typename S::T* __restrict__ fout,
                                                                   const uint32_t* __restrict__ bulk_bits, Geom g,
                                                                   StepParams p, int z0, int* __restrict__ diverged) {
    const int chunk = blockIdx.x + 1;
    const int x = chunk * 32 + threadIdx.x;
    const int y = 1 + blockIdx.y * kBulkRows + threadIdx.y;
    const int z = z0 + blockIdx.z;
    if (y >= g.ny - 1) return;
    const size_t row = (size_t)z * g.ny + y;
    const uint32_t bits = __ldg(bulk_bits + row * g.wpr + chunk);
    if (!((bits >> threadIdx.x) & 1u)) return;
    const uint32_t c = (uint32_t)(row * g.nx + x);
    bulk_cell<Q, S, false>(fin, fout, g, p, x, y, z, c, diverged);
}

// One inlet or outlet cell (x = 0 or x = nx-1, fluid): equilibrium at the
// inlet (LbmReference.cpp:269-273); at the outlet, equilibrium from the
// upstream neighbour's fIn moments with rho relaxed toward 1
// (LbmReference.cpp:275-327).
template <int Q, class S>
__device__ __forceinline__ void plane_cell(const typename S::T* __restrict__ fin, typename S::T* __restrict__ fout,
                                           const Geom& g, const StepParams& p, int x, size_t c) {
    float f[Q];
    if (x == p.inlet_x) {
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            f[i] = p.feq_inlet[i];
        });
    } else {
        const size_t nb = p.reverse ? c + 1 : c - 1;
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            f[i] = load_pop_c<Q, S, i>(fin, g.n, nb);
        });
        float nr, nu, nv, nw;
        moments<Q>(f, nr, nu, nv, nw);
        const float rho = nr > 1e-6f ? 1.0f + 0.999f * (nr - 1.0f) : 1.0f;
        equilibrium_all<Q>(rho, nu, nv, nw, f);
    }
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        store_pop_c<Q, S, i>(fout, g.n, c, f[i]);
    });
}

// The inlet / outlet cells a warp of the pair kernels holds, updated by the
// whole warp for the 16-bit formats: lane i < Q takes population i, so a
// cell's Q loads and Q stores are one instruction each for the warp instead
// of Q for one lane while the other lanes wait. The values, the moments
// (direction order, shared by shuffles) and the equilibrium are those of
// plane_cell. Every lane of the warp calls row_end_cells together; `plane`
// holds this lane's bits (1: cell x, 2: cell x + 1). (The FP32 kernels keep
// plane_cell: there the warp-wide version costs more registers than the
// kernel has to spare.)
template <int Q, class S>
__device__ __forceinline__ void row_end_cell(const typename S::T* __restrict__ fin, typename S::T* __restrict__ fout,
                                             const Geom& g, const StepParams& p, int px, size_t pc) {
    const unsigned lane = threadIdx.x & 31;
    const bool mine = lane < (unsigned)Q;
    const unsigned i = mine ? lane : 0u;
    const float wi = lattice_w_rt<Q>(i);
    typename S::T* dst = fout + (size_t)i * g.n + pc;
    if (px == p.inlet_x) {  // feq_inlet[i]: the equilibrium at rho 1, u = (inlet_ux, 0, 0)
        const float ux = p.inlet_ux;
        const float v = equilibrium_rt<Q>(i, 1.0f, ux, 0.0f, 0.0f, speed2(ux, 0.0f, 0.0f));
        if (mine) *dst = S::enc(v, wi);
        return;
    }
    const size_t nb = p.reverse ? pc + 1 : pc - 1;
    const float own = S::dec(S::ld(fin + (size_t)i * g.n + nb), wi);
    float f[Q];
    static_for<0, Q>([&](auto I) { f[decltype(I)::value] = __shfl_sync(0xffffffffu, own, decltype(I)::value); });
    float nr, nu, nv, nw;
    moments<Q>(f, nr, nu, nv, nw);
    const float rho = nr > 1e-6f ? 1.0f + 0.999f * (nr - 1.0f) : 1.0f;
    const float o = equilibrium_rt<Q>(i, rho, nu, nv, nw, speed2(nu, nv, nw));
    if (mine) *dst = S::enc(o, wi);
}

template <int Q, class S>
__device__ __forceinline__ void row_end_cells(const typename S::T* __restrict__ fin, typename S::T* __restrict__ fout,
                                              const Geom& g, const StepParams& p, unsigned plane, int x, uint32_t c) {
    unsigned m = __ballot_sync(0xffffffffu, plane != 0u);
    while (m) {  // uniform: at most the two row ends
        const int src = __ffs(m) - 1;
        m &= m - 1u;
        const unsigned sp = __shfl_sync(0xffffffffu, plane, src);
        const int sx = __shfl_sync(0xffffffffu, x, src);
        const uint32_t sc = __shfl_sync(0xffffffffu, c, src);
        if (sp & 1u) row_end_cell<Q, S>(fin, fout, g, p, sx, (size_t)sc);
        if (sp & 2u) row_end_cell<Q, S>(fin, fout, g, p, sx + 1, (size_t)sc + 1);
    }
}

// Bulk cells of lattices with even nx, two x-adjacent cells per thread, every
// row and every 64-cell chunk. A warp covers cells [64*blockIdx.x, +64) of one
// row, so whether it touches a Y/Z domain face (`face`) or the first or last
// chunk of the row (`edge`) is uniform across the warp:
//   * interior warps, and the full pairs of edge warps off the faces, run
//     the pure pair pull (aligned 2-element loads for the e_x = 0
//     directions, pair stores);
//   * face warps, and the partial pairs of edge warps, run the general pair
//     path: sources off the Y/Z edge come from the cell's own mirrored /
//     bounced plane (the choice is per direction and uniform across the
//     row), cells that are not bulk cells here keep in-bounds addresses and
//     are not stored;
//   * the lane holding an x = 0 or x = nx-1 cell first updates that inlet /
//     outlet cell.
// Stores the pair's post-collision values (full floats for the exact
// format, scaled offsets otherwise): one 2-element store per plane for a full
// pair, element stores for the valid cell of a partial one. The full / partial
// test is made once for all Q planes: per plane it costs a divergence-safe
// branch (BSSY / BSYNC) for each of the Q stores.
template <int Q, class S>
__device__ __forceinline__ void store_pair(const PlanePtrs& pp, uint32_t c, const float2 (&v)[Q], unsigned pair) {
    using L = Lattice<Q>;
    using T = typename S::T;
    auto enc = [&](auto I) {
        constexpr int i = decltype(I)::value;
        if constexpr (S::kExact)
            return S::enc2(v[i].x, v[i].y, L::w(i));
        else
            return S::pack2(v[i].x, v[i].y);
    };
    if (pair == 3u) {
        static_for<0, Q>([&](auto I) {
            T* dst = static_cast<T*>(pp.dst[decltype(I)::value]);
            *reinterpret_cast<typename S::T2*>(dst + c) = enc(I);
        });
    } else {  // one cell of the pair (pair is 1 or 2): one element store per plane
        const uint32_t ec = pair == 1u ? c : c + 1u;
        static_for<0, Q>([&](auto I) {
            T* dst = static_cast<T*>(pp.dst[decltype(I)::value]);
            const typename S::T2 h = enc(I);
            dst[ec] = pair == 1u ? h.x : h.y;
        });
    }
}

// Blocks of k_bulk_pairs when its interior warps run in k_bulk_tiles: the
// shell as a 1D list of (chunk, 8-row block, z) items in three regions,
//   E  the first and last chunk of every row block of every layer,
//   F  the other chunks of the row blocks that hold y = 0 or y = ny-1, in
//      layers off the Z faces,
//   G  the other chunks of every row block of the Z-face layers,
// so no block is launched only to find nothing to do. n == 0: the whole
// lattice, blockIdx = (chunk, row block, z - z0).
struct PairsShell {
    unsigned long long n, ne, nf;  // items in all, in E, in F
    int gx, nyb;                   // chunks per row, 8-row blocks per layer
    int z0, zi0;                   // first layer of the range, first layer off the Z faces
    int nyf;                       // row blocks in F (1 or 2)
    int nzf, zf[2];                // Z-face layers in the range
};

__device__ __forceinline__ void shell_item(const PairsShell& sh, int& bx, int& by, int& z) {
    unsigned long long it = blockIdx.x;
    if (it < sh.ne) {
        bx = (it & 1ull) ? sh.gx - 1 : 0;
        const unsigned long long r = it >> 1;
        by = (int)(r % sh.nyb);
        z = sh.z0 + (int)(r / sh.nyb);
        return;
    }
    it -= sh.ne;
    const int inner = sh.gx - 2;
    bx = 1 + (int)(it % inner);
    const unsigned long long r = it / inner;
    if (it < sh.nf) {
        by = (r % sh.nyf) ? sh.nyb - 1 : 0;
        z = sh.zi0 + (int)(r / sh.nyf);
    } else {
        const unsigned long long q = r - sh.nf / inner;
        by = (int)(q % sh.nyb);
        z = (q / sh.nyb) ? sh.zf[1] : sh.zf[0];
    }
}

// One block of k_bulk_pairs: the 64 x kBulkRows cells of x chunk bx, row
// block by, layer z. shell: the launch covers the shell only (interior warps
// leave). k_bulk_pairs_tiles runs the same code for the tiles of many
// lattices in one launch.
template <int Q, class S>
__device__ __forceinline__ void pairs_tile(const typename S::T* __restrict__ fin, typename S::T* __restrict__ fout,
                                           const uint32_t* __restrict__ bulk_bits, const Geom& g,
                                           const StepParams& p, const PlanePtrs& pp, int* __restrict__ diverged,
                                           int bx, int by, int z, bool shell) {
    using L = Lattice<Q>;
    using T = typename S::T;
    const int y = by * kBulkRows + threadIdx.y;
    if (y >= g.ny) return;
    const size_t row = (size_t)z * g.ny + y;
    const int k = 2 * threadIdx.x;
    const int w = 2 * bx + (k >> 5);
    const uint32_t bits = w < g.wpr ? __ldg(bulk_bits + row * g.wpr + w) : 0u;
    const int x = 64 * bx + k;
    unsigned pair = (bits >> (k & 31)) & 3u;
    unsigned plane = 0;  // fluid inlet / outlet cells of this pair
    if (x == 0) {
        plane |= pair & 1u;
        pair &= ~1u;
    }
    if (x + 1 == g.nx - 1) {
        plane |= pair & 2u;
        pair &= ~2u;
    }
    const uint32_t c = (uint32_t)(row * g.nx + x);
    if constexpr (!S::kExact) {  // the row-end cells by the whole warp (no interior warp holds one)
        row_end_cells<Q, S>(fin, fout, g, p, plane, x, c);
        plane = 0;
    }
    if (!(pair | plane)) return;
    const bool face = (y == 0) | (y == g.ny - 1) | (z == 0) | (z == g.nz - 1);
    const bool edge = (bx == 0) | (64 * bx + 64 >= g.nx);
    if (shell && !face && !edge) return;  // an interior warp: done by k_bulk_tiles

    // FP32: the one lane of a row end that holds an inlet or outlet cell finishes it alone
    if (plane) plane_cell<Q, S>(fin, fout, g, p, plane == 1u ? x : x + 1, plane == 1u ? c : (size_t)c + 1);
    if (!pair) return;
    float2 v[Q];
    if (!face) {
        if (pair != 3u && !edge) {  // one of the two is next to a wall (a boundary-list cell)
            const uint32_t cc = pair == 1u ? c : c + 1u;
            bulk_cell<Q, S, false>(fin, fout, g, p, x + (pair == 1u ? 0 : 1), y, z, cc, diverged);
            return;
        }
        // Full pairs, and in row-end warps every pair: the plain pull. Off the
        // Y/Z faces every source of a row lies inside the population set, also
        // for a cell that is not stored here (an inlet / outlet or wall cell
        // next to a pair cell), so a row-end warp runs one uniform path, with
        // the masked pair collision of the general path for its partial pairs.
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const T* src = static_cast<const T*>(pp.src[i]);
            if constexpr (S::kExact) {
                v[i] = L::ex(i) == 0 ? S::dec2(S::ld2(src + c), L::w(i))
                                     : make_float2(S::dec(S::ld(src + c), L::w(i)),
                                                   S::dec(S::ld(src + c + 1u), L::w(i)));
            } else {
                v[i] = L::ex(i) == 0 ? S::raw2(S::ld2(src + c))
                                     : make_float2(S::raw(S::ld(src + c)), S::raw(S::ld(src + c + 1u)));
            }
        });
        if (collide_pair<Q, S>(v, p.tau, p.cs) & pair) atomicOr(diverged, 1);
        store_pair<Q, S>(pp, c, v, pair);
        return;
    }
    // general pair path: face rows, and partial pairs of the row-end chunks
    const bool va = pair & 1u, vb = pair & 2u;
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const int py = y - L::ey(i), pz = z - L::ez(i);
        const bool oy = py < 0 || py >= g.ny;
        const bool oz = pz < 0 || pz >= g.nz;
        const bool out = oy || oz;  // the same for the whole row
        const int plane = out ? edge_plane<Q, i>(oy, oz, p) : i;
        const uint32_t off = out ? 0u : (uint32_t)link_offset<Q>(i, g);
        const uint32_t sa = va ? c - off : c;
        const uint32_t sb = vb ? c + 1u - off : c + 1u;
        const T* base = fin + (size_t)plane * g.n;
        if constexpr (S::kExact)
            v[i] = make_float2(S::dec(S::ld(base + sa), L::w(i)), S::dec(S::ld(base + sb), L::w(i)));
        else
            v[i] = make_float2(S::raw(S::ld(base + sa)), S::raw(S::ld(base + sb)));
    });
    const unsigned bad = collide_pair<Q, S>(v, p.tau, p.cs) & pair;
    if (bad) atomicOr(diverged, 1);
    store_pair<Q, S>(pp, c, v, pair);
}

template <int Q, class S>
__global__ void __launch_bounds__(32 * kBulkRows, 4) k_bulk_pairs(const typename S::T* __restrict__ fin,
                                                                typename S::T* __restrict__ fout,
                                                                const uint32_t* __restrict__ bulk_bits, Geom g,
                                                                StepParams p, PlanePtrs pp, int z0,
                                                                int* __restrict__ diverged, PairsShell sh) {
    int bx = blockIdx.x, by = blockIdx.y, z = z0 + blockIdx.z;
    if (sh.n) shell_item(sh, bx, by, z);
    pairs_tile<Q, S>(fin, fout, bulk_bits, g, p, pp, diverged, bx, by, z, sh.n != 0);
}

// The bulk step of many lattices in one launch of one block per tile: the
// blocks of each lattice's own k_bulk_pairs launch, in its order, the
// lattices one after another, so they follow each other through the GPU with
// no launch boundary between them. Every lattice's k_bulk_pairs parameters
// travel in this launch's parameters (constant bank): a block finds its
// lattice by a binary search there and runs k_bulk_pairs' per-tile code, so
// a batch step is bit-identical to stepping each lattice alone.
template <int Q, class S>
__global__ void __launch_bounds__(32 * kBulkRows, 4) k_bulk_pairs_tiles(const __grid_constant__ TileLaunch t) {
    using T = typename S::T;
    const unsigned w = blockIdx.x;
    int lo = 0, hi = t.nlat - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t.l[mid].first <= w) lo = mid;
        else hi = mid - 1;
    }
    const TileLattice& d = t.l[lo];
    const unsigned local = w - d.first;
    const unsigned gx = (unsigned)d.gx, gy = (unsigned)d.gy;
    const unsigned r = local / gx;
    const unsigned z = r / gy;
    pairs_tile<Q, S>(static_cast<const T*>(d.fin), static_cast<T*>(d.fout), d.bits, d.g, d.p, d.pp, d.diverged,
                     (int)(local - r * gx), (int)(r - z * gy), (int)z, false);
}

// k_bulk_pairs with the learned closure (16-bit offset storage). The MLP is a
// warp-wide tensor-core operation, so no lane leaves before it: lanes without
// a bulk pair run it on zero offsets and store nothing. Loads and stores are
// those of k_bulk_pairs (aligned pair loads in interior warps for full pairs,
// the general masked path otherwise); between them the collision runs in two
// halves around the closure (moments2, closure_warp_mlp, relax2). Warps never
// wait for one another: the closure's shared memory is private to each warp.
template <int Q, class S>
__global__ void __launch_bounds__(32 * kBulkRows, 4) k_bulk_pairs_learned(const typename S::T* __restrict__ fin,
                                                                        typename S::T* __restrict__ fout,
                                                                        const uint32_t* __restrict__ bulk_bits,
                                                                        Geom g, StepParams p, PlanePtrs pp, int z0,
                                                                        int* __restrict__ diverged, ClosureDev cl) {
    static_assert(!S::kExact, "the learned closure runs on the 16-bit offset formats");
    using L = Lattice<Q>;
    using T = typename S::T;
    __shared__ uint32_t s_in[kBulkRows][32 * 8];
    __shared__ float2 s_out[kBulkRows][32];
    __shared__ float2 s_mo[kBulkRows][12][32];  // the relaxation's moments while the MLP runs
    const int y = blockIdx.y * kBulkRows + threadIdx.y;
    const int z = z0 + blockIdx.z;
    if (y >= g.ny) return;  // the whole warp: one row
    const size_t row = (size_t)z * g.ny + y;
    const int k = 2 * threadIdx.x;
    const int w = 2 * blockIdx.x + (k >> 5);
    const uint32_t bits = w < g.wpr ? __ldg(bulk_bits + row * g.wpr + w) : 0u;
    const int x = 64 * blockIdx.x + k;
    unsigned pair = (bits >> (k & 31)) & 3u;
    unsigned plane = 0;
    if (x == 0) {
        plane |= pair & 1u;
        pair &= ~1u;
    }
    if (x + 1 == g.nx - 1) {
        plane |= pair & 2u;
        pair &= ~2u;
    }
    const uint32_t c = (uint32_t)(row * g.nx + x);
    const bool face = (y == 0) | (y == g.ny - 1) | (z == 0) | (z == g.nz - 1);
    row_end_cells<Q, S>(fin, fout, g, p, plane, x, c);
    const bool va = pair & 1u, vb = pair & 2u;

    // The load path is chosen per warp: off the Y/Z faces every lane takes
    // the pure pair pull (every source of a row off the faces lies inside the
    // lattice, also for the cells a lane does not store: the inlet / outlet
    // cell of a row end and wall cells), the masked general path on the faces.
    // Lanes beyond the row load their own row and store nothing.
    const bool fast = !face;
    const uint32_t cs = x < g.nx ? c : (uint32_t)(row * g.nx);
    float2 v[Q];
    if (fast) {
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const T* src = static_cast<const T*>(pp.src[i]);
            v[i] = L::ex(i) == 0 ? S::raw2(S::ld2(src + cs))
                                 : make_float2(S::raw(S::ld(src + cs)), S::raw(S::ld(src + cs + 1u)));
        });
    } else {
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const int py = y - L::ey(i), pz = z - L::ez(i);
            const bool oy = py < 0 || py >= g.ny;
            const bool oz = pz < 0 || pz >= g.nz;
            const bool out = oy || oz;
            const int pl = out ? edge_plane<Q, i>(oy, oz, p) : i;
            const uint32_t off = out ? 0u : (uint32_t)link_offset<Q>(i, g);
            const uint32_t sa = va ? c - off : cs;
            const uint32_t sb = vb ? c + 1u - off : cs + 1u;
            const T* base = fin + (size_t)pl * g.n;
            v[i] = make_float2(S::raw(S::ld(base + sa)), S::raw(S::ld(base + sb)));
        });
    }
    Mom2 mo;
    const unsigned bad = moments2<Q>(v, mo) & pair;
    // everything besides nu_t is settled before the MMA, so only the moments
    // stay live across it. The range test goes input by input, each stage
    // only in warps where some lane is still in range (warp votes, so the
    // branches stay uniform); the inputs are packed for the MLP only where
    // it runs.
    // both cells' wall distances in one aligned load (x and nx are even)
    const unsigned wd = pair ? (unsigned)__ldg(reinterpret_cast<const unsigned short*>(cl.wall + c)) : 0xffffu;
    float ra, rb;
    const float xa0 = closure_x0(mo.pp.x, mo.inv.x, ra), xb0 = closure_x0(mo.pp.y, mo.inv.y, rb);
    bool la = closure_wall_ok(cl, wd & 0xffu) && closure_x0_in_range(cl, xa0);
    bool lb = closure_wall_ok(cl, wd >> 8) && closure_x0_in_range(cl, xb0);
    float xa1 = 0.0f, xa2 = 0.0f, xb1 = 0.0f, xb2 = 0.0f;
    if (__any_sync(0xffffffffu, la || lb)) {
        closure_x12(mo.pxx.x, mo.pyy.x, mo.pzz.x, mo.pxy.x, mo.pxz.x, mo.pyz.x, ra, xa1, xa2);
        closure_x12(mo.pxx.y, mo.pyy.y, mo.pzz.y, mo.pxy.y, mo.pxz.y, mo.pyz.y, rb, xb1, xb2);
        la = la && closure_x12_in_range(cl, xa1, xa2);
        lb = lb && closure_x12_in_range(cl, xb1, xb2);
    }
    // the Smagorinsky fallback only where some lane of the warp needs it
    float sga = 0.0f, sgb = 0.0f, dsa = 0.0f, dsb = 0.0f;
    if (closure_anchored(cl) || __any_sync(0xffffffffu, !(la && lb))) {
        sga = smagorinsky_g(mo.pp.x, mo.rho.x, mo.inv.x, p.tau, p.cs);
        sgb = smagorinsky_g(mo.pp.y, mo.rho.y, mo.inv.y, p.tau, p.cs);
        if (closure_anchored(cl)) {
            dsa = smagorinsky_d3(mo.pp.x, mo.rho.x, mo.inv.x, p.tau, p.cs);
            dsb = smagorinsky_d3(mo.pp.y, mo.rho.y, mo.inv.y, p.tau, p.cs);
        }
    }
    // A cell outside the training range takes the Smagorinsky value, so a
    // warp with no cell in range has no use for the MLP and skips it (the
    // result is the same): it relaxes with Smagorinsky and is done.
    const unsigned need = __ballot_sync(0xffffffffu, la || lb);
    if (!need) {
        if (!pair) return;
        relax2<Q>(v, mo, make_float2(sga, sgb));
        if (bad) atomicOr(diverged, 1);
        store_pair<Q, S>(pp, c, v, pair);
        return;
    }
    // The MLP path. The moments the relaxation needs wait in shared memory
    // (this warp's own slice) while the MLP holds the registers.
    float2* sm = &s_mo[threadIdx.y][0][threadIdx.x];
    sm[0 * 32] = mo.rho, sm[1 * 32] = mo.drho, sm[2 * 32] = mo.u2, sm[3 * 32] = mo.ux;
    sm[4 * 32] = mo.uy, sm[5 * 32] = mo.uz, sm[6 * 32] = mo.pxx, sm[7 * 32] = mo.pyy;
    sm[8 * 32] = mo.pzz, sm[9 * 32] = mo.pxy, sm[10 * 32] = mo.pxz, sm[11 * 32] = mo.pyz;
    // row tiles of the MLP (8 lanes each) with a cell in range
    const unsigned tiles = ((need & 0xffu) ? 1u : 0u) | ((need & 0xff00u) ? 2u : 0u) |
                           ((need & 0xff0000u) ? 4u : 0u) | ((need & 0xff000000u) ? 8u : 0u);
    uint32_t* in = &s_in[threadIdx.y][threadIdx.x * 8];
    closure_pack_inputs(cl, xa0, xa1, xa2, (float)(wd & 0xffu) * 0.0625f, in);
    closure_pack_inputs(cl, xb0, xb1, xb2, (float)(wd >> 8) * 0.0625f, in + 4);
    __syncwarp();
    const float2 nu = closure_warp_mlp(cl.frag, s_in[threadIdx.y], s_out[threadIdx.y], tiles);
    if (!pair) return;
    Mom2 mr;
    mr.rho = sm[0 * 32], mr.drho = sm[1 * 32], mr.u2 = sm[2 * 32], mr.ux = sm[3 * 32];
    mr.uy = sm[4 * 32], mr.uz = sm[5 * 32], mr.pxx = sm[6 * 32], mr.pyy = sm[7 * 32];
    mr.pzz = sm[8 * 32], mr.pxy = sm[9 * 32], mr.pxz = sm[10 * 32], mr.pyz = sm[11 * 32];
    float2 gr;
    gr.x = la ? closure_g(cl, nu.x, p.tau, dsa) : sga;
    gr.y = lb ? closure_g(cl, nu.y, p.tau, dsb) : sgb;
    relax2<Q>(v, mr, gr);
    if (bad) atomicOr(diverged, 1);
    store_pair<Q, S>(pp, c, v, pair);
}

// k_bulk_pairs_learned with the MLP on the tcgen05 tensor cores
// (FC_OPTION_TC_CLOSURE): the same loads, inputs, fallback and stores, but
// the MLP runs once for the block's 512 cells (closure_cta_mlp), in blocks
// where some cell is in the training range (a block-wide vote); the other
// blocks relax with Smagorinsky at once. So no warp leaves before the vote:
// rows past the lattice and lanes without a bulk pair load nothing or
// in-lattice values and store nothing. Each block serializes its three
// layers (MMA, commit, TMEM read-back, barrier), and with four blocks per SM
// nothing hides those waits: in a developed flow this kernel takes twice the
// time of the warp-level one, which stays the default.
template <int Q, class S>
__global__ void __launch_bounds__(32 * kBulkRows, 4) k_bulk_pairs_learned_tc(const typename S::T* __restrict__ fin,
                                                                           typename S::T* __restrict__ fout,
                                                                           const uint32_t* __restrict__ bulk_bits,
                                                                           Geom g, StepParams p, PlanePtrs pp, int z0,
                                                                           int* __restrict__ diverged, ClosureDev cl) {
    static_assert(!S::kExact, "the learned closure runs on the 16-bit offset formats");
    using L = Lattice<Q>;
    using T = typename S::T;
    __shared__ TcSmem tsm;
    const int y = blockIdx.y * kBulkRows + threadIdx.y;
    const int z = z0 + blockIdx.z;
    const bool row_ok = y < g.ny;  // the whole warp: one row
    const size_t row = (size_t)z * g.ny + (row_ok ? y : 0);
    const int k = 2 * threadIdx.x;
    const int w = 2 * blockIdx.x + (k >> 5);
    const uint32_t bits = row_ok && w < g.wpr ? __ldg(bulk_bits + row * g.wpr + w) : 0u;
    const int x = 64 * blockIdx.x + k;
    unsigned pair = (bits >> (k & 31)) & 3u;
    unsigned plane = 0;
    if (x == 0) {
        plane |= pair & 1u;
        pair &= ~1u;
    }
    if (x + 1 == g.nx - 1) {
        plane |= pair & 2u;
        pair &= ~2u;
    }
    const uint32_t c = (uint32_t)(row * g.nx + x);
    const bool face = (y == 0) | (y == g.ny - 1) | (z == 0) | (z == g.nz - 1);
    row_end_cells<Q, S>(fin, fout, g, p, plane, x, c);
    const bool va = pair & 1u, vb = pair & 2u;

    // The load path is chosen per warp: off the Y/Z faces every lane takes
    // the pure pair pull (every source of a row off the faces lies inside the
    // lattice, also for the cells a lane does not store: the inlet / outlet
    // cell of a row end and wall cells), the masked general path on the faces.
    // Lanes beyond the row load their own row and store nothing.
    const uint32_t cs = x < g.nx ? c : (uint32_t)(row * g.nx);
    float2 v[Q];
    if (!row_ok) {
        static_for<0, Q>([&](auto I) { v[decltype(I)::value] = make_float2(0.0f, 0.0f); });
    } else if (!face) {
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const T* src = static_cast<const T*>(pp.src[i]);
            v[i] = L::ex(i) == 0 ? S::raw2(S::ld2(src + cs))
                                 : make_float2(S::raw(S::ld(src + cs)), S::raw(S::ld(src + cs + 1u)));
        });
    } else {
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const int py = y - L::ey(i), pz = z - L::ez(i);
            const bool oy = py < 0 || py >= g.ny;
            const bool oz = pz < 0 || pz >= g.nz;
            const bool out = oy || oz;
            const int pl = out ? edge_plane<Q, i>(oy, oz, p) : i;
            const uint32_t off = out ? 0u : (uint32_t)link_offset<Q>(i, g);
            const uint32_t sa = va ? c - off : cs;
            const uint32_t sb = vb ? c + 1u - off : cs + 1u;
            const T* base = fin + (size_t)pl * g.n;
            v[i] = make_float2(S::raw(S::ld(base + sa)), S::raw(S::ld(base + sb)));
        });
    }
    Mom2 mo;
    const unsigned bad = moments2<Q>(v, mo) & pair;
    // The range test goes input by input, each stage only in warps where
    // some lane is still in range (warp votes keep the branches uniform).
    float ra, rb;
    const float xa0 = closure_x0(mo.pp.x, mo.inv.x, ra), xb0 = closure_x0(mo.pp.y, mo.inv.y, rb);
    const unsigned wd = pair ? (unsigned)__ldg(reinterpret_cast<const unsigned short*>(cl.wall + c)) : 0xffffu;
    bool la = row_ok && closure_wall_ok(cl, wd & 0xffu) && closure_x0_in_range(cl, xa0);
    bool lb = row_ok && closure_wall_ok(cl, wd >> 8) && closure_x0_in_range(cl, xb0);
    float xa1 = 0.0f, xa2 = 0.0f, xb1 = 0.0f, xb2 = 0.0f;
    if (__any_sync(0xffffffffu, la || lb)) {
        closure_x12(mo.pxx.x, mo.pyy.x, mo.pzz.x, mo.pxy.x, mo.pxz.x, mo.pyz.x, ra, xa1, xa2);
        closure_x12(mo.pxx.y, mo.pyy.y, mo.pzz.y, mo.pxy.y, mo.pxz.y, mo.pyz.y, rb, xb1, xb2);
        la = la && closure_x12_in_range(cl, xa1, xa2);
        lb = lb && closure_x12_in_range(cl, xb1, xb2);
    }
    // the Smagorinsky fallback only where some lane of the warp needs it
    float sga = 0.0f, sgb = 0.0f, dsa = 0.0f, dsb = 0.0f;
    if (closure_anchored(cl) || __any_sync(0xffffffffu, !(la && lb))) {
        sga = smagorinsky_g(mo.pp.x, mo.rho.x, mo.inv.x, p.tau, p.cs);
        sgb = smagorinsky_g(mo.pp.y, mo.rho.y, mo.inv.y, p.tau, p.cs);
        if (closure_anchored(cl)) {
            dsa = smagorinsky_d3(mo.pp.x, mo.rho.x, mo.inv.x, p.tau, p.cs);
            dsb = smagorinsky_d3(mo.pp.y, mo.rho.y, mo.inv.y, p.tau, p.cs);
        }
    }
    // A cell outside the training range takes the Smagorinsky value, so a
    // block with no cell in range has no use for the MLP and skips it (the
    // result is the same).
    const bool live = __any_sync(0xffffffffu, la || lb);
    float2 g2 = make_float2(sga, sgb);
    if (__syncthreads_or(live)) {
        uint4 ia, ib;
        closure_pack_inputs(cl, xa0, xa1, xa2, (float)(wd & 0xffu) * 0.0625f, reinterpret_cast<uint32_t*>(&ia));
        closure_pack_inputs(cl, xb0, xb1, xb2, (float)(wd >> 8) * 0.0625f, reinterpret_cast<uint32_t*>(&ib));
        const float2 nu = closure_cta_mlp(tsm, cl, ia, ib, live, diverged);
        if (la) g2.x = closure_g(cl, nu.x, p.tau, dsa);
        if (lb) g2.y = closure_g(cl, nu.y, p.tau, dsb);
    }
    if (!pair) return;
    relax2<Q>(v, mo, g2);
    if (bad) atomicOr(diverged, 1);
    store_pair<Q, S>(pp, c, v, pair);
}

// The closure's inputs and nu_t for every cell of the current population set
// as stored (no streaming; `layout` a PopLayout of aa.cuh): the same device
// code as the fused kernels, for checking the inference against a CPU
// evaluation. Two cells per lane. Solid cells count as holding f = w, what
// a ping-pong set keeps there (in place their slots carry the neighbours'
// bounced populations).
// out[5*c .. 5*c+4] = inputs 0-3 and nu_t; in_range[c] = 1 when the learned
// value is used. With out == nullptr it only counts, into counts[0] the
// cells in range and into counts[1] the 64-cell warps with any cell in range
// (the warps that run the MLP in a step).
template <int Q, class S>
__global__ void __launch_bounds__(128) k_closure_probe(const typename S::T* __restrict__ f,
                                                       const uint8_t* __restrict__ solid, Geom g, ClosureDev cl,
                                                       float* __restrict__ out, uint8_t* __restrict__ in_range,
                                                       unsigned long long* __restrict__ counts, int layout) {
    static_assert(!S::kExact, "the learned closure runs on the 16-bit offset formats");
    __shared__ uint32_t s_in[4][32 * 8];
    __shared__ float2 s_out[4][32];
    const size_t c = 2 * ((size_t)blockIdx.x * blockDim.x + threadIdx.x);
    const bool ha = c < g.n, hb = c + 1 < g.n;
    const bool la = ha && !solid[c], lb = hb && !solid[c + 1];  // read the stored values
    auto coords = [&](size_t cc, int& x, int& y, int& z) {
        z = (int)(cc / g.nxy);
        const size_t rem = cc - (size_t)z * g.nxy;
        y = (int)(rem / (size_t)g.nx);
        x = (int)(rem - (size_t)y * g.nx);
    };
    int xa = 0, ya = 0, za = 0, xb = 0, yb = 0, zb = 0;
    if (ha) coords(c, xa, ya, za);
    if (hb) coords(c + 1, xb, yb, zb);
    float2 v[Q];
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        v[i] = make_float2(la ? S::raw(S::ld(f + pop_slot<Q, i>(c, xa, ya, za, g, layout))) : 0.0f,
                           lb ? S::raw(S::ld(f + pop_slot<Q, i>(c + 1, xb, yb, zb, g, layout))) : 0.0f);
    });
    Mom2 mo;
    moments2<Q>(v, mo);
    float ia[4], ib[4];
    closure_invariants(mo.pxx.x, mo.pyy.x, mo.pzz.x, mo.pxy.x, mo.pxz.x, mo.pyz.x, mo.pp.x, mo.inv.x, ia[0], ia[1],
                       ia[2]);
    closure_invariants(mo.pxx.y, mo.pyy.y, mo.pzz.y, mo.pxy.y, mo.pxz.y, mo.pyz.y, mo.pp.y, mo.inv.y, ib[0], ib[1],
                       ib[2]);
    ia[3] = ha ? (float)cl.wall[c] * 0.0625f : 0.0f;
    ib[3] = hb ? (float)cl.wall[c + 1] * 0.0625f : 0.0f;
    const int warp = threadIdx.x >> 5;
    if (!out) {
        const bool ra = ha && closure_wall_ok(cl, cl.wall[c]) && closure_in_range(cl, ia[0], ia[1], ia[2]);
        const bool rb = hb && closure_wall_ok(cl, cl.wall[c + 1]) && closure_in_range(cl, ib[0], ib[1], ib[2]);
        const unsigned cells = __popc(__ballot_sync(0xffffffffu, ra)) + __popc(__ballot_sync(0xffffffffu, rb));
        if ((threadIdx.x & 31) == 0 && cells) {
            atomicAdd(counts, (unsigned long long)cells);
            atomicAdd(counts + 1, 1ull);
        }
        return;
    }
    uint32_t* in = &s_in[warp][(threadIdx.x & 31) * 8];
    closure_pack_inputs(cl, ia[0], ia[1], ia[2], ia[3], in);
    closure_pack_inputs(cl, ib[0], ib[1], ib[2], ib[3], in + 4);
    __syncwarp();
    const float2 nu = closure_warp_mlp(cl.frag, s_in[warp], s_out[warp]);
    if (ha) {
        for (int k = 0; k < 4; ++k) out[5 * c + k] = ia[k];
        out[5 * c + 4] = nu.x;
        in_range[c] = closure_wall_ok(cl, cl.wall[c]) && closure_in_range(cl, ia[0], ia[1], ia[2]) ? 1 : 0;
    }
    if (hb) {
        for (int k = 0; k < 4; ++k) out[5 * (c + 1) + k] = ib[k];
        out[5 * (c + 1) + 4] = nu.y;
        in_range[c + 1] = closure_wall_ok(cl, cl.wall[c + 1]) && closure_in_range(cl, ib[0], ib[1], ib[2]) ? 1 : 0;
    }
}

// The bulk step of many lattices in one persistent launch over a work-list of
// tiles (64 x ROWS cells of one z layer) spanning every lattice of a batch.
// Blocks stride over chunks of kBatchChunk consecutive tiles (block b takes
// chunks b, b + G, b + 2G, ...), which interleaves cheap and costly tiles
// across blocks. A block's tiles only ever move forward, so it searches for
// a tile's lattice (binary search over the lattices' first items) only when
// the tile passes the end of the current one, and keeps that lattice's
// descriptor (geometry, step parameters, plane pointers) in shared memory
// meanwhile. The tile's (x chunk, row group, z) is divided out once per
// chunk in 32-bit arithmetic and stepped from tile to tile after that. The
// per-tile work and arithmetic are those of k_bulk_pairs, so a batch step is
// bit-identical to stepping each lattice alone.
template <int Q, class S, int ROWS>
__global__ void __launch_bounds__(32 * ROWS, 32 / ROWS) k_bulk_pairs_batch(const BatchLattice* __restrict__ lat,
                                                                           int nlat, unsigned long long total,
                                                                           int parity) {
    using L = Lattice<Q>;
    using T = typename S::T;
    __shared__ BatchLattice sl;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    unsigned long long cur_end = 0;  // one past the current lattice's last tile
    int bx = 0, ty = 0, z = 0;       // the tile: x chunk, row group, z layer
    const unsigned long long chunks = (total + kBatchChunk - 1) / kBatchChunk;
    for (unsigned long long ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
    bool fresh = true;
    for (unsigned long long w = ch * kBatchChunk; w < min(total, (ch + 1) * kBatchChunk); ++w) {
        if (w >= cur_end) {  // w and cur_end are the same for every thread of the block
            int lo = 0, hi = nlat - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(&lat[mid].first) <= w) lo = mid;
                else hi = mid - 1;
            }
            __syncthreads();
            const int* srcw = reinterpret_cast<const int*>(lat + lo);
            int* dstw = reinterpret_cast<int*>(&sl);
            for (int k = tid; k < (int)(sizeof(BatchLattice) / 4); k += 32 * ROWS) dstw[k] = __ldg(srcw + k);
            __syncthreads();
            cur_end = lo + 1 < nlat ? __ldg(&lat[lo + 1].first) : total;
            fresh = true;
        }
        if (fresh) {  // a lattice has fewer than 2^32 tiles
            const unsigned local = (unsigned)(w - sl.first);
            const unsigned t = local / (unsigned)sl.gx;
            bx = (int)(local - t * (unsigned)sl.gx);
            z = (int)(t / (unsigned)sl.gy);
            ty = (int)(t - (unsigned)z * (unsigned)sl.gy);
            fresh = false;
        } else if (++bx == sl.gx) {
            bx = 0;
            if (++ty == sl.gy) {
                ty = 0;
                ++z;
            }
        }
        const Geom& g = sl.g;
        const StepParams& p = sl.p;
        const int side = sl.cur ^ parity;
        const PlanePtrs& pp = sl.pp[side];
        const T* __restrict__ fin = static_cast<const T*>(sl.pop[side]);
        T* __restrict__ fout = static_cast<T*>(const_cast<void*>(sl.pop[side ^ 1]));
        const int y = ty * ROWS + threadIdx.y;
        if (y >= g.ny) continue;
        const size_t row = (size_t)z * g.ny + y;
        const int k = 2 * threadIdx.x;
        const int wd = 2 * bx + (k >> 5);
        const uint32_t bits = wd < g.wpr ? __ldg(sl.bits + row * g.wpr + wd) : 0u;
        const int x = 64 * bx + k;
        unsigned pair = (bits >> (k & 31)) & 3u;
        unsigned plane = 0;
        if (x == 0) {
            plane |= pair & 1u;
            pair &= ~1u;
        }
        if (x + 1 == g.nx - 1) {
            plane |= pair & 2u;
            pair &= ~2u;
        }
        if (!(pair | plane)) continue;
        const uint32_t c = (uint32_t)(row * g.nx + x);
        const bool face = (y == 0) | (y == g.ny - 1) | (z == 0) | (z == g.nz - 1);
        const bool edge = (bx == 0) | (64 * bx + 64 >= g.nx);
        if (plane) plane_cell<Q, S>(fin, fout, g, p, plane == 1u ? x : x + 1, plane == 1u ? c : (size_t)c + 1);
        if (!pair) continue;
        float2 v[Q];
        if (!face) {  // as k_bulk_pairs
            if (pair != 3u && !edge) {
                const uint32_t cc = pair == 1u ? c : c + 1u;
                bulk_cell<Q, S, false>(fin, fout, g, p, x + (pair == 1u ? 0 : 1), y, z, cc, sl.diverged);
                continue;
            }
            static_for<0, Q>([&](auto I) {
                constexpr int i = decltype(I)::value;
                const T* src = static_cast<const T*>(pp.src[i]);
                if constexpr (S::kExact) {
                    v[i] = L::ex(i) == 0 ? S::dec2(S::ld2(src + c), L::w(i))
                                         : make_float2(S::dec(S::ld(src + c), L::w(i)),
                                                       S::dec(S::ld(src + c + 1u), L::w(i)));
                } else {
                    v[i] = L::ex(i) == 0 ? S::raw2(S::ld2(src + c))
                                         : make_float2(S::raw(S::ld(src + c)), S::raw(S::ld(src + c + 1u)));
                }
            });
            if (collide_pair<Q, S>(v, p.tau, p.cs) & pair) atomicOr(sl.diverged, 1);
            store_pair<Q, S>(pp, c, v, pair);
            continue;
        }
        const bool va = pair & 1u, vb = pair & 2u;
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const int py = y - L::ey(i), pz = z - L::ez(i);
            const bool oy = py < 0 || py >= g.ny;
            const bool oz = pz < 0 || pz >= g.nz;
            const bool out = oy || oz;
            const int pl = out ? edge_plane<Q, i>(oy, oz, p) : i;
            const uint32_t off = out ? 0u : (uint32_t)link_offset<Q>(i, g);
            const uint32_t sa = va ? c - off : c;
            const uint32_t sb = vb ? c + 1u - off : c + 1u;
            const T* base = fin + (size_t)pl * g.n;
            if constexpr (S::kExact)
                v[i] = make_float2(S::dec(S::ld(base + sa), L::w(i)), S::dec(S::ld(base + sb), L::w(i)));
            else
                v[i] = make_float2(S::raw(S::ld(base + sa)), S::raw(S::ld(base + sb)));
        });
        const unsigned bad = collide_pair<Q, S>(v, p.tau, p.cs) & pair;
        if (bad) atomicOr(sl.diverged, 1);
        store_pair<Q, S>(pp, c, v, pair);
    }
    }
}

template <int Q, class S>
__global__ void __launch_bounds__(32 * kBulkRows) k_bulk_shell(const typename S::T* __restrict__ fin,
                                                                typename S::T* __restrict__ fout,
                                                                const uint32_t* __restrict__ bulk_bits, Geom g,
                                                                StepParams p, ShellPlan sp, int* __restrict__ diverged) {
    // one warp per (row, chunk) item of the shell
    unsigned long long item = (unsigned long long)blockIdx.x * kBulkRows + threadIdx.y;
    int chunk, y, z;
    if (item < sp.n_a) {  // Y-face rows, every chunk
        chunk = (int)(item % g.wpr);
        const unsigned long long r = item / g.wpr;
        y = sp.yf[(int)(r % sp.nyf)];
        z = sp.z0 + (int)(r / sp.nyf);
    } else if ((item -= sp.n_a) < sp.n_b) {  // Z-face rows off the Y faces, every chunk
        chunk = (int)(item % g.wpr);
        const unsigned long long r = item / g.wpr;
        y = 1 + (int)(r % sp.nyi);
        z = sp.zf[(int)(r / sp.nyi)];
    } else if ((item -= sp.n_b) < sp.n_c) {  // end chunks of interior rows
        chunk = sp.cend[(int)(item % sp.ncend)];
        const unsigned long long r = item / sp.ncend;
        y = 1 + (int)(r % sp.nyi);
        z = sp.zi0 + (int)(r / sp.nyi);
    } else {
        return;
    }
    const size_t row = (size_t)z * g.ny + y;
    const uint32_t bits = __ldg(bulk_bits + row * g.wpr + chunk);
    if (!((bits >> threadIdx.x) & 1u)) return;
    const int x = chunk * 32 + threadIdx.x;
    const uint32_t c = (uint32_t)(row * g.nx + x);
    bulk_cell<Q, S, true>(fin, fout, g, p, x, y, z, c, diverged);
}

// Boundary-list entries: fluid cells with a solid neighbour (off the
// inlet/outlet planes) and the solid cells an outlet reads. Every link's source
// address is formed with selects first and all loads issue together.
template <int Q, class S>
__device__ __forceinline__ void boundary_entry(const typename S::T* __restrict__ fin,
                                               typename S::T* __restrict__ fout, const BoundaryList& bl, uint32_t e,
                                               const Geom& g, const StepParams& p, int* __restrict__ diverged) {
    using L = Lattice<Q>;
    const uint32_t c = __ldg(bl.cells + e);
    const unsigned long long lk = __ldg(bl.links + e);
    const unsigned cls = (unsigned)(lk >> kClassShift) & 7u;
    const uint32_t nxy = (uint32_t)g.nxy;
    const uint32_t z = c / nxy;
    const uint32_t rem = c - z * nxy;
    const uint32_t y = rem / (uint32_t)g.nx;

    float f[Q];
    if (cls == kCellSolidFill) {  // solid cell: f_i = w_i (LbmReference.cpp:264-267)
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            store_pop_c<Q, S, i>(fout, g.n, c, L::w(i));
        });
        return;
    }
    // Fluid cell next to a wall (LbmReference.cpp:329-383).
    const uint32_t co0 = __ldg(bl.coef_off + e);
    uint32_t bzmask = 0;  // directions that carry a Bouzidi coefficient pair
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if ((((unsigned)(lk >> (3 * i))) & 6u) == 2u) bzmask |= 1u << i;
    });
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        constexpr int op = L::opp(i);
        const unsigned kind = (unsigned)(lk >> (3 * i)) & 7u;
        int pa = op;
        size_t sa = c;
        if (kind == kLinkStream) {
            pa = i;
            sa = (size_t)c - link_offset<Q>(i, g);
        } else if (kind == kLinkEdge) {
            const int py = (int)y - L::ey(i), pz = (int)z - L::ez(i);
            pa = edge_plane<Q, i>(py < 0 || py >= g.ny, pz < 0 || pz >= g.nz, p);
        }
        const float va = load_plane<Q, S>(fin, pa, g.n, sa, L::w(i));
        float v = va;
        if (kind == kLinkBzNear || kind == kLinkBzFar) {
            const float2 k = __ldg(bl.coef + co0 + __popc(bzmask & ((1u << i) - 1u)));
            const int pb = kind == kLinkBzNear ? op : i;
            const size_t sb = kind == kLinkBzNear ? (size_t)c + link_offset<Q>(i, g) : (size_t)c;
            const float vb = load_plane<Q, S>(fin, pb, g.n, sb, L::w(i));
            v = k.x * va + k.y * vb;
        }
        f[i] = v;
    });
    if (collide<Q, S::kExact>(f, p.tau, p.cs)) atomicOr(diverged, 1);
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
    const uint32_t e = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= end) return;
    boundary_entry<Q, S>(fin, fout, bl, e, g, p, diverged);
}

// The boundary-list entries of every lattice of a batch in one launch: a
// thread takes one entry of the concatenated lists and finds its lattice by
// binary search over the lattices' first entries.
template <int Q, class S>
__global__ void __launch_bounds__(128) k_boundary_pull_batch(const BatchLattice* __restrict__ lat, int nlat,
                                                              unsigned long long total, int parity) {
    const unsigned long long w = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= total) return;
    int lo = 0, hi = nlat - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&lat[mid].bnd_first) <= w) lo = mid;
        else hi = mid - 1;
    }
    const BatchLattice& L = lat[lo];
    const int side = L.cur ^ parity;
    boundary_entry<Q, S>(static_cast<const typename S::T*>(L.pop[side]),
                         static_cast<typename S::T*>(const_cast<void*>(L.pop[side ^ 1])), L.bl,
                         (uint32_t)(w - L.bnd_first), L.g, L.p, L.diverged);
}

// k_boundary_pull with the learned closure (16-bit offset storage): the same
// link handling in float populations, then the two-phase collision on
// offsets (f - w) * 2^8 with the warp-wide closure. Every lane of a warp runs
// the closure; only live fluid entries store.
template <int Q, class S>
__global__ void __launch_bounds__(128) k_boundary_pull_learned(const typename S::T* __restrict__ fin,
                                                                typename S::T* __restrict__ fout, BoundaryList bl,
                                                                uint32_t begin, uint32_t end, Geom g, StepParams p,
                                                                int* __restrict__ diverged, ClosureDev cl) {
    static_assert(!S::kExact, "the learned closure runs on the 16-bit offset formats");
    using L = Lattice<Q>;
    __shared__ uint32_t s_in[4][32 * 8];
    __shared__ float2 s_out[4][32];
    const uint32_t e = begin + blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = e < end;
    const uint32_t c = live ? __ldg(bl.cells + e) : 0u;
    const unsigned long long lk = live ? __ldg(bl.links + e) : 0ull;
    const unsigned cls = (unsigned)(lk >> kClassShift) & 7u;
    const bool fluid = live && cls != kCellSolidFill;
    if (live && !fluid) {  // solid cell: f_i = w_i (LbmReference.cpp:264-267)
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            store_pop_c<Q, S, i>(fout, g.n, c, L::w(i));
        });
    }
    const uint32_t nxy = (uint32_t)g.nxy;
    const uint32_t z = c / nxy;
    const uint32_t rem = c - z * nxy;
    const uint32_t y = rem / (uint32_t)g.nx;
    float2 h[Q];
    if (fluid) {
        const uint32_t co0 = __ldg(bl.coef_off + e);
        uint32_t bzmask = 0;
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            if ((((unsigned)(lk >> (3 * i))) & 6u) == 2u) bzmask |= 1u << i;
        });
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            constexpr int op = L::opp(i);
            const unsigned kind = (unsigned)(lk >> (3 * i)) & 7u;
            int pa = op;
            size_t sa = c;
            if (kind == kLinkStream) {
                pa = i;
                sa = (size_t)c - link_offset<Q>(i, g);
            } else if (kind == kLinkEdge) {
                const int py = (int)y - L::ey(i), pz = (int)z - L::ez(i);
                pa = edge_plane<Q, i>(py < 0 || py >= g.ny, pz < 0 || pz >= g.nz, p);
            }
            const float va = load_plane<Q, S>(fin, pa, g.n, sa, L::w(i));
            float v = va;
            if (kind == kLinkBzNear || kind == kLinkBzFar) {
                const float2 kk = __ldg(bl.coef + co0 + __popc(bzmask & ((1u << i) - 1u)));
                const int pb = kind == kLinkBzNear ? op : i;
                const size_t sb = kind == kLinkBzNear ? (size_t)c + link_offset<Q>(i, g) : (size_t)c;
                const float vb = load_plane<Q, S>(fin, pb, g.n, sb, L::w(i));
                v = kk.x * va + kk.y * vb;
            }
            h[i] = make_float2((v - L::w(i)) * 256.0f, 0.0f);
        });
    } else {
        static_for<0, Q>([&](auto I) { h[decltype(I)::value] = make_float2(0.0f, 0.0f); });
    }
    Mom2 mo;
    const unsigned bad = moments2<Q>(h, mo) & (fluid ? 1u : 0u);
    float x0, x1, x2;
    closure_invariants(mo.pxx.x, mo.pyy.x, mo.pzz.x, mo.pxy.x, mo.pxz.x, mo.pyz.x, mo.pp.x, mo.inv.x, x0, x1, x2);
    const float x3 = fluid ? (float)__ldg(cl.wall + c) * 0.0625f : 0.0f;
    const bool lin = fluid && closure_wall_ok(cl, __ldg(cl.wall + c)) && closure_in_range(cl, x0, x1, x2);
    const float sg = smagorinsky_g(mo.pp.x, mo.rho.x, mo.inv.x, p.tau, p.cs);
    const float ds = closure_anchored(cl) ? smagorinsky_d3(mo.pp.x, mo.rho.x, mo.inv.x, p.tau, p.cs) : 0.0f;
    const int warp = threadIdx.x >> 5;
    uint32_t* in = &s_in[warp][(threadIdx.x & 31) * 8];
    closure_pack_inputs(cl, x0, x1, x2, x3, in);
    closure_pack_inputs(cl, 0.0f, 0.0f, 0.0f, 0.0f, in + 4);
    __syncwarp();
    float2 nu = make_float2(0.0f, 0.0f);  // warps with no cell in range skip the MLP
    if (__any_sync(0xffffffffu, lin)) nu = closure_warp_mlp(cl.frag, s_in[warp], s_out[warp]);
    if (!fluid) return;
    const float gx = lin ? closure_g(cl, nu.x, p.tau, ds) : sg;
    relax2<Q>(h, mo, make_float2(gx, gx));
    if (bad) atomicOr(diverged, 1);
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        store_pop_c<Q, S, i>(fout, g.n, c, L::w(i) + h[i].x * (1.0f / 256.0f));
    });
}

// Plane pointers of a ping-pong step (PlanePtrs in lbm_internal.h).
template <int Q, class S>
static PlanePtrs pp_of(const void* fin, void* fout, const Geom& g) {
    PlanePtrs pp{};
    for (int i = 0; i < Q; ++i) {
        const long long off = (long long)Lattice<Q>::ex(i) + (long long)Lattice<Q>::ey(i) * g.nx +
                              (long long)Lattice<Q>::ez(i) * g.nxy;
        pp.src[i] = (const typename S::T*)fin + ((long long)i * (long long)g.n - off);
        pp.dst[i] = (typename S::T*)fout + (size_t)i * g.n;
    }
    return pp;
}

template <int Q, class S>
static cudaError_t bulk_t(const void* fin, void* fout, const uint32_t* bits, const Geom& g, const StepParams& p,
                          int z0, int zc, int* dv, cudaStream_t s, int* launched, int staged) {
    *launched = 0;
    if (zc <= 0) return cudaSuccess;
    const int z1 = z0 + zc;
    dim3 block(32, kBulkRows, 1);
    if (g.nx % 2 == 0) {  // pairs start on even cells: every row through k_bulk_pairs
        PairsShell sh{};
        if (staged) {  // the interior warps' rows staged in shared memory by TMA
            int nl = 0;
            cudaError_t e = launch_bulk_staged(Q, storage_code<S>(), fin, fout, bits, g, p, z0, zc, dv, s, &nl);
            if (e != cudaSuccess) return e;
            *launched += nl;
            sh.gx = (g.nx + 63) / 64;
            sh.nyb = (g.ny + kBulkRows - 1) / kBulkRows;
            sh.z0 = z0;
            sh.zi0 = z0 > 1 ? z0 : 1;
            const int zi1 = z1 < g.nz - 1 ? z1 : g.nz - 1;
            sh.nyf = sh.nyb >= 2 ? 2 : 1;
            sh.nzf = 0;
            if (z0 <= 0 && 0 < z1) sh.zf[sh.nzf++] = 0;
            if (g.nz > 1 && z0 <= g.nz - 1 && g.nz - 1 < z1) sh.zf[sh.nzf++] = g.nz - 1;
            sh.ne = 2ull * sh.nyb * zc;
            sh.nf = zi1 > sh.zi0 ? (unsigned long long)(sh.gx - 2) * sh.nyf * (zi1 - sh.zi0) : 0ull;
            const unsigned long long ng = (unsigned long long)(sh.gx - 2) * sh.nyb * sh.nzf;
            sh.n = sh.ne + sh.nf + ng;
            if (sh.n == 0) return cudaSuccess;
            k_bulk_pairs<Q, S><<<(unsigned)sh.n, block, 0, s>>>((const typename S::T*)fin, (typename S::T*)fout, bits, g,
                                                                p, pp_of<Q, S>(fin, fout, g), z0, dv, sh);
            ++*launched;
            return cudaGetLastError();
        }
        dim3 grid((unsigned)((g.nx + 63) / 64), (unsigned)((g.ny + kBulkRows - 1) / kBulkRows), (unsigned)zc);
        k_bulk_pairs<Q, S><<<grid, block, 0, s>>>((const typename S::T*)fin, (typename S::T*)fout, bits, g, p,
                                                  pp_of<Q, S>(fin, fout, g), z0, dv, sh);
        ++*launched;
        return cudaGetLastError();
    }
    // odd nx: one-cell interior kernel + shell kernel (planes ride in the shell's row-end warps)
    const int zi0 = z0 > 1 ? z0 : 1, zi1 = z1 < g.nz - 1 ? z1 : g.nz - 1;
    if (g.wpr > 2 && g.ny > 2 && zi1 > zi0) {
        const unsigned gy = (unsigned)((g.ny - 2 + kBulkRows - 1) / kBulkRows);
        dim3 grid((unsigned)(g.wpr - 2), gy, (unsigned)(zi1 - zi0));
        k_bulk_interior<Q, S><<<grid, block, 0, s>>>((const typename S::T*)fin, (typename S::T*)fout, bits, g, p, zi0,
                                                     dv);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        ++*launched;
    }
    ShellPlan sp{};
    sp.z0 = z0;
    sp.nyf = 0;
    sp.yf[sp.nyf++] = 0;
    if (g.ny > 1) sp.yf[sp.nyf++] = g.ny - 1;
    sp.nyi = g.ny > 2 ? g.ny - 2 : 0;
    sp.nzf = 0;
    if (z0 <= 0 && 0 < z1) sp.zf[sp.nzf++] = 0;
    if (g.nz > 1 && z0 <= g.nz - 1 && g.nz - 1 < z1) sp.zf[sp.nzf++] = g.nz - 1;
    sp.zi0 = zi0;
    sp.ncend = 0;
    sp.cend[sp.ncend++] = 0;
    if (g.wpr > 1) sp.cend[sp.ncend++] = g.wpr - 1;
    sp.n_a = (unsigned long long)sp.nyf * zc * g.wpr;
    sp.n_b = (unsigned long long)sp.nzf * sp.nyi * g.wpr;
    sp.n_c = zi1 > zi0 ? (unsigned long long)(zi1 - zi0) * sp.nyi * sp.ncend : 0ull;
    const unsigned long long items = sp.n_a + sp.n_b + sp.n_c;
    if (items == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((items + kBulkRows - 1) / kBulkRows);
    k_bulk_shell<Q, S><<<blocks, block, 0, s>>>((const typename S::T*)fin, (typename S::T*)fout, bits, g, p, sp, dv);
    ++*launched;
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

template <int Q, class S>
static cudaError_t bulk_learned_t(const void* fin, void* fout, const uint32_t* bits, const Geom& g,
                                  const StepParams& p, int z0, int zc, int* dv, cudaStream_t s, int* launched,
                                  const ClosureDev& cl, int tc) {
    *launched = 0;
    if constexpr (S::kExact) {
        return cudaErrorNotSupported;
    } else {
        if (zc <= 0) return cudaSuccess;
        if (g.nx % 2 != 0) return cudaErrorNotSupported;
        PlanePtrs pp{};
        for (int i = 0; i < Q; ++i) {
            const long long off = (long long)Lattice<Q>::ex(i) + (long long)Lattice<Q>::ey(i) * g.nx +
                                  (long long)Lattice<Q>::ez(i) * g.nxy;
            pp.src[i] = (const typename S::T*)fin + ((long long)i * (long long)g.n - off);
            pp.dst[i] = (typename S::T*)fout + (size_t)i * g.n;
        }
        dim3 block(32, kBulkRows, 1);
        dim3 grid((unsigned)((g.nx + 63) / 64), (unsigned)((g.ny + kBulkRows - 1) / kBulkRows), (unsigned)zc);
        if (tc)
            k_bulk_pairs_learned_tc<Q, S><<<grid, block, 0, s>>>((const typename S::T*)fin, (typename S::T*)fout,
                                                                 bits, g, p, pp, z0, dv, cl);
        else
            k_bulk_pairs_learned<Q, S><<<grid, block, 0, s>>>((const typename S::T*)fin, (typename S::T*)fout, bits,
                                                              g, p, pp, z0, dv, cl);
        ++*launched;
        return cudaGetLastError();
    }
}

template <int Q, class S>
static cudaError_t boundary_learned_t(const void* fin, void* fout, const BoundaryList& bl, uint32_t b, uint32_t e,
                                      const Geom& g, const StepParams& p, int* dv, cudaStream_t s,
                                      const ClosureDev& cl) {
    if constexpr (S::kExact) {
        return cudaErrorNotSupported;
    } else {
        if (e <= b) return cudaSuccess;
        const unsigned threads = 128;
        const unsigned blocks = (e - b + threads - 1) / threads;
        k_boundary_pull_learned<Q, S><<<blocks, threads, 0, s>>>((const typename S::T*)fin, (typename S::T*)fout, bl,
                                                                 b, e, g, p, dv, cl);
        return cudaGetLastError();
    }
}

template <int Q, class S>
static cudaError_t closure_probe_t(const void* f, const uint8_t* solid, const Geom& g, const ClosureDev& cl,
                                   float* out, uint8_t* in_range, unsigned long long* counts, int layout,
                                   cudaStream_t s) {
    if constexpr (S::kExact) {
        return cudaErrorNotSupported;
    } else {
        const size_t pairs = (g.n + 1) / 2;
        k_closure_probe<Q, S><<<(unsigned)((pairs + 127) / 128), 128, 0, s>>>((const typename S::T*)f, solid, g, cl,
                                                                              out, in_range, counts, layout);
        return cudaGetLastError();
    }
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
                             const Geom& g, const StepParams& p, int z0, int zc, int* diverged, cudaStream_t s,
                             int* launched, int staged) {
    const int st = staged && g.nx % 2 == 0 && staged_eligible(storage, g) ? 1 : 0;
    FC_DISPATCH(q, storage, bulk_t, fin, fout, bulk_bits, g, p, z0, zc, diverged, s, launched, st);
}

cudaError_t launch_boundary_pull(int q, int storage, const void* fin, void* fout, const BoundaryList& bl,
                                 uint32_t begin, uint32_t end, const Geom& g, const StepParams& p, int* diverged,
                                 cudaStream_t s) {
    FC_DISPATCH(q, storage, boundary_t, fin, fout, bl, begin, end, g, p, diverged, s);
}

cudaError_t launch_bulk_pull_learned(int q, int storage, const void* fin, void* fout, const uint32_t* bulk_bits,
                                     const Geom& g, const StepParams& p, int z0, int zc, int* diverged,
                                     cudaStream_t s, int* launched, const ClosureDev& cl, int tc) {
    FC_DISPATCH(q, storage, bulk_learned_t, fin, fout, bulk_bits, g, p, z0, zc, diverged, s, launched, cl, tc);
}

cudaError_t launch_boundary_pull_learned(int q, int storage, const void* fin, void* fout, const BoundaryList& bl,
                                         uint32_t begin, uint32_t end, const Geom& g, const StepParams& p,
                                         int* diverged, cudaStream_t s, const ClosureDev& cl) {
    FC_DISPATCH(q, storage, boundary_learned_t, fin, fout, bl, begin, end, g, p, diverged, s, cl);
}

template <int Q, class S>
static cudaError_t bulk_batch_t(int rows, const BatchLattice* lat, int nlat, unsigned long long total, int parity,
                                int grid, cudaStream_t s) {
    if (total == 0) return cudaSuccess;
    if (rows == 4)
        k_bulk_pairs_batch<Q, S, 4><<<grid, dim3(32, 4), 0, s>>>(lat, nlat, total, parity);
    else if (rows == 8)
        k_bulk_pairs_batch<Q, S, 8><<<grid, dim3(32, 8), 0, s>>>(lat, nlat, total, parity);
    else if (rows == 16)
        k_bulk_pairs_batch<Q, S, 16><<<grid, dim3(32, 16), 0, s>>>(lat, nlat, total, parity);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

template <int Q, class S>
static cudaError_t bulk_tiles_t(const TileLaunch& t, cudaStream_t s) {
    if (t.tiles == 0) return cudaSuccess;
    if (t.nlat < 1 || t.nlat > kTileLaunchLattices || t.tiles > 0x7fffffffu) return cudaErrorInvalidValue;
    k_bulk_pairs_tiles<Q, S><<<t.tiles, dim3(32, kBulkRows), 0, s>>>(t);
    return cudaGetLastError();
}

cudaError_t launch_bulk_tiles(int q, int storage, const TileLaunch& t, cudaStream_t s) {
    FC_DISPATCH(q, storage, bulk_tiles_t, t, s);
}

template <int Q, class S>
static cudaError_t batch_resident_t(int rows, int* nb) {
    if (rows == 4) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(nb, k_bulk_pairs_batch<Q, S, 4>, 128, 0);
    if (rows == 8) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(nb, k_bulk_pairs_batch<Q, S, 8>, 256, 0);
    if (rows == 16) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(nb, k_bulk_pairs_batch<Q, S, 16>, 512, 0);
    return cudaErrorInvalidValue;
}

cudaError_t launch_bulk_batch(int q, int storage, int rows, const BatchLattice* lat, int nlat,
                              unsigned long long total, int parity, int grid, cudaStream_t s) {
    FC_DISPATCH(q, storage, bulk_batch_t, rows, lat, nlat, total, parity, grid, s);
}

template <int Q, class S>
static cudaError_t boundary_batch_t(const BatchLattice* lat, int nlat, unsigned long long total, int parity,
                                    cudaStream_t s) {
    if (total == 0) return cudaSuccess;
    k_boundary_pull_batch<Q, S><<<(unsigned)((total + 127) / 128), 128, 0, s>>>(lat, nlat, total, parity);
    return cudaGetLastError();
}

cudaError_t launch_boundary_batch(int q, int storage, const BatchLattice* lat, int nlat, unsigned long long total,
                                  int parity, cudaStream_t s) {
    FC_DISPATCH(q, storage, boundary_batch_t, lat, nlat, total, parity, s);
}

static cudaError_t batch_resident_dispatch(int q, int storage, int rows, int* nb) {
    FC_DISPATCH(q, storage, batch_resident_t, rows, nb);
}

int bulk_batch_resident(int q, int storage, int rows) {
    int nb = 0;
    return batch_resident_dispatch(q, storage, rows, &nb) == cudaSuccess ? nb : 0;
}

cudaError_t launch_closure_probe(int q, int storage, const void* f, const uint8_t* solid, const Geom& g,
                                 const ClosureDev& cl, float* out, uint8_t* in_range, unsigned long long* counts,
                                 int layout, cudaStream_t s) {
    FC_DISPATCH(q, storage, closure_probe_t, f, solid, g, cl, out, in_range, counts, layout, s);
}

}  // namespace fc
