// The LBM step on one population set updated in place with the AA pattern
// (the layouts and the argument that no two threads touch one slot are in
// aa.cuh). The kernels mirror the ping-pong ones of lbm_step.cu cell for
// cell: the same classification, the same collision of a cell pair or a
// single cell, the same boundary-link handling and inlet / outlet rules, so
// every stored value is the one the ping-pong step stores; only the slots
// change.
//
//   k_bulk_pairs_aa   bulk cells, two x-adjacent cells per thread. An even
//                     step reads and writes each cell's own slots (aligned
//                     pair loads and stores in every direction); an odd step
//                     pulls from the upstream cells and pushes to the
//                     downstream ones (aligned pairs for e_x = 0, element
//                     accesses otherwise). Row-end warps take the same
//                     loads plus the inlet / outlet rules; face warps take
//                     the general path with the edge rules.
//   k_boundary_aa     the boundary list. The Bouzidi far-side partner
//                     f*_i(c), which the pulling cell c + e_i overwrites in
//                     place, comes from the side buffer the entry itself
//                     filled last step.
//   k_aa_prime_*      fill the side buffers from a state set by a seed or
//                     a population load.
//   *_learned         the bulk and boundary kernels with the learned
//                     closure (16-bit formats), the same slots around the
//                     collision and warp-wide MLP of the ping-pong learned
//                     kernels.
//
// Outlet moments: the outlet reads the moments of its upstream neighbour's
// post-collision populations (LbmReference.cpp:275-327), which in place sit
// in other threads' slots. The cells at x = 1 and x = nx-2 (both flow
// directions) write the moments of what they store into a per-row buffer;
// a step of parity k reads buffer k and writes buffer k ^ 1.
#include "aa.cuh"
#include "closure.cuh"
#include "step_common.cuh"

namespace fc {

namespace {

template <class S>
__device__ __forceinline__ typename S::T ld_plain(const typename S::T* p) {
    return *p;  // a coherent load: the kernel writes the same array
}
template <class S>
__device__ __forceinline__ typename S::T2 ld2_plain(const typename S::T* p) {
    return *reinterpret_cast<const typename S::T2*>(p);
}

__device__ __forceinline__ size_t outm_index(const AaSide& sd, int par, int col, size_t row) {
    return ((size_t)par * 2 + (size_t)col) * sd.rows + row;
}

// Moments of the values a ping-pong read would decode from what is stored
// for post-collision values f (full floats).
template <int Q, class S>
__device__ __forceinline__ float4 stored_moments(const float (&f)[Q]) {
    float d[Q];
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        d[i] = S::dec(S::enc(f[i], Lattice<Q>::w(i)), Lattice<Q>::w(i));
    });
    float r, u, v, w;
    moments<Q>(d, r, u, v, w);
    return make_float4(r, u, v, w);
}

// The two cells' decoded stored values after collide_pair (v holds full
// floats for the exact format, scaled offsets for the 16-bit ones).
template <int Q, class S>
__device__ __forceinline__ void pair_stored(const float2 (&v)[Q], float (&a)[Q], float (&b)[Q]) {
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if constexpr (S::kExact) {
            a[i] = v[i].x;
            b[i] = v[i].y;
        } else {
            const typename S::T2 h = S::pack2(v[i].x, v[i].y);
            a[i] = S::dec(h.x, Lattice<Q>::w(i));
            b[i] = S::dec(h.y, Lattice<Q>::w(i));
        }
    });
}

template <int Q>
__device__ __forceinline__ float4 plain_moments(const float (&d)[Q]) {
    float r, u, v, w;
    moments<Q>(d, r, u, v, w);
    return make_float4(r, u, v, w);
}

// Column of the outlet-moment buffer a cell at x feeds, or -1.
__device__ __forceinline__ int outm_col(int x, const Geom& g) { return x == 1 ? 0 : (x == g.nx - 2 ? 1 : -1); }

// Slot of f*_i(c) that the step writes: even, plane opp(i) of c; odd, plane i
// of c + e_i, or plane opp(i) of c when c + e_i is off the lattice.
template <int Q, int I, bool Odd>
__device__ __forceinline__ size_t out_slot(uint32_t c, int x, int y, int z, const Geom& g) {
    using L = Lattice<Q>;
    if constexpr (Odd) {
        const int tx = x + L::ex(I), ty = y + L::ey(I), tz = z + L::ez(I);
        if (tx >= 0 && ty >= 0 && tz >= 0 && tx < g.nx && ty < g.ny && tz < g.nz)
            return (size_t)I * g.n + (size_t)((long long)c + link_offset<Q>(I, g));
    }
    return (size_t)L::opp(I) * g.n + c;
}

// One interior bulk cell (the one-cell path of k_bulk_pairs).
template <int Q, class S, bool Odd>
__device__ __forceinline__ void aa_interior_cell(typename S::T* f, const Geom& g, const StepParams& p, uint32_t c,
                                                 int* __restrict__ diverged) {
    using L = Lattice<Q>;
    float v[Q];
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const size_t s = Odd ? (size_t)L::opp(i) * g.n + (size_t)((long long)c - link_offset<Q>(i, g))
                             : (size_t)i * g.n + c;
        v[i] = S::dec(ld_plain<S>(f + s), L::w(i));
    });
    if (collide<Q, S::kExact>(v, p.tau, p.cs)) atomicOr(diverged, 1);
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const size_t d = Odd ? (size_t)i * g.n + (size_t)((long long)c + link_offset<Q>(i, g))
                             : (size_t)L::opp(i) * g.n + c;
        f[d] = S::enc(v[i], L::w(i));
    });
}

// One inlet or outlet cell (plane_cell of lbm_step.cu).
template <int Q, class S, bool Odd>
__device__ __forceinline__ void aa_plane_cell(typename S::T* f, const Geom& g, const StepParams& p, const AaSide& sd,
                                              int x, int y, int z, uint32_t c, size_t row) {
    using L = Lattice<Q>;
    float v[Q];
    if (x == p.inlet_x) {
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            v[i] = p.feq_inlet[i];
        });
    } else {
        const float4 m = sd.outm[outm_index(sd, Odd ? 1 : 0, p.reverse ? 0 : 1, row)];
        const float rho = m.x > 1e-6f ? 1.0f + 0.999f * (m.x - 1.0f) : 1.0f;
        equilibrium_all<Q>(rho, m.y, m.z, m.w, v);
    }
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        f[out_slot<Q, i, Odd>(c, x, y, z, g)] = S::enc(v[i], L::w(i));
    });
}

// aa_plane_cell for the 16-bit formats by the whole warp: lane i < Q takes
// population i of the cell (the equilibrium for its run-time direction and
// its slot), so the cell's Q stores are one instruction for the warp. The
// values are aa_plane_cell's. Every lane of the warp calls aa_row_end_cells
// together; `plane` holds this lane's bits (1: cell x, 2: cell x + 1).
template <int Q, class S, bool Odd>
__device__ __forceinline__ void aa_row_end_cell(typename S::T* f, const Geom& g, const StepParams& p,
                                                const AaSide& sd, int px, int y, int z, uint32_t pc, size_t row) {
    const unsigned lane = threadIdx.x & 31;
    const bool mine = lane < (unsigned)Q;
    const unsigned i = mine ? lane : 0u;
    float v;
    if (px == p.inlet_x) {
        const float ux = p.inlet_ux;
        v = equilibrium_rt<Q>(i, 1.0f, ux, 0.0f, 0.0f, speed2(ux, 0.0f, 0.0f));
    } else {
        const float4 m = sd.outm[outm_index(sd, Odd ? 1 : 0, p.reverse ? 0 : 1, row)];
        const float rho = m.x > 1e-6f ? 1.0f + 0.999f * (m.x - 1.0f) : 1.0f;
        v = equilibrium_rt<Q>(i, rho, m.y, m.z, m.w, speed2(m.y, m.z, m.w));
    }
    // the slot out_slot<Q, i, Odd> names, for the run-time direction
    const unsigned opp = i == 0 ? 0u : ((i - 1u) ^ 1u) + 1u;
    size_t slot = (size_t)opp * g.n + pc;
    if constexpr (Odd) {
        const int ex = (int)lattice_e_rt<Q, 0>(i), ey = (int)lattice_e_rt<Q, 1>(i), ez = (int)lattice_e_rt<Q, 2>(i);
        const int tx = px + ex, ty = y + ey, tz = z + ez;
        if (tx >= 0 && ty >= 0 && tz >= 0 && tx < g.nx && ty < g.ny && tz < g.nz)
            slot = (size_t)i * g.n + (size_t)((long long)pc + ex + (long long)ey * g.nx + (long long)ez * g.nxy);
    }
    if (mine) f[slot] = S::enc(v, lattice_w_rt<Q>(i));
}

template <int Q, class S, bool Odd>
__device__ __forceinline__ void aa_row_end_cells(typename S::T* f, const Geom& g, const StepParams& p,
                                                 const AaSide& sd, unsigned plane, int x, int y, int z, uint32_t c,
                                                 size_t row) {
    unsigned m = __ballot_sync(0xffffffffu, plane != 0u);
    while (m) {  // uniform: at most the two row ends
        const int src = __ffs(m) - 1;
        m &= m - 1u;
        const unsigned sp = __shfl_sync(0xffffffffu, plane, src);
        const int sx = __shfl_sync(0xffffffffu, x, src);
        const uint32_t sc = __shfl_sync(0xffffffffu, c, src);
        if (sp & 1u) aa_row_end_cell<Q, S, Odd>(f, g, p, sd, sx, y, z, sc, row);
        if (sp & 2u) aa_row_end_cell<Q, S, Odd>(f, g, p, sd, sx + 1, y, z, sc + 1u, row);
    }
}

}  // namespace

// Bulk cells (bulk mask) of lattices with even nx; see the file comment.
template <int Q, class S, bool Odd>
__global__ void __launch_bounds__(32 * kBulkRows, 4) k_bulk_pairs_aa(typename S::T* f,
                                                                   const uint32_t* __restrict__ bulk_bits, Geom g,
                                                                   StepParams p, PlanePtrs pp, int z0,
                                                                   int* __restrict__ diverged, AaSide sd) {
    using L = Lattice<Q>;
    using T = typename S::T;
    using T2 = typename S::T2;
    const int y = blockIdx.y * kBulkRows + threadIdx.y;
    const int z = z0 + blockIdx.z;
    if (y >= g.ny) return;
    const size_t row = (size_t)z * g.ny + y;
    const int k = 2 * threadIdx.x;
    const int w = 2 * blockIdx.x + (k >> 5);
    const uint32_t bits = w < g.wpr ? __ldg(bulk_bits + row * g.wpr + w) : 0u;
    const int x = 64 * blockIdx.x + k;
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
    if constexpr (!S::kExact) {  // the row-end cells by the whole warp
        aa_row_end_cells<Q, S, Odd>(f, g, p, sd, plane, x, y, z, c, row);
        plane = 0;
    }
    if (!(pair | plane)) return;
    const bool face = (y == 0) | (y == g.ny - 1) | (z == 0) | (z == g.nz - 1);
    const bool edge = (blockIdx.x == 0) | (64 * (int)blockIdx.x + 64 >= g.nx);

    float2 v[Q];
    if (!face) {
        // Off the Y/Z faces every source slot of a row lies inside the set,
        // also for a cell this lane does not store (the inlet / outlet cell of
        // a row end, a wall cell), so row-end warps take the same loads; their
        // partial pairs keep the masked pair collision of the ping-pong step.
        if (pair != 3u && !edge) {
            aa_interior_cell<Q, S, Odd>(f, g, p, pair == 1u ? c : c + 1u, diverged);
            return;
        }
        if (plane) {
            const int px = plane == 1u ? x : x + 1;
            aa_plane_cell<Q, S, Odd>(f, g, p, sd, px, y, z, plane == 1u ? c : c + 1u, row);
        }
        if (!pair) return;
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const T* src = static_cast<const T*>(pp.src[i]);
            if (!Odd || L::ex(i) == 0) {
                const T2 h = ld2_plain<S>(src + c);
                if constexpr (S::kExact)
                    v[i] = S::dec2(h, L::w(i));
                else
                    v[i] = S::raw2(h);
            } else {
                const T ha = ld_plain<S>(src + c), hb = ld_plain<S>(src + c + 1u);
                if constexpr (S::kExact)
                    v[i] = make_float2(S::dec(ha, L::w(i)), S::dec(hb, L::w(i)));
                else
                    v[i] = make_float2(S::raw(ha), S::raw(hb));
            }
        });
        if (collide_pair<Q, S>(v, p.tau, p.cs) & pair) atomicOr(diverged, 1);
        if (pair == 3u) {
            static_for<0, Q>([&](auto I) {
                constexpr int i = decltype(I)::value;
                T* dst = static_cast<T*>(pp.dst[i]);
                T2 h;
                if constexpr (S::kExact)
                    h = S::enc2(v[i].x, v[i].y, L::w(i));
                else
                    h = S::pack2(v[i].x, v[i].y);
                if (!Odd || L::ex(i) == 0) {
                    *reinterpret_cast<T2*>(dst + c) = h;
                } else {
                    dst[c] = h.x;
                    dst[c + 1u] = h.y;
                }
            });
        } else {  // a partial pair of a row-end warp: its valid cell only (pair is 1 or 2)
            const uint32_t ec = pair == 1u ? c : c + 1u;
            static_for<0, Q>([&](auto I) {
                constexpr int i = decltype(I)::value;
                if constexpr (S::kExact) {
                    const T2 h = S::enc2(v[i].x, v[i].y, L::w(i));
                    T* dst = static_cast<T*>(pp.dst[i]) + c;
                    if (pair & 1u) dst[0] = h.x;
                    if (pair & 2u) dst[1] = h.y;
                } else {
                    const T2 h = S::pack2(v[i].x, v[i].y);
                    static_cast<T*>(pp.dst[i])[ec] = pair == 1u ? h.x : h.y;
                }
            });
        }
        if (edge) {  // upstream-neighbour moments for the outlets of both flow directions
            const int ca = (pair & 1u) ? outm_col(x, g) : -1, cb = (pair & 2u) ? outm_col(x + 1, g) : -1;
            if (ca >= 0 || cb >= 0) {
                float a[Q], b[Q];
                pair_stored<Q, S>(v, a, b);
                if (ca >= 0) sd.outm[outm_index(sd, Odd ? 0 : 1, ca, row)] = plain_moments<Q>(a);
                if (cb >= 0) sd.outm[outm_index(sd, Odd ? 0 : 1, cb, row)] = plain_moments<Q>(b);
            }
        }
        return;
    }
    // general pair path (face rows)
    if (plane) {
        const int px = plane == 1u ? x : x + 1;
        aa_plane_cell<Q, S, Odd>(f, g, p, sd, px, y, z, plane == 1u ? c : c + 1u, row);
    }
    if (!pair) return;
    const bool va = pair & 1u, vb = pair & 2u;
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const int py = y - L::ey(i), pz = z - L::ez(i);
        const bool oy = py < 0 || py >= g.ny;
        const bool oz = pz < 0 || pz >= g.nz;
        const bool out = oy || oz;  // the same for the whole row
        // off the edge: the mirrored / bounced population of the cell itself,
        // kept in its own opposite slot in both layouts
        const int m = out ? edge_plane<Q, i>(oy, oz, p) : i;
        const int rplane = out ? L::opp(m) : (Odd ? L::opp(i) : i);
        const uint32_t off = (out || !Odd) ? 0u : (uint32_t)link_offset<Q>(i, g);
        const uint32_t sa = va ? c - off : c;
        const uint32_t sb = vb ? c + 1u - off : c + 1u;
        const T* base = f + (size_t)rplane * g.n;
        const T ha = ld_plain<S>(base + sa), hb = ld_plain<S>(base + sb);
        if constexpr (S::kExact)
            v[i] = make_float2(S::dec(ha, L::w(i)), S::dec(hb, L::w(i)));
        else
            v[i] = make_float2(S::raw(ha), S::raw(hb));
    });
    const unsigned bad = collide_pair<Q, S>(v, p.tau, p.cs) & pair;
    if (bad) atomicOr(diverged, 1);
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        T2 h;
        if constexpr (S::kExact)
            h = S::enc2(v[i].x, v[i].y, L::w(i));
        else
            h = S::pack2(v[i].x, v[i].y);
        // pair cells never sit on x = 0 or x = nx-1, so only y / z can leave
        const int ty = y + L::ey(i), tz = z + L::ez(i);
        const bool inside = ty >= 0 && ty < g.ny && tz >= 0 && tz < g.nz;
        const bool push = Odd && inside;
        T* dst = f + (push ? (size_t)i * g.n + (size_t)((long long)c + link_offset<Q>(i, g))
                           : (size_t)L::opp(i) * g.n + c);
        if (pair == 3u && (!push || L::ex(i) == 0)) {
            *reinterpret_cast<T2*>(dst) = h;
        } else {
            if (va) dst[0] = h.x;
            if (vb) dst[1] = h.y;
        }
    });
    // upstream-neighbour moments for the outlets of both flow directions
    const int ca = va ? outm_col(x, g) : -1, cb = vb ? outm_col(x + 1, g) : -1;
    if (ca >= 0 || cb >= 0) {
        float a[Q], b[Q];
        pair_stored<Q, S>(v, a, b);
        if (ca >= 0) sd.outm[outm_index(sd, Odd ? 0 : 1, ca, row)] = plain_moments<Q>(a);
        if (cb >= 0) sd.outm[outm_index(sd, Odd ? 0 : 1, cb, row)] = plain_moments<Q>(b);
    }
}

// Boundary-list entries (boundary_entry of lbm_step.cu, in place).
template <int Q, class S, bool Odd>
__global__ void __launch_bounds__(128) k_boundary_aa(typename S::T* f, BoundaryList bl, uint32_t begin, uint32_t end,
                                                     Geom g, StepParams p, int* __restrict__ diverged, AaSide sd) {
    using L = Lattice<Q>;
    using T = typename S::T;
    const uint32_t e = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= end) return;
    const uint32_t c = __ldg(bl.cells + e);
    const unsigned long long lk = __ldg(bl.links + e);
    const unsigned cls = (unsigned)(lk >> kClassShift) & 7u;
    const uint32_t nxy = (uint32_t)g.nxy;
    const int z = (int)(c / nxy);
    const uint32_t rem = c - (uint32_t)z * nxy;
    const int y = (int)(rem / (uint32_t)g.nx);
    const int x = (int)(rem - (uint32_t)y * (uint32_t)g.nx);
    const size_t row = (size_t)z * g.ny + y;
    const int col = outm_col(x, g);

    if (cls == kCellSolidFill) {
        // f_i = w_i (LbmReference.cpp:264-267). In place the solid cell's
        // slots carry its neighbours' bounced populations, so only the
        // outlet's view of it, the moments, is written.
        if (col >= 0) {
            float wv[Q];
            static_for<0, Q>([&](auto I) {
                constexpr int i = decltype(I)::value;
                wv[i] = L::w(i);
            });
            sd.outm[outm_index(sd, Odd ? 0 : 1, col, row)] = stored_moments<Q, S>(wv);
        }
        return;
    }
    const uint32_t co0 = __ldg(bl.coef_off + e);
    uint32_t bzmask = 0;
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if ((((unsigned)(lk >> (3 * i))) & 6u) == 2u) bzmask |= 1u << i;
    });
    T* bz = static_cast<T*>(sd.bz);
    float v[Q];
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        constexpr int op = L::opp(i);
        const unsigned kind = (unsigned)(lk >> (3 * i)) & 7u;
        const size_t off = (size_t)link_offset<Q>(i, g);
        size_t sa;
        if (kind == kLinkStream) {  // f*_i(c - e_i)
            sa = Odd ? (size_t)op * g.n + (c - off) : (size_t)i * g.n + c;
        } else if (kind == kLinkEdge) {  // f*_m(c) for the mirrored / bounced m
            const int py = y - L::ey(i), pz = z - L::ez(i);
            const int m = edge_plane<Q, i>(py < 0 || py >= g.ny, pz < 0 || pz >= g.nz, p);
            sa = (size_t)L::opp(m) * g.n + c;
        } else {  // f*_op(c); before an even step it sits in the solid neighbour c - e_i
            sa = Odd ? (size_t)i * g.n + c : (size_t)op * g.n + (c - off);
        }
        const float va = S::dec(ld_plain<S>(f + sa), L::w(i));
        float r = va;
        if (kind == kLinkBzNear || kind == kLinkBzFar) {
            const uint32_t slot = co0 + __popc(bzmask & ((1u << i) - 1u));
            const float2 kc = __ldg(bl.coef + slot);
            float vb;
            if (kind == kLinkBzNear) {  // f*_op(c + e_i)
                const size_t sb = Odd ? (size_t)i * g.n + (c + off) : (size_t)op * g.n + c;
                vb = S::dec(ld_plain<S>(f + sb), L::w(i));
            } else {  // f*_i(c), kept from the previous step
                vb = S::dec(bz[slot], L::w(i));
            }
            r = kc.x * va + kc.y * vb;
        }
        v[i] = r;
    });
    if (collide<Q, S::kExact>(v, p.tau, p.cs)) atomicOr(diverged, 1);
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const T t = S::enc(v[i], L::w(i));
        f[out_slot<Q, i, Odd>(c, x, y, z, g)] = t;
        if ((((unsigned)(lk >> (3 * i))) & 7u) == kLinkBzFar) bz[co0 + __popc(bzmask & ((1u << i) - 1u))] = t;
    });
    if (col >= 0) sd.outm[outm_index(sd, Odd ? 0 : 1, col, row)] = stored_moments<Q, S>(v);
}

// Stores of a cell pair after the collision (v: scaled offsets or full
// floats, as collide_pair leaves them): the aligned form for full pairs off
// the faces (fast), or the general masked form with the edge and
// outlet-moment rules (the cells feeding the outlet moments, x = 1 and
// nx-2, always sit in partial pairs).
template <int Q, class S, bool Odd>
__device__ __forceinline__ void aa_store_pair(typename S::T* f, const PlanePtrs& pp, const Geom& g, const AaSide& sd,
                                              const float2 (&v)[Q], uint32_t c, int x, int y, int z, size_t row,
                                              unsigned pair, bool fast) {
    using L = Lattice<Q>;
    using T = typename S::T;
    using T2 = typename S::T2;
    if (fast && pair == 3u) {
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            T* dst = static_cast<T*>(pp.dst[i]);
            const T2 h = S::kExact ? S::enc2(v[i].x, v[i].y, L::w(i)) : S::pack2(v[i].x, v[i].y);
            if (!Odd || L::ex(i) == 0) {
                *reinterpret_cast<T2*>(dst + c) = h;
            } else {
                dst[c] = h.x;
                dst[c + 1u] = h.y;
            }
        });
        return;
    }
    const bool va = pair & 1u, vb = pair & 2u;
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const T2 h = S::kExact ? S::enc2(v[i].x, v[i].y, L::w(i)) : S::pack2(v[i].x, v[i].y);
        // pair cells never sit on x = 0 or x = nx-1, so only y / z can leave
        const int ty = y + L::ey(i), tz = z + L::ez(i);
        const bool inside = ty >= 0 && ty < g.ny && tz >= 0 && tz < g.nz;
        const bool push = Odd && inside;
        T* dst = f + (push ? (size_t)i * g.n + (size_t)((long long)c + link_offset<Q>(i, g))
                           : (size_t)L::opp(i) * g.n + c);
        if (pair == 3u && (!push || L::ex(i) == 0)) {
            *reinterpret_cast<T2*>(dst) = h;
        } else {
            if (va) dst[0] = h.x;
            if (vb) dst[1] = h.y;
        }
    });
    const int ca = va ? outm_col(x, g) : -1, cb = vb ? outm_col(x + 1, g) : -1;
    if (ca >= 0 || cb >= 0) {
        float a[Q], b[Q];
        pair_stored<Q, S>(v, a, b);
        if (ca >= 0) sd.outm[outm_index(sd, Odd ? 0 : 1, ca, row)] = plain_moments<Q>(a);
        if (cb >= 0) sd.outm[outm_index(sd, Odd ? 0 : 1, cb, row)] = plain_moments<Q>(b);
    }
}

// k_bulk_pairs_aa with the learned closure (16-bit offset formats): the slots
// of k_bulk_pairs_aa around the two-phase collision and warp-wide MLP of
// k_bulk_pairs_learned, so every stored value is the one the ping-pong
// learned step stores. The MLP is a warp-wide tensor-core operation, so no
// lane leaves before it: lanes without a bulk pair read in-lattice slots and
// store nothing, and partial pairs take the pair collision with masked
// stores, as in the ping-pong learned kernel.
template <int Q, class S, bool Odd>
__global__ void __launch_bounds__(32 * kBulkRows, 4) k_bulk_pairs_aa_learned(typename S::T* f,
                                                                           const uint32_t* __restrict__ bulk_bits,
                                                                           Geom g, StepParams p, PlanePtrs pp, int z0,
                                                                           int* __restrict__ diverged, AaSide sd,
                                                                           ClosureDev cl) {
    static_assert(!S::kExact, "the learned closure runs on the 16-bit offset formats");
    using L = Lattice<Q>;
    using T = typename S::T;
    using T2 = typename S::T2;
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
    const uint32_t cs = x < g.nx ? c : (uint32_t)(row * g.nx);  // lanes past the row end read its first pair
    const bool face = (y == 0) | (y == g.ny - 1) | (z == 0) | (z == g.nz - 1);
    // off the faces every source slot lies inside the set (k_bulk_pairs_aa)
    const bool fast = !face;
    aa_row_end_cells<Q, S, Odd>(f, g, p, sd, plane, x, y, z, c, row);

    float2 v[Q];
    if (fast) {
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const T* src = static_cast<const T*>(pp.src[i]);
            if (!Odd || L::ex(i) == 0)
                v[i] = S::raw2(ld2_plain<S>(src + cs));
            else
                v[i] = make_float2(S::raw(ld_plain<S>(src + cs)), S::raw(ld_plain<S>(src + cs + 1u)));
        });
    } else {
        const bool va = pair & 1u, vb = pair & 2u;
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const int py = y - L::ey(i), pz = z - L::ez(i);
            const bool oy = py < 0 || py >= g.ny;
            const bool oz = pz < 0 || pz >= g.nz;
            const bool out = oy || oz;
            const int m = out ? edge_plane<Q, i>(oy, oz, p) : i;
            const int rplane = out ? L::opp(m) : (Odd ? L::opp(i) : i);
            const uint32_t off = (out || !Odd) ? 0u : (uint32_t)link_offset<Q>(i, g);
            const uint32_t sa = va ? c - off : cs;
            const uint32_t sb = vb ? c + 1u - off : cs + 1u;
            const T* base = f + (size_t)rplane * g.n;
            v[i] = make_float2(S::raw(ld_plain<S>(base + sa)), S::raw(ld_plain<S>(base + sb)));
        });
    }
    Mom2 mo;
    const unsigned bad = moments2<Q>(v, mo) & pair;
    // the range test, the Smagorinsky fallback and the MLP as in
    // k_bulk_pairs_learned (warp votes keep every branch uniform)
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
    float sga = 0.0f, sgb = 0.0f, dsa = 0.0f, dsb = 0.0f;
    if (closure_anchored(cl) || __any_sync(0xffffffffu, !(la && lb))) {
        sga = smagorinsky_g(mo.pp.x, mo.rho.x, mo.inv.x, p.tau, p.cs);
        sgb = smagorinsky_g(mo.pp.y, mo.rho.y, mo.inv.y, p.tau, p.cs);
        if (closure_anchored(cl)) {
            dsa = smagorinsky_d3(mo.pp.x, mo.rho.x, mo.inv.x, p.tau, p.cs);
            dsb = smagorinsky_d3(mo.pp.y, mo.rho.y, mo.inv.y, p.tau, p.cs);
        }
    }
    const unsigned need = __ballot_sync(0xffffffffu, la || lb);
    if (!need) {
        if (!pair) return;
        relax2<Q>(v, mo, make_float2(sga, sgb));
        if (bad) atomicOr(diverged, 1);
        aa_store_pair<Q, S, Odd>(f, pp, g, sd, v, c, x, y, z, row, pair, fast);
        return;
    }
    float2* sm = &s_mo[threadIdx.y][0][threadIdx.x];
    sm[0 * 32] = mo.rho, sm[1 * 32] = mo.drho, sm[2 * 32] = mo.u2, sm[3 * 32] = mo.ux;
    sm[4 * 32] = mo.uy, sm[5 * 32] = mo.uz, sm[6 * 32] = mo.pxx, sm[7 * 32] = mo.pyy;
    sm[8 * 32] = mo.pzz, sm[9 * 32] = mo.pxy, sm[10 * 32] = mo.pxz, sm[11 * 32] = mo.pyz;
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
    aa_store_pair<Q, S, Odd>(f, pp, g, sd, v, c, x, y, z, row, pair, fast);
}

// k_boundary_aa with the learned closure: the slots of k_boundary_aa around
// the collision of k_boundary_pull_learned (link values in floats, then the
// two-phase collision on offsets with the warp-wide closure). Every lane of
// a warp runs the closure; only live fluid entries store.
template <int Q, class S, bool Odd>
__global__ void __launch_bounds__(128) k_boundary_aa_learned(typename S::T* f, BoundaryList bl, uint32_t begin,
                                                             uint32_t end, Geom g, StepParams p,
                                                             int* __restrict__ diverged, AaSide sd, ClosureDev cl) {
    static_assert(!S::kExact, "the learned closure runs on the 16-bit offset formats");
    using L = Lattice<Q>;
    using T = typename S::T;
    __shared__ uint32_t s_in[4][32 * 8];
    __shared__ float2 s_out[4][32];
    const uint32_t e = begin + blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = e < end;
    const uint32_t c = live ? __ldg(bl.cells + e) : 0u;
    const unsigned long long lk = live ? __ldg(bl.links + e) : 0ull;
    const unsigned cls = (unsigned)(lk >> kClassShift) & 7u;
    const bool fluid = live && cls != kCellSolidFill;
    const uint32_t nxy = (uint32_t)g.nxy;
    const int z = (int)(c / nxy);
    const uint32_t rem = c - (uint32_t)z * nxy;
    const int y = (int)(rem / (uint32_t)g.nx);
    const int x = (int)(rem - (uint32_t)y * (uint32_t)g.nx);
    const size_t row = (size_t)z * g.ny + y;
    const int col = live ? outm_col(x, g) : -1;
    if (live && !fluid && col >= 0) {  // a solid cell: only the outlet's view of it (k_boundary_aa)
        float wv[Q];
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            wv[i] = L::w(i);
        });
        sd.outm[outm_index(sd, Odd ? 0 : 1, col, row)] = stored_moments<Q, S>(wv);
    }
    T* bz = static_cast<T*>(sd.bz);
    const uint32_t co0 = fluid ? __ldg(bl.coef_off + e) : 0u;
    uint32_t bzmask = 0;
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if ((((unsigned)(lk >> (3 * i))) & 6u) == 2u) bzmask |= 1u << i;
    });
    float2 h[Q];
    if (fluid) {
        static_for<0, Q>([&](auto I) {
            constexpr int i = decltype(I)::value;
            constexpr int op = L::opp(i);
            const unsigned kind = (unsigned)(lk >> (3 * i)) & 7u;
            const size_t off = (size_t)link_offset<Q>(i, g);
            size_t sa;
            if (kind == kLinkStream) {  // f*_i(c - e_i)
                sa = Odd ? (size_t)op * g.n + (c - off) : (size_t)i * g.n + c;
            } else if (kind == kLinkEdge) {  // f*_m(c) for the mirrored / bounced m
                const int py = y - L::ey(i), pz = z - L::ez(i);
                const int m = edge_plane<Q, i>(py < 0 || py >= g.ny, pz < 0 || pz >= g.nz, p);
                sa = (size_t)L::opp(m) * g.n + c;
            } else {  // f*_op(c); before an even step it sits in the solid neighbour c - e_i
                sa = Odd ? (size_t)i * g.n + c : (size_t)op * g.n + (c - off);
            }
            const float va = S::dec(ld_plain<S>(f + sa), L::w(i));
            float r = va;
            if (kind == kLinkBzNear || kind == kLinkBzFar) {
                const uint32_t slot = co0 + __popc(bzmask & ((1u << i) - 1u));
                const float2 kc = __ldg(bl.coef + slot);
                float vb;
                if (kind == kLinkBzNear) {  // f*_op(c + e_i)
                    const size_t sb = Odd ? (size_t)i * g.n + (c + off) : (size_t)op * g.n + c;
                    vb = S::dec(ld_plain<S>(f + sb), L::w(i));
                } else {  // f*_i(c), kept from the previous step
                    vb = S::dec(bz[slot], L::w(i));
                }
                r = kc.x * va + kc.y * vb;
            }
            h[i] = make_float2((r - L::w(i)) * 256.0f, 0.0f);
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
    float vf[Q];
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        vf[i] = L::w(i) + h[i].x * (1.0f / 256.0f);
        const T t = S::enc(vf[i], L::w(i));
        f[out_slot<Q, i, Odd>(c, x, y, z, g)] = t;
        if ((((unsigned)(lk >> (3 * i))) & 7u) == kLinkBzFar) bz[co0 + __popc(bzmask & ((1u << i) - 1u))] = t;
    });
    if (col >= 0) sd.outm[outm_index(sd, Odd ? 0 : 1, col, row)] = stored_moments<Q, S>(vf);
}

// Side buffers from the current state (`layout`, read by a step of parity
// par): the Bouzidi far-side values of every boundary entry ...
template <int Q, class S>
__global__ void __launch_bounds__(128) k_aa_prime_links(const typename S::T* f, BoundaryList bl, uint32_t count,
                                                        Geom g, AaSide sd, int layout) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const unsigned long long lk = __ldg(bl.links + e);
    if ((((unsigned)(lk >> kClassShift)) & 7u) == kCellSolidFill) return;
    const uint32_t c = __ldg(bl.cells + e);
    const uint32_t nxy = (uint32_t)g.nxy;
    const int z = (int)(c / nxy);
    const uint32_t rem = c - (uint32_t)z * nxy;
    const int y = (int)(rem / (uint32_t)g.nx);
    const int x = (int)(rem - (uint32_t)y * (uint32_t)g.nx);
    const uint32_t co0 = __ldg(bl.coef_off + e);
    uint32_t bzmask = 0;
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if ((((unsigned)(lk >> (3 * i))) & 6u) == 2u) bzmask |= 1u << i;
    });
    typename S::T* bz = static_cast<typename S::T*>(sd.bz);
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if ((((unsigned)(lk >> (3 * i))) & 7u) == kLinkBzFar)
            bz[co0 + __popc(bzmask & ((1u << i) - 1u))] = f[pop_slot<Q, i>(c, x, y, z, g, layout)];
    });
}

// ... and the moments of the cells at x = 1 and x = nx-2 of every row.
template <int Q, class S>
__global__ void __launch_bounds__(128) k_aa_prime_rows(const typename S::T* f, Geom g, AaSide sd, int layout,
                                                       int par) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * sd.rows) return;
    const int col = (int)(t / sd.rows);
    const size_t row = t - (size_t)col * sd.rows;
    const int z = (int)(row / (size_t)g.ny), y = (int)(row - (size_t)z * g.ny);
    const int x = col == 0 ? 1 : g.nx - 2;
    const size_t c = row * g.nx + x;
    float d[Q];
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        d[i] = S::dec(f[pop_slot<Q, i>(c, x, y, z, g, layout)], Lattice<Q>::w(i));
    });
    sd.outm[outm_index(sd, par, col, row)] = plain_moments<Q>(d);
}

template <int Q, class S>
static cudaError_t bulk_aa_t(void* f, const uint32_t* bits, const Geom& g, const StepParams& p, int z0, int zc,
                             int* dv, cudaStream_t s, int* launched, int odd, const AaSide& sd) {
    *launched = 0;
    if (zc <= 0) return cudaSuccess;
    if (g.nx % 2 != 0 || g.nx < 4) return cudaErrorNotSupported;
    using T = typename S::T;
    T* base = static_cast<T*>(f);
    PlanePtrs pp{};
    for (int i = 0; i < Q; ++i) {
        const long long off = (long long)Lattice<Q>::ex(i) + (long long)Lattice<Q>::ey(i) * g.nx +
                              (long long)Lattice<Q>::ez(i) * g.nxy;
        const long long pi = (long long)i * (long long)g.n, po = (long long)Lattice<Q>::opp(i) * (long long)g.n;
        pp.src[i] = base + (odd ? po - off : pi);
        pp.dst[i] = base + (odd ? pi + off : po);
    }
    dim3 block(32, kBulkRows, 1);
    dim3 grid((unsigned)((g.nx + 63) / 64), (unsigned)((g.ny + kBulkRows - 1) / kBulkRows), (unsigned)zc);
    if (odd)
        k_bulk_pairs_aa<Q, S, true><<<grid, block, 0, s>>>(base, bits, g, p, pp, z0, dv, sd);
    else
        k_bulk_pairs_aa<Q, S, false><<<grid, block, 0, s>>>(base, bits, g, p, pp, z0, dv, sd);
    ++*launched;
    return cudaGetLastError();
}

template <int Q, class S>
static cudaError_t boundary_aa_t(void* f, const BoundaryList& bl, uint32_t b, uint32_t e, const Geom& g,
                                 const StepParams& p, int* dv, cudaStream_t s, int odd, const AaSide& sd) {
    if (e <= b) return cudaSuccess;
    const unsigned threads = 128;
    const unsigned blocks = (e - b + threads - 1) / threads;
    if (odd)
        k_boundary_aa<Q, S, true><<<blocks, threads, 0, s>>>((typename S::T*)f, bl, b, e, g, p, dv, sd);
    else
        k_boundary_aa<Q, S, false><<<blocks, threads, 0, s>>>((typename S::T*)f, bl, b, e, g, p, dv, sd);
    return cudaGetLastError();
}

template <int Q, class S>
static cudaError_t bulk_aa_learned_t(void* f, const uint32_t* bits, const Geom& g, const StepParams& p, int z0, int zc,
                                     int* dv, cudaStream_t s, int* launched, int odd, const AaSide& sd,
                                     const ClosureDev& cl) {
    *launched = 0;
    if constexpr (S::kExact) {
        return cudaErrorNotSupported;
    } else {
        if (zc <= 0) return cudaSuccess;
        if (g.nx % 2 != 0 || g.nx < 4) return cudaErrorNotSupported;
        using T = typename S::T;
        T* base = static_cast<T*>(f);
        PlanePtrs pp{};
        for (int i = 0; i < Q; ++i) {
            const long long off = (long long)Lattice<Q>::ex(i) + (long long)Lattice<Q>::ey(i) * g.nx +
                                  (long long)Lattice<Q>::ez(i) * g.nxy;
            const long long pi = (long long)i * (long long)g.n, po = (long long)Lattice<Q>::opp(i) * (long long)g.n;
            pp.src[i] = base + (odd ? po - off : pi);
            pp.dst[i] = base + (odd ? pi + off : po);
        }
        dim3 block(32, kBulkRows, 1);
        dim3 grid((unsigned)((g.nx + 63) / 64), (unsigned)((g.ny + kBulkRows - 1) / kBulkRows), (unsigned)zc);
        if (odd)
            k_bulk_pairs_aa_learned<Q, S, true><<<grid, block, 0, s>>>(base, bits, g, p, pp, z0, dv, sd, cl);
        else
            k_bulk_pairs_aa_learned<Q, S, false><<<grid, block, 0, s>>>(base, bits, g, p, pp, z0, dv, sd, cl);
        ++*launched;
        return cudaGetLastError();
    }
}

template <int Q, class S>
static cudaError_t boundary_aa_learned_t(void* f, const BoundaryList& bl, uint32_t b, uint32_t e, const Geom& g,
                                         const StepParams& p, int* dv, cudaStream_t s, int odd, const AaSide& sd,
                                         const ClosureDev& cl) {
    if constexpr (S::kExact) {
        return cudaErrorNotSupported;
    } else {
        if (e <= b) return cudaSuccess;
        const unsigned threads = 128;
        const unsigned blocks = (e - b + threads - 1) / threads;
        if (odd)
            k_boundary_aa_learned<Q, S, true><<<blocks, threads, 0, s>>>((typename S::T*)f, bl, b, e, g, p, dv, sd, cl);
        else
            k_boundary_aa_learned<Q, S, false><<<blocks, threads, 0, s>>>((typename S::T*)f, bl, b, e, g, p, dv, sd,
                                                                          cl);
        return cudaGetLastError();
    }
}

template <int Q, class S>
static cudaError_t aa_prime_t(const void* f, const BoundaryList& bl, uint32_t count, const Geom& g, const AaSide& sd,
                              int par, cudaStream_t s) {
    const int layout = aa_layout(par);
    if (count > 0) {
        k_aa_prime_links<Q, S><<<(count + 127) / 128, 128, 0, s>>>((const typename S::T*)f, bl, count, g, sd, layout);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    k_aa_prime_rows<Q, S><<<(unsigned)((2 * sd.rows + 127) / 128), 128, 0, s>>>((const typename S::T*)f, g, sd, layout,
                                                                               par);
    return cudaGetLastError();
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

cudaError_t launch_bulk_aa(int q, int storage, void* f, const uint32_t* bulk_bits, const Geom& g, const StepParams& p,
                           int z0, int zc, int* diverged, cudaStream_t s, int* launched, int odd, const AaSide& sd) {
    FC_DISPATCH(q, storage, bulk_aa_t, f, bulk_bits, g, p, z0, zc, diverged, s, launched, odd, sd);
}

cudaError_t launch_boundary_aa(int q, int storage, void* f, const BoundaryList& bl, uint32_t begin, uint32_t end,
                               const Geom& g, const StepParams& p, int* diverged, cudaStream_t s, int odd,
                               const AaSide& sd) {
    FC_DISPATCH(q, storage, boundary_aa_t, f, bl, begin, end, g, p, diverged, s, odd, sd);
}

cudaError_t launch_bulk_aa_learned(int q, int storage, void* f, const uint32_t* bulk_bits, const Geom& g,
                                   const StepParams& p, int z0, int zc, int* diverged, cudaStream_t s, int* launched,
                                   int odd, const AaSide& sd, const ClosureDev& cl) {
    FC_DISPATCH(q, storage, bulk_aa_learned_t, f, bulk_bits, g, p, z0, zc, diverged, s, launched, odd, sd, cl);
}

cudaError_t launch_boundary_aa_learned(int q, int storage, void* f, const BoundaryList& bl, uint32_t begin,
                                       uint32_t end, const Geom& g, const StepParams& p, int* diverged,
                                       cudaStream_t s, int odd, const AaSide& sd, const ClosureDev& cl) {
    FC_DISPATCH(q, storage, boundary_aa_learned_t, f, bl, begin, end, g, p, diverged, s, odd, sd, cl);
}

cudaError_t launch_aa_prime(int q, int storage, const void* f, const BoundaryList& bl, uint32_t count, const Geom& g,
                            const AaSide& sd, int par, cudaStream_t s) {
    FC_DISPATCH(q, storage, aa_prime_t, f, bl, count, g, sd, par, s);
}

}  // namespace fc
