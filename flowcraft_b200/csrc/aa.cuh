// Where a population lives between steps: the plane-major layout of a
// ping-pong set, or the two layouts of a single set streamed in place with
// the AA pattern.
//
// Pull streaming reads f*_i(c - e_i), the post-collision population i of the
// upstream cell. With one set updated in place, the AA pattern alternates two
// kinds of step:
//   even  reads cell c's own slots and writes its own slots: f*_i(c) goes
//         to plane opp(i) of cell c;
//   odd   reads f*_i(c - e_i) from plane opp(i) of c - e_i and writes f*_i(c)
//         to plane i of c + e_i, the cell that pulls it next.
// So between steps, post-collision population p of cell c = (x, y, z) sits:
//   before an even step (kLayoutAAEven): in plane p of c + e_p, or, when
//       c + e_p is off the lattice, in plane opp(p) of c itself;
//   before an odd step (kLayoutAAOdd): in plane opp(p) of c.
// Both maps are one-to-one onto the Q*n slots. In either step every thread
// writes exactly the slots its own pulls read: the stream sources, the
// bounce-back and free-slip sources (a population that would leave the
// lattice stays in the cell's own opposite slot), and the Bouzidi near-side
// partner. The two reads that fall in another thread's slots, the Bouzidi
// far-side partner f*_i(c) and the outlet's neighbour moments, are carried
// from the step before in small side buffers (lbm_step.cu).
#pragma once

#include <cstddef>

#include "lattice.cuh"
#include "lbm_internal.h"

namespace fc {

enum PopLayout : int { kLayoutPlanes = 0, kLayoutAAEven = 1, kLayoutAAOdd = 2 };

// Layout of a set that a step of parity `odd` reads.
__host__ __device__ constexpr int aa_layout(int odd) { return odd ? kLayoutAAOdd : kLayoutAAEven; }

template <int Q>
__device__ __forceinline__ long long aa_link(int p, const Geom& g) {
    using L = Lattice<Q>;
    return (long long)L::ex(p) + (long long)L::ey(p) * g.nx + (long long)L::ez(p) * g.nxy;
}

// Slot index (plane * n + cell) of post-collision population P of cell c.
template <int Q, int P>
__device__ __forceinline__ size_t pop_slot(size_t c, int x, int y, int z, const Geom& g, int layout) {
    using L = Lattice<Q>;
    if (layout == kLayoutPlanes) return (size_t)P * g.n + c;
    if (layout == kLayoutAAEven) {
        const int tx = x + L::ex(P), ty = y + L::ey(P), tz = z + L::ez(P);
        if (tx >= 0 && ty >= 0 && tz >= 0 && tx < g.nx && ty < g.ny && tz < g.nz)
            return (size_t)P * g.n + (size_t)((long long)c + aa_link<Q>(P, g));
    }
    return (size_t)L::opp(P) * g.n + c;
}

// The same with a run-time direction.
template <int Q>
__device__ __forceinline__ size_t pop_slot_rt(int p, size_t c, int x, int y, int z, const Geom& g, int layout) {
    size_t r = 0;
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if (i == p) r = pop_slot<Q, i>(c, x, y, z, g, layout);
    });
    return r;
}

}  // namespace fc
