// Readback kernels: macroscopic field, raw populations, and the FP64
// statistics reduction.
//
// The field follows LbmReference::ReadbackField (LbmReference.cpp:475-500):
// fluid cells get (rho, ux, uy, uz) from the current post-collision state;
// solid cells get the momentum-exchange force of their fluid neighbours,
// (|F| / (6 sum w), Fx, Fy, Fz) (LbmReference::SolidCellForce,
// LbmReference.cpp:127-148), with the same Bouzidi reconstruction the step
// uses. Only the moments are computed — the step never writes a
// 16-byte-per-cell macro buffer the way the reference's GPU kernel does
// (shaders/lbm_step.comp.glsl:360-363), which saves 16 B of HBM traffic per
// cell update.
#include <mutex>

#include "aa.cuh"
#include "collide.cuh"
#include "fc_lbm.h"
#include "lbm_internal.h"
#include "storage.cuh"

namespace fc {

__device__ __forceinline__ bool inb(const Geom& g, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && x < g.nx && y < g.ny && z < g.nz;
}
__device__ __forceinline__ size_t cidx(const Geom& g, int x, int y, int z) { return ((size_t)z * g.ny + y) * g.nx + x; }

// Post-collision population P of cell c = (x, y, z) under `layout` (aa.cuh).
template <int Q, class S, int P>
__device__ __forceinline__ float load_at(const typename S::T* __restrict__ f, size_t c, int x, int y, int z,
                                         const Geom& g, int layout) {
    return S::dec(S::ld(f + pop_slot<Q, P>(c, x, y, z, g, layout)), Lattice<Q>::w(P));
}

// InterpolatedBounceBack for fluid node a (cell ca) whose direction-i
// upstream neighbour s (cell cs) is solid (LbmReference.cpp:100-122).
template <int Q, class S, int I>
__device__ float bounce_rt(const typename S::T* __restrict__ f, const uint8_t* __restrict__ solid,
                           const float* __restrict__ sdf, const Geom& g, int ax, int ay, int az, size_t ca,
                           size_t cs, int layout) {
    using L = Lattice<Q>;
    constexpr int op = L::opp(I);
    const float plain = load_at<Q, S, op>(f, ca, ax, ay, az, g, layout);
    if (!sdf) return plain;
    const float phi_f = sdf[ca], phi_s = sdf[cs];
    if (!isfinite(phi_f) || !isfinite(phi_s)) return plain;
    const float denom = phi_f - phi_s;
    if (!(denom > 1e-4f)) return plain;
    float q = phi_f / denom;
    q = (q < 0.0f) ? 0.0f : ((1.0f < q) ? 1.0f : q);
    if (q < 0.5f) {
        const int fx = ax + L::ex(I), fy = ay + L::ey(I), fz = az + L::ez(I);
        if (!inb(g, fx, fy, fz) || solid[cidx(g, fx, fy, fz)]) return plain;
        return 2.0f * q * plain + (1.0f - 2.0f * q) * load_at<Q, S, op>(f, cidx(g, fx, fy, fz), fx, fy, fz, g, layout);
    }
    const float inv = 1.0f / (2.0f * q);
    return inv * plain + (1.0f - inv) * load_at<Q, S, I>(f, ca, ax, ay, az, g, layout);
}

template <int Q, class S>
__device__ float4 solid_force(const typename S::T* __restrict__ f, const uint8_t* __restrict__ solid,
                              const float* __restrict__ sdf, const Geom& g, int x, int y, int z, size_t c,
                              int layout) {
    using L = Lattice<Q>;
    float fx = 0.0f, fy = 0.0f, fz = 0.0f, ws = 0.0f;
    static_for<1, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        constexpr int X = L::ex(i), Y = L::ey(i), Z = L::ez(i);
        const int ax = x + X, ay = y + Y, az = z + Z;
        if (!inb(g, ax, ay, az)) return;
        const size_t ca = cidx(g, ax, ay, az);
        if (solid[ca]) return;
        const float plain = load_at<Q, S, L::opp(i)>(f, ca, ax, ay, az, g, layout);
        const float bounced = bounce_rt<Q, S, i>(f, solid, sdf, g, ax, ay, az, ca, c, layout);
        const float dp = (plain + bounced) - 2.0f * L::w(i);
        if constexpr (X > 0) fx = fx - dp;
        if constexpr (X < 0) fx = fx + dp;
        if constexpr (Y > 0) fy = fy - dp;
        if constexpr (Y < 0) fy = fy + dp;
        if constexpr (Z > 0) fz = fz - dp;
        if constexpr (Z < 0) fz = fz + dp;
        ws = ws + L::w(i);
    });
    const float mag = sqrtf((fx * fx + fy * fy) + fz * fz);
    const float stress = (ws > 0.0f) ? (mag / (6.0f * ws)) : 0.0f;
    return make_float4(stress, fx, fy, fz);
}

template <int Q, class S>
__device__ __forceinline__ float4 fluid_moments(const typename S::T* __restrict__ f, const Geom& g, size_t c, int x,
                                                int y, int z, int layout) {
    float p[Q];
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        p[i] = load_at<Q, S, i>(f, c, x, y, z, g, layout);
    });
    float rho, ux, uy, uz;
    moments<Q>(p, rho, ux, uy, uz);
    return make_float4(rho, ux, uy, uz);
}

template <int Q, class S, int Lay>
__global__ void __launch_bounds__(256) k_field(const typename S::T* __restrict__ f, const uint8_t* __restrict__ solid,
                                                const float* __restrict__ sdf, Geom g, size_t cell0, size_t cells,
                                                float4* __restrict__ out, int layout_in) {
    // the layout is a compile-time constant, so every slot folds to its
    // formula (plane * n + c for plane-major states)
    const int layout = Lay;
    (void)layout_in;
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cells) return;
    const size_t c = cell0 + k;
    const int z = (int)(c / (size_t)g.nxy);
    const size_t rem = c - (size_t)z * g.nxy;
    const int y = (int)(rem / g.nx);
    const int x = (int)(rem - (size_t)y * g.nx);
    out[k] = solid[c] ? solid_force<Q, S>(f, solid, sdf, g, x, y, z, c, layout)
                      : fluid_moments<Q, S>(f, g, c, x, y, z, layout);
}

// ProbeSliceHealth's verdict on the device (LbmSolver.cpp:699-716): the
// field values k_field gives for cells [cell0, cell0 + cells), then every
// value finite, and for fluid cells rho > 0 and |u|^2 <= 4 (the same float
// operations as the host check). Any failing cell sets *flag.
template <int Q, class S, int Lay>
__global__ void __launch_bounds__(256) k_probe_health(const typename S::T* __restrict__ f,
                                                       const uint8_t* __restrict__ solid, const float* __restrict__ sdf,
                                                       Geom g, size_t cell0, size_t cells, int* __restrict__ flag,
                                                       int layout_in) {
    const int layout = Lay;
    (void)layout_in;
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = false;
    if (k < cells) {
        const size_t c = cell0 + k;
        const int z = (int)(c / (size_t)g.nxy);
        const size_t rem = c - (size_t)z * g.nxy;
        const int y = (int)(rem / g.nx);
        const int x = (int)(rem - (size_t)y * g.nx);
        const bool sc = solid[c] != 0;
        const float4 v = sc ? solid_force<Q, S>(f, solid, sdf, g, x, y, z, c, layout)
                            : fluid_moments<Q, S>(f, g, c, x, y, z, layout);
        bad = !isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z) || !isfinite(v.w);
        if (!bad && !sc) {
            const float sp2 = v.y * v.y + v.z * v.z + v.w * v.w;
            bad = v.x <= 0.0f || sp2 > 4.0f;
        }
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

template <int Q, class S, int Lay>
__global__ void k_pops_out(const typename S::T* __restrict__ f, const uint8_t* __restrict__ solid,
                           int solid_is_weight, Geom g, size_t cell0, size_t cells, float* __restrict__ out,
                           int layout_in) {
    // the layout is a compile-time constant, so every slot folds to its
    // formula (plane * n + c for plane-major states)
    const int layout = Lay;
    (void)layout_in;
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cells) return;
    const size_t c = cell0 + k;
    int x = 0, y = 0, z = 0;
    if (layout != kLayoutPlanes) {  // the plane-major slot needs no coordinates
        z = (int)(c / (size_t)g.nxy);
        const size_t rem = c - (size_t)z * g.nxy;
        y = (int)(rem / g.nx);
        x = (int)(rem - (size_t)y * g.nx);
    }
    const bool sw = solid_is_weight && solid[c];
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        out[(size_t)i * cells + k] = sw ? Lattice<Q>::w(i) : load_at<Q, S, i>(f, c, x, y, z, g, layout);
    });
}

template <int Q, class S, int Lay>
__global__ void k_pops_in(typename S::T* __restrict__ f, Geom g, size_t cell0, size_t cells,
                          const float* __restrict__ in, int layout_in) {
    // the layout is a compile-time constant, so every slot folds to its
    // formula (plane * n + c for plane-major states)
    const int layout = Lay;
    (void)layout_in;
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cells) return;
    const size_t c = cell0 + k;
    int x = 0, y = 0, z = 0;
    if (layout != kLayoutPlanes) {
        z = (int)(c / (size_t)g.nxy);
        const size_t rem = c - (size_t)z * g.nxy;
        y = (int)(rem / g.nx);
        x = (int)(rem - (size_t)y * g.nx);
    }
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        f[pop_slot<Q, i>(c, x, y, z, g, layout)] = S::enc(in[(size_t)i * cells + k], Lattice<Q>::w(i));
    });
}

// ---- statistics (LbmReference::ComputeStats, LbmReference.cpp:502-585) ----
// Slots: 0 density sum, 1 speed sum, 2 mass, 3..5 force sums, 6 fluid count,
// 7 min density, 8 max density, 9 max speed, 10 max stress, 11 NaN flag.
constexpr int kStatsThreads = 256;

struct StatAcc {
    double dsum = 0.0, ssum = 0.0, fx = 0.0, fy = 0.0, fz = 0.0, count = 0.0;
    float mn = 1e30f, mx = -1e30f, vmax = 0.0f, smax = 0.0f;
    int nan = 0;
};

__device__ __forceinline__ void stat_merge(StatAcc& a, const StatAcc& b) {
    a.dsum += b.dsum;
    a.ssum += b.ssum;
    a.fx += b.fx;
    a.fy += b.fy;
    a.fz += b.fz;
    a.count += b.count;
    a.mn = fminf(a.mn, b.mn);
    a.mx = fmaxf(a.mx, b.mx);
    a.vmax = fmaxf(a.vmax, b.vmax);
    a.smax = fmaxf(a.smax, b.smax);
    a.nan |= b.nan;
}

__device__ __forceinline__ void stat_block_reduce(StatAcc& acc, double* out) {
    __shared__ StatAcc sh[kStatsThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        StatAcc b;
        b.dsum = __shfl_down_sync(0xffffffffu, acc.dsum, o);
        b.ssum = __shfl_down_sync(0xffffffffu, acc.ssum, o);
        b.fx = __shfl_down_sync(0xffffffffu, acc.fx, o);
        b.fy = __shfl_down_sync(0xffffffffu, acc.fy, o);
        b.fz = __shfl_down_sync(0xffffffffu, acc.fz, o);
        b.count = __shfl_down_sync(0xffffffffu, acc.count, o);
        b.mn = __shfl_down_sync(0xffffffffu, acc.mn, o);
        b.mx = __shfl_down_sync(0xffffffffu, acc.mx, o);
        b.vmax = __shfl_down_sync(0xffffffffu, acc.vmax, o);
        b.smax = __shfl_down_sync(0xffffffffu, acc.smax, o);
        b.nan = __shfl_down_sync(0xffffffffu, acc.nan, o);
        stat_merge(acc, b);
    }
    if (lane == 0) sh[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        StatAcc t = sh[0];
        for (int w = 1; w < kStatsThreads / 32; ++w) stat_merge(t, sh[w]);
        out[0] = t.dsum;
        out[1] = t.ssum;
        out[2] = t.dsum;  // mass: the reference sums rho over fluid cells
        out[3] = t.fx;
        out[4] = t.fy;
        out[5] = t.fz;
        out[6] = t.count;
        out[7] = t.mn;
        out[8] = t.mx;
        out[9] = t.vmax;
        out[10] = t.smax;
        out[11] = t.nan;
    }
}

template <int Q, class S, int Lay>
__global__ void __launch_bounds__(kStatsThreads) k_stats(const typename S::T* __restrict__ f,
                                                         const uint8_t* __restrict__ solid,
                                                         const float* __restrict__ sdf, Geom g,
                                                         double* __restrict__ partials, int layout_in) {
    // the layout is a compile-time constant, so every slot folds to its
    // formula (plane * n + c for plane-major states)
    const int layout = Lay;
    (void)layout_in;
    StatAcc acc;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < g.n; c += (size_t)gridDim.x * blockDim.x) {
        const bool sol = solid[c];
        // cell coordinates only where they are used: the solid-cell force and
        // the in-place layouts (the plane-major slot is plane * n + c)
        int x = 0, y = 0, z = 0;
        if (sol || layout != kLayoutPlanes) {
            z = (int)(c / (size_t)g.nxy);
            const size_t rem = c - (size_t)z * g.nxy;
            y = (int)(rem / g.nx);
            x = (int)(rem - (size_t)y * g.nx);
        }
        if (sol) {
            const float4 v = solid_force<Q, S>(f, solid, sdf, g, x, y, z, c, layout);
            if (isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w)) {
                acc.fx += (double)v.y;
                acc.fy += (double)v.z;
                acc.fz += (double)v.w;
                acc.smax = fmaxf(acc.smax, v.x);
            }
            continue;
        }
        const float4 m = fluid_moments<Q, S>(f, g, c, x, y, z, layout);
        if (!isfinite(m.x) || !isfinite(m.y) || !isfinite(m.z) || !isfinite(m.w)) {
            acc.nan = 1;
            continue;
        }
        const float sp = sqrtf(speed2(m.y, m.z, m.w));
        acc.mn = fminf(acc.mn, m.x);
        acc.mx = fmaxf(acc.mx, m.x);
        acc.vmax = fmaxf(acc.vmax, sp);
        acc.dsum += (double)m.x;
        acc.ssum += (double)sp;
        acc.count += 1.0;
    }
    stat_block_reduce(acc, partials + (size_t)blockIdx.x * kStatsSlots);
}

__global__ void __launch_bounds__(kStatsThreads) k_stats_final(const double* __restrict__ partials, int blocks,
                                                               double* __restrict__ result) {
    StatAcc acc;
    for (int b = threadIdx.x; b < blocks; b += blockDim.x) {
        const double* p = partials + (size_t)b * kStatsSlots;
        StatAcc t;
        t.dsum = p[0];
        t.ssum = p[1];
        t.fx = p[3];
        t.fy = p[4];
        t.fz = p[5];
        t.count = p[6];
        t.mn = (float)p[7];
        t.mx = (float)p[8];
        t.vmax = (float)p[9];
        t.smax = (float)p[10];
        t.nan = p[11] != 0.0;
        stat_merge(acc, t);
    }
    stat_block_reduce(acc, result);
}

// ---- aerodynamic forces (FieldOverlay::ComputeAerodynamicForces, FieldOverlay.cpp:469-621) ----
// Slots: 0-2 force sums, 3 lift weight sum, 4-6 lift-weighted position sums,
// 7 force weight sum, 8-10 force-weighted sums, 11-13 geometric position sums,
// 14 solid count, 15 max solid z, 16 min loaded stress, 17 max loaded stress,
// 18 NaN flag. All sums are FP64; a solid cell whose field entry is not finite
// only raises the flag (the reference skips it after counting its position).
enum AeroSlot { kAfx = 0, kAlw = 3, kAlwx = 4, kAfw = 7, kAfwx = 8, kAgx = 11, kAcount = 14, kAmaxz = 15,
                kAlo = 16, kAhi = 17, kAnan = 18 };

__device__ __forceinline__ void aero_init(double* a) {
    for (int k = 0; k < kAeroSlots; ++k) a[k] = 0.0;
    a[kAmaxz] = -1.0;
    a[kAlo] = 1e30;
    a[kAhi] = -1e30;
}

__device__ __forceinline__ void aero_merge(double* a, const double* b) {
    for (int k = 0; k <= kAcount; ++k) a[k] += b[k];
    a[kAmaxz] = fmax(a[kAmaxz], b[kAmaxz]);
    a[kAlo] = fmin(a[kAlo], b[kAlo]);
    a[kAhi] = fmax(a[kAhi], b[kAhi]);
    a[kAnan] = fmax(a[kAnan], b[kAnan]);
}

// Block reduction in a fixed order (shuffle tree, then warps in order).
__device__ void aero_block_reduce(double* a, double* out) {
    __shared__ double sh[kStatsThreads / 32][kAeroSlots];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        double b[kAeroSlots];
        for (int k = 0; k < kAeroSlots; ++k) b[k] = __shfl_down_sync(0xffffffffu, a[k], o);
        aero_merge(a, b);
    }
    if (lane == 0)
        for (int k = 0; k < kAeroSlots; ++k) sh[warp][k] = a[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kStatsThreads / 32; ++w) aero_merge(a, sh[w]);
        for (int k = 0; k < kAeroSlots; ++k) out[k] = a[k];
    }
}

template <int Q, class S, int Lay>
__global__ void __launch_bounds__(kStatsThreads) k_aero(const typename S::T* __restrict__ f,
                                                        const uint8_t* __restrict__ solid,
                                                        const float* __restrict__ sdf, Geom g, float cs, float ox,
                                                        float oy, float oz, double* __restrict__ partials,
                                                        int layout_in) {
    // the layout is a compile-time constant, so every slot folds to its
    // formula (plane * n + c for plane-major states)
    const int layout = Lay;
    (void)layout_in;
    double a[kAeroSlots];
    aero_init(a);
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < g.n; c += (size_t)gridDim.x * blockDim.x) {
        if (!solid[c]) continue;
        const int z = (int)(c / (size_t)g.nxy);
        const size_t rem = c - (size_t)z * g.nxy;
        const int y = (int)(rem / g.nx);
        const int x = (int)(rem - (size_t)y * g.nx);
        // VoxelGrid::CellCenter (VoxelGrid.h:53-55) in float
        const float px = ox + ((float)y + 0.5f) * cs;
        const float py = oy + ((float)x + 0.5f) * cs;
        const float pz = oz + ((float)z + 0.5f) * cs;
        a[kAgx] += (double)px;
        a[kAgx + 1] += (double)py;
        a[kAgx + 2] += (double)pz;
        a[kAcount] += 1.0;
        a[kAmaxz] = fmax(a[kAmaxz], (double)z);
        const float4 v = solid_force<Q, S>(f, solid, sdf, g, x, y, z, c, layout);
        if (!isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z) || !isfinite(v.w)) {
            a[kAnan] = 1.0;
            continue;
        }
        a[kAfx] += (double)v.y;
        a[kAfx + 1] += (double)v.z;
        a[kAfx + 2] += (double)v.w;
        const double wl = fabs((double)v.w);
        a[kAlw] += wl;
        a[kAlwx] += wl * px;
        a[kAlwx + 1] += wl * py;
        a[kAlwx + 2] += wl * pz;
        const double wf = sqrt((double)v.y * v.y + (double)v.z * v.z + (double)v.w * v.w);
        a[kAfw] += wf;
        a[kAfwx] += wf * px;
        a[kAfwx + 1] += wf * py;
        a[kAfwx + 2] += wf * pz;
        if (v.x > 0.0f) {
            a[kAlo] = fmin(a[kAlo], (double)v.x);
            a[kAhi] = fmax(a[kAhi], (double)v.x);
        }
    }
    aero_block_reduce(a, partials + (size_t)blockIdx.x * kAeroSlots);
}

// Reduces the partials, then computes the centre of pressure and the lift
// arrow's base from a 5x5 patch of columns around it (FieldOverlay.cpp:
// 580-618), one column per thread.
__global__ void __launch_bounds__(kStatsThreads) k_aero_final(const double* __restrict__ partials, int blocks,
                                                              const uint8_t* __restrict__ solid, Geom g, float cs,
                                                              float ox, float oy, float oz,
                                                              double* __restrict__ result) {
    __shared__ double tot[kAeroSlots];
    __shared__ float cp[3];
    __shared__ int col_top;
    double a[kAeroSlots];
    aero_init(a);
    for (int b = threadIdx.x; b < blocks; b += blockDim.x) aero_merge(a, partials + (size_t)b * kAeroSlots);
    aero_block_reduce(a, tot);
    if (threadIdx.x == 0) {
        col_top = -1;
        const double lw = tot[kAlw], fw = tot[kAfw], count = tot[kAcount];
        float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
        if (lw > 1e-9) {
            c0 = (float)(tot[kAlwx] / lw), c1 = (float)(tot[kAlwx + 1] / lw), c2 = (float)(tot[kAlwx + 2] / lw);
        } else if (fw > 1e-9) {
            c0 = (float)(tot[kAfwx] / fw), c1 = (float)(tot[kAfwx + 1] / fw), c2 = (float)(tot[kAfwx + 2] / fw);
        } else if (count > 0.0) {
            const double inv = 1.0 / count;
            c0 = (float)(tot[kAgx] * inv), c1 = (float)(tot[kAgx + 1] * inv), c2 = (float)(tot[kAgx + 2] * inv);
        }
        cp[0] = c0, cp[1] = c1, cp[2] = c2;
    }
    __syncthreads();
    if (threadIdx.x < 25) {
        const int nxm = g.nx - 1 > 0 ? g.nx - 1 : 0, nym = g.ny - 1 > 0 ? g.ny - 1 : 0;
        int gx = (int)floorf((cp[1] - oy) / cs), gy = (int)floorf((cp[0] - ox) / cs);
        gx = gx < 0 ? 0 : (gx > nxm ? nxm : gx);
        gy = gy < 0 ? 0 : (gy > nym ? nym : gy);
        int x = gx + (int)(threadIdx.x % 5) - 2, y = gy + (int)(threadIdx.x / 5) - 2;
        x = x < 0 ? 0 : (x > nxm ? nxm : x);
        y = y < 0 ? 0 : (y > nym ? nym : y);
        for (int z = g.nz - 1; z >= 0; --z)
            if (solid[((size_t)z * g.ny + y) * g.nx + x]) {
                atomicMax(&col_top, z);
                break;
            }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int maxz = (int)tot[kAmaxz];
        const int eff = col_top >= 0 ? col_top : (maxz > 0 ? maxz : 0);
        float lo = (float)tot[kAlo], hi = (float)tot[kAhi];
        if (lo > hi) {
            lo = 0.0f;
            hi = 1e-6f;
        } else {
            lo = 0.0f;
            if (!(hi > lo)) hi = lo + 1e-6f;
        }
        result[0] = tot[kAfx];
        result[1] = tot[kAfx + 1];
        result[2] = tot[kAfx + 2];
        result[3] = tot[kAlw];
        result[4] = tot[kAfw];
        result[5] = tot[kAcount];
        result[6] = lo;
        result[7] = hi;
        result[8] = tot[kAnan];
        result[9] = cp[0];
        result[10] = cp[1];
        result[11] = cp[2];
        result[12] = cp[0];
        result[13] = cp[1];
        result[14] = oz + ((float)eff + 1.0f) * cs;
        result[15] = (double)maxz;
    }
}

int stats_blocks(const Geom& g) {
    const size_t want = (g.n + kStatsThreads * 8 - 1) / (kStatsThreads * 8);
    const size_t cap = 148 * 16;
    return (int)(want < 1 ? 1 : (want > cap ? cap : want));
}

// Launches KERNEL<Q, S, layout> for the run-time `layout` (PopLayout).
#define FC_LAYOUT_LAUNCH(KERNEL, GRID, BLOCK, ...)                                        \
    do {                                                                                  \
        if (layout == kLayoutAAEven)                                                      \
            KERNEL<Q, S, kLayoutAAEven><<<GRID, BLOCK, 0, s>>>(__VA_ARGS__);              \
        else if (layout == kLayoutAAOdd)                                                  \
            KERNEL<Q, S, kLayoutAAOdd><<<GRID, BLOCK, 0, s>>>(__VA_ARGS__);               \
        else                                                                              \
            KERNEL<Q, S, kLayoutPlanes><<<GRID, BLOCK, 0, s>>>(__VA_ARGS__);              \
    } while (0)

template <int Q, class S>
static cudaError_t field_t(const void* f, const uint8_t* solid, const float* sdf, const Geom& g, size_t cell0,
                           size_t cells, float* out, int layout, cudaStream_t s) {
    if (cells == 0) return cudaSuccess;
    FC_LAYOUT_LAUNCH(k_field, (unsigned)((cells + 255) / 256), 256, (const typename S::T*)f, solid, sdf, g, cell0,
                     cells, (float4*)out, layout);
    return cudaGetLastError();
}

template <int Q, class S>
static cudaError_t probe_health_t(const void* f, const uint8_t* solid, const float* sdf, const Geom& g, size_t cell0,
                                  size_t cells, int* flag, int layout, cudaStream_t s) {
    if (cells == 0) return cudaSuccess;
    FC_LAYOUT_LAUNCH(k_probe_health, (unsigned)((cells + 255) / 256), 256, (const typename S::T*)f, solid, sdf, g,
                     cell0, cells, flag, layout);
    return cudaGetLastError();
}

template <int Q, class S>
static cudaError_t pops_out_t(const void* f, const uint8_t* solid, int sw, const Geom& g, size_t cell0, size_t cells,
                              float* out, int layout, cudaStream_t s) {
    if (cells == 0) return cudaSuccess;
    FC_LAYOUT_LAUNCH(k_pops_out, (unsigned)((cells + 255) / 256), 256, (const typename S::T*)f, solid, sw, g, cell0,
                     cells, out, layout);
    return cudaGetLastError();
}

template <int Q, class S>
static cudaError_t pops_in_t(void* f, const Geom& g, size_t cell0, size_t cells, const float* in, int layout,
                             cudaStream_t s) {
    if (cells == 0) return cudaSuccess;
    FC_LAYOUT_LAUNCH(k_pops_in, (unsigned)((cells + 255) / 256), 256, (typename S::T*)f, g, cell0, cells, in, layout);
    return cudaGetLastError();
}

template <int Q, class S>
static cudaError_t stats_t(const void* f, const uint8_t* solid, const float* sdf, const Geom& g, double* partials,
                           int blocks, double* result, int layout, cudaStream_t s) {
    FC_LAYOUT_LAUNCH(k_stats, blocks, kStatsThreads, (const typename S::T*)f, solid, sdf, g, partials, layout);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_stats_final<<<1, kStatsThreads, 0, s>>>(partials, blocks, result);
    return cudaGetLastError();
}

#define FC_DISPATCH(q, storage, FN, ...)                               \
    do {                                                               \
        if ((q) == 19) {                                               \
            if ((storage) == 0) return FN<19, StoreF32>(__VA_ARGS__);  \
            if ((storage) == 1) return FN<19, StoreF16>(__VA_ARGS__);  \
            if ((storage) == 2) return FN<19, StoreBF16>(__VA_ARGS__); \
        } else if ((q) == 15) {                                        \
            if ((storage) == 0) return FN<15, StoreF32>(__VA_ARGS__);  \
            if ((storage) == 1) return FN<15, StoreF16>(__VA_ARGS__);  \
            if ((storage) == 2) return FN<15, StoreBF16>(__VA_ARGS__); \
        }                                                              \
        return cudaErrorInvalidValue;                                  \
    } while (0)

cudaError_t launch_field(int q, int storage, const void* f, const uint8_t* solid, const float* sdf, const Geom& g,
                         size_t cell0, size_t cells, float* out, int layout, cudaStream_t s) {
    FC_DISPATCH(q, storage, field_t, f, solid, sdf, g, cell0, cells, out, layout, s);
}

cudaError_t launch_probe_health(int q, int storage, const void* f, const uint8_t* solid, const float* sdf,
                                const Geom& g, size_t cell0, size_t cells, int* flag, int layout, cudaStream_t s) {
    FC_DISPATCH(q, storage, probe_health_t, f, solid, sdf, g, cell0, cells, flag, layout, s);
}

cudaError_t launch_pops_out(int q, int storage, const void* f, const uint8_t* solid, int solid_is_weight,
                            const Geom& g, size_t cell0, size_t cells, float* out, int layout, cudaStream_t s) {
    FC_DISPATCH(q, storage, pops_out_t, f, solid, solid_is_weight, g, cell0, cells, out, layout, s);
}

cudaError_t launch_pops_in(int q, int storage, void* f, const Geom& g, size_t cell0, size_t cells, const float* in,
                           int layout, cudaStream_t s) {
    FC_DISPATCH(q, storage, pops_in_t, f, g, cell0, cells, in, layout, s);
}

cudaError_t launch_stats(int q, int storage, const void* f, const uint8_t* solid, const float* sdf, const Geom& g,
                         double* partials, int blocks, double* result, int layout, cudaStream_t s) {
    FC_DISPATCH(q, storage, stats_t, f, solid, sdf, g, partials, blocks, result, layout, s);
}

template <int Q, class S>
static cudaError_t aero_t(const void* f, const uint8_t* solid, const float* sdf, const Geom& g, float cs, float ox,
                          float oy, float oz, double* partials, int blocks, double* result, int layout,
                          cudaStream_t s) {
    FC_LAYOUT_LAUNCH(k_aero, blocks, kStatsThreads, (const typename S::T*)f, solid, sdf, g, cs, ox, oy, oz, partials,
                     layout);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_aero_final<<<1, kStatsThreads, 0, s>>>(partials, blocks, solid, g, cs, ox, oy, oz, result);
    return cudaGetLastError();
}

cudaError_t launch_aero(int q, int storage, const void* f, const uint8_t* solid, const float* sdf, const Geom& g,
                        float cell_size, float ox, float oy, float oz, double* partials, int blocks, double* result,
                        int layout, cudaStream_t s) {
    FC_DISPATCH(q, storage, aero_t, f, solid, sdf, g, cell_size, ox, oy, oz, partials, blocks, result, layout, s);
}

}  // namespace fc

// ---- statistics without allocation (fc_lbm_stats_noalloc) ----
// The same k_stats / k_stats_final kernels as fc_lbm_readback_stats, with the
// per-block partials in a fixed file-scope device array instead of memory the
// solver allocated. The array holds 4096 blocks' partials (4096 * 12 doubles
// = 384 KiB). The block count follows the allocating path's rule, one block
// per 2048 cells, capped here by the array instead of at 148 * 16: the
// reduction is grid-stride, so every cell is covered whatever the count, and
// below the allocating path's cap (4.8M cells) both paths form the same
// partial sums. Lattices are limited to 2^29 cells. Each launch writes every
// slot of the partials it uses before the final kernel reads them, so nothing
// has to be cleared between calls.
//
// The device address of the array is looked up once per device and cached for
// the life of the process. A cudaDeviceReset destroys the module that holds
// the array, so that cached address does not survive a reset; the header
// documents this.
namespace {

constexpr int kNoAllocMaxBlocks = 4096;
constexpr size_t kNoAllocCellsPerBlock = size_t(1) << 11;  // kStatsThreads * 8, as stats_blocks()
static_assert(fc::kStatsSlots == FC_LBM_STATS_SLOTS, "slot count must match the header");

static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxBlocks * fc::kStatsSlots];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_scratch[kNoAllocMaxDevices] = {};

}  // namespace

extern "C" FC_LBM_API int fc_lbm_stats_noalloc(const void* populations, const uint8_t* solid,
                                               const float* signed_distance, int32_t nx, int32_t ny, int32_t nz,
                                               int32_t model, int32_t storage, double* out_slots, void* stream) {
    if (!populations || !solid || !out_slots) return FC_LBM_ERR_INVALID_ARG;
    if (nx <= 0 || ny <= 0 || nz <= 0) return FC_LBM_ERR_INVALID_ARG;
    if (model != FC_LATTICE_D3Q15 && model != FC_LATTICE_D3Q19) return FC_LBM_ERR_INVALID_ARG;
    if (storage < FC_STORAGE_FP32 || storage > FC_STORAGE_BF16_OFFSET) return FC_LBM_ERR_INVALID_ARG;
    const size_t n = (size_t)nx * (size_t)ny * (size_t)nz;
    if (n > FC_LBM_NOALLOC_MAX_CELLS) return FC_LBM_ERR_TOO_LARGE;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return FC_LBM_ERR_CUDA;
    if (dev >= kNoAllocMaxDevices) return FC_LBM_ERR_UNSUPPORTED;
    double* scratch = nullptr;
    {
        // set-up, once per device, with that device current: the symbol's
        // host-side name is not a device address
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_scratch[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) return FC_LBM_ERR_CUDA;
            g_noalloc_scratch[dev] = static_cast<double*>(p);
        }
        scratch = g_noalloc_scratch[dev];
    }
    fc::Geom g{};
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.wpr = (nx + 31) / 32;
    g.nxy = (long long)nx * ny;
    g.n = n;
    const size_t want = (n + kNoAllocCellsPerBlock - 1) / kNoAllocCellsPerBlock;
    const int blocks = (int)(want < 1 ? 1 : (want > (size_t)kNoAllocMaxBlocks ? (size_t)kNoAllocMaxBlocks : want));
    const int q = model == FC_LATTICE_D3Q19 ? 19 : 15;
    const cudaError_t e = fc::launch_stats(q, storage, populations, solid, signed_distance, g, scratch, blocks,
                                           out_slots, fc::kLayoutPlanes, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? FC_LBM_OK : FC_LBM_ERR_CUDA;
}
