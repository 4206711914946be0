// Smoke-trail particles advected on the device (FlowCraft/SmokeTrail.cpp):
// SmokeTrailSystem::Step, Reset / ScatterRandom, Respawn and ShiftPlane over
// particles whose trails live in device memory, with the velocity sampled
// straight from the solver's populations instead of from a host copy of
// the whole field.
//
// Velocity: the reference interpolates (ux, uy, uz) of the 4-float field
// readback trilinearly between the 8 cells around a point
// (SampleVelocityInterpolated, SmokeTrail.cpp:69-116). Here each of the 8
// corners takes the moments of its populations (the same moments<Q> the
// field readback uses, so the same values), 0 at solid cells, and the
// blend runs in the reference's order with no fused multiply-adds, so a
// particle moves exactly as the reference moves it through the field.
//
// World space follows VoxelGrid::CellCenter (VoxelGrid.h:54-56): grid x is
// world Y, grid y is world X, z is z, cell centres at (index + 0.5) * cell.
//
// Random draws (respawn and scatter positions) come from a counter-based
// hash of (seed, particle, draw counter), not the reference's mt19937, so
// the particles an exit respawns land elsewhere than the reference's do;
// the rules (inlet face, 8 attempts at a non-solid cell, jitter inside the
// cell along the free axes) are the reference's.
#include "aa.cuh"
#include "collide.cuh"
#include "lbm_internal.h"
#include "storage.cuh"

namespace fc {

namespace {

struct V3 {
    float x, y, z;
};

__device__ __forceinline__ V3 v_add(V3 a, V3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 v_sub(V3 a, V3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 v_mul(V3 a, float s) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
// a + (b - a) * t, as the reference's Vec3 expressions round it
__device__ __forceinline__ V3 v_lerp(V3 a, V3 b, float t) { return v_add(a, v_mul(v_sub(b, a), t)); }

__device__ __forceinline__ bool in_grid(const Geom& g, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && x < g.nx && y < g.ny && z < g.nz;
}
__device__ __forceinline__ size_t cell_of(const Geom& g, int x, int y, int z) {
    return ((size_t)z * g.ny + y) * g.nx + x;
}

// splitmix64 of (seed, particle, draw): uniform in [0, 1)
__device__ __forceinline__ float rand01(unsigned long long seed, unsigned long long particle, unsigned long long draw) {
    unsigned long long z = seed + 0x9e3779b97f4a7c15ull * (particle * 0x100000001b3ull + draw + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return (float)(z >> 40) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ int rand_int(unsigned long long seed, unsigned long long particle, unsigned long long draw,
                                        int n) {
    int v = (int)(rand01(seed, particle, draw) * (float)n);
    return v < n ? v : n - 1;
}

// VoxelGrid::CellCenter (VoxelGrid.h:54-56)
__device__ __forceinline__ V3 cell_center(const SmokeParams& sp, int x, int y, int z) {
    return {__fadd_rn(sp.ox, __fmul_rn(__fadd_rn((float)y, 0.5f), sp.cs)),
            __fadd_rn(sp.oy, __fmul_rn(__fadd_rn((float)x, 0.5f), sp.cs)),
            __fadd_rn(sp.oz, __fmul_rn(__fadd_rn((float)z, 0.5f), sp.cs))};
}

// CellAt (SmokeTrail.cpp:36-61): the grid cell holding a world point
__device__ __forceinline__ bool cell_at(const SmokeParams& sp, const Geom& g, V3 pos, int& x, int& y, int& z) {
    const V3 l = {__fsub_rn(pos.x, sp.ox), __fsub_rn(pos.y, sp.oy), __fsub_rn(pos.z, sp.oz)};
    x = (int)floorf(__fdiv_rn(l.y, sp.cs));
    y = (int)floorf(__fdiv_rn(l.x, sp.cs));
    z = (int)floorf(__fdiv_rn(l.z, sp.cs));
    return in_grid(g, x, y, z);
}

// World velocity (uy, ux, uz) of a cell: the moments of its populations,
// 0 at a solid cell.
template <int Q, class S>
__device__ __forceinline__ V3 cell_velocity(const typename S::T* __restrict__ f, const uint8_t* __restrict__ solid,
                                            const Geom& g, int x, int y, int z, int layout) {
    x = x < 0 ? 0 : (x > g.nx - 1 ? g.nx - 1 : x);
    y = y < 0 ? 0 : (y > g.ny - 1 ? g.ny - 1 : y);
    z = z < 0 ? 0 : (z > g.nz - 1 ? g.nz - 1 : z);
    const size_t c = cell_of(g, x, y, z);
    if (solid[c]) return {0.0f, 0.0f, 0.0f};
    float p[Q];
    static_for<0, Q>([&](auto I) {
        constexpr int i = decltype(I)::value;
        p[i] = S::dec(S::ld(f + pop_slot<Q, i>(c, x, y, z, g, layout)), Lattice<Q>::w(i));
    });
    float rho, ux, uy, uz;
    moments<Q>(p, rho, ux, uy, uz);
    return {uy, ux, uz};
}

// SampleVelocityInterpolated (SmokeTrail.cpp:69-116)
template <int Q, class S>
__device__ V3 sample_velocity(const typename S::T* __restrict__ f, const uint8_t* __restrict__ solid, const Geom& g,
                              const SmokeParams& sp, V3 pos, int layout) {
    const V3 l = {__fsub_rn(pos.x, sp.ox), __fsub_rn(pos.y, sp.oy), __fsub_rn(pos.z, sp.oz)};
    const float gxf = __fsub_rn(__fdiv_rn(l.y, sp.cs), 0.5f);
    const float gyf = __fsub_rn(__fdiv_rn(l.x, sp.cs), 0.5f);
    const float gzf = __fsub_rn(__fdiv_rn(l.z, sp.cs), 0.5f);
    const int gx0 = (int)floorf(gxf), gy0 = (int)floorf(gyf), gz0 = (int)floorf(gzf);
    const float tx = __fsub_rn(gxf, (float)gx0), ty = __fsub_rn(gyf, (float)gy0), tz = __fsub_rn(gzf, (float)gz0);
    auto s = [&](int dx, int dy, int dz) { return cell_velocity<Q, S>(f, solid, g, gx0 + dx, gy0 + dy, gz0 + dz, layout); };
    const V3 c000 = s(0, 0, 0), c100 = s(1, 0, 0), c010 = s(0, 1, 0), c110 = s(1, 1, 0);
    const V3 c001 = s(0, 0, 1), c101 = s(1, 0, 1), c011 = s(0, 1, 1), c111 = s(1, 1, 1);
    const V3 c00 = v_lerp(c000, c100, tx), c10 = v_lerp(c010, c110, tx);
    const V3 c01 = v_lerp(c001, c101, tx), c11 = v_lerp(c011, c111, tx);
    const V3 c0 = v_lerp(c00, c10, ty), c1 = v_lerp(c01, c11, ty);
    return v_lerp(c0, c1, tz);
}

// PickCell (SmokeTrail.cpp:163-182): up to 8 draws of the free axes for a
// non-solid cell; the fixed coordinates (or the grid's centre on a free
// axis) when all 8 land in solid.
__device__ void pick_cell(const uint8_t* __restrict__ solid, const Geom& g, const SmokeParams& sp, int p,
                          unsigned long long& draw, int fx, int fy, int fz, int& ox, int& oy, int& oz) {
    ox = fx >= 0 ? fx : g.nx / 2;
    oy = fy >= 0 ? fy : g.ny / 2;
    oz = fz >= 0 ? fz : g.nz / 2;
    for (int attempt = 0; attempt < 8; ++attempt) {
        const int tx = fx >= 0 ? fx : rand_int(sp.seed, p, draw++, g.nx);
        const int ty = fy >= 0 ? fy : rand_int(sp.seed, p, draw++, g.ny);
        const int tz = fz >= 0 ? fz : rand_int(sp.seed, p, draw++, g.nz);
        if (!solid[cell_of(g, tx, ty, tz)]) {
            ox = tx, oy = ty, oz = tz;
            return;
        }
    }
}

// JitteredCellCenter (SmokeTrail.cpp:27-34): a point in the cell, uniform
// along the free grid axes (jitter in grid terms, swapped into world terms)
__device__ V3 jittered_center(const SmokeParams& sp, int p, unsigned long long& draw, int x, int y, int z, bool xf,
                              bool yf, bool zf) {
    const float jx = xf ? 0.0f : __fmul_rn(__fsub_rn(rand01(sp.seed, p, draw++), 0.5f), sp.cs);
    const float jy = yf ? 0.0f : __fmul_rn(__fsub_rn(rand01(sp.seed, p, draw++), 0.5f), sp.cs);
    const float jz = zf ? 0.0f : __fmul_rn(__fsub_rn(rand01(sp.seed, p, draw++), 0.5f), sp.cs);
    return v_add(cell_center(sp, x, y, z), V3{jy, jx, jz});
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ void trail_reset(const ParticleSet& ps, int p, V3 pos) {
    ps.trail[(size_t)p * ps.length] = make_float4(pos.x, pos.y, pos.z, 0.0f);
    ps.head[p] = 0;
    ps.len[p] = 1;
}

// Respawn (SmokeTrail.cpp:184-204): the inlet face, or the confinement plane
__device__ void respawn(const uint8_t* __restrict__ solid, const Geom& g, const SmokeParams& sp, const ParticleSet& ps,
                        int p, unsigned long long& draw) {
    const int fx = sp.confine_axis == 0 ? clampi(sp.confine_index, 0, g.nx - 1) : (sp.reverse ? g.nx - 1 : 0);
    const int fy = sp.confine_axis == 1 ? clampi(sp.confine_index, 0, g.ny - 1) : -1;
    const int fz = sp.confine_axis == 2 ? clampi(sp.confine_index, 0, g.nz - 1) : -1;
    int x, y, z;
    pick_cell(solid, g, sp, p, draw, fx, fy, fz, x, y, z);
    // the reference passes (fixedY < 0, fixedZ < 0) as the "fixed" flags
    // here (SmokeTrail.cpp:203), so a respawned point is jittered only along
    // a confined y / z axis; kept as is
    trail_reset(ps, p, jittered_center(sp, p, draw, x, y, z, true, fy < 0, fz < 0));
}

}  // namespace

// SmokeTrailSystem::Step (SmokeTrail.cpp:278-343), one thread per particle.
template <int Q, class S>
__global__ void __launch_bounds__(128) k_particles_step(const typename S::T* __restrict__ f, int layout,
                                                        const uint8_t* __restrict__ solid, Geom g, ParticleSet ps,
                                                        SmokeParams sp) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ps.count) return;
    unsigned long long draw = sp.counter;  // this call's draws: sp.counter .. sp.counter + 99
    const int n = ps.len[p];
    if (n == 0) {
        if (!sp.suspend) respawn(solid, g, sp, ps, p, draw);
        return;
    }
    const int h = ps.head[p];
    const float4 cf = ps.trail[(size_t)p * ps.length + h];
    const V3 cur = {cf.x, cf.y, cf.z};
    int cx, cy, cz;
    if (!cell_at(sp, g, cur, cx, cy, cz) || solid[cell_of(g, cx, cy, cz)]) {
        if (sp.suspend)
            ps.len[p] = 0;  // vanish until respawning resumes
        else
            respawn(solid, g, sp, ps, p, draw);
        return;
    }
    V3 vel = sample_velocity<Q, S>(static_cast<const typename S::T*>(f), solid, g, sp, cur, layout);
    // confined: no motion along the plane's normal (a grid axis, so the
    // world component it maps to)
    if (sp.confine_axis == 0) vel.y = 0.0f;
    if (sp.confine_axis == 1) vel.x = 0.0f;
    if (sp.confine_axis == 2) vel.z = 0.0f;
    const V3 next = v_add(cur, v_mul(vel, sp.scale));
    const int nh = h + 1 == ps.length ? 0 : h + 1;
    ps.trail[(size_t)p * ps.length + nh] = make_float4(next.x, next.y, next.z, 0.0f);
    ps.head[p] = nh;
    ps.len[p] = n < ps.length ? n + 1 : n;
}

// ScatterRandom (SmokeTrail.cpp:206-220): every particle to a single fresh
// point in a random non-solid cell of the domain or the confinement plane.
__global__ void __launch_bounds__(128) k_particles_scatter(const uint8_t* __restrict__ solid, Geom g, ParticleSet ps,
                                                           SmokeParams sp) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ps.count) return;
    unsigned long long draw = sp.counter;
    const int fx = sp.confine_axis == 0 ? clampi(sp.confine_index, 0, g.nx - 1) : -1;
    const int fy = sp.confine_axis == 1 ? clampi(sp.confine_index, 0, g.ny - 1) : -1;
    const int fz = sp.confine_axis == 2 ? clampi(sp.confine_index, 0, g.nz - 1) : -1;
    int x, y, z;
    pick_cell(solid, g, sp, p, draw, fx, fy, fz, x, y, z);
    trail_reset(ps, p, jittered_center(sp, p, draw, x, y, z, fx >= 0, fy >= 0, fz >= 0));
}

// ShiftPlane (SmokeTrail.cpp:222-255): every kept trail point onto the new
// plane along the same axis.
__global__ void __launch_bounds__(128) k_particles_shift(Geom g, ParticleSet ps, SmokeParams sp) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ps.count) return;
    const int a = sp.confine_axis;
    const int idx = clampi(sp.confine_index, 0, (a == 0 ? g.nx : (a == 1 ? g.ny : g.nz)) - 1);
    const V3 c = cell_center(sp, a == 0 ? idx : 0, a == 1 ? idx : 0, a == 2 ? idx : 0);
    for (int k = 0; k < ps.length; ++k) {
        float4& v = ps.trail[(size_t)p * ps.length + k];
        if (a == 0) v.y = c.y;
        if (a == 1) v.x = c.x;
        if (a == 2) v.z = c.z;
    }
}

// Trails oldest -> newest: out[(p * length + k) * 3 + 0..2], lens[p].
__global__ void __launch_bounds__(128) k_particles_gather(ParticleSet ps, float* __restrict__ out,
                                                          int* __restrict__ lens) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ps.count) return;
    const int n = ps.len[p], h = ps.head[p];
    lens[p] = n;
    for (int k = 0; k < ps.length; ++k) {
        float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (k < n) {
            int src = h - (n - 1) + k;
            if (src < 0) src += ps.length;
            v = ps.trail[(size_t)p * ps.length + src];
        }
        float* o = out + ((size_t)p * ps.length + k) * 3;
        o[0] = v.x, o[1] = v.y, o[2] = v.z;
    }
}

// Every particle to the single given point pos[p * 3 + 0..2].
__global__ void __launch_bounds__(128) k_particles_set(ParticleSet ps, const float* __restrict__ pos) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ps.count) return;
    trail_reset(ps, p, V3{pos[3 * (size_t)p], pos[3 * (size_t)p + 1], pos[3 * (size_t)p + 2]});
}

template <int Q, class S>
static cudaError_t particles_step_t(const void* f, int layout, const uint8_t* solid, const Geom& g,
                                    const ParticleSet& ps, const SmokeParams& sp, cudaStream_t s) {
    if (ps.count <= 0) return cudaSuccess;
    k_particles_step<Q, S><<<(ps.count + 127) / 128, 128, 0, s>>>((const typename S::T*)f, layout, solid, g, ps, sp);
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

cudaError_t launch_particles_step(int q, int storage, const void* f, int layout, const uint8_t* solid, const Geom& g,
                                  const ParticleSet& ps, const SmokeParams& sp, cudaStream_t s) {
    FC_DISPATCH(q, storage, particles_step_t, f, layout, solid, g, ps, sp, s);
}

cudaError_t launch_particles_scatter(const uint8_t* solid, const Geom& g, const ParticleSet& ps, const SmokeParams& sp,
                                     cudaStream_t s) {
    if (ps.count <= 0) return cudaSuccess;
    k_particles_scatter<<<(ps.count + 127) / 128, 128, 0, s>>>(solid, g, ps, sp);
    return cudaGetLastError();
}

cudaError_t launch_particles_shift(const Geom& g, const ParticleSet& ps, const SmokeParams& sp, cudaStream_t s) {
    if (ps.count <= 0) return cudaSuccess;
    k_particles_shift<<<(ps.count + 127) / 128, 128, 0, s>>>(g, ps, sp);
    return cudaGetLastError();
}

cudaError_t launch_particles_gather(const ParticleSet& ps, float* out, int* lens, cudaStream_t s) {
    if (ps.count <= 0) return cudaSuccess;
    k_particles_gather<<<(ps.count + 127) / 128, 128, 0, s>>>(ps, out, lens);
    return cudaGetLastError();
}

cudaError_t launch_particles_set(const ParticleSet& ps, const float* pos, cudaStream_t s) {
    if (ps.count <= 0) return cudaSuccess;
    k_particles_set<<<(ps.count + 127) / 128, 128, 0, s>>>(ps, pos);
    return cudaGetLastError();
}

}  // namespace fc
