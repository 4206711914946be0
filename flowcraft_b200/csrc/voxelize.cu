// Mesh voxelizer on the device: FlowCraft's Voxelizer::Voxelize
// (FlowCraft/Voxelizer.cpp:136-485) producing the solver's boundary input, the
// VoxelGrid solid mask and signed distance (FlowCraft/VoxelGrid.h:13-61),
// bit-identical to the reference's CPU build.
//
// Pipeline (one stream, blocking call):
//   1. grid: bounds of the vertices by a two-level reduction whose ties keep
//      the lowest vertex index, which is std::min/std::max's first-wins rule
//      (Mesh.h:56-59) even for signed zeros; then the padded domain, cell size
//      and dims exactly as Voxelizer.cpp:146-166;
//   2. triangles: one thread per triangle computes its unit normal and its
//      clamped cell box (Voxelizer.cpp:206-235) and counts the 8x8x8 raster
//      tiles the box touches; an exclusive scan places every (tile, triangle)
//      pair, written in triangle order; a stable radix sort on the tile id
//      groups them by tile keeping triangle order inside each tile, and a
//      run-length encode gives each occupied tile its triangle list;
//   3. raster: one 512-thread block per occupied tile, one cell per thread,
//      triangles staged through shared memory in index order; each cell keeps
//      its running signed distance, best normal projection and solid bit in
//      registers and applies the reference's update rule (Voxelizer.cpp:
//      236-293) for every triangle whose box holds it, so every cell sees the
//      same triangles in the same order as the CPU loop and rounds the same
//      IEEE operations (the library is built without FMA contraction, with
//      IEEE division and square root);
//   4. flood fill: fluid cells 6-connected to cell (0,0,0) are the exterior
//      (Voxelizer.cpp:295-454). Labels start as the start of each x-run in a
//      32-cell row segment (one warp ballot), then runs are joined across
//      segment, row and layer boundaries with a lock-free union-find that
//      links the larger root under the smaller (Playne & Hawick, "A new
//      algorithm for parallel connected-component labelling on GPUs", IEEE
//      TPDS 2018). The root of any component is its smallest cell index, so
//      the exterior is the component whose root is 0;
//   5. finalize: unreached fluid becomes solid and the signed distance is
//      reconciled with the classification (Voxelizer.cpp:456-481).
//
// Every loop over the union-find forest is bounded: labels strictly decrease
// along a parent chain, and the loops also stop after a fixed iteration count,
// setting an error bit the host turns into FC_LBM_ERR_CUDA.
#include <cuda_runtime.h>

#include <chrono>
#include <climits>
#include <cmath>
#include <cstdint>
#include <thread>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>
#include <cub/device/device_scan.cuh>

#include "fc_lbm.h"

namespace {

constexpr int kTile = 8;                    // raster tile edge (cells)
constexpr int kTileCells = kTile * kTile * kTile;
constexpr int kTriWords = 18;               // a[3] b[3] c[3] n[3] lo[3] hi[3]
constexpr int kBoundsBlocks = 148;
constexpr int kBoundsThreads = 256;
constexpr unsigned kMaxFindHops = 1u << 26;
constexpr int kMaxMergeRetries = 1 << 20;
constexpr int kWaitTimeoutMs = 600000;
constexpr int kErrBadIndex = 1;
constexpr int kErrUnionBound = 2;

struct Tri {
    float a[3], b[3], c[3], n[3];
    int lo[3], hi[3];  // clamped cell box, grid axes (x spans world y, y spans world x)
};
static_assert(sizeof(Tri) == kTriWords * 4, "triangle record layout");

struct V3 {
    float x, y, z;
};

__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 vmul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 vcross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float vlen(V3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
__device__ __forceinline__ float min3(float a, float b, float c) {
    float m = a;
    if (b < m) m = b;
    if (c < m) m = c;
    return m;
}
__device__ __forceinline__ float max3(float a, float b, float c) {
    float m = a;
    if (m < b) m = b;
    if (m < c) m = c;
    return m;
}

// float -> int as the x86-64 host converts it (cvttss2si): truncation in
// range, INT_MIN for NaN and out-of-range values. The device's own conversion
// saturates instead, which would change the clamped box of a triangle lying
// more than 2^31 cells outside the grid.
__device__ __forceinline__ int to_int_host(float f) {
    return (f >= -2147483648.0f && f < 2147483648.0f) ? (int)f : INT_MIN;
}

// Closest point on triangle (a, b, c) to p: Ericson's Voronoi-region method,
// the operation order of Voxelizer.cpp:89-129.
__device__ __forceinline__ V3 closest_on_triangle(V3 p, V3 a, V3 b, V3 c) {
    const V3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a);
    const float d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) return a;
    const V3 bp = vsub(p, b);
    const float d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) return b;
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float v = d1 / (d1 - d3);
        return vadd(a, vmul(ab, v));
    }
    const V3 cp = vsub(p, c);
    const float d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) return c;
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float w = d2 / (d2 - d6);
        return vadd(a, vmul(ac, w));
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return vadd(b, vmul(vsub(c, b), w));
    }
    const float denom = 1.0f / (va + vb + vc);
    const float v = vb * denom, w = vc * denom;
    return vadd(vadd(a, vmul(ab, v)), vmul(ac, w));
}

// ---- 1. grid from the mesh bounds ----

// (value, vertex index) with "smaller value, then smaller index" order: the
// minimum over a set is the first vertex holding the smallest value, which is
// what a sequential `min = std::min(min, v)` keeps (it never replaces an equal
// value, so -0.0 and +0.0 keep whichever came first). For the maximum the
// value order flips and the index order stays.
struct Pick {
    float v;
    unsigned i;
};
__device__ __forceinline__ Pick pick_min(Pick a, Pick b) {
    return (b.v < a.v || (b.v == a.v && b.i < a.i)) ? b : a;
}
__device__ __forceinline__ Pick pick_max(Pick a, Pick b) {
    return (a.v < b.v || (b.v == a.v && b.i < a.i)) ? b : a;
}

__device__ __forceinline__ Pick shfl_pick(Pick p, int off) {
    p.v = __shfl_down_sync(0xffffffffu, p.v, off);
    p.i = __shfl_down_sync(0xffffffffu, p.i, off);
    return p;
}

// The reduction's identity is the reference's starting value (FLT_MAX for the
// minimum, lowest() for the maximum) with an index behind every vertex, so a
// vertex equal to it (or NaN, which never compares less) leaves the same
// bits the sequential loop leaves.
__global__ void __launch_bounds__(kBoundsThreads) k_bounds_partial(const float* __restrict__ pos, unsigned nv,
                                                                   Pick* __restrict__ partial) {
    Pick mn[3], mx[3];
    for (int k = 0; k < 3; ++k) {
        mn[k] = {3.402823466e38f, 0xffffffffu};
        mx[k] = {-3.402823466e38f, 0xffffffffu};
    }
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
        for (int k = 0; k < 3; ++k) {
            const Pick p{pos[3 * (size_t)i + k], i};
            mn[k] = pick_min(mn[k], p);
            mx[k] = pick_max(mx[k], p);
        }
    }
    __shared__ Pick s[6][kBoundsThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < 3; ++k) {
        for (int off = 16; off > 0; off >>= 1) {
            mn[k] = pick_min(mn[k], shfl_pick(mn[k], off));
            mx[k] = pick_max(mx[k], shfl_pick(mx[k], off));
        }
        if (lane == 0) {
            s[k][warp] = mn[k];
            s[3 + k][warp] = mx[k];
        }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int k = threadIdx.x;
        Pick r = s[k][0];
        for (int w = 1; w < kBoundsThreads / 32; ++w) r = k < 3 ? pick_min(r, s[k][w]) : pick_max(r, s[k][w]);
        partial[blockIdx.x * 6 + k] = r;
    }
}

struct GridOut {
    int dims[3];
    float cell;
    float origin[3];
};

// Voxelizer.cpp:146-166, one thread.
__global__ void k_grid_final(const Pick* __restrict__ partial, int blocks, int target_res, float padx, float pady,
                             float padz, GridOut* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Pick r[6];
    for (int k = 0; k < 6; ++k) {
        r[k] = partial[k];
        for (int b = 1; b < blocks; ++b) r[k] = k < 3 ? pick_min(r[k], partial[b * 6 + k]) : pick_max(r[k], partial[b * 6 + k]);
    }
    const V3 mn{r[0].v, r[1].v, r[2].v}, mx{r[3].v, r[4].v, r[5].v};
    const V3 size = vsub(mx, mn);
    const V3 pad{size.x * padx, size.y * pady, size.z * padz};
    const V3 dmin = vsub(mn, pad), dmax = vadd(mx, pad);
    const V3 dsize = vsub(dmax, dmin);
    const float longest = max3(dsize.x, dsize.y, dsize.z);
    const int res = target_res > 4 ? target_res : 4;
    float cs = longest / (float)res;
    if (cs < 1e-6f) cs = 1e-6f;
    const int nx = to_int_host(ceilf(dsize.y / cs)), ny = to_int_host(ceilf(dsize.x / cs)),
              nz = to_int_host(ceilf(dsize.z / cs));
    out->dims[0] = nx > 1 ? nx : 1;
    out->dims[1] = ny > 1 ? ny : 1;
    out->dims[2] = nz > 1 ? nz : 1;
    out->cell = cs;
    out->origin[0] = dmin.x;
    out->origin[1] = dmin.y;
    out->origin[2] = dmin.z;
}

// ---- 2. triangle records and tile binning ----

struct GridDev {
    int nx, ny, nz;
    int tx, ty, tz;  // tiles per axis
    float cs, cr;
    float ox, oy, oz;
};

__global__ void k_tri_prep(const float* __restrict__ pos, unsigned nv, const uint32_t* __restrict__ idx,
                           unsigned ntri, GridDev g, Tri* __restrict__ tris, unsigned long long* __restrict__ counts,
                           int* __restrict__ err) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > ntri) return;
    if (t == ntri) {  // the scan's trailing slot, so offsets[ntri] is the pair total
        counts[t] = 0;
        return;
    }
    const uint32_t i0 = idx[3 * (size_t)t], i1 = idx[3 * (size_t)t + 1], i2 = idx[3 * (size_t)t + 2];
    if (i0 >= nv || i1 >= nv || i2 >= nv) {
        atomicOr(err, kErrBadIndex);
        counts[t] = 0;
        return;
    }
    const V3 a{pos[3 * (size_t)i0], pos[3 * (size_t)i0 + 1], pos[3 * (size_t)i0 + 2]};
    const V3 b{pos[3 * (size_t)i1], pos[3 * (size_t)i1 + 1], pos[3 * (size_t)i1 + 2]};
    const V3 c{pos[3 * (size_t)i2], pos[3 * (size_t)i2 + 1], pos[3 * (size_t)i2 + 2]};
    const V3 rn = vcross(vsub(b, a), vsub(c, a));
    const float nl = vlen(rn);
    Tri r;
    r.a[0] = a.x, r.a[1] = a.y, r.a[2] = a.z;
    r.b[0] = b.x, r.b[1] = b.y, r.b[2] = b.z;
    r.c[0] = c.x, r.c[1] = c.y, r.c[2] = c.z;
    unsigned long long cnt = 0;
    if (nl <= 1e-12f) {  // zero-area triangles touch no cell
        r.n[0] = r.n[1] = r.n[2] = 0.0f;
        r.lo[0] = r.lo[1] = r.lo[2] = 1;
        r.hi[0] = r.hi[1] = r.hi[2] = 0;
    } else {
        const V3 un = vmul(rn, 1.0f / nl);
        r.n[0] = un.x, r.n[1] = un.y, r.n[2] = un.z;
        const V3 tmin{min3(a.x, b.x, c.x), min3(a.y, b.y, c.y), min3(a.z, b.z, c.z)};
        const V3 tmax{max3(a.x, b.x, c.x), max3(a.y, b.y, c.y), max3(a.z, b.z, c.z)};
        int lo0 = to_int_host(floorf((tmin.y - g.cr - g.oy) / g.cs));
        int lo1 = to_int_host(floorf((tmin.x - g.cr - g.ox) / g.cs));
        int lo2 = to_int_host(floorf((tmin.z - g.cr - g.oz) / g.cs));
        int hi0 = to_int_host(ceilf((tmax.y + g.cr - g.oy) / g.cs));
        int hi1 = to_int_host(ceilf((tmax.x + g.cr - g.ox) / g.cs));
        int hi2 = to_int_host(ceilf((tmax.z + g.cr - g.oz) / g.cs));
        lo0 = lo0 < 0 ? 0 : lo0;
        lo1 = lo1 < 0 ? 0 : lo1;
        lo2 = lo2 < 0 ? 0 : lo2;
        hi0 = hi0 > g.nx - 1 ? g.nx - 1 : hi0;
        hi1 = hi1 > g.ny - 1 ? g.ny - 1 : hi1;
        hi2 = hi2 > g.nz - 1 ? g.nz - 1 : hi2;
        r.lo[0] = lo0, r.lo[1] = lo1, r.lo[2] = lo2;
        r.hi[0] = hi0, r.hi[1] = hi1, r.hi[2] = hi2;
        if (lo0 <= hi0 && lo1 <= hi1 && lo2 <= hi2)
            cnt = (unsigned long long)(hi0 / kTile - lo0 / kTile + 1) * (hi1 / kTile - lo1 / kTile + 1) *
                  (hi2 / kTile - lo2 / kTile + 1);
    }
    tris[t] = r;
    counts[t] = cnt;
}

__global__ void k_tri_emit(const Tri* __restrict__ tris, const unsigned long long* __restrict__ offsets,
                           unsigned ntri, GridDev g, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntri) return;
    const unsigned long long off = offsets[t], end = offsets[t + 1];
    if (off == end) return;
    const Tri& r = tris[t];
    const int x0 = r.lo[0] / kTile, x1 = r.hi[0] / kTile;
    const int y0 = r.lo[1] / kTile, y1 = r.hi[1] / kTile;
    const int z0 = r.lo[2] / kTile, z1 = r.hi[2] / kTile;
    unsigned long long o = off;
    for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y)
            for (int x = x0; x <= x1; ++x) {
                keys[o] = (uint32_t)(((size_t)z * g.ty + y) * g.tx + x);
                vals[o] = t;
                ++o;
            }
}

// ---- 3. raster ----

__global__ void k_vox_init(uint8_t* __restrict__ solid, float* __restrict__ sdf, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        solid[i] = 0;
        sdf[i] = INFINITY;
    }
}

__global__ void __launch_bounds__(kTileCells) k_vox_raster(const Tri* __restrict__ tris,
                                                          const uint32_t* __restrict__ tile_tris,
                                                          const uint32_t* __restrict__ run_tile,
                                                          const uint32_t* __restrict__ run_len,
                                                          const unsigned long long* __restrict__ run_off, GridDev g,
                                                          uint8_t* __restrict__ solid, float* __restrict__ sdf) {
    __shared__ Tri s_tri[kTileCells];
    const uint32_t tile = run_tile[blockIdx.x];
    const unsigned count = run_len[blockIdx.x];
    const unsigned long long first = run_off[blockIdx.x];
    const int tx = (int)(tile % (uint32_t)g.tx);
    const int ty = (int)((tile / (uint32_t)g.tx) % (uint32_t)g.ty);
    const int tz = (int)(tile / ((uint32_t)g.tx * (uint32_t)g.ty));
    const int x = tx * kTile + (threadIdx.x & 7);
    const int y = ty * kTile + ((threadIdx.x >> 3) & 7);
    const int z = tz * kTile + (threadIdx.x >> 6);
    const bool inside = x < g.nx && y < g.ny && z < g.nz;
    // CellCenter: world x from grid y, world y from grid x (VoxelGrid.h:43-56)
    const V3 ctr{g.ox + ((float)y + 0.5f) * g.cs, g.oy + ((float)x + 0.5f) * g.cs, g.oz + ((float)z + 0.5f) * g.cs};
    const float tie = g.cs * 1e-3f;
    float sd = INFINITY, bp = -1.0f;
    bool sol = false;
    for (unsigned base = 0; base < count; base += kTileCells) {
        const unsigned m = count - base < (unsigned)kTileCells ? count - base : (unsigned)kTileCells;
        __syncthreads();
        if (threadIdx.x < m) s_tri[threadIdx.x] = tris[tile_tris[first + base + threadIdx.x]];
        __syncthreads();
        if (!inside) continue;
        for (unsigned k = 0; k < m; ++k) {
            const Tri& r = s_tri[k];
            if (x < r.lo[0] || x > r.hi[0] || y < r.lo[1] || y > r.hi[1] || z < r.lo[2] || z > r.hi[2]) continue;
            const V3 a{r.a[0], r.a[1], r.a[2]}, b{r.b[0], r.b[1], r.b[2]}, c{r.c[0], r.c[1], r.c[2]};
            const V3 un{r.n[0], r.n[1], r.n[2]};
            const V3 cl = closest_on_triangle(ctr, a, b, c);
            const V3 diff = vsub(ctr, cl);
            const float dist = vlen(diff);
            const float nd = vdot(diff, un);
            const float and_ = fabsf(nd);
            const float bd = fabsf(sd);
            // Voxelizer.cpp:258-290: a clearly nearer triangle replaces the
            // cell's distance; within the tie tolerance the one whose normal
            // points more directly at the cell decides the sign
            if (dist + tie < bd) {
                sd = nd < 0.0f ? -dist : dist;
                bp = and_;
            } else if (dist <= bd + tie) {
                if (and_ > bp) {
                    const float md = dist < bd ? dist : bd;
                    sd = nd < 0.0f ? -md : md;
                    bp = and_;
                } else if (dist < bd) {
                    sd = sd < 0.0f ? -dist : dist;
                }
            }
            if (dist <= g.cr) sol = true;
        }
    }
    if (inside) {
        const size_t i = ((size_t)z * g.ny + y) * g.nx + x;
        solid[i] = sol ? 1 : 0;
        sdf[i] = sd;
    }
}

// ---- 4. flood fill (connected components of fluid cells) ----

__device__ __forceinline__ uint32_t find_root(const uint32_t* __restrict__ L, uint32_t a, int* err) {
    for (unsigned hop = 0; hop < kMaxFindHops; ++hop) {
        const uint32_t p = __ldcg(L + a);
        if (p == a) return a;
        a = p;
    }
    atomicOr(err, kErrUnionBound);
    return a;
}

__device__ void unite(uint32_t* L, uint32_t a, uint32_t b, int* err) {
    for (int it = 0; it < kMaxMergeRetries; ++it) {
        a = find_root(L, a, err);
        b = find_root(L, b, err);
        if (a == b) return;
        if (a < b) {
            const uint32_t old = atomicMin(L + b, a);
            if (old == b) return;
            b = old;
        } else {
            const uint32_t old = atomicMin(L + a, b);
            if (old == a) return;
            a = old;
        }
    }
    atomicOr(err, kErrUnionBound);
}

// One warp per 32-cell segment of an x row; segments never straddle rows.
struct SegPos {
    size_t row;  // z * ny + y
    int x, y, z;
    bool valid;
};

__device__ __forceinline__ SegPos seg_pos(int nx, int ny, int nz, int wpr) {
    const size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    SegPos s;
    const size_t row = warp / (size_t)wpr;
    s.row = row;
    s.x = (int)(warp % (size_t)wpr) * 32 + lane;
    s.y = (int)(row % (size_t)ny);
    s.z = (int)(row / (size_t)ny);
    s.valid = s.z < nz;
    return s;
}

__global__ void k_ff_init(const uint8_t* __restrict__ solid, uint32_t* __restrict__ L, int nx, int ny, int nz,
                          int wpr) {
    const SegPos s = seg_pos(nx, ny, nz, wpr);
    if (!s.valid) return;  // warp-uniform
    const int lane = threadIdx.x & 31;
    const size_t i = s.row * nx + s.x;
    const bool fl = s.x < nx && !solid[i];
    const unsigned F = __ballot_sync(0xffffffffu, fl);
    const unsigned starts = F & ~(F << 1);
    if (fl) {
        const unsigned upto = starts & (0xffffffffu >> (31 - lane));
        const int start = 31 - __clz(upto);
        L[i] = (uint32_t)(s.row * nx + (s.x - lane + start));
    }
}

// Joins runs across the segment's left edge and to the row below and the layer
// below. Within a segment only the first cell of every stretch where both the
// cell and its neighbour are fluid unites: the rest of the stretch is already
// in the same runs on both sides.
__global__ void k_ff_merge(const uint8_t* __restrict__ solid, uint32_t* __restrict__ L, int nx, int ny, int nz,
                           int wpr, int* __restrict__ err) {
    const SegPos s = seg_pos(nx, ny, nz, wpr);
    if (!s.valid) return;
    const int lane = threadIdx.x & 31;
    const size_t i = s.row * nx + s.x;
    const bool in = s.x < nx;
    const bool fl = in && !solid[i];
    const unsigned F = __ballot_sync(0xffffffffu, fl);
    if (lane == 0 && fl && s.x > 0 && !solid[i - 1]) unite(L, (uint32_t)i, (uint32_t)(i - 1), err);
    if (s.y > 0) {
        const unsigned B = F & __ballot_sync(0xffffffffu, in && !solid[i - nx]);
        if ((B & ~(B << 1)) >> lane & 1u) unite(L, (uint32_t)i, (uint32_t)(i - nx), err);
    }
    if (s.z > 0) {
        const size_t layer = (size_t)nx * ny;
        const unsigned B = F & __ballot_sync(0xffffffffu, in && !solid[i - layer]);
        if ((B & ~(B << 1)) >> lane & 1u) unite(L, (uint32_t)i, (uint32_t)(i - layer), err);
    }
}

// ---- 5. finalize ----

__global__ void k_vox_finalize(uint8_t* __restrict__ solid, float* __restrict__ sdf, const uint32_t* __restrict__ L,
                               size_t n, float cr, int* __restrict__ err) {
    // cell 0 keeps its class through this pass (fluid there is the root 0 of
    // its own component), so every thread may read it
    const bool seed = solid[0] == 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        bool s = solid[i] != 0;
        if (!s) s = !seed || find_root(L, L[i], err) != 0u;
        const float d = fabsf(sdf[i]);
        if (!s)
            sdf[i] = d;
        else if (d > cr)
            sdf[i] = -d;
        solid[i] = s ? 1 : 0;
    }
}

// ---- host side ----

int wait_on(cudaStream_t s) {
    cudaEvent_t ev;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return FC_LBM_ERR_CUDA;
    if (cudaEventRecord(ev, s) != cudaSuccess) {
        cudaEventDestroy(ev);
        return FC_LBM_ERR_CUDA;
    }
    const auto t0 = std::chrono::steady_clock::now();
    int sleep_us = 20;
    int rc = FC_LBM_OK;
    for (;;) {
        const cudaError_t q = cudaEventQuery(ev);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) {
            rc = FC_LBM_ERR_CUDA;
            break;
        }
        if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(kWaitTimeoutMs)) {
            rc = FC_LBM_ERR_TIMEOUT;
            break;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(sleep_us));
        if (sleep_us < 2000) sleep_us *= 2;
    }
    cudaEventDestroy(ev);
    return rc;
}

// Stream-ordered scratch allocations, freed together on the same stream when
// the call returns (every path that hands results back has waited first).
struct Scratch {
    cudaStream_t s;
    void* ptrs[24] = {};
    int n = 0;
    explicit Scratch(cudaStream_t st) : s(st) {}
    template <class T>
    cudaError_t get(T** p, size_t bytes) {
        *p = nullptr;
        if (n >= 24) return cudaErrorInvalidValue;
        void* q = nullptr;
        const cudaError_t e = cudaMallocAsync(&q, bytes ? bytes : 16, s);
        if (e != cudaSuccess) return e;
        ptrs[n++] = q;
        *p = static_cast<T*>(q);
        return cudaSuccess;
    }
    ~Scratch() {
        for (int i = n - 1; i >= 0; --i) cudaFreeAsync(ptrs[i], s);
    }
};

int code_of(cudaError_t e) {
    if (e == cudaSuccess) return FC_LBM_OK;
    if (e == cudaErrorMemoryAllocation) return FC_LBM_ERR_OUT_OF_MEMORY;
    return FC_LBM_ERR_CUDA;
}

#define VX_TRY(expr)                                   \
    do {                                               \
        const cudaError_t _e = (expr);                 \
        if (_e != cudaSuccess) return code_of(_e);     \
    } while (0)

#define VX_RC(expr)                     \
    do {                                \
        const int _rc = (expr);         \
        if (_rc != FC_LBM_OK) return _rc; \
    } while (0)

int bits_for(uint64_t v) {
    int b = 1;
    while (b < 32 && (uint64_t(1) << b) <= v) ++b;
    return b;
}

int grid_on_device(const float* d_pos, size_t nv, const fc_voxel_params* p, cudaStream_t s, Scratch& sc,
                   GridOut* host) {
    Pick* partial = nullptr;
    GridOut* d_out = nullptr;
    VX_TRY(sc.get(&partial, sizeof(Pick) * 6 * kBoundsBlocks));
    VX_TRY(sc.get(&d_out, sizeof(GridOut)));
    k_bounds_partial<<<kBoundsBlocks, kBoundsThreads, 0, s>>>(d_pos, (unsigned)nv, partial);
    VX_TRY(cudaGetLastError());
    k_grid_final<<<1, 32, 0, s>>>(partial, kBoundsBlocks, p->target_resolution, p->padding[0], p->padding[1],
                                  p->padding[2], d_out);
    VX_TRY(cudaGetLastError());
    VX_TRY(cudaMemcpyAsync(host, d_out, sizeof(GridOut), cudaMemcpyDeviceToHost, s));
    VX_RC(wait_on(s));
    return FC_LBM_OK;
}

int voxelize_on_device(const float* d_pos, size_t nv, const uint32_t* d_idx, size_t ni, const int32_t dims[3],
                       float cell_size, const float origin[3], uint8_t* d_solid, float* d_sdf, cudaStream_t s,
                       Scratch& sc) {
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    const size_t n = (size_t)nx * ny * nz;
    GridDev g;
    g.nx = nx, g.ny = ny, g.nz = nz;
    g.tx = (nx + kTile - 1) / kTile, g.ty = (ny + kTile - 1) / kTile, g.tz = (nz + kTile - 1) / kTile;
    g.cs = cell_size;
    g.cr = cell_size * 0.8660254f;
    g.ox = origin[0], g.oy = origin[1], g.oz = origin[2];
    const unsigned ntri = (unsigned)(ni / 3);
    const uint64_t ntiles = (uint64_t)g.tx * g.ty * g.tz;

    int* d_err = nullptr;
    VX_TRY(sc.get(&d_err, sizeof(int)));
    VX_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), s));
    const int init_blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)148 * 16);
    k_vox_init<<<init_blocks, 256, 0, s>>>(d_solid, d_sdf, n);
    VX_TRY(cudaGetLastError());

    if (ntri > 0) {
        Tri* tris = nullptr;
        unsigned long long *counts = nullptr, *offsets = nullptr;
        VX_TRY(sc.get(&tris, sizeof(Tri) * ntri));
        VX_TRY(sc.get(&counts, sizeof(unsigned long long) * (ntri + 1)));
        VX_TRY(sc.get(&offsets, sizeof(unsigned long long) * (ntri + 1)));
        k_tri_prep<<<(ntri + 1 + 255) / 256, 256, 0, s>>>(d_pos, (unsigned)nv, d_idx, ntri, g, tris, counts, d_err);
        VX_TRY(cudaGetLastError());
        size_t tmp_bytes = 0;
        VX_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, counts, offsets, (int64_t)ntri + 1, s));
        void* tmp = nullptr;
        VX_TRY(sc.get(&tmp, tmp_bytes));
        VX_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, counts, offsets, (int64_t)ntri + 1, s));
        unsigned long long pairs = 0;
        int herr = 0;
        VX_TRY(cudaMemcpyAsync(&pairs, offsets + ntri, sizeof(pairs), cudaMemcpyDeviceToHost, s));
        VX_TRY(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
        VX_RC(wait_on(s));
        if (herr & kErrBadIndex) return FC_LBM_ERR_INVALID_ARG;
        if (pairs > (unsigned long long)INT32_MAX) return FC_LBM_ERR_TOO_LARGE;
        if (pairs > 0) {
            uint32_t *k0, *k1, *v0, *v1, *run_tile, *run_len;
            unsigned long long* run_off = nullptr;
            int* d_runs = nullptr;
            VX_TRY(sc.get(&k0, 4 * pairs));
            VX_TRY(sc.get(&k1, 4 * pairs));
            VX_TRY(sc.get(&v0, 4 * pairs));
            VX_TRY(sc.get(&v1, 4 * pairs));
            k_tri_emit<<<(ntri + 255) / 256, 256, 0, s>>>(tris, offsets, ntri, g, k0, v0);
            VX_TRY(cudaGetLastError());
            cub::DoubleBuffer<uint32_t> kb(k0, k1), vb(v0, v1);
            const int end_bit = bits_for(ntiles);
            size_t sort_bytes = 0;
            VX_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, kb, vb, (int)pairs, 0, end_bit, s));
            void* sort_tmp = nullptr;
            VX_TRY(sc.get(&sort_tmp, sort_bytes));
            VX_TRY(cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, kb, vb, (int)pairs, 0, end_bit, s));
            const uint64_t max_runs = std::min<uint64_t>(pairs, ntiles);
            VX_TRY(sc.get(&run_tile, 4 * max_runs));
            VX_TRY(sc.get(&run_len, 4 * max_runs));
            VX_TRY(sc.get(&run_off, 8 * max_runs));
            VX_TRY(sc.get(&d_runs, sizeof(int)));
            size_t rle_bytes = 0;
            VX_TRY(cub::DeviceRunLengthEncode::Encode(nullptr, rle_bytes, kb.Current(), run_tile, run_len, d_runs,
                                                       (int)pairs, s));
            void* rle_tmp = nullptr;
            VX_TRY(sc.get(&rle_tmp, rle_bytes));
            VX_TRY(cub::DeviceRunLengthEncode::Encode(rle_tmp, rle_bytes, kb.Current(), run_tile, run_len, d_runs,
                                                       (int)pairs, s));
            int runs = 0;
            VX_TRY(cudaMemcpyAsync(&runs, d_runs, sizeof(int), cudaMemcpyDeviceToHost, s));
            VX_RC(wait_on(s));
            size_t scan2 = 0;
            VX_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan2, run_len, run_off, (int64_t)runs, s));
            void* scan2_tmp = nullptr;
            VX_TRY(sc.get(&scan2_tmp, scan2));
            VX_TRY(cub::DeviceScan::ExclusiveSum(scan2_tmp, scan2, run_len, run_off, (int64_t)runs, s));
            if (runs > 0) {
                k_vox_raster<<<runs, kTileCells, 0, s>>>(tris, vb.Current(), run_tile, run_len, run_off, g, d_solid,
                                                         d_sdf);
                VX_TRY(cudaGetLastError());
            }
        }
    }

    uint32_t* L = nullptr;
    VX_TRY(sc.get(&L, sizeof(uint32_t) * n));
    const int wpr = (nx + 31) / 32;
    const size_t segs = (size_t)wpr * ny * nz;
    const size_t ff_blocks = (segs * 32 + 255) / 256;
    if (ff_blocks > (size_t)INT32_MAX) return FC_LBM_ERR_TOO_LARGE;
    k_ff_init<<<(unsigned)ff_blocks, 256, 0, s>>>(d_solid, L, nx, ny, nz, wpr);
    VX_TRY(cudaGetLastError());
    k_ff_merge<<<(unsigned)ff_blocks, 256, 0, s>>>(d_solid, L, nx, ny, nz, wpr, d_err);
    VX_TRY(cudaGetLastError());
    k_vox_finalize<<<init_blocks, 256, 0, s>>>(d_solid, d_sdf, L, n, g.cr, d_err);
    VX_TRY(cudaGetLastError());
    int herr = 0;
    VX_TRY(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    VX_RC(wait_on(s));
    return herr ? FC_LBM_ERR_CUDA : FC_LBM_OK;
}

bool finite3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

}  // namespace

extern "C" {

FC_LBM_API int fc_lbm_voxel_grid(const float* positions, size_t vertex_count, const fc_voxel_params* params,
                                 int32_t memory, int32_t dims[3], float* cell_size, float origin[3], void* stream) {
    if (!positions || !params || !dims || !cell_size || !origin) return FC_LBM_ERR_INVALID_ARG;
    if (memory != FC_MEMORY_HOST && memory != FC_MEMORY_DEVICE) return FC_LBM_ERR_INVALID_ARG;
    if (vertex_count == 0 || vertex_count >= 0xffffffffu) return FC_LBM_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    GridOut out{};
    int rc;
    {
        Scratch sc(s);
        const float* d_pos = positions;
        if (memory == FC_MEMORY_HOST) {
            float* p = nullptr;
            VX_TRY(sc.get(&p, 12 * vertex_count));
            VX_TRY(cudaMemcpyAsync(p, positions, 12 * vertex_count, cudaMemcpyHostToDevice, s));
            d_pos = p;
        }
        rc = grid_on_device(d_pos, vertex_count, params, s, sc, &out);
    }
    if (rc != FC_LBM_OK) return rc;
    for (int k = 0; k < 3; ++k) {
        dims[k] = out.dims[k];
        origin[k] = out.origin[k];
    }
    *cell_size = out.cell;
    return FC_LBM_OK;
}

FC_LBM_API int fc_lbm_voxelize(const float* positions, size_t vertex_count, const uint32_t* indices,
                               size_t index_count, const int32_t dims[3], float cell_size, const float origin[3],
                               int32_t memory, uint8_t* solid, float* signed_distance, void* stream) {
    if (!dims || !origin || !solid || !signed_distance) return FC_LBM_ERR_INVALID_ARG;
    if (memory != FC_MEMORY_HOST && memory != FC_MEMORY_DEVICE) return FC_LBM_ERR_INVALID_ARG;
    if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0) return FC_LBM_ERR_INVALID_ARG;
    if (!(cell_size > 0.0f) || !std::isfinite(cell_size) || !finite3(origin)) return FC_LBM_ERR_INVALID_ARG;
    if (index_count >= 3 && (!positions || !indices || vertex_count == 0)) return FC_LBM_ERR_INVALID_ARG;
    if (vertex_count >= 0xffffffffu || index_count / 3 >= 0xffffffffu) return FC_LBM_ERR_TOO_LARGE;
    const size_t n = (size_t)dims[0] * dims[1] * dims[2];
    if (n >= 0xffffffffull) return FC_LBM_ERR_TOO_LARGE;  // labels are 32-bit cell indices
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch sc(s);
    const float* d_pos = positions;
    const uint32_t* d_idx = indices;
    uint8_t* d_solid = solid;
    float* d_sdf = signed_distance;
    const size_t ni = index_count - index_count % 3;
    if (memory == FC_MEMORY_HOST) {
        if (ni > 0) {
            float* p = nullptr;
            uint32_t* q = nullptr;
            VX_TRY(sc.get(&p, 12 * vertex_count));
            VX_TRY(sc.get(&q, 4 * ni));
            VX_TRY(cudaMemcpyAsync(p, positions, 12 * vertex_count, cudaMemcpyHostToDevice, s));
            VX_TRY(cudaMemcpyAsync(q, indices, 4 * ni, cudaMemcpyHostToDevice, s));
            d_pos = p;
            d_idx = q;
        }
        VX_TRY(sc.get(&d_solid, n));
        VX_TRY(sc.get(&d_sdf, 4 * n));
    }
    VX_RC(voxelize_on_device(d_pos, vertex_count, d_idx, ni, dims, cell_size, origin, d_solid, d_sdf, s, sc));
    if (memory == FC_MEMORY_HOST) {
        VX_TRY(cudaMemcpyAsync(solid, d_solid, n, cudaMemcpyDeviceToHost, s));
        VX_TRY(cudaMemcpyAsync(signed_distance, d_sdf, 4 * n, cudaMemcpyDeviceToHost, s));
        VX_RC(wait_on(s));
    }
    return FC_LBM_OK;
}

}  // extern "C"
