/*
 * ORACLE — test infrastructure only; the product never links or calls it.
 *
 * A plain-C restatement of FlowCraft's mesh voxelizer
 * (FlowCraft/Voxelizer.cpp:136-485), single-threaded, built with
 * -ffp-contract=off so every float operation rounds as in the reference:
 *
 *   1. grid from the mesh bounds, padding and target resolution
 *      (Voxelizer.cpp:146-166), or a grid given explicitly;
 *   2. rasterization: for every triangle in index order and every cell of its
 *      conservatively grown bounding box, the closest point on the triangle
 *      (Ericson's Voronoi-region method, Voxelizer.cpp:89-129), the signed
 *      distance with the reference's tie-breaking between near-equal
 *      distances, and solid = 1 within sqrt(3)/2 cells (Voxelizer.cpp:206-293);
 *   3. flood fill: fluid cells not 6-connected to cell (0,0,0) become solid
 *      (the reference finds the same components with slab-parallel flood fills
 *      stitched by union-find, Voxelizer.cpp:295-454; a single breadth-first
 *      fill from the seed gives the identical classification);
 *   4. sign reconciliation (Voxelizer.cpp:456-481).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    float x, y, z;
} v3;

static v3 vsub(v3 a, v3 b) { return (v3){a.x - b.x, a.y - b.y, a.z - b.z}; }
static v3 vadd(v3 a, v3 b) { return (v3){a.x + b.x, a.y + b.y, a.z + b.z}; }
static v3 vmul(v3 a, float s) { return (v3){a.x * s, a.y * s, a.z * s}; }
static float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 vcross(v3 a, v3 b) { return (v3){a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
static float vlen(v3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
static float fmin3(float a, float b, float c) {
    float m = a;
    if (b < m) m = b;
    if (c < m) m = c;
    return m;
}
static float fmax3(float a, float b, float c) {
    float m = a;
    if (m < b) m = b;
    if (m < c) m = c;
    return m;
}

/* Closest point on triangle (a, b, c) to p (Voxelizer.cpp:89-129). */
static v3 closest_on_triangle(v3 p, v3 a, v3 b, v3 c) {
    v3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a);
    float d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) return a;
    v3 bp = vsub(p, b);
    float d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) return b;
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float v = d1 / (d1 - d3);
        return vadd(a, vmul(ab, v));
    }
    v3 cp = vsub(p, c);
    float d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) return c;
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        float w = d2 / (d2 - d6);
        return vadd(a, vmul(ac, w));
    }
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return vadd(b, vmul(vsub(c, b), w));
    }
    float denom = 1.0f / (va + vb + vc);
    float v = vb * denom, w = vc * denom;
    return vadd(vadd(a, vmul(ab, v)), vmul(ac, w));
}

/* Grid of Voxelizer::Voxelize for a mesh (Voxelizer.cpp:146-166): grid x is
 * world y (the flow axis), grid y is world x. Returns 0, or -1 for an empty
 * mesh. */
int voxo_grid_for_mesh(const float* pos, size_t nv, int target_res, float padx, float pady, float padz, int* dims,
                       float* cell, float* origin) {
    if (nv == 0) return -1;
    v3 mn = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
    v3 mx = {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
    for (size_t i = 0; i < nv; ++i) {
        float x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        if (x < mn.x) mn.x = x;
        if (y < mn.y) mn.y = y;
        if (z < mn.z) mn.z = z;
        if (mx.x < x) mx.x = x;
        if (mx.y < y) mx.y = y;
        if (mx.z < z) mx.z = z;
    }
    v3 size = vsub(mx, mn);
    v3 pad = {size.x * padx, size.y * pady, size.z * padz};
    v3 dmin = vsub(mn, pad), dmax = vadd(mx, pad);
    v3 dsize = vsub(dmax, dmin);
    float longest = fmax3(dsize.x, dsize.y, dsize.z);
    int res = target_res > 4 ? target_res : 4;
    float cs = longest / (float)res;
    if (cs < 1e-6f) cs = 1e-6f;
    int nx = (int)ceilf(dsize.y / cs), ny = (int)ceilf(dsize.x / cs), nz = (int)ceilf(dsize.z / cs);
    dims[0] = nx > 1 ? nx : 1;
    dims[1] = ny > 1 ? ny : 1;
    dims[2] = nz > 1 ? nz : 1;
    *cell = cs;
    origin[0] = dmin.x;
    origin[1] = dmin.y;
    origin[2] = dmin.z;
    return 0;
}

/* Voxelizes the mesh onto the given grid; solid / sdf hold nx*ny*nz entries. */
int voxo_voxelize(const float* pos, size_t nv, const uint32_t* idx, size_t ni, const int* dims, float cs,
                  const float* origin, uint8_t* solid, float* sdf) {
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    const size_t n = (size_t)nx * ny * nz;
    const v3 org = {origin[0], origin[1], origin[2]};
    float* best_proj = (float*)malloc(sizeof(float) * n);
    uint8_t* reached = (uint8_t*)calloc(n, 1);
    size_t* queue = (size_t*)malloc(sizeof(size_t) * (n ? n : 1));
    if (!best_proj || !reached || !queue) {
        free(best_proj);
        free(reached);
        free(queue);
        return -1;
    }
    memset(solid, 0, n);
    for (size_t i = 0; i < n; ++i) {
        sdf[i] = INFINITY;
        best_proj[i] = -1.0f;
    }
    const float cr = cs * 0.8660254f;
    const float tie = cs * 1e-3f;
    (void)nv;
    for (size_t t = 0; t + 2 < ni; t += 3) {
        const float* p0 = pos + 3 * (size_t)idx[t];
        const float* p1 = pos + 3 * (size_t)idx[t + 1];
        const float* p2 = pos + 3 * (size_t)idx[t + 2];
        v3 a = {p0[0], p0[1], p0[2]}, b = {p1[0], p1[1], p1[2]}, c = {p2[0], p2[1], p2[2]};
        v3 rn = vcross(vsub(b, a), vsub(c, a));
        float nl = vlen(rn);
        if (nl <= 1e-12f) continue;
        v3 un = vmul(rn, 1.0f / nl);
        v3 tmin = {fmin3(a.x, b.x, c.x), fmin3(a.y, b.y, c.y), fmin3(a.z, b.z, c.z)};
        v3 tmax = {fmax3(a.x, b.x, c.x), fmax3(a.y, b.y, c.y), fmax3(a.z, b.z, c.z)};
        int minX = (int)floorf((tmin.y - cr - org.y) / cs);
        int minY = (int)floorf((tmin.x - cr - org.x) / cs);
        int minZ = (int)floorf((tmin.z - cr - org.z) / cs);
        int maxX = (int)ceilf((tmax.y + cr - org.y) / cs);
        int maxY = (int)ceilf((tmax.x + cr - org.x) / cs);
        int maxZ = (int)ceilf((tmax.z + cr - org.z) / cs);
        if (minX < 0) minX = 0;
        if (minY < 0) minY = 0;
        if (minZ < 0) minZ = 0;
        if (maxX > nx - 1) maxX = nx - 1;
        if (maxY > ny - 1) maxY = ny - 1;
        if (maxZ > nz - 1) maxZ = nz - 1;
        for (int z = minZ; z <= maxZ; ++z)
            for (int y = minY; y <= maxY; ++y)
                for (int x = minX; x <= maxX; ++x) {
                    size_t i = ((size_t)z * ny + y) * nx + x;
                    /* CellCenter: world x from grid y, world y from grid x (VoxelGrid.h:43-56) */
                    v3 ctr = vadd(org, (v3){((float)y + 0.5f) * cs, ((float)x + 0.5f) * cs, ((float)z + 0.5f) * cs});
                    v3 cl = closest_on_triangle(ctr, a, b, c);
                    v3 diff = vsub(ctr, cl);
                    float dist = vlen(diff);
                    float nd = vdot(diff, un);
                    float and_ = fabsf(nd);
                    float sd = nd < 0.0f ? -dist : dist;
                    float bd = fabsf(sdf[i]);
                    if (dist + tie < bd) {
                        sdf[i] = sd;
                        best_proj[i] = and_;
                    } else if (dist <= bd + tie) {
                        if (and_ > best_proj[i]) {
                            float md = dist < bd ? dist : bd;
                            sdf[i] = nd < 0.0f ? -md : md;
                            best_proj[i] = and_;
                        } else if (dist < bd) {
                            sdf[i] = sdf[i] < 0.0f ? -dist : dist;
                        }
                    }
                    if (dist <= cr) solid[i] = 1;
                }
    }
    /* flood fill from the seed cell (0,0,0) over 6-connected fluid cells */
    size_t head = 0, tail = 0;
    if (n > 0 && !solid[0]) {
        reached[0] = 1;
        queue[tail++] = 0;
    }
    const size_t layer = (size_t)nx * ny;
    while (head < tail) {
        size_t cur = queue[head++];
        int cz = (int)(cur / layer);
        size_t rem = cur - (size_t)cz * layer;
        int cy = (int)(rem / nx), cx = (int)(rem - (size_t)cy * nx);
        const int nb[6][3] = {{cx - 1, cy, cz}, {cx + 1, cy, cz}, {cx, cy - 1, cz},
                              {cx, cy + 1, cz}, {cx, cy, cz - 1}, {cx, cy, cz + 1}};
        for (int k = 0; k < 6; ++k) {
            int x = nb[k][0], y = nb[k][1], z = nb[k][2];
            if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) continue;
            size_t j = ((size_t)z * ny + y) * nx + x;
            if (solid[j] || reached[j]) continue;
            reached[j] = 1;
            queue[tail++] = j;
        }
    }
    for (size_t i = 0; i < n; ++i)
        if (!solid[i] && !reached[i]) solid[i] = 1;
    /* sign reconciliation */
    for (size_t i = 0; i < n; ++i) {
        float d = fabsf(sdf[i]);
        if (!solid[i])
            sdf[i] = d;
        else if (d > cr)
            sdf[i] = -d;
    }
    free(best_proj);
    free(reached);
    free(queue);
    return 0;
}
