// Host-side packing of the learned closure's weights and the wall-distance
// input (closure.cuh holds the device inference).
#include <cuda_runtime.h>

#include <cstring>

#include "lbm_internal.h"

namespace fc {

namespace {

// float -> bfloat16 bits, round to nearest even (NaN stays NaN).
uint16_t to_bf16(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0u;
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

uint32_t pair_bits(float lo, float hi) { return (uint32_t)to_bf16(lo) | ((uint32_t)to_bf16(hi) << 16); }

uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

}  // namespace

// Fragment order of the warp MMA (closure.cuh): lane L = 4g + t holds, for a
// B fragment of K x 8 (col-major), rows 2t, 2t+1 (and 2t+8, 2t+9 for K = 16)
// of column g. The first layer's K = 8 rows are inputs 0-4, the constant 1
// (row 5, carrying b1) and two zero rows; the second layer's bias is the
// K = 8 fragment whose row 0 is b2 (multiplied by a constant-1 column).
void pack_closure(const float* w1, const float* b1, const float* w2, const float* b2, const float* w3, float b3,
                  float out_scale, uint4* out) {
    constexpr int H = kClosureHidden;
    auto W1 = [&](int k, int j) { return k < kClosureIn ? w1[k * H + j] : (k == kClosureIn ? b1[j] : 0.0f); };
    auto B2 = [&](int k, int j) { return k == 0 ? b2[j] : 0.0f; };
    auto W2 = [&](int k, int j) { return w2[k * H + j]; };
    auto W3 = [&](int k, int j) { return j == 0 ? w3[k] * out_scale : 0.0f; };  // N padded to 8
    for (int lane = 0; lane < 32; ++lane) {
        const int g = lane >> 2, t = lane & 3;
        uint32_t gw[kClosureGroups][4] = {};
        for (int n = 0; n < 4; ++n) {
            gw[0][n] = pair_bits(W1(2 * t, 8 * n + g), W1(2 * t + 1, 8 * n + g));
            gw[1][n] = pair_bits(B2(2 * t, 8 * n + g), B2(2 * t + 1, 8 * n + g));
        }
        for (int n = 0; n < 4; ++n)
            for (int s = 0; s < 2; ++s) {
                const int col = 8 * n + g, k0 = 16 * s + 2 * t;
                gw[2 + n][2 * s] = pair_bits(W2(k0, col), W2(k0 + 1, col));
                gw[2 + n][2 * s + 1] = pair_bits(W2(k0 + 8, col), W2(k0 + 9, col));
            }
        for (int s = 0; s < 2; ++s) {
            const int k0 = 16 * s + 2 * t;
            gw[6][2 * s] = pair_bits(W3(k0, g), W3(k0 + 1, g));
            gw[6][2 * s + 1] = pair_bits(W3(k0 + 8, g), W3(k0 + 9, g));
        }
        gw[7][0] = fbits(b3 * out_scale);
        for (int grp = 0; grp < kClosureGroups; ++grp)
            out[grp * 32 + lane] = make_uint4(gw[grp][0], gw[grp][1], gw[grp][2], gw[grp][3]);
    }
}

namespace {

__global__ void k_wall_init(const uint8_t* __restrict__ solid, uint8_t* __restrict__ d, size_t n) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        d[c] = solid[c] ? 0 : (uint8_t)kWallFar;
}

// One relaxation sweep of the 3x3x3 chamfer distance: d(c) = min over the 26
// neighbours of d(n) + 16, 23 or 28 (1, ~sqrt2, ~sqrt3 cells in 1/16 steps).
__global__ void k_wall_relax(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, Geom g) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < g.n; c += (size_t)gridDim.x * blockDim.x) {
        const int v = in[c];
        if (v == 0) {
            out[c] = 0;
            continue;
        }
        const int z = (int)(c / (size_t)g.nxy);
        const size_t rem = c - (size_t)z * g.nxy;
        const int y = (int)(rem / g.nx);
        const int x = (int)(rem - (size_t)y * g.nx);
        int best = v;
        for (int dz = -1; dz <= 1; ++dz) {
            const int zz = z + dz;
            if (zz < 0 || zz >= g.nz) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int yy = y + dy;
                if (yy < 0 || yy >= g.ny) continue;
                const size_t rowc = ((size_t)zz * g.ny + yy) * g.nx;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int xx = x + dx;
                    if (xx < 0 || xx >= g.nx) continue;
                    const int m = (dx != 0) + (dy != 0) + (dz != 0);
                    if (m == 0) continue;
                    const int cand = (int)in[rowc + xx] + (m == 1 ? 16 : (m == 2 ? 23 : 28));
                    best = cand < best ? cand : best;
                }
            }
        }
        out[c] = (uint8_t)(best < kWallFar ? best : kWallFar);
    }
}

}  // namespace

cudaError_t launch_wall_distance(const uint8_t* solid, const Geom& g, uint8_t* out, uint8_t* tmp, cudaStream_t s) {
    const int blocks = (int)((g.n + 255) / 256 < 148 * 32 ? (g.n + 255) / 256 : 148 * 32);
    // 16 Jacobi sweeps (an even count leaves the result in `out`)
    k_wall_init<<<blocks, 256, 0, s>>>(solid, out, g.n);
    cudaError_t e = cudaGetLastError();
    for (int it = 0; it < 16 && e == cudaSuccess; it += 2) {
        k_wall_relax<<<blocks, 256, 0, s>>>(out, tmp, g);
        k_wall_relax<<<blocks, 256, 0, s>>>(tmp, out, g);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace fc
