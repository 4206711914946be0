// Host-side packing of the learned closure's weights, the wall-distance
// input, and the extraction of training samples from a finer lattice
// (closure.cuh holds the device inference).
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <thread>

#include <cub/device/device_scan.cuh>

#include "fc_lbm.h"
#include "lattice.cuh"
#include "lbm_internal.h"
#include "storage.cuh"

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

// The tensor-core MLP's operands B (N x K, K-major): element (n, k) of a
// block sits at (n / 8) * SBO + (k / 8) * 128 + (n % 8) * 16 + (k % 8) * 2
// bytes, SBO = K * 16 bytes (one 8-row group of all K core matrices).
//   W1  bytes    0-1023: n = hidden unit (32), k = input 0-4, 5 the constant 1 (b1), rest 0 (K = 16)
//   W2  bytes 1024-3071: n = hidden unit of layer 2 (32), k = layer-1 unit (K = 32)
//   B2  bytes 3072-4095: n = hidden unit of layer 2, k = 0 carries b2, rest 0 (K = 16)
//   W3  bytes 4096-5119: n = 0 carries w3 * out_scale, rows 1-15 zero (N = 16, K = 32)
void pack_closure_tc(const float* w1, const float* b1, const float* w2, const float* b2, const float* w3,
                     float out_scale, uint8_t* out) {
    constexpr int H = kClosureHidden;
    std::memset(out, 0, kTcWeightBytes);
    auto put = [&](int base, int kdim, int n, int k, float v) {
        const uint16_t b = to_bf16(v);
        const int off = base + (n / 8) * (kdim * 16) + (k / 8) * 128 + (n % 8) * 16 + (k % 8) * 2;
        std::memcpy(out + off, &b, 2);
    };
    for (int n = 0; n < H; ++n) {
        for (int k = 0; k < kClosureIn; ++k) put(0, 16, n, k, w1[k * H + n]);
        put(0, 16, n, kClosureIn, b1[n]);
        for (int k = 0; k < H; ++k) put(1024, 32, n, k, w2[k * H + n]);
        put(3072, 16, n, 0, b2[n]);
    }
    for (int k = 0; k < H; ++k) put(4096, 32, 0, k, w3[k] * out_scale);
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

// ---- training samples: a 2x box filter of a fine lattice ----
//
// Coarse cell X covers the fine cells 2X + {0,1}^3. From the fine
// populations it gets the box-filtered density, momentum, momentum flux and
// viscous stress:
//   rho = <rho_f>, u = <rho_f u_f> / rho,
//   tau_sgs = <rho_f u_f u_f> - rho u u          (the resolved sub-grid stress),
//   V = <V_f>                                    (the fine cells' viscous stress).
// V_f is the whole viscous stress a fine cell carries, molecular and its own
// Smagorinsky eddy viscosity: its stored populations are post-collision, so
// their non-equilibrium stress is Pi* = (1 - 1/tau_f') Pi_neq with the cell's
// tau_f' = (tau_f + sqrt(tau_f^2 + k |Pi_neq| / rho)) / 2, k = 18 sqrt2 Cs^2
// (the step's Smagorinsky). Eliminating Pi_neq gives
//   (tau_f' - tau_f) (1 - tau_f') = k |Pi*| / (4 rho),
// a quadratic whose root next to tau_f is tau_f', and then
//   V_f = 2 rho c_s^2 (tau_f' - 1/2) S_f = (tau_f' - 1/2) / (1 - tau_f') Pi*.
// The filtered flow's momentum balance carries the stress V - tau_sgs, so
// with S the strain of the filtered velocity by central differences over
// the coarse neighbours, the coarse cell's total viscosity is the
// least-squares fit of (V - tau_sgs)_dev = 2 rho nu S_dev, and the target
// eddy viscosity is that minus the coarse molecular viscosity:
//   nu* = max(0, (V - tau_sgs)_dev : S_dev / (2 rho S_dev : S_dev) - (tau_c - 1/2) / 3).
// (Viscosity and strain are in each lattice's own units; their product, a
// stress, is the same number on both.)
// The inputs are those a coarse cell relaxing with tau_c + 3 nu* sees: the
// regularized scheme's non-equilibrium stress is Pi = -2 rho c_s^2 tau_eff S
// (Chapman-Enskog), so the samples carry the invariants of
// Pi = -(2/3) rho (tau_c + 3 nu*) S, the coarse wall distance and the filter
// width. Velocities keep their lattice value under the 2x coarsening
// (dx and dt both double), strains and viscosities are in coarse units.
namespace {

constexpr int kCoarseFields = 16;  // rho, u (3), tau_sgs (6), V (6)
constexpr int kWaitTimeoutMs = 600000;

// Waits for `s` by polling an event with a growing sleep, so a stuck device
// surfaces as a timeout status instead of a hang.
cudaError_t wait_bounded(cudaStream_t s, bool* timed_out) {
    *timed_out = false;
    cudaEvent_t ev;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(ev, s);
    const auto t0 = std::chrono::steady_clock::now();
    int sleep_us = 20;
    while (e == cudaSuccess) {
        const cudaError_t q = cudaEventQuery(ev);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) {
            e = q;
            break;
        }
        if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(kWaitTimeoutMs)) {
            *timed_out = true;
            break;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(sleep_us));
        if (sleep_us < 2000) sleep_us *= 2;
    }
    cudaEventDestroy(ev);
    return e;
}

template <int Q, class S>
__global__ void k_coarse_fields(const typename S::T* __restrict__ f, const uint8_t* __restrict__ solid, Geom fg,
                                Geom cg, float tau_f, float cs_f, uint8_t* __restrict__ csolid,
                                float* __restrict__ cf) {
    using L = Lattice<Q>;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < cg.n; c += (size_t)gridDim.x * blockDim.x) {
        const int zc = (int)(c / (size_t)cg.nxy);
        const size_t rem = c - (size_t)zc * cg.nxy;
        const int yc = (int)(rem / cg.nx);
        const int xc = (int)(rem - (size_t)yc * cg.nx);
        bool any_solid = false;
        double rs = 0, mx = 0, my = 0, mz = 0, uu[6] = {0, 0, 0, 0, 0, 0}, vs[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 8; ++k) {
            const size_t fc = ((size_t)(2 * zc + (k >> 2)) * fg.ny + (2 * yc + ((k >> 1) & 1))) * fg.nx +
                              (2 * xc + (k & 1));
            if (solid[fc]) {
                any_solid = true;
                continue;
            }
            float rho = 0.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
            double m2[6] = {0, 0, 0, 0, 0, 0};  // sum f e_a e_b: xx yy zz xy xz yz
            static_for<0, Q>([&](auto I) {
                constexpr int i = decltype(I)::value;
                constexpr int X = L::ex(i), Y = L::ey(i), Z = L::ez(i);
                const float v = load_pop_c<Q, S, i>(f, fg.n, fc);
                rho += v;
                if constexpr (X != 0) jx += (float)X * v;
                if constexpr (Y != 0) jy += (float)Y * v;
                if constexpr (Z != 0) jz += (float)Z * v;
                m2[0] += (double)(X * X) * v, m2[1] += (double)(Y * Y) * v, m2[2] += (double)(Z * Z) * v;
                m2[3] += (double)(X * Y) * v, m2[4] += (double)(X * Z) * v, m2[5] += (double)(Y * Z) * v;
            });
            const double ux = jx / rho, uy = jy / rho, uz = jz / rho;
            // the cell's post-collision non-equilibrium stress, its relaxation
            // time and its viscous stress (see above)
            const double pr = (double)rho / 3.0;
            const double pst[6] = {m2[0] - pr - rho * ux * ux, m2[1] - pr - rho * uy * uy, m2[2] - pr - rho * uz * uz,
                                   m2[3] - rho * ux * uy, m2[4] - rho * ux * uz, m2[5] - rho * uy * uz};
            const double pmag = sqrt(pst[0] * pst[0] + pst[1] * pst[1] + pst[2] * pst[2] +
                                     2.0 * (pst[3] * pst[3] + pst[4] * pst[4] + pst[5] * pst[5]));
            const double kq = 18.0 * 1.41421356 * (double)cs_f * (double)cs_f;
            const double disc = (1.0 - tau_f) * (1.0 - tau_f) - kq * pmag / (rho > 1e-6f ? (double)rho : 1e-6);
            const double te = 0.5 * ((1.0 + tau_f) - sqrt(disc > 0.0 ? disc : 0.0));
            const double vf = (te - 0.5) / (1.0 - te);
            for (int k = 0; k < 6; ++k) vs[k] += vf * pst[k];
            rs += rho;
            mx += jx, my += jy, mz += jz;
            uu[0] += rho * ux * ux, uu[1] += rho * uy * uy, uu[2] += rho * uz * uz;
            uu[3] += rho * ux * uy, uu[4] += rho * ux * uz, uu[5] += rho * uy * uz;
        }
        csolid[c] = any_solid ? 1 : 0;
        float* o = cf + c * kCoarseFields;
        if (any_solid) {
            for (int k = 0; k < kCoarseFields; ++k) o[k] = 0.0f;
            continue;
        }
        const double rho = rs / 8.0, ux = mx / rs, uy = my / rs, uz = mz / rs;
        o[0] = (float)rho, o[1] = (float)ux, o[2] = (float)uy, o[3] = (float)uz;
        o[4] = (float)(uu[0] / 8.0 - rho * ux * ux), o[5] = (float)(uu[1] / 8.0 - rho * uy * uy);
        o[6] = (float)(uu[2] / 8.0 - rho * uz * uz), o[7] = (float)(uu[3] / 8.0 - rho * ux * uy);
        o[8] = (float)(uu[4] / 8.0 - rho * ux * uz), o[9] = (float)(uu[5] / 8.0 - rho * uy * uz);
        for (int k = 0; k < 6; ++k) o[10 + k] = (float)(vs[k] / 8.0);
    }
}

struct SampleOut {
    bool valid;
    float row[6];
};

__device__ SampleOut coarse_sample(const uint8_t* __restrict__ csolid, const float* __restrict__ cf,
                                   const uint8_t* __restrict__ cwall, const Geom& cg, size_t c, float tau_c,
                                   float filter_width) {
    SampleOut r{};
    const int z = (int)(c / (size_t)cg.nxy);
    const size_t rem = c - (size_t)z * cg.nxy;
    const int y = (int)(rem / cg.nx);
    const int x = (int)(rem - (size_t)y * cg.nx);
    // off the inlet/outlet planes and the domain faces, with fluid neighbours
    if (x < 2 || x > cg.nx - 3 || y < 1 || y > cg.ny - 2 || z < 1 || z > cg.nz - 2 || csolid[c]) return r;
    const size_t nb[6] = {c - 1, c + 1, c - (size_t)cg.nx, c + (size_t)cg.nx, c - (size_t)cg.nxy, c + (size_t)cg.nxy};
    for (int k = 0; k < 6; ++k)
        if (csolid[nb[k]]) return r;
    double g[3][3];  // g[a][b] = d u_b / d x_a
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) g[a][b] = 0.5 * ((double)cf[nb[2 * a + 1] * kCoarseFields + 1 + b] -
                                                       (double)cf[nb[2 * a] * kCoarseFields + 1 + b]);
    double sm[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) sm[a][b] = 0.5 * (g[a][b] + g[b][a]);
    const double tr = (sm[0][0] + sm[1][1] + sm[2][2]) / 3.0;
    double sd[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) sd[a][b] = sm[a][b] - (a == b ? tr : 0.0);
    const float* o = cf + c * kCoarseFields;
    const double rho = o[0];
    // the stress the coarse cell's viscosity must carry: V - tau_sgs
    const double t6[6] = {o[10] - o[4], o[11] - o[5], o[12] - o[6], o[13] - o[7], o[14] - o[8], o[15] - o[9]};
    const double ttr = (t6[0] + t6[1] + t6[2]) / 3.0;
    const double td[3][3] = {{t6[0] - ttr, t6[3], t6[4]}, {t6[3], t6[1] - ttr, t6[5]}, {t6[4], t6[5], t6[2] - ttr}};
    double tds = 0.0, sds = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            tds += td[a][b] * sd[a][b];
            sds += sd[a][b] * sd[a][b];
        }
    if (!(sds > 1e-18) || !(rho > 0.0)) return r;
    double nu = tds / (2.0 * rho * sds) - ((double)tau_c - 0.5) / 3.0;
    nu = nu > 0.0 ? nu : 0.0;
    // the stress a coarse cell relaxing with tau_c + 3 nu carries
    const double k = -(2.0 / 3.0) * rho * ((double)tau_c + 3.0 * nu);
    double p[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) p[a][b] = k * sm[a][b];
    double pp = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) pp += p[a][b] * p[a][b];
    const double mag = sqrt(pp);
    const double ri = mag > 0.0 ? 1.0 / mag : 0.0;
    const double det = p[0][0] * (p[1][1] * p[2][2] - p[1][2] * p[2][1]) -
                       p[0][1] * (p[1][0] * p[2][2] - p[1][2] * p[2][0]) +
                       p[0][2] * (p[1][0] * p[2][1] - p[1][1] * p[2][0]);
    r.row[0] = (float)log2(mag / rho + 1e-12);
    r.row[1] = (float)((p[0][0] + p[1][1] + p[2][2]) * ri);
    r.row[2] = (float)(det * ri * ri * ri);
    r.row[3] = (float)cwall[c] * 0.0625f;
    r.row[4] = filter_width;
    r.row[5] = (float)nu;
    r.valid = true;
    return r;
}

__global__ void k_sample_flags(const uint8_t* __restrict__ csolid, const float* __restrict__ cf,
                               const uint8_t* __restrict__ cwall, Geom cg, float tau_c, float filter_width,
                               uint32_t* __restrict__ flags) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < cg.n; c += (size_t)gridDim.x * blockDim.x)
        flags[c] = coarse_sample(csolid, cf, cwall, cg, c, tau_c, filter_width).valid ? 1u : 0u;
}

__global__ void k_sample_write(const uint8_t* __restrict__ csolid, const float* __restrict__ cf,
                               const uint8_t* __restrict__ cwall, Geom cg, float tau_c, float filter_width,
                               const uint32_t* __restrict__ pos, float* __restrict__ out) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < cg.n; c += (size_t)gridDim.x * blockDim.x) {
        const SampleOut so = coarse_sample(csolid, cf, cwall, cg, c, tau_c, filter_width);
        if (!so.valid) continue;
        float* row = out + (size_t)pos[c] * 6;
        for (int k = 0; k < 6; ++k) row[k] = so.row[k];
    }
}

template <int Q, class S>
cudaError_t coarse_fields_t(const void* f, const uint8_t* solid, const Geom& fg, const Geom& cg, float tau_f,
                            float cs_f, uint8_t* csolid, float* cf, cudaStream_t s) {
    const int blocks = (int)((cg.n + 255) / 256 < 148 * 16 ? (cg.n + 255) / 256 : 148 * 16);
    k_coarse_fields<Q, S><<<blocks, 256, 0, s>>>((const typename S::T*)f, solid, fg, cg, tau_f, cs_f, csolid, cf);
    return cudaGetLastError();
}

cudaError_t coarse_fields(int q, int storage, const void* f, const uint8_t* solid, const Geom& fg, const Geom& cg,
                          float tau_f, float cs_f, uint8_t* csolid, float* cf, cudaStream_t s) {
    if (q == 19) {
        if (storage == 0) return coarse_fields_t<19, StoreF32>(f, solid, fg, cg, tau_f, cs_f, csolid, cf, s);
        if (storage == 1) return coarse_fields_t<19, StoreF16>(f, solid, fg, cg, tau_f, cs_f, csolid, cf, s);
        if (storage == 2) return coarse_fields_t<19, StoreBF16>(f, solid, fg, cg, tau_f, cs_f, csolid, cf, s);
    } else if (q == 15) {
        if (storage == 0) return coarse_fields_t<15, StoreF32>(f, solid, fg, cg, tau_f, cs_f, csolid, cf, s);
        if (storage == 1) return coarse_fields_t<15, StoreF16>(f, solid, fg, cg, tau_f, cs_f, csolid, cf, s);
        if (storage == 2) return coarse_fields_t<15, StoreBF16>(f, solid, fg, cg, tau_f, cs_f, csolid, cf, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace

int closure_samples(int q, int storage, const void* f, const uint8_t* solid, const Geom& fg, float tau_f, float cs_f,
                    float tau_c, float filter_width, float* out, int64_t capacity, int64_t* count, cudaStream_t s) {
    Geom cg{};
    cg.nx = fg.nx / 2, cg.ny = fg.ny / 2, cg.nz = fg.nz / 2;
    cg.wpr = (cg.nx + 31) / 32;
    cg.nxy = (long long)cg.nx * cg.ny;
    cg.n = (size_t)cg.nx * cg.ny * cg.nz;
    *count = 0;
    if (cg.nx < 5 || cg.ny < 3 || cg.nz < 3) return FC_LBM_ERR_INVALID_ARG;
    uint8_t *csolid = nullptr, *cwall = nullptr, *tmp = nullptr;
    float* cf = nullptr;
    uint32_t *flags = nullptr, *pos = nullptr;
    void* scan_tmp = nullptr;
    size_t scan_bytes = 0;
    int rc = FC_LBM_OK;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == FC_LBM_OK) rc = e == cudaErrorMemoryAllocation ? FC_LBM_ERR_OUT_OF_MEMORY
                                                                                     : FC_LBM_ERR_CUDA;
        return rc == FC_LBM_OK;
    };
    const int blocks = (int)((cg.n + 255) / 256 < 148 * 16 ? (cg.n + 255) / 256 : 148 * 16);
    uint32_t total = 0;
    bool timed_out = false;
    if (ok(cudaMallocAsync(&csolid, cg.n, s)) && ok(cudaMallocAsync(&cwall, cg.n, s)) &&
        ok(cudaMallocAsync(&tmp, cg.n, s)) && ok(cudaMallocAsync(&cf, cg.n * kCoarseFields * sizeof(float), s)) &&
        ok(cudaMallocAsync(&flags, cg.n * sizeof(uint32_t), s)) &&
        ok(cudaMallocAsync(&pos, (cg.n + 1) * sizeof(uint32_t), s)) &&
        ok(coarse_fields(q, storage, f, solid, fg, cg, tau_f, cs_f, csolid, cf, s)) &&
        ok(launch_wall_distance(csolid, cg, cwall, tmp, s))) {
        k_sample_flags<<<blocks, 256, 0, s>>>(csolid, cf, cwall, cg, tau_c, filter_width, flags);
        if (ok(cudaGetLastError()) && ok(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, flags, pos, (int64_t)cg.n, s)) &&
            ok(cudaMallocAsync(&scan_tmp, scan_bytes, s)) &&
            ok(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, flags, pos, (int64_t)cg.n, s))) {
            uint32_t last[2] = {0, 0};
            if (ok(cudaMemcpyAsync(&last[0], pos + cg.n - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s)) &&
                ok(cudaMemcpyAsync(&last[1], flags + cg.n - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s)) &&
                ok(wait_bounded(s, &timed_out))) {
                if (timed_out) rc = FC_LBM_ERR_TIMEOUT;
                total = last[0] + last[1];
                *count = total;
                if (rc != FC_LBM_OK) {
                } else if ((int64_t)total > capacity) {
                    rc = FC_LBM_ERR_TOO_LARGE;
                } else if (out && total > 0) {
                    k_sample_write<<<blocks, 256, 0, s>>>(csolid, cf, cwall, cg, tau_c, filter_width, pos, out);
                    ok(cudaGetLastError());
                }
            }
        }
    }
    for (void* p : {(void*)csolid, (void*)cwall, (void*)tmp, (void*)cf, (void*)flags, (void*)pos, scan_tmp})
        if (p) cudaFreeAsync(p, s);
    return rc;
}

}  // namespace fc
