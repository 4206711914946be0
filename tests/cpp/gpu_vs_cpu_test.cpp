// The reference's headless GPU-vs-CPU consistency test
// (tests/gpu_vs_cpu_test.cpp:21-80) restated against this library: the
// CUDA solver through fc::LbmSolver (include/fc_lbm_solver.hpp) versus the
// CPU oracle (oracle/lbm_oracle.c, the restatement pinned to LbmReference)
// on the same 48x24x24 sphere, tau 0.6, U 0.05, Cs 0.12, mid-speed seed,
// 60 steps, both lattices. The reference passes at max|drho| < 0.01,
// max|du| < 0.01, mean|du| < 0.001 (its GPU stores FP16); the FP32 path
// here must be bit-identical, so the test also counts differing floats.
//
// A third check runs fc::Voxelize against the voxelizer oracle.
//
// Exit code: 0 pass, 1 fail, 2 no device (as the reference's test).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <map>
#include <cstdio>
#include <cstring>
#include <vector>

#include "fc_lbm_solver.hpp"

extern "C" {
struct oracle_params {
    float tau, inlet_velocity;
    int32_t reverse_flow, free_slip_y, free_slip_z;
    float smagorinsky_cs;
};
struct oracle_lbm;
oracle_lbm* oracle32_create(int nx, int ny, int nz, int q, const uint8_t* solid, const float* sdf, size_t sdf_count,
                            const oracle_params* p, int seed_mid, int threads);
void oracle32_step(oracle_lbm* o, int n);
void oracle32_readback_field(oracle_lbm* o, float* out);
void oracle32_destroy(oracle_lbm* o);
int voxo_grid_for_mesh(const float* pos, size_t nv, int target_res, float padx, float pady, float padz, int* dims,
                       float* cell, float* origin);
int voxo_voxelize(const float* pos, size_t nv, const uint32_t* idx, size_t ni, const int* dims, float cs,
                  const float* origin, uint8_t* solid, float* sdf);
}

struct Vec3 {
    float x = 0, y = 0, z = 0;
};
// Same field names as FlowCraft's VoxelGrid (FlowCraft/VoxelGrid.h:13-61).
struct VoxelGrid {
    int nx = 0, ny = 0, nz = 0;
    float cellSize = 1.0f;
    Vec3 origin;
    std::vector<uint8_t> solid;
    std::vector<float> signedDistance;
    size_t CellCount() const { return (size_t)nx * ny * nz; }
    size_t Index(int x, int y, int z) const { return ((size_t)z * ny + y) * nx + x; }
};

// Icosahedron subdivided `level` times onto a sphere (outward winding).
static void icosphere(int level, float r, Vec3 c, std::vector<Vec3>& pos, std::vector<uint32_t>& idx) {
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    std::vector<std::array<double, 3>> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                                            {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    auto norm = [](std::array<double, 3> a) {
        const double l = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        return std::array<double, 3>{a[0] / l, a[1] / l, a[2] / l};
    };
    for (auto& p : v) p = norm(p);
    std::vector<std::array<uint32_t, 3>> f = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11},
                                              {1, 5, 9}, {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                                              {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8}, {3, 8, 9},
                                              {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    for (int l = 0; l < level; ++l) {
        std::map<std::pair<uint32_t, uint32_t>, uint32_t> mid;
        auto m = [&](uint32_t a, uint32_t b) {
            auto key = std::make_pair(std::min(a, b), std::max(a, b));
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            v.push_back(norm({v[a][0] + v[b][0], v[a][1] + v[b][1], v[a][2] + v[b][2]}));
            return mid[key] = (uint32_t)(v.size() - 1);
        };
        std::vector<std::array<uint32_t, 3>> nf;
        for (auto& tri : f) {
            const uint32_t ab = m(tri[0], tri[1]), bc = m(tri[1], tri[2]), ca = m(tri[2], tri[0]);
            nf.push_back({tri[0], ab, ca});
            nf.push_back({tri[1], bc, ab});
            nf.push_back({tri[2], ca, bc});
            nf.push_back({ab, bc, ca});
        }
        f = nf;
    }
    pos.clear();
    idx.clear();
    for (auto& p : v) pos.push_back({(float)(p[0] * r + c.x), (float)(p[1] * r + c.y), (float)(p[2] * r + c.z)});
    for (auto& tri : f) idx.insert(idx.end(), tri.begin(), tri.end());
}

// fc::Voxelize (the GPU voxelizer) against the voxelizer oracle on an
// icosphere, at the reference's default padding.
static bool voxelizer_check() {
    std::vector<Vec3> pos;
    std::vector<uint32_t> idx;
    icosphere(3, 10.0f, Vec3{5.0f, 7.0f, -3.0f}, pos, idx);
    fc::VoxelizerParams vp;
    vp.targetResolution = 80;
    VoxelGrid g;
    int status = 0;
    if (!fc::Voxelize(pos, idx, vp, g, &status)) {
        std::printf("voxelizer: fc::Voxelize failed with status %d\n", status);
        return false;
    }
    std::vector<float> flat;
    for (auto& p : pos) flat.insert(flat.end(), {p.x, p.y, p.z});
    int dims[3];
    float cell, origin[3];
    voxo_grid_for_mesh(flat.data(), pos.size(), vp.targetResolution, 0.3f, 1.0f, 0.5f, dims, &cell, origin);
    const size_t n = (size_t)dims[0] * dims[1] * dims[2];
    std::vector<uint8_t> solid(n);
    std::vector<float> sdf(n);
    voxo_voxelize(flat.data(), pos.size(), idx.data(), idx.size(), dims, cell, origin, solid.data(), sdf.data());
    const bool same_grid = g.nx == dims[0] && g.ny == dims[1] && g.nz == dims[2] && g.cellSize == cell &&
                           g.origin.x == origin[0] && g.origin.y == origin[1] && g.origin.z == origin[2];
    const bool ok = same_grid && g.solid == solid &&
                    std::memcmp(g.signedDistance.data(), sdf.data(), n * sizeof(float)) == 0;
    size_t solid_cells = 0;
    for (uint8_t b : solid) solid_cells += b;
    std::printf("voxelizer icosphere L3 (%zu triangles) on %dx%dx%d: %zu solid cells, bit-identical %s\n",
                idx.size() / 3, g.nx, g.ny, g.nz, solid_cells, ok ? "yes" : "no");
    std::printf("  -> %s\n", ok ? "PASS" : "FAIL");
    return ok;
}

int main() {
    for (fc::LatticeModel model : {fc::LatticeModel::D3Q19, fc::LatticeModel::D3Q15}) {
        VoxelGrid grid;
        grid.nx = 48; grid.ny = 24; grid.nz = 24;
        grid.solid.assign(grid.CellCount(), 0);
        grid.signedDistance.assign(grid.CellCount(), 1e30f);
        const float cx = 20, cy = 12, cz = 12, r = 5;
        for (int z = 0; z < grid.nz; ++z)
            for (int y = 0; y < grid.ny; ++y)
                for (int x = 0; x < grid.nx; ++x) {
                    float d = std::sqrt((x + .5f - cx) * (x + .5f - cx) + (y + .5f - cy) * (y + .5f - cy) +
                                        (z + .5f - cz) * (z + .5f - cz)) - r;
                    size_t i = grid.Index(x, y, z);
                    grid.signedDistance[i] = d;
                    grid.solid[i] = d < 0 ? 1 : 0;
                }

        fc::LbmSolver::Params gp; gp.tau = 0.6f; gp.inletVelocity = 0.05f; gp.smagorinskyCs = 0.12f;
        oracle_params cp{gp.tau, gp.inletVelocity, gp.reverseFlow, gp.freeSlipY, gp.freeSlipZ, gp.smagorinskyCs};

        fc::LbmSolver gpu;
        if (!gpu.Init(0, grid, model)) {
            std::printf("GPU Init failed: %s\n", gpu.LastError().c_str());
            return gpu.LastError().find("no CUDA device") != std::string::npos ? 2 : 1;
        }
        gpu.Reset(gp, true);
        const int q = model == fc::LatticeModel::D3Q19 ? 19 : 15;
        oracle_lbm* cpu = oracle32_create(grid.nx, grid.ny, grid.nz, q, grid.solid.data(),
                                          grid.signedDistance.data(), grid.CellCount(), &cp, 1, 0);

        const int kSteps = 60;
        gpu.Step(nullptr, kSteps);
        oracle32_step(cpu, kSteps);

        std::vector<float> g = gpu.ReadbackField(), c(grid.CellCount() * 4);
        oracle32_readback_field(cpu, c.data());
        double maxRho = 0, maxU = 0, sumU = 0; size_t n = 0, differing = 0; bool nan = false;
        for (size_t i = 0; i < grid.CellCount(); ++i) {
            for (int k = 0; k < 4; ++k) differing += std::memcmp(&g[i * 4 + k], &c[i * 4 + k], 4) != 0;
            if (grid.solid[i]) continue;
            for (int k = 0; k < 4; ++k) if (!std::isfinite(g[i * 4 + k])) nan = true;
            maxRho = std::max<double>(maxRho, std::fabs(g[i * 4] - c[i * 4]));
            for (int k = 1; k < 4; ++k) {
                double e = std::fabs(g[i * 4 + k] - c[i * 4 + k]);
                maxU = std::max(maxU, e); sumU += e; ++n;
            }
        }
        fc::LbmSolver::Stats st = gpu.ReadbackStats();
        std::printf("%s: max|drho|=%.3g  max|du|=%.3g  mean|du|=%.3g  differing floats=%zu  Fx=%.5f%s\n",
                    q == 19 ? "D3Q19" : "D3Q15", maxRho, maxU, sumU / double(n), differing, st.forceX,
                    nan ? "  NaN!" : "");
        bool ok = !nan && maxRho < 0.01 && maxU < 0.01 && sumU / double(n) < 0.001 && differing == 0 && st.valid;
        std::printf("  -> %s\n", ok ? "PASS" : "FAIL");
        oracle32_destroy(cpu);
        if (!ok) return 1;
        gpu.Shutdown();
    }
    return voxelizer_check() ? 0 : 1;
}
