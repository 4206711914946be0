// The reference's headless GPU-vs-CPU consistency test
// (tests/gpu_vs_cpu_test.cpp:21-80) restated against this library: the
// CUDA solver through fc::LbmSolver (include/fc_lbm_solver.hpp) versus the
// CPU oracle (oracle/lbm_oracle.c, the restatement pinned to LbmReference)
// on the same 48x24x24 sphere, tau 0.6, U 0.05, Cs 0.12, mid-speed seed,
// 60 steps, both lattices. The reference passes at max|drho| < 0.01,
// max|du| < 0.01, mean|du| < 0.001 (its GPU stores FP16); the FP32 path
// here must be bit-identical, so the test also counts differing floats.
//
// Exit code: 0 pass, 1 fail, 2 no device (as the reference's test).
#include <cmath>
#include <cstdint>
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
    return 0;
}
