// fc_lbm_solver.hpp — C++ host mirror of FlowCraft's LbmSolver
// (FlowCraft/LbmSolver.h:59-230) over the C ABI in fc_lbm.h.
//
// Same method names, argument meanings and error behaviour as the reference
// class, so a caller switches backends by swapping the type:
//   - Init(device, grid, model) returns false and sets LastError() on failure;
//   - Reset/ResetFromField/SetParams/Step/StepRange/AdvanceSubstep return
//     void, and ResetFromField ignores a mis-sized field (LbmSolver.cpp:430);
//   - ReadbackField/ReadbackFieldRange/ReadbackStats/ProbeSliceHealth block.
// The SDL_GPUDevice* becomes a CUDA device ordinal and the
// SDL_GPUCommandBuffer* a cudaStream_t (any pointer-sized stream handle;
// nullptr = the solver's own stream). Init() accepts any grid type with the
// fields of FlowCraft's VoxelGrid (nx, ny, nz, cellSize, origin.{x,y,z},
// solid, signedDistance), including that VoxelGrid itself.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "fc_lbm.h"

namespace fc {

enum class LatticeModel { D3Q15 = FC_LATTICE_D3Q15, D3Q19 = FC_LATTICE_D3Q19 };

enum class Storage { FP32 = FC_STORAGE_FP32, FP16Offset = FC_STORAGE_FP16_OFFSET, BF16Offset = FC_STORAGE_BF16_OFFSET };
// PingPong keeps two population copies (the reference's scheme); InPlace one,
// streamed with the AA pattern (bit-identical results, half the memory).
enum class Streaming { PingPong = FC_STREAMING_PINGPONG, InPlace = FC_STREAMING_AA };

struct Vec3f {
    float x = 0.0f, y = 0.0f, z = 0.0f;
};

class LbmSolver {
public:
    // LbmSolver::Params (LbmSolver.h:61-100), same defaults.
    struct Params {
        float tau = 0.8f;
        float inletVelocity = 0.05f;
        bool reverseFlow = false;
        bool freeSlipY = true;
        bool freeSlipZ = true;
        float smagorinskyCs = 0.12f;
    };

    // LbmSolver::Stats (LbmSolver.h:172-184). centerOfPressure/liftBaseZ are
    // filled by the caller from the field, as in the reference.
    struct Stats {
        float avgDensity = 0.0f, minDensity = 0.0f, maxDensity = 0.0f;
        float avgSpeed = 0.0f, maxSpeed = 0.0f;
        float forceX = 0.0f, forceY = 0.0f, forceZ = 0.0f;
        float maxStress = 0.0f;
        Vec3f centerOfPressure;
        float liftBaseZ = 0.0f;
        bool hasNaN = false;
        bool valid = false;
        double totalMass = 0.0;  // FP64 device sum (LbmReference::Stats has it too)
    };

    LbmSolver() { fc_lbm_create(&h_); }
    ~LbmSolver() { fc_lbm_destroy(h_); }
    LbmSolver(const LbmSolver&) = delete;
    LbmSolver& operator=(const LbmSolver&) = delete;

    template <class Grid>
    // The reference's Init(device, grid, model); storage, streaming and the
    // FC_OPTION_* flags are additions with the reference's behaviour as
    // defaults.
    bool Init(int device, const Grid& grid, LatticeModel model, Storage storage = Storage::FP32,
              Streaming streaming = Streaming::PingPong, int32_t flags = 0) {
        fc_grid_desc d{};
        d.nx = grid.nx;
        d.ny = grid.ny;
        d.nz = grid.nz;
        d.cell_size = grid.cellSize;
        d.origin[0] = grid.origin.x;
        d.origin[1] = grid.origin.y;
        d.origin[2] = grid.origin.z;
        d.solid = grid.solid.data();
        const size_t cells = (size_t)grid.nx * grid.ny * grid.nz;
        // a missing or mis-sized SDF means plain bounce-back (LbmReference.cpp:162-166)
        d.signed_distance = grid.signedDistance.size() == cells ? grid.signedDistance.data() : nullptr;
        d.memory = FC_MEMORY_HOST;
        fc_options o{device, (int32_t)storage, (int32_t)streaming, flags};
        model_ = model;
        const bool ok = fc_lbm_init(h_, &d, (int32_t)model, &o) == FC_LBM_OK;
        if (ok) {
            solidCpu_.assign(grid.solid.begin(), grid.solid.end());
            fc_lbm_dims(h_, &nx_, &ny_, &nz_);
        }
        return ok;
    }
    void Shutdown() {
        fc_lbm_shutdown(h_);
        nx_ = ny_ = nz_ = 0;
    }
    std::string LastError() const { return fc_lbm_last_error(h_); }

    void Reset(const Params& params, bool seedAtMidSpeed = false) {
        fc_params p = toC(params);
        fc_lbm_reset(h_, &p, seedAtMidSpeed ? 1 : 0);
    }
    void ResetFromField(const std::vector<float>& field) { fc_lbm_reset_from_field(h_, field.data(), field.size()); }
    void SetParams(const Params& params) {
        fc_params p = toC(params);
        fc_lbm_set_params(h_, &p);
    }

    void Step(void* cmd, int numSubsteps) { fc_lbm_step(h_, cmd, numSubsteps); }
    void StepRange(void* cmd, int zStart, int zCount) { fc_lbm_step_range(h_, cmd, zStart, zCount); }
    void AdvanceSubstep() { fc_lbm_advance_substep(h_); }

    Stats ReadbackStats() {
        Stats s;
        fc_stats c{};
        if (fc_lbm_readback_stats(h_, &c) != FC_LBM_OK) return s;
        s.avgDensity = c.avg_density;
        s.minDensity = c.min_density;
        s.maxDensity = c.max_density;
        s.avgSpeed = c.avg_speed;
        s.maxSpeed = c.max_speed;
        s.forceX = c.force_x;
        s.forceY = c.force_y;
        s.forceZ = c.force_z;
        s.maxStress = c.max_stress;
        s.hasNaN = c.has_nan != 0;
        s.valid = c.valid != 0;
        s.totalMass = c.total_mass;
        return s;
    }
    std::vector<float> ReadbackField() {
        std::vector<float> field;
        if (!IsValid()) return field;
        field.resize(CellCount() * 4);
        fc_lbm_readback_field(h_, field.data(), field.size());
        return field;
    }
    void ReadbackFieldRange(int zStart, int zCount, std::vector<float>& outField) {
        fc_lbm_readback_field_range(h_, zStart, zCount, outField.data(), outField.size());
    }
    bool ProbeSliceHealth(int zLayer) {
        int32_t d = 0;
        fc_lbm_probe_slice_health(h_, zLayer, &d);
        return d != 0;
    }
    // FieldOverlay::ComputeAerodynamicForces (FieldOverlay.cpp:469-621) of the
    // current state, integrated on the device in FP64. The returned struct
    // has the reference's fields plus the FP64 sums; `ok` false on failure.
    fc_aero_forces AerodynamicForces(bool* ok = nullptr) {
        fc_aero_forces a{};
        const int rc = fc_lbm_aero_forces(h_, &a);
        if (ok) *ok = rc == FC_LBM_OK;
        return a;
    }
    // LbmReference::HasDiverged (LbmReference.h:129), a device flag here.
    bool HasDiverged() {
        int32_t d = 0;
        fc_lbm_has_diverged(h_, &d);
        return d != 0;
    }
    bool Sync(int timeoutMs = -1) { return fc_lbm_sync(h_, timeoutMs) == FC_LBM_OK; }
    // The learned sub-grid closure (an addition; nullptr returns to
    // Smagorinsky). The weights are copied.
    bool SetClosure(const fc_closure* closure) { return fc_lbm_set_closure(h_, closure) == FC_LBM_OK; }

    const std::vector<uint8_t>& SolidMask() const { return solidCpu_; }
    bool IsValid() const { return fc_lbm_is_valid(h_) != 0; }
    LatticeModel Model() const { return model_; }
    int Nx() const { return nx_; }
    int Ny() const { return ny_; }
    int Nz() const { return nz_; }
    size_t CellCount() const { return (size_t)nx_ * ny_ * nz_; }
    fc_lbm* Handle() const { return h_; }

private:
    static fc_params toC(const Params& p) {
        return fc_params{p.tau, p.inletVelocity, p.reverseFlow ? 1 : 0, p.freeSlipY ? 1 : 0, p.freeSlipZ ? 1 : 0,
                         p.smagorinskyCs};
    }
    fc_lbm* h_ = nullptr;
    LatticeModel model_ = LatticeModel::D3Q19;
    std::vector<uint8_t> solidCpu_;
    int32_t nx_ = 0, ny_ = 0, nz_ = 0;
};

// Voxelizer::Voxelize (FlowCraft/Voxelizer.h:12-53) on the GPU, bit-identical
// to the reference's CPU voxelizer. `Grid` is any type with the fields of
// FlowCraft's VoxelGrid (nx, ny, nz, cellSize, origin.{x,y,z}, solid,
// signedDistance), `Vec` any type with float members x, y, z. Runs on the
// current CUDA device and blocks until the grid is on the host. Returns false
// (grid left empty) when the CUDA call fails, with the status in *status.
struct VoxelizerParams {
    int targetResolution = 640;
    Vec3f paddingFactor{0.3f, 1.0f, 0.5f};
};

template <class Grid, class Vec>
bool Voxelize(const std::vector<Vec>& positions, const std::vector<uint32_t>& indices, const VoxelizerParams& params,
              Grid& grid, int* status = nullptr) {
    grid = Grid{};
    if (status) *status = FC_LBM_OK;
    if (positions.empty() || indices.size() < 3) return true;  // the reference's empty grid
    std::vector<float> pos(positions.size() * 3);
    for (size_t i = 0; i < positions.size(); ++i) {
        pos[3 * i] = positions[i].x;
        pos[3 * i + 1] = positions[i].y;
        pos[3 * i + 2] = positions[i].z;
    }
    fc_voxel_params p{params.targetResolution,
                      {params.paddingFactor.x, params.paddingFactor.y, params.paddingFactor.z}};
    int32_t dims[3] = {0, 0, 0};
    float cell = 0.0f, origin[3] = {0.0f, 0.0f, 0.0f};
    int rc = fc_lbm_voxel_grid(pos.data(), positions.size(), &p, FC_MEMORY_HOST, dims, &cell, origin, nullptr);
    std::vector<uint8_t> solid;
    std::vector<float> sdf;
    if (rc == FC_LBM_OK) {
        const size_t n = (size_t)dims[0] * dims[1] * dims[2];
        solid.resize(n);
        sdf.resize(n);
        rc = fc_lbm_voxelize(pos.data(), positions.size(), indices.data(), indices.size(), dims, cell, origin,
                             FC_MEMORY_HOST, solid.data(), sdf.data(), nullptr);
    }
    if (status) *status = rc;
    if (rc != FC_LBM_OK) return false;
    grid.nx = dims[0];
    grid.ny = dims[1];
    grid.nz = dims[2];
    grid.cellSize = cell;
    grid.origin.x = origin[0];
    grid.origin.y = origin[1];
    grid.origin.z = origin[2];
    grid.solid = std::move(solid);
    grid.signedDistance = std::move(sdf);
    return true;
}

}  // namespace fc
