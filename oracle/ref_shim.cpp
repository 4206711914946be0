// ORACLE — test infrastructure only. A C-callable shim over FlowCraft's own
// CPU solver class LbmReference (FlowCraft/LbmReference.h:39-181), compiled
// together with the reference's unmodified FlowCraft/LbmReference.cpp by
// oracle/Makefile into oracle/_ref/. It exposes the same entry points as the
// restated oracle (lbm_oracle.c) so tests can run either against the same
// inputs; it is used to pin the restatement and to generate golden fixtures,
// and as the CPU baseline that bench.py times.
#include <cstdint>
#include <cstring>
#include <vector>

#include "LbmReference.h"

extern "C" {

struct oracle_params {
    float tau;
    float inlet_velocity;
    int32_t reverse_flow;
    int32_t free_slip_y;
    int32_t free_slip_z;
    float smagorinsky_cs;
};

struct oracle_stats {
    double avg_density, min_density, max_density;
    double avg_speed, max_speed;
    double force_x, force_y, force_z;
    double max_stress;
    double total_mass;
    int32_t has_nan;
    int32_t fluid_count_lo;
};

struct ref_lbm {
    LbmReference solver;
    size_t cells = 0;
};

static LbmReference::Params to_params(const oracle_params* p) {
    LbmReference::Params r;
    r.tau = p->tau;
    r.inletVelocity = p->inlet_velocity;
    r.reverseFlow = p->reverse_flow != 0;
    r.freeSlipY = p->free_slip_y != 0;
    r.freeSlipZ = p->free_slip_z != 0;
    r.smagorinskyCs = p->smagorinsky_cs;
    return r;
}

ref_lbm* ref_create(int nx, int ny, int nz, int q, const uint8_t* solid, const float* sdf, size_t sdf_count,
                    const oracle_params* p, int seed_mid) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || (q != 19 && q != 15)) return nullptr;
    VoxelGrid grid;
    grid.nx = nx;
    grid.ny = ny;
    grid.nz = nz;
    grid.cellSize = 1.0f;
    grid.solid.assign(solid, solid + grid.CellCount());
    if (sdf && sdf_count > 0) grid.signedDistance.assign(sdf, sdf + sdf_count);
    ref_lbm* r = new ref_lbm();
    r->cells = grid.CellCount();
    r->solver.Init(grid, q == 19 ? LatticeModel::D3Q19 : LatticeModel::D3Q15, to_params(p), seed_mid != 0);
    return r;
}

void ref_destroy(ref_lbm* r) { delete r; }

void ref_reset(ref_lbm* r, int seed_mid) { r->solver.Reset(seed_mid != 0); }

int ref_reset_from_field(ref_lbm* r, const float* field, size_t count) {
    std::vector<float> v(field, field + count);
    r->solver.ResetFromField(v);
    return count == r->cells * 4 ? 0 : -1;
}

void ref_set_params(ref_lbm* r, const oracle_params* p) { r->solver.SetParams(to_params(p)); }

void ref_step(ref_lbm* r, int n) {
    for (int i = 0; i < n; ++i) r->solver.Step();
}

int ref_has_diverged(const ref_lbm* r) { return r->solver.HasDiverged() ? 1 : 0; }

void ref_readback_field(ref_lbm* r, float* out) {
    std::vector<float> f = r->solver.ReadbackField();
    std::memcpy(out, f.data(), f.size() * sizeof(float));
}

void ref_stats(ref_lbm* r, oracle_stats* s) {
    LbmReference::Stats st = r->solver.ComputeStats();
    std::memset(s, 0, sizeof(*s));
    s->avg_density = st.avgDensity;
    s->min_density = st.minDensity;
    s->max_density = st.maxDensity;
    s->avg_speed = st.avgSpeed;
    s->max_speed = st.maxSpeed;
    s->force_x = st.forceX;
    s->force_y = st.forceY;
    s->force_z = st.forceZ;
    s->max_stress = st.maxStress;
    s->total_mass = st.totalMass;
    s->has_nan = st.hasNaN ? 1 : 0;
}

}  // extern "C"

// ---- Voxelizer (FlowCraft/Voxelizer.cpp:136-485) ----
#include "Voxelizer.h"

extern "C" {

struct ref_voxels {
    VoxelGrid grid;
};

ref_voxels* ref_voxelize(const float* positions, size_t vertex_count, const uint32_t* indices, size_t index_count,
                         int target_resolution, float pad_x, float pad_y, float pad_z) {
    std::vector<Vec3> pos(vertex_count);
    for (size_t i = 0; i < vertex_count; ++i) pos[i] = Vec3(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
    std::vector<uint32_t> idx(indices, indices + index_count);
    Voxelizer::Params p;
    p.targetResolution = target_resolution;
    p.paddingFactor = Vec3(pad_x, pad_y, pad_z);
    ref_voxels* v = new ref_voxels();
    v->grid = Voxelizer::Voxelize(pos, idx, p);
    return v;
}

void ref_voxels_info(const ref_voxels* v, int* dims, float* cell_size, float* origin) {
    dims[0] = v->grid.nx;
    dims[1] = v->grid.ny;
    dims[2] = v->grid.nz;
    *cell_size = v->grid.cellSize;
    origin[0] = v->grid.origin.x;
    origin[1] = v->grid.origin.y;
    origin[2] = v->grid.origin.z;
}

void ref_voxels_copy(const ref_voxels* v, uint8_t* solid, float* sdf) {
    std::memcpy(solid, v->grid.solid.data(), v->grid.solid.size());
    std::memcpy(sdf, v->grid.signedDistance.data(), v->grid.signedDistance.size() * sizeof(float));
}

void ref_voxels_free(ref_voxels* v) { delete v; }

}  // extern "C"

// ---- FieldOverlay::ComputeAerodynamicForces (FlowCraft/FieldOverlay.cpp:469-621) ----
#include "FieldOverlay.h"

extern "C" {

struct ref_aero {
    float force[3];
    float min_stress, max_stress;
    float center_of_pressure[3];
    float lift_arrow_base[3];
    int32_t has_nan;
};

void ref_aero_forces(int nx, int ny, int nz, float cell_size, const float* origin, const uint8_t* solid,
                     const float* field, ref_aero* out) {
    VoxelGrid grid;
    grid.nx = nx;
    grid.ny = ny;
    grid.nz = nz;
    grid.cellSize = cell_size;
    grid.origin = Vec3(origin[0], origin[1], origin[2]);
    grid.solid.assign(solid, solid + grid.CellCount());
    std::vector<float> f(field, field + grid.CellCount() * 4);
    FieldOverlay::AerodynamicForces a = FieldOverlay::ComputeAerodynamicForces(grid, f);
    out->force[0] = a.forceX;
    out->force[1] = a.forceY;
    out->force[2] = a.forceZ;
    out->min_stress = a.minStress;
    out->max_stress = a.maxStress;
    out->center_of_pressure[0] = a.centerOfPressure.x;
    out->center_of_pressure[1] = a.centerOfPressure.y;
    out->center_of_pressure[2] = a.centerOfPressure.z;
    out->lift_arrow_base[0] = a.liftArrowBase.x;
    out->lift_arrow_base[1] = a.liftArrowBase.y;
    out->lift_arrow_base[2] = a.liftArrowBase.z;
    out->has_nan = a.hasNaN ? 1 : 0;
}

}  // extern "C"

// ---- SmokeTrailSystem::Step (FlowCraft/SmokeTrail.cpp:278-343) ----
// The particle state is private to the class; the shim opens it (and only
// it: the standard headers and FieldOverlay.h are already included above)
// so a test can seed given positions, run the reference's own Step on a
// field, and read the trails back.
#include <random>
#define private public
#include "SmokeTrail.h"
#undef private

extern "C" {

// Seeds `count` particles at pos[p*3 .. +2] (world units), runs `steps`
// Step() calls on `field` (4 floats per cell), and writes every trail,
// oldest point first, to out[(p * trail_length + k) * 3 + 0..2] with its
// point count in lens[p]. confine_axis < 0: unconfined.
int ref_smoke_step(int nx, int ny, int nz, float cell_size, const float* origin, const uint8_t* solid,
                   const float* field, int count, int trail_length, const float* pos, int steps, int reverse,
                   float mm_per_sec, float dt, int confine_axis, int confine_index, float* out, int* lens) {
    VoxelGrid grid;
    grid.nx = nx;
    grid.ny = ny;
    grid.nz = nz;
    grid.cellSize = cell_size;
    grid.origin = Vec3(origin[0], origin[1], origin[2]);
    const size_t n = (size_t)nx * ny * nz;
    grid.solid.assign(solid, solid + n);
    std::vector<float> f(field, field + n * 4);
    SmokeTrailSystem::PlaneConfinement conf{};
    const SmokeTrailSystem::PlaneConfinement* cp = nullptr;
    if (confine_axis >= 0) {
        conf.axis = static_cast<SliceAxis>(confine_axis);
        conf.index = confine_index;
        cp = &conf;
    }
    SmokeTrailSystem sys;
    sys.Reset(grid, reverse != 0, count, trail_length, cp);
    for (int p = 0; p < count; ++p) {
        sys.particles_[(size_t)p].trail.clear();
        sys.particles_[(size_t)p].trail.push_back(Vec3(pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]));
    }
    for (int s = 0; s < steps; ++s) sys.Step(grid, f, reverse != 0, mm_per_sec, dt, false, cp);
    for (int p = 0; p < count; ++p) {
        const auto& t = sys.particles_[(size_t)p].trail;
        lens[p] = (int)t.size();
        for (int k = 0; k < trail_length; ++k) {
            float* o = out + ((size_t)p * trail_length + k) * 3;
            if (k < (int)t.size()) {
                o[0] = t[(size_t)k].x, o[1] = t[(size_t)k].y, o[2] = t[(size_t)k].z;
            } else {
                o[0] = o[1] = o[2] = 0.0f;
            }
        }
    }
    return 0;
}

}  // extern "C"
