/*
 * fc_lbm.h — C ABI of the B200 Lattice-Boltzmann solver (libfc_lbm.so).
 *
 * Drop-in replacement for the SDL_GPU compute backend of FlowCraft's
 * `LbmSolver` (FlowCraft/LbmSolver.h:59-230). Each entry point names the
 * reference method it replaces. Differences from the reference interface:
 *   - the SDL_GPUDevice becomes a CUDA device ordinal (fc_lbm_options);
 *   - the SDL_GPUCommandBuffer argument of Step/StepRange becomes a
 *     cudaStream_t passed as `void*` (NULL = the solver's own stream);
 *   - every call returns an int status (FC_LBM_OK or a negative FC_LBM_ERR_*)
 *     instead of bool/void, and no C++ exception crosses this boundary.
 *     fc_lbm_last_error() keeps the reference's LastError() string.
 *
 * Plain pointers and sizes only: no CUDA, torch or C++ types appear in the
 * signatures. The handle is not thread-safe (the reference serialises every
 * call on one mutex, FlowCraft/main.cpp:366-368); one handle, one stream.
 *
 * Data layout seen by callers (identical to the reference):
 *   cell index  = (z*ny + y)*nx + x,
 *   field       = 4 floats per cell: (rho, ux, uy, uz) at fluid cells,
 *                 (stress, Fx, Fy, Fz) at solid cells
 *                 (FlowCraft/LbmReference.cpp:475-500).
 */
#ifndef FC_LBM_H
#define FC_LBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FC_LBM_ABI_VERSION 1

#if defined(__GNUC__)
#define FC_LBM_API __attribute__((visibility("default")))
#else
#define FC_LBM_API
#endif

/* Status codes. */
#define FC_LBM_OK 0
#define FC_LBM_ERR_INVALID_ARG (-1)
#define FC_LBM_ERR_OUT_OF_MEMORY (-2)
#define FC_LBM_ERR_CUDA (-3)
#define FC_LBM_ERR_TIMEOUT (-4)
#define FC_LBM_ERR_NOT_INITIALIZED (-5)
#define FC_LBM_ERR_UNSUPPORTED (-6)

/* LatticeModel, same enumerator order as FlowCraft/LatticeModel.h:12. */
#define FC_LATTICE_D3Q15 0
#define FC_LATTICE_D3Q19 1

/* Population storage in HBM. FP32 reproduces LbmReference bit-for-bit;
 * the 16-bit formats store (f_i - w_i) * 2^8 and collide in FP32. */
#define FC_STORAGE_FP32 0
#define FC_STORAGE_FP16_OFFSET 1
#define FC_STORAGE_BF16_OFFSET 2

/* Streaming scheme. PINGPONG keeps two population copies (pull scheme, the
 * reference's layout); AA keeps one copy updated in place, half the device
 * memory, with results bit-identical to PINGPONG (also with the learned
 * closure). AA needs an even nx >= 4 and does not combine with batches,
 * closure samples or layer copies (FC_LBM_ERR_UNSUPPORTED). */
#define FC_STREAMING_PINGPONG 0
#define FC_STREAMING_AA 1

/* Where the pointers in fc_grid_desc live. */
#define FC_MEMORY_HOST 0
#define FC_MEMORY_DEVICE 1

/* Geometry input: FlowCraft's VoxelGrid (FlowCraft/VoxelGrid.h:13-61).
 * `solid` holds nx*ny*nz bytes (nonzero = solid). `signed_distance` holds
 * nx*ny*nz floats (positive in fluid, negative in solid, +-inf far from the
 * surface) or is NULL, in which case every wall link uses plain halfway
 * bounce-back (the reference's behaviour for a missing or mis-sized SDF,
 * LbmReference.cpp:162-166). The solver copies both arrays; neither is
 * retained. */
typedef struct fc_grid_desc {
    int32_t nx, ny, nz;
    float cell_size;
    float origin[3];
    const uint8_t* solid;
    const float* signed_distance;
    int32_t memory; /* FC_MEMORY_HOST or FC_MEMORY_DEVICE */
} fc_grid_desc;

/* LbmSolver::Params (FlowCraft/LbmSolver.h:61-100); the defaults there are
 * tau 0.8, inlet 0.05, reverse 0, free-slip Y/Z 1, Cs 0.12. */
typedef struct fc_params {
    float tau;
    float inlet_velocity;
    int32_t reverse_flow;
    int32_t free_slip_y;
    int32_t free_slip_z;
    float smagorinsky_cs;
} fc_params;

/* fc_options.flags bits. TMA_STAGING runs the interior rows of the
 * ping-pong bulk step (16-bit formats, nx a multiple of 8 above 128, ny, nz
 * >= 3) through a kernel that stages 8-row tiles of the source rows in
 * shared memory with TMA tensor copies, instead of loading them directly;
 * results are identical. It is off by default: on B200 the direct loads are
 * faster (the step is issue-bound, not latency-bound). */
#define FC_OPTION_TMA_STAGING 1
/* TC_CLOSURE evaluates the learned closure's MLP in the ping-pong bulk step
 * on the tcgen05 tensor cores, once per block of 512 cells (shared-memory
 * operands, TMEM accumulators), instead of per warp with mma.sync. Results
 * agree to the FP32 rounding of the accumulation. It is off by default:
 * each block waits on its three layers in turn, and on B200 the step takes
 * twice as long in a developed flow. The in-place (AA) learned step and the
 * boundary list keep the warp-level MLP. */
#define FC_OPTION_TC_CLOSURE 2

typedef struct fc_options {
    int32_t device;    /* CUDA device ordinal */
    int32_t storage;   /* FC_STORAGE_* */
    int32_t streaming; /* FC_STREAMING_* */
    int32_t flags;     /* FC_OPTION_* bits, 0 for the defaults; other bits are rejected */
} fc_options;

/* LbmSolver::Stats (FlowCraft/LbmSolver.h:172-184) plus the FP64 sums the
 * device reduction produces (LbmReference::ComputeStats,
 * LbmReference.cpp:502-585, also reports total mass). */
typedef struct fc_stats {
    float avg_density, min_density, max_density;
    float avg_speed, max_speed;
    float force_x, force_y, force_z;
    float max_stress;
    int32_t has_nan;
    int32_t valid;
    double total_mass;
    double force_sum[3];
    double density_sum;
    double speed_sum;
    uint64_t fluid_cells;
} fc_stats;

/* FieldOverlay::AerodynamicForces (FieldOverlay.h:186-195) plus the FP64
 * sums behind it. */
typedef struct fc_aero_forces {
    float force[3];              /* forceX/Y/Z: the FP64 sums rounded to float */
    float min_stress, max_stress;
    float center_of_pressure[3]; /* world units */
    float lift_arrow_base[3];
    int32_t has_nan;
    double force_sum[3];         /* FP64 surface integral of the momentum-exchange force */
    double lift_weight_sum;      /* sum of |Fz| over solid cells */
    double force_weight_sum;     /* sum of |F| over solid cells */
    uint64_t solid_cells;
} fc_aero_forces;

typedef struct fc_lbm fc_lbm;

/* Allocates an empty solver object (no device work). Pair with destroy. */
FC_LBM_API int fc_lbm_create(fc_lbm** out);
/* Releases everything, including the object. NULL is accepted. */
FC_LBM_API void fc_lbm_destroy(fc_lbm* h);

/* LbmSolver::Init (LbmSolver.cpp:205-366). model: FC_LATTICE_*. opts may be
 * NULL (device 0, FP32, ping-pong). On failure every device resource is
 * released and fc_lbm_last_error() says why. */
FC_LBM_API int fc_lbm_init(fc_lbm* h, const fc_grid_desc* grid, int32_t model, const fc_options* opts);
/* LbmSolver::Shutdown (LbmSolver.cpp:368-387). The object stays reusable. */
FC_LBM_API int fc_lbm_shutdown(fc_lbm* h);
/* LbmSolver::LastError (LbmSolver.h:110). Never NULL. */
FC_LBM_API const char* fc_lbm_last_error(const fc_lbm* h);

/* LbmSolver::Reset (LbmSolver.cpp:389-427): stores params, seeds every cell
 * with the uniform equilibrium (quiescent, or the mid-speed seed). */
FC_LBM_API int fc_lbm_reset(fc_lbm* h, const fc_params* params, int32_t seed_at_mid_speed);
/* LbmSolver::ResetFromField (LbmSolver.cpp:429-472): per-cell equilibrium
 * from a 4-float-per-cell field. count must be 4*nx*ny*nz floats; a
 * mismatch returns FC_LBM_ERR_INVALID_ARG and leaves the state untouched
 * (the reference silently ignores it, LbmSolver.cpp:430). */
FC_LBM_API int fc_lbm_reset_from_field(fc_lbm* h, const float* field, size_t count);
/* LbmSolver::SetParams (LbmSolver.h:135): live, no state change. Rejects a
 * non-finite value, tau <= 0.5 or Cs < 0 with FC_LBM_ERR_INVALID_ARG. */
FC_LBM_API int fc_lbm_set_params(fc_lbm* h, const fc_params* params);
FC_LBM_API int fc_lbm_get_params(const fc_lbm* h, fc_params* out);

/* LbmSolver::Step (LbmSolver.cpp:556-562): n full substeps, enqueued on
 * `stream` (cudaStream_t; NULL = the solver's own stream). Asynchronous. */
FC_LBM_API int fc_lbm_step(fc_lbm* h, void* stream, int32_t n);
/* LbmSolver::StepRange (LbmSolver.cpp:543-554): one substep restricted to
 * z in [z_start, z_start + z_count); call fc_lbm_advance_substep once after
 * chunks covering the full z range. */
FC_LBM_API int fc_lbm_step_range(fc_lbm* h, void* stream, int32_t z_start, int32_t z_count);
/* LbmSolver::AdvanceSubstep (LbmSolver.h:170). */
FC_LBM_API int fc_lbm_advance_substep(fc_lbm* h);

/* LbmSolver::ReadbackField (LbmSolver.cpp:722-737). Blocking. `out` holds
 * count = 4*nx*ny*nz floats. */
FC_LBM_API int fc_lbm_readback_field(fc_lbm* h, float* out, size_t count);
/* LbmSolver::ReadbackFieldRange (LbmSolver.cpp:584-651): writes z-layers
 * [z_start, z_start+z_count) into their slots of a full-size (4*N) array. */
FC_LBM_API int fc_lbm_readback_field_range(fc_lbm* h, int32_t z_start, int32_t z_count, float* out, size_t count);
/* LbmSolver::ReadbackStats (LbmSolver.cpp:739-788), reduced on the device
 * with FP64 accumulators; only the stats struct crosses to the host. */
FC_LBM_API int fc_lbm_readback_stats(fc_lbm* h, fc_stats* out);
/* LbmSolver::ProbeSliceHealth (LbmSolver.cpp:653-720): *diverged = 1 when
 * any cell of layer z (clamped) is non-finite, or a fluid cell has rho <= 0
 * or |u|^2 > 4. */
FC_LBM_API int fc_lbm_probe_slice_health(fc_lbm* h, int32_t z, int32_t* diverged);
/* LbmReference::HasDiverged (LbmReference.h:129): sticky device flag set by
 * the step kernels for any streamed fluid cell that goes non-finite,
 * rho <= 0 or |u|^2 > 4; cleared by reset. Waits for queued work. */
FC_LBM_API int fc_lbm_has_diverged(fc_lbm* h, int32_t* diverged);

/* LbmSolver::SolidMask (LbmSolver.h:224): copies the solver's nx*ny*nz
 * solid bytes into `out`. */
FC_LBM_API int fc_lbm_copy_solid_mask(const fc_lbm* h, uint8_t* out, size_t count);
/* LbmSolver::IsValid / Model / Nx / Ny / Nz (LbmSolver.h:226-230). */
FC_LBM_API int fc_lbm_is_valid(const fc_lbm* h);
FC_LBM_API int fc_lbm_model(const fc_lbm* h);
FC_LBM_API int fc_lbm_dims(const fc_lbm* h, int32_t* nx, int32_t* ny, int32_t* nz);

/* Waits up to timeout_ms (< 0 = forever) for the solver's queued work;
 * FC_LBM_ERR_TIMEOUT if it is still running. Polls, never spins on the GPU. */
FC_LBM_API int fc_lbm_sync(fc_lbm* h, int32_t timeout_ms);
/* The solver's own stream (a cudaStream_t), for callers that order work
 * against it. */
FC_LBM_API int fc_lbm_get_stream(const fc_lbm* h, void** stream);
/* Number of cells handled by the boundary-list kernel and of interpolated
 * (Bouzidi) links; diagnostics for tests and the bench. */
FC_LBM_API int fc_lbm_boundary_info(const fc_lbm* h, uint64_t* boundary_cells, uint64_t* bouzidi_links, uint64_t* bulk_cells);
/* Runs n full substeps on the solver's own stream with CUDA events around
 * every kernel launch, waits, and reports the device time of the whole
 * sequence and the summed durations of the bulk and boundary-list kernels
 * (ms). Measurement aid for benchmarks; results equal fc_lbm_step's. */
FC_LBM_API int fc_lbm_step_timed(fc_lbm* h, int32_t n, float* total_ms, float* bulk_ms, float* boundary_ms);
/* Kernel launches this handle has enqueued since init (bench accounting). */
FC_LBM_API int fc_lbm_launch_count(const fc_lbm* h, uint64_t* launches);

/* Raw populations of the current state in the reference's natural layout
 * (post-collision, f[i*N + cell]) decoded to FP32: Q*N floats. Solid cells
 * read back as the reference holds them (the seed before the first step,
 * w_i after it) although the step never streams them. For checkpoints and
 * exhaustive tests. */
FC_LBM_API int fc_lbm_save_populations(fc_lbm* h, float* out, size_t count);
/* Restores a state written by fc_lbm_save_populations (Q*N floats). */
FC_LBM_API int fc_lbm_load_populations(fc_lbm* h, const float* in, size_t count);

/* FieldOverlay::ComputeAerodynamicForces (FieldOverlay.cpp:469-621) on the
 * current state, without the 4-float-per-cell field readback it takes in the
 * reference: the solid cells' momentum-exchange forces (the field's solid
 * entries) are summed on the device in FP64, the centre of pressure is the
 * |Fz|-weighted mean cell centre (|F|-weighted, then geometric, when the
 * weights vanish), and the lift arrow's base sits one cell above the top skin
 * in a 5x5 column patch around it. World positions use the grid's cell size
 * and origin from fc_lbm_init. Blocking. */
FC_LBM_API int fc_lbm_aero_forces(fc_lbm* h, fc_aero_forces* out);

/* ---- Learned sub-grid closure ----
 * An MLP (5 inputs -> 32 -> 32 -> 1, ReLU) predicting the eddy viscosity
 * nu_t, evaluated per cell inside the collision on the tensor cores (BF16,
 * FP32 accumulate) in place of the constant-coefficient Smagorinsky closure
 * (LbmReference.cpp:439-444): tau_eff = tau + 3 nu_t. This has no reference
 * counterpart. Inputs: 0 log2(|Pi_neq|/rho), 1 tr(Pi_neq)/|Pi_neq|,
 * 2 det(Pi_neq)/|Pi_neq|^3, 3 distance to the nearest solid cell in cells
 * (3x3x3 chamfer, 1/16-cell steps, capped at 15.9), 4 the filter width. A
 * cell whose inputs 0-2 leave [lo, hi] (the training range) keeps the
 * Smagorinsky tau_eff. Weights are input-major: w1[k*32 + j] feeds input k
 * to hidden unit j; nu_t = relu(w3 . h2 + b3) * out_scale. */
#define FC_CLOSURE_INPUTS 5
#define FC_CLOSURE_HIDDEN 32
typedef struct fc_closure {
    const float* w1; /* [5][32] */
    const float* b1; /* [32] */
    const float* w2; /* [32][32] */
    const float* b2; /* [32] */
    const float* w3; /* [32] */
    float b3;
    float out_scale;
    float mean[FC_CLOSURE_INPUTS]; /* input normalization: (x - mean) / std */
    float std[FC_CLOSURE_INPUTS];
    float lo[3], hi[3];            /* training range of inputs 0-2 */
    float filter_width;            /* input 4 for this lattice */
    float min_wall_distance;       /* cells nearer a wall than this (in cells) keep Smagorinsky; 0 = none */
    float trust_factor;            /* 0 = off; k >= 1: 3 nu_t held in [d/k, d k], d = 3 nu_t of Smagorinsky */
} fc_closure;

/* Installs the closure (copied; NULL returns to Smagorinsky) for every later
 * step, under either streaming scheme. Needs FP16/BF16 offset storage and an
 * even nx (FC_LBM_ERR_UNSUPPORTED otherwise). The first call computes the
 * wall distance field (one byte per cell). Blocking. */
FC_LBM_API int fc_lbm_set_closure(fc_lbm* h, const fc_closure* c);
/* The closure evaluated on the current populations as stored, by the same
 * device code as the step: out[5*c .. 5*c+4] = inputs 0-3 and nu_t,
 * in_range[c] = 1 where the learned nu_t is used. Host arrays; cells must be
 * nx*ny*nz. For checking the inference. */
FC_LBM_API int fc_lbm_closure_probe(fc_lbm* h, float* out, uint8_t* in_range, size_t cells);
/* How much of the current state the closure covers: the cells whose inputs
 * are in the training range, and the groups of 64 consecutive cells that
 * hold at least one of them. When nx is a multiple of 64 those groups are the
 * step kernel's warps, and the count is the number of warps that evaluate
 * the MLP in a step; the others keep Smagorinsky and skip it. Blocking. */
FC_LBM_API int fc_lbm_closure_coverage(fc_lbm* h, uint64_t* cells_in_range, uint64_t* warps_with_mlp);
/* The wall-distance input (1/16-cell steps, 255 = 15.94 cells or more). */
FC_LBM_API int fc_lbm_wall_distance(fc_lbm* h, uint8_t* out, size_t cells);

/* Training samples for the closure from this (fine) lattice: its current
 * populations are box-filtered 2x2x2 onto a lattice of half the size; every
 * coarse cell off the faces and the inlet/outlet planes whose 6 neighbours
 * are fluid gives one row of 6 floats (inputs 0-4 and the target nu_t),
 * written to the DEVICE array `out` in coarse-cell order. The target is the
 * eddy viscosity that carries the filtered flow's stress: the least-squares
 * fit of the box-filtered viscous stress of the fine cells (molecular plus
 * this lattice's Smagorinsky, at its tau and Cs) minus the resolved sub-grid
 * stress, against the filtered strain (central differences), less the coarse
 * molecular viscosity, clipped at 0; the inputs are those of a coarse cell
 * relaxing with the coarse molecular tau plus 3 nu_t.
 * *count receives the number of rows; with out NULL or capacity too small
 * nothing is written (FC_LBM_ERR_TOO_LARGE when rows did not fit). Blocking.
 * No reference counterpart. */
FC_LBM_API int fc_lbm_closure_samples(fc_lbm* h, float filter_width, float* out, int64_t capacity, int64_t* count);

/* ---- Training the closure's MLP (no reference counterpart) ----
 * params: FC_MLP_PARAMS floats, w1[5*32], b1[32], w2[32*32], b2[32], w3[32],
 * b3 (the fc_closure layout, unscaled), on the device like every array here.
 * x: n rows of the 5 normalized inputs; y: n targets. The output is linear
 * (training); inference applies relu and out_scale. All calls are
 * asynchronous on `stream`. */
#define FC_MLP_PARAMS 1281
#define FC_MLP_GRAD_SCRATCH 190000 /* floats */
FC_LBM_API int fc_lbm_mlp_forward(const float* params, const float* x, int64_t n, float* y, void* stream);
/* grad = d/dparams of the mean squared error over rows idx[0..n) (idx NULL:
 * rows 0..n-1), *loss (device double, or NULL) = that error. Deterministic:
 * the same inputs give the same bits. scratch: FC_MLP_GRAD_SCRATCH floats. */
FC_LBM_API int fc_lbm_mlp_grad(const float* params, const float* x, const float* y, const int64_t* idx, int64_t n,
                               float* grad, double* loss, float* scratch, void* stream);
/* One Adam step (Kingma & Ba 2015) with bias correction; step counts from 1. */
FC_LBM_API int fc_lbm_mlp_adam(float* params, const float* grad, float* m, float* v, int32_t step, float lr,
                               float beta1, float beta2, float eps, void* stream);

/* Copies the Q populations of z-layer `z` between a population set and a
 * contiguous DEVICE buffer of Q*nx*ny elements (storage format, plane i
 * first): `next` = 0 is the current set, 1 the set the in-progress step
 * writes (between fc_lbm_step_range and fc_lbm_advance_substep);
 * `to_buffer` = 1 packs into the buffer, 0 unpacks from it. Asynchronous on
 * `stream`. The halo exchange of a lattice split into z-slabs across GPUs
 * (flowcraft_b200/shard.py) is built on it; no reference counterpart. */
FC_LBM_API int fc_lbm_layer_copy(fc_lbm* h, int32_t z, int32_t next, void* buffer, int32_t to_buffer, void* stream);
/* The same for the planes whose e_z equals `ez` only (+1 or -1; 0 = all Q
 * planes, as fc_lbm_layer_copy): their rows, in plane order, are the first
 * FC_LBM_DIR_PLANES rows of the buffer. A step of the layer next to a halo
 * reads only the halo's planes that stream toward it (e_z = +1 from the
 * layer below, -1 from the layer above), so a per-step halo exchange moves 5
 * of the Q planes. No reference counterpart. */
#define FC_LBM_DIR_PLANES 5
FC_LBM_API int fc_lbm_layer_copy_dir(fc_lbm* h, int32_t z, int32_t next, void* buffer, int32_t to_buffer, int32_t ez,
                                     void* stream);

/* ---- Asynchronous field readback (overlapped with stepping) ----
 * What FlowCraft's ReadbackFieldPacedGPU (main.cpp:2506-2555) does with
 * adaptive blocking z-chunks so that a readback never stalls the solver:
 * here one kernel snapshots the whole 4-float field (ReadbackField's layout)
 * of the state every queued step leaves into a device buffer (16 bytes per
 * cell, allocated on the first call) on a side stream, and the copy to
 * `out` follows on that stream. The call returns at once; steps enqueued
 * afterwards run while the copy is in flight and only the first one that
 * overwrites the population set the snapshot reads waits for the snapshot
 * kernel (not for the copy). `out` must stay valid until
 * fc_lbm_readback_wait returns; page-locked memory (fc_lbm_alloc_pinned)
 * lets the copy run asynchronously. One readback at a time: a second call
 * first waits for the first. */
FC_LBM_API int fc_lbm_readback_field_async(fc_lbm* h, float* out, size_t count);
/* Waits (bounded, -1 = no limit) until the pending readback's copy has
 * landed; FC_LBM_OK at once when none is pending. */
FC_LBM_API int fc_lbm_readback_wait(fc_lbm* h, int32_t timeout_ms);
/* Page-locked host memory for asynchronous readbacks. */
FC_LBM_API int fc_lbm_alloc_pinned(size_t bytes, void** out);
FC_LBM_API int fc_lbm_free_pinned(void* p);

/* ---- Smoke-trail particles (SmokeTrailSystem, FlowCraft/SmokeTrail.h:26-184) ----
 * Particles with short trails advected through the solver's own velocity,
 * sampled on the device from the current populations (the velocity the field
 * readback would report, trilinearly interpolated as SampleVelocityInterpolated
 * does, SmokeTrail.cpp:69-116) instead of from a host copy of the field.
 * Positions are world coordinates (VoxelGrid::CellCenter: grid x is world Y,
 * grid y is world X). `confine_axis` < 0 means unconfined, else the grid axis
 * (0 x, 1 y, 2 z) of a PlaneConfinement at `confine_index`. Random draws come
 * from a counter-based hash of `seed` (the reference uses std::mt19937), so
 * respawned particles land elsewhere than the reference's; the rules are the
 * reference's. All calls are ordered on the solver's stream. */
/* SmokeTrailSystem::Reset (SmokeTrail.cpp:257-276): `count` particles with
 * trails of max(trail_length, 2) points, scattered over the domain (or plane).
 * Allocates the particle buffers. */
FC_LBM_API int fc_lbm_particles_reset(fc_lbm* h, int32_t count, int32_t trail_length, uint64_t seed,
                                      int32_t confine_axis, int32_t confine_index);
/* SmokeTrailSystem::Step (SmokeTrail.cpp:278-343): one advection of every
 * particle by the current velocity x mm_per_sec_per_lattice_unit x
 * min(dt_seconds, 0.1); a particle that left the grid or entered a solid cell
 * respawns at the inlet face (or plane), or vanishes with suspend_respawn.
 * dt_seconds <= 0 does nothing. Asynchronous. */
FC_LBM_API int fc_lbm_particles_step(fc_lbm* h, int32_t reverse_flow, float mm_per_sec_per_lattice_unit,
                                     float dt_seconds, int32_t suspend_respawn, int32_t confine_axis,
                                     int32_t confine_index);
/* SmokeTrailSystem::ScatterRandom (SmokeTrail.cpp:206-220). */
FC_LBM_API int fc_lbm_particles_scatter(fc_lbm* h, int32_t confine_axis, int32_t confine_index);
/* SmokeTrailSystem::ShiftPlane (SmokeTrail.cpp:222-255): every trail point onto
 * the plane at confine_index along confine_axis (0..2). */
FC_LBM_API int fc_lbm_particles_shift_plane(fc_lbm* h, int32_t confine_axis, int32_t confine_index);
/* Every trail, oldest point first: points[(p * L + k) * 3 + 0..2] for
 * k < lens[p], zeros after (L = the trail length of the last reset). Blocks. */
FC_LBM_API int fc_lbm_particles_read(fc_lbm* h, float* points, size_t points_count, int32_t* lens,
                                     size_t lens_count);
/* Every particle to the single point points[p * 3 + 0..2] (world units),
 * trail cleared. Blocks. */
FC_LBM_API int fc_lbm_particles_set(fc_lbm* h, const float* points, size_t points_count);

/* ---- Batches: many lattices stepped together (no reference counterpart) ----
 * For sweeps such as a set of angles of attack: the members (initialized
 * handles on one device, one lattice model and storage format, even nx, no
 * learned closure) step together. Every step is one persistent bulk launch
 * over a work-list of the tiles of all members (or, when that is faster,
 * each member's own bulk kernel, run side by side on forked streams) and one
 * launch over all their boundary lists; pairs of steps replay as one CUDA
 * graph. Results are
 * bit-identical to stepping every member with fc_lbm_step. The members keep
 * their own state and API; they must outlive the batch and must not step on
 * their own while a batch step is queued. */
typedef struct fc_lbm_batch fc_lbm_batch;
#define FC_LBM_BATCH_CANDIDATES 8
FC_LBM_API int fc_lbm_batch_create(fc_lbm* const* members, int32_t count, fc_lbm_batch** out);
FC_LBM_API void fc_lbm_batch_destroy(fc_lbm_batch* b);
FC_LBM_API const char* fc_lbm_batch_last_error(const fc_lbm_batch* b);
/* n steps of every member; asynchronous, ordered after and before the
 * members' own streams. An odd n leaves the next call to rebuild its graph. */
FC_LBM_API int fc_lbm_batch_step(fc_lbm_batch* b, int32_t n);
/* The block shape of the batch's bulk launch: rows in {4, 8, 16} (a block is
 * 32 x rows threads over 64 x rows cells) with grid_mult in {1, 2} (a
 * persistent launch of resident blocks per SM times this, each block taking
 * chunks of 8 tiles), or rows 8 with grid_mult 0 (one block per tile over the
 * tiles of every lattice, each lattice's in the order of its own launch, the
 * lattices one after another; one launch per 32 lattices). rows 0
 * replaces the batch launch by each member's own bulk kernel (the one
 * fc_lbm_step launches), spread over 4 forked streams; grid_mult is then
 * unused. Default 8, 1. */
FC_LBM_API int fc_lbm_batch_config(fc_lbm_batch* b, int32_t rows, int32_t grid_mult);
/* Autotuner: times each of the FC_LBM_BATCH_CANDIDATES shapes (rows 4, 8, 16
 * x grid_mult 1, 2, in that order, then rows 8 with grid_mult 0, then rows 0)
 * over `steps` (rounded up to even) real steps after 2 warm-up steps, and
 * keeps the fastest. Every member advances by 8 x (steps + 2) steps (the
 * candidates compute identical results).
 * ms_per_step (may be NULL) receives each candidate's time. Blocking. */
FC_LBM_API int fc_lbm_batch_tune(fc_lbm_batch* b, int32_t steps, int32_t* rows, int32_t* grid_mult,
                                 float* ms_per_step);

/* Statistics of a population set computed without allocating anything: no
 * cudaMalloc, cudaFree or allocating library call happens inside. This entry
 * point has no counterpart in the reference. It is meant for callers that
 * cannot allocate device memory: applications whose own pool allocator owns
 * all of the GPU's memory, runs under a fixed memory budget that must not hit
 * out-of-memory halfway through, and latency-critical loops in which a
 * cudaMalloc or cudaFree could synchronize the device and stall stepping.
 *
 * All pointers are device memory on the calling thread's current device:
 * `populations` holds Q*N values in `storage`'s format (FC_STORAGE_*), laid
 * out f[i*N + cell] with N = nx*ny*nz (plane-major, the layout of a ping-pong
 * set and of fc_lbm_save_populations; a set streamed in place with
 * FC_STREAMING_AA keeps population i of a cell in other slots between steps,
 * and passing it here is a caller error that the call cannot detect: it reads
 * the wrong slots); `solid` holds N bytes;
 * `signed_distance` holds N floats or is NULL. The result is written to the
 * device buffer `out_slots` (FC_LBM_STATS_SLOTS doubles: density sum, speed
 * sum, mass, Fx, Fy, Fz, fluid cell count, min density, max density, max
 * speed, max stress, NaN flag), asynchronously on `stream` (a cudaStream_t;
 * NULL = the default stream).
 *
 * The reduction's per-block partial sums live in one fixed 384 KiB array
 * inside the library, which every GPU that loads the library holds until the
 * process exits. It covers lattices up to FC_LBM_NOALLOC_MAX_CELLS cells;
 * larger ones are refused with FC_LBM_ERR_TOO_LARGE before any work is
 * queued. The first call on each device looks up that array's device address
 * once and keeps it for the life of the process; make that first call before
 * any stream capture begins. The kept address does not survive
 * cudaDeviceReset (the reset unloads the array), so do not call this entry
 * point on a device after resetting it. Every call reuses the same array, so
 * two calls whose work overlaps on the GPU (on different streams without
 * ordering) race; order them on one stream or with events. */
#define FC_LBM_STATS_SLOTS 12
#define FC_LBM_NOALLOC_MAX_CELLS 536870912ull
#define FC_LBM_ERR_TOO_LARGE (-7)
FC_LBM_API int fc_lbm_stats_noalloc(const void* populations, const uint8_t* solid, const float* signed_distance,
                                    int32_t nx, int32_t ny, int32_t nz, int32_t model, int32_t storage,
                                    double* out_slots, void* stream);

/* ---- Mesh voxelizer ----
 * Replaces Voxelizer::Voxelize (FlowCraft/Voxelizer.h:44-45,
 * Voxelizer.cpp:136-485), the producer of the VoxelGrid that fc_lbm_init
 * consumes. The results are bit-identical to the reference's CPU voxelizer:
 * the same cells, the same solid mask and the same float signed distances
 * (positive in the fluid, negative in the solid, +-infinity where no triangle
 * came within reach), computed on the current device. Positions are float
 * triples (x, y, z) in world units; indices are uint32 triples, one per
 * triangle, any trailing remainder ignored as in the reference. Grid x spans
 * world y (the flow axis) and grid y spans world x (VoxelGrid.h:43-56). With
 * `memory` = FC_MEMORY_DEVICE every array is device memory on the current
 * device; with FC_MEMORY_HOST every array is host memory. Both calls block
 * until their results are ready; their work runs on `stream` (a cudaStream_t;
 * NULL = the default stream). */
typedef struct fc_voxel_params {
    int32_t target_resolution; /* cells along the padded domain's longest axis; reference default 640 */
    float padding[3];          /* padding per side as a fraction of the model's extent; default {0.3, 1.0, 0.5} */
} fc_voxel_params;

/* The grid Voxelize derives for a mesh (Voxelizer.cpp:146-166): dims (nx, ny,
 * nz), cell size and world origin of the padded domain. The caller handles the
 * reference's empty-grid case (no vertices or fewer than 3 indices) itself;
 * vertex_count = 0 returns FC_LBM_ERR_INVALID_ARG. */
FC_LBM_API int fc_lbm_voxel_grid(const float* positions, size_t vertex_count, const fc_voxel_params* params,
                                 int32_t memory, int32_t dims[3], float* cell_size, float origin[3], void* stream);

/* Voxelizes the mesh onto an explicit grid: `solid` receives nx*ny*nz bytes
 * (0 fluid, 1 solid) and `signed_distance` nx*ny*nz floats, indexed
 * (z*ny + y)*nx + x. On the grid from fc_lbm_voxel_grid this is
 * Voxelizer::Voxelize; any other grid (a chosen cell size and origin) runs the
 * same rasterization, flood fill from cell (0,0,0) and sign reconciliation.
 * Returns FC_LBM_ERR_INVALID_ARG for an index outside the vertex array, and
 * FC_LBM_ERR_TOO_LARGE for grids of 2^32-1 cells or more. */
FC_LBM_API int fc_lbm_voxelize(const float* positions, size_t vertex_count, const uint32_t* indices,
                               size_t index_count, const int32_t dims[3], float cell_size, const float origin[3],
                               int32_t memory, uint8_t* solid, float* signed_distance, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FC_LBM_H */
