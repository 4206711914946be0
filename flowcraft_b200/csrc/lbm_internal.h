// Shared between the kernel translation units and the C-ABI host code.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace fc {

// Grid geometry passed by value to every kernel.
struct Geom {
    int nx, ny, nz;
    int wpr;        // 32-bit words per x-row of the bulk bitmask = ceil(nx/32)
    long long nxy;  // nx*ny
    size_t n;       // nx*ny*nz (SoA plane stride)
};

// Live parameters of one step (LbmSolver::Params, LbmSolver.h:61-100).
struct StepParams {
    float tau;
    float cs;
    float inlet_ux;  // signed: -inletVelocity when reverse_flow
    int inlet_x;     // 0, or nx-1 when reverse_flow
    int outlet_x;    // nx-1, or 0 when reverse_flow
    int reverse;
    int slip_y, slip_z;
    // Inlet equilibrium feq_i(rho = 1, u = (inlet_ux, 0, 0)), computed on the
    // host with the reference's float operations (LbmReference.cpp:9-13).
    float feq_inlet[19];
};

// Per-direction plane pointers of one step, computed on the host:
// src[i] = fin + i*n - (e_x + e_y nx + e_z nx ny) (the upstream neighbour of
// cell c in plane i is src[i][c]) and dst[i] = fout + i*n. Passing them as
// kernel parameters leaves one index-times-stride per access in the kernel.
struct PlanePtrs {
    const void* src[19];
    void* dst[19];
};

// Work plan of the bulk shell kernel for one z range (see lbm_step.cu).
struct ShellPlan {
    unsigned long long n_a, n_b, n_c;  // warp items in the three regions
    int z0;                            // first z of the range (region a)
    int zi0;                           // first interior z (region c)
    int nyf, yf[2];                    // Y-face rows
    int nyi;                           // interior rows per layer (ny - 2)
    int nzf, zf[2];                    // Z-face layers inside the range
    int ncend, cend[2];                // end chunks of a row
};

// Per-link handling codes of a boundary-list cell, 3 bits per direction.
enum LinkKind : unsigned {
    kLinkStream = 0,   // upstream neighbour is interior fluid: plain pull
    kLinkBounce = 1,   // plain halfway bounce-back: f_opp(x)
    kLinkBzNear = 2,   // Bouzidi, q < 1/2: c1*f_opp(x) + c2*f_opp(x+e_i)
    kLinkBzFar = 3,    // Bouzidi, q >= 1/2: c1*f_opp(x) + c2*f_i(x)
    kLinkEdge = 4,     // off the Y/Z domain edge: free-slip mirror or bounce-back, decided per step
};
// Cell class, stored in bits 60..62 of the 64-bit link word.
enum CellClass : unsigned {
    kCellFluid = 0,      // fluid cell with a solid neighbour
    kCellSolidFill = 2,  // solid cell at x = 1 or x = nx-2 (an outlet's neighbour)
};
constexpr int kClassShift = 60;

// Device-side boundary list (sorted by cell index).
struct BoundaryList {
    const uint32_t* cells;
    const unsigned long long* links;
    const uint32_t* coef_off;
    const float2* coef;
};

// ---- launchers (defined in the .cu files) ----
// storage: 0 fp32, 1 fp16 offset, 2 bf16 offset; q: 15 or 19.
// Bulk cells of z range [z0, z0+zc): interior + shell kernels. *launched
// receives the number of kernels enqueued (0..2).
// Learned closure (closure.cuh): fragment-ordered weights, the per-cell wall
// distance and the input normalization, passed to the kernels by value.
constexpr int kClosureIn = 5;
constexpr int kClosureHidden = 32;
// 8 groups of 4 words per lane, 32 lanes (fragment order, pack_closure):
//   0 W1 with b1 as the row of K slot 5 (n-tiles 0-3)   1 b2 as a K = 8
//   fragment row (n-tiles 0-3)   2-5 W2 (one group per n-tile: k0 b0, k0 b1,
//   k1 b0, k1 b1)   6 W3 (k0 b0, k0 b1, k1 b0, k1 b1)   7 b3 (word 0, FP32)
constexpr int kClosureGroups = 8;
constexpr int kClosureVec = kClosureGroups * 32;  // uint4 entries
constexpr int kWallFar = 255;                     // wall-distance byte for 15.94+ cells

// Bytes of the closure's weight image for the tensor-core MLP (closure_tc.cuh):
// W1 (32 x 16), W2 (32 x 32), the b2 block (32 x 16) and W3 (16 x 32), BF16,
// each K-major in 8-row x 16-byte core matrices.
constexpr int kTcWeightBytes = 5120;

struct ClosureDev {
    const uint4* frag;    // kClosureVec entries
    const uint4* tcw;     // kTcWeightBytes: the weight image of the tensor-core MLP
    float b3;             // output bias, out_scale folded in
    const uint8_t* wall;  // per-cell wall distance, 1/16-cell steps
    float mean[kClosureIn];
    float inv_std[kClosureIn];
    float lo[3], hi[3];   // training range of inputs 0-2 (fallback outside)
    float filter_width;   // input 4
    unsigned wall_min;    // wall-distance byte below which a cell keeps Smagorinsky (0: none)
    float trust;          // > 0: 3 nu_t held in [ds / trust, ds * trust] around Smagorinsky's ds
    float inv_trust;      // 1 / trust
};

// Host: packs FP32 weights (w1 [5][32], b1 [32], w2 [32][32], b2 [32], w3 [32],
// b3; input-major, nu_t = relu(z) * out_scale) into kClosureVec fragment-ordered
// entries: BF16 weights and hidden-layer biases, FP32 output bias.
void pack_closure(const float* w1, const float* b1, const float* w2, const float* b2, const float* w3, float b3,
                  float out_scale, uint4* out);
// Host: the same weights (the same BF16 values) as the tensor-core MLP's
// shared-memory image, kTcWeightBytes bytes into `out`.
void pack_closure_tc(const float* w1, const float* b1, const float* w2, const float* b2, const float* w3,
                     float out_scale, uint8_t* out);
// Chamfer distance (in 1/16 cells, capped at kWallFar) from every cell to the
// nearest solid cell; `tmp` is a scratch array of g.n bytes.
cudaError_t launch_wall_distance(const uint8_t* solid, const Geom& g, uint8_t* out, uint8_t* tmp, cudaStream_t s);

// Training samples of the closure from a 2x box filter of this lattice
// (closure.cu), a Smagorinsky run with tau_f and Cs cs_f: rows (inputs 0-4,
// target nu_t) written to device `out` in
// coarse cell order. Returns an FC_LBM_* status; *count is the sample count
// (also when it exceeds `capacity`, FC_LBM_ERR_TOO_LARGE). Waits for `s`
// (bounded: FC_LBM_ERR_TIMEOUT).
int closure_samples(int q, int storage, const void* f, const uint8_t* solid, const Geom& fg, float tau_f, float cs_f,
                    float tau_c, float filter_width, float* out, int64_t capacity, int64_t* count, cudaStream_t s);

// `tc`: the MLP on the tcgen05 tensor cores, once per block (closure_tc.cuh),
// instead of the warp-level mma.sync MLP.
cudaError_t launch_bulk_pull_learned(int q, int storage, const void* fin, void* fout, const uint32_t* bulk_bits,
                                     const Geom& g, const StepParams& p, int z0, int zc, int* diverged,
                                     cudaStream_t s, int* launched, const ClosureDev& cl, int tc = 0);
cudaError_t launch_closure_probe(int q, int storage, const void* f, const uint8_t* solid, const Geom& g,
                                 const ClosureDev& cl, float* out, uint8_t* in_range, unsigned long long* counts,
                                 int layout, cudaStream_t s);

// One lattice of a batch (fc_lbm_batch): everything the persistent bulk
// kernel needs, in device memory. pp[k] are the plane pointers of a step that
// reads pop[k] and writes pop[1 - k]; a step of parity `par` reads
// pop[cur ^ par]. Work items (tiles of 64 x ROWS cells of one z layer) of
// lattice k are first .. first + gx * gy * nz - 1.
struct BatchLattice {
    Geom g;
    StepParams p;
    PlanePtrs pp[2];
    const void* pop[2];
    const uint32_t* bits;
    int* diverged;
    unsigned long long first;      // first bulk work item
    unsigned long long bnd_first;  // first entry in the concatenated boundary lists
    BoundaryList bl;
    int gx, gy;
    int cur;
    int pad;
};

// The persistent bulk kernel of a batch (all lattices even nx, one model and
// storage): `grid` blocks of 32 x rows threads loop over `total` work items.
// rows is 4, 8 or 16.
cudaError_t launch_bulk_batch(int q, int storage, int rows, const BatchLattice* lat, int nlat,
                              unsigned long long total, int parity, int grid, cudaStream_t s);
// One lattice of a one-block-per-tile batch launch (k_bulk_pairs_tiles) for
// one step: its k_bulk_pairs parameters, passed by value with the launch.
struct TileLattice {
    Geom g;
    StepParams p;
    PlanePtrs pp;
    const void* fin;
    void* fout;
    const uint32_t* bits;
    int* diverged;
    unsigned first;  // the launch's first block that is this lattice's
    int gx, gy;      // x chunks per row, 8-row blocks per layer
};
// Lattices per launch: the parameters stay under the 32 KB kernel-parameter
// limit.
constexpr int kTileLaunchLattices = 32;
struct TileLaunch {
    TileLattice l[kTileLaunchLattices];
    int nlat;
    unsigned tiles;  // blocks of the launch
};
// The bulk step of up to kTileLaunchLattices lattices of a batch as one block
// per tile of 64 x 8 cells: block w steps tile w - first of the last lattice
// whose first <= w.
cudaError_t launch_bulk_tiles(int q, int storage, const TileLaunch& t, cudaStream_t s);
// The boundary-list entries of every lattice of a batch in one launch
// (`total` = the sum of the lattices' list lengths).
cudaError_t launch_boundary_batch(int q, int storage, const BatchLattice* lat, int nlat, unsigned long long total,
                                  int parity, cudaStream_t s);
// Blocks of the batch kernel resident per SM (occupancy), or 0.
int bulk_batch_resident(int q, int storage, int rows);

// Side buffers of a lattice streamed in place (lbm_step_aa.cu): `bz` holds
// one stored population per Bouzidi coefficient slot (the far-side partner
// f*_i(c) of that link from the previous step), `outm` 2 parities x 2
// columns x `rows` (= ny * nz) moments (rho, ux, uy, uz) of the cells at
// x = 1 and x = nx-2 for the outlets.
struct AaSide {
    void* bz;
    float4* outm;
    size_t rows;
};
// One in-place step's bulk and boundary kernels; `odd` is the step's parity
// (0: reads the kLayoutAAEven state, 1: kLayoutAAOdd). Even nx >= 4 only.
cudaError_t launch_bulk_aa(int q, int storage, void* f, const uint32_t* bulk_bits, const Geom& g, const StepParams& p,
                           int z0, int zc, int* diverged, cudaStream_t s, int* launched, int odd, const AaSide& sd);
cudaError_t launch_boundary_aa(int q, int storage, void* f, const BoundaryList& bl, uint32_t begin, uint32_t end,
                               const Geom& g, const StepParams& p, int* diverged, cudaStream_t s, int odd,
                               const AaSide& sd);
// The same with the learned closure (16-bit offset formats).
cudaError_t launch_bulk_aa_learned(int q, int storage, void* f, const uint32_t* bulk_bits, const Geom& g,
                                   const StepParams& p, int z0, int zc, int* diverged, cudaStream_t s, int* launched,
                                   int odd, const AaSide& sd, const ClosureDev& cl);
cudaError_t launch_boundary_aa_learned(int q, int storage, void* f, const BoundaryList& bl, uint32_t begin,
                                       uint32_t end, const Geom& g, const StepParams& p, int* diverged,
                                       cudaStream_t s, int odd, const AaSide& sd, const ClosureDev& cl);
// Fills the side buffers from the state a step of parity `par` reads (after a
// seed or a population load); `count` = boundary-list length.
cudaError_t launch_aa_prime(int q, int storage, const void* f, const BoundaryList& bl, uint32_t count, const Geom& g,
                            const AaSide& sd, int par, cudaStream_t s);

// `staged`: run the interior rows through k_bulk_tiles (8-row tiles staged
// in shared memory by TMA tensor copies) when the lattice allows it
// (staged_eligible), the rest through k_bulk_pairs.
cudaError_t launch_bulk_pull(int q, int storage, const void* fin, void* fout, const uint32_t* bulk_bits,
                             const Geom& g, const StepParams& p, int z0, int zc, int* diverged, cudaStream_t s,
                             int* launched, int staged = 0);
// The interior rows only (lbm_step_staged.cu): rows off the Y/Z faces,
// 64-cell chunks off the row ends.
cudaError_t launch_bulk_staged(int q, int storage, const void* fin, void* fout, const uint32_t* bulk_bits,
                               const Geom& g, const StepParams& p, int z0, int zc, int* diverged, cudaStream_t s,
                               int* launched);
// nx a multiple of 16 bytes' worth of elements, nx > 128, ny, nz >= 3.
bool staged_eligible(int storage, const Geom& g);
cudaError_t launch_boundary_pull_learned(int q, int storage, const void* fin, void* fout, const BoundaryList& bl,
                                         uint32_t begin, uint32_t end, const Geom& g, const StepParams& p,
                                         int* diverged, cudaStream_t s, const ClosureDev& cl);
cudaError_t launch_boundary_pull(int q, int storage, const void* fin, void* fout, const BoundaryList& bl,
                                 uint32_t begin, uint32_t end, const Geom& g, const StepParams& p, int* diverged,
                                 cudaStream_t s);

// `layout` (every launcher that reads or writes a whole state): where the
// populations sit between steps, a PopLayout of aa.cuh: 0 plane-major
// (ping-pong), 1 / 2 one set streamed in place before an even / odd step.
cudaError_t launch_seed_uniform(int q, int storage, void* f, const Geom& g, float rho, float ux, float uy, float uz,
                                int layout, cudaStream_t s);
cudaError_t launch_seed_field(int q, int storage, void* f, const Geom& g, const float* field, const uint8_t* solid,
                              size_t cell0, size_t cells, int layout, cudaStream_t s);

cudaError_t launch_field(int q, int storage, const void* f, const uint8_t* solid, const float* sdf, const Geom& g,
                         size_t cell0, size_t cells, float* out, int layout, cudaStream_t s);
// ProbeSliceHealth's verdict for cells [cell0, cell0 + cells) on the device:
// *flag (device, cleared by the caller) becomes nonzero if a cell fails.
cudaError_t launch_probe_health(int q, int storage, const void* f, const uint8_t* solid, const float* sdf,
                                const Geom& g, size_t cell0, size_t cells, int* flag, int layout, cudaStream_t s);
cudaError_t launch_pops_out(int q, int storage, const void* f, const uint8_t* solid, int solid_is_weight,
                            const Geom& g, size_t cell0, size_t cells, float* out, int layout, cudaStream_t s);
cudaError_t launch_pops_in(int q, int storage, void* f, const Geom& g, size_t cell0, size_t cells,
                           const float* in, int layout, cudaStream_t s);

// Stats: `partials` holds stats_partial_doubles() doubles per block of
// stats_blocks(); `result` receives kStatsSlots doubles.
constexpr int kStatsSlots = 12;
int stats_blocks(const Geom& g);
cudaError_t launch_stats(int q, int storage, const void* f, const uint8_t* solid, const float* sdf, const Geom& g,
                         double* partials, int blocks, double* result, int layout, cudaStream_t s);

// Aerodynamic force integral (FieldOverlay::ComputeAerodynamicForces). The
// partials take stats_blocks(g) * kAeroSlots doubles; `result` receives
// kAeroResult doubles: force sums (3), lift and force weight sums, solid
// count, stress range (2), NaN flag, centre of pressure (3), lift arrow base
// (3).
constexpr int kAeroSlots = 20;
constexpr int kAeroResult = 16;
cudaError_t launch_aero(int q, int storage, const void* f, const uint8_t* solid, const float* sdf, const Geom& g,
                        float cell_size, float ox, float oy, float oz, double* partials, int blocks, double* result,
                        int layout, cudaStream_t s);

// Smoke-trail particles (particles.cu): trails of `length` points per
// particle in a ring (head = newest point, len = points kept, 0 = inactive).
struct ParticleSet {
    float4* trail;  // count * length points (x, y, z world, w unused)
    int* head;
    int* len;
    int count, length;
};
struct SmokeParams {
    float ox, oy, oz, cs;      // grid origin and cell size (world units)
    int reverse;               // inlet face at x = nx-1
    float scale;               // mm per second per lattice unit x dt (dt capped at 0.1 s)
    int suspend;               // vanish instead of respawning
    int confine_axis;          // -1 none, 0 / 1 / 2: the grid axis a plane fixes
    int confine_index;
    unsigned long long seed, counter;  // random draws: hash(seed, particle, counter + k)
};
cudaError_t launch_particles_step(int q, int storage, const void* f, int layout, const uint8_t* solid, const Geom& g,
                                  const ParticleSet& ps, const SmokeParams& sp, cudaStream_t s);
cudaError_t launch_particles_scatter(const uint8_t* solid, const Geom& g, const ParticleSet& ps, const SmokeParams& sp,
                                     cudaStream_t s);
cudaError_t launch_particles_shift(const Geom& g, const ParticleSet& ps, const SmokeParams& sp, cudaStream_t s);
cudaError_t launch_particles_gather(const ParticleSet& ps, float* out, int* lens, cudaStream_t s);
cudaError_t launch_particles_set(const ParticleSet& ps, const float* pos, cudaStream_t s);

// Setup (geometry classification and boundary-list construction).
// counts[0] += flagged (boundary-list) cells, counts[1] += bulk cells.
cudaError_t launch_classify(int q, const uint8_t* solid, const Geom& g, uint8_t* flags, uint32_t* bulk_bits,
                            unsigned long long* counts, cudaStream_t s);
cudaError_t launch_links(int q, const uint32_t* cells, size_t count, const uint8_t* solid, const float* sdf,
                         const Geom& g, unsigned long long* links, uint32_t* nbz, const uint32_t* coef_off,
                         float2* coef, cudaStream_t s);
cudaError_t launch_z_offsets(const uint32_t* cells, size_t count, const Geom& g, uint32_t* z_begin, cudaStream_t s);
// Ordered stream compaction of flagged cell indices (CUB); temp sized by the
// first call with temp == nullptr.
cudaError_t select_flagged_cells(void* temp, size_t& temp_bytes, const uint8_t* flags, uint32_t* out,
                                 uint32_t* count_out, size_t n, cudaStream_t s);
cudaError_t exclusive_scan_u32(void* temp, size_t& temp_bytes, const uint32_t* in, uint32_t* out, size_t n,
                               cudaStream_t s);

}  // namespace fc
