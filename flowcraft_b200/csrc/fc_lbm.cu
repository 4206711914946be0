// Host side of the C ABI declared in include/fc_lbm.h: the CUDA-backed
// replacement of FlowCraft's SDL_GPU LbmSolver (FlowCraft/LbmSolver.cpp).
//
// One handle owns one lattice on one device: the population set(s), the
// solid mask and SDF (for readback forces), the bit-packed bulk mask, the
// compacted boundary list with its Bouzidi coefficients, a stream, and
// pinned staging for transfers. Device memory is allocated in fc_lbm_init
// and released in fc_lbm_shutdown; stepping and readback allocate nothing.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fc_lbm.h"
#include "aa.cuh"
#include "lattice.cuh"
#include "lbm_internal.h"

using fc::Geom;

struct fc_lbm {
    std::string err;
    bool valid = false;
    int device = 0;
    int q = 19;
    int model = FC_LATTICE_D3Q19;
    int storage = FC_STORAGE_FP32;
    int streaming = FC_STREAMING_PINGPONG;
    int flags = 0;  // FC_OPTION_* bits
    Geom g{};
    fc_params params{0.8f, 0.05f, 0, 1, 1, 0.12f};  // LbmSolver::Params defaults (LbmSolver.h:61-100)
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_own = nullptr, ev_foreign = nullptr, ev_sync = nullptr;
    void* pop[2] = {nullptr, nullptr};  // AA streaming: one set, pop[1] == pop[0]
    int cur = 0;                         // AA streaming: the next step's parity
    void* d_aa_bz = nullptr;             // AA side buffers (lbm_internal.h AaSide)
    float4* d_aa_outm = nullptr;
    uint8_t* d_solid = nullptr;
    float* d_sdf = nullptr;
    uint32_t* d_bulk_bits = nullptr;
    uint32_t* d_cells = nullptr;
    unsigned long long* d_links = nullptr;
    uint32_t* d_coef_off = nullptr;
    float2* d_coef = nullptr;
    std::vector<uint32_t> z_begin;
    size_t n_bnd = 0, n_bz = 0, n_bulk = 0;
    int* d_diverged = nullptr;
    double* d_stats_partials = nullptr;
    double* d_stats_result = nullptr;
    int stats_blocks = 0;
    double* d_aero_partials = nullptr;
    double* d_aero_result = nullptr;
    float cell_size = 1.0f;
    float origin[3] = {0.0f, 0.0f, 0.0f};
    bool closure_on = false;  // learned closure in place of Smagorinsky
    fc::ClosureDev closure{};
    uint4* d_closure = nullptr;
    uint4* d_closure_tc = nullptr;  // the weight image of the tensor-core MLP
    uint8_t* d_wall = nullptr;
    float* d_stage = nullptr;
    float* h_stage = nullptr;
    size_t stage_floats = 0;
    std::vector<uint8_t> solid_cpu;
    uint64_t steps_since_reset = 0;
    uint64_t launches = 0;
    // asynchronous field readback: a snapshot kernel on rb_stream into
    // d_snap, then the host copy; ev_snap marks the snapshot kernel's end
    float* d_snap = nullptr;
    cudaStream_t rb_stream = nullptr;
    cudaEvent_t ev_snap = nullptr, ev_rb = nullptr;
    bool rb_pending = false;
    int snap_set = -1;  // population set the pending snapshot reads
    // smoke-trail particles (particles.cu)
    fc::ParticleSet parts{nullptr, nullptr, nullptr, 0, 0};
    float* d_part_io = nullptr;  // count * length * 3 floats: trail readout / position upload
    int* d_part_lens = nullptr;
    unsigned long long part_seed = 0, part_counter = 0;
};

namespace {

constexpr size_t kStageFloats = size_t(1) << 24;  // 64 MiB device + 64 MiB pinned host
constexpr int kTransferTimeoutMs = 600000;

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~DeviceGuard() {
        int now = -1;
        if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
    }
};

int fail(fc_lbm* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

int cuda_fail(fc_lbm* h, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (e == cudaErrorMemoryAllocation) return fail(h, FC_LBM_ERR_OUT_OF_MEMORY, m);
    return fail(h, FC_LBM_ERR_CUDA, m);
}

#define FC_TRY(h, expr, what)                                 \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) return cuda_fail(h, _e, what); \
    } while (0)

#define FC_RC(expr)               \
    do {                          \
        int _rc = (expr);         \
        if (_rc != FC_LBM_OK) return _rc; \
    } while (0)

template <class T>
void dfree(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// Waits for everything queued on the handle's stream. Polls with a growing
// sleep so the host never spins on the GPU and a stuck device surfaces as a
// timeout status rather than a hang.
int wait_stream(fc_lbm* h, int timeout_ms) {
    cudaError_t e = cudaEventRecord(h->ev_sync, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaEventRecord");
    auto t0 = std::chrono::steady_clock::now();
    int sleep_us = 5;
    for (;;) {
        e = cudaEventQuery(h->ev_sync);
        if (e == cudaSuccess) return FC_LBM_OK;
        if (e != cudaErrorNotReady) return cuda_fail(h, e, "device work failed");
        if (timeout_ms >= 0) {
            auto ms =
                std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
            if (ms >= timeout_ms) return fail(h, FC_LBM_ERR_TIMEOUT, "timed out waiting for the device");
        }
        std::this_thread::sleep_for(std::chrono::microseconds(sleep_us));
        sleep_us = std::min(sleep_us * 2, 500);
    }
}

bool params_ok(const fc_params* p) {
    return p && std::isfinite(p->tau) && std::isfinite(p->inlet_velocity) && std::isfinite(p->smagorinsky_cs) &&
           p->tau > 0.5f && p->smagorinsky_cs >= 0.0f;
}

fc::StepParams step_params(const fc_lbm* h) {
    fc::StepParams s{};
    const fc_params& p = h->params;
    s.tau = p.tau;
    s.cs = p.smagorinsky_cs;
    s.reverse = p.reverse_flow != 0;
    s.inlet_x = s.reverse ? h->g.nx - 1 : 0;  // LbmReference.cpp:253-255
    s.outlet_x = s.reverse ? 0 : h->g.nx - 1;
    s.inlet_ux = s.reverse ? -p.inlet_velocity : p.inlet_velocity;
    s.slip_y = p.free_slip_y != 0;
    s.slip_z = p.free_slip_z != 0;
    // Equilibrium(dir, rho = 1, ux = inlet_ux, 0, 0) as LbmReference.cpp:9-13
    // computes it (host code is built without FMA contraction).
    for (int i = 0; i < 19; ++i) s.feq_inlet[i] = 0.0f;
    for (int i = 0; i < h->q; ++i) {
        int ex, ey, ez;
        float w;
        if (h->q == 19) {
            ex = fc::Lattice<19>::ex(i), ey = fc::Lattice<19>::ey(i), ez = fc::Lattice<19>::ez(i);
            w = fc::Lattice<19>::w(i);
        } else {
            ex = fc::Lattice<15>::ex(i), ey = fc::Lattice<15>::ey(i), ez = fc::Lattice<15>::ez(i);
            w = fc::Lattice<15>::w(i);
        }
        const float rho = 1.0f, ux = s.inlet_ux, uy = 0.0f, uz = 0.0f;
        const float eu = (float)ex * ux + (float)ey * uy + (float)ez * uz;
        const float u2 = ux * ux + uy * uy + uz * uz;
        s.feq_inlet[i] = w * rho * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * u2);
    }
    return s;
}

void release(fc_lbm* h) {
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->rb_stream) {
        cudaStreamSynchronize(h->rb_stream);
        cudaStreamDestroy(h->rb_stream);
        h->rb_stream = nullptr;
    }
    if (h->ev_snap) cudaEventDestroy(h->ev_snap);
    if (h->ev_rb) cudaEventDestroy(h->ev_rb);
    h->ev_snap = h->ev_rb = nullptr;
    h->rb_pending = false;
    h->snap_set = -1;
    dfree(h->d_snap);
    if (h->pop[1] == h->pop[0]) h->pop[1] = nullptr;  // one in-place set
    dfree(h->pop[0]);
    dfree(h->pop[1]);
    dfree(h->d_solid);
    dfree(h->d_sdf);
    dfree(h->d_bulk_bits);
    dfree(h->d_cells);
    dfree(h->d_links);
    dfree(h->d_coef_off);
    dfree(h->d_coef);
    dfree(h->d_diverged);
    dfree(h->d_stats_partials);
    dfree(h->d_stats_result);
    dfree(h->d_aero_partials);
    dfree(h->d_aero_result);
    dfree(h->d_closure);
    dfree(h->d_closure_tc);
    dfree(h->d_wall);
    dfree(h->d_aa_bz);
    dfree(h->d_aa_outm);
    dfree(h->parts.trail);
    dfree(h->parts.head);
    dfree(h->parts.len);
    dfree(h->d_part_io);
    dfree(h->d_part_lens);
    h->parts.count = h->parts.length = 0;
    h->closure_on = false;
    dfree(h->d_stage);
    if (h->h_stage) cudaFreeHost(h->h_stage);
    h->h_stage = nullptr;
    if (h->ev_own) cudaEventDestroy(h->ev_own);
    if (h->ev_foreign) cudaEventDestroy(h->ev_foreign);
    if (h->ev_sync) cudaEventDestroy(h->ev_sync);
    h->ev_own = h->ev_foreign = h->ev_sync = nullptr;
    if (h->stream) cudaStreamDestroy(h->stream);
    h->stream = nullptr;
    h->z_begin.clear();
    h->solid_cpu.clear();
    h->solid_cpu.shrink_to_fit();
    h->n_bnd = h->n_bz = h->n_bulk = 0;
    h->valid = false;
    h->cur = 0;
    h->steps_since_reset = 0;
}

// Copies `bytes` from host or device memory into device memory, staging host
// data through the pinned buffer.
int upload(fc_lbm* h, void* dst, const void* src, size_t bytes, bool src_device) {
    if (src_device) {
        FC_TRY(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, h->stream), "copy geometry");
        return FC_LBM_OK;
    }
    const size_t chunk = h->stage_floats * sizeof(float);
    for (size_t off = 0; off < bytes; off += chunk) {
        const size_t nb = std::min(chunk, bytes - off);
        FC_RC(wait_stream(h, kTransferTimeoutMs));
        std::memcpy(h->h_stage, (const char*)src + off, nb);
        FC_TRY(h, cudaMemcpyAsync((char*)dst + off, h->h_stage, nb, cudaMemcpyHostToDevice, h->stream),
               "upload geometry");
    }
    return wait_stream(h, kTransferTimeoutMs);
}

// Classifies every cell and builds the boundary list (see lbm_setup.cu).
int build_boundary(fc_lbm* h) {
    const Geom& g = h->g;
    struct Temp {
        uint8_t* flags = nullptr;
        unsigned long long* counts = nullptr;
        uint32_t* sel_count = nullptr;
        uint32_t* nbz = nullptr;
        void* cub = nullptr;
        ~Temp() {
            dfree(flags);
            dfree(counts);
            dfree(sel_count);
            dfree(nbz);
            if (cub) cudaFree(cub);
        }
    } t;
    FC_TRY(h, cudaMalloc(&t.flags, g.n), "alloc classify flags");
    FC_TRY(h, cudaMalloc(&t.counts, 2 * sizeof(unsigned long long)), "alloc counters");
    FC_TRY(h, cudaMalloc(&t.sel_count, sizeof(uint32_t)), "alloc counter");
    FC_TRY(h, cudaMemsetAsync(t.counts, 0, 2 * sizeof(unsigned long long), h->stream), "clear counters");
    FC_TRY(h, fc::launch_classify(h->q, h->d_solid, g, t.flags, h->d_bulk_bits, t.counts, h->stream), "classify");
    h->launches++;
    unsigned long long counts[2] = {0, 0};
    FC_TRY(h, cudaMemcpyAsync(h->h_stage, t.counts, sizeof(counts), cudaMemcpyDeviceToHost, h->stream), "read counts");
    FC_RC(wait_stream(h, kTransferTimeoutMs));
    std::memcpy(counts, h->h_stage, sizeof(counts));
    h->n_bnd = (size_t)counts[0];
    h->n_bulk = (size_t)counts[1];

    h->z_begin.assign((size_t)g.nz + 1, 0);
    if (h->n_bnd == 0) return FC_LBM_OK;

    FC_TRY(h, cudaMalloc(&h->d_cells, h->n_bnd * sizeof(uint32_t)), "alloc boundary list");
    size_t cub_bytes = 0, scan_bytes = 0;
    FC_TRY(h, fc::select_flagged_cells(nullptr, cub_bytes, t.flags, h->d_cells, t.sel_count, g.n, h->stream),
           "select sizing");
    FC_TRY(h, fc::exclusive_scan_u32(nullptr, scan_bytes, nullptr, nullptr, h->n_bnd, h->stream), "scan sizing");
    cub_bytes = std::max(cub_bytes, scan_bytes);
    FC_TRY(h, cudaMalloc(&t.cub, cub_bytes), "alloc select temp");
    FC_TRY(h, fc::select_flagged_cells(t.cub, cub_bytes, t.flags, h->d_cells, t.sel_count, g.n, h->stream),
           "select boundary cells");
    dfree(t.flags);  // 1 byte per cell, no longer needed

    FC_TRY(h, cudaMalloc(&h->d_links, h->n_bnd * sizeof(unsigned long long)), "alloc links");
    FC_TRY(h, cudaMalloc(&h->d_coef_off, h->n_bnd * sizeof(uint32_t)), "alloc coefficient offsets");
    FC_TRY(h, cudaMalloc(&t.nbz, h->n_bnd * sizeof(uint32_t)), "alloc link counts");
    FC_TRY(h, fc::launch_links(h->q, h->d_cells, h->n_bnd, h->d_solid, h->d_sdf, g, h->d_links, t.nbz, nullptr,
                               nullptr, h->stream),
           "resolve links");
    FC_TRY(h, fc::exclusive_scan_u32(t.cub, cub_bytes, t.nbz, h->d_coef_off, h->n_bnd, h->stream), "scan links");
    uint32_t tail[2] = {0, 0};
    FC_TRY(h, cudaMemcpyAsync(h->h_stage, h->d_coef_off + (h->n_bnd - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost,
                              h->stream),
           "read link total");
    FC_TRY(h, cudaMemcpyAsync((char*)h->h_stage + 4, t.nbz + (h->n_bnd - 1), sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, h->stream),
           "read link total");
    FC_RC(wait_stream(h, kTransferTimeoutMs));
    std::memcpy(tail, h->h_stage, sizeof(tail));
    h->n_bz = (size_t)tail[0] + tail[1];
    if (h->n_bz > 0) {
        FC_TRY(h, cudaMalloc(&h->d_coef, h->n_bz * sizeof(float2)), "alloc Bouzidi coefficients");
        FC_TRY(h, fc::launch_links(h->q, h->d_cells, h->n_bnd, h->d_solid, h->d_sdf, g, h->d_links, nullptr,
                                   h->d_coef_off, h->d_coef, h->stream),
               "fill Bouzidi coefficients");
    }
    uint32_t* d_zb = nullptr;
    FC_TRY(h, cudaMalloc(&d_zb, ((size_t)g.nz + 1) * sizeof(uint32_t)), "alloc z offsets");
    cudaError_t e = fc::launch_z_offsets(h->d_cells, h->n_bnd, g, d_zb, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->h_stage, d_zb, ((size_t)g.nz + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            h->stream);
    int rc = e == cudaSuccess ? wait_stream(h, kTransferTimeoutMs) : cuda_fail(h, e, "z offsets");
    if (rc == FC_LBM_OK) std::memcpy(h->z_begin.data(), h->h_stage, ((size_t)g.nz + 1) * sizeof(uint32_t));
    cudaFree(d_zb);
    h->launches += 4;
    return rc;
}

// Orders work on a caller's stream after the handle's stream (and back).
int enter_stream(fc_lbm* h, cudaStream_t s) {
    if (s == h->stream) return FC_LBM_OK;
    FC_TRY(h, cudaEventRecord(h->ev_own, h->stream), "order streams");
    FC_TRY(h, cudaStreamWaitEvent(s, h->ev_own, 0), "order streams");
    return FC_LBM_OK;
}
int leave_stream(fc_lbm* h, cudaStream_t s) {
    if (s == h->stream) return FC_LBM_OK;
    FC_TRY(h, cudaEventRecord(h->ev_foreign, s), "order streams");
    FC_TRY(h, cudaStreamWaitEvent(h->stream, h->ev_foreign, 0), "order streams");
    return FC_LBM_OK;
}

bool in_place(const fc_lbm* h) { return h->streaming == FC_STREAMING_AA; }

// Where the current state's populations sit (aa.cuh PopLayout).
int layout_of(const fc_lbm* h) { return in_place(h) ? fc::aa_layout(h->cur) : fc::kLayoutPlanes; }

fc::AaSide aa_side(const fc_lbm* h) { return fc::AaSide{h->d_aa_bz, h->d_aa_outm, (size_t)h->g.ny * h->g.nz}; }

fc::BoundaryList boundary_list(const fc_lbm* h) {
    return fc::BoundaryList{h->d_cells, h->d_links, h->d_coef_off, h->d_coef};
}

// After a seed or a population load of an in-place lattice: the side
// buffers from the new state.
int aa_prime(fc_lbm* h) {
    if (!in_place(h)) return FC_LBM_OK;
    FC_TRY(h, fc::launch_aa_prime(h->q, h->storage, h->pop[0], boundary_list(h), (uint32_t)h->n_bnd, h->g, aa_side(h),
                                  h->cur, h->stream),
           "prime in-place side buffers");
    h->launches += 2;
    return FC_LBM_OK;
}

// Work on stream s that overwrites population set `set` waits until a
// pending asynchronous readback's snapshot kernel has read it.
int guard_snapshot(fc_lbm* h, cudaStream_t s, int set) {
    if (h->rb_pending && (in_place(h) || set == h->snap_set))
        FC_TRY(h, cudaStreamWaitEvent(s, h->ev_snap, 0), "order after readback snapshot");
    return FC_LBM_OK;
}

// The two step kernels, with or without the learned closure, ping-pong or in place.
cudaError_t launch_bulk(fc_lbm* h, const fc::StepParams& p, const void* fin, void* fout, int z0, int zc,
                        cudaStream_t s, int* nl) {
    if (in_place(h) && h->closure_on)
        return fc::launch_bulk_aa_learned(h->q, h->storage, h->pop[0], h->d_bulk_bits, h->g, p, z0, zc,
                                          h->d_diverged, s, nl, h->cur, aa_side(h), h->closure);
    if (in_place(h))
        return fc::launch_bulk_aa(h->q, h->storage, h->pop[0], h->d_bulk_bits, h->g, p, z0, zc, h->d_diverged, s, nl,
                                  h->cur, aa_side(h));
    if (h->closure_on)
        return fc::launch_bulk_pull_learned(h->q, h->storage, fin, fout, h->d_bulk_bits, h->g, p, z0, zc,
                                            h->d_diverged, s, nl, h->closure,
                                            (h->flags & FC_OPTION_TC_CLOSURE) ? 1 : 0);
    return fc::launch_bulk_pull(h->q, h->storage, fin, fout, h->d_bulk_bits, h->g, p, z0, zc, h->d_diverged, s, nl,
                                (h->flags & FC_OPTION_TMA_STAGING) ? 1 : 0);
}

cudaError_t launch_boundary(fc_lbm* h, const fc::StepParams& p, const void* fin, void* fout, uint32_t b, uint32_t e,
                            cudaStream_t s) {
    const fc::BoundaryList bl = boundary_list(h);
    if (in_place(h) && h->closure_on)
        return fc::launch_boundary_aa_learned(h->q, h->storage, h->pop[0], bl, b, e, h->g, p, h->d_diverged, s,
                                              h->cur, aa_side(h), h->closure);
    if (in_place(h))
        return fc::launch_boundary_aa(h->q, h->storage, h->pop[0], bl, b, e, h->g, p, h->d_diverged, s, h->cur,
                                      aa_side(h));
    if (h->closure_on)
        return fc::launch_boundary_pull_learned(h->q, h->storage, fin, fout, bl, b, e, h->g, p, h->d_diverged, s,
                                                h->closure);
    return fc::launch_boundary_pull(h->q, h->storage, fin, fout, bl, b, e, h->g, p, h->d_diverged, s);
}

int step_range_on(fc_lbm* h, cudaStream_t s, int z0, int zc) {
    const int z1 = std::min(h->g.nz, z0 + zc);
    z0 = std::max(0, z0);
    if (z1 <= z0) return FC_LBM_OK;
    const fc::StepParams p = step_params(h);
    const void* fin = h->pop[h->cur];
    void* fout = h->pop[1 - h->cur];
    FC_RC(guard_snapshot(h, s, 1 - h->cur));
    if (h->n_bulk > 0) {
        int nl = 0;
        FC_TRY(h, launch_bulk(h, p, fin, fout, z0, z1 - z0, s, &nl), "bulk step");
        h->launches += nl;
    }
    const uint32_t b = h->z_begin[(size_t)z0], e = h->z_begin[(size_t)z1];
    if (e > b) {
        FC_TRY(h, launch_boundary(h, p, fin, fout, b, e, s), "boundary step");
        h->launches++;
    }
    return FC_LBM_OK;
}

int check_ready(fc_lbm* h) {
    if (!h) return FC_LBM_ERR_INVALID_ARG;
    if (!h->valid) return fail(h, FC_LBM_ERR_NOT_INITIALIZED, "solver not initialized");
    return FC_LBM_OK;
}

// Macroscopic field of cells [cell0, cell0 + cells) into host memory `out`
// (4 floats per cell), chunked through the staging buffers.
int field_to_host(fc_lbm* h, size_t cell0, size_t cells, float* out) {
    const size_t chunk = h->stage_floats / 4;
    for (size_t done = 0; done < cells; done += chunk) {
        const size_t nc = std::min(chunk, cells - done);
        FC_TRY(h, fc::launch_field(h->q, h->storage, h->pop[h->cur], h->d_solid, h->d_sdf, h->g, cell0 + done, nc,
                                   h->d_stage, layout_of(h), h->stream),
               "field kernel");
        h->launches++;
        FC_TRY(h, cudaMemcpyAsync(h->h_stage, h->d_stage, nc * 4 * sizeof(float), cudaMemcpyDeviceToHost, h->stream),
               "field download");
        FC_RC(wait_stream(h, kTransferTimeoutMs));
        std::memcpy(out + (cell0 + done) * 4, h->h_stage, nc * 4 * sizeof(float));
    }
    return FC_LBM_OK;
}

}  // namespace

extern "C" {

int fc_lbm_create(fc_lbm** out) {
    if (!out) return FC_LBM_ERR_INVALID_ARG;
    *out = new (std::nothrow) fc_lbm();
    return *out ? FC_LBM_OK : FC_LBM_ERR_OUT_OF_MEMORY;
}

void fc_lbm_destroy(fc_lbm* h) {
    if (!h) return;
    if (h->valid || h->stream) {
        DeviceGuard dg(h->device);
        release(h);
    }
    delete h;
}

const char* fc_lbm_last_error(const fc_lbm* h) { return h ? h->err.c_str() : "null handle"; }

int fc_lbm_shutdown(fc_lbm* h) {
    if (!h) return FC_LBM_ERR_INVALID_ARG;
    DeviceGuard dg(h->device);
    release(h);
    return FC_LBM_OK;
}

int fc_lbm_init(fc_lbm* h, const fc_grid_desc* grid, int32_t model, const fc_options* opts) {
    if (!h) return FC_LBM_ERR_INVALID_ARG;
    {
        DeviceGuard dg(h->device);
        release(h);  // LbmSolver::Init starts with Shutdown (LbmSolver.cpp:206)
    }
    h->err.clear();
    if (!grid || !grid->solid) return fail(h, FC_LBM_ERR_INVALID_ARG, "grid and grid->solid are required");
    if (grid->nx <= 0 || grid->ny <= 0 || grid->nz <= 0)
        return fail(h, FC_LBM_ERR_INVALID_ARG, "grid dimensions must be positive");
    if (model != FC_LATTICE_D3Q15 && model != FC_LATTICE_D3Q19)
        return fail(h, FC_LBM_ERR_INVALID_ARG, "unknown lattice model");
    fc_options o{0, FC_STORAGE_FP32, FC_STREAMING_PINGPONG, 0};
    if (opts) o = *opts;
    if (o.storage < FC_STORAGE_FP32 || o.storage > FC_STORAGE_BF16_OFFSET)
        return fail(h, FC_LBM_ERR_INVALID_ARG, "unknown storage format");
    if (o.streaming != FC_STREAMING_PINGPONG && o.streaming != FC_STREAMING_AA)
        return fail(h, FC_LBM_ERR_INVALID_ARG, "unknown streaming mode");
    if (o.flags & ~(FC_OPTION_TMA_STAGING | FC_OPTION_TC_CLOSURE))
        return fail(h, FC_LBM_ERR_INVALID_ARG, "unknown option flags");
    if (o.streaming == FC_STREAMING_AA && (grid->nx % 2 != 0 || grid->nx < 4))
        return fail(h, FC_LBM_ERR_UNSUPPORTED, "AA (in-place) streaming needs an even nx of at least 4");
    const size_t n = (size_t)grid->nx * (size_t)grid->ny * (size_t)grid->nz;
    if (n >= (size_t(1) << 32))
        return fail(h, FC_LBM_ERR_INVALID_ARG, "grid too large: at most 2^32-1 cells per lattice");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(h, FC_LBM_ERR_CUDA, "no CUDA device available");
    if (o.device < 0 || o.device >= ndev) return fail(h, FC_LBM_ERR_INVALID_ARG, "device ordinal out of range");

    h->device = o.device;
    DeviceGuard dg(h->device);
    h->model = model;
    h->q = model == FC_LATTICE_D3Q19 ? 19 : 15;
    h->storage = o.storage;
    h->streaming = o.streaming;
    h->flags = o.flags;
    h->g.nx = grid->nx;
    h->g.ny = grid->ny;
    h->g.nz = grid->nz;
    h->g.wpr = (grid->nx + 31) / 32;
    h->cell_size = grid->cell_size;
    for (int k = 0; k < 3; ++k) h->origin[k] = grid->origin[k];
    h->g.nxy = (long long)grid->nx * grid->ny;
    h->g.n = n;

    const size_t elem = h->storage == FC_STORAGE_FP32 ? 4 : 2;
    const size_t pop_bytes = (size_t)h->q * n * elem;
    const size_t bits_bytes = (size_t)grid->ny * grid->nz * h->g.wpr * sizeof(uint32_t);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        const size_t sets = o.streaming == FC_STREAMING_AA ? 1 : 2;
        const size_t need = sets * pop_bytes + n * (1 + (grid->signed_distance ? 4 : 0)) + bits_bytes + n /*flags*/;
        if (need > free_b) {
            char buf[256];
            std::snprintf(buf, sizeof(buf), "grid too large: %zu cells need %.2f GiB of device memory, %.2f GiB free",
                          n, need / 1073741824.0, free_b / 1073741824.0);
            return fail(h, FC_LBM_ERR_OUT_OF_MEMORY, buf);
        }
    }

    auto init_body = [&]() -> int {
        FC_TRY(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "create stream");
        FC_TRY(h, cudaEventCreateWithFlags(&h->ev_own, cudaEventDisableTiming), "create event");
        FC_TRY(h, cudaEventCreateWithFlags(&h->ev_foreign, cudaEventDisableTiming), "create event");
        FC_TRY(h, cudaEventCreateWithFlags(&h->ev_sync, cudaEventDisableTiming), "create event");
        h->stage_floats = kStageFloats;
        FC_TRY(h, cudaMalloc(&h->d_stage, h->stage_floats * sizeof(float)), "alloc staging");
        FC_TRY(h, cudaMallocHost(&h->h_stage, h->stage_floats * sizeof(float)), "alloc pinned staging");
        FC_TRY(h, cudaMalloc(&h->pop[0], pop_bytes), "alloc populations");
        if (in_place(h))
            h->pop[1] = h->pop[0];  // readbacks use pop[cur] under either scheme
        else
            FC_TRY(h, cudaMalloc(&h->pop[1], pop_bytes), "alloc populations");
        FC_TRY(h, cudaMalloc(&h->d_solid, n), "alloc solid mask");
        if (grid->signed_distance) FC_TRY(h, cudaMalloc(&h->d_sdf, n * sizeof(float)), "alloc SDF");
        FC_TRY(h, cudaMalloc(&h->d_bulk_bits, bits_bytes), "alloc bulk mask");
        FC_TRY(h, cudaMalloc(&h->d_diverged, sizeof(int)), "alloc divergence flag");
        h->stats_blocks = fc::stats_blocks(h->g);
        FC_TRY(h, cudaMalloc(&h->d_stats_partials, (size_t)h->stats_blocks * fc::kStatsSlots * sizeof(double)),
               "alloc stats partials");
        FC_TRY(h, cudaMalloc(&h->d_stats_result, fc::kStatsSlots * sizeof(double)), "alloc stats result");
        FC_TRY(h, cudaMalloc(&h->d_aero_partials, (size_t)h->stats_blocks * fc::kAeroSlots * sizeof(double)),
               "alloc force partials");
        FC_TRY(h, cudaMalloc(&h->d_aero_result, fc::kAeroResult * sizeof(double)), "alloc force result");
        FC_TRY(h, cudaMemsetAsync(h->d_diverged, 0, sizeof(int), h->stream), "clear flag");
        const bool dev = grid->memory == FC_MEMORY_DEVICE;
        FC_RC(upload(h, h->d_solid, grid->solid, n, dev));
        if (grid->signed_distance) FC_RC(upload(h, h->d_sdf, grid->signed_distance, n * sizeof(float), dev));
        FC_RC(build_boundary(h));
        if (in_place(h)) {
            FC_TRY(h, cudaMalloc(&h->d_aa_bz, std::max<size_t>(h->n_bz, 1) * elem), "alloc in-place link buffer");
            FC_TRY(h, cudaMalloc(&h->d_aa_outm, 4 * (size_t)grid->ny * grid->nz * sizeof(float4)),
                   "alloc in-place outlet buffer");
        }
        h->solid_cpu.resize(n);
        if (dev) {
            FC_TRY(h, cudaMemcpy(h->solid_cpu.data(), grid->solid, n, cudaMemcpyDeviceToHost), "copy solid mask");
        } else {
            std::memcpy(h->solid_cpu.data(), grid->solid, n);
        }
        // A defined state before the first Reset: quiescent equilibrium.
        h->cur = 0;
        FC_TRY(h, fc::launch_seed_uniform(h->q, h->storage, h->pop[0], h->g, 1.0f, 0.0f, 0.0f, 0.0f, layout_of(h),
                                          h->stream),
               "seed");
        h->launches++;
        FC_RC(aa_prime(h));
        return wait_stream(h, kTransferTimeoutMs);
    };
    int rc = init_body();
    if (rc != FC_LBM_OK) {
        std::string keep = h->err;
        release(h);
        h->err = keep;
        return rc;
    }
    h->cur = 0;
    h->steps_since_reset = 0;
    h->valid = true;
    return FC_LBM_OK;
}

int fc_lbm_reset(fc_lbm* h, const fc_params* params, int32_t seed_mid) {
    FC_RC(check_ready(h));
    if (!params_ok(params)) return fail(h, FC_LBM_ERR_INVALID_ARG, "invalid params (tau must exceed 0.5, Cs >= 0)");
    DeviceGuard dg(h->device);
    h->params = *params;
    // LbmReference::Reset / LbmSolver::Reset seed (LbmReference.cpp:193-202).
    float rho = 1.0f, ux = 0.0f;
    if (seed_mid) {
        const float u = h->params.inlet_velocity;
        const float mid = 0.5f * u;
        ux = h->params.reverse_flow ? -mid : mid;
        const float dev = 0.5f * (u * u - mid * mid);
        rho = 1.0f + 3.0f * dev;
    }
    h->cur = 0;
    FC_RC(guard_snapshot(h, h->stream, 0));
    FC_TRY(h, fc::launch_seed_uniform(h->q, h->storage, h->pop[0], h->g, rho, ux, 0.0f, 0.0f, layout_of(h), h->stream),
           "seed");
    FC_TRY(h, cudaMemsetAsync(h->d_diverged, 0, sizeof(int), h->stream), "clear flag");
    h->launches++;
    FC_RC(aa_prime(h));
    h->steps_since_reset = 0;
    return FC_LBM_OK;
}

int fc_lbm_reset_from_field(fc_lbm* h, const float* field, size_t count) {
    FC_RC(check_ready(h));
    if (!field || count != h->g.n * 4)
        return fail(h, FC_LBM_ERR_INVALID_ARG, "field must hold exactly 4 floats per cell");
    DeviceGuard dg(h->device);
    h->cur = 0;
    FC_RC(guard_snapshot(h, h->stream, 0));
    const size_t chunk = h->stage_floats / 4;
    for (size_t c0 = 0; c0 < h->g.n; c0 += chunk) {
        const size_t nc = std::min(chunk, h->g.n - c0);
        FC_RC(wait_stream(h, kTransferTimeoutMs));
        std::memcpy(h->h_stage, field + c0 * 4, nc * 4 * sizeof(float));
        FC_TRY(h, cudaMemcpyAsync(h->d_stage, h->h_stage, nc * 4 * sizeof(float), cudaMemcpyHostToDevice, h->stream),
               "field upload");
        FC_TRY(h, fc::launch_seed_field(h->q, h->storage, h->pop[0], h->g, h->d_stage, h->d_solid, c0, nc,
                                        layout_of(h), h->stream),
               "seed from field");
        h->launches++;
    }
    FC_TRY(h, cudaMemsetAsync(h->d_diverged, 0, sizeof(int), h->stream), "clear flag");
    FC_RC(aa_prime(h));
    h->steps_since_reset = 0;
    return wait_stream(h, kTransferTimeoutMs);
}

int fc_lbm_set_params(fc_lbm* h, const fc_params* params) {
    if (!h) return FC_LBM_ERR_INVALID_ARG;
    if (!params_ok(params)) return fail(h, FC_LBM_ERR_INVALID_ARG, "invalid params (tau must exceed 0.5, Cs >= 0)");
    h->params = *params;
    return FC_LBM_OK;
}

int fc_lbm_get_params(const fc_lbm* h, fc_params* out) {
    if (!h || !out) return FC_LBM_ERR_INVALID_ARG;
    *out = h->params;
    return FC_LBM_OK;
}

int fc_lbm_step(fc_lbm* h, void* stream, int32_t n) {
    FC_RC(check_ready(h));
    if (n < 0) return fail(h, FC_LBM_ERR_INVALID_ARG, "negative step count");
    DeviceGuard dg(h->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    FC_RC(enter_stream(h, s));
    for (int k = 0; k < n; ++k) {
        FC_RC(step_range_on(h, s, 0, h->g.nz));
        h->cur = 1 - h->cur;
        h->steps_since_reset++;
    }
    return leave_stream(h, s);
}

int fc_lbm_step_range(fc_lbm* h, void* stream, int32_t z_start, int32_t z_count) {
    FC_RC(check_ready(h));
    DeviceGuard dg(h->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    FC_RC(enter_stream(h, s));
    FC_RC(step_range_on(h, s, z_start, z_count));
    return leave_stream(h, s);
}

int fc_lbm_advance_substep(fc_lbm* h) {
    FC_RC(check_ready(h));
    h->cur = 1 - h->cur;
    h->steps_since_reset++;
    return FC_LBM_OK;
}

int fc_lbm_readback_field(fc_lbm* h, float* out, size_t count) {
    FC_RC(check_ready(h));
    if (!out || count != h->g.n * 4) return fail(h, FC_LBM_ERR_INVALID_ARG, "output must hold 4 floats per cell");
    DeviceGuard dg(h->device);
    return field_to_host(h, 0, h->g.n, out);
}

int fc_lbm_readback_field_range(fc_lbm* h, int32_t z_start, int32_t z_count, float* out, size_t count) {
    FC_RC(check_ready(h));
    if (!out || count != h->g.n * 4) return fail(h, FC_LBM_ERR_INVALID_ARG, "output must hold 4 floats per cell");
    const int z1 = std::min(h->g.nz, z_start + z_count);
    const int z0 = std::max(0, z_start);
    if (z1 <= z0) return FC_LBM_OK;
    DeviceGuard dg(h->device);
    return field_to_host(h, (size_t)z0 * h->g.nxy, (size_t)(z1 - z0) * h->g.nxy, out);
}

int fc_lbm_readback_stats(fc_lbm* h, fc_stats* out) {
    FC_RC(check_ready(h));
    if (!out) return FC_LBM_ERR_INVALID_ARG;
    DeviceGuard dg(h->device);
    FC_TRY(h, fc::launch_stats(h->q, h->storage, h->pop[h->cur], h->d_solid, h->d_sdf, h->g, h->d_stats_partials,
                               h->stats_blocks, h->d_stats_result, layout_of(h), h->stream),
           "stats kernel");
    h->launches += 2;
    FC_TRY(h, cudaMemcpyAsync(h->h_stage, h->d_stats_result, fc::kStatsSlots * sizeof(double), cudaMemcpyDeviceToHost,
                              h->stream),
           "stats download");
    FC_RC(wait_stream(h, kTransferTimeoutMs));
    double r[fc::kStatsSlots];
    std::memcpy(r, h->h_stage, sizeof(r));
    std::memset(out, 0, sizeof(*out));
    const double fluid = r[6];
    out->fluid_cells = (uint64_t)fluid;
    out->density_sum = r[0];
    out->speed_sum = r[1];
    out->total_mass = r[2];
    out->force_sum[0] = r[3];
    out->force_sum[1] = r[4];
    out->force_sum[2] = r[5];
    if (fluid > 0) {
        out->avg_density = (float)(r[0] / fluid);
        out->avg_speed = (float)(r[1] / fluid);
        out->min_density = (float)r[7];
        out->max_density = (float)r[8];
    }
    out->max_speed = (float)r[9];
    out->max_stress = (float)r[10];
    out->force_x = (float)r[3];
    out->force_y = (float)r[4];
    out->force_z = (float)r[5];
    out->has_nan = r[11] != 0.0;
    out->valid = 1;
    return FC_LBM_OK;
}

int fc_lbm_aero_forces(fc_lbm* h, fc_aero_forces* out) {
    FC_RC(check_ready(h));
    if (!out) return FC_LBM_ERR_INVALID_ARG;
    DeviceGuard dg(h->device);
    FC_TRY(h, fc::launch_aero(h->q, h->storage, h->pop[h->cur], h->d_solid, h->d_sdf, h->g, h->cell_size,
                              h->origin[0], h->origin[1], h->origin[2], h->d_aero_partials, h->stats_blocks,
                              h->d_aero_result, layout_of(h), h->stream),
           "force kernel");
    h->launches += 2;
    FC_TRY(h, cudaMemcpyAsync(h->h_stage, h->d_aero_result, fc::kAeroResult * sizeof(double), cudaMemcpyDeviceToHost,
                              h->stream),
           "force download");
    FC_RC(wait_stream(h, kTransferTimeoutMs));
    double r[fc::kAeroResult];
    std::memcpy(r, h->h_stage, sizeof(r));
    std::memset(out, 0, sizeof(*out));
    for (int k = 0; k < 3; ++k) {
        out->force_sum[k] = r[k];
        out->force[k] = (float)r[k];
        out->center_of_pressure[k] = (float)r[9 + k];
        out->lift_arrow_base[k] = (float)r[12 + k];
    }
    out->lift_weight_sum = r[3];
    out->force_weight_sum = r[4];
    out->solid_cells = (uint64_t)r[5];
    out->min_stress = (float)r[6];
    out->max_stress = (float)r[7];
    out->has_nan = r[8] != 0.0;
    return FC_LBM_OK;
}

int fc_lbm_set_closure(fc_lbm* h, const fc_closure* c) {
    FC_RC(check_ready(h));
    if (!c) {
        h->closure_on = false;
        return FC_LBM_OK;
    }
    if (h->storage == FC_STORAGE_FP32)
        return fail(h, FC_LBM_ERR_UNSUPPORTED, "the learned closure runs on the FP16/BF16 offset storage formats");
    if (h->g.nx % 2 != 0) return fail(h, FC_LBM_ERR_UNSUPPORTED, "the learned closure needs an even nx");
    if (!c->w1 || !c->b1 || !c->w2 || !c->b2 || !c->w3)
        return fail(h, FC_LBM_ERR_INVALID_ARG, "closure weights missing");
    bool ok = std::isfinite(c->b3) && std::isfinite(c->out_scale) && c->out_scale > 0.0f &&
              std::isfinite(c->filter_width);
    for (int k = 0; k < FC_CLOSURE_INPUTS; ++k) ok = ok && std::isfinite(c->mean[k]) && c->std[k] > 0.0f;
    for (int k = 0; k < 3; ++k) ok = ok && !(c->lo[k] > c->hi[k]);
    ok = ok && std::isfinite(c->min_wall_distance) && c->min_wall_distance >= 0.0f && std::isfinite(c->trust_factor) &&
         (c->trust_factor == 0.0f || c->trust_factor >= 1.0f);
    const int H = FC_CLOSURE_HIDDEN;
    for (int i = 0; i < FC_CLOSURE_INPUTS * H && ok; ++i) ok = std::isfinite(c->w1[i]);
    for (int i = 0; i < H * H && ok; ++i) ok = std::isfinite(c->w2[i]);
    for (int i = 0; i < H && ok; ++i)
        ok = std::isfinite(c->b1[i]) && std::isfinite(c->b2[i]) && std::isfinite(c->w3[i]);
    if (!ok)
        return fail(h, FC_LBM_ERR_INVALID_ARG,
                    "closure parameters must be finite, with std > 0, out_scale > 0, min_wall_distance >= 0 and "
                    "trust_factor 0 or >= 1");
    DeviceGuard dg(h->device);
    if (!h->d_wall) {
        uint8_t* tmp = nullptr;
        FC_TRY(h, cudaMalloc(&h->d_wall, h->g.n), "alloc wall distance");
        cudaError_t e = cudaMalloc(&tmp, h->g.n);
        if (e == cudaSuccess) e = fc::launch_wall_distance(h->d_solid, h->g, h->d_wall, tmp, h->stream);
        const int rc = e == cudaSuccess ? wait_stream(h, kTransferTimeoutMs) : cuda_fail(h, e, "wall distance");
        if (tmp) cudaFree(tmp);
        if (rc != FC_LBM_OK) {
            dfree(h->d_wall);
            return rc;
        }
    }
    if (!h->d_closure) FC_TRY(h, cudaMalloc(&h->d_closure, fc::kClosureVec * sizeof(uint4)), "alloc closure");
    if (!h->d_closure_tc) FC_TRY(h, cudaMalloc(&h->d_closure_tc, fc::kTcWeightBytes), "alloc closure");
    std::vector<uint4> frag(fc::kClosureVec);
    fc::pack_closure(c->w1, c->b1, c->w2, c->b2, c->w3, c->b3, c->out_scale, frag.data());
    std::vector<uint4> tcw(fc::kTcWeightBytes / sizeof(uint4));
    fc::pack_closure_tc(c->w1, c->b1, c->w2, c->b2, c->w3, c->out_scale, reinterpret_cast<uint8_t*>(tcw.data()));
    // ordered after any step already queued on the solver's stream
    FC_TRY(h, cudaMemcpyAsync(h->d_closure, frag.data(), frag.size() * sizeof(uint4), cudaMemcpyHostToDevice,
                              h->stream),
           "upload closure");
    FC_TRY(h, cudaMemcpyAsync(h->d_closure_tc, tcw.data(), fc::kTcWeightBytes, cudaMemcpyHostToDevice, h->stream),
           "upload closure");
    FC_RC(wait_stream(h, kTransferTimeoutMs));
    fc::ClosureDev cd{};
    cd.frag = h->d_closure;
    cd.tcw = h->d_closure_tc;
    cd.b3 = c->b3 * c->out_scale;  // as the fragment image folds it
    cd.wall = h->d_wall;
    for (int k = 0; k < FC_CLOSURE_INPUTS; ++k) {
        cd.mean[k] = c->mean[k];
        cd.inv_std[k] = 1.0f / c->std[k];
    }
    for (int k = 0; k < 3; ++k) {
        cd.lo[k] = c->lo[k];
        cd.hi[k] = c->hi[k];
    }
    cd.filter_width = c->filter_width;
    // the wall-distance bytes count 1/16 cells; a cell keeps Smagorinsky below this byte
    const float wm = std::ceil(c->min_wall_distance * 16.0f);
    cd.wall_min = wm > 255.0f ? 256u : (unsigned)wm;
    cd.trust = c->trust_factor;
    cd.inv_trust = c->trust_factor > 0.0f ? 1.0f / c->trust_factor : 0.0f;
    h->closure = cd;
    h->closure_on = true;
    return FC_LBM_OK;
}

int fc_lbm_closure_samples(fc_lbm* h, float filter_width, float* out, int64_t capacity, int64_t* count) {
    FC_RC(check_ready(h));
    if (!count || capacity < 0 || !std::isfinite(filter_width)) return FC_LBM_ERR_INVALID_ARG;
    if (in_place(h)) return fail(h, FC_LBM_ERR_UNSUPPORTED, "closure samples need ping-pong streaming");
    DeviceGuard dg(h->device);
    FC_RC(wait_stream(h, kTransferTimeoutMs));  // every queued step first
    // the molecular relaxation time of the 2x coarser lattice (nu halves)
    const float tau_c = 0.5f + 0.5f * (h->params.tau - 0.5f);
    const int rc = fc::closure_samples(h->q, h->storage, h->pop[h->cur], h->d_solid, h->g, h->params.tau,
                                       h->params.smagorinsky_cs, tau_c, filter_width, out, capacity, count, h->stream);
    h->launches += 5;
    if (rc != FC_LBM_OK && rc != FC_LBM_ERR_TOO_LARGE) return fail(h, rc, "closure samples failed");
    return rc;
}

int fc_lbm_closure_probe(fc_lbm* h, float* out, uint8_t* in_range, size_t cells) {
    FC_RC(check_ready(h));
    if (!h->closure_on) return fail(h, FC_LBM_ERR_NOT_INITIALIZED, "no learned closure set");
    if (!out || !in_range || cells != h->g.n) return FC_LBM_ERR_INVALID_ARG;
    DeviceGuard dg(h->device);
    float* d_out = nullptr;
    uint8_t* d_rng = nullptr;
    FC_TRY(h, cudaMalloc(&d_out, h->g.n * 5 * sizeof(float)), "alloc probe");
    cudaError_t e = cudaMalloc(&d_rng, h->g.n);
    if (e == cudaSuccess)
        e = fc::launch_closure_probe(h->q, h->storage, h->pop[h->cur], h->d_solid, h->g, h->closure, d_out, d_rng,
                                     nullptr, layout_of(h), h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, d_out, h->g.n * 5 * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(in_range, d_rng, h->g.n, cudaMemcpyDeviceToHost, h->stream);
    const int rc = e == cudaSuccess ? wait_stream(h, kTransferTimeoutMs) : cuda_fail(h, e, "closure probe");
    cudaFree(d_out);
    if (d_rng) cudaFree(d_rng);
    h->launches++;
    return rc;
}

int fc_lbm_closure_coverage(fc_lbm* h, uint64_t* cells_in_range, uint64_t* warps_with_mlp) {
    FC_RC(check_ready(h));
    if (!h->closure_on) return fail(h, FC_LBM_ERR_NOT_INITIALIZED, "no learned closure set");
    if (!cells_in_range || !warps_with_mlp) return FC_LBM_ERR_INVALID_ARG;
    DeviceGuard dg(h->device);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(h->d_stats_result);  // 2 slots, reused
    FC_TRY(h, cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), h->stream), "clear counts");
    FC_TRY(h, fc::launch_closure_probe(h->q, h->storage, h->pop[h->cur], h->d_solid, h->g, h->closure, nullptr,
                                       nullptr, d, layout_of(h), h->stream),
           "closure coverage");
    h->launches++;
    FC_TRY(h, cudaMemcpyAsync(h->h_stage, d, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream),
           "coverage download");
    FC_RC(wait_stream(h, kTransferTimeoutMs));
    unsigned long long r[2];
    std::memcpy(r, h->h_stage, sizeof(r));
    *cells_in_range = r[0];
    *warps_with_mlp = r[1];
    return FC_LBM_OK;
}

int fc_lbm_wall_distance(fc_lbm* h, uint8_t* out, size_t cells) {
    FC_RC(check_ready(h));
    if (!out || cells != h->g.n) return FC_LBM_ERR_INVALID_ARG;
    DeviceGuard dg(h->device);
    uint8_t* d = h->d_wall;
    uint8_t* own = nullptr;
    uint8_t* tmp = nullptr;
    cudaError_t e = cudaSuccess;
    if (!d) {
        e = cudaMalloc(&own, h->g.n);
        if (e == cudaSuccess) e = cudaMalloc(&tmp, h->g.n);
        if (e == cudaSuccess) e = fc::launch_wall_distance(h->d_solid, h->g, own, tmp, h->stream);
        d = own;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, h->g.n, cudaMemcpyDeviceToHost, h->stream);
    const int rc = e == cudaSuccess ? wait_stream(h, kTransferTimeoutMs) : cuda_fail(h, e, "wall distance");
    if (own) cudaFree(own);
    if (tmp) cudaFree(tmp);
    return rc;
}

int fc_lbm_layer_copy(fc_lbm* h, int32_t z, int32_t next, void* buffer, int32_t to_buffer, void* stream) {
    FC_RC(check_ready(h));
    if (!buffer || z < 0 || z >= h->g.nz) return FC_LBM_ERR_INVALID_ARG;
    if (in_place(h)) return fail(h, FC_LBM_ERR_UNSUPPORTED, "layer copies need ping-pong streaming");
    DeviceGuard dg(h->device);
    const size_t elem = h->storage == FC_STORAGE_FP32 ? 4 : 2;
    const size_t width = (size_t)h->g.nxy * elem, pitch = h->g.n * elem;
    char* pop = static_cast<char*>(h->pop[next ? 1 - h->cur : h->cur]) + (size_t)z * width;
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    FC_RC(enter_stream(h, s));
    if (!to_buffer) FC_RC(guard_snapshot(h, s, next ? 1 - h->cur : h->cur));
    // one strided copy: Q planes of one layer <-> Q contiguous rows
    const cudaError_t e = to_buffer ? cudaMemcpy2DAsync(buffer, width, pop, pitch, width, (size_t)h->q,
                                                        cudaMemcpyDeviceToDevice, s)
                                    : cudaMemcpy2DAsync(pop, pitch, buffer, width, width, (size_t)h->q,
                                                        cudaMemcpyDeviceToDevice, s);
    FC_TRY(h, e, "layer copy");
    return leave_stream(h, s);
}

int fc_lbm_layer_copy_dir(fc_lbm* h, int32_t z, int32_t next, void* buffer, int32_t to_buffer, int32_t ez,
                          void* stream) {
    if (ez == 0) return fc_lbm_layer_copy(h, z, next, buffer, to_buffer, stream);
    FC_RC(check_ready(h));
    if (!buffer || z < 0 || z >= h->g.nz || (ez != 1 && ez != -1)) return FC_LBM_ERR_INVALID_ARG;
    if (in_place(h)) return fail(h, FC_LBM_ERR_UNSUPPORTED, "layer copies need ping-pong streaming");
    DeviceGuard dg(h->device);
    const size_t elem = h->storage == FC_STORAGE_FP32 ? 4 : 2;
    const size_t width = (size_t)h->g.nxy * elem, pitch = h->g.n * elem;
    char* pop = static_cast<char*>(h->pop[next ? 1 - h->cur : h->cur]) + (size_t)z * width;
    char* buf = static_cast<char*>(buffer);
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    FC_RC(enter_stream(h, s));
    if (!to_buffer) FC_RC(guard_snapshot(h, s, next ? 1 - h->cur : h->cur));
    // one copy per plane with that e_z: FC_LBM_DIR_PLANES contiguous rows
    int row = 0;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < h->q && e == cudaSuccess; ++i) {
        const int eiz = h->q == 19 ? fc::Lattice<19>::ez(i) : fc::Lattice<15>::ez(i);
        if (eiz != ez) continue;
        char* plane = pop + (size_t)i * pitch;
        char* r = buf + (size_t)row * width;
        e = to_buffer ? cudaMemcpyAsync(r, plane, width, cudaMemcpyDeviceToDevice, s)
                      : cudaMemcpyAsync(plane, r, width, cudaMemcpyDeviceToDevice, s);
        ++row;
    }
    FC_TRY(h, e, "layer copy");
    if (row != FC_LBM_DIR_PLANES) return fail(h, FC_LBM_ERR_CUDA, "unexpected plane count per e_z");
    return leave_stream(h, s);
}

int fc_lbm_probe_slice_health(fc_lbm* h, int32_t z, int32_t* diverged) {
    FC_RC(check_ready(h));
    if (!diverged) return FC_LBM_ERR_INVALID_ARG;
    DeviceGuard dg(h->device);
    const int gz = std::min(std::max(z, 0), h->g.nz - 1);  // LbmSolver.cpp:655
    const size_t layer = (size_t)h->g.nxy;
    // the layer's field values and the reference's checks on them
    // (LbmSolver.cpp:699-716), evaluated on the device: one flag comes back
    int* d_flag = reinterpret_cast<int*>(h->d_stage);
    FC_TRY(h, cudaMemsetAsync(d_flag, 0, sizeof(int), h->stream), "clear probe flag");
    FC_TRY(h, fc::launch_probe_health(h->q, h->storage, h->pop[h->cur], h->d_solid, h->d_sdf, h->g,
                                      (size_t)gz * layer, layer, d_flag, layout_of(h), h->stream),
           "probe kernel");
    h->launches++;
    FC_TRY(h, cudaMemcpyAsync(h->h_stage, d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "probe download");
    FC_RC(wait_stream(h, kTransferTimeoutMs));
    *diverged = *reinterpret_cast<const int*>(h->h_stage) != 0 ? 1 : 0;
    return FC_LBM_OK;
}

int fc_lbm_has_diverged(fc_lbm* h, int32_t* diverged) {
    FC_RC(check_ready(h));
    if (!diverged) return FC_LBM_ERR_INVALID_ARG;
    DeviceGuard dg(h->device);
    FC_TRY(h, cudaMemcpyAsync(h->h_stage, h->d_diverged, sizeof(int), cudaMemcpyDeviceToHost, h->stream),
           "flag download");
    FC_RC(wait_stream(h, kTransferTimeoutMs));
    int v = 0;
    std::memcpy(&v, h->h_stage, sizeof(int));
    *diverged = v != 0;
    return FC_LBM_OK;
}

int fc_lbm_copy_solid_mask(const fc_lbm* h, uint8_t* out, size_t count) {
    if (!h || !out) return FC_LBM_ERR_INVALID_ARG;
    if (!h->valid) return FC_LBM_ERR_NOT_INITIALIZED;
    if (count != h->solid_cpu.size()) return FC_LBM_ERR_INVALID_ARG;
    std::memcpy(out, h->solid_cpu.data(), count);
    return FC_LBM_OK;
}

int fc_lbm_is_valid(const fc_lbm* h) { return h && h->valid ? 1 : 0; }

int fc_lbm_model(const fc_lbm* h) { return h ? h->model : FC_LBM_ERR_INVALID_ARG; }

int fc_lbm_dims(const fc_lbm* h, int32_t* nx, int32_t* ny, int32_t* nz) {
    if (!h) return FC_LBM_ERR_INVALID_ARG;
    if (nx) *nx = h->valid ? h->g.nx : 0;
    if (ny) *ny = h->valid ? h->g.ny : 0;
    if (nz) *nz = h->valid ? h->g.nz : 0;
    return FC_LBM_OK;
}

int fc_lbm_sync(fc_lbm* h, int32_t timeout_ms) {
    FC_RC(check_ready(h));
    DeviceGuard dg(h->device);
    return wait_stream(h, timeout_ms);
}

int fc_lbm_get_stream(const fc_lbm* h, void** stream) {
    if (!h || !stream) return FC_LBM_ERR_INVALID_ARG;
    if (!h->valid) return FC_LBM_ERR_NOT_INITIALIZED;
    *stream = (void*)h->stream;
    return FC_LBM_OK;
}

int fc_lbm_boundary_info(const fc_lbm* h, uint64_t* boundary_cells, uint64_t* bouzidi_links, uint64_t* bulk_cells) {
    if (!h) return FC_LBM_ERR_INVALID_ARG;
    if (boundary_cells) *boundary_cells = h->n_bnd;
    if (bouzidi_links) *bouzidi_links = h->n_bz;
    if (bulk_cells) *bulk_cells = h->n_bulk;
    return FC_LBM_OK;
}

int fc_lbm_step_timed(fc_lbm* h, int32_t n, float* total_ms, float* bulk_ms, float* boundary_ms) {
    FC_RC(check_ready(h));
    if (n < 0) return fail(h, FC_LBM_ERR_INVALID_ARG, "negative step count");
    DeviceGuard dg(h->device);
    std::vector<cudaEvent_t> ev((size_t)n * 4 + 2, nullptr);
    auto destroy = [&]() {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    };
    for (cudaEvent_t& e : ev) {
        cudaError_t ce = cudaEventCreate(&e);
        if (ce != cudaSuccess) {
            destroy();
            return cuda_fail(h, ce, "create timing event");
        }
    }
    const uint32_t b = h->z_begin[0], e = h->z_begin[(size_t)h->g.nz];
    int rc = FC_LBM_OK;
    cudaEventRecord(ev[0], h->stream);
    for (int k = 0; k < n && rc == FC_LBM_OK; ++k) {
        const fc::StepParams p = step_params(h);
        const void* fin = h->pop[h->cur];
        void* fout = h->pop[1 - h->cur];
        rc = guard_snapshot(h, h->stream, 1 - h->cur);
        if (rc != FC_LBM_OK) break;
        cudaEventRecord(ev[2 + 4 * k], h->stream);
        cudaError_t ce = cudaSuccess;
        if (h->n_bulk > 0) {
            int nl = 0;
            ce = launch_bulk(h, p, fin, fout, 0, h->g.nz, h->stream, &nl);
            h->launches += nl;
        }
        cudaEventRecord(ev[3 + 4 * k], h->stream);
        cudaEventRecord(ev[4 + 4 * k], h->stream);
        if (ce == cudaSuccess && e > b) {
            ce = launch_boundary(h, p, fin, fout, b, e, h->stream);
            h->launches++;
        }
        cudaEventRecord(ev[5 + 4 * k], h->stream);
        if (ce != cudaSuccess) rc = cuda_fail(h, ce, "timed step");
        h->cur = 1 - h->cur;
        h->steps_since_reset++;
    }
    cudaEventRecord(ev[1], h->stream);
    if (rc == FC_LBM_OK) rc = wait_stream(h, kTransferTimeoutMs);
    if (rc == FC_LBM_OK) {
        float t = 0.0f, tb = 0.0f, td = 0.0f, x = 0.0f;
        cudaEventElapsedTime(&t, ev[0], ev[1]);
        for (int k = 0; k < n; ++k) {
            cudaEventElapsedTime(&x, ev[2 + 4 * k], ev[3 + 4 * k]);
            tb += x;
            cudaEventElapsedTime(&x, ev[4 + 4 * k], ev[5 + 4 * k]);
            td += x;
        }
        if (total_ms) *total_ms = t;
        if (bulk_ms) *bulk_ms = tb;
        if (boundary_ms) *boundary_ms = td;
    }
    destroy();
    return rc;
}

int fc_lbm_launch_count(const fc_lbm* h, uint64_t* launches) {
    if (!h || !launches) return FC_LBM_ERR_INVALID_ARG;
    *launches = h->launches;
    return FC_LBM_OK;
}

int fc_lbm_save_populations(fc_lbm* h, float* out, size_t count) {
    FC_RC(check_ready(h));
    if (!out || count != (size_t)h->q * h->g.n)
        return fail(h, FC_LBM_ERR_INVALID_ARG, "output must hold Q floats per cell");
    DeviceGuard dg(h->device);
    const size_t chunk = h->stage_floats / (size_t)h->q;
    const int solid_w = h->steps_since_reset > 0 ? 1 : 0;
    for (size_t c0 = 0; c0 < h->g.n; c0 += chunk) {
        const size_t nc = std::min(chunk, h->g.n - c0);
        FC_TRY(h, fc::launch_pops_out(h->q, h->storage, h->pop[h->cur], h->d_solid, solid_w, h->g, c0, nc, h->d_stage,
                                      layout_of(h), h->stream),
               "population readout");
        h->launches++;
        FC_TRY(h, cudaMemcpyAsync(h->h_stage, h->d_stage, nc * h->q * sizeof(float), cudaMemcpyDeviceToHost, h->stream),
               "population download");
        FC_RC(wait_stream(h, kTransferTimeoutMs));
        for (int i = 0; i < h->q; ++i)
            std::memcpy(out + (size_t)i * h->g.n + c0, h->h_stage + (size_t)i * nc, nc * sizeof(float));
    }
    return FC_LBM_OK;
}

int fc_lbm_load_populations(fc_lbm* h, const float* in, size_t count) {
    FC_RC(check_ready(h));
    if (!in || count != (size_t)h->q * h->g.n)
        return fail(h, FC_LBM_ERR_INVALID_ARG, "input must hold Q floats per cell");
    DeviceGuard dg(h->device);
    const size_t chunk = h->stage_floats / (size_t)h->q;
    for (size_t c0 = 0; c0 < h->g.n; c0 += chunk) {
        const size_t nc = std::min(chunk, h->g.n - c0);
        FC_RC(wait_stream(h, kTransferTimeoutMs));
        for (int i = 0; i < h->q; ++i)
            std::memcpy(h->h_stage + (size_t)i * nc, in + (size_t)i * h->g.n + c0, nc * sizeof(float));
        FC_TRY(h, cudaMemcpyAsync(h->d_stage, h->h_stage, nc * h->q * sizeof(float), cudaMemcpyHostToDevice, h->stream),
               "population upload");
        FC_RC(guard_snapshot(h, h->stream, h->cur));
        FC_TRY(h, fc::launch_pops_in(h->q, h->storage, h->pop[h->cur], h->g, c0, nc, h->d_stage, layout_of(h),
                                     h->stream),
               "population write");
        h->launches++;
    }
    FC_RC(aa_prime(h));
    // The loaded state is a post-step state: solid cells hold what was given.
    h->steps_since_reset = 0;
    return wait_stream(h, kTransferTimeoutMs);
}

// ---- asynchronous field readback ----
int fc_lbm_readback_field_async(fc_lbm* h, float* out, size_t count) {
    FC_RC(check_ready(h));
    if (!out || count != h->g.n * 4) return fail(h, FC_LBM_ERR_INVALID_ARG, "output must hold 4 floats per cell");
    DeviceGuard dg(h->device);
    if (h->rb_pending) FC_RC(fc_lbm_readback_wait(h, kTransferTimeoutMs));
    if (!h->rb_stream) {
        FC_TRY(h, cudaStreamCreateWithFlags(&h->rb_stream, cudaStreamNonBlocking), "create readback stream");
        FC_TRY(h, cudaEventCreateWithFlags(&h->ev_snap, cudaEventDisableTiming), "create event");
        FC_TRY(h, cudaEventCreateWithFlags(&h->ev_rb, cudaEventDisableTiming), "create event");
    }
    if (!h->d_snap) FC_TRY(h, cudaMalloc(&h->d_snap, h->g.n * 4 * sizeof(float)), "alloc readback snapshot");
    // the snapshot reads the state every step queued so far leaves
    FC_TRY(h, cudaEventRecord(h->ev_own, h->stream), "order readback");
    FC_TRY(h, cudaStreamWaitEvent(h->rb_stream, h->ev_own, 0), "order readback");
    FC_TRY(h, fc::launch_field(h->q, h->storage, h->pop[h->cur], h->d_solid, h->d_sdf, h->g, 0, h->g.n, h->d_snap,
                               layout_of(h), h->rb_stream),
           "snapshot field");
    h->launches++;
    FC_TRY(h, cudaEventRecord(h->ev_snap, h->rb_stream), "snapshot event");
    h->snap_set = in_place(h) ? 0 : h->cur;
    h->rb_pending = true;
    FC_TRY(h, cudaMemcpyAsync(out, h->d_snap, h->g.n * 4 * sizeof(float), cudaMemcpyDeviceToHost, h->rb_stream),
           "field download");
    FC_TRY(h, cudaEventRecord(h->ev_rb, h->rb_stream), "readback event");
    return FC_LBM_OK;
}

int fc_lbm_readback_wait(fc_lbm* h, int32_t timeout_ms) {
    FC_RC(check_ready(h));
    if (!h->rb_pending) return FC_LBM_OK;
    DeviceGuard dg(h->device);
    auto t0 = std::chrono::steady_clock::now();
    int sleep_us = 5;
    for (;;) {
        const cudaError_t e = cudaEventQuery(h->ev_rb);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) return cuda_fail(h, e, "readback failed");
        if (timeout_ms >= 0 &&
            std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count() >=
                timeout_ms)
            return fail(h, FC_LBM_ERR_TIMEOUT, "timed out waiting for the readback");
        std::this_thread::sleep_for(std::chrono::microseconds(sleep_us));
        sleep_us = std::min(sleep_us * 2, 500);
    }
    h->rb_pending = false;
    h->snap_set = -1;
    return FC_LBM_OK;
}

int fc_lbm_alloc_pinned(size_t bytes, void** out) {
    if (!out) return FC_LBM_ERR_INVALID_ARG;
    *out = nullptr;
    const cudaError_t e = cudaMallocHost(out, bytes);
    if (e == cudaErrorMemoryAllocation) return FC_LBM_ERR_OUT_OF_MEMORY;
    return e == cudaSuccess ? FC_LBM_OK : FC_LBM_ERR_CUDA;
}

int fc_lbm_free_pinned(void* p) {
    if (!p) return FC_LBM_OK;
    return cudaFreeHost(p) == cudaSuccess ? FC_LBM_OK : FC_LBM_ERR_CUDA;
}

// ---- smoke-trail particles (SmokeTrailSystem, FlowCraft/SmokeTrail.h:26-184) ----
}  // extern "C"

namespace {

fc::SmokeParams smoke_params(const fc_lbm* h, int32_t confine_axis, int32_t confine_index) {
    fc::SmokeParams sp{};
    sp.ox = h->origin[0];
    sp.oy = h->origin[1];
    sp.oz = h->origin[2];
    sp.cs = h->cell_size;
    sp.confine_axis = confine_axis >= 0 && confine_axis <= 2 ? confine_axis : -1;
    sp.confine_index = confine_index;
    sp.seed = h->part_seed;
    sp.counter = h->part_counter;
    return sp;
}

// Draws one particle may take in one call: 8 attempts x 3 axes + 3 jitters.
constexpr unsigned long long kDrawsPerCall = 32;

}  // namespace

extern "C" {

int fc_lbm_particles_reset(fc_lbm* h, int32_t count, int32_t trail_length, uint64_t seed, int32_t confine_axis,
                           int32_t confine_index) {
    FC_RC(check_ready(h));
    if (count < 0 || count > (1 << 26)) return fail(h, FC_LBM_ERR_INVALID_ARG, "particle count out of range");
    DeviceGuard dg(h->device);
    const int length = std::max(trail_length, 2);  // SmokeTrail.cpp:259
    if ((long long)count * length > (1ll << 30)) return fail(h, FC_LBM_ERR_INVALID_ARG, "trails too long");
    FC_RC(wait_stream(h, kTransferTimeoutMs));
    dfree(h->parts.trail);
    dfree(h->parts.head);
    dfree(h->parts.len);
    dfree(h->d_part_io);
    dfree(h->d_part_lens);
    h->parts = fc::ParticleSet{nullptr, nullptr, nullptr, count, length};
    if (count > 0) {
        FC_TRY(h, cudaMalloc(&h->parts.trail, (size_t)count * length * sizeof(float4)), "alloc particle trails");
        FC_TRY(h, cudaMalloc(&h->parts.head, (size_t)count * sizeof(int)), "alloc particles");
        FC_TRY(h, cudaMalloc(&h->parts.len, (size_t)count * sizeof(int)), "alloc particles");
        FC_TRY(h, cudaMalloc(&h->d_part_io, (size_t)count * length * 3 * sizeof(float)), "alloc particle readout");
        FC_TRY(h, cudaMalloc(&h->d_part_lens, (size_t)count * sizeof(int)), "alloc particle readout");
    }
    h->part_seed = seed;
    h->part_counter = 0;
    // Reset scatters over the whole domain (SmokeTrail.cpp:257-276)
    FC_TRY(h, fc::launch_particles_scatter(h->d_solid, h->g, h->parts, smoke_params(h, confine_axis, confine_index),
                                           h->stream),
           "scatter particles");
    h->part_counter += kDrawsPerCall;
    h->launches++;
    return FC_LBM_OK;
}

int fc_lbm_particles_step(fc_lbm* h, int32_t reverse_flow, float mm_per_sec_per_lattice_unit, float dt_seconds,
                          int32_t suspend_respawn, int32_t confine_axis, int32_t confine_index) {
    FC_RC(check_ready(h));
    if (!std::isfinite(mm_per_sec_per_lattice_unit) || !std::isfinite(dt_seconds)) return FC_LBM_ERR_INVALID_ARG;
    if (h->parts.count == 0 || dt_seconds <= 0.0f) return FC_LBM_OK;  // SmokeTrail.cpp:281
    DeviceGuard dg(h->device);
    fc::SmokeParams sp = smoke_params(h, confine_axis, confine_index);
    sp.reverse = reverse_flow != 0;
    sp.suspend = suspend_respawn != 0;
    const float dt = std::min(dt_seconds, 0.1f);  // kMaxDtSeconds, SmokeTrail.cpp:296-297
    sp.scale = mm_per_sec_per_lattice_unit * dt;
    FC_TRY(h, fc::launch_particles_step(h->q, h->storage, h->pop[h->cur], layout_of(h), h->d_solid, h->g, h->parts,
                                        sp, h->stream),
           "advect particles");
    h->part_counter += kDrawsPerCall;
    h->launches++;
    return FC_LBM_OK;
}

int fc_lbm_particles_scatter(fc_lbm* h, int32_t confine_axis, int32_t confine_index) {
    FC_RC(check_ready(h));
    DeviceGuard dg(h->device);
    FC_TRY(h, fc::launch_particles_scatter(h->d_solid, h->g, h->parts, smoke_params(h, confine_axis, confine_index),
                                           h->stream),
           "scatter particles");
    h->part_counter += kDrawsPerCall;
    h->launches++;
    return FC_LBM_OK;
}

int fc_lbm_particles_shift_plane(fc_lbm* h, int32_t confine_axis, int32_t confine_index) {
    FC_RC(check_ready(h));
    if (confine_axis < 0 || confine_axis > 2) return FC_LBM_ERR_INVALID_ARG;
    DeviceGuard dg(h->device);
    FC_TRY(h, fc::launch_particles_shift(h->g, h->parts, smoke_params(h, confine_axis, confine_index), h->stream),
           "shift particles");
    h->launches++;
    return FC_LBM_OK;
}

int fc_lbm_particles_read(fc_lbm* h, float* points, size_t points_count, int32_t* lens, size_t lens_count) {
    FC_RC(check_ready(h));
    const size_t np = (size_t)h->parts.count, nl = (size_t)h->parts.length;
    if (!points || !lens || points_count != np * nl * 3 || lens_count != np) return FC_LBM_ERR_INVALID_ARG;
    if (np == 0) return FC_LBM_OK;
    DeviceGuard dg(h->device);
    FC_TRY(h, fc::launch_particles_gather(h->parts, h->d_part_io, h->d_part_lens, h->stream), "gather trails");
    h->launches++;
    FC_TRY(h, cudaMemcpyAsync(points, h->d_part_io, np * nl * 3 * sizeof(float), cudaMemcpyDeviceToHost, h->stream),
           "trail download");
    FC_TRY(h, cudaMemcpyAsync(lens, h->d_part_lens, np * sizeof(int), cudaMemcpyDeviceToHost, h->stream),
           "trail download");
    return wait_stream(h, kTransferTimeoutMs);
}

int fc_lbm_particles_set(fc_lbm* h, const float* points, size_t points_count) {
    FC_RC(check_ready(h));
    const size_t np = (size_t)h->parts.count;
    if (!points || points_count != np * 3) return FC_LBM_ERR_INVALID_ARG;
    if (np == 0) return FC_LBM_OK;
    DeviceGuard dg(h->device);
    FC_TRY(h, cudaMemcpyAsync(h->d_part_io, points, np * 3 * sizeof(float), cudaMemcpyHostToDevice, h->stream),
           "position upload");
    FC_TRY(h, fc::launch_particles_set(h->parts, h->d_part_io, h->stream), "set particles");
    h->launches++;
    return wait_stream(h, kTransferTimeoutMs);
}

// ---- batches: many lattices stepped together (fc_lbm_batch) ----
}  // extern "C"

struct fc_lbm_batch {
    std::vector<fc_lbm*> m;
    int device = 0, q = 19, storage = FC_STORAGE_FP32, model = FC_LATTICE_D3Q19;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    fc::BatchLattice* d_lat = nullptr;
    std::vector<fc::BatchLattice> h_lat;
    // grid_mult 0: the one-block-per-tile launches of each step parity
    std::vector<fc::TileLaunch> tiles[2];
    unsigned long long total = 0;   // bulk work items
    unsigned long long btotal = 0;  // boundary-list entries
    int rows = 8, mult = 1, grid = 0;  // rows 0: every member's own bulk launch
    cudaGraphExec_t exec = nullptr;
    // forked streams of the per-member bulk launches (rows 0)
    static constexpr int kFork = 4;
    cudaStream_t fork[kFork] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kFork] = {};
    std::vector<uint64_t> sig;  // member state the descriptors and the graph were built for
    std::string err;
};

namespace {

// The autotuner's candidates, in the order of fc_lbm_batch_tune's times: the
// persistent launch's block shapes, the one-block-per-tile launch, then every
// member's own bulk kernel.
constexpr int kBatchCand[FC_LBM_BATCH_CANDIDATES][2] = {{4, 1}, {4, 2}, {8, 1}, {8, 2}, {16, 1}, {16, 2},
                                                      {8, 0}, {0, 1}};

int bfail(fc_lbm_batch* b, int code, const std::string& msg) {
    b->err = msg;
    return code;
}

int bcuda(fc_lbm_batch* b, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return FC_LBM_OK;
    return bfail(b, e == cudaErrorMemoryAllocation ? FC_LBM_ERR_OUT_OF_MEMORY : FC_LBM_ERR_CUDA,
                 std::string(what) + ": " + cudaGetErrorName(e));
}

#define FB_TRY(b, expr, what)                          \
    do {                                               \
        const int _rc = bcuda((b), (expr), (what));    \
        if (_rc != FC_LBM_OK) return _rc;              \
    } while (0)

uint64_t fbits64(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

std::vector<uint64_t> batch_signature(const fc_lbm_batch* b) {
    std::vector<uint64_t> v{(uint64_t)b->rows, (uint64_t)b->mult};
    for (const fc_lbm* h : b->m) {
        v.push_back((uint64_t)(uintptr_t)h->pop[0]);
        v.push_back((uint64_t)(uintptr_t)h->pop[1]);
        v.push_back((uint64_t)h->cur);
        v.push_back(fbits64(h->params.tau) | (fbits64(h->params.inlet_velocity) << 32));
        v.push_back(fbits64(h->params.smagorinsky_cs) | ((uint64_t)h->params.reverse_flow << 32) |
                    ((uint64_t)h->params.free_slip_y << 33) | ((uint64_t)h->params.free_slip_z << 34));
    }
    return v;
}

// Descriptors of every member for the current block shape, uploaded.
int batch_build(fc_lbm_batch* b) {
    const size_t elem = b->storage == FC_STORAGE_FP32 ? 4 : 2;
    b->h_lat.assign(b->m.size(), fc::BatchLattice{});
    unsigned long long first = 0, bfirst = 0;
    for (size_t k = 0; k < b->m.size(); ++k) {
        fc_lbm* h = b->m[k];
        fc::BatchLattice& d = b->h_lat[k];
        d.g = h->g;
        d.p = step_params(h);
        for (int side = 0; side < 2; ++side) {
            const char* in = static_cast<const char*>(h->pop[side]);
            char* out = static_cast<char*>(h->pop[1 - side]);
            for (int i = 0; i < b->q; ++i) {
                const long long off = (long long)(b->q == 19 ? fc::Lattice<19>::ex(i) : fc::Lattice<15>::ex(i)) +
                                      (long long)(b->q == 19 ? fc::Lattice<19>::ey(i) : fc::Lattice<15>::ey(i)) *
                                          h->g.nx +
                                      (long long)(b->q == 19 ? fc::Lattice<19>::ez(i) : fc::Lattice<15>::ez(i)) *
                                          h->g.nxy;
                d.pp[side].src[i] = in + ((long long)i * (long long)h->g.n - off) * (long long)elem;
                d.pp[side].dst[i] = out + (size_t)i * h->g.n * elem;
            }
        }
        d.pop[0] = h->pop[0];
        d.pop[1] = h->pop[1];
        const uint32_t b0 = h->z_begin[0], b1 = h->z_begin[(size_t)h->g.nz];
        d.bl = fc::BoundaryList{h->d_cells ? h->d_cells + b0 : nullptr, h->d_links ? h->d_links + b0 : nullptr,
                                h->d_coef_off ? h->d_coef_off + b0 : nullptr, h->d_coef};
        d.bnd_first = bfirst;
        bfirst += b1 > b0 ? b1 - b0 : 0;
        d.bits = h->d_bulk_bits;
        d.diverged = h->d_diverged;
        const int rows = b->rows ? b->rows : 8;  // rows 0: the work-list is not used
        d.gx = (h->g.nx + 63) / 64;
        d.gy = (h->g.ny + rows - 1) / rows;
        d.first = first;
        d.cur = h->cur;
        first += (unsigned long long)d.gx * d.gy * h->g.nz;
    }
    b->total = first;
    b->btotal = bfirst;
    for (int par = 0; par < 2; ++par) {  // one block per tile: up to 32 lattices per launch
        b->tiles[par].clear();
        if (!b->rows || b->mult != 0) continue;
        for (size_t k = 0; k < b->m.size(); ++k) {
            const fc::BatchLattice& d = b->h_lat[k];
            const unsigned long long n = (unsigned long long)d.gx * d.gy * d.g.nz;
            if (b->tiles[par].empty() || b->tiles[par].back().nlat == fc::kTileLaunchLattices ||
                b->tiles[par].back().tiles + n > 0x7fffffffull) {
                if (n > 0x7fffffffull) return bfail(b, FC_LBM_ERR_UNSUPPORTED, "one block per tile: 2^31 tiles at most");
                b->tiles[par].emplace_back();
                std::memset(&b->tiles[par].back(), 0, sizeof(fc::TileLaunch));
            }
            fc::TileLaunch& t = b->tiles[par].back();
            fc::TileLattice& l = t.l[t.nlat++];
            const int side = d.cur ^ par;
            l.g = d.g;
            l.p = d.p;
            l.pp = d.pp[side];
            l.fin = d.pop[side];
            l.fout = const_cast<void*>(d.pop[side ^ 1]);
            l.bits = d.bits;
            l.diverged = d.diverged;
            l.first = t.tiles;
            l.gx = d.gx;
            l.gy = d.gy;
            t.tiles += (unsigned)n;
        }
    }
    const int resident = fc::bulk_batch_resident(b->q, b->storage, b->rows ? b->rows : 8);
    int sms = 0;
    FB_TRY(b, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device), "SM count");
    if (resident <= 0) return bfail(b, FC_LBM_ERR_CUDA, "batch kernel occupancy query failed");
    b->grid = sms * resident * b->mult;  // 0: one block per work item
    FB_TRY(b, cudaMemcpyAsync(b->d_lat, b->h_lat.data(), b->h_lat.size() * sizeof(fc::BatchLattice),
                              cudaMemcpyHostToDevice, b->stream),
           "upload batch descriptors");
    return FC_LBM_OK;
}

// Every member's own bulk kernel (the launch fc_lbm_step makes), spread over
// the forked streams so that small lattices run side by side, and meanwhile
// the batch's boundary-list launch on the batch stream (it writes only
// boundary-list cells and reads only the input sets, so it shares nothing
// with the bulk kernels); joined back into the batch stream. Under stream
// capture the fork and join become graph dependencies.
int batch_bulk_members(fc_lbm_batch* b, int parity) {
    const int nf = (int)std::min<size_t>(fc_lbm_batch::kFork, b->m.size());
    FB_TRY(b, cudaEventRecord(b->ev_fork, b->stream), "fork event");
    for (int j = 0; j < nf; ++j) FB_TRY(b, cudaStreamWaitEvent(b->fork[j], b->ev_fork, 0), "fork");
    cudaError_t e = cudaSuccess;
    for (size_t k = 0; k < b->m.size() && e == cudaSuccess; ++k) {
        fc_lbm* h = b->m[k];
        if (h->n_bulk == 0) continue;
        const int side = h->cur ^ parity;
        int nl = 0;
        e = launch_bulk(h, step_params(h), h->pop[side], h->pop[1 - side], 0, h->g.nz, b->fork[k % nf], &nl);
    }
    if (e == cudaSuccess)
        e = fc::launch_boundary_batch(b->q, b->storage, b->d_lat, (int)b->m.size(), b->btotal, parity, b->stream);
    // always join, so that a capture can end
    for (int j = 0; j < nf; ++j) {
        const cudaError_t r = cudaEventRecord(b->ev_join[j], b->fork[j]);
        const cudaError_t w = r == cudaSuccess ? cudaStreamWaitEvent(b->stream, b->ev_join[j], 0) : r;
        if (e == cudaSuccess) e = w;
    }
    return bcuda(b, e, "batch member bulk step");
}

// One step of every member (parity relative to the members' current sets).
int batch_step_direct(fc_lbm_batch* b, int parity) {
    if (b->rows == 0)
        return batch_bulk_members(b, parity);  // the boundary launch runs beside the members' bulk kernels
    if (b->mult == 0)
        for (const fc::TileLaunch& t : b->tiles[parity])
            FB_TRY(b, fc::launch_bulk_tiles(b->q, b->storage, t, b->stream), "batch bulk step");
    else
        FB_TRY(b, fc::launch_bulk_batch(b->q, b->storage, b->rows, b->d_lat, (int)b->m.size(), b->total, parity,
                                        b->grid, b->stream),
               "batch bulk step");
    FB_TRY(b, fc::launch_boundary_batch(b->q, b->storage, b->d_lat, (int)b->m.size(), b->btotal, parity, b->stream),
           "batch boundary step");
    return FC_LBM_OK;
}

int batch_prepare(fc_lbm_batch* b, bool want_graph) {
    const std::vector<uint64_t> sig = batch_signature(b);
    if (sig != b->sig) {
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        FC_RC(batch_build(b));
        b->sig = sig;
    }
    if (want_graph && !b->exec) {
        // two steps, one of each parity: a replay leaves every member on its own set
        cudaGraph_t graph = nullptr;
        FB_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        int rc = batch_step_direct(b, 0);
        if (rc == FC_LBM_OK) rc = batch_step_direct(b, 1);
        const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
        if (rc != FC_LBM_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        FB_TRY(b, e, "end capture");
        const cudaError_t ie = cudaGraphInstantiate(&b->exec, graph, 0);
        cudaGraphDestroy(graph);
        FB_TRY(b, ie, "instantiate graph");
    }
    return FC_LBM_OK;
}

// Every call that steps the batch re-checks its members: a member may have
// been shut down, re-initialized or given a learned closure since the batch
// was created, and the batch kernels would then step it with the wrong
// closure or layout instead of reproducing fc_lbm_step.
int batch_check(fc_lbm_batch* b) {
    for (fc_lbm* h : b->m) {
        if (!h->valid || h->device != b->device || h->q != b->q || h->storage != b->storage)
            return bfail(b, FC_LBM_ERR_INVALID_ARG, "a batch member changed (shut down or re-initialized)");
        if (h->closure_on)
            return bfail(b, FC_LBM_ERR_UNSUPPORTED, "a batch member has a learned closure (set after batch create)");
        if (in_place(h) || h->g.nx % 2 != 0)
            return bfail(b, FC_LBM_ERR_UNSUPPORTED, "a batch member was re-initialized with AA streaming or odd nx");
    }
    return FC_LBM_OK;
}

int batch_enter(fc_lbm_batch* b) {
    for (fc_lbm* h : b->m) {
        FB_TRY(b, cudaEventRecord(b->ev, h->stream), "member event");
        FB_TRY(b, cudaStreamWaitEvent(b->stream, b->ev, 0), "wait member");
        if (h->rb_pending) FB_TRY(b, cudaStreamWaitEvent(b->stream, h->ev_snap, 0), "wait member readback snapshot");
    }
    return FC_LBM_OK;
}

int batch_leave(fc_lbm_batch* b) {
    FB_TRY(b, cudaEventRecord(b->ev, b->stream), "batch event");
    for (fc_lbm* h : b->m) FB_TRY(b, cudaStreamWaitEvent(h->stream, b->ev, 0), "member wait");
    return FC_LBM_OK;
}

int batch_wait(fc_lbm_batch* b) {
    FB_TRY(b, cudaEventRecord(b->ev, b->stream), "batch event");
    const auto t0 = std::chrono::steady_clock::now();
    int sleep_us = 20;
    for (;;) {
        const cudaError_t q = cudaEventQuery(b->ev);
        if (q == cudaSuccess) return FC_LBM_OK;
        if (q != cudaErrorNotReady) return bcuda(b, q, "batch wait");
        if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(kTransferTimeoutMs))
            return bfail(b, FC_LBM_ERR_TIMEOUT, "batch wait timed out");
        std::this_thread::sleep_for(std::chrono::microseconds(sleep_us));
        if (sleep_us < 2000) sleep_us *= 2;
    }
}

void batch_advance(fc_lbm_batch* b, int n, uint64_t launches_per_step) {
    for (fc_lbm* h : b->m) {
        if (n & 1) h->cur = 1 - h->cur;
        h->steps_since_reset += (uint64_t)n;
        h->launches += (uint64_t)n * launches_per_step;  // shared launches, counted in every member
    }
}

}  // namespace

extern "C" {

int fc_lbm_batch_create(fc_lbm* const* members, int32_t count, fc_lbm_batch** out) {
    if (!out) return FC_LBM_ERR_INVALID_ARG;
    *out = nullptr;
    if (!members || count <= 0 || count > 4096) return FC_LBM_ERR_INVALID_ARG;
    fc_lbm* h0 = members[0];
    if (!h0 || !h0->valid) return FC_LBM_ERR_NOT_INITIALIZED;
    for (int k = 0; k < count; ++k) {
        fc_lbm* h = members[k];
        if (!h || !h->valid) return FC_LBM_ERR_NOT_INITIALIZED;
        if (h->device != h0->device || h->q != h0->q || h->storage != h0->storage) return FC_LBM_ERR_INVALID_ARG;
        if (h->g.nx % 2 != 0 || h->closure_on || in_place(h)) return FC_LBM_ERR_UNSUPPORTED;
        for (int j = 0; j < k; ++j)
            if (members[j] == h) return FC_LBM_ERR_INVALID_ARG;
    }
    auto* b = new (std::nothrow) fc_lbm_batch();
    if (!b) return FC_LBM_ERR_OUT_OF_MEMORY;
    b->m.assign(members, members + count);
    b->device = h0->device;
    b->q = h0->q;
    b->storage = h0->storage;
    b->model = h0->model;
    DeviceGuard dg(b->device);
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    for (int j = 0; j < fc_lbm_batch::kFork && e == cudaSuccess; ++j) {
        e = cudaStreamCreateWithFlags(&b->fork[j], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join[j], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaMalloc(&b->d_lat, (size_t)count * sizeof(fc::BatchLattice));
    if (e != cudaSuccess) {
        fc_lbm_batch_destroy(b);
        return e == cudaErrorMemoryAllocation ? FC_LBM_ERR_OUT_OF_MEMORY : FC_LBM_ERR_CUDA;
    }
    *out = b;
    return FC_LBM_OK;
}

void fc_lbm_batch_destroy(fc_lbm_batch* b) {
    if (!b) return;
    DeviceGuard dg(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->d_lat) cudaFree(b->d_lat);
    if (b->ev) cudaEventDestroy(b->ev);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    for (int j = 0; j < fc_lbm_batch::kFork; ++j) {
        if (b->fork[j]) {
            cudaStreamSynchronize(b->fork[j]);
            cudaStreamDestroy(b->fork[j]);
        }
        if (b->ev_join[j]) cudaEventDestroy(b->ev_join[j]);
    }
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char* fc_lbm_batch_last_error(const fc_lbm_batch* b) { return b ? b->err.c_str() : "null batch"; }

int fc_lbm_batch_step(fc_lbm_batch* b, int32_t n) {
    if (!b || n < 0) return FC_LBM_ERR_INVALID_ARG;
    FC_RC(batch_check(b));
    if (n == 0) return FC_LBM_OK;
    DeviceGuard dg(b->device);
    FC_RC(batch_enter(b));
    FC_RC(batch_prepare(b, n >= 2));
    for (int k = 0; k + 1 < n; k += 2) FB_TRY(b, cudaGraphLaunch(b->exec, b->stream), "graph launch");
    if (n & 1) FC_RC(batch_step_direct(b, 0));
    batch_advance(b, n, 2);
    return batch_leave(b);
}

int fc_lbm_batch_config(fc_lbm_batch* b, int32_t rows, int32_t grid_mult) {
    if (!b) return FC_LBM_ERR_INVALID_ARG;
    if ((rows != 0 && rows != 4 && rows != 8 && rows != 16) || grid_mult < 0 || grid_mult > 2 ||
        (grid_mult == 0 && rows != 8))
        return bfail(b, FC_LBM_ERR_INVALID_ARG, "rows must be 0, 4, 8 or 16 and grid_mult 1 or 2 (or 0 with rows 8)");
    b->rows = rows;
    b->mult = grid_mult;
    return FC_LBM_OK;
}

int fc_lbm_batch_tune(fc_lbm_batch* b, int32_t steps, int32_t* rows, int32_t* grid_mult, float* ms_per_step) {
    if (!b || steps < 1) return FC_LBM_ERR_INVALID_ARG;
    FC_RC(batch_check(b));
    DeviceGuard dg(b->device);
    const int timed = steps + (steps & 1);  // even: every member ends on its own set
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    FB_TRY(b, cudaEventCreate(&t0), "timing event");
    if (cudaEventCreate(&t1) != cudaSuccess) {
        cudaEventDestroy(t0);
        return bfail(b, FC_LBM_ERR_CUDA, "timing event");
    }
    int rc = batch_enter(b);
    float best = 1e30f;
    int best_r = 8, best_m = 1, idx = 0;
    for (const auto& cand : kBatchCand) {
        const int r = cand[0], mu = cand[1];
        if (rc != FC_LBM_OK) break;
        b->rows = r;
        b->mult = mu;
        rc = batch_prepare(b, false);
        for (int k = 0; k < 2 && rc == FC_LBM_OK; ++k) rc = batch_step_direct(b, k);  // warm-up
        if (rc == FC_LBM_OK) rc = bcuda(b, cudaEventRecord(t0, b->stream), "timing");
        for (int k = 0; k < timed && rc == FC_LBM_OK; ++k) rc = batch_step_direct(b, k & 1);
        if (rc == FC_LBM_OK) rc = bcuda(b, cudaEventRecord(t1, b->stream), "timing");
        if (rc == FC_LBM_OK) rc = batch_wait(b);
        float ms = 0.0f;
        if (rc == FC_LBM_OK) rc = bcuda(b, cudaEventElapsedTime(&ms, t0, t1), "timing");
        const float per = ms / (float)timed;
        if (ms_per_step) ms_per_step[idx] = per;
        if (rc == FC_LBM_OK && per < best) {
            best = per;
            best_r = r;
            best_m = mu;
        }
        ++idx;
        batch_advance(b, timed + 2, 2);
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    b->rows = best_r;
    b->mult = best_m;
    if (rows) *rows = best_r;
    if (grid_mult) *grid_mult = best_m;
    if (rc == FC_LBM_OK) rc = batch_leave(b);
    return rc;
}

}  // extern "C"
