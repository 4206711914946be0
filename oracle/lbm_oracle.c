/*
 * ORACLE — test infrastructure only. Nothing in the product library links,
 * loads or calls this file; only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg use it, and only to check results.
 *
 * A plain-C restatement of FlowCraft's CPU Lattice-Boltzmann step
 * (FlowCraft/LbmReference.cpp) written from the algorithm, compiled twice:
 *   -DFC_REAL_DOUBLE=0  -> float arithmetic, the same IEEE operation order as
 *                          the reference (build with -ffp-contract=off); its
 *                          outputs are pinned bit-for-bit against the
 *                          reference compiled from its own sources and against
 *                          the committed golden fixtures;
 *   -DFC_REAL_DOUBLE=1  -> double arithmetic with exact lattice weights: the
 *                          FP64 error reference every GPU result is measured
 *                          against.
 *
 * Layout (as the reference, FlowCraft/LbmReference.h:134-135):
 *   cell = (z*ny + y)*nx + x,  population i of a cell at f[i*cellCount + cell].
 * Lattice direction order, weights and `opposite` follow
 * FlowCraft/LatticeModel.h:20-64.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#ifndef FC_REAL_DOUBLE
#define FC_REAL_DOUBLE 0
#endif

#if FC_REAL_DOUBLE
typedef double real;
#define K(x) x
#define RSQRT sqrt
#define RFINITE(v) isfinite(v)
#define SYM(name) oracle64_##name
#else
typedef float real;
#define K(x) x##f
#define RSQRT sqrtf
#define RFINITE(v) isfinite(v)
#define SYM(name) oracle32_##name
#endif

#define FC_MAXQ 19

typedef struct {
    float tau;
    float inlet_velocity;
    int32_t reverse_flow;
    int32_t free_slip_y;
    int32_t free_slip_z;
    float smagorinsky_cs;
} oracle_params;

typedef struct {
    double avg_density, min_density, max_density;
    double avg_speed, max_speed;
    double force_x, force_y, force_z;
    double max_stress;
    double total_mass;
    int32_t has_nan;
    int32_t fluid_count_lo; /* fluid cell count (low 31 bits), informational */
} oracle_stats;

typedef struct {
    int nx, ny, nz, q;
    size_t n;             /* cell count */
    int ex[FC_MAXQ], ey[FC_MAXQ], ez[FC_MAXQ], opp[FC_MAXQ];
    int mirror_y[FC_MAXQ], mirror_z[FC_MAXQ];
    real w[FC_MAXQ];
    uint8_t* solid;
    real* sdf;            /* NULL -> plain halfway bounce-back everywhere */
    real* f[2];
    int cur;
    int threads;
    int diverged;
    real tau, inlet_u, cs;
    int reverse, slip_y, slip_z;
    /* learned closure (see SYM(set_closure)); off when closure_on == 0 */
    int closure_on;
    float cw1[5 * 32], cb1[32], cw2[32 * 32], cb2[32], cw3[32], cb3;
    float cmean[5], cinv_std[5], clo[3], chi[3], cfilter;
    int cwall_min;  /* wall-distance byte below which a cell keeps Smagorinsky */
    float ctrust;   /* > 0: 3 nu_t held within [d / ctrust, d * ctrust] of Smagorinsky's d */
    uint8_t* wall;
} oracle_lbm;

/* Lattice tables: FlowCraft/LatticeModel.h:20-43 (D3Q19) and :45-64 (D3Q15).
 * The velocity vectors and the pairing order are what parity depends on. */
static const int kQ19[19][4] = {
    {0, 0, 0, 0},  {1, 0, 0, 2},  {-1, 0, 0, 1}, {0, 1, 0, 4},   {0, -1, 0, 3},  {0, 0, 1, 6},  {0, 0, -1, 5},
    {1, 1, 0, 8},  {-1, -1, 0, 7}, {1, -1, 0, 10}, {-1, 1, 0, 9}, {1, 0, 1, 12},  {-1, 0, -1, 11}, {1, 0, -1, 14},
    {-1, 0, 1, 13}, {0, 1, 1, 16}, {0, -1, -1, 15}, {0, 1, -1, 18}, {0, -1, 1, 17}};
static const int kQ15[15][4] = {
    {0, 0, 0, 0},   {1, 0, 0, 2},   {-1, 0, 0, 1},  {0, 1, 0, 4},   {0, -1, 0, 3},
    {0, 0, 1, 6},   {0, 0, -1, 5},  {1, 1, 1, 8},   {-1, -1, -1, 7}, {1, 1, -1, 10},
    {-1, -1, 1, 9}, {1, -1, 1, 12}, {-1, 1, -1, 11}, {-1, 1, 1, 14}, {1, -1, -1, 13}};

static void setup_lattice(oracle_lbm* o, int q) {
    o->q = q;
    for (int i = 0; i < q; ++i) {
        const int* d = (q == 19) ? kQ19[i] : kQ15[i];
        o->ex[i] = d[0];
        o->ey[i] = d[1];
        o->ez[i] = d[2];
        o->opp[i] = d[3];
        int s = abs(d[0]) + abs(d[1]) + abs(d[2]);
        if (q == 19) {
            o->w[i] = s == 0 ? K(1.0) / K(3.0) : (s == 1 ? K(1.0) / K(18.0) : K(1.0) / K(36.0));
        } else {
            o->w[i] = s == 0 ? K(2.0) / K(9.0) : (s == 1 ? K(1.0) / K(9.0) : K(1.0) / K(72.0));
        }
    }
    /* Reflection tables found by search (LbmReference.cpp:168-183). */
    for (int i = 0; i < q; ++i) {
        o->mirror_y[i] = 0;
        o->mirror_z[i] = 0;
        for (int j = 0; j < q; ++j) {
            if (o->ex[j] == o->ex[i] && o->ey[j] == -o->ey[i] && o->ez[j] == o->ez[i]) o->mirror_y[i] = j;
            if (o->ex[j] == o->ex[i] && o->ey[j] == o->ey[i] && o->ez[j] == -o->ez[i]) o->mirror_z[i] = j;
        }
    }
}

/* Second-order equilibrium, LbmReference.cpp:9-13. Operation order kept:
 * eu = (ex*ux + ey*uy) + ez*uz;  w*rho*(((1 + 3eu) + 4.5eu*eu) - 1.5u2). */
static inline real feq(const oracle_lbm* o, int i, real rho, real ux, real uy, real uz) {
    real eu = (real)o->ex[i] * ux + (real)o->ey[i] * uy + (real)o->ez[i] * uz;
    real u2 = ux * ux + uy * uy + uz * uz;
    return o->w[i] * rho * (K(1.0) + K(3.0) * eu + K(4.5) * eu * eu - K(1.5) * u2);
}

static inline size_t cidx(const oracle_lbm* o, int x, int y, int z) {
    return ((size_t)z * (size_t)o->ny + (size_t)y) * (size_t)o->nx + (size_t)x;
}
static inline int inb(const oracle_lbm* o, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && x < o->nx && y < o->ny && z < o->nz;
}
static inline int is_solid(const oracle_lbm* o, int x, int y, int z) {
    return inb(o, x, y, z) && o->solid[cidx(o, x, y, z)] != 0;
}
#define POP(f, i, c) ((f)[(size_t)(i) * o->n + (c)])

/* Moments of one cell, LbmReference.cpp:43-61 (divide only when rho > 1e-6). */
static void moments(const oracle_lbm* o, const real* f, size_t c, real* rho, real* ux, real* uy, real* uz) {
    real r = K(0.0), a = K(0.0), b = K(0.0), d = K(0.0);
    for (int i = 0; i < o->q; ++i) {
        real fi = POP(f, i, c);
        r += fi;
        a += fi * (real)o->ex[i];
        b += fi * (real)o->ey[i];
        d += fi * (real)o->ez[i];
    }
    if (r > K(1e-6)) {
        a /= r;
        b /= r;
        d /= r;
    }
    *rho = r;
    *ux = a;
    *uy = b;
    *uz = d;
}

/* Bouzidi / Mei-Luo-Shyy interpolated bounce-back for fluid node (x,y,z)
 * whose direction-i upstream neighbour (sx,sy,sz) is solid,
 * LbmReference.cpp:100-122. Falls back to plain f_opp(x) on missing or
 * non-finite SDF, denom <= 1e-4, or (q < 1/2) an unusable further node. */
static real bouzidi(const oracle_lbm* o, const real* f, int x, int y, int z, size_t c, int i, int sx, int sy,
                    int sz) {
    int op = o->opp[i];
    real plain = POP(f, op, c);
    if (!o->sdf) return plain;
    real phi_f = o->sdf[c];
    real phi_s = o->sdf[cidx(o, sx, sy, sz)];
    if (!RFINITE(phi_f) || !RFINITE(phi_s)) return plain;
    real denom = phi_f - phi_s;
    if (!(denom > K(1e-4))) return plain;
    real q = phi_f / denom;
    if (q < K(0.0)) q = K(0.0);
    if (q > K(1.0)) q = K(1.0);
    if (q < K(0.5)) {
        int fx = x + o->ex[i], fy = y + o->ey[i], fz = z + o->ez[i];
        if (!inb(o, fx, fy, fz) || is_solid(o, fx, fy, fz)) return plain;
        return K(2.0) * q * plain + (K(1.0) - K(2.0) * q) * POP(f, op, cidx(o, fx, fy, fz));
    }
    real inv2q = K(1.0) / (K(2.0) * q);
    return inv2q * plain + (K(1.0) - inv2q) * POP(f, i, c);
}

/* Momentum-exchange force on one solid cell, LbmReference.cpp:127-148. */
static void solid_force(const oracle_lbm* o, const real* f, int x, int y, int z, real* stress, real* fxo, real* fyo,
                        real* fzo) {
    real fx = K(0.0), fy = K(0.0), fz = K(0.0), wsum = K(0.0);
    for (int i = 1; i < o->q; ++i) {
        int ax = x + o->ex[i], ay = y + o->ey[i], az = z + o->ez[i];
        if (!inb(o, ax, ay, az) || is_solid(o, ax, ay, az)) continue;
        size_t fc = cidx(o, ax, ay, az);
        real plain = POP(f, o->opp[i], fc);
        real bounced = bouzidi(o, f, ax, ay, az, fc, i, x, y, z);
        real dp = (plain + bounced) - K(2.0) * o->w[i];
        fx -= (real)o->ex[i] * dp;
        fy -= (real)o->ey[i] * dp;
        fz -= (real)o->ez[i] * dp;
        wsum += o->w[i];
    }
    real mag = RSQRT(fx * fx + fy * fy + fz * fz);
    *stress = (wsum > K(0.0)) ? (mag / (K(6.0) * wsum)) : K(0.0);
    *fxo = fx;
    *fyo = fy;
    *fzo = fz;
}

/* ---- z-slab worker pool (the reference forks std::threads per call,
 *      LbmReference.cpp:24-39; a per-call pthread fork/join is the same). ---- */
typedef struct {
    oracle_lbm* o;
    int z0, z1, tid;
    void* ctx;
    void (*body)(oracle_lbm*, int, int, int, void*);
} slab_job;

static void* slab_entry(void* arg) {
    slab_job* j = (slab_job*)arg;
    j->body(j->o, j->z0, j->z1, j->tid, j->ctx);
    return NULL;
}

static int thread_count(const oracle_lbm* o) {
    int t = o->threads;
    if (t <= 0) {
        long c = sysconf(_SC_NPROCESSORS_ONLN);
        t = c > 0 ? (int)c : 1;
    }
    if (t > o->nz) t = o->nz > 0 ? o->nz : 1;
    if (t > 256) t = 256;
    return t;
}

static void parallel_z(oracle_lbm* o, void (*body)(oracle_lbm*, int, int, int, void*), void* ctx) {
    int t = thread_count(o);
    int per = (o->nz + t - 1) / t;
    pthread_t th[256];
    slab_job jobs[256];
    int started = 0;
    for (int k = 0; k < t; ++k) {
        int z0 = k * per, z1 = z0 + per < o->nz ? z0 + per : o->nz;
        if (z0 >= z1) break;
        jobs[k].o = o;
        jobs[k].z0 = z0;
        jobs[k].z1 = z1;
        jobs[k].tid = k;
        jobs[k].ctx = ctx;
        jobs[k].body = body;
        if (t == 1 || pthread_create(&th[k], NULL, slab_entry, &jobs[k]) != 0) {
            slab_entry(&jobs[k]);
            th[k] = 0;
        }
        started = k + 1;
    }
    for (int k = 0; k < started; ++k)
        if (th[k]) pthread_join(th[k], NULL);
}

/* ---- seeding, LbmReference.cpp:192-239 ---- */
typedef struct {
    real rho, ux, uy, uz;
    const float* field;
} seed_ctx;

static void seed_body(oracle_lbm* o, int z0, int z1, int tid, void* vctx) {
    (void)tid;
    seed_ctx* s = (seed_ctx*)vctx;
    size_t layer = (size_t)o->nx * (size_t)o->ny;
    for (size_t c = (size_t)z0 * layer; c < (size_t)z1 * layer; ++c) {
        real rho = s->rho, ux = s->ux, uy = s->uy, uz = s->uz;
        if (s->field) {
            int sol = o->solid[c] != 0;
            rho = sol ? K(1.0) : (real)s->field[c * 4 + 0];
            ux = sol ? K(0.0) : (real)s->field[c * 4 + 1];
            uy = sol ? K(0.0) : (real)s->field[c * 4 + 2];
            uz = sol ? K(0.0) : (real)s->field[c * 4 + 3];
        }
        for (int i = 0; i < o->q; ++i) POP(o->f[0], i, c) = feq(o, i, rho, ux, uy, uz);
    }
}

void SYM(reset)(oracle_lbm* o, int seed_mid) {
    seed_ctx s = {K(1.0), K(0.0), K(0.0), K(0.0), NULL};
    if (seed_mid) {
        /* Bernoulli-consistent mid-speed seed, LbmReference.cpp:194-202. */
        real mid = K(0.5) * o->inlet_u;
        s.ux = o->reverse ? -mid : mid;
        real dev = K(0.5) * (o->inlet_u * o->inlet_u - mid * mid);
        s.rho = K(1.0) + K(3.0) * dev;
    }
    parallel_z(o, seed_body, &s);
    o->cur = 0;
    o->diverged = 0;
}

int SYM(reset_from_field)(oracle_lbm* o, const float* field, size_t count) {
    if (count != o->n * 4) return -1; /* the reference ignores a mis-sized field */
    o->diverged = 0;
    seed_ctx s = {K(1.0), K(0.0), K(0.0), K(0.0), field};
    parallel_z(o, seed_body, &s);
    o->cur = 0;
    return 0;
}

void SYM(set_params)(oracle_lbm* o, const oracle_params* p) {
    o->tau = (real)p->tau;
    o->inlet_u = (real)p->inlet_velocity;
    o->cs = (real)p->smagorinsky_cs;
    o->reverse = p->reverse_flow != 0;
    o->slip_y = p->free_slip_y != 0;
    o->slip_z = p->free_slip_z != 0;
}

oracle_lbm* SYM(create)(int nx, int ny, int nz, int q, const uint8_t* solid, const float* sdf, size_t sdf_count,
                        const oracle_params* p, int seed_mid, int threads) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || (q != 19 && q != 15)) return NULL;
    oracle_lbm* o = (oracle_lbm*)calloc(1, sizeof(oracle_lbm));
    if (!o) return NULL;
    o->nx = nx;
    o->ny = ny;
    o->nz = nz;
    o->n = (size_t)nx * (size_t)ny * (size_t)nz;
    o->threads = threads;
    setup_lattice(o, q);
    o->solid = (uint8_t*)malloc(o->n);
    o->f[0] = (real*)malloc(sizeof(real) * (size_t)q * o->n);
    o->f[1] = (real*)malloc(sizeof(real) * (size_t)q * o->n);
    if (!o->solid || !o->f[0] || !o->f[1]) {
        free(o->solid);
        free(o->f[0]);
        free(o->f[1]);
        free(o);
        return NULL;
    }
    memcpy(o->solid, solid, o->n);
    /* An SDF whose size differs from the grid is treated as absent
     * (LbmReference.cpp:162-166). */
    if (sdf && sdf_count == o->n) {
        o->sdf = (real*)malloc(sizeof(real) * o->n);
        for (size_t c = 0; c < o->n; ++c) o->sdf[c] = (real)sdf[c];
    }
    memset(o->f[1], 0, sizeof(real) * (size_t)q * o->n);
    SYM(set_params)(o, p);
    SYM(reset)(o, seed_mid);
    return o;
}

void SYM(destroy)(oracle_lbm* o) {
    if (!o) return;
    free(o->wall);
    free(o->solid);
    free(o->sdf);
    free(o->f[0]);
    free(o->f[1]);
    free(o);
}

/* ---- learned closure: the CUDA library's closure (closure.cuh) restated ----
 * Distance to the nearest solid cell: 16 Jacobi sweeps of the 3x3x3 chamfer
 * mask (16 / 23 / 28 sixteenths of a cell), capped at 255. */
void SYM(wall_distance)(int nx, int ny, int nz, const uint8_t* solid, uint8_t* out) {
    size_t n = (size_t)nx * ny * nz;
    uint8_t* tmp = (uint8_t*)malloc(n ? n : 1);
    for (size_t c = 0; c < n; ++c) out[c] = solid[c] ? 0 : 255;
    for (int it = 0; it < 16; ++it) {
        const uint8_t* in = (it % 2 == 0) ? out : tmp;
        uint8_t* dst = (it % 2 == 0) ? tmp : out;
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    size_t c = ((size_t)z * ny + y) * nx + x;
                    int best = in[c];
                    if (best == 0) {
                        dst[c] = 0;
                        continue;
                    }
                    for (int dz = -1; dz <= 1; ++dz)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dx = -1; dx <= 1; ++dx) {
                                int xx = x + dx, yy = y + dy, zz = z + dz;
                                int m = (dx != 0) + (dy != 0) + (dz != 0);
                                if (m == 0 || xx < 0 || yy < 0 || zz < 0 || xx >= nx || yy >= ny || zz >= nz) continue;
                                int cand = in[((size_t)zz * ny + yy) * nx + xx] + (m == 1 ? 16 : (m == 2 ? 23 : 28));
                                if (cand < best) best = cand;
                            }
                    dst[c] = (uint8_t)(best < 255 ? best : 255);
                }
    }
    free(tmp);
}

/* float -> bfloat16 -> float, round to nearest even */
static float bf16r(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return x;
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    memcpy(&x, &u, 4);
    return x;
}

/* Installs the closure: the weights as the library packs them (BF16 weights
 * and hidden-layer biases, out_scale folded into the last layer, FP32 output
 * bias), the input
 * normalization and training range, the wall distance (computed here
 * when `wall` is NULL), the near-wall fallback distance `wall_min` (cells)
 * and the Smagorinsky trust factor `trust` (0: off). w1 NULL turns the
 * closure off. */
int SYM(set_closure)(oracle_lbm* o, const float* w1, const float* b1, const float* w2, const float* b2,
                     const float* w3, float b3, float out_scale, const float* mean, const float* std,
                     const float* lo, const float* hi, float filter_width, const uint8_t* wall, float wall_min,
                     float trust) {
    if (!w1) {
        o->closure_on = 0;
        return 0;
    }
    for (int i = 0; i < 5 * 32; ++i) o->cw1[i] = bf16r(w1[i]);
    for (int i = 0; i < 32 * 32; ++i) o->cw2[i] = bf16r(w2[i]);
    for (int i = 0; i < 32; ++i) {
        o->cb1[i] = bf16r(b1[i]);
        o->cb2[i] = bf16r(b2[i]);
        o->cw3[i] = bf16r(w3[i] * out_scale);
    }
    o->cb3 = b3 * out_scale;
    for (int k = 0; k < 5; ++k) {
        o->cmean[k] = mean[k];
        o->cinv_std[k] = 1.0f / std[k];
    }
    for (int k = 0; k < 3; ++k) {
        o->clo[k] = lo[k];
        o->chi[k] = hi[k];
    }
    o->cfilter = filter_width;
    {
        float wm = ceilf(wall_min * 16.0f);
        o->cwall_min = wm > 255.0f ? 256 : (int)wm;
    }
    o->ctrust = trust;
    if (!o->wall) o->wall = (uint8_t*)malloc(o->n ? o->n : 1);
    if (wall)
        memcpy(o->wall, wall, o->n);
    else
        SYM(wall_distance)(o->nx, o->ny, o->nz, o->solid, o->wall);
    o->closure_on = 1;
    return 0;
}

/* The closure's raw inputs 0-2 from Pi_neq and rho (closure_invariants). */
static void closure_inputs(real pxx, real pyy, real pzz, real pxy, real pxz, real pyz, real rho, float* x) {
    real pp = pxx * pxx + pyy * pyy + pzz * pzz + K(2.0) * (pxy * pxy + pxz * pxz + pyz * pyz);
    real mag = RSQRT(pp);
    real r = pp > K(0.0) ? K(1.0) / mag : K(0.0);
    real inv = rho > K(1e-6) ? K(1.0) / rho : K(1.0);
    x[0] = (float)log2((double)(mag * inv) + 1e-12);
    x[1] = (float)((pxx + pyy + pzz) * r);
    real det = pxx * (pyy * pzz - pyz * pyz) - pxy * (pxy * pzz - pyz * pxz) + pxz * (pxy * pyz - pyy * pxz);
    x[2] = (float)(det * r * r * r);
}

/* nu_t of one cell, or -1 when inputs 0-2 leave the training range. Inputs,
 * weights and hidden activations are rounded to BF16 as on the tensor cores;
 * the sums are accumulated in double. */
static float closure_nu(const oracle_lbm* o, const float* x3) {
    float x[5] = {x3[0], x3[1], x3[2], x3[3], o->cfilter};
    for (int k = 0; k < 3; ++k)
        if (!(x[k] >= o->clo[k] && x[k] <= o->chi[k])) return -1.0f;
    if ((int)(x3[3] * 16.0f) < o->cwall_min) return -1.0f; /* near-wall fallback */
    float a[5], h1[32], h2[32];
    for (int k = 0; k < 5; ++k) a[k] = bf16r((x[k] - o->cmean[k]) * o->cinv_std[k]);
    for (int j = 0; j < 32; ++j) {
        double s = o->cb1[j];
        for (int k = 0; k < 5; ++k) s += (double)a[k] * o->cw1[k * 32 + j];
        h1[j] = bf16r(s > 0.0 ? (float)s : 0.0f);
    }
    for (int j = 0; j < 32; ++j) {
        double s = o->cb2[j];
        for (int k = 0; k < 32; ++k) s += (double)h1[k] * o->cw2[k * 32 + j];
        h2[j] = bf16r(s > 0.0 ? (float)s : 0.0f);
    }
    double z = o->cb3;
    for (int k = 0; k < 32; ++k) z += (double)h2[k] * o->cw3[k];
    return z > 0.0 ? (float)z : 0.0f;
}

/* Batch evaluation for tests: nu_t (or -1 outside the range) of n cells from
 * their inputs 0-3 (x[4*i .. 4*i+3]). */
void SYM(closure_eval)(const oracle_lbm* o, const float* x, size_t n, float* nu) {
    for (size_t i = 0; i < n; ++i) nu[i] = closure_nu(o, x + 4 * i);
}

/* ---- one fused pull-stream + BC + regularized collision step,
 *      LbmReference.cpp:241-469 ---- */
static void step_body(oracle_lbm* o, int z0, int z1, int tid, void* vctx) {
    (void)tid;
    (void)vctx;
    const real* fi = o->f[o->cur];
    real* fo = o->f[1 - o->cur];
    const int q = o->q;
    int inlet_x = o->reverse ? o->nx - 1 : 0;
    int outlet_x = o->reverse ? 0 : o->nx - 1;
    real inlet_ux = o->reverse ? -o->inlet_u : o->inlet_u;
    int bad = 0;
    for (int z = z0; z < z1; ++z) {
        for (int y = 0; y < o->ny; ++y) {
            for (int x = 0; x < o->nx; ++x) {
                size_t c = cidx(o, x, y, z);
                if (o->solid[c]) { /* :264-267 */
                    for (int i = 0; i < q; ++i) POP(fo, i, c) = o->w[i];
                    continue;
                }
                if (x == inlet_x) { /* :269-273 */
                    for (int i = 0; i < q; ++i) POP(fo, i, c) = feq(o, i, K(1.0), inlet_ux, K(0.0), K(0.0));
                    continue;
                }
                if (x == outlet_x) { /* :275-327, neighbour moments from fIn */
                    int nxb = o->reverse ? x + 1 : x - 1;
                    real nr, nu, nv, nw;
                    moments(o, fi, cidx(o, nxb, y, z), &nr, &nu, &nv, &nw);
                    real rho = nr > K(1e-6) ? K(1.0) + K(0.999) * (nr - K(1.0)) : K(1.0);
                    for (int i = 0; i < q; ++i) POP(fo, i, c) = feq(o, i, rho, nu, nv, nw);
                    continue;
                }
                real fp[FC_MAXQ];
                for (int i = 0; i < q; ++i) { /* :329-383 */
                    int px = x - o->ex[i], py = y - o->ey[i], pz = z - o->ez[i];
                    int in = inb(o, px, py, pz);
                    if (in && !o->solid[cidx(o, px, py, pz)]) {
                        fp[i] = POP(fi, i, cidx(o, px, py, pz));
                    } else if (in) {
                        fp[i] = bouzidi(o, fi, x, y, z, c, i, px, py, pz);
                    } else {
                        int out_y = py < 0 || py >= o->ny;
                        int out_z = pz < 0 || pz >= o->nz;
                        int mirror_ok = (!out_y || o->slip_y) && (!out_z || o->slip_z);
                        if ((out_y || out_z) && mirror_ok) {
                            int d = i;
                            if (out_y) d = o->mirror_y[d];
                            if (out_z) d = o->mirror_z[d];
                            fp[i] = POP(fi, d, c);
                        } else {
                            fp[i] = POP(fi, o->opp[i], c);
                        }
                    }
                }
                real rho = K(0.0), ux = K(0.0), uy = K(0.0), uz = K(0.0);
                for (int i = 0; i < q; ++i) {
                    rho += fp[i];
                    ux += fp[i] * (real)o->ex[i];
                    uy += fp[i] * (real)o->ey[i];
                    uz += fp[i] * (real)o->ez[i];
                }
                if (rho > K(1e-6)) {
                    ux /= rho;
                    uy /= rho;
                    uz /= rho;
                }
                if (!RFINITE(rho) || !RFINITE(ux) || !RFINITE(uy) || !RFINITE(uz) || rho <= K(0.0) ||
                    (ux * ux + uy * uy + uz * uz) > K(4.0))
                    bad = 1;
                /* Regularized (Latt-Chopard) collision, :422-453. */
                const real cs2 = K(1.0) / K(3.0);
                real pxx = K(0.0), pyy = K(0.0), pzz = K(0.0), pxy = K(0.0), pxz = K(0.0), pyz = K(0.0);
                for (int i = 0; i < q; ++i) {
                    real e = feq(o, i, rho, ux, uy, uz);
                    real ne = fp[i] - e;
                    fp[i] = e;
                    real ex = (real)o->ex[i], ey = (real)o->ey[i], ez = (real)o->ez[i];
                    pxx += ex * ex * ne;
                    pyy += ey * ey * ne;
                    pzz += ez * ez * ne;
                    pxy += ex * ey * ne;
                    pxz += ex * ez * ne;
                    pyz += ey * ez * ne;
                }
                /* Smagorinsky relaxation time, :439-444. */
                real pimag = RSQRT(pxx * pxx + pyy * pyy + pzz * pzz + K(2.0) * (pxy * pxy + pxz * pxz + pyz * pyz));
                real rden = rho > K(1e-6) ? rho : K(1e-6);
                real tau_eff = K(0.5) * (o->tau + RSQRT(o->tau * o->tau +
                                                       K(18.0) * K(1.41421356) * o->cs * o->cs * pimag / rden));
                if (o->closure_on) { /* learned closure in place of Smagorinsky */
                    float xin[4];
                    closure_inputs(pxx, pyy, pzz, pxy, pxz, pyz, rho, xin);
                    xin[3] = (float)o->wall[c] * 0.0625f;
                    float nu = closure_nu(o, xin);
                    if (nu >= 0.0f) {
                        real d = K(3.0) * (real)nu;
                        if (o->ctrust > 0.0f) { /* anchored to Smagorinsky's 3 nu_t */
                            real ds = tau_eff - o->tau;
                            real dlo = ds / (real)o->ctrust, dhi = ds * (real)o->ctrust;
                            d = d < dlo ? dlo : (d > dhi ? dhi : d);
                        }
                        tau_eff = o->tau + d;
                    }
                }
                real omega = K(1.0) / tau_eff;
                for (int i = 0; i < q; ++i) {
                    real ex = (real)o->ex[i], ey = (real)o->ey[i], ez = (real)o->ez[i];
                    real qxx = ex * ex - cs2, qyy = ey * ey - cs2, qzz = ez * ez - cs2;
                    real qxy = ex * ey, qxz = ex * ez, qyz = ey * ez;
                    real reg = (o->w[i] * K(4.5)) * (qxx * pxx + qyy * pyy + qzz * pzz + K(2.0) * qxy * pxy +
                                                     K(2.0) * qxz * pxz + K(2.0) * qyz * pyz);
                    POP(fo, i, c) = fp[i] + (K(1.0) - omega) * reg;
                }
            }
        }
    }
    if (bad) __atomic_store_n(&o->diverged, 1, __ATOMIC_RELAXED);
}

void SYM(step)(oracle_lbm* o, int n) {
    for (int s = 0; s < n; ++s) {
        parallel_z(o, step_body, NULL);
        o->cur = 1 - o->cur;
    }
}

int SYM(has_diverged)(const oracle_lbm* o) { return o->diverged; }

/* ---- readback, LbmReference.cpp:475-500: 4 values per cell,
 *      fluid (rho,ux,uy,uz) / solid (stress,Fx,Fy,Fz) ---- */
typedef struct {
    float* out32;
    double* out64;
} field_ctx;

static void field_body(oracle_lbm* o, int z0, int z1, int tid, void* vctx) {
    (void)tid;
    field_ctx* fc = (field_ctx*)vctx;
    const real* f = o->f[o->cur];
    for (int z = z0; z < z1; ++z)
        for (int y = 0; y < o->ny; ++y)
            for (int x = 0; x < o->nx; ++x) {
                size_t c = cidx(o, x, y, z);
                real v[4];
                if (o->solid[c])
                    solid_force(o, f, x, y, z, &v[0], &v[1], &v[2], &v[3]);
                else
                    moments(o, f, c, &v[0], &v[1], &v[2], &v[3]);
                for (int k = 0; k < 4; ++k) {
                    if (fc->out32) fc->out32[c * 4 + k] = (float)v[k];
                    if (fc->out64) fc->out64[c * 4 + k] = (double)v[k];
                }
            }
}

void SYM(readback_field)(oracle_lbm* o, float* out) {
    field_ctx fc = {out, NULL};
    parallel_z(o, field_body, &fc);
}

void SYM(readback_field_f64)(oracle_lbm* o, double* out) {
    field_ctx fc = {NULL, out};
    parallel_z(o, field_body, &fc);
}

/* Raw populations of the current state in the reference's natural layout
 * (post-collision, pre-streaming), converted to float / double. */
void SYM(get_populations)(const oracle_lbm* o, float* out32, double* out64) {
    const real* f = o->f[o->cur];
    size_t total = (size_t)o->q * o->n;
    for (size_t k = 0; k < total; ++k) {
        if (out32) out32[k] = (float)f[k];
        if (out64) out64[k] = (double)f[k];
    }
}

/* ---- statistics, LbmReference.cpp:502-585 (per-slab partials in double) ---- */
typedef struct {
    double mn, mx, vmax, smax;
    double dsum, ssum, mass, fxs, fys, fzs;
    size_t fluid;
    int nan;
} stat_part;

static void stats_body(oracle_lbm* o, int z0, int z1, int tid, void* vctx) {
    stat_part* p = &((stat_part*)vctx)[tid];
    const real* f = o->f[o->cur];
    p->mn = 1e30;
    p->mx = -1e30;
    for (int z = z0; z < z1; ++z)
        for (int y = 0; y < o->ny; ++y)
            for (int x = 0; x < o->nx; ++x) {
                size_t c = cidx(o, x, y, z);
                if (o->solid[c]) {
                    real st, a, b, d;
                    solid_force(o, f, x, y, z, &st, &a, &b, &d);
                    if (RFINITE(st) && RFINITE(a) && RFINITE(b) && RFINITE(d)) {
                        p->fxs += (double)a;
                        p->fys += (double)b;
                        p->fzs += (double)d;
                        if ((double)st > p->smax) p->smax = (double)st;
                    }
                    continue;
                }
                real rho, ux, uy, uz;
                moments(o, f, c, &rho, &ux, &uy, &uz);
                if (!RFINITE(rho) || !RFINITE(ux) || !RFINITE(uy) || !RFINITE(uz)) {
                    p->nan = 1;
                    continue;
                }
                real sp = RSQRT(ux * ux + uy * uy + uz * uz);
                if ((double)rho < p->mn) p->mn = (double)rho;
                if ((double)rho > p->mx) p->mx = (double)rho;
                if ((double)sp > p->vmax) p->vmax = (double)sp;
                p->dsum += (double)rho;
                p->ssum += (double)sp;
                p->mass += (double)rho;
                p->fluid++;
            }
}

void SYM(stats)(oracle_lbm* o, oracle_stats* s) {
    stat_part parts[256];
    memset(parts, 0, sizeof(parts));
    parallel_z(o, stats_body, parts);
    memset(s, 0, sizeof(*s));
    double mn = 1e30, mx = -1e30, vmax = 0.0, smax = 0.0, ds = 0.0, ss = 0.0, mass = 0.0;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    size_t fluid = 0;
    int t = thread_count(o);
    for (int k = 0; k < t; ++k) {
        stat_part* p = &parts[k];
        s->has_nan |= p->nan;
        if (p->smax > smax) smax = p->smax;
        fx += p->fxs;
        fy += p->fys;
        fz += p->fzs;
        if (p->fluid == 0) continue;
        if (p->mn < mn) mn = p->mn;
        if (p->mx > mx) mx = p->mx;
        if (p->vmax > vmax) vmax = p->vmax;
        ds += p->dsum;
        ss += p->ssum;
        mass += p->mass;
        fluid += p->fluid;
    }
    s->force_x = fx;
    s->force_y = fy;
    s->force_z = fz;
    s->max_stress = smax;
    s->max_speed = vmax;
    s->total_mass = mass;
    if (fluid > 0) {
        s->min_density = mn;
        s->max_density = mx;
        s->avg_density = ds / (double)fluid;
        s->avg_speed = ss / (double)fluid;
    }
    s->fluid_count_lo = (int32_t)(fluid & 0x7fffffff);
}
