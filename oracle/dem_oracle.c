/*
 * dem_oracle.c -- CPU restatement of the world DEM step (test infrastructure only).
 *
 * Built with -ffp-contract=off: every fused multiply-add below is an explicit fmaf,
 * placed where the CUDA kernels of libworld_b200 place theirs, so both sides round
 * identically. Grain visiting order is canonical: the reference's 27-cell stencil
 * order (src/find_neighbors_kernel.cu:132-158, dx outer, dz inner) and, inside a
 * cell, ascending grain id. The reference fills cells with atomicAdd slots
 * (src/find_neighbors_kernel.cu:91) and so has no defined order inside a cell; the
 * canonical order is the one deterministic choice consistent with it.
 *
 * The dense-grid bucketing (one count per cell, then a fill) is the reference's
 * algorithm (src/find_neighbors_kernel.cu:46-112) without the per-cell capacity: no
 * grain is dropped, and cells above particles_per_cell are only counted, as the
 * reference's overflow counter does (src/find_neighbors_kernel.cu:92-95).
 */
#include "dem_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int dem_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void dem_set_num_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

void dem_params_derive(dem_params* p, float normal_stiffness, float tangential_stiffness,
                       float particle_radius) {
    const int compat = !(normal_stiffness > 0.f);
    p->k_n = compat ? p->max_force / particle_radius : normal_stiffness;
    if (!compat && !(p->max_force > 0.f)) p->max_force = INFINITY;
    p->k_t = tangential_stiffness > 0.f ? tangential_stiffness : (2.f / 7.f) * p->k_n;
    const float pi = 3.14159265358979323846f;
    p->ln_e = (p->restitution > 0.f && p->restitution < 1.f) ? logf(p->restitution) : 0.f;
    p->damp_den = sqrtf(fmaf(p->ln_e, p->ln_e, pi * pi));
    p->clamp_overlap = compat ? particle_radius : p->max_force / p->k_n;
    p->radius = particle_radius;
}

/* float -> int32 truncation with the saturating behaviour of CUDA's cvt.rzi.s32.f32
 * (NaN -> 0, out of range -> INT32_MIN / INT32_MAX), which is what
 * static_cast<int>(float) does in the reference kernels. */
static inline int32_t f2i_rz_sat(float t) {
    if (t != t) return 0;
    if (t >= 2147483648.0f) return INT32_MAX;
    if (t < -2147483648.0f) return INT32_MIN;
    return (int32_t)t;
}

static inline int32_t clampi(int32_t v, int32_t lo, int32_t hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

/* reference src/find_neighbors_kernel.cu:11-22 */
static inline int32_t cell_axis(float x, float lo, float hi, int32_t g) {
    const float t = (x - lo) / (hi - lo) * (float)g;
    return clampi(f2i_rz_sat(t), 0, g - 1);
}

static inline void cell_coords(const dem_params* p, const float* s, int32_t* c) {
    c[0] = cell_axis(s[0], p->lo[0], p->hi[0], p->grid[0]);
    c[1] = cell_axis(s[1], p->lo[1], p->hi[1], p->grid[1]);
    c[2] = cell_axis(s[2], p->lo[2], p->hi[2], p->grid[2]);
}

/* reference src/find_neighbors_kernel.cu:27-30 (x slowest, z fastest) */
static inline int64_t flat_cell(const dem_params* p, int32_t x, int32_t y, int32_t z) {
    return ((int64_t)x * p->grid[1] + y) * p->grid[2] + z;
}

void dem_cell_keys(const dem_params* p, int64_t n, const float* state, int32_t* keys) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        int32_t c[3];
        cell_coords(p, state + 6 * i, c);
        keys[i] = (int32_t)flat_cell(p, c[0], c[1], c[2]);
    }
}

/* ---------------------------------------------------------------------------------
 * Dense-grid bucketing. start[c]..start[c+1] indexes sorted[], grains of cell c by
 * ascending id. Buffers are kept between calls (the oracle is single-user).
 * ------------------------------------------------------------------------------- */
typedef struct cells {
    int64_t num_cells;
    int32_t* start;   /* num_cells + 1 */
    int32_t* fill;    /* num_cells */
    int32_t* sorted;  /* n */
    int32_t* key;     /* n */
    int64_t cap_cells, cap_n;
} cells;

static cells g_cells;


static int64_t build_cells(const dem_params* p, int64_t n, const float* state) {
    cells* C = &g_cells;
    const int64_t nc = (int64_t)p->grid[0] * p->grid[1] * p->grid[2];
    if (nc + 1 > C->cap_cells) {
        free(C->start); free(C->fill);
        C->start = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nc + 1));
        C->fill = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nc + 1));
        C->cap_cells = nc + 1;
    }
    if (n > C->cap_n) {
        free(C->sorted); free(C->key);
        C->sorted = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
        C->key = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
        C->cap_n = n;
    }
    C->num_cells = nc;
    memset(C->fill, 0, sizeof(int32_t) * (size_t)nc);
    dem_cell_keys(p, n, state, C->key);
    /* count (pass 1 of the reference marks, pass 3 reserves slots) */
    for (int64_t i = 0; i < n; ++i) C->fill[C->key[i]]++;
    int64_t overflow = 0;
    int32_t acc = 0;
    for (int64_t c = 0; c < nc; ++c) {
        const int32_t k = C->fill[c];
        if (k > p->particles_per_cell) ++overflow;
        C->start[c] = acc;
        C->fill[c] = acc;
        acc += k;
    }
    C->start[nc] = acc;
    /* fill in ascending id order -> ids ascending inside every cell */
    for (int64_t i = 0; i < n; ++i) C->sorted[C->fill[C->key[i]]++] = (int32_t)i;
    return overflow;
}

/* Visit the canonical candidates of grain i: stencil order, ascending id per cell. */
#define FOR_EACH_CANDIDATE(P, STATE, I, J, ...)                                         \
    do {                                                                                \
        int32_t cc_[3];                                                                 \
        cell_coords((P), (STATE) + 6 * (I), cc_);                                       \
        for (int dx_ = -1; dx_ <= 1; ++dx_) {                                           \
            const int32_t nx_ = cc_[0] + dx_;                                           \
            if (nx_ < 0 || nx_ >= (P)->grid[0]) continue;                               \
            for (int dy_ = -1; dy_ <= 1; ++dy_) {                                       \
                const int32_t ny_ = cc_[1] + dy_;                                       \
                if (ny_ < 0 || ny_ >= (P)->grid[1]) continue;                           \
                for (int dz_ = -1; dz_ <= 1; ++dz_) {                                   \
                    const int32_t nz_ = cc_[2] + dz_;                                   \
                    if (nz_ < 0 || nz_ >= (P)->grid[2]) continue;                       \
                    const int64_t c_ = flat_cell((P), nx_, ny_, nz_);                   \
                    for (int32_t s_ = g_cells.start[c_]; s_ < g_cells.start[c_ + 1];    \
                         ++s_) {                                                        \
                        const int64_t J = g_cells.sorted[s_];                           \
                        if (J == (I)) continue;                                         \
                        __VA_ARGS__                                                     \
                    }                                                                   \
                }                                                                       \
            }                                                                           \
        }                                                                               \
    } while (0)

/* Pair geometry shared by candidates, forces and energy. */
static inline float pair_norm(const float* si, const float* sj, float* d) {
    d[0] = si[0] - sj[0];
    d[1] = si[1] - sj[1];
    d[2] = si[2] - sj[2];
    float ns = d[0] * d[0];
    ns = fmaf(d[1], d[1], ns);
    ns = fmaf(d[2], d[2], ns);
    return sqrtf(ns);
}

/* dist = |delta| - r_i - r_j, subtracting the larger radius first: symmetric in
 * (i, j) and identical to the reference's norm - radius - radius for equal radii
 * (src/compute_rhs_kernel.cu:161). */
static inline float pair_dist(float norm, float ri, float rj) {
    const float rmax = ri > rj ? ri : rj;
    const float rmin = ri > rj ? rj : ri;
    return (norm - rmax) - rmin;
}

int64_t dem_candidates(const dem_params* p, int64_t n, const float* state,
                       const float* radius, int64_t* offsets, int32_t* cand,
                       uint8_t* contact, int64_t cap, int64_t* overflow_cells) {
    const int64_t ovf = build_cells(p, n, state);
    if (overflow_cells) *overflow_cells = ovf;
    offsets[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t cnt = 0;
        FOR_EACH_CANDIDATE(p, state, i, j, { (void)j; ++cnt; });
        offsets[i + 1] = offsets[i] + cnt;
    }
    const int64_t total = offsets[n];
    if (total > cap) return total;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        int64_t k = offsets[i];
        const float* si = state + 6 * i;
        FOR_EACH_CANDIDATE(p, state, i, j, {
            float d[3];
            const float norm = pair_norm(si, state + 6 * j, d);
            const float dist = pair_dist(norm, radius[i], radius[j]);
            cand[k] = (int32_t)j;
            contact[k] = (uint8_t)(dist < 0.f);
            ++k;
        });
    }
    return total;
}

/* reference src/compute_rhs_kernel.cu:41-47, with logf(e) and the denominator
 * precomputed on the host: c = ((-2 sqrt(m k)) ln e) / sqrt(pi^2 + ln^2 e). */
static inline float damping(const dem_params* p, float m) {
    if (p->restitution <= 0.f) return 2.f * sqrtf(p->k_n * m);
    if (p->restitution >= 1.f) return 0.f;
    return ((-2.f * sqrtf(m * p->k_n)) * p->ln_e) / p->damp_den;
}

/* reference src/compute_rhs_kernel.cu:66-78 (viscous, capped at mu |F_n|) */
static inline void viscous_friction(float* f, const float* vt, float limit, float c) {
    float vt_sq = vt[0] * vt[0];
    vt_sq = fmaf(vt[1], vt[1], vt_sq);
    vt_sq = fmaf(vt[2], vt[2], vt_sq);
    const float v = sqrtf(vt_sq);
    if (v < 1e-8f) return;
    const float mag = fminf(limit, c * v);
    f[0] = f[0] - (mag * vt[0]) / v;
    f[1] = f[1] - (mag * vt[1]) / v;
    f[2] = f[2] - (mag * vt[2]) / v;
}

typedef struct hist_io {
    const int32_t* cnt_in; const int32_t* part_in; const float* xi_in;
    int32_t* cnt_out; int32_t* part_out; float* xi_out;
    int64_t overflow;
} hist_io;

/* Tangential spring with history (Cundall-Strack), capped at mu |F_n| with the
 * spring reset to the cap on slip. xi is rotated onto the current tangent plane,
 * advanced by v_t dt, and F_t = -k_t xi. No reference function: extension. */
static inline void spring_friction(const dem_params* p, float* f, const float* vt,
                                   const float* nrm, float limit, int64_t i,
                                   int32_t partner, hist_io* h, int32_t* newcnt) {
    float xi[3] = {0.f, 0.f, 0.f};
    const int32_t oc = h->cnt_in[i];
    for (int32_t k = 0; k < oc; ++k) {
        if (h->part_in[i * DEM_HIST_CAP + k] == partner) {
            const float* x = h->xi_in + (i * DEM_HIST_CAP + k) * 3;
            xi[0] = x[0]; xi[1] = x[1]; xi[2] = x[2];
            break;
        }
    }
    float xn = xi[0] * nrm[0];
    xn = fmaf(xi[1], nrm[1], xn);
    xn = fmaf(xi[2], nrm[2], xn);
    float ft[3];
    for (int a = 0; a < 3; ++a) {
        xi[a] = fmaf(-xn, nrm[a], xi[a]);
        xi[a] = fmaf(p->dt, vt[a], xi[a]);
        ft[a] = -p->k_t * xi[a];
    }
    float ft_sq = ft[0] * ft[0];
    ft_sq = fmaf(ft[1], ft[1], ft_sq);
    ft_sq = fmaf(ft[2], ft[2], ft_sq);
    if (ft_sq > limit * limit) {
        const float s = limit / sqrtf(ft_sq);
        for (int a = 0; a < 3; ++a) { ft[a] = ft[a] * s; xi[a] = xi[a] * s; }
    }
    f[0] = f[0] + ft[0];
    f[1] = f[1] + ft[1];
    f[2] = f[2] + ft[2];
    const int32_t slot = *newcnt;
    if (slot < DEM_HIST_CAP) {
        h->part_out[i * DEM_HIST_CAP + slot] = partner;
        float* x = h->xi_out + (i * DEM_HIST_CAP + slot) * 3;
        x[0] = xi[0]; x[1] = xi[1]; x[2] = xi[2];
        *newcnt = slot + 1;
    } else {
#pragma omp atomic
        h->overflow += 1;
    }
}

/* Force on grain i divided by its mass -> acc[3]. reference
 * src/compute_rhs_kernel.cu:99-210 (gravity, six walls, pairs, rhs = F/m). */
static void grain_acc(const dem_params* p, int64_t i, const float* state,
                      const float* radius, const float* mass, hist_io* h, float* acc) {
    const float* si = state + 6 * i;
    const float pos[3] = {si[0], si[1], si[2]};
    const float vel[3] = {si[3], si[4], si[5]};
    const float ri = radius[i];
    const float mi = mass[i];
    const float k = p->k_n;
    const float F = p->max_force;
    const float mu = p->friction;
    float f[3] = {0.f, 0.f, 0.f};
    int32_t newcnt = 0;
    const float c_wall = damping(p, mi);

    f[2] = fmaf(-mi, p->gravity, f[2]);

    for (int a = 0; a < 3; ++a) {
        float vt[3];
        for (int b = 0; b < 3; ++b) vt[b] = (b == a) ? 0.f : vel[b];
        const float dl = (pos[a] - p->wall_lo[a]) - ri;
        const float fl = fmaxf(0.f, fminf(F, -k * dl));
        f[a] = f[a] + fl;
        if (dl < 0.f) {
            f[a] = fmaf(-c_wall, vel[a], f[a]);
            if (p->history) {
                float nrm[3] = {0.f, 0.f, 0.f};
                nrm[a] = 1.f;
                spring_friction(p, f, vt, nrm, mu * fl, i, -1 - 2 * a, h, &newcnt);
            } else {
                viscous_friction(f, vt, mu * fl, c_wall);
            }
        }
        const float du = (p->wall_hi[a] - pos[a]) - ri;
        const float fu = fmaxf(0.f, fminf(F, -k * du));
        f[a] = f[a] - fu;
        if (du < 0.f) {
            f[a] = fmaf(-c_wall, vel[a], f[a]);
            if (p->history) {
                float nrm[3] = {0.f, 0.f, 0.f};
                nrm[a] = -1.f;
                spring_friction(p, f, vt, nrm, mu * fu, i, -2 - 2 * a, h, &newcnt);
            } else {
                viscous_friction(f, vt, mu * fu, c_wall);
            }
        }
    }

    FOR_EACH_CANDIDATE(p, state, i, j, {
        const float* sj = state + 6 * j;
        float d[3];
        const float norm = pair_norm(si, sj, d);
        const float dist = pair_dist(norm, ri, radius[j]);
        if (dist < 0.f) {
            const float nrm[3] = {d[0] / norm, d[1] / norm, d[2] / norm};
            const float fp = fmaxf(0.f, fminf(F, -k * dist));
            f[0] = fmaf(fp, nrm[0], f[0]);
            f[1] = fmaf(fp, nrm[1], f[1]);
            f[2] = fmaf(fp, nrm[2], f[2]);
            const float mj = mass[j];
            const float msum = mi + mj;
            const float mred = (msum > 0.f) ? (mi * mj) / msum : 0.f;
            const float c = damping(p, mred);
            const float vr[3] = {vel[0] - sj[3], vel[1] - sj[4], vel[2] - sj[5]};
            float vn = vr[0] * nrm[0];
            vn = fmaf(vr[1], nrm[1], vn);
            vn = fmaf(vr[2], nrm[2], vn);
            const float cvn = c * vn;
            float vt[3];
            for (int a = 0; a < 3; ++a) {
                f[a] = fmaf(-cvn, nrm[a], f[a]);
                vt[a] = fmaf(-vn, nrm[a], vr[a]);
            }
            if (p->history) {
                spring_friction(p, f, vt, nrm, mu * fp, i, (int32_t)j, h, &newcnt);
            } else {
                viscous_friction(f, vt, mu * fp, c);
            }
        }
    });

    if (p->history) h->cnt_out[i] = newcnt;
    acc[0] = f[0] / mi;
    acc[1] = f[1] / mi;
    acc[2] = f[2] / mi;
}

static int64_t rhs_pass(const dem_params* p, int64_t n, const float* state,
                        const float* radius, const float* mass, hist_io* h, float* acc) {
    const int64_t ovf = build_cells(p, n, state);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) grain_acc(p, i, state, radius, mass, h, acc + 3 * i);
    return ovf;
}

int dem_compute_rhs(const dem_params* p, int64_t n, const float* state,
                    const float* radius, const float* mass,
                    const int32_t* hcnt_in, const int32_t* hpart_in, const float* hxi_in,
                    int32_t* hcnt_out, int32_t* hpart_out, float* hxi_out,
                    float* rhs, int64_t* overflow_cells, int64_t* hist_overflow) {
    hist_io h = {hcnt_in, hpart_in, hxi_in, hcnt_out, hpart_out, hxi_out, 0};
    float* acc = (float*)malloc(sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
    const int64_t ovf = rhs_pass(p, n, state, radius, mass, &h, acc);
    for (int64_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            rhs[6 * i + a] = state[6 * i + 3 + a];
            rhs[6 * i + 3 + a] = acc[3 * i + a];
        }
    }
    free(acc);
    if (overflow_cells) *overflow_cells = ovf;
    if (hist_overflow) *hist_overflow = h.overflow;
    return 0;
}

/* rhs = [v, F/m] at the state the forces were evaluated on (before the update),
 * as the reference's device_rhs holds it (src/compute_rhs_kernel.cu:207-210). */
static void record_rhs(float* rhs_out, const float* state, const float* acc, int64_t n) {
    if (!rhs_out) return;
    for (int64_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            rhs_out[6 * i + a] = state[6 * i + 3 + a];
            rhs_out[6 * i + 3 + a] = acc[3 * i + a];
        }
    }
}

int dem_step(const dem_params* p, int64_t n, float* state, const float* radius,
             const float* mass, int32_t* hcnt, int32_t* hpart, float* hxi,
             float* rhs_out, int32_t* picard_used, float* picard_residual,
             int64_t* overflow_cells, int64_t* hist_overflow) {
    const size_t nn = (size_t)(n > 0 ? n : 1);
    float* acc = (float*)malloc(sizeof(float) * 3 * nn);
    int32_t* ncnt = NULL; int32_t* npart = NULL; float* nxi = NULL;
    if (p->history) {
        ncnt = (int32_t*)malloc(sizeof(int32_t) * nn);
        npart = (int32_t*)malloc(sizeof(int32_t) * nn * DEM_HIST_CAP);
        nxi = (float*)malloc(sizeof(float) * nn * DEM_HIST_CAP * 3);
    }
    hist_io h = {hcnt, hpart, hxi, ncnt, npart, nxi, 0};
    int64_t ovf = 0;
    int32_t used = 1;
    float residual = 0.f;
    const float dt = p->dt;
    if (p->integrator == 0) {
        /* reference src/semi_implicit_euler_kernel.cu:4-16 */
        ovf += rhs_pass(p, n, state, radius, mass, &h, acc);
        record_rhs(rhs_out, state, acc, n);
        for (int64_t i = 0; i < n; ++i) {
            float* s = state + 6 * i;
            for (int a = 0; a < 3; ++a) s[3 + a] = fmaf(dt, acc[3 * i + a], s[3 + a]);
            for (int a = 0; a < 3; ++a) s[a] = fmaf(dt, s[3 + a], s[a]);
        }
    } else {
        /* reference src/particle_dynamics.cu:270-279 and
         * src/backward_euler_picard_kernel.cu:4-17; stops early once
         * max |x_{k+1} - x_k| < picard_tolerance when a tolerance is set. */
        float* sn = (float*)malloc(sizeof(float) * 6 * nn);
        memcpy(sn, state, sizeof(float) * 6 * (size_t)n);
        used = 0;
        for (int32_t k = 0; k < p->picard_iterations; ++k) {
            h.overflow = 0;
            ovf += rhs_pass(p, n, state, radius, mass, &h, acc);
            record_rhs(rhs_out, state, acc, n);
            float res = 0.f;
            for (int64_t i = 0; i < n; ++i) {
                float* s = state + 6 * i;
                const float* s0 = sn + 6 * i;
                for (int a = 0; a < 3; ++a) {
                    const float v = fmaf(dt, acc[3 * i + a], s0[3 + a]);
                    const float x = fmaf(dt, v, s0[a]);
                    const float r = fabsf(x - s[a]);
                    if (r > res || r != r) res = r;
                    s[3 + a] = v;
                    s[a] = x;
                }
            }
            residual = res;
            ++used;
            if (p->picard_tolerance > 0.f && res < p->picard_tolerance) break;
        }
        free(sn);
    }
    if (p->history) {
        memcpy(hcnt, ncnt, sizeof(int32_t) * (size_t)n);
        memcpy(hpart, npart, sizeof(int32_t) * (size_t)n * DEM_HIST_CAP);
        memcpy(hxi, nxi, sizeof(float) * (size_t)n * DEM_HIST_CAP * 3);
        free(ncnt); free(npart); free(nxi);
    }
    free(acc);
    if (picard_used) *picard_used = used;
    if (picard_residual) *picard_residual = residual;
    if (overflow_cells) *overflow_cells = ovf;
    if (hist_overflow) *hist_overflow = h.overflow;
    return 0;
}

/* reference src/density_grid_kernel.cu:25-40 */
static inline void axis_weights(float x, float lo, float hi, int32_t size, int32_t* i0,
                                int32_t* i1, float* w0, float* w1) {
    if (size <= 1) { *i0 = 0; *i1 = 0; *w0 = 1.f; *w1 = 0.f; return; }
    const float h = (hi - lo) / (float)(size - 1);
    const float u = (x - lo) / h;
    const float base = floorf(u);
    const float frac = u - base;
    const int32_t b = f2i_rz_sat(base);
    *i0 = clampi(b, 0, size - 1);
    *i1 = clampi((int32_t)((uint32_t)b + 1u), 0, size - 1);
    *w0 = 1.f - frac;
    *w1 = frac;
}

void dem_deposit(const dem_params* p, int64_t n, const float* state, const float* mass,
                 double* grid) {
    const int32_t sx = p->dgrid[0], sy = p->dgrid[1], sz = p->dgrid[2];
    const int64_t nodes = (int64_t)sx * sy * sz;
    memset(grid, 0, sizeof(double) * 4 * (size_t)nodes);
    for (int64_t i = 0; i < n; ++i) {
        const float m = mass[i];
        if (m == 0.f) continue;
        const float* s = state + 6 * i;
        int32_t ix[2], iy[2], iz[2];
        float wx[2], wy[2], wz[2];
        axis_weights(s[0], p->lo[0], p->hi[0], sx, &ix[0], &ix[1], &wx[0], &wx[1]);
        axis_weights(s[1], p->lo[1], p->hi[1], sy, &iy[0], &iy[1], &wy[0], &wy[1]);
        axis_weights(s[2], p->lo[2], p->hi[2], sz, &iz[0], &iz[1], &wz[0], &wz[1]);
        const float mom[3] = {m * s[3], m * s[4], m * s[5]};
        for (int cx = 0; cx < 2; ++cx)
            for (int cy = 0; cy < 2; ++cy)
                for (int cz = 0; cz < 2; ++cz) {
                    const float w = wx[cx] * wy[cy] * wz[cz];
                    if (w == 0.f) continue;
                    const int64_t node = ((int64_t)ix[cx] * sy + iy[cy]) * sz + iz[cz];
                    grid[node] += (double)(m * w);
                    for (int a = 0; a < 3; ++a)
                        grid[(a + 1) * nodes + node] += (double)(mom[a] * w);
                }
    }
}

/* reference src/energy_kernel.cu:22-27, clamp point generalised to F/k_n */
static inline float contact_energy(float delta, float clamp_d, float F, float k) {
    if (delta <= 0.f) return 0.f;
    if (delta <= clamp_d) return 0.5f * k * delta * delta;
    return 0.5f * F * clamp_d + F * (delta - clamp_d);
}

double dem_energy(const dem_params* p, int64_t n, const float* state, const float* radius,
                  const float* mass, const int32_t* hcnt, const int32_t* hpart,
                  const float* hxi, int64_t* overflow_cells) {
    const int64_t ovf = build_cells(p, n, state);
    if (overflow_cells) *overflow_cells = ovf;
    const float F = p->max_force, k = p->k_n, cd = p->clamp_overlap;
    double total = 0.0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
    for (int64_t i = 0; i < n; ++i) {
        const float* s = state + 6 * i;
        const float m = mass[i];
        const float ri = radius[i];
        float ss = s[3] * s[3];
        ss = fmaf(s[4], s[4], ss);
        ss = fmaf(s[5], s[5], ss);
        double e = (double)(0.5f * m * ss);
        e += (double)((m * p->gravity) * (s[2] - p->wall_lo[2]));
        for (int a = 0; a < 3; ++a) {
            e += (double)contact_energy(ri - (s[a] - p->wall_lo[a]), cd, F, k);
            e += (double)contact_energy(ri - (p->wall_hi[a] - s[a]), cd, F, k);
        }
        FOR_EACH_CANDIDATE(p, state, i, j, {
            if (j > i) {
                float d[3];
                const float norm = pair_norm(s, state + 6 * j, d);
                e += (double)contact_energy((ri + radius[j]) - norm, cd, F, k);
            }
        });
        if (p->history && hcnt) {
            for (int32_t q = 0; q < hcnt[i]; ++q) {
                const int32_t partner = hpart[i * DEM_HIST_CAP + q];
                if (partner >= 0 && partner <= i) continue;
                const float* x = hxi + (i * DEM_HIST_CAP + q) * 3;
                float xs = x[0] * x[0];
                xs = fmaf(x[1], x[1], xs);
                xs = fmaf(x[2], x[2], xs);
                e += (double)(0.5f * p->k_t * xs);
            }
        }
        total += e;
    }
    return total;
}

void dem_momentum(int64_t n, const float* state, const float* mass, double* out3) {
    double px = 0.0, py = 0.0, pz = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double m = mass[i];
        px += m * state[6 * i + 3];
        py += m * state[6 * i + 4];
        pz += m * state[6 * i + 5];
    }
    out3[0] = px; out3[1] = py; out3[2] = pz;
}
