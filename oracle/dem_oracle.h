/*
 * dem_oracle.h -- CPU restatement of the world DEM step (test infrastructure).
 *
 * THIS IS THE ORACLE, NOT THE PRODUCT. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference leg of bench.py may load it, and only as the checker or as
 * the timed CPU baseline. The product path (libworld_b200.so) never calls into it.
 *
 * It restates, in plain C99 (+ optional OpenMP over grains), the reference's step:
 *   src/find_neighbors_kernel.cu:11-161   cell keys, 27-cell candidate lists
 *   src/compute_rhs_kernel.cu:41-210      gravity, walls, pair spring-dashpot, friction
 *   src/semi_implicit_euler_kernel.cu:4-16, src/backward_euler_picard_kernel.cu:4-17,
 *   src/particle_dynamics.cu:264-281      the two integrators and the Picard loop
 *   src/density_grid_kernel.cu:25-83      node-centred CIC deposit
 *   src/energy_kernel.cu:22-80            total energy
 * plus the extensions that have no reference function (per-grain radius and mass,
 * explicit normal stiffness, tangential spring with per-pair history, Picard tolerance).
 *
 * Every floating-point expression is written with the association and the fused
 * multiply-adds that the CUDA kernels use (C99 fmaf, compiled with -ffp-contract=off),
 * so that the GPU path and this file agree bit for bit when they visit grains in the
 * same order: cells in the reference's stencil order (dx, dy, dz ascending), grains
 * inside a cell by ascending grain id.
 */
#ifndef DEM_ORACLE_H
#define DEM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Tangential-history capacity per grain (pair and wall contacts). */
#define DEM_HIST_CAP 24

typedef struct dem_params {
    float lo[3], hi[3];          /* domain box: cell mapping and CIC grid span */
    int32_t grid[3];             /* collision grid cells per axis */
    int32_t particles_per_cell;  /* capacity used only for overflow counting */
    int32_t dgrid[3];            /* CIC nodes per axis */
    float gravity;
    float radius;                /* global radius (compat clamp point in the energy) */
    float max_force;             /* spring clamp; +inf disables it */
    float wall_lo[3], wall_hi[3];/* wall_x_min, wall_y_min, floor_z / wall_x_max, wall_y_max, ceiling_z */
    float restitution;
    float friction;              /* Coulomb mu */
    float k_n;                   /* normal stiffness (compat: max_force / radius) */
    float k_t;                   /* tangential stiffness (history mode) */
    float clamp_overlap;         /* overlap at which the clamp engages (compat: radius) */
    float ln_e;                  /* logf(restitution), computed once on the host */
    float damp_den;              /* sqrtf(fmaf(ln_e, ln_e, pi*pi)) */
    float dt;
    int32_t history;             /* 0: viscous friction (reference); 1: tangential spring */
    int32_t integrator;          /* 0: semi-implicit Euler; 1: backward Euler / Picard */
    int32_t picard_iterations;   /* fixed count, or the cap when picard_tolerance > 0 */
    float picard_tolerance;      /* <= 0: fixed count (reference behaviour) */
} dem_params;

/* Fill the derived fields (k_n, the clamp, k_t, ln_e, damp_den, clamp_overlap,
 * radius) from the base fields already set and the three config values below:
 * compat mode (normal_stiffness <= 0) takes k_n = max_force / particle_radius as
 * the reference does (src/compute_rhs_kernel.cu:92). */
void dem_params_derive(dem_params* p, float normal_stiffness, float tangential_stiffness,
                       float particle_radius);

/* Number of OpenMP threads the oracle uses (1 when built without OpenMP). */
int dem_num_threads(void);
void dem_set_num_threads(int threads);

/* Cell key of every grain (reference src/find_neighbors_kernel.cu:11-40). */
void dem_cell_keys(const dem_params* p, int64_t n, const float* state, int32_t* keys);

/* Canonical candidate lists (reference src/find_neighbors_kernel.cu:119-161), CSR by
 * grain id: offsets[n+1]; cand[offsets[i]..offsets[i+1]) in stencil order, ids
 * ascending inside a cell; contact[k] = 1 when the pair overlaps (dist < 0).
 * Returns the total number of candidates; cand/contact are written only when the
 * total fits in cap. *overflow_cells gets the number of cells above capacity. */
int64_t dem_candidates(const dem_params* p, int64_t n, const float* state,
                       const float* radius, int64_t* offsets, int32_t* cand,
                       uint8_t* contact, int64_t cap, int64_t* overflow_cells);

/* rhs = [v, F/m] at the given state (reference src/compute_rhs_kernel.cu:81-212).
 * History rows are read from h*_in and the updated rows written to h*_out (history
 * mode only; pass NULL otherwise). Returns 0. */
int dem_compute_rhs(const dem_params* p, int64_t n, const float* state,
                    const float* radius, const float* mass,
                    const int32_t* hcnt_in, const int32_t* hpart_in, const float* hxi_in,
                    int32_t* hcnt_out, int32_t* hpart_out, float* hxi_out,
                    float* rhs, int64_t* overflow_cells, int64_t* hist_overflow);

/* One take_step() (reference src/particle_dynamics.cu:264-281) in place. History
 * arrays are in/out (committed rows). rhs_out (nullable) receives the last rhs.
 * *picard_used receives the number of Picard iterations run (1 for SIE). */
int dem_step(const dem_params* p, int64_t n, float* state, const float* radius,
             const float* mass, int32_t* hcnt, int32_t* hpart, float* hxi,
             float* rhs_out, int32_t* picard_used, float* picard_residual,
             int64_t* overflow_cells, int64_t* hist_overflow);

/* CIC deposit (reference src/density_grid_kernel.cu:25-83) accumulated in double:
 * grid[4 * nodes], channel-major, node = (ix*ny + iy)*nz + iz. */
void dem_deposit(const dem_params* p, int64_t n, const float* state, const float* mass,
                 double* grid);

/* Total energy (reference src/energy_kernel.cu:22-80): per-term FP32 as the
 * reference, accumulated in double. Adds the tangential-spring energy in history mode. */
double dem_energy(const dem_params* p, int64_t n, const float* state, const float* radius,
                  const float* mass, const int32_t* hcnt, const int32_t* hpart,
                  const float* hxi, int64_t* overflow_cells);

/* Total momentum sum(m v) in double. */
void dem_momentum(int64_t n, const float* state, const float* mass, double* out3);

#ifdef __cplusplus
}
#endif
#endif
