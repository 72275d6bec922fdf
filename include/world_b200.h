/*
 * world_b200.h -- C ABI of libworld_b200.so, the B200 (sm_100a) DEM step.
 *
 * The reference exposes its step only as the C++ class ParticleDynamics
 * (src/particle_dynamics.h:17-141), statically linked into every driver, plus the
 * YAML loader load_config (src/sim_config.h:202-205). This header is the drop-in
 * boundary for that path: plain C types, no exceptions, every call returns an int
 * status (0 = ok, > 0 = ok with a warning, < 0 = error; wd_last_error() has the
 * message). One handle per host thread; each handle owns its CUDA stream and its
 * device buffers. The C++ class mirroring ParticleDynamics member for member is in
 * include/world_b200/particle_dynamics.hpp; Python reaches the same calls through
 * ctypes (world_b200/_lib.py).
 *
 * Arrays crossing this boundary use the reference's layouts:
 *   state      float[6n]  AoS [x y z vx vy vz] per grain (src/sim_config.h:14-15)
 *   positions  float[3n]  AoS [x y z]          (src/particle_dynamics.h:34-37)
 *   rhs        float[6n]  AoS [v, F/m]          (src/compute_rhs_kernel.cu:207-210)
 *   grid       float[4*nodes] channel-major [m, m vx, m vy, m vz], node =
 *              (ix*ny + iy)*nz + iz             (src/density_grid_kernel.h:18-24)
 * all indexed by the caller's grain id, whatever order the device keeps them in.
 */
#ifndef WORLD_B200_H
#define WORLD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define WD_OK 0
#define WD_WARN_DEFAULTS 1     /* config file missing: defaults kept (src/sim_config.cpp:157-161) */
#define WD_WARN_UNKNOWN_KEY 2  /* unknown key ignored (src/sim_config.cpp:47-50) */
#define WD_ERR_INVALID (-1)    /* bad argument */
#define WD_ERR_CUDA (-2)       /* CUDA runtime error (the reference aborts: src/cuda_check.h:7-12) */
#define WD_ERR_IO (-3)         /* state file unreadable or short (the reference exits: src/particle_dynamics.cu:213-229) */
#define WD_ERR_CONFIG (-4)     /* value that does not parse (the reference throws from std::stof) */
#define WD_ERR_OOM (-5)        /* device allocation failed */
#define WD_ERR_CAPACITY (-6)   /* a caller buffer or a fixed capacity is too small */

/* Tangential-history capacity per grain (pair plus wall contacts). */
#define WD_HIST_CAP 24

typedef struct wd_config wd_config;
typedef struct wd_sim wd_sim;

/* Message of the last failing call on this thread (never NULL). */
const char* wd_last_error(void);

/* Library version string. */
const char* wd_version(void);

/* ---- configuration: SimConfig + load_config (src/sim_config.h:64-205) ----------- */

/* New config holding the reference's built-in defaults (src/sim_config.h:68-199). */
int wd_config_create(wd_config** out);
int wd_config_destroy(wd_config* cfg);
int wd_config_copy(const wd_config* src, wd_config** out);

/* Apply a YAML file on top of cfg with load_config's semantics
 * (src/sim_config.cpp:153-195): "section:" headers, "key: value", "[a, b]" lists, "#"
 * comments; unknown keys warn; a missing file warns and keeps cfg. */
int wd_config_load_yaml(wd_config* cfg, const char* path);

/* Set one "section.key" from its text form, exactly as a YAML line would
 * (src/sim_config.cpp:54-149). Returns WD_WARN_UNKNOWN_KEY for unknown keys. */
int wd_config_set(wd_config* cfg, const char* section, const char* key, const char* value);

/* Read one "section.key" back as text (floats as %.9g, lists as "[a, b]"). */
int wd_config_get(const wd_config* cfg, const char* section, const char* key, char* buf,
                  size_t buf_len);

/* Host-only: the initial grains cfg's initialization section describes
 * (initialize_to_cube / two_particles / single_particle / from_file,
 * src/particle_dynamics.cu:128-235). *n receives the grain count; state (6n) and
 * material (n) are written only when n <= capacity. No device is touched. */
int wd_initial_state(const wd_config* cfg, float* state, int32_t* material, int64_t capacity,
                     int64_t* n);

/* ---- construction: ParticleDynamics(const SimConfig&) (src/particle_dynamics.cu:10-94) */

/* Build the initial state from cfg's initialization section (cube, two_particles,
 * single_particle or file: src/particle_dynamics.cu:22-30,165-235) and upload it. */
int wd_create(const wd_config* cfg, wd_sim** out);

/* Build from caller arrays (length n): state AoS6; material ids (NULL: the config's
 * particle_material); radius (NULL: physics.particle_radius); mass (NULL: from
 * physics.density when set, else the material table). */
int wd_create_from_arrays(const wd_config* cfg, int64_t n, const float* state,
                          const int32_t* material, const float* radius, const float* mass,
                          wd_sim** out);

int wd_destroy(wd_sim* sim);

/* ---- batched scenes (extension) --------------------------------------------------
 * No reference counterpart as one call: it replaces the dataset and ensemble
 * drivers' loop of one ParticleDynamics per design row (src/dataset.cpp:163-232,
 * src/chaos.cpp:176-206). num_scenes independent scenes share one handle and
 * one step: scene k's grains take the grain ids [first_k, first_k + counts[k]) in
 * every state, positions, rhs and history array; its density field is the
 * 4 * nodes_k floats that start at float 4 * node_first_k of the handle's grid
 * (wd_density_grid_nodes gives the sum of nodes_k), laid out channel-major like a
 * single scene's grid. History partners are global grain ids. Each scene's
 * results equal its own single-scene run bit for bit. The scenes must share the
 * time integrator, Picard iteration count, history mode and dt; a batch runs
 * Picard with a fixed iteration count (picard_tolerance 0). radii / masses may be
 * NULL (or hold NULL entries) for the configs' defaults; materials likewise. A NULL
 * states (or a NULL entry) builds that scene from its config's initialization
 * section, as wd_create does; counts is read only for the scenes given a state. */
int wd_create_batch(const wd_config* const* cfgs, int32_t num_scenes, const int64_t* counts,
                    const float* const* states, const int32_t* const* materials,
                    const float* const* radii, const float* const* masses, wd_sim** out);
/* Number of scenes (1 for a handle from wd_create / wd_create_from_arrays). */
int wd_scene_count(const wd_sim* sim, int32_t* scenes);
/* Grain id range and density-node range of one scene. */
int wd_scene_range(const wd_sim* sim, int32_t scene, int64_t* first, int64_t* count,
                   int64_t* node_first, int64_t* nodes);
/* Per scene: energy (FP64, one value per scene) and momentum (3 per scene). */
int wd_compute_scene_energies(wd_sim* sim, double* energies);
int wd_compute_scene_momenta(wd_sim* sim, double* momenta);
/* Per scene: grid_overflow_count() and is_stable() (src/particle_dynamics.cu:311-347),
 * the checks the dataset driver makes of each rollout at every checkpoint
 * (src/dataset.cpp:203-206). A single-scene handle answers for its one scene. */
int wd_scene_overflow_counts(wd_sim* sim, int64_t* counts);
int wd_scene_stability(wd_sim* sim, int32_t* stable);
/* Stop (frozen != 0) or restart one scene of a batch: the step leaves a frozen
 * scene's grains where they are and drops their tangential history. The dataset
 * driver stops a diverged rollout this way (src/dataset.cpp:198-208 stops stepping
 * it). */
int wd_freeze_scene(wd_sim* sim, int32_t scene, int32_t frozen);
/* Ensemble divergence of every scene from reference_scene (src/chaos.cpp:47-78,
 * 190-222), computed on the device from the current state and a fresh density
 * deposit: metrics3[3k] = sqrt(mean_i |x_i^(k) - x_i^(ref)|^2) over grains with the
 * same index, metrics3[3k+1] = ||rho^(k) - rho^(ref)|| / ||rho^(ref)|| (mass
 * channel), metrics3[3k+2] = |com^(k) - com^(ref)| in node units. Every scene needs
 * the same grain count and density grid. */
int wd_chaos_metrics(wd_sim* sim, int32_t reference_scene, double* metrics3);

/* ---- stepping: take_step() (src/particle_dynamics.cu:264-281) -------------------- */

/* nsteps x take_step(), launched asynchronously on the handle's stream. */
int wd_step(wd_sim* sim, int64_t nsteps);

/* dt is re-read at every step, as the reference re-applies sim.dt
 * (src/particle_dynamics.cu:268,276). */
int wd_set_dt(wd_sim* sim, float dt);
int wd_get_dt(const wd_sim* sim, float* dt);
/* Simulated time, float, advanced by dt per step (src/particle_dynamics.cu:280). */
int wd_get_time(const wd_sim* sim, float* time);
int wd_set_time(wd_sim* sim, float time);
int wd_get_n(const wd_sim* sim, int64_t* n);
/* Picard iterations run in the last step and its final residual max|x_{k+1}-x_k|. */
int wd_get_picard_stats(const wd_sim* sim, int32_t* iterations, float* residual);

/* ---- state in and out: host_state / device_state / positions / device_rhs -------- */

/* device_state.copy_from_host(host_state) (src/device_vector.h:30-49): state AoS6. */
int wd_set_state(wd_sim* sim, const float* state);
/* host_state.copy_from_device(device_state): state AoS6 by grain id. */
int wd_get_state(wd_sim* sim, float* state);
/* unpack_state() positions (src/particle_dynamics.cu:109-124): AoS3 by grain id. */
int wd_get_positions(wd_sim* sim, float* positions);
/* device_rhs of the last step (src/particle_dynamics.h:42): AoS6 [v, F/m]. */
int wd_get_rhs(wd_sim* sim, float* rhs);
/* host_mass / host_material per grain, and per-grain radius. */
int wd_get_grain_props(const wd_sim* sim, float* radius, float* mass, int32_t* material);

/* Device-pointer variants for zero-copy callers (PyTorch): the same layouts, in
 * device memory, ordered on the handle's stream. */
int wd_set_state_device(wd_sim* sim, const float* d_state);
int wd_get_state_device(wd_sim* sim, float* d_state);
int wd_get_positions_device(wd_sim* sim, float* d_positions);
/* Use an external stream (cudaStream_t as void*); NULL restores the own stream. */
int wd_set_stream(wd_sim* sim, void* stream);
int wd_get_stream(const wd_sim* sim, void** stream);
/* Block until all work queued on the handle's streams (steps and copies) is done. */
int wd_synchronize(wd_sim* sim);
/* Asynchronous host I/O (extension): uploads and downloads run on two copy streams,
 * through double-buffered device staging, ordered against the steps by events, so a
 * loop of set_state / step / get_positions overlaps the upload of one step with the
 * step before and the download of the step before that. The host buffers (pinned for
 * real overlap) must stay valid and unchanged until wd_synchronize. wd_io_join orders
 * the step stream after every copy issued so far and the copy streams after the step
 * stream's current point. */
int wd_set_state_async(wd_sim* sim, const float* state);
int wd_get_positions_async(wd_sim* sim, float* positions);
int wd_io_join(wd_sim* sim);

/* ---- files and frames ------------------------------------------------------------ */

/* The reference's state file (int32 n + 6n float32 by grain id), readable by its
 * initialize_from_file (src/particle_dynamics.cu:212-235). */
int wd_write_state_file(wd_sim* sim, const char* path);
/* Checkpoint (extension: the reference saves no more than the state file): the state
 * file at path plus "<path>.sidecar" (magic "WDCKPT01", version 1: time, dt, radius,
 * mass, material and the tangential springs by grain id). A handle created from it
 * with the same config continues bit for bit as the saved one would have. Single-scene
 * handles only. */
int wd_write_checkpoint(wd_sim* sim, const char* path);
int wd_create_from_checkpoint(const wd_config* cfg, const char* path, wd_sim** out);
/* The broadcast frame of src/broadcast.cpp:95-108: frame[0..3n) positions by grain id,
 * frame[3n] = simulated time, frame[3n+1..3n+5] = meta5 (real-time ratio,
 * find-neighbors, compute-rhs, take-step and unpack times in ms; NULL: zeros). */
int wd_pack_frame(wd_sim* sim, const float* meta5, float* frame);

/* ---- reverse pass (extension: the reference has no derivatives) ------------------
 * Gradients of a loss on the state at the end of a window of semi-implicit Euler
 * steps with respect to the state at its start and to the contact parameters
 * (mu, restitution, k_n), by a hand-written adjoint of the fused contact + integrator
 * step: the contact set and the clamp / stick-slip / viscous-cap branches of each
 * step are those the forward took. The window is recorded with checkpoints every
 * checkpoint_every steps; the reverse pass replays one segment at a time from its
 * checkpoint. Single-scene handles; semi-implicit Euler only. */

/* mu, restitution and k_n (physics.normal_stiffness; k_t follows as 2/7 k_n unless
 * physics.tangential_stiffness is set) of a live handle. */
int wd_set_contact_params(wd_sim* sim, float mu, float restitution, float k_n);
/* steps x take_step() from the current state, keeping the checkpoints.
 * WD_ERR_CAPACITY if a grain ran out of spring slots in the window. */
int wd_adjoint_record(wd_sim* sim, int64_t steps, int32_t checkpoint_every);
/* Device pointers, AoS3 by grain id: d_gx, d_gv = dL/dx, dL/dv at the window's end
 * (NULL: zero); d_gx0, d_gv0 receive dL/dx, dL/dv at its start (NULL: skipped);
 * theta3 (host) receives dL/dmu, dL/de, dL/dk_n. The handle is left at the window's
 * end, as after wd_adjoint_record. */
int wd_adjoint_backward(wd_sim* sim, const float* d_gx, const float* d_gv, float* d_gx0,
                        float* d_gv0, double* theta3);
/* Adjoint of compute_density_grid at the current state: d_ggrid (device, 4*nodes,
 * channel-major) = dL/dgrid; d_gx, d_gv (device, AoS3 by grain id) receive dL/dx and
 * dL/dv. The CIC weights are differentiated inside their cells. */
int wd_deposit_vjp(wd_sim* sim, const float* d_ggrid, float* d_gx, float* d_gv);

/* ---- tangential history (extension: no reference counterpart) ------------------- */

/* Per grain id: count[n], partner[n*WD_HIST_CAP] (grain id, or -1-2a / -2-2a for the
 * lower / upper wall of axis a), xi[n*WD_HIST_CAP*3] tangential displacement. */
int wd_get_history(wd_sim* sim, int32_t* count, int32_t* partner, float* xi);
int wd_set_history(wd_sim* sim, const int32_t* count, const int32_t* partner,
                   const float* xi);

/* ---- on-demand fields: compute_density_grid / compute_total_energy -------------- */

/* density_grid_nodes() (src/particle_dynamics.cu:283-286). */
int wd_density_grid_nodes(const wd_sim* sim, int64_t* nodes);
/* compute_density_grid() (src/particle_dynamics.cu:289-293): writes 4*nodes floats
 * to grid (host). Deterministic: order-independent fixed-point accumulation. */
int wd_compute_density_grid(wd_sim* sim, float* grid);
int wd_compute_density_grid_device(wd_sim* sim, float* d_grid);
/* compute_total_energy() (src/particle_dynamics.cu:296-308), summed in FP64. Like
 * the reference it re-runs the neighbor search on the current positions first. */
int wd_compute_total_energy(wd_sim* sim, double* energy);
/* Per-grain terms of compute_total_energy, by grain id (n doubles): kinetic, gravity
 * and wall energy of the grain, the pair energy of its contacts with larger-id grains
 * and the spring energy of its stored springs whose partner has a larger id (or is a
 * wall). Summed over any partition of the grains they give the total once; the slab
 * decomposition (world_b200/slab.py) sums its owned grains' and all-reduces. No
 * counterpart in the reference (src/energy_kernel.cu:30-80 sums in one atomic). */
int wd_grain_energies(wd_sim* sim, double* energies);
/* Total momentum sum(m v) in FP64 (extension). */
int wd_compute_momentum(wd_sim* sim, double* momentum3);

/* ---- diagnostics (src/particle_dynamics.cu:311-347) ------------------------------ */

/* is_stable(): every position finite and inside the domain box. */
int wd_is_stable(wd_sim* sim, int32_t* stable);
/* compute_max_acceleration(): max |F/m| of the last step's rhs. */
int wd_compute_max_acceleration(wd_sim* sim, float* max_accel);
/* grid_overflow_count(): lifetime count of (cell, search) incidents with more than
 * particles_per_cell grains in a cell (src/find_neighbors_kernel.cu:230-234). No
 * grain is dropped here: the sorted search has no per-cell capacity. */
int wd_grid_overflow_count(wd_sim* sim, int64_t* count);
/* Switch the Verlet-list skin of a live handle (0: grid search every step). The
 * trajectory does not depend on it. */
int wd_set_neighbor_skin(wd_sim* sim, float skin);
/* Autotuner (extension): times `steps` steps for each neighbor skin in {0, 0.05,
 * 0.1, 0.15, 0.2, 0.3, 0.4} mean diameters, contact-kernel block size in {128, 256} and, with
 * lists, its variant (per-lane with 48 or 64 registers, warp-cooperative, bulk-staged)
 * from the same saved state, keeps
 * the fastest and restores the state (results do not depend on the choice). With
 * cache_path, a line "key skin block variant" keyed by grain count,
 * scenes, grid, SM count, history, integrator and launch mode is reused or appended.
 * skin_out / block_out (may be NULL) receive the choice. */
int wd_autotune(wd_sim* sim, int32_t steps, const char* cache_path, float* skin_out,
                int32_t* block_out);
/* The current schedule: neighbor skin, contact-kernel block size, and the list
 * contact kernel variant: 48 or 64 (registers per thread of the per-lane kernel), 0
 * (the warp-cooperative kernel, 256 threads) or 1 / 2 (the bulk-staged persistent
 * kernel, 256 threads, 48 / 64 registers: per-slot arrays copied into shared memory by
 * cp.async.bulk two tiles ahead). wd_set_contact_kernel sets the last two (the
 * autotuner's other choices); results do not depend on them. */
int wd_get_tuning(const wd_sim* sim, float* skin, int32_t* block, int32_t* variant);
int wd_set_contact_kernel(wd_sim* sim, int32_t block, int32_t variant);
/* Verlet-list build kernel (no counterpart in the reference): 0 (default) one thread per
 * grain reading its candidates from global memory; 1 each block of 256 grains stages the
 * union of its stencil rows in shared memory by bulk copies first (single scenes; the
 * same lists). Measured on a B200, 2^20-grain collapsed column: 0.185 ms per build with
 * 0, 0.24 ms with 1. */
int wd_set_build_kernel(wd_sim* sim, int32_t tiled);
/* Test hook for the bulk-staged contact kernel's bounded waits (no counterpart in the
 * reference). wait_us: the limit of each wait for a stage of bulk copies (0: one
 * second). stall != 0: each warp's first stage is made to expect 16 bytes that no copy
 * delivers, so its wait runs out; the kernel then returns without finishing that warp's
 * tiles, and the next synchronizing call returns WD_ERR_CUDA once with "did not
 * complete within its wait limit". The state of that step is invalid, slot order
 * included: restore one with wd_set_state (which then starts from the grain-id order
 * and no stored springs; wd_set_history restores those). No copy is ever left in
 * flight. Handles with Verlet lists only. */
int wd_debug_stage_wait(wd_sim* sim, int32_t stall, int32_t wait_us);
/* Verlet lists: steps so far whose contact kernel measured the exact displacement
 * since the build (reading the build positions). The other steps decide on a bound:
 * the last exact value plus the largest per-step displacement of each step since. */
int wd_list_exact_count(wd_sim* sim, int64_t* steps);
/* Lifetime count of (grain, step) pairs in which the list contact kernels found a
 * grain's contacts out of the canonical visiting order (a cell crossing since the last
 * build) and evaluated them in sorted order instead (no counterpart in the reference). */
int wd_list_resort_count(wd_sim* sim, int64_t* grains);
/* Backward Euler / Picard: iterations executed so far (iterations that a converged
 * step skipped are not counted), and, on Verlet lists, the steps whose iterate went
 * beyond the lists' validity bound and that were redone with the per-iteration search
 * (their iterations count twice). */
int wd_picard_counts(wd_sim* sim, int64_t* iterations, int64_t* redos);
/* Verlet lists (simulation.neighbor_skin > 0): builds so far, kernels one build
 * launches, and the mean list length of the last build (0 without lists). */
int wd_list_stats(wd_sim* sim, int64_t* builds, int32_t* kernels_each, double* mean_length);
/* Lifetime count of contacts that found no free history slot (WD_HIST_CAP). */
int wd_history_overflow_count(wd_sim* sim, int64_t* count);
/* find_neighbors_wct / compute_rhs_wct / take_step_wct / density_grid_wct
 * (src/particle_dynamics.cu:350-358): lifetime ms, recorded when
 * drivers.kernel_timing is true. The contact kernel integrates in its epilogue, so
 * take_step_wct stays 0 and compute_rhs_wct covers forces plus integration. */
int wd_timings(wd_sim* sim, float* ms4);
/* Switch drivers.kernel_timing at run time (the reference fixes it at construction,
 * src/sim_config.h:165): 1 = direct launches with events per phase, 0 = one graph
 * launch per step. */
int wd_set_kernel_timing(wd_sim* sim, int32_t enabled);
/* Lifetime count of neighbor searches that ran the full radix sort (first search, or
 * more grains changing cell than the incremental path takes); *kernels_each
 * receives the kernels such a search adds. */
int wd_radix_search_count(wd_sim* sim, int64_t* count, int32_t* kernels_each);
/* Kernels one step launches on the incremental search path (launch accounting). */
int wd_kernels_per_step(const wd_sim* sim, int64_t* kernels);

/* ---- allocation-free CIC deposit (no counterpart in the reference) ---------------
 * For callers that cannot call cudaMalloc: processes whose device memory is owned by
 * another framework's allocator (an ML runtime that reserves the GPU's memory up
 * front, PyTorch's caching allocator holding the pool) and loops that must not
 * allocate while they run. Same field as wd_compute_density_grid, from caller-owned
 * device arrays: d_state AoS6 per grain, d_mass per grain (0 skips the grain), the
 * node-centred grid [lo, hi] with size[a] nodes per axis, d_grid = 4*nodes floats.
 * The scratch (64-bit accumulators and channel bounds) is one static device array
 * sized for WD_NOALLOC_MAX_NODES nodes (8 MiB), held by every GPU that loads the
 * library until the process exits; larger grids return WD_ERR_CAPACITY. Every call
 * looks that array's address up in the current context (cudaGetSymbolAddress, host
 * side only), so it stays valid after cudaDeviceReset; the first call on a device
 * also loads the library's device code there and should come before any stream
 * capture. Every call shares the array and clears it first, so calls that overlap on
 * the GPU (different streams or threads) race. A NaN or infinite mass or momentum
 * makes its whole channel NaN. Work is queued on `stream` (cudaStream_t as void*,
 * NULL = default stream). */
#define WD_NOALLOC_MAX_NODES (64 * 64 * 64)
int wd_deposit_grid_noalloc(const float* d_state, const float* d_mass, int64_t n,
                            const float* lo3, const float* hi3, const int32_t* size3,
                            float* d_grid, void* stream);

/* ---- parity probes: the reference's public device_neighbors buffer
 * (src/particle_dynamics.h:48-52) and its cell mapping -------------------------- */

/* Cell key of every grain at the current positions, by grain id
 * (src/find_neighbors_kernel.cu:11-40). */
int wd_debug_cell_keys(wd_sim* sim, int32_t* keys);
/* The sorted order of the last neighbor search: cell key and grain id per slot,
 * ascending by (key, id). */
int wd_debug_sorted(wd_sim* sim, int32_t* keys, int32_t* ids);
/* Candidate lists at the current positions, CSR by grain id: offsets[n+1];
 * cand[offsets[i]..offsets[i+1]) in stencil order, ids ascending inside a cell;
 * contact[k] = 1 when that pair overlaps. *total receives the candidate count;
 * cand/contact are written only when it fits in cap. */
int wd_debug_candidates(wd_sim* sim, int64_t* offsets, int32_t* cand, uint8_t* contact,
                        int64_t cap, int64_t* total);

#ifdef __cplusplus
}
#endif
#endif
