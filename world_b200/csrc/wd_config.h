// wd_config.h -- host-side configuration of the DEM step.
//
// Same fields, defaults and YAML semantics as the reference's SimConfig / load_config
// (src/sim_config.h:28-205, src/sim_config.cpp:54-195). New keys live in the existing
// sections and default to the reference's behaviour when absent:
//   simulation.history            false  -> viscous tangential friction (reference)
//   simulation.neighbor_skin      0      -> neighbor search every step (reference); > 0:
//                                           Verlet lists with this skin (m), rebuilt when
//                                           a grain has moved 0.49 skin since the build
//   physics.normal_stiffness      0      -> k_n = max_force / particle_radius
//   physics.tangential_stiffness  0      -> k_t = 2/7 k_n when history is on
//   physics.density               0      -> masses from the material table
//   time_integration.picard_tolerance 0  -> fixed picard_iterations (reference)
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace wd {

struct Config {
    // simulation
    float dt = 0.0001f;
    int grid[3] = {32, 32, 32};
    int particles_per_cell = 64;
    int threads_per_block = 256;
    int dgrid[3] = {32, 32, 32};
    bool history = false;
    float neighbor_skin = 0.f;
    // domain
    float dom_lo[3] = {-1.f, -1.f, -1.f};
    float dom_hi[3] = {1.f, 1.f, 1.f};
    // physics
    float gravity = 9.81f;
    float particle_radius = 0.01f;
    float max_force = 100.f;
    float floor_z = -1.f, ceiling_z = 1.f;
    float wall_x_min = -1.f, wall_x_max = 1.f, wall_y_min = -1.f, wall_y_max = 1.f;
    float restitution = 0.3f;
    float friction = 0.5f;
    float normal_stiffness = 0.f;
    float tangential_stiffness = 0.f;
    float density = 0.f;
    // materials
    std::vector<float> masses{0.f, 0.04f};
    // initialization
    std::string init_type = "cube";
    std::string init_state_path;
    float init_x0 = -0.5f, init_y0 = 0.f, init_z0 = 0.f;
    float init_vx0 = 0.f, init_vy0 = 0.f, init_vz0 = 0.f;
    float init_jitter = 0.f;
    unsigned init_seed = 12345u;
    float init_perturbation = 0.f;
    unsigned init_perturbation_seed = 1u;
    float cube_length[3] = {0.2f, 0.2f, 0.2f};
    float two_particle_separation = 0.1f;
    int particle_material = 1;
    // rendering / drivers (kept so every reference file loads without warnings)
    int num_triangles = 20;
    int port = 8081;
    int steps_per_frame = 10;
    int profiling_outer_iters = 10;
    int profiling_steps_per_iter = 10;
    bool kernel_timing = true;
    std::vector<float> sweep_dt, sweep_max_force, sweep_restitution;
    std::string stability_mode = "fixed_time";
    float stability_sim_time = 0.1f;
    float stability_acceleration_cutoff = 0.01f;
    int stability_steps_per_steadiness_check = 100;
    float model_problem_sim_time = 1.0f;
    float dataset_sim_time = 2.0f;
    int dataset_checkpoints = 10;
    // time integration
    std::string time_integrator = "semi_implicit_euler";
    int picard_iterations = 3;
    float picard_tolerance = 0.f;
};

// Status values shared with the C ABI.
enum Status : int {
    kOk = 0,
    kWarnDefaults = 1,
    kWarnUnknownKey = 2,
    kErrInvalid = -1,
    kErrCuda = -2,
    kErrIo = -3,
    kErrConfig = -4,
    kErrOom = -5,
    kErrCapacity = -6,
};

// Set one section.key from text; returns kOk, kWarnUnknownKey or kErrConfig.
int config_set(Config& cfg, const std::string& section, const std::string& key,
               const std::string& value, std::string* err);
// Read one section.key as text; kErrInvalid for unknown keys.
int config_get(const Config& cfg, const std::string& section, const std::string& key,
               std::string* out);
// Apply a YAML file on top of cfg; kWarnDefaults if the file cannot be opened.
int config_load_yaml(Config& cfg, const std::string& path, std::string* err);

// Initial grains built from cfg's initialization section.
struct Grains {
    std::vector<float> state;     // 6n AoS
    std::vector<int32_t> material;
};
int build_initial_grains(const Config& cfg, Grains* out, std::string* err);

// Thread-local last-error message of the C ABI.
void set_last_error(const std::string& msg);

}  // namespace wd
