// particle_dynamics.hpp -- header-only C++ drop-in for the reference's ParticleDynamics,
// SimConfig and load_config (src/particle_dynamics.h:17-141, src/sim_config.h:14-205),
// implemented over the C ABI of libworld_b200.so (include/world_b200.h).
//
// The reference's drivers and tests use these names unqualified; they are declared in
// namespace world_b200 and, unless WORLD_B200_NO_GLOBAL_NAMES is defined, brought into
// the global namespace. Members keep the reference's names and meanings:
//   config, time, n, dt (writable: re-applied at the next take_step, as the reference
//   re-reads it), positions, host_state, device_state.copy_from_host(host_state),
//   host_mass (material table), host_material, host_density_grid, grid sizes,
//   take_step, unpack_state, compute_density_grid, density_grid_nodes,
//   compute_total_energy, is_stable, compute_max_acceleration, grid_overflow_count,
//   find_neighbors_wct / compute_rhs_wct / take_step_wct / density_grid_wct.
// Where the reference aborts or exits on an error, these throw std::runtime_error.
#pragma once

#include <chrono>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../world_b200.h"

namespace world_b200 {

constexpr int kDim = 3;
constexpr int kStateStride = 2 * kDim;
constexpr int kStencilCells = 27;

struct DomainParams {
    float x_min, x_max, y_min, y_max, z_min, z_max;
};

struct PhysicsParams {
    float gravity;
    float particle_radius;
    float max_force;
    float floor_z, ceiling_z, wall_x_min, wall_x_max, wall_y_min, wall_y_max;
    float restitution;
    float friction;
    // extensions (0 = the reference's behaviour)
    float normal_stiffness = 0.f;
    float tangential_stiffness = 0.f;
    float density = 0.f;
};

// Same members and defaults as the reference's SimConfig (src/sim_config.h:64-200),
// plus the library's extension keys.
struct SimConfig {
    float dt = 0.0001f;
    int collision_grid_size_x = 32, collision_grid_size_y = 32, collision_grid_size_z = 32;
    int particles_per_cell = 64;
    int threads_per_block = 256;
    int density_grid_size_x = 32, density_grid_size_y = 32, density_grid_size_z = 32;
    DomainParams domain{-1.0f, 1.0f, -1.0f, 1.0f, -1.0f, 1.0f};
    PhysicsParams physics{9.81f, 0.01f, 100.0f, -1.0f, 1.0f, -1.0f, 1.0f, -1.0f, 1.0f, 0.3f, 0.5f};
    std::vector<float> masses{0.0f, 0.04f};
    std::string init_type = "cube";
    std::string init_state_path = "";
    float init_x0 = -0.5f, init_y0 = 0.0f, init_z0 = 0.0f;
    float init_vx0 = 0.0f, init_vy0 = 0.0f, init_vz0 = 0.0f;
    float init_jitter = 0.0f;
    unsigned int init_seed = 12345u;
    float init_perturbation = 0.0f;
    unsigned int init_perturbation_seed = 1u;
    float cube_length_x = 0.2f, cube_length_y = 0.2f, cube_length_z = 0.2f;
    float two_particle_separation = 0.1f;
    int particle_material = 1;
    int num_triangles = 20;
    int port = 8081;
    int steps_per_frame = 10;
    int profiling_outer_iters = 10;
    int profiling_steps_per_iter = 10;
    bool kernel_timing = true;
    std::vector<float> sweep_dt{}, sweep_max_force{}, sweep_restitution{};
    std::string stability_mode = "fixed_time";
    float stability_sim_time = 0.1f;
    float stability_acceleration_cutoff = 0.01f;
    int stability_steps_per_steadiness_check = 100;
    float model_problem_sim_time = 1.0f;
    float dataset_sim_time = 2.0f;
    int dataset_checkpoints = 10;
    std::string time_integrator = "semi_implicit_euler";
    int picard_iterations = 3;
    // extensions
    bool history = false;
    float picard_tolerance = 0.0f;
    float neighbor_skin = 0.0f;
};

namespace detail {

inline void check(int status, const char* what) {
    if (status < 0) throw std::runtime_error(std::string(what) + ": " + wd_last_error());
}

inline std::string ftext(float v) {
    char b[48];
    std::snprintf(b, sizeof(b), "%.9g", static_cast<double>(v));
    return b;
}

inline std::string ltext(const std::vector<float>& v) {
    std::string s = "[";
    for (size_t i = 0; i < v.size(); ++i) s += (i ? ", " : "") + ftext(v[i]);
    return s + "]";
}

// Visit every (section, key, member) of SimConfig; `io` reads or writes it.
template <typename Io>
void visit(SimConfig& c, Io&& io) {
    io("simulation", "dt", c.dt);
    io("simulation", "collision_grid_size_x", c.collision_grid_size_x);
    io("simulation", "collision_grid_size_y", c.collision_grid_size_y);
    io("simulation", "collision_grid_size_z", c.collision_grid_size_z);
    io("simulation", "particles_per_cell", c.particles_per_cell);
    io("simulation", "threads_per_block", c.threads_per_block);
    io("simulation", "density_grid_size_x", c.density_grid_size_x);
    io("simulation", "density_grid_size_y", c.density_grid_size_y);
    io("simulation", "density_grid_size_z", c.density_grid_size_z);
    io("simulation", "history", c.history);
    io("simulation", "neighbor_skin", c.neighbor_skin);
    io("domain", "x_min", c.domain.x_min);
    io("domain", "x_max", c.domain.x_max);
    io("domain", "y_min", c.domain.y_min);
    io("domain", "y_max", c.domain.y_max);
    io("domain", "z_min", c.domain.z_min);
    io("domain", "z_max", c.domain.z_max);
    io("physics", "gravity", c.physics.gravity);
    io("physics", "particle_radius", c.physics.particle_radius);
    io("physics", "max_force", c.physics.max_force);
    io("physics", "floor_z", c.physics.floor_z);
    io("physics", "ceiling_z", c.physics.ceiling_z);
    io("physics", "wall_x_min", c.physics.wall_x_min);
    io("physics", "wall_x_max", c.physics.wall_x_max);
    io("physics", "wall_y_min", c.physics.wall_y_min);
    io("physics", "wall_y_max", c.physics.wall_y_max);
    io("physics", "restitution", c.physics.restitution);
    io("physics", "friction", c.physics.friction);
    io("physics", "normal_stiffness", c.physics.normal_stiffness);
    io("physics", "tangential_stiffness", c.physics.tangential_stiffness);
    io("physics", "density", c.physics.density);
    io("materials", "masses", c.masses);
    io("initialization", "type", c.init_type);
    io("initialization", "state_path", c.init_state_path);
    io("initialization", "x0", c.init_x0);
    io("initialization", "y0", c.init_y0);
    io("initialization", "z0", c.init_z0);
    io("initialization", "vx0", c.init_vx0);
    io("initialization", "vy0", c.init_vy0);
    io("initialization", "vz0", c.init_vz0);
    io("initialization", "jitter", c.init_jitter);
    io("initialization", "seed", c.init_seed);
    io("initialization", "perturbation", c.init_perturbation);
    io("initialization", "perturbation_seed", c.init_perturbation_seed);
    io("initialization", "cube_length_x", c.cube_length_x);
    io("initialization", "cube_length_y", c.cube_length_y);
    io("initialization", "cube_length_z", c.cube_length_z);
    io("initialization", "two_particle_separation", c.two_particle_separation);
    io("initialization", "particle_material", c.particle_material);
    io("rendering", "num_triangles", c.num_triangles);
    io("drivers", "port", c.port);
    io("drivers", "steps_per_frame", c.steps_per_frame);
    io("drivers", "profiling_outer_iters", c.profiling_outer_iters);
    io("drivers", "profiling_steps_per_iter", c.profiling_steps_per_iter);
    io("drivers", "kernel_timing", c.kernel_timing);
    io("sweep", "dt", c.sweep_dt);
    io("sweep", "max_force", c.sweep_max_force);
    io("sweep", "restitution", c.sweep_restitution);
    io("stability", "mode", c.stability_mode);
    io("stability", "sim_time", c.stability_sim_time);
    io("stability", "acceleration_cutoff", c.stability_acceleration_cutoff);
    io("stability", "steps_per_steadiness_check", c.stability_steps_per_steadiness_check);
    io("model_problem", "sim_time", c.model_problem_sim_time);
    io("dataset", "sim_time", c.dataset_sim_time);
    io("dataset", "checkpoints", c.dataset_checkpoints);
    io("time_integration", "solver", c.time_integrator);
    io("time_integration", "picard_iterations", c.picard_iterations);
    io("time_integration", "picard_tolerance", c.picard_tolerance);
}

struct Writer {
    wd_config* cfg;
    void put(const char* s, const char* k, const std::string& v) {
        check(wd_config_set(cfg, s, k, v.c_str()), "wd_config_set");
    }
    void operator()(const char* s, const char* k, float& v) { put(s, k, ftext(v)); }
    void operator()(const char* s, const char* k, int& v) { put(s, k, std::to_string(v)); }
    void operator()(const char* s, const char* k, unsigned& v) { put(s, k, std::to_string(v)); }
    void operator()(const char* s, const char* k, bool& v) { put(s, k, v ? "true" : "false"); }
    void operator()(const char* s, const char* k, std::string& v) { put(s, k, v); }
    void operator()(const char* s, const char* k, std::vector<float>& v) { put(s, k, ltext(v)); }
};

struct Reader {
    const wd_config* cfg;
    std::string get(const char* s, const char* k) {
        char buf[4096];
        check(wd_config_get(cfg, s, k, buf, sizeof(buf)), "wd_config_get");
        return buf;
    }
    void operator()(const char* s, const char* k, float& v) { v = std::stof(get(s, k)); }
    void operator()(const char* s, const char* k, int& v) { v = std::stoi(get(s, k)); }
    void operator()(const char* s, const char* k, unsigned& v) {
        v = static_cast<unsigned>(std::stoul(get(s, k)));
    }
    void operator()(const char* s, const char* k, bool& v) { v = get(s, k) == "true"; }
    void operator()(const char* s, const char* k, std::string& v) { v = get(s, k); }
    void operator()(const char* s, const char* k, std::vector<float>& v) {
        const std::string t = get(s, k);
        v.clear();
        size_t i = 1;
        while (i < t.size()) {
            const size_t j = t.find_first_of(",]", i);
            const std::string item = t.substr(i, j - i);
            if (item.find_first_not_of(" ") != std::string::npos) v.push_back(std::stof(item));
            if (j == std::string::npos || t[j] == ']') break;
            i = j + 1;
        }
    }
};

struct ConfigHandle {
    wd_config* p = nullptr;
    ConfigHandle() { check(wd_config_create(&p), "wd_config_create"); }
    ~ConfigHandle() { wd_config_destroy(p); }
    ConfigHandle(const ConfigHandle&) = delete;
    ConfigHandle& operator=(const ConfigHandle&) = delete;
};

}  // namespace detail

// load_config(path) (src/sim_config.cpp:153-195): defaults, then the file's keys.
inline SimConfig load_config(const std::string& path) {
    detail::ConfigHandle h;
    detail::check(wd_config_load_yaml(h.p, path.c_str()), "load_config");
    SimConfig c;
    detail::visit(c, detail::Reader{h.p});
    return c;
}

class ParticleDynamics {
public:
    // device_state.copy_from_host(host_state), as the reference's tests push edits.
    struct DeviceState {
        ParticleDynamics* owner;
        void copy_from_host(const std::vector<float>& host) {
            detail::check(wd_set_state(owner->sim_, host.data()), "device_state.copy_from_host");
        }
    };

    SimConfig config;
    float time = 0.f;
    float last_time = 0.f;
    std::chrono::steady_clock::time_point last_wall_clock_time;
    float real_time_ratio = 0.f;
    int n = 0;
    float dt = 0.f;
    int collision_grid_size_x, collision_grid_size_y, collision_grid_size_z;
    int particles_per_cell;
    std::vector<float> positions;
    std::vector<float> host_state;
    DeviceState device_state{this};
    std::vector<int> host_material;
    std::vector<float> host_mass;
    std::vector<float> host_density_grid;
    int density_grid_size_x, density_grid_size_y, density_grid_size_z;
    float time_unpack_state = 0.f;

    explicit ParticleDynamics(const SimConfig& config_ = SimConfig{}) : config(config_) {
        detail::ConfigHandle h;
        detail::visit(config, detail::Writer{h.p});
        detail::check(wd_create(h.p, &sim_), "ParticleDynamics");
        int64_t count = 0;
        wd_get_n(sim_, &count);
        n = static_cast<int>(count);
        dt = config.dt;
        applied_dt_ = dt;
        collision_grid_size_x = config.collision_grid_size_x;
        collision_grid_size_y = config.collision_grid_size_y;
        collision_grid_size_z = config.collision_grid_size_z;
        particles_per_cell = config.particles_per_cell;
        density_grid_size_x = config.density_grid_size_x;
        density_grid_size_y = config.density_grid_size_y;
        density_grid_size_z = config.density_grid_size_z;
        positions.resize(static_cast<size_t>(kDim) * n);
        host_state.resize(static_cast<size_t>(kStateStride) * n);
        host_material.resize(n);
        wd_get_grain_props(sim_, nullptr, nullptr, host_material.data());
        host_mass = config.masses;
        host_density_grid.resize(4 * density_grid_nodes());
        last_wall_clock_time = std::chrono::steady_clock::now();
        unpack_state();
    }

    ~ParticleDynamics() { wd_destroy(sim_); }
    ParticleDynamics(const ParticleDynamics&) = delete;
    ParticleDynamics& operator=(const ParticleDynamics&) = delete;

    void take_step() {
        if (dt != applied_dt_) {
            detail::check(wd_set_dt(sim_, dt), "wd_set_dt");
            applied_dt_ = dt;
        }
        detail::check(wd_step(sim_, 1), "take_step");
        time += dt;
    }

    void unpack_state() {
        const auto t0 = std::chrono::steady_clock::now();
        detail::check(wd_get_state(sim_, host_state.data()), "unpack_state");
        for (int i = 0; i < n; ++i)
            for (int a = 0; a < kDim; ++a)
                positions[static_cast<size_t>(kDim) * i + a] = host_state[static_cast<size_t>(kStateStride) * i + a];
        time_unpack_state = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        real_time_ratio = get_real_time_ratio();
    }

    float get_real_time_ratio() {
        const auto now = std::chrono::steady_clock::now();
        const double wall = std::chrono::duration<double>(now - last_wall_clock_time).count();
        const float ratio = wall > 0.0 ? (time - last_time) / static_cast<float>(wall) : 0.f;
        last_time = time;
        last_wall_clock_time = now;
        return ratio;
    }

    size_t density_grid_nodes() const {
        int64_t nodes = 0;
        wd_density_grid_nodes(sim_, &nodes);
        return static_cast<size_t>(nodes);
    }

    size_t compute_density_grid() {
        detail::check(wd_compute_density_grid(sim_, host_density_grid.data()), "compute_density_grid");
        return host_density_grid.size();
    }

    float compute_total_energy() {
        double e = 0.0;
        detail::check(wd_compute_total_energy(sim_, &e), "compute_total_energy");
        return static_cast<float>(e);
    }

    bool is_stable() {
        int32_t ok = 0;
        detail::check(wd_is_stable(sim_, &ok), "is_stable");
        return ok != 0;
    }

    float compute_max_acceleration() {
        float a = 0.f;
        detail::check(wd_compute_max_acceleration(sim_, &a), "compute_max_acceleration");
        return a;
    }

    int grid_overflow_count() const {
        int64_t c = 0;
        detail::check(wd_grid_overflow_count(sim_, &c), "grid_overflow_count");
        return static_cast<int>(c);
    }

    float find_neighbors_wct() const { return timing(0); }
    float compute_rhs_wct() const { return timing(1); }
    float take_step_wct() const { return timing(2); }
    float density_grid_wct() const { return timing(3); }

    wd_sim* handle() const { return sim_; }

private:
    wd_sim* sim_ = nullptr;
    float applied_dt_ = 0.f;

    float timing(int which) const {
        float ms[4] = {0.f, 0.f, 0.f, 0.f};
        detail::check(wd_timings(sim_, ms), "wd_timings");
        return ms[which];
    }
};

}  // namespace world_b200

#ifndef WORLD_B200_NO_GLOBAL_NAMES
using world_b200::DomainParams;
using world_b200::kDim;
using world_b200::kStateStride;
using world_b200::kStencilCells;
using world_b200::load_config;
using world_b200::ParticleDynamics;
using world_b200::PhysicsParams;
using world_b200::SimConfig;
#endif
