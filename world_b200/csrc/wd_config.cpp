// wd_config.cpp -- YAML-subset loader and initial-state builders.
//
// Parsing follows src/sim_config.cpp:14-195 line for line in behaviour: comments
// start at '#', a bare "name:" opens a section, "key: value" assigns, "[a, b]" is a
// float list, unknown keys warn and are skipped, a missing file keeps the defaults.
// Where the reference lets std::stof/std::stoi throw (and the process terminate),
// this returns kErrConfig with the offending line instead.
#include "wd_config.h"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <functional>
#include <random>
#include <sstream>

namespace wd {

namespace {

thread_local std::string t_last_error;

std::string trim(const std::string& s) {
    const std::size_t first = s.find_first_not_of(" \t\r\n");
    if (first == std::string::npos) return "";
    const std::size_t last = s.find_last_not_of(" \t\r\n");
    return s.substr(first, last - first + 1);
}

std::string unquote(const std::string& s) {
    if (s.size() >= 2 && (s.front() == '"' || s.front() == '\'') && s.back() == s.front())
        return s.substr(1, s.size() - 2);
    return s;
}

std::vector<float> parse_float_list(const std::string& value) {
    std::vector<float> out;
    std::string inner = trim(value);
    if (inner.size() >= 2 && inner.front() == '[' && inner.back() == ']')
        inner = inner.substr(1, inner.size() - 2);
    std::stringstream ss(inner);
    std::string item;
    while (std::getline(ss, item, ',')) {
        const std::string t = trim(item);
        if (!t.empty()) out.push_back(std::stof(t));
    }
    return out;
}

std::string fmt_float(float v) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.9g", static_cast<double>(v));
    return buf;
}

std::string fmt_list(const std::vector<float>& v) {
    std::string s = "[";
    for (size_t i = 0; i < v.size(); ++i) {
        if (i) s += ", ";
        s += fmt_float(v[i]);
    }
    return s + "]";
}

enum class Kind { F, I, U, B, S, SQ, L };

struct Entry {
    const char* section;
    const char* key;
    Kind kind;
    std::function<void*(Config&)> field;
};

#define WD_E(sec, key, kind, member) \
    Entry{sec, key, kind, [](Config& c) -> void* { return static_cast<void*>(&(c.member)); }}

const std::vector<Entry>& registry() {
    static const std::vector<Entry> entries = {
        WD_E("simulation", "dt", Kind::F, dt),
        WD_E("simulation", "collision_grid_size_x", Kind::I, grid[0]),
        WD_E("simulation", "collision_grid_size_y", Kind::I, grid[1]),
        WD_E("simulation", "collision_grid_size_z", Kind::I, grid[2]),
        WD_E("simulation", "particles_per_cell", Kind::I, particles_per_cell),
        WD_E("simulation", "threads_per_block", Kind::I, threads_per_block),
        WD_E("simulation", "density_grid_size_x", Kind::I, dgrid[0]),
        WD_E("simulation", "density_grid_size_y", Kind::I, dgrid[1]),
        WD_E("simulation", "density_grid_size_z", Kind::I, dgrid[2]),
        WD_E("simulation", "history", Kind::B, history),
        WD_E("simulation", "neighbor_skin", Kind::F, neighbor_skin),
        WD_E("domain", "x_min", Kind::F, dom_lo[0]),
        WD_E("domain", "x_max", Kind::F, dom_hi[0]),
        WD_E("domain", "y_min", Kind::F, dom_lo[1]),
        WD_E("domain", "y_max", Kind::F, dom_hi[1]),
        WD_E("domain", "z_min", Kind::F, dom_lo[2]),
        WD_E("domain", "z_max", Kind::F, dom_hi[2]),
        WD_E("physics", "gravity", Kind::F, gravity),
        WD_E("physics", "particle_radius", Kind::F, particle_radius),
        WD_E("physics", "max_force", Kind::F, max_force),
        WD_E("physics", "floor_z", Kind::F, floor_z),
        WD_E("physics", "ceiling_z", Kind::F, ceiling_z),
        WD_E("physics", "wall_x_min", Kind::F, wall_x_min),
        WD_E("physics", "wall_x_max", Kind::F, wall_x_max),
        WD_E("physics", "wall_y_min", Kind::F, wall_y_min),
        WD_E("physics", "wall_y_max", Kind::F, wall_y_max),
        WD_E("physics", "restitution", Kind::F, restitution),
        WD_E("physics", "friction", Kind::F, friction),
        WD_E("physics", "normal_stiffness", Kind::F, normal_stiffness),
        WD_E("physics", "tangential_stiffness", Kind::F, tangential_stiffness),
        WD_E("physics", "density", Kind::F, density),
        WD_E("materials", "masses", Kind::L, masses),
        WD_E("initialization", "type", Kind::SQ, init_type),
        WD_E("initialization", "state_path", Kind::SQ, init_state_path),
        WD_E("initialization", "x0", Kind::F, init_x0),
        WD_E("initialization", "y0", Kind::F, init_y0),
        WD_E("initialization", "z0", Kind::F, init_z0),
        WD_E("initialization", "vx0", Kind::F, init_vx0),
        WD_E("initialization", "vy0", Kind::F, init_vy0),
        WD_E("initialization", "vz0", Kind::F, init_vz0),
        WD_E("initialization", "jitter", Kind::F, init_jitter),
        WD_E("initialization", "seed", Kind::U, init_seed),
        WD_E("initialization", "perturbation", Kind::F, init_perturbation),
        WD_E("initialization", "perturbation_seed", Kind::U, init_perturbation_seed),
        WD_E("initialization", "cube_length_x", Kind::F, cube_length[0]),
        WD_E("initialization", "cube_length_y", Kind::F, cube_length[1]),
        WD_E("initialization", "cube_length_z", Kind::F, cube_length[2]),
        WD_E("initialization", "two_particle_separation", Kind::F, two_particle_separation),
        WD_E("initialization", "particle_material", Kind::I, particle_material),
        WD_E("rendering", "num_triangles", Kind::I, num_triangles),
        WD_E("drivers", "port", Kind::I, port),
        WD_E("drivers", "steps_per_frame", Kind::I, steps_per_frame),
        WD_E("drivers", "profiling_outer_iters", Kind::I, profiling_outer_iters),
        WD_E("drivers", "profiling_steps_per_iter", Kind::I, profiling_steps_per_iter),
        WD_E("drivers", "kernel_timing", Kind::B, kernel_timing),
        WD_E("sweep", "dt", Kind::L, sweep_dt),
        WD_E("sweep", "max_force", Kind::L, sweep_max_force),
        WD_E("sweep", "restitution", Kind::L, sweep_restitution),
        WD_E("stability", "mode", Kind::SQ, stability_mode),
        WD_E("stability", "sim_time", Kind::F, stability_sim_time),
        WD_E("stability", "acceleration_cutoff", Kind::F, stability_acceleration_cutoff),
        WD_E("stability", "steps_per_steadiness_check", Kind::I,
             stability_steps_per_steadiness_check),
        WD_E("model_problem", "sim_time", Kind::F, model_problem_sim_time),
        WD_E("dataset", "sim_time", Kind::F, dataset_sim_time),
        WD_E("dataset", "checkpoints", Kind::I, dataset_checkpoints),
        // The reference stores the solver name without unquoting
        // (src/sim_config.cpp:148); kept as is.
        WD_E("time_integration", "solver", Kind::S, time_integrator),
        WD_E("time_integration", "picard_iterations", Kind::I, picard_iterations),
        WD_E("time_integration", "picard_tolerance", Kind::F, picard_tolerance),
    };
    return entries;
}

#undef WD_E

const Entry* find_entry(const std::string& section, const std::string& key) {
    for (const Entry& e : registry())
        if (section == e.section && key == e.key) return &e;
    return nullptr;
}

}  // namespace

void set_last_error(const std::string& msg) { t_last_error = msg; }
const char* last_error_cstr() { return t_last_error.c_str(); }

int config_set(Config& cfg, const std::string& section, const std::string& key,
               const std::string& value, std::string* err) {
    const Entry* e = find_entry(section, key);
    if (!e) {
        std::fprintf(stderr, "load_config: ignoring unknown key '%s.%s'\n", section.c_str(),
                     key.c_str());
        return kWarnUnknownKey;
    }
    void* field = e->field(cfg);
    try {
        switch (e->kind) {
            case Kind::F: *static_cast<float*>(field) = std::stof(value); break;
            case Kind::I: *static_cast<int*>(field) = std::stoi(value); break;
            case Kind::U:
                *static_cast<unsigned*>(field) = static_cast<unsigned>(std::stoi(value));
                break;
            case Kind::B: *static_cast<bool*>(field) = (value == "true"); break;
            case Kind::S: *static_cast<std::string*>(field) = value; break;
            case Kind::SQ: *static_cast<std::string*>(field) = unquote(value); break;
            case Kind::L: *static_cast<std::vector<float>*>(field) = parse_float_list(value); break;
        }
    } catch (const std::exception&) {
        if (err) *err = "config: cannot parse '" + value + "' for '" + section + "." + key + "'";
        return kErrConfig;
    }
    return kOk;
}

int config_get(const Config& cfg_in, const std::string& section, const std::string& key,
               std::string* out) {
    const Entry* e = find_entry(section, key);
    if (!e) return kErrInvalid;
    Config& cfg = const_cast<Config&>(cfg_in);
    void* field = e->field(cfg);
    switch (e->kind) {
        case Kind::F: *out = fmt_float(*static_cast<float*>(field)); break;
        case Kind::I: *out = std::to_string(*static_cast<int*>(field)); break;
        case Kind::U: *out = std::to_string(*static_cast<unsigned*>(field)); break;
        case Kind::B: *out = *static_cast<bool*>(field) ? "true" : "false"; break;
        case Kind::S:
        case Kind::SQ: *out = *static_cast<std::string*>(field); break;
        case Kind::L: *out = fmt_list(*static_cast<std::vector<float>*>(field)); break;
    }
    return kOk;
}

int config_load_yaml(Config& cfg, const std::string& path, std::string* err) {
    std::ifstream in(path);
    if (!in) {
        std::fprintf(stderr, "load_config: could not open '%s'; using built-in defaults.\n",
                     path.c_str());
        return kWarnDefaults;
    }
    std::string section, line;
    int status = kOk;
    while (std::getline(in, line)) {
        const std::size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        line = trim(line);
        if (line.empty()) continue;
        const std::size_t colon = line.find(':');
        if (colon == std::string::npos) {
            std::fprintf(stderr, "load_config: skipping malformed line '%s'\n", line.c_str());
            continue;
        }
        const std::string key = trim(line.substr(0, colon));
        const std::string value = trim(line.substr(colon + 1));
        if (value.empty()) {
            section = key;
            continue;
        }
        const int rc = config_set(cfg, section, key, value, err);
        if (rc < 0) return rc;
        if (rc > status) status = rc;
    }
    return status == kWarnUnknownKey ? kWarnUnknownKey : kOk;
}

// reference src/particle_dynamics.cu:165-209
static void init_cube(const Config& cfg, Grains* g) {
    const float radius = cfg.particle_radius;
    const float origin[3] = {cfg.init_x0, cfg.init_y0, cfg.init_z0};
    int nps[3];
    for (int a = 0; a < 3; ++a) nps[a] = static_cast<int>(cfg.cube_length[a] / (2 * radius));
    const int n = nps[0] * nps[1] * nps[2];
    g->state.assign(static_cast<size_t>(n) * 6, 0.f);
    g->material.assign(static_cast<size_t>(n), cfg.particle_material);
    const float velocity[3] = {cfg.init_vx0, cfg.init_vy0, cfg.init_vz0};
    std::mt19937 rng(cfg.init_seed);
    std::uniform_real_distribution<float> jitter(-cfg.init_jitter * radius,
                                                 cfg.init_jitter * radius);
    std::mt19937 perturbation_rng(cfg.init_perturbation_seed);
    std::uniform_real_distribution<float> perturbation(-cfg.init_perturbation * radius,
                                                       cfg.init_perturbation * radius);
    for (int i = 0; i < nps[0]; ++i)
        for (int j = 0; j < nps[1]; ++j)
            for (int k = 0; k < nps[2]; ++k) {
                const int lattice[3] = {i, j, k};
                const int p = (i * nps[1] + j) * nps[2] + k;
                for (int a = 0; a < 3; ++a) {
                    const float base =
                        origin[a] + static_cast<float>(lattice[a]) * 2.f * 1.01f * radius;
                    const float jit = cfg.init_jitter > 0.f ? jitter(rng) : 0.f;
                    const float per =
                        cfg.init_perturbation > 0.f ? perturbation(perturbation_rng) : 0.f;
                    g->state[6 * static_cast<size_t>(p) + a] = base + jit + per;
                    g->state[6 * static_cast<size_t>(p) + 3 + a] = velocity[a];
                }
            }
}

int build_initial_grains(const Config& cfg, Grains* g, std::string* err) {
    g->state.clear();
    g->material.clear();
    if (cfg.init_type == "file") {
        // reference src/particle_dynamics.cu:212-235
        FILE* f = std::fopen(cfg.init_state_path.c_str(), "rb");
        if (!f) {
            if (err) *err = "initialize_from_file: could not open '" + cfg.init_state_path + "'";
            return kErrIo;
        }
        int32_t count = 0;
        if (std::fread(&count, sizeof(int32_t), 1, f) != 1 || count <= 0) {
            std::fclose(f);
            if (err) *err = "initialize_from_file: bad particle count in '" + cfg.init_state_path + "'";
            return kErrIo;
        }
        const size_t expected = static_cast<size_t>(count) * 6;
        g->state.resize(expected);
        const size_t got = std::fread(g->state.data(), sizeof(float), expected, f);
        std::fclose(f);
        if (got != expected) {
            if (err)
                *err = "initialize_from_file: '" + cfg.init_state_path + "' is short of " +
                       std::to_string(expected) + " floats";
            return kErrIo;
        }
        g->material.assign(static_cast<size_t>(count), cfg.particle_material);
    } else if (cfg.init_type == "two_particles") {
        // reference src/particle_dynamics.cu:128-145
        g->state = {cfg.init_x0, cfg.init_y0, cfg.init_z0, 0.f, 0.f, 0.f,
                    cfg.init_x0, cfg.init_y0, cfg.init_z0 + cfg.two_particle_separation,
                    0.f, 0.f, 0.f};
        g->material.assign(2, cfg.particle_material);
    } else if (cfg.init_type == "single_particle") {
        // reference src/particle_dynamics.cu:148-162
        g->state = {cfg.init_x0, cfg.init_y0, cfg.init_z0, cfg.init_vx0, cfg.init_vy0,
                    cfg.init_vz0};
        g->material.assign(1, cfg.particle_material);
    } else {
        init_cube(cfg, g);
    }
    return kOk;
}

}  // namespace wd
