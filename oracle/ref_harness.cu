// ref_harness.cu -- C entry points over the reference's own ParticleDynamics.
//
// Test infrastructure. Built by oracle/build.py together with the reference's
// unmodified sources (src/*.cu, src/sim_config.cpp) into oracle/_ref/libref_world.so.
// It only constructs the reference's class and reads its public members
// (src/particle_dynamics.h:17-141); nothing of the reference is re-implemented here.
// Used by the GPU parity tests and by tests/golden/make_golden.py to record the
// reference's outputs on seeded inputs.
#include <cstring>
#include <string>

#include "particle_dynamics.h"
#include "sim_config.h"

extern "C" {

void* ref_create(const char* yaml_path) {
    const SimConfig cfg = load_config(yaml_path);
    return new ParticleDynamics(cfg);
}

void ref_destroy(void* h) { delete static_cast<ParticleDynamics*>(h); }

int ref_n(void* h) { return static_cast<ParticleDynamics*>(h)->n; }

void ref_step(void* h, int steps) {
    auto* sim = static_cast<ParticleDynamics*>(h);
    for (int k = 0; k < steps; ++k) sim->take_step();
}

void ref_set_dt(void* h, float dt) { static_cast<ParticleDynamics*>(h)->dt = dt; }

float ref_time(void* h) { return static_cast<ParticleDynamics*>(h)->time; }

void ref_get_state(void* h, float* out) {
    auto* sim = static_cast<ParticleDynamics*>(h);
    sim->host_state.copy_from_device(sim->device_state);
    std::memcpy(out, sim->host_state.data(), sizeof(float) * sim->host_state.size());
}

void ref_set_state(void* h, const float* in) {
    auto* sim = static_cast<ParticleDynamics*>(h);
    std::memcpy(sim->host_state.data(), in, sizeof(float) * sim->host_state.size());
    sim->device_state.copy_from_host(sim->host_state);
}

void ref_get_rhs(void* h, float* out) {
    auto* sim = static_cast<ParticleDynamics*>(h);
    HostVector<float> tmp(sim->device_rhs.size());
    tmp.copy_from_device(sim->device_rhs);
    std::memcpy(out, tmp.data(), sizeof(float) * tmp.size());
}

int ref_neighbor_stride(void* h) {
    auto* sim = static_cast<ParticleDynamics*>(h);
    return kStencilCells * sim->particles_per_cell;
}

void ref_get_neighbors(void* h, int* out) {
    auto* sim = static_cast<ParticleDynamics*>(h);
    HostVector<int> tmp(sim->device_neighbors.size());
    tmp.copy_from_device(sim->device_neighbors);
    std::memcpy(out, tmp.data(), sizeof(int) * tmp.size());
}

long long ref_density_nodes(void* h) {
    return static_cast<long long>(static_cast<ParticleDynamics*>(h)->density_grid_nodes());
}

void ref_density(void* h, float* out) {
    auto* sim = static_cast<ParticleDynamics*>(h);
    const size_t count = sim->compute_density_grid();
    std::memcpy(out, sim->host_density_grid.data(), sizeof(float) * count);
}

float ref_energy(void* h) { return static_cast<ParticleDynamics*>(h)->compute_total_energy(); }

int ref_overflow(void* h) { return static_cast<ParticleDynamics*>(h)->grid_overflow_count(); }

int ref_is_stable(void* h) { return static_cast<ParticleDynamics*>(h)->is_stable() ? 1 : 0; }

float ref_max_accel(void* h) {
    return static_cast<ParticleDynamics*>(h)->compute_max_acceleration();
}

}  // extern "C"
