// The reference's ParticleDynamics tests (test/particle_dynamics_test.cpp:16-285) written
// against the C++ drop-in include/world_b200/particle_dynamics.hpp, with the same
// statements the reference's GoogleTest cases make. A minimal runner replaces
// GoogleTest (not available offline). `reference_cases config` runs the host-only
// cases; `reference_cases all` needs a GPU.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "world_b200/particle_dynamics.hpp"

static int g_failures = 0;
#define EXPECT(cond)                                                                 \
    do {                                                                             \
        if (!(cond)) {                                                               \
            std::fprintf(stderr, "%s:%d: expectation failed: %s\n", __FILE__, __LINE__, #cond); \
            ++g_failures;                                                            \
        }                                                                            \
    } while (0)
#define EXPECT_NEAR(a, b, tol) EXPECT(std::fabs(static_cast<double>(a) - static_cast<double>(b)) <= (tol))

static void ConfigDefaultsAndYaml() {
    SimConfig defaults;
    EXPECT(defaults.collision_grid_size_x == 32 && defaults.particles_per_cell == 64);
    const char* path = "reference_cases_config.yaml";
    FILE* f = std::fopen(path, "w");
    std::fprintf(f, "simulation:\n  dt: 0.001\n  collision_grid_size_x: 100\nphysics:\n"
                    "  friction: 0.25\nmaterials:\n  masses: [0.0, 0.8]\n"
                    "initialization:\n  type: \"single_particle\"\n");
    std::fclose(f);
    const SimConfig c = load_config(path);
    std::remove(path);
    EXPECT_NEAR(c.dt, 0.001f, 0.0);
    EXPECT(c.collision_grid_size_x == 100 && c.collision_grid_size_y == 32);
    EXPECT_NEAR(c.physics.friction, 0.25f, 0.0);
    EXPECT(c.masses.size() == 2 && c.masses[1] == 0.8f);
    EXPECT(c.init_type == "single_particle");
    const SimConfig missing = load_config("no_such_reference_cases.yaml");
    EXPECT(missing.collision_grid_size_x == 32);
}

static void RunsStablyForFixedIterations() {
    ParticleDynamics sim;
    for (int i = 0; i < 100; ++i) sim.take_step();
    EXPECT(sim.is_stable());
}

static void FreeFallMatchesKinematics() {
    ParticleDynamics sim;
    for (int i = 0; i < sim.n; ++i)
        for (int a = 0; a < kDim; ++a) sim.host_state[kStateStride * i + kDim + a] = 0.0f;
    sim.device_state.copy_from_host(sim.host_state);
    const float z0 = sim.host_state[2];
    const int steps = 100;
    for (int i = 0; i < steps; ++i) sim.take_step();
    sim.unpack_state();
    const float expected = -9.81f * sim.dt * sim.dt * static_cast<float>(steps) *
                           static_cast<float>(steps + 1) / 2.0f;
    EXPECT_NEAR(sim.positions[2] - z0, expected, 1e-6);
}

static void ParticleDoesNotPenetrateFloor() {
    ParticleDynamics sim;
    const float start[kStateStride] = {0.5f, 0.5f, -0.5f, 0.0f, 0.0f, 0.0f};
    for (int a = 0; a < kStateStride; ++a) sim.host_state[a] = start[a];
    sim.device_state.copy_from_host(sim.host_state);
    for (int i = 0; i < 20000; ++i) sim.take_step();
    sim.unpack_state();
    EXPECT(sim.positions[2] >= -1.0f + 0.01f - 1e-3f);
    EXPECT(sim.is_stable());
}

static void RepeatedRunsAreDeterministic() {
    auto run = [](std::vector<float>& out) {
        ParticleDynamics sim;
        for (int i = 0; i < 50; ++i) sim.take_step();
        sim.unpack_state();
        out = sim.positions;
    };
    std::vector<float> a, b;
    run(a);
    run(b);
    EXPECT(a.size() == b.size());
    for (size_t i = 0; i < a.size(); ++i) EXPECT(a[i] == b[i]);
}

static void GridOverflowIsCountedAndStaysInBounds() {
    SimConfig config;
    config.collision_grid_size_x = config.collision_grid_size_y = config.collision_grid_size_z = 1;
    config.particles_per_cell = 2;
    ParticleDynamics sim(config);
    EXPECT(sim.n > config.particles_per_cell);
    EXPECT(sim.grid_overflow_count() == 0);
    sim.take_step();
    EXPECT(sim.grid_overflow_count() > 0);
    sim.unpack_state();
    for (float c : sim.positions) EXPECT(std::isfinite(c));
}

static void TotalEnergyNeverIncreases() {
    ParticleDynamics sim;
    float previous = sim.compute_total_energy();
    const float initial = previous;
    EXPECT(initial > 0.0f);
    const float tolerance = 1e-3f * initial;
    for (int interval = 0; interval < 12; ++interval) {
        for (int step = 0; step < 100; ++step) sim.take_step();
        const float current = sim.compute_total_energy();
        EXPECT(current <= previous + tolerance);
        previous = current;
    }
    EXPECT(previous < initial);
}

static void DensityGridConservesTotalMass() {
    SimConfig config;
    config.init_jitter = 0.3f;
    ParticleDynamics sim(config);
    for (int step = 0; step < 250; ++step) sim.take_step();
    sim.compute_density_grid();
    double deposited = 0.0;
    for (size_t node = 0; node < sim.density_grid_nodes(); ++node) deposited += sim.host_density_grid[node];
    sim.unpack_state();
    double expected = 0.0;
    for (int i = 0; i < sim.n; ++i) expected += sim.host_mass[sim.host_material[i]];
    EXPECT(expected > 0.0);
    EXPECT_NEAR(deposited, expected, 1e-4 * expected);
}

static void DensityGridPutsGrainOnNodeAtSingleNode() {
    SimConfig config;
    config.init_type = "single_particle";
    config.density_grid_size_x = config.density_grid_size_y = config.density_grid_size_z = 5;
    config.init_x0 = -0.5f;
    config.init_y0 = 0.0f;
    config.init_z0 = 0.5f;
    ParticleDynamics sim(config);
    sim.compute_density_grid();
    const int expected_node = (1 * 5 + 2) * 5 + 3;
    const float m = sim.host_mass[config.particle_material];
    for (size_t node = 0; node < sim.density_grid_nodes(); ++node) {
        if (static_cast<int>(node) == expected_node) EXPECT_NEAR(sim.host_density_grid[node], m, 1e-6 * m);
        else EXPECT_NEAR(sim.host_density_grid[node], 0.0, 1e-6 * m);
    }
}

static void DensityGridSplitsCellCenterEightWays() {
    SimConfig config;
    config.init_type = "single_particle";
    config.density_grid_size_x = config.density_grid_size_y = config.density_grid_size_z = 5;
    config.init_x0 = -0.75f;
    config.init_y0 = -0.25f;
    config.init_z0 = 0.25f;
    ParticleDynamics sim(config);
    sim.compute_density_grid();
    const float m = sim.host_mass[config.particle_material];
    int nonzero = 0;
    float total = 0.0f;
    for (size_t node = 0; node < sim.density_grid_nodes(); ++node) {
        const float value = sim.host_density_grid[node];
        total += value;
        if (value > 1e-9f) {
            ++nonzero;
            EXPECT_NEAR(value, m / 8.0f, 1e-5 * m);
        }
    }
    EXPECT(nonzero == 8);
    EXPECT_NEAR(total, m, 1e-5 * m);
}

static void DensityGridMomentumMatchesMassTimesVelocity() {
    SimConfig config;
    config.init_type = "single_particle";
    config.init_vx0 = 2.0f;
    config.init_vy0 = -3.0f;
    config.init_vz0 = 0.5f;
    ParticleDynamics sim(config);
    sim.compute_density_grid();
    const size_t nodes = sim.density_grid_nodes();
    const float m = sim.host_mass[config.particle_material];
    const float expected_velocity[kDim] = {2.0f, -3.0f, 0.5f};
    for (int a = 0; a < kDim; ++a) {
        double momentum = 0.0;
        for (size_t node = 0; node < nodes; ++node) momentum += sim.host_density_grid[(a + 1) * nodes + node];
        const double want = static_cast<double>(m) * expected_velocity[a];
        EXPECT_NEAR(momentum, want, 1e-4 * std::fabs(want) + 1e-9);
    }
}

static void CubeGrainsReceiveInitialVelocity() {
    SimConfig config;
    config.init_vx0 = 1.5f;
    config.init_vy0 = -0.5f;
    config.init_vz0 = 0.25f;
    config.physics.gravity = 0.0f;
    ParticleDynamics sim(config);
    EXPECT(sim.n > 1);
    const float expected[kDim] = {1.5f, -0.5f, 0.25f};
    for (int i = 0; i < sim.n; ++i)
        for (int a = 0; a < kDim; ++a) EXPECT(sim.host_state[kStateStride * i + kDim + a] == expected[a]);
    std::vector<float> before(sim.positions.begin(), sim.positions.end());
    const int steps = 50;
    for (int step = 0; step < steps; ++step) sim.take_step();
    sim.unpack_state();
    const float elapsed = sim.dt * static_cast<float>(steps);
    for (int a = 0; a < kDim; ++a) {
        const float moved = sim.positions[a] - before[a];
        EXPECT_NEAR(moved, expected[a] * elapsed, 1e-4 * std::fabs(expected[a] * elapsed) + 1e-6);
    }
}

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "all";
    struct Case { const char* name; std::function<void()> fn; bool gpu; };
    const Case cases[] = {
        {"ConfigDefaultsAndYaml", ConfigDefaultsAndYaml, false},
        {"RunsStablyForFixedIterations", RunsStablyForFixedIterations, true},
        {"FreeFallMatchesKinematics", FreeFallMatchesKinematics, true},
        {"ParticleDoesNotPenetrateFloor", ParticleDoesNotPenetrateFloor, true},
        {"RepeatedRunsAreDeterministic", RepeatedRunsAreDeterministic, true},
        {"GridOverflowIsCountedAndStaysInBounds", GridOverflowIsCountedAndStaysInBounds, true},
        {"TotalEnergyNeverIncreases", TotalEnergyNeverIncreases, true},
        {"DensityGridConservesTotalMass", DensityGridConservesTotalMass, true},
        {"DensityGridPutsGrainOnNodeAtSingleNode", DensityGridPutsGrainOnNodeAtSingleNode, true},
        {"DensityGridSplitsCellCenterEightWays", DensityGridSplitsCellCenterEightWays, true},
        {"DensityGridMomentumMatchesMassTimesVelocity", DensityGridMomentumMatchesMassTimesVelocity, true},
        {"CubeGrainsReceiveInitialVelocity", CubeGrainsReceiveInitialVelocity, true},
    };
    int ran = 0;
    for (const Case& c : cases) {
        if (mode == "config" && c.gpu) continue;
        const int before = g_failures;
        try {
            c.fn();
        } catch (const std::exception& e) {
            std::fprintf(stderr, "%s: exception: %s\n", c.name, e.what());
            ++g_failures;
        }
        std::printf("[%s] %s\n", g_failures == before ? "  OK  " : " FAIL ", c.name);
        ++ran;
    }
    std::printf("%d cases, %d failed expectations\n", ran, g_failures);
    return g_failures == 0 ? 0 : 1;
}
