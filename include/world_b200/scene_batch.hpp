// scene_batch.hpp -- C++ face of the batched-scene calls of libworld_b200.so
// (wd_create_batch and the per-scene calls in include/world_b200.h).
//
// The reference runs its dataset rows and ensemble members one ParticleDynamics at a
// time (src/dataset.cpp:186-224, src/chaos.cpp:176-224). SceneBatch holds many such
// simulations in one handle and one step; scene k keeps the grain ids
// [range(k).first, range(k).first + range(k).count) of the batch-wide arrays and the
// density-field floats [4 * range(k).node_first, 4 * (range(k).node_first +
// range(k).nodes)), laid out like a single simulation's host_density_grid.
#pragma once

#include <cstdint>
#include <vector>

#include "particle_dynamics.hpp"

namespace world_b200 {

struct SceneRange {
    int64_t first = 0, count = 0, node_first = 0, nodes = 0;
};

class SceneBatch {
public:
    std::vector<SimConfig> configs;
    int n = 0;             // grains over all scenes
    float time = 0.f;      // simulated time, advanced by dt per step for every scene
    float dt = 0.f;
    std::vector<float> positions;          // 3n, by batch grain id
    std::vector<float> host_density_grid;  // 4 * nodes over all scenes

    // Every scene built from its config's initialization section, as
    // ParticleDynamics(config) builds one.
    explicit SceneBatch(const std::vector<SimConfig>& cfgs) : configs(cfgs) {
        if (cfgs.empty()) throw std::runtime_error("SceneBatch: no scenes");
        std::vector<detail::ConfigHandle> handles(cfgs.size());
        std::vector<const wd_config*> ptrs(cfgs.size());
        for (size_t k = 0; k < cfgs.size(); ++k) {
            SimConfig c = cfgs[k];
            detail::visit(c, detail::Writer{handles[k].p});
            ptrs[k] = handles[k].p;
        }
        detail::check(wd_create_batch(ptrs.data(), static_cast<int32_t>(cfgs.size()), nullptr,
                                      nullptr, nullptr, nullptr, nullptr, &sim_),
                      "SceneBatch");
        int64_t count = 0;
        wd_get_n(sim_, &count);
        n = static_cast<int>(count);
        dt = cfgs[0].dt;
        ranges_.resize(cfgs.size());
        for (size_t k = 0; k < cfgs.size(); ++k) {
            SceneRange& r = ranges_[k];
            detail::check(wd_scene_range(sim_, static_cast<int32_t>(k), &r.first, &r.count,
                                         &r.node_first, &r.nodes),
                          "wd_scene_range");
        }
        int64_t nodes = 0;
        wd_density_grid_nodes(sim_, &nodes);
        positions.resize(static_cast<size_t>(kDim) * n);
        host_density_grid.resize(4 * static_cast<size_t>(nodes));
    }

    ~SceneBatch() { wd_destroy(sim_); }
    SceneBatch(const SceneBatch&) = delete;
    SceneBatch& operator=(const SceneBatch&) = delete;

    int scenes() const { return static_cast<int>(ranges_.size()); }
    const SceneRange& range(int k) const { return ranges_.at(k); }

    // steps x take_step() for every scene that is not frozen
    void take_steps(int steps) {
        detail::check(wd_step(sim_, steps), "take_steps");
        detail::check(wd_get_time(sim_, &time), "wd_get_time");
    }

    void unpack_positions() {
        detail::check(wd_get_positions(sim_, positions.data()), "unpack_positions");
    }

    void compute_density_grid() {
        detail::check(wd_compute_density_grid(sim_, host_density_grid.data()),
                      "compute_density_grid");
    }

    // Scene k's 4 * nodes floats of host_density_grid (after compute_density_grid),
    // channel-major with the mass channel first.
    const float* scene_grid(int k) const {
        return host_density_grid.data() + 4 * static_cast<size_t>(ranges_.at(k).node_first);
    }

    std::vector<int64_t> overflow_counts() {
        std::vector<int64_t> v(ranges_.size());
        detail::check(wd_scene_overflow_counts(sim_, v.data()), "wd_scene_overflow_counts");
        return v;
    }

    std::vector<int32_t> stability() {
        std::vector<int32_t> v(ranges_.size());
        detail::check(wd_scene_stability(sim_, v.data()), "wd_scene_stability");
        return v;
    }

    void freeze(int k) { detail::check(wd_freeze_scene(sim_, k, 1), "wd_freeze_scene"); }

    // Per scene: {grain RMS separation, field relative difference, COM displacement}
    // from reference_scene.
    std::vector<double> chaos_metrics(int reference_scene) {
        std::vector<double> v(3 * ranges_.size());
        detail::check(wd_chaos_metrics(sim_, reference_scene, v.data()), "wd_chaos_metrics");
        return v;
    }

    wd_sim* handle() const { return sim_; }

private:
    wd_sim* sim_ = nullptr;
    std::vector<SceneRange> ranges_;
};

}  // namespace world_b200

#ifndef WORLD_B200_NO_GLOBAL_NAMES
using world_b200::SceneBatch;
using world_b200::SceneRange;
#endif
