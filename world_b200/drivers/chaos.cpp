// chaos -- what is predictable about a granular interaction, on batched scenes.
//
//   chaos [config.yaml] [members]
//
// Same command line and outputs as the reference's build/bin/chaos
// (src/chaos.cpp:80-240): E members share the config and differ only by a uniform
// random displacement of initialization.perturbation x radius per grain and axis
// (member 0 unperturbed, member m seeded 1000 + m). At each of dataset.checkpoints
// checkpoints every member m >= 1 is compared with member 0: per-grain RMS
// separation, relative l2 difference of the mass field, and centre-of-mass
// displacement (node units). Written to chaos/divergence.csv (member, checkpoint,
// time, grain_rms_displacement, field_relative_difference, com_displacement) and
// chaos/final_fields.bin (int32 members, int32 nodes, then the terminal mass field
// of member 0, 1, ..., float32 each).
//
// The reference runs the members one after another against stored checkpoints of
// member 0. Here the members are the scenes of one SceneBatch (member 0 included in
// every batch of at most B members, default 64) and the three measures are reduced
// on the device (wd_chaos_metrics).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <string>
#include <vector>

#include "world_b200/scene_batch.hpp"

namespace {
constexpr const char* kOutputDir = "chaos";
}

int main(int argc, char** argv) {
    std::vector<std::string> pos;
    int batch = 64;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--batch" && i + 1 < argc) {
            batch = std::max(2, std::atoi(argv[++i]));
        } else {
            pos.push_back(a);
        }
    }
    const std::string config_path = pos.size() > 0 ? pos[0] : "chaos/ensemble.yaml";
    const int members = pos.size() > 1 ? std::atoi(pos[1].c_str()) : 16;
    SimConfig base;
    try {
        base = load_config(config_path);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "chaos: %s\n", e.what());
        return 1;
    }
    if (base.init_perturbation <= 0.0f) {
        std::fprintf(stderr,
                     "chaos: initialization.perturbation is 0, so every member would be "
                     "identical.\nSet it to the perturbation magnitude you want to study.\n");
        return 1;
    }
    if (members < 2) {
        std::fprintf(stderr, "chaos: need at least 2 members, got %d\n", members);
        return 1;
    }
    const int K = base.dataset_checkpoints;
    const float total_time = base.dataset_sim_time;
    if (K <= 0) {
        std::fprintf(stderr, "chaos: dataset.checkpoints must be > 0\n");
        return 1;
    }
    std::vector<float> times(K);
    for (int k = 0; k < K; ++k)
        times[k] = total_time * static_cast<float>(k + 1) / static_cast<float>(K);
    std::error_code ec;
    std::filesystem::create_directories(kOutputDir, ec);
    if (ec) {
        std::fprintf(stderr, "chaos: could not create '%s'\n", kOutputDir);
        return 1;
    }
    const std::string path = std::string(kOutputDir) + "/divergence.csv";
    std::FILE* out = std::fopen(path.c_str(), "w");
    if (!out) {
        std::fprintf(stderr, "chaos: could not open '%s'\n", path.c_str());
        return 1;
    }
    std::fprintf(out, "member,checkpoint,time,grain_rms_displacement,"
                      "field_relative_difference,com_displacement\n");
    const std::string fields_path = std::string(kOutputDir) + "/final_fields.bin";
    std::FILE* fields = std::fopen(fields_path.c_str(), "wb");
    if (!fields) {
        std::fprintf(stderr, "chaos: could not open '%s'\n", fields_path.c_str());
        return 1;
    }
    const int steps = std::max(1, static_cast<int>(
        total_time / (static_cast<float>(K) * base.dt) + 0.5f));
    const size_t nodes = static_cast<size_t>(base.density_grid_size_x) *
                         base.density_grid_size_y * base.density_grid_size_z;
    {
        const int32_t header[2] = {members, static_cast<int32_t>(nodes)};
        std::fwrite(header, sizeof(int32_t), 2, fields);
    }
    const int per_batch = std::max(1, std::min(batch, members) - 1);  // besides member 0
    bool reference_written = false;
    try {
        for (int m0 = 1; m0 < members; m0 += per_batch) {
            const int count = std::min(per_batch, members - m0);
            std::vector<SimConfig> cfgs;
            SimConfig ref = base;
            ref.init_perturbation = 0.0f;  // member 0 is unperturbed
            cfgs.push_back(ref);
            for (int m = m0; m < m0 + count; ++m) {
                SimConfig c = base;
                c.init_perturbation_seed = static_cast<unsigned int>(1000 + m);
                cfgs.push_back(c);
            }
            SceneBatch sim(cfgs);
            const int n0 = static_cast<int>(sim.range(0).count);
            for (int q = 1; q < sim.scenes(); ++q) {
                if (sim.range(q).count != n0) {
                    std::fprintf(stderr, "chaos: member %d has %lld grains, reference had %d\n",
                                 m0 + q - 1, static_cast<long long>(sim.range(q).count), n0);
                    return 1;
                }
            }
            if (!reference_written) {
                std::printf("reference: %d grains, %d checkpoints, %d steps each, grid %dx%dx%d\n",
                            n0, K, steps, base.density_grid_size_x, base.density_grid_size_y,
                            base.density_grid_size_z);
            }
            // rows[(member - m0) * K + k]
            std::vector<double> rows(static_cast<size_t>(3) * count * K);
            for (int k = 0; k < K; ++k) {
                sim.take_steps(steps);
                const std::vector<double> m = sim.chaos_metrics(0);
                for (int q = 1; q <= count; ++q)
                    for (int c = 0; c < 3; ++c)
                        rows[3 * (static_cast<size_t>(q - 1) * K + k) + c] = m[3 * q + c];
            }
            // terminal mass fields
            sim.compute_density_grid();
            if (!reference_written) {
                std::fwrite(sim.scene_grid(0), sizeof(float), nodes, fields);
                reference_written = true;
            }
            for (int q = 1; q <= count; ++q) {
                for (int k = 0; k < K; ++k) {
                    const double* r = &rows[3 * (static_cast<size_t>(q - 1) * K + k)];
                    std::fprintf(out, "%d,%d,%.9g,%.9g,%.9g,%.9g\n", m0 + q - 1, k,
                                 static_cast<double>(times[k]), r[0], r[1], r[2]);
                }
                std::fwrite(sim.scene_grid(q), sizeof(float), nodes, fields);
            }
            std::fflush(out);
            std::printf("\rmember %d/%d", m0 + count - 1, members - 1);
            std::fflush(stdout);
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "\nchaos: %s\n", e.what());
        std::fclose(out);
        std::fclose(fields);
        return 1;
    }
    std::printf("\n");
    std::fclose(out);
    std::fclose(fields);
    std::printf("Wrote %s (%d perturbed members, perturbation = %.3g x radius)\n", path.c_str(),
                members - 1, static_cast<double>(base.init_perturbation));
    return 0;
}
