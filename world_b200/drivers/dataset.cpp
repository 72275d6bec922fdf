// dataset -- training-set generator for the outcome surrogate, on batched scenes.
//
//   dataset [config.yaml] [design.csv] [output_dir] [--batch B]
//
// Same command line, inputs and outputs as the reference's build/bin/dataset
// (src/dataset.cpp:126-240): one rollout per row of the design CSV, the row's
// parameters applied on top of the base config, the density field recorded at K
// evenly spaced checkpoints (t_k = (k + 1) / K * dataset.sim_time), written to
// output_dir/grids.bin ("RTPGRD01" header, then grids[rollout][checkpoint][4][nx][ny][nz]
// float32) and output_dir/manifest.csv (rollout, the parameters, status, final_time,
// overflow_cells, deposited_mass). A rollout whose grid overflows or that leaves the
// domain is "diverged": it stops there, and its remaining checkpoints are zero-filled.
//
// The reference steps one ParticleDynamics per row. Here up to B rows (default 128)
// run as the scenes of one SceneBatch, all advanced by one step; a diverged row is
// frozen in place. Each row's trajectory is the one its own simulation would follow.
// Unknown design columns are rejected before anything is written (the reference
// stops at the first row that uses one, after writing the headers).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "world_b200/scene_batch.hpp"

namespace {

constexpr char kMagic[8] = {'R', 'T', 'P', 'G', 'R', 'D', '0', '1'};
constexpr int kChannels = 4;  // mass, then momentum per axis

struct Design {
    std::vector<std::string> names;
    std::vector<std::vector<float>> rows;
};

// Whitespace and a trailing carriage return (CRLF files from Python's csv module)
// are not part of a cell.
std::string trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

bool read_design(const std::string& path, Design* d) {
    std::ifstream in(path);
    if (!in) {
        std::fprintf(stderr,
                     "dataset: could not open design '%s'.\n"
                     "Generate one first:  surrogate/.venv/bin/python surrogate/make_design.py\n",
                     path.c_str());
        return false;
    }
    std::string line;
    bool header = true;
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        std::stringstream ss(line);
        std::string cell;
        if (header) {
            while (std::getline(ss, cell, ',')) d->names.push_back(trim(cell));
            header = false;
            continue;
        }
        std::vector<float> row;
        while (std::getline(ss, cell, ',')) row.push_back(std::stof(trim(cell)));
        if (row.size() != d->names.size()) {
            std::fprintf(stderr, "dataset: design row has %zu values, expected %zu\n", row.size(),
                         d->names.size());
            return false;
        }
        d->rows.push_back(row);
    }
    return true;
}

const char* const kColumns[] = {"throw_vx", "throw_vy", "throw_vz", "release_z",
                                "grain_mass", "restitution", "friction"};

bool known_column(const std::string& name) {
    for (const char* c : kColumns)
        if (name == c) return true;
    return false;
}

// One design row on top of the base config (src/dataset.cpp:96-124). grain_mass sets
// every non-void material's mass, so the grain count is the same for every row.
SimConfig config_for_row(const SimConfig& base, const Design& d, const std::vector<float>& row) {
    SimConfig c = base;
    for (size_t j = 0; j < d.names.size(); ++j) {
        const std::string& name = d.names[j];
        const float v = row[j];
        if (name == "throw_vx") c.init_vx0 = v;
        else if (name == "throw_vy") c.init_vy0 = v;
        else if (name == "throw_vz") c.init_vz0 = v;
        else if (name == "release_z") c.init_z0 = v;
        else if (name == "grain_mass") {
            for (size_t m = 1; m < c.masses.size(); ++m) c.masses[m] = v;
        } else if (name == "restitution") c.physics.restitution = v;
        else if (name == "friction") c.physics.friction = v;
    }
    return c;
}

}  // namespace

int main(int argc, char** argv) {
    std::vector<std::string> pos;
    int batch = 128;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--batch" && i + 1 < argc) {
            batch = std::max(1, std::atoi(argv[++i]));
        } else {
            pos.push_back(a);
        }
    }
    const std::string config_path = pos.size() > 0 ? pos[0] : "dataset/blob_throw.yaml";
    const std::string design_path = pos.size() > 1 ? pos[1] : "dataset/design.csv";
    const std::string out_dir = pos.size() > 2 ? pos[2] : "dataset";

    SimConfig base;
    Design design;
    try {
        base = load_config(config_path);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "dataset: %s\n", e.what());
        return 1;
    }
    if (!read_design(design_path, &design)) return 1;
    for (const std::string& name : design.names) {
        if (!known_column(name)) {
            std::fprintf(stderr, "dataset: design column '%s' is not a known parameter\n",
                         name.c_str());
            return 1;
        }
    }
    const int R = static_cast<int>(design.rows.size());
    const int K = base.dataset_checkpoints;
    if (R == 0 || K <= 0) {
        std::fprintf(stderr, "dataset: nothing to do (%d rollouts, %d checkpoints)\n", R, K);
        return 1;
    }
    std::vector<float> times(K);
    for (int k = 0; k < K; ++k)
        times[k] = base.dataset_sim_time * static_cast<float>(k + 1) / static_cast<float>(K);

    std::error_code ec;
    std::filesystem::create_directories(out_dir, ec);
    if (ec) {
        std::fprintf(stderr, "dataset: could not create '%s'\n", out_dir.c_str());
        return 1;
    }
    const int nx = base.density_grid_size_x, ny = base.density_grid_size_y,
              nz = base.density_grid_size_z;
    const size_t snapshot = static_cast<size_t>(kChannels) * nx * ny * nz;
    const std::string grid_path = out_dir + "/grids.bin";
    std::FILE* grids = std::fopen(grid_path.c_str(), "wb");
    if (!grids) {
        std::fprintf(stderr, "dataset: could not open '%s' for writing\n", grid_path.c_str());
        return 1;
    }
    std::fwrite(kMagic, 1, 8, grids);
    const int32_t header[7] = {R, K, kChannels, nx, ny, nz,
                               static_cast<int32_t>(design.names.size())};
    std::fwrite(header, sizeof(int32_t), 7, grids);
    std::fwrite(times.data(), sizeof(float), times.size(), grids);
    const long long data_start = 8 + 7 * 4 + 4LL * K;

    const std::string manifest_path = out_dir + "/manifest.csv";
    std::FILE* manifest = std::fopen(manifest_path.c_str(), "w");
    if (!manifest) {
        std::fprintf(stderr, "dataset: could not open '%s' for writing\n", manifest_path.c_str());
        return 1;
    }
    std::fprintf(manifest, "rollout");
    for (const std::string& name : design.names) std::fprintf(manifest, ",%s", name.c_str());
    std::fprintf(manifest, ",status,final_time,overflow_cells,deposited_mass\n");

    // rows per batch: also bounded so the batch's collision cells stay below 2^31
    const double cells = static_cast<double>(base.collision_grid_size_x) *
                         base.collision_grid_size_y * base.collision_grid_size_z;
    const int by_cells = static_cast<int>(std::max(1.0, 2147483647.0 / std::max(cells, 1.0)));
    const int B = std::max(1, std::min({batch, by_cells, R}));
    const std::vector<float> zeros(snapshot, 0.f);
    int num_ok = 0, num_diverged = 0;

    try {
        for (int r0 = 0; r0 < R; r0 += B) {
            const int S = std::min(B, R - r0);
            std::vector<SimConfig> cfgs;
            for (int k = 0; k < S; ++k) cfgs.push_back(config_for_row(base, design, design.rows[r0 + k]));
            SceneBatch sim(cfgs);
            const int steps = std::max(1, static_cast<int>(
                base.dataset_sim_time / (static_cast<float>(K) * cfgs[0].dt) + 0.5f));
            std::vector<char> diverged(S, 0);
            std::vector<int> overflow(S, 0);
            std::vector<float> final_time(S, 0.f);
            std::vector<double> deposited(S, 0.0);
            for (int k = 0; k < K; ++k) {
                sim.take_steps(steps);
                // polled once per checkpoint, as the reference does
                const std::vector<int64_t> ov = sim.overflow_counts();
                const std::vector<int32_t> ok = sim.stability();
                for (int q = 0; q < S; ++q) {
                    if (diverged[q]) continue;
                    overflow[q] = static_cast<int>(ov[q]);
                    final_time[q] = sim.time;
                    if (ov[q] > 0 || !ok[q]) {
                        diverged[q] = 1;
                        sim.freeze(q);
                    }
                }
                sim.compute_density_grid();
                for (int q = 0; q < S; ++q) {
                    const long long at =
                        data_start + 4LL * static_cast<long long>(snapshot) *
                                         (static_cast<long long>(r0 + q) * K + k);
                    std::fseek(grids, at, SEEK_SET);
                    const float* src = diverged[q] ? zeros.data() : sim.scene_grid(q);
                    std::fwrite(src, sizeof(float), snapshot, grids);
                    if (!diverged[q] && k == K - 1) {
                        double m = 0.0;
                        const size_t nodes = snapshot / kChannels;
                        for (size_t i = 0; i < nodes; ++i) m += src[i];
                        deposited[q] = m;
                    }
                }
            }
            for (int q = 0; q < S; ++q) {
                std::fprintf(manifest, "%d", r0 + q);
                for (float v : design.rows[r0 + q]) std::fprintf(manifest, ",%.9g", static_cast<double>(v));
                std::fprintf(manifest, ",%s,%.9g,%d,%.9g\n", diverged[q] ? "diverged" : "ok",
                             static_cast<double>(final_time[q]), overflow[q], deposited[q]);
                if (diverged[q]) ++num_diverged; else ++num_ok;
            }
            std::fflush(manifest);
            std::printf("\rrollout %d/%d  ok=%d diverged=%d", r0 + S, R, num_ok, num_diverged);
            std::fflush(stdout);
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "\ndataset: %s\n", e.what());
        std::fclose(grids);
        std::fclose(manifest);
        return 1;
    }
    std::printf("\n");
    std::fclose(grids);
    std::fclose(manifest);
    std::printf("Wrote %s (%d rollouts x %d checkpoints x %d channels x %dx%dx%d)\n",
                grid_path.c_str(), R, K, kChannels, nx, ny, nz);
    std::printf("Wrote %s (%d ok, %d diverged)\n", manifest_path.c_str(), num_ok, num_diverged);
    return 0;
}
