// State files, checkpoints and the broadcast frame, over the library's own C ABI.
//
// State file (the reference's format; reader src/particle_dynamics.cu:212-235, writer
// surrogate/decode_particles.py:355-361): int32 n, then 6n float32 [x y z vx vy vz].
//
// A checkpoint is that file plus a sidecar "<path>.sidecar" holding what the state file
// lacks for a bit-identical resume (the reference saves none of it):
//   char magic[8] = "WDCKPT01"; uint32 version = 2; uint32 flags (bit 0: history)
//   int64 n; float32 time; float32 dt; uint64 state_hash (version 2 only: 64-bit
//   FNV-1a of the state file's bytes, so a sidecar never pairs with another state)
//   float32 radius[n]; float32 mass[n]; int32 material[n]
//   history only: int32 count[n]; int32 partner[n * 24]; float32 xi[n * 24 * 3]
// all little-endian, arrays by grain id. The neighbor order is canonical (cell key,
// then grain id), so it needs no saving: the first search of the resumed handle
// rebuilds it. Both files are written under temporary names and renamed into place,
// the state file first; a crash between the two renames leaves a new state file with
// the old sidecar, which the hash rejects. Version-1 sidecars (no hash) still load.
//
// Broadcast frame (src/broadcast.cpp:95-108): 3n position floats by grain id, then
// sim time, real-time ratio, find-neighbors / compute-rhs / take-step / unpack times.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/world_b200.h"
#include "wd_config.h"

namespace {

constexpr char kMagic[8] = {'W', 'D', 'C', 'K', 'P', 'T', '0', '1'};
constexpr uint32_t kVersion = 2;
constexpr int kCap = WD_HIST_CAP;

int fail(int code, const std::string& msg) {
    wd::set_last_error(msg);
    return code;
}

struct File {
    std::FILE* f = nullptr;
    File(const std::string& path, const char* mode) : f(std::fopen(path.c_str(), mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
    template <typename T>
    bool put(const T* p, size_t count) { return std::fwrite(p, sizeof(T), count, f) == count; }
    template <typename T>
    bool get(T* p, size_t count) { return std::fread(p, sizeof(T), count, f) == count; }
};

uint64_t fnv1a(uint64_t h, const void* data, size_t bytes) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (size_t k = 0; k < bytes; ++k) {
        h ^= p[k];
        h *= 0x100000001b3ull;
    }
    return h;
}
constexpr uint64_t kFnvBasis = 0xcbf29ce484222325ull;

uint64_t state_hash(int32_t count, const std::vector<float>& state) {
    return fnv1a(fnv1a(kFnvBasis, &count, sizeof(count)), state.data(),
                 state.size() * sizeof(float));
}

bool is_batch(const wd_sim* sim) {
    int32_t scenes = 1;
    wd_scene_count(sim, &scenes);
    return scenes != 1;
}

}  // namespace

extern "C" {

namespace {

// The state file's bytes for `sim`: its grain count and 6n floats.
int read_state(wd_sim* sim, const char* who, int32_t* count, std::vector<float>* state) {
    int64_t n = 0;
    int rc = wd_get_n(sim, &n);
    if (rc) return rc;
    if (n > INT32_MAX) return fail(WD_ERR_INVALID, std::string(who) + ": n does not fit int32");
    state->resize(static_cast<size_t>(6) * n);
    rc = wd_get_state(sim, state->data());
    if (rc) return rc;
    *count = static_cast<int32_t>(n);
    return WD_OK;
}

bool write_state_bytes(const std::string& path, int32_t count, const std::vector<float>& state) {
    File out(path, "wb");
    const bool ok = out.f && out.put(&count, 1) && out.put(state.data(), state.size());
    if (!out.f) return false;
    const bool closed = std::fclose(out.f) == 0;
    out.f = nullptr;
    return ok && closed;
}

}  // namespace

int wd_write_state_file(wd_sim* sim, const char* path) {
    if (!sim || !path) return fail(WD_ERR_INVALID, "wd_write_state_file: NULL argument");
    int32_t count = 0;
    std::vector<float> state;
    const int rc = read_state(sim, "wd_write_state_file", &count, &state);
    if (rc) return rc;
    if (!write_state_bytes(path, count, state))
        return fail(WD_ERR_IO, std::string("wd_write_state_file: cannot write ") + path);
    return WD_OK;
}

int wd_write_checkpoint(wd_sim* sim, const char* path) {
    if (!sim || !path) return fail(WD_ERR_INVALID, "wd_write_checkpoint: NULL argument");
    if (is_batch(sim)) return fail(WD_ERR_INVALID, "wd_write_checkpoint: not for a batch of scenes");
    int32_t count32 = 0;
    std::vector<float> state;
    int rc = read_state(sim, "wd_write_checkpoint", &count32, &state);
    if (rc) return rc;
    const int64_t n = count32;
    float time = 0.f, dt = 0.f;
    wd_get_time(sim, &time);
    wd_get_dt(sim, &dt);
    std::vector<float> radius(n), mass(n);
    std::vector<int32_t> material(n);
    rc = wd_get_grain_props(sim, radius.data(), mass.data(), material.data());
    if (rc) return rc;
    std::vector<int32_t> count(n), partner(static_cast<size_t>(n) * kCap);
    std::vector<float> xi(static_cast<size_t>(n) * kCap * 3);
    rc = wd_get_history(sim, count.data(), partner.data(), xi.data());
    if (rc) return rc;
    // springs are saved when any is stored (a handle without history reports none;
    // an empty history resumes the same as a fresh one)
    bool history = false;
    for (int32_t c : count) history |= c > 0;
    const uint32_t flags = history ? 1u : 0u;
    const uint64_t hash = state_hash(count32, state);
    const std::string state_tmp = std::string(path) + ".tmp";
    const std::string side = std::string(path) + ".sidecar";
    const std::string side_tmp = side + ".tmp";
    if (!write_state_bytes(state_tmp, count32, state))
        return fail(WD_ERR_IO, "wd_write_checkpoint: cannot write " + state_tmp);
    {
        File out(side_tmp, "wb");
        bool ok = out.f && out.put(kMagic, 8) && out.put(&kVersion, 1) && out.put(&flags, 1) &&
                  out.put(&n, 1) && out.put(&time, 1) && out.put(&dt, 1) && out.put(&hash, 1) &&
                  out.put(radius.data(), radius.size()) && out.put(mass.data(), mass.size()) &&
                  out.put(material.data(), material.size());
        if (ok && history)
            ok = out.put(count.data(), count.size()) && out.put(partner.data(), partner.size()) &&
                 out.put(xi.data(), xi.size());
        if (out.f) {
            ok = (std::fclose(out.f) == 0) && ok;
            out.f = nullptr;
        }
        if (!ok) {
            std::remove(state_tmp.c_str());
            std::remove(side_tmp.c_str());
            return fail(WD_ERR_IO, "wd_write_checkpoint: cannot write " + side_tmp);
        }
    }
    if (std::rename(state_tmp.c_str(), path) != 0)
        return fail(WD_ERR_IO, std::string("wd_write_checkpoint: cannot rename into ") + path);
    if (std::rename(side_tmp.c_str(), side.c_str()) != 0)
        return fail(WD_ERR_IO, "wd_write_checkpoint: cannot rename into " + side);
    return WD_OK;
}

int wd_create_from_checkpoint(const wd_config* cfg, const char* path, wd_sim** out) {
    if (!cfg || !path || !out) return fail(WD_ERR_INVALID, "wd_create_from_checkpoint: NULL argument");
    *out = nullptr;
    File in(path, "rb");
    int32_t count = 0;
    if (!in.f || !in.get(&count, 1) || count <= 0)
        return fail(WD_ERR_IO, std::string("wd_create_from_checkpoint: cannot read ") + path);
    const int64_t n = count;
    std::vector<float> state(static_cast<size_t>(6) * n);
    if (!in.get(state.data(), state.size()))
        return fail(WD_ERR_IO, std::string("wd_create_from_checkpoint: short state file ") + path);
    const std::string side = std::string(path) + ".sidecar";
    File sc(side, "rb");
    char magic[8];
    uint32_t version = 0, flags = 0;
    int64_t sn = 0;
    float time = 0.f, dt = 0.f;
    if (!sc.f || !sc.get(magic, 8) || std::memcmp(magic, kMagic, 8) != 0 || !sc.get(&version, 1) ||
        !sc.get(&flags, 1) || !sc.get(&sn, 1) || !sc.get(&time, 1) || !sc.get(&dt, 1))
        return fail(WD_ERR_IO, "wd_create_from_checkpoint: missing or bad sidecar " + side);
    if (version != 1 && version != kVersion)
        return fail(WD_ERR_IO, "wd_create_from_checkpoint: sidecar version " + std::to_string(version));
    if (sn != n)
        return fail(WD_ERR_IO, "wd_create_from_checkpoint: sidecar is for " + std::to_string(sn) +
                                   " grains, state file has " + std::to_string(n));
    if (version >= 2) {
        uint64_t hash = 0;
        if (!sc.get(&hash, 1))
            return fail(WD_ERR_IO, "wd_create_from_checkpoint: short sidecar " + side);
        if (hash != state_hash(count, state))
            return fail(WD_ERR_IO, "wd_create_from_checkpoint: " + side +
                                       " was written with another state file than " + path);
    }
    std::vector<float> radius(n), mass(n);
    std::vector<int32_t> material(n);
    if (!sc.get(radius.data(), radius.size()) || !sc.get(mass.data(), mass.size()) ||
        !sc.get(material.data(), material.size()))
        return fail(WD_ERR_IO, "wd_create_from_checkpoint: short sidecar " + side);
    std::vector<int32_t> hcount, partner;
    std::vector<float> xi;
    if (flags & 1u) {
        hcount.resize(n);
        partner.resize(static_cast<size_t>(n) * kCap);
        xi.resize(static_cast<size_t>(n) * kCap * 3);
        if (!sc.get(hcount.data(), hcount.size()) || !sc.get(partner.data(), partner.size()) ||
            !sc.get(xi.data(), xi.size()))
            return fail(WD_ERR_IO, "wd_create_from_checkpoint: short history in " + side);
    }
    wd_sim* sim = nullptr;
    int rc = wd_create_from_arrays(cfg, n, state.data(), material.data(), radius.data(),
                                   mass.data(), &sim);
    if (rc) return rc;
    rc = wd_set_dt(sim, dt);
    if (rc == WD_OK) rc = wd_set_time(sim, time);
    if (rc == WD_OK && (flags & 1u)) {
        rc = wd_set_history(sim, hcount.data(), partner.data(), xi.data());
        if (rc) {
            const std::string msg = wd_last_error();
            wd_destroy(sim);
            return fail(rc, "wd_create_from_checkpoint: the config has history off but the "
                            "checkpoint carries springs (" + msg + ")");
        }
    }
    if (rc) {
        wd_destroy(sim);
        return rc;
    }
    *out = sim;
    return WD_OK;
}

int wd_pack_frame(wd_sim* sim, const float* meta5, float* frame) {
    if (!sim || !frame) return fail(WD_ERR_INVALID, "wd_pack_frame: NULL argument");
    int64_t n = 0;
    int rc = wd_get_n(sim, &n);
    if (rc) return rc;
    rc = wd_get_positions(sim, frame);
    if (rc) return rc;
    float time = 0.f;
    wd_get_time(sim, &time);
    frame[3 * n] = time;
    for (int k = 0; k < 5; ++k) frame[3 * n + 1 + k] = meta5 ? meta5[k] : 0.f;
    return WD_OK;
}

}  // extern "C"
