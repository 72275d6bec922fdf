// wd_sim.cu -- the simulation handle behind the C ABI (include/world_b200.h).
//
// Replaces class ParticleDynamics (src/particle_dynamics.h:17-141,
// src/particle_dynamics.cu:10-358). Differences in mechanism, not in meaning:
//   * state lives on the device as sorted SoA (float4 x,y,z,r / float4 vx,vy,vz,m /
//     int id); the caller always sees AoS by grain id;
//   * a step is one CUDA graph launch on the handle's stream (search, gather,
//     contact+integrate), instead of eleven launches each followed by
//     cudaDeviceSynchronize (src/kernel.cu:31-38);
//   * errors come back as status codes; nothing calls exit() or abort().
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/world_b200.h"
#include "wd_config.h"
#include "wd_kernels.h"

namespace wd {
const char* last_error_cstr();
}

struct wd_config {
    wd::Config cfg;
};

namespace {

using wd::DevParams;

constexpr const char* kVersion = "world_b200 0.1.0 (sm_100a)";

int fail(int code, const std::string& msg) {
    wd::set_last_error(msg);
    return code;
}

#define WD_CUDA(call)                                                                   \
    do {                                                                                \
        const cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) {                                                        \
            return fail(e_ == cudaErrorMemoryAllocation ? WD_ERR_OOM : WD_ERR_CUDA,     \
                        std::string(#call) + ": " + cudaGetErrorString(e_));            \
        }                                                                               \
    } while (0)

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
}

int key_bits(uint64_t cells) {
    int b = 0;
    uint64_t v = cells > 0 ? cells - 1 : 0;
    while (v) {
        ++b;
        v >>= 1;
    }
    return b;
}

}  // namespace

struct wd_sim {
    wd::Config cfg;
    int n = 0;
    DevParams P{};
    float dt = 0.f;
    float time = 0.f;
    bool picard = false;
    int picard_iters = 1;

    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t aux_stream = nullptr;   // captures the radix path's conditional body

    // sorted SoA: A = state, B = step gather, C = on-demand gather
    float4 *posA = nullptr, *velA = nullptr, *posB = nullptr, *velB = nullptr;
    float4 *posC = nullptr, *velC = nullptr;
    int *idsA = nullptr, *idsB = nullptr, *idsC = nullptr;
    float4 *npos[2] = {nullptr, nullptr}, *nvel[2] = {nullptr, nullptr};
    float4* acc = nullptr;
    float4* hist[2] = {nullptr, nullptr};
    int* hcnt_slot = nullptr;                     // committed counts, state slot order
    int* hcnt_g = nullptr;                        // gathered counts (semi-implicit Euler)
    int* hcnt_snap[2] = {nullptr, nullptr};       // step-start counts, permuted (Picard)
    int hist_cur = 0;

    wd::SearchBuffers sb{};
    uint64_t num_cells = 0;

    // scenes: one for a plain simulation, S for a batch. Per-scene parameters live on
    // the device only for S > 1 (kernels then look each grain's scene up).
    int scenes = 1;
    std::vector<wd::Config> scene_cfg;
    std::vector<DevParams> scene_P;
    std::vector<int64_t> scene_off;       // S+1 grain offsets (grain ids of scene s)
    std::vector<int64_t> scene_nodes_off; // S+1 CIC node offsets
    DevParams* d_scene_P = nullptr;
    int* sceneA = nullptr;
    int* sceneB = nullptr;
    int* sceneC = nullptr;
    int* d_seg = nullptr;                 // S+1 segment starts (int)
    int* d_chunk_base = nullptr;          // S+1 reduction chunk offsets
    int total_chunks = 0;
    double* grain_vals = nullptr;         // 3n per-grain values for reductions
    double* scene_sums = nullptr;         // 3S per-scene sums
    unsigned long long* scene_overflow = nullptr;  // S lifetime overflow counts (batch)
    int* scene_unstable = nullptr;        // S is_stable flags (batch)
    // chaos metrics: node segments of the batch's density field
    int* d_node_seg = nullptr;
    int* d_node_chunk = nullptr;
    int node_chunks = 0;
    double* node_vals = nullptr;          // 6 values per node
    double* chaos_partials = nullptr;
    double* chaos_sums = nullptr;         // 6 per scene
    double* grain_sums = nullptr;         // 1 per scene
    float* chaos_grid = nullptr;          // 4 * nodes floats

    // Verlet lists (simulation.neighbor_skin > 0, semi-implicit Euler): the state
    // ping-pongs between the A and B buffers; lpar counts the swaps mod 2.
    // asynchronous host I/O: uploads on io_up, downloads on io_down, double-buffered
    // device staging; events order them against the step stream
    cudaStream_t io_up = nullptr, io_down = nullptr;
    float* io_in[2] = {nullptr, nullptr};
    float* io_out[2] = {nullptr, nullptr};
    cudaEvent_t ev_in_ready[2] = {nullptr, nullptr}, ev_in_free[2] = {nullptr, nullptr};
    cudaEvent_t ev_out_ready[2] = {nullptr, nullptr}, ev_out_free[2] = {nullptr, nullptr};
    cudaEvent_t ev_join = nullptr;
    int io_i = 0, io_o = 0;

    bool lists = false;
    int lpar = 0;
    int force_block = wd::kBlock;   // threads per block of the contact kernel
    int force_minb = 1;             // list contact kernel variant (1: bulk-staged)
    // Picard with lists: scratch iterate buffers (and, for a redo's gather, ids / scenes)
    float4* xpos = nullptr;
    float4* xvel = nullptr;
    int* xids = nullptr;
    int* xscene = nullptr;
    float4* rhs_vel = nullptr;      // the last iterate's velocity, slot order of rhs_ids
    int* rhs_ids = nullptr;
    int* nbr = nullptr;
    int* nbr_cnt = nullptr;
    float4* xbuild = nullptr;
    uint32_t* list_ctrl = nullptr;
    bool build_tiled = false;   // list builds stage each block's neighbour window
    bool slots_invalid = false; // a contact step stopped part-way: slot order to reset
    unsigned long long* list_len = nullptr;
    unsigned* tail_count = nullptr;  // block ticket of the contact kernel's fused decision
    bool need_build = false;         // host-side change: rebuild before the next step

    // reverse pass: snapshots of the step state (checkpoints of a recorded window and
    // the states of the segment being replayed) and the adjoint buffers
    struct Snap {
        float4* pos = nullptr;
        float4* vel = nullptr;
        int* ids = nullptr;
        uint32_t* keys = nullptr;
        int* hcnt = nullptr;
        float4* hist = nullptr;
        float time = 0.f;
    };
    std::vector<Snap> adj_ckpt;
    Snap adj_end;
    // one replayed step: its sorted input state, in-counts, springs, contacts
    struct TapeStep {
        float4* pos = nullptr;
        float4* vel = nullptr;
        int* ids = nullptr;
        int* hcnt = nullptr;
        float4* hist = nullptr;
        int* cnt_id = nullptr;
        int* clist = nullptr;
        int* ccnt = nullptr;
    };
    std::vector<TapeStep> adj_tape;
    unsigned long long* adj_ovf = nullptr;
    // captured replay / walk-back graphs per (segment length, parity); -1: replay
    std::map<std::pair<int, int>, cudaGraphExec_t> adj_graphs;
    int64_t adj_steps = 0;
    int adj_every = 0;
    float4* adj_lx[2] = {nullptr, nullptr};
    float4* adj_lv[2] = {nullptr, nullptr};
    float4* adj_lxi[2] = {nullptr, nullptr};
    float4* adj_lvt = nullptr;
    float4* adj_lf = nullptr;
    int* adj_cnt_next = nullptr;
    double* adj_theta = nullptr;

    unsigned long long* counters = nullptr;
    uint32_t* picard_res = nullptr;
    int* picard_used = nullptr;
    double* partials = nullptr;
    double* red_out = nullptr;

    uint32_t* dep_bounds = nullptr;
    unsigned long long* dep_acc = nullptr;
    float* dep_out = nullptr;
    int64_t dep_nodes = 0;

    float* staging = nullptr;   // 6n floats
    int64_t* cand_offsets = nullptr;
    int* cand_count = nullptr;

    std::vector<float> radius, mass;
    std::vector<int32_t> material;

    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    // list mode (semi-implicit Euler): the list build as device-launchable graphs per
    // step parity -- the search head (keys, mover sort), then the mover path (merge) or
    // the radix path, each followed by the gather and the listing; the contact kernel
    // tail-launches the head when it decides a build, the mover kernel the rest
    cudaGraphExec_t dev_head[2] = {nullptr, nullptr};
    cudaGraphExec_t dev_mover[2] = {nullptr, nullptr};
    cudaGraphExec_t dev_radix[2] = {nullptr, nullptr};
    // searched semi-implicit Euler steps: the step graph holds the search head (keys,
    // mover sort) and a kernel that tail-launches the rest of the step as one of two
    // device-launchable graphs: the mover path (merge) or the radix path, each followed
    // by the gather and the contact kernel
    cudaGraphExec_t dev_step_mover[2] = {nullptr, nullptr};
    cudaGraphExec_t dev_step_radix[2] = {nullptr, nullptr};
    bool graph_dirty = true;
    int kernels_per_step = 0;

    // kernel_timing: lifetime ms [search, contact+integrate, integrate, deposit]
    float wct[4] = {0.f, 0.f, 0.f, 0.f};
    std::vector<cudaEvent_t> ev_pool;
    std::vector<cudaEvent_t> ev_pending;  // triples: t0, t1, t2 per timed step
    std::vector<uint8_t> ev_contact_first;  // per triple: t0-t1 is the contact phase
};

namespace {

void clear_adj_graphs(wd_sim* s) {
    for (auto& kv : s->adj_graphs) cudaGraphExecDestroy(kv.second);
    s->adj_graphs.clear();
}

void destroy_graphs(wd_sim* s) {
    // steps still in flight may yet tail-launch the device graphs: let them finish first
    if (s->stream) cudaStreamSynchronize(s->stream);
    clear_adj_graphs(s);
    for (auto& g : s->graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    for (cudaGraphExec_t* set : {s->dev_head, s->dev_mover, s->dev_radix, s->dev_step_mover,
                                 s->dev_step_radix}) {
        for (int q = 0; q < 2; ++q) {
            if (set[q]) cudaGraphExecDestroy(set[q]);
            set[q] = nullptr;
        }
    }
    s->graph_dirty = true;
}

cudaError_t request_list_build(wd_sim* s);

// ---- snapshots of the step state, for the reverse pass ---------------------------

void free_snap(wd_sim::Snap& q) {
    void* ptrs[] = {q.pos, q.vel, q.ids, q.keys, q.hcnt, q.hist};
    for (void* p : ptrs) cudaFree(p);
    q = wd_sim::Snap{};
}

void free_tape(wd_sim* s) {
    clear_adj_graphs(s);
    for (auto& q : s->adj_ckpt) free_snap(q);
    free_snap(s->adj_end);
    for (auto& t : s->adj_tape) {
        void* ptrs[] = {t.pos, t.vel, t.ids, t.hcnt, t.hist, t.cnt_id, t.clist, t.ccnt};
        for (void* p : ptrs) cudaFree(p);
    }
    cudaFree(s->adj_ovf);
    s->adj_ovf = nullptr;
    s->adj_ckpt.clear();
    s->adj_tape.clear();
    s->adj_steps = 0;
    s->adj_every = 0;
}

cudaError_t alloc_tape_step(wd_sim* s, wd_sim::TapeStep& t) {
    const size_t n = static_cast<size_t>(s->n);
    cudaError_t e = dalloc(&t.pos, n);
    if (e == cudaSuccess) e = dalloc(&t.vel, n);
    if (e == cudaSuccess) e = dalloc(&t.ids, n);
    if (e == cudaSuccess) e = dalloc(&t.clist, n * wd::kAdjContacts);
    if (e == cudaSuccess) e = dalloc(&t.ccnt, n);
    if (e == cudaSuccess && s->P.history) e = dalloc(&t.hcnt, n);
    if (e == cudaSuccess && s->P.history) e = dalloc(&t.hist, n * wd::kHistCap);
    if (e == cudaSuccess && s->P.history) e = dalloc(&t.cnt_id, n);
    return e;
}

cudaError_t alloc_snap(wd_sim* s, wd_sim::Snap& q) {
    const size_t n = static_cast<size_t>(s->n);
    cudaError_t e = dalloc(&q.pos, n);
    if (e == cudaSuccess) e = dalloc(&q.vel, n);
    if (e == cudaSuccess) e = dalloc(&q.ids, n);
    if (e == cudaSuccess) e = dalloc(&q.keys, n);
    if (e == cudaSuccess && s->P.history) e = dalloc(&q.hcnt, n);
    if (e == cudaSuccess && s->P.history) e = dalloc(&q.hist, n * wd::kHistCap);
    return e;
}

// The state a step reads: sorted state, the keys of its slots (the incremental search
// compares against them), the stored springs and their counts, and the time.
cudaError_t take_snap(wd_sim* s, wd_sim::Snap& q) {
    const size_t n = static_cast<size_t>(s->n);
    cudaStream_t st = s->stream;
    cudaError_t e = cudaMemcpyAsync(q.pos, s->posA, n * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(q.vel, s->velA, n * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(q.ids, s->idsA, n * sizeof(int), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(q.keys, s->sb.slot_keys, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && s->P.history) {
        e = cudaMemcpyAsync(q.hcnt, s->hcnt_slot, n * sizeof(int), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(q.hist, s->hist[s->hist_cur], n * wd::kHistCap * sizeof(float4),
                                cudaMemcpyDeviceToDevice, st);
    }
    q.time = s->time;
    return e;
}

cudaError_t put_snap(wd_sim* s, const wd_sim::Snap& q) {
    const size_t n = static_cast<size_t>(s->n);
    cudaStream_t st = s->stream;
    cudaError_t e = cudaMemcpyAsync(s->posA, q.pos, n * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->velA, q.vel, n * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->idsA, q.ids, n * sizeof(int), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->sb.slot_keys, q.keys, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && s->P.history) {
        e = cudaMemcpyAsync(s->hcnt_slot, q.hcnt, n * sizeof(int), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->hist[s->hist_cur], q.hist, n * wd::kHistCap * sizeof(float4),
                                cudaMemcpyDeviceToDevice, st);
    }
    s->time = q.time;
    if (e == cudaSuccess) e = request_list_build(s);
    return e;
}

void free_sim(wd_sim* s) {
    if (!s) return;
    destroy_graphs(s);
    void* bufs[] = {s->posA, s->velA, s->posB, s->velB, s->posC, s->velC, s->idsA, s->idsB,
                    s->idsC, s->npos[0], s->npos[1], s->nvel[0], s->nvel[1], s->acc,
                    s->hist[0], s->hist[1], s->hcnt_slot, s->hcnt_g, s->hcnt_snap[0],
                    s->hcnt_snap[1], s->sb.key_by_id,
                    s->sb.slot_of_id, s->sb.keys[0], s->sb.keys[1], s->sb.vals[0],
                    s->sb.vals[1], s->sb.table_keys, s->sb.slot_keys, s->sb.newkey, s->sb.moved,
                    s->sb.blk_cnt, s->sb.blk_off, s->sb.ctrl, s->sb.mv_key, s->sb.mv_slot,
                    s->sb.src, s->sb.tile_counts, s->sb.digit_totals,
                    s->sb.table, s->counters, s->picard_res, s->picard_used, s->partials,
                    s->red_out, s->dep_bounds, s->dep_acc, s->dep_out, s->staging,
                    s->cand_offsets, s->cand_count, s->d_scene_P, s->sceneA, s->sceneB,
                    s->sceneC, s->d_seg, s->d_chunk_base, s->grain_vals, s->scene_sums,
                    s->scene_overflow, s->scene_unstable, s->d_node_seg, s->d_node_chunk,
                    s->node_vals, s->chaos_partials, s->chaos_sums, s->grain_sums,
                    s->chaos_grid, s->nbr, s->nbr_cnt, s->xbuild, s->list_ctrl, s->list_len,
                    s->tail_count, s->xpos, s->xvel, s->xids, s->xscene, s->rhs_vel, s->rhs_ids};
    for (void* b : bufs)
        if (b) cudaFree(b);
    for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : s->ev_pending) cudaEventDestroy(e);
    free_tape(s);
    for (int b = 0; b < 2; ++b) {
        cudaFree(s->io_in[b]);
        cudaFree(s->io_out[b]);
        cudaEvent_t evs[] = {s->ev_in_ready[b], s->ev_in_free[b], s->ev_out_ready[b], s->ev_out_free[b]};
        for (cudaEvent_t e : evs)
            if (e) cudaEventDestroy(e);
    }
    if (s->ev_join) cudaEventDestroy(s->ev_join);
    if (s->io_up) cudaStreamDestroy(s->io_up);
    if (s->io_down) cudaStreamDestroy(s->io_down);
    void* adj[] = {s->adj_lx[0], s->adj_lx[1], s->adj_lv[0], s->adj_lv[1], s->adj_lxi[0],
                   s->adj_lxi[1], s->adj_lvt, s->adj_lf, s->adj_cnt_next, s->adj_theta};
    for (void* p : adj) cudaFree(p);
    if (s->own_stream) cudaStreamDestroy(s->own_stream);
    if (s->aux_stream) cudaStreamDestroy(s->aux_stream);
    delete s;
}

// Derived physics constants; the same derivation is restated by the oracle.
DevParams make_params(const wd::Config& c, int n, float dt) {
    DevParams P{};
    for (int a = 0; a < 3; ++a) {
        P.lo[a] = c.dom_lo[a];
        P.hi[a] = c.dom_hi[a];
        P.grid[a] = c.grid[a];
        // cell_axis's fast path: the float box length as the kernels round it
        const float len = P.hi[a] - P.lo[a];
        P.inv_len[a] = static_cast<float>(1.0 / static_cast<double>(len));
        P.cell_err[a] = static_cast<float>(std::ldexp(static_cast<double>(P.grid[a]) + 1.0, -20));
        P.cell_len[a] = static_cast<float>(static_cast<double>(len) / P.grid[a] * (1.0 - 1e-6));
    }
    P.cell_min = std::min(P.cell_len[0], std::min(P.cell_len[1], P.cell_len[2]));
    P.ppc = c.particles_per_cell;
    P.gravity = c.gravity;
    const bool compat_k = !(c.normal_stiffness > 0.f);
    P.k_n = compat_k ? c.max_force / c.particle_radius : c.normal_stiffness;
    P.max_force = (!compat_k && !(c.max_force > 0.f)) ? INFINITY : c.max_force;
    P.k_t = c.tangential_stiffness > 0.f ? c.tangential_stiffness : (2.f / 7.f) * P.k_n;
    P.restitution = c.restitution;
    const float pi = 3.14159265358979323846f;
    P.ln_e = (c.restitution > 0.f && c.restitution < 1.f) ? logf(c.restitution) : 0.f;
    P.damp_den = sqrtf(fmaf(P.ln_e, P.ln_e, pi * pi));
    P.mu = c.friction;
    P.dt = dt;
    P.wall_lo[0] = c.wall_x_min; P.wall_lo[1] = c.wall_y_min; P.wall_lo[2] = c.floor_z;
    P.wall_hi[0] = c.wall_x_max; P.wall_hi[1] = c.wall_y_max; P.wall_hi[2] = c.ceiling_z;
    P.clamp_overlap = compat_k ? c.particle_radius : P.max_force / P.k_n;
    P.picard_tol = c.picard_tolerance;
    P.history = c.history ? 1 : 0;
    P.n = n;
    for (int a = 0; a < 3; ++a) P.dgrid[a] = c.dgrid[a];
    P.cell_base = 0;
    P.node_base = 0;
    P.frozen = 0;
    P.skin = c.neighbor_skin;
    return P;
}

// Scene tables of the A / B / C arrays (empty for a single scene).
wd::SceneTab tab(const wd_sim* s, const int* scene) {
    return s->scenes > 1 ? wd::SceneTab{s->d_scene_P, scene} : wd::SceneTab{nullptr, nullptr};
}

wd::Segments segments(const wd_sim* s) {
    return wd::Segments{s->d_seg, s->d_chunk_base, s->scenes, s->total_chunks};
}

// List mode: the buffers holding the state after a step become the A buffers.
void swap_state(wd_sim* s) {
    std::swap(s->posA, s->posB);
    std::swap(s->velA, s->velB);
    std::swap(s->idsA, s->idsB);
    if (s->P.history) std::swap(s->hcnt_slot, s->hcnt_g);
    if (s->scenes > 1) std::swap(s->sceneA, s->sceneB);
    s->lpar ^= 1;
}

// The state changed outside a step: the next step rebuilds the lists.
cudaError_t request_list_build(wd_sim* s) {
    if (!s->lists) return cudaSuccess;
    s->need_build = true;
    return cudaMemsetAsync(s->list_ctrl + wd::kLcForce, 1, 1, s->stream);
}

// One neighbor search. Inside graph capture the radix path goes into an IF
// conditional node that the mover kernel switches on only when it is needed, so
// the common step launches no idle radix kernels; outside capture every kernel is
// launched and the idle path returns at once.
cudaError_t enqueue_search(wd_sim* s, wd::Skip skip, uint32_t* zero_res, int zero_res_count,
                           bool capture, cudaStream_t st) {
    const DevParams& P = s->P;
    if (!capture) {
        wd::launch_search(P, tab(s, s->sceneA), s->posA, s->idsA, s->sb, skip, zero_res,
                          zero_res_count, s->counters, st);
        return cudaGetLastError();
    }
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle cond;
    e = cudaGraphConditionalHandleCreate(&cond, graph, 0, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return e;
    wd::launch_search_head(P, tab(s, s->sceneA), s->posA, s->idsA, s->sb, skip, zero_res,
                           zero_res_count, true, cond, s->counters, st);
    e = cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps);
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    e = cudaGraphAddNode(&node, graph, deps, ndeps, &cp);
    if (e != cudaSuccess) return e;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(s->aux_stream, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return e;
    wd::launch_search_radix(P, s->idsA, s->sb, skip, s->aux_stream);
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(s->aux_stream, &captured);
    if (e != cudaSuccess) return e;
    e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return e;
    wd::launch_search_merge(P, s->idsA, s->sb, skip, st);
    return cudaGetLastError();
}

// One take_step() enqueued on st (captured into the step graph when `capture`).
// History rows are indexed by grain id and ping-pong by step parity; their counts
// travel with the state in slot order (committed in hcnt_slot, gathered into hcnt_g,
// or for Picard into the permuted step-start snapshots hcnt_snap). `mid`, when given,
// is recorded between the search and the contact kernel (semi-implicit Euler only).
// The arguments of a searched step's contact kernel (state B -> A).
wd::ForceArgs step_force_args(wd_sim* s, int parity) {
    const bool batch = s->scenes > 1;
    wd::ForceArgs fa{};
    fa.pos = s->posB; fa.vel = s->velB; fa.ids = s->idsB; fa.table = s->sb.table;
    fa.pos_out = s->posA; fa.vel_out = s->velA; fa.ids_out = s->idsA; fa.acc_out = s->acc;
    fa.hist_in = s->hist[parity];
    fa.hist_out = s->hist[parity ^ 1];
    fa.hcnt_out = s->hcnt_slot;
    fa.counters = s->counters;
    fa.scene_params = batch ? s->d_scene_P : nullptr;
    fa.scene = s->sceneB;
    fa.scene_out = s->sceneA;
    return fa;
}

// A searched semi-implicit Euler step after its search: gather into the new order (B),
// then the contact kernel (B -> A).
void enqueue_step_tail(wd_sim* s, int parity, cudaStream_t st, cudaEvent_t mid) {
    const DevParams& P = s->P;
    const bool hist = P.history != 0, batch = s->scenes > 1;
    const wd::Skip none{nullptr, 0.f};
    wd::launch_gather(P, s->sb, s->posA, s->velA, s->posB, s->velB, s->idsB, nullptr, nullptr,
                      nullptr, nullptr, false, hist ? s->hcnt_slot : nullptr,
                      hist ? s->hcnt_g : nullptr, batch ? s->sceneA : nullptr,
                      batch ? s->sceneB : nullptr, true, s->counters, s->scene_overflow,
                      s->d_scene_P, none, st);
    if (mid) cudaEventRecord(mid, st);
    wd::ForceArgs fa = step_force_args(s, parity);
    fa.hcnt_in = s->hcnt_g;
    wd::launch_force(P, fa, false, none, st, s->force_block);
}

cudaError_t enqueue_step(wd_sim* s, int parity, cudaStream_t st, bool capture,
                         cudaEvent_t mid = nullptr) {
    const DevParams& P = s->P;
    const bool hist = P.history != 0;
    wd::ForceArgs fa{};
    fa.pos = s->posB; fa.vel = s->velB; fa.ids = s->idsB; fa.table = s->sb.table;
    fa.pos_out = s->posA; fa.vel_out = s->velA; fa.ids_out = s->idsA; fa.acc_out = s->acc;
    fa.hist_in = s->hist[parity];
    fa.hist_out = s->hist[parity ^ 1];
    fa.hcnt_out = s->hcnt_slot;
    fa.counters = s->counters;
    const bool batch = s->scenes > 1;
    fa.scene_params = batch ? s->d_scene_P : nullptr;
    fa.scene = s->sceneB;
    fa.scene_out = s->sceneA;
    const wd::Skip none{nullptr, 0.f};
    if (!s->picard) {
        if (capture && s->dev_step_mover[parity] != nullptr) {
            // the search head here, the rest of the step tail-launched from the device
            wd::launch_search_head(P, tab(s, s->sceneA), s->posA, s->idsA, s->sb, none, nullptr,
                                   0, false, 0, s->counters, st);
            wd::launch_graph_pick(s->sb.ctrl + 1, s->dev_step_mover[parity],
                                  s->dev_step_radix[parity], s->counters, st);
            return cudaGetLastError();
        }
        cudaError_t e = enqueue_search(s, none, nullptr, 0, capture, st);
        if (e != cudaSuccess) return e;
        enqueue_step_tail(s, parity, st, mid);
        return cudaGetLastError();
    }
    for (int k = 0; k < s->picard_iters; ++k) {
        const wd::Skip skip{k == 0 ? nullptr : s->picard_res + (k - 1), P.picard_tol};
        cudaError_t e = enqueue_search(s, skip, k == 0 ? s->picard_res : nullptr, s->picard_iters,
                                       capture, st);
        if (e != cudaSuccess) return e;
        const int nb = k & 1;
        const int* cnt_src = k == 0 ? s->hcnt_slot : s->hcnt_snap[nb ^ 1];
        wd::launch_gather(P, s->sb, s->posA, s->velA, s->posB, s->velB, s->idsB,
                          k == 0 ? nullptr : s->npos[nb ^ 1], k == 0 ? nullptr : s->nvel[nb ^ 1],
                          s->npos[nb], s->nvel[nb], k == 0, hist ? cnt_src : nullptr,
                          hist ? s->hcnt_snap[nb] : nullptr, batch ? s->sceneA : nullptr,
                          batch ? s->sceneB : nullptr, true, s->counters, s->scene_overflow, s->d_scene_P, skip, st);
        fa.hcnt_in = s->hcnt_snap[nb];
        fa.npos = s->npos[nb];
        fa.nvel = s->nvel[nb];
        fa.res_slot = s->picard_res + k;
        fa.picard_used = s->picard_used;
        fa.iter = k;
        wd::launch_force(P, fa, true, skip, st, s->force_block);
    }
    return cudaGetLastError();
}

// List build: search and gather the state (A) into the new order (B), list the
// neighbors of the sorted state, copy it back to A. `gate` skips it all when the
// step's decision says no build (direct launches); in a graph it is the body of an
// IF node and runs ungated.
void enqueue_list_build_tail(wd_sim* s, wd::Skip gate, cudaStream_t st);

void enqueue_list_build(wd_sim* s, wd::Skip gate, cudaStream_t st) {
    wd::launch_search(s->P, tab(s, s->sceneA), s->posA, s->idsA, s->sb, gate, nullptr, 0,
                      s->counters, st);
    enqueue_list_build_tail(s, gate, st);
}

// The build after the search: gather into the new order, list, copy back.
void enqueue_list_build_tail(wd_sim* s, wd::Skip gate, cudaStream_t st) {
    const DevParams& P = s->P;
    const bool hist = P.history != 0, batch = s->scenes > 1;
    wd::launch_gather(P, s->sb, s->posA, s->velA, s->posB, s->velB, s->idsB, nullptr, nullptr,
                      nullptr, nullptr, false, hist ? s->hcnt_slot : nullptr,
                      hist ? s->hcnt_g : nullptr, batch ? s->sceneA : nullptr,
                      batch ? s->sceneB : nullptr, true, s->counters, s->scene_overflow,
                      s->d_scene_P, gate, st);
    wd::ListCopy cp{s->velB, s->idsB, hist ? s->hcnt_g : nullptr, batch ? s->sceneB : nullptr,
                    s->posA, s->velA, s->idsA, hist ? s->hcnt_slot : nullptr,
                    batch ? s->sceneA : nullptr};
    wd::launch_list_build(P, tab(s, s->sceneB), s->posB, s->sb.table, s->nbr, s->nbr_cnt,
                          s->xbuild, s->list_ctrl, cp, gate, s->counters, s->build_tiled, st);
}

// Inside a capture on st: an IF node on `cond` after everything captured so far, its
// body the list build of the current A buffers.
cudaError_t capture_if_build(wd_sim* s, cudaStream_t st, cudaGraphConditionalHandle cond) {
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps);
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    e = cudaGraphAddNode(&node, graph, deps, ndeps, &cp);
    if (e != cudaSuccess) return e;
    e = cudaStreamBeginCaptureToGraph(s->aux_stream, cp.conditional.phGraph_out[0], nullptr,
                                      nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return e;
    enqueue_list_build(s, wd::Skip{nullptr, 0.f}, s->aux_stream);
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(s->aux_stream, &captured);
    if (e != cudaSuccess) return e;
    return cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
}

// A conditional handle of the graph being captured on st (reset to 0 every launch).
cudaError_t capture_cond(cudaStream_t st, cudaGraphConditionalHandle* cond) {
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, nullptr, nullptr);
    if (e != cudaSuccess) return e;
    return cudaGraphConditionalHandleCreate(cond, graph, 0, cudaGraphCondAssignDefault);
}

// Decide and, when needed, build (an IF node in a graph; gated launches otherwise).
// thr: the build threshold on max |x - x_build| (m).
cudaError_t enqueue_list_decide_build(wd_sim* s, float thr, cudaStream_t st, bool capture) {
    if (!capture) {
        wd::launch_list_decide(s->list_ctrl, thr, s->picard, s->counters, false, 0, st);
        enqueue_list_build(s, wd::Skip{s->list_ctrl + wd::kLcDecision, 0.5f}, st);
        return cudaGetLastError();
    }
    cudaGraphConditionalHandle cond;
    cudaError_t e = capture_cond(st, &cond);
    if (e != cudaSuccess) return e;
    wd::launch_list_decide(s->list_ctrl, thr, s->picard, s->counters, true, cond, st);
    return capture_if_build(s, st, cond);
}

// Redo of a list-mode Picard step whose iterates left the lists' validity bound: the
// step-start state is copied into B and stepped there by the per-iteration search
// (the scratch buffers take the search's gathered copy).
cudaError_t enqueue_picard_redo(wd_sim* s, int parity, cudaStream_t st) {
    const bool hist = s->P.history != 0, batch = s->scenes > 1;
    const wd::Skip none{nullptr, 0.f};
    wd::launch_list_copy(s->n, s->posA, s->velA, s->idsA, hist ? s->hcnt_slot : nullptr,
                         batch ? s->sceneA : nullptr, s->posB, s->velB, s->idsB,
                         hist ? s->hcnt_g : nullptr, batch ? s->sceneB : nullptr, none, st);
    float4 *pa = s->posA, *pb = s->posB, *va = s->velA, *vb = s->velB;
    int *ia = s->idsA, *ib = s->idsB, *ha = s->hcnt_slot, *hb = s->hcnt_g;
    int *sa = s->sceneA, *sbn = s->sceneB;
    s->posA = pb; s->velA = vb; s->idsA = ib; s->hcnt_slot = hb; s->sceneA = sbn;
    s->posB = s->xpos; s->velB = s->xvel; s->idsB = s->xids; s->sceneB = s->xscene;
    cudaError_t e = enqueue_step(s, parity, st, false, nullptr);
    // the searched step's rhs pairs its last gathered iterate with the forces
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->rhs_vel, s->xvel, sizeof(float4) * s->n, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->rhs_ids, s->xids, sizeof(int) * s->n, cudaMemcpyDeviceToDevice, st);
    s->posA = pa; s->posB = pb; s->velA = va; s->velB = vb; s->idsA = ia; s->idsB = ib;
    s->hcnt_slot = ha; s->hcnt_g = hb; s->sceneA = sa; s->sceneB = sbn;
    return e;
}

// One list-mode backward Euler / Picard step: decide, build if needed, then the
// iterations on the lists (iterates alternate between B and the scratch buffers,
// integrating from the state in A), the last iterate into B, and, when an iterate left
// the lists' validity bound, the redo. Builds start at 0.30 skin so that iterates
// rarely reach the validity bound (kListValid) within a step.
cudaError_t enqueue_step_list_picard(wd_sim* s, int parity, cudaStream_t st, bool capture,
                                     cudaEvent_t mid) {
    const DevParams& P = s->P;
    const bool hist = P.history != 0, batch = s->scenes > 1;
    const float build_at = wd::kPicardBuildAt * P.skin, valid = wd::kListValid * P.skin;
    cudaError_t e = enqueue_list_decide_build(s, build_at, st, capture);
    if (e != cudaSuccess) return e;
    if (mid) cudaEventRecord(mid, st);
    e = cudaMemsetAsync(s->picard_res, 0, sizeof(uint32_t) * s->picard_iters, st);
    if (e != cudaSuccess) return e;
    for (int k = 0; k < s->picard_iters; ++k) {
        wd::ListArgs a{};
        const bool in_b = k > 0 && ((k - 1) & 1) == 0;
        a.pos = k == 0 ? s->posA : (in_b ? s->posB : s->xpos);
        a.vel = k == 0 ? s->velA : (in_b ? s->velB : s->xvel);
        a.ids = s->idsA; a.table = s->sb.table;
        a.pos_out = (k & 1) == 0 ? s->posB : s->xpos;
        a.vel_out = (k & 1) == 0 ? s->velB : s->xvel;
        a.ids_out = s->idsB; a.acc_out = s->acc;
        a.hist_in = hist ? s->hist[parity] : nullptr;
        a.hcnt_in = hist ? s->hcnt_slot : nullptr;
        a.hist_out = hist ? s->hist[parity ^ 1] : nullptr;
        a.hcnt_out = hist ? s->hcnt_g : nullptr;
        a.counters = s->counters;
        a.nbr = s->nbr; a.nbr_cnt = s->nbr_cnt; a.xbuild = s->xbuild; a.list_ctrl = s->list_ctrl;
        a.scene_params = batch ? s->d_scene_P : nullptr;
        a.scene = s->sceneA;
        a.scene_out = s->sceneB;
        a.xn = s->posA; a.vn = s->velA;
        a.res_slot = s->picard_res + k;
        a.picard_used = s->picard_used;
        a.iter = k;
        a.viol_thr = valid * valid;
        a.skip = wd::Skip{k == 0 ? nullptr : s->picard_res + (k - 1), P.picard_tol};
        a.rhs_vel = s->rhs_vel;
        a.rhs_ids = s->rhs_ids;
        wd::launch_force_list(P, a, st, s->force_block, s->force_minb == 4 ? 4 : 5, true);
    }
    wd::launch_list_finalize(s->n, s->picard_used, s->xpos, s->xvel, s->posB, s->velB, st);
    if (!capture) {
        wd::launch_list_picard_check(s->list_ctrl, s->counters, false, 0, st);
        uint32_t redo = 0;
        e = cudaMemcpyAsync(&redo, s->list_ctrl + wd::kLcRedo, sizeof(redo), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
        if (redo) e = enqueue_picard_redo(s, parity, st);
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    e = cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle cond;
    e = cudaGraphConditionalHandleCreate(&cond, graph, 0, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return e;
    wd::launch_list_picard_check(s->list_ctrl, s->counters, true, cond, st);
    e = cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps);
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    e = cudaGraphAddNode(&node, graph, deps, ndeps, &cp);
    if (e != cudaSuccess) return e;
    e = cudaStreamBeginCaptureToGraph(s->aux_stream, cp.conditional.phGraph_out[0], nullptr,
                                      nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return e;
    const cudaError_t re = enqueue_picard_redo(s, parity, s->aux_stream);
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(s->aux_stream, &captured);
    if (re != cudaSuccess) return re;
    if (e != cudaSuccess) return e;
    e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// One list-mode step: decide, build if needed, contacts + integration from A into B.
// The buffers a list step's build works on: the step's new state (B) as the build's
// input (A), gathered through the C buffers; the step's input (A, the rhs getter's
// velocities and ids) stays as it is. Restored when the view ends.
struct BuildView {
    wd_sim* s;
    float4 *pa, *pb, *va, *vb;
    int *ia, *ib, *ha, *hb, *sa, *sbn;
    explicit BuildView(wd_sim* w)
        : s(w), pa(w->posA), pb(w->posB), va(w->velA), vb(w->velB), ia(w->idsA), ib(w->idsB),
          ha(w->hcnt_slot), hb(w->hcnt_g), sa(w->sceneA), sbn(w->sceneB) {
        s->posA = pb; s->velA = vb; s->idsA = ib; s->hcnt_slot = hb; s->sceneA = sbn;
        s->posB = s->posC; s->velB = s->velC; s->idsB = s->idsC; s->hcnt_g = ha;
        s->sceneB = s->sceneC;
    }
    ~BuildView() {
        s->posA = pa; s->posB = pb; s->velA = va; s->velB = vb; s->idsA = ia; s->idsB = ib;
        s->hcnt_slot = ha; s->hcnt_g = hb; s->sceneA = sa; s->sceneB = sbn;
    }
};

// One device-launchable graph: what `body` enqueues, captured on the auxiliary stream,
// instantiated for device launch and uploaded.
template <class Body>
cudaError_t capture_device_graph(wd_sim* s, cudaGraphExec_t* out, Body body) {
    *out = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s->aux_stream, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return e;
    body(s->aux_stream);
    const cudaError_t be = cudaGetLastError();
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(s->aux_stream, &g);
    if (be != cudaSuccess || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return be != cudaSuccess ? be : e;
    }
    e = cudaGraphInstantiate(out, g, cudaGraphInstantiateFlagDeviceLaunch);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *out = nullptr;
        return e;
    }
    return cudaGraphUpload(*out, s->aux_stream);
}

// The list build of the step graph of parity q as device graphs (see dev_head), on the
// buffers that graph's build sees. On failure none is kept and the step graph holds
// the build in a conditional node instead.
cudaError_t capture_device_builds(wd_sim* s, int q) {
    const DevParams& P = s->P;
    const wd::Skip none{nullptr, 0.f};
    BuildView view(s);
    cudaError_t e = capture_device_graph(s, &s->dev_mover[q], [&](cudaStream_t st) {
        wd::launch_search_merge(P, s->idsA, s->sb, none, st);
        enqueue_list_build_tail(s, none, st);
    });
    if (e == cudaSuccess)
        e = capture_device_graph(s, &s->dev_radix[q], [&](cudaStream_t st) {
            wd::launch_search_radix(P, s->idsA, s->sb, none, st);
            enqueue_list_build_tail(s, none, st);
        });
    if (e == cudaSuccess)
        e = capture_device_graph(s, &s->dev_head[q], [&](cudaStream_t st) {
            wd::launch_search_head(P, tab(s, s->sceneA), s->posA, s->idsA, s->sb, none, nullptr,
                                   0, false, 0, s->counters, st);
            // the path the mover kernel picked (ctrl[1]: the radix sort)
            wd::launch_graph_pick(s->sb.ctrl + 1, s->dev_mover[q], s->dev_radix[q], s->counters,
                                  st);
        });
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->aux_stream);
    if (e != cudaSuccess) {
        for (cudaGraphExec_t* x : {&s->dev_head[q], &s->dev_mover[q], &s->dev_radix[q]}) {
            if (*x) cudaGraphExecDestroy(*x);
            *x = nullptr;
        }
        cudaGetLastError();
    }
    return e;
}

// The rest of a searched step of parity q as device graphs (see dev_step_mover). On
// failure none is kept and the step graph holds the radix path in a conditional node.
cudaError_t capture_device_search_steps(wd_sim* s, int q) {
    const DevParams& P = s->P;
    const wd::Skip none{nullptr, 0.f};
    cudaError_t e = capture_device_graph(s, &s->dev_step_mover[q], [&](cudaStream_t st) {
        wd::launch_search_merge(P, s->idsA, s->sb, none, st);
        enqueue_step_tail(s, q, st, nullptr);
    });
    if (e == cudaSuccess)
        e = capture_device_graph(s, &s->dev_step_radix[q], [&](cudaStream_t st) {
            wd::launch_search_radix(P, s->idsA, s->sb, none, st);
            enqueue_step_tail(s, q, st, nullptr);
        });
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->aux_stream);
    if (e != cudaSuccess) {
        for (cudaGraphExec_t* x : {&s->dev_step_mover[q], &s->dev_step_radix[q]}) {
            if (*x) cudaGraphExecDestroy(*x);
            *x = nullptr;
        }
        cudaGetLastError();
    }
    return e;
}

// One list-mode step: decide, build if needed, contacts + integration from A into B.
cudaError_t enqueue_step_list(wd_sim* s, int parity, cudaStream_t st, bool capture,
                              cudaEvent_t mid = nullptr) {
    if (s->picard) return enqueue_step_list_picard(s, parity, st, capture, mid);
    const DevParams& P = s->P;
    const bool hist = P.history != 0, batch = s->scenes > 1;
    // in a graph, the build is either tail-launched from the device (its graphs exist)
    // or an IF node that the contact kernel switches
    const bool device_build = capture && s->dev_head[parity] != nullptr;
    cudaGraphConditionalHandle cond = 0;
    if (capture && !device_build) {
        const cudaError_t e = capture_cond(st, &cond);
        if (e != cudaSuccess) return e;
    }
    wd::ListArgs a{};
    a.thr = wd::kListValid * P.skin;
    a.tail_count = s->tail_count;
    a.use_cond = capture && !device_build ? 1 : 0;
    a.cond = cond;
    a.pos = s->posA; a.vel = s->velA; a.ids = s->idsA; a.table = s->sb.table;
    a.pos_out = s->posB; a.vel_out = s->velB; a.ids_out = s->idsB; a.acc_out = s->acc;
    a.hist_in = hist ? s->hist[parity] : nullptr;
    a.hcnt_in = hist ? s->hcnt_slot : nullptr;
    a.hist_out = hist ? s->hist[parity ^ 1] : nullptr;
    a.hcnt_out = hist ? s->hcnt_g : nullptr;
    a.counters = s->counters;
    a.nbr = s->nbr; a.nbr_cnt = s->nbr_cnt; a.xbuild = s->xbuild; a.list_ctrl = s->list_ctrl;
    a.scene_params = batch ? s->d_scene_P : nullptr;
    a.scene = s->sceneA;
    a.scene_out = s->sceneB;
    wd::launch_force_list(P, a, st, s->force_block, s->force_minb);
    if (mid) cudaEventRecord(mid, st);
    if (device_build) {
        // the build the kernel's last block decided on (kLcDecision), from the device
        wd::launch_graph_if(s->list_ctrl + wd::kLcDecision, s->dev_head[parity], s->counters, st);
        return cudaGetLastError();
    }
    // the build the kernel's last block decided on, of the new state in B
    cudaError_t e = cudaSuccess;
    {
        BuildView view(s);
        if (capture) e = capture_if_build(s, st, cond);
        else enqueue_list_build(s, wd::Skip{s->list_ctrl + wd::kLcDecision, 0.5f}, st);
    }
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// Before a list-mode step: lists that a host-side change invalidated (creation, state
// upload, snapshot restore, skin switch) are rebuilt outside the step graph, the build
// counted and the displacement bound reset by a forced decision.
cudaError_t enqueue_pending_build(wd_sim* s, cudaStream_t st) {
    if (!s->need_build) return cudaSuccess;
    s->need_build = false;
    if (s->picard) return cudaSuccess;  // the Picard step decides at its start
    return enqueue_list_decide_build(s, wd::kListValid * s->P.skin, st, false);
}

cudaError_t enqueue_any_step(wd_sim* s, int parity, cudaStream_t st, bool capture,
                             cudaEvent_t mid = nullptr) {
    return s->lists ? enqueue_step_list(s, parity, st, capture, mid)
                    : enqueue_step(s, parity, st, capture, mid);
}

int build_graphs(wd_sim* s) {
    destroy_graphs(s);
    const int count = (s->P.history || s->lists) ? 2 : 1;
    for (int parity = 0; parity < count; ++parity) {
        cudaGraph_t g = nullptr;
        // list mode: capture the graph of parity q with the buffers it will see
        const bool swapped = s->lists && s->lpar != parity;
        if (swapped) swap_state(s);
        // semi-implicit Euler on lists: the build as device-launched graphs (kept only
        // when they instantiate; otherwise the step graph holds an IF node)
        if (s->lists && !s->picard) capture_device_builds(s, parity);
        if (!s->lists && !s->picard) capture_device_search_steps(s, parity);
        WD_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t ce = enqueue_any_step(s, parity, s->stream, true);
        const cudaError_t ee = cudaStreamEndCapture(s->stream, &g);
        if (swapped) swap_state(s);
        if (ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            WD_CUDA(ce);
        }
        WD_CUDA(ee);
        size_t nodes = 0;
        cudaGraphGetNodes(g, nullptr, &nodes);
        s->kernels_per_step = static_cast<int>(nodes);
        const cudaError_t e = cudaGraphInstantiate(&s->graph[parity], g, 0);
        cudaGraphDestroy(g);
        WD_CUDA(e);
    }
    s->graph_dirty = false;
    return WD_OK;
}

int flush_timings(wd_sim* s) {
    if (s->ev_pending.empty()) return WD_OK;
    WD_CUDA(cudaEventSynchronize(s->ev_pending.back()));
    for (size_t i = 0; i + 2 < s->ev_pending.size(); i += 3) {
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, s->ev_pending[i], s->ev_pending[i + 1]);
        cudaEventElapsedTime(&b, s->ev_pending[i + 1], s->ev_pending[i + 2]);
        if (s->ev_contact_first[i / 3]) std::swap(a, b);
        s->wct[0] += a;
        s->wct[1] += b;
    }
    for (cudaEvent_t e : s->ev_pending) s->ev_pool.push_back(e);
    s->ev_pending.clear();
    s->ev_contact_first.clear();
    return WD_OK;
}

cudaEvent_t take_event(wd_sim* s) {
    if (!s->ev_pool.empty()) {
        cudaEvent_t e = s->ev_pool.back();
        s->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Timed step (drivers.kernel_timing): direct launches with events around the
// search and the contact phase; accumulated lazily, no per-step host sync. Picard
// interleaves search and contact per iteration, so its whole step counts as contact.
// A semi-implicit Euler list step runs its contact kernel first and the (gated) list
// build for the next step after it.
int timed_step(wd_sim* s, int parity) {
    if (s->ev_pending.size() >= 3 * 256) {
        const int rc = flush_timings(s);
        if (rc) return rc;
    }
    cudaStream_t st = s->stream;
    cudaEvent_t e0 = take_event(s), e1 = take_event(s), e2 = take_event(s);
    WD_CUDA(cudaEventRecord(e0, st));
    if (s->picard) WD_CUDA(cudaEventRecord(e1, st));
    WD_CUDA(enqueue_any_step(s, parity, st, false, s->picard ? nullptr : e1));
    WD_CUDA(cudaEventRecord(e2, st));
    WD_CUDA(cudaGetLastError());
    s->ev_pending.push_back(e0);
    s->ev_pending.push_back(e1);
    s->ev_pending.push_back(e2);
    s->ev_contact_first.push_back(s->lists && !s->picard ? 1 : 0);
    return WD_OK;
}

// The C state buffers: on-demand searches and the list build's gather scratch.
cudaError_t alloc_c_buffers(wd_sim* s) {
    if (s->posC) return cudaSuccess;
    cudaError_t e = dalloc(&s->posC, s->n);
    if (e == cudaSuccess) e = dalloc(&s->velC, s->n);
    if (e == cudaSuccess) e = dalloc(&s->idsC, s->n);
    if (e == cudaSuccess && s->scenes > 1) e = dalloc(&s->sceneC, s->n);
    return e;
}

// Search on the current state into the C buffers (energy, probes).
int ondemand_search(wd_sim* s) {
    const bool batch = s->scenes > 1;
    WD_CUDA(alloc_c_buffers(s));
    const wd::Skip none{nullptr, 0.f};
    wd::launch_search(s->P, tab(s, s->sceneA), s->posA, s->idsA, s->sb, none, nullptr, 0,
                      s->counters, s->stream);
    wd::launch_gather(s->P, s->sb, s->posA, s->velA, s->posC, s->velC, s->idsC, nullptr, nullptr,
                      nullptr, nullptr, false, nullptr, nullptr, batch ? s->sceneA : nullptr,
                      batch ? s->sceneC : nullptr, false, s->counters, s->scene_overflow, s->d_scene_P, none, s->stream);
    WD_CUDA(cudaGetLastError());
    return WD_OK;
}

int sync_stream(wd_sim* s) {
    WD_CUDA(cudaStreamSynchronize(s->stream));
    WD_CUDA(cudaGetLastError());
    if (s->lists && !s->picard) {
        // a list build whose device-side graph launch failed did not run
        unsigned long long failed = 0;
        WD_CUDA(cudaMemcpy(&failed, s->counters + wd::kCntLaunchFail, sizeof(failed),
                           cudaMemcpyDeviceToHost));
        if (failed) {
            WD_CUDA(cudaMemset(s->counters + wd::kCntLaunchFail, 0, sizeof(failed)));
            WD_CUDA(request_list_build(s));
            return fail(WD_ERR_CUDA, "list build: a device-side graph launch failed; the "
                                     "steps since the last synchronisation are invalid");
        }
    }
    if (s->lists && (s->force_minb == 1 || s->force_minb == 2)) {
        // the bulk-staged contact kernel flags stages that never arrived (bounded waits)
        unsigned long long stalls = 0;
        WD_CUDA(cudaMemcpy(&stalls, s->counters + wd::kCntStageTimeout, sizeof(stalls),
                           cudaMemcpyDeviceToHost));
        if (stalls) {
            // reported once: the handle stays usable. The step stopped part-way, so even
            // its slot order may be mixed (the first step after a build rewrites the
            // ids); the next state upload starts from a fresh slot order.
            WD_CUDA(cudaMemset(s->counters + wd::kCntStageTimeout, 0, sizeof(stalls)));
            s->slots_invalid = true;
            return fail(WD_ERR_CUDA, "contact kernel: a bulk copy into shared memory did not "
                                     "complete within its wait limit; the state is invalid");
        }
    }
    return WD_OK;
}

int alloc_sim(wd_sim* s) {
    const int n = s->n;
    WD_CUDA(cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking));
    WD_CUDA(cudaStreamCreateWithFlags(&s->aux_stream, cudaStreamNonBlocking));
    s->stream = s->own_stream;
    WD_CUDA(dalloc(&s->posA, n)); WD_CUDA(dalloc(&s->velA, n)); WD_CUDA(dalloc(&s->idsA, n));
    WD_CUDA(dalloc(&s->posB, n)); WD_CUDA(dalloc(&s->velB, n)); WD_CUDA(dalloc(&s->idsB, n));
    WD_CUDA(dalloc(&s->acc, n));
    if (s->picard) {
        for (int b = 0; b < 2; ++b) {
            WD_CUDA(dalloc(&s->npos[b], n));
            WD_CUDA(dalloc(&s->nvel[b], n));
        }
    }
    if (s->P.history) {
        for (int b = 0; b < 2; ++b)
            WD_CUDA(dalloc(&s->hist[b], static_cast<size_t>(n) * wd::kHistCap));
        WD_CUDA(dalloc(&s->hcnt_slot, n));
        WD_CUDA(cudaMemset(s->hcnt_slot, 0, sizeof(int) * static_cast<size_t>(n)));
        WD_CUDA(dalloc(&s->hcnt_g, n));
        if (s->picard) {
            WD_CUDA(dalloc(&s->hcnt_snap[0], n));
            WD_CUDA(dalloc(&s->hcnt_snap[1], n));
        }
    }
    wd::SearchBuffers& sb = s->sb;
    WD_CUDA(dalloc(&sb.key_by_id, n));
    WD_CUDA(dalloc(&sb.slot_of_id, n));
    for (int b = 0; b < 2; ++b) {
        WD_CUDA(dalloc(&sb.keys[b], n));
        WD_CUDA(dalloc(&sb.vals[b], n));
    }
    WD_CUDA(dalloc(&sb.table_keys, n));
    WD_CUDA(cudaMemset(sb.table_keys, 0xFF, sizeof(uint32_t) * static_cast<size_t>(n)));
    WD_CUDA(dalloc(&sb.slot_keys, n));
    WD_CUDA(cudaMemset(sb.slot_keys, 0xFF, sizeof(uint32_t) * static_cast<size_t>(n)));
    WD_CUDA(dalloc(&sb.newkey, n));
    WD_CUDA(dalloc(&sb.moved, (static_cast<size_t>(n) + 31) / 32));
    sb.num_blocks = wd::blocks_for(n);
    WD_CUDA(dalloc(&sb.blk_cnt, sb.num_blocks));
    WD_CUDA(dalloc(&sb.blk_off, static_cast<size_t>(sb.num_blocks) + 1));
    WD_CUDA(dalloc(&sb.ctrl, 2));
    WD_CUDA(cudaMemset(sb.ctrl, 0, 2 * sizeof(int)));
    WD_CUDA(dalloc(&sb.mv_key, wd::kMoverCap));
    WD_CUDA(dalloc(&sb.mv_slot, wd::kMoverCap));
    WD_CUDA(dalloc(&sb.src, n));
    WD_CUDA(wd::search_prepare());
    sb.num_tiles = static_cast<int>((static_cast<int64_t>(n) + wd::kSortTile - 1) / wd::kSortTile);
    const int bits = key_bits(s->num_cells);
    sb.passes = bits > 0 ? (bits + wd::kRadixBits - 1) / wd::kRadixBits : 1;
    sb.out = wd::radix_output(sb.passes);
    WD_CUDA(dalloc(&sb.tile_counts, static_cast<size_t>(wd::kRadix) * sb.num_tiles));
    WD_CUDA(dalloc(&sb.digit_totals, static_cast<size_t>(wd::kRadix) * sb.passes));
    WD_CUDA(dalloc(&sb.table, s->num_cells));
    WD_CUDA(cudaMemset(sb.table, 0xFF, sizeof(int2) * s->num_cells));
    WD_CUDA(dalloc(&s->counters, wd::kNumCounters));
    WD_CUDA(cudaMemset(s->counters, 0, sizeof(unsigned long long) * wd::kNumCounters));
    WD_CUDA(dalloc(&s->picard_res, s->picard_iters > 0 ? s->picard_iters : 1));
    WD_CUDA(cudaMemset(s->picard_res, 0, sizeof(uint32_t) * (s->picard_iters > 0 ? s->picard_iters : 1)));
    WD_CUDA(dalloc(&s->picard_used, 1));
    WD_CUDA(cudaMemset(s->picard_used, 0, sizeof(int)));
    WD_CUDA(dalloc(&s->red_out, 4));
    WD_CUDA(dalloc(&s->staging, static_cast<size_t>(6) * n));
    s->dep_nodes = s->scene_nodes_off.back();
    // per-scene reduction layout (segments of the sorted order, 256-grain chunks)
    const int S = s->scenes;
    std::vector<int> seg(S + 1), chunk(S + 1);
    chunk[0] = 0;
    for (int k = 0; k <= S; ++k) seg[k] = static_cast<int>(s->scene_off[k]);
    for (int k = 0; k < S; ++k)
        chunk[k + 1] = chunk[k] + static_cast<int>((s->scene_off[k + 1] - s->scene_off[k] + wd::kBlock - 1) / wd::kBlock);
    s->total_chunks = chunk[S];
    WD_CUDA(dalloc(&s->d_seg, S + 1));
    WD_CUDA(dalloc(&s->d_chunk_base, S + 1));
    WD_CUDA(cudaMemcpy(s->d_seg, seg.data(), sizeof(int) * (S + 1), cudaMemcpyHostToDevice));
    WD_CUDA(cudaMemcpy(s->d_chunk_base, chunk.data(), sizeof(int) * (S + 1), cudaMemcpyHostToDevice));
    WD_CUDA(dalloc(&s->partials, static_cast<size_t>(3) * s->total_chunks));
    WD_CUDA(dalloc(&s->scene_sums, static_cast<size_t>(3) * S));
    WD_CUDA(dalloc(&s->grain_vals, static_cast<size_t>(3) * n));
    if (S > 1) {
        WD_CUDA(dalloc(&s->d_scene_P, S));
        WD_CUDA(cudaMemcpy(s->d_scene_P, s->scene_P.data(), sizeof(DevParams) * S, cudaMemcpyHostToDevice));
        WD_CUDA(dalloc(&s->sceneA, n));
        WD_CUDA(dalloc(&s->sceneB, n));
        WD_CUDA(dalloc(&s->scene_overflow, S));
        WD_CUDA(cudaMemset(s->scene_overflow, 0, sizeof(unsigned long long) * S));
        WD_CUDA(dalloc(&s->scene_unstable, S));
    }
    if (s->lists) {
        WD_CUDA(dalloc(&s->nbr, static_cast<size_t>(n) * wd::kNbrCap));
        WD_CUDA(dalloc(&s->nbr_cnt, n));
        WD_CUDA(dalloc(&s->xbuild, n));
        WD_CUDA(dalloc(&s->list_ctrl, wd::kLcWords));
        WD_CUDA(dalloc(&s->list_len, 1));
        WD_CUDA(dalloc(&s->tail_count, 1));
        WD_CUDA(cudaMemset(s->tail_count, 0, sizeof(unsigned)));
        WD_CUDA(alloc_c_buffers(s));
        uint32_t init[wd::kLcWords] = {};
        init[wd::kLcForce] = 1u;  // the first step builds
        WD_CUDA(cudaMemcpy(s->list_ctrl, init, sizeof(init), cudaMemcpyHostToDevice));
        s->need_build = true;
        if (s->picard) {
            WD_CUDA(dalloc(&s->xpos, n));
            WD_CUDA(dalloc(&s->xvel, n));
            WD_CUDA(dalloc(&s->xids, n));
            WD_CUDA(dalloc(&s->rhs_vel, n));
            WD_CUDA(dalloc(&s->rhs_ids, n));
            if (S > 1) WD_CUDA(dalloc(&s->xscene, n));
        }
    }
    return WD_OK;
}

int upload_initial(wd_sim* s, const float* state) {
    const int n = s->n;
    std::vector<float4> pos(n), vel(n);
    std::vector<int> ids(n);
    for (int i = 0; i < n; ++i) {
        const float* q = state + 6 * static_cast<size_t>(i);
        pos[i] = make_float4(q[0], q[1], q[2], s->radius[i]);
        vel[i] = make_float4(q[3], q[4], q[5], s->mass[i]);
        ids[i] = i;
    }
    WD_CUDA(cudaMemcpy(s->posA, pos.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    WD_CUDA(cudaMemcpy(s->velA, vel.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    WD_CUDA(cudaMemcpy(s->idsA, ids.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    // B mirrors A until the first step, so get_rhs before a step reads defined data.
    WD_CUDA(cudaMemcpy(s->posB, s->posA, sizeof(float4) * n, cudaMemcpyDeviceToDevice));
    WD_CUDA(cudaMemcpy(s->velB, s->velA, sizeof(float4) * n, cudaMemcpyDeviceToDevice));
    WD_CUDA(cudaMemcpy(s->idsB, s->idsA, sizeof(int) * n, cudaMemcpyDeviceToDevice));
    if (s->rhs_vel) {
        WD_CUDA(cudaMemcpy(s->rhs_vel, s->velA, sizeof(float4) * n, cudaMemcpyDeviceToDevice));
        WD_CUDA(cudaMemcpy(s->rhs_ids, s->idsA, sizeof(int) * n, cudaMemcpyDeviceToDevice));
    }
    WD_CUDA(cudaMemset(s->acc, 0, sizeof(float4) * n));
    if (s->scenes > 1) {
        std::vector<int> sc(n);
        for (int k = 0; k < s->scenes; ++k)
            for (int64_t i = s->scene_off[k]; i < s->scene_off[k + 1]; ++i) sc[i] = k;
        WD_CUDA(cudaMemcpy(s->sceneA, sc.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
        WD_CUDA(cudaMemcpy(s->sceneB, sc.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    }
    return WD_OK;
}

// Per-grain radius and mass of one scene (the reference's mass table, or density).
int scene_grains(const wd::Config& cfg, int64_t n, const int32_t* material, const float* radius,
                 const float* mass, std::vector<float>& r_out, std::vector<float>& m_out,
                 std::vector<int32_t>& mat_out) {
    for (int64_t i = 0; i < n; ++i) {
        const int32_t mat = material ? material[i] : cfg.particle_material;
        const float r = radius ? radius[i] : cfg.particle_radius;
        float m;
        if (mass) {
            m = mass[i];
        } else if (cfg.density > 0.f) {
            const double rd = r;
            m = static_cast<float>(static_cast<double>(cfg.density) * 4.0 / 3.0 * 3.14159265358979323846 * rd * rd * rd);
        } else {
            if (mat < 0 || static_cast<size_t>(mat) >= cfg.masses.size())
                return fail(WD_ERR_INVALID, "wd_create: material id " + std::to_string(mat) +
                                                " has no entry in materials.masses");
            m = cfg.masses[mat];
        }
        r_out.push_back(r);
        m_out.push_back(m);
        mat_out.push_back(mat);
    }
    return WD_OK;
}

int check_scene_config(const wd::Config& cfg, bool have_radius) {
    for (int a = 0; a < 3; ++a) {
        if (cfg.grid[a] <= 0) return fail(WD_ERR_INVALID, "wd_create: collision grid sizes must be > 0");
        if (cfg.dgrid[a] <= 0) return fail(WD_ERR_INVALID, "wd_create: density grid sizes must be > 0");
    }
    if (!(cfg.particle_radius > 0.f) && !have_radius)
        return fail(WD_ERR_INVALID, "wd_create: physics.particle_radius must be > 0");
    if (cfg.picard_iterations < 1 && cfg.time_integrator != "semi_implicit_euler")
        return fail(WD_ERR_INVALID, "wd_create: picard_iterations must be >= 1");
    return WD_OK;
}

// S scenes in one handle. Scene k's grains get the global ids [off_k, off_k + n_k);
// its collision cells and CIC nodes are placed after those of the scenes before it.
// All scenes share the integrator, Picard settings, history mode and dt; a batch
// (S > 1) runs Picard with a fixed iteration count only.
int create_scenes(const wd::Config* const* cfgs, int S, const int64_t* counts,
                  const float* const* states, const int32_t* const* materials,
                  const float* const* radii, const float* const* masses, wd_sim** out) {
    if (!out) return fail(WD_ERR_INVALID, "wd_create: out is NULL");
    *out = nullptr;
    if (S < 1 || !cfgs || !counts || !states) return fail(WD_ERR_INVALID, "wd_create: no scenes");
    int64_t total = 0;
    uint64_t cells = 0;
    int64_t nodes = 0;
    const wd::Config& c0 = *cfgs[0];
    for (int k = 0; k < S; ++k) {
        if (!cfgs[k] || !states[k]) return fail(WD_ERR_INVALID, "wd_create: NULL scene config or state");
        const wd::Config& c = *cfgs[k];
        int rc = check_scene_config(c, radii && radii[k]);
        if (rc) return rc;
        if (counts[k] <= 0) return fail(WD_ERR_INVALID, "wd_create: every scene needs grains");
        const bool picard = c0.time_integrator != "semi_implicit_euler";
        if (k > 0 && (c.time_integrator != c0.time_integrator || c.history != c0.history ||
                      c.dt != c0.dt || (picard && c.picard_iterations != c0.picard_iterations) ||
                      c.neighbor_skin != c0.neighbor_skin))
            return fail(WD_ERR_INVALID, "wd_create: scenes of a batch must share the integrator, "
                                        "Picard iterations, history mode, neighbor skin and dt");
        if (c.neighbor_skin < 0.f) return fail(WD_ERR_INVALID, "wd_create: simulation.neighbor_skin must be >= 0");
        total += counts[k];
        cells += static_cast<uint64_t>(c.grid[0]) * c.grid[1] * c.grid[2];
        nodes += static_cast<int64_t>(c.dgrid[0]) * c.dgrid[1] * c.dgrid[2];
    }
    if (S > 1 && c0.time_integrator != "semi_implicit_euler" && c0.picard_tolerance > 0.f)
        return fail(WD_ERR_INVALID, "wd_create: a batch of scenes runs Picard with a fixed "
                                    "iteration count (time_integration.picard_tolerance: 0)");
    if (total > (int64_t{1} << 30)) return fail(WD_ERR_INVALID, "wd_create: grain count must be in [1, 2^30]");
    if (cells >= (uint64_t{1} << 32))
        return fail(WD_ERR_INVALID, "wd_create: collision grids exceed 2^32 cells in total");
    if (nodes >= (int64_t{1} << 31)) return fail(WD_ERR_INVALID, "wd_create: density grids too large");

    wd_sim* s = new wd_sim();
    s->cfg = c0;
    s->scenes = S;
    s->n = static_cast<int>(total);
    s->dt = c0.dt;
    s->picard = c0.time_integrator != "semi_implicit_euler";
    s->picard_iters = s->picard ? c0.picard_iterations : 1;
    s->lists = c0.neighbor_skin > 0.f;
    s->num_cells = cells;
    s->scene_off.assign(1, 0);
    s->scene_nodes_off.assign(1, 0);
    uint64_t cell_base = 0;
    for (int k = 0; k < S; ++k) {
        const wd::Config& c = *cfgs[k];
        s->scene_cfg.push_back(c);
        const size_t first = s->radius.size();
        int rc = scene_grains(c, counts[k], materials ? materials[k] : nullptr,
                              radii ? radii[k] : nullptr, masses ? masses[k] : nullptr, s->radius,
                              s->mass, s->material);
        if (rc) {
            delete s;
            return rc;
        }
        DevParams Q = make_params(c, static_cast<int>(counts[k]), s->dt);
        float rmax = 0.f;
        for (size_t i = first; i < s->radius.size(); ++i) rmax = fmaxf(rmax, s->radius[i]);
        Q.rmax = rmax;
        Q.cell_base = static_cast<uint32_t>(cell_base);
        Q.node_base = static_cast<int>(s->scene_nodes_off.back());
        s->scene_P.push_back(Q);
        cell_base += static_cast<uint64_t>(c.grid[0]) * c.grid[1] * c.grid[2];
        s->scene_off.push_back(s->scene_off.back() + counts[k]);
        s->scene_nodes_off.push_back(s->scene_nodes_off.back() +
                                     static_cast<int64_t>(c.dgrid[0]) * c.dgrid[1] * c.dgrid[2]);
    }
    // whole-handle parameters: scene 0's physics for a single scene; for a batch only
    // n, dt, history and the Picard settings are read from it
    s->P = s->scene_P[0];
    s->P.n = s->n;
    std::vector<float> all_state(static_cast<size_t>(6) * s->n);
    for (int k = 0; k < S; ++k)
        std::memcpy(all_state.data() + 6 * s->scene_off[k], states[k],
                    sizeof(float) * 6 * static_cast<size_t>(counts[k]));
    int rc = alloc_sim(s);
    if (rc == WD_OK) rc = upload_initial(s, all_state.data());
    if (rc != WD_OK) {
        const std::string msg = wd::last_error_cstr();
        free_sim(s);
        return fail(rc, msg);
    }
    *out = s;
    return WD_OK;
}

int create_impl(const wd::Config& cfg, int64_t n64, const float* state,
                const int32_t* material, const float* radius, const float* mass,
                wd_sim** out) {
    if (n64 <= 0 || n64 > (int64_t{1} << 30))
        return fail(WD_ERR_INVALID, "wd_create: grain count must be in [1, 2^30]");
    if (!state) return fail(WD_ERR_INVALID, "wd_create: state is NULL");
    const wd::Config* cfgs[1] = {&cfg};
    const int64_t counts[1] = {n64};
    const float* states[1] = {state};
    const int32_t* mats[1] = {material};
    const float* radii[1] = {radius};
    const float* masses[1] = {mass};
    return create_scenes(cfgs, 1, counts, states, mats, radii, masses, out);
}

}  // namespace

// ============================== C ABI ==============================================

extern "C" {

const char* wd_last_error(void) { return wd::last_error_cstr(); }
const char* wd_version(void) { return kVersion; }

int wd_config_create(wd_config** out) {
    if (!out) return fail(WD_ERR_INVALID, "wd_config_create: out is NULL");
    *out = new wd_config();
    return WD_OK;
}

int wd_config_destroy(wd_config* cfg) {
    delete cfg;
    return WD_OK;
}

int wd_config_copy(const wd_config* src, wd_config** out) {
    if (!src || !out) return fail(WD_ERR_INVALID, "wd_config_copy: NULL argument");
    *out = new wd_config(*src);
    return WD_OK;
}

int wd_config_load_yaml(wd_config* cfg, const char* path) {
    if (!cfg || !path) return fail(WD_ERR_INVALID, "wd_config_load_yaml: NULL argument");
    std::string err;
    const int rc = wd::config_load_yaml(cfg->cfg, path, &err);
    if (rc < 0) return fail(rc, err);
    if (rc == WD_WARN_DEFAULTS)
        wd::set_last_error(std::string("load_config: could not open '") + path + "'");
    return rc;
}

int wd_config_set(wd_config* cfg, const char* section, const char* key, const char* value) {
    if (!cfg || !section || !key || !value) return fail(WD_ERR_INVALID, "wd_config_set: NULL argument");
    std::string err;
    const int rc = wd::config_set(cfg->cfg, section, key, value, &err);
    if (rc < 0) return fail(rc, err);
    if (rc == WD_WARN_UNKNOWN_KEY)
        wd::set_last_error(std::string("unknown key '") + section + "." + key + "'");
    return rc;
}

int wd_config_get(const wd_config* cfg, const char* section, const char* key, char* buf,
                  size_t buf_len) {
    if (!cfg || !section || !key || !buf) return fail(WD_ERR_INVALID, "wd_config_get: NULL argument");
    std::string v;
    if (wd::config_get(cfg->cfg, section, key, &v) != WD_OK)
        return fail(WD_ERR_INVALID, std::string("unknown key '") + section + "." + key + "'");
    if (v.size() + 1 > buf_len) return fail(WD_ERR_CAPACITY, "wd_config_get: buffer too small");
    std::memcpy(buf, v.c_str(), v.size() + 1);
    return WD_OK;
}

int wd_initial_state(const wd_config* cfg, float* state, int32_t* material, int64_t capacity,
                     int64_t* n) {
    if (!cfg || !n) return fail(WD_ERR_INVALID, "wd_initial_state: NULL argument");
    wd::Grains g;
    std::string err;
    const int rc = wd::build_initial_grains(cfg->cfg, &g, &err);
    if (rc < 0) return fail(rc, err);
    *n = static_cast<int64_t>(g.material.size());
    if (*n <= capacity) {
        if (state) std::memcpy(state, g.state.data(), g.state.size() * sizeof(float));
        if (material) std::memcpy(material, g.material.data(), g.material.size() * sizeof(int32_t));
    }
    return WD_OK;
}

int wd_create(const wd_config* cfg, wd_sim** out) {
    if (!cfg) return fail(WD_ERR_INVALID, "wd_create: cfg is NULL");
    wd::Grains g;
    std::string err;
    const int rc = wd::build_initial_grains(cfg->cfg, &g, &err);
    if (rc < 0) return fail(rc, err);
    if (g.material.empty()) return fail(WD_ERR_INVALID, "wd_create: initialization produced no grains");
    return create_impl(cfg->cfg, static_cast<int64_t>(g.material.size()), g.state.data(),
                       g.material.data(), nullptr, nullptr, out);
}

int wd_create_from_arrays(const wd_config* cfg, int64_t n, const float* state,
                          const int32_t* material, const float* radius, const float* mass,
                          wd_sim** out) {
    if (!cfg) return fail(WD_ERR_INVALID, "wd_create_from_arrays: cfg is NULL");
    return create_impl(cfg->cfg, n, state, material, radius, mass, out);
}

int wd_create_batch(const wd_config* const* cfgs, int32_t num_scenes, const int64_t* counts,
                    const float* const* states, const int32_t* const* materials,
                    const float* const* radii, const float* const* masses, wd_sim** out) {
    if (!cfgs || num_scenes < 1) return fail(WD_ERR_INVALID, "wd_create_batch: no scenes");
    const int S = num_scenes;
    std::vector<const wd::Config*> c(S);
    std::vector<wd::Grains> built(S);
    std::vector<int64_t> cnt(S);
    std::vector<const float*> st(S);
    std::vector<const int32_t*> mat(S);
    for (int k = 0; k < S; ++k) {
        if (!cfgs[k]) return fail(WD_ERR_INVALID, "wd_create_batch: NULL config");
        c[k] = &cfgs[k]->cfg;
        mat[k] = materials ? materials[k] : nullptr;
        if (states && states[k]) {
            if (!counts) return fail(WD_ERR_INVALID, "wd_create_batch: states given without counts");
            st[k] = states[k];
            cnt[k] = counts[k];
            continue;
        }
        // no state: the scene's own initialization section, as wd_create
        std::string err;
        const int rc = wd::build_initial_grains(*c[k], &built[k], &err);
        if (rc < 0) return fail(rc, err);
        if (built[k].material.empty())
            return fail(WD_ERR_INVALID, "wd_create_batch: scene " + std::to_string(k) +
                                            " initialization produced no grains");
        st[k] = built[k].state.data();
        cnt[k] = static_cast<int64_t>(built[k].material.size());
        if (!mat[k]) mat[k] = built[k].material.data();
    }
    return create_scenes(c.data(), S, cnt.data(), st.data(), mat.data(), radii, masses, out);
}

int wd_scene_count(const wd_sim* sim, int32_t* scenes) {
    if (!sim || !scenes) return fail(WD_ERR_INVALID, "wd_scene_count: NULL argument");
    *scenes = sim->scenes;
    return WD_OK;
}

int wd_scene_range(const wd_sim* sim, int32_t scene, int64_t* first, int64_t* count,
                   int64_t* node_first, int64_t* nodes) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_scene_range: NULL handle");
    if (scene < 0 || scene >= sim->scenes) return fail(WD_ERR_INVALID, "wd_scene_range: scene out of range");
    if (first) *first = sim->scene_off[scene];
    if (count) *count = sim->scene_off[scene + 1] - sim->scene_off[scene];
    if (node_first) *node_first = sim->scene_nodes_off[scene];
    if (nodes) *nodes = sim->scene_nodes_off[scene + 1] - sim->scene_nodes_off[scene];
    return WD_OK;
}

int wd_destroy(wd_sim* sim) {
    if (!sim) return WD_OK;
    if (sim->stream) cudaStreamSynchronize(sim->stream);
    free_sim(sim);
    return WD_OK;
}

int wd_step(wd_sim* sim, int64_t nsteps) {
    if (!sim || nsteps < 0) return fail(WD_ERR_INVALID, "wd_step: bad argument");
    for (int64_t k = 0; k < nsteps; ++k) {
        const int parity = sim->lists ? sim->lpar : (sim->P.history ? sim->hist_cur : 0);
        if (sim->lists) WD_CUDA(enqueue_pending_build(sim, sim->stream));
        if (sim->cfg.kernel_timing) {
            const int rc = timed_step(sim, parity);
            if (rc) return rc;
        } else {
            if (sim->graph_dirty) {
                const int rc = build_graphs(sim);
                if (rc) return rc;
            }
            WD_CUDA(cudaGraphLaunch(sim->graph[parity], sim->stream));
        }
        if (sim->lists) swap_state(sim);
        if (sim->P.history) sim->hist_cur ^= 1;
        sim->time += sim->dt;
    }
    return WD_OK;
}

int wd_set_dt(wd_sim* sim, float dt) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_set_dt: NULL handle");
    if (dt != sim->dt) {
        sim->dt = dt;
        sim->P.dt = dt;
        for (DevParams& Q : sim->scene_P) Q.dt = dt;
        clear_adj_graphs(sim);
        if (sim->d_scene_P) {
            // ordered after the steps already queued, before the next one
            WD_CUDA(cudaMemcpyAsync(sim->d_scene_P, sim->scene_P.data(),
                                    sizeof(DevParams) * sim->scene_P.size(),
                                    cudaMemcpyHostToDevice, sim->stream));
            int rc = sync_stream(sim);
            if (rc) return rc;
        }
        sim->graph_dirty = true;
    }
    return WD_OK;
}

int wd_get_dt(const wd_sim* sim, float* dt) {
    if (!sim || !dt) return fail(WD_ERR_INVALID, "wd_get_dt: NULL argument");
    *dt = sim->dt;
    return WD_OK;
}

int wd_get_time(const wd_sim* sim, float* t) {
    if (!sim || !t) return fail(WD_ERR_INVALID, "wd_get_time: NULL argument");
    *t = sim->time;
    return WD_OK;
}

int wd_set_time(wd_sim* sim, float t) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_set_time: NULL handle");
    sim->time = t;
    return WD_OK;
}

int wd_get_n(const wd_sim* sim, int64_t* n) {
    if (!sim || !n) return fail(WD_ERR_INVALID, "wd_get_n: NULL argument");
    *n = sim->n;
    return WD_OK;
}

int wd_get_picard_stats(const wd_sim* sim_c, int32_t* iterations, float* residual) {
    wd_sim* sim = const_cast<wd_sim*>(sim_c);
    if (!sim) return fail(WD_ERR_INVALID, "wd_get_picard_stats: NULL handle");
    int rc = sync_stream(sim);
    if (rc) return rc;
    int used = 1;
    float res = 0.f;
    if (sim->picard) {
        WD_CUDA(cudaMemcpy(&used, sim->picard_used, sizeof(int), cudaMemcpyDeviceToHost));
        if (used > 0) {
            uint32_t bits = 0;
            WD_CUDA(cudaMemcpy(&bits, sim->picard_res + (used - 1), sizeof(uint32_t),
                               cudaMemcpyDeviceToHost));
            std::memcpy(&res, &bits, sizeof(float));
        }
    }
    if (iterations) *iterations = used;
    if (residual) *residual = res;
    return WD_OK;
}

// Slots back to grain-id order with each grain's radius, mass and scene (as at
// creation) and no stored springs, after a step that stopped part-way.
static int reset_slot_order(wd_sim* s) {
    const int n = s->n;
    std::vector<float4> pos(n), vel(n);
    std::vector<int> ids(n);
    for (int i = 0; i < n; ++i) {
        pos[i] = make_float4(0.f, 0.f, 0.f, s->radius[i]);
        vel[i] = make_float4(0.f, 0.f, 0.f, s->mass[i]);
        ids[i] = i;
    }
    WD_CUDA(cudaStreamSynchronize(s->stream));
    WD_CUDA(cudaMemcpy(s->posA, pos.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    WD_CUDA(cudaMemcpy(s->velA, vel.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    WD_CUDA(cudaMemcpy(s->idsA, ids.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    WD_CUDA(cudaMemcpy(s->idsB, ids.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    if (s->scenes > 1) {
        std::vector<int> sc(n);
        for (int k = 0; k < s->scenes; ++k)
            for (int64_t i = s->scene_off[k]; i < s->scene_off[k + 1]; ++i) sc[i] = k;
        WD_CUDA(cudaMemcpy(s->sceneA, sc.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
        WD_CUDA(cudaMemcpy(s->sceneB, sc.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    }
    if (s->P.history) {
        WD_CUDA(cudaMemset(s->hcnt_slot, 0, sizeof(int) * n));
        WD_CUDA(cudaMemset(s->hcnt_g, 0, sizeof(int) * n));
    }
    s->slots_invalid = false;
    return WD_OK;
}

int wd_set_state_device(wd_sim* sim, const float* d_state) {
    if (!sim || !d_state) return fail(WD_ERR_INVALID, "wd_set_state_device: NULL argument");
    if (sim->slots_invalid) {
        const int rc = reset_slot_order(sim);
        if (rc) return rc;
    }
    wd::launch_state_from_aos(sim->n, d_state, sim->posA, sim->velA, sim->idsA, sim->stream);
    WD_CUDA(cudaGetLastError());
    WD_CUDA(request_list_build(sim));
    return WD_OK;
}

int wd_set_state(wd_sim* sim, const float* state) {
    if (!sim || !state) return fail(WD_ERR_INVALID, "wd_set_state: NULL argument");
    WD_CUDA(cudaMemcpyAsync(sim->staging, state, sizeof(float) * 6 * static_cast<size_t>(sim->n),
                            cudaMemcpyHostToDevice, sim->stream));
    return wd_set_state_device(sim, sim->staging);
}

int wd_get_state_device(wd_sim* sim, float* d_state) {
    if (!sim || !d_state) return fail(WD_ERR_INVALID, "wd_get_state_device: NULL argument");
    wd::launch_state_to_aos(sim->n, sim->posA, sim->velA, sim->idsA, d_state, sim->stream);
    WD_CUDA(cudaGetLastError());
    return WD_OK;
}

int wd_get_state(wd_sim* sim, float* state) {
    if (!sim || !state) return fail(WD_ERR_INVALID, "wd_get_state: NULL argument");
    int rc = wd_get_state_device(sim, sim->staging);
    if (rc) return rc;
    WD_CUDA(cudaMemcpyAsync(state, sim->staging, sizeof(float) * 6 * static_cast<size_t>(sim->n),
                            cudaMemcpyDeviceToHost, sim->stream));
    return sync_stream(sim);
}

int wd_get_positions_device(wd_sim* sim, float* d_pos) {
    if (!sim || !d_pos) return fail(WD_ERR_INVALID, "wd_get_positions_device: NULL argument");
    wd::launch_positions_to_aos(sim->n, sim->posA, sim->idsA, d_pos, sim->stream);
    WD_CUDA(cudaGetLastError());
    return WD_OK;
}

int wd_get_positions(wd_sim* sim, float* positions) {
    if (!sim || !positions) return fail(WD_ERR_INVALID, "wd_get_positions: NULL argument");
    int rc = wd_get_positions_device(sim, sim->staging);
    if (rc) return rc;
    WD_CUDA(cudaMemcpyAsync(positions, sim->staging, sizeof(float) * 3 * static_cast<size_t>(sim->n),
                            cudaMemcpyDeviceToHost, sim->stream));
    return sync_stream(sim);
}

int wd_get_rhs(wd_sim* sim, float* rhs) {
    if (!sim || !rhs) return fail(WD_ERR_INVALID, "wd_get_rhs: NULL argument");
    const bool picard_lists = sim->lists && sim->picard;
    wd::launch_rhs_to_aos(sim->n, picard_lists ? sim->rhs_vel : sim->velB, sim->acc,
                          picard_lists ? sim->rhs_ids : sim->idsB, sim->staging, sim->stream);
    WD_CUDA(cudaGetLastError());
    WD_CUDA(cudaMemcpyAsync(rhs, sim->staging, sizeof(float) * 6 * static_cast<size_t>(sim->n),
                            cudaMemcpyDeviceToHost, sim->stream));
    return sync_stream(sim);
}

int wd_get_grain_props(const wd_sim* sim, float* radius, float* mass, int32_t* material) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_get_grain_props: NULL handle");
    const size_t n = static_cast<size_t>(sim->n);
    if (radius) std::memcpy(radius, sim->radius.data(), n * sizeof(float));
    if (mass) std::memcpy(mass, sim->mass.data(), n * sizeof(float));
    if (material) std::memcpy(material, sim->material.data(), n * sizeof(int32_t));
    return WD_OK;
}

int wd_set_stream(wd_sim* sim, void* stream) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_set_stream: NULL handle");
    WD_CUDA(cudaStreamSynchronize(sim->stream));
    sim->stream = stream ? static_cast<cudaStream_t>(stream) : sim->own_stream;
    return WD_OK;
}

int wd_get_stream(const wd_sim* sim, void** stream) {
    if (!sim || !stream) return fail(WD_ERR_INVALID, "wd_get_stream: NULL argument");
    *stream = static_cast<void*>(sim->stream);
    return WD_OK;
}

int wd_synchronize(wd_sim* sim) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_synchronize: NULL handle");
    if (sim->io_up) WD_CUDA(cudaStreamSynchronize(sim->io_up));
    if (sim->io_down) WD_CUDA(cudaStreamSynchronize(sim->io_down));
    return sync_stream(sim);
}

static int io_setup(wd_sim* s) {
    if (s->io_up) return WD_OK;
    const size_t n = static_cast<size_t>(s->n);
    WD_CUDA(cudaStreamCreateWithFlags(&s->io_up, cudaStreamNonBlocking));
    WD_CUDA(cudaStreamCreateWithFlags(&s->io_down, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
        WD_CUDA(dalloc(&s->io_in[b], 6 * n));
        WD_CUDA(dalloc(&s->io_out[b], 3 * n));
        cudaEvent_t* evs[] = {&s->ev_in_ready[b], &s->ev_in_free[b], &s->ev_out_ready[b],
                              &s->ev_out_free[b]};
        for (cudaEvent_t* e : evs) WD_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    WD_CUDA(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming));
    return WD_OK;
}

int wd_set_state_async(wd_sim* sim, const float* state) {
    if (!sim || !state) return fail(WD_ERR_INVALID, "wd_set_state_async: NULL argument");
    int rc = io_setup(sim);
    if (rc) return rc;
    const int i = sim->io_i;
    sim->io_i ^= 1;
    const size_t bytes = sizeof(float) * 6 * static_cast<size_t>(sim->n);
    WD_CUDA(cudaStreamWaitEvent(sim->io_up, sim->ev_in_free[i], 0));
    WD_CUDA(cudaMemcpyAsync(sim->io_in[i], state, bytes, cudaMemcpyHostToDevice, sim->io_up));
    WD_CUDA(cudaEventRecord(sim->ev_in_ready[i], sim->io_up));
    WD_CUDA(cudaStreamWaitEvent(sim->stream, sim->ev_in_ready[i], 0));
    wd::launch_state_from_aos(sim->n, sim->io_in[i], sim->posA, sim->velA, sim->idsA, sim->stream);
    WD_CUDA(cudaGetLastError());
    WD_CUDA(cudaEventRecord(sim->ev_in_free[i], sim->stream));
    WD_CUDA(request_list_build(sim));
    return WD_OK;
}

int wd_get_positions_async(wd_sim* sim, float* positions) {
    if (!sim || !positions) return fail(WD_ERR_INVALID, "wd_get_positions_async: NULL argument");
    int rc = io_setup(sim);
    if (rc) return rc;
    const int j = sim->io_o;
    sim->io_o ^= 1;
    const size_t bytes = sizeof(float) * 3 * static_cast<size_t>(sim->n);
    WD_CUDA(cudaStreamWaitEvent(sim->stream, sim->ev_out_free[j], 0));
    wd::launch_positions_to_aos(sim->n, sim->posA, sim->idsA, sim->io_out[j], sim->stream);
    WD_CUDA(cudaGetLastError());
    WD_CUDA(cudaEventRecord(sim->ev_out_ready[j], sim->stream));
    WD_CUDA(cudaStreamWaitEvent(sim->io_down, sim->ev_out_ready[j], 0));
    WD_CUDA(cudaMemcpyAsync(positions, sim->io_out[j], bytes, cudaMemcpyDeviceToHost, sim->io_down));
    WD_CUDA(cudaEventRecord(sim->ev_out_free[j], sim->io_down));
    return WD_OK;
}

int wd_io_join(wd_sim* sim) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_io_join: NULL handle");
    int rc = io_setup(sim);
    if (rc) return rc;
    // the step stream waits for every copy issued so far, the copy streams for the step stream
    WD_CUDA(cudaEventRecord(sim->ev_join, sim->io_up));
    WD_CUDA(cudaStreamWaitEvent(sim->stream, sim->ev_join, 0));
    WD_CUDA(cudaEventRecord(sim->ev_join, sim->io_down));
    WD_CUDA(cudaStreamWaitEvent(sim->stream, sim->ev_join, 0));
    WD_CUDA(cudaEventRecord(sim->ev_join, sim->stream));
    WD_CUDA(cudaStreamWaitEvent(sim->io_up, sim->ev_join, 0));
    WD_CUDA(cudaStreamWaitEvent(sim->io_down, sim->ev_join, 0));
    return WD_OK;
}

int wd_get_history(wd_sim* sim, int32_t* count, int32_t* partner, float* xi) {
    if (!sim || !count || !partner || !xi) return fail(WD_ERR_INVALID, "wd_get_history: NULL argument");
    const size_t n = static_cast<size_t>(sim->n);
    if (!sim->P.history) {
        std::memset(count, 0, n * sizeof(int32_t));
        return WD_OK;
    }
    int rc = sync_stream(sim);
    if (rc) return rc;
    std::vector<float4> rows(n * wd::kHistCap);
    // counts live in state-slot order: map them back to grain ids
    std::vector<int32_t> slot_count(n), slot_id(n);
    WD_CUDA(cudaMemcpy(slot_count.data(), sim->hcnt_slot, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    WD_CUDA(cudaMemcpy(slot_id.data(), sim->idsA, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < n; ++k) count[slot_id[k]] = slot_count[k];
    WD_CUDA(cudaMemcpy(rows.data(), sim->hist[sim->hist_cur], rows.size() * sizeof(float4),
                       cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < wd::kHistCap; ++k) {
            const float4 e = rows[i * wd::kHistCap + k];
            const bool live = k < count[i];
            int32_t p;
            std::memcpy(&p, &e.w, sizeof(int32_t));
            partner[i * wd::kHistCap + k] = live ? p : 0;
            float* x = xi + (i * wd::kHistCap + k) * 3;
            x[0] = live ? e.x : 0.f;
            x[1] = live ? e.y : 0.f;
            x[2] = live ? e.z : 0.f;
        }
    return WD_OK;
}

int wd_set_history(wd_sim* sim, const int32_t* count, const int32_t* partner, const float* xi) {
    if (!sim || !count || !partner || !xi) return fail(WD_ERR_INVALID, "wd_set_history: NULL argument");
    if (!sim->P.history) return fail(WD_ERR_INVALID, "wd_set_history: simulation.history is off");
    const size_t n = static_cast<size_t>(sim->n);
    std::vector<float4> rows(n * wd::kHistCap);
    for (size_t i = 0; i < n; ++i) {
        if (count[i] < 0 || count[i] > wd::kHistCap)
            return fail(WD_ERR_INVALID, "wd_set_history: count out of range");
        for (int k = 0; k < wd::kHistCap; ++k) {
            const float* x = xi + (i * wd::kHistCap + k) * 3;
            float w;
            std::memcpy(&w, &partner[i * wd::kHistCap + k], sizeof(float));
            rows[i * wd::kHistCap + k] = make_float4(x[0], x[1], x[2], w);
        }
    }
    int rc = sync_stream(sim);
    if (rc) return rc;
    std::vector<int32_t> slot_count(n), slot_id(n);
    WD_CUDA(cudaMemcpy(slot_id.data(), sim->idsA, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < n; ++k) slot_count[k] = count[slot_id[k]];
    WD_CUDA(cudaMemcpy(sim->hcnt_slot, slot_count.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
    WD_CUDA(cudaMemcpy(sim->hist[sim->hist_cur], rows.data(), rows.size() * sizeof(float4),
                       cudaMemcpyHostToDevice));
    return WD_OK;
}

int wd_density_grid_nodes(const wd_sim* sim, int64_t* nodes) {
    if (!sim || !nodes) return fail(WD_ERR_INVALID, "wd_density_grid_nodes: NULL argument");
    *nodes = sim->dep_nodes;
    return WD_OK;
}

int wd_compute_density_grid_device(wd_sim* sim, float* d_grid) {
    if (!sim || !d_grid) return fail(WD_ERR_INVALID, "wd_compute_density_grid_device: NULL argument");
    if (!sim->dep_acc) {
        WD_CUDA(dalloc(&sim->dep_bounds, static_cast<size_t>(4) * sim->scenes));
        WD_CUDA(dalloc(&sim->dep_acc, static_cast<size_t>(4) * sim->dep_nodes));
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (sim->cfg.kernel_timing) {
        e0 = take_event(sim);
        e1 = take_event(sim);
        WD_CUDA(cudaEventRecord(e0, sim->stream));
    }
    if (sim->scenes > 1)
        wd::launch_deposit_batch(sim->n, sim->posA, sim->velA, tab(sim, sim->sceneA), sim->scenes,
                                 sim->dep_nodes, sim->dep_bounds, sim->dep_acc, d_grid, sim->stream);
    else
        wd::launch_deposit(sim->n, sim->posA, sim->velA, sim->cfg.dom_lo, sim->cfg.dom_hi,
                           sim->cfg.dgrid, sim->dep_bounds, sim->dep_acc, d_grid, sim->stream);
    WD_CUDA(cudaGetLastError());
    if (e0) {
        WD_CUDA(cudaEventRecord(e1, sim->stream));
        WD_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        sim->wct[3] += ms;
        sim->ev_pool.push_back(e0);
        sim->ev_pool.push_back(e1);
    }
    return WD_OK;
}

int wd_compute_density_grid(wd_sim* sim, float* grid) {
    if (!sim || !grid) return fail(WD_ERR_INVALID, "wd_compute_density_grid: NULL argument");
    if (!sim->dep_out) WD_CUDA(dalloc(&sim->dep_out, static_cast<size_t>(4) * sim->dep_nodes));
    int rc = wd_compute_density_grid_device(sim, sim->dep_out);
    if (rc) return rc;
    WD_CUDA(cudaMemcpyAsync(grid, sim->dep_out, sizeof(float) * 4 * static_cast<size_t>(sim->dep_nodes),
                            cudaMemcpyDeviceToHost, sim->stream));
    return sync_stream(sim);
}

int wd_compute_scene_energies(wd_sim* sim, double* energies) {
    if (!sim || !energies) return fail(WD_ERR_INVALID, "wd_compute_scene_energies: NULL argument");
    int rc = ondemand_search(sim);
    if (rc) return rc;
    wd::launch_energy(sim->P, tab(sim, sim->sceneC), sim->posC, sim->velC, sim->idsC,
                      sim->sb.table, sim->hist[sim->hist_cur], sim->hcnt_slot, sim->sb.src,
                      segments(sim), sim->grain_vals, sim->partials, sim->scene_sums, sim->stream);
    WD_CUDA(cudaGetLastError());
    WD_CUDA(cudaMemcpyAsync(energies, sim->scene_sums, sizeof(double) * sim->scenes,
                            cudaMemcpyDeviceToHost, sim->stream));
    return sync_stream(sim);
}

int wd_grain_energies(wd_sim* sim, double* energies) {
    if (!sim || !energies) return fail(WD_ERR_INVALID, "wd_grain_energies: NULL argument");
    int rc = ondemand_search(sim);
    if (rc) return rc;
    wd::launch_energy(sim->P, tab(sim, sim->sceneC), sim->posC, sim->velC, sim->idsC,
                      sim->sb.table, sim->hist[sim->hist_cur], sim->hcnt_slot, sim->sb.src,
                      segments(sim), sim->grain_vals, sim->partials, sim->scene_sums, sim->stream);
    WD_CUDA(cudaGetLastError());
    const size_t n = static_cast<size_t>(sim->n);
    std::vector<double> by_slot(n);
    std::vector<int32_t> ids(n);
    WD_CUDA(cudaMemcpyAsync(by_slot.data(), sim->grain_vals, n * sizeof(double),
                            cudaMemcpyDeviceToHost, sim->stream));
    WD_CUDA(cudaMemcpyAsync(ids.data(), sim->idsC, n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            sim->stream));
    rc = sync_stream(sim);
    if (rc) return rc;
    for (size_t k = 0; k < n; ++k) energies[ids[k]] = by_slot[k];
    return WD_OK;
}

int wd_compute_total_energy(wd_sim* sim, double* energy) {
    if (!sim || !energy) return fail(WD_ERR_INVALID, "wd_compute_total_energy: NULL argument");
    std::vector<double> e(sim->scenes);
    int rc = wd_compute_scene_energies(sim, e.data());
    if (rc) return rc;
    double t = 0.0;
    for (double v : e) t += v;
    *energy = t;
    return WD_OK;
}

int wd_compute_scene_momenta(wd_sim* sim, double* momenta) {
    if (!sim || !momenta) return fail(WD_ERR_INVALID, "wd_compute_scene_momenta: NULL argument");
    wd::launch_momentum(sim->n, sim->velA, segments(sim), sim->grain_vals, sim->partials,
                        sim->scene_sums, sim->stream);
    WD_CUDA(cudaGetLastError());
    WD_CUDA(cudaMemcpyAsync(momenta, sim->scene_sums, 3 * sizeof(double) * sim->scenes,
                            cudaMemcpyDeviceToHost, sim->stream));
    return sync_stream(sim);
}

int wd_compute_momentum(wd_sim* sim, double* momentum3) {
    if (!sim || !momentum3) return fail(WD_ERR_INVALID, "wd_compute_momentum: NULL argument");
    std::vector<double> m(static_cast<size_t>(3) * sim->scenes);
    int rc = wd_compute_scene_momenta(sim, m.data());
    if (rc) return rc;
    for (int a = 0; a < 3; ++a) {
        double t = 0.0;
        for (int k = 0; k < sim->scenes; ++k) t += m[3 * k + a];
        momentum3[a] = t;
    }
    return WD_OK;
}

int wd_is_stable(wd_sim* sim, int32_t* stable) {
    if (!sim || !stable) return fail(WD_ERR_INVALID, "wd_is_stable: NULL argument");
    WD_CUDA(cudaMemsetAsync(sim->counters + wd::kCntUnstable, 0, sizeof(unsigned long long), sim->stream));
    wd::launch_stability(sim->P, tab(sim, sim->sceneA), sim->posA, sim->counters, nullptr,
                         sim->stream);
    WD_CUDA(cudaGetLastError());
    unsigned long long flag = 0;
    WD_CUDA(cudaMemcpyAsync(&flag, sim->counters + wd::kCntUnstable, sizeof(flag),
                            cudaMemcpyDeviceToHost, sim->stream));
    int rc = sync_stream(sim);
    if (rc) return rc;
    *stable = flag ? 0 : 1;
    return WD_OK;
}

int wd_compute_max_acceleration(wd_sim* sim, float* max_accel) {
    if (!sim || !max_accel) return fail(WD_ERR_INVALID, "wd_compute_max_acceleration: NULL argument");
    WD_CUDA(cudaMemsetAsync(sim->counters + wd::kCntMaxAccel, 0, sizeof(unsigned long long), sim->stream));
    wd::launch_max_accel(sim->n, sim->acc, sim->counters, sim->stream);
    WD_CUDA(cudaGetLastError());
    unsigned long long bits = 0;
    WD_CUDA(cudaMemcpyAsync(&bits, sim->counters + wd::kCntMaxAccel, sizeof(bits),
                            cudaMemcpyDeviceToHost, sim->stream));
    int rc = sync_stream(sim);
    if (rc) return rc;
    const uint32_t b = static_cast<uint32_t>(bits);
    std::memcpy(max_accel, &b, sizeof(float));
    return WD_OK;
}

static int read_counter(wd_sim* sim, int which, int64_t* out) {
    unsigned long long v = 0;
    WD_CUDA(cudaMemcpyAsync(&v, sim->counters + which, sizeof(v), cudaMemcpyDeviceToHost, sim->stream));
    int rc = sync_stream(sim);
    if (rc) return rc;
    *out = static_cast<int64_t>(v);
    return WD_OK;
}

int wd_grid_overflow_count(wd_sim* sim, int64_t* count) {
    if (!sim || !count) return fail(WD_ERR_INVALID, "wd_grid_overflow_count: NULL argument");
    return read_counter(sim, wd::kCntGridOverflow, count);
}

int wd_history_overflow_count(wd_sim* sim, int64_t* count) {
    if (!sim || !count) return fail(WD_ERR_INVALID, "wd_history_overflow_count: NULL argument");
    return read_counter(sim, wd::kCntHistOverflow, count);
}

int wd_radix_search_count(wd_sim* sim, int64_t* count, int32_t* kernels_each) {
    if (!sim || !count) return fail(WD_ERR_INVALID, "wd_radix_search_count: NULL argument");
    if (kernels_each) *kernels_each = 1 + 3 * sim->sb.passes;
    return read_counter(sim, wd::kCntRadixSearches, count);
}

int wd_timings(wd_sim* sim, float* ms4) {
    if (!sim || !ms4) return fail(WD_ERR_INVALID, "wd_timings: NULL argument");
    int rc = flush_timings(sim);
    if (rc) return rc;
    for (int i = 0; i < 4; ++i) ms4[i] = sim->wct[i];
    return WD_OK;
}

int wd_set_kernel_timing(wd_sim* sim, int32_t enabled) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_set_kernel_timing: NULL handle");
    sim->cfg.kernel_timing = enabled != 0;
    return WD_OK;
}

int wd_kernels_per_step(const wd_sim* sim_c, int64_t* kernels) {
    wd_sim* sim = const_cast<wd_sim*>(sim_c);
    if (!sim || !kernels) return fail(WD_ERR_INVALID, "wd_kernels_per_step: NULL argument");
    // keys, mover kernel, merge, gather, contact per search; a search that takes the
    // radix path adds 1 + 3 per pass (wd_radix_search_count)
    // list mode: the contact kernel (its last block decides the next build) and, in graph
    // mode, the kernel that launches a decided build from the device; builds add
    // wd_list_stats' count (Picard: the decision, the iterations, the last iterate's
    // copy, the redo check)
    if (sim->lists && !sim->picard) {
        const bool device = sim->dev_head[0] != nullptr || sim->dev_head[1] != nullptr;
        *kernels = device ? 2 : 1;
    } else if (!sim->lists && !sim->picard) {
        // the searched step: with its tail launched from the device, the path-pick kernel
        const bool device = sim->dev_step_mover[0] != nullptr || sim->dev_step_mover[1] != nullptr;
        *kernels = device ? 6 : 5;
    } else {
        *kernels = sim->lists ? sim->picard_iters + 3 : static_cast<int64_t>(5) * sim->picard_iters;
    }
    return WD_OK;
}

int wd_debug_cell_keys(wd_sim* sim, int32_t* keys) {
    if (!sim || !keys) return fail(WD_ERR_INVALID, "wd_debug_cell_keys: NULL argument");
    int32_t* d = reinterpret_cast<int32_t*>(sim->staging);
    wd::launch_cell_keys_by_id(sim->P, tab(sim, sim->sceneA), sim->posA, sim->idsA, d, sim->stream);
    WD_CUDA(cudaGetLastError());
    WD_CUDA(cudaMemcpyAsync(keys, d, sizeof(int32_t) * static_cast<size_t>(sim->n),
                            cudaMemcpyDeviceToHost, sim->stream));
    return sync_stream(sim);
}

int wd_debug_sorted(wd_sim* sim, int32_t* keys, int32_t* ids) {
    if (!sim || !keys || !ids) return fail(WD_ERR_INVALID, "wd_debug_sorted: NULL argument");
    int rc = ondemand_search(sim);
    if (rc) return rc;
    const size_t bytes = sizeof(int32_t) * static_cast<size_t>(sim->n);
    WD_CUDA(cudaMemcpyAsync(keys, sim->sb.keys[sim->sb.out], bytes, cudaMemcpyDeviceToHost, sim->stream));
    WD_CUDA(cudaMemcpyAsync(ids, sim->sb.vals[sim->sb.out], bytes, cudaMemcpyDeviceToHost, sim->stream));
    return sync_stream(sim);
}

int wd_debug_candidates(wd_sim* sim, int64_t* offsets, int32_t* cand, uint8_t* contact,
                        int64_t cap, int64_t* total) {
    if (!sim || !offsets || !total) return fail(WD_ERR_INVALID, "wd_debug_candidates: NULL argument");
    int rc = ondemand_search(sim);
    if (rc) return rc;
    const int n = sim->n;
    if (!sim->cand_count) {
        WD_CUDA(dalloc(&sim->cand_count, n));
        WD_CUDA(dalloc(&sim->cand_offsets, static_cast<size_t>(n) + 1));
    }
    wd::launch_candidate_count(sim->P, tab(sim, sim->sceneC), sim->posC, sim->idsC, sim->sb.table,
                               sim->cand_count, sim->stream);
    WD_CUDA(cudaGetLastError());
    std::vector<int> counts(n);
    WD_CUDA(cudaMemcpyAsync(counts.data(), sim->cand_count, sizeof(int) * n, cudaMemcpyDeviceToHost, sim->stream));
    rc = sync_stream(sim);
    if (rc) return rc;
    offsets[0] = 0;
    for (int i = 0; i < n; ++i) offsets[i + 1] = offsets[i] + counts[i];
    *total = offsets[n];
    if (!cand || !contact || *total > cap) return WD_OK;
    int* d_cand = nullptr;
    uint8_t* d_contact = nullptr;
    WD_CUDA(dalloc(&d_cand, static_cast<size_t>(*total)));
    WD_CUDA(dalloc(&d_contact, static_cast<size_t>(*total)));
    WD_CUDA(cudaMemcpyAsync(sim->cand_offsets, offsets, sizeof(int64_t) * (n + 1),
                            cudaMemcpyHostToDevice, sim->stream));
    wd::launch_candidate_fill(sim->P, tab(sim, sim->sceneC), sim->posC, sim->idsC, sim->sb.table,
                              sim->cand_offsets, d_cand, d_contact, sim->stream);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(cand, d_cand, sizeof(int32_t) * static_cast<size_t>(*total),
                            cudaMemcpyDeviceToHost, sim->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(contact, d_contact, static_cast<size_t>(*total), cudaMemcpyDeviceToHost,
                            sim->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sim->stream);
    cudaFree(d_cand);
    cudaFree(d_contact);
    WD_CUDA(e);
    return WD_OK;
}

// Skin switch on a live handle (the autotuner's knob): list buffers on first use; on
// entering list mode the current buffers are labelled with the spring parity.
static int apply_skin(wd_sim* s, float skin) {
    if (skin < 0.f) return fail(WD_ERR_INVALID, "neighbor skin must be >= 0");
    const bool lists = skin > 0.f;
    if (lists && !s->nbr) {
        const int n = s->n;
        WD_CUDA(dalloc(&s->nbr, static_cast<size_t>(n) * wd::kNbrCap));
        WD_CUDA(dalloc(&s->nbr_cnt, n));
        WD_CUDA(dalloc(&s->xbuild, n));
        WD_CUDA(dalloc(&s->list_ctrl, wd::kLcWords));
        WD_CUDA(dalloc(&s->list_len, 1));
        WD_CUDA(dalloc(&s->tail_count, 1));
        WD_CUDA(alloc_c_buffers(s));
        WD_CUDA(cudaMemsetAsync(s->list_ctrl, 0, sizeof(uint32_t) * wd::kLcWords, s->stream));
        WD_CUDA(cudaMemsetAsync(s->tail_count, 0, sizeof(unsigned), s->stream));
    }
    if (lists && s->picard && !s->xpos) {
        const int n = s->n;
        WD_CUDA(dalloc(&s->xpos, n));
        WD_CUDA(dalloc(&s->xvel, n));
        WD_CUDA(dalloc(&s->xids, n));
        WD_CUDA(dalloc(&s->rhs_vel, n));
        WD_CUDA(dalloc(&s->rhs_ids, n));
        // the rhs getter reads these in list mode: start them at the current rhs source
        WD_CUDA(cudaMemcpyAsync(s->rhs_vel, s->velB, sizeof(float4) * n, cudaMemcpyDeviceToDevice, s->stream));
        WD_CUDA(cudaMemcpyAsync(s->rhs_ids, s->idsB, sizeof(int) * n, cudaMemcpyDeviceToDevice, s->stream));
        if (s->scenes > 1) WD_CUDA(dalloc(&s->xscene, n));
    }
    if (lists && !s->lists) s->lpar = s->P.history ? s->hist_cur : s->lpar;
    s->lists = lists;
    s->cfg.neighbor_skin = skin;
    s->P.skin = skin;
    for (size_t k = 0; k < s->scene_P.size(); ++k) {
        s->scene_P[k].skin = skin;
        s->scene_cfg[k].neighbor_skin = skin;
    }
    if (s->d_scene_P)
        WD_CUDA(cudaMemcpyAsync(s->d_scene_P, s->scene_P.data(), sizeof(DevParams) * s->scene_P.size(),
                                cudaMemcpyHostToDevice, s->stream));
    WD_CUDA(request_list_build(s));
    s->graph_dirty = true;
    clear_adj_graphs(s);
    return sync_stream(s);
}

static std::string tune_key(const wd_sim* s) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    char buf[256];
    std::snprintf(buf, sizeof(buf), "n=%d,scenes=%d,grid=%dx%dx%d,sm=%d,hist=%d,picard=%d,graph=%d",
                  s->n, s->scenes, s->cfg.grid[0], s->cfg.grid[1], s->cfg.grid[2], sms,
                  s->P.history, s->picard ? 1 : 0, s->cfg.kernel_timing ? 0 : 1);
    return buf;
}

int wd_picard_counts(wd_sim* sim, int64_t* iterations, int64_t* redos) {
    if (!sim || !iterations || !redos) return fail(WD_ERR_INVALID, "wd_picard_counts: NULL argument");
    const int rc = read_counter(sim, wd::kCntPicardIters, iterations);
    return rc ? rc : read_counter(sim, wd::kCntPicardRedos, redos);
}

int wd_list_resort_count(wd_sim* sim, int64_t* grains) {
    if (!sim || !grains) return fail(WD_ERR_INVALID, "wd_list_resort_count: NULL argument");
    return read_counter(sim, wd::kCntListResort, grains);
}

int wd_list_exact_count(wd_sim* sim, int64_t* steps) {
    if (!sim || !steps) return fail(WD_ERR_INVALID, "wd_list_exact_count: NULL argument");
    return read_counter(sim, wd::kCntListExact, steps);
}

int wd_list_stats(wd_sim* sim, int64_t* builds, int32_t* kernels_each, double* mean_length) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_list_stats: NULL handle");
    if (kernels_each) {
        // device-launched builds: the head (keys, mover sort, path pick) and the mover
        // path (merge, gather, listing); in a conditional node or direct launches: every
        // search kernel (the radix ones return at once when idle), gather and listing
        const bool device = sim->dev_head[0] != nullptr || sim->dev_head[1] != nullptr;
        *kernels_each = !sim->lists ? 0 : device ? 6 : 2 + (1 + 3 * sim->sb.passes) + 1 + 2;
    }
    if (builds) {
        int rc = read_counter(sim, wd::kCntListBuilds, builds);
        if (rc) return rc;
    }
    if (mean_length) {
        *mean_length = 0.0;
        if (sim->lists) {
            WD_CUDA(cudaMemsetAsync(sim->list_len, 0, sizeof(unsigned long long), sim->stream));
            wd::launch_list_length(sim->n, sim->nbr_cnt, sim->list_len, sim->stream);
            WD_CUDA(cudaGetLastError());
            unsigned long long total = 0;
            WD_CUDA(cudaMemcpyAsync(&total, sim->list_len, sizeof(total), cudaMemcpyDeviceToHost,
                                    sim->stream));
            int rc = sync_stream(sim);
            if (rc) return rc;
            *mean_length = static_cast<double>(total) / static_cast<double>(sim->n);
        }
    }
    return WD_OK;
}

// ---- reverse pass -------------------------------------------------------------------

// Replay of one segment from the state restored into A (the checkpoint): each step's
// sorted input, contacts and springs go to the tape; the springs are read from and
// written to the tape, not to the handle's own rows.
cudaError_t adj_replay_body(wd_sim* s, int len, bool capture, cudaStream_t st) {
    const DevParams& P = s->P;
    const bool hist = P.history != 0;
    const int n = s->n;
    const wd::Skip none{nullptr, 0.f};
    for (int k = 0; k < len; ++k) {
        wd_sim::TapeStep& T = s->adj_tape[static_cast<size_t>(k)];
        wd_sim::TapeStep& T1 = s->adj_tape[static_cast<size_t>(k) + 1];
        cudaError_t e = enqueue_search(s, none, nullptr, 0, capture, st);
        if (e != cudaSuccess) return e;
        wd::launch_gather(P, s->sb, s->posA, s->velA, T.pos, T.vel, T.ids, nullptr, nullptr,
                          nullptr, nullptr, false, hist ? s->hcnt_slot : nullptr,
                          hist ? T.hcnt : nullptr, nullptr, nullptr, true, s->counters, nullptr,
                          nullptr, none, st);
        wd::launch_contact_record(P, T.pos, s->sb.table, T.clist, T.ccnt, s->adj_ovf, st);
        if (hist) wd::launch_counts_by_id(n, T.ids, T.hcnt, T.cnt_id, st);
        wd::ForceArgs fa{};
        fa.pos = T.pos; fa.vel = T.vel; fa.ids = T.ids; fa.table = s->sb.table;
        fa.pos_out = s->posA; fa.vel_out = s->velA; fa.ids_out = s->idsA;
        fa.acc_out = s->acc;
        fa.hist_in = hist ? T.hist : nullptr;
        fa.hcnt_in = hist ? T.hcnt : nullptr;
        fa.hist_out = hist ? T1.hist : nullptr;
        fa.hcnt_out = hist ? s->hcnt_slot : nullptr;
        fa.counters = s->counters;
        wd::launch_force(P, fa, false, none, st, s->force_block);
    }
    if (hist)
        wd::launch_counts_by_id(n, s->idsA, s->hcnt_slot,
                                s->adj_tape[static_cast<size_t>(len)].cnt_id, st);
    return cudaGetLastError();
}

// Walk one segment back, the adjoints starting in buffer `cur`.
cudaError_t adj_back_body(wd_sim* s, int len, int cur, cudaStream_t st) {
    const DevParams& P = s->P;
    const bool hist = P.history != 0;
    const int n = s->n;
    const size_t rows = static_cast<size_t>(n) * wd::kHistCap;
    for (int t = len - 1; t >= 0; --t) {
        const wd_sim::TapeStep& T = s->adj_tape[static_cast<size_t>(t)];
        const wd_sim::TapeStep& T1 = s->adj_tape[static_cast<size_t>(t) + 1];
        if (hist) {
            cudaError_t e = cudaMemsetAsync(s->adj_lxi[cur ^ 1], 0, rows * sizeof(float4), st);
            if (e != cudaSuccess) return e;
        }
        wd::launch_adj_prep(n, P.dt, T.vel, T.ids, s->adj_lx[cur], s->adj_lv[cur], s->adj_lvt,
                            s->adj_lf, st);
        wd::AdjArgs a{};
        a.pos = T.pos; a.vel = T.vel; a.ids = T.ids; a.table = nullptr;
        a.hist_in = hist ? T.hist : nullptr;
        a.hcnt_in = hist ? T.hcnt : nullptr;
        a.hist_next = hist ? T1.hist : nullptr;
        a.hcnt_next = hist ? T1.cnt_id : nullptr;
        a.clist = T.clist; a.ccnt = T.ccnt;
        a.lx = s->adj_lx[cur]; a.lvt = s->adj_lvt; a.lf = s->adj_lf;
        a.lxi = hist ? s->adj_lxi[cur] : nullptr;
        a.lx_out = s->adj_lx[cur ^ 1]; a.lv_out = s->adj_lv[cur ^ 1];
        a.lxi_out = hist ? s->adj_lxi[cur ^ 1] : nullptr;
        a.theta = s->adj_theta;
        a.kt_from_kn = s->cfg.tangential_stiffness > 0.f ? 0 : 1;
        wd::launch_adj_step(P, a, st);
        cur ^= 1;
    }
    return cudaGetLastError();
}

// One replay (parity -1) or walk-back segment, from a graph captured once per
// (length, parity) and kept until the step parameters or the tape change.
cudaError_t run_adj_graph(wd_sim* s, int len, int parity) {
    const auto key = std::make_pair(len, parity);
    auto it = s->adj_graphs.find(key);
    if (it == s->adj_graphs.end()) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        const cudaError_t ce = parity < 0 ? adj_replay_body(s, len, true, s->stream)
                                          : adj_back_body(s, len, parity, s->stream);
        e = cudaStreamEndCapture(s->stream, &g);
        if (ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return ce;
        }
        if (e != cudaSuccess) return e;
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return e;
        it = s->adj_graphs.emplace(key, exec).first;
    }
    return cudaGraphLaunch(it->second, s->stream);
}

int wd_get_tuning(const wd_sim* sim, float* skin, int32_t* block, int32_t* variant) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_get_tuning: NULL handle");
    if (skin) *skin = sim->cfg.neighbor_skin;
    if (block) *block = sim->force_minb <= 2 ? wd::kBlock : sim->force_block;
    if (variant)
        *variant = sim->force_minb <= 2 ? sim->force_minb : (sim->force_minb == 4 ? 64 : 48);
    return WD_OK;
}

int wd_set_build_kernel(wd_sim* sim, int32_t tiled) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_set_build_kernel: NULL handle");
    int rc = sync_stream(sim);
    if (rc) return rc;
    sim->build_tiled = tiled != 0;
    sim->graph_dirty = true;
    return WD_OK;
}

int wd_set_contact_kernel(wd_sim* sim, int32_t block, int32_t variant) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_set_contact_kernel: NULL handle");
    if (block < 32 || block > wd::kBlock || block % 32)
        return fail(WD_ERR_INVALID, "wd_set_contact_kernel: block must be a multiple of 32 up to 256");
    if (variant != 48 && variant != 64 && (variant < 0 || variant > 2))
        return fail(WD_ERR_INVALID, "wd_set_contact_kernel: variant must be 48, 64, 0, 1 or 2");
    int rc = sync_stream(sim);
    if (rc) return rc;
    sim->force_block = block;
    sim->force_minb = variant <= 2 ? variant : (variant == 64 ? 4 : 5);
    sim->graph_dirty = true;
    clear_adj_graphs(sim);
    return WD_OK;
}

int wd_debug_stage_wait(wd_sim* sim, int32_t stall, int32_t wait_us) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_debug_stage_wait: NULL handle");
    if (!sim->list_ctrl)
        return fail(WD_ERR_INVALID, "wd_debug_stage_wait: the handle has no Verlet lists");
    if (wait_us < 0) return fail(WD_ERR_INVALID, "wd_debug_stage_wait: wait_us must be >= 0");
    int rc = sync_stream(sim);
    if (rc) return rc;
    const uint32_t words[2] = {stall ? 1u : 0u, static_cast<uint32_t>(wait_us)};
    WD_CUDA(cudaMemcpy(sim->list_ctrl + wd::kLcStallTest, words, sizeof(words),
                       cudaMemcpyHostToDevice));
    return WD_OK;
}

int wd_set_neighbor_skin(wd_sim* sim, float skin) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_set_neighbor_skin: NULL handle");
    int rc = sync_stream(sim);
    if (rc) return rc;
    return apply_skin(sim, skin);
}

int wd_autotune(wd_sim* sim, int32_t steps, const char* cache_path, float* skin_out,
                int32_t* block_out) {
    if (!sim || steps < 1) return fail(WD_ERR_INVALID, "wd_autotune: bad argument");
    const std::string key = tune_key(sim);
    float best_skin = sim->cfg.neighbor_skin;
    int best_block = sim->force_block;
    int best_minb = sim->force_minb;
    bool cached = false;
    if (cache_path) {
        if (std::FILE* f = std::fopen(cache_path, "r")) {
            char line[512];
            while (std::fgets(line, sizeof(line), f)) {
                char k[300];
                float sk = 0.f;
                int bl = 0, mb = 5;
                if (std::sscanf(line, "%299s %f %d %d", k, &sk, &bl, &mb) >= 3 && key == k) {
                    best_skin = sk;
                    best_block = bl;
                    best_minb = (mb == 4 || (mb >= 0 && mb <= 2)) ? mb : 5;
                    cached = true;
                }
            }
            std::fclose(f);
        }
    }
    int rc = sync_stream(sim);
    if (rc) return rc;
    if (!cached) {
        // every candidate gives the same trajectory (lists and the block size change
        // the schedule, not the arithmetic): time each from the same saved state
        double mean_r = 0.0;
        for (float r : sim->radius) mean_r += r;
        mean_r /= static_cast<double>(sim->radius.size());
        const float d = static_cast<float>(2.0 * mean_r);
        std::vector<float> skins = {0.f};
        for (float f : {0.05f, 0.1f, 0.15f, 0.2f, 0.3f, 0.4f}) skins.push_back(f * d);
        // (block, variant): variant 5 / 4 = per-lane list kernel with 48 / 64 registers,
        // 0 = warp-cooperative list kernel, 1 / 2 = bulk-staged persistent list kernel
        // with 48 / 64 registers (256 threads each)
        const int cands[][2] = {{128, 5}, {256, 5}, {128, 4}, {256, 4}, {256, 0}, {256, 1},
                                {256, 2}};
        const int ncands = static_cast<int>(sizeof(cands) / sizeof(cands[0]));
        wd_sim::Snap snap;
        WD_CUDA(alloc_snap(sim, snap));
        WD_CUDA(take_snap(sim, snap));
        unsigned long long saved[wd::kNumCounters];
        WD_CUDA(cudaMemcpyAsync(saved, sim->counters, sizeof(saved), cudaMemcpyDeviceToHost, sim->stream));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        float best_ms = INFINITY;
        for (float sk : skins) {
            for (int cand = 0; cand < ncands && rc == WD_OK; ++cand) {
                const int bl = cands[cand][0];
                const int mb = cands[cand][1];
                if (sk == 0.f && mb != 5) continue;  // the searched kernel has one variant
                if (sim->picard && mb <= 2) continue;  // Picard: the per-lane kernel only
                rc = apply_skin(sim, sk);
                if (rc == WD_OK) {
                    sim->force_block = bl;
                    sim->force_minb = mb;
                    sim->graph_dirty = true;
                    const cudaError_t e = put_snap(sim, snap);
                    if (e != cudaSuccess) rc = fail(WD_ERR_CUDA, cudaGetErrorString(e));
                }
                if (rc == WD_OK) rc = wd_step(sim, 2);  // graphs, first list build
                if (rc == WD_OK) {
                    cudaEventRecord(e0, sim->stream);
                    rc = wd_step(sim, steps);
                    cudaEventRecord(e1, sim->stream);
                }
                if (rc == WD_OK) rc = sync_stream(sim);
                if (rc != WD_OK) break;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best_ms) {
                    best_ms = ms;
                    best_skin = sk;
                    best_block = bl;
                    best_minb = mb;
                }
            }
            if (rc != WD_OK) break;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rc == WD_OK) {
            const cudaError_t e = put_snap(sim, snap);
            if (e != cudaSuccess) rc = fail(WD_ERR_CUDA, cudaGetErrorString(e));
        }
        if (rc == WD_OK) {
            cudaMemcpyAsync(sim->counters, saved, sizeof(saved), cudaMemcpyHostToDevice, sim->stream);
            rc = sync_stream(sim);
        }
        free_snap(snap);
        if (rc) return rc;
        if (cache_path) {
            if (std::FILE* f = std::fopen(cache_path, "a")) {
                std::fprintf(f, "%s %.9g %d %d\n", key.c_str(), static_cast<double>(best_skin),
                             best_block, best_minb);
                std::fclose(f);
            }
        }
    }
    rc = apply_skin(sim, best_skin);
    if (rc) return rc;
    sim->force_block = best_block;
    sim->force_minb = best_minb;
    sim->graph_dirty = true;
    if (skin_out) *skin_out = best_skin;
    if (block_out) *block_out = best_block;
    return WD_OK;
}

int wd_set_contact_params(wd_sim* sim, float mu, float restitution, float k_n) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_set_contact_params: NULL handle");
    if (sim->scenes != 1) return fail(WD_ERR_INVALID, "wd_set_contact_params: not for a batch of scenes");
    if (!(k_n > 0.f) || !(mu >= 0.f) || !(restitution >= 0.f))
        return fail(WD_ERR_INVALID, "wd_set_contact_params: need mu >= 0, restitution >= 0, k_n > 0");
    if (sim->cfg.friction == mu && sim->cfg.restitution == restitution &&
        sim->cfg.normal_stiffness == k_n)
        return WD_OK;  // unchanged: keep the captured graphs
    int rc = sync_stream(sim);
    if (rc) return rc;
    sim->cfg.friction = mu;
    sim->cfg.restitution = restitution;
    sim->cfg.normal_stiffness = k_n;
    const float rmax = sim->P.rmax;
    sim->P = make_params(sim->cfg, sim->n, sim->dt);
    sim->P.rmax = rmax;
    sim->scene_P[0] = sim->P;
    sim->scene_cfg[0] = sim->cfg;
    sim->graph_dirty = true;
    clear_adj_graphs(sim);
    return WD_OK;
}

int wd_adjoint_record(wd_sim* sim, int64_t steps, int32_t checkpoint_every) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_adjoint_record: NULL handle");
    if (sim->picard) return fail(WD_ERR_INVALID, "wd_adjoint_record: the reverse pass covers semi-implicit Euler only");
    if (sim->scenes != 1) return fail(WD_ERR_INVALID, "wd_adjoint_record: not for a batch of scenes");
    if (steps < 1 || checkpoint_every < 1) return fail(WD_ERR_INVALID, "wd_adjoint_record: steps and checkpoint_every must be >= 1");
    int rc = sync_stream(sim);
    if (rc) return rc;
    // snapshots are kept between windows and grown when a window needs more
    const size_t nck = static_cast<size_t>((steps + checkpoint_every - 1) / checkpoint_every);
    sim->adj_steps = 0;
    for (size_t k = sim->adj_ckpt.size(); k < nck; ++k) {
        sim->adj_ckpt.emplace_back();
        WD_CUDA(alloc_snap(sim, sim->adj_ckpt.back()));
    }
    if (!sim->adj_end.pos) WD_CUDA(alloc_snap(sim, sim->adj_end));
    int64_t hist_over0 = 0;
    rc = read_counter(sim, wd::kCntHistOverflow, &hist_over0);
    if (rc) return rc;
    for (int64_t k = 0; k < steps; ++k) {
        if (k % checkpoint_every == 0) WD_CUDA(take_snap(sim, sim->adj_ckpt[static_cast<size_t>(k / checkpoint_every)]));
        rc = wd_step(sim, 1);
        if (rc) return rc;
    }
    WD_CUDA(take_snap(sim, sim->adj_end));
    int64_t hist_over1 = 0;
    rc = read_counter(sim, wd::kCntHistOverflow, &hist_over1);
    if (rc) return rc;
    sim->adj_steps = steps;
    sim->adj_every = checkpoint_every;
    if (hist_over1 != hist_over0)
        return fail(WD_ERR_CAPACITY, "wd_adjoint_record: a grain ran out of spring slots in the "
                                     "window; the reverse pass needs every spring stored");
    return WD_OK;
}

int wd_adjoint_backward(wd_sim* sim, const float* d_gx, const float* d_gv, float* d_gx0,
                        float* d_gv0, double* theta3) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_adjoint_backward: NULL handle");
    if (sim->adj_steps < 1) return fail(WD_ERR_INVALID, "wd_adjoint_backward: no window recorded (wd_adjoint_record)");
    const int n = sim->n;
    cudaStream_t st = sim->stream;
    const bool hist = sim->P.history != 0;
    if (!sim->adj_lvt) {
        for (int b = 0; b < 2; ++b) {
            WD_CUDA(dalloc(&sim->adj_lx[b], n));
            WD_CUDA(dalloc(&sim->adj_lv[b], n));
            if (hist) WD_CUDA(dalloc(&sim->adj_lxi[b], static_cast<size_t>(n) * wd::kHistCap));
        }
        WD_CUDA(dalloc(&sim->adj_lvt, n));
        WD_CUDA(dalloc(&sim->adj_lf, n));
        WD_CUDA(dalloc(&sim->adj_cnt_next, n));
        WD_CUDA(dalloc(&sim->adj_theta, static_cast<size_t>(3) * n));
    }
    const int every = sim->adj_every;
    if (sim->adj_tape.size() < static_cast<size_t>(every) + 1) clear_adj_graphs(sim);
    for (size_t k = sim->adj_tape.size(); k < static_cast<size_t>(every) + 1; ++k) {
        sim->adj_tape.emplace_back();
        WD_CUDA(alloc_tape_step(sim, sim->adj_tape.back()));
    }
    if (!sim->adj_ovf) WD_CUDA(dalloc(&sim->adj_ovf, 1));
    WD_CUDA(cudaMemsetAsync(sim->adj_ovf, 0, sizeof(unsigned long long), st));
    unsigned long long saved[wd::kNumCounters];
    WD_CUDA(cudaMemcpyAsync(saved, sim->counters, sizeof(saved), cudaMemcpyDeviceToHost, st));
    int rc = sync_stream(sim);
    if (rc) return rc;

    int cur = 0;
    wd::launch_aos3_to_f4(n, d_gx, sim->adj_lx[0], st);
    wd::launch_aos3_to_f4(n, d_gv, sim->adj_lv[0], st);
    if (hist)
        WD_CUDA(cudaMemsetAsync(sim->adj_lxi[0], 0, sizeof(float4) * n * wd::kHistCap, st));
    WD_CUDA(cudaMemsetAsync(sim->adj_theta, 0, sizeof(double) * 3 * n, st));
    const DevParams& P = sim->P;
    const wd::Skip none{nullptr, 0.f};
    const size_t rows = static_cast<size_t>(n) * wd::kHistCap;
    const int64_t nseg = static_cast<int64_t>(sim->adj_ckpt.size() == 0 ? 0 :
                                              (sim->adj_steps + every - 1) / every);
    for (int64_t seg = nseg - 1; seg >= 0; --seg) {
        const int64_t s0 = seg * every;
        const int len = static_cast<int>(std::min<int64_t>(sim->adj_steps, s0 + every) - s0);
        // replay the segment from its checkpoint, recording each step's sorted input,
        // contacts and springs on the tape (the springs live on the tape meanwhile)
        const wd_sim::Snap& ck = sim->adj_ckpt[static_cast<size_t>(seg)];
        WD_CUDA(put_snap(sim, ck));
        if (hist)
            WD_CUDA(cudaMemcpyAsync(sim->adj_tape[0].hist, ck.hist, rows * sizeof(float4),
                                    cudaMemcpyDeviceToDevice, st));
        WD_CUDA(run_adj_graph(sim, len, -1));
        WD_CUDA(run_adj_graph(sim, len, cur));
        if (len % 2) cur ^= 1;
    }
    if (d_gx0) wd::launch_f4_to_aos3(n, sim->adj_lx[cur], d_gx0, st);
    if (d_gv0) wd::launch_f4_to_aos3(n, sim->adj_lv[cur], d_gv0, st);
    wd::launch_segment_sums(sim->adj_theta, n, 3, segments(sim), sim->partials, sim->scene_sums, st);
    WD_CUDA(cudaGetLastError());
    double th[3];
    unsigned long long ovf = 0;
    WD_CUDA(cudaMemcpyAsync(th, sim->scene_sums, sizeof(th), cudaMemcpyDeviceToHost, st));
    WD_CUDA(cudaMemcpyAsync(&ovf, sim->adj_ovf, sizeof(ovf), cudaMemcpyDeviceToHost, st));
    // back to the window's end, counters as they were
    WD_CUDA(put_snap(sim, sim->adj_end));
    WD_CUDA(cudaMemcpyAsync(sim->counters, saved, sizeof(saved), cudaMemcpyHostToDevice, st));
    rc = sync_stream(sim);
    if (rc) return rc;
    if (ovf)
        return fail(WD_ERR_CAPACITY, "wd_adjoint_backward: a grain had more than " +
                                         std::to_string(wd::kAdjContacts) +
                                         " pair contacts in one step of the window");
    if (theta3) {
        const float e = sim->cfg.restitution;
        theta3[0] = th[0];
        theta3[1] = (e > 0.f && e < 1.f) ? th[1] / static_cast<double>(e) : 0.0;
        theta3[2] = th[2];
    }
    return WD_OK;
}

int wd_deposit_vjp(wd_sim* sim, const float* d_ggrid, float* d_gx, float* d_gv) {
    if (!sim || !d_ggrid) return fail(WD_ERR_INVALID, "wd_deposit_vjp: NULL argument");
    if (sim->scenes != 1) return fail(WD_ERR_INVALID, "wd_deposit_vjp: not for a batch of scenes");
    const int n = sim->n;
    if (!sim->adj_lvt) {
        for (int b = 0; b < 2; ++b) {
            WD_CUDA(dalloc(&sim->adj_lx[b], n));
            WD_CUDA(dalloc(&sim->adj_lv[b], n));
        }
        WD_CUDA(dalloc(&sim->adj_lvt, n));
        WD_CUDA(dalloc(&sim->adj_lf, n));
        WD_CUDA(dalloc(&sim->adj_cnt_next, n));
        WD_CUDA(dalloc(&sim->adj_theta, static_cast<size_t>(3) * n));
        if (sim->P.history)
            for (int b = 0; b < 2; ++b)
                WD_CUDA(dalloc(&sim->adj_lxi[b], static_cast<size_t>(n) * wd::kHistCap));
    }
    wd::launch_deposit_vjp(n, sim->posA, sim->velA, sim->idsA, sim->cfg.dom_lo, sim->cfg.dom_hi,
                           sim->cfg.dgrid, d_ggrid, sim->adj_lvt, sim->adj_lf, sim->stream);
    if (d_gx) wd::launch_f4_to_aos3(n, sim->adj_lvt, d_gx, sim->stream);
    if (d_gv) wd::launch_f4_to_aos3(n, sim->adj_lf, d_gv, sim->stream);
    WD_CUDA(cudaGetLastError());
    return sync_stream(sim);
}

// ---- batched scenes: per-scene diagnostics and ensemble metrics -----------------

int wd_scene_overflow_counts(wd_sim* sim, int64_t* counts) {
    if (!sim || !counts) return fail(WD_ERR_INVALID, "wd_scene_overflow_counts: NULL argument");
    if (sim->scenes == 1) return read_counter(sim, wd::kCntGridOverflow, counts);
    std::vector<unsigned long long> v(sim->scenes);
    WD_CUDA(cudaMemcpyAsync(v.data(), sim->scene_overflow, sizeof(unsigned long long) * v.size(),
                            cudaMemcpyDeviceToHost, sim->stream));
    const int rc = sync_stream(sim);
    if (rc) return rc;
    for (int k = 0; k < sim->scenes; ++k) counts[k] = static_cast<int64_t>(v[k]);
    return WD_OK;
}

int wd_scene_stability(wd_sim* sim, int32_t* stable) {
    if (!sim || !stable) return fail(WD_ERR_INVALID, "wd_scene_stability: NULL argument");
    if (sim->scenes == 1) return wd_is_stable(sim, stable);
    WD_CUDA(cudaMemsetAsync(sim->counters + wd::kCntUnstable, 0, sizeof(unsigned long long), sim->stream));
    WD_CUDA(cudaMemsetAsync(sim->scene_unstable, 0, sizeof(int) * sim->scenes, sim->stream));
    wd::launch_stability(sim->P, tab(sim, sim->sceneA), sim->posA, sim->counters,
                         sim->scene_unstable, sim->stream);
    WD_CUDA(cudaGetLastError());
    std::vector<int> v(sim->scenes);
    WD_CUDA(cudaMemcpyAsync(v.data(), sim->scene_unstable, sizeof(int) * v.size(),
                            cudaMemcpyDeviceToHost, sim->stream));
    const int rc = sync_stream(sim);
    if (rc) return rc;
    for (int k = 0; k < sim->scenes; ++k) stable[k] = v[k] ? 0 : 1;
    return WD_OK;
}

int wd_freeze_scene(wd_sim* sim, int32_t scene, int32_t frozen) {
    if (!sim) return fail(WD_ERR_INVALID, "wd_freeze_scene: NULL handle");
    if (sim->scenes == 1) return fail(WD_ERR_INVALID, "wd_freeze_scene: not a batch of scenes");
    if (scene < 0 || scene >= sim->scenes) return fail(WD_ERR_INVALID, "wd_freeze_scene: scene out of range");
    sim->scene_P[scene].frozen = frozen ? 1 : 0;
    // ordered after the steps already queued, before the next one
    WD_CUDA(cudaMemcpyAsync(sim->d_scene_P + scene, &sim->scene_P[scene], sizeof(DevParams),
                            cudaMemcpyHostToDevice, sim->stream));
    return sync_stream(sim);
}

int wd_chaos_metrics(wd_sim* sim, int32_t reference_scene, double* metrics3) {
    if (!sim || !metrics3) return fail(WD_ERR_INVALID, "wd_chaos_metrics: NULL argument");
    const int S = sim->scenes;
    if (reference_scene < 0 || reference_scene >= S)
        return fail(WD_ERR_INVALID, "wd_chaos_metrics: reference scene out of range");
    const int64_t n0 = sim->scene_off[1] - sim->scene_off[0];
    for (int k = 0; k < S; ++k) {
        const wd::Config& c = sim->scene_cfg[k];
        const wd::Config& c0 = sim->scene_cfg[0];
        if (sim->scene_off[k + 1] - sim->scene_off[k] != n0 ||
            c.dgrid[0] != c0.dgrid[0] || c.dgrid[1] != c0.dgrid[1] || c.dgrid[2] != c0.dgrid[2])
            return fail(WD_ERR_INVALID, "wd_chaos_metrics: every scene needs the same grain "
                                        "count and density grid");
    }
    const int total_nodes = static_cast<int>(sim->dep_nodes);
    if (!sim->d_node_seg) {
        std::vector<int> seg(S + 1), chunk(S + 1);
        chunk[0] = 0;
        for (int k = 0; k <= S; ++k) seg[k] = static_cast<int>(sim->scene_nodes_off[k]);
        for (int k = 0; k < S; ++k)
            chunk[k + 1] = chunk[k] + static_cast<int>((seg[k + 1] - seg[k] + wd::kBlock - 1) / wd::kBlock);
        sim->node_chunks = chunk[S];
        WD_CUDA(dalloc(&sim->d_node_seg, S + 1));
        WD_CUDA(dalloc(&sim->d_node_chunk, S + 1));
        WD_CUDA(cudaMemcpy(sim->d_node_seg, seg.data(), sizeof(int) * (S + 1), cudaMemcpyHostToDevice));
        WD_CUDA(cudaMemcpy(sim->d_node_chunk, chunk.data(), sizeof(int) * (S + 1), cudaMemcpyHostToDevice));
        WD_CUDA(dalloc(&sim->node_vals, static_cast<size_t>(6) * total_nodes));
        WD_CUDA(dalloc(&sim->chaos_partials, static_cast<size_t>(6) * sim->node_chunks));
        WD_CUDA(dalloc(&sim->chaos_sums, static_cast<size_t>(6) * S));
        WD_CUDA(dalloc(&sim->grain_sums, S));
        WD_CUDA(dalloc(&sim->chaos_grid, static_cast<size_t>(4) * total_nodes));
    }
    int rc = wd_compute_density_grid_device(sim, sim->chaos_grid);
    if (rc) return rc;
    float* pos3 = reinterpret_cast<float*>(sim->staging);
    rc = wd_get_positions_device(sim, pos3);
    if (rc) return rc;
    const wd::Segments nodes{sim->d_node_seg, sim->d_node_chunk, S, sim->node_chunks};
    wd::launch_chaos(sim->n, pos3, segments(sim), sim->grain_vals, sim->partials, sim->grain_sums,
                     total_nodes, sim->chaos_grid, nodes, reference_scene, sim->cfg.dgrid[1],
                     sim->cfg.dgrid[2], sim->node_vals, sim->chaos_partials, sim->chaos_sums,
                     sim->stream);
    WD_CUDA(cudaGetLastError());
    std::vector<double> g(S), f(static_cast<size_t>(6) * S);
    WD_CUDA(cudaMemcpyAsync(g.data(), sim->grain_sums, sizeof(double) * S, cudaMemcpyDeviceToHost,
                            sim->stream));
    WD_CUDA(cudaMemcpyAsync(f.data(), sim->chaos_sums, sizeof(double) * 6 * S,
                            cudaMemcpyDeviceToHost, sim->stream));
    rc = sync_stream(sim);
    if (rc) return rc;
    const double* fr = &f[6 * static_cast<size_t>(reference_scene)];
    double com_ref[3];
    for (int a = 0; a < 3; ++a) com_ref[a] = fr[2] > 0.0 ? fr[3 + a] / fr[2] : 0.0;
    for (int k = 0; k < S; ++k) {
        const double* fk = &f[6 * static_cast<size_t>(k)];
        metrics3[3 * k] = std::sqrt(g[k] / static_cast<double>(n0));
        metrics3[3 * k + 1] = fk[1] > 0.0 ? std::sqrt(fk[0] / fk[1]) : 0.0;
        double dd = 0.0;
        for (int a = 0; a < 3; ++a) {
            const double com = fk[2] > 0.0 ? fk[3 + a] / fk[2] : 0.0;
            dd += (com - com_ref[a]) * (com - com_ref[a]);
        }
        metrics3[3 * k + 2] = std::sqrt(dd);
    }
    return WD_OK;
}

}  // extern "C"
