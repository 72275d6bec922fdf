// wd_kernels.h -- host-side launchers of the sm_100a kernels (wd_search.cu,
// wd_contact.cu, wd_fields.cu). All launches are asynchronous on the given stream.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "wd_device.cuh"

namespace wd {

constexpr int kBlock = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kBlock * kSortItems;  // keys per radix-sort tile
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

inline int blocks_for(int64_t n, int block = kBlock) {
    return static_cast<int>((n + block - 1) / block);
}

// Incremental search: at most this many grains may change cell between searches
// for the mover path (a bitonic sort on one 8-CTA cluster, kMoverThreads per CTA);
// more falls back to the radix sort.
constexpr int kMoverCap = 8192;
constexpr int kMoverThreads = 1024;

// Buffers of one neighbor search (sorted by (cell key, grain id)).
struct SearchBuffers {
    uint32_t* key_by_id;     // n: cell key of grain id (radix path)
    int* slot_of_id;         // n: slot of grain id in the source state arrays (radix path)
    uint32_t* keys[2];       // n: radix ping-pong; keys[out] = sorted keys
    uint32_t* vals[2];       // n: vals[out] = grain id of each sorted position
    uint32_t* table_keys;    // n: sorted keys of the search that last wrote the table
    uint32_t* slot_keys;     // n: key of each state slot at the last step search
    uint32_t* newkey;        // n: key of each state slot now
    uint32_t* moved;         // n/32 words: bit set when a slot's key changed
    int* blk_cnt;            // movers per 256-slot block
    int* blk_off;            // exclusive prefix of blk_cnt
    int* ctrl;               // [0] mover count, [1] 1 = radix path this search
    unsigned long long* mv_key;  // kMoverCap: (key << 32 | id) of each mover
    uint32_t* mv_slot;       // kMoverCap: its state slot
    int* src;                // n: state slot of each sorted position
    uint32_t* tile_counts;   // kRadix * num_tiles
    uint32_t* digit_totals;  // kRadix * max_passes
    int2* table;             // num_cells: [start, end) of each occupied cell
    int num_tiles;
    int num_blocks;          // ceil(n / kBlock)
    int passes;              // radix passes for the key width
    int out;                 // index of the radix output buffers
};

// Picard early exit: kernels return at once when prev_res != nullptr and
// *prev_res (float bits) < tol. tol <= 0 never skips.
struct Skip {
    const uint32_t* prev_res;
    float tol;
};

// A search orders the state slots by (cell key, grain id) into keys[out] (sorted
// keys), vals[out] (grain ids) and src (source slot of each position). It has three
// parts, split so a CUDA graph can put the radix path under a conditional node:
//   head  -- keys of every slot, mover bits, and the cluster mover kernel, which
//            picks the path (ctrl[1]) and sets `cond` when use_cond;
//   radix -- stable LSD radix sort of all keys (runs when ctrl[1]);
//   merge -- merges the sorted movers into the still-sorted rest (idle when ctrl[1]).
void launch_search_head(const DevParams& P, SceneTab T, const float4* pos, const int* ids,
                        SearchBuffers& sb, Skip skip, uint32_t* zero_res, int zero_res_count,
                        bool use_cond, cudaGraphConditionalHandle cond,
                        unsigned long long* counters, cudaStream_t st);
void launch_search_radix(const DevParams& P, const int* ids, SearchBuffers& sb, Skip skip,
                         cudaStream_t st);
void launch_search_merge(const DevParams& P, const int* ids, SearchBuffers& sb, Skip skip,
                         cudaStream_t st);
// All three parts in stream order (outside graph capture).
void launch_search(const DevParams& P, SceneTab T, const float4* pos, const int* ids,
                   SearchBuffers& sb, Skip skip, uint32_t* zero_res, int zero_res_count,
                   unsigned long long* counters, cudaStream_t st);

// One-time kernel attributes (the mover kernel's shared memory); call before capture.
cudaError_t search_prepare();
// Index of the radix output buffers for a number of passes.
int radix_output(int passes);

// Gather the source state into sorted order (and the Picard snapshot when given),
// fused with the run table. History counts travel with the state in slot order:
// cnt_dst[p] = cnt_src[src[p]] (both NULL without history). step_search: the sorted
// order becomes the state's slot order, so the slot keys are recorded for the next
// search's mover test.
void launch_gather(const DevParams& P, SearchBuffers& sb, const float4* posA,
                   const float4* velA, float4* posB, float4* velB, int* idsB,
                   const float4* nposA, const float4* nvelA, float4* nposB, float4* nvelB,
                   bool snap_from_state, const int* cnt_src, int* cnt_dst, const int* scene_src,
                   int* scene_dst, bool step_search, unsigned long long* counters,
                   unsigned long long* scene_overflow, const DevParams* scene_params, Skip skip,
                   cudaStream_t st);

struct ForceArgs {
    const float4* pos; const float4* vel; const int* ids;  // sorted step input
    const int2* table;
    float4* pos_out; float4* vel_out; int* ids_out;        // integrated state
    float4* acc_out;                                       // F/m per slot
    const float4* npos; const float4* nvel;                // Picard x^n, v^n
    const float4* hist_in;                                 // committed rows, by grain id
    const int* hcnt_in;                                    // their counts, by sorted slot
    float4* hist_out;                                      // new rows, by grain id
    int* hcnt_out;                                         // new counts, by sorted slot
    unsigned long long* counters;
    uint32_t* res_slot;                                    // Picard residual (bits)
    int* picard_used;
    int iter;
    const DevParams* scene_params;                         // batched scenes (or NULL)
    const int* scene;                                      // scene of each input slot
    int* scene_out;                                        // scene of each output slot
};

// Scene segments of the sorted order, for per-scene reductions: seg[S+1] grain
// offsets (scene s holds sorted positions [seg[s], seg[s+1])), chunk_base[S+1] prefix
// of ceil(n_s / kBlock).
struct Segments {
    const int* seg;
    const int* chunk_base;
    int scenes;
    int total_chunks;
};

// block: threads per block (a multiple of 32, at most kBlock; the autotuner's choice)
void launch_force(const DevParams& P, const ForceArgs& a, bool picard, Skip skip,
                  cudaStream_t st, int block = kBlock);

// Verlet lists (simulation.neighbor_skin > 0). list_ctrl words:
// [0] max |x - x_build|^2 over the last step's output (float bits; measured only when
// [7] was set), [1] a list overflowed, [2] rebuild requested by the host, [3] this
// step's decision (1.0f: rebuild). Picard: [4] an iteration started from an iterate
// kListValid skin or more from its build position, [5] this step's redo decision (1.0f: redo
// with the per-iteration search). [6] max |x_out - x_in|^2 of the last step (float
// bits), [7] the contact kernel measures [0] this step, [8..9] (double) a bound on
// max |x - x_build| of the current state.
// Verlet-list validity: every grain within kListValid skins of its build position.
// Pairs not listed were >= r_i + r_j + skin apart at the build; after displacements of
// at most kListValid skin each they are still >= r_i + r_j + 0.02 skin apart (10 um at
// a 0.5 mm skin, many orders of magnitude above the float rounding of the distance
// tests). Picard builds earlier, at kPicardBuildAt, so that its iterates rarely leave.
constexpr float kListValid = 0.49f;
constexpr float kPicardBuildAt = 0.30f;
// kLcStallTest / kLcWaitUs: the bulk-staged contact kernel's wait test. A nonzero
// kLcStallTest makes each warp's first stage expect 16 bytes that no copy delivers (no
// copy is issued for it), so its bounded wait runs out; kLcWaitUs is that wait's limit
// in microseconds (0: one second).
enum ListCtrl {
    kLcDisp = 0, kLcOverflow = 1, kLcForce = 2, kLcDecision = 3, kLcViol = 4, kLcRedo = 5,
    kLcStep = 6, kLcExact = 7, kLcBound = 8, kLcStallTest = 10, kLcWaitUs = 11, kLcWords = 12
};
struct ListArgs {
    const float4* pos; const float4* vel; const int* ids;  // state of the step
    const int2* table;                                     // fresh only at a build
    float4* pos_out; float4* vel_out; int* ids_out; float4* acc_out;
    const float4* hist_in; const int* hcnt_in;
    float4* hist_out; int* hcnt_out;
    unsigned long long* counters;
    const int* nbr; const int* nbr_cnt; const float4* xbuild;
    uint32_t* list_ctrl;
    const DevParams* scene_params; const int* scene; int* scene_out;
    // backward Euler / Picard: the step-start state, the iteration's residual slot,
    // the iteration counter, the list-validity bound on the iterate, the convergence skip
    const float4* xn; const float4* vn;
    uint32_t* res_slot; int* picard_used; int iter;
    float viol_thr;
    Skip skip;
    float4* rhs_vel; int* rhs_ids;    // the iterate's velocity and ids, for the rhs getter
    // semi-implicit Euler: the build decision for the next step, made by the kernel's
    // last block (threshold on max |x - x_build|, block ticket, the build's IF node)
    float thr; unsigned* tail_count; int use_cond; cudaGraphConditionalHandle cond;
};
// Device-side launches of the list build's graphs (wd_launch.cu, the one translation
// unit built with relocatable device code for the device runtime): one thread
// tail-launches `graph` when *flag is nonzero (the step's build decision), or `on_zero`
// / `on_one` by *flag (the search's path). The launched graph runs once the graph that
// holds the launching kernel has completed; later work of the stream waits for it. A
// failed launch counts in counters[kCntLaunchFail].
void launch_graph_if(const uint32_t* flag, cudaGraphExec_t graph, unsigned long long* counters,
                     cudaStream_t st);
void launch_graph_pick(const int* flag, cudaGraphExec_t on_zero, cudaGraphExec_t on_one,
                       unsigned long long* counters, cudaStream_t st);
void launch_list_decide(uint32_t* list_ctrl, float thr, bool always_exact,
                        unsigned long long* counters,
                        bool use_cond, cudaGraphConditionalHandle cond, cudaStream_t st);
// The sorted state a list build copies back into the step's buffers (one pass with the
// listing: pos is read there anyway).
struct ListCopy {
    const float4* vel; const int* ids; const int* hcnt; const int* scene;
    float4* pos_out; float4* vel_out; int* ids_out; int* hcnt_out; int* scene_out;
};
// tiled: a single scene's build with each block's neighbour window staged in shared
// memory (k_list_build_tiled); otherwise one thread per slot reading global memory.
void launch_list_build(const DevParams& P, SceneTab T, const float4* pos, const int2* table,
                       int* nbr, int* nbr_cnt, float4* xbuild, uint32_t* list_ctrl,
                       const ListCopy& cp, Skip skip, unsigned long long* counters, bool tiled,
                       cudaStream_t st);
void launch_list_copy(int n, const float4* pos, const float4* vel, const int* ids,
                      const int* hcnt, const int* scene, float4* pos_out, float4* vel_out,
                      int* ids_out, int* hcnt_out, int* scene_out, Skip skip, cudaStream_t st);
// min_blocks: the kernel variant. 5 / 4: per-lane kernel with 48 / 64 registers per
// thread; 0: warp-cooperative; 1 / 2: bulk-staged persistent (kBlock threads) with 48
// / 64 registers. Picard runs the per-lane kernel (4 or 5).
void launch_force_list(const DevParams& P, const ListArgs& a, cudaStream_t st,
                       int block = kBlock, int min_blocks = 5, bool picard = false);
// Picard with lists: the last iterate into the B buffers when the last executed
// iteration wrote the scratch ones; then the redo decision.
void launch_list_finalize(int n, const int* picard_used, const float4* xpos,
                          const float4* xvel, float4* pos, float4* vel, cudaStream_t st);
void launch_list_picard_check(uint32_t* list_ctrl, unsigned long long* counters, bool use_cond,
                              cudaGraphConditionalHandle cond, cudaStream_t st);
void launch_list_length(int n, const int* nbr_cnt, unsigned long long* out, cudaStream_t st);

// Total energy per scene at the sorted state (after a search): per-grain FP64 sums,
// then fixed-order per-segment reductions into out[scene]. hcnt is in state-slot
// order; src maps each sorted position to its state slot.
void launch_energy(const DevParams& P, SceneTab T, const float4* pos, const float4* vel,
                   const int* ids, const int2* table, const float4* hist, const int* hcnt,
                   const int* src, const Segments& g, double* per_grain, double* partials,
                   double* out, cudaStream_t st);

// Candidate probes (CSR by grain id).
void launch_candidate_count(const DevParams& P, SceneTab T, const float4* pos, const int* ids,
                            const int2* table, int* count_by_id, cudaStream_t st);
void launch_candidate_fill(const DevParams& P, SceneTab T, const float4* pos, const int* ids,
                           const int2* table, const int64_t* offsets_by_id, int* cand,
                           uint8_t* contact, cudaStream_t st);

// State conversion between the sorted SoA and the caller's AoS-by-id layouts.
void launch_state_to_aos(int n, const float4* pos, const float4* vel, const int* ids,
                         float* out6, cudaStream_t st);
void launch_positions_to_aos(int n, const float4* pos, const int* ids, float* out3,
                             cudaStream_t st);
void launch_rhs_to_aos(int n, const float4* vel_used, const float4* acc, const int* ids,
                       float* out6, cudaStream_t st);
void launch_state_from_aos(int n, const float* in6, float4* pos, float4* vel, const int* ids,
                           cudaStream_t st);
void launch_cell_keys_by_id(const DevParams& P, SceneTab T, const float4* pos, const int* ids,
                            int32_t* keys, cudaStream_t st);

// CIC deposit: deterministic fixed-point accumulation (see wd_fields.cu).
void launch_deposit(int n, const float4* pos, const float4* vel, const float* lo,
                    const float* hi, const int* dgrid, uint32_t* bounds,
                    unsigned long long* acc, float* out, cudaStream_t st);
// One field per scene, scene after scene; bounds holds 4 words per scene.
void launch_deposit_batch(int n, const float4* pos, const float4* vel, SceneTab T, int scenes,
                          int64_t total_nodes, uint32_t* bounds, unsigned long long* acc,
                          float* out, cudaStream_t st);

// Reductions (per scene: out3[3 * scene + axis]).
void launch_segment_sums(const double* values, int n, int comps, const Segments& g,
                         double* partials, double* out, cudaStream_t st);
void launch_momentum(int n, const float4* vel, const Segments& g, double* per_grain,
                     double* partials, double* out3, cudaStream_t st);
void launch_max_accel(int n, const float4* acc, unsigned long long* counters,
                      cudaStream_t st);
// is_stable: sets counters[kCntUnstable]; a batch also flags scene_unstable[scene].
void launch_stability(const DevParams& P, SceneTab T, const float4* pos,
                      unsigned long long* counters, int* scene_unstable, cudaStream_t st);

int reduction_blocks(int n);

// Reverse pass (wd_adjoint.cu). Adjoint arrays are float4 (x, y, z, unused) by grain
// id; spring rows are kHistCap entries per grain id.
struct AdjArgs {
    const float4* pos; const float4* vel; const int* ids;  // sorted state of step t
    const int2* table;
    const float4* hist_in; const int* hcnt_in;     // springs at t (counts by sorted slot)
    const float4* hist_next; const int* hcnt_next; // springs at t+1 (counts by id)
    const int* clist; const int* ccnt;             // pair contacts per slot (kAdjContacts)
    const float4* lx; const float4* lvt; const float4* lf; const float4* lxi;
    float4* lx_out; float4* lv_out; float4* lxi_out;
    double* theta;                                  // [3][n], accumulated
    int kt_from_kn;
};
constexpr int kAdjContacts = 32;  // pair contacts per grain the reverse pass records
void launch_contact_record(const DevParams& P, const float4* pos, const int2* table, int* clist,
                           int* ccnt, unsigned long long* overflow, cudaStream_t st);
void launch_adj_prep(int n, float dt, const float4* vel, const int* ids, const float4* lx,
                     const float4* lv, float4* lvt, float4* lf, cudaStream_t st);
void launch_adj_step(const DevParams& P, const AdjArgs& a, cudaStream_t st);
void launch_counts_by_id(int n, const int* ids, const int* cnt_slot, int* cnt_id,
                         cudaStream_t st);
// AoS3 floats by grain id <-> float4 by grain id (a == nullptr: zeros).
void launch_aos3_to_f4(int n, const float* a, float4* o, cudaStream_t st);
void launch_f4_to_aos3(int n, const float4* a, float* o, cudaStream_t st);
void launch_deposit_vjp(int n, const float4* pos, const float4* vel, const int* ids,
                        const float* lo, const float* hi, const int* size, const float* g,
                        float4* gx, float4* gv, cudaStream_t st);

// Ensemble metrics (wd_ensemble.cu): per scene, the sum over grains of the squared
// separation from the reference scene's grain with the same index (grain_sums), and
// the six node sums sum (rho - rho_ref)^2, sum rho_ref^2, sum rho, sum rho*ix,
// sum rho*iy, sum rho*iz of the mass channel (node_sums[6 * scene + c]).
void launch_chaos(int n, const float* pos3, const Segments& grains, double* grain_vals,
                  double* grain_partials, double* grain_sums, int total_nodes, const float* grid,
                  const Segments& nodes, int ref, int ny, int nz, double* node_vals,
                  double* node_partials, double* node_sums, cudaStream_t st);

}  // namespace wd
