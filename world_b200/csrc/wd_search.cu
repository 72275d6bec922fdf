// wd_search.cu -- neighbor search for sm_100a: cell keys, ordering by (cell key,
// grain id), run table, gather into sorted SoA.
//
// Replaces the reference's four-pass dense bucketing (src/find_neighbors_kernel.cu:
// 46-161: atomicCAS marks, atomicAdd compaction, atomicAdd slot fill, flat candidate
// rows of 27*particles_per_cell ints). Here:
//   * the key of every grain is the reference's cell mapping; grains are ordered by
//     (key, grain id): deterministic, no per-cell capacity, nothing dropped;
//   * between steps few grains change cell, so the search re-sorts only those
//     ("movers": a bitonic sort on one 8-CTA cluster over distributed shared memory)
//     and merges them into the still-sorted rest
//     by binary search; the first search, or one with more than kMoverCap movers,
//     runs a stable LSD radix sort of all keys instead. The choice is made on the
//     device, so both paths sit in the same CUDA graph and the idle one returns at
//     once. Both produce the same order;
//   * the run table is a dense [start, end) per cell, but only the cells of the
//     previous search are cleared (O(n), not the reference's O(cells) memset);
//   * no candidate list is materialised: the contact kernel walks the sorted runs.
#include <cstdio>

#include <cooperative_groups.h>

#include "wd_kernels.h"

namespace wd {

namespace {

__device__ __forceinline__ bool skipped(const Skip& s) {
    return s.prev_res != nullptr && s.tol > 0.f && __uint_as_float(*s.prev_res) < s.tol;
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Movers among slots [0, q): block prefix plus the bits of the words before q.
__device__ __forceinline__ int movers_before(const uint32_t* __restrict__ bits,
                                             const int* __restrict__ blk_off, int q) {
    const int b = q / kBlock;
    int c = blk_off[b];
    const int w0 = b * (kBlock / 32), wq = q >> 5;
    for (int w = w0; w < wq; ++w) c += __popc(bits[w]);
    const int r = q & 31;
    if (r) c += __popc(bits[wq] & ((1u << r) - 1u));
    return c;
}

// Search pass 1: key of every state slot, mover bits and per-block mover counts;
// clear the runs of the previous search; zero the radix digit totals.
template <bool BATCH>
__global__ void __launch_bounds__(kBlock)
k_keys(DevParams P, SceneTab T, const float4* __restrict__ pos, uint32_t* __restrict__ newkey,
       uint32_t* __restrict__ moved, int* __restrict__ blk_cnt, int num_blocks,
       const uint32_t* __restrict__ slot_keys, const uint32_t* __restrict__ table_keys,
       int2* __restrict__ table, uint32_t* __restrict__ digit_totals, int totals_count,
       uint32_t* __restrict__ zero_res, int zero_res_count, Skip skip) {
    if (skipped(skip)) return;
    __shared__ int warp_movers[kBlock / 32];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < totals_count) digit_totals[s] = 0u;
    if (zero_res != nullptr && s < zero_res_count) zero_res[s] = 0u;
    bool mv = false;
    if (s < P.n) {
        const DevParams& Q = scene_params<BATCH>(P, T, s);
        const float4 p = pos[s];
        int cx, cy, cz;
        cell_coords(Q, p.x, p.y, p.z, cx, cy, cz);
        const uint32_t key = Q.cell_base + flat_cell(Q, cx, cy, cz);
        newkey[s] = key;
        mv = key != slot_keys[s];
        const uint32_t kp = table_keys[s];
        if (kp != kNoKey && (s == 0 || table_keys[s - 1] != kp)) table[kp] = make_int2(-1, -1);
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, mv);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        if (s < P.n) moved[s >> 5] = ballot;
        warp_movers[warp] = __popc(ballot);
    }
    __syncthreads();
    if (threadIdx.x == 0 && blockIdx.x < num_blocks) {
        int c = 0;
#pragma unroll
        for (int w = 0; w < kBlock / 32; ++w) c += warp_movers[w];
        blk_cnt[blockIdx.x] = c;
    }
}

// Block-wide exclusive scan of one value per thread (THREADS threads).
template <int THREADS>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < THREADS / 32 ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < THREADS / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    const uint32_t before = (warp > 0 ? warp_sums[warp - 1] : 0u) + x - v;
    if (total) *total = warp_sums[THREADS / 32 - 1];
    __syncthreads();
    return before;
}

__device__ __forceinline__ bool radix_idle(const int* ctrl) { return ctrl != nullptr && ctrl[1] == 0; }
__device__ __forceinline__ bool mover_idle(const int* ctrl) { return ctrl[1] != 0; }

// Radix path: key and slot of every grain by id, so the sort input is in id order
// and a stable sort yields (key, id) order.
__global__ void __launch_bounds__(kBlock)
k_by_id(int n, const int* __restrict__ ids, const uint32_t* __restrict__ newkey,
        uint32_t* __restrict__ key_by_id, int* __restrict__ slot_of_id,
        const int* __restrict__ ctrl, Skip skip) {
    if (skipped(skip) || radix_idle(ctrl)) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int i = ids[s];
    key_by_id[i] = newkey[s];
    slot_of_id[i] = s;
}

// Radix pass, step 1: digit histogram of one tile (warp-aggregated shared atomics:
// nearly sorted input puts most keys of a tile on one digit).
__global__ void __launch_bounds__(kBlock)
k_sort_hist(const uint32_t* __restrict__ keys, int n, int shift, int num_tiles,
            uint32_t* __restrict__ counts, uint32_t* __restrict__ totals,
            const int* __restrict__ ctrl, Skip skip) {
    if (skipped(skip) || radix_idle(ctrl)) return;
    __shared__ uint32_t h[kRadix];
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) h[d] = 0u;
    __syncthreads();
    const int base = blockIdx.x * kSortTile;
    const unsigned lane_lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int idx = base + k * kBlock + threadIdx.x;
        const bool valid = idx < n;
        const uint32_t d = valid ? (keys[idx] >> shift) & (kRadix - 1) : kRadix;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (valid && (peers & lane_lt) == 0u) atomicAdd(&h[d], static_cast<uint32_t>(__popc(peers)));
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
        const uint32_t c = h[d];
        counts[static_cast<size_t>(d) * num_tiles + blockIdx.x] = c;
        if (c) atomicAdd(&totals[d], c);
    }
}

// Radix pass, step 2: one block per digit turns that digit's per-tile counts into
// global output offsets (digit base + exclusive scan over tiles).
__global__ void __launch_bounds__(kBlock)
k_sort_scan(uint32_t* __restrict__ counts, const uint32_t* __restrict__ totals, int num_tiles,
            const int* __restrict__ ctrl, Skip skip) {
    if (skipped(skip) || radix_idle(ctrl)) return;
    const int d = blockIdx.x;
    uint32_t part = 0u;
    for (int t = threadIdx.x; t < d; t += blockDim.x) part += totals[t];
    uint32_t base = 0u;
    block_exclusive_scan<kBlock>(part, &base);
    uint32_t* col = counts + static_cast<size_t>(d) * num_tiles;
    const int chunk = (num_tiles + kBlock - 1) / kBlock;
    const int t0 = threadIdx.x * chunk;
    uint32_t sum = 0u;
    for (int t = t0; t < min(t0 + chunk, num_tiles); ++t) sum += col[t];
    uint32_t run = base + block_exclusive_scan<kBlock>(sum, nullptr);
    for (int t = t0; t < min(t0 + chunk, num_tiles); ++t) {
        const uint32_t c = col[t];
        col[t] = run;
        run += c;
    }
}

// Radix pass, step 3: stable scatter. Each warp ranks its 256 consecutive keys in 8
// rounds of 32 with __match_any_sync; warps are then offset by the per-digit counts
// of the warps before them, and the tile by its scanned global offset.
template <bool IOTA>
__global__ void __launch_bounds__(kBlock)
k_sort_scatter(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
               uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, int n,
               int shift, int num_tiles, const uint32_t* __restrict__ offsets,
               const int* __restrict__ ctrl, Skip skip) {
    if (skipped(skip) || radix_idle(ctrl)) return;
    constexpr int kWarps = kBlock / 32;
    __shared__ uint32_t wh[kWarps][kRadix];
    __shared__ uint32_t toff[kRadix];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
        toff[d] = offsets[static_cast<size_t>(d) * num_tiles + blockIdx.x];
#pragma unroll
        for (int w = 0; w < kWarps; ++w) wh[w][d] = 0u;
    }
    __syncthreads();
    const unsigned lane_lt = lanemask_lt();
    const int base = blockIdx.x * kSortTile + warp * (32 * kSortItems);
    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int idx = base + r * 32 + lane;
        const bool valid = idx < n;
        key[r] = valid ? keys_in[idx] : 0u;
        val[r] = valid ? (IOTA ? static_cast<uint32_t>(idx) : vals_in[idx]) : 0u;
        const uint32_t d = valid ? (key[r] >> shift) & (kRadix - 1) : kRadix;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned lt = peers & lane_lt;
        const uint32_t before = valid ? wh[warp][d] : 0u;
        __syncwarp();
        if (valid && lt == 0u) wh[warp][d] = before + static_cast<uint32_t>(__popc(peers));
        __syncwarp();
        rank[r] = before + static_cast<uint32_t>(__popc(lt));
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
        uint32_t run = 0u;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = wh[w][d];
            wh[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int idx = base + r * 32 + lane;
        if (idx < n) {
            const uint32_t d = (key[r] >> shift) & (kRadix - 1);
            const uint32_t dst = toff[d] + wh[warp][d] + rank[r];
            keys_out[dst] = key[r];
            vals_out[dst] = val[r];
        }
    }
}

// Search pass 2, one thread-block cluster of kMoverCtas CTAs (one CTA per SM, the
// cluster's shared memories together holding kMoverCap movers, one per thread): mover
// offsets per 256-slot block, the mover count and the path. When the movers fit
// kMoverCap they are compacted from the bit mask (only blocks that have movers are
// read) into the distributed shared memory and sorted by (key << 32 | id) with a
// bitonic network whose stages across CTAs use remote shared-memory accesses (DSMEM)
// and a cluster barrier, the others a CTA barrier; otherwise ctrl[1] selects the radix
// sort, and when the search runs inside a CUDA graph the radix path's conditional node
// is switched on. (A single CTA did the same network on one SM, issue-bound at about
// 100 us for 8192 movers.)
constexpr int kMoverCtas = 8;
constexpr int kMoverPer = kMoverCap / kMoverCtas;  // elements per CTA: one per thread
static_assert(kMoverPer == kMoverThreads, "one mover element per thread");

__global__ void __cluster_dims__(kMoverCtas, 1, 1) __launch_bounds__(kMoverThreads)
k_movers(int n, const int* __restrict__ blk_cnt, int* __restrict__ blk_off, int num_blocks,
         const uint32_t* __restrict__ moved, const uint32_t* __restrict__ newkey,
         const int* __restrict__ ids, unsigned long long* __restrict__ mv_key,
         uint32_t* __restrict__ mv_slot, int* __restrict__ ctrl, int use_cond,
         cudaGraphConditionalHandle cond, unsigned long long* __restrict__ counters, Skip skip) {
    namespace cg = cooperative_groups;
    if (skipped(skip)) return;  // the same flag for every CTA of the cluster
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = static_cast<int>(cluster.block_rank());
    __shared__ unsigned long long k[kMoverPer];
    __shared__ uint32_t v[kMoverPer];
    __shared__ uint32_t cta_total;
    __shared__ uint32_t s_off, s_m;
    const int tid = static_cast<int>(threadIdx.x);
    const int g = rank * kMoverPer + tid;  // the cluster-wide thread, owner of element g
    const int gthreads = kMoverCtas * kMoverThreads;
    const int chunk = (num_blocks + gthreads - 1) / gthreads;
    const int b0 = min(g * chunk, num_blocks);
    const int b1 = min(b0 + chunk, num_blocks);
    uint32_t sum = 0u;
    for (int b = b0; b < b1; ++b) sum += static_cast<uint32_t>(blk_cnt[b]);
    uint32_t total = 0u;
    const uint32_t first_local = block_exclusive_scan<kMoverThreads>(sum, &total);
    if (tid == 0) cta_total = total;
    cluster.sync();  // every CTA's total visible
    if (tid == 0) {
        uint32_t off = 0u, m = 0u;
        for (int r = 0; r < kMoverCtas; ++r) {
            const uint32_t t = *cluster.map_shared_rank(&cta_total, r);
            if (r < rank) off += t;
            m += t;
        }
        s_off = off;
        s_m = m;
    }
    cluster.sync();  // remote reads done before any CTA may leave
    const uint32_t total_all = s_m;
    uint32_t run = s_off + first_local;
    for (int b = b0; b < b1; ++b) {
        blk_off[b] = static_cast<int>(run);
        run += static_cast<uint32_t>(blk_cnt[b]);
    }
    const int m = static_cast<int>(total_all);
    const int full = total_all > static_cast<uint32_t>(kMoverCap) ? 1 : 0;
    if (rank == 0 && tid == 0) {
        blk_off[num_blocks] = m;
        ctrl[0] = m;
        ctrl[1] = full;
        if (use_cond) cudaGraphSetConditional(cond, static_cast<unsigned>(full));
        if (full) atomicAdd(&counters[kCntRadixSearches], 1ull);
    }
    if (full || m == 0) return;  // the same decision in every CTA
    // compaction in slot order, each mover stored in the CTA that owns its position
    run = s_off + first_local;
    for (int b = b0; b < b1; ++b) {
        if (blk_cnt[b] == 0) continue;
        const int w0 = b * (kBlock / 32);
        for (int w = w0; w < w0 + kBlock / 32 && 32 * w < n; ++w) {
            uint32_t bits = moved[w];
            while (bits) {
                const int lane = __ffs(bits) - 1;
                bits &= bits - 1u;
                const int slot = 32 * w + lane;
                const int owner = static_cast<int>(run) / kMoverPer;
                const int at = static_cast<int>(run) % kMoverPer;
                *cluster.map_shared_rank(&k[at], owner) =
                    (static_cast<unsigned long long>(newkey[slot]) << 32) |
                    static_cast<uint32_t>(ids[slot]);
                *cluster.map_shared_rank(&v[at], owner) = static_cast<uint32_t>(slot);
                ++run;
            }
        }
    }
    int p = 1;
    while (p < m) p <<= 1;
    if (g >= m && g < p) {
        k[tid] = ~0ull;
        v[tid] = 0u;
    }
    cluster.sync();  // the compacted movers and the padding visible everywhere
    for (int size = 2; size <= p; size <<= 1) {
        int stride = size >> 1;
        for (; stride >= 32; stride >>= 1) {
            const int j = g ^ stride;
            if (g < p && j > g) {
                const bool up = (g & size) == 0;
                unsigned long long* kj = cluster.map_shared_rank(&k[j % kMoverPer], j / kMoverPer);
                uint32_t* vj = cluster.map_shared_rank(&v[j % kMoverPer], j / kMoverPer);
                const unsigned long long a = k[tid], c = *kj;
                if ((a > c) == up) {
                    k[tid] = c;
                    *kj = a;
                    const uint32_t t = v[tid];
                    v[tid] = *vj;
                    *vj = t;
                }
            }
            // a stage that crosses CTAs, or precedes one, ends at a cluster barrier
            const bool cross = stride >= kMoverPer;
            const bool next_cross = (stride >> 1) >= kMoverPer;
            if (cross || next_cross) cluster.sync();
            else __syncthreads();
        }
        // strides below 32 pair lanes of one warp: exchanged through shuffles, no barrier
        // (an element at or above p is padding that sorts last; its lane still shuffles)
        unsigned long long a = k[tid];
        uint32_t av = v[tid];
        const bool up = (g & size) == 0;
        for (; stride > 0; stride >>= 1) {
            const unsigned long long c = __shfl_xor_sync(0xffffffffu, a, stride);
            const uint32_t cv = __shfl_xor_sync(0xffffffffu, av, stride);
            const bool lower = (g & stride) == 0;  // this lane holds the lower index
            // ascending: the lower index keeps the smaller key; descending: the larger
            const bool take = lower == up ? c < a : c > a;
            if (take && g < p) {
                a = c;
                av = cv;
            }
        }
        k[tid] = a;
        v[tid] = av;
        // the next size starts with a stride >= 32 (or none): across warps, maybe CTAs
        if ((size << 1) <= p && size >= kMoverPer) cluster.sync();
        else __syncthreads();
    }
    if (g < m) {
        mv_key[g] = k[tid];
        mv_slot[g] = v[tid];
    }
}

// Mover path, merge: final position of every grain. A stayer keeps its rank among
// stayers and moves up by the movers sorted below it; a mover's position is its rank
// among movers plus the stayers below it (a binary search over the previous order,
// which is sorted by (key, id), minus the movers in that prefix).
__global__ void __launch_bounds__(kBlock)
k_merge(int n, const uint32_t* __restrict__ newkey, const uint32_t* __restrict__ slot_keys,
        const int* __restrict__ ids, const uint32_t* __restrict__ moved,
        const int* __restrict__ blk_off, const unsigned long long* __restrict__ mv_key,
        const uint32_t* __restrict__ mv_slot, uint32_t* __restrict__ skey,
        uint32_t* __restrict__ sid, int* __restrict__ src, const int* __restrict__ ctrl,
        Skip skip) {
    if (skipped(skip) || mover_idle(ctrl)) return;
    const int m = ctrl[0];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n && !((moved[t >> 5] >> (t & 31)) & 1u)) {
        const uint32_t key = newkey[t];
        const uint32_t id = static_cast<uint32_t>(ids[t]);
        const unsigned long long x = (static_cast<unsigned long long>(key) << 32) | id;
        int lo = 0, hi = m;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (mv_key[mid] < x) lo = mid + 1; else hi = mid;
        }
        const int pos = t - movers_before(moved, blk_off, t) + lo;
        skey[pos] = key;
        sid[pos] = id;
        src[pos] = t;
    }
    if (t < m) {
        const unsigned long long x = mv_key[t];
        int lo = 0, hi = n;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const unsigned long long y =
                (static_cast<unsigned long long>(slot_keys[mid]) << 32) | static_cast<uint32_t>(ids[mid]);
            if (y < x) lo = mid + 1; else hi = mid;
        }
        const int pos = t + lo - movers_before(moved, blk_off, lo);
        skey[pos] = static_cast<uint32_t>(x >> 32);
        sid[pos] = static_cast<uint32_t>(x & 0xffffffffu);
        src[pos] = static_cast<int>(mv_slot[t]);
    }
}

// Gather into sorted order, fused with the run table: each position copies its grain
// from its source state slot (the radix path resolves the slot from the grain id),
// the first and last position of every run write the cell's [start, end), step
// searches record the new slot keys, and a run longer than particles_per_cell (its
// first key equals the key ppc positions later) is counted as an overflow.
template <bool SNAP, bool SNAP_FROM_STATE>
__global__ void __launch_bounds__(kBlock)
k_gather(int n, int ppc, const uint32_t* __restrict__ skey, const uint32_t* __restrict__ sid,
         const int* __restrict__ src, const int* __restrict__ slot_of_id,
         const int* __restrict__ ctrl, const float4* __restrict__ posA,
         const float4* __restrict__ velA, float4* __restrict__ posB, float4* __restrict__ velB,
         int* __restrict__ idsB, const float4* __restrict__ nposA,
         const float4* __restrict__ nvelA, float4* __restrict__ nposB,
         float4* __restrict__ nvelB, const int* __restrict__ cnt_src, int* __restrict__ cnt_dst,
         const int* __restrict__ scene_src, int* __restrict__ scene_dst,
         int2* __restrict__ table, uint32_t* __restrict__ table_keys,
         uint32_t* __restrict__ slot_keys, unsigned long long* __restrict__ counters,
         unsigned long long* __restrict__ scene_overflow,
         const DevParams* __restrict__ scene_params, Skip skip) {
    if (skipped(skip)) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t id = sid[s];
    const int p = ctrl[1] ? slot_of_id[id] : src[s];
    const float4 x = posA[p], v = velA[p];
    posB[s] = x;
    velB[s] = v;
    idsB[s] = static_cast<int>(id);
    if (SNAP) {
        if (SNAP_FROM_STATE) {
            nposB[s] = x;
            nvelB[s] = v;
        } else {
            nposB[s] = nposA[p];
            nvelB[s] = nvelA[p];
        }
    }
    if (cnt_dst) cnt_dst[s] = cnt_src[p];
    if (scene_dst) scene_dst[s] = scene_src[p];
    const uint32_t k = skey[s];
    table_keys[s] = k;
    if (slot_keys) slot_keys[s] = k;
    int* e = reinterpret_cast<int*>(&table[k]);
    if (s == 0 || skey[s - 1] != k) {
        e[0] = s;
        // a run holds one scene's grains: its own particles_per_cell applies
        const int cap = scene_params ? scene_params[scene_src[p]].ppc : ppc;
        if (s + cap < n && skey[s + cap] == k) {
            atomicAdd(&counters[kCntGridOverflow], 1ull);
            if (scene_overflow) atomicAdd(&scene_overflow[scene_src[p]], 1ull);
        }
    }
    if (s == n - 1 || skey[s + 1] != k) e[1] = s + 1;
}

// Candidate probes: the same traversal as the contact kernel.
template <bool BATCH>
__global__ void __launch_bounds__(kBlock)
k_cand_count(DevParams P0, SceneTab T, const float4* __restrict__ pos, const int* __restrict__ ids,
             const int2* __restrict__ table, int* __restrict__ count_by_id) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P0.n) return;
    const DevParams& P = scene_params<BATCH>(P0, T, s);
    const float4 pi = pos[s];
    int cx, cy, cz;
    cell_coords(P, pi.x, pi.y, pi.z, cx, cy, cz);
    int c = 0;
    for (int dx = -1; dx <= 1; ++dx) {
        const int nx = cx + dx;
        if (nx < 0 || nx >= P.grid[0]) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int ny = cy + dy;
            if (ny < 0 || ny >= P.grid[1]) continue;
            int lo, hi;
            column_range(P, table, nx, ny, cz, lo, hi);
            if (hi > lo) c += hi - lo - ((s >= lo && s < hi) ? 1 : 0);
        }
    }
    count_by_id[ids[s]] = c;
}

template <bool BATCH>
__global__ void __launch_bounds__(kBlock)
k_cand_fill(DevParams P0, SceneTab T, const float4* __restrict__ pos, const int* __restrict__ ids,
            const int2* __restrict__ table, const int64_t* __restrict__ offsets,
            int* __restrict__ cand, uint8_t* __restrict__ contact) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P0.n) return;
    const DevParams& P = scene_params<BATCH>(P0, T, s);
    const float4 pi = pos[s];
    int cx, cy, cz;
    cell_coords(P, pi.x, pi.y, pi.z, cx, cy, cz);
    int64_t k = offsets[ids[s]];
    for (int dx = -1; dx <= 1; ++dx) {
        const int nx = cx + dx;
        if (nx < 0 || nx >= P.grid[0]) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int ny = cy + dy;
            if (ny < 0 || ny >= P.grid[1]) continue;
            int lo, hi;
            column_range(P, table, nx, ny, cz, lo, hi);
            for (int j = lo; j < hi; ++j) {
                if (j == s) continue;
                const float4 pj = pos[j];
                float3 d;
                const float ns = pair_norm_sq(pi, pj, d);
                const float dist = pair_dist(sqrtf(ns), pi.w, pj.w);
                cand[k] = ids[j];
                contact[k] = dist < 0.f ? 1 : 0;
                ++k;
            }
        }
    }
}

__global__ void k_state_to_aos(int n, const float4* __restrict__ pos,
                               const float4* __restrict__ vel, const int* __restrict__ ids,
                               float* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 x = pos[s], v = vel[s];
    float* o = out + 6 * static_cast<int64_t>(ids[s]);
    o[0] = x.x; o[1] = x.y; o[2] = x.z; o[3] = v.x; o[4] = v.y; o[5] = v.z;
}

__global__ void k_positions_to_aos(int n, const float4* __restrict__ pos,
                                   const int* __restrict__ ids, float* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 x = pos[s];
    float* o = out + 3 * static_cast<int64_t>(ids[s]);
    o[0] = x.x; o[1] = x.y; o[2] = x.z;
}

__global__ void k_rhs_to_aos(int n, const float4* __restrict__ vel,
                             const float4* __restrict__ acc, const int* __restrict__ ids,
                             float* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 v = vel[s], a = acc[s];
    float* o = out + 6 * static_cast<int64_t>(ids[s]);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = a.x; o[4] = a.y; o[5] = a.z;
}

__global__ void k_state_from_aos(int n, const float* __restrict__ in, float4* __restrict__ pos,
                                 float4* __restrict__ vel, const int* __restrict__ ids) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float* q = in + 6 * static_cast<int64_t>(ids[s]);
    pos[s] = make_float4(q[0], q[1], q[2], pos[s].w);
    vel[s] = make_float4(q[3], q[4], q[5], vel[s].w);
}

// Cell key of every grain within its own scene's grid, by grain id.
template <bool BATCH>
__global__ void k_cell_keys_by_id(DevParams P0, SceneTab T, const float4* __restrict__ pos,
                                  const int* __restrict__ ids, int32_t* __restrict__ keys) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P0.n) return;
    const DevParams& P = scene_params<BATCH>(P0, T, s);
    const float4 p = pos[s];
    int cx, cy, cz;
    cell_coords(P, p.x, p.y, p.z, cx, cy, cz);
    keys[ids[s]] = static_cast<int32_t>(flat_cell(P, cx, cy, cz));
}

}  // namespace

void launch_search_head(const DevParams& P, SceneTab T, const float4* pos, const int* ids,
                        SearchBuffers& sb, Skip skip, uint32_t* zero_res, int zero_res_count,
                        bool use_cond, cudaGraphConditionalHandle cond,
                        unsigned long long* counters, cudaStream_t st) {
    const int n = P.n;
    const int totals = kRadix * sb.passes;
    const int kb = blocks_for(n > totals ? n : totals);
    if (T.params) {
        k_keys<true><<<kb, kBlock, 0, st>>>(P, T, pos, sb.newkey, sb.moved, sb.blk_cnt,
                                            sb.num_blocks, sb.slot_keys, sb.table_keys, sb.table,
                                            sb.digit_totals, totals, zero_res, zero_res_count, skip);
    } else {
        k_keys<false><<<kb, kBlock, 0, st>>>(P, T, pos, sb.newkey, sb.moved, sb.blk_cnt,
                                             sb.num_blocks, sb.slot_keys, sb.table_keys, sb.table,
                                             sb.digit_totals, totals, zero_res, zero_res_count, skip);
    }
    k_movers<<<kMoverCtas, kMoverThreads, 0, st>>>(n, sb.blk_cnt, sb.blk_off, sb.num_blocks,
                                                       sb.moved, sb.newkey, ids, sb.mv_key,
                                                       sb.mv_slot, sb.ctrl, use_cond ? 1 : 0,
                                                       cond, counters, skip);
}

void launch_search_radix(const DevParams& P, const int* ids, SearchBuffers& sb, Skip skip,
                         cudaStream_t st) {
    const int n = P.n;
    k_by_id<<<blocks_for(n), kBlock, 0, st>>>(n, ids, sb.newkey, sb.key_by_id, sb.slot_of_id,
                                              sb.ctrl, skip);
    int cur = 0;
    const uint32_t* kin = sb.key_by_id;
    const uint32_t* vin = nullptr;
    for (int pass = 0; pass < sb.passes; ++pass) {
        const int shift = pass * kRadixBits;
        uint32_t* totals_p = sb.digit_totals + kRadix * pass;
        k_sort_hist<<<sb.num_tiles, kBlock, 0, st>>>(kin, n, shift, sb.num_tiles, sb.tile_counts,
                                                     totals_p, sb.ctrl, skip);
        k_sort_scan<<<kRadix, kBlock, 0, st>>>(sb.tile_counts, totals_p, sb.num_tiles, sb.ctrl, skip);
        if (pass == 0) {
            k_sort_scatter<true><<<sb.num_tiles, kBlock, 0, st>>>(
                kin, vin, sb.keys[cur], sb.vals[cur], n, shift, sb.num_tiles, sb.tile_counts,
                sb.ctrl, skip);
        } else {
            k_sort_scatter<false><<<sb.num_tiles, kBlock, 0, st>>>(
                kin, vin, sb.keys[cur], sb.vals[cur], n, shift, sb.num_tiles, sb.tile_counts,
                sb.ctrl, skip);
        }
        kin = sb.keys[cur];
        vin = sb.vals[cur];
        cur ^= 1;
    }
}

void launch_search_merge(const DevParams& P, const int* ids, SearchBuffers& sb, Skip skip,
                         cudaStream_t st) {
    const int n = P.n;
    k_merge<<<blocks_for(n), kBlock, 0, st>>>(n, sb.newkey, sb.slot_keys, ids, sb.moved, sb.blk_off,
                                              sb.mv_key, sb.mv_slot, sb.keys[sb.out],
                                              sb.vals[sb.out], sb.src, sb.ctrl, skip);
}

void launch_search(const DevParams& P, SceneTab T, const float4* pos, const int* ids,
                   SearchBuffers& sb, Skip skip, uint32_t* zero_res, int zero_res_count,
                   unsigned long long* counters, cudaStream_t st) {
    launch_search_head(P, T, pos, ids, sb, skip, zero_res, zero_res_count, false, 0, counters, st);
    launch_search_radix(P, ids, sb, skip, st);
    launch_search_merge(P, ids, sb, skip, st);
}

cudaError_t search_prepare() { return cudaSuccess; }

int radix_output(int passes) { return (passes - 1) & 1; }

void launch_gather(const DevParams& P, SearchBuffers& sb, const float4* posA,
                   const float4* velA, float4* posB, float4* velB, int* idsB,
                   const float4* nposA, const float4* nvelA, float4* nposB, float4* nvelB,
                   bool snap_from_state, const int* cnt_src, int* cnt_dst, const int* scene_src,
                   int* scene_dst, bool step_search, unsigned long long* counters,
                   unsigned long long* scene_overflow, const DevParams* scene_params, Skip skip,
                   cudaStream_t st) {
    const int nb = blocks_for(P.n);
    const uint32_t* skey = sb.keys[sb.out];
    const uint32_t* sid = sb.vals[sb.out];
    uint32_t* slot_keys = step_search ? sb.slot_keys : nullptr;
    if (nposB == nullptr) {
        k_gather<false, false><<<nb, kBlock, 0, st>>>(
            P.n, P.ppc, skey, sid, sb.src, sb.slot_of_id, sb.ctrl, posA, velA, posB, velB, idsB,
            nullptr, nullptr, nullptr, nullptr, cnt_src, cnt_dst, scene_src, scene_dst, sb.table,
            sb.table_keys, slot_keys, counters, scene_overflow, scene_params, skip);
    } else if (snap_from_state) {
        k_gather<true, true><<<nb, kBlock, 0, st>>>(
            P.n, P.ppc, skey, sid, sb.src, sb.slot_of_id, sb.ctrl, posA, velA, posB, velB, idsB,
            nullptr, nullptr, nposB, nvelB, cnt_src, cnt_dst, scene_src, scene_dst, sb.table,
            sb.table_keys, slot_keys, counters, scene_overflow, scene_params, skip);
    } else {
        k_gather<true, false><<<nb, kBlock, 0, st>>>(
            P.n, P.ppc, skey, sid, sb.src, sb.slot_of_id, sb.ctrl, posA, velA, posB, velB, idsB,
            nposA, nvelA, nposB, nvelB, cnt_src, cnt_dst, scene_src, scene_dst, sb.table,
            sb.table_keys, slot_keys, counters, scene_overflow, scene_params, skip);
    }
}

void launch_candidate_count(const DevParams& P, SceneTab T, const float4* pos, const int* ids,
                            const int2* table, int* count_by_id, cudaStream_t st) {
    if (T.params) k_cand_count<true><<<blocks_for(P.n), kBlock, 0, st>>>(P, T, pos, ids, table, count_by_id);
    else k_cand_count<false><<<blocks_for(P.n), kBlock, 0, st>>>(P, T, pos, ids, table, count_by_id);
}

void launch_candidate_fill(const DevParams& P, SceneTab T, const float4* pos, const int* ids,
                           const int2* table, const int64_t* offsets_by_id, int* cand,
                           uint8_t* contact, cudaStream_t st) {
    if (T.params)
        k_cand_fill<true><<<blocks_for(P.n), kBlock, 0, st>>>(P, T, pos, ids, table, offsets_by_id,
                                                              cand, contact);
    else
        k_cand_fill<false><<<blocks_for(P.n), kBlock, 0, st>>>(P, T, pos, ids, table, offsets_by_id,
                                                               cand, contact);
}

void launch_state_to_aos(int n, const float4* pos, const float4* vel, const int* ids,
                         float* out6, cudaStream_t st) {
    k_state_to_aos<<<blocks_for(n), kBlock, 0, st>>>(n, pos, vel, ids, out6);
}

void launch_positions_to_aos(int n, const float4* pos, const int* ids, float* out3,
                             cudaStream_t st) {
    k_positions_to_aos<<<blocks_for(n), kBlock, 0, st>>>(n, pos, ids, out3);
}

void launch_rhs_to_aos(int n, const float4* vel_used, const float4* acc, const int* ids,
                       float* out6, cudaStream_t st) {
    k_rhs_to_aos<<<blocks_for(n), kBlock, 0, st>>>(n, vel_used, acc, ids, out6);
}

void launch_state_from_aos(int n, const float* in6, float4* pos, float4* vel, const int* ids,
                           cudaStream_t st) {
    k_state_from_aos<<<blocks_for(n), kBlock, 0, st>>>(n, in6, pos, vel, ids);
}

void launch_cell_keys_by_id(const DevParams& P, SceneTab T, const float4* pos, const int* ids,
                            int32_t* keys, cudaStream_t st) {
    if (T.params) k_cell_keys_by_id<true><<<blocks_for(P.n), kBlock, 0, st>>>(P, T, pos, ids, keys);
    else k_cell_keys_by_id<false><<<blocks_for(P.n), kBlock, 0, st>>>(P, T, pos, ids, keys);
}

}  // namespace wd
