// wd_lists.cu -- Verlet neighbor lists for the semi-implicit Euler and the backward
// Euler / Picard steps.
//
// The reference searches the grid every step (src/particle_dynamics.cu:264-281). With
// simulation.neighbor_skin = s > 0 the search runs only when needed: a build sorts the
// grains as the search does, and lists, for every grain, the grains whose centres are
// closer than r_i + r_j + s, in the contact kernel's canonical visiting order (stencil
// cell, then grain id). Until some grain has moved 0.49 s from where the build saw it
// (kListValid), every contact of every step is in the lists (a pair not listed is still
// >= r_i + r_j + 0.02 s apart), so the step computes the same contact set as the
// searched step.
//
// The results are bit-identical to the searched step because forces are accumulated
// in the same order: the kernel checks that the contacts it meets arrive in canonical
// order for the current positions ((stencil offset of the partner's current cell,
// partner id) non-decreasing); a grain for which a cell crossing broke that order
// re-sorts its contacts before accumulating them.
//
// Between builds the state stays in one order and ping-pongs between two buffers; a
// build gathers it into the new order, lists the neighbors, and copies it back.
//
// Picard iterates every force evaluation of a step on the same lists. Builds start at
// 0.30 skin instead of 0.49, and each iteration checks that its input iterate is still
// within 0.49 skin of the build; if one is not, the step is redone from its start
// state with the per-iteration search, so the results stay those of the searched step.
#include <algorithm>

#include "wd_kernels.h"

namespace wd {
namespace {

__device__ __forceinline__ bool skipped(const Skip& s) {
    return s.prev_res != nullptr && s.tol > 0.f && __uint_as_float(*s.prev_res) < s.tol;
}

// One thread: decide whether this step builds (the decision word, kLcDecision) and
// switch the build's conditional node where the graph holds one. The decision needs a bound B on max |x - x_build| of the current state:
// the exact maximum when the last contact kernel measured it (it then read the build
// positions), otherwise the previous bound plus the largest displacement of the last
// step (triangle inequality), so that most steps read no build positions. The measured
// squares carry float rounding of a few ulps, covered by the factor 1 + 2^-16. The
// next kernel measures exactly when B is within two last-step displacements of the
// threshold, so a build is triggered by the bound only when the exact value is close.
// A NaN or infinite displacement makes B infinite: the step builds.
// One thread. Volatile accesses: the fused form runs in the last block of a contact
// kernel whose other blocks updated these words with atomics.
__device__ bool list_decide_core(uint32_t* ctrl_, float thr, int always_exact,
                                 unsigned long long* counters) {
    volatile uint32_t* ctrl = ctrl_;
    volatile double* bound = reinterpret_cast<volatile double*>(ctrl_ + kLcBound);
    const double grow = 1.0 + 1.0 / 65536.0;
    const double step = sqrt(static_cast<double>(__uint_as_float(ctrl[kLcStep]))) * grow;
    double b = ctrl[kLcExact] != 0u
                   ? sqrt(static_cast<double>(__uint_as_float(ctrl[kLcDisp]))) * grow
                   : *bound + step;
    const bool build = ctrl[kLcForce] != 0u || ctrl[kLcOverflow] != 0u || !(b < thr);
    ctrl[kLcDecision] = build ? __float_as_uint(1.f) : 0u;
    if (build) {
        b = 0.0;
        ctrl[kLcOverflow] = 0u;
        ctrl[kLcForce] = 0u;
        counters[kCntListBuilds] += 1ull;
    }
    *bound = b;
    ctrl[kLcDisp] = 0u;
    ctrl[kLcStep] = 0u;
    const bool exact = always_exact || (!build && !(b + 2.0 * step < thr));
    ctrl[kLcExact] = exact ? 1u : 0u;
    if (exact) counters[kCntListExact] += 1ull;
    return build;
}

__global__ void k_list_decide(uint32_t* __restrict__ ctrl, float thr, int always_exact,
                              unsigned long long* __restrict__ counters, int use_cond,
                              cudaGraphConditionalHandle cond) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const bool build = list_decide_core(ctrl, thr, always_exact, counters);
    if (use_cond) cudaGraphSetConditional(cond, build ? 1u : 0u);
}

// The decision fused into the tail of a semi-implicit Euler list kernel: the last block
// to finish (every block's displacement atomics done) decides whether the lists are
// rebuilt before the next step: it switches the build's conditional node where the step
// graph holds one, or leaves the decision word to the kernel that launches the build's
// graphs from the device (wd_launch.cu). All threads
// of every block call it. The barrier orders the block's atomics before thread 0's
// fence and ticket (the grid-barrier pattern: one fence per block, not per thread).
__device__ __forceinline__ void list_tail_decide(const ListArgs& A) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned ticket = atomicAdd(A.tail_count, 1u);
        if (ticket == gridDim.x - 1) {
            __threadfence();
            const bool build = list_decide_core(A.list_ctrl, A.thr, 0, A.counters);
            *reinterpret_cast<volatile unsigned*>(A.tail_count) = 0u;
            if (A.use_cond) cudaGraphSetConditional(A.cond, build ? 1u : 0u);
        }
    }
}

// Grains in cells two apart along an axis are more than a cell width apart, so the 27
// stencil cells hold every contact; but when 2 r_max + skin exceeds a cell width, a pair
// two cells apart can be closer than r_i + r_j + skin and meet before the next build.
// A build then walks the outer shell of the 5 x 5 x 5 block too, cell by cell where its
// box lies within the grain's reach r_i + r_max + skin (only grains near a face of their
// cell, so few). Each shell cell is visited in the pass of the first axis along which
// it lies two cells away; its grains follow the stencil's in the list.
template <typename Visit>
__device__ __forceinline__ void list_far_shell(const DevParams& P, const int2* __restrict__ table,
                                               const float4* __restrict__ pos, float4 pi,
                                               int cx, int cy, int cz, Visit& visit) {
    const float reach_max = (pi.w + P.rmax) + P.skin;
    // the grain's offset in its cell per axis (the fast path's t minus the index) and the
    // cell mapping's rounding margin, in cells
    const float f0 = ((pi.x - P.lo[0]) * P.inv_len[0]) * static_cast<float>(P.grid[0]) -
                     static_cast<float>(cx);
    const float f1 = ((pi.y - P.lo[1]) * P.inv_len[1]) * static_cast<float>(P.grid[1]) -
                     static_cast<float>(cy);
    const float f2 = ((pi.z - P.lo[2]) * P.inv_len[2]) * static_cast<float>(P.grid[2]) -
                     static_cast<float>(cz);
    // distance from the grain to the box of cell c + o along axis a, shortened by the
    // margin (a NaN offset gives 0: every cell in reach)
    auto gap = [&](int a, int o) {
        const float f = a == 0 ? f0 : (a == 1 ? f1 : f2);
        const float g = o == 0 ? 0.f
                      : o == 1 ? 1.f - f
                      : o == -1 ? f
                      : o == 2 ? 2.f - f
                               : 1.f + f;
        const float m = 2.f * (a == 0 ? P.cell_err[0] : (a == 1 ? P.cell_err[1] : P.cell_err[2])) + 1e-4f;
        const float len = a == 0 ? P.cell_len[0] : (a == 1 ? P.cell_len[1] : P.cell_len[2]);
        return fmaxf(0.f, g - m) * len;
    };
    const float r2 = (reach_max * reach_max) * 1.0001f;
    // a cell two away along two axes is at least sqrt(2) cell widths (less the margins)
    // away: in reach only for a reach above about 1.4 cells
    // (an offset f lies in [-err, 1 + err] and the margin is 2 err + 1e-4 cells)
    const float w = P.cell_min * (1.f - 3.f * fmaxf(P.cell_err[0], fmaxf(P.cell_err[1], P.cell_err[2])) - 1e-4f);
    const bool two_axes = r2 > 2.f * w * w;
    for (int a = 0; a < 3; ++a) {
        // b < c: the other two axes; an axis before a stays within one cell (a is the
        // first axis at which the cell lies two away)
        const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
        for (int side = -2; side <= 2; side += 4) {
            const float ga = gap(a, side);
            if (ga * ga > r2) continue;
            const int bl = (b < a || !two_axes) ? -1 : -2;
            const int cl = (c < a || !two_axes) ? -1 : -2;
            for (int ob = bl; ob <= -bl; ++ob) {
                const float gb = gap(b, ob);
                if (ga * ga + gb * gb > r2) continue;
                for (int oc = cl; oc <= -cl; ++oc) {
                    const float gc = gap(c, oc);
                    if (ga * ga + gb * gb + gc * gc > r2) continue;
                    const int nx = cx + (a == 0 ? side : ob);
                    const int ny = cy + (a == 0 ? ob : (a == 1 ? side : oc));
                    const int nz = cz + (a == 2 ? side : oc);
                    if (nx < 0 || nx >= P.grid[0] || ny < 0 || ny >= P.grid[1] || nz < 0 ||
                        nz >= P.grid[2])
                        continue;
                    const int2 e = __ldg(&table[P.cell_base + flat_cell(P, nx, ny, nz)]);
                    for (int j = e.x; j < e.y; ++j) visit(j, __ldg(&pos[j]));
                }
            }
        }
    }
}

// The list of every grain, from the run table of the build's sorted state: the
// contact kernel's stencil walk with the skin added to the contact distance. The sorted
// state is copied back into the step's buffers on the way.
template <bool BATCH>
__global__ void __launch_bounds__(kBlock)
k_list_build(DevParams P0, SceneTab T, const float4* __restrict__ pos,
             const int2* __restrict__ table, int* __restrict__ nbr, int* __restrict__ nbr_cnt,
             float4* __restrict__ xbuild, uint32_t* __restrict__ ctrl, ListCopy cp, Skip skip) {
    if (skipped(skip)) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = P0.n;
    if (s >= n) return;
    const DevParams& P = scene_params<BATCH>(P0, T, s);
    const float4 pi = pos[s];
    cp.pos_out[s] = pi;
    cp.vel_out[s] = cp.vel[s];
    cp.ids_out[s] = cp.ids[s];
    if (cp.hcnt) cp.hcnt_out[s] = cp.hcnt[s];
    if (BATCH) cp.scene_out[s] = cp.scene[s];
    int cx, cy, cz;
    cell_coords(P, pi.x, pi.y, pi.z, cx, cy, cz);
    // the nine rows' slot ranges first (27 independent table loads), then the
    // candidates two at a time, in the stencil order
    int lo[9], hi[9];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int nx = cx + r - 1;
        if (nx >= 0 && nx < P.grid[0]) {
            row_ranges(P, table, nx, cy, cz, lo + 3 * r, hi + 3 * r);
        } else {
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                lo[3 * r + t] = 0;
                hi[3 * r + t] = 0;
            }
        }
    }
    int cnt = 0;
    auto visit = [&](int j, float4 pj) {
        if (j == s) return;
        float3 d;
        const float ns = pair_norm_sq(pi, pj, d);
        const float reach = (pi.w + pj.w) + P.skin;
        if (ns < reach * reach) {
            if (cnt < kNbrCap) nbr[static_cast<int64_t>(cnt) * n + s] = j;
            ++cnt;
        }
    };
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        int j = lo[r];
        const int e = hi[r];
        // an empty row has lo = INT_MAX, hi = 0: the difference does not overflow
        for (; e - j > 1; j += 2) {
            const float4 a = __ldg(&pos[j]);
            const float4 b = __ldg(&pos[j + 1]);
            visit(j, a);
            visit(j + 1, b);
        }
        if (j < e) visit(j, __ldg(&pos[j]));
    }
    if ((pi.w + P.rmax) + P.skin > P.cell_min) list_far_shell(P, table, pos, pi, cx, cy, cz, visit);
    nbr_cnt[s] = cnt;
    xbuild[s] = pi;
    if (cnt > kNbrCap) atomicOr(&ctrl[kLcOverflow], 1u);
}

__global__ void __launch_bounds__(kBlock)
k_list_copy(int n, const float4* __restrict__ pos, const float4* __restrict__ vel,
            const int* __restrict__ ids, const int* __restrict__ hcnt,
            const int* __restrict__ scene, float4* __restrict__ pos_out,
            float4* __restrict__ vel_out, int* __restrict__ ids_out, int* __restrict__ hcnt_out,
            int* __restrict__ scene_out, Skip skip) {
    if (skipped(skip)) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    pos_out[s] = pos[s];
    vel_out[s] = vel[s];
    ids_out[s] = ids[s];
    if (hcnt) hcnt_out[s] = hcnt[s];
    if (scene) scene_out[s] = scene[s];
}

// Position of a partner in the canonical visiting order: the stencil offset of its
// current cell (dx, then dy, then dz, ascending), then its id.
__device__ __forceinline__ unsigned long long visit_key(const DevParams& P, int cx, int cy,
                                                        int cz, float4 pj, int jd) {
    int jx, jy, jz;
    cell_coords(P, pj.x, pj.y, pj.z, jx, jy, jz);
    const int sidx = ((jx - cx + 1) * 3 + (jy - cy + 1)) * 3 + (jz - cz + 1);
    return (static_cast<unsigned long long>(static_cast<unsigned>(sidx)) << 32) |
           static_cast<unsigned>(jd);
}

// |x1 - x0|^2 as float bits; NaN compares above every float, so a diverging grain
// reports +inf and forces a build.
__device__ __forceinline__ uint32_t disp_sq_bits(float3 x1, float3 x0) {
    const float ex = x1.x - x0.x, ey = x1.y - x0.y, ez = x1.z - x0.z;
    const float d2 = ex * ex + ey * ey + ez * ez;
    return d2 >= 0.f ? __float_as_uint(d2) : 0x7f800000u;
}
__device__ __forceinline__ uint32_t disp_sq_bits(float3 x1, float4 x0) {
    return disp_sq_bits(x1, make_float3(x0.x, x0.y, x0.z));
}

// Warp maxima of the displacement measures into list_ctrl (the exact one only on the
// steps that measure it; the per-step one for semi-implicit Euler).
template <bool PICARD>
__device__ __forceinline__ void list_disp_report(uint32_t* ctrl, bool exact, uint32_t disp_bits,
                                                 uint32_t step_bits) {
    if (exact) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            disp_bits = max(disp_bits, __shfl_xor_sync(0xffffffffu, disp_bits, o));
        if ((threadIdx.x & 31) == 0 && disp_bits != 0u) atomicMax(&ctrl[kLcDisp], disp_bits);
    }
    if (!PICARD) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            step_bits = max(step_bits, __shfl_xor_sync(0xffffffffu, step_bits, o));
        if ((threadIdx.x & 31) == 0 && step_bits != 0u) atomicMax(&ctrl[kLcStep], step_bits);
    }
}

// Asks L1 for the line holding p; nothing is read into registers, so a later __ldg of
// p finds it on chip without holding registers in between.
__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// The contacts of a grain whose list entries a cell crossing re-ordered, in canonical
// order: each pass takes the smallest visiting key above the last. (Inlined: an
// out-of-line call copies the parameter structs to local memory at kernel entry, which
// was measured to cost more than the code it moves away.)
template <bool HIST>
__device__ __forceinline__ void list_contacts_sorted(const DevParams& P, const ListArgs& A, int s,
                                                  int n, int cnt, float4 pi, float3 vel,
                                                  float mi, float cut, int cx, int cy, int cz,
                                                  float3& f, HistRow& h) {
    const float ri = pi.w;
    long long done = -1;
    for (;;) {
        long long best = 0x7fffffffffffffffll;
        int bj = -1;
        for (int e = 0; e < cnt; ++e) {
            const int j = __ldg(&A.nbr[static_cast<int64_t>(e) * n + s]);
            const float4 pj = __ldg(&A.pos[j]);
            float3 d;
            const float ns = pair_norm_sq(pi, pj, d);
            if (ns > cut) continue;
            const float dist = pair_dist(sqrtf(ns), ri, pj.w);
            if (!(dist < 0.f)) continue;
            const long long key =
                static_cast<long long>(visit_key(P, cx, cy, cz, pj, __ldg(&A.ids[j])));
            if (key > done && key < best) {
                best = key;
                bj = j;
            }
        }
        if (bj < 0) break;
        done = best;
        const float4 pj = __ldg(&A.pos[bj]);
        float3 d;
        const float ns = pair_norm_sq(pi, pj, d);
        const float norm = sqrtf(ns);
        const float dist = pair_dist(norm, ri, pj.w);
        const float4 vj = __ldg(&A.vel[bj]);
        pair_force<HIST>(P, d, norm, dist, vel, mi, vj, static_cast<int>(best & 0xffffffffll),
                         f, h, A.counters);
    }
}

// The same for a grain whose contacts the scan found (bitmask over list entries): each
// pass visits the contacts only, and takes the smallest visiting key above the last.
template <bool HIST>
__device__ __forceinline__ void list_contacts_sorted_mask(const DevParams& P, const ListArgs& A,
                                                       int s, int n, unsigned long long hits,
                                                       float4 pi, float3 vel, float mi, int cx,
                                                       int cy, int cz, float3& f, HistRow& h) {
    const float ri = pi.w;
    long long done = -1;
    for (;;) {
        long long best = 0x7fffffffffffffffll;
        int be = -1;
        for (unsigned long long m = hits; m; m &= m - 1ull) {
            const int e = __ffsll(static_cast<long long>(m)) - 1;
            const int j = __ldg(&A.nbr[static_cast<int64_t>(e) * n + s]);
            const long long key = static_cast<long long>(
                visit_key(P, cx, cy, cz, __ldg(&A.pos[j]), __ldg(&A.ids[j])));
            if (key > done && key < best) {
                best = key;
                be = e;
            }
        }
        if (be < 0) break;
        done = best;
        const int j = __ldg(&A.nbr[static_cast<int64_t>(be) * n + s]);
        const float4 pj = __ldg(&A.pos[j]);
        float3 d;
        const float ns = pair_norm_sq(pi, pj, d);
        const float norm = sqrtf(ns);
        const float dist = pair_dist(norm, ri, pj.w);
        const float4 vj = __ldg(&A.vel[j]);
        pair_force<HIST>(P, d, norm, dist, vel, mi, vj, static_cast<int>(best & 0xffffffffll),
                         f, h, A.counters);
    }
}

// The contacts of a grain whose list overflowed, from the run table of the build that
// ran this step (the stencil walk of the searched kernel).
template <bool HIST>
__device__ __forceinline__ void list_contacts_table(const DevParams& P, const ListArgs& A, int s,
                                                 float4 pi, float3 vel, float mi, float cut,
                                                 int cx, int cy, int cz, float3& f, HistRow& h) {
    const float ri = pi.w;
    for (int dx = -1; dx <= 1; ++dx) {
        const int nx = cx + dx;
        if (nx < 0 || nx >= P.grid[0]) continue;
        int lo[3], hi[3];
        row_ranges(P, A.table, nx, cy, cz, lo, hi);
        for (int t = 0; t < 3; ++t) {
            for (int j = lo[t]; j < hi[t]; ++j) {
                const float4 pj = __ldg(&A.pos[j]);
                float3 d;
                const float ns = pair_norm_sq(pi, pj, d);
                if (ns > cut || j == s) continue;
                const float norm = sqrtf(ns);
                const float dist = pair_dist(norm, ri, pj.w);
                if (!(dist < 0.f)) continue;
                const float4 vj = __ldg(&A.vel[j]);
                const int partner = HIST ? __ldg(&A.ids[j]) : 0;
                pair_force<HIST>(P, d, norm, dist, vel, mi, vj, partner, f, h, A.counters);
            }
        }
    }
}

// One grain of the list contact kernels, its per-slot values already loaded: contacts
// from the list in canonical order (or the run table when the list overflowed), the
// integrator, the displacement measures (maxima folded into disp_bits / step_bits /
// res_bits, viol or-ed). warp_listed: some grain of the calling warp has a list entry
// (warp-uniform). order_out: write the slot's id (and scene) too. Between builds
// the slot order is fixed and the ids of both state buffers agree, so only the first
// step after a build (whose gather reordered one buffer) and Picard write them.
template <bool HIST, bool BATCH, bool PICARD, bool PREFETCH = false>
__device__ __forceinline__ void list_grain(const DevParams& P0, const ListArgs& A, int s, int n,
                                           int scene, float4 pi, float4 vi, int id, int cnt,
                                           float4 xb, int hcnt_in, bool exact, bool order_out,
                                           bool warp_listed, uint32_t& disp_bits,
                                           uint32_t& step_bits, uint32_t& res_bits, bool& viol) {
    const DevParams& P = BATCH ? A.scene_params[scene] : P0;
    if (PICARD) {
        // the rhs of a Picard step pairs the last iterate's velocity with its forces
        A.rhs_vel[s] = vi;
        A.rhs_ids[s] = id;
        if (A.iter > 0) {
            const float ex = pi.x - xb.x, ey = pi.y - xb.y, ez = pi.z - xb.z;
            viol |= !(ex * ex + ey * ey + ez * ez < A.viol_thr);
        }
    }
    if (BATCH && P.frozen) {
        A.pos_out[s] = pi;
        A.vel_out[s] = vi;
        if (order_out) {
            A.ids_out[s] = id;
            A.scene_out[s] = scene;
        }
        A.acc_out[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (HIST) A.hcnt_out[s] = 0;
    } else {
        const float3 pos = make_float3(pi.x, pi.y, pi.z);
        const float3 vel = make_float3(vi.x, vi.y, vi.z);
        const float ri = pi.w, mi = vi.w;
        float3 f = make_float3(0.f, 0.f, 0.f);
        HistRow h;
        if (HIST) {
            h.in = A.hist_in + static_cast<int64_t>(id) * kHistCap;
            h.in_count = hcnt_in;
            h.out = A.hist_out + static_cast<int64_t>(id) * kHistCap;
            h.out_count = 0;
            // the first stored spring is probed first: on its way while the list is scanned
            if (PREFETCH && hcnt_in > 0) prefetch_l1(h.in);
        }
        wall_forces<HIST>(P, pos, vel, ri, mi, f, h, A.counters);
        // the list contacts, skipped as a whole by warps in which no grain has a list
        // entry (ballistic grains: the contact code's registers stay out of their path)
        if (warp_listed) {
            const float3 f_walls = f;
            const int out_walls = HIST ? h.out_count : 0;
            const float cut = contact_cutoff_sq(ri, P.rmax);
            // the grain's cell orders its contacts; a grain without list entries needs none
            int cx = 0, cy = 0, cz = 0;
            if (cnt > 0) cell_coords(P, pi.x, pi.y, pi.z, cx, cy, cz);
            bool ordered = true;
            if (cnt <= kNbrCap) {
                // scan: which entries are contacts, four entries' loads in flight at a
                // time (index loads, then the partners' positions), one bit each
                unsigned long long hits = 0ull;
                for (int e0 = 0; e0 < cnt; e0 += 4) {
                    int jj[4];
                    float4 pp[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        jj[u] = e0 + u < cnt ? __ldg(&A.nbr[static_cast<int64_t>(e0 + u) * n + s]) : s;
#pragma unroll
                    for (int u = 0; u < 4; ++u) pp[u] = __ldg(&A.pos[jj[u]]);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        float3 d;
                        const float ns = pair_norm_sq(pi, pp[u], d);
                        const bool hit = e0 + u < cnt && !(ns > cut) &&
                                         pair_dist(sqrtf(ns), ri, pp[u].w) < 0.f;
                        hits |= hit ? (1ull << (e0 + u)) : 0ull;
                        // the contact's partner id and velocity are read after the scan
                        if (PREFETCH && hit) {
                            prefetch_l1(&A.ids[jj[u]]);
                            prefetch_l1(&A.vel[jj[u]]);
                        }
                    }
                }
                // the contacts, in list order, while they arrive in canonical order (the
                // partner's values are re-read: L1 hits, same arithmetic as the scan)
                const unsigned long long all_hits = hits;
                unsigned long long last = 0ull;
                while (hits) {
                    const int e = __ffsll(static_cast<long long>(hits)) - 1;
                    hits &= hits - 1ull;
                    const int j = __ldg(&A.nbr[static_cast<int64_t>(e) * n + s]);
                    const float4 pj = __ldg(&A.pos[j]);
                    float3 d;
                    const float ns = pair_norm_sq(pi, pj, d);
                    const float norm = sqrtf(ns);
                    const float dist = pair_dist(norm, ri, pj.w);
                    const int jd = __ldg(&A.ids[j]);
                    const unsigned long long key = visit_key(P, cx, cy, cz, pj, jd);
                    if (key < last) {
                        ordered = false;
                        break;
                    }
                    last = key;
                    const float4 vj = __ldg(&A.vel[j]);
                    pair_force<HIST>(P, d, norm, dist, vel, mi, vj, jd, f, h, A.counters);
                }
                if (!ordered) {
                    // a cell crossing re-ordered this grain's contacts: redo them in
                    // canonical order
                    f = f_walls;
                    if (HIST) h.out_count = out_walls;
                    atomicAdd(&A.counters[kCntListResort], 1ull);
                    list_contacts_sorted_mask<HIST>(P, A, s, n, all_hits, pi, vel, mi, cx, cy, cz,
                                                    f, h);
                }
            } else {
                // list overflow: this step built the lists, so the run table is fresh
                list_contacts_table<HIST>(P, A, s, pi, vel, mi, cut, cx, cy, cz, f, h);
            }
        }
        if (HIST) A.hcnt_out[s] = h.out_count;
        const float3 a = make_float3(f.x / mi, f.y / mi, f.z / mi);
        float3 v1, x1;
        if (!PICARD) {
            v1 = make_float3(fmaf(P.dt, a.x, vel.x), fmaf(P.dt, a.y, vel.y),
                             fmaf(P.dt, a.z, vel.z));
            x1 = make_float3(fmaf(P.dt, v1.x, pos.x), fmaf(P.dt, v1.y, pos.y),
                             fmaf(P.dt, v1.z, pos.z));
        } else {
            const float4 xn = A.xn[s], vn = A.vn[s];
            v1 = make_float3(fmaf(P.dt, a.x, vn.x), fmaf(P.dt, a.y, vn.y),
                             fmaf(P.dt, a.z, vn.z));
            x1 = make_float3(fmaf(P.dt, v1.x, xn.x), fmaf(P.dt, v1.y, xn.y),
                             fmaf(P.dt, v1.z, xn.z));
            res_bits = max(res_bits, __float_as_uint(fabsf(x1.x - pos.x)));
            res_bits = max(res_bits, __float_as_uint(fabsf(x1.y - pos.y)));
            res_bits = max(res_bits, __float_as_uint(fabsf(x1.z - pos.z)));
        }
        A.pos_out[s] = make_float4(x1.x, x1.y, x1.z, ri);
        A.vel_out[s] = make_float4(v1.x, v1.y, v1.z, mi);
        if (order_out) {
            A.ids_out[s] = id;
            if (BATCH) A.scene_out[s] = scene;
        }
        A.acc_out[s] = make_float4(a.x, a.y, a.z, 0.f);
        if (exact) disp_bits = max(disp_bits, disp_sq_bits(x1, xb));
        if (!PICARD) step_bits = max(step_bits, disp_sq_bits(x1, pos));
    }
}

// MINB resident blocks per SM: 5 caps registers at 48 (more warps, a few spills), 4 at
// 64 (no spills); the autotuner picks. The 64-register form also prefetches, into L1,
// each contact's partner id and velocity when the scan finds it, and the grain's first
// stored spring (measured: 2% on a settled column; at 48 registers the prefetches'
// addresses added spills and cost more than they saved).
// PICARD: one backward-Euler / Picard iteration (src/backward_euler_picard_kernel.cu:4-17):
// forces at the iterate (pos, vel), integration from the step-start state (xn, vn), the
// residual max |x_{k+1} - x_k|; an iterate that has left the lists' validity bound marks
// the step for a redo.
template <bool HIST, bool BATCH, int MINB, bool PICARD>
__global__ void __launch_bounds__(kBlock, MINB)
k_force_list(DevParams P0, ListArgs A) {
    if (PICARD && skipped(A.skip)) return;
    const int n = P0.n;
    uint32_t disp_bits = 0u, step_bits = 0u;
    uint32_t res_bits = 0u;
    bool viol = false;
    // build positions are read only on the steps that measure the exact displacement;
    // ids only right after a build
    const bool exact = PICARD || A.list_ctrl[kLcExact] != 0u;
    const bool order_out = PICARD || A.list_ctrl[kLcDecision] != 0u;
    // a grid-stride loop: semi-implicit Euler launches one wave (its fused build decision
    // then waits once per block, not once per block of a many-wave grid); Picard launches
    // one slot per thread
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const int s = base + threadIdx.x;
        const bool live = s < n;
        // every per-slot load issued up front: they are independent, and the kernel is
        // bound by their latency when lists are short
        int scene = 0, id = 0, cnt = 0, hcnt_in = 0;
        float4 pi = make_float4(0.f, 0.f, 0.f, 0.f), vi = pi, xb = pi;
        if (live) {
            scene = BATCH ? A.scene[s] : 0;
            pi = A.pos[s];
            vi = A.vel[s];
            id = A.ids[s];
            cnt = A.nbr_cnt[s];
            hcnt_in = HIST ? A.hcnt_in[s] : 0;
            if (exact) xb = A.xbuild[s];
        }
        const bool warp_listed = __any_sync(0xffffffffu, cnt != 0);
        if (live)
            list_grain<HIST, BATCH, PICARD, MINB == 4 && !PICARD>(
                P0, A, s, n, scene, pi, vi, id, cnt, xb, hcnt_in, exact, order_out, warp_listed,
                disp_bits, step_bits, res_bits, viol);
    }
    list_disp_report<PICARD>(A.list_ctrl, exact, disp_bits, step_bits);
    if (!PICARD) list_tail_decide(A);
    if (PICARD) {
        // max of non-negative float bits (NaN above +inf, so it is kept)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) res_bits = max(res_bits, __shfl_xor_sync(0xffffffffu, res_bits, o));
        if ((threadIdx.x & 31) == 0 && res_bits != 0u) atomicMax(A.res_slot, res_bits);
        if (__any_sync(0xffffffffu, viol) && (threadIdx.x & 31) == 0) atomicOr(&A.list_ctrl[kLcViol], 1u);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            *A.picard_used = A.iter + 1;
            A.counters[kCntPicardIters] += 1ull;
        }
    }
}

// ---- bulk-staged list kernel -------------------------------------------------------
// Persistent warps over tiles of 32 slots. Each warp keeps two tiles in flight: lane 0
// issues the tile's per-slot arrays (x, v, ids, list count, spring count, scene, and
// the build positions on measuring steps) as 1-D bulk copies (cp.async.bulk, the TMA
// engine; each copy reads this GPU's memory into the issuing CTA only) into the warp's
// shared stage, completing on an mbarrier; the lanes compute the tile before while the
// next arrives. The per-slot loads, whose
// latency binds the per-lane kernel, leave the critical path. Contacts, forces and the
// integrator are the per-lane kernel's (list_grain), so the results are identical.
constexpr int kStageWarps = kBlock / 32;
constexpr int kStageTile = 32;
struct __align__(16) SlotStage {
    float4 pos[kStageTile];
    float4 vel[kStageTile];
    float4 xb[kStageTile];
    int ids[kStageTile];
    int cnt[kStageTile];
    int hcnt[kStageTile];
    int scene[kStageTile];
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// global -> this CTA's shared memory, completing `bytes` on bar (16-byte aligned
// addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for a phase: false after limit_ns without completion.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

template <bool HIST, bool BATCH>
__device__ __forceinline__ void stage_issue(const ListArgs& A, int tile, bool exact,
                                            SlotStage& S, uint64_t* bar) {
    const int s0 = tile * kStageTile;
    constexpr uint32_t f4 = kStageTile * sizeof(float4), i4 = kStageTile * sizeof(int);
    const uint32_t bytes = 2u * f4 + 2u * i4 + (HIST ? i4 : 0u) + (BATCH ? i4 : 0u) +
                           (exact ? f4 : 0u);
    mbar_expect_tx(bar, bytes);
    bulk_g2s(S.pos, A.pos + s0, f4, bar);
    bulk_g2s(S.vel, A.vel + s0, f4, bar);
    bulk_g2s(S.ids, A.ids + s0, i4, bar);
    bulk_g2s(S.cnt, A.nbr_cnt + s0, i4, bar);
    if (HIST) bulk_g2s(S.hcnt, A.hcnt_in + s0, i4, bar);
    if (BATCH) bulk_g2s(S.scene, A.scene + s0, i4, bar);
    if (exact) bulk_g2s(S.xb, A.xbuild + s0, f4, bar);
}

// MINB: resident blocks per SM (5: 48 registers per thread, 4: 64). Tiles: warp w of W
// takes tiles w, w + W, w + 2W, ... (claiming the last rounds from a shared counter
// instead was measured slower: the claims serialize on one address just when every
// warp needs its next tile).
template <bool HIST, bool BATCH, int MINB>
__global__ void __launch_bounds__(kBlock, MINB)
k_force_list_staged(DevParams P0, ListArgs A) {
    __shared__ SlotStage stage[kStageWarps][2];
    __shared__ uint64_t bars[kStageWarps][2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int n = P0.n;
    const int tiles = (n + kStageTile - 1) / kStageTile;
    const int whole = n / kStageTile;  // tiles with 32 slots go through the stages
    const int W = gridDim.x * kStageWarps;
    const int first = blockIdx.x * kStageWarps + w;
    const bool exact = A.list_ctrl[kLcExact] != 0u;
    const bool order_out = A.list_ctrl[kLcDecision] != 0u;  // first step after a build
    const uint32_t wait_us = A.list_ctrl[kLcWaitUs];
    const uint64_t limit_ns = wait_us ? 1000ull * wait_us : 1000000000ull;
    const bool stall_test = A.list_ctrl[kLcStallTest] != 0u;
    SlotStage* S = stage[w];
    uint64_t* bar = bars[w];
    // tiles of iterations it (cur, in stage it & 1) and it + 1 (nxt), in registers
    int cur = first, nxt = first + W;
    if (lane == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init_fence();
        if (cur < whole) {
            if (stall_test) mbar_expect_tx(&bar[0], 16u);   // nothing will arrive
            else stage_issue<HIST, BATCH>(A, cur, exact, S[0], &bar[0]);
        }
        if (nxt < whole) stage_issue<HIST, BATCH>(A, nxt, exact, S[1], &bar[1]);
    }
    __syncwarp();
    uint32_t disp_bits = 0u, step_bits = 0u, res_bits = 0u;
    bool viol = false, failed = false;
    int it = 0;
    for (;; ++it) {
        const int st = it & 1;
        const int t = cur;
        if (t >= tiles) break;
        const int s = t * kStageTile + lane;
        float4 pi = make_float4(0.f, 0.f, 0.f, 0.f), vi = pi, xb = pi;
        int id = 0, cnt = 0, hcnt_in = 0, scene = 0;
        if (t < whole) {
            const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar[st], (it >> 1) & 1, limit_ns));
            if (!ok) {
                failed = true;
                break;
            }
            const SlotStage& T = S[st];
            pi = T.pos[lane];
            vi = T.vel[lane];
            id = T.ids[lane];
            cnt = T.cnt[lane];
            if (HIST) hcnt_in = T.hcnt[lane];
            if (BATCH) scene = T.scene[lane];
            if (exact) xb = T.xb[lane];
            __syncwarp();
            // the stage is read: refill it with the tile two ahead
            const int tn = nxt + W;
            if (lane == 0 && tn < whole) stage_issue<HIST, BATCH>(A, tn, exact, S[st], &bar[st]);
            cur = nxt;
            nxt = tn;
        } else {
            // the ragged last tile: plain loads, nothing after it
            cur = nxt;
            nxt = tiles;
            if (s < n) {
                pi = A.pos[s];
                vi = A.vel[s];
                id = A.ids[s];
                cnt = A.nbr_cnt[s];
                if (HIST) hcnt_in = A.hcnt_in[s];
                if (BATCH) scene = A.scene[s];
                if (exact) xb = A.xbuild[s];
            }
        }
        const bool warp_listed = __any_sync(0xffffffffu, cnt != 0);
        if (s < n)
            list_grain<HIST, BATCH, false>(P0, A, s, n, scene, pi, vi, id, cnt, xb, hcnt_in,
                                           exact, order_out, warp_listed, disp_bits,
                                           step_bits, res_bits, viol);
    }
    if (failed) {
        // a stage never completed: flag it and drain what this warp still has in flight
        // (bounded); the step is left unfinished for the host to report
        if (lane == 0) {
            atomicAdd(&A.counters[kCntStageTimeout], 1ull);
            if (cur < whole) mbar_wait(&bar[it & 1], (it >> 1) & 1, limit_ns);
            if (nxt < whole) mbar_wait(&bar[(it + 1) & 1], ((it + 1) >> 1) & 1, limit_ns);
        }
    } else {
        list_disp_report<false>(A.list_ctrl, exact, disp_bits, step_bits);
    }
    list_tail_decide(A);
}

// ---- list build with the tile's neighbour window staged in shared memory ----------
// One block per 256 consecutive sorted slots (single scene). Every grain's candidates
// lie in its nine stencil rows (three z-consecutive cells of one column each, one slot
// range per row); over the tile, row r's ranges lie inside [min lo_r, max hi_r). Those
// nine hulls, merged where they overlap (consecutive columns of one x-plane are
// consecutive in slot order), are copied into shared memory once by bulk copies
// (cp.async.bulk, this GPU's memory into this CTA, completing on an mbarrier), and the
// threads read their candidates there: 27 position loads per grain from L2 become a
// few per grain. A window above kWinCap positions, or a copy that does not complete
// within the bounded wait, falls back to global loads. Same lists, same order.
constexpr int kWinCap = 2560;   // positions (40 KB): five blocks per SM

__global__ void __launch_bounds__(kBlock)
k_list_build_tiled(DevParams P, const float4* __restrict__ pos, const int2* __restrict__ table,
                   int* __restrict__ nbr, int* __restrict__ nbr_cnt, float4* __restrict__ xbuild,
                   uint32_t* __restrict__ ctrl, ListCopy cp, Skip skip,
                   unsigned long long* __restrict__ counters) {
    if (skipped(skip)) return;
    __shared__ float4 win[kWinCap];
    __shared__ int hull_lo[9], hull_hi[9], row_off[9];
    __shared__ int staged;
    __shared__ __align__(8) uint64_t bar;
    const int n = P.n;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = s < n;
    if (threadIdx.x < 9) {
        hull_lo[threadIdx.x] = 0x7fffffff;
        hull_hi[threadIdx.x] = 0;
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    int lo[9], hi[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        lo[r] = 0x7fffffff;
        hi[r] = 0;
    }
    if (live) {
        pi = pos[s];
        cp.pos_out[s] = pi;
        cp.vel_out[s] = cp.vel[s];
        cp.ids_out[s] = cp.ids[s];
        if (cp.hcnt) cp.hcnt_out[s] = cp.hcnt[s];
        int cx, cy, cz;
        cell_coords(P, pi.x, pi.y, pi.z, cx, cy, cz);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const int nx = cx + r - 1;
            if (nx >= 0 && nx < P.grid[0]) row_ranges(P, table, nx, cy, cz, lo + 3 * r, hi + 3 * r);
        }
    }
    __syncthreads();   // hull initialisation and the barrier's init visible
    if (live) {
#pragma unroll
        for (int r = 0; r < 9; ++r) {
            if (lo[r] < hi[r]) {
                atomicMin(&hull_lo[r], lo[r]);
                atomicMax(&hull_hi[r], hi[r]);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // merge the nine hulls into disjoint ranges (ascending), stage them if they fit
        int idx[9], m = 0;
        for (int r = 0; r < 9; ++r)
            if (hull_lo[r] < hull_hi[r]) idx[m++] = r;
        for (int a = 1; a < m; ++a) {          // insertion sort by hull start
            const int v = idx[a];
            int b = a - 1;
            while (b >= 0 && hull_lo[idx[b]] > hull_lo[v]) {
                idx[b + 1] = idx[b];
                --b;
            }
            idx[b + 1] = v;
        }
        int mlo[9], mhi[9], nm = 0, total = 0;
        for (int a = 0; a < m; ++a) {
            const int r = idx[a];
            if (nm > 0 && hull_lo[r] <= mhi[nm - 1]) {
                mhi[nm - 1] = max(mhi[nm - 1], hull_hi[r]);
            } else {
                mlo[nm] = hull_lo[r];
                mhi[nm] = hull_hi[r];
                ++nm;
            }
        }
        for (int k = 0; k < nm; ++k) total += mhi[k] - mlo[k];
        const bool fits = nm > 0 && total <= kWinCap;
        staged = fits ? 1 : 0;
        if (fits) {
            int base[9];
            int acc = 0;
            for (int k = 0; k < nm; ++k) {
                base[k] = acc;
                acc += mhi[k] - mlo[k];
            }
            for (int a = 0; a < m; ++a) {
                const int r = idx[a];
                int k = 0;
                while (!(hull_lo[r] >= mlo[k] && hull_hi[r] <= mhi[k])) ++k;
                row_off[r] = base[k] - mlo[k];
            }
            mbar_expect_tx(&bar, static_cast<uint32_t>(total) * 16u);
            for (int k = 0; k < nm; ++k)
                bulk_g2s(&win[base[k]], pos + mlo[k], static_cast<uint32_t>(mhi[k] - mlo[k]) * 16u, &bar);
        }
    }
    __syncthreads();
    bool use_win = staged != 0;
    if (use_win) {
        const bool ok = mbar_wait(&bar, 0u, 1000000000ull);
        if (!__syncthreads_and(ok)) {
            if (threadIdx.x == 0) atomicAdd(&counters[kCntStageTimeout], 1ull);
            use_win = false;
        }
    }
    if (!live) return;
    int cnt = 0;
    auto visit = [&](int j, float4 pj) {
        if (j == s) return;
        float3 d;
        const float ns = pair_norm_sq(pi, pj, d);
        const float reach = (pi.w + pj.w) + P.skin;
        if (ns < reach * reach) {
            if (cnt < kNbrCap) nbr[static_cast<int64_t>(cnt) * n + s] = j;
            ++cnt;
        }
    };
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        int j = lo[r];
        const int e = hi[r];
        if (use_win) {
            if (j < e) {
                const float4* w = win + row_off[r];
                for (; j < e; ++j) visit(j, w[j]);
            }
        } else {
            for (; e - j > 1; j += 2) {
                const float4 a = __ldg(&pos[j]);
                const float4 b = __ldg(&pos[j + 1]);
                visit(j, a);
                visit(j + 1, b);
            }
            if (j < e) visit(j, __ldg(&pos[j]));
        }
    }
    if ((pi.w + P.rmax) + P.skin > P.cell_min) {
        // the outer shell, from global memory (the window holds the stencil only)
        int cx, cy, cz;
        cell_coords(P, pi.x, pi.y, pi.z, cx, cy, cz);
        list_far_shell(P, table, pos, pi, cx, cy, cz, visit);
    }
    nbr_cnt[s] = cnt;
    xbuild[s] = pi;
    if (cnt > kNbrCap) atomicOr(&ctrl[kLcOverflow], 1u);
}

// The last executed Picard iteration k wrote the B buffers when k is even and the
// scratch buffers when k is odd (iterations alternate, starting in B).
__global__ void __launch_bounds__(kBlock)
k_list_finalize(int n, const int* __restrict__ used, const float4* __restrict__ xpos,
                const float4* __restrict__ xvel, float4* __restrict__ pos,
                float4* __restrict__ vel) {
    if ((*used & 1) != 0) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    pos[s] = xpos[s];
    vel[s] = xvel[s];
}

__global__ void k_list_picard_check(uint32_t* __restrict__ ctrl,
                                    unsigned long long* __restrict__ counters, int use_cond,
                                    cudaGraphConditionalHandle cond) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const bool redo = ctrl[kLcViol] != 0u;
    ctrl[kLcViol] = 0u;
    ctrl[kLcRedo] = redo ? __float_as_uint(1.f) : 0u;
    if (redo) {
        ctrl[kLcForce] = 1u;  // the redo re-sorts the state: build next step
        counters[kCntPicardRedos] += 1ull;
    }
    if (use_cond) cudaGraphSetConditional(cond, redo ? 1u : 0u);
}

// Warp-cooperative variant: a contact's work (spring lookup, Coulomb cap, dashpot) is
// spread over the lanes of the warp instead of running on its grain's lane alone, then
// every grain accumulates its contacts' terms in order. The per-lane kernel above
// spends most issue slots on one or two active lanes when contacts are sparse.
//
// Per warp: rounds over the list entries (e = 0, 1, ...) find the contacts of the 32
// grains and queue them (partner slot, owner lane, owner's contact rank); a full queue
// (kCoopCap) or the last round flushes it: the lanes compute the queued contacts' terms
// (pair_terms, the springs written to their final rows), each grain's terms land in
// its own run of the buffer, and each lane accumulates its run in order. Contacts are
// found in list order, which is the canonical order unless a cell crossing changed it;
// such a grain redoes its contacts in canonical order on its own lane at the end.
constexpr int kCoopWarps = kBlock / 32;
constexpr int kCoopCap = 64;

struct CoopWarp {
    int qj[kCoopCap];
    unsigned char qg[kCoopCap];
    unsigned char qr[kCoopCap];
    PairTerms terms[kCoopCap];
    float4 pos[32], vel[32];
    int id[32], hin[32], outw[32], first[32], off[32], scene[32];
};

template <bool HIST, bool BATCH>
__device__ __forceinline__ void coop_flush(const DevParams& P0, const ListArgs& A, CoopWarp& W,
                                           int q, int lane, int my_count, int& bstart,
                                           bool reorder, float3& f) {
    __syncwarp();
    const int c = my_count - bstart;
    int off = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, off, o);
        if (lane >= o) off += y;
    }
    off -= c;
    W.first[lane] = bstart;
    W.off[lane] = off;
    __syncwarp();
    for (int i = lane; i < q; i += 32) {
        const int j = W.qj[i];
        const int g = W.qg[i];
        const int r = W.qr[i];
        const DevParams& P = BATCH ? A.scene_params[W.scene[g]] : P0;
        const float4 pi = W.pos[g], vi = W.vel[g];
        const float4 pj = __ldg(&A.pos[j]);
        const float4 vj = __ldg(&A.vel[j]);
        const int jd = __ldg(&A.ids[j]);
        float3 d;
        const float ns = pair_norm_sq(pi, pj, d);
        const float norm = sqrtf(ns);
        const float dist = pair_dist(norm, pi.w, pj.w);
        const int gid = W.id[g];
        float3 xi = HIST ? find_spring(A.hist_in + static_cast<int64_t>(gid) * kHistCap, W.hin[g], jd)
                         : make_float3(0.f, 0.f, 0.f);
        W.terms[W.off[g] + (r - W.first[g])] =
            pair_terms<HIST>(P, d, norm, dist, make_float3(vi.x, vi.y, vi.z), vi.w, vj, xi);
        if (HIST) {
            const int slot = W.outw[g] + r;
            if (slot < kHistCap)
                A.hist_out[static_cast<int64_t>(gid) * kHistCap + slot] =
                    make_float4(xi.x, xi.y, xi.z, __int_as_float(jd));
        }
    }
    __syncwarp();
    if (!reorder)
        for (int k = 0; k < c; ++k) pair_accumulate<HIST>(f, W.terms[off + k]);
    __syncwarp();
    bstart = my_count;
}

// One slot per lane of the warp-cooperative kernel (all lanes of the warp together).
template <bool HIST, bool BATCH>
__device__ __forceinline__ void coop_slot(const DevParams& P0, const ListArgs& A, CoopWarp& W, int s, bool exact,
                                          bool order_out, uint32_t& disp_bits,
                                          uint32_t& step_bits) {
    const int lane = threadIdx.x & 31;
    const int n = P0.n;
    const bool active = s < n;
    // per-slot loads, up front
    const int scene = (BATCH && active) ? A.scene[s] : 0;
    const float4 pi = active ? A.pos[s] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 vi = active ? A.vel[s] : make_float4(0.f, 0.f, 0.f, 1.f);
    const int id = active ? A.ids[s] : 0;
    const int cnt_raw = active ? A.nbr_cnt[s] : 0;
    const float4 xb = (active && exact) ? A.xbuild[s] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int hcnt_in = (HIST && active) ? A.hcnt_in[s] : 0;
    const DevParams& P = BATCH ? A.scene_params[scene] : P0;
    const bool frozen = BATCH && active && P.frozen;
    const bool work = active && !frozen;
    const float3 pos = make_float3(pi.x, pi.y, pi.z);
    const float3 vel = make_float3(vi.x, vi.y, vi.z);
    const float ri = pi.w, mi = vi.w;
    float3 f = make_float3(0.f, 0.f, 0.f);
    HistRow h;
    h.in = A.hist_in + static_cast<int64_t>(id) * kHistCap;
    h.in_count = hcnt_in;
    h.out = A.hist_out + static_cast<int64_t>(id) * kHistCap;
    h.out_count = 0;
    if (work) wall_forces<HIST>(P, pos, vel, ri, mi, f, h, A.counters);
    const float3 f_walls = f;
    const int out_walls = HIST ? h.out_count : 0;
    W.pos[lane] = pi;
    W.vel[lane] = vi;
    W.id[lane] = id;
    W.hin[lane] = hcnt_in;
    W.outw[lane] = out_walls;
    W.scene[lane] = scene;
    const float cut = contact_cutoff_sq(ri, P.rmax);
    int cx = 0, cy = 0, cz = 0;
    if (work) cell_coords(P, pi.x, pi.y, pi.z, cx, cy, cz);
    const bool listed = work && cnt_raw <= kNbrCap;
    const int cnt = listed ? cnt_raw : 0;
    const int rounds = __reduce_max_sync(0xffffffffu, cnt);
    int q = 0, my_count = 0, bstart = 0;
    bool reorder = false;
    unsigned long long last = 0ull;
    for (int e = 0; e < rounds; ++e) {
        bool hit = false;
        int j = 0;
        if (e < cnt) {
            j = __ldg(&A.nbr[static_cast<int64_t>(e) * n + s]);
            const float4 pj = __ldg(&A.pos[j]);
            float3 d;
            const float ns = pair_norm_sq(pi, pj, d);
            if (!(ns > cut)) {
                const float dist = pair_dist(sqrtf(ns), ri, pj.w);
                if (dist < 0.f) {
                    hit = true;
                    const unsigned long long key = visit_key(P, cx, cy, cz, pj, __ldg(&A.ids[j]));
                    if (key < last) reorder = true;
                    last = key;
                }
            }
        }
        const unsigned b = __ballot_sync(0xffffffffu, hit);
        const int add = __popc(b);
        if (q + add > kCoopCap) {
            coop_flush<HIST, BATCH>(P0, A, W, q, lane, my_count, bstart, reorder, f);
            q = 0;
        }
        if (hit) {
            const int at = q + __popc(b & ((1u << lane) - 1u));
            W.qj[at] = j;
            W.qg[at] = static_cast<unsigned char>(lane);
            W.qr[at] = static_cast<unsigned char>(my_count);
            ++my_count;
        }
        q += add;
    }
    if (rounds > 0) coop_flush<HIST, BATCH>(P0, A, W, q, lane, my_count, bstart, reorder, f);
    if (work) {
        if (!listed) {
            // list overflow: this step built the lists, so the run table is fresh
            h.out_count = out_walls;
            list_contacts_table<HIST>(P, A, s, pi, vel, mi, cut, cx, cy, cz, f, h);
        } else if (reorder) {
            // a cell crossing re-ordered this grain's contacts: redo them in canonical order
            f = f_walls;
            h.out_count = out_walls;
            list_contacts_sorted<HIST>(P, A, s, n, cnt, pi, vel, mi, cut, cx, cy, cz, f, h);
        } else if (HIST) {
            h.out_count = min(out_walls + my_count, kHistCap);
            if (out_walls + my_count > kHistCap)
                atomicAdd(&A.counters[kCntHistOverflow],
                          static_cast<unsigned long long>(out_walls + my_count - kHistCap));
        }
        if (HIST) A.hcnt_out[s] = h.out_count;
        const float3 a = make_float3(f.x / mi, f.y / mi, f.z / mi);
        const float3 v1 = make_float3(fmaf(P.dt, a.x, vel.x), fmaf(P.dt, a.y, vel.y),
                                      fmaf(P.dt, a.z, vel.z));
        const float3 x1 = make_float3(fmaf(P.dt, v1.x, pos.x), fmaf(P.dt, v1.y, pos.y),
                                      fmaf(P.dt, v1.z, pos.z));
        A.pos_out[s] = make_float4(x1.x, x1.y, x1.z, ri);
        A.vel_out[s] = make_float4(v1.x, v1.y, v1.z, mi);
        if (order_out) {
            A.ids_out[s] = id;
            if (BATCH) A.scene_out[s] = scene;
        }
        A.acc_out[s] = make_float4(a.x, a.y, a.z, 0.f);
        if (exact) disp_bits = max(disp_bits, disp_sq_bits(x1, xb));
        step_bits = max(step_bits, disp_sq_bits(x1, pos));
    } else if (frozen) {
        A.pos_out[s] = pi;
        A.vel_out[s] = vi;
        if (order_out) {
            A.ids_out[s] = id;
            A.scene_out[s] = scene;
        }
        A.acc_out[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (HIST) A.hcnt_out[s] = 0;
    }
}

// Grid-stride over warps of 32 slots (one wave for the fused build decision).
template <bool HIST, bool BATCH>
__global__ void __launch_bounds__(kBlock, 4)
k_force_list_coop(DevParams P0, ListArgs A) {
    __shared__ CoopWarp warps[kCoopWarps];
    CoopWarp& W = warps[threadIdx.x >> 5];
    const bool exact = A.list_ctrl[kLcExact] != 0u;
    const bool order_out = A.list_ctrl[kLcDecision] != 0u;  // first step after a build
    uint32_t disp_bits = 0u, step_bits = 0u;
    for (int base = blockIdx.x * blockDim.x; base < P0.n; base += gridDim.x * blockDim.x)
        coop_slot<HIST, BATCH>(P0, A, W, base + threadIdx.x, exact, order_out, disp_bits,
                               step_bits);
    list_disp_report<false>(A.list_ctrl, exact, disp_bits, step_bits);
    list_tail_decide(A);
}

__global__ void __launch_bounds__(kBlock)
k_list_length(int n, const int* __restrict__ cnt, unsigned long long* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long v = s < n ? static_cast<unsigned long long>(min(cnt[s], kNbrCap + 1)) : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(out, v);
}

}  // namespace

void launch_list_decide(uint32_t* list_ctrl, float thr, bool always_exact,
                        unsigned long long* counters,
                        bool use_cond, cudaGraphConditionalHandle cond, cudaStream_t st) {
    k_list_decide<<<1, 32, 0, st>>>(list_ctrl, thr, always_exact ? 1 : 0, counters,
                                    use_cond ? 1 : 0, cond);
}

void launch_list_build(const DevParams& P, SceneTab T, const float4* pos, const int2* table,
                       int* nbr, int* nbr_cnt, float4* xbuild, uint32_t* list_ctrl,
                       const ListCopy& cp, Skip skip, unsigned long long* counters, bool tiled,
                       cudaStream_t st) {
    if (tiled && !T.params) {
        k_list_build_tiled<<<blocks_for(P.n), kBlock, 0, st>>>(P, pos, table, nbr, nbr_cnt, xbuild,
                                                               list_ctrl, cp, skip, counters);
        return;
    }
    if (T.params)
        k_list_build<true><<<blocks_for(P.n), kBlock, 0, st>>>(P, T, pos, table, nbr, nbr_cnt,
                                                                xbuild, list_ctrl, cp, skip);
    else
        k_list_build<false><<<blocks_for(P.n), kBlock, 0, st>>>(P, T, pos, table, nbr, nbr_cnt,
                                                                 xbuild, list_ctrl, cp, skip);
}

void launch_list_copy(int n, const float4* pos, const float4* vel, const int* ids,
                      const int* hcnt, const int* scene, float4* pos_out, float4* vel_out,
                      int* ids_out, int* hcnt_out, int* scene_out, Skip skip, cudaStream_t st) {
    k_list_copy<<<blocks_for(n), kBlock, 0, st>>>(n, pos, vel, ids, hcnt, scene, pos_out,
                                                  vel_out, ids_out, hcnt_out, scene_out, skip);
}

// Blocks of one full wave of a kernel at `block` threads (a multiple of 32 up to 256):
// the SM count times the resident blocks per SM, cached per kernel, device and block
// size (devices beyond the first 64 query each time).
template <auto Kernel>
int one_wave(int block) {
    constexpr int kDevs = 64;
    static int cache[kDevs][9] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int local = 0;
    int& occ = (dev >= 0 && dev < kDevs) ? cache[dev][(block / 32) % 9] : local;
    if (occ == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, Kernel, block, 0);
        occ = occ < 1 ? 1 : occ;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms * occ;
}

template <bool HIST, bool BATCH, int MINB>
void force_list_staged(const DevParams& P, const ListArgs& a, cudaStream_t st) {
    // persistent: as many blocks as fit at once, at most one warp per tile
    const int tiles = (P.n + kStageTile - 1) / kStageTile;
    const int want = (tiles + kStageWarps - 1) / kStageWarps;
    const int nb = std::min(want, one_wave<k_force_list_staged<HIST, BATCH, MINB>>(kBlock));
    k_force_list_staged<HIST, BATCH, MINB><<<nb < 1 ? 1 : nb, kBlock, 0, st>>>(P, a);
}

template <bool HIST, bool BATCH, int MINB, bool PICARD>
void force_list_launch(const DevParams& P, const ListArgs& a, cudaStream_t st, int block) {
    int nb = blocks_for(P.n, block);
    // semi-implicit Euler: one wave (grid-stride), so the fused build decision's
    // per-block wait happens once per resident block
    if (!PICARD) nb = std::min(nb, one_wave<k_force_list<HIST, BATCH, MINB, PICARD>>(block));
    k_force_list<HIST, BATCH, MINB, PICARD><<<nb, block, 0, st>>>(P, a);
}

template <int MINB, bool PICARD>
void force_list_variant(const DevParams& P, const ListArgs& a, cudaStream_t st, int block) {
    const bool batch = a.scene_params != nullptr;
    if (P.history) {
        if (batch) force_list_launch<true, true, MINB, PICARD>(P, a, st, block);
        else force_list_launch<true, false, MINB, PICARD>(P, a, st, block);
    } else {
        if (batch) force_list_launch<false, true, MINB, PICARD>(P, a, st, block);
        else force_list_launch<false, false, MINB, PICARD>(P, a, st, block);
    }
}

void launch_list_finalize(int n, const int* picard_used, const float4* xpos,
                          const float4* xvel, float4* pos, float4* vel, cudaStream_t st) {
    k_list_finalize<<<blocks_for(n), kBlock, 0, st>>>(n, picard_used, xpos, xvel, pos, vel);
}

void launch_list_picard_check(uint32_t* list_ctrl, unsigned long long* counters, bool use_cond,
                              cudaGraphConditionalHandle cond, cudaStream_t st) {
    k_list_picard_check<<<1, 32, 0, st>>>(list_ctrl, counters, use_cond ? 1 : 0, cond);
}

void launch_force_list(const DevParams& P, const ListArgs& a, cudaStream_t st, int block,
                       int min_blocks, bool picard) {
    if (picard) {
        // the per-lane kernel (the cooperative one has no Picard form)
        if (min_blocks == 4) force_list_variant<4, true>(P, a, st, block == 0 ? kBlock : block);
        else force_list_variant<5, true>(P, a, st, block);
        return;
    }
    if (min_blocks == 1 || min_blocks == 2) {
        // bulk-staged persistent kernel (kBlock threads; 1: 48 registers, 2: 64)
        const bool batch = a.scene_params != nullptr;
        const bool r64 = min_blocks == 2;
        if (P.history) {
            if (batch) r64 ? force_list_staged<true, true, 4>(P, a, st) : force_list_staged<true, true, 5>(P, a, st);
            else r64 ? force_list_staged<true, false, 4>(P, a, st) : force_list_staged<true, false, 5>(P, a, st);
        } else {
            if (batch) r64 ? force_list_staged<false, true, 4>(P, a, st) : force_list_staged<false, true, 5>(P, a, st);
            else r64 ? force_list_staged<false, false, 4>(P, a, st) : force_list_staged<false, false, 5>(P, a, st);
        }
        return;
    }
    if (min_blocks == 0) {
        // warp-cooperative kernel: its shared queues are sized for kBlock threads; one
        // wave, grid-stride
        const int nb = blocks_for(P.n, kBlock);
        const bool batch = a.scene_params != nullptr;
        if (P.history) {
            if (batch) {
                k_force_list_coop<true, true><<<std::min(nb, one_wave<k_force_list_coop<true, true>>(kBlock)), kBlock, 0, st>>>(P, a);
            } else {
                k_force_list_coop<true, false><<<std::min(nb, one_wave<k_force_list_coop<true, false>>(kBlock)), kBlock, 0, st>>>(P, a);
            }
        } else {
            if (batch) {
                k_force_list_coop<false, true><<<std::min(nb, one_wave<k_force_list_coop<false, true>>(kBlock)), kBlock, 0, st>>>(P, a);
            } else {
                k_force_list_coop<false, false><<<std::min(nb, one_wave<k_force_list_coop<false, false>>(kBlock)), kBlock, 0, st>>>(P, a);
            }
        }
    } else if (min_blocks == 4) {
        force_list_variant<4, false>(P, a, st, block);
    } else {
        force_list_variant<5, false>(P, a, st, block);
    }
}

void launch_list_length(int n, const int* nbr_cnt, unsigned long long* out, cudaStream_t st) {
    k_list_length<<<blocks_for(n), kBlock, 0, st>>>(n, nbr_cnt, out);
}

}  // namespace wd
