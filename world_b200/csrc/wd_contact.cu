// wd_contact.cu -- fused contact force + integrator, and the FP64 energy reduction.
//
// One thread per grain in (cell, id) order. The thread walks the 9 neighbor
// columns of its cell; the three z-cells of each column are consecutive runs of the
// sorted arrays, so the candidates of a column are one contiguous slot range read
// straight from the sorted SoA (float4 position+radius, float4 velocity+mass). Each
// thread sums only its own force: no force atomics and a fixed summation order
// (stencil order, ids ascending inside a cell), hence bit-reproducible steps.
//
// Physics per contact: reference src/compute_rhs_kernel.cu:81-212 (gravity, six
// walls, clamped linear spring, normal dashpot from restitution, Coulomb-capped
// friction), generalised to per-grain radius and mass, with the tangential spring
// and its per-pair history as an option. The integrator runs in the epilogue:
// semi-implicit Euler (src/semi_implicit_euler_kernel.cu:4-16) or one backward
// Euler / Picard update from the step-start snapshot
// (src/backward_euler_picard_kernel.cu:4-17).
#include "wd_kernels.h"

namespace wd {

namespace {

__device__ __forceinline__ bool skipped(const Skip& s) {
    return s.prev_res != nullptr && s.tol > 0.f && __uint_as_float(*s.prev_res) < s.tol;
}

// 5 resident blocks of 256 per SM (<= 51 registers): the candidate loop is
// latency-bound, so occupancy matters more than the few values the rarely taken
// contact path may keep in local memory.
template <bool HIST, bool PICARD, bool BATCH>
__global__ void __launch_bounds__(kBlock, 5)
k_force(DevParams P0, ForceArgs A, Skip skip) {
    if (PICARD && skipped(skip)) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t res_bits = 0u;
    if (s < P0.n) {
        const int scene = BATCH ? A.scene[s] : 0;
        const DevParams& P = BATCH ? A.scene_params[scene] : P0;
        const float4 pi = A.pos[s];
        const float4 vi = A.vel[s];
        const int id = A.ids[s];
        if (BATCH && P.frozen) {
            // a stopped scene (a diverged rollout): state copied through unchanged
            A.pos_out[s] = pi;
            A.vel_out[s] = vi;
            A.ids_out[s] = id;
            A.scene_out[s] = scene;
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
                h.in_count = A.hcnt_in[s];
                h.out = A.hist_out + static_cast<int64_t>(id) * kHistCap;
                h.out_count = 0;
            }
            wall_forces<HIST>(P, pos, vel, ri, mi, f, h, A.counters);

            const float cut = contact_cutoff_sq(ri, P.rmax);
            int cx, cy, cz;
            cell_coords(P, pi.x, pi.y, pi.z, cx, cy, cz);
            for (int dx = -1; dx <= 1; ++dx) {
                const int nx = cx + dx;
                if (nx < 0 || nx >= P.grid[0]) continue;
                int lo[3], hi[3];
                row_ranges(P, A.table, nx, cy, cz, lo, hi);
    #pragma unroll
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
            if (HIST) A.hcnt_out[s] = h.out_count;

            const float3 a = make_float3(f.x / mi, f.y / mi, f.z / mi);
            float3 v1, x1;
            if (!PICARD) {
                v1 = make_float3(fmaf(P.dt, a.x, vel.x), fmaf(P.dt, a.y, vel.y),
                                 fmaf(P.dt, a.z, vel.z));
                x1 = make_float3(fmaf(P.dt, v1.x, pos.x), fmaf(P.dt, v1.y, pos.y),
                                 fmaf(P.dt, v1.z, pos.z));
            } else {
                const float4 xn = A.npos[s], vn = A.nvel[s];
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
            A.ids_out[s] = id;
            if (BATCH) A.scene_out[s] = scene;
            A.acc_out[s] = make_float4(a.x, a.y, a.z, 0.f);
        }
    }
    if (PICARD) {
        // max of non-negative float bits (NaN above +inf, so it is kept)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            res_bits = max(res_bits, __shfl_xor_sync(0xffffffffu, res_bits, o));
        if ((threadIdx.x & 31) == 0 && res_bits != 0u) atomicMax(A.res_slot, res_bits);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            *A.picard_used = A.iter + 1;
            A.counters[kCntPicardIters] += 1ull;
        }
    }
}

// Deterministic block sum of doubles (fixed tree for a fixed launch shape).
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double ws[kBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) ws[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (warp == 0) {
        t = lane < kBlock / 32 ? ws[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    return t;  // valid in thread 0
}

// reference src/energy_kernel.cu:30-80: kinetic + gravity + wall and pair elastic
// energy (pairs counted from the lower grain id), plus the tangential spring energy
// 1/2 k_t |xi|^2 of stored contacts in history mode. Terms in FP32 as the
// reference, the grain's sum in FP64, written per sorted position for the segmented
// reduction below.
template <bool HIST, bool BATCH>
__global__ void __launch_bounds__(kBlock)
k_energy(DevParams P0, SceneTab T, const float4* __restrict__ pos, const float4* __restrict__ vel,
         const int* __restrict__ ids, const int2* __restrict__ table,
         const float4* __restrict__ hist, const int* __restrict__ hcnt,
         const int* __restrict__ src, double* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P0.n) return;
    const DevParams& P = scene_params<BATCH>(P0, T, s);
    double e = 0.0;
    const float4 pi = pos[s], vi = vel[s];
    const int id = ids[s];
    const float m = vi.w, ri = pi.w;
    const float F = P.max_force, k = P.k_n, cd = P.clamp_overlap;
    float ss = vi.x * vi.x;
    ss = fmaf(vi.y, vi.y, ss);
    ss = fmaf(vi.z, vi.z, ss);
    e += static_cast<double>(0.5f * m * ss);
    e += static_cast<double>((m * P.gravity) * (pi.z - P.wall_lo[2]));
    const float p3[3] = {pi.x, pi.y, pi.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        e += static_cast<double>(contact_energy(ri - (p3[a] - P.wall_lo[a]), cd, F, k));
        e += static_cast<double>(contact_energy(ri - (P.wall_hi[a] - p3[a]), cd, F, k));
    }
    int cx, cy, cz;
    cell_coords(P, pi.x, pi.y, pi.z, cx, cy, cz);
    for (int dx = -1; dx <= 1; ++dx) {
        const int nx = cx + dx;
        if (nx < 0 || nx >= P.grid[0]) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int ny = cy + dy;
            if (ny < 0 || ny >= P.grid[1]) continue;
            int lo, hi;
            column_range(P, table, nx, ny, cz, lo, hi);
            for (int j = lo; j < hi; ++j) {
                if (j == s || ids[j] <= id) continue;
                const float4 pj = pos[j];
                float3 d;
                const float ns = pair_norm_sq(pi, pj, d);
                if (!maybe_contact(ns, ri, pj.w)) continue;
                e += static_cast<double>(contact_energy((ri + pj.w) - sqrtf(ns), cd, F, k));
            }
        }
    }
    if (HIST) {
        const int c = hcnt[src[s]];
        for (int q = 0; q < c; ++q) {
            const float4 x = hist[static_cast<int64_t>(id) * kHistCap + q];
            const int partner = __float_as_int(x.w);
            if (partner >= 0 && partner <= id) continue;
            float xs = x.x * x.x;
            xs = fmaf(x.y, x.y, xs);
            xs = fmaf(x.z, x.z, xs);
            e += static_cast<double>(0.5f * P.k_t * xs);
        }
    }
    out[s] = e;
}

// Segmented sums, step 1: one block per 256-grain chunk of a scene's segment (chunks
// are aligned to the segment start, so a scene reduces the same way alone or in a
// batch). comps values per grain, component-major: v[c * n + slot].
__global__ void __launch_bounds__(kBlock)
k_segment_chunks(const double* __restrict__ v, int n, int comps, const int* __restrict__ seg,
                 const int* __restrict__ chunk_base, int scenes, double* __restrict__ partials,
                 int total_chunks) {
    const int b = blockIdx.x;
    int lo = 0, hi = scenes;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (chunk_base[mid] <= b) lo = mid; else hi = mid;
    }
    const int sc = lo;
    const int first = seg[sc] + (b - chunk_base[sc]) * kBlock;
    const int i = first + static_cast<int>(threadIdx.x);
    for (int c = 0; c < comps; ++c) {
        const double x = i < seg[sc + 1] ? v[static_cast<int64_t>(c) * n + i] : 0.0;
        const double t = block_sum(x);
        if (threadIdx.x == 0) partials[static_cast<int64_t>(c) * total_chunks + b] = t;
    }
}

// Segmented sums, step 2: one block per scene sums its chunk partials in a fixed order.
__global__ void __launch_bounds__(kBlock)
k_segment_finish(const double* __restrict__ partials, const int* __restrict__ chunk_base,
                 int comps, int total_chunks, double* __restrict__ out) {
    const int sc = blockIdx.x;
    const int c0 = chunk_base[sc], c1 = chunk_base[sc + 1];
    for (int c = 0; c < comps; ++c) {
        double x = 0.0;
        for (int i = c0 + static_cast<int>(threadIdx.x); i < c1; i += blockDim.x)
            x += partials[static_cast<int64_t>(c) * total_chunks + i];
        const double t = block_sum(x);
        if (threadIdx.x == 0) out[sc * comps + c] = t;
    }
}

__global__ void __launch_bounds__(kBlock)
k_momentum(int n, const float4* __restrict__ vel, double* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 v = vel[s];
    const double m = v.w;
    out[s] = m * v.x;
    out[static_cast<int64_t>(n) + s] = m * v.y;
    out[2 * static_cast<int64_t>(n) + s] = m * v.z;
}

// reference src/particle_dynamics.cu:328-344: sqrt(ax^2 + ay^2 + az^2), unfused.
__global__ void __launch_bounds__(kBlock)
k_max_accel(int n, const float4* __restrict__ acc, unsigned long long* __restrict__ counters) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t b = 0u;
    if (s < n) {
        const float4 a = acc[s];
        float sq = 0.f;
        sq = sq + a.x * a.x;
        sq = sq + a.y * a.y;
        sq = sq + a.z * a.z;
        b = __float_as_uint(sqrtf(sq));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    if ((threadIdx.x & 31) == 0 && b)
        atomicMax(reinterpret_cast<unsigned int*>(&counters[kCntMaxAccel]), b);
}

// reference src/particle_dynamics.cu:311-325: finite and inside the domain box.
template <bool BATCH>
__global__ void __launch_bounds__(kBlock)
k_stability(DevParams P0, SceneTab T, const float4* __restrict__ pos,
            unsigned long long* __restrict__ counters, int* __restrict__ scene_unstable) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P0.n) return;
    const DevParams& P = scene_params<BATCH>(P0, T, s);
    const float4 p = pos[s];
    const float q[3] = {p.x, p.y, p.z};
    bool bad = false;
#pragma unroll
    for (int a = 0; a < 3; ++a) bad |= !isfinite(q[a]) || q[a] < P.lo[a] || q[a] > P.hi[a];
    if (bad) {
        atomicOr(&counters[kCntUnstable], 1ull);
        if (BATCH && scene_unstable) scene_unstable[T.scene[s]] = 1;
    }
}

}  // namespace

void launch_force(const DevParams& P, const ForceArgs& a, bool picard, Skip skip,
                  cudaStream_t st, int block) {
    const int nb = blocks_for(P.n, block);
    const bool batch = a.scene_params != nullptr;
#define WD_FORCE(H, PI, B) k_force<H, PI, B><<<nb, block, 0, st>>>(P, a, skip)
    if (P.history) {
        if (picard) { if (batch) WD_FORCE(true, true, true); else WD_FORCE(true, true, false); }
        else { if (batch) WD_FORCE(true, false, true); else WD_FORCE(true, false, false); }
    } else {
        if (picard) { if (batch) WD_FORCE(false, true, true); else WD_FORCE(false, true, false); }
        else { if (batch) WD_FORCE(false, false, true); else WD_FORCE(false, false, false); }
    }
#undef WD_FORCE
}

int reduction_blocks(int n) { return blocks_for(n > 0 ? n : 1); }

void launch_segment_sums(const double* values, int n, int comps, const Segments& g,
                         double* partials, double* out, cudaStream_t st) {
    k_segment_chunks<<<g.total_chunks, kBlock, 0, st>>>(values, n, comps, g.seg, g.chunk_base,
                                                        g.scenes, partials, g.total_chunks);
    k_segment_finish<<<g.scenes, kBlock, 0, st>>>(partials, g.chunk_base, comps, g.total_chunks, out);
}

void launch_energy(const DevParams& P, SceneTab T, const float4* pos, const float4* vel,
                   const int* ids, const int2* table, const float4* hist, const int* hcnt,
                   const int* src, const Segments& g, double* per_grain, double* partials,
                   double* out, cudaStream_t st) {
    const int nb = reduction_blocks(P.n);
    const bool batch = T.params != nullptr;
    if (P.history) {
        if (batch) k_energy<true, true><<<nb, kBlock, 0, st>>>(P, T, pos, vel, ids, table, hist, hcnt, src, per_grain);
        else k_energy<true, false><<<nb, kBlock, 0, st>>>(P, T, pos, vel, ids, table, hist, hcnt, src, per_grain);
    } else {
        if (batch) k_energy<false, true><<<nb, kBlock, 0, st>>>(P, T, pos, vel, ids, table, hist, hcnt, src, per_grain);
        else k_energy<false, false><<<nb, kBlock, 0, st>>>(P, T, pos, vel, ids, table, hist, hcnt, src, per_grain);
    }
    launch_segment_sums(per_grain, P.n, 1, g, partials, out, st);
}

void launch_momentum(int n, const float4* vel, const Segments& g, double* per_grain,
                     double* partials, double* out3, cudaStream_t st) {
    k_momentum<<<reduction_blocks(n), kBlock, 0, st>>>(n, vel, per_grain);
    launch_segment_sums(per_grain, n, 3, g, partials, out3, st);
}

void launch_max_accel(int n, const float4* acc, unsigned long long* counters,
                      cudaStream_t st) {
    k_max_accel<<<blocks_for(n), kBlock, 0, st>>>(n, acc, counters);
}

void launch_stability(const DevParams& P, SceneTab T, const float4* pos,
                      unsigned long long* counters, int* scene_unstable, cudaStream_t st) {
    if (T.params)
        k_stability<true><<<blocks_for(P.n), kBlock, 0, st>>>(P, T, pos, counters, scene_unstable);
    else
        k_stability<false><<<blocks_for(P.n), kBlock, 0, st>>>(P, T, pos, counters, nullptr);
}

}  // namespace wd
