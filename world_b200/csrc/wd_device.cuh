// wd_device.cuh -- parameters and per-contact arithmetic shared by the sm_100a kernels.
//
// The library is compiled with -fmad=false: the only fused multiply-adds are the
// explicit fmaf() calls below, placed where nvcc contracts the reference's own
// expressions (e.g. `force[a] += f_pair * normal[a]`). Division and sqrt are the
// IEEE-rounded ones (-prec-div, -prec-sqrt), so a CPU restatement with the same
// operation order reproduces these kernels bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace wd {

constexpr int kHistCap = 24;          // tangential-history slots per grain
constexpr uint32_t kNoKey = 0xFFFFFFFFu;
constexpr int kNbrCap = 48;            // Verlet-list entries per grain

// Lifetime counters kept on the device.
enum Counter : int {
    kCntGridOverflow = 0,   // (cell, search) incidents above particles_per_cell
    kCntHistOverflow = 1,   // contacts without a free history slot
    kCntUnstable = 2,       // scratch for is_stable
    kCntMaxAccel = 3,       // scratch for compute_max_acceleration (float bits)
    kCntRadixSearches = 4,  // searches that took the full radix-sort path
    kCntListBuilds = 5,     // Verlet-list builds
    kCntPicardRedos = 6,    // list-mode Picard steps redone with the per-iteration search
    kCntPicardIters = 7,    // Picard iterations executed (contact-kernel launches that ran)
    kCntListExact = 8,      // list steps whose contact kernel read the build positions
    kCntStageTimeout = 9,   // bulk-staged contact kernel: stages that never completed
    kCntListResort = 10,    // list contact kernels: grains whose contacts were re-ordered
    kCntLaunchFail = 11,    // device-side launches of a list build's graphs that failed
    kNumCounters = 12,
};

// Everything a step kernel needs, passed by value (baked into the captured graph).
struct DevParams {
    float lo[3], hi[3];        // domain box
    int grid[3];               // collision grid
    float inv_len[3];          // 1 / (hi - lo) rounded to float, per axis (cell_axis)
    float cell_err[3];         // (grid + 1) * 2^-20: cell_axis's fast-path margin
    float cell_len[3];         // cell width (hi - lo) / grid, rounded down
    float cell_min;            // the smallest of the three
    int ppc;                   // particles_per_cell
    float gravity;
    float max_force;           // clamp (+inf: none)
    float k_n, k_t;
    float restitution, ln_e, damp_den;
    float mu;
    float dt;
    float wall_lo[3], wall_hi[3];
    float clamp_overlap;
    float picard_tol;
    float rmax;                // largest grain radius (conservative candidate cutoff)
    int history;
    int n;                     // grains (of the scene, in a scene's own entry)
    uint32_t cell_base;        // first cell key of the scene (0 for a single scene)
    int dgrid[3];              // CIC nodes per axis
    int node_base;             // first CIC node of the scene in the batch's field
    int frozen;                // batch only: the step leaves this scene's grains as they are
    float skin;                // Verlet-list skin (0: search every step)
};

// Scenes of a batch: per-scene parameters and the scene of each slot of the arrays a
// kernel reads. A single scene passes params == nullptr and uses the kernel's own
// DevParams; batched kernels (template flag BATCH) look each grain's scene up.
struct SceneTab {
    const DevParams* params;
    const int* scene;
};

template <bool BATCH>
__device__ __forceinline__ const DevParams& scene_params(const DevParams& P, const SceneTab& T,
                                                         int slot) {
    if (BATCH) return T.params[T.scene[slot]];
    return P;
}

// reference src/find_neighbors_kernel.cu:11-22. __float2int_rz is cvt.rzi.s32.f32,
// the conversion static_cast<int>(float) compiles to.
__device__ __forceinline__ int cell_axis_exact(float x, float lo, float hi, int g) {
    const float t = (x - lo) / (hi - lo) * static_cast<float>(g);
    return min(g - 1, max(0, __float2int_rz(t)));
}

// The same integer without the division where that is provably safe. With u = x - lo
// (the same rounded difference), t' = (u * inv) * g, inv = 1/(hi - lo) rounded, differs
// from the reference's t = (u / (hi - lo)) * g by at most 5 roundings of 2^-24 relative:
// below (g + 1) 2^-21.4 for t' in [-0.5, g + 0.5), a third of `err` = (g + 1) 2^-20. So
// where t' is farther than err from every integer, trunc(t) and floor(t') agree after
// the clamp to [0, g - 1] (t' < -0.5 and t' >= g + 0.5 clamp alike); elsewhere, and
// for NaN, the exact expression decides. About 2 err of all values take it.
__device__ __forceinline__ int cell_axis(float x, float lo, float hi, int g, float inv, float err) {
    const float t = ((x - lo) * inv) * static_cast<float>(g);
    if (t >= -0.5f && t < static_cast<float>(g) + 0.5f) {
        const float k = floorf(t);
        const float f = t - k;
        if (f >= err && f <= 1.f - err) return min(g - 1, max(0, static_cast<int>(k)));
    } else if (t < -0.5f) {
        return 0;
    } else if (t >= static_cast<float>(g) + 0.5f) {
        return g - 1;
    }
    return cell_axis_exact(x, lo, hi, g);
}

__device__ __forceinline__ void cell_coords(const DevParams& P, float x, float y, float z,
                                            int& cx, int& cy, int& cz) {
    cx = cell_axis(x, P.lo[0], P.hi[0], P.grid[0], P.inv_len[0], P.cell_err[0]);
    cy = cell_axis(y, P.lo[1], P.hi[1], P.grid[1], P.inv_len[1], P.cell_err[1]);
    cz = cell_axis(z, P.lo[2], P.hi[2], P.grid[2], P.inv_len[2], P.cell_err[2]);
}

// reference src/find_neighbors_kernel.cu:27-30 (x slowest, z fastest).
__device__ __forceinline__ uint32_t flat_cell(const DevParams& P, int x, int y, int z) {
    return (static_cast<uint32_t>(x) * static_cast<uint32_t>(P.grid[1]) +
            static_cast<uint32_t>(y)) * static_cast<uint32_t>(P.grid[2]) +
           static_cast<uint32_t>(z);
}

// reference src/compute_rhs_kernel.cu:41-47 with logf(e) and the denominator
// sqrtf(pi^2 + ln^2 e) computed once on the host.
__device__ __forceinline__ float damping(const DevParams& P, float m) {
    if (P.restitution <= 0.f) return 2.f * sqrtf(P.k_n * m);
    if (P.restitution >= 1.f) return 0.f;
    return ((-2.f * sqrtf(m * P.k_n)) * P.ln_e) / P.damp_den;
}

// reference src/compute_rhs_kernel.cu:66-78: the friction force is -term (zero below
// the 1e-8 m/s cutoff; f - 0 is f exactly).
__device__ __forceinline__ float3 viscous_term(float3 vt, float limit, float c) {
    float vt_sq = vt.x * vt.x;
    vt_sq = fmaf(vt.y, vt.y, vt_sq);
    vt_sq = fmaf(vt.z, vt.z, vt_sq);
    const float v = sqrtf(vt_sq);
    if (v < 1e-8f) return make_float3(0.f, 0.f, 0.f);
    const float mag = fminf(limit, c * v);
    return make_float3((mag * vt.x) / v, (mag * vt.y) / v, (mag * vt.z) / v);
}

__device__ __forceinline__ void viscous_friction(float3& f, float3 vt, float limit, float c) {
    const float3 t = viscous_term(vt, limit, c);
    f.x = f.x - t.x;
    f.y = f.y - t.y;
    f.z = f.z - t.z;
}

// Tangential spring with per-pair history (Cundall-Strack), capped at mu |F_n| with
// the spring reset to the cap on slip. The stored displacement is rotated onto the
// current tangent plane, advanced by v_t dt, and F_t = -k_t xi. Extension: the
// reference's friction is the viscous form above.
struct HistRow {
    const float4* in;   // old row of this grain (kHistCap entries)
    int in_count;
    float4* out;        // new row
    int out_count;
    int cursor = 0;     // where the next search of the old row starts
};

// Stored spring of `partner` in a row (zero if the contact is new).
__device__ __forceinline__ float3 find_spring(const float4* row, int count, int partner) {
    for (int k = 0; k < count; ++k) {
        const float4 e = row[k];
        if (__float_as_int(e.w) == partner) return make_float3(e.x, e.y, e.z);
    }
    return make_float3(0.f, 0.f, 0.f);
}

// The same search started at the entry after the last match, wrapping around. A row
// holds each partner at most once, so the entry found is the one above; the row was
// written in the order the contacts were visited, and the next step visits the same
// contacts in the same order, so a lasting contact is found at its first probe.
__device__ __forceinline__ float3 find_spring(HistRow& h, int partner) {
    int k = h.cursor;
    for (int t = 0; t < h.in_count; ++t, ++k) {
        if (k >= h.in_count) k = 0;
        const float4 e = h.in[k];
        if (__float_as_int(e.w) == partner) {
            h.cursor = k + 1;
            return make_float3(e.x, e.y, e.z);
        }
    }
    return make_float3(0.f, 0.f, 0.f);
}

// The spring's step: rotate onto the tangent plane, advance by v_t dt, cap at `limit`.
// Returns the tangential force; xi becomes the new spring.
__device__ __forceinline__ float3 spring_step(const DevParams& P, float3 vt, float3 nrm,
                                              float limit, float3& xi) {
    float xn = xi.x * nrm.x;
    xn = fmaf(xi.y, nrm.y, xn);
    xn = fmaf(xi.z, nrm.z, xn);
    xi.x = fmaf(-xn, nrm.x, xi.x);
    xi.y = fmaf(-xn, nrm.y, xi.y);
    xi.z = fmaf(-xn, nrm.z, xi.z);
    xi.x = fmaf(P.dt, vt.x, xi.x);
    xi.y = fmaf(P.dt, vt.y, xi.y);
    xi.z = fmaf(P.dt, vt.z, xi.z);
    float3 ft = make_float3(-P.k_t * xi.x, -P.k_t * xi.y, -P.k_t * xi.z);
    float ft_sq = ft.x * ft.x;
    ft_sq = fmaf(ft.y, ft.y, ft_sq);
    ft_sq = fmaf(ft.z, ft.z, ft_sq);
    if (ft_sq > limit * limit) {
        const float s = limit / sqrtf(ft_sq);
        ft.x = ft.x * s; ft.y = ft.y * s; ft.z = ft.z * s;
        xi.x = xi.x * s; xi.y = xi.y * s; xi.z = xi.z * s;
    }
    return ft;
}

__device__ __forceinline__ void spring_friction(const DevParams& P, float3& f, float3 vt,
                                                float3 nrm, float limit, int partner,
                                                HistRow& h, unsigned long long* counters) {
    float3 xi = find_spring(h, partner);
    const float3 ft = spring_step(P, vt, nrm, limit, xi);
    f.x = f.x + ft.x;
    f.y = f.y + ft.y;
    f.z = f.z + ft.z;
    if (h.out_count < kHistCap) {
        h.out[h.out_count] = make_float4(xi.x, xi.y, xi.z, __int_as_float(partner));
        ++h.out_count;
    } else {
        atomicAdd(&counters[kCntHistOverflow], 1ull);
    }
}

// Gravity and the six walls: reference src/compute_rhs_kernel.cu:114-146.
template <bool HIST>
__device__ __forceinline__ void wall_forces(const DevParams& P, float3 pos, float3 vel,
                                            float ri, float mi, float3& f, HistRow& h,
                                            unsigned long long* counters) {
    const float k = P.k_n, F = P.max_force;
    // the dashpot coefficient only where a wall is touched (most grains touch none)
    auto c_wall = [&]() { return damping(P, mi); };
    f.z = fmaf(-mi, P.gravity, f.z);
    const float p3[3] = {pos.x, pos.y, pos.z};
    const float v3[3] = {vel.x, vel.y, vel.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float3 vt = make_float3(a == 0 ? 0.f : vel.x, a == 1 ? 0.f : vel.y,
                                      a == 2 ? 0.f : vel.z);
        float fa = a == 0 ? f.x : (a == 1 ? f.y : f.z);
        const float dl = (p3[a] - P.wall_lo[a]) - ri;
        const float fl = fmaxf(0.f, fminf(F, -k * dl));
        fa = fa + fl;
        if (a == 0) f.x = fa; else if (a == 1) f.y = fa; else f.z = fa;
        if (dl < 0.f) {
            const float cw = c_wall();
            fa = fmaf(-cw, v3[a], fa);
            if (a == 0) f.x = fa; else if (a == 1) f.y = fa; else f.z = fa;
            if (HIST) {
                const float3 nrm = make_float3(a == 0 ? 1.f : 0.f, a == 1 ? 1.f : 0.f,
                                               a == 2 ? 1.f : 0.f);
                spring_friction(P, f, vt, nrm, P.mu * fl, -1 - 2 * a, h, counters);
            } else {
                viscous_friction(f, vt, P.mu * fl, cw);
            }
        }
        fa = a == 0 ? f.x : (a == 1 ? f.y : f.z);
        const float du = (P.wall_hi[a] - p3[a]) - ri;
        const float fu = fmaxf(0.f, fminf(F, -k * du));
        fa = fa - fu;
        if (a == 0) f.x = fa; else if (a == 1) f.y = fa; else f.z = fa;
        if (du < 0.f) {
            const float cw = c_wall();
            fa = fmaf(-cw, v3[a], fa);
            if (a == 0) f.x = fa; else if (a == 1) f.y = fa; else f.z = fa;
            if (HIST) {
                const float3 nrm = make_float3(a == 0 ? -1.f : 0.f, a == 1 ? -1.f : 0.f,
                                               a == 2 ? -1.f : 0.f);
                spring_friction(P, f, vt, nrm, P.mu * fu, -2 - 2 * a, h, counters);
            } else {
                viscous_friction(f, vt, P.mu * fu, cw);
            }
        }
    }
}

// Squared centre distance, accumulated as the reference's loop contracts it.
__device__ __forceinline__ float pair_norm_sq(float4 pi, float4 pj, float3& d) {
    d = make_float3(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z);
    float ns = d.x * d.x;
    ns = fmaf(d.y, d.y, ns);
    ns = fmaf(d.z, d.z, ns);
    return ns;
}

// dist = |delta| - r_i - r_j with the larger radius subtracted first: symmetric in
// (i, j) and equal to the reference's norm - radius - radius for equal radii.
__device__ __forceinline__ float pair_dist(float norm, float ri, float rj) {
    const float rmax = fmaxf(ri, rj), rmin = fminf(ri, rj);
    return (norm - rmax) - rmin;
}

// Conservative early-out: ns above this can never give dist < 0.
__device__ __forceinline__ bool maybe_contact(float ns, float ri, float rj) {
    const float rs = ri + rj;
    return ns <= rs * rs * 1.001f;
}

// Per-grain form with the scene's largest radius: one compare per candidate, still
// conservative (the exact dist < 0 test decides).
__device__ __forceinline__ float contact_cutoff_sq(float ri, float rmax) {
    const float rs = ri + rmax;
    return rs * rs * 1.001f;
}

// One pair contact's quantities (reference src/compute_rhs_kernel.cu:150-204, dist < 0
// branch): the normal force fp along nrm, the dashpot term cvn, and the friction t
// (the spring's force, added, in history mode; the viscous term, subtracted,
// otherwise). With springs, xi enters as the stored spring and leaves as the new one.
struct PairTerms {
    float fp, cvn;
    float3 nrm, t;
};

template <bool HIST>
__device__ __forceinline__ PairTerms pair_terms(const DevParams& P, float3 d, float norm,
                                                float dist, float3 vel, float mi, float4 vj,
                                                float3& xi) {
    PairTerms q;
    q.nrm = make_float3(d.x / norm, d.y / norm, d.z / norm);
    q.fp = fmaxf(0.f, fminf(P.max_force, -P.k_n * dist));
    const float mj = vj.w;
    const float msum = mi + mj;
    const float mred = (msum > 0.f) ? (mi * mj) / msum : 0.f;
    const float c = damping(P, mred);
    const float3 vr = make_float3(vel.x - vj.x, vel.y - vj.y, vel.z - vj.z);
    float vn = vr.x * q.nrm.x;
    vn = fmaf(vr.y, q.nrm.y, vn);
    vn = fmaf(vr.z, q.nrm.z, vn);
    q.cvn = c * vn;
    const float3 vt = make_float3(fmaf(-vn, q.nrm.x, vr.x), fmaf(-vn, q.nrm.y, vr.y),
                                  fmaf(-vn, q.nrm.z, vr.z));
    const float limit = P.mu * q.fp;
    q.t = HIST ? spring_step(P, vt, q.nrm, limit, xi) : viscous_term(vt, limit, c);
    return q;
}

// The contact's share of the grain's force, in the reference's order: normal force,
// dashpot, friction.
template <bool HIST>
__device__ __forceinline__ void pair_accumulate(float3& f, const PairTerms& q) {
    f.x = fmaf(q.fp, q.nrm.x, f.x);
    f.y = fmaf(q.fp, q.nrm.y, f.y);
    f.z = fmaf(q.fp, q.nrm.z, f.z);
    f.x = fmaf(-q.cvn, q.nrm.x, f.x);
    f.y = fmaf(-q.cvn, q.nrm.y, f.y);
    f.z = fmaf(-q.cvn, q.nrm.z, f.z);
    if (HIST) {
        f.x = f.x + q.t.x;
        f.y = f.y + q.t.y;
        f.z = f.z + q.t.z;
    } else {
        f.x = f.x - q.t.x;
        f.y = f.y - q.t.y;
        f.z = f.z - q.t.z;
    }
}

// One pair contact accumulated into f, its spring read from and written to h.
template <bool HIST>
__device__ __forceinline__ void pair_force(const DevParams& P, float3 d, float norm,
                                           float dist, float3 vel, float mi, float4 vj,
                                           int partner, float3& f, HistRow& h,
                                           unsigned long long* counters) {
    float3 xi = HIST ? find_spring(h, partner) : make_float3(0.f, 0.f, 0.f);
    const PairTerms q = pair_terms<HIST>(P, d, norm, dist, vel, mi, vj, xi);
    pair_accumulate<HIST>(f, q);
    if (HIST) {
        if (h.out_count < kHistCap) {
            h.out[h.out_count] = make_float4(xi.x, xi.y, xi.z, __int_as_float(partner));
            ++h.out_count;
        } else {
            atomicAdd(&counters[kCntHistOverflow], 1ull);
        }
    }
}

// reference src/energy_kernel.cu:22-27, clamp point generalised to F/k_n.
__device__ __forceinline__ float contact_energy(float delta, float clamp_d, float F, float k) {
    if (delta <= 0.f) return 0.f;
    if (delta <= clamp_d) return 0.5f * k * delta * delta;
    return 0.5f * F * clamp_d + F * (delta - clamp_d);
}

// Slot ranges of the three columns (nx, cy-1 .. cy+1) around cell z = cz: nine run
// table loads issued together, one latency instead of three. Columns outside the
// grid come back empty (lo >= hi).
__device__ __forceinline__ void row_ranges(const DevParams& P, const int2* __restrict__ table,
                                           int nx, int cy, int cz, int lo[3], int hi[3]) {
    const uint32_t gy = static_cast<uint32_t>(P.grid[1]), gz = static_cast<uint32_t>(P.grid[2]);
    table += P.cell_base;
    int2 e[3][3];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        const int ny = cy + t - 1;
        const bool col_ok = ny >= 0 && ny < P.grid[1];
        const uint32_t base = (static_cast<uint32_t>(nx) * gy + static_cast<uint32_t>(ny)) * gz;
#pragma unroll
        for (int z = 0; z < 3; ++z) {
            const int zz = cz + z - 1;
            e[t][z] = (col_ok && zz >= 0 && zz < P.grid[2])
                          ? __ldg(&table[base + static_cast<uint32_t>(zz)])
                          : make_int2(-1, -1);
        }
    }
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        lo[t] = 0x7fffffff;
        hi[t] = 0;
#pragma unroll
        for (int z = 0; z < 3; ++z) {
            if (e[t][z].x >= 0) {
                lo[t] = min(lo[t], e[t][z].x);
                hi[t] = max(hi[t], e[t][z].y);
            }
        }
    }
}

// Range of sorted slots covering cells (x, y, z-1 .. z+1): the three runs are
// consecutive in (key, id) order, so one [lo, hi) spans them in stencil order.
__device__ __forceinline__ void column_range(const DevParams& P, const int2* __restrict__ table,
                                             int nx, int ny, int cz, int& lo, int& hi) {
    const int zlo = max(cz - 1, 0), zhi = min(cz + 1, P.grid[2] - 1);
    const uint32_t base = P.cell_base + flat_cell(P, nx, ny, 0);
    lo = 0x7fffffff;
    hi = 0;
    for (int z = zlo; z <= zhi; ++z) {
        const int2 e = __ldg(&table[base + static_cast<uint32_t>(z)]);
        if (e.x >= 0) {
            lo = min(lo, e.x);
            hi = max(hi, e.y);
        }
    }
}

}  // namespace wd
