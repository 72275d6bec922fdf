// wd_adjoint.cu -- reverse pass of the semi-implicit Euler step, and of the CIC deposit.
//
// Step t maps (x, v, springs) to (x', v', springs'): F from the contacts, then
// v' = v + dt F / m and x' = x + dt v' (src/semi_implicit_euler_kernel.cu:4-16). Given
// the adjoints (lx', lv', lxi') of step t's outputs, k_adj_step returns those of its
// inputs and adds the step's share of dL/d(mu, ln e, k_n):
//   lvt = lv' + dt lx',  lF = dt / m lvt,
//   lx = lx' + sum over contacts J_x^T [lF-side; lxi-side],  lv = lvt + sum J_v^T [...].
// A pair force and its new spring are odd in (d, v_rel, xi) with d = x_i - x_j, and the
// two grains keep mirrored copies of the spring, so grain i alone can apply the pair's
// whole contribution to its own adjoints: with respect to d and v_rel the weights are
// (lF_i - lF_j, lxi'_ij - lxi'_ji); with respect to i's stored spring and the parameters
// they are (lF_i, lxi'_ij). Every grain gathers; nothing is scattered.
//
// The contact set, clamp, slip and viscous-cap branches are those of the forward step
// (wd_adjoint.cuh evaluates the laws with the forward's own float operations).
#include "wd_adjoint.cuh"
#include "wd_kernels.h"

namespace wd {
namespace {

struct AdjStep {
    // sorted state of step t (the step's gathered copy) and its run table
    const float4* pos;
    const float4* vel;
    const int* ids;
    const int2* table;
    // springs of step t (rows by grain id, counts by sorted slot) and of step t+1
    // (rows and counts by grain id)
    const float4* hist_in;
    const int* hcnt_in;
    const float4* hist_next;
    const int* hcnt_next;
    // the step's pair contacts per sorted slot, in the forward's visiting order
    const int* clist;
    const int* ccnt;
    // adjoints of step t's outputs, by grain id
    const float4* lx;
    const float4* lvt;     // lv' + dt lx'
    const float4* lf;      // dt / m * lvt
    const float4* lxi;     // rows like hist_next
    // adjoints of step t's inputs, by grain id
    float4* lx_out;
    float4* lv_out;
    float4* lxi_out;       // rows like hist_in (zeroed before the launch)
    double* theta;         // [3][n]: d/dmu, d/d ln e, d/dk_n, accumulated
    int kt_from_kn;
};

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }

template <class S>
__device__ __forceinline__ Theta<S> make_theta(const DevParams& P, int kt_from_kn, int seed_block) {
    Theta<S> th;
    th.mu = lift<S>(P.mu);
    th.L = lift<S>(P.ln_e);
    th.k = lift<S>(P.k_n);
    if (seed_block) {
        th.mu = dseed<3>(P.mu, 0);
        th.L = dseed<3>(P.ln_e, 1);
        th.k = dseed<3>(P.k_n, 2);
    }
    th.kt = kt_from_kn ? lift<S>(2.f / 7.f) * th.k : lift<S>(P.k_t);
    return th;
}

// Row search: index of partner in a spring row, -1 if absent (first match, as the
// forward's lookup).
__device__ __forceinline__ int row_find(const float4* row, int count, int partner) {
    for (int k = 0; k < count; ++k)
        if (__float_as_int(row[k].w) == partner) return k;
    return -1;
}

// Weighted sums of one Jacobian block: out[c] += sum_o J_f[o][c] wf[o] + J_xi[o][c] wxi[o].
__device__ __forceinline__ void vjp_add(const ContactOut<Dual<3>>& o, float3 wf, float3 wx,
                                        float out[3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
        out[c] += o.f[0].d[c] * wf.x + o.f[1].d[c] * wf.y + o.f[2].d[c] * wf.z +
                  o.xi[0].d[c] * wx.x + o.xi[1].d[c] * wx.y + o.xi[2].d[c] * wx.z;
}

using D3 = Dual<3>;

template <bool HIST>
__device__ __forceinline__ void pair_blocks(const DevParams& P, const AdjStep& A, float3 d,
                                            float3 vr, float3 xi, float ri, float rj, float mi,
                                            float mj, float3 w_rel_f, float3 w_rel_x,
                                            float3 w_own_f, float3 w_own_x, float ax[3],
                                            float av[3], float axi[3], double th[3]) {
    const float dv[3] = {d.x, d.y, d.z}, vv[3] = {vr.x, vr.y, vr.z}, xv[3] = {xi.x, xi.y, xi.z};
    const Theta<D3> th0 = make_theta<D3>(P, A.kt_from_kn, 0);
    for (int blk = 0; blk < 4; ++blk) {
        D3 dd[3], vd[3], xd[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            dd[c] = dseed<3>(dv[c], blk == 0 ? c : -1);
            vd[c] = dseed<3>(vv[c], blk == 1 ? c : -1);
            xd[c] = dseed<3>(xv[c], blk == 2 ? c : -1);
        }
        const Theta<D3> tt = blk == 3 ? make_theta<D3>(P, A.kt_from_kn, 1) : th0;
        ContactOut<D3> o;
        pair_t<D3, HIST>(P, tt, dd, vd, xd, ri, rj, mi, mj, o);
        if (blk == 0) vjp_add(o, w_rel_f, w_rel_x, ax);
        else if (blk == 1) vjp_add(o, w_rel_f, w_rel_x, av);
        else if (blk == 2) vjp_add(o, w_own_f, w_own_x, axi);
        else {
            float t[3] = {0.f, 0.f, 0.f};
            vjp_add(o, w_own_f, w_own_x, t);
#pragma unroll
            for (int c = 0; c < 3; ++c) th[c] += t[c];
        }
    }
}

template <bool HIST>
__device__ __forceinline__ void wall_blocks(const DevParams& P, const AdjStep& A, float3 x,
                                            float3 v, float3 xi, float ri, float mi, int a,
                                            bool upper, float3 wf, float3 wx, float ax[3],
                                            float av[3], float axi[3], double th[3]) {
    const float xv[3] = {x.x, x.y, x.z}, vv[3] = {v.x, v.y, v.z}, sv[3] = {xi.x, xi.y, xi.z};
    const Theta<D3> th0 = make_theta<D3>(P, A.kt_from_kn, 0);
    for (int blk = 0; blk < 4; ++blk) {
        D3 xd[3], vd[3], sd[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            xd[c] = dseed<3>(xv[c], blk == 0 ? c : -1);
            vd[c] = dseed<3>(vv[c], blk == 1 ? c : -1);
            sd[c] = dseed<3>(sv[c], blk == 2 ? c : -1);
        }
        const Theta<D3> tt = blk == 3 ? make_theta<D3>(P, A.kt_from_kn, 1) : th0;
        ContactOut<D3> o;
        wall_t<D3, HIST>(P, tt, xd, vd, sd, ri, mi, a, upper, o);
        if (blk == 0) vjp_add(o, wf, wx, ax);
        else if (blk == 1) vjp_add(o, wf, wx, av);
        else if (blk == 2) vjp_add(o, wf, wx, axi);
        else {
            float t[3] = {0.f, 0.f, 0.f};
            vjp_add(o, wf, wx, t);
#pragma unroll
            for (int c = 0; c < 3; ++c) th[c] += t[c];
        }
    }
}

// lvt = lv' + dt lx' and lF = dt / m lvt, by grain id.
__global__ void __launch_bounds__(kBlock)
k_adj_prep(int n, float dt, const float4* __restrict__ vel, const int* __restrict__ ids,
           const float4* __restrict__ lx, const float4* __restrict__ lv,
           float4* __restrict__ lvt, float4* __restrict__ lf) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int id = ids[s];
    const float m = vel[s].w;
    const float4 x = lx[id], v = lv[id];
    const float4 t = make_float4(fmaf(dt, x.x, v.x), fmaf(dt, x.y, v.y), fmaf(dt, x.z, v.z), 0.f);
    lvt[id] = t;
    const float g = m != 0.f ? dt / m : 0.f;
    lf[id] = make_float4(g * t.x, g * t.y, g * t.z, 0.f);
}

template <bool HIST>
__global__ void __launch_bounds__(kBlock)
k_adj_step(DevParams P, AdjStep A) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n) return;
    const float4 pi = A.pos[s];
    const float4 vi = A.vel[s];
    const int id = A.ids[s];
    const float3 pos = f3(pi), vel = f3(vi);
    const float ri = pi.w, mi = vi.w;
    const float3 lf_i = f3(A.lf[id]);
    const float3 zero = make_float3(0.f, 0.f, 0.f);
    const float4* in_row = HIST ? A.hist_in + static_cast<int64_t>(id) * kHistCap : nullptr;
    const int in_count = HIST ? A.hcnt_in[s] : 0;
    int out_count = 0;
    float ax[3] = {0.f, 0.f, 0.f}, av[3] = {0.f, 0.f, 0.f};
    double th[3] = {0.0, 0.0, 0.0};

    // walls, in the forward's order: axis 0 lower, upper, axis 1, axis 2
    const float p3[3] = {pos.x, pos.y, pos.z};
    for (int a = 0; a < 3; ++a) {
        for (int up = 0; up < 2; ++up) {
            const float dl = up ? (P.wall_hi[a] - p3[a]) - ri : (p3[a] - P.wall_lo[a]) - ri;
            if (!(dl < 0.f)) continue;
            const int partner = up ? -2 - 2 * a : -1 - 2 * a;
            float3 xi = zero, lxi_own = zero;
            int k_in = -1;
            if (HIST) {
                k_in = row_find(in_row, in_count, partner);
                if (k_in >= 0) xi = f3(in_row[k_in]);
                if (out_count < kHistCap)
                    lxi_own = f3(A.lxi[static_cast<int64_t>(id) * kHistCap + out_count]);
                ++out_count;
            }
            float axi[3] = {0.f, 0.f, 0.f};
            wall_blocks<HIST>(P, A, pos, vel, xi, ri, mi, a, up != 0, lf_i, lxi_own, ax, av, axi, th);
            if (HIST && k_in >= 0)
                A.lxi_out[static_cast<int64_t>(id) * kHistCap + k_in] =
                    make_float4(axi[0], axi[1], axi[2], 0.f);
        }
    }

    // pairs, in the forward's visiting order (recorded by the replay)
    const int nc = A.ccnt[s];
    for (int e = 0; e < nc; ++e) {
        const int j = A.clist[static_cast<int64_t>(e) * P.n + s];
        const float4 pj = A.pos[j];
        float3 d;
        pair_norm_sq(pi, pj, d);
        const float4 vj = A.vel[j];
        const int jd = A.ids[j];
        const float3 lf_j = f3(A.lf[jd]);
        float3 xi = zero, lxi_ij = zero, lxi_ji = zero;
        int k_in = -1;
        if (HIST) {
            k_in = row_find(in_row, in_count, jd);
            if (k_in >= 0) xi = f3(in_row[k_in]);
            if (out_count < kHistCap)
                lxi_ij = f3(A.lxi[static_cast<int64_t>(id) * kHistCap + out_count]);
            ++out_count;
            const float4* jrow = A.hist_next + static_cast<int64_t>(jd) * kHistCap;
            const int kj = row_find(jrow, A.hcnt_next[jd], id);
            if (kj >= 0) lxi_ji = f3(A.lxi[static_cast<int64_t>(jd) * kHistCap + kj]);
        }
        const float3 w_rel_f = make_float3(lf_i.x - lf_j.x, lf_i.y - lf_j.y, lf_i.z - lf_j.z);
        const float3 w_rel_x = make_float3(lxi_ij.x - lxi_ji.x, lxi_ij.y - lxi_ji.y,
                                           lxi_ij.z - lxi_ji.z);
        const float3 vr = make_float3(vel.x - vj.x, vel.y - vj.y, vel.z - vj.z);
        float axi[3] = {0.f, 0.f, 0.f};
        pair_blocks<HIST>(P, A, d, vr, xi, ri, pj.w, mi, vj.w, w_rel_f, w_rel_x, lf_i,
                          lxi_ij, ax, av, axi, th);
        if (HIST && k_in >= 0)
            A.lxi_out[static_cast<int64_t>(id) * kHistCap + k_in] =
                make_float4(axi[0], axi[1], axi[2], 0.f);
    }
    const float4 lx = A.lx[id], lvt = A.lvt[id];
    A.lx_out[id] = make_float4(lx.x + ax[0], lx.y + ax[1], lx.z + ax[2], 0.f);
    A.lv_out[id] = make_float4(lvt.x + av[0], lvt.y + av[1], lvt.z + av[2], 0.f);
#pragma unroll
    for (int c = 0; c < 3; ++c) A.theta[static_cast<int64_t>(c) * P.n + id] += th[c];
}

// The pair contacts of every sorted slot in the contact kernel's visiting order
// (run-table stencil walk, the same tests), for the reverse pass.
__global__ void __launch_bounds__(kBlock)
k_contact_record(DevParams P, const float4* __restrict__ pos, const int2* __restrict__ table,
                 int* __restrict__ clist, int* __restrict__ ccnt,
                 unsigned long long* __restrict__ overflow) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n) return;
    const float4 pi = pos[s];
    const float ri = pi.w;
    const float cut = contact_cutoff_sq(ri, P.rmax);
    int cx, cy, cz;
    cell_coords(P, pi.x, pi.y, pi.z, cx, cy, cz);
    int cnt = 0;
    for (int dx = -1; dx <= 1; ++dx) {
        const int nx = cx + dx;
        if (nx < 0 || nx >= P.grid[0]) continue;
        int lo[3], hi[3];
        row_ranges(P, table, nx, cy, cz, lo, hi);
        for (int t = 0; t < 3; ++t) {
            for (int j = lo[t]; j < hi[t]; ++j) {
                const float4 pj = __ldg(&pos[j]);
                float3 d;
                const float ns = pair_norm_sq(pi, pj, d);
                if (ns > cut || j == s) continue;
                const float dist = pair_dist(sqrtf(ns), ri, pj.w);
                if (!(dist < 0.f)) continue;
                if (cnt < kAdjContacts) clist[static_cast<int64_t>(cnt) * P.n + s] = j;
                ++cnt;
            }
        }
    }
    if (cnt > kAdjContacts) {
        atomicAdd(overflow, 1ull);
        cnt = kAdjContacts;
    }
    ccnt[s] = cnt;
}

// Counts of a spring snapshot by grain id (snapshots keep them by sorted slot).
__global__ void __launch_bounds__(kBlock)
k_counts_by_id(int n, const int* __restrict__ ids, const int* __restrict__ cnt_slot,
               int* __restrict__ cnt_id) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) cnt_id[ids[s]] = cnt_slot[s];
}

// reference src/density_grid_kernel.cu:25-40 with d(frac)/dx = 1/h.
__device__ __forceinline__ void axis_weights_d(float x, float lo, float hi, int size, int& i0,
                                               int& i1, float& w0, float& w1, float& dw) {
    if (size <= 1) {
        i0 = 0; i1 = 0; w0 = 1.f; w1 = 0.f; dw = 0.f;
        return;
    }
    const float h = (hi - lo) / static_cast<float>(size - 1);
    const float u = (x - lo) / h;
    const float base = floorf(u);
    const float frac = u - base;
    const int b = __float2int_rz(base);
    i0 = min(size - 1, max(0, b));
    i1 = min(size - 1, max(0, static_cast<int>(static_cast<unsigned>(b) + 1u)));
    w0 = 1.f - frac;
    w1 = frac;
    dw = 1.f / h;
}

// Adjoint of the CIC deposit at the current state: for node weights w(x) and
// contributions m w, m v_a w, gx = sum_corners dw/dx (m G0 + m v.G_mom), gv_a = sum w m G_a.
__global__ void __launch_bounds__(kBlock)
k_deposit_vjp(int n, const float4* __restrict__ pos, const float4* __restrict__ vel,
              const int* __restrict__ ids, float lo0, float lo1, float lo2, float hi0, float hi1,
              float hi2, int sx, int sy, int sz, const float* __restrict__ g,
              float4* __restrict__ gx, float4* __restrict__ gv) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 x = pos[s], v = vel[s];
    const int id = ids[s];
    const float m = v.w;
    float ax[3] = {0.f, 0.f, 0.f}, av[3] = {0.f, 0.f, 0.f};
    if (m != 0.f) {
        int ix[2], iy[2], iz[2];
        float wx[2], wy[2], wz[2], dx, dy, dz;
        axis_weights_d(x.x, lo0, hi0, sx, ix[0], ix[1], wx[0], wx[1], dx);
        axis_weights_d(x.y, lo1, hi1, sy, iy[0], iy[1], wy[0], wy[1], dy);
        axis_weights_d(x.z, lo2, hi2, sz, iz[0], iz[1], wz[0], wz[1], dz);
        const float sgn[2] = {-1.f, 1.f};
        const int64_t nodes = static_cast<int64_t>(sx) * sy * sz;
        for (int cx = 0; cx < 2; ++cx)
            for (int cy = 0; cy < 2; ++cy)
                for (int cz = 0; cz < 2; ++cz) {
                    const int64_t node = (static_cast<int64_t>(ix[cx]) * sy + iy[cy]) * sz + iz[cz];
                    const float g0 = g[node], g1 = g[nodes + node], g2 = g[2 * nodes + node],
                                g3 = g[3 * nodes + node];
                    const float w = wx[cx] * wy[cy] * wz[cz];
                    const float val = m * (g0 + v.x * g1 + v.y * g2 + v.z * g3);
                    ax[0] += sgn[cx] * dx * wy[cy] * wz[cz] * val;
                    ax[1] += sgn[cy] * dy * wx[cx] * wz[cz] * val;
                    ax[2] += sgn[cz] * dz * wx[cx] * wy[cy] * val;
                    av[0] += w * m * g1;
                    av[1] += w * m * g2;
                    av[2] += w * m * g3;
                }
    }
    gx[id] = make_float4(ax[0], ax[1], ax[2], 0.f);
    gv[id] = make_float4(av[0], av[1], av[2], 0.f);
}

}  // namespace

void launch_adj_prep(int n, float dt, const float4* vel, const int* ids, const float4* lx,
                     const float4* lv, float4* lvt, float4* lf, cudaStream_t st) {
    k_adj_prep<<<blocks_for(n), kBlock, 0, st>>>(n, dt, vel, ids, lx, lv, lvt, lf);
}

void launch_contact_record(const DevParams& P, const float4* pos, const int2* table, int* clist,
                           int* ccnt, unsigned long long* overflow, cudaStream_t st) {
    k_contact_record<<<blocks_for(P.n), kBlock, 0, st>>>(P, pos, table, clist, ccnt, overflow);
}

void launch_adj_step(const DevParams& P, const AdjArgs& a, cudaStream_t st) {
    AdjStep A;
    A.pos = a.pos; A.vel = a.vel; A.ids = a.ids; A.table = a.table;
    A.hist_in = a.hist_in; A.hcnt_in = a.hcnt_in; A.hist_next = a.hist_next;
    A.hcnt_next = a.hcnt_next; A.clist = a.clist; A.ccnt = a.ccnt; A.lx = a.lx; A.lvt = a.lvt; A.lf = a.lf; A.lxi = a.lxi;
    A.lx_out = a.lx_out; A.lv_out = a.lv_out; A.lxi_out = a.lxi_out; A.theta = a.theta;
    A.kt_from_kn = a.kt_from_kn;
    if (P.history) k_adj_step<true><<<blocks_for(P.n), kBlock, 0, st>>>(P, A);
    else k_adj_step<false><<<blocks_for(P.n), kBlock, 0, st>>>(P, A);
}

void launch_counts_by_id(int n, const int* ids, const int* cnt_slot, int* cnt_id, cudaStream_t st) {
    k_counts_by_id<<<blocks_for(n), kBlock, 0, st>>>(n, ids, cnt_slot, cnt_id);
}

void launch_deposit_vjp(int n, const float4* pos, const float4* vel, const int* ids,
                        const float* lo, const float* hi, const int* size, const float* g,
                        float4* gx, float4* gv, cudaStream_t st) {
    k_deposit_vjp<<<blocks_for(n), kBlock, 0, st>>>(n, pos, vel, ids, lo[0], lo[1], lo[2], hi[0],
                                                    hi[1], hi[2], size[0], size[1], size[2], g,
                                                    gx, gv);
}

}  // namespace wd

namespace wd {
namespace {

__global__ void __launch_bounds__(kBlock)
k_aos3_to_f4(int n, const float* __restrict__ a, float4* __restrict__ o) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    o[i] = a ? make_float4(a[3 * static_cast<int64_t>(i)], a[3 * static_cast<int64_t>(i) + 1],
                           a[3 * static_cast<int64_t>(i) + 2], 0.f)
             : make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void __launch_bounds__(kBlock)
k_f4_to_aos3(int n, const float4* __restrict__ a, float* __restrict__ o) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = a[i];
    o[3 * static_cast<int64_t>(i)] = v.x;
    o[3 * static_cast<int64_t>(i) + 1] = v.y;
    o[3 * static_cast<int64_t>(i) + 2] = v.z;
}

}  // namespace

void launch_aos3_to_f4(int n, const float* a, float4* o, cudaStream_t st) {
    k_aos3_to_f4<<<blocks_for(n), kBlock, 0, st>>>(n, a, o);
}

void launch_f4_to_aos3(int n, const float4* a, float* o, cudaStream_t st) {
    k_f4_to_aos3<<<blocks_for(n), kBlock, 0, st>>>(n, a, o);
}

}  // namespace wd
