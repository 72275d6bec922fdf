// wd_fields.cu -- node-centred CIC deposit of mass and momentum.
//
// Weights and layout follow reference src/density_grid_kernel.cu:25-83 (node-centred
// spacing (hi-lo)/(size-1), indices clamped, zero-mass grains skipped, channel-major
// [m, m vx, m vy, m vz], node = (ix*ny + iy)*nz + iz). The reference accumulates with
// float atomicAdd, so its field changes with thread timing. Here every contribution
// (the same float product the reference adds) is converted to a 64-bit fixed-point
// integer with a power-of-two scale chosen per channel from a bound on the channel's
// total, and accumulated with integer atomics: integer addition is associative, so
// the field is bit-identical run to run and is the correctly rounded sum up to the
// 2^-62-relative quantum. Grains are visited in cell order, so neighbouring lanes hit
// the same nodes; identical nodes inside a warp are combined before the atomic.
#include <cfloat>
#include <cmath>

#include "wd_kernels.h"

namespace wd {

namespace {

// reference src/density_grid_kernel.cu:25-40
__device__ __forceinline__ void axis_weights(float x, float lo, float hi, int size, int& i0,
                                             int& i1, float& w0, float& w1) {
    if (size <= 1) {
        i0 = 0; i1 = 0; w0 = 1.f; w1 = 0.f;
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
}

struct DepositGeom {
    float lo[3], hi[3];
    int size[3];
};

// Channel bounds: max |m| and max |m v_a| over grains (float bits; max of
// non-negative floats is order-independent).
__global__ void __launch_bounds__(kBlock)
k_deposit_bounds(int n, const float4* __restrict__ vel, uint32_t* __restrict__ bounds) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t b[4] = {0u, 0u, 0u, 0u};
    if (s < n) {
        const float4 v = vel[s];
        const float m = v.w;
        if (m != 0.f) {
            b[0] = __float_as_uint(fabsf(m));
            b[1] = __float_as_uint(fabsf(m * v.x));
            b[2] = __float_as_uint(fabsf(m * v.y));
            b[3] = __float_as_uint(fabsf(m * v.z));
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        uint32_t x = b[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = max(x, __shfl_xor_sync(0xffffffffu, x, o));
        if ((threadIdx.x & 31) == 0 && x) atomicMax(&bounds[c], x);
    }
}

// Scale 2^(62-e) with n * bound < 2^e, so every partial sum stays below 2^62.
__device__ __forceinline__ double channel_scale(int n, uint32_t bound_bits) {
    const double b = static_cast<double>(__uint_as_float(bound_bits)) * static_cast<double>(n);
    if (!(b > 0.0) || !isfinite(b)) return 1.0;
    int e;
    frexp(b, &e);
    return ldexp(1.0, 62 - e);
}

// Adds up q over each run of adjacent lanes that hold the same key: a segmented inclusive
// scan by shuffles (one step per doubling of the longest run in the warp), after which the
// last lane of each run holds the run's total. Returns true on that lane. Grains arrive in
// cell order, so lanes that deposit on one node are mostly adjacent; a node that comes back
// later in the warp forms a second run with its own atomic. The values are integers, so the
// node totals do not depend on how the lanes are grouped.
__device__ __forceinline__ bool run_totals(long long key, long long (&q)[4]) {
    const int lane = threadIdx.x & 31;
    const long long prev = __shfl_up_sync(0xffffffffu, key, 1);
    const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || prev != key);
    const bool last = lane == 31 || ((heads >> (lane + 1)) & 1u);
    if (heads == 0xffffffffu) return true;
    const int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
    const unsigned longest = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(lane - start + 1));
    for (unsigned d = 1; d < longest; d <<= 1) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const long long t = __shfl_up_sync(0xffffffffu, q[c], d);
            if (lane - static_cast<int>(d) >= start) q[c] += t;
        }
    }
    return last;
}

__global__ void __launch_bounds__(kBlock)
k_deposit(int n, const float4* __restrict__ pos, const float4* __restrict__ vel,
          DepositGeom g, const uint32_t* __restrict__ bounds,
          unsigned long long* __restrict__ acc) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nodes = static_cast<int64_t>(g.size[0]) * g.size[1] * g.size[2];
    double scale[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) scale[c] = channel_scale(n, bounds[c]);
    bool active = s < n;
    float4 x = make_float4(0.f, 0.f, 0.f, 0.f), v = x;
    if (active) {
        x = pos[s];
        v = vel[s];
        active = v.w != 0.f;
    }
    int ix[2] = {0, 0}, iy[2] = {0, 0}, iz[2] = {0, 0};
    float wx[2] = {0.f, 0.f}, wy[2] = {0.f, 0.f}, wz[2] = {0.f, 0.f};
    const float m = v.w;
    const float mom[3] = {m * v.x, m * v.y, m * v.z};
    if (active) {
        axis_weights(x.x, g.lo[0], g.hi[0], g.size[0], ix[0], ix[1], wx[0], wx[1]);
        axis_weights(x.y, g.lo[1], g.hi[1], g.size[1], iy[0], iy[1], wy[0], wy[1]);
        axis_weights(x.z, g.lo[2], g.hi[2], g.size[2], iz[0], iz[1], wz[0], wz[1]);
    }
#pragma unroll
    for (int cx = 0; cx < 2; ++cx)
#pragma unroll
        for (int cy = 0; cy < 2; ++cy)
#pragma unroll
            for (int cz = 0; cz < 2; ++cz) {
                const float w = wx[cx] * wy[cy] * wz[cz];
                const bool live = active && w != 0.f;
                const long long node =
                    live ? (static_cast<long long>(ix[cx]) * g.size[1] + iy[cy]) * g.size[2] + iz[cz]
                         : -1ll;
                long long q[4] = {0, 0, 0, 0};
                if (live) {
                    q[0] = __double2ll_rn(static_cast<double>(m * w) * scale[0]);
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        q[a + 1] = __double2ll_rn(static_cast<double>(mom[a] * w) * scale[a + 1]);
                }
                // combine adjacent lanes that hit the same node, then one atomic per run
                const bool tail = run_totals(node, q);
                if (live && tail) {
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        if (q[c] != 0)
                            atomicAdd(&acc[c * nodes + node], static_cast<unsigned long long>(q[c]));
                }
            }
}

__global__ void __launch_bounds__(kBlock)
k_deposit_finish(int n, int64_t nodes, const uint32_t* __restrict__ bounds,
                 const unsigned long long* __restrict__ acc, float* __restrict__ out) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= 4 * nodes) return;
    const int c = static_cast<int>(t / nodes);
    // a NaN or infinite mass or momentum makes its whole channel NaN (the bound is the
    // largest |value| by its bits, so it is not finite exactly when some value is not)
    if (!(__uint_as_float(bounds[c]) <= FLT_MAX)) {
        out[t] = __uint_as_float(0x7fc00000u);
        return;
    }
    const double inv = 1.0 / channel_scale(n, bounds[c]);
    out[t] = static_cast<float>(static_cast<double>(static_cast<long long>(acc[t])) * inv);
}

// Batched scenes: one field per scene, laid out scene after scene
// ([scene][4][nodes of that scene]); each grain deposits with its own scene's grid and
// the channel scale of its scene (bounds and grain count per scene), so a scene's
// field is bit-identical to the one it gets alone.
__global__ void __launch_bounds__(kBlock)
k_deposit_bounds_batch(int n, const float4* __restrict__ vel, SceneTab T,
                       uint32_t* __restrict__ bounds) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 v = vel[s];
    const float m = v.w;
    if (m == 0.f) return;
    uint32_t* b = bounds + 4 * T.scene[s];
    atomicMax(&b[0], __float_as_uint(fabsf(m)));
    atomicMax(&b[1], __float_as_uint(fabsf(m * v.x)));
    atomicMax(&b[2], __float_as_uint(fabsf(m * v.y)));
    atomicMax(&b[3], __float_as_uint(fabsf(m * v.z)));
}

__global__ void __launch_bounds__(kBlock)
k_deposit_batch(int n, const float4* __restrict__ pos, const float4* __restrict__ vel, SceneTab T,
                const uint32_t* __restrict__ bounds, unsigned long long* __restrict__ acc) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    bool active = s < n;
    int sc = 0;
    float4 x = make_float4(0.f, 0.f, 0.f, 0.f), v = x;
    if (active) {
        sc = T.scene[s];
        x = pos[s];
        v = vel[s];
        active = v.w != 0.f;
    }
    const DevParams& Q = T.params[sc];
    const int64_t nodes = static_cast<int64_t>(Q.dgrid[0]) * Q.dgrid[1] * Q.dgrid[2];
    unsigned long long* a = acc + 4 * static_cast<int64_t>(Q.node_base);
    double scale[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) scale[c] = channel_scale(Q.n, bounds[4 * sc + c]);
    int ix[2] = {0, 0}, iy[2] = {0, 0}, iz[2] = {0, 0};
    float wx[2] = {0.f, 0.f}, wy[2] = {0.f, 0.f}, wz[2] = {0.f, 0.f};
    const float m = v.w;
    const float mom[3] = {m * v.x, m * v.y, m * v.z};
    if (active) {
        axis_weights(x.x, Q.lo[0], Q.hi[0], Q.dgrid[0], ix[0], ix[1], wx[0], wx[1]);
        axis_weights(x.y, Q.lo[1], Q.hi[1], Q.dgrid[1], iy[0], iy[1], wy[0], wy[1]);
        axis_weights(x.z, Q.lo[2], Q.hi[2], Q.dgrid[2], iz[0], iz[1], wz[0], wz[1]);
    }
#pragma unroll
    for (int cx = 0; cx < 2; ++cx)
#pragma unroll
        for (int cy = 0; cy < 2; ++cy)
#pragma unroll
            for (int cz = 0; cz < 2; ++cz) {
                const float w = wx[cx] * wy[cy] * wz[cz];
                const bool live = active && w != 0.f;
                const long long node =
                    live ? (static_cast<long long>(ix[cx]) * Q.dgrid[1] + iy[cy]) * Q.dgrid[2] + iz[cz]
                         : -1ll;
                // lanes combine only within one scene: key the runs on (scene, node)
                const long long key = live ? (static_cast<long long>(sc) << 40) | node : -1ll;
                long long q[4] = {0, 0, 0, 0};
                if (live) {
                    q[0] = __double2ll_rn(static_cast<double>(m * w) * scale[0]);
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                        q[k + 1] = __double2ll_rn(static_cast<double>(mom[k] * w) * scale[k + 1]);
                }
                // combine adjacent lanes that hit the same node, then one atomic per run
                const bool tail = run_totals(key, q);
                if (live && tail) {
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        if (q[c] != 0)
                            atomicAdd(&a[c * nodes + node], static_cast<unsigned long long>(q[c]));
                }
            }
}

__global__ void __launch_bounds__(kBlock)
k_deposit_finish_batch(const DevParams* __restrict__ params, int scenes, int64_t total,
                       const uint32_t* __restrict__ bounds,
                       const unsigned long long* __restrict__ acc, float* __restrict__ out) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= total) return;
    int lo = 0, hi = scenes;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (4 * static_cast<int64_t>(params[mid].node_base) <= t) lo = mid; else hi = mid;
    }
    const DevParams& Q = params[lo];
    const int64_t nodes = static_cast<int64_t>(Q.dgrid[0]) * Q.dgrid[1] * Q.dgrid[2];
    const int c = static_cast<int>((t - 4 * static_cast<int64_t>(Q.node_base)) / nodes);
    if (!(__uint_as_float(bounds[4 * lo + c]) <= FLT_MAX)) {   // non-finite input: NaN channel
        out[t] = __uint_as_float(0x7fc00000u);
        return;
    }
    const double inv = 1.0 / channel_scale(Q.n, bounds[4 * lo + c]);
    out[t] = static_cast<float>(static_cast<double>(static_cast<long long>(acc[t])) * inv);
}

}  // namespace

void launch_deposit(int n, const float4* pos, const float4* vel, const float* lo,
                    const float* hi, const int* dgrid, uint32_t* bounds,
                    unsigned long long* acc, float* out, cudaStream_t st) {
    DepositGeom g;
    for (int a = 0; a < 3; ++a) {
        g.lo[a] = lo[a];
        g.hi[a] = hi[a];
        g.size[a] = dgrid[a];
    }
    const int64_t nodes = static_cast<int64_t>(dgrid[0]) * dgrid[1] * dgrid[2];
    cudaMemsetAsync(bounds, 0, 4 * sizeof(uint32_t), st);
    cudaMemsetAsync(acc, 0, 4 * nodes * sizeof(unsigned long long), st);
    if (n > 0) {
        k_deposit_bounds<<<blocks_for(n), kBlock, 0, st>>>(n, vel, bounds);
        k_deposit<<<blocks_for(n), kBlock, 0, st>>>(n, pos, vel, g, bounds, acc);
    }
    k_deposit_finish<<<static_cast<int>((4 * nodes + kBlock - 1) / kBlock), kBlock, 0, st>>>(
        n, nodes, bounds, acc, out);
}

void launch_deposit_batch(int n, const float4* pos, const float4* vel, SceneTab T, int scenes,
                          int64_t total_nodes, uint32_t* bounds, unsigned long long* acc,
                          float* out, cudaStream_t st) {
    cudaMemsetAsync(bounds, 0, 4 * sizeof(uint32_t) * static_cast<size_t>(scenes), st);
    cudaMemsetAsync(acc, 0, 4 * total_nodes * sizeof(unsigned long long), st);
    if (n > 0) {
        k_deposit_bounds_batch<<<blocks_for(n), kBlock, 0, st>>>(n, vel, T, bounds);
        k_deposit_batch<<<blocks_for(n), kBlock, 0, st>>>(n, pos, vel, T, bounds, acc);
    }
    k_deposit_finish_batch<<<static_cast<int>((4 * total_nodes + kBlock - 1) / kBlock), kBlock, 0,
                             st>>>(T.params, scenes, 4 * total_nodes, bounds, acc, out);
}

}  // namespace wd

// ---------------------------------------------------------------------------------
// Allocation-free variant of the deposit for callers that cannot call cudaMalloc
// (device memory owned by another framework's allocator, or a loop that must not
// allocate). Inputs are the caller's own device arrays in the reference's AoS
// layout; the scratch is the static array below, one per device, never freed.
// ---------------------------------------------------------------------------------
#include <string>

#include "../../include/world_b200.h"
#include "wd_config.h"

namespace {

constexpr long long kNoAllocNodes = WD_NOALLOC_MAX_NODES;
// 4 channels of 64-bit accumulators, then 2 words holding the four 32-bit bounds.
static __device__ __align__(256) unsigned long long g_deposit_scratch[4 * kNoAllocNodes + 2];


__global__ void __launch_bounds__(wd::kBlock)
k_deposit_bounds_aos(int n, const float* __restrict__ state, const float* __restrict__ mass,
                     uint32_t* __restrict__ bounds) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t b[4] = {0u, 0u, 0u, 0u};
    if (s < n) {
        const float m = mass[s];
        if (m != 0.f) {
            const float* q = state + 6 * static_cast<int64_t>(s);
            b[0] = __float_as_uint(fabsf(m));
            b[1] = __float_as_uint(fabsf(m * q[3]));
            b[2] = __float_as_uint(fabsf(m * q[4]));
            b[3] = __float_as_uint(fabsf(m * q[5]));
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        uint32_t x = b[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = max(x, __shfl_xor_sync(0xffffffffu, x, o));
        if ((threadIdx.x & 31) == 0 && x) atomicMax(&bounds[c], x);
    }
}

// Same contributions, scale and per-warp combining as k_deposit; integer sums make
// the field independent of the order grains arrive in.
__global__ void __launch_bounds__(wd::kBlock)
k_deposit_aos(int n, const float* __restrict__ state, const float* __restrict__ mass,
              wd::DepositGeom g, const uint32_t* __restrict__ bounds,
              unsigned long long* __restrict__ acc) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nodes = static_cast<int64_t>(g.size[0]) * g.size[1] * g.size[2];
    double scale[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) scale[c] = wd::channel_scale(n, bounds[c]);
    bool active = s < n;
    float p[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float m = 0.f;
    if (active) {
        const float* q = state + 6 * static_cast<int64_t>(s);
#pragma unroll
        for (int a = 0; a < 6; ++a) p[a] = q[a];
        m = mass[s];
        active = m != 0.f;
    }
    int ix[2] = {0, 0}, iy[2] = {0, 0}, iz[2] = {0, 0};
    float wx[2] = {0.f, 0.f}, wy[2] = {0.f, 0.f}, wz[2] = {0.f, 0.f};
    const float mom[3] = {m * p[3], m * p[4], m * p[5]};
    if (active) {
        wd::axis_weights(p[0], g.lo[0], g.hi[0], g.size[0], ix[0], ix[1], wx[0], wx[1]);
        wd::axis_weights(p[1], g.lo[1], g.hi[1], g.size[1], iy[0], iy[1], wy[0], wy[1]);
        wd::axis_weights(p[2], g.lo[2], g.hi[2], g.size[2], iz[0], iz[1], wz[0], wz[1]);
    }
#pragma unroll
    for (int cx = 0; cx < 2; ++cx)
#pragma unroll
        for (int cy = 0; cy < 2; ++cy)
#pragma unroll
            for (int cz = 0; cz < 2; ++cz) {
                const float w = wx[cx] * wy[cy] * wz[cz];
                const bool live = active && w != 0.f;
                const long long node =
                    live ? (static_cast<long long>(ix[cx]) * g.size[1] + iy[cy]) * g.size[2] + iz[cz]
                         : -1ll;
                long long q[4] = {0, 0, 0, 0};
                if (live) {
                    q[0] = __double2ll_rn(static_cast<double>(m * w) * scale[0]);
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        q[a + 1] = __double2ll_rn(static_cast<double>(mom[a] * w) * scale[a + 1]);
                }
                // combine adjacent lanes that hit the same node, then one atomic per run
                const bool tail = wd::run_totals(node, q);
                if (live && tail) {
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        if (q[c] != 0)
                            atomicAdd(&acc[c * nodes + node], static_cast<unsigned long long>(q[c]));
                }
            }
}

// Device address of the scratch array in the current device's context. Looked up on
// every call (a host-side table lookup, no allocation and no device work), so the
// address stays right after a cudaDeviceReset or when another context is made current.
cudaError_t scratch_for_current_device(unsigned long long** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_deposit_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned long long*>(p);
    return cudaSuccess;
}

}  // namespace

extern "C" int wd_deposit_grid_noalloc(const float* d_state, const float* d_mass, int64_t n,
                                       const float* lo3, const float* hi3, const int32_t* size3,
                                       float* d_grid, void* stream_v) {
    if (!lo3 || !hi3 || !size3 || !d_grid || (n > 0 && (!d_state || !d_mass))) {
        wd::set_last_error("wd_deposit_grid_noalloc: NULL argument");
        return WD_ERR_INVALID;
    }
    if (n < 0 || n > (int64_t{1} << 30)) {
        wd::set_last_error("wd_deposit_grid_noalloc: grain count must be in [0, 2^30]");
        return WD_ERR_INVALID;
    }
    for (int a = 0; a < 3; ++a) {
        if (size3[a] < 1) {
            wd::set_last_error("wd_deposit_grid_noalloc: grid sizes must be >= 1");
            return WD_ERR_INVALID;
        }
    }
    const int64_t nodes = static_cast<int64_t>(size3[0]) * size3[1] * size3[2];
    if (nodes > kNoAllocNodes) {
        wd::set_last_error("wd_deposit_grid_noalloc: grid of " + std::to_string(nodes) +
                           " nodes exceeds the fixed scratch of " +
                           std::to_string(kNoAllocNodes) + " nodes (64^3)");
        return WD_ERR_CAPACITY;
    }
    unsigned long long* scratch = nullptr;
    cudaError_t e = scratch_for_current_device(&scratch);
    if (e != cudaSuccess) {
        wd::set_last_error(std::string("wd_deposit_grid_noalloc: cudaGetSymbolAddress: ") +
                           cudaGetErrorString(e));
        return WD_ERR_CUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream_v);
    unsigned long long* acc = scratch;
    uint32_t* bounds = reinterpret_cast<uint32_t*>(scratch + 4 * kNoAllocNodes);
    wd::DepositGeom g;
    for (int a = 0; a < 3; ++a) {
        g.lo[a] = lo3[a];
        g.hi[a] = hi3[a];
        g.size[a] = size3[a];
    }
    // the array keeps the previous call's sums: clear what this call reads
    e = cudaMemsetAsync(bounds, 0, 4 * sizeof(uint32_t), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(acc, 0, static_cast<size_t>(4 * nodes) * sizeof(unsigned long long), st);
    if (e == cudaSuccess && n > 0) {
        const int ni = static_cast<int>(n);
        k_deposit_bounds_aos<<<wd::blocks_for(ni), wd::kBlock, 0, st>>>(ni, d_state, d_mass, bounds);
        k_deposit_aos<<<wd::blocks_for(ni), wd::kBlock, 0, st>>>(ni, d_state, d_mass, g, bounds, acc);
    }
    if (e == cudaSuccess) {
        wd::k_deposit_finish<<<static_cast<int>((4 * nodes + wd::kBlock - 1) / wd::kBlock), wd::kBlock, 0,
                               st>>>(static_cast<int>(n), nodes, bounds, acc, d_grid);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        wd::set_last_error(std::string("wd_deposit_grid_noalloc: ") + cudaGetErrorString(e));
        return WD_ERR_CUDA;
    }
    return WD_OK;
}
