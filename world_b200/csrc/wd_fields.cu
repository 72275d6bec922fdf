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
                // combine lanes that hit the same node, then one atomic per node
                const unsigned peers = __match_any_sync(0xffffffffu, node);
                const int leader = __ffs(peers) - 1;
                const int lane = threadIdx.x & 31;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    long long sum = 0;
                    unsigned rest = peers;
                    while (rest) {
                        const int src = __ffs(rest) - 1;
                        rest &= rest - 1u;
                        sum += __shfl_sync(peers, q[c], src);
                    }
                    q[c] = sum;
                }
                if (live && lane == leader) {
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
    const double inv = 1.0 / channel_scale(n, bounds[c]);
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

}  // namespace wd
