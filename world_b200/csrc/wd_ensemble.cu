// Ensemble metrics over the scenes of a batch, on the device.
//
// The reference's chaos driver (src/chaos.cpp:47-78,176-206) runs its members one
// after another and compares each with the unperturbed member on the host: the
// per-grain RMS separation sqrt(mean_i |x_i^(e) - x_i^(ref)|^2), the relative l2
// difference of the mass field ||rho^(e) - rho^(ref)|| / ||rho^(ref)|| and the
// displacement of the field's centre of mass (in node units). Here all members are
// scenes of one batch, so the three measures come from per-grain and per-node FP64
// terms reduced per scene with the segmented sums of wd_contact.cu.
#include "wd_device.cuh"
#include "wd_kernels.h"

namespace wd {
namespace {

__device__ __forceinline__ int segment_of(const int* __restrict__ seg, int scenes, int i) {
    int lo = 0, hi = scenes;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (seg[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// Squared separation of grain i of scene e from grain i of the reference scene
// (chaos.cpp:196-205: differences and squares in FP64, axes summed in order).
__global__ void __launch_bounds__(kBlock)
k_chaos_grains(int n, const float* __restrict__ pos3, const int* __restrict__ seg, int scenes,
               int ref, double* __restrict__ out) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const int e = segment_of(seg, scenes, g);
    double sq = 0.0;
    if (e != ref) {
        const int r = seg[ref] + (g - seg[e]);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double d = static_cast<double>(pos3[3 * static_cast<int64_t>(g) + a]) -
                             static_cast<double>(pos3[3 * static_cast<int64_t>(r) + a]);
            sq += d * d;
        }
    }
    out[g] = sq;
}

// Per node of the batch's field (scene after scene): (rho - rho_ref)^2, rho_ref^2,
// rho, rho*ix, rho*iy, rho*iz, component-major. Node (ix, iy, iz) of a scene's
// mass channel sits at (ix * ny + iy) * nz + iz of its block (chaos.cpp:64-66).
__global__ void __launch_bounds__(kBlock)
k_chaos_nodes(int total, const float* __restrict__ grid, const int* __restrict__ nseg,
              int scenes, int ref, int ny, int nz, double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int e = segment_of(nseg, scenes, t);
    const int node = t - nseg[e];
    const double m = grid[4 * static_cast<int64_t>(nseg[e]) + node];
    const double mr = grid[4 * static_cast<int64_t>(nseg[ref]) + node];
    const double d = m - mr;
    const int iz = node % nz;
    const int iy = (node / nz) % ny;
    const int ix = node / (nz * ny);
    const int64_t T = total;
    out[t] = d * d;
    out[T + t] = mr * mr;
    out[2 * T + t] = m;
    out[3 * T + t] = m * ix;
    out[4 * T + t] = m * iy;
    out[5 * T + t] = m * iz;
}

}  // namespace

void launch_chaos(int n, const float* pos3, const Segments& grains, double* grain_vals,
                  double* grain_partials, double* grain_sums, int total_nodes, const float* grid,
                  const Segments& nodes, int ref, int ny, int nz, double* node_vals,
                  double* node_partials, double* node_sums, cudaStream_t st) {
    k_chaos_grains<<<blocks_for(n), kBlock, 0, st>>>(n, pos3, grains.seg, grains.scenes, ref,
                                                     grain_vals);
    launch_segment_sums(grain_vals, n, 1, grains, grain_partials, grain_sums, st);
    k_chaos_nodes<<<blocks_for(total_nodes), kBlock, 0, st>>>(total_nodes, grid, nodes.seg,
                                                              nodes.scenes, ref, ny, nz, node_vals);
    launch_segment_sums(node_vals, total_nodes, 6, nodes, node_partials, node_sums, st);
}

}  // namespace wd
