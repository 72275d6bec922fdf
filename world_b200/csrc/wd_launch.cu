// wd_launch.cu -- device-side launches of the Verlet-list build's CUDA graphs.
//
// In a list-mode semi-implicit Euler step the contact kernel decides at its end
// whether the lists must be rebuilt before the next step. A conditional node after it
// costs about 8 us of device time per step even when not taken; instead, one thread
// of a one-block kernel tail-launches the build's device-launchable graph only when the
// decision says so (the launched graph runs after the step's graph has completed, and
// the next step's graph waits for it). Inside the build, the same kind of kernel picks
// the mover path's or the radix path's graph after the mover sort.
//
// This is the only translation unit compiled with relocatable device code (the device
// runtime's cudaGraphLaunch): elsewhere -rdc would put the device ABI on the contact
// kernels and raise their spills.
#include "wd_kernels.h"

namespace wd {
namespace {

__global__ void k_graph_if(const uint32_t* __restrict__ flag, cudaGraphExec_t graph,
                           unsigned long long* __restrict__ counters) {
    if (threadIdx.x != 0 || *flag == 0u) return;
    if (cudaGraphLaunch(graph, cudaStreamGraphTailLaunch) != cudaSuccess)
        atomicAdd(&counters[kCntLaunchFail], 1ull);
}

__global__ void k_graph_pick(const int* __restrict__ flag, cudaGraphExec_t on_zero,
                             cudaGraphExec_t on_one, unsigned long long* __restrict__ counters) {
    if (threadIdx.x != 0) return;
    if (cudaGraphLaunch(*flag != 0 ? on_one : on_zero, cudaStreamGraphTailLaunch) != cudaSuccess)
        atomicAdd(&counters[kCntLaunchFail], 1ull);
}

}  // namespace

void launch_graph_if(const uint32_t* flag, cudaGraphExec_t graph, unsigned long long* counters,
                     cudaStream_t st) {
    k_graph_if<<<1, 32, 0, st>>>(flag, graph, counters);
}

void launch_graph_pick(const int* flag, cudaGraphExec_t on_zero, cudaGraphExec_t on_one,
                       unsigned long long* counters, cudaStream_t st) {
    k_graph_pick<<<1, 32, 0, st>>>(flag, on_zero, on_one, counters);
}

}  // namespace wd
