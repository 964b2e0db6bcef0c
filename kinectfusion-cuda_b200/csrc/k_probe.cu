// k_probe.cu -- an on-device read-bandwidth probe: the L2 (or HBM) figure the raycaster's
// gather rate is read against.  Not part of the reference's path.
#include "kf_host.h"

namespace kf {

// Every thread streams float4s of the buffer, round after round, through L2 (bypassing L1),
// and sums them.  A buffer under the 126 MB L2 stays resident after the first round.
__global__ void __launch_bounds__(256) read_probe_kernel(const float4* __restrict__ buf, long long n4, int rounds,
                                                         float* sink) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    float acc = 0.f;
    for (int r = 0; r < rounds; ++r)
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
            const float4 v = __ldcg(buf + i);
            acc += (v.x + v.y) + (v.z + v.w);
        }
    // a store that depends on every thread's sum keeps the loads; the buffer holds zeros, so
    // only thread 0 of each block writes
    if (threadIdx.x == 0 || acc == -1.0f) sink[blockIdx.x] = acc;
}

cudaError_t launch_read_probe(const float4* buf, long long n4, int rounds, float* sink, int grid, cudaStream_t st) {
    read_probe_kernel<<<grid, 256, 0, st>>>(buf, n4, rounds, sink);
    return cudaGetLastError();
}

}  // namespace kf
