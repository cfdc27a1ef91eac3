// probe.cu - device read bandwidth of a buffer, for the gather kernels' L2 roofline.
//
// The projector kernels read the field copy (64 MiB for a 256^3 FP32 volume, replicated
// corners included) mostly out of L1 and L2, so their bandwidth ceiling is the rate at
// which the SMs can read an L2-resident buffer, not the HBM copy rate.  A torch copy of an
// L2-resident buffer understates that rate (it also writes, and its launch shape is not
// chosen for it); this kernel only reads: every thread issues four independent 16-byte
// loads per iteration with the L1-bypassing .cg hint, over a grid of eight 256-thread
// blocks per SM, repeated `passes` times over the buffer in one launch.
#include "launch.h"

namespace dpt {
namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeBlocksPerSm = 8;
constexpr int kProbeUnroll = 4;

__global__ void __launch_bounds__(kProbeThreads) k_read_probe(const float4* __restrict__ buffer, int64_t quads,
                                                              int passes, float* __restrict__ sink)
{
    const int64_t stride = (int64_t)gridDim.x * kProbeThreads;
    float sum = 0.0f;
    for (int pass = 0; pass < passes; ++pass) {
        for (int64_t first = (int64_t)blockIdx.x * kProbeThreads + threadIdx.x; first < quads;
             first += stride * kProbeUnroll) {
            float4 v[kProbeUnroll];
#pragma unroll
            for (int u = 0; u < kProbeUnroll; ++u) {
                const int64_t index = first + u * stride;
                v[u] = index < quads ? __ldcg(buffer + index) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
#pragma unroll
            for (int u = 0; u < kProbeUnroll; ++u) sum += (v[u].x + v[u].y) + (v[u].z + v[u].w);
        }
    }
    // the loads must not be dead: a store that only a NaN sum takes
    if (sum != sum) sink[0] = sum;
}

}  // namespace
}  // namespace dpt

extern "C" int dpt_b200_read_probe(const void* buffer, int64_t bytes, int32_t passes, float* sink, void* stream)
{
    if (buffer == nullptr || sink == nullptr) return DPT_E_NULL;
    if (bytes <= 0 || bytes % 16 != 0 || passes < 1) return DPT_E_SHAPE;
    if (reinterpret_cast<uintptr_t>(buffer) % 16 != 0) return DPT_E_ALIGN;
    int device = 0, sms = 0;
    cudaError_t error = cudaGetDevice(&device);
    if (error == cudaSuccess) error = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (error != cudaSuccess) return (int)error;
    dpt::k_read_probe<<<sms * dpt::kProbeBlocksPerSm, dpt::kProbeThreads, 0, (cudaStream_t)stream>>>(
        static_cast<const float4*>(buffer), bytes / 16, passes, sink);
    return (int)cudaGetLastError();
}
