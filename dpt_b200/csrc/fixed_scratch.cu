// fixed_scratch.cu - a pose-VJP entry point that allocates nothing.
//
// Some callers cannot call cudaMalloc once they are running: a pose-tracking loop in an
// interventional or robotic guidance process that reserves all of its device memory at
// start-up (an allocation can block on the device and break its latency budget), or a
// plugin hosted by an application that owns the GPU memory and hands out none.  For them
// dpt_b200_pose_vjp_fixed computes the per-view pose cotangent with its per-block FP64
// partials in the file-scope array below instead of caller-allocated scratch, reads the
// FP32 field directly (no corner-replicated copy) and allocates nothing.
//
// The array holds kPosePartialCapacity doubles (1 MiB) in every device that loads this
// library, for as long as the process lives.  Its name is only a host-side stand-in for
// the device symbol: host code must pass the device address, which every call looks up with
// cudaGetSymbolAddress on the current device (so a device reset between calls is harmless).
// The first call on a device also loads the library's device code there, so it should come
// before any stream capture.  All calls share the array, so calls whose work overlaps on the
// GPU (different streams, or different threads on the same device) race and must be
// serialised by the caller.  Every partial that a call reads is written by the same call
// first, so nothing needs clearing.
#include "launch.h"

static constexpr size_t kPosePartialCapacity = 1 << 17;  // doubles (1 MiB)
static __device__ __align__(256) double g_pose_partials[kPosePartialCapacity];

extern "C" int dpt_b200_pose_vjp_fixed(const dpt_problem* problem, const dpt_rays* rays,
                                       const float* field, const void* cotangent, int32_t components,
                                       double* pose_gradient, int32_t* status, void* stream)
{
    if (!field || !cotangent || !pose_gradient || !status) return DPT_E_NULL;
    if (components != 12 && components != 6) return DPT_E_FLAGS;
    int code = dpt::check_problem(problem);
    if (code != DPT_OK) return code;
    if (problem->field_dtype != DPT_F32) return DPT_E_DTYPE;
    // the mixed and fast samplings are fixed-pose forms
    if (problem->arith == DPT_ARITH_MIXED || problem->arith == DPT_ARITH_FAST) return DPT_E_FLAGS;
    dpt_problem direct = *problem;
    direct.layout = DPT_LAYOUT_DIRECT;  // sample the caller's field: no replicated copy
    if ((code = dpt::check_rays(&direct, rays)) != DPT_OK) return code;
    int tiles_x;
    const int tiles = dpt::tiles_per_view(direct, &tiles_x, dpt::kVjpBlock);
    if ((size_t)rays->view_count * (size_t)tiles * (size_t)components > kPosePartialCapacity)
        return DPT_E_CAPACITY;

    void* symbol = nullptr;
    cudaError_t error = cudaGetSymbolAddress(&symbol, g_pose_partials);
    if (error != cudaSuccess) return (int)error;
    double* partials = static_cast<double*>(symbol);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    // field scan and rigid-pose check only (a null copy pointer writes no scratch)
    error = dpt::launch_prepare_field(direct, field, nullptr, rays->poses, status, s);
    if (error != cudaSuccess) return (int)error;
    const dpt::RayArgs args = dpt::make_ray_args(direct, *rays, status, dpt::kVjpBlock);
    error = dpt::launch_vjp(direct, args, field, cotangent,
                            components == 12 ? DPT_VJP_POSE12 : DPT_VJP_POSE6, nullptr, partials, s);
    if (error != cudaSuccess) return (int)error;
    error = dpt::launch_finish_pose(rays->view_begin, rays->view_count, tiles, components, partials,
                                    pose_gradient, 0, status, s);
    return error == cudaSuccess ? DPT_OK : (int)error;
}
