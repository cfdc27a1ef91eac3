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
// the device symbol: host code must pass the device address, which the first call on each
// device obtains with cudaGetSymbolAddress while that device is current.  That first call
// therefore does a little set-up and should come before any stream capture.  All calls
// share the array, so calls whose work overlaps on the GPU (different streams, or
// different threads on the same device) race and must be serialised by the caller.  Every
// partial that a call reads is written by the same call first, so nothing needs clearing.
#include <mutex>

#include "launch.h"

static constexpr size_t kPosePartialCapacity = 1 << 17;  // doubles (1 MiB)
static __device__ __align__(256) double g_pose_partials[kPosePartialCapacity];

namespace {

constexpr int kMaxDevices = 64;

std::mutex g_setup_mutex;
double* g_partials_address[kMaxDevices] = {};

// Device address of g_pose_partials on the current device (looked up once per device).
int partials_address(double** address)
{
    int device = -1;
    cudaError_t error = cudaGetDevice(&device);
    if (error != cudaSuccess) return (int)error;
    if (device < 0 || device >= kMaxDevices) return DPT_E_RANGE;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_address[device]) {
        void* symbol = nullptr;
        error = cudaGetSymbolAddress(&symbol, g_pose_partials);
        if (error != cudaSuccess) return (int)error;
        g_partials_address[device] = static_cast<double*>(symbol);
    }
    *address = g_partials_address[device];
    return DPT_OK;
}

}  // namespace

extern "C" int dpt_b200_pose_vjp_fixed(const dpt_problem* problem, const dpt_rays* rays,
                                       const float* field, const void* cotangent, int32_t components,
                                       double* pose_gradient, int32_t* status, void* stream)
{
    if (!problem || !rays || !field || !cotangent || !pose_gradient || !status || !rays->poses)
        return DPT_E_NULL;
    if (problem->field_dtype != DPT_F32) return DPT_E_DTYPE;
    if (components != 12 && components != 6) return DPT_E_FLAGS;
    // the mixed and fast samplings are fixed-pose forms
    if (problem->arith == DPT_ARITH_MIXED || problem->arith == DPT_ARITH_FAST) return DPT_E_FLAGS;
    dpt_problem direct = *problem;
    direct.layout = DPT_LAYOUT_DIRECT;  // sample the caller's field: no replicated copy
    // the size query returns 0 for every problem the other entry points reject
    if (dpt_b200_accumulator_bytes(&direct) == 0) return DPT_E_SHAPE;
    if (rays->view_begin < 0 || rays->view_count < 1 ||
        rays->view_begin + (int64_t)rays->view_count > direct.views || rays->view_count > 65535)
        return DPT_E_RANGE;
    if (direct.ray_kind == DPT_RAYS_PANELS ? !rays->view_table
                                           : (!rays->ray_sources || !rays->ray_endpoints))
        return DPT_E_NULL;
    int tiles_x;
    const int tiles = dpt::tiles_per_view(direct, &tiles_x, dpt::kVjpBlock);
    if ((size_t)rays->view_count * (size_t)tiles * (size_t)components > kPosePartialCapacity)
        return DPT_E_CAPACITY;

    double* partials = nullptr;
    int code = partials_address(&partials);
    if (code != DPT_OK) return code;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    // field scan and rigid-pose check only (a null copy pointer writes no scratch)
    cudaError_t error = dpt::launch_prepare_field(direct, field, nullptr, rays->poses, status, s);
    if (error != cudaSuccess) return (int)error;
    const dpt::RayArgs args = dpt::make_ray_args(direct, *rays, status, dpt::kVjpBlock);
    error = dpt::launch_vjp(direct, args, field, cotangent,
                            components == 12 ? DPT_VJP_POSE12 : DPT_VJP_POSE6, nullptr, partials, s);
    if (error != cudaSuccess) return (int)error;
    error = dpt::launch_finish_pose(rays->view_begin, rays->view_count, tiles, components, partials,
                                    pose_gradient, 0, status, s);
    return error == cudaSuccess ? DPT_OK : (int)error;
}
