// launch.h - host launchers shared between the kernel translation units and the C ABI.
#pragma once

#include <cuda_runtime.h>

#include "../../include/dpt_b200.h"
#include "common.cuh"

namespace dpt {

// DPT_OK, or the DPT_E_* code of the first rule a problem (or its ray description) breaks.
int check_problem(const dpt_problem* p);
int check_rays(const dpt_problem* p, const dpt_rays* r);

// Fill a RayArgs record for views [view_begin, view_begin + view_count) and blocks of
// `threads` threads (kBlock for the forward and count kernels, kVjpBlock for the VJP).
RayArgs make_ray_args(const dpt_problem& p, const dpt_rays& r, int32_t* status, int threads);

// Detector columns per block tile (panels) and blocks per view for the ray kernels.
// Detector columns per block tile (panels), the columns a block of `threads` threads covers,
// and blocks per view for the ray kernels.
int block_cols(const dpt_problem& p);
int tile_cols(const dpt_problem& p, int threads);
int tiles_per_view(const dpt_problem& p, int* tiles_x, int threads);

cudaError_t launch_prepare_field(const dpt_problem& p, const void* field, void* packed,
                                 const double* poses, int32_t* status, cudaStream_t stream);
cudaError_t launch_forward(const dpt_problem& p, const RayArgs& a, const void* packed, void* image,
                           cudaStream_t stream);
// One launch over `count` problems that share arith, layout and image dtype.
cudaError_t launch_forward_packed(int count, const dpt_problem* problems, const RayArgs* args,
                                  const void* const* packed, void* const* images, cudaStream_t stream);
cudaError_t launch_counts(const dpt_problem& p, const RayArgs& a, double* lower, double* upper,
                          int32_t* realised, cudaStream_t stream);
cudaError_t launch_vjp(const dpt_problem& p, const RayArgs& a, const void* packed,
                       const void* cotangent, int flags, float* accumulator, double* partials,
                       cudaStream_t stream);
cudaError_t launch_forward_moments(const dpt_problem& p, const RayArgs& a, const void* packed,
                                   float* image, float* moments, int64_t stride, cudaStream_t stream);
cudaError_t launch_pose_from_moments(const dpt_problem& p, const RayArgs& a, const float* moments,
                                     int64_t stride, const void* cotangent, int flags,
                                     double* partials, cudaStream_t stream);
cudaError_t launch_finish_pose(int view_begin, int view_count, int tiles, int components,
                               const double* partials, double* gradient, int accumulate,
                               int32_t* status, cudaStream_t stream);
cudaError_t launch_fold(const dpt_problem& p, float* accumulator, double* total,
                        int accumulate_total, void* gradient, int gradient_dtype, int clear,
                        int32_t* status, cudaStream_t stream);

// Deterministic adjoint gather (gather.cu).  Plan layout (FP64 words): per view a header of
// kGatherHeaderWords (culling metrics, cone coefficients, cone flag), then per ray of every
// view a record of kGatherRayWords.
constexpr int kGatherHeaderWords = 32;
constexpr int kGatherColumnError = 0, kGatherRowError = 1, kGatherPointError = 2, kGatherFallback = 5,
              kGatherCoefficients = 6, kGatherCone = 18;
constexpr int kGatherRayWords = 16;
constexpr int kRayOrigin = 0, kRayDirection = 3, kRayLength = 6, kRayLower = 7, kRaySpan = 8, kRayStep = 9,
              kRayError = 10, kRayUpper = 13;

struct GatherArgs {
    Grid grid;
    int views;       // views of the plan (and of this call)
    int view_begin;  // first absolute view
    int rows, cols, samples, ray_kind;
    int cells;       // cell-Gauss integration (DPT_ARITH_CELLS) instead of midpoint samples
    const double* poses;       // absolute view indexing
    const double* view_table;  // absolute view indexing
    const double* ray_sources;
    const double* ray_endpoints;
    int32_t* status;           // absolute view indexing
};

cudaError_t launch_gather_prepare(const GatherArgs& a, double* plan, cudaStream_t stream);
cudaError_t launch_gather_count(const GatherArgs& a, const double* plan, int max_rays, unsigned long long* totals,
                                cudaStream_t stream);
cudaError_t launch_gather(const GatherArgs& a, const double* plan, const void* cotangent, int seed_dtype,
                          void* out, int out_dtype, int accumulate, cudaStream_t stream);

}  // namespace dpt
