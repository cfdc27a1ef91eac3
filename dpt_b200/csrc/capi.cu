// capi.cu - extern "C" entry points: argument checks, then kernel launches on the caller's
// stream.  No entry point allocates device or host memory.
#include <cstdint>

#include "launch.h"

namespace dpt {

int block_cols(const dpt_problem& p) { return p.block_cols == 0 ? kDefaultBlockCols : p.block_cols; }

int tile_cols(const dpt_problem& p, int threads)
{
    const int cols = block_cols(p);
    return cols * 4 <= threads ? cols : threads / 4;  // at least one 8x4 warp tile per row band
}

int tiles_per_view(const dpt_problem& p, int* tiles_x, int threads)
{
    if (p.ray_kind == DPT_RAYS_BUNDLE) {
        const int64_t rays = (int64_t)p.rows * p.cols;
        *tiles_x = (int)((rays + threads - 1) / threads);
        return *tiles_x;
    }
    const int cols = tile_cols(p, threads), rows = threads / cols;
    *tiles_x = (p.cols + cols - 1) / cols;
    const int tiles_y = (p.rows + rows - 1) / rows;
    return *tiles_x * tiles_y;
}

RayArgs make_ray_args(const dpt_problem& p, const dpt_rays& r, int32_t* status, int threads)
{
    RayArgs a;
    a.grid.nx = p.nx;
    a.grid.ny = p.ny;
    a.grid.nz = p.nz;
    for (int k = 0; k < 9; ++k) a.grid.m[k] = p.object_to_grid[k];
    for (int k = 0; k < 3; ++k) a.grid.g0[k] = p.grid_origin[k];
    a.views = r.view_count;
    a.view_begin = r.view_begin;
    a.rows = p.rows;
    a.cols = p.cols;
    a.samples = p.samples;
    a.ray_kind = p.ray_kind;
    a.tiles_per_view = tiles_per_view(p, &a.tiles_x, threads);
    a.block_threads = threads;
    a.block_cols = tile_cols(p, threads);
    a.block_rows = threads / a.block_cols;
    a.warps_x = a.block_cols / 8;
    a.view_group = DPT_VIEW_GROUP;
    a.poses = r.poses;
    a.view_table = r.view_table;
    a.ray_sources = r.ray_sources;
    a.ray_endpoints = r.ray_endpoints;
    a.status = status;
    return a;
}

// Argument checks shared by every entry point that takes a problem and rays.
constexpr int64_t kMaxIndex = 2147483647;  // signed 32-bit indexing, as the reference

int check_problem(const dpt_problem* p)
{
    if (!p) return DPT_E_NULL;
    if (p->nx < 1 || p->ny < 1 || p->nz < 1 || p->views < 1 || p->rows < 1 || p->cols < 1 ||
        p->samples < 1)
        return DPT_E_SHAPE;
    const int64_t voxels = (int64_t)p->nx * p->ny * p->nz;
    if (voxels > kMaxIndex || (int64_t)p->rows * p->cols > kMaxIndex ||
        (int64_t)p->rows * p->cols * p->views > kMaxIndex * 4)
        return DPT_E_SHAPE;
    if (p->ray_kind != DPT_RAYS_PANELS && p->ray_kind != DPT_RAYS_BUNDLE) return DPT_E_FLAGS;
    if (p->image_dtype != DPT_F32 && p->image_dtype != DPT_F64) return DPT_E_DTYPE;
    if (p->field_dtype != DPT_F32 && p->field_dtype != DPT_F16 && p->field_dtype != DPT_BF16)
        return DPT_E_DTYPE;
    if (p->arith < DPT_ARITH_F32 || p->arith > DPT_ARITH_CELLS) return DPT_E_DTYPE;
    // the reference FP32 arithmetic reads FP32 storage (reference ProjectionSpec rule); the
    // others decode FP16/BF16 values in the pack kernel
    if (p->field_dtype != DPT_F32 && p->arith == DPT_ARITH_F32) return DPT_E_DTYPE;
    if (p->field_domain != DPT_DOMAIN_PHYSICAL && p->field_domain != DPT_DOMAIN_SIGNED) return DPT_E_FLAGS;
    if (p->layout != DPT_LAYOUT_REPLICATED && p->layout != DPT_LAYOUT_DIRECT) return DPT_E_FLAGS;
    if (p->layout == DPT_LAYOUT_DIRECT && p->field_dtype != DPT_F32) return DPT_E_DTYPE;
    if (p->block_cols != 0 && p->block_cols != 8 && p->block_cols != 16 && p->block_cols != 32 &&
        p->block_cols != 64)
        return DPT_E_FLAGS;
    // FP32 grid coordinates are exact integers only up to 2^24 (reference projection.py:548).
    if (p->arith != DPT_ARITH_F64 && p->arith != DPT_ARITH_CELLS &&
        (p->nx > (1 << 24) || p->ny > (1 << 24) || p->nz > (1 << 24)))
        return DPT_E_SHAPE;
    return DPT_OK;
}

int check_rays(const dpt_problem* p, const dpt_rays* r)
{
    if (!r || !r->poses) return DPT_E_NULL;
    if (r->view_begin < 0 || r->view_count < 1 || r->view_begin + (int64_t)r->view_count > p->views)
        return DPT_E_RANGE;
    if (p->ray_kind == DPT_RAYS_PANELS && !r->view_table) return DPT_E_NULL;
    if (p->ray_kind == DPT_RAYS_BUNDLE && (!r->ray_sources || !r->ray_endpoints)) return DPT_E_NULL;
    return DPT_OK;
}

}  // namespace dpt

namespace {

using dpt::check_problem;
using dpt::check_rays;

constexpr int kMaxViewsPerLaunch = 65535;   // views per launch of the ray kernels

bool aligned(const void* p, uintptr_t bytes) { return (reinterpret_cast<uintptr_t>(p) % bytes) == 0; }

int to_code(cudaError_t e) { return e == cudaSuccess ? DPT_OK : (int)e; }

// Launch `body` on chunks of at most kMaxViewsPerLaunch views, and few enough that the 1-D
// grid of views x tiles stays below 2^31 blocks.
template <typename Body>
int chunked(const dpt_problem* p, const dpt_rays* r, int32_t* status, int threads, Body body)
{
    int tiles_x;
    const int64_t tiles = dpt::tiles_per_view(*p, &tiles_x, threads);
    const int64_t by_grid = ((int64_t)1 << 31) / (tiles > 0 ? tiles : 1) - 1;
    const int32_t most = (int32_t)(by_grid < kMaxViewsPerLaunch ? (by_grid < 1 ? 1 : by_grid) : kMaxViewsPerLaunch);
    for (int32_t first = 0; first < r->view_count; first += most) {
        dpt_rays part = *r;
        part.view_begin = r->view_begin + first;
        part.view_count = r->view_count - first < most ? r->view_count - first : most;
        const dpt::RayArgs a = dpt::make_ray_args(*p, part, status, threads);
        const int code = body(a, first);
        if (code != DPT_OK) return code;
    }
    return DPT_OK;
}

}  // namespace

extern "C" {

int dpt_b200_abi_version(void) { return DPT_B200_ABI_VERSION; }

const char* dpt_b200_error_string(int code)
{
    switch (code) {
    case DPT_OK: return "ok";
    case DPT_E_NULL: return "a required pointer is null";
    case DPT_E_SHAPE: return "a size is out of range";
    case DPT_E_DTYPE: return "unsupported dtype or arithmetic combination";
    case DPT_E_FLAGS: return "inconsistent flags";
    case DPT_E_RANGE: return "view range outside the problem";
    case DPT_E_ALIGN: return "a pointer is not aligned as required";
    case DPT_E_CAPACITY: return "a fixed-capacity buffer is too small";
    default: return code > 0 ? cudaGetErrorString((cudaError_t)code) : "unknown error";
    }
}

size_t dpt_b200_packed_bytes(const dpt_problem* p)
{
    if (check_problem(p) != DPT_OK) return 0;
    if (p->layout == DPT_LAYOUT_DIRECT) return 0;
    // compensated form: two float4 of polynomial coefficients per cell; else one 16-byte record
    if (p->arith == DPT_ARITH_F32C) return (size_t)p->nx * p->ny * p->nz * 32u;
    return (size_t)p->nx * p->ny * p->nz * 16u;
}

size_t dpt_b200_accumulator_bytes(const dpt_problem* p)
{
    if (check_problem(p) != DPT_OK) return 0;
    return (size_t)p->nx * p->ny * p->nz * 32u;
}

size_t dpt_b200_pose_partials_bytes(const dpt_problem* p, int32_t view_count)
{
    if (check_problem(p) != DPT_OK || view_count < 1) return 0;
    int tiles_x;
    const int tiles = dpt::tiles_per_view(*p, &tiles_x, dpt::kVjpBlock);
    return (size_t)view_count * tiles * 12u * sizeof(double);
}

int dpt_b200_prepare_field(const dpt_problem* p, const void* field, void* packed,
                           const double* poses, int32_t* status, void* stream)
{
    int code = check_problem(p);
    if (code != DPT_OK) return code;
    if (!field || !poses || !status) return DPT_E_NULL;
    if (p->layout == DPT_LAYOUT_DIRECT) packed = nullptr;
    if (packed && !aligned(packed, 16)) return DPT_E_ALIGN;
    return to_code(dpt::launch_prepare_field(*p, field, packed, poses, status,
                                             static_cast<cudaStream_t>(stream)));
}

int dpt_b200_forward(const dpt_problem* p, const dpt_rays* r, const void* packed, void* image,
                     int32_t* status, void* stream)
{
    int code = check_problem(p);
    if (code != DPT_OK) return code;
    if ((code = check_rays(p, r)) != DPT_OK) return code;
    if (!packed || !image || !status) return DPT_E_NULL;
    if (!aligned(packed, 16)) return DPT_E_ALIGN;
    const int64_t rays_per_view = (int64_t)p->rows * p->cols;
    const size_t element = p->image_dtype == DPT_F64 ? 8 : 4;
    return chunked(p, r, status, dpt::kForwardBlock, [&](const dpt::RayArgs& a, int32_t first) {
        char* out = static_cast<char*>(image) + (size_t)first * rays_per_view * element;
        return to_code(dpt::launch_forward(*p, a, packed, out, static_cast<cudaStream_t>(stream)));
    });
}

int dpt_b200_forward_packed(int32_t count, const dpt_problem* problems, const dpt_rays* rays,
                            const void* const* packed, void* const* images, int32_t* const* status, void* stream)
{
    if (count < 1) return DPT_E_SHAPE;
    if (count > DPT_MAX_PACK) return DPT_E_CAPACITY;
    if (!problems || !rays || !packed || !images || !status) return DPT_E_NULL;
    dpt::RayArgs args[DPT_MAX_PACK];
    for (int32_t k = 0; k < count; ++k) {
        const dpt_problem* p = problems + k;
        int code = check_problem(p);
        if (code != DPT_OK) return code;
        if ((code = check_rays(p, rays + k)) != DPT_OK) return code;
        if (!packed[k] || !images[k] || !status[k]) return DPT_E_NULL;
        if (!aligned(packed[k], 16)) return DPT_E_ALIGN;
        // one kernel instantiation serves the pack
        if (p->arith != problems[0].arith || p->layout != problems[0].layout ||
            p->image_dtype != problems[0].image_dtype)
            return DPT_E_FLAGS;
        if (rays[k].view_count > kMaxViewsPerLaunch) return DPT_E_RANGE;
        args[k] = dpt::make_ray_args(*p, rays[k], status[k], dpt::kForwardBlock);
    }
    return to_code(dpt::launch_forward_packed(count, problems, args, packed, images, static_cast<cudaStream_t>(stream)));
}

size_t dpt_b200_moments_bytes(const dpt_problem* p, int32_t view_count)
{
    if (check_problem(p) != DPT_OK || view_count < 1) return 0;
    return (size_t)9 * sizeof(float) * (size_t)view_count * (size_t)p->rows * (size_t)p->cols;
}

int dpt_b200_forward_moments(const dpt_problem* p, const dpt_rays* r, const void* packed, float* image,
                             float* moments, int32_t* status, void* stream)
{
    int code = check_problem(p);
    if (code != DPT_OK) return code;
    if ((code = check_rays(p, r)) != DPT_OK) return code;
    if ((p->arith != DPT_ARITH_F32 && p->arith != DPT_ARITH_F32C) || p->image_dtype != DPT_F32)
        return DPT_E_DTYPE;
    if (!packed || !image || !moments || !status) return DPT_E_NULL;
    if (!aligned(packed, 16)) return DPT_E_ALIGN;
    const int64_t rays_per_view = (int64_t)p->rows * p->cols;
    const int64_t stride = rays_per_view * r->view_count;
    return chunked(p, r, status, dpt::kVjpBlock, [&](const dpt::RayArgs& a, int32_t first) {
        const int64_t offset = (int64_t)first * rays_per_view;
        return to_code(dpt::launch_forward_moments(*p, a, packed, image + offset, moments + offset, stride,
                                                   static_cast<cudaStream_t>(stream)));
    });
}

int dpt_b200_pose_from_moments(const dpt_problem* p, const dpt_rays* r, const float* moments,
                               const void* cotangent, int32_t flags, double* pose_partials,
                               int32_t* status, void* stream)
{
    int code = check_problem(p);
    if (code != DPT_OK) return code;
    if ((code = check_rays(p, r)) != DPT_OK) return code;
    if (p->arith != DPT_ARITH_F32 && p->arith != DPT_ARITH_F32C) return DPT_E_DTYPE;
    if (!moments || !cotangent || !pose_partials || !status) return DPT_E_NULL;
    if (flags != DPT_VJP_POSE12 && flags != DPT_VJP_POSE6 && flags != DPT_VJP_PER_RAY6) return DPT_E_FLAGS;
    const int64_t rays_per_view = (int64_t)p->rows * p->cols;
    const int64_t stride = rays_per_view * r->view_count;
    const size_t element = p->image_dtype == DPT_F64 ? 8 : 4;
    int tiles_x;
    const int tiles = dpt::tiles_per_view(*p, &tiles_x, dpt::kVjpBlock);
    return chunked(p, r, status, dpt::kVjpBlock, [&](const dpt::RayArgs& a, int32_t first) {
        const int64_t offset = (int64_t)first * rays_per_view;
        const char* seed = static_cast<const char*>(cotangent) + (size_t)offset * element;
        const int64_t per_view = (flags & DPT_VJP_PER_RAY6) ? rays_per_view * 6
                                 : (int64_t)tiles * ((flags & DPT_VJP_POSE12) ? 12 : 6);
        return to_code(dpt::launch_pose_from_moments(*p, a, moments + offset, stride, seed, flags,
                                                     pose_partials + (int64_t)first * per_view,
                                                     static_cast<cudaStream_t>(stream)));
    });
}

int dpt_b200_vjp(const dpt_problem* p, const dpt_rays* r, const void* packed,
                 const void* cotangent, int32_t flags, float* accumulator, double* pose_partials,
                 int32_t* status, void* stream)
{
    int code = check_problem(p);
    if (code != DPT_OK) return code;
    if ((code = check_rays(p, r)) != DPT_OK) return code;
    if (!packed || !cotangent || !status) return DPT_E_NULL;
    if (!aligned(packed, 16)) return DPT_E_ALIGN;
    const int pose_bits = flags & (DPT_VJP_POSE12 | DPT_VJP_POSE6 | DPT_VJP_PER_RAY6);
    if (flags & ~(DPT_VJP_VOLUME | DPT_VJP_POSE12 | DPT_VJP_POSE6 | DPT_VJP_PER_RAY6))
        return DPT_E_FLAGS;
    if (!(flags & DPT_VJP_VOLUME) && !pose_bits) return DPT_E_FLAGS;
    if (pose_bits && (pose_bits & (pose_bits - 1))) return DPT_E_FLAGS;  // one pose form
    if ((flags & DPT_VJP_PER_RAY6) && (flags & DPT_VJP_VOLUME)) return DPT_E_FLAGS;
    // the mixed and fast samplings are fixed-pose forms (reference ProjectionSpec rule)
    if (pose_bits && (p->arith == DPT_ARITH_MIXED || p->arith == DPT_ARITH_FAST)) return DPT_E_FLAGS;
    if ((flags & DPT_VJP_VOLUME) && !accumulator) return DPT_E_NULL;
    if (accumulator && !aligned(accumulator, 32)) return DPT_E_ALIGN;
    if (pose_bits && !pose_partials) return DPT_E_NULL;
    const int64_t rays_per_view = (int64_t)p->rows * p->cols;
    const size_t element = p->image_dtype == DPT_F64 ? 8 : 4;
    int tiles_x;
    const int tiles = dpt::tiles_per_view(*p, &tiles_x, dpt::kVjpBlock);
    return chunked(p, r, status, dpt::kVjpBlock, [&](const dpt::RayArgs& a, int32_t first) {
        const char* seed = static_cast<const char*>(cotangent) + (size_t)first * rays_per_view * element;
        double* partials = pose_partials;
        if (partials) {
            const int64_t per_view = (flags & DPT_VJP_PER_RAY6) ? rays_per_view * 6
                                     : (int64_t)tiles * ((flags & DPT_VJP_POSE12) ? 12 : 6);
            partials += (int64_t)first * per_view;
        }
        return to_code(dpt::launch_vjp(*p, a, packed, seed, flags, accumulator, partials,
                                       static_cast<cudaStream_t>(stream)));
    });
}

int dpt_b200_finish_pose(const dpt_problem* p, int32_t view_begin, int32_t view_count,
                         int32_t components,
                         const double* pose_partials, double* pose_gradient, int32_t accumulate,
                         int32_t* status, void* stream)
{
    int code = check_problem(p);
    if (code != DPT_OK) return code;
    if (!pose_partials || !pose_gradient || !status) return DPT_E_NULL;
    if (components != 12 && components != 6) return DPT_E_FLAGS;
    if (view_begin < 0 || view_count < 1 || view_begin + (int64_t)view_count > p->views)
        return DPT_E_RANGE;
    int tiles_x;
    const int tiles = dpt::tiles_per_view(*p, &tiles_x, dpt::kVjpBlock);
    return to_code(dpt::launch_finish_pose(view_begin, view_count, tiles, components, pose_partials,
                                           pose_gradient, accumulate, status,
                                           static_cast<cudaStream_t>(stream)));
}

int dpt_b200_fold_volume(const dpt_problem* p, float* accumulator, double* total,
                         int32_t accumulate_total, void* gradient, int32_t gradient_dtype,
                         int32_t clear, int32_t* status, void* stream)
{
    int code = check_problem(p);
    if (code != DPT_OK) return code;
    if (!accumulator || !status) return DPT_E_NULL;
    if (!total && !gradient) return DPT_E_NULL;
    if (gradient && gradient_dtype != DPT_F32 && gradient_dtype != DPT_F64) return DPT_E_DTYPE;
    return to_code(dpt::launch_fold(*p, accumulator, total, accumulate_total, gradient,
                                    gradient_dtype, clear, status,
                                    static_cast<cudaStream_t>(stream)));
}

int dpt_b200_counts(const dpt_problem* p, const dpt_rays* r, double* lower, double* upper,
                    int32_t* realised, int32_t* status, void* stream)
{
    int code = check_problem(p);
    if (code != DPT_OK) return code;
    if ((code = check_rays(p, r)) != DPT_OK) return code;
    if (!lower || !upper || !realised || !status) return DPT_E_NULL;
    const int64_t rays_per_view = (int64_t)p->rows * p->cols;
    return chunked(p, r, status, dpt::kBlock, [&](const dpt::RayArgs& a, int32_t first) {
        const int64_t offset = (int64_t)first * rays_per_view;
        return to_code(dpt::launch_counts(*p, a, lower + offset, upper + offset, realised + offset,
                                          static_cast<cudaStream_t>(stream)));
    });
}

// ------------------------------------------------------------ deterministic adjoint gather

namespace {

int check_gather(const dpt_problem* p, const dpt_rays* r)
{
    int code = check_problem(p);
    if (code != DPT_OK) return code;
    if ((code = check_rays(p, r)) != DPT_OK) return code;
    // the canonical weights of the gather are the strict FP64 forward's (midpoint or cell-Gauss)
    if (p->arith != DPT_ARITH_F64 && p->arith != DPT_ARITH_CELLS) return DPT_E_DTYPE;
    return DPT_OK;
}

dpt::GatherArgs gather_args(const dpt_problem& p, const dpt_rays& r, int32_t* status)
{
    dpt::GatherArgs a;
    a.grid.nx = p.nx;
    a.grid.ny = p.ny;
    a.grid.nz = p.nz;
    for (int k = 0; k < 9; ++k) a.grid.m[k] = p.object_to_grid[k];
    for (int k = 0; k < 3; ++k) a.grid.g0[k] = p.grid_origin[k];
    a.views = r.view_count;
    a.view_begin = r.view_begin;
    a.rows = p.rows;
    a.cols = p.cols;
    a.samples = p.samples;
    a.ray_kind = p.ray_kind;
    a.cells = p.arith == DPT_ARITH_CELLS;
    a.poses = r.poses;
    a.view_table = r.view_table;
    a.ray_sources = r.ray_sources;
    a.ray_endpoints = r.ray_endpoints;
    a.status = status;
    return a;
}

}  // namespace

size_t dpt_b200_gather_plan_bytes(const dpt_problem* p, int32_t view_count)
{
    if (check_problem(p) != DPT_OK || view_count < 1 || view_count > p->views) return 0;
    const size_t words = (size_t)view_count * dpt::kGatherHeaderWords +
                         (size_t)view_count * p->rows * p->cols * dpt::kGatherRayWords;
    return words * sizeof(double);
}

int dpt_b200_gather_prepare(const dpt_problem* p, const dpt_rays* r, double* plan, int32_t* status, void* stream)
{
    int code = check_gather(p, r);
    if (code != DPT_OK) return code;
    if (!plan || !status) return DPT_E_NULL;
    if (!aligned(plan, 8)) return DPT_E_ALIGN;
    if (r->view_count > kMaxViewsPerLaunch) return DPT_E_SHAPE;
    return to_code(dpt::launch_gather_prepare(gather_args(*p, *r, status), plan, static_cast<cudaStream_t>(stream)));
}

int dpt_b200_gather_count(const dpt_problem* p, const dpt_rays* r, const double* plan, int32_t max_rays_per_voxel,
                          int64_t* totals, void* stream)
{
    int code = check_gather(p, r);
    if (code != DPT_OK) return code;
    if (!plan || !totals) return DPT_E_NULL;
    if (p->arith != DPT_ARITH_F64) return DPT_E_DTYPE;  // sample culling is for midpoint plans
    if (max_rays_per_voxel < 1) return DPT_E_SHAPE;
    if (!aligned(plan, 8) || !aligned(totals, 8)) return DPT_E_ALIGN;
    return to_code(dpt::launch_gather_count(gather_args(*p, *r, nullptr), plan, max_rays_per_voxel,
                                            reinterpret_cast<unsigned long long*>(totals),
                                            static_cast<cudaStream_t>(stream)));
}

int dpt_b200_gather(const dpt_problem* p, const dpt_rays* r, const double* plan, const void* cotangent,
                    void* gradient, int32_t gradient_dtype, int32_t accumulate, int32_t* status, void* stream)
{
    int code = check_gather(p, r);
    if (code != DPT_OK) return code;
    if (!plan || !cotangent || !gradient || !status) return DPT_E_NULL;
    if (gradient_dtype != DPT_F32 && gradient_dtype != DPT_F64) return DPT_E_DTYPE;
    if (!aligned(plan, 8)) return DPT_E_ALIGN;
    return to_code(dpt::launch_gather(gather_args(*p, *r, status), plan, cotangent, p->image_dtype, gradient,
                                      gradient_dtype, accumulate, static_cast<cudaStream_t>(stream)));
}

}  // extern "C"
