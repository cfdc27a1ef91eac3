// reduce.cu - per-view pose reduction and the fold of the per-cell volume accumulator.
//
// finish_pose replaces the reference's FP64 tile tree (python/dpt/_reductions.py:27-63,
// python/dpt/kernels/reductions.py:11-61): one block per view reduces that view's block
// partials in a fixed order, so the result is deterministic.
//
// fold gathers, for every voxel, the corner slots of the (up to eight) cells that touch
// it, sums them in FP64 in a fixed order and optionally adds them into an FP64 running
// total.  This is where the FP32 per-batch sums are widened to FP64, as the reference
// does every 8 views (python/dpt/torch/_projection_ops.py:304-352).  The final pass also
// scans the gradient for non-finite values (reference python/dpt/projection.py:470-499).
// Each warp walks 31-voxel columns up z with the cell records in registers; the accumulator
// is then cleared for the next batch with one memset (fold + clear of a 256^3 batch 0.24 ms;
// a shared-memory staged 16x4x16 tile took 0.45 ms, bound by its staging and index math).
#include "launch.h"

namespace dpt {
namespace {

__global__ void __launch_bounds__(256) k_finish_pose(int view_begin, int tiles, int components,
                                                     const double* __restrict__ partials,
                                                     double* __restrict__ gradient,
                                                     int accumulate, int32_t* status)
{
    __shared__ double tree[256];
    const int view = blockIdx.x;
    const double* base = partials + (int64_t)view * tiles * components;
    for (int k = 0; k < components; ++k) {
        double s = 0.0;
        for (int b = threadIdx.x; b < tiles; b += 256) s += base[(int64_t)b * components + k];
        tree[threadIdx.x] = s;
        __syncthreads();
        for (int width = 128; width > 0; width >>= 1) {
            if (threadIdx.x < width) tree[threadIdx.x] += tree[threadIdx.x + width];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            double value = tree[0];
            double* out = gradient + (int64_t)view * components + k;
            if (accumulate) value += *out;
            *out = value;
            if (!isfinite(value)) atomicOr(status + view_begin + view, 2);
        }
        __syncthreads();
    }
}

// A warp folds 31 consecutive voxels in x (lane l >= 1 folds voxel
// x0 + l - 1 and holds the records of that voxel's own cell; lane 0 holds the cell below the
// first voxel), one y row per warp (eight per block), and walks kColumnDepth voxels up z.
// Each step loads the two cell rows (y and y - 1) at z and keeps the two rows at z - 1 from
// the step before, so a record is loaded twice (by the warps of rows y and y + 1, which share
// the block's L1) and the bit-1 x slots come from the lane below by shuffle.  The eight
// slots are summed in a fixed order (z bit 0 before bit 1, then y, then x);
// a source that does not exist (past an edge, or the never-written cells at n - 1) reads as
// +0, which leaves the FP64 sum unchanged (it starts at +0 and never becomes -0).
constexpr int kColumnLanes = 31, kColumnWarps = 8, kColumnDepth = 16;

__device__ __forceinline__ void load_record(const float4* records, int64_t cell, bool valid, float* s)
{
    float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f), b = a;
    if (valid) {
        a = __ldg(records + 2 * cell);
        b = __ldg(records + 2 * cell + 1);
    }
    s[0] = a.x; s[1] = a.y; s[2] = a.z; s[3] = a.w;
    s[4] = b.x; s[5] = b.y; s[6] = b.z; s[7] = b.w;
}

template <typename G>
__global__ void __launch_bounds__(256) k_fold_columns(int nx, int ny, int nz, const float* __restrict__ acc,
                                                      double* __restrict__ total, int accumulate_total,
                                                      G* __restrict__ gradient, int32_t* status)
{
    const int tiles_x = (nx + kColumnLanes - 1) / kColumnLanes, tiles_y = (ny + kColumnWarps - 1) / kColumnWarps;
    const int tile = blockIdx.x;
    const int tz = tile / (tiles_x * tiles_y), rest = tile - tz * tiles_x * tiles_y;
    const int ty = rest / tiles_x, tx = rest - ty * tiles_x;
    const int lane = threadIdx.x & 31;
    const int x = tx * kColumnLanes + lane - 1;
    const int y = ty * kColumnWarps + (threadIdx.x >> 5);
    const int z_begin = tz * kColumnDepth, z_end = min(z_begin + kColumnDepth, nz);
    const float4* records = reinterpret_cast<const float4*>(acc);
    // the cells whose bit-1 y / z corners land on this voxel (the voxel's own cell on a
    // one-cell axis)
    const int ym = ny == 1 ? 0 : y - 1;
    const bool own_ok = x >= 0 && x < nx && y < ny;
    const bool minus_ok = own_ok && ym >= 0;
    const bool folds = lane >= 1 && x < nx && y < ny;
    auto cell = [&](int cy, int cz) { return ((int64_t)cz * ny + cy) * nx + x; };
    float own_prev[8], minus_prev[8], own_cur[8], minus_cur[8];
    const int zm = nz == 1 ? 0 : z_begin - 1;
    load_record(records, cell(y, zm), own_ok && zm >= 0, own_prev);
    load_record(records, cell(ym, zm), minus_ok && zm >= 0, minus_prev);
    const bool single_x = nx == 1;
    auto below = [&](float v) {
        const float w = __shfl_up_sync(0xffffffffu, v, 1);
        return single_x ? v : w;
    };
    bool bad = false;
    for (int z = z_begin; z < z_end; ++z) {
        load_record(records, cell(y, z), own_ok, own_cur);
        load_record(records, cell(ym, z), minus_ok, minus_cur);
        const float x1[4] = {below(own_cur[1]), below(minus_cur[3]), below(own_prev[5]), below(minus_prev[7])};
        double sum = 0.0;
        sum += (double)own_cur[0];
        sum += (double)x1[0];
        sum += (double)minus_cur[2];
        sum += (double)x1[1];
        sum += (double)own_prev[4];
        sum += (double)x1[2];
        sum += (double)minus_prev[6];
        sum += (double)x1[3];
        if (folds) {
            const int64_t index = ((int64_t)z * ny + y) * nx + x;
            double value = sum;
            if (total) {
                if (accumulate_total) value += total[index];
                total[index] = value;
            }
            if (gradient) {
                const G out = (G)value;
                gradient[index] = out;
                bad = bad || !isfinite(out);
            }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            own_prev[k] = own_cur[k];
            minus_prev[k] = minus_cur[k];
        }
    }
    const unsigned any = __ballot_sync(0xffffffffu, bad);
    if (any && lane == 0) atomicOr(status, 2);
}

}  // namespace

cudaError_t launch_finish_pose(int view_begin, int view_count, int tiles, int components,
                               const double* partials, double* gradient, int accumulate,
                               int32_t* status, cudaStream_t stream)
{
    k_finish_pose<<<view_count, 256, 0, stream>>>(view_begin, tiles, components, partials,
                                                  gradient, accumulate, status);
    return cudaGetLastError();
}

cudaError_t launch_fold(const dpt_problem& p, float* accumulator, double* total,
                        int accumulate_total, void* gradient, int gradient_dtype, int clear,
                        int32_t* status, cudaStream_t stream)
{
    const unsigned blocks = (unsigned)(((p.nx + kColumnLanes - 1) / kColumnLanes) *
                                       ((p.ny + kColumnWarps - 1) / kColumnWarps) *
                                       ((p.nz + kColumnDepth - 1) / kColumnDepth));
    if (gradient_dtype == DPT_F64)
        k_fold_columns<double><<<blocks, 256, 0, stream>>>(p.nx, p.ny, p.nz, accumulator, total,
                                                          accumulate_total, static_cast<double*>(gradient), status);
    else
        k_fold_columns<float><<<blocks, 256, 0, stream>>>(p.nx, p.ny, p.nz, accumulator, total,
                                                         accumulate_total, static_cast<float*>(gradient), status);
    cudaError_t error = cudaGetLastError();
    if (error == cudaSuccess && clear)
        error = cudaMemsetAsync(accumulator, 0, (size_t)p.nx * p.ny * p.nz * 32u, stream);
    return error;
}

}  // namespace dpt
