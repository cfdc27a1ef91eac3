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
// Every accumulator slot is read by exactly one voxel thread, so the same thread clears
// it for the next batch.
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

// (cell, bit) pairs along one axis whose corner lands on coordinate x: min(c + b, n-1) == x
// with 0 <= c <= max(n-2, 0).
__device__ __forceinline__ int axis_sources(int x, int n, int* cells, int* bits)
{
    if (n == 1) {
        cells[0] = 0; bits[0] = 0;
        cells[1] = 0; bits[1] = 1;
        return 2;
    }
    int count = 0;
    if (x <= n - 2) { cells[count] = x; bits[count] = 0; ++count; }
    if (x >= 1) { cells[count] = x - 1; bits[count] = 1; ++count; }
    return count;
}

template <typename G>
__global__ void __launch_bounds__(256) k_fold(int nx, int ny, int nz, float* __restrict__ acc,
                                              double* __restrict__ total, int accumulate_total,
                                              G* __restrict__ gradient, int clear, int32_t* status)
{
    const int64_t voxels = (int64_t)nx * ny * nz;
    const int64_t index = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = false;
    if (index < voxels) {
        const int x = (int)(index % nx);
        const int64_t rest = index / nx;
        const int y = (int)(rest % ny), z = (int)(rest / ny);
        int cx[2], bx[2], cy[2], by[2], cz[2], bz[2];
        const int kx = axis_sources(x, nx, cx, bx);
        const int ky = axis_sources(y, ny, cy, by);
        const int kz = axis_sources(z, nz, cz, bz);
        double sum = 0.0;
        for (int iz = 0; iz < kz; ++iz)
            for (int iy = 0; iy < ky; ++iy)
                for (int ix = 0; ix < kx; ++ix) {
                    const int64_t cell = ((int64_t)cz[iz] * ny + cy[iy]) * nx + cx[ix];
                    float* slot = acc + 8 * cell + (bx[ix] | (by[iy] << 1) | (bz[iz] << 2));
                    sum += (double)*slot;
                    if (clear) *slot = 0.0f;
                }
        double value = sum;
        if (total) {
            if (accumulate_total) value += total[index];
            total[index] = value;
        }
        if (gradient) {
            const G out = (G)value;
            gradient[index] = out;
            bad = !isfinite(out);
        }
    }
    const unsigned any = __ballot_sync(0xffffffffu, bad);
    if (any && (threadIdx.x & 31) == 0) atomicOr(status, 2);
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
    const int64_t voxels = (int64_t)p.nx * p.ny * p.nz;
    const unsigned blocks = (unsigned)((voxels + 255) / 256);
    if (gradient_dtype == DPT_F64)
        k_fold<double><<<blocks, 256, 0, stream>>>(p.nx, p.ny, p.nz, accumulator, total,
                                                   accumulate_total, static_cast<double*>(gradient),
                                                   clear, status);
    else
        k_fold<float><<<blocks, 256, 0, stream>>>(p.nx, p.ny, p.nz, accumulator, total,
                                                  accumulate_total, static_cast<float*>(gradient),
                                                  clear, status);
    return cudaGetLastError();
}

}  // namespace dpt
