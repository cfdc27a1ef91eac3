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
// The cell records of a 16x4x4 voxel tile are staged through shared memory with coalesced
// loads; the accumulator is then cleared for the next batch with one memset.
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

// Fold tile: 16 x 4 x 16 voxels per 256-thread block, each thread folding four voxels spaced
// 4 apart in z.  The cells that touch those voxels are [x0-1, x0+16) x [y0-1, y0+4) x
// [z0-1, z0+16): 17 x 5 x 17 records of 32 bytes (1.4 record reads per voxel), loaded with
// coalesced 16-byte loads and stored corner-major in shared memory (one FP32 array per
// corner), so that the 32 lanes of a warp, which fold consecutive voxels in x, read 32
// consecutive words of one corner array: no bank conflicts.
constexpr int kFoldX = 16, kFoldY = 4, kFoldZ = 16, kFoldPasses = 4;
constexpr int kHaloX = kFoldX + 1, kHaloY = kFoldY + 1, kHaloZ = kFoldZ + 1;
constexpr int kHaloCells = kHaloX * kHaloY * kHaloZ;
constexpr size_t kFoldShared = 8 * kHaloCells * sizeof(float);  // 46,240 bytes

template <typename G>
__global__ void __launch_bounds__(256) k_fold(int nx, int ny, int nz, const float* __restrict__ acc,
                                              double* __restrict__ total, int accumulate_total,
                                              G* __restrict__ gradient, int32_t* status)
{
    extern __shared__ float corners[];  // [8][kHaloCells]
    const int tiles_x = (nx + kFoldX - 1) / kFoldX, tiles_y = (ny + kFoldY - 1) / kFoldY;
    const int tile = blockIdx.x;
    const int tz = tile / (tiles_x * tiles_y), rest = tile - tz * tiles_x * tiles_y;
    const int ty = rest / tiles_x, tx = rest - ty * tiles_x;
    const int x0 = tx * kFoldX, y0 = ty * kFoldY, z0 = tz * kFoldZ;
    const float4* records = reinterpret_cast<const float4*>(acc);
    for (int i = threadIdx.x; i < 2 * kHaloCells; i += 256) {
        const int half = i & 1, c = i >> 1;
        const int cz = c / (kHaloX * kHaloY), cr = c - cz * kHaloX * kHaloY;
        const int cy = cr / kHaloX, cx = cr - cy * kHaloX;
        const int gx = x0 - 1 + cx, gy = y0 - 1 + cy, gz = z0 - 1 + cz;
        float4 value = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (gx >= 0 && gy >= 0 && gz >= 0 && gx < nx && gy < ny && gz < nz)
            value = __ldg(records + 2 * (((int64_t)gz * ny + gy) * nx + gx) + half);
        float* base = corners + 4 * half * kHaloCells + c;
        base[0] = value.x;
        base[kHaloCells] = value.y;
        base[2 * kHaloCells] = value.z;
        base[3 * kHaloCells] = value.w;
    }
    __syncthreads();
    const int lx = threadIdx.x % kFoldX, ly = (threadIdx.x / kFoldX) % kFoldY, lz0 = threadIdx.x / (kFoldX * kFoldY);
    const int x = x0 + lx, y = y0 + ly;
    bool bad = false;
    if (x < nx && y < ny) {
        int cxs[2], bxs[2], cys[2], bys[2];
        const int kx = axis_sources(x, nx, cxs, bxs);
        const int ky = axis_sources(y, ny, cys, bys);
#pragma unroll
        for (int pass = 0; pass < kFoldPasses; ++pass) {
            const int z = z0 + lz0 + pass * (kFoldZ / kFoldPasses);
            if (z >= nz) break;
            int czs[2], bzs[2];
            const int kz = axis_sources(z, nz, czs, bzs);
            double sum = 0.0;
            for (int iz = 0; iz < kz; ++iz)
                for (int iy = 0; iy < ky; ++iy)
                    for (int ix = 0; ix < kx; ++ix) {
                        const int c = ((czs[iz] - z0 + 1) * kHaloY + (cys[iy] - y0 + 1)) * kHaloX + (cxs[ix] - x0 + 1);
                        const int corner = bxs[ix] | (bys[iy] << 1) | (bzs[iz] << 2);
                        sum += (double)corners[corner * kHaloCells + c];
                    }
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
    const unsigned blocks = (unsigned)(((p.nx + kFoldX - 1) / kFoldX) * ((p.ny + kFoldY - 1) / kFoldY) *
                                       ((p.nz + kFoldZ - 1) / kFoldZ));
    if (gradient_dtype == DPT_F64)
        k_fold<double><<<blocks, 256, kFoldShared, stream>>>(p.nx, p.ny, p.nz, accumulator, total,
                                                   accumulate_total, static_cast<double*>(gradient), status);
    else
        k_fold<float><<<blocks, 256, kFoldShared, stream>>>(p.nx, p.ny, p.nz, accumulator, total,
                                                  accumulate_total, static_cast<float*>(gradient), status);
    cudaError_t error = cudaGetLastError();
    if (error == cudaSuccess && clear)
        error = cudaMemsetAsync(accumulator, 0, (size_t)p.nx * p.ny * p.nz * 32u, stream);
    return error;
}

}  // namespace dpt
