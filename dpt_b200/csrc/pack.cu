// pack.cu - field validation, rigid-pose validation and corner-replicated field copies.
//
// One pass over the field (reference kernels/projection_checks.py:20-56 field scan) also
// writes the layout the sampling kernels read: for FP32 storage a float4 "quad" per voxel
// holding the (x, x+1) x (y, y+1) corners of its z plane, for FP16/BF16 storage a 16-byte
// "octet" with all eight corners.  A sample then needs two (FP32) or one (half) 16-byte
// loads instead of eight 4- or 2-byte gathers.  Corner indices clamp to n-1 exactly like
// corner_index (reference kernels/projection.py:217-222), so every sample sees the same
// values as a direct gather.
#include "launch.h"

namespace dpt {
namespace {

__device__ __forceinline__ float half_bits_to_float(uint16_t h)
{
    return __half2float(__ushort_as_half(h));
}
__device__ __forceinline__ float bf16_bits_to_float(uint16_t b)
{
    return __uint_as_float((uint32_t)b << 16);
}

// Rigid pose: finite, R^T R = I within 1e-10, det(R) >= 0 (reference kernels/geometry.py:55-74).
__device__ bool rigid_pose(const double* p)
{
    bool valid = true;
    for (int k = 0; k < 12; ++k) valid = valid && isfinite(p[k]);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double product = fma(p[6 + i], p[6 + j], fma(p[3 + i], p[3 + j], p[i] * p[j]));
            if (fabs(product - (i == j ? 1.0 : 0.0)) > 1e-10) valid = false;
        }
    const double det = p[0] * (p[4] * p[8] - p[5] * p[7]) - p[1] * (p[3] * p[8] - p[5] * p[6]) +
                       p[2] * (p[3] * p[7] - p[4] * p[6]);
    if (det < 0.0) valid = false;
    return valid;
}

struct PackArgs {
    int nx, ny, nz;
    int64_t voxels;
    int views;
    const double* poses;
    int32_t* status;
};

__device__ __forceinline__ void flag_field(bool bad, int32_t* status)
{
    const unsigned any = __ballot_sync(__activemask(), bad);
    if (any && (threadIdx.x & 31) == (__ffs(any) - 1)) atomicOr(status, 8);
}

__device__ __forceinline__ void check_pose(const PackArgs& a, int64_t index)
{
    if (index < a.views) {
        double p[12];
        for (int k = 0; k < 12; ++k) p[k] = a.poses[12 * index + k];
        if (!rigid_pose(p)) atomicOr(a.status + index, 1);
    }
}

__global__ void __launch_bounds__(256) k_pack_quad(PackArgs a, const float* __restrict__ field,
                                                   float4* __restrict__ quad)
{
    const int64_t index = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    check_pose(a, index);
    if (index >= a.voxels) return;
    const int x = (int)(index % a.nx);
    const int64_t rest = index / a.nx;
    const int y = (int)(rest % a.ny), z = (int)(rest / a.ny);
    const int x1 = min(x + 1, a.nx - 1), y1 = min(y + 1, a.ny - 1);
    const int64_t row0 = ((int64_t)z * a.ny + y) * a.nx, row1 = ((int64_t)z * a.ny + y1) * a.nx;
    const float v = field[index];
    flag_field(!isfinite(v) || v < 0.0f, a.status);
    if (quad) quad[index] = make_float4(v, field[row0 + x1], field[row1 + x], field[row1 + x1]);
}

template <bool kBF16>
__global__ void __launch_bounds__(256) k_pack_octet(PackArgs a, const uint16_t* __restrict__ field,
                                                    uint4* __restrict__ octet)
{
    const int64_t index = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    check_pose(a, index);
    if (index >= a.voxels) return;
    const int x = (int)(index % a.nx);
    const int64_t rest = index / a.nx;
    const int y = (int)(rest % a.ny), z = (int)(rest / a.ny);
    const int x1 = min(x + 1, a.nx - 1), y1 = min(y + 1, a.ny - 1), z1 = min(z + 1, a.nz - 1);
    const int64_t r00 = ((int64_t)z * a.ny + y) * a.nx, r10 = ((int64_t)z * a.ny + y1) * a.nx;
    const int64_t r01 = ((int64_t)z1 * a.ny + y) * a.nx, r11 = ((int64_t)z1 * a.ny + y1) * a.nx;
    const uint16_t own = field[index];
    const float v = kBF16 ? bf16_bits_to_float(own) : half_bits_to_float(own);
    flag_field(!isfinite(v) || v < 0.0f, a.status);
    // corner c = (x bit, y bit, z bit); corners 2k (low half) and 2k+1 (high half) per word
    if (!octet) return;
    const uint32_t w0 = (uint32_t)field[r00 + x] | ((uint32_t)field[r00 + x1] << 16);
    const uint32_t w1 = (uint32_t)field[r10 + x] | ((uint32_t)field[r10 + x1] << 16);
    const uint32_t w2 = (uint32_t)field[r01 + x] | ((uint32_t)field[r01 + x1] << 16);
    const uint32_t w3 = (uint32_t)field[r11 + x] | ((uint32_t)field[r11 + x1] << 16);
    octet[index] = make_uint4(w0, w1, w2, w3);
}

}  // namespace

cudaError_t launch_prepare_field(const dpt_problem& p, const void* field, void* packed,
                                 const double* poses, int32_t* status, cudaStream_t stream)
{
    PackArgs a;
    a.nx = p.nx;
    a.ny = p.ny;
    a.nz = p.nz;
    a.voxels = (int64_t)p.nx * p.ny * p.nz;
    a.views = p.views;
    a.poses = poses;
    a.status = status;
    const int64_t work = a.voxels > a.views ? a.voxels : a.views;
    const unsigned blocks = (unsigned)((work + 255) / 256);
    if (p.field_dtype == DPT_F32) {
        k_pack_quad<<<blocks, 256, 0, stream>>>(a, static_cast<const float*>(field),
                                                static_cast<float4*>(packed));
    } else if (p.field_dtype == DPT_BF16) {
        k_pack_octet<true><<<blocks, 256, 0, stream>>>(a, static_cast<const uint16_t*>(field),
                                                       static_cast<uint4*>(packed));
    } else {
        k_pack_octet<false><<<blocks, 256, 0, stream>>>(a, static_cast<const uint16_t*>(field),
                                                        static_cast<uint4*>(packed));
    }
    return cudaGetLastError();
}

}  // namespace dpt
