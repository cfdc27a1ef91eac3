// pack.cu - field validation, rigid-pose validation and corner-replicated field copies.
//
// One pass over the field (reference kernels/projection_checks.py:20-56 field scan) also
// writes the layout the sampling kernels read: for the FP32 and FP64 arithmetic a float4
// "quad" per voxel holding the (x, x+1) x (y, y+1) corners of its z plane; for the
// compensated form (FP32, FP16 or BF16 storage) the eight polynomial coefficients of the
// cell.  A sample then needs two 16-byte loads instead of eight gathers.  Corner indices
// clamp to n-1 exactly like
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

struct PackArgs {
    int nx, ny, nz;
    int signed_domain;  // DPT_DOMAIN_SIGNED: only non-finite values are flagged
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

template <int kDtype>
__device__ __forceinline__ float decode(const void* field, int64_t index)
{
    if constexpr (kDtype == DPT_F32) return static_cast<const float*>(field)[index];
    else if constexpr (kDtype == DPT_BF16) return bf16_bits_to_float(static_cast<const uint16_t*>(field)[index]);
    else return half_bits_to_float(static_cast<const uint16_t*>(field)[index]);
}

__device__ __forceinline__ bool out_of_domain(const PackArgs& a, float v)
{
    return !isfinite(v) || (!a.signed_domain && v < 0.0f);
}

// FP32 corner quads of any storage type (half values decoded exactly).
template <int kDtype>
__global__ void __launch_bounds__(256) k_pack_quad(PackArgs a, const void* __restrict__ field,
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
    const float v = decode<kDtype>(field, index);
    flag_field(out_of_domain(a, v), a.status);
    if (quad)
        quad[index] = make_float4(v, decode<kDtype>(field, row0 + x1), decode<kDtype>(field, row1 + x),
                                  decode<kDtype>(field, row1 + x1));
}

// Polynomial copy of the compensated precision form: per cell the coefficients of
// f = c0 + c1 x + c2 y + c3 z + c4 xy + c5 xz + c6 yz + c7 xyz from its eight decoded corner
// values (clamped like corner_index), in the order and FP32 arithmetic of PolyCache.

template <int kDtype>
__global__ void __launch_bounds__(256) k_pack_poly(PackArgs a, const void* __restrict__ field,
                                                   float4* __restrict__ coef)
{
    const int64_t index = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    check_pose(a, index);
    if (index >= a.voxels) return;
    const int x = (int)(index % a.nx);
    const int64_t rest = index / a.nx;
    const int y = (int)(rest % a.ny), z = (int)(rest / a.ny);
    const float own = decode<kDtype>(field, index);
    flag_field(out_of_domain(a, own), a.status);
    if (!coef) return;  // validation only
    const int x1 = min(x + 1, a.nx - 1), y1 = min(y + 1, a.ny - 1), z1 = min(z + 1, a.nz - 1);
    const int64_t r00 = ((int64_t)z * a.ny + y) * a.nx, r10 = ((int64_t)z * a.ny + y1) * a.nx;
    const int64_t r01 = ((int64_t)z1 * a.ny + y) * a.nx, r11 = ((int64_t)z1 * a.ny + y1) * a.nx;
    float v[8];
    v[0] = own;
    v[1] = decode<kDtype>(field, r00 + x1);
    v[2] = decode<kDtype>(field, r10 + x);
    v[3] = decode<kDtype>(field, r10 + x1);
    v[4] = decode<kDtype>(field, r01 + x);
    v[5] = decode<kDtype>(field, r01 + x1);
    v[6] = decode<kDtype>(field, r11 + x);
    v[7] = decode<kDtype>(field, r11 + x1);
    const float c1 = v[1] - v[0], c2 = v[2] - v[0], c3 = v[4] - v[0];
    const float c4 = (v[3] - v[2]) - c1, c5 = (v[5] - v[4]) - c1, c6 = (v[6] - v[4]) - c2;
    const float c7 = ((v[7] - v[6]) - (v[5] - v[4])) - c4;
    coef[2 * index] = make_float4(v[0], c1, c2, c3);
    coef[2 * index + 1] = make_float4(c4, c5, c6, c7);
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
    a.signed_domain = p.field_domain == DPT_DOMAIN_SIGNED;
    a.views = p.views;
    a.poses = poses;
    a.status = status;
    const int64_t work = a.voxels > a.views ? a.voxels : a.views;
    const unsigned blocks = (unsigned)((work + 255) / 256);
    if (p.arith == DPT_ARITH_F32C) {
        float4* coef = static_cast<float4*>(packed);
        if (p.field_dtype == DPT_F32)
            k_pack_poly<DPT_F32><<<blocks, 256, 0, stream>>>(a, field, coef);
        else if (p.field_dtype == DPT_BF16)
            k_pack_poly<DPT_BF16><<<blocks, 256, 0, stream>>>(a, field, coef);
        else
            k_pack_poly<DPT_F16><<<blocks, 256, 0, stream>>>(a, field, coef);
    } else {
        float4* quad = static_cast<float4*>(packed);
        if (p.field_dtype == DPT_F32)
            k_pack_quad<DPT_F32><<<blocks, 256, 0, stream>>>(a, field, quad);
        else if (p.field_dtype == DPT_BF16)
            k_pack_quad<DPT_BF16><<<blocks, 256, 0, stream>>>(a, field, quad);
        else
            k_pack_quad<DPT_F16><<<blocks, 256, 0, stream>>>(a, field, quad);
    }
    return cudaGetLastError();
}

}  // namespace dpt
