// common.cuh - device arithmetic shared by the projector kernels.
//
// Floating-point contract: this code is compiled with -fmad=false.  Every fused
// multiply-add is an explicit fma()/fmaf(); every other operation is one IEEE
// rounding.  Where the reference projector (hcltech-robotics/dpt) writes
// a*b + c*d this code computes fma(c, d, a*b); a + b*c is fma(b, c, a).  With
// that contract the FP32 forward reproduces the reference sample sequence of
// python/dpt/kernels/projection_fp32.py exactly, and the FP64 forward that of
// python/dpt/kernels/projection.py.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

#include "../../include/dpt_b200.h"

namespace dpt {

constexpr int kBlock = 256;      // threads per block of the count kernels
#ifndef DPT_FORWARD_THREADS
#define DPT_FORWARD_THREADS 128  // 16x8 detector tiles: 5% faster than 256 (FP32, 256^3, 512^2, S = 1024)
#endif
constexpr int kForwardBlock = DPT_FORWARD_THREADS;  // threads per block of the forward kernel
// Build-time tuning of the VJP launch (results do not depend on it beyond the FP64 order of
// the per-block pose partials): 128-thread blocks (a 16x8 detector tile) keep five blocks of
// the ~96-register kernel resident per SM, 20 warps against 16 with 256-thread blocks, which
// measured 12% faster on the 256^3 / 512^2 / S=1024 full scan.
#ifndef DPT_VJP_THREADS
#define DPT_VJP_THREADS 128
#endif
constexpr int kVjpBlock = DPT_VJP_THREADS;  // threads per block of the VJP kernel
constexpr int kDefaultBlockCols = 16;  // default block tile: 16 x 16 detector pixels
constexpr int kMaxPack = DPT_MAX_PACK;  // problems of one packed forward launch

struct Grid {
    int nx, ny, nz;
    double m[9];   // object_to_grid, row-major
    double g0[3];  // grid origin (object mm)
};

// Kernel arguments passed by value (fits the 4 KB parameter space).
struct RayArgs {
    Grid grid;
    int views;           // views in this launch
    int view_begin;      // first absolute view of this launch
    int rows, cols;      // rays per view = rows*cols
    int samples;
    int ray_kind;
    int tiles_x;         // column tiles per view (panels)
    int tiles_per_view;  // blocks per view
    int block_cols;      // detector columns per block tile (panels): 8, 16, 32 or 64
    int block_rows;      // detector rows per block tile: block_threads / block_cols
    int warps_x;         // warps along the columns of a block tile: block_cols / 8
    int block_threads;   // threads per block
    int view_group;      // views per block-order group (see block_work)
    const double* poses;       // absolute view indexing
    const double* view_table;  // absolute view indexing
    const double* ray_sources;
    const double* ray_endpoints;
    int32_t* status;           // absolute view indexing
};

// ---------------------------------------------------------------- helpers

__device__ __forceinline__ bool finite3(double a, double b, double c)
{
    return isfinite(a) && isfinite(b) && isfinite(c);
}
__device__ __forceinline__ bool finite3f(float a, float b, float c)
{
    return isfinite(a) && isfinite(b) && isfinite(c);
}

// r = A v, A row-major: fma(a2, v2, fma(a1, v1, a0*v0)).
__device__ __forceinline__ void matvec(const double* a, const double* v, double* r)
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
        r[i] = fma(a[3 * i + 2], v[2], fma(a[3 * i + 1], v[1], a[3 * i] * v[0]));
}

// r = A^T v.
__device__ __forceinline__ void matvec_t(const double* a, const double* v, double* r)
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
        r[i] = fma(a[6 + i], v[2], fma(a[3 + i], v[1], a[i] * v[0]));
}

// Rigid pose: finite, R^T R = I within 1e-10, det(R) >= 0 (reference kernels/geometry.py:55-74).
__device__ __forceinline__ bool rigid_pose(const double* p)
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

// Views per group of the block order of the ray kernels.  The 1-D grid walks groups of
// view_group consecutive views; inside a group the blocks of one detector tile for all of the
// group's views are consecutive.  The blocks resident at one time then cover a few tiles of
// several neighbouring views, whose rays cross nearly the same cells: the field copy and the
// volume accumulator records they touch are shared in L2 instead of each view streaming the
// whole volume through it (a launch's blocks are dispatched roughly in index order).
#ifndef DPT_VIEW_GROUP
#define DPT_VIEW_GROUP 32
#endif

// Blocks of a launch over a.views views and a.tiles_per_view tiles per view.
__host__ __device__ __forceinline__ unsigned ray_blocks(const RayArgs& a)
{
    return (unsigned)a.tiles_per_view * (unsigned)a.views;
}

// (view within the launch, detector tile) of block b of the launch's order.
__device__ __forceinline__ void block_work_at(const RayArgs& a, int b, int* view_local, int* tile)
{
    const int per_group = a.view_group * a.tiles_per_view;
    const int g = b / per_group;
    const int r = b - g * per_group;
    const int first = g * a.view_group;
    const int views = min(a.view_group, a.views - first);
    const int t = r / views;
    *tile = t;
    *view_local = first + (r - t * views);
}

// (view within the launch, detector tile) of this block.
__device__ __forceinline__ void block_work(const RayArgs& a, int* view_local, int* tile)
{
    block_work_at(a, (int)blockIdx.x, view_local, tile);
}

// Ray index inside its view -> (pixel) for the tiled panel mapping, or the bundle index.
// Returns false for padding threads.
__device__ __forceinline__ bool ray_of_thread(const RayArgs& a, int tile, int* pixel)
{
    const int t = threadIdx.x;
    if (a.ray_kind == DPT_RAYS_BUNDLE) {
        const int index = tile * a.block_threads + t;
        *pixel = index;
        return index < a.rows * a.cols;
    }
    // block tile of block_cols x block_rows pixels; each warp covers 8 columns x 4 rows.
    const int warp = t >> 5, lane = t & 31;
    const int wy = warp / a.warps_x, wx = warp - wy * a.warps_x;
    const int tile_row = tile / a.tiles_x, tile_col = tile - tile_row * a.tiles_x;
    const int col = tile_col * a.block_cols + wx * 8 + (lane & 7);
    const int row = tile_row * a.block_rows + wy * 4 + (lane >> 3);
    *pixel = row * a.cols + col;
    return row < a.rows && col < a.cols;
}

// Source and endpoint (world mm) of ray `pixel` of absolute view `view`.
__device__ __forceinline__ void ray_endpoints(const RayArgs& a, const double* w, int view, int pixel,
                                              double* source, double* end)
{
    if (a.ray_kind == DPT_RAYS_BUNDLE) {
        const int64_t ray = (int64_t)view * a.rows * a.cols + pixel;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            source[k] = __ldg(a.ray_sources + 3 * ray + k);
            end[k] = __ldg(a.ray_endpoints + 3 * ray + k);
        }
        return;
    }
    const int r = pixel / a.cols;
    const double row = (double)r, column = (double)(pixel - r * a.cols);
    const int mode = (int)w[DPT_VIEW_MODE_WORD];
    if (mode == DPT_PANEL_CONE) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            source[k] = w[k];
            end[k] = fma(row, w[9 + k], fma(column, w[6 + k], w[3 + k]));
        }
    } else if (mode == DPT_PANEL_PARALLEL) {
        const double cu = column * w[12], rv = row * w[13], length = w[14];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            end[k] = fma(rv, w[9 + k], fma(cu, w[6 + k], w[3 + k]));
            source[k] = end[k] - length * w[k];
        }
    } else {
        const double radius = w[14];
        const double angle = column * w[12] / radius;
        double s, c;
        sincos(angle, &s, &c);
        const double c1 = c - 1.0, sr = s * radius, rv = row * w[13];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            source[k] = w[k];
            end[k] = fma(rv, w[9 + k], fma(sr, w[6 + k], fma(c1, w[15 + k], w[3 + k])));
        }
    }
}

// FP64 ray in grid-index coordinates (reference kernels/projection.py:79-102).
struct Ray64 {
    double origin[3], direction[3];
    double os[3], od[3];    // object-frame source and direction
    double wsr[3], wd[3];   // world source minus translation, world direction
    double length;
};

__device__ __forceinline__ void ray_setup(const Grid& g, const double* pose, const double* source,
                                          const double* end, Ray64& r)
{
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r.wsr[k] = source[k] - pose[9 + k];
        r.wd[k] = end[k] - source[k];
    }
    matvec_t(pose, r.wsr, r.os);
    matvec_t(pose, r.wd, r.od);
    double rel[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) rel[k] = r.os[k] - g.g0[k];
    matvec(g.m, rel, r.origin);
    matvec(g.m, r.od, r.direction);
    r.length = sqrt(fma(r.wd[2], r.wd[2], fma(r.wd[1], r.wd[1], r.wd[0] * r.wd[0])));
}

__device__ __forceinline__ bool valid_ray(const Ray64& r)
{
    return finite3(r.origin[0], r.origin[1], r.origin[2]) &&
           finite3(r.direction[0], r.direction[1], r.direction[2]) &&
           finite3(r.os[0], r.os[1], r.os[2]) && finite3(r.od[0], r.od[1], r.od[2]) &&
           finite3(r.wsr[0], r.wsr[1], r.wsr[2]) && finite3(r.wd[0], r.wd[1], r.wd[2]) &&
           isfinite(r.length) && r.length > 0.0;
}

// Slab clip of t in [0,1] against [-0.5, n-0.5] per axis with the active-face derivatives
// (reference kernels/projection_fp32.py:78-109 and kernels/projection.py:147-184).
template <typename T>
struct Interval {
    T lower, upper;
    int lower_axis, upper_axis;  // -1: the segment end itself (no face derivative)
    T lower_velocity, upper_velocity;

    __device__ __forceinline__ void clip(const T* origin, const T* direction, int nx, int ny, int nz)
    {
        lower = T(0);
        upper = T(1);
        lower_axis = upper_axis = -1;
        lower_velocity = upper_velocity = T(1);
        const int shape[3] = {nx, ny, nz};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const T low = T(-0.5), high = T(shape[a]) - T(0.5), velocity = direction[a];
            if (velocity == T(0)) {
                if (origin[a] < low || origin[a] > high) upper = T(-1);
            } else {
                T first = (low - origin[a]) / velocity;
                T last = (high - origin[a]) / velocity;
                if (first > last) {
                    const T t = first;
                    first = last;
                    last = t;
                }
                if (first > lower) {
                    lower = first;
                    lower_axis = a;
                    lower_velocity = velocity;
                }
                if (last < upper) {
                    upper = last;
                    upper_axis = a;
                    upper_velocity = velocity;
                }
            }
        }
    }

    // d lower / d origin[a] = -1/v, d lower / d direction[a] = -lower/v on the active axis.
    __device__ __forceinline__ void lower_gradients(T* og, T* dg) const
    {
#pragma unroll
        for (int a = 0; a < 3; ++a) og[a] = dg[a] = T(0);
        if (lower_axis >= 0) {
#pragma unroll
            for (int a = 0; a < 3; ++a)
                if (a == lower_axis) {
                    og[a] = -T(1) / lower_velocity;
                    dg[a] = -lower / lower_velocity;
                }
        }
    }
    __device__ __forceinline__ void upper_gradients(T* og, T* dg) const
    {
#pragma unroll
        for (int a = 0; a < 3; ++a) og[a] = dg[a] = T(0);
        if (upper_axis >= 0) {
#pragma unroll
            for (int a = 0; a < 3; ++a)
                if (a == upper_axis) {
                    og[a] = -T(1) / upper_velocity;
                    dg[a] = -upper / upper_velocity;
                }
        }
    }
};

// Half-cell support test.
__device__ __forceinline__ bool inside(float x, float y, float z, float hx, float hy, float hz)
{
    return x >= -0.5f && y >= -0.5f && z >= -0.5f && x <= hx && y <= hy && z <= hz;
}
__device__ __forceinline__ bool inside(double x, double y, double z, int nx, int ny, int nz)
{
    return x >= -0.5 && y >= -0.5 && z >= -0.5 && x <= (double)nx - 0.5 &&
           y <= (double)ny - 0.5 && z <= (double)nz - 0.5;
}

// One axis of the clamped cell coordinate: lower = min(floor(clamp(p,0,n-1)), max(n-2,0)).
struct Axis32 {
    int lower;
    float fraction;
};
__device__ __forceinline__ Axis32 axis32(float p, float high, int cap)
{
    const float value = fminf(fmaxf(p, 0.0f), high);
    Axis32 r;
    r.lower = min((int)floorf(value), cap);
    r.fraction = value - (float)r.lower;
    return r;
}

struct Axis64 {
    int lower;
    double fraction;
};
__device__ __forceinline__ Axis64 axis64(double p, double high, int cap)
{
    const double value = fmin(fmax(p, 0.0), high);
    Axis64 r;
    r.lower = min((int)floor(value), cap);
    r.fraction = value - (double)r.lower;
    return r;
}

// FP32 scatter increment: one rounded product, then |x| < 2^-126 flushed to signed zero
// (reference kernels/projection_fp32.py:240-258; CUDA FP32 global atomics flush the same).
__device__ __forceinline__ float scatter_increment(float factor, float weight)
{
    const float increment = factor * weight;
    return fabsf(increment) < 0x1p-126f ? copysignf(0.0f, increment) : increment;
}

// Vector reduction of four FP32 values into 16-byte aligned global memory.
__device__ __forceinline__ void red_add_v4(float* address, float a, float b, float c, float d)
{
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(address), "f"(a), "f"(b),
                 "f"(c), "f"(d)
                 : "memory");
}

// ------------------------------------------------------------ field access

// Corner-replicated copies of the field, written by the pack kernel.
//  Quad (FP32): quad[(z*ny+y)*nx+x] = (v(x,y,z), v(x+1,y,z), v(x,y+1,z), v(x+1,y+1,z)),
//               indices clamped to n-1 like corner_index.  A cell reads quad at z and at
//               min(z+1, nz-1): corners 0-3 and 4-7.
//  Poly (compensated form, any storage): the cell's trilinear coefficients, two float4.
struct QuadF32 {
    static constexpr bool kCoefficients = false;
    const float4* quad;
    int nx, ny, nz;
    // corners of the cell whose flat index (z*ny + y)*nx + x is `cell` (32-bit: the problem
    // checks bound the voxel count below 2^31)
    __device__ __forceinline__ void load_at(int cell, int, int, int lz, float* v) const
    {
        const float4* p = quad + cell;
        const float4 a = __ldg(p);
        const float4 b = __ldg(lz + 1 < nz ? p + nx * ny : p);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    }
    __device__ __forceinline__ void load(int lx, int ly, int lz, float* v) const
    {
        const int64_t plane = (int64_t)nx * ny;
        const int64_t base = (int64_t)ly * nx + lx;
        const int64_t z1 = lz + 1 < nz ? lz + 1 : nz - 1;
        const float4 a = __ldg(quad + (int64_t)lz * plane + base);
        const float4 b = __ldg(quad + z1 * plane + base);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    }
};

struct PlainF32 {
    static constexpr bool kCoefficients = false;
    const float* field;
    int nx, ny, nz;
    __device__ __forceinline__ void load_at(int, int lx, int ly, int lz, float* v) const
    {
        load(lx, ly, lz, v);
    }
    __device__ __forceinline__ void load(int lx, int ly, int lz, float* v) const
    {
        const int x1 = min(lx + 1, nx - 1), y1 = min(ly + 1, ny - 1), z1 = min(lz + 1, nz - 1);
        const int64_t r00 = ((int64_t)lz * ny + ly) * nx, r10 = ((int64_t)lz * ny + y1) * nx;
        const int64_t r01 = ((int64_t)z1 * ny + ly) * nx, r11 = ((int64_t)z1 * ny + y1) * nx;
        v[0] = __ldg(field + r00 + lx); v[1] = __ldg(field + r00 + x1);
        v[2] = __ldg(field + r10 + lx); v[3] = __ldg(field + r10 + x1);
        v[4] = __ldg(field + r01 + lx); v[5] = __ldg(field + r01 + x1);
        v[6] = __ldg(field + r11 + lx); v[7] = __ldg(field + r11 + x1);
    }
};

// Polynomial copy (compensated precision form): per cell the FP32 coefficients c0..c7 of its
// trilinear polynomial as two float4, formed by the pack kernel from the decoded corner values
// with the arithmetic of PolyCache, so a sample loads its coefficients instead of its corners.
struct PolyF32 {
    static constexpr bool kCoefficients = true;
    const float4* coef;
    int nx, ny, nz;
    __device__ __forceinline__ void coefficients_at(int cell, float* c) const
    {
        const float4* p = coef + 2 * (int64_t)cell;
        const float4 a = __ldg(p), b = __ldg(p + 1);
        c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = a.w;
        c[4] = b.x; c[5] = b.y; c[6] = b.z; c[7] = b.w;
    }
};

// Trilinear weight of corner c: (f0 f1) f2 with f = 1 - fraction for a 0 bit.
__device__ __forceinline__ void corner_weights(float fx, float fy, float fz, float* w)
{
    const float ax = 1.0f - fx, ay = 1.0f - fy, az = 1.0f - fz;
    w[0] = (ax * ay) * az;
    w[1] = (fx * ay) * az;
    w[2] = (ax * fy) * az;
    w[3] = (fx * fy) * az;
    w[4] = (ax * ay) * fz;
    w[5] = (fx * ay) * fz;
    w[6] = (ax * fy) * fz;
    w[7] = (fx * fy) * fz;
}

// value = fmaf(w_c, v_c, value) over corners 0..7 from zero.
__device__ __forceinline__ float interpolate(const float* w, const float* v)
{
    float value = fmaf(w[0], v[0], 0.0f);
#pragma unroll
    for (int c = 1; c < 8; ++c) value = fmaf(w[c], v[c], value);
    return value;
}

// Grid-space slope of the FP32 pose path (reference kernels/projection_fp32.py:196-208).
__device__ __forceinline__ void slope32(float fx, float fy, float fz, const float* v, float sx,
                                        float sy, float sz, float* g)
{
    const float ax = 1.0f - fx, ay = 1.0f - fy, az = 1.0f - fz;
    const float x0 = fmaf(fy, v[3] - v[2], ay * (v[1] - v[0]));
    const float x1 = fmaf(fy, v[7] - v[6], ay * (v[5] - v[4]));
    g[0] = sx * fmaf(fz, x1, az * x0);
    const float y0 = fmaf(fx, v[3] - v[1], ax * (v[2] - v[0]));
    const float y1 = fmaf(fx, v[7] - v[5], ax * (v[6] - v[4]));
    g[1] = sy * fmaf(fz, y1, az * y0);
    const float z0 = fmaf(fx, v[5] - v[1], ax * (v[4] - v[0]));
    const float z1 = fmaf(fx, v[7] - v[3], ax * (v[6] - v[2]));
    g[2] = sz * fmaf(fy, z1, ay * z0);
}

// FP64 weighted-lerp value (reference kernels/projection.py:249-260).
__device__ __forceinline__ double interpolate64(double fx, double fy, double fz, const double* v)
{
    const double ax = 1.0 - fx, ay = 1.0 - fy, az = 1.0 - fz;
    const double x00 = fma(fx, v[1], ax * v[0]), x10 = fma(fx, v[3], ax * v[2]);
    const double x01 = fma(fx, v[5], ax * v[4]), x11 = fma(fx, v[7], ax * v[6]);
    const double xy0 = fma(fy, x10, ay * x00), xy1 = fma(fy, x11, ay * x01);
    return fma(fz, xy1, az * xy0);
}

// FP64 slope (reference kernels/projection.py:261-273).
__device__ __forceinline__ void slope64(double fx, double fy, double fz, const double* v, double sx,
                                        double sy, double sz, double* g)
{
    const double ax = 1.0 - fx, ay = 1.0 - fy, az = 1.0 - fz;
    const double dx0 = fma(fy, v[3] - v[2], ay * (v[1] - v[0]));
    const double dx1 = fma(fy, v[7] - v[6], ay * (v[5] - v[4]));
    const double dy0 = fma(fx, v[3] - v[1], ax * (v[2] - v[0]));
    const double dy1 = fma(fx, v[7] - v[5], ax * (v[6] - v[4]));
    const double dz0 = fma(fx, v[5] - v[1], ax * (v[4] - v[0]));
    const double dz1 = fma(fx, v[7] - v[3], ax * (v[6] - v[2]));
    g[0] = sx * fma(fz, dx1, az * dx0);
    g[1] = sy * fma(fz, dy1, az * dy0);
    g[2] = sz * fma(fy, dz1, ay * dz0);
}

// Grid bounds used by every sample (computed once per thread).
struct FieldDims {
    int nx, ny, nz;
    float hx, hy, hz;   // n - 0.5: upper end of the half-cell support
    float mx, my, mz;   // n - 1: clamp bound
    int cx, cy, cz;     // max(n - 2, 0): largest lower cell index
    bool packed;        // interior coordinates stay below 2^23 (interior_fraction2 applies)
    __device__ __forceinline__ void init(const Grid& g)
    {
        nx = g.nx; ny = g.ny; nz = g.nz;
        hx = (float)nx - 0.5f; hy = (float)ny - 0.5f; hz = (float)nz - 0.5f;
        mx = (float)(nx - 1); my = (float)(ny - 1); mz = (float)(nz - 1);
        cx = max(nx - 2, 0); cy = max(ny - 2, 0); cz = max(nz - 2, 0);
        packed = nx <= (1 << 23) && ny <= (1 << 23) && nz <= (1 << 23);
    }
};

// A ray whose grid-space origin and direction are below 1e30 in magnitude has only finite
// sample points (each point is o + t d with t in [0, 1]), so its samples need no finiteness
// test; other rays take the general path.
__device__ __forceinline__ bool moderate(const float* o, const float* d)
{
    const float m = fmaxf(fmaxf(fmaxf(fabsf(o[0]), fabsf(o[1])), fmaxf(fabsf(o[2]), fabsf(d[0]))),
                          fmaxf(fabsf(d[1]), fabsf(d[2])));
    return m < 1e30f;
}
// The compensated form walks cell runs (segment form) while a ray's samples lie at most one
// cell plane apart on average, (|s_x| + |s_y|) + |s_z| <= 1 for the per-sample step s in grid
// units; sparser samples take the per-sample form (walking every plane between them costs
// more than evaluating each sample), as do rays whose coordinates reach 1e30.
__device__ __forceinline__ bool segment_form(const float* entry, const float* sv)
{
    return moderate(entry, sv) && (fabsf(sv[0]) + fabsf(sv[1])) + fabsf(sv[2]) <= 1.0f;
}
__device__ __forceinline__ bool moderate(const double* o, const double* d)
{
    const double m = fmax(fmax(fmax(fabs(o[0]), fabs(o[1])), fmax(fabs(o[2]), fabs(d[0]))),
                          fmax(fabs(d[1]), fabs(d[2])));
    return m < 1e300;
}

// The midpoints of one ray are monotone in the sample index along every axis (each point
// is an fma that is monotone in its sample parameter), so the samples inside the half-cell
// support form one contiguous run.  Find its ends [first, last] (first > last when empty);
// samples outside the run contribute exactly zero and need not be visited.
template <typename Inside>
__device__ __forceinline__ void inside_run(int samples, Inside inside_at, int& first, int& last)
{
    first = 0;
    last = samples - 1;
    while (first <= last && !inside_at(first)) ++first;
    while (last > first && !inside_at(last)) --last;
}

// The current cell's eight corner values.  With kReuse they are reloaded only when the
// sample enters another cell; without, every sample loads them (no branch in the loop: the
// choice of the kernels whose loop body is long enough that the branch costs more than the
// L1 hit it saves).
template <class Field, bool kReuse = true>
struct CellCache {
    float v[8];
    int cell = -1;
    __device__ __forceinline__ void fetch(const Field& f, int lx, int ly, int lz, int index)
    {
        if constexpr (kReuse) {
            if (index != cell) {
                f.load_at(index, lx, ly, lz, v);
                cell = index;
            }
        } else {
            f.load_at(index, lx, ly, lz, v);
        }
    }
};

// The current cell's eight corner values widened to FP64 once per cell.
template <class Field>
struct WideCellCache {
    double v[8];
    int cell = -1;
    __device__ __forceinline__ void fetch(const Field& f, int lx, int ly, int lz, int index)
    {
        if (index != cell) {
            float narrow[8];
            f.load_at(index, lx, ly, lz, narrow);
#pragma unroll
            for (int c = 0; c < 8; ++c) v[c] = (double)narrow[c];
            cell = index;
        }
    }
};

// Axis coordinate of a point known to satisfy 0 <= p < n-1 (the interior of the grid): the
// clamp and the cap of axis32 are then no-ops, so this is the same lower cell and fraction.
__device__ __forceinline__ Axis32 interior_axis(float p)
{
    Axis32 r;
    r.lower = __float2int_rd(p);
    r.fraction = p - (float)r.lower;
    return r;
}

// Interior run of the inside run: the samples whose point satisfies 0 <= p < n-1 on every
// axis (all clamps inactive, all slope masks 1).  Also contiguous by monotonicity.
template <typename Interior>
__device__ __forceinline__ void interior_run(int first, int last, Interior interior_at, int& ifirst,
                                             int& ilast)
{
    ifirst = first;
    while (ifirst <= last && !interior_at(ifirst)) ++ifirst;
    ilast = last;
    while (ilast > ifirst && !interior_at(ilast)) --ilast;
    if (ifirst > last) ilast = ifirst - 1;
}

// Trilinear polynomial of a cell, f = c0 + c1 x + c2 y + c3 z + c4 xy + c5 xz + c6 yz + c7 xyz,
// formed in FP32 from the eight corner values when a ray enters the cell (the arithmetic of
// the compensated precision form).
template <class Field, bool kReuse = true>
struct PolyCache {
    float c[8];
    int cell = -1;
    __device__ __forceinline__ void fetch(const Field& f, int lx, int ly, int lz, int index)
    {
        if constexpr (kReuse) {
            if (index == cell) return;
            cell = index;
        }
        if constexpr (Field::kCoefficients) {
            f.coefficients_at(index, c);
        } else {
            float v[8];
            f.load_at(index, lx, ly, lz, v);
            c[0] = v[0];
            c[1] = v[1] - v[0];
            c[2] = v[2] - v[0];
            c[3] = v[4] - v[0];
            c[4] = (v[3] - v[2]) - c[1];
            c[5] = (v[5] - v[4]) - c[1];
            c[6] = (v[6] - v[4]) - c[2];
            c[7] = ((v[7] - v[6]) - (v[5] - v[4])) - c[4];
        }
    }
    // value, and when `g` is given the derivatives d/dfx, d/dfy, d/dfz
    __device__ __forceinline__ float eval(float fx, float fy, float fz, float* g = nullptr) const
    {
        const float a = fmaf(c[7], fz, c[4]), b = fmaf(c[5], fz, c[1]);
        const float gx = fmaf(a, fy, b);
        const float e = fmaf(c[6], fz, c[2]), h = fmaf(c[3], fz, c[0]);
        if (g) {
            g[0] = gx;
            g[1] = fmaf(a, fx, e);
            g[2] = fmaf(fx, fmaf(c[7], fy, c[5]), fmaf(c[6], fy, c[3]));
        }
        return fmaf(gx, fx, fmaf(e, fy, h));
    }
};

// ------------------------------------------------ compensated form: cell runs in closed form
//
// For rays whose grid origin and direction stay below 1e30, the samples inside the support,
// [first, last], are grouped into runs of consecutive samples in one interpolation cell by
// walking the cell planes along the ray.  Along a run the fractions are f + j d (j = 0..n-1,
// d the per-sample step; d = 0 on an axis in its half-cell margin, whose fraction is clamped),
// so the run's sum of the cell polynomial, its slope sums and the volume moments are
// polynomials in j of degree <= 3: closed forms in the power sums S1 = sum j, S2 = sum j^2,
// S3 = sum j^3.  Cost per cell crossed instead of per sample.

struct CellRun {
    int i0, n;             // first sample of the run and its sample count
    int lx, ly, lz, cell;  // interpolation cell (lower corner, clamped) and its flat index
    int interior;          // bit k set: axis k inside its cell range (its slope is active)
    float f[3], d[3];      // fractions at sample i0 and their change per sample
    float nf, s1, s2, s3;  // n and the power sums of j over 0..n-1
};

// Walk the cell planes from sample `first` to `last` (sample i at entry + (i + 0.5) sv) and
// call `action(run)` for every run with at least one sample.  Each step advances every axis
// whose plane is the nearest, so the walk ends within nx + ny + nz + 3 steps.  The plane an
// axis meets next is kept as an exact float coordinate; it is crossed at sample coordinate
// (plane - entry) / sv, computed as (plane - entry) * (1 / sv), or never (+inf) when it lies
// outside the cell planes 0..n-1 or the ray does not move on that axis.
// Power sums of short runs, tabulated once per block: entry n holds (n, S1, S2, S3) for
// j = 0..n-1 as walk_cells forms them (exact integers rounded once to FP32, S3 = S1 * S1 in
// FP32), so a run of at most kRunSumTable samples reads its sums instead of forming them.
constexpr int kRunSumTable = 64;
__device__ __forceinline__ float4 run_power_sums(int n)
{
    const unsigned m = (unsigned)n;
    const unsigned s1 = m * (m - 1u) / 2u;
    const float f1 = (float)s1;
    return make_float4((float)n, f1, (float)(s1 * (2u * m - 1u) / 3u), f1 * f1);
}
__device__ __forceinline__ void fill_run_sums(float4* table)
{
    for (int n = threadIdx.x; n <= kRunSumTable; n += blockDim.x) table[n] = run_power_sums(n);
}

template <typename Action>
__device__ __forceinline__ void walk_cells(const FieldDims& dims, const float* entry, const float* sv,
                                           int first, int last, Action action, const float4* sums = nullptr)
{
    const int shape[3] = {dims.nx, dims.ny, dims.nz};
    const float top_plane[3] = {dims.mx, dims.my, dims.mz};  // n - 1
    const float inf = __int_as_float(0x7f800000);
    float inverse[3], next[3], plane[3], stepf[3];
    int axis_cell[3], step[3];
    {
        const float offset = (float)first + 0.5f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int c = (int)floorf(fmaf(offset, sv[k], entry[k]));
            axis_cell[k] = c < -1 ? -1 : (c > shape[k] - 1 ? shape[k] - 1 : c);
            inverse[k] = sv[k] != 0.0f ? 1.0f / sv[k] : 0.0f;
            step[k] = sv[k] > 0.0f ? 1 : -1;
            stepf[k] = (float)step[k];
            plane[k] = (float)(axis_cell[k] + (sv[k] > 0.0f ? 1 : 0));
        }
    }
    auto crossing = [&](int k) {
        const bool valid = sv[k] != 0.0f && plane[k] >= 0.0f && plane[k] <= top_plane[k];
        return valid ? (plane[k] - entry[k]) * inverse[k] : inf;
    };
#pragma unroll
    for (int k = 0; k < 3; ++k) next[k] = crossing(k);
    const float end_limit = (float)(last + 1);
    int i = first;
    const int limit = shape[0] + shape[1] + shape[2] + 4;
    for (int walk = 0; walk < limit; ++walk) {
        const float nearest = fminf(next[0], fminf(next[1], next[2]));
        const float t = nearest - 0.5f;
        const int end = !(t < end_limit) ? last + 1 : (t <= (float)i ? i : (int)ceilf(t));
        if (end > i) {
            CellRun r;
            r.i0 = i;
            r.n = end - i;
            const float offset = (float)i + 0.5f;
            int lower[3];
            r.interior = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int top = shape[k] - 2 < 0 ? 0 : shape[k] - 2;
                const bool interior = axis_cell[k] >= 0 && axis_cell[k] <= shape[k] - 2;
                lower[k] = interior ? axis_cell[k] : (axis_cell[k] < 0 ? 0 : top);
                const float margin = (axis_cell[k] < 0 || shape[k] == 1) ? 0.0f : 1.0f;
                r.f[k] = interior ? fmaf(offset, sv[k], entry[k]) - (float)axis_cell[k] : margin;
                r.d[k] = interior ? sv[k] : 0.0f;
                r.interior |= interior ? 1 << k : 0;
            }
            r.lx = lower[0];
            r.ly = lower[1];
            r.lz = lower[2];
            r.cell = (lower[2] * dims.ny + lower[1]) * dims.nx + lower[0];
            // power sums of j = 0..n-1 (exact integers, rounded once to FP32); 32-bit
            // arithmetic is exact up to n = 1024
            if (sums && r.n <= kRunSumTable) {
                const float4 e = sums[r.n];
                r.nf = e.x;
                r.s1 = e.y;
                r.s2 = e.z;
                r.s3 = e.w;
            } else {
                if (r.n <= 1024) {
                    const float4 e = run_power_sums(r.n);
                    r.s1 = e.y;
                    r.s2 = e.z;
                } else {
                    const int64_t m = r.n;
                    r.s1 = (float)(m * (m - 1) / 2);
                    r.s2 = (float)(m * (m - 1) * (2 * m - 1) / 6);
                }
                r.nf = (float)r.n;
                r.s3 = r.s1 * r.s1;
            }
            action(r);
        }
        i = end;
        if (i > last) break;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (next[k] == nearest) {
                axis_cell[k] += step[k];
                plane[k] += stepf[k];
                next[k] = crossing(k);
            }
        }
    }
}

// The run cell's polynomial at the run's first fractions: value, slopes d/dfx, d/dfy, d/dfz and
// the bilinear terms a = c4 + c7 z, t1 = c5 + c7 y, t2 = c6 + c7 x (the arithmetic of
// PolyCache::eval, extended).
struct RunPoly {
    float value, gx, gy, gz, a, t1, t2, c7;
};

__device__ __forceinline__ RunPoly run_poly(const float* c, const float* f)
{
    RunPoly o;
    const float fx = f[0], fy = f[1], fz = f[2];
    o.a = fmaf(c[7], fz, c[4]);
    const float b = fmaf(c[5], fz, c[1]);
    o.gx = fmaf(o.a, fy, b);
    const float e = fmaf(c[6], fz, c[2]), h = fmaf(c[3], fz, c[0]);
    o.value = fmaf(o.gx, fx, fmaf(e, fy, h));
    o.gy = fmaf(o.a, fx, e);
    o.t1 = fmaf(c[7], fy, c[5]);
    o.t2 = fmaf(c[7], fx, c[6]);
    o.gz = fmaf(fx, o.t1, fmaf(c[6], fy, c[3]));
    o.c7 = c[7];
    return o;
}

// Sum over the run of the cell polynomial: n A + S1 B + S2 C + S3 D.
__device__ __forceinline__ float run_sum(const CellRun& r, const RunPoly& o)
{
    const float dx = r.d[0], dy = r.d[1], dz = r.d[2];
    const float dxy = dx * dy, dxz = dx * dz, dyz = dy * dz;
    const float B = fmaf(o.gz, dz, fmaf(o.gy, dy, o.gx * dx));
    const float C = fmaf(o.t2, dyz, fmaf(o.t1, dxz, o.a * dxy));
    const float D = o.c7 * (dxy * dz);
    return fmaf(r.s3, D, fmaf(r.s2, C, fmaf(r.s1, B, r.nf * o.value)));
}

// Kahan-compensated FP32 sum.
struct Kahan32 {
    float sum = 0.0f, carry = 0.0f;
    __device__ __forceinline__ void add(float value)
    {
        const float y = value - carry;
        const float t = sum + y;
        carry = (t - sum) - y;
        sum = t;
    }
    __device__ __forceinline__ double value() const { return (double)sum - (double)carry; }
};

// ------------------------------------------------------ FP64 cell-Gauss integration
//
// Reference kernels/projection.py:522-746: the clipped ray is split at every interpolation
// plane (integer grid coordinates 0..n-1; the half-cell margins are segments of their own)
// and each segment, on which the trilinear field is a cubic in the ray parameter, is
// integrated exactly with the two-node Gauss rule.  The arithmetic follows the reference
// step for step (the FMA-corrected reciprocal crossings, ties advanced together), so the
// segments and nodes are the reference's.

// Strict FP64 sample (reference sample_field / sample_cell_fraction): zero outside the
// half-cell support; the value and, when `g` is given, the slope-masked grid gradient.
template <class Field>
__device__ __forceinline__ double sample_strict64(const Field& f, const FieldDims& d, const double* p,
                                                  double* g)
{
    if (g) g[0] = g[1] = g[2] = 0.0;
    if (!inside(p[0], p[1], p[2], d.nx, d.ny, d.nz)) return 0.0;
    const double mx = (double)(d.nx - 1), my = (double)(d.ny - 1), mz = (double)(d.nz - 1);
    const Axis64 X = axis64(p[0], mx, d.cx), Y = axis64(p[1], my, d.cy), Z = axis64(p[2], mz, d.cz);
    float v32[8];
    f.load_at((Z.lower * d.ny + Y.lower) * d.nx + X.lower, X.lower, Y.lower, Z.lower, v32);
    double v[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) v[c] = (double)v32[c];
    if (g) {
        const double sx = (p[0] >= 0.0 && p[0] < mx) ? 1.0 : 0.0;
        const double sy = (p[1] >= 0.0 && p[1] < my) ? 1.0 : 0.0;
        const double sz = (p[2] >= 0.0 && p[2] < mz) ? 1.0 : 0.0;
        slope64(X.fraction, Y.fraction, Z.fraction, v, sx, sy, sz, g);
    }
    return interpolate64(X.fraction, Y.fraction, Z.fraction, v);
}

struct GaussSegment {
    double end, radius, first_position, second_position;
    double first[3], second[3];  // the two Gauss nodes
    int lower[3];                // interpolation cell of the segment centre
    bool shared;                 // both nodes in that cell (one combined scatter)
};

struct CellWalk64 {
    int plane[3], step[3];
    double next[3], inverse[3];

    // reference crossing_quotient (:530-541): cached reciprocal with one FMA correction
    __device__ static double quotient(double delta, double direction, double inverse)
    {
        if (inverse == 0.0) return delta / direction;
        const double q = delta * inverse;
        if (!isfinite(q) || fabs(q) < 2.2250738585072014e-308) return delta / direction;
        return fma(fma(-q, direction, delta), inverse, q);
    }
    __device__ double crossing(const Ray64& r, int axis, const int* shape, double upper) const
    {
        if (r.direction[axis] == 0.0 || plane[axis] < 0 || plane[axis] >= shape[axis]) return upper;
        const double c = quotient((double)plane[axis] - r.origin[axis], r.direction[axis], inverse[axis]);
        return c < upper ? c : upper;
    }
    // reference begin_cells (:559-611)
    __device__ void begin(const Ray64& r, double lower, double upper, const int* shape)
    {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double entry = fma(lower, r.direction[a], r.origin[a]);
            const double v = r.direction[a];
            inverse[a] = 0.0;
            step[a] = 0;
            plane[a] = 0;
            if (v != 0.0) {
                const double inv = 1.0 / v;
                if (isfinite(inv) && fabs(inv) >= 2.2250738585072014e-308 && fabs(v) >= 2.2250738585072014e-308)
                    inverse[a] = inv;
            }
            if (v > 0.0) {
                step[a] = 1;
                const int c = (int)ceil(entry);
                plane[a] = c > 0 ? c : 0;
            } else if (v < 0.0) {
                step[a] = -1;
                const int c = (int)floor(entry);
                plane[a] = c < shape[a] - 1 ? c : shape[a] - 1;
            }
            double c = crossing(r, a, shape, upper);
            if (c <= lower) {
                plane[a] += step[a];
                c = crossing(r, a, shape, upper);
            }
            next[a] = c;
        }
    }
    // reference cell_segment (:614-646)
    __device__ void segment(const Ray64& r, double start, const FieldDims& d, GaussSegment& s) const
    {
        const double n12 = next[1] < next[2] ? next[1] : next[2];
        s.end = next[0] < n12 ? next[0] : n12;
        s.radius = (s.end - start) * 0.5;
        const double centre = start + s.radius;
        const double offset = s.radius / sqrt(3.0);
        s.first_position = centre - offset;
        s.second_position = centre + offset;
        double mid[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            s.first[a] = fma(s.first_position, r.direction[a], r.origin[a]);
            s.second[a] = fma(s.second_position, r.direction[a], r.origin[a]);
            mid[a] = fma(centre, r.direction[a], r.origin[a]);
        }
        const int shape[3] = {d.nx, d.ny, d.nz}, cap[3] = {d.cx, d.cy, d.cz};
        s.shared = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double high = (double)(shape[a] - 1);
            s.lower[a] = axis64(mid[a], high, cap[a]).lower;
            const double low = (double)s.lower[a], up = low + 1.0;
            const double c1 = fmin(fmax(s.first[a], 0.0), high), c2 = fmin(fmax(s.second[a], 0.0), high);
            if (c1 < low || c2 < low) s.shared = false;
            if (s.lower[a] < shape[a] - 2 && (c1 >= up || c2 >= up)) s.shared = false;
        }
    }
    // reference advance_cells (:649-660)
    __device__ void advance(const Ray64& r, const int* shape, double end, double upper)
    {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (next[a] <= end) {
                plane[a] += step[a];
                next[a] = crossing(r, a, shape, upper);
            }
        }
    }
};

// Compensated ray sum of the precision form: 16-sample blocks summed serially in FP32,
// block sums added with Kahan compensation.  Blocks are aligned to the sample index.
struct BlockSum {
    float block = 0.0f, sum = 0.0f, carry = 0.0f;
    __device__ __forceinline__ void kahan(float value)
    {
        const float y = value - carry;
        const float t = sum + y;
        carry = (t - sum) - y;
        sum = t;
    }
    __device__ __forceinline__ void add(float value, int index, int samples)
    {
        block = block + value;
        if ((index & 15) == 15 || index == samples - 1) {
            kahan(block);
            block = 0.0f;
        }
    }
    // the blocks after sample `last` hold only zeros: close the open block, then add the
    // zero block sums (which can still move the compensation into the sum)
    __device__ __forceinline__ void finish(int last, int samples)
    {
        if (last >= samples - 1) return;  // the block of the last sample is already closed
        if ((last & 15) != 15) {          // close the block containing `last`
            kahan(block);
            block = 0.0f;
        }
        // one zero sum per later block; once the compensation is zero they change nothing
        for (int start = (last | 15) + 1; start < samples && carry != 0.0f; start += 16) kahan(0.0f);
    }
    __device__ __forceinline__ double value() const { return (double)sum - (double)carry; }
};

// FP32 product with results below the normal range flushed to signed zero: the scatter
// increment of the reference (a rounded product, then |x| < 2^-126 -> 0, as CUDA's global
// FP32 atomics treat subnormal operands), in one instruction.
__device__ __forceinline__ float mul_ftz(float a, float b)
{
    float r;
    asm("mul.rn.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}

// ------------------------------------------------------------ packed FP32 pairs
//
// sm_100 executes add/sub/mul/fma on two FP32 lanes held in one 64-bit register pair per
// instruction, each lane rounded exactly as the scalar instruction rounds it.  The FP32
// sample loops evaluate two consecutive samples of a ray per instruction wherever their
// arithmetic is lane-wise (positions, coordinates, floors, corner weights, slopes, scatter
// increments): half the issue slots for the same results bit for bit.  Serial sums (the ray
// sum, the moments, a cell run's corner sums) stay scalar, sample i before sample i + 1.
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pack2(float lo, float hi)
{
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ f32x2 splat2(float v) { return pack2(v, v); }
__device__ __forceinline__ float lo2(f32x2 v)
{
    float a, b;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
    return a;
}
__device__ __forceinline__ float hi2(f32x2 v)
{
    float a, b;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
    return b;
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b)
{
    f32x2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b)
{
    f32x2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b)
{
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
// lane-wise mul_ftz: results below the normal range flushed to signed zero
__device__ __forceinline__ f32x2 mul_ftz2(f32x2 a, f32x2 b)
{
    f32x2 r;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c)
{
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// Floor of two coordinates known to satisfy 0 <= p < 2^23 on the FP32 pipe: p + 2^23 rounded
// toward -inf is 2^23 + floor(p) exactly (the sum lies in [2^23, 2^24), where the floats are
// the integers), so its bit pattern is 0x4B000000 + floor(p) and subtracting 2^23 again gives
// floor(p) exactly.  The fraction p - floor(p) is exact (Sterbenz), so this equals
// interior_axis lane by lane.  Returns the fractions; `biased` receives the biased floors.
constexpr float kFloorMagic = 8388608.0f;  // 2^23
constexpr int kFloorBias = 0x4B000000;     // bit pattern of 2^23
__device__ __forceinline__ f32x2 interior_fraction2(f32x2 p, f32x2* biased)
{
    f32x2 t;
    asm("add.rm.f32x2 %0, %1, %2;" : "=l"(t) : "l"(p), "l"(splat2(kFloorMagic)));
    *biased = t;
    return sub2(p, sub2(t, splat2(kFloorMagic)));
}
__device__ __forceinline__ int biased_lo(f32x2 t) { return __float_as_int(lo2(t)) - kFloorBias; }
__device__ __forceinline__ int biased_hi(f32x2 t) { return __float_as_int(hi2(t)) - kFloorBias; }

// Trilinear corner weights of two samples, (f0 f1) f2 per lane (corner_weights lane-wise).
__device__ __forceinline__ void corner_weights2(f32x2 fx, f32x2 fy, f32x2 fz, f32x2* w, f32x2* ax_out = nullptr,
                                                f32x2* ay_out = nullptr, f32x2* az_out = nullptr)
{
    const f32x2 one = splat2(1.0f);
    const f32x2 ax = sub2(one, fx), ay = sub2(one, fy), az = sub2(one, fz);
    const f32x2 p00 = mul2(ax, ay), p10 = mul2(fx, ay), p01 = mul2(ax, fy), p11 = mul2(fx, fy);
    w[0] = mul2(p00, az);
    w[1] = mul2(p10, az);
    w[2] = mul2(p01, az);
    w[3] = mul2(p11, az);
    w[4] = mul2(p00, fz);
    w[5] = mul2(p10, fz);
    w[6] = mul2(p01, fz);
    w[7] = mul2(p11, fz);
    if (ax_out) *ax_out = ax;
    if (ay_out) *ay_out = ay;
    if (az_out) *az_out = az;
}

// Interior slopes of two samples (slope32 with every mask 1), from each sample's eight corner
// values: the twelve differences per sample are scalar, their combination lane-wise.
__device__ __forceinline__ void slope2(f32x2 fx, f32x2 fy, f32x2 fz, f32x2 ax, f32x2 ay, f32x2 az,
                                       const float* u, const float* v, f32x2* g)
{
    const f32x2 d10 = pack2(u[1] - u[0], v[1] - v[0]), d32 = pack2(u[3] - u[2], v[3] - v[2]);
    const f32x2 d54 = pack2(u[5] - u[4], v[5] - v[4]), d76 = pack2(u[7] - u[6], v[7] - v[6]);
    g[0] = fma2(fz, fma2(fy, d76, mul2(ay, d54)), mul2(az, fma2(fy, d32, mul2(ay, d10))));
    const f32x2 d20 = pack2(u[2] - u[0], v[2] - v[0]), d31 = pack2(u[3] - u[1], v[3] - v[1]);
    const f32x2 d64 = pack2(u[6] - u[4], v[6] - v[4]), d75 = pack2(u[7] - u[5], v[7] - v[5]);
    g[1] = fma2(fz, fma2(fx, d75, mul2(ax, d64)), mul2(az, fma2(fx, d31, mul2(ax, d20))));
    const f32x2 d40 = pack2(u[4] - u[0], v[4] - v[0]), d51 = pack2(u[5] - u[1], v[5] - v[1]);
    const f32x2 d62 = pack2(u[6] - u[2], v[6] - v[2]), d73 = pack2(u[7] - u[3], v[7] - v[3]);
    g[2] = fma2(fy, fma2(fx, d73, mul2(ax, d62)), mul2(ay, fma2(fx, d51, mul2(ax, d40))));
}

// Per-block staging of the view's pose (12 doubles) and panel record.
struct ViewShared {
    double pose[12];
    double table[DPT_VIEW_WORDS];
};

__device__ __forceinline__ void stage_view(const RayArgs& a, int view, ViewShared& s)
{
    const int t = threadIdx.x;
    if (t < 12) s.pose[t] = a.poses[12 * (int64_t)view + t];
    if (a.ray_kind == DPT_RAYS_PANELS && t >= 32 && t < 32 + DPT_VIEW_WORDS)
        s.table[t - 32] = a.view_table[(int64_t)view * DPT_VIEW_WORDS + (t - 32)];
    __syncthreads();
}

}  // namespace dpt
