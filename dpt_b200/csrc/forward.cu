// forward.cu - optical depth and per-ray clip counts.
//
// One thread marches one ray; a 128-thread block covers a 16x8 detector tile (each warp
// an 8x4 sub-tile) so the 32 rays of a warp sample neighbouring voxels at every step and
// their corner loads share L1 lines.  One launch covers every view of a call, where the
// reference launches once per view; the blocks run in groups of neighbouring views (block_work).
//
// Arithmetic per mode (reference hcltech-robotics/dpt):
//   F32  - python/dpt/kernels/projection_fp32.py:334-374 (FP64 setup, FP32 clip, fmaf
//          midpoints, fmaf corner sum, serial FP32 total, total *= length*step)
//   F64  - python/dpt/kernels/projection.py:802-846 with the midpoint integrator 770-799
//   F32C - FP64 setup and clip; FP32 marching p_i = entry + (i+0.5) step_vector (the mixed
//          recurrence of python/dpt/kernels/projection.py:368-392); the samples of each cell
//          run summed in closed form from the cell's trilinear polynomial, the run sums added
//          with Kahan compensation and scaled by length*step in FP64 (this library's
//          precision form, no reference counterpart).
//
// Samples inside the support form one run; within it the interior run (0 <= p < n-1 on every
// axis) skips the clamps of the cell coordinate.  Both are exact rewrites of the per-sample
// tests, so every mode keeps its arithmetic bit for bit.
#include <type_traits>

#include "launch.h"

#ifndef DPT_FORWARD_REUSE
#define DPT_FORWARD_REUSE 1  // FP32 forward: reload the corners only when the sample enters another cell
#endif

namespace dpt {
namespace {

// FP32 sample of the field at grid point (x, y, z): zero outside the half-cell support.
template <class Field>
__device__ __forceinline__ float sample32(const Field& f, const FieldDims& d, float x, float y,
                                          float z)
{
    if (!inside(x, y, z, d.hx, d.hy, d.hz)) return 0.0f;
    const Axis32 X = axis32(x, d.mx, d.cx), Y = axis32(y, d.my, d.cy), Z = axis32(z, d.mz, d.cz);
    float v[8], w[8];
    f.load(X.lower, Y.lower, Z.lower, v);
    corner_weights(X.fraction, Y.fraction, Z.fraction, w);
    return interpolate(w, v);
}

template <class Field>
__device__ __forceinline__ double sample64(const Field& f, const Grid& g, const double* p)
{
    if (!inside(p[0], p[1], p[2], g.nx, g.ny, g.nz)) return 0.0;
    const Axis64 X = axis64(p[0], (double)(g.nx - 1), max(g.nx - 2, 0));
    const Axis64 Y = axis64(p[1], (double)(g.ny - 1), max(g.ny - 2, 0));
    const Axis64 Z = axis64(p[2], (double)(g.nz - 1), max(g.nz - 2, 0));
    float v32[8];
    f.load(X.lower, Y.lower, Z.lower, v32);
    double v[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) v[c] = (double)v32[c];
    return interpolate64(X.fraction, Y.fraction, Z.fraction, v);
}

template <typename Out>
__device__ __forceinline__ bool finite_out(double value)
{
    return isfinite((Out)value);
}

// The rays of one detector tile of one view: every thread of the block calls it (stage_view
// synchronises the block), padding threads return after the staging.
template <int kArith, class Field, typename Out>
__device__ __forceinline__ void forward_tile(const RayArgs& a, const Field& f, Out* __restrict__ image,
                                             int view_local, int tile, ViewShared& vs, const float4* run_sums)
{
    const int view = a.view_begin + view_local;
    stage_view(a, view, vs);  // synchronises the block (the table is ready)
    int pixel;
    if (!ray_of_thread(a, tile, &pixel)) return;

    double source[3], end[3];
    ray_endpoints(a, vs.table, view, pixel, source, end);
    Ray64 r;
    ray_setup(a.grid, vs.pose, source, end, r);
    const int S = a.samples;
    int bits = 0;
    double result = 0.0;

    if constexpr (kArith == DPT_ARITH_F32) {
        const float o[3] = {(float)r.origin[0], (float)r.origin[1], (float)r.origin[2]};
        const float d[3] = {(float)r.direction[0], (float)r.direction[1], (float)r.direction[2]};
        const float length = (float)r.length;
        if (!valid_ray(r) || !finite3f(o[0], o[1], o[2]) || !finite3f(d[0], d[1], d[2]) ||
            !isfinite(length) || length <= 0.0f) {
            bits = 2;
        } else {
            Interval<float> iv;
            iv.clip(o, d, a.grid.nx, a.grid.ny, a.grid.nz);
            float total = 0.0f;
            if (iv.upper > iv.lower) {
                FieldDims dims;
                dims.init(a.grid);
                const float step = (iv.upper - iv.lower) / (float)S;
                auto at = [&](int i, float& x, float& y, float& z) {
                    const float position = fmaf((float)i + 0.5f, step, iv.lower);
                    x = fmaf(position, d[0], o[0]);
                    y = fmaf(position, d[1], o[1]);
                    z = fmaf(position, d[2], o[2]);
                };
                if (!moderate(o, d)) {
                    bool finite = true;
                    for (int i = 0; i < S; ++i) {
                        float x, y, z;
                        at(i, x, y, z);
                        finite = finite && finite3f(x, y, z);
                        total = total + sample32(f, dims, x, y, z);
                    }
                    if (!finite) bits |= 2;
                } else {
                    int first, last;
                    inside_run(S, [&](int i) {
                        float x, y, z;
                        at(i, x, y, z);
                        return inside(x, y, z, dims.hx, dims.hy, dims.hz);
                    }, first, last);
                    int ifirst, ilast;
                    interior_run(first, last, [&](int i) {
                        float x, y, z;
                        at(i, x, y, z);
                        return x >= 0.0f && x < dims.mx && y >= 0.0f && y < dims.my && z >= 0.0f && z < dims.mz;
                    }, ifirst, ilast);
                    CellCache<Field, DPT_FORWARD_REUSE != 0> cache;
                    auto add = [&](Axis32 X, Axis32 Y, Axis32 Z) {
                        cache.fetch(f, X.lower, Y.lower, Z.lower, (Z.lower * dims.ny + Y.lower) * dims.nx + X.lower);
                        float w[8];
                        corner_weights(X.fraction, Y.fraction, Z.fraction, w);
                        total = total + interpolate(w, cache.v);
                    };
                    auto margin = [&](int i) {
                        float x, y, z;
                        at(i, x, y, z);
                        add(axis32(x, dims.mx, dims.cx), axis32(y, dims.my, dims.cy), axis32(z, dims.mz, dims.cz));
                    };
                    const int split = min(ifirst, last + 1);
                    for (int i = first; i < split; ++i) margin(i);
#pragma unroll 4
                    for (int i = ifirst; i <= ilast; ++i) {
                        float x, y, z;
                        at(i, x, y, z);
                        add(interior_axis(x), interior_axis(y), interior_axis(z));
                    }
                    for (int i = max(ilast + 1, split); i <= last; ++i) margin(i);
                    // the zero samples after the run: adding +0 only turns -0 into +0
                    if (last < S - 1) total = total + 0.0f;
                }
                total = total * (length * step);
            }
            if (!isfinite(total)) bits |= 2;
            result = total;
        }
    } else if constexpr (kArith == DPT_ARITH_CELLS) {
        // reference integration="cell_gauss" (kernels/projection.py:717-746, segment action
        // :695-711): two Gauss nodes per cell segment, L = length * sum radius * value
        if (!valid_ray(r)) {
            bits = 2;
        } else {
            Interval<double> iv;
            iv.clip(r.origin, r.direction, a.grid.nx, a.grid.ny, a.grid.nz);
            double integral = 0.0;
            if (iv.upper > iv.lower) {
                FieldDims dims;
                dims.init(a.grid);
                const int shape[3] = {dims.nx, dims.ny, dims.nz};
                CellWalk64 walk;
                walk.begin(r, iv.lower, iv.upper, shape);
                double start = iv.lower;
                const int64_t limit = (int64_t)shape[0] + shape[1] + shape[2] + 1;
                for (int64_t segments = 0; start < iv.upper && segments < limit; ++segments) {
                    GaussSegment s;
                    walk.segment(r, start, dims, s);
                    if (s.end <= start) {
                        bits |= 2;
                        break;
                    }
                    if (!finite3(s.first[0], s.first[1], s.first[2]) ||
                        !finite3(s.second[0], s.second[1], s.second[2]))
                        bits |= 2;
                    integral = fma(s.radius, sample_strict64(f, dims, s.first, nullptr), integral);
                    integral = fma(s.radius, sample_strict64(f, dims, s.second, nullptr), integral);
                    start = s.end;
                    walk.advance(r, shape, s.end, iv.upper);
                }
                if (start < iv.upper) bits |= 2;
                integral = integral * r.length;
            }
            result = integral;
            if (!finite_out<Out>(result)) bits |= 2;
        }
    } else if constexpr (kArith == DPT_ARITH_MIXED || kArith == DPT_ARITH_FAST) {
        // reference mixed_float32 / fast_float32 (kernels/projection.py:296-392): FP64 clip,
        // FP32 marching and clamped corner weights, the corner sum in FP64 (MIXED) or as an
        // FP32 fmaf chain promoted to the FP64 ray sum (FAST)
        if (!valid_ray(r)) {
            bits = 2;
        } else {
            Interval<double> iv;
            iv.clip(r.origin, r.direction, a.grid.nx, a.grid.ny, a.grid.nz);
            double integral = 0.0;
            if (iv.upper > iv.lower) {
                FieldDims dims;
                dims.init(a.grid);
                const double step = (iv.upper - iv.lower) / (double)S;
                float entry[3], sv[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    entry[k] = (float)fma(iv.lower, r.direction[k], r.origin[k]);
                    sv[k] = (float)(step * r.direction[k]);
                }
                auto at = [&](int i, float& x, float& y, float& z) {
                    const float offset = (float)i + 0.5f;
                    x = fmaf(offset, sv[0], entry[0]);
                    y = fmaf(offset, sv[1], entry[1]);
                    z = fmaf(offset, sv[2], entry[2]);
                };
                // MIXED keeps the cell's corners widened to FP64, so a sample widens only its
                // eight weights (the products w_c v_c are exact in FP64 either way)
                std::conditional_t<kArith == DPT_ARITH_FAST, CellCache<Field>, WideCellCache<Field>> cache;
                auto add = [&](Axis32 X, Axis32 Y, Axis32 Z) {
                    cache.fetch(f, X.lower, Y.lower, Z.lower, (Z.lower * dims.ny + Y.lower) * dims.nx + X.lower);
                    float w[8];
                    corner_weights(X.fraction, Y.fraction, Z.fraction, w);
                    if constexpr (kArith == DPT_ARITH_FAST) {
                        float value = 0.0f;
#pragma unroll
                        for (int c = 0; c < 8; ++c) value = fmaf(w[c], cache.v[c], value);
                        integral = integral + (double)value;
                    } else {
                        double value = 0.0;
#pragma unroll
                        for (int c = 0; c < 8; ++c) value = fma((double)w[c], cache.v[c], value);
                        integral = integral + value;
                    }
                };
                auto sample = [&](int i) {
                    float x, y, z;
                    at(i, x, y, z);
                    if (inside(x, y, z, dims.hx, dims.hy, dims.hz))
                        add(axis32(x, dims.mx, dims.cx), axis32(y, dims.my, dims.cy), axis32(z, dims.mz, dims.cz));
                    else
                        integral = integral + 0.0;
                };
                if (!moderate(entry, sv)) {
                    bool finite = true;
                    for (int i = 0; i < S; ++i) {
                        float x, y, z;
                        at(i, x, y, z);
                        finite = finite && finite3f(x, y, z);
                        sample(i);
                    }
                    if (!finite) bits |= 2;
                } else {
                    int first, last;
                    inside_run(S, [&](int i) {
                        float x, y, z;
                        at(i, x, y, z);
                        return inside(x, y, z, dims.hx, dims.hy, dims.hz);
                    }, first, last);
                    int ifirst, ilast;
                    interior_run(first, last, [&](int i) {
                        float x, y, z;
                        at(i, x, y, z);
                        return x >= 0.0f && x < dims.mx && y >= 0.0f && y < dims.my && z >= 0.0f && z < dims.mz;
                    }, ifirst, ilast);
                    const int split = min(ifirst, last + 1);
                    for (int i = first; i < split; ++i) sample(i);
#pragma unroll 2
                    for (int i = ifirst; i <= ilast; ++i) {
                        float x, y, z;
                        at(i, x, y, z);
                        add(interior_axis(x), interior_axis(y), interior_axis(z));
                    }
                    for (int i = max(ilast + 1, split); i <= last; ++i) sample(i);
                    // the zero samples after the run: adding +0 only turns -0 into +0
                    if (last < S - 1) integral = integral + 0.0;
                }
                integral = integral * (r.length * step);
            }
            result = integral;
            if (!finite_out<Out>(result)) bits |= 2;
        }
    } else if constexpr (kArith == DPT_ARITH_F64) {
        if (!valid_ray(r)) {
            bits = 2;
        } else {
            Interval<double> iv;
            iv.clip(r.origin, r.direction, a.grid.nx, a.grid.ny, a.grid.nz);
            double integral = 0.0;
            if (iv.upper > iv.lower) {
                const double step = (iv.upper - iv.lower) / (double)S;
                auto at = [&](int i, double* p) {
                    const double position = fma((double)i + 0.5, step, iv.lower);
#pragma unroll
                    for (int k = 0; k < 3; ++k) p[k] = fma(position, r.direction[k], r.origin[k]);
                };
                if (!moderate(r.origin, r.direction)) {
                    bool finite = true;
                    for (int i = 0; i < S; ++i) {
                        double p[3];
                        at(i, p);
                        finite = finite && finite3(p[0], p[1], p[2]);
                        integral = integral + sample64(f, a.grid, p);
                    }
                    if (!finite) bits |= 2;
                } else {
                    int first, last;
                    inside_run(S, [&](int i) {
                        double p[3];
                        at(i, p);
                        return inside(p[0], p[1], p[2], a.grid.nx, a.grid.ny, a.grid.nz);
                    }, first, last);
                    const double mx = (double)(a.grid.nx - 1), my = (double)(a.grid.ny - 1), mz = (double)(a.grid.nz - 1);
                    const int cx = max(a.grid.nx - 2, 0), cy = max(a.grid.ny - 2, 0), cz = max(a.grid.nz - 2, 0);
                    WideCellCache<Field> cache;
#pragma unroll 2
                    for (int i = first; i <= last; ++i) {
                        double p[3];
                        at(i, p);
                        const Axis64 X = axis64(p[0], mx, cx), Y = axis64(p[1], my, cy), Z = axis64(p[2], mz, cz);
                        cache.fetch(f, X.lower, Y.lower, Z.lower, (Z.lower * a.grid.ny + Y.lower) * a.grid.nx + X.lower);
                        integral = integral + interpolate64(X.fraction, Y.fraction, Z.fraction, cache.v);
                    }
                    if (last < S - 1) integral = integral + 0.0;
                }
                integral = integral * (r.length * step);
            }
            result = integral;
            if (!finite_out<Out>(result)) bits |= 2;
        }
    } else {
        if (!valid_ray(r)) {
            bits = 2;
        } else {
            Interval<double> iv;
            iv.clip(r.origin, r.direction, a.grid.nx, a.grid.ny, a.grid.nz);
            if (iv.upper > iv.lower) {
                FieldDims dims;
                dims.init(a.grid);
                const double step = (iv.upper - iv.lower) / (double)S;
                float entry[3], sv[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    entry[k] = (float)fma(iv.lower, r.direction[k], r.origin[k]);
                    sv[k] = (float)(step * r.direction[k]);
                }
                auto at = [&](int i, float& x, float& y, float& z) {
                    const float offset = (float)i + 0.5f;
                    x = fmaf(offset, sv[0], entry[0]);
                    y = fmaf(offset, sv[1], entry[1]);
                    z = fmaf(offset, sv[2], entry[2]);
                };
                double total;
                if (!segment_form(entry, sv)) {
                    // per-sample form: polynomial samples, blocked compensated sum
                    BlockSum acc;
                    PolyCache<Field> cache;
                    bool finite = true;
                    for (int i = 0; i < S; ++i) {
                        float x, y, z;
                        at(i, x, y, z);
                        finite = finite && finite3f(x, y, z);
                        if (inside(x, y, z, dims.hx, dims.hy, dims.hz)) {
                            const Axis32 X = axis32(x, dims.mx, dims.cx), Y = axis32(y, dims.my, dims.cy),
                                         Z = axis32(z, dims.mz, dims.cz);
                            cache.fetch(f, X.lower, Y.lower, Z.lower, (Z.lower * dims.ny + Y.lower) * dims.nx + X.lower);
                            acc.add(cache.eval(X.fraction, Y.fraction, Z.fraction), i, S);
                        } else {
                            acc.add(0.0f, i, S);
                        }
                    }
                    if (!finite) bits |= 2;
                    total = acc.value();
                } else {
                    // segment form: closed-form sums over the cell runs, compensated across runs
                    int first, last;
                    inside_run(S, [&](int i) {
                        float x, y, z;
                        at(i, x, y, z);
                        return inside(x, y, z, dims.hx, dims.hy, dims.hz);
                    }, first, last);
                    Kahan32 acc;
                    if (first <= last) {
                        walk_cells(dims, entry, sv, first, last, [&](const CellRun& run) {
                            PolyCache<Field, false> cell;
                            cell.fetch(f, run.lx, run.ly, run.lz, run.cell);
                            acc.add(run_sum(run, run_poly(cell.c, run.f)));
                        }, run_sums);
                    }
                    total = acc.value();
                }
                result = total * (r.length * step);
            }
            if (!finite_out<Out>(result)) bits |= 2;
        }
    }
    const int64_t rays_per_view = (int64_t)a.rows * a.cols;
    image[view_local * rays_per_view + pixel] = (Out)result;
    if (bits) atomicOr(a.status + view, bits);
}

template <int kArith, class Field, typename Out>
__global__ void __launch_bounds__(kForwardBlock) k_forward(RayArgs a, Field f, Out* __restrict__ image)
{
    __shared__ ViewShared vs;
    __shared__ float4 run_sums[kArith == DPT_ARITH_F32C ? kRunSumTable + 1 : 1];
    if (kArith == DPT_ARITH_F32C) fill_run_sums(run_sums);
    int view_local, tile;
    block_work(a, &view_local, &tile);
    forward_tile<kArith, Field, Out>(a, f, image, view_local, tile, vs, run_sums);
}

// Forward of several problems of one arithmetic in one launch.  The work items are the (view,
// tile) blocks of every problem, problem by problem (each in its own grouped-view order), one
// block per item, so the block scheduler hands items to SMs as they free up.  (A grid of the
// resident blocks walking the items with a fixed stride ran 8 views of 512^2 at S = 512 in
// 27.1 ms per 8 requests against 20.1 ms for one block per item: a fixed split cannot follow
// the unequal cost of rays that cross the volume and rays that miss it.)  No block waits on
// another.  The descriptors travel as the kernel's parameter (up to kMaxPack).
template <class Field>
struct PackedForward {
    int count;                // problems
    int total;                // work items of all problems
    int first[kMaxPack + 1];  // first work item of problem r; first[count] = total
    RayArgs args[kMaxPack];
    Field fields[kMaxPack];
    void* images[kMaxPack];
};
// the whole descriptor set is one kernel parameter: 32,764 bytes at most (CUDA 12.1, Volta on)
static_assert(sizeof(PackedForward<QuadF32>) <= 32764, "packed descriptors exceed the parameter space");

// Blocks per SM the packed kernel is compiled for: the occupancy the single-problem kernel of
// the same arithmetic reaches (its register count at 128 threads).  Indexing the descriptors
// with a run-time problem number costs registers the single-problem kernel takes from the
// constant bank; without the bound the FP32 form drops from 9 to 7 resident blocks and runs
// 8 requests of 8 views of 512^2 at S = 512 in 20.1 ms against 18.6 ms with it.
template <int kArith>
constexpr int packed_min_blocks()
{
    return kArith == DPT_ARITH_F32 || kArith == DPT_ARITH_FAST ? 9
         : kArith == DPT_ARITH_F64 ? 7
         : kArith == DPT_ARITH_CELLS ? 5
         : 8;  // compensated, mixed
}

template <int kArith, class Field, typename Out>
__global__ void __launch_bounds__(kForwardBlock, packed_min_blocks<kArith>())
    k_forward_packed(const __grid_constant__ PackedForward<Field> p)
{
    __shared__ ViewShared vs;
    __shared__ float4 run_sums[kArith == DPT_ARITH_F32C ? kRunSumTable + 1 : 1];
    if (kArith == DPT_ARITH_F32C) fill_run_sums(run_sums);
    const int item = blockIdx.x;
    int lo = 0, hi = p.count - 1;  // the problem r with first[r] <= item < first[r + 1]
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p.first[mid] <= item)
            lo = mid;
        else
            hi = mid - 1;
    }
    const RayArgs& a = p.args[lo];
    int view_local, tile;
    block_work_at(a, item - p.first[lo], &view_local, &tile);
    forward_tile<kArith, Field, Out>(a, p.fields[lo], static_cast<Out*>(p.images[lo]), view_local, tile, vs,
                                     run_sums);
}

// Per-ray interval and number of midpoints inside the support, in each mode's arithmetic.
template <int kArith>
__global__ void __launch_bounds__(kBlock) k_counts(RayArgs a, double* __restrict__ lower,
                                                   double* __restrict__ upper,
                                                   int32_t* __restrict__ realised)
{
    __shared__ ViewShared vs;
    int view_local, tile;
    block_work(a, &view_local, &tile);
    const int view = a.view_begin + view_local;
    stage_view(a, view, vs);
    int pixel;
    if (!ray_of_thread(a, tile, &pixel)) return;
    double source[3], end[3];
    ray_endpoints(a, vs.table, view, pixel, source, end);
    Ray64 r;
    ray_setup(a.grid, vs.pose, source, end, r);
    const int S = a.samples;
    int count = 0;
    double lo = 0.0, hi = -1.0;
    FieldDims dims;
    dims.init(a.grid);
    if (kArith == DPT_ARITH_F32) {
        const float o[3] = {(float)r.origin[0], (float)r.origin[1], (float)r.origin[2]};
        const float d[3] = {(float)r.direction[0], (float)r.direction[1], (float)r.direction[2]};
        const float length = (float)r.length;
        if (valid_ray(r) && finite3f(o[0], o[1], o[2]) && finite3f(d[0], d[1], d[2]) &&
            isfinite(length) && length > 0.0f) {
            Interval<float> iv;
            iv.clip(o, d, a.grid.nx, a.grid.ny, a.grid.nz);
            lo = iv.lower;
            hi = iv.upper;
            if (iv.upper > iv.lower) {
                const float step = (iv.upper - iv.lower) / (float)S;
                for (int i = 0; i < S; ++i) {
                    const float position = fmaf((float)i + 0.5f, step, iv.lower);
                    count += inside(fmaf(position, d[0], o[0]), fmaf(position, d[1], o[1]),
                                    fmaf(position, d[2], o[2]), dims.hx, dims.hy, dims.hz);
                }
            }
        }
    } else if (valid_ray(r)) {
        Interval<double> iv;
        iv.clip(r.origin, r.direction, a.grid.nx, a.grid.ny, a.grid.nz);
        lo = iv.lower;
        hi = iv.upper;
        if (iv.upper > iv.lower) {
            const double step = (iv.upper - iv.lower) / (double)S;
            if (kArith == DPT_ARITH_F64) {
                for (int i = 0; i < S; ++i) {
                    const double position = fma((double)i + 0.5, step, iv.lower);
                    count += inside(fma(position, r.direction[0], r.origin[0]),
                                    fma(position, r.direction[1], r.origin[1]),
                                    fma(position, r.direction[2], r.origin[2]), a.grid.nx,
                                    a.grid.ny, a.grid.nz);
                }
            } else {
                float entry[3], sv[3];
                for (int k = 0; k < 3; ++k) {
                    entry[k] = (float)fma(iv.lower, r.direction[k], r.origin[k]);
                    sv[k] = (float)(step * r.direction[k]);
                }
                for (int i = 0; i < S; ++i) {
                    const float offset = (float)i + 0.5f;
                    count += inside(fmaf(offset, sv[0], entry[0]), fmaf(offset, sv[1], entry[1]),
                                    fmaf(offset, sv[2], entry[2]), dims.hx, dims.hy, dims.hz);
                }
            }
        }
    }
    const int64_t index = view_local * (int64_t)a.rows * a.cols + pixel;
    lower[index] = lo;
    upper[index] = hi;
    realised[index] = count;
}

template <int kArith, class Field>
cudaError_t forward_with(const dpt_problem& p, const RayArgs& a, const Field& f, void* image,
                         dim3 grid, cudaStream_t stream)
{
    if (p.image_dtype == DPT_F64)
        k_forward<kArith, Field, double><<<grid, kForwardBlock, 0, stream>>>(a, f, static_cast<double*>(image));
    else
        k_forward<kArith, Field, float><<<grid, kForwardBlock, 0, stream>>>(a, f, static_cast<float*>(image));
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_forward(const dpt_problem& p, const RayArgs& a, const void* packed, void* image,
                           cudaStream_t stream)
{
    const dim3 grid(ray_blocks(a));
    if (p.arith == DPT_ARITH_F32C && p.layout == DPT_LAYOUT_REPLICATED) {
        PolyF32 f{static_cast<const float4*>(packed), p.nx, p.ny, p.nz};
        return forward_with<DPT_ARITH_F32C>(p, a, f, image, grid, stream);
    }
    // direct gathers from the caller's FP32 field, or the FP32 corner quads (decoded from any
    // storage type by the pack kernel)
    auto run = [&](const auto& f) -> cudaError_t {
        switch (p.arith) {
        case DPT_ARITH_F32: return forward_with<DPT_ARITH_F32>(p, a, f, image, grid, stream);
        case DPT_ARITH_F64: return forward_with<DPT_ARITH_F64>(p, a, f, image, grid, stream);
        case DPT_ARITH_MIXED: return forward_with<DPT_ARITH_MIXED>(p, a, f, image, grid, stream);
        case DPT_ARITH_FAST: return forward_with<DPT_ARITH_FAST>(p, a, f, image, grid, stream);
        case DPT_ARITH_CELLS: return forward_with<DPT_ARITH_CELLS>(p, a, f, image, grid, stream);
        default: return forward_with<DPT_ARITH_F32C>(p, a, f, image, grid, stream);
        }
    };
    if (p.layout == DPT_LAYOUT_DIRECT) return run(PlainF32{static_cast<const float*>(packed), p.nx, p.ny, p.nz});
    return run(QuadF32{static_cast<const float4*>(packed), p.nx, p.ny, p.nz});
}

namespace {

template <int kArith, class Field, typename Out>
cudaError_t packed_with(int count, const RayArgs* args, const Field* fields, void* const* images,
                        cudaStream_t stream)
{
    PackedForward<Field> p{};
    p.count = count;
    int64_t total = 0;
    for (int r = 0; r < count; ++r) {
        p.first[r] = (int)total;
        total += (int64_t)ray_blocks(args[r]);
        p.args[r] = args[r];
        p.fields[r] = fields[r];
        p.images[r] = images[r];
    }
    if (total >= ((int64_t)1 << 31)) return cudaErrorInvalidValue;
    p.first[count] = p.total = (int)total;
    if (total < 1) return cudaSuccess;
    k_forward_packed<kArith, Field, Out><<<(unsigned)total, kForwardBlock, 0, stream>>>(p);
    return cudaGetLastError();
}

template <int kArith, class Field>
cudaError_t packed_out(const dpt_problem& p0, int count, const RayArgs* args, const Field* fields,
                       void* const* images, cudaStream_t stream)
{
    if (p0.image_dtype == DPT_F64) return packed_with<kArith, Field, double>(count, args, fields, images, stream);
    return packed_with<kArith, Field, float>(count, args, fields, images, stream);
}

}  // namespace

cudaError_t launch_forward_packed(int count, const dpt_problem* problems, const RayArgs* args,
                                  const void* const* packed, void* const* images, cudaStream_t stream)
{
    const dpt_problem& p0 = problems[0];
    auto fields_of = [&](auto make, auto* fields) {
        for (int r = 0; r < count; ++r) fields[r] = make(problems[r], packed[r]);
    };
    if (p0.arith == DPT_ARITH_F32C && p0.layout == DPT_LAYOUT_REPLICATED) {
        PolyF32 fields[kMaxPack];
        fields_of([](const dpt_problem& p, const void* ptr) {
            return PolyF32{static_cast<const float4*>(ptr), p.nx, p.ny, p.nz};
        }, fields);
        return packed_out<DPT_ARITH_F32C>(p0, count, args, fields, images, stream);
    }
    auto run = [&](const auto* fields) -> cudaError_t {
        using FieldT = std::remove_cv_t<std::remove_pointer_t<decltype(fields)>>;
        switch (p0.arith) {
        case DPT_ARITH_F32: return packed_out<DPT_ARITH_F32, FieldT>(p0, count, args, fields, images, stream);
        case DPT_ARITH_F64: return packed_out<DPT_ARITH_F64, FieldT>(p0, count, args, fields, images, stream);
        case DPT_ARITH_MIXED: return packed_out<DPT_ARITH_MIXED, FieldT>(p0, count, args, fields, images, stream);
        case DPT_ARITH_FAST: return packed_out<DPT_ARITH_FAST, FieldT>(p0, count, args, fields, images, stream);
        case DPT_ARITH_CELLS: return packed_out<DPT_ARITH_CELLS, FieldT>(p0, count, args, fields, images, stream);
        default: return packed_out<DPT_ARITH_F32C, FieldT>(p0, count, args, fields, images, stream);
        }
    };
    if (p0.layout == DPT_LAYOUT_DIRECT) {
        PlainF32 fields[kMaxPack];
        fields_of([](const dpt_problem& p, const void* ptr) {
            return PlainF32{static_cast<const float*>(ptr), p.nx, p.ny, p.nz};
        }, fields);
        return run(static_cast<const PlainF32*>(fields));
    }
    QuadF32 fields[kMaxPack];
    fields_of([](const dpt_problem& p, const void* ptr) {
        return QuadF32{static_cast<const float4*>(ptr), p.nx, p.ny, p.nz};
    }, fields);
    return run(static_cast<const QuadF32*>(fields));
}

cudaError_t launch_counts(const dpt_problem& p, const RayArgs& a, double* lower, double* upper,
                          int32_t* realised, cudaStream_t stream)
{
    const dim3 grid(ray_blocks(a));
    if (p.arith == DPT_ARITH_F32)
        k_counts<DPT_ARITH_F32><<<grid, kBlock, 0, stream>>>(a, lower, upper, realised);
    else if (p.arith == DPT_ARITH_F64 || p.arith == DPT_ARITH_CELLS)
        k_counts<DPT_ARITH_F64><<<grid, kBlock, 0, stream>>>(a, lower, upper, realised);
    else  // F32C, MIXED and FAST share the FP64 clip and the FP32 marching
        k_counts<DPT_ARITH_F32C><<<grid, kBlock, 0, stream>>>(a, lower, upper, realised);
    return cudaGetLastError();
}

}  // namespace dpt
