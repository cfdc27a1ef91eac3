// gather.cu - deterministic voxel-driven transpose of the strict FP64 projection, midpoint or
// cell-Gauss (reference python/dpt/projection.py:1087-1405, kernels
// python/dpt/kernels/projection_adjoint.py).
//
// out[v] = sum over views, rays p and midpoint samples s of the corner weight of voxel v at
// sample s of ray p, times cotangent[p] |e - s| span / S, summed per voxel in FP64 in a fixed
// order: views ascending (each view's sum formed from zero and then added to the running
// value, as a per-view loop with accumulation would), then detector rows, columns and samples
// ascending.  One thread owns one voxel, so the result is bitwise reproducible and does not
// depend on the launch.
//
// A prepared plan holds, per ray, the FP64 ray in grid coordinates with its clip interval
// and a bound on the rounding of its sample points, and per view the culling metrics.  Each
// voxel then visits only the rays and samples that can reach its support box: for cone
// panels the detector rectangle of the box's perspective image (outward-rounded interval
// arithmetic, widened by the largest detector-coordinate error measured on the rays
// themselves), for every ray the sample-index range of its passage through the box.  Both
// bounds are conservative, so a culled sum visits every non-zero term in the same order as
// the sum over all rays and samples and is bitwise equal to it.
#include <cstdint>

#include "launch.h"

namespace dpt {
namespace {

constexpr int kGatherThreads = 128;
#ifndef DPT_GATHER_MIN_BLOCKS
#define DPT_GATHER_MIN_BLOCKS 6  // resident 128-thread blocks per SM the midpoint gather is compiled for
#endif

// The adjacent double below / above x (nextafter toward -inf / +inf): one integer step of the
// bit pattern, with NaN and the infinity in the direction of travel unchanged and a zero
// stepping to the smallest subnormal.
__device__ __forceinline__ double down(double x)
{
    if (x != x || x == -INFINITY) return x;
    if (x == 0.0) return -4.9406564584124654e-324;
    return __longlong_as_double(__double_as_longlong(x) + (x > 0.0 ? -1 : 1));
}
__device__ __forceinline__ double up(double x)
{
    if (x != x || x == INFINITY) return x;
    if (x == 0.0) return 4.9406564584124654e-324;
    return __longlong_as_double(__double_as_longlong(x) + (x > 0.0 ? 1 : -1));
}

// Enclosure of the real dot product a . b of stored FP64 vectors (every primitive rounded
// outward; reference enclosed_dot).
__device__ __forceinline__ void enclosed_dot(const double* a, const double* b, double* r)
{
    double lo = 0.0, hi = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double product = a[k] * b[k];
        lo = down(lo + down(product));
        hi = up(hi + up(product));
    }
    r[0] = lo;
    r[1] = hi;
}

// Enclosure of c . (x - o) over the box lower <= x <= upper (reference enclosed_box_dot).
__device__ __forceinline__ void enclosed_box_dot(const double* c, const double* lower, const double* upper,
                                                 const double* o, double* r)
{
    double lo = 0.0, hi = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double first = down(lower[k] - o[k]), last = up(upper[k] - o[k]);
        const double a = c[k] >= 0.0 ? first : last, b = c[k] >= 0.0 ? last : first;
        lo = down(lo + down(c[k] * a));
        hi = up(hi + up(c[k] * b));
    }
    r[0] = lo;
    r[1] = hi;
}

// Enclosure of n / d; NaNs when an input is not finite or d contains zero.
__device__ __forceinline__ void enclosed_quotient(const double* n, const double* d, double* r)
{
    r[0] = r[1] = NAN;
    if (!isfinite(n[0]) || !isfinite(n[1]) || !isfinite(d[0]) || !isfinite(d[1]) || !(d[0] > 0.0 || d[1] < 0.0))
        return;
    double lo = INFINITY, hi = -INFINITY;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const double q = n[i] / d[j];
            if (!isfinite(q)) return;
            lo = fmin(lo, down(q));
            hi = fmax(hi, up(q));
        }
    r[0] = lo;
    r[1] = hi;
}

// Rounding radius of o + t d (t in [0, 1], fused or not) on one axis.
__device__ __forceinline__ double point_radius(double o, double d)
{
    return up(1.7763568394002505e-15 * fmax(fabs(o), fabs(d)));
}

__device__ __forceinline__ void store_max(double* slot, double value)
{
    // nonnegative doubles (and +inf, NaN) order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long*>(slot), (unsigned long long)__double_as_longlong(value));
}

// Pose check (bit 1) and cone coefficients of one view (reference prepare_cone_coefficients):
// the common ray origin o
// in grid coordinates and c1 = row x d0, c2 = d0 x column, c3 = column x row, so that a grid
// point x projects to detector column (c1 . (x - o)) / (c3 . (x - o)) and row
// (c2 . (x - o)) / (c3 . (x - o)), d0 the direction of pixel 0 and column, row the grid-space
// detector steps.  Any rounding here is absorbed by the errors measured on the rays.
__global__ void k_gather_views(GatherArgs a, double* __restrict__ plan)
{
    const int view = blockIdx.x * blockDim.x + threadIdx.x;
    if (view >= a.views) return;
    double* h = plan + (int64_t)view * kGatherHeaderWords;
#pragma unroll
    for (int k = 0; k < kGatherHeaderWords; ++k) h[k] = 0.0;
    const int absolute = a.view_begin + view;
    const double* pose = a.poses + (int64_t)absolute * 12;
    if (!rigid_pose(pose)) atomicOr(a.status + absolute, 1);
    const double* w = a.view_table ? a.view_table + (int64_t)absolute * DPT_VIEW_WORDS : nullptr;
    const bool cone = a.ray_kind == DPT_RAYS_PANELS && (int)w[DPT_VIEW_MODE_WORD] == DPT_PANEL_CONE;
    h[kGatherCone] = cone ? 1.0 : 0.0;
    if (!cone) return;
    double source[3], end[3];
    RayArgs ra;
    ra.ray_kind = a.ray_kind;
    ra.cols = a.cols;
    ray_endpoints(ra, w, absolute, 0, source, end);
    Ray64 r;
    ray_setup(a.grid, pose, source, end, r);
    double column[3], row[3], object[3];
    matvec_t(pose, w + 6, object);
    matvec(a.grid.m, object, column);
    matvec_t(pose, w + 9, object);
    matvec(a.grid.m, object, row);
    const double* d = r.direction;
    double* c = h + kGatherCoefficients;
#pragma unroll
    for (int k = 0; k < 3; ++k) c[k] = r.origin[k];
    c[3] = row[1] * d[2] - row[2] * d[1];
    c[4] = row[2] * d[0] - row[0] * d[2];
    c[5] = row[0] * d[1] - row[1] * d[0];
    c[6] = d[1] * column[2] - d[2] * column[1];
    c[7] = d[2] * column[0] - d[0] * column[2];
    c[8] = d[0] * column[1] - d[1] * column[0];
    c[9] = column[1] * row[2] - column[2] * row[1];
    c[10] = column[2] * row[0] - column[0] * row[2];
    c[11] = column[0] * row[1] - column[1] * row[0];
}

// One record per ray (reference get_prepare_rays): the FP64 grid-space ray of the forward,
// its clip interval, sample step and point-rounding radii; invalid rays and non-finite sample
// points set bit 2; the per-view maxima of the point radii and, for cone views, of the
// distance between each ray's modelled detector coordinates and its own pixel.
__global__ void __launch_bounds__(256) k_gather_rays(GatherArgs a, double* __restrict__ plan)
{
    const int view = blockIdx.y;
    const int pixel = blockIdx.x * blockDim.x + threadIdx.x;
    const int rays_per_view = a.rows * a.cols;
    if (pixel >= rays_per_view) return;
    const int absolute = a.view_begin + view;
    double* h = plan + (int64_t)view * kGatherHeaderWords;
    double* rec = plan + (int64_t)a.views * kGatherHeaderWords +
                  ((int64_t)view * rays_per_view + pixel) * kGatherRayWords;
    const double* w = a.view_table ? a.view_table + (int64_t)absolute * DPT_VIEW_WORDS : nullptr;
    RayArgs ra;
    ra.ray_kind = a.ray_kind;
    ra.cols = a.cols;
    ra.rows = a.rows;
    ra.ray_sources = a.ray_sources;
    ra.ray_endpoints = a.ray_endpoints;
    double source[3], end[3];
    ray_endpoints(ra, w, absolute, pixel, source, end);
    Ray64 r;
    ray_setup(a.grid, a.poses + (int64_t)absolute * 12, source, end, r);
    int bits = valid_ray(r) ? 0 : 2;
    Interval<double> iv;
    iv.clip(r.origin, r.direction, a.grid.nx, a.grid.ny, a.grid.nz);
    const double span = fmax(iv.upper - iv.lower, 0.0);
    const double step = span / (double)a.samples;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        rec[kRayOrigin + k] = r.origin[k];
        rec[kRayDirection + k] = r.direction[k];
        const double radius = point_radius(r.origin[k], r.direction[k]);
        rec[kRayError + k] = radius;
        store_max(h + kGatherPointError + k, radius);
    }
    rec[kRayLength] = r.length;
    rec[kRayLower] = iv.lower;
    rec[kRaySpan] = span;
    rec[kRayStep] = step;
    rec[kRayUpper] = iv.upper;
    if (a.cells && bits == 0 && iv.upper - iv.lower > 0.0) {
        // every segment of the cell walk must advance and have finite Gauss nodes (reference
        // get_gather cell_gauss, projection_adjoint.py:105-146); checked once per ray here
        const int shape[3] = {a.grid.nx, a.grid.ny, a.grid.nz};
        FieldDims dims;
        dims.init(a.grid);
        CellWalk64 walk;
        walk.begin(r, iv.lower, iv.upper, shape);
        double start = iv.lower;
        const int64_t limit = (int64_t)shape[0] + shape[1] + shape[2] + 1;
        for (int64_t n = 0; start < iv.upper && n < limit; ++n) {
            GaussSegment seg;
            walk.segment(r, start, dims, seg);
            if (seg.end <= start) {
                bits |= 2;
                break;
            }
            if (!finite3(seg.first[0], seg.first[1], seg.first[2]) || !finite3(seg.second[0], seg.second[1], seg.second[2]))
                bits |= 2;
            start = seg.end;
            walk.advance(r, shape, seg.end, iv.upper);
        }
        if (start < iv.upper) bits |= 2;
    }
    // every sample point is finite when |origin| and |direction| are moderate (points are
    // o + t d with t in [0, 1]); otherwise check them all
    if (!a.cells && span > 0.0 && !moderate(r.origin, r.direction)) {
        for (int i = 0; i < a.samples; ++i) {
            const double position = fma((double)i + 0.5, step, iv.lower);
            if (!finite3(fma(position, r.direction[0], r.origin[0]), fma(position, r.direction[1], r.origin[1]),
                         fma(position, r.direction[2], r.origin[2]))) {
                bits |= 2;
                break;
            }
        }
    }
    if (h[kGatherCone] != 0.0) {
        const double* c = h + kGatherCoefficients;
        double den[2], num[2], col[2], rw[2];
        enclosed_dot(c + 9, r.direction, den);
        enclosed_dot(c + 3, r.direction, num);
        enclosed_quotient(num, den, col);
        enclosed_dot(c + 6, r.direction, num);
        enclosed_quotient(num, den, rw);
        if (!isfinite(col[0]) || !isfinite(col[1]) || !isfinite(rw[0]) || !isfinite(rw[1])) {
            store_max(h + kGatherFallback, 1.0);
        } else {
            const int rr = pixel / a.cols;
            const double column = (double)(pixel - rr * a.cols), row = (double)rr;
            store_max(h + kGatherColumnError, fmax(fabs(down(col[0] - column)), fabs(up(col[1] + (-column)))));
            store_max(h + kGatherRowError, fmax(fabs(down(rw[0] - row)), fabs(up(rw[1] + (-row)))));
        }
    }
    if (bits) atomicOr(a.status + absolute, bits);
}

// Support box of voxel (x, y, z): the grid points at which it can be a corner of the clamped
// trilinear cell (reference voxel_support), [i - 1, i + 1] per axis, widened to the half-cell
// margin at the first and last two indices (where clamping keeps a zero-weight corner in the
// cell; that term still carries the canonical overflow semantics).
__device__ __forceinline__ void voxel_support(const int* index, const int* shape, double* lower, double* upper)
{
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lower[k] = (double)(index[k] - 1);
        upper[k] = (double)(index[k] + 1);
        if (index[k] <= 1) lower[k] = -0.5;
        if (index[k] >= shape[k] - 2) upper[k] = (double)shape[k] - 0.5;
    }
}

// Detector rectangle [first_row, last_row) x [first_col, last_col) that can see the box
// (reference pixel_bounds); the whole panel for non-cone views and ill-conditioned cases.
struct Rect {
    int first_row, last_row, first_col, last_col;
    bool fallback;
};

__device__ __forceinline__ Rect pixel_bounds(const double* h, const double* lower, const double* upper, int rows,
                                             int cols)
{
    Rect r{0, rows, 0, cols, false};
    if (h[kGatherCone] == 0.0) return r;
    double lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = down(lower[k] - h[kGatherPointError + k]);
        hi[k] = up(upper[k] + h[kGatherPointError + k]);
    }
    const double* c = h + kGatherCoefficients;
    double den[2], num[2], column[2], row[2];
    enclosed_box_dot(c + 9, lo, hi, c, den);
    enclosed_box_dot(c + 3, lo, hi, c, num);
    enclosed_quotient(num, den, column);
    enclosed_box_dot(c + 6, lo, hi, c, num);
    enclosed_quotient(num, den, row);
    bool fallback = h[kGatherFallback] != 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) fallback = fallback || !isfinite(h[k]);
    fallback = fallback || !isfinite(column[0]) || !isfinite(column[1]) || !isfinite(row[0]) || !isfinite(row[1]);
    if (fallback) {
        r.fallback = true;
        return r;
    }
    column[0] = down(column[0] - h[kGatherColumnError]);
    column[1] = up(column[1] + h[kGatherColumnError]);
    row[0] = down(row[0] - h[kGatherRowError]);
    row[1] = up(row[1] + h[kGatherRowError]);
    if (column[1] < 0.0 || row[1] < 0.0 || column[0] > (double)(cols - 1) || row[0] > (double)(rows - 1)) {
        r.last_row = r.last_col = 0;
        return r;
    }
    r.first_col = (int)ceil(fmax(column[0], 0.0));
    r.last_col = (int)floor(fmin(column[1], (double)(cols - 1))) + 1;
    r.first_row = (int)ceil(fmax(row[0], 0.0));
    r.last_row = (int)floor(fmin(row[1], (double)(rows - 1))) + 1;
    return r;
}

// Sample indices [first, last) of a ray whose points can lie in the box (reference
// enclosed_support_interval / enclosed_sample_indices / sample_bounds).
__device__ __forceinline__ void sample_bounds(const double* ray, const double* lower, const double* upper,
                                              int samples, int& first, int& last)
{
    first = 0;
    last = samples;
    if (ray[kRaySpan] <= 0.0) {
        last = 0;
        return;
    }
    if (ray[kRayStep] <= 0.0) return;
    double lo = -1.776356839400251e-15, hi = 1.0 + 1.776356839400251e-15;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double o = ray[kRayOrigin + k], d = ray[kRayDirection + k];
        const double a0 = down(lower[k] - ray[kRayError + k]), b0 = up(upper[k] + ray[kRayError + k]);
        if (d == 0.0) {
            if (o < a0 || o > b0) {
                last = 0;
                return;
            }
        } else {
            double a = down(a0 - o), b = up(b0 - o);
            if (d < 0.0) {
                const double t = a;
                a = b;
                b = t;
            }
            a = down(a / d);
            b = up(b / d);
            if (!isfinite(a) || !isfinite(b)) return;  // all samples
            lo = fmax(lo, a);
            hi = fmin(hi, b);
        }
    }
    if (lo > hi) {
        last = 0;
        return;
    }
    const double radius = 1.776356839400251e-15, base = ray[kRayLower], step = ray[kRayStep];
    const double low = down(down(lo - radius) - base), high = up(up(hi + radius) - base);
    const double i0 = down(down(low / step) - 0.5), i1 = up(up(high / step) - 0.5);
    if (!isfinite(i0) || !isfinite(i1)) return;
    if (i1 < 0.0 || i0 > (double)(samples - 1)) {
        last = 0;
        return;
    }
    first = (int)ceil(fmax(i0, 0.0));
    last = (int)floor(fmin(i1, (double)(samples - 1))) + 1;
}

// a b c d without premature overflow or underflow of the partial products: the mantissas
// multiply in [2^-4, 1), the exponents add, one final scaling (reference numerics product4).
__device__ __forceinline__ double range_product(double a, double b, double c, double d)
{
    if (!isfinite(a) || !isfinite(b) || !isfinite(c) || !isfinite(d)) return a * b * c * d;
    if (a == 0.0 || b == 0.0 || c == 0.0 || d == 0.0) return 0.0;
    int ea, eb, ec, ed;
    const double ma = frexp(a, &ea), mb = frexp(b, &eb), mc = frexp(c, &ec), md = frexp(d, &ed);
    return ldexp(ma * mb * mc * md, ea + eb + ec + ed);
}

// The terms of sample point q for voxel (vx, vy, vz): corners of q's clamped cell in corner
// order 0..7 that land on the voxel, each the seed times its strict trilinear factors in axis
// order (reference point_contribution / scaled_corner_weight).
__device__ __forceinline__ double point_terms(const double* q, const int* shape, const int* voxel, double seed)
{
    if (!inside(q[0], q[1], q[2], shape[0], shape[1], shape[2])) return 0.0;
    int lower[3];
    double fraction[3];
    unsigned match[3];  // bit b of axis k: corner bit b on that axis lands on the voxel
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const Axis64 ax = axis64(q[k], (double)(shape[k] - 1), max(shape[k] - 2, 0));
        lower[k] = ax.lower;
        fraction[k] = ax.fraction;
        match[k] = (min(lower[k], shape[k] - 1) == voxel[k] ? 1u : 0u) |
                   (min(lower[k] + 1, shape[k] - 1) == voxel[k] ? 2u : 0u);
    }
    double result = 0.0;
    if (!(match[0] && match[1] && match[2])) return result;
#pragma unroll
    for (int corner = 0; corner < 8; ++corner) {
        const int bx = corner & 1, by = (corner >> 1) & 1, bz = (corner >> 2) & 1;
        if ((match[0] >> bx & 1u) && (match[1] >> by & 1u) && (match[2] >> bz & 1u)) {
            double term = seed;
            term *= bx ? fraction[0] : 1.0 - fraction[0];
            term *= by ? fraction[1] : 1.0 - fraction[1];
            term *= bz ? fraction[2] : 1.0 - fraction[2];
            result += term;
        }
    }
    return result;
}

template <typename TSeed, typename TOut>
__global__ void __launch_bounds__(kGatherThreads, DPT_GATHER_MIN_BLOCKS) k_gather(GatherArgs a, const double* __restrict__ plan,
                                                           const TSeed* __restrict__ cotangent,
                                                           TOut* __restrict__ out, int accumulate)
{
    const int64_t voxel = (int64_t)blockIdx.x * kGatherThreads + threadIdx.x;
    const int shape[3] = {a.grid.nx, a.grid.ny, a.grid.nz};
    const int64_t voxels = (int64_t)shape[0] * shape[1] * shape[2];
    if (voxel >= voxels) return;
    const int index[3] = {(int)(voxel % shape[0]), (int)((voxel / shape[0]) % shape[1]),
                          (int)(voxel / ((int64_t)shape[0] * shape[1]))};
    double lower[3], upper[3];
    voxel_support(index, shape, lower, upper);
    const int rays_per_view = a.rows * a.cols;
    const double* records = plan + (int64_t)a.views * kGatherHeaderWords;
    TOut value = accumulate ? out[voxel] : (TOut)0.0;
    bool running = accumulate != 0;  // whether `value` holds a sum yet
    for (int view = 0; view < a.views; ++view) {
        const double* h = plan + (int64_t)view * kGatherHeaderWords;
        const Rect rect = pixel_bounds(h, lower, upper, a.rows, a.cols);
        double total = 0.0;
        for (int row = rect.first_row; row < rect.last_row; ++row) {
            for (int col = rect.first_col; col < rect.last_col; ++col) {
                const int pixel = row * a.cols + col;
                const int64_t ray_index = (int64_t)view * rays_per_view + pixel;
                const double seed = (double)cotangent[ray_index];
                if (seed == 0.0) continue;
                const double* ray = records + ray_index * kGatherRayWords;
                int first, last;
                sample_bounds(ray, lower, upper, a.samples, first, last);
                if (first >= last) continue;
                const double factor = seed * ray[kRayLength];
                double scale = factor * ray[kRaySpan] / (double)a.samples;
                if (!isfinite(factor))
                    scale = range_product(seed, ray[kRayLength], ray[kRaySpan], 1.0 / (double)a.samples);
                const double o[3] = {ray[kRayOrigin], ray[kRayOrigin + 1], ray[kRayOrigin + 2]};
                const double d[3] = {ray[kRayDirection], ray[kRayDirection + 1], ray[kRayDirection + 2]};
                const double base = ray[kRayLower], step = ray[kRayStep];
                double offset = (double)first + 0.5;  // s + 1/2, exact
                for (int s = first; s < last; ++s, offset += 1.0) {
                    const double position = fma(offset, step, base);
                    const double q[3] = {fma(position, d[0], o[0]), fma(position, d[1], o[1]),
                                         fma(position, d[2], o[2])};
                    total += point_terms(q, shape, index, scale);
                }
            }
        }
        value = running ? (TOut)(total + (double)value) : (TOut)total;
        running = true;
    }
    out[voxel] = value;
    if (!isfinite((double)value)) atomicOr(a.status + a.view_begin, 2);
}

// a b c without premature overflow or underflow of the partial products (reference numerics
// product3).
__device__ __forceinline__ double range_product(double a, double b, double c)
{
    if (!isfinite(a) || !isfinite(b) || !isfinite(c)) return a * b * c;
    if (a == 0.0 || b == 0.0 || c == 0.0) return 0.0;
    int ea, eb, ec;
    const double ma = frexp(a, &ea), mb = frexp(b, &eb), mc = frexp(c, &ec);
    return ldexp(ma * mb * mc, ea + eb + ec);
}

// Both Gauss nodes of a segment whose nodes share its interpolation cell (reference
// cell_contribution): per corner of that cell landing on the voxel, first + second, a node
// outside the support weighted by zero.
__device__ __forceinline__ double cell_terms(const GaussSegment& s, const int* shape, const int* voxel, double seed)
{
    unsigned match[3];
    double f1[3], f2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        match[k] = (min(s.lower[k], shape[k] - 1) == voxel[k] ? 1u : 0u) |
                   (min(s.lower[k] + 1, shape[k] - 1) == voxel[k] ? 2u : 0u);
        const double high = (double)(shape[k] - 1);
        f1[k] = fmin(fmax(s.first[k], 0.0), high) - (double)s.lower[k];
        f2[k] = fmin(fmax(s.second[k], 0.0), high) - (double)s.lower[k];
    }
    double result = 0.0;
    if (!(match[0] && match[1] && match[2])) return result;
    const double a = inside(s.first[0], s.first[1], s.first[2], shape[0], shape[1], shape[2]) ? seed : 0.0;
    const double b = inside(s.second[0], s.second[1], s.second[2], shape[0], shape[1], shape[2]) ? seed : 0.0;
#pragma unroll
    for (int corner = 0; corner < 8; ++corner) {
        const int bx = corner & 1, by = (corner >> 1) & 1, bz = (corner >> 2) & 1;
        if ((match[0] >> bx & 1u) && (match[1] >> by & 1u) && (match[2] >> bz & 1u)) {
            double first = a, second = b;
            first *= bx ? f1[0] : 1.0 - f1[0];
            first *= by ? f1[1] : 1.0 - f1[1];
            first *= bz ? f1[2] : 1.0 - f1[2];
            second *= bx ? f2[0] : 1.0 - f2[0];
            second *= by ? f2[1] : 1.0 - f2[1];
            second *= bz ? f2[2] : 1.0 - f2[2];
            result += first + second;
        }
    }
    return result;
}

// The same fixed-order gather for cell-Gauss integration (reference get_gather with
// cell_gauss, projection_adjoint.py:105-146): each candidate ray's cell walk from its entry,
// two Gauss nodes per segment weighted by cotangent |e - s| radius.  The walk of every ray
// was validated when the plan was written.
template <typename TSeed, typename TOut>
__global__ void __launch_bounds__(kGatherThreads) k_gather_cells(GatherArgs a, const double* __restrict__ plan,
                                                                 const TSeed* __restrict__ cotangent,
                                                                 TOut* __restrict__ out, int accumulate)
{
    const int64_t voxel = (int64_t)blockIdx.x * kGatherThreads + threadIdx.x;
    const int shape[3] = {a.grid.nx, a.grid.ny, a.grid.nz};
    const int64_t voxels = (int64_t)shape[0] * shape[1] * shape[2];
    if (voxel >= voxels) return;
    const int index[3] = {(int)(voxel % shape[0]), (int)((voxel / shape[0]) % shape[1]),
                          (int)(voxel / ((int64_t)shape[0] * shape[1]))};
    double lower[3], upper[3];
    voxel_support(index, shape, lower, upper);
    FieldDims dims;
    dims.init(a.grid);
    const int rays_per_view = a.rows * a.cols;
    const double* records = plan + (int64_t)a.views * kGatherHeaderWords;
    const int64_t limit = (int64_t)shape[0] + shape[1] + shape[2] + 1;
    TOut value = accumulate ? out[voxel] : (TOut)0.0;
    bool running = accumulate != 0;
    for (int view = 0; view < a.views; ++view) {
        const Rect rect = pixel_bounds(plan + (int64_t)view * kGatherHeaderWords, lower, upper, a.rows, a.cols);
        double total = 0.0;
        for (int row = rect.first_row; row < rect.last_row; ++row) {
            for (int col = rect.first_col; col < rect.last_col; ++col) {
                const int64_t ray_index = (int64_t)view * rays_per_view + row * a.cols + col;
                const double seed = (double)cotangent[ray_index];
                if (seed == 0.0) continue;
                const double* rec = records + ray_index * kGatherRayWords;
                const double lo = rec[kRayLower], hi = rec[kRayUpper];
                if (hi - lo <= 0.0) continue;
                Ray64 r;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    r.origin[k] = rec[kRayOrigin + k];
                    r.direction[k] = rec[kRayDirection + k];
                }
                const double factor = seed * rec[kRayLength];
                CellWalk64 walk;
                walk.begin(r, lo, hi, shape);
                double start = lo;
                for (int64_t n = 0; start < hi && n < limit; ++n) {
                    GaussSegment s;
                    walk.segment(r, start, dims, s);
                    if (s.end <= start) break;
                    double vf = factor * s.radius;
                    if (!isfinite(factor)) vf = range_product(seed, rec[kRayLength], s.radius);
                    if (s.shared) {
                        total += cell_terms(s, shape, index, vf);
                    } else {
                        total += point_terms(s.first, shape, index, vf);
                        total += point_terms(s.second, shape, index, vf);
                    }
                    start = s.end;
                    walk.advance(r, shape, s.end, hi);
                }
            }
        }
        value = running ? (TOut)(total + (double)value) : (TOut)total;
        running = true;
    }
    out[voxel] = value;
    if (!isfinite((double)value)) atomicOr(a.status + a.view_begin, 2);
}

// Per-voxel work of a plan (reference get_count_gather_work): candidate rays, sample nodes,
// voxels whose candidate rectangle exceeds `max_rays` in some view, and fallback voxels.
__global__ void __launch_bounds__(kGatherThreads) k_gather_count(GatherArgs a, const double* __restrict__ plan,
                                                                 int max_rays, unsigned long long* totals)
{
    const int64_t voxel = (int64_t)blockIdx.x * kGatherThreads + threadIdx.x;
    const int shape[3] = {a.grid.nx, a.grid.ny, a.grid.nz};
    const int64_t voxels = (int64_t)shape[0] * shape[1] * shape[2];
    unsigned long long rays = 0, nodes = 0, limited = 0, fallbacks = 0;
    if (voxel < voxels) {
        const int index[3] = {(int)(voxel % shape[0]), (int)((voxel / shape[0]) % shape[1]),
                              (int)(voxel / ((int64_t)shape[0] * shape[1]))};
        double lower[3], upper[3];
        voxel_support(index, shape, lower, upper);
        const int rays_per_view = a.rows * a.cols;
        const double* records = plan + (int64_t)a.views * kGatherHeaderWords;
        bool over = false, fell = false;
        for (int view = 0; view < a.views; ++view) {
            const Rect rect = pixel_bounds(plan + (int64_t)view * kGatherHeaderWords, lower, upper, a.rows, a.cols);
            const int64_t count =
                (int64_t)max(rect.last_row - rect.first_row, 0) * max(rect.last_col - rect.first_col, 0);
            fell = fell || rect.fallback;
            if (count > max_rays) {
                over = true;
                continue;
            }
            rays += (unsigned long long)count;
            for (int row = rect.first_row; row < rect.last_row; ++row)
                for (int col = rect.first_col; col < rect.last_col; ++col) {
                    int first, last;
                    sample_bounds(records + ((int64_t)view * rays_per_view + row * a.cols + col) * kGatherRayWords,
                                  lower, upper, a.samples, first, last);
                    nodes += (unsigned long long)max(last - first, 0);
                }
        }
        limited = over ? 1 : 0;
        fallbacks = fell ? 1 : 0;
    }
    // warp totals, then one atomic per warp and counter (integer sums: order-free)
    for (int offset = 16; offset > 0; offset >>= 1) {
        rays += __shfl_down_sync(0xffffffffu, rays, offset);
        nodes += __shfl_down_sync(0xffffffffu, nodes, offset);
        limited += __shfl_down_sync(0xffffffffu, limited, offset);
        fallbacks += __shfl_down_sync(0xffffffffu, fallbacks, offset);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(totals + 0, rays);
        atomicAdd(totals + 1, nodes);
        atomicAdd(totals + 2, limited);
        atomicAdd(totals + 3, fallbacks);
    }
}

}  // namespace

cudaError_t launch_gather_prepare(const GatherArgs& a, double* plan, cudaStream_t stream)
{
    k_gather_views<<<(a.views + 127) / 128, 128, 0, stream>>>(a, plan);
    const dim3 grid((unsigned)((a.rows * a.cols + 255) / 256), (unsigned)a.views);
    k_gather_rays<<<grid, 256, 0, stream>>>(a, plan);
    return cudaGetLastError();
}

cudaError_t launch_gather_count(const GatherArgs& a, const double* plan, int max_rays, unsigned long long* totals,
                                cudaStream_t stream)
{
    const int64_t voxels = (int64_t)a.grid.nx * a.grid.ny * a.grid.nz;
    cudaMemsetAsync(totals, 0, 4 * sizeof(unsigned long long), stream);
    k_gather_count<<<(unsigned)((voxels + kGatherThreads - 1) / kGatherThreads), kGatherThreads, 0, stream>>>(
        a, plan, max_rays, totals);
    return cudaGetLastError();
}

cudaError_t launch_gather(const GatherArgs& a, const double* plan, const void* cotangent, int seed_dtype,
                          void* out, int out_dtype, int accumulate, cudaStream_t stream)
{
    const int64_t voxels = (int64_t)a.grid.nx * a.grid.ny * a.grid.nz;
    const unsigned blocks = (unsigned)((voxels + kGatherThreads - 1) / kGatherThreads);
    auto run = [&](auto seed_type, auto out_type) {
        using TS = decltype(seed_type);
        using TO = decltype(out_type);
        if (a.cells)
            k_gather_cells<TS, TO><<<blocks, kGatherThreads, 0, stream>>>(
                a, plan, static_cast<const TS*>(cotangent), static_cast<TO*>(out), accumulate);
        else
            k_gather<TS, TO><<<blocks, kGatherThreads, 0, stream>>>(
                a, plan, static_cast<const TS*>(cotangent), static_cast<TO*>(out), accumulate);
    };
    if (seed_dtype == DPT_F64 && out_dtype == DPT_F64)
        run(double{}, double{});
    else if (seed_dtype == DPT_F64)
        run(double{}, float{});
    else if (out_dtype == DPT_F64)
        run(float{}, double{});
    else
        run(float{}, float{});
    return cudaGetLastError();
}

}  // namespace dpt
