/*
 * projector_oracle.c - CPU ORACLE for the projector.  TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, scalar and unoptimised, the arithmetic of the reference
 * projector (hcltech-robotics/dpt) so that the CUDA kernels can be checked
 * against it.  It is called only by tests/, by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline arm; the product never links or calls it.
 *
 * Reference files restated (paths inside the reference project):
 *   python/dpt/kernels/projection.py       ray_for_pixel 79-102, valid_ray 110-121,
 *                                          inside_support 124-134, finite_interval 147-184,
 *                                          cell_lower/cell_fraction/corner_index 199-222,
 *                                          sample_cell_fraction 236-274, midpoint forward
 *                                          770-846, strict VJP 873-1237
 *   python/dpt/kernels/projection_fp32.py  FP32 clip 78-109, sample_position/point 116-127,
 *                                          coordinates 130-140, sample_field 157-177,
 *                                          sample_pose_field 180-209, scatter_increment
 *                                          240-258, cell-run aggregation 261-331 and
 *                                          459-548, forward 334-374, VJP 377-617
 *   python/dpt/kernels/geometry.py         unpack 13-21, local-right adjoint 24-52,
 *                                          rigid-pose check 55-74
 *   python/dpt/kernels/batched_geometry.py generate 8-39 (parallel / curved panels)
 *   python/dpt/kernels/projection_checks.py field/finite scans 20-28
 *
 * Floating-point contract.  Compile with -ffp-contract=off: every fused
 * multiply-add below is an explicit fma()/fmaf(), every other operation is a
 * single IEEE-rounded operation.  Where the reference writes a*b + c*d (which
 * its JIT may contract) this restatement uses fma(c, d, a*b); where it writes
 * a + b*c it uses fma(b, c, a).  The CUDA kernels follow the same contract, so
 * forward images, clip intervals and sample counts agree bit for bit.
 *
 * The DPT_ARITH_F32C form (FP64 clip, FP32 marching, trilinear-polynomial samples,
 * blocked compensated sum, moment-based scatter) has no reference counterpart: it is
 * the projector library's storage-precision form, restated here from its own definition
 * and checked in the tests against F64.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/dpt_b200.h"

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ storage */

static float half_to_float(uint16_t h)
{
    uint32_t sign = (uint32_t)(h >> 15) << 31;
    uint32_t exponent = (h >> 10) & 0x1f;
    uint32_t mantissa = h & 0x3ff;
    uint32_t bits;
    if (exponent == 0) {
        if (mantissa == 0) {
            bits = sign;
        } else {
            /* subnormal half: value = mantissa * 2^-24, exact in float */
            float value = (float)mantissa * 5.9604644775390625e-08f;
            memcpy(&bits, &value, 4);
            bits |= sign;
        }
    } else if (exponent == 31) {
        bits = sign | 0x7f800000u | (mantissa << 13);
    } else {
        bits = sign | ((exponent + 112) << 23) | (mantissa << 13);
    }
    float out;
    memcpy(&out, &bits, 4);
    return out;
}

static float bf16_to_float(uint16_t b)
{
    uint32_t bits = (uint32_t)b << 16;
    float out;
    memcpy(&out, &bits, 4);
    return out;
}

static float field_value(const dpt_problem* p, const void* field, int64_t index)
{
    switch (p->field_dtype) {
    case DPT_F16:
        return half_to_float(((const uint16_t*)field)[index]);
    case DPT_BF16:
        return bf16_to_float(((const uint16_t*)field)[index]);
    default:
        return ((const float*)field)[index];
    }
}

/* --------------------------------------------------------------- ray setup */

typedef struct {
    double origin[3], direction[3];           /* grid-index coordinates */
    double object_source[3], object_direction[3];
    double world_source_relative[3], world_direction[3];
    double length;
} ray64_t;

/* r = A v for a row-major 3x3 A, accumulated as fma(a2,v2, fma(a1,v1, a0*v0)). */
static void matvec(const double* a, const double* v, double* r)
{
    for (int i = 0; i < 3; ++i)
        r[i] = fma(a[3 * i + 2], v[2], fma(a[3 * i + 1], v[1], a[3 * i] * v[0]));
}

/* r = A^T v. */
static void matvec_t(const double* a, const double* v, double* r)
{
    for (int i = 0; i < 3; ++i)
        r[i] = fma(a[6 + i], v[2], fma(a[3 + i], v[1], a[i] * v[0]));
}

/* Source and endpoint of ray `pixel` (index inside its view).  Cone panels follow
 * kernels/projection.py:88-93 (end = d0 + c*(u du) + r*(v dv)); parallel and
 * curved panels follow kernels/batched_geometry.py:17-38. */
static void ray_endpoints(const dpt_problem* p, const double* view_table, const double* sources,
                          const double* endpoints, int view, int64_t pixel, double* source,
                          double* end)
{
    if (p->ray_kind == DPT_RAYS_BUNDLE) {
        int64_t ray = (int64_t)view * p->rows * p->cols + pixel;
        for (int a = 0; a < 3; ++a) {
            source[a] = sources[3 * ray + a];
            end[a] = endpoints[3 * ray + a];
        }
        return;
    }
    const double* w = view_table + (int64_t)view * DPT_VIEW_WORDS;
    double row = (double)(pixel / p->cols), column = (double)(pixel % p->cols);
    int mode = (int)w[DPT_VIEW_MODE_WORD];
    if (mode == DPT_PANEL_CONE) {
        for (int a = 0; a < 3; ++a) {
            source[a] = w[a];
            end[a] = fma(row, w[9 + a], fma(column, w[6 + a], w[3 + a]));
        }
        return;
    }
    double du = w[12], dv = w[13], length = w[14];
    if (mode == DPT_PANEL_PARALLEL) {
        double cu = column * du, rv = row * dv;
        for (int a = 0; a < 3; ++a) {
            end[a] = fma(rv, w[9 + a], fma(cu, w[6 + a], w[3 + a]));
            source[a] = end[a] - length * w[a];
        }
        return;
    }
    /* curved: angle = c*du/R; end = o + (cos-1) radial + sin R u + r dv v */
    double angle = column * du / length;
    double c1 = cos(angle) - 1.0, s = sin(angle) * length, rv = row * dv;
    for (int a = 0; a < 3; ++a) {
        source[a] = w[a];
        end[a] = fma(rv, w[9 + a], fma(s, w[6 + a], fma(c1, w[15 + a], w[3 + a])));
    }
}

/* kernels/projection.py:79-102 */
static void ray_setup(const dpt_problem* p, const double* pose, const double* source,
                      const double* end, ray64_t* r)
{
    double rel[3];
    for (int a = 0; a < 3; ++a) {
        r->world_source_relative[a] = source[a] - pose[9 + a];
        r->world_direction[a] = end[a] - source[a];
    }
    matvec_t(pose, r->world_source_relative, r->object_source);
    matvec_t(pose, r->world_direction, r->object_direction);
    for (int a = 0; a < 3; ++a)
        rel[a] = r->object_source[a] - p->grid_origin[a];
    matvec(p->object_to_grid, rel, r->origin);
    matvec(p->object_to_grid, r->object_direction, r->direction);
    const double* d = r->world_direction;
    r->length = sqrt(fma(d[2], d[2], fma(d[1], d[1], d[0] * d[0])));
}

static int finite3(const double* v) { return isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]); }
static int finite3f(const float* v) { return isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]); }

/* kernels/projection.py:110-121 */
static int valid_ray(const ray64_t* r)
{
    return finite3(r->origin) && finite3(r->direction) && finite3(r->object_source) &&
           finite3(r->object_direction) && finite3(r->world_source_relative) &&
           finite3(r->world_direction) && isfinite(r->length) && r->length > 0.0;
}

/* ----------------------------------------------------------------- clipping */

typedef struct {
    float lower, upper;
    float lower_origin[3], lower_direction[3], upper_origin[3], upper_direction[3];
} interval32_t;

typedef struct {
    double lower, upper;
    double lower_origin[3], lower_direction[3], upper_origin[3], upper_direction[3];
} interval64_t;

/* kernels/projection_fp32.py:78-109 */
static void clip32(const float* origin, const float* direction, const int* shape,
                   interval32_t* iv)
{
    memset(iv, 0, sizeof(*iv));
    iv->lower = 0.0f;
    iv->upper = 1.0f;
    for (int a = 0; a < 3; ++a) {
        float low = -0.5f, high = (float)shape[a] - 0.5f, velocity = direction[a];
        if (velocity == 0.0f) {
            if (origin[a] < low || origin[a] > high)
                iv->upper = -1.0f;
        } else {
            float first = (low - origin[a]) / velocity;
            float last = (high - origin[a]) / velocity;
            if (first > last) {
                float t = first;
                first = last;
                last = t;
            }
            if (first > iv->lower) {
                iv->lower = first;
                memset(iv->lower_origin, 0, sizeof(iv->lower_origin));
                memset(iv->lower_direction, 0, sizeof(iv->lower_direction));
                iv->lower_origin[a] = -1.0f / velocity;
                iv->lower_direction[a] = -first / velocity;
            }
            if (last < iv->upper) {
                iv->upper = last;
                memset(iv->upper_origin, 0, sizeof(iv->upper_origin));
                memset(iv->upper_direction, 0, sizeof(iv->upper_direction));
                iv->upper_origin[a] = -1.0f / velocity;
                iv->upper_direction[a] = -last / velocity;
            }
        }
    }
}

/* kernels/projection.py:147-184 */
static void clip64(const double* origin, const double* direction, const int* shape,
                   interval64_t* iv)
{
    memset(iv, 0, sizeof(*iv));
    iv->lower = 0.0;
    iv->upper = 1.0;
    for (int a = 0; a < 3; ++a) {
        double low = -0.5, high = (double)shape[a] - 0.5, velocity = direction[a];
        if (velocity == 0.0) {
            if (origin[a] < low || origin[a] > high)
                iv->upper = -1.0;
        } else {
            double first = (low - origin[a]) / velocity;
            double last = (high - origin[a]) / velocity;
            if (first > last) {
                double t = first;
                first = last;
                last = t;
            }
            if (first > iv->lower) {
                iv->lower = first;
                memset(iv->lower_origin, 0, sizeof(iv->lower_origin));
                memset(iv->lower_direction, 0, sizeof(iv->lower_direction));
                iv->lower_origin[a] = -1.0 / velocity;
                iv->lower_direction[a] = -first / velocity;
            }
            if (last < iv->upper) {
                iv->upper = last;
                memset(iv->upper_origin, 0, sizeof(iv->upper_origin));
                memset(iv->upper_direction, 0, sizeof(iv->upper_direction));
                iv->upper_origin[a] = -1.0 / velocity;
                iv->upper_direction[a] = -last / velocity;
            }
        }
    }
}

/* ------------------------------------------------------------ interpolation */

static int inside32(const float* q, const int* shape)
{
    return finite3f(q) && q[0] >= -0.5f && q[1] >= -0.5f && q[2] >= -0.5f &&
           q[0] <= (float)shape[0] - 0.5f && q[1] <= (float)shape[1] - 0.5f &&
           q[2] <= (float)shape[2] - 0.5f;
}

static int inside64(const double* q, const int* shape)
{
    return finite3(q) && q[0] >= -0.5 && q[1] >= -0.5 && q[2] >= -0.5 &&
           q[0] <= (double)shape[0] - 0.5 && q[1] <= (double)shape[1] - 0.5 &&
           q[2] <= (double)shape[2] - 0.5;
}

static int64_t corner_index(const int* lower, const int* shape, int corner)
{
    int x = lower[0] + (corner & 1), y = lower[1] + ((corner >> 1) & 1),
        z = lower[2] + ((corner >> 2) & 1);
    if (x > shape[0] - 1) x = shape[0] - 1;
    if (y > shape[1] - 1) y = shape[1] - 1;
    if (z > shape[2] - 1) z = shape[2] - 1;
    return ((int64_t)z * shape[1] + y) * shape[0] + x;
}

static int cell_floor(double value, int n)
{
    int lower = (int)floor(value), cap = n - 2 > 0 ? n - 2 : 0;
    return lower < cap ? lower : cap;
}

/* kernels/projection_fp32.py:130-140: lower cell, fraction and in-range slope mask. */
static void coordinates32(const float* q, const int* shape, int* lower, float* fraction,
                          float* slope)
{
    for (int a = 0; a < 3; ++a) {
        float high = (float)(shape[a] - 1);
        float value = q[a] < 0.0f ? 0.0f : (q[a] > high ? high : q[a]);
        lower[a] = cell_floor((double)value, shape[a]);
        fraction[a] = value - (float)lower[a];
        slope[a] = (q[a] >= 0.0f && q[a] < high) ? 1.0f : 0.0f;
    }
}

/* kernels/projection.py:199-214 */
static void coordinates64(const double* q, const int* shape, int* lower, double* fraction,
                          double* slope)
{
    for (int a = 0; a < 3; ++a) {
        double high = (double)(shape[a] - 1);
        double value = q[a] < 0.0 ? 0.0 : (q[a] > high ? high : q[a]);
        lower[a] = cell_floor(value, shape[a]);
        fraction[a] = value - (double)lower[a];
        slope[a] = (q[a] >= 0.0 && q[a] < high) ? 1.0 : 0.0;
    }
}

/* (f0 f1) f2 with f = 1 - fraction for a 0 bit, kernels/projection_fp32.py:143-154 */
static float corner_weight32(const float* fraction, int corner)
{
    float f[3];
    for (int a = 0; a < 3; ++a)
        f[a] = ((corner >> a) & 1) ? fraction[a] : 1.0f - fraction[a];
    return (f[0] * f[1]) * f[2];
}

/* MIXED / FAST sample of one FP32 point (kernels/projection.py:326-352): zero outside the
 * support; else the FP32 clamped coordinates and corner weights, and the corner sum in FP64
 * (MIXED, fma(w, v, value)) or FP32 (FAST, fmaf(w, v, value)) from zero. */
static double sample_mixed32(const dpt_problem* p, const void* field, const float* q, const int* shape)
{
    if (!inside32(q, shape)) return 0.0;
    int lower[3];
    float f[3], slope[3];
    coordinates32(q, shape, lower, f, slope);
    if (p->arith == DPT_ARITH_FAST) {
        float value = 0.0f;
        for (int c = 0; c < 8; ++c)
            value = fmaf(corner_weight32(f, c), field_value(p, field, corner_index(lower, shape, c)), value);
        return (double)value;
    }
    double value = 0.0;
    for (int c = 0; c < 8; ++c)
        value = fma((double)corner_weight32(f, c), (double)field_value(p, field, corner_index(lower, shape, c)),
                    value);
    return value;
}

/* sample_pose_field, kernels/projection_fp32.py:180-209 (value and grid slope). */
static float sample32(const dpt_problem* p, const void* field, const float* q, const int* shape,
                      float* gradient)
{
    if (gradient) gradient[0] = gradient[1] = gradient[2] = 0.0f;
    if (!inside32(q, shape)) return 0.0f;
    int lower[3];
    float fraction[3], slope[3], v[8];
    coordinates32(q, shape, lower, fraction, slope);
    float value = 0.0f;
    for (int c = 0; c < 8; ++c) {
        v[c] = field_value(p, field, corner_index(lower, shape, c));
        value = fmaf(corner_weight32(fraction, c), v[c], value);
    }
    if (gradient) {
        float fx = fraction[0], fy = fraction[1], fz = fraction[2];
        float ax = 1.0f - fx, ay = 1.0f - fy, az = 1.0f - fz;
        float x0 = fmaf(fy, v[3] - v[2], ay * (v[1] - v[0]));
        float x1 = fmaf(fy, v[7] - v[6], ay * (v[5] - v[4]));
        gradient[0] = slope[0] * fmaf(fz, x1, az * x0);
        float y0 = fmaf(fx, v[3] - v[1], ax * (v[2] - v[0]));
        float y1 = fmaf(fx, v[7] - v[5], ax * (v[6] - v[4]));
        gradient[1] = slope[1] * fmaf(fz, y1, az * y0);
        float z0 = fmaf(fx, v[5] - v[1], ax * (v[4] - v[0]));
        float z1 = fmaf(fx, v[7] - v[3], ax * (v[6] - v[2]));
        gradient[2] = slope[2] * fmaf(fy, z1, ay * z0);
    }
    return value;
}

/* sample_cell_fraction, kernels/projection.py:236-274 (weighted lerps in FP64). */
static double sample64(const dpt_problem* p, const void* field, const double* q,
                       const int* shape, double* gradient)
{
    if (gradient) gradient[0] = gradient[1] = gradient[2] = 0.0;
    if (!inside64(q, shape)) return 0.0;
    int lower[3];
    double f[3], slope[3], v[8];
    coordinates64(q, shape, lower, f, slope);
    for (int c = 0; c < 8; ++c)
        v[c] = (double)field_value(p, field, corner_index(lower, shape, c));
    double fx = f[0], fy = f[1], fz = f[2], ax = 1.0 - fx, ay = 1.0 - fy, az = 1.0 - fz;
    double x00 = fma(fx, v[1], ax * v[0]), x10 = fma(fx, v[3], ax * v[2]);
    double x01 = fma(fx, v[5], ax * v[4]), x11 = fma(fx, v[7], ax * v[6]);
    double xy0 = fma(fy, x10, ay * x00), xy1 = fma(fy, x11, ay * x01);
    double value = fma(fz, xy1, az * xy0);
    if (gradient) {
        double dx00 = v[1] - v[0], dx10 = v[3] - v[2], dx01 = v[5] - v[4], dx11 = v[7] - v[6];
        double dx0 = fma(fy, dx10, ay * dx00), dx1 = fma(fy, dx11, ay * dx01);
        double dy0 = fma(fx, v[3] - v[1], ax * (v[2] - v[0]));
        double dy1 = fma(fx, v[7] - v[5], ax * (v[6] - v[4]));
        double dz0 = fma(fx, v[5] - v[1], ax * (v[4] - v[0]));
        double dz1 = fma(fx, v[7] - v[3], ax * (v[6] - v[2]));
        gradient[0] = slope[0] * fma(fz, dx1, az * dx0);
        gradient[1] = slope[1] * fma(fz, dy1, az * dy0);
        gradient[2] = slope[2] * fma(fy, dz1, ay * dz0);
    }
    return value;
}

/* F32C sample: value and grid slope from the trilinear polynomial of the cell,
 * f = c0 + c1 x + c2 y + c3 z + c4 xy + c5 xz + c6 yz + c7 xyz, coefficients formed in FP32
 * from the eight corners in the order below and evaluated with fmaf. */
static float sample32c(const dpt_problem* p, const void* field, const float* q, const int* shape,
                       float* gradient, float* fraction_out)
{
    if (gradient) gradient[0] = gradient[1] = gradient[2] = 0.0f;
    if (!inside32(q, shape)) return 0.0f;
    int lower[3];
    float f[3], slope[3], v[8];
    coordinates32(q, shape, lower, f, slope);
    if (fraction_out) memcpy(fraction_out, f, sizeof(f));
    for (int c = 0; c < 8; ++c) v[c] = field_value(p, field, corner_index(lower, shape, c));
    const float c0 = v[0], c1 = v[1] - v[0], c2 = v[2] - v[0], c3 = v[4] - v[0];
    const float c4 = (v[3] - v[2]) - c1, c5 = (v[5] - v[4]) - c1, c6 = (v[6] - v[4]) - c2;
    const float c7 = ((v[7] - v[6]) - (v[5] - v[4])) - c4;
    const float fx = f[0], fy = f[1], fz = f[2];
    const float a = fmaf(c7, fz, c4), b = fmaf(c5, fz, c1);
    const float gx = fmaf(a, fy, b);
    const float e = fmaf(c6, fz, c2), h = fmaf(c3, fz, c0);
    const float value = fmaf(gx, fx, fmaf(e, fy, h));
    if (gradient) {
        gradient[0] = slope[0] * gx;
        gradient[1] = slope[1] * fmaf(a, fx, e);
        gradient[2] = slope[2] * fmaf(fx, fmaf(c7, fy, c5), fmaf(c6, fy, c3));
    }
    return value;
}

/* Compensated sum of 16-sample blocks: each block summed serially in FP32, the block sums
 * added with Kahan compensation. */
typedef struct {
    float block, sum, carry;
} blocksum_t;

static void blocksum_add(blocksum_t* s, float value, int index, int samples)
{
    s->block += value;
    if ((index & 15) == 15 || index == samples - 1) {
        float y = s->block - s->carry;
        float t = s->sum + y;
        s->carry = (t - s->sum) - y;
        s->sum = t;
        s->block = 0.0f;
    }
}

/* ------------------------------------------------------------ ray geometry */

typedef struct {
    /* common per-ray quantities, FP64 setup plus the arithmetic's own clip */
    ray64_t r;
    int valid;
    /* F32 */
    float o32[3], d32[3], len32;
    interval32_t iv32;
    /* F64 and F32C */
    interval64_t iv64;
} ray_t;

static int ray_prepare(const dpt_problem* p, const double* pose, const double* source,
                       const double* end, ray_t* ray)
{
    int shape[3] = {p->nx, p->ny, p->nz};
    ray_setup(p, pose, source, end, &ray->r);
    ray->valid = valid_ray(&ray->r);
    if (p->arith == DPT_ARITH_F32) {
        for (int a = 0; a < 3; ++a) {
            ray->o32[a] = (float)ray->r.origin[a];
            ray->d32[a] = (float)ray->r.direction[a];
        }
        ray->len32 = (float)ray->r.length;
        ray->valid = ray->valid && finite3f(ray->o32) && finite3f(ray->d32) &&
                     isfinite(ray->len32) && ray->len32 > 0.0f;
        if (ray->valid) clip32(ray->o32, ray->d32, shape, &ray->iv32);
    } else if (ray->valid) {
        clip64(ray->r.origin, ray->r.direction, shape, &ray->iv64);
    }
    return ray->valid;
}

/* F32C marching: entry = o + lower d and per-sample step vector, both rounded once to FP32
 * (the mixed-midpoint recurrence of kernels/projection.py:368-392). */
static void march32c(const ray_t* ray, int samples, float* entry, float* step_vector)
{
    double span = ray->iv64.upper - ray->iv64.lower, step = span / (double)samples;
    for (int a = 0; a < 3; ++a) {
        entry[a] = (float)fma(ray->iv64.lower, ray->r.direction[a], ray->r.origin[a]);
        step_vector[a] = (float)(step * ray->r.direction[a]);
    }
}

static void point32c(const float* entry, const float* step_vector, int index, float* q)
{
    float offset = (float)index + 0.5f;
    for (int a = 0; a < 3; ++a)
        q[a] = fmaf(offset, step_vector[a], entry[a]);
}

/* ------------------------------------------------- F32C segment form (moderate rays)
 * The samples inside the support, [first, last], are grouped into runs of consecutive
 * samples in one interpolation cell by walking the cell planes along the ray.  Along the
 * run the fractions are f + j d (j = 0..n-1, d the per-sample step; d = 0 on an axis in its
 * half-cell margin, where the fraction is clamped), so the run's sum of the cell polynomial,
 * its slope sums and the volume moments are polynomials in j of degree <= 3, evaluated in
 * closed form with the power sums S1 = sum j, S2 = sum j^2, S3 = sum j^3.  Rays whose grid
 * origin or direction reach 1e30, or whose samples lie more than one cell plane apart on
 * average, take the per-sample form instead. */

static int moderate32c(const float* entry, const float* step_vector)
{
    float m = 0.0f;
    for (int a = 0; a < 3; ++a) {
        m = fmaxf(m, fabsf(entry[a]));
        m = fmaxf(m, fabsf(step_vector[a]));
    }
    return m < 1e30f;
}

/* Segment form while the samples lie at most one cell plane apart on average,
 * (|s_x| + |s_y|) + |s_z| <= 1 (this library's rule; sparser samples take the per-sample
 * form, whose sums round differently). */
static int segment_form32c(const float* entry, const float* step_vector)
{
    const float planes = (fabsf(step_vector[0]) + fabsf(step_vector[1])) + fabsf(step_vector[2]);
    return moderate32c(entry, step_vector) && planes <= 1.0f;
}

/* First and last samples inside the support (first > last when none): the points are
 * monotone in the sample index on every axis, so the inside samples form one run. */
static void inside_run32c(const float* entry, const float* step_vector, const int* shape, int S,
                          int* first, int* last)
{
    float q[3];
    int f = 0, l = S - 1;
    for (; f <= l; ++f) {
        point32c(entry, step_vector, f, q);
        if (inside32(q, shape)) break;
    }
    for (; l > f; --l) {
        point32c(entry, step_vector, l, q);
        if (inside32(q, shape)) break;
    }
    *first = f;
    *last = l;
}

typedef struct {
    int i0, n;        /* first sample of the run and its sample count */
    int cell[3];      /* interpolation cell (lower corner, clamped to the grid) */
    int interior[3];  /* 1 where the axis lies inside its cell range (slope active) */
    float f[3], d[3]; /* fractions at sample i0 and their per-sample change */
    float nf, s1, s2, s3;
} run32c_t;

/* sample-index coordinate u (sample i at u = i + 0.5) where the ray meets the next cell
 * plane on axis k, or +inf when none is left inside the support */
static float crossing32c(const float* entry, const float* inverse, const float* step_vector,
                         const int* plane_cell, const int* shape, int k)
{
    if (step_vector[k] > 0.0f && plane_cell[k] + 1 <= shape[k] - 1)
        return ((float)(plane_cell[k] + 1) - entry[k]) * inverse[k];
    if (step_vector[k] < 0.0f && plane_cell[k] >= 0)
        return ((float)plane_cell[k] - entry[k]) * inverse[k];
    return INFINITY;
}

static void make_run32c(const float* entry, const float* step_vector, const int* shape,
                        const int* axis_cell, int i0, int n, run32c_t* r)
{
    float q[3];
    point32c(entry, step_vector, i0, q);
    r->i0 = i0;
    r->n = n;
    for (int k = 0; k < 3; ++k) {
        const int top = shape[k] - 2 < 0 ? 0 : shape[k] - 2;
        if (axis_cell[k] >= 0 && axis_cell[k] <= shape[k] - 2) {
            r->cell[k] = axis_cell[k];
            r->f[k] = q[k] - (float)axis_cell[k];
            r->d[k] = step_vector[k];
            r->interior[k] = 1;
        } else {
            r->cell[k] = axis_cell[k] < 0 ? 0 : top;
            r->f[k] = (axis_cell[k] < 0 || shape[k] == 1) ? 0.0f : 1.0f;
            r->d[k] = 0.0f;
            r->interior[k] = 0;
        }
    }
    const int64_t m = n;
    r->nf = (float)m;
    r->s1 = (float)(m * (m - 1) / 2);
    r->s2 = (float)(m * (m - 1) * (2 * m - 1) / 6);
    r->s3 = r->s1 * r->s1;
}

typedef void (*run_action32c)(void* context, const run32c_t* run);

/* Walk the cell planes from sample `first` to `last`, calling `action` on every run with at
 * least one sample.  Each step advances every axis whose plane is the nearest, so the walk
 * ends after at most nx + ny + nz + 3 steps. */
static void traverse32c(const float* entry, const float* step_vector, const int* shape, int first,
                        int last, run_action32c action, void* context)
{
    float q[3], inverse[3], next[3];
    int axis_cell[3];
    point32c(entry, step_vector, first, q);
    for (int k = 0; k < 3; ++k) {
        int c = (int)floorf(q[k]);
        axis_cell[k] = c < -1 ? -1 : (c > shape[k] - 1 ? shape[k] - 1 : c);
        inverse[k] = step_vector[k] != 0.0f ? 1.0f / step_vector[k] : 0.0f;
    }
    for (int k = 0; k < 3; ++k) next[k] = crossing32c(entry, inverse, step_vector, axis_cell, shape, k);
    int i = first;
    const int limit = shape[0] + shape[1] + shape[2] + 4;
    for (int walk = 0; walk < limit; ++walk) {
        const float nearest = fminf(next[0], fminf(next[1], next[2]));
        const float t = nearest - 0.5f;
        const int end = !(t < (float)(last + 1)) ? last + 1 : (t <= (float)i ? i : (int)ceilf(t));
        if (end > i) {
            run32c_t run;
            make_run32c(entry, step_vector, shape, axis_cell, i, end - i, &run);
            action(context, &run);
        }
        i = end;
        if (i > last) break;
        for (int k = 0; k < 3; ++k) {
            if (next[k] == nearest) {
                axis_cell[k] += step_vector[k] > 0.0f ? 1 : -1;
                next[k] = crossing32c(entry, inverse, step_vector, axis_cell, shape, k);
            }
        }
    }
}

/* The cell polynomial f = c0 + c1 x + c2 y + c3 z + c4 xy + c5 xz + c6 yz + c7 xyz of the run's
 * cell and its value and slopes at the run's first fractions. */
typedef struct {
    float c[8];
    float value, gx, gy, gz;
    float a, t1, t2; /* c4 + c7 z, c5 + c7 y, c6 + c7 x */
} runpoly32c_t;

static void run_poly32c(const dpt_problem* p, const void* field, const run32c_t* r, runpoly32c_t* o)
{
    int shape[3] = {p->nx, p->ny, p->nz};
    float v[8];
    for (int c = 0; c < 8; ++c) v[c] = field_value(p, field, corner_index(r->cell, shape, c));
    float* c = o->c;
    c[0] = v[0];
    c[1] = v[1] - v[0];
    c[2] = v[2] - v[0];
    c[3] = v[4] - v[0];
    c[4] = (v[3] - v[2]) - c[1];
    c[5] = (v[5] - v[4]) - c[1];
    c[6] = (v[6] - v[4]) - c[2];
    c[7] = ((v[7] - v[6]) - (v[5] - v[4])) - c[4];
    const float fx = r->f[0], fy = r->f[1], fz = r->f[2];
    o->a = fmaf(c[7], fz, c[4]);
    const float b = fmaf(c[5], fz, c[1]);
    o->gx = fmaf(o->a, fy, b);
    const float e = fmaf(c[6], fz, c[2]), h = fmaf(c[3], fz, c[0]);
    o->value = fmaf(o->gx, fx, fmaf(e, fy, h));
    o->gy = fmaf(o->a, fx, e);
    o->t1 = fmaf(c[7], fy, c[5]);
    o->t2 = fmaf(c[7], fx, c[6]);
    o->gz = fmaf(fx, o->t1, fmaf(c[6], fy, c[3]));
}

/* sum over the run of the cell polynomial: n A + S1 B + S2 C + S3 D */
static float run_sum32c(const run32c_t* r, const runpoly32c_t* o)
{
    const float dx = r->d[0], dy = r->d[1], dz = r->d[2];
    const float dxy = dx * dy, dxz = dx * dz, dyz = dy * dz;
    const float B = fmaf(o->gz, dz, fmaf(o->gy, dy, o->gx * dx));
    const float C = fmaf(o->t2, dyz, fmaf(o->t1, dxz, o->a * dxy));
    const float D = o->c[7] * (dxy * dz);
    return fmaf(r->s3, D, fmaf(r->s2, C, fmaf(r->s1, B, r->nf * o->value)));
}

typedef struct {
    float sum, carry;
} kahan32_t;

static void kahan_add32(kahan32_t* k, float value)
{
    const float y = value - k->carry;
    const float t = k->sum + y;
    k->carry = (t - k->sum) - y;
    k->sum = t;
}

typedef struct {
    const dpt_problem* p;
    const void* field;
    kahan32_t total;
} fwd_context32c;

static void forward_action32c(void* context, const run32c_t* run)
{
    fwd_context32c* ctx = (fwd_context32c*)context;
    runpoly32c_t o;
    run_poly32c(ctx->p, ctx->field, run, &o);
    kahan_add32(&ctx->total, run_sum32c(run, &o));
}

/* ------------------------------------------------------ FP64 cell-Gauss integration
 * kernels/projection.py:522-746: the clipped ray [lower, upper] is split at every
 * interpolation plane (integer grid coordinates 0..n-1 on each axis; the half-cell margins
 * are segments of their own) and each segment, on which the field is a cubic in t, is
 * integrated exactly with the two-node Gauss rule. */

typedef struct {
    int plane[3], step[3];
    double next[3], inverse[3];
} cells_t;

typedef struct {
    double end, radius, first_position, second_position;
    double first_point[3], second_point[3];
    int lower[3];
    int shared;
} segment_t;

/* kernels/projection.py:530-541: cached reciprocal with one FMA correction */
static double crossing_quotient(double delta, double direction, double inverse)
{
    if (inverse == 0.0) return delta / direction;
    const double quotient = delta * inverse;
    if (!isfinite(quotient) || fabs(quotient) < 2.2250738585072014e-308) return delta / direction;
    return fma(fma(-quotient, direction, delta), inverse, quotient);
}

/* :543-556 */
static double cell_crossing(const ray64_t* r, int axis, int plane, const int* shape, double upper,
                            double inverse)
{
    if (r->direction[axis] == 0.0 || plane < 0 || plane >= shape[axis]) return upper;
    const double c = crossing_quotient((double)plane - r->origin[axis], r->direction[axis], inverse);
    return c < upper ? c : upper;
}

/* :559-611: next strictly forward plane per axis, half-cell edge planes included */
static void begin_cells(const ray64_t* r, const interval64_t* iv, const int* shape, cells_t* t)
{
    memset(t, 0, sizeof(*t));
    for (int a = 0; a < 3; ++a) {
        const double entry = fma(iv->lower, r->direction[a], r->origin[a]);
        const double v = r->direction[a];
        if (v != 0.0) {
            const double inverse = 1.0 / v;
            if (isfinite(inverse) && fabs(inverse) >= 2.2250738585072014e-308 &&
                fabs(v) >= 2.2250738585072014e-308)
                t->inverse[a] = inverse;
        }
        if (v > 0.0) {
            t->step[a] = 1;
            const int c = (int)ceil(entry);
            t->plane[a] = c > 0 ? c : 0;
        } else if (v < 0.0) {
            t->step[a] = -1;
            const int c = (int)floor(entry);
            t->plane[a] = c < shape[a] - 1 ? c : shape[a] - 1;
        }
        double crossing = cell_crossing(r, a, t->plane[a], shape, iv->upper, t->inverse[a]);
        if (crossing <= iv->lower) {
            t->plane[a] += t->step[a];
            crossing = cell_crossing(r, a, t->plane[a], shape, iv->upper, t->inverse[a]);
        }
        t->next[a] = crossing;
    }
}

/* :199-206 */
static void cell_lower64(const double* q, const int* shape, int* lower)
{
    for (int a = 0; a < 3; ++a) {
        const double high = (double)(shape[a] - 1);
        const double c = q[a] < 0.0 ? 0.0 : (q[a] > high ? high : q[a]);
        lower[a] = cell_floor(c, shape[a]);
    }
}

/* :614-646: Gauss nodes of the segment from `start` to the nearest plane */
static void cell_segment(const ray64_t* r, const cells_t* t, double start, const int* shape, segment_t* s)
{
    const double n12 = t->next[1] < t->next[2] ? t->next[1] : t->next[2];
    s->end = t->next[0] < n12 ? t->next[0] : n12;
    s->radius = (s->end - start) * 0.5;
    const double centre = start + s->radius;
    const double offset = s->radius / sqrt(3.0);
    s->first_position = centre - offset;
    s->second_position = centre + offset;
    double centre_point[3];
    for (int a = 0; a < 3; ++a) {
        s->first_point[a] = fma(s->first_position, r->direction[a], r->origin[a]);
        s->second_point[a] = fma(s->second_position, r->direction[a], r->origin[a]);
        centre_point[a] = fma(centre, r->direction[a], r->origin[a]);
    }
    cell_lower64(centre_point, shape, s->lower);
    s->shared = 1;
    for (int a = 0; a < 3; ++a) {
        const double low = (double)s->lower[a], up = low + 1.0, high = (double)(shape[a] - 1);
        const double first = s->first_point[a] < 0.0 ? 0.0 : (s->first_point[a] > high ? high : s->first_point[a]);
        const double second = s->second_point[a] < 0.0 ? 0.0 : (s->second_point[a] > high ? high : s->second_point[a]);
        if (first < low || second < low) s->shared = 0;
        if (s->lower[a] < shape[a] - 2 && (first >= up || second >= up)) s->shared = 0;
    }
}

/* :649-660: advance every axis whose plane the segment reached (ties together) */
static void advance_cells(cells_t* t, const ray64_t* r, const int* shape, double end, double upper)
{
    for (int a = 0; a < 3; ++a) {
        if (t->next[a] <= end) {
            t->plane[a] += t->step[a];
            t->next[a] = cell_crossing(r, a, t->plane[a], shape, upper, t->inverse[a]);
        }
    }
}

/* :663-674: value at a clipped endpoint, clamped into the support first */
static double support_value(const dpt_problem* p, const void* field, const double* q, const int* shape)
{
    double bounded[3];
    for (int a = 0; a < 3; ++a) {
        const double high = (double)shape[a] - 0.5;
        bounded[a] = q[a] < -0.5 ? -0.5 : (q[a] > high ? high : q[a]);
    }
    return sample64(p, field, bounded, shape, NULL);
}

/* :717-746 with the segment action :695-711: returns status bits, the integral in *out */
static int forward_cells(const dpt_problem* p, const void* field, const ray_t* ray, double* out)
{
    int shape[3] = {p->nx, p->ny, p->nz}, status = 0;
    const interval64_t* iv = &ray->iv64;
    double integral = 0.0;
    if (iv->upper > iv->lower) {
        cells_t t;
        begin_cells(&ray->r, iv, shape, &t);
        double start = iv->lower;
        int64_t segments = 0, limit = (int64_t)shape[0] + shape[1] + shape[2] + 1;
        while (start < iv->upper && segments < limit) {
            segment_t s;
            cell_segment(&ray->r, &t, start, shape, &s);
            if (s.end <= start) {
                status |= 2;
                break;
            }
            if (!finite3(s.first_point) || !finite3(s.second_point)) status |= 2;
            integral = fma(s.radius, sample64(p, field, s.first_point, shape, NULL), integral);
            integral = fma(s.radius, sample64(p, field, s.second_point, shape, NULL), integral);
            start = s.end;
            advance_cells(&t, &ray->r, shape, s.end, iv->upper);
            ++segments;
        }
        if (start < iv->upper) status |= 2;
        integral *= ray->r.length;
    }
    *out = integral;
    if (!isfinite(p->image_dtype == DPT_F32 ? (double)(float)integral : integral)) status |= 2;
    return status;
}

/* ((seed w0) w1) w2 with w = 1 - f for a 0 bit (scaled_corner_weight, :396-404) */
static double scaled_corner64(const double* fraction, int corner, double seed)
{
    double contribution = seed;
    for (int a = 0; a < 3; ++a) contribution *= ((corner >> a) & 1) ? fraction[a] : 1.0 - fraction[a];
    return contribution;
}

static void fraction64(const double* q, const int* lower, const int* shape, double* fraction)
{
    for (int a = 0; a < 3; ++a) {
        const double high = (double)(shape[a] - 1);
        const double c = q[a] < 0.0 ? 0.0 : (q[a] > high ? high : q[a]);
        fraction[a] = c - (double)lower[a];
    }
}

/* get_scatter_field (:421-479), strict coordinates, FP32 increments */
static int scatter_point64(const dpt_problem* p, double* gradient, const double* q, double seed)
{
    int shape[3] = {p->nx, p->ny, p->nz}, status = 0, lower[3];
    if (!finite3(q)) status |= 2;
    if (!inside64(q, shape)) return status;
    double fraction[3];
    cell_lower64(q, shape, lower);
    fraction64(q, lower, shape, fraction);
    for (int c = 0; c < 8; ++c) {
        const float rounded = (float)scaled_corner64(fraction, c, seed);
        if (!isfinite(rounded)) status |= 2;
        gradient[corner_index(lower, shape, c)] += (double)rounded;
    }
    return status;
}

/* get_scatter_cell (:482-515): both nodes in one cell, corner terms summed in FP64 first */
static int scatter_cell64(const dpt_problem* p, double* gradient, const segment_t* s, double seed)
{
    int shape[3] = {p->nx, p->ny, p->nz}, status = 0;
    if (!finite3(s->first_point) || !finite3(s->second_point)) status |= 2;
    double f1[3], f2[3];
    fraction64(s->first_point, s->lower, shape, f1);
    fraction64(s->second_point, s->lower, shape, f2);
    const int in1 = inside64(s->first_point, shape), in2 = inside64(s->second_point, shape);
    for (int c = 0; c < 8; ++c) {
        const double first = scaled_corner64(f1, c, in1 ? seed : 0.0);
        const double second = scaled_corner64(f2, c, in2 ? seed : 0.0);
        const float rounded = (float)(first + second);
        if (!isfinite(rounded)) status |= 2;
        gradient[corner_index(s->lower, shape, c)] += (double)rounded;
    }
    return status;
}

/* Packed-12 and local-right 6 pose rows from the object-space source and direction
 * cotangents (kernels/projection.py:1184-1210, kernels/geometry.py:39-52). */
static void pose_rows64(const ray_t* ray, const double* sa, const double* da, double* g12, double* g6)
{
    if (g12) {
        const double* wsr = ray->r.world_source_relative;
        const double* wd = ray->r.world_direction;
        for (int row = 0; row < 3; ++row)
            for (int col = 0; col < 3; ++col)
                g12[3 * row + col] = fma(wd[row], da[col], wsr[row] * sa[col]);
        g12[12] = sa[0];
        g12[13] = sa[1];
        g12[14] = sa[2];
    }
    if (g6) {
        const double* os = ray->r.object_source;
        const double* od = ray->r.object_direction;
        g6[0] = -sa[0];
        g6[1] = -sa[1];
        g6[2] = -sa[2];
        g6[3] = fma(-da[2], od[1], da[1] * od[2]) + fma(-sa[2], os[1], sa[1] * os[2]);
        g6[4] = fma(-da[0], od[2], da[2] * od[0]) + fma(-sa[0], os[2], sa[2] * os[0]);
        g6[5] = fma(-da[1], od[0], da[0] * od[1]) + fma(-sa[1], os[0], sa[0] * os[1]);
    }
}

/* Cell-Gauss VJP of one ray (kernels/projection.py:935-1024 and the shared tail
 * 1152-1210): Gauss-node gradients weighted by the radius (origin) and radius x position
 * (direction), the endpoint terms of the zero-extended support, factor = seed*length. */
static int vjp_ray_cells(const dpt_problem* p, const void* field, const ray_t* ray, double seed,
                         int flags, double* gradient, double* g12, double* g6)
{
    int shape[3] = {p->nx, p->ny, p->nz}, status = 0;
    const int active_volume = (flags & DPT_VJP_VOLUME) != 0;
    const int active_pose = (flags & (DPT_VJP_POSE12 | DPT_VJP_POSE6 | DPT_VJP_PER_RAY6)) != 0;
    const interval64_t* iv = &ray->iv64;
    double span = iv->upper - iv->lower;
    if (!isfinite(seed)) status |= 2;
    if (seed == 0.0) span = 0.0;
    if (!(span > 0.0)) return status;
    const double factor = seed * ray->r.length;
    double og[3] = {0.0, 0.0, 0.0}, dg[3] = {0.0, 0.0, 0.0};
    cells_t t;
    begin_cells(&ray->r, iv, shape, &t);
    double start = iv->lower;
    int64_t segments = 0, limit = (int64_t)shape[0] + shape[1] + shape[2] + 1;
    while (start < iv->upper && segments < limit) {
        segment_t s;
        cell_segment(&ray->r, &t, start, shape, &s);
        if (s.end <= start) {
            status |= 2;
            break;
        }
        if (!finite3(s.first_point) || !finite3(s.second_point)) status |= 2;
        if (active_pose) {
            double g1[3], g2[3];
            sample64(p, field, s.first_point, shape, g1);
            sample64(p, field, s.second_point, shape, g2);
            const double r1 = s.radius * s.first_position, r2 = s.radius * s.second_position;
            for (int a = 0; a < 3; ++a) {
                og[a] = fma(s.radius, g1[a], og[a]);
                og[a] = fma(s.radius, g2[a], og[a]);
                dg[a] = fma(r1, g1[a], dg[a]);
                dg[a] = fma(r2, g2[a], dg[a]);
            }
        }
        if (active_volume) {
            const double volume_factor = factor * s.radius;
            if (s.shared) {
                status |= scatter_cell64(p, gradient, &s, volume_factor);
            } else {
                status |= scatter_point64(p, gradient, s.first_point, volume_factor);
                status |= scatter_point64(p, gradient, s.second_point, volume_factor);
            }
        }
        start = s.end;
        advance_cells(&t, &ray->r, shape, s.end, iv->upper);
        ++segments;
    }
    if (start < iv->upper) status |= 2;
    if (!active_pose) return status;
    double lower_point[3], upper_point[3];
    for (int a = 0; a < 3; ++a) {
        lower_point[a] = fma(iv->lower, ray->r.direction[a], ray->r.origin[a]);
        upper_point[a] = fma(iv->upper, ray->r.direction[a], ray->r.origin[a]);
    }
    const double lower_value = support_value(p, field, lower_point, shape);
    const double upper_value = support_value(p, field, upper_point, shape);
    for (int a = 0; a < 3; ++a) {
        og[a] = og[a] + fma(-lower_value, iv->lower_origin[a], upper_value * iv->upper_origin[a]);
        dg[a] = dg[a] + fma(-lower_value, iv->lower_direction[a], upper_value * iv->upper_direction[a]);
    }
    double sa[3], da[3];
    matvec_t(p->object_to_grid, og, sa);
    matvec_t(p->object_to_grid, dg, da);
    for (int a = 0; a < 3; ++a) {
        sa[a] = factor * sa[a];
        da[a] = factor * da[a];
    }
    pose_rows64(ray, sa, da, g12, g6);
    return status;
}

/* ------------------------------------------------------------------ forward */

/* One ray's optical depth; returns status bits. */
static int forward_ray(const dpt_problem* p, const void* field, const ray_t* ray, double* out)
{
    int shape[3] = {p->nx, p->ny, p->nz}, status = 0, S = p->samples;
    *out = 0.0;
    if (!ray->valid) return 2;
    if (p->arith == DPT_ARITH_F32) {
        /* kernels/projection_fp32.py:359-372 */
        const interval32_t* iv = &ray->iv32;
        float total = 0.0f;
        if (iv->upper > iv->lower) {
            float step = (iv->upper - iv->lower) / (float)S;
            for (int i = 0; i < S; ++i) {
                float position = fmaf((float)i + 0.5f, step, iv->lower), q[3];
                for (int a = 0; a < 3; ++a) q[a] = fmaf(position, ray->d32[a], ray->o32[a]);
                if (!finite3f(q)) status |= 2;
                total += sample32(p, field, q, shape, NULL);
            }
            total *= ray->len32 * step;
        }
        if (!isfinite(total)) status |= 2;
        *out = total;
    } else if (p->arith == DPT_ARITH_F64) {
        /* kernels/projection.py:826-844 with get_midpoint_integrator 770-799 */
        const interval64_t* iv = &ray->iv64;
        double integral = 0.0;
        if (iv->upper > iv->lower) {
            double step = (iv->upper - iv->lower) / (double)S;
            for (int i = 0; i < S; ++i) {
                double position = fma((double)i + 0.5, step, iv->lower), q[3];
                for (int a = 0; a < 3; ++a) q[a] = fma(position, ray->r.direction[a], ray->r.origin[a]);
                if (!finite3(q)) status |= 2;
                integral += sample64(p, field, q, shape, NULL);
            }
            integral *= ray->r.length * step;
        }
        *out = integral;
        if (!isfinite(p->image_dtype == DPT_F32 ? (double)(float)integral : integral)) status |= 2;
    } else if (p->arith == DPT_ARITH_CELLS) {
        status |= forward_cells(p, field, ray, out);
    } else if (p->arith == DPT_ARITH_MIXED || p->arith == DPT_ARITH_FAST) {
        /* kernels/projection.py:296-392 (mixed_coordinates, mixed_corner_weight,
         * sample_mixed_field / sample_float32_field, begin_midpoints, mixed_point_fma) with the
         * midpoint integrator 770-799: FP32 points and weights; MIXED sums w*v in FP64, FAST
         * in an FP32 fmaf cell sum promoted to the FP64 ray sum. */
        const interval64_t* iv = &ray->iv64;
        double integral = 0.0;
        if (iv->upper > iv->lower) {
            float entry[3], stepv[3];
            march32c(ray, S, entry, stepv);
            for (int i = 0; i < S; ++i) {
                float q[3];
                point32c(entry, stepv, i, q);
                if (!finite3f(q)) status |= 2;
                integral += sample_mixed32(p, field, q, shape);
            }
            double step = (iv->upper - iv->lower) / (double)S;
            integral *= ray->r.length * step;
        }
        *out = integral;
        if (!isfinite(p->image_dtype == DPT_F32 ? (double)(float)integral : integral)) status |= 2;
    } else {
        /* F32C: FP32 polynomial samples, blocked compensated sum, FP64 scale. */
        const interval64_t* iv = &ray->iv64;
        double integral = 0.0;
        if (iv->upper > iv->lower) {
            float entry[3], stepv[3];
            march32c(ray, S, entry, stepv);
            double total;
            if (segment_form32c(entry, stepv)) {
                int first, last;
                inside_run32c(entry, stepv, shape, S, &first, &last);
                fwd_context32c ctx = {p, field, {0.0f, 0.0f}};
                if (first <= last) traverse32c(entry, stepv, shape, first, last, forward_action32c, &ctx);
                total = (double)ctx.total.sum - (double)ctx.total.carry;
            } else {
                blocksum_t acc = {0.0f, 0.0f, 0.0f};
                for (int i = 0; i < S; ++i) {
                    float q[3];
                    point32c(entry, stepv, i, q);
                    if (!finite3f(q)) status |= 2;
                    blocksum_add(&acc, sample32c(p, field, q, shape, NULL, NULL), i, S);
                }
                total = (double)acc.sum - (double)acc.carry;
            }
            double step = (iv->upper - iv->lower) / (double)S;
            integral = total * (ray->r.length * step);
        }
        *out = integral;
        if (!isfinite(p->image_dtype == DPT_F32 ? (double)(float)integral : integral)) status |= 2;
    }
    return status;
}

static void store_image(const dpt_problem* p, void* image, int64_t index, double value)
{
    if (p->image_dtype == DPT_F64)
        ((double*)image)[index] = value;
    else
        ((float*)image)[index] = (float)value;
}

static double load_image(const dpt_problem* p, const void* image, int64_t index)
{
    if (p->image_dtype == DPT_F64) return ((const double*)image)[index];
    return (double)((const float*)image)[index];
}

int oracle_forward(const dpt_problem* p, const double* poses, const double* view_table,
                   const double* sources, const double* endpoints, const void* field,
                   void* image, int32_t* status, int threads)
{
    int64_t per_view = (int64_t)p->rows * p->cols, total = per_view * p->views;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int64_t ray_index = 0; ray_index < total; ++ray_index) {
        int view = (int)(ray_index / per_view);
        int64_t pixel = ray_index % per_view;
        double source[3], end[3], out;
        ray_t ray;
        ray_endpoints(p, view_table, sources, endpoints, view, pixel, source, end);
        ray_prepare(p, poses + 12 * view, source, end, &ray);
        int bits = forward_ray(p, field, &ray, &out);
        store_image(p, image, ray_index, out);
        if (bits) {
#ifdef _OPENMP
#pragma omp atomic
#endif
            status[view] |= bits;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ counts */

int oracle_counts(const dpt_problem* p, const double* poses, const double* view_table,
                  const double* sources, const double* endpoints, double* lower, double* upper,
                  int32_t* realised, int threads)
{
    int shape[3] = {p->nx, p->ny, p->nz};
    int64_t per_view = (int64_t)p->rows * p->cols, total = per_view * p->views;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int64_t ray_index = 0; ray_index < total; ++ray_index) {
        int view = (int)(ray_index / per_view);
        double source[3], end[3];
        ray_t ray;
        ray_endpoints(p, view_table, sources, endpoints, view, ray_index % per_view, source, end);
        ray_prepare(p, poses + 12 * view, source, end, &ray);
        int count = 0;
        double lo = 0.0, hi = -1.0;
        if (ray.valid && p->arith == DPT_ARITH_F32) {
            lo = ray.iv32.lower;
            hi = ray.iv32.upper;
            if (ray.iv32.upper > ray.iv32.lower) {
                float step = (ray.iv32.upper - ray.iv32.lower) / (float)p->samples;
                for (int i = 0; i < p->samples; ++i) {
                    float position = fmaf((float)i + 0.5f, step, ray.iv32.lower), q[3];
                    for (int a = 0; a < 3; ++a) q[a] = fmaf(position, ray.d32[a], ray.o32[a]);
                    count += inside32(q, shape);
                }
            }
        } else if (ray.valid && (p->arith == DPT_ARITH_F64 || p->arith == DPT_ARITH_CELLS)) {
            lo = ray.iv64.lower;
            hi = ray.iv64.upper;
            if (hi > lo) {
                double step = (hi - lo) / (double)p->samples;
                for (int i = 0; i < p->samples; ++i) {
                    double position = fma((double)i + 0.5, step, lo), q[3];
                    for (int a = 0; a < 3; ++a) q[a] = fma(position, ray.r.direction[a], ray.r.origin[a]);
                    count += inside64(q, shape);
                }
            }
        } else if (ray.valid) {
            lo = ray.iv64.lower;
            hi = ray.iv64.upper;
            if (hi > lo) {
                float entry[3], stepv[3];
                march32c(&ray, p->samples, entry, stepv);
                for (int i = 0; i < p->samples; ++i) {
                    float q[3];
                    point32c(entry, stepv, i, q);
                    count += inside32(q, shape);
                }
            }
        }
        lower[ray_index] = lo;
        upper[ray_index] = hi;
        realised[ray_index] = count;
    }
    return 0;
}

/* --------------------------------------------------------------------- VJP */

/* scatter_increment, kernels/projection_fp32.py:240-258: one rounded product, then the
 * flush of |x| < 2^-126 to signed zero that CUDA global FP32 atomics apply. */
static float scatter_increment(float factor, float weight)
{
    float increment = factor * weight;
    if (fabsf(increment) < 0x1p-126f) return copysignf(0.0f, increment);
    return increment;
}

typedef struct {
    double* gradient; /* private FP64 volume accumulator */
    int shape[3];
    int pending[3];
    float sums[8];
    int carry; /* shared-face carry (volume-only VJP), kernels/projection_fp32.py:396 */
} scatter_t;

static void flush_all(scatter_t* s)
{
    for (int c = 0; c < 8; ++c) {
        s->gradient[corner_index(s->pending, s->shape, c)] += (double)s->sums[c];
        s->sums[c] = 0.0f;
    }
}

/* transition_cell, kernels/projection_fp32.py:272-331 */
static void transition(scatter_t* s, const int* next)
{
    int* lo = s->pending;
    if (s->shape[0] > 1 && s->shape[1] > 1 && s->shape[2] > 1) {
        int d[3] = {next[0] - lo[0], next[1] - lo[1], next[2] - lo[2]};
        for (int axis = 0; axis < 3; ++axis) {
            int o1 = (axis + 1) % 3, o2 = (axis + 2) % 3;
            if (d[o1] == 0 && d[o2] == 0 && (d[axis] == 1 || d[axis] == -1)) {
                int shared_bit = d[axis] == 1 ? 1 : 0;
                float carried[8] = {0};
                for (int c = 0; c < 8; ++c) {
                    if (((c >> axis) & 1) == shared_bit)
                        carried[c ^ (1 << axis)] = s->sums[c];
                    else
                        s->gradient[corner_index(lo, s->shape, c)] += (double)s->sums[c];
                }
                memcpy(s->sums, carried, sizeof(carried));
                return;
            }
        }
    }
    flush_all(s);
}

/* One ray of the FP32 joint VJP, kernels/projection_fp32.py:411-602. */
static int vjp_ray_f32(const dpt_problem* p, const void* field, const ray_t* ray, float seed,
                       int flags, scatter_t* sc, double* g12, double* g6)
{
    int shape[3] = {p->nx, p->ny, p->nz}, status = 0, S = p->samples;
    int active_volume = (flags & DPT_VJP_VOLUME) != 0;
    int active_pose = (flags & (DPT_VJP_POSE12 | DPT_VJP_POSE6 | DPT_VJP_PER_RAY6)) != 0;
    const interval32_t* iv = &ray->iv32;
    float span = iv->upper - iv->lower;
    if (!isfinite(seed)) status |= 2;
    if (!(span > 0.0f && seed != 0.0f)) return status;
    float step = span / (float)S;
    float physical_step = ray->len32 * step;
    float volume_factor = seed * physical_step;
    float mean = 0.0f, direct_origin[3] = {0}, direct_direction[3] = {0};
    float shift_lower = 0.0f, shift_upper = 0.0f;
    int bounded = isfinite(volume_factor) && fabsf(volume_factor) <= 1.0f;
    sc->pending[0] = sc->pending[1] = sc->pending[2] = -1;
    memset(sc->sums, 0, sizeof(sc->sums));
    for (int i = 0; i < S; ++i) {
        float position = fmaf((float)i + 0.5f, step, iv->lower), q[3];
        for (int a = 0; a < 3; ++a) q[a] = fmaf(position, ray->d32[a], ray->o32[a]);
        if (!finite3f(q)) status |= 2;
        if (active_pose) {
            float g[3];
            float value = sample32(p, field, q, shape, g);
            mean += value;
            for (int a = 0; a < 3; ++a) {
                direct_origin[a] += g[a];
                direct_direction[a] = fmaf(position, g[a], direct_direction[a]);
            }
            float alpha = ((float)i + 0.5f) / (float)S;
            float along = fmaf(g[2], ray->d32[2], fmaf(g[1], ray->d32[1], g[0] * ray->d32[0]));
            shift_lower = fmaf(1.0f - alpha, along, shift_lower);
            shift_upper = fmaf(alpha, along, shift_upper);
        }
        if (active_volume) {
            if (inside32(q, shape)) {
                int lower[3];
                float fraction[3], slope[3];
                coordinates32(q, shape, lower, fraction, slope);
                if (lower[0] != sc->pending[0] || lower[1] != sc->pending[1] ||
                    lower[2] != sc->pending[2]) {
                    if (sc->pending[0] >= 0) {
                        if (sc->carry && bounded)
                            transition(sc, lower);
                        else
                            flush_all(sc);
                    } else {
                        memset(sc->sums, 0, sizeof(sc->sums));
                    }
                    memcpy(sc->pending, lower, sizeof(lower));
                }
                for (int c = 0; c < 8; ++c) {
                    float increment = scatter_increment(volume_factor, corner_weight32(fraction, c));
                    if (bounded) {
                        sc->sums[c] += increment;
                    } else if (!isfinite(increment)) {
                        status |= 2;
                        sc->gradient[corner_index(lower, shape, c)] += (double)increment;
                    } else {
                        float partial = sc->sums[c] + increment;
                        if (!isfinite(partial)) {
                            sc->gradient[corner_index(lower, shape, c)] += (double)sc->sums[c];
                            sc->sums[c] = increment;
                        } else {
                            sc->sums[c] = partial;
                        }
                    }
                }
            } else if (sc->pending[0] >= 0) {
                flush_all(sc);
                sc->pending[0] = sc->pending[1] = sc->pending[2] = -1;
            }
        }
    }
    if (active_volume && sc->pending[0] >= 0) flush_all(sc);
    if (!active_pose) return status;

    /* kernels/projection_fp32.py:549-602 */
    float lower_seed = fmaf(span, shift_lower, -mean);
    float upper_seed = fmaf(span, shift_upper, mean);
    float og[3], dg[3];
    for (int a = 0; a < 3; ++a) {
        og[a] = fmaf(upper_seed, iv->upper_origin[a],
                     fmaf(lower_seed, iv->lower_origin[a], span * direct_origin[a]));
        dg[a] = fmaf(upper_seed, iv->upper_direction[a],
                     fmaf(lower_seed, iv->lower_direction[a], span * direct_direction[a]));
    }
    float factor = (seed * ray->len32) / (float)S;
    double og64[3] = {og[0], og[1], og[2]}, dg64[3] = {dg[0], dg[1], dg[2]};
    double sa[3], da[3];
    matvec_t(p->object_to_grid, og64, sa);
    matvec_t(p->object_to_grid, dg64, da);
    for (int a = 0; a < 3; ++a) {
        sa[a] = (double)factor * sa[a];
        da[a] = (double)factor * da[a];
    }
    if (g12) {
        const double* wsr = ray->r.world_source_relative;
        const double* wd = ray->r.world_direction;
        for (int row = 0; row < 3; ++row)
            for (int col = 0; col < 3; ++col)
                g12[3 * row + col] = fma(wd[row], da[col], wsr[row] * sa[col]);
        /* translation = -(R sa); R is the pose rotation, supplied through g12[12..20] */
    }
    if (g6) {
        /* local-right adjoint, kernels/geometry.py:24-52 */
        const double* os = ray->r.object_source;
        const double* od = ray->r.object_direction;
        g6[0] = -sa[0];
        g6[1] = -sa[1];
        g6[2] = -sa[2];
        g6[3] = fma(-da[2], od[1], da[1] * od[2]) + fma(-sa[2], os[1], sa[1] * os[2]);
        g6[4] = fma(-da[0], od[2], da[2] * od[0]) + fma(-sa[0], os[2], sa[2] * os[0]);
        g6[5] = fma(-da[1], od[0], da[0] * od[1]) + fma(-sa[1], os[0], sa[0] * os[1]);
    }
    /* store the source adjoint for the translation rows */
    if (g12) {
        g12[12] = sa[0];
        g12[13] = sa[1];
        g12[14] = sa[2];
    }
    return status;
}

/* One ray of the strict FP64 joint VJP (midpoint), kernels/projection.py:922-1217, with
 * FP32-rounded volume increments (scatter_realised, kernels/projection.py:407-430). */
/* MIXED / FAST volume VJP (fixed pose), kernels/projection.py:1026-1106 with the mixed scatter
 * of get_scatter_field (:431-479): volume_factor = seed*length*span/S in FP64; every inside
 * sample adds, per corner, the FP32 rounding of volume_factor * (double)w_c, w_c the FP32
 * corner weight of the forward. */
static int vjp_ray_mixed(const dpt_problem* p, const ray_t* ray, double seed, scatter_t* sc)
{
    int shape[3] = {p->nx, p->ny, p->nz}, status = 0, S = p->samples;
    const interval64_t* iv = &ray->iv64;
    double span = iv->upper - iv->lower;
    if (!isfinite(seed)) status |= 2;
    if (seed == 0.0) span = 0.0;
    if (!(span > 0.0)) return status;
    double volume_factor = seed * ray->r.length * span / (double)S;
    float entry[3], stepv[3];
    march32c(ray, S, entry, stepv);
    for (int i = 0; i < S; ++i) {
        float q[3], f[3], slope[3];
        int lower[3];
        point32c(entry, stepv, i, q);
        if (!finite3f(q)) status |= 2;
        if (!inside32(q, shape)) continue;
        coordinates32(q, shape, lower, f, slope);
        for (int c = 0; c < 8; ++c) {
            float rounded = (float)(volume_factor * (double)corner_weight32(f, c));
            if (!isfinite(rounded)) status |= 2;
            sc->gradient[corner_index(lower, shape, c)] += (double)rounded;
        }
    }
    return status;
}

static int vjp_ray_f64(const dpt_problem* p, const void* field, const ray_t* ray, double seed,
                       int flags, scatter_t* sc, double* g12, double* g6)
{
    int shape[3] = {p->nx, p->ny, p->nz}, status = 0, S = p->samples;
    int active_volume = (flags & DPT_VJP_VOLUME) != 0;
    int active_pose = (flags & (DPT_VJP_POSE12 | DPT_VJP_POSE6 | DPT_VJP_PER_RAY6)) != 0;
    const interval64_t* iv = &ray->iv64;
    double span = iv->upper - iv->lower;
    if (!isfinite(seed)) status |= 2;
    if (seed == 0.0) span = 0.0;
    if (!(span > 0.0)) return status;
    double factor = seed * ray->r.length;
    double step = span / (double)S;
    double volume_factor = factor * span / (double)S;
    int power_of_two = S > 0 && (S & (S - 1)) == 0;
    double inverse_samples = power_of_two ? 1.0 / (double)S : 0.0;
    double mean = 0.0, direct_origin[3] = {0}, direct_direction[3] = {0};
    double shift_lower = 0.0, shift_upper = 0.0;
    for (int i = 0; i < S; ++i) {
        double alpha = power_of_two ? ((double)i + 0.5) * inverse_samples
                                    : ((double)i + 0.5) / (double)S;
        double position = fma((double)i + 0.5, step, iv->lower), q[3];
        for (int a = 0; a < 3; ++a) q[a] = fma(position, ray->r.direction[a], ray->r.origin[a]);
        if (!finite3(q)) status |= 2;
        int supported = inside64(q, shape);
        if (active_pose) {
            double g[3];
            double value = sample64(p, field, q, shape, g);
            mean += value;
            for (int a = 0; a < 3; ++a) {
                direct_origin[a] += g[a];
                direct_direction[a] = fma(position, g[a], direct_direction[a]);
            }
            const double* d = ray->r.direction;
            double along = fma(g[2], d[2], fma(g[1], d[1], g[0] * d[0]));
            shift_lower = fma(1.0 - alpha, along, shift_lower);
            shift_upper = fma(alpha, along, shift_upper);
        }
        if (active_volume && supported) {
            int lower[3];
            double fraction[3], slope[3];
            coordinates64(q, shape, lower, fraction, slope);
            for (int c = 0; c < 8; ++c) {
                double contribution = volume_factor;
                for (int a = 0; a < 3; ++a)
                    contribution *= ((c >> a) & 1) ? fraction[a] : 1.0 - fraction[a];
                float rounded = (float)contribution;
                if (!isfinite(rounded)) status |= 2;
                sc->gradient[corner_index(lower, shape, c)] += (double)rounded;
            }
        }
    }
    if (!active_pose) return status;
    double lower_seed = fma(span, shift_lower, -mean);
    double upper_seed = fma(span, shift_upper, mean);
    double og[3], dg[3];
    for (int a = 0; a < 3; ++a) {
        og[a] = fma(upper_seed, iv->upper_origin[a],
                    fma(lower_seed, iv->lower_origin[a], span * direct_origin[a]));
        dg[a] = fma(upper_seed, iv->upper_direction[a],
                    fma(lower_seed, iv->lower_direction[a], span * direct_direction[a]));
    }
    factor /= (double)S;
    double sa[3], da[3];
    matvec_t(p->object_to_grid, og, sa);
    matvec_t(p->object_to_grid, dg, da);
    for (int a = 0; a < 3; ++a) {
        sa[a] = factor * sa[a];
        da[a] = factor * da[a];
    }
    if (g12) {
        const double* wsr = ray->r.world_source_relative;
        const double* wd = ray->r.world_direction;
        for (int row = 0; row < 3; ++row)
            for (int col = 0; col < 3; ++col)
                g12[3 * row + col] = fma(wd[row], da[col], wsr[row] * sa[col]);
        g12[12] = sa[0];
        g12[13] = sa[1];
        g12[14] = sa[2];
    }
    if (g6) {
        const double* os = ray->r.object_source;
        const double* od = ray->r.object_direction;
        g6[0] = -sa[0];
        g6[1] = -sa[1];
        g6[2] = -sa[2];
        g6[3] = fma(-da[2], od[1], da[1] * od[2]) + fma(-sa[2], os[1], sa[1] * os[2]);
        g6[4] = fma(-da[0], od[2], da[2] * od[0]) + fma(-sa[0], os[2], sa[2] * os[0]);
        g6[5] = fma(-da[1], od[0], da[0] * od[1]) + fma(-sa[1], os[0], sa[0] * os[1]);
    }
    return status;
}

/* F32C volume scatter: per run of samples in one cell, FP32 moments of the fractions
 * (count, fx, fy, fz, fx fy, fx fz, fy fz, fx fy fz) expand at the end of the run into the
 * eight corner weight sums, which are scaled by the ray's factor once. */
typedef struct {
    int pending[3];
    float m[8];
} moments_t;

static int flush_moments(const dpt_problem* p, moments_t* mo, float factor, double* gradient)
{
    int shape[3] = {p->nx, p->ny, p->nz}, status = 0;
    const float* m = mo->m;
    float corner[8];
    corner[7] = m[7];
    corner[3] = m[4] - m[7];
    corner[5] = m[5] - m[7];
    corner[6] = m[6] - m[7];
    corner[1] = (m[1] - m[4]) - corner[5];
    corner[2] = (m[2] - m[4]) - corner[6];
    corner[4] = (m[3] - m[5]) - corner[6];
    corner[0] = ((m[0] - m[1]) - (m[2] - m[4])) - corner[4];
    for (int c = 0; c < 8; ++c) {
        float increment = factor * corner[c];
        if (!isfinite(increment)) status |= 2;
        gradient[corner_index(mo->pending, shape, c)] += (double)increment;
    }
    memset(mo->m, 0, sizeof(mo->m));
    return status;
}

/* F32C pose chain: clip-face seeds and the FP64 chain through M^T from the mean value,
 * G = sum grad and H = sum alpha grad of one ray (alpha_i = (i + 0.5) / S). */
static int pose_chain32c(const dpt_problem* p, const ray_t* ray, double seed, double span,
                         double mean64, const double* Gd, const double* Hd, double* g12, double* g6)
{
    const interval64_t* iv = &ray->iv64;
    int S = p->samples;
    const double* d = ray->r.direction;
    double g_along = fma(Gd[2], d[2], fma(Gd[1], d[1], Gd[0] * d[0]));
    double h_along = fma(Hd[2], d[2], fma(Hd[1], d[1], Hd[0] * d[0]));
    double shift_upper = h_along, shift_lower = g_along - h_along;
    double lower_seed = fma(span, shift_lower, -mean64);
    double upper_seed = fma(span, shift_upper, mean64);
    double og[3], dg[3];
    for (int a = 0; a < 3; ++a) {
        double direct_direction = fma(span, Hd[a], iv->lower * Gd[a]);
        og[a] = fma(upper_seed, iv->upper_origin[a],
                    fma(lower_seed, iv->lower_origin[a], span * Gd[a]));
        dg[a] = fma(upper_seed, iv->upper_direction[a],
                    fma(lower_seed, iv->lower_direction[a], span * direct_direction));
    }
    double factor = seed * ray->r.length / (double)S;
    double sa[3], da[3];
    matvec_t(p->object_to_grid, og, sa);
    matvec_t(p->object_to_grid, dg, da);
    for (int a = 0; a < 3; ++a) {
        sa[a] = factor * sa[a];
        da[a] = factor * da[a];
    }
    if (g12) {
        const double* wsr = ray->r.world_source_relative;
        const double* wd = ray->r.world_direction;
        for (int row = 0; row < 3; ++row)
            for (int col = 0; col < 3; ++col)
                g12[3 * row + col] = fma(wd[row], da[col], wsr[row] * sa[col]);
        g12[12] = sa[0];
        g12[13] = sa[1];
        g12[14] = sa[2];
    }
    if (g6) {
        const double* os = ray->r.object_source;
        const double* od = ray->r.object_direction;
        g6[0] = -sa[0];
        g6[1] = -sa[1];
        g6[2] = -sa[2];
        g6[3] = fma(-da[2], od[1], da[1] * od[2]) + fma(-sa[2], os[1], sa[1] * os[2]);
        g6[4] = fma(-da[0], od[2], da[2] * od[0]) + fma(-sa[0], os[2], sa[2] * os[0]);
        g6[5] = fma(-da[1], od[0], da[0] * od[1]) + fma(-sa[1], os[0], sa[0] * os[1]);
    }
    return 0;
}

typedef struct {
    const dpt_problem* p;
    const void* field;
    int active_volume, active_pose, status;
    float volume_factor;
    double* gradient;
    kahan32_t mean;
    float G[3], Hs[3];
} vjp_context32c;

/* One run of the segment form's VJP: the pose sums G = sum grad and Hs = sum (i + 0.5) grad
 * and the compensated sum of the values, and the eight moments of the fractions expanded
 * into the run cell's corner sums. */
static void vjp_action32c(void* context, const run32c_t* r)
{
    vjp_context32c* ctx = (vjp_context32c*)context;
    const float dx = r->d[0], dy = r->d[1], dz = r->d[2];
    const float dxy = dx * dy, dxz = dx * dz, dyz = dy * dz;
    const float nf = r->nf, s1 = r->s1, s2 = r->s2, s3 = r->s3;
    if (ctx->active_pose) {
        runpoly32c_t o;
        run_poly32c(ctx->p, ctx->field, r, &o);
        kahan_add32(&ctx->mean, run_sum32c(r, &o));
        float g0[3] = {o.gx, o.gy, o.gz};
        float g1[3] = {fmaf(o.t1, dz, o.a * dy), fmaf(o.t2, dz, o.a * dx), fmaf(o.t2, dy, o.t1 * dx)};
        float g2[3] = {o.c[7] * dyz, o.c[7] * dxz, o.c[7] * dxy};
        const float offset = (float)r->i0 + 0.5f;
        for (int k = 0; k < 3; ++k) {
            if (!r->interior[k]) g0[k] = g1[k] = g2[k] = 0.0f;
            const float sg = fmaf(s2, g2[k], fmaf(s1, g1[k], nf * g0[k]));
            const float sj = fmaf(s3, g2[k], fmaf(s2, g1[k], s1 * g0[k]));
            ctx->G[k] = ctx->G[k] + sg;
            ctx->Hs[k] = ctx->Hs[k] + fmaf(offset, sg, sj);
        }
    }
    if (ctx->active_volume) {
        const float fx = r->f[0], fy = r->f[1], fz = r->f[2];
        const float fxy = fx * fy, fxz = fx * fz, fyz = fy * fz;
        moments_t mo;
        memcpy(mo.pending, r->cell, sizeof(mo.pending));
        float* m = mo.m;
        m[0] = nf;
        m[1] = fmaf(s1, dx, nf * fx);
        m[2] = fmaf(s1, dy, nf * fy);
        m[3] = fmaf(s1, dz, nf * fz);
        m[4] = fmaf(s2, dxy, fmaf(s1, fmaf(fx, dy, fy * dx), nf * fxy));
        m[5] = fmaf(s2, dxz, fmaf(s1, fmaf(fx, dz, fz * dx), nf * fxz));
        m[6] = fmaf(s2, dyz, fmaf(s1, fmaf(fy, dz, fz * dy), nf * fyz));
        m[7] = fmaf(s3, dxy * dz,
                    fmaf(s2, fmaf(fz, dxy, fmaf(fy, dxz, fx * dyz)),
                         fmaf(s1, fmaf(fyz, dx, fmaf(fxz, dy, fxy * dz)), nf * (fxy * fz))));
        ctx->status |= flush_moments(ctx->p, &mo, ctx->volume_factor, ctx->gradient);
    }
}

/* One ray of the F32C VJP: FP64 clip and clip-face chain, FP32 marching, polynomial
 * values and slopes, blocked compensated mean, pose moments G = sum grad and
 * H = sum alpha grad, moment-based volume scatter. */
static int vjp_ray_f32c(const dpt_problem* p, const void* field, const ray_t* ray, double seed,
                        int flags, scatter_t* sc, double* g12, double* g6)
{
    int shape[3] = {p->nx, p->ny, p->nz}, status = 0, S = p->samples;
    int active_volume = (flags & DPT_VJP_VOLUME) != 0;
    int active_pose = (flags & (DPT_VJP_POSE12 | DPT_VJP_POSE6 | DPT_VJP_PER_RAY6)) != 0;
    const interval64_t* iv = &ray->iv64;
    double span = iv->upper - iv->lower;
    if (!isfinite(seed)) status |= 2;
    if (!(span > 0.0 && seed != 0.0)) return status;
    double step = span / (double)S;
    float volume_factor = (float)(seed * ray->r.length * step);
    float entry[3], stepv[3];
    march32c(ray, S, entry, stepv);
    if (segment_form32c(entry, stepv)) {
        int first, last;
        inside_run32c(entry, stepv, shape, S, &first, &last);
        vjp_context32c ctx;
        memset(&ctx, 0, sizeof(ctx));
        ctx.p = p;
        ctx.field = field;
        ctx.active_volume = active_volume;
        ctx.active_pose = active_pose;
        ctx.volume_factor = volume_factor;
        ctx.gradient = sc->gradient;
        if (first <= last) traverse32c(entry, stepv, shape, first, last, vjp_action32c, &ctx);
        status |= ctx.status;
        if (!active_pose) return status;
        const double mean_seg = (double)ctx.mean.sum - (double)ctx.mean.carry;
        double G_seg[3], H_seg[3];
        for (int a = 0; a < 3; ++a) {
            G_seg[a] = ctx.G[a];
            H_seg[a] = (double)ctx.Hs[a] / (double)S;
        }
        return status | pose_chain32c(p, ray, seed, span, mean_seg, G_seg, H_seg, g12, g6);
    }
    blocksum_t mean = {0.0f, 0.0f, 0.0f};
    float G[3] = {0}, H[3] = {0};
    float inv_s = 1.0f / (float)S;
    moments_t mo;
    memset(&mo, 0, sizeof(mo));
    mo.pending[0] = mo.pending[1] = mo.pending[2] = -1;
    for (int i = 0; i < S; ++i) {
        float q[3], g[3], f[3];
        point32c(entry, stepv, i, q);
        if (!finite3f(q)) status |= 2;
        int in = inside32(q, shape);
        if (active_pose) {
            float value = sample32c(p, field, q, shape, g, NULL);
            blocksum_add(&mean, value, i, S);
            float alpha = ((float)i + 0.5f) * inv_s;
            for (int a = 0; a < 3; ++a) {
                G[a] += g[a];
                H[a] = fmaf(alpha, g[a], H[a]);
            }
        }
        if (active_volume) {
            if (in) {
                int lower[3];
                float slope[3];
                coordinates32(q, shape, lower, f, slope);
                if (lower[0] != mo.pending[0] || lower[1] != mo.pending[1] || lower[2] != mo.pending[2]) {
                    if (mo.pending[0] >= 0) status |= flush_moments(p, &mo, volume_factor, sc->gradient);
                    memcpy(mo.pending, lower, sizeof(lower));
                }
                float fxy = f[0] * f[1];
                mo.m[0] += 1.0f;
                mo.m[1] += f[0];
                mo.m[2] += f[1];
                mo.m[3] += f[2];
                mo.m[4] += fxy;
                mo.m[5] += f[0] * f[2];
                mo.m[6] += f[1] * f[2];
                mo.m[7] += fxy * f[2];
            } else if (mo.pending[0] >= 0) {
                status |= flush_moments(p, &mo, volume_factor, sc->gradient);
                mo.pending[0] = mo.pending[1] = mo.pending[2] = -1;
            }
        }
    }
    if (active_volume && mo.pending[0] >= 0) status |= flush_moments(p, &mo, volume_factor, sc->gradient);
    if (!active_pose) return status;
    double Gd[3] = {G[0], G[1], G[2]}, Hd[3] = {H[0], H[1], H[2]};
    double mean64 = (double)mean.sum - (double)mean.carry;
    return status | pose_chain32c(p, ray, seed, span, mean64, Gd, Hd, g12, g6);
}

/*
 * Joint VJP over all rays.
 *   volume_gradient: voxels doubles, accumulated (+=) in FP64 when DPT_VJP_VOLUME.
 *   pose_gradient:   DPT_VJP_POSE12 -> views x 12, DPT_VJP_POSE6 -> views x 6,
 *                    DPT_VJP_PER_RAY6 -> rays x 6 (overwritten).
 * Per-view pose sums run over rays in order, in FP64.
 */
int oracle_vjp(const dpt_problem* p, const double* poses, const double* view_table,
               const double* sources, const double* endpoints, const void* field,
               const void* cotangent, int32_t flags, double* volume_gradient,
               double* pose_gradient, int32_t* status, int threads)
{
    int64_t per_view = (int64_t)p->rows * p->cols, total = per_view * p->views;
    int64_t voxels = (int64_t)p->nx * p->ny * p->nz;
    int components = (flags & DPT_VJP_POSE12) ? 12 : 6;
    int want_pose = (flags & (DPT_VJP_POSE12 | DPT_VJP_POSE6 | DPT_VJP_PER_RAY6)) != 0;
    int nthreads = 1;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
    nthreads = omp_get_max_threads();
#endif
    /* Per-thread private volume accumulators; bounded to keep host memory modest. */
    int64_t limit_threads = (int64_t)(16ll << 30) / (voxels * 8 > 0 ? voxels * 8 : 1);
    if (limit_threads < 1) limit_threads = 1;
    if (nthreads > limit_threads) nthreads = (int)limit_threads;
    double** privates = NULL;
    if (flags & DPT_VJP_VOLUME) {
        privates = (double**)calloc((size_t)nthreads, sizeof(double*));
        for (int t = 0; t < nthreads; ++t) {
            privates[t] = (double*)calloc((size_t)voxels, sizeof(double));
            if (!privates[t]) return -1;
        }
    }
    double* per_ray = NULL;
    if (want_pose) {
        per_ray = (double*)calloc((size_t)total * 15 + 1, sizeof(double));
        if (!per_ray) return -1;
    }
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads)
#endif
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        scatter_t sc;
        memset(&sc, 0, sizeof(sc));
        sc.shape[0] = p->nx;
        sc.shape[1] = p->ny;
        sc.shape[2] = p->nz;
        sc.gradient = privates ? privates[tid] : NULL;
        sc.carry = (flags & DPT_VJP_VOLUME) && !want_pose;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
        for (int64_t ray_index = 0; ray_index < total; ++ray_index) {
            int view = (int)(ray_index / per_view);
            double source[3], end[3], g12[15] = {0}, g6[6] = {0};
            ray_t ray;
            ray_endpoints(p, view_table, sources, endpoints, view, ray_index % per_view, source, end);
            ray_prepare(p, poses + 12 * view, source, end, &ray);
            double seed = load_image(p, cotangent, ray_index);
            int bits = 0;
            if (!ray.valid) {
                bits = 2;
            } else if (p->arith == DPT_ARITH_F32) {
                bits = vjp_ray_f32(p, field, &ray, (float)seed, flags, &sc,
                                   (flags & DPT_VJP_POSE12) ? g12 : NULL,
                                   (flags & (DPT_VJP_POSE6 | DPT_VJP_PER_RAY6)) ? g6 : NULL);
            } else if (p->arith == DPT_ARITH_F64) {
                bits = vjp_ray_f64(p, field, &ray, seed, flags, &sc,
                                   (flags & DPT_VJP_POSE12) ? g12 : NULL,
                                   (flags & (DPT_VJP_POSE6 | DPT_VJP_PER_RAY6)) ? g6 : NULL);
            } else if (p->arith == DPT_ARITH_MIXED || p->arith == DPT_ARITH_FAST) {
                bits = (flags & DPT_VJP_VOLUME) ? vjp_ray_mixed(p, &ray, seed, &sc) : 0;
            } else if (p->arith == DPT_ARITH_CELLS) {
                bits = vjp_ray_cells(p, field, &ray, seed, flags, sc.gradient,
                                     (flags & DPT_VJP_POSE12) ? g12 : NULL,
                                     (flags & (DPT_VJP_POSE6 | DPT_VJP_PER_RAY6)) ? g6 : NULL);
            } else {
                bits = vjp_ray_f32c(p, field, &ray, seed, flags, &sc,
                                    (flags & DPT_VJP_POSE12) ? g12 : NULL,
                                    (flags & (DPT_VJP_POSE6 | DPT_VJP_PER_RAY6)) ? g6 : NULL);
            }
            if (want_pose) {
                double* slot = per_ray + 15 * ray_index;
                if (flags & DPT_VJP_POSE12) {
                    /* translation rows -(R sa), kernels/projection_fp32.py:591-593 */
                    const double* R = poses + 12 * view;
                    double t[3];
                    matvec(R, g12 + 12, t);
                    for (int k = 0; k < 9; ++k) slot[k] = g12[k];
                    for (int a = 0; a < 3; ++a) slot[9 + a] = -t[a];
                } else {
                    for (int k = 0; k < 6; ++k) slot[k] = g6[k];
                }
                if (flags & DPT_VJP_PER_RAY6)
                    for (int k = 0; k < 6; ++k)
                        if (!isfinite(slot[k])) bits |= 2;
            }
            if (bits) {
#ifdef _OPENMP
#pragma omp atomic
#endif
                status[view] |= bits;
            }
        }
    }
    if (privates) {
        for (int64_t v = 0; v < voxels; ++v) {
            double sum = 0.0;
            for (int t = 0; t < nthreads; ++t) sum += privates[t][v];
            volume_gradient[v] += sum;
        }
        for (int t = 0; t < nthreads; ++t) free(privates[t]);
        free(privates);
    }
    if (want_pose) {
        if (flags & DPT_VJP_PER_RAY6) {
            for (int64_t r = 0; r < total; ++r)
                for (int k = 0; k < 6; ++k) pose_gradient[6 * r + k] = per_ray[15 * r + k];
        } else {
            for (int view = 0; view < p->views; ++view) {
                for (int k = 0; k < components; ++k) {
                    double sum = 0.0;
                    for (int64_t px = 0; px < per_view; ++px)
                        sum += per_ray[15 * ((int64_t)view * per_view + px) + k];
                    pose_gradient[components * view + k] = sum;
                    if (!isfinite(sum)) status[view] |= 2;
                }
            }
        }
        free(per_ray);
    }
    return 0;
}

/* ------------------------------------------------------------------- checks */

/* kernels/projection_checks.py:20-24 (physical field: finite and non-negative) */
int oracle_check_field(const dpt_problem* p, const void* field, int64_t voxels)
{
    for (int64_t v = 0; v < voxels; ++v) {
        float value = field_value(p, field, v);
        if (!isfinite(value) || (p->field_domain != DPT_DOMAIN_SIGNED && value < 0.0f)) return 8;
    }
    return 0;
}

/* kernels/geometry.py:55-74: finite, R^T R = I to 1e-10, det >= 0. */
int oracle_check_pose(const double* pose)
{
    for (int k = 0; k < 12; ++k)
        if (!isfinite(pose[k])) return 1;
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            double product = 0.0;
            for (int k = 0; k < 3; ++k) product += pose[3 * k + i] * pose[3 * k + j];
            if (fabs(product - (i == j ? 1.0 : 0.0)) > 1e-10) return 1;
        }
    }
    const double* r = pose;
    double det = r[0] * (r[4] * r[8] - r[5] * r[7]) - r[1] * (r[3] * r[8] - r[5] * r[6]) +
                 r[2] * (r[3] * r[7] - r[4] * r[6]);
    return det < 0.0 ? 1 : 0;
}

int oracle_abi_version(void) { return DPT_B200_ABI_VERSION; }

/* ---------------------------------------------------- deterministic adjoint gather */

/* a b c d with the mantissas multiplied in [2^-4, 1) and the exponents added, one final
 * scaling (numerics.py product4, :11-62) */
static double range_product4(double a, double b, double c, double d)
{
    if (!isfinite(a) || !isfinite(b) || !isfinite(c) || !isfinite(d)) return a * b * c * d;
    if (a == 0.0 || b == 0.0 || c == 0.0 || d == 0.0) return 0.0;
    int ea, eb, ec, ed;
    double ma = frexp(a, &ea), mb = frexp(b, &eb), mc = frexp(c, &ec), md = frexp(d, &ed);
    return ldexp(ma * mb * mc * md, ea + eb + ec + ed);
}

/* point_contribution (projection_adjoint.py:34-45): the corner terms of sample q that land on
 * `voxel`, in corner order, each scaled_corner_weight */
static double point_contribution(int64_t voxel, const double* q, const int* shape, double seed)
{
    double result = 0.0;
    if (!inside64(q, shape)) return result;
    int lower[3];
    double fraction[3];
    cell_lower64(q, shape, lower);
    fraction64(q, lower, shape, fraction);
    for (int c = 0; c < 8; ++c)
        if (corner_index(lower, shape, c) == voxel) result += scaled_corner64(fraction, c, seed);
    return result;
}

/* get_gather (projection_adjoint.py:73-170), midpoint: every view's sum over all of its rays
 * and samples, formed from zero per view and added to the running value (a per-view loop
 * with accumulation), FP64 or FP32 output.  cotangent has the image dtype. */
int oracle_gather(const dpt_problem* p, const double* poses, const double* view_table,
                  const double* sources, const double* endpoints, const void* cotangent, void* out,
                  int out_dtype, int accumulate, int32_t* status, int threads)
{
    const int shape[3] = {p->nx, p->ny, p->nz}, S = p->samples;
    const int64_t voxels = (int64_t)p->nx * p->ny * p->nz, per_view = (int64_t)p->rows * p->cols;
    int bits = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 16) reduction(| : bits)
#endif
    for (int64_t voxel = 0; voxel < voxels; ++voxel) {
        double value = 0.0;
        int running = accumulate;
        if (accumulate) value = out_dtype == DPT_F64 ? ((double*)out)[voxel] : (double)((float*)out)[voxel];
        for (int view = 0; view < p->views; ++view) {
            double total = 0.0;
            for (int64_t pixel = 0; pixel < per_view; ++pixel) {
                double source[3], end[3];
                ray_t ray;
                ray_endpoints(p, view_table, sources, endpoints, view, pixel, source, end);
                ray_setup(p, poses + 12 * view, source, end, &ray.r);
                if (!valid_ray(&ray.r)) {
                    bits |= 2;
                    continue;
                }
                const double seed = (double)load_image(p, cotangent, (int64_t)view * per_view + pixel);
                if (seed == 0.0) continue;
                clip64(ray.r.origin, ray.r.direction, shape, &ray.iv64);
                const double span = ray.iv64.upper - ray.iv64.lower;
                if (span <= 0.0) continue;
                const double factor = seed * ray.r.length;
                const double step = span / (double)S;
                double scale = factor * span / (double)S;
                if (!isfinite(factor)) scale = range_product4(seed, ray.r.length, span, 1.0 / (double)S);
                for (int i = 0; i < S; ++i) {
                    double position = fma((double)i + 0.5, step, ray.iv64.lower), q[3];
                    for (int a = 0; a < 3; ++a) q[a] = fma(position, ray.r.direction[a], ray.r.origin[a]);
                    if (!finite3(q)) bits |= 2;
                    total += point_contribution(voxel, q, shape, scale);
                }
            }
            if (out_dtype == DPT_F64)
                value = running ? total + value : total;
            else
                value = (double)(float)(running ? total + value : total);
            running = 1;
        }
        if (out_dtype == DPT_F64)
            ((double*)out)[voxel] = value;
        else
            ((float*)out)[voxel] = (float)value;
        if (!isfinite(value)) bits |= 2;
    }
    status[0] |= bits;
    return 0;
}

/* product3 (numerics.py:11-52) */
static double range_product3(double a, double b, double c)
{
    if (!isfinite(a) || !isfinite(b) || !isfinite(c)) return a * b * c;
    if (a == 0.0 || b == 0.0 || c == 0.0) return 0.0;
    int ea, eb, ec;
    double ma = frexp(a, &ea), mb = frexp(b, &eb), mc = frexp(c, &ec);
    return ldexp(ma * mb * mc, ea + eb + ec);
}

/* cell_contribution (projection_adjoint.py:48-70): both Gauss nodes of a shared cell, per
 * matching corner first + second */
static double cell_contribution(int64_t voxel, const segment_t* s, const int* shape, double seed)
{
    double result = 0.0, f1[3], f2[3];
    fraction64(s->first_point, s->lower, shape, f1);
    fraction64(s->second_point, s->lower, shape, f2);
    for (int c = 0; c < 8; ++c) {
        if (corner_index(s->lower, shape, c) != voxel) continue;
        const double first = scaled_corner64(f1, c, inside64(s->first_point, shape) ? seed : 0.0);
        const double second = scaled_corner64(f2, c, inside64(s->second_point, shape) ? seed : 0.0);
        result += first + second;
    }
    return result;
}

/* get_gather with cell_gauss (projection_adjoint.py:105-146): every ray's cell segments, views
 * summed as oracle_gather does. */
int oracle_gather_cells(const dpt_problem* p, const double* poses, const double* view_table,
                        const double* sources, const double* endpoints, const void* cotangent, void* out,
                        int out_dtype, int accumulate, int32_t* status, int threads)
{
    const int shape[3] = {p->nx, p->ny, p->nz};
    const int64_t voxels = (int64_t)p->nx * p->ny * p->nz, per_view = (int64_t)p->rows * p->cols;
    int bits = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 16) reduction(| : bits)
#endif
    for (int64_t voxel = 0; voxel < voxels; ++voxel) {
        double value = 0.0;
        int running = accumulate;
        if (accumulate) value = out_dtype == DPT_F64 ? ((double*)out)[voxel] : (double)((float*)out)[voxel];
        for (int view = 0; view < p->views; ++view) {
            double total = 0.0;
            for (int64_t pixel = 0; pixel < per_view; ++pixel) {
                double source[3], end[3];
                ray_t ray;
                ray_endpoints(p, view_table, sources, endpoints, view, pixel, source, end);
                ray_setup(p, poses + 12 * view, source, end, &ray.r);
                if (!valid_ray(&ray.r)) {
                    bits |= 2;
                    continue;
                }
                const double seed = (double)load_image(p, cotangent, (int64_t)view * per_view + pixel);
                if (seed == 0.0) continue;
                clip64(ray.r.origin, ray.r.direction, shape, &ray.iv64);
                const interval64_t* iv = &ray.iv64;
                if (iv->upper - iv->lower <= 0.0) continue;
                const double factor = seed * ray.r.length;
                cells_t t;
                begin_cells(&ray.r, iv, shape, &t);
                double start = iv->lower;
                int64_t segments = 0, limit = (int64_t)shape[0] + shape[1] + shape[2] + 1;
                while (start < iv->upper && segments < limit) {
                    segment_t s;
                    cell_segment(&ray.r, &t, start, shape, &s);
                    if (s.end <= start) {
                        bits |= 2;
                        break;
                    }
                    if (!finite3(s.first_point) || !finite3(s.second_point)) bits |= 2;
                    double vf = factor * s.radius;
                    if (!isfinite(factor)) vf = range_product3(seed, ray.r.length, s.radius);
                    if (s.shared) {
                        total += cell_contribution(voxel, &s, shape, vf);
                    } else {
                        total += point_contribution(voxel, s.first_point, shape, vf);
                        total += point_contribution(voxel, s.second_point, shape, vf);
                    }
                    start = s.end;
                    advance_cells(&t, &ray.r, shape, s.end, iv->upper);
                    ++segments;
                }
                if (start < iv->upper) bits |= 2;
            }
            if (out_dtype == DPT_F64)
                value = running ? total + value : total;
            else
                value = (double)(float)(running ? total + value : total);
            running = 1;
        }
        if (out_dtype == DPT_F64)
            ((double*)out)[voxel] = value;
        else
            ((float*)out)[voxel] = (float)value;
        if (!isfinite(value)) bits |= 2;
    }
    status[0] |= bits;
    return 0;
}
