/*
 * pointwise_oracle.c - CPU restatement of the reference's image-space transmission and
 * objective kernels.  TEST INFRASTRUCTURE ONLY: the checker for the CUDA pointwise path,
 * never called by the product.
 *
 * Each function follows the reference file and lines cited beside it
 * (hcltech-robotics/dpt, python/dpt/...).  Local arithmetic is FP64 rounded once into the
 * destination; built with -ffp-contract=off so every fused multiply-add is the explicit
 * fma() written here.  Scalar sums use the same fixed tree as the CUDA kernels: 256-wide
 * tiles, each summed pairwise (t[i] += t[i + w] for w = 128, 64, ..., 1), level after level
 * until one row is left (reference python/dpt/_reductions.py:27-63).  The FP32 exponential
 * is the C library's expf, so transmission values may differ from the GPU's in the last
 * units in the last place; the tests state those budgets.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define TILE 256

/* ---- fixed reduction tree ------------------------------------------------------------ */

static double tile_sum(const double *values, int64_t begin, int64_t count)
{
    double t[TILE];
    for (int i = 0; i < TILE; ++i) t[i] = begin + i < count ? values[begin + i] : 0.0;
    for (int w = TILE / 2; w > 0; w >>= 1)
        for (int i = 0; i < w; ++i) t[i] += t[i + w];
    return t[0];
}

/* Sum `count` rows through 256-wide tiles; an empty sum is zero. */
static double tree_sum(const double *rows, int64_t count)
{
    if (count <= 0) return 0.0;
    double *level = malloc(sizeof(double) * (size_t)count);
    memcpy(level, rows, sizeof(double) * (size_t)count);
    while (count > 1) {
        const int64_t next = (count + TILE - 1) / TILE;
        for (int64_t b = 0; b < next; ++b) level[b] = tile_sum(level, b * TILE, count);
        count = next;
    }
    const double total = level[0];
    free(level);
    return total;
}

/* Per-pixel terms -> per-block partials -> tree (the two stages the kernels run).  With U
 * vector groups per thread a block covers 1024 U pixels: thread t (0..255) sums, in (u, j)
 * order, pixels 4 (256 (U b + u) + t) + j for u < U, j < 4 (absent pixels add zero); the
 * block's 256 thread sums are then summed pairwise.  The shared-beam VJP runs with U = 2,
 * the objective with U = 1. */
#define VJP_UNROLL 2
#define OBJECTIVE_UNROLL 1

static double pixel_tree_sum(const double *terms, int64_t count, int unroll)
{
    if (count <= 0) return 0.0;
    const int64_t block_pixels = (int64_t)TILE * 4 * unroll;
    const int64_t blocks = (count + block_pixels - 1) / block_pixels;
    double *partials = malloc(sizeof(double) * (size_t)blocks);
    double threads[TILE];
    for (int64_t b = 0; b < blocks; ++b) {
        for (int t = 0; t < TILE; ++t) {
            double sum = 0.0;
            for (int u = 0; u < unroll; ++u)
                for (int j = 0; j < 4; ++j) {
                    const int64_t p = ((b * unroll + u) * TILE + t) * 4 + j;
                    sum += p < count ? terms[p] : 0.0;
                }
            threads[t] = sum;
        }
        partials[b] = tile_sum(threads, 0, TILE);
    }
    const double total = tree_sum(partials, blocks);
    free(partials);
    return total;
}

double oracle_tree_sum(const double *values, int64_t count) { return tree_sum(values, count); }

/* ---- transmission (python/dpt/kernels/transmission.py) ------------------------------- */

/* transmission_factor, :81-89 */
static double factor_of(float depth)
{
    if (depth <= 64.0f) return (double)expf(-depth);
    return exp(-(double)depth);
}

/* removed_primary, :44-58 */
static float removed_of(float depth)
{
    const double x = (double)depth;
    if (x == 0.0) return 0.0f;
    if (x > 0.0 && x <= 2.98023223876953125e-8) return depth;
    if (x <= 0.5) return (float)(-expm1(-x));
    return (float)(1.0 - exp(-x));
}

/* optical_depth_from_decrement, :60-73 */
static float depth_of(float decrement)
{
    const double x = (double)decrement;
    if (x == 0.0) return 0.0f;
    if (x > 0.0 && x <= 2.98023223876953125e-8) return decrement;
    if (x <= 0.5) return (float)(-log1p(-x));
    return (float)(-log(1.0 - x));
}

static float beam_at(int mode, const float *beam, float scalar, int64_t p)
{
    if (mode == 2) return beam[0];
    if (mode == 3) return beam[p];
    return scalar;
}

/* finite_nonnegative / finite_seed / decrement_domain, :305-326; returns bit 1 or 0 */
int oracle_check_values(const float *values, int64_t count, int rule)
{
    for (int64_t p = 0; p < count; ++p) {
        const float v = values[p];
        int bad = !isfinite(v);
        if (rule != 1) bad = bad || v < 0.0f;
        if (rule == 2) bad = bad || v >= 1.0f;
        if (bad) return 1;
    }
    return 0;
}

/* get_forward_kernel, :91-144 (null outputs are skipped) */
void oracle_transmit(const float *depth, int64_t count, int beam_mode, const float *beam, float beam_scalar,
                     float *transmission, float *counts, float *log_transmission, float *removed)
{
    for (int64_t p = 0; p < count; ++p) {
        const float L = depth[p];
        const double factor = factor_of(L);
        if (transmission) transmission[p] = (float)factor;
        if (counts) {
            float c = (float)((double)beam_at(beam_mode, beam, beam_scalar, p) * factor);
            counts[p] = c == 0.0f ? 0.0f : c;
        }
        if (log_transmission) log_transmission[p] = -L;
        if (removed) {
            const float r = removed_of(L);
            removed[p] = r == 0.0f ? 0.0f : r;
        }
    }
}

/* get_vjp_kernel with weighted_depth_adjoint and checked_gradient, :146-237; the shared
 * beam's gradient is the tree sum of get_beam_partial_kernel's terms, :239-268.  Returns the
 * status bits (2 for an overflowing FP32 gradient). */
int oracle_transmit_vjp(const float *depth, int64_t count, int beam_mode, const float *beam, float beam_scalar,
                        const float *seed_t, const float *seed_n, const float *seed_log, const float *seed_r,
                        float *grad_depth, float *grad_beam_pixels, float *grad_beam_shared)
{
    int bits = 0;
    double *terms = grad_beam_shared ? malloc(sizeof(double) * (size_t)(count ? count : 1)) : NULL;
    for (int64_t p = 0; p < count; ++p) {
        const double a = seed_t ? (double)seed_t[p] : 0.0;
        const double b = seed_n ? (double)seed_n[p] : 0.0;
        const double c = seed_log ? (double)seed_log[p] : 0.0;
        const double r = seed_r ? (double)seed_r[p] : 0.0;
        const double factor = (seed_t || seed_n || seed_r) ? factor_of(depth[p]) : 0.0;
        if (grad_depth) {
            const double n0 = seed_n ? (double)beam_at(beam_mode, beam, beam_scalar, p) : 0.0;
            const double derivative = fma(-(b * n0), factor, (r - a) * factor) - c;
            grad_depth[p] = (float)derivative;
            if (!isfinite(grad_depth[p])) bits |= 2;
        }
        if (grad_beam_pixels) {
            grad_beam_pixels[p] = (float)(b * factor);
            if (!isfinite(grad_beam_pixels[p])) bits |= 2;
        }
        if (terms) terms[p] = b * factor;
    }
    if (grad_beam_shared) {
        grad_beam_shared[0] = (float)(seed_n ? pixel_tree_sum(terms, count, VJP_UNROLL) : 0.0);
        if (!isfinite(grad_beam_shared[0])) bits |= 2;
        free(terms);
    }
    return bits;
}

/* get_inverse_kernel, :270-283 */
void oracle_depth_from_removed(const float *removed, int64_t count, float *depth)
{
    for (int64_t p = 0; p < count; ++p) {
        const float L = depth_of(removed[p]);
        depth[p] = L == 0.0f ? 0.0f : L;
    }
}

/* get_inverse_vjp_kernel, :285-303 */
int oracle_depth_from_removed_vjp(const float *removed, const float *seed, int64_t count, float *grad)
{
    int bits = 0;
    for (int64_t p = 0; p < count; ++p) {
        grad[p] = (float)((double)seed[p] / (1.0 - (double)removed[p]));
        if (!isfinite(grad[p])) bits |= 2;
    }
    return bits;
}

/* ---- objectives (python/dpt/kernels/objectives.py) ----------------------------------- */

/* poisson_half_deviance, :100-131 */
static double half_deviance(double predicted, double observed)
{
    if (observed == 0.0) return predicted;
    const double difference = predicted - observed;
    if (fabs(difference) <= 0.25 * observed) {
        const double ratio = difference / observed;
        const double s = ratio / (2.0 + ratio);
        const double square = s * s;
        double series = 1.0 / 23.0;
        for (int term = 0; term < 10; ++term) series = fma(square, series, 1.0 / (double)(21 - 2 * term));
        return observed * fma(-(2.0 * s * square), series, ratio * s);
    }
    const double quotient = observed / predicted;
    if (quotient > 0.0 && isfinite(quotient)) return fma(observed, log(quotient), difference);
    return fma(observed, log(observed) - log(predicted), difference);
}

double oracle_poisson_half_deviance(double predicted, double observed)
{
    return half_deviance(predicted, observed);
}

/* observation_validation_kernel and validation_kernel, :23-98; prediction may be null.
 * prediction_dtype: 0 float, 1 double.  Returns the status bits. */
int oracle_objective_check(const void *prediction, int prediction_dtype, const float *observation,
                           const float *weights, const uint8_t *valid, int64_t count, int poisson,
                           int integer_counts)
{
    int bits = 0;
    for (int64_t p = 0; p < count; ++p) {
        int active = 1;
        if (valid) {
            if (valid[p] > 1) bits |= 1;
            active = valid[p] == 1;
        }
        if (!active) continue;
        const float b = observation[p];
        int invalid = !isfinite(b);
        if (poisson) {
            invalid = invalid || b < 0.0f;
            if (integer_counts) invalid = invalid || floorf(b) != b;
        }
        if (weights) invalid = invalid || !isfinite(weights[p]) || weights[p] < 0.0f;
        if (invalid) bits |= 1;
        if (prediction) {
            const double a = prediction_dtype ? ((const double *)prediction)[p] : (double)((const float *)prediction)[p];
            if (!isfinite(a))
                bits |= 2;
            else if (poisson && (a < 0.0 || (a == 0.0 && b > 0.0f)))
                bits |= 8;
        }
    }
    return bits;
}

/* evaluation_kernel, :133-211, and the FP64 tree of _reductions.py.  prediction_dtype 0:
 * FP32 prediction and seed; 1: FP64.  `wide` selects the FP64-precision forms.  The seed is
 * (weight x derivative) x seed_scale rounded once.  Returns the status bits. */
int oracle_objective(const void *prediction, int prediction_dtype, int wide, const float *observation,
                     const float *weights, const uint8_t *valid, int64_t count, int poisson, double normalisation,
                     double seed_scale, void *seed, double *loss)
{
    int bits = 0;
    double *terms = malloc(sizeof(double) * (size_t)(count ? count : 1));
    for (int64_t p = 0; p < count; ++p) {
        terms[p] = 0.0;
        int active = 1;
        if (valid) {
            if (valid[p] > 1) bits |= 1;
            active = valid[p] == 1;
        }
        if (!active) {
            if (seed) {
                if (prediction_dtype) ((double *)seed)[p] = 0.0;
                else ((float *)seed)[p] = 0.0f;
            }
            continue;
        }
        const double predicted =
            prediction_dtype ? ((const double *)prediction)[p] : (double)((const float *)prediction)[p];
        if (!isfinite(predicted))
            bits |= 2;
        else if (poisson && predicted < 0.0)
            bits |= 8;
        const double observed = (double)observation[p];
        double weight = normalisation;
        if (weights) weight *= (double)weights[p];
        const double difference = predicted - observed;
        double derivative = difference;
        double value = 0.5 * difference * difference;
        if (poisson) {
            if (observed == 0.0) {
                value = predicted;
                derivative = 1.0;
            } else {
                if (isfinite(predicted) && predicted <= 0.0) bits |= 8;
                derivative = difference / predicted;
                value = half_deviance(predicted, observed);
            }
        }
        if (wide && !poisson)
            value = (0.5 * weight * difference) * difference;
        else
            value *= weight;
        if (!isfinite(value)) bits |= 2;
        terms[p] = value;
        if (seed) {
            double weighted = weight * derivative;
            if (wide && poisson && !isfinite(derivative)) weighted = (weight * difference) / predicted;
            const double scaled = weighted * seed_scale;
            if (prediction_dtype) {
                ((double *)seed)[p] = scaled;
                if (!isfinite(scaled)) bits |= 2;
            } else {
                const float rounded = (float)scaled;
                ((float *)seed)[p] = rounded;
                if (!isfinite(rounded)) bits |= 2;
            }
        }
    }
    if (loss) {
        loss[0] = pixel_tree_sum(terms, count, OBJECTIVE_UNROLL);
        if (!isfinite(loss[0])) bits |= 2;
    }
    free(terms);
    return bits;
}
