// pointwise.cu - the image-space steps on either side of the projection in a recovery loop:
// Beer-Lambert transmission (reference python/dpt/kernels/transmission.py) and the fused
// objective value and image-space seed (reference python/dpt/kernels/objectives.py:133-211).
//
// One thread per pixel.  Local arithmetic is FP64 and rounds once into each FP32 (or FP64)
// destination, as the reference does.  Scalar results (an objective's loss, an active
// shared beam's gradient) are reduced without floating-point atomics: the pixel kernel
// writes one FP64 partial per 256-pixel tile, then a fixed tree of 256-wide tiles
// (reference python/dpt/_reductions.py:27-63) reduces them and one thread rounds the total
// into its destination, so every sum is deterministic for a given pixel count.
//
// Checks of fixed inputs (finite, nonnegative, inside a domain) are separate launches that
// write nothing but the status word, so a checked host call can reject its inputs before any
// output is touched (reference python/dpt/transmission.py:278-305, objectives.py:252-270).
// Status bits: 1 invalid input, 2 an unrepresentable result, 8 a prediction outside the
// Poisson trial domain.
#include <cstdint>

#include "launch.h"

namespace dpt {
namespace {

constexpr int kTile = 256;

__device__ __forceinline__ void flag(int32_t* status, int bits)
{
    if (bits) atomicOr(status, bits);
}

// Fixed-order sum of one value per thread of a 256-thread block (pairwise tree in shared
// memory); the total is valid in thread 0.
__device__ __forceinline__ double tile_sum(double value, double* tree)
{
    tree[threadIdx.x] = value;
    __syncthreads();
    for (int width = kTile / 2; width > 0; width >>= 1) {
        if (threadIdx.x < width) tree[threadIdx.x] += tree[threadIdx.x + width];
        __syncthreads();
    }
    return tree[0];
}

// exp(-L) kept in FP64 until every requested product is formed (reference
// kernels/transmission.py:81-89): the FP32 exponential while exp(-L) is a normal FP32 value.
__device__ __forceinline__ double transmission_factor(float depth)
{
    if (depth <= 64.0f) return (double)expf(-depth);
    return exp(-(double)depth);
}

// 1 - exp(-L) without cancellation (reference kernels/transmission.py:44-58): below 2^-25
// the input itself is the correctly rounded result.
__device__ __forceinline__ float removed_primary(float depth)
{
    const double x = (double)depth;
    if (x == 0.0) return 0.0f;
    if (x > 0.0 && x <= 2.98023223876953125e-8) return depth;
    if (x <= 0.5) return (float)(-expm1(-x));
    return (float)(1.0 - exp(-x));
}

// -log(1 - delta) without cancellation (reference kernels/transmission.py:60-73).
__device__ __forceinline__ float depth_from_decrement(float decrement)
{
    const double x = (double)decrement;
    if (x == 0.0) return 0.0f;
    if (x > 0.0 && x <= 2.98023223876953125e-8) return decrement;
    if (x <= 0.5) return (float)(-log1p(-x));
    return (float)(-log(1.0 - x));
}

__device__ __forceinline__ float illumination(int beam_mode, const float* beam, float scalar, int64_t p)
{
    if (beam_mode == DPT_BEAM_DEVICE_SCALAR) return beam[0];
    if (beam_mode == DPT_BEAM_PER_PIXEL) return beam[p];
    return scalar;
}

// Input rules of the reference's check kernels (kernels/transmission.py:305-326).
__global__ void __launch_bounds__(kTile) k_check_values(const float* __restrict__ values, int64_t count,
                                                        int rule, int32_t* status)
{
    const int64_t p = (int64_t)blockIdx.x * kTile + threadIdx.x;
    if (p >= count) return;
    const float v = values[p];
    bool bad = !isfinite(v);
    if (rule != DPT_CHECK_FINITE) bad = bad || v < 0.0f;
    if (rule == DPT_CHECK_DECREMENT) bad = bad || v >= 1.0f;
    if (bad) atomicOr(status, 1);
}

// Forward map (reference get_forward_kernel, kernels/transmission.py:91-144).  Counts are
// formed from the FP64 factor, never from a stored FP32 transmission; -0 results become +0.
__global__ void __launch_bounds__(kTile) k_transmit(const float* __restrict__ depth, int64_t count, int mask,
                                                    int beam_mode, const float* __restrict__ beam,
                                                    float beam_scalar, float* __restrict__ transmission,
                                                    float* __restrict__ counts, float* __restrict__ log_t,
                                                    float* __restrict__ removed)
{
    const int64_t p = (int64_t)blockIdx.x * kTile + threadIdx.x;
    if (p >= count) return;
    const float L = depth[p];
    if (mask & (DPT_OUT_TRANSMISSION | DPT_OUT_COUNTS)) {
        const double factor = transmission_factor(L);
        if (mask & DPT_OUT_TRANSMISSION) transmission[p] = (float)factor;
        if (mask & DPT_OUT_COUNTS) {
            float c = (float)((double)illumination(beam_mode, beam, beam_scalar, p) * factor);
            if (c == 0.0f) c = 0.0f;
            counts[p] = c;
        }
    }
    if (mask & DPT_OUT_LOG_TRANSMISSION) log_t[p] = -L;
    if (mask & DPT_OUT_REMOVED) {
        float r = removed_primary(L);
        if (r == 0.0f) r = 0.0f;
        removed[p] = r;
    }
}

// Round an FP64 derivative once into FP32 and flag overflow (reference checked_gradient).
__device__ __forceinline__ float checked(double value, int& bits)
{
    const float rounded = (float)value;
    if (!isfinite(rounded)) bits |= 2;
    return rounded;
}

// Pointwise VJP (reference get_vjp_kernel / weighted_depth_adjoint / get_beam_partial_kernel,
// kernels/transmission.py:146-268): d/dL of sum cT T + cN n0 T - cLog L + cR (1 - T), the
// per-pixel beam gradient cN T, and for a shared beam one FP64 partial of sum cN T per tile.
// A missing cotangent is zero; `accumulate` adds the destination before the single rounding.
__global__ void __launch_bounds__(kTile) k_transmit_vjp(
    const float* __restrict__ depth, int64_t count, int beam_mode, const float* __restrict__ beam,
    float beam_scalar, const float* __restrict__ seed_t, const float* __restrict__ seed_n,
    const float* __restrict__ seed_log, const float* __restrict__ seed_r, float* __restrict__ grad_depth,
    float* __restrict__ grad_beam, double* __restrict__ beam_partials, int accumulate, int32_t* status)
{
    __shared__ double tree[kTile];
    const int64_t p = (int64_t)blockIdx.x * kTile + threadIdx.x;
    double beam_term = 0.0;
    int bits = 0;
    if (p < count) {
        const float L = depth[p];
        const double a = seed_t ? (double)seed_t[p] : 0.0;
        const double b = seed_n ? (double)seed_n[p] : 0.0;
        const double c = seed_log ? (double)seed_log[p] : 0.0;
        const double r = seed_r ? (double)seed_r[p] : 0.0;
        const double factor = (seed_t || seed_n || seed_r) ? transmission_factor(L) : 0.0;
        if (grad_depth) {
            const double n0 = seed_n ? (double)illumination(beam_mode, beam, beam_scalar, p) : 0.0;
            const double optical = (r - a) * factor;
            double derivative = fma(-(b * n0), factor, optical) - c;
            if (accumulate) derivative += (double)grad_depth[p];
            grad_depth[p] = checked(derivative, bits);
        }
        beam_term = b * factor;
        if (grad_beam) {
            double derivative = beam_term;
            if (accumulate) derivative += (double)grad_beam[p];
            grad_beam[p] = checked(derivative, bits);
        }
    }
    if (beam_partials) {
        const double total = tile_sum(beam_term, tree);
        if (threadIdx.x == 0) beam_partials[blockIdx.x] = total;
    }
    flag(status, bits);
}

__global__ void __launch_bounds__(kTile) k_depth_from_removed(const float* __restrict__ decrement,
                                                              int64_t count, float* __restrict__ depth)
{
    const int64_t p = (int64_t)blockIdx.x * kTile + threadIdx.x;
    if (p >= count) return;
    float L = depth_from_decrement(decrement[p]);
    if (L == 0.0f) L = 0.0f;
    depth[p] = L;
}

// d/d delta of -log(1 - delta) is 1 / (1 - delta) (reference get_inverse_vjp_kernel).
__global__ void __launch_bounds__(kTile) k_depth_from_removed_vjp(const float* __restrict__ decrement,
                                                                  const float* __restrict__ seed,
                                                                  int64_t count, float* __restrict__ grad,
                                                                  int accumulate, int32_t* status)
{
    const int64_t p = (int64_t)blockIdx.x * kTile + threadIdx.x;
    if (p >= count) return;
    int bits = 0;
    double derivative = (double)seed[p] / (1.0 - (double)decrement[p]);
    if (accumulate) derivative += (double)grad[p];
    grad[p] = checked(derivative, bits);
    flag(status, bits);
}

// Poisson half-deviance mu - y + y log(y / mu) without cancellation (reference
// kernels/objectives.py:100-131): near equality log1p(r) = 2 atanh(s), s = r / (2 + r), with
// the linear term removed analytically and the odd series summed to its 23rd-order term.
__device__ __forceinline__ double poisson_half_deviance(double predicted, double observed)
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

// Fixed-input and trial-domain checks (reference observation_validation_kernel and
// validation_kernel, kernels/objectives.py:23-98).  A null prediction checks the
// observation, weights and mask alone.
template <typename T>
__global__ void __launch_bounds__(kTile) k_objective_check(const T* __restrict__ prediction,
                                                           const float* __restrict__ observation,
                                                           const float* __restrict__ weights,
                                                           const uint8_t* __restrict__ valid, int64_t count,
                                                           int poisson, int integer_counts, int32_t* status)
{
    const int64_t p = (int64_t)blockIdx.x * kTile + threadIdx.x;
    if (p >= count) return;
    int bits = 0;
    bool active = true;
    if (valid) {
        if (valid[p] > 1) bits |= 1;
        active = valid[p] == 1;
    }
    if (active) {
        const float b = observation[p];
        bool invalid = !isfinite(b);
        if (poisson) {
            invalid = invalid || b < 0.0f;
            if (integer_counts) invalid = invalid || floorf(b) != b;
        }
        if (weights) invalid = invalid || !isfinite(weights[p]) || weights[p] < 0.0f;
        if (invalid) bits |= 1;
        if (prediction) {
            const T a = prediction[p];
            if (!isfinite(a))
                bits |= 2;
            else if (poisson && (a < (T)0 || (a == (T)0 && b > 0.0f)))
                bits |= 8;
        }
    }
    flag(status, bits);
}

// Objective terms and the image-space seed (reference evaluation_kernel,
// kernels/objectives.py:133-211).  kind: half squared error or Poisson half-deviance; each
// active pixel's loss is weighted by normalisation x weights[p] and summed per tile into
// `partials` (skipped when null).  `kWide` selects the FP64-precision forms: the squared
// loss as (0.5 w d) d and a Poisson seed recomputed as (w d) / mu when w / mu overflows.
// The seed is (w x derivative) x seed_scale rounded once into TOut; seed_scale = 1 except
// where a scalar upstream cotangent is folded in before that rounding.
template <typename TIn, typename TOut, bool kWide>
__global__ void __launch_bounds__(kTile) k_objective(const TIn* __restrict__ prediction,
                                                     const float* __restrict__ observation,
                                                     const float* __restrict__ weights,
                                                     const uint8_t* __restrict__ valid, int64_t count,
                                                     int poisson, double normalisation, double seed_scale,
                                                     TOut* __restrict__ seed, double* __restrict__ partials,
                                                     int32_t* status)
{
    __shared__ double tree[kTile];
    const int64_t p = (int64_t)blockIdx.x * kTile + threadIdx.x;
    double loss = 0.0;
    int bits = 0;
    if (p < count) {
        bool active = true;
        if (valid) {
            if (valid[p] > 1) bits |= 1;
            active = valid[p] == 1;
        }
        if (active) {
            const double predicted = (double)prediction[p];
            if (!isfinite(predicted))
                bits |= 2;
            else if (poisson && predicted < 0.0)
                bits |= 8;
            const double observed = (double)observation[p];
            double weight = normalisation;
            if (weights) weight *= (double)weights[p];
            const double difference = predicted - observed;
            double derivative = difference;
            loss = 0.5 * difference * difference;
            if (poisson) {
                if (observed == 0.0) {
                    loss = predicted;
                    derivative = 1.0;
                } else {
                    if (isfinite(predicted) && predicted <= 0.0) bits |= 8;
                    derivative = difference / predicted;
                    loss = poisson_half_deviance(predicted, observed);
                }
            }
            if (kWide && !poisson)
                loss = (0.5 * weight * difference) * difference;
            else
                loss *= weight;
            if (!isfinite(loss)) bits |= 2;
            if (seed) {
                double weighted = weight * derivative;
                if (kWide && poisson && !isfinite(derivative)) weighted = (weight * difference) / predicted;
                const TOut result = (TOut)(weighted * seed_scale);
                seed[p] = result;
                if (!isfinite((double)result)) bits |= 2;
            }
        } else if (seed) {
            seed[p] = (TOut)0.0;
        }
    }
    if (partials) {
        const double total = tile_sum(loss, tree);
        if (threadIdx.x == 0) partials[blockIdx.x] = total;
    }
    flag(status, bits);
}

// One level of the reduction tree: block b sums rows [256 b, 256 b + 256) of `source`.
__global__ void __launch_bounds__(kTile) k_reduce(const double* __restrict__ source, int64_t count,
                                                  double* __restrict__ destination)
{
    __shared__ double tree[kTile];
    const int64_t index = (int64_t)blockIdx.x * kTile + threadIdx.x;
    const double total = tile_sum(index < count ? source[index] : 0.0, tree);
    if (threadIdx.x == 0) destination[blockIdx.x] = total;
}

// Store the tree's root once (reference kernels/reductions.py:39-61): an empty sum is zero,
// `accumulate` adds the destination first, a non-finite stored value sets bit 2.
template <typename T>
__global__ void k_finish(const double* __restrict__ root, int nonempty, T* __restrict__ destination,
                         int accumulate, int32_t* status)
{
    double value = nonempty ? root[0] : 0.0;
    if (accumulate) value += (double)destination[0];
    const T result = (T)value;
    destination[0] = result;
    if (!isfinite((double)result)) atomicOr(status, 2);
}

int64_t tiles(int64_t count) { return (count + kTile - 1) / kTile; }

// Rows of scratch the tree above `count` first-level rows needs (all levels after the first).
int64_t tree_rows(int64_t count)
{
    int64_t rows = 0;
    while (count > 1) {
        count = tiles(count);
        rows += count;
    }
    return rows;
}

// Reduce `count` FP64 rows of `first` through 256-wide tiles in `scratch` and store the total.
template <typename T>
void finish_tree(const double* first, int64_t count, double* scratch, T* destination, int accumulate,
                 int32_t* status, cudaStream_t stream)
{
    const double* previous = first;
    const int nonempty = count > 0;
    while (count > 1) {
        const int64_t next = tiles(count);
        k_reduce<<<(unsigned)next, kTile, 0, stream>>>(previous, count, scratch);
        previous = scratch;
        scratch += next;
        count = next;
    }
    k_finish<T><<<1, 1, 0, stream>>>(previous, nonempty, destination, accumulate, status);
}

int launched() { return (int)cudaGetLastError(); }

}  // namespace
}  // namespace dpt

using dpt::kTile;

extern "C" {

size_t dpt_b200_reduction_bytes(int64_t count)
{
    if (count < 0) return 0;
    const int64_t first = count ? dpt::tiles(count) : 0;
    return (size_t)(first + dpt::tree_rows(first) + 1) * sizeof(double);
}

int dpt_b200_check_values(const float* values, int64_t count, int32_t rule, int32_t* status, void* stream)
{
    if (count < 0 || count > INT32_MAX) return DPT_E_SHAPE;
    if (rule < DPT_CHECK_FINITE_NONNEGATIVE || rule > DPT_CHECK_DECREMENT) return DPT_E_FLAGS;
    if (!status || (count && !values)) return DPT_E_NULL;
    if (!count) return DPT_OK;
    dpt::k_check_values<<<(unsigned)dpt::tiles(count), kTile, 0, static_cast<cudaStream_t>(stream)>>>(
        values, count, rule, status);
    return dpt::launched();
}

int dpt_b200_transmit(const float* depth, int64_t count, int32_t mask, int32_t beam_mode, const float* beam,
                      float beam_scalar, float* transmission, float* counts, float* log_transmission,
                      float* removed, void* stream)
{
    if (count < 0 || count > INT32_MAX) return DPT_E_SHAPE;
    if (mask < 1 || mask > 15 || beam_mode < DPT_BEAM_NONE || beam_mode > DPT_BEAM_PER_PIXEL) return DPT_E_FLAGS;
    if ((mask & DPT_OUT_COUNTS) && beam_mode == DPT_BEAM_NONE) return DPT_E_FLAGS;
    if (count && !depth) return DPT_E_NULL;
    if (((mask & DPT_OUT_TRANSMISSION) && !transmission) || ((mask & DPT_OUT_COUNTS) && !counts) ||
        ((mask & DPT_OUT_LOG_TRANSMISSION) && !log_transmission) || ((mask & DPT_OUT_REMOVED) && !removed))
        return DPT_E_NULL;
    if ((mask & DPT_OUT_COUNTS) && beam_mode >= DPT_BEAM_DEVICE_SCALAR && !beam) return DPT_E_NULL;
    if (!count) return DPT_OK;
    dpt::k_transmit<<<(unsigned)dpt::tiles(count), kTile, 0, static_cast<cudaStream_t>(stream)>>>(
        depth, count, mask, beam_mode, beam, beam_scalar, transmission, counts, log_transmission, removed);
    return dpt::launched();
}

int dpt_b200_transmit_vjp(const float* depth, int64_t count, int32_t beam_mode, const float* beam,
                          float beam_scalar, const float* seed_transmission, const float* seed_counts,
                          const float* seed_log_transmission, const float* seed_removed, float* grad_depth,
                          float* grad_beam, double* scratch, int32_t accumulate, int32_t* status,
                          void* stream)
{
    if (count < 0 || count > INT32_MAX) return DPT_E_SHAPE;
    if (beam_mode < DPT_BEAM_NONE || beam_mode > DPT_BEAM_PER_PIXEL) return DPT_E_FLAGS;
    if (seed_counts && beam_mode == DPT_BEAM_NONE) return DPT_E_FLAGS;
    if (grad_beam && beam_mode < DPT_BEAM_DEVICE_SCALAR) return DPT_E_FLAGS;
    if (!grad_depth && !grad_beam) return DPT_E_FLAGS;
    if (!status || (count && !depth)) return DPT_E_NULL;
    if (seed_counts && beam_mode >= DPT_BEAM_DEVICE_SCALAR && !beam) return DPT_E_NULL;
    const bool shared = grad_beam && beam_mode == DPT_BEAM_DEVICE_SCALAR;
    if (shared && !scratch) return DPT_E_NULL;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool per_pixel = grad_beam && beam_mode == DPT_BEAM_PER_PIXEL;
    const bool partials = shared && seed_counts && count;
    if (count && (grad_depth || per_pixel || partials)) {
        dpt::k_transmit_vjp<<<(unsigned)dpt::tiles(count), kTile, 0, s>>>(
            depth, count, beam_mode, beam, beam_scalar, seed_transmission, seed_counts, seed_log_transmission,
            seed_removed, grad_depth, per_pixel ? grad_beam : nullptr, partials ? scratch : nullptr, accumulate,
            status);
    }
    if (shared) {
        const int64_t rows = partials ? dpt::tiles(count) : 0;
        dpt::finish_tree<float>(scratch, rows, scratch + rows, grad_beam, accumulate, status, s);
    }
    return dpt::launched();
}

int dpt_b200_depth_from_removed(const float* removed, int64_t count, float* depth, void* stream)
{
    if (count < 0 || count > INT32_MAX) return DPT_E_SHAPE;
    if (count && (!removed || !depth)) return DPT_E_NULL;
    if (!count) return DPT_OK;
    dpt::k_depth_from_removed<<<(unsigned)dpt::tiles(count), kTile, 0, static_cast<cudaStream_t>(stream)>>>(
        removed, count, depth);
    return dpt::launched();
}

int dpt_b200_depth_from_removed_vjp(const float* removed, const float* seed, int64_t count, float* grad,
                                    int32_t accumulate, int32_t* status, void* stream)
{
    if (count < 0 || count > INT32_MAX) return DPT_E_SHAPE;
    if (!status || (count && (!removed || !seed || !grad))) return DPT_E_NULL;
    if (!count) return DPT_OK;
    dpt::k_depth_from_removed_vjp<<<(unsigned)dpt::tiles(count), kTile, 0, static_cast<cudaStream_t>(stream)>>>(
        removed, seed, count, grad, accumulate, status);
    return dpt::launched();
}

int dpt_b200_objective_check(const void* prediction, int32_t prediction_dtype, const float* observation,
                             const float* weights, const uint8_t* valid, int64_t count, int32_t kind,
                             int32_t integer_counts, int32_t* status, void* stream)
{
    if (count < 0 || count > INT32_MAX) return DPT_E_SHAPE;
    if (kind != DPT_OBJECTIVE_SQUARED_ERROR && kind != DPT_OBJECTIVE_POISSON) return DPT_E_FLAGS;
    if (prediction_dtype != DPT_F32 && prediction_dtype != DPT_F64) return DPT_E_DTYPE;
    if (!status || (count && !observation)) return DPT_E_NULL;
    if (!count) return DPT_OK;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const unsigned blocks = (unsigned)dpt::tiles(count);
    const int poisson = kind == DPT_OBJECTIVE_POISSON;
    if (prediction_dtype == DPT_F64)
        dpt::k_objective_check<double><<<blocks, kTile, 0, s>>>(static_cast<const double*>(prediction),
                                                                observation, weights, valid, count, poisson,
                                                                integer_counts, status);
    else
        dpt::k_objective_check<float><<<blocks, kTile, 0, s>>>(static_cast<const float*>(prediction),
                                                               observation, weights, valid, count, poisson,
                                                               integer_counts, status);
    return dpt::launched();
}

int dpt_b200_objective(const void* prediction, int32_t prediction_dtype, int32_t wide, const float* observation,
                       const float* weights, const uint8_t* valid, int64_t count, int32_t kind,
                       double normalisation, double seed_scale, void* seed, double* scratch, double* loss,
                       int32_t* status, void* stream)
{
    if (count < 0 || count > INT32_MAX) return DPT_E_SHAPE;
    if (kind != DPT_OBJECTIVE_SQUARED_ERROR && kind != DPT_OBJECTIVE_POISSON) return DPT_E_FLAGS;
    if (prediction_dtype != DPT_F32 && prediction_dtype != DPT_F64) return DPT_E_DTYPE;
    if (prediction_dtype == DPT_F64 && !wide) return DPT_E_DTYPE;
    if (!seed && !loss) return DPT_E_FLAGS;
    if (!status || (count && (!prediction || !observation)) || (loss && !scratch)) return DPT_E_NULL;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int poisson = kind == DPT_OBJECTIVE_POISSON;
    double* partials = loss ? scratch : nullptr;
    if (count) {
        const unsigned blocks = (unsigned)dpt::tiles(count);
        if (prediction_dtype == DPT_F64)
            dpt::k_objective<double, double, true><<<blocks, kTile, 0, s>>>(
                static_cast<const double*>(prediction), observation, weights, valid, count, poisson, normalisation,
                seed_scale, static_cast<double*>(seed), partials, status);
        else if (wide)
            dpt::k_objective<float, float, true><<<blocks, kTile, 0, s>>>(
                static_cast<const float*>(prediction), observation, weights, valid, count, poisson, normalisation,
                seed_scale, static_cast<float*>(seed), partials, status);
        else
            dpt::k_objective<float, float, false><<<blocks, kTile, 0, s>>>(
                static_cast<const float*>(prediction), observation, weights, valid, count, poisson, normalisation,
                seed_scale, static_cast<float*>(seed), partials, status);
    }
    if (loss) {
        const int64_t rows = dpt::tiles(count);
        dpt::finish_tree<double>(scratch, rows, scratch + rows, loss, 0, status, s);
    }
    return dpt::launched();
}

int dpt_b200_reduce_sum(const double* values, int64_t count, double* scratch, double* total, int32_t* status,
                        void* stream)
{
    if (count < 0 || count > INT32_MAX) return DPT_E_SHAPE;
    if (!status || !total || (count && !values) || (count > 1 && !scratch)) return DPT_E_NULL;
    dpt::finish_tree<double>(values, count, scratch, total, 0, status, static_cast<cudaStream_t>(stream));
    return dpt::launched();
}

}  // extern "C"
