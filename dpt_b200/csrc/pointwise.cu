// pointwise.cu - the image-space steps on either side of the projection in a recovery loop:
// Beer-Lambert transmission (reference python/dpt/kernels/transmission.py) and the fused
// objective value and image-space seed (reference python/dpt/kernels/objectives.py:133-211).
//
// These kernels stream HBM: each thread owns U 16-byte vector groups of 4 pixels (group u
// of thread t in block b starts at pixel 4 (256 (U b + u) + t)), issues every load before any
// arithmetic so that enough bytes are in flight to cover DRAM latency, and falls back to
// scalar accesses for a ragged tail or when a caller's pointer is not 16-byte aligned.
// Local arithmetic is FP64 and rounds once into each FP32 (or FP64) destination, as the
// reference does.  Scalar results (an objective's loss, an active shared beam's gradient)
// are reduced without floating-point atomics: each thread sums its 4 U terms in (u, j)
// order, the block sums its 256 threads pairwise into one FP64 partial per 1024 U pixels,
// then a fixed tree of 256-wide tiles (reference python/dpt/_reductions.py:27-63) reduces
// the partials and one thread rounds the total into its destination, so every sum is
// deterministic for a given pixel count.
//
// Checks of fixed inputs (finite, nonnegative, inside a domain) are separate launches that
// write nothing but the status word, so a checked host call can reject its inputs before any
// output is touched (reference python/dpt/transmission.py:278-305, objectives.py:252-270).
// Status bits: 1 invalid input, 2 an unrepresentable result, 8 a prediction outside the
// Poisson trial domain.
#include <cstdint>
#include <initializer_list>

#include "launch.h"

namespace dpt {
namespace {

constexpr int kTile = 256;                           // threads per block
constexpr int kVec = 4;                              // pixels per vector group
// Vector groups per thread of each kernel: four (16 pixels) for the streaming kernels, fewer
// where FP64 latency or register pressure wants more resident warps instead.
constexpr int kStreamUnroll = 4;
constexpr int kVjpUnroll = 2;
constexpr int kObjectiveUnroll = 1;

__device__ __forceinline__ void flag(int32_t* status, int bits)
{
    if (bits) atomicOr(status, bits);
}

// First pixel of this thread's vector group u (U groups per thread).
template <int U>
__device__ __forceinline__ int64_t group_first(int u)
{
    return (((int64_t)blockIdx.x * U + u) * kTile + threadIdx.x) * kVec;
}

// Streaming loads and stores of one group: one 16-byte access when the group is whole and
// the pointer aligned, else element by element (absent elements read as zero, not stored).
__device__ __forceinline__ void load4(const float* __restrict__ ptr, int64_t p, int64_t count, bool vec, float* v)
{
    if (vec && p + kVec <= count) {
        const float4 x = __ldcs(reinterpret_cast<const float4*>(ptr + p));
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else {
#pragma unroll
        for (int j = 0; j < kVec; ++j) v[j] = p + j < count ? ptr[p + j] : 0.0f;
    }
}

__device__ __forceinline__ void load4(const double* __restrict__ ptr, int64_t p, int64_t count, bool vec, double* v)
{
    if (vec && p + kVec <= count) {
        const double2 a = __ldcs(reinterpret_cast<const double2*>(ptr + p));
        const double2 b = __ldcs(reinterpret_cast<const double2*>(ptr + p + 2));
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else {
#pragma unroll
        for (int j = 0; j < kVec; ++j) v[j] = p + j < count ? ptr[p + j] : 0.0;
    }
}

__device__ __forceinline__ void load4(const uint8_t* __restrict__ ptr, int64_t p, int64_t count, bool vec, uint8_t* v)
{
    if (vec && p + kVec <= count) {
        const uchar4 x = *reinterpret_cast<const uchar4*>(ptr + p);
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else {
#pragma unroll
        for (int j = 0; j < kVec; ++j) v[j] = p + j < count ? ptr[p + j] : 0;
    }
}

__device__ __forceinline__ void store4(float* __restrict__ ptr, int64_t p, int64_t count, bool vec, const float* v)
{
    if (vec && p + kVec <= count) {
        __stcs(reinterpret_cast<float4*>(ptr + p), make_float4(v[0], v[1], v[2], v[3]));
    } else {
#pragma unroll
        for (int j = 0; j < kVec; ++j)
            if (p + j < count) ptr[p + j] = v[j];
    }
}

__device__ __forceinline__ void store4(double* __restrict__ ptr, int64_t p, int64_t count, bool vec, const double* v)
{
    if (vec && p + kVec <= count) {
        __stcs(reinterpret_cast<double2*>(ptr + p), make_double2(v[0], v[1]));
        __stcs(reinterpret_cast<double2*>(ptr + p + 2), make_double2(v[2], v[3]));
    } else {
#pragma unroll
        for (int j = 0; j < kVec; ++j)
            if (p + j < count) ptr[p + j] = v[j];
    }
}

// The thread's kVec U pixels of `ptr` (group u, element j at index kVec u + j).
template <int U, typename T>
__device__ __forceinline__ void load_all(const T* __restrict__ ptr, int64_t count, bool vec, T* v)
{
#pragma unroll
    for (int u = 0; u < U; ++u) load4(ptr, group_first<U>(u), count, vec, v + kVec * u);
}

template <int U, typename T>
__device__ __forceinline__ void store_all(T* __restrict__ ptr, int64_t count, bool vec, const T* v)
{
#pragma unroll
    for (int u = 0; u < U; ++u) store4(ptr, group_first<U>(u), count, vec, v + kVec * u);
}

template <int U>
__device__ __forceinline__ int64_t pixel_at(int k) { return group_first<U>(k / kVec) + k % kVec; }

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
                                                        int rule, int vec, int32_t* status)
{
    constexpr int U = kStreamUnroll, kPixels = kVec * U;
    float v[kPixels];
    load_all<U>(values, count, vec, v);
    bool bad = false;
#pragma unroll
    for (int k = 0; k < kPixels; ++k) {
        bool b = !isfinite(v[k]);
        if (rule != DPT_CHECK_FINITE) b = b || v[k] < 0.0f;
        if (rule == DPT_CHECK_DECREMENT) b = b || v[k] >= 1.0f;
        bad = bad || (b && pixel_at<U>(k) < count);
    }
    if (bad) atomicOr(status, 1);
}

// Forward map (reference get_forward_kernel, kernels/transmission.py:91-144).  Counts are
// formed from the FP64 factor, never from a stored FP32 transmission; -0 results become +0.
__global__ void __launch_bounds__(kTile) k_transmit(const float* __restrict__ depth, int64_t count, int mask,
                                                    int beam_mode, const float* __restrict__ beam,
                                                    float beam_scalar, float* __restrict__ transmission,
                                                    float* __restrict__ counts, float* __restrict__ log_t,
                                                    float* __restrict__ removed, int vec)
{
    constexpr int U = kStreamUnroll, kPixels = kVec * U;
    float L[kPixels], n0[kPixels], out[kPixels];
    load_all<U>(depth, count, vec, L);
    const bool per_pixel = (mask & DPT_OUT_COUNTS) && beam_mode == DPT_BEAM_PER_PIXEL;
    if (per_pixel) load_all<U>(beam, count, vec, n0);
    const float shared = beam_mode == DPT_BEAM_DEVICE_SCALAR && (mask & DPT_OUT_COUNTS) ? beam[0] : beam_scalar;
    if (mask & DPT_OUT_TRANSMISSION) {
#pragma unroll
        for (int k = 0; k < kPixels; ++k) out[k] = (float)transmission_factor(L[k]);
        store_all<U>(transmission, count, vec, out);
    }
    if (mask & DPT_OUT_COUNTS) {
#pragma unroll
        for (int k = 0; k < kPixels; ++k) {
            const float c = (float)((double)(per_pixel ? n0[k] : shared) * transmission_factor(L[k]));
            out[k] = c == 0.0f ? 0.0f : c;
        }
        store_all<U>(counts, count, vec, out);
    }
    if (mask & DPT_OUT_LOG_TRANSMISSION) {
#pragma unroll
        for (int k = 0; k < kPixels; ++k) out[k] = -L[k];
        store_all<U>(log_t, count, vec, out);
    }
    if (mask & DPT_OUT_REMOVED) {
#pragma unroll
        for (int k = 0; k < kPixels; ++k) {
            const float r = removed_primary(L[k]);
            out[k] = r == 0.0f ? 0.0f : r;
        }
        store_all<U>(removed, count, vec, out);
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
// per-pixel beam gradient cN T, and for a shared beam one FP64 partial of sum cN T per block.
// A missing cotangent is zero; `accumulate` adds the destination before the single rounding.
__global__ void __launch_bounds__(kTile) k_transmit_vjp(
    const float* __restrict__ depth, int64_t count, int beam_mode, const float* __restrict__ beam,
    float beam_scalar, const float* __restrict__ seed_t, const float* __restrict__ seed_n,
    const float* __restrict__ seed_log, const float* __restrict__ seed_r, float* __restrict__ grad_depth,
    float* __restrict__ grad_beam, double* __restrict__ beam_partials, int accumulate, int vec, int32_t* status)
{
    constexpr int U = kVjpUnroll, kPixels = kVec * U;
    __shared__ double tree[kTile];
    float L[kPixels], a[kPixels], b[kPixels], c[kPixels], r[kPixels], n0[kPixels], out[kPixels];
    load_all<U>(depth, count, vec, L);
#pragma unroll
    for (int k = 0; k < kPixels; ++k) a[k] = b[k] = c[k] = r[k] = 0.0f;
    if (seed_t) load_all<U>(seed_t, count, vec, a);
    if (seed_n) load_all<U>(seed_n, count, vec, b);
    if (seed_log) load_all<U>(seed_log, count, vec, c);
    if (seed_r) load_all<U>(seed_r, count, vec, r);
    const bool per_pixel = seed_n && grad_depth && beam_mode == DPT_BEAM_PER_PIXEL;
    if (per_pixel) load_all<U>(beam, count, vec, n0);
    const float shared = seed_n && beam_mode == DPT_BEAM_DEVICE_SCALAR ? beam[0] : beam_scalar;
    const bool exponential = seed_t || seed_n || seed_r;
    int bits = 0;
    if (grad_depth) {
        if (accumulate) load_all<U>(grad_depth, count, vec, out);
#pragma unroll
        for (int k = 0; k < kPixels; ++k) {
            // absent cotangents enter as FP64 zeros without a conversion (the XU pipe that
            // converts FP32 to FP64 bounds this kernel)
            const double factor = exponential ? transmission_factor(L[k]) : 0.0;
            const double ak = seed_t ? (double)a[k] : 0.0, bk = seed_n ? (double)b[k] : 0.0;
            const double ck = seed_log ? (double)c[k] : 0.0, rk = seed_r ? (double)r[k] : 0.0;
            const double beam_k = seed_n ? (double)(per_pixel ? n0[k] : shared) : 0.0;
            const double optical = (rk - ak) * factor;
            double derivative = fma(-(bk * beam_k), factor, optical) - ck;
            if (accumulate) derivative += (double)out[k];
            const float rounded = (float)derivative;
            if (!isfinite(rounded) && pixel_at<U>(k) < count) bits |= 2;
            out[k] = rounded;
        }
        store_all<U>(grad_depth, count, vec, out);
    }
    if (grad_beam) {
        if (accumulate) load_all<U>(grad_beam, count, vec, out);
#pragma unroll
        for (int k = 0; k < kPixels; ++k) {
            double derivative = (double)b[k] * (exponential ? transmission_factor(L[k]) : 0.0);
            if (accumulate) derivative += (double)out[k];
            const float rounded = (float)derivative;
            if (!isfinite(rounded) && pixel_at<U>(k) < count) bits |= 2;
            out[k] = rounded;
        }
        store_all<U>(grad_beam, count, vec, out);
    }
    if (beam_partials) {
        double sum = 0.0;
#pragma unroll
        for (int k = 0; k < kPixels; ++k) sum += pixel_at<U>(k) < count ? (double)b[k] * transmission_factor(L[k]) : 0.0;
        const double total = tile_sum(sum, tree);
        if (threadIdx.x == 0) beam_partials[blockIdx.x] = total;
    }
    flag(status, bits);
}

__global__ void __launch_bounds__(kTile) k_depth_from_removed(const float* __restrict__ decrement,
                                                              int64_t count, float* __restrict__ depth, int vec)
{
    constexpr int U = kStreamUnroll, kPixels = kVec * U;
    float v[kPixels];
    load_all<U>(decrement, count, vec, v);
#pragma unroll
    for (int k = 0; k < kPixels; ++k) {
        const float L = depth_from_decrement(v[k]);
        v[k] = L == 0.0f ? 0.0f : L;
    }
    store_all<U>(depth, count, vec, v);
}

// d/d delta of -log(1 - delta) is 1 / (1 - delta) (reference get_inverse_vjp_kernel).
__global__ void __launch_bounds__(kTile) k_depth_from_removed_vjp(const float* __restrict__ decrement,
                                                                  const float* __restrict__ seed,
                                                                  int64_t count, float* __restrict__ grad,
                                                                  int accumulate, int vec, int32_t* status)
{
    constexpr int U = kStreamUnroll, kPixels = kVec * U;
    float d[kPixels], s[kPixels], out[kPixels];
    load_all<U>(decrement, count, vec, d);
    load_all<U>(seed, count, vec, s);
    if (accumulate) load_all<U>(grad, count, vec, out);
    int bits = 0;
#pragma unroll
    for (int k = 0; k < kPixels; ++k) {
        double derivative = (double)s[k] / (1.0 - (double)d[k]);
        if (accumulate) derivative += (double)out[k];
        const float rounded = (float)derivative;
        if (!isfinite(rounded) && pixel_at<U>(k) < count) bits |= 2;
        out[k] = rounded;
    }
    store_all<U>(grad, count, vec, out);
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
                                                           int poisson, int integer_counts, int vec, int32_t* status)
{
    constexpr int U = kStreamUnroll, kPixels = kVec * U;
    T mu[kPixels];
    float y[kPixels], w[kPixels];
    uint8_t m[kPixels];
    load_all<U>(observation, count, vec, y);
    if (prediction) load_all<U>(prediction, count, vec, mu);
    if (weights) load_all<U>(weights, count, vec, w);
    if (valid) load_all<U>(valid, count, vec, m);
    int bits = 0;
#pragma unroll
    for (int k = 0; k < kPixels; ++k) {
        if (pixel_at<U>(k) >= count) continue;
        bool active = true;
        if (valid) {
            if (m[k] > 1) bits |= 1;
            active = m[k] == 1;
        }
        if (!active) continue;
        bool invalid = !isfinite(y[k]);
        if (poisson) {
            invalid = invalid || y[k] < 0.0f;
            if (integer_counts) invalid = invalid || floorf(y[k]) != y[k];
        }
        if (weights) invalid = invalid || !isfinite(w[k]) || w[k] < 0.0f;
        if (invalid) bits |= 1;
        if (prediction) {
            if (!isfinite(mu[k]))
                bits |= 2;
            else if (poisson && (mu[k] < (T)0 || (mu[k] == (T)0 && y[k] > 0.0f)))
                bits |= 8;
        }
    }
    flag(status, bits);
}

// Objective terms and the image-space seed (reference evaluation_kernel,
// kernels/objectives.py:133-211).  kind: half squared error or Poisson half-deviance; each
// active pixel's loss is weighted by normalisation x weights[p] and summed per block into
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
                                                     int vec, int32_t* status)
{
    constexpr int U = kObjectiveUnroll, kPixels = kVec * U;
    __shared__ double tree[kTile];
    TIn mu[kPixels];
    float y[kPixels], w[kPixels];
    uint8_t m[kPixels];
    TOut out[kPixels];
    load_all<U>(prediction, count, vec, mu);
    load_all<U>(observation, count, vec, y);
    if (weights) load_all<U>(weights, count, vec, w);
    if (valid) load_all<U>(valid, count, vec, m);
    double sum = 0.0;
    int bits = 0;
#pragma unroll
    for (int k = 0; k < kPixels; ++k) {
        double loss = 0.0;
        out[k] = (TOut)0.0;
        if (pixel_at<U>(k) < count && (!valid || m[k] == 1)) {
            const double predicted = (double)mu[k];
            if (!isfinite(predicted))
                bits |= 2;
            else if (poisson && predicted < 0.0)
                bits |= 8;
            const double observed = (double)y[k];
            double weight = normalisation;
            if (weights) weight *= (double)w[k];
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
                out[k] = (TOut)(weighted * seed_scale);
                if (!isfinite((double)out[k])) bits |= 2;
            }
        }
        if (valid && pixel_at<U>(k) < count && m[k] > 1) bits |= 1;
        sum += loss;
    }
    if (seed) store_all<U>(seed, count, vec, out);
    if (partials) {
        const double total = tile_sum(sum, tree);
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

// Blocks of a pixel kernel with U groups per thread (1024 U pixels each): also its
// first-level partial count.
template <int U>
int64_t blocks_for(int64_t count)
{
    constexpr int64_t pixels = (int64_t)kTile * kVec * U;
    return (count + pixels - 1) / pixels;
}

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

// Vector accesses need every array 16-byte aligned (the uint8 mask 4-byte aligned).
bool aligned(std::initializer_list<const void*> pointers, const void* mask = nullptr)
{
    for (const void* ptr : pointers)
        if (ptr && reinterpret_cast<uintptr_t>(ptr) % 16) return false;
    return !mask || reinterpret_cast<uintptr_t>(mask) % 4 == 0;
}

int launched() { return (int)cudaGetLastError(); }

}  // namespace
}  // namespace dpt

using dpt::kTile;

extern "C" {

size_t dpt_b200_reduction_bytes(int64_t count)
{
    if (count < 0) return 0;
    // covers both a pixel kernel's partials and its tree, and a tree over `count` rows
    const int64_t first = count ? dpt::tiles(count) : 0;
    return (size_t)(first + dpt::tree_rows(first) + 1) * sizeof(double);
}

int dpt_b200_check_values(const float* values, int64_t count, int32_t rule, int32_t* status, void* stream)
{
    if (count < 0 || count > INT32_MAX) return DPT_E_SHAPE;
    if (rule < DPT_CHECK_FINITE_NONNEGATIVE || rule > DPT_CHECK_DECREMENT) return DPT_E_FLAGS;
    if (!status || (count && !values)) return DPT_E_NULL;
    if (!count) return DPT_OK;
    dpt::k_check_values<<<(unsigned)dpt::blocks_for<dpt::kStreamUnroll>(count), kTile, 0, static_cast<cudaStream_t>(stream)>>>(
        values, count, rule, dpt::aligned({values}), status);
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
    const float* pixel_beam = (mask & DPT_OUT_COUNTS) && beam_mode == DPT_BEAM_PER_PIXEL ? beam : nullptr;
    const bool vec = dpt::aligned({depth, pixel_beam, transmission, counts, log_transmission, removed});
    dpt::k_transmit<<<(unsigned)dpt::blocks_for<dpt::kStreamUnroll>(count), kTile, 0, static_cast<cudaStream_t>(stream)>>>(
        depth, count, mask, beam_mode, beam, beam_scalar, transmission, counts, log_transmission, removed, vec);
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
        const float* pixel_beam = beam_mode == DPT_BEAM_PER_PIXEL ? beam : nullptr;
        const bool vec = dpt::aligned({depth, pixel_beam, seed_transmission, seed_counts, seed_log_transmission,
                                       seed_removed, grad_depth, per_pixel ? grad_beam : nullptr});
        dpt::k_transmit_vjp<<<(unsigned)dpt::blocks_for<dpt::kVjpUnroll>(count), kTile, 0, s>>>(
            depth, count, beam_mode, beam, beam_scalar, seed_transmission, seed_counts, seed_log_transmission,
            seed_removed, grad_depth, per_pixel ? grad_beam : nullptr, partials ? scratch : nullptr, accumulate,
            vec, status);
    }
    if (shared) {
        const int64_t rows = partials ? dpt::blocks_for<dpt::kVjpUnroll>(count) : 0;
        dpt::finish_tree<float>(scratch, rows, scratch + rows, grad_beam, accumulate, status, s);
    }
    return dpt::launched();
}

int dpt_b200_depth_from_removed(const float* removed, int64_t count, float* depth, void* stream)
{
    if (count < 0 || count > INT32_MAX) return DPT_E_SHAPE;
    if (count && (!removed || !depth)) return DPT_E_NULL;
    if (!count) return DPT_OK;
    dpt::k_depth_from_removed<<<(unsigned)dpt::blocks_for<dpt::kStreamUnroll>(count), kTile, 0, static_cast<cudaStream_t>(stream)>>>(
        removed, count, depth, dpt::aligned({removed, depth}));
    return dpt::launched();
}

int dpt_b200_depth_from_removed_vjp(const float* removed, const float* seed, int64_t count, float* grad,
                                    int32_t accumulate, int32_t* status, void* stream)
{
    if (count < 0 || count > INT32_MAX) return DPT_E_SHAPE;
    if (!status || (count && (!removed || !seed || !grad))) return DPT_E_NULL;
    if (!count) return DPT_OK;
    dpt::k_depth_from_removed_vjp<<<(unsigned)dpt::blocks_for<dpt::kStreamUnroll>(count), kTile, 0,
                                    static_cast<cudaStream_t>(stream)>>>(
        removed, seed, count, grad, accumulate, dpt::aligned({removed, seed, grad}), status);
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
    const unsigned blocks = (unsigned)dpt::blocks_for<dpt::kStreamUnroll>(count);
    const int poisson = kind == DPT_OBJECTIVE_POISSON;
    const bool vec = dpt::aligned({prediction, observation, weights}, valid);
    if (prediction_dtype == DPT_F64)
        dpt::k_objective_check<double><<<blocks, kTile, 0, s>>>(static_cast<const double*>(prediction),
                                                                observation, weights, valid, count, poisson,
                                                                integer_counts, vec, status);
    else
        dpt::k_objective_check<float><<<blocks, kTile, 0, s>>>(static_cast<const float*>(prediction),
                                                               observation, weights, valid, count, poisson,
                                                               integer_counts, vec, status);
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
    const int64_t blocks = dpt::blocks_for<dpt::kObjectiveUnroll>(count);
    if (count) {
        const bool vec = dpt::aligned({prediction, observation, weights, seed}, valid);
        if (prediction_dtype == DPT_F64)
            dpt::k_objective<double, double, true><<<(unsigned)blocks, kTile, 0, s>>>(
                static_cast<const double*>(prediction), observation, weights, valid, count, poisson, normalisation,
                seed_scale, static_cast<double*>(seed), partials, vec, status);
        else if (wide)
            dpt::k_objective<float, float, true><<<(unsigned)blocks, kTile, 0, s>>>(
                static_cast<const float*>(prediction), observation, weights, valid, count, poisson, normalisation,
                seed_scale, static_cast<float*>(seed), partials, vec, status);
        else
            dpt::k_objective<float, float, false><<<(unsigned)blocks, kTile, 0, s>>>(
                static_cast<const float*>(prediction), observation, weights, valid, count, poisson, normalisation,
                seed_scale, static_cast<float*>(seed), partials, vec, status);
    }
    if (loss) dpt::finish_tree<double>(scratch, blocks, scratch + blocks, loss, 0, status, s);
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
