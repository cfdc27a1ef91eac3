// vjp.cu - discrete VJP of the projector: volume cotangent and rigid-pose cotangent.
//
// Samples are recomputed exactly as in the forward (no per-sample state is stored).
//
// Volume: while consecutive samples of a ray stay in one interpolation cell their eight
// corner increments accumulate in registers (the cell-run aggregation of the reference,
// python/dpt/kernels/projection_fp32.py:459-548); when the ray leaves the cell the eight
// sums go to a per-cell accumulator record of 32 bytes with two 16-byte vector reductions
// (red.global.add.v4.f32) instead of eight scalar atomics.  The fold kernel (reduce.cu)
// later gathers each voxel's corner slots, so the accumulator needs no atomics on voxels
// shared by neighbouring cells.
//
// Pose: per ray the moments of the reference (mean, sum grad, sum t grad, the two clip
// shifts) are accumulated in the sample arithmetic, chained through the clip-face
// derivatives and M^T in FP64 (python/dpt/kernels/projection_fp32.py:549-602,
// python/dpt/kernels/projection.py:1140-1217), then reduced per block with a fixed
// warp-shuffle tree into FP64 partials that finish_pose reduces per view.
#include <type_traits>

#include "launch.h"

// DPT_VJP_REUSE=1 keeps the last cell's values across samples (fewer loads, one more branch
// per sample: 3% slower measured).
#ifndef DPT_VJP_REUSE
#define DPT_VJP_REUSE 0
#endif
// Resident blocks per SM the register allocation must allow, per arithmetic (128-thread
// blocks).  The kernels are latency bound, so occupancy pays for a few spilled registers:
// the compensated form's cell walk measured 0.71 ms per 512^2 view (S = 1024) at four
// blocks (118 registers), 0.59 at eight (64 registers, 376 bytes spilled to L1); the FP32
// form 1.17 ms at five blocks (96 registers), 1.15 at six (80 registers, 12 bytes spilled).
#ifndef DPT_VJP_MIN_BLOCKS_F32
#define DPT_VJP_MIN_BLOCKS_F32 6
#endif
#ifndef DPT_VJP_MIN_BLOCKS_F32C
#define DPT_VJP_MIN_BLOCKS_F32C 8
#endif
// FP32 pose moments: alpha_i = (i + 0.5) / S as one multiplication by 1/S when S is a power
// of two (both exact), else from a per-block table of IEEE quotients
#ifndef DPT_VJP_POW2_ALPHA
#define DPT_VJP_POW2_ALPHA 1
#endif
// The compensated form's forward that stores the pose moments (no scatter) measured 158.6 ->
// 153.4 ms per 360-view full scan at nine blocks (56 registers), 155.4 at ten.
#ifndef DPT_VJP_MIN_BLOCKS_F32C_FORWARD
#define DPT_VJP_MIN_BLOCKS_F32C_FORWARD 9
#endif
// The compensated joint volume + pose pass: 237.9 ms per full scan at eight blocks (64
// registers, 376 bytes spilled), 247.3 at seven, 252.6 at six, 249.7 at nine, 310.3 at ten.
#ifndef DPT_VJP_MIN_BLOCKS_F32C_JOINT
#define DPT_VJP_MIN_BLOCKS_F32C_JOINT 8
#endif
// The FP32 forward that stores the pose moments: 289.1 ms per full scan at six blocks (80
// registers, 84 bytes spilled), 289.5 at five (88 registers, none spilled), 316.0 at seven;
// the occupancy does not matter where the FP32 pipe binds.
#ifndef DPT_VJP_MIN_BLOCKS_F32_MOMENTS
#define DPT_VJP_MIN_BLOCKS_F32_MOMENTS 6
#endif
// Strict FP64: the full-scan joint VJP (launches of two views) measured 86.7 ms per 32 views
// at three blocks (160 registers), 84.3 at four (128, 68 bytes spilled), 83.2 at five (96,
// 376 bytes spilled to L1).  The cell-Gauss joint VJP: 61.5 ms per 32 views at three blocks,
// 59.3 at four, 66.0 at five.  The mixed and fast forms keep three.
#ifndef DPT_VJP_MIN_BLOCKS_F64
#define DPT_VJP_MIN_BLOCKS_F64 5
#endif
#ifndef DPT_VJP_MIN_BLOCKS_CELLS
#define DPT_VJP_MIN_BLOCKS_CELLS 4
#endif
#ifndef DPT_VJP_MIN_BLOCKS_FP64_OTHER
#define DPT_VJP_MIN_BLOCKS_FP64_OTHER 3
#endif

namespace dpt {
namespace {

// whether the VJP keeps the last cell's values across samples (CellCache / PolyCache kReuse)
constexpr bool kVjpReuse = DPT_VJP_REUSE != 0;

constexpr int kAlphaTable = 2048;

__device__ __forceinline__ void flush_cell(float* acc, int cell, const float* cs)
{
    float* slot = acc + 8 * (int64_t)cell;
    red_add_v4(slot, cs[0], cs[1], cs[2], cs[3]);
    red_add_v4(slot + 4, cs[4], cs[5], cs[6], cs[7]);
}

// Pose outputs from the source/direction adjoints (FP64).
//   mode 12: packed rows d L / d R[row][col] = wsr[row] sa[col] + wd[row] da[col] and
//            d L / d t = -(R sa)   (reference kernels/projection_fp32.py:584-593)
//   mode 6 / -6: local-right tangent (-sa, sa x os + da x od)  (reference kernels/geometry.py:24-52)
__device__ __forceinline__ void pose_rows(int mode, const Ray64& r, const double* pose,
                                          const double* sa, const double* da, double* g)
{
    if (mode == 12) {
#pragma unroll
        for (int row = 0; row < 3; ++row)
#pragma unroll
            for (int col = 0; col < 3; ++col)
                g[3 * row + col] = fma(r.wd[row], da[col], r.wsr[row] * sa[col]);
        double t[3];
        matvec(pose, sa, t);
#pragma unroll
        for (int k = 0; k < 3; ++k) g[9 + k] = -t[k];
    } else {
        const double* os = r.os;
        const double* od = r.od;
        g[0] = -sa[0];
        g[1] = -sa[1];
        g[2] = -sa[2];
        g[3] = fma(-da[2], od[1], da[1] * od[2]) + fma(-sa[2], os[1], sa[1] * os[2]);
        g[4] = fma(-da[0], od[2], da[2] * od[0]) + fma(-sa[0], os[2], sa[2] * os[0]);
        g[5] = fma(-da[1], od[0], da[0] * od[1]) + fma(-sa[1], os[0], sa[0] * os[1]);
    }
}

// Pose epilogue: recompute the FP64 ray of `pixel` (a few hundred FP64 operations once per
// ray) instead of keeping its 24 registers alive across the sample loop, then form the rows.
// The empty asm with a memory clobber makes the compiler reload the view record from shared
// memory here, so the recomputation cannot be folded into the pre-loop ray setup.
__device__ __forceinline__ void pose_epilogue(const RayArgs& a, const ViewShared& vs, int view, int pixel,
                                           int mode, const double* sa, const double* da, double* g)
{
    asm volatile("" ::: "memory");
    double source[3], end[3];
    ray_endpoints(a, vs.table, view, pixel, source, end);
    Ray64 r;
    ray_setup(a.grid, vs.pose, source, end, r);
    pose_rows(mode, r, vs.pose, sa, da, g);
}

// Split pose VJP (FP32 arithmetic).  The pose moments of a ray (mean, sum of slopes, sum of
// position-weighted slopes and the two clip shifts) do not depend on its cotangent, so a
// training step can gather them during its forward pass (kStoreMoments: the kernel samples
// once, writes the image and the nine moments and no gradient) and finish the pose VJP
// without sampling (kLoadMoments: read the moments, apply the cotangent and the clip-face
// chain); the volume VJP then runs alone.  The moments are the same FP32 values the joint
// kernel forms, so every result is unchanged.
constexpr int kJointMoments = 0, kStoreMoments = 1, kLoadMoments = 2;
// FP32: mean, dO[3], dD[3], shift_lower, shift_upper; compensated: the mean's sum and
// compensation, G[3], H[3] and whether H is the cell-run sum (to divide by S) or already
// alpha-weighted (per-sample form)
constexpr int kMomentWords = 9;

struct MomentArgs {
    float* moments;  // kMomentWords x stride FP32, word k of ray r at k * stride + r
    int64_t stride;  // rays of the call
    float* image;    // kStoreMoments: the forward image (FP32)
};

// kPow2: nx and ny are powers of two, so the interior pairs form their flat cell index with
// shifts (integer pipe) instead of two multiply-adds on the FP32 pipe, which binds the
// moment-storing forward (full scan at 256^3: 289.0 -> 283.7 ms, the same values).
template <int kArith, class Field, bool kVol, bool kPose, typename Seed, int kMoments = kJointMoments,
          bool kPow2 = false>
__global__ void __launch_bounds__(kVjpBlock, kArith == DPT_ARITH_F32C
                                                  ? (kMoments == kStoreMoments ? DPT_VJP_MIN_BLOCKS_F32C_FORWARD
                                                     : (kVol && kPose)             ? DPT_VJP_MIN_BLOCKS_F32C_JOINT
                                                                                   : DPT_VJP_MIN_BLOCKS_F32C)
                                                  : kArith == DPT_ARITH_F32 ? (kMoments == kStoreMoments ? DPT_VJP_MIN_BLOCKS_F32_MOMENTS
                                                                                                         : DPT_VJP_MIN_BLOCKS_F32)
                                                  : kArith == DPT_ARITH_F64   ? DPT_VJP_MIN_BLOCKS_F64
                                                  : kArith == DPT_ARITH_CELLS ? DPT_VJP_MIN_BLOCKS_CELLS
                                                                              : DPT_VJP_MIN_BLOCKS_FP64_OTHER)
    k_vjp(RayArgs a, Field f, const Seed* __restrict__ cot,
                                                int mode, float* __restrict__ acc,
                                                double* __restrict__ partials, MomentArgs ma)
{
    static_assert(kMoments == kJointMoments ||
                      ((kArith == DPT_ARITH_F32 || kArith == DPT_ARITH_F32C) && !kVol && kPose),
                  "split pose moments: FP32 or compensated arithmetic, pose only");
    __shared__ ViewShared vs;
    __shared__ double warp_sums[kVjpBlock / 32][12];
    __shared__ float4 run_sums[kArith == DPT_ARITH_F32C && kMoments != kLoadMoments ? kRunSumTable + 1 : 1];
    if (kArith == DPT_ARITH_F32C && kMoments != kLoadMoments) fill_run_sums(run_sums);
    // alpha_i = (i + 0.5) / S of the FP32 pose moments, each one IEEE division, tabulated
    // once per block for the first kAlphaTable samples (later samples divide directly)
    __shared__ float alpha_table[kArith == DPT_ARITH_F32 && kPose && kMoments != kLoadMoments ? kAlphaTable : 1];
    // one cell run's sums into its 32-byte accumulator record
    auto flush_run = [&](int cell, const float* sums) { flush_cell(acc, cell, sums); };
    int view_local, tile;
    block_work(a, &view_local, &tile);
    const int view = a.view_begin + view_local;
    if (kArith == DPT_ARITH_F32 && kPose && kMoments != kLoadMoments) {
        const int n = min(a.samples, kAlphaTable);
        for (int k = threadIdx.x; k < n; k += kVjpBlock) alpha_table[k] = ((float)k + 0.5f) / (float)a.samples;
    }
    stage_view(a, view, vs);
    int pixel;
    const bool active = ray_of_thread(a, tile, &pixel);
    const int64_t rays_per_view = (int64_t)a.rows * a.cols;
    const int S = a.samples;
    double g[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) g[k] = 0.0;
    int bits = 0;
    float stored[kMoments == kStoreMoments ? kMomentWords : 1] = {};
    float stored_image = 0.0f;

    if (active) {
        double source[3], end[3];
        ray_endpoints(a, vs.table, view, pixel, source, end);
        Ray64 r;
        ray_setup(a.grid, vs.pose, source, end, r);
        const int64_t ray_index = view_local * rays_per_view + pixel;
        // a forward pass that stores moments has no cotangent yet: sample as for a unit seed
        const double seed_in = kMoments == kStoreMoments ? 1.0 : (double)cot[ray_index];
        FieldDims dims;
        dims.init(a.grid);

        if constexpr (kArith == DPT_ARITH_F32) {
            const float o[3] = {(float)r.origin[0], (float)r.origin[1], (float)r.origin[2]};
            const float d[3] = {(float)r.direction[0], (float)r.direction[1], (float)r.direction[2]};
            const float length = (float)r.length;
            if (!valid_ray(r) || !finite3f(o[0], o[1], o[2]) || !finite3f(d[0], d[1], d[2]) ||
                !isfinite(length) || length <= 0.0f) {
                bits = 2;
            } else {
                Interval<float> iv;
                iv.clip(o, d, dims.nx, dims.ny, dims.nz);
                const float span = iv.upper - iv.lower;
                const float seed = (float)seed_in;
                if (!isfinite(seed)) bits |= 2;
                if (span > 0.0f && seed != 0.0f) {
                    const float step = span / (float)S;
                    const float physical_step = length * step;
                    const float vf = seed * physical_step;
                    const bool bounded = isfinite(vf) && fabsf(vf) <= 1.0f;
                    float mean = 0.0f, dO[3] = {0.0f, 0.0f, 0.0f}, dD[3] = {0.0f, 0.0f, 0.0f};
                    float sl = 0.0f, su = 0.0f;
                    bool trailing_zero = false;
                    float cs[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c) cs[c] = 0.0f;
                    int pending = -1;
                    CellCache<Field, kVjpReuse> cache;
                    auto position_at = [&](int i) { return fmaf((float)i + 0.5f, step, iv.lower); };
                    const int shift_x = kPow2 ? __ffs(dims.nx) - 1 : 0, shift_y = kPow2 ? __ffs(dims.ny) - 1 : 0;
                    const float inverse_samples = 1.0f / (float)S;
                    // One midpoint.  mode 0: general (support and finiteness tested); 1: on the
                    // inside run (both known to pass); 2: on the interior run (no clamp active,
                    // slope masks 1).
                    // `bounded` (every increment finite and at most 1 in magnitude) is fixed
                    // per ray: the march is instantiated for both values so the sample loop
                    // carries no test of it
                    auto visit = [&](int i, int mode, auto bounded_tag, auto pow2_tag) {
                        constexpr bool kBounded = decltype(bounded_tag)::value;
                        const bool known_inside = mode > 0;
                        const float position = position_at(i);
                        const float x = fmaf(position, d[0], o[0]);
                        const float y = fmaf(position, d[1], o[1]);
                        const float z = fmaf(position, d[2], o[2]);
                        bool in = true;
                        if (!known_inside) {
                            if (!finite3f(x, y, z)) bits |= 2;
                            in = inside(x, y, z, dims.hx, dims.hy, dims.hz);
                        }
                        Axis32 X{0, 0.0f}, Y{0, 0.0f}, Z{0, 0.0f};
                        float w[8];
                        int cell = -1;
                        if (mode == 2) {
                            X = interior_axis(x);
                            Y = interior_axis(y);
                            Z = interior_axis(z);
                        } else if (in) {
                            X = axis32(x, dims.mx, dims.cx);
                            Y = axis32(y, dims.my, dims.cy);
                            Z = axis32(z, dims.mz, dims.cz);
                        }
                        if (in) {
                            corner_weights(X.fraction, Y.fraction, Z.fraction, w);
                            cell = (Z.lower * dims.ny + Y.lower) * dims.nx + X.lower;
                        }
                        if (kPose) {
                            float value = 0.0f, gs[3] = {0.0f, 0.0f, 0.0f};
                            if (in) {
                                cache.fetch(f, X.lower, Y.lower, Z.lower, cell);
                                value = interpolate(w, cache.v);
                                const bool core = mode == 2;
                                const float sx = (core || (x >= 0.0f && x < dims.mx)) ? 1.0f : 0.0f;
                                const float sy = (core || (y >= 0.0f && y < dims.my)) ? 1.0f : 0.0f;
                                const float sz = (core || (z >= 0.0f && z < dims.mz)) ? 1.0f : 0.0f;
                                slope32(X.fraction, Y.fraction, Z.fraction, cache.v, sx, sy, sz, gs);
                            }
                            mean = mean + value;
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                dO[k] = dO[k] + gs[k];
                                dD[k] = fmaf(position, gs[k], dD[k]);
                            }
                            // S a power of two: (i + 0.5) / S is exact, and so is the product
                            // with the exact reciprocal
                            float alpha;
                            if constexpr (decltype(pow2_tag)::value)
                                alpha = ((float)i + 0.5f) * inverse_samples;
                            else
                                alpha = i < kAlphaTable ? alpha_table[i] : ((float)i + 0.5f) / (float)S;
                            const float along = fmaf(gs[2], d[2], fmaf(gs[1], d[1], gs[0] * d[0]));
                            sl = fmaf(1.0f - alpha, along, sl);
                            su = fmaf(alpha, along, su);
                        }
                        if (kVol) {
                            if (in) {
                                if constexpr (kBounded) {
                                    // a run's first increments start its sums (0 + x differs
                                    // from x only for x = -0, and a -0 run sum leaves the
                                    // +0-initialised accumulator slot exactly as +0 does):
                                    // 234.8 ms per full-scan volume pass, 235.9 with zeroing
                                    if (cell != pending) {
                                        if (pending >= 0) flush_run(pending, cs);
                                        pending = cell;
#pragma unroll
                                        for (int c = 0; c < 8; ++c) cs[c] = mul_ftz(vf, w[c]);
                                    } else {
#pragma unroll
                                        for (int c = 0; c < 8; ++c) cs[c] = cs[c] + mul_ftz(vf, w[c]);
                                    }
                                } else {
                                    // increments that may be non-finite or large: each one is
                                    // checked, and a sum that would overflow is flushed first
                                    if (cell != pending) {
                                        if (pending >= 0) flush_run(pending, cs);
#pragma unroll
                                        for (int c = 0; c < 8; ++c) cs[c] = 0.0f;
                                        pending = cell;
                                    }
                                    float* slot = acc + 8 * (int64_t)cell;
#pragma unroll
                                    for (int c = 0; c < 8; ++c) {
                                        const float inc = scatter_increment(vf, w[c]);
                                        if (!isfinite(inc)) {
                                            bits |= 2;
                                            atomicAdd(slot + c, inc);
                                        } else {
                                            const float partial = cs[c] + inc;
                                            if (!isfinite(partial)) {
                                                atomicAdd(slot + c, cs[c]);
                                                cs[c] = inc;
                                            } else {
                                                cs[c] = partial;
                                            }
                                        }
                                    }
                                }
                            } else if (pending >= 0) {
                                flush_run(pending, cs);
#pragma unroll
                                for (int c = 0; c < 8; ++c) cs[c] = 0.0f;
                                pending = -1;
                            }
                        }
                    };
                    // Samples i and i + 1 of the interior run, lane-wise where the arithmetic is
                    // (see "packed FP32 pairs" in common.cuh); the serial sums take sample i,
                    // then sample i + 1, so every moment, increment and run sum is the value
                    // the two visits of mode 2 form.  `ip` holds (i + 0.5, i + 1.5).
                    auto visit_pair = [&](int i, f32x2 ip, auto bounded_tag, auto pow2_tag) {
                        (void)bounded_tag;
                        const f32x2 position = fma2(ip, splat2(step), splat2(iv.lower));
                        const f32x2 x = fma2(position, splat2(d[0]), splat2(o[0]));
                        const f32x2 y = fma2(position, splat2(d[1]), splat2(o[1]));
                        const f32x2 z = fma2(position, splat2(d[2]), splat2(o[2]));
                        f32x2 bx, by, bz;
                        const f32x2 fx = interior_fraction2(x, &bx);
                        const f32x2 fy = interior_fraction2(y, &by);
                        const f32x2 fz = interior_fraction2(z, &bz);
                        f32x2 w[8], ax, ay, az;
                        corner_weights2(fx, fy, fz, w, &ax, &ay, &az);
                        const int lx0 = biased_lo(bx), ly0 = biased_lo(by), lz0 = biased_lo(bz);
                        const int lx1 = biased_hi(bx), ly1 = biased_hi(by), lz1 = biased_hi(bz);
                        int cell0, cell1;
                        if constexpr (kPow2) {
                            cell0 = (((lz0 << shift_y) + ly0) << shift_x) + lx0;
                            cell1 = (((lz1 << shift_y) + ly1) << shift_x) + lx1;
                        } else {
                            cell0 = (lz0 * dims.ny + ly0) * dims.nx + lx0;
                            cell1 = (lz1 * dims.ny + ly1) * dims.nx + lx1;
                        }
                        if (kPose) {
                            float u[8], v[8];
                            f.load_at(cell0, lx0, ly0, lz0, u);
                            f.load_at(cell1, lx1, ly1, lz1, v);
                            float wu[8], wv[8];
#pragma unroll
                            for (int c = 0; c < 8; ++c) {
                                wu[c] = lo2(w[c]);
                                wv[c] = hi2(w[c]);
                            }
                            const float value0 = interpolate(wu, u), value1 = interpolate(wv, v);
                            f32x2 gs[3];
                            slope2(fx, fy, fz, ax, ay, az, u, v, gs);
                            mean = mean + value0;
                            mean = mean + value1;
                            const float p0 = lo2(position), p1 = hi2(position);
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                dO[k] = dO[k] + lo2(gs[k]);
                                dO[k] = dO[k] + hi2(gs[k]);
                                dD[k] = fmaf(p0, lo2(gs[k]), dD[k]);
                                dD[k] = fmaf(p1, hi2(gs[k]), dD[k]);
                            }
                            f32x2 alpha;
                            if constexpr (decltype(pow2_tag)::value)
                                alpha = mul2(ip, splat2(inverse_samples));
                            else
                                alpha = pack2(i < kAlphaTable ? alpha_table[i] : ((float)i + 0.5f) / (float)S,
                                              i + 1 < kAlphaTable ? alpha_table[i + 1] : ((float)i + 1.5f) / (float)S);
                            const f32x2 along = fma2(gs[2], splat2(d[2]), fma2(gs[1], splat2(d[1]), mul2(gs[0], splat2(d[0]))));
                            const f32x2 rest = sub2(splat2(1.0f), alpha);
                            sl = fmaf(lo2(rest), lo2(along), sl);
                            sl = fmaf(hi2(rest), hi2(along), sl);
                            su = fmaf(lo2(alpha), lo2(along), su);
                            su = fmaf(hi2(alpha), hi2(along), su);
                        }
                        if (kVol) {
                            // bounded increments only (the pair loop runs for bounded rays)
                            f32x2 inc[8];
#pragma unroll
                            for (int c = 0; c < 8; ++c) inc[c] = mul_ftz2(splat2(vf), w[c]);
                            if (cell0 != pending) {
                                if (pending >= 0) flush_run(pending, cs);
                                pending = cell0;
#pragma unroll
                                for (int c = 0; c < 8; ++c) cs[c] = lo2(inc[c]);
                            } else {
#pragma unroll
                                for (int c = 0; c < 8; ++c) cs[c] = cs[c] + lo2(inc[c]);
                            }
                            if (cell1 != pending) {
                                flush_run(pending, cs);
                                pending = cell1;
#pragma unroll
                                for (int c = 0; c < 8; ++c) cs[c] = hi2(inc[c]);
                            } else {
#pragma unroll
                                for (int c = 0; c < 8; ++c) cs[c] = cs[c] + hi2(inc[c]);
                            }
                        }
                    };
                    auto march = [&](auto bounded_tag, auto pow2_tag) {
                    if (!moderate(o, d)) {
                        for (int i = 0; i < S; ++i) visit(i, 0, bounded_tag, pow2_tag);
                    } else {
                        // samples outside the inside run add exact zeros to every moment
                        int first, last;
                        inside_run(S, [&](int i) {
                            const float position = position_at(i);
                            return inside(fmaf(position, d[0], o[0]), fmaf(position, d[1], o[1]),
                                          fmaf(position, d[2], o[2]), dims.hx, dims.hy, dims.hz);
                        }, first, last);
                        int ifirst, ilast;
                        interior_run(first, last, [&](int i) {
                            const float position = position_at(i);
                            const float x = fmaf(position, d[0], o[0]), y = fmaf(position, d[1], o[1]),
                                        z = fmaf(position, d[2], o[2]);
                            return x >= 0.0f && x < dims.mx && y >= 0.0f && y < dims.my && z >= 0.0f && z < dims.mz;
                        }, ifirst, ilast);
                        const int split = min(ifirst, last + 1);
                        for (int i = first; i < split; ++i) visit(i, 1, bounded_tag, pow2_tag);
                        int i = ifirst;
                        // the pair floors need interior coordinates below 2^23, and the pair
                        // scatter bounded increments
                        if (dims.packed && (!kVol || decltype(bounded_tag)::value)) {
                            f32x2 ip = pack2((float)i + 0.5f, (float)i + 1.5f);
                            for (; i + 1 <= ilast; i += 2) {
                                visit_pair(i, ip, bounded_tag, pow2_tag);
                                ip = add2(ip, splat2(2.0f));
                            }
                        }
                        for (; i <= ilast; ++i) visit(i, 2, bounded_tag, pow2_tag);
                        for (int i = max(ilast + 1, split); i <= last; ++i) visit(i, 1, bounded_tag, pow2_tag);
                        trailing_zero = last < S - 1;
                    }
                    };
                    if constexpr (kMoments == kLoadMoments) {
                        const float* m = ma.moments + ray_index;
                        mean = m[0];
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            dO[k] = m[(1 + k) * ma.stride];
                            dD[k] = m[(4 + k) * ma.stride];
                        }
                        sl = m[7 * ma.stride];
                        su = m[8 * ma.stride];
                    } else {
                        // the pose moments' alpha_i by one multiplication when S is a power of two
                        auto run = [&](auto bounded_tag) {
                            if constexpr (kPose && DPT_VJP_POW2_ALPHA != 0) {
                                if ((S & (S - 1)) == 0)
                                    march(bounded_tag, std::true_type{});
                                else
                                    march(bounded_tag, std::false_type{});
                            } else {
                                march(bounded_tag, std::false_type{});
                            }
                        };
                        if (bounded)
                            run(std::true_type{});
                        else
                            run(std::false_type{});
                    }
                    if (kVol && pending >= 0) flush_run(pending, cs);
                    if constexpr (kMoments == kStoreMoments) {
                        // the forward image: the same serial sum the forward kernel forms (a
                        // trailing zero sample only turns -0 into +0), scaled by length*step
                        float total = trailing_zero ? mean + 0.0f : mean;
                        total = total * physical_step;
                        if (!isfinite(total)) bits |= 2;
                        stored_image = total;
                        stored[0] = mean;
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            stored[1 + k] = dO[k];
                            stored[4 + k] = dD[k];
                        }
                        stored[7] = sl;
                        stored[8] = su;
                    } else if (kPose) {
                        float lo_o[3], lo_d[3], up_o[3], up_d[3];
                        iv.lower_gradients(lo_o, lo_d);
                        iv.upper_gradients(up_o, up_d);
                        const float lower_seed = fmaf(span, sl, -mean);
                        const float upper_seed = fmaf(span, su, mean);
                        double og[3], dg[3];
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            og[k] = (double)fmaf(upper_seed, up_o[k], fmaf(lower_seed, lo_o[k], span * dO[k]));
                            dg[k] = (double)fmaf(upper_seed, up_d[k], fmaf(lower_seed, lo_d[k], span * dD[k]));
                        }
                        const double factor = (double)((seed * length) / (float)S);
                        double sa[3], da[3];
                        matvec_t(a.grid.m, og, sa);
                        matvec_t(a.grid.m, dg, da);
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            sa[k] = factor * sa[k];
                            da[k] = factor * da[k];
                        }
                        pose_epilogue(a, vs, view, pixel, mode, sa, da, g);
                    }
                }
            }
        } else if constexpr (kArith == DPT_ARITH_MIXED || kArith == DPT_ARITH_FAST) {
            // reference mixed / fast sampling, fixed pose (kernels/projection.py:1026-1106 with
            // the mixed scatter :431-479): each inside sample adds, per corner, the FP32
            // rounding of volume_factor * w_c, w_c the forward's FP32 corner weight
            if (!valid_ray(r)) {
                bits = 2;
            } else if (kVol) {
                Interval<double> iv;
                iv.clip(r.origin, r.direction, dims.nx, dims.ny, dims.nz);
                double span = iv.upper - iv.lower;
                const double seed = seed_in;
                if (!isfinite(seed)) bits |= 2;
                if (seed == 0.0) span = 0.0;
                if (span > 0.0) {
                    const double vf = seed * r.length * span / (double)S;
                    const double step = span / (double)S;
                    float entry[3], sv[3];
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        entry[k] = (float)fma(iv.lower, r.direction[k], r.origin[k]);
                        sv[k] = (float)(step * r.direction[k]);
                    }
                    float cs[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c) cs[c] = 0.0f;
                    int pending = -1;
                    auto flush = [&]() {
                        flush_cell(acc, pending, cs);
#pragma unroll
                        for (int c = 0; c < 8; ++c) cs[c] = 0.0f;
                    };
                    auto visit = [&](int i, bool general) {
                        const float offset = (float)i + 0.5f;
                        const float x = fmaf(offset, sv[0], entry[0]);
                        const float y = fmaf(offset, sv[1], entry[1]);
                        const float z = fmaf(offset, sv[2], entry[2]);
                        if (general) {
                            if (!finite3f(x, y, z)) bits |= 2;
                            if (!inside(x, y, z, dims.hx, dims.hy, dims.hz)) {
                                if (pending >= 0) flush();
                                pending = -1;
                                return;
                            }
                        }
                        const Axis32 X = axis32(x, dims.mx, dims.cx), Y = axis32(y, dims.my, dims.cy),
                                     Z = axis32(z, dims.mz, dims.cz);
                        const int cell = (Z.lower * dims.ny + Y.lower) * dims.nx + X.lower;
                        if (cell != pending) {
                            if (pending >= 0) flush();
                            pending = cell;
                        }
                        float w[8];
                        corner_weights(X.fraction, Y.fraction, Z.fraction, w);
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            const float increment = (float)(vf * (double)w[c]);
                            if (!isfinite(increment)) bits |= 2;
                            cs[c] = cs[c] + increment;
                        }
                    };
                    if (!moderate(entry, sv)) {
                        for (int i = 0; i < S; ++i) visit(i, true);
                    } else {
                        int first, last;
                        inside_run(S, [&](int i) {
                            const float offset = (float)i + 0.5f;
                            return inside(fmaf(offset, sv[0], entry[0]), fmaf(offset, sv[1], entry[1]),
                                          fmaf(offset, sv[2], entry[2]), dims.hx, dims.hy, dims.hz);
                        }, first, last);
                        for (int i = first; i <= last; ++i) visit(i, false);
                    }
                    if (pending >= 0) flush();
                }
            }
        } else if constexpr (kArith == DPT_ARITH_CELLS) {
            // reference cell-Gauss VJP (kernels/projection.py:935-1024 and the shared tail
            // 1152-1210): Gauss-node gradients weighted by radius (origin) and radius times
            // position (direction), the zero-extended support's endpoint terms, factor =
            // seed * length; the scatter combines a shared cell's two nodes before rounding
            if (!valid_ray(r)) {
                bits = 2;
            } else {
                Interval<double> iv;
                iv.clip(r.origin, r.direction, dims.nx, dims.ny, dims.nz);
                double span = iv.upper - iv.lower;
                const double seed = seed_in;
                if (!isfinite(seed)) bits |= 2;
                if (seed == 0.0) span = 0.0;
                if (span > 0.0) {
                    const double factor = seed * r.length;
                    const int shape[3] = {dims.nx, dims.ny, dims.nz}, cap[3] = {dims.cx, dims.cy, dims.cz};
                    double og[3] = {0.0, 0.0, 0.0}, dg[3] = {0.0, 0.0, 0.0};
                    // one node's FP64 corner terms ((seed w0) w1) w2 relative to cell `lower`
                    auto corner_terms = [&](const double* q, const int* lower, double vf, double* t) {
                        double fr[3];
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            fr[k] = fmin(fmax(q[k], 0.0), (double)(shape[k] - 1)) - (double)lower[k];
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            double contribution = vf * ((c & 1) ? fr[0] : 1.0 - fr[0]);
                            contribution = contribution * ((c & 2) ? fr[1] : 1.0 - fr[1]);
                            t[c] = contribution * ((c & 4) ? fr[2] : 1.0 - fr[2]);
                        }
                    };
                    auto scatter_node = [&](const double* q, double vf) {
                        if (!inside(q[0], q[1], q[2], dims.nx, dims.ny, dims.nz)) return;
                        int lower[3];
#pragma unroll
                        for (int k = 0; k < 3; ++k) lower[k] = axis64(q[k], (double)(shape[k] - 1), cap[k]).lower;
                        double t[8];
                        corner_terms(q, lower, vf, t);
                        float c32[8];
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            c32[c] = (float)t[c];
                            if (!isfinite(c32[c])) bits |= 2;
                        }
                        flush_cell(acc, (lower[2] * dims.ny + lower[1]) * dims.nx + lower[0], c32);
                    };
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
                        if (kPose) {
                            double g1[3], g2[3];
                            sample_strict64(f, dims, s.first, g1);
                            sample_strict64(f, dims, s.second, g2);
                            const double r1 = s.radius * s.first_position, r2 = s.radius * s.second_position;
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                og[k] = fma(s.radius, g1[k], og[k]);
                                og[k] = fma(s.radius, g2[k], og[k]);
                                dg[k] = fma(r1, g1[k], dg[k]);
                                dg[k] = fma(r2, g2[k], dg[k]);
                            }
                        }
                        if (kVol) {
                            const double vf = factor * s.radius;
                            if (s.shared) {
                                const bool in1 = inside(s.first[0], s.first[1], s.first[2], dims.nx, dims.ny, dims.nz);
                                const bool in2 = inside(s.second[0], s.second[1], s.second[2], dims.nx, dims.ny, dims.nz);
                                double t1[8], t2[8];
                                corner_terms(s.first, s.lower, in1 ? vf : 0.0, t1);
                                corner_terms(s.second, s.lower, in2 ? vf : 0.0, t2);
                                float c32[8];
#pragma unroll
                                for (int c = 0; c < 8; ++c) {
                                    c32[c] = (float)(t1[c] + t2[c]);
                                    if (!isfinite(c32[c])) bits |= 2;
                                }
                                flush_cell(acc, (s.lower[2] * dims.ny + s.lower[1]) * dims.nx + s.lower[0], c32);
                            } else {
                                scatter_node(s.first, vf);
                                scatter_node(s.second, vf);
                            }
                        }
                        start = s.end;
                        walk.advance(r, shape, s.end, iv.upper);
                    }
                    if (start < iv.upper) bits |= 2;
                    if (kPose) {
                        double lower_point[3], upper_point[3];
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            // support_value (:663-674): the endpoint clamped into the support
                            const double high = (double)shape[k] - 0.5;
                            lower_point[k] = fmin(fmax(fma(iv.lower, r.direction[k], r.origin[k]), -0.5), high);
                            upper_point[k] = fmin(fmax(fma(iv.upper, r.direction[k], r.origin[k]), -0.5), high);
                        }
                        const double lower_value = sample_strict64(f, dims, lower_point, nullptr);
                        const double upper_value = sample_strict64(f, dims, upper_point, nullptr);
                        double lo_o[3], lo_d[3], up_o[3], up_d[3];
                        iv.lower_gradients(lo_o, lo_d);
                        iv.upper_gradients(up_o, up_d);
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            og[k] = og[k] + fma(-lower_value, lo_o[k], upper_value * up_o[k]);
                            dg[k] = dg[k] + fma(-lower_value, lo_d[k], upper_value * up_d[k]);
                        }
                        double sa[3], da[3];
                        matvec_t(a.grid.m, og, sa);
                        matvec_t(a.grid.m, dg, da);
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            sa[k] = factor * sa[k];
                            da[k] = factor * da[k];
                        }
                        pose_epilogue(a, vs, view, pixel, mode, sa, da, g);
                    }
                }
            }
        } else if constexpr (kArith == DPT_ARITH_F64) {
            if (!valid_ray(r)) {
                bits = 2;
            } else {
                Interval<double> iv;
                iv.clip(r.origin, r.direction, dims.nx, dims.ny, dims.nz);
                double span = iv.upper - iv.lower;
                const double seed = seed_in;
                if (!isfinite(seed)) bits |= 2;
                if (seed == 0.0) span = 0.0;
                if (span > 0.0) {
                    double factor = seed * r.length;
                    const double step = span / (double)S;
                    const double vf = factor * span / (double)S;
                    const bool power_of_two = (S & (S - 1)) == 0;
                    const double inverse_samples = power_of_two ? 1.0 / (double)S : 0.0;
                    const double mx = (double)(dims.nx - 1), my = (double)(dims.ny - 1), mz = (double)(dims.nz - 1);
                    double mean = 0.0, dO[3] = {0.0, 0.0, 0.0}, dD[3] = {0.0, 0.0, 0.0};
                    double sl = 0.0, su = 0.0;
                    // a cell run's sums of the FP32-rounded increments, in FP32 as the reference
                    // adds them (FP32 atomics into the FP32 accumulator)
                    float cs[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c) cs[c] = 0.0f;
                    int pending = -1;
                    // the cell's corners widened to FP64 once per cell (exact)
                    WideCellCache<Field> cache;
                    auto flush64 = [&]() {
                        flush_cell(acc, pending, cs);
#pragma unroll
                        for (int c = 0; c < 8; ++c) cs[c] = 0.0f;
                    };
                    auto point_at = [&](int i, double& position, double* p) {
                        position = fma((double)i + 0.5, step, iv.lower);
#pragma unroll
                        for (int k = 0; k < 3; ++k) p[k] = fma(position, r.direction[k], r.origin[k]);
                    };
                    auto visit = [&](int i, bool known_inside) {
                        const double alpha = power_of_two ? ((double)i + 0.5) * inverse_samples
                                                          : ((double)i + 0.5) / (double)S;
                        double position, p[3];
                        point_at(i, position, p);
                        bool in = true;
                        if (!known_inside) {
                            if (!finite3(p[0], p[1], p[2])) bits |= 2;
                            in = inside(p[0], p[1], p[2], dims.nx, dims.ny, dims.nz);
                        }
                        Axis64 X{0, 0.0}, Y{0, 0.0}, Z{0, 0.0};
                        int cell = -1;
                        if (in) {
                            X = axis64(p[0], mx, dims.cx);
                            Y = axis64(p[1], my, dims.cy);
                            Z = axis64(p[2], mz, dims.cz);
                            cell = (Z.lower * dims.ny + Y.lower) * dims.nx + X.lower;
                        }
                        if (kPose) {
                            double value = 0.0, gs[3] = {0.0, 0.0, 0.0};
                            if (in) {
                                cache.fetch(f, X.lower, Y.lower, Z.lower, cell);
                                const double* v = cache.v;
                                value = interpolate64(X.fraction, Y.fraction, Z.fraction, v);
                                const double sx = (p[0] >= 0.0 && p[0] < mx) ? 1.0 : 0.0;
                                const double sy = (p[1] >= 0.0 && p[1] < my) ? 1.0 : 0.0;
                                const double sz = (p[2] >= 0.0 && p[2] < mz) ? 1.0 : 0.0;
                                slope64(X.fraction, Y.fraction, Z.fraction, v, sx, sy, sz, gs);
                            }
                            mean = mean + value;
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                dO[k] = dO[k] + gs[k];
                                dD[k] = fma(position, gs[k], dD[k]);
                            }
                            const double along =
                                fma(gs[2], r.direction[2], fma(gs[1], r.direction[1], gs[0] * r.direction[0]));
                            sl = fma(1.0 - alpha, along, sl);
                            su = fma(alpha, along, su);
                        }
                        if (kVol) {
                            if (in) {
                                if (cell != pending) {
                                    if (pending >= 0) flush64();
                                    pending = cell;
                                }
                                const double fx = X.fraction, fy = Y.fraction, fz = Z.fraction;
#pragma unroll
                                for (int c = 0; c < 8; ++c) {
                                    double contribution = vf * ((c & 1) ? fx : 1.0 - fx);
                                    contribution = contribution * ((c & 2) ? fy : 1.0 - fy);
                                    contribution = contribution * ((c & 4) ? fz : 1.0 - fz);
                                    const float rounded = (float)contribution;
                                    if (!isfinite(rounded)) bits |= 2;
                                    cs[c] = cs[c] + rounded;
                                }
                            } else if (pending >= 0) {
                                flush64();
                                pending = -1;
                            }
                        }
                    };
                    if (!moderate(r.origin, r.direction)) {
                        for (int i = 0; i < S; ++i) visit(i, false);
                    } else {
                        int first, last;
                        inside_run(S, [&](int i) {
                            double position, p[3];
                            point_at(i, position, p);
                            return inside(p[0], p[1], p[2], dims.nx, dims.ny, dims.nz);
                        }, first, last);
                        for (int i = first; i <= last; ++i) visit(i, true);
                    }
                    if (kVol && pending >= 0) flush64();
                    if (kPose) {
                        double lo_o[3], lo_d[3], up_o[3], up_d[3];
                        iv.lower_gradients(lo_o, lo_d);
                        iv.upper_gradients(up_o, up_d);
                        const double lower_seed = fma(span, sl, -mean);
                        const double upper_seed = fma(span, su, mean);
                        double og[3], dg[3];
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            og[k] = fma(upper_seed, up_o[k], fma(lower_seed, lo_o[k], span * dO[k]));
                            dg[k] = fma(upper_seed, up_d[k], fma(lower_seed, lo_d[k], span * dD[k]));
                        }
                        factor = factor / (double)S;
                        double sa[3], da[3];
                        matvec_t(a.grid.m, og, sa);
                        matvec_t(a.grid.m, dg, da);
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            sa[k] = factor * sa[k];
                            da[k] = factor * da[k];
                        }
                        pose_epilogue(a, vs, view, pixel, mode, sa, da, g);
                    }
                }
            }
        } else {
            // F32C: FP64 clip; FP32 marching; per cell run (closed form over the run's
            // samples): the compensated mean, pose sums G = sum grad and H = sum alpha grad
            // from the cell's trilinear polynomial, and the eight moments of the fractions
            // expanded into the cell's eight corner sums.
            if (!valid_ray(r)) {
                bits = 2;
            } else {
                Interval<double> iv;
                iv.clip(r.origin, r.direction, dims.nx, dims.ny, dims.nz);
                const double span = iv.upper - iv.lower;
                const double seed = seed_in;
                if (!isfinite(seed)) bits |= 2;
                if (span > 0.0 && seed != 0.0) {
                    const double step = span / (double)S;
                    const float vf = (float)(seed * r.length * step);
                    float entry[3], sv[3];
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        entry[k] = (float)fma(iv.lower, r.direction[k], r.origin[k]);
                        sv[k] = (float)(step * r.direction[k]);
                    }
                    double mean64 = 0.0, Gd[3] = {0.0, 0.0, 0.0}, Hd[3] = {0.0, 0.0, 0.0};
                    // eight moments of a run's fractions -> its cell's eight corner sums, scaled
                    auto scatter_moments = [&](int cell, const float* m) {
                        float corner[8];
                        corner[7] = m[7];
                        corner[3] = m[4] - m[7];
                        corner[5] = m[5] - m[7];
                        corner[6] = m[6] - m[7];
                        corner[1] = (m[1] - m[4]) - corner[5];
                        corner[2] = (m[2] - m[4]) - corner[6];
                        corner[4] = (m[3] - m[5]) - corner[6];
                        corner[0] = ((m[0] - m[1]) - (m[2] - m[4])) - corner[4];
                        bool finite = true;
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            corner[c] = vf * corner[c];
                            finite = finite && isfinite(corner[c]);
                        }
                        if (!finite) bits |= 2;
                        flush_cell(acc, cell, corner);
                    };
                    float words[kMomentWords] = {};
                    if constexpr (kMoments == kLoadMoments) {
#pragma unroll
                        for (int k = 0; k < kMomentWords; ++k) words[k] = ma.moments[k * ma.stride + ray_index];
                    } else if (segment_form(entry, sv)) {
                        // segment form: every cell run in closed form
                        int first, last;
                        inside_run(S, [&](int i) {
                            const float offset = (float)i + 0.5f;
                            return inside(fmaf(offset, sv[0], entry[0]), fmaf(offset, sv[1], entry[1]),
                                          fmaf(offset, sv[2], entry[2]), dims.hx, dims.hy, dims.hz);
                        }, first, last);
                        Kahan32 mean;
                        float G[3] = {0.0f, 0.0f, 0.0f}, Hs[3] = {0.0f, 0.0f, 0.0f};
                        if (first <= last) {
                            walk_cells(dims, entry, sv, first, last, [&](const CellRun& run) {
                                const float dx = run.d[0], dy = run.d[1], dz = run.d[2];
                                const float dxy = dx * dy, dxz = dx * dz, dyz = dy * dz;
                                const float nf = run.nf, s1 = run.s1, s2 = run.s2, s3 = run.s3;
                                if (kPose) {
                                    PolyCache<Field, false> cell;
                                    cell.fetch(f, run.lx, run.ly, run.lz, run.cell);
                                    const RunPoly o = run_poly(cell.c, run.f);
                                    mean.add(run_sum(run, o));
                                    float g0[3] = {o.gx, o.gy, o.gz};
                                    float g1[3] = {fmaf(o.t1, dz, o.a * dy), fmaf(o.t2, dz, o.a * dx),
                                                   fmaf(o.t2, dy, o.t1 * dx)};
                                    float g2[3] = {o.c7 * dyz, o.c7 * dxz, o.c7 * dxy};
                                    const float offset = (float)run.i0 + 0.5f;
#pragma unroll
                                    for (int k = 0; k < 3; ++k) {
                                        if (!((run.interior >> k) & 1)) g0[k] = g1[k] = g2[k] = 0.0f;
                                        const float sg = fmaf(s2, g2[k], fmaf(s1, g1[k], nf * g0[k]));
                                        const float sj = fmaf(s3, g2[k], fmaf(s2, g1[k], s1 * g0[k]));
                                        G[k] = G[k] + sg;
                                        Hs[k] = Hs[k] + fmaf(offset, sg, sj);
                                    }
                                }
                                if (kVol) {
                                    const float fx = run.f[0], fy = run.f[1], fz = run.f[2];
                                    const float fxy = fx * fy, fxz = fx * fz, fyz = fy * fz;
                                    float m[8];
                                    m[0] = nf;
                                    m[1] = fmaf(s1, dx, nf * fx);
                                    m[2] = fmaf(s1, dy, nf * fy);
                                    m[3] = fmaf(s1, dz, nf * fz);
                                    m[4] = fmaf(s2, dxy, fmaf(s1, fmaf(fx, dy, fy * dx), nf * fxy));
                                    m[5] = fmaf(s2, dxz, fmaf(s1, fmaf(fx, dz, fz * dx), nf * fxz));
                                    m[6] = fmaf(s2, dyz, fmaf(s1, fmaf(fy, dz, fz * dy), nf * fyz));
                                    m[7] = fmaf(s3, dxy * dz,
                                                fmaf(s2, fmaf(fz, dxy, fmaf(fy, dxz, fx * dyz)),
                                                     fmaf(s1, fmaf(fyz, dx, fmaf(fxz, dy, fxy * dz)),
                                                          nf * (fxy * fz))));
                                    scatter_moments(run.cell, m);
                                }
                            }, run_sums);
                        }
                        words[0] = mean.sum;
                        words[1] = mean.carry;
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            words[2 + k] = G[k];
                            words[5 + k] = Hs[k];
                        }
                    } else {
                        // per-sample form (samples more than a cell plane apart, or rays
                        // reaching 1e30 in grid coordinates)
                        const float inv_s = 1.0f / (float)S;
                        BlockSum mean;
                        float G[3] = {0.0f, 0.0f, 0.0f}, H[3] = {0.0f, 0.0f, 0.0f};
                        float m[8];
#pragma unroll
                        for (int c = 0; c < 8; ++c) m[c] = 0.0f;
                        int pending = -1;
                        PolyCache<Field, kVjpReuse> cache;
                        for (int i = 0; i < S; ++i) {
                            const float offset = (float)i + 0.5f;
                            const float x = fmaf(offset, sv[0], entry[0]);
                            const float y = fmaf(offset, sv[1], entry[1]);
                            const float z = fmaf(offset, sv[2], entry[2]);
                            if (!finite3f(x, y, z)) bits |= 2;
                            const bool in = inside(x, y, z, dims.hx, dims.hy, dims.hz);
                            Axis32 X{0, 0.0f}, Y{0, 0.0f}, Z{0, 0.0f};
                            int cell = -1;
                            if (in) {
                                X = axis32(x, dims.mx, dims.cx);
                                Y = axis32(y, dims.my, dims.cy);
                                Z = axis32(z, dims.mz, dims.cz);
                                cell = (Z.lower * dims.ny + Y.lower) * dims.nx + X.lower;
                            }
                            if (kPose) {
                                float value = 0.0f, gs[3] = {0.0f, 0.0f, 0.0f};
                                if (in) {
                                    cache.fetch(f, X.lower, Y.lower, Z.lower, cell);
                                    value = cache.eval(X.fraction, Y.fraction, Z.fraction, gs);
                                    if (!(x >= 0.0f && x < dims.mx)) gs[0] = 0.0f * gs[0];
                                    if (!(y >= 0.0f && y < dims.my)) gs[1] = 0.0f * gs[1];
                                    if (!(z >= 0.0f && z < dims.mz)) gs[2] = 0.0f * gs[2];
                                }
                                mean.add(value, i, S);
                                const float alpha = offset * inv_s;
#pragma unroll
                                for (int k = 0; k < 3; ++k) {
                                    G[k] = G[k] + gs[k];
                                    H[k] = fmaf(alpha, gs[k], H[k]);
                                }
                            }
                            if (kVol) {
                                if (in) {
                                    if (cell != pending) {
                                        if (pending >= 0) {
                                            scatter_moments(pending, m);
#pragma unroll
                                            for (int c = 0; c < 8; ++c) m[c] = 0.0f;
                                        }
                                        pending = cell;
                                    }
                                    const float fx = X.fraction, fy = Y.fraction, fz = Z.fraction;
                                    const float fxy = fx * fy;
                                    m[0] = m[0] + 1.0f;
                                    m[1] = m[1] + fx;
                                    m[2] = m[2] + fy;
                                    m[3] = m[3] + fz;
                                    m[4] = m[4] + fxy;
                                    m[5] = m[5] + fx * fz;
                                    m[6] = m[6] + fy * fz;
                                    m[7] = m[7] + fxy * fz;
                                } else if (pending >= 0) {
                                    scatter_moments(pending, m);
#pragma unroll
                                    for (int c = 0; c < 8; ++c) m[c] = 0.0f;
                                    pending = -1;
                                }
                            }
                        }
                        if (kVol && pending >= 0) scatter_moments(pending, m);
                        words[0] = mean.sum;
                        words[1] = mean.carry;
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            words[2 + k] = G[k];
                            words[5 + k] = H[k];
                        }
                        words[8] = 1.0f;
                    }
                    if (kPose) {
                        mean64 = (double)words[0] - (double)words[1];
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            Gd[k] = words[2 + k];
                            Hd[k] = words[8] != 0.0f ? (double)words[5 + k] : (double)words[5 + k] / (double)S;
                        }
                    }
                    if constexpr (kMoments == kStoreMoments) {
                        // the forward image of the compensated form, as the forward kernel forms it
                        const float total = (float)(mean64 * (r.length * step));
                        if (!isfinite(total)) bits |= 2;
                        stored_image = total;
#pragma unroll
                        for (int k = 0; k < kMomentWords; ++k) stored[k] = words[k];
                    } else if (kPose) {
                        const double* dr = r.direction;
                        const double g_along = fma(Gd[2], dr[2], fma(Gd[1], dr[1], Gd[0] * dr[0]));
                        const double h_along = fma(Hd[2], dr[2], fma(Hd[1], dr[1], Hd[0] * dr[0]));
                        const double su = h_along, sl = g_along - h_along;
                        const double lower_seed = fma(span, sl, -mean64);
                        const double upper_seed = fma(span, su, mean64);
                        double lo_o[3], lo_d[3], up_o[3], up_d[3];
                        iv.lower_gradients(lo_o, lo_d);
                        iv.upper_gradients(up_o, up_d);
                        double og[3], dg[3];
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            const double direct_direction = fma(span, Hd[k], iv.lower * Gd[k]);
                            og[k] = fma(upper_seed, up_o[k], fma(lower_seed, lo_o[k], span * Gd[k]));
                            dg[k] = fma(upper_seed, up_d[k], fma(lower_seed, lo_d[k], span * direct_direction));
                        }
                        const double factor = seed * r.length / (double)S;
                        double sa[3], da[3];
                        matvec_t(a.grid.m, og, sa);
                        matvec_t(a.grid.m, dg, da);
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            sa[k] = factor * sa[k];
                            da[k] = factor * da[k];
                        }
                        pose_epilogue(a, vs, view, pixel, mode, sa, da, g);
                    }
                }
            }
        }
    }

    if constexpr (kMoments == kStoreMoments) {
        if (active) {
            const int64_t ray_index = view_local * rays_per_view + pixel;
            ma.image[ray_index] = stored_image;
#pragma unroll
            for (int k = 0; k < kMomentWords; ++k) ma.moments[k * ma.stride + ray_index] = stored[k];
        }
        if (bits) atomicOr(a.status + view, bits);
        return;
    }
    if (kPose) {
        if (mode < 0) {
            if (active) {
                double* out = partials + 6 * (view_local * rays_per_view + pixel);
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    out[k] = g[k];
                    if (!isfinite(g[k])) bits |= 2;
                }
            }
        } else {
            const int components = mode;
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
            for (int k = 0; k < 12; ++k) {
                if (k < components) {
                    double v = g[k];
#pragma unroll
                    for (int offset = 16; offset > 0; offset >>= 1)
                        v += __shfl_down_sync(0xffffffffu, v, offset);
                    if (lane == 0) warp_sums[warp][k] = v;
                }
            }
            __syncthreads();
            if (threadIdx.x < components) {
                double total = 0.0;
#pragma unroll
                for (int w = 0; w < kVjpBlock / 32; ++w) total += warp_sums[w][threadIdx.x];
                partials[((int64_t)view_local * a.tiles_per_view + tile) * components +
                         threadIdx.x] = total;
            }
        }
    }
    if (bits) atomicOr(a.status + view, bits);
}

template <int kArith, class Field, typename Seed>
cudaError_t vjp_with(const RayArgs& a, const Field& f, const Seed* cot, int flags, float* acc,
                     double* partials, cudaStream_t stream)
{
    const dim3 grid(ray_blocks(a));
    const bool volume = (flags & DPT_VJP_VOLUME) != 0;
    const bool pose = (flags & (DPT_VJP_POSE12 | DPT_VJP_POSE6 | DPT_VJP_PER_RAY6)) != 0;
    const int mode = (flags & DPT_VJP_POSE12) ? 12 : ((flags & DPT_VJP_PER_RAY6) ? -6 : 6);
    if constexpr (kArith == DPT_ARITH_MIXED || kArith == DPT_ARITH_FAST) {
        // fixed-pose forms: the C ABI admits the volume cotangent only
        if (pose || !volume) return cudaErrorInvalidValue;
        k_vjp<kArith, Field, true, false, Seed><<<grid, kVjpBlock, 0, stream>>>(a, f, cot, mode, acc, partials, MomentArgs{});
    } else {
        if (volume && pose)
            k_vjp<kArith, Field, true, true, Seed><<<grid, kVjpBlock, 0, stream>>>(a, f, cot, mode, acc, partials, MomentArgs{});
        else if (volume)
            k_vjp<kArith, Field, true, false, Seed><<<grid, kVjpBlock, 0, stream>>>(a, f, cot, mode, acc, partials, MomentArgs{});
        else
            k_vjp<kArith, Field, false, true, Seed><<<grid, kVjpBlock, 0, stream>>>(a, f, cot, mode, acc, partials, MomentArgs{});
    }
    return cudaGetLastError();
}

template <int kArith, class Field>
cudaError_t vjp_seed(const dpt_problem& p, const RayArgs& a, const Field& f, const void* cot,
                     int flags, float* acc, double* partials, cudaStream_t stream)
{
    if (p.image_dtype == DPT_F64)
        return vjp_with<kArith>(a, f, static_cast<const double*>(cot), flags, acc, partials, stream);
    return vjp_with<kArith>(a, f, static_cast<const float*>(cot), flags, acc, partials, stream);
}

}  // namespace

cudaError_t launch_vjp(const dpt_problem& p, const RayArgs& a, const void* packed,
                       const void* cotangent, int flags, float* accumulator, double* partials,
                       cudaStream_t stream)
{
    if (p.arith == DPT_ARITH_F32C && p.layout == DPT_LAYOUT_REPLICATED) {
        PolyF32 f{static_cast<const float4*>(packed), p.nx, p.ny, p.nz};
        return vjp_seed<DPT_ARITH_F32C>(p, a, f, cotangent, flags, accumulator, partials, stream);
    }
    // direct gathers from the caller's FP32 field, or the FP32 corner quads (decoded from any
    // storage type by the pack kernel)
    auto run = [&](const auto& f) -> cudaError_t {
        switch (p.arith) {
        case DPT_ARITH_F32:
            return vjp_seed<DPT_ARITH_F32>(p, a, f, cotangent, flags, accumulator, partials, stream);
        case DPT_ARITH_F64:
            return vjp_seed<DPT_ARITH_F64>(p, a, f, cotangent, flags, accumulator, partials, stream);
        case DPT_ARITH_MIXED:
            return vjp_seed<DPT_ARITH_MIXED>(p, a, f, cotangent, flags, accumulator, partials, stream);
        case DPT_ARITH_FAST:
            return vjp_seed<DPT_ARITH_FAST>(p, a, f, cotangent, flags, accumulator, partials, stream);
        case DPT_ARITH_CELLS:
            return vjp_seed<DPT_ARITH_CELLS>(p, a, f, cotangent, flags, accumulator, partials, stream);
        default:
            return vjp_seed<DPT_ARITH_F32C>(p, a, f, cotangent, flags, accumulator, partials, stream);
        }
    };
    if (p.layout == DPT_LAYOUT_DIRECT) return run(PlainF32{static_cast<const float*>(packed), p.nx, p.ny, p.nz});
    return run(QuadF32{static_cast<const float4*>(packed), p.nx, p.ny, p.nz});
}

// Forward image plus the pose moments of every ray (FP32 or compensated arithmetic; see
// kStoreMoments).
cudaError_t launch_forward_moments(const dpt_problem& p, const RayArgs& a, const void* packed,
                                   float* image, float* moments, int64_t stride, cudaStream_t stream)
{
    const dim3 grid(ray_blocks(a));
    const MomentArgs ma{moments, stride, image};
    const bool pow2 = (p.nx & (p.nx - 1)) == 0 && (p.ny & (p.ny - 1)) == 0;
    auto run = [&](auto arith, const auto& f) {
        using FieldT = std::decay_t<decltype(f)>;
        constexpr int kArith = decltype(arith)::value;
        if constexpr (kArith == DPT_ARITH_F32) {
            if (pow2) {
                k_vjp<kArith, FieldT, false, true, float, kStoreMoments, true>
                    <<<grid, kVjpBlock, 0, stream>>>(a, f, nullptr, 6, nullptr, nullptr, ma);
                return;
            }
        }
        k_vjp<kArith, FieldT, false, true, float, kStoreMoments>
            <<<grid, kVjpBlock, 0, stream>>>(a, f, nullptr, 6, nullptr, nullptr, ma);
    };
    using F32 = std::integral_constant<int, DPT_ARITH_F32>;
    using F32C = std::integral_constant<int, DPT_ARITH_F32C>;
    const PlainF32 direct{static_cast<const float*>(packed), p.nx, p.ny, p.nz};
    if (p.arith == DPT_ARITH_F32C) {
        if (p.layout == DPT_LAYOUT_DIRECT)
            run(F32C{}, direct);
        else
            run(F32C{}, PolyF32{static_cast<const float4*>(packed), p.nx, p.ny, p.nz});
    } else if (p.layout == DPT_LAYOUT_DIRECT) {
        run(F32{}, direct);
    } else {
        run(F32{}, QuadF32{static_cast<const float4*>(packed), p.nx, p.ny, p.nz});
    }
    return cudaGetLastError();
}

// Pose VJP from stored moments: no sampling, the field is not read.
cudaError_t launch_pose_from_moments(const dpt_problem& p, const RayArgs& a, const float* moments,
                                     int64_t stride, const void* cotangent, int flags,
                                     double* partials, cudaStream_t stream)
{
    const dim3 grid(ray_blocks(a));
    const int mode = (flags & DPT_VJP_POSE12) ? 12 : ((flags & DPT_VJP_PER_RAY6) ? -6 : 6);
    const MomentArgs ma{const_cast<float*>(moments), stride, nullptr};
    const PlainF32 none{nullptr, p.nx, p.ny, p.nz};
    auto run = [&](auto arith, const auto* seed) {
        using SeedT = std::remove_cv_t<std::remove_pointer_t<decltype(seed)>>;
        k_vjp<decltype(arith)::value, PlainF32, false, true, SeedT, kLoadMoments>
            <<<grid, kVjpBlock, 0, stream>>>(a, none, seed, mode, nullptr, partials, ma);
    };
    using F32 = std::integral_constant<int, DPT_ARITH_F32>;
    using F32C = std::integral_constant<int, DPT_ARITH_F32C>;
    if (p.image_dtype == DPT_F64) {
        const double* seed = static_cast<const double*>(cotangent);
        if (p.arith == DPT_ARITH_F32C) run(F32C{}, seed); else run(F32{}, seed);
    } else {
        const float* seed = static_cast<const float*>(cotangent);
        if (p.arith == DPT_ARITH_F32C) run(F32C{}, seed); else run(F32{}, seed);
    }
    return cudaGetLastError();
}

}  // namespace dpt
