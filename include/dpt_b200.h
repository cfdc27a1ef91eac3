/*
 * dpt_b200.h - C ABI of the B200 differentiable CT projector.
 *
 * The projector integrates a sampled attenuation field mu (mm^-1) along finite
 * source-to-detector segments: clipped midpoint sampling of the trilinear,
 * half-cell-extended field, then L = |e - s| * step * sum_i mu(p_i).  Its VJP
 * returns the volume cotangent (adjoint backprojection) and the per-view rigid
 * pose cotangent.
 *
 * Every compute entry point borrows caller memory and allocates nothing: the
 * field, geometry, outputs and scratch are device pointers owned by the
 * caller, work is enqueued on the caller's cudaStream_t (passed as void*), and
 * the call returns as soon as the kernels are enqueued.  Device diagnostics are
 * OR-ed into per-view int32 status words with the reference projector's bits:
 *   1 = invalid rigid pose, 2 = non-finite projection / gradient / cotangent,
 *   8 = field not finite or negative.
 * Host-side argument errors are returned as negative DPT_E* codes; a CUDA launch
 * error is returned as its positive cudaError_t value.
 *
 * The reference interfaces these entry points replace (hcltech-robotics/dpt):
 *   dpt_b200_prepare_field  <- python/dpt/torch/_projection_ops.py:197-211 (_validate:
 *                              field scan + rigid-pose check) and the field upload of
 *                              python/dpt/projection.py:747-809
 *   dpt_b200_forward        <- python/dpt/projection.py:747-809 (project_optical_depth),
 *                              kernels python/dpt/kernels/projection_fp32.py:334-374 and
 *                              python/dpt/kernels/projection.py:802-846
 *   dpt_b200_vjp            <- python/dpt/projection.py:871-1018 (projection_vjp) and
 *                              1021-1084 (projection_pose_sensitivities), kernels
 *                              python/dpt/kernels/projection_fp32.py:377-617 and
 *                              python/dpt/kernels/projection.py:873-1237
 *   dpt_b200_fold_volume    <- python/dpt/torch/_projection_ops.py:304-352 (FP64 widening
 *                              of the FP32 volume gradient) plus the gradient finite scan
 *                              python/dpt/projection.py:470-499
 *   dpt_b200_finish_pose    <- python/dpt/_reductions.py:27-63 (FP64 tile tree and finish)
 *   dpt_b200_counts         <- per-ray clip interval of python/dpt/kernels/projection_fp32.py:78-109
 *                              and python/dpt/kernels/projection.py:147-184 (no separate
 *                              reference entry point; exported for bit-exact count checks)
 *   dpt_b200_gather_prepare <- python/dpt/projection.py:1087-1247 (prepare_projection_adjoint),
 *                              kernels python/dpt/kernels/projection_adjoint.py:184-368
 *   dpt_b200_gather_count   <- python/dpt/kernels/projection_adjoint.py:371-581 (bounds, work count)
 *   dpt_b200_gather         <- python/dpt/projection.py:1250-1405 (projection_adjoint_gather),
 *                              kernels python/dpt/kernels/projection_adjoint.py:34-170, 583-635
 *
 * and, for the image-space steps either side of the projection (declared at the end):
 *   dpt_b200_transmit       <- python/dpt/transmission.py:307-397 (transmit), kernels
 *                              python/dpt/kernels/transmission.py:91-144
 *   dpt_b200_transmit_vjp   <- python/dpt/transmission.py:480-605 (transmission_vjp), kernels
 *                              python/dpt/kernels/transmission.py:146-268
 *   dpt_b200_depth_from_removed(_vjp) <- python/dpt/transmission.py:607-730
 *   dpt_b200_check_values   <- python/dpt/kernels/transmission.py:305-326 (input rules)
 *   dpt_b200_objective(_check) <- python/dpt/objectives.py:189-305 (evaluate_objective),
 *                              kernels python/dpt/kernels/objectives.py:23-211
 *   dpt_b200_reduce_sum     <- python/dpt/objectives.py:414-450 (reduce_objective_components)
 */
#ifndef DPT_B200_H
#define DPT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DPT_B200_ABI_VERSION 4

/* Storage / output element types. */
enum {
    DPT_F32 = 0,
    DPT_F64 = 1,
    DPT_F16 = 2,
    DPT_BF16 = 3
};

/* Sample-loop arithmetic.
 *  DPT_ARITH_F32   FP64 ray setup, FP32 clip, FP32 fmaf interpolation and serial FP32 ray sum
 *                  (the reference "fp32" Projector, kernels/projection_fp32.py).
 *  DPT_ARITH_F64   FP64 ray setup, clip, interpolation and sum (the reference "fp64" Projector,
 *                  kernels/projection.py strict midpoint).
 *  DPT_ARITH_F32C  FP64 ray setup and clip, FP32 marching, closed-form sums over the cell runs
 *                  of each ray, compensated FP32 sum over runs; the precision form for
 *                  FP16/BF16 (and FP32) storage (no reference counterpart).
 *  DPT_ARITH_MIXED FP64 setup and clip, FP32 marching and corner weights, FP64 products and
 *                  ray sum (the reference "mixed_float32" sampling, kernels/projection.py:296-392);
 *                  fixed pose: the VJP takes DPT_VJP_VOLUME only.
 *  DPT_ARITH_FAST  as MIXED with an FP32 fmaf cell sum promoted to the FP64 ray sum (the
 *                  reference "fast_float32" sampling); fixed pose.
 *  DPT_ARITH_CELLS FP64 cell-Gauss integration: the clipped ray is split at every interpolation
 *                  plane and each cubic segment integrated exactly with two Gauss nodes (the
 *                  reference integration="cell_gauss", kernels/projection.py:522-746); `samples`
 *                  is ignored. */
enum {
    DPT_ARITH_F32 = 0,
    DPT_ARITH_F64 = 1,
    DPT_ARITH_F32C = 2,
    DPT_ARITH_MIXED = 3,
    DPT_ARITH_FAST = 4,
    DPT_ARITH_CELLS = 5
};

/* Field value domain (reference ProjectionSpec.field_domain). */
enum {
    DPT_DOMAIN_PHYSICAL = 0, /* attenuation: finite and non-negative (status bit 8 otherwise) */
    DPT_DOMAIN_SIGNED = 1    /* signed_linear: any finite value (e.g. a linearised increment) */
};

/* How rays are described. */
enum {
    DPT_RAYS_PANELS = 0, /* per-view panel table (cone, parallel or curved), row-major pixels */
    DPT_RAYS_BUNDLE = 1  /* explicit FP64 source/endpoint arrays, one pose per view */
};

/* Panel table: DPT_VIEW_WORDS doubles per view. */
#define DPT_VIEW_WORDS 20
enum {
    DPT_PANEL_CONE = 0,     /* words 0-2 source, 3-5 first pixel centre, 6-8 u*du, 9-11 v*dv */
    DPT_PANEL_PARALLEL = 1, /* words 0-2 unit direction, 3-5 first pixel centre, 6-8 u, 9-11 v,
                               12 du, 13 dv, 14 segment length */
    DPT_PANEL_CURVED = 2    /* words 0-2 source, 3-5 first pixel centre, 6-8 u, 9-11 v,
                               12 du, 13 dv, 14 radius, 15-17 radial vector */
};
#define DPT_VIEW_MODE_WORD 18

/* Field layouts read by the sampling kernels.
 *  DPT_LAYOUT_REPLICATED  copy written by dpt_b200_prepare_field (default): the cell's eight
 *                         FP32 polynomial coefficients (32 bytes per voxel) for DPT_ARITH_F32C,
 *                         else an FP32 corner quad (16 bytes per voxel) decoded from any
 *                         storage type.
 *  DPT_LAYOUT_DIRECT      eight gathers per sample straight from the caller's FP32 field;
 *                         `packed` then points at the field itself (no copy, FP32 only). */
enum {
    DPT_LAYOUT_REPLICATED = 0,
    DPT_LAYOUT_DIRECT = 1
};

/* VJP flags. */
enum {
    DPT_VJP_VOLUME = 1,      /* scatter the volume cotangent into the accumulator */
    DPT_VJP_POSE12 = 2,      /* per-view packed 12-entry pose cotangent (row-major R, t) */
    DPT_VJP_POSE6 = 4,       /* per-view local-right tangent (tx,ty,tz,rx,ry,rz) */
    DPT_VJP_PER_RAY6 = 8     /* per-ray local-right 6-row Jacobian (weighted by the cotangent) */
};

/* Error codes (negative). */
enum {
    DPT_OK = 0,
    DPT_E_NULL = -1,       /* a required pointer is null */
    DPT_E_SHAPE = -2,      /* a size is out of range */
    DPT_E_DTYPE = -3,      /* unsupported dtype / arithmetic combination */
    DPT_E_FLAGS = -4,      /* inconsistent flags */
    DPT_E_RANGE = -5,      /* view range outside the problem */
    DPT_E_ALIGN = -6,      /* a pointer is not aligned as required */
    DPT_E_CAPACITY = -7    /* a fixed-capacity buffer is too small */
};

/* Fixed description of one projection problem. */
typedef struct dpt_problem {
    int32_t nx, ny, nz;     /* grid sample counts; field is x fastest: (z*ny + y)*nx + x */
    int32_t views;          /* number of views */
    int32_t rows, cols;     /* detector shape per view; bundles use rows=1, cols=rays per view */
    int32_t samples;        /* midpoint samples per ray */
    int32_t ray_kind;       /* DPT_RAYS_* */
    int32_t arith;          /* DPT_ARITH_* */
    int32_t field_dtype;    /* DPT_F32, DPT_F16 or DPT_BF16 */
    int32_t image_dtype;    /* DPT_F32 or DPT_F64: image and cotangent element type */
    int32_t layout;         /* DPT_LAYOUT_*: how the sampling kernels read the field */
    int32_t block_cols;     /* panels: detector columns per 256-ray block tile: 8, 16, 32 or 64
                               (the tile is then 32, 16, 8 or 4 rows high); 0 selects 16 */
    int32_t field_domain;   /* DPT_DOMAIN_*: which field values prepare_field accepts */
    int32_t reserved;       /* 0 */
    double object_to_grid[9]; /* diag(1/h) G^T, row-major: grid index = M (x_object - origin) */
    double grid_origin[3];    /* object mm of sample (0,0,0) */
} dpt_problem;

/* Ray description for one call.  All pointers are device pointers. */
typedef struct dpt_rays {
    const double* poses;        /* views x 12, row-major object-to-world R then t (mm) */
    const double* view_table;   /* views x DPT_VIEW_WORDS, for DPT_RAYS_PANELS */
    const double* ray_sources;  /* views*rows*cols x 3, for DPT_RAYS_BUNDLE */
    const double* ray_endpoints;/* views*rows*cols x 3, for DPT_RAYS_BUNDLE */
    int32_t view_begin;         /* first view of this call */
    int32_t view_count;         /* number of views of this call */
} dpt_rays;

/* Library identity. */
int dpt_b200_abi_version(void);
const char* dpt_b200_error_string(int code);

/* Scratch sizes in bytes (all 256-byte aligned allocations are sufficient). */
size_t dpt_b200_packed_bytes(const dpt_problem* problem);
size_t dpt_b200_accumulator_bytes(const dpt_problem* problem);
size_t dpt_b200_pose_partials_bytes(const dpt_problem* problem, int32_t view_count);

/* Validate the field (bit 8 into status[0]) and every view's rigid pose (bit 1 into
 * status[view]); write the corner-replicated copy of the field used by the sampling
 * kernels into `packed` (dpt_b200_packed_bytes, 16-byte aligned).  A null `packed`
 * only validates (an unchanged field whose copy is still current). */
int dpt_b200_prepare_field(const dpt_problem* problem, const void* field, void* packed,
                           const double* poses, int32_t* status, void* stream);

/* Optical depth of views [view_begin, view_begin+view_count): `image` holds
 * view_count*rows*cols elements of image_dtype in view, row, column order. */
int dpt_b200_forward(const dpt_problem* problem, const dpt_rays* rays, const void* packed,
                     void* image, int32_t* status, void* stream);

/* Discrete VJP of the same views.  `cotangent` matches `image` of dpt_b200_forward.
 * DPT_VJP_VOLUME adds into `accumulator` (dpt_b200_accumulator_bytes, zeroed by the caller
 * before its first use).  A pose flag writes per-block FP64 partials into `pose_partials`
 * (dpt_b200_pose_partials_bytes); dpt_b200_finish_pose turns them into gradients.
 * DPT_VJP_PER_RAY6 writes 6 doubles per ray into `pose_partials` instead. */
int dpt_b200_vjp(const dpt_problem* problem, const dpt_rays* rays, const void* packed,
                 const void* cotangent, int32_t flags, float* accumulator,
                 double* pose_partials, int32_t* status, void* stream);

/* Forward of several problems in one launch: `count` (<= DPT_MAX_PACK) problems
 * of one arithmetic, one field layout and one image dtype (else DPT_E_FLAGS), each with its
 * own rays, field copy (`packed[i]`, as for dpt_b200_forward), image and status words.  One
 * block runs each (view, tile) item of every problem, so many small requests fill the GPU with
 * one launch and no tail between them (2^31 - 1 items at most, else a CUDA error); each image
 * equals its own dpt_b200_forward bit for bit.  No reference counterpart (the reference launches each
 * view of each call separately); a serving loop's batching of small forward requests. */
#define DPT_MAX_PACK 64
int dpt_b200_forward_packed(int32_t count, const dpt_problem* problems, const dpt_rays* rays,
                            const void* const* packed, void* const* images, int32_t* const* status,
                            void* stream);

/* Split pose VJP (DPT_ARITH_F32 or DPT_ARITH_F32C, FP32 images).  A ray's pose moments (its
 * sample sum, sums of the grid slopes and of the position-weighted slopes, and for FP32 the
 * two clip shifts: 9 FP32 words) do not depend on its cotangent.  dpt_b200_forward_moments writes the forward image
 * (identical to dpt_b200_forward) and stores the moments, word k of ray i of the call at
 * moments[k * view_count*rows*cols + i] (dpt_b200_moments_bytes);
 * dpt_b200_pose_from_moments then forms the pose partials of dpt_b200_vjp for one pose
 * form (DPT_VJP_POSE12, POSE6 or PER_RAY6) from the moments and the cotangent without
 * sampling the field, so a training step samples twice (forward with moments, volume VJP)
 * instead of three times.  Results equal those of dpt_b200_vjp with the same flags.
 * Replaces the pose part of python/dpt/projection.py:871-1018 (projection_vjp), kernels
 * python/dpt/kernels/projection_fp32.py:443-458 and 549-615. */
size_t dpt_b200_moments_bytes(const dpt_problem* problem, int32_t view_count);
int dpt_b200_forward_moments(const dpt_problem* problem, const dpt_rays* rays, const void* packed,
                             float* image, float* moments, int32_t* status, void* stream);
int dpt_b200_pose_from_moments(const dpt_problem* problem, const dpt_rays* rays, const float* moments,
                               const void* cotangent, int32_t flags, double* pose_partials,
                               int32_t* status, void* stream);

/* Reduce the pose partials of a dpt_b200_vjp call over views [view_begin, view_begin +
 * view_count) in a fixed FP64 order into `pose_gradient` (view_count x components,
 * components 12 or 6); accumulate != 0 adds.  Non-finite results set bit 2 of
 * status[view]. */
int dpt_b200_finish_pose(const dpt_problem* problem, int32_t view_begin, int32_t view_count,
                         int32_t components,
                         const double* pose_partials, double* pose_gradient, int32_t accumulate,
                         int32_t* status, void* stream);

/* Fold the corner accumulator into per-voxel sums.  `total` (voxels doubles, may be null)
 * receives total (+)= fold in FP64.  When `gradient` is non-null the final FP32
 * (gradient_dtype DPT_F32) or FP64 gradient is written from total (or from the fold when
 * total is null) and scanned for non-finite values (bit 2 into status[0]).  The accumulator
 * is cleared for the next batch when clear != 0. */
int dpt_b200_fold_volume(const dpt_problem* problem, float* accumulator, double* total,
                         int32_t accumulate_total, void* gradient, int32_t gradient_dtype,
                         int32_t clear, int32_t* status, void* stream);

/* Per-ray clip interval (the arithmetic's own lower/upper, as doubles) and the number of
 * midpoint samples that fall inside the half-cell support. */
int dpt_b200_counts(const dpt_problem* problem, const dpt_rays* rays, double* lower,
                    double* upper, int32_t* realised, int32_t* status, void* stream);

/* Pose cotangent of views [view_begin, view_begin+view_count) without any caller scratch
 * and without allocating: for callers that cannot call cudaMalloc while they run (a
 * guidance or tracking loop that reserves its device memory up front, or a plugin whose
 * host application owns the GPU memory).  No counterpart in the reference.  The per-block
 * partials live in a fixed 1 MiB device array inside the library (view_count x blocks per
 * view x components <= 131072, else DPT_E_CAPACITY); the FP32 field is read directly.
 * Every call looks up that array's device address on the current device; the first call on
 * a device also loads the library's device code there, so make it before any stream
 * capture.  Calls that overlap on the GPU share the array and race.  Arithmetic: FP32,
 * FP64, compensated or cell-Gauss (the direct-gather form of each); the problem and rays
 * are checked as by dpt_b200_vjp.  `pose_gradient` is view_count x components (12 packed
 * or 6 local-right); status as dpt_b200_vjp. */
int dpt_b200_pose_vjp_fixed(const dpt_problem* problem, const dpt_rays* rays, const float* field,
                            const void* cotangent, int32_t components, double* pose_gradient,
                            int32_t* status, void* stream);

/* ---------------------------------------------------------------------------------------
 * Deterministic adjoint gather: out[v] = sum_p A[p, v] cotangent[p] for the strict FP64
 * projection, midpoint (arith DPT_ARITH_F64) or cell-Gauss (DPT_ARITH_CELLS; the plan of such
 * a problem validates every ray's cell walk and is not counted), one thread per voxel summing in FP64 in a fixed
 * order (views ascending, each view's sum added to the running value; then detector rows,
 * columns and samples ascending), so the result is bitwise reproducible.  A plan holds the
 * rays of views [view_begin, view_begin + view_count) of `rays` and their culling metrics;
 * the culled sum is bitwise equal to the sum over all rays and samples.
 * ------------------------------------------------------------------------------------- */

/* Bytes of a plan for `view_count` views (32 + 16 x rays per view doubles per view). */
size_t dpt_b200_gather_plan_bytes(const dpt_problem* problem, int32_t view_count);

/* Write the plan: ray records, point-rounding bounds, cone culling metrics.  Invalid rays and
 * non-finite sample points set bit 2 in their view's status word (the plan is then unusable). */
int dpt_b200_gather_prepare(const dpt_problem* problem, const dpt_rays* rays, double* plan,
                            int32_t* status, void* stream);

/* totals[0..3] = candidate rays, sample nodes, voxels over `max_rays_per_voxel` candidate rays
 * in some view, voxels whose culling fell back to the whole panel (summed over views). */
int dpt_b200_gather_count(const dpt_problem* problem, const dpt_rays* rays, const double* plan,
                          int32_t max_rays_per_voxel, int64_t* totals, void* stream);

/* gradient (voxels, DPT_F32 or DPT_F64) = (accumulate ? gradient : 0) + gather of the
 * cotangent (view_count x rows x cols, problem->image_dtype); a non-finite result sets bit 2
 * in status[view_begin]. */
int dpt_b200_gather(const dpt_problem* problem, const dpt_rays* rays, const double* plan,
                    const void* cotangent, void* gradient, int32_t gradient_dtype,
                    int32_t accumulate, int32_t* status, void* stream);

/* ---------------------------------------------------------------------------------------
 * Image-space transmission and objectives.  One thread per pixel; `count` pixels of
 * contiguous device arrays, count <= 2^31 - 1.  FP64 local arithmetic rounded once into
 * each destination.  Scalar results go through a fixed FP64 tree of 256-wide tiles in the
 * caller's `scratch` (dpt_b200_reduction_bytes(count) bytes), so they are deterministic.
 * Compute calls write no input-rule diagnostics: a checked caller runs the matching
 * check call first, reads `status`, and only then computes.  Status bits (status[0]):
 * 1 invalid input, 2 unrepresentable output or gradient, 8 Poisson prediction outside
 * its trial domain.
 * ------------------------------------------------------------------------------------- */

/* Transmission outputs (mask bits) and open-beam forms. */
enum {
    DPT_OUT_TRANSMISSION = 1,      /* T = exp(-L) */
    DPT_OUT_COUNTS = 2,            /* n0 T, formed from the FP64 factor */
    DPT_OUT_LOG_TRANSMISSION = 4,  /* -L (IEEE negation) */
    DPT_OUT_REMOVED = 8            /* 1 - T = -expm1(-L) */
};
enum {
    DPT_BEAM_NONE = 0,
    DPT_BEAM_SCALAR = 1,           /* host scalar `beam_scalar` */
    DPT_BEAM_DEVICE_SCALAR = 2,    /* beam[0] */
    DPT_BEAM_PER_PIXEL = 3         /* beam[p] */
};
/* Input rules of dpt_b200_check_values. */
enum {
    DPT_CHECK_FINITE_NONNEGATIVE = 0,
    DPT_CHECK_FINITE = 1,
    DPT_CHECK_DECREMENT = 2        /* finite, 0 <= v < 1 */
};
/* Objective kinds. */
enum {
    DPT_OBJECTIVE_SQUARED_ERROR = 0,  /* 0.5 (mu - y)^2 */
    DPT_OBJECTIVE_POISSON = 1         /* half-deviance mu - y + y log(y / mu) */
};

/* FP64 scratch bytes of the reduction tree over `count` pixels (or `count` FP64 rows). */
size_t dpt_b200_reduction_bytes(int64_t count);

/* OR bit 1 into status[0] for any value that breaks `rule`. */
int dpt_b200_check_values(const float* values, int64_t count, int32_t rule, int32_t* status,
                          void* stream);

/* Write the outputs selected by `mask` (each non-null when selected). */
int dpt_b200_transmit(const float* depth, int64_t count, int32_t mask, int32_t beam_mode,
                      const float* beam, float beam_scalar, float* transmission, float* counts,
                      float* log_transmission, float* removed, void* stream);

/* grad_depth = -T cT - n0 T cN - cLog + T cR (null cotangents are zero); grad_beam = T cN
 * per pixel (DPT_BEAM_PER_PIXEL) or its fixed-order FP64 sum rounded into grad_beam[0]
 * (DPT_BEAM_DEVICE_SCALAR, needs `scratch`).  At least one gradient; `accumulate` adds
 * each destination before its single rounding. */
int dpt_b200_transmit_vjp(const float* depth, int64_t count, int32_t beam_mode, const float* beam,
                          float beam_scalar, const float* seed_transmission,
                          const float* seed_counts, const float* seed_log_transmission,
                          const float* seed_removed, float* grad_depth, float* grad_beam,
                          double* scratch, int32_t accumulate, int32_t* status, void* stream);

/* depth = -log1p(-removed) and its VJP grad = seed / (1 - removed). */
int dpt_b200_depth_from_removed(const float* removed, int64_t count, float* depth, void* stream);
int dpt_b200_depth_from_removed_vjp(const float* removed, const float* seed, int64_t count,
                                    float* grad, int32_t accumulate, int32_t* status,
                                    void* stream);

/* Fixed-input rules (bit 1) for observation, weights (may be null) and valid (uint8 0/1, may
 * be null) and, with a non-null prediction (DPT_F32 or DPT_F64), bit 2 for a non-finite
 * prediction and bit 8 for a Poisson prediction < 0 or == 0 against a positive count. */
int dpt_b200_objective_check(const void* prediction, int32_t prediction_dtype,
                             const float* observation, const float* weights,
                             const uint8_t* valid, int64_t count, int32_t kind,
                             int32_t integer_counts, int32_t* status, void* stream);

/* loss[0] = sum_p valid_p normalisation weights_p ell(prediction_p, observation_p) (FP64;
 * null skips the loss) and seed_p = d/d prediction_p of that term times seed_scale, rounded
 * once into the prediction's dtype (null skips the seed).  `wide` selects the FP64
 * precision forms (required for DPT_F64; with DPT_F32 the FP32 prediction is widened). */
int dpt_b200_objective(const void* prediction, int32_t prediction_dtype, int32_t wide,
                       const float* observation, const float* weights, const uint8_t* valid,
                       int64_t count, int32_t kind, double normalisation, double seed_scale,
                       void* seed, double* scratch, double* loss, int32_t* status,
                       void* stream);

/* total[0] = fixed-order FP64 sum of `count` values (zero when empty). */
int dpt_b200_reduce_sum(const double* values, int64_t count, double* scratch, double* total,
                        int32_t* status, void* stream);

/* ---- measurement --------------------------------------------------------------------
 * No reference counterpart: the roofline the benchmark reports for the gather kernels.
 * Reads `bytes` (a multiple of 16) from the 16-byte aligned device `buffer` `passes` times
 * in one launch (no writes; `sink` is one device float that is written only if the
 * buffer's sum is NaN).  Bandwidth = passes * bytes / launch time; for a buffer that fits
 * in L2 this is the L2 read rate of the device. */
int dpt_b200_read_probe(const void* buffer, int64_t bytes, int32_t passes, float* sink, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DPT_B200_H */
