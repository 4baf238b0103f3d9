/*
 * pacman_b200 -- C ABI of the B200 (sm_100a) RBF-PUM transfer.
 *
 * Drop-in engine for PACMAN's RBF-PUM path (messahelramzi/pacman).  Plain C
 * types only: no C++, CUDA or torch types cross this boundary, no exception
 * crosses it, every entry point returns 0 or a negative PACMAN_B200_ERR_*
 * code, and pacman_b200_last_error() gives the calling thread's message
 * (the convention of the reference's C shim, src/fortran_interface.cpp:84-90).
 *
 * Pointers may be host memory or CUDA device memory of the selected device;
 * each one is classified with cudaPointerGetAttributes.  Points are row-major
 * [count x dim] doubles, values are row-major [n_source x n_fields] doubles,
 * outputs are row-major [n_target x n_fields] doubles.  Inputs are never
 * modified.  Targets outside every patch receive 0 (the reference zero-fills,
 * src/common/transfer.hxx:101-110).
 */
#ifndef PACMAN_B200_H
#define PACMAN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PACMAN_B200_ABI_VERSION 6

#if defined(__GNUC__)
#define PACMAN_B200_API __attribute__((visibility("default")))
#else
#define PACMAN_B200_API
#endif

/* Error codes. */
#define PACMAN_B200_OK 0
#define PACMAN_B200_ERR_INVALID (-1)    /* bad argument (std::invalid_argument in the reference) */
#define PACMAN_B200_ERR_DIMENSION (-2)  /* dim not in {1,2,3} (std::runtime_error in the reference) */
#define PACMAN_B200_ERR_CUDA (-3)       /* CUDA runtime error or no usable device */
#define PACMAN_B200_ERR_NOMEM (-4)      /* device allocation failed */
#define PACMAN_B200_ERR_DEGENERATE (-5) /* zero or non-finite patch radius */
#define PACMAN_B200_ERR_LIMIT (-6)      /* a documented size limit was exceeded */

/* Basis selector bytes, identical to PACMAN::RbfFunctions (src/interface.hpp:25-31). */
#define PACMAN_B200_WENDLAND_C0 0x10
#define PACMAN_B200_WENDLAND_C2 0x11
#define PACMAN_B200_WENDLAND_C4 0x12
#define PACMAN_B200_WENDLAND_C6 0x13
#define PACMAN_B200_WENDLAND_C8 0x14

/* Execution-space selector bytes of PACMAN::ExecSpaces
 * (src/common/execspaces.hpp:17-24).  All of them select the B200 path. */
#define PACMAN_B200_EXEC_SERIAL 0x00
#define PACMAN_B200_EXEC_OPENMP 0x01
#define PACMAN_B200_EXEC_THREADS 0x02
#define PACMAN_B200_EXEC_CUDA 0x03
#define PACMAN_B200_EXEC_HIP 0x04
#define PACMAN_B200_EXEC_SYCL 0x05

/* Precision of the per-patch solves. */
#define PACMAN_B200_FP64 0  /* the reference algorithm: unpivoted LU in FP64 */
#define PACMAN_B200_MIXED 1 /* Cholesky (A is symmetric positive definite):
                               small patches in FP64 registers, the column
                               updates of large patches as split-integer
                               products on the int8 tensor cores (FP64-level
                               accuracy); a failed patch is re-solved by the
                               FP64 LU */

typedef struct pacman_b200_options {
  int32_t nodes_per_cluster; /* 50: RbfPumInterpolator default, src/rbf_pum/interpolator.hxx:39 */
  double relative_overlap;   /* 0.15: interpolator.hxx:40 */
  double support_radius;     /* 0.1: interpolator.hxx:41 (absolute basis support) */
  int32_t precision;         /* PACMAN_B200_FP64 or PACMAN_B200_MIXED */
  int32_t device;            /* CUDA device ordinal, -1 = the current device */
  void *stream;              /* cudaStream_t to run on, NULL = a library-owned stream */
} pacman_b200_options;

typedef struct pacman_b200_stats {
  double radius;            /* patch radius (clusters_radius.hpp:121-124) */
  int64_t num_candidates;   /* candidate centres before pruning */
  int64_t num_patches;      /* K, surviving centres */
  int64_t sum_n, sum_m;     /* total patch sources / targets */
  int64_t max_n;            /* largest patch */
  int64_t patches_fp32;     /* patches factored in FP32: always 0 (the mixed
                               path emulates FP64 products on the int8 tensor
                               cores instead; FP32 factors of these matrices
                               do not refine to the 1e-10 bound) */
  int64_t patches_fp64;     /* patches solved at FP64 accuracy */
  int64_t patches_fallback; /* mixed-path patches re-solved by the FP64 LU
                               (non-positive pivot or a pipeline time-out) */
  int64_t dropped_axis_patches; /* patches whose linear polynomial lost an axis */
  double ms_geometry;       /* device time of radius + centres + membership */
  double ms_solve;          /* device time of the patch solves */
  double ms_total;          /* device time of the whole call */
  int64_t kernel_launches;  /* this library's kernel launches in the call */
  double ms_factor;         /* device time of the dense factorisations */
  double factor_flops;      /* algorithmic FLOPs of those factorisations */
  /* With PACMAN_B200_TIME_KERNELS: the step launches of the large-patch
   * Cholesky (the dominant kernels), each bracketed by CUDA events on its
   * own stream: the span of device time during which at least one of them
   * runs (slot groups run concurrently on their streams, so this is the
   * union of the launch intervals, not their sum), their algorithmic
   * FP64-equivalent FLOPs (2 * 64^3 per tile product) and launch count. */
  double ms_update;
  double update_flops;
  int64_t update_launches;
  /* Patches solved from factorisations kept by an earlier execute
   * (PACMAN_B200_KEEP_FACTORS). */
  int64_t factors_reused;
  /* The same three figures per kind of step launch: the column updates on
   * the int8 tensor cores (k_col_step_ws) and those in FP64 (k_col_step).
   * The FLOPs of a step count (j + 1) tile products per row tile: the j of
   * the column update and one for the triangular solve. */
  double ms_update_i8;
  double update_flops_i8;
  int64_t update_launches_i8;
  double ms_update_f64;
  double update_flops_f64;
  int64_t update_launches_f64;
  /* Host synchronisations (waits for the device) inside the call. */
  int64_t host_syncs;
  /* 64 x 64 x 64 tile products of the column updates on the int8 tensor
   * cores alone (j per row tile and per next diagonal tile at step j); each
   * is 34 int8 digit products (slice pairs a + b <= 9 of 7 slices). */
  double mma_products_i8;
} pacman_b200_stats;

/* Fills the reference's defaults (50, 0.15, 0.1, FP64, current device). */
PACMAN_B200_API void pacman_b200_options_init(pacman_b200_options *opts);

/*
 * One RBF-PUM transfer, the engine behind PACMAN::rbf_interpolate
 * (replaces src/rbf_interface.cpp:101-130 -> RbfPumInterpolator,
 * src/rbf_pum/interpolator.hpp:58-94) for n_fields fields at once.
 * opts may be NULL (defaults); stats may be NULL.
 */
PACMAN_B200_API int pacman_b200_rbf_interpolate(int32_t dim, int32_t rbf_function,
                                 const double *source_points, int64_t n_source,
                                 const double *source_values, int32_t n_fields,
                                 const double *target_points, int64_t n_target,
                                 double *target_values,
                                 const pacman_b200_options *opts,
                                 pacman_b200_stats *stats);

/* One problem of a batched call. */
typedef struct pacman_b200_problem {
  int32_t dim;                 /* 1, 2 or 3 */
  int32_t rbf_function;        /* PACMAN_B200_WENDLAND_C0 .. C8 */
  const double *source_points; /* n_source x dim, row-major (host or device) */
  int64_t n_source;
  const double *source_values; /* n_source x n_fields, row-major */
  int32_t n_fields;            /* 1 .. 8 */
  const double *target_points; /* n_target x dim, row-major */
  int64_t n_target;
  double *target_values;       /* out: n_target x n_fields (host or device) */
} pacman_b200_problem;

/*
 * Many independent transfers in one call.  No counterpart in the reference,
 * which runs one transfer per call: here the geometry is built per problem,
 * then the patches of all problems that share (dim, rbf_function, n_fields)
 * are solved together in one set of launches, and each problem's
 * partition-of-unity sum is formed from them.  Results equal
 * pacman_b200_rbf_interpolate on each problem.  opts (shared by all problems,
 * may be NULL) and stats (totals, may be NULL) as there.
 */
PACMAN_B200_API int pacman_b200_rbf_interpolate_batch(const pacman_b200_problem *problems,
                                                      int32_t count,
                                                      const pacman_b200_options *opts,
                                                      pacman_b200_stats *stats);

/* Reusable transfer plan: the geometry (patch radius, centre cover, patch
 * membership lists; src/rbf_pum/interpolator.hpp:76-92 and solver.hpp:45-66)
 * is built once and each execute solves for new source values.  The plan
 * copies the points to the device; the caller may free them afterwards. */
typedef struct pacman_b200_plan pacman_b200_plan;

PACMAN_B200_API int pacman_b200_plan_create(int32_t dim, const double *source_points, int64_t n_source,
                            const double *target_points, int64_t n_target,
                            const pacman_b200_options *opts, pacman_b200_plan **plan);
PACMAN_B200_API int pacman_b200_plan_execute(pacman_b200_plan *plan, int32_t rbf_function,
                             const double *source_values, int32_t n_fields,
                             double *target_values, pacman_b200_stats *stats);
PACMAN_B200_API void pacman_b200_plan_destroy(pacman_b200_plan *plan);

/* Adjoint of the transfer (no counterpart in the reference, which only
 * evaluates the forward map).  execute_ex with PACMAN_B200_SAVE_FOR_ADJOINT
 * keeps the per-patch coefficients of that call; plan_adjoint then applies
 * the transpose of the (fixed-geometry, linear in the values) transfer to an
 * upstream gradient grad_target_values [n_target x n_fields]:
 *   grad_source_values [n_source x n_fields] = M^T grad   (may be NULL),
 *   grad_target_points [n_target x dim]       = d <grad, out> / d targets
 *                                               at fixed patch membership
 *                                               (may be NULL). */
#define PACMAN_B200_SAVE_FOR_ADJOINT 1u
/* Times every launch of the dominant kernel with CUDA events on its stream
 * (one slot group, no concurrent groups) and reports it in the stats. */
#define PACMAN_B200_TIME_KERNELS 2u
/* Reusable factorisations (precision PACMAN_B200_MIXED; no counterpart in
 * the reference, which refactors every patch matrix on every call).  The
 * patch matrices depend only on the geometry and the basis, so a coupling
 * loop that transfers new values over fixed point sets factors them once:
 * the first execute with this flag factors every patch and keeps the
 * factors in the plan (device memory: about n^2 doubles per patch, n^2 / 2
 * rounded up to 64 x 64 tiles for the large ones); later executes with the
 * flag and the same basis run only the polynomial block, the triangular
 * solves and the evaluation.  Another basis refactors and replaces them; an
 * execute without the flag leaves them untouched; pacman_b200_plan_shard
 * drops them.  Precision PACMAN_B200_FP64 keeps nothing. */
#define PACMAN_B200_KEEP_FACTORS 4u
PACMAN_B200_API int pacman_b200_plan_execute_ex(pacman_b200_plan *plan, int32_t rbf_function,
                                                const double *source_values, int32_t n_fields,
                                                double *target_values, uint32_t flags,
                                                pacman_b200_stats *stats);
PACMAN_B200_API int pacman_b200_plan_adjoint(pacman_b200_plan *plan,
                                             const double *grad_target_values,
                                             double *grad_source_values,
                                             double *grad_target_points);

/* Geometry of a plan, for inspection and parity tests.
 * info[0] = K, info[1] = candidates, info[2] = total source memberships,
 * info[3] = total target memberships; *radius = patch radius. */
PACMAN_B200_API int pacman_b200_plan_info(const pacman_b200_plan *plan, double *radius, int64_t info[4]);
/* Patch centres, K x dim row-major (host or device buffer). */
PACMAN_B200_API int pacman_b200_plan_centers(const pacman_b200_plan *plan, double *centers);
/* Membership lists in CSR form (ascending point ids within a patch):
 * which = 0 sources, 1 targets; offsets has K+1 entries. */
PACMAN_B200_API int pacman_b200_plan_patch_lists(const pacman_b200_plan *plan, int32_t which,
                                 int64_t *offsets, int32_t *indices);
/* Per (patch, target) local interpolant values of the last execute, in the
 * order of the target membership lists, times n_fields. */
PACMAN_B200_API int pacman_b200_plan_local_values(const pacman_b200_plan *plan, double *local);

/* Per-patch status words of the plan's last execute, K entries into host
 * memory: which patches lost a polynomial axis, which were re-solved and
 * why.  No counterpart in the reference, which has no per-patch checks
 * after its LU (src/rbf_pum/solver/utils/serial_solve.hpp:76-84).  Bits: */
#define PACMAN_B200_PATCH_DROPPED_AXIS 1 /* the linear polynomial lost an axis */
#define PACMAN_B200_PATCH_NONFINITE 2    /* a non-finite local value */
#define PACMAN_B200_PATCH_BREAKDOWN 4    /* non-positive Cholesky pivot (mixed) */
#define PACMAN_B200_PATCH_TIMEOUT 8      /* a bounded tensor-core pipeline wait gave up */
#define PACMAN_B200_PATCH_RESOLVED 16    /* re-solved by the FP64 LU after 2, 4 or 8 */
PACMAN_B200_API int pacman_b200_plan_patch_status(const pacman_b200_plan *plan, int32_t *status);

/*
 * Finite-element transfer of the reference's PACMAN::fe_interpolate
 * (src/interface.hpp:76-80, src/interface.cpp:89-121) for the method
 * NEAREST_NEAREST (0xF0, src/common/types.hpp:29-37; FTNearest.hpp:27-56):
 * target_values[t] = source_values[nearest source] (lowest index on ties), 0
 * without sources; target_status[t] = 0 (OUTSIDE: the reference's
 * NEAREST_NEAREST leaves the zero-initialised status as it is; may be NULL).
 * The point-based method reads no connectivity, so none is passed.  Other
 * methods return PACMAN_B200_ERR_INVALID.  Arrays may be host or device
 * memory of opts->device; opts (device, stream) may be NULL.
 */
#define PACMAN_B200_FE_NEAREST_NEAREST 0xF0
PACMAN_B200_API int pacman_b200_fe_interpolate(int32_t dim, int32_t method,
                                               const double *source_points, int64_t n_source,
                                               const double *source_values,
                                               const double *target_points, int64_t n_target,
                                               double *target_values, int32_t *target_status,
                                               const pacman_b200_options *opts);

/*
 * Moving least squares transfer of the reference's PACMAN::MLS_interpolate
 * (src/interface.hpp:148-170, src/mls_interface.cpp; the arithmetic of
 * ArborX 2.1's Interpolation::MovingLeastSquares with its defaults, called at
 * src/mls/interpolator.hpp:49-77): for each target the K nearest sources
 * (K = 3, 6, 10 in 1D, 2D, 3D; lowest index on ties; all sources when fewer),
 * Wendland C0 weights over 1.1 x the farthest neighbour's distance, and the
 * value at the target of the weighted least-squares quadratic (pseudo-inverse
 * of the moment matrix, eigenvalues below 1e-13 of the largest dropped).
 * One scalar field; 0 at every target without sources.  Arrays may be host or
 * device memory of opts->device; opts (device, stream) may be NULL.  Errors:
 * PACMAN_B200_ERR_INVALID (null pointer with a non-zero count, negative
 * count), PACMAN_B200_ERR_DIMENSION, PACMAN_B200_ERR_LIMIT (counts >= 2^31).
 */
PACMAN_B200_API int pacman_b200_mls_interpolate(int32_t dim, const double *source_points,
                                                int64_t n_source, const double *source_values,
                                                const double *target_points, int64_t n_target,
                                                double *target_values,
                                                const pacman_b200_options *opts);

/*
 * Target sharding of one transfer over `world` GPUs, one process per GPU
 * (no counterpart in the reference, which runs on one device).  Every rank
 * creates the same plan (all sources, all targets: the patch cover depends on
 * both) and calls this with its rank.  The targets are cut into `world`
 * ranges of their Morton order over the source bounding box, balanced by the
 * solve cost n^3 of the patches each range needs; the cut uses integer data
 * only, so all ranks agree on it.  Afterwards an execute solves only the
 * patches holding an owned target, writes the owned targets' values (bit-
 * identical to the unsharded transfer) and zero elsewhere: the sum over the
 * ranks (one all-reduce) is the whole result.  The adjoint of a sharded plan
 * gives this shard's contribution to the source-value gradient and the
 * owned targets' coordinate gradients.  A plan is sharded once.
 */
PACMAN_B200_API int pacman_b200_plan_shard(pacman_b200_plan *plan, int32_t rank, int32_t world);

/* Targets of the plan's shard (all targets for an unsharded plan): their
 * number in *count, and, when owned is not NULL, their indices ascending
 * (*count entries). */
PACMAN_B200_API int pacman_b200_plan_owned_targets(const pacman_b200_plan *plan, int64_t *count,
                                                   int32_t *owned);

/*
 * Patch radius (the transfer's cluster-size heuristic: 2*dim+1 sample points
 * projected onto their nearest source, k-th nearest source distance with
 * k = nodes_per_cluster, median) WITHOUT ANY DEVICE ALLOCATION.  No
 * counterpart in the reference: it exists for callers that cannot let a
 * library allocate device memory, e.g. a coupled code that reserves the GPU
 * for its own pool allocator at start-up.  Its working memory is one fixed
 * 16 KiB file-scope __device__ array, present on every GPU that loads this
 * library until the process exits.  Every call resolves that array's address
 * (cudaGetSymbolAddress) in the context current on the calling thread, so a
 * cudaDeviceReset or a context the caller made current is followed.  The
 * call synchronises the stream to read the radius back, so it cannot be
 * captured into a CUDA graph.  Calls share the array: calls that overlap on
 * the GPU race and must be serialised by the caller.
 * source_points: device memory of the current device, row-major [n x dim];
 * limits: dim <= 3 (the array holds at most 7 samples), 1 <= n <= 2^31 - 1.
 * stream: cudaStream_t (NULL = default stream); the call returns after
 * *radius (host or device pointer) has been written.  A radius that is zero
 * or not finite (all sources coincide) is written and reported as
 * PACMAN_B200_ERR_DEGENERATE, as the full transfer reports it.
 */
PACMAN_B200_API int pacman_b200_patch_radius_noalloc(int32_t dim, const double *source_points,
                                                     int64_t n_source, int32_t nodes_per_cluster,
                                                     void *stream, double *radius);

/* Message of the last error on the calling thread ("" if none). */
PACMAN_B200_API const char *pacman_b200_last_error(void);
PACMAN_B200_API int32_t pacman_b200_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PACMAN_B200_H */
