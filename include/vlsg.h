/*
 * vlsg.h -- C ABI of the B200 level-set advection library (libvlsgpu.so).
 *
 * This is the boundary a host front binds to in place of
 * viennals::Advect<T,D>::apply (include/viennals/lsAdvect.hpp:1017-1043 of
 * ViennaLS 5.8.3).  Every entry point takes plain pointers and sizes, returns
 * an int status (VLSG_OK == 0, negative on error) and leaves a message for
 * vlsg_last_error(), mirroring the error model of the reference (log + return,
 * lsAdvect.hpp:1019-1027) and the handle/last-error style of the reference's
 * own GPU interface (lsOxidationBiCGSTABInterface.hpp:27-73).
 *
 * Threading: one context == one CUDA stream; a context must be used by one
 * host thread at a time (viennals::Advect is not re-entrant either).
 *
 * Level-set exchange format: a level set is the sequence that the reference's
 * viennahrle::ConstSparseIterator yields -- defined points (index, value) and
 * undefined runs (start index, sign) in HRLE lexicographic order (x fastest,
 * highest dimension slowest).  Upload takes both lists; download returns the
 * defined points in the same order.  Values are in grid units (signed
 * distance / gridDelta), as lsDomain stores them.
 */
#ifndef VLSG_H
#define VLSG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VLSG_OK 0
#define VLSG_ERR_ARGUMENT -1     /* bad argument / unsupported option        */
#define VLSG_ERR_CUDA -2         /* CUDA runtime error                       */
#define VLSG_ERR_CAPACITY -3     /* pool / brick map capacity exceeded        */
#define VLSG_ERR_STATE -4        /* call out of order (no grid, no level set) */
#define VLSG_ERR_NUMERIC -5      /* time step <= 0, step limit reached        */
#define VLSG_ERR_DEVICE_CHECK -6 /* a kernel's own bounds check fired         */
#define VLSG_ERR_CALLBACK -7     /* the host velocity callback failed         */

#define VLSG_MAX_LEVEL_SETS 8
#define VLSG_MAX_MATERIALS 16

/* SpatialSchemeEnum, lsAdvectIntegrationSchemes.hpp:10-23 (same values). */
enum vlsg_spatial_scheme {
  VLSG_ENGQUIST_OSHER_1ST_ORDER = 0,
  VLSG_ENGQUIST_OSHER_2ND_ORDER = 1,
  VLSG_LAX_FRIEDRICHS_1ST_ORDER = 2,
  VLSG_LAX_FRIEDRICHS_2ND_ORDER = 3,
  VLSG_LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER = 4,
  VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER = 5,
  VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_2ND_ORDER = 6,
  VLSG_LOCAL_LAX_FRIEDRICHS_1ST_ORDER = 7,
  VLSG_LOCAL_LAX_FRIEDRICHS_2ND_ORDER = 8,
  VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER = 9,
  VLSG_WENO_3RD_ORDER = 10,
  VLSG_WENO_5TH_ORDER = 11
};

/* TemporalSchemeEnum, lsAdvectIntegrationSchemes.hpp:31-35. */
enum vlsg_temporal_scheme {
  VLSG_FORWARD_EULER = 0,
  VLSG_RUNGE_KUTTA_2ND_ORDER = 1,
  VLSG_RUNGE_KUTTA_3RD_ORDER = 2
};

/* viennahrle::BoundaryType (python/viennals/_core.pyi:25-30). */
enum vlsg_boundary {
  VLSG_REFLECTIVE_BOUNDARY = 0,
  VLSG_INFINITE_BOUNDARY = 1,
  VLSG_PERIODIC_BOUNDARY = 2,
  VLSG_POS_INFINITE_BOUNDARY = 3,
  VLSG_NEG_INFINITE_BOUNDARY = 4
};

/* Storage / stencil precision of a context.  FP64 reproduces the reference's
 * Advect<double,3> rule for rule; FP32 stores phi and evaluates the stencils
 * in float, keeping the CFL reduction, the advected time and the RK stage
 * combination in double. */
enum vlsg_precision { VLSG_FP64 = 0, VLSG_FP32 = 1 };

/* All setters of viennals::Advect (lsAdvect.hpp:856-969) in one struct.
 * vlsg_default_params() fills the reference defaults (lsAdvect.hpp:64-79). */
typedef struct vlsg_advect_params {
  int32_t spatial_scheme;          /* setSpatialScheme            :936 */
  int32_t temporal_scheme;         /* setTemporalScheme           :949 */
  double time_step_ratio;          /* setTimeStepRatio (0.4999)   :885 */
  double dissipation_alpha;        /* setDissipationAlpha (1.0)   :955 */
  double advection_time;           /* setAdvectionTime (0)        :873 */
  int32_t single_step;             /* setSingleStep               :879 */
  int32_t calculate_normal_vectors;/* setCalculateNormalVectors   :891 */
  int32_t ignore_voids;            /* setIgnoreVoids (must be 0)  :899 */
  int32_t adaptive_time_stepping;  /* setAdaptiveTimeStepping     :904 */
  uint32_t adaptive_subdivisions;  /*   (20)                      :904 */
  int32_t check_dissipation;       /* setCheckDissipation (1)     :958 */
  int32_t save_advection_velocities; /* setSaveAdvectionVelocities :916 */
  int32_t update_point_data;       /* setUpdatePointData (1)      :962 */
  uint32_t max_steps;              /* guard against dt == 0 loops (0 = 1e7) */
  double max_dissipation;          /* StencilLocalLaxFriedrichsScalar::
                                      setMaxDissipation (lsStencilLocalLax
                                      FriedrichsScalar.hpp:215); <= 0 means
                                      no limit (the reference's default) */
  int32_t track_point_data;        /* carry the top level set's point data
                                      through the advection (the source ids
                                      of translateFromMultiData); read it with
                                      vlsg_download_point_data.  Implied by
                                      save_advection_velocities. */
  int32_t fp32_compensation;       /* FP32 contexts: the value update and the
                                      RK stage combination keep their FP64
                                      result as an FP32 value plus an FP32
                                      compensation term (the top level set
                                      and its RK copy); downloads return the
                                      sum.  Costs about 18% of an RK3 step;
                                      0 (default): the FP64 results are
                                      rounded to FP32 once. */
} vlsg_advect_params;

/* Getters of viennals::Advect (lsAdvect.hpp:920-932) plus work counters. */
typedef struct vlsg_advect_result {
  double advected_time;        /* getAdvectedTime     */
  double current_time_step;    /* getCurrentTimeStep  */
  uint32_t number_of_time_steps; /* getNumberOfTimeSteps */
  uint32_t number_of_stages;   /* forward-Euler stages executed */
  uint64_t point_updates;      /* sum over stages of active points */
  uint64_t kernel_launches;    /* kernels this library launched */
} vlsg_advect_result;

/* Device velocity functor: evaluates, for material m (clamped to
 * n_materials-1) and unit normal n,
 *   scalar = rate[m]
 *          + sum_k (n_k > 0 ? lin_pos : lin_neg)[m][k] * n_k
 *          + sum_k (n_k > 0 ? abs_pos : abs_neg)[m][k] * |n_k|
 *          + sum_k (n_k > 0 ? sq_pos  : sq_neg )[m][k] * (n_k * n_k)
 * in exactly that order, skipping terms whose coefficient is 0 (so a
 * constant field never reads a normal), and vector = vec[m].
 * This covers the fields of the reference's tests and examples
 * (TimeIntegration.cpp:17-35, Advection.cpp:25-44,
 * MultiMaterialEtch.cpp:30-49, SquareEtch.cpp:26-41).  Any other
 * VelocityField goes through vlsg_set_velocity_callback. */
typedef struct vlsg_velocity_desc {
  int32_t n_materials;
  double rate[VLSG_MAX_MATERIALS];
  double lin_pos[VLSG_MAX_MATERIALS][3];
  double lin_neg[VLSG_MAX_MATERIALS][3];
  double abs_pos[VLSG_MAX_MATERIALS][3];
  double abs_neg[VLSG_MAX_MATERIALS][3];
  double sq_pos[VLSG_MAX_MATERIALS][3];
  double sq_neg[VLSG_MAX_MATERIALS][3];
  double vec[VLSG_MAX_MATERIALS][3];
  /* getDissipationAlpha(direction, material, centralDifferences) =
   * alpha[material][direction] (lsVelocityField.hpp:35-38; the scheme
   * LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER asks it, e.g. the constant
   * per-direction alphas of SquareEtch.cpp:66-83). */
  double alpha[VLSG_MAX_MATERIALS][3];
} vlsg_velocity_desc;

/* Host velocity callback (viennals::VelocityField<T>::getScalarVelocity and
 * getVectorVelocity, lsVelocityField.hpp:17-30, batched).  Called with n
 * queries; coords = index * gridDelta, normals as the scheme computes them,
 * point_ids = HRLE linear id of the centre point.  Must fill scalar_out[n]
 * and vector_out[3n]; return 0 on success.  It may be called from several
 * host threads at once for disjoint batches (as the reference calls the
 * virtuals from OpenMP threads, lsAdvect.hpp:464). */
typedef int (*vlsg_velocity_cb)(void *user, int64_t n, const double *coords,
                                const int32_t *materials,
                                const double *normals,
                                const uint64_t *point_ids, double *scalar_out,
                                double *vector_out);

/* Host dissipation-alpha callback (VelocityField::getDissipationAlpha,
 * lsVelocityField.hpp:35-38, batched) for LOCAL_LAX_FRIEDRICHS_ANALYTICAL
 * with a host velocity callback: n queries of (direction, material, the
 * three central differences of lsLocalLaxFriedrichsAnalytical.hpp:199-209);
 * fills alpha_out[n]; returns 0 on success.  Without one, the alphas are 0
 * (the reference's default). */
typedef int (*vlsg_alpha_cb)(void *user, int64_t n, const int32_t *directions,
                             const int32_t *materials,
                             const double *central_differences,
                             double *alpha_out);

/* A level set as the velocity-update callback sees it: defined points and
 * undefined runs in HRLE order (valid during the call only). */
typedef struct vlsg_levelset_view {
  int64_t n_points;
  const int32_t *indices; /* 3 per point */
  const double *values;
  int64_t n_runs;
  const int32_t *run_start; /* 3 per run */
  const int8_t *run_sign;
  int32_t width;
} vlsg_levelset_view;

/* setVelocityUpdateCallback (lsAdvect.hpp:966-969): called by the RK2/RK3
 * schemes between stages with the top level set (lsAdvectIntegrationSchemes
 * .hpp:88-89, :129-130, :147-149), e.g. to recompute the velocity field it
 * feeds.  Returning non-zero ends apply() with VLSG_ERR_CALLBACK (the
 * reference ignores the callback's bool). */
typedef int (*vlsg_update_cb)(void *user, const vlsg_levelset_view *top);

typedef struct vlsg_context vlsg_context;

/* Library / context lifetime ---------------------------------------------- */
int vlsg_version(void);
const char *vlsg_last_error(const vlsg_context *ctx); /* ctx may be NULL */
int vlsg_create(vlsg_context **out, int32_t device, int32_t precision);
int vlsg_destroy(vlsg_context *ctx);
void vlsg_default_params(vlsg_advect_params *p);
/* The CUDA stream (cudaStream_t) every kernel of the context runs on; a
 * caller may hand in its own stream (NULL restores the context's own). */
int vlsg_set_stream(vlsg_context *ctx, void *stream);
int vlsg_get_stream(vlsg_context *ctx, void **stream);

/* Grid: Domain(bounds, boundaryConditions, gridDelta), lsDomain.hpp:68-78.
 * grid_min/grid_max are INDEX bounds (floor(min/dx), ceil(max/dx)); for a
 * periodic direction the points are grid_min..grid_max-1, for a reflective
 * one grid_min..grid_max, an infinite direction is unbounded.
 * dim = 2 (Advect<T,2>): grid_min, grid_max and boundary hold 2 entries; the
 * level set is held as the plane z = 0 of a grid periodic in z with period
 * 1, so every z neighbour of a point is the point itself and every z
 * difference is 0.  Every index array of the other entry points keeps 3
 * int32 per point or run start, the third 0 (downloads return 0 there); the
 * velocity field sees coordinates and normals with a zero z component.
 * The schemes that ask the velocity field around a point (LocalLaxFriedrichs,
 * LLF-analytical, Stencil-LLF) ask it at the plane's 3x3 box only, in the
 * directions x and y, as the 2D reference does. */
int vlsg_set_grid(vlsg_context *ctx, int32_t dim, const int64_t *grid_min,
                  const int64_t *grid_max, const int32_t *boundary,
                  double grid_delta);

/* Level sets are numbered bottom (0) to top (n-1) like the vector passed to
 * Advect (lsAdvect.hpp:46-53); the top one is advected and must wrap the
 * others.  vlsg_set_level_set_count drops slots >= n. */
int vlsg_set_level_set_count(vlsg_context *ctx, int32_t n);
int vlsg_upload_levelset(vlsg_context *ctx, int32_t slot, int64_t n_points,
                         const int32_t *indices, const double *values,
                         int64_t n_runs, const int32_t *run_start,
                         const int8_t *run_sign, int32_t width);
int vlsg_count_points(vlsg_context *ctx, int32_t slot, int64_t *n_points);
int vlsg_download_levelset(vlsg_context *ctx, int32_t slot, int64_t capacity,
                           int32_t *indices, double *values, int32_t *width);

/* Undefined runs of a level set in HRLE order -- what viennahrle's sparse
 * iterators yield besides the defined points (lsDomain.hpp:51-52: an
 * undefined run carries +-max with its sign) -- over the box [min - 1,
 * max + 1] of the defined points: one run before the box, per z-plane one
 * run before and one after its rows, per row a run at its head (or one for
 * a row without points) and one after every point not followed by its +x
 * neighbour, one run after the box; a run with the previous run's sign and
 * no defined point between them is merged into it.  Start indices below the
 * box are -(2^20 - 2).  Writes *n_runs; with capacity < *n_runs nothing is
 * written and VLSG_ERR_CAPACITY is returned (call with capacity 0 to ask). */
int vlsg_download_runs(vlsg_context *ctx, int32_t slot, int64_t capacity,
                       int32_t *run_start, int8_t *run_sign, int64_t *n_runs);

/* Point data of the top level set after vlsg_advect with track_point_data
 * or save_advection_velocities (replaces reading Domain::getPointData()
 * after Advect::apply).  Per defined point, in the order of
 * vlsg_download_levelset:
 *   source[i]      the index (in the download order of the top level set as
 *                  it was when that vlsg_advect started) of the point whose
 *                  data point i now carries -- the source ids the reference's
 *                  Expand, Reduce, Prune, BooleanOperation and rebuildLS pass
 *                  to translateFromMultiData (lsExpand.hpp:110-150,
 *                  lsAdvect.hpp:318-410, lsBooleanOperation.hpp:104-114);
 *                  -1 where the reference records none;
 *   velocity[i]    "AdvectionVelocities": the rate of the last value update
 *                  (lsAdvect.hpp:764-767, 794), with save_advection_velocities;
 *   dissipation[i] "Dissipation" (lsAdvect.hpp:795); 0 without it.
 * *has_point_data = 0 (and nothing else written) when the top level set
 * carries none: no tracking was asked for, or update_point_data was 0, in
 * which case rebuildLS drops all point data (lsAdvect.hpp:418-423).
 * Only the top level set (slot = count - 1); VLSG_ERR_CAPACITY when capacity
 * is below the number of points (vlsg_count_points). */
int vlsg_download_point_data(vlsg_context *ctx, int32_t slot, int64_t capacity,
                             int64_t *source, double *velocity, double *dissipation,
                             int32_t *has_point_data);

/* Values of arbitrary grid points of a level set (indices are mapped through
 * the boundary conditions): the defined value, or +-DBL_MAX carrying the sign
 * of the undefined region -- what viennahrle's iterators return for them
 * (lsDomain.hpp:51-52).  Used to rebuild the undefined runs of a downloaded
 * level set. */
int vlsg_get_values(vlsg_context *ctx, int32_t slot, int64_t n,
                    const int32_t *indices, double *values);

/* vlsg_get_values without any device allocation.  It has no counterpart in
 * the reference.  It serves callers that may not allocate device memory once
 * their set-up is done: an application whose memory pool (a framework's
 * caching allocator, a fixed budget shared with other GPU work) already holds
 * the device's free memory, or a loop that must not stall the other streams
 * of the device, which cudaMalloc and cudaFree can do.  vlsg_get_values
 * stages the query indices and the returned values in device buffers it
 * allocates and frees on every call; this entry point stages them instead in
 * one static device array of the library, sized for VLSG_NOALLOC_MAX_QUERIES
 * queries (1.25 MiB per GPU, held until the process exits).
 *   - n > VLSG_NOALLOC_MAX_QUERIES is rejected with VLSG_ERR_CAPACITY.
 *   - The level sets must already be on the device (after vlsg_advect,
 *     vlsg_count_points, vlsg_download_levelset or vlsg_get_values), because
 *     moving them there allocates; otherwise VLSG_ERR_STATE.
 *   - The array is taken at set-up: the first time a context on a device
 *     moves its level sets there, the library looks up the array's device
 *     address with that device current (once per device).  Under lazy module
 *     loading (the CUDA default) that lookup is what places the array in
 *     device memory, so it happens while the set-up allocates anyway, not in
 *     a later no-allocation call.  Do that set-up before any stream capture
 *     on the device.
 *   - All calls share the array.  Calls that overlap on the GPU (contexts on
 *     the same device driven from several host threads at once) race on it.
 *     Each call writes every byte it reads, so nothing needs clearing between
 *     calls.
 * Same arguments, results and synchronisation as vlsg_get_values. */
#define VLSG_NOALLOC_MAX_QUERIES 65536
int vlsg_get_values_noalloc(vlsg_context *ctx, int32_t slot, int64_t n,
                            const int32_t *indices, double *values);

/* Comparison of two level sets held by contexts on the same device (they may
 * differ in precision), for the precision report of the FP32 path against
 * the FP64 path.  No counterpart in Advect itself; the volume and Chamfer
 * figures restate the rules of lsCompareVolume.hpp:272-287 (a cell is inside
 * when the average of its 8 corner values is <= 0; counted over the map box)
 * and lsCompareChamfer.hpp:148-242 (nodes on grid edges between defined
 * points of opposite sign, interpolated as lsToSurfaceMesh.hpp:339-361, here
 * without merging close nodes; mean / RMS / max nearest-node distances).
 * Distances are in grid units (multiply by gridDelta). */
typedef struct vlsg_compare_result {
  int64_t points_a, points_b;           /* defined points */
  int64_t common_points;                /* defined in both */
  int64_t defined_only_a, defined_only_b;
  int64_t active_a, active_b;           /* defined with |phi| <= 0.5 */
  int64_t active_only_a, active_only_b; /* active in one, not active in the other */
  double max_abs_diff, rms_abs_diff;    /* |phi_a - phi_b| on the common points */
  int64_t inside_cells_a, inside_cells_b;
  int64_t nodes_a, nodes_b;
  double chamfer_ab, chamfer_ba;        /* mean nearest-node distance a->b, b->a */
  double chamfer_mean, chamfer_rms, chamfer_max;
  int64_t chamfer_unresolved;           /* nodes with no node within 4 cells */
  int64_t diff_above[4];                /* common points with |phi_a - phi_b| above
                                           1e-6, 1e-5, 1e-4, 1e-3 (grid units) */
} vlsg_compare_result;
int vlsg_compare(vlsg_context *a, int32_t slot_a, vlsg_context *b, int32_t slot_b,
                 vlsg_compare_result *out);

/* setVelocityUpdateCallback (lsAdvect.hpp:966-969); NULL clears it. */
int vlsg_set_velocity_update_callback(vlsg_context *ctx, vlsg_update_cb cb, void *user);

/* Spatial sharding of one level-set domain over several contexts (one per
 * GPU), each holding a slab of the band plus ghost layers.  No counterpart in
 * Advect: the reference's only decomposition is its OpenMP segments, whose
 * per-thread time-step minima and alpha maxima it reduces in critical
 * sections (lsAdvect.hpp:595-606, :186-191); these two calls are that
 * reduction across contexts.
 *
 * vlsg_set_owned_region: only active points with index[axis] in [lo, hi)
 * contribute to the time step, the Lax-Friedrichs alphas and the point-update
 * count; the other (ghost) points are advanced all the same.  axis = -1 (the
 * default) owns everything; only axis 2 (the slowest index of the HRLE order)
 * is supported, and not with STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER.
 *
 * vlsg_set_reduction_callback: called from vlsg_advect with this context's
 * partial values before they are used -- the smallest per-point time step of
 * a rate pass (n = 1, op VLSG_REDUCE_MIN; DBL_MAX when it has none), the
 * alphas of the Lax-Friedrichs schemes (n = 3, VLSG_REDUCE_MAX) and the
 * "moved down" flag of a stage combination with lower layers (n = 1,
 * VLSG_REDUCE_MAX).  The callback replaces values[] by the reduction over all
 * shards (e.g. an all-reduce) and returns 0; every shard must call vlsg_advect
 * with the same parameters so that the calls line up.  NULL clears it. */
#define VLSG_REDUCE_MIN 0
#define VLSG_REDUCE_MAX 1
typedef int (*vlsg_reduce_cb)(void *user, double *values, int32_t n, int32_t op);
int vlsg_set_owned_region(vlsg_context *ctx, int32_t axis, int64_t lo, int64_t hi);
int vlsg_set_reduction_callback(vlsg_context *ctx, vlsg_reduce_cb cb, void *user);

/* PrepareStencilLocalLaxFriedrichs (lsStencilLocalLaxFriedrichsScalar.hpp:
 * 423-477) on the context's level sets: is_depo[i] tells whether level set i
 * is deposited on (n entries, missing ones false); the top level set becomes
 * the layer wrapping STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER advects. */
int vlsg_prepare_stencil_llf(vlsg_context *ctx, const int32_t *is_depo, int32_t n);
/* FinalizeStencilLocalLaxFriedrichs (:480-492): restores the usual wrapping
 * (top = inverted top united with the level set below; needs two). */
int vlsg_finalize_stencil_llf(vlsg_context *ctx);

/* Advect::prepareLS (lsAdvect.hpp:972-1015): Expand the top level set to the
 * width the spatial scheme reads (vlsg_spatial_scheme); VLSG_ERR_ARGUMENT for
 * an unknown scheme ("Advect: Discretization scheme not found."). */
int vlsg_prepare_ls(vlsg_context *ctx, int32_t spatial_scheme);

/* Velocity plugin: either a device functor or a host callback. */
int vlsg_set_velocity_functor(vlsg_context *ctx, const vlsg_velocity_desc *v);
int vlsg_set_velocity_callback(vlsg_context *ctx, vlsg_velocity_cb cb,
                               void *user);
/* With a host velocity callback: the dissipation alphas of
 * LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER (NULL clears it). */
int vlsg_set_dissipation_alpha_callback(vlsg_context *ctx, vlsg_alpha_cb cb,
                                        void *user);

/* Advect::apply(), lsAdvect.hpp:1017-1043. */
int vlsg_advect(vlsg_context *ctx, const vlsg_advect_params *params,
                vlsg_advect_result *result);

/* Batching form: advance n independent contexts (each with its own grid,
 * level sets and velocity functor) with the same parameters.  A pool of
 * `threads` host threads (0: min(n, 32)) drives them, each context on its own
 * CUDA stream, so the kernels of many small domains run side by side on the
 * GPU.  results[i] receives context i's getters; the return value is the
 * first failing context's status (its message in vlsg_last_error(ctxs[i])).
 * Results are bit-identical to calling vlsg_advect on each context in turn.
 * No counterpart in Advect (one Advect per domain); it replaces the loop a
 * caller would write over many Advect objects. */
int vlsg_advect_batch(vlsg_context **ctxs, int32_t n, const vlsg_advect_params *params,
                      vlsg_advect_result *results, int32_t threads);

/* Batching form, in one context: many independent domains (each with its own
 * grid, one level set and a velocity functor) share one brick pool, and every
 * band pass, rate pass and value update of a time step is ONE kernel launch
 * over the bricks of all domains.  Each domain keeps its own gridDelta,
 * velocity and time step; the time steps are reduced per domain on the
 * device, so a step needs no host synchronisation until its end.  No
 * counterpart in Advect: it replaces a loop over many Advect objects
 * (examples/SquareEtch/SquareEtch.cpp:189-229 advances one domain per
 * Advect), with results bit-identical to advancing each domain by itself
 * (vlsg_advect on one context per domain).
 * Limits: every domain periodic in x and y with extents that are multiples
 * of 8 points and infinite in z; one level set per domain; one time step per
 * vlsg_batch_advect (advection_time 0); device velocity functors; not with
 * global LAX_FRIEDRICHS, STENCIL_LOCAL_LAX_FRIEDRICHS, voids, point data or
 * FP32 compensation (VLSG_ERR_ARGUMENT); a domain whose first stage gets no
 * positive time step (no active point, zero velocity) ends the step with
 * VLSG_ERR_DEVICE_CHECK.  vlsg_set_grid returns the context to one domain. */
typedef struct vlsg_batch_domain {
  const int64_t *grid_min, *grid_max; /* index bounds, 3 each (vlsg_set_grid) */
  const int32_t *boundary;            /* 3: PERIODIC, PERIODIC, INFINITE */
  double grid_delta;
  int64_t n_points;                   /* as vlsg_upload_levelset */
  const int32_t *indices;
  const double *values;
  int64_t n_runs;
  const int32_t *run_start;
  const int8_t *run_sign;
  int32_t width;
  const vlsg_velocity_desc *velocity;
} vlsg_batch_domain;
int vlsg_batch_set_domains(vlsg_context *ctx, int32_t n, const vlsg_batch_domain *domains);
/* One time step of every domain; results[d] receives domain d's getters. */
int vlsg_batch_advect(vlsg_context *ctx, const vlsg_advect_params *params,
                      vlsg_advect_result *results);
/* Domain d's defined points in HRLE order, in its own indices. */
int vlsg_batch_count_points(vlsg_context *ctx, int32_t domain, int64_t *n_points);
int vlsg_batch_download(vlsg_context *ctx, int32_t domain, int64_t capacity,
                        int32_t *indices, double *values, int32_t *width);
/* Domain d's undefined runs, in the layout and with the capacity protocol
 * of vlsg_download_runs (built on the host from point queries). */
int vlsg_batch_download_runs(vlsg_context *ctx, int32_t domain, int64_t capacity,
                             int32_t *run_start, int8_t *run_sign, int64_t *n_runs);
/* vlsg_get_values for domain d (its indices, mapped through its periodic
 * boundaries). */
int vlsg_batch_get_values(vlsg_context *ctx, int32_t domain, int64_t n,
                          const int32_t *indices, double *values);

/* Timing of the last vlsg_advect: per kernel family, device milliseconds and
 * algorithmic bytes, as measured with CUDA events on the context stream
 * (filled only when profiling is switched on with vlsg_set_profiling). */
typedef struct vlsg_kernel_stat {
  char name[32];
  uint64_t launches;
  double device_ms;
  double algorithmic_bytes;
} vlsg_kernel_stat;
int vlsg_set_profiling(vlsg_context *ctx, int32_t on);
int vlsg_get_kernel_stats(vlsg_context *ctx, int32_t capacity,
                          vlsg_kernel_stat *out, int32_t *count);

#ifdef __cplusplus
}
#endif
#endif /* VLSG_H */
