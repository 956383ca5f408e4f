/* inductioneq.h -- C ABI of the B200 (sm_100a) InductionEq time-stepping library.
 *
 * Drop-in boundary for the reference's MatCL-driven OpenCL kernels
 * (IANW-Projects/InductionEq v1.1.1).  The reference host (MATLAB) compiles a list of
 * source files with a "-DKEY=VAL" settings string and then runs lists of named kernels
 * that all receive the same argument vector:
 *     cl_run_kernel(device, kernel_path_list, settings)            -- compile
 *     t = cl_run_kernel(device, names, g_range, l_range, args..., 0) -- run
 * (matlab/+induction_eq/compute_numerical_solution.m:23,179-181; the MatCL mex itself is
 * not part of the reference).  This header replaces that pair:
 *     ieq_create(settings, kernel_path_list)   <- cl_run_kernel(dev, paths, settings)
 *     ieq_run_kernels(names, g_range, args)    <- cl_run_kernel(dev, names, g, l, args..., 0)
 * plus one typed entry point per reference kernel (inductioneq_kernels.h) and the fused,
 * graph-captured paths that the B200 build adds (time stepping, CG cleaning, norms).
 *
 * Conventions
 *   - Plain pointers and sizes only.  Field arguments are DEVICE pointers in the
 *     reference layout: a vector field is REAL4 AoS (x,y,z,w; w = 0) of num_nodes_pad
 *     entries, a scalar field num_nodes_pad REALs, `time` two REALs
 *     (time[0] = start of the step, time[1] = stage time).  Node index
 *     idx = ix + NX*(iy + NY*iz) (include/utils.h:66-68).
 *   - REAL is double unless the settings say -DREAL=float.
 *   - Every function returns ieq_status; ieq_last_error() describes the last failure.
 *   - One CUDA stream per context; calls on one context are not thread safe, separate
 *     contexts are independent.  Work is asynchronous on that stream unless stated.
 */
#ifndef INDUCTIONEQ_H
#define INDUCTIONEQ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ieq_status {
  IEQ_OK = 0,
  IEQ_ERR_SETTINGS = 1,       /* unknown/contradictory -D settings or kernel path list   */
  IEQ_ERR_SHAPE = 2,          /* grid too small for the operator, bad g_range           */
  IEQ_ERR_CUDA = 3,           /* a CUDA runtime call failed                              */
  IEQ_ERR_NAN = 4,            /* a non-finite value was detected in a result             */
  IEQ_ERR_NOT_CONVERGED = 5,  /* CG stopped at max_iterations above the threshold        */
  IEQ_ERR_TIMEOUT = 6,        /* a bounded device wait gave up                           */
  IEQ_ERR_UNKNOWN_KERNEL = 7, /* a kernel name the reference does not define             */
  IEQ_ERR_ARG = 8             /* null/misaligned pointer, wrong argument count           */
} ieq_status;

typedef struct ieq_ctx ieq_ctx;

/* Create a context from the reference's settings string and kernel path list.
 * settings: the concatenation generate_settings.m produces (" -DNODES_X=40 -DDX=5.1e-02
 *   -DUSE_UIBJ_PRODUCT=1 ... -cl-mad-enable"); OpenCL compiler options are accepted and
 *   ignored.  Keys this library adds (all optional): -DIEQ_INTEGRATOR=<name of one of the
 *   six integrators> (host-side I_TI('time_integrator')), -DIEQ_VARIABLE_U=1
 *   (I_RunOps('variable_u')), -DTC_OMEGA=<rotation rate of the rotation_gaussian case>;
 *   and, choosing kernels of the fused time stepping without changing its results beyond
 *   the compiler's FMA contraction: -DIEQ_STAGE_KERNEL=AUTO|COLUMN|NODE|BRICK|LIST|ZMARCH
 *   (ZMARCH: the one-pass Hall stage that marches through z -- curl, E = J x B, dissipation
 *   and update in one kernel -- wherever it can run; AUTO does not take it: it measured
 *   slower than the curl + stage kernel pair), -DIEQ_ZMARCH_TZ=<z planes per CTA of that
 *   kernel; 0 chosen per grid>,
 *   -DIEQ_COL_BLOCK=XxYxZ / -DIEQ_CURL_BLOCK=XxYxZ (128-thread block shapes of the column
 *   stage and curl kernels), -DIEQ_COL_PAIRS=0|1|4 (nodes per thread: one; the measured
 *   default; FP32 quads on every grid), -DIEQ_XBAND=0|1|2 (a box's x boundary columns in a
 *   launch of their own: never, where measured faster, wherever possible), -DIEQ_PDL=0|1
 *   (programmatic dependent launch of the column kernels).
 * kernel_paths: the kernel_path_list (compute_numerical_solution_setup.m:57-122).  Only
 *   the base names matter: the operator header ({2,4,6}thOrder[Extended].h) selects the SBP
 *   operator, "<testcase>.h" the testcase, artificial_dissipation.cl enables dissipation.
 * device: CUDA device ordinal. */
ieq_status ieq_create(ieq_ctx **ctx, const char *settings, const char *const *kernel_paths,
                      int n_paths, int device);
void ieq_destroy(ieq_ctx *ctx);
const char *ieq_last_error(const ieq_ctx *ctx);
const char *ieq_status_string(ieq_status s);

/* Sizes the reference host derives in initialize.m:31-48. */
size_t ieq_num_nodes(const ieq_ctx *ctx);
size_t ieq_num_nodes_pad(const ieq_ctx *ctx);
size_t ieq_num_groups(const ieq_ctx *ctx);
int ieq_real_size(const ieq_ctx *ctx); /* 8 (double) or 4 (float) */

/* Device memory owned by the context (freed by ieq_free or ieq_destroy).  Memory
 * allocated elsewhere (e.g. by PyTorch) may be passed to every call as well. */
ieq_status ieq_alloc(ieq_ctx *ctx, size_t bytes, void **dptr);
ieq_status ieq_free(ieq_ctx *ctx, void *dptr);
ieq_status ieq_upload(ieq_ctx *ctx, void *dst, const void *host_src, size_t bytes);
ieq_status ieq_download(ieq_ctx *ctx, void *host_dst, const void *src, size_t bytes);
ieq_status ieq_memset(ieq_ctx *ctx, void *dst, int value, size_t bytes);
ieq_status ieq_synchronize(ieq_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their own work. */
void *ieq_stream(ieq_ctx *ctx);

/* MatCL-form list call: enqueue every kernel of `names` in order, each with the same
 * argument vector `args` (device pointers, n_args of them).  g_range as in the reference
 * host (3D node range, or {num_nodes_pad,1,1} for the reductions, or the CG interior
 * range NODES-2*BNODES).  If elapsed_seconds is not NULL the call synchronises and
 * returns the device time of the list (cudaEvent), like MatCL's return value. */
ieq_status ieq_run_kernels(ieq_ctx *ctx, const char *const *names, int n_names,
                           const uint32_t g_range[3], void *const *args, int n_args,
                           double *elapsed_seconds);

/* The same with HOST arrays, copied in before and back after the list, in place, as the
 * MatCL mex does with MATLAB arrays.  arg_bytes[i] is the size of host array i. */
ieq_status ieq_run_kernels_host(ieq_ctx *ctx, const char *const *names, int n_names,
                                const uint32_t g_range[3], void *const *host_args,
                                const size_t *arg_bytes, int n_args, double *elapsed_seconds);

/* ---------------------------------------------------------------- fused B200 paths */

/* num_steps time steps of the configured integrator (-DIEQ_INTEGRATOR), the loop of
 * compute_numerical_solution.m:174-192, with the stage kernels fused as far as the data
 * flow allows and the step captured in a CUDA graph.  Field arguments as for the
 * reference kernels of that integrator (b3 is ignored by the 2N schemes and may be NULL).
 * Results equal running rk_step() kernel lists through ieq_run_kernels. */
ieq_status ieq_time_steps(ieq_ctx *ctx, void *b, void *b2, void *b3, void *curlB_rho, void *u,
                          void *rho, void *time, int num_steps);

/* ieq_time_steps with the per-step diagnostics of the reference's save_integrals_over_time
 * loop (compute_numerical_solution.m:153-193): before every step the mass-weighted energy
 * norm2(b), the divergence norm sqrt(norm2_S(calc_div(b))) and the L2 error
 * sqrt(norm2_diff(b, analytical_b(time[0]))) are evaluated on the device in one pass and
 * collected into a device series (inside the step graph when there is no cleaning).  With
 * clean_max_iterations > 0, B is cleaned after every step (ieq_clean_div with that cap and
 * clean_threshold), as the reference does when divergence cleaning is on.  energy,
 * divergence_norm, l2_error: host arrays of num_steps entries, or NULL.  Synchronises. */
ieq_status ieq_time_steps_integrals(ieq_ctx *ctx, void *b, void *b2, void *b3, void *curlB_rho, void *u,
                                    void *rho, void *time, int num_steps, int clean_max_iterations,
                                    double clean_threshold, double *energy, double *divergence_norm,
                                    double *l2_error);

/* Divergence cleaning, matlab/+induction_eq/clean_div.m:36-79, device resident: CG on
 * (-Laplace) phi = div B over the interior, stopping when the unweighted squared
 * residual <= absolute_error_threshold^2 or after max_iterations, then B is projected.
 * The CG vectors (phi, r, u, Laplacian), the dot products, alpha/beta and the divergence and
 * projection arithmetic are FP64 whatever REAL is (with REAL=float this is the precision
 * form: FP32 state, FP64 solve).  Returns IEQ_ERR_NOT_CONVERGED (with B still projected)
 * if the cap was hit. */
ieq_status ieq_clean_div(ieq_ctx *ctx, void *b, int max_iterations,
                         double absolute_error_threshold, int *iterations,
                         double *residual_norm2, double *initial_divergence_norm);

/* Mass-weighted squared norms (kernel_operator.cl:11-137), reduced on the device in a
 * fixed order (bitwise reproducible) and returned to the host in FP64. */
ieq_status ieq_norm2_value(ieq_ctx *ctx, const void *vec_field, double *result);
ieq_status ieq_norm2_diff_value(ieq_ctx *ctx, const void *vec_a, const void *vec_b,
                                double *result);
ieq_status ieq_norm2_S_value(ieq_ctx *ctx, const void *scalar_field, double *result);
ieq_status ieq_dot_value(ieq_ctx *ctx, const void *a, const void *b, double *result);
/* The same unweighted dot product (kernel_dot_product.cl:47-74 summed like the host of
 * clean_div.m:47-79) over the elements [first, first + count) of two scalar fields of the
 * context's grid only: one rank's owned planes in a z-slab decomposition, whose per-rank
 * sums are then added across the ranks.  IEQ_ERR_SHAPE if the range leaves the grid's nodes. */
ieq_status ieq_dot_range(ieq_ctx *ctx, const void *a, const void *b, uint64_t first, uint64_t count,
                         double *result);

/* Result metrics of compute_numerical_solution.m:198-250 at time t: abs/rel L2 error
 * against b_analytical(t), ||div B|| and the energy.  work_vec/work_scalar are scratch
 * fields of the context's layout. */
typedef struct ieq_results {
  double abs_err, rel_err, divergence_norm, energy;
} ieq_results;
ieq_status ieq_compute_results(ieq_ctx *ctx, const void *b, double t, void *work_vec,
                               void *work_scalar, ieq_results *out);

/* IEQ_ERR_NAN if any x/y/z component of the vector field is not finite, else IEQ_OK. */
ieq_status ieq_check_finite(ieq_ctx *ctx, const void *vec_field);

/* Test hook of the TMA brick kernels' bounded mbarrier waits (failure-path tests): with
 * first_wait_gives_up = 1 every brick's first wait for its halo copies gives up at once, so
 * the brick records a time-out, waits for its copies with the production limit before it
 * leaves (no copy is left writing into shared memory) and the next ieq_time_steps returns
 * IEQ_ERR_TIMEOUT; 0 restores the production waits.  A brick that leaves with copies still
 * outstanding after that second wait is reported as a different IEQ_ERR_TIMEOUT message:
 * the context's results are then undefined and it should be destroyed. */
ieq_status ieq_test_brick_wait(ieq_ctx *ctx, int first_wait_gives_up);

/* The reference kernel list of one time step of the configured integrator, as the MATLAB
 * host builds it (compute_numerical_solution_setup.m:140-371): names separated by '\n'
 * written to `names` (NUL-terminated; `capacity` bytes) and their number to *count.  With
 * names == NULL only the count is returned.  Hosts that interleave their own work between
 * the kernels of a step (the z-slab decomposition's ghost exchanges) run the list through
 * ieq_run_kernels one name at a time. */
ieq_status ieq_step_kernels(ieq_ctx *ctx, char *names, size_t capacity, int *count);

/* Profiling (the per-kernel counterpart of the kernel time MatCL returns): every launch of
 * one ieq_time_steps step is captured alone, `repeats` times back to back, into a CUDA graph
 * and timed with events around the graph; records[k] gets the label and average device
 * time (ms) of launch k, in launch order.  The fields are advanced by the repeated
 * launches and hold no solution afterwards.  Synchronises. */
typedef struct ieq_kernel_record {
  char name[40];
  double ms;
} ieq_kernel_record;
ieq_status ieq_profile_step(ieq_ctx *ctx, void *b, void *b2, void *b3, void *curlB_rho, void *u,
                            void *rho, void *time, int repeats, int max_records,
                            ieq_kernel_record *records, int *n_records);

/* ---------------------------------------------------------------- batched form */

/* Many independent solves of uneven grid sizes and SBP orders advanced together: every
 * SSPRK33 stage of every solve is processed by one persistent kernel over a queue of tiles,
 * the whole run captured in a CUDA graph.  No counterpart in the reference (which runs one
 * grid per process); each solve is a context made by ieq_create, and the result of every
 * solve equals ieq_time_steps on its own context.  Restrictions: REAL=double, SSPRK33,
 * classical operators, no Hall term, no dissipation, constant velocity. */
typedef struct ieq_batch ieq_batch;
ieq_status ieq_batch_create(ieq_batch **batch, ieq_ctx *const *solves, int n_solves);
void ieq_batch_destroy(ieq_batch *batch);
const char *ieq_batch_last_error(const ieq_batch *batch);
void *ieq_batch_stream(ieq_batch *batch);
/* tile (brick) shape of one solve's tiles, tx*ty*tz = 256 nodes (chosen by the autotuner) */
ieq_status ieq_batch_set_tile(ieq_batch *batch, int solve, int tx, int ty, int tz);
/* fields[5*i + 0..4] = solve i's b, b2, b3, u, time (device pointers, reference layout) */
ieq_status ieq_batch_bind(ieq_batch *batch, void *const *fields);
/* num_steps steps of all bound solves, captured in one CUDA graph, by
 *   mode IEQ_BATCH_PERSISTENT (1): one persistent kernel over the tile queue, stages
 *     separated by a bounded software grid barrier;
 *   mode IEQ_BATCH_STAGES (0): one kernel over the tile queue per stage;
 *   mode IEQ_BATCH_BRANCHES (2): one graph branch per solve (its fused column kernels on its
 *     own stream), the branches running concurrently.
 * IEQ_ERR_TIMEOUT if a bounded grid barrier gave up.  Syncs. */
#define IEQ_BATCH_STAGES 0
#define IEQ_BATCH_PERSISTENT 1
#define IEQ_BATCH_BRANCHES 2
ieq_status ieq_batch_run(ieq_batch *batch, int num_steps, int mode);
/* copy the solves' b, b2, b3 back into the bound fields */
ieq_status ieq_batch_unbind(ieq_batch *batch);
long long ieq_batch_total_tiles(const ieq_batch *batch);
int ieq_batch_grid(const ieq_batch *batch);
/* Test hook of the persistent mode's bounded grid barrier (failure-path tests): every later
 * ieq_batch_run waits for `extra_arrivals` (0 or 1) blocks beyond the grid -- 1 is a block
 * that never arrives, so each wait runs out after `spin_limit` 64-ns sleeps (<= 0: the
 * production limit, about 1.3 s) and the run returns IEQ_ERR_TIMEOUT.  (0, 0) restores the
 * production barrier; every run starts from a reset barrier state. */
ieq_status ieq_batch_test_barrier(ieq_batch *batch, int extra_arrivals, long long spin_limit);

/* ---------------------------------------------------------------- stage-by-stage stepping */

/* The fused time step of ieq_time_steps enqueued one RK stage at a time, for a caller that
 * acts between stages -- the z-slab decomposition of one solve over several GPUs refreshes
 * the ghost planes of the state fields after every stage.  No counterpart in the reference
 * (its host runs whole kernel lists).
 *   ieq_stages_begin copies the fields (reference layout) into the context's fused state and
 *     returns the stages of one step of the configured integrator;
 *   ieq_stages_run enqueues stage `stage` (0 .. stages_per_step - 1, in order; after the last
 *     stage the next stage 0 starts a new step) on the context's stream;
 *   ieq_stages_field gives the state field `field` (0: b1, 1: b2, 2: b3 or db of the
 *     three-field schemes) as it stands after the last stage run: the device address of its x
 *     plane, the y and z planes following at component_stride elements (REAL); the fused path
 *     alternates some fields between two buffers, so ask after every stage;
 *   ieq_stages_end copies the state back into the fields.
 * The fields may not be used by other calls on the context between begin and end. */
ieq_status ieq_stages_begin(ieq_ctx *ctx, void *b, void *b2, void *b3, void *curlB_rho, void *u,
                            int *stages_per_step);
ieq_status ieq_stages_run(ieq_ctx *ctx, void *rho, void *time, int stage);
ieq_status ieq_stages_field(ieq_ctx *ctx, int field, void **base, long long *component_stride);
ieq_status ieq_stages_end(ieq_ctx *ctx, void *b, void *b2, void *b3, void *curlB_rho, void *u, const void *rho);

/* ---------------------------------------------------------------- discrete adjoint */

/* Hand-written discrete adjoint of the spatial operator F(b) = DB (volume terms, Hall term
 * with J = curl(b)/rho, high-order and first-order dissipation, inflow SAT, Hall outflow SAT)
 * at fixed u and rho, and of the SSPRK33 and 2N steps.  No counterpart in the reference.
 * FP64 only.  The Hall outflow SAT switches on the sign of 0.5u - J: it is differentiated with
 * the switch held (its derivative away from tv = 0).  Adaptive dissipation is linearised at b
 * (kappa's derivative inside its thresholds; none exists at them).  Vector fields in the
 * reference layout. */
/* out = F'(b) v (tangent linear) */
ieq_status ieq_operator_jvp(ieq_ctx *ctx, const void *b, const void *v, const void *u, const void *rho,
                            void *out);
/* out = F'(b)^T w */
ieq_status ieq_operator_vjp(ieq_ctx *ctx, const void *b, const void *w, const void *u, const void *rho,
                            void *out);
/* lambda <- (d b_{n+1} / d b_n)^T lambda for one SSPRK33 step with stage states s1 = b_n,
 * s2 = b^(2), s3 = b^(3) starting at time t0 (u from u_analytical at the stage times when
 * -DIEQ_VARIABLE_U=1, else the given u) */
ieq_status ieq_ssprk33_step_vjp(ieq_ctx *ctx, const void *s1, const void *s2, const void *s3, double t0,
                                void *lambda, const void *u, const void *rho);
/* Gradient through num_steps steps of the configured integrator (any of the six) from b0 at
 * t = 0: lambda holds dL/db(T) on entry and dL/db0 on return.  The forward run is checkpointed
 * every checkpoint_every steps and each segment recomputed (the input of every stage kept)
 * during the reverse sweep.  SSPRK33 and the 2N schemes have step adjoints of their own (a 2N
 * step reversed stage by stage: mu2 += B_s mu1, mu1 += h F'^T mu2, mu2 = A_s mu2); the 2R
 * schemes and SSPRK104 -- and every integrator with -DIEQ_ADJOINT_PROGRAM=1 -- reverse the
 * step's register program (each stage K = h F(R_src) and its register updates, transposed in
 * reverse order); that form needs the fused kernels (not -DIEQ_STAGE_KERNEL=LIST). */
ieq_status ieq_adjoint_steps(ieq_ctx *ctx, const void *b0, void *lambda, const void *u, const void *rho,
                             int num_steps, int checkpoint_every);

/* ---------------------------------------------------------------- allocation-free dot */

/* FP64 dot product sum_i a[i]*b[i] of two device arrays of n doubles, written to the device
 * scalar result[0] on `stream` (a cudaStream_t; NULL = the default stream).  No counterpart
 * in the reference: it exists for callers that cannot let a library allocate device memory --
 * hosts whose device memory belongs to their own pool (a framework's caching allocator, a
 * MATLAB mex working within a fixed budget) and time loops that must not allocate once they
 * run.  It needs no context and calls no cudaMalloc, cudaFree or allocating library routine:
 * its scratch (one FP64 partial per 2048 elements) is a fixed 32 KiB array in the library's
 * device image, which every GPU that loads the library holds until the process exits.
 *   - n may be at most IEQ_NOALLOC_DOT_MAX_ELEMENTS; larger n returns IEQ_ERR_SHAPE and
 *     launches nothing.  NULL pointers return IEQ_ERR_ARG.
 *   - Every call looks up the scratch array's device address for the calling thread's
 *     current device (cudaGetSymbolAddress, which allocates nothing); the first call on a
 *     device also loads the library's device image there, so make it before any stream
 *     capture.
 *   - All calls share the one scratch array, which keeps the last call's partials.  Every
 *     partial a call reads was written earlier in that call, so nothing needs clearing, but
 *     calls that overlap on the GPU (other streams, other threads) race: order them.
 *   - The sum is taken in a fixed order: repeated calls give bitwise identical results. */
#define IEQ_NOALLOC_DOT_MAX_ELEMENTS 8388608
ieq_status ieq_dot_product_noalloc(const double *a, const double *b, uint64_t n, double *result,
                                   void *stream);

/* The FP64 arithmetic rate of `device` in GFLOP/s (2 per fused multiply-add), measured with
 * an FMA loop of `iterations` steps per chain (8 independent chains per thread, 8 blocks of
 * 256 threads per SM) timed with CUDA events: the FP64 roof the stencil kernels are graded
 * against beside the HBM bandwidth.  No counterpart in the reference (a measurement aid). */
ieq_status ieq_fp64_fma_rate(int device, int iterations, double *gflops);

#ifdef __cplusplus
}
#endif

#include "inductioneq_kernels.h"

#endif /* INDUCTIONEQ_H */
