/* baemm.h -- C ABI of libbaemm_cuda.so, the B200 (sm_100a) implementation of
 * BAEMM's boundary-element Helmholtz operator path.
 *
 * Every entry point replaces one public member of the reference class
 * BAEMM::Helmholtz_OpenCL (HenrikSchumacher/BAEMM); the reference interface is
 * cited beside each declaration (path:line within that project).  The C++
 * drop-in class in Helmholtz_CUDA.hpp wraps these calls with the reference's
 * templated signatures.
 *
 * Conventions
 *   - Plain pointers and sizes only.  Complex arrays are interleaved (re, im)
 *     pairs, row-major "rows x ld" exactly as the reference lays them out.
 *     `_z` = complex<double> external data, `_c` = complex<float>, `_d` = double.
 *   - Host-pointer entry points copy inputs to the device and results back
 *     (the reference's semantics).  `_dev_` entry points take device pointers
 *     and run on the context's stream without host synchronisation.
 *   - Every call returns a baemm_status; 0 is success.  The text of the last
 *     error of a context is available from baemm_last_error().
 *   - A context is externally synchronised: one thread at a time (the
 *     reference class is not thread-safe either).
 *   - There is no CPU fallback: without a usable CUDA device baemm_create
 *     fails with BAEMM_ERR_CUDA.
 */
#ifndef BAEMM_H
#define BAEMM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct baemm_ctx baemm_ctx;

typedef enum baemm_status
{
    BAEMM_OK                = 0,
    BAEMM_ERR_ARG           = 1,  /* invalid argument (null pointer, bad size, ld < wave_count, ...) */
    BAEMM_ERR_CUDA          = 2,  /* a CUDA call failed; see baemm_last_error */
    BAEMM_ERR_ALLOC         = 3,  /* device or host allocation failed */
    BAEMM_ERR_NOT_LOADED    = 4,  /* operator applied before baemm_load_boundary_operators */
    BAEMM_ERR_NOT_CONVERGED = 5,  /* a solver stopped at its iteration limit */
    BAEMM_ERR_SIZE          = 6,  /* size outside the supported range */
    BAEMM_ERR_TIMEOUT       = 7   /* a bounded device-side wait gave up */
} baemm_status;

/* Wave types (BAEMM_Common.hpp:7-11). */
#define BAEMM_WAVE_PLANE  201
#define BAEMM_WAVE_RADIAL 202

/* Arithmetic of the dense boundary-operator apply (no reference counterpart;
 * the reference has FP32 only, Definitions.hpp:3-6). */
#define BAEMM_APPLY_FP32 0   /* plain: FP32 generation and FP32 SIMT contraction */
#define BAEMM_APPLY_TC   1   /* compensated: split hi+lo operands on the tensor cores, FP32 accumulate;
                              * needs wave_chunk_size a multiple of 16 and wave_count <= 512, other
                              * shapes run the plain FP32 kernel; FP32 values below 1.2e-38 are
                              * flushed to zero in this form */
#define BAEMM_APPLY_FP64 2   /* FP64 generation and contraction */

/* Solver statistics of the last GMRES / CG run (the reference discards them,
 * FarField.hpp:764, 870). */
typedef struct baemm_solve_stats
{
    int32_t gmres_iterations;
    int32_t gmres_converged;
    double  gmres_relative_residual;
    int32_t cg_iterations;         /* max over the mass-inverse calls of that solve */
    int32_t cg_converged;
    int32_t refinement_steps;      /* FP64 iterative-refinement steps (0 = none) */
    double  seconds;
} baemm_solve_stats;

/* User operator on n x 3 real host arrays (the M and P callables of
 * GaussNewtonSolve, FarField.hpp:457-479). */
typedef void (*baemm_real_op)(const double *x, double *y, void *user);

/* ---- lifecycle ---------------------------------------------------------- */

/* Helmholtz_OpenCL(coords, nv, tris, nt, meas, nm, device_num, threads)
 * (Helmholtz_OpenCL.hpp:175-249) and the variant without device_num
 * (Helmholtz_OpenCL.hpp:109-159; pass device = 0).  coords: nv x 3,
 * triangles: nt x 3 (0-based), meas_directions: nm x 3.  cpu_threads is
 * accepted for signature parity and bounds the host threads of set-up.
 * At most 2^28 triangles, vertices and measurement directions each
 * (BAEMM_ERR_SIZE beyond: the sparse operators and kernels index with int32). */
int baemm_create(const double *coords, int64_t vertex_count,
                 const int64_t *triangles, int64_t simplex_count,
                 const double *meas_directions, int64_t meas_count,
                 int device, int cpu_threads, baemm_ctx **out);
int baemm_create_i32(const double *coords, int64_t vertex_count,
                     const int32_t *triangles, int64_t simplex_count,
                     const double *meas_directions, int64_t meas_count,
                     int device, int cpu_threads, baemm_ctx **out);
/* Replace the mesh of a context, keeping its device, stream, measurement
 * directions and settings (no reference counterpart: the reference constructs
 * a new Helmholtz_OpenCL per mesh).  Device buffers only grow, so a mesh no
 * larger than one the context held before allocates nothing; a serving loop
 * re-meshes pooled contexts instead of creating and destroying them (a
 * cudaFree synchronises the whole device).  Unloads the boundary operators;
 * synchronises the context's stream. */
int baemm_set_mesh(baemm_ctx *ctx, const double *coords, int64_t vertex_count,
                   const int64_t *triangles, int64_t simplex_count);
/* ~Helmholtz_OpenCL (Helmholtz_OpenCL.hpp:251-282). */
void baemm_destroy(baemm_ctx *ctx);
const char *baemm_last_error(const baemm_ctx *ctx);
/* DeviceInfo (Helmholtz_OpenCL.hpp:343-391); writes a NUL-terminated text. */
int baemm_device_info(baemm_ctx *ctx, char *buf, size_t len);
/* ClassName (Helmholtz_OpenCL.hpp:395-398): "Helmholtz_CUDA". */
const char *baemm_class_name(void);
/* The CUDA stream the context runs on (cudaStream_t). */
void *baemm_stream(baemm_ctx *ctx);
/* Use an external stream (e.g. a framework's current stream); NULL = own
 * (non-blocking) stream; cudaStreamLegacy ((void *)0x1) = the legacy default
 * stream.  Work enqueued afterwards is ordered after the work already queued
 * on the previous stream (an event, no host synchronisation).  The stream must
 * outlive its use by the context.  No reference counterpart (the reference
 * owns its OpenCL queue). */
int baemm_set_stream(baemm_ctx *ctx, void *stream);
int baemm_synchronize(baemm_ctx *ctx);

/* ---- getters / setters (GetSetters.hpp, MemberVariables.hpp:93-98) ------- */
int64_t baemm_vertex_count(const baemm_ctx *ctx);          /* GetSetters.hpp:103-106 */
int64_t baemm_simplex_count(const baemm_ctx *ctx);         /* GetSetters.hpp:108-111 */
int64_t baemm_meas_count(const baemm_ctx *ctx);            /* GetSetters.hpp:164-167 */
int baemm_get_wave_count(const baemm_ctx *ctx);            /* GetSetters.hpp:130-133 */
int baemm_get_wave_chunk_size(const baemm_ctx *ctx);       /* GetSetters.hpp:142-145 */
int baemm_set_wave_chunk_size(baemm_ctx *ctx, int wcs);    /* GetSetters.hpp:147-152 */
int baemm_get_block_size(const baemm_ctx *ctx);            /* GetSetters.hpp:159-162 */
int baemm_set_block_size(baemm_ctx *ctx, int block_size);  /* GetSetters.hpp:180-188 (recorded; tiles are chosen by the library) */
int baemm_use_diagonal(baemm_ctx *ctx, int use_it);        /* GetSetters.hpp:210-213 */
int baemm_set_gmres_params(baemm_ctx *ctx, int max_iter, int max_restarts); /* MemberVariables.hpp:97-98 */
int baemm_get_gmres_params(const baemm_ctx *ctx, int *max_iter, int *max_restarts);
int baemm_set_apply_mode(baemm_ctx *ctx, int mode);        /* BAEMM_APPLY_*; no reference counterpart */
int baemm_get_apply_mode(const baemm_ctx *ctx);
/* Kernel tuning knobs (no reference counterpart; results are the same sums):
 *   BAEMM_TUNE_DENSE_VARIANT  plain FP32 dense kernel: 0 scalar FMA (default),
 *                             1 / 2 packed FP32x2 with 1 / 2 targets per thread
 *   BAEMM_TUNE_TC_SEGMENT     tensor-core form: 16-source tiles accumulated in
 *                             TMEM before each partial sum is added to the FP32
 *                             sums in shared memory (default 16; bounds the
 *                             tensor-core accumulation chain)
 *   BAEMM_TUNE_TC_CTAS        tensor-core form: persistent grid size (default 0 =
 *                             one CTA per SM)
 *   BAEMM_TUNE_TC_STAGGER     tensor-core form: CTA k starts its sweep of the
 *                             source tiles at tile (k % 8) * value (default 0:
 *                             all in step); -1 spreads the starts over all tiles
 *   BAEMM_TUNE_TC_GEN_WARPS   tensor-core form: warps evaluating the kernel
 *                             entries, 8 or 16 (default 16)
 *   BAEMM_TUNE_TC_CHUNKS      tensor-core form: 16-column groups per work unit,
 *                             1, 2 or 4 (default 0: the most the wave shape
 *                             allows; fewer give small meshes more work units)
 *   BAEMM_TUNE_TC_SHARE       tensor-core form: most 16-column groups with one
 *                             wavenumber that share one evaluation of the
 *                             kernel entries, 1, 2 or 4 (default 4; used by the
 *                             mixed BIE and DtN coefficient forms) */
#define BAEMM_TUNE_DENSE_VARIANT 1
#define BAEMM_TUNE_TC_SEGMENT    2
#define BAEMM_TUNE_TC_CTAS       3
#define BAEMM_TUNE_TC_STAGGER    4
#define BAEMM_TUNE_TC_GEN_WARPS  5
#define BAEMM_TUNE_TC_CHUNKS     6
#define BAEMM_TUNE_TC_SHARE      7
int baemm_set_tuning(baemm_ctx *ctx, int key, int value);
int baemm_get_tuning(const baemm_ctx *ctx, int key);
/* Groups of 16 columns per shared entry evaluation that the tensor-core apply
 * of the loaded operators uses (1, 2 or 4; from the wavenumbers, the operator
 * combination, BAEMM_TUNE_TC_CHUNKS and BAEMM_TUNE_TC_SHARE), or a negative
 * error code when no operators are loaded. */
int baemm_tc_entry_sharing(const baemm_ctx *ctx);
/* CUDA graphs for the solvers' inner operators (no reference counterpart;
 * default off).  When on, the GMRES operator apply and the CG mass inverse of
 * BoundaryPotential / DirichletToNeumann / FarField and the derivative solves
 * run as fixed launch sequences: the second call with the same operands is
 * captured (thread-local capture mode, on the context's stream) and later
 * calls replay the graph, which saves the launch overhead that dominates small
 * meshes.  Graphs are dropped when the library reallocates a device buffer or
 * when the mesh, the loaded operators, the apply mode or the tuning change;
 * they are not used on the legacy default stream or while profiling.  Results
 * are the same as without graphs.  baemm_graph_stats counts captures and
 * replays since the context was created. */
int baemm_set_graphs(baemm_ctx *ctx, int on);
int baemm_graph_stats(const baemm_ctx *ctx, int64_t *captures, int64_t *replays);
/* Autotuner (no reference counterpart): times the dense-kernel settings of
 * `mode` on the loaded operators, with the mesh and wave counts of the
 * context, `repeats` timed runs each (>= 1), keeps the fastest in the context
 * and reports it.  BAEMM_APPLY_FP32: the three plain variants;
 * BAEMM_APPLY_TC: generator warps {16, 8} x chunk groups per unit {4, 2, 1}
 * (those the wave shape allows) at segment 16, then segments {8, 32} around
 * the winner.  A TC request whose wave shape the tensor-core form does not
 * support tunes the plain kernel.  The choice is cached for the process per
 * (device, simplex and vertex count, wave_count, wave_chunk_size, form,
 * operator structure): a later call with the same key applies it without
 * timing (cached = 1, before_ms = -1).  Requires
 * baemm_load_boundary_operators; synchronises the context. */
typedef struct baemm_tune_result
{
    int32_t apply_mode;      /* the form tuned (BAEMM_APPLY_*) */
    int32_t dense_variant;   /* chosen BAEMM_TUNE_DENSE_VARIANT (plain form) */
    int32_t tc_segment;      /* chosen BAEMM_TUNE_TC_SEGMENT (tensor-core form) */
    int32_t tc_ctas;         /* BAEMM_TUNE_TC_CTAS in force */
    int32_t tc_stagger;      /* BAEMM_TUNE_TC_STAGGER in force */
    int32_t candidates;      /* settings timed */
    double  best_ms;         /* dense-kernel time of the chosen setting */
    double  before_ms;       /* dense-kernel time of the setting in force before (-1: cached) */
    int32_t tc_gen_warps;    /* chosen BAEMM_TUNE_TC_GEN_WARPS */
    int32_t tc_chunks;       /* chunk groups per work unit in force */
    int32_t cached;          /* 1: taken from the process cache, nothing timed */
    int32_t reserved;
} baemm_tune_result;
int baemm_autotune(baemm_ctx *ctx, int mode, int repeats, baemm_tune_result *out);
/* Empties the autotuner's process cache (the next baemm_autotune times again). */
void baemm_autotune_forget(void);
/* FP64 iterative refinement around the inner GMRES (0 = off, the reference's
 * behaviour).  When on, the solve's outer residual uses the FP64 apply and
 * the inner GMRES uses the context's apply mode. No reference counterpart. */
int baemm_set_refinement(baemm_ctx *ctx, int max_steps, double inner_tol);
/* Areas / TriangleAreas (GetSetters.hpp:123-126, 195-198): nt floats. */
int baemm_get_areas(baemm_ctx *ctx, float *out);
/* TriangleNormals / TriangleMidpoints (GetSetters.hpp:200-208): nt x 4 floats (w = 0). */
int baemm_get_triangle_normals(baemm_ctx *ctx, float *out4);
int baemm_get_triangle_midpoints(baemm_ctx *ctx, float *out4);
/* SingleLayerDiagonal (GetSetters.hpp:190-193): nt floats. */
int baemm_get_single_layer_diagonal(baemm_ctx *ctx, float *out);
/* MassMatrix (GetSetters.hpp:113-116) as CSR: outer (nv+1), inner (nnz),
 * values (nnz).  Call with outer == NULL to query *nnz only. */
int baemm_get_mass_matrix(baemm_ctx *ctx, int64_t *outer, int32_t *inner, float *values, int64_t *nnz);
/* CurlOp (Initialize.hpp:146-211; the reference builds it as a member and no
 * public method uses it): 3 simplex_count x vertex_count CSR, rows 3 t + d
 * (d = x, y, z) of triangle t, the three vertex columns of the triangle in
 * ascending order; value = (area * nu_t x grad phi_v)[d] in FP32, phi_v the P1
 * basis function of vertex v.  outer: 3 simplex_count + 1, inner and values:
 * 9 simplex_count.  Call with outer == NULL to query *nnz only. */
int baemm_get_curl_operator(baemm_ctx *ctx, int64_t *outer, int32_t *inner, float *values, int64_t *nnz);
/* Statistics of the last solve on this context. */
int baemm_last_solve_stats(const baemm_ctx *ctx, baemm_solve_stats *out);

/* ---- parameters and operators -------------------------------------------- */

/* LoadParameters (LoadParameters.hpp:20-81): kappa (wave_chunk_count reals),
 * coeff (wave_chunk_count x 4 complex: mass, SL, DL, adjoint DL).  SL/DL/DL'
 * are scaled by factor/(4 pi).  wave_count must be a multiple of wcs. */
int baemm_load_parameters(baemm_ctx *ctx, const double *kappa, const double *coeff,
                          int wave_count, int wave_chunk_size, double factor);
/* LoadBoundaryOperators_PL / UnloadBoundaryOperators_PL
 * (ApplyBoundaryOperators.hpp:261-284). */
int baemm_load_boundary_operators(baemm_ctx *ctx, const double *kappa, const double *coeff,
                                  int wave_count, int wave_chunk_size);
int baemm_unload_boundary_operators(baemm_ctx *ctx);

/* ApplyBoundaryOperators_PL (ApplyBoundaryOperators.hpp:289-391), operators
 * already loaded: C_out = alpha * A * B_in + beta * C_out on vertex_count x
 * wave_count blocks, A = c0 M + c1 SL + c2 DL + c3 DL' per wave chunk. */
int baemm_apply_boundary_operators_z(baemm_ctx *ctx, const double alpha[2], const double *B_in, int64_t ldB,
                                     const double beta[2], double *C_out, int64_t ldC);
int baemm_apply_boundary_operators_c(baemm_ctx *ctx, const float alpha[2], const float *B_in, int64_t ldB,
                                     const float beta[2], float *C_out, int64_t ldC);
int baemm_apply_boundary_operators_dev_z(baemm_ctx *ctx, const double alpha[2], const double *B_in, int64_t ldB,
                                         const double beta[2], double *C_out, int64_t ldC);
int baemm_apply_boundary_operators_dev_c(baemm_ctx *ctx, const float alpha[2], const float *B_in, int64_t ldB,
                                         const float beta[2], float *C_out, int64_t ldC);
/* Allocation-free variant of baemm_apply_boundary_operators_dev_c.  No
 * counterpart in the reference.  For callers that cannot allocate device
 * memory while they run (hosts that own all device memory through their own
 * pool or budget, servers that must not grow their footprint after start-up,
 * loops that cannot afford cudaMalloc's implicit synchronisation): the
 * triangle-level intermediate blocks live in one fixed 32 MiB __device__
 * array of the library instead of cudaMalloc'ed buffers, so the call
 * allocates and frees nothing.
 * Limit: 2 * simplex_count * wave_count * 8 bytes <= 32 MiB, else
 * BAEMM_ERR_SIZE.  Plain FP32 apply mode only; operators loaded beforehand.
 * The array's device address is looked up on the first call on a device
 * (make it before any stream capture) and cached for the process, so
 * cudaDeviceReset is not supported while the library is loaded.  All calls
 * share the array: calls that overlap on the GPU race and must be serialised
 * by the caller.  The call records no phase timings. */
int baemm_apply_boundary_operators_noalloc_dev_c(baemm_ctx *ctx, const float alpha[2], const float *B_in,
                                                 int64_t ldB, const float beta[2], float *C_out, int64_t ldC);
/* The overload that loads, applies and unloads in one call
 * (ApplyBoundaryOperators.hpp:238-256). */
int baemm_apply_boundary_operators_full_z(baemm_ctx *ctx, const double alpha[2], const double *B_in, int64_t ldB,
                                          const double beta[2], double *C_out, int64_t ldC,
                                          const double *kappa, const double *coeff, int wave_count,
                                          int wave_chunk_size);

/* ApplyFarFieldOperators_PL (ApplyFarFieldOperators.hpp:334-412):
 * C_out (meas_count x wave_count) = alpha * (c1 FF_SL + c2 FF_DL) B_in + beta * C_out.
 * The `_loaded` variant uses the parameters already loaded
 * (ApplyFarFieldOperators.hpp:356-359). */
int baemm_apply_far_field_operators_z(baemm_ctx *ctx, const double alpha[2], const double *B_in, int64_t ldB,
                                      const double beta[2], double *C_out, int64_t ldC,
                                      const double *kappa, const double *coeff, int wave_count,
                                      int wave_chunk_size);
int baemm_apply_far_field_operators_loaded_z(baemm_ctx *ctx, const double alpha[2], const double *B_in,
                                             int64_t ldB, const double beta[2], double *C_out, int64_t ldC);
int baemm_apply_far_field_operators_dev_z(baemm_ctx *ctx, const double alpha[2], const double *B_in, int64_t ldB,
                                          const double beta[2], double *C_out, int64_t ldC);

/* One row shard of ApplyBoundaryOperators_PL for an apply split by target
 * triangles over several GPUs (no reference counterpart; the reference runs on
 * one device).  On device blocks:
 *   C_out = alpha * AvOp^T|rows (K[rows, :] + SL diagonal) AvOp B_in
 *           [+ alpha * c0 * Mass B_in  if with_mass]  + beta * C_out,
 * rows = triangles [row_begin, row_end), every source included.  For a
 * partition of [0, simplex_count) into shards, with with_mass and beta on one
 * shard only (beta = 0 on the others), the shards' C_out sum to the full apply;
 * one all-reduce of the vertex block combines them (baemm_b200.sharded). */
int baemm_apply_boundary_operators_rows_dev_z(baemm_ctx *ctx, const double alpha[2], const double *B_in, int64_t ldB,
                                              const double beta[2], double *C_out, int64_t ldC, int64_t row_begin,
                                              int64_t row_end, int with_mass);
int baemm_apply_boundary_operators_rows_dev_c(baemm_ctx *ctx, const float alpha[2], const float *B_in, int64_t ldB,
                                              const float beta[2], float *C_out, int64_t ldC, int64_t row_begin,
                                              int64_t row_end, int with_mass);

/* Packing of concurrent solves' tensor-core applies into one launch (no
 * reference counterpart; the reference solves one request per GMRES call,
 * FarField.hpp:706-708).  Contexts attached to one packer (same device, each
 * driven by its own thread, e.g. the slots of a server) submit the dense
 * stage of every operator apply inside their solves (BoundaryPotential,
 * DirichletToNeumann, FarField, the derivatives) to the packer instead of
 * launching it.  A submission waits until every attached context that is
 * inside a solve has submitted too, or until max_wait_us has passed, and then
 * one persistent tensor-core launch covers all pending problems of the same
 * operator structure, chunk grouping and warp count (whole target blocks per
 * CTA, longest first), after which each context's stream continues.  Only
 * problems whose own launch cannot fill the GPU (at most two 128-triangle
 * target blocks per SM, counting chunk groups) are packed; larger ones launch
 * alone.  Each
 * problem's result is the same whatever it is packed with.  Applies outside
 * the KI coefficient structure of the solve operators (and row shards) are
 * launched alone as before; with a packer the solve's operator apply is not
 * captured in a CUDA graph (the mass inverse still is).  Destroy a packer only
 * after detaching every context from it.
 * baemm_packer_create returns NULL on failure (message: baemm_last_error(NULL)). */
typedef struct baemm_packer baemm_packer;
baemm_packer *baemm_packer_create(int device, int max_wait_us);
void baemm_packer_destroy(baemm_packer *packer);
int baemm_set_packer(baemm_ctx *ctx, baemm_packer *packer);   /* NULL detaches */
int baemm_packer_stats(const baemm_packer *packer, int64_t *launches, int64_t *problems);

/* Self-test of the tensor-core kernel's bounded pipeline waits (no reference
 * counterpart): one warp on `device` waits on an mbarrier that nothing
 * arrives on, through the same wait code as the kernel's pipeline stages.
 * The wait gives up after its bound (200 ms of device time); *code receives
 * the error code it wrote (99) and *elapsed_ms the time until it gave up.
 * Faults, traps and hangs nothing; the device stays usable.  Errors: message
 * in baemm_last_error(NULL). */
int baemm_selftest_bounded_wait(int device, double *elapsed_ms, int *code);

/* Device time of one CG iteration of the mass inverse on this context's mesh,
 * on the path its solves take (no reference counterpart): 2 * columns real
 * columns (columns complex), `iterations` iterations with no column allowed
 * to converge.  out[0] = ms per iteration, out[1] = algorithmic bytes of one
 * iteration (matvec, update and p update), out[2] = 1 when the mesh (at most
 * 16384 vertices) takes the one-launch path (one block per column, every
 * iteration in one launch), 0 for the three-launches-per-iteration kernels
 * of larger meshes. */
int baemm_profile_cg(baemm_ctx *ctx, int columns, int iterations, double out[3]);

/* The dense stage alone, the device counterpart of the reference's private
 * BoundaryOperatorKernel() (BoundaryOperatorKernel.hpp:5-28, kernel
 * BoundaryOperatorKernel.cl:5-239; no public counterpart): on device
 * triangle blocks (simplex_count x wave_count, leading dimension wave_count),
 *   C_tri[i, :] = sum_{j != i} A_ij(kappa) B_tri[j, :],  i in [row_begin, row_end),
 * with the loaded operators and the current apply mode: _c in the plain FP32
 * or the tensor-core form, _z in the FP64 form (BAEMM_APPLY_FP64 required).
 * Rows outside the range are left untouched.  No AvOp, diagonal or mass. */
int baemm_boundary_operator_kernel_dev_c(baemm_ctx *ctx, const float *B_tri, float *C_tri, int64_t row_begin,
                                         int64_t row_end);
int baemm_boundary_operator_kernel_dev_z(baemm_ctx *ctx, const double *B_tri, double *C_tri, int64_t row_begin,
                                         int64_t row_end);

/* ApplyNearFieldOperators_PL (ApplyNearFieldOperators.hpp:56-122, kernel
 * NearFieldOperatorKernel.cl:5-194): the boundary potential of the vertex
 * values B_in (vertex_count x wave_count) at evaluation points,
 *   C_out (point_count x wave_count) = alpha * (c1 SL + c2 DL)(points) AvOp B_in
 *                                      + beta * C_out,
 * no pair excluded, c0 (mass) and c3 (adjoint double layer) not used.
 * evaluation_points: point_count x 3.  Uses the loaded parameters (the
 * reference's overload without kappa_list); returns without touching C_out
 * when none are loaded or neither layer is present, as the reference does.
 * The arithmetic is the context's apply mode (FP32, tensor-core, FP64).
 * The reference writes C_out with leading dimension wave_count whatever ldC_out
 * is (ApplyNearFieldOperators.hpp:76,112-116); here ldC is honoured (the same
 * when ldC == wave_count).  A point that coincides with a triangle midpoint
 * gives non-finite values in its row, as in the reference (r = 0).  At most
 * 2^28 points per call (BAEMM_ERR_SIZE beyond). */
int baemm_apply_near_field_operators_z(baemm_ctx *ctx, const double alpha[2], const double *B_in, int64_t ldB,
                                       const double beta[2], double *C_out, int64_t ldC,
                                       const double *evaluation_points, int64_t point_count);
int baemm_apply_near_field_operators_c(baemm_ctx *ctx, const float alpha[2], const float *B_in, int64_t ldB,
                                       const float beta[2], float *C_out, int64_t ldC,
                                       const float *evaluation_points, int64_t point_count);
/* The overload with kappa_list / coeff_list (ApplyNearFieldOperators.hpp:27-50):
 * loads the parameters first, as LoadParameters does. */
int baemm_apply_near_field_operators_full_z(baemm_ctx *ctx, const double alpha[2], const double *B_in, int64_t ldB,
                                            const double beta[2], double *C_out, int64_t ldC, const double *kappa,
                                            const double *coeff, int wave_count, int wave_chunk_size,
                                            const double *evaluation_points, int64_t point_count);
/* Device-pointer forms (no reference counterpart): B_in, C_out and
 * evaluation_points (point_count x 3 doubles) in device memory; enqueued on the
 * context's stream without host synchronisation. */
int baemm_apply_near_field_operators_dev_z(baemm_ctx *ctx, const double alpha[2], const double *B_in, int64_t ldB,
                                           const double beta[2], double *C_out, int64_t ldC,
                                           const double *evaluation_points, int64_t point_count);
int baemm_apply_near_field_operators_dev_c(baemm_ctx *ctx, const float alpha[2], const float *B_in, int64_t ldB,
                                           const float beta[2], float *C_out, int64_t ldC,
                                           const double *evaluation_points, int64_t point_count);

/* CreateIncidentWave_PL (CreateIncidentWave.hpp:21-50): weak-form incident
 * waves, C_out (vertex_count x wave_count) = alpha * wave + beta * C_out.
 * incident_directions: inc_count x 3 (plane directions or point sources). */
int baemm_create_incident_wave_z(baemm_ctx *ctx, const double alpha[2], const double *incident_directions,
                                 int inc_count, const double beta[2], double *C_out, int64_t ldC,
                                 const double *kappa, const double *coeff, int wave_count, int wave_chunk_size,
                                 int wave_type);
/* The overload with the loaded parameters (CreateIncidentWave.hpp:55-124):
 * the parameters of the last baemm_load_parameters call (factor as given
 * there; the overload above loads with 4 pi), wave_chunk_size directions.
 * C_out is left untouched when nothing is loaded or neither layer is present. */
int baemm_create_incident_wave_loaded_z(baemm_ctx *ctx, const double alpha[2], const double *incident_directions,
                                        const double beta[2], double *C_out, int64_t ldC, int wave_type);

/* CreateHerglotzWave_PL (CreateHerglotzWave.hpp:25-44): weak-form Herglotz
 * waves of the kernel g (meas_count x wave_count). */
int baemm_create_herglotz_wave_z(baemm_ctx *ctx, const double alpha[2], const double *g, int64_t ldg,
                                 const double beta[2], double *C_out, int64_t ldC,
                                 const double *kappa, const double *coeff, int wave_count, int wave_chunk_size);
/* The overload with the loaded parameters (CreateHerglotzWave.hpp:51-95):
 * the parameters of the last baemm_load_parameters call (the overload above
 * loads with factor 4 pi / meas_count). */
int baemm_create_herglotz_wave_loaded_z(baemm_ctx *ctx, const double alpha[2], const double *g, int64_t ldg,
                                        const double beta[2], double *C_out, int64_t ldC);

/* ApplyMassInverse (ApplyMassInverse.hpp:6-156): Y = M^-1 X by CG
 * (<= 20 iterations, lumped-mass preconditioner).  _z: nrhs complex columns,
 * _d: nrhs real columns. */
int baemm_apply_mass_inverse_z(baemm_ctx *ctx, const double *X, int64_t ldX, double *Y, int64_t ldY,
                               int nrhs, double cg_tol);
int baemm_apply_mass_inverse_d(baemm_ctx *ctx, const double *X, int64_t ldX, double *Y, int64_t ldY,
                               int nrhs, double cg_tol);
/* ApplyLumpedMassInverse (ApplyMassInverse.hpp:161-197). */
int baemm_apply_lumped_mass_inverse_z(baemm_ctx *ctx, const double *X, int64_t ldX, double *Y, int64_t ldY,
                                      int nrhs);
int baemm_apply_lumped_mass_inverse_d(baemm_ctx *ctx, const double *X, int64_t ldX, double *Y, int64_t ldY,
                                      int nrhs);
/* MassMatrix().Dot as used by callers (Example_GaussNewton/main.cpp:391-395):
 * Y = alpha M X + beta Y on nrhs real columns. */
int baemm_mass_dot_d(baemm_ctx *ctx, double alpha, const double *X, int64_t ldX, double beta, double *Y,
                     int64_t ldY, int nrhs);

/* ---- solvers (FarField.hpp) ---------------------------------------------- */

/* FarField<WC> (FarField.hpp:28-70); Y_out: meas_count x (wcc*wcs). */
int baemm_far_field(baemm_ctx *ctx, const double *kappa, int wave_chunk_count, const double *inc_directions,
                    int wave_chunk_size, double *Y_out, int wave_type, double cg_tol, double gmres_tol);
/* FarField_parameters (FarField.hpp:90-144) with coupling parameters eta. */
int baemm_far_field_parameters(baemm_ctx *ctx, const double *kappa, int wave_chunk_count,
                               const double *inc_directions, int wave_chunk_size, double *Y_out, int wave_type,
                               const double *eta, double cg_tol, double gmres_tol);
/* BoundaryPotential (FarField.hpp:626-658): solves (1/2 M - i kappa SL + DL) phi = wave;
 * writes the used coefficients to coeff (wcc x 4 complex). */
int baemm_boundary_potential(baemm_ctx *ctx, const double *kappa, double *coeff, const double *wave, double *phi,
                             int wave_chunk_count, int wave_chunk_size, double cg_tol, double gmres_tol);
/* DirichletToNeumann (FarField.hpp:790-879): solves (1/2 M - i kappa SL + DL') psi = wave. */
int baemm_dirichlet_to_neumann(baemm_ctx *ctx, const double *kappa, const double *wave, double *neumann_trace,
                               int wave_chunk_count, int wave_chunk_size, double cg_tol, double gmres_tol);
/* Derivative_FF_Helper (FarField.hpp:148-207); du_dn: vertex_count x wc. */
int baemm_derivative_ff_helper(baemm_ctx *ctx, const double *kappa, int wave_chunk_count,
                               const double *inc_directions, int wave_chunk_size, double *du_dn, int wave_type,
                               double cg_tol, double gmres_tol);
/* Derivative_FF (FarField.hpp:227-321).  X_in: vertex_count x 3 reals,
 * Y_out: meas_count x wc.  *du_dn == NULL: the library allocates it with
 * calloc (release with baemm_free or free) and fills it, as the reference
 * does (FarField.hpp:273-283). */
int baemm_derivative_ff(baemm_ctx *ctx, const double *kappa, int wave_chunk_count, const double *inc_directions,
                        int wave_chunk_size, const double *X_in, double *Y_out, double **du_dn, int wave_type,
                        double cg_tol, double gmres_tol);
/* AdjointDerivative_FF (FarField.hpp:342-428).  g: meas_count x wc complex,
 * Y_out: vertex_count x 3 reals. */
int baemm_adjoint_derivative_ff(baemm_ctx *ctx, const double *kappa, int wave_chunk_count,
                                const double *inc_directions, int wave_chunk_size, const double *g, double *Y_out,
                                double **du_dn, int wave_type, double cg_tol, double gmres_tol);
/* GaussNewtonSolve (FarField.hpp:457-604): X = alpha (M + DF* DF)^-1 B + beta X
 * by GMRES (solver = 0, the reference) or CG (solver = 1) on 3 * vertex_count
 * reals.  M and P act on vertex_count x 3 host arrays.  *succeeded receives
 * the reference's bool. */
int baemm_gauss_newton_solve(baemm_ctx *ctx, const double *kappa, int wave_chunk_count,
                             const double *inc_directions, int wave_chunk_size, baemm_real_op M, void *M_user,
                             baemm_real_op P, void *P_user, double alpha, const double *B_in, int64_t ldB,
                             double beta, double *X_out, int64_t ldX, double **du_dn, int wave_type, double cg_tol,
                             double gmres_tol_inner, double gmres_tol_outer, int solver, int *succeeded);

/* ---- tracing (the reference's Tools profiler, ptic/ptoc) -------------------- */

/* Device time of the Krylov-vector kernels on this context's mesh (no
 * reference counterpart; a measurement hook for ApplyMassInverse.hpp:48-156
 * and the GMRES of FarField.hpp:706-708 as implemented here):
 *   the CG mass inverse (the GMRES preconditioner) on 2 * columns real
 *   columns for `iterations` iterations, and one Gram-Schmidt pass of a GMRES
 *   iteration on `columns` complex columns against `basis` vectors.
 * out[0..4]: mean ms per launch of {cg_matvec, cg_update, cg_pupdate,
 * gs_dot, gs_update}; out[5..9]: their algorithmic bytes per launch (every
 * operand read or written once: the mass CSR, the lumped inverse and the
 * n x c vectors the kernel touches). */
int baemm_profile_krylov(baemm_ctx *ctx, int columns, int iterations, int basis, double out[10]);

/* Per-phase CUDA-event timing of boundary applies on this context (0 = off). */
int baemm_set_profiling(baemm_ctx *ctx, int on);
/* Device milliseconds of the last boundary apply: ms3[0] AvOp, ms3[1] dense
 * kernel, ms3[2] epilogue (AvOp^T + SL diagonal + mass).  Synchronises on
 * the apply.  Needs profiling on. */
int baemm_last_apply_times(baemm_ctx *ctx, float *ms3);
/* Number of kernels this library has launched in the process so far. */
int64_t baemm_kernel_launch_count(void);

/* Release memory the library allocated for the caller (du_dn). */
void baemm_free(void *p);

#ifdef __cplusplus
}
#endif
#endif /* BAEMM_H */
