/*
 * cudafusion_b200.h — C ABI of the B200 (sm_100a) non-rigid warp-field solve.
 *
 * This library replaces one path of CUDAFusion: the per-frame Gauss-Newton +
 * block-Jacobi PCG solve over a dual-quaternion deformation graph and the node
 * update around it.  Every entry point below names the reference interface it
 * stands in for (file:line inside the CUDAFusion project).
 *
 * Conventions
 *  - All pointers named d_* are device pointers owned by the caller.
 *  - `stream` is a cudaStream_t passed as void* so that this header needs no
 *    CUDA include; NULL means the legacy default stream.
 *  - Every call is asynchronous on `stream` unless it returns statistics to
 *    host memory (those calls synchronise `stream` before returning).
 *  - Calls return a cf_status; no call terminates the process (the reference's
 *    CUDA_CHECK exits, include/types.h:14-20).
 *  - A handle is not thread-safe: use one handle per host thread.
 */
#ifndef CUDAFUSION_B200_H
#define CUDAFUSION_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CF_API __attribute__((visibility("default")))
#else
#define CF_API
#endif

#ifdef __cplusplus
extern "C" {
#define CF_ALIGN16 alignas(16)
#else
#define CF_ALIGN16 _Alignas(16)
#endif

#define CF_K_NEIGHBORS 4 /* skinning nodes per point, include/types.h:182 */
#define CF_K_GRAPH 8     /* graph neighbours per node, include/types.h:183 */
#define CF_BLOCK_DIM 6   /* include/types.h:212 */
#define CF_BLOCK_SIZE 36 /* include/types.h:213 */
#define CF_MAX_GN_ITERS 32
#define CF_MAX_NODES_DEFAULT 8192 /* WarpField::MAX_NODES, include/warp_field.h:14 */
/* learned initial increment (no reference counterpart) */
#define CF_MPNN_IN 20
#define CF_MPNN_HIDDEN 64
#define CF_MPNN_OUT 6
#define CF_MPNN_PARAMS 19526
#define CF_MPNN_ROT_SCALE 10.0f     /* rotation-vector features: rad x 10 */
#define CF_MPNN_TRANS_SCALE 100.0f  /* translation features: m x 100 (cm) */
#define CF_MPNN_RES_SCALE 1000.0f   /* residual features: m x 1000 (mm) */

/* ------------------------------------------------------------------------ */
/* Byte-compatible mirrors of the reference structs (include/types.h).       */
/* ------------------------------------------------------------------------ */

typedef struct cf_vec3 { float x, y, z; } cf_vec3;           /* float3 */
typedef struct cf_quat { CF_ALIGN16 float x; float y, z, w; } cf_quat; /* float4 (16-B aligned) */

/* DualQuat, include/types.h:86-94 (32 B, 16-B aligned).  real = rotation
 * quaternion (x,y,z,w); dual = 0.5 * t * real.  A node transform is read as
 * centred at its node: T(p) = R (p - c) + c + t. */
typedef struct cf_dual_quat {
  cf_quat real;
  cf_quat dual;
} cf_dual_quat;

/* DeformNode, include/types.h:185-192 (96 B). */
typedef struct cf_deform_node {
  cf_vec3 pos;
  cf_vec3 normal;
  float radius;
  int neighbors[CF_K_GRAPH];
  float neighbor_w[CF_K_GRAPH];
  int num_neighbors;
} cf_deform_node;

/* Correspondence, include/types.h:198-206 (76 B; `valid` is a C++ bool). */
typedef struct cf_correspondence {
  cf_vec3 src;    /* skinned (live) point */
  cf_vec3 dst;    /* target point */
  cf_vec3 normal; /* target normal */
  int node_ids[CF_K_NEIGHBORS];
  float node_ws[CF_K_NEIGHBORS];
  float weight;
  uint8_t valid;
  uint8_t pad_[3];
} cf_correspondence;

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */

typedef enum cf_status {
  CF_OK = 0,
  CF_ERR_INVALID_ARG = 1,  /* null pointer, negative size, bad alignment */
  CF_ERR_OOM = 2,          /* device allocation failed */
  CF_ERR_NON_FINITE = 3,   /* a NaN/Inf reached the solution or the energy */
  CF_ERR_TIMEOUT = 4,      /* a bounded in-kernel barrier gave up waiting */
  CF_ERR_CUDA = 5,         /* any other CUDA runtime error */
  CF_ERR_CAPACITY = 6,     /* a size exceeds what the handle was created for */
  CF_ERR_NOT_IMPLEMENTED = 7,
  CF_ERR_NO_DEVICE = 8
} cf_status;

CF_API const char* cf_status_string(cf_status s);

/* ------------------------------------------------------------------------ */
/* Solver parameters: GaussNewtonSolver::Params, include/solver.h:13-22.     */
/* Field order and defaults are the reference's.                             */
/* ------------------------------------------------------------------------ */

typedef struct cf_gn_params {
  int gn_iterations;    /* 3 */
  int pcg_iterations;   /* 10 */
  float pcg_tolerance;  /* 1e-4: absolute ||r|| stop, solver_kernels.cu:669 */
  float lambda_smooth;  /* 1.0: ARAP weight */
  float lambda_rot;     /* 1.0: kept for layout; the reference never reads it */
  float lambda_damping; /* 1e-2: relative Levenberg damping, solver_kernels.cu:167-194 */
  int debug;            /* 0 */
} cf_gn_params;

/* Fills the reference defaults (include/solver.h:15-21). */
CF_API cf_status cf_gn_params_default(cf_gn_params* p);

/* Opaque solver handle: owns the block pattern, the BSR values, the rhs, the
 * block-Jacobi inverses and the PCG vectors (the reference allocates the same
 * set in GaussNewtonSolver's constructor, kernels/solver_kernels.cu:486-496). */
typedef struct cf_gn cf_gn;

/* GaussNewtonSolver::GaussNewtonSolver(const Params&, int max_nodes),
 * include/solver.h:24.  `max_corrs` bounds num_corrs of later calls (the
 * reference sizes nothing by it because it accumulates with atomics). */
CF_API cf_status cf_gn_create(const cf_gn_params* params, int max_nodes, int max_corrs,
                       cf_gn** out);
CF_API cf_status cf_gn_destroy(cf_gn* h);
CF_API cf_status cf_gn_set_params(cf_gn* h, const cf_gn_params* params);
CF_API cf_status cf_gn_get_params(const cf_gn* h, cf_gn_params* params);

/* GaussNewtonSolver::solve, include/solver.h:29-35 and
 * kernels/solver_kernels.cu:543-570: ONE linearisation at the given
 * correspondences (src already skinned) -> delta_x [6*num_nodes], ordered
 * (w_x, w_y, w_z, v_x, v_y, v_z) per node.  The transforms are read only by
 * the ARAP term.  The block pattern is rebuilt when num_nodes differs from the
 * previous call, exactly like the reference (solver_kernels.cu:553-561). */
CF_API cf_status cf_gn_linearize_solve(cf_gn* h, const cf_correspondence* d_corrs,
                                int num_corrs, const cf_deform_node* d_nodes,
                                const cf_dual_quat* d_transforms, int num_nodes,
                                float* d_delta_x, void* stream);

/* Options (no reference counterpart; the defaults reproduce the reference):
 *  CF_OPT_ARAP_CONSISTENT  0: the reference's ARAP rotation Jacobian
 *                          (kernels/solver_kernels.cu:140-165, rows q x e_a);
 *                          1: the consistent derivative e_a x q of the left
 *                          update.  With 0 the GN energy can rise for large
 *                          lambda_smooth, exactly as in the reference.
 *  CF_OPT_PCG_CTAS         CTAs of the grid-wide PCG kernel (0 = automatic).
 *  CF_OPT_PCG_MODE         0: automatic (single cluster up to 32 rows per
 *                          CTA of a 16-CTA cluster, else grid-wide or, past
 *                          the GPU's shared memory, streaming); 1: grid-wide
 *                          cooperative PCG with the system in shared memory
 *                          (streaming when it does not fit); 2: single-
 *                          cluster PCG (upper blocks in distributed shared
 *                          memory) when the system fits the cluster's shared
 *                          memory (else grid-wide); 3: streaming PCG (A re-read from HBM
 *                          through TMA bulk copies every iteration, vectors
 *                          in global memory; the automatic choice for systems
 *                          larger than the GPU's shared memory).
 *  CF_OPT_PCG_PIPELINED    0: the reference's PCG (two reductions per
 *                          iteration); 1: pipelined PCG, the same iterates in
 *                          exact arithmetic with one reduction per iteration
 *                          (FP64 recurrences), shared-memory grid-wide mode
 *                          only.
 *  CF_OPT_GRAPH            1 (default): cf_gn_solve / cf_gn_solve_batched
 *                          run their launch sequence (binning, G x (residual,
 *                          assembly, PCG), energy) as a CUDA graph, captured
 *                          on the first call with given sizes, pointers of the
 *                          node and transform arrays, parameters and options,
 *                          replayed on later calls (new correspondence
 *                          buffers of the same sizes replay it too).  Not used
 *                          on the legacy default stream, while profiling, or
 *                          when the caller is capturing `stream` itself.
 *                          0: direct launches. */
#define CF_OPT_ARAP_CONSISTENT 1
#define CF_OPT_PCG_CTAS 2
#define CF_OPT_PCG_MODE 3
#define CF_OPT_PCG_PIPELINED 4
#define CF_OPT_GRAPH 5
/* read only (cf_gn_get_option): 1 when the last solve ran as a CUDA graph */
#define CF_OPT_GRAPH_ACTIVE 6
/* Polls of a PCG grid barrier before it gives up (0 = the default, 1<<22):
 * the kernel then records CF_ERR_TIMEOUT, every later barrier of the launch
 * returns at once, and the solve returns CF_ERR_TIMEOUT with the context
 * intact (its transforms are then not a solution). */
#define CF_OPT_SPIN_LIMIT 7
/* Test hook for the failure path above: every PCG group barrier also waits
 * for this many arrivals that never come (0 in normal use). */
#define CF_OPT_TEST_BARRIER_EXTRA 8
/* Blocks per shared-memory tile of the streaming PCG: 256 (default) or 128. */
#define CF_OPT_STREAM_TILE 9
/* read only: the PCG kernel the current pattern runs (0 before the first
 * solve, 1 grid-wide, 2 single cluster, 3 streaming) */
#define CF_OPT_PCG_ACTIVE 10
CF_API cf_status cf_gn_set_option(cf_gn* h, int option, int value);
CF_API cf_status cf_gn_get_option(const cf_gn* h, int option, int* value);

/* Synchronises `stream` and converts the device error flags of the last
 * solve (bounded-barrier timeout, non-finite result) into a status. */
CF_API cf_status cf_gn_check(cf_gn* h, void* stream);

/* Forces a rebuild of the block pattern from d_nodes on the next solve (the
 * reference keys its cache on num_nodes only, solver_kernels.cu:554; this
 * closes that gap for callers that change topology at constant N). */
CF_API cf_status cf_gn_invalidate_pattern(cf_gn* h);

/* GaussNewtonSolver::system_matrix() / rhs(), include/solver.h:38-39: copies
 * the last assembled system to HOST memory.  Any pointer may be NULL; the
 * counts are returned through num_rows/num_blocks.  Synchronises `stream`. */
CF_API cf_status cf_gn_get_system(cf_gn* h, int* num_rows, int* num_blocks,
                           int* h_row_ptr, int* h_col_idx, float* h_values,
                           float* h_rhs, void* stream);

/* Statistics of the last solve (host copy). */
typedef struct cf_solve_stats {
  double energy_initial;                   /* E at the first linearisation point */
  double energy_final;                     /* E after the last node update */
  double energy_per_iter[CF_MAX_GN_ITERS]; /* E at each linearisation point */
  int pcg_iterations[CF_MAX_GN_ITERS];     /* PCG iterations run per GN iteration */
  double pcg_residual[CF_MAX_GN_ITERS];    /* final ||r|| per GN iteration */
  int gn_iterations_run;
  int num_blocks;          /* nnzb of the block pattern */
  int precond_fallbacks;   /* diagonal blocks whose Cholesky failed (last GN it.) */
  int error_flags;         /* bit 0: barrier timeout, bit 1: non-finite */
  int init_rejected;       /* learned solve: 1 when the predicted start was not kept */
  double energy_warm_start; /* learned solve: E at the warm start */
  double energy_predicted;  /* learned solve: E at the network's predicted start */
} cf_solve_stats;

/* One problem of the multi-iteration solve.  The correspondences carry the
 * canonical point separately: each GN iteration re-skins it with the current
 * node transforms (se3_math.cuh:450-510), which in the reference happens
 * upstream of the solver (src/skinning_kernels.cu:29-63). */
typedef struct cf_problem {
  const cf_deform_node* nodes;     /* device, num_nodes */
  int num_nodes;
  const float* canon_points;       /* device, 3*num_corrs, xyz per correspondence */
  const cf_correspondence* corrs;  /* device, num_corrs; src is ignored */
  int num_corrs;
  float max_rot;                   /* twist clamp per node (rad), <=0: off */
  float max_trans;                 /* twist clamp per node (m),   <=0: off */
  float update_scale;              /* 1.0 */
} cf_problem;

/* G full Gauss-Newton iterations (G = params.gn_iterations) on one problem:
 * per iteration re-skin -> assemble -> block-Jacobi PCG -> clamped DQ update
 * T_i <- exp(dx_i) * T_i (src/warp_field.cu:250-291), then the energy at the
 * final transforms.  d_transforms is updated in place.  `stats` may be NULL
 * (then the call does not synchronise). */
CF_API cf_status cf_gn_solve(cf_gn* h, const cf_problem* problem,
                      cf_dual_quat* d_transforms, cf_solve_stats* stats,
                      void* stream);

/* Autotuner (no reference counterpart).  Times the PCG configurations that
 * matter for these problems — the system held in shared memory (grid of the
 * automatic size, one or two CTAs per SM) or streamed through TMA tiles (256
 * or 128 blocks per tile; automatic or one CTA per SM) — on the actual
 * problems (the caller's transforms are read, never written; the candidates
 * run on scratch copies, which this call allocates), leaves the fastest set
 * on the handle and remembers it per (SM count, problem count, total nodes and
 * correspondences, GN / PCG iterations): in the process, and in the file named
 * by the environment variable CF_AUTOTUNE_CACHE when set.  A remembered
 * shape is applied without timing (from_cache = 1).  One problem: tuned for
 * cf_gn_solve; several: for cf_gn_solve_batched.  Synchronises `stream`. */
typedef struct cf_tune_result {
  int pcg_mode;     /* the chosen CF_OPT_PCG_MODE */
  int pcg_ctas;     /* the chosen CF_OPT_PCG_CTAS (0 = automatic) */
  int stream_tile;  /* the chosen CF_OPT_STREAM_TILE */
  int candidates;   /* distinct configurations timed */
  double ms_best;   /* median ms of a solve with the choice */
  double ms_default; /* median ms of a solve with the configuration in effect before */
  int from_cache;
} cf_tune_result;
CF_API cf_status cf_gn_autotune(cf_gn* h, const cf_problem* problems, int num_problems,
                                cf_dual_quat* const* d_transforms, cf_tune_result* out, void* stream);

/* Statistics of the handle's last solve, read without running it again
 * (for a caller that ran it with stats = NULL): `num` records in the order of
 * the solve's non-empty problems.  Synchronises `stream`. */
CF_API cf_status cf_gn_last_stats(cf_gn* h, cf_solve_stats* stats, int num, void* stream);

/* Batched solve (no counterpart in the reference, which solves one warp
 * field per call): num_problems independent problems of uneven size, each
 * with its own graph, correspondences, clamps and transforms
 * (d_transforms[p], a host array of device pointers, updated in place), run
 * through G GN iterations together — one launch per phase for the whole
 * batch, one PCG CTA group with its own reductions and stopping test per
 * problem.  The handle's max_nodes / max_corrs bound the batch totals; one
 * problem holds at most 48000 nodes; at most 1024 problems.  Problems with
 * no nodes are skipped.  `stats` (may be NULL: no synchronisation) receives
 * num_problems records, num_blocks being the batch's total. */
CF_API cf_status cf_gn_solve_batched(cf_gn* h, const cf_problem* problems, int num_problems,
                                     cf_dual_quat* const* d_transforms, cf_solve_stats* stats,
                                     void* stream);

/* Per-phase device timing (no reference counterpart; the reference times the
 * whole solve with std::chrono, include/fusion_app.h:386-391).  When enabled,
 * every kernel launch of a solve is bracketed by CUDA events on the launch
 * stream; cf_gn_profile_read synchronises and returns, per phase slot, the
 * summed device milliseconds and the launch count since the last enable.
 * cf_gn_launch_count returns the total kernel launches made by the handle. */
#define CF_PROF_SLOTS 12
CF_API cf_status cf_gn_profile_enable(cf_gn* h, int on);
CF_API cf_status cf_gn_profile_read(cf_gn* h, double* ms, int* launches, int n_slots);
CF_API const char* cf_gn_profile_name(int slot);
CF_API cf_status cf_gn_launch_count(const cf_gn* h, long long* launches);

/* ------------------------------------------------------------------------ */
/* Learned initial increment (no counterpart in the reference, whose every   */
/* frame starts GN from a zero increment).                                    */
/* ------------------------------------------------------------------------ */

/* A message-passing network over the deformation graph that predicts each
 * node's increment for the coming frame: 3 layers (each node's features with
 * the mean of its graph neighbours'), hidden 64, BF16 parameters and
 * activations, FP32 accumulation; output = the last frame's increment plus a
 * learned correction.  Features per node (CF_MPNN_IN = 20): the increments
 * (rotation vector x CF_MPNN_ROT_SCALE, translation x CF_MPNN_TRANS_SCALE) of
 * the last three frames, and the mean and max |residual| (x CF_MPNN_RES_SCALE)
 * of the node's correspondences at the warm start.  Parameters: a flat FP32
 * vector of CF_MPNN_PARAMS (W0 [64][40], b0, W1 [64][128], b1, W2 [64][128],
 * b2, Wo [6][64], bo).  Created with zero parameters (the prediction is then
 * the last frame's increment). */
typedef struct cf_mpnn cf_mpnn;
CF_API cf_status cf_mpnn_create(int max_nodes, cf_mpnn** out);
CF_API cf_status cf_mpnn_destroy(cf_mpnn* net);
/* Sets the FP32 parameters (n = CF_MPNN_PARAMS) and resets the optimiser. */
CF_API cf_status cf_mpnn_set_weights(cf_mpnn* net, const float* h_params, int n);
CF_API cf_status cf_mpnn_get_weights(cf_mpnn* net, float* h_params, int n);
/* The graph for forward / training: d_nbr [num_nodes][CF_K_GRAPH] neighbour
 * indices, -1 = none (synchronises; builds the reverse graph on the host). */
CF_API cf_status cf_mpnn_set_graph(cf_mpnn* net, const int* d_nbr, int num_nodes, void* stream);
/* d_out [N][6] = the predicted increments in feature units. */
CF_API cf_status cf_mpnn_forward(cf_mpnn* net, const float* d_features, float* d_out, void* stream);
/* Loss = mean squared error against d_targets [N][6] (feature units), its
 * gradient into h_grad [CF_MPNN_PARAMS] (either may be NULL); synchronises. */
CF_API cf_status cf_mpnn_gradients(cf_mpnn* net, const float* d_features, const float* d_targets,
                                   float* h_grad, double* h_loss, void* stream);
/* One Adam step (learning rate lr) on the loss above; h_loss may be NULL
 * (then no synchronisation). */
CF_API cf_status cf_mpnn_train_step(cf_mpnn* net, const float* d_features, const float* d_targets,
                                    float lr, double* h_loss, void* stream);
/* Per node the increment (rotation vector, translation) taking d_from to
 * d_to: d_to = D (x) d_from, as centred DQs of the same node; d_out [n][6]. */
CF_API cf_status cf_dq_increments(const cf_dual_quat* d_to, const cf_dual_quat* d_from, int n,
                                  float* d_out, void* stream);
/* The network's features of `problem` at the warm start d_transforms
 * (= T_{t-1}) with d_history = [T_{t-2}, T_{t-3}, T_{t-4}] (3 x num_nodes
 * DQs); d_features [num_nodes][CF_MPNN_IN]. */
CF_API cf_status cf_gn_features(cf_gn* h, const cf_problem* problem, const cf_dual_quat* d_transforms,
                                const cf_dual_quat* d_history, float* d_features, void* stream);
/* cf_gn_solve from a learned start: features, the network's increment
 * applied to the warm start, kept only if its energy is below the warm
 * start's (stats->init_rejected otherwise: the plain warm start is used),
 * then params.gn_iterations GN iterations.  Runs as one CUDA graph like
 * cf_gn_solve. */
CF_API cf_status cf_gn_solve_learned(cf_gn* h, cf_mpnn* net, const cf_problem* problem,
                                     cf_dual_quat* d_transforms, const cf_dual_quat* d_history,
                                     cf_solve_stats* stats, void* stream);

/* Allocation-free energy (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory where they need the energy
 * (a per-frame loop working inside a fixed memory budget owned by a host
 * application; code that must not stall on cudaMalloc/cudaFree, which can
 * synchronise the device and fail under memory pressure).  Computes the
 * solve's IRLS energy E(T) = sum_c fw_c r_c^2 + sum_edges lambda_eff |r_ij|^2
 * at d_transforms for `problem` (max_rot/max_trans/update_scale unused) and
 * writes it to *d_energy (device).  Allocates nothing: its scratch is a static
 * device array of this library sized for CF_NOALLOC_MAX_NODES nodes (about
 * 260 KB, held on every GPU that loads the library until exit); larger
 * problems return CF_ERR_CAPACITY.  Every call made outside a stream capture
 * looks the scratch address up on the current device (cudaGetSymbolAddress),
 * so a device reset between calls is harmless; the first call on a device
 * must therefore come before any stream capture (a capturing first call
 * returns CF_ERR_CUDA).  Calls share the scratch: calls that overlap on the
 * GPU race and must be serialised by the caller.  Asynchronous on `stream`. */
#define CF_NOALLOC_MAX_NODES 8192
CF_API cf_status cf_energy_noalloc(const cf_problem* problem, const cf_dual_quat* d_transforms,
                                   float lambda_smooth, double* d_energy, void* stream);

/* ------------------------------------------------------------------------ */
/* Warp field: WarpField, include/warp_field.h:12-126 (the solve-path subset)*/
/* ------------------------------------------------------------------------ */

/* WarpField::apply_twist_increment, include/warp_field.h:92-94 and
 * src/warp_field.cu:250-291,1121-1141: per node, twist = update_scale*dx,
 * clamp ||w||<=max_rot and ||v||<=max_trans (when > 0), then
 * T_i <- dq_mul(dq_from_twist(twist), T_i). */
CF_API cf_status cf_warp_apply_twist(cf_dual_quat* d_transforms, const float* d_delta_x,
                              int num_nodes, float max_rot, float max_trans,
                              float update_scale, void* stream);

/* DQ skinning of points: warp_point, include/se3_math.cuh:450-510, as used by
 * skin_vertices_from_voxel_knn_kernel (src/skinning_kernels.cu:29-63) with
 * per-point node ids/weights instead of a voxel lookup.  d_out may alias
 * d_points. */
CF_API cf_status cf_warp_skin_points(const float* d_points, const int* d_node_ids,
                              const float* d_node_ws, int num_points,
                              const cf_deform_node* d_nodes,
                              const cf_dual_quat* d_transforms, int num_nodes,
                              float* d_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Projective correspondence search: the producer of the solve's input.     */
/* DynamicFusionPipeline::find_correspondences, include/fusion_app.h:1791-1845:*/
/* compute_pixel_knn_kernel (kernels/tsdf_kernels.cu:573-604) followed by    */
/* find_correspondences_kernel (kernels/tsdf_kernels.cu:386-563).           */
/* ------------------------------------------------------------------------ */

/* CameraIntrinsics, include/types.h:148-162: project(p) = (fx x/z + cx,
 * fy y/z + cy), unproject(u, v, z) = (z (u-cx)/fx, z (v-cy)/fy, z). */
typedef struct cf_camera {
  float fx, fy, cx, cy;
  int width, height;
} cf_camera;

/* Mat4, include/types.h:26-60: row-major rigid transform, p' = M[0:3,0:3] p
 * + M[0:3,3]. */
typedef struct cf_mat4 {
  float m[4][4];
} cf_mat4;

/* The search thresholds of the reference's pipeline parameters
 * (config/params.yaml:60-63; the stock values are 0.2, 0.0, 0.0, 50). */
typedef struct cf_corr_params {
  float dist_threshold;  /* a pair needs |n_dst . (v_live - v_dst)| < this (m) */
  float angle_threshold; /* and |n_live . n_dst| >= this */
  float view_threshold;  /* a live pixel needs |n_live . view ray| >= this */
  int search_radius_px;  /* (2r+1)^2 window around the projection; < 0 acts as 0 */
} cf_corr_params;

/* One frame's inputs, all device arrays of width*height pixels in row-major
 * order, owned by the caller.  The node ids/weights of a pixel come either
 * from d_pixel_knn/d_pixel_knn_w (what find_correspondences_kernel reads) or,
 * when d_pixel_knn is NULL, from the canonical voxel the pixel's ray hit
 * (compute_pixel_knn_kernel fused into the search). */
typedef struct cf_corr_frame {
  const float* d_live_vertices; /* float3 [H*W]: raycast live surface (world); |v| < 1e-6 = none */
  const float* d_live_normals;  /* float3 [H*W]; |n| < 1e-6 = none */
  const float* d_depth;         /* float [H*W]: observed depth (m); <= 0 = none */
  const float* d_depth_normals; /* float3 [H*W] (camera frame); |n| < 1e-6 = none */
  const int* d_pixel_knn;       /* int [H*W][CF_K_NEIGHBORS] or NULL */
  const float* d_pixel_knn_w;   /* float [H*W][CF_K_NEIGHBORS] */
  const int* d_hit_voxel_idx;   /* int [H*W]: canonical voxel hit per pixel, < 0 = none */
  const int* d_voxel_knn;       /* int [num_voxels][CF_K_NEIGHBORS] */
  const float* d_voxel_knn_w;   /* float [num_voxels][CF_K_NEIGHBORS] */
  long long num_voxels;         /* voxel indices >= this count as none */
  int* d_pixel_knn_out;         /* optional (voxel path): the gathered per-pixel ids ... */
  float* d_pixel_knn_w_out;     /* ... and weights, as compute_pixel_knn_kernel writes them */
} cf_corr_frame;

/* Opaque search handle: owns the per-pixel candidate records and the row
 * chunks' partial results (88 B per pixel of the largest frame). */
typedef struct cf_corr_search cf_corr_search;
CF_API cf_status cf_corr_search_create(int max_width, int max_height, cf_corr_search** out);
CF_API cf_status cf_corr_search_destroy(cf_corr_search* h);

/* find_correspondences_kernel over every pixel of a cam->width x
 * cam->height frame: project the live vertex with T_cam_world, search the
 * (2r+1)^2 depth pixels around the projection in row-major order and keep
 * the first candidate of least point-to-plane distance among those within
 * max(3 d, d + 0.03) m (d = dist_threshold) whose normal agrees; the pair is
 * (src = live vertex, dst / normal = the candidate mapped by T_world_cam,
 * weight = the reference's squared mean of distance, normal and view
 * confidences, node ids/weights of the pixel).  Writes all H*W records
 * (invalid ones: valid = 0, weight = 0, ids = -1, other fields 0), the valid
 * count to *d_num_valid and, when d_stats is not NULL, the reference's six
 * debug counters (invalid_live, out_proj, no_depth, far, angle, valid) to
 * d_stats[0..5]; both are overwritten, not accumulated.  FP32 with fused
 * multiply-add accumulation and IEEE division and square roots (the
 * reference's build uses approximate ones: results agree to rounding, and a
 * candidate choice can differ where two candidates tie to a few ulps).
 * Asynchronous on `stream`. */
CF_API cf_status cf_find_correspondences(cf_corr_search* h, const cf_corr_frame* frame, const cf_camera* cam,
                                         const cf_mat4* T_cam_world, const cf_mat4* T_world_cam,
                                         const cf_corr_params* params, cf_correspondence* d_corrs,
                                         int* d_num_valid, int* d_stats, void* stream);

/* compute_pixel_knn_kernel, kernels/tsdf_kernels.cu:573-604: per pixel the
 * CF_K_NEIGHBORS node ids/weights of its hit voxel, (-1, 0) where none. */
CF_API cf_status cf_compute_pixel_knn(const int* d_hit_voxel_idx, int width, int height, const int* d_voxel_knn,
                                      const float* d_voxel_knn_w, long long num_voxels, int* d_pixel_knn,
                                      float* d_pixel_knn_w, void* stream);

/* Kernel launches made through the handle since its creation. */
CF_API cf_status cf_corr_search_launch_count(const cf_corr_search* h, long long* launches);

/* Tuning knob (no reference counterpart): the search splits the rows each
 * 32 x 8 tile of pixels scans into `chunks` parts run by separate CTAs
 * (1..8; 0, the default, picks the count per frame from the tile count and
 * the SM count).  Results do not depend on it. */
CF_API cf_status cf_corr_search_set_chunks(cf_corr_search* h, int chunks);

/* ------------------------------------------------------------------------ */
/* Live-surface prediction: the deformed mesh rasterised into the live maps */
/* the correspondence search reads.                                         */
/* DynamicFusionPipeline::rasterize_deformed_mesh_live_surface,             */
/* include/fusion_app.h:1216-1318: skin_vertices_from_voxel_knn_kernel       */
/* (src/skinning_kernels.cu:29-63), rasterize_triangles_z_kernel and         */
/* resolve_rasterized_triangles_kernel (src/mesh_raster_kernels.cu:76-200). */
/* ------------------------------------------------------------------------ */

/* The canonical voxel grid (TSDFParams origin / voxel_size / dims,
 * include/types.h): voxel (x, y, z) has index (z * dims[1] + y) * dims[0] + x. */
typedef struct cf_voxel_grid {
  float origin[3];
  float voxel_size;
  int dims[3];
} cf_voxel_grid;

/* skin_vertices_from_voxel_knn_kernel: each canonical vertex is warped by the
 * CF_K_NEIGHBORS nodes of the voxel it lies in (warp_point,
 * include/se3_math.cuh:450-510); a vertex outside the grid, or with no nodes
 * at all (num_nodes == 0 or no voxel tables), is copied.  d_voxel_knn /
 * d_voxel_knn_w hold CF_K_NEIGHBORS entries per voxel of the grid.
 * Asynchronous on `stream`. */
CF_API cf_status cf_skin_mesh_vertices(const float* d_canonical, float* d_warped, int num_vertices,
                                       const cf_voxel_grid* grid, const cf_deform_node* d_nodes,
                                       const cf_dual_quat* d_transforms, int num_nodes, const int* d_voxel_knn,
                                       const float* d_voxel_knn_w, void* stream);

/* Opaque raster handle: owns the 64-bit depth/triangle buffer of the largest
 * frame (8 B per pixel), a per-triangle record and list entry (120 B per
 * triangle) and, for cf_predict_live_surface, each node's plain dual
 * quaternion (32 B per node); the latter two are allocated by the first call
 * with a larger mesh or graph, which then synchronises `stream`. */
typedef struct cf_raster cf_raster;
CF_API cf_status cf_raster_create(int max_width, int max_height, cf_raster** out);
CF_API cf_status cf_raster_destroy(cf_raster* h);

/* The rasterisation and resolve of rasterize_deformed_mesh_live_surface: the
 * triangles (int3, indices into both vertex arrays) of the warped mesh are
 * projected with T_cam_world and cam; each pixel keeps the nearest triangle
 * covering its centre (ties: the lower triangle index); the pixel's live
 * vertex is the warped triangle interpolated at the centre, its normal the
 * warped face normal, and its hit voxel the voxel of the canonical triangle
 * interpolated there (-1 outside the grid).  Writes every pixel of the
 * cam->width x cam->height maps (no hit: zero vertex and normal, voxel -1).
 * FP32 with fused multiply-add accumulation and IEEE division and square
 * roots (the reference's build uses approximate ones: results agree to
 * rounding).  Asynchronous on `stream`. */
CF_API cf_status cf_rasterize_live_surface(cf_raster* h, const float* d_canonical, const float* d_warped,
                                           const int* d_triangles, int num_vertices, int num_triangles,
                                           const cf_camera* cam, const cf_mat4* T_cam_world,
                                           const cf_voxel_grid* grid, float* d_live_vertices,
                                           float* d_live_normals, int* d_hit_voxel_idx, void* stream);

/* rasterize_deformed_mesh_live_surface once the mesh is extracted: the
 * canonical vertices skinned into d_warped (the skinning of
 * cf_skin_mesh_vertices, from each node's plain dual quaternion computed once
 * per call on the handle when the voxel tables are 16-byte aligned), then
 * rasterised and resolved (cf_rasterize_live_surface), on one stream.  On a
 * stream of the caller's the launches are captured once and replayed as a
 * CUDA graph while the arguments and the handle's buffers are unchanged.
 * Asynchronous on `stream`. */
CF_API cf_status cf_predict_live_surface(cf_raster* h, const float* d_canonical, float* d_warped, const int* d_triangles,
                                         int num_vertices, int num_triangles, const cf_deform_node* d_nodes,
                                         const cf_dual_quat* d_transforms, int num_nodes, const int* d_voxel_knn,
                                         const float* d_voxel_knn_w, const cf_camera* cam,
                                         const cf_mat4* T_cam_world, const cf_voxel_grid* grid,
                                         float* d_live_vertices, float* d_live_normals, int* d_hit_voxel_idx,
                                         void* stream);

/* Kernel launches made through the handle since its creation. */
CF_API cf_status cf_raster_launch_count(const cf_raster* h, long long* launches);

/* ------------------------------------------------------------------------ */
/* Update validation and line search: the GN step's acceptance.             */
/* The body of DynamicFusionPipeline's GN loop after the solve,             */
/* include/fusion_app.h:409-641, with correspondence_rmse (:1331-1350) and  */
/* upload_scaled_delta_x (:1352-1375), kept on the device.                 */
/* ------------------------------------------------------------------------ */

/* Per-node increment statistics of the validation (fusion_app.h:409-490):
 * rn = |dx[0:3]|, tn = |dx[3:6]|; the raw and the scaled-and-clamped
 * (er = min(update_scale rn, max_rot), et likewise) sums and maxima, summed
 * in FP64 on the device (the reference sums in FP32 in node order). */
typedef struct cf_update_stats {
  double rot_sum, trans_sum, eff_rot_sum, eff_trans_sum;
  float rot_max, trans_max, eff_rot_max, eff_trans_max;
  int finite;    /* every rn and tn finite */
  int num_nodes;
  int iter_ok;   /* the reference's acceptance of the increment (:480-489) */
  int pad_;
} cf_update_stats;

/* The validation's thresholds and the line search's parameters (the
 * pipeline's params_: update_scale, max_update_rot, max_update_trans,
 * max_dx_mean, min_valid_corrs). */
typedef struct cf_line_search_params {
  float update_scale;
  float max_update_rot;
  float max_update_trans;
  float max_dx_mean;
  int min_valid_corrs;
  int pad_;
} cf_line_search_params;

/* The validation statistics and decision for d_delta_x [6*num_nodes]
 * (synchronises `stream`). */
CF_API cf_status cf_validate_update(const float* d_delta_x, int num_nodes, const cf_line_search_params* params,
                                    cf_update_stats* stats, void* stream);

/* upload_scaled_delta_x (fusion_app.h:1352-1375) on the device: per node the
 * rotation part scaled by min(1, max_rot / |w|) and the translation part by
 * min(1, max_trans / |v|) (a bound <= 0 leaves it), both times `scale`. */
CF_API cf_status cf_scale_delta(const float* d_delta_x, int num_nodes, float max_rot, float max_trans, float scale,
                                float* d_out, void* stream);

/* correspondence_rmse (fusion_app.h:1331-1350) on the device: over the
 * records with valid set and weight > 0, r = n . (src - dst) in FP64 (the
 * difference in FP32), sum w r^2 and sum w; d_out[0] = sum, d_out[1] = wsum
 * (device doubles, overwritten).  RMSE = sqrt(sum / wsum), +inf when wsum is
 * 0.  The sums run per block over fixed slices and then in block order, so
 * a result does not depend on scheduling.  d_partials: 2 x CF_RMSE_BLOCKS
 * device doubles of scratch.  Asynchronous on `stream`. */
#define CF_RMSE_BLOCKS 296
CF_API cf_status cf_correspondence_rmse(const cf_correspondence* d_corrs, int num_corrs, double* d_partials,
                                        double* d_out, void* stream);

#define CF_LINE_SEARCH_TRIALS 10
/* device doubles of cf_line_search's d_scratch_rmse */
#define CF_LINE_SEARCH_SCRATCH (2 * CF_RMSE_BLOCKS + 3 * CF_LINE_SEARCH_TRIALS)

/* The line search of fusion_app.h:493-641 for one GN iteration, on the
 * device.  With update_scale <= 0 or a non-finite base_rmse it does nothing
 * (best_scale 0), as the reference breaks there.  Otherwise, for each of the
 * ten trial scales (update_scale x 1, 1/2, 1/4, 1/8, 1/16 and their
 * negatives) the saved transforms are restored, the scaled increment applied
 * (cf_scale_delta, then cf_warp_apply_twist with the clamps and scale 1), the
 * mesh re-predicted (cf_predict_live_surface into frame's live maps and hit
 * voxels), the correspondences searched again (cf_find_correspondences into
 * d_corrs / d_num_valid, the node lists gathered from frame's voxel tables)
 * and their RMSE reduced (cf_correspondence_rmse).  A trial is kept when its
 * valid count reaches min_valid_corrs and (int)(0.75 base_valid) and its
 * RMSE is finite and below the best so far (starting at base_rmse).  The
 * ten trials are enqueued without synchronising and read back once.  Then
 * the saved transforms are restored and, when a trial was kept, its
 * increment applied, the mesh skinned with it and the kept trial's maps,
 * hit voxels, records, valid count and pixel node lists put back (a copy of
 * that trial's outputs held on `search` while the trials run: the same bits
 * as predicting and searching again); when none was, the maps and records
 * stay the last trial's, as in the reference.  The first call, and a call
 * on a larger frame, allocates that copy (104 B per pixel, 136 B with the
 * pixel node lists) and synchronises.  d_transforms holds the warp on entry
 * and the accepted warp on exit; d_scratch_transforms (num_nodes), d_scratch_delta
 * (6 num_nodes) and d_scratch_rmse (CF_LINE_SEARCH_SCRATCH doubles) are the
 * caller's device scratch.  *best_scale = 0 means no update; trial_rmse /
 * trial_valid (CF_LINE_SEARCH_TRIALS each, may be NULL) receive every
 * trial's result.  Synchronises `stream`. */
CF_API cf_status cf_line_search(cf_raster* raster, cf_corr_search* search, const float* d_mesh_canonical,
                                float* d_mesh_warped, const int* d_mesh_triangles, int num_vertices,
                                int num_triangles, const cf_voxel_grid* grid, const cf_deform_node* d_nodes,
                                cf_dual_quat* d_transforms, int num_nodes, const int* d_voxel_knn,
                                const float* d_voxel_knn_w, const float* d_delta_x,
                                const cf_line_search_params* params, cf_corr_frame* frame, const cf_camera* cam,
                                const cf_mat4* T_cam_world, const cf_mat4* T_world_cam,
                                const cf_corr_params* corr_params, cf_correspondence* d_corrs, int* d_num_valid,
                                double base_rmse, int base_valid, cf_dual_quat* d_scratch_transforms,
                                float* d_scratch_delta, double* d_scratch_rmse, float* best_scale,
                                double* best_rmse, double* trial_rmse, int* trial_valid, void* stream);

/* ------------------------------------------------------------------------ */
/* Warped TSDF integration: TSDFVolume::integrate (src/tsdf_volume.cu:23-60,  */
/* include/tsdf_volume.h:27-35) with tsdf_integrate_kernel                    */
/* (kernels/tsdf_kernels.cu:85-174), and the gate's counts,                   */
/* mark_optimized_voxels (include/fusion_app.h:1321-1328,                     */
/* kernels/tsdf_kernels.cu:606-650).                                          */
/* ------------------------------------------------------------------------ */

/* TSDFVoxel, include/types.h:168-176 (12 bytes; a new voxel is tsdf 1,
 * weight 0, colour 128 128 128). */
typedef struct cf_tsdf_voxel {
  float tsdf;
  float weight;
  uint8_t color[3];
  uint8_t pad;
} cf_tsdf_voxel;

/* TSDFVolume::Params, include/tsdf_volume.h:10-19 (stock: 256^3, 0.006 m,
 * truncation 0.03 m, origin (-0.768, -0.768, 0.5), decay 0.9, cap 50).
 * Voxel (x, y, z) has index (z * dims[1] + y) * dims[0] + x and centre
 * origin + (v + 0.5) voxel_size. */
typedef struct cf_tsdf_params {
  int dims[3];
  float voxel_size;
  float truncation;
  float origin[3];
  float decay_alpha; /* the old weight is multiplied by this before an update */
  float max_weight;  /* the updated weight is capped here */
} cf_tsdf_params;

/* The TSDFVolume constructor's initial state (src/tsdf_volume.cu:11-19) for
 * num_voxels voxels.  Asynchronous on `stream`. */
CF_API cf_status cf_tsdf_reset(cf_tsdf_voxel* d_voxels, long long num_voxels, void* stream);

/* T_cam_world as TSDFVolume::integrate forms it from camera_pose (the
 * transposed rotation and -R^T t, src/tsdf_volume.cu:34-50); the bottom row
 * is 0 0 0 1. */
CF_API cf_status cf_tsdf_world_to_camera(const cf_mat4* camera_pose, cf_mat4* T_cam_world);

/* TSDFVolume::integrate: the depth map (cam->width x cam->height, metres,
 * <= 0 = none) is fused into d_voxels (params->dims voxels) seen from
 * camera_pose (camera -> world).  With nodes (d_nodes, d_transforms and
 * num_nodes > 0) each voxel centre is warped by the CF_K_NEIGHBORS entries of
 * its d_voxel_knn / d_voxel_knn_w lists (both 16-byte aligned) and, when
 * d_voxel_opt_counts is given, a voxel whose count is below min_opt_count is
 * skipped; without nodes the integration is rigid (KinectFusion) and the
 * lists and counts are not read.  d_scratch_plain holds num_nodes dual
 * quaternions of the caller's device scratch (may be NULL without nodes).
 * Only tsdf and weight are written.  The volume must have fewer than 2^31
 * voxels.  FP32 with IEEE division (the reference's build uses approximate
 * division: results agree to rounding).  Asynchronous on `stream`. */
CF_API cf_status cf_tsdf_integrate(cf_tsdf_voxel* d_voxels, const cf_tsdf_params* params, const float* d_depth,
                                   const cf_camera* cam, const cf_mat4* camera_pose, const cf_deform_node* d_nodes,
                                   const cf_dual_quat* d_transforms, int num_nodes, const int* d_voxel_knn,
                                   const float* d_voxel_knn_w, const int* d_voxel_opt_counts, int min_opt_count,
                                   cf_dual_quat* d_scratch_plain, void* stream);

/* The warped voxel centres cf_tsdf_integrate projects (3 floats per voxel,
 * index order into d_points); with num_nodes == 0 the canonical centres.
 * Asynchronous on `stream`. */
CF_API cf_status cf_tsdf_warp_voxel_centres(float* d_points, const cf_tsdf_params* params,
                                            const cf_deform_node* d_nodes, const cf_dual_quat* d_transforms,
                                            int num_nodes, const int* d_voxel_knn, const float* d_voxel_knn_w,
                                            cf_dual_quat* d_scratch_plain, void* stream);

/* mark_optimized_voxels_kernel: every pixel with a valid correspondence of
 * weight > 0 and a canonical voxel d_canonical_vidx[px] >= 0 marks the voxels
 * of the 3x3x3 block around it inside the grid (dims): a voxel whose
 * d_voxel_opt_frame differs from frame_id takes frame_id and its
 * d_voxel_opt_counts rises by one.  Asynchronous on `stream`. */
CF_API cf_status cf_mark_optimized_voxels(const cf_correspondence* d_corrs, const int* d_canonical_vidx,
                                          int num_pixels, const int dims[3], int frame_id,
                                          int* d_voxel_opt_counts, int* d_voxel_opt_frame, void* stream);

/* WarpField::compute_voxel_knn, include/warp_field.h:72-74 and
 * src/warp_field.cu:957-981, with compute_voxel_knn_kernel (:299-405): the
 * voxel kNN field of the volume d_voxels (params: dims, origin, voxel_size)
 * over the num_nodes nodes d_nodes.  For every voxel v (index
 * (z * dims[1] + y) * dims[0] + x) it writes d_voxel_knn[4v..4v+3] and
 * d_voxel_knn_w[4v..4v+3]: ids -1 and weights 0 when the voxel's weight is
 * <= 0; otherwise the 4 nodes with the smallest squared distance to the
 * centre origin + (v + 0.5) voxel_size, ties to the lower index, nearest
 * first (-1 / 0 past the number of nodes), each weighted exp(-d / (2 r^2)),
 * r = max(radius, 1e-6), normalised by their sum when it exceeds 1e-8.  The
 * ids are the reference's bit for bit; the weights agree to float rounding.
 * The caller owns both outputs (4 entries per voxel, 16-byte aligned; the
 * reference reallocates its DeviceArrays here).  num_nodes == 0 writes
 * nothing, like the reference.  At most 49152 nodes (CF_ERR_CAPACITY).
 * Asynchronous on `stream`. */
CF_API cf_status cf_compute_voxel_knn(const cf_tsdf_voxel* d_voxels, const cf_tsdf_params* params,
                                      const cf_deform_node* d_nodes, int num_nodes, int* d_voxel_knn,
                                      float* d_voxel_knn_w, void* stream);

/* Library / device information. */
CF_API cf_status cf_get_version(int* major, int* minor, int* patch);
CF_API cf_status cf_last_cuda_error(char* buf, size_t len);

#ifdef __cplusplus
}
#endif

#endif /* CUDAFUSION_B200_H */
