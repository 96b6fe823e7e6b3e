// cf_internal.h — structures shared by the host API (cf_api.cu) and the
// kernel launchers (cf_kernels.cu).  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cudafusion_b200.h"

namespace cf {

constexpr int kThreads = 256;
constexpr int kErrTimeoutBit = 1;   // bounded barrier gave up
constexpr int kErrNonFiniteBit = 2; // NaN/Inf in the solution or energy
constexpr int kStatsSlots = CF_MAX_GN_ITERS + 1;
// float4 per ARAP edge in Pattern::edge_terms: diagonal block + rhs of i (7),
// of j (7), off-diagonal block (9)
constexpr int kEdgeTerms4 = 23;

// Device-side statistics of one solve (copied to cf_solve_stats on request).
struct DevStats {
  double energy[kStatsSlots];          // energy at each linearisation point; [G] = final
  double pcg_res[CF_MAX_GN_ITERS];     // final ||r|| per GN iteration
  int pcg_iters[CF_MAX_GN_ITERS];
  int fallbacks;                        // Cholesky fallbacks of the last GN iteration
  int init_rejected;                    // learned solve: the predicted start was not kept
  double gate[2];                       // learned solve: energy at the warm start, at the prediction
};

// One problem of a solve as the kernels see it; a single solve is a batch of
// one.  Correspondences and nodes of all problems live in one concatenated
// index space (node ids inside the packed records are global).
struct ProbDesc {
  const cf_correspondence* corrs;  // the caller's rows, indexed locally
  const float* canon;              // canonical points (nullptr: linearise at src)
  const cf_deform_node* nodes;     // the caller's nodes (batched solves gather them)
  cf_dual_quat* T;                 // the caller's transforms (batched solves gather/scatter)
  long long cnt_off;               // first histogram word of this problem in Work::cnt
  int M, N;
  int corr_off, node_off;          // first correspondence / node in the concatenated space
  int bin_cta0, bin_ctas, chunk;   // sort CTAs of this problem, correspondences per CTA
  int e_cta0, e_ctas;              // residual / energy CTAs, one FP64 partial each
  float max_rot, max_trans, update_scale;
  int pad_[2];
};
static_assert(sizeof(ProbDesc) == 96, "ProbDesc has no padding (compared bytewise)");

// Per-call problem table (device copies of the host arrays).
struct Table {
  int P = 0;
  int n_bin = 0, n_e = 0;    // total sort / energy CTAs
  int M = 0, N = 0;          // concatenated sizes
  int max_N = 0;             // largest problem (shared-memory histograms)
  int max_chunk = 0;         // most correspondences of one sort CTA
  ProbDesc* desc = nullptr;  // [P]
  int* bin_prob = nullptr;   // [n_bin] problem of each sort CTA
  long long bin_cap = 0;     // capacity of bin_prob
  int* e_prob = nullptr;     // [n_e] problem of each energy CTA
  int* node_prob = nullptr;  // [N] problem of each node
};

// Block pattern and everything derived from the graph topology.  Built on
// the host (cold path, kernels/solver_kernels.cu:498-541) and uploaded.
struct Pattern {
  int P = 1;               // problems (block-diagonal union for batched solves)
  int* prob_edge_off = nullptr;  // [P+1] ARAP edges of each problem (edge_ijk order)
  int* pcg_cta_off = nullptr;    // [P+1] PCG CTA group of each problem
  int* pcg_prob = nullptr;       // [pcg_ctas] problem of each PCG CTA
  int N = 0;
  int nnzb = 0;
  int n_upper = 0;      // blocks with col >= row (incl. diagonal)
  int n_edges = 0;      // ARAP edges visited by the reference (lower endpoint owns)
  int max_upper_row = 0;  // max upper blocks in one row
  int* row_ptr = nullptr;   // [N+1]
  int* col_idx = nullptr;   // [nnzb]
  int* diag_pos = nullptr;  // [N]
  int* trans_pos = nullptr; // [nnzb] position of the transposed block
  int* upper_pos = nullptr; // [n_upper]
  int* upper_row = nullptr; // [n_upper]
  int* arap_row_ptr = nullptr;  // [N+1]
  int* arap_row_inc = nullptr;  // (edge << 1) | role, role 0 = lower endpoint
  int* arap_blk_ptr = nullptr;  // [n_upper+1] over upper off-diagonal blocks
  int* arap_blk_edge = nullptr;
  int* edge_ijk = nullptr;      // [3*n_edges] i, j, k (slot in i's list)
  float4* edge_terms = nullptr; // [kEdgeTerms4*n_edges] per GN iteration: the edge's block contributions
  double* edge_energy = nullptr; // [n_edges] per GN iteration: el |r|^2
  // per-pattern work arrays
  float* values = nullptr;  // [nnzb*36]
  int* seg_off = nullptr;   // [nnzb]
  int* seg_cnt = nullptr;   // [nnzb]
  int n_off = 0;            // off-diagonal upper blocks
  int* off_upper = nullptr; // [n_off] their upper indices
  // single-cluster PCG (cf_pcg_cluster.cu)
  int use_cluster = 0;
  int clu_C = 0;
  int clu_smem = 0;
  int clu_nup_max = 0, clu_nlow_max = 0, clu_rows_max = 0, clu_halo_max = 0;
  int* clu_row_begin = nullptr;  // [clu_C+1]
  int* ustart = nullptr;         // [N+1] first upper index of each row
  int* low_ptr = nullptr;        // [N+1] lower blocks (j, i), j < i, of row i, in order of j
  int* clu_opnd = nullptr;       // [n_upper] operand slot of the block's column in its CTA: own row, or rows + halo slot
  int* clu_push = nullptr;       // [n_upper] off-diagonal (i, j): (owner of row j << 24) | receive slot of (j, i) there; -1 diagonal
  int* clu_halo_ptr = nullptr;   // [clu_C+1]
  int* clu_halo = nullptr;       // per CTA, its remote columns: (owner << 24) | row local to the owner
  // grid PCG partition
  int pcg_ctas = 0;
  int* pcg_row_begin = nullptr;  // [pcg_ctas+1]
  int pcg_smem = 0;
  int pcg_a_in_smem = 0;
  int pcg_pipelined = 0;
  int* g_vidx = nullptr;      // [nnzb] operand slot of each block's column in its CTA ([own | halo])
  int* g_halo_ptr = nullptr;  // [pcg_ctas+1]
  int* g_halo_col = nullptr;  // distinct columns of other CTAs touched by each CTA
  // streaming PCG (cf_pcg_stream.cu): A streamed from HBM in tiles of whole rows
  int pcg_stream = 0;
  int st_tile_blocks = 256;    // blocks per tile (256 or 128)
  int* st_tile_ptr = nullptr;  // [pcg_ctas+1] into st_tile_row
  int* st_tile_row = nullptr;  // per CTA: its tiles' first rows, then its end row
  int* st_tile_cols = nullptr; // [entries of st_tile_row][tile blocks] each tile's column indices, -1 padded
};

// Per-handle work buffers sized by (max_nodes, max_corrs).
struct Work {
  int max_nodes = 0, max_corrs = 0;
  int bin_ctas_max = 0;
  float4* pk_src = nullptr;  // xyz: canonical point (solve) or src (linearise); w: effective weight
  float4* pk_dst = nullptr;
  float4* pk_nrm = nullptr;
  int4* pk_ids = nullptr;
  float4* pk_ws = nullptr;
  float4* c_srcfw = nullptr;  // skinned src, fw (0 = skipped)
  float4* c_nres = nullptr;   // normal, residual
  float2* c_fr = nullptr;     // (weight, residual) per correspondence, for the learned start's features
  int* cnt = nullptr;         // per sort CTA, a histogram over its problem's nodes
  long long cnt_cap = 0;      // words allocated for cnt
  int* node_total = nullptr;  // [max_nodes]
  int* row_order = nullptr;   // [max_nodes] rows by decreasing incidence count (launch order of the per-row kernels)
  int4* asm_meta = nullptr;   // [3*max_nodes] per launch position: the assembly's row metadata, written by the expand
  int* inc_start = nullptr;   // [max_nodes+1]
  int* inc = nullptr;         // [4*max_corrs]: (c << 2) | a
  int* trip = nullptr;        // [16*max_corrs]: (c << 4) | (a << 2) | b
  int2* ekeys = nullptr;      // [4*max_corrs]: per incidence, column keys of its 4 slots
  float* rhs = nullptr;       // [6*max_nodes]
  cf_dual_quat* plain = nullptr;  // [max_nodes]
  float* x = nullptr;         // [6*max_nodes]
  float* z = nullptr;
  float* p0 = nullptr;
  float* p1 = nullptr;
  double* partials = nullptr;  // [2 bufs][3 slots][max pcg ctas]
  unsigned* barrier = nullptr;  // [max pcg ctas] one arrival counter per PCG CTA group
  int* err = nullptr;
  double* e_data_part = nullptr;  // [kEnergyCtas + kMaxProblems] one partial per energy CTA
  double* e_arap_part = nullptr;  // [max_nodes] per row
  DevStats* stats = nullptr;      // [kMaxProblems]
  // streaming PCG: residual, A p and the FP32 block inverses in global memory
  float* r = nullptr;       // [6*max_nodes]
  float* ap = nullptr;      // [6*max_nodes]
  float* minv32 = nullptr;  // [36*max_nodes]
  cf_dual_quat* T_save = nullptr;  // [max_nodes] learned solve: the warm start
  // batched solves: the problems' nodes and transforms, concatenated
  cf_deform_node* nodes_cat = nullptr;  // [max_nodes]
  cf_dual_quat* T_cat = nullptr;        // [max_nodes]
  long long* timers = nullptr;  // [kTimerSlots] phase cycles of the grid PCG (debug)
};

constexpr int kEnergyCtas = 512;  // residual/energy CTAs of a single solve (with the edge CTAs, one wave at 4 per SM)
constexpr int kMaxPcgCtas = 1024;
constexpr int kSortCorrs = 4096;     // correspondences per sort CTA of a batched solve (at least)
constexpr int kMaxSortCtas = 1 << 16;
constexpr int kClusterAutoRows = 32;  // rows per CTA up to which mode 0 picks the single-cluster PCG
constexpr int kMaxProblems = 1024;       // problems per batched solve
constexpr int kMaxProblemNodes = 48000;  // nodes per problem (per-CTA histograms in shared memory)

struct SolveArgs {
  const cf_deform_node* nodes;
  int N;
  int M;
  float lambda_smooth;
  float lambda_damping;
  int pcg_iterations;
  float pcg_tolerance;
  int arap_consistent;
  // node update (solve) or plain delta_x output (linearise)
  cf_dual_quat* transforms;  // in/out
  float* delta_x;            // non-null: write dx here and do not update
  float max_rot, max_trans, update_scale;
  unsigned spin_limit;
  unsigned bar_extra;  // test hook: arrivals every group barrier waits for beyond its CTAs (0)
  long long* timers;  // non-null: CTA 0 of the grid PCG accumulates phase cycles here
  Table tb;           // the problems of this solve
};
constexpr int kTimerSlots = 16;

#ifdef __CUDACC__
// clock64 phase timer of one thread of the persistent PCG kernels (debug;
// a.timers == nullptr disables it)
struct PhaseClock {
  long long* out;
  long long last;
  long long acc[kTimerSlots];
  __device__ PhaseClock(long long* o) : out(o), last(0) {
#ifdef __CUDA_ARCH__
    last = clock64();
#endif
    for (int i = 0; i < kTimerSlots; i++) acc[i] = 0;
  }
  __device__ __forceinline__ void mark(int slot) {
#ifdef __CUDA_ARCH__
    if (!out) return;
    const long long t = clock64();
    acc[slot] += t - last;
    last = t;
#endif
  }
  __device__ void flush() {
    if (!out) return;
    for (int i = 0; i < kTimerSlots; i++) atomicAdd(reinterpret_cast<unsigned long long*>(out + i), (unsigned long long)acc[i]);
  }
};
#endif


// ---- launchers (cf_kernels.cu) ----
cudaError_t launch_pack_count(const Work& w, const Table& tb, cudaStream_t s);
cudaError_t launch_bin_scan(const Work& w, const Table& tb, cudaStream_t s);
cudaError_t launch_row_order(const Work& w, int N, cudaStream_t s);
cudaError_t launch_bin_scatter(const Work& w, const Table& tb, cudaStream_t s);
cudaError_t launch_expand(const Work& w, const Pattern& p, int N, cudaStream_t s);
cudaError_t launch_node_plain(const Work& w, const cf_deform_node* nodes, const cf_dual_quat* T, int N,
                              cudaStream_t s);
cudaError_t launch_residual(const Work& w, const Table& tb, const Pattern& p, const SolveArgs& a,
                            const cf_dual_quat* T, bool skin, cudaStream_t s, bool fr = false);
cudaError_t launch_batch_gather(const Work& w, const Table& tb, cudaStream_t s);
cudaError_t launch_batch_scatter(const Work& w, const Table& tb, cudaStream_t s);
cudaError_t launch_assemble(const Work& w, const Pattern& p, const SolveArgs& a, const cf_dual_quat* T,
                            cudaStream_t s);
cudaError_t launch_pcg(const Work& w, const Pattern& p, const SolveArgs& a, int gn_slot, cudaStream_t s);
cudaError_t launch_residual_energy(const Work& w, const Pattern& p, const SolveArgs& a, int slot, cudaStream_t s);
cudaError_t launch_final_energy(const Work& w, const Pattern& p, const SolveArgs& a, int slot, cudaStream_t s);
cudaError_t launch_apply_twist(cf_dual_quat* T, const float* dx, int N, float max_rot, float max_trans,
                               float scale, cudaStream_t s);
// cf_corr.cu: projective correspondence search
constexpr int kCorrMaxChunks = 8;
struct CorrScratch {
  float4* A;       // per pixel: unprojected point (x, y, z) and normal x
  float2* B;       // per pixel: normal y, z
  float* part_pd;  // [kCorrMaxChunks][pixels]: each row chunk's best distance ...
  int* part_idx;   // ... and candidate
  int* flag;       // set when a value could make a distance NaN
  int sms;
};
int corr_pick_chunks(int tiles, int sms, int radius, int W, int H);
// cf_linesearch.cu: the GN step's acceptance
cudaError_t launch_update_stats(const float* dx, int N, float update_scale, float max_rot, float max_trans,
                                double* sums, unsigned* maxima, int* finite, cudaStream_t s);
cudaError_t launch_scale_delta(const float* dx, int N, float max_rot, float max_trans, float scale, float* out,
                               cudaStream_t s);
// The line search's record of its best trial (ls_keep_kernel).
struct LsKeepArgs {
  const double* slot;
  const double* best_in;  // nullptr: best0
  double best0;
  double* best_out;
  int* kept;
  int trial, min_valid, need, nbuf;
  const int* src[8];
  int* dst[8];
  size_t words[8];
};
cudaError_t launch_ls_keep(const LsKeepArgs& a, cudaStream_t s);
cudaError_t launch_corr_rmse(const cf_correspondence* corrs, int M, double* partials, double* out, const int* valid,
                             cudaStream_t s);
cudaError_t launch_tsdf_plain(const cf_deform_node* nodes, const cf_dual_quat* T, cf_dual_quat* plain, int N,
                              cudaStream_t s);
cudaError_t launch_tsdf_integrate(float* vox, const cf_tsdf_params* p, const float* depth, const cf_camera* cam,
                                  const float* cw, const int* knn, const float* knn_w, const cf_dual_quat* plain,
                                  int N, const int* counts, int min_opt, cudaStream_t s);
cudaError_t launch_tsdf_centres(float* out, const cf_tsdf_params* p, const int* knn, const float* knn_w,
                                const cf_dual_quat* plain, int N, cudaStream_t s);
cudaError_t launch_mark_optimized(const cf_correspondence* corrs, const int* vidx, int P, const int dims[3],
                                  int frame, int* counts, int* frames, cudaStream_t s);
cudaError_t launch_tsdf_init(cf_tsdf_voxel* vox, unsigned V, cudaStream_t s);
// cf_voxelknn.cu: the voxel kNN field (variant 0: default pruning, 1: tile
// pruning only, 2: tile and warp pruning)
int voxel_knn_max_nodes();
cudaError_t launch_voxel_knn(const float* vox, const cf_tsdf_params* p, const cf_deform_node* nodes, int N,
                             int* ids, float* ws, int variant, cudaStream_t s);
// cf_raster.cu: live-surface prediction
cudaError_t launch_mesh_skin(const float* canon, float* warped, int V, const cf_voxel_grid* grid,
                             const cf_deform_node* nodes, const cf_dual_quat* T, int N, const int* vk, const float* vw,
                             cudaStream_t s);
cudaError_t launch_mesh_skin_plain(const float* canon, float* warped, int V, const cf_voxel_grid* grid,
                                   const cf_dual_quat* plain, int N, const int* vk, const float* vw, cudaStream_t s);
cudaError_t launch_raster(const float* canon, const float* warped, const int* tris, int V, int NT,
                          const cf_camera* cam, const cf_mat4* Tcw, const cf_voxel_grid* grid,
                          unsigned long long* ztri, float4* cache, int* big, unsigned long long* big_ctr, float* lv,
                          float* ln, int* hit, cudaStream_t s, long long* launches);
cudaError_t launch_corr_search(const cf_corr_frame* f, const cf_camera* cam, const cf_mat4* Tcw, const cf_mat4* Twc,
                               const cf_corr_params* p, const CorrScratch& sc, int chunks, cf_correspondence* out,
                               int* num_valid, int* stats, cudaStream_t s, long long* launches);
cudaError_t launch_pixel_knn(const int* hit, int P, const int* vk, const float* vw, long long num_voxels, int* pk,
                             float* pw, cudaStream_t s);
cudaError_t launch_skin_points(const float* pts, const int* ids, const float* ws, int M,
                               const cf_deform_node* nodes, const cf_dual_quat* T, int N, float* out,
                               cudaStream_t s);
cudaError_t launch_energy_noalloc(const cf_problem* pr, const cf_dual_quat* T, float lambda, double* d_energy,
                                  cudaStream_t s);
int pcg_grid_smem_bytes(int nblk, int nrows, int nhalo, bool a_in_smem, bool pipelined);
int pcg_max_active_ctas(int smem, bool a_in_smem, bool pipelined);
int expand_smem_bytes(int max_upper_row, int N);

int pcg_cluster_smem_bytes(int nup_max, int nlow_max, int rows_max, int nhalo_max, int C);
int pcg_cluster_max_active(int C, int smem);
cudaError_t launch_pcg_cluster(const Work& w, const Pattern& p, const SolveArgs& a, int gn_slot, cudaStream_t s);

// The learned initial increment (cf_mpnn.cu): parameters, graph, activations.
struct Mpnn {
  int max_nodes = 0, N = 0;
  long long step = 0;
  float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;  // FP32 master, Adam moments, gradient
  void* wb = nullptr;                                            // BF16 parameters
  int* nbr = nullptr;       // [N][8] neighbour lists, -1 = none
  float* inv_deg = nullptr;  // [N]
  int *rev_ptr = nullptr, *rev_idx = nullptr;  // reverse graph (training)
  float *feat = nullptr, *tgt = nullptr, *out = nullptr;
  void *h1 = nullptr, *h2 = nullptr, *h3 = nullptr;  // BF16 activations [N][64]
  float *dh = nullptr, *dh2 = nullptr, *dcat = nullptr, *part = nullptr;
  double *loss_part = nullptr, *loss = nullptr;
};
int mpnn_param_count();
cudaError_t mpnn_alloc(Mpnn& m, int max_nodes);
void mpnn_free(Mpnn& m);
cudaError_t mpnn_refresh_bf16(const Mpnn& m, cudaStream_t s);
cudaError_t mpnn_graph_from_nodes(Mpnn& m, const cf_deform_node* nodes, int N, cudaStream_t s);
cudaError_t mpnn_forward(const Mpnn& m, const float* feat, float* out, cudaStream_t s);
cudaError_t mpnn_gradients(Mpnn& m, const float* feat, const float* tgt, cudaStream_t s);
cudaError_t mpnn_adam(Mpnn& m, float lr, cudaStream_t s);
cudaError_t launch_increments(const cf_dual_quat* to, const cf_dual_quat* from, int n, float* out, cudaStream_t s);
cudaError_t launch_features(const Work& w, const cf_dual_quat* T, const cf_dual_quat* hist, int N, float* feat,
                            cudaStream_t s);
cudaError_t launch_apply_prediction(const Work& w, cf_dual_quat* T, const cf_deform_node* nodes, const float* pred,
                                    int N, cudaStream_t s);
cudaError_t launch_gate_prediction(const Work& w, cf_dual_quat* T, const cf_deform_node* nodes, int N,
                                   cudaStream_t s);

int pcg_stream_smem_bytes(int tile_blocks);
int pcg_stream_max_active_ctas(int tile_blocks);
cudaError_t launch_pcg_stream(const Work& w, const Pattern& p, const SolveArgs& a, int gn_slot, cudaStream_t s);

}  // namespace cf
