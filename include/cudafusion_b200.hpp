// cudafusion_b200.hpp — C++ drop-in for CUDAFusion's solve-path classes.
//
//   cudafusion_b200::GaussNewtonSolver     include/solver.h:10-89
//   cudafusion_b200::WarpField             include/warp_field.h:12-126 (solve-path subset)
//   cudafusion_b200::CorrespondenceSearch  DynamicFusionPipeline::find_correspondences,
//                                          include/fusion_app.h:1791-1845
//   cudafusion_b200::LiveSurfaceRaster     DynamicFusionPipeline::rasterize_deformed_mesh_live_surface,
//                                          include/fusion_app.h:1216-1318 (after the mesh extraction)
//
// Header-only, on top of the C ABI (cudafusion_b200.h, link libcfb200.so).
// The classes keep the reference's constructor and method signatures and
// its observable behaviour: every call synchronises the device before it
// returns, solve() (re)allocates delta_x to 6*num_nodes floats
// (solver_kernels.cu:551), apply_twist_increment() refreshes the host mirror
// (warp_field.cu:1135-1140).  The reference's own types are accepted
// unchanged: any array type with the members `data`, `count` and
// `allocate(n)` (the reference's DeviceArray<T>, include/types.h:100-142)
// and the structs DualQuat / DeformNode / Correspondence, whose byte layouts
// are checked here at compile time.  Errors throw cudafusion_b200::Error (the
// reference exits through CUDA_CHECK; define CF_DROPIN_EXIT_ON_ERROR to get
// that behaviour instead).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "cudafusion_b200.h"

namespace cudafusion_b200 {

struct Error : std::runtime_error {
  cf_status status;
  Error(cf_status s, const char* where)
      : std::runtime_error(std::string(where) + ": " + cf_status_string(s)), status(s) {}
};

inline void check(cf_status s, const char* where) {
  if (s == CF_OK) return;
#ifdef CF_DROPIN_EXIT_ON_ERROR
  std::fprintf(stderr, "cudafusion_b200 error in %s: %s\n", where, cf_status_string(s));
  std::exit(1);
#else
  throw Error(s, where);
#endif
}

// The caller's DualQuat / DeformNode / Correspondence (include/types.h:86-94,
// 185-192, 198-206) against the ABI structs: sizes, the DualQuat alignment,
// and the byte offset of every field, so a reordered or retyped member fails
// to compile instead of being read at the wrong place.
template <class Node>
constexpr bool node_layout_matches() {
  return sizeof(Node) == sizeof(cf_deform_node) && offsetof(Node, pos) == offsetof(cf_deform_node, pos) &&
         offsetof(Node, normal) == offsetof(cf_deform_node, normal) &&
         offsetof(Node, radius) == offsetof(cf_deform_node, radius) &&
         offsetof(Node, neighbors) == offsetof(cf_deform_node, neighbors) &&
         offsetof(Node, neighbor_w) == offsetof(cf_deform_node, neighbor_w) &&
         offsetof(Node, num_neighbors) == offsetof(cf_deform_node, num_neighbors);
}

template <class DQ>
constexpr bool dq_layout_matches() {
  return sizeof(DQ) == sizeof(cf_dual_quat) && alignof(DQ) == alignof(cf_dual_quat) &&
         offsetof(DQ, real) == offsetof(cf_dual_quat, real) && offsetof(DQ, dual) == offsetof(cf_dual_quat, dual);
}

template <class Corr>
constexpr bool corr_layout_matches() {
  return sizeof(Corr) == sizeof(cf_correspondence) && offsetof(Corr, src) == offsetof(cf_correspondence, src) &&
         offsetof(Corr, dst) == offsetof(cf_correspondence, dst) &&
         offsetof(Corr, normal) == offsetof(cf_correspondence, normal) &&
         offsetof(Corr, node_ids) == offsetof(cf_correspondence, node_ids) &&
         offsetof(Corr, node_ws) == offsetof(cf_correspondence, node_ws) &&
         offsetof(Corr, weight) == offsetof(cf_correspondence, weight) &&
         offsetof(Corr, valid) == offsetof(cf_correspondence, valid);
}

template <class Node, class DQ, class Corr>
constexpr bool layouts_match() {
  return node_layout_matches<Node>() && dq_layout_matches<DQ>() && corr_layout_matches<Corr>();
}

// CameraIntrinsics (include/types.h:148-162) and Mat4 (:26-60).
template <class Cam>
constexpr bool camera_layout_matches() {
  return sizeof(Cam) == sizeof(cf_camera) && offsetof(Cam, fx) == offsetof(cf_camera, fx) &&
         offsetof(Cam, fy) == offsetof(cf_camera, fy) && offsetof(Cam, cx) == offsetof(cf_camera, cx) &&
         offsetof(Cam, cy) == offsetof(cf_camera, cy) && offsetof(Cam, width) == offsetof(cf_camera, width) &&
         offsetof(Cam, height) == offsetof(cf_camera, height);
}

template <class M4>
constexpr bool mat4_layout_matches() {
  return sizeof(M4) == sizeof(cf_mat4) && offsetof(M4, m) == 0;
}

// TSDFVoxel (include/types.h:168-176) and TSDFVolume::Params
// (include/tsdf_volume.h:10-19).
template <class Voxel>
constexpr bool voxel_layout_matches() {
  return sizeof(Voxel) == sizeof(cf_tsdf_voxel) && offsetof(Voxel, tsdf) == offsetof(cf_tsdf_voxel, tsdf) &&
         offsetof(Voxel, weight) == offsetof(cf_tsdf_voxel, weight) &&
         offsetof(Voxel, color) == offsetof(cf_tsdf_voxel, color);
}

template <class Params>
constexpr bool tsdf_params_layout_matches() {
  return sizeof(Params) == sizeof(cf_tsdf_params) && offsetof(Params, dims) == offsetof(cf_tsdf_params, dims) &&
         offsetof(Params, voxel_size) == offsetof(cf_tsdf_params, voxel_size) &&
         offsetof(Params, truncation) == offsetof(cf_tsdf_params, truncation) &&
         offsetof(Params, origin) == offsetof(cf_tsdf_params, origin) &&
         offsetof(Params, decay_alpha) == offsetof(cf_tsdf_params, decay_alpha) &&
         offsetof(Params, max_weight) == offsetof(cf_tsdf_params, max_weight);
}

class GaussNewtonSolver {
 public:
  // GaussNewtonSolver::Params, include/solver.h:13-22 (same fields and defaults)
  struct Params {
    int gn_iterations = 3;
    int pcg_iterations = 10;
    float pcg_tolerance = 1e-4f;
    float lambda_smooth = 1.0f;
    float lambda_rot = 1.0f;
    float lambda_damping = 1e-2f;
    bool debug = false;
  };

  // include/solver.h:24.  max_corrs bounds num_corrs of later solves.
  explicit GaussNewtonSolver(const Params& p, int max_nodes, int max_corrs = 1 << 20) : params_(p) {
    cf_gn_params cp = to_c(p);
    check(cf_gn_create(&cp, max_nodes, max_corrs, &h_), "GaussNewtonSolver");
  }
  ~GaussNewtonSolver() {
    if (h_) cf_gn_destroy(h_);
  }
  GaussNewtonSolver(const GaussNewtonSolver&) = delete;
  GaussNewtonSolver& operator=(const GaussNewtonSolver&) = delete;

  // include/solver.h:29-35: one linearisation -> delta_x [6*num_nodes].
  template <class CorrArray, class Node, class DQ, class FloatArray>
  void solve(const CorrArray& corrs, int num_corrs, const Node* d_nodes, const DQ* d_transforms, int num_nodes,
             FloatArray& delta_x) {
    using Corr = typename std::remove_pointer<decltype(corrs.data)>::type;
    static_assert(layouts_match<Node, DQ, Corr>(), "struct layouts differ from include/types.h");
    delta_x.allocate((size_t)num_nodes * 6);
    check(cf_gn_linearize_solve(h_, reinterpret_cast<const cf_correspondence*>(corrs.data), num_corrs,
                                reinterpret_cast<const cf_deform_node*>(d_nodes),
                                reinterpret_cast<const cf_dual_quat*>(d_transforms), num_nodes,
                                reinterpret_cast<float*>(delta_x.data), nullptr),
          "GaussNewtonSolver::solve");
    check(cf_gn_check(h_, nullptr), "GaussNewtonSolver::solve");
  }

  // Host copies of the assembled system (system_matrix() / rhs(),
  // include/solver.h:38-39, which return device BSR storage in the reference).
  void system_matrix(std::vector<int>& row_ptr, std::vector<int>& col_idx, std::vector<float>& values) {
    int n = 0, nb = 0;
    check(cf_gn_get_system(h_, &n, &nb, nullptr, nullptr, nullptr, nullptr, nullptr), "system_matrix");
    row_ptr.resize(n + 1);
    col_idx.resize(nb);
    values.resize((size_t)nb * 36);
    check(cf_gn_get_system(h_, &n, &nb, row_ptr.data(), col_idx.data(), values.data(), nullptr, nullptr),
          "system_matrix");
  }
  void rhs(std::vector<float>& b) {
    int n = 0, nb = 0;
    check(cf_gn_get_system(h_, &n, &nb, nullptr, nullptr, nullptr, nullptr, nullptr), "rhs");
    b.resize((size_t)n * 6);
    check(cf_gn_get_system(h_, &n, &nb, nullptr, nullptr, nullptr, b.data(), nullptr), "rhs");
  }

  // G full GN iterations with re-skinning from canonical points (no
  // reference counterpart: the reference runs this loop on the host around
  // solve(), include/fusion_app.h:256-646).
  template <class Node, class Corr, class DQ>
  cf_solve_stats solve_frame(const Node* d_nodes, int num_nodes, const float* d_canon, const Corr* d_corrs,
                             int num_corrs, DQ* d_transforms, float max_rot, float max_trans,
                             float update_scale = 1.0f) {
    static_assert(layouts_match<Node, DQ, Corr>(), "struct layouts differ from include/types.h");
    cf_problem pr;
    pr.nodes = reinterpret_cast<const cf_deform_node*>(d_nodes);
    pr.num_nodes = num_nodes;
    pr.canon_points = d_canon;
    pr.corrs = reinterpret_cast<const cf_correspondence*>(d_corrs);
    pr.num_corrs = num_corrs;
    pr.max_rot = max_rot;
    pr.max_trans = max_trans;
    pr.update_scale = update_scale;
    cf_solve_stats st;
    check(cf_gn_solve(h_, &pr, reinterpret_cast<cf_dual_quat*>(d_transforms), &st, nullptr), "solve_frame");
    return st;
  }

  cf_gn* handle() { return h_; }
  const Params& params() const { return params_; }

 private:
  static cf_gn_params to_c(const Params& p) {
    cf_gn_params c;
    c.gn_iterations = p.gn_iterations;
    c.pcg_iterations = p.pcg_iterations;
    c.pcg_tolerance = p.pcg_tolerance;
    c.lambda_smooth = p.lambda_smooth;
    c.lambda_rot = p.lambda_rot;
    c.lambda_damping = p.lambda_damping;
    c.debug = p.debug ? 1 : 0;
    return c;
  }
  Params params_;
  cf_gn* h_ = nullptr;
};

// The solve-path part of WarpField: node storage, transforms with
// save/restore, the twist update, and the voxel kNN field.  Graph
// construction (add_nodes_*, prune_nodes) stays with the reference.  Node
// and DQ are the caller's DeformNode / DualQuat types.
template <class Node, class DQ>
class WarpField {
 public:
  static constexpr int MAX_NODES = CF_MAX_NODES_DEFAULT;  // include/warp_field.h:14

  explicit WarpField(float node_radius, int max_nodes = MAX_NODES) : node_radius_(node_radius), max_nodes_(max_nodes) {
    static_assert(node_layout_matches<Node>() && dq_layout_matches<DQ>(), "DeformNode / DualQuat layouts");
    check_cuda(cudaMalloc(&d_nodes_, sizeof(Node) * max_nodes), "WarpField");
    check_cuda(cudaMalloc(&d_T_, sizeof(DQ) * max_nodes), "WarpField");
    check_cuda(cudaMalloc(&d_Tprev_, sizeof(DQ) * max_nodes), "WarpField");
  }
  ~WarpField() {
    cudaFree(d_nodes_);
    cudaFree(d_T_);
    cudaFree(d_Tprev_);
  }
  WarpField(const WarpField&) = delete;
  WarpField& operator=(const WarpField&) = delete;

  int num_nodes() const { return n_; }
  Node* device_nodes() { return d_nodes_; }
  DQ* device_transforms() { return d_T_; }
  DQ* device_transforms_prev() { return d_Tprev_; }
  const Node* device_nodes() const { return d_nodes_; }
  const DQ* device_transforms() const { return d_T_; }

  // src/warp_field.cu:1160-1177: identity transforms when the count changes
  void upload_nodes(const std::vector<Node>& nodes) {
    const int n = (int)std::min<size_t>(nodes.size(), (size_t)max_nodes_);
    h_nodes_.assign(nodes.begin(), nodes.begin() + n);
    check_cuda(cudaMemcpy(d_nodes_, h_nodes_.data(), sizeof(Node) * n, cudaMemcpyHostToDevice), "upload_nodes");
    if ((int)h_T_.size() != n) {
      h_T_.assign(n, identity());
      check_cuda(cudaMemcpy(d_T_, h_T_.data(), sizeof(DQ) * n, cudaMemcpyHostToDevice), "upload_nodes");
      check_cuda(cudaMemcpy(d_Tprev_, h_T_.data(), sizeof(DQ) * n, cudaMemcpyHostToDevice), "upload_nodes");
    }
    n_ = n;
  }
  // src/warp_field.cu:1179-1192
  void upload_transforms(const std::vector<DQ>& T) {
    int n = (int)std::min<size_t>(T.size(), (size_t)max_nodes_);
    if (n_ == 0) n_ = n;
    n = std::min(n, n_);
    h_T_.assign(T.begin(), T.begin() + n);
    check_cuda(cudaMemcpy(d_T_, h_T_.data(), sizeof(DQ) * n, cudaMemcpyHostToDevice), "upload_transforms");
    check_cuda(cudaMemcpy(d_Tprev_, h_T_.data(), sizeof(DQ) * n, cudaMemcpyHostToDevice), "upload_transforms");
  }
  std::vector<Node> download_nodes() const { return h_nodes_; }
  std::vector<DQ> download_transforms() const { return h_T_; }

  // src/warp_field.cu:1106-1119
  void save_transforms() {
    check_cuda(cudaMemcpy(d_Tprev_, d_T_, sizeof(DQ) * n_, cudaMemcpyDeviceToDevice), "save_transforms");
  }
  void restore_transforms() {
    check_cuda(cudaMemcpy(d_T_, d_Tprev_, sizeof(DQ) * n_, cudaMemcpyDeviceToDevice), "restore_transforms");
    h_T_.resize(n_);
    check_cuda(cudaMemcpy(h_T_.data(), d_T_, sizeof(DQ) * n_, cudaMemcpyDeviceToHost), "restore_transforms");
  }
  // src/warp_field.cu:1143-1148
  void reset_transforms() {
    h_T_.assign(n_, identity());
    check_cuda(cudaMemcpy(d_T_, h_T_.data(), sizeof(DQ) * n_, cudaMemcpyHostToDevice), "reset_transforms");
  }
  // src/warp_field.cu:1121-1141: T_i <- exp(clamp(scale * dx_i)) * T_i, then the host mirror
  template <class FloatArray>
  void apply_twist_increment(const FloatArray& delta_x, float max_rot, float max_trans, float update_scale = 1.0f) {
    if (n_ == 0) return;
    check(cf_warp_apply_twist(reinterpret_cast<cf_dual_quat*>(d_T_), reinterpret_cast<const float*>(delta_x.data),
                              n_, max_rot, max_trans, update_scale, nullptr),
          "apply_twist_increment");
    check_cuda(cudaDeviceSynchronize(), "apply_twist_increment");
    h_T_.resize(n_);
    check_cuda(cudaMemcpy(h_T_.data(), d_T_, sizeof(DQ) * n_, cudaMemcpyDeviceToHost), "apply_twist_increment");
  }

  // include/warp_field.h:72-74, src/warp_field.cu:957-981: the voxel kNN
  // field of `volume` (the reference's TSDFVolume: params() with dims,
  // origin and voxel_size, device_data() of 12-byte voxels) over this
  // field's nodes.  Like the reference: nothing happens without nodes, the
  // two arrays are (re)allocated to 4 entries per voxel, and the call
  // synchronises.
  template <class Volume, class IntArray, class FloatArray>
  void compute_voxel_knn(const Volume& volume, IntArray& d_voxel_knn, FloatArray& d_voxel_knn_w) {
    using Voxel = typename std::remove_cv<typename std::remove_pointer<decltype(volume.device_data())>::type>::type;
    static_assert(voxel_layout_matches<Voxel>(), "TSDFVoxel layout");
    if (n_ == 0) return;
    const auto& p = volume.params();
    const size_t total = (size_t)p.dims.x * (size_t)p.dims.y * (size_t)p.dims.z;
    d_voxel_knn.allocate(total * CF_K_NEIGHBORS);
    d_voxel_knn_w.allocate(total * CF_K_NEIGHBORS);
    cf_tsdf_params cp{};
    cp.dims[0] = p.dims.x;
    cp.dims[1] = p.dims.y;
    cp.dims[2] = p.dims.z;
    cp.voxel_size = p.voxel_size;
    cp.origin[0] = p.origin.x;
    cp.origin[1] = p.origin.y;
    cp.origin[2] = p.origin.z;
    check(cf_compute_voxel_knn(reinterpret_cast<const cf_tsdf_voxel*>(volume.device_data()), &cp,
                               reinterpret_cast<const cf_deform_node*>(d_nodes_), n_,
                               reinterpret_cast<int*>(d_voxel_knn.data), reinterpret_cast<float*>(d_voxel_knn_w.data),
                               nullptr),
          "WarpField::compute_voxel_knn");
    check_cuda(cudaDeviceSynchronize(), "WarpField::compute_voxel_knn");
  }

  float node_radius() const { return node_radius_; }

 private:
  static DQ identity() {
    cf_dual_quat d = {{0.f, 0.f, 0.f, 1.f}, {0.f, 0.f, 0.f, 0.f}};
    DQ out;
    static_assert(sizeof(out) == sizeof(d), "layout");
    std::memcpy(&out, &d, sizeof(d));
    return out;
  }
  static void check_cuda(cudaError_t e, const char* where) {
    if (e != cudaSuccess) check(CF_ERR_CUDA, where);
  }
  float node_radius_;
  int max_nodes_;
  int n_ = 0;
  Node* d_nodes_ = nullptr;
  DQ* d_T_ = nullptr;
  DQ* d_Tprev_ = nullptr;
  std::vector<Node> h_nodes_;
  std::vector<DQ> h_T_;
};

// The projective correspondence search on the pipeline's own buffers.  Cam,
// M4 and Corr are the caller's CameraIntrinsics, Mat4 and Correspondence.
class CorrespondenceSearch {
 public:
  CorrespondenceSearch(int max_width, int max_height) {
    check(cf_corr_search_create(max_width, max_height, &h_), "CorrespondenceSearch");
  }
  ~CorrespondenceSearch() { cf_corr_search_destroy(h_); }
  CorrespondenceSearch(const CorrespondenceSearch&) = delete;
  CorrespondenceSearch& operator=(const CorrespondenceSearch&) = delete;

  // find_correspondences: searches, synchronises and returns the valid count
  // (d_stats, when given, receives the six debug counters).
  template <class Cam, class M4, class Corr>
  int find_correspondences(const cf_corr_frame& frame, const Cam& cam, const M4& T_cam_world, const M4& T_world_cam,
                           const cf_corr_params& params, Corr* d_corrs, int* d_num_valid, int* d_stats = nullptr) {
    static_assert(camera_layout_matches<Cam>() && mat4_layout_matches<M4>() && corr_layout_matches<Corr>(),
                  "CameraIntrinsics / Mat4 / Correspondence layouts");
    check(cf_find_correspondences(h_, &frame, reinterpret_cast<const cf_camera*>(&cam),
                                  reinterpret_cast<const cf_mat4*>(&T_cam_world),
                                  reinterpret_cast<const cf_mat4*>(&T_world_cam), &params,
                                  reinterpret_cast<cf_correspondence*>(d_corrs), d_num_valid, d_stats, nullptr),
          "find_correspondences");
    int n = 0;
    check_cuda(cudaMemcpy(&n, d_num_valid, sizeof(int), cudaMemcpyDeviceToHost), "find_correspondences");
    return n;
  }
  cf_corr_search* handle() { return h_; }

 private:
  static void check_cuda(cudaError_t e, const char* where) {
    if (e != cudaSuccess) check(CF_ERR_CUDA, where);
  }
  cf_corr_search* h_ = nullptr;
};

// The live-surface prediction: mesh skinning, rasterisation and resolve into
// the pipeline's live maps.  Node / DQ / Cam / M4 are the caller's
// DeformNode, DualQuat, CameraIntrinsics and Mat4; vertices are float3.
class LiveSurfaceRaster {
 public:
  LiveSurfaceRaster(int max_width, int max_height) {
    check(cf_raster_create(max_width, max_height, &h_), "LiveSurfaceRaster");
  }
  ~LiveSurfaceRaster() { cf_raster_destroy(h_); }
  LiveSurfaceRaster(const LiveSurfaceRaster&) = delete;
  LiveSurfaceRaster& operator=(const LiveSurfaceRaster&) = delete;

  // rasterize_deformed_mesh_live_surface after the mesh is extracted;
  // synchronises, as the reference does.
  template <class V3, class I3, class Node, class DQ, class Cam, class M4>
  void predict(const V3* d_canonical, V3* d_warped, const I3* d_triangles, int num_vertices, int num_triangles,
               const Node* d_nodes, const DQ* d_transforms, int num_nodes, const int* d_voxel_knn,
               const float* d_voxel_knn_w, const Cam& cam, const M4& T_cam_world, const cf_voxel_grid& grid,
               V3* d_live_vertices, V3* d_live_normals, int* d_hit_voxel_idx) {
    static_assert(sizeof(V3) == 3 * sizeof(float) && sizeof(I3) == 3 * sizeof(int), "float3 / int3");
    static_assert(node_layout_matches<Node>() && dq_layout_matches<DQ>() && camera_layout_matches<Cam>() &&
                      mat4_layout_matches<M4>(),
                  "DeformNode / DualQuat / CameraIntrinsics / Mat4 layouts");
    check(cf_predict_live_surface(h_, reinterpret_cast<const float*>(d_canonical), reinterpret_cast<float*>(d_warped),
                                  reinterpret_cast<const int*>(d_triangles), num_vertices, num_triangles,
                                  reinterpret_cast<const cf_deform_node*>(d_nodes),
                                  reinterpret_cast<const cf_dual_quat*>(d_transforms), num_nodes, d_voxel_knn,
                                  d_voxel_knn_w, reinterpret_cast<const cf_camera*>(&cam),
                                  reinterpret_cast<const cf_mat4*>(&T_cam_world), &grid,
                                  reinterpret_cast<float*>(d_live_vertices), reinterpret_cast<float*>(d_live_normals),
                                  d_hit_voxel_idx, nullptr),
          "rasterize_deformed_mesh_live_surface");
    if (cudaDeviceSynchronize() != cudaSuccess) check(CF_ERR_CUDA, "rasterize_deformed_mesh_live_surface");
  }
  cf_raster* handle() { return h_; }

 private:
  cf_raster* h_ = nullptr;
};

// TSDFVolume::integrate (src/tsdf_volume.cu:23-60) over a volume the caller
// owns (TSDFVolume::device_data(), the reference's 12-byte TSDFVoxel), and
// DynamicFusionPipeline::mark_optimized_voxels (include/fusion_app.h:1321-1328).
// Holds the per-node scratch of up to max_nodes dual quaternions; synchronises,
// as the reference does.
class TSDFIntegrator {
 public:
  explicit TSDFIntegrator(int max_nodes) : cap_(max_nodes) {
    if (max_nodes < 0) check(CF_ERR_INVALID_ARG, "TSDFIntegrator");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
      cudaGetLastError();
      check(CF_ERR_NO_DEVICE, "TSDFIntegrator");
    }
    if (cap_ > 0 && cudaMalloc(&plain_, sizeof(cf_dual_quat) * (size_t)cap_) != cudaSuccess) {
      cudaGetLastError();
      check(CF_ERR_OOM, "TSDFIntegrator");
    }
  }
  ~TSDFIntegrator() { cudaFree(plain_); }
  TSDFIntegrator(const TSDFIntegrator&) = delete;
  TSDFIntegrator& operator=(const TSDFIntegrator&) = delete;

  // Params = TSDFVolume::Params (include/tsdf_volume.h:10-19); nodes == nullptr
  // or num_nodes == 0 integrates rigidly.
  template <class Voxel, class Params, class Cam, class M4, class Node = cf_deform_node, class DQ = cf_dual_quat>
  void integrate(Voxel* d_voxels, const Params& params, const float* d_depth, const Cam& cam, const M4& camera_pose,
                 const Node* d_nodes = nullptr, const DQ* d_transforms = nullptr, int num_nodes = 0,
                 const int* d_voxel_knn = nullptr, const float* d_voxel_knn_w = nullptr,
                 const int* d_voxel_opt_counts = nullptr, int min_opt_count = 0) {
    static_assert(voxel_layout_matches<Voxel>() && tsdf_params_layout_matches<Params>(),
                  "TSDFVoxel / TSDFVolume::Params layouts");
    static_assert(node_layout_matches<Node>() && dq_layout_matches<DQ>() && camera_layout_matches<Cam>() &&
                      mat4_layout_matches<M4>(),
                  "DeformNode / DualQuat / CameraIntrinsics / Mat4 layouts");
    if (d_nodes && num_nodes > cap_) check(CF_ERR_CAPACITY, "TSDFVolume::integrate");
    check(cf_tsdf_integrate(reinterpret_cast<cf_tsdf_voxel*>(d_voxels),
                            reinterpret_cast<const cf_tsdf_params*>(&params), d_depth,
                            reinterpret_cast<const cf_camera*>(&cam), reinterpret_cast<const cf_mat4*>(&camera_pose),
                            reinterpret_cast<const cf_deform_node*>(d_nodes),
                            reinterpret_cast<const cf_dual_quat*>(d_transforms), num_nodes, d_voxel_knn,
                            d_voxel_knn_w, d_voxel_opt_counts, min_opt_count, plain_, nullptr),
          "TSDFVolume::integrate");
    if (cudaDeviceSynchronize() != cudaSuccess) check(CF_ERR_CUDA, "TSDFVolume::integrate");
  }

  // mark_optimized_voxels_kernel; Dims = int3.
  template <class Corr, class Dims>
  static void mark_optimized_voxels(const Corr* d_corrs, const int* d_canonical_vidx, int num_pixels,
                                    const Dims& dims, int frame_id, int* d_voxel_opt_counts,
                                    int* d_voxel_opt_frame) {
    static_assert(corr_layout_matches<Corr>() && sizeof(Dims) == 3 * sizeof(int),
                  "Correspondence / int3 layouts");
    check(cf_mark_optimized_voxels(reinterpret_cast<const cf_correspondence*>(d_corrs), d_canonical_vidx, num_pixels,
                                   reinterpret_cast<const int*>(&dims), frame_id, d_voxel_opt_counts,
                                   d_voxel_opt_frame, nullptr),
          "mark_optimized_voxels");
    if (cudaDeviceSynchronize() != cudaSuccess) check(CF_ERR_CUDA, "mark_optimized_voxels");
  }

 private:
  int cap_ = 0;
  cf_dual_quat* plain_ = nullptr;
};

}  // namespace cudafusion_b200
