// The C++ drop-in classes instantiated with CUDAFusion's own types, taken
// from the reference's headers themselves (include/types.h: Mat4,
// CameraIntrinsics, DualQuat, DeviceArray<T>, TSDFVoxel, DeformNode,
// Correspondence; include/tsdf_volume.h: TSDFVolume::Params) rather than
// restated.  Compile-only (-c): every layout check of cudafusion_b200.hpp
// (sizes and the byte offset of every field) runs against the reference's
// definitions, and each templated method is instantiated with them.
#include "types.h"
#include "tsdf_volume.h"
#include "cudafusion_b200.hpp"

namespace cf = cudafusion_b200;

static_assert(cf::layouts_match<DeformNode, DualQuat, Correspondence>(),
              "DeformNode / DualQuat / Correspondence layouts");
static_assert(cf::camera_layout_matches<CameraIntrinsics>(), "CameraIntrinsics layout");
static_assert(cf::mat4_layout_matches<Mat4>(), "Mat4 layout");
static_assert(cf::voxel_layout_matches<TSDFVoxel>(), "TSDFVoxel layout");
static_assert(cf::tsdf_params_layout_matches<TSDFVolume::Params>(), "TSDFVolume::Params layout");

// Never called: referencing the methods instantiates them with the
// reference's types, so their own static_asserts are evaluated too.
void instantiate_with_reference_types(cf::GaussNewtonSolver& solver, cf::WarpField<DeformNode, DualQuat>& warp,
                                      cf::CorrespondenceSearch& search, cf::LiveSurfaceRaster& raster,
                                      cf::TSDFIntegrator& tsdf, const DeviceArray<Correspondence>& corrs,
                                      DeviceArray<float>& delta_x, const float3* canon, float3* warped,
                                      const int3* tris, const float* depth, int* ints, float* floats,
                                      TSDFVoxel* voxels, const cf_corr_frame& frame, const cf_corr_params& cprm,
                                      const cf_voxel_grid& grid) {
  CameraIntrinsics cam{};
  Mat4 pose;
  TSDFVolume::Params tp;
  solver.solve(corrs, 0, warp.device_nodes(), warp.device_transforms(), 0, delta_x);
  solver.solve_frame(warp.device_nodes(), 0, floats, corrs.data, 0, warp.device_transforms(), 0.f, 0.f);
  warp.apply_twist_increment(delta_x, 0.f, 0.f);
  search.find_correspondences(frame, cam, pose, pose, cprm, corrs.data, ints);
  raster.predict(canon, warped, tris, 0, 0, warp.device_nodes(), warp.device_transforms(), 0, ints, floats, cam,
                 pose, grid, warped, warped, ints);
  tsdf.integrate(voxels, tp, depth, cam, pose, warp.device_nodes(), warp.device_transforms(), 0, ints, floats, ints,
                 0);
  cf::TSDFIntegrator::mark_optimized_voxels(corrs.data, ints, 0, tp.dims, 0, ints, ints);
}

// WarpField::compute_voxel_knn over the reference's TSDFVolume and DeviceArrays.
void instantiate_voxel_knn(cf::WarpField<DeformNode, DualQuat>& warp, const TSDFVolume& volume,
                           DeviceArray<int>& knn, DeviceArray<float>& knn_w) {
  warp.compute_voxel_knn(volume, knn, knn_w);
}
