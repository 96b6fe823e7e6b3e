// The correspondence search, the live-surface prediction and the TSDF
// integration through the C++ drop-in classes, with the reference's type
// layouts (include/types.h:26-60, 148-176, 198-206, include/tsdf_volume.h:10-19).  Compiled with -Wall -Werror: the templates instantiate
// against these types.
//
// usage: dropin_frontend nodev   (no GPU: the constructors must throw
//                                 CF_ERR_NO_DEVICE, not fall back)
#include <cstdio>
#include <string>

#include "cudafusion_b200.hpp"

struct CameraIntrinsics {
  float fx, fy, cx, cy;
  int width, height;
};
struct Mat4 {
  float m[4][4];
};
struct DualQuat {
  float4 real;
  float4 dual;
};
struct DeformNode {
  float3 pos;
  float3 normal;
  float radius;
  int neighbors[8];
  float neighbor_w[8];
  int num_neighbors;
};
struct TSDFVoxel {
  float tsdf;
  float weight;
  uchar3 color;
  uint8_t pad;
};
struct TSDFParams {
  int3 dims;
  float voxel_size;
  float truncation;
  float3 origin;
  float decay_alpha;
  float max_weight;
};
struct Correspondence {
  float3 src, dst, normal;
  int node_ids[4];
  float node_ws[4];
  float weight;
  bool valid;
};

// Instantiates the classes' templates (never called without a device).
void frame(cudafusion_b200::CorrespondenceSearch& cs, cudafusion_b200::LiveSurfaceRaster& ras,
           cudafusion_b200::TSDFIntegrator& tsdf) {
  CameraIntrinsics cam = {570.342f, 570.342f, 320.f, 240.f, 640, 480};
  Mat4 I = {{{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}}};
  cf_voxel_grid g = {{0.f, 0.f, 0.f}, 0.004f, {64, 64, 64}};
  float3 *v = nullptr, *lv = nullptr, *ln = nullptr;
  int3* t = nullptr;
  int* hit = nullptr;
  DeformNode* nodes = nullptr;
  DualQuat* T = nullptr;
  ras.predict(v, v, t, 0, 0, nodes, T, 0, nullptr, nullptr, cam, I, g, lv, ln, hit);
  cf_corr_frame f = {};
  cf_corr_params p = {0.2f, 0.f, 0.f, 50};
  Correspondence* corrs = nullptr;
  int* nv = nullptr;
  std::printf("valid %d\n", cs.find_correspondences(f, cam, I, I, p, corrs, nv));
  TSDFVoxel* vox = nullptr;
  TSDFParams tp = {{256, 256, 256}, 0.006f, 0.03f, {-0.768f, -0.768f, 0.5f}, 0.9f, 50.f};
  const float* depth = nullptr;
  tsdf.integrate(vox, tp, depth, cam, I);
  tsdf.integrate(vox, tp, depth, cam, I, nodes, T, 0, hit, nullptr, hit, 3);
  cudafusion_b200::TSDFIntegrator::mark_optimized_voxels(corrs, hit, 0, tp.dims, 1, hit, hit);
}

int main(int argc, char** argv) {
  if (argc >= 2 && std::string(argv[1]) == "nodev") {
    int caught = 0;
    try {
      cudafusion_b200::CorrespondenceSearch cs(640, 480);
    } catch (const cudafusion_b200::Error& e) {
      caught += e.status == CF_ERR_NO_DEVICE;
      std::printf("CorrespondenceSearch: status %d (%s)\n", (int)e.status, e.what());
    }
    try {
      cudafusion_b200::LiveSurfaceRaster ras(640, 480);
    } catch (const cudafusion_b200::Error& e) {
      caught += e.status == CF_ERR_NO_DEVICE;
      std::printf("LiveSurfaceRaster: status %d (%s)\n", (int)e.status, e.what());
    }
    try {
      cudafusion_b200::TSDFIntegrator tsdf(2048);
    } catch (const cudafusion_b200::Error& e) {
      caught += e.status == CF_ERR_NO_DEVICE;
      std::printf("TSDFIntegrator: status %d (%s)\n", (int)e.status, e.what());
    }
    return caught == 3 ? 0 : 1;
  }
  cudafusion_b200::CorrespondenceSearch cs(640, 480);
  cudafusion_b200::LiveSurfaceRaster ras(640, 480);
  cudafusion_b200::TSDFIntegrator tsdf(2048);
  (void)frame;
  return 0;
}
