// The correspondence search and the live-surface prediction through the C++
// drop-in classes, with the reference's type layouts (include/types.h:26-60,
// 148-162, 198-206).  Compiled with -Wall -Werror: the templates instantiate
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
struct Correspondence {
  float3 src, dst, normal;
  int node_ids[4];
  float node_ws[4];
  float weight;
  bool valid;
};

// Instantiates both classes' templates (never called without a device).
void frame(cudafusion_b200::CorrespondenceSearch& cs, cudafusion_b200::LiveSurfaceRaster& ras) {
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
    return caught == 2 ? 0 : 1;
  }
  cudafusion_b200::CorrespondenceSearch cs(640, 480);
  cudafusion_b200::LiveSurfaceRaster ras(640, 480);
  (void)frame;
  return 0;
}
