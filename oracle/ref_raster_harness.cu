// ref_raster_harness.cu — thin driver of the reference's own live-surface
// prediction, linked with the unmodified src/mesh_raster_kernels.cu and
// src/skinning_kernels.cu (oracle/Makefile target `ref`, built for sm_100a
// with --use_fast_math as the reference ships).  TEST AND REFERENCE-ARM
// INFRASTRUCTURE ONLY: used by the GPU parity tests, by the script that makes
// the golden fixtures and by `bench.py --impl reference --workload raster`.
//
// refr_run does what DynamicFusionPipeline::rasterize_deformed_mesh_live_surface
// does (include/fusion_app.h:1216-1318) once the mesh is extracted: zero the
// live maps, fill the hit voxels with -1, optionally skin the mesh
// (skin_vertices_from_voxel_knn_kernel), fill the depth buffer with ones,
// rasterize_triangles_z_kernel, resolve_rasterized_triangles_kernel,
// synchronise.
#include <cuda_runtime.h>

#include "mesh_raster_kernels.h"
#include "skinning_kernels.h"
#include "types.h"

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

struct RefRaster {
  int W = 0, H = 0, V = 0, NT = 0, N = 0;
  long long G = 0;
  float3 *canon = nullptr, *warped = nullptr, *lv = nullptr, *ln = nullptr;
  int3* tris = nullptr;
  int* hit = nullptr;
  unsigned long long* ztri = nullptr;
  DeformNode* nodes = nullptr;
  DualQuat* T = nullptr;
  int* vk = nullptr;
  float* vw = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};

inline int blocks256(int n) { return (n + 255) / 256; }

}  // namespace

REF_EXPORT void refr_destroy(void* hp) {
  RefRaster* h = (RefRaster*)hp;
  if (!h) return;
  cudaFree(h->canon); cudaFree(h->warped); cudaFree(h->lv); cudaFree(h->ln); cudaFree(h->tris);
  cudaFree(h->hit); cudaFree(h->ztri); cudaFree(h->nodes); cudaFree(h->T); cudaFree(h->vk); cudaFree(h->vw);
  if (h->e0) cudaEventDestroy(h->e0);
  if (h->e1) cudaEventDestroy(h->e1);
  delete h;
}

// Allocates and uploads one mesh frame (host arrays; nodes / T / voxel
// tables may be null when the caller passes warped vertices).
REF_EXPORT void* refr_create(int W, int H, const float* canon, const float* warped, int V, const int* tris, int NT,
                             const DeformNode* nodes, const DualQuat* T, int N, const int* vk, const float* vw,
                             long long G) {
  RefRaster* h = new RefRaster();
  h->W = W; h->H = H; h->V = V; h->NT = NT; h->N = N; h->G = G;
  const size_t P = (size_t)W * H;
  bool ok = cudaMalloc(&h->canon, (size_t)V * sizeof(float3)) == cudaSuccess &&
            cudaMalloc(&h->warped, (size_t)V * sizeof(float3)) == cudaSuccess &&
            cudaMalloc(&h->tris, (size_t)(NT > 0 ? NT : 1) * sizeof(int3)) == cudaSuccess &&
            cudaMalloc(&h->lv, P * sizeof(float3)) == cudaSuccess &&
            cudaMalloc(&h->ln, P * sizeof(float3)) == cudaSuccess &&
            cudaMalloc(&h->hit, P * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&h->ztri, P * sizeof(unsigned long long)) == cudaSuccess &&
            cudaEventCreate(&h->e0) == cudaSuccess && cudaEventCreate(&h->e1) == cudaSuccess;
  ok = ok && cudaMemcpy(h->canon, canon, (size_t)V * sizeof(float3), cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(h->warped, warped, (size_t)V * sizeof(float3), cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok && NT > 0) ok = cudaMemcpy(h->tris, tris, (size_t)NT * sizeof(int3), cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok && N > 0 && nodes && T && vk && vw && G > 0) {
    ok = cudaMalloc(&h->nodes, (size_t)N * sizeof(DeformNode)) == cudaSuccess &&
         cudaMalloc(&h->T, (size_t)N * sizeof(DualQuat)) == cudaSuccess &&
         cudaMalloc(&h->vk, (size_t)G * K_NEIGHBORS * sizeof(int)) == cudaSuccess &&
         cudaMalloc(&h->vw, (size_t)G * K_NEIGHBORS * sizeof(float)) == cudaSuccess &&
         cudaMemcpy(h->nodes, nodes, (size_t)N * sizeof(DeformNode), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->T, T, (size_t)N * sizeof(DualQuat), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->vk, vk, (size_t)G * K_NEIGHBORS * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->vw, vw, (size_t)G * K_NEIGHBORS * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess;
  }
  if (!ok) {
    refr_destroy(h);
    return nullptr;
  }
  return h;
}

// One prediction.  cam = {fx, fy, cx, cy}; T_cw row-major 4x4; grid = {ox,
// oy, oz, voxel_size}; dims[3].  skin != 0 warps the canonical mesh by the
// uploaded graph first (the warped vertices uploaded at create are replaced).
// *ms = device time of the whole sequence (CUDA events).  Returns 0, or -1 on
// a CUDA error.
REF_EXPORT int refr_run(void* hp, const float* cam, const float* T_cw, const float* grid, const int* dims, int skin,
                        float* ms) {
  RefRaster* h = (RefRaster*)hp;
  CameraIntrinsics c;
  c.fx = cam[0]; c.fy = cam[1]; c.cx = cam[2]; c.cy = cam[3];
  c.width = h->W; c.height = h->H;
  Mat4 cw;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) cw.m[i][j] = T_cw[4 * i + j];
  const float3 origin = make_float3(grid[0], grid[1], grid[2]);
  const int3 d3 = make_int3(dims[0], dims[1], dims[2]);
  const size_t P = (size_t)h->W * h->H;
  cudaEventRecord(h->e0);
  cudaMemset(h->lv, 0, P * sizeof(float3));
  cudaMemset(h->ln, 0, P * sizeof(float3));
  cudaMemset(h->hit, 0xff, P * sizeof(int));
  if (skin && h->nodes)
    skin_vertices_from_voxel_knn_kernel<<<blocks256(h->V), 256>>>(h->canon, h->warped, h->V, origin, grid[3], d3,
                                                              h->nodes, h->T, h->N, h->vk, h->vw);
  cudaMemset(h->ztri, 0xff, P * sizeof(unsigned long long));
  if (h->NT > 0) {
    rasterize_triangles_z_kernel<<<blocks256(h->NT), 256>>>(h->canon, h->warped, h->tris, h->V, h->NT, c, cw, h->ztri);
    resolve_rasterized_triangles_kernel<<<blocks256((int)P), 256>>>(h->canon, h->warped, h->tris, h->V, c, cw, origin,
                                                                 grid[3], d3, h->ztri, h->lv, h->ln, h->hit);
  }
  cudaEventRecord(h->e1);
  if (cudaDeviceSynchronize() != cudaSuccess) return -1;
  if (ms) cudaEventElapsedTime(ms, h->e0, h->e1);
  return 0;
}

// Copies the last run's maps and the warped vertices (any pointer may be null).
REF_EXPORT int refr_download(void* hp, float* lv, float* ln, int* hit, float* warped, unsigned long long* ztri) {
  RefRaster* h = (RefRaster*)hp;
  const size_t P = (size_t)h->W * h->H;
  bool ok = true;
  if (lv) ok = ok && cudaMemcpy(lv, h->lv, P * sizeof(float3), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (ln) ok = ok && cudaMemcpy(ln, h->ln, P * sizeof(float3), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (hit) ok = ok && cudaMemcpy(hit, h->hit, P * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (warped) ok = ok && cudaMemcpy(warped, h->warped, (size_t)h->V * sizeof(float3), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (ztri) ok = ok && cudaMemcpy(ztri, h->ztri, P * sizeof(unsigned long long), cudaMemcpyDeviceToHost) == cudaSuccess;
  return ok ? 0 : -1;
}
