// ref_tsdf_harness.cu — thin driver of the reference's own TSDF integration,
// linked with the unmodified src/tsdf_volume.cu and kernels/tsdf_kernels.cu
// (oracle/Makefile target `ref`, built for sm_100a with --use_fast_math as
// the reference ships).  TEST INFRASTRUCTURE ONLY: used by the script that
// makes the golden fixtures and by the GPU parity tests.
//
// reft_upload keeps one frame's inputs on the device; reft_integrate calls
// TSDFVolume::integrate (src/tsdf_volume.cu:23-60), the reference's public
// entry, on a volume whose voxels the caller uploaded; reft_mark launches
// mark_optimized_voxels_kernel as DynamicFusionPipeline::mark_optimized_voxels
// does (include/fusion_app.h:1321-1328).
#include <cuda_runtime.h>

#include "tsdf_kernels.h"
#include "tsdf_volume.h"
#include "types.h"

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

namespace {
struct RefTsdf {
  TSDFVolume* vol = nullptr;
  long long V = 0;
  int W = 0, H = 0, N = 0;
  DeviceArray<float> depth;
  DeviceArray<float3> normals;
  DeformNode* dn = nullptr;
  DualQuat* dT = nullptr;
  int* dk = nullptr;
  float* dw = nullptr;
  int* dc = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};
template <typename T>
bool up(T** d, const void* h, size_t n) {
  if (cudaMalloc(d, n * sizeof(T)) != cudaSuccess) return false;
  return cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
}
}  // namespace

// dims[3], origin[3]; the TSDFVolume constructor initialises the voxels.
REF_EXPORT void* reft_create(const int* dims, float voxel_size, float truncation, const float* origin, float decay,
                             float max_weight) {
  TSDFVolume::Params p;
  p.dims = make_int3(dims[0], dims[1], dims[2]);
  p.voxel_size = voxel_size;
  p.truncation = truncation;
  p.origin = make_float3(origin[0], origin[1], origin[2]);
  p.decay_alpha = decay;
  p.max_weight = max_weight;
  RefTsdf* h = new RefTsdf();
  h->vol = new TSDFVolume(p);
  h->V = (long long)dims[0] * dims[1] * dims[2];
  cudaEventCreate(&h->e0);
  cudaEventCreate(&h->e1);
  return h;
}

REF_EXPORT void reft_destroy(void* hp) {
  RefTsdf* h = (RefTsdf*)hp;
  if (!h) return;
  cudaFree(h->dn); cudaFree(h->dT); cudaFree(h->dk); cudaFree(h->dw); cudaFree(h->dc);
  if (h->e0) cudaEventDestroy(h->e0);
  if (h->e1) cudaEventDestroy(h->e1);
  delete h->vol;
  delete h;
}

// The voxels as 12-byte records (tsdf, weight, colour bytes).
REF_EXPORT int reft_set_voxels(void* hp, const void* vox) {
  RefTsdf* h = (RefTsdf*)hp;
  return cudaMemcpy(h->vol->device_data(), vox, (size_t)h->V * sizeof(TSDFVoxel), cudaMemcpyHostToDevice) ==
                 cudaSuccess ? 0 : -1;
}
REF_EXPORT int reft_get_voxels(void* hp, void* vox) {
  RefTsdf* h = (RefTsdf*)hp;
  return cudaMemcpy(vox, h->vol->device_data(), (size_t)h->V * sizeof(TSDFVoxel), cudaMemcpyDeviceToHost) ==
                 cudaSuccess ? 0 : -1;
}

// Uploads one frame's inputs, kept on the device until the next upload:
// depth (W x H); N == 0 integrates rigidly; counts may be null.  Returns 0,
// or -1 on a CUDA error.
REF_EXPORT int reft_upload(void* hp, const float* depth, int W, int H, const DeformNode* nodes, const DualQuat* T,
                           int N, const int* vk, const float* vw, const int* counts) {
  RefTsdf* h = (RefTsdf*)hp;
  cudaFree(h->dn); cudaFree(h->dT); cudaFree(h->dk); cudaFree(h->dw); cudaFree(h->dc);
  h->dn = nullptr; h->dT = nullptr; h->dk = nullptr; h->dw = nullptr; h->dc = nullptr;
  h->W = W; h->H = H; h->N = N;
  h->depth.allocate((size_t)W * H);
  h->normals.allocate((size_t)W * H);
  bool ok = cudaMemcpy(h->depth.data, depth, (size_t)W * H * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok && N > 0) {
    ok = up(&h->dn, nodes, N) && up(&h->dT, T, N) && up(&h->dk, vk, (size_t)h->V * K_NEIGHBORS) &&
         up(&h->dw, vw, (size_t)h->V * K_NEIGHBORS);
    if (ok && counts) ok = up(&h->dc, counts, (size_t)h->V);
  }
  return ok ? 0 : -1;
}

// One TSDFVolume::integrate on the uploaded frame: cam = {fx, fy, cx, cy},
// pose row-major 4x4 (camera -> world).  *ms = its device time (CUDA
// events around the call, which synchronises).  Returns 0, or -1 on a CUDA
// error.
REF_EXPORT int reft_integrate(void* hp, const float* cam, const float* pose, int min_opt, float* ms) {
  RefTsdf* h = (RefTsdf*)hp;
  CameraIntrinsics c;
  c.fx = cam[0]; c.fy = cam[1]; c.cx = cam[2]; c.cy = cam[3];
  c.width = h->W; c.height = h->H;
  Mat4 m;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) m.m[i][j] = pose[4 * i + j];
  cudaEventRecord(h->e0);
  h->vol->integrate(h->depth, h->normals, c, m, h->dn, h->dT, h->N, h->dk, h->dw, h->dc, min_opt);
  cudaEventRecord(h->e1);
  if (cudaDeviceSynchronize() != cudaSuccess) return -1;
  if (ms) cudaEventElapsedTime(ms, h->e0, h->e1);
  return 0;
}

// mark_optimized_voxels_kernel on host arrays: corrs (P records), vidx (P),
// counts / frames (V, updated in place).
REF_EXPORT int reft_mark(const Correspondence* corrs, const int* vidx, int P, const int* dims, int frame, int* counts,
                         int* frames) {
  const long long V = (long long)dims[0] * dims[1] * dims[2];
  Correspondence* dc = nullptr;
  int *dv = nullptr, *dn = nullptr, *df = nullptr;
  bool ok = up(&dc, corrs, P) && up(&dv, vidx, P) && up(&dn, counts, V) && up(&df, frames, V);
  if (ok) {
    mark_optimized_voxels_kernel<<<(P + 255) / 256, 256>>>(dc, dv, P, make_int3(dims[0], dims[1], dims[2]), frame,
                                                           dn, df);
    ok = cudaDeviceSynchronize() == cudaSuccess &&
         cudaMemcpy(counts, dn, V * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(frames, df, V * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess;
  }
  cudaFree(dc); cudaFree(dv); cudaFree(dn); cudaFree(df);
  return ok ? 0 : -1;
}
