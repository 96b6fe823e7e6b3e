// ref_voxelknn_harness.cu — thin driver of the reference's own voxel kNN
// field, linked with the unmodified src/warp_field.cu, src/tsdf_volume.cu and
// kernels/tsdf_kernels.cu (oracle/Makefile target `ref`, built for sm_100a with
// --use_fast_math as the reference ships).  TEST AND REFERENCE-ARM
// INFRASTRUCTURE ONLY: used by the script that makes the golden fixture, by the
// GPU parity tests and by `bench.py --impl reference --workload voxelknn`.
//
// refk_compute calls WarpField::compute_voxel_knn (src/warp_field.cu:957-981),
// the reference's public entry, on a TSDFVolume whose voxels the caller
// uploaded and a WarpField holding the caller's nodes; it launches
// compute_voxel_knn_kernel (:299-405) on 8x8 blocks and synchronises.
#include <cuda_runtime.h>

#include <vector>

#include "tsdf_volume.h"
#include "types.h"
#include "warp_field.h"

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

// src/warp_field.cu:299 (external linkage there; launched here by its host stub)
__global__ void compute_voxel_knn_kernel(const TSDFVoxel* voxels, int3 dims, float3 origin, float voxel_size,
                                         const DeformNode* nodes, int num_nodes, int* knn_ids, float* knn_ws);

namespace {
struct RefKnn {
  TSDFVolume* vol = nullptr;
  WarpField* warp = nullptr;
  long long V = 0;
  DeviceArray<int> knn;
  DeviceArray<float> knn_w;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};
}  // namespace

// dims[3], origin[3]; the TSDFVolume constructor initialises the voxels.
REF_EXPORT void* refk_create(const int* dims, float voxel_size, const float* origin, int max_nodes) {
  TSDFVolume::Params p;
  p.dims = make_int3(dims[0], dims[1], dims[2]);
  p.voxel_size = voxel_size;
  p.origin = make_float3(origin[0], origin[1], origin[2]);
  RefKnn* h = new RefKnn();
  h->vol = new TSDFVolume(p);
  h->warp = new WarpField(0.02f, max_nodes);
  h->V = (long long)dims[0] * dims[1] * dims[2];
  cudaEventCreate(&h->e0);
  cudaEventCreate(&h->e1);
  return h;
}

REF_EXPORT void refk_destroy(void* hp) {
  RefKnn* h = (RefKnn*)hp;
  if (!h) return;
  if (h->e0) cudaEventDestroy(h->e0);
  if (h->e1) cudaEventDestroy(h->e1);
  delete h->warp;
  delete h->vol;
  delete h;
}

// The voxels as 12-byte records (tsdf, weight, colour bytes).
REF_EXPORT int refk_set_voxels(void* hp, const void* vox) {
  RefKnn* h = (RefKnn*)hp;
  return cudaMemcpy(h->vol->device_data(), vox, (size_t)h->V * sizeof(TSDFVoxel), cudaMemcpyHostToDevice) ==
                 cudaSuccess ? 0 : -1;
}

// WarpField::upload_nodes (the reference's own node upload).
REF_EXPORT int refk_set_nodes(void* hp, const DeformNode* nodes, int n) {
  RefKnn* h = (RefKnn*)hp;
  h->warp->upload_nodes(std::vector<DeformNode>(nodes, nodes + n));
  return (int)cudaDeviceSynchronize();
}

// One WarpField::compute_voxel_knn; *ms = its time by CUDA events on the
// legacy stream (the call allocates its outputs and synchronises); the field
// is copied to ids / ws (V * 4 each) when they are not null.
REF_EXPORT int refk_compute(void* hp, int* ids, float* ws, float* ms) {
  RefKnn* h = (RefKnn*)hp;
  cudaEventRecord(h->e0, 0);
  h->warp->compute_voxel_knn(*h->vol, h->knn, h->knn_w);
  cudaEventRecord(h->e1, 0);
  cudaEventSynchronize(h->e1);
  if (ms) cudaEventElapsedTime(ms, h->e0, h->e1);
  if (ids && cudaMemcpy(ids, h->knn.data, sizeof(int) * 4 * (size_t)h->V, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  if (ws && cudaMemcpy(ws, h->knn_w.data, sizeof(float) * 4 * (size_t)h->V, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  return (int)cudaGetLastError();
}

// The kernel alone, as WarpField::compute_voxel_knn launches it (8x8 blocks,
// one z slice per grid layer), into the outputs of the last refk_compute:
// *ms by CUDA events around the launch on the legacy stream.
REF_EXPORT int refk_kernel(void* hp, float* ms) {
  RefKnn* h = (RefKnn*)hp;
  if (!h->knn.data || !h->knn_w.data) return -1;
  const TSDFVolume::Params& p = h->vol->params();
  dim3 block(8, 8, 1);
  dim3 grid((p.dims.x + block.x - 1) / block.x, (p.dims.y + block.y - 1) / block.y, p.dims.z);
  cudaEventRecord(h->e0, 0);
  compute_voxel_knn_kernel<<<grid, block>>>(h->vol->device_data(), p.dims, p.origin, p.voxel_size,
                                            h->warp->device_nodes(), h->warp->num_nodes(), h->knn.data,
                                            h->knn_w.data);
  cudaEventRecord(h->e1, 0);
  cudaEventSynchronize(h->e1);
  if (ms) cudaEventElapsedTime(ms, h->e0, h->e1);
  return (int)cudaGetLastError();
}
