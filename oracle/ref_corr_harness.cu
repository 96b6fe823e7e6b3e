// ref_corr_harness.cu — thin driver of the reference's own correspondence
// search, linked with the unmodified kernels/tsdf_kernels.cu (oracle/Makefile
// target `ref`, built for sm_100a with --use_fast_math as the reference
// ships).  TEST AND REFERENCE-ARM INFRASTRUCTURE ONLY: used by the GPU parity tests,
// by the script that makes the golden fixtures and by
// `bench.py --impl reference --workload corr`.
//
// refc_run does what DynamicFusionPipeline::find_correspondences does
// (include/fusion_app.h:1791-1845): zero the correspondences, the valid count
// and the debug counters; compute_pixel_knn_kernel and
// find_correspondences_kernel on 16x16 blocks; synchronise; read the count.
#include <cuda_runtime.h>

#include "tsdf_kernels.h"
#include "types.h"

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

struct RefCorr {
  int W = 0, H = 0;
  long long V = 0;
  float3 *lv = nullptr, *ln = nullptr, *dn = nullptr;
  float* depth = nullptr;
  int* hit = nullptr;
  int* vk = nullptr;
  float* vw = nullptr;
  int* pk = nullptr;
  float* pw = nullptr;
  Correspondence* corrs = nullptr;
  int* num_valid = nullptr;
  int* stats = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};

}  // namespace

REF_EXPORT void refc_destroy(void* hp) {
  RefCorr* h = (RefCorr*)hp;
  if (!h) return;
  cudaFree(h->lv); cudaFree(h->ln); cudaFree(h->dn); cudaFree(h->depth);
  cudaFree(h->hit); cudaFree(h->vk); cudaFree(h->vw); cudaFree(h->pk); cudaFree(h->pw);
  cudaFree(h->corrs); cudaFree(h->num_valid); cudaFree(h->stats);
  if (h->e0) cudaEventDestroy(h->e0);
  if (h->e1) cudaEventDestroy(h->e1);
  delete h;
}

// Allocates the frame buffers and uploads one frame (host arrays).
REF_EXPORT void* refc_create(int W, int H, const float* lv, const float* ln, const float* depth, const float* dn,
                             const int* hit, const int* vk, const float* vw, long long V) {
  RefCorr* h = new RefCorr();
  h->W = W;
  h->H = H;
  h->V = V;
  const size_t P = (size_t)W * H, V1 = V > 0 ? (size_t)V : 1;
  bool ok = cudaMalloc(&h->lv, P * sizeof(float3)) == cudaSuccess &&
            cudaMalloc(&h->ln, P * sizeof(float3)) == cudaSuccess &&
            cudaMalloc(&h->dn, P * sizeof(float3)) == cudaSuccess &&
            cudaMalloc(&h->depth, P * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&h->hit, P * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&h->vk, V1 * K_NEIGHBORS * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&h->vw, V1 * K_NEIGHBORS * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&h->pk, P * K_NEIGHBORS * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&h->pw, P * K_NEIGHBORS * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&h->corrs, P * sizeof(Correspondence)) == cudaSuccess &&
            cudaMalloc(&h->num_valid, sizeof(int)) == cudaSuccess &&
            cudaMalloc(&h->stats, 6 * sizeof(int)) == cudaSuccess &&
            cudaEventCreate(&h->e0) == cudaSuccess && cudaEventCreate(&h->e1) == cudaSuccess;
  ok = ok && cudaMemcpy(h->lv, lv, P * sizeof(float3), cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(h->ln, ln, P * sizeof(float3), cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(h->dn, dn, P * sizeof(float3), cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(h->depth, depth, P * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(h->hit, hit, P * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok && V > 0)
    ok = cudaMemcpy(h->vk, vk, (size_t)V * K_NEIGHBORS * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->vw, vw, (size_t)V * K_NEIGHBORS * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    refc_destroy(h);
    return nullptr;
  }
  return h;
}

// Re-uploads one frame's per-pixel inputs into the buffers made by refc_create.
REF_EXPORT int refc_upload(void* hp, const float* lv, const float* ln, const float* depth, const float* dn,
                           const int* hit) {
  RefCorr* h = (RefCorr*)hp;
  const size_t P = (size_t)h->W * h->H;
  bool ok = cudaMemcpy(h->lv, lv, P * sizeof(float3), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(h->ln, ln, P * sizeof(float3), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(h->dn, dn, P * sizeof(float3), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(h->depth, depth, P * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(h->hit, hit, P * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
  return ok ? 0 : -1;
}

// One find_correspondences call.  cam = {fx, fy, cx, cy}; T_cw, T_wc row-major
// 4x4.  *ms = device time from the first memset to the end of the search
// kernel (CUDA events).  Returns the valid count, or -1 on a CUDA error.
REF_EXPORT int refc_run(void* hp, const float* cam, const float* T_cw, const float* T_wc, float dist_threshold,
                        float angle_threshold, float view_threshold, int search_radius_px, int debug, float* ms) {
  RefCorr* h = (RefCorr*)hp;
  CameraIntrinsics c;
  c.fx = cam[0];
  c.fy = cam[1];
  c.cx = cam[2];
  c.cy = cam[3];
  c.width = h->W;
  c.height = h->H;
  Mat4 cw, wc;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      cw.m[i][j] = T_cw[4 * i + j];
      wc.m[i][j] = T_wc[4 * i + j];
    }
  const size_t P = (size_t)h->W * h->H;
  cudaEventRecord(h->e0);
  cudaMemset(h->num_valid, 0, sizeof(int));
  cudaMemset(h->stats, 0, 6 * sizeof(int));
  cudaMemset(h->corrs, 0, P * sizeof(Correspondence));
  dim3 block(16, 16);
  dim3 grid((h->W + block.x - 1) / block.x, (h->H + block.y - 1) / block.y);
  compute_pixel_knn_kernel<<<grid, block>>>(h->hit, h->W, h->H, h->vk, h->vw, h->pk, h->pw);
  find_correspondences_kernel<<<grid, block>>>(h->lv, h->ln, h->depth, h->dn, h->corrs, h->num_valid, h->W, h->H, c,
                                               cw, wc, h->pk, h->pw, dist_threshold, angle_threshold,
                                               view_threshold, search_radius_px, debug ? h->stats : nullptr);
  cudaEventRecord(h->e1);
  if (cudaDeviceSynchronize() != cudaSuccess) return -1;
  int n = 0;
  if (cudaMemcpy(&n, h->num_valid, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  if (ms) cudaEventElapsedTime(ms, h->e0, h->e1);
  return n;
}

// Copies the last run's records, per-pixel node lists and debug counters.
REF_EXPORT int refc_download(void* hp, Correspondence* corrs, int* pk, float* pw, int* stats) {
  RefCorr* h = (RefCorr*)hp;
  const size_t P = (size_t)h->W * h->H;
  bool ok = true;
  if (corrs) ok = ok && cudaMemcpy(corrs, h->corrs, P * sizeof(Correspondence), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (pk) ok = ok && cudaMemcpy(pk, h->pk, P * K_NEIGHBORS * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (pw) ok = ok && cudaMemcpy(pw, h->pw, P * K_NEIGHBORS * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (stats) ok = ok && cudaMemcpy(stats, h->stats, 6 * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess;
  return ok ? 0 : -1;
}

REF_EXPORT int refc_sizeof_correspondence() { return (int)sizeof(Correspondence); }
