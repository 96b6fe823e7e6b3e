// ref_cuda_harness.cu — thin driver of the reference's own CUDA solver,
// linked with the unmodified kernels/solver_kernels.cu and src/warp_field.cu
// (oracle/Makefile target `ref`, built for sm_100a with --use_fast_math as the
// reference ships).  TEST AND REFERENCE-ARM INFRASTRUCTURE ONLY: used by the GPU
// parity tests and by `bench.py --impl reference`.
//
// Per GN iteration it does what the reference pipeline does around the solve
// (include/fusion_app.h:253-390,525-550 without the re-rendering):
//   skin every correspondence's canonical point with warp_point
//   (include/se3_math.cuh:450-510)  ->  GaussNewtonSolver::solve
//   ->  WarpField::apply_twist_increment(delta_x, max_rot, max_trans, scale).
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "se3_math.cuh"
#include "solver.h"
#include "warp_field.h"

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

__global__ void harness_skin_kernel(const float* canon, Correspondence* corrs, int m, const DeformNode* nodes,
                                    const DualQuat* transforms) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  Correspondence& c = corrs[i];
  float3 p = make_float3(canon[3 * i], canon[3 * i + 1], canon[3 * i + 2]);
  c.src = warp_point(p, nodes, transforms, c.node_ids, c.node_ws);
}

struct RefHandle {
  GaussNewtonSolver* solver = nullptr;
  WarpField* warp = nullptr;
  DeviceArray<Correspondence> corrs;
  DeviceArray<float> canon;
  DeviceArray<float> delta_x;
  int num_nodes = 0;
  int num_corrs = 0;
};

GaussNewtonSolver::Params to_params(const int* iparams, const float* fparams) {
  GaussNewtonSolver::Params p;
  p.gn_iterations = iparams[0];
  p.pcg_iterations = iparams[1];
  p.debug = iparams[2] != 0;
  p.pcg_tolerance = fparams[0];
  p.lambda_smooth = fparams[1];
  p.lambda_rot = fparams[2];
  p.lambda_damping = fparams[3];
  return p;
}

}  // namespace

// iparams = {gn_iterations, pcg_iterations, debug}; fparams = {pcg_tolerance,
// lambda_smooth, lambda_rot, lambda_damping}.
REF_EXPORT void* ref_create(const int* iparams, const float* fparams, int max_nodes) {
  RefHandle* h = new RefHandle();
  h->solver = new GaussNewtonSolver(to_params(iparams, fparams), max_nodes);
  h->warp = new WarpField(0.02f, max_nodes);
  return h;
}

REF_EXPORT void ref_destroy(void* hp) {
  RefHandle* h = (RefHandle*)hp;
  delete h->solver;
  delete h->warp;
  delete h;
}

// Uploads one problem: nodes, canonical points, correspondences, transforms.
REF_EXPORT int ref_upload(void* hp, const DeformNode* nodes, int n, const float* canon, const Correspondence* corrs,
                          int m, const DualQuat* transforms) {
  RefHandle* h = (RefHandle*)hp;
  h->warp->upload_nodes(std::vector<DeformNode>(nodes, nodes + n));
  h->warp->upload_transforms(std::vector<DualQuat>(transforms, transforms + n));
  h->corrs.upload(std::vector<Correspondence>(corrs, corrs + m));
  h->canon.upload(std::vector<float>(canon, canon + 3 * (size_t)m));
  h->num_nodes = n;
  h->num_corrs = m;
  return (int)cudaDeviceSynchronize();
}

REF_EXPORT int ref_set_transforms(void* hp, const DualQuat* transforms, int n) {
  RefHandle* h = (RefHandle*)hp;
  h->warp->upload_transforms(std::vector<DualQuat>(transforms, transforms + n));
  return (int)cudaDeviceSynchronize();
}

REF_EXPORT int ref_get_transforms(void* hp, DualQuat* out, int n) {
  RefHandle* h = (RefHandle*)hp;
  cudaError_t e = cudaMemcpy(out, h->warp->device_transforms(), sizeof(DualQuat) * n, cudaMemcpyDeviceToHost);
  return (int)e;
}

// One GaussNewtonSolver::solve at the uploaded correspondences' own src
// (no skinning), delta_x to host.
REF_EXPORT int ref_linearize_solve(void* hp, float* dx_out) {
  RefHandle* h = (RefHandle*)hp;
  h->solver->solve(h->corrs, h->num_corrs, h->warp->device_nodes(), h->warp->device_transforms(), h->num_nodes,
                   h->delta_x);
  cudaError_t e = cudaMemcpy(dx_out, h->delta_x.data, sizeof(float) * 6 * h->num_nodes, cudaMemcpyDeviceToHost);
  return (int)e;
}

// The assembled system of the last solve (host copies).
REF_EXPORT int ref_get_system(void* hp, int* row_ptr, int* col_idx, float* values, float* rhs) {
  RefHandle* h = (RefHandle*)hp;
  const BSRMatrix& A = h->solver->system_matrix();
  cudaMemcpy(row_ptr, A.row_ptr.data, sizeof(int) * (A.num_block_rows + 1), cudaMemcpyDeviceToHost);
  cudaMemcpy(col_idx, A.col_idx.data, sizeof(int) * A.num_blocks, cudaMemcpyDeviceToHost);
  cudaMemcpy(values, A.values.data, sizeof(float) * 36 * (size_t)A.num_blocks, cudaMemcpyDeviceToHost);
  cudaMemcpy(rhs, h->solver->rhs().data, sizeof(float) * 6 * h->num_nodes, cudaMemcpyDeviceToHost);
  return A.num_blocks;
}

// G x (skin -> solve -> apply_twist_increment) on the uploaded problem; the
// transforms stay on the device.  Returns a cudaError_t.
REF_EXPORT int ref_gn_solve(void* hp, int gn_iterations, float max_rot, float max_trans, float update_scale) {
  RefHandle* h = (RefHandle*)hp;
  for (int g = 0; g < gn_iterations; g++) {
    int block = 256;
    int grid = (h->num_corrs + block - 1) / block;
    harness_skin_kernel<<<grid, block>>>(h->canon.data, h->corrs.data, h->num_corrs, h->warp->device_nodes(),
                                         h->warp->device_transforms());
    cudaDeviceSynchronize();
    h->solver->solve(h->corrs, h->num_corrs, h->warp->device_nodes(), h->warp->device_transforms(), h->num_nodes,
                     h->delta_x);
    h->warp->apply_twist_increment(h->delta_x, max_rot, max_trans, update_scale);
  }
  return (int)cudaDeviceSynchronize();
}

// Same as ref_gn_solve, timed with CUDA events on the legacy stream; *ms out.
REF_EXPORT int ref_gn_solve_timed(void* hp, int gn_iterations, float max_rot, float max_trans, float update_scale,
                                  float* ms) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, 0);
  int rc = ref_gn_solve(hp, gn_iterations, max_rot, max_trans, update_scale);
  cudaEventRecord(b, 0);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

// Skinned sources of the last iteration (host copy of corrs[].src).
REF_EXPORT int ref_get_corrs(void* hp, Correspondence* out) {
  RefHandle* h = (RefHandle*)hp;
  return (int)cudaMemcpy(out, h->corrs.data, sizeof(Correspondence) * h->num_corrs, cudaMemcpyDeviceToHost);
}
