// ref_host_shim.cu — C shim over the reference's own __host__ __device__ se3
// functions (include/se3_math.cuh) and its host skinning copy
// (include/fusion_math.h:32-78), compiled for the HOST from the reference
// headers in place (oracle/Makefile target `ref`).  TEST INFRASTRUCTURE ONLY:
// it produces the known-answer vectors that pin the oracle.
#include "se3_math.cuh"
#include "fusion_math.h"

#include <vector>

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

REF_EXPORT void ref_exp_se3(const float* tw, float* T16) {
  Mat4 T = exp_se3(tw);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) T16[i * 4 + j] = T.m[i][j];
}

REF_EXPORT void ref_mat4_to_dq(const float* T16, DualQuat* out) {
  Mat4 T;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) T.m[i][j] = T16[i * 4 + j];
  *out = mat4_to_dq(T);
}

REF_EXPORT void ref_dq_from_twist(const float* tw, DualQuat* out) { *out = dq_from_twist(tw); }

REF_EXPORT void ref_dq_mul(const DualQuat* a, const DualQuat* b, DualQuat* out) { *out = dq_mul(*a, *b); }

REF_EXPORT void ref_dq_centered(const DualQuat* a, const float* c, DualQuat* out) {
  *out = dq_centered(*a, make_float3(c[0], c[1], c[2]));
}

REF_EXPORT void ref_dq_transform_point(const DualQuat* a, const float* p, float* out) {
  float3 r = dq_transform_point(*a, make_float3(p[0], p[1], p[2]));
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

REF_EXPORT void ref_dq_transform_point_centered(const DualQuat* a, const float* p, const float* c, float* out) {
  float3 r = dq_transform_point_centered(*a, make_float3(p[0], p[1], p[2]), make_float3(c[0], c[1], c[2]));
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

// warp_point_dual_quat_host over M points with per-point node ids/weights.
REF_EXPORT void ref_skin(const float* canon, const int* ids, const float* ws, int M, const DeformNode* nodes,
                         const DualQuat* T, int N, float* out) {
  std::vector<DeformNode> vn(nodes, nodes + N);
  std::vector<DualQuat> vt(T, T + N);
  for (int c = 0; c < M; c++) {
    float3 r = warp_point_dual_quat_host(make_float3(canon[3 * c], canon[3 * c + 1], canon[3 * c + 2]), vn, vt,
                                         ids + 4 * c, ws + 4 * c);
    out[3 * c] = r.x; out[3 * c + 1] = r.y; out[3 * c + 2] = r.z;
  }
}

REF_EXPORT int ref_struct_sizes(int* out) {
  out[0] = (int)sizeof(DualQuat);
  out[1] = (int)sizeof(DeformNode);
  out[2] = (int)sizeof(Correspondence);
  return 3;
}
