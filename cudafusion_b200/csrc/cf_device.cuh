// cf_device.cuh — device-side types and math shared by the sm_100a kernels.
//
// The SE(3)/DQ functions restate include/se3_math.cuh (CUDAFusion) in FP32
// with the reference's operand order so that results match the reference to
// rounding; each cites the reference lines it follows.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cudafusion_b200.h"

namespace cf {

constexpr int kK = CF_K_NEIGHBORS;  // 4 skinning nodes
constexpr int kG = CF_K_GRAPH;      // 8 graph neighbours

// error bits written by kernels into the handle's device status word
constexpr int kErrTimeout = 1;    // == kErrTimeoutBit (cf_internal.h)
constexpr int kErrNonFinite = 2;  // == kErrNonFiniteBit

struct DQ {
  float4 r, d;
};

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ DQ load_dq(const cf_dual_quat* p) {
  const float4* q = reinterpret_cast<const float4*>(p);
  DQ d;
  d.r = __ldg(q);
  d.d = __ldg(q + 1);
  return d;
}
// through L1: for DQs written by an earlier launch and not during this one
__device__ __forceinline__ DQ load_dq_ldg(const cf_dual_quat* p) {
  const float4* q = reinterpret_cast<const float4*>(p);
  DQ d;
  d.r = __ldg(q);
  d.d = __ldg(q + 1);
  return d;
}
__device__ __forceinline__ DQ load_dq_cg(const cf_dual_quat* p) {
  const float4* q = reinterpret_cast<const float4*>(p);
  DQ d;
  d.r = __ldcg(q);
  d.d = __ldcg(q + 1);
  return d;
}
__device__ __forceinline__ void store_dq(cf_dual_quat* p, DQ d) {
  float4* q = reinterpret_cast<float4*>(p);
  q[0] = d.r;
  q[1] = d.d;
}
__device__ __forceinline__ float3 node_pos(const cf_deform_node* n, int i) {
  const float* p = reinterpret_cast<const float*>(n + i);
  return f3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
}

// ---- quaternion / dual-quaternion math (se3_math.cuh:205-415) ----
__device__ __forceinline__ float4 qmul(float4 a, float4 b) {
  return make_float4(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
                     a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
__device__ __forceinline__ float4 qconj(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }
__device__ __forceinline__ float qdot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__device__ __forceinline__ float4 qnormalize(float4 q) {
  float n = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  if (n < 1e-12f) return make_float4(0.f, 0.f, 0.f, 1.f);
  return make_float4(q.x / n, q.y / n, q.z / n, q.w / n);
}
__device__ __forceinline__ DQ dq_identity() {
  DQ d;
  d.r = make_float4(0.f, 0.f, 0.f, 1.f);
  d.d = make_float4(0.f, 0.f, 0.f, 0.f);
  return d;
}
// se3_math.cuh:302-328
__device__ __forceinline__ DQ dq_normalize(DQ d) {
  float n = sqrtf(d.r.x * d.r.x + d.r.y * d.r.y + d.r.z * d.r.z + d.r.w * d.r.w);
  if (n < 1e-12f) return dq_identity();
  float inv = 1.f / n;
  d.r.x *= inv; d.r.y *= inv; d.r.z *= inv; d.r.w *= inv;
  d.d.x *= inv; d.d.y *= inv; d.d.z *= inv; d.d.w *= inv;
  return d;
}
// se3_math.cuh:330-340
__device__ __forceinline__ DQ dq_mul(DQ a, DQ b) {
  DQ r;
  r.r = qmul(a.r, b.r);
  float4 u = qmul(a.r, b.d), v = qmul(a.d, b.r);
  r.d = make_float4(u.x + v.x, u.y + v.y, u.z + v.z, u.w + v.w);
  return dq_normalize(r);
}
// se3_math.cuh:349-360
__device__ __forceinline__ float3 dq_rotate(DQ d, float3 p) {
  float4 r = qmul(qmul(d.r, make_float4(p.x, p.y, p.z, 0.f)), qconj(d.r));
  return f3(r.x, r.y, r.z);
}
// se3_math.cuh:362-368
__device__ __forceinline__ float3 dq_translation(DQ d) {
  float4 t = qmul(d.d, qconj(d.r));
  return f3(2.f * t.x, 2.f * t.y, 2.f * t.z);
}
// se3_math.cuh:370-377
__device__ __forceinline__ float3 dq_transform_point(DQ d, float3 p) {
  float3 r = dq_rotate(d, p), t = dq_translation(d);
  return f3(r.x + t.x, r.y + t.y, r.z + t.z);
}
// se3_math.cuh:379-388
__device__ __forceinline__ float3 dq_transform_point_centered(DQ d, float3 p, float3 c) {
  float3 rp = dq_transform_point(d, p), rc = dq_rotate(d, c);
  return f3(rp.x + c.x - rc.x, rp.y + c.y - rc.y, rp.z + c.z - rc.z);
}
// se3_math.cuh:390-415: node-centred DQ -> plain DQ
__device__ __forceinline__ DQ dq_centered(DQ d, float3 c) {
  float3 t = dq_translation(d), rc = dq_rotate(d, c);
  float3 ct = f3(t.x + c.x - rc.x, t.y + c.y - rc.y, t.z + c.z - rc.z);
  DQ o;
  o.r = qnormalize(d.r);
  o.d = qmul(make_float4(ct.x, ct.y, ct.z, 0.f), o.r);
  o.d.x *= 0.5f; o.d.y *= 0.5f; o.d.z *= 0.5f; o.d.w *= 0.5f;
  return dq_normalize(o);
}

// se3_math.cuh:40-98 (exp) composed with :244-300 (matrix -> DQ): dq_from_twist.
__device__ __forceinline__ DQ dq_from_twist(const float* tw) {
  float ox = tw[0], oy = tw[1], oz = tw[2], vx = tw[3], vy = tw[4], vz = tw[5];
  float th = sqrtf(ox * ox + oy * oy + oz * oz);
  float A, B, C;
  if (th < 1e-6f) {
    A = 1.f; B = 0.5f; C = 1.f / 6.f;
  } else {
    float it = 1.f / th, it2 = it * it;
    float s = sinf(th), c = cosf(th);
    A = s * it;
    B = (1.f - c) * it2;
    C = (th - s) * it2 * it;
  }
  float m00 = 1.f - B * (oy * oy + oz * oz), m01 = B * ox * oy - A * oz, m02 = B * ox * oz + A * oy;
  float m10 = B * ox * oy + A * oz, m11 = 1.f - B * (ox * ox + oz * oz), m12 = B * oy * oz - A * ox;
  float m20 = B * ox * oz - A * oy, m21 = B * oy * oz + A * ox, m22 = 1.f - B * (ox * ox + oy * oy);
  float v00 = 1.f - C * (oy * oy + oz * oz), v01 = C * ox * oy - B * oz, v02 = C * ox * oz + B * oy;
  float v10 = C * ox * oy + B * oz, v11 = 1.f - C * (ox * ox + oz * oz), v12 = C * oy * oz - B * ox;
  float v20 = C * ox * oz - B * oy, v21 = C * oy * oz + B * ox, v22 = 1.f - C * (ox * ox + oy * oy);
  float tx = v00 * vx + v01 * vy + v02 * vz;
  float ty = v10 * vx + v11 * vy + v12 * vz;
  float tz = v20 * vx + v21 * vy + v22 * vz;
  float tr = m00 + m11 + m22;
  float4 q;
  if (tr > 0.f) {
    float s = sqrtf(tr + 1.f) * 2.f;
    q.w = 0.25f * s; q.x = (m21 - m12) / s; q.y = (m02 - m20) / s; q.z = (m10 - m01) / s;
  } else if (m00 > m11 && m00 > m22) {
    float s = sqrtf(1.f + m00 - m11 - m22) * 2.f;
    q.w = (m21 - m12) / s; q.x = 0.25f * s; q.y = (m01 + m10) / s; q.z = (m02 + m20) / s;
  } else if (m11 > m22) {
    float s = sqrtf(1.f + m11 - m00 - m22) * 2.f;
    q.w = (m02 - m20) / s; q.x = (m01 + m10) / s; q.y = 0.25f * s; q.z = (m12 + m21) / s;
  } else {
    float s = sqrtf(1.f + m22 - m00 - m11) * 2.f;
    q.w = (m10 - m01) / s; q.x = (m02 + m20) / s; q.y = (m12 + m21) / s; q.z = 0.25f * s;
  }
  q = qnormalize(q);
  float4 qd = qmul(make_float4(tx, ty, tz, 0.f), q);
  DQ o;
  o.r = q;
  o.d = make_float4(qd.x * 0.5f, qd.y * 0.5f, qd.z * 0.5f, qd.w * 0.5f);
  return o;
}

// src/warp_field.cu:250-291: scale, clamp rotation and translation norms,
// exponentiate, left-compose.
__device__ __forceinline__ DQ twist_update(DQ T, const float* dx, float max_rot, float max_trans, float scale) {
  float tw[6];
#pragma unroll
  for (int k = 0; k < 6; k++) tw[k] = scale * dx[k];
  float rn = sqrtf(tw[0] * tw[0] + tw[1] * tw[1] + tw[2] * tw[2]);
  if (max_rot > 0.f && rn > max_rot) {
    float s = max_rot / rn;
    tw[0] *= s; tw[1] *= s; tw[2] *= s;
  }
  float tn = sqrtf(tw[3] * tw[3] + tw[4] * tw[4] + tw[5] * tw[5]);
  if (max_trans > 0.f && tn > max_trans) {
    float s = max_trans / tn;
    tw[3] *= s; tw[4] *= s; tw[5] *= s;
  }
  return dq_mul(dq_from_twist(tw), T);
}

// warp_point (se3_math.cuh:450-510) centring each node DQ on the fly: node
// ids outside 0..N-1 and weights below 1e-8 are skipped; no weight left
// copies the point.
__device__ __forceinline__ float3 skin_point_centered(float3 p, const int* ids, const float* ws,
                                                      const cf_deform_node* __restrict__ nodes,
                                                      const cf_dual_quat* __restrict__ T, int N) {
  float4 br = make_float4(0.f, 0.f, 0.f, 0.f), bd = make_float4(0.f, 0.f, 0.f, 0.f);
  float wsum = 0.f;
  for (int k = 0; k < kK; k++) {
    int nid = ids[k];
    float wk = ws[k];
    if (nid < 0 || nid >= N || wk < 1e-8f) continue;
    DQ d = dq_centered(load_dq_cg(T + nid), node_pos(nodes, nid));
    if (qdot(d.r, br) < 0.f) {
      d.r.x = -d.r.x; d.r.y = -d.r.y; d.r.z = -d.r.z; d.r.w = -d.r.w;
      d.d.x = -d.d.x; d.d.y = -d.d.y; d.d.z = -d.d.z; d.d.w = -d.d.w;
    }
    br.x += wk * d.r.x; br.y += wk * d.r.y; br.z += wk * d.r.z; br.w += wk * d.r.w;
    bd.x += wk * d.d.x; bd.y += wk * d.d.y; bd.z += wk * d.d.z; bd.w += wk * d.d.w;
    wsum += wk;
  }
  if (wsum < 1e-8f) return p;
  DQ b;
  b.r = br;
  b.d = bd;
  return dq_transform_point(dq_normalize(b), p);
}

// se3_math.cuh:450-510 with the per-node plain DQs (dq_centered of each node)
// computed once per GN iteration instead of once per (point, node).
__device__ __forceinline__ float3 blend_warp(float3 p, int4 ids, float4 ws, const cf_dual_quat* plain, int N) {
  float4 br = make_float4(0.f, 0.f, 0.f, 0.f), bd = make_float4(0.f, 0.f, 0.f, 0.f);
  float wsum = 0.f;
  int idv[4] = {ids.x, ids.y, ids.z, ids.w};
  float wv[4] = {ws.x, ws.y, ws.z, ws.w};
#pragma unroll
  for (int k = 0; k < kK; k++) {
    int nid = idv[k];
    float w = wv[k];
    if (nid < 0 || nid >= N || w < 1e-8f) continue;
    DQ d = load_dq_ldg(plain + nid);  // (the plain DQs come from an earlier launch)
    if (qdot(d.r, br) < 0.f) {
      d.r.x = -d.r.x; d.r.y = -d.r.y; d.r.z = -d.r.z; d.r.w = -d.r.w;
      d.d.x = -d.d.x; d.d.y = -d.d.y; d.d.z = -d.d.z; d.d.w = -d.d.w;
    }
    br.x += w * d.r.x; br.y += w * d.r.y; br.z += w * d.r.z; br.w += w * d.r.w;
    bd.x += w * d.d.x; bd.y += w * d.d.y; bd.z += w * d.d.z; bd.w += w * d.d.w;
    wsum += w;
  }
  if (wsum < 1e-8f) return p;
  DQ b;
  b.r = br;
  b.d = bd;
  b = dq_normalize(b);
  return dq_transform_point(b, p);
}

// kernels/solver_kernels.cu:13-24
__device__ __forceinline__ float huber_w(float r, float delta) {
  float a = fabsf(r);
  return (a <= delta) ? 1.f : delta / a;
}

// se3_math.cuh:121-145
__device__ __forceinline__ void jac_row(float3 src, float3 x, float3 n, float w, float* J) {
  float3 l = sub3(src, x);
  float3 cp = cross3(l, n);
  J[0] = w * cp.x; J[1] = w * cp.y; J[2] = w * cp.z;
  J[3] = w * n.x; J[4] = w * n.y; J[5] = w * n.z;
}

// 6x6 FP64 Cholesky inverse (se3_math.cuh:152-202); false if not SPD.
__device__ inline bool inv6_chol_d(const double* A, double* Ainv) {
  double L[6][6];
#pragma unroll
  for (int i = 0; i < 6; i++)
#pragma unroll
    for (int j = 0; j < 6; j++) L[i][j] = 0.0;
  for (int i = 0; i < 6; i++)
    for (int j = 0; j <= i; j++) {
      double s = A[i * 6 + j];
      for (int k = 0; k < j; k++) s -= L[i][k] * L[j][k];
      if (i == j) {
        if (!(s > 0.0)) return false;
        L[i][j] = sqrt(s);
      } else {
        L[i][j] = s / L[j][j];
      }
    }
  for (int col = 0; col < 6; col++) {
    double y[6], x[6];
    for (int i = 0; i < 6; i++) {
      double s = (i == col) ? 1.0 : 0.0;
      for (int k = 0; k < i; k++) s -= L[i][k] * y[k];
      y[i] = s / L[i][i];
    }
    for (int i = 5; i >= 0; i--) {
      double s = y[i];
      for (int k = i + 1; k < 6; k++) s -= L[k][i] * x[k];
      x[i] = s / L[i][i];
    }
    for (int i = 0; i < 6; i++) Ainv[i * 6 + col] = x[i];
  }
  return true;
}

// Block-Jacobi inverse of one row, (A_rr + 1e-4 I)^-1 in FP64
// (kernels/solver_kernels.cu:358-399), computed by a group of 8 lanes of one
// warp (lane l of the group = threadIdx.x & 7): lane 0 factors A = L L^T
// keeping reciprocal pivots, lanes 0..5 then solve one column each.  The
// diagonal fallback of the reference applies when the factorisation fails.
// blk: the 36 floats of the diagonal block; S: 72 doubles of group scratch;
// Minv: 36 doubles out.  Every lane of the warp must call it (it syncs the
// warp); `active` is false for groups without a row.  Returns the fallback flag.
__device__ inline bool inv6_group(const float* blk, double* S, double* Minv, bool active) {
  const int l = threadIdx.x & 7;
  double* L = S;       // lower factor, reciprocal pivots on the diagonal (row-major, lower triangle)
  double* D = S + 36;  // A + 1e-4 I
  if (active)
    for (int q = l; q < 36; q += 8) D[q] = (double)blk[q] + ((q % 7 == 0) ? (double)1e-4f : 0.0);
  __syncwarp();
  int ok = 1;
  if (active && l == 0) {
    // the factor in registers (fully unrolled): no dependent shared-memory
    // round trip per multiply-add of the elimination
    double f[21];  // row i, column j <= i at i*(i+1)/2 + j
#pragma unroll
    for (int i = 0; i < 6; i++)
#pragma unroll
      for (int j = 0; j <= i; j++) {
        double s = D[i * 6 + j];
#pragma unroll
        for (int k = 0; k < j; k++) s -= f[i * (i + 1) / 2 + k] * f[j * (j + 1) / 2 + k];
        if (i == j) {
          ok &= (s > 0.0) ? 1 : 0;  // a failed pivot leaves NaN behind it, never read (ok == 0)
          f[i * (i + 1) / 2 + i] = 1.0 / sqrt(s);
        } else {
          f[i * (i + 1) / 2 + j] = s * f[j * (j + 1) / 2 + j];
        }
      }
#pragma unroll
    for (int i = 0; i < 6; i++)
#pragma unroll
      for (int j = 0; j <= i; j++) L[i * 6 + j] = f[i * (i + 1) / 2 + j];
  }
  ok = __shfl_sync(0xffffffffu, ok, (threadIdx.x & 31) & ~7);
  __syncwarp();
  if (active && l < 6) {
    if (ok) {
      double f[21];
#pragma unroll
      for (int i = 0; i < 6; i++)
#pragma unroll
        for (int j = 0; j <= i; j++) f[i * (i + 1) / 2 + j] = L[i * 6 + j];
      double y[6], x[6];
#pragma unroll
      for (int i = 0; i < 6; i++) {
        double s = (i == l) ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < i; k++) s -= f[i * (i + 1) / 2 + k] * y[k];
        y[i] = s * f[i * (i + 1) / 2 + i];
      }
#pragma unroll
      for (int i = 5; i >= 0; i--) {
        double s = y[i];
#pragma unroll
        for (int k = i + 1; k < 6; k++) s -= f[k * (k + 1) / 2 + i] * x[k];
        x[i] = s * f[i * (i + 1) / 2 + i];
      }
#pragma unroll
      for (int i = 0; i < 6; i++) Minv[i * 6 + l] = x[i];
    } else {
      for (int q = 0; q < 6; q++) Minv[l * 6 + q] = (q == l) ? 1.0 / (D[l * 6 + l] + (double)1e-6f) : 0.0;
    }
  }
  __syncwarp();
  return active && !ok;
}

// ---- small helpers ----
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ float sel4(float4 v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }
__device__ __forceinline__ int sel4i(int4 v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
  float y = v - c;
  float t = s + y;
  c = (t - s) - y;
  s = t;
}


// ARAP edge (kernels/solver_kernels.cu:225-289): residual, effective weight,
// and the two lever arms of the Jacobians.
struct Edge {
  float el;
  float3 r, qi, qj;
};

__device__ __forceinline__ Edge eval_edge(const cf_deform_node* nodes, const cf_dual_quat* T, int i, int j, int k,
                                          float lambda) {
  Edge o;
  const float* nwp = reinterpret_cast<const float*>(nodes + i) + 15 + k;  // neighbor_w[k]
  float nw = fmaxf(__ldg(nwp), 0.05f);
  float3 xi = node_pos(nodes, i), xj = node_pos(nodes, j);
  DQ Ti = load_dq_ldg(T + i), Tj = load_dq_ldg(T + j);  // (T comes from an earlier launch)
  float3 ti_xj = dq_transform_point_centered(Ti, xj, xi);
  float3 ti_xi = dq_transform_point_centered(Ti, xi, xi);
  float3 tj_xj = dq_transform_point_centered(Tj, xj, xj);
  float3 rest = sub3(xi, xj), curr = sub3(ti_xi, tj_xj);
  float dr = sqrtf(rest.x * rest.x + rest.y * rest.y + rest.z * rest.z);
  float dc = sqrtf(curr.x * curr.x + curr.y * curr.y + curr.z * curr.z);
  float strain = fabsf(dc - dr) / fmaxf(dr, 1e-6f);
  float ratio = strain / 0.25f;
  float sw = expf(-(ratio * ratio));
  o.r = sub3(ti_xj, tj_xj);
  float rn = sqrtf(o.r.x * o.r.x + o.r.y * o.r.y + o.r.z * o.r.z);
  float el = lambda * nw * huber_w(rn, 0.05f) * sw;
  o.el = (el > 1e-8f) ? el : 0.f;
  o.qi = sub3(ti_xj, xi);
  o.qj = sub3(tj_xj, xj);
  return o;
}

// 6x3 ARAP Jacobian of kernels/solver_kernels.cu:140-165 (sgn = +1), or the
// consistent sign (sgn = -1) on the rotation rows.
__device__ __forceinline__ void arap_jac(float3 q, float sgn, float J[6][3]) {
  J[0][0] = 0.f; J[0][1] = sgn * q.z; J[0][2] = -sgn * q.y;
  J[1][0] = -sgn * q.z; J[1][1] = 0.f; J[1][2] = sgn * q.x;
  J[2][0] = sgn * q.y; J[2][1] = -sgn * q.x; J[2][2] = 0.f;
  J[3][0] = 1.f; J[3][1] = 0.f; J[3][2] = 0.f;
  J[4][0] = 0.f; J[4][1] = 1.f; J[4][2] = 0.f;
  J[5][0] = 0.f; J[5][1] = 0.f; J[5][2] = 1.f;
}


// ---- warp helpers ----
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---- memory-order primitives for the bounded grid barrier ----
// asynchronous global -> shared copies (16, 8 or 4 B: both addresses aligned to the size)
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_gpu_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier over `nblocks` co-resident CTAs (cooperative launch).  The
// counter only grows; instance `gen` (0-based) waits for (gen+1)*nblocks
// arrivals.  The wait is bounded: after `spin_limit` polls it records
// kErrTimeout in *err and returns, and once *err is set every later barrier
// returns at once, so a stuck grid drains instead of hanging.
__device__ __forceinline__ void grid_barrier(unsigned* counter, unsigned gen, unsigned nblocks, int* err,
                                             unsigned spin_limit) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    red_release_gpu_add(counter, 1u);
    unsigned target = (gen + 1u) * nblocks;
    unsigned polls = 0;
    while (ld_acquire_gpu(counter) < target) {
      if (*(volatile int*)err != 0) break;
      if (++polls > spin_limit) {
        atomicOr(err, kErrTimeout);
        break;
      }
      if (polls > 64) __nanosleep(polls > 4096 ? 256 : 32);
    }
    __threadfence();
  }
  __syncthreads();
}

}  // namespace cf
