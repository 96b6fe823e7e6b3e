/*
 * cf_oracle_voxelknn.c — CPU oracle of the voxel kNN field.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it, and only as the checker (or as
 * the timed CPU baseline).
 *
 * Restates compute_voxel_knn_kernel (src/warp_field.cu:299-405), launched by
 * WarpField::compute_voxel_knn (src/warp_field.cu:957-981), voxel by voxel:
 *   - a voxel whose weight is <= 0 gets ids -1 and weights 0 (:319-327);
 *   - otherwise the centre origin + (v + 0.5) voxel_size (:329-332) is
 *     compared with every node in index order; a node replaces the last of
 *     the 4 best when its squared distance is strictly below it, then bubbles
 *     up past strictly larger distances (:343-373), so the list holds the 4
 *     smallest (distance, index) pairs among the nodes closer than 1e30;
 *   - each found node's weight is exp(-d / (2 r^2)) with r = max(radius,
 *     1e-6), normalised by their sum when it exceeds 1e-8 (:375-404).
 *
 * Arithmetic: the centre is fmaf(v + 0.5, voxel_size, origin) and the squared
 * distance fmaf(dz, dz, fmaf(dx, dx, dy * dy)), the contraction of the
 * reference's device build (pinned by the golden fixture made from its kernel
 * and by the two voxels of the 256^3 benchmark volume whose order a different
 * nesting changes); the weights use expf and IEEE division (the reference's
 * build uses --use_fast_math, so weights agree with it to rounding, not bit
 * for bit).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

#define CFO_EXPORT __attribute__((visibility("default")))

#define VK_K 4
#define NODE_FLOATS 24 /* DeformNode, 96 bytes: pos 0-2, normal 3-5, radius 6, ... */

static inline float vk_centre(long long v, float vs, float o) { return fmaf((float)v + 0.5f, vs, o); }

static inline float vk_dist2(float px, float py, float pz, const float* q) {
  float dx = px - q[0], dy = py - q[1], dz = pz - q[2];
  return fmaf(dz, dz, fmaf(dx, dx, dy * dy));
}

/* One voxel's list; `vox` = the 12-byte voxel records as floats (tsdf,
 * weight, colour). */
static void vk_one(const float* vox, const int* dims, const float* origin, float vs, const float* nodes,
                   int num_nodes, long long vidx, int* ids, float* ws) {
  const float weight = vox[3 * vidx + 1];
  if (weight <= 0.f || num_nodes == 0) {
    for (int k = 0; k < VK_K; ++k) {
      ids[k] = -1;
      ws[k] = 0.f;
    }
    return;
  }
  const long long plane = (long long)dims[0] * dims[1];
  const long long z = vidx / plane, r = vidx - z * plane;
  const long long y = r / dims[0], x = r - y * dims[0];
  const float px = vk_centre(x, vs, origin[0]), py = vk_centre(y, vs, origin[1]), pz = vk_centre(z, vs, origin[2]);
  float bd[VK_K];
  int bi[VK_K];
  for (int k = 0; k < VK_K; ++k) {
    bd[k] = 1e30f;
    bi[k] = -1;
  }
  for (int n = 0; n < num_nodes; ++n) {
    const float d = vk_dist2(px, py, pz, nodes + (size_t)NODE_FLOATS * n);
    if (d < bd[VK_K - 1]) {
      bd[VK_K - 1] = d;
      bi[VK_K - 1] = n;
      for (int k = VK_K - 2; k >= 0; --k) {
        if (bd[k + 1] < bd[k]) {
          float td = bd[k];
          bd[k] = bd[k + 1];
          bd[k + 1] = td;
          int ti = bi[k];
          bi[k] = bi[k + 1];
          bi[k + 1] = ti;
        }
      }
    }
  }
  float w[VK_K], sum = 0.f;
  for (int k = 0; k < VK_K; ++k) {
    if (bi[k] < 0) {
      w[k] = 0.f;
      continue;
    }
    const float rad = fmaxf(nodes[(size_t)NODE_FLOATS * bi[k] + 6], 1e-6f);
    w[k] = expf(-bd[k] / (2.0f * rad * rad));
    sum += w[k];
  }
  const float inv = sum > 1e-8f ? 1.0f / sum : 0.0f;
  for (int k = 0; k < VK_K; ++k) {
    ids[k] = bi[k];
    ws[k] = w[k] * inv;
  }
}

/* Voxels [lo, hi) of the volume: knn_ids / knn_ws hold (hi - lo) * 4
 * entries, the lists of voxels lo .. hi-1 in order.  num_nodes == 0 leaves
 * them untouched (the reference returns before its launch,
 * src/warp_field.cu:962-963). */
CFO_EXPORT void cfo_voxel_knn(const float* vox, const int* dims, const float* origin, float voxel_size,
                              const float* nodes, int num_nodes, long long lo, long long hi, int* knn_ids,
                              float* knn_ws, int nthreads) {
  if (num_nodes == 0) return;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads > 0 ? nthreads : 1)
  for (long long v = lo; v < hi; ++v)
    vk_one(vox, dims, origin, voxel_size, nodes, num_nodes, v, knn_ids + VK_K * (v - lo), knn_ws + VK_K * (v - lo));
}

/* The same for an explicit list of voxel indices (a sample of a volume). */
CFO_EXPORT void cfo_voxel_knn_list(const float* vox, const int* dims, const float* origin, float voxel_size,
                                   const float* nodes, int num_nodes, const long long* vidx, long long count,
                                   int* knn_ids, float* knn_ws, int nthreads) {
  if (num_nodes == 0) return;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads > 0 ? nthreads : 1)
  for (long long c = 0; c < count; ++c)
    vk_one(vox, dims, origin, voxel_size, nodes, num_nodes, vidx[c], knn_ids + VK_K * c, knn_ws + VK_K * c);
}
