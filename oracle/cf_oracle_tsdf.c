/*
 * cf_oracle_tsdf.c — CPU oracle of the warped TSDF integration and of the
 * optimisation counts that gate it.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it, and only as the checker (or as
 * the timed CPU baseline).
 *
 * Restates, voxel by voxel and pixel by pixel:
 *   kernels/tsdf_kernels.cu:85-174   tsdf_integrate_kernel
 *   src/tsdf_volume.cu:11-19         the initial voxel state
 *   src/tsdf_volume.cu:34-50         T_cam_world from camera_pose
 *   kernels/tsdf_kernels.cu:606-650  mark_optimized_voxels_kernel
 * The warp of each voxel centre is the caller's: `live` holds the warped
 * centres (3 floats per voxel, from the oracle's skinning or from the device
 * under test), NULL integrates rigidly at the centres.
 *
 * Arithmetic: the centre is fmaf(v + 0.5, voxel_size, origin); the rigid
 * transform's rows are three-term fused sums (left to right) plus the
 * translation; every other operation is one IEEE-rounded operation and the
 * averaged numerator is fmaf(tsdf, decayed, observation) (built with
 * -ffp-contract=off).  The reference's build uses --use_fast_math, so it
 * agrees with this restatement to rounding.
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#define CFO_EXPORT __attribute__((visibility("default")))

static inline float ts_dot(float ax, float ay, float az, float bx, float by, float bz) {
  return fmaf(az, bz, fmaf(ay, by, ax * bx));
}
/* __float2int_rn: round half to even; NaN -> 0; saturating */
static inline int ts_f2i_rn(float x) {
  if (isnan(x)) return 0;
  if (x >= 2147483648.0f) return INT_MAX;
  if (x < -2147483648.0f) return INT_MIN;
  return (int)rintf(x);
}

/* The TSDFVolume constructor's voxels: tsdf 1, weight 0, colour 128. */
CFO_EXPORT void cfo_tsdf_reset(float* vox, long long n) {
  for (long long i = 0; i < n; ++i) {
    vox[3 * i] = 1.f;
    vox[3 * i + 1] = 0.f;
    uint32_t c = 0x00808080u;
    memcpy(vox + 3 * i + 2, &c, 4);
  }
}

/* src/tsdf_volume.cu:34-50; rows[12] = T_cam_world rows 0..2 */
CFO_EXPORT void cfo_tsdf_world_to_camera(const float* pose, float* rows) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) rows[4 * i + j] = pose[4 * j + i];
  for (int i = 0; i < 3; ++i) {
    float a = rows[4 * i] * pose[3], b = rows[4 * i + 1] * pose[7], c = rows[4 * i + 2] * pose[11];
    rows[4 * i + 3] = -((a + b) + c);
  }
}

/* Voxel centres of voxels [lo, hi) (kernels/tsdf_kernels.cu:117-121). */
CFO_EXPORT void cfo_tsdf_centres(const int* dims, const float* origin, float vs, long long lo, long long hi,
                                 float* out) {
  const long long plane = (long long)dims[0] * dims[1];
  for (long long i = lo; i < hi; ++i) {
    const long long z = i / plane, r = i - z * plane, y = r / dims[0], x = r - y * dims[0];
    float* o = out + 3 * (i - lo);
    o[0] = fmaf((float)x + 0.5f, vs, origin[0]);
    o[1] = fmaf((float)y + 0.5f, vs, origin[1]);
    o[2] = fmaf((float)z + 0.5f, vs, origin[2]);
  }
}

/* tsdf_integrate_kernel over voxels [lo, hi): vox (3 floats per voxel,
 * indexed from 0), live (3 floats per voxel of the range, or NULL for the
 * centres), counts (NULL = no gate; applied only with gate != 0), cam =
 * fx fy cx cy, rows = T_cam_world rows.  Returns the voxels updated. */
CFO_EXPORT long long cfo_tsdf_integrate(float* vox, const int* dims, const float* origin, float vs, float trunc,
                                        const float* depth, int W, int H, const float* cam, const float* rows,
                                        const float* live, const int* counts, int gate, int min_opt, float alpha,
                                        float max_w, long long lo, long long hi) {
  long long updated = 0;
  float cen[3];
  for (long long i = lo; i < hi; ++i) {
    if (gate && counts && counts[i] < min_opt) continue;
    const float* p;
    if (live) {
      p = live + 3 * (i - lo);
    } else {
      cfo_tsdf_centres(dims, origin, vs, i, i + 1, cen);
      p = cen;
    }
    const float cx = ts_dot(rows[0], rows[1], rows[2], p[0], p[1], p[2]) + rows[3];
    const float cy = ts_dot(rows[4], rows[5], rows[6], p[0], p[1], p[2]) + rows[7];
    const float cz = ts_dot(rows[8], rows[9], rows[10], p[0], p[1], p[2]) + rows[11];
    if (cz <= 0.f) continue;
    const int u = ts_f2i_rn((cam[0] * cx) / cz + cam[2]);
    const int v = ts_f2i_rn((cam[1] * cy) / cz + cam[3]);
    if (u < 0 || u >= W || v < 0 || v >= H) continue;
    const float d = depth[(long long)v * W + u];
    if (d <= 0.f) continue;
    const float sdf = d - cz;
    if (sdf < -trunc) continue;
    const float obs = fminf(1.f, sdf / trunc);
    float* cell = vox + 3 * i;
    const float decayed = cell[1] * alpha;
    const float new_w = decayed + 1.f;
    cell[0] = fmaf(cell[0], decayed, obs) / new_w;
    cell[1] = fminf(new_w, max_w);
    ++updated;
  }
  return updated;
}

/* mark_optimized_voxels_kernel, pixel by pixel.  valid / weight are the
 * correspondence records' fields. */
CFO_EXPORT void cfo_mark_optimized_voxels(const uint8_t* valid, const float* weight, const int* vidx_map, int P,
                                          const int* dims, int frame, int* counts, int* frames) {
  for (int px = 0; px < P; ++px) {
    if (!valid[px] || weight[px] <= 0.f) continue;
    const int vidx = vidx_map[px];
    if (vidx < 0) continue;
    const int vx = vidx % dims[0], vy = (vidx / dims[0]) % dims[1], vz = vidx / (dims[0] * dims[1]);
    for (int oz = -1; oz <= 1; ++oz) {
      const int z = vz + oz;
      if (z < 0 || z >= dims[2]) continue;
      for (int oy = -1; oy <= 1; ++oy) {
        const int y = vy + oy;
        if (y < 0 || y >= dims[1]) continue;
        for (int ox = -1; ox <= 1; ++ox) {
          const int x = vx + ox;
          if (x < 0 || x >= dims[0]) continue;
          const int n = (z * dims[1] + y) * dims[0] + x;
          const int prev = frames[n];
          frames[n] = frame;
          if (prev != frame) counts[n] += 1;
        }
      }
    }
  }
}
