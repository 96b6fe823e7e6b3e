/*
 * cf_oracle_raster.c — CPU oracle of the live-surface rasterisation.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it, and only as the checker (or as
 * the timed CPU baseline).
 *
 * Restates, triangle by triangle and pixel by pixel:
 *   src/mesh_raster_kernels.cu:76-133   rasterize_triangles_z_kernel
 *   src/mesh_raster_kernels.cu:135-200  resolve_rasterized_triangles_kernel
 *   src/mesh_raster_kernels.cu:8-72     edge_fn, cross3, normalize3, voxel_index,
 *                                       project_triangle
 *   src/skinning_kernels.cu:13-24       the canonical voxel of a point
 * The depth test keeps the least (depth bits << 32 | triangle) per pixel, as the
 * reference's 64-bit atomicMin does, so the triangle order does not matter.
 *
 * Arithmetic: three-term product sums and interpolations accumulate left to
 * right by fused multiply-adds, a*b - c*d is fmaf(a, b, -(c*d)), everything
 * else is one IEEE-rounded operation (built with -ffp-contract=off).  The
 * reference's build uses --use_fast_math; tests/golden holds its outputs on
 * small meshes (made on a B200), against which this oracle is checked to
 * rounding.
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CFO_EXPORT __attribute__((visibility("default")))

typedef struct { float x, y; } rs_f2;
typedef struct { float x, y, z; } rs_f3;

static inline float rs_dot(float ax, float ay, float az, float bx, float by, float bz) {
  return fmaf(az, bz, fmaf(ay, by, ax * bx));
}
static inline float rs_dp(float a, float b, float c, float d) { return fmaf(a, b, -(c * d)); }
static inline float rs_edge(rs_f2 a, rs_f2 b, rs_f2 p) { return rs_dp(p.x - a.x, b.y - a.y, p.y - a.y, b.x - a.x); }
static inline rs_f3 rs_sub(rs_f3 a, rs_f3 b) { rs_f3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline rs_f3 rs_cross(rs_f3 a, rs_f3 b) {
  rs_f3 r = {rs_dp(a.y, b.z, a.z, b.y), rs_dp(a.z, b.x, a.x, b.z), rs_dp(a.x, b.y, a.y, b.x)};
  return r;
}
static inline float rs_norm(rs_f3 v) { return sqrtf(rs_dot(v.x, v.y, v.z, v.x, v.y, v.z)); }
static inline rs_f3 rs_normalize(rs_f3 v) {
  float n = rs_norm(v);
  if (n > 1e-9f) {
    rs_f3 r = {v.x / n, v.y / n, v.z / n};
    return r;
  }
  return v;
}
static inline float rs_lerp3(float w0, float w1, float w2, float a, float b, float c) {
  return fmaf(w2, c, fmaf(w1, b, w0 * a));
}
static inline rs_f3 rs_ld3(const float* p, int i) { rs_f3 r = {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; return r; }
/* __float2int_rd / __float2int_ru: NaN -> 0, saturating */
static inline int rs_f2i(float x) {
  if (isnan(x)) return 0;
  if (x >= 2147483648.0f) return INT_MAX;
  if (x < -2147483648.0f) return INT_MIN;
  return (int)x;
}

typedef struct {
  float fx, fy, cx, cy;
  int W, H;
  const float* cw;
  float ox, oy, oz, vs;
  int dx, dy, dz;
} rs_k;

/* voxel_index (src/mesh_raster_kernels.cu:36-45) */
static int rs_voxel(const rs_k* k, rs_f3 p) {
  int vx = rs_f2i(floorf((p.x - k->ox) / k->vs));
  int vy = rs_f2i(floorf((p.y - k->oy) / k->vs));
  int vz = rs_f2i(floorf((p.z - k->oz) / k->vs));
  if (vx < 0 || vx >= k->dx || vy < 0 || vy >= k->dy || vz < 0 || vz >= k->dz) return -1;
  return (vz * k->dy + vy) * k->dx + vx;
}

/* project_triangle (src/mesh_raster_kernels.cu:47-72) */
static int rs_project(const rs_k* k, const float* warped, const int* t, rs_f3 wc[3], rs_f3 cc[3], rs_f2 p[3],
                      float* area) {
  const float* r = k->cw;
  for (int j = 0; j < 3; j++) {
    wc[j] = rs_ld3(warped, t[j]);
    cc[j].x = rs_dot(r[0], r[1], r[2], wc[j].x, wc[j].y, wc[j].z) + r[3];
    cc[j].y = rs_dot(r[4], r[5], r[6], wc[j].x, wc[j].y, wc[j].z) + r[7];
    cc[j].z = rs_dot(r[8], r[9], r[10], wc[j].x, wc[j].y, wc[j].z) + r[11];
  }
  if (cc[0].z <= 0.0f || cc[1].z <= 0.0f || cc[2].z <= 0.0f) return 0;
  for (int j = 0; j < 3; j++) {
    p[j].x = k->fx * cc[j].x / cc[j].z + k->cx;
    p[j].y = k->fy * cc[j].y / cc[j].z + k->cy;
  }
  *area = rs_edge(p[0], p[1], p[2]);
  return fabsf(*area) >= 1e-6f;
}

static int rs_valid(const int* t, int V) {
  return t[0] >= 0 && t[1] >= 0 && t[2] >= 0 && t[0] < V && t[1] < V && t[2] < V;
}

static int rs_bary(const rs_f2 p[3], float area, rs_f2 q, float* w0, float* w1, float* w2) {
  *w0 = rs_edge(p[1], p[2], q) / area;
  *w1 = rs_edge(p[2], p[0], q) / area;
  *w2 = rs_edge(p[0], p[1], q) / area;
  return !(*w0 < -1e-5f || *w1 < -1e-5f || *w2 < -1e-5f);
}

/* Rasterises NT triangles (int3) of the warped mesh and resolves every pixel
 * of the W x H maps: lv / ln float3 [W*H] (zero where nothing is hit), hit
 * int [W*H] (-1 where nothing is hit or outside the grid).  cam = {fx, fy,
 * cx, cy}; T_cw row-major 4x4; grid = {ox, oy, oz, voxel_size}; dims[3].
 * ztri (W*H, may be NULL) receives the per-pixel depth keys.  Returns the
 * number of pixels hit. */
CFO_EXPORT int cfo_rasterize(const float* canon, const float* warped, const int* tris, int V, int NT, int W, int H,
                             const float* cam, const float* T_cw, const float* grid, const int* dims, float* lv,
                             float* ln, int* hit, uint64_t* ztri_out) {
  rs_k k = {cam[0], cam[1], cam[2], cam[3], W, H, T_cw, grid[0], grid[1], grid[2], grid[3], dims[0], dims[1], dims[2]};
  const size_t P = (size_t)W * H;
  uint64_t* z = ztri_out ? ztri_out : (uint64_t*)malloc(P * sizeof(uint64_t));
  if (!z) return -1;
  for (size_t i = 0; i < P; i++) z[i] = ~(uint64_t)0;
  for (int ti = 0; ti < NT; ti++) {
    const int* t = tris + 3 * (size_t)ti;
    if (!rs_valid(t, V)) continue;
    rs_f3 wc[3], cc[3];
    rs_f2 p[3];
    float area = 0.f;
    if (!rs_project(&k, warped, t, wc, cc, p, &area)) continue;
    int min_u = rs_f2i(floorf(fminf(p[0].x, fminf(p[1].x, p[2].x))));
    int max_u = rs_f2i(ceilf(fmaxf(p[0].x, fmaxf(p[1].x, p[2].x))));
    int min_v = rs_f2i(floorf(fminf(p[0].y, fminf(p[1].y, p[2].y))));
    int max_v = rs_f2i(ceilf(fmaxf(p[0].y, fmaxf(p[1].y, p[2].y))));
    if (min_u < 0) min_u = 0;
    if (max_u > W - 1) max_u = W - 1;
    if (min_v < 0) min_v = 0;
    if (max_v > H - 1) max_v = H - 1;
    if (min_u > max_u || min_v > max_v) continue;
    if (rs_norm(rs_normalize(rs_cross(rs_sub(wc[1], wc[0]), rs_sub(wc[2], wc[0])))) < 1e-6f) continue;
    for (int y = min_v; y <= max_v; y++)
      for (int x = min_u; x <= max_u; x++) {
        float w0, w1, w2;
        rs_f2 q = {(float)x + 0.5f, (float)y + 0.5f};
        if (!rs_bary(p, area, q, &w0, &w1, &w2)) continue;
        float zz = rs_lerp3(w0, w1, w2, cc[0].z, cc[1].z, cc[2].z);
        if (zz <= 0.0f || !isfinite(zz)) continue;
        uint32_t zb;
        memcpy(&zb, &zz, 4);
        uint64_t packed = ((uint64_t)zb << 32) | (uint32_t)ti;
        uint64_t* slot = z + (size_t)y * W + x;
        if (packed < *slot) *slot = packed;
      }
  }
  int nhit = 0;
  for (size_t px = 0; px < P; px++) {
    rs_f3 v = {0, 0, 0}, n = {0, 0, 0};
    int h = -1;
    if (z[px] != ~(uint64_t)0) {
      int ti = (int)(z[px] & 0xffffffffu);
      const int* t = tris + 3 * (size_t)ti;
      rs_f3 wc[3], cc[3];
      rs_f2 p[3];
      float area = 0.f, w0, w1, w2;
      int y = (int)(px / W), x = (int)(px - (size_t)y * W);
      rs_f2 q = {(float)x + 0.5f, (float)y + 0.5f};
      if (rs_valid(t, V) && rs_project(&k, warped, t, wc, cc, p, &area) && rs_bary(p, area, q, &w0, &w1, &w2)) {
        v.x = rs_lerp3(w0, w1, w2, wc[0].x, wc[1].x, wc[2].x);
        v.y = rs_lerp3(w0, w1, w2, wc[0].y, wc[1].y, wc[2].y);
        v.z = rs_lerp3(w0, w1, w2, wc[0].z, wc[1].z, wc[2].z);
        n = rs_normalize(rs_cross(rs_sub(wc[1], wc[0]), rs_sub(wc[2], wc[0])));
        rs_f3 c0 = rs_ld3(canon, t[0]), c1 = rs_ld3(canon, t[1]), c2 = rs_ld3(canon, t[2]);
        rs_f3 cp = {rs_lerp3(w0, w1, w2, c0.x, c1.x, c2.x), rs_lerp3(w0, w1, w2, c0.y, c1.y, c2.y),
                    rs_lerp3(w0, w1, w2, c0.z, c1.z, c2.z)};
        h = rs_voxel(&k, cp);
        nhit++;
      }
    }
    lv[3 * px] = v.x; lv[3 * px + 1] = v.y; lv[3 * px + 2] = v.z;
    ln[3 * px] = n.x; ln[3 * px + 1] = n.y; ln[3 * px + 2] = n.z;
    hit[px] = h;
  }
  if (!ztri_out) free(z);
  return nhit;
}

/* The canonical voxel of each point (src/skinning_kernels.cu:13-24), -1
 * outside the grid. */
CFO_EXPORT void cfo_voxel_of_points(const float* pts, int n, const float* grid, const int* dims, int* out) {
  rs_k k;
  memset(&k, 0, sizeof(k));
  k.ox = grid[0]; k.oy = grid[1]; k.oz = grid[2]; k.vs = grid[3];
  k.dx = dims[0]; k.dy = dims[1]; k.dz = dims[2];
  for (int i = 0; i < n; i++) out[i] = rs_voxel(&k, rs_ld3(pts, i));
}
