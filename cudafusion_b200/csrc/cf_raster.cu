// cf_raster.cu — live-surface prediction: the deformed mesh rasterised into
// the live vertex / normal / canonical-voxel maps the correspondence search
// reads.
//
// Restates DynamicFusionPipeline::rasterize_deformed_mesh_live_surface
// (include/fusion_app.h:1216-1318): skin_vertices_from_voxel_knn_kernel
// (src/skinning_kernels.cu:29-63) warps every canonical mesh vertex by the
// nodes of its voxel; rasterize_triangles_z_kernel
// (src/mesh_raster_kernels.cu:76-133) projects each warped triangle and keeps,
// per pixel centre it covers, the least (depth, triangle) pair by a 64-bit
// atomic min; resolve_rasterized_triangles_kernel (:135-200) turns each
// pixel's triangle into the live vertex, the face normal and the canonical
// voxel.
//
// Arithmetic, as in the correspondence search: three-term product sums and
// interpolations accumulate left to right by fused multiply-adds, a
// difference of products a*b - c*d is fmaf(a, b, -(c*d)), and every other
// operation is one IEEE-rounded operation; the CPU oracle performs the same
// operations, so the two agree bit for bit.
//
// Launches per frame: mesh_skin_kernel (one thread per vertex, when the caller
// skins); raster_kernel (one thread per triangle: the set-up, the record the
// resolve reads, and the pixels of a box of up to 64; a larger box goes to a
// list); raster_big_kernel (one warp per listed triangle, its pixels shared
// out over the lanes); resolve_kernel (one thread per pixel; it writes every pixel
// and resets the depth buffer and the list for the next frame, which replaces
// the reference's three memsets).  A pixel centre is tested against each edge
// without dividing unless the edge value lies within a narrow band of the
// threshold.
#include <cmath>

#include "cf_device.cuh"
#include "cf_internal.h"

namespace cf {

namespace {

constexpr unsigned long long kRsEmpty = 0xffffffffffffffffull;
// The rounded quotient w = e / area is below -1e-5f exactly when the real
// quotient is below this midpoint of -1e-5f and the float beneath it (the
// midpoint itself rounds to -1e-5f, its even neighbour).
constexpr double kRsOutside = -1.0000000202126103e-05;

struct RasterConsts {
  float fx, fy, cx, cy;
  int W, H;
  float cw[12];  // T_cam_world, rows 0..2
  float ox, oy, oz, vs;
  int dx, dy, dz;
};

__device__ __forceinline__ float rs_dot(float ax, float ay, float az, float bx, float by, float bz) {
  return fmaf(az, bz, fmaf(ay, by, __fmul_rn(ax, bx)));
}
// a*b - c*d
__device__ __forceinline__ float rs_dp(float a, float b, float c, float d) { return fmaf(a, b, -__fmul_rn(c, d)); }
// edge_fn (src/mesh_raster_kernels.cu:8-11): (p.x-a.x)(b.y-a.y) - (p.y-a.y)(b.x-a.x)
__device__ __forceinline__ float rs_edge(float2 a, float2 b, float2 p) {
  return rs_dp(__fsub_rn(p.x, a.x), __fsub_rn(b.y, a.y), __fsub_rn(p.y, a.y), __fsub_rn(b.x, a.x));
}
__device__ __forceinline__ float3 rs_sub(float3 a, float3 b) {
  return make_float3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}
__device__ __forceinline__ float3 rs_cross(float3 a, float3 b) {
  return make_float3(rs_dp(a.y, b.z, a.z, b.y), rs_dp(a.z, b.x, a.x, b.z), rs_dp(a.x, b.y, a.y, b.x));
}
__device__ __forceinline__ float rs_norm(float3 v) { return __fsqrt_rn(rs_dot(v.x, v.y, v.z, v.x, v.y, v.z)); }
__device__ __forceinline__ float3 rs_normalize(float3 v) {
  const float n = rs_norm(v);
  return n > 1e-9f ? make_float3(__fdiv_rn(v.x, n), __fdiv_rn(v.y, n), __fdiv_rn(v.z, n)) : v;
}
__device__ __forceinline__ float3 rs_ld3(const float* p, int i) {
  return make_float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}
// w0 a + w1 b + w2 c, accumulated left to right
__device__ __forceinline__ float rs_lerp3(float w0, float w1, float w2, float a, float b, float c) {
  return fmaf(w2, c, fmaf(w1, b, __fmul_rn(w0, a)));
}

// The voxel of canonical point p (src/mesh_raster_kernels.cu:36-45,
// src/skinning_kernels.cu:13-24), -1 outside the grid.
__device__ __forceinline__ int rs_voxel(const RasterConsts& k, float3 p) {
  const int vx = __float2int_rd(__fdiv_rn(__fsub_rn(p.x, k.ox), k.vs));
  const int vy = __float2int_rd(__fdiv_rn(__fsub_rn(p.y, k.oy), k.vs));
  const int vz = __float2int_rd(__fdiv_rn(__fsub_rn(p.z, k.oz), k.vs));
  if (vx < 0 || vx >= k.dx || vy < 0 || vy >= k.dy || vz < 0 || vz >= k.dz) return -1;
  return (vz * k.dy + vy) * k.dx + vx;
}

// project_triangle (src/mesh_raster_kernels.cu:47-72): the warped corners,
// their camera-frame points, their projections and the signed area.
__device__ __forceinline__ bool rs_project(const RasterConsts& k, const float* __restrict__ warped, int3 t,
                                           float3 wc[3], float3 cc[3], float2 p[3], float& area) {
  const int ids[3] = {t.x, t.y, t.z};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    wc[j] = rs_ld3(warped, ids[j]);
    const float* r = k.cw;
    cc[j] = make_float3(__fadd_rn(rs_dot(r[0], r[1], r[2], wc[j].x, wc[j].y, wc[j].z), r[3]),
                        __fadd_rn(rs_dot(r[4], r[5], r[6], wc[j].x, wc[j].y, wc[j].z), r[7]),
                        __fadd_rn(rs_dot(r[8], r[9], r[10], wc[j].x, wc[j].y, wc[j].z), r[11]));
  }
  if (cc[0].z <= 0.f || cc[1].z <= 0.f || cc[2].z <= 0.f) return false;
#pragma unroll
  for (int j = 0; j < 3; ++j)
    p[j] = make_float2(__fadd_rn(__fdiv_rn(__fmul_rn(k.fx, cc[j].x), cc[j].z), k.cx),
                       __fadd_rn(__fdiv_rn(__fmul_rn(k.fy, cc[j].y), cc[j].z), k.cy));
  area = rs_edge(p[0], p[1], p[2]);
  return fabsf(area) >= 1e-6f;
}

__device__ __forceinline__ bool rs_valid_tri(int3 t, int V) {
  return t.x >= 0 && t.y >= 0 && t.z >= 0 && t.x < V && t.y < V && t.z < V;
}

// Barycentric weights of pixel centre q; false where the centre is outside
// the triangle by more than 1e-5 (src/mesh_raster_kernels.cu:116-121).
__device__ __forceinline__ bool rs_bary(const float2 p[3], float area, float2 q, float& w0, float& w1, float& w2) {
  w0 = __fdiv_rn(rs_edge(p[1], p[2], q), area);
  w1 = __fdiv_rn(rs_edge(p[2], p[0], q), area);
  w2 = __fdiv_rn(rs_edge(p[0], p[1], q), area);
  return !(w0 < -1e-5f || w1 < -1e-5f || w2 < -1e-5f);
}

__global__ void mesh_skin_kernel(const float* __restrict__ canon, float* __restrict__ warped, int V,
                                 const RasterConsts k, const cf_deform_node* __restrict__ nodes,
                                 const cf_dual_quat* __restrict__ T, int N, const int* __restrict__ vk,
                                 const float* __restrict__ vw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  const float3 p = rs_ld3(canon, i);
  float3 o = p;
  if (N > 0 && nodes && T && vk && vw) {
    const int v = rs_voxel(k, p);
    if (v >= 0) o = skin_point_centered(p, vk + (size_t)v * kK, vw + (size_t)v * kK, nodes, T, N);
  }
  warped[3 * i] = o.x;
  warped[3 * i + 1] = o.y;
  warped[3 * i + 2] = o.z;
}

// Whether e / area rounds below -1e-5f, mostly without the division: e is
// compared with the exact threshold kRsOutside * area (an FP64 product of
// 25- and 24-bit significands, so exact) through a float band around it
// (lo, hi rounded outward); only an e inside the band pays the division.
struct RsEdgeTest {
  float lo, hi;  // the band around the threshold
  bool pos;      // area > 0
};
__device__ __forceinline__ RsEdgeTest rs_edge_test(float area) {
  const double t = __dmul_rn(kRsOutside, (double)area);
  const double pad = fabs(t) * 0x1p-20 + 0x1p-140;
  RsEdgeTest r;
  r.lo = __double2float_rd(t - pad);
  r.hi = __double2float_ru(t + pad);
  r.pos = area > 0.f;
  return r;
}
__device__ __forceinline__ bool rs_out(const RsEdgeTest& g, float e, float area) {
  if (g.pos ? e < g.lo : e > g.hi) return true;
  if (g.pos ? e > g.hi : e < g.lo) return false;
  return __fdiv_rn(e, area) < -1e-5f;
}

// The per-triangle record the raster leaves for the resolve: the projected
// corners, the area, the face normal and the warped and canonical corners,
// 7 float4 (112 B), so that a pixel's owner is one record away.
constexpr int kRsRec = 7;
constexpr int kRsSmallBox = 64;  // boxes up to this many pixels: one thread; larger: one warp

// A drawn triangle's set-up in registers.
struct RsTri {
  float2 p0, p1, p2;
  float area, lo, hi, z0, z1, z2;
  int min_u, min_v, bw, bh;
};

// The reference's per-pixel test and depth-key atomic for pixel (x, y) of
// triangle ti (src/mesh_raster_kernels.cu:112-131), the edge tests without
// division outside the threshold band.
__device__ __forceinline__ void rs_fragment(const RsTri& r, int ti, int x, int y, const RasterConsts& k,
                                            unsigned long long* __restrict__ ztri) {
  const float2 q = make_float2(__fadd_rn((float)x, 0.5f), __fadd_rn((float)y, 0.5f));
  const float e0 = rs_edge(r.p1, r.p2, q), e1 = rs_edge(r.p2, r.p0, q), e2 = rs_edge(r.p0, r.p1, q);
  RsEdgeTest g;
  g.lo = r.lo;
  g.hi = r.hi;
  g.pos = r.area > 0.f;
  if (rs_out(g, e0, r.area) || rs_out(g, e1, r.area) || rs_out(g, e2, r.area)) return;
  const float z = rs_lerp3(__fdiv_rn(e0, r.area), __fdiv_rn(e1, r.area), __fdiv_rn(e2, r.area), r.z0, r.z1, r.z2);
  if (!(z > 0.f) || !isfinite(z)) return;
  atomicMin(ztri + (size_t)y * k.W + x, ((unsigned long long)__float_as_uint(z) << 32) | (unsigned)ti);
}

// Set-up of triangle ti (rasterize_triangles_z_kernel up to the pixel loop,
// src/mesh_raster_kernels.cu:86-110); false when it draws nothing.  A drawn
// triangle's record goes to the cache (when given).
__device__ __forceinline__ bool rs_setup(int ti, const float* __restrict__ canon, const float* __restrict__ warped,
                                         const int3* __restrict__ tris, int V, const RasterConsts& k,
                                         float4* __restrict__ cache, RsTri& r) {
  const int3 t = tris[ti];
  float3 wc[3], cc[3];
  float2 p[3];
  float area = 0.f;
  if (!rs_valid_tri(t, V) || !rs_project(k, warped, t, wc, cc, p, area)) return false;
  r.min_u = max(0, __float2int_rd(fminf(p[0].x, fminf(p[1].x, p[2].x))));
  const int max_u = min(k.W - 1, __float2int_ru(fmaxf(p[0].x, fmaxf(p[1].x, p[2].x))));
  r.min_v = max(0, __float2int_rd(fminf(p[0].y, fminf(p[1].y, p[2].y))));
  const int max_v = min(k.H - 1, __float2int_ru(fmaxf(p[0].y, fmaxf(p[1].y, p[2].y))));
  if (r.min_u > max_u || r.min_v > max_v) return false;
  const float3 fn = rs_normalize(rs_cross(rs_sub(wc[1], wc[0]), rs_sub(wc[2], wc[0])));
  if (rs_norm(fn) < 1e-6f) return false;
  if (cache) {
    const float3 c0 = rs_ld3(canon, t.x), c1 = rs_ld3(canon, t.y), c2 = rs_ld3(canon, t.z);
    float4* rec = cache + (size_t)kRsRec * ti;
    rec[0] = make_float4(p[0].x, p[0].y, p[1].x, p[1].y);
    rec[1] = make_float4(p[2].x, p[2].y, area, fn.x);
    rec[2] = make_float4(fn.y, fn.z, wc[0].x, wc[0].y);
    rec[3] = make_float4(wc[0].z, wc[1].x, wc[1].y, wc[1].z);
    rec[4] = make_float4(wc[2].x, wc[2].y, wc[2].z, c0.x);
    rec[5] = make_float4(c0.y, c0.z, c1.x, c1.y);
    rec[6] = make_float4(c1.z, c2.x, c2.y, c2.z);
  }
  const RsEdgeTest g = rs_edge_test(area);
  r.p0 = p[0];
  r.p1 = p[1];
  r.p2 = p[2];
  r.area = area;
  r.lo = g.lo;
  r.hi = g.hi;
  r.z0 = cc[0].z;
  r.z1 = cc[1].z;
  r.z2 = cc[2].z;
  r.bw = max_u - r.min_u + 1;
  r.bh = max_v - r.min_v + 1;
  return true;
}

// One thread per triangle: a box of up to kRsSmallBox pixels is drawn here;
// a larger one goes to the big list for raster_big_kernel.
__global__ void __launch_bounds__(256) raster_kernel(const float* __restrict__ canon, const float* __restrict__ warped,
                                                     const int3* __restrict__ tris, int V, int NT,
                                                     const RasterConsts k, unsigned long long* __restrict__ ztri,
                                                     float4* __restrict__ cache, int* __restrict__ big,
                                                     int* __restrict__ big_count) {
  const int ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= NT) return;
  RsTri r;
  if (!rs_setup(ti, canon, warped, tris, V, k, cache, r)) return;
  if (r.bw * r.bh > kRsSmallBox) {
    big[atomicAdd(big_count, 1)] = ti;
    return;
  }
  for (int y = r.min_v; y < r.min_v + r.bh; ++y)
    for (int x = r.min_u; x < r.min_u + r.bw; ++x) rs_fragment(r, ti, x, y, k, ztri);
}

// The big list, one warp per triangle: every lane repeats the set-up (the
// same operations, so the same values) and the lanes stride over the box's
// pixels.  The 64-bit min is order-free: the keys equal a sequential pass's.
__global__ void __launch_bounds__(256) raster_big_kernel(const float* __restrict__ canon,
                                                         const float* __restrict__ warped,
                                                         const int3* __restrict__ tris, int V, const RasterConsts k,
                                                         unsigned long long* __restrict__ ztri,
                                                         const int* __restrict__ big,
                                                         const int* __restrict__ big_count) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int n = *big_count;
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < n; w += warps) {
    const int ti = big[w];
    RsTri r;
    if (!rs_setup(ti, canon, warped, tris, V, k, nullptr, r)) continue;  // drew in raster_kernel: cannot fail
    const int cnt = r.bw * r.bh;
    const float inv_w = 1.f / (float)r.bw;
    for (int idx = lane; idx < cnt; idx += 32) {
      int row = __float2int_rz((float)idx * inv_w);
      if (row * r.bw > idx) --row;
      if ((row + 1) * r.bw <= idx) ++row;
      rs_fragment(r, ti, r.min_u + (idx - row * r.bw), r.min_v + row, k, ztri);
    }
  }
}

__global__ void __launch_bounds__(256) resolve_kernel(const RasterConsts k, unsigned long long* __restrict__ ztri,
                                                      const float4* __restrict__ cache, float* __restrict__ lv,
                                                      float* __restrict__ ln, int* __restrict__ hit,
                                                      int* __restrict__ big_count) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  if (px == 0) *big_count = 0;  // the big list is consumed: ready for the next frame
  if (px >= k.W * k.H) return;
  const unsigned long long packed = ztri[px];
  ztri[px] = kRsEmpty;  // ready for the next frame
  float3 v = make_float3(0.f, 0.f, 0.f), n = v;
  int h = -1;
  if (packed != kRsEmpty) {
    // the owner's record: the projection, area, face normal and corners that
    // resolve_rasterized_triangles_kernel recomputes (src/mesh_raster_kernels.cu:162-199)
    const int ti = (int)(packed & 0xffffffffull);
    const float4* rec = cache + (size_t)kRsRec * ti;
    const float4 r0 = rec[0], r1 = rec[1];
    const float2 p[3] = {make_float2(r0.x, r0.y), make_float2(r0.z, r0.w), make_float2(r1.x, r1.y)};
    const float area = r1.z;
    float w0, w1, w2;
    const int y = px / k.W, x = px - y * k.W;
    if (rs_bary(p, area, make_float2(__fadd_rn((float)x, 0.5f), __fadd_rn((float)y, 0.5f)), w0, w1, w2)) {
      const float4 r2 = rec[2], r3 = rec[3], r4 = rec[4], r5 = rec[5], r6 = rec[6];
      v = make_float3(rs_lerp3(w0, w1, w2, r2.z, r3.y, r4.x), rs_lerp3(w0, w1, w2, r2.w, r3.z, r4.y),
                      rs_lerp3(w0, w1, w2, r3.x, r3.w, r4.z));
      n = make_float3(r1.w, r2.x, r2.y);
      h = rs_voxel(k, make_float3(rs_lerp3(w0, w1, w2, r4.w, r5.z, r6.y), rs_lerp3(w0, w1, w2, r5.x, r5.w, r6.z),
                                  rs_lerp3(w0, w1, w2, r5.y, r6.x, r6.w)));
    }
  }
  lv[3 * px] = v.x;
  lv[3 * px + 1] = v.y;
  lv[3 * px + 2] = v.z;
  ln[3 * px] = n.x;
  ln[3 * px + 1] = n.y;
  ln[3 * px + 2] = n.z;
  hit[px] = h;
}

RasterConsts raster_consts(const cf_camera* cam, const cf_mat4* Tcw, const cf_voxel_grid* g) {
  RasterConsts k;
  k.fx = cam ? cam->fx : 0.f;
  k.fy = cam ? cam->fy : 0.f;
  k.cx = cam ? cam->cx : 0.f;
  k.cy = cam ? cam->cy : 0.f;
  k.W = cam ? cam->width : 0;
  k.H = cam ? cam->height : 0;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 4; ++c) k.cw[4 * r + c] = Tcw ? Tcw->m[r][c] : (r == c ? 1.f : 0.f);
  k.ox = g->origin[0];
  k.oy = g->origin[1];
  k.oz = g->origin[2];
  k.vs = g->voxel_size;
  k.dx = g->dims[0];
  k.dy = g->dims[1];
  k.dz = g->dims[2];
  return k;
}

}  // namespace

cudaError_t launch_mesh_skin(const float* canon, float* warped, int V, const cf_voxel_grid* grid,
                             const cf_deform_node* nodes, const cf_dual_quat* T, int N, const int* vk, const float* vw,
                             cudaStream_t s) {
  if (V <= 0) return cudaSuccess;
  const RasterConsts k = raster_consts(nullptr, nullptr, grid);
  mesh_skin_kernel<<<(V + 255) / 256, 256, 0, s>>>(canon, warped, V, k, nodes, T, N, vk, vw);
  return cudaGetLastError();
}

cudaError_t launch_raster(const float* canon, const float* warped, const int* tris, int V, int NT,
                          const cf_camera* cam, const cf_mat4* Tcw, const cf_voxel_grid* grid,
                          unsigned long long* ztri, float4* cache, int* big, int* big_count, float* lv, float* ln,
                          int* hit, cudaStream_t s, long long* launches) {
  const RasterConsts k = raster_consts(cam, Tcw, grid);
  const int P = k.W * k.H;
  if (P == 0) return cudaSuccess;
  const int3* t3 = reinterpret_cast<const int3*>(tris);
  if (NT > 0) {
    // the big list is at most NT long; its kernel strides over it, one warp per
    // triangle, with a grid of 8 CTAs of 8 warps per SM
    static int sms_times_8 = 0;
    if (sms_times_8 == 0) {
      int dev = 0, sms = 148;
      if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      sms_times_8 = 8 * sms;
    }
    raster_kernel<<<(NT + 255) / 256, 256, 0, s>>>(canon, warped, t3, V, NT, k, ztri, cache, big, big_count);
    raster_big_kernel<<<sms_times_8, 256, 0, s>>>(canon, warped, t3, V, k, ztri, big, big_count);
    *launches += 2;
  }
  resolve_kernel<<<(P + 255) / 256, 256, 0, s>>>(k, ztri, cache, lv, ln, hit, big_count);
  *launches += 1;
  return cudaGetLastError();
}

}  // namespace cf
