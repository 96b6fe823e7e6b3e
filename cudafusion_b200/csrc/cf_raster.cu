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
// resolve reads, and the pixels of a box of up to 128; a larger box goes to a
// list as row items); raster_big_kernel (one warp per row item, the row's
// pixels shared out over the lanes); resolve_kernel (one thread per two
// pixels; it writes every pixel and resets the depth buffer and the list for
// the next frame, which replaces the reference's three memsets).  Only the
// pixels of each row's conservative span are tested (a pixel outside it
// cannot pass), and a pixel centre is tested against each edge without
// dividing unless the edge value lies within a narrow band of the threshold.
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

// The same skinning from the nodes' plain dual quaternions (dq_centered of
// each node, computed once per call by the caller's launch), blended as the
// solve's skinning does: no per-vertex centring.  The lists are read as one
// 16-byte load each.
__global__ void mesh_skin_plain_kernel(const float* __restrict__ canon, float* __restrict__ warped, int V,
                                       const RasterConsts k, const cf_dual_quat* __restrict__ plain, int N,
                                       const int4* __restrict__ vk, const float4* __restrict__ vw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  const float3 p = rs_ld3(canon, i);
  float3 o = p;
  const int v = rs_voxel(k, p);
  if (v >= 0) o = blend_warp(p, __ldg(vk + v), __ldg(vw + v), plain, N);
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
constexpr int kRsSmallBox = 128;  // boxes up to this many pixels: one thread; larger: one warp

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

// A drawn triangle's set-up again, from its record in the cache: the same
// fields rs_setup computed (the corners and area as stored, the band from the
// area, each corner's camera depth from its warped corner, the box from the
// corners), by the same operations.
__device__ __forceinline__ void rs_from_record(const float4* __restrict__ rec, const RasterConsts& k, RsTri& r) {
  const float4 r0 = rec[0], r1 = rec[1], r2 = rec[2], r3 = rec[3], r4 = rec[4];
  const float2 p[3] = {make_float2(r0.x, r0.y), make_float2(r0.z, r0.w), make_float2(r1.x, r1.y)};
  const float3 wc[3] = {make_float3(r2.z, r2.w, r3.x), make_float3(r3.y, r3.z, r3.w), make_float3(r4.x, r4.y, r4.z)};
  const float* c = k.cw;
  r.z0 = __fadd_rn(rs_dot(c[8], c[9], c[10], wc[0].x, wc[0].y, wc[0].z), c[11]);
  r.z1 = __fadd_rn(rs_dot(c[8], c[9], c[10], wc[1].x, wc[1].y, wc[1].z), c[11]);
  r.z2 = __fadd_rn(rs_dot(c[8], c[9], c[10], wc[2].x, wc[2].y, wc[2].z), c[11]);
  r.min_u = max(0, __float2int_rd(fminf(p[0].x, fminf(p[1].x, p[2].x))));
  const int max_u = min(k.W - 1, __float2int_ru(fmaxf(p[0].x, fmaxf(p[1].x, p[2].x))));
  r.min_v = max(0, __float2int_rd(fminf(p[0].y, fminf(p[1].y, p[2].y))));
  const int max_v = min(k.H - 1, __float2int_ru(fmaxf(p[0].y, fmaxf(p[1].y, p[2].y))));
  const RsEdgeTest g = rs_edge_test(r1.z);
  r.p0 = p[0];
  r.p1 = p[1];
  r.p2 = p[2];
  r.area = r1.z;
  r.lo = g.lo;
  r.hi = g.hi;
  r.bw = max_u - r.min_u + 1;
  r.bh = max_v - r.min_v + 1;
}

// Row spans: the pixels of a row whose centres can pass the edge tests.  For
// edge i, from a to b, the test computes e = fmaf(dx, B, -(dy * C)) with
// dx = q.x - a.x, dy = q.y - a.y, B = b.y - a.y and C = b.x - a.x each
// rounded once, so |e - (X B - Y C)| <= 3.01 u (|X||B| + |Y||C|) + 2^-140
// for the exact X = q.x - a.x, Y = q.y - a.y (u = 2^-24; the last term for
// results in the subnormal range).  A centre passes only when s e >= Lb (s the
// sign of the area, Lb the outer edge of the test's band), hence only when
// s (X B - Y C) >= Lb - 4u (Xmax |B| + |Y||C|) - 2^-140, Xmax bounding |X|
// over the box.  For B != 0 that bounds X in each row: X >= R + Y C/B -
// 4u |Y||C/B| when s B > 0, X <= R + Y C/B + 4u |Y||C/B| when s B < 0, with
// R = (Lb - 4u Xmax |B| - 2^-140) / (s B).  The float evaluation of the
// bound, fmaf(q.y - a.y, C/B, base), is widened by 32u times the magnitudes
// it combines, which exceeds the sum of its rounding errors and of the
// 4u |Y||C/B| term.  An edge with B == 0 bounds nothing; since the rounded
// B of the three edges are the signed differences of the corners' y, a
// triangle of nonzero area has an edge of each sign, so every row gets a
// lower and an upper bound.  A pixel outside its row's span fails the
// reference's test, so skipping it leaves the depth keys unchanged.
struct RsSpan {
  float ay[3], slope[3], base[3];
  int kind[3];  // +1: lower bound on x, -1: upper bound, 0: none
};

__device__ __forceinline__ void rs_span_edge(float2 a, float2 b, float s, float Lb, float xlo, float xhi, float ylo,
                                             float yhi, float& ay, float& slope, float& base, int& kind) {
  constexpr float u = 0x1p-24f;
  const float B = __fsub_rn(b.y, a.y), C = __fsub_rn(b.x, a.x);
  ay = a.y;
  slope = 0.f;
  base = 0.f;
  kind = 0;
  if (B == 0.f) return;
  const float sB = s * B;
  const float xmax = fmaxf(fabsf(__fsub_rn(xlo, a.x)), fabsf(__fsub_rn(xhi, a.x)));
  const float ymax = fmaxf(fabsf(__fsub_rn(ylo, a.y)), fabsf(__fsub_rn(yhi, a.y)));
  const float ex = __fmul_rn(__fmul_rn(xmax, fabsf(B)), 5.f * u);  // >= 4u Xmax |B| after its own roundings
  const float R = __fdiv_rn(__fsub_rn(__fsub_rn(Lb, ex), 0x1p-140f), sB);
  slope = __fdiv_rn(C, B);
  const float mag = __fadd_rn(__fadd_rn(__fmul_rn(fabsf(slope), ymax), fabsf(a.x)), __fadd_rn(fabsf(R), 1.f));
  const float margin = __fadd_rn(__fmul_rn(mag, 32.f * u), 1e-6f);
  kind = sB > 0.f ? 1 : -1;
  // the pixel index bound: x >= bound - 0.5 (lower) or x <= bound - 0.5 (upper)
  base = __fsub_rn(__fadd_rn(a.x, R), 0.5f);
  base = kind > 0 ? __fsub_rn(base, margin) : __fadd_rn(base, margin);
}

__device__ __forceinline__ void rs_span_setup(const RsTri& r, RsSpan& sp) {
  const float s = r.area > 0.f ? 1.f : -1.f;
  const float Lb = r.area > 0.f ? r.lo : -r.hi;
  const float xlo = __fadd_rn((float)r.min_u, 0.5f), xhi = __fadd_rn((float)(r.min_u + r.bw - 1), 0.5f);
  const float ylo = __fadd_rn((float)r.min_v, 0.5f), yhi = __fadd_rn((float)(r.min_v + r.bh - 1), 0.5f);
  rs_span_edge(r.p1, r.p2, s, Lb, xlo, xhi, ylo, yhi, sp.ay[0], sp.slope[0], sp.base[0], sp.kind[0]);
  rs_span_edge(r.p2, r.p0, s, Lb, xlo, xhi, ylo, yhi, sp.ay[1], sp.slope[1], sp.base[1], sp.kind[1]);
  rs_span_edge(r.p0, r.p1, s, Lb, xlo, xhi, ylo, yhi, sp.ay[2], sp.slope[2], sp.base[2], sp.kind[2]);
}

// The span [x0, x1] of row y, inside the box (empty when x0 > x1).  A NaN
// bound (an infinite slope at a zero offset) is ignored by fmaxf / fminf.
__device__ __forceinline__ void rs_span_row(const RsTri& r, const RsSpan& sp, int y, int& x0, int& x1) {
  const float qy = __fadd_rn((float)y, 0.5f);
  float lo = -1e9f, hi = 1e9f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float t = fmaf(__fsub_rn(qy, sp.ay[i]), sp.slope[i], sp.base[i]);
    if (sp.kind[i] > 0) lo = fmaxf(lo, t);
    if (sp.kind[i] < 0) hi = fminf(hi, t);
  }
  x0 = max(r.min_u, __float2int_ru(fminf(lo, 1e9f)));
  x1 = min(r.min_u + r.bw - 1, __float2int_rd(fmaxf(hi, -1e9f)));
}

// One thread per triangle: the set-up, the record, and the pixels of a box
// of up to kRsSmallBox, row by row over the rows' spans.  A larger box joins
// the big list as one entry and ceil(rows / G) row items: a single 64-bit
// atomic on big_ctr (entries in the high word, items in the low word) gives
// the entry its index and its first item, so the entries' first items
// increase with their index.  128-thread CTAs at 9 per SM: 5120 warps of a
// 164k-triangle mesh fit in one wave.
__global__ void __launch_bounds__(128, 9) raster_kernel(const float* __restrict__ canon, const float* __restrict__ warped,
                                                        const int3* __restrict__ tris, int V, int NT,
                                                        const RasterConsts k, int G,
                                                        unsigned long long* __restrict__ ztri,
                                                        float4* __restrict__ cache, int2* __restrict__ big,
                                                        unsigned long long* __restrict__ big_ctr) {
  const int ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= NT) return;
  RsTri r;
  if (!rs_setup(ti, canon, warped, tris, V, k, cache, r)) return;
  if (r.bw * r.bh > kRsSmallBox) {
    const unsigned items = (unsigned)((r.bh + G - 1) / G);
    const unsigned long long old = atomicAdd(big_ctr, (1ull << 32) | items);
    big[(int)(old >> 32)] = make_int2(ti, (int)(unsigned)old);
    return;
  }
  RsSpan sp;
  rs_span_setup(r, sp);
  for (int y = r.min_v; y < r.min_v + r.bh; ++y) {
    int x0, x1;
    rs_span_row(r, sp, y, x0, x1);
    for (int x = x0; x <= x1; ++x) rs_fragment(r, ti, x, y, k, ztri);
  }
}

// The big list, one warp per row item: the warp finds the item's entry (the
// last whose first item is at or below it) by a 32-way search, rebuilds the
// entry's set-up from its record (the same values) and shares each row's span
// out over its lanes.  The 64-bit min is order-free: the keys
// equal a sequential pass's.
__global__ void __launch_bounds__(256) raster_big_kernel(const float4* __restrict__ cache, const RasterConsts k,
                                                         int G, unsigned long long* __restrict__ ztri,
                                                         const int2* __restrict__ big,
                                                         const unsigned long long* __restrict__ big_ctr) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const unsigned long long ctr = *big_ctr;
  const int n = (int)(ctr >> 32);
  const unsigned total = (unsigned)ctr;
  for (unsigned item = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); item < total; item += warps) {
    // entries [lo, hi) hold the answer; big[lo].y <= item always (big[0].y == 0)
    int lo = 0, hi = n;
    while (hi - lo > 32) {
      const int step = (hi - lo + 31) >> 5;
      const int at = lo + lane * step;
      const unsigned m = __ballot_sync(0xffffffffu, at < hi && (unsigned)big[at].y <= item);
      const int last = 31 - __clz(m);  // lane 0 always qualifies
      lo += last * step;
      hi = min(hi, lo + step);
    }
    const unsigned m = __ballot_sync(0xffffffffu, lo + lane < hi && (unsigned)big[lo + lane].y <= item);
    const int2 e = big[lo + 31 - __clz(m)];
    RsTri r;
    rs_from_record(cache + (size_t)kRsRec * e.x, k, r);
    RsSpan sp;
    rs_span_setup(r, sp);
    const int y0 = r.min_v + (int)(item - (unsigned)e.y) * G;
    const int y1 = min(r.min_v + r.bh, y0 + G);
    for (int y = y0; y < y1; ++y) {
      int x0, x1;
      rs_span_row(r, sp, y, x0, x1);
      for (int x = x0 + lane; x <= x1; x += 32) rs_fragment(r, e.x, x, y, k, ztri);
    }
  }
}

// One thread per two pixels (px and px + half: both rows coalesced), every
// load of both issued before either is used, so that the grid fits one wave.
__device__ __forceinline__ void rs_resolve_px(const RasterConsts& k, int px, unsigned long long packed,
                                              const float4 (&rc)[kRsRec], float* __restrict__ lv,
                                              float* __restrict__ ln, int* __restrict__ hit) {
  float3 v = make_float3(0.f, 0.f, 0.f), n = v;
  int h = -1;
  if (packed != kRsEmpty) {
    // the owner's record: the projection, area, face normal and corners that
    // resolve_rasterized_triangles_kernel recomputes (src/mesh_raster_kernels.cu:162-199)
    const float2 p[3] = {make_float2(rc[0].x, rc[0].y), make_float2(rc[0].z, rc[0].w), make_float2(rc[1].x, rc[1].y)};
    const float area = rc[1].z;
    float w0, w1, w2;
    const int y = px / k.W, x = px - y * k.W;
    if (rs_bary(p, area, make_float2(__fadd_rn((float)x, 0.5f), __fadd_rn((float)y, 0.5f)), w0, w1, w2)) {
      const float4 r2 = rc[2], r3 = rc[3], r4 = rc[4], r5 = rc[5], r6 = rc[6];
      v = make_float3(rs_lerp3(w0, w1, w2, r2.z, r3.y, r4.x), rs_lerp3(w0, w1, w2, r2.w, r3.z, r4.y),
                      rs_lerp3(w0, w1, w2, r3.x, r3.w, r4.z));
      n = make_float3(rc[1].w, r2.x, r2.y);
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

__global__ void __launch_bounds__(256) resolve_kernel(const RasterConsts k, unsigned long long* __restrict__ ztri,
                                                      const float4* __restrict__ cache, float* __restrict__ lv,
                                                      float* __restrict__ ln, int* __restrict__ hit,
                                                      unsigned long long* __restrict__ big_ctr) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) *big_ctr = 0;  // the big list is consumed: ready for the next frame
  const int P = k.W * k.H, half = (P + 1) >> 1;
  if (t >= half) return;
  const int pa = t, pb = t + half;
  const bool hb = pb < P;
  const unsigned long long ka = ztri[pa], kb = hb ? ztri[pb] : kRsEmpty;
  ztri[pa] = kRsEmpty;  // ready for the next frame
  if (hb) ztri[pb] = kRsEmpty;
  float4 ra[kRsRec], rb[kRsRec];
  if (ka != kRsEmpty) {
    const float4* rec = cache + (size_t)kRsRec * (int)(ka & 0xffffffffull);
#pragma unroll
    for (int q = 0; q < kRsRec; ++q) ra[q] = rec[q];
  }
  if (kb != kRsEmpty) {
    const float4* rec = cache + (size_t)kRsRec * (int)(kb & 0xffffffffull);
#pragma unroll
    for (int q = 0; q < kRsRec; ++q) rb[q] = rec[q];
  }
  rs_resolve_px(k, pa, ka, ra, lv, ln, hit);
  if (hb) rs_resolve_px(k, pb, kb, rb, lv, ln, hit);
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

cudaError_t launch_mesh_skin_plain(const float* canon, float* warped, int V, const cf_voxel_grid* grid,
                                   const cf_dual_quat* plain, int N, const int* vk, const float* vw, cudaStream_t s) {
  if (V <= 0) return cudaSuccess;
  const RasterConsts k = raster_consts(nullptr, nullptr, grid);
  mesh_skin_plain_kernel<<<(V + 255) / 256, 256, 0, s>>>(canon, warped, V, k, plain, N,
                                                         reinterpret_cast<const int4*>(vk),
                                                         reinterpret_cast<const float4*>(vw));
  return cudaGetLastError();
}

cudaError_t launch_raster(const float* canon, const float* warped, const int* tris, int V, int NT,
                          const cf_camera* cam, const cf_mat4* Tcw, const cf_voxel_grid* grid,
                          unsigned long long* ztri, float4* cache, int* big, unsigned long long* big_ctr, float* lv,
                          float* ln, int* hit, cudaStream_t s, long long* launches) {
  const RasterConsts k = raster_consts(cam, Tcw, grid);
  const int P = k.W * k.H;
  if (P == 0) return cudaSuccess;
  const int3* t3 = reinterpret_cast<const int3*>(tris);
  int2* big2 = reinterpret_cast<int2*>(big);
  if (NT > 0) {
    // rows per big-list item: 1 unless NT * H items could pass 2^31 (the
    // counter's low word then stays below 2^32)
    const long long worst = (long long)NT * k.H;
    const int G = worst < (1LL << 31) ? 1 : (int)((worst >> 31) + 1);
    // the big list's kernel strides over the row items, one warp per item,
    // with a grid of 2 CTAs of 8 warps per SM
    static int sms_times_2 = 0;
    if (sms_times_2 == 0) {
      int dev = 0, sms = 148;
      if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      sms_times_2 = 2 * sms;
    }
    raster_kernel<<<(NT + 127) / 128, 128, 0, s>>>(canon, warped, t3, V, NT, k, G, ztri, cache, big2, big_ctr);
    raster_big_kernel<<<sms_times_2, 256, 0, s>>>(cache, k, G, ztri, big2, big_ctr);
    *launches += 2;
  }
  resolve_kernel<<<((P + 1) / 2 + 255) / 256, 256, 0, s>>>(k, ztri, cache, lv, ln, hit, big_ctr);
  *launches += 1;
  return cudaGetLastError();
}

}  // namespace cf
