// cf_corr.cu — projective correspondence search (point-to-plane ICP pairs).
//
// Restates DynamicFusionPipeline::find_correspondences
// (include/fusion_app.h:1791-1845): compute_pixel_knn_kernel
// (kernels/tsdf_kernels.cu:573-604) then find_correspondences_kernel
// (kernels/tsdf_kernels.cu:386-563).  Per live pixel: reject a missing live
// vertex or normal, project the vertex into the depth camera, reject a
// projection behind the camera or off the image and a normal seen edge-on,
// then scan the (2r+1)^2 depth pixels around the projection in row-major
// order.  A candidate is skipped without depth, farther than the Euclidean cap
// max(3 d, d + 0.03), without a normal, with |n_live . n_dst| below the angle
// threshold, or with a point-to-plane distance above d or not below the best
// so far; otherwise it becomes the best.  The pair stores the live vertex, the
// best candidate and its normal mapped back to the world, the squared mean of
// the three confidences and the pixel's node ids/weights.
//
// Arithmetic.  Every three-term product sum is accumulated left to right by
// fused multiply-adds, fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)); every other
// operation is a single IEEE-rounded add, multiply, divide or square root.  The
// CPU oracle performs the same operations, so the two agree bit for bit.  (The
// reference is built with --use_fast_math, whose divide and square root are
// approximations; its results agree with these to rounding.)
//
// Launches per frame:
//  corr_prep_kernel    per depth pixel one 24-byte candidate record: the
//                      unprojected point and the normal.  The two skip cases
//                      are folded into z (0: no depth; -1: no normal) with x, y
//                      and the normal's x so large that the record's
//                      point-to-plane distance is +inf.
//                      The reference recomputes the unprojection, two
//                      divisions, for every (pixel, candidate) pair.
//  corr_search_kernel  one thread per two vertically adjacent live pixels (one
//                      shared-memory load serves both windows; each pixel still
//                      meets its candidates in row-major order), 32 x 16 pixels
//                      per CTA, and
//                      blockIdx.z = one of C chunks of the rows that the CTA's
//                      windows cover (C from a cost model of the waves of
//                      tiles x C CTAs over the resident slots).  The CTA stages
//                      its chunk in shared memory one band of rows at a time;
//                      each thread scans its window's rows in the chunk in
//                      row-major order with the reference's acceptance rule,
//                      applied to groups of 4 consecutive candidates (one min
//                      per candidate, one compare per group, the group's first
//                      column found again at the end).  The Euclidean test
//                      compares the
//                      squared distance with the largest float whose IEEE
//                      square root is within the cap (exact: the rounded
//                      square root is monotonic), and is left out for a band
//                      whose bounding box of real points lies within the cap.  With one chunk the kernel writes the
//                      records itself; otherwise each (chunk, pixel) leaves its
//                      best distance and candidate for
//  corr_merge_kernel   which takes the chunks in row order with the same
//                      strict-less rule.  That reproduces one sequential scan
//                      because no distance can be NaN: every value entering
//                      the search is finite and at most 1e18 in magnitude, so
//                      no product sum overflows.  A pixel or frame holding any
//                      other value is rescanned sequentially with the
//                      reference's rule as it stands (a NaN distance is
//                      accepted).  The record write gathers the pixel's node
//                      lists and reduces the counters per warp.
#include <cfloat>
#include <climits>
#include <cmath>

#include "cf_internal.h"

namespace cf {

namespace {

constexpr int kCsTx = 32;
constexpr int kCsTy = 8;
constexpr int kCsPy = 2 * kCsTy;  // pixel rows per tile: each thread scans two
constexpr int kCsThreads = kCsTx * kCsTy;
constexpr int kCsSmem = 55 * 1024;  // one band of records; 4 CTAs per SM with the 1 KB reserve each
constexpr int kCsCtasPerSm = 4;
constexpr int kCsRecBytes = (int)(sizeof(float4) + sizeof(float2));
constexpr float kCsBig = 1e18f;  // squares and three-term sums of such values stay finite in FP32
constexpr float kCsFar = 1e30f;  // x, y and normal x of a skip record: its distance overflows to +inf

struct CorrConsts {
  float fx, fy, cx, cy;
  int W, H, P, radius, chunks;
  float cw[12];  // T_cam_world, rows 0..2
  float wc[12];  // T_world_cam, rows 0..2
  float dist_thr, angle_thr, view_thr;
  float cap, s_max, normal_eps, view_eps;
};

struct KnnSrc {
  const int* pixel_knn;
  const float* pixel_knn_w;
  const int* hit;
  const int* voxel_knn;
  const float* voxel_knn_w;
  long long num_voxels;
  int* pixel_knn_out;
  float* pixel_knn_w_out;
};

__device__ __forceinline__ float cs_dot(float ax, float ay, float az, float bx, float by, float bz) {
  return fmaf(az, bz, fmaf(ay, by, __fmul_rn(ax, bx)));
}

// Mat4::transform_point / transform_normal (include/types.h:37-57) on rows
// r[0..11] = M[0][0..3], M[1][0..3], M[2][0..3].
__device__ __forceinline__ float3 cs_point(const float* r, float x, float y, float z) {
  return make_float3(__fadd_rn(cs_dot(r[0], r[1], r[2], x, y, z), r[3]),
                     __fadd_rn(cs_dot(r[4], r[5], r[6], x, y, z), r[7]),
                     __fadd_rn(cs_dot(r[8], r[9], r[10], x, y, z), r[11]));
}
__device__ __forceinline__ float3 cs_normal(const float* r, float x, float y, float z) {
  return make_float3(cs_dot(r[0], r[1], r[2], x, y, z), cs_dot(r[4], r[5], r[6], x, y, z),
                     cs_dot(r[8], r[9], r[10], x, y, z));
}
// normalize3, include/se3_math.cuh:28-33.
__device__ __forceinline__ float3 cs_normalize(float3 v) {
  const float n = __fsqrt_rn(cs_dot(v.x, v.y, v.z, v.x, v.y, v.z));
  return n > 1e-9f ? make_float3(__fdiv_rn(v.x, n), __fdiv_rn(v.y, n), __fdiv_rn(v.z, n)) : v;
}
__device__ __forceinline__ float cs_norm(float x, float y, float z) { return __fsqrt_rn(cs_dot(x, y, z, x, y, z)); }
__device__ __forceinline__ bool cs_small(float v) { return fabsf(v) <= kCsBig; }  // false for NaN and inf

__global__ void corr_prep_kernel(const float* __restrict__ depth, const float* __restrict__ dn, int W, int H,
                                 float fx, float fy, float cx, float cy, float4* __restrict__ A,
                                 float2* __restrict__ B, int* __restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W * H) return;
  const int y = i / W, x = i - y * W;
  const float d = depth[i];
  float4 a = make_float4(kCsFar, kCsFar, 0.f, kCsFar);
  float2 b = make_float2(0.f, 0.f);
  if (!(d <= 0.f)) {
    const float nx = dn[3 * i], ny = dn[3 * i + 1], nz = dn[3 * i + 2];
    if (cs_norm(nx, ny, nz) < 1e-6f) {
      a.z = -1.f;
    } else {
      // CameraIntrinsics::unproject, include/types.h:157-161
      a.x = __fdiv_rn(__fmul_rn(d, __fsub_rn((float)x, cx)), fx);
      a.y = __fdiv_rn(__fmul_rn(d, __fsub_rn((float)y, cy)), fy);
      a.z = d;
      a.w = nx;
      b = make_float2(ny, nz);
      if (!(cs_small(a.x) && cs_small(a.y) && cs_small(d) && cs_small(nx) && cs_small(ny) && cs_small(nz)))
        atomicOr(flag, 1);
    }
  }
  A[i] = a;
  B[i] = b;
}

// The per-pixel part of find_correspondences_kernel before the window scan.
struct CsPixel {
  int code;      // debug counter when the pixel stops here, else -1
  bool search;   // the window is scanned
  bool special;  // the scan must run sequentially with the reference's NaN behaviour
  int pu, pv;
  float3 vl, vc, nc;
  float view_cos;
};

__device__ __forceinline__ CsPixel cs_pixel(const CorrConsts& k, const float* __restrict__ lv,
                                            const float* __restrict__ ln, int px, int frame_flag) {
  CsPixel p;
  p.code = -1;
  p.search = false;
  p.special = false;
  p.pu = p.pv = 0;
  p.vl = make_float3(lv[3 * px], lv[3 * px + 1], lv[3 * px + 2]);
  p.vc = p.nc = make_float3(0.f, 0.f, 0.f);
  p.view_cos = 0.f;
  const float3 nl = make_float3(ln[3 * px], ln[3 * px + 1], ln[3 * px + 2]);
  if (cs_norm(p.vl.x, p.vl.y, p.vl.z) < 1e-6f || cs_norm(nl.x, nl.y, nl.z) < 1e-6f) {
    p.code = 0;
    return p;
  }
  p.vc = cs_point(k.cw, p.vl.x, p.vl.y, p.vl.z);
  if (p.vc.z <= 0.f) {
    p.code = 1;
    return p;
  }
  // CameraIntrinsics::project, include/types.h:152-155
  p.pu = __float2int_rn(__fadd_rn(__fdiv_rn(__fmul_rn(k.fx, p.vc.x), p.vc.z), k.cx));
  p.pv = __float2int_rn(__fadd_rn(__fdiv_rn(__fmul_rn(k.fy, p.vc.y), p.vc.z), k.cy));
  if (p.pu < 0 || p.pu >= k.W || p.pv < 0 || p.pv >= k.H) {
    p.code = 1;
    return p;
  }
  p.nc = cs_normal(k.cw, nl.x, nl.y, nl.z);
  const float3 vd = cs_normalize(make_float3(-p.vc.x, -p.vc.y, -p.vc.z));
  p.view_cos = fabsf(cs_dot(p.nc.x, p.nc.y, p.nc.z, vd.x, vd.y, vd.z));
  if (p.view_cos < k.view_thr) {
    p.code = 4;
    return p;
  }
  p.search = true;
  p.special = frame_flag != 0 || !(cs_small(p.vc.x) && cs_small(p.vc.y) && cs_small(p.vc.z) && cs_small(p.nc.x) &&
                                   cs_small(p.nc.y) && cs_small(p.nc.z));
  return p;
}

// The scan state of one pixel: its projection, camera-frame point and normal,
// and the best candidate so far.
struct CsScan {
  int pu, pv;
  float vx, vy, vz, nx, ny, nz;
  float best;
  int bi;
  bool on;  // the pixel is scanned here
};

__device__ __forceinline__ CsScan cs_scan_state(const CsPixel& p, bool on, float dist_thr) {
  CsScan q;
  q.pu = p.pu;
  q.pv = p.pv;
  q.vx = p.vc.x;
  q.vy = p.vc.y;
  q.vz = p.vc.z;
  q.nx = p.nc.x;
  q.ny = p.nc.y;
  q.nz = p.nc.z;
  q.best = dist_thr;
  q.bi = -1;
  q.on = on;
  return q;
}

// A candidate's point-to-plane distance, +inf where the reference would skip
// it (finite values only).  A skip record's far-away point and huge normal
// make its distance +inf by themselves.  kCheckS: apply the Euclidean cap
// (left out where the band's bounding box proves every record within it);
// kAngle: apply the angle threshold.
template <bool kAngle, bool kCheckS>
__device__ __forceinline__ float cs_pd(const CsScan& q, const float4& a, const float2& b, const CorrConsts& k) {
  const float ex = __fsub_rn(q.vx, a.x), ey = __fsub_rn(q.vy, a.y), ez = __fsub_rn(q.vz, a.z);
  float pd = fabsf(cs_dot(a.w, b.x, b.y, ex, ey, ez));
  if (kCheckS) pd = cs_dot(ex, ey, ez, ex, ey, ez) <= k.s_max ? pd : INFINITY;
  if (kAngle) pd = fabsf(cs_dot(q.nx, q.ny, q.nz, a.w, b.x, b.y)) < k.angle_thr ? INFINITY : pd;
  return pd;
}

// The acceptance rule over columns lo..hi of one row, for one pixel or for
// two at one load each, by groups of kCsGroup consecutive candidates: the
// group's minimum distance (one min per candidate) replaces the best when
// strictly below it, and q.bi keeps the first candidate of that group.  The
// winning group is the first one holding the least distance, as in the
// reference's scan; cs_resolve finds the first candidate in it reaching that
// distance.  best starts at the distance bound and only falls, so a kept
// distance is below the bound.
constexpr int kCsGroup = 4;

__device__ __forceinline__ void cs_keep(CsScan& q, float m, int idx) {
  const bool acc = m < q.best;
  q.best = acc ? m : q.best;
  q.bi = acc ? idx : q.bi;
}

template <bool kAngle, bool kCheckS>
__device__ __forceinline__ void cs_seg1(const float4* ra, const float2* rb, int lo, int hi, int row_base, CsScan& q,
                                        const CorrConsts& k) {
  int xx = lo;
  for (; xx + kCsGroup - 1 <= hi; xx += kCsGroup) {
    float m = INFINITY;
#pragma unroll
    for (int j = 0; j < kCsGroup; ++j) m = fminf(m, cs_pd<kAngle, kCheckS>(q, ra[xx + j], rb[xx + j], k));
    cs_keep(q, m, row_base + xx);
  }
  for (; xx <= hi; ++xx) cs_keep(q, cs_pd<kAngle, kCheckS>(q, ra[xx], rb[xx], k), row_base + xx);
}

template <bool kAngle, bool kCheckS>
__device__ __forceinline__ void cs_seg2(const float4* ra, const float2* rb, int lo, int hi, int row_base, CsScan& q0,
                                        CsScan& q1, const CorrConsts& k) {
  int xx = lo;
  for (; xx + kCsGroup - 1 <= hi; xx += kCsGroup) {
    float m0 = INFINITY, m1 = INFINITY;
#pragma unroll
    for (int j = 0; j < kCsGroup; ++j) {
      const float4 a = ra[xx + j];
      const float2 b = rb[xx + j];
      m0 = fminf(m0, cs_pd<kAngle, kCheckS>(q0, a, b, k));
      m1 = fminf(m1, cs_pd<kAngle, kCheckS>(q1, a, b, k));
    }
    cs_keep(q0, m0, row_base + xx);
    cs_keep(q1, m1, row_base + xx);
  }
  for (; xx <= hi; ++xx) {
    const float4 a = ra[xx];
    const float2 b = rb[xx];
    cs_keep(q0, cs_pd<kAngle, kCheckS>(q0, a, b, k), row_base + xx);
    cs_keep(q1, cs_pd<kAngle, kCheckS>(q1, a, b, k), row_base + xx);
  }
}

// The first candidate of the kept group whose distance equals the best
// (recomputed with the cap test: where it was left out it holds anyway).
template <bool kAngle>
__device__ __forceinline__ void cs_resolve(CsScan& q, const float4* __restrict__ A, const float2* __restrict__ B,
                                           const CorrConsts& k) {
  if (!q.on || q.bi < 0) return;
  const int last = min(q.bi + kCsGroup - 1, (q.bi / k.W) * k.W + k.W - 1);
  for (int i = q.bi; i <= last; ++i)
    if (cs_pd<kAngle, true>(q, A[i], B[i], k) == q.best) {
      q.bi = i;
      return;
    }
}

// Row yy of the two pixels' windows (ra/rb: the row's records indexed by
// image column).  Each pixel still meets its candidates in increasing column
// order: the row splits into the part only one window covers on the left,
// the shared part, and the part only one covers on the right.
template <bool kAngle, bool kCheckS>
__device__ __forceinline__ void cs_pair_row(const float4* ra, const float2* rb, int yy, CsScan& q0, CsScan& q1,
                                            const CorrConsts& k) {
  const int r = k.radius, row_base = yy * k.W;
  const bool in0 = q0.on && yy >= q0.pv - r && yy <= q0.pv + r;
  const bool in1 = q1.on && yy >= q1.pv - r && yy <= q1.pv + r;
  const int l0 = max(0, q0.pu - r), h0 = min(k.W - 1, q0.pu + r);
  const int l1 = max(0, q1.pu - r), h1 = min(k.W - 1, q1.pu + r);
  if (in0 && in1) {
    const int slo = max(l0, l1), shi = min(h0, h1);
    if (slo <= shi) {
      if (l0 < slo) cs_seg1<kAngle, kCheckS>(ra, rb, l0, slo - 1, row_base, q0, k);
      else if (l1 < slo) cs_seg1<kAngle, kCheckS>(ra, rb, l1, slo - 1, row_base, q1, k);
      cs_seg2<kAngle, kCheckS>(ra, rb, slo, shi, row_base, q0, q1, k);
      if (h0 > shi) cs_seg1<kAngle, kCheckS>(ra, rb, shi + 1, h0, row_base, q0, k);
      else if (h1 > shi) cs_seg1<kAngle, kCheckS>(ra, rb, shi + 1, h1, row_base, q1, k);
    } else {
      cs_seg1<kAngle, kCheckS>(ra, rb, l0, h0, row_base, q0, k);
      cs_seg1<kAngle, kCheckS>(ra, rb, l1, h1, row_base, q1, k);
    }
  } else if (in0) {
    cs_seg1<kAngle, kCheckS>(ra, rb, l0, h0, row_base, q0, k);
  } else if (in1) {
    cs_seg1<kAngle, kCheckS>(ra, rb, l1, h1, row_base, q1, k);
  }
}

// Whether every record of a band whose real points lie in the box lo..hi is
// within the Euclidean cap of the pixel's point: the box's farthest corner,
// with a relative margin of 1e-4 over the few-ulp rounding of the squared
// distances, is below the bound.
__device__ __forceinline__ bool cs_within_cap(const CsScan& q, const float* lo, const float* hi, float s_max) {
  if (!q.on) return true;
  if (lo[0] > hi[0]) return true;  // no real record in the band
  const float dx = fmaxf(fabsf(q.vx - lo[0]), fabsf(q.vx - hi[0]));
  const float dy = fmaxf(fabsf(q.vy - lo[1]), fabsf(q.vy - hi[1]));
  const float dz = fmaxf(fabsf(q.vz - lo[2]), fabsf(q.vz - hi[2]));
  return (dx * dx + dy * dy + dz * dz) * 1.0001f <= s_max;
}

// find_correspondences_kernel's loop as it stands (kernels/tsdf_kernels.cu:470-524),
// for pixels or frames whose values could make a distance NaN.
__device__ __forceinline__ int cs_rescan(const CorrConsts& k, const CsPixel& p, const float4* __restrict__ A,
                                         const float2* __restrict__ B, bool& saw_depth) {
  const int r = k.radius;
  const int x0 = max(0, p.pu - r), x1 = min(k.W - 1, p.pu + r);
  const int y0 = max(0, p.pv - r), y1 = min(k.H - 1, p.pv + r);
  float best = k.dist_thr;
  int bi = -1;
  for (int yy = y0; yy <= y1; ++yy)
    for (int xx = x0; xx <= x1; ++xx) {
      const float4 a = A[yy * k.W + xx];
      if (a.z == 0.f) continue;
      saw_depth = true;
      if (a.z < 0.f) continue;
      const float ex = __fsub_rn(p.vc.x, a.x), ey = __fsub_rn(p.vc.y, a.y), ez = __fsub_rn(p.vc.z, a.z);
      if (cs_dot(ex, ey, ez, ex, ey, ez) > k.s_max) continue;
      const float2 b = B[yy * k.W + xx];
      if (fabsf(cs_dot(p.nc.x, p.nc.y, p.nc.z, a.w, b.x, b.y)) < k.angle_thr) continue;
      const float pd = fabsf(cs_dot(a.w, b.x, b.y, ex, ey, ez));
      if (pd > k.dist_thr || pd >= best) continue;
      best = pd;
      bi = yy * k.W + xx;
    }
  return bi;
}

// Whether the pixel's window holds any depth (no_depth vs far, for the
// debug counters of a pixel without a pair).
__device__ __forceinline__ bool cs_any_depth(const CorrConsts& k, const CsPixel& p, const float4* __restrict__ A) {
  const int r = k.radius;
  const int x0 = max(0, p.pu - r), x1 = min(k.W - 1, p.pu + r);
  const int y0 = max(0, p.pv - r), y1 = min(k.H - 1, p.pv + r);
  for (int yy = y0; yy <= y1; ++yy)
    for (int xx = x0; xx <= x1; ++xx)
      if (A[yy * k.W + xx].z != 0.f) return true;
  return false;
}

// Writes pixel px's record from its winner bi (-1: none) and adds the
// pixel to the valid count and to its debug counter (code, -1: none), both
// reduced per warp first.  Called by every thread of the warp, whose lanes
// hold consecutive pixels (the in-image ones a prefix): each lane's 19-word
// record goes to the warp's staging area (kCsRecWords words per lane, in
// shared memory), and the warp writes its records' words out in order, 32
// consecutive words per store.
constexpr int kCsRecWords = (int)(sizeof(cf_correspondence) / 4);
static_assert(sizeof(cf_correspondence) == 4 * kCsRecWords, "a record is whole words");
__device__ __forceinline__ void cs_emit(const CorrConsts& k, const CsPixel& p, bool inimg, int px, int bi, int code,
                                        const float4* __restrict__ A, const float2* __restrict__ B,
                                        const KnnSrc& knn, cf_correspondence* __restrict__ out,
                                        int* __restrict__ num_valid, int* __restrict__ stats, int lane,
                                        float* __restrict__ stage) {
  const bool valid = bi >= 0;
  if (inimg) {
    int ids[CF_K_NEIGHBORS];
    float ws[CF_K_NEIGHBORS];
#pragma unroll
    for (int j = 0; j < CF_K_NEIGHBORS; ++j) {
      ids[j] = -1;
      ws[j] = 0.f;
    }
    if (knn.pixel_knn) {
      if (valid) {
#pragma unroll
        for (int j = 0; j < CF_K_NEIGHBORS; ++j) {
          ids[j] = knn.pixel_knn[(size_t)px * CF_K_NEIGHBORS + j];
          ws[j] = knn.pixel_knn_w[(size_t)px * CF_K_NEIGHBORS + j];
        }
      }
    } else if (knn.hit) {
      const int v = knn.hit[px];
      if (v >= 0 && (long long)v < knn.num_voxels) {
#pragma unroll
        for (int j = 0; j < CF_K_NEIGHBORS; ++j) {
          ids[j] = knn.voxel_knn[(size_t)v * CF_K_NEIGHBORS + j];
          ws[j] = knn.voxel_knn_w[(size_t)v * CF_K_NEIGHBORS + j];
        }
      }
      if (knn.pixel_knn_out) {
#pragma unroll
        for (int j = 0; j < CF_K_NEIGHBORS; ++j) {
          knn.pixel_knn_out[(size_t)px * CF_K_NEIGHBORS + j] = ids[j];
          knn.pixel_knn_w_out[(size_t)px * CF_K_NEIGHBORS + j] = ws[j];
        }
      }
    }
    float3 src = make_float3(0.f, 0.f, 0.f), dst = src, nrm = src;
    float weight = 0.f;
    if (valid) {
      const float4 a = A[bi];
      const float2 b = B[bi];
      const float ex = __fsub_rn(p.vc.x, a.x), ey = __fsub_rn(p.vc.y, a.y), ez = __fsub_rn(p.vc.z, a.z);
      const float euclid = __fsqrt_rn(cs_dot(ex, ey, ez, ex, ey, ez));
      const float cosv = fabsf(cs_dot(p.nc.x, p.nc.y, p.nc.z, a.w, b.x, b.y));
      src = p.vl;
      dst = cs_point(k.wc, a.x, a.y, a.z);
      nrm = cs_normalize(cs_normal(k.wc, a.w, b.x, b.y));
      // kernels/tsdf_kernels.cu:510-514
      const float phi_d = fmaxf(0.f, __fsub_rn(1.f, __fdiv_rn(euclid, k.cap)));
      const float phi_n = fmaxf(0.f, __fsub_rn(1.f, __fdiv_rn(__fsub_rn(1.f, cosv), k.normal_eps)));
      const float phi_v = fmaxf(0.f, __fsub_rn(1.f, __fdiv_rn(__fsub_rn(1.f, p.view_cos), k.view_eps)));
      const float c = __fdiv_rn(__fadd_rn(__fadd_rn(phi_d, phi_n), phi_v), 3.f);
      weight = __fmul_rn(c, c);
    } else {
#pragma unroll
      for (int j = 0; j < CF_K_NEIGHBORS; ++j) {
        ids[j] = -1;
        ws[j] = 0.f;
      }
    }
    float* o = stage + lane * kCsRecWords;
    o[0] = src.x; o[1] = src.y; o[2] = src.z;
    o[3] = dst.x; o[4] = dst.y; o[5] = dst.z;
    o[6] = nrm.x; o[7] = nrm.y; o[8] = nrm.z;
#pragma unroll
    for (int j = 0; j < CF_K_NEIGHBORS; ++j) {
      o[9 + j] = __int_as_float(ids[j]);
      o[13 + j] = ws[j];
    }
    o[17] = weight;
    o[18] = __int_as_float(valid ? 1 : 0);  // bool valid + 3 zero pad bytes
  }
  {
    const unsigned mi = __ballot_sync(0xffffffffu, inimg);
    const int px0 = __shfl_sync(0xffffffffu, px, 0);
    __syncwarp();
    if (mi & 1u) {
      float* dst = reinterpret_cast<float*>(out + px0);
      const int words = __popc(mi) * kCsRecWords;
      for (int w = lane; w < words; w += 32) dst[w] = stage[w];
    }
    __syncwarp();
  }
  const unsigned mv = __ballot_sync(0xffffffffu, valid);
  if (lane == 0 && mv) atomicAdd(num_valid, __popc(mv));
  if (stats) {
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const unsigned m = __ballot_sync(0xffffffffu, code == c);
      if (lane == 0 && m) atomicAdd(stats + c, __popc(m));
    }
  }
}

// One thread per vertically adjacent pixel pair, 32 x 16 pixels per CTA.
// kDirect: one chunk covers every row, and the kernel resolves each pixel and
// writes its record itself (no partials, no merge launch).
template <bool kAngle, bool kDirect>
__global__ void __launch_bounds__(kCsThreads, kCsCtasPerSm)
    corr_search_kernel(const CorrConsts k, const float* __restrict__ lv, const float* __restrict__ ln,
                       const float4* __restrict__ A, const float2* __restrict__ B, const int* __restrict__ flag,
                       float* __restrict__ part_pd, int* __restrict__ part_idx, const KnnSrc knn,
                       cf_correspondence* __restrict__ out, int* __restrict__ num_valid, int* __restrict__ stats) {
  extern __shared__ float4 cs_smem[];
  __shared__ int s_box[4];  // min pu, max pu, min pv, max pv of the pixels scanned here
  __shared__ float s_bb[kCsThreads / 32][6];  // per warp: the band's real-point box (min xyz, max xyz)
  const int tid = threadIdx.y * kCsTx + threadIdx.x;
  const int x = blockIdx.x * kCsTx + threadIdx.x;
  const int y0 = blockIdx.y * kCsPy + 2 * threadIdx.y, y1 = y0 + 1;
  const int chunk = blockIdx.z;
  const bool img0 = x < k.W && y0 < k.H, img1 = x < k.W && y1 < k.H;
  const int px0 = img0 ? y0 * k.W + x : 0, px1 = img1 ? y1 * k.W + x : 0;
  if (tid == 0) {
    s_box[0] = INT_MAX;
    s_box[1] = INT_MIN;
    s_box[2] = INT_MAX;
    s_box[3] = INT_MIN;
  }
  const int frame_flag = *flag;
  CsScan q0, q1;
  {
    CsPixel p;
    p.search = false;
    p.special = false;
    p.pu = p.pv = 0;
    p.vc = p.nc = make_float3(0.f, 0.f, 0.f);
    if (img0) p = cs_pixel(k, lv, ln, px0, frame_flag);
    q0 = cs_scan_state(p, img0 && p.search && !p.special, k.dist_thr);
    p.search = false;
    p.special = false;
    p.pu = p.pv = 0;
    if (img1) p = cs_pixel(k, lv, ln, px1, frame_flag);
    q1 = cs_scan_state(p, img1 && p.search && !p.special, k.dist_thr);
  }
  __syncthreads();
  if (q0.on) {
    atomicMin(&s_box[0], q0.pu);
    atomicMax(&s_box[1], q0.pu);
    atomicMin(&s_box[2], q0.pv);
    atomicMax(&s_box[3], q0.pv);
  }
  if (q1.on) {
    atomicMin(&s_box[0], q1.pu);
    atomicMax(&s_box[1], q1.pu);
    atomicMin(&s_box[2], q1.pv);
    atomicMax(&s_box[3], q1.pv);
  }
  __syncthreads();

  if (s_box[0] <= s_box[1]) {  // uniform over the CTA
    const int r = k.radius;
    const int xlo = max(0, s_box[0] - r), xhi = min(k.W - 1, s_box[1] + r);
    const int ylo = max(0, s_box[2] - r), yhi = min(k.H - 1, s_box[3] + r);
    const int per = (yhi - ylo + k.chunks) / k.chunks;  // ceil(rows / chunks)
    const int c0 = ylo + chunk * per, c1 = min(yhi, c0 + per - 1);
    const int wu = xhi - xlo + 1;
    const int band = kCsSmem / (kCsRecBytes * wu);
    // rows either pixel's window covers
    const int plo = min(q0.on ? q0.pv : INT_MAX, q1.on ? q1.pv : INT_MAX) - r;
    const int phi = max(q0.on ? q0.pv : INT_MIN, q1.on ? q1.pv : INT_MIN) + r;
    const bool any = q0.on || q1.on;
    if (c0 <= c1 && band >= 1) {
      float4* sA = cs_smem;
      float2* sB = reinterpret_cast<float2*>(cs_smem + (size_t)band * wu);
      for (int yb = c0; yb <= c1; yb += band) {
        const int rows = min(band, c1 - yb + 1);
        // the band's records, and the bounding box of their real points
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int j = tid; j < rows * wu; j += kCsThreads) {
          const int rr = j / wu;
          const int g = (yb + rr) * k.W + xlo + (j - rr * wu);
          const float4 a = A[g];
          sA[j] = a;
          sB[j] = B[g];
          if (a.z > 0.f) {
            lo[0] = fminf(lo[0], a.x);
            lo[1] = fminf(lo[1], a.y);
            lo[2] = fminf(lo[2], a.z);
            hi[0] = fmaxf(hi[0], a.x);
            hi[1] = fmaxf(hi[1], a.y);
            hi[2] = fmaxf(hi[2], a.z);
          }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c)
          for (int o = 16; o; o >>= 1) {
            lo[c] = fminf(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
            hi[c] = fmaxf(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
          }
        if ((tid & 31) == 0)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            s_bb[tid >> 5][c] = lo[c];
            s_bb[tid >> 5][3 + c] = hi[c];
          }
        __syncthreads();
        if (any) {
#pragma unroll
          for (int w = 0; w < kCsThreads / 32; ++w)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              lo[c] = fminf(lo[c], s_bb[w][c]);
              hi[c] = fmaxf(hi[c], s_bb[w][3 + c]);
            }
          const int ya = max(yb, plo), yz = min(yb + rows - 1, phi);
          if (cs_within_cap(q0, lo, hi, k.s_max) && cs_within_cap(q1, lo, hi, k.s_max)) {
            for (int yy = ya; yy <= yz; ++yy) {
              const int o = (yy - yb) * wu - xlo;
              cs_pair_row<kAngle, false>(sA + o, sB + o, yy, q0, q1, k);
            }
          } else {
            for (int yy = ya; yy <= yz; ++yy) {
              const int o = (yy - yb) * wu - xlo;
              cs_pair_row<kAngle, true>(sA + o, sB + o, yy, q0, q1, k);
            }
          }
        }
        __syncthreads();
      }
    } else if (c0 <= c1 && any) {  // the union is wider than a band buffer row: read through L1
      const int ya = max(c0, plo), yz = min(c1, phi);
      for (int yy = ya; yy <= yz; ++yy)
        cs_pair_row<kAngle, true>(A + (size_t)yy * k.W, B + (size_t)yy * k.W, yy, q0, q1, k);
    }
  }
  cs_resolve<kAngle>(q0, A, B, k);
  cs_resolve<kAngle>(q1, A, B, k);
  if (kDirect) {
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      const bool img = h == 0 ? img0 : img1;
      const int px = h == 0 ? px0 : px1;
      const int best_i = h == 0 ? q0.bi : q1.bi;
      CsPixel p;
      p.search = false;
      p.code = -1;
      if (img) p = cs_pixel(k, lv, ln, px, frame_flag);
      int code = p.code;
      int bi = -1;
      if (p.search) {
        bool saw_depth = false;
        if (p.special) {
          bi = cs_rescan(k, p, A, B, saw_depth);
        } else {
          bi = best_i;
          if (bi < 0 && stats) saw_depth = cs_any_depth(k, p, A);
        }
        code = bi >= 0 ? 5 : (saw_depth ? 3 : 2);
      }
      // the band buffer is free once every band is scanned: stage the records there
      cs_emit(k, p, img, px, bi, code, A, B, knn, out, num_valid, stats, threadIdx.x,
              reinterpret_cast<float*>(cs_smem) + threadIdx.y * (32 * kCsRecWords));
    }
  } else {
    if (img0) {
      part_pd[(size_t)chunk * k.P + px0] = q0.best;
      part_idx[(size_t)chunk * k.P + px0] = q0.bi;
    }
    if (img1) {
      part_pd[(size_t)chunk * k.P + px1] = q1.best;
      part_idx[(size_t)chunk * k.P + px1] = q1.bi;
    }
  }
}

__global__ void __launch_bounds__(256)
    corr_merge_kernel(const CorrConsts k, const float* __restrict__ lv, const float* __restrict__ ln,
                      const float4* __restrict__ A, const float2* __restrict__ B, const int* __restrict__ flag,
                      const float* __restrict__ part_pd, const int* __restrict__ part_idx, const KnnSrc knn,
                      cf_correspondence* __restrict__ out, int* __restrict__ num_valid, int* __restrict__ stats) {
  __shared__ float s_stage[256 / 32][32 * kCsRecWords];
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const bool inimg = px < k.P;
  CsPixel p;
  p.search = false;
  p.code = -1;
  if (inimg) p = cs_pixel(k, lv, ln, px, *flag);
  int code = p.code;
  int bi = -1;
  if (p.search) {
    bool saw_depth = false;
    if (p.special) {
      bi = cs_rescan(k, p, A, B, saw_depth);
    } else {
      float best = k.dist_thr;
      for (int c = 0; c < k.chunks; ++c) {
        const int i = part_idx[(size_t)c * k.P + px];
        const float pd = part_pd[(size_t)c * k.P + px];
        if (i >= 0 && pd < best) {
          best = pd;
          bi = i;
        }
      }
      if (bi < 0 && stats) saw_depth = cs_any_depth(k, p, A);
    }
    code = bi >= 0 ? 5 : (saw_depth ? 3 : 2);
  }
  cs_emit(k, p, inimg, px, bi, code, A, B, knn, out, num_valid, stats, threadIdx.x & 31, s_stage[threadIdx.x >> 5]);
}

__global__ void pixel_knn_kernel(const int* __restrict__ hit, int P, const int* __restrict__ vk,
                                 const float* __restrict__ vw, long long num_voxels, int* __restrict__ pk,
                                 float* __restrict__ pw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const int v = hit[i];
  const bool ok = v >= 0 && (long long)v < num_voxels;
#pragma unroll
  for (int j = 0; j < CF_K_NEIGHBORS; ++j) {
    pk[(size_t)i * CF_K_NEIGHBORS + j] = ok ? vk[(size_t)v * CF_K_NEIGHBORS + j] : -1;
    pw[(size_t)i * CF_K_NEIGHBORS + j] = ok ? vw[(size_t)v * CF_K_NEIGHBORS + j] : 0.f;
  }
}

// Largest float s with sqrtf(s) <= cap (IEEE square roots on both sides), so
// that sqrtf(s) > cap exactly when s > bound.
float sqrt_bound(float cap) {
  if (std::isnan(cap)) return NAN;  // sqrtf(s) > NaN never holds; neither does s > NaN
  if (cap < 0.f) return -INFINITY;
  if (std::isinf(cap)) return INFINITY;
  float s = cap * cap;
  if (std::isinf(s)) s = FLT_MAX;
  while (s > 0.f && std::sqrt(s) > cap) s = std::nextafter(s, 0.f);
  for (;;) {
    const float up = std::nextafter(s, INFINITY);
    if (std::isinf(up) || !(std::sqrt(up) <= cap)) break;
    s = up;
  }
  return s;
}

}  // namespace

// Row chunks per tile.  Rough model in SM clocks: a CTA scans 512 pixels x
// S/C candidates at about 1.9 candidates per clock (7.5 per SM, 4 CTAs) after
// a fixed ~3000-clock set-up, the CTAs run in ceil(tiles x C / slots) waves,
// and more than one chunk adds the merge launch (~20000 clocks).  One chunk
// writes the records from the search kernel itself.
int corr_pick_chunks(int tiles, int sms, int radius, int W, int H) {
  const double slots = (double)(sms > 0 ? sms : 1) * kCsCtasPerSm;
  const double side_x = std::fmin(2.0 * radius + 1.0, (double)W), side_y = std::fmin(2.0 * radius + 1.0, (double)H);
  const double scan = 512.0 * side_x * side_y / 1.9;
  int best_c = 1;
  double best = 1e300;
  for (int c = 1; c <= kCorrMaxChunks; ++c) {
    const double t = std::ceil((double)tiles * c / slots) * (3000.0 + scan / c) + (c > 1 ? 20000.0 : 0.0);
    if (t < best * (1.0 - 1e-9)) {
      best = t;
      best_c = c;
    }
  }
  return best_c;
}

cudaError_t launch_corr_search(const cf_corr_frame* f, const cf_camera* cam, const cf_mat4* Tcw, const cf_mat4* Twc,
                               const cf_corr_params* p, const CorrScratch& sc, int chunks, cf_correspondence* out,
                               int* num_valid, int* stats, cudaStream_t s, long long* launches) {
  cudaError_t e = cudaSuccess;
  const int W = cam->width, H = cam->height;
  CorrConsts k;
  k.fx = cam->fx;
  k.fy = cam->fy;
  k.cx = cam->cx;
  k.cy = cam->cy;
  k.W = W;
  k.H = H;
  k.P = W * H;
  // a window wider than the image reads the same pixels as the image itself
  const int span = W > H ? W : H;
  k.radius = p->search_radius_px < 0 ? 0 : (p->search_radius_px > span ? span : p->search_radius_px);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 4; ++c) {
      k.cw[4 * r + c] = Tcw->m[r][c];
      k.wc[4 * r + c] = Twc->m[r][c];
    }
  k.dist_thr = p->dist_threshold;
  k.angle_thr = p->angle_threshold;
  k.view_thr = p->view_threshold;
  // kernels/tsdf_kernels.cu:456-458
  const float d3 = 3.0f * p->dist_threshold, d2 = p->dist_threshold + 0.03f;
  k.cap = std::fmax(d3, d2);
  const float ne = 1.0f - p->angle_threshold, ve = 1.0f - p->view_threshold;
  k.normal_eps = std::fmax(ne, 1e-4f);
  k.view_eps = std::fmax(ve, 1e-4f);
  k.s_max = sqrt_bound(k.cap);

  KnnSrc knn;
  knn.pixel_knn = f->d_pixel_knn;
  knn.pixel_knn_w = f->d_pixel_knn_w;
  knn.hit = f->d_pixel_knn ? nullptr : f->d_hit_voxel_idx;
  knn.voxel_knn = f->d_voxel_knn;
  knn.voxel_knn_w = f->d_voxel_knn_w;
  knn.num_voxels = f->d_voxel_knn ? f->num_voxels : 0;
  knn.pixel_knn_out = f->d_pixel_knn ? nullptr : f->d_pixel_knn_out;
  knn.pixel_knn_w_out = f->d_pixel_knn ? nullptr : f->d_pixel_knn_w_out;

  e = cudaMemsetAsync(num_valid, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  if (stats) {
    e = cudaMemsetAsync(stats, 0, 6 * sizeof(int), s);
    if (e != cudaSuccess) return e;
  }
  if (W == 0 || H == 0) return cudaSuccess;
  // a NaN bound defeats the strict-less rule (the reference then accepts every
  // candidate it reaches) and an infinite one lets a skip record pass the
  // Euclidean test: such calls take the sequential scan throughout
  e = cudaMemsetAsync(sc.flag, std::isfinite(p->dist_threshold) ? 0 : 1, sizeof(int), s);
  if (e != cudaSuccess) return e;

  const dim3 tiles((W + kCsTx - 1) / kCsTx, (H + kCsPy - 1) / kCsPy);
  // the partials hold kCorrMaxChunks entries per pixel of the largest frame
  k.chunks = chunks > 0 ? (chunks > kCorrMaxChunks ? kCorrMaxChunks : chunks)
                        : corr_pick_chunks((int)(tiles.x * tiles.y), sc.sms, k.radius, W, H);
  const bool angle = p->angle_threshold > 0.f, direct = k.chunks == 1;
  auto kern = angle ? (direct ? corr_search_kernel<true, true> : corr_search_kernel<true, false>)
                    : (direct ? corr_search_kernel<false, true> : corr_search_kernel<false, false>);
  // per device and cheap: set on every call rather than cached per device
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kCsSmem);
  if (e != cudaSuccess) return e;

  corr_prep_kernel<<<(k.P + 255) / 256, 256, 0, s>>>(f->d_depth, f->d_depth_normals, W, H, k.fx, k.fy, k.cx, k.cy,
                                                      sc.A, sc.B, sc.flag);
  const dim3 grid(tiles.x, tiles.y, k.chunks);
  kern<<<grid, dim3(kCsTx, kCsTy), kCsSmem, s>>>(k, f->d_live_vertices, f->d_live_normals, sc.A, sc.B, sc.flag,
                                                 sc.part_pd, sc.part_idx, knn, out, num_valid, stats);
  *launches += 2;
  if (!direct) {
    corr_merge_kernel<<<(k.P + 255) / 256, 256, 0, s>>>(k, f->d_live_vertices, f->d_live_normals, sc.A, sc.B,
                                                        sc.flag, sc.part_pd, sc.part_idx, knn, out, num_valid, stats);
    *launches += 1;
  }
  return cudaGetLastError();
}

cudaError_t launch_pixel_knn(const int* hit, int P, const int* vk, const float* vw, long long num_voxels, int* pk,
                             float* pw, cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  pixel_knn_kernel<<<(P + 255) / 256, 256, 0, s>>>(hit, P, vk, vw, num_voxels, pk, pw);
  return cudaGetLastError();
}

}  // namespace cf
