// cf_voxelknn.cu — the voxel kNN field: for every voxel of the canonical
// volume that holds data, its CF_K_NEIGHBORS nearest deformation nodes and
// their skinning weights, the field the TSDF integration, the mesh skinning
// and the correspondence search read.
//
// Restates WarpField::compute_voxel_knn (src/warp_field.cu:957-981) with
// compute_voxel_knn_kernel (:299-405).  Per voxel: a voxel whose weight is
// <= 0 gets ids -1 and weights 0; otherwise its centre origin + (v + 0.5)
// voxel_size is compared with the nodes, and the list keeps the 4 smallest
// (squared distance, node index) pairs among the nodes closer than 1e30 (the
// reference's strict-less insertion in index order with its bubble-up yields
// exactly that set and order); each found node weighs exp(-d / (2 r^2)), r =
// max(radius, 1e-6), normalised by the sum when it exceeds 1e-8.
//
// The reference compares every such voxel with every node (N squared
// distances per voxel, nodes re-read from global memory).  Here a persistent
// CTA owns 8x8x8-voxel tiles, with the nodes (position, radius) staged once
// in shared memory.  Per tile, an exact bound prunes the nodes: over the
// axis-aligned box of the tile's voxel centres, the 4th smallest maximum
// squared distance R is an upper bound of every voxel's 4th distance, so only
// nodes whose minimum squared distance to the box is <= R (with a relative
// margin of 1e-4, far above the few ulps of the per-voxel rounding) can be in
// a voxel's list.  Each warp covers a 4x4x2 sub-box and prunes the tile's
// candidates again the same way.  The per-voxel squared distances and the
// (distance, index) comparisons are then exactly the reference's, over the
// candidates only, so the ids are identical whatever order the candidates
// come in.
//
// Arithmetic: the centre is fmaf(v + 0.5, voxel_size, origin) and the squared
// distance fmaf(dz, dz, fmaf(dx, dx, dy * dy)): the reference's device build
// contracts d.x*d.x + d.y*d.y + d.z*d.z that way (of the six nestings, only
// it and an unfused dx^2 + dy^2 reproduce the reference's order on the two
// voxels of the 256^3 benchmark volume where the roundings decide it); the
// weights use expf and IEEE division (the reference's build uses
// --use_fast_math: weights agree to rounding).
//
// Layout: the volume is the reference's array of 12-byte voxels (only the
// weight is read, once, with evict-first loads); the field is int4 ids and
// float4 weights per voxel in index order (x fastest), written with
// streaming stores — 32 of the 44 algorithmic bytes per voxel.
#include <cmath>
#include <cstdint>

#include "cf_device.cuh"
#include "cf_internal.h"

namespace cf {

namespace {

constexpr int kVkThreads = 512;                       // one 8x8x8 tile, a voxel per thread
constexpr int kVkWarps = kVkThreads / 32;
constexpr int kVkWarpCap = 256;                       // a warp's own candidate list
constexpr int kVkSmemNodesMax = 8192;                 // nodes staged in shared memory up to here
constexpr float kVkMargin = 1.0f + 1e-4f;             // relative slack of the pruning bound

struct VkConsts {
  int dx, dy, dz;
  float ox, oy, oz, vs;
  int N;
  int tx, ty;      // tiles along x and y
  unsigned tiles;  // tiles in the volume
};

__device__ __forceinline__ float vk_centre(int v, float vs, float o) { return fmaf(__fadd_rn((float)v, 0.5f), vs, o); }

__device__ __forceinline__ float vk_dist2(float px, float py, float pz, float4 q) {
  const float ex = __fsub_rn(px, q.x), ey = __fsub_rn(py, q.y), ez = __fsub_rn(pz, q.z);
  return fmaf(ez, ez, fmaf(ex, ex, __fmul_rn(ey, ey)));
}

// Minimum and maximum squared distance from q to the box [lo, hi].
__device__ __forceinline__ void vk_box_dist2(float4 q, float3 lo, float3 hi, float& dmin, float& dmax) {
  const float ax = fmaxf(fmaxf(lo.x - q.x, q.x - hi.x), 0.f), bx = fmaxf(fabsf(q.x - lo.x), fabsf(q.x - hi.x));
  const float ay = fmaxf(fmaxf(lo.y - q.y, q.y - hi.y), 0.f), by = fmaxf(fabsf(q.y - lo.y), fabsf(q.y - hi.y));
  const float az = fmaxf(fmaxf(lo.z - q.z, q.z - hi.z), 0.f), bz = fmaxf(fabsf(q.z - lo.z), fabsf(q.z - hi.z));
  dmin = ax * ax + ay * ay + az * az;
  dmax = bx * bx + by * by + bz * bz;
}

// Sorted insert of v into t[0..3] (ascending); NaN never enters.
__device__ __forceinline__ void vk_top4_push(float (&t)[4], float v) {
  if (!(v < t[3])) return;
  t[3] = v;
  if (t[3] < t[2]) { const float s = t[2]; t[2] = t[3]; t[3] = s; }
  if (t[2] < t[1]) { const float s = t[1]; t[1] = t[2]; t[2] = s; }
  if (t[1] < t[0]) { const float s = t[0]; t[0] = t[1]; t[1] = s; }
}

// The 4th smallest value held by the warp's lanes (each lane's t sorted).
__device__ __forceinline__ float vk_warp_4th(float (&t)[4]) {
  float m = 0.f;
  for (int r = 0; r < 4; ++r) {
    m = t[0];
    for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
    const unsigned own = __ballot_sync(0xffffffffu, t[0] == m);
    if (own && lane_id() == __ffs(own) - 1) {
      t[0] = t[1];
      t[1] = t[2];
      t[2] = t[3];
      t[3] = INFINITY;
    }
  }
  return m;  // +inf when the warp held fewer than 4 finite values
}

template <bool kSmemNodes>
__device__ __forceinline__ float4 vk_node(const float4* sn, const cf_deform_node* __restrict__ nodes, int i) {
  if (kSmemNodes) return sn[i];
  const float* p = reinterpret_cast<const float*>(nodes + i);
  return make_float4(__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 6));
}

// Lexicographic (distance, index) insert into the sorted list (bd, bi).
__device__ __forceinline__ void vk_insert(float (&bd)[4], int (&bi)[4], float d, int j) {
  if (!(d < bd[3] || (d == bd[3] && j < bi[3]))) return;
  bd[3] = d;
  bi[3] = j;
#pragma unroll
  for (int k = 2; k >= 0; --k) {
    if (bd[k + 1] < bd[k] || (bd[k + 1] == bd[k] && bi[k + 1] < bi[k])) {
      const float td = bd[k];
      bd[k] = bd[k + 1];
      bd[k + 1] = td;
      const int ti = bi[k];
      bi[k] = bi[k + 1];
      bi[k + 1] = ti;
    }
  }
}

// The warp's voxel-centre box, from its lanes' (in-range) centres.
__device__ __forceinline__ void vk_warp_box(bool in, float px, float py, float pz, float3& lo, float3& hi) {
  float a = in ? px : INFINITY, b = in ? py : INFINITY, c = in ? pz : INFINITY;
  float d = in ? px : -INFINITY, e = in ? py : -INFINITY, f = in ? pz : -INFINITY;
  for (int o = 16; o > 0; o >>= 1) {
    a = fminf(a, __shfl_xor_sync(0xffffffffu, a, o));
    b = fminf(b, __shfl_xor_sync(0xffffffffu, b, o));
    c = fminf(c, __shfl_xor_sync(0xffffffffu, c, o));
    d = fmaxf(d, __shfl_xor_sync(0xffffffffu, d, o));
    e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, o));
    f = fmaxf(f, __shfl_xor_sync(0xffffffffu, f, o));
  }
  lo = make_float3(a, b, c);
  hi = make_float3(d, e, f);
}

template <bool kSmemNodes, bool kWarpPrune>
__global__ void __launch_bounds__(kVkThreads, 3)
    voxel_knn_kernel(const VkConsts k, const float* __restrict__ vox, const cf_deform_node* __restrict__ nodes,
                     int4* __restrict__ out_ids, float4* __restrict__ out_ws) {
  extern __shared__ float4 vk_smem[];
  float4* sn = vk_smem;                                                  // [N] position, radius
  int* cand = reinterpret_cast<int*>(vk_smem + (kSmemNodes ? k.N : 0));  // [N] the tile's candidates
  int* wcand = cand + k.N;                                               // [warps][kVkWarpCap]
  float* sdmin = reinterpret_cast<float*>(wcand + kVkWarps * kVkWarpCap);  // [N] (shared-memory nodes only)
  __shared__ float s_red[kVkWarps][4];
  __shared__ float s_bound;
  __shared__ int s_count;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = k.N;
  if (kSmemNodes) {
    for (int i = tid; i < N; i += kVkThreads) {
      const float* p = reinterpret_cast<const float*>(nodes + i);
      sn[i] = make_float4(__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 6));
    }
  }
  // voxel of this thread within a tile: warp w covers the 4x4x2 sub-box
  // (w & 1, (w >> 1) & 1, w >> 2), lane l its voxel (l & 3, (l >> 2) & 3, l >> 4)
  const int ox = ((warp & 1) << 2) | (lane & 3);
  const int oy = (((warp >> 1) & 1) << 2) | ((lane >> 2) & 3);
  const int oz = ((warp >> 2) << 1) | (lane >> 4);
  // The CTA's tiles are blockIdx.x + j * gridDim.x: their (x, y, z) tile
  // coordinates advance by the grid stride with carries, no division per
  // tile.  This thread's voxel of a tile, and its weight (0 outside the
  // volume); the next tile's weight is loaded ahead, so that its DRAM round
  // trip overlaps the work on the current tile.
  const unsigned tiles_xy = (unsigned)k.tx * (unsigned)k.ty;
  const unsigned G = gridDim.x;
  const uint3 step = make_uint3(G % (unsigned)k.tx, (G / (unsigned)k.tx) % (unsigned)k.ty, G / tiles_xy);
  auto advance = [&](uint3 c) -> uint3 {
    c.x += step.x;
    unsigned cy = step.y;
    if (c.x >= (unsigned)k.tx) {
      c.x -= (unsigned)k.tx;
      ++cy;
    }
    c.y += cy;
    unsigned cz = step.z;
    if (c.y >= (unsigned)k.ty) {
      c.y -= (unsigned)k.ty;
      ++cz;
    }
    c.z += cz;
    return c;
  };
  auto voxel_of = [&](uint3 c, int& x, int& y, int& z) -> bool {
    x = (int)c.x * 8 + ox;
    y = (int)c.y * 8 + oy;
    z = (int)c.z * 8 + oz;
    return x < k.dx && y < k.dy && z < k.dz;  // (a tile past the last has z >= dz)
  };
  auto weight_of = [&](uint3 c) -> float {
    int x, y, z;
    if (!voxel_of(c, x, y, z)) return 0.f;
    return __ldcs(vox + 3 * (((size_t)z * (size_t)k.dy + (size_t)y) * (size_t)k.dx + (size_t)x) + 1);
  };
  uint3 c_cur = make_uint3(blockIdx.x % (unsigned)k.tx, (blockIdx.x / (unsigned)k.tx) % (unsigned)k.ty,
                           blockIdx.x / tiles_xy);
  float w_next = weight_of(c_cur);
  for (unsigned t = blockIdx.x; t < k.tiles; t += G) {
    int x, y, z;
    const bool in = voxel_of(c_cur, x, y, z);
    const unsigned tx = c_cur.x, ty = c_cur.y, tz = c_cur.z;
    const size_t vidx = ((size_t)z * (size_t)k.dy + (size_t)y) * (size_t)k.dx + (size_t)x;
    const float wv = w_next;
    c_cur = advance(c_cur);
    w_next = weight_of(c_cur);
    // src/warp_field.cu:319: only voxels with weight > 0 (a NaN weight is not <= 0)
    const bool active = in && !(wv <= 0.f);
    if (!__syncthreads_or(active)) {
      if (in) {
        __stcs(out_ids + vidx, make_int4(-1, -1, -1, -1));
        __stcs(out_ws + vidx, make_float4(0.f, 0.f, 0.f, 0.f));
      }
      continue;
    }
    const float px = vk_centre(x, k.vs, k.ox), py = vk_centre(y, k.vs, k.oy), pz = vk_centre(z, k.vs, k.oz);
    // the box of the tile's in-range voxel centres (the centre is monotonic
    // in the index for either sign of the voxel size)
    const int xe = min((int)tx * 8 + 7, k.dx - 1), ye = min((int)ty * 8 + 7, k.dy - 1);
    const int ze = min((int)tz * 8 + 7, k.dz - 1);
    const float ax = vk_centre((int)tx * 8, k.vs, k.ox), bx = vk_centre(xe, k.vs, k.ox);
    const float ay = vk_centre((int)ty * 8, k.vs, k.oy), by = vk_centre(ye, k.vs, k.oy);
    const float az = vk_centre((int)tz * 8, k.vs, k.oz), bz = vk_centre(ze, k.vs, k.oz);
    const float3 lo = make_float3(fminf(ax, bx), fminf(ay, by), fminf(az, bz));
    const float3 hi = make_float3(fmaxf(ax, bx), fmaxf(ay, by), fmaxf(az, bz));

    // 1. R = the 4th smallest maximum squared distance to the box: each
    // thread keeps its 4 smallest, each warp pops its 4 smallest into s_red,
    // warp 0 takes the 4th smallest of those
    if (tid == 0) s_count = 0;
    {
      float r4[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
      for (int i = tid; i < N; i += kVkThreads) {
        float dmin, dmax;
        vk_box_dist2(vk_node<kSmemNodes>(sn, nodes, i), lo, hi, dmin, dmax);
        vk_top4_push(r4, dmax);
        if (kSmemNodes) sdmin[i] = dmin;  // read back by the same thread in step 2
      }
      for (int r = 0; r < 4; ++r) {
        float m = r4[0];
        for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
        const unsigned own = __ballot_sync(0xffffffffu, r4[0] == m);
        if (own && lane == __ffs(own) - 1) {
          r4[0] = r4[1];
          r4[1] = r4[2];
          r4[2] = r4[3];
          r4[3] = INFINITY;
        }
        if (lane == 0) s_red[warp][r] = m;
      }
    }
    __syncthreads();
    if (warp == 0) {
      float r4[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
      for (int q = lane; q < kVkWarps * 4; q += 32) vk_top4_push(r4, s_red[q >> 2][q & 3]);
      const float R = vk_warp_4th(r4);
      if (lane == 0) s_bound = R * kVkMargin;
    }
    __syncthreads();
    const float bound = s_bound;

    // 2. the tile's candidates: minimum squared distance to the box <= bound
    for (int base = 0; base < N; base += kVkThreads) {
      const int i = base + tid;
      bool keep = false;
      if (i < N) {
        float dmin = 0.f, dmax;
        if (kSmemNodes)
          dmin = sdmin[i];
        else
          vk_box_dist2(vk_node<kSmemNodes>(sn, nodes, i), lo, hi, dmin, dmax);
        keep = dmin <= bound;
      }
      const unsigned b = __ballot_sync(0xffffffffu, keep);
      int pos = 0;
      if (lane == 0 && b) pos = atomicAdd(&s_count, __popc(b));
      pos = __shfl_sync(0xffffffffu, pos, 0);
      if (keep) cand[pos + __popc(b & lanemask_lt())] = i;
    }
    __syncthreads();
    const int C = s_count;
    const int* list = cand;
    int L = C;

    // 2b. the warp's own candidates over its 4x4x2 sub-box
    if (kWarpPrune && __any_sync(0xffffffffu, active)) {
      float3 wlo, whi;
      vk_warp_box(in, px, py, pz, wlo, whi);
      float r4[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
      for (int c = lane; c < C; c += 32) {
        float dmin, dmax;
        vk_box_dist2(vk_node<kSmemNodes>(sn, nodes, cand[c]), wlo, whi, dmin, dmax);
        vk_top4_push(r4, dmax);
      }
      const float wb = vk_warp_4th(r4) * kVkMargin;
      int* wl = wcand + warp * kVkWarpCap;
      int n = 0;
      for (int c0 = 0; c0 < C; c0 += 32) {
        const int c = c0 + lane;
        bool keep = false;
        int id = 0;
        if (c < C) {
          id = cand[c];
          float dmin, dmax;
          vk_box_dist2(vk_node<kSmemNodes>(sn, nodes, id), wlo, whi, dmin, dmax);
          keep = dmin <= wb;
        }
        const unsigned b = __ballot_sync(0xffffffffu, keep);
        const int at = n + __popc(b & lanemask_lt());
        if (keep && at < kVkWarpCap) wl[at] = id;
        n += __popc(b);
      }
      __syncwarp();
      if (n <= kVkWarpCap) {
        list = wl;
        L = n;
      }
    }

    // 3. the voxel's list over the candidates, then its weights
    if (active) {
      float bd[4] = {1e30f, 1e30f, 1e30f, 1e30f};
      int bi[4] = {-1, -1, -1, -1};
      for (int c = 0; c < L; ++c) {
        const int j = list[c];
        vk_insert(bd, bi, vk_dist2(px, py, pz, vk_node<kSmemNodes>(sn, nodes, j)), j);
      }
      float w[4], sum = 0.f;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        w[q] = 0.f;
        if (bi[q] < 0) continue;
        const float r = fmaxf(vk_node<kSmemNodes>(sn, nodes, bi[q]).w, 1e-6f);
        w[q] = expf(__fdiv_rn(-bd[q], __fmul_rn(__fmul_rn(2.0f, r), r)));
        sum = __fadd_rn(sum, w[q]);
      }
      const float inv = sum > 1e-8f ? __fdiv_rn(1.0f, sum) : 0.0f;
      __stcs(out_ids + vidx, make_int4(bi[0], bi[1], bi[2], bi[3]));
      __stcs(out_ws + vidx, make_float4(__fmul_rn(w[0], inv), __fmul_rn(w[1], inv), __fmul_rn(w[2], inv),
                                        __fmul_rn(w[3], inv)));
    } else if (in) {
      __stcs(out_ids + vidx, make_int4(-1, -1, -1, -1));
      __stcs(out_ws + vidx, make_float4(0.f, 0.f, 0.f, 0.f));
    }
    __syncthreads();  // the candidate lists are rewritten by the next tile
  }
}

template <bool kSmemNodes, bool kWarpPrune>
cudaError_t launch_vk(const VkConsts& k, const float* vox, const cf_deform_node* nodes, int4* ids, float4* ws,
                      cudaStream_t s) {
  auto kern = voxel_knn_kernel<kSmemNodes, kWarpPrune>;
  const size_t smem = (kSmemNodes ? 20 * (size_t)k.N : 0) + 4 * (size_t)k.N + 4 * (size_t)kVkWarps * kVkWarpCap;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kVkThreads, smem)) != cudaSuccess) return e;
  const unsigned grid = (unsigned)std::min<long long>((long long)k.tiles, (long long)std::max(1, per_sm) * sms);
  kern<<<grid, kVkThreads, smem, s>>>(k, vox, nodes, ids, ws);
  return cudaGetLastError();
}

}  // namespace

int voxel_knn_max_nodes() { return 49152; }

cudaError_t launch_voxel_knn(const float* vox, const cf_tsdf_params* p, const cf_deform_node* nodes, int N,
                             int* ids, float* ws, int variant, cudaStream_t s) {
  VkConsts k;
  k.dx = p->dims[0];
  k.dy = p->dims[1];
  k.dz = p->dims[2];
  k.ox = p->origin[0];
  k.oy = p->origin[1];
  k.oz = p->origin[2];
  k.vs = p->voxel_size;
  k.N = N;
  k.tx = (k.dx + 7) / 8;
  k.ty = (k.dy + 7) / 8;
  k.tiles = (unsigned)k.tx * (unsigned)k.ty * (unsigned)((k.dz + 7) / 8);
  int4* oi = reinterpret_cast<int4*>(ids);
  float4* ow = reinterpret_cast<float4*>(ws);
  const bool smem_nodes = N <= kVkSmemNodesMax;
#ifndef CF_VK_WARP_PRUNE
#define CF_VK_WARP_PRUNE 1
#endif
  const bool warp_prune = variant == 0 ? CF_VK_WARP_PRUNE != 0 : variant == 2;
  if (smem_nodes && warp_prune) return launch_vk<true, true>(k, vox, nodes, oi, ow, s);
  if (smem_nodes) return launch_vk<true, false>(k, vox, nodes, oi, ow, s);
  if (warp_prune) return launch_vk<false, true>(k, vox, nodes, oi, ow, s);
  return launch_vk<false, false>(k, vox, nodes, oi, ow, s);
}

}  // namespace cf
