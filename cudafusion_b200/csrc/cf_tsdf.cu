// cf_tsdf.cu — warped TSDF integration: the step after the solve that fuses
// the frame's depth into the canonical volume through the updated warp.
//
// Restates TSDFVolume::integrate (src/tsdf_volume.cu:23-60) with
// tsdf_integrate_kernel (kernels/tsdf_kernels.cu:85-174), and the gate's
// bookkeeping DynamicFusionPipeline::mark_optimized_voxels
// (include/fusion_app.h:1321-1328) with mark_optimized_voxels_kernel
// (kernels/tsdf_kernels.cu:606-650).
//
// Per voxel: the centre origin + (v + 0.5) voxel_size; when warping, a voxel
// whose optimisation count is below the minimum is left alone, and the centre
// is warped by its voxel's CF_K_NEIGHBORS nodes (warp_point,
// include/se3_math.cuh:450-510); the point is moved into the camera, projected
// and rounded to a pixel; a pixel with depth d > 0 gives sdf = d - z, which is
// dropped below -truncation and else truncated to min(1, sdf / truncation);
// the voxel's weight decays by decay_alpha before the observation of weight 1
// is averaged in, and is capped at max_weight.
//
// Layout: the volume is the reference's array of 12-byte voxels (tsdf,
// weight, colour, pad), x fastest.  Gated and warped (the pipeline's case),
// persistent warps stream the counts 256 voxels at a time and queue the few
// voxels past the gate, updating them 32 at a time (tsdf_gated_kernel);
// otherwise one thread per voxel in index order, so a warp reads 32
// consecutive kNN lists (2 x 512 B, one 16-byte load each) and voxels (384 B)
// and writes back only tsdf and weight.
// The streams read once use evict-first loads; the depth map (1.2 MB at
// 640x480) and the nodes stay in L2.  Each node's plain dual quaternion
// (dq_centered) is computed once per call by tsdf_plain_kernel instead of once
// per (voxel, neighbour), which the reference does.
//
// Arithmetic: the centre is fmaf(v + 0.5, voxel_size, origin); its warp
// (ts_warp) rounds every operation explicitly, shared by the integration and
// the centres entry point; the rigid
// transform's rows are three-term fused sums plus the translation; the
// projection, the sdf, its quotient and the averaged tsdf are IEEE-rounded,
// the averaged numerator is fmaf(tsdf, decayed, observation).  The CPU oracle
// performs the same operations.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>

#include "cf_device.cuh"
#include "cf_internal.h"

namespace cf {

namespace {

constexpr int kTsThreads = 256;

struct TsdfConsts {
  int dx, dy, dz;
  float ox, oy, oz, vs, trunc;
  float fx, fy, cx, cy;
  int W, H;
  float cw[12];  // rows 0..2 of T_cam_world
  float alpha, max_w;
  int min_opt;
};

__device__ __forceinline__ float ts_dot(float ax, float ay, float az, float bx, float by, float bz) {
  return fmaf(az, bz, fmaf(ay, by, __fmul_rn(ax, bx)));
}

// The centre of voxel i (kernels/tsdf_kernels.cu:117-121).
__device__ __forceinline__ float3 ts_centre(const TsdfConsts& k, unsigned i) {
  const unsigned plane = (unsigned)k.dx * (unsigned)k.dy;
  const unsigned z = i / plane, r = i - z * plane;
  const unsigned y = r / (unsigned)k.dx, x = r - y * (unsigned)k.dx;
  return make_float3(fmaf(__fadd_rn((float)x, 0.5f), k.vs, k.ox), fmaf(__fadd_rn((float)y, 0.5f), k.vs, k.oy),
                     fmaf(__fadd_rn((float)z, 0.5f), k.vs, k.oz));
}

__global__ void tsdf_plain_kernel(const cf_deform_node* __restrict__ nodes, const cf_dual_quat* __restrict__ T,
                                  cf_dual_quat* __restrict__ plain, int N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) store_dq(plain + i, dq_centered(load_dq_cg(T + i), node_pos(nodes, i)));
}

// The voxel centre's warp (warp_point, include/se3_math.cuh:450-510, over the
// nodes' plain dual quaternions) with every operation rounded explicitly:
// sums of products accumulate left to right by fused multiply-adds, square
// root and quotients are IEEE.  The integration and the centres entry point
// share it, so they compute the same bits whichever kernel inlines it.
__device__ __forceinline__ float ts_qdot(float4 a, float4 b) {
  return fmaf(a.w, b.w, fmaf(a.z, b.z, fmaf(a.y, b.y, __fmul_rn(a.x, b.x))));
}
__device__ __forceinline__ float4 ts_qmul(float4 a, float4 b) {
  return make_float4(fmaf(-a.z, b.y, fmaf(a.y, b.z, fmaf(a.x, b.w, __fmul_rn(a.w, b.x)))),
                     fmaf(a.z, b.x, fmaf(a.y, b.w, fmaf(-a.x, b.z, __fmul_rn(a.w, b.y)))),
                     fmaf(a.z, b.w, fmaf(-a.y, b.x, fmaf(a.x, b.y, __fmul_rn(a.w, b.z)))),
                     fmaf(-a.z, b.z, fmaf(-a.y, b.y, fmaf(-a.x, b.x, __fmul_rn(a.w, b.w)))));
}
__device__ __forceinline__ float3 ts_warp(float3 p, int4 ids, float4 ws, const cf_dual_quat* __restrict__ plain,
                                          int N) {
  float4 br = make_float4(0.f, 0.f, 0.f, 0.f), bd = br;
  float wsum = 0.f;
  const int idv[4] = {ids.x, ids.y, ids.z, ids.w};
  const float wv[4] = {ws.x, ws.y, ws.z, ws.w};
#pragma unroll
  for (int k = 0; k < kK; k++) {
    const int nid = idv[k];
    const float w = wv[k];
    if (nid < 0 || nid >= N || w < 1e-8f) continue;
    DQ d = load_dq_ldg(plain + nid);  // (the plain DQs come from an earlier launch)
    if (ts_qdot(d.r, br) < 0.f) {
      d.r = make_float4(-d.r.x, -d.r.y, -d.r.z, -d.r.w);
      d.d = make_float4(-d.d.x, -d.d.y, -d.d.z, -d.d.w);
    }
    br = make_float4(fmaf(w, d.r.x, br.x), fmaf(w, d.r.y, br.y), fmaf(w, d.r.z, br.z), fmaf(w, d.r.w, br.w));
    bd = make_float4(fmaf(w, d.d.x, bd.x), fmaf(w, d.d.y, bd.y), fmaf(w, d.d.z, bd.z), fmaf(w, d.d.w, bd.w));
    wsum = __fadd_rn(wsum, w);
  }
  if (wsum < 1e-8f) return p;
  const float n = __fsqrt_rn(ts_qdot(br, br));
  if (n < 1e-12f) return p;  // the identity transform
  const float inv = __fdiv_rn(1.f, n);
  const float4 r = make_float4(__fmul_rn(br.x, inv), __fmul_rn(br.y, inv), __fmul_rn(br.z, inv), __fmul_rn(br.w, inv));
  const float4 dd = make_float4(__fmul_rn(bd.x, inv), __fmul_rn(bd.y, inv), __fmul_rn(bd.z, inv), __fmul_rn(bd.w, inv));
  const float4 rc = make_float4(-r.x, -r.y, -r.z, r.w);
  const float4 rp = ts_qmul(ts_qmul(r, make_float4(p.x, p.y, p.z, 0.f)), rc);
  const float4 t = ts_qmul(dd, rc);
  return make_float3(__fadd_rn(rp.x, __fmul_rn(2.f, t.x)), __fadd_rn(rp.y, __fmul_rn(2.f, t.y)),
                     __fadd_rn(rp.z, __fmul_rn(2.f, t.z)));
}

// One voxel's update (kernels/tsdf_kernels.cu:117-173) once it is past the
// gate: centre, warp, camera, pixel, sdf, weighted average.
template <bool kWarp>
__device__ __forceinline__ void ts_update(const TsdfConsts& k, float* __restrict__ vox, unsigned i,
                                          const float* __restrict__ depth, const int4* __restrict__ knn,
                                          const float4* __restrict__ knn_w, const cf_dual_quat* __restrict__ plain,
                                          int N) {
  float3 p = ts_centre(k, i);
  if (kWarp) p = ts_warp(p, __ldcs(knn + i), __ldcs(knn_w + i), plain, N);
  const float* r = k.cw;
  const float cxp = __fadd_rn(ts_dot(r[0], r[1], r[2], p.x, p.y, p.z), r[3]);
  const float cyp = __fadd_rn(ts_dot(r[4], r[5], r[6], p.x, p.y, p.z), r[7]);
  const float czp = __fadd_rn(ts_dot(r[8], r[9], r[10], p.x, p.y, p.z), r[11]);
  if (czp <= 0.f) return;
  // CameraIntrinsics::project (include/types.h:152-155), then __float2int_rn
  const int u = __float2int_rn(__fadd_rn(__fdiv_rn(__fmul_rn(k.fx, cxp), czp), k.cx));
  const int v = __float2int_rn(__fadd_rn(__fdiv_rn(__fmul_rn(k.fy, cyp), czp), k.cy));
  if (u < 0 || u >= k.W || v < 0 || v >= k.H) return;
  const float d = __ldg(depth + (size_t)v * k.W + u);
  if (d <= 0.f) return;
  const float sdf = __fsub_rn(d, czp);
  if (sdf < -k.trunc) return;
  const float obs = fminf(1.f, __fdiv_rn(sdf, k.trunc));
  float* cell = vox + 3 * (size_t)i;
  const float t_old = __ldcs(cell), w_old = __ldcs(cell + 1);
  const float decayed = __fmul_rn(w_old, k.alpha);
  const float new_w = __fadd_rn(decayed, 1.f);
  __stcs(cell, __fdiv_rn(fmaf(t_old, decayed, obs), new_w));
  __stcs(cell + 1, fminf(new_w, k.max_w));
}

// Every voxel, one thread each (no gate, or a count array that is not
// 16-byte aligned).
template <bool kWarp, bool kGate>
__global__ void __launch_bounds__(kTsThreads)
    tsdf_integrate_kernel(const TsdfConsts k, float* __restrict__ vox, unsigned V, const float* __restrict__ depth,
                          const int4* __restrict__ knn, const float4* __restrict__ knn_w,
                          const cf_dual_quat* __restrict__ plain, int N, const int* __restrict__ counts) {
  const unsigned i = blockIdx.x * kTsThreads + threadIdx.x;
  if (i >= V) return;
  if (kGate && __ldcs(counts + i) < k.min_opt) return;
  ts_update<kWarp>(k, vox, i, depth, knn, knn_w, plain, N);
}

// The gated warp (the stock pipeline's case: a few per cent of the voxels
// pass).  Persistent warps stream the counts in tiles of 256 voxels (two
// 16-byte loads per lane, the next tile's issued before the current tile is
// worked), keep the voxels past the gate in a per-warp queue in shared memory
// (a warp scan of the lanes' counts of passing voxels) and update the queue
// 32 voxels at a time, one per lane, so that the count stream keeps enough
// bytes in flight and no lane idles on a gated voxel.  Each voxel's update is
// ts_update's, so the values equal the one-thread-per-voxel kernel's.
constexpr int kTsTile = 256, kTsQueue = 32 + kTsTile;
__device__ __forceinline__ void ts_load_counts(const int* __restrict__ counts, unsigned V, unsigned tile, int lane,
                                               int4 (&c)[2]) {
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const unsigned base = tile * kTsTile + h * 128 + 4 * lane;
    if (base + 4 <= V) {
      c[h] = __ldcs(reinterpret_cast<const int4*>(counts + base));
    } else {
      c[h].x = base < V ? __ldcs(counts + base) : INT_MIN;
      c[h].y = base + 1 < V ? __ldcs(counts + base + 1) : INT_MIN;
      c[h].z = base + 2 < V ? __ldcs(counts + base + 2) : INT_MIN;
      c[h].w = base + 3 < V ? __ldcs(counts + base + 3) : INT_MIN;
    }
  }
}

__global__ void __launch_bounds__(kTsThreads)
    tsdf_gated_kernel(const TsdfConsts k, float* __restrict__ vox, unsigned V, const float* __restrict__ depth,
                      const int4* __restrict__ knn, const float4* __restrict__ knn_w,
                      const cf_dual_quat* __restrict__ plain, int N, const int* __restrict__ counts) {
  __shared__ unsigned s_queue[kTsThreads / 32][kTsQueue];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  unsigned* q = s_queue[wl];
  const unsigned nwarps = gridDim.x * (kTsThreads / 32);
  const unsigned tiles = (V + kTsTile - 1) / kTsTile;
  unsigned tile = blockIdx.x * (kTsThreads / 32) + wl;
  int qlen = 0;  // uniform in the warp
  int4 cur[2];
  if (tile < tiles) ts_load_counts(counts, V, tile, lane, cur);
  for (; tile < tiles; tile += nwarps) {
    int4 nxt[2];
    if (tile + nwarps < tiles) ts_load_counts(counts, V, tile + nwarps, lane, nxt);
    // this lane's passing voxels: 8 bits, voxel (h * 128 + 4 * lane + j)
    unsigned bits = 0;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      bits |= (unsigned)(cur[h].x >= k.min_opt) << (4 * h);
      bits |= (unsigned)(cur[h].y >= k.min_opt) << (4 * h + 1);
      bits |= (unsigned)(cur[h].z >= k.min_opt) << (4 * h + 2);
      bits |= (unsigned)(cur[h].w >= k.min_opt) << (4 * h + 3);
    }
    const int n = __popc(bits);
    int incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int x = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += x;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    int at = qlen + incl - n;
    while (bits) {
      const int j = __ffs(bits) - 1;
      bits &= bits - 1;
      const unsigned i = tile * kTsTile + (j >> 2) * 128 + 4 * lane + (j & 3);
      q[at++] = i;
    }
    qlen += total;
    __syncwarp();
    while (qlen >= 32) {
      qlen -= 32;
      ts_update<true>(k, vox, q[qlen + lane], depth, knn, knn_w, plain, N);
    }
    __syncwarp();
    if (tile + nwarps < tiles) {
      cur[0] = nxt[0];
      cur[1] = nxt[1];
    }
  }
  if (lane < qlen) ts_update<true>(k, vox, q[lane], depth, knn, knn_w, plain, N);
}

__global__ void __launch_bounds__(kTsThreads)
    tsdf_centres_kernel(const TsdfConsts k, float* __restrict__ out, unsigned V, const int4* __restrict__ knn,
                        const float4* __restrict__ knn_w, const cf_dual_quat* __restrict__ plain, int N) {
  const unsigned i = blockIdx.x * kTsThreads + threadIdx.x;
  if (i >= V) return;
  float3 p = ts_centre(k, i);
  if (N > 0) p = ts_warp(p, __ldcs(knn + i), __ldcs(knn_w + i), plain, N);
  out[3 * (size_t)i] = p.x;
  out[3 * (size_t)i + 1] = p.y;
  out[3 * (size_t)i + 2] = p.z;
}

// mark_optimized_voxels_kernel: each pixel with a valid, positively weighted
// correspondence and a canonical voxel marks the 3x3x3 voxels around it
// (those inside the grid) as optimised in this frame; a voxel's count rises
// once per frame however many pixels mark it.
__global__ void mark_opt_kernel(const cf_correspondence* __restrict__ corrs, const int* __restrict__ vidx_map,
                                int P, int dx, int dy, int dz, int frame, int* __restrict__ counts,
                                int* __restrict__ frames) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  if (px >= P) return;
  const cf_correspondence& c = corrs[px];
  if (!c.valid || c.weight <= 0.f) return;
  const int vidx = vidx_map[px];
  if (vidx < 0) return;
  const int vx = vidx % dx, vy = (vidx / dx) % dy, vz = vidx / (dx * dy);
  for (int oz = -1; oz <= 1; ++oz) {
    const int z = vz + oz;
    if (z < 0 || z >= dz) continue;
    for (int oy = -1; oy <= 1; ++oy) {
      const int y = vy + oy;
      if (y < 0 || y >= dy) continue;
      for (int ox = -1; ox <= 1; ++ox) {
        const int x = vx + ox;
        if (x < 0 || x >= dx) continue;
        const int n = (z * dy + y) * dx + x;
        if (atomicExch(frames + n, frame) != frame) atomicAdd(counts + n, 1);
      }
    }
  }
}

__global__ void tsdf_init_kernel(cf_tsdf_voxel* __restrict__ vox, unsigned V) {
  const unsigned i = blockIdx.x * kTsThreads + threadIdx.x;
  if (i >= V) return;
  float* f = reinterpret_cast<float*>(vox + i);
  f[0] = 1.f;
  f[1] = 0.f;
  // colour (128, 128, 128) and pad 0, little-endian
  reinterpret_cast<unsigned*>(f)[2] = 0x00808080u;
}

TsdfConsts make_consts(const cf_tsdf_params* p, const cf_camera* cam, const float* cw, int min_opt) {
  TsdfConsts k;
  k.dx = p->dims[0];
  k.dy = p->dims[1];
  k.dz = p->dims[2];
  k.ox = p->origin[0];
  k.oy = p->origin[1];
  k.oz = p->origin[2];
  k.vs = p->voxel_size;
  k.trunc = p->truncation;
  k.alpha = p->decay_alpha;
  k.max_w = p->max_weight;
  k.min_opt = min_opt;
  if (cam) {
    k.fx = cam->fx;
    k.fy = cam->fy;
    k.cx = cam->cx;
    k.cy = cam->cy;
    k.W = cam->width;
    k.H = cam->height;
  } else {
    k.fx = k.fy = k.cx = k.cy = 0.f;
    k.W = k.H = 0;
  }
  for (int j = 0; j < 12; ++j) k.cw[j] = cw ? cw[j] : 0.f;
  return k;
}

unsigned blocks_of(unsigned V) { return (V + kTsThreads - 1) / kTsThreads; }

}  // namespace

cudaError_t launch_tsdf_plain(const cf_deform_node* nodes, const cf_dual_quat* T, cf_dual_quat* plain, int N,
                              cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  tsdf_plain_kernel<<<(N + 127) / 128, 128, 0, s>>>(nodes, T, plain, N);
  return cudaGetLastError();
}

cudaError_t launch_tsdf_integrate(float* vox, const cf_tsdf_params* p, const float* depth, const cf_camera* cam,
                                  const float* cw, const int* knn, const float* knn_w, const cf_dual_quat* plain,
                                  int N, const int* counts, int min_opt, cudaStream_t s) {
  const unsigned V = (unsigned)p->dims[0] * (unsigned)p->dims[1] * (unsigned)p->dims[2];
  if (V == 0) return cudaSuccess;
  const TsdfConsts k = make_consts(p, cam, cw, min_opt);
  const int4* kn = reinterpret_cast<const int4*>(knn);
  const float4* kw = reinterpret_cast<const float4*>(knn_w);
  const bool warp = plain != nullptr && N > 0;
  if (warp && counts && (reinterpret_cast<uintptr_t>(counts) & 15u) == 0) {
    // persistent: as many CTAs as are resident at once, fewer when the volume
    // has fewer tiles
    static unsigned resident = 0;
    if (resident == 0) {
      int dev = 0, sms = 148, per_sm = 1;
      if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tsdf_gated_kernel, kTsThreads, 0) != cudaSuccess ||
          per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
      }
      resident = (unsigned)(sms * per_sm);
    }
    const unsigned tiles = (V + kTsTile - 1) / kTsTile;
    const unsigned ctas = std::min<unsigned>(resident, (tiles + kTsThreads / 32 - 1) / (kTsThreads / 32));
    tsdf_gated_kernel<<<ctas, kTsThreads, 0, s>>>(k, vox, V, depth, kn, kw, plain, N, counts);
  } else if (warp && counts)
    tsdf_integrate_kernel<true, true><<<blocks_of(V), kTsThreads, 0, s>>>(k, vox, V, depth, kn, kw, plain, N, counts);
  else if (warp)
    tsdf_integrate_kernel<true, false><<<blocks_of(V), kTsThreads, 0, s>>>(k, vox, V, depth, kn, kw, plain, N, nullptr);
  else
    tsdf_integrate_kernel<false, false><<<blocks_of(V), kTsThreads, 0, s>>>(k, vox, V, depth, nullptr, nullptr,
                                                                             nullptr, 0, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_tsdf_centres(float* out, const cf_tsdf_params* p, const int* knn, const float* knn_w,
                                const cf_dual_quat* plain, int N, cudaStream_t s) {
  const unsigned V = (unsigned)p->dims[0] * (unsigned)p->dims[1] * (unsigned)p->dims[2];
  if (V == 0) return cudaSuccess;
  const TsdfConsts k = make_consts(p, nullptr, nullptr, 0);
  tsdf_centres_kernel<<<blocks_of(V), kTsThreads, 0, s>>>(k, out, V, reinterpret_cast<const int4*>(knn),
                                                          reinterpret_cast<const float4*>(knn_w), plain, N);
  return cudaGetLastError();
}

cudaError_t launch_mark_optimized(const cf_correspondence* corrs, const int* vidx, int P, const int dims[3],
                                  int frame, int* counts, int* frames, cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  mark_opt_kernel<<<(P + 255) / 256, 256, 0, s>>>(corrs, vidx, P, dims[0], dims[1], dims[2], frame, counts, frames);
  return cudaGetLastError();
}

cudaError_t launch_tsdf_init(cf_tsdf_voxel* vox, unsigned V, cudaStream_t s) {
  if (V == 0) return cudaSuccess;
  tsdf_init_kernel<<<blocks_of(V), kTsThreads, 0, s>>>(vox, V);
  return cudaGetLastError();
}

}  // namespace cf
