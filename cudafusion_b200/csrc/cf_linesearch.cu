// cf_linesearch.cu — the GN step's acceptance on the device: the increment's
// validation statistics, the scaled and clamped trial increment and the
// correspondence RMSE.
//
// DynamicFusionPipeline runs these on the host after downloading the
// increment (include/fusion_app.h:409-490) and, for each of the line
// search's ten trials, every correspondence record (correspondence_rmse,
// :1331-1350; 23 MB at 640x480).  Here they are reductions over device
// arrays that stay on the stream, so the whole line search is enqueued
// without a host round trip (cf_line_search in cf_api.cu drives it).
#include <cmath>

#include "cf_internal.h"

namespace cf {

namespace {

constexpr int kLsThreads = 256;

__device__ __forceinline__ float ls_norm3(float a, float b, float c) {
  return __fsqrt_rn(fmaf(c, c, fmaf(b, b, __fmul_rn(a, a))));
}

// Per node rn = |dx[0:3]|, tn = |dx[3:6]|; sums in FP64 and maxima of the raw
// and of the scaled-and-clamped values (fusion_app.h:434-458); a non-finite
// rn or tn clears out->finite.  Block partials then atomics: maxima of
// non-negative floats compare as their bit patterns.
__global__ void __launch_bounds__(kLsThreads) update_stats_kernel(const float* __restrict__ dx, int N,
                                                                   float update_scale, float max_rot,
                                                                   float max_trans, double* __restrict__ sums,
                                                                   unsigned* __restrict__ maxima,
                                                                   int* __restrict__ finite) {
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  float m[4] = {0.f, 0.f, 0.f, 0.f};
  bool fin = true;
  for (int i = blockIdx.x * kLsThreads + threadIdx.x; i < N; i += gridDim.x * kLsThreads) {
    const float* d = dx + 6 * (size_t)i;
    const float rn = ls_norm3(d[0], d[1], d[2]), tn = ls_norm3(d[3], d[4], d[5]);
    fin = fin && isfinite(rn) && isfinite(tn);
    float er = __fmul_rn(update_scale, rn), et = __fmul_rn(update_scale, tn);
    if (max_rot > 0.f) er = fminf(er, max_rot);
    if (max_trans > 0.f) et = fminf(et, max_trans);
    s[0] += rn;
    s[1] += tn;
    s[2] += er;
    s[3] += et;
    m[0] = fmaxf(m[0], rn);
    m[1] = fmaxf(m[1], tn);
    m[2] = fmaxf(m[2], er);
    m[3] = fmaxf(m[3], et);
  }
  __shared__ double rs[4][kLsThreads / 32];
  __shared__ float rm[4][kLsThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    double v = s[c];
    float mv = m[c];
    for (int o = 16; o; o >>= 1) {
      v += __shfl_xor_sync(0xffffffffu, v, o);
      mv = fmaxf(mv, __shfl_xor_sync(0xffffffffu, mv, o));
    }
    if (lane == 0) {
      rs[c][w] = v;
      rm[c][w] = mv;
    }
  }
  if (!__all_sync(0xffffffffu, fin) && lane == 0) atomicExch(finite, 0);
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0.0;
    float mv = 0.f;
    for (int j = 0; j < kLsThreads / 32; ++j) {
      v += rs[threadIdx.x][j];
      mv = fmaxf(mv, rm[threadIdx.x][j]);
    }
    atomicAdd(sums + threadIdx.x, v);
    atomicMax(maxima + threadIdx.x, __float_as_uint(mv));
  }
}

// upload_scaled_delta_x (fusion_app.h:1352-1375): per node rs = max_rot / rn
// when rn exceeds a positive max_rot (else 1), ts likewise, then
// dx[k] * (rs * scale) and dx[k] * (ts * scale).
__global__ void scale_delta_kernel(const float* __restrict__ dx, int N, float max_rot, float max_trans, float scale,
                                   float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float* d = dx + 6 * (size_t)i;
  const float rn = ls_norm3(d[0], d[1], d[2]), tn = ls_norm3(d[3], d[4], d[5]);
  float rs = 1.f, ts = 1.f;
  if (max_rot > 0.f && rn > max_rot) rs = __fdiv_rn(max_rot, rn);
  if (max_trans > 0.f && tn > max_trans) ts = __fdiv_rn(max_trans, tn);
  const float fr = __fmul_rn(rs, scale), ft = __fmul_rn(ts, scale);
  float* o = out + 6 * (size_t)i;
#pragma unroll
  for (int k = 0; k < 3; ++k) o[k] = __fmul_rn(d[k], fr);
#pragma unroll
  for (int k = 3; k < 6; ++k) o[k] = __fmul_rn(d[k], ft);
}

// correspondence_rmse's sums (fusion_app.h:1336-1347): block b sums the
// records of its fixed slice in index order per thread and then in thread
// order; rmse_final_kernel adds the blocks in block order.  Deterministic.
__global__ void __launch_bounds__(kLsThreads) rmse_partial_kernel(const cf_correspondence* __restrict__ corrs, int M,
                                                                   double* __restrict__ part) {
  const int per = (M + gridDim.x - 1) / gridDim.x;
  const int lo = blockIdx.x * per, hi = min(M, lo + per);
  double s = 0.0, ws = 0.0;
  for (int c = lo + threadIdx.x; c < hi; c += kLsThreads) {
    const cf_correspondence& r = corrs[c];
    if (!r.valid || !(r.weight > 0.f)) continue;
    const float dx = __fsub_rn(r.src.x, r.dst.x), dy = __fsub_rn(r.src.y, r.dst.y), dz = __fsub_rn(r.src.z, r.dst.z);
    const double e = fma((double)r.normal.z, (double)dz, fma((double)r.normal.y, (double)dy,
                                                              (double)r.normal.x * (double)dx));
    const double w = (double)fmaxf(0.f, r.weight);
    s = fma(w * e, e, s);
    ws += w;
  }
  __shared__ double sh[2][kLsThreads];
  sh[0][threadIdx.x] = s;
  sh[1][threadIdx.x] = ws;
  __syncthreads();
  if (threadIdx.x < 2) {
    double v = 0.0;
    for (int j = 0; j < kLsThreads; ++j) v += sh[threadIdx.x][j];
    part[2 * blockIdx.x + threadIdx.x] = v;
  }
}

// out[0..1] = the block sums in block order; with `valid` also out[2] = the
// search's valid count (the line search keeps each trial's in its slot).
__global__ void rmse_final_kernel(const double* __restrict__ part, int blocks, double* __restrict__ out,
                                  const int* __restrict__ valid) {
  if (threadIdx.x < 2) {
    double v = 0.0;
    for (int b = 0; b < blocks; ++b) v += part[2 * b + threadIdx.x];
    out[threadIdx.x] = v;
  }
  if (threadIdx.x == 2 && valid) out[2] = (double)*valid;
}

// After a trial's RMSE (slot: its sum, wsum and valid count): whether the
// trial is the best so far under the line search's acceptance rule
// (fusion_app.h:575-582, the host's arithmetic: IEEE double quotient and
// square root), chaining the best RMSE from best_in (or best0) to best_out;
// a kept trial's index goes to *kept and its outputs (4-byte words) are
// copied aside, so that the accepted trial need not be predicted and searched
// again.
__global__ void __launch_bounds__(256) ls_keep_kernel(LsKeepArgs a) {
  const double sum = a.slot[0], wsum = a.slot[1];
  const int valid = (int)a.slot[2];
  const double rmse = wsum > 0.0 ? sqrt(sum / wsum) : (double)INFINITY;
  const double best = a.best_in ? *a.best_in : a.best0;
  const bool take = valid >= a.min_valid && valid >= a.need && isfinite(rmse) && rmse < best;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *a.best_out = take ? rmse : best;
    if (take) *a.kept = a.trial;
  }
  if (!take) return;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (int b = 0; b < a.nbuf; ++b) {
    const int* src = a.src[b];
    int* dst = a.dst[b];
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.words[b]; i += stride) dst[i] = src[i];
  }
}

}  // namespace

cudaError_t launch_ls_keep(const LsKeepArgs& a, cudaStream_t s) {
  ls_keep_kernel<<<296, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_update_stats(const float* dx, int N, float update_scale, float max_rot, float max_trans,
                                double* sums, unsigned* maxima, int* finite, cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  int blocks = (N + kLsThreads - 1) / kLsThreads;
  if (blocks > 148) blocks = 148;
  update_stats_kernel<<<blocks, kLsThreads, 0, s>>>(dx, N, update_scale, max_rot, max_trans, sums, maxima, finite);
  return cudaGetLastError();
}

cudaError_t launch_scale_delta(const float* dx, int N, float max_rot, float max_trans, float scale, float* out,
                               cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  scale_delta_kernel<<<(N + 255) / 256, 256, 0, s>>>(dx, N, max_rot, max_trans, scale, out);
  return cudaGetLastError();
}

cudaError_t launch_corr_rmse(const cf_correspondence* corrs, int M, double* partials, double* out, const int* valid,
                             cudaStream_t s) {
  rmse_partial_kernel<<<CF_RMSE_BLOCKS, kLsThreads, 0, s>>>(corrs, M, partials);
  rmse_final_kernel<<<1, 32, 0, s>>>(partials, CF_RMSE_BLOCKS, out, valid);
  return cudaGetLastError();
}

}  // namespace cf
