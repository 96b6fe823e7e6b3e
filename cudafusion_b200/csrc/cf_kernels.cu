// cf_kernels.cu — sm_100a kernels of the warp-field Gauss-Newton solve.
//
// Per solve (the correspondences' node ids are fixed for all GN iterations):
//   pack_count    AoS Correspondence -> SoA packs + per-CTA node histograms
//   bin_scan_*    deterministic exclusive offsets (node, CTA)
//   bin_scatter   stable counting sort of incidences (c, slot) by node
//   expand        per block row: incidences -> (c, a, b) entries grouped by
//                 upper block column (the segmented layout of J^T W J)
// Per GN iteration:
//   node_plain    node-centred DQ -> plain DQ (once per node, not per point)
//   residual      DQ skinning + point-to-plane residual + Huber weight
//   assemble      one warp per upper block: register accumulation over the
//                 block's entry segment (Kahan on diagonal blocks), ARAP edges,
//                 damping, warp reduction, block + transpose store.  No atomics.
//   pcg           persistent cooperative block-Jacobi PCG: A rows resident in
//                 shared memory, FP64 block inverses and dot products, two
//                 bounded grid barriers per iteration, fused clamped DQ update.
// The reference (CUDAFusion kernels/solver_kernels.cu) assembles with float
// atomicAdd and runs PCG as ~10 synchronised launches per iteration.
#include <cooperative_groups.h>

#include "cf_device.cuh"
#include "cf_internal.h"

namespace cf {

namespace {

constexpr int kWords = 19;  // sizeof(cf_correspondence) / 4
static_assert(sizeof(cf_correspondence) == 76, "Correspondence layout");
static_assert(sizeof(cf_deform_node) == 96, "DeformNode layout");
static_assert(sizeof(cf_dual_quat) == 32, "DualQuat layout");

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

// Block-wide double sum; result valid in thread 0.
__device__ __forceinline__ double block_sum_d(double v, double* red) {
  v = warp_sum_d(v);
  int w = threadIdx.x >> 5;
  __syncthreads();
  if (lane_id() == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = (lane_id() < (int)(blockDim.x >> 5)) ? red[lane_id()] : 0.0;
    t = warp_sum_d(t);
  }
  return t;
}

// ----------------------------------------------------------------------------
// pack + count
// ----------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) pack_count_kernel(const cf_correspondence* __restrict__ corrs,
                                                              const float* __restrict__ canon, int M, int N,
                                                              int chunk, Work w) {
  extern __shared__ int hist[];
  __shared__ __align__(16) uint32_t stage[kThreads * kWords];
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += kThreads) hist[i] = 0;
  const bool al16 = ((reinterpret_cast<uintptr_t>(corrs) & 15u) == 0);
  const int cb = blockIdx.x * chunk;
  const int ce = min(M, cb + chunk);
  __syncthreads();
  for (int t0 = cb; t0 < ce; t0 += kThreads) {
    const int n = min(kThreads, ce - t0);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(corrs) + (size_t)t0 * kWords;
    const int nw = n * kWords;
    if (al16 && (nw & 3) == 0) {
      const uint4* s4 = reinterpret_cast<const uint4*>(src);
      uint4* d4 = reinterpret_cast<uint4*>(stage);
      for (int i = tid; i < (nw >> 2); i += kThreads) d4[i] = __ldg(s4 + i);
    } else {
      for (int i = tid; i < nw; i += kThreads) stage[i] = __ldg(src + i);
    }
    __syncthreads();
    if (tid < n) {
      const uint32_t* rec = stage + tid * kWords;
      const int c = t0 + tid;
      float3 p;
      if (canon) {
        p = f3(__ldg(canon + 3 * (size_t)c), __ldg(canon + 3 * (size_t)c + 1), __ldg(canon + 3 * (size_t)c + 2));
      } else {
        p = f3(__uint_as_float(rec[0]), __uint_as_float(rec[1]), __uint_as_float(rec[2]));
      }
      const bool valid = (rec[18] & 0xffu) != 0;
      const float weight = __uint_as_float(rec[17]);
      const float we = valid ? weight : 0.f;  // <= 0 or NaN: never contributes
      int4 ids = make_int4((int)rec[9], (int)rec[10], (int)rec[11], (int)rec[12]);
      float4 ws = make_float4(__uint_as_float(rec[13]), __uint_as_float(rec[14]), __uint_as_float(rec[15]),
                              __uint_as_float(rec[16]));
      w.pk_src[c] = make_float4(p.x, p.y, p.z, we);
      w.pk_dst[c] = make_float4(__uint_as_float(rec[3]), __uint_as_float(rec[4]), __uint_as_float(rec[5]), 0.f);
      w.pk_nrm[c] = make_float4(__uint_as_float(rec[6]), __uint_as_float(rec[7]), __uint_as_float(rec[8]), 0.f);
      w.pk_ids[c] = ids;
      w.pk_ws[c] = ws;
      if (we > 0.f) {
#pragma unroll
        for (int k = 0; k < kK; k++) {
          int id = sel4i(ids, k);
          float wk = sel4(ws, k);
          if (id >= 0 && id < N && wk > 1e-8f) atomicAdd(&hist[id], 1);
        }
      }
    }
    __syncthreads();
  }
  int* out = w.cnt + (size_t)blockIdx.x * N;
  for (int i = tid; i < N; i += kThreads) out[i] = hist[i];
}

// cnt[k][n] -> exclusive prefix over k (in place); node_total[n] = sum.
__global__ void bin_scan_nodes_kernel(Work w, int N, int bin_ctas) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  int run = 0;
  for (int k = 0; k < bin_ctas; k++) {
    int* p = w.cnt + (size_t)k * N + n;
    int v = *p;
    *p = run;
    run += v;
  }
  w.node_total[n] = run;
}

// inc_start = exclusive scan of node_total (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024) bin_scan_total_kernel(Work w, int N) {
  __shared__ int wsum[32];
  const int tid = threadIdx.x;
  const int per = (N + 1023) / 1024;
  const int b = tid * per, e = min(N, b + per);
  int loc = 0;
  for (int i = b; i < e; i++) loc += w.node_total[i];
  // block exclusive scan of loc
  int v = loc;
  const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) wsum[wid] = v;
  __syncthreads();
  if (wid == 0) {
    int s = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    wsum[lane] = s;
  }
  __syncthreads();
  int excl = v - loc + (wid > 0 ? wsum[wid - 1] : 0);
  for (int i = b; i < e; i++) {
    w.inc_start[i] = excl;
    excl += w.node_total[i];
  }
  if (tid == 1023) w.inc_start[N] = wsum[31];
}

// Stable scatter of incidences: order within a node = (tile, slot, corr).
__global__ void __launch_bounds__(kThreads) bin_scatter_kernel(Work w, int M, int N, int chunk) {
  extern __shared__ int cursor[];
  __shared__ int wkey[kThreads / 32][32];
  __shared__ int wcnt[kThreads / 32][32];
  __shared__ int wlen[kThreads / 32];
  const int tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  const int* base = w.cnt + (size_t)blockIdx.x * N;
  for (int i = tid; i < N; i += kThreads) cursor[i] = w.inc_start[i] + base[i];
  const int cb = blockIdx.x * chunk;
  const int ce = min(M, cb + chunk);
  __syncthreads();
  for (int t0 = cb; t0 < ce; t0 += kThreads) {
    const int c = t0 + tid;
    const bool live = c < ce;
    int4 ids = make_int4(-1, -1, -1, -1);
    float4 ws = make_float4(0.f, 0.f, 0.f, 0.f);
    float we = 0.f;
    if (live) {
      ids = w.pk_ids[c];
      ws = w.pk_ws[c];
      we = w.pk_src[c].w;
    }
#pragma unroll 1
    for (int a = 0; a < kK; a++) {
      int id = sel4i(ids, a);
      float wa = sel4(ws, a);
      int key = (live && we > 0.f && id >= 0 && id < N && wa > 1e-8f) ? id : -1;
      unsigned peers = __match_any_sync(0xffffffffu, key);
      int rank = __popc(peers & lanemask_lt());
      bool leader = (__ffs(peers) - 1) == lane;
      bool last = (31 - __clz(peers)) == lane;
      unsigned lead_mask = __ballot_sync(0xffffffffu, leader && key >= 0);
      if (leader && key >= 0) {
        int slot = __popc(lead_mask & lanemask_lt());
        wkey[warp][slot] = key;
        wcnt[warp][slot] = __popc(peers);
      }
      if (lane == 0) wlen[warp] = __popc(lead_mask);
      __syncthreads();
      int pos = 0;
      bool is_last = false;
      if (key >= 0) {
        int prefix = 0;
        for (int v = 0; v < warp; v++)
          for (int s = 0; s < wlen[v]; s++)
            if (wkey[v][s] == key) prefix += wcnt[v][s];
        is_last = last;
        if (is_last)
          for (int v = warp + 1; v < kThreads / 32 && is_last; v++)
            for (int s = 0; s < wlen[v]; s++)
              if (wkey[v][s] == key) is_last = false;
        pos = cursor[key] + prefix + rank;
        w.inc[pos] = (c << 2) | a;
      }
      __syncthreads();
      if (is_last) cursor[key] = pos + 1;
      __syncthreads();
    }
  }
}

// One warp per block row: expand its incidences into (c, a, b) entries for
// every valid slot b whose node is an upper column of the row present in the
// pattern (find_block < 0 drops the term, solver_kernels.cu:123-125), grouped
// by column with a stable counting sort.
__device__ __forceinline__ int find_col(const int* cols, int n, int v) {
  int lo = 0, hi = n - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int x = cols[mid];
    if (x == v) return mid;
    if (x < v) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

__global__ void __launch_bounds__(kThreads) expand_kernel(Work w, Pattern pt, int N, int U) {
  extern __shared__ int sm[];
  const int lane = lane_id(), wib = threadIdx.x >> 5;
  const int r = blockIdx.x * (kThreads / 32) + wib;
  if (r >= N) return;
  int* scol = sm + wib * 3 * U;
  int* scnt = scol + U;
  int* scur = scnt + U;
  const int dpos = pt.diag_pos[r];
  const int nu = pt.row_ptr[r + 1] - dpos;
  for (int l = lane; l < nu; l += 32) {
    scol[l] = pt.col_idx[dpos + l];
    scnt[l] = 0;
  }
  __syncwarp();
  const int i0 = w.inc_start[r], i1 = w.inc_start[r + 1];
  const int base = 4 * i0;
  for (int pass = 0; pass < 2; pass++) {
    for (int t = i0; t < i1; t += 32) {
      const int idx = t + lane;
      const int e = idx < i1 ? w.inc[idx] : -1;
      const int c = e >> 2, a = e & 3;
      int4 ids = make_int4(-1, -1, -1, -1);
      float4 ws = make_float4(0.f, 0.f, 0.f, 0.f);
      if (e >= 0) {
        ids = w.pk_ids[c];
        ws = w.pk_ws[c];
      }
#pragma unroll 1
      for (int b = 0; b < kK; b++) {
        int key = -1;
        if (e >= 0) {
          int nb = sel4i(ids, b);
          if (nb >= r && nb < N && sel4(ws, b) > 1e-8f) key = find_col(scol, nu, nb);
        }
        unsigned peers = __match_any_sync(0xffffffffu, key);
        bool leader = (__ffs(peers) - 1) == lane;
        if (pass == 0) {
          if (key >= 0 && leader) scnt[key] += __popc(peers);
        } else {
          if (key >= 0) {
            int pos = scur[key] + __popc(peers & lanemask_lt());
            w.trip[base + pos] = (c << 4) | (a << 2) | b;
          }
          __syncwarp();
          if (key >= 0 && leader) scur[key] += __popc(peers);
        }
        __syncwarp();
      }
    }
    if (pass == 0) {
      if (lane == 0) {
        int run = 0;
        for (int l = 0; l < nu; l++) {
          scur[l] = run;
          pt.seg_off[dpos + l] = base + run;
          pt.seg_cnt[dpos + l] = scnt[l];
          run += scnt[l];
        }
      }
      __syncwarp();
    }
  }
}

// ----------------------------------------------------------------------------
// per-iteration kernels
// ----------------------------------------------------------------------------
__global__ void node_plain_kernel(const cf_deform_node* __restrict__ nodes, const cf_dual_quat* __restrict__ T,
                                  cf_dual_quat* __restrict__ plain, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  store_dq(plain + i, dq_centered(load_dq_cg(T + i), node_pos(nodes, i)));
}

template <bool SKIN>
__global__ void __launch_bounds__(kThreads) residual_kernel(Work w, int M, int N) {
  __shared__ double red[32];
  double e = 0.0;
  for (int c = blockIdx.x * kThreads + threadIdx.x; c < M; c += gridDim.x * kThreads) {
    float4 s = w.pk_src[c];
    if (!(s.w > 0.f)) continue;
    float3 src = f3(s.x, s.y, s.z);
    if (SKIN) src = blend_warp(src, w.pk_ids[c], w.pk_ws[c], w.plain, N);
    float4 d = w.pk_dst[c];
    float4 n = w.pk_nrm[c];
    // kernels/solver_kernels.cu:76-85
    float res = n.x * (src.x - d.x) + n.y * (src.y - d.y) + n.z * (src.z - d.z);
    float fw = fmaxf(s.w, 0.f) * huber_w(res, 0.2f);
    if (!(fw > 1e-8f)) {
      fw = 0.f;
    } else {
      e += (double)fw * (double)res * (double)res;
    }
    w.c_srcfw[c] = make_float4(src.x, src.y, src.z, fw);
    w.c_nres[c] = make_float4(n.x, n.y, n.z, res);
  }
  double t = block_sum_d(e, red);
  if (threadIdx.x == 0) w.e_data_part[blockIdx.x] = t;
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
  DQ Ti = load_dq_cg(T + i), Tj = load_dq_cg(T + j);
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

struct AsmArgs {
  const cf_deform_node* nodes;
  const cf_dual_quat* T;
  int N;
  float lambda_smooth, lambda_damping, arap_sgn;
};

__global__ void __launch_bounds__(kThreads) assemble_kernel(Work w, Pattern pt, AsmArgs aa) {
  const int lane = lane_id();
  const int u = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (u >= pt.n_upper) return;
  const int pos = pt.upper_pos[u];
  const int r = pt.upper_row[u];
  const int j = pt.col_idx[pos];
  const float3 xr = node_pos(aa.nodes, r);
  const int off = pt.seg_off[pos], cnt = pt.seg_cnt[pos];
  float* out = pt.values + (size_t)pos * 36;
  if (j == r) {
    // ---- diagonal block: 21 upper entries + rhs, Kahan-compensated ----
    float s[21], k[21], bs[6], bk[6];
#pragma unroll
    for (int q = 0; q < 21; q++) s[q] = k[q] = 0.f;
#pragma unroll
    for (int q = 0; q < 6; q++) bs[q] = bk[q] = 0.f;
    for (int e = off + lane; e < off + cnt; e += 32) {
      const int t = w.trip[e];
      const int c = t >> 4, a = (t >> 2) & 3, b = t & 3;
      const float4 sf = w.c_srcfw[c];
      if (sf.w == 0.f) continue;
      const float4 nr = w.c_nres[c];
      const float4 w4 = w.pk_ws[c];
      const float3 src = f3(sf.x, sf.y, sf.z), n = f3(nr.x, nr.y, nr.z);
      float Ja[6], Jb[6];
      jac_row(src, xr, n, sel4(w4, a), Ja);
      jac_row(src, xr, n, sel4(w4, b), Jb);
      float fJa[6];
#pragma unroll
      for (int p = 0; p < 6; p++) fJa[p] = sf.w * Ja[p];
      int idx = 0;
#pragma unroll
      for (int p = 0; p < 6; p++)
#pragma unroll
        for (int q = p; q < 6; q++) kahan_add(s[idx], k[idx], fJa[p] * Jb[q]), idx++;
      if (a == b) {
#pragma unroll
        for (int p = 0; p < 6; p++) kahan_add(bs[p], bk[p], -sf.w * Ja[p] * nr.w);
      }
    }
    // ARAP edges incident to r (kernels/solver_kernels.cu:293-313, 337-350)
    double earap = 0.0;
    const int a0 = pt.arap_row_ptr[r], a1 = pt.arap_row_ptr[r + 1];
    for (int e = a0 + lane; e < a1; e += 32) {
      const int inc = pt.arap_row_inc[e];
      const int ed = inc >> 1, role = inc & 1;
      const int ei = pt.edge_ijk[3 * ed], ej = pt.edge_ijk[3 * ed + 1], ek = pt.edge_ijk[3 * ed + 2];
      Edge ev = eval_edge(aa.nodes, aa.T, ei, ej, ek, aa.lambda_smooth);
      if (ev.el == 0.f) continue;
      float J[6][3];
      arap_jac(role == 0 ? ev.qi : ev.qj, aa.arap_sgn, J);
      int idx = 0;
#pragma unroll
      for (int p = 0; p < 6; p++)
#pragma unroll
        for (int q = p; q < 6; q++) {
          float v = 0.f;
          v += J[p][0] * J[q][0];
          v += J[p][1] * J[q][1];
          v += J[p][2] * J[q][2];
          kahan_add(s[idx], k[idx], ev.el * v);
          idx++;
        }
      const float rr[3] = {ev.r.x, ev.r.y, ev.r.z};
#pragma unroll
      for (int p = 0; p < 6; p++) {
        float v = 0.f;
        v += J[p][0] * rr[0];
        v += J[p][1] * rr[1];
        v += J[p][2] * rr[2];
        kahan_add(bs[p], bk[p], role == 0 ? -ev.el * v : ev.el * v);
      }
      if (role == 0) earap += (double)ev.el * ((double)rr[0] * rr[0] + (double)rr[1] * rr[1] + (double)rr[2] * rr[2]);
    }
    // fold the compensation, reduce across the warp (every lane gets all sums)
#pragma unroll
    for (int q = 0; q < 21; q++) s[q] = warp_sum_f(s[q] - k[q]);
#pragma unroll
    for (int q = 0; q < 6; q++) bs[q] = warp_sum_f(bs[q] - bk[q]);
    earap = warp_sum_d(earap);
    // relative Levenberg damping on the diagonal (solver_kernels.cu:183-193)
    {
      int idx = 0;
#pragma unroll
      for (int p = 0; p < 6; p++) {
        float d = s[idx];
        float fl = (p < 3) ? 1e-3f : 1e-2f;
        s[idx] = d + aa.lambda_damping * fmaxf(fabsf(d), fl);
        idx += 6 - p;
      }
    }
    // lane l < 36 stores element l of the symmetric block
    if (lane < 36) {
      int p = lane / 6, q = lane % 6;
      int lo = min(p, q), hi = max(p, q);
      int uidx = lo * 6 - lo * (lo - 1) / 2 + (hi - lo);
      float v = 0.f;
#pragma unroll
      for (int t = 0; t < 21; t++)
        if (t == uidx) v = s[t];
      out[lane] = v;
    }
    if (lane < 4) {
      // elements 32..35 of the block go to lanes 0..3
      int l = 32 + lane;
      int p = l / 6, q = l % 6;
      int lo = min(p, q), hi = max(p, q);
      int uidx = lo * 6 - lo * (lo - 1) / 2 + (hi - lo);
      float v = 0.f;
#pragma unroll
      for (int t = 0; t < 21; t++)
        if (t == uidx) v = s[t];
      out[l] = v;
    }
    if (lane < 6) {
      float v = 0.f;
#pragma unroll
      for (int t = 0; t < 6; t++)
        if (t == lane) v = bs[t];
      w.rhs[r * 6 + lane] = v;
    }
    if (lane == 0) w.e_arap_part[r] = earap;
  } else {
    // ---- off-diagonal upper block (r, j), j > r ----
    const float3 xj = node_pos(aa.nodes, j);
    float acc[36];
#pragma unroll
    for (int q = 0; q < 36; q++) acc[q] = 0.f;
    for (int e = off + lane; e < off + cnt; e += 32) {
      const int t = w.trip[e];
      const int c = t >> 4, a = (t >> 2) & 3, b = t & 3;
      const float4 sf = w.c_srcfw[c];
      if (sf.w == 0.f) continue;
      const float4 nr = w.c_nres[c];
      const float4 w4 = w.pk_ws[c];
      const float3 src = f3(sf.x, sf.y, sf.z), n = f3(nr.x, nr.y, nr.z);
      float Ja[6], Jb[6];
      jac_row(src, xr, n, sel4(w4, a), Ja);
      jac_row(src, xj, n, sel4(w4, b), Jb);
#pragma unroll
      for (int p = 0; p < 6; p++) {
        float f = sf.w * Ja[p];
#pragma unroll
        for (int q = 0; q < 6; q++) acc[p * 6 + q] += f * Jb[q];
      }
    }
    // ARAP edges (r, j) visited from r (solver_kernels.cu:315-324)
    const int b0 = pt.arap_blk_ptr[u], b1 = pt.arap_blk_ptr[u + 1];
    for (int e = b0 + lane; e < b1; e += 32) {
      const int ed = pt.arap_blk_edge[e];
      const int ei = pt.edge_ijk[3 * ed], ej = pt.edge_ijk[3 * ed + 1], ek = pt.edge_ijk[3 * ed + 2];
      Edge ev = eval_edge(aa.nodes, aa.T, ei, ej, ek, aa.lambda_smooth);
      if (ev.el == 0.f) continue;
      float Ji[6][3], Jj[6][3];
      arap_jac(ev.qi, aa.arap_sgn, Ji);
      arap_jac(ev.qj, aa.arap_sgn, Jj);
#pragma unroll
      for (int p = 0; p < 6; p++)
#pragma unroll
        for (int q = 0; q < 6; q++) {
          float v = 0.f;
          v += Ji[p][0] * Jj[q][0];
          v += Ji[p][1] * Jj[q][1];
          v += Ji[p][2] * Jj[q][2];
          acc[p * 6 + q] += -ev.el * v;
        }
    }
#pragma unroll
    for (int q = 0; q < 36; q++) acc[q] = warp_sum_f(acc[q]);
    float* outT = pt.values + (size_t)pt.trans_pos[pos] * 36;
    // lane l stores element l (and l+32 for l < 4) of the block and its transpose
#pragma unroll
    for (int h = 0; h < 2; h++) {
      int l = lane + 32 * h;
      if (l < 36) {
        float v = 0.f;
#pragma unroll
        for (int t = 0; t < 36; t++)
          if (t == l) v = acc[t];
        out[l] = v;
        outT[(l % 6) * 6 + (l / 6)] = v;
      }
    }
  }
}

// ----------------------------------------------------------------------------
// persistent block-Jacobi PCG (kernels/solver_kernels.cu:616-687)
// ----------------------------------------------------------------------------
struct PcgArgs {
  Work w;
  Pattern pt;
  SolveArgs a;
  int slot;
};

__host__ __device__ inline int align16(int x) { return (x + 15) & ~15; }

struct PcgLayout {
  int a, col, rowptr, pg, minv, x, r, ap, p, red, total;
};

__host__ __device__ inline PcgLayout pcg_layout(int nblk, int nrows, bool a_smem) {
  PcgLayout L;
  int o = 0;
  L.a = o; o += a_smem ? align16(nblk * 36 * 4) : 0;
  L.col = o; o += align16(nblk * 4);
  L.rowptr = o; o += align16((nrows + 1) * 4);
  L.pg = o; o += align16(nblk * 6 * 4);
  L.minv = o; o += align16(nrows * 36 * 8);
  L.x = o; o += align16(nrows * 6 * 4);
  L.r = o; o += align16(nrows * 6 * 4);
  L.ap = o; o += align16(nrows * 6 * 4);
  L.p = o; o += align16(nrows * 6 * 4);
  L.red = o; o += 64 * 8;
  L.total = o;
  return L;
}

// Reads the per-CTA partials of reduction slot `s` and returns the grid sum
// (the same bits on every CTA: fixed order, xor butterfly).
__device__ __forceinline__ double grid_total(const double* parts, int G, double* bcast) {
  if (threadIdx.x < 32) {
    double v = 0.0;
    for (int k = lane_id(); k < G; k += 32) v += __ldcg(parts + k);
    v = warp_sum_d(v);
    if (threadIdx.x == 0) *bcast = v;
  }
  __syncthreads();
  double t = *bcast;
  __syncthreads();
  return t;
}

// 6x6 FP64 Cholesky inverse (se3_math.cuh:152-202); false if not SPD.
__device__ bool inv6_chol_d(const double* A, double* Ainv) {
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

template <bool A_SMEM>
__global__ void __launch_bounds__(kThreads, 1) pcg_kernel(PcgArgs P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Work& w = P.w;
  const Pattern& pt = P.pt;
  const SolveArgs& a = P.a;
  const int tid = threadIdx.x;
  const int cta = blockIdx.x, G = gridDim.x;
  const int r0 = pt.pcg_row_begin[cta], r1 = pt.pcg_row_begin[cta + 1];
  const int nrows = r1 - r0;
  const int b0 = pt.row_ptr[r0], b1 = pt.row_ptr[r1];
  const int nblk = b1 - b0;
  const PcgLayout L = pcg_layout(nblk, nrows, A_SMEM);
  float* sA = reinterpret_cast<float*>(smem + L.a);
  int* sCol = reinterpret_cast<int*>(smem + L.col);
  int* sRow = reinterpret_cast<int*>(smem + L.rowptr);
  float* sPg = reinterpret_cast<float*>(smem + L.pg);
  double* sMinv = reinterpret_cast<double*>(smem + L.minv);
  float* sX = reinterpret_cast<float*>(smem + L.x);
  float* sR = reinterpret_cast<float*>(smem + L.r);
  float* sAp = reinterpret_cast<float*>(smem + L.ap);
  float* sP = reinterpret_cast<float*>(smem + L.p);
  double* sRed = reinterpret_cast<double*>(smem + L.red);
  const float* gA = pt.values + (size_t)b0 * 36;
  const int n6 = nrows * 6;
  unsigned gen = 0;
  int* err = w.err;
  __shared__ int s_fallbacks;

  // ---- prologue: rows of A into shared memory, block inverses, r = b ----
  if (tid == 0) s_fallbacks = 0;
  if (A_SMEM) {
    const float4* g4 = reinterpret_cast<const float4*>(gA);
    float4* s4 = reinterpret_cast<float4*>(sA);
    for (int i = tid; i < nblk * 9; i += kThreads) s4[i] = __ldcg(g4 + i);
  }
  for (int i = tid; i < nblk; i += kThreads) sCol[i] = pt.col_idx[b0 + i];
  for (int i = tid; i <= nrows; i += kThreads) sRow[i] = pt.row_ptr[r0 + i] - b0;
  __syncthreads();
  for (int i = tid; i < nrows; i += kThreads) {
    const int dl = pt.diag_pos[r0 + i] - b0;
    double D[36];
    for (int q = 0; q < 36; q++) D[q] = A_SMEM ? (double)sA[dl * 36 + q] : (double)__ldcg(gA + dl * 36 + q);
    for (int q = 0; q < 6; q++) D[q * 6 + q] += (double)1e-4f;  // solver_kernels.cu:382-383
    double* Mi = sMinv + i * 36;
    if (!inv6_chol_d(D, Mi)) {  // diagonal fallback, solver_kernels.cu:387-395
      for (int q = 0; q < 36; q++) Mi[q] = 0.0;
      for (int q = 0; q < 6; q++) Mi[q * 6 + q] = 1.0 / (D[q * 6 + q] + (double)1e-6f);
      atomicAdd(&s_fallbacks, 1);
    }
  }
  for (int t = tid; t < n6; t += kThreads) {
    sX[t] = 0.f;
    sR[t] = __ldcg(w.rhs + r0 * 6 + t);
  }
  __syncthreads();
  // z = M^-1 r ; partial r.z and b.b
  double prz = 0.0, pbb = 0.0;
  for (int t = tid; t < n6; t += kThreads) {
    const int i = t / 6, c = t % 6;
    const double* Mi = sMinv + i * 36 + c * 6;
    const float* ri = sR + i * 6;
    double zz = 0.0;
#pragma unroll
    for (int q = 0; q < 6; q++) zz += Mi[q] * (double)ri[q];
    float zf = (float)zz;
    w.z[r0 * 6 + t] = zf;
    prz += (double)sR[t] * (double)zf;
    pbb += (double)sR[t] * (double)sR[t];
  }
  double* part = w.partials;  // [2][2][G]
  {
    double t1 = block_sum_d(prz, sRed);
    double t2 = block_sum_d(pbb, sRed + 8);
    if (tid == 0) {
      part[(0 * 2 + 0) * G + cta] = t1;
      part[(0 * 2 + 1) * G + cta] = t2;
      if (s_fallbacks) atomicAdd(&w.stats->fallbacks, s_fallbacks);
    }
  }
  // energy of this linearisation point (CTA 0): data partials + ARAP rows
  if (cta == 0 && tid >= 32 && tid < 64) {
    double v = 0.0;
    for (int k = tid - 32; k < kEnergyCtas; k += 32) v += w.e_data_part[k];
    for (int k = tid - 32; k < a.N; k += 32) v += w.e_arap_part[k];
    v = warp_sum_d(v);
    if (tid == 32) {
      w.stats->energy[P.slot] = v;
      if (!isfinite(v)) atomicOr(err, kErrNonFinite);
    }
  }
  grid_barrier(w.barrier, gen++, G, err, a.spin_limit);
  double rz = grid_total(part + (0 * 2 + 0) * G, G, sRed + 16);
  double rr_last = grid_total(part + (0 * 2 + 1) * G, G, sRed + 16);

  int used = 0;
  float betaf = 0.f;
  const float* pold = w.p1;  // p_{-1} (unused at it = 0)
  for (int it = 0; it < a.pcg_iterations; it++) {
    float* pnew = (it & 1) ? w.p1 : w.p0;
    // ---- p_it on the columns this CTA touches: p = z + beta * p_old ----
    for (int e = tid; e < nblk * 6; e += kThreads) {
      const int bl = e / 6, c = e % 6;
      const int jj = sCol[bl];
      const float zj = __ldcg(w.z + jj * 6 + c);
      sPg[e] = (it == 0) ? zj : __fmaf_rn(betaf, __ldcg(pold + jj * 6 + c), zj);
    }
    for (int t = tid; t < n6; t += kThreads) {
      const float zi = __ldcg(w.z + r0 * 6 + t);
      const float pi = (it == 0) ? zi : __fmaf_rn(betaf, __ldcg(pold + r0 * 6 + t), zi);
      sP[t] = pi;
      pnew[r0 * 6 + t] = pi;
    }
    __syncthreads();
    // ---- Ap on own rows (solver_kernels.cu:406-432) ----
    double ppap = 0.0;
    for (int t = tid; t < n6; t += kThreads) {
      const int i = t / 6, c = t % 6;
      float acc = 0.f;
      for (int bl = sRow[i]; bl < sRow[i + 1]; bl++) {
        const float* Ab = A_SMEM ? (sA + bl * 36 + c * 6) : (gA + bl * 36 + c * 6);
        const float* pg = sPg + bl * 6;
#pragma unroll
        for (int q = 0; q < 6; q++) acc = __fmaf_rn(A_SMEM ? Ab[q] : __ldcg(Ab + q), pg[q], acc);
      }
      sAp[t] = acc;
      ppap += (double)sP[t] * (double)acc;
    }
    {
      const int buf = gen & 1;
      double t1 = block_sum_d(ppap, sRed);
      if (tid == 0) part[(buf * 2 + 0) * G + cta] = t1;
      grid_barrier(w.barrier, gen++, G, err, a.spin_limit);
      const double pAp = grid_total(part + (buf * 2 + 0) * G, G, sRed + 16);
      if (fabs(pAp) < 1e-12) break;  // solver_kernels.cu:647-653
      const float af = (float)(rz / pAp);
      // ---- x += a p ; r -= a Ap ; z = M^-1 r ----
      for (int t = tid; t < n6; t += kThreads) {
        sX[t] = __fmaf_rn(af, sP[t], sX[t]);
        sR[t] = __fmaf_rn(-af, sAp[t], sR[t]);
      }
      __syncthreads();
      double prr = 0.0, przn = 0.0;
      for (int t = tid; t < n6; t += kThreads) {
        const int i = t / 6, c = t % 6;
        const double* Mi = sMinv + i * 36 + c * 6;
        const float* ri = sR + i * 6;
        double zz = 0.0;
#pragma unroll
        for (int q = 0; q < 6; q++) zz += Mi[q] * (double)ri[q];
        const float zf = (float)zz;
        w.z[r0 * 6 + t] = zf;
        prr += (double)sR[t] * (double)sR[t];
        przn += (double)sR[t] * (double)zf;
      }
      const int buf2 = gen & 1;
      double t2 = block_sum_d(prr, sRed);
      double t3 = block_sum_d(przn, sRed + 8);
      if (tid == 0) {
        part[(buf2 * 2 + 0) * G + cta] = t2;
        part[(buf2 * 2 + 1) * G + cta] = t3;
      }
      grid_barrier(w.barrier, gen++, G, err, a.spin_limit);
      const double rr = grid_total(part + (buf2 * 2 + 0) * G, G, sRed + 16);
      const double rzn = grid_total(part + (buf2 * 2 + 1) * G, G, sRed + 16);
      used = it + 1;
      rr_last = rr;
      if (sqrt(rr) < (double)a.pcg_tolerance) break;  // solver_kernels.cu:669
      betaf = (float)(rzn / rz);
      rz = rzn;
      pold = pnew;
    }
  }

  // ---- epilogue: delta_x out, or the clamped DQ update fused per node ----
  bool bad = false;
  for (int t = tid; t < n6; t += kThreads) bad |= !isfinite(sX[t]);
  if (bad) atomicOr(err, kErrNonFinite);
  if (a.delta_x) {
    for (int t = tid; t < n6; t += kThreads) a.delta_x[r0 * 6 + t] = sX[t];
  } else {
    for (int i = tid; i < nrows; i += kThreads) {
      const int node = r0 + i;
      DQ Tn = twist_update(load_dq_cg(a.transforms + node), sX + i * 6, a.max_rot, a.max_trans, a.update_scale);
      store_dq(a.transforms + node, Tn);
      store_dq(w.plain + node, dq_centered(Tn, node_pos(a.nodes, node)));
    }
  }
  if (cta == 0 && tid == 0) {
    w.stats->pcg_iters[P.slot] = used;
    w.stats->pcg_res[P.slot] = sqrt(rr_last);
  }
}

// Energy at the current transforms (after the last update): data term with
// the final skinning, plus the ARAP edges; fixed grid, per-CTA partials.
__global__ void __launch_bounds__(kThreads) energy_kernel(Work w, Pattern pt, const cf_deform_node* nodes,
                                                          const cf_dual_quat* T, int M, int N, float lambda) {
  __shared__ double red[32];
  double e = 0.0;
  for (int c = blockIdx.x * kThreads + threadIdx.x; c < M; c += gridDim.x * kThreads) {
    float4 s = w.pk_src[c];
    if (!(s.w > 0.f)) continue;
    float3 src = blend_warp(f3(s.x, s.y, s.z), w.pk_ids[c], w.pk_ws[c], w.plain, N);
    float4 d = w.pk_dst[c];
    float4 n = w.pk_nrm[c];
    float res = n.x * (src.x - d.x) + n.y * (src.y - d.y) + n.z * (src.z - d.z);
    float fw = fmaxf(s.w, 0.f) * huber_w(res, 0.2f);
    if (fw > 1e-8f) e += (double)fw * (double)res * (double)res;
  }
  for (int ed = blockIdx.x * kThreads + threadIdx.x; ed < pt.n_edges; ed += gridDim.x * kThreads) {
    Edge ev = eval_edge(nodes, T, pt.edge_ijk[3 * ed], pt.edge_ijk[3 * ed + 1], pt.edge_ijk[3 * ed + 2], lambda);
    if (ev.el > 0.f)
      e += (double)ev.el * ((double)ev.r.x * ev.r.x + (double)ev.r.y * ev.r.y + (double)ev.r.z * ev.r.z);
  }
  double t = block_sum_d(e, red);
  if (threadIdx.x == 0) w.e_data_part[blockIdx.x] = t;
}

__global__ void energy_reduce_kernel(Work w, int slot) {
  double v = 0.0;
  for (int k = threadIdx.x; k < kEnergyCtas; k += 32) v += w.e_data_part[k];
  v = warp_sum_d(v);
  if (threadIdx.x == 0) {
    w.stats->energy[slot] = v;
    if (!isfinite(v)) atomicOr(w.err, kErrNonFinite);
  }
}

// WarpField::apply_twist_increment (src/warp_field.cu:250-291).
__global__ void apply_twist_kernel(cf_dual_quat* __restrict__ T, const float* __restrict__ dx, int N, float max_rot,
                                   float max_trans, float scale) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  float d[6];
#pragma unroll
  for (int k = 0; k < 6; k++) d[k] = dx[i * 6 + k];
  store_dq(T + i, twist_update(load_dq_cg(T + i), d, max_rot, max_trans, scale));
}

// warp_point per point (se3_math.cuh:450-510), centring each node DQ on the fly.
__global__ void skin_points_kernel(const float* __restrict__ pts, const int* __restrict__ ids,
                                   const float* __restrict__ ws, int M, const cf_deform_node* __restrict__ nodes,
                                   const cf_dual_quat* __restrict__ T, int N, float* out) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= M) return;
  float3 p = f3(pts[3 * c], pts[3 * c + 1], pts[3 * c + 2]);
  float4 br = make_float4(0.f, 0.f, 0.f, 0.f), bd = make_float4(0.f, 0.f, 0.f, 0.f);
  float wsum = 0.f;
  for (int k = 0; k < kK; k++) {
    int nid = ids[4 * c + k];
    float wk = ws[4 * c + k];
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
  float3 o = p;
  if (wsum >= 1e-8f) {
    DQ b;
    b.r = br;
    b.d = bd;
    o = dq_transform_point(dq_normalize(b), p);
  }
  out[3 * c] = o.x;
  out[3 * c + 1] = o.y;
  out[3 * c + 2] = o.z;
}

inline int cdiv(int a, int b) { return (a + b - 1) / b; }

}  // namespace

// ----------------------------------------------------------------------------
// launchers
// ----------------------------------------------------------------------------
cudaError_t launch_pack_count(const Work& w, const cf_correspondence* corrs, const float* canon, int M, int N,
                              int bin_ctas, int chunk, cudaStream_t s) {
  if (M <= 0) return cudaSuccess;
  size_t smem = (size_t)N * sizeof(int);
  cudaError_t e = cudaFuncSetAttribute(pack_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  pack_count_kernel<<<bin_ctas, kThreads, smem, s>>>(corrs, canon, M, N, chunk, w);
  return cudaGetLastError();
}

cudaError_t launch_bin_scan(const Work& w, int N, int bin_ctas, cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  bin_scan_nodes_kernel<<<cdiv(N, 128), 128, 0, s>>>(w, N, bin_ctas);
  bin_scan_total_kernel<<<1, 1024, 0, s>>>(w, N);
  return cudaGetLastError();
}

cudaError_t launch_bin_scatter(const Work& w, int M, int N, int bin_ctas, int chunk, cudaStream_t s) {
  if (M <= 0) return cudaSuccess;
  size_t smem = (size_t)N * sizeof(int);
  cudaError_t e = cudaFuncSetAttribute(bin_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  bin_scatter_kernel<<<bin_ctas, kThreads, smem, s>>>(w, M, N, chunk);
  return cudaGetLastError();
}

int expand_smem_bytes(int U) { return (kThreads / 32) * 3 * U * (int)sizeof(int); }

cudaError_t launch_expand(const Work& w, const Pattern& p, int N, cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  int U = p.max_upper_row;
  size_t smem = (size_t)expand_smem_bytes(U);
  cudaError_t e = cudaFuncSetAttribute(expand_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  expand_kernel<<<cdiv(N, kThreads / 32), kThreads, smem, s>>>(w, p, N, U);
  return cudaGetLastError();
}

cudaError_t launch_node_plain(const Work& w, const cf_deform_node* nodes, const cf_dual_quat* T, int N,
                              cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  node_plain_kernel<<<cdiv(N, 128), 128, 0, s>>>(nodes, T, w.plain, N);
  return cudaGetLastError();
}

cudaError_t launch_residual(const Work& w, int M, int N, bool skin, cudaStream_t s) {
  if (skin)
    residual_kernel<true><<<kEnergyCtas, kThreads, 0, s>>>(w, M, N);
  else
    residual_kernel<false><<<kEnergyCtas, kThreads, 0, s>>>(w, M, N);
  return cudaGetLastError();
}

cudaError_t launch_assemble(const Work& w, const Pattern& p, const SolveArgs& a, const cf_dual_quat* T,
                            cudaStream_t s) {
  if (p.n_upper <= 0) return cudaSuccess;
  AsmArgs aa;
  aa.nodes = a.nodes;
  aa.T = T;
  aa.N = a.N;
  aa.lambda_smooth = a.lambda_smooth;
  aa.lambda_damping = a.lambda_damping;
  aa.arap_sgn = a.arap_consistent ? -1.f : 1.f;
  assemble_kernel<<<cdiv(p.n_upper, kThreads / 32), kThreads, 0, s>>>(w, p, aa);
  return cudaGetLastError();
}

int pcg_smem_bytes(int max_blocks, int max_rows, bool a_in_smem) {
  return pcg_layout(max_blocks, max_rows, a_in_smem).total;
}

cudaError_t pcg_prepare(int smem, bool a_in_smem) {
  if (a_in_smem)
    return cudaFuncSetAttribute(pcg_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  return cudaFuncSetAttribute(pcg_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

int pcg_max_active_ctas(int smem, bool a_in_smem) {
  int per_sm = 0, dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (a_in_smem)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<true>, kThreads, smem);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<false>, kThreads, smem);
  return per_sm * sms;
}

cudaError_t launch_pcg(const Work& w, const Pattern& p, const SolveArgs& a, int gn_slot, cudaStream_t s) {
  if (a.N <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(w.barrier, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  PcgArgs P;
  P.w = w;
  P.pt = p;
  P.a = a;
  P.slot = gn_slot;
  void* args[] = {&P};
  if (p.pcg_a_in_smem)
    return cudaLaunchCooperativeKernel((void*)pcg_kernel<true>, dim3(p.pcg_ctas), dim3(kThreads), args,
                                       (size_t)p.pcg_smem, s);
  return cudaLaunchCooperativeKernel((void*)pcg_kernel<false>, dim3(p.pcg_ctas), dim3(kThreads), args,
                                     (size_t)p.pcg_smem, s);
}

cudaError_t launch_final_energy(const Work& w, const Pattern& p, const SolveArgs& a, int slot, cudaStream_t s) {
  energy_kernel<<<kEnergyCtas, kThreads, 0, s>>>(w, p, a.nodes, a.transforms, a.M, a.N, a.lambda_smooth);
  energy_reduce_kernel<<<1, 32, 0, s>>>(w, slot);
  return cudaGetLastError();
}

cudaError_t launch_apply_twist(cf_dual_quat* T, const float* dx, int N, float max_rot, float max_trans,
                               float scale, cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  apply_twist_kernel<<<cdiv(N, 128), 128, 0, s>>>(T, dx, N, max_rot, max_trans, scale);
  return cudaGetLastError();
}

cudaError_t launch_skin_points(const float* pts, const int* ids, const float* ws, int M,
                               const cf_deform_node* nodes, const cf_dual_quat* T, int N, float* out,
                               cudaStream_t s) {
  if (M <= 0) return cudaSuccess;
  skin_points_kernel<<<cdiv(M, 256), 256, 0, s>>>(pts, ids, ws, M, nodes, T, N, out);
  return cudaGetLastError();
}

}  // namespace cf
