// cf_kernels.cu — sm_100a kernels of the warp-field Gauss-Newton solve.
//
// Per solve (the correspondences' node ids are fixed for all GN iterations):
//   pack_count    AoS Correspondence -> SoA packs + per-CTA node histograms
//   bin_scan_*    deterministic exclusive offsets (node, CTA)
//   bin_scatter   stable counting sort of incidences (c, slot) by node
//   expand        (cf_assemble.cu) per block row: incidences -> (c, a, b)
//                 entries grouped by upper block column
// Per GN iteration:
//   node_plain    node-centred DQ -> plain DQ (once per node, not per point)
//   residual      DQ skinning + point-to-plane residual + Huber weight
//   assemble      (cf_assemble.cu) a CTA per diagonal block (Kahan), a warp
//                 per off-diagonal block, ARAP, damping, rhs.
// Every kernel works on a table of problems (ProbDesc): a single solve is a
// batch of one; a batched solve concatenates its problems' correspondences
// and nodes, and each sort / energy CTA belongs to exactly one problem.
// The PCG kernels live in cf_pcg_grid.cu (grid-wide cooperative) and
// cf_pcg_cluster.cu (one thread-block cluster).
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
__global__ void __launch_bounds__(kThreads) pack_count_kernel(Table tb, Work w) {
  extern __shared__ int hist[];
  __shared__ __align__(16) uint32_t stage2[2][kThreads * kWords];  // double-buffered tiles of records
  __shared__ __align__(16) float cstage[2][kThreads * 3];           // and of canonical points
  const int tid = threadIdx.x;
  const ProbDesc d = tb.desc[tb.bin_prob[blockIdx.x]];
  const int N = d.N, lc = blockIdx.x - d.bin_cta0;
  for (int i = tid; i < N; i += kThreads) hist[i] = 0;
  const cf_correspondence* corrs = d.corrs;
  const float* canon = d.canon;
  const bool al16 = ((reinterpret_cast<uintptr_t>(corrs) & 15u) == 0);
  const bool cal16 = ((reinterpret_cast<uintptr_t>(canon) & 15u) == 0);
  const int cb = lc * d.chunk;
  const int ce = min(d.M, cb + d.chunk);
  // the next tile's records are in flight (cp.async) while this one is packed
  auto issue = [&](int t0, int b) {
    const int nt = min(kThreads, ce - t0), nw = nt * kWords;
    const uint32_t* src = reinterpret_cast<const uint32_t*>(corrs) + (size_t)t0 * kWords;
    uint32_t* buf = stage2[b];
    if (al16 && (nw & 3) == 0) {
      for (int i = tid; i < (nw >> 2); i += kThreads) cp_async16(buf + 4 * i, src + 4 * i);
    } else {
      for (int i = tid; i < nw; i += kThreads) cp_async4(buf + i, src + i);
    }
    if (canon) {
      const float* csrc = canon + 3 * (size_t)t0;
      if (cal16 && ((3 * nt) & 3) == 0) {
        for (int i = tid; i < (3 * nt) >> 2; i += kThreads) cp_async16(cstage[b] + 4 * i, csrc + 4 * i);
      } else {
        for (int i = tid; i < 3 * nt; i += kThreads) cp_async4(cstage[b] + i, csrc + i);
      }
    }
    cp_async_commit();
  };
  if (cb < ce) issue(cb, 0);
  __syncthreads();
  for (int t0 = cb, it = 0; t0 < ce; t0 += kThreads, it++) {
    const int n = min(kThreads, ce - t0);
    const uint32_t* stage = stage2[it & 1];
    const float* cst = cstage[it & 1];
    if (t0 + kThreads < ce) {
      issue(t0 + kThreads, (it & 1) ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (tid < n) {
      const uint32_t* rec = stage + tid * kWords;
      const int cl = t0 + tid;           // row of the caller's array
      const int c = d.corr_off + cl;     // concatenated index
      float3 p;
      if (canon) {
        p = f3(cst[3 * tid], cst[3 * tid + 1], cst[3 * tid + 2]);
      } else {
        p = f3(__uint_as_float(rec[0]), __uint_as_float(rec[1]), __uint_as_float(rec[2]));
      }
      const bool valid = (rec[18] & 0xffu) != 0;
      const float weight = __uint_as_float(rec[17]);
      const float we = valid ? weight : 0.f;  // <= 0 or NaN: never contributes
      int lid[kK];
#pragma unroll
      for (int k = 0; k < kK; k++) lid[k] = (int)rec[9 + k];
      // node ids become global; an id outside [0, N) is no node (-1)
      int4 ids;
      ids.x = (lid[0] >= 0 && lid[0] < N) ? lid[0] + d.node_off : -1;
      ids.y = (lid[1] >= 0 && lid[1] < N) ? lid[1] + d.node_off : -1;
      ids.z = (lid[2] >= 0 && lid[2] < N) ? lid[2] + d.node_off : -1;
      ids.w = (lid[3] >= 0 && lid[3] < N) ? lid[3] + d.node_off : -1;
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
          if (lid[k] >= 0 && lid[k] < N && sel4(ws, k) > 1e-8f) atomicAdd(&hist[lid[k]], 1);
        }
      }
    }
    __syncthreads();
  }
  int* out = w.cnt + d.cnt_off + (size_t)lc * N;
  for (int i = tid; i < N; i += kThreads) out[i] = hist[i];
}

// Per node: exclusive prefix of its counts over its problem's sort CTAs (in
// place); node_total[n] = sum.  32 nodes per CTA, lane = node (coalesced
// over the sort-CTA index k); the k range is split over the 8 warps: segment
// sums with all loads in flight, a prefix over the warps, then each warp
// rewrites its segment.
__global__ void __launch_bounds__(kThreads) bin_scan_nodes_kernel(Table tb, Work w) {
  __shared__ int seg[kThreads / 32][32];
  const int lane = lane_id(), wid = threadIdx.x >> 5;
  const int n = blockIdx.x * 32 + lane;
  int bc = 0, stride = 0;
  int* p = nullptr;
  if (n < tb.N) {
    const ProbDesc& d = tb.desc[tb.node_prob[n]];
    bc = d.bin_ctas;
    stride = d.N;
    p = w.cnt + d.cnt_off + (n - d.node_off);
  }
  const int per = (bc + kThreads / 32 - 1) / (kThreads / 32);
  const int k0 = min(bc, wid * per), k1 = min(bc, k0 + per);
  int s = 0;
  for (int k = k0; k < k1; k += 8) {
    int v[8];
#pragma unroll
    for (int b = 0; b < 8; b++) v[b] = (k + b < k1) ? p[(size_t)(k + b) * stride] : 0;
#pragma unroll
    for (int b = 0; b < 8; b++) s += v[b];
  }
  seg[wid][lane] = s;
  __syncthreads();
  int run = 0;
  for (int v = 0; v < wid; v++) run += seg[v][lane];
  if (wid == kThreads / 32 - 1 && n < tb.N) w.node_total[n] = run + s;
  for (int k = k0; k < k1; k += 8) {
    int v[8];
#pragma unroll
    for (int b = 0; b < 8; b++) v[b] = (k + b < k1) ? p[(size_t)(k + b) * stride] : 0;
#pragma unroll
    for (int b = 0; b < 8; b++)
      if (k + b < k1) {
        p[(size_t)(k + b) * stride] = run;
        run += v[b];
      }
  }
}

// Rows in order of decreasing incidence count (buckets of 16 incidences),
// so that the per-row kernels (expand, assembly) start their longest rows
// first and the last wave holds short ones.  The order inside a bucket is
// whatever the atomics give: it changes the schedule only, never a result.
constexpr int kOrderBuckets = 1024;
__device__ __forceinline__ void row_order_body(const Work& w, int N) {
  __shared__ int hist[kOrderBuckets];
  __shared__ int wsum[kOrderBuckets / 32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  hist[tid] = 0;
  __syncthreads();
  for (int i = tid; i < N; i += kOrderBuckets)
    atomicAdd(&hist[kOrderBuckets - 1 - min(w.node_total[i] >> 4, kOrderBuckets - 1)], 1);
  __syncthreads();
  const int v = hist[tid];
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int x = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += x;
  }
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int t = wsum[lane], ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int x = __shfl_up_sync(0xffffffffu, ti, o);
      if (lane >= o) ti += x;
    }
    wsum[lane] = ti - t;
  }
  __syncthreads();
  hist[tid] = wsum[wid] + incl - v;
  __syncthreads();
  for (int i = tid; i < N; i += kOrderBuckets) {
    const int pos = atomicAdd(&hist[kOrderBuckets - 1 - min(w.node_total[i] >> 4, kOrderBuckets - 1)], 1);
    w.row_order[pos] = i;
  }
}
__global__ void __launch_bounds__(kOrderBuckets) row_order_kernel(Work w, int N) { row_order_body(w, N); }

// inc_start = exclusive scan of node_total (one CTA of 1024 threads), then
// the rows' launch order.
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
  __syncthreads();
  row_order_body(w, N);  // the launch order of the per-row kernels, from the same totals
}


// Stable scatter of incidences: order within a node = (tile, slot, corr).
__global__ void __launch_bounds__(kThreads) bin_scatter_kernel(Table tb, Work w) {
  extern __shared__ int cursor[];
  __shared__ int wkey[kThreads / 32][32];
  __shared__ int wcnt[kThreads / 32][32];
  __shared__ int wlen[kThreads / 32];
  const int tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  const ProbDesc d = tb.desc[tb.bin_prob[blockIdx.x]];
  const int N = d.N, lc = blockIdx.x - d.bin_cta0;
  const int* base = w.cnt + d.cnt_off + (size_t)lc * N;
  for (int i = tid; i < N; i += kThreads) cursor[i] = w.inc_start[d.node_off + i] + base[i];
  const int cb = d.corr_off + lc * d.chunk;
  const int ce = d.corr_off + min(d.M, lc * d.chunk + d.chunk);
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
      const int id = sel4i(ids, a);
      const float wa = sel4(ws, a);
      // local node of this problem (packed ids are global or -1)
      const int key = (live && we > 0.f && id >= 0 && wa > 1e-8f) ? id - d.node_off : -1;
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

// Stable scatter of incidences with per-warp cursors (problems of at most
// kWarpScatterNodes nodes): the sort CTA's correspondences are split into 8
// contiguous warp ranges; order within a node = (warp range, round of 32
// correspondences, slot, lane).  Pass 1 counts per (warp, node) in 16-bit
// shared counters, pass 2 turns them into offsets below the CTA's base, pass
// 3 writes; no CTA barrier inside a pass.
constexpr int kScatterWarps = kThreads / 32;
constexpr int kWarpScatterSmem = 200 * 1024;
__device__ __forceinline__ int scatter_key(const ProbDesc& d, bool live, int a, const int4& ids, const float4& ws,
                                           float we) {
  if (!live) return -1;
  const int id = sel4i(ids, a);
  return (we > 0.f && id >= 0 && sel4(ws, a) > 1e-8f) ? id - d.node_off : -1;
}
__global__ void __launch_bounds__(kThreads) bin_scatter_warp_kernel(Table tb, Work w) {
  extern __shared__ int sbase[];  // [N] CTA base of each node, then [8][N] 16-bit warp offsets
  const int tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  const ProbDesc d = tb.desc[tb.bin_prob[blockIdx.x]];
  const int N = d.N, lc = blockIdx.x - d.bin_cta0;
  unsigned short* wcnt = reinterpret_cast<unsigned short*>(sbase + N);
  unsigned short* mine = wcnt + (size_t)warp * N;
  const int* base = w.cnt + d.cnt_off + (size_t)lc * N;
  for (int i = tid; i < N; i += kThreads) sbase[i] = w.inc_start[d.node_off + i] + base[i];
  for (int i = tid; i < kScatterWarps * N; i += kThreads) wcnt[i] = 0;
  const int cb = d.corr_off + lc * d.chunk;
  const int ce = d.corr_off + min(d.M, lc * d.chunk + d.chunk);
  const int per = (ce - cb + kScatterWarps - 1) / kScatterWarps;
  const int wb = min(ce, cb + warp * per), we_ = min(ce, wb + per);
  __syncthreads();
  // pass 1: counts per (warp, node)
  for (int t0 = wb; t0 < we_; t0 += 32) {
    const int c = t0 + lane;
    const bool live = c < we_;
    int4 ids = make_int4(-1, -1, -1, -1);
    float4 ws = make_float4(0.f, 0.f, 0.f, 0.f);
    float wgt = 0.f;
    if (live) {
      ids = w.pk_ids[c];
      ws = w.pk_ws[c];
      wgt = w.pk_src[c].w;
    }
#pragma unroll
    for (int a = 0; a < kK; a++) {
      const int key = scatter_key(d, live, a, ids, ws, wgt);
      const unsigned peers = __match_any_sync(0xffffffffu, key);
      if (key >= 0 && (__ffs(peers) - 1) == lane) mine[key] += (unsigned short)__popc(peers);
      __syncwarp();
    }
  }
  __syncthreads();
  // pass 2: per node, the warps' offsets below the CTA base
  for (int i = tid; i < N; i += kThreads) {
    unsigned run = 0;
#pragma unroll
    for (int v = 0; v < kScatterWarps; v++) {
      const unsigned t = wcnt[(size_t)v * N + i];
      wcnt[(size_t)v * N + i] = (unsigned short)run;
      run += t;
    }
  }
  __syncthreads();
  // pass 3: the writes, in the order of pass 1
  for (int t0 = wb; t0 < we_; t0 += 32) {
    const int c = t0 + lane;
    const bool live = c < we_;
    int4 ids = make_int4(-1, -1, -1, -1);
    float4 ws = make_float4(0.f, 0.f, 0.f, 0.f);
    float wgt = 0.f;
    if (live) {
      ids = w.pk_ids[c];
      ws = w.pk_ws[c];
      wgt = w.pk_src[c].w;
    }
#pragma unroll
    for (int a = 0; a < kK; a++) {
      const int key = scatter_key(d, live, a, ids, ws, wgt);
      const unsigned peers = __match_any_sync(0xffffffffu, key);
      if (key >= 0) w.inc[sbase[key] + mine[key] + __popc(peers & lanemask_lt())] = (c << 2) | a;
      __syncwarp();
      if (key >= 0 && (__ffs(peers) - 1) == lane) mine[key] += (unsigned short)__popc(peers);
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

// Correspondences [c0, c1) of energy CTA `cta` (a contiguous share of its
// problem's rows).
__device__ __forceinline__ void e_range(const Table& tb, const ProbDesc& d, int cta, int& c0, int& c1) {
  const int lc = cta - d.e_cta0;
  const int per = (d.M + d.e_ctas - 1) / d.e_ctas;
  c0 = d.corr_off + min(d.M, lc * per);
  c1 = d.corr_off + min(d.M, lc * per + per);
}

struct EdgeArgs {
  const int* edge_ijk;
  int n_edges;
  const cf_deform_node* nodes;
  const cf_dual_quat* T;
  float lambda, arap_sgn;
  float4* out;     // [kEdgeTerms4 * n_edges]
  double* energy;  // [n_edges]
  int edge_ctas;   // the launch's first CTAs
  float2* fr;      // non-null: (weight, residual) per correspondence, for the features
};

__device__ __forceinline__ int tri6(int p, int q) { return p * 6 - p * (p - 1) / 2 + (q - p); }

// CTAs after the correspondence ones: every ARAP edge (i, j) at the current
// transforms (kernels/solver_kernels.cu:202-352: strain and Huber weight,
// residual r, Jacobians J_i, J_j of both endpoints), written as its complete
// contributions for the assembly: the diagonal blocks of i and j (upper
// triangle el J J^T and rhs -+el J r, 27 + pad floats each), the
// off-diagonal block -el J_i J_j^T (36 floats) and the energy el |r|^2 (FP64).
__device__ void edge_terms_cta(const EdgeArgs& ea, int cta) {
  const int ed = cta * kThreads + threadIdx.x;
  if (ed >= ea.n_edges) return;
  const Edge ev = eval_edge(ea.nodes, ea.T, ea.edge_ijk[3 * ed], ea.edge_ijk[3 * ed + 1], ea.edge_ijk[3 * ed + 2],
                            ea.lambda);
  float Ji[6][3], Jj[6][3];
  arap_jac(ev.qi, ea.arap_sgn, Ji);
  arap_jac(ev.qj, ea.arap_sgn, Jj);
  const float rr[3] = {ev.r.x, ev.r.y, ev.r.z};
  float di[28], dj[28], o[36];
#pragma unroll
  for (int p = 0; p < 6; p++)
#pragma unroll
    for (int q = p; q < 6; q++) {
      float ti = 0.f, tj = 0.f;
      ti += Ji[p][0] * Ji[q][0];
      ti += Ji[p][1] * Ji[q][1];
      ti += Ji[p][2] * Ji[q][2];
      tj += Jj[p][0] * Jj[q][0];
      tj += Jj[p][1] * Jj[q][1];
      tj += Jj[p][2] * Jj[q][2];
      di[tri6(p, q)] = ev.el * ti;
      dj[tri6(p, q)] = ev.el * tj;
    }
#pragma unroll
  for (int p = 0; p < 6; p++) {
    float ti = 0.f, tj = 0.f;
    ti += Ji[p][0] * rr[0];
    ti += Ji[p][1] * rr[1];
    ti += Ji[p][2] * rr[2];
    tj += Jj[p][0] * rr[0];
    tj += Jj[p][1] * rr[1];
    tj += Jj[p][2] * rr[2];
    di[21 + p] = -ev.el * ti;
    dj[21 + p] = ev.el * tj;
  }
  di[27] = dj[27] = 0.f;
#pragma unroll
  for (int p = 0; p < 6; p++)
#pragma unroll
    for (int q = 0; q < 6; q++) {
      float t = 0.f;
      t += Ji[p][0] * Jj[q][0];
      t += Ji[p][1] * Jj[q][1];
      t += Ji[p][2] * Jj[q][2];
      o[p * 6 + q] = -ev.el * t;
    }
  float4* out = ea.out + (size_t)kEdgeTerms4 * ed;
#pragma unroll
  for (int k = 0; k < 7; k++) out[k] = make_float4(di[4 * k], di[4 * k + 1], di[4 * k + 2], di[4 * k + 3]);
#pragma unroll
  for (int k = 0; k < 7; k++) out[7 + k] = make_float4(dj[4 * k], dj[4 * k + 1], dj[4 * k + 2], dj[4 * k + 3]);
#pragma unroll
  for (int k = 0; k < 9; k++) out[14 + k] = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
  ea.energy[ed] =
      ev.el > 0.f ? (double)ev.el * ((double)rr[0] * rr[0] + (double)rr[1] * rr[1] + (double)rr[2] * rr[2]) : 0.0;
}

// The edge CTAs come first: their per-thread chains are the longest of the
// launch, so they start while the correspondence CTAs fill the rest.
template <bool SKIN>
__global__ void __launch_bounds__(kThreads) residual_kernel(Table tb, Work w, EdgeArgs ea) {
  __shared__ double red[32];
  if ((int)blockIdx.x < ea.edge_ctas) {
    edge_terms_cta(ea, blockIdx.x);
    return;
  }
  const int cta = blockIdx.x - ea.edge_ctas;
  const ProbDesc d = tb.desc[tb.e_prob[cta]];
  int c0, c1;
  e_range(tb, d, cta, c0, c1);
  const int N = tb.N;
  double e = 0.0;
  for (int c = c0 + threadIdx.x; c < c1; c += kThreads) {
    // every load of the correspondence issued together, then the skinning gathers
    const float4 s = w.pk_src[c];
    const float4 dd = w.pk_dst[c];
    const float4 n = w.pk_nrm[c];
    int4 ids = make_int4(-1, -1, -1, -1);
    float4 ws4 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (SKIN) {
      ids = w.pk_ids[c];
      ws4 = w.pk_ws[c];
    }
    if (!(s.w > 0.f)) continue;
    float3 src = f3(s.x, s.y, s.z);
    if (SKIN) src = blend_warp(src, ids, ws4, w.plain, N);
    // kernels/solver_kernels.cu:76-85
    float res = n.x * (src.x - dd.x) + n.y * (src.y - dd.y) + n.z * (src.z - dd.z);
    float fw = fmaxf(s.w, 0.f) * huber_w(res, 0.2f);
    if (!(fw > 1e-8f)) {
      fw = 0.f;
    } else {
      e += (double)fw * (double)res * (double)res;
    }
    w.c_srcfw[c] = make_float4(src.x, src.y, src.z, fw);
    w.c_nres[c] = make_float4(n.x, n.y, n.z, res);
    if (ea.fr) ea.fr[c] = make_float2(fw, res);
  }
  double t = block_sum_d(e, red);
  if (threadIdx.x == 0) w.e_data_part[cta] = t;
}

// Energy at the current transforms (after the last update): data term with
// the final skinning, plus the problem's ARAP edges; per-CTA partials.
__global__ void __launch_bounds__(kThreads) energy_kernel(Table tb, Work w, Pattern pt, const cf_deform_node* nodes,
                                                          const cf_dual_quat* T, float lambda) {
  __shared__ double red[32];
  const int prob = tb.e_prob[blockIdx.x];
  const ProbDesc d = tb.desc[prob];
  int c0, c1;
  e_range(tb, d, blockIdx.x, c0, c1);
  const int N = tb.N;
  double e = 0.0;
  for (int c = c0 + threadIdx.x; c < c1; c += kThreads) {
    float4 s = w.pk_src[c];
    if (!(s.w > 0.f)) continue;
    float3 src = blend_warp(f3(s.x, s.y, s.z), w.pk_ids[c], w.pk_ws[c], w.plain, N);
    float4 dd = w.pk_dst[c];
    float4 n = w.pk_nrm[c];
    float res = n.x * (src.x - dd.x) + n.y * (src.y - dd.y) + n.z * (src.z - dd.z);
    float fw = fmaxf(s.w, 0.f) * huber_w(res, 0.2f);
    if (fw > 1e-8f) e += (double)fw * (double)res * (double)res;
  }
  const int e0 = pt.prob_edge_off[prob], ne = pt.prob_edge_off[prob + 1] - e0;
  const int lc = blockIdx.x - d.e_cta0, per = (ne + d.e_ctas - 1) / d.e_ctas;
  const int ea = e0 + min(ne, lc * per), eb = e0 + min(ne, lc * per + per);
  for (int ed = ea + threadIdx.x; ed < eb; ed += kThreads) {
    Edge ev = eval_edge(nodes, T, pt.edge_ijk[3 * ed], pt.edge_ijk[3 * ed + 1], pt.edge_ijk[3 * ed + 2], lambda);
    if (ev.el > 0.f)
      e += (double)ev.el * ((double)ev.r.x * ev.r.x + (double)ev.r.y * ev.r.y + (double)ev.r.z * ev.r.z);
  }
  double t = block_sum_d(e, red);
  if (threadIdx.x == 0) w.e_data_part[blockIdx.x] = t;
}

// Sum of p[0..n) by `stride` threads starting at `t`, in a fixed order per
// thread, with 8 loads in flight at a time.
__device__ __forceinline__ double strided_sum(const double* p, int n, int t, int stride) {
  double v = 0.0;
  for (int k0 = t; k0 < n; k0 += 8 * stride) {
    double x[8];
#pragma unroll
    for (int b = 0; b < 8; b++) x[b] = k0 + b * stride < n ? __ldcg(p + k0 + b * stride) : 0.0;
#pragma unroll
    for (int b = 0; b < 8; b++)
      if (k0 + b * stride < n) v += x[b];
  }
  return v;
}

// One warp per problem: its energy = the sum of its CTAs' partials.
__global__ void energy_reduce_kernel(Table tb, Work w, int slot) {
  const ProbDesc d = tb.desc[blockIdx.x];
  double v = strided_sum(w.e_data_part + d.e_cta0, d.e_ctas, threadIdx.x, 32);
  v = warp_sum_d(v);
  if (threadIdx.x == 0) {
    if (slot >= 0) {
      w.stats[blockIdx.x].energy[slot] = v;
      if (!isfinite(v)) atomicOr(w.err, kErrNonFinite);
    } else {
      w.stats[blockIdx.x].gate[-slot - 1] = v;  // energies compared by the learned solve's gate
    }
  }
}

// One warp per problem: the energy at the transforms the residual launch just
// linearised at, from that launch's own partials (data-term CTA partials and
// per-edge ARAP energies) -- no second skinning pass.
// One CTA of 1024 threads per problem.
__global__ void __launch_bounds__(1024) residual_energy_kernel(Table tb, Work w, Pattern pt, int slot) {
  __shared__ double red[32];
  const ProbDesc d = tb.desc[blockIdx.x];
  const int e0 = pt.prob_edge_off[blockIdx.x], e1 = pt.prob_edge_off[blockIdx.x + 1];
  double v = strided_sum(w.e_data_part + d.e_cta0, d.e_ctas, threadIdx.x, 1024) +
             strided_sum(pt.edge_energy + e0, e1 - e0, threadIdx.x, 1024);
  v = warp_sum_d(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x >= 32) return;
  v = warp_sum_d(red[threadIdx.x]);
  if (threadIdx.x == 0) {
    if (slot >= 0) {
      w.stats[blockIdx.x].energy[slot] = v;
      if (!isfinite(v)) atomicOr(w.err, kErrNonFinite);
    } else {
      w.stats[blockIdx.x].gate[-slot - 1] = v;
    }
  }
}

// Batched solves: each problem's nodes (neighbour ids made global) and
// transforms into the concatenated arrays.
__global__ void batch_gather_kernel(Table tb, Work w) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= tb.N) return;
  const ProbDesc d = tb.desc[tb.node_prob[n]];
  const int l = n - d.node_off;
  cf_deform_node nd = d.nodes[l];
  const int nn = min(max(nd.num_neighbors, 0), CF_K_GRAPH);
#pragma unroll
  for (int k = 0; k < CF_K_GRAPH; k++) {
    const int j = nd.neighbors[k];
    nd.neighbors[k] = (k < nn && j >= 0 && j < d.N) ? j + d.node_off : -1;
  }
  w.nodes_cat[n] = nd;
  store_dq(w.T_cat + n, load_dq_cg(d.T + l));
}

__global__ void batch_scatter_kernel(Table tb, Work w) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= tb.N) return;
  const ProbDesc d = tb.desc[tb.node_prob[n]];
  store_dq(d.T + (n - d.node_off), load_dq_cg(w.T_cat + n));
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
  const float3 o = skin_point_centered(f3(pts[3 * c], pts[3 * c + 1], pts[3 * c + 2]), ids + 4 * c, ws + 4 * c,
                                       nodes, T, N);
  out[3 * c] = o.x;
  out[3 * c + 1] = o.y;
  out[3 * c + 2] = o.z;
}

inline int cdiv(int a, int b) { return (a + b - 1) / b; }

}  // namespace

// ----------------------------------------------------------------------------
// launchers
// ----------------------------------------------------------------------------
cudaError_t launch_pack_count(const Work& w, const Table& tb, cudaStream_t s) {
  if (tb.n_bin <= 0) return cudaSuccess;
  const int smem = tb.max_N * (int)sizeof(int);
  cudaError_t e = cudaFuncSetAttribute(pack_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  pack_count_kernel<<<tb.n_bin, kThreads, smem, s>>>(tb, w);
  return cudaGetLastError();
}

cudaError_t launch_bin_scan(const Work& w, const Table& tb, cudaStream_t s) {
  if (tb.N <= 0) return cudaSuccess;
  bin_scan_nodes_kernel<<<cdiv(tb.N, 32), kThreads, 0, s>>>(tb, w);
  static_assert(kOrderBuckets == 1024, "the scan CTA also orders the rows");
  bin_scan_total_kernel<<<1, 1024, 0, s>>>(w, tb.N);
  return cudaGetLastError();
}

cudaError_t launch_row_order(const Work& w, int N, cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  row_order_kernel<<<1, kOrderBuckets, 0, s>>>(w, N);
  return cudaGetLastError();
}

cudaError_t launch_bin_scatter(const Work& w, const Table& tb, cudaStream_t s) {
  if (tb.n_bin <= 0) return cudaSuccess;
  // per-warp cursors: 20 B of shared memory per node, counts below 2^16
  const int wsmem = tb.max_N * (int)(sizeof(int) + kScatterWarps * sizeof(unsigned short));
  if (wsmem <= kWarpScatterSmem && (long long)tb.max_chunk * kK < 65536) {
    cudaError_t e = cudaFuncSetAttribute(bin_scatter_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kWarpScatterSmem);
    if (e != cudaSuccess) return e;
    bin_scatter_warp_kernel<<<tb.n_bin, kThreads, wsmem, s>>>(tb, w);
    return cudaGetLastError();
  }
  const int smem = tb.max_N * (int)sizeof(int);
  cudaError_t e = cudaFuncSetAttribute(bin_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  bin_scatter_kernel<<<tb.n_bin, kThreads, smem, s>>>(tb, w);
  return cudaGetLastError();
}

cudaError_t launch_node_plain(const Work& w, const cf_deform_node* nodes, const cf_dual_quat* T, int N,
                              cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  node_plain_kernel<<<cdiv(N, 128), 128, 0, s>>>(nodes, T, w.plain, N);
  return cudaGetLastError();
}

cudaError_t launch_residual(const Work& w, const Table& tb, const Pattern& p, const SolveArgs& a,
                            const cf_dual_quat* T, bool skin, cudaStream_t s, bool fr) {
  EdgeArgs ea;
  ea.edge_ijk = p.edge_ijk;
  ea.n_edges = p.n_edges;
  ea.nodes = a.nodes;
  ea.T = T;
  ea.lambda = a.lambda_smooth;
  ea.arap_sgn = a.arap_consistent ? -1.f : 1.f;
  ea.out = p.edge_terms;
  ea.energy = p.edge_energy;
  ea.edge_ctas = cdiv(p.n_edges, kThreads);
  ea.fr = fr ? w.c_fr : nullptr;
  const int grid = tb.n_e + ea.edge_ctas;
  if (grid <= 0) return cudaSuccess;
  if (skin)
    residual_kernel<true><<<grid, kThreads, 0, s>>>(tb, w, ea);
  else
    residual_kernel<false><<<grid, kThreads, 0, s>>>(tb, w, ea);
  return cudaGetLastError();
}

cudaError_t launch_residual_energy(const Work& w, const Pattern& p, const SolveArgs& a, int slot, cudaStream_t s) {
  if (a.tb.P <= 0) return cudaSuccess;
  residual_energy_kernel<<<a.tb.P, 1024, 0, s>>>(a.tb, w, p, slot);
  return cudaGetLastError();
}

cudaError_t launch_final_energy(const Work& w, const Pattern& p, const SolveArgs& a, int slot, cudaStream_t s) {
  if (a.tb.n_e <= 0) return cudaSuccess;
  energy_kernel<<<a.tb.n_e, kThreads, 0, s>>>(a.tb, w, p, a.nodes, a.transforms, a.lambda_smooth);
  energy_reduce_kernel<<<a.tb.P, 32, 0, s>>>(a.tb, w, slot);
  return cudaGetLastError();
}

cudaError_t launch_batch_gather(const Work& w, const Table& tb, cudaStream_t s) {
  if (tb.N <= 0) return cudaSuccess;
  batch_gather_kernel<<<cdiv(tb.N, 128), 128, 0, s>>>(tb, w);
  return cudaGetLastError();
}

cudaError_t launch_batch_scatter(const Work& w, const Table& tb, cudaStream_t s) {
  if (tb.N <= 0) return cudaSuccess;
  batch_scatter_kernel<<<cdiv(tb.N, 128), 128, 0, s>>>(tb, w);
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
