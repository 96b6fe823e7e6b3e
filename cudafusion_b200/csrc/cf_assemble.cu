// cf_assemble.cu — atomic-free assembly of J^T W J / J^T W r (6x6 BSR).
//
// expand (once per solve): one CTA per block row r turns the row's
//   incidences (c, a) — correspondence c has node r in slot a — into entries
//   (c, a, b) for every valid slot b whose node is an upper column of row r
//   present in the pattern (find_block < 0 drops the term, as in
//   kernels/solver_kernels.cu:123-125), grouped by column with a stable
//   counting sort: order within a column = (warp, round, sub-round, slot,
//   lane), fixed by the incidence order, so the assembly is deterministic.
// assemble (every GN iteration), one launch:
//   CTAs [0, N)        the diagonal block of row r: 8 warps share the row's
//                      segment (4 entries per lane per round, loads issued
//                      before the arithmetic), Kahan-compensated partials are
//                      combined in warp order, then the ARAP terms, the
//                      damping and the rhs.
//   CTAs [N, ...)      one warp per off-diagonal upper block (r, j), j > r,
//                      written with its transpose.
#include "cf_device.cuh"
#include "cf_internal.h"

namespace cf {

namespace {

constexpr int kWarps = kThreads / 32;
constexpr int kEpl = 4;  // incidences per lane per round of expand
constexpr int kRound = 32 * kEpl;

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

// keys of an incidence: lb (16 bits) per slot b, 0xffff = none
__device__ __forceinline__ int key_of(int2 kk, int b) {
  unsigned v = (b < 2) ? (unsigned)kk.x : (unsigned)kk.y;
  v = (b & 1) ? (v >> 16) : (v & 0xffffu);
  return v == 0xffffu ? -1 : (int)v;
}

__global__ void __launch_bounds__(kThreads) expand_kernel(Work w, Pattern pt, int N, int U) {
  extern __shared__ int sm[];
  int* scol = sm;                  // [U]
  int* wcnt = scol + U;            // [kWarps][U]
  const int lane = lane_id(), wid = threadIdx.x >> 5;
  const int r = blockIdx.x;
  const int dpos = pt.diag_pos[r];
  const int nu = pt.row_ptr[r + 1] - dpos;
  for (int l = threadIdx.x; l < nu; l += kThreads) scol[l] = pt.col_idx[dpos + l];
  for (int l = threadIdx.x; l < kWarps * U; l += kThreads) wcnt[l] = 0;
  __syncthreads();
  int* mycnt = wcnt + wid * U;
  const int i0 = w.inc_start[r], i1 = w.inc_start[r + 1];
  const int base = 4 * i0;
  // ---- pass 1: keys (stored) and per-warp counts ----
  for (int t = i0 + wid * kRound; t < i1; t += kWarps * kRound) {
    int e[kEpl];
    int4 ids[kEpl];
    float4 ws[kEpl];
#pragma unroll
    for (int k = 0; k < kEpl; k++) {
      const int idx = t + lane + 32 * k;
      e[k] = idx < i1 ? w.inc[idx] : -1;
    }
#pragma unroll
    for (int k = 0; k < kEpl; k++) {
      if (e[k] >= 0) {
        ids[k] = w.pk_ids[e[k] >> 2];
        ws[k] = w.pk_ws[e[k] >> 2];
      } else {
        ids[k] = make_int4(-1, -1, -1, -1);
        ws[k] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
#pragma unroll
    for (int k = 0; k < kEpl; k++) {
      unsigned kv[4];
#pragma unroll
      for (int b = 0; b < kK; b++) {
        int key = -1;
        if (e[k] >= 0) {
          const int nb = sel4i(ids[k], b);
          if (nb >= r && nb < N && sel4(ws[k], b) > 1e-8f) key = find_col(scol, nu, nb);
        }
        kv[b] = key < 0 ? 0xffffu : (unsigned)key;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        if (key >= 0 && (__ffs(peers) - 1) == lane) mycnt[key] += __popc(peers);
        __syncwarp();
      }
      const int idx = t + lane + 32 * k;
      if (idx < i1) w.ekeys[idx] = make_int2((int)(kv[0] | (kv[1] << 16)), (int)(kv[2] | (kv[3] << 16)));
    }
  }
  __syncthreads();
  // ---- segments: column-major over (column, warp) ----
  if (threadIdx.x == 0) {
    int run = 0;
    for (int l = 0; l < nu; l++) {
      pt.seg_off[dpos + l] = base + run;
      int c0 = run;
      for (int v = 0; v < kWarps; v++) {
        const int c = wcnt[v * U + l];
        wcnt[v * U + l] = run;  // becomes the warp's cursor
        run += c;
      }
      pt.seg_cnt[dpos + l] = run - c0;
    }
  }
  __syncthreads();
  // ---- pass 2: stable scatter of the entries ----
  for (int t = i0 + wid * kRound; t < i1; t += kWarps * kRound) {
    int e[kEpl];
    int2 kk[kEpl];
#pragma unroll
    for (int k = 0; k < kEpl; k++) {
      const int idx = t + lane + 32 * k;
      e[k] = idx < i1 ? w.inc[idx] : -1;
      kk[k] = idx < i1 ? w.ekeys[idx] : make_int2(-1, -1);
    }
#pragma unroll
    for (int k = 0; k < kEpl; k++) {
#pragma unroll
      for (int b = 0; b < kK; b++) {
        const int key = e[k] >= 0 ? key_of(kk[k], b) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        if (key >= 0) {
          const int pos = mycnt[key] + __popc(peers & lanemask_lt());
          w.trip[base + pos] = ((e[k] >> 2) << 4) | ((e[k] & 3) << 2) | b;
        }
        __syncwarp();
        if (key >= 0 && (__ffs(peers) - 1) == lane) mycnt[key] += __popc(peers);
        __syncwarp();
      }
    }
  }
}

struct AsmArgs {
  const cf_deform_node* nodes;
  const cf_dual_quat* T;
  int N;
  float lambda_smooth, lambda_damping, arap_sgn;
};

// index of (p, q), p <= q, in the packed upper triangle of a 6x6 block
__host__ __device__ constexpr int tri(int p, int q) { return p * 6 - p * (p - 1) / 2 + (q - p); }

// Per-warp staging of the gathered per-correspondence records: kStages
// rounds of 32 entries, 3 float4 each (skinned src + fw, normal + residual,
// skin weights), brought in by cp.async so that a warp keeps up to
// 3*kStages 16-byte gathers per lane in flight without holding them in
// registers.  Layout [stage][field][lane]: a lane reads consecutive 16 B.
constexpr int kStages = 8;
constexpr int kStageFloats4 = kStages * 3 * 32;  // float4 per warp

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ float4* stage_smem() {
  extern __shared__ float4 stage_buf[];
  return stage_buf;
}

// Stages entries t + s*stride + lane (s < kStages) of a segment ending at
// `end`; tv[s] is the entry word of stage s for this lane (-1 if none).
__device__ __forceinline__ void stage_entries(const Work& w, int t, int stride, int end, float4* buf, int* tv) {
  const int lane = lane_id();
#pragma unroll
  for (int s = 0; s < kStages; s++) {
    const int e = t + s * stride + lane;
    tv[s] = e < end ? __ldg(w.trip + e) : -1;
  }
#pragma unroll
  for (int s = 0; s < kStages; s++) {
    if (tv[s] >= 0) {
      const int c = tv[s] >> 4;
      cp_async16(buf + (s * 3 + 0) * 32 + lane, w.c_srcfw + c);
      cp_async16(buf + (s * 3 + 1) * 32 + lane, w.c_nres + c);
      cp_async16(buf + (s * 3 + 2) * 32 + lane, w.pk_ws + c);
    }
  }
  cp_async_commit_wait_all();
  __syncwarp();
}

// diagonal block of row r: CTA-wide, values v[0,21) upper entries, v[21,27) rhs
__device__ void assemble_diag(const Work& w, const Pattern& pt, const AsmArgs& aa, int r) {
  __shared__ float sred[kWarps][28];
  const int lane = lane_id(), wid = threadIdx.x >> 5;
  const int pos = pt.diag_pos[r];
  const float3 xr = node_pos(aa.nodes, r);
  const int off = pt.seg_off[pos], end = off + pt.seg_cnt[pos];
  float s[27], k[27];
#pragma unroll
  for (int q = 0; q < 27; q++) s[q] = k[q] = 0.f;
  float4* buf = stage_smem() + wid * kStageFloats4;
  // all 8 warps share every round: stage s of warp w covers entries
  // t + (s*8 + w)*32 + lane
  for (int t = off; t < end; t += kWarps * kStages * 32) {
    int tv[kStages];
    stage_entries(w, t + wid * 32, kWarps * 32, end, buf, tv);
#pragma unroll
    for (int j = 0; j < kStages; j++) {
      if (tv[j] < 0) continue;
      const float4 sf = buf[(j * 3 + 0) * 32 + lane];
      if (sf.w == 0.f) continue;
      const float4 nr = buf[(j * 3 + 1) * 32 + lane];
      const float4 w4 = buf[(j * 3 + 2) * 32 + lane];
      const int a = (tv[j] >> 2) & 3, b = tv[j] & 3;
      const float3 src = f3(sf.x, sf.y, sf.z), n = f3(nr.x, nr.y, nr.z);
      float Ja[6], Jb[6], fJa[6];
      jac_row(src, xr, n, sel4(w4, a), Ja);
      jac_row(src, xr, n, sel4(w4, b), Jb);
#pragma unroll
      for (int p = 0; p < 6; p++) fJa[p] = sf.w * Ja[p];
#pragma unroll
      for (int p = 0; p < 6; p++)
#pragma unroll
        for (int q = p; q < 6; q++) kahan_add(s[tri(p, q)], k[tri(p, q)], fJa[p] * Jb[q]);
      if (a == b) {
#pragma unroll
        for (int p = 0; p < 6; p++) kahan_add(s[21 + p], k[21 + p], -sf.w * Ja[p] * nr.w);
      }
    }
    __syncwarp();
  }
  // ARAP edges incident to r, spread over warp 0..7 lanes (kernels/solver_kernels.cu:293-313, 337-350)
  double earap = 0.0;
  const int a0 = pt.arap_row_ptr[r], a1 = pt.arap_row_ptr[r + 1];
  for (int e = a0 + threadIdx.x; e < a1; e += kThreads) {
    const int inc = pt.arap_row_inc[e];
    const int ed = inc >> 1, role = inc & 1;
    Edge ev = eval_edge(aa.nodes, aa.T, pt.edge_ijk[3 * ed], pt.edge_ijk[3 * ed + 1], pt.edge_ijk[3 * ed + 2],
                        aa.lambda_smooth);
    if (ev.el == 0.f) continue;
    float J[6][3];
    arap_jac(role == 0 ? ev.qi : ev.qj, aa.arap_sgn, J);
#pragma unroll
    for (int p = 0; p < 6; p++)
#pragma unroll
      for (int q = p; q < 6; q++) {
        float t = 0.f;
        t += J[p][0] * J[q][0];
        t += J[p][1] * J[q][1];
        t += J[p][2] * J[q][2];
        kahan_add(s[tri(p, q)], k[tri(p, q)], ev.el * t);
      }
    const float rr[3] = {ev.r.x, ev.r.y, ev.r.z};
#pragma unroll
    for (int p = 0; p < 6; p++) {
      float t = 0.f;
      t += J[p][0] * rr[0];
      t += J[p][1] * rr[1];
      t += J[p][2] * rr[2];
      kahan_add(s[21 + p], k[21 + p], role == 0 ? -ev.el * t : ev.el * t);
    }
    if (role == 0) earap += (double)ev.el * ((double)rr[0] * rr[0] + (double)rr[1] * rr[1] + (double)rr[2] * rr[2]);
  }
  // fold the compensation, reduce each warp, combine warps in order (Kahan)
#pragma unroll
  for (int q = 0; q < 27; q++) s[q] = warp_sum_f(s[q] - k[q]);
  earap = warp_sum_d(earap);
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < 27; q++) sred[wid][q] = s[q];
  }
  __syncthreads();
  if (wid == 0) {
    float tot = 0.f, comp = 0.f;
    if (lane < 27) {
      for (int v = 0; v < kWarps; v++) kahan_add(tot, comp, sred[v][lane]);
      tot -= comp;
    }
    // damping on the diagonal entries (solver_kernels.cu:183-193)
    const int dp = (lane == tri(0, 0)) ? 0 : (lane == tri(1, 1)) ? 1 : (lane == tri(2, 2)) ? 2
                 : (lane == tri(3, 3)) ? 3 : (lane == tri(4, 4)) ? 4 : (lane == tri(5, 5)) ? 5 : -1;
    if (dp >= 0) tot = tot + aa.lambda_damping * fmaxf(fabsf(tot), dp < 3 ? 1e-3f : 1e-2f);
    if (lane < 27) sred[0][lane] = tot;
  }
  __syncthreads();
  float* out = pt.values + (size_t)pos * 36;
  if (threadIdx.x < 36) {
    const int p = threadIdx.x / 6, q = threadIdx.x % 6;
    out[threadIdx.x] = sred[0][tri(min(p, q), max(p, q))];
  } else if (threadIdx.x >= 64 && threadIdx.x < 70) {
    w.rhs[r * 6 + threadIdx.x - 64] = sred[0][21 + threadIdx.x - 64];
  }
  // energy: per-warp ARAP sums combined in warp order by thread 0
  __shared__ double swe[kWarps];
  if (lane == 0) swe[wid] = earap;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int v = 0; v < kWarps; v++) t += swe[v];
    w.e_arap_part[r] = t;
  }
}

// off-diagonal upper block (r, j), j > r: one warp
__device__ void assemble_off(const Work& w, const Pattern& pt, const AsmArgs& aa, int u) {
  const int lane = lane_id();
  const int pos = pt.upper_pos[u], r = pt.upper_row[u], j = pt.col_idx[pos];
  const float3 xr = node_pos(aa.nodes, r), xj = node_pos(aa.nodes, j);
  const int off = pt.seg_off[pos], end = off + pt.seg_cnt[pos];
  float acc[36];
#pragma unroll
  for (int q = 0; q < 36; q++) acc[q] = 0.f;
  float4* buf = stage_smem() + (threadIdx.x >> 5) * kStageFloats4;
  for (int t = off; t < end; t += kStages * 32) {
    int tv[kStages];
    stage_entries(w, t, 32, end, buf, tv);
#pragma unroll
    for (int e = 0; e < kStages; e++) {
      if (tv[e] < 0) continue;
      const float4 sf = buf[(e * 3 + 0) * 32 + lane];
      if (sf.w == 0.f) continue;
      const float4 nr = buf[(e * 3 + 1) * 32 + lane];
      const float4 w4 = buf[(e * 3 + 2) * 32 + lane];
      const int a = (tv[e] >> 2) & 3, b = tv[e] & 3;
      const float3 src = f3(sf.x, sf.y, sf.z), n = f3(nr.x, nr.y, nr.z);
      float Ja[6], Jb[6];
      jac_row(src, xr, n, sel4(w4, a), Ja);
      jac_row(src, xj, n, sel4(w4, b), Jb);
#pragma unroll
      for (int p = 0; p < 6; p++) {
        const float f = sf.w * Ja[p];
#pragma unroll
        for (int q = 0; q < 6; q++) acc[p * 6 + q] += f * Jb[q];
      }
    }
    __syncwarp();
  }
  // ARAP edges (r, j) visited from r (solver_kernels.cu:315-324)
  const int e0 = pt.arap_blk_ptr[u], e1 = pt.arap_blk_ptr[u + 1];
  for (int e = e0 + lane; e < e1; e += 32) {
    const int ed = pt.arap_blk_edge[e];
    Edge ev = eval_edge(aa.nodes, aa.T, pt.edge_ijk[3 * ed], pt.edge_ijk[3 * ed + 1], pt.edge_ijk[3 * ed + 2],
                        aa.lambda_smooth);
    if (ev.el == 0.f) continue;
    float Ji[6][3], Jj[6][3];
    arap_jac(ev.qi, aa.arap_sgn, Ji);
    arap_jac(ev.qj, aa.arap_sgn, Jj);
#pragma unroll
    for (int p = 0; p < 6; p++)
#pragma unroll
      for (int q = 0; q < 6; q++) {
        float t = 0.f;
        t += Ji[p][0] * Jj[q][0];
        t += Ji[p][1] * Jj[q][1];
        t += Ji[p][2] * Jj[q][2];
        acc[p * 6 + q] += -ev.el * t;
      }
  }
#pragma unroll
  for (int q = 0; q < 36; q++) acc[q] = warp_sum_f(acc[q]);
  float* out = pt.values + (size_t)pos * 36;
  float* outT = pt.values + (size_t)pt.trans_pos[pos] * 36;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int l = lane + 32 * h;
    if (l < 36) {
      float val = 0.f;
#pragma unroll
      for (int t = 0; t < 36; t++)
        if (t == l) val = acc[t];
      out[l] = val;
      outT[(l % 6) * 6 + (l / 6)] = val;
    }
  }
}

__global__ void __launch_bounds__(kThreads, 2) assemble_kernel(Work w, Pattern pt, AsmArgs aa) {
  if ((int)blockIdx.x < aa.N) {
    assemble_diag(w, pt, aa, blockIdx.x);
  } else {
    const int k = ((int)blockIdx.x - aa.N) * kWarps + (threadIdx.x >> 5);
    if (k < pt.n_off) assemble_off(w, pt, aa, pt.off_upper[k]);
  }
}

inline int cdiv_(int a, int b) { return (a + b - 1) / b; }

}  // namespace

int expand_smem_bytes(int U) { return (1 + kWarps) * U * (int)sizeof(int); }

cudaError_t launch_expand(const Work& w, const Pattern& p, int N, cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  const int U = p.max_upper_row;
  const size_t smem = (size_t)expand_smem_bytes(U);
  cudaError_t e = cudaFuncSetAttribute(expand_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  expand_kernel<<<N, kThreads, smem, s>>>(w, p, N, U);
  return cudaGetLastError();
}

cudaError_t launch_assemble(const Work& w, const Pattern& p, const SolveArgs& a, const cf_dual_quat* T,
                            cudaStream_t s) {
  if (a.N <= 0) return cudaSuccess;
  AsmArgs aa;
  aa.nodes = a.nodes;
  aa.T = T;
  aa.N = a.N;
  aa.lambda_smooth = a.lambda_smooth;
  aa.lambda_damping = a.lambda_damping;
  aa.arap_sgn = a.arap_consistent ? -1.f : 1.f;
  const int smem = kWarps * kStageFloats4 * (int)sizeof(float4);
  cudaError_t e = cudaFuncSetAttribute(assemble_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  assemble_kernel<<<a.N + cdiv_(p.n_off, kWarps), kThreads, smem, s>>>(w, p, aa);
  return cudaGetLastError();
}

}  // namespace cf
