// cf_assemble.cu — atomic-free assembly of J^T W J / J^T W r (6x6 BSR).
//
// expand (once per solve): one CTA per block row r turns the row's
//   incidences (c, a) — correspondence c has node r in slot a — into entries
//   (ii, b), ii the incidence's position in the row's list, for every valid
//   slot b whose node is an upper column of row r present in the pattern
//   (find_block < 0 drops the term, as in kernels/solver_kernels.cu:123-125),
//   grouped by column with a stable counting sort: order within a column =
//   (warp, round, sub-round, slot, lane), fixed by the incidence order, so
//   the assembly is deterministic.
// assemble (every GN iteration): one CTA per block row, described at
//   assemble_kernel.  The ARAP terms of every edge (weight, residual and the
//   two rotated offsets of kernels/solver_kernels.cu:202-352) are evaluated
//   once per GN iteration by the residual launch (cf_kernels.cu).
#include "cf_device.cuh"
#include "cf_internal.h"

namespace cf {

namespace {

constexpr int kWarps = kThreads / 32;
constexpr int kEpl = 2;  // incidences per lane per round of expand
constexpr int kExpandStage = 2048;  // incidences of a row kept in shared memory between the passes of expand
constexpr int kColMap = 16384;      // nodes up to which expand finds a column through a node -> column map
// incidences of a row staged by the assembly (60 KB with their entries; 92 %
// of the incidences of the full frame), and ARAP edges of a row / of its
// upper blocks staged (rows have ~16): with them the CTA fits 3 per SM
// (measured: 64.5 us per GN vs 66.4 at 768 / 64)
constexpr int kStageCap = 896;
constexpr int kRowEdges = 32;
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
  int2* s_k = reinterpret_cast<int2*>(sm);  // [kExpandStage] keys of the staged incidences
  int* s_e = sm + 2 * kExpandStage;         // [kExpandStage] the staged incidences
  int* scol = s_e + kExpandStage;           // [U]
  int* wcnt = scol + U;                     // [kWarps][U]
  int* cmap = wcnt + kWarps * U;            // [N] node -> column (only the row's columns written)
  const int lane = lane_id(), wid = threadIdx.x >> 5;
  const int r = w.row_order[blockIdx.x];  // longest rows first
  const int dpos = pt.diag_pos[r];
  const int nu = pt.row_ptr[r + 1] - dpos;
  const bool use_map = N <= kColMap;
  for (int l = threadIdx.x; l < nu; l += kThreads) {
    const int c = pt.col_idx[dpos + l];
    scol[l] = c;
    if (use_map) cmap[c] = l;
  }
  for (int l = threadIdx.x; l < kWarps * U; l += kThreads) wcnt[l] = 0;
  __syncthreads();
  // column of node nb in this row, or -1.  The map is written only at the
  // row's columns: an entry read elsewhere holds whatever shared memory held
  // and is accepted only if it points at a column equal to nb.
  auto col_of = [&](int nb) -> int {
    if (!use_map) return find_col(scol, nu, nb);
    const int l = cmap[nb];
    return ((unsigned)l < (unsigned)nu && scol[l] == nb) ? l : -1;
  };
  int* mycnt = wcnt + wid * U;
  const int i0 = w.inc_start[r], i1 = w.inc_start[r + 1];
  const int base = 4 * i0;
  const bool staged = i1 - i0 <= kExpandStage;  // else the second pass re-reads global memory
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
          if (nb >= r && nb < N && sel4(ws[k], b) > 1e-8f) key = col_of(nb);
        }
        kv[b] = key < 0 ? 0xffffu : (unsigned)key;
        if (key >= 0) atomicAdd(&mycnt[key], 1);  // counts only: order comes from pass 2
      }
      const int idx = t + lane + 32 * k;
      if (idx < i1) {
        const int2 kk = make_int2((int)(kv[0] | (kv[1] << 16)), (int)(kv[2] | (kv[3] << 16)));
        if (staged) {
          s_k[idx - i0] = kk;
          s_e[idx - i0] = e[k];
        } else {
          w.ekeys[idx] = kk;
        }
      }
    }
  }
  __syncthreads();
  // ---- segments: column-major over (column, warp); warp 0, lane = column ----
  if (wid == 0) {
    int carry = 0;
    for (int l0 = 0; l0 < nu; l0 += 32) {
      const int l = l0 + lane;
      int c[kWarps], tot = 0;
#pragma unroll
      for (int v = 0; v < kWarps; v++) {
        c[v] = l < nu ? wcnt[v * U + l] : 0;
        tot += c[v];
      }
      int incl = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += x;
      }
      if (l < nu) {
        int run = carry + incl - tot;
        pt.seg_off[dpos + l] = base + run;
        pt.seg_cnt[dpos + l] = tot;
#pragma unroll
        for (int v = 0; v < kWarps; v++) {
          wcnt[v * U + l] = run;  // becomes the warp's cursor
          run += c[v];
        }
      }
      carry += __shfl_sync(0xffffffffu, incl, 31);
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
      e[k] = idx < i1 ? (staged ? s_e[idx - i0] : w.inc[idx]) : -1;
      kk[k] = idx < i1 ? (staged ? s_k[idx - i0] : w.ekeys[idx]) : make_int2(-1, -1);
    }
#pragma unroll
    for (int k = 0; k < kEpl; k++) {
      const int ii = t + lane + 32 * k - i0;  // the incidence's position in the row's list
#pragma unroll
      for (int b = 0; b < kK; b++) {
        const int key = e[k] >= 0 ? key_of(kk[k], b) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        if (key >= 0) {
          const int pos = mycnt[key] + __popc(peers & lanemask_lt());
          w.trip[base + pos] = (ii << 2) | b;
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
  int N;
  int stage_cap;  // incidences of a row staged in shared memory
  float lambda_damping;
};

// index of (p, q), p <= q, in the packed upper triangle of a 6x6 block
__host__ __device__ constexpr int tri(int p, int q) { return p * 6 - p * (p - 1) / 2 + (q - p); }

// The row's incidence records (skinned src + fw, normal + residual, skin
// weights) and entries: the first `ns` / `nt` staged in shared memory, the
// rest (rows beyond the staging capacity) read from global memory.
struct RowRecords {
  const float4* s_sf;
  const float4* s_nr;
  const float4* s_ws;
  const int* s_a;     // slot a of each staged incidence
  const int* s_trip;  // the row's entries (ii << 2) | b
  const int* inc;     // the row's incidences (c << 2) | a
  const int* trip;    // the row's entries in global memory
  int ns, nt;
  __device__ __forceinline__ void get(const Work& w, int ii, float4& sf, float4& nr, float4& ws) const {
    if (ii < ns) {
      sf = s_sf[ii];
      nr = s_nr[ii];
      ws = s_ws[ii];
    } else {
      const int c = __ldg(inc + ii) >> 2;
      sf = __ldcg(w.c_srcfw + c);
      nr = __ldcg(w.c_nres + c);
      ws = __ldg(w.pk_ws + c);
    }
  }
  __device__ __forceinline__ int slot(int ii) const { return ii < ns ? s_a[ii] : (__ldg(inc + ii) & 3); }
  __device__ __forceinline__ int entry(int t) const { return t < nt ? s_trip[t] : __ldg(trip + t); }
};

// Reduce-scatter of 32 per-lane values: afterwards a[0] of lane l holds the
// warp's sum of value l (31 exchanges instead of 32 x 5 for a butterfly per
// value; fixed pairing, so the result is deterministic).
__device__ __forceinline__ void reduce_scatter32(float* a) {
  const int lane = lane_id();
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const bool up = (lane & s) != 0;
#pragma unroll
    for (int k = 0; k < s; k++) {
      const float send = up ? a[k] : a[k + s];
      const float keep = up ? a[k + s] : a[k];
      a[k] = keep + __shfl_xor_sync(0xffffffffu, send, s);
    }
  }
}

constexpr int kPartVals = 42;  // 36 block values + 6 rhs (diagonal block only)

// One CTA per block row r.
//  1. stage: the row's entry list, its incidences' slots and records
//     (cp.async, one wait)
//  2. windows: the row's blocks (diagonal first, then the upper off-diagonal
//     blocks) are cut into windows of 32 entries; warp w takes a contiguous
//     run of W/8 windows, accumulates lane-private sums of
//     fw J_a J_b^T (and -fw J_a r for the diagonal) and, whenever it leaves a
//     block, reduce-scatters them into a partial slot of that block
//  3. combine: per block value, the warps' partials in warp order (Kahan on
//     the diagonal block), the ARAP terms of the block's edges (precomputed
//     by the residual launch), the damping; blocks written with their
//     transposes, the rhs and the row's ARAP energy.
// 3 CTAs per SM (80 registers, 74 KB of shared memory each): the per-row
// phases are latency chains, so rows in flight matter more than registers
__global__ void __launch_bounds__(kThreads, 3) assemble_kernel(Work w, Pattern pt, AsmArgs aa) {
  extern __shared__ float4 stage_buf[];
  const int r = w.row_order[blockIdx.x], lane = lane_id(), wid = threadIdx.x >> 5;  // longest rows first
  const int cap = aa.stage_cap;
  const int i0 = w.inc_start[r], n_inc = w.inc_start[r + 1] - i0;
  const int dpos = pt.diag_pos[r], nb = pt.row_ptr[r + 1] - dpos;  // upper blocks of the row, diagonal first
  const int U = pt.max_upper_row;
  const int Up = (U + 4) & ~3;
  float4* s_eterm = stage_buf + 3 * cap;     // [kRowEdges][7]: the row's share of its edges' diagonal terms
  float4* s_bterm = s_eterm + 7 * kRowEdges; // [kRowEdges][9]: off-diagonal terms of the row's blocks' edges
  double* s_eng = reinterpret_cast<double*>(s_bterm + 9 * kRowEdges);  // [kRowEdges] energies of the row's edges
  int* s_a = reinterpret_cast<int*>(s_eng + kRowEdges);
  int* s_trip = s_a + cap;
  int* s_wpre = s_trip + 4 * cap;  // [Up] window prefix per block
  int4* s_blk = reinterpret_cast<int4*>(s_wpre + Up);  // [Up] (segment start, count, column, transpose position)
  int* s_boff = reinterpret_cast<int*>(s_blk + Up);    // [Up] first block edge of each upper block
  int* s_erole = s_boff + Up;                          // [kRowEdges] role of each row edge
  float* s_part = reinterpret_cast<float*>(s_erole + kRowEdges);  // [U+8][42]
  RowRecords R;
  R.ns = min(n_inc, cap);
  R.nt = min(pt.seg_off[dpos + nb - 1] + pt.seg_cnt[dpos + nb - 1] - 4 * i0, 4 * cap);
  R.s_sf = stage_buf;
  R.s_nr = stage_buf + cap;
  R.s_ws = stage_buf + 2 * cap;
  R.s_a = s_a;
  R.s_trip = s_trip;
  R.inc = w.inc + i0;
  R.trip = w.trip + 4 * (size_t)i0;
  // block info, ARAP terms of the row's edges and of its blocks' edges
  const int u0 = pt.ustart[r];
  const int a0 = pt.arap_row_ptr[r], a1 = pt.arap_row_ptr[r + 1] - a0, na = min(a1, kRowEdges);
  const int be0 = pt.arap_blk_ptr[u0 + 1];  // the row's off-diagonal upper blocks are u0+1 .. u0+nb-1
  const int be1 = pt.arap_blk_ptr[u0 + nb] - be0, nbe = min(be1, kRowEdges);
  for (int k = threadIdx.x; k < nb; k += kThreads) {
    const int pos = dpos + k;
    s_blk[k] = make_int4(pt.seg_off[pos] - 4 * i0, pt.seg_cnt[pos], pt.col_idx[pos], pt.trans_pos[pos]);
    s_boff[k] = k == 0 ? 0 : pt.arap_blk_ptr[u0 + k] - be0;
  }
  // (threads from the back, so that they overlap the block-info loads)
  const int te = kThreads - 1 - threadIdx.x;
  if (te < na) {
    const int inc = pt.arap_row_inc[a0 + te];
    const int ed = inc >> 1, role = inc & 1;
    s_erole[te] = role;
    const float4* src = pt.edge_terms + (size_t)kEdgeTerms4 * ed + 7 * role;
#pragma unroll
    for (int k = 0; k < 7; k++) cp_async16(s_eterm + 7 * te + k, src + k);
    s_eng[te] = role == 0 ? pt.edge_energy[ed] : 0.0;
  } else if (te >= kRowEdges && te < kRowEdges + nbe) {
    const int e = te - kRowEdges;
    const float4* src = pt.edge_terms + (size_t)kEdgeTerms4 * pt.arap_blk_edge[be0 + e] + 14;
#pragma unroll
    for (int k = 0; k < 9; k++) cp_async16(s_bterm + 9 * e + k, src + k);
  }
  for (int t = threadIdx.x; t < R.nt; t += kThreads) s_trip[t] = __ldg(R.trip + t);
  for (int ii = threadIdx.x; ii < R.ns; ii += kThreads) {
    const int e = __ldg(R.inc + ii);
    const int c = e >> 2;
    s_a[ii] = e & 3;
    cp_async16(stage_buf + ii, w.c_srcfw + c);
    cp_async16(stage_buf + cap + ii, w.c_nres + c);
    cp_async16(stage_buf + 2 * cap + ii, w.pk_ws + c);
  }
  cp_async_commit_wait_all();
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int k = 0; k < nb; k++) {
      s_wpre[k] = run;
      run += (s_blk[k].y + 31) >> 5;
    }
    s_wpre[nb] = run;
  }
  __syncthreads();

  // ---- 2. windows ----
  const int W = s_wpre[nb];
  const int wa = (int)((long long)W * wid / kWarps), wb = (int)((long long)W * (wid + 1) / kWarps);
  const float3 xr = node_pos(aa.nodes, r);
  int k = 0;
  while (k < nb && s_wpre[k + 1] <= wa) k++;
  // lane-private sums: an off-diagonal block's 36 values (p * 6 + q); the
  // diagonal block's upper triangle (tri(p, q)) and its rhs (21 + p)
  float acc[36];
#pragma unroll
  for (int q = 0; q < 36; q++) acc[q] = 0.f;
  float3 xc = node_pos(aa.nodes, k < nb ? s_blk[k].z : r);
  int seg0 = k < nb ? s_blk[k].x : 0, segn = k < nb ? s_blk[k].y : 0;
  for (int win = wa; win < wb; win++) {
    const int t = seg0 + (win - s_wpre[k]) * 32 + lane;
    if (t < seg0 + segn) {
      const int e = R.entry(t);
      const int ii = e >> 2, b = e & 3;
      float4 sf, nr, w4;
      R.get(w, ii, sf, nr, w4);
      if (sf.w != 0.f) {
        const int a = R.slot(ii);
        const float3 src = f3(sf.x, sf.y, sf.z), n = f3(nr.x, nr.y, nr.z);
        float Ja[6], Jb[6];
        jac_row(src, xr, n, sel4(w4, a), Ja);
        jac_row(src, xc, n, sel4(w4, b), Jb);
        if (k == 0) {  // (the block index is uniform in the warp)
#pragma unroll
          for (int p = 0; p < 6; p++) {
            const float f = sf.w * Ja[p];
#pragma unroll
            for (int q = p; q < 6; q++) acc[tri(p, q)] += f * Jb[q];
          }
          if (a == b) {
#pragma unroll
            for (int p = 0; p < 6; p++) acc[21 + p] += -sf.w * Ja[p] * nr.w;
          }
        } else {
#pragma unroll
          for (int p = 0; p < 6; p++) {
            const float f = sf.w * Ja[p];
#pragma unroll
            for (int q = 0; q < 6; q++) acc[p * 6 + q] += f * Jb[q];
          }
        }
      }
    }
    // leaving block k (next window belongs to another block, or the run ends)
    if (win + 1 == wb || win + 1 == s_wpre[k + 1]) {
      float* dst = s_part + (size_t)(k + wid) * kPartVals;
      if (k == 0) {  // 27 values (acc[27..31] stay zero): one reduce-scatter
        reduce_scatter32(acc);
        if (lane < 27) dst[lane] = acc[0];
      } else {
        float extra[4] = {acc[32], acc[33], acc[34], acc[35]};
        reduce_scatter32(acc);
        dst[lane] = acc[0];
        // the last 4 values: halved over lane bits 4 and 3 (3 exchanges),
        // then summed over bits 2..0; lane 8g holds value 2 (g >> 1) + (g & 1)
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const bool up = (lane & 16) != 0;
          const float send = up ? extra[q] : extra[q + 2];
          const float keep = up ? extra[q + 2] : extra[q];
          extra[q] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
        {
          const bool up = (lane & 8) != 0;
          const float send = up ? extra[0] : extra[1];
          const float keep = up ? extra[1] : extra[0];
          extra[0] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) extra[0] += __shfl_xor_sync(0xffffffffu, extra[0], o);
        if ((lane & 7) == 0) dst[32 + 2 * ((lane >> 4) & 1) + ((lane >> 3) & 1)] = extra[0];
      }
#pragma unroll
      for (int q = 0; q < 36; q++) acc[q] = 0.f;
      if (win + 1 < wb) {
        k++;
        while (k < nb && s_wpre[k + 1] <= win + 1) k++;
        xc = node_pos(aa.nodes, s_blk[k].z);
        seg0 = s_blk[k].x;
        segn = s_blk[k].y;
      }
    }
  }
  __syncthreads();

  // ---- 3. combine ----
  const int nwork = 27 + 36 * (nb - 1);
  for (int item = threadIdx.x; item < nwork; item += kThreads) {
    int kb, v;
    if (item < 27) {
      kb = 0;
      v = item;
    } else {
      kb = 1 + (item - 27) / 36;
      v = (item - 27) % 36;
    }
    // warps that touched block kb, in warp order
    const int w0 = s_wpre[kb], w1 = s_wpre[kb + 1];
    float tot = 0.f, comp = 0.f;
    if (w1 > w0) {
      const int idx = v;  // diagonal block: tri(p, q), then the rhs at 21 + p; off-diagonal: p * 6 + q
      for (int ww = 0; ww < kWarps; ww++) {  // the warps whose window runs met block kb
        const int a_w = (int)((long long)W * ww / kWarps), b_w = (int)((long long)W * (ww + 1) / kWarps);
        if (a_w >= b_w || a_w >= w1 || b_w <= w0) continue;
        const float x = s_part[(size_t)(kb + ww) * kPartVals + idx];
        if (kb == 0) kahan_add(tot, comp, x); else tot += x;
      }
      tot -= comp;
      comp = 0.f;
    }
    const int pos = dpos + kb;
    if (kb == 0) {
      // ARAP edges incident to r (kernels/solver_kernels.cu:293-313, 337-350)
      for (int e = 0; e < a1; e++) {
        float x;
        if (e < na) {
          x = reinterpret_cast<const float*>(s_eterm + 7 * e)[v];
        } else {
          const int inc = pt.arap_row_inc[a0 + e];
          x = reinterpret_cast<const float*>(pt.edge_terms + (size_t)kEdgeTerms4 * (inc >> 1) + 7 * (inc & 1))[v];
        }
        kahan_add(tot, comp, x);
      }
      tot -= comp;
      if (v < 21) {
        int p = 0;
        while (tri(p, 5) < v) p++;
        const int q = v - tri(p, p) + p;
        // damping on the diagonal entries (solver_kernels.cu:183-193)
        if (p == q) tot = tot + aa.lambda_damping * fmaxf(fabsf(tot), p < 3 ? 1e-3f : 1e-2f);
        float* out = pt.values + (size_t)pos * 36;
        out[p * 6 + q] = tot;
        out[q * 6 + p] = tot;
      } else {
        w.rhs[r * 6 + (v - 21)] = tot;
      }
    } else {
      // ARAP edges (r, j) visited from r (solver_kernels.cu:315-324)
      const int e0 = s_boff[kb], e1 = kb + 1 < nb ? s_boff[kb + 1] : be1;
      for (int e = e0; e < e1; e++) {
        tot += e < nbe ? reinterpret_cast<const float*>(s_bterm + 9 * e)[v]
                       : reinterpret_cast<const float*>(pt.edge_terms + (size_t)kEdgeTerms4 *
                                                                          pt.arap_blk_edge[be0 + e] + 14)[v];
      }
      pt.values[(size_t)pos * 36 + v] = tot;
      pt.values[(size_t)s_blk[kb].w * 36 + (v % 6) * 6 + v / 6] = tot;
    }
  }
  if (threadIdx.x == kThreads - 1) {  // the row's ARAP energy: edges owned by r
    double t = 0.0;
    for (int e = 0; e < a1; e++) {
      if (e < na) {
        t += s_eng[e];
      } else {
        const int inc = pt.arap_row_inc[a0 + e];
        if (!(inc & 1)) t += pt.edge_energy[inc >> 1];
      }
    }
    w.e_arap_part[r] = t;
  }
}

}  // namespace

int expand_smem_bytes(int U, int N) {
  return 3 * kExpandStage * (int)sizeof(int) + (1 + kWarps) * U * (int)sizeof(int) +
         (N <= kColMap ? N * (int)sizeof(int) : 0);
}

cudaError_t launch_expand(const Work& w, const Pattern& p, int N, cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  const int U = p.max_upper_row;
  const size_t smem = (size_t)expand_smem_bytes(U, N);
  cudaError_t e = cudaFuncSetAttribute(expand_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  expand_kernel<<<N, kThreads, smem, s>>>(w, p, N, U);
  return cudaGetLastError();
}

int assemble_smem_bytes(int max_upper_row) {
  const int Up = (max_upper_row + 4) & ~3;
  return kStageCap * (3 * (int)sizeof(float4) + 5 * (int)sizeof(int)) + kRowEdges * 16 * (int)sizeof(float4) +
         kRowEdges * 8 + Up * (4 + 16 + 4) + kRowEdges * 4 + (max_upper_row + kWarps) * kPartVals * 4;
}

cudaError_t launch_assemble(const Work& w, const Pattern& p, const SolveArgs& a, const cf_dual_quat* T,
                            cudaStream_t s) {
  (void)T;  // the transforms enter through the ARAP terms of the residual launch
  if (a.N <= 0) return cudaSuccess;
  AsmArgs aa;
  aa.nodes = a.nodes;
  aa.N = a.N;
  aa.stage_cap = kStageCap;
  aa.lambda_damping = a.lambda_damping;
  const int smem = assemble_smem_bytes(p.max_upper_row);
  cudaError_t e = cudaFuncSetAttribute(assemble_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  assemble_kernel<<<a.N, kThreads, smem, s>>>(w, p, aa);
  return cudaGetLastError();
}

}  // namespace cf
