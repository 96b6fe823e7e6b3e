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
// staged incidences per assembly thread (the stage capacity is kStageCap)
constexpr int kIncPerThread = (kStageCap + kThreads - 1) / kThreads;
static_assert(kIncPerThread * kThreads >= kStageCap && kStageCap % 4 == 0, "assembly staging layout");

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
    // the assembly's metadata of this launch position, so that its first
    // load is one 48-byte record instead of a chain of dependent lookups:
    // {row, first incidence, incidences, diagonal position}, {upper blocks,
    // first upper-block index, first ARAP incidence, ARAP incidences},
    // {first block edge past the diagonal, block edges, entries, 0}
    if (lane == 0) {
      const int u0 = pt.ustart[r];
      const int a0 = pt.arap_row_ptr[r], a1 = pt.arap_row_ptr[r + 1];
      const int be0 = pt.arap_blk_ptr[u0 + 1], be1 = pt.arap_blk_ptr[u0 + nu];
      int4* m = w.asm_meta + 3 * (size_t)blockIdx.x;
      m[0] = make_int4(r, i0, i1 - i0, dpos);
      m[1] = make_int4(nu, u0, a0, a1 - a0);
      m[2] = make_int4(be0, be1 - be0, carry, 0);
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

// The row's incidence records, staged as the factors the windows need:
// U = ((src - x_r) x n, fw w_a) and N = (n, fw w_a r), with the skin weights
// of the correspondence (for w_b) and the slot a; the first `ns` / `nt` staged
// in shared memory, the rest (rows beyond the staging capacity) formed from
// global memory.
struct RowRecords {
  const float4* s_u;
  const float4* s_n;
  const float4* s_ws;
  const int* s_a;     // slot a of each staged incidence
  const int* s_trip;  // the row's entries (ii << 2) | b
  const int* inc;     // the row's incidences (c << 2) | a
  const int* trip;    // the row's entries in global memory
  float3 xr;          // the row's node
  int ns, nt;
  __device__ __forceinline__ void get(const Work& w, int ii, float4& u, float4& n, float4& ws, int& a) const {
    if (ii < ns) {
      u = s_u[ii];
      n = s_n[ii];
      ws = s_ws[ii];
      a = s_a[ii];
    } else {
      const int e = __ldg(inc + ii);
      const int c = e >> 2;
      a = e & 3;
      const float4 sf = __ldcg(w.c_srcfw + c), nr = __ldcg(w.c_nres + c);
      ws = __ldg(w.pk_ws + c);
      factor(sf, nr, sel4(ws, a), xr, u, n);
    }
  }
  // (src, fw), (n, r) and w_a -> U, N
  __device__ __forceinline__ static void factor(float4 sf, float4 nr, float wa, float3 xr, float4& u, float4& n) {
    const float3 l = sub3(f3(sf.x, sf.y, sf.z), xr);
    const float3 cp = cross3(l, f3(nr.x, nr.y, nr.z));
    const float fwa = sf.w * wa;
    u = make_float4(cp.x, cp.y, cp.z, fwa);
    n = make_float4(nr.x, nr.y, nr.z, fwa * nr.w);
  }
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

// Per block, the sums the windows accumulate (g = fw w_a w_b, u = (src - x_r)
// x n of the row's node, n the normal):
//   [0, 6)   S_uu = sum g u u^T (upper triangle: 00 01 02 11 12 22)
//   [6, 15)  S_un = sum g u n^T (row-major)
//   [15, 21) S_nn = sum g n n^T (upper triangle)
//   [21, 27) the rhs, diagonal block only: -sum fw w_a r (u, n)
// With d = x_c - x_r and D = [d]_x (D v = d x v), the column node's
// u_c = u - D n, so the block J_a^T ... sum is
//   [[S_uu + S_un D, S_un], [S_un^T + S_nn D, S_nn]],
// the off-diagonal block of kernels/solver_kernels.cu:113-137 regrouped (the
// diagonal block is the same with D = 0).
constexpr int kSums = 21;
constexpr int kPartVals = 27;
__host__ __device__ constexpr int sym3(int p, int q) {
  return p <= q ? p * 3 - p * (p - 1) / 2 + (q - p) : q * 3 - q * (q - 1) / 2 + (p - q);
}

// One CTA per block row r.
//  1. stage: the row's entry list, its incidences' slots and records
//     (cp.async, one wait), then each staged incidence's factors U and N
//  2. windows: the row's blocks (diagonal first, then the upper off-diagonal
//     blocks) are cut into windows of 32 entries; warp w takes a contiguous
//     run of W/8 windows, accumulates lane-private sums of the 21 products of
//     g (u, n) (u, n)^T (and the rhs for the diagonal) and, whenever it
//     leaves a block, reduce-scatters them into a partial slot of that block
//  3. combine: per block, the warps' partials in warp order (Kahan on the
//     diagonal block); then per block value its expansion, the ARAP terms of
//     the block's edges (precomputed by the residual launch) and the damping;
//     blocks written with their transposes, the rhs and the row's ARAP energy.
__global__ void __launch_bounds__(kThreads, 3) assemble_kernel(Work w, Pattern pt, AsmArgs aa) {
  extern __shared__ float4 stage_buf[];
  // the row's metadata (written by the expand, longest rows first)
  const int4 m0 = __ldg(w.asm_meta + 3 * (size_t)blockIdx.x), m1 = __ldg(w.asm_meta + 3 * (size_t)blockIdx.x + 1),
             m2 = __ldg(w.asm_meta + 3 * (size_t)blockIdx.x + 2);
  const int r = m0.x, lane = lane_id(), wid = threadIdx.x >> 5;
  const int cap = aa.stage_cap;
  const int i0 = m0.y, n_inc = m0.z;
  const int dpos = m0.w, nb = m1.x;  // upper blocks of the row, diagonal first
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
  float* s_part = reinterpret_cast<float*>(s_erole + kRowEdges);  // [U+8][27]
  float* s_sum = s_part + (size_t)(U + kWarps) * kPartVals;       // [U][27] the blocks' sums
  RowRecords R;
  R.ns = min(n_inc, cap);
  R.nt = min(m2.z, 4 * cap);
  R.s_u = stage_buf;
  R.s_n = stage_buf + cap;
  R.s_ws = stage_buf + 2 * cap;
  R.s_a = s_a;
  R.s_trip = s_trip;
  R.inc = w.inc + i0;
  R.trip = w.trip + 4 * (size_t)i0;
  R.xr = node_pos(aa.nodes, r);
  // block info, ARAP terms of the row's edges and of its blocks' edges
  const int u0 = m1.y;
  const int a0 = m1.z, a1 = m1.w, na = min(a1, kRowEdges);
  const int be0 = m2.x;  // the row's off-diagonal upper blocks are u0+1 .. u0+nb-1
  const int be1 = m2.y, nbe = min(be1, kRowEdges);
  // Every plain load is issued before the first cp.async (whose memory
  // clobber would otherwise hold later loads back), so that the row's
  // incidences, ARAP incidences and block information arrive in one round
  // trip after the metadata; everything else is copied asynchronously.
  float4* su = stage_buf;
  float4* sn = stage_buf + cap;
  int ev[kIncPerThread];
#pragma unroll
  for (int k = 0; k < kIncPerThread; k++) {
    const int ii = threadIdx.x + k * kThreads;
    ev[k] = ii < R.ns ? __ldg(R.inc + ii) : 0;
  }
  // (threads from the back take the edges, so that they overlap the block-info loads)
  const int te = kThreads - 1 - threadIdx.x;
  const bool row_edge = te < na, blk_edge = te >= kRowEdges && te < kRowEdges + nbe;
  int einc = 0;
  if (row_edge) einc = __ldg(pt.arap_row_inc + a0 + te);
  else if (blk_edge) einc = __ldg(pt.arap_blk_edge + be0 + (te - kRowEdges));
  for (int k = threadIdx.x; k < nb; k += kThreads) {
    const int pos = dpos + k;
    s_blk[k] = make_int4(pt.seg_off[pos] - 4 * i0, pt.seg_cnt[pos], pt.col_idx[pos], pt.trans_pos[pos]);
    s_boff[k] = k == 0 ? 0 : pt.arap_blk_ptr[u0 + k] - be0;
  }
  // the entries, 16 B at a time (the row's list starts 16-B aligned and
  // holds 4 slots per incidence, so the last chunk stays inside it)
  for (int t4 = threadIdx.x; 4 * t4 < R.nt; t4 += kThreads) cp_async16(s_trip + 4 * t4, R.trip + 4 * t4);
  if (row_edge) {
    const int ed = einc >> 1, role = einc & 1;
    s_erole[te] = role;
    const float4* src = pt.edge_terms + (size_t)kEdgeTerms4 * ed + 7 * role;
#pragma unroll
    for (int k = 0; k < 7; k++) cp_async16(s_eterm + 7 * te + k, src + k);
    if (role == 0) cp_async8(s_eng + te, pt.edge_energy + ed);
    else s_eng[te] = 0.0;
  } else if (blk_edge) {
    const float4* src = pt.edge_terms + (size_t)kEdgeTerms4 * einc + 14;
#pragma unroll
    for (int k = 0; k < 9; k++) cp_async16(s_bterm + 9 * (te - kRowEdges) + k, src + k);
  }
#pragma unroll
  for (int k = 0; k < kIncPerThread; k++) {
    const int ii = threadIdx.x + k * kThreads;
    if (ii < R.ns) {
      const int c = ev[k] >> 2;
      s_a[ii] = ev[k] & 3;
      cp_async16(su + ii, w.c_srcfw + c);
      cp_async16(sn + ii, w.c_nres + c);
      cp_async16(stage_buf + 2 * cap + ii, w.pk_ws + c);
    }
  }
  cp_async_commit_wait_all();
  // each thread turns the records it staged into the factors (its own
  // copies: no barrier needed between the wait and the rewrite)
  for (int ii = threadIdx.x; ii < R.ns; ii += kThreads) {
    float4 u, n;
    RowRecords::factor(su[ii], sn[ii], sel4(R.s_ws[ii], s_a[ii]), R.xr, u, n);
    su[ii] = u;
    sn[ii] = n;
  }
  __syncthreads();
  if (wid == 0) {  // window prefix over the blocks: a warp scan, 32 blocks at a time
    int carry = 0;
    for (int k0 = 0; k0 < nb; k0 += 32) {
      const int k = k0 + lane;
      const int v = k < nb ? (s_blk[k].y + 31) >> 5 : 0;
      int incl = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += x;
      }
      if (k < nb) s_wpre[k] = carry + incl - v;
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) s_wpre[nb] = carry;
  }
  __syncthreads();

  // ---- 2. windows ----
  const int W = s_wpre[nb];
  const int wa = (int)((long long)W * wid / kWarps), wb = (int)((long long)W * (wid + 1) / kWarps);
  int k = 0;
  while (k < nb && s_wpre[k + 1] <= wa) k++;
  // lane-private sums (the layout above); the 5 slots past the diagonal
  // block's 27 stay zero for the reduce-scatter
  float acc[32];
#pragma unroll
  for (int q = 0; q < 32; q++) acc[q] = 0.f;
  int seg0 = k < nb ? s_blk[k].x : 0, segn = k < nb ? s_blk[k].y : 0;
  for (int win = wa; win < wb; win++) {
    const int t = seg0 + (win - s_wpre[k]) * 32 + lane;
    if (t < seg0 + segn) {
      const int e = R.entry(t);
      const int ii = e >> 2, b = e & 3;
      float4 u, n, w4;
      int a;
      R.get(w, ii, u, n, w4, a);
      const float g = u.w * sel4(w4, b);
      if (g != 0.f) {
        const float gu[3] = {g * u.x, g * u.y, g * u.z};
        const float gn[3] = {g * n.x, g * n.y, g * n.z};
        const float uu[3] = {u.x, u.y, u.z};
        const float nn[3] = {n.x, n.y, n.z};
#pragma unroll
        for (int p = 0; p < 3; p++) {
#pragma unroll
          for (int q = p; q < 3; q++) {
            acc[sym3(p, q)] += gu[p] * uu[q];
            acc[15 + sym3(p, q)] += gn[p] * nn[q];
          }
#pragma unroll
          for (int q = 0; q < 3; q++) acc[6 + 3 * p + q] += gu[p] * nn[q];
        }
        if (k == 0 && a == b) {  // (the block index is uniform in the warp)
#pragma unroll
          for (int p = 0; p < 3; p++) {
            acc[21 + p] += -n.w * uu[p];
            acc[24 + p] += -n.w * nn[p];
          }
        }
      }
    }
    // leaving block k (next window belongs to another block, or the run ends)
    if (win + 1 == wb || win + 1 == s_wpre[k + 1]) {
      reduce_scatter32(acc);
      if (lane < kPartVals) s_part[(size_t)(k + wid) * kPartVals + lane] = acc[0];
#pragma unroll
      for (int q = 0; q < 32; q++) acc[q] = 0.f;
      if (win + 1 < wb) {
        k++;
        while (k < nb && s_wpre[k + 1] <= win + 1) k++;
        seg0 = s_blk[k].x;
        segn = s_blk[k].y;
      }
    }
  }
  __syncthreads();

  // ---- 3a. the blocks' sums: the warps' partials in warp order ----
  for (int item = threadIdx.x; item < kPartVals + kSums * (nb - 1); item += kThreads) {
    const int kb = item < kPartVals ? 0 : 1 + (item - kPartVals) / kSums;
    const int v = item < kPartVals ? item : (item - kPartVals) % kSums;
    const int w0 = s_wpre[kb], w1 = s_wpre[kb + 1];
    float tot = 0.f, comp = 0.f;
    for (int ww = 0; ww < kWarps && w1 > w0; ww++) {  // the warps whose window runs met block kb
      const int a_w = (int)((long long)W * ww / kWarps), b_w = (int)((long long)W * (ww + 1) / kWarps);
      if (a_w >= b_w || a_w >= w1 || b_w <= w0) continue;
      const float x = s_part[(size_t)(kb + ww) * kPartVals + v];
      if (kb == 0) kahan_add(tot, comp, x); else tot += x;
    }
    s_sum[(size_t)kb * kPartVals + v] = tot - comp;
  }
  __syncthreads();

  // ---- 3b. per block value: expansion, ARAP terms, damping ----
  const int pos0 = dpos;
  for (int item = threadIdx.x; item < 27 + 36 * (nb - 1); item += kThreads) {
    int kb, v;
    if (item < 27) {
      kb = 0;
      v = item;
    } else {
      kb = 1 + (item - 27) / 36;
      v = (item - 27) % 36;
    }
    const float* S = s_sum + (size_t)kb * kPartVals;
    const int pos = pos0 + kb;
    if (kb == 0) {
      // diagonal block: upper triangle tri(p, q) (21) and the rhs (6)
      float tot, comp = 0.f;
      int p = 0, q = 0;
      if (v < 21) {
        while (tri(p, 5) < v) p++;
        q = v - tri(p, p) + p;
        tot = p < 3 ? (q < 3 ? S[sym3(p, q)] : S[6 + 3 * p + (q - 3)]) : S[15 + sym3(p - 3, q - 3)];
      } else {
        tot = S[v];
      }
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
        // damping on the diagonal entries (solver_kernels.cu:183-193)
        if (p == q) tot = tot + aa.lambda_damping * fmaxf(fabsf(tot), p < 3 ? 1e-3f : 1e-2f);
        float* out = pt.values + (size_t)pos * 36;
        out[p * 6 + q] = tot;
        out[q * 6 + p] = tot;
      } else {
        w.rhs[r * 6 + (v - 21)] = tot;
      }
    } else {
      const int p = v / 6, q = v % 6;
      float tot;
      if (p < 3 && q >= 3) {
        tot = S[6 + 3 * p + (q - 3)];  // S_un
      } else if (p >= 3 && q >= 3) {
        tot = S[15 + sym3(p - 3, q - 3)];  // S_nn
      } else {
        // (S_uu + S_un D)[p][q] or (S_un^T + S_nn D)[p - 3][q]:
        // D[k][q] = e_k . (d x e_q), d = x_c - x_r
        const float3 xc = node_pos(aa.nodes, s_blk[kb].z);
        const float d[3] = {xc.x - R.xr.x, xc.y - R.xr.y, xc.z - R.xr.z};
        // column q of D: d x e_q
        const float dq[3] = {q == 0 ? 0.f : q == 1 ? -d[2] : d[1], q == 0 ? d[2] : q == 1 ? 0.f : -d[0],
                             q == 0 ? -d[1] : q == 1 ? d[0] : 0.f};
        if (p < 3) {
          tot = S[sym3(p, q)] + S[6 + 3 * p] * dq[0] + S[6 + 3 * p + 1] * dq[1] + S[6 + 3 * p + 2] * dq[2];
        } else {
          const int pp = p - 3;
          tot = S[6 + 3 * q + pp] + S[15 + sym3(pp, 0)] * dq[0] + S[15 + sym3(pp, 1)] * dq[1] +
                S[15 + sym3(pp, 2)] * dq[2];
        }
      }
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
         kRowEdges * 8 + Up * (4 + 16 + 4) + kRowEdges * 4 + (2 * max_upper_row + kWarps) * kPartVals * 4;
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
