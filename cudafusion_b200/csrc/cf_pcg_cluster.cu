// cf_pcg_cluster.cu — block-Jacobi PCG of one problem inside ONE thread-block
// cluster (sm_100a).
//
// The system of a frame (N ~ 2k nodes, ~11k upper 6x6 blocks) fits in the
// distributed shared memory of a 16-CTA cluster.  Each CTA keeps the upper
// blocks (col >= row) of a contiguous range of block rows in its shared
// memory; the lower blocks are read transposed from the CTA that owns them
// (ld through cluster-mapped shared memory), the search direction p of other
// CTAs is read the same way, and the dot-product partials are exchanged in
// the leader CTA's shared memory.  All synchronisation is the hardware
// cluster barrier: no global-memory round trip inside the PCG loop.
// Schedule and guards follow kernels/solver_kernels.cu:616-687 (PCG from
// x = 0, |p.Ap| < 1e-12 stops before the update, ||r|| < tol after it);
// FP64 block inverses and dot products, FP32 matrix and vectors.
#include <cooperative_groups.h>

#include "cf_device.cuh"
#include "cf_internal.h"

namespace cg = cooperative_groups;

namespace cf {

namespace {

__host__ __device__ inline int al16(int x) { return (x + 15) & ~15; }

struct CluLayout {
  int a, ucol, urow, lpk, lrow, pgu, pgl, p, z, r, x, ap, minv, scr, parts, red, total;
};

__host__ __device__ inline CluLayout clu_layout(int nup, int nlow, int rows, int C, bool a_smem) {
  CluLayout L;
  int o = 0;
  L.a = o; o += a_smem ? al16(nup * 36 * 4) : 0;
  L.ucol = o; o += al16(nup * 4);
  L.urow = o; o += al16((rows + 1) * 4);
  L.lpk = o; o += al16(nlow * 8);
  L.lrow = o; o += al16((rows + 1) * 4);
  L.pgu = o; o += al16(nup * 6 * 4);
  L.pgl = o; o += al16(nlow * 6 * 4);
  L.p = o; o += al16(rows * 6 * 4);
  L.z = o; o += al16(rows * 6 * 4);
  L.r = o; o += al16(rows * 6 * 4);
  L.x = o; o += al16(rows * 6 * 4);
  L.ap = o; o += al16(rows * 6 * 4);
  L.minv = o; o += al16(rows * 36 * 8);
  L.scr = o; o += (kThreads / 8) * 72 * 8;
  L.parts = o; o += al16(4 * C * 8);
  L.red = o; o += 64 * 8;
  L.total = o;
  return L;
}

struct CluArgs {
  Work w;
  Pattern pt;
  SolveArgs a;
  int slot;
};

__device__ __forceinline__ double block_sum(double v, double* red) {
  v = warp_sum_d(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
    t = warp_sum_d(t);
  }
  return t;
}

// Sum of the C partials of slot s held by the leader; same bits on every CTA.
__device__ __forceinline__ double cluster_total(const double* leader_parts, int s, int C, double* bcast) {
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x & 31;
    double v = (lane < C) ? leader_parts[s * C + lane] : 0.0;
    v = warp_sum_d(v);
    if (lane == 0) *bcast = v;
  }
  __syncthreads();
  double t = *bcast;
  __syncthreads();
  return t;
}

template <bool A_SMEM>
__global__ void __launch_bounds__(kThreads, 1) pcg_cluster_kernel(CluArgs P) {
  extern __shared__ __align__(16) unsigned char smem[];
  cg::cluster_group cluster = cg::this_cluster();
  const Work& w = P.w;
  const Pattern& pt = P.pt;
  const SolveArgs& a = P.a;
  const int C = (int)cluster.num_blocks();
  const int crank = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  const int r0 = pt.clu_row_begin[crank], r1 = pt.clu_row_begin[crank + 1];
  const int nrows = r1 - r0;
  const int u0 = pt.ustart[r0], u1 = pt.ustart[r1];
  const int nup = u1 - u0;
  const int l0 = pt.low_ptr[r0], l1 = pt.low_ptr[r1];
  const int nlow = l1 - l0;
  const CluLayout L = clu_layout(pt.clu_nup_max, pt.clu_nlow_max, pt.clu_rows_max, C, A_SMEM);
  float* sA = reinterpret_cast<float*>(smem + L.a);
  int* sUcol = reinterpret_cast<int*>(smem + L.ucol);
  int* sUrow = reinterpret_cast<int*>(smem + L.urow);
  int2* sLpk = reinterpret_cast<int2*>(smem + L.lpk);
  int* sLrow = reinterpret_cast<int*>(smem + L.lrow);
  float* sPgu = reinterpret_cast<float*>(smem + L.pgu);
  float* sPgl = reinterpret_cast<float*>(smem + L.pgl);
  float* sP = reinterpret_cast<float*>(smem + L.p);
  float* sZ = reinterpret_cast<float*>(smem + L.z);
  float* sR = reinterpret_cast<float*>(smem + L.r);
  float* sX = reinterpret_cast<float*>(smem + L.x);
  float* sAp = reinterpret_cast<float*>(smem + L.ap);
  double* sMinv = reinterpret_cast<double*>(smem + L.minv);
  double* sParts = reinterpret_cast<double*>(smem + L.parts);
  double* sRed = reinterpret_cast<double*>(smem + L.red);
  double* lparts = cluster.map_shared_rank(sParts, 0);
  const int n6 = nrows * 6;
  int* err = w.err;

  // ---- prologue ----
  cluster.sync();  // every CTA of the cluster is running before any DSMEM access
  for (int e = tid; e < nup * 9; e += kThreads) {
    const int k = e / 9, q = e % 9;
    const float4* g = reinterpret_cast<const float4*>(pt.values + (size_t)pt.upper_pos[u0 + k] * 36);
    if (A_SMEM) reinterpret_cast<float4*>(sA)[e] = __ldcg(g + q);
    if (q == 0) sUcol[k] = pt.col_idx[pt.upper_pos[u0 + k]];
  }
  for (int i = tid; i <= nrows; i += kThreads) {
    sUrow[i] = pt.ustart[r0 + i] - u0;
    sLrow[i] = pt.low_ptr[r0 + i] - l0;
  }
  for (int k = tid; k < nlow; k += kThreads) sLpk[k] = make_int2(pt.low_pack[l0 + k], pt.low_jl[l0 + k]);
  __syncthreads();
  // block-Jacobi inverses in FP64, one 8-lane group per row
  {
    double* scr = reinterpret_cast<double*>(smem + L.scr) + (tid >> 3) * 72;
    int nfb = 0;
    for (int i0 = 0; i0 < nrows; i0 += kThreads / 8) {
      const int i = i0 + (tid >> 3);
      const bool act = i < nrows;
      const int k = act ? sUrow[i] : 0;  // first upper block of a row is its diagonal
      const float* blk = A_SMEM ? (sA + k * 36) : (pt.values + (size_t)pt.upper_pos[u0 + k] * 36);
      nfb += inv6_group(blk, scr, sMinv + (act ? i : 0) * 36, act) && (tid & 7) == 0;
    }
    if (nfb) atomicAdd(&w.stats->fallbacks, nfb);
  }
  __syncthreads();
  double prz = 0.0, pbb = 0.0;
  for (int t = tid; t < n6; t += kThreads) {
    const int i = t / 6, c = t % 6;
    float ri[6];
#pragma unroll
    for (int q = 0; q < 6; q++) ri[q] = __ldcg(w.rhs + (r0 + i) * 6 + q);
    const double* Mi = sMinv + i * 36 + c * 6;
    double zz = 0.0;
#pragma unroll
    for (int q = 0; q < 6; q++) zz += Mi[q] * (double)ri[q];
    const float zf = (float)zz;
    sR[t] = ri[c];
    sX[t] = 0.f;
    sZ[t] = zf;
    sP[t] = zf;
    prz += (double)ri[c] * (double)zf;
    pbb += (double)ri[c] * (double)ri[c];
  }
  {
    double t1 = block_sum(prz, sRed);
    double t2 = block_sum(pbb, sRed + 8);
    if (tid == 0) {
      lparts[0 * C + crank] = t1;
      lparts[1 * C + crank] = t2;
    }
  }
  if (crank == 0 && tid >= 32 && tid < 64) {  // energy of this linearisation point
    double v = 0.0;
    const int ne = a.tb.desc[0].e_ctas;  // the cluster path serves single solves
    for (int k = tid - 32; k < ne; k += 32) v += w.e_data_part[k];
    for (int k = tid - 32; k < a.N; k += 32) v += w.e_arap_part[k];
    v = warp_sum_d(v);
    if (tid == 32) {
      w.stats->energy[P.slot] = v;
      if (!isfinite(v)) atomicOr(err, kErrNonFinite);
    }
  }
  cluster.sync();
  double rz = cluster_total(lparts, 0, C, sRed + 16);
  double rr_last = cluster_total(lparts, 1, C, sRed + 16);
  int used = 0;
  float betaf = 0.f;
  for (int it = 0; it < a.pcg_iterations; it++) {
    if (it > 0) {
      for (int t = tid; t < n6; t += kThreads) sP[t] = __fmaf_rn(betaf, sP[t], sZ[t]);
    }
    cluster.sync();  // p of every CTA final
    // ---- gather p for the upper and lower blocks (local or cluster-mapped) ----
    for (int e = tid; e < nup * 6; e += kThreads) {
      const int k = e / 6, c = e % 6;
      const int j = sUcol[k];
      float v;
      if (j >= r0 && j < r1) {
        v = sP[(j - r0) * 6 + c];
      } else {
        const int owner = pt.cta_of_row[j];
        const float* rp = cluster.map_shared_rank(sP, owner);
        v = rp[(j - pt.clu_row_begin[owner]) * 6 + c];
      }
      sPgu[e] = v;
    }
    for (int e = tid; e < nlow * 6; e += kThreads) {
      const int k = e / 6, c = e % 6;
      const int2 pk = sLpk[k];
      const int owner = pk.x >> 24;
      const float* rp = (owner == crank) ? sP : cluster.map_shared_rank(sP, owner);
      sPgl[e] = rp[pk.y * 6 + c];
    }
    __syncthreads();
    // ---- Ap = sum_upper A_ij p_j + sum_lower A_ji^T p_j ----
    double ppap = 0.0;
    for (int t = tid; t < n6; t += kThreads) {
      const int i = t / 6, c = t % 6;
      float acc = 0.f;
      for (int k = sUrow[i]; k < sUrow[i + 1]; k++) {
        const float* Ab = A_SMEM ? (sA + k * 36 + c * 6) : (pt.values + (size_t)pt.upper_pos[u0 + k] * 36 + c * 6);
        const float* pg = sPgu + k * 6;
#pragma unroll
        for (int q = 0; q < 6; q++) acc = __fmaf_rn(A_SMEM ? Ab[q] : __ldcg(Ab + q), pg[q], acc);
      }
      for (int k = sLrow[i]; k < sLrow[i + 1]; k++) {
        const int2 pk = sLpk[k];
        const int owner = pk.x >> 24, slot = pk.x & 0xffffff;
        const float* pg = sPgl + k * 6;
        if (A_SMEM) {
          const float* Ab = ((owner == crank) ? sA : cluster.map_shared_rank(sA, owner)) + slot * 36 + c;
#pragma unroll
          for (int q = 0; q < 6; q++) acc = __fmaf_rn(Ab[q * 6], pg[q], acc);
        } else {
          const int u = pt.ustart[pt.clu_row_begin[owner]] + slot;
          const float* Ab = pt.values + (size_t)pt.upper_pos[u] * 36 + c;
#pragma unroll
          for (int q = 0; q < 6; q++) acc = __fmaf_rn(__ldcg(Ab + q * 6), pg[q], acc);
        }
      }
      sAp[t] = acc;
      ppap += (double)sP[t] * (double)acc;
    }
    {
      double t1 = block_sum(ppap, sRed);
      if (tid == 0) lparts[2 * C + crank] = t1;
    }
    cluster.sync();
    const double pAp = cluster_total(lparts, 2, C, sRed + 16);
    if (fabs(pAp) < 1e-12) break;  // solver_kernels.cu:647-653
    const float af = (float)(rz / pAp);
    double prr = 0.0, przn = 0.0;
    for (int t = tid; t < n6; t += kThreads) {
      sX[t] = __fmaf_rn(af, sP[t], sX[t]);
      sR[t] = __fmaf_rn(-af, sAp[t], sR[t]);
    }
    __syncthreads();
    for (int t = tid; t < n6; t += kThreads) {
      const int i = t / 6, c = t % 6;
      const double* Mi = sMinv + i * 36 + c * 6;
      const float* ri = sR + i * 6;
      double zz = 0.0;
#pragma unroll
      for (int q = 0; q < 6; q++) zz += Mi[q] * (double)ri[q];
      const float zf = (float)zz;
      sZ[t] = zf;
      prr += (double)sR[t] * (double)sR[t];
      przn += (double)sR[t] * (double)zf;
    }
    {
      double t2 = block_sum(prr, sRed);
      double t3 = block_sum(przn, sRed + 8);
      if (tid == 0) {
        lparts[0 * C + crank] = t2;
        lparts[1 * C + crank] = t3;
      }
    }
    cluster.sync();
    const double rr = cluster_total(lparts, 0, C, sRed + 16);
    const double rzn = cluster_total(lparts, 1, C, sRed + 16);
    used = it + 1;
    rr_last = rr;
    if (sqrt(rr) < (double)a.pcg_tolerance) break;  // solver_kernels.cu:669
    betaf = (float)(rzn / rz);
    rz = rzn;
  }
  cluster.sync();  // no CTA leaves while others may still read its shared memory

  // ---- epilogue ----
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
  if (crank == 0 && tid == 0) {
    w.stats->pcg_iters[P.slot] = used;
    w.stats->pcg_res[P.slot] = sqrt(rr_last);
  }
}

template <bool A_SMEM>
cudaError_t config_kernel(int C, int smem) {
  auto k = pcg_cluster_kernel<A_SMEM>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  if (C > 8) e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

template <bool A_SMEM>
int max_clusters(int C, int smem) {
  if (config_kernel<A_SMEM>(C, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, pcg_cluster_kernel<A_SMEM>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

}  // namespace

int pcg_cluster_smem_bytes(int nup_max, int nlow_max, int rows_max, int C, bool a_in_smem) {
  return clu_layout(nup_max, nlow_max, rows_max, C, a_in_smem).total;
}

int pcg_cluster_max_active(int C, int smem, bool a_in_smem) {
  return a_in_smem ? max_clusters<true>(C, smem) : max_clusters<false>(C, smem);
}

cudaError_t launch_pcg_cluster(const Work& w, const Pattern& p, const SolveArgs& a, int gn_slot, cudaStream_t s) {
  if (a.N <= 0) return cudaSuccess;
  CluArgs P;
  P.w = w;
  P.pt = p;
  P.a = a;
  P.slot = gn_slot;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(p.clu_C);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = p.clu_smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = p.clu_C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (p.clu_a_in_smem) return cudaLaunchKernelEx(&cfg, pcg_cluster_kernel<true>, P);
  return cudaLaunchKernelEx(&cfg, pcg_cluster_kernel<false>, P);
}

}  // namespace cf
