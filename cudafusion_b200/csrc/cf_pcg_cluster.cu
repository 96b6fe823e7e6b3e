// cf_pcg_cluster.cu — block-Jacobi PCG of one problem inside ONE thread-block
// cluster (sm_100a).
//
// A frame's system (N ~ 2k nodes, ~11k upper 6x6 blocks) fits in the shared
// memory of a 16-CTA cluster when only the upper blocks (col >= row) are
// kept: each CTA holds those of a contiguous range of block rows (balanced by
// upper-block count).  The SpMV uses every stored block twice: A_ij p_j for
// its own row i, and the transposed product A_ij^T p_i, which belongs to row
// j and is pushed into a receive slot of row j's owner (a distributed
// shared-memory store, one slot per lower block, so the owner adds them in a
// fixed order).  The operand p of other CTAs' rows (the CTA's halo) is
// formed locally as z + beta p_old from the owners' z and p_old, read
// through cluster-mapped shared memory, so p itself is never waited for.
// Dot-product partials are stored into every CTA's partial slots, so each
// CTA sums the same values in the same order from its own shared memory.
//
// Three cluster barriers per iteration (after the pushes, after p.Ap, after
// r.r and r.z), no global-memory round trip inside the loop.  Schedule and
// guards follow kernels/solver_kernels.cu:616-687 (PCG from x = 0,
// |p.Ap| < 1e-12 stops before the update, ||r|| < tol after it); FP64 block
// inverses and dot products, FP32 matrix and vectors.
#include <cooperative_groups.h>

#include "cf_device.cuh"
#include "cf_internal.h"

namespace cg = cooperative_groups;

namespace cf {

namespace {

__host__ __device__ inline int al16(int x) { return (x + 15) & ~15; }

constexpr int kInvScratch = (kThreads / 8) * 72 * 8;  // inv6_group scratch, on the receive buffer

struct CluLayout {
  int a, opnd, push, urow, lrow, halo, recv, v0, v1, z, r, x, ap, minv, tn, parts, red, total;
};

// parts: [4 slots][C] -- p.Ap | r.r | r.z | energy share -- one column per CTA
__host__ __device__ inline CluLayout clu_layout(int nup, int nlow, int rows, int nhalo, int C) {
  CluLayout L;
  int o = 0;
  L.a = o; o += al16(nup * 36 * 4);
  L.opnd = o; o += al16(nup * 4);
  L.push = o; o += al16(nup * 4);
  L.urow = o; o += al16((rows + 1) * 4);
  L.lrow = o; o += al16((rows + 1) * 4);
  L.halo = o; o += al16(nhalo * 4);
  {  // the receive buffer doubles as prologue scratch: staged upper positions, then the inverses' scratch
    int rb = al16(nlow * 6 * 4);
    rb = rb > kInvScratch ? rb : kInvScratch;
    rb = rb > al16(nup * 4) ? rb : al16(nup * 4);
    L.recv = o; o += rb;
  }
  L.v0 = o; o += al16((rows + nhalo) * 6 * 4);
  L.v1 = o; o += al16((rows + nhalo) * 6 * 4);
  L.z = o; o += al16(rows * 6 * 4);
  L.r = o; o += al16(rows * 6 * 4);
  L.x = o; o += al16(rows * 6 * 4);
  L.ap = o; o += al16(rows * 6 * 4);
  L.minv = o; o += al16(rows * 36 * 8);
  L.tn = o; o += al16(rows * 48);
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

// CTA sums of NS values (warp sums, then the eight warp sums in a fixed
// tree), stored by lane r of warp 0 into slot slots[k] column `crank` of
// CTA r's partials: after the next cluster barrier every CTA holds every
// CTA's sums in its own shared memory.
template <int NS>
__device__ __forceinline__ void broadcast_sums(const cg::cluster_group& cl, const double (&v)[NS],
                                               const int (&slots)[NS], double* parts, double* red, int C,
                                               int crank) {
  static_assert(kThreads == 256, "eight warps per CTA");
  const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double ws[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) ws[k] = warp_sum_d(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NS; k++) red[k * 8 + wi] = ws[k];
  }
  __syncthreads();
  if (wi == 0 && lane < C) {
    double* dst = cl.map_shared_rank(parts, lane);
#pragma unroll
    for (int k = 0; k < NS; k++) {
      const double* r = red + k * 8;
      dst[slots[k] * C + crank] = ((r[0] + r[4]) + (r[2] + r[6])) + ((r[1] + r[5]) + (r[3] + r[7]));
    }
  }
}

__global__ void __launch_bounds__(kThreads, 1) pcg_cluster_kernel(CluArgs P) {
  extern __shared__ __align__(16) unsigned char smem[];
  cg::cluster_group cluster = cg::this_cluster();
  const Work& w = P.w;
  const Pattern& pt = P.pt;
  const SolveArgs& a = P.a;
  const int C = (int)cluster.num_blocks();
  const int crank = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  const ProbDesc pd = a.tb.desc[0];  // the cluster path serves single solves
  DevStats* st = w.stats;
  const int r0 = pt.clu_row_begin[crank], r1 = pt.clu_row_begin[crank + 1];
  const int nrows = r1 - r0;
  const int u0 = pt.ustart[r0], nup = pt.ustart[r1] - u0;
  const int l0 = pt.low_ptr[r0];
  const int h0 = pt.clu_halo_ptr[crank], nhalo = pt.clu_halo_ptr[crank + 1] - h0;
  const CluLayout L = clu_layout(pt.clu_nup_max, pt.clu_nlow_max, pt.clu_rows_max, pt.clu_halo_max, C);
  float* sA = reinterpret_cast<float*>(smem + L.a);
  int* sOpnd = reinterpret_cast<int*>(smem + L.opnd);
  int* sPush = reinterpret_cast<int*>(smem + L.push);
  int* sUrow = reinterpret_cast<int*>(smem + L.urow);
  int* sLrow = reinterpret_cast<int*>(smem + L.lrow);
  int* sHalo = reinterpret_cast<int*>(smem + L.halo);
  float* sRecv = reinterpret_cast<float*>(smem + L.recv);
  float* sV0 = reinterpret_cast<float*>(smem + L.v0);
  float* sV1 = reinterpret_cast<float*>(smem + L.v1);
  float* sZ = reinterpret_cast<float*>(smem + L.z);
  float* sR = reinterpret_cast<float*>(smem + L.r);
  float* sX = reinterpret_cast<float*>(smem + L.x);
  float* sAp = reinterpret_cast<float*>(smem + L.ap);
  double* sMinv = reinterpret_cast<double*>(smem + L.minv);
  float4* sTn = reinterpret_cast<float4*>(smem + L.tn);
  double* sParts = reinterpret_cast<double*>(smem + L.parts);
  double* sRed = reinterpret_cast<double*>(smem + L.red);
  const int n6 = nrows * 6, h6 = nhalo * 6;
  int spl_log = 0;  // lanes per row element of the SpMV: 1, 2 or 4, all in one pass
  while (spl_log < 2 && (n6 << (spl_log + 1)) <= kThreads) spl_log++;
  const int spl = 1 << spl_log;
  int* err = w.err;
  PhaseClock clk((a.timers && crank == 0 && tid == 0) ? a.timers : nullptr);

  // Distributed shared memory may be touched only once every CTA of the
  // cluster runs: arrive now, wait before the first remote store.
  asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");

  // ---- prologue: indices, then the upper blocks, all by cp.async ----
  int* sUpos = reinterpret_cast<int*>(smem + L.recv);  // staged upper positions (receive buffer unused yet)
  for (int k = tid; k < nup; k += kThreads) {
    cp_async4(sUpos + k, pt.upper_pos + u0 + k);
    cp_async4(sOpnd + k, pt.clu_opnd + u0 + k);
    cp_async4(sPush + k, pt.clu_push + u0 + k);
  }
  for (int k = tid; k < nhalo; k += kThreads) cp_async4(sHalo + k, pt.clu_halo + h0 + k);
  if (!a.delta_x)  // the epilogue's operands (transform, node position)
    for (int i = tid; i < nrows; i += kThreads) {
      const float4* tq = reinterpret_cast<const float4*>(a.transforms + r0 + i);
      cp_async16(sTn + 3 * i, tq);
      cp_async16(sTn + 3 * i + 1, tq + 1);
      const float* np = reinterpret_cast<const float*>(a.nodes + r0 + i);
      float* sp = reinterpret_cast<float*>(sTn + 3 * i + 2);
      cp_async4(sp, np);
      cp_async4(sp + 1, np + 1);
      cp_async4(sp + 2, np + 2);
    }
  for (int i = tid; i <= nrows; i += kThreads) {
    sUrow[i] = pt.ustart[r0 + i] - u0;
    sLrow[i] = pt.low_ptr[r0 + i] - l0;
  }
  cp_async_commit_wait_all();
  __syncthreads();
  for (int e = tid; e < nup * 9; e += kThreads) {
    const int k = e / 9, q = e - 9 * k;
    cp_async16(sA + 36 * k + 4 * q, pt.values + (size_t)sUpos[k] * 36 + 4 * q);
  }
  cp_async_commit_wait_all();
  __syncthreads();
  clk.mark(0);  // staging
  // block-Jacobi inverses in FP64, one 8-lane group per row (the first upper
  // block of a row is its diagonal)
  {
    double* scr = reinterpret_cast<double*>(smem + L.recv) + (tid >> 3) * 72;
    int nfb = 0;
    for (int i0 = 0; i0 < nrows; i0 += kThreads / 8) {
      const int i = i0 + (tid >> 3);
      const bool act = i < nrows;
      nfb += inv6_group(sA + (act ? sUrow[i] : 0) * 36, scr, sMinv + (act ? i : 0) * 36, act) && (tid & 7) == 0;
    }
    if (nfb) atomicAdd(&st->fallbacks, nfb);
  }
  __syncthreads();
  clk.mark(1);  // inverses
  // r = b, x = 0, z = M^-1 r; this CTA's share of the energy at the
  // linearisation point (the data partials, then the ARAP node partials)
  auto minv_row = [&](int t) -> double {
    const int i = t / 6, c = t % 6;
    const double* Mi = sMinv + i * 36 + c * 6;
    const float* ri = sR + i * 6;
    double zz = 0.0;
#pragma unroll
    for (int q = 0; q < 6; q++) zz += Mi[q] * (double)ri[q];
    return zz;
  };
  double prz = 0.0, pbb = 0.0, pen = 0.0;
  for (int t = tid; t < n6; t += kThreads) {
    const float rt = __ldcg(w.rhs + r0 * 6 + t);
    sR[t] = rt;
    sX[t] = 0.f;
    pbb += (double)rt * rt;
  }
  {
    const int n1 = pd.e_ctas, n = pd.e_ctas + pd.N, chunk = (n + C - 1) / C;
    const int k1 = min(n, (crank + 1) * chunk);
    for (int k0 = crank * chunk + tid; k0 < k1; k0 += kThreads * 4) {
      double x[4];
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const int k = k0 + kThreads * b;
        x[b] = k < k1 ? (k < n1 ? __ldcg(w.e_data_part + pd.e_cta0 + k) : __ldcg(w.e_arap_part + pd.node_off + (k - n1)))
                      : 0.0;
      }
#pragma unroll
      for (int b = 0; b < 4; b++)
        if (k0 + kThreads * b < k1) pen += x[b];
    }
  }
  __syncthreads();
  for (int t = tid; t < n6; t += kThreads) {
    const float zf = (float)minv_row(t);
    sZ[t] = zf;
    prz += (double)sR[t] * zf;
  }
  asm volatile("barrier.cluster.wait.aligned;" ::: "memory");
  {
    const double v3[3] = {pbb, prz, pen};
    const int s3[3] = {1, 2, 3};
    broadcast_sums<3>(cluster, v3, s3, sParts, sRed, C, crank);
  }
  clk.mark(2);  // r, z, energy share
  cluster.sync();  // C0: every CTA's z, the first partials and (first of all) every CTA is running
  if (crank == 0 && tid == 0) {
    double e = 0.0;
    for (int r = 0; r < C; r++) e += sParts[3 * C + r];
    st->energy[P.slot] = e;
    if (!isfinite(e)) atomicOr(err, kErrNonFinite);
  }
  clk.mark(3);  // C0

  double rz = 0.0, rr_last = 0.0;
  int used = 0;
  float betaf = 0.f;
  for (int it = 0;; it++) {
    // ---- the last reduction, from this CTA's copies of every CTA's partials ----
    {
      double srr = 0.0, srz = 0.0;
      for (int r = 0; r < C; r++) {
        srr += sParts[1 * C + r];
        srz += sParts[2 * C + r];
      }
      if (it == 0) {
        rz = srz;
        rr_last = srr;
      } else {
        used = it;
        rr_last = srr;
        if (sqrt(srr) < (double)a.pcg_tolerance) break;  // solver_kernels.cu:669
        betaf = (float)(srz / rz);
        rz = srz;
      }
    }
    if (it >= a.pcg_iterations) break;
    clk.mark(4);  // reduction
    float* V = (it & 1) ? sV1 : sV0;
    float* Vold = (it & 1) ? sV0 : sV1;
    // ---- p = z + beta p_old: own rows, and the halo from the owners' z and p_old ----
    for (int t = tid; t < n6; t += kThreads) V[t] = (it == 0) ? sZ[t] : __fmaf_rn(betaf, Vold[t], sZ[t]);
    for (int e = tid; e < h6; e += kThreads) {
      const int hk = sHalo[e / 6], o = hk >> 24, jl = hk & 0xffffff, c = e % 6;
      const float zr = cluster.map_shared_rank(sZ, o)[jl * 6 + c];
      V[n6 + e] = (it == 0) ? zr : __fmaf_rn(betaf, cluster.map_shared_rank(Vold, o)[jl * 6 + c], zr);
    }
    __syncthreads();
    clk.mark(5);  // p and halo
    // ---- Ap (solver_kernels.cu:406-432): the upper blocks of own rows, and
    //      their transposed products pushed to the rows of their columns.
    //      spl adjacent lanes per row element (as many as the CTA's threads
    //      allow, up to 4): lane k takes the row's blocks k, k + spl, ...,
    //      the lanes' sums combined by an xor butterfly ----
    for (int u0 = 0; u0 < n6 * spl; u0 += kThreads) {
      const int u = u0 + tid, t = u >> spl_log, kk = u & (spl - 1);
      float y = 0.f;
      if (t < n6) {
        const int i = t / 6, c = t % 6;
        float pi[6];
#pragma unroll
        for (int q = 0; q < 6; q++) pi[q] = V[i * 6 + q];
        for (int k = sUrow[i] + kk; k < sUrow[i + 1]; k += spl) {
          const float* Ab = sA + k * 36;
          const float* vj = V + sOpnd[k] * 6;
#pragma unroll
          for (int q = 0; q < 6; q++) y = __fmaf_rn(Ab[c * 6 + q], vj[q], y);
          const int pk = sPush[k];
          if (pk >= 0) {
            float uu = 0.f;
#pragma unroll
            for (int q = 0; q < 6; q++) uu = __fmaf_rn(Ab[q * 6 + c], pi[q], uu);
            cluster.map_shared_rank(sRecv, pk >> 24)[(pk & 0xffffff) * 6 + c] = uu;
          }
        }
      }
      for (int o = spl >> 1; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
      if (kk == 0 && t < n6) sAp[t] = y;
    }
    clk.mark(6);  // upper products, pushes
    cluster.sync();  // B: every transposed product delivered
    clk.mark(7);
    double ppap = 0.0;
    for (int t = tid; t < n6; t += kThreads) {
      const int i = t / 6, c = t % 6;
      float y = sAp[t];
      for (int l = sLrow[i]; l < sLrow[i + 1]; l++) y += sRecv[l * 6 + c];
      sAp[t] = y;
      ppap += (double)V[t] * y;
    }
    {
      const double v1[1] = {ppap};
      const int s1[1] = {0};
      broadcast_sums<1>(cluster, v1, s1, sParts, sRed, C, crank);
    }
    clk.mark(8);  // received products, p.Ap
    cluster.sync();  // A: p.Ap
    clk.mark(9);
    double pAp = 0.0;
    for (int r = 0; r < C; r++) pAp += sParts[r];
    if (fabs(pAp) < 1e-12) break;  // solver_kernels.cu:647-653
    const float af = (float)(rz / pAp);
    for (int t = tid; t < n6; t += kThreads) {
      sX[t] = __fmaf_rn(af, V[t], sX[t]);
      sR[t] = __fmaf_rn(-af, sAp[t], sR[t]);
    }
    __syncthreads();
    double prr = 0.0, przn = 0.0;
    for (int t = tid; t < n6; t += kThreads) {
      const float zf = (float)minv_row(t);
      sZ[t] = zf;
      prr += (double)sR[t] * sR[t];
      przn += (double)sR[t] * zf;
    }
    {
      const double v2[2] = {prr, przn};
      const int s2[2] = {1, 2};
      broadcast_sums<2>(cluster, v2, s2, sParts, sRed, C, crank);
    }
    clk.mark(10);  // x, r, z
    cluster.sync();  // C: r.r and r.z
    clk.mark(11);
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
      DQ T0;
      T0.r = sTn[3 * i];
      T0.d = sTn[3 * i + 1];
      const float4 xp = sTn[3 * i + 2];
      DQ Tn = twist_update(T0, sX + i * 6, pd.max_rot, pd.max_trans, pd.update_scale);
      store_dq(a.transforms + node, Tn);
      store_dq(w.plain + node, dq_centered(Tn, f3(xp.x, xp.y, xp.z)));
    }
  }
  clk.mark(12);  // epilogue
  clk.flush();
  if (crank == 0 && tid == 0) {
    st->pcg_iters[P.slot] = used;
    st->pcg_res[P.slot] = sqrt(rr_last);
  }
}

cudaError_t config_kernel(int C, int smem) {
  // the device's opt-in maximum, not this plan's size: another handle's plan
  // (with more shared memory) launches the same kernel
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (smem > optin) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(pcg_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
  if (e != cudaSuccess) return e;
  if (C > 8) e = cudaFuncSetAttribute(pcg_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

}  // namespace

int pcg_cluster_smem_bytes(int nup_max, int nlow_max, int rows_max, int nhalo_max, int C) {
  return clu_layout(nup_max, nlow_max, rows_max, nhalo_max, C).total;
}

int pcg_cluster_max_active(int C, int smem) {
  if (config_kernel(C, smem) != cudaSuccess) {
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
  if (cudaOccupancyMaxActiveClusters(&n, pcg_cluster_kernel, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
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
  return cudaLaunchKernelEx(&cfg, pcg_cluster_kernel, P);
}

}  // namespace cf
