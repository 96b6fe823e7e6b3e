// cf_pcg_grid.cu — persistent cooperative block-Jacobi PCG over the whole GPU.
//
// One cooperative launch per GN iteration.  Each CTA owns a contiguous range
// of block rows (balanced by block count); its rows of A stay in shared memory
// for the whole solve, its block-Jacobi inverses are computed in FP64 in the
// prologue, and its state vectors never leave shared memory.  Only the
// exchange vector of the halo (the columns of other CTAs' rows that this
// CTA's blocks touch, a deduplicated per-CTA list) and the dot-product
// partials go through global memory, around a fence-free release/acquire
// grid barrier with a bounded wait.
//
// Two schedules (kernels/solver_kernels.cu:616-687 semantics in both: x0 = 0,
// |p.Ap| < 1e-12 stops before the update, ||r|| < tol after it):
//   standard   the reference's PCG; FP32 vectors, FP64 dot products; two
//              reductions per iteration.  p of the halo is formed locally as
//              z + beta*p_old from the exchanged z and p_old, so p itself is
//              never waited for.
//   pipelined  Ghysels-Vanroose pipelined PCG: the same iterates in exact
//              arithmetic with ONE reduction (gamma, delta, ||r||^2) per
//              iteration overlapped with the SpMV operand exchange; its
//              recurrences run in FP64 (the SpMV stays FP32).
#include "cf_device.cuh"
#include "cf_internal.h"

namespace cf {

namespace {

__host__ __device__ inline int gal16(int x) { return (x + 15) & ~15; }

struct GLayout {
  int a, vidx, rowptr, halo, v, minv, scr, st, red, tn, total;
};

// v : the SpMV operand, [own rows | halo] x 6 floats.
// st: standard  -> z, x, r, ap (FP32, own rows) + halo z and halo p_old;
//     pipelined -> x r u w z q s p (FP64, own rows) + n (FP32, own rows).
__host__ __device__ inline GLayout glayout(int nblk, int nrows, int nhalo, bool a_smem, bool pipe) {
  GLayout L;
  int o = 0;
  L.a = o; o += a_smem ? gal16(nblk * 36 * 4) : 0;
  L.vidx = o; o += gal16(nblk * 4);
  L.rowptr = o; o += gal16((nrows + 1) * 4);
  L.halo = o; o += gal16(nhalo * 4);
  L.v = o; o += gal16((nrows + nhalo) * 6 * 4);
  L.minv = o; o += gal16(nrows * 36 * 8);
  L.scr = o; o += (kThreads / 8) * 72 * 8;  // inversion scratch, 72 doubles per 8-lane group
  L.st = o;
  o += pipe ? gal16(nrows * 6 * 8) * 8 + gal16(nrows * 6 * 4) : gal16((nrows + nhalo) * 6 * 4) + gal16(nrows * 6 * 4) * 4;
  L.red = o; o += 64 * 8;
  L.tn = o; o += gal16(nrows * 48);  // per row: the transform and the node position, read in the prologue
  L.total = o;
  return L;
}

struct GridArgs {
  Work w;
  Pattern pt;
  SolveArgs a;
  int slot;
};

__device__ __forceinline__ double bsum(double v, double* red) {
  v = warp_sum_d(v);
  const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[wi] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
    t = warp_sum_d(t);
  }
  return t;
}

// Fence-free grid barrier: the arrive is a release RMW on one counter
// (cumulative over the CTA's writes ordered before it by bar.sync), the wait
// an acquire poll.  (Per-CTA flags polled by every CTA measured 2-3x slower
// on B200: G*G acquire loads per round.)  Bounded: gives up after spin_limit
// polls, records kErrTimeout, and every later barrier of the launch returns
// within 32 polls.
// The arrive and the bounded wait of the barrier, by one thread.
__device__ __forceinline__ void arrive_wait(unsigned* ctr, unsigned gen, int G, int* err, unsigned spin_limit,
                                            unsigned extra) {
  red_release_gpu_add(ctr, 1u);
  const unsigned target = (gen + 1u) * (unsigned)G + extra;
  unsigned polls = 0;
  while (ld_acquire_gpu(ctr) < target) {
    // the error word only every 32 polls: a poll is then one round trip
    // to L2, not two
    if ((polls & 31) == 31 && *(volatile int*)err != 0) break;
    if (++polls > spin_limit) {
      atomicOr(err, kErrTimeout);
      break;
    }
    if (polls > 256) __nanosleep(polls > 8192 ? 256 : 20);
  }
}

__device__ __forceinline__ void gbar(unsigned* ctr, unsigned gen, int G, int cta, int* err, unsigned spin_limit,
                                     unsigned extra) {
  (void)cta;
  __syncthreads();
  if (threadIdx.x == 0) arrive_wait(ctr, gen, G, err, spin_limit, extra);
  __syncthreads();
}

// CTA sums of NS values stored as this CTA's partials, with ONE CTA barrier:
// warp sums, then thread 0 adds the eight warp sums in the xor-butterfly
// order of warp_sum_d (the bits of a second warp-level sum) and stores them.
// On return only thread 0 has stored; it arrives at the grid barrier next,
// its release covering every write of the CTA ordered before the bar.sync.
template <int NS>
__device__ __forceinline__ void publish_sums(const double (&v)[NS], double* red, double* const (&dst)[NS]) {
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
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NS; k++) {
      const double* r = red + k * 8;
      *dst[k] = ((r[0] + r[4]) + (r[2] + r[6])) + ((r[1] + r[5]) + (r[3] + r[7]));
    }
  }
}

// A warp sums NS slots of the G partials of a CTA group (slot stride
// `stride`) in one pass: each lane issues all its loads before it adds them
// (one round trip to L2 for up to 32 * kPartBatch CTAs), in a fixed order
// per lane, then an xor butterfly, so every CTA gets the same bits; results
// to red[dst..dst+NS).
constexpr int kPartBatch = 8;
template <int NS>
__device__ __forceinline__ void wsum_parts(const double* parts, int G, int stride, double* red, int dst) {
  const int lane = threadIdx.x & 31;
  double v[NS];
#pragma unroll
  for (int s = 0; s < NS; s++) v[s] = 0.0;
  for (int k0 = lane; k0 < G; k0 += 32 * kPartBatch) {
    double x[kPartBatch][NS];
#pragma unroll
    for (int b = 0; b < kPartBatch; b++) {
      const int k = k0 + 32 * b;
#pragma unroll
      for (int s = 0; s < NS; s++) x[b][s] = (k < G) ? __ldcg(parts + s * stride + k) : 0.0;
    }
#pragma unroll
    for (int b = 0; b < kPartBatch; b++)
      if (k0 + 32 * b < G) {
#pragma unroll
        for (int s = 0; s < NS; s++) v[s] += x[b][s];
      }
  }
#pragma unroll
  for (int s = 0; s < NS; s++) {
    v[s] = warp_sum_d(v[s]);
    if (lane == 0) red[dst + s] = v[s];
  }
}

template <bool A_SMEM, bool PIPE>
__global__ void __launch_bounds__(kThreads, 1) pcg_grid_kernel(GridArgs P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Work& w = P.w;
  const Pattern& pt = P.pt;
  const SolveArgs& a = P.a;
  const int tid = threadIdx.x;
  // CTA groups: each problem of the table has its own CTAs, barrier and partials
  const int cta = blockIdx.x, GT = gridDim.x;
  const int prob = pt.pcg_prob[cta];
  const int gb = pt.pcg_cta_off[prob], G = pt.pcg_cta_off[prob + 1] - gb, gcta = cta - gb;
  const ProbDesc pd = a.tb.desc[prob];
  DevStats* st = w.stats + prob;
  unsigned* bar = w.barrier + prob;
  const int r0 = pt.pcg_row_begin[cta], r1 = pt.pcg_row_begin[cta + 1];
  const int nrows = r1 - r0;
  const int b0 = pt.row_ptr[r0], b1 = pt.row_ptr[r1];
  const int nblk = b1 - b0;
  const int h0 = pt.g_halo_ptr[cta], nhalo = pt.g_halo_ptr[cta + 1] - h0;
  const GLayout L = glayout(nblk, nrows, nhalo, A_SMEM, PIPE);
  float* sA = reinterpret_cast<float*>(smem + L.a);
  int* sVidx = reinterpret_cast<int*>(smem + L.vidx);
  int* sRow = reinterpret_cast<int*>(smem + L.rowptr);
  int* sHalo = reinterpret_cast<int*>(smem + L.halo);
  float* sV = reinterpret_cast<float*>(smem + L.v);  // exchange vector: [own rows | halo] x 6
  double* sMinv = reinterpret_cast<double*>(smem + L.minv);
  double* sRed = reinterpret_cast<double*>(smem + L.red);
  const float* gA = pt.values + (size_t)b0 * 36;
  const int n6 = nrows * 6, h6 = nhalo * 6;
  int* err = w.err;
  double* part = w.partials;  // [2 bufs][3 slots][GT], this group's at [gb, gb + G)
  unsigned gen = 0;
  PhaseClock clk((a.timers && cta == 0 && tid == 0) ? a.timers : nullptr);
  (void)gcta;

  // ---- prologue: A rows, indices, halo list, FP64 block inverses ----
  // staged with cp.async: every copy of the CTA in flight at once, one wait
  if (A_SMEM)
    for (int i = tid; i < nblk * 9; i += kThreads) cp_async16(sA + 4 * i, gA + 4 * i);
  for (int i = tid; i < nblk; i += kThreads) cp_async4(sVidx + i, pt.g_vidx + b0 + i);
  for (int i = tid; i < nhalo; i += kThreads) cp_async4(sHalo + i, pt.g_halo_col + h0 + i);
  // the epilogue's operands (transform, node position), loaded now so that
  // their latency hides behind the solve
  float4* sTn = reinterpret_cast<float4*>(smem + L.tn);
  if (!a.delta_x)
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
  for (int i = tid; i <= nrows; i += kThreads) sRow[i] = pt.row_ptr[r0 + i] - b0;
  cp_async_commit_wait_all();
  __syncthreads();
  clk.mark(12);  // A, indices
  // block-Jacobi inverses in FP64, one 8-lane group per row
  {
    double* scr = reinterpret_cast<double*>(smem + L.scr) + (tid >> 3) * 72;
    int nfb = 0;
    for (int i0 = 0; i0 < nrows; i0 += kThreads / 8) {
      const int i = i0 + (tid >> 3);
      const bool act = i < nrows;
      const int dl = act ? pt.diag_pos[r0 + i] - b0 : 0;
      const float* blk = A_SMEM ? (sA + dl * 36) : (gA + dl * 36);
      nfb += inv6_group(blk, scr, sMinv + (act ? i : 0) * 36, act) && (tid & 7) == 0;
    }
    if (nfb) atomicAdd(&st->fallbacks, nfb);
  }
  clk.mark(13);  // inverses
  // The energy of this problem's linearisation point, summed by warps 1..7 of
  // the group's first CTA while thread 0 waits at the first grid barrier:
  // per thread in a fixed order (loads in flight together), then per warp,
  // then the seven warp sums in a fixed tree by thread 32 after the barrier.
  auto energy_warps = [&]() {
    if (gcta != 0 || tid < 32) return;
    const int n1 = pd.e_ctas, n = pd.e_ctas + pd.N;
    const double* p1 = w.e_data_part + pd.e_cta0;
    const double* p2 = w.e_arap_part + pd.node_off;
    double v = 0.0;
    for (int k0 = tid - 32; k0 < n; k0 += (kThreads - 32) * 8) {
      double x[8];
#pragma unroll
      for (int b = 0; b < 8; b++) {
        const int k = k0 + (kThreads - 32) * b;
        x[b] = k < n1 ? __ldcg(p1 + k) : (k < n ? __ldcg(p2 + (k - n1)) : 0.0);
      }
#pragma unroll
      for (int b = 0; b < 8; b++)
        if (k0 + (kThreads - 32) * b < n) v += x[b];
    }
    v = warp_sum_d(v);
    if ((tid & 31) == 0) sRed[40 + (tid >> 5)] = v;
  };
  auto energy_store = [&]() {  // after a CTA barrier that follows energy_warps
    if (gcta != 0 || tid != 32) return;
    const double* r = sRed + 41;
    const double v = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + r[6]);
    st->energy[P.slot] = v;
    if (!isfinite(v)) atomicOr(err, kErrNonFinite);
  };
  static_assert(kThreads == 256, "energy_store sums seven warps");

  // y = A v over own rows (v = sV, own rows then halo), FP32
  auto spmv_row = [&](int t) -> float {
    const int i = t / 6, c = t % 6;
    float acc = 0.f;
    for (int bl = sRow[i]; bl < sRow[i + 1]; bl++) {
      const float* Ab = A_SMEM ? (sA + bl * 36 + c * 6) : (gA + bl * 36 + c * 6);
      const float* vv = sV + sVidx[bl] * 6;
#pragma unroll
      for (int q = 0; q < 6; q++) acc = __fmaf_rn(A_SMEM ? Ab[q] : __ldcg(Ab + q), vv[q], acc);
    }
    return acc;
  };
  // z_t = (M^-1 v)_t for own row element t, FP64
  auto minv_row = [&](int t, auto vget) -> double {
    const int i = t / 6, c = t % 6;
    const double* Mi = sMinv + i * 36 + c * 6;
    double zz = 0.0;
#pragma unroll
    for (int q = 0; q < 6; q++) zz += Mi[q] * vget(i * 6 + q);
    return zz;
  };

  int used = 0;
  double rr_last = 0.0;
  if (!PIPE) {
    // ================= standard PCG =================
    // sZ: z of own rows then halo; sV: the previous p, own rows then halo (the
    // SpMV forms p = z + beta p_old as it reads, so p is never stored for the
    // halo); sPn: this iteration's p of own rows
    const int vs = gal16(n6 * 4) / 4, zs = gal16((n6 + h6) * 4) / 4;
    float* sZ = reinterpret_cast<float*>(smem + L.st);
    float* sX = sZ + zs;
    float* sR = sX + vs;
    float* sAp = sR + vs;
    float* sPn = sAp + vs;
    // lanes per row element of the SpMV: 4, 2 or 1, as many as the CTA's threads allow
    const int spl_log = (n6 * 4 <= kThreads) ? 2 : (n6 * 2 <= kThreads) ? 1 : 0, spl = 1 << spl_log;
    double prz = 0.0, pbb = 0.0;
    for (int t = tid; t < n6; t += kThreads) {
      const float rt = __ldcg(w.rhs + r0 * 6 + t);
      sR[t] = rt;
      sX[t] = 0.f;
      pbb += (double)rt * rt;
    }
    __syncthreads();
    for (int t = tid; t < n6; t += kThreads) {
      const float zf = (float)minv_row(t, [&](int k) { return (double)sR[k]; });
      sZ[t] = zf;
      w.z[r0 * 6 + t] = zf;
      prz += (double)sR[t] * zf;
    }
    {
      const int buf = gen & 1;
      const double v2[2] = {prz, pbb};
      double* const d2[2] = {part + (buf * 3 + 0) * GT + cta, part + (buf * 3 + 1) * GT + cta};
      publish_sums<2>(v2, sRed, d2);
    }
    clk.mark(0);  // prologue
    if (tid == 0)
      arrive_wait(bar, gen, G, err, a.spin_limit, a.bar_extra);
    else
      energy_warps();
    gen++;
    __syncthreads();
    energy_store();
    clk.mark(1);  // first barrier
    double rz = 0.0;
    float betaf = 0.f;
    for (int it = 0;; it++) {
      const float* pold = (it & 1) ? w.p0 : w.p1;  // p_{it-1} lives in buffer (it-1)&1
      float* pnew = (it & 1) ? w.p1 : w.p0;
      // ---- one round trip: the reduction behind the last barrier and the halo ----
      {
        const int buf = (gen - 1) & 1;
        if (tid < 32) {
          wsum_parts<2>(part + (buf * 3 + 0) * GT + gb, G, GT, sRed, 16);
        } else {
          for (int e = tid - 32; e < h6; e += kThreads - 32) {
            const int col = sHalo[e / 6], c = e % 6;
            sZ[n6 + e] = __ldcg(w.z + col * 6 + c);
            if (it > 0) sV[n6 + e] = __ldcg(pold + col * 6 + c);
          }
        }
        __syncthreads();
      }
      clk.mark(2);  // partials + halo
      if (it == 0) {
        rz = sRed[16];
        rr_last = sRed[17];
      } else {
        const double rr = sRed[16], rzn = sRed[17];
        used = it;
        rr_last = rr;
        if (sqrt(rr) < (double)a.pcg_tolerance) break;  // solver_kernels.cu:669
        betaf = (float)(rzn / rz);
        rz = rzn;
      }
      if (it >= a.pcg_iterations) break;
      clk.mark(3);  // (p is formed inside the SpMV)
      // ---- p = z + beta p_old and Ap (solver_kernels.cu:406-432), p.Ap ----
      // S adjacent lanes per row element, lane k over the row's blocks k, k+S, ...,
      // combined by an xor butterfly: the CTA's time is its longest row / S.
      // Each operand value is formed as it is read, fmaf(beta, p_old, z) (z
      // alone in the first iteration), the value the p update would store.
      const bool first = it == 0;
      double ppap = 0.0;
      for (int u0 = 0; u0 < n6 * spl; u0 += kThreads) {
        const int u = u0 + tid, t = u >> spl_log, k = u & (spl - 1);
        float y = 0.f;
        if (t < n6) {
          const int i = t / 6, c = t % 6;
          for (int bl = sRow[i] + k; bl < sRow[i + 1]; bl += spl) {
            const float* Ab = A_SMEM ? (sA + bl * 36 + c * 6) : (gA + bl * 36 + c * 6);
            const int o = sVidx[bl] * 6;
            const float* zz = sZ + o;
            const float* pp = sV + o;
#pragma unroll
            for (int q = 0; q < 6; q++) {
              const float pv = first ? zz[q] : __fmaf_rn(betaf, pp[q], zz[q]);
              y = __fmaf_rn(A_SMEM ? Ab[q] : __ldcg(Ab + q), pv, y);
            }
          }
        }
        for (int o = spl >> 1; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        if (k == 0 && t < n6) {
          const float pt_ = first ? sZ[t] : __fmaf_rn(betaf, sV[t], sZ[t]);
          sPn[t] = pt_;
          pnew[r0 * 6 + t] = pt_;
          sAp[t] = y;
          ppap += (double)pt_ * y;
        }
      }
      clk.mark(4);  // spmv
      {
        const double v1[1] = {ppap};
        double* const d1[1] = {part + ((gen & 1) * 3 + 0) * GT + cta};
        publish_sums<1>(v1, sRed, d1);
      }
      clk.mark(5);  // block sum
      if (tid < 32) {  // warp 0 waits and reads the partials; the others wait at the CTA barrier
        if (tid == 0) arrive_wait(bar, gen, G, err, a.spin_limit, a.bar_extra);
        clk.mark(6);  // barrier A
        __syncwarp();
        wsum_parts<1>(part + ((gen & 1) * 3 + 0) * GT + gb, G, GT, sRed, 18);
      }
      gen++;
      __syncthreads();
      clk.mark(7);  // pAp partials
      const double pAp = sRed[18];
      if (fabs(pAp) < 1e-12) break;  // solver_kernels.cu:647-653
      const float af = (float)(rz / pAp);
      for (int t = tid; t < n6; t += kThreads) {
        sX[t] = __fmaf_rn(af, sPn[t], sX[t]);
        sR[t] = __fmaf_rn(-af, sAp[t], sR[t]);
        sV[t] = sPn[t];  // p_old of the next iteration
      }
      __syncthreads();
      double prr = 0.0, przn = 0.0;
      for (int t = tid; t < n6; t += kThreads) {
        const float zf = (float)minv_row(t, [&](int k) { return (double)sR[k]; });
        sZ[t] = zf;
        w.z[r0 * 6 + t] = zf;
        prr += (double)sR[t] * sR[t];
        przn += (double)sR[t] * zf;
      }
      clk.mark(8);  // x, r, z updates
      {
        const int buf = gen & 1;
        const double v2[2] = {prr, przn};
        double* const d2[2] = {part + (buf * 3 + 0) * GT + cta, part + (buf * 3 + 1) * GT + cta};
        publish_sums<2>(v2, sRed, d2);
      }
      clk.mark(9);  // block sums
      if (tid == 0) arrive_wait(bar, gen, G, err, a.spin_limit, a.bar_extra);
      gen++;
      __syncthreads();
      clk.mark(10);  // barrier B
    }
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
  } else {
    // ================= pipelined PCG (Ghysels-Vanroose) =================
    const int ds = gal16(n6 * 8) / 8;
    double* vX = reinterpret_cast<double*>(smem + L.st);
    double* vR = vX + ds;
    double* vU = vR + ds;
    double* vW = vU + ds;
    double* vZ = vW + ds;
    double* vQ = vZ + ds;
    double* vS = vQ + ds;
    double* vP = vS + ds;
    float* sN = reinterpret_cast<float*>(vP + ds);
    float* xb[2] = {w.p0, w.p1};
    // r = b, x = z = q = s = p = 0, u = M^-1 r; publish u
    for (int t = tid; t < n6; t += kThreads) {
      vR[t] = (double)__ldcg(w.rhs + r0 * 6 + t);
      vX[t] = vZ[t] = vQ[t] = vS[t] = vP[t] = 0.0;
    }
    __syncthreads();
    for (int t = tid; t < n6; t += kThreads) {
      const double u = minv_row(t, [&](int k) { return vR[k]; });
      vU[t] = u;
      const float uf = (float)u;
      sV[t] = uf;
      xb[gen & 1][r0 * 6 + t] = uf;
    }
    __syncthreads();
    if (tid == 0)
      arrive_wait(bar, gen, G, err, a.spin_limit, a.bar_extra);
    else
      energy_warps();
    gen++;
    __syncthreads();
    energy_store();
    for (int e = tid; e < h6; e += kThreads) sV[n6 + e] = __ldcg(xb[(gen - 1) & 1] + sHalo[e / 6] * 6 + e % 6);
    __syncthreads();
    // w = A u ; then the first reduction and m = M^-1 w
    for (int t = tid; t < n6; t += kThreads) vW[t] = (double)spmv_row(t);
    __syncthreads();
    auto reduce_and_publish = [&]() {
      double pg = 0.0, pd = 0.0, pr = 0.0;
      for (int t = tid; t < n6; t += kThreads) {
        pg += vR[t] * vU[t];
        pd += vW[t] * vU[t];
        pr += vR[t] * vR[t];
        const float mf = (float)minv_row(t, [&](int k) { return vW[k]; });
        xb[gen & 1][r0 * 6 + t] = mf;
        sN[t] = mf;  // stage m; copied into the operand after the barrier
      }
      const int buf = gen & 1;
      const double t1 = bsum(pg, sRed), t2 = bsum(pd, sRed + 8), t3 = bsum(pr, sRed + 24);
      if (tid == 0) {
        part[(buf * 3 + 0) * GT + cta] = t1;
        part[(buf * 3 + 1) * GT + cta] = t2;
        part[(buf * 3 + 2) * GT + cta] = t3;
      }
      gbar(bar, gen++, G, cta, err, a.spin_limit, a.bar_extra);
    };
    reduce_and_publish();
    double gamma_prev = 0.0, alpha_prev = 0.0;
    for (int it = 0;; it++) {
      {
        const int buf = (gen - 1) & 1;
        if (tid < 32) {
          wsum_parts<3>(part + (buf * 3 + 0) * GT + gb, G, GT, sRed, 16);
        } else {
          for (int e = tid - 32; e < h6; e += kThreads - 32)
            sV[n6 + e] = __ldcg(xb[buf] + sHalo[e / 6] * 6 + e % 6);
        }
        for (int t = tid; t < n6; t += kThreads) sV[t] = sN[t];
        __syncthreads();
      }
      const double gamma = sRed[16], delta = sRed[17], rr = sRed[18];
      rr_last = rr;
      if (it > 0) {
        used = it;
        if (sqrt(rr) < (double)a.pcg_tolerance) break;  // solver_kernels.cu:669
      }
      if (it >= a.pcg_iterations) break;
      const double beta = (it > 0) ? gamma / gamma_prev : 0.0;
      const double pAp = (it > 0) ? delta - beta * gamma / alpha_prev : delta;  // = p.Ap
      if (fabs(pAp) < 1e-12) break;  // solver_kernels.cu:647-653
      const double alpha = gamma / pAp;
      for (int t = tid; t < n6; t += kThreads) {
        const double n = (double)spmv_row(t);
        const double m = (double)sV[t];
        vZ[t] = n + beta * vZ[t];
        vQ[t] = m + beta * vQ[t];
        vS[t] = vW[t] + beta * vS[t];
        vP[t] = vU[t] + beta * vP[t];
        vX[t] += alpha * vP[t];
        vR[t] -= alpha * vS[t];
        vU[t] -= alpha * vQ[t];
        vW[t] -= alpha * vZ[t];
      }
      __syncthreads();
      gamma_prev = gamma;
      alpha_prev = alpha;
      if (it + 1 >= a.pcg_iterations) {
        used = it + 1;
        // final ||r|| for the statistics
        double pr = 0.0;
        for (int t = tid; t < n6; t += kThreads) pr += vR[t] * vR[t];
        const double t3 = bsum(pr, sRed);
        if (tid == 0) part[((gen & 1) * 3 + 2) * GT + cta] = t3;
        gbar(bar, gen++, G, cta, err, a.spin_limit, a.bar_extra);
        if (tid < 32) wsum_parts<1>(part + (((gen - 1) & 1) * 3 + 2) * GT + gb, G, GT, sRed, 18);
        __syncthreads();
        rr_last = sRed[18];
        break;
      }
      reduce_and_publish();
    }
    // ---- epilogue ----
    float* xf = sN;
    bool bad = false;
    for (int t = tid; t < n6; t += kThreads) {
      xf[t] = (float)vX[t];
      bad |= !isfinite(xf[t]);
    }
    if (bad) atomicOr(err, kErrNonFinite);
    __syncthreads();
    if (a.delta_x) {
      for (int t = tid; t < n6; t += kThreads) a.delta_x[r0 * 6 + t] = xf[t];
    } else {
      for (int i = tid; i < nrows; i += kThreads) {
        const int node = r0 + i;
        DQ T0;
        T0.r = sTn[3 * i];
        T0.d = sTn[3 * i + 1];
        const float4 xp = sTn[3 * i + 2];
        DQ Tn = twist_update(T0, xf + i * 6, pd.max_rot, pd.max_trans, pd.update_scale);
        store_dq(a.transforms + node, Tn);
        store_dq(w.plain + node, dq_centered(Tn, f3(xp.x, xp.y, xp.z)));
      }
    }
  }
  clk.mark(11);  // epilogue
  clk.flush();
  if (gcta == 0 && tid == 0) {
    st->pcg_iters[P.slot] = used;
    st->pcg_res[P.slot] = sqrt(rr_last);
  }
}

template <bool A, bool PP>
cudaError_t set_smem(int smem) {
  // the device's opt-in maximum, not this plan's size: another handle's plan
  // (with more shared memory) launches the same kernel
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (smem > optin) return cudaErrorInvalidValue;
  return cudaFuncSetAttribute(pcg_grid_kernel<A, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
}

template <bool A, bool PP>
int occupancy(int smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_grid_kernel<A, PP>, kThreads, smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return per_sm;
}

}  // namespace

int pcg_grid_smem_bytes(int nblk, int nrows, int nhalo, bool a_in_smem, bool pipelined) {
  return glayout(nblk, nrows, nhalo, a_in_smem, pipelined).total;
}

int pcg_max_active_ctas(int smem, bool a_in_smem, bool pipelined) {
  cudaError_t e = a_in_smem ? (pipelined ? set_smem<true, true>(smem) : set_smem<true, false>(smem))
                            : (pipelined ? set_smem<false, true>(smem) : set_smem<false, false>(smem));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int per_sm = a_in_smem ? (pipelined ? occupancy<true, true>(smem) : occupancy<true, false>(smem))
                         : (pipelined ? occupancy<false, true>(smem) : occupancy<false, false>(smem));
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return per_sm * sms;
}

cudaError_t launch_pcg(const Work& w, const Pattern& p, const SolveArgs& a, int gn_slot, cudaStream_t s) {
  if (a.N <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(w.barrier, 0, sizeof(unsigned) * (size_t)p.P, s);
  if (e != cudaSuccess) return e;
  GridArgs P;
  P.w = w;
  P.pt = p;
  P.a = a;
  P.slot = gn_slot;
  void* args[] = {&P};
  void* fn;
  if (p.pcg_a_in_smem)
    fn = p.pcg_pipelined ? (void*)pcg_grid_kernel<true, true> : (void*)pcg_grid_kernel<true, false>;
  else
    fn = p.pcg_pipelined ? (void*)pcg_grid_kernel<false, true> : (void*)pcg_grid_kernel<false, false>;
  return cudaLaunchCooperativeKernel(fn, dim3(p.pcg_ctas), dim3(kThreads), args, (size_t)p.pcg_smem, s);
}

}  // namespace cf
