// cf_pcg_stream.cu — persistent block-Jacobi PCG for systems larger than the
// GPU's shared memory (big problems, batches).
//
// Same schedule and semantics as the shared-memory kernel (cf_pcg_grid.cu):
// the reference's PCG (kernels/solver_kernels.cu:616-687: x0 = 0, the
// |p.Ap| < 1e-12 guard before the update, ||r|| < tol after it), FP32
// vectors, FP64 dot products, FP64 block inverses (stored FP32), two grid
// reductions per iteration, one CTA group per problem.  What differs is where
// the data lives: every iteration streams the CTA's block rows of A from HBM
// through a ring of shared-memory stages filled by TMA bulk copies
// (cp.async.bulk, completion on an mbarrier), and the vectors stay in global
// memory.  A tile is a run of whole block rows of at most TB blocks.
//
// Per iteration, per CTA:
//   SpMV   thread per block of the tile: y_b = A_b (z_j + beta p_old_j), the
//          operand formed on the fly from the exchanged z and p_old (so p
//          itself is never waited for); then thread per (row, component):
//          the row's block products summed in block order, p and Ap written,
//          p.Ap accumulated.  -> group reduction (barrier A)
//   update thread per row: x += alpha p, r -= alpha Ap, z = M^-1 r, r.r and
//          r.z accumulated.  -> group reduction (barrier B)
// The tiles of the next iteration are prefetched while the reductions run;
// copies still in flight when the loop ends are drained before exit.  Each
// stage also brings the tile's column indices (a padded copy made with the
// pattern), so the SpMV operand of tile t + 1 is gathered while tile t's rows
// are summed: one exposed gather per iteration instead of one per tile.
#include "cf_device.cuh"
#include "cf_internal.h"

namespace cf {

namespace {

// tile: up to TB blocks of whole rows (one thread per block): 256 (36,864 B)
// or 128, the autotuner's choice
constexpr int kStages = 2;
constexpr int kPartStride = 7;  // padded 6-float partial row
// polls of a tile copy's completion before it counts as lost: a copy always
// completes, so this is far above any real wait and independent of the
// barrier's (settable) limit; a CTA never exits with its copy in flight
// unless this runs out
constexpr unsigned kCopyWaitLimit = 1u << 26;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// TMA bulk copy global -> shared, completion counted on `bar` (16-B aligned
// addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of `bar`; false (and the timeout bit) when
// it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err, unsigned limit) {
  for (unsigned polls = 0; !mbar_try_wait(bar, parity);) {
    if (++polls > limit) {
      atomicOr(err, kErrTimeout);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ double bsum_s(double v, double* red) {
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

// group barrier: release arrive on the group's counter, bounded acquire poll
__device__ __forceinline__ void gbar_s(unsigned* ctr, unsigned gen, int G, int* err, unsigned spin_limit,
                                       unsigned extra) {
  __syncthreads();
  if (threadIdx.x == 0) {
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
  __syncthreads();
}

__device__ __forceinline__ void ld6(const float* p, float* v) {
  const float2 a = __ldcg(reinterpret_cast<const float2*>(p));
  const float2 b = __ldcg(reinterpret_cast<const float2*>(p) + 1);
  const float2 c = __ldcg(reinterpret_cast<const float2*>(p) + 2);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y;
}
__device__ __forceinline__ void st6(float* p, const float* v) {
  reinterpret_cast<float2*>(p)[0] = make_float2(v[0], v[1]);
  reinterpret_cast<float2*>(p)[1] = make_float2(v[2], v[3]);
  reinterpret_cast<float2*>(p)[2] = make_float2(v[4], v[5]);
}

struct StreamArgs {
  Work w;
  Pattern pt;
  SolveArgs a;
  int slot;
};

template <int TB>
__global__ void __launch_bounds__(kThreads, 2) pcg_stream_kernel(StreamArgs P) {
  static_assert(TB <= kThreads, "one thread per block of a tile");
  constexpr int kTileBlocks = TB, kTileBytes = TB * 36 * 4, kStageBytes = kTileBytes + TB * 4;
  extern __shared__ __align__(128) unsigned char smem[];
  float* ring = reinterpret_cast<float*>(smem);                           // [kStages] x (A tile, column indices)
  float* sPart = reinterpret_cast<float*>(smem + kStages * kStageBytes);  // [kTileBlocks][7]
  double* sRed = reinterpret_cast<double*>(smem + kStages * kStageBytes + kTileBlocks * kPartStride * 4);  // [64]
  auto stageA = [&](int s) { return reinterpret_cast<const float*>(smem + (size_t)s * kStageBytes); };
  auto stageC = [&](int s) { return reinterpret_cast<const int*>(smem + (size_t)s * kStageBytes + kTileBytes); };
  __shared__ uint64_t mbar[kStages];
  const Work& w = P.w;
  const Pattern& pt = P.pt;
  const SolveArgs& a = P.a;
  const int tid = threadIdx.x;
  const int cta = blockIdx.x, GT = gridDim.x;
  const int prob = pt.pcg_prob[cta];
  const int gb = pt.pcg_cta_off[prob], G = pt.pcg_cta_off[prob + 1] - gb, gcta = cta - gb;
  const ProbDesc pd = a.tb.desc[prob];
  DevStats* st = w.stats + prob;
  unsigned* bar = w.barrier + prob;
  int* err = w.err;
  double* part = w.partials;  // [2 bufs][3 slots][GT]
  const int r0 = pt.pcg_row_begin[cta], r1 = pt.pcg_row_begin[cta + 1];
  const int t_begin = pt.st_tile_ptr[cta], n_tiles = pt.st_tile_ptr[cta + 1] - t_begin - 1;
  const int* trow = pt.st_tile_row + t_begin;  // n_tiles + 1 row boundaries
  unsigned gen = 0;

  if (tid == 0) {
    for (int s = 0; s < kStages; s++) mbar_init(&mbar[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // ring state, identical in every thread: the next tile to issue and the
  // next to consume (counted over the whole launch), per-stage phase bits
  long long issued = 0, consumed = 0;
  unsigned phase_bits = 0;
  auto issue = [&](long long k) {  // thread 0: tile k % n_tiles into stage k % kStages
    const int t = (int)(k % n_tiles), s = (int)(k % kStages);
    const int b0 = pt.row_ptr[trow[t]], b1 = pt.row_ptr[trow[t + 1]];
    const unsigned bytes = (unsigned)(b1 - b0) * 144u;
    unsigned char* dst = smem + (size_t)s * kStageBytes;
    fence_proxy_async();
    mbar_expect_tx(&mbar[s], bytes + TB * 4u);
    bulk_g2s(dst, pt.values + (size_t)b0 * 36, bytes, &mbar[s]);
    bulk_g2s(dst + kTileBytes, pt.st_tile_cols + (size_t)(t_begin + t) * TB, TB * 4u, &mbar[s]);
  };
  auto top_up = [&]() {  // keep kStages tiles in flight
    while (issued < consumed + kStages) {
      if (tid == 0 && n_tiles > 0) issue(issued);
      issued++;
    }
  };

  // ---- prologue: block-Jacobi inverses (FP64, stored FP32), energy ----
  // (the ring is free until the first tiles are issued: it holds the
  // inversion scratch, 108 doubles per 8-lane group)
  {
    double* scr = reinterpret_cast<double*>(ring) + (tid >> 3) * 108;
    double* outd = scr + 72;
    int nfb = 0;
    for (int i0 = r0; i0 < r1; i0 += kThreads / 8) {
      const int i = i0 + (tid >> 3);
      const bool act = i < r1;
      const float* blk = pt.values + (size_t)(act ? pt.diag_pos[i] : 0) * 36;
      nfb += inv6_group(blk, scr, outd, act) && (tid & 7) == 0;
      if (act)
        for (int q = tid & 7; q < 36; q += 8) w.minv32[(size_t)i * 36 + q] = (float)outd[q];
      __syncwarp();
    }
    if (nfb) atomicAdd(&st->fallbacks, nfb);
  }
  __syncthreads();
  if (gcta == 0) {  // energy of this problem's linearisation point (fixed-order tree)
    double v = 0.0;
    for (int k = tid; k < pd.e_ctas; k += kThreads) v += __ldcg(w.e_data_part + pd.e_cta0 + k);
    for (int k = tid; k < pd.N; k += kThreads) v += __ldcg(w.e_arap_part + pd.node_off + k);
    v = bsum_s(v, sRed + 32);
    if (tid == 0) {
      st->energy[P.slot] = v;
      if (!isfinite(v)) atomicOr(err, kErrNonFinite);
    }
  }
  __syncthreads();
  top_up();  // the first tiles stream in during the first reduction

  // r = b, x = 0, z = M^-1 r; r.z and b.b
  double prz = 0.0, pbb = 0.0;
  for (int i = r0 + tid; i < r1; i += kThreads) {
    float rr[6], zz[6], M[36];
    ld6(w.rhs + (size_t)i * 6, rr);
    for (int q = 0; q < 36; q++) M[q] = w.minv32[(size_t)i * 36 + q];
#pragma unroll
    for (int c = 0; c < 6; c++) {
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < 6; q++) s += (double)M[c * 6 + q] * (double)rr[q];
      zz[c] = (float)s;
      prz += (double)rr[c] * zz[c];
      pbb += (double)rr[c] * rr[c];
    }
    const float zero[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    st6(w.r + (size_t)i * 6, rr);
    st6(w.x + (size_t)i * 6, zero);
    st6(w.z + (size_t)i * 6, zz);
  }
  {
    const double t1 = bsum_s(prz, sRed), t2 = bsum_s(pbb, sRed + 8);
    if (tid == 0) {
      part[(0 * 3 + 0) * GT + cta] = t1;
      part[(0 * 3 + 1) * GT + cta] = t2;
    }
  }
  gbar_s(bar, gen++, G, err, a.spin_limit, a.bar_extra);

  int used = 0;
  double rz = 0.0, rr_last = 0.0;
  float betaf = 0.f;
  bool ok = true;
  for (int it = 0;; it++) {
    // the reduction behind the last barrier (fixed order: every CTA gets the same bits)
    if (tid < 32) {
      const int buf = (gen - 1) & 1;
      double v0 = 0.0, v1 = 0.0;
      for (int k = tid; k < G; k += 32) {
        v0 += __ldcg(part + (buf * 3 + 0) * GT + gb + k);
        v1 += __ldcg(part + (buf * 3 + 1) * GT + gb + k);
      }
      v0 = warp_sum_d(v0);
      v1 = warp_sum_d(v1);
      if (tid == 0) {
        sRed[16] = v0;
        sRed[17] = v1;
      }
    }
    __syncthreads();
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
    if (it >= a.pcg_iterations || *(volatile int*)err) break;
    const float* pold = (it & 1) ? w.p0 : w.p1;
    float* pnew = (it & 1) ? w.p1 : w.p0;
    // ---- Ap = A (z + beta p_old), p = z + beta p_old, p.Ap ----
    double ppap = 0.0;
    // the operand of the tile in stage s (its column indices came with A;
    // -1 pads past the tile's blocks): z_j and p_old_j into registers
    float gz[6], gp[6];
    auto gather = [&](int s) {
      const int j = stageC(s)[tid < TB ? tid : 0];
      if (tid < TB && j >= 0) {
        ld6(w.z + (size_t)j * 6, gz);
        if (it > 0) ld6(pold + (size_t)j * 6, gp);
      }
    };
    for (int t = 0; t < n_tiles; t++) {
      const int s = (int)(consumed % kStages);
      if (!mbar_wait(&mbar[s], (phase_bits >> s) & 1u, err, kCopyWaitLimit)) ok = false;
      if (t == 0) gather(s);  // (later tiles were gathered during the previous one)
      phase_bits ^= 1u << s;
      const float* A = stageA(s);
      const int ra = trow[t], rb_ = trow[t + 1];
      const int b0 = pt.row_ptr[ra], nb = pt.row_ptr[rb_] - b0;
      if (tid < nb) {
        float v[6];
#pragma unroll
        for (int q = 0; q < 6; q++) v[q] = (it > 0) ? __fmaf_rn(betaf, gp[q], gz[q]) : gz[q];
        const float4* A4 = reinterpret_cast<const float4*>(A + tid * 36);
        float Ab[36];
#pragma unroll
        for (int k = 0; k < 9; k++) {
          const float4 f = A4[k];
          Ab[4 * k] = f.x; Ab[4 * k + 1] = f.y; Ab[4 * k + 2] = f.z; Ab[4 * k + 3] = f.w;
        }
#pragma unroll
        for (int c = 0; c < 6; c++) {
          float acc = 0.f;
#pragma unroll
          for (int q = 0; q < 6; q++) acc = __fmaf_rn(Ab[c * 6 + q], v[q], acc);
          sPart[tid * kPartStride + c] = acc;
        }
      }
      if (t + 1 < n_tiles) {  // the next tile's operand, in flight during this tile's row sums
        const int s2 = (int)((consumed + 1) % kStages);
        if (!mbar_wait(&mbar[s2], (phase_bits >> s2) & 1u, err, kCopyWaitLimit)) ok = false;
        gather(s2);
      }
      __syncthreads();
      consumed++;
      top_up();  // stage s is free: refill it (tiles wrap into the next iteration)
      for (int e = tid; e < (rb_ - ra) * 6; e += kThreads) {
        const int i = ra + e / 6, c = e % 6;
        const int q0 = pt.row_ptr[i] - b0, q1 = pt.row_ptr[i + 1] - b0;
        float y = 0.f;
        for (int q = q0; q < q1; q++) y += sPart[q * kPartStride + c];
        const float zi = __ldcg(w.z + (size_t)i * 6 + c);
        const float pi = (it > 0) ? __fmaf_rn(betaf, __ldcg(pold + (size_t)i * 6 + c), zi) : zi;
        pnew[(size_t)i * 6 + c] = pi;
        w.ap[(size_t)i * 6 + c] = y;
        ppap += (double)pi * y;
      }
      __syncthreads();
    }
    {
      const double t1 = bsum_s(ppap, sRed);
      if (tid == 0) part[((gen & 1) * 3 + 0) * GT + cta] = t1;
    }
    gbar_s(bar, gen++, G, err, a.spin_limit, a.bar_extra);
    if (tid < 32) {
      double v0 = 0.0;
      for (int k = tid; k < G; k += 32) v0 += __ldcg(part + (((gen - 1) & 1) * 3 + 0) * GT + gb + k);
      v0 = warp_sum_d(v0);
      if (tid == 0) sRed[18] = v0;
    }
    __syncthreads();
    const double pAp = sRed[18];
    if (fabs(pAp) < 1e-12 || !ok) break;  // solver_kernels.cu:647-653
    const float af = (float)(rz / pAp);
    // ---- x += alpha p, r -= alpha Ap, z = M^-1 r; r.r, r.z ----
    double prr = 0.0, przn = 0.0;
    for (int i = r0 + tid; i < r1; i += kThreads) {
      float xx[6], rr[6], pp[6], ap[6], zz[6], M[36];
      ld6(w.x + (size_t)i * 6, xx);
      ld6(w.r + (size_t)i * 6, rr);
      ld6(pnew + (size_t)i * 6, pp);
      ld6(w.ap + (size_t)i * 6, ap);
      const float4* m4 = reinterpret_cast<const float4*>(w.minv32 + (size_t)i * 36);
#pragma unroll
      for (int k = 0; k < 9; k++) {
        const float4 f = __ldcg(m4 + k);
        M[4 * k] = f.x; M[4 * k + 1] = f.y; M[4 * k + 2] = f.z; M[4 * k + 3] = f.w;
      }
#pragma unroll
      for (int c = 0; c < 6; c++) {
        xx[c] = __fmaf_rn(af, pp[c], xx[c]);
        rr[c] = __fmaf_rn(-af, ap[c], rr[c]);
      }
#pragma unroll
      for (int c = 0; c < 6; c++) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < 6; q++) s += (double)M[c * 6 + q] * (double)rr[q];
        zz[c] = (float)s;
        prr += (double)rr[c] * rr[c];
        przn += (double)rr[c] * zz[c];
      }
      st6(w.x + (size_t)i * 6, xx);
      st6(w.r + (size_t)i * 6, rr);
      st6(w.z + (size_t)i * 6, zz);
    }
    {
      const double t1 = bsum_s(prr, sRed), t2 = bsum_s(przn, sRed + 8);
      if (tid == 0) {
        part[((gen & 1) * 3 + 0) * GT + cta] = t1;
        part[((gen & 1) * 3 + 1) * GT + cta] = t2;
      }
    }
    gbar_s(bar, gen++, G, err, a.spin_limit, a.bar_extra);
  }
  // ---- drain the prefetched tiles, then the epilogue ----
  while (consumed < issued) {
    const int s = (int)(consumed % kStages);
    if (n_tiles > 0) mbar_wait(&mbar[s], (phase_bits >> s) & 1u, err, kCopyWaitLimit);
    phase_bits ^= 1u << s;
    consumed++;
  }
  __syncthreads();
  bool bad = false;
  for (int i = r0 + tid; i < r1; i += kThreads) {
    float xx[6];
    ld6(w.x + (size_t)i * 6, xx);
#pragma unroll
    for (int c = 0; c < 6; c++) bad |= !isfinite(xx[c]);
    if (a.delta_x) {
      st6(a.delta_x + (size_t)i * 6, xx);
    } else {
      DQ Tn = twist_update(load_dq_cg(a.transforms + i), xx, pd.max_rot, pd.max_trans, pd.update_scale);
      store_dq(a.transforms + i, Tn);
      store_dq(w.plain + i, dq_centered(Tn, node_pos(a.nodes, i)));
    }
  }
  if (bad) atomicOr(err, kErrNonFinite);
  if (gcta == 0 && tid == 0) {
    st->pcg_iters[P.slot] = used;
    st->pcg_res[P.slot] = sqrt(rr_last);
  }
}

}  // namespace

int pcg_stream_smem_bytes(int tb) { return kStages * tb * 148 + tb * kPartStride * 4 + 64 * 8; }
static_assert(kStages * 128 * 144 >= (kThreads / 8) * 108 * 8, "the ring holds the inversion scratch");

namespace {
void* stream_fn(int tb) { return tb == 128 ? (void*)pcg_stream_kernel<128> : (void*)pcg_stream_kernel<256>; }
}  // namespace

int pcg_stream_max_active_ctas(int tb) {
  const int smem = pcg_stream_smem_bytes(tb);
  if (cudaFuncSetAttribute(stream_fn(tb), cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stream_fn(tb), kThreads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return per_sm * sms;
}

cudaError_t launch_pcg_stream(const Work& w, const Pattern& p, const SolveArgs& a, int gn_slot, cudaStream_t s) {
  if (a.N <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(w.barrier, 0, sizeof(unsigned) * (size_t)p.P, s);
  if (e != cudaSuccess) return e;
  StreamArgs P;
  P.w = w;
  P.pt = p;
  P.a = a;
  P.slot = gn_slot;
  void* args[] = {&P};
  return cudaLaunchCooperativeKernel(stream_fn(p.st_tile_blocks), dim3(p.pcg_ctas), dim3(kThreads), args,
                                     (size_t)pcg_stream_smem_bytes(p.st_tile_blocks), s);
}

}  // namespace cf
