// cf_mpnn.cu — the learned initial increment: a message-passing network over
// the deformation graph, its training kernels, and the per-node features and
// increments it works on.  (No counterpart in the reference, which starts
// every frame's GN from a zero increment.)
//
// Network (per node i, neighbours N(i) = the node's graph list, K <= 8):
//   x_i   = 20 features: the node's increments of the last three frames
//           (rotation vector scaled by 10, translation in cm), and the mean
//           and max |point-to-plane residual| (mm) of its correspondences at
//           the warm start
//   h1_i  = relu(W0 [x_i, mean_j x_j] + b0)          20+20 -> 64
//   h2_i  = relu(W1 [h1_i, mean_j h1_j] + b1)        64+64 -> 64
//   h3_i  = relu(W2 [h2_i, mean_j h2_j] + b2)        64+64 -> 64
//   out_i = Wo h3_i + bo + x_i[0:6]                  64 -> 6 (a correction to
//           repeating the last frame's increment), in the scaled units of x
// Parameters and activations are BF16 (parameters kept in FP32 for Adam and
// rounded to BF16 after every step); every sum accumulates in FP32, in a
// fixed order, so forward and gradients are deterministic.  The layers are
// tiny (N x 128 x 64): the forward runs on the tensor cores (BF16 mma.sync
// over shared-memory tiles of 16 nodes), the gradients on CUDA cores over
// tiles of 32 (per-CTA partial sums reduced in CTA order).
#include <cuda_bf16.h>

#include "cf_device.cuh"
#include "cf_internal.h"

namespace cf {

namespace {

constexpr int kIn = CF_MPNN_IN, kHid = CF_MPNN_HIDDEN, kOut = CF_MPNN_OUT;
constexpr int kTileNodes = 32;

// parameter offsets (floats) in the flat vector: W0 b0 W1 b1 W2 b2 Wo bo
constexpr int kW0 = 0, kB0 = kW0 + kHid * 2 * kIn, kW1 = kB0 + kHid, kB1 = kW1 + kHid * 2 * kHid,
              kW2 = kB1 + kHid, kB2 = kW2 + kHid * 2 * kHid, kWo = kB2 + kHid, kBo = kWo + kOut * kHid,
              kParams = kBo + kOut;
static_assert(kParams == CF_MPNN_PARAMS, "parameter count");

__device__ __forceinline__ float bf(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ __nv_bfloat16 tobf(float v) { return __float2bfloat16_rn(v); }

// Forward of one message-passing layer over a tile of kFwdTile = 16 nodes on
// the tensor cores: out = act(W [in_i, mean_j in_j] + b) as one
// mma.sync.m16n8k16 (BF16 operands, FP32 accumulation) per 16 input columns
// and 8 output units, a warp per 8 units.  FIRST: `in` is the FP32 feature
// array (rounded to BF16 on load).  AGG=false (output layer): out = W in + b
// + x[0:6] (FP32 out).  The node's own inputs are BF16 already; the FP32
// neighbour mean enters as two BF16 terms, hi = bf16(mean) and lo =
// bf16(mean - hi), both against the same weight columns, so it keeps ~16
// significant bits.  Operands sit in shared memory as BF16 rows: each half of
// [in, mean] padded with zeros to a multiple of 16 columns, W padded the same
// way (and to a multiple of 8 units), row strides 8 elements past the padded
// width so that the fragment loads of the 8 row groups x 4 column pairs hit
// 32 distinct banks.  Loads are issued before use: the weights as 16-B chunks,
// the neighbour lists, then the neighbours' features.  Accumulation: the bias,
// then the 16-column steps in ascending order, then the mean's low terms.
constexpr int kFwdTile = 16;
template <int DIN, int DOUT, bool AGG>
struct FwdShape {
  static constexpr int DINP = (DIN + 15) / 16 * 16;
  static constexpr int CAT = AGG ? 2 * DIN : DIN;      // the weight row's width in global memory
  static constexpr int CATP = AGG ? 2 * DINP : DINP;   // ... padded, in shared memory
  static constexpr int DOUTP = (DOUT + 7) / 8 * 8;
  static constexpr int LD = CATP + 8;                  // BF16 row stride of sW and sX
  static constexpr int LDL = DINP + 8;                 // ... of the mean's low terms
  static constexpr int SMEM = (DOUTP * LD + kFwdTile * LD + (AGG ? kFwdTile * LDL : 0)) * 2 + DOUTP * 4;
};

__device__ __forceinline__ unsigned ld_bf16x2(const __nv_bfloat16* p) {
  return *reinterpret_cast<const unsigned*>(p);
}
// D += A B: A 16x16 row-major (4 regs), B 16x8 column-major (2 regs), D 16x8 FP32
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                               unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

template <int DIN, int DOUT, bool FIRST, bool AGG, bool RELU>
__global__ void __launch_bounds__(kThreads) layer_fwd(const void* in_, const int* __restrict__ nbr,
                                                      const float* __restrict__ inv_deg,
                                                      const __nv_bfloat16* __restrict__ W,
                                                      const __nv_bfloat16* __restrict__ b, void* out_,
                                                      const float* __restrict__ x_skip, int N) {
  using S = FwdShape<DIN, DOUT, AGG>;
  constexpr int CAT = S::CAT, CATP = S::CATP, DINP = S::DINP, DOUTP = S::DOUTP, LD = S::LD, LDL = S::LDL;
  static_assert(CAT % 8 == 0, "weight rows in 16-B chunks");
  extern __shared__ __align__(16) unsigned char fsm_raw[];
  __nv_bfloat16* sW = reinterpret_cast<__nv_bfloat16*>(fsm_raw);  // [DOUTP][LD]
  __nv_bfloat16* sX = sW + DOUTP * LD;                            // [kFwdTile][LD]: in | mean (hi)
  __nv_bfloat16* sLo = sX + kFwdTile * LD;                        // [kFwdTile][LDL]: mean (lo)
  float* sB = reinterpret_cast<float*>(sLo + (AGG ? kFwdTile * LDL : 0));  // [DOUTP]
  const int tid = threadIdx.x;
  const int n0 = blockIdx.x * kFwdTile;
  const __nv_bfloat16 zero = tobf(0.f);
  // column c of a global weight row -> its padded column
  auto wcol = [](int c) { return c < DIN ? c : DINP + (c - DIN); };
  {
    constexpr int NCH = DOUT * CAT / 8, PER = (NCH + kThreads - 1) / kThreads;
    uint4 wv[PER];
#pragma unroll
    for (int j = 0; j < PER; j++) {
      const int q = tid + j * kThreads;
      if (q < NCH) wv[j] = __ldg(reinterpret_cast<const uint4*>(W) + q);
    }
#pragma unroll
    for (int j = 0; j < PER; j++) {
      const int q = tid + j * kThreads;
      if (q < NCH) {
        const __nv_bfloat16* h = reinterpret_cast<const __nv_bfloat16*>(&wv[j]);
#pragma unroll
        for (int t = 0; t < 8; t++) {
          const int idx = 8 * q + t, u = idx / CAT, c = idx % CAT;
          sW[u * LD + wcol(c)] = h[t];
        }
      }
    }
    // the padding (columns past each half's width, units past DOUT): zeros
    constexpr int PADC = CATP - CAT;
    if constexpr (PADC > 0) {
      for (int e = tid; e < DOUT * PADC; e += kThreads) {
        const int u = e / PADC, pc = e % PADC;
        const int col = AGG ? (pc < DINP - DIN ? DIN + pc : DINP + DIN + (pc - (DINP - DIN))) : DIN + pc;
        sW[u * LD + col] = zero;
      }
    }
    for (int e = tid; e < (DOUTP - DOUT) * CATP; e += kThreads) sW[(DOUT + e / CATP) * LD + e % CATP] = zero;
  }
  for (int k = tid; k < DOUTP; k += kThreads) sB[k] = k < DOUT ? bf(b[k]) : 0.f;
  auto load_in = [&](int i, int k) -> float {
    if (FIRST) return bf(tobf(reinterpret_cast<const float*>(in_)[(size_t)i * DIN + k]));
    return bf(reinterpret_cast<const __nv_bfloat16*>(in_)[(size_t)i * DIN + k]);
  };
  {
    constexpr int NE = kFwdTile * DIN, EPT = (NE + kThreads - 1) / kThreads;
    int jn[EPT][CF_K_GRAPH];
#pragma unroll
    for (int j = 0; j < EPT; j++) {
      const int e = tid + j * kThreads, i = n0 + e / DIN;
      const bool ok = e < NE && i < N;
#pragma unroll
      for (int q = 0; q < CF_K_GRAPH; q++) jn[j][q] = (AGG && ok) ? nbr[(size_t)i * CF_K_GRAPH + q] : -1;
    }
#pragma unroll
    for (int j = 0; j < EPT; j++) {
      const int e = tid + j * kThreads, s = e / DIN, k = e % DIN, i = n0 + s;
      if (e >= NE) continue;
      float v = 0.f, a = 0.f;
      if (i < N) {
        v = load_in(i, k);
        if (AGG) {
          float x[CF_K_GRAPH];
#pragma unroll
          for (int q = 0; q < CF_K_GRAPH; q++) x[q] = jn[j][q] >= 0 ? load_in(jn[j][q], k) : 0.f;
#pragma unroll
          for (int q = 0; q < CF_K_GRAPH; q++)
            if (jn[j][q] >= 0) a += x[q];
          a *= inv_deg[i];
        }
      }
      sX[s * LD + k] = tobf(v);  // exact: v is a BF16 value
      if (AGG) {
        const __nv_bfloat16 hi = tobf(a);
        sX[s * LD + DINP + k] = hi;
        sLo[s * LDL + k] = tobf(a - bf(hi));
      }
    }
    // the input padding columns: zeros
    constexpr int PADX = DINP - DIN;
    if constexpr (PADX > 0) {
      for (int e = tid; e < kFwdTile * PADX; e += kThreads) {
        const int s = e / PADX, k = DIN + e % PADX;
        sX[s * LD + k] = zero;
        if (AGG) {
          sX[s * LD + DINP + k] = zero;
          sLo[s * LDL + k] = zero;
        }
      }
    }
  }
  __syncthreads();
  auto store = [&](int i, int u, float acc) {
    if (RELU) acc = fmaxf(acc, 0.f);
    if (AGG) {
      reinterpret_cast<__nv_bfloat16*>(out_)[(size_t)i * DOUT + u] = tobf(acc);
    } else {
      reinterpret_cast<float*>(out_)[(size_t)i * DOUT + u] = acc + x_skip[(size_t)i * kIn + u];
    }
  };
  // fragments of m16n8k16: row group g = lane / 4, column pair t = lane % 4
  const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  for (int nt = warp; nt < DOUTP / 8; nt += kThreads / 32) {
    const int u0 = nt * 8;
    float d[4];
    d[0] = d[2] = sB[u0 + 2 * t];
    d[1] = d[3] = sB[u0 + 2 * t + 1];
    const __nv_bfloat16* wr = sW + (u0 + g) * LD + 2 * t;
    const __nv_bfloat16* x0 = sX + g * LD + 2 * t;
    const __nv_bfloat16* x8 = sX + (g + 8) * LD + 2 * t;
#pragma unroll
    for (int k0 = 0; k0 < CATP; k0 += 16)
      mma_bf16_16816(d, ld_bf16x2(x0 + k0), ld_bf16x2(x8 + k0), ld_bf16x2(x0 + k0 + 8), ld_bf16x2(x8 + k0 + 8),
                     ld_bf16x2(wr + k0), ld_bf16x2(wr + k0 + 8));
    if (AGG) {
      const __nv_bfloat16* l0 = sLo + g * LDL + 2 * t;
      const __nv_bfloat16* l8 = sLo + (g + 8) * LDL + 2 * t;
#pragma unroll
      for (int k0 = 0; k0 < DINP; k0 += 16)
        mma_bf16_16816(d, ld_bf16x2(l0 + k0), ld_bf16x2(l8 + k0), ld_bf16x2(l0 + k0 + 8), ld_bf16x2(l8 + k0 + 8),
                       ld_bf16x2(wr + DINP + k0), ld_bf16x2(wr + DINP + k0 + 8));
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int i = n0 + g + 8 * h;
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int u = u0 + 2 * t + e;
        if (i < N && u < DOUT) store(i, u, d[2 * h + e]);
      }
    }
  }
}

// Output layer backward over a tile: loss = mean over N*6 of (out - target)^2;
// dh3 = Wo^T dy; per-CTA partial gradients of Wo, bo and the loss.
__global__ void __launch_bounds__(kThreads) out_bwd(const float* __restrict__ out, const float* __restrict__ tgt,
                                                    const __nv_bfloat16* __restrict__ h3,
                                                    const __nv_bfloat16* __restrict__ Wo, float* __restrict__ dh3,
                                                    float* __restrict__ part, double* __restrict__ loss_part, int N) {
  __shared__ float sdy[kTileNodes * kOut];
  __shared__ float sh[kTileNodes * kHid];
  __shared__ float sW[kOut * kHid];
  __shared__ double sl[kThreads / 32];
  const int n0 = blockIdx.x * kTileNodes;
  const float scale = 2.f / (6.f * (float)N);
  for (int k = threadIdx.x; k < kOut * kHid; k += kThreads) sW[k] = bf(Wo[k]);
  double l = 0.0;
  for (int e = threadIdx.x; e < kTileNodes * kOut; e += kThreads) {
    const int s = e / kOut, c = e % kOut, i = n0 + s;
    float d = 0.f;
    if (i < N) {
      d = out[(size_t)i * kOut + c] - tgt[(size_t)i * kOut + c];
      l += (double)d * d;
    }
    sdy[e] = d * scale;
  }
  for (int e = threadIdx.x; e < kTileNodes * kHid; e += kThreads) {
    const int i = n0 + e / kHid;
    sh[e] = i < N ? bf(h3[(size_t)i * kHid + e % kHid]) : 0.f;
  }
  l = warp_sum_d(l);
  if ((threadIdx.x & 31) == 0) sl[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < kThreads / 32; q++) t += sl[q];
    loss_part[blockIdx.x] = t;
  }
  // dh3 = Wo^T dy
  for (int e = threadIdx.x; e < kTileNodes * kHid; e += kThreads) {
    const int s = e / kHid, k = e % kHid, i = n0 + s;
    if (i >= N) continue;
    float a = 0.f;
#pragma unroll
    for (int c = 0; c < kOut; c++) a = fmaf(sW[c * kHid + k], sdy[s * kOut + c], a);
    dh3[(size_t)i * kHid + k] = a;
  }
  // partial gradients: Wo[c][k] = sum_s dy[s][c] h3[s][k], bo[c] = sum_s dy[s][c]
  float* p = part + (size_t)blockIdx.x * (kOut * kHid + kOut);
  for (int q = threadIdx.x; q < kOut * kHid + kOut; q += kThreads) {
    float a = 0.f;
    if (q < kOut * kHid) {
      const int c = q / kHid, k = q % kHid;
      for (int s = 0; s < kTileNodes; s++) a = fmaf(sdy[s * kOut + c], sh[s * kHid + k], a);
    } else {
      for (int s = 0; s < kTileNodes; s++) a += sdy[s * kOut + (q - kOut * kHid)];
    }
    p[q] = a;
  }
}

// Hidden layer backward over a tile: dz = dh * (h > 0); partial gradients of
// W (DOUT x 2 DIN) and b; dcat = W^T dz (FP32, [N][2 DIN]).
template <int DIN, bool FIRST>
__global__ void __launch_bounds__(kThreads) layer_bwd(const void* in_, const int* __restrict__ nbr,
                                                      const float* __restrict__ inv_deg,
                                                      const __nv_bfloat16* __restrict__ W,
                                                      const __nv_bfloat16* __restrict__ h,
                                                      const float* __restrict__ dh, float* __restrict__ dcat,
                                                      float* __restrict__ part, int N) {
  constexpr int CAT = 2 * DIN, DOUT = kHid;
  extern __shared__ float smem[];
  float* sW = smem;                       // [DOUT][CAT]
  float* sX = sW + DOUT * CAT;            // [32][CAT]
  float* sZ = sX + kTileNodes * CAT;      // [32][DOUT]
  const int n0 = blockIdx.x * kTileNodes;
  for (int k = threadIdx.x; k < DOUT * CAT; k += kThreads) sW[k] = bf(W[k]);
  auto load_in = [&](int i, int k) -> float {
    if (FIRST) return bf(tobf(reinterpret_cast<const float*>(in_)[(size_t)i * DIN + k]));
    return bf(reinterpret_cast<const __nv_bfloat16*>(in_)[(size_t)i * DIN + k]);
  };
  for (int e = threadIdx.x; e < kTileNodes * DIN; e += kThreads) {
    const int s = e / DIN, k = e % DIN, i = n0 + s;
    float v = 0.f, a = 0.f;
    if (i < N) {
      v = load_in(i, k);
#pragma unroll
      for (int q = 0; q < CF_K_GRAPH; q++) {
        const int j = nbr[(size_t)i * CF_K_GRAPH + q];
        if (j >= 0) a += load_in(j, k);
      }
      a *= inv_deg[i];
    }
    sX[s * CAT + k] = v;
    sX[s * CAT + DIN + k] = a;
  }
  for (int e = threadIdx.x; e < kTileNodes * DOUT; e += kThreads) {
    const int i = n0 + e / DOUT;
    float z = 0.f;
    if (i < N) {
      const size_t o = (size_t)i * DOUT + e % DOUT;
      z = bf(h[o]) > 0.f ? dh[o] : 0.f;
    }
    sZ[e] = z;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kTileNodes * CAT; e += kThreads) {
    const int s = e / CAT, k = e % CAT, i = n0 + s;
    if (i >= N) continue;
    float a = 0.f;
#pragma unroll 8
    for (int u = 0; u < DOUT; u++) a = fmaf(sW[u * CAT + k], sZ[s * DOUT + u], a);
    dcat[(size_t)i * CAT + k] = a;
  }
  float* p = part + (size_t)blockIdx.x * (DOUT * CAT + DOUT);
  for (int q = threadIdx.x; q < DOUT * CAT + DOUT; q += kThreads) {
    float a = 0.f;
    if (q < DOUT * CAT) {
      const int u = q / CAT, k = q % CAT;
      for (int s = 0; s < kTileNodes; s++) a = fmaf(sZ[s * DOUT + u], sX[s * CAT + k], a);
    } else {
      for (int s = 0; s < kTileNodes; s++) a += sZ[s * DOUT + (q - DOUT * CAT)];
    }
    p[q] = a;
  }
}

// d in_j = dcat_j[0:DIN] + sum over the nodes i that list j (reverse graph,
// fixed order) of inv_deg_i * dcat_i[DIN:2 DIN]
template <int DIN>
__global__ void grad_gather(const float* __restrict__ dcat, const int* __restrict__ rev_ptr,
                            const int* __restrict__ rev_idx, const float* __restrict__ inv_deg,
                            float* __restrict__ din, int N) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N * DIN) return;
  const int j = e / DIN, k = e % DIN;
  float a = dcat[(size_t)j * 2 * DIN + k];
  for (int q = rev_ptr[j]; q < rev_ptr[j + 1]; q++) {
    const int i = rev_idx[q];
    a = fmaf(inv_deg[i], dcat[(size_t)i * 2 * DIN + DIN + k], a);
  }
  din[e] = a;
}

// grad[p] = sum over CTAs (in order) of part[cta][p]
__global__ void reduce_parts(const float* __restrict__ part, int ctas, int np, float* __restrict__ grad) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  float a = 0.f;
  for (int c = 0; c < ctas; c++) a += part[(size_t)c * np + q];
  grad[q] = a;
}

__global__ void reduce_loss(const double* __restrict__ part, int n, double* __restrict__ out, int N) {
  double a = 0.0;
  for (int k = threadIdx.x; k < n; k += 32) a += part[k];
  a = warp_sum_d(a);
  if (threadIdx.x == 0) *out = a / (6.0 * N);
}

// Adam (FP32 master weights), then the BF16 copy
__global__ void adam_step(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                          const float* __restrict__ g, __nv_bfloat16* __restrict__ wb, int n, float lr, float b1,
                          float b2, float c1, float c2, float eps) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float gg = g[q];
  const float mm = b1 * m[q] + (1.f - b1) * gg;
  const float vv = b2 * v[q] + (1.f - b2) * gg * gg;
  m[q] = mm;
  v[q] = vv;
  const float ww = w[q] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  w[q] = ww;
  wb[q] = tobf(ww);
}

__global__ void to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, int n) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) wb[q] = tobf(w[q]);
}

// graph of a problem's nodes: neighbour lists (-1 = none) and 1/degree
__global__ void graph_from_nodes(const cf_deform_node* __restrict__ nodes, int N, int* __restrict__ nbr,
                                 float* __restrict__ inv_deg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int nn = min(max(nodes[i].num_neighbors, 0), CF_K_GRAPH);
  int deg = 0;
#pragma unroll
  for (int k = 0; k < CF_K_GRAPH; k++) {
    const int j = nodes[i].neighbors[k];
    const bool ok = k < nn && j >= 0 && j < N;
    nbr[(size_t)i * CF_K_GRAPH + k] = ok ? j : -1;
    deg += ok;
  }
  inv_deg[i] = deg ? 1.f / (float)deg : 0.f;
}

// ---- increments between node transforms (centred DQs of the same node) ----

// rotation vector of a unit quaternion (w >= 0 hemisphere)
__device__ __forceinline__ float3 quat_log(float4 q) {
  if (q.w < 0.f) q = make_float4(-q.x, -q.y, -q.z, -q.w);
  const float s = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z);
  const float ang = 2.f * atan2f(s, q.w);
  const float f = s > 1e-12f ? ang / s : 2.f;
  return f3(q.x * f, q.y * f, q.z * f);
}
__device__ __forceinline__ float4 quat_exp(float3 w) {
  const float th = sqrtf(w.x * w.x + w.y * w.y + w.z * w.z);
  float sn, cs;
  sincosf(0.5f * th, &sn, &cs);
  const float f = th > 1e-12f ? sn / th : 0.5f;
  return make_float4(w.x * f, w.y * f, w.z * f, cs);
}
// (w, t) with T_to = D(w, t) (x) T_from: R_D = R_to R_from^T, t_D = t_to - R_D t_from
__device__ __forceinline__ void dq_increment(DQ to, DQ from, float* o) {
  const float4 qd = qmul(qnormalize(to.r), qconj(qnormalize(from.r)));
  const float3 w = quat_log(qd);
  const float3 tt = dq_translation(to), tf = dq_translation(from);
  DQ d;
  d.r = qd;
  const float3 rt = dq_rotate(d, tf);
  o[0] = w.x; o[1] = w.y; o[2] = w.z;
  o[3] = tt.x - rt.x; o[4] = tt.y - rt.y; o[5] = tt.z - rt.z;
}
// D(w, t) (x) T
__device__ __forceinline__ DQ dq_apply_increment(DQ T, const float* o) {
  DQ d;
  d.r = quat_exp(f3(o[0], o[1], o[2]));
  const float3 tT = dq_translation(T);
  const float3 rt = dq_rotate(d, tT);
  const float3 t = f3(rt.x + o[3], rt.y + o[4], rt.z + o[5]);
  DQ out;
  out.r = qnormalize(qmul(d.r, qnormalize(T.r)));
  out.d = qmul(make_float4(t.x, t.y, t.z, 0.f), out.r);
  out.d.x *= 0.5f; out.d.y *= 0.5f; out.d.z *= 0.5f; out.d.w *= 0.5f;
  return out;
}

__global__ void increments_kernel(const cf_dual_quat* __restrict__ to, const cf_dual_quat* __restrict__ from, int n,
                                  float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float o[6];
  dq_increment(load_dq_cg(to + i), load_dq_cg(from + i), o);
#pragma unroll
  for (int k = 0; k < 6; k++) out[(size_t)i * 6 + k] = o[k];
}

// Features of every node at the warm start T (= T_{t-1}) with the history
// hist = [T_{t-2}, T_{t-3}, T_{t-4}]: the three increments (scaled) and the
// mean / max |residual| (mm) of the node's valid correspondences (the
// residual launch at T must have run; warp per node over its incidences).
__global__ void features_kernel(const cf_dual_quat* __restrict__ T, const cf_dual_quat* __restrict__ hist, int N,
                                const int* __restrict__ inc_start, const int* __restrict__ inc,
                                const float2* __restrict__ c_fr, float* __restrict__ feat) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= N) return;
  float s = 0.f, mx = 0.f;
  int cnt = 0;
  // 4 incidences per lane in flight: their ids, then the (weight, residual)
  // pair of each (8 B, written by the residual launch), summed in incidence order
  const int q1 = inc_start[i + 1];
  for (int q0 = inc_start[i] + lane; q0 < q1; q0 += 4 * 32) {
    int c[4];
#pragma unroll
    for (int b = 0; b < 4; b++) c[b] = q0 + 32 * b < q1 ? (inc[q0 + 32 * b] >> 2) : -1;
    float f[4], r[4];
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const float2 fr = c[b] >= 0 ? __ldg(c_fr + c[b]) : make_float2(0.f, 0.f);
      f[b] = fr.x;
      r[b] = fr.y;
    }
#pragma unroll
    for (int b = 0; b < 4; b++)
      if (f[b] > 0.f) {
        const float ra = fabsf(r[b]);
        s += ra;
        mx = fmaxf(mx, ra);
        cnt++;
      }
  }
  s = warp_sum_f(s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  }
  if (lane < 3) {
    const DQ a = load_dq_cg(lane == 0 ? T + i : hist + (size_t)(lane - 1) * N + i);
    const DQ b = load_dq_cg(hist + (size_t)lane * N + i);
    float o[6];
    dq_increment(a, b, o);
#pragma unroll
    for (int k = 0; k < 3; k++) feat[(size_t)i * kIn + 6 * lane + k] = o[k] * CF_MPNN_ROT_SCALE;
#pragma unroll
    for (int k = 3; k < 6; k++) feat[(size_t)i * kIn + 6 * lane + k] = o[k] * CF_MPNN_TRANS_SCALE;
  } else if (lane == 3) {
    feat[(size_t)i * kIn + 18] = cnt ? s / (float)cnt * CF_MPNN_RES_SCALE : 0.f;
    feat[(size_t)i * kIn + 19] = mx * CF_MPNN_RES_SCALE;
  }
}

// T <- D(prediction) (x) T for every node (the warm start kept in T_save),
// and the node-centred plain DQs for the skinning
__global__ void apply_prediction(cf_dual_quat* __restrict__ T, cf_dual_quat* __restrict__ T_save,
                                 cf_dual_quat* __restrict__ plain, const cf_deform_node* __restrict__ nodes,
                                 const float* __restrict__ pred, int N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const DQ t0 = load_dq_cg(T + i);
  store_dq(T_save + i, t0);
  float o[6];
#pragma unroll
  for (int k = 0; k < 3; k++) o[k] = pred[(size_t)i * kOut + k] / CF_MPNN_ROT_SCALE;
#pragma unroll
  for (int k = 3; k < 6; k++) o[k] = pred[(size_t)i * kOut + k] / CF_MPNN_TRANS_SCALE;
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 6; k++) ok &= isfinite(o[k]);
  const DQ t1 = ok ? dq_apply_increment(t0, o) : t0;
  store_dq(T + i, t1);
  store_dq(plain + i, dq_centered(t1, node_pos(nodes, i)));
}

// Keeps the predicted start only if its energy is below the warm start's
// (gate[0] warm start, gate[1] prediction); otherwise restores the warm start.
__global__ void gate_prediction(cf_dual_quat* __restrict__ T, const cf_dual_quat* __restrict__ T_save,
                                cf_dual_quat* __restrict__ plain, const cf_deform_node* __restrict__ nodes,
                                DevStats* __restrict__ st, int N) {
  const bool reject = !(st->gate[1] <= st->gate[0]);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) st->init_rejected = reject ? 1 : 0;
  if (!reject || i >= N) return;
  const DQ t0 = load_dq_cg(T_save + i);
  store_dq(T + i, t0);
  store_dq(plain + i, dq_centered(t0, node_pos(nodes, i)));
}

inline int cdiv(int a, int b) { return (a + b - 1) / b; }

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

int mpnn_param_count() { return kParams; }

static int layer_bwd_smem(int din) { return (kHid * 2 * din + kTileNodes * 2 * din + kTileNodes * kHid) * 4; }

template <typename T>
static cudaError_t alloc_n(T** p, size_t n) {
  *p = nullptr;
  return cudaMalloc((void**)p, (n ? n : 1) * sizeof(T));
}

cudaError_t mpnn_alloc(Mpnn& m, int max_nodes) {
  m.max_nodes = max_nodes;
  const size_t N = (size_t)max_nodes;
  const int ctas = cdiv(max_nodes, kTileNodes);
  cudaError_t e;
#define A_(p, n) if ((e = alloc_n(&(p), (n))) != cudaSuccess) return e
  A_(m.w, kParams); A_(m.m, kParams); A_(m.v, kParams); A_(m.g, kParams);
  if ((e = cudaMalloc(&m.wb, sizeof(__nv_bfloat16) * kParams)) != cudaSuccess) return e;
  A_(m.nbr, N * CF_K_GRAPH); A_(m.inv_deg, N);
  A_(m.rev_ptr, N + 1); A_(m.rev_idx, N * CF_K_GRAPH);
  A_(m.feat, N * kIn); A_(m.tgt, N * kOut); A_(m.out, N * kOut);
  if ((e = cudaMalloc(&m.h1, sizeof(__nv_bfloat16) * N * kHid)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&m.h2, sizeof(__nv_bfloat16) * N * kHid)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&m.h3, sizeof(__nv_bfloat16) * N * kHid)) != cudaSuccess) return e;
  A_(m.dh, N * kHid); A_(m.dh2, N * kHid); A_(m.dcat, N * 2 * kHid);
  A_(m.part, (size_t)ctas * (kHid * 2 * kHid + kHid)); A_(m.loss_part, (size_t)ctas); A_(m.loss, 1);
#undef A_
  if ((e = cudaMemset(m.m, 0, sizeof(float) * kParams)) != cudaSuccess) return e;
  return cudaMemset(m.v, 0, sizeof(float) * kParams);
}

void mpnn_free(Mpnn& m) {
  void* ps[] = {m.w, m.m, m.v, m.g, m.wb, m.nbr, m.inv_deg, m.rev_ptr, m.rev_idx, m.feat, m.tgt, m.out,
                m.h1, m.h2, m.h3, m.dh, m.dh2, m.dcat, m.part, m.loss_part, m.loss};
  for (void* p : ps)
    if (p) cudaFree(p);
  m = Mpnn();
}

cudaError_t mpnn_refresh_bf16(const Mpnn& m, cudaStream_t s) {
  to_bf16<<<cdiv(kParams, 256), 256, 0, s>>>(m.w, reinterpret_cast<__nv_bfloat16*>(m.wb), kParams);
  return cudaGetLastError();
}

cudaError_t mpnn_graph_from_nodes(Mpnn& m, const cf_deform_node* nodes, int N, cudaStream_t s) {
  m.N = N;
  if (N <= 0) return cudaSuccess;
  graph_from_nodes<<<cdiv(N, 128), 128, 0, s>>>(nodes, N, m.nbr, m.inv_deg);
  return cudaGetLastError();
}

cudaError_t mpnn_forward(const Mpnn& m, const float* feat, float* out, cudaStream_t s) {
  const int N = m.N;
  if (N <= 0) return cudaSuccess;
  const int g = cdiv(N, kFwdTile);
  const __nv_bfloat16* wb = reinterpret_cast<const __nv_bfloat16*>(m.wb);
  const int s0 = FwdShape<kIn, kHid, true>::SMEM, s1 = FwdShape<kHid, kHid, true>::SMEM,
            so = FwdShape<kHid, kOut, false>::SMEM;
  cudaError_t e = cudaFuncSetAttribute(layer_fwd<kHid, kHid, false, true, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, s1);
  if (e != cudaSuccess) return e;
  layer_fwd<kIn, kHid, true, true, true><<<g, kThreads, s0, s>>>(feat, m.nbr, m.inv_deg, wb + kW0, wb + kB0, m.h1,
                                                                  nullptr, N);
  layer_fwd<kHid, kHid, false, true, true><<<g, kThreads, s1, s>>>(m.h1, m.nbr, m.inv_deg, wb + kW1, wb + kB1, m.h2,
                                                                    nullptr, N);
  layer_fwd<kHid, kHid, false, true, true><<<g, kThreads, s1, s>>>(m.h2, m.nbr, m.inv_deg, wb + kW2, wb + kB2, m.h3,
                                                                    nullptr, N);
  layer_fwd<kHid, kOut, false, false, false><<<g, kThreads, so, s>>>(m.h3, nullptr, nullptr, wb + kWo, wb + kBo, out,
                                                                      feat, N);
  return cudaGetLastError();
}


// forward + backward at (feat, tgt): loss (device) and the gradient m.g
cudaError_t mpnn_gradients(Mpnn& m, const float* feat, const float* tgt, cudaStream_t s) {
  const int N = m.N;
  if (N <= 0) return cudaSuccess;
  const int g = cdiv(N, kTileNodes);
  cudaError_t e = mpnn_forward(m, feat, m.out, s);
  if (e != cudaSuccess) return e;
  const __nv_bfloat16* wb = reinterpret_cast<const __nv_bfloat16*>(m.wb);
  out_bwd<<<g, kThreads, 0, s>>>(m.out, tgt, reinterpret_cast<const __nv_bfloat16*>(m.h3), wb + kWo, m.dh, m.part,
                                 m.loss_part, N);
  reduce_parts<<<cdiv(kOut * kHid + kOut, 128), 128, 0, s>>>(m.part, g, kOut * kHid + kOut, m.g + kWo);
  reduce_loss<<<1, 32, 0, s>>>(m.loss_part, g, m.loss, N);
  const int sm64 = layer_bwd_smem(kHid), sm20 = layer_bwd_smem(kIn);
  if ((e = cudaFuncSetAttribute(layer_bwd<kHid, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm64)) !=
      cudaSuccess)
    return e;
  // layer 3 (h2 -> h3)
  layer_bwd<kHid, false><<<g, kThreads, sm64, s>>>(m.h2, m.nbr, m.inv_deg, wb + kW2,
                                                   reinterpret_cast<const __nv_bfloat16*>(m.h3), m.dh, m.dcat, m.part, N);
  reduce_parts<<<cdiv(kHid * 2 * kHid + kHid, 128), 128, 0, s>>>(m.part, g, kHid * 2 * kHid + kHid, m.g + kW2);
  grad_gather<kHid><<<cdiv(N * kHid, 256), 256, 0, s>>>(m.dcat, m.rev_ptr, m.rev_idx, m.inv_deg, m.dh2, N);
  // layer 2 (h1 -> h2)
  layer_bwd<kHid, false><<<g, kThreads, sm64, s>>>(m.h1, m.nbr, m.inv_deg, wb + kW1,
                                                   reinterpret_cast<const __nv_bfloat16*>(m.h2), m.dh2, m.dcat, m.part, N);
  reduce_parts<<<cdiv(kHid * 2 * kHid + kHid, 128), 128, 0, s>>>(m.part, g, kHid * 2 * kHid + kHid, m.g + kW1);
  grad_gather<kHid><<<cdiv(N * kHid, 256), 256, 0, s>>>(m.dcat, m.rev_ptr, m.rev_idx, m.inv_deg, m.dh, N);
  // layer 1 (x -> h1)
  layer_bwd<kIn, true><<<g, kThreads, sm20, s>>>(feat, m.nbr, m.inv_deg, wb + kW0,
                                                 reinterpret_cast<const __nv_bfloat16*>(m.h1), m.dh, m.dcat, m.part, N);
  reduce_parts<<<cdiv(kHid * 2 * kIn + kHid, 128), 128, 0, s>>>(m.part, g, kHid * 2 * kIn + kHid, m.g + kW0);
  return cudaGetLastError();
}

cudaError_t mpnn_adam(Mpnn& m, float lr, cudaStream_t s) {
  m.step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)m.step), c2 = 1.f - powf(b2, (float)m.step);
  adam_step<<<cdiv(kParams, 256), 256, 0, s>>>(m.w, m.m, m.v, m.g, reinterpret_cast<__nv_bfloat16*>(m.wb), kParams,
                                                lr, b1, b2, c1, c2, 1e-8f);
  return cudaGetLastError();
}

cudaError_t launch_increments(const cf_dual_quat* to, const cf_dual_quat* from, int n, float* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  increments_kernel<<<cdiv(n, 128), 128, 0, s>>>(to, from, n, out);
  return cudaGetLastError();
}

cudaError_t launch_features(const Work& w, const cf_dual_quat* T, const cf_dual_quat* hist, int N, float* feat,
                            cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  features_kernel<<<cdiv(N * 32, 256), 256, 0, s>>>(T, hist, N, w.inc_start, w.inc, w.c_fr, feat);
  return cudaGetLastError();
}

cudaError_t launch_apply_prediction(const Work& w, cf_dual_quat* T, const cf_deform_node* nodes, const float* pred,
                                    int N, cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  apply_prediction<<<cdiv(N, 128), 128, 0, s>>>(T, w.T_save, w.plain, nodes, pred, N);
  return cudaGetLastError();
}

cudaError_t launch_gate_prediction(const Work& w, cf_dual_quat* T, const cf_deform_node* nodes, int N,
                                   cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  gate_prediction<<<cdiv(N, 128), 128, 0, s>>>(T, w.T_save, w.plain, nodes, w.stats, N);
  return cudaGetLastError();
}

}  // namespace cf
