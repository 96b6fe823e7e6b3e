// cf_noalloc.cu — energy of a warp-field problem without allocating anything.
//
// Some callers cannot allocate device memory where they need this number:
// a tracking loop that runs every frame under a fixed memory budget handed
// to it by a host application (which owns every allocation), or code that
// must not stall — cudaMalloc and cudaFree can synchronise the device and can
// fail under memory pressure.  cf_energy_noalloc serves them: it computes the
// same IRLS energy as the solve reports (data term + ARAP term at the given
// transforms) using only the caller's buffers and a scratch area that lives
// in this library's own static device memory.
//
// The scratch is a file-scope __device__ array of fixed size: the per-node
// plain dual quaternions for at most CF_NOALLOC_MAX_NODES nodes and one FP64
// partial sum per CTA of the energy kernel.  Every GPU that loads this library
// holds it until the process exits.  Host code cannot use the array's name as
// a device address (it is a host-side stand-in), so the first call on each
// device, with that device current, looks the address up with
// cudaGetSymbolAddress and caches it; make that first call before capturing
// the stream into a graph.  All calls share the one array and it keeps the
// last call's contents: calls that overlap on the GPU (two streams, two host
// threads on one device) race on it and must be serialised by the caller.
#include <mutex>

#include "cf_device.cuh"
#include "cf_internal.h"

namespace cf {

namespace {

constexpr int kNaCtas = 592;  // fixed grid: one partial per CTA, fully rewritten each call
constexpr size_t kNaPlainBytes = (size_t)CF_NOALLOC_MAX_NODES * sizeof(cf_dual_quat);
constexpr size_t kNaBytes = kNaPlainBytes + (size_t)kNaCtas * sizeof(double);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

std::mutex g_mu;
constexpr int kMaxDevices = 64;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

__global__ void na_plain_kernel(const cf_deform_node* __restrict__ nodes, const cf_dual_quat* __restrict__ T,
                                cf_dual_quat* __restrict__ plain, int N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  store_dq(plain + i, dq_centered(load_dq_cg(T + i), node_pos(nodes, i)));
}

// Data term over the AoS correspondences plus the ARAP edges enumerated from
// the node lists in the reference's visiting order (each unordered pair from
// its lower endpoint, kernels/solver_kernels.cu:225-233).
__global__ void __launch_bounds__(kThreads) na_energy_kernel(const cf_correspondence* __restrict__ corrs,
                                                             const float* __restrict__ canon, int M,
                                                             const cf_deform_node* __restrict__ nodes,
                                                             const cf_dual_quat* __restrict__ T, int N, float lambda,
                                                             const cf_dual_quat* __restrict__ plain,
                                                             double* __restrict__ part) {
  __shared__ double red[kThreads / 32];
  double e = 0.0;
  const int stride = gridDim.x * kThreads;
  for (int c = blockIdx.x * kThreads + threadIdx.x; c < M; c += stride) {
    const cf_correspondence& k = corrs[c];
    const float we = k.valid ? k.weight : 0.f;
    if (!(we > 0.f)) continue;
    const float3 p = f3(canon[3 * (size_t)c], canon[3 * (size_t)c + 1], canon[3 * (size_t)c + 2]);
    const int4 ids = make_int4(k.node_ids[0], k.node_ids[1], k.node_ids[2], k.node_ids[3]);
    const float4 ws = make_float4(k.node_ws[0], k.node_ws[1], k.node_ws[2], k.node_ws[3]);
    const float3 src = blend_warp(p, ids, ws, plain, N);
    const float res = k.normal.x * (src.x - k.dst.x) + k.normal.y * (src.y - k.dst.y) + k.normal.z * (src.z - k.dst.z);
    const float fw = fmaxf(we, 0.f) * huber_w(res, 0.2f);
    if (fw > 1e-8f) e += (double)fw * (double)res * (double)res;
  }
  for (int q = blockIdx.x * kThreads + threadIdx.x; q < N * CF_K_GRAPH; q += stride) {
    const int i = q / CF_K_GRAPH, k = q % CF_K_GRAPH;
    if (k >= min(nodes[i].num_neighbors, CF_K_GRAPH)) continue;
    const int j = nodes[i].neighbors[k];
    if (j < 0 || j >= N || j <= i) continue;
    const Edge ev = eval_edge(nodes, T, i, j, k, lambda);
    if (ev.el > 0.f)
      e += (double)ev.el * ((double)ev.r.x * ev.r.x + (double)ev.r.y * ev.r.y + (double)ev.r.z * ev.r.z);
  }
  e = warp_sum_d(e);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kThreads / 32 ? red[threadIdx.x] : 0.0;
    t = warp_sum_d(t);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
  }
}

__global__ void na_reduce_kernel(const double* __restrict__ part, double* __restrict__ out) {
  double v = 0.0;
  for (int k = threadIdx.x; k < kNaCtas; k += 32) v += part[k];
  v = warp_sum_d(v);
  if (threadIdx.x == 0) *out = v;
}

}  // namespace

// Device address of the static scratch on the current device.  Looked up
// again on every call made outside a stream capture (cheap), so a context
// torn down and re-created (cudaDeviceReset) never leaves a stale address;
// inside a capture the address of the last uncaptured call is used.
cudaError_t noalloc_scratch(cudaStream_t s, void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_mu);
  if (cap == cudaStreamCaptureStatusNone || !g_scratch_ptr[dev]) {
    if (cap != cudaStreamCaptureStatusNone) return cudaErrorStreamCaptureUnsupported;
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

cudaError_t launch_energy_noalloc(const cf_problem* pr, const cf_dual_quat* T, float lambda, double* d_energy,
                                  cudaStream_t s) {
  void* base = nullptr;
  cudaError_t e = noalloc_scratch(s, &base);
  if (e != cudaSuccess) return e;
  cf_dual_quat* plain = reinterpret_cast<cf_dual_quat*>(base);
  double* part = reinterpret_cast<double*>(static_cast<unsigned char*>(base) + kNaPlainBytes);
  const int N = pr->num_nodes, M = pr->num_corrs;
  if (N > 0) na_plain_kernel<<<(N + 127) / 128, 128, 0, s>>>(pr->nodes, T, plain, N);
  na_energy_kernel<<<kNaCtas, kThreads, 0, s>>>(pr->corrs, pr->canon_points, M, pr->nodes, T, N, lambda, plain,
                                                part);
  na_reduce_kernel<<<1, 32, 0, s>>>(part, d_energy);
  return cudaGetLastError();
}

}  // namespace cf
