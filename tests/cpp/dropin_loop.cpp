// The reference's per-frame loop written against the C++ drop-in classes.
//
// Types below have the byte layouts of CUDAFusion's include/types.h
// (DualQuat, DeformNode, Correspondence, DeviceArray<T>), which is what a
// caller of the drop-in holds.  The loop is the one of
// DynamicFusionPipeline::process_frame (include/fusion_app.h:386-390 and
// :525-550): solve() then WarpField::apply_twist_increment(), G times, the
// correspondences' src fixed.  Then one solve_frame() (the whole loop on the
// GPU) from the same start.
//
// usage: dropin_loop nodev
//        dropin_loop <dir> <G> <P> <lambda_smooth> <max_rot> <max_trans>
//   <dir> holds nodes.bin, corrs.bin, canon.bin, init.bin (raw structs);
//   writes loop.bin, frame.bin (final transforms), dx0.bin, sys.bin.
#include <cstdio>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "cudafusion_b200.hpp"

struct DualQuat {
  float4 real;
  float4 dual;
};
struct DeformNode {
  float3 pos;
  float3 normal;
  float radius;
  int neighbors[8];
  float neighbor_w[8];
  int num_neighbors;
};
struct Correspondence {
  float3 src, dst, normal;
  int node_ids[4];
  float node_ws[4];
  float weight;
  bool valid;
};
template <class T>
struct DeviceArray {
  T* data = nullptr;
  size_t count = 0;
  DeviceArray() = default;
  DeviceArray(const DeviceArray&) = delete;
  ~DeviceArray() { release(); }
  void allocate(size_t n) {
    release();
    count = n;
    if (n && cudaMalloc(&data, n * sizeof(T)) != cudaSuccess) {
      std::fprintf(stderr, "cudaMalloc failed\n");
      std::exit(2);
    }
  }
  void release() {
    if (data) cudaFree(data);
    data = nullptr;
    count = 0;
  }
  void upload(const std::vector<T>& v) {
    if (count != v.size()) allocate(v.size());
    cudaMemcpy(data, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  }
  void download(std::vector<T>& v) const {
    v.resize(count);
    cudaMemcpy(v.data(), data, count * sizeof(T), cudaMemcpyDeviceToHost);
  }
};
static_assert(sizeof(DualQuat) == 32 && sizeof(DeformNode) == 96 && sizeof(Correspondence) == 76, "layouts");

template <class T>
static std::vector<T> read_all(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  std::vector<char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  std::vector<T> v(b.size() / sizeof(T));
  std::memcpy(v.data(), b.data(), v.size() * sizeof(T));
  return v;
}
template <class T>
static void write_all(const std::string& path, const std::vector<T>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
}

namespace cfb = cudafusion_b200;

int main(int argc, char** argv) {
  if (argc >= 2 && std::string(argv[1]) == "nodev") {
    // Without a GPU the constructor must fail loudly, not fall back.
    try {
      cfb::GaussNewtonSolver s(cfb::GaussNewtonSolver::Params{}, 64, 1024);
    } catch (const cfb::Error& e) {
      std::printf("status %d %s\n", (int)e.status, e.what());
      return e.status == CF_ERR_NO_DEVICE ? 0 : 3;
    }
    return 4;
  }
  if (argc < 7) return 1;
  const std::string dir = argv[1];
  cfb::GaussNewtonSolver::Params prm;
  prm.gn_iterations = std::atoi(argv[2]);
  prm.pcg_iterations = std::atoi(argv[3]);
  prm.lambda_smooth = (float)std::atof(argv[4]);
  const float max_rot = (float)std::atof(argv[5]), max_trans = (float)std::atof(argv[6]);

  auto nodes = read_all<DeformNode>(dir + "/nodes.bin");
  auto corrs_h = read_all<Correspondence>(dir + "/corrs.bin");
  auto canon = read_all<float>(dir + "/canon.bin");
  auto init = read_all<DualQuat>(dir + "/init.bin");
  const int N = (int)nodes.size(), M = (int)corrs_h.size();

  try {
    cfb::GaussNewtonSolver solver(prm, N, M);
    cfb::WarpField<DeformNode, DualQuat> warp(0.025f, N);
    warp.upload_nodes(nodes);
    warp.upload_transforms(init);

    DeviceArray<Correspondence> corrs;
    corrs.upload(corrs_h);
    DeviceArray<float> delta_x;
    for (int g = 0; g < prm.gn_iterations; g++) {
      solver.solve(corrs, M, warp.device_nodes(), warp.device_transforms(), warp.num_nodes(), delta_x);
      if (g == 0) {
        std::vector<float> dx;
        delta_x.download(dx);
        write_all(dir + "/dx0.bin", dx);
        std::vector<int> rp, ci;
        std::vector<float> vals, b;
        solver.system_matrix(rp, ci, vals);
        solver.rhs(b);
        std::vector<float> sys(vals);
        sys.insert(sys.end(), b.begin(), b.end());
        write_all(dir + "/sys.bin", sys);
      }
      warp.apply_twist_increment(delta_x, max_rot, max_trans, 1.0f);
    }
    write_all(dir + "/loop.bin", warp.download_transforms());

    // save/restore round trip, then the whole loop on the GPU from the start
    warp.save_transforms();
    warp.reset_transforms();
    warp.restore_transforms();
    warp.upload_transforms(init);
    DeviceArray<float> d_canon;
    d_canon.upload(canon);
    cf_solve_stats st = solver.solve_frame(warp.device_nodes(), N, d_canon.data, corrs.data, M,
                                           warp.device_transforms(), max_rot, max_trans);
    std::vector<DualQuat> out(N);
    cudaMemcpy(out.data(), warp.device_transforms(), sizeof(DualQuat) * N, cudaMemcpyDeviceToHost);
    write_all(dir + "/frame.bin", out);
    std::printf("energy %.17g %.17g\n", st.energy_initial, st.energy_final);
  } catch (const cfb::Error& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 5;
  }
  return 0;
}
