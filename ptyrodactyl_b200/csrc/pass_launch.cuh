// Launchers of the pass kernel, one translation unit per grid edge (pass_<n>.cu).
// Each returns the cudaError_t of its launch as int (0 = success).
#pragma once
#include <atomic>

#include "ms_pass.cuh"

namespace ptyro {

// Number of engine kernels enqueued by this process (all devices, all threads).
extern std::atomic<unsigned long long> g_launches;

template <int N1, int N2, int AXIS>
int launch_pass_t(const PassArgs& a, int grid_y, cudaStream_t st) {
  using Geo = PassGeom<N1, N2>;
  constexpr int N = Geo::N, G = Geo::G;
  constexpr int kMaxWarps = 8;
  const int warps = N / G < kMaxWarps ? (N / G > 0 ? N / G : 1) : kMaxWarps;
  const size_t smem = Geo::smem_bytes(warps);
  static bool attr_done = false;  // once per template instance
  if (!attr_done) {
    cudaFuncSetAttribute(ms_pass_kernel<N1, N2, AXIS, kMaxWarps>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)Geo::smem_bytes(kMaxWarps));
    attr_done = true;
  }
  const int lines = warps * G;
  dim3 grid((N + lines - 1) / lines, grid_y);
  ms_pass_kernel<N1, N2, AXIS, kMaxWarps><<<grid, warps * 32, smem, st>>>(a);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

#define PTYRO_DEFINE_PASS_LAUNCHER(NN, N1, N2)                                   \
  int launch_pass_##NN(int axis, const PassArgs& a, int grid_y, cudaStream_t st) { \
    return axis == 0 ? launch_pass_t<N1, N2, 0>(a, grid_y, st)                     \
                     : launch_pass_t<N1, N2, 1>(a, grid_y, st);                    \
  }

int launch_pass_16(int axis, const PassArgs& a, int grid_y, cudaStream_t st);
int launch_pass_32(int axis, const PassArgs& a, int grid_y, cudaStream_t st);
int launch_pass_64(int axis, const PassArgs& a, int grid_y, cudaStream_t st);
int launch_pass_128(int axis, const PassArgs& a, int grid_y, cudaStream_t st);
int launch_pass_256(int axis, const PassArgs& a, int grid_y, cudaStream_t st);
int launch_pass_512(int axis, const PassArgs& a, int grid_y, cudaStream_t st);
int launch_pass_1024(int axis, const PassArgs& a, int grid_y, cudaStream_t st);

}  // namespace ptyro
