// Diagnostics: a dense FP32 FMA stream that measures the CUDA-core FP32 ceiling of
// the device it runs on (the denominator of the multislice roofline), and a
// self-test of the bounded tile wait of the TMA pass kernels.
#include <cuda_runtime.h>

#include <atomic>

#include "../../include/ptyro_b200.h"
#include "ms_wait.cuh"

namespace ptyro {
extern std::atomic<unsigned long long> g_launches;

__global__ void __launch_bounds__(256) k_fma_stream(float* out, int iters) {
  float a[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) a[u] = (float)(threadIdx.x + u);
  const float b = 0.9999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int u = 0; u < 8; ++u) a[u] = fmaf(a[u], b, c);
  }
  float s = 0.f;
#pragma unroll
  for (int u = 0; u < 8; ++u) s += a[u];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Every warp arms its own mbarrier for `kBytes` of a copy that is never issued, so
// the phase never completes and warp_wait_tile gives up after `polls` polls, as a
// pass kernel's warp would if its TMA tile never landed. Nothing is in flight.
__global__ void k_wait_timeout_test(int polls, unsigned int* status, int* skipped) {
  constexpr uint32_t kBytes = 4096;
  __shared__ __align__(8) uint64_t bars[32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t bar = smem_u32(&bars[warp]);
  if (lane == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_expect_tx(bar, kBytes);
  }
  __syncwarp();
  if (!warp_wait_tile(bar, polls, status)) {
    if (lane == 0) atomicAdd(skipped, 1);
    return;  // the pass kernels' give-up path: the warp does no further work
  }
}
}  // namespace ptyro

extern "C" int ptyro_fp32_fma_probe(float* out, int32_t blocks, int32_t iters, void* stream) {
  if (!out || blocks <= 0 || iters <= 0) return PTYRO_ERR_INVALID;
  ptyro::k_fma_stream<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters);
  ptyro::g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError() == cudaSuccess ? PTYRO_OK : PTYRO_ERR_CUDA;
}

extern "C" int ptyro_test_wait_timeout(int32_t warps, int32_t polls, uint32_t* status, int32_t* skipped_warps,
                                       void* stream) {
  if (!status || !skipped_warps || warps < 1 || warps > 32 || polls < 1 || polls > (1 << 20))
    return PTYRO_ERR_INVALID;
  ptyro::k_wait_timeout_test<<<1, warps * 32, 0, (cudaStream_t)stream>>>(polls, (unsigned int*)status,
                                                                          (int*)skipped_warps);
  ptyro::g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError() == cudaSuccess ? PTYRO_OK : PTYRO_ERR_CUDA;
}
