// Diagnostics: a dense FP32 FMA stream that measures the CUDA-core FP32 ceiling of
// the device it runs on (the denominator of the multislice roofline).
#include <cuda_runtime.h>

#include <atomic>

#include "../../include/ptyro_b200.h"

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
}  // namespace ptyro

extern "C" int ptyro_fp32_fma_probe(float* out, int32_t blocks, int32_t iters, void* stream) {
  if (!out || blocks <= 0 || iters <= 0) return PTYRO_ERR_INVALID;
  ptyro::k_fma_stream<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters);
  ptyro::g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError() == cudaSuccess ? PTYRO_OK : PTYRO_ERR_CUDA;
}
