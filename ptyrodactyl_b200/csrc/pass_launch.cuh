// Launchers of the pass kernel, one translation unit per grid edge (pass_<n>.cu).
// Each returns the cudaError_t of its launch as int (0 = success).
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <mutex>

#include "ms_bwd.cuh"
#include "ms_bwd_lam.cuh"
#include "ms_jvp.cuh"
#include "ms_half.cuh"
#include "ms_pair.cuh"
#include "ms_pipe.cuh"

namespace ptyro {

// Number of engine kernels enqueued by this process (all devices, all threads).
extern std::atomic<unsigned long long> g_launches;

// Per-device one-time setup for state that CUDA keeps per device, such as a kernel's
// dynamic shared memory limit (cudaFuncSetAttribute): once(f) runs f once for every
// device ordinal below kDevices (the current device), and every time for higher
// ordinals. Threads that launch on the same device at once (one per lane) wait for
// the first call to finish, so none launches before the attribute is set.
struct DeviceOnce {
  static constexpr int kDevices = 64;
  std::once_flag flag[kDevices];
  // runs f once per device; callers on that device that arrive meanwhile wait until it
  // has returned (so no thread launches before the attribute is set)
  template <class F>
  void once(F&& f) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevices) {
      f();
      return;
    }
    std::call_once(flag[dev], f);
  }
};

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda), or null.
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The batch's wave slots as a 3-D tensor (x, y, slot) of 8-byte elements with box
// (cols, rows, 1) (rows = N by default), for the TMA column passes. The last few encodings are reused. False
// if the driver offers no encoder or rejects the map (the caller then uses plain loads).
inline bool wave_tensor_map(float2* wave, int n, int slots, int cols, CUtensorMap* out, int rows = 0) {
  if (rows <= 0) rows = n;
  if (rows > 256 || n % rows != 0) return false;  // TMA box dimensions are at most 256
  struct Entry {
    float2* wave;
    int n, slots, cols, rows;
    CUtensorMap map;
  };
  constexpr int kEntries = 8;
  static std::mutex mu;
  static Entry cache[kEntries] = {};
  static int next = 0;
  std::lock_guard<std::mutex> lock(mu);
  for (const Entry& e : cache) {
    if (e.wave == wave && e.n == n && e.slots == slots && e.cols == cols && e.rows == rows && wave != nullptr) {
      *out = e.map;
      return true;
    }
  }
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || (reinterpret_cast<uintptr_t>(wave) & 15) != 0) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)slots};
  const cuuint64_t strides[2] = {(cuuint64_t)n * 8, (cuuint64_t)n * n * 8};
  const cuuint32_t box[3] = {(cuuint32_t)cols, (cuuint32_t)rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUtensorMap m;
  if (enc(&m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, wave, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  cache[next] = {wave, n, slots, cols, rows, m};
  next = (next + 1) % kEntries;
  *out = m;
  return true;
}

template <int N1, int N2, int AXIS, int MINB, bool STEADY>
int launch_pass_s(const PassArgs& a, int grid_y, cudaStream_t st) {
  using Geo = PassGeom<N1, N2>;
  constexpr int N = Geo::N;
  constexpr int W = Geo::kWarps;
  const size_t smem = STEADY ? Geo::smem_bytes_steady(W) : Geo::smem_bytes(W);
  static DeviceOnce attr_done;  // per device: the attribute is per-device state
  attr_done.once([&] {
    cudaFuncSetAttribute(ms_pass_kernel<N1, N2, AXIS, W, MINB, STEADY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  });
  dim3 grid(N / Geo::kLines, grid_y);
  ms_pass_kernel<N1, N2, AXIS, W, MINB, STEADY><<<grid, W * 32, smem, st>>>(a);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

template <int N1, int N2, int AXIS, bool TMA>
int launch_bwd_w(const BwdArgs& a, int grid_y, cudaStream_t st, const CUtensorMap* pmap = nullptr,
                 const CUtensorMap* lmap = nullptr) {
  using Geo = PassGeom<N1, N2>;
  constexpr int N = Geo::N;
  constexpr int W = Geo::kWarps;
  constexpr int MINB = N2 <= 16 ? 2 : 1;  // two resident CTAs where the register budget allows
  const size_t smem = bwd_smem_bytes<N1, N2>(W);
  static DeviceOnce attr_done;  // per device: the attribute is per-device state
  attr_done.once([&] {
    cudaFuncSetAttribute(ms_bwd_pass_kernel<N1, N2, AXIS, W, MINB, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  });
  static const CUtensorMap kNoMap = {};
  dim3 grid(N / Geo::kLines, grid_y);
  ms_bwd_pass_kernel<N1, N2, AXIS, W, MINB, TMA>
      <<<grid, W * 32, smem, st>>>(a, pmap ? *pmap : kNoMap, lmap ? *lmap : kNoMap);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

// The lambda-only adjoint pass (ms_bwd_lam.cuh): two lines per thread, direct access.
template <int N1, int N2, int AXIS, bool TMA>
int launch_bwd_lam_w(const BwdArgs& a, int grid_y, cudaStream_t st, const CUtensorMap* lmap = nullptr) {
  constexpr int N = N1 * N2, G = 32 / N1;
  constexpr int W = N / (2 * G) < 8 ? N / (2 * G) : 8;  // line pairs per CTA tile the grid
  using PG = PairGeom<N1, N2, W>;
  const size_t smem = sizeof(float2) * 2 * (size_t)N + PG::kXbuf;
  static DeviceOnce attr_done;  // per device: the attribute is per-device state
  attr_done.once([&] { cudaFuncSetAttribute(ms_bwd_lam_kernel<N1, N2, AXIS, W, 2, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem); });
  static const CUtensorMap kNoMap = {};
  dim3 grid(N / PG::kLines, grid_y);
  ms_bwd_lam_kernel<N1, N2, AXIS, W, 2, TMA><<<grid, W * 32, smem, st>>>(a, lmap ? *lmap : kNoMap);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

// lambda-only adjoint passes; variant bit 11 (2048): 256^2 column passes move lambda's
// column blocks by TMA (not the initial pass, which reads the amplitudes)
template <int N1, int N2, int AXIS>
int launch_bwd_lam_t(const BwdArgs& a, int grid_y, cudaStream_t st, int variant) {
  if constexpr (AXIS == 1 && N1 * N2 == 256) {
    CUtensorMap lmap;
    if ((variant & 2048) && !a.init && wave_tensor_map(a.lam, N1 * N2, grid_y, 2 * (32 / N1), &lmap))
      return launch_bwd_lam_w<N1, N2, AXIS, true>(a, grid_y, st, &lmap);
  }
  return launch_bwd_lam_w<N1, N2, AXIS, false>(a, grid_y, st);
}

// variant bit 11 (2048): 256^2 adjoint column passes move their column blocks by TMA
template <int N1, int N2, int AXIS>
int launch_bwd_t(const BwdArgs& a, int grid_y, cudaStream_t st, int variant) {
  if constexpr (N2 <= 16) {  // two lines of lambda fit in a thread's registers
    if (a.lam_only) return launch_bwd_lam_t<N1, N2, AXIS>(a, grid_y, st, variant);
  }
  if constexpr (AXIS == 1 && N1 * N2 == 256) {
    CUtensorMap pmap, lmap;
    if ((variant & 2048) && !a.init && wave_tensor_map(a.psi, N1 * N2, grid_y, 32 / N1, &pmap) &&
        wave_tensor_map(a.lam, N1 * N2, grid_y, 32 / N1, &lmap))
      return launch_bwd_w<N1, N2, AXIS, true>(a, grid_y, st, &pmap, &lmap);
  }
  return launch_bwd_w<N1, N2, AXIS, false>(a, grid_y, st);
}

template <int N1, int N2, int AXIS>
int launch_jvp_t(const JvpArgs& a, int grid_y, cudaStream_t st) {
  using Geo = PassGeom<N1, N2>;
  constexpr int N = Geo::N;
  constexpr int W = Geo::kWarps;
  constexpr int MINB = N2 <= 16 ? 2 : 1;
  const size_t smem = bwd_smem_bytes<N1, N2>(W);
  static DeviceOnce attr_done;  // per device: the attribute is per-device state
  attr_done.once([&] {
    cudaFuncSetAttribute(ms_jvp_pass_kernel<N1, N2, AXIS, W, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  });
  dim3 grid(N / Geo::kLines, grid_y);
  ms_jvp_pass_kernel<N1, N2, AXIS, W, MINB><<<grid, W * 32, smem, st>>>(a);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

// Steady passes: persistent, prefetching CTAs; the grid holds exactly the CTAs that
// can be resident at once (line tiles x rows), each walking several slots.
template <int N1, int N2, int AXIS, int MINB>
int launch_pipe_t(const PassArgs& a, int nslots, cudaStream_t st) {
  using Geo = PassGeom<N1, N2>;
  constexpr int W = Geo::kWarps;
  using PG = PipeGeom<N1, N2, AXIS, W>;
  const size_t smem = PG::smem_bytes();
  static int resident_of[DeviceOnce::kDevices] = {};  // CTAs of this kernel per SM x SMs, per device
  int dev = 0;
  cudaGetDevice(&dev);
  int resident = dev >= 0 && dev < DeviceOnce::kDevices ? resident_of[dev] : 0;
  if (!resident) {
    cudaFuncSetAttribute(ms_pass_pipe_kernel<N1, N2, AXIS, W, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ms_pass_pipe_kernel<N1, N2, AXIS, W, MINB>, W * 32,
                                                  smem);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    resident = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
    if (dev >= 0 && dev < DeviceOnce::kDevices) resident_of[dev] = resident;
  }
  const int tiles = Geo::N / Geo::kLines;
  int rows = resident / tiles;
  if (rows < 1) rows = 1;
  if (rows > nslots) rows = nslots;
  dim3 grid(tiles, rows);
  ms_pass_pipe_kernel<N1, N2, AXIS, W, MINB><<<grid, W * 32, smem, st>>>(a, nslots);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

// Steady passes with two lines per thread in paired FP32 arithmetic (ms_pair.cuh).
template <int N1, int N2, int AXIS, int W, int MINB, bool PRE, bool DIRECT = false, bool TMA = false,
          bool GEN = false>
int launch_pair_w(const PassArgs& a, int grid_y, cudaStream_t st, const CUtensorMap* wmap = nullptr) {
  using PG = PairGeom<N1, N2, W, PRE>;
  const size_t smem = PG::smem_bytes();
  static DeviceOnce attr_done;  // per device: the attribute is per-device state
  attr_done.once([&] {
    cudaFuncSetAttribute(ms_pass_pair_kernel<N1, N2, AXIS, W, MINB, PRE, DIRECT, TMA, GEN>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  static const CUtensorMap kNoMap = {};
  dim3 grid(PG::N / PG::kLines, grid_y);
  ms_pass_pair_kernel<N1, N2, AXIS, W, MINB, PRE, DIRECT, TMA, GEN>
      <<<grid, W * 32, smem, st>>>(a, wmap ? *wmap : kNoMap);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}


// variant bit 5 (32): transmission rows prefetched into shared memory, 3 CTAs/SM
// variant bit 6 (64): 8 warps per CTA, 2 CTAs/SM
// variant bit 7 (128): column passes access their column pairs in global memory directly
template <int N1, int N2, int AXIS>
int launch_pair_t(const PassArgs& a, int grid_y, cudaStream_t st, int variant) {
  constexpr int G = 32 / N1;
  constexpr int N = N1 * N2;
  constexpr int W4 = N / (2 * G) < 4 ? N / (2 * G) : 4;
  constexpr int W8 = N / (2 * G) < 8 ? N / (2 * G) : 8;
  const bool pre = (variant & 32) && a.win == nullptr && a.field_n == N;
  if constexpr (AXIS == 1 && N == 256 && W8 == 8) {
    // variant bit 11 (2048, with bits 6 and 7): column blocks moved by TMA
    CUtensorMap wmap;
    if ((variant & 2048) && (variant & 64) && (variant & 128) &&
        wave_tensor_map(a.wave, N, grid_y, 2 * G, &wmap))
      return launch_pair_w<N1, N2, AXIS, W8, 16 / W8, false, true, true>(a, grid_y, st, &wmap);
  }
  if (AXIS == 1 && (variant & 128)) {
    if (variant & 64) return launch_pair_w<N1, N2, AXIS, W8, 16 / W8, false, true>(a, grid_y, st);
    return launch_pair_w<N1, N2, AXIS, W4, 16 / W4, false, true>(a, grid_y, st);
  }
  if (variant & 64) return launch_pair_w<N1, N2, AXIS, W8, 16 / W8, false>(a, grid_y, st);
  if (pre) return launch_pair_w<N1, N2, AXIS, W4, 3, true>(a, grid_y, st);
  return launch_pair_w<N1, N2, AXIS, W4, 16 / W4, false>(a, grid_y, st);
}

// Steady passes with the halves of each line paired (ms_half.cuh), N2 == 2 N1.
template <int N1, int N2, int AXIS, int MINB, bool TMA>
int launch_half_w(const PassArgs& a, int grid_y, cudaStream_t st, const CUtensorMap* wmap = nullptr) {
  using Geo = PassGeom<N1, N2>;
  constexpr int W = Geo::kWarps;
  const size_t smem = Geo::smem_bytes(W);
  static DeviceOnce attr_done;  // per device: the attribute is per-device state
  attr_done.once([&] {
    cudaFuncSetAttribute(ms_pass_half_kernel<N1, N2, AXIS, W, MINB, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  });
  static const CUtensorMap kNoMap = {};
  dim3 grid(Geo::N / Geo::kLines, grid_y);
  ms_pass_half_kernel<N1, N2, AXIS, W, MINB, TMA><<<grid, W * 32, smem, st>>>(a, wmap ? *wmap : kNoMap);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

// variant bit 11 (2048): 512^2 column passes move their column blocks by TMA
template <int N1, int N2, int AXIS, int MINB>
int launch_half_t(const PassArgs& a, int grid_y, cudaStream_t st, int variant) {
  if constexpr (AXIS == 1 && N1 * N2 == 512) {
    CUtensorMap wmap;
    if ((variant & 2048) && wave_tensor_map(a.wave, N1 * N2, grid_y, 32 / N1, &wmap, 256))
      return launch_half_w<N1, N2, AXIS, MINB, true>(a, grid_y, st, &wmap);
  }
  return launch_half_w<N1, N2, AXIS, MINB, false>(a, grid_y, st);
}

// tune bit 8 (value 256): steady passes of N2 == 2 N1 shapes run the half-paired kernel
// (bit 9, value 512: with one CTA per SM and up to 255 registers).
// tune bit 4 (value 16): steady passes run the paired two-lines-per-thread kernel.
// tune bit 2 (value 4) selects the persistent double-buffered kernel for steady
// passes (measured slower than the one-slot-per-CTA kernel on B200 at 128-512^2)
template <int N1, int N2, int AXIS, int MINB>
int launch_pass_t(const PassArgs& a0, int grid_y, cudaStream_t st, int variant) {
  // tune bit 3 (value 8): column passes access global memory directly (no staging tile)
  PassArgs a = a0;
  if (AXIS == 1 && (variant & 8)) a.direct = 1;
  if constexpr (N2 == 2 * N1) {
    if (is_steady_pass(a) && (variant & 256) && a.pf != nullptr)
      return (variant & 512) ? launch_half_t<N1, N2, AXIS, 1>(a, grid_y, st, variant)
                             : launch_half_t<N1, N2, AXIS, 2>(a, grid_y, st, variant);
  }
  if (is_steady_pass(a) && (variant & 16) && a.pf != nullptr)
    return launch_pair_t<N1, N2, AXIS>(a, grid_y, st, variant);
  if constexpr (N1 == N2 && N1 * N2 == 256) {
    // tune bit 12 (4096, with bits 4, 6 and 7): the first and last slice passes run the
    // paired kernel too (column passes with TMA blocks when bit 11 is set)
    if ((variant & 4096) && (variant & 16) && (variant & 64) && (variant & 128) && is_edge_slice_pass(a) &&
        a.pf != nullptr) {
      constexpr int G = 32 / N1;
      if constexpr (AXIS == 1) {
        CUtensorMap wmap;
        if ((variant & 2048) && wave_tensor_map(a.wave, N1 * N2, grid_y, 2 * G, &wmap))
          return launch_pair_w<N1, N2, AXIS, 8, 2, false, true, true, true>(a, grid_y, st, &wmap);
        return launch_pair_w<N1, N2, AXIS, 8, 2, false, true, false, true>(a, grid_y, st);
      } else {
        return launch_pair_w<N1, N2, AXIS, 8, 2, false, false, false, true>(a, grid_y, st);
      }
    }
  }
  if (is_steady_pass(a) && a.tw2 != nullptr && (variant & 4)) return launch_pipe_t<N1, N2, AXIS, MINB>(a, grid_y, st);
  return is_steady_pass(a) ? launch_pass_s<N1, N2, AXIS, MINB, true>(a, grid_y, st)
                           : launch_pass_s<N1, N2, AXIS, MINB, false>(a, grid_y, st);
}

template <int N1, int N2, int AXIS, int MINB>
int launch_pass_multi_t(const PassArgs* descs, const int2* rows, int nrows, cudaStream_t st) {
  using Geo = PassGeom<N1, N2>;
  constexpr int W = Geo::kWarps;
  const size_t smem = Geo::smem_bytes(W);
  static DeviceOnce attr_done;  // per device: the attribute is per-device state
  attr_done.once([&] {
    cudaFuncSetAttribute(ms_pass_multi_kernel<N1, N2, AXIS, W, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  });
  dim3 grid(Geo::N / Geo::kLines, nrows);
  ms_pass_multi_kernel<N1, N2, AXIS, W, MINB><<<grid, W * 32, smem, st>>>(descs, rows);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

// Steady forward passes of several jobs with two lines per thread (N <= 256) or the
// two halves of each line paired (512); returns -1 where no paired kernel serves the
// shape.
template <int N1, int N2, int AXIS>
int launch_pass_pair_multi_t(const PassArgs* descs, const int2* rows, int nrows, cudaStream_t st) {
  if constexpr (N1 * N2 == 512 && N2 == 2 * N1) {  // half-paired lines (ms_half.cuh), 2 CTAs per SM
    using Geo = PassGeom<N1, N2>;
    constexpr int W = Geo::kWarps;
    const size_t smem = Geo::smem_bytes(W);
    static DeviceOnce attr_done;  // per device: the attribute is per-device state
    attr_done.once([&] {
      cudaFuncSetAttribute(ms_pass_half_multi_kernel<N1, N2, AXIS, W, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
    });
    dim3 grid(Geo::N / Geo::kLines, nrows);
    ms_pass_half_multi_kernel<N1, N2, AXIS, W, 2><<<grid, W * 32, smem, st>>>(descs, rows);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return (int)cudaGetLastError();
  } else if constexpr (N1 * N2 > 256) {
    return -1;
  } else {
    constexpr int G = 32 / N1;
    constexpr int N = N1 * N2;
    constexpr int W = N == 256 ? 8 : (N / (2 * G) < 4 ? N / (2 * G) : 4);
    constexpr int MINB = 16 / W;
    using PG = PairGeom<N1, N2, W, false>;
    const size_t smem = PG::smem_bytes();
    static DeviceOnce attr_done;  // per device: the attribute is per-device state
    attr_done.once([&] {
      cudaFuncSetAttribute(ms_pass_pair_multi_kernel<N1, N2, AXIS, W, MINB>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    dim3 grid(N / PG::kLines, nrows);
    ms_pass_pair_multi_kernel<N1, N2, AXIS, W, MINB><<<grid, W * 32, smem, st>>>(descs, rows);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return (int)cudaGetLastError();
  }
}

template <int N1, int N2, int AXIS>
int launch_bwd_multi_t(const BwdArgs* descs, const int2* rows, int nrows, cudaStream_t st) {
  using Geo = PassGeom<N1, N2>;
  constexpr int W = Geo::kWarps;
  constexpr int MINB = N2 <= 16 ? 2 : 1;
  const size_t smem = bwd_smem_bytes<N1, N2>(W);
  static DeviceOnce attr_done;  // per device: the attribute is per-device state
  attr_done.once([&] {
    cudaFuncSetAttribute(ms_bwd_multi_kernel<N1, N2, AXIS, W, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  });
  dim3 grid(Geo::N / Geo::kLines, nrows);
  ms_bwd_multi_kernel<N1, N2, AXIS, W, MINB><<<grid, W * 32, smem, st>>>(descs, rows);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

// variant bit (1 << axis) selects the 3-CTAs-per-SM register budget where the
// shape allows it (N2 <= 16); otherwise 2 (N2 <= 16) or 1 (N2 = 32) CTAs per SM.
#define PTYRO_DEFINE_PASS_LAUNCHER(NN, N1, N2)                                                   \
  int launch_pass_##NN(int axis, const PassArgs& a, int grid_y, cudaStream_t st, int variant) {  \
    constexpr int lo = (N2) <= 16 ? 2 : 1, hi = (N2) <= 16 ? 3 : 1;                              \
    const bool occ = (variant >> axis) & 1;                                                      \
    if (axis == 0)                                                                               \
      return occ ? launch_pass_t<N1, N2, 0, hi>(a, grid_y, st, variant)                          \
                 : launch_pass_t<N1, N2, 0, lo>(a, grid_y, st, variant);                         \
    return occ ? launch_pass_t<N1, N2, 1, hi>(a, grid_y, st, variant)                            \
               : launch_pass_t<N1, N2, 1, lo>(a, grid_y, st, variant);                           \
  }                                                                                              \
  /* TMA completion waits of this unit's passes that hit their poll limit (current device) */ \
  unsigned int pair_wait_timeouts_##NN() {                                                      \
    unsigned int v = 0;                                                                          \
    if (cudaMemcpyFromSymbol(&v, g_pair_wait_timeouts, sizeof v) != cudaSuccess) return 0xffffffffu; \
    return v;                                                                                    \
  }                                                                                              \
  int launch_bwd_##NN(int axis, const BwdArgs& a, int grid_y, cudaStream_t st, int variant) {   \
    return axis == 0 ? launch_bwd_t<N1, N2, 0>(a, grid_y, st, variant)                          \
                     : launch_bwd_t<N1, N2, 1>(a, grid_y, st, variant);                         \
  }                                                                                              \
  int launch_jvp_##NN(int axis, const JvpArgs& a, int grid_y, cudaStream_t st) {                \
    return axis == 0 ? launch_jvp_t<N1, N2, 0>(a, grid_y, st) : launch_jvp_t<N1, N2, 1>(a, grid_y, st); \
  }                                                                                              \
  int launch_pass_multi_##NN(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st,  \
                             int variant) {                                                      \
    constexpr int lo = (N2) <= 16 ? 2 : 1, hi = (N2) <= 16 ? 3 : 1;                              \
    const bool occ = (variant >> axis) & 1;                                                      \
    if (axis == 0)                                                                               \
      return occ ? launch_pass_multi_t<N1, N2, 0, hi>(d, r, nr, st) : launch_pass_multi_t<N1, N2, 0, lo>(d, r, nr, st); \
    return occ ? launch_pass_multi_t<N1, N2, 1, hi>(d, r, nr, st) : launch_pass_multi_t<N1, N2, 1, lo>(d, r, nr, st);   \
  }                                                                                              \
  int launch_pass_pair_multi_##NN(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st) { \
    return axis == 0 ? launch_pass_pair_multi_t<N1, N2, 0>(d, r, nr, st)                         \
                     : launch_pass_pair_multi_t<N1, N2, 1>(d, r, nr, st);                        \
  }                                                                                              \
  int launch_bwd_multi_##NN(int axis, const BwdArgs* d, const int2* r, int nr, cudaStream_t st) {  \
    return axis == 0 ? launch_bwd_multi_t<N1, N2, 0>(d, r, nr, st) : launch_bwd_multi_t<N1, N2, 1>(d, r, nr, st); \
  }

int launch_pass_multi_16(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st, int variant);
int launch_bwd_multi_16(int axis, const BwdArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_pair_multi_16(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_multi_32(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st, int variant);
int launch_bwd_multi_32(int axis, const BwdArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_pair_multi_32(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_multi_64(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st, int variant);
int launch_bwd_multi_64(int axis, const BwdArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_pair_multi_64(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_multi_128(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st, int variant);
int launch_bwd_multi_128(int axis, const BwdArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_pair_multi_128(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_multi_256(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st, int variant);
int launch_bwd_multi_256(int axis, const BwdArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_pair_multi_256(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_multi_512(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st, int variant);
int launch_bwd_multi_512(int axis, const BwdArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_pair_multi_512(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_multi_1024(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st, int variant);
int launch_bwd_multi_1024(int axis, const BwdArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_pass_pair_multi_1024(int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st);
int launch_jvp_16(int axis, const JvpArgs& a, int grid_y, cudaStream_t st);
int launch_jvp_32(int axis, const JvpArgs& a, int grid_y, cudaStream_t st);
int launch_jvp_64(int axis, const JvpArgs& a, int grid_y, cudaStream_t st);
int launch_jvp_128(int axis, const JvpArgs& a, int grid_y, cudaStream_t st);
int launch_jvp_256(int axis, const JvpArgs& a, int grid_y, cudaStream_t st);
int launch_jvp_512(int axis, const JvpArgs& a, int grid_y, cudaStream_t st);
int launch_jvp_1024(int axis, const JvpArgs& a, int grid_y, cudaStream_t st);
int launch_bwd_16(int axis, const BwdArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_bwd_32(int axis, const BwdArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_bwd_64(int axis, const BwdArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_bwd_128(int axis, const BwdArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_bwd_256(int axis, const BwdArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_bwd_512(int axis, const BwdArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_bwd_1024(int axis, const BwdArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_pass_16(int axis, const PassArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_pass_32(int axis, const PassArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_pass_64(int axis, const PassArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_pass_128(int axis, const PassArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_pass_256(int axis, const PassArgs& a, int grid_y, cudaStream_t st, int variant);
unsigned int pair_wait_timeouts_16();
unsigned int pair_wait_timeouts_32();
unsigned int pair_wait_timeouts_64();
unsigned int pair_wait_timeouts_128();
unsigned int pair_wait_timeouts_256();
unsigned int pair_wait_timeouts_512();
unsigned int pair_wait_timeouts_1024();
int launch_pass_512(int axis, const PassArgs& a, int grid_y, cudaStream_t st, int variant);
int launch_pass_1024(int axis, const PassArgs& a, int grid_y, cudaStream_t st, int variant);

}  // namespace ptyro
