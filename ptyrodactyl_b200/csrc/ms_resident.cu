// The wave-resident multislice forward (see ms_resident.cuh).
#include "ms_resident.cuh"

#include "pass_launch.cuh"

namespace ptyro {

template <int N1, int N2, int WARPS>
struct ResGeom {
  static constexpr int N = N1 * N2;
  static constexpr int G = 32 / N1;         // line pairs per warp
  static constexpr int kPairs = WARPS * G;  // line pairs per iteration of a pass
  static_assert((N / 2) % kPairs == 0, "the CTA's line pairs must tile the grid");
  static constexpr int kIters = (N / 2) / kPairs;
  // Row pitch of the resident wave, in float2: N + 4 (== 4 mod 8). Row passes: the line
  // pairs (2p, 2p + 1) of a warp start 2 * pitch * 8 == 64 bytes apart modulo the
  // 128-byte bank window, so each 8-byte load of a warp (4 pairs x 8 lanes) takes the
  // minimum two wavefronts. Column passes: consecutive rows sit 32 bytes apart modulo
  // 128, so the 16-byte column-pair reads of a warp (8 rows x 64 bytes) cover every
  // bank exactly four times, the minimum four wavefronts.
  static constexpr int kPitch = N + 4;
  static constexpr size_t kWave = sizeof(float2) * (size_t)N * kPitch;
  static constexpr size_t kTables = sizeof(float2) * 2 * (size_t)N;  // twiddles, propagator factor
  static constexpr size_t kXbuf = sizeof(Pair) * (size_t)kPairs * PairBuf<N1, N2>::kSize;
  static constexpr size_t kSmem = kWave + kTables + kXbuf;
};

// One pass of pass index k over the CTA's wave W (rows for AXIS 0, columns for AXIS 1).
template <int N1, int N2, int WARPS, int AXIS>
__device__ __forceinline__ void resident_pass(const ResidentArgs& a, const int b, const int k, float2* W,
                                              const float2* tw, const float2* pfs, Pair* xbuf) {
  using RG = ResGeom<N1, N2, WARPS>;
  constexpr int N = RG::N, G = RG::G, P = RG::kPitch;
  const int S = a.num_slices;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = AXIS == 0 ? (lane % N1) : (lane / G);
  const int gl = AXIS == 0 ? (lane / N1) : (lane % G);
  Pair* buf = xbuf + (warp * G + gl) * PairBuf<N1, N2>::kSize;
  // the pass engine's program of pass k
  const int op1 = k <= 1 ? (int)OP_IFFT : (k <= S ? (int)OP_CONV : (int)OP_FFT);
  const int op2 = (k == 0 || k == S + 1) ? (int)OP_NONE : (k == S ? (int)OP_FFT : (int)OP_CONV);
  const size_t NN = (size_t)N * N;

#pragma unroll 1
  for (int it = 0; it < RG::kIters; ++it) {
    const int la = 2 * (it * RG::kPairs + warp * G + gl), lb = la + 1;
    Pair v[N2];
    // ---- load: the shifted probe spectrum (k = 0), the wave in k-order along this
    // axis (k = 1: the y part of the probe's inverse transform), or natural order
    if (k == 0) {  // rows (AXIS 0): k-order along x
      const float2* ra = a.ramp_x + (size_t)b * N;
      const float2 rla = a.ramp_y[(size_t)b * N + la], rlb = a.ramp_y[(size_t)b * N + lb];
#pragma unroll
      for (int r = 0; r < N2; ++r) {
        const int kk = korder_index<N1, N2>(t, r);
        v[r] = make_pair(cmul(cmul(a.probe_k[(size_t)la * N + kk], ra[kk]), rla),
                         cmul(cmul(a.probe_k[(size_t)lb * N + kk], ra[kk]), rlb));
      }
    } else {
#pragma unroll
      for (int r = 0; r < N2; ++r) {
        const int e = k == 1 ? korder_index<N1, N2>(t, r) : t + N1 * r;
        if (AXIS == 0) {
          v[r] = make_pair(W[la * P + e], W[lb * P + e]);
        } else {
          const float4 q = *reinterpret_cast<const float4*>(W + e * P + la);
          v[r] = {make_float2(q.x, q.z), make_float2(q.y, q.w)};
        }
      }
    }
    // ---- op1
    bool korder;
    if (op1 == OP_IFFT) {
      line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
#pragma unroll
      for (int j = 0; j < N2; ++j) v[j] = cscale(v[j], a.scale);
      korder = false;
    } else if (op1 == OP_CONV) {
      line_nat_to_k<N1, N2, -1>(v, t, buf, tw);
#pragma unroll
      for (int r = 0; r < N2; ++r) v[r] = cmul(v[r], pfs[korder_index<N1, N2>(t, r)]);
      line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
      korder = false;
    } else {  // OP_FFT: the pattern pass
      line_nat_to_k<N1, N2, -1>(v, t, buf, tw);
      korder = true;
    }
    if (k == S + 1) {  // ---- w |A|^2, fftshifted (frequency k lands at (k + N/2) mod N)
      float* out = a.pattern + (size_t)b * NN;
      const float wm = a.weights[0];
      const int lsa = (la + N / 2) % N, lsb = (lb + N / 2) % N;
#pragma unroll
      for (int r = 0; r < N2; ++r) {
        const int ks = (korder_index<N1, N2>(t, r) + N / 2) % N;
        const float2 va = pair_a(v[r]), vb = pair_b(v[r]);
        const float ia = fmaf(wm, fmaf(va.x, va.x, va.y * va.y), 0.f);
        const float ib = fmaf(wm, fmaf(vb.x, vb.x, vb.y * vb.y), 0.f);
        const size_t oa = AXIS == 0 ? (size_t)lsa * N + ks : (size_t)ks * N + lsa;
        const size_t ob = AXIS == 0 ? (size_t)lsb * N + ks : (size_t)ks * N + lsb;
        out[oa] = a.accumulate ? out[oa] + ia : ia;
        out[ob] = a.accumulate ? out[ob] + ib : ib;
      }
      continue;
    }
    // ---- transmission T_{k-1}: row-major rows for row passes, the transposed table for columns
    if (k >= 1) {
      const float2* T = (AXIS == 0 ? a.trans : a.trans_t) + (size_t)(k - 1) * NN;
      const float2* Ta = T + (size_t)la * N;
      const float2* Tb = T + (size_t)lb * N;
#pragma unroll
      for (int j = 0; j < N2; ++j) v[j] = cmul(v[j], __ldg(Ta + t + N1 * j), __ldg(Tb + t + N1 * j));
    }
    // ---- op2
    if (op2 == OP_CONV) {
      line_nat_to_k<N1, N2, -1>(v, t, buf, tw);
#pragma unroll
      for (int r = 0; r < N2; ++r) v[r] = cmul(v[r], pfs[korder_index<N1, N2>(t, r)]);
      line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
    } else if (op2 == OP_FFT) {
      line_nat_to_k<N1, N2, -1>(v, t, buf, tw);
      korder = true;
    }
    // ---- store back into the resident wave
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const int e = korder ? korder_index<N1, N2>(t, r) : t + N1 * r;
      if (AXIS == 0) {
        W[la * P + e] = pair_a(v[r]);
        W[lb * P + e] = pair_b(v[r]);
      } else {
        *reinterpret_cast<float4*>(W + e * P + la) = make_float4(v[r].re.x, v[r].im.x, v[r].re.y, v[r].im.y);
      }
    }
  }
}

template <int N1, int N2, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 1) ms_resident_kernel(ResidentArgs a) {
  using RG = ResGeom<N1, N2, WARPS>;
  constexpr int N = RG::N;
  extern __shared__ float4 smem4[];
  float2* W = reinterpret_cast<float2*>(smem4);
  float2* tw = W + (size_t)N * RG::kPitch;  // tw[k2 * N1 + t] = W_N^{t k2}
  float2* pfs = tw + N;
  Pair* xbuf = reinterpret_cast<Pair*>(pfs + N);
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int k2 = i / N1, tt = i % N1;
    tw[i] = a.tw[(tt * k2) % N];
    pfs[i] = a.pf[i];
  }
  __syncthreads();
  const int b = blockIdx.x;
#pragma unroll 1
  for (int k = 0; k <= a.num_slices + 1; ++k) {
    if ((k & 1) == 0)
      resident_pass<N1, N2, WARPS, 0>(a, b, k, W, tw, pfs, xbuf);
    else
      resident_pass<N1, N2, WARPS, 1>(a, b, k, W, tw, pfs, xbuf);
    __syncthreads();  // the next pass reads the other axis' lines
  }
}

template <int N1, int N2, int WARPS>
static int launch_resident_t(const ResidentArgs& a, int nb, cudaStream_t st) {
  using RG = ResGeom<N1, N2, WARPS>;
  static DeviceOnce attr_done;  // per device: the attribute is per-device state
  attr_done.once([&] { cudaFuncSetAttribute(ms_resident_kernel<N1, N2, WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)RG::kSmem); });
  ms_resident_kernel<N1, N2, WARPS><<<nb, WARPS * 32, RG::kSmem, st>>>(a);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

int launch_resident(int n, const ResidentArgs& a, int nb, cudaStream_t st) {
  if (nb <= 0) return 0;
  switch (n) {
    case 16: return launch_resident_t<4, 4, 1>(a, nb, st);
    case 32: return launch_resident_t<4, 8, 2>(a, nb, st);
    case 64: return launch_resident_t<8, 8, 8>(a, nb, st);
    case 128: return launch_resident_t<8, 16, 8>(a, nb, st);
    default: return (int)cudaErrorInvalidValue;
  }
}

size_t resident_smem_bytes(int n) {
  switch (n) {
    case 16: return ResGeom<4, 4, 1>::kSmem;
    case 32: return ResGeom<4, 8, 2>::kSmem;
    case 64: return ResGeom<8, 8, 8>::kSmem;
    case 128: return ResGeom<8, 16, 8>::kSmem;
    default: return 0;
  }
}

}  // namespace ptyro
