// One "pass" of the batched multislice engine: every line (row or column) of every
// wave slot in a batch is loaded once from HBM/L2, pushed through a short program
// of 1-D transforms and elementwise factors in registers, and stored once.
//
// Because the Fresnel propagator is separable, P(q) = Py(qy) Px(qx), the 2-D step
// ifft2(P fft2(.)) equals a 1-D convolution along y followed by one along x, and
// the two commute. A pass along one axis can therefore finish slice s-1's
// convolution along that axis, apply T_s, and start slice s's convolution along the
// same axis, touching the wave in memory once per slice:
//   pass k (k >= 1):  [axis part of op_{k-1}]  x T_{k-1}  [axis part of op_k]
// with op_0 = IFFT2 of the shifted probe spectrum, op_j = Conv_{j-1}, op_S = FFT2.
#pragma once
#include "fft_core.cuh"

namespace ptyro {

enum SrcKind : int { SRC_WAVE = 0, SRC_PROBE = 1 };
enum OpKind : int { OP_NONE = 0, OP_FFT = 1, OP_IFFT = 2, OP_CONV = 3, OP_CONV_CONJ = 4 };
enum DstKind : int { DST_WAVE = 0, DST_PATTERN = 1 };

struct PassArgs {
  float2* wave;            // wave slots, slot w occupies wave[w*N*N, (w+1)*N*N), row-major [y][x]
  const float2* probe_k;   // (M, N, N) spectrum of the beam modes (SRC_PROBE)
  const float2* ramp_y;    // (B, N) shift ramp along y per probe of the batch (SRC_PROBE)
  const float2* ramp_x;    // (B, N) shift ramp along x
  const float2* trans;     // (S, N, N) transmission exp(i sigma V), row-major
  const float2* pf;        // (N) 1-D propagator factor along this axis, already divided by N
  const float2* tw;        // (N) forward twiddles exp(-2 pi i j / N)
  float* pattern;          // (B, N, N) fftshifted intensity (DST_PATTERN)
  const float* weights;    // (M) incoherent mode weights (DST_PATTERN)
  int n_modes;
  int src, op1, t_slice, op2, dst;
  int t_conj;              // multiply by conj(T) instead of T
  float scale;             // factor applied after op1 == OP_IFFT
};

template <int N1, int N2>
struct PassGeom {
  static constexpr int N = N1 * N2;
  static constexpr int G = 32 / N1;  // lines per warp
  static_assert(N2 % N1 == 0, "N2 must be a multiple of N1");
  static_assert(32 % N1 == 0, "N1 must divide the warp");
  static size_t smem_bytes(int warps) {
    return sizeof(float2) * ((size_t)N + (size_t)warps * G * LineBuf<N1, N2>::kSize);
  }
};

// op on registers in natural distribution; returns true if the result is k-order.
template <int N1, int N2>
__device__ __forceinline__ bool apply_op(int op, float2 (&v)[N2], int t, float2* buf, const float2* tw,
                                         const float2* __restrict__ pf, float scale) {
  if (op == OP_FFT) {
    line_nat_to_k<N1, N2, -1>(v, t, buf, tw);
    return true;
  }
  if (op == OP_CONV || op == OP_CONV_CONJ) {
    line_nat_to_k<N1, N2, -1>(v, t, buf, tw);
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const float2 p = __ldg(pf + korder_index<N1, N2>(t, r));
      v[r] = op == OP_CONV ? cmul(v[r], p) : cmulc(v[r], p);
    }
    line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
    return false;
  }
  return false;
}

template <int N1, int N2, int AXIS, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) ms_pass_kernel(PassArgs a) {
  using Geo = PassGeom<N1, N2>;
  using LB = LineBuf<N1, N2>;
  constexpr int N = Geo::N;
  constexpr int G = Geo::G;
  extern __shared__ float2 smem[];
  float2* tw = smem;
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = a.tw[i];
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Row passes put consecutive lanes along x inside a line; column passes put them
  // across neighbouring columns, so both load full 32-byte sectors.
  const int t = AXIS == 0 ? (lane % N1) : (lane / G);
  const int gl = AXIS == 0 ? (lane / N1) : (lane % G);
  const int warps = blockDim.x >> 5;
  const int line = blockIdx.x * (warps * G) + warp * G + gl;
  if (blockIdx.x * (warps * G) + warp * G >= N) return;  // whole warp idle (N < lines per CTA)
  float2* buf = smem + N + (warp * G + gl) * LB::kSize;
  const size_t NN = (size_t)N * N;
  auto off = [&](int e) -> size_t { return AXIS == 0 ? (size_t)line * N + e : (size_t)e * N + line; };

  const bool to_pattern = a.dst == DST_PATTERN;
  const int mcount = to_pattern ? a.n_modes : 1;
  float acc[N2];
#pragma unroll
  for (int r = 0; r < N2; ++r) acc[r] = 0.f;

  for (int m = 0; m < mcount; ++m) {
    const int slot = to_pattern ? blockIdx.y * a.n_modes + m : blockIdx.y;
    float2* w = a.wave + (size_t)slot * NN;
    float2 v[N2];
    bool korder;
    // ---- load
    if (a.src == SRC_PROBE) {
      const int b = blockIdx.y / a.n_modes;
      const int mode = blockIdx.y % a.n_modes;
      const float2* pk = a.probe_k + (size_t)mode * NN;
      const float2 rl = AXIS == 0 ? a.ramp_y[(size_t)b * N + line] : a.ramp_x[(size_t)b * N + line];
      const float2* ra = (AXIS == 0 ? a.ramp_x : a.ramp_y) + (size_t)b * N;
#pragma unroll
      for (int r = 0; r < N2; ++r) {
        const int k = korder_index<N1, N2>(t, r);
        v[r] = cmul(cmul(pk[off(k)], ra[k]), rl);
      }
      korder = true;
    } else if (a.op1 == OP_IFFT) {
#pragma unroll
      for (int r = 0; r < N2; ++r) v[r] = w[off(korder_index<N1, N2>(t, r))];
      korder = true;
    } else {
#pragma unroll
      for (int j = 0; j < N2; ++j) v[j] = w[off(t + N1 * j)];
      korder = false;
    }
    // ---- op1
    if (a.op1 == OP_IFFT) {
      line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
#pragma unroll
      for (int j = 0; j < N2; ++j) v[j] = cscale(v[j], a.scale);
      korder = false;
    } else if (a.op1 != OP_NONE) {
      korder = apply_op<N1, N2>(a.op1, v, t, buf, tw, a.pf, a.scale);
    }
    // ---- transmission
    if (a.t_slice >= 0) {
      const float2* T = a.trans + (size_t)a.t_slice * NN;
#pragma unroll
      for (int j = 0; j < N2; ++j) {
        const float2 tv = __ldg(T + off(t + N1 * j));
        v[j] = a.t_conj ? cmulc(v[j], tv) : cmul(v[j], tv);
      }
    }
    // ---- op2
    if (a.op2 != OP_NONE) korder = apply_op<N1, N2>(a.op2, v, t, buf, tw, a.pf, a.scale);
    // ---- store
    if (to_pattern) {
      const float wm = a.weights[m];
#pragma unroll
      for (int r = 0; r < N2; ++r) acc[r] = fmaf(wm, fmaf(v[r].x, v[r].x, v[r].y * v[r].y), acc[r]);
    } else if (korder) {
#pragma unroll
      for (int r = 0; r < N2; ++r) w[off(korder_index<N1, N2>(t, r))] = v[r];
    } else {
#pragma unroll
      for (int j = 0; j < N2; ++j) w[off(t + N1 * j)] = v[j];
    }
  }
  if (to_pattern) {
    // fftshift on store: frequency index k lands at (k + N/2) mod N on both axes.
    float* out = a.pattern + (size_t)blockIdx.y * NN;
    const int ls = (line + N / 2) % N;
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const int ks = (korder_index<N1, N2>(t, r) + N / 2) % N;
      const size_t o = AXIS == 0 ? (size_t)ls * N + ks : (size_t)ks * N + ls;
      out[o] = acc[r];
    }
  }
}

}  // namespace ptyro
