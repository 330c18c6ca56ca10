// Tangent (forward-mode) pass of the multislice engine: the Jacobian-vector
// product J v of the 4D-STEM forward model for a tangent v = (dV, dmodes).
//
// Forward, per probe and mode: phi_s = T_s psi_s, psi_{s+1} = U phi_s with
// U = ifft2 diag(P) fft2, A = fft2(phi_{S-1}), I = sum_m w_m |A_m|^2. Linearised
// (T_s = exp(i sigma V_s), so dT_s = i sigma dV_s T_s):
//   dpsi_0   = shift(dmodes)
//   dphi_s   = T_s (dpsi_s + i sigma dV_s psi_s)
//   dpsi_s+1 = U dphi_s
//   dI       = sum_m w_m 2 Re(conj(A_m) dA_m)
// The tangent obeys the same operator as the wave, so one pass carries both waves
// of a line through the forward's schedule in lockstep (the same passes, the same
// transforms) and couples them only at the slice point.
#pragma once
#include "ms_bwd.cuh"

namespace ptyro {

struct JvpArgs {
  float2* psi;             // wave slots (B*M planes)
  float2* dpsi;            // tangent slots
  const float2* probe_k;   // (M, N, N) spectra of the modes (SRC_PROBE)
  const float2* dprobe_k;  // (M, N, N) spectra of the tangent modes, or null (zero tangent)
  const float2* ramp_y;    // (B, N) shift ramps
  const float2* ramp_x;
  const float2* trans;     // (S, F, F) T, row-major
  const float2* trans_t;   // transposed
  const float* sdv;        // (S, F, F) sigma * dV, row-major, or null (zero tangent)
  const float* sdv_t;      // transposed
  const int* win;          // (B, 2) window origins, or null
  int field_n;
  const float2* pf;        // (N) propagator factor / N
  const float2* tw;        // (N) forward twiddles
  float* pattern;          // (B, N, N) fftshifted intensities, or null
  float* dpattern;         // (B, N, N) fftshifted tangent intensities
  const float* weights;    // (M)
  int n_modes;
  int src, op1, t_slice, op2, dst;
  float scale;             // factor applied after op1 == OP_IFFT
};

// Row of `line` in a periodic F x F field plane (row-major for rows, transposed
// table for columns); element e of the line sits at (e + *off) & (F - 1).
template <int AXIS, typename T>
__device__ __forceinline__ const T* field_row(const T* rowmaj, const T* colmaj, int field_n, int t_slice,
                                              const int* win, int b, int line, int* off) {
  int wy = 0, wx = 0;
  if (win) {
    wy = win[2 * b];
    wx = win[2 * b + 1];
  }
  *off = AXIS == 0 ? wx : wy;
  const T* P = (AXIS == 0 ? rowmaj : colmaj) + (size_t)t_slice * field_n * field_n;
  return P + (size_t)((line + (AXIS == 0 ? wy : wx)) & (field_n - 1)) * field_n;
}

template <int N1, int N2, typename T>
__device__ __forceinline__ bool jvp_op(int op, T (&v)[N2], int t, T* buf, const float2* tw, const float2* pf,
                                       float scale) {
  if (op == OP_IFFT) {
    line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
#pragma unroll
    for (int j = 0; j < N2; ++j) v[j] = cscale(v[j], scale);
    return false;
  }
  return apply_op<N1, N2>(op, v, t, buf, tw, pf);
}

template <int N1, int N2, int AXIS, int WARPS>
__device__ __forceinline__ void jvp_body(const JvpArgs& a, const int yslot) {
  using Geo = PassGeom<N1, N2>;
  constexpr int N = Geo::N;
  constexpr int G = Geo::G;
  constexpr int lines = WARPS * G;
  static_assert(N % lines == 0, "lines per CTA must divide N");
  constexpr int pitch = lines + G;
  constexpr int kTileIters = N * lines / (WARPS * 32);
  extern __shared__ float2 smem[];
  float2* tw = smem;
  float2* work = smem + N;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int k2 = i / N1, tt = i % N1;
    tw[i] = a.tw[(tt * k2) % N];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = AXIS == 0 ? (lane % N1) : (lane / G);
  const int gl = AXIS == 0 ? (lane / N1) : (lane % G);
  const int lc = warp * G + gl;
  const int line0 = blockIdx.x * lines;
  const int line = line0 + lc;
  // the wave and its tangent ride as one Pair per element (half 0, half 1)
  Pair* buf = reinterpret_cast<Pair*>(work) + lc * PairBuf<N1, N2>::kSize;
  const size_t NN = (size_t)N * N;
  auto off = [&](int e) -> size_t { return AXIS == 0 ? (size_t)line * N + e : (size_t)e * N + line; };
  const bool to_pattern = a.dst == DST_PATTERN;
  const int mcount = to_pattern ? a.n_modes : 1;
  float acc[N2], dacc[N2];
#pragma unroll
  for (int r = 0; r < N2; ++r) acc[r] = dacc[r] = 0.f;

  for (int m = 0; m < mcount; ++m) {
    const int slot = to_pattern ? yslot * a.n_modes + m : yslot;
    const int b = slot / a.n_modes;
    float2* Wp = a.psi + (size_t)slot * NN;
    float2* Wd = a.dpsi + (size_t)slot * NN;
    Pair q[N2];
    const bool korder_in = a.src == SRC_PROBE || a.op1 == OP_IFFT;
    // ---- load both waves
    if (a.src == SRC_PROBE) {
      const int mode = slot % a.n_modes;
      const float2* pk = a.probe_k + (size_t)mode * NN;
      const float2* dk = a.dprobe_k ? a.dprobe_k + (size_t)mode * NN : nullptr;
      const float2 rl = AXIS == 0 ? a.ramp_y[(size_t)b * N + line] : a.ramp_x[(size_t)b * N + line];
      const float2* ra = (AXIS == 0 ? a.ramp_x : a.ramp_y) + (size_t)b * N;
#pragma unroll
      for (int r = 0; r < N2; ++r) {
        const int k = korder_index<N1, N2>(t, r);
        const float2 f = cmul(ra[k], rl);
        q[r] = make_pair(cmul(pk[off(k)], f), dk ? cmul(dk[off(k)], f) : make_float2(0.f, 0.f));
      }
    } else if (AXIS == 0) {
      bwd_load_half<N1, N2, AXIS, 0>(Wp, q, korder_in, t, line, lc, work, pitch);
      bwd_load_half<N1, N2, AXIS, 1>(Wd, q, korder_in, t, line, lc, work, pitch);
    } else {
      __syncthreads();
      tile_load<N, lines, pitch, WARPS * 32>(Wp, work, line0);
      __syncthreads();
      bwd_load_half<N1, N2, AXIS, 0>(Wp, q, korder_in, t, line, lc, work, pitch);
      __syncthreads();
      tile_load<N, lines, pitch, WARPS * 32>(Wd, work, line0);
      __syncthreads();
      bwd_load_half<N1, N2, AXIS, 1>(Wd, q, korder_in, t, line, lc, work, pitch);
      __syncthreads();
    }
    bool korder = korder_in;
    // ---- op1 on both
    if (a.op1 != OP_NONE) korder = jvp_op<N1, N2>(a.op1, q, t, buf, tw, a.pf, a.scale);
    // ---- slice point: dphi = T (dpsi + i sigma dV psi), phi = T psi
    if (a.t_slice >= 0) {
      int eoff;
      const float2* T = field_row<AXIS>(a.trans, a.trans_t, a.field_n, a.t_slice, a.win, b, line, &eoff);
      const int fm = a.field_n - 1;
      if (a.sdv) {
        int doff;
        const float* D = field_row<AXIS>(a.sdv, a.sdv_t, a.field_n, a.t_slice, a.win, b, line, &doff);
#pragma unroll
        for (int j = 0; j < N2; ++j) {
          const float e = __ldg(D + ((t + N1 * j + doff) & fm));
          q[j].re.y = fmaf(-e, q[j].im.x, q[j].re.y);
          q[j].im.y = fmaf(e, q[j].re.x, q[j].im.y);
        }
      }
#pragma unroll
      for (int j = 0; j < N2; ++j) q[j] = cmul(q[j], __ldg(T + ((t + N1 * j + eoff) & fm)));
    }
    // ---- op2 on both
    if (a.op2 != OP_NONE) korder = jvp_op<N1, N2>(a.op2, q, t, buf, tw, a.pf, a.scale);
    // ---- store
    if (to_pattern) {
      const float wm = a.weights[m];
#pragma unroll
      for (int r = 0; r < N2; ++r) {
        const float2 v = pair_a(q[r]), u = pair_b(q[r]);
        acc[r] = fmaf(wm, fmaf(v.x, v.x, v.y * v.y), acc[r]);
        dacc[r] = fmaf(2.f * wm, fmaf(v.x, u.x, v.y * u.y), dacc[r]);
      }
    } else if (AXIS == 0) {
#pragma unroll
      for (int r = 0; r < N2; ++r) {
        const size_t o = off(korder ? korder_index<N1, N2>(t, r) : t + N1 * r);
        Wp[o] = pair_a(q[r]);
        Wd[o] = pair_b(q[r]);
      }
    } else {
      for (int wv = 0; wv < 2; ++wv) {
        __syncthreads();
#pragma unroll
        for (int r = 0; r < N2; ++r)
          work[(korder ? korder_index<N1, N2>(t, r) : t + N1 * r) * pitch + lc] = wv == 0 ? pair_a(q[r]) : pair_b(q[r]);
        __syncthreads();
        tile_store<N, lines, pitch, WARPS * 32>(wv == 0 ? Wp : Wd, work, line0);
      }
    }
  }
  if (to_pattern) {
    // fftshift on store: frequency index k lands at (k + N/2) mod N on both axes.
    for (int o2 = 0; o2 < 2; ++o2) {
      float* out = (o2 == 0 ? a.pattern : a.dpattern);
      if (!out) continue;
      out += (size_t)yslot * NN;
      if (AXIS == 0) {
        const int ls = (line + N / 2) % N;
#pragma unroll
        for (int r = 0; r < N2; ++r) {
          const int ks = (korder_index<N1, N2>(t, r) + N / 2) % N;
          out[(size_t)ls * N + ks] = o2 == 0 ? acc[r] : dacc[r];
        }
      } else {
        float* tile = reinterpret_cast<float*>(work);
        __syncthreads();
#pragma unroll
        for (int r = 0; r < N2; ++r) tile[korder_index<N1, N2>(t, r) * pitch + lc] = o2 == 0 ? acc[r] : dacc[r];
        __syncthreads();
#pragma unroll 8
        for (int it = 0; it < kTileIters; ++it) {
          const int i = threadIdx.x + it * WARPS * 32;
          const int rr = i / lines, c = i % lines;
          out[(size_t)((rr + N / 2) % N) * N + (line0 + c + N / 2) % N] = tile[rr * pitch + c];
        }
      }
    }
  }
}

template <int N1, int N2, int AXIS, int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) ms_jvp_pass_kernel(JvpArgs a) {
  jvp_body<N1, N2, AXIS, WARPS>(a, blockIdx.y);
}

}  // namespace ptyro
