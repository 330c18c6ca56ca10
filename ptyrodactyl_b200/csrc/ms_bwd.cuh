// Adjoint pass of the multislice engine (reverse-mode gradient).
//
// Forward, per probe and mode: phi_s = psi_s T_s, psi_{s+1} = U phi_s with
// U = ifft2 diag(P) fft2 (unitary), A = fft2(phi_{S-1}), I = sum_m w_m |A_m|^2
// (stored fftshifted). With g = dL/dI and lam = dL/dconj(.):
//   lam_A          = N^2 w_m ifftshift(g) A          (so lam_phi_{S-1} = ifft2(lam_A))
//   dL/dV_s        = 2 sigma Im(conj(phi_s) lam_phi_s)
//   lam_phi_{s-1}  = U^H (conj(T_s) lam_phi_s)
//   phi_{s-1}      = U^H (conj(T_s) phi_s)            (the forward run backwards)
// The adjoint and the reconstructed forward wave obey the same operator, so one
// pass carries both waves of a line through it in lockstep; at each slice point
// the pair is in registers and the pass emits the per-pixel dV contribution. The
// reconstructed wave is replaced by the checkpoint stored in the forward where one
// exists, which bounds the rounding drift of running U backwards. Passes follow
// the forward's schedule: op'_0 = IFFT2, op'_j = U^H, op'_S = FFT2 (adjoint only).
#pragma once
#include "ms_pair.cuh"

namespace ptyro {

struct BwdArgs {
  float2* psi;             // reconstructed forward wave slots (B*M planes)
  float2* lam;             // adjoint slots
  const float2* amp;       // init: far-field amplitude residual of slot w at amp + w * res_stride
  const float* gpat;       // init: upstream dL/dI (B, N, N), fftshifted like the patterns
  const float* weights;    // (M)
  const float2* ckpt;      // checkpoint plane of this pass's slice point (slot stride res_stride), or null
  size_t res_stride;
  const float2* trans;     // (S, F, F) T, row-major
  const float2* trans_t;   // transposed
  const float4* trans_p;   // T interleaved by line pairs (rows), or null: the lambda-only pass's one
  const float4* trans_pt;  // 16-byte load per element pair; and the transposed table's column pairs
  const int* win;          // (B, 2) window origins in the field, or null
  int field_n;             // F (== N without windows)
  const float2* pf;        // (N) propagator factor / N (conjugated in use)
  const float2* tw;        // (N) forward twiddles
  const float2* ramp_y;    // (B, N) shift ramps (beam-gradient epilogue)
  const float2* ramp_x;
  float* contrib;          // (B*M, N, N) row-major dV contribution of this pass's slice point, or null
  int n_modes;
  int init;                // 1: psi <- amp, lam <- N^2 w g amp (k-order loads), op1 must be OP_IFFT
  int op1, t_slice, op2;   // op1 on both waves; T point (conj T) ; op2 on lam (and psi unless psi_done)
  int psi_done;            // the forward wave is not needed after this pass's slice point
  int beam_epi;            // op2 / op1 ends in k-order: multiply lam by conj(ramp along this axis)
  float sigma2;            // 2 sigma
  float scale;             // 1/N after OP_IFFT
  unsigned int* status;    // the call's device status word (PTYRO_STATUS_* bits), or null
  int lam_only;            // every slice point has a checkpoint: carry lambda only (ms_bwd_lam.cuh)
};

// Shared memory of an adjoint pass: twiddles + max(paired exchange buffers, tile).
template <int N1, int N2>
size_t bwd_smem_bytes(int warps) {
  constexpr int N = N1 * N2, G = 32 / N1;
  const size_t lines = (size_t)warps * G;
  const size_t xbuf = sizeof(Pair) * lines * PairBuf<N1, N2>::kSize;
  const size_t tile = sizeof(float2) * (size_t)N * (lines + G);
  return sizeof(float2) * (size_t)N + (xbuf > tile ? xbuf : tile);
}

// Read one wave of a line from global memory (rows) or the staged tile (columns)
// into half H (0: the forward wave, 1: the adjoint) of the paired registers.
template <int N1, int N2, int AXIS, int H>
__device__ __forceinline__ void bwd_load_half(const float2* w, Pair (&v)[N2], bool korder, int t, int line, int lc,
                                              const float2* work, int pitch) {
  constexpr int N = N1 * N2;
#pragma unroll
  for (int r = 0; r < N2; ++r) {
    const int e = korder ? korder_index<N1, N2>(t, r) : t + N1 * r;
    const float2 x = AXIS == 0 ? w[(size_t)line * N + e] : work[e * pitch + lc];
    if (H == 0) {
      v[r].re.x = x.x;
      v[r].im.x = x.y;
    } else {
      v[r].re.y = x.x;
      v[r].im.y = x.y;
    }
  }
}

// The forward wave psi and the adjoint lambda of a line go through identical
// operators, so they are carried as one Pair per element (half 0 = psi, half 1 =
// lambda) and every transform step is one paired f32x2 operation for both.
// TMA (column passes without the k-space init): each warp's block of G columns x N
// rows of psi and of lambda comes in with two tiled TMA copies issued together at the
// start (pmap / lmap: the slots as 3-D tensors (x, y, slot), box G x N x 1) into its
// own exchange buffers, and goes back the same way, instead of two rounds through
// the CTA's column tile with barriers; the dV contribution keeps the tile (a box of
// G floats is narrower than TMA's 16-byte minimum).
template <int N1, int N2, int AXIS, int WARPS, bool TMA = false>
__device__ __forceinline__ void bwd_body(const BwdArgs& a, const int slot, const CUtensorMap* pmap = nullptr,
                                         const CUtensorMap* lmap = nullptr) {
  using Geo = PassGeom<N1, N2>;
  using LB = LineBuf<N1, N2>;
  constexpr int N = Geo::N;
  constexpr int G = Geo::G;
  constexpr int lines = WARPS * G;
  static_assert(N % lines == 0, "lines per CTA must divide N");
  static_assert(!TMA || (AXIS == 1 && N <= 256 && G * 8 % 16 == 0), "TMA moves whole column blocks");
  constexpr int pitch = lines + G;
  constexpr uint32_t kBlock = sizeof(float2) * G * N;  // one wave's column block of a warp
  static_assert(!TMA || sizeof(Pair) * G * PairBuf<N1, N2>::kSize >= 2 * kBlock + 127,
                "the warp's exchange buffers must hold both column blocks at 128-byte alignment");
  __shared__ __align__(8) uint64_t bwd_bar[TMA ? WARPS : 1];
  extern __shared__ float2 smem[];
  float2* tw = smem;
  float2* work = smem + N;
  float2* stg = nullptr;  // TMA staging: psi block, then lambda block, [row][G]
  uint32_t bar = 0;
  bool tile_ok = true;  // false once this warp's tile wait gave up
  if (TMA) {
    const int wp = threadIdx.x >> 5;
    const uintptr_t base = reinterpret_cast<uintptr_t>(reinterpret_cast<Pair*>(work) + (size_t)(wp * G) * PairBuf<N1, N2>::kSize);
    stg = reinterpret_cast<float2*>((base + 127) & ~(uintptr_t)127);
    bar = smem_u32(&bwd_bar[wp]);
    if ((threadIdx.x & 31) == 0) {
      const bool with_psi = a.op1 != OP_FFT;
      const int x = blockIdx.x * lines + wp * G;
      mbar_init(bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      mbar_expect_tx(bar, (with_psi ? 2u : 1u) * kBlock);
      if (with_psi) tma_load_3d(smem_u32(stg), pmap, x, 0, slot, bar);
      tma_load_3d(smem_u32(stg + G * N), lmap, x, 0, slot, bar);
    }
  }
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
  // exchange buffer of the line (Pair elements)
  Pair* buf = reinterpret_cast<Pair*>(work) + lc * PairBuf<N1, N2>::kSize;
  const size_t NN = (size_t)N * N;
  const int b = slot / a.n_modes, m = slot % a.n_modes;
  auto off = [&](int e) -> size_t { return AXIS == 0 ? (size_t)line * N + e : (size_t)e * N + line; };

  float2* Wp = a.psi + (size_t)slot * NN;
  float2* Wl = a.lam + (size_t)slot * NN;
  const bool korder_in = a.init || a.op1 == OP_IFFT;
  Pair v[N2];

  // ---- load both waves (column passes stage each through the tile in turn)
  if (a.init) {
    // row pass over k-space: psi = A, lam = N^2 w_m g(shifted) A
    const float2* A = a.amp + (size_t)slot * a.res_stride;
    const float* g = a.gpat + (size_t)b * NN;
    const float s = (float)N * (float)N * a.weights[m];
    const int ks_line = (line + N / 2) % N;
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const int k = korder_index<N1, N2>(t, r);
      const float2 av = A[off(k)];
      const float gv = AXIS == 0 ? g[(size_t)ks_line * N + (k + N / 2) % N] : g[(size_t)((k + N / 2) % N) * N + ks_line];
      v[r] = make_pair(av, cscale(av, s * gv));
    }
  } else if (AXIS == 0) {
    if (a.op1 != OP_FFT) {
      bwd_load_half<N1, N2, AXIS, 0>(Wp, v, korder_in, t, line, lc, work, pitch);
    } else {
#pragma unroll
      for (int r = 0; r < N2; ++r) v[r].re.x = v[r].im.x = 0.f;  // psi is not carried
    }
    bwd_load_half<N1, N2, AXIS, 1>(Wl, v, korder_in, t, line, lc, work, pitch);
  } else if (TMA) {
    // a warp whose copies never landed computes on stale shared memory but writes no
    // wave back; it still takes part in the dV tile's block barriers below
    tile_ok = warp_wait_tile(bar, kTileWaitPolls, a.status);
    if (a.op1 == OP_FFT) {
#pragma unroll
      for (int r = 0; r < N2; ++r) v[r].re.x = v[r].im.x = 0.f;
    } else {
      bwd_load_half<N1, N2, AXIS, 0>(Wp, v, korder_in, t, line, gl, stg, G);
    }
    bwd_load_half<N1, N2, AXIS, 1>(Wl, v, korder_in, t, line, gl, stg + G * N, G);
  } else {
    if (a.op1 == OP_FFT) {
#pragma unroll
      for (int r = 0; r < N2; ++r) v[r].re.x = v[r].im.x = 0.f;
    }
    for (int wv = a.op1 == OP_FFT ? 1 : 0; wv < 2; ++wv) {
      const float2* W = wv == 0 ? Wp : Wl;
      __syncthreads();
      tile_load<N, lines, pitch, WARPS * 32>(W, work, line0);
      __syncthreads();
      if (wv == 0) bwd_load_half<N1, N2, AXIS, 0>(W, v, korder_in, t, line, lc, work, pitch);
      else bwd_load_half<N1, N2, AXIS, 1>(W, v, korder_in, t, line, lc, work, pitch);
    }
    __syncthreads();
  }

  // ---- op1 on both
  if (a.op1 == OP_IFFT) {
    line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
#pragma unroll
    for (int j = 0; j < N2; ++j) v[j] = cscale(v[j], a.scale);
  } else if (a.op1 == OP_CONV_CONJ || a.op1 == OP_FFT) {
    apply_op<N1, N2>(a.op1, v, t, buf, tw, a.pf);
  }

  // ---- slice point: checkpoint refresh, dV contribution, conj(T)
  float cv[N2];
  if (a.t_slice >= 0) {
    if (a.ckpt) {
      const float2* ck = a.ckpt + (size_t)slot * a.res_stride;
#pragma unroll
      for (int j = 0; j < N2; ++j) {
        const float2 c = ck[off(t + N1 * j)];
        v[j].re.x = c.x;
        v[j].im.x = c.y;
      }
    }
#pragma unroll
    for (int j = 0; j < N2; ++j) cv[j] = a.sigma2 * (v[j].re.x * v[j].im.y - v[j].im.x * v[j].re.y);
    int eoff;
    const float2* T = trans_row<AXIS>(a.trans, a.trans_t, a.field_n, a.t_slice, a.win, b, line, &eoff);
    const int fm = a.field_n - 1;
#pragma unroll
    for (int j = 0; j < N2; ++j) v[j] = cmulc(v[j], __ldg(T + ((t + N1 * j + eoff) & fm)));
  }

  // ---- op2 (psi too, even where it is no longer needed: it rides in the same instructions)
  bool lam_k = a.op1 == OP_FFT;
  if (a.op2 == OP_CONV_CONJ) {
    apply_op<N1, N2>(OP_CONV_CONJ, v, t, buf, tw, a.pf);
  } else if (a.op2 == OP_FFT) {
    apply_op<N1, N2>(OP_FFT, v, t, buf, tw, a.pf);
    lam_k = true;
  }
  if (a.beam_epi) {
    // lam is k-order along this axis: multiply conj(ramp(k)) of this axis
    const float2* ra = (AXIS == 0 ? a.ramp_x : a.ramp_y) + (size_t)b * N;
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const float2 l = cmulc(pair_b(v[r]), ra[korder_index<N1, N2>(t, r)]);
      v[r].re.y = l.x;
      v[r].im.y = l.y;
    }
  }

  // ---- store
  const bool store_psi = !a.psi_done && a.op1 != OP_FFT;
  if (AXIS == 0) {
    if (store_psi) {
#pragma unroll
      for (int j = 0; j < N2; ++j) Wp[off(t + N1 * j)] = pair_a(v[j]);
    }
#pragma unroll
    for (int r = 0; r < N2; ++r) Wl[off(lam_k ? korder_index<N1, N2>(t, r) : t + N1 * r)] = pair_b(v[r]);
    if (a.t_slice >= 0 && a.contrib) {
      float* C = a.contrib + (size_t)slot * NN;
#pragma unroll
      for (int j = 0; j < N2; ++j) C[off(t + N1 * j)] = cv[j];
    }
  } else if (TMA) {
    __syncwarp();  // every lane has read the last exchange
    if (store_psi) {
#pragma unroll
      for (int j = 0; j < N2; ++j) stg[(t + N1 * j) * G + gl] = pair_a(v[j]);
    }
#pragma unroll
    for (int r = 0; r < N2; ++r) stg[G * N + (lam_k ? korder_index<N1, N2>(t, r) : t + N1 * r) * G + gl] = pair_b(v[r]);
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0 && tile_ok) {
      const int x = line0 + warp * G;
      if (store_psi) tma_store_3d(pmap, x, 0, slot, smem_u32(stg));
      tma_store_3d(lmap, x, 0, slot, smem_u32(stg + G * N));
      tma_store_wait_read();
    }
    if (a.t_slice >= 0 && a.contrib) {
      __syncthreads();  // every warp's copies have read its staging before the tile reuses it
      float* tile = reinterpret_cast<float*>(work);
#pragma unroll
      for (int j = 0; j < N2; ++j) tile[(t + N1 * j) * pitch + lc] = cv[j];
      __syncthreads();
      tile_store<N, lines, pitch, WARPS * 32>(a.contrib + (size_t)slot * NN, reinterpret_cast<const float*>(work),
                                              line0);
    }
  } else {
    for (int wv = 0; wv < 3; ++wv) {
      if (wv == 0 && !store_psi) continue;
      if (wv == 2 && !(a.t_slice >= 0 && a.contrib)) continue;
      __syncthreads();
      if (wv == 0) {
#pragma unroll
        for (int j = 0; j < N2; ++j) work[(t + N1 * j) * pitch + lc] = pair_a(v[j]);
      } else if (wv == 1) {
#pragma unroll
        for (int r = 0; r < N2; ++r)
          work[(lam_k ? korder_index<N1, N2>(t, r) : t + N1 * r) * pitch + lc] = pair_b(v[r]);
      } else {
        float* tile = reinterpret_cast<float*>(work);
#pragma unroll
        for (int j = 0; j < N2; ++j) tile[(t + N1 * j) * pitch + lc] = cv[j];
      }
      __syncthreads();
      if (wv < 2) {
        tile_store<N, lines, pitch, WARPS * 32>(wv == 0 ? Wp : Wl, work, line0);
      } else {
        tile_store<N, lines, pitch, WARPS * 32>(a.contrib + (size_t)slot * NN,
                                                reinterpret_cast<const float*>(work), line0);
      }
    }
  }
}


template <int N1, int N2, int AXIS, int WARPS, int MINB, bool TMA = false>
__global__ void __launch_bounds__(WARPS * 32, MINB)
    ms_bwd_pass_kernel(BwdArgs a, const __grid_constant__ CUtensorMap pmap, const __grid_constant__ CUtensorMap lmap) {
  bwd_body<N1, N2, AXIS, WARPS, TMA>(a, blockIdx.y, &pmap, &lmap);
}

// Adjoint passes of several jobs in one launch (see ms_pass_multi_kernel).
template <int N1, int N2, int AXIS, int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) ms_bwd_multi_kernel(const BwdArgs* __restrict__ descs,
                                                                        const int2* __restrict__ rows) {
  const int2 r = rows[blockIdx.y];
  bwd_body<N1, N2, AXIS, WARPS>(descs[r.x], r.y);
}

}  // namespace ptyro
