// Adjoint pass that carries only the adjoint wave, for gradients whose forward kept
// the wave at every slice (checkpoint spacing 1), grids up to 256^2.
//
// The lockstep adjoint (ms_bwd.cuh) pairs the forward wave psi and the adjoint lambda
// of one line and runs psi backward through U^H conj(T) alongside lambda, replacing
// it by the stored wave wherever a checkpoint exists. With a checkpoint at every
// slice point psi is never needed between slice points: lambda's recursion does not
// involve psi, and the dV contribution 2 sigma Im(conj(phi_s) lambda_s) takes phi_s
// straight from the stored residual. This pass therefore pairs the adjoints of two
// neighbouring lines (like the forward's paired pass), which halves the transform work
// of every adjoint pass; each paired operation rounds as the lockstep kernel's lambda
// half does, so the gradients are bit-identical to the lockstep adjoint at spacing 1.
// Row passes read and write lines directly; column passes read and write the two
// neighbouring columns of a lane pair as 16-byte pieces, or (TMA, 256^2, as the
// forward's paired column pass) move each warp's block of 2 G columns x N rows of
// lambda with one tiled TMA copy into and out of its own exchange buffers, with the
// bounded mbarrier wait of warp_wait_tile.
#pragma once
#include "ms_bwd.cuh"
#include "ms_pair.cuh"

namespace ptyro {

// Asynchronous prefetch of `bytes` (a multiple of 16, 16-byte aligned) of global
// memory into L2; nothing is written to shared memory and nothing waits on it.
__device__ __forceinline__ void prefetch_l2_bulk(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// a * conj(w) with a different w per line: the operations of cmulc(Pair, w) per lane
__device__ __forceinline__ Pair cmulc(Pair a, float2 wa, float2 wb) {
  const float2 wx = make_float2(wa.x, wb.x), wy = make_float2(wa.y, wb.y);
  return {__ffma2_rn(a.re, wx, __fmul2_rn(a.im, wy)), __ffma2_rn(a.im, wx, __fmul2_rn(a.re, make_float2(-wa.y, -wb.y)))};
}

template <int N1, int N2, int AXIS, int WARPS, bool TMA>
__device__ __forceinline__ void bwd_lam_body(const BwdArgs& a, const int slot, const CUtensorMap& lmap) {
  using PG = PairGeom<N1, N2, WARPS>;
  using PB = PairBuf<N1, N2>;
  constexpr int N = PG::N, G = PG::G, lines = PG::kLines;
  static_assert(!TMA || (AXIS == 1 && N <= 256), "TMA moves whole columns of a column pass");
  constexpr uint32_t kWarpBytes = sizeof(float2) * 2 * G * N;  // one warp's column block
  static_assert(!TMA || sizeof(Pair) * G * PB::kSize >= kWarpBytes + 127,
                "the warp's exchange buffers must hold its column block at 128-byte alignment");
  __shared__ __align__(8) uint64_t tma_bar[TMA ? WARPS : 1];
  extern __shared__ float4 smem4[];
  float2* tw = reinterpret_cast<float2*>(smem4);  // tw[k2 * N1 + t] = W_N^{t k2}
  float2* pfs = tw + N;                           // propagator factor / N
  Pair* xbuf = reinterpret_cast<Pair*>(pfs + N);
  // TMA staging: this warp's exchange buffers, rounded up to 128 bytes; [row][2 G columns]
  float2* stg = nullptr;
  uint32_t bar = 0;
  if (TMA) {
    const int wp = threadIdx.x >> 5;
    const uintptr_t base = reinterpret_cast<uintptr_t>(xbuf + (size_t)(wp * G) * PB::kSize);
    stg = reinterpret_cast<float2*>((base + 127) & ~(uintptr_t)127);
    bar = smem_u32(&tma_bar[wp]);
    if ((threadIdx.x & 31) == 0) {
      mbar_init(bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      mbar_expect_tx(bar, kWarpBytes);
      tma_load_3d(smem_u32(stg), &lmap, blockIdx.x * lines + wp * 2 * G, 0, slot, bar);
    }
  }
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int k2 = i / N1, tt = i % N1;
    tw[i] = a.tw[(tt * k2) % N];
    pfs[i] = a.pf[i];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = AXIS == 0 ? (lane % N1) : (lane / G);
  const int gl = AXIS == 0 ? (lane / N1) : (lane % G);
  const int lp = warp * G + gl;
  const int la = blockIdx.x * lines + 2 * lp, lb = la + 1;
  Pair* buf = xbuf + lp * PB::kSize;
  const size_t NN = (size_t)N * N;
  const int b = slot / a.n_modes, m = slot % a.n_modes;
  float2* Wl = a.lam + (size_t)slot * NN;
  // the stored wave phi_s of the CTA's lines, wanted after the first transform: its
  // DRAM latency overlaps that transform (rows: one contiguous block; columns: one
  // row segment of the CTA's columns per thread)
  if (a.t_slice >= 0) {
    const float2* ck0 = a.ckpt + (size_t)slot * a.res_stride;
    const int line0 = blockIdx.x * lines;
    if (AXIS == 0) {
      constexpr uint32_t kChunk = 4096;
      constexpr uint32_t kBytes = sizeof(float2) * (uint32_t)lines * N;
      if (threadIdx.x < kBytes / kChunk)
        prefetch_l2_bulk(reinterpret_cast<const char*>(ck0 + (size_t)line0 * N) + threadIdx.x * kChunk, kChunk);
    } else {
      for (int e = threadIdx.x; e < N; e += blockDim.x)
        prefetch_l2_bulk(ck0 + (size_t)e * N + line0, sizeof(float2) * lines);
    }
  }
  const bool korder_in = a.init || a.op1 == OP_IFFT;
  Pair v[N2];

  // ---- load lambda of both lines
  if (a.init) {  // lam = N^2 w_m g(shifted) A in k-space
    const float2* A = a.amp + (size_t)slot * a.res_stride;
    const float* g = a.gpat + (size_t)b * NN;
    const float s = (float)N * (float)N * a.weights[m];
    const int ksa = (la + N / 2) % N, ksb = (lb + N / 2) % N;
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const int k = korder_index<N1, N2>(t, r), kq = (k + N / 2) % N;
      const float2 aa = __ldcs(A + (AXIS == 0 ? (size_t)la * N + k : (size_t)k * N + la));
      const float2 ab = __ldcs(A + (AXIS == 0 ? (size_t)lb * N + k : (size_t)k * N + lb));
      const float ga = AXIS == 0 ? g[(size_t)ksa * N + kq] : g[(size_t)kq * N + ksa];
      const float gb = AXIS == 0 ? g[(size_t)ksb * N + kq] : g[(size_t)kq * N + ksb];
      v[r] = make_pair(cscale(aa, s * ga), cscale(ab, s * gb));
    }
  } else {
    // a warp whose copy never landed leaves its lines untouched (no barrier follows)
    if (TMA && !warp_wait_tile(bar, kTileWaitPolls, a.status)) return;
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const int e = korder_in ? korder_index<N1, N2>(t, r) : t + N1 * r;
      if (AXIS == 0) {
        v[r] = make_pair(Wl[(size_t)la * N + e], Wl[(size_t)lb * N + e]);
      } else {
        const float4 q = TMA ? *reinterpret_cast<const float4*>(stg + (size_t)e * (2 * G) + 2 * gl)
                             : *reinterpret_cast<const float4*>(Wl + (size_t)e * N + la);
        v[r] = {make_float2(q.x, q.z), make_float2(q.y, q.w)};
      }
    }
  }

  // ---- op1
  if (a.op1 == OP_IFFT) {
    line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
#pragma unroll
    for (int j = 0; j < N2; ++j) v[j] = cscale(v[j], a.scale);
  } else if (a.op1 == OP_CONV_CONJ || a.op1 == OP_FFT) {
    apply_op<N1, N2>(a.op1, v, t, buf, tw, pfs);
  }

  // ---- slice point: dV contribution from the stored wave phi_s (stored at once, so
  // it holds no registers through the second transform), then conj(T_s). phi_s is
  // read and the contribution written with streaming hints (each is touched once), so
  // that the batch's lambda slots stay in L2 between passes.
  if (a.t_slice >= 0) {
    const float2* ck = a.ckpt + (size_t)slot * a.res_stride;
    float* C = a.contrib ? a.contrib + (size_t)slot * NN : nullptr;
#pragma unroll
    for (int j = 0; j < N2; ++j) {
      const int e = t + N1 * j;
      float2 pa, pb;
      if (AXIS == 0) {
        pa = __ldcs(ck + (size_t)la * N + e);
        pb = __ldcs(ck + (size_t)lb * N + e);
      } else {
        const float4 q = __ldcs(reinterpret_cast<const float4*>(ck + (size_t)e * N + la));
        pa = make_float2(q.x, q.y);
        pb = make_float2(q.z, q.w);
      }
      const float cva = a.sigma2 * (pa.x * v[j].im.x - pa.y * v[j].re.x);
      const float cvb = a.sigma2 * (pb.x * v[j].im.y - pb.y * v[j].re.y);
      if (C) {
        if (AXIS == 0) {
          __stcs(C + (size_t)la * N + e, cva);
          __stcs(C + (size_t)lb * N + e, cvb);
        } else {
          __stcs(reinterpret_cast<float2*>(C + (size_t)e * N + la), make_float2(cva, cvb));
        }
      }
    }
    // the pair's lines sit at field lines la + lo, la + 1 + lo: one interleaved entry
    // (T[2p].re, T[2p+1].re, T[2p].im, T[2p+1].im) serves both when lo is even, and
    // multiplies with the same operations as the two plain loads
    const float4* TP = AXIS == 0 ? a.trans_p : a.trans_pt;
    int lo = 0, eo = 0;
    if (a.win) {
      lo = AXIS == 0 ? a.win[2 * b] : a.win[2 * b + 1];
      eo = AXIS == 0 ? a.win[2 * b + 1] : a.win[2 * b];
    }
    const int fm = a.field_n - 1;
    if (TP != nullptr && (lo & 1) == 0) {
      const float4* row =
          TP + ((size_t)a.t_slice * (a.field_n / 2) + (size_t)(((la + lo) & fm) >> 1)) * a.field_n;
#pragma unroll
      for (int j = 0; j < N2; ++j) {
        const float4 q = __ldg(row + ((t + N1 * j + eo) & fm));
        const float2 wx = make_float2(q.x, q.y), wy = make_float2(q.z, q.w);
        v[j] = {__ffma2_rn(v[j].re, wx, __fmul2_rn(v[j].im, wy)),
                __ffma2_rn(v[j].im, wx, __fmul2_rn(v[j].re, make_float2(-q.z, -q.w)))};
      }
    } else {
      int oa, ob;
      const float2* Ta = trans_row<AXIS>(a.trans, a.trans_t, a.field_n, a.t_slice, a.win, b, la, &oa);
      const float2* Tb = trans_row<AXIS>(a.trans, a.trans_t, a.field_n, a.t_slice, a.win, b, lb, &ob);
#pragma unroll
      for (int j = 0; j < N2; ++j)
        v[j] = cmulc(v[j], __ldg(Ta + ((t + N1 * j + oa) & fm)), __ldg(Tb + ((t + N1 * j + ob) & fm)));
    }
  }

  // ---- op2, and the beam-gradient epilogue (lambda k-order along this axis times conj(ramp))
  bool lam_k = a.op1 == OP_FFT;
  if (a.op2 == OP_CONV_CONJ) {
    apply_op<N1, N2>(OP_CONV_CONJ, v, t, buf, tw, pfs);
  } else if (a.op2 == OP_FFT) {
    apply_op<N1, N2>(OP_FFT, v, t, buf, tw, pfs);
    lam_k = true;
  }
  if (a.beam_epi) {
    const float2* ra = (AXIS == 0 ? a.ramp_x : a.ramp_y) + (size_t)b * N;
#pragma unroll
    for (int r = 0; r < N2; ++r) v[r] = cmulc(v[r], ra[korder_index<N1, N2>(t, r)]);
  }

  // ---- store lambda
  if (TMA) {
    __syncwarp();  // every lane has read the last exchange
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const int e = lam_k ? korder_index<N1, N2>(t, r) : t + N1 * r;
      *reinterpret_cast<float4*>(stg + (size_t)e * (2 * G) + 2 * gl) =
          make_float4(v[r].re.x, v[r].im.x, v[r].re.y, v[r].im.y);
    }
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) {
      tma_store_3d(&lmap, la, 0, slot, smem_u32(stg));
      tma_store_wait_read();
    }
    return;
  }
#pragma unroll
  for (int r = 0; r < N2; ++r) {
    const int e = lam_k ? korder_index<N1, N2>(t, r) : t + N1 * r;
    if (AXIS == 0) {
      Wl[(size_t)la * N + e] = pair_a(v[r]);
      Wl[(size_t)lb * N + e] = pair_b(v[r]);
    } else {
      *reinterpret_cast<float4*>(Wl + (size_t)e * N + la) = make_float4(v[r].re.x, v[r].im.x, v[r].re.y, v[r].im.y);
    }
  }
}

template <int N1, int N2, int AXIS, int WARPS, int MINB, bool TMA = false>
__global__ void __launch_bounds__(WARPS * 32, MINB) ms_bwd_lam_kernel(BwdArgs a, const __grid_constant__ CUtensorMap lmap) {
  bwd_lam_body<N1, N2, AXIS, WARPS, TMA>(a, blockIdx.y, lmap);
}

}  // namespace ptyro
