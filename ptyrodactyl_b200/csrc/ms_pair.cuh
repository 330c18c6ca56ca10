// Steady-state pass with two lines per thread in paired FP32 arithmetic.
//
// The middle slices' program (wave -> conv, x T, conv -> wave) is identical for
// every line, so each thread carries the same element positions of two neighbouring
// lines (A, B) as Pair values: real parts (A, B) and imaginary parts (A, B) in
// register pairs. Every add, multiply and fma of the line transforms is then one
// add/mul/fma.f32x2 instruction for both lines (sm_100), halving the issue slots of
// the FP32 work, and twiddles and propagator factors are read once for two lines.
// Results are bit-identical to the one-line kernel (each paired operation rounds
// as the scalar one it replaces).
//
// Per CTA: WARPS warps, 32 / N1 line pairs per warp. Row passes read and write the
// lines directly; column passes stage the CTA's block of 2 * pairs columns through a
// shared tile (row pitch lines + 4 float2, so 16-byte column-pair reads of eight
// lanes fall in distinct banks).
#pragma once
#include <cuda.h>

#include "ms_pass.cuh"
#include "ms_wait.cuh"

namespace ptyro {

// plain 3-D tiled TMA load of box (x, y, z) into this CTA's own shared memory only
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z), "r"(src)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void tma_store_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Exchange buffer of one line pair (Pair elements): same (k2, n1) index layout as
// LineBuf, padded to 4 mod 8 Pairs so the two line pairs of a warp start 64 bytes
// apart modulo the 128-byte bank window.
template <int N1, int N2>
struct PairBuf {
  static constexpr int kRaw = N2 * (N1 + 1);
  static constexpr int kSize = ((kRaw + 7) / 8) * 8 + 4;
};

template <int N1, int N2, int WARPS, bool PRE = false>
struct PairGeom {
  static constexpr int N = N1 * N2;
  static constexpr int G = 32 / N1;          // line pairs per warp
  static constexpr int kPairs = WARPS * G;   // line pairs per CTA
  static constexpr int kLines = 2 * kPairs;  // lines per CTA
  static constexpr int kPitch = kLines + 4;  // column tile row pitch (float2)
  static_assert(N % kLines == 0, "lines per CTA must divide N");
  static constexpr size_t kXbuf = sizeof(Pair) * (size_t)kPairs * PairBuf<N1, N2>::kSize;
  static constexpr size_t kTile = sizeof(float2) * (size_t)N * kPitch;
  static constexpr size_t kWork = kXbuf > kTile ? kXbuf : kTile;
  // twiddles + propagator factor + max(exchange buffers, column tile)
  // [+ the transmission rows of the CTA's lines, prefetched]
  static size_t smem_bytes() {
    return sizeof(float2) * 2 * (size_t)N + kWork + (PRE ? sizeof(float2) * (size_t)kLines * N : 0);
  }
};

// a * w with w = ((wA.x, wB.x), (wA.y, wB.y)): the operations of cmul(Pair, wA, wB)
__device__ __forceinline__ Pair cmul_pp(Pair a, Pair w) {
  return {__ffma2_rn(a.re, w.re, __fmul2_rn(a.im, make_float2(-w.im.x, -w.im.y))),
          __ffma2_rn(a.re, w.im, __fmul2_rn(a.im, w.re))};
}

// PRE: the transmission rows of the thread's two lines are copied into shared
// memory with cp.async at the start (each thread copies exactly the elements it
// multiplies, so waiting for its own copies suffices); windows need PRE = false.
// DIRECT (column passes): each lane pair reads and writes its two neighbouring
// columns straight from global memory as 16-byte pieces (32 contiguous bytes per row
// and lane pair), with no staging tile and no barriers.
// TMA (column passes of 256^2 grids): each warp moves its block of 2 G columns x N
// rows of the slot with one tiled TMA copy (wmap: the batch's wave slots as a 3-D
// tensor (x, y, slot) of 8-byte elements, box 2 G x N x 1), into and out of its own
// exchange buffers, instead of 16-byte loads and stores per row and lane pair; the
// wait on the copy's mbarrier gives up after a bounded number of polls, and then
// the warp flags the call's status word and skips its lines (warp_wait_tile).
// GEN: the first and last slice passes too: op1 may be OP_IFFT (the wave arrives
// transformed along this axis; inverse transform and a.scale instead of finishing a
// convolution) and op2 OP_FFT (forward transform instead of starting one). With
// N1 == N2 a thread's k-order positions are its natural ones (t + N1 r), so loads
// and stores are unchanged.
template <int N1, int N2, int AXIS, int WARPS, bool PRE, bool DIRECT, bool TMA, bool GEN>
__device__ __forceinline__ void pair_body(const PassArgs& a, const int slot, const CUtensorMap& wmap) {
  using PG = PairGeom<N1, N2, WARPS, PRE>;
  using PB = PairBuf<N1, N2>;
  constexpr int N = PG::N, G = PG::G, lines = PG::kLines, pitch = PG::kPitch;
  static_assert(!GEN || N1 == N2, "first / last passes need k-order positions equal to natural ones");
  const int op1 = GEN ? a.op1 : (int)OP_CONV, op2 = GEN ? a.op2 : (int)OP_CONV;
  static_assert(!TMA || (AXIS == 1 && DIRECT && !PRE && N <= 256), "TMA moves whole columns of a direct column pass");
  constexpr uint32_t kWarpBytes = sizeof(float2) * 2 * G * N;  // one warp's column block
  static_assert(!TMA || sizeof(Pair) * G * PB::kSize >= kWarpBytes + 127,
                "the warp's exchange buffers must hold its column block at 128-byte alignment");
  __shared__ __align__(8) uint64_t tma_bar[TMA ? WARPS : 1];
  extern __shared__ float4 smem4[];
  float2* tw = reinterpret_cast<float2*>(smem4);  // tw[k2 * N1 + t] = W_N^{t k2}
  float2* pfs = tw + N;                           // propagator factor along this axis
  float2* work = pfs + N;                         // column tile; aliases the exchange buffers
  Pair* xbuf = reinterpret_cast<Pair*>(work);
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
      tma_load_3d(smem_u32(stg), &wmap, blockIdx.x * lines + wp * 2 * G, 0, slot, bar);
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
  const int lp = warp * G + gl;  // line pair within the CTA
  const int line0 = blockIdx.x * lines;
  const int la = line0 + 2 * lp, lb = la + 1;
  Pair* buf = xbuf + lp * PB::kSize;
  float2* w = a.wave + (size_t)slot * N * N;
  float2* tpre = reinterpret_cast<float2*>(reinterpret_cast<char*>(work) + PG::kWork) + (size_t)(2 * lp) * N;
  if (PRE) {
    const float2* T = (AXIS == 0 ? a.trans : a.trans_t) + (size_t)a.t_slice * N * N;
#pragma unroll
    for (int j = 0; j < N2; ++j) {
      cp_async8(tpre + t + N1 * j, T + (size_t)la * N + t + N1 * j);
      cp_async8(tpre + N + t + N1 * j, T + (size_t)lb * N + t + N1 * j);
    }
    cp_async_commit();
  }
  Pair v[N2];

  // ---- load (natural distribution: element t + N1 j of lines A and B)
  if (AXIS == 0) {
#pragma unroll
    for (int j = 0; j < N2; ++j)
      v[j] = make_pair(w[(size_t)la * N + t + N1 * j], w[(size_t)lb * N + t + N1 * j]);
  } else if (TMA) {
    // a warp whose copy never landed leaves its lines untouched (no barrier follows)
    if (!warp_wait_tile(bar, kTileWaitPolls, a.status)) return;
#pragma unroll
    for (int j = 0; j < N2; ++j) {
      const float4 q = *reinterpret_cast<const float4*>(stg + (t + N1 * j) * (2 * G) + 2 * gl);
      v[j] = {make_float2(q.x, q.z), make_float2(q.y, q.w)};
    }
  } else if (DIRECT) {
#pragma unroll
    for (int j = 0; j < N2; ++j) {
      const float4 q = *reinterpret_cast<const float4*>(w + (size_t)(t + N1 * j) * N + la);
      v[j] = {make_float2(q.x, q.z), make_float2(q.y, q.w)};
    }
  } else {
    tile_load<N, lines, pitch, WARPS * 32>(w, work, line0);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < N2; ++j) {
      const float4 q = *reinterpret_cast<const float4*>(work + (t + N1 * j) * pitch + 2 * lp);
      v[j] = {make_float2(q.x, q.z), make_float2(q.y, q.w)};
    }
    __syncthreads();  // the tile becomes the exchange buffers
  }

  // ---- finish slice s-1's convolution along this axis (or the probe's inverse transform)
  if (op1 == OP_IFFT) {
    line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
#pragma unroll
    for (int j = 0; j < N2; ++j) v[j] = cscale(v[j], a.scale);
  } else {
    line_nat_to_k<N1, N2, -1>(v, t, buf, tw);
#pragma unroll
    for (int r = 0; r < N2; ++r) v[r] = cmul(v[r], pfs[korder_index<N1, N2>(t, r)]);
    line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
  }

  // ---- transmission T_s (row-major table for rows, transposed for columns)
  if (PRE) {
    cp_async_wait<0>();
#pragma unroll
    for (int j = 0; j < N2; ++j) v[j] = cmul(v[j], tpre[t + N1 * j], tpre[N + t + N1 * j]);
  } else {
    // the pair's lines sit at field lines la + lo, la + 1 + lo: one interleaved entry
    // serves both when lo is even (la is even)
    const float4* TP = AXIS == 0 ? a.trans_p : a.trans_pt;
    int lo = 0, eo = 0;
    if (a.win) {
      const int b = slot / a.n_modes;
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
        v[j] = cmul_pp(v[j], {make_float2(q.x, q.y), make_float2(q.z, q.w)});
      }
    } else {
      int oa, ob;
      const float2* Ta = trans_row<AXIS>(a.trans, a.trans_t, a.field_n, a.t_slice, a.win, slot / a.n_modes, la, &oa);
      const float2* Tb = trans_row<AXIS>(a.trans, a.trans_t, a.field_n, a.t_slice, a.win, slot / a.n_modes, lb, &ob);
#pragma unroll
      for (int j = 0; j < N2; ++j)
        v[j] = cmul(v[j], __ldg(Ta + ((t + N1 * j + oa) & fm)), __ldg(Tb + ((t + N1 * j + ob) & fm)));
    }
  }

  // gradient-mode checkpoint: the wave right after the T multiply
  if (a.ckpt_store) {
    float2* ck = a.ckpt_store + (size_t)slot * a.res_stride;
#pragma unroll
    for (int j = 0; j < N2; ++j) {
      // streaming stores: the residuals are read once, by the adjoint, and must not
      // push the batch's wave slots out of L2
      if (AXIS == 0) {
        __stcs(ck + (size_t)la * N + t + N1 * j, pair_a(v[j]));
        __stcs(ck + (size_t)lb * N + t + N1 * j, pair_b(v[j]));
      } else {
        __stcs(reinterpret_cast<float4*>(ck + (size_t)(t + N1 * j) * N + la),
               make_float4(v[j].re.x, v[j].im.x, v[j].re.y, v[j].im.y));
      }
    }
  }

  // ---- start slice s's convolution along this axis (or the far field's forward transform)
  if (op2 == OP_FFT) {
    line_nat_to_k<N1, N2, -1>(v, t, buf, tw);
  } else {
    line_nat_to_k<N1, N2, -1>(v, t, buf, tw);
#pragma unroll
    for (int r = 0; r < N2; ++r) v[r] = cmul(v[r], pfs[korder_index<N1, N2>(t, r)]);
    line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
  }

  // ---- store
  if (AXIS == 0) {
#pragma unroll
    for (int j = 0; j < N2; ++j) {
      w[(size_t)la * N + t + N1 * j] = pair_a(v[j]);
      w[(size_t)lb * N + t + N1 * j] = pair_b(v[j]);
    }
  } else if (TMA) {
    __syncwarp();  // every lane has read the last exchange
#pragma unroll
    for (int j = 0; j < N2; ++j)
      *reinterpret_cast<float4*>(stg + (t + N1 * j) * (2 * G) + 2 * gl) =
          make_float4(v[j].re.x, v[j].im.x, v[j].re.y, v[j].im.y);
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) {
      tma_store_3d(&wmap, la, 0, slot, smem_u32(stg));
      tma_store_wait_read();
    }
  } else if (DIRECT) {
#pragma unroll
    for (int j = 0; j < N2; ++j)
      *reinterpret_cast<float4*>(w + (size_t)(t + N1 * j) * N + la) =
          make_float4(v[j].re.x, v[j].im.x, v[j].re.y, v[j].im.y);
  } else {
    __syncthreads();  // every warp is done with its exchange buffer
#pragma unroll
    for (int j = 0; j < N2; ++j)
      *reinterpret_cast<float4*>(work + (t + N1 * j) * pitch + 2 * lp) =
          make_float4(v[j].re.x, v[j].im.x, v[j].re.y, v[j].im.y);
    __syncthreads();
    tile_store<N, lines, pitch, WARPS * 32>(w, work, line0);
  }
}

template <int N1, int N2, int AXIS, int WARPS, int MINB, bool PRE, bool DIRECT = false, bool TMA = false,
          bool GEN = false>
__global__ void __launch_bounds__(WARPS * 32, MINB)
    ms_pass_pair_kernel(PassArgs a, const __grid_constant__ CUtensorMap wmap) {
  pair_body<N1, N2, AXIS, WARPS, PRE, DIRECT, TMA, GEN>(a, blockIdx.y, wmap);
}

// Steady passes of several jobs in one launch (the scheduler's paired rows): CTA row
// y works on slot rows[y].y of the job whose arguments are descs[rows[y].x], copied
// into shared memory once per CTA. Column passes read their column pairs directly.
template <int N1, int N2, int AXIS, int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB)
    ms_pass_pair_multi_kernel(const PassArgs* __restrict__ descs, const int2* __restrict__ rows) {
  __shared__ __align__(16) PassArgs sa;
  const int2 r = rows[blockIdx.y];
  static_assert(sizeof(PassArgs) % 4 == 0, "descriptor copy in 32-bit words");
  const uint32_t* src = reinterpret_cast<const uint32_t*>(descs + r.x);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&sa);
  for (int i = threadIdx.x; i < (int)(sizeof(PassArgs) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  const CUtensorMap none = {};
  pair_body<N1, N2, AXIS, WARPS, false, AXIS == 1, false, false>(sa, r.y, none);
}

}  // namespace ptyro
