// Pipelined steady-state pass: persistent CTAs walk the wave slots of a batch and
// prefetch the next slot's lines into shared memory with cp.async while the
// current slot is transformed, so global-load latency hides behind the FFT work.
//
// Program (the middle slices): wave -> conv, x T, conv -> wave. Per CTA two tiles
// hold its block of lines of two consecutive slots: row passes keep `lines` full
// rows (contiguous in global memory), column passes keep all N rows of `lines`
// columns. Once a tile has been read into registers
// it serves as the warps' exchange buffers; column results go back through it so
// global stores move whole row segments.
#pragma once
#include "ms_pass.cuh"

namespace ptyro {

template <int N1, int N2, int AXIS, int WARPS>
struct PipeGeom {
  static constexpr int N = N1 * N2;
  static constexpr int G = 32 / N1;
  static constexpr int kLines = WARPS * G;
  // row passes: pitch kSize (>= N + 8, = 8 mod 16: the two lines of a warp fall in
  // different bank halves); column passes: lines + G (t * pitch + lc spreads banks)
  static constexpr int kRowPitch = AXIS == 0 ? LineBuf<N1, N2>::kSize : kLines + G;
  static constexpr int kTileRows = AXIS == 0 ? kLines : N;
  static constexpr int kXbuf = kLines * LineBuf<N1, N2>::kSize;
  static constexpr int kTile = kTileRows * kRowPitch > kXbuf ? kTileRows * kRowPitch : kXbuf;
  // 16-byte copies where every tile row starts 16-byte aligned, else 8-byte copies
  static constexpr int kChunkElems = kRowPitch % 2 == 0 ? 2 : 1;
  static constexpr int kChunksPerRow = (AXIS == 0 ? N : kLines) / kChunkElems;
  static constexpr int kChunks = kTileRows * kChunksPerRow;
  static_assert(kChunks % (WARPS * 32) == 0, "tile chunks must divide evenly among the threads");
  static_assert(kTile % 2 == 0, "the second tile must start 16-byte aligned");
  static_assert(AXIS != 0 || kRowPitch >= N, "a row must fit in the row pitch");
  // twiddles come from a global (k2, t) table, so shared memory holds the two tiles only
  static size_t smem_bytes() { return sizeof(float2) * 2 * (size_t)kTile; }
};

// issue the async copy of slot `slot`'s block of lines into `tile`
template <int N1, int N2, int AXIS, int WARPS>
__device__ __forceinline__ void pipe_issue(const float2* __restrict__ wave, int slot, int line0, float2* tile) {
  using PG = PipeGeom<N1, N2, AXIS, WARPS>;
  constexpr int N = PG::N;
  const float2* w = wave + (size_t)slot * N * N;
#pragma unroll
  for (int it = 0; it < PG::kChunks / (WARPS * 32); ++it) {
    const int c = threadIdx.x + it * WARPS * 32;
    const int r = c / PG::kChunksPerRow, k = (c % PG::kChunksPerRow) * PG::kChunkElems;
    const float2* src = AXIS == 0 ? w + (size_t)(line0 + r) * N + k : w + (size_t)r * N + line0 + k;
    if (PG::kChunkElems == 2) cp_async16(tile + r * PG::kRowPitch + k, src);
    else cp_async8(tile + r * PG::kRowPitch + k, src);
  }
  cp_async_commit();
}

template <int N1, int N2, int AXIS, int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) ms_pass_pipe_kernel(PassArgs a, int nslots) {
  using PG = PipeGeom<N1, N2, AXIS, WARPS>;
  using LB = LineBuf<N1, N2>;
  constexpr int N = PG::N, G = PG::G, lines = PG::kLines, pitch = PG::kRowPitch;
  extern __shared__ float2 smem[];
  const float2* tw = a.tw2;  // tw2[k2 * N1 + t] = W_N^{t k2}, read through L1
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = AXIS == 0 ? (lane % N1) : (lane / G);
  const int gl = AXIS == 0 ? (lane / N1) : (lane % G);
  const int lc = warp * G + gl;
  const int line0 = blockIdx.x * lines;
  const int line = line0 + lc;
  const size_t NN = (size_t)N * N;
  const int fm = a.field_n - 1;
  int slot = blockIdx.y;
  if (slot >= nslots) return;  // whole CTA idle (uniform)
  pipe_issue<N1, N2, AXIS, WARPS>(a.wave, slot, line0, smem);
  int cur = 0;
  for (; slot < nslots; slot += gridDim.y) {
    const int next = slot + gridDim.y;
    if (next < nslots) {
      pipe_issue<N1, N2, AXIS, WARPS>(a.wave, next, line0, smem + (cur ^ 1) * PG::kTile);
      cp_async_wait<1>();  // every group but the newest (this slot's tile) has landed
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    float2* tile = smem + cur * PG::kTile;
    float2 v[N2];
#pragma unroll
    for (int j = 0; j < N2; ++j)
      v[j] = AXIS == 0 ? tile[lc * pitch + t + N1 * j] : tile[(t + N1 * j) * pitch + lc];
    __syncthreads();  // the tile becomes the exchange buffers
    float2* buf = tile + lc * LB::kSize;
    apply_op<N1, N2>(OP_CONV, v, t, buf, tw, a.pf);
    {
      int eoff;
      const float2* T = trans_row<AXIS>(a.trans, a.trans_t, a.field_n, a.t_slice, a.win, slot / a.n_modes, line,
                                        &eoff);
#pragma unroll
      for (int j = 0; j < N2; ++j) v[j] = cmul(v[j], __ldg(T + ((t + N1 * j + eoff) & fm)));
      if (a.ckpt_store) {
        float2* ck = a.ckpt_store + (size_t)slot * a.res_stride;
#pragma unroll
        for (int j = 0; j < N2; ++j)
          ck[AXIS == 0 ? (size_t)line * N + t + N1 * j : (size_t)(t + N1 * j) * N + line] = v[j];
      }
    }
    apply_op<N1, N2>(OP_CONV, v, t, buf, tw, a.pf);
    float2* w = a.wave + (size_t)slot * NN;
    if (AXIS == 0) {
#pragma unroll
      for (int j = 0; j < N2; ++j) w[(size_t)line * N + t + N1 * j] = v[j];
      __syncthreads();  // this tile is refilled by the next-but-one prefetch
    } else {
      __syncthreads();
#pragma unroll
      for (int j = 0; j < N2; ++j) tile[(t + N1 * j) * pitch + lc] = v[j];
      __syncthreads();
      tile_store<N, lines, pitch, WARPS * 32>(w, tile, line0);
      __syncthreads();
    }
    cur ^= 1;
  }
}

}  // namespace ptyro
