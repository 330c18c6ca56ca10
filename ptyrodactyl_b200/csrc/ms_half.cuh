// Steady-state pass for lines of N = N1 * 2 N1 points (512 = 16 x 32) with the two
// halves of each thread's work paired in f32x2 arithmetic.
//
// A thread owns 2 N1 points of one line. Two lines per thread (ms_pair.cuh) would
// not fit in registers here, so the pairing is inside the line:
//   natural order:   Pair j = (x[t + N1 j], x[t + N1 (j + N1)]),  j < N1
//   in-thread DFT:   decimation in frequency, a_j = x_j + x_{j+N1},
//                    b_j = (x_j - x_{j+N1}) W_{2 N1}^j, then one paired N1-point DFT
//                    gives (X[2k], X[2k+1]) in Pair k
//   exchange:        thread t of the second stage takes rows k2 = 2t and 2t + 1 of
//                    every column, exactly the Pairs the first stage produced, so the
//                    exchange moves whole Pairs (16 bytes) and the N1-point DFTs of
//                    the second stage pair too: thread t ends with
//                    Pair k1 = (X[2t + N2 k1], X[2t + 1 + N2 k1])
//   inverse:         the mirror image (paired group DFTs, exchange, paired N1-point
//                    DFT of (even, odd) inputs, decimation-in-time final stage), which
//                    returns each value to the thread and the pairing it came from.
// Every step that treats the pair halves alike runs as paired instructions; only
// the two radix-2 stages that join the halves run scalar.
#pragma once
#include "ms_pair.cuh"

namespace ptyro {

template <int N1, int N2>
struct HalfLine {
  static_assert(N2 == 2 * N1, "the half-paired line needs N2 == 2 N1");
  static constexpr int N = N1 * N2;
  static constexpr int H = N1;  // Pairs per thread
};

// a * conj(w) with w = ((wA.x, wB.x), (wA.y, wB.y)): the operations of
// cmul(Pair, conj(wA), conj(wB))
__device__ __forceinline__ Pair cmulc_pp(Pair a, Pair w) {
  return {__ffma2_rn(a.re, w.re, __fmul2_rn(a.im, w.im)),
          __ffma2_rn(a.re, make_float2(-w.im.x, -w.im.y), __fmul2_rn(a.im, w.re))};
}

// Exchange buffer of one line: Pair entry (m, n1) holds rows 2m and 2m + 1 (of the
// N2 rows k2) of column n1 at m * (N1 + 1) + n1, so one 16-byte store and one
// 16-byte load move a Pair between the two stages without repacking; both access
// patterns (m fixed, n1 = lane; n1 fixed, m = lane) put the 8 lanes of each
// quarter-warp phase in distinct banks. It fits in the line's LineBuf region.
template <int N1, int N2>
struct HalfBuf {
  static constexpr int kRow = N1 + 1;
  static_assert(N2 == 2 * N1 && sizeof(Pair) * (N2 / 2) * kRow <= sizeof(float2) * LineBuf<N1, N2>::kSize,
                "the Pair exchange buffer must fit in the line's buffer");
  __device__ static __forceinline__ int at(int m, int n1) { return m * kRow + n1; }
};

// Tables of the half-paired kernel, Pair-shaped so that each lookup is one 16-byte
// load: twiddles twp[m * N1 + t] = (W_N^{2m t}, W_N^{(2m+1) t}) and propagator factors
// pfp[k1 * N1 + t] = (P[2t + N2 k1], P[2t + 1 + N2 k1]), the factors of the k-order
// Pair k1 of thread t.
template <int N1, int N2>
__device__ __forceinline__ void half_tables(const float2* __restrict__ tw_g, const float2* __restrict__ pf_g,
                                            Pair* twp, Pair* pfp) {
  constexpr int N = N1 * N2;
  for (int i = threadIdx.x; i < N / 2; i += blockDim.x) {
    const int m = i / N1, t = i % N1;
    twp[i] = make_pair(tw_g[(t * 2 * m) % N], tw_g[(t * (2 * m + 1)) % N]);
    pfp[i] = make_pair(pf_g[2 * t + N2 * m], pf_g[2 * t + 1 + N2 * m]);
  }
}

// forward, natural (j, j + H) pairs -> k-order Pairs; DIR = -1. Thread t ends with
// Pair k1 = (X[2t + N2 k1], X[2t + 1 + N2 k1]).
template <int N1, int N2, int DIR>
__device__ __forceinline__ void half_nat_to_k(Pair (&p)[N1], int t, Pair* buf, const Pair* twp) {
  using HB = HalfBuf<N1, N2>;
  constexpr int H = N1;
  // decimation in frequency: a_j = x_j + x_{j+H}, b_j = (x_j - x_{j+H}) W_{2H}^j
#pragma unroll
  for (int j = 0; j < H; ++j) {
    const float2 xa = pair_a(p[j]), xb = pair_b(p[j]);
    const float2 a = cadd(xa, xb);
    const float2 b = twmul64<DIR>(csub(xa, xb), j * (64 / (2 * H)));
    p[j] = make_pair(a, b);
  }
  dft<H, DIR, 1, 0, H>(p);  // Pair k = (Y[2k], Y[2k+1])
  // twiddles W_N^{t k2}, k2 = 2k and 2k + 1
  if (t != 0) {
#pragma unroll
    for (int k = 0; k < H; ++k) p[k] = DIR < 0 ? cmul_pp(p[k], twp[k * N1 + t]) : cmulc_pp(p[k], twp[k * N1 + t]);
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < H; ++k) buf[HB::at(k, t)] = p[k];
  __syncwarp();
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) p[n1] = buf[HB::at(t, n1)];  // (Y_{n1}[2t], Y_{n1}[2t+1])
  dft<N1, DIR, 1, 0, N1>(p);
}

// inverse, k-order Pairs -> natural (j, j + H) pairs; DIR = +1
template <int N1, int N2, int DIR>
__device__ __forceinline__ void half_k_to_nat(Pair (&p)[N1], int t, Pair* buf, const Pair* twp) {
  using HB = HalfBuf<N1, N2>;
  constexpr int H = N1;
  dft<N1, DIR, 1, 0, N1>(p);  // Pair n1 = (rows 2t, 2t + 1 of column n1)
  __syncwarp();
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) buf[HB::at(t, n1)] = p[n1];
  __syncwarp();
#pragma unroll
  for (int m = 0; m < H; ++m) p[m] = buf[HB::at(m, t)];
  if (t != 0) {
#pragma unroll
    for (int m = 0; m < H; ++m) p[m] = DIR < 0 ? cmul_pp(p[m], twp[m * N1 + t]) : cmulc_pp(p[m], twp[m * N1 + t]);
  }
  dft<H, DIR, 1, 0, H>(p);  // Pair j = (E_j, O_j): transforms of the even and odd inputs
  // decimation in time: x_j = E_j + W_{2H}^j O_j, x_{j+H} = E_j - W_{2H}^j O_j
#pragma unroll
  for (int j = 0; j < H; ++j) {
    float2 e = pair_a(p[j]), o = pair_b(p[j]);
    bfly<DIR>(e, o, j * (64 / (2 * H)));
    p[j] = make_pair(e, o);
  }
}

// TMA (column passes of 512^2 grids): each warp's block of G columns x N rows comes
// in and goes back as N / 256 tiled TMA copies of 256 rows (wmap: the slots as a 3-D
// tensor (x, y, slot), box G x 256 x 1) through its own exchange buffers, instead of
// the CTA's column tile and its barriers; bounded mbarrier wait as in ms_pair.cuh.
template <int N1, int N2, int AXIS, int WARPS, bool TMA>
__device__ __forceinline__ void half_body(const PassArgs& a, const int slot, const CUtensorMap& wmap) {
  using Geo = PassGeom<N1, N2>;
  using LB = LineBuf<N1, N2>;
  constexpr int N = Geo::N, G = Geo::G, H = N1;
  constexpr int lines = WARPS * G;
  static_assert(N % lines == 0, "lines per CTA must divide N");
  constexpr int pitch = lines + G;
  constexpr int kBoxRows = N < 256 ? N : 256;
  constexpr uint32_t kWarpBytes = sizeof(float2) * G * N;
  static_assert(!TMA || (AXIS == 1 && N % kBoxRows == 0 && (G * 8) % 16 == 0), "TMA moves whole column blocks");
  static_assert(!TMA || sizeof(float2) * G * LB::kSize >= kWarpBytes + 127,
                "the warp's exchange buffers must hold its column block at 128-byte alignment");
  __shared__ __align__(8) uint64_t half_bar[TMA ? WARPS : 1];
  extern __shared__ float2 smem[];
  Pair* twp = reinterpret_cast<Pair*>(smem);          // N / 2 Pairs
  Pair* pfp = reinterpret_cast<Pair*>(smem + N);      // N / 2 Pairs
  float2* work = smem + 2 * N;
  float2* stg = nullptr;  // TMA staging: [row][G]
  uint32_t bar = 0;
  if (TMA) {
    const int wp = threadIdx.x >> 5;
    const uintptr_t base = reinterpret_cast<uintptr_t>(work + (size_t)(wp * G) * LB::kSize);
    stg = reinterpret_cast<float2*>((base + 127) & ~(uintptr_t)127);
    bar = smem_u32(&half_bar[wp]);
    if ((threadIdx.x & 31) == 0) {
      mbar_init(bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      mbar_expect_tx(bar, kWarpBytes);
#pragma unroll
      for (int y = 0; y < N; y += kBoxRows)
        tma_load_3d(smem_u32(stg + (size_t)y * G), &wmap, blockIdx.x * lines + wp * G, y, slot, bar);
    }
  }
  half_tables<N1, N2>(a.tw, a.pf, twp, pfp);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = AXIS == 0 ? (lane % N1) : (lane / G);
  const int gl = AXIS == 0 ? (lane / N1) : (lane % G);
  const int lc = warp * G + gl;
  const int line0 = blockIdx.x * lines;
  const int line = line0 + lc;
  Pair* buf = reinterpret_cast<Pair*>(work + lc * LB::kSize);
  float2* w = a.wave + (size_t)slot * N * N;
  auto off = [&](int e) -> size_t { return AXIS == 0 ? (size_t)line * N + e : (size_t)e * N + line; };
  Pair p[H];

  // ---- load: Pair j = elements t + N1 j and t + N1 (j + H)
  if (AXIS == 0) {
#pragma unroll
    for (int j = 0; j < H; ++j) p[j] = make_pair(w[off(t + N1 * j)], w[off(t + N1 * (j + H))]);
  } else if (TMA) {
    // a warp whose copies never landed leaves its lines untouched (no barrier follows)
    if (!warp_wait_tile(bar, kTileWaitPolls, a.status)) return;
#pragma unroll
    for (int j = 0; j < H; ++j) p[j] = make_pair(stg[(t + N1 * j) * G + gl], stg[(t + N1 * (j + H)) * G + gl]);
  } else {
    tile_load<N, lines, pitch, WARPS * 32>(w, work, line0);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < H; ++j)
      p[j] = make_pair(work[(t + N1 * j) * pitch + lc], work[(t + N1 * (j + H)) * pitch + lc]);
    __syncthreads();
  }

  // ---- finish slice s-1's convolution along this axis
  half_nat_to_k<N1, N2, -1>(p, t, buf, twp);
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) p[k1] = cmul_pp(p[k1], pfp[k1 * N1 + t]);
  half_k_to_nat<N1, N2, +1>(p, t, buf, twp);

  // ---- transmission (and the gradient-mode checkpoint)
  {
    const float4* TH = AXIS == 0 ? a.trans_h : a.trans_ht;
    if (TH != nullptr && a.win == nullptr) {  // one entry holds the factors of both halves
      const float4* row = TH + ((size_t)a.t_slice * N + line) * (N / 2);
#pragma unroll
      for (int j = 0; j < H; ++j) {
        const float4 q = __ldg(row + t + N1 * j);
        p[j] = cmul_pp(p[j], {make_float2(q.x, q.y), make_float2(q.z, q.w)});
      }
    } else {
      int eoff;
      const float2* T = trans_row<AXIS>(a.trans, a.trans_t, a.field_n, a.t_slice, a.win, slot / a.n_modes, line,
                                        &eoff);
      const int fm = a.field_n - 1;
#pragma unroll
      for (int j = 0; j < H; ++j)
        p[j] = cmul(p[j], __ldg(T + ((t + N1 * j + eoff) & fm)), __ldg(T + ((t + N1 * (j + H) + eoff) & fm)));
    }
    if (a.ckpt_store) {
      float2* ck = a.ckpt_store + (size_t)slot * a.res_stride;
#pragma unroll
      for (int j = 0; j < H; ++j) {
        __stcs(ck + off(t + N1 * j), pair_a(p[j]));  // read once, by the adjoint
        __stcs(ck + off(t + N1 * (j + H)), pair_b(p[j]));
      }
    }
  }

  // ---- start slice s's convolution along this axis
  half_nat_to_k<N1, N2, -1>(p, t, buf, twp);
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) p[k1] = cmul_pp(p[k1], pfp[k1 * N1 + t]);
  half_k_to_nat<N1, N2, +1>(p, t, buf, twp);

  // ---- store
  if (AXIS == 0) {
#pragma unroll
    for (int j = 0; j < H; ++j) {
      w[off(t + N1 * j)] = pair_a(p[j]);
      w[off(t + N1 * (j + H))] = pair_b(p[j]);
    }
  } else if (TMA) {
    __syncwarp();  // every lane has read the last exchange
#pragma unroll
    for (int j = 0; j < H; ++j) {
      stg[(t + N1 * j) * G + gl] = pair_a(p[j]);
      stg[(t + N1 * (j + H)) * G + gl] = pair_b(p[j]);
    }
    fence_proxy_async_smem();
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
      for (int y = 0; y < N; y += kBoxRows)
        tma_store_3d(&wmap, line0 + warp * G, y, slot, smem_u32(stg + (size_t)y * G));
      tma_store_wait_read();
    }
  } else {
    __syncthreads();
#pragma unroll
    for (int j = 0; j < H; ++j) {
      work[(t + N1 * j) * pitch + lc] = pair_a(p[j]);
      work[(t + N1 * (j + H)) * pitch + lc] = pair_b(p[j]);
    }
    __syncthreads();
    tile_store<N, lines, pitch, WARPS * 32>(w, work, line0);
  }
}

template <int N1, int N2, int AXIS, int WARPS, int MINB, bool TMA = false>
__global__ void __launch_bounds__(WARPS * 32, MINB)
    ms_pass_half_kernel(PassArgs a, const __grid_constant__ CUtensorMap wmap) {
  half_body<N1, N2, AXIS, WARPS, TMA>(a, blockIdx.y, wmap);
}

// Steady passes of several jobs in one launch (the scheduler's half-paired rows):
// CTA row y works on slot rows[y].y of the job descs[rows[y].x], copied into shared
// memory once per CTA; column passes stage through the CTA's column tile.
template <int N1, int N2, int AXIS, int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB)
    ms_pass_half_multi_kernel(const PassArgs* __restrict__ descs, const int2* __restrict__ rows) {
  __shared__ __align__(16) PassArgs sa;
  const int2 r = rows[blockIdx.y];
  const uint32_t* src = reinterpret_cast<const uint32_t*>(descs + r.x);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&sa);
  for (int i = threadIdx.x; i < (int)(sizeof(PassArgs) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  const CUtensorMap none = {};
  half_body<N1, N2, AXIS, WARPS, false>(sa, r.y, none);
}

}  // namespace ptyro
