// Register-resident FFT building blocks for the multislice pass kernels (sm_100a).
//
// A line of N = N1 * N2 complex points is owned by N1 threads of one warp.
// "Natural" distribution: thread t holds x[t + N1*j], j in [0, N2).
// "K-order" distribution: thread t holds X[k2 + N2*k1] for k2 = t + N1*g,
//   g in [0, N2/N1), k1 in [0, N1), at register index g*N1 + k1.
// A forward transform maps natural -> k-order with one warp-local exchange
// through shared memory (four-step factorisation: N2-point DFTs, twiddles
// W_N^{t k2}, N1-point DFTs). The inverse maps k-order -> natural by running the
// same steps backwards, so a forward/inverse pair (a Fresnel convolution along
// one axis) returns every value to the thread that loaded it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "unit_consts.cuh"

namespace ptyro {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// Two complex values of two different lines that go through identical arithmetic,
// kept as (real parts, imaginary parts) so that every operation is one paired FP32
// instruction (add / mul / fma .f32x2 on sm_100): the pair costs one issue slot
// where two scalar instructions would cost two. Each paired operation rounds
// exactly like the scalar float2 operation it replaces.
struct alignas(16) Pair {
  float2 re;  // (line A, line B)
  float2 im;
};
__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, dup2(-1.f), a); }
__device__ __forceinline__ Pair cadd(Pair a, Pair b) { return {__fadd2_rn(a.re, b.re), __fadd2_rn(a.im, b.im)}; }
__device__ __forceinline__ Pair csub(Pair a, Pair b) { return {sub2(a.re, b.re), sub2(a.im, b.im)}; }
// a * w with the same w for both lines: (a.x w.x - a.y w.y, a.x w.y + a.y w.x)
__device__ __forceinline__ Pair cmul(Pair a, float2 w) {
  return {__ffma2_rn(a.re, dup2(w.x), __fmul2_rn(a.im, dup2(-w.y))),
          __ffma2_rn(a.re, dup2(w.y), __fmul2_rn(a.im, dup2(w.x)))};
}
// a * conj(w)
__device__ __forceinline__ Pair cmulc(Pair a, float2 w) {
  return {__ffma2_rn(a.re, dup2(w.x), __fmul2_rn(a.im, dup2(w.y))),
          __ffma2_rn(a.im, dup2(w.x), __fmul2_rn(a.re, dup2(-w.y)))};
}
// a * w with a different w per line: (wA, wB)
__device__ __forceinline__ Pair cmul(Pair a, float2 wa, float2 wb) {
  const float2 wx = make_float2(wa.x, wb.x), wy = make_float2(wa.y, wb.y);
  return {__ffma2_rn(a.re, wx, __fmul2_rn(a.im, make_float2(-wa.y, -wb.y))),
          __ffma2_rn(a.re, wy, __fmul2_rn(a.im, wx))};
}
__device__ __forceinline__ Pair cscale(Pair a, float s) { return {__fmul2_rn(a.re, dup2(s)), __fmul2_rn(a.im, dup2(s))}; }
__device__ __forceinline__ Pair make_pair(float2 a, float2 b) { return {make_float2(a.x, b.x), make_float2(a.y, b.y)}; }
__device__ __forceinline__ float2 pair_a(Pair p) { return make_float2(p.re.x, p.im.x); }
__device__ __forceinline__ float2 pair_b(Pair p) { return make_float2(p.re.y, p.im.y); }

// exp(DIR * 2 pi i k / 64) for k in [0, 64); DIR = -1 forward, +1 inverse. The
// first-quadrant values come from unit_consts.cuh (float32 roots chosen so that the
// tables and stages built from them neither gain nor lose energy on average); the
// other quadrants follow by exact rotations by i.
template <int DIR>
__device__ __forceinline__ float2 w64(int k) {
  k &= 63;
  const int q = k >> 4, r = k & 15;
  const float c0 = unit_c(r), s0 = unit_s(r);
  float c, s;
  if (q == 0) { c = c0; s = s0; }
  else if (q == 1) { c = -s0; s = c0; }
  else if (q == 2) { c = -c0; s = -s0; }
  else { c = s0; s = -c0; }
  return make_float2(c, DIR < 0 ? -s : s);
}

// Factored form of W_64^k for the butterflies: w = m (1 + i t) when A is true
// (|cos| >= |sin|), w = m (t + i) otherwise. First-quadrant (m, t) come from
// bfly_m / bfly_t (r <= 8: m ~ cos, t ~ tan; r > 8 uses r' = 16 - r with the roles of
// cos and sin swapped); multiplying by i^q and conjugating (DIR = -1) only moves
// signs between m and t and switches the form.
struct FactTw {
  float m, t;
  bool a;
};
template <int DIR>
__device__ __forceinline__ FactTw fact_tw(int k) {
  k &= 63;
  const int q = k >> 4, r = k & 15;
  FactTw f = r <= 8 ? FactTw{bfly_m(r), bfly_t(r), true} : FactTw{bfly_m(16 - r), bfly_t(16 - r), false};
  for (int i = 0; i < q; ++i) {  // times i: m (1 + i t) -> m (-t + i); m (t + i) -> (-m) (1 - i t)
    if (f.a) f = FactTw{f.m, -f.t, false};
    else f = FactTw{-f.m, -f.t, true};
  }
  if (DIR < 0) {  // conjugate: m (1 - i t) -> form A with -t; m (t - i) = (-m) (-t + i)
    if (f.a) f.t = -f.t;
    else f = FactTw{-f.m, -f.t, false};
  }
  return f;
}

// b * W_64^k (W = exp(DIR 2 pi i / 64)) with the exact cases folded at compile time.
template <int DIR>
__device__ __forceinline__ float2 twmul64(float2 b, int k) {
  k &= 63;
  if (k == 0) return b;
  if (k == 32) return make_float2(-b.x, -b.y);
  if (k == 16) return DIR < 0 ? make_float2(b.y, -b.x) : make_float2(-b.y, b.x);
  if (k == 48) return DIR < 0 ? make_float2(-b.y, b.x) : make_float2(b.y, -b.x);
  return cmul(b, w64<DIR>(k));
}

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }
__host__ __device__ constexpr int bitrev(int i, int bits) {
  return bits == 0 ? 0 : (((i & 1) << (bits - 1)) | bitrev(i >> 1, bits - 1));
}

// Butterflies u +- b W_64^k. The exact twiddles (k = 0, 16, 32, 48) become additions
// of the swapped parts. Every other twiddle is held factored (fact_tw) as
// c (1 + i t) when |c| >= |s| and s (t + i) otherwise, so b w costs two fmas
// and the two outputs u +- (scale) q two more each: six fused operations instead of
// a complex multiply and two complex additions (eight). The scalar and the paired
// versions perform the same operations, so they round identically.
template <int DIR>
__device__ __forceinline__ void bfly(Pair& u, Pair& b, int k) {
  k &= 63;
  Pair o1, o2;
  if (k == 0) {
    o1 = cadd(u, b); o2 = csub(u, b);
  } else if (k == 32) {
    o1 = csub(u, b); o2 = cadd(u, b);
  } else if ((k == 16 && DIR < 0) || (k == 48 && DIR > 0)) {  // w = (b.y, -b.x)
    o1 = {__fadd2_rn(u.re, b.im), sub2(u.im, b.re)};
    o2 = {sub2(u.re, b.im), __fadd2_rn(u.im, b.re)};
  } else if (k == 16 || k == 48) {  // w = (-b.y, b.x)
    o1 = {sub2(u.re, b.im), __fadd2_rn(u.im, b.re)};
    o2 = {__fadd2_rn(u.re, b.im), sub2(u.im, b.re)};
  } else {
    const FactTw f = fact_tw<DIR>(k);
    if (f.a) {  // b w = c (b.re - t b.im, b.im + t b.re)
      const float t = f.t, c = f.m;
      const Pair q = {__ffma2_rn(dup2(-t), b.im, b.re), __ffma2_rn(dup2(t), b.re, b.im)};
      o1 = {__ffma2_rn(dup2(c), q.re, u.re), __ffma2_rn(dup2(c), q.im, u.im)};
      o2 = {__ffma2_rn(dup2(-c), q.re, u.re), __ffma2_rn(dup2(-c), q.im, u.im)};
    } else {  // b w = s (t b.re - b.im, t b.im + b.re), real part kept negated
      const float t = f.t, sn = f.m;
      const Pair q = {__ffma2_rn(dup2(-t), b.re, b.im), __ffma2_rn(dup2(t), b.im, b.re)};
      o1 = {__ffma2_rn(dup2(-sn), q.re, u.re), __ffma2_rn(dup2(sn), q.im, u.im)};
      o2 = {__ffma2_rn(dup2(sn), q.re, u.re), __ffma2_rn(dup2(-sn), q.im, u.im)};
    }
  }
  u = o1;
  b = o2;
}
template <int DIR>
__device__ __forceinline__ void bfly(float2& u, float2& b, int k) {
  k &= 63;
  if (k == 0 || k == 16 || k == 32 || k == 48) {
    const float2 w = twmul64<DIR>(b, k);
    const float2 o1 = cadd(u, w), o2 = csub(u, w);
    u = o1;
    b = o2;
    return;
  }
  const FactTw f = fact_tw<DIR>(k);
  float2 o1, o2;
  if (f.a) {
    const float t = f.t, c = f.m;
    const float2 q = make_float2(fmaf(-t, b.y, b.x), fmaf(t, b.x, b.y));
    o1 = make_float2(fmaf(c, q.x, u.x), fmaf(c, q.y, u.y));
    o2 = make_float2(fmaf(-c, q.x, u.x), fmaf(-c, q.y, u.y));
  } else {
    const float t = f.t, sn = f.m;
    const float2 q = make_float2(fmaf(-t, b.x, b.y), fmaf(t, b.y, b.x));
    o1 = make_float2(fmaf(-sn, q.x, u.x), fmaf(sn, q.y, u.y));
    o2 = make_float2(fmaf(sn, q.x, u.x), fmaf(-sn, q.y, u.y));
  }
  u = o1;
  b = o2;
}

// One radix-2 stage (butterfly span HALF) of an R-point decimation-in-time DFT.
template <int R, int DIR, int HALF, typename T>
__device__ __forceinline__ void dit_stage(T (&t)[R]) {
  constexpr int LEN = 2 * HALF;
  constexpr int TW = 64 / LEN;
#pragma unroll
  for (int i = 0; i < R; i += LEN) {
#pragma unroll
    for (int j = 0; j < HALF; ++j) bfly<DIR>(t[i + j], t[i + j + HALF], j * TW);
  }
  if constexpr (LEN < R) dit_stage<R, DIR, LEN>(t);
}

template <int R>
struct BitRev {
  int v[R];
  constexpr BitRev() : v() {
    for (int i = 0; i < R; ++i) v[i] = bitrev(i, ilog2(R));
  }
};

// In-register DFT of size R (power of two, R <= 64) over a[O + S*i], i in [0,R),
// natural order in and out, unnormalised. Radix-2 decimation in time with every
// index and twiddle resolved at compile time.
template <int R, int DIR, int S, int O, int L, typename T>
__device__ __forceinline__ void dft(T (&a)[L]) {
  static_assert(R >= 1 && R <= 64 && (R & (R - 1)) == 0, "radix must be a power of two <= 64");
  static_assert(O + S * (R - 1) < L, "dft range exceeds register array");
  if constexpr (R == 1) {
    return;
  } else {
    constexpr BitRev<R> br;
    T t[R];
#pragma unroll
    for (int i = 0; i < R; ++i) t[i] = a[O + S * br.v[i]];
    dit_stage<R, DIR, 1>(t);
#pragma unroll
    for (int i = 0; i < R; ++i) a[O + S * i] = t[i];
  }
}

// The N1-point DFTs over each contiguous group g*N1 .. g*N1+N1-1.
template <int N1, int N2, int DIR, int G = 0, typename T>
__device__ __forceinline__ void dft_groups(T (&v)[N2]) {
  if constexpr (G < N2 / N1) {
    dft<N1, DIR, 1, G * N1, N2>(v);
    dft_groups<N1, N2, DIR, G + 1>(v);
  }
}

// Shared-memory exchange buffer of one line: entry (k2, n1) sits at
// k2 * (N1 + 1) + n1 so the strided k-order reads fall in distinct banks; the
// per-line footprint is padded so neighbouring lines start 8 float2 apart mod 16.
template <int N1, int N2>
struct LineBuf {
  static constexpr int kRow = N1 + 1;
  static constexpr int kRaw = N2 * kRow;
  static constexpr int kSize = ((kRaw + 15) / 16) * 16 + 8;
  __device__ static __forceinline__ int at(int k2, int n1) { return k2 * kRow + n1; }
};

// natural -> k-order transform of one line, unnormalised. DIR = -1 forward.
// tw[k2 * N1 + t] = exp(-2 pi i t k2 / N) (shared memory; lanes of one k2 read
// consecutive entries, so the table is read without bank conflicts).
template <int N1, int N2, int DIR, typename T>
__device__ __forceinline__ void line_nat_to_k(T (&v)[N2], int t, T* buf, const float2* tw) {
  using LB = LineBuf<N1, N2>;
  dft<N2, DIR, 1, 0, N2>(v);
  if (t != 0) {
#pragma unroll
    for (int k2 = 1; k2 < N2; ++k2) {
      const float2 w = tw[k2 * N1 + t];
      v[k2] = DIR < 0 ? cmul(v[k2], w) : cmulc(v[k2], w);
    }
  }
  __syncwarp();
#pragma unroll
  for (int k2 = 0; k2 < N2; ++k2) buf[LB::at(k2, t)] = v[k2];
  __syncwarp();
#pragma unroll
  for (int g = 0; g < N2 / N1; ++g)
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[g * N1 + n1] = buf[LB::at(t + N1 * g, n1)];
  dft_groups<N1, N2, DIR>(v);
}

// k-order -> natural transform of one line, unnormalised. DIR = +1 inverse.
template <int N1, int N2, int DIR, typename T>
__device__ __forceinline__ void line_k_to_nat(T (&v)[N2], int t, T* buf, const float2* tw) {
  using LB = LineBuf<N1, N2>;
  dft_groups<N1, N2, DIR>(v);
  __syncwarp();
#pragma unroll
  for (int g = 0; g < N2 / N1; ++g)
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) buf[LB::at(t + N1 * g, n1)] = v[g * N1 + n1];
  __syncwarp();
#pragma unroll
  for (int k2 = 0; k2 < N2; ++k2) v[k2] = buf[LB::at(k2, t)];
  if (t != 0) {
#pragma unroll
    for (int k2 = 1; k2 < N2; ++k2) {
      const float2 w = tw[k2 * N1 + t];
      v[k2] = DIR < 0 ? cmul(v[k2], w) : cmulc(v[k2], w);
    }
  }
  dft<N2, DIR, 1, 0, N2>(v);
}

// k-order register index r -> frequency index along the line.
template <int N1, int N2>
__device__ __forceinline__ int korder_index(int t, int r) {
  const int g = r / N1, k1 = r % N1;
  return (t + N1 * g) + N2 * k1;
}

}  // namespace ptyro
