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
//
// Row passes (AXIS 0) read and write each line directly: the N1 lanes of a line
// touch consecutive addresses. Column passes (AXIS 1) stage the CTA's block of
// columns through a shared-memory tile so that global traffic moves whole
// row segments (lines-per-CTA x 8 bytes, 128 B at 256^2) in both directions; they
// read the transmission from a transposed copy for the same reason.
#pragma once
#include "fft_core.cuh"

namespace ptyro {

// asynchronous global -> shared copies (completion tracked per thread by groups)
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

enum SrcKind : int { SRC_WAVE = 0, SRC_PROBE = 1 };
enum OpKind : int { OP_NONE = 0, OP_FFT = 1, OP_IFFT = 2, OP_CONV = 3, OP_CONV_CONJ = 4 };
enum DstKind : int { DST_WAVE = 0, DST_PATTERN = 1 };

struct PassArgs {
  float2* wave;            // wave slots, slot w occupies wave[w*N*N, (w+1)*N*N), row-major [y][x]
  const float2* probe_k;   // (M, N, N) spectrum of the beam modes (SRC_PROBE)
  const float2* ramp_y;    // (B, N) shift ramp along y per probe of the batch (SRC_PROBE)
  const float2* ramp_x;    // (B, N) shift ramp along x
  const float2* trans;     // (S, F, F) transmission exp(i sigma V), row-major [y][x]
  const float2* trans_t;   // (S, F, F) the same, transposed [x][y]
  // the same interleaved by line pairs for paired passes, or null: trans_p[s][y/2][x] =
  // (T[2p][x].re, T[2p+1][x].re, T[2p][x].im, T[2p+1][x].im) with p = y/2; trans_pt
  // likewise over column pairs of trans_t
  const float4* trans_p;
  const float4* trans_pt;
  // for half-paired passes (F == N), or null: trans_h[s][y][x] = (T[y][x].re,
  // T[y][x+N/2].re, T[y][x].im, T[y][x+N/2].im) for x < N/2; trans_ht likewise over
  // the transposed table
  const float4* trans_h;
  const float4* trans_ht;
  const int* win;          // (B, 2) window origins (y, x) in the field for this batch, or null
  int field_n;             // F (== N without windows); power of two

  const float2* pf;        // (N) 1-D propagator factor along this axis, already divided by N
  const float2* tw;        // (N) forward twiddles exp(-2 pi i j / N)
  const float2* tw2;       // (N) the same in the (k2, t) order the line transforms read: [k2 * N1 + t]
  float* pattern;          // (B, N, N) fftshifted intensity (DST_PATTERN)
  const float* weights;    // (M) incoherent mode weights (DST_PATTERN)
  int n_modes;
  int src, op1, t_slice, op2, dst;
  int t_conj;              // multiply by conj(T) instead of T
  float scale;             // factor applied after op1 == OP_IFFT
  // gradient-mode residuals (null when not recording): the wave right after the
  // T multiply is stored to ckpt_store (checkpoint plane), and a pattern pass stores
  // the complex far-field amplitude (unshifted, both axes transformed) to amp_store.
  // Plane of slot w: base + w * res_stride.
  float2* ckpt_store;
  float2* amp_store;
  size_t res_stride;
  int accumulate;          // pattern pass adds into the output instead of overwriting it
  // virtual detectors fused into the pattern pass: bit d of det_mask[ky * N + kx]
  // (unshifted frequency order) puts that pixel in detector d; each line's masked
  // intensity sum goes to det_part[(slot * N + line) * n_det + d]. pattern may then
  // be null (no pattern is stored).
  const uint32_t* det_mask;
  float* det_part;
  int n_det;
  int direct;              // column passes: read and write the columns straight from global memory
  // beam tilt per mode: (M, 2, N) complex factors, [m][0][y] and [m][1][x], applied
  // in real space right after the probe's inverse transform completes (the pass with
  // src == SRC_WAVE and op1 == OP_IFFT), or null
  const float2* tilt;
  int amp_shift;           // amp_store receives the fftshifted amplitude with plane stride res_stride
  unsigned int* status;    // the call's device status word (PTYRO_STATUS_* bits), or null
};

template <int N1, int N2>
struct PassGeom {
  static constexpr int N = N1 * N2;
  static constexpr int G = 32 / N1;  // lines per warp
  static_assert(N2 % N1 == 0, "N2 must be a multiple of N1");
  static_assert(32 % N1 == 0, "N1 must divide the warp");
  static constexpr int kWarps = N / G < 8 ? N / G : 8;  // lines per CTA = kWarps * G divides N
  static constexpr int kLines = kWarps * G;
  static int warps_for() { return kWarps; }
  // twiddle table + propagator factor + max(exchange buffers, column tile)
  static size_t smem_bytes(int warps) {
    const size_t lines = (size_t)warps * G;
    const size_t xbuf = lines * LineBuf<N1, N2>::kSize;
    const size_t tile = (size_t)N * (lines + G);
    return sizeof(float2) * ((size_t)2 * N + (xbuf > tile ? xbuf : tile));
  }
  // steady passes also keep the transmission rows of their lines (prefetched)
  static size_t smem_bytes_steady(int warps) { return smem_bytes(warps) + sizeof(float2) * (size_t)warps * G * N; }
};

// Column passes: copy the CTA's block of LINES columns (all N rows) between a plane
// in global memory and the shared staging tile (row pitch PITCH float2). Global
// accesses move LINES consecutive elements per row; loads keep up to 8 per thread
// in flight.
template <int N, int LINES, int PITCH, int THREADS, typename T2>
__device__ __forceinline__ void tile_load(const T2* __restrict__ W, T2* work, int line0) {
  constexpr int kIters = N * LINES / THREADS;
  constexpr int kChunk = kIters < 8 ? kIters : 8;
#pragma unroll 1
  for (int c0 = 0; c0 < kIters; c0 += kChunk) {
    T2 stage[kChunk];
#pragma unroll
    for (int u = 0; u < kChunk; ++u) {
      const int i = threadIdx.x + (c0 + u) * THREADS;
      stage[u] = W[(size_t)(i / LINES) * N + line0 + i % LINES];
    }
#pragma unroll
    for (int u = 0; u < kChunk; ++u) {
      const int i = threadIdx.x + (c0 + u) * THREADS;
      work[(i / LINES) * PITCH + i % LINES] = stage[u];
    }
  }
}

template <int N, int LINES, int PITCH, int THREADS, typename T2>
__device__ __forceinline__ void tile_store(T2* __restrict__ W, const T2* work, int line0) {
  constexpr int kIters = N * LINES / THREADS;
#pragma unroll 8
  for (int it = 0; it < kIters; ++it) {
    const int i = threadIdx.x + it * THREADS;
    W[(size_t)(i / LINES) * N + line0 + i % LINES] = work[(i / LINES) * PITCH + i % LINES];
  }
}

// Transmission row of `line` for a probe whose window starts at (wy, wx) in the
// periodic F x F field; element e of the line is at index (e + off) & (F - 1).
template <int AXIS>
__device__ __forceinline__ const float2* trans_row(const float2* trans, const float2* trans_t, int field_n,
                                                   int t_slice, const int* win, int b, int line, int* off) {
  int wy = 0, wx = 0;
  if (win) {
    wy = win[2 * b];
    wx = win[2 * b + 1];
  }
  const int fm = field_n - 1;
  *off = AXIS == 0 ? wx : wy;
  const float2* T = (AXIS == 0 ? trans : trans_t) + (size_t)t_slice * field_n * field_n;
  return T + (size_t)((line + (AXIS == 0 ? wy : wx)) & fm) * field_n;
}

// op on registers in natural distribution; returns true if the result is k-order.
template <int N1, int N2, typename T>
__device__ __forceinline__ bool apply_op(int op, T (&v)[N2], int t, T* buf, const float2* tw, const float2* pf) {
  if (op == OP_FFT) {
    line_nat_to_k<N1, N2, -1>(v, t, buf, tw);
    return true;
  }
  if (op == OP_CONV || op == OP_CONV_CONJ) {
    line_nat_to_k<N1, N2, -1>(v, t, buf, tw);
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const float2 p = pf[korder_index<N1, N2>(t, r)];
      v[r] = op == OP_CONV ? cmul(v[r], p) : cmulc(v[r], p);
    }
    line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
    return false;
  }
  return false;
}

// The pass on wave slot `yslot` of the job described by `a` (one CTA per
// (line tile, slot); for pattern passes the slot index is the probe index).
// STEADY compiles the program of the middle slices (wave -> conv, x T, conv ->
// wave) in as constants, so the branches of the other programs disappear.
template <int N1, int N2, int AXIS, int WARPS, bool STEADY = false>
__device__ __forceinline__ void pass_body(const PassArgs& a, const int yslot) {
  const int src = STEADY ? (int)SRC_WAVE : a.src;
  const int op1 = STEADY ? (int)OP_CONV : a.op1;
  const int op2 = STEADY ? (int)OP_CONV : a.op2;
  const int dst = STEADY ? (int)DST_WAVE : a.dst;
  const bool has_t = STEADY ? true : a.t_slice >= 0;
  using Geo = PassGeom<N1, N2>;
  using LB = LineBuf<N1, N2>;
  constexpr int N = Geo::N;
  constexpr int G = Geo::G;
  extern __shared__ float2 smem[];
  float2* tw = smem;            // tw[k2 * N1 + t] = W_N^{t k2}
  float2* pfs = smem + N;       // propagator factor along this axis
  float2* work = smem + 2 * N;  // exchange buffers; column passes alias the staging tile here
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int k2 = i / N1, tt = i % N1;
    tw[i] = a.tw[(tt * k2) % N];
    if (a.pf) pfs[i] = a.pf[i];
  }
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = AXIS == 0 ? (lane % N1) : (lane / G);
  const int gl = AXIS == 0 ? (lane / N1) : (lane % G);
  constexpr int lines = WARPS * G;          // lines per CTA (blockDim.x == WARPS * 32); divides N
  static_assert(N % lines == 0, "lines per CTA must divide N");
  constexpr int pitch = lines + G;          // staging-tile row pitch (float2): t*pitch + gl spreads banks
  constexpr int kTileIters = N * lines / (WARPS * 32);
  const int lc = warp * G + gl;             // line within the CTA
  const int line0 = blockIdx.x * lines;
  const int line = line0 + lc;
  float2* buf = work + lc * LB::kSize;
  const size_t NN = (size_t)N * N;
  auto off = [&](int e) -> size_t { return AXIS == 0 ? (size_t)line * N + e : (size_t)e * N + line; };

  // steady passes without windows prefetch their transmission row into shared
  // memory at the start; each thread copies exactly the elements it multiplies, so
  // waiting for its own copies is enough (no barrier)
  constexpr int kWork = (WARPS * G * LB::kSize > N * (WARPS * G + G)) ? WARPS * G * LB::kSize
                                                                     : N * (WARPS * G + G);
  float2* tpre = work + kWork + lc * N;
  const bool pre = STEADY && a.win == nullptr && a.field_n == N;
  if (pre) {
    const float2* Trow = (AXIS == 0 ? a.trans : a.trans_t) + (size_t)a.t_slice * NN + (size_t)line * N;
#pragma unroll
    for (int j = 0; j < N2; ++j) cp_async8(tpre + t + N1 * j, Trow + t + N1 * j);
    cp_async_commit();
  }
  const bool to_pattern = dst == DST_PATTERN;
  const int mcount = to_pattern ? a.n_modes : 1;
  float acc[N2];
#pragma unroll
  for (int r = 0; r < N2; ++r) acc[r] = 0.f;
  bool korder = false;

  for (int m = 0; m < mcount; ++m) {
    const int slot = to_pattern ? yslot * a.n_modes + m : yslot;
    float2* w = a.wave + (size_t)slot * NN;
    float2 v[N2];
    const bool load_k = src == SRC_PROBE || op1 == OP_IFFT;
    // ---- load
    if (src == SRC_PROBE) {
      const int b = yslot / a.n_modes;
      const int mode = yslot % a.n_modes;
      const float2* pk = a.probe_k + (size_t)mode * NN;
      const float2 rl = AXIS == 0 ? a.ramp_y[(size_t)b * N + line] : a.ramp_x[(size_t)b * N + line];
      const float2* ra = (AXIS == 0 ? a.ramp_x : a.ramp_y) + (size_t)b * N;
#pragma unroll
      for (int r = 0; r < N2; ++r) {
        const int k = korder_index<N1, N2>(t, r);
        v[r] = cmul(cmul(pk[off(k)], ra[k]), rl);
      }
    } else if (AXIS == 0 || a.direct) {
      if (load_k) {
#pragma unroll
        for (int r = 0; r < N2; ++r) v[r] = w[off(korder_index<N1, N2>(t, r))];
      } else {
#pragma unroll
        for (int j = 0; j < N2; ++j) v[j] = w[off(t + N1 * j)];
      }
    } else {
      __syncthreads();  // the tile aliases other warps' exchange buffers
      tile_load<N, lines, pitch, WARPS * 32>(w, work, line0);
      __syncthreads();
      if (load_k) {
#pragma unroll
        for (int r = 0; r < N2; ++r) v[r] = work[korder_index<N1, N2>(t, r) * pitch + lc];
      } else {
#pragma unroll
        for (int j = 0; j < N2; ++j) v[j] = work[(t + N1 * j) * pitch + lc];
      }
      __syncthreads();
    }
    korder = load_k;
    // ---- op1
    if (op1 == OP_IFFT) {
      line_k_to_nat<N1, N2, +1>(v, t, buf, tw);
#pragma unroll
      for (int j = 0; j < N2; ++j) v[j] = cscale(v[j], a.scale);
      korder = false;
    } else if (op1 != OP_NONE) {
      korder = apply_op<N1, N2>(op1, v, t, buf, tw, pfs);
    }
    // ---- beam tilt (real space, natural distribution)
    if (!STEADY && a.tilt && src == SRC_WAVE && op1 == OP_IFFT) {
      const float2* ty = a.tilt + (size_t)(slot % a.n_modes) * 2 * N;
      const float2* tx = ty + N;
      const float2 tl = AXIS == 0 ? ty[line] : tx[line];
      const float2* te = AXIS == 0 ? tx : ty;
#pragma unroll
      for (int j = 0; j < N2; ++j) v[j] = cmul(v[j], cmul(te[t + N1 * j], tl));
    }
    // ---- transmission (natural distribution; row-major table for rows, transposed for columns)
    if (has_t) {
      if (pre) {
        cp_async_wait<0>();
#pragma unroll
        for (int j = 0; j < N2; ++j) v[j] = cmul(v[j], tpre[t + N1 * j]);
      } else {
        int eoff;
        const float2* T = trans_row<AXIS>(a.trans, a.trans_t, a.field_n, a.t_slice, a.win, yslot / a.n_modes,
                                          line, &eoff);
        const int fm = a.field_n - 1;
#pragma unroll
        for (int j = 0; j < N2; ++j) {
          const float2 tv = __ldg(T + ((t + N1 * j + eoff) & fm));
          v[j] = a.t_conj ? cmulc(v[j], tv) : cmul(v[j], tv);
        }
      }
      if (a.ckpt_store) {
        float2* ck = a.ckpt_store + (size_t)slot * a.res_stride;
#pragma unroll
        for (int j = 0; j < N2; ++j) __stcs(ck + off(t + N1 * j), v[j]);  // read once, by the adjoint
      }
    }
    // ---- op2
    if (op2 != OP_NONE) korder = apply_op<N1, N2>(op2, v, t, buf, tw, pfs);
    // ---- store
    if (to_pattern) {
      if (a.pattern || a.n_det > 0) {
        const float wm = a.weights[m];
#pragma unroll
        for (int r = 0; r < N2; ++r) acc[r] = fmaf(wm, fmaf(v[r].x, v[r].x, v[r].y * v[r].y), acc[r]);
      }
      if (a.amp_store) {
        float2* am = a.amp_store + (size_t)slot * a.res_stride;
        if (a.amp_shift) {
          const int ls = (line + N / 2) % N;
#pragma unroll
          for (int r = 0; r < N2; ++r) {
            const int ks = (korder_index<N1, N2>(t, r) + N / 2) % N;
            am[AXIS == 0 ? (size_t)ls * N + ks : (size_t)ks * N + ls] = v[r];
          }
        } else {
#pragma unroll
          for (int r = 0; r < N2; ++r) am[off(korder_index<N1, N2>(t, r))] = v[r];
        }
      }
    } else if (AXIS == 0 || a.direct) {
      if (korder) {
#pragma unroll
        for (int r = 0; r < N2; ++r) w[off(korder_index<N1, N2>(t, r))] = v[r];
      } else {
#pragma unroll
        for (int j = 0; j < N2; ++j) w[off(t + N1 * j)] = v[j];
      }
    } else {
      __syncthreads();  // every warp is done with its exchange buffer
      if (korder) {
#pragma unroll
        for (int r = 0; r < N2; ++r) work[korder_index<N1, N2>(t, r) * pitch + lc] = v[r];
      } else {
#pragma unroll
        for (int j = 0; j < N2; ++j) work[(t + N1 * j) * pitch + lc] = v[j];
      }
      __syncthreads();
      tile_store<N, lines, pitch, WARPS * 32>(w, work, line0);
    }
  }
  if (to_pattern && a.n_det > 0) {
    uint32_t mb[N2];
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const int k = korder_index<N1, N2>(t, r);
      mb[r] = __ldg(a.det_mask + (AXIS == 0 ? (size_t)line * N + k : (size_t)k * N + line));
    }
    float* part = a.det_part + ((size_t)yslot * N + line) * a.n_det;
    for (int d = 0; d < a.n_det; ++d) {
      float s = 0.f;
#pragma unroll
      for (int r = 0; r < N2; ++r) s += ((mb[r] >> d) & 1u) ? acc[r] : 0.f;
      // the lanes of one line differ in t: lane % N1 for rows, lane / G for columns
      if (AXIS == 0) {
#pragma unroll
        for (int o = N1 / 2; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      } else {
#pragma unroll
        for (int o = 16; o >= G; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      }
      if (t == 0) part[d] = s;
    }
  }
  if (to_pattern && a.pattern) {
    // fftshift on store: frequency index k lands at (k + N/2) mod N on both axes.
    float* out = a.pattern + (size_t)yslot * NN;
    if (AXIS == 0) {
      const int ls = (line + N / 2) % N;
#pragma unroll
      for (int r = 0; r < N2; ++r) {
        const int ks = (korder_index<N1, N2>(t, r) + N / 2) % N;
        const size_t o = (size_t)ls * N + ks;
        out[o] = a.accumulate ? out[o] + acc[r] : acc[r];
      }
    } else {
      float* tile = reinterpret_cast<float*>(work);
      __syncthreads();
#pragma unroll
      for (int r = 0; r < N2; ++r) tile[korder_index<N1, N2>(t, r) * pitch + lc] = acc[r];
      __syncthreads();
#pragma unroll 8
      for (int it = 0; it < kTileIters; ++it) {
        const int i = threadIdx.x + it * WARPS * 32;
        const int rr = i / lines, c = i % lines;
        const size_t o = (size_t)((rr + N / 2) % N) * N + (line0 + c + N / 2) % N;
        out[o] = a.accumulate ? out[o] + tile[rr * pitch + c] : tile[rr * pitch + c];
      }
    }
  }
}


// MINB: resident CTAs per SM the register allocation must allow (occupancy variant).
template <int N1, int N2, int AXIS, int WARPS, int MINB, bool STEADY = false>
__global__ void __launch_bounds__(WARPS * 32, MINB) ms_pass_kernel(PassArgs a) {
  pass_body<N1, N2, AXIS, WARPS, STEADY>(a, blockIdx.y);
}

// a pass running the middle-slice program (see pass_body's STEADY)
// The first (op1 = IFFT) and last (op2 = FFT) slice passes: wave in, one T multiply,
// wave out, no tilt.
inline bool is_edge_slice_pass(const PassArgs& a) {
  return a.src == SRC_WAVE && a.dst == DST_WAVE && a.t_slice >= 0 && !a.t_conj && a.tilt == nullptr &&
         (a.op1 == OP_IFFT || a.op1 == OP_CONV) && (a.op2 == OP_FFT || a.op2 == OP_CONV) &&
         !(a.op1 == OP_CONV && a.op2 == OP_CONV);
}

inline bool is_steady_pass(const PassArgs& a) {
  return a.src == SRC_WAVE && a.op1 == OP_CONV && a.op2 == OP_CONV && a.dst == DST_WAVE && a.t_slice >= 0 &&
         !a.t_conj;
}

// Passes of several jobs in one launch: CTA row y works on slot rows[y].y of the
// job whose arguments are descs[rows[y].x]. Jobs may differ in potential, probe,
// slice count and progress; they share the grid edge and the axis.
template <int N1, int N2, int AXIS, int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) ms_pass_multi_kernel(const PassArgs* __restrict__ descs,
                                                                         const int2* __restrict__ rows) {
  const int2 r = rows[blockIdx.y];
  pass_body<N1, N2, AXIS, WARPS>(descs[r.x], r.y);
}

}  // namespace ptyro
