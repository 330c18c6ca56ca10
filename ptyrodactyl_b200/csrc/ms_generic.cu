// Multislice forward and adjoint on arbitrary H x W grids (any sizes, square or not,
// powers of two or not), as the reference allows (its fftfreq grids and probe_shape
// take any size: src/ptyrodactyl/multislice/simulations.py:162-225, :334-431).
//
// The fused pass engine (ms_pass.cuh and friends) covers square power-of-two grids
// 16..1024. Everything else runs here, batched over probes but one stage per launch:
//   shift  : psi_k = fft2(beam) * exp(-2 pi i (qy y + qx x))   (phase in double)
//   per s  : psi *= T_s; unless last: psi = ifft2(P * fft2(psi))
//   pattern: sum_m w_m |fftshift(fft2(psi))|^2
// with the 1-D transforms done by a four-step DFT in shared memory: N = N1 N2 (N1 the
// divisor of N nearest sqrt(N)), N1-point DFTs over stride-N2 subsequences, then
// N2-point DFTs with the four-step twiddle folded into one table index (n2 k mod N),
// each a direct sum: N1 + N2 complex multiply-adds per point and transform (a prime N
// becomes one direct N-point DFT). Residuals keep the wave after every slice's T
// multiply and the far-field amplitude; the adjoint runs lambda backward with the same
// stages (conj T, conj P) and adds each slice's dV contribution over the slots in slot
// order (no atomics).
#include <cuda_runtime.h>
#include <math.h>

#include <atomic>
#include <mutex>
#include <string>

#include "../../include/ptyro_b200.h"

namespace ptyro {
extern std::atomic<unsigned long long> g_launches;
void set_error_message(const std::string& msg);

namespace {

constexpr double kPi = 3.14159265358979323846;
// CODATA 2018 (reference: src/ptyrodactyl/types/constants.py:60-96)
constexpr double kH = 6.62607015e-34, kME = 9.1093837015e-31, kE = 1.602176634e-19, kC = 2.99792458e8;

double wavelength(double kv) {
  const double ev = kv * 1000.0 * kE;
  return 1e10 * sqrt(((kH * kH) * (kC * kC)) / (ev * (2.0 * kME * (kC * kC) + ev)));
}
double sigma_of(double kv) {
  const double volt = kv * 1000.0, ev = kE * volt, einstein = kME * (kC * kC);
  return ((2 * kPi / (wavelength(kv) * volt)) * (einstein + ev)) / ((2 * einstein) + ev);
}

int err(int code, const std::string& msg) {
  set_error_message(msg);
  return code;
}
int launched(const char* what, int count = 1) {
  g_launches.fetch_add((unsigned long long)count, std::memory_order_relaxed);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PTYRO_OK : err(PTYRO_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }
unsigned blocks(size_t n, int threads = 256) {
  const size_t b = (n + threads - 1) / threads;
  return (unsigned)(b > 148u * 32u ? 148u * 32u : (b ? b : 1));
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ double fftfreq(int k, int n, double d) {
  return (double)(k <= (n - 1) / 2 ? k : k - n) / (n * d);
}

// ---------------------------------------------------------------- the line transform
// One CTA transforms L lines of length N in place (forward: sign -1, unnormalised;
// inverse: sign +1, scaled by 1/N). Line j of plane p starts at p * plane + j * ls and
// its element e sits e * es further on.
__global__ void k_dft_lines(float2* __restrict__ data, int planes, int lines, long long plane, long long ls,
                            long long es, int N, int N1, int L, int inverse, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  float2* a = sm;                     // [L][N] input
  float2* y = sm + (size_t)L * N;     // [L][N] after the N1-point DFTs, [l][k1 * N2 + n2]
  float2* t = y + (size_t)L * N;      // [N] forward roots exp(-2 pi i j / N)
  const int N2 = N / N1;
  const long long total_lines = (long long)planes * lines;
  const long long l0 = (long long)blockIdx.x * L;
  for (int i = threadIdx.x; i < N; i += blockDim.x) t[i] = tw[i];
  // load: along each line for rows (es == 1), across the L lines of a row for columns,
  // so consecutive threads touch consecutive addresses either way
  const bool along = es == 1;
  for (int i = threadIdx.x; i < L * N; i += blockDim.x) {
    const int e = along ? i % N : i / L, l = along ? i / N : i % L;
    const long long gl = l0 + l;
    if (gl < total_lines) {
      const long long p = gl / lines, j = gl % lines;
      a[(size_t)l * N + e] = data[p * plane + j * ls + (long long)e * es];
    }
  }
  __syncthreads();
  // N1-point DFTs: y[k1 * N2 + n2] = sum_n1 x[N2 n1 + n2] w^(N2 n1 k1)
  for (int i = threadIdx.x; i < L * N; i += blockDim.x) {
    const int l = i / N, r = i % N, k1 = r / N2, n2 = r % N2;
    const float2* x = a + (size_t)l * N;
    float2 acc = make_float2(0.f, 0.f);
    const int step = (int)(((long long)N2 * k1) % N);
    int idx = 0;
    for (int n1 = 0; n1 < N1; ++n1) {
      const float2 w = t[idx];
      const float2 v = x[N2 * n1 + n2];
      const float2 m = inverse ? cmulc(v, w) : cmul(v, w);
      acc.x += m.x;
      acc.y += m.y;
      idx += step;
      if (idx >= N) idx -= N;
    }
    y[(size_t)l * N + r] = acc;
  }
  __syncthreads();
  // N2-point DFTs with the four-step twiddle: X[k] = sum_n2 y[(k mod N1) N2 + n2] w^(n2 k)
  const float scale = inverse ? 1.0f / (float)N : 1.0f;
  for (int i = threadIdx.x; i < L * N; i += blockDim.x) {
    const int l = i / N, k = i % N, k1 = k % N1;
    const float2* yy = y + (size_t)l * N + (size_t)k1 * N2;
    float2 acc = make_float2(0.f, 0.f);
    int idx = 0;
    for (int n2 = 0; n2 < N2; ++n2) {
      const float2 w = t[idx];
      const float2 m = inverse ? cmulc(yy[n2], w) : cmul(yy[n2], w);
      acc.x += m.x;
      acc.y += m.y;
      idx += k;
      if (idx >= N) idx -= N;
    }
    a[(size_t)l * N + k] = make_float2(acc.x * scale, acc.y * scale);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < L * N; i += blockDim.x) {
    const int e = along ? i % N : i / L, l = along ? i / N : i % L;
    const long long gl = l0 + l;
    if (gl < total_lines) {
      const long long p = gl / lines, j = gl % lines;
      data[p * plane + j * ls + (long long)e * es] = a[(size_t)l * N + e];
    }
  }
}

__global__ void k_roots(int n, float2* __restrict__ tw) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double s, c;
  sincospi(-2.0 * (double)j / (double)n, &s, &c);
  tw[j] = make_float2((float)c, (float)s);
}

int divisor_near_sqrt(int n) {
  int best = 1;
  for (int d = 1; (long long)d * d <= n; ++d)
    if (n % d == 0) best = d;
  return best;
}

// Transform `planes` H x W planes along one axis (0: rows of length W, 1: columns of length H).
int dft_axis(float2* data, int planes, int H, int W, int axis, bool inverse, const float2* tw, cudaStream_t st) {
  if (planes <= 0) return PTYRO_OK;
  const int N = axis == 0 ? W : H, lines = axis == 0 ? H : W;
  if (N == 1) return PTYRO_OK;
  const long long ls = axis == 0 ? W : 1, es = axis == 0 ? 1 : W;
  int L = 6144 / N;  // lines per CTA: two [L][N] buffers of 8 bytes stay within 96 KB
  L = L < 1 ? 1 : (L > 32 ? 32 : L);
  const size_t smem = sizeof(float2) * ((size_t)2 * L * N + N);
  static std::once_flag attr[64];  // per device; concurrent callers wait for the first
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64)
    std::call_once(attr[dev], [] {
      cudaFuncSetAttribute(k_dft_lines, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    });
  else
    cudaFuncSetAttribute(k_dft_lines, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  const long long total = (long long)planes * lines;
  k_dft_lines<<<(unsigned)((total + L - 1) / L), 256, smem, st>>>(data, planes, lines, (long long)H * W, ls, es, N,
                                                                  divisor_near_sqrt(N), L, inverse ? 1 : 0, tw);
  return launched("k_dft_lines");
}

int fft2_planes(float2* data, int planes, int H, int W, bool inverse, const float2* twH, const float2* twW,
                cudaStream_t st) {
  int rc = dft_axis(data, planes, H, W, 0, inverse, twW, st);
  if (rc) return rc;
  return dft_axis(data, planes, H, W, 1, inverse, twH, st);
}

// ---------------------------------------------------------------- elementwise stages
__global__ void k_gm_transmission(const float* __restrict__ V, long long sy, long long sx, long long ss, int H,
                                  int W, int S, double sigma, float2* __restrict__ T, int conj_t) {
  const size_t total = (size_t)S * H * W;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / ((size_t)H * W)), y = (int)((i / W) % H), x = (int)(i % W);
    double sn, cs;
    sincos(sigma * (double)V[(long long)y * sy + (long long)x * sx + (long long)s * ss], &sn, &cs);
    T[i] = make_float2((float)cs, (float)(conj_t ? -sn : sn));
  }
}

// propagation_func (simulations.py:213-224): exp(-i pi lambda dz (qy^2 + qx^2)), q = fftfreq
__global__ void k_gm_propagator(int H, int W, double calib, double lam_dz, float2* __restrict__ P) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)H * W) return;
  const double qy = fftfreq((int)(i / W), H, calib), qx = fftfreq((int)(i % W), W, calib);
  double s, c;
  sincos(-kPi * lam_dz * (qx * qx + qy * qy), &s, &c);
  P[i] = make_float2((float)c, (float)s);
}

__global__ void k_gm_gather_modes(const float2* __restrict__ modes, long long sy, long long sx, long long sm, int H,
                                  int W, int M, float2* __restrict__ out) {
  const size_t total = (size_t)M * H * W;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(i / ((size_t)H * W)), y = (int)((i / W) % H), x = (int)(i % W);
    out[i] = modes[(long long)y * sy + (long long)x * sx + (long long)m * sm];
  }
}

// shift_beam_fourier (simulations.py:1282-1321): spectrum times exp(-2 pi i (qy y + qx x)),
// the phase summed in double before its exponential, for slot (b, m) of the batch
__global__ void k_gm_shift(const float2* __restrict__ probe_k, const double* __restrict__ pos, int nb, int M, int H,
                           int W, double calib, float2* __restrict__ wave) {
  const size_t hw = (size_t)H * W, total = (size_t)nb * M * hw;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t slot = i / hw, px = i % hw;
    const int b = (int)(slot / M), m = (int)(slot % M);
    const double qy = fftfreq((int)(px / W), H, calib), qx = fftfreq((int)(px % W), W, calib);
    double s, c;
    sincospi(-2.0 * (qy * pos[2 * b] + qx * pos[2 * b + 1]), &s, &c);
    wave[i] = cmul(probe_k[(size_t)m * hw + px], make_float2((float)c, (float)s));
  }
}

// wave slots times a plane shared by all slots (T_s or P), optionally conjugated; with
// store != null the product is also copied to the slot's residual plane
__global__ void k_gm_mul(float2* __restrict__ wave, size_t slots, size_t hw, const float2* __restrict__ f, int conj_f,
                         float2* __restrict__ store, size_t store_stride) {
  const size_t total = slots * hw;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t px = i % hw;
    const float2 v = conj_f ? cmulc(wave[i], f[px]) : cmul(wave[i], f[px]);
    wave[i] = v;
    if (store) store[(i / hw) * store_stride + px] = v;
  }
}

// sum_m w_m |A|^2, fftshifted (frequency k at (k + n/2) mod n on both axes)
__global__ void k_gm_intensity(const float2* __restrict__ wave, const float* __restrict__ w, int nb, int M, int H,
                               int W, float* __restrict__ out, int accumulate, float2* __restrict__ amp_store,
                               size_t amp_stride) {
  const size_t hw = (size_t)H * W, total = (size_t)nb * hw;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t b = i / hw, px = i % hw;
    const int ky = (int)(px / W), kx = (int)(px % W);
    float acc = 0.f;
    for (int m = 0; m < M; ++m) {
      const float2 a = wave[(b * M + m) * hw + px];
      acc = fmaf(w[m], fmaf(a.x, a.x, a.y * a.y), acc);
      if (amp_store) amp_store[(b * M + m) * amp_stride + px] = a;
    }
    const size_t o = b * hw + (size_t)((ky + H / 2) % H) * W + (kx + W / 2) % W;
    out[o] = accumulate ? out[o] + acc : acc;
  }
}

// ---------------------------------------------------------------- adjoint stages
// lam = H W w_m g(fftshift k) A(k): the cotangent of the far-field amplitude (k-space)
__global__ void k_gm_lam_init(const float2* __restrict__ res, size_t res_stride, size_t amp_off,
                              const float* __restrict__ g, const float* __restrict__ w, int nb, int M, int H, int W,
                              float2* __restrict__ lam) {
  const size_t hw = (size_t)H * W, total = (size_t)nb * M * hw;
  const float hwf = (float)H * (float)W;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t slot = i / hw, px = i % hw;
    const int b = (int)(slot / M), m = (int)(slot % M);
    const int ky = (int)(px / W), kx = (int)(px % W);
    const float2 a = res[slot * res_stride + amp_off + px];
    const float gv = g[(size_t)b * hw + (size_t)((ky + H / 2) % H) * W + (kx + W / 2) % W];
    const float s = hwf * w[m] * gv;
    lam[i] = make_float2(a.x * s, a.y * s);
  }
}

// dV_s(y, x) += sum over the slots, in slot order, of 2 sigma Im(conj(phi_s) lam)
__global__ void k_gm_dv(const float2* __restrict__ res, size_t res_stride, size_t phi_off,
                        const float2* __restrict__ lam, size_t slots, int H, int W, float sigma2, float* __restrict__ dv,
                        long long sy, long long sx, long long ss, int s) {
  const size_t hw = (size_t)H * W;
  const size_t px = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (px >= hw) return;
  float acc = 0.f;
  for (size_t k = 0; k < slots; ++k) {
    const float2 p = res[k * res_stride + phi_off + px], l = lam[k * hw + px];
    acc += sigma2 * (p.x * l.y - p.y * l.x);
  }
  const int y = (int)(px / W), x = (int)(px % W);
  dv[(long long)y * sy + (long long)x * sx + (long long)s * ss] += acc;
}

// G_p = fft2(lam_psi0) conj(R_p) in place (R the shift ramp of k_gm_shift)
__global__ void k_gm_unshift(float2* __restrict__ lam, const double* __restrict__ pos, int nb, int M, int H, int W,
                             double calib) {
  const size_t hw = (size_t)H * W, total = (size_t)nb * M * hw;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t px = i % hw;
    const int b = (int)(i / hw / M);
    const double qy = fftfreq((int)(px / W), H, calib), qx = fftfreq((int)(px % W), W, calib);
    double s, c;
    sincospi(-2.0 * (qy * pos[2 * b] + qx * pos[2 * b + 1]), &s, &c);
    lam[i] = cmulc(lam[i], make_float2((float)c, (float)s));
  }
}

__global__ void k_gm_sum_slots(const float2* __restrict__ g, int nb, int M, size_t hw, float2* __restrict__ acc) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)M * hw) return;
  const size_t m = i / hw, px = i % hw;
  float2 s = acc[i];
  for (int b = 0; b < nb; ++b) {
    const float2 v = g[((size_t)b * M + m) * hw + px];
    s.x += v.x;
    s.y += v.y;
  }
  acc[i] = s;
}

// dL/d(y, x)_p = 4 pi / (H W) sum_k (qy, qx) Im(conj(G_p) B), one CTA per probe
__global__ void __launch_bounds__(256) k_gm_position_grad(const float2* __restrict__ G, const float2* __restrict__ B,
                                                          int M, int H, int W, double calib, double* out) {
  __shared__ double red[8][2];
  const size_t hw = (size_t)H * W;
  const int b = blockIdx.x;
  double sy = 0.0, sx = 0.0;
  for (int m = 0; m < M; ++m) {
    const float2* g = G + ((size_t)b * M + m) * hw;
    const float2* bk = B + (size_t)m * hw;
    for (size_t i = threadIdx.x; i < hw; i += blockDim.x) {
      const double qy = fftfreq((int)(i / W), H, calib), qx = fftfreq((int)(i % W), W, calib);
      const double im = (double)g[i].x * bk[i].y - (double)g[i].y * bk[i].x;
      sy += qy * im;
      sx += qx * im;
    }
  }
  for (int o = 16; o >= 1; o >>= 1) {
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5][0] = sy;
    red[threadIdx.x >> 5][1] = sx;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][threadIdx.x];
    out[2 * (size_t)b + threadIdx.x] = 4.0 * kPi / ((double)H * W) * s;
  }
}

__global__ void k_gm_write_modes(const float2* __restrict__ beam, int H, int W, int M, float2* __restrict__ out,
                                 long long sy, long long sx, long long sm) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)M * H * W) return;
  const int m = (int)(i / ((size_t)H * W)), y = (int)((i / W) % H), x = (int)(i % W);
  out[(long long)y * sy + (long long)x * sx + (long long)m * sm] = make_float2(2.f * beam[i].x, -2.f * beam[i].y);
}

__global__ void k_gm_zero_pot(float* dv, long long sy, long long sx, long long ss, int H, int W, int S) {
  const size_t total = (size_t)S * H * W;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / ((size_t)H * W)), y = (int)((i / W) % H), x = (int)(i % W);
    dv[(long long)y * sy + (long long)x * sx + (long long)s * ss] = 0.f;
  }
}

// ---------------------------------------------------------------- layouts and checks
struct GmLayout {
  size_t status, twH, twW, trans, prop, probe_k, waves, lam, beam, total;
  int batch;
};

GmLayout gm_layout(const ptyro_ms_params* p, int H, int W, bool backward) {
  GmLayout L = {};
  const size_t hw = (size_t)H * W;
  const int M = p->num_modes;
  int b = p->batch > 0 ? p->batch : (int)(64.0 * 1024 * 1024 / (8.0 * hw * M));
  if (b < 1) b = 1;
  if (b > p->num_probes && p->num_probes > 0) b = p->num_probes;
  L.batch = b;
  size_t o = 0;
  L.status = o; o = align_up(o + PTYRO_WS_STATUS_BYTES);
  L.twH = o; o = align_up(o + 8 * (size_t)H);
  L.twW = o; o = align_up(o + 8 * (size_t)W);
  L.trans = o; o = align_up(o + 8 * hw * p->num_slices);
  L.prop = o; o = align_up(o + 8 * hw);
  L.probe_k = o; o = align_up(o + 8 * hw * M);
  L.waves = o; o = align_up(o + 8 * hw * M * (size_t)b);
  if (backward) {
    L.lam = L.waves;  // the adjoint's slots
    L.beam = o; o = align_up(o + 8 * hw * M);
  }
  L.total = o;
  return L;
}

int gm_validate(const ptyro_ms_params* p, int H, int W) {
  if (!p) return err(PTYRO_ERR_INVALID, "params is NULL");
  if (H < 1 || W < 1 || H > 4096 || W > 4096) return err(PTYRO_ERR_INVALID, "grid height and width must be in [1, 4096]");
  if (p->num_slices < 1) return err(PTYRO_ERR_INVALID, "num_slices must be >= 1");
  if (p->num_modes < 1) return err(PTYRO_ERR_INVALID, "num_modes must be >= 1");
  if (p->num_probes < 0) return err(PTYRO_ERR_INVALID, "num_probes must be >= 0");
  if (p->windows || (p->field_n != 0 && !(p->field_n == H && H == W)))
    return err(PTYRO_ERR_UNSUPPORTED, "the any-size path has no potential-field windows");
  if (!(p->voltage_kv > 0) || !(p->calib_ang > 0) || !(p->shift_calib_ang > 0) || !isfinite(p->slice_thickness_ang))
    return err(PTYRO_ERR_INVALID, "voltage, calibrations and slice thickness must be finite and positive");
  return PTYRO_OK;
}

int gm_workspace(const GmLayout& L, void* ws, size_t bytes) {
  if (!ws) return err(PTYRO_ERR_WORKSPACE, "workspace is NULL");
  if (((uintptr_t)ws & 255) != 0) return err(PTYRO_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  if (bytes < L.total)
    return err(PTYRO_ERR_WORKSPACE, "workspace too small: need " + std::to_string(L.total) + " bytes");
  return PTYRO_OK;
}

// twiddles, transmission (conj for the adjoint), propagator (conj for the adjoint)
int gm_setup(const ptyro_ms_params* p, int H, int W, const GmLayout& L, char* ws, const float* V, bool adjoint,
             cudaStream_t st) {
  const double lam = wavelength(p->voltage_kv);
  const size_t hw = (size_t)H * W;
  if (cudaMemsetAsync(ws + L.status, 0, sizeof(unsigned int), st) != cudaSuccess)
    return err(PTYRO_ERR_CUDA, "clearing the status word");
  k_roots<<<(H + 255) / 256, 256, 0, st>>>(H, (float2*)(ws + L.twH));
  k_roots<<<(W + 255) / 256, 256, 0, st>>>(W, (float2*)(ws + L.twW));
  k_gm_transmission<<<blocks(hw * p->num_slices), 256, 0, st>>>(V, p->pot_stride_y, p->pot_stride_x, p->pot_stride_s, H,
                                                                W, p->num_slices, sigma_of(p->voltage_kv),
                                                                (float2*)(ws + L.trans), adjoint ? 1 : 0);
  k_gm_propagator<<<(unsigned)((hw + 255) / 256), 256, 0, st>>>(H, W, p->calib_ang, lam * p->slice_thickness_ang,
                                                                (float2*)(ws + L.prop));
  return launched("any-size setup", 4);
}

int gm_forward(const ptyro_ms_params* p, int H, int W, const float* V, const float* modes, const float* weights,
               const double* positions, float* patterns, float2* residuals, void* workspace, size_t bytes,
               cudaStream_t st) {
  int rc = gm_validate(p, H, W);
  if (rc) return rc;
  if (p->num_probes == 0) return PTYRO_OK;
  if (!V || !modes || !weights || !positions || !patterns) return err(PTYRO_ERR_INVALID, "NULL array argument");
  const GmLayout L = gm_layout(p, H, W, false);
  if ((rc = gm_workspace(L, workspace, bytes))) return rc;
  char* ws = (char*)workspace;
  if ((rc = gm_setup(p, H, W, L, ws, V, false, st))) return rc;
  const int S = p->num_slices, M = p->num_modes;
  const size_t hw = (size_t)H * W;
  const float2 *twH = (const float2*)(ws + L.twH), *twW = (const float2*)(ws + L.twW);
  const float2 *T = (const float2*)(ws + L.trans), *P = (const float2*)(ws + L.prop);
  float2* pk = (float2*)(ws + L.probe_k);
  float2* wave = (float2*)(ws + L.waves);
  k_gm_gather_modes<<<blocks(hw * M), 256, 0, st>>>((const float2*)modes, p->mode_stride_y, p->mode_stride_x,
                                                    p->mode_stride_m, H, W, M, pk);
  if ((rc = launched("k_gm_gather_modes"))) return rc;
  if ((rc = fft2_planes(pk, M, H, W, false, twH, twW, st))) return rc;
  const size_t res_stride = (size_t)(S + 1) * hw;  // (phi_0 .. phi_{S-1}, amplitude) per slot
  for (int b0 = 0; b0 < p->num_probes; b0 += L.batch) {
    const int nb = p->num_probes - b0 < L.batch ? p->num_probes - b0 : L.batch;
    const size_t slots = (size_t)nb * M;
    float2* res = residuals ? residuals + (size_t)b0 * M * res_stride : nullptr;
    k_gm_shift<<<blocks(slots * hw), 256, 0, st>>>(pk, positions + 2 * (size_t)b0, nb, M, H, W, p->shift_calib_ang,
                                                   wave);
    if ((rc = launched("k_gm_shift"))) return rc;
    if ((rc = fft2_planes(wave, (int)slots, H, W, true, twH, twW, st))) return rc;
    for (int s = 0; s < S; ++s) {
      k_gm_mul<<<blocks(slots * hw), 256, 0, st>>>(wave, slots, hw, T + (size_t)s * hw, 0,
                                                   res ? res + (size_t)s * hw : nullptr, res_stride);
      if ((rc = launched("k_gm_mul"))) return rc;
      if (s == S - 1) break;
      if ((rc = fft2_planes(wave, (int)slots, H, W, false, twH, twW, st))) return rc;
      k_gm_mul<<<blocks(slots * hw), 256, 0, st>>>(wave, slots, hw, P, 0, nullptr, 0);
      if ((rc = launched("k_gm_mul"))) return rc;
      if ((rc = fft2_planes(wave, (int)slots, H, W, true, twH, twW, st))) return rc;
    }
    if ((rc = fft2_planes(wave, (int)slots, H, W, false, twH, twW, st))) return rc;
    k_gm_intensity<<<blocks((size_t)nb * hw), 256, 0, st>>>(wave, weights, nb, M, H, W, patterns + (size_t)b0 * hw,
                                                            (p->flags & PTYRO_FLAG_ACCUMULATE) != 0,
                                                            res ? res + (size_t)S * hw : nullptr, res_stride);
    if ((rc = launched("k_gm_intensity"))) return rc;
  }
  return PTYRO_OK;
}

int gm_backward(const ptyro_ms_params* p, int H, int W, const float* V, const float* modes, const float* weights,
                const double* positions, const float2* residuals, const float* g, float* grad_potential,
                float* grad_modes, double* grad_positions, void* workspace, size_t bytes, cudaStream_t st) {
  int rc = gm_validate(p, H, W);
  if (rc) return rc;
  if (!V || !weights || !positions || !grad_potential || !grad_modes || (p->num_probes > 0 && (!residuals || !g)))
    return err(PTYRO_ERR_INVALID, "NULL array argument");
  if (grad_positions && !modes) return err(PTYRO_ERR_INVALID, "position gradients need the beam modes");
  const GmLayout L = gm_layout(p, H, W, true);
  if ((rc = gm_workspace(L, workspace, bytes))) return rc;
  char* ws = (char*)workspace;
  if ((rc = gm_setup(p, H, W, L, ws, V, true, st))) return rc;
  const int S = p->num_slices, M = p->num_modes;
  const size_t hw = (size_t)H * W;
  const float2 *twH = (const float2*)(ws + L.twH), *twW = (const float2*)(ws + L.twW);
  const float2 *Tc = (const float2*)(ws + L.trans), *Pc = (const float2*)(ws + L.prop);
  float2* lam = (float2*)(ws + L.lam);
  float2* beam = (float2*)(ws + L.beam);
  float2* pk = (float2*)(ws + L.probe_k);
  k_gm_zero_pot<<<blocks(hw * S), 256, 0, st>>>(grad_potential, p->pot_stride_y, p->pot_stride_x, p->pot_stride_s, H,
                                                W, S);
  if (cudaMemsetAsync(beam, 0, 8 * hw * M, st) != cudaSuccess) return err(PTYRO_ERR_CUDA, "clearing the beam sum");
  if ((rc = launched("k_gm_zero_pot"))) return rc;
  if (grad_positions) {
    k_gm_gather_modes<<<blocks(hw * M), 256, 0, st>>>((const float2*)modes, p->mode_stride_y, p->mode_stride_x,
                                                      p->mode_stride_m, H, W, M, pk);
    if ((rc = launched("k_gm_gather_modes"))) return rc;
    if ((rc = fft2_planes(pk, M, H, W, false, twH, twW, st))) return rc;
  }
  const float sigma2 = (float)(2.0 * sigma_of(p->voltage_kv));
  const size_t res_stride = (size_t)(S + 1) * hw;
  for (int b0 = 0; b0 < p->num_probes; b0 += L.batch) {
    const int nb = p->num_probes - b0 < L.batch ? p->num_probes - b0 : L.batch;
    const size_t slots = (size_t)nb * M;
    const float2* res = residuals + (size_t)b0 * M * res_stride;
    k_gm_lam_init<<<blocks(slots * hw), 256, 0, st>>>(res, res_stride, (size_t)S * hw, g + (size_t)b0 * hw,
                                                      weights, nb, M, H, W, lam);
    if ((rc = launched("k_gm_lam_init"))) return rc;
    if ((rc = fft2_planes(lam, (int)slots, H, W, true, twH, twW, st))) return rc;  // lambda of phi_{S-1}
    for (int s = S - 1; s >= 0; --s) {
      k_gm_dv<<<(unsigned)((hw + 255) / 256), 256, 0, st>>>(res, res_stride, (size_t)s * hw, lam, slots, H, W,
                                                            sigma2, grad_potential, p->pot_stride_y, p->pot_stride_x,
                                                            p->pot_stride_s, s);
      k_gm_mul<<<blocks(slots * hw), 256, 0, st>>>(lam, slots, hw, Tc + (size_t)s * hw, 0, nullptr, 0);  // conj(T)
      if ((rc = launched("any-size adjoint slice", 2))) return rc;
      if (s == 0) break;
      if ((rc = fft2_planes(lam, (int)slots, H, W, false, twH, twW, st))) return rc;
      k_gm_mul<<<blocks(slots * hw), 256, 0, st>>>(lam, slots, hw, Pc, 1, nullptr, 0);  // conj(P)
      if ((rc = launched("k_gm_mul"))) return rc;
      if ((rc = fft2_planes(lam, (int)slots, H, W, true, twH, twW, st))) return rc;
    }
    // beam: G_p = fft2(lam_psi0) conj(R_p), summed over probes in order
    if ((rc = fft2_planes(lam, (int)slots, H, W, false, twH, twW, st))) return rc;
    k_gm_unshift<<<blocks(slots * hw), 256, 0, st>>>(lam, positions + 2 * (size_t)b0, nb, M, H, W,
                                                     p->shift_calib_ang);
    if ((rc = launched("k_gm_unshift"))) return rc;
    if (grad_positions) {
      k_gm_position_grad<<<nb, 256, 0, st>>>(lam, pk, M, H, W, p->shift_calib_ang, grad_positions + 2 * (size_t)b0);
      if ((rc = launched("k_gm_position_grad"))) return rc;
    }
    k_gm_sum_slots<<<(unsigned)((hw * M + 255) / 256), 256, 0, st>>>(lam, nb, M, hw, beam);
    if ((rc = launched("k_gm_sum_slots"))) return rc;
  }
  // beam gradient = ifft2(sum_p G_p), returned as conj(2 .) (JAX's convention)
  if ((rc = fft2_planes(beam, M, H, W, true, twH, twW, st))) return rc;
  k_gm_write_modes<<<(unsigned)((hw * M + 255) / 256), 256, 0, st>>>(beam, H, W, M, (float2*)grad_modes,
                                                                     p->mode_stride_y, p->mode_stride_x,
                                                                     p->mode_stride_m);
  return launched("k_gm_write_modes");
}

// ---------------------------------------------------------------- forward mode
// The forward with its tangent (ptyro_ms_jvp on any grid): per slot the wave psi and its
// tangent dpsi go through the same slice operators, the tangent picking up the
// potential's tangent at each transmission: dphi = T (dpsi + i sigma dV psi), phi = T psi
// (stem_4d's jvp). Both waves sit in one array (psi planes first, then dpsi planes), so
// every transform runs on all of them at once.
__global__ void k_gm_jvp_slice(float2* __restrict__ wave, float2* __restrict__ dwave, size_t slots, int H, int W,
                               const float2* __restrict__ T, const float* __restrict__ dV, long long sy, long long sx,
                               long long ss, int s, float sigma) {
  const size_t hw = (size_t)H * W, total = slots * hw;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t px = i % hw;
    const float2 t = T[px], v = wave[i];
    float2 d = dwave[i];
    if (dV) {  // dpsi + i sigma dV psi
      const float a = sigma * dV[(long long)(px / W) * sy + (long long)(px % W) * sx + (long long)s * ss];
      d = make_float2(fmaf(-a, v.y, d.x), fmaf(a, v.x, d.y));
    }
    dwave[i] = cmul(d, t);
    wave[i] = cmul(v, t);
  }
}

// I = sum_m w_m |A|^2 and dI = sum_m w_m 2 Re(conj(A) dA), fftshifted like k_gm_intensity
__global__ void k_gm_jvp_out(const float2* __restrict__ wave, const float2* __restrict__ dwave,
                             const float* __restrict__ w, int nb, int M, int H, int W, float* __restrict__ out,
                             float* __restrict__ tangent) {
  const size_t hw = (size_t)H * W, total = (size_t)nb * hw;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t b = i / hw, px = i % hw;
    const int ky = (int)(px / W), kx = (int)(px % W);
    float acc = 0.f, dacc = 0.f;
    for (int m = 0; m < M; ++m) {
      const float2 a = wave[(b * M + m) * hw + px], da = dwave[(b * M + m) * hw + px];
      acc = fmaf(w[m], fmaf(a.x, a.x, a.y * a.y), acc);
      dacc = fmaf(w[m], 2.f * fmaf(a.x, da.x, a.y * da.y), dacc);
    }
    const size_t o = b * hw + (size_t)((ky + H / 2) % H) * W + (kx + W / 2) % W;
    if (out) out[o] = acc;
    tangent[o] = dacc;
  }
}

struct GmJvpLayout {
  GmLayout L;      // status, roots, tables, probe spectra and the batch
  size_t dprobe_k;  // tangent probe spectra (M planes)
  size_t waves2;    // psi and dpsi of the batch's slots
  size_t total;
};

GmJvpLayout gm_jvp_layout(const ptyro_ms_params* p, int H, int W) {
  GmJvpLayout J;
  J.L = gm_layout(p, H, W, false);
  const size_t hw = (size_t)H * W;
  size_t o = J.L.total;
  J.dprobe_k = o; o = align_up(o + 8 * hw * p->num_modes);
  J.waves2 = o; o = align_up(o + 2 * 8 * hw * p->num_modes * (size_t)J.L.batch);
  J.total = o;
  return J;
}

int gm_jvp(const ptyro_ms_params* p, int H, int W, const float* V, const float* dV, const float* modes,
           const float* dmodes, const float* weights, const double* positions, float* patterns, float* tangent,
           void* workspace, size_t bytes, cudaStream_t st) {
  int rc = gm_validate(p, H, W);
  if (rc) return rc;
  if (p->num_probes == 0) return PTYRO_OK;
  if (!V || !modes || !weights || !positions || !tangent) return err(PTYRO_ERR_INVALID, "NULL array argument");
  if (p->flags & PTYRO_FLAG_ACCUMULATE) return err(PTYRO_ERR_INVALID, "the tangent forward does not accumulate");
  const GmJvpLayout J = gm_jvp_layout(p, H, W);
  GmLayout Lw = J.L;
  Lw.total = J.total;
  if ((rc = gm_workspace(Lw, workspace, bytes))) return rc;
  char* ws = (char*)workspace;
  const GmLayout& L = J.L;
  if ((rc = gm_setup(p, H, W, L, ws, V, false, st))) return rc;
  const int S = p->num_slices, M = p->num_modes;
  const size_t hw = (size_t)H * W;
  const float2 *twH = (const float2*)(ws + L.twH), *twW = (const float2*)(ws + L.twW);
  const float2 *T = (const float2*)(ws + L.trans), *P = (const float2*)(ws + L.prop);
  float2* pk = (float2*)(ws + L.probe_k);
  float2* dpk = (float2*)(ws + J.dprobe_k);
  k_gm_gather_modes<<<blocks(hw * M), 256, 0, st>>>((const float2*)modes, p->mode_stride_y, p->mode_stride_x,
                                                    p->mode_stride_m, H, W, M, pk);
  if (dmodes)
    k_gm_gather_modes<<<blocks(hw * M), 256, 0, st>>>((const float2*)dmodes, p->mode_stride_y, p->mode_stride_x,
                                                      p->mode_stride_m, H, W, M, dpk);
  else if (cudaMemsetAsync(dpk, 0, 8 * hw * M, st) != cudaSuccess)
    return err(PTYRO_ERR_CUDA, "clearing the tangent probe spectra");
  if ((rc = launched("k_gm_gather_modes", dmodes ? 2 : 1))) return rc;
  if ((rc = fft2_planes(pk, M, H, W, false, twH, twW, st))) return rc;
  if ((rc = fft2_planes(dpk, M, H, W, false, twH, twW, st))) return rc;
  const float sigma = (float)sigma_of(p->voltage_kv);
  for (int b0 = 0; b0 < p->num_probes; b0 += L.batch) {
    const int nb = p->num_probes - b0 < L.batch ? p->num_probes - b0 : L.batch;
    const size_t slots = (size_t)nb * M;
    float2* wave = (float2*)(ws + J.waves2);
    float2* dwave = wave + slots * hw;  // both waves contiguous: one transform call for all planes
    k_gm_shift<<<blocks(slots * hw), 256, 0, st>>>(pk, positions + 2 * (size_t)b0, nb, M, H, W, p->shift_calib_ang,
                                                   wave);
    k_gm_shift<<<blocks(slots * hw), 256, 0, st>>>(dpk, positions + 2 * (size_t)b0, nb, M, H, W,
                                                   p->shift_calib_ang, dwave);
    if ((rc = launched("k_gm_shift", 2))) return rc;
    if ((rc = fft2_planes(wave, (int)(2 * slots), H, W, true, twH, twW, st))) return rc;
    for (int s = 0; s < S; ++s) {
      k_gm_jvp_slice<<<blocks(slots * hw), 256, 0, st>>>(wave, dwave, slots, H, W, T + (size_t)s * hw, dV,
                                                         p->pot_stride_y, p->pot_stride_x, p->pot_stride_s, s, sigma);
      if ((rc = launched("k_gm_jvp_slice"))) return rc;
      if (s == S - 1) break;
      if ((rc = fft2_planes(wave, (int)(2 * slots), H, W, false, twH, twW, st))) return rc;
      k_gm_mul<<<blocks(2 * slots * hw), 256, 0, st>>>(wave, 2 * slots, hw, P, 0, nullptr, 0);
      if ((rc = launched("k_gm_mul"))) return rc;
      if ((rc = fft2_planes(wave, (int)(2 * slots), H, W, true, twH, twW, st))) return rc;
    }
    if ((rc = fft2_planes(wave, (int)(2 * slots), H, W, false, twH, twW, st))) return rc;
    k_gm_jvp_out<<<blocks((size_t)nb * hw), 256, 0, st>>>(wave, dwave, weights, nb, M, H, W,
                                                          patterns ? patterns + (size_t)b0 * hw : nullptr,
                                                          tangent + (size_t)b0 * hw);
    if ((rc = launched("k_gm_jvp_out"))) return rc;
  }
  return PTYRO_OK;
}

// ---------------------------------------------------------------- make_probe, any shape
// make_probe (simulations.py:395-431) on an H x W grid: the aperture |q| <= alpha/lambda
// times exp(-i chi) on the reference's grid, q along x = (arange(-W/2, W/2) rolled by
// W // 2) / (W 0.01 pm) (likewise y), then ifft2 and ifftshift (roll by -(n // 2)).
__global__ void k_gm_aperture(int H, int W, double fovy, double fovx, double lam, double l_max, double c1, double c3,
                              double c5, float2* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)H * W) return;
  const int y = (int)(i / W), x = (int)(i % W);
  const double lx = (-W / 2.0 + (double)(((x - W / 2) % W + W) % W)) / fovx;
  const double ly = (-H / 2.0 + (double)(((y - H / 2) % H + H) % H)) / fovy;
  const double q = sqrt(lx * lx + ly * ly);
  if (!(q <= l_max)) {
    out[i] = make_float2(0.f, 0.f);
    return;
  }
  const double p = lam * q, p2 = p * p;
  const double chi = ((c1 * p2) / 2) + ((c3 * 1e7 * (p2 * p2)) / 4) + ((c5 * 1e7 * (p2 * p2 * p2)) / 6);
  double s, c;
  sincos(-((2 * kPi * chi) / lam), &s, &c);
  out[i] = make_float2((float)c, (float)s);
}

__global__ void k_gm_ifftshift(const float2* __restrict__ in, int H, int W, float2* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)H * W) return;
  const int y = (int)(i / W), x = (int)(i % W);
  out[i] = in[(size_t)((y + H / 2) % H) * W + (x + W / 2) % W];
}

// ---------------------------------------------------------------- mode-weight gradient
// Each CTA of row m sums a fixed share of the (probe, pixel) terms g |A|^2 in float64 and
// writes one partial; the second kernel adds the partials in order (deterministic).
__global__ void __launch_bounds__(256) k_weight_grad_part(const float2* __restrict__ res, const float* __restrict__ g,
                                                          int P, int M, int H, int W, size_t slot_stride,
                                                          size_t amp_off, double* __restrict__ part) {
  __shared__ double red[8];
  const int m = blockIdx.y;
  const size_t hw = (size_t)H * W, total = (size_t)P * hw;
  double acc = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t pr = i / hw, px = i % hw;
    const int ky = (int)(px / W), kx = (int)(px % W);
    const float2 a = res[(pr * M + m) * slot_stride + amp_off + px];
    const float gv = g[pr * hw + (size_t)((ky + H / 2) % H) * W + (kx + W / 2) % W];
    acc += (double)gv * ((double)a.x * a.x + (double)a.y * a.y);
  }
  for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    part[(size_t)m * gridDim.x + blockIdx.x] = s;
  }
}

__global__ void k_weight_grad_final(const double* __restrict__ part, int blocks, int M, double* out) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  double s = 0.0;
  for (int b = 0; b < blocks; ++b) s += part[(size_t)m * blocks + b];
  out[m] = s;
}

}  // namespace

int weight_grad_hw(int P, int M, int H, int W, size_t slot_stride, size_t amp_off, const float2* res, const float* g,
                   double* out, double* part, int nblocks, cudaStream_t st) {
  k_weight_grad_part<<<dim3(nblocks, M), 256, 0, st>>>(res, g, P, M, H, W, slot_stride, amp_off, part);
  k_weight_grad_final<<<(M + 63) / 64, 64, 0, st>>>(part, nblocks, M, out);
  g_launches.fetch_add(2, std::memory_order_relaxed);
  return cudaGetLastError() == cudaSuccess ? PTYRO_OK : PTYRO_ERR_CUDA;
}
}  // namespace ptyro

extern "C" {

size_t ptyro_gm_fft_workspace_bytes(int32_t height, int32_t width) {
  if (height < 1 || width < 1 || height > 4096 || width > 4096) return 0;
  return ptyro::align_up(8 * (size_t)height) + ptyro::align_up(8 * (size_t)width);
}

int ptyro_gm_fft2(int32_t height, int32_t width, int32_t count, int32_t inverse, float* data, void* workspace,
                  size_t workspace_bytes, void* stream) {
  using namespace ptyro;
  const int H = height, W = width;
  if (H < 1 || W < 1 || H > 4096 || W > 4096) return err(PTYRO_ERR_INVALID, "fft2: height and width must be in [1, 4096]");
  if (count < 0) return err(PTYRO_ERR_INVALID, "fft2: count must be >= 0");
  if (count == 0) return PTYRO_OK;
  if (!data) return err(PTYRO_ERR_INVALID, "fft2: data is NULL");
  if (!workspace || workspace_bytes < ptyro_gm_fft_workspace_bytes(H, W))
    return err(PTYRO_ERR_WORKSPACE, "fft2: workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  float2* twH = (float2*)workspace;
  float2* twW = (float2*)((char*)workspace + align_up(8 * (size_t)H));
  k_roots<<<(H + 255) / 256, 256, 0, st>>>(H, twH);
  k_roots<<<(W + 255) / 256, 256, 0, st>>>(W, twW);
  int rc = launched("fft2 roots", 2);
  if (rc) return rc;
  return fft2_planes((float2*)data, count, H, W, inverse != 0, twH, twW, st);
}

size_t ptyro_gm_make_probe_workspace_bytes(int32_t height, int32_t width) {
  if (height < 1 || width < 1 || height > 4096 || width > 4096) return 0;
  return ptyro::align_up(8 * (size_t)height) + ptyro::align_up(8 * (size_t)width) +
         ptyro::align_up(8 * (size_t)height * width);
}

int ptyro_gm_make_probe(int32_t height, int32_t width, double voltage_kv, double aperture_mrad,
                        double probe_calibration_pm, double defocus_ang, double c3_ang, double c5_ang, float* probe,
                        void* workspace, size_t workspace_bytes, void* stream) {
  using namespace ptyro;
  const int H = height, W = width;
  if (H < 1 || W < 1 || H > 4096 || W > 4096) return err(PTYRO_ERR_INVALID, "probe_shape must be in [1, 4096]^2");
  if (!(voltage_kv > 0)) return err(PTYRO_ERR_INVALID, "voltage_kv must be > 0");
  if (!(aperture_mrad > 0)) return err(PTYRO_ERR_INVALID, "aperture_mrad must be > 0");
  if (!(probe_calibration_pm > 0)) return err(PTYRO_ERR_INVALID, "probe_calibration_pm must be > 0");
  if (!isfinite(defocus_ang) || !isfinite(c3_ang) || !isfinite(c5_ang))
    return err(PTYRO_ERR_INVALID, "aberration coefficients must be finite");
  if (!probe) return err(PTYRO_ERR_INVALID, "make_probe: probe is NULL");
  if (!workspace || workspace_bytes < ptyro_gm_make_probe_workspace_bytes(H, W))
    return err(PTYRO_ERR_WORKSPACE, "make_probe: workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  float2* twH = (float2*)ws;
  float2* twW = (float2*)(ws + align_up(8 * (size_t)H));
  float2* a = (float2*)(ws + align_up(8 * (size_t)H) + align_up(8 * (size_t)W));
  const double lam = wavelength(voltage_kv);
  const size_t hw = (size_t)H * W;
  k_roots<<<(H + 255) / 256, 256, 0, st>>>(H, twH);
  k_roots<<<(W + 255) / 256, 256, 0, st>>>(W, twW);
  k_gm_aperture<<<(unsigned)((hw + 255) / 256), 256, 0, st>>>(H, W, H * 0.01 * probe_calibration_pm,
                                                              W * 0.01 * probe_calibration_pm, lam,
                                                              (aperture_mrad / 1000.0) / lam, defocus_ang, c3_ang,
                                                              c5_ang, a);
  int rc = launched("make_probe setup", 3);
  if (rc) return rc;
  if ((rc = fft2_planes(a, 1, H, W, true, twH, twW, st))) return rc;
  k_gm_ifftshift<<<(unsigned)((hw + 255) / 256), 256, 0, st>>>(a, H, W, (float2*)probe);
  return launched("make_probe ifftshift");
}

size_t ptyro_gm_weight_grad_workspace_bytes(const ptyro_ms_params* p, int32_t height, int32_t width) {
  if (ptyro::gm_validate(p, height, width)) return 0;
  return ptyro::align_up(sizeof(double) * 296 * (size_t)p->num_modes);
}

int ptyro_gm_weight_grad(const ptyro_ms_params* p, int32_t height, int32_t width, const float* residuals,
                         const float* grad_patterns, double* grad_weights, void* workspace, size_t workspace_bytes,
                         void* stream) {
  using namespace ptyro;
  int rc = gm_validate(p, height, width);
  if (rc) return rc;
  if (!grad_weights || (p->num_probes > 0 && (!residuals || !grad_patterns)))
    return err(PTYRO_ERR_INVALID, "NULL array argument");
  if (!workspace || workspace_bytes < ptyro_gm_weight_grad_workspace_bytes(p, height, width))
    return err(PTYRO_ERR_WORKSPACE, "workspace too small for the weight gradient");
  const size_t hw = (size_t)height * width;
  if (p->num_probes == 0)
    return cudaMemsetAsync(grad_weights, 0, 8 * (size_t)p->num_modes, (cudaStream_t)stream) == cudaSuccess
               ? PTYRO_OK : err(PTYRO_ERR_CUDA, "clearing the weight gradient");
  rc = weight_grad_hw(p->num_probes, p->num_modes, height, width, (size_t)(p->num_slices + 1) * hw,
                      (size_t)p->num_slices * hw, (const float2*)residuals, grad_patterns, grad_weights,
                      (double*)workspace, 296, (cudaStream_t)stream);
  return rc ? err(rc, "mode-weight gradient: launch failed") : PTYRO_OK;
}

size_t ptyro_gm_jvp_workspace_bytes(const ptyro_ms_params* p, int32_t height, int32_t width) {
  if (ptyro::gm_validate(p, height, width)) return 0;
  return ptyro::gm_jvp_layout(p, height, width).total;
}

int ptyro_gm_jvp(const ptyro_ms_params* p, int32_t height, int32_t width, const float* potential,
                 const float* tangent_potential, const float* modes, const float* tangent_modes, const float* weights,
                 const double* positions, float* patterns, float* tangent, void* workspace, size_t workspace_bytes,
                 void* stream) {
  return ptyro::gm_jvp(p, height, width, potential, tangent_potential, modes, tangent_modes, weights, positions,
                       patterns, tangent, workspace, workspace_bytes, (cudaStream_t)stream);
}

size_t ptyro_gm_workspace_bytes(const ptyro_ms_params* p, int32_t height, int32_t width) {
  if (ptyro::gm_validate(p, height, width)) return 0;
  return ptyro::gm_layout(p, height, width, false).total;
}

size_t ptyro_gm_residual_bytes(const ptyro_ms_params* p, int32_t height, int32_t width) {
  if (ptyro::gm_validate(p, height, width)) return 0;
  return 8 * (size_t)height * width * (size_t)(p->num_slices + 1) * p->num_modes * (size_t)p->num_probes;
}

int ptyro_gm_forward(const ptyro_ms_params* p, int32_t height, int32_t width, const float* potential,
                     const float* modes, const float* weights, const double* positions, float* patterns,
                     float* residuals, void* workspace, size_t workspace_bytes, void* stream) {
  return ptyro::gm_forward(p, height, width, potential, modes, weights, positions, patterns, (float2*)residuals,
                           workspace, workspace_bytes, (cudaStream_t)stream);
}

size_t ptyro_gm_backward_workspace_bytes(const ptyro_ms_params* p, int32_t height, int32_t width) {
  if (ptyro::gm_validate(p, height, width)) return 0;
  return ptyro::gm_layout(p, height, width, true).total;
}

int ptyro_gm_backward(const ptyro_ms_params* p, int32_t height, int32_t width, const float* potential,
                      const float* modes, const float* weights, const double* positions, const float* residuals,
                      const float* grad_patterns, float* grad_potential, float* grad_modes, double* grad_positions,
                      void* workspace, size_t workspace_bytes, void* stream) {
  return ptyro::gm_backward(p, height, width, potential, modes, weights, positions, (const float2*)residuals,
                            grad_patterns, grad_potential, grad_modes, grad_positions, workspace, workspace_bytes,
                            (cudaStream_t)stream);
}

}  // extern "C"
