// B200 multislice 4D-STEM engine: setup kernels, pass scheduling and the C-ABI
// declared in include/ptyro_b200.h.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include <atomic>
#include <string>

#include "../../include/ptyro_b200.h"
#include "ms_pass.cuh"
#include "pass_launch.cuh"

namespace ptyro {

// ---------------------------------------------------------------- errors
static thread_local std::string g_err;

void set_error_message(const std::string& msg) { g_err = msg; }

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

std::atomic<unsigned long long> g_launches{0};

// Every launch site outside the pass launchers reports through here.
static int check_launch(const char* what, int launches = 1) {
  g_launches.fetch_add((unsigned long long)launches, std::memory_order_relaxed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(PTYRO_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return PTYRO_OK;
}

// ---------------------------------------------------------------- physics scalars
// CODATA 2018 values (reference: src/ptyrodactyl/types/constants.py:60-96)
constexpr double kH = 6.62607015e-34;
constexpr double kME = 9.1093837015e-31;
constexpr double kE = 1.602176634e-19;
constexpr double kC = 2.99792458e8;

// relativistic_wavelength_ang (types/constants.py:291-340)
double wavelength_ang(double kv) {
  const double ev = kv * 1000.0 * kE;
  const double num = (kH * kH) * (kC * kC);
  const double den = ev * (2.0 * kME * (kC * kC) + ev);
  return 1e10 * sqrt(num / den);
}

// interaction constant of transmission_func (multislice/simulations.py:150-157)
double interaction_sigma(double kv) {
  const double volt = kv * 1000.0;
  const double ev = kE * volt;
  const double lam = wavelength_ang(kv);
  const double einstein = kME * (kC * kC);
  return ((2 * M_PI / (lam * volt)) * (einstein + ev)) / ((2 * einstein) + ev);
}

// ---------------------------------------------------------------- setup kernels
__device__ __forceinline__ double fftfreq(int k, int n, double d) {
  return (double)(k <= (n - 1) / 2 ? k : k - n) / (n * d);
}

__global__ void k_twiddle(int n, float2* tw) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double s, c;
  sincospi(-2.0 * (double)j / (double)n, &s, &c);
  tw[j] = make_float2((float)c, (float)s);
}

// 1-D factor of propagation_func (simulations.py:213-224): exp(-i pi lambda dz q^2) * scale
__global__ void k_propagator(int n, double calib, double lam_dz, double scale, float2* pf) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double q = fftfreq(k, n, calib);
  double s, c;
  sincos(-M_PI * lam_dz * q * q, &s, &c);
  pf[k] = make_float2((float)(c * scale), (float)(s * scale));
}

// full 2-D propagator table exp(-i pi lambda dz (qx^2 + qy^2)) for the plain path
__global__ void k_propagator2d(int n, double calib, double lam_dz, float2* p2) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)n * n) return;
  const int y = (int)(i / n), x = (int)(i % n);
  const double qy = fftfreq(y, n, calib), qx = fftfreq(x, n, calib);
  double s, c;
  sincos(-M_PI * lam_dz * (qx * qx + qy * qy), &s, &c);
  p2[i] = make_float2((float)c, (float)s);
}

// transmission_func (simulations.py:105-159): T_s = exp(i sigma V_s), evaluated in
// double and rounded once; written row-major (S, N, N) and transposed (S, N^T).
__global__ void k_transmission(const float* __restrict__ V, long long sy, long long sx, long long ss,
                               int n, int S, double sigma, float2* __restrict__ T, float2* __restrict__ TT) {
  const size_t total = (size_t)S * n * n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / ((size_t)n * n));
    const int y = (int)((i / n) % n);
    const int x = (int)(i % n);
    const double ph = sigma * (double)V[(long long)y * sy + (long long)x * sx + (long long)s * ss];
    double sn, cs;
    sincos(ph, &sn, &cs);
    const float2 v = make_float2((float)cs, (float)sn);
    T[i] = v;
    TT[(size_t)s * n * n + (size_t)x * n + y] = v;
  }
}

// strided beam modes [y][x][m] -> contiguous (M, N, N)
__global__ void k_gather_modes(const float2* __restrict__ modes, long long sy, long long sx, long long sm,
                               int n, int M, float2* __restrict__ out) {
  const size_t total = (size_t)M * n * n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(i / ((size_t)n * n));
    const int y = (int)((i / n) % n);
    const int x = (int)(i % n);
    out[i] = modes[(long long)y * sy + (long long)x * sx + (long long)m * sm];
  }
}

// shift_beam_fourier's ramp (simulations.py:1282-1321), split into its separable
// factors: exp(-2 pi i qy y_p) and exp(-2 pi i qx x_p), q = fftfreq(n, d=calib).
__global__ void k_ramps(const double* __restrict__ pos, int nb, int n, double calib,
                        float2* __restrict__ ry, float2* __restrict__ rx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb * n) return;
  const int b = i / n, k = i % n;
  const double q = fftfreq(k, n, calib);
  double s, c;
  sincospi(-2.0 * q * pos[2 * b + 0], &s, &c);
  ry[i] = make_float2((float)c, (float)s);
  sincospi(-2.0 * q * pos[2 * b + 1], &s, &c);
  rx[i] = make_float2((float)c, (float)s);
}

// make_probe's aperture and aberration (simulations.py:395-427, :491-497) on the
// unshifted grid: a = [|q| <= alpha/lambda] exp(-i chi(|q|)).
__global__ void k_probe_aperture(int n, double fov, double lam, double l_max, double c1, double c3,
                                 double c5, float2* out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)n * n) return;
  const int y = (int)(i / n), x = (int)(i % n);
  const double ly = (double)(y < n / 2 ? y : y - n) / fov;
  const double lx = (double)(x < n / 2 ? x : x - n) / fov;
  const double q = sqrt(lx * lx + ly * ly);
  if (!(q <= l_max)) { out[i] = make_float2(0.f, 0.f); return; }
  const double p = lam * q;
  const double p2 = p * p;
  const double chi = ((c1 * p2) / 2) + ((c3 * 1e7 * (p2 * p2)) / 4) + ((c5 * 1e7 * (p2 * p2 * p2)) / 6);
  const double chi_probe = (2 * M_PI * chi) / lam;
  double s, c;
  sincos(-chi_probe, &s, &c);
  out[i] = make_float2((float)c, (float)s);
}

// in-place fftshift == ifftshift for even n: swap (y, x) with (y+n/2, x+n/2) mod n
__global__ void k_swap_quadrants(int n, int count, float2* data) {
  const size_t half = (size_t)(n / 2) * n;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= half * count) return;
  const size_t plane = i / half, r = i % half;
  const int y = (int)(r / n), x = (int)(r % n);
  float2* d = data + plane * (size_t)n * n;
  const size_t a = (size_t)y * n + x;
  const size_t b = (size_t)(y + n / 2) * n + (x + n / 2) % n;
  const float2 t = d[a];
  d[a] = d[b];
  d[b] = t;
}

// ---- plain-path elementwise kernels (one wave, one stage per launch)
__global__ void k_plain_shift(const float2* __restrict__ pk, const float2* __restrict__ ry,
                              const float2* __restrict__ rx, int n, int M, float2* __restrict__ w) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)M * n * n) return;
  const int y = (int)((i / n) % n), x = (int)(i % n);
  w[i] = cmul(pk[i], cmul(ry[y], rx[x]));
}

__global__ void k_plain_mul_plane(float2* __restrict__ w, const float2* __restrict__ f, int n, int M) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)M * n * n) return;
  w[i] = cmul(w[i], f[i % ((size_t)n * n)]);
}

__global__ void k_plain_intensity(const float2* __restrict__ w, const float* __restrict__ wt, int n, int M,
                                  float* __restrict__ out) {
  const size_t nn = (size_t)n * n;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  float acc = 0.f;
  for (int m = 0; m < M; ++m) {
    const float2 v = w[m * nn + i];
    acc = fmaf(wt[m], fmaf(v.x, v.x, v.y * v.y), acc);
  }
  const int y = (int)(i / n), x = (int)(i % n);
  out[(size_t)((y + n / 2) % n) * n + (x + n / 2) % n] = acc;
}

// ---------------------------------------------------------------- pass dispatch
struct Shape {
  int n1, n2;
};

static bool shape_for(int n, Shape* s) {
  switch (n) {
    case 16: *s = {4, 4}; return true;
    case 32: *s = {4, 8}; return true;
    case 64: *s = {8, 8}; return true;
    case 128: *s = {8, 16}; return true;
    case 256: *s = {16, 16}; return true;
    case 512: *s = {16, 32}; return true;
    case 1024: *s = {32, 32}; return true;
    default: return false;
  }
}

static int launch_pass(int n, int axis, const PassArgs& a, int grid_y, cudaStream_t st, int variant = 0) {
  if (grid_y <= 0) return PTYRO_OK;
  int rc;
  switch (n) {
    case 16: rc = launch_pass_16(axis, a, grid_y, st, variant); break;
    case 32: rc = launch_pass_32(axis, a, grid_y, st, variant); break;
    case 64: rc = launch_pass_64(axis, a, grid_y, st, variant); break;
    case 128: rc = launch_pass_128(axis, a, grid_y, st, variant); break;
    case 256: rc = launch_pass_256(axis, a, grid_y, st, variant); break;
    case 512: rc = launch_pass_512(axis, a, grid_y, st, variant); break;
    case 1024: rc = launch_pass_1024(axis, a, grid_y, st, variant); break;
    default: return fail(PTYRO_ERR_UNSUPPORTED, "grid edge not compiled");
  }
  if (rc != 0) return fail(PTYRO_ERR_CUDA, std::string("ms_pass_kernel: ") + cudaGetErrorString((cudaError_t)rc));
  return PTYRO_OK;
}

// plain 1-D transform passes over `count` planes: fft2 / ifft2 in natural layout
static int fft2_planes(int n, int count, bool inverse, float2* data, const float2* tw, cudaStream_t st) {
  PassArgs a = {};
  a.wave = data;
  a.tw = tw;
  a.n_modes = 1;
  a.src = SRC_WAVE;
  a.op1 = inverse ? OP_IFFT : OP_FFT;
  a.t_slice = -1;
  a.op2 = OP_NONE;
  a.dst = DST_WAVE;
  a.scale = 1.0f / (float)n;
  int rc = launch_pass(n, 0, a, count, st);
  if (rc) return rc;
  return launch_pass(n, 1, a, count, st);
}

// ---------------------------------------------------------------- workspace layout
static size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static int field_of(const ptyro_ms_params* p) { return p->field_n > 0 ? p->field_n : p->n; }

struct Layout {
  size_t tw, pf, trans, trans_t, probe_k, ramp_y, ramp_x, waves, p2, total;
  int batch;
};

static int auto_batch(const ptyro_ms_params* p) {
  // Keep the batch's wave slots near 64 MB so they stay resident in the 126 MB L2.
  const double slot = 8.0 * p->n * (double)p->n * p->num_modes;
  int b = (int)(64.0 * 1024 * 1024 / slot);
  if (b < 1) b = 1;
  if (b > p->num_probes) b = p->num_probes > 0 ? p->num_probes : 1;
  return b;
}

static Layout layout_for(const ptyro_ms_params* p) {
  Layout L = {};
  const size_t nn = (size_t)p->n * p->n;
  L.batch = p->batch > 0 ? (p->batch < p->num_probes ? p->batch : (p->num_probes > 0 ? p->num_probes : 1))
                         : auto_batch(p);
  size_t o = 0;
  L.tw = o; o = align_up(o + 8 * (size_t)p->n);
  L.pf = o; o = align_up(o + 8 * (size_t)p->n);
  const size_t ff = (size_t)field_of(p) * field_of(p);
  L.trans = o; o = align_up(o + 8 * ff * p->num_slices);
  L.trans_t = o; o = align_up(o + 8 * ff * p->num_slices);
  L.probe_k = o; o = align_up(o + 8 * nn * p->num_modes);
  L.ramp_y = o; o = align_up(o + 8 * (size_t)p->n * L.batch);
  L.ramp_x = o; o = align_up(o + 8 * (size_t)p->n * L.batch);
  L.waves = o; o = align_up(o + 8 * nn * p->num_modes * (size_t)L.batch);
  L.p2 = o; o = align_up(o + 8 * nn);  // plain path only
  L.total = o;
  return L;
}


static int validate(const ptyro_ms_params* p) {
  if (!p) return fail(PTYRO_ERR_INVALID, "params is NULL");
  if (p->field_n != 0 && (!is_pow2(p->field_n) || p->field_n < p->n || p->field_n > 8192))
    return fail(PTYRO_ERR_INVALID, "field_n must be 0 or a power of two in [n, 8192]");
  if (!is_pow2(p->n) || p->n < 16 || p->n > 1024)
    return fail(PTYRO_ERR_UNSUPPORTED, "grid edge n must be a power of two in [16, 1024], got " +
                                           std::to_string(p->n));
  if (p->num_slices < 1) return fail(PTYRO_ERR_INVALID, "num_slices must be >= 1");
  if (p->num_modes < 1) return fail(PTYRO_ERR_INVALID, "num_modes must be >= 1");
  if (p->num_probes < 0) return fail(PTYRO_ERR_INVALID, "num_probes must be >= 0");
  if (p->batch < 0) return fail(PTYRO_ERR_INVALID, "batch must be >= 0");
  if (!(p->voltage_kv > 0) || !isfinite(p->voltage_kv)) return fail(PTYRO_ERR_INVALID, "voltage_kv must be > 0");
  if (!(p->slice_thickness_ang > 0) || !isfinite(p->slice_thickness_ang))
    return fail(PTYRO_ERR_INVALID, "slice_thickness must be > 0");
  if (!(p->calib_ang > 0) || !isfinite(p->calib_ang)) return fail(PTYRO_ERR_INVALID, "calib must be > 0");
  if (!(p->shift_calib_ang > 0) || !isfinite(p->shift_calib_ang))
    return fail(PTYRO_ERR_INVALID, "real_space_calib_ang must be > 0");
  if ((size_t)p->num_modes * p->num_probes > 65535u * 16u)
    return fail(PTYRO_ERR_INVALID, "too many probe modes");
  return PTYRO_OK;
}

static int check_workspace(const Layout& L, void* ws, size_t bytes) {
  if (!ws) return fail(PTYRO_ERR_WORKSPACE, "workspace is NULL");
  if (((uintptr_t)ws & 255) != 0) return fail(PTYRO_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  if (bytes < L.total)
    return fail(PTYRO_ERR_WORKSPACE, "workspace too small: need " + std::to_string(L.total) + " bytes, got " +
                                         std::to_string(bytes));
  return PTYRO_OK;
}

static unsigned blocks_for(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  return (unsigned)(b > 148u * 64u ? 148u * 64u : (b ? b : 1));
}

// Everything a forward needs before the probe loop: twiddles, propagator factor,
// transmission table and the beam spectrum.
static int forward_setup(const ptyro_ms_params* p, const Layout& L, char* ws, const float* potential,
                         const float* modes, cudaStream_t st) {
  const int n = p->n;
  const size_t nn = (size_t)n * n;
  float2* tw = (float2*)(ws + L.tw);
  float2* pf = (float2*)(ws + L.pf);
  float2* T = (float2*)(ws + L.trans);
  float2* pk = (float2*)(ws + L.probe_k);
  const double lam = wavelength_ang(p->voltage_kv);
  k_twiddle<<<(n + 255) / 256, 256, 0, st>>>(n, tw);
  k_propagator<<<(n + 255) / 256, 256, 0, st>>>(n, p->calib_ang, lam * p->slice_thickness_ang, 1.0 / n, pf);
  const int F = field_of(p);
  k_transmission<<<blocks_for((size_t)F * F * p->num_slices, 256), 256, 0, st>>>(
      potential, p->pot_stride_y, p->pot_stride_x, p->pot_stride_s, F, p->num_slices,
      interaction_sigma(p->voltage_kv), T, (float2*)(ws + L.trans_t));
  k_gather_modes<<<blocks_for(nn * p->num_modes, 256), 256, 0, st>>>(
      (const float2*)modes, p->mode_stride_y, p->mode_stride_x, p->mode_stride_m, n, p->num_modes, pk);
  int rc = check_launch("forward setup", 4);
  if (rc) return rc;
  return fft2_planes(n, p->num_modes, false, pk, tw, st);
}

// Batched forward over all probes. With residuals != null (gradient mode) every
// pass whose slice point s has s % ckpt_every == 0 also stores the wave after the
// T multiply, and the pattern pass stores the complex far-field amplitude:
// residual planes per (probe, mode) slot = ceil(S / ckpt_every) checkpoints + 1.
static int forward_impl(const ptyro_ms_params* p, int ckpt_every, const float* potential, const float* modes,
                        const float* weights, const double* positions, float* patterns, float2* residuals,
                        void* workspace, size_t workspace_bytes, void* stream) {
  int rc = validate(p);
  if (rc) return rc;
  if (p->num_probes == 0) return PTYRO_OK;
  if (!potential || !modes || !weights || !positions || !patterns)
    return fail(PTYRO_ERR_INVALID, "NULL array argument");
  const Layout L = layout_for(p);
  rc = check_workspace(L, workspace, workspace_bytes);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  rc = forward_setup(p, L, ws, potential, modes, st);
  if (rc) return rc;
  const int n = p->n, S = p->num_slices, M = p->num_modes;
  const size_t nn = (size_t)n * n;
  const int C = residuals ? (S + ckpt_every - 1) / ckpt_every : 0;
  const size_t res_stride = (size_t)(C + 1) * nn;
  float2* ry = (float2*)(ws + L.ramp_y);
  float2* rx = (float2*)(ws + L.ramp_x);
  PassArgs a = {};
  a.wave = (float2*)(ws + L.waves);
  a.probe_k = (const float2*)(ws + L.probe_k);
  a.ramp_y = ry;
  a.ramp_x = rx;
  a.trans = (const float2*)(ws + L.trans);
  a.trans_t = (const float2*)(ws + L.trans_t);
  a.pf = (const float2*)(ws + L.pf);
  a.tw = (const float2*)(ws + L.tw);
  a.weights = weights;
  a.n_modes = M;
  a.scale = 1.0f / (float)n;
  a.res_stride = res_stride;
  a.field_n = field_of(p);
  for (int b0 = 0; b0 < p->num_probes; b0 += L.batch) {
    const int nb = p->num_probes - b0 < L.batch ? p->num_probes - b0 : L.batch;
    float2* res_base = residuals ? residuals + (size_t)b0 * M * res_stride : nullptr;
    a.win = p->windows ? (const int*)p->windows + 2 * (size_t)b0 : nullptr;
    k_ramps<<<(nb * n + 255) / 256, 256, 0, st>>>(positions + 2 * (size_t)b0, nb, n, p->shift_calib_ang, ry, rx);
    if ((rc = check_launch("k_ramps"))) return rc;
    // pass 0: x part of the IFFT2 of the shifted probe spectrum
    PassArgs q = a;
    q.src = SRC_PROBE; q.op1 = OP_IFFT; q.t_slice = -1; q.op2 = OP_NONE; q.dst = DST_WAVE;
    if ((rc = launch_pass(n, 0, q, nb * M, st, p->tune))) return rc;
    for (int k = 1; k <= S; ++k) {
      q = a;
      q.src = SRC_WAVE;
      q.op1 = k == 1 ? OP_IFFT : OP_CONV;
      q.t_slice = k - 1;
      q.op2 = k == S ? OP_FFT : OP_CONV;
      q.dst = DST_WAVE;
      if (res_base && (k - 1) % ckpt_every == 0) q.ckpt_store = res_base + (size_t)((k - 1) / ckpt_every) * nn;
      if ((rc = launch_pass(n, k % 2, q, nb * M, st, p->tune))) return rc;
    }
    q = a;
    q.src = SRC_WAVE; q.op1 = OP_FFT; q.t_slice = -1; q.op2 = OP_NONE; q.dst = DST_PATTERN;
    q.pattern = patterns + (size_t)b0 * nn;
    if (res_base) q.amp_store = res_base + (size_t)C * nn;
    if ((rc = launch_pass(n, (S + 1) % 2, q, nb, st, p->tune))) return rc;
  }
  return PTYRO_OK;
}

// ---------------------------------------------------------------- gradient
__global__ void k_zero_pot(float* dv, long long sy, long long sx, long long ss, int n, int S) {
  const size_t total = (size_t)S * n * n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / ((size_t)n * n)), y = (int)((i / n) % n), x = (int)(i % n);
    dv[(long long)y * sy + (long long)x * sx + (long long)s * ss] = 0.f;
  }
}

__global__ void k_zero2(float2* d, size_t count) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    d[i] = make_float2(0.f, 0.f);
}

// dV_s += sum over slots of the per-slot contributions, in slot order (deterministic).
__global__ void k_reduce_dv(const float* __restrict__ contrib, int nslots, int n, float* dv, long long sy,
                            long long sx, long long ss, int s) {
  const size_t nn = (size_t)n * n;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  float acc = 0.f;
  for (int w = 0; w < nslots; ++w) acc += contrib[(size_t)w * nn + i];
  const int y = (int)(i / n), x = (int)(i % n);
  dv[(long long)y * sy + (long long)x * sx + (long long)s * ss] += acc;
}

// Windowed runs: field pixel (fy, fx) of dV_s collects the contribution of every
// slot whose n x n window (origin modulo F) covers it, added in slot order (no
// atomics). Loads of 8 slots are issued together before they are summed, so a
// thread keeps several reads in flight; neighbouring threads read neighbouring
// pixels of the same slot plane.
constexpr int kReduceWinStaged = 4096;

__global__ void __launch_bounds__(256) k_reduce_dv_win(const float* __restrict__ contrib, int nb, int M, int n,
                                                       int F, const int* __restrict__ win, float* dv, long long sy,
                                                       long long sx, long long ss, int s) {
  extern __shared__ int swin[];
  const bool staged = nb <= kReduceWinStaged;  // window origins in shared memory when they fit
  if (staged)
    for (int i = threadIdx.x; i < 2 * nb; i += blockDim.x) swin[i] = win ? win[i] : 0;
  __syncthreads();
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)F * F) return;
  const int fy = (int)(i / F), fx = (int)(i % F);
  const int fm = F - 1;
  const size_t nn = (size_t)n * n;
  float acc = 0.f;
  for (int b0 = 0; b0 < nb; b0 += 8) {
    float v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int bb = b0 + u;
      v[u] = 0.f;
      if (bb < nb) {
        const int wy = staged ? swin[2 * bb] : (win ? win[2 * bb] : 0);
        const int wx = staged ? swin[2 * bb + 1] : (win ? win[2 * bb + 1] : 0);
        const int ly = (fy - wy) & fm, lx = (fx - wx) & fm;
        if (ly < n && lx < n) {
          const float* cp = contrib + (size_t)bb * M * nn + (size_t)ly * n + lx;
          float t = cp[0];
          for (int m = 1; m < M; ++m) t += cp[(size_t)m * nn];
          v[u] = t;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) acc += v[u];
  }
  dv[(long long)fy * sy + (long long)fx * sx + (long long)s * ss] += acc;
}

static int launch_reduce_dv_win(const float* contrib, int nb, int M, int n, int F, const int* win, float* dv,
                                long long sy, long long sx, long long ss, int s, cudaStream_t st) {
  const size_t ff = (size_t)F * F;
  const size_t smem = nb <= kReduceWinStaged ? 2 * sizeof(int) * (size_t)nb : 0;
  k_reduce_dv_win<<<(unsigned)((ff + 255) / 256), 256, smem, st>>>(
      contrib, nb, M, n, F, win, dv, sy, sx, ss, s);
  return check_launch("k_reduce_dv_win");
}

// beam spectrum gradient: acc[m] += sum_b lam[b*M + m], in probe order.
__global__ void k_reduce_beam(const float2* __restrict__ lam, int nb, int M, int n, float2* acc) {
  const size_t nn = (size_t)n * n;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn * M) return;
  const int m = (int)(i / nn);
  const size_t px = i % nn;
  float2 s = acc[i];
  for (int b = 0; b < nb; ++b) s = cadd(s, lam[((size_t)b * M + m) * nn + px]);
  acc[i] = s;
}

// JAX's gradient convention for a complex input of a real loss: conj(2 dL/dconj(z)).
__global__ void k_write_grad_modes(const float2* __restrict__ lam_beam, int n, int M, float2* out, long long sy,
                                   long long sx, long long sm) {
  const size_t nn = (size_t)n * n;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn * M) return;
  const int m = (int)(i / nn), y = (int)((i % nn) / n), x = (int)(i % n);
  const float2 v = lam_beam[i];
  out[(long long)y * sy + (long long)x * sx + (long long)m * sm] = make_float2(2.f * v.x, -2.f * v.y);
}

struct BwdLayout {
  size_t tw, pf, trans, trans_t, ramp_y, ramp_x, psi, lam, contrib, beam, total;
  int batch;
};

static BwdLayout bwd_layout_for(const ptyro_ms_params* p) {
  BwdLayout L = {};
  const size_t nn = (size_t)p->n * p->n;
  if (p->batch > 0) {
    L.batch = p->batch < p->num_probes ? p->batch : (p->num_probes > 0 ? p->num_probes : 1);
  } else {
    // 64 MiB per wave set (forward + adjoint = 128 MiB): measured faster than an
    // L2-resident 32 MiB set at 256^2 (fewer, fuller launches and reductions)
    int b = (int)(64.0 * 1024 * 1024 / (8.0 * nn * p->num_modes));
    if (b < 1) b = 1;
    L.batch = b > p->num_probes ? (p->num_probes > 0 ? p->num_probes : 1) : b;
  }
  const size_t slots = (size_t)L.batch * p->num_modes;
  size_t o = 0;
  L.tw = o; o = align_up(o + 8 * (size_t)p->n);
  L.pf = o; o = align_up(o + 8 * (size_t)p->n);
  const size_t ff = (size_t)field_of(p) * field_of(p);
  L.trans = o; o = align_up(o + 8 * ff * p->num_slices);
  L.trans_t = o; o = align_up(o + 8 * ff * p->num_slices);
  L.ramp_y = o; o = align_up(o + 8 * (size_t)p->n * L.batch);
  L.ramp_x = o; o = align_up(o + 8 * (size_t)p->n * L.batch);
  L.psi = o; o = align_up(o + 8 * nn * slots);
  L.lam = o; o = align_up(o + 8 * nn * slots);
  L.contrib = o; o = align_up(o + 4 * nn * slots);
  L.beam = o; o = align_up(o + 8 * nn * p->num_modes);
  L.total = o;
  return L;
}

static int launch_bwd(int n, int axis, const BwdArgs& a, int grid_y, cudaStream_t st) {
  if (grid_y <= 0) return PTYRO_OK;
  int rc;
  switch (n) {
    case 16: rc = launch_bwd_16(axis, a, grid_y, st); break;
    case 32: rc = launch_bwd_32(axis, a, grid_y, st); break;
    case 64: rc = launch_bwd_64(axis, a, grid_y, st); break;
    case 128: rc = launch_bwd_128(axis, a, grid_y, st); break;
    case 256: rc = launch_bwd_256(axis, a, grid_y, st); break;
    case 512: rc = launch_bwd_512(axis, a, grid_y, st); break;
    case 1024: rc = launch_bwd_1024(axis, a, grid_y, st); break;
    default: return fail(PTYRO_ERR_UNSUPPORTED, "grid edge not compiled");
  }
  if (rc != 0) return fail(PTYRO_ERR_CUDA, std::string("ms_bwd_pass_kernel: ") + cudaGetErrorString((cudaError_t)rc));
  return PTYRO_OK;
}

static int backward_impl(const ptyro_ms_params* p, int ckpt_every, const float* potential, const float* weights,
                         const double* positions, const float2* residuals, const float* grad_patterns,
                         float* grad_potential, float* grad_modes, void* workspace, size_t workspace_bytes,
                         void* stream) {
  int rc = validate(p);
  if (rc) return rc;
  if (ckpt_every < 1) return fail(PTYRO_ERR_INVALID, "ckpt_every must be >= 1");
  if (!potential || !weights || !positions || !residuals || !grad_patterns || !grad_potential || !grad_modes)
    return fail(PTYRO_ERR_INVALID, "NULL array argument");
  const BwdLayout L = bwd_layout_for(p);
  if (!workspace) return fail(PTYRO_ERR_WORKSPACE, "workspace is NULL");
  if (((uintptr_t)workspace & 255) != 0) return fail(PTYRO_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  if (workspace_bytes < L.total)
    return fail(PTYRO_ERR_WORKSPACE, "workspace too small: need " + std::to_string(L.total) + " bytes, got " +
                                         std::to_string(workspace_bytes));
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  const int n = p->n, S = p->num_slices, M = p->num_modes;
  const size_t nn = (size_t)n * n;
  const int C = (S + ckpt_every - 1) / ckpt_every;
  const size_t res_stride = (size_t)(C + 1) * nn;
  const double lam = wavelength_ang(p->voltage_kv);
  float2* tw = (float2*)(ws + L.tw);
  float2* beam = (float2*)(ws + L.beam);
  k_twiddle<<<(n + 255) / 256, 256, 0, st>>>(n, tw);
  k_propagator<<<(n + 255) / 256, 256, 0, st>>>(n, p->calib_ang, lam * p->slice_thickness_ang, 1.0 / n,
                                                (float2*)(ws + L.pf));
  const int F = field_of(p);
  const bool windowed = p->windows != nullptr || F != n;
  k_transmission<<<blocks_for((size_t)F * F * S, 256), 256, 0, st>>>(potential, p->pot_stride_y, p->pot_stride_x,
                                                                     p->pot_stride_s, F, S,
                                                                     interaction_sigma(p->voltage_kv),
                                                                     (float2*)(ws + L.trans), (float2*)(ws + L.trans_t));
  k_zero_pot<<<blocks_for((size_t)F * F * S, 256), 256, 0, st>>>(grad_potential, p->pot_stride_y, p->pot_stride_x,
                                                                 p->pot_stride_s, F, S);
  k_zero2<<<blocks_for(nn * M, 256), 256, 0, st>>>(beam, nn * M);
  if ((rc = check_launch("backward setup", 5))) return rc;
  BwdArgs a = {};
  a.psi = (float2*)(ws + L.psi);
  a.lam = (float2*)(ws + L.lam);
  a.weights = weights;
  a.res_stride = res_stride;
  a.trans = (const float2*)(ws + L.trans);
  a.trans_t = (const float2*)(ws + L.trans_t);
  a.pf = (const float2*)(ws + L.pf);
  a.tw = tw;
  a.ramp_y = (const float2*)(ws + L.ramp_y);
  a.ramp_x = (const float2*)(ws + L.ramp_x);
  a.n_modes = M;
  a.sigma2 = (float)(2.0 * interaction_sigma(p->voltage_kv));
  a.field_n = F;
  a.scale = 1.0f / (float)n;
  float* contrib = (float*)(ws + L.contrib);
  for (int b0 = 0; b0 < p->num_probes; b0 += L.batch) {
    const int nb = p->num_probes - b0 < L.batch ? p->num_probes - b0 : L.batch;
    const float2* res_base = residuals + (size_t)b0 * M * res_stride;
    const int* win = p->windows ? (const int*)p->windows + 2 * (size_t)b0 : nullptr;
    a.win = win;
    k_ramps<<<(nb * n + 255) / 256, 256, 0, st>>>(positions + 2 * (size_t)b0, nb, n, p->shift_calib_ang,
                                                  (float2*)(ws + L.ramp_y), (float2*)(ws + L.ramp_x));
    if ((rc = check_launch("k_ramps"))) return rc;
    BwdArgs q = a;
    q.init = 1;
    q.amp = res_base + (size_t)C * nn;
    q.gpat = grad_patterns + (size_t)b0 * nn;
    q.op1 = OP_IFFT; q.t_slice = -1; q.op2 = OP_NONE;
    if ((rc = launch_bwd(n, 0, q, nb * M, st))) return rc;
    for (int k = 1; k <= S; ++k) {
      const int s = S - k;
      q = a;
      q.op1 = k == 1 ? OP_IFFT : OP_CONV_CONJ;
      q.t_slice = s;
      q.ckpt = (s % ckpt_every == 0) ? res_base + (size_t)(s / ckpt_every) * nn : nullptr;
      q.contrib = contrib;
      q.op2 = k == S ? OP_FFT : OP_CONV_CONJ;
      q.psi_done = k == S;
      q.beam_epi = k == S;
      if ((rc = launch_bwd(n, k % 2, q, nb * M, st))) return rc;
      if (windowed) {
        if ((rc = launch_reduce_dv_win(contrib, nb, M, n, F, win, grad_potential, p->pot_stride_y,
                                       p->pot_stride_x, p->pot_stride_s, s, st)))
          return rc;
      } else {
        k_reduce_dv<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(contrib, nb * M, n, grad_potential,
                                                                   p->pot_stride_y, p->pot_stride_x, p->pot_stride_s, s);
        if ((rc = check_launch("k_reduce_dv"))) return rc;
      }
    }
    q = a;
    q.op1 = OP_FFT; q.t_slice = -1; q.op2 = OP_NONE; q.psi_done = 1; q.beam_epi = 1;
    if ((rc = launch_bwd(n, (S + 1) % 2, q, nb * M, st))) return rc;
    k_reduce_beam<<<(unsigned)((nn * M + 255) / 256), 256, 0, st>>>(a.lam, nb, M, n, beam);
    if ((rc = check_launch("k_reduce_beam"))) return rc;
  }
  // beam = ifft2(sum_p conj(R_p) fft2(lam_psi0_p)); gradient = conj(2 beam)
  if ((rc = fft2_planes(n, M, true, beam, tw, st))) return rc;
  k_write_grad_modes<<<(unsigned)((nn * M + 255) / 256), 256, 0, st>>>(beam, n, M, (float2*)grad_modes,
                                                                       p->mode_stride_y, p->mode_stride_x,
                                                                       p->mode_stride_m);
  return check_launch("k_write_grad_modes");
}

}  // namespace ptyro

using namespace ptyro;

extern "C" {

int ptyro_version(void) { return 100; }

const char* ptyro_last_error(void) { return g_err.c_str(); }

size_t ptyro_ms_workspace_bytes(const ptyro_ms_params* p) {
  if (validate(p)) return 0;
  return layout_for(p).total;
}

int ptyro_ms_forward(const ptyro_ms_params* p, const float* potential, const float* modes,
                     const float* weights, const double* positions, float* patterns, void* workspace,
                     size_t workspace_bytes, void* stream) {
  return forward_impl(p, 0, potential, modes, weights, positions, patterns, nullptr, workspace, workspace_bytes,
                      stream);
}

size_t ptyro_ms_residual_bytes(const ptyro_ms_params* p, int32_t ckpt_every) {
  if (validate(p) || ckpt_every < 1) return 0;
  const int C = (p->num_slices + ckpt_every - 1) / ckpt_every;
  return 8 * (size_t)p->n * p->n * (size_t)(C + 1) * p->num_modes * (size_t)p->num_probes;
}

size_t ptyro_ms_backward_workspace_bytes(const ptyro_ms_params* p) {
  if (validate(p)) return 0;
  return bwd_layout_for(p).total;
}

int ptyro_ms_forward_ckpt(const ptyro_ms_params* p, int32_t ckpt_every, const float* potential, const float* modes,
                          const float* weights, const double* positions, float* patterns, float* residuals,
                          void* workspace, size_t workspace_bytes, void* stream) {
  if (ckpt_every < 1) return fail(PTYRO_ERR_INVALID, "ckpt_every must be >= 1");
  if (!residuals && p && p->num_probes > 0) return fail(PTYRO_ERR_INVALID, "residuals is NULL");
  return forward_impl(p, ckpt_every, potential, modes, weights, positions, patterns, (float2*)residuals, workspace,
                      workspace_bytes, stream);
}

int ptyro_ms_backward(const ptyro_ms_params* p, int32_t ckpt_every, const float* potential, const float* weights,
                      const double* positions, const float* residuals, const float* grad_patterns,
                      float* grad_potential, float* grad_modes, void* workspace, size_t workspace_bytes,
                      void* stream) {
  return backward_impl(p, ckpt_every, potential, weights, positions, (const float2*)residuals, grad_patterns,
                       grad_potential, grad_modes, workspace, workspace_bytes, stream);
}

int ptyro_ms_forward_plain(const ptyro_ms_params* p, const float* potential, const float* modes,
                           const float* weights, const double* positions, float* patterns, void* workspace,
                           size_t workspace_bytes, void* stream) {
  int rc = validate(p);
  if (rc) return rc;
  if (p->num_probes == 0) return PTYRO_OK;
  if (!potential || !modes || !weights || !positions || !patterns)
    return fail(PTYRO_ERR_INVALID, "NULL array argument");
  if (p->windows || field_of(p) != p->n)
    return fail(PTYRO_ERR_UNSUPPORTED, "the plain per-position path has no windowed mode");
  const Layout L = layout_for(p);
  rc = check_workspace(L, workspace, workspace_bytes);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  rc = forward_setup(p, L, ws, potential, modes, st);
  if (rc) return rc;
  const int n = p->n, S = p->num_slices, M = p->num_modes;
  const size_t nn = (size_t)n * n;
  const double lam = wavelength_ang(p->voltage_kv);
  float2* p2 = (float2*)(ws + L.p2);
  k_propagator2d<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(n, p->calib_ang, lam * p->slice_thickness_ang, p2);
  if ((rc = check_launch("plain propagator table"))) return rc;
  const float2* tw = (const float2*)(ws + L.tw);
  const float2* T = (const float2*)(ws + L.trans);
  const float2* pk = (const float2*)(ws + L.probe_k);
  float2* ry = (float2*)(ws + L.ramp_y);
  float2* rx = (float2*)(ws + L.ramp_x);
  float2* w = (float2*)(ws + L.waves);
  const unsigned eb = (unsigned)((nn * M + 255) / 256);
  for (int i = 0; i < p->num_probes; ++i) {
    k_ramps<<<(n + 255) / 256, 256, 0, st>>>(positions + 2 * (size_t)i, 1, n, p->shift_calib_ang, ry, rx);
    k_plain_shift<<<eb, 256, 0, st>>>(pk, ry, rx, n, M, w);
    if ((rc = check_launch("plain shift", 2))) return rc;
    if ((rc = fft2_planes(n, M, true, w, tw, st))) return rc;
    for (int s = 0; s < S; ++s) {
      k_plain_mul_plane<<<eb, 256, 0, st>>>(w, T + (size_t)s * nn, n, M);
      if ((rc = check_launch("plain transmission"))) return rc;
      if (s == S - 1) break;
      if ((rc = fft2_planes(n, M, false, w, tw, st))) return rc;
      k_plain_mul_plane<<<eb, 256, 0, st>>>(w, p2, n, M);
      if ((rc = check_launch("plain propagator"))) return rc;
      if ((rc = fft2_planes(n, M, true, w, tw, st))) return rc;
    }
    if ((rc = fft2_planes(n, M, false, w, tw, st))) return rc;
    k_plain_intensity<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(w, weights, n, M, patterns + (size_t)i * nn);
    if ((rc = check_launch("plain intensity"))) return rc;
  }
  return PTYRO_OK;
}

unsigned long long ptyro_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int ptyro_ms_steady_pass(const ptyro_ms_params* p, int32_t axis, int32_t reps, void* workspace,
                         size_t workspace_bytes, void* stream) {
  int rc = validate(p);
  if (rc) return rc;
  if (axis != 0 && axis != 1) return fail(PTYRO_ERR_INVALID, "axis must be 0 or 1");
  if (reps < 0) return fail(PTYRO_ERR_INVALID, "reps must be >= 0");
  if (p->num_slices < 2) return fail(PTYRO_ERR_INVALID, "steady pass needs num_slices >= 2");
  const Layout L = layout_for(p);
  if ((rc = check_workspace(L, workspace, workspace_bytes))) return rc;
  char* ws = (char*)workspace;
  PassArgs a = {};
  a.wave = (float2*)(ws + L.waves);
  a.trans = (const float2*)(ws + L.trans);
  a.trans_t = (const float2*)(ws + L.trans_t);
  a.pf = (const float2*)(ws + L.pf);
  a.tw = (const float2*)(ws + L.tw);
  a.n_modes = p->num_modes;
  a.scale = 1.0f / (float)p->n;
  a.src = SRC_WAVE;
  a.op1 = OP_CONV;
  a.t_slice = 1;
  a.op2 = OP_CONV;
  a.dst = DST_WAVE;
  a.field_n = field_of(p);
  for (int r = 0; r < reps; ++r)
    if ((rc = launch_pass(p->n, axis, a, L.batch * p->num_modes, (cudaStream_t)stream, p->tune))) return rc;
  return PTYRO_OK;
}

size_t ptyro_fft_workspace_bytes(int32_t n) { return align_up(8 * (size_t)(n > 0 ? n : 0)); }

int ptyro_fft2(int32_t n, int32_t count, int32_t inverse, float* data, void* workspace, size_t workspace_bytes,
               void* stream) {
  Shape s;
  if (!shape_for(n, &s)) return fail(PTYRO_ERR_UNSUPPORTED, "fft2: n must be a power of two in [16, 1024]");
  if (count < 0) return fail(PTYRO_ERR_INVALID, "fft2: count must be >= 0");
  if (count == 0) return PTYRO_OK;
  if (!data) return fail(PTYRO_ERR_INVALID, "fft2: data is NULL");
  if (!workspace || workspace_bytes < ptyro_fft_workspace_bytes(n))
    return fail(PTYRO_ERR_WORKSPACE, "fft2: workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  float2* tw = (float2*)workspace;
  k_twiddle<<<(n + 255) / 256, 256, 0, st>>>(n, tw);
  int rc = check_launch("k_twiddle");
  if (rc) return rc;
  return fft2_planes(n, count, inverse != 0, (float2*)data, tw, st);
}

int ptyro_make_probe(int32_t n, double voltage_kv, double aperture_mrad, double probe_calibration_pm,
                     double defocus_ang, double c3_ang, double c5_ang, float* probe, void* workspace,
                     size_t workspace_bytes, void* stream) {
  Shape s;
  if (!shape_for(n, &s)) return fail(PTYRO_ERR_UNSUPPORTED, "make_probe: n must be a power of two in [16, 1024]");
  if (!(voltage_kv > 0)) return fail(PTYRO_ERR_INVALID, "voltage_kv must be > 0");
  if (!(aperture_mrad > 0)) return fail(PTYRO_ERR_INVALID, "aperture_mrad must be > 0");
  if (!(probe_calibration_pm > 0)) return fail(PTYRO_ERR_INVALID, "probe_calibration_pm must be > 0");
  if (!isfinite(defocus_ang) || !isfinite(c3_ang) || !isfinite(c5_ang))
    return fail(PTYRO_ERR_INVALID, "aberration coefficients must be finite");
  if (!probe) return fail(PTYRO_ERR_INVALID, "make_probe: probe is NULL");
  if (!workspace || workspace_bytes < ptyro_fft_workspace_bytes(n))
    return fail(PTYRO_ERR_WORKSPACE, "make_probe: workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  const double lam = wavelength_ang(voltage_kv);
  const double l_max = (aperture_mrad / 1000.0) / lam;
  const double fov = n * 0.01 * probe_calibration_pm;
  const size_t nn = (size_t)n * n;
  k_probe_aperture<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(n, fov, lam, l_max, defocus_ang, c3_ang, c5_ang,
                                                                 (float2*)probe);
  float2* tw = (float2*)workspace;
  k_twiddle<<<(n + 255) / 256, 256, 0, st>>>(n, tw);
  int rc = check_launch("make_probe setup", 2);
  if (rc) return rc;
  if ((rc = fft2_planes(n, 1, true, (float2*)probe, tw, st))) return rc;
  k_swap_quadrants<<<(unsigned)((nn / 2 + 255) / 256), 256, 0, st>>>(n, 1, (float2*)probe);
  return check_launch("make_probe ifftshift");
}

}  // extern "C"
