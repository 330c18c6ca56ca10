// Internals of the B200 multislice engine shared by its translation units
// (ms_engine.cu: the C-ABI; ms_sched.cu: the multi-job scheduler): physics
// scalars, setup and reduction kernels, workspace layouts and the forward and
// adjoint drivers. Everything here has internal linkage except the error state
// and the launch counter, which are defined once in ms_engine.cu.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include <atomic>
#include <string>

#include "../../include/ptyro_b200.h"
#include "ms_pass.cuh"
#include "ms_resident.cuh"
#include "pass_launch.cuh"

namespace ptyro {

// ---------------------------------------------------------------- errors
extern thread_local std::string g_err;

void set_error_message(const std::string& msg);

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}


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
static double wavelength_ang(double kv) {
  const double ev = kv * 1000.0 * kE;
  const double num = (kH * kH) * (kC * kC);
  const double den = ev * (2.0 * kME * (kC * kC) + ev);
  return 1e10 * sqrt(num / den);
}

// interaction constant of transmission_func (multislice/simulations.py:150-157)
static double interaction_sigma(double kv) {
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

// exp(-2 pi i j / n) in float32. Entries at multiples of n / 64 are 64th roots of
// unity and take the energy-balanced constants of the butterflies (w64); every other
// entry is evaluated in double and rounded to nearest.
__device__ __forceinline__ float2 unit_root(int j, int n) {
  if ((j * 64) % n == 0) return w64<-1>((j * 64) / n);
  double s, c;
  sincospi(-2.0 * (double)j / (double)n, &s, &c);
  return make_float2((float)c, (float)s);
}

static __global__ void k_twiddle(int n, float2* tw) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  tw[j] = unit_root(j, n);
}

// twiddles in line-transform order: tw2[k2 * n1 + t] = exp(-2 pi i t k2 / n)
static __global__ void k_twiddle2(int n, int n1, float2* tw2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k2 = i / n1, t = i % n1;
  tw2[i] = unit_root((t * k2) % n, n);
}

// 1-D factor of propagation_func (simulations.py:213-224): exp(-i pi lambda dz q^2) * scale
static __global__ void k_propagator(int n, double calib, double lam_dz, double scale, float2* pf) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double q = fftfreq(k, n, calib);
  double s, c;
  sincos(-M_PI * lam_dz * q * q, &s, &c);
  pf[k] = make_float2((float)(c * scale), (float)(s * scale));
}

// full 2-D propagator table exp(-i pi lambda dz (qx^2 + qy^2)) for the plain path
static __global__ void k_propagator2d(int n, double calib, double lam_dz, float2* p2) {
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
static __global__ void k_transmission(const float* __restrict__ V, long long sy, long long sx, long long ss,
                               int n, int S, double sigma, float2* __restrict__ T, float2* __restrict__ TT,
                               float* __restrict__ TP = nullptr, float* __restrict__ TPT = nullptr,
                               float* __restrict__ TH = nullptr, float* __restrict__ THT = nullptr) {
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
    if (TP) {  // line-pair interleaved copies: component (line & 1) holds re, 2 + (line & 1) im
      const size_t pr = (((size_t)s * (n / 2) + (size_t)(y >> 1)) * n + x) * 4 + (y & 1);
      TP[pr] = v.x;
      TP[pr + 2] = v.y;
      const size_t pc = (((size_t)s * (n / 2) + (size_t)(x >> 1)) * n + y) * 4 + (x & 1);
      TPT[pc] = v.x;
      TPT[pc + 2] = v.y;
    }
    if (TH) {  // half-pair interleaved copies: component (element >= n/2) holds re, 2 + it im
      const int h = n / 2;
      const size_t hr = (((size_t)s * n + y) * h + (x % h)) * 4 + (x >= h);
      TH[hr] = v.x;
      TH[hr + 2] = v.y;
      const size_t hc = (((size_t)s * n + x) * h + (y % h)) * 4 + (y >= h);
      THT[hc] = v.x;
      THT[hc + 2] = v.y;
    }
  }
}

// strided beam modes [y][x][m] -> contiguous (M, N, N)
static __global__ void k_gather_modes(const float2* __restrict__ modes, long long sy, long long sx, long long sm,
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
static __global__ void k_ramps(const double* __restrict__ pos, int nb, int n, double calib,
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
static __global__ void k_probe_aperture(int n, double fov, double lam, double l_max, double c1, double c3,
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
static __global__ void k_swap_quadrants(int n, int count, float2* data) {
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
static __global__ void k_plain_shift(const float2* __restrict__ pk, const float2* __restrict__ ry,
                              const float2* __restrict__ rx, int n, int M, float2* __restrict__ w) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)M * n * n) return;
  const int y = (int)((i / n) % n), x = (int)(i % n);
  w[i] = cmul(pk[i], cmul(ry[y], rx[x]));
}

static __global__ void k_plain_mul_plane(float2* __restrict__ w, const float2* __restrict__ f, int n, int M) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)M * n * n) return;
  w[i] = cmul(w[i], f[i % ((size_t)n * n)]);
}

static __global__ void k_plain_intensity(const float2* __restrict__ w, const float* __restrict__ wt, int n, int M,
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

// ptyro_ms_params.tune bit of the wave-resident kernel (ms_resident.cuh)
constexpr int kTuneResident = 32768;
// tune bit: keep the lockstep adjoint (psi and lambda together) even when every slice
// point has a checkpoint, instead of the lambda-only pass (ms_bwd_lam.cuh)
constexpr int kTuneLockstepAdjoint = 65536;

static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static int field_of(const ptyro_ms_params* p) { return p->field_n > 0 ? p->field_n : p->n; }

struct Layout {
  size_t status, tw, tw2, pf, trans, trans_t, trans_p, trans_pt, trans_h, trans_ht, probe_k, ramp_y, ramp_x, waves, p2,
      total;
  int batch;
  bool paired_t;  // line-pair interleaved transmission tables present (tune bit 16384 at 256^2)
  bool half_t;    // half-pair interleaved tables present (tune bit 16384 at 512^2 without a field)
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
  L.status = o; o = align_up(o + PTYRO_WS_STATUS_BYTES);  // the call's device status word
  L.tw = o; o = align_up(o + 8 * (size_t)p->n);
  L.tw2 = o; o = align_up(o + 8 * (size_t)p->n);
  L.pf = o; o = align_up(o + 8 * (size_t)p->n);
  const size_t ff = (size_t)field_of(p) * field_of(p);
  L.trans = o; o = align_up(o + 8 * ff * p->num_slices);
  L.trans_t = o; o = align_up(o + 8 * ff * p->num_slices);
  L.paired_t = p->n == 256 && (p->tune & 16384) && (p->tune & 16) && (p->tune & 64);
  if (L.paired_t) {
    L.trans_p = o; o = align_up(o + 8 * ff * p->num_slices);
    L.trans_pt = o; o = align_up(o + 8 * ff * p->num_slices);
  }
  L.half_t = p->n == 512 && field_of(p) == p->n && (p->tune & 16384) && (p->tune & 256);
  if (L.half_t) {
    L.trans_h = o; o = align_up(o + 8 * ff * p->num_slices);
    L.trans_ht = o; o = align_up(o + 8 * ff * p->num_slices);
  }
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

// Zero the call's device status word (a memset node when the stream is being captured).
static int clear_status(void* status, cudaStream_t st) {
  const cudaError_t e = cudaMemsetAsync(status, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return fail(PTYRO_ERR_CUDA, std::string("clearing the status word: ") + cudaGetErrorString(e));
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
  Shape sh;
  shape_for(n, &sh);
  k_twiddle<<<(n + 255) / 256, 256, 0, st>>>(n, tw);
  k_twiddle2<<<(n + 255) / 256, 256, 0, st>>>(n, sh.n1, (float2*)(ws + L.tw2));
  k_propagator<<<(n + 255) / 256, 256, 0, st>>>(n, p->calib_ang, lam * p->slice_thickness_ang, 1.0 / n, pf);
  const int F = field_of(p);
  k_transmission<<<blocks_for((size_t)F * F * p->num_slices, 256), 256, 0, st>>>(
      potential, p->pot_stride_y, p->pot_stride_x, p->pot_stride_s, F, p->num_slices,
      interaction_sigma(p->voltage_kv), T, (float2*)(ws + L.trans_t),
      L.paired_t ? (float*)(ws + L.trans_p) : nullptr, L.paired_t ? (float*)(ws + L.trans_pt) : nullptr,
      L.half_t ? (float*)(ws + L.trans_h) : nullptr, L.half_t ? (float*)(ws + L.trans_ht) : nullptr);
  k_gather_modes<<<blocks_for(nn * p->num_modes, 256), 256, 0, st>>>(
      (const float2*)modes, p->mode_stride_y, p->mode_stride_x, p->mode_stride_m, n, p->num_modes, pk);
  int rc = check_launch("forward setup", 5);
  if (rc) return rc;
  return fft2_planes(n, p->num_modes, false, pk, tw, st);
}

// Arguments of forward pass k (0 .. S+1) for the probe batch [b0, b0 + nb).
struct FwdPlan {
  PassArgs a;
  int axis;
  int rows;  // CTA rows: wave slots, or probes for the pattern pass
};

struct FwdBuffers {
  unsigned int* status;
  float2* waves;
  const float2* probe_k;
  const float2 *ramp_y, *ramp_x, *trans, *trans_t, *pf, *tw, *tw2;
  const float4 *trans_p, *trans_pt;  // or null
  const float4 *trans_h, *trans_ht;  // or null
};

static FwdBuffers fwd_buffers(const Layout& L, char* ws) {
  FwdBuffers b;
  b.status = (unsigned int*)(ws + L.status);
  b.waves = (float2*)(ws + L.waves);
  b.probe_k = (const float2*)(ws + L.probe_k);
  b.ramp_y = (const float2*)(ws + L.ramp_y);
  b.ramp_x = (const float2*)(ws + L.ramp_x);
  b.trans = (const float2*)(ws + L.trans);
  b.trans_t = (const float2*)(ws + L.trans_t);
  b.pf = (const float2*)(ws + L.pf);
  b.tw = (const float2*)(ws + L.tw);
  b.tw2 = (const float2*)(ws + L.tw2);
  b.trans_p = L.paired_t ? (const float4*)(ws + L.trans_p) : nullptr;
  b.trans_pt = L.paired_t ? (const float4*)(ws + L.trans_pt) : nullptr;
  b.trans_h = L.half_t ? (const float4*)(ws + L.trans_h) : nullptr;
  b.trans_ht = L.half_t ? (const float4*)(ws + L.trans_ht) : nullptr;
  return b;
}

// Virtual detectors of a forward: the mask (n, n), the detector count and the
// per-line partial sums (batch, n, n_det) the pattern pass writes.
struct DetOut {
  const uint32_t* mask;
  int n_det;
  float* part;
  double* out;  // (P, n_det)
};

// Optional extras of a forward: beam tilts (M, 2, n) applied after the probe's
// inverse transform, and fftshifted amplitudes (P, M, n, n) stored by the pattern pass.
struct FwdExtras {
  const float2* tilt;
  float2* amplitudes;
};

static FwdPlan fwd_pass_plan(const ptyro_ms_params* p, const FwdBuffers& B, const float* weights, float* patterns,
                             float2* res_base, int ckpt_every, int C, int b0, int nb, int k,
                             const DetOut* det = nullptr, const FwdExtras* ex = nullptr) {
  const int n = p->n, S = p->num_slices, M = p->num_modes;
  const size_t nn = (size_t)n * n;
  FwdPlan r;
  PassArgs& a = r.a;
  a = PassArgs{};
  a.status = B.status;
  a.wave = B.waves;
  a.probe_k = B.probe_k;
  a.ramp_y = B.ramp_y;
  a.ramp_x = B.ramp_x;
  a.trans = B.trans;
  a.trans_t = B.trans_t;
  a.trans_p = B.trans_p;
  a.trans_pt = B.trans_pt;
  a.trans_h = B.trans_h;
  a.trans_ht = B.trans_ht;
  a.pf = B.pf;
  a.tw = B.tw;
  a.tw2 = B.tw2;
  a.weights = weights;
  a.n_modes = M;
  a.scale = 1.0f / (float)n;
  a.res_stride = (size_t)(C + 1) * nn;
  a.field_n = field_of(p);
  a.win = p->windows ? (const int*)p->windows + 2 * (size_t)b0 : nullptr;
  if (k == 0) {  // x part of the IFFT2 of the shifted probe spectrum
    a.src = SRC_PROBE; a.op1 = OP_IFFT; a.t_slice = -1; a.op2 = OP_NONE; a.dst = DST_WAVE;
    r.axis = 0;
    r.rows = nb * M;
  } else if (k <= S) {
    a.src = SRC_WAVE;
    a.op1 = k == 1 ? OP_IFFT : OP_CONV;
    a.t_slice = k - 1;
    a.op2 = k == S ? OP_FFT : OP_CONV;
    a.dst = DST_WAVE;
    if (res_base && (k - 1) % ckpt_every == 0) a.ckpt_store = res_base + (size_t)((k - 1) / ckpt_every) * nn;
    if (ex && k == 1) a.tilt = ex->tilt;
    r.axis = k % 2;
    r.rows = nb * M;
  } else {  // last axis of the FFT2, |.|^2, fftshifted store
    a.src = SRC_WAVE; a.op1 = OP_FFT; a.t_slice = -1; a.op2 = OP_NONE; a.dst = DST_PATTERN;
    a.pattern = patterns ? patterns + (size_t)b0 * nn : nullptr;
    a.accumulate = (p->flags & PTYRO_FLAG_ACCUMULATE) != 0;
    if (det && det->n_det > 0) {
      a.det_mask = det->mask;
      a.det_part = det->part;
      a.n_det = det->n_det;
    }
    if (res_base) a.amp_store = res_base + (size_t)C * nn;
    if (ex && ex->amplitudes) {
      a.amp_store = ex->amplitudes + (size_t)b0 * M * nn;
      a.res_stride = nn;
      a.amp_shift = 1;
    }
    r.axis = (S + 1) % 2;
    r.rows = nb;
  }
  return r;
}

// Batched forward over all probes. With residuals != null (gradient mode) every
// pass whose slice point s has s % ckpt_every == 0 also stores the wave after the
// T multiply, and the pattern pass stores the complex far-field amplitude:
// residual planes per (probe, mode) slot = ceil(S / ckpt_every) checkpoints + 1.
// Detector sums of `nb` probes: out[b][d] (+)= sum over the n line partials, in
// line order (deterministic).
static __global__ void k_det_reduce(const float* __restrict__ part, int nb, int n, int n_det, double* out,
                                    int accumulate) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb * n_det) return;
  const int b = i / n_det, d = i % n_det;
  double s = 0.0;
  for (int l = 0; l < n; ++l) s += (double)part[((size_t)b * n + l) * n_det + d];
  out[i] = accumulate ? out[i] + s : s;
}

// Bytes of the per-line detector partials behind the forward layout.
static size_t det_part_bytes(const Layout& L, int n, int n_det) {
  return n_det > 0 ? align_up(4 * (size_t)L.batch * n * n_det) : 0;
}

// Masked sums of stored (fftshifted) patterns: one CTA per pattern, float64
// accumulation, the warps' sums added in warp order (deterministic). Pixel (y, x)
// of a stored pattern holds frequency ((y + n/2) mod n, (x + n/2) mod n).
constexpr int kDetThreads = 256;

// Per-detector CTA totals: each warp's shuffle sum, then the warps' sums in warp
// order (deterministic), written to row[0 .. n_det).
__device__ __forceinline__ void det_block_sums(const double (&acc)[PTYRO_MAX_DETECTORS], int n_det,
                                               double (*red)[PTYRO_MAX_DETECTORS], double* row) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 0; d < PTYRO_MAX_DETECTORS; ++d) {
    if (d >= n_det) break;
    double s = acc[d];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp][d] = s;
  }
  __syncthreads();
  if (threadIdx.x < n_det) {
    double s = 0.0;
    for (int w = 0; w < kDetThreads / 32; ++w) s += red[w][threadIdx.x];
    row[threadIdx.x] = s;
  }
}

static __global__ void __launch_bounds__(kDetThreads) k_detect_patterns(const float* __restrict__ pat, int n,
                                                                        const uint32_t* __restrict__ mask,
                                                                        int n_det, double* out) {
  __shared__ double red[kDetThreads / 32][PTYRO_MAX_DETECTORS];
  const size_t nn = (size_t)n * n;
  const float* p = pat + (size_t)blockIdx.x * nn;
  double acc[PTYRO_MAX_DETECTORS];
#pragma unroll
  for (int d = 0; d < PTYRO_MAX_DETECTORS; ++d) acc[d] = 0.0;
  const int h = n / 2, m = n - 1;
  for (size_t i = threadIdx.x; i < nn; i += kDetThreads) {
    const int y = (int)(i / n), x = (int)(i % n);
    const float v = p[i];
    const uint32_t b = __ldg(mask + (size_t)((y + h) & m) * n + ((x + h) & m));
#pragma unroll
    for (int d = 0; d < PTYRO_MAX_DETECTORS; ++d)
      if (d < n_det && ((b >> d) & 1u)) acc[d] += (double)v;
  }
  det_block_sums(acc, n_det, red, out + (size_t)blockIdx.x * n_det);
}

// The same sums for patterns of any height x width, the mask given in the stored
// patterns' own (fftshifted) pixel order: pixel i of every pattern against mask[i],
// as the reference's annular_detector multiplies each pattern by its mask.
static __global__ void __launch_bounds__(kDetThreads) k_detect_patterns_stored(const float* __restrict__ pat,
                                                                               int hw,
                                                                               const uint32_t* __restrict__ mask,
                                                                               int n_det, double* out) {
  __shared__ double red[kDetThreads / 32][PTYRO_MAX_DETECTORS];
  const float* p = pat + (size_t)blockIdx.x * hw;
  double acc[PTYRO_MAX_DETECTORS];
#pragma unroll
  for (int d = 0; d < PTYRO_MAX_DETECTORS; ++d) acc[d] = 0.0;
  for (int i = threadIdx.x; i < hw; i += kDetThreads) {
    const float v = p[i];
    const uint32_t b = __ldg(mask + i);
#pragma unroll
    for (int d = 0; d < PTYRO_MAX_DETECTORS; ++d)
      if (d < n_det && ((b >> d) & 1u)) acc[d] += (double)v;
  }
  det_block_sums(acc, n_det, red, out + (size_t)blockIdx.x * n_det);
}

static int detect_patterns(const float* patterns, int count, int n, const uint32_t* mask, int n_det, double* out,
                           cudaStream_t st) {
  k_detect_patterns<<<count, kDetThreads, 0, st>>>(patterns, n, mask, n_det, out);
  return check_launch("k_detect_patterns");
}

// Patterns streamed to host memory (ptyro_ms_forward_to_host): after each probe batch
// the batch's patterns are copied on `copy` once `ready` (recorded after the batch's
// pattern pass) has fired, while later batches compute; at the end the call's stream
// waits for `copied`, recorded after the last copy. Waits take the event's latest
// record at the time of the call, so one `ready` event serves every batch.
struct HostStream {
  float* host = nullptr;
  cudaStream_t copy = nullptr;
  cudaEvent_t ready = nullptr, copied = nullptr;
  ~HostStream() {
    if (ready) cudaEventDestroy(ready);
    if (copied) cudaEventDestroy(copied);
  }
};

static int copy_batch_to_host(const HostStream* hs, const float* patterns, int b0, int nb, size_t nn,
                              cudaStream_t st) {
  if (!hs) return PTYRO_OK;
  if (cudaEventRecord(hs->ready, st) != cudaSuccess || cudaStreamWaitEvent(hs->copy, hs->ready, 0) != cudaSuccess ||
      cudaMemcpyAsync(hs->host + (size_t)b0 * nn, patterns + (size_t)b0 * nn, sizeof(float) * nn * (size_t)nb,
                      cudaMemcpyDeviceToHost, hs->copy) != cudaSuccess)
    return fail(PTYRO_ERR_CUDA, "streaming the patterns to host memory failed");
  return PTYRO_OK;
}

static int forward_impl(const ptyro_ms_params* p, int ckpt_every, const float* potential, const float* modes,
                        const float* weights, const double* positions, float* patterns, float2* residuals,
                        void* workspace, size_t workspace_bytes, void* stream, const DetOut* det_in = nullptr,
                        const FwdExtras* ex = nullptr, const HostStream* hs = nullptr) {
  int rc = validate(p);
  if (rc) return rc;
  if (p->num_probes == 0) return PTYRO_OK;
  const bool has_det = det_in && det_in->n_det > 0;
  const bool has_amp = ex && ex->amplitudes;
  if (!potential || !modes || !positions || (!patterns && !has_det && !has_amp) ||
      (!weights && (patterns || has_det)))
    return fail(PTYRO_ERR_INVALID, "NULL array argument");
  if (has_det && (!det_in->mask || !det_in->out)) return fail(PTYRO_ERR_INVALID, "NULL detector argument");
  const Layout L = layout_for(p);
  if (has_det) {
    if (workspace_bytes < L.total + det_part_bytes(L, p->n, det_in->n_det))
      return fail(PTYRO_ERR_WORKSPACE, "workspace too small for the detector partials: need " +
                                           std::to_string(L.total + det_part_bytes(L, p->n, det_in->n_det)));
    workspace_bytes = L.total;
  }
  rc = check_workspace(L, workspace, workspace_bytes);
  if (rc) return rc;
  DetOut det = {};
  if (has_det) {
    det = *det_in;
    det.part = (float*)((char*)workspace + L.total);
  }
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  if ((rc = clear_status(ws + L.status, st))) return rc;
  rc = forward_setup(p, L, ws, potential, modes, st);
  if (rc) return rc;
  const int n = p->n, S = p->num_slices, M = p->num_modes;
  const size_t nn = (size_t)n * n;
  const int C = residuals ? (S + ckpt_every - 1) / ckpt_every : 0;
  const size_t res_stride = (size_t)(C + 1) * nn;
  const FwdBuffers B = fwd_buffers(L, ws);
  // tune bit 32768: the wave-resident kernel (one CTA per probe, wave in shared memory
  // across all slices) where it applies: N <= 128, one mode, no field windows, no
  // residuals, detectors, tilts or amplitude output
  const bool resident = (p->tune & kTuneResident) && resident_smem_bytes(n) > 0 && M == 1 && !residuals &&
                        !has_det && !ex && !p->windows && field_of(p) == n;
  for (int b0 = 0; b0 < p->num_probes; b0 += L.batch) {
    const int nb = p->num_probes - b0 < L.batch ? p->num_probes - b0 : L.batch;
    float2* res_base = residuals ? residuals + (size_t)b0 * M * res_stride : nullptr;
    k_ramps<<<(nb * n + 255) / 256, 256, 0, st>>>(positions + 2 * (size_t)b0, nb, n, p->shift_calib_ang,
                                                  (float2*)B.ramp_y, (float2*)B.ramp_x);
    if ((rc = check_launch("k_ramps"))) return rc;
    if (resident) {
      ResidentArgs ra = {};
      ra.probe_k = B.probe_k;
      ra.ramp_y = B.ramp_y;
      ra.ramp_x = B.ramp_x;
      ra.trans = B.trans;
      ra.trans_t = B.trans_t;
      ra.pf = B.pf;
      ra.tw = B.tw;
      ra.weights = weights;
      ra.pattern = patterns + (size_t)b0 * nn;
      ra.num_slices = S;
      ra.accumulate = (p->flags & PTYRO_FLAG_ACCUMULATE) != 0;
      ra.scale = 1.0f / (float)n;
      const int e = launch_resident(n, ra, nb, st);
      if (e != 0) return fail(PTYRO_ERR_CUDA, std::string("ms_resident_kernel: ") + cudaGetErrorString((cudaError_t)e));
      if ((rc = copy_batch_to_host(hs, patterns, b0, nb, nn, st))) return rc;
      continue;
    }
    for (int k = 0; k <= S + 1; ++k) {
      const FwdPlan f = fwd_pass_plan(p, B, weights, patterns, res_base, ckpt_every, C, b0, nb, k,
                                      has_det ? &det : nullptr, ex);
      if ((rc = launch_pass(n, f.axis, f.a, f.rows, st, p->tune))) return rc;
    }
    if (has_det) {
      k_det_reduce<<<(nb * det.n_det + 127) / 128, 128, 0, st>>>(det.part, nb, n, det.n_det,
                                                                  det.out + (size_t)b0 * det.n_det,
                                                                  (p->flags & PTYRO_FLAG_ACCUMULATE) != 0);
      if ((rc = check_launch("k_det_reduce"))) return rc;
    }
    if ((rc = copy_batch_to_host(hs, patterns, b0, nb, nn, st))) return rc;
  }
  if (hs && (cudaEventRecord(hs->copied, hs->copy) != cudaSuccess || cudaStreamWaitEvent(st, hs->copied, 0) != cudaSuccess))
    return fail(PTYRO_ERR_CUDA, "joining the pattern copies failed");
  return PTYRO_OK;
}

// ---------------------------------------------------------------- gradient
static __global__ void k_zero_pot(float* dv, long long sy, long long sx, long long ss, int n, int S) {
  const size_t total = (size_t)S * n * n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / ((size_t)n * n)), y = (int)((i / n) % n), x = (int)(i % n);
    dv[(long long)y * sy + (long long)x * sx + (long long)s * ss] = 0.f;
  }
}

static __global__ void k_zero2(float2* d, size_t count) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    d[i] = make_float2(0.f, 0.f);
}

// dV_s += sum over slots of the per-slot contributions, in slot order (deterministic),
// for a group of `planes` contribution planes (plane j, `pstride` floats apart, holds
// slice s0 - j); four planes are summed together so that their loads overlap.
static __global__ void k_reduce_dv(const float* __restrict__ contrib, int nslots, int n, float* dv, long long sy,
                                   long long sx, long long ss, int s0, int planes, long long pstride) {
  const size_t nn = (size_t)n * n;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const int y = (int)(i / n), x = (int)(i % n);
  for (int j0 = 0; j0 < planes; j0 += 4) {
    const int jn = planes - j0 < 4 ? planes - j0 : 4;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (int w = 0; w < nslots; ++w) {
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
        if (jj < jn) acc[jj] += __ldcs(contrib + (j0 + jj) * pstride + (size_t)w * nn + i);  // read once
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
      if (jj < jn) dv[(long long)y * sy + (long long)x * sx + (long long)(s0 - j0 - jj) * ss] += acc[jj];
  }
}

// Windowed runs: field pixel (fy, fx) of dV_s collects the contribution of every
// slot whose n x n window (origin modulo F) covers it, added in a fixed order (no
// atomics, deterministic). A CTA covers a TX x TY tile of the field (TX, TY <= n,
// TX TY = 64). First every thread classifies some of the slots (a window meets the
// tile iff it holds one of the tile's corner rows and one of its corner columns, both
// lengths being at most n), then warp 0 lists the meeting slots in slot order with
// their plane base and window origin. A batch's windows cluster (neighbouring scan
// positions), so central pixels collect many contributions: each pixel's list is
// split into kReduceQ contiguous parts summed by kReduceQ threads, 8 loads in flight
// each, and the parts are added in order. Neighbouring threads read neighbouring
// pixels of the same plane. Every listed slot takes the same path (local row and
// column from the window origin, one bounds test), and a single-mode run (M1) drops
// the mode loop: the loop body stays small, since instruction fetch, not DRAM, is
// what this kernel waits on most.
constexpr int kReduceQ = 4;
constexpr int kPartPlanes = 12;  // planes whose parts are staged between two barriers

// 4 CTAs per SM (64 registers): more resident warps pay for its short loads
template <bool M1>
static __global__ void __launch_bounds__(256, 4) k_reduce_dv_win(const float* __restrict__ contrib, int nb, int M, int n,
                                                       int F, const int* __restrict__ win, float* dv, long long sy,
                                                       long long sx, long long ss, int s0, int planes,
                                                       long long pstride, int tx_log2) {
  extern __shared__ long long shl[];
  long long* sbase = shl;                                    // listed: plane base of the slot
  int2* sorg = reinterpret_cast<int2*>(shl + nb);            // listed: window origin (wy, wx)
  int2* sall = sorg + nb;                                    // per slot: window origin
  int* sflag = reinterpret_cast<int*>(sall + nb);            // per slot: meets the tile
  __shared__ int count;
  __shared__ float part[kPartPlanes][256];
  constexpr int kPix = 256 / kReduceQ;  // pixels per tile
  const int TX = 1 << tx_log2, TY = kPix >> tx_log2;
  const int fx0 = (int)blockIdx.x * TX, fy0 = (int)blockIdx.y * TY;
  const int fm = F - 1;
  for (int bb = (int)threadIdx.x; bb < nb; bb += (int)blockDim.x) {
    const int wy = win ? win[2 * bb] : 0, wx = win ? win[2 * bb + 1] : 0;
    const bool rows = ((fy0 - wy) & fm) < n || ((fy0 + TY - 1 - wy) & fm) < n;
    const bool cols = ((fx0 - wx) & fm) < n || ((fx0 + TX - 1 - wx) & fm) < n;
    sall[bb] = make_int2(wy, wx);
    sflag[bb] = rows && cols;
  }
  __syncthreads();
  const size_t nn = (size_t)n * n;
  if (threadIdx.x < 32) {
    int c = 0;
    for (int b0 = 0; b0 < nb; b0 += 32) {
      const int bb = b0 + (int)threadIdx.x;
      const int f = bb < nb ? sflag[bb] : 0;
      const unsigned mask = __ballot_sync(0xffffffffu, f != 0);
      if (f) {
        const int pos = c + __popc(mask & ((1u << threadIdx.x) - 1u));
        sbase[pos] = (long long)bb * (M1 ? 1 : M) * (long long)nn;
        sorg[pos] = sall[bb];
      }
      c += __popc(mask);
    }
    if (threadIdx.x == 0) count = c;
  }
  __syncthreads();
  const int pix = (int)threadIdx.x & (kPix - 1), q = (int)threadIdx.x / kPix;
  const int tx = pix & (TX - 1), ty = pix >> tx_log2;
  const int fx = fx0 + tx, fy = fy0 + ty;
  const int cnt = count;
  const int kb = (int)(((long long)cnt * q) / kReduceQ), ke = (int)(((long long)cnt * (q + 1)) / kReduceQ);
  // planes (slices) four at a time: one listing serves every plane, and each thread
  // keeps one independent sum per plane in flight; the parts of up to kPartPlanes
  // planes wait in shared memory, so the threads meet once per kPartPlanes planes
  for (int g0 = 0; g0 < planes; g0 += kPartPlanes) {
    const int gn = planes - g0 < kPartPlanes ? planes - g0 : kPartPlanes;
    for (int j0 = g0; j0 < g0 + gn; j0 += 4) {
      const int jn = g0 + gn - j0 < 4 ? g0 + gn - j0 : 4;
      const float* cplane = contrib + j0 * pstride;
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      for (int k0 = kb; k0 < ke; k0 += 8) {
        float v[8][4];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int k = k0 + u;
          const bool in = k < ke;
          const int2 o = in ? sorg[k] : make_int2(0, 0);
          const int ly = (fy - o.x) & fm, lx = (fx - o.y) & fm;
          const bool ok = in && (ly | lx) < n;  // n is a power of two
          const float* cp = cplane + (ok ? sbase[k] + (long long)ly * n + lx : 0);
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            float t = 0.f;
            if (ok && jj < jn) {  // contributions are read once
              t = __ldcs(cp + jj * pstride);
              if (!M1)
                for (int m = 1; m < M; ++m) t += __ldcs(cp + jj * pstride + (size_t)m * nn);
            }
            v[u][jj] = t;
          }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) acc[jj] += v[u][jj];
      }
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
        if (jj < jn) part[j0 - g0 + jj][threadIdx.x] = acc[jj];
    }
    __syncthreads();
    if (q == 0) {
      for (int jj = 0; jj < gn; ++jj) {
        float sum = part[jj][pix];
#pragma unroll
        for (int r = 1; r < kReduceQ; ++r) sum += part[jj][r * kPix + pix];
        dv[(long long)fy * sy + (long long)fx * sx + (long long)(s0 - g0 - jj) * ss] += sum;
      }
    }
    __syncthreads();  // part is refilled by the next planes
  }
}

static int launch_reduce_dv_win(const float* contrib, int nb, int M, int n, int F, const int* win, float* dv,
                                long long sy, long long sx, long long ss, int s0, int planes, long long pstride,
                                cudaStream_t st) {
  // tile TX x TY = 256 / kReduceQ pixels with TX, TY <= n (n and F are powers of two, n >= 16)
  const int tx = n < 32 ? n : 32;
  int tx_log2 = 0;
  while ((1 << tx_log2) < tx) ++tx_log2;
  const int ty = (256 / kReduceQ) / tx;
  constexpr int kChunk = 1024;  // probes listed per launch (32 bytes of shared memory each)
  const dim3 grid((unsigned)(F / tx), (unsigned)(F / ty));
  for (int c0 = 0; c0 < nb; c0 += kChunk) {  // chunks add into dv in probe order
    const int cn = nb - c0 < kChunk ? nb - c0 : kChunk;
    const float* cbase = contrib + (size_t)c0 * M * n * n;
    const int* wbase = win ? win + 2 * (size_t)c0 : nullptr;
    if (M == 1)
      k_reduce_dv_win<true><<<grid, 256, 32 * (size_t)cn, st>>>(cbase, cn, M, n, F, wbase, dv, sy, sx, ss, s0, planes,
                                                                 pstride, tx_log2);
    else
      k_reduce_dv_win<false><<<grid, 256, 32 * (size_t)cn, st>>>(cbase, cn, M, n, F, wbase, dv, sy, sx, ss, s0, planes,
                                                                  pstride, tx_log2);
    int rc = check_launch("k_reduce_dv_win");
    if (rc) return rc;
  }
  return PTYRO_OK;
}

// beam spectrum gradient: acc[m] += sum_b lam[b*M + m], in probe order.
static __global__ void k_reduce_beam(const float2* __restrict__ lam, int nb, int M, int n, float2* acc) {
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
static __global__ void k_write_grad_modes(const float2* __restrict__ lam_beam, int n, int M, float2* out, long long sy,
                                   long long sx, long long sm) {
  const size_t nn = (size_t)n * n;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn * M) return;
  const int m = (int)(i / nn), y = (int)((i % nn) / n), x = (int)(i % n);
  const float2 v = lam_beam[i];
  out[(long long)y * sy + (long long)x * sx + (long long)m * sm] = make_float2(2.f * v.x, -2.f * v.y);
}

struct BwdLayout {
  size_t status, tw, pf, trans, trans_t, trans_p, trans_pt, ramp_y, ramp_x, psi, lam, contrib, beam, probe_k, total;
  int batch;
  bool paired_t;  // line-pair interleaved transmission tables (as the forward's, 256^2)
  int dgroup;  // slices whose dV contributions are kept before one reduction adds them
};

// Contribution planes kept per batch: the reduction of a group of slices lists each
// tile's windows once and overlaps the slices' loads.
constexpr size_t kContribGroupBytes = (size_t)512 << 20;

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
  L.status = o; o = align_up(o + PTYRO_WS_STATUS_BYTES);  // the call's device status word
  L.tw = o; o = align_up(o + 8 * (size_t)p->n);
  L.pf = o; o = align_up(o + 8 * (size_t)p->n);
  const size_t ff = (size_t)field_of(p) * field_of(p);
  L.trans = o; o = align_up(o + 8 * ff * p->num_slices);
  L.trans_t = o; o = align_up(o + 8 * ff * p->num_slices);
  L.paired_t = p->n == 256 && (p->tune & 16384) && (p->tune & 16) && (p->tune & 64);
  if (L.paired_t) {
    L.trans_p = o; o = align_up(o + 8 * ff * p->num_slices);
    L.trans_pt = o; o = align_up(o + 8 * ff * p->num_slices);
  }
  L.ramp_y = o; o = align_up(o + 8 * (size_t)p->n * L.batch);
  L.ramp_x = o; o = align_up(o + 8 * (size_t)p->n * L.batch);
  L.psi = o; o = align_up(o + 8 * nn * slots);
  L.lam = o; o = align_up(o + 8 * nn * slots);
  const size_t plane = 4 * nn * slots;
  size_t d = kContribGroupBytes / plane;
  d = d < 1 ? 1 : (d > (size_t)p->num_slices ? (size_t)p->num_slices : d);
  L.dgroup = (int)(d < 1 ? 1 : d);
  L.contrib = o; o = align_up(o + plane * L.dgroup);
  L.beam = o; o = align_up(o + 8 * nn * p->num_modes);
  L.probe_k = o; o = align_up(o + 8 * nn * p->num_modes);  // position gradients only
  L.total = o;
  return L;
}

// dL/d(position) of every probe of a batch from the adjoint left in k-space by the
// last passes, G_p = fft2(lam_psi0_p) conj(R_p), and the probe spectra B_m:
// psi0_p = ifft2(B R_p), R_p = exp(-2 pi i (qy y_p + qx x_p)), so
// dL/dy_p = 2 Re sum_r conj(lam) d psi0/dy = (4 pi / N^2) sum_{m,k} qy Im(conj(G) B)
// (Parseval), likewise x. One CTA per probe, float64 accumulation, warps added in
// order (deterministic).
static __global__ void __launch_bounds__(256) k_position_grad(const float2* __restrict__ G, const float2* __restrict__ B,
                                                              int n, int M, double shift_calib, double* out) {
  __shared__ double red[8][2];
  const size_t nn = (size_t)n * n;
  const int b = blockIdx.x;
  double sy = 0.0, sx = 0.0;
  for (int m = 0; m < M; ++m) {
    const float2* g = G + ((size_t)b * M + m) * nn;
    const float2* bk = B + (size_t)m * nn;
    for (size_t i = threadIdx.x; i < nn; i += blockDim.x) {
      const int ky = (int)(i / n), kx = (int)(i % n);
      const double qy = (double)(ky < n / 2 ? ky : ky - n) / (n * shift_calib);
      const double qx = (double)(kx < n / 2 ? kx : kx - n) / (n * shift_calib);
      const float2 gv = g[i], bv = bk[i];
      const double im = (double)gv.x * bv.y - (double)gv.y * bv.x;  // Im(conj(G) B)
      sy += qy * im;
      sx += qx * im;
    }
  }
  for (int o = 16; o >= 1; o >>= 1) {
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    red[warp][0] = sy;
    red[warp][1] = sx;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][threadIdx.x];
    out[2 * (size_t)b + threadIdx.x] = 4.0 * 3.14159265358979323846 / ((double)n * n) * s;
  }
}

static int launch_bwd(int n, int axis, const BwdArgs& a, int grid_y, cudaStream_t st, int variant = 0) {
  if (grid_y <= 0) return PTYRO_OK;
  int rc;
  switch (n) {
    case 16: rc = launch_bwd_16(axis, a, grid_y, st, variant); break;
    case 32: rc = launch_bwd_32(axis, a, grid_y, st, variant); break;
    case 64: rc = launch_bwd_64(axis, a, grid_y, st, variant); break;
    case 128: rc = launch_bwd_128(axis, a, grid_y, st, variant); break;
    case 256: rc = launch_bwd_256(axis, a, grid_y, st, variant); break;
    case 512: rc = launch_bwd_512(axis, a, grid_y, st, variant); break;
    case 1024: rc = launch_bwd_1024(axis, a, grid_y, st, variant); break;
    default: return fail(PTYRO_ERR_UNSUPPORTED, "grid edge not compiled");
  }
  if (rc != 0) return fail(PTYRO_ERR_CUDA, std::string("ms_bwd_pass_kernel: ") + cudaGetErrorString((cudaError_t)rc));
  return PTYRO_OK;
}

// Arguments of adjoint pass k (0 .. S+1) for the probe batch [b0, b0 + nb).
struct BwdPlan {
  BwdArgs a;
  int axis;
  int rows;
  int slice;  // slice point whose dV contribution the pass writes, or -1
};

struct BwdBuffers {
  unsigned int* status;
  float2 *psi, *lam;
  float* contrib;
  const float2 *trans, *trans_t, *pf, *tw, *ramp_y, *ramp_x;
  const float4 *trans_p = nullptr, *trans_pt = nullptr;  // interleaved tables, or null
  int dgroup = 1;             // contribution planes: slice point i (in adjoint order) writes plane i % dgroup
  size_t contrib_plane = 0;   // floats between planes
};

static BwdPlan bwd_pass_plan(const ptyro_ms_params* p, const BwdBuffers& B, const float* weights,
                             const float2* res_base, const float* gpat_batch, int ckpt_every, int C, int b0, int nb,
                             int k) {
  const int n = p->n, S = p->num_slices, M = p->num_modes;
  const size_t nn = (size_t)n * n;
  BwdPlan r;
  BwdArgs& a = r.a;
  a = BwdArgs{};
  a.status = B.status;
  a.psi = B.psi;
  a.lam = B.lam;
  a.weights = weights;
  a.res_stride = (size_t)(C + 1) * nn;
  a.trans = B.trans;
  a.trans_t = B.trans_t;
  a.trans_p = B.trans_p;
  a.trans_pt = B.trans_pt;
  a.pf = B.pf;
  a.tw = B.tw;
  a.ramp_y = B.ramp_y;
  a.ramp_x = B.ramp_x;
  a.n_modes = M;
  a.sigma2 = (float)(2.0 * interaction_sigma(p->voltage_kv));
  a.scale = 1.0f / (float)n;
  a.field_n = field_of(p);
  a.win = p->windows ? (const int*)p->windows + 2 * (size_t)b0 : nullptr;
  r.rows = nb * M;
  r.slice = -1;
  if (k == 0) {  // psi <- A, lam <- N^2 w g A, then the x part of the IFFT2 of both
    a.init = 1;
    a.amp = res_base + (size_t)C * nn;
    a.gpat = gpat_batch;
    a.op1 = OP_IFFT; a.t_slice = -1; a.op2 = OP_NONE;
    r.axis = 0;
  } else if (k <= S) {
    const int s = S - k;
    a.op1 = k == 1 ? OP_IFFT : OP_CONV_CONJ;
    a.t_slice = s;
    a.ckpt = (s % ckpt_every == 0) ? res_base + (size_t)(s / ckpt_every) * nn : nullptr;
    a.contrib = B.contrib + (size_t)((k - 1) % B.dgroup) * B.contrib_plane;
    a.op2 = k == S ? OP_FFT : OP_CONV_CONJ;
    a.psi_done = k == S;
    a.beam_epi = k == S;
    r.axis = k % 2;
    r.slice = s;
  } else {  // the other axis of FFT2(lam_psi0) times conj(ramp)
    a.op1 = OP_FFT; a.t_slice = -1; a.op2 = OP_NONE; a.psi_done = 1; a.beam_epi = 1;
    r.axis = (S + 1) % 2;
  }
  // a checkpoint at every slice point: the lambda-only pass (tune bit 65536 keeps the lockstep one)
  a.lam_only = ckpt_every == 1 && n <= 256 && !(p->tune & kTuneLockstepAdjoint);
  return r;
}

// ---------------------------------------------------------------- mode-weight gradient
// dL/dw_m = sum_p sum_k g_p(fftshift(k)) |A_pm(k)|^2 over the far-field amplitudes the
// residual-recording forward stored (unshifted). Each CTA of row m sums a fixed share
// of the (probe, pixel) elements in float64 and writes one partial; a second kernel adds
// the partials in order (deterministic).
constexpr int kWeightGradBlocks = 296;

static size_t weight_grad_workspace_bytes(int num_modes) {
  return align_up(sizeof(double) * (size_t)kWeightGradBlocks * (size_t)num_modes);
}

// the reduction itself (ms_generic.cu), for any H x W: sum_p sum_k g_p(fftshift k) |A_pm(k)|^2
int weight_grad_hw(int P, int M, int H, int W, size_t slot_stride, size_t amp_off, const float2* res, const float* g,
                   double* out, double* part, int blocks, cudaStream_t st);

static int weight_grad(const ptyro_ms_params* p, int ckpt_every, const float2* residuals, const float* g,
                       double* out, double* part, cudaStream_t st) {
  const int n = p->n, M = p->num_modes, P = p->num_probes;
  const size_t nn = (size_t)n * n;
  const int C = (p->num_slices + ckpt_every - 1) / ckpt_every;
  if (P == 0) {
    const cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * (size_t)M, st);
    return e == cudaSuccess ? PTYRO_OK : fail(PTYRO_ERR_CUDA, cudaGetErrorString(e));
  }
  const int rc = weight_grad_hw(P, M, n, n, (size_t)(C + 1) * nn, (size_t)C * nn, residuals, g, out, part,
                                kWeightGradBlocks, st);
  return rc ? fail(rc, "mode-weight gradient: launch failed") : PTYRO_OK;
}

// dV of a group of `planes` slices (plane j: slice s0 - j, pstride floats apart)
static int launch_reduce_dv_group(const ptyro_ms_params* p, const float* contrib, int planes, size_t pstride, int nb,
                                  int b0, float* dv, int s0, cudaStream_t st) {
  const int n = p->n, M = p->num_modes, F = field_of(p);
  const size_t nn = (size_t)n * n;
  if (p->windows != nullptr || F != n) {
    const int* win = p->windows ? (const int*)p->windows + 2 * (size_t)b0 : nullptr;
    return launch_reduce_dv_win(contrib, nb, M, n, F, win, dv, p->pot_stride_y, p->pot_stride_x, p->pot_stride_s,
                                s0, planes, (long long)pstride, st);
  }
  k_reduce_dv<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(contrib, nb * M, n, dv, p->pot_stride_y,
                                                             p->pot_stride_x, p->pot_stride_s, s0, planes,
                                                             (long long)pstride);
  return check_launch("k_reduce_dv");
}

static int launch_reduce_dv_any(const ptyro_ms_params* p, const float* contrib, int nb, int b0, float* dv, int s,
                                cudaStream_t st) {
  return launch_reduce_dv_group(p, contrib, 1, 0, nb, b0, dv, s, st);
}

static int backward_impl(const ptyro_ms_params* p, int ckpt_every, const float* potential, const float* weights,
                         const double* positions, const float2* residuals, const float* grad_patterns,
                         float* grad_potential, float* grad_modes, void* workspace, size_t workspace_bytes,
                         void* stream, const float* modes = nullptr, double* grad_positions = nullptr) {
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
  if ((rc = clear_status(ws + L.status, st))) return rc;
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
  k_transmission<<<blocks_for((size_t)F * F * S, 256), 256, 0, st>>>(potential, p->pot_stride_y, p->pot_stride_x,
                                                                     p->pot_stride_s, F, S,
                                                                     interaction_sigma(p->voltage_kv),
                                                                     (float2*)(ws + L.trans), (float2*)(ws + L.trans_t),
                                                                     L.paired_t ? (float*)(ws + L.trans_p) : nullptr,
                                                                     L.paired_t ? (float*)(ws + L.trans_pt) : nullptr);
  k_zero_pot<<<blocks_for((size_t)F * F * S, 256), 256, 0, st>>>(grad_potential, p->pot_stride_y, p->pot_stride_x,
                                                                 p->pot_stride_s, F, S);
  k_zero2<<<blocks_for(nn * M, 256), 256, 0, st>>>(beam, nn * M);
  if ((rc = check_launch("backward setup", 5))) return rc;
  if (grad_positions) {
    if (!modes) return fail(PTYRO_ERR_INVALID, "position gradients need the beam modes");
    float2* pk = (float2*)(ws + L.probe_k);
    k_gather_modes<<<blocks_for(nn * M, 256), 256, 0, st>>>((const float2*)modes, p->mode_stride_y,
                                                            p->mode_stride_x, p->mode_stride_m, n, M, pk);
    if ((rc = check_launch("k_gather_modes"))) return rc;
    if ((rc = fft2_planes(n, M, false, pk, tw, st))) return rc;
  }
  BwdBuffers B;
  B.status = (unsigned int*)(ws + L.status);
  B.psi = (float2*)(ws + L.psi);
  B.lam = (float2*)(ws + L.lam);
  B.contrib = (float*)(ws + L.contrib);
  B.dgroup = L.dgroup;
  B.contrib_plane = nn * (size_t)L.batch * M;
  B.trans = (const float2*)(ws + L.trans);
  B.trans_t = (const float2*)(ws + L.trans_t);
  B.trans_p = L.paired_t ? (const float4*)(ws + L.trans_p) : nullptr;
  B.trans_pt = L.paired_t ? (const float4*)(ws + L.trans_pt) : nullptr;
  B.pf = (const float2*)(ws + L.pf);
  B.tw = tw;
  B.ramp_y = (const float2*)(ws + L.ramp_y);
  B.ramp_x = (const float2*)(ws + L.ramp_x);
  for (int b0 = 0; b0 < p->num_probes; b0 += L.batch) {
    const int nb = p->num_probes - b0 < L.batch ? p->num_probes - b0 : L.batch;
    const float2* res_base = residuals + (size_t)b0 * M * res_stride;
    k_ramps<<<(nb * n + 255) / 256, 256, 0, st>>>(positions + 2 * (size_t)b0, nb, n, p->shift_calib_ang,
                                                  (float2*)B.ramp_y, (float2*)B.ramp_x);
    if ((rc = check_launch("k_ramps"))) return rc;
    for (int k = 0; k <= S + 1; ++k) {
      const BwdPlan b = bwd_pass_plan(p, B, weights, res_base, grad_patterns + (size_t)b0 * nn, ckpt_every, C, b0,
                                      nb, k);
      if ((rc = launch_bwd(n, b.axis, b.a, b.rows, st, p->tune))) return rc;
      // slice points k = 1 .. S (slice S - k) fill planes (k - 1) % dgroup; a full group,
      // or the last slice point, is reduced into dV in one launch
      if (b.slice >= 0 && ((k - 1) % L.dgroup == L.dgroup - 1 || k == S)) {
        const int i0 = (k - 1) - (k - 1) % L.dgroup;
        if ((rc = launch_reduce_dv_group(p, B.contrib, k - i0, B.contrib_plane, nb, b0, grad_potential, S - 1 - i0,
                                         st)))
          return rc;
      }
    }
    if (grad_positions) {
      k_position_grad<<<nb, 256, 0, st>>>(B.lam, (const float2*)(ws + L.probe_k), n, M, p->shift_calib_ang,
                                          grad_positions + 2 * (size_t)b0);
      if ((rc = check_launch("k_position_grad"))) return rc;
    }
    k_reduce_beam<<<(unsigned)((nn * M + 255) / 256), 256, 0, st>>>(B.lam, nb, M, n, beam);
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
