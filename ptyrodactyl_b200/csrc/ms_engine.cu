// B200 multislice 4D-STEM engine: the C-ABI declared in include/ptyro_b200.h.
#include "engine.cuh"

namespace ptyro {
thread_local std::string g_err;
std::atomic<unsigned long long> g_launches{0};
void set_error_message(const std::string& msg) { g_err = msg; }
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

int ptyro_ms_forward_to_host(const ptyro_ms_params* p, const float* potential, const float* modes,
                             const float* weights, const double* positions, float* patterns, float* host_patterns,
                             void* workspace, size_t workspace_bytes, void* stream, void* copy_stream) {
  if (!host_patterns) return fail(PTYRO_ERR_INVALID, "host_patterns is NULL");
  if (p && (p->flags & PTYRO_FLAG_ACCUMULATE))
    return fail(PTYRO_ERR_INVALID, "an accumulating forward cannot stream its patterns to the host");
  if (!copy_stream || copy_stream == stream)
    return fail(PTYRO_ERR_INVALID, "copy_stream must be a stream of its own (not NULL, not stream)");
  HostStream hs;
  hs.host = host_patterns;
  hs.copy = (cudaStream_t)copy_stream;
  if (cudaEventCreateWithFlags(&hs.ready, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&hs.copied, cudaEventDisableTiming) != cudaSuccess)
    return fail(PTYRO_ERR_CUDA, "cudaEventCreateWithFlags failed");
  return forward_impl(p, 0, potential, modes, weights, positions, patterns, nullptr, workspace, workspace_bytes,
                      stream, nullptr, nullptr, &hs);
}

size_t ptyro_ms_detect_workspace_bytes(const ptyro_ms_params* p, int32_t num_det) {
  if (validate(p) || num_det < 1 || num_det > PTYRO_MAX_DETECTORS) return 0;
  const Layout L = layout_for(p);
  return L.total + det_part_bytes(L, p->n, num_det);
}

int ptyro_ms_forward_detect(const ptyro_ms_params* p, const float* potential, const float* modes,
                            const float* weights, const double* positions, const uint32_t* det_mask,
                            int32_t num_det, double* det_out, float* patterns, void* workspace,
                            size_t workspace_bytes, void* stream) {
  if (num_det < 1 || num_det > PTYRO_MAX_DETECTORS)
    return fail(PTYRO_ERR_INVALID, "num_det must be in [1, " + std::to_string(PTYRO_MAX_DETECTORS) + "]");
  const DetOut det = {det_mask, num_det, nullptr, det_out};
  return forward_impl(p, 0, potential, modes, weights, positions, patterns, nullptr, workspace, workspace_bytes,
                      stream, &det);
}

int ptyro_detect_patterns(const float* patterns, int64_t num_patterns, int32_t n, const uint32_t* det_mask,
                          int32_t num_det, double* det_out, void* stream) {
  if (n < 2 || n > 8192 || (n & (n - 1)) != 0)
    return fail(PTYRO_ERR_UNSUPPORTED, "pattern edge must be a power of two in [2, 8192]");
  if (num_patterns < 0 || num_patterns > 0x7fffffffLL) return fail(PTYRO_ERR_INVALID, "num_patterns out of range");
  if (num_det < 1 || num_det > PTYRO_MAX_DETECTORS)
    return fail(PTYRO_ERR_INVALID, "num_det must be in [1, " + std::to_string(PTYRO_MAX_DETECTORS) + "]");
  if (num_patterns == 0) return PTYRO_OK;
  if (!patterns || !det_mask || !det_out) return fail(PTYRO_ERR_INVALID, "NULL array argument");
  return detect_patterns(patterns, (int)num_patterns, n, det_mask, num_det, det_out, (cudaStream_t)stream);
}

int ptyro_detect_patterns_hw(const float* patterns, int64_t num_patterns, int32_t height, int32_t width,
                             const uint32_t* det_mask, int32_t num_det, double* det_out, void* stream) {
  if (height < 1 || width < 1 || height > 8192 || width > 8192)
    return fail(PTYRO_ERR_INVALID, "pattern height and width must be in [1, 8192]");
  if (num_patterns < 0 || num_patterns > 0x7fffffffLL) return fail(PTYRO_ERR_INVALID, "num_patterns out of range");
  if (num_det < 1 || num_det > PTYRO_MAX_DETECTORS)
    return fail(PTYRO_ERR_INVALID, "num_det must be in [1, " + std::to_string(PTYRO_MAX_DETECTORS) + "]");
  if (num_patterns == 0) return PTYRO_OK;
  if (!patterns || !det_mask || !det_out) return fail(PTYRO_ERR_INVALID, "NULL array argument");
  k_detect_patterns_stored<<<(unsigned)num_patterns, kDetThreads, 0, (cudaStream_t)stream>>>(
      patterns, height * width, det_mask, num_det, det_out);
  return check_launch("k_detect_patterns_stored");
}

int ptyro_ms_forward_tilted(const ptyro_ms_params* p, const float* potential, const float* modes,
                            const float* weights, const double* positions, const float* tilts, float* patterns,
                            void* workspace, size_t workspace_bytes, void* stream) {
  if (!tilts && p && p->num_probes > 0) return fail(PTYRO_ERR_INVALID, "tilts is NULL");
  const FwdExtras ex = {(const float2*)tilts, nullptr};
  return forward_impl(p, 0, potential, modes, weights, positions, patterns, nullptr, workspace, workspace_bytes,
                      stream, nullptr, &ex);
}

int ptyro_ms_amplitudes(const ptyro_ms_params* p, const float* potential, const float* modes,
                        const double* positions, const float* tilts, float* amplitudes, void* workspace,
                        size_t workspace_bytes, void* stream) {
  if (!amplitudes && p && p->num_probes > 0) return fail(PTYRO_ERR_INVALID, "amplitudes is NULL");
  if (p && (p->flags & PTYRO_FLAG_ACCUMULATE))
    return fail(PTYRO_ERR_INVALID, "amplitudes cannot be accumulated");
  const FwdExtras ex = {(const float2*)tilts, (float2*)amplitudes};
  return forward_impl(p, 0, potential, modes, nullptr, positions, nullptr, nullptr, workspace, workspace_bytes,
                      stream, nullptr, &ex);
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

int ptyro_ms_backward_positions(const ptyro_ms_params* p, int32_t ckpt_every, const float* potential,
                                const float* modes, const float* weights, const double* positions,
                                const float* residuals, const float* grad_patterns, float* grad_potential,
                                float* grad_modes, double* grad_positions, void* workspace, size_t workspace_bytes,
                                void* stream) {
  if (!grad_positions && p && p->num_probes > 0) return fail(PTYRO_ERR_INVALID, "grad_positions is NULL");
  return backward_impl(p, ckpt_every, potential, weights, positions, (const float2*)residuals, grad_patterns,
                       grad_potential, grad_modes, workspace, workspace_bytes, stream, modes, grad_positions);
}

size_t ptyro_ms_weight_grad_workspace_bytes(const ptyro_ms_params* p) {
  if (validate(p)) return 0;
  return weight_grad_workspace_bytes(p->num_modes);
}

int ptyro_ms_weight_grad(const ptyro_ms_params* p, int32_t ckpt_every, const float* residuals,
                         const float* grad_patterns, double* grad_weights, void* workspace, size_t workspace_bytes,
                         void* stream) {
  int rc = validate(p);
  if (rc) return rc;
  if (ckpt_every < 1) return fail(PTYRO_ERR_INVALID, "ckpt_every must be >= 1");
  if (!grad_weights) return fail(PTYRO_ERR_INVALID, "grad_weights is NULL");
  if (p->num_probes > 0 && (!residuals || !grad_patterns)) return fail(PTYRO_ERR_INVALID, "NULL array argument");
  if (!workspace || workspace_bytes < weight_grad_workspace_bytes(p->num_modes))
    return fail(PTYRO_ERR_WORKSPACE, "workspace too small for the weight gradient");
  return weight_grad(p, ckpt_every, (const float2*)residuals, grad_patterns, grad_weights, (double*)workspace,
                     (cudaStream_t)stream);
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

unsigned int ptyro_pass_wait_timeouts(void) {
  unsigned int (*const units[])() = {pair_wait_timeouts_16,  pair_wait_timeouts_32,  pair_wait_timeouts_64,
                                     pair_wait_timeouts_128, pair_wait_timeouts_256, pair_wait_timeouts_512,
                                     pair_wait_timeouts_1024};
  unsigned long long total = 0;
  for (auto f : units) total += f();
  return total > 0xffffffffull ? 0xffffffffu : (unsigned int)total;
}

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
  a.status = (unsigned int*)(ws + L.status);
  a.wave = (float2*)(ws + L.waves);
  a.trans = (const float2*)(ws + L.trans);
  a.trans_t = (const float2*)(ws + L.trans_t);
  if (L.paired_t) {  // written by the forward that filled this workspace
    a.trans_p = (const float4*)(ws + L.trans_p);
    a.trans_pt = (const float4*)(ws + L.trans_pt);
  }
  if (L.half_t) {
    a.trans_h = (const float4*)(ws + L.trans_h);
    a.trans_ht = (const float4*)(ws + L.trans_ht);
  }
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
