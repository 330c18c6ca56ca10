// Forward-mode (tangent) product of the 4D-STEM forward model: the C-ABI
// ptyro_ms_jvp declared in include/ptyro_b200.h. The passes follow the forward's
// schedule exactly (ms_jvp.cuh carries the wave and its tangent together).
#include "engine.cuh"

namespace ptyro {

// sigma * dV (strided [y][x][s]) -> row-major and transposed (S, F, F) tables
static __global__ void k_tangent_table(const float* __restrict__ dV, long long sy, long long sx, long long ss, int n,
                                       int S, double sigma, float* __restrict__ D, float* __restrict__ DT) {
  const size_t total = (size_t)S * n * n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / ((size_t)n * n));
    const int y = (int)((i / n) % n);
    const int x = (int)(i % n);
    const float v = (float)(sigma * (double)dV[(long long)y * sy + (long long)x * sx + (long long)s * ss]);
    D[i] = v;
    DT[(size_t)s * n * n + (size_t)x * n + y] = v;
  }
}

static int launch_jvp(int n, int axis, const JvpArgs& a, int grid_y, cudaStream_t st) {
  if (grid_y <= 0) return PTYRO_OK;
  int rc;
  switch (n) {
    case 16: rc = launch_jvp_16(axis, a, grid_y, st); break;
    case 32: rc = launch_jvp_32(axis, a, grid_y, st); break;
    case 64: rc = launch_jvp_64(axis, a, grid_y, st); break;
    case 128: rc = launch_jvp_128(axis, a, grid_y, st); break;
    case 256: rc = launch_jvp_256(axis, a, grid_y, st); break;
    case 512: rc = launch_jvp_512(axis, a, grid_y, st); break;
    case 1024: rc = launch_jvp_1024(axis, a, grid_y, st); break;
    default: return fail(PTYRO_ERR_UNSUPPORTED, "grid edge not compiled");
  }
  if (rc != 0) return fail(PTYRO_ERR_CUDA, std::string("ms_jvp_pass_kernel: ") + cudaGetErrorString((cudaError_t)rc));
  return PTYRO_OK;
}

// Workspace: the forward's layout, then the tangent slots, the tangent probe
// spectra and the two sigma * dV tables.
struct JvpLayout {
  Layout L;
  size_t dwaves, dprobe_k, sdv, sdv_t, total;
};

static JvpLayout jvp_layout_for(const ptyro_ms_params* p) {
  JvpLayout J;
  J.L = layout_for(p);
  const size_t nn = (size_t)p->n * p->n, ff = (size_t)field_of(p) * field_of(p);
  size_t o = J.L.total;
  J.dwaves = o; o = align_up(o + 8 * nn * p->num_modes * (size_t)J.L.batch);
  J.dprobe_k = o; o = align_up(o + 8 * nn * p->num_modes);
  J.sdv = o; o = align_up(o + 4 * ff * p->num_slices);
  J.sdv_t = o; o = align_up(o + 4 * ff * p->num_slices);
  J.total = o;
  return J;
}

static int jvp_impl(const ptyro_ms_params* p, const float* potential, const float* dpotential, const float* modes,
                    const float* dmodes, const float* weights, const double* positions, float* patterns,
                    float* dpatterns, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = validate(p);
  if (rc) return rc;
  if (p->num_probes == 0) return PTYRO_OK;
  if (!potential || !modes || !weights || !positions || !dpatterns)
    return fail(PTYRO_ERR_INVALID, "NULL array argument");
  const JvpLayout J = jvp_layout_for(p);
  const Layout& L = J.L;
  if (!workspace) return fail(PTYRO_ERR_WORKSPACE, "workspace is NULL");
  if (((uintptr_t)workspace & 255) != 0) return fail(PTYRO_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  if (workspace_bytes < J.total)
    return fail(PTYRO_ERR_WORKSPACE, "workspace too small: need " + std::to_string(J.total) + " bytes, got " +
                                         std::to_string(workspace_bytes));
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  if ((rc = clear_status(ws + L.status, st))) return rc;
  if ((rc = forward_setup(p, L, ws, potential, modes, st))) return rc;
  const int n = p->n, S = p->num_slices, M = p->num_modes, F = field_of(p);
  const size_t nn = (size_t)n * n;
  float2* dpk = (float2*)(ws + J.dprobe_k);
  if (dmodes) {
    k_gather_modes<<<blocks_for(nn * M, 256), 256, 0, st>>>((const float2*)dmodes, p->mode_stride_y,
                                                            p->mode_stride_x, p->mode_stride_m, n, M, dpk);
    if ((rc = check_launch("k_gather_modes"))) return rc;
    if ((rc = fft2_planes(n, M, false, dpk, (const float2*)(ws + L.tw), st))) return rc;
  }
  if (dpotential) {
    k_tangent_table<<<blocks_for((size_t)F * F * S, 256), 256, 0, st>>>(
        dpotential, p->pot_stride_y, p->pot_stride_x, p->pot_stride_s, F, S, interaction_sigma(p->voltage_kv),
        (float*)(ws + J.sdv), (float*)(ws + J.sdv_t));
    if ((rc = check_launch("k_tangent_table"))) return rc;
  }
  const FwdBuffers B = fwd_buffers(L, ws);
  JvpArgs a = {};
  a.psi = B.waves;
  a.dpsi = (float2*)(ws + J.dwaves);
  a.probe_k = B.probe_k;
  a.dprobe_k = dmodes ? dpk : nullptr;
  a.ramp_y = B.ramp_y;
  a.ramp_x = B.ramp_x;
  a.trans = B.trans;
  a.trans_t = B.trans_t;
  a.sdv = dpotential ? (const float*)(ws + J.sdv) : nullptr;
  a.sdv_t = dpotential ? (const float*)(ws + J.sdv_t) : nullptr;
  a.field_n = F;
  a.pf = B.pf;
  a.tw = B.tw;
  a.weights = weights;
  a.n_modes = M;
  a.scale = 1.0f / (float)n;
  for (int b0 = 0; b0 < p->num_probes; b0 += L.batch) {
    const int nb = p->num_probes - b0 < L.batch ? p->num_probes - b0 : L.batch;
    a.win = p->windows ? (const int*)p->windows + 2 * (size_t)b0 : nullptr;
    k_ramps<<<(nb * n + 255) / 256, 256, 0, st>>>(positions + 2 * (size_t)b0, nb, n, p->shift_calib_ang,
                                                  (float2*)B.ramp_y, (float2*)B.ramp_x);
    if ((rc = check_launch("k_ramps"))) return rc;
    for (int k = 0; k <= S + 1; ++k) {
      int axis, rows;
      if (k == 0) {  // x part of the IFFT2 of the shifted probe spectra
        a.src = SRC_PROBE; a.op1 = OP_IFFT; a.t_slice = -1; a.op2 = OP_NONE; a.dst = DST_WAVE;
        axis = 0;
        rows = nb * M;
      } else if (k <= S) {
        a.src = SRC_WAVE; a.op1 = k == 1 ? OP_IFFT : OP_CONV; a.t_slice = k - 1;
        a.op2 = k == S ? OP_FFT : OP_CONV; a.dst = DST_WAVE;
        axis = k % 2;
        rows = nb * M;
      } else {  // last axis of the FFT2; intensities and their tangents, fftshifted
        a.src = SRC_WAVE; a.op1 = OP_FFT; a.t_slice = -1; a.op2 = OP_NONE; a.dst = DST_PATTERN;
        a.pattern = patterns ? patterns + (size_t)b0 * nn : nullptr;
        a.dpattern = dpatterns + (size_t)b0 * nn;
        axis = (S + 1) % 2;
        rows = nb;
      }
      if ((rc = launch_jvp(n, axis, a, rows, st))) return rc;
    }
  }
  return PTYRO_OK;
}

}  // namespace ptyro

using namespace ptyro;

extern "C" {

size_t ptyro_ms_jvp_workspace_bytes(const ptyro_ms_params* p) {
  if (validate(p)) return 0;
  return jvp_layout_for(p).total;
}

int ptyro_ms_jvp(const ptyro_ms_params* p, const float* potential, const float* tangent_potential,
                 const float* modes, const float* tangent_modes, const float* weights, const double* positions,
                 float* patterns, float* tangent_patterns, void* workspace, size_t workspace_bytes, void* stream) {
  return jvp_impl(p, potential, tangent_potential, modes, tangent_modes, weights, positions, patterns,
                  tangent_patterns, workspace, workspace_bytes, stream);
}

}  // extern "C"
