/*
 * ptyro_b200 — C-ABI of the B200 multislice 4D-STEM engine.
 *
 * Plain pointers and sizes only. Every array argument is a DEVICE pointer unless
 * its comment says HOST; every call only enqueues work on `stream` (a
 * cudaStream_t passed as void*), never synchronises and never allocates: scratch
 * comes from the caller's `workspace`, sized by ptyro_ms_workspace_bytes().
 * Complex arrays are interleaved complex64 (re, im float pairs).
 *
 * Each entry point replaces one step of the reference's JAX path
 * (ptyrodactyl 2026.5.31, paths relative to its project root); the citation
 * names the function whose arithmetic and argument meaning it keeps.
 *
 * Return value: PTYRO_OK or an error code; ptyro_last_error() gives the message
 * of the last failure on the calling host thread.
 *
 * Device status: the first PTYRO_WS_STATUS_BYTES of every engine workspace
 * (ptyro_ms_forward and its variants, ptyro_ms_backward*, ptyro_ms_jvp) hold the
 * call's device status word, a uint32 at offset 0. Each call zeroes it on its
 * stream before its first kernel and its kernels OR PTYRO_STATUS_* bits into it.
 * Since the call does not synchronise, its return value cannot report these: the
 * caller reads the word once the stream has run the call (for an XLA FFI handler:
 * copy it into an output flag buffer and raise on the host, like eqx.error_if)
 * and treats any set bit as a failed call whose outputs are unusable.
 */
#ifndef PTYRO_B200_H
#define PTYRO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PTYRO_OK 0
#define PTYRO_ERR_INVALID 1     /* bad shape, size or scalar (reference: ValueError) */
#define PTYRO_ERR_WORKSPACE 2   /* workspace too small or misaligned */
#define PTYRO_ERR_CUDA 3        /* a launch failed */
#define PTYRO_ERR_UNSUPPORTED 4 /* grid size outside the compiled set */

#define PTYRO_WS_STATUS_BYTES 256 /* the status block at the start of each workspace */
/* Status bit: a bounded wait for a tile copy (TMA) gave up; the warps that gave up
 * left their lines of the wave unwritten, so the call's results are wrong. */
#define PTYRO_STATUS_WAIT_TIMEOUT 1u

/* ptyro_ms_params.flags: add sum_m w_m |A_m|^2 into `patterns` instead of
 * overwriting them (frozen-phonon averaging: one forward per configuration with
 * weights scaled by 1/configurations; the plain and gradient paths ignore it). */
#define PTYRO_FLAG_ACCUMULATE 1

/* Geometry and physics scalars of one multislice job.
 * The potential is V[y][x][s] with element strides pot_stride_{y,x,s} (the
 * reference stores slices last, PotentialSlices.slices (H, W, S)); the beam is
 * modes[y][x][m] with complex-element strides mode_stride_{y,x,m}
 * (ProbeModes.modes (H, W, M)). */
typedef struct ptyro_ms_params {
  int32_t n;                   /* grid edge H == W; power of two in [16, 1024] */
  int32_t num_slices;          /* S >= 1 */
  int32_t num_modes;           /* M >= 1 */
  int32_t num_probes;          /* P >= 0 scan positions */
  int32_t batch;               /* probes in flight per batch; 0 = automatic */
  int32_t tune;                /* kernel variant bits (0 = default): bit a (a = 0, 1) selects
                                  the 3-CTAs-per-SM register budget for passes along axis a;
                                  bit 2 the persistent double-buffered steady-pass kernel */
  int32_t field_n;             /* 0, or edge F of a larger periodic potential field (power of
                                  two, n <= F <= 8192) from which every probe reads an n x n
                                  window; the potential (and its gradient) is then F x F x S */
  int32_t flags;               /* PTYRO_FLAG_* bits */
  double voltage_kv;           /* MicroscopeConfig.voltage_kv */
  double slice_thickness_ang;  /* PotentialSlices.slice_thickness */
  double calib_ang;            /* min(PotentialSlices.calib, ProbeModes.calib): propagator grid */
  double shift_calib_ang;      /* DetectorConfig.real_space_calib_ang: shift-ramp grid */
  int64_t pot_stride_y, pot_stride_x, pot_stride_s;
  int64_t mode_stride_y, mode_stride_x, mode_stride_m;
  const int32_t* windows;      /* DEVICE (P, 2) int32 (y, x) window origins in the field, or
                                  NULL (all windows at 0); taken modulo F. The windowed run
                                  stands in for the reference's tiled workflow, which crops a
                                  tile of the sample around each position
                                  (src/ptyrodactyl/workflows/stem_4d.py:553) */
} ptyro_ms_params;

/* Library version, major*10000 + minor*100 + patch. */
int ptyro_version(void);

/* Message of the last failed call on this host thread ("" if none). */
const char* ptyro_last_error(void);

/* Workspace bytes ptyro_ms_forward / ptyro_ms_forward_plain need for `p`. */
size_t ptyro_ms_workspace_bytes(const ptyro_ms_params* p);

/* Batched fused 4D-STEM forward model.
 * Replaces stem_4d (src/ptyrodactyl/multislice/simulations.py:1330-1443) with its
 * shift_beam_fourier (:1236-1327), the slice loop of
 * _cbed_amplitude_from_slice_provider (:501-603) and the incoherent mode sum of
 * apply_distribution (src/ptyrodactyl/multislice/reduce.py:29-89).
 *   potential  float32 V[y][x][s] (strided, see ptyro_ms_params), volt-Angstrom
 *   modes      complex64 beam modes[y][x][m] (strided)
 *   weights    float32 (M) normalised mode weights
 *   positions  float64 (P, 2) (y, x) shifts; the reference passes
 *              DetectorConfig.scan_positions_px here and its q grid makes them
 *              act as Angstrom
 *   patterns   float32 (P, N, N) out: fftshifted sum_m w_m |A_m|^2 per position */
int ptyro_ms_forward(const ptyro_ms_params* p, const float* potential, const float* modes,
                     const float* weights, const double* positions, float* patterns,
                     void* workspace, size_t workspace_bytes, void* stream);

/* ptyro_ms_forward whose patterns also stream to host memory: after each probe batch's
 * pattern pass, the batch's patterns (in `patterns`, device) are copied into
 * host_patterns ((P, n, n) float32; page-locked for the copies to overlap) on
 * copy_stream while later batches compute; `stream` waits for the last copy, so work
 * ordered after the call on `stream` sees every pattern on the host. One setup for all
 * batches, and only the last batch's copy is not hidden. copy_stream: a stream of its
 * own (not NULL, not stream); no PTYRO_FLAG_ACCUMULATE; not for stream capture. */
int ptyro_ms_forward_to_host(const ptyro_ms_params* p, const float* potential, const float* modes,
                             const float* weights, const double* positions, float* patterns, float* host_patterns,
                             void* workspace, size_t workspace_bytes, void* stream, void* copy_stream);

/* Residual bytes ptyro_ms_forward_ckpt writes for `p`: per (probe, mode) one
 * complex64 N x N plane per checkpoint (slices 0, K, 2K, ... for K = ckpt_every)
 * plus one plane for the far-field amplitude. */
size_t ptyro_ms_residual_bytes(const ptyro_ms_params* p, int32_t ckpt_every);

/* ptyro_ms_forward that also records the residuals the gradient needs: the wave
 * after every K-th transmission multiply and the complex far-field amplitude, as
 * `residuals` (P, M, ceil(S/K) + 1, N, N) complex64. The reverse pass of
 * jax.value_and_grad through stem_4d (src/ptyrodactyl/multislice/multislice_recon.py:1940,
 * :1915-1966) would instead keep every slice's wave of the lax.scan.
 * Workspace: ptyro_ms_workspace_bytes(p). */
int ptyro_ms_forward_ckpt(const ptyro_ms_params* p, int32_t ckpt_every, const float* potential,
                          const float* modes, const float* weights, const double* positions,
                          float* patterns, float* residuals, void* workspace, size_t workspace_bytes,
                          void* stream);

/* Workspace bytes ptyro_ms_backward needs for `p` (p->batch probes per batch, 0 = automatic). */
size_t ptyro_ms_backward_workspace_bytes(const ptyro_ms_params* p);

/* Vector-Jacobian product of stem_4d: given dL/d(patterns) (P, N, N) float32 in the
 * patterns' fftshifted layout and the residuals of ptyro_ms_forward_ckpt (same p,
 * same ckpt_every), write
 *   grad_potential  float32 dL/dV with the potential's strides (p->pot_stride_*),
 *   grad_modes      complex64 gradient of the beam modes with the modes' strides, in
 *                   JAX's convention for a real loss: conj(2 dL/dconj(z)) = dL/dRe - i dL/dIm.
 * Matches jax.vjp / jax.grad through stem_4d in the reference (the gradient that
 * multislice_recon.py:1940 takes w.r.t. the potential and the beam). Mode weights and
 * positions are treated as constants. Sums over probes are in a fixed order.
 * Workspace: ptyro_ms_backward_workspace_bytes(p). */
int ptyro_ms_backward(const ptyro_ms_params* p, int32_t ckpt_every, const float* potential,
                      const float* weights, const double* positions, const float* residuals,
                      const float* grad_patterns, float* grad_potential, float* grad_modes,
                      void* workspace, size_t workspace_bytes, void* stream);

/* ptyro_ms_backward plus the gradient of L with respect to every scan position:
 * grad_positions float64 (P, 2) (y, x), in the units of `positions`. The
 * reconstruction loops that refine positions (single_slice_poscorrected,
 * single_slice_multi_modal, multi_slice_multi_modal,
 * src/ptyrodactyl/multislice/multislice_recon.py:671-2227) differentiate stem_4d
 * with respect to scan_positions_px; this is that derivative. `modes` as in
 * ptyro_ms_forward. Workspace: ptyro_ms_backward_workspace_bytes(p). */
int ptyro_ms_backward_positions(const ptyro_ms_params* p, int32_t ckpt_every, const float* potential,
                                const float* modes, const float* weights, const double* positions,
                                const float* residuals, const float* grad_patterns, float* grad_potential,
                                float* grad_modes, double* grad_positions, void* workspace, size_t workspace_bytes,
                                void* stream);

/* Workspace bytes of ptyro_ms_weight_grad for `p` (its num_modes). */
size_t ptyro_ms_weight_grad_workspace_bytes(const ptyro_ms_params* p);

/* Gradient of the loss with respect to the incoherent mode weights of stem_4d
 * (apply_distribution, src/ptyrodactyl/multislice/reduce.py:29-89: I = sum_m w_m |A_m|^2):
 * grad_weights[m] = sum_p sum_k dL/dI_p(k) |A_pm(k)|^2, float64 (M,), from the far-field
 * amplitudes stored by ptyro_ms_forward_ckpt (same p, same ckpt_every) and dL/d(patterns)
 * (P, N, N) in the patterns' fftshifted layout. Deterministic (fixed partial sums added
 * in order). The reference differentiates through the weights with jax.grad. */
int ptyro_ms_weight_grad(const ptyro_ms_params* p, int32_t ckpt_every, const float* residuals,
                         const float* grad_patterns, double* grad_weights, void* workspace, size_t workspace_bytes,
                         void* stream);

/* The same model run the plain way: one scan position at a time, one kernel per
 * stage (shift, and per slice transmission multiply, FFT2, propagator multiply,
 * IFFT2, then FFT2 and |.|^2), the way the reference's vmap body reads
 * (simulations.py:1396-1427 around :501-603). Kept as the comparison baseline. */
int ptyro_ms_forward_plain(const ptyro_ms_params* p, const float* potential, const float* modes,
                           const float* weights, const double* positions, float* patterns,
                           void* workspace, size_t workspace_bytes, void* stream);

/* ptyro_ms_forward with a beam tilt per mode: tilts is complex64 (M, 2, n), row
 * [m][0] the factors along y and [m][1] along x, multiplied into mode m's wave in real
 * space after the scan shift, before the first slice. This is the tilt phase ramp
 * that cbed_image's ensemble branch applies per coherence sample
 * (_apply_tilt_phase_ramp, src/ptyrodactyl/multislice/simulations.py:891-946), after
 * stem_4d's scan shift. Workspace: ptyro_ms_workspace_bytes(p). */
int ptyro_ms_forward_tilted(const ptyro_ms_params* p, const float* potential, const float* modes,
                            const float* weights, const double* positions, const float* tilts, float* patterns,
                            void* workspace, size_t workspace_bytes, void* stream);

/* Complex far-field amplitudes of every (probe, mode): complex64 (P, M, n, n),
 * fftshifted. Replaces cbed_amplitude (src/ptyrodactyl/multislice/simulations.py:
 * 606-679) at the probe's own place (positions zero) or shifted per position as in
 * stem_4d. tilts as in ptyro_ms_forward_tilted, or NULL. No weights: nothing is
 * summed. PTYRO_FLAG_ACCUMULATE is rejected. Workspace: ptyro_ms_workspace_bytes(p). */
int ptyro_ms_amplitudes(const ptyro_ms_params* p, const float* potential, const float* modes,
                        const double* positions, const float* tilts, float* amplitudes, void* workspace,
                        size_t workspace_bytes, void* stream);

/* Workspace bytes ptyro_ms_jvp needs for `p` (0 when invalid). */
size_t ptyro_ms_jvp_workspace_bytes(const ptyro_ms_params* p);

/* Forward-mode product of the forward model: the patterns and their directional
 * derivative along (tangent_potential, tangent_modes). This is the jax.jvp that
 * jvp_operator / jtj_operator (src/ptyrodactyl/jacobian/operators.py:30-186) take
 * through stem_4d (src/ptyrodactyl/multislice/simulations.py:1330-1443):
 *   tangent_potential  float32 dV with the potential's strides, or NULL (zero)
 *   tangent_modes      complex64 dmodes with the modes' strides, or NULL (zero)
 *   patterns           float32 (P, n, n) intensities, or NULL to skip them
 *   tangent_patterns   float32 (P, n, n) dI, fftshifted like the patterns
 * Windows (ptyro_ms_params.windows) apply to the tangent potential as to V. */
int ptyro_ms_jvp(const ptyro_ms_params* p, const float* potential, const float* tangent_potential,
                 const float* modes, const float* tangent_modes, const float* weights, const double* positions,
                 float* patterns, float* tangent_patterns, void* workspace, size_t workspace_bytes, void* stream);

/* Most virtual detectors one forward or one ptyro_detect_patterns call evaluates. */
#define PTYRO_MAX_DETECTORS 32

/* Workspace bytes ptyro_ms_forward_detect needs for `p` and `num_det` detectors
 * (0 when invalid). */
size_t ptyro_ms_detect_workspace_bytes(const ptyro_ms_params* p, int32_t num_det);

/* ptyro_ms_forward with virtual detectors fused into the pattern pass: the
 * integration step of annular_detector (src/ptyrodactyl/multislice/simulations.py:
 * 1539-1656) runs on each far-field intensity while it is in registers.
 *   det_mask  uint32 (n, n) in UNSHIFTED frequency order [ky][kx]: bit d set puts
 *             the pixel in detector d (the reference's annular mask is built on the
 *             fftshifted grid; pixel (i, j) there is frequency (i - n/2, j - n/2))
 *   num_det   1 .. PTYRO_MAX_DETECTORS
 *   det_out   float64 (P, num_det) masked intensity sums
 *   patterns  float32 (P, n, n) fftshifted intensities, or NULL to store none
 * PTYRO_FLAG_ACCUMULATE adds into det_out (and patterns). */
int ptyro_ms_forward_detect(const ptyro_ms_params* p, const float* potential, const float* modes,
                            const float* weights, const double* positions, const uint32_t* det_mask,
                            int32_t num_det, double* det_out, float* patterns, void* workspace,
                            size_t workspace_bytes, void* stream);

/* Masked sums of stored fftshifted patterns (P, n, n) float32: det_out[p][d] = sum of
 * the pixels of pattern p whose frequency has bit d set in det_mask (unshifted
 * order, as above). The vmap'd integration of annular_detector
 * (simulations.py:1620-1636). n a power of two in [2, 8192]. No workspace. */
int ptyro_detect_patterns(const float* patterns, int64_t num_patterns, int32_t n, const uint32_t* det_mask,
                          int32_t num_det, double* det_out, void* stream);

/* Masked sums of stored patterns of any height x width, (P, height, width) float32:
 * det_out[p][d] = sum of the pixels i of pattern p with bit d set in det_mask[i],
 * the mask in the stored patterns' own (fftshifted) pixel order, (height, width).
 * annular_detector (simulations.py:1539-1656) at every probe_shape, including the
 * any-size grids of ptyro_gm_forward. height, width in [1, 8192]. No workspace. */
int ptyro_detect_patterns_hw(const float* patterns, int64_t num_patterns, int32_t height, int32_t width,
                             const uint32_t* det_mask, int32_t num_det, double* det_out, void* stream);

/* Probe formation. Replaces make_probe (src/ptyrodactyl/multislice/simulations.py:334-431)
 * with aberration (:434-498): aperture |q| <= alpha/lambda times exp(-i chi),
 * ifftshift(ifft2(.)). Writes a complex64 (n, n) probe to `probe`.
 * Workspace: ptyro_fft_workspace_bytes(n). */
int ptyro_make_probe(int32_t n, double voltage_kv, double aperture_mrad, double probe_calibration_pm,
                     double defocus_ang, double c3_ang, double c5_ang, float* probe,
                     void* workspace, size_t workspace_bytes, void* stream);

/* Workspace bytes for ptyro_fft2 / ptyro_make_probe at edge n. */
size_t ptyro_fft_workspace_bytes(int32_t n);

/* In-place batched 2-D FFT of `count` contiguous complex64 (n, n) planes, with
 * numpy/JAX conventions: inverse != 0 gives ifft2 (1/n^2 scaling), else fft2.
 * Stands in for the jnp.fft.fft2/ifft2 calls of the path (simulations.py:429,
 * :585-589, :601, :1287, :1319). */
int ptyro_fft2(int32_t n, int32_t count, int32_t inverse, float* data, void* workspace,
               size_t workspace_bytes, void* stream);

/* Engine kernels enqueued by this process so far (all threads and devices).
 * Lets a caller count the launches of a timed region. */
unsigned long long ptyro_launch_count(void);

/* Device-side waits of the pass kernels (the TMA copies of the column passes,
 * tune bit 2048) that gave up after their poll limit on the current device, summed
 * over grid edges; 0 means every copy completed. No counterpart in the reference (a health
 * check of this engine's bounded waits). */
unsigned int ptyro_pass_wait_timeouts(void);

/* `reps` launches of the steady-state pass (finish slice s-1's convolution along
 * `axis`, multiply T_1, start slice s's convolution) over the batch of wave slots
 * held in `workspace` by a preceding ptyro_ms_forward with the same `p`. The
 * workspace must hold finite values. Used to time the dominant kernel alone; the
 * reference has no counterpart (its slice step is _scan_fn, simulations.py:544-597). */
int ptyro_ms_steady_pass(const ptyro_ms_params* p, int32_t axis, int32_t reps, void* workspace,
                         size_t workspace_bytes, void* stream);

/* Diagnostic: `blocks` x 256 threads each run iters*128 dependent-free FP32 FMAs
 * and write one float to out[blocks*256]. FLOPs = blocks*256*iters*256. Measures
 * the FP32 ceiling used as the roofline denominator; no reference counterpart. */
int ptyro_fp32_fma_probe(float* out, int32_t blocks, int32_t iters, void* stream);

/* Self-test of the bounded tile wait the TMA column passes use: one CTA of `warps`
 * warps (1..32) arms an mbarrier for a copy that is never issued, so every warp's
 * wait gives up after `polls` polls (1..2^20) and takes the pass kernels' give-up
 * path: the warp skips its work, *skipped_warps (DEVICE int32) counts it and
 * PTYRO_STATUS_WAIT_TIMEOUT is ORed into *status (DEVICE uint32). Nothing is in
 * flight when the CTA exits. No counterpart in the reference. */
int ptyro_test_wait_timeout(int32_t warps, int32_t polls, uint32_t* status, int32_t* skipped_warps,
                            void* stream);

/* Projected potential of one atom, averaged from a supersampled grid: replaces
 * single_atom_potential (src/ptyrodactyl/multislice/atom_potentials.py:588-681) with
 * lobato_projected_potential / kirkland_projected_potential
 * (src/ptyrodactyl/multislice/form_factors.py:322-439).
 *   parameterization  0 = Lobato--Van Dyck, 1 = Kirkland
 *   coeffs            HOST double: Lobato a1..a5, b1..b5 (10 values); Kirkland a1, b1,
 *                     a2, b2, a3, b3 (Lorentzian), c1, d1, c2, d2, c3, d3 (Gaussian) (12)
 *   pixel_size        Angstrom; the supersampled step is pixel_size / supersampling
 *   h, w              output grid; supersampled point k of an axis of K = edge *
 *                     supersampling points sits at (k - K/2) * step
 *   center_x, center_y  the atom's position, Angstrom (0, 0: the supersampled grid's centre)
 *   out               DEVICE float64 (h, w), volt-Angstrom: the mean of each pixel's
 *                     supersampling^2 values */
int ptyro_atom_potential(int32_t parameterization, const double* coeffs, double pixel_size, int32_t h, int32_t w,
                         double center_x, double center_y, int32_t supersampling, double* out, void* stream);

/* ---- Any grid size. The entry points above take square power-of-two grids 16..1024
 * (p->n). These take any height x width (each 1..4096), as the reference does
 * (fftfreq of any size, simulations.py:162-225; any probe_shape), with p->n ignored,
 * no potential-field windows, and every slice's wave kept as a residual (checkpoint
 * spacing 1). The 1-D transforms are four-step DFTs with direct sums (N1 + N2 complex
 * multiply-adds per point for N = N1 N2), slower than the fused path; results follow
 * the same arithmetic (stem_4d, simulations.py:1330-1443, and its jax.grad). */
size_t ptyro_gm_workspace_bytes(const ptyro_ms_params* p, int32_t height, int32_t width);

/* Residual bytes ptyro_gm_forward writes when `residuals` is not NULL: per (probe,
 * mode) the wave after each of the S transmission multiplies and the far-field
 * amplitude, (P, M, S + 1, height, width) complex64. */
size_t ptyro_gm_residual_bytes(const ptyro_ms_params* p, int32_t height, int32_t width);

/* ptyro_ms_forward / ptyro_ms_forward_ckpt on a height x width grid: patterns (P, H, W)
 * fftshifted (odd sizes shift by floor(N/2), as numpy's fftshift); residuals NULL or
 * ptyro_gm_residual_bytes. p->flags PTYRO_FLAG_ACCUMULATE adds into patterns. */
int ptyro_gm_forward(const ptyro_ms_params* p, int32_t height, int32_t width, const float* potential,
                     const float* modes, const float* weights, const double* positions, float* patterns,
                     float* residuals, void* workspace, size_t workspace_bytes, void* stream);

size_t ptyro_gm_backward_workspace_bytes(const ptyro_ms_params* p, int32_t height, int32_t width);

/* ptyro_ms_backward(_positions) on a height x width grid, from ptyro_gm_forward's
 * residuals: dL/dV (potential strides), the modes' gradient in JAX's convention, and
 * dL/d(positions) (P, 2) when grad_positions is not NULL (then modes is needed). */
int ptyro_gm_backward(const ptyro_ms_params* p, int32_t height, int32_t width, const float* potential,
                      const float* modes, const float* weights, const double* positions, const float* residuals,
                      const float* grad_patterns, float* grad_potential, float* grad_modes, double* grad_positions,
                      void* workspace, size_t workspace_bytes, void* stream);

/* ptyro_ms_jvp on a height x width grid: patterns (NULL or (P, H, W)) and their
 * directional derivative `tangent` (P, H, W) along (tangent_potential, tangent_modes),
 * either of which may be NULL (zero); tangents have the potential's / modes' strides. */
size_t ptyro_gm_jvp_workspace_bytes(const ptyro_ms_params* p, int32_t height, int32_t width);
int ptyro_gm_jvp(const ptyro_ms_params* p, int32_t height, int32_t width, const float* potential,
                 const float* tangent_potential, const float* modes, const float* tangent_modes, const float* weights,
                 const double* positions, float* patterns, float* tangent, void* workspace, size_t workspace_bytes,
                 void* stream);

/* numpy fft2 / ifft2 of `count` contiguous height x width complex64 planes in place,
 * any height and width in [1, 4096] (inverse scaled by 1 / (height width)). */
size_t ptyro_gm_fft_workspace_bytes(int32_t height, int32_t width);
int ptyro_gm_fft2(int32_t height, int32_t width, int32_t count, int32_t inverse, float* data, void* workspace,
                  size_t workspace_bytes, void* stream);

/* make_probe (simulations.py:334-431) for any probe_shape (height x width, 1..4096 each):
 * the aperture and aberration on the reference's rolled-arange frequency grid, ifft2
 * and ifftshift; probe (height, width) complex64. */
size_t ptyro_gm_make_probe_workspace_bytes(int32_t height, int32_t width);
int ptyro_gm_make_probe(int32_t height, int32_t width, double voltage_kv, double aperture_mrad,
                        double probe_calibration_pm, double defocus_ang, double c3_ang, double c5_ang, float* probe,
                        void* workspace, size_t workspace_bytes, void* stream);

/* ptyro_ms_weight_grad from ptyro_gm_forward's residuals. */
size_t ptyro_gm_weight_grad_workspace_bytes(const ptyro_ms_params* p, int32_t height, int32_t width);
int ptyro_gm_weight_grad(const ptyro_ms_params* p, int32_t height, int32_t width, const float* residuals,
                         const float* grad_patterns, double* grad_weights, void* workspace, size_t workspace_bytes,
                         void* stream);

/* Workspace bytes of ptyro_atom_slices for edge n and num_types atom types. */
size_t ptyro_atom_slices_workspace_bytes(int32_t n, int32_t num_types);

/* Potential slices built on the device from atoms, the slice builder of the
 * reference's atom-backed path (_compute_slice_potential,
 * src/ptyrodactyl/multislice/parallelized.py:54-169; used by stem4d_sharded :348).
 *   atom_coords     DEVICE float64 (N, 3) x, y, z in Angstrom
 *   atom_types      DEVICE int32 (N) indices into atom_potentials
 *   slice_z_bounds  HOST float64 (S, 2) [z_min, z_max) per slice
 *   atom_potentials DEVICE float32 (T, n, n) per-type projected potentials (V A)
 *   atom_mask       DEVICE float32 (N) inclusion weights, or NULL
 *   slices          DEVICE float32 out, V[y][x][s] at strides (sy, sx, ss)
 * Atoms land on floor(coord / calib) mod n; each type's delta grid is circularly
 * convolved with its kernel (FFT), and the types are summed. */
int ptyro_atom_slices(int32_t n, int32_t num_atoms, int32_t num_types, int32_t num_slices, const double* atom_coords,
                      const int32_t* atom_types, const double* slice_z_bounds, const float* atom_potentials,
                      const float* atom_mask, double calib_ang, float* slices, int64_t sy, int64_t sx, int64_t ss,
                      void* workspace, size_t workspace_bytes, void* stream);

/* Workspace bytes of ptyro_place_atoms (0 when invalid). */
size_t ptyro_place_atoms_workspace_bytes(int32_t n, int32_t num_types, int32_t num_atoms);

/* Sub-pixel placement of crystal_potential_slices (src/ptyrodactyl/multislice/
 * atom_potentials.py:826-994): slice s = real(ifft2(sum over its atoms of
 * fft2(P_type) exp(2 pi i (kx shift_x + ky shift_y)))), k = fftfreq(n) per pixel.
 *   shift_y, shift_x   float64 device (num_atoms): the atom's offset from the grid
 *                      centre in pixels ((coord - min) / pixel_size - n / 2)
 *   group_offsets_host int32 HOST (num_slices * num_types + 1): the atoms are sorted
 *                      by (slice, type); group g = s * num_types + t holds atoms
 *                      [offsets[g], offsets[g+1])
 *   atom_potentials    float32 device (num_types, n, n) per-type lookup potentials
 *   slices             float32 (n, n, num_slices) written with strides (sy, sx, ss) */
int ptyro_place_atoms(int32_t n, int32_t num_atoms, int32_t num_types, int32_t num_slices, const double* shift_y,
                      const double* shift_x, const int32_t* group_offsets_host, const float* atom_potentials,
                      float* slices, int64_t sy, int64_t sx, int64_t ss, void* workspace, size_t workspace_bytes,
                      void* stream);

/* Scratch bytes of ptyro_clip_resize: a (P, hc, wo) float32 intermediate. */
size_t ptyro_clip_resize_workspace_bytes(int64_t num_patterns, int32_t hc, int32_t wo);

/* clip_cbed (src/ptyrodactyl/plots/figuring.py:37-117) over P stored float32 patterns
 * (P, h, w): the crop rows [y0, y0 + hc) and columns [x0, x0 + wc), resized by the
 * separable weight matrices wy (ho, hc) and wx (wo, wc) (row-major float32: output
 * index major) into out (P, ho, wo). The caller builds the weights of the resize
 * method (jax.image.resize "linear" for the reference). */
int ptyro_clip_resize(const float* patterns, int64_t num_patterns, int32_t h, int32_t w, int32_t y0, int32_t x0,
                      int32_t hc, int32_t wc, const float* wy, int32_t ho, const float* wx, int32_t wo, float* out,
                      void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------- scheduler
 * Continuous batching of forward and gradient jobs of any grid edge, slice count
 * and scan size (the batching and serving patterns; no reference counterpart:
 * the reference runs one jitted stem_4d call at a time). Jobs wait until their
 * scratch fits in the caller-provided arena and their probes in flight fit the slot
 * budget; each ptyro_sched_step advances every running job by one pass, the
 * passes of all running jobs with the same grid edge going out as one multi-job
 * launch per (forward/adjoint, axis). Inputs and outputs are the caller's device
 * buffers; they must stay valid until the job is DONE, FAILED or CANCELLED. */
#define PTYRO_JOB_FORWARD 0
#define PTYRO_JOB_GRADIENT 1

#define PTYRO_JOB_QUEUED 0
#define PTYRO_JOB_RUNNING 1
#define PTYRO_JOB_DONE 2
#define PTYRO_JOB_FAILED 3
#define PTYRO_JOB_CANCELLED 4

typedef struct ptyro_sched ptyro_sched;

typedef struct ptyro_job_desc {
  ptyro_ms_params p;          /* geometry; p.batch = probes in flight (0 = automatic) */
  int32_t kind;               /* PTYRO_JOB_FORWARD or PTYRO_JOB_GRADIENT */
  int32_t ckpt_every;         /* gradient jobs: checkpoint spacing (0 = ceil(sqrt(S))) */
  const float* potential;     /* as ptyro_ms_forward */
  const float* modes;
  const float* weights;
  const double* positions;
  float* patterns;            /* out (P, n, n) */
  const float* targets;       /* gradient jobs: measured patterns (P, n, n), fftshifted */
  float* grad_potential;      /* gradient jobs, out: d(loss)/dV with the potential's strides */
  float* grad_modes;          /* gradient jobs, out: JAX-convention gradient of the modes */
  float* loss;                /* gradient jobs, out: amplitude loss sum (sqrt(I) - sqrt(target))^2 */
  void* ready_event;          /* optional cudaEvent_t: the job's inputs are ready once it completes */
} ptyro_job_desc;

/* Device scratch bytes a job takes from the arena while it runs (0 if invalid). */
size_t ptyro_sched_job_bytes(const ptyro_job_desc* d);

/* New scheduler on `device` (must be current) with `arena` (DEVICE, 256-byte
 * aligned) as its only device memory and at most `max_slots` wave slots in flight. */
int ptyro_sched_create(int32_t device, void* arena, size_t arena_bytes, int32_t max_slots, ptyro_sched** out);

/* Waits for all issued work and frees the scheduler's host resources. */
int ptyro_sched_destroy(ptyro_sched* s);

/* Queue a job (copied); `*id` identifies it. Invalid jobs, and jobs larger than
 * the arena, are rejected here. Thread-safe. */
int ptyro_sched_submit(ptyro_sched* s, const ptyro_job_desc* d, int64_t* id);

/* Cancel a queued or running job (running: no further passes are issued). */
int ptyro_sched_cancel(ptyro_sched* s, int64_t id);

/* Retire finished jobs, admit queued ones, issue one pass of every running job. */
int ptyro_sched_step(ptyro_sched* s, int32_t* running, int32_t* queued);

/* PTYRO_JOB_* state of a job. Thread-safe. */
int ptyro_sched_job_state(ptyro_sched* s, int64_t id, int32_t* state);

/* Forget a finished job. */
int ptyro_sched_release(ptyro_sched* s, int64_t id);

/* Free arena bytes and free wave slots. */
int ptyro_sched_memory(ptyro_sched* s, size_t* free_bytes, int32_t* free_slots);

/* Recorded batch plans: a fixed set of jobs (any mix of grid edges, slice counts,
 * scan sizes, forward and gradient; no ready events) run as the scheduler runs them,
 * every job advancing one pass per tick in the same multi-job launches, but
 * recorded once. ptyro_plan_create simulates the ticks on the host and copies every
 * tick's descriptors into the arena (a synchronous copy: call it outside stream
 * capture); ptyro_plan_launch then only enqueues kernels and memsets on `stream`,
 * so it can be captured into a CUDA graph and replayed; each launch recomputes every
 * job from its current inputs. The jobs of each grid edge run on a stream of the
 * plan's own, forked from `stream` and joined back to it with events (a captured
 * graph gets one branch per grid edge). Results are bit-identical to the same jobs run
 * through ptyro_sched_*. The arena (DEVICE, 256-byte aligned, ptyro_plan_bytes)
 * holds every job's scratch at once; one launch at a time per plan. */
typedef struct ptyro_plan ptyro_plan;
size_t ptyro_plan_bytes(const ptyro_job_desc* jobs, int32_t num_jobs);
int ptyro_plan_create(int32_t device, const ptyro_job_desc* jobs, int32_t num_jobs, void* arena, size_t arena_bytes,
                      ptyro_plan** out);
int ptyro_plan_launch(ptyro_plan* plan, void* stream);
/* Device address of job `job`'s status word (uint32, PTYRO_STATUS_* bits; cleared by
 * every launch of the plan). */
int ptyro_plan_job_status(const ptyro_plan* plan, int32_t job, void** status_word);
int ptyro_plan_destroy(ptyro_plan* plan);

/* Bytes of the fixed device scratch array behind ptyro_ms_forward_noalloc. */
#define PTYRO_STATIC_SCRATCH_BYTES (64u * 1024u * 1024u)

/* Forward model that allocates nothing and takes no workspace, for callers that
 * cannot allocate device memory: a host that owns all of it (an XLA FFI handler
 * without a workspace operand, a fixed-budget plugin host) or code running during
 * CUDA stream capture, where cudaMalloc is not allowed. No counterpart in the
 * reference (JAX allocates for its own path).
 * Same arguments and results as ptyro_ms_forward minus the workspace; the scratch
 * is a PTYRO_STATIC_SCRATCH_BYTES array in the library's device image, held on
 * every GPU that loads the library until exit. Every call made outside stream
 * capture looks up that array's address on the current device; captured calls reuse
 * it, so make one call on each device before any stream capture. Calls on a device
 * share the array, so calls that overlap on the GPU race: serialise them on one
 * stream. The batch is the largest that fits; when not one probe fits with the
 * default variant's optional interleaved transmission tables, they are left out
 * (bit-identical results). Jobs whose scratch still does not fit (e.g. a 1024^2 grid
 * with many slices) are rejected with PTYRO_ERR_WORKSPACE before anything is
 * launched. The call has no way to return the device status word, so if a bounded
 * wait inside the forward gave up, `patterns` is filled with NaN. */
int ptyro_ms_forward_noalloc(const ptyro_ms_params* p, const float* potential, const float* modes,
                             const float* weights, const double* positions, float* patterns, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PTYRO_B200_H */
