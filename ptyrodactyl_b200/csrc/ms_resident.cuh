// Wave-resident multislice forward for grids up to 128 x 128: one CTA per probe keeps
// the probe's complex64 wave in shared memory across all slices.
//
// The pass engine (ms_pass.cuh, ms_pair.cuh) moves every wave slot through L2/HBM
// once per slice. For N <= 128 the whole wave (128 KB at 128^2) fits in one CTA's
// shared memory, so here a CTA runs the same schedule of alternating row and column
// passes on its own wave without leaving the SM:
//   pass 0 (rows)        : x part of the IFFT2 of the shifted probe spectrum
//   pass k (1..S, k % 2) : [axis part of op_{k-1}]  x T_{k-1}  [axis part of op_k]
//   pass S+1             : last axis of the FFT2, w |.|^2, fftshifted store
// with a block barrier between passes. Each pass uses the paired line transforms of
// the pass engine (two lines per thread, f32x2 arithmetic, per-warp exchange buffers)
// with the same operations in the same order, so the patterns are bit-identical to
// the pass engine's. Only the transmission rows (shared by all probes, L2-resident)
// and the probe spectrum come from global memory; one launch runs a probe batch
// through every slice instead of S + 2 launches.
//
// Scope: N in {16, 32, 64, 128}, one probe mode, no potential field windows, no
// gradient residuals, detectors, tilts or amplitude output (the driver uses the
// pass engine for those).
#pragma once
#include <cuda_runtime.h>

namespace ptyro {

struct ResidentArgs {
  const float2* probe_k;  // (N, N) spectrum of the beam mode
  const float2* ramp_y;   // (B, N) shift ramp along y per probe of the batch
  const float2* ramp_x;   // (B, N) along x
  const float2* trans;    // (S, N, N) exp(i sigma V), row-major
  const float2* trans_t;  // (S, N, N) transposed
  const float2* pf;       // (N) propagator factor / N
  const float2* tw;       // (N) forward twiddles exp(-2 pi i j / N)
  const float* weights;   // (1) mode weight
  float* pattern;         // (B, N, N) fftshifted intensities of the batch
  int num_slices;
  int accumulate;         // add into pattern instead of overwriting
  float scale;            // 1 / N after an inverse transform
};

// Launch over the `nb` probes of a batch (one CTA each); returns a cudaError_t as int.
int launch_resident(int n, const ResidentArgs& a, int nb, cudaStream_t st);

// Shared memory one CTA of the resident kernel needs at edge n (0 if n is unsupported).
size_t resident_smem_bytes(int n);

}  // namespace ptyro
