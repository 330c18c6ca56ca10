// Generated by gen_unit_consts.py; do not edit by hand.
// float32 roots of unity W_64^r = exp(2 pi i r / 64) chosen among the neighbours
// of the exact values (phase error <= 4.5e-08 rad) so that the expected energy
// change of each transform built from them is close to zero.
#pragma once

namespace ptyro {

// factored butterfly twiddle M (1 + i T) for r = 0..8 (r > 8 uses 16 - r swapped)
__device__ __forceinline__ float bfly_m(int r) {
  switch (r) {
    case 0: return 1.0f;
    case 1: return 0.9951847195625305f;  // |w| - 1 = -7.42e-09, phase error -2.85e-09
    case 2: return 0.9807852506637573f;  // |w| - 1 = -2.18e-08, phase error +4.29e-08
    case 3: return 0.9569403529167175f;  // |w| - 1 = +2.07e-08, phase error +9.07e-09
    case 4: return 0.9238795638084412f;  // |w| - 1 = +2.53e-08, phase error -2.07e-08
    case 5: return 0.8819212913513184f;  // |w| - 1 = +1.12e-08, phase error -3.63e-08
    case 6: return 0.8314695954322815f;  // |w| - 1 = -1.98e-09, phase error +2.74e-08
    case 7: return 0.7730104327201843f;  // |w| - 1 = -7.42e-09, phase error +2.35e-08
    case 8: return 0.7071067690849304f;  // |w| - 1 = -1.71e-08, phase error +0.00e+00
    default: return 0.0f;
  }
}

__device__ __forceinline__ float bfly_t(int r) {
  switch (r) {
    case 0: return 0.0f;
    case 1: return 0.09849140048027039f;
    case 2: return 0.19891241192817688f;
    case 3: return 0.3033466935157776f;
    case 4: return 0.41421353816986084f;
    case 5: return 0.5345110893249512f;
    case 6: return 0.6681786775588989f;
    case 7: return 0.8206788301467896f;
    case 8: return 1.0f;
    default: return 0.0f;
  }
}

// cos and sin of 2 pi r / 64 for plain complex multiplies, r = 0..15
__device__ __host__ __forceinline__ float unit_c(int r) {
  switch (r) {
    case 0: return 1.0f;
    case 1: return 0.9951847195625305f;  // |w| - 1 = -4.80e-09, phase error +2.38e-08
    case 2: return 0.9807853102684021f;  // |w| - 1 = +2.67e-08, phase error -1.88e-08
    case 3: return 0.9569403529167175f;  // |w| - 1 = +2.97e-08, phase error +3.88e-08
    case 4: return 0.9238795638084412f;  // |w| - 1 = +2.65e-08, phase error -1.77e-08
    case 5: return 0.8819212317466736f;  // |w| - 1 = -2.53e-08, phase error +2.19e-08
    case 6: return 0.8314695954322815f;  // |w| - 1 = -7.49e-09, phase error +1.92e-08
    case 7: return 0.7730104327201843f;  // |w| - 1 = -2.19e-08, phase error +5.85e-09
    case 8: return 0.7071067690849304f;  // |w| - 1 = -1.71e-08, phase error +0.00e+00
    case 9: return 0.6343932747840881f;  // |w| - 1 = -2.19e-08, phase error -5.85e-09
    case 10: return 0.5555702447891235f;  // |w| - 1 = -7.49e-09, phase error -1.92e-08
    case 11: return 0.47139671444892883f;  // |w| - 1 = +1.33e-08, phase error +3.25e-08
    case 12: return 0.3826834261417389f;  // |w| - 1 = -2.85e-08, phase error -5.08e-09
    case 13: return 0.290284663438797f;  // |w| - 1 = +1.24e-08, phase error +1.82e-08
    case 14: return 0.19509029388427734f;  // |w| - 1 = +2.38e-08, phase error +3.34e-08
    case 15: return 0.09801716357469559f;  // |w| - 1 = -4.80e-09, phase error -2.38e-08
    default: return 0.0f;
  }
}

__device__ __host__ __forceinline__ float unit_s(int r) {
  switch (r) {
    case 0: return 0.0f;
    case 1: return 0.09801716357469559f;
    case 2: return 0.19509030878543854f;
    case 3: return 0.2902847230434418f;
    case 4: return 0.3826834261417389f;
    case 5: return 0.4713967442512512f;
    case 6: return 0.5555702447891235f;
    case 7: return 0.6343932747840881f;
    case 8: return 0.7071067690849304f;
    case 9: return 0.7730104327201843f;
    case 10: return 0.8314695954322815f;
    case 11: return 0.8819212913513184f;
    case 12: return 0.9238795042037964f;
    case 13: return 0.9569403529167175f;
    case 14: return 0.9807853102684021f;
    case 15: return 0.9951847195625305f;
    default: return 0.0f;
  }
}

// expected energy change per transform (spread-out data):
//    8-point DIT DFT: -8.56e-09
//   16-point DIT DFT: -1.76e-10
//   32-point DIT DFT: -1.93e-09
//   64th-root entries of the   16-point four-step table: -9.06e-09
//   64th-root entries of the   32-point four-step table: -3.37e-10
//   64th-root entries of the   64-point four-step table: -8.50e-10
//   64th-root entries of the  128-point four-step table: -4.02e-11
//   64th-root entries of the  256-point four-step table: +1.72e-10
//   64th-root entries of the  512-point four-step table: -9.53e-11
//   64th-root entries of the 1024-point four-step table: -1.38e-10

}  // namespace ptyro
