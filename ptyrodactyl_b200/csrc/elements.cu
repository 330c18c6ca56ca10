// Projected potential of one atom on a supersampled grid, averaged to the target grid:
// single_atom_potential (src/ptyrodactyl/multislice/atom_potentials.py:588-681) with the
// Lobato--Van Dyck and Kirkland parametrisations (multislice/form_factors.py:322-439).
//
// One thread per output pixel evaluates the potential in double precision at the
// pixel's s x s supersampled points (coordinate (k - K/2) * pixel / s along each axis,
// K = edge * s, r = sqrt(dx^2 + dy^2 + 1e-10)) and averages them, as the reference's
// reshape-and-mean downsampling does. The modified Bessel functions K0 and K1 are the
// reference's own approximations (bessel_kv, atom_potentials.py:95-450): the
// polynomial forms of Abramowitz & Stegun 9.8.5 / 9.8.7 for x <= 2 (with I0 and I1),
// and 9.8.6 / 9.8.8 for x > 2, so the potentials agree with the reference's to
// rounding rather than only to those approximations' accuracy (~1e-7).
#include <cuda_runtime.h>
#include <math.h>

#include <atomic>
#include <string>

#include "../../include/ptyro_b200.h"

namespace ptyro {
extern std::atomic<unsigned long long> g_launches;
void set_error_message(const std::string& msg);

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kMottBethe = 47.87801;  // C_MB, volt Angstrom^2 (types/constants.py:104)

__device__ double bessel_k0_ref(double x) {
  if (x <= 2.0) {  // A&S 9.8.5: -ln(x/2) I0(x) + sum_k c_k (x^2/4)^k
    const double c[7] = {-0.57721566, 0.42278420, 0.23069756, 0.03488590, 0.00262698, 0.00010750, 0.00000740};
    const double x2 = (x * x) / 4.0;
    double p = 1.0, poly = 0.0;
    for (int k = 0; k < 7; ++k) {
      poly += c[k] * p;
      p *= x2;
    }
    return -log(x / 2.0) * cyl_bessel_i0(x) + poly;
  }
  const double y = 2.0 / x;  // A&S 9.8.6
  const double poly = 1.25331414 + y * (-0.07832358 + y * (0.02189568 + y * (-0.01062446 + y * (0.00587872 +
                                                                                                 y * (-0.00251540 + y * 0.00053208)))));
  return exp(-x) / sqrt(x) * poly;
}

__device__ double bessel_k1_ref(double x) {
  if (x <= 2.0) {  // A&S 9.8.7: ln(x/2) I1(x) + (1/x) sum_k d_k (x^2/4)^k
    const double d[7] = {1.0, 0.15443144, -0.67278579, -0.18156897, -0.01919402, -0.00110404, -0.00004686};
    const double x2 = (x * x) / 4.0;
    double p = 1.0, poly = 0.0;
    for (int k = 0; k < 7; ++k) {
      poly += d[k] * p;
      p *= x2;
    }
    return log(x / 2.0) * cyl_bessel_i1(x) + poly / x;
  }
  const double y = 2.0 / x;  // A&S 9.8.8
  const double poly = 1.25331414 + y * (0.23498619 + y * (-0.03655620 + y * (0.01504268 + y * (-0.00780353 +
                                                                                                y * (0.00325614 + y * -0.00068245)))));
  return exp(-x) / sqrt(x) * poly;
}

struct ElementCoeffs {
  double v[12];  // Lobato: a1..a5, b1..b5; Kirkland: a1, b1, a2, b2, a3, b3, c1, d1, c2, d2, c3, d3
};

// Lobato and Van Dyck (2014) Eq. 16: 2 pi C_MB sum_i [a_i / b_i K0(2 pi r / sqrt(b_i))
//                                               + a_i pi r / b_i^1.5 K1(2 pi r / sqrt(b_i))]
__device__ double lobato_potential(const ElementCoeffs& c, double r) {
  double sum = 0.0;
  for (int i = 0; i < 5; ++i) {
    const double a = c.v[i], b = c.v[5 + i];
    const double arg = 2.0 * kPi * r / sqrt(b);
    sum += a / b * bessel_k0_ref(arg) + a * kPi * r / pow(b, 1.5) * bessel_k1_ref(arg);
  }
  return 2.0 * kPi * kMottBethe * sum;
}

// Kirkland: 4 pi^2 a0 e_k sum_i a_i K0(2 pi r sqrt(b_i)) + 2 pi^2 a0 e_k sum_i c_i / d_i exp(-pi^2 r^2 / d_i),
// with the reference's a0 = 0.5292, e_k = 14.4 and its term order
__device__ double kirkland_potential(const ElementCoeffs& c, double r) {
  double lt[3], gt[3];
  for (int i = 0; i < 3; ++i) {
    lt[i] = c.v[2 * i] * bessel_k0_ref(2.0 * kPi * r * sqrt(c.v[2 * i + 1]));
    const double ci = c.v[6 + 2 * i], di = c.v[7 + 2 * i];
    gt[i] = ci / di * exp(-(kPi * kPi) * (r * r) / di);
  }
  const double lpre = 4.0 * (kPi * kPi) * 0.5292 * 14.4, gpre = 2.0 * (kPi * kPi) * 0.5292 * 14.4;
  return lpre * (lt[0] + lt[1] + lt[2]) + gpre * (gt[0] + gt[1] + gt[2]);
}

__global__ void k_atom_potential(ElementCoeffs c, int kirkland, double pixel_size, int h, int w, double cx,
                                 double cy, int s, double* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)h * w) return;
  const int oy = (int)(i / w), ox = (int)(i % w);
  const double step = pixel_size / s;
  const int hs = h * s, ws = w * s;
  double acc = 0.0;
  for (int a = 0; a < s; ++a) {
    const double y = (double)(oy * s + a - hs / 2) * step;
    for (int b = 0; b < s; ++b) {
      const double x = (double)(ox * s + b - ws / 2) * step;
      const double dx = x - cx, dy = y - cy;
      double r = sqrt(dx * dx + dy * dy + 1e-10);
      r = fmax(r, 1e-10);
      acc += kirkland ? kirkland_potential(c, r) : lobato_potential(c, r);
    }
  }
  out[i] = acc / (double)(s * s);
}

}  // namespace
}  // namespace ptyro

extern "C" int ptyro_atom_potential(int32_t parameterization, const double* coeffs, double pixel_size, int32_t h,
                                    int32_t w, double center_x, double center_y, int32_t supersampling, double* out,
                                    void* stream) {
  using namespace ptyro;
  if (parameterization != 0 && parameterization != 1) {
    set_error_message("parameterization must be 0 (Lobato) or 1 (Kirkland)");
    return PTYRO_ERR_INVALID;
  }
  if (!coeffs || !out) {
    set_error_message("NULL array argument");
    return PTYRO_ERR_INVALID;
  }
  if (h < 1 || w < 1 || (long long)h * w > (1LL << 28) || supersampling < 1 || supersampling > 64 ||
      !(pixel_size > 0) || !isfinite(pixel_size)) {
    set_error_message("grid, supersampling and pixel size must be positive (grid <= 2^28 pixels, supersampling <= 64)");
    return PTYRO_ERR_INVALID;
  }
  ElementCoeffs c;
  const int count = parameterization == 0 ? 10 : 12;
  for (int k = 0; k < 12; ++k) c.v[k] = k < count ? coeffs[k] : 0.0;
  for (int k = 0; k < count; ++k) {
    const bool scale = parameterization == 0 ? k >= 5 : (k % 2 == 1);
    if (!isfinite(c.v[k]) || (scale && !(c.v[k] > 0))) {
      set_error_message("coefficients must be finite with positive scales");
      return PTYRO_ERR_INVALID;
    }
  }
  const long long total = (long long)h * w;
  k_atom_potential<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      c, parameterization, pixel_size, h, w, center_x, center_y, supersampling, out);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error_message(std::string("k_atom_potential: ") + cudaGetErrorString(e));
    return PTYRO_ERR_CUDA;
  }
  return PTYRO_OK;
}
