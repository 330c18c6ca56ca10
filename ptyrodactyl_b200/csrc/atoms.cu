// On-device potential slices from atoms: the slice builder of the reference's
// atom-backed path (_compute_slice_potential, src/ptyrodactyl/multislice/parallelized.py:54-169).
// Per slice: scatter the atoms with z_min <= z < z_max to floor(coord / calib) mod n
// per type, FFT2 the type planes, multiply by each type's kernel spectrum and sum,
// IFFT2, keep the real part.
#include "engine.cuh"

namespace ptyro {

static __global__ void k_real_to_complex(const float* __restrict__ src, size_t count, float2* __restrict__ dst) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = make_float2(src[i], 0.f);
}

// atoms of the slice add their weight at their pixel; weights are 1 unless a mask is
// given, so the sums are exact whatever the order of the additions
static __global__ void k_scatter_atoms(const double* __restrict__ coords, const int* __restrict__ types,
                                       const float* __restrict__ mask, int num_atoms, int num_types, double z_min,
                                       double z_max, double calib, int n, float2* __restrict__ delta) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= num_atoms) return;
  const double z = coords[3 * i + 2];
  if (!(z >= z_min && z < z_max)) return;
  const int t = types[i];
  if (t < 0 || t >= num_types) return;
  const float wgt = mask ? mask[i] : 1.0f;
  long long xi = (long long)floor(coords[3 * i + 0] / calib) % n;
  long long yi = (long long)floor(coords[3 * i + 1] / calib) % n;
  if (xi < 0) xi += n;
  if (yi < 0) yi += n;
  atomicAdd(&delta[((size_t)t * n + yi) * n + xi].x, wgt);
}

static __global__ void k_combine_types(const float2* __restrict__ delta_k, const float2* __restrict__ kern_k,
                                       int num_types, size_t nn, float2* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (size_t)gridDim.x * blockDim.x) {
    float2 acc = make_float2(0.f, 0.f);
    for (int t = 0; t < num_types; ++t) acc = cadd(acc, cmul(delta_k[t * nn + i], kern_k[t * nn + i]));
    out[i] = acc;
  }
}

static __global__ void k_store_slice(const float2* __restrict__ c, int n, float* __restrict__ slices, long long sy,
                                     long long sx, long long ss, int s) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)n * n) return;
  const int y = (int)(i / n), x = (int)(i % n);
  slices[(long long)y * sy + (long long)x * sx + (long long)s * ss] = c[i].x;
}

// ---------------------------------------------------------------- sub-pixel placement
// crystal_potential_slices (src/ptyrodactyl/multislice/atom_potentials.py:826-994,
// 1364-1510): every atom adds real(ifft2(fft2(P_type) exp(2 pi i (kx sx + ky sy))))
// to its slice, k = fftfreq(n) in cycles per pixel, (sy, sx) the atom's offset from
// the grid centre in pixels. Summed over the atoms of a slice this is
// real(ifft2(sum_t fft2(P_t) Z_t)) with the structure factor
// Z_t(ky, kx) = sum over the slice's type-t atoms of e_y(ky) e_x(kx), a complex
// product of per-atom phase tables (a small GEMM over atoms, computed here in FP32
// with tiles of the tables in shared memory).

// per-atom phase tables: ex[a][j] = exp(2 pi i k_j sx_a), ey likewise (double-precision argument)
static __global__ void k_phase_tables(const double* __restrict__ sy, const double* __restrict__ sx, int num_atoms,
                                      int n, float2* __restrict__ ey, float2* __restrict__ ex) {
  const size_t total = (size_t)num_atoms * n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int a = (int)(i / n), j = (int)(i % n);
    const double kj = (double)(j < n / 2 ? j : j - n);  // fftfreq numerator
    double s, c;
    sincospi(2.0 * kj * sy[a] / n, &s, &c);
    ey[i] = make_float2((float)c, (float)s);
    sincospi(2.0 * kj * sx[a] / n, &s, &c);
    ex[i] = make_float2((float)c, (float)s);
  }
}

// Z(ky, kx) = sum_{a in [a0, a1)} ey[a][ky] ex[a][kx]; one 16 x 16 tile per CTA (256 threads)
constexpr int kSfChunk = 32;
static __global__ void __launch_bounds__(256) k_structure_factor(const float2* __restrict__ ey,
                                                                 const float2* __restrict__ ex, int a0, int a1, int n,
                                                                 float2* __restrict__ z) {
  __shared__ float2 sey[kSfChunk][16];
  __shared__ float2 sex[kSfChunk][16];
  const int ky0 = blockIdx.y * 16, kx0 = blockIdx.x * 16;
  const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
  float2 acc = make_float2(0.f, 0.f);
  for (int c0 = a0; c0 < a1; c0 += kSfChunk) {
    const int cnt = a1 - c0 < kSfChunk ? a1 - c0 : kSfChunk;
    for (int i = threadIdx.x; i < cnt * 16; i += 256) {
      const int r = i / 16, k = i % 16;
      sey[r][k] = ey[(size_t)(c0 + r) * n + ky0 + k];
      sex[r][k] = ex[(size_t)(c0 + r) * n + kx0 + k];
    }
    __syncthreads();
    for (int r = 0; r < cnt; ++r) {
      const float2 a = sey[r][ty], b = sex[r][tx];
      acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
      acc.y = fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y));
    }
    __syncthreads();
  }
  z[(size_t)(ky0 + ty) * n + kx0 + tx] = acc;
}

}  // namespace ptyro

using namespace ptyro;

extern "C" {

size_t ptyro_atom_slices_workspace_bytes(int32_t n, int32_t num_types) {
  if (n <= 0 || num_types <= 0) return 0;
  const size_t nn = (size_t)n * n;
  return align_up(8 * (size_t)n) + 2 * align_up(8 * nn * num_types) + align_up(8 * nn);
}

int ptyro_atom_slices(int32_t n, int32_t num_atoms, int32_t num_types, int32_t num_slices, const double* atom_coords,
                      const int32_t* atom_types, const double* slice_z_bounds_host, const float* atom_potentials,
                      const float* atom_mask, double calib_ang, float* slices, int64_t sy, int64_t sx, int64_t ss,
                      void* workspace, size_t workspace_bytes, void* stream) {
  Shape sh;
  if (!shape_for(n, &sh)) return fail(PTYRO_ERR_UNSUPPORTED, "atom slices: n must be a power of two in [16, 1024]");
  if (num_atoms < 0 || num_types < 1 || num_slices < 1)
    return fail(PTYRO_ERR_INVALID, "atom slices: need num_atoms >= 0, num_types >= 1, num_slices >= 1");
  if (!(calib_ang > 0)) return fail(PTYRO_ERR_INVALID, "calib must be > 0");
  if ((num_atoms && (!atom_coords || !atom_types)) || !slice_z_bounds_host || !atom_potentials || !slices)
    return fail(PTYRO_ERR_INVALID, "NULL array argument");
  const size_t need = ptyro_atom_slices_workspace_bytes(n, num_types);
  if (!workspace || workspace_bytes < need || ((uintptr_t)workspace & 255))
    return fail(PTYRO_ERR_WORKSPACE, "atom slices: workspace too small or misaligned: need " + std::to_string(need));
  cudaStream_t st = (cudaStream_t)stream;
  const size_t nn = (size_t)n * n;
  char* ws = (char*)workspace;
  float2* tw = (float2*)ws;
  float2* kern = (float2*)(ws + align_up(8 * (size_t)n));
  float2* delta = (float2*)((char*)kern + align_up(8 * nn * num_types));
  float2* acc = (float2*)((char*)delta + align_up(8 * nn * num_types));
  k_twiddle<<<(n + 255) / 256, 256, 0, st>>>(n, tw);
  k_real_to_complex<<<blocks_for(nn * num_types, 256), 256, 0, st>>>(atom_potentials, nn * num_types, kern);
  int rc = check_launch("atom slices setup", 2);
  if (rc) return rc;
  if ((rc = fft2_planes(n, num_types, false, kern, tw, st))) return rc;
  for (int s = 0; s < num_slices; ++s) {
    k_zero2<<<blocks_for(nn * num_types, 256), 256, 0, st>>>(delta, nn * num_types);
    if (num_atoms > 0)
      k_scatter_atoms<<<(num_atoms + 255) / 256, 256, 0, st>>>(atom_coords, atom_types, atom_mask, num_atoms,
                                                               num_types, slice_z_bounds_host[2 * s],
                                                               slice_z_bounds_host[2 * s + 1], calib_ang, n, delta);
    if ((rc = check_launch("k_scatter_atoms", num_atoms > 0 ? 2 : 1))) return rc;
    if ((rc = fft2_planes(n, num_types, false, delta, tw, st))) return rc;
    k_combine_types<<<blocks_for(nn, 256), 256, 0, st>>>(delta, kern, num_types, nn, acc);
    if ((rc = check_launch("k_combine_types"))) return rc;
    if ((rc = fft2_planes(n, 1, true, acc, tw, st))) return rc;
    k_store_slice<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(acc, n, slices, sy, sx, ss, s);
    if ((rc = check_launch("k_store_slice"))) return rc;
  }
  return PTYRO_OK;
}

size_t ptyro_place_atoms_workspace_bytes(int32_t n, int32_t num_types, int32_t num_atoms) {
  if (n <= 0 || num_types <= 0 || num_atoms < 0) return 0;
  const size_t nn = (size_t)n * n;
  return align_up(8 * (size_t)n) + 2 * align_up(8 * nn * num_types) + align_up(8 * nn) +
         2 * align_up(8 * (size_t)n * (num_atoms > 0 ? num_atoms : 1));
}

int ptyro_place_atoms(int32_t n, int32_t num_atoms, int32_t num_types, int32_t num_slices, const double* shift_y,
                      const double* shift_x, const int32_t* group_offsets_host, const float* atom_potentials,
                      float* slices, int64_t sy, int64_t sx, int64_t ss, void* workspace, size_t workspace_bytes,
                      void* stream) {
  Shape sh;
  if (!shape_for(n, &sh)) return fail(PTYRO_ERR_UNSUPPORTED, "place atoms: n must be a power of two in [16, 1024]");
  if (num_atoms < 0 || num_types < 1 || num_slices < 1)
    return fail(PTYRO_ERR_INVALID, "place atoms: need num_atoms >= 0, num_types >= 1, num_slices >= 1");
  if ((num_atoms && (!shift_y || !shift_x)) || !group_offsets_host || !atom_potentials || !slices)
    return fail(PTYRO_ERR_INVALID, "NULL array argument");
  const int groups = num_slices * num_types;
  if (group_offsets_host[0] != 0 || group_offsets_host[groups] != num_atoms)
    return fail(PTYRO_ERR_INVALID, "place atoms: group offsets must run from 0 to num_atoms");
  for (int g = 0; g < groups; ++g)
    if (group_offsets_host[g + 1] < group_offsets_host[g])
      return fail(PTYRO_ERR_INVALID, "place atoms: group offsets must not decrease");
  const size_t need = ptyro_place_atoms_workspace_bytes(n, num_types, num_atoms);
  if (!workspace || workspace_bytes < need || ((uintptr_t)workspace & 255))
    return fail(PTYRO_ERR_WORKSPACE, "place atoms: workspace too small or misaligned: need " + std::to_string(need));
  cudaStream_t st = (cudaStream_t)stream;
  const size_t nn = (size_t)n * n;
  char* ws = (char*)workspace;
  float2* tw = (float2*)ws;
  float2* kern = (float2*)(ws + align_up(8 * (size_t)n));
  float2* zs = (float2*)((char*)kern + align_up(8 * nn * num_types));
  float2* acc = (float2*)((char*)zs + align_up(8 * nn * num_types));
  float2* ey = (float2*)((char*)acc + align_up(8 * nn));
  float2* ex = (float2*)((char*)ey + align_up(8 * (size_t)n * (num_atoms > 0 ? num_atoms : 1)));
  k_twiddle<<<(n + 255) / 256, 256, 0, st>>>(n, tw);
  k_real_to_complex<<<blocks_for(nn * num_types, 256), 256, 0, st>>>(atom_potentials, nn * num_types, kern);
  int launches = 2;
  if (num_atoms > 0) {
    k_phase_tables<<<blocks_for((size_t)num_atoms * n, 256), 256, 0, st>>>(shift_y, shift_x, num_atoms, n, ey, ex);
    ++launches;
  }
  int rc = check_launch("place atoms setup", launches);
  if (rc) return rc;
  if ((rc = fft2_planes(n, num_types, false, kern, tw, st))) return rc;
  const dim3 grid(n / 16, n / 16);
  for (int s = 0; s < num_slices; ++s) {
    for (int t = 0; t < num_types; ++t) {
      const int a0 = group_offsets_host[s * num_types + t], a1 = group_offsets_host[s * num_types + t + 1];
      k_structure_factor<<<grid, 256, 0, st>>>(ey, ex, a0, a1, n, zs + (size_t)t * nn);
    }
    if ((rc = check_launch("k_structure_factor", num_types))) return rc;
    k_combine_types<<<blocks_for(nn, 256), 256, 0, st>>>(zs, kern, num_types, nn, acc);
    if ((rc = check_launch("k_combine_types"))) return rc;
    if ((rc = fft2_planes(n, 1, true, acc, tw, st))) return rc;
    k_store_slice<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(acc, n, slices, sy, sx, ss, s);
    if ((rc = check_launch("k_store_slice"))) return rc;
  }
  return PTYRO_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- CBED clip + resize
// clip_cbed (src/ptyrodactyl/plots/figuring.py:37-117) over a batch of stored
// patterns: the central crop [y0, y0 + hc) x [x0, x0 + wc), then a separable linear
// resize given as dense weight matrices wy (ho x hc) and wx (wo x wc), applied along
// x into a (P, hc, wo) scratch and then along y.
namespace ptyro {

static __global__ void k_resize_x(const float* __restrict__ pat, int h, int w, int y0, int x0, int hc, int wc,
                                  const float* __restrict__ wx, int wo, size_t count, float* __restrict__ tmp) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const int ox = (int)(i % wo);
    const int iy = (int)((i / wo) % hc);
    const size_t p = i / ((size_t)wo * hc);
    const float* row = pat + (p * h + (size_t)(y0 + iy)) * w + x0;
    const float* wr = wx + (size_t)ox * wc;
    float acc = 0.f;
    for (int ix = 0; ix < wc; ++ix) acc = fmaf(wr[ix], row[ix], acc);
    tmp[i] = acc;
  }
}

static __global__ void k_resize_y(const float* __restrict__ tmp, int hc, int wo, const float* __restrict__ wy, int ho,
                                  size_t count, float* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const int ox = (int)(i % wo);
    const int oy = (int)((i / wo) % ho);
    const size_t p = i / ((size_t)wo * ho);
    const float* col = tmp + p * hc * wo + ox;
    const float* wr = wy + (size_t)oy * hc;
    float acc = 0.f;
    for (int iy = 0; iy < hc; ++iy) acc = fmaf(wr[iy], col[(size_t)iy * wo], acc);
    out[i] = acc;
  }
}

}  // namespace ptyro

extern "C" {

size_t ptyro_clip_resize_workspace_bytes(int64_t num_patterns, int32_t hc, int32_t wo) {
  if (num_patterns < 0 || hc <= 0 || wo <= 0) return 0;
  return align_up(4 * (size_t)(num_patterns > 0 ? num_patterns : 1) * hc * wo);
}

int ptyro_clip_resize(const float* patterns, int64_t num_patterns, int32_t h, int32_t w, int32_t y0, int32_t x0,
                      int32_t hc, int32_t wc, const float* wy, int32_t ho, const float* wx, int32_t wo, float* out,
                      void* workspace, size_t workspace_bytes, void* stream) {
  if (num_patterns < 0 || h <= 0 || w <= 0 || hc <= 0 || wc <= 0 || ho <= 0 || wo <= 0)
    return fail(PTYRO_ERR_INVALID, "clip resize: sizes must be positive");
  if (y0 < 0 || x0 < 0 || y0 + hc > h || x0 + wc > w)
    return fail(PTYRO_ERR_INVALID, "clip resize: the crop must lie inside the pattern");
  if (num_patterns == 0) return PTYRO_OK;
  if (!patterns || !wy || !wx || !out) return fail(PTYRO_ERR_INVALID, "NULL array argument");
  const size_t need = ptyro_clip_resize_workspace_bytes(num_patterns, hc, wo);
  if (!workspace || workspace_bytes < need)
    return fail(PTYRO_ERR_WORKSPACE, "clip resize: workspace too small: need " + std::to_string(need));
  cudaStream_t st = (cudaStream_t)stream;
  float* tmp = (float*)workspace;
  const size_t c1 = (size_t)num_patterns * hc * wo, c2 = (size_t)num_patterns * ho * wo;
  k_resize_x<<<blocks_for(c1, 256), 256, 0, st>>>(patterns, h, w, y0, x0, hc, wc, wx, wo, c1, tmp);
  k_resize_y<<<blocks_for(c2, 256), 256, 0, st>>>(tmp, hc, wo, wy, ho, c2, out);
  return check_launch("clip resize", 2);
}

}  // extern "C"
