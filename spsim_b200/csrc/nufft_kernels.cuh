// Non-uniform FFT structure factor (internal C++ interface).
//
// F(q_k) = sum_e f_e(|q_k|) sum_{j in e} w_j exp(-2 pi i q_k . r_j) for an
// arbitrary q list, as a type-3 non-uniform transform per element:
//   1. spread   b_l = sum_j w_j e^{-2 pi i C.x_j} psi1(l - x_j / h)  on a real-space
//               grid of n1 points per axis (x_j = r_j - centre, C = centre of the
//               q box, h = 1 / (2 sigma1 S), S = half-width of the q box)
//   2. pad      b_l / phi2hat((l - n1/2) / n2) into an n2 = sigma2 n1 grid at
//               index (l - n1/2) mod n2, zeros elsewhere
//   3. FFT      forward (e^{-2 pi i m p / n2}) over the n2 grid (cuFFT, batched
//               over elements), then packed as FP32 with the elements interleaved
//   4. interp   T(q') = sum_p g_p phi2(n2 h q' - p), F = e^{-2 pi i q.c}
//               sum_e f_e T_e(q') / prod_d psi1hat(h_d q'_d)
// psi1, phi2: "exponential of semicircle" kernels exp(beta (sqrt(1 - (2u/w)^2) - 1))
// of width w grid points; q' = q - C.  Spreading, FFT and the interpolation's
// row sums in FP64; the packed grid and its contraction along x in FP32.
#pragma once

#include <cuda_runtime.h>

#include "sf_device.cuh"

namespace spsim {

constexpr int NUFFT_MIN_W = 4;
constexpr int NUFFT_MAX_W = 16;  // spreading; the interpolation goes to 15
constexpr int NUFFT_MAX_COEF = 2 * NUFFT_MAX_W + 2;  // psi1hat trapezoid nodes at spacing 1/4 over [0, w/2]

struct NufftGeom {
  int n1[3];          // spreading grid points per axis (x, y, z), even
  int n2[3];          // FFT grid points per axis, even
  int w1, w2;         // kernel widths (grid points)
  double beta1, beta2;
  double inv_h[3];    // 1 / h (h: spreading grid spacing, m)
  double h[3];
  double L[3];        // h n2: q' (1/m) -> FFT-grid coordinate
  double cq[3];       // centre of the q box (1/m)
  double center[3];   // molecule centre (m)
};

struct NufftInterp {
  NufftGeom g;
  const float *hkl;   // AoS float3 q, or nullptr
  const double *q64;  // AoS double3 q, or nullptr
  long long npix;
  int tile_nx;        // > 0: the q list is a detector of rows of tile_nx pixels, taken in 16 x 8 tiles
  int has_rot;
  double rot[9];      // q' = R q (row-major)
  int npat;           // patterns (blockIdx.y); outputs [npat][npix]
  const double *rots; // device, 9 per pattern (row-major), or nullptr (then has_rot / rot)
  const float4 *packed;  // [n_groups][n2z][n2y][n2x][halves] (nufft_pack)
  long long cell2;       // n2x n2y n2z
  int halves;            // float4 per cell and group (two elements each)
  int n_groups;
  int n_elem;
  const float *coeffs;  // n_elem x 9 atomsf coefficients
  double B;
  int delta_atoms;
  int n_coef;           // psi1hat(xi) = sum_k a_k cos(2 pi xi k / 4)
  double psi_a[NUFFT_MAX_COEF];
  float2 *F;
  float *I;
};

// Bounding box of R q over a q list: out[0..2] = min, out[3..5] = max, as
// order-preserving 64-bit keys (initialise with nufft_bounds_init).
cudaError_t nufft_bounds(const float *hkl, const double *q64, long long npix, const double *rot,
                         unsigned long long *keys, cudaStream_t st);
double nufft_key_to_double(unsigned long long k);
unsigned long long nufft_double_to_key(double d);

// Step 1.  atoms: element-sorted FP64 records; seg: n_elem + 1 segment starts;
// grid (zeroed): `copies` x [n_elem][n1z][n1y][n1x], atom j adding into copy
// j mod copies (several copies spread the updates of one cell when the grid is
// small next to the atom count).  An atom whose stencil leaves the grid is
// skipped and sets err[0].
cudaError_t nufft_spread(const AtomD *atoms, const int *seg, int n_elem, int n_atoms, const NufftGeom &g,
                         double2 *grid, int copies, int *err, cudaStream_t st);
// Step 2: zero `fine` and scatter the deconvolved spreading grid (the sum of
// its copies) into it.  dec: 1 / phi2hat per spreading-grid index, x then y
// then z.
cudaError_t nufft_pad(const double2 *small, double2 *fine, const NufftGeom &g, int n_elem, int copies,
                      const double *dec, cudaStream_t st);
// Step 3b: FP32 element-interleaved copy of the FFT output for step 4
// (nufft_pack_groups(n_elem) x cells2 x nufft_pack_halves(n_elem) float4).
int nufft_pack_halves(int n_elem);
int nufft_pack_groups(int n_elem);
cudaError_t nufft_pack(const double2 *fine, float4 *packed, long long cells2, int n_elem, cudaStream_t st);
// Step 4.
cudaError_t nufft_interp(const NufftInterp &a, cudaStream_t st);

}  // namespace spsim
