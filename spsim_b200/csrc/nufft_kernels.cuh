// Non-uniform FFT structure factor (internal C++ interface).
//
// F(q_k) = sum_e f_e(|q_k|) sum_{j in e} w_j exp(-2 pi i q_k . r_j) for an
// arbitrary q list, as a type-3 non-uniform transform per element:
//   1. spread   b_l = sum_j w_j e^{-2 pi i C.x_j} psi1(l - x_j / h)  on a real-space
//               grid of n1 points per axis (x_j = r_j - centre, C = centre of the
//               q box, h = 1 / (2 sigma1 S), S = half-width of the q box)
//   2. pad      b_l / phi2hat((l - n1/2) / n2) into an n2 = sigma2 n1 grid at
//               index (l - n1/2) mod n2, zeros elsewhere
//   3. FFT      forward (e^{-2 pi i m p / n2}) over the n2 grid: pruned x, y, z
//               passes (steps 2 and 3 together, only the output box that step 4
//               reads), written as FP32 with the elements interleaved
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
  int pmin[3];        // FFT output box read by the interpolation: frequency indices
  int m[3];           // pmin .. pmin + m - 1 (taken mod n2), m along each axis
};

// One axis of the pruned FFT passes (nufft_fft.cu)
constexpr int NUFFT_FFT_MAX = 6144;  // longest transform: two FP64 lines in shared memory
struct FftAxis {
  int n;        // transform length (n2 along the axis)
  int nin;      // input points: spreading-grid index l at frequency index (l - nin/2) mod n
  int nout;     // output points: box index i from frequency index (p0 + i) mod n
  int p0;
  int ld;       // shared-memory line stride (double2): n (+ n/8 padding slots), 1 mod 8
  int pad;      // padded positions (powers of two)
  int nst;      // Stockham stages and their radices (odd ones first)
  int rad[16];
  const double2 *tw;  // device: exp(-2 pi i k / n), k < n
};
struct FftPassX {
  FftAxis ax;
  const double *small;   // spreading grid, copies x [E][re, im][n1z][n1y][n1x]
  long long copy_stride; // doubles between copies
  long long cells1;      // n1x n1y n1z
  int copies;
  const double *dec;     // 1 / phi2hat per spreading-grid index: x, then y, then z
  int n1y, n1z;
  long long lines;       // E n1z n1y
  int per_cta;
  double2 *out;          // [E][n1z][n1y][mx]
};
struct FftPassY {
  FftAxis ax;
  const double2 *in;     // [E][n1z][n1y][mx]
  double2 *out;          // [E][n1z][my][mx]
  int mx, per_cta;
};
struct FftPassZ {
  FftAxis ax;
  const double2 *in;     // [E][n1z][my][mx]
  float2 *packed;        // [groups][mz][my][mx][slots]
  int mx, my, n_elem, slots, n_groups;
  int per_cta, per_elem;
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
  const float4 *packed;  // [n_groups][m_z][m_y][m_x][halves] (the z pass of nufft_fft3)
  long long cell2;       // box cells m_x m_y m_z
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
// grid (zeroed, FP64): `copies` x [n_elem][re, im][n1z][n1y][n1x], atom j
// adding into copy j mod copies (several copies spread the updates of one cell
// when the grid is small next to the atom count).  An atom whose stencil
// leaves the grid is skipped and sets err[0].
cudaError_t nufft_spread(const AtomD *atoms, const int *seg, int n_elem, int n_atoms, const NufftGeom &g,
                         double *grid, int copies, int *err, cudaStream_t st);
// Step 2: zero `fine` and scatter the deconvolved spreading grid (the sum of
// its copies) into it.  dec: 1 / phi2hat per spreading-grid index, x then y
// then z.
cudaError_t nufft_pad(const double2 *small, double2 *fine, const NufftGeom &g, int n_elem, int copies,
                      const double *dec, cudaStream_t st);
// Steps 2-3 by the hand-written passes: x (with the sum of the spreading-grid
// copies and the deconvolution), y, z (with the FP32 element-interleaved
// output of nufft_pack_groups(n_elem) x box cells x nufft_pack_halves(n_elem)
// float4).  fa: E n1z n1y m_x, fb: E n1z m_y m_x double2.
int nufft_pack_halves(int n_elem);
int nufft_pack_groups(int n_elem);
int nufft_fft_axis(int n, int nin, int pmin, int nout, const double2 *tw, FftAxis *ax);  // 0, or -1: n unsupported
void nufft_fft_twiddles(int n, double2 *tw);  // host table exp(-2 pi i k / n)
cudaError_t nufft_fft3(const double *small, int copies, const double *dec, const NufftGeom &g, int n_elem,
                       const FftAxis ax[3], double2 *fa, double2 *fb, float4 *packed, cudaStream_t st);
// Step 4.  Detector q sets (tile_nx > 0) take the tile path unless the mode is
// 1 (the per-pixel path everywhere; both give the same bits).
cudaError_t nufft_interp(const NufftInterp &a, cudaStream_t st);
void nufft_set_interp_mode(int mode);
int nufft_interp_mode();

}  // namespace spsim
