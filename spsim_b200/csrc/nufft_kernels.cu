// Non-uniform FFT structure factor kernels for sm_100a: q-box bounds, atom
// spreading, deconvolution/zero-padding and interpolation at the pixels' q.
// The FFT between the last two steps is cuFFT's.  The transform replaces the
// reference's per-element NNFFT (src/diffraction.c:528-675, dispatched from
// src/spsim.c:120-126): atoms -> q list, unit atom weights, then the
// form factor of |q| with the B factor (src/diffraction.c:390-400).
#include "nufft_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace spsim {

// ---------------------------------------------------------------------------
// exponential-of-semicircle kernel of width w (grid points), at offset u

__device__ __forceinline__ double es_kernel(double u, double inv_half_w, double beta) {
  const double t = u * inv_half_w;
  const double a = 1.0 - t * t;
  return a >= 0.0 ? exp(beta * (sqrt(a) - 1.0)) : 0.0;
}

// ---------------------------------------------------------------------------
// q box

__host__ __device__ inline unsigned long long nufft_key(double d) {
#ifdef __CUDA_ARCH__
  const unsigned long long u = (unsigned long long)__double_as_longlong(d);
#else
  unsigned long long u;
  std::memcpy(&u, &d, sizeof(u));
#endif
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

unsigned long long nufft_double_to_key(double d) { return nufft_key(d); }

double nufft_key_to_double(unsigned long long k) {
  const unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double d;
  std::memcpy(&d, &u, sizeof(d));
  return d;
}

struct RotArg {
  double r[9];
  int on;
};

__global__ void nufft_bounds_kernel(const float *__restrict__ hkl, const double *__restrict__ q64, long long npix,
                                    RotArg rot, unsigned long long *__restrict__ keys) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npix;
       p += (long long)gridDim.x * blockDim.x) {
    double a, b, c;
    if (hkl) {
      a = hkl[3 * p];
      b = hkl[3 * p + 1];
      c = hkl[3 * p + 2];
    } else {
      a = q64[3 * p];
      b = q64[3 * p + 1];
      c = q64[3 * p + 2];
    }
    double q[3] = {a, b, c};
    if (rot.on) {
      q[0] = rot.r[0] * a + rot.r[1] * b + rot.r[2] * c;
      q[1] = rot.r[3] * a + rot.r[4] * b + rot.r[5] * c;
      q[2] = rot.r[6] * a + rot.r[7] * b + rot.r[8] * c;
    }
    for (int d = 0; d < 3; ++d) {
      lo[d] = fmin(lo[d], q[d]);
      hi[d] = fmax(hi[d], q[d]);
    }
  }
  for (int d = 0; d < 3; ++d)
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
  if ((threadIdx.x & 31) == 0 && lo[0] <= hi[0]) {
    for (int d = 0; d < 3; ++d) {
      atomicMin(keys + d, nufft_key(lo[d]));
      atomicMax(keys + 3 + d, nufft_key(hi[d]));
    }
  }
}

cudaError_t nufft_bounds(const float *hkl, const double *q64, long long npix, const double *rot,
                         unsigned long long *keys, cudaStream_t st) {
  unsigned long long init[6];
  for (int d = 0; d < 3; ++d) {
    init[d] = ~0ull;
    init[3 + d] = 0ull;
  }
  cudaError_t e = cudaMemcpyAsync(keys, init, sizeof(init), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess || npix <= 0) return e;
  RotArg r;
  r.on = rot != nullptr;
  for (int k = 0; k < 9; ++k) r.r[k] = rot ? rot[k] : (k % 4 == 0 ? 1.0 : 0.0);
  const long long blocks = std::min<long long>((npix + 255) / 256, 148 * 8);
  nufft_bounds_kernel<<<(unsigned)blocks, 256, 0, st>>>(hkl, q64, npix, r, keys);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// step 1: spreading, one warp per atom, FP64 atomics into the (L2-resident)
// spreading grid

constexpr int SPREAD_WARPS = 8;

__global__ void __launch_bounds__(32 * SPREAD_WARPS) nufft_spread_kernel(const AtomD *__restrict__ atoms,
                                                                         const int *__restrict__ seg, int n_elem,
                                                                         int n_atoms, const NufftGeom g,
                                                                         double2 *__restrict__ grid,
                                                                         int *__restrict__ err) {
  __shared__ double kv[SPREAD_WARPS][3][NUFFT_MAX_W];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * SPREAD_WARPS + warp;
  if (j >= n_atoms) return;
  const AtomD a = atoms[j];
  if (a.w == 0.0f) return;  // segment padding (and atoms of zero weight)
  int e = 0;
  while (e + 1 < n_elem && j >= seg[e + 1]) ++e;
  const double xs[3] = {a.x, a.y, a.z};
  const int w = g.w1;
  double s[3];
  int l0[3];
  for (int d = 0; d < 3; ++d) {
    s[d] = xs[d] * g.inv_h[d] + 0.5 * g.n1[d];
    l0[d] = (int)ceil(s[d] - 0.5 * w);
    if (!(l0[d] >= 0 && l0[d] + w <= g.n1[d])) {  // also catches NaN positions
      if (lane == 0) atomicOr(err, 1);
      return;
    }
  }
  const double inv_half_w = 2.0 / w;
  for (int i = lane; i < 3 * w; i += 32) {
    const int d = i / w, k = i - d * w;
    kv[warp][d][k] = es_kernel(s[d] - (double)(l0[d] + k), inv_half_w, g.beta1);
  }
  __syncwarp();
  // w_j e^{-2 pi i C.x_j}
  double t = g.cq[0] * a.x + g.cq[1] * a.y + g.cq[2] * a.z;
  t -= rint(t);
  double sn, cs;
  sincospi(2.0 * t, &sn, &cs);
  const double cr = (double)a.w * cs, ci = -(double)a.w * sn;
  const long long n1x = g.n1[0], n1y = g.n1[1];
  double2 *base = grid + (long long)e * n1x * n1y * g.n1[2] + ((long long)l0[2] * n1y + l0[1]) * n1x + l0[0];
  const int ww = w * w;
  for (int c = lane; c < ww * w; c += 32) {
    const int iz = c / ww, r = c - iz * ww, iy = r / w, ix = r - iy * w;
    const double v = kv[warp][2][iz] * kv[warp][1][iy] * kv[warp][0][ix];
    double2 *p = base + ((long long)iz * n1y + iy) * n1x + ix;
    atomicAdd(&p->x, v * cr);
    atomicAdd(&p->y, v * ci);
  }
}

cudaError_t nufft_spread(const AtomD *atoms, const int *seg, int n_elem, int n_atoms, const NufftGeom &g,
                         double2 *grid, int *err, cudaStream_t st) {
  if (n_atoms <= 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((n_atoms + SPREAD_WARPS - 1) / SPREAD_WARPS);
  nufft_spread_kernel<<<blocks, 32 * SPREAD_WARPS, 0, st>>>(atoms, seg, n_elem, n_atoms, g, grid, err);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// step 2: deconvolution by phi2hat and zero-padding into the FFT grid.
// Spreading-grid index l holds mode m = l - n1/2, stored at FFT index m mod n2.

__global__ void nufft_pad_kernel(const double2 *__restrict__ small, double2 *__restrict__ fine, const NufftGeom g,
                                 int n_elem, const double *__restrict__ dec) {
  const int n2x = g.n2[0], n2y = g.n2[1], n2z = g.n2[2];
  const int n1x = g.n1[0], n1y = g.n1[1], n1z = g.n1[2];
  const double *decx = dec, *decy = dec + n1x, *decz = dec + n1x + n1y;
  const int py = blockIdx.y;
  const int my = (py < n2y / 2 ? py : py - n2y) + n1y / 2;
  const bool iny = my >= 0 && my < n1y;
  for (int ez = blockIdx.z; ez < n_elem * n2z; ez += gridDim.z) {
    const int e = ez / n2z, pz = ez - e * n2z;
    const int mz = (pz < n2z / 2 ? pz : pz - n2z) + n1z / 2;
    const bool inyz = iny && mz >= 0 && mz < n1z;
    double2 *out = fine + (((long long)e * n2z + pz) * n2y + py) * n2x;
    const double2 *in = inyz ? small + (((long long)e * n1z + mz) * n1y + my) * n1x : small;
    const double dyz = inyz ? decy[my] * decz[mz] : 0.0;
    for (int px = blockIdx.x * blockDim.x + threadIdx.x; px < n2x; px += gridDim.x * blockDim.x) {
      const int mx = (px < n2x / 2 ? px : px - n2x) + n1x / 2;
      double2 v = make_double2(0.0, 0.0);
      if (inyz && mx >= 0 && mx < n1x) {
        const double2 b = in[mx];
        const double d = dyz * decx[mx];
        v = make_double2(b.x * d, b.y * d);
      }
      out[px] = v;
    }
  }
}

cudaError_t nufft_pad(const double2 *small, double2 *fine, const NufftGeom &g, int n_elem, const double *dec,
                      cudaStream_t st) {
  const int threads = 128;
  dim3 grid((unsigned)std::min((g.n2[0] + threads - 1) / threads, 8), (unsigned)g.n2[1],
            (unsigned)std::min(n_elem * g.n2[2], 65535));
  nufft_pad_kernel<<<grid, threads, 0, st>>>(small, fine, g, n_elem, dec);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// step 4: interpolation at each pixel's q, form factors, deconvolution by
// psi1hat, centre phase.  One thread per pixel; the stencil is W^3 FFT-grid
// points, each element's grid read at the same offsets.

__device__ __forceinline__ double psi1_hat(double xi, const double *__restrict__ a, int n) {
  // sum_k a_k cos(2 pi xi k / 4) by Clenshaw's recurrence in T_k(cos(pi xi / 2))
  const double x = cospi(0.5 * xi);
  double b1 = 0.0, b2 = 0.0;
  for (int k = n - 1; k >= 1; --k) {
    const double b0 = fma(2.0 * x, b1, a[k] - b2);
    b2 = b1;
    b1 = b0;
  }
  return fma(x, b1, a[0] - b2);
}

template <int W>
__global__ void __launch_bounds__(128) nufft_interp_kernel(const __grid_constant__ NufftInterp a) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.npix) return;
  const NufftGeom &g = a.g;
  double h0, h1, h2;
  if (a.hkl) {
    h0 = a.hkl[3 * p];
    h1 = a.hkl[3 * p + 1];
    h2 = a.hkl[3 * p + 2];
  } else {
    h0 = a.q64[3 * p];
    h1 = a.q64[3 * p + 1];
    h2 = a.q64[3 * p + 2];
  }
  double q[3] = {h0, h1, h2};
  if (a.has_rot) {
    q[0] = a.rot[0] * h0 + a.rot[1] * h1 + a.rot[2] * h2;
    q[1] = a.rot[3] * h0 + a.rot[4] * h1 + a.rot[5] * h2;
    q[2] = a.rot[6] * h0 + a.rot[7] * h1 + a.rot[8] * h2;
  }
  const int n2x = g.n2[0], n2y = g.n2[1], n2z = g.n2[2];
  double t[3];
  int b[3];
  double D = 1.0;
  for (int d = 0; d < 3; ++d) {
    const double qp = q[d] - g.cq[d];
    t[d] = qp * g.L[d];
    const double p0 = ceil(t[d] - 0.5 * W);
    t[d] -= p0;  // stencil offsets: t - i, i = 0 .. W-1
    int s = (int)p0 % g.n2[d];
    b[d] = s < 0 ? s + g.n2[d] : s;
    D *= psi1_hat(g.h[d] * qp, a.psi_a, a.n_coef);
  }
  const double ihw = 2.0 / W;
  double kx[W], ky[W];
  int ix[W], iy[W];
#pragma unroll
  for (int i = 0; i < W; ++i) {
    kx[i] = es_kernel(t[0] - i, ihw, g.beta2);
    ky[i] = es_kernel(t[1] - i, ihw, g.beta2);
    ix[i] = b[0] + i >= n2x ? b[0] + i - n2x : b[0] + i;
    iy[i] = b[1] + i >= n2y ? b[1] + i - n2y : b[1] + i;
  }
  // |q| of the unrotated list for the form factors, as the direct path
  const double s2 = [&] {
    const double d = sqrt(h0 * h0 + h1 * h1 + h2 * h2) * 1e-10;
    return d * d * 0.25;
  }();
  double fr = 0.0, fi = 0.0;
  for (int e0 = 0; e0 < a.n_elem; e0 += 4) {
    const int ne = min(4, a.n_elem - e0);
    const double2 *gr = a.grid + (long long)e0 * a.cell2;
    double ar[4] = {0.0, 0.0, 0.0, 0.0}, ai[4] = {0.0, 0.0, 0.0, 0.0};
    for (int iz = 0; iz < W; ++iz) {
      const double kz = es_kernel(t[2] - iz, ihw, g.beta2);
      const int zz = b[2] + iz >= n2z ? b[2] + iz - n2z : b[2] + iz;
      const double2 *plane = gr + (long long)zz * n2y * n2x;
#pragma unroll
      for (int jy = 0; jy < W; ++jy) {
        const double2 *row = plane + (long long)iy[jy] * n2x;
        double sr[4] = {0.0, 0.0, 0.0, 0.0}, si[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int jx = 0; jx < W; ++jx) {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            if (e < ne) {
              const double2 v = __ldg(row + (long long)e * a.cell2 + ix[jx]);
              sr[e] = fma(kx[jx], v.x, sr[e]);
              si[e] = fma(kx[jx], v.y, si[e]);
            }
          }
        }
        const double kzy = kz * ky[jy];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          ar[e] = fma(kzy, sr[e], ar[e]);
          ai[e] = fma(kzy, si[e], ai[e]);
        }
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (e >= ne) break;
      double f = 1.0;
      if (!a.delta_atoms) {
        // src/diffraction.c:183-193, as ff_table_kernel
        const float *c = a.coeffs + 9 * (e0 + e);
        f = 0.0;
        for (int i = 0; i < 4; ++i) f += (double)c[i] * exp(-((double)c[i + 4] + a.B) * s2);
        f += (double)c[8] * exp(-a.B * s2);
      }
      fr = fma(f, ar[e], fr);
      fi = fma(f, ai[e], fi);
    }
  }
  const double inv = 1.0 / D;
  fr *= inv;
  fi *= inv;
  if (a.I) a.I[p] = (float)(fr * fr + fi * fi);
  if (a.F) {
    double tc = q[0] * g.center[0] + q[1] * g.center[1] + q[2] * g.center[2];
    tc -= rint(tc);
    double sn, cs;
    sincospi(2.0 * tc, &sn, &cs);
    a.F[p] = make_float2((float)(fr * cs + fi * sn), (float)(fi * cs - fr * sn));
  }
}

template <int W>
static cudaError_t interp_t(const NufftInterp &a, cudaStream_t st) {
  const unsigned blocks = (unsigned)((a.npix + 127) / 128);
  nufft_interp_kernel<W><<<blocks, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t nufft_interp(const NufftInterp &a, cudaStream_t st) {
  if (a.npix <= 0) return cudaSuccess;
  switch (a.g.w2) {
    case 4: return interp_t<4>(a, st);
    case 5: return interp_t<5>(a, st);
    case 6: return interp_t<6>(a, st);
    case 7: return interp_t<7>(a, st);
    case 8: return interp_t<8>(a, st);
    case 9: return interp_t<9>(a, st);
    case 10: return interp_t<10>(a, st);
    case 11: return interp_t<11>(a, st);
    case 12: return interp_t<12>(a, st);
    case 13: return interp_t<13>(a, st);
    case 14: return interp_t<14>(a, st);
    case 15: return interp_t<15>(a, st);
    case 16: return interp_t<16>(a, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace spsim
