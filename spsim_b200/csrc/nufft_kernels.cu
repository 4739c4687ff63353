// Non-uniform FFT structure factor kernels for sm_100a: q-box bounds, atom
// spreading and interpolation at the pixels' q.  The deconvolution, padding
// and FFT between the two are the passes of nufft_fft.cu.  The transform replaces the
// reference's per-element NNFFT (src/diffraction.c:528-675, dispatched from
// src/spsim.c:119-123): atoms -> q list, unit atom weights, then the
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
                                                                         double *__restrict__ grid, int copies,
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
  // warps take the grid copies in turn: fewer updates of one cell in flight;
  // real and imaginary parts in separate planes, so that a half-warp's
  // atomics on one stencil row cover 96 contiguous bytes, not 192
  const long long cells1 = n1x * n1y * g.n1[2];
  double *base = grid + 2 * ((long long)(j % copies) * n_elem + e) * cells1 + ((long long)l0[2] * n1y + l0[1]) * n1x +
                 l0[0];
  // lane = (y parity, x offset): half-warps cover two stencil rows per step
  static_assert(NUFFT_MAX_W <= 16, "one stencil row per half-warp");
  const int ix = lane & 15, iy0 = lane >> 4;
  if (ix < w) {
    const double kxr = kv[warp][0][ix] * cr, kxi = kv[warp][0][ix] * ci;
    for (int iz = 0; iz < w; ++iz) {
      const double kz = kv[warp][2][iz];
      double *plane = base + (long long)iz * n1y * n1x + ix;
      for (int iy = iy0; iy < w; iy += 2) {
        const double v = kz * kv[warp][1][iy];
        double *p = plane + (long long)iy * n1x;
        atomicAdd(p, v * kxr);
        atomicAdd(p + cells1, v * kxi);
      }
    }
  }
}

cudaError_t nufft_spread(const AtomD *atoms, const int *seg, int n_elem, int n_atoms, const NufftGeom &g,
                         double *grid, int copies, int *err, cudaStream_t st) {
  if (n_atoms <= 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((n_atoms + SPREAD_WARPS - 1) / SPREAD_WARPS);
  nufft_spread_kernel<<<blocks, 32 * SPREAD_WARPS, 0, st>>>(atoms, seg, n_elem, n_atoms, g, grid, std::max(copies, 1),
                                                            err);
  return cudaGetLastError();
}

// the interpolation's FP32 grid holds elements in groups of 2 x halves,
// halves float4 (two elements each) per cell and group
int nufft_pack_halves(int n_elem) { return n_elem <= 2 ? 1 : 2; }
int nufft_pack_groups(int n_elem) { return (n_elem + 2 * nufft_pack_halves(n_elem) - 1) / (2 * nufft_pack_halves(n_elem)); }

// ---------------------------------------------------------------------------
// step 4: interpolation at each pixel's q, form factors, deconvolution by
// psi1hat, centre phase.  One thread per pixel; the stencil is W^3 grid points,
// all elements of a group read together.  Each x row of the stencil is
// contracted in FP32 (W terms), the rows summed in FP64.

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

// 32 bytes (four elements, FP32 complex) in one 256-bit load; p 32-byte aligned
__device__ __forceinline__ void ld_cell32(const float4 *p, float4 &a, float4 &b) {
  asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
               : "l"(p));
}

// Pixel tiles of a detector q list: a block takes 16 x 8 neighbouring pixels.
constexpr int INTERP_TX = 16, INTERP_TY = 8, INTERP_THREADS = INTERP_TX * INTERP_TY;
// The tile path stages the tile's grid region in shared memory when it spans
// at most REGION_MAX_X points along x and REGION_MAX_CELLS points in all
// (four elements: 32 bytes a point, 55 KB); other tiles read per pixel.
constexpr int REGION_MAX_X = 16;
constexpr int REGION_MAX_CELLS = 1728;

static int g_interp_mode = 0;  // 0: tile path for detector q sets, 1: per-pixel path everywhere

// A pixel's interpolation stencil: the first grid point b of its W^3 stencil
// in the output box along each axis, the offsets t (stencil point i has weight
// phi2(t - i)), the deconvolution D = prod_d psi1hat(h_d q'_d), s^2 = (|q|/2)^2
// in 1/A^2 for the form factors, and q = R q_list for the centre phase.
struct Stencil {
  double q[3];
  double t[3];
  int b[3];
  double D;
  double s2;
};

template <int W>
__device__ __forceinline__ void stencil_of(const NufftInterp &a, long long p, int pattern, Stencil &s) {
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
  s.q[0] = h0;
  s.q[1] = h1;
  s.q[2] = h2;
  const double *R = a.rots ? a.rots + 9 * pattern : (a.has_rot ? a.rot : nullptr);
  if (R) {
    s.q[0] = R[0] * h0 + R[1] * h1 + R[2] * h2;
    s.q[1] = R[3] * h0 + R[4] * h1 + R[5] * h2;
    s.q[2] = R[6] * h0 + R[7] * h1 + R[8] * h2;
  }
  s.D = 1.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double qp = s.q[d] - g.cq[d];
    s.t[d] = qp * g.L[d];
    const double p0 = ceil(s.t[d] - 0.5 * W);
    s.t[d] -= p0;  // stencil offsets: t - i, i = 0 .. W-1
    // stencil start in the output box; the box holds every q of the list
    // with a margin, the clamp only keeps the reads inside it
    s.b[d] = min(max((int)p0 - g.pmin[d], 0), g.m[d] - W);
    s.D *= psi1_hat(g.h[d] * qp, a.psi_a, a.n_coef);
  }
  // |q| of the unrotated list for the form factors, as the direct path
  const double d = sqrt(h0 * h0 + h1 * h1 + h2 * h2) * 1e-10;
  s.s2 = d * d * 0.25;
}

// The element sums of group grp (acc: re, im of its 2H elements) into F, with
// the form factors (src/diffraction.c:183-193, as ff_table_kernel).
template <int H>
__device__ __forceinline__ void add_group(const NufftInterp &a, int grp, const double (&acc)[4 * H], double s2,
                                          double &fr, double &fi) {
#pragma unroll
  for (int k = 0; k < 2 * H; ++k) {
    const int e = grp * 2 * H + k;
    if (e >= a.n_elem) break;
    double f = 1.0;
    if (!a.delta_atoms) {
      const float *c = a.coeffs + 9 * e;
      f = 0.0;
      for (int i = 0; i < 4; ++i) f += (double)c[i] * exp(-((double)c[i + 4] + a.B) * s2);
      f += (double)c[8] * exp(-a.B * s2);
    }
    fr = fma(f, acc[2 * k], fr);
    fi = fma(f, acc[2 * k + 1], fi);
  }
}

__device__ __forceinline__ void write_pixel(const NufftInterp &a, long long out, const Stencil &s, double fr,
                                            double fi) {
  const double inv = 1.0 / s.D;
  fr *= inv;
  fi *= inv;
  if (a.I) a.I[out] = (float)(fr * fr + fi * fi);
  if (a.F) {
    double tc = s.q[0] * a.g.center[0] + s.q[1] * a.g.center[1] + s.q[2] * a.g.center[2];
    tc -= rint(tc);
    double sn, cs;
    sincospi(2.0 * tc, &sn, &cs);
    a.F[out] = make_float2((float)(fr * cs + fi * sn), (float)(fi * cs - fr * sn));
  }
}

// A pixel's stencil weights and grid offsets along x and y (z: per plane).
template <int W, int H>
struct StencilXY {
  float kx[W];
  double ky[W];
  int ix[W], iy[W];
};

template <int W, int H>
__device__ __forceinline__ void stencil_xy(const NufftGeom &g, const Stencil &s, StencilXY<W, H> &w) {
  const double ihw = 2.0 / W;
#pragma unroll
  for (int i = 0; i < W; ++i) {
    w.kx[i] = (float)es_kernel(s.t[0] - i, ihw, g.beta2);
    w.ky[i] = es_kernel(s.t[1] - i, ihw, g.beta2);
    w.ix[i] = (s.b[0] + i) * H;
    w.iy[i] = s.b[1] + i;
  }
}

// One group's W^3 stencil read per pixel from the grid (L1-cached 256-bit
// loads): x rows contracted in FP32, rows summed in FP64.
template <int W, int H>
__device__ __forceinline__ void direct_group(const NufftInterp &a, int grp, const Stencil &s,
                                             const StencilXY<W, H> &w, double (&acc)[4 * H]) {
  const NufftGeom &g = a.g;
  const double ihw = 2.0 / W;
  const long long row_stride = (long long)g.m[0] * H, plane_stride = row_stride * g.m[1];
  const float4 *gr = a.packed + (long long)grp * a.cell2 * H;
#pragma unroll
  for (int k = 0; k < 4 * H; ++k) acc[k] = 0.0;
  for (int iz = 0; iz < W; ++iz) {
    const double kz = es_kernel(s.t[2] - iz, ihw, g.beta2);
    const float4 *plane = gr + (long long)(s.b[2] + iz) * plane_stride;
#pragma unroll
    for (int jy = 0; jy < W; ++jy) {
      const float4 *row = plane + (long long)w.iy[jy] * row_stride;
      float v4[4 * H];
#pragma unroll
      for (int k = 0; k < 4 * H; ++k) v4[k] = 0.0f;
#pragma unroll
      for (int jx = 0; jx < W; ++jx) {
        float4 v[H];
        if constexpr (H == 2)
          ld_cell32(row + w.ix[jx], v[0], v[1]);
        else
          v[0] = __ldg(row + w.ix[jx]);
#pragma unroll
        for (int h = 0; h < H; ++h) {
          v4[4 * h + 0] = fmaf(w.kx[jx], v[h].x, v4[4 * h + 0]);
          v4[4 * h + 1] = fmaf(w.kx[jx], v[h].y, v4[4 * h + 1]);
          v4[4 * h + 2] = fmaf(w.kx[jx], v[h].z, v4[4 * h + 2]);
          v4[4 * h + 3] = fmaf(w.kx[jx], v[h].w, v4[4 * h + 3]);
        }
      }
      const double kzy = kz * w.ky[jy];
#pragma unroll
      for (int k = 0; k < 4 * H; ++k) acc[k] = fma(kzy, (double)v4[k], acc[k]);
    }
  }
}

// Per-pixel path: one thread per pixel of any q list (16 x 8 tiles of a
// detector's pixels, so that neighbouring stencils share L1 lines).
template <int W, int H>
__global__ void __launch_bounds__(INTERP_THREADS, W <= 11 ? 3 : 1)
    nufft_interp_kernel(const __grid_constant__ NufftInterp a) {
  long long p;
  if (a.tile_nx > 0) {
    const int tiles_x = (a.tile_nx + INTERP_TX - 1) / INTERP_TX;
    const long long x = (long long)(blockIdx.x % tiles_x) * INTERP_TX + threadIdx.x % INTERP_TX;
    const long long y = (long long)(blockIdx.x / tiles_x) * INTERP_TY + threadIdx.x / INTERP_TX;
    if (x >= a.tile_nx) return;
    p = y * a.tile_nx + x;
  } else {
    p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  }
  if (p >= a.npix) return;
  Stencil s;
  stencil_of<W>(a, p, blockIdx.y, s);
  StencilXY<W, H> w;
  stencil_xy<W, H>(a.g, s, w);
  double fr = 0.0, fi = 0.0;
  for (int grp = 0; grp < a.n_groups; ++grp) {
    double acc[4 * H];
    direct_group<W, H>(a, grp, s, w, acc);
    add_group<H>(a, grp, acc, s.s2, fr, fi);
  }
  write_pixel(a, (long long)blockIdx.y * a.npix + p, s, fr, fi);
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}

// Tile path (detector q sets): the block's 128 pixels walk their tile's grid
// region together.  The region (the union of the W^3 stencils, E_x x E_y x
// E_z points) is staged in shared memory by 16-byte asynchronous copies; for
// every (z, y) row of it every thread reads the same points (shared-memory
// broadcasts, one wavefront a 16-byte load for the whole warp, where each
// pixel's own 256-bit loads cost eight) and contracts them with its own x
// weights, zero outside its stencil, on packed f32x2 FMAs.  Zero weights add
// exact zeros, in the per-pixel path's order, so that both paths give the same
// bits.  Rows outside every stencil of a warp are skipped.
template <int W, int H>
__global__ void __launch_bounds__(INTERP_THREADS, 3) nufft_interp_tile_kernel(const __grid_constant__ NufftInterp a) {
  extern __shared__ float4 region[];  // [E_z][E_y][E_x][H]
  __shared__ double wgt[2][W][INTERP_THREADS];  // y and z stencil weights per thread
  __shared__ int box[6];                        // smallest and largest stencil start per axis
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tiles_x = (a.tile_nx + INTERP_TX - 1) / INTERP_TX;
  const long long px = (long long)(blockIdx.x % tiles_x) * INTERP_TX + tid % INTERP_TX;
  const long long py = (long long)(blockIdx.x / tiles_x) * INTERP_TY + tid / INTERP_TX;
  const long long p = py * a.tile_nx + px;
  const bool active = px < a.tile_nx && p < a.npix;
  const NufftGeom &g = a.g;
  const double ihw = 2.0 / W;
  Stencil s;
  if (active) stencil_of<W>(a, p, blockIdx.y, s);
  if (tid < 3) {
    box[tid] = 0x7fffffff;
    box[3 + tid] = -0x7fffffff;
  }
#pragma unroll
  for (int i = 0; i < W; ++i) {
    wgt[0][i][tid] = active ? es_kernel(s.t[1] - i, ihw, g.beta2) : 0.0;
    wgt[1][i][tid] = active ? es_kernel(s.t[2] - i, ihw, g.beta2) : 0.0;
  }
  __syncthreads();
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int lo = __reduce_min_sync(0xffffffffu, active ? s.b[d] : 0x7fffffff);
    const int hi = __reduce_max_sync(0xffffffffu, active ? s.b[d] : -0x7fffffff);
    if (lane == 0) {
      atomicMin(&box[d], lo);
      atomicMax(&box[3 + d], hi);
    }
  }
  __syncthreads();
  const int r0x = box[0], r0y = box[1], r0z = box[2];
  const int ex = box[3] - r0x + W, ey = box[4] - r0y + W, ez = box[5] - r0z + W;
  double fr = 0.0, fi = 0.0;
  if (ex <= REGION_MAX_X && ex * ey * ez <= REGION_MAX_CELLS) {
    // this pixel's x weights over the region's columns (zero outside its stencil)
    float kxr[REGION_MAX_X];
    const int ox = active ? s.b[0] - r0x : 0, oy = active ? s.b[1] - r0y : 0, oz = active ? s.b[2] - r0z : 0;
#pragma unroll
    for (int x = 0; x < REGION_MAX_X; ++x) {
      const int i = x - ox;
      kxr[x] = active && i >= 0 && i < W ? (float)es_kernel(s.t[0] - i, ihw, g.beta2) : 0.0f;
    }
    const int rowlen = ex * H, nrow = ey * ez;  // float4 per region row (<= 32), rows
    for (int grp = 0; grp < a.n_groups; ++grp) {
      if (grp > 0) __syncthreads();  // the previous group's region is read
      const float4 *src = a.packed + (long long)grp * a.cell2 * H;
      for (int r = warp; r < nrow; r += INTERP_THREADS / 32) {
        const int z = r / ey, y = r - z * ey;
        if (lane < rowlen)
          cp_async16(region + r * rowlen + lane,
                     src + (((long long)(r0z + z) * g.m[1] + r0y + y) * g.m[0] + r0x) * H + lane);
      }
      asm volatile("cp.async.wait_all;" ::: "memory");
      __syncthreads();
      double acc[4 * H];
#pragma unroll
      for (int k = 0; k < 4 * H; ++k) acc[k] = 0.0;
      for (int z = 0; z < ez; ++z) {
        const int jz = z - oz;
        const double kz = jz >= 0 && jz < W ? wgt[1][jz][tid] : 0.0;
        if (!__any_sync(0xffffffffu, kz != 0.0)) continue;
        for (int y = 0; y < ey; ++y) {
          const int jy = y - oy;
          const double kzy = kz * (jy >= 0 && jy < W ? wgt[0][jy][tid] : 0.0);
          if (!__any_sync(0xffffffffu, kzy != 0.0)) continue;
          const float4 *row = region + (z * ey + y) * rowlen;
          float2 v2[2 * H];
#pragma unroll
          for (int k = 0; k < 2 * H; ++k) v2[k] = make_float2(0.0f, 0.0f);
#pragma unroll
          for (int x = 0; x < REGION_MAX_X; ++x) {
            if (x < ex) {
              const float2 w = make_float2(kxr[x], kxr[x]);
#pragma unroll
              for (int h = 0; h < H; ++h) {
                const float4 c = row[x * H + h];
                v2[2 * h] = __ffma2_rn(w, make_float2(c.x, c.y), v2[2 * h]);
                v2[2 * h + 1] = __ffma2_rn(w, make_float2(c.z, c.w), v2[2 * h + 1]);
              }
            }
          }
#pragma unroll
          for (int k = 0; k < 2 * H; ++k) {
            acc[2 * k] = fma(kzy, (double)v2[k].x, acc[2 * k]);
            acc[2 * k + 1] = fma(kzy, (double)v2[k].y, acc[2 * k + 1]);
          }
        }
      }
      if (active) add_group<H>(a, grp, acc, s.s2, fr, fi);
    }
  } else if (active) {
    StencilXY<W, H> w;
    stencil_xy<W, H>(g, s, w);
    for (int grp = 0; grp < a.n_groups; ++grp) {
      double acc[4 * H];
      direct_group<W, H>(a, grp, s, w, acc);
      add_group<H>(a, grp, acc, s.s2, fr, fi);
    }
  }
  if (active) write_pixel(a, (long long)blockIdx.y * a.npix + p, s, fr, fi);
}

template <int W>
static cudaError_t interp_t(const NufftInterp &a, cudaStream_t st) {
  long long blocks = (a.npix + INTERP_THREADS - 1) / INTERP_THREADS;
  if (a.tile_nx > 0) {
    const long long rows = (a.npix + a.tile_nx - 1) / a.tile_nx;
    blocks = ((a.tile_nx + INTERP_TX - 1) / INTERP_TX) * ((rows + INTERP_TY - 1) / INTERP_TY);
  }
  const dim3 grid((unsigned)blocks, (unsigned)std::max(a.npat, 1));
  // a stencil wider than 11 points leaves no region of 1,728 points room to
  // hold a tile's spread: such widths read per pixel
  if constexpr (W <= 11) if (a.tile_nx > 0 && g_interp_mode == 0) {
    const size_t smem = (size_t)REGION_MAX_CELLS * a.halves * sizeof(float4);
    cudaError_t e;
    if (a.halves == 1) {
      e = cudaFuncSetAttribute(nufft_interp_tile_kernel<W, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem);
      if (e == cudaSuccess) nufft_interp_tile_kernel<W, 1><<<grid, INTERP_THREADS, smem, st>>>(a);
    } else {
      e = cudaFuncSetAttribute(nufft_interp_tile_kernel<W, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem);
      if (e == cudaSuccess) nufft_interp_tile_kernel<W, 2><<<grid, INTERP_THREADS, smem, st>>>(a);
    }
    return e != cudaSuccess ? e : cudaGetLastError();
  }
  if (a.halves == 1)
    nufft_interp_kernel<W, 1><<<grid, INTERP_THREADS, 0, st>>>(a);
  else
    nufft_interp_kernel<W, 2><<<grid, INTERP_THREADS, 0, st>>>(a);
  return cudaGetLastError();
}

void nufft_set_interp_mode(int mode) { g_interp_mode = mode; }
int nufft_interp_mode() { return g_interp_mode; }

cudaError_t nufft_interp(const NufftInterp &a, cudaStream_t st) {
  if (a.npix <= 0) return cudaSuccess;
  if (a.halves != 1 && a.halves != 2) return cudaErrorInvalidValue;
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
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace spsim
