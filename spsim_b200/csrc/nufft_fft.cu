// FFT passes of the NUFFT structure factor for sm_100a: the deconvolved
// spreading grid of every element, zero-padded to the FFT grid, transformed
// along x, then y, then z, each pass a batch of 1-D FP64 transforms in shared
// memory.  The passes are pruned at both ends: a pass reads only the n1
// spreading-grid points of its lines (the padding is never stored) and writes
// only the box of output frequencies that the interpolation reads, so the
// FFT grid never exists in full.  The z pass writes its box straight into the
// FP32 element-interleaved layout of the interpolation.
//
// Transform: mixed-radix Stockham autosort (radices 7, 5, 3, 8, 4, 2), one
// stage per shared-memory round trip between two line buffers.  Stage with
// radix R after radices of product Ns: for butterfly j < N/R, k = j mod Ns,
//   v_t = x[j + t N/R] exp(-2 pi i t k / (Ns R)),  v = DFT_R(v),
//   y[(j - k) R + k + t Ns] = v_t.
#include "nufft_kernels.cuh"

#include <algorithm>
#include <cmath>

namespace spsim {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }  // -i a

// DFT_R in place, y_k = sum_n v_n exp(-2 pi i n k / R); w[m] = exp(-2 pi i m / R)
template <int R>
struct Dft;

template <>
struct Dft<2> {
  static __device__ __forceinline__ void run(double2 *v, const double2 *) {
    const double2 a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
  }
};

template <>
struct Dft<4> {
  static __device__ __forceinline__ void run(double2 *v, const double2 *) {
    const double2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    const double2 s13 = cadd(v[1], v[3]), d13 = mul_mi(csub(v[1], v[3]));
    v[0] = cadd(s02, s13);
    v[2] = csub(s02, s13);
    v[1] = cadd(d02, d13);
    v[3] = csub(d02, d13);
  }
};

template <>
struct Dft<8> {
  // even and odd halves as DFT_4, joined by exp(-2 pi i k / 8)
  static __device__ __forceinline__ void run(double2 *v, const double2 *) {
    double2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4>::run(e, nullptr);
    Dft<4>::run(o, nullptr);
    const double r = M_SQRT1_2;
    o[1] = make_double2((o[1].x + o[1].y) * r, (o[1].y - o[1].x) * r);
    o[2] = mul_mi(o[2]);
    o[3] = make_double2((o[3].y - o[3].x) * r, -(o[3].x + o[3].y) * r);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = cadd(e[k], o[k]);
      v[k + 4] = csub(e[k], o[k]);
    }
  }
};

// odd R: pairs n, R - n share cos(2 pi n k / R) and sin(2 pi n k / R)
template <int R>
struct DftOdd {
  static __device__ __forceinline__ void run(double2 *v, const double2 *w) {
    constexpr int h = (R - 1) / 2;
    double2 S[h], D[h];
#pragma unroll
    for (int n = 1; n <= h; ++n) {
      S[n - 1] = cadd(v[n], v[R - n]);
      D[n - 1] = csub(v[n], v[R - n]);
    }
    double2 y[R];
    y[0] = v[0];
#pragma unroll
    for (int n = 0; n < h; ++n) y[0] = cadd(y[0], S[n]);
#pragma unroll
    for (int k = 1; k <= h; ++k) {
      double2 A = v[0], B = make_double2(0.0, 0.0);
#pragma unroll
      for (int n = 1; n <= h; ++n) {
        const double c = w[(n * k) % R].x, s = -w[(n * k) % R].y;
        A.x = fma(S[n - 1].x, c, A.x);
        A.y = fma(S[n - 1].y, c, A.y);
        B.x = fma(D[n - 1].x, s, B.x);
        B.y = fma(D[n - 1].y, s, B.y);
      }
      y[k] = make_double2(A.x + B.y, A.y - B.x);      // A - i B
      y[R - k] = make_double2(A.x - B.y, A.y + B.x);  // A + i B
    }
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = y[k];
  }
};
template <>
struct Dft<3> : DftOdd<3> {};
template <>
struct Dft<5> : DftOdd<5> {};
template <>
struct Dft<7> : DftOdd<7> {};

// Position i of a line in shared memory.  A stage with Ns = 1 has thread j
// write positions j R + t: for an odd first radix (every n with an odd
// factor) that stride already spreads a quarter-warp's 16-byte stores over
// all banks, and positions are plain (PAD false).  A power-of-two n starts
// with R = 8: there one padding slot follows every 8 positions, so that the
// stride becomes 9 slots (PAD true).  Lines are ld >= pos(n - 1) + 1 slots
// apart.
template <bool PAD>
__device__ __forceinline__ int pad(int i) {
  return PAD ? i + (i >> 3) : i;
}

// n / d for 0 <= n, n d < 2^32 by a multiply-high (the block-uniform d's
// magic computed once per loop)
struct FastDiv {
  unsigned m;
  int d;
};
__device__ __forceinline__ FastDiv fdiv_make(int d) {
  FastDiv f;
  f.d = d;
  f.m = d == 1 ? 0u : 0xFFFFFFFFu / (unsigned)d + 1u;
  return f;
}
__device__ __forceinline__ int fdiv(int n, const FastDiv &f) { return f.d == 1 ? n : (int)__umulhi((unsigned)n, f.m); }

constexpr int FFT_THREADS = 256;
constexpr int FFT_MAX_LINES = 64;  // lines of one block (x pass: its per-line scales)

template <int R, bool PAD>
__device__ __forceinline__ void radix_stage(const double2 *__restrict__ src, double2 *__restrict__ dst, int lines,
                                            const FftAxis &ax, int Ns) {
  const int N = ax.n, Nr = N / R, tstep = N / (Ns * R), ld = ax.ld;
  const FastDiv dNr = fdiv_make(Nr), dNs = fdiv_make(Ns);
  double2 w[R];
  if constexpr (R & 1) {
#pragma unroll
    for (int m = 0; m < R; ++m) w[m] = __ldg(ax.tw + m * Nr);
  }
  const int items = lines * Nr;
  for (int it = threadIdx.x; it < items; it += FFT_THREADS) {
    const int c = fdiv(it, dNr), j = it - c * Nr;
    const int q = fdiv(j, dNs), k = j - q * Ns;
    const double2 *s = src + c * ld;
    double2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = s[pad<PAD>(j + t * Nr)];
    if (Ns > 1) {
      // exp(-2 pi i t k / (Ns R)) as powers of the t = 1 twiddle (R - 1 table
      // loads per butterfly measured slower: the L1 path is the busier one)
      const double2 w1 = __ldg(ax.tw + k * tstep);
      double2 wt = w1;
      v[1] = cmul(v[1], w1);
#pragma unroll
      for (int t = 2; t < R; ++t) {
        wt = cmul(wt, w1);
        v[t] = cmul(v[t], wt);
      }
    }
    Dft<R>::run(v, w);
    double2 *d = dst + c * ld;
    const int o = q * Ns * R + k;
#pragma unroll
    for (int t = 0; t < R; ++t) d[pad<PAD>(o + t * Ns)] = v[t];
  }
}

// all stages on `lines` lines of buffer a (b: the other buffer); returns the
// buffer that holds the transforms.  Entered and left with the block in step.
template <bool PAD>
__device__ double2 *stockham(double2 *a, double2 *b, int lines, const FftAxis &ax) {
  int Ns = 1;
  for (int s = 0; s < ax.nst; ++s) {
    const int R = ax.rad[s];
    switch (R) {
      case 8: radix_stage<8, PAD>(a, b, lines, ax, Ns); break;
      case 4: radix_stage<4, PAD>(a, b, lines, ax, Ns); break;
      case 2: radix_stage<2, PAD>(a, b, lines, ax, Ns); break;
      case 3: radix_stage<3, PAD>(a, b, lines, ax, Ns); break;
      case 5: radix_stage<5, PAD>(a, b, lines, ax, Ns); break;
      default: radix_stage<7, PAD>(a, b, lines, ax, Ns); break;
    }
    __syncthreads();
    double2 *t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

// zero the padding of `lines` lines: frequency indices [nin - nin/2, n - nin/2)
template <bool PAD>
__device__ __forceinline__ void zero_padding(double2 *buf, int lines, const FftAxis &ax) {
  const int nz = ax.n - ax.nin, first = ax.nin - ax.nin / 2;
  if (nz <= 0) return;
  const FastDiv dz = fdiv_make(nz);
  for (int i = threadIdx.x; i < lines * nz; i += FFT_THREADS) {
    const int c = fdiv(i, dz), q = i - c * nz;
    buf[c * ax.ld + pad<PAD>(first + q)] = make_double2(0.0, 0.0);
  }
}

template <bool PAD>
__device__ __forceinline__ int in_pos(int l, const FftAxis &ax) {
  const int m = l - ax.nin / 2;
  return pad<PAD>(m < 0 ? m + ax.n : m);
}

template <bool PAD>
__device__ __forceinline__ int out_pos(int o, const FftAxis &ax) {
  int p = ax.p0 + o;
  if (p >= ax.n) p %= ax.n;
  return pad<PAD>(p);
}

// Loads of a pass are issued KL per thread before any is stored to shared
// memory, so that a block has its whole input in flight at once.
constexpr int KL = 8;

// x pass: lines (e, lz, ly) of the spreading grid (the sum of its copies),
// times the separable deconvolution dec (x at the input, y z at the output:
// the transform is linear); out [E n1z n1y][nout]
template <bool PAD>
__global__ void __launch_bounds__(FFT_THREADS, 3) nufft_fft_x_kernel(const __grid_constant__ FftPassX a) {
  extern __shared__ double2 sm[];
  __shared__ double line_scale[FFT_MAX_LINES];
  __shared__ long long line_at[FFT_MAX_LINES];  // offset of the line's real part in the spreading grid
  const FftAxis &ax = a.ax;
  const long long line0 = (long long)blockIdx.x * a.per_cta;
  const int nl = (int)min((long long)a.per_cta, a.lines - line0);
  double2 *b0 = sm, *b1 = sm + (long long)a.per_cta * ax.ld;
  if (threadIdx.x < nl) {
    // line (e, lz, ly): real part at e 2 cells1 + (lz n1y + ly) n1x
    const long long line = line0 + threadIdx.x, per_elem = (long long)a.n1z * a.n1y, e = line / per_elem;
    const int ly = (int)(line % a.n1y), lz = (int)((line / a.n1y) % a.n1z);
    line_scale[threadIdx.x] = a.dec[ax.nin + ly] * a.dec[ax.nin + a.n1y + lz];
    line_at[threadIdx.x] = e * 2 * a.cells1 + (line - e * per_elem) * ax.nin;
  }
  zero_padding<PAD>(b0, nl, ax);
  const int total = nl * ax.nin;
  const FastDiv dnin = fdiv_make(ax.nin);
  __syncthreads();  // line_at
  for (int base = 0; base < total; base += KL * FFT_THREADS) {
    double2 v[KL];
#pragma unroll
    for (int u = 0; u < KL; ++u) {
      const int i = base + u * FFT_THREADS + threadIdx.x;
      if (i < total) {
        const int c = fdiv(i, dnin), lx = i - c * ax.nin;
        const double *re = a.small + line_at[c] + lx;
        v[u] = make_double2(re[0], re[a.cells1]);
        for (int k = 1; k < a.copies; ++k) v[u] = cadd(v[u], make_double2(re[k * a.copy_stride], re[k * a.copy_stride + a.cells1]));
      }
    }
#pragma unroll
    for (int u = 0; u < KL; ++u) {
      const int i = base + u * FFT_THREADS + threadIdx.x;
      if (i < total) {
        const int c = fdiv(i, dnin), lx = i - c * ax.nin;
        const double d = a.dec[lx];
        b0[c * ax.ld + in_pos<PAD>(lx, ax)] = make_double2(v[u].x * d, v[u].y * d);
      }
    }
  }
  __syncthreads();
  const double2 *r = stockham<PAD>(b0, b1, nl, ax);
  double2 *out = a.out + line0 * ax.nout;
  const FastDiv dnout = fdiv_make(ax.nout);
  for (int i = threadIdx.x; i < nl * ax.nout; i += FFT_THREADS) {
    const int c = fdiv(i, dnout), o = i - c * ax.nout;
    const double2 x = r[c * ax.ld + out_pos<PAD>(o, ax)];
    out[i] = make_double2(x.x * line_scale[c], x.y * line_scale[c]);
  }
}

// y pass: columns of [E n1z][n1y][mx], per_cta neighbouring columns of one
// (e, lz) plane; out [E n1z][nout][mx].  Thread t takes column t mod nc and
// rows t / nc + m (256 / nc).
template <bool PAD>
__global__ void __launch_bounds__(FFT_THREADS, 3) nufft_fft_y_kernel(const __grid_constant__ FftPassY a) {
  extern __shared__ double2 sm[];
  const FftAxis &ax = a.ax;
  const int tiles = (a.mx + a.per_cta - 1) / a.per_cta;
  const long long pl = blockIdx.x / tiles;  // (e, lz) plane
  const int x0 = (int)(blockIdx.x - pl * tiles) * a.per_cta, nc = min(a.per_cta, a.mx - x0);
  double2 *b0 = sm, *b1 = sm + a.per_cta * ax.ld;
  zero_padding<PAD>(b0, nc, ax);
  const int c = threadIdx.x % nc, r0 = threadIdx.x / nc, step = FFT_THREADS / nc;
  const bool on = r0 < step;
  const double2 *in = a.in + pl * ax.nin * a.mx + x0 + c;
  for (int base = r0; base < ax.nin; base += KL * step) {
    double2 v[KL];
#pragma unroll
    for (int u = 0; u < KL; ++u) {
      const int ly = base + u * step;
      if (on && ly < ax.nin) v[u] = in[(long long)ly * a.mx];
    }
#pragma unroll
    for (int u = 0; u < KL; ++u) {
      const int ly = base + u * step;
      if (on && ly < ax.nin) b0[c * ax.ld + in_pos<PAD>(ly, ax)] = v[u];
    }
  }
  __syncthreads();
  const double2 *r = stockham<PAD>(b0, b1, nc, ax);
  if (!on) return;
  double2 *out = a.out + pl * ax.nout * a.mx + x0 + c;
  for (int o = r0; o < ax.nout; o += step) out[(long long)o * a.mx] = r[c * ax.ld + out_pos<PAD>(o, ax)];
}

// z pass: columns of [E][n1z][my][mx] for elements [e0, e0 + per_elem) and
// per_cta neighbouring x of one y; out: the interpolation's FP32 grid,
// float2 slots [group][nout][my][mx][slots], element e in group e / slots,
// slot e mod slots; slots past the last element are written as zeros
template <bool PAD>
__global__ void __launch_bounds__(FFT_THREADS, 3) nufft_fft_z_kernel(const __grid_constant__ FftPassZ a) {
  extern __shared__ double2 sm[];
  const FftAxis &ax = a.ax;
  const int x0 = blockIdx.x * a.per_cta, nc = min(a.per_cta, a.mx - x0);
  const int py = blockIdx.y;
  const int e0 = blockIdx.z * a.per_elem, ne = min(a.per_elem, a.n_elem - e0);
  const int lines = ne * nc;  // line l: element e0 + l / nc, column l mod nc
  double2 *b0 = sm, *b1 = sm + a.per_elem * a.per_cta * ax.ld;
  zero_padding<PAD>(b0, lines, ax);
  const long long plane = (long long)a.my * a.mx;
  {
    const int l = threadIdx.x % lines, r0 = threadIdx.x / lines, step = FFT_THREADS / lines;
    const bool on = r0 < step;
    const int el = l / nc, c = l - el * nc;
    const double2 *in = a.in + (long long)(e0 + el) * ax.nin * plane + (long long)py * a.mx + x0 + c;
    for (int base = r0; base < ax.nin; base += KL * step) {
      double2 v[KL];
#pragma unroll
      for (int u = 0; u < KL; ++u) {
        const int lz = base + u * step;
        if (on && lz < ax.nin) v[u] = in[lz * plane];
      }
#pragma unroll
      for (int u = 0; u < KL; ++u) {
        const int lz = base + u * step;
        if (on && lz < ax.nin) b0[l * ax.ld + in_pos<PAD>(lz, ax)] = v[u];
      }
    }
  }
  __syncthreads();
  const double2 *r = stockham<PAD>(b0, b1, lines, ax);
  // slots written by this block: its elements, and the empty slots after the
  // last element when the block holds it; thread t takes slot t mod nw of
  // column (t / nw) mod nc, outputs t / (nw nc) + m (256 / (nw nc))
  const int e_end = e0 + ne == a.n_elem ? a.n_groups * a.slots : e0 + ne;
  const int nw = e_end - e0, lw = nw * nc;
  const int el = threadIdx.x % nw, c = (threadIdx.x / nw) % nc, o0 = threadIdx.x / lw, step = FFT_THREADS / lw;
  if (o0 >= step) return;
  const int e = e0 + el, grp = e / a.slots;
  float2 *out = a.packed + (((long long)grp * ax.nout * a.my + py) * a.mx + x0 + c) * a.slots + (e - grp * a.slots);
  const long long ostride = plane * a.slots;
  for (int o = o0; o < ax.nout; o += step) {
    float2 v = make_float2(0.0f, 0.0f);
    if (el < ne) {
      const double2 d = r[(el * nc + c) * ax.ld + out_pos<PAD>(o, ax)];
      v = make_float2((float)d.x, (float)d.y);
    }
    out[o * ostride] = v;
  }
}

// ---------------------------------------------------------------------------
// host side

// padded layout for powers of two (the transform's first radix is even)
static bool pad_of(int n) { return (n & (n - 1)) == 0; }

// line stride: room for the (padded) positions, rounded up to 1 mod 8 so that
// neighbouring lines start 4 banks apart
static int ld_of(int n) {
  const int l = pad_of(n) ? n + (n + 7) / 8 : n;
  return l + (9 - l % 8) % 8;
}

int nufft_fft_axis(int n, int nin, int pmin, int nout, const double2 *tw, FftAxis *ax) {
  if (n < 2 || n > NUFFT_FFT_MAX || nin < 1 || nin > n || nout < 1) return -1;
  FftAxis a;
  a.n = n;
  a.nin = nin;
  a.nout = nout;
  a.p0 = ((pmin % n) + n) % n;
  a.ld = ld_of(n);
  a.pad = pad_of(n) ? 1 : 0;
  a.tw = tw;
  a.nst = 0;
  int m = n;
  for (int r : {7, 5, 3, 8, 4, 2})
    while (m % r == 0) {
      if (a.nst == (int)(sizeof(a.rad) / sizeof(a.rad[0]))) return -1;
      a.rad[a.nst++] = r;
      m /= r;
    }
  if (m != 1) return -1;
  *ax = a;
  return 0;
}

void nufft_fft_twiddles(int n, double2 *tw) {
  for (int k = 0; k < n; ++k) {
    const long double t = 2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)n;
    tw[k] = make_double2((double)std::cos(t), (double)-std::sin(t));
  }
}

static constexpr size_t kSmemBudget = 72 * 1024;  // three blocks per SM
static const size_t kSmemMax = 2 * (size_t)std::max(ld_of(NUFFT_FFT_MAX), ld_of(4096)) * sizeof(double2);  // one line

static cudaError_t smem_opt_in() {
  static thread_local int done_dev = -1;
  int dev;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev == done_dev) return e;
  for (const void *f : {(const void *)nufft_fft_x_kernel<false>, (const void *)nufft_fft_y_kernel<false>,
                        (const void *)nufft_fft_z_kernel<false>, (const void *)nufft_fft_x_kernel<true>,
                        (const void *)nufft_fft_y_kernel<true>, (const void *)nufft_fft_z_kernel<true>}) {
    e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax);
    if (e != cudaSuccess) return e;
  }
  done_dev = dev;
  return cudaSuccess;
}

static int lines_for(const FftAxis &ax, int cap) {
  cap = std::min(cap, FFT_MAX_LINES);
  const size_t line = 2 * (size_t)ax.ld * sizeof(double2);
  return (int)std::max<size_t>(1, std::min<size_t>(cap, kSmemBudget / line));
}

cudaError_t nufft_fft3(const double *small, int copies, const double *dec, const NufftGeom &g, int n_elem,
                       const FftAxis ax[3], double2 *fa, double2 *fb, float4 *packed, cudaStream_t st) {
  cudaError_t e = smem_opt_in();
  if (e != cudaSuccess) return e;
  const int mx = ax[0].nout, my = ax[1].nout;
  {
    FftPassX p;
    p.ax = ax[0];
    p.small = small;
    p.copies = std::max(copies, 1);
    p.cells1 = (long long)g.n1[0] * g.n1[1] * g.n1[2];
    p.copy_stride = 2 * (long long)n_elem * p.cells1;
    p.dec = dec;
    p.n1y = g.n1[1];
    p.n1z = g.n1[2];
    p.lines = (long long)n_elem * g.n1[2] * g.n1[1];
    p.per_cta = lines_for(ax[0], 16);
    p.out = fa;
    const size_t smem = 2 * (size_t)p.per_cta * ax[0].ld * sizeof(double2);
    const long long blocks = (p.lines + p.per_cta - 1) / p.per_cta;
    if (p.ax.pad)
      nufft_fft_x_kernel<true><<<(unsigned)blocks, FFT_THREADS, smem, st>>>(p);
    else
      nufft_fft_x_kernel<false><<<(unsigned)blocks, FFT_THREADS, smem, st>>>(p);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  {
    FftPassY p;
    p.ax = ax[1];
    p.in = fa;
    p.out = fb;
    p.mx = mx;
    p.per_cta = lines_for(ax[1], 16);
    const size_t smem = 2 * (size_t)p.per_cta * ax[1].ld * sizeof(double2);
    const long long blocks = (long long)((mx + p.per_cta - 1) / p.per_cta) * n_elem * g.n1[2];
    if (p.ax.pad)
      nufft_fft_y_kernel<true><<<(unsigned)blocks, FFT_THREADS, smem, st>>>(p);
    else
      nufft_fft_y_kernel<false><<<(unsigned)blocks, FFT_THREADS, smem, st>>>(p);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  {
    FftPassZ p;
    p.ax = ax[2];
    p.in = fb;
    p.packed = (float2 *)packed;
    p.mx = mx;
    p.my = my;
    p.n_elem = n_elem;
    p.slots = 2 * nufft_pack_halves(n_elem);
    p.n_groups = nufft_pack_groups(n_elem);
    const int cols = lines_for(ax[2], 64);
    if (cols >= n_elem) {
      p.per_elem = n_elem;
      p.per_cta = std::min(16, cols / n_elem);
    } else {
      p.per_elem = std::min(cols, p.slots);
      p.per_cta = 1;
    }
    const size_t smem = 2 * (size_t)p.per_elem * p.per_cta * ax[2].ld * sizeof(double2);
    const dim3 grid((unsigned)((mx + p.per_cta - 1) / p.per_cta), (unsigned)my,
                    (unsigned)((n_elem + p.per_elem - 1) / p.per_elem));
    if (p.ax.pad)
      nufft_fft_z_kernel<true><<<grid, FFT_THREADS, smem, st>>>(p);
    else
      nufft_fft_z_kernel<false><<<grid, FFT_THREADS, smem, st>>>(p);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace spsim
