// Detector chain after the structure factor, fused per pixel:
//   Thomson factor            src/diffraction.c:1109-1144
//   pixel solid angle         src/diffraction.c:1146-1187
//   photons = T * Omega * I * I0                         :1190-1204
//   photon count (Poisson)    src/noise.c:32-51  (counter-based Philox stream 0
//                             instead of GSL's unseeded global generator)
//   electrons                 src/amplification.c:54-74
//   real output               src/amplification.c:77-116 (Philox stream 1 readout noise)
//   noiseless output          src/amplification.c:119-155
// Float/double choices follow the reference line by line so that the
// deterministic outputs agree with it to float rounding.
#include "chain_kernels.cuh"

namespace spsim {

// ---- Philox4x32-10 (Salmon et al., SC'11) ----------------------------------

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
    const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
    c[0] = n0;
    c[1] = n1;
    c[2] = n2;
    c[3] = n3;
    k0 += W0;
    k1 += W1;
  }
}

struct PhiloxStream {
  uint32_t ctr[4];
  uint32_t k0, k1;
  uint32_t buf[4];
  int left;
  __device__ PhiloxStream(uint32_t item, uint32_t pattern, uint32_t sid, uint64_t seed) {
    ctr[0] = item;
    ctr[1] = pattern;
    ctr[2] = sid;
    ctr[3] = 0;
    k0 = (uint32_t)seed;
    k1 = (uint32_t)(seed >> 32);
    left = 0;
  }
  __device__ float uniform() {  // (0, 1)
    if (left == 0) {
      buf[0] = ctr[0];
      buf[1] = ctr[1];
      buf[2] = ctr[2];
      buf[3] = ctr[3];
      philox4x32_10(buf, k0, k1);
      ++ctr[3];
      left = 4;
    }
    const uint32_t x = buf[4 - left--];
    return ((float)(x >> 8) + 0.5f) * 5.9604644775390625e-8f;
  }
  __device__ float normal() {  // Box-Muller, first of the pair
    const float a = uniform(), b = uniform();
    return sqrtf(-2.0f * logf(a)) * cosf(6.2831853071795864f * b);
  }
};

// Poisson(lam): inversion below 10, Hormann's PTRS transformed rejection
// (Insurance: Math. & Econ. 12 (1993) 39-45) up to 1000, and the reference's
// Gaussian approximation (int)(lam + N(0, sqrt(lam))) above (src/noise.c:42-46).
__device__ float poisson_sample(PhiloxStream &s, float lam) {
  if (!(lam > 0.0f)) return 0.0f;
  if (lam >= 1000.0f) {
    const float v = lam + sqrtf(lam) * s.normal();
    return (float)(int)v;
  }
  if (lam < 10.0f) {
    const float u = s.uniform();
    float p = expf(-lam), F = p;
    int k = 0;
    while (u > F && k < 200) {
      ++k;
      p *= lam / (float)k;
      F += p;
    }
    return (float)k;
  }
  const float slam = sqrtf(lam), loglam = logf(lam);
  const float b = 0.931f + 2.53f * slam;
  const float a = -0.059f + 0.02483f * b;
  const float inv_alpha = 1.1239f + 1.1328f / (b - 3.4f);
  const float vr = 0.9277f - 3.6224f / (b - 2.0f);
  for (int it = 0; it < 64; ++it) {
    const float U = s.uniform() - 0.5f;
    const float V = s.uniform();
    const float us = 0.5f - fabsf(U);
    const float k = floorf((2.0f * a / us + b) * U + lam + 0.43f);
    if (us >= 0.07f && V <= vr) return k;
    if (k < 0.0f || (us < 0.013f && V > us)) continue;
    if (logf(V) + logf(inv_alpha) - logf(a / (us * us) + b) <= -lam + k * loglam - lgammaf(k + 1.0f)) return k;
  }
  return (float)(int)(lam + slam * s.normal());
}

// ---- per-pixel geometry factors --------------------------------------------

__device__ __forceinline__ float thomson_factor(const ChainDev &c, int x, int y) {
  const double r0 = 2.81794e-15;
  double pf = 1.0;
  if (c.polarization != 0) {
    const double px = ((x - (c.nx - 1.0) / 2.0) / c.nx) * c.width - c.cx;
    const double py = ((y - (c.ny - 1.0) / 2.0) / c.ny) * c.height - c.cy;
    const double r = sqrt(px * px + py * py + c.distance * c.distance);
    if (c.polarization == 1) {
      const double chi = asin(py / r);
      pf = cos(chi) * cos(chi);
    } else if (c.polarization == 2) {
      const double chi = asin(px / r);
      pf = cos(chi) * cos(chi);
    } else if (c.polarization == 3) {
      const double chi = asin(sqrt(px * px + py * py) / r);
      pf = (1.0 + cos(chi) * cos(chi)) / 2.0;
    }
  }
  return (float)((r0 * r0) * pf);
}

__device__ __forceinline__ float solid_angle_factor(const ChainDev &c, int x, int y) {
  if (c.nz > 1 || c.spherical) {
    const double r = c.distance;
    return (float)(c.pw * c.ph / (r * r));
  }
  const double px = ((x - (c.nx - 1.0) / 2.0) / c.nx) * c.width - c.cx;
  const double py = ((y - (c.ny - 1.0) / 2.0) / c.ny) * c.height - c.cy;
  double inc = atan(sqrt(px * px + py * py) / c.distance);
  inc = cos(inc);
  inc = inc * inc * inc;
  return (float)(c.pw * c.ph / (c.distance * c.distance) * inc);
}

// ---- fused chain -------------------------------------------------------------

__global__ void chain_pixel_kernel(ChainDev c, const float *__restrict__ I, ChainOut o) {
  const long long i = c.i0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.i1) return;
  const int x = (int)(i % c.nx);
  const int y = (int)((i / c.nx) % c.ny);
  const float T = thomson_factor(c, x, y);
  const float Om = solid_angle_factor(c, x, y);
  if (o.thomson) o.thomson[i] = T;
  if (o.solid_angle) o.solid_angle[i] = Om;
  if (!I) return;
  const float ph = T * Om * I[i] * c.beam_intensity;
  if (o.photons) o.photons[i] = ph;
  if (o.noiseless && c.unbinned) o.noiseless[i] = ph * c.qe * c.epp_noiseless * c.adc;
  if (!o.counts && !o.electrons && !o.real_out) return;
  PhiloxStream s((uint32_t)i, c.pattern, 0u, c.seed);
  const float cnt = poisson_sample(s, ph * c.qe);
  if (o.counts) o.counts[i] = cnt;
  const float el = cnt * c.epp;
  if (o.electrons) o.electrons[i] = el;
  if (o.real_out && c.unbinned) {
    float v = 0.0f;
    v += (el + c.dark_t);
    PhiloxStream r((uint32_t)i, c.pattern, 1u, c.seed);
    v += c.readout * r.normal();
    if (v < 0) v = 0;
    v *= c.adc;
    if (c.clamp && c.maxv != 0.0f && v > c.maxv) v = c.maxv;
    o.real_out[i] = v;
  }
}

// Binned outputs (binning > 1): sums in the reference's loop order.
__global__ void chain_bin_kernel(ChainDev c, const float *__restrict__ photons, const float *__restrict__ electrons,
                                 float *__restrict__ real_out, float *__restrict__ noiseless) {
  const int bnx = c.nx / c.bx, bny = c.ny / c.by;
  const long long b = c.b0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= c.b1) return;
  const int x = (int)(b % bnx), y = (int)((b / bnx) % bny), z = (int)(b / ((long long)bnx * bny));
  float acc_r = 0.0f, acc_n = 0.0f;
  for (int zi = 0; zi < c.bz; ++zi)
    for (int yi = 0; yi < c.by; ++yi)
      for (int xi = 0; xi < c.bx; ++xi) {
        const long long src = ((long long)(z * c.bz + zi) * c.ny + (y * c.by + yi)) * c.nx + (x * c.bx + xi);
        if (real_out) acc_r += (electrons[src] + c.dark_t);
        if (noiseless) acc_n += (photons[src] * c.qe * c.epp_noiseless * c.adc);
      }
  if (real_out) {
    PhiloxStream r((uint32_t)b, c.pattern, 1u, c.seed);
    acc_r += c.readout * r.normal();
    if (acc_r < 0) acc_r = 0;
    acc_r *= c.adc;
    if (c.clamp && c.maxv != 0.0f && acc_r > c.maxv) acc_r = c.maxv;
    real_out[b] = acc_r;
  }
  if (noiseless) noiseless[b] = acc_n;
}

__global__ void poisson_kernel(long long n, const float *__restrict__ lam, uint64_t seed, uint32_t pattern,
                               float *__restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  PhiloxStream s((uint32_t)i, pattern, 0u, seed);
  out[i] = poisson_sample(s, lam[i]);
}

__global__ void photons_kernel(long long n, const float *__restrict__ T, const float *__restrict__ Om,
                               const float *__restrict__ I, float I0, float *__restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = T[i] * Om[i] * I[i] * I0;
}

__global__ void counts_kernel(ChainDev c, long long n, const float *__restrict__ ph, float *__restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  PhiloxStream s((uint32_t)i, c.pattern, 0u, c.seed);
  out[i] = poisson_sample(s, ph[i] * c.qe);
}

__global__ void electrons_kernel(long long n, const float *__restrict__ cnt, float epp, float *__restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = cnt[i] * epp;
}

cudaError_t launch_photons(long long n, const float *T, const float *Om, const float *I, float I0, float *out,
                           cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  photons_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, T, Om, I, I0, out);
  return cudaGetLastError();
}

cudaError_t launch_counts(const ChainDev &c, const float *ph, float *out, cudaStream_t st) {
  const long long n = (long long)c.nx * c.ny * c.nz;
  if (n <= 0) return cudaSuccess;
  counts_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(c, n, ph, out);
  return cudaGetLastError();
}

cudaError_t launch_electrons(const ChainDev &c, const float *cnt, float *out, cudaStream_t st) {
  const long long n = (long long)c.nx * c.ny * c.nz;
  if (n <= 0) return cudaSuccess;
  electrons_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, cnt, c.epp, out);
  return cudaGetLastError();
}

cudaError_t launch_binned(const ChainDev &c, const float *electrons, const float *photons, float *real_out,
                          float *noiseless, cudaStream_t st) {
  const long long nb = c.b1 - c.b0;
  if (nb <= 0) return cudaSuccess;
  chain_bin_kernel<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(c, photons, electrons, real_out, noiseless);
  return cudaGetLastError();
}

cudaError_t launch_chain(const ChainDev &c, const float *I, const ChainOut &o, float *scratch_ph, float *scratch_el,
                         cudaStream_t st) {
  const long long n = c.i1 - c.i0;
  if (n <= 0) return cudaSuccess;
  ChainOut po = o;
  if (!c.unbinned) {
    // the binning pass needs photons / electrons even when the caller does not
    if (o.noiseless && !po.photons) po.photons = scratch_ph;
    if (o.real_out && !po.electrons) po.electrons = scratch_el;
    po.noiseless = nullptr;
    po.real_out = nullptr;
  }
  chain_pixel_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(c, I, po);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || c.unbinned || (!o.noiseless && !o.real_out) || !I) return e;
  const long long nb = c.b1 - c.b0;
  if (nb <= 0) return cudaSuccess;
  chain_bin_kernel<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(c, po.photons, po.electrons, o.real_out,
                                                                 o.noiseless);
  return cudaGetLastError();
}

cudaError_t launch_poisson(long long n, const float *lam, uint64_t seed, uint32_t pattern, float *out,
                           cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  poisson_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, lam, seed, pattern, out);
  return cudaGetLastError();
}

}  // namespace spsim
