// Pipe-throughput probe for the roofline of the structure-factor kernels.
// Each kernel runs independent arithmetic chains (FP32 FMA, packed f32x2 FMA,
// both mixed, MUFU sin, ALU logic, packed FMA with logic riding along, FP64
// FMA alone and beside packed FP32, FP64->FP32 conversion) or the
// structure-factor inner loop in isolation (term32, term64), and
// stores one value per thread; the host prints lane-operations per clock per SM
// and a JSON line with the measured FP32-FMA and MUFU rates (ops/s) that
// bench.py uses as the measured peak of R = min(P_FMA/5, P_MUFU/2); bench.py
// builds it (nvcc, sm_100a) into _build/pipe_probe on first use.
#include <cstdio>
#include <cstring>
#include <cuda_runtime.h>
#include "spsim_b200/csrc/sincos_poly.h"
#define N_IT 4096
__global__ void k_ffma(float *out, float b, float c) {
  float a[16];
  for (int i = 0; i < 16; ++i) a[i] = threadIdx.x * 1e-3f + i;
  for (int it = 0; it < N_IT; ++it)
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = fmaf(a[i], b, c);
  float s = 0; for (int i = 0; i < 16; ++i) s += a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
__global__ void k_ffma2(float2 *out, float b, float c) {
  float2 a[8];
  for (int i = 0; i < 8; ++i) a[i] = make_float2(threadIdx.x * 1e-3f + i, i);
  const float2 bb = make_float2(b, b), cc = make_float2(c, c);
  for (int it = 0; it < N_IT; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = __ffma2_rn(a[i], bb, cc);
  float2 s = make_float2(0, 0); for (int i = 0; i < 8; ++i) s = __fadd2_rn(s, a[i]);
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
// 8 packed chains + 8 scalar chains: FMA lane-ops per iteration = 16 + 8
__global__ void k_mixed(float *out, float b, float c) {
  float2 a[8]; float d[8];
  for (int i = 0; i < 8; ++i) { a[i] = make_float2(threadIdx.x * 1e-3f + i, i); d[i] = i * 0.5f; }
  const float2 bb = make_float2(b, b), cc = make_float2(c, c);
  for (int it = 0; it < N_IT; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) { a[i] = __ffma2_rn(a[i], bb, cc); d[i] = fmaf(d[i], b, c); }
  }
  float s = 0; for (int i = 0; i < 8; ++i) s += a[i].x + a[i].y + d[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
__global__ void k_mufu(float *out, float b) {
  float a[8];
  for (int i = 0; i < 8; ++i) a[i] = threadIdx.x * 1e-3f + i;
  for (int it = 0; it < N_IT / 4; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) { float x; asm("sin.approx.ftz.f32 %0, %1;" : "=f"(x) : "f"(a[i])); a[i] = x + b; }
  float s = 0; for (int i = 0; i < 8; ++i) s += a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
__global__ void k_alu(unsigned *out, unsigned b) {
  unsigned a[16];
  for (int i = 0; i < 16; ++i) a[i] = threadIdx.x + i;
  for (int it = 0; it < N_IT; ++it)
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = (a[i] ^ b) & (a[i] | 0x9e3779b9u);  // one LOP3
  unsigned s = 0; for (int i = 0; i < 16; ++i) s ^= a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
// packed FMA chains with interleaved scalar ALU selects (the quadrant pattern)
__global__ void k_ffma2_alu(float2 *out, float b, float c, unsigned m) {
  float2 a[8]; unsigned u[8];
  for (int i = 0; i < 8; ++i) { a[i] = make_float2(threadIdx.x * 1e-3f + i, i); u[i] = threadIdx.x + i; }
  const float2 bb = make_float2(b, b), cc = make_float2(c, c);
  for (int it = 0; it < N_IT; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) { a[i] = __ffma2_rn(a[i], bb, cc); u[i] = (u[i] ^ m) & (u[i] | 0x9e3779b9u); }
  float s = 0; unsigned t = 0; for (int i = 0; i < 8; ++i) { s += a[i].x + a[i].y; t ^= u[i]; }
  out[blockIdx.x * blockDim.x + threadIdx.x] = make_float2(s, (float)t);
}
// FP64 fused multiply-add chains
__global__ void k_dfma(double *out, double b, double c) {
  double a[8];
  for (int i = 0; i < 8; ++i) a[i] = threadIdx.x * 1e-3 + i;
  for (int it = 0; it < N_IT / 2; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = fma(a[i], b, c);
  double s = 0; for (int i = 0; i < 8; ++i) s += a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
// packed FP32 chains and FP64 chains interleaved: counts FMA lane-ops; 4 DFMA per 16 FMA lane-ops ride along
__global__ void k_ffma2_dfma(float2 *out, float b, float c, double bd, double cd) {
  float2 a[8]; double d[4];
  for (int i = 0; i < 8; ++i) a[i] = make_float2(threadIdx.x * 1e-3f + i, i);
  for (int i = 0; i < 4; ++i) d[i] = threadIdx.x * 1e-3 + i;
  const float2 bb = make_float2(b, b), cc = make_float2(c, c);
  for (int it = 0; it < N_IT; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = __ffma2_rn(a[i], bb, cc);
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] = fma(d[i], bd, cd);
  }
  float s = 0; double t = 0; for (int i = 0; i < 8; ++i) s += a[i].x + a[i].y;
  for (int i = 0; i < 4; ++i) t += d[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = make_float2(s, (float)t);
}
// FP64 -> FP32 conversions (one F2F per op; the DADD keeps the chain dependent)
__global__ void k_f2f(float *out, double b) {
  double a[8]; float f[8];
  for (int i = 0; i < 8; ++i) { a[i] = threadIdx.x * 1e-3 + i; f[i] = 0; }
  for (int it = 0; it < N_IT / 4; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) { a[i] = a[i] * b + 1e-3; f[i] += __double2float_rn(a[i]); }
  float s = 0; for (int i = 0; i < 8; ++i) s += f[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// 32-bit integer multiply-add chains, multiplier in a register (kernel argument)
__global__ void k_imad(unsigned *out, unsigned m) {
  unsigned a[16];
  for (int i = 0; i < 16; ++i) a[i] = threadIdx.x + i;
  for (int it = 0; it < N_IT; ++it)
#pragma unroll
    for (int i = 0; i < 16; ++i) asm("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[i]) : "r"(m), "r"((unsigned)i));
  unsigned s = 0; for (int i = 0; i < 16; ++i) s ^= a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// FP64 -> int32 (round to nearest) -> FP64 conversions: two conversions per op
__global__ void k_cvt(double *out, double b) {
  double a[8];
  for (int i = 0; i < 8; ++i) a[i] = threadIdx.x * 1e-3 + i;
  for (int it = 0; it < N_IT / 4; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = (double)__double2int_rn(a[i] * b);
  double s = 0; for (int i = 0; i < 8; ++i) s += a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// FP64 tensor-core MMA (m8n8k4): 8 independent accumulator tiles per warp;
// 8 x 8 x 4 = 256 FMA per MMA per warp, i.e. 8 FP64 FMA lane-ops per thread
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}
__global__ void k_dmma(double *out, double a, double b) {
  double d[8][2];
  for (int i = 0; i < 8; ++i) d[i][0] = d[i][1] = threadIdx.x * 1e-3 + i;
  const double aa = a + threadIdx.x * 1e-9, bb = b - threadIdx.x * 1e-9;
  for (int it = 0; it < N_IT / 8; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) dmma(d[i][0], d[i][1], aa, bb);
  double s = 0; for (int i = 0; i < 8; ++i) s += d[i][0] + d[i][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
// packed FP32 chains with FP64 MMAs riding along: counts FMA lane-ops; 2 MMAs
// (16 FP64 FMA lane-ops per thread) per 16 FP32 FMA lane-ops
__global__ void k_ffma2_dmma(float2 *out, float b, float c, double ad, double bd) {
  float2 a[8]; double d[2][2];
  for (int i = 0; i < 8; ++i) a[i] = make_float2(threadIdx.x * 1e-3f + i, i);
  for (int i = 0; i < 2; ++i) d[i][0] = d[i][1] = threadIdx.x * 1e-3 + i;
  const float2 bb = make_float2(b, b), cc = make_float2(c, c);
  for (int it = 0; it < N_IT; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = __ffma2_rn(a[i], bb, cc);
#pragma unroll
    for (int i = 0; i < 2; ++i) dmma(d[i][0], d[i][1], ad, bd);
  }
  float s = 0; double t = 0; for (int i = 0; i < 8; ++i) s += a[i].x + a[i].y;
  for (int i = 0; i < 2; ++i) t += d[i][0] + d[i][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = make_float2(s, (float)t);
}
// FP64 vector FMA chains with FP64 MMAs riding along: counts DFMA lane-ops; 1 MMA per 4 DFMA
__global__ void k_dfma_dmma(double *out, double b, double c, double ad, double bd) {
  double a[4]; double d[2][2];
  for (int i = 0; i < 4; ++i) a[i] = threadIdx.x * 1e-3 + i;
  for (int i = 0; i < 2; ++i) d[i][0] = d[i][1] = threadIdx.x * 1e-3 + i;
  for (int it = 0; it < N_IT / 2; ++it) {
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = fma(a[i], b, c);
    dmma(d[it & 1][0], d[it & 1][1], ad, bd);
  }
  double s = 0; for (int i = 0; i < 4; ++i) s += a[i];
  for (int i = 0; i < 2; ++i) s += d[i][0] + d[i][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// ---- the structure-factor inner loop in isolation: 256 atoms in shared
// memory, PP pixel pairs per thread, every term of the half-cycle polynomial
// form.  term32: compensated FP32 phase (Q_hi.R_hi + cross term);
// term64: FP64 phase and FP64 half-cycle reduction, FP32 polynomial.
#define PP 2
#define N_ATOMS 256
__device__ __forceinline__ float2 f2v(float a) { return make_float2(a, a); }
__device__ __forceinline__ void half_poly2(float2 y, float2 &S, float2 &C) {
  const float2 z = __fmul2_rn(y, y);
  float2 ps = __ffma2_rn(z, f2v(SPSIM_HALF_S4), f2v(SPSIM_HALF_S3));
  ps = __ffma2_rn(z, ps, f2v(SPSIM_HALF_S2));
  ps = __ffma2_rn(z, ps, f2v(SPSIM_HALF_S1));
  ps = __ffma2_rn(z, ps, f2v(SPSIM_HALF_S0));
  float2 pc = __ffma2_rn(z, f2v(SPSIM_HALF_C5), f2v(SPSIM_HALF_C4));
  pc = __ffma2_rn(z, pc, f2v(SPSIM_HALF_C3));
  pc = __ffma2_rn(z, pc, f2v(SPSIM_HALF_C2));
  pc = __ffma2_rn(z, pc, f2v(SPSIM_HALF_C1));
  pc = __ffma2_rn(z, pc, f2v(SPSIM_HALF_C0));
  S = __fmul2_rn(y, ps);
  C = pc;
}
__device__ __forceinline__ void dhalf_poly2(float2 y, float2 &S, float2 &C) {
  const float2 z = __fmul2_rn(y, y);
  float2 ps = __ffma2_rn(z, f2v(SPSIM_DHALF_S4), f2v(SPSIM_DHALF_S3));
  ps = __ffma2_rn(z, ps, f2v(SPSIM_DHALF_S2));
  ps = __ffma2_rn(z, ps, f2v(SPSIM_DHALF_S1));
  ps = __ffma2_rn(z, ps, f2v(SPSIM_DHALF_S0));
  float2 pc = __ffma2_rn(z, f2v(SPSIM_DHALF_C4), f2v(SPSIM_DHALF_C3));
  pc = __ffma2_rn(z, pc, f2v(SPSIM_DHALF_C2));
  pc = __ffma2_rn(z, pc, f2v(SPSIM_DHALF_C1));
  pc = __ffma2_rn(z, pc, f2v(SPSIM_DHALF_C0));
  S = __fmul2_rn(y, ps);
  C = pc;
}
// (-1)^k w: bit 0 of k moved to the sign bit.  SIGN 0: shift and xor (two
// logic ops); SIGN 1: one integer multiply-add with the multiplier 2^31 held
// in a register (adding 2^31 flips the sign bit).
template <int SIGN>
__device__ __forceinline__ float signed_w(float w, unsigned kbits, unsigned m31) {
  if (SIGN == 0) return __uint_as_float(__float_as_uint(w) ^ (kbits << 31));
  unsigned r;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(kbits), "r"(m31), "r"(__float_as_uint(w)));
  return __uint_as_float(r);
}
template <int SIGN>
__global__ void __launch_bounds__(256) k_term32(float4 *out, int reps, unsigned m31) {
  __shared__ float4 hi[N_ATOMS], lo[N_ATOMS];
  for (int i = threadIdx.x; i < N_ATOMS; i += blockDim.x) {
    hi[i] = make_float4((i % 37) * 3.0f, (i % 29) * 5.0f, (i % 31) * 7.0f, 1.0f);
    lo[i] = make_float4(i * 1e-4f, -i * 2e-4f, i * 3e-5f, 0.0f);
  }
  __syncthreads();
  float2 qh[PP][3], q[PP][3], ql[PP][3], bc[PP], bs[PP];
  for (int j = 0; j < PP; ++j)
    for (int d = 0; d < 3; ++d) {
      qh[j][d] = make_float2((threadIdx.x + d + j) * 0.25f, (threadIdx.x + 2 * d + j) * 0.125f);
      ql[j][d] = make_float2(1e-5f * d, -2e-5f * j);
      q[j][d] = __fadd2_rn(qh[j][d], ql[j][d]);
      bc[j] = bs[j] = make_float2(0.f, 0.f);
    }
  for (int r = 0; r < reps; ++r)
    for (int a = 0; a < N_ATOMS; ++a) {
      const float4 H = hi[a], L = lo[a];
#pragma unroll
      for (int j = 0; j < PP; ++j) {
        float2 u = __fmul2_rn(qh[j][0], f2v(H.x));
        u = __ffma2_rn(qh[j][1], f2v(H.y), u);
        u = __ffma2_rn(qh[j][2], f2v(H.z), u);
        float2 c = __fmul2_rn(q[j][0], f2v(L.x));
        c = __ffma2_rn(q[j][1], f2v(L.y), c);
        c = __ffma2_rn(q[j][2], f2v(L.z), c);
        c = __ffma2_rn(ql[j][0], f2v(H.x), c);
        c = __ffma2_rn(ql[j][1], f2v(H.y), c);
        c = __ffma2_rn(ql[j][2], f2v(H.z), c);
        const float2 t = __ffma2_rn(u, f2v(2.0f), f2v(12582912.0f));
        const float2 kf = __fadd2_rn(t, f2v(-12582912.0f));
        const float2 y = __fadd2_rn(__ffma2_rn(kf, f2v(-0.5f), u), c);
        float2 S, C;
        half_poly2(y, S, C);
        const float2 ws = make_float2(signed_w<SIGN>(H.w, __float_as_uint(t.x), m31),
                                      signed_w<SIGN>(H.w, __float_as_uint(t.y), m31));
        bc[j] = __ffma2_rn(ws, C, bc[j]);
        bs[j] = __ffma2_rn(ws, S, bs[j]);
      }
    }
  float4 o = make_float4(0, 0, 0, 0);
  for (int j = 0; j < PP; ++j) { o.x += bc[j].x; o.y += bc[j].y; o.z += bs[j].x; o.w += bs[j].y; }
  out[blockIdx.x * blockDim.x + threadIdx.x] = o;
}
// term64 with the rounding of 2u done by conversions (XU pipe): k = rint(2u)
// as an integer, back to FP64, one DFMA for u - k/2.  RED 0: the magic-number
// rounding (two more FP64 operations, no conversions).
template <int SIGN, int RED = 0>
__global__ void __launch_bounds__(256) k_term64(float4 *out, int reps, unsigned m31) {
  __shared__ double4 at[N_ATOMS];
  for (int i = threadIdx.x; i < N_ATOMS; i += blockDim.x)
    at[i] = make_double4((i % 37) * 3.01, (i % 29) * 5.03, (i % 31) * 7.07, 1.0);
  __syncthreads();
  double q[2 * PP][3];
  float2 bc[PP], bs[PP];
  for (int j = 0; j < 2 * PP; ++j)
    for (int d = 0; d < 3; ++d) q[j][d] = (threadIdx.x + d + j) * 0.2500123;
  for (int j = 0; j < PP; ++j) bc[j] = bs[j] = make_float2(0.f, 0.f);
  const double M = 6755399441055744.0;  // 1.5 * 2^52
  for (int r = 0; r < reps; ++r)
    for (int a = 0; a < N_ATOMS; ++a) {
      const double4 A = at[a];
      const float w = (float)A.w;
#pragma unroll
      for (int j = 0; j < PP; ++j) {
        double t2[2];
        float yv[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          double u = q[2 * j + h][0] * A.x;
          u = fma(q[2 * j + h][1], A.y, u);
          u = fma(q[2 * j + h][2], A.z, u);
          if (RED == 0) {
            const double t = fma(u, 2.0, M);
            const double kf = t - M;
            yv[h] = __double2float_rn(fma(kf, -0.5, u));
            t2[h] = t;
          } else {
            const int k = __double2int_rn(2.0 * u);
            yv[h] = __double2float_rn(fma((double)k, -0.5, u));
            t2[h] = __hiloint2double(0, k);
          }
        }
        float2 S, C;
        dhalf_poly2(make_float2(yv[0], yv[1]), S, C);
        const float2 ws = make_float2(signed_w<SIGN>(w, (unsigned)__double2loint(t2[0]), m31),
                                      signed_w<SIGN>(w, (unsigned)__double2loint(t2[1]), m31));
        bc[j] = __ffma2_rn(ws, C, bc[j]);
        bs[j] = __ffma2_rn(ws, S, bs[j]);
      }
    }
  float4 o = make_float4(0, 0, 0, 0);
  for (int j = 0; j < PP; ++j) { o.x += bc[j].x; o.y += bc[j].y; o.z += bs[j].x; o.w += bs[j].y; }
  out[blockIdx.x * blockDim.x + threadIdx.x] = o;
}

static double g_fma = 0, g_mufu = 0, g_dfma = 0, g_imad = 0, g_alu = 0;

int main() {
  int sms; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  int clk; cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, 0);
  const int blocks = sms * 8, threads = 256;
  void *buf; cudaMalloc(&buf, (size_t)blocks * threads * 16);  // 16 B per thread: the widest store (float4)
  cudaEvent_t e0, e1; cudaEventCreate(&e0); cudaEventCreate(&e1);
  const double thr = (double)blocks * threads;
  auto run = [&](const char *name, auto launch, double ops_per_thread) {
    launch(); cudaDeviceSynchronize();
    cudaEventRecord(e0); for (int r = 0; r < 5; ++r) launch(); cudaEventRecord(e1); cudaEventSynchronize(e1);
    float ms; cudaEventElapsedTime(&ms, e0, e1); ms /= 5;
    double per_s = thr * ops_per_thread / (ms * 1e-3);
    printf("%-12s %8.3f ms  %.4e lane-ops/s  %.1f lane-ops/clk/SM (at %.0f MHz)\n", name, ms, per_s,
           per_s / sms / (clk * 1e3), clk / 1e3);
    if (name[0] == 'f' && name[1] == 'f' && name[4] == 0) g_fma = per_s > g_fma ? per_s : g_fma;
    if (name[0] == 'm') g_mufu = per_s;
    if (!strcmp(name, "dfma")) g_dfma = per_s;
    if (!strcmp(name, "imad")) g_imad = per_s;
    if (!strcmp(name, "alu_lop3")) g_alu = per_s;
  };
  run("ffma", [&] { k_ffma<<<blocks, threads>>>((float *)buf, 0.999f, 1e-3f); }, 16.0 * N_IT);
  run("ffma2", [&] { k_ffma2<<<blocks, threads>>>((float2 *)buf, 0.999f, 1e-3f); }, 16.0 * N_IT);
  run("mixed", [&] { k_mixed<<<blocks, threads>>>((float *)buf, 0.999f, 1e-3f); }, 24.0 * N_IT);
  run("mufu_sin", [&] { k_mufu<<<blocks, threads>>>((float *)buf, 0.5f); }, 8.0 * (N_IT / 4));
  run("alu_lop3", [&] { k_alu<<<blocks, threads>>>((unsigned *)buf, 0x1234u); }, 16.0 * N_IT);
  run("ffma2+alu", [&] { k_ffma2_alu<<<blocks, threads>>>((float2 *)buf, 0.999f, 1e-3f, 0x55u); }, 16.0 * N_IT);
  printf("(ffma2+alu counts only FMA lane-ops; 8 ALU ops per 16 FMA lane-ops ride along)\n");
  run("dfma", [&] { k_dfma<<<blocks, threads>>>((double *)buf, 0.999, 1e-3); }, 8.0 * (N_IT / 2));
  run("imad", [&] { k_imad<<<blocks, threads>>>((unsigned *)buf, 0x9e3779b9u); }, 16.0 * N_IT);
  run("ffma2+dfma", [&] { k_ffma2_dfma<<<blocks, threads>>>((float2 *)buf, 0.999f, 1e-3f, 0.999, 1e-3); },
      16.0 * N_IT);
  printf("(ffma2+dfma counts only FMA lane-ops; 4 DFMA per 16 FMA lane-ops ride along)\n");
  run("f2f_dmul", [&] { k_f2f<<<blocks, threads>>>((float *)buf, 0.999); }, 8.0 * (N_IT / 4));
  run("cvt_d2i2d", [&] { k_cvt<<<blocks, threads>>>((double *)buf, 1.001); }, 8.0 * (N_IT / 4));
  printf("(cvt_d2i2d counts round trips: DMUL + F2I.F64 + I2F.F64 each)\n");
  run("dmma", [&] { k_dmma<<<blocks, threads>>>((double *)buf, 0.999, 1e-3); }, 8.0 * 8 * (N_IT / 8));
  printf("(dmma counts FP64 FMA lane-ops: 8 per thread per m8n8k4)\n");
  run("ffma2+dmma", [&] { k_ffma2_dmma<<<blocks, threads>>>((float2 *)buf, 0.999f, 1e-3f, 0.999, 1e-3); },
      16.0 * N_IT);
  printf("(ffma2+dmma counts only FP32 FMA lane-ops; 16 FP64 MMA lane-ops per 16 ride along)\n");
  run("dfma+dmma", [&] { k_dfma_dmma<<<blocks, threads>>>((double *)buf, 0.999, 1e-3, 0.999, 1e-3); },
      4.0 * (N_IT / 2));
  printf("(dfma+dmma counts only DFMA lane-ops; 8 FP64 MMA lane-ops per 4 ride along)\n");
  const int reps = 16;
  const unsigned m31 = 0x80000000u;
  run("term32", [&] { k_term32<0><<<blocks, threads>>>((float4 *)buf, reps, m31); }, 2.0 * PP * N_ATOMS * reps);
  run("term32_imad", [&] { k_term32<1><<<blocks, threads>>>((float4 *)buf, reps, m31); }, 2.0 * PP * N_ATOMS * reps);
  run("term64", [&] { k_term64<0><<<blocks, threads>>>((float4 *)buf, reps, m31); }, 2.0 * PP * N_ATOMS * reps);
  run("term64_imad", [&] { k_term64<1><<<blocks, threads>>>((float4 *)buf, reps, m31); }, 2.0 * PP * N_ATOMS * reps);
  run("term64_cvt", [&] { k_term64<1, 1><<<blocks, threads>>>((float4 *)buf, reps, m31); }, 2.0 * PP * N_ATOMS * reps);
  printf("(term32 / term64 count structure-factor terms)\n");
  printf("{\"fma_lane_ops_per_s\": %.6e, \"mufu_ops_per_s\": %.6e, \"dfma_lane_ops_per_s\": %.6e, "
         "\"imad_lane_ops_per_s\": %.6e, \"alu_lane_ops_per_s\": %.6e, \"sms\": %d, \"clock_mhz\": %.0f}\n",
         g_fma, g_mufu, g_dfma, g_imad, g_alu, sms, clk / 1e3);
  cudaError_t e = cudaGetLastError(); printf("status %s\n", cudaGetErrorString(e));
  return e != cudaSuccess;
}
