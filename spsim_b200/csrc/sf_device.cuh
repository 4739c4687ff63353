// Device-side data layout and helpers for the structure-factor kernels.
//
// Atom record (two float4 per atom, element-sorted, each element segment
// padded with zero-weight atoms to a multiple of ATOM_GROUP):
//   a0 = {hx, hy, hz, w}   coarse part R_hi of (r - centre), on the molecule's
//                          power-of-two grid dr; w = occ * sqrt(illumination)
//   a1 = {lx, ly, lz, b}   remainder R_lo = (r - centre) - R_hi; b = per-atom B (A^2)
// Pixel q is split the same way on the q set's grid dq, so that Q_hi . R_hi
// is exact in FP32 (<= 22 significant bits per product, dq*dr a power of two)
// and the phase u = q.(r - c) in cycles is
//   u = Q_hi.R_hi (exact)  +  [Q.R_lo + Q_lo.R_hi]  (small cross term, FP32)
// reduced modulo a quarter (or whole) cycle before sin/cos.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sincos_poly.h"

namespace spsim {

constexpr int PREC_MODE_POLY = 0;  // FMA-pipe minimax sin/cos (SPSIM_PREC_F32)
constexpr int PREC_MODE_MUFU = 1;  // MUFU sin/cos (SPSIM_PREC_F32_FAST)

constexpr int ATOM_GROUP = 8;        // segment padding and inner unroll
constexpr int TILE_ATOMS = 128;      // atoms per shared-memory tile (4 KiB)
constexpr int RING_STAGES = 3;       // bulk-copy ring depth
constexpr int MAX_ELEM = 100;

// Magic constant 1.5 * 2^23: x + MAGIC rounds x to the nearest integer for
// |x| < 2^22 and leaves that integer in the low mantissa bits.
constexpr float RINT_MAGIC = 12582912.0f;

// Work-item / pattern descriptors (host-built, device-read).
struct TileDesc {      // one shared-memory tile of a molecule
  int atom_begin;      // padded atom index
  int count;           // atoms in tile, multiple of ATOM_GROUP
  int elem;            // element slot (row of the form-factor table)
  int last;            // 1 if the tile ends its element segment
};

// FP64-phase record of one padded atom (32 bytes): r - centre in FP64, the
// weight w = occ * sqrt(illumination) and the per-atom B factor.
struct __align__(16) AtomD {
  double x, y, z;
  float w, b;
};

struct SfPattern {
  const float4 *atoms;     // 2 float4 per padded atom
  const float4 *atoms2;    // the same records duplicated for pixel pairs: 4 float4 per atom,
                           // {hx,hx,hy,hy} {hz,hz,w,w} {lx,lx,ly,ly} {lz,lz,b,b}
  const AtomD *atomsd;     // FP64-phase records, one per padded atom
  const TileDesc *tiles;   // molecule tile table
  int n_tiles;
  int n_elem;
  int per_atom_b;
  int has_rot;
  const double *ff;        // [n_elem][npix] FP64 form factors for this pattern
  long long npix;
  const float *hkl;        // AoS float3 q (1/m), or nullptr
  const double *q64;       // AoS double3 q (1/m), or nullptr
  double rot[9];           // row-major, applied as q' = R q
  double qscale;           // phase-space q = qscale * R q (wavelength sample of a spectrum; 1 otherwise)
  double s2scale;          // 1 / qscale^2: per-atom B factors use the unscaled |q|, like the form factors
  double center[3];        // molecule centre (m)
  float dq, inv_dq;        // pixel grid step (power of two) and its inverse
  double2 *acc;            // FP64 accumulator [npix] (zeroed before the forward)
  float2 *F;               // complex64 output [npix] or nullptr
  float *I;                // intensity output [npix] or nullptr
  long long tile0;         // first pixel-tile index of this pattern in a grid-mapped launch
  const int *mol_err;      // the molecule's range word (atoms moved past its bounds), or nullptr
  int *plan_err;           // where the finalizing kernel reports it
};

struct WorkItem {      // one CTA's unit of work
  int pattern;
  int pixel_tile;
  int k0, k1;          // tile range [k0, k1) of the molecule
};

// ---------------------------------------------------------------------------
// shared-memory barriers and bulk copies (inline PTX, sm_90+ forms)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after ~`limit_cycles` SM clocks and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, long long limit_cycles) {
  if (mbar_try_wait(bar, parity)) return true;
  long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit_cycles) return false;
  }
  return true;
}

// 1-D bulk copy global -> shared completing on an mbarrier (no multicast).
__device__ __forceinline__ void bulk_copy_g2s(void *smem_dst, const void *gmem_src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// ---------------------------------------------------------------------------
// per-term arithmetic

// sin(2 pi y), cos(2 pi y) for |y| <= 3/16 cycle: minimax polynomials on the
// FMA pipe (coefficients from gen_sincos_poly.py).
__device__ __forceinline__ void sincos_quad_poly(float y, float &s, float &c) {
  const float z = y * y;
  float ps = fmaf(z, SPSIM_QUAD_S4, SPSIM_QUAD_S3);
  ps = fmaf(z, ps, SPSIM_QUAD_S2);
  ps = fmaf(z, ps, SPSIM_QUAD_S1);
  ps = fmaf(z, ps, SPSIM_QUAD_S0);
  float pc = fmaf(z, SPSIM_QUAD_C4, SPSIM_QUAD_C3);
  pc = fmaf(z, pc, SPSIM_QUAD_C2);
  pc = fmaf(z, pc, SPSIM_QUAD_C1);
  pc = fmaf(z, pc, SPSIM_QUAD_C0);
  s = y * ps;
  c = pc;
}

// sin(2 pi y), cos(2 pi y) for |y| <= 5/16 cycle (half-cycle reduction plus
// the phase cross term): the wider-range pair from gen_sincos_poly.py.
__device__ __forceinline__ void sincos_half_poly(float y, float &s, float &c) {
  const float z = y * y;
  float ps = fmaf(z, SPSIM_HALF_S4, SPSIM_HALF_S3);
  ps = fmaf(z, ps, SPSIM_HALF_S2);
  ps = fmaf(z, ps, SPSIM_HALF_S1);
  ps = fmaf(z, ps, SPSIM_HALF_S0);
  float pc = fmaf(z, SPSIM_HALF_C5, SPSIM_HALF_C4);
  pc = fmaf(z, pc, SPSIM_HALF_C3);
  pc = fmaf(z, pc, SPSIM_HALF_C2);
  pc = fmaf(z, pc, SPSIM_HALF_C1);
  pc = fmaf(z, pc, SPSIM_HALF_C0);
  s = y * ps;
  c = pc;
}

// packed f32x2 arithmetic (sm_100): two lanes' worth of FP32 per instruction
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }

// sin(2 pi y), cos(2 pi y) of two phases |y| <= 1/4 cycle (the DHALF pair)
__device__ __forceinline__ void sincos_dhalf_poly2(float2 y, float2 &S, float2 &C) {
  const float2 z = mul2(y, y);
  float2 ps = fma2(z, f2(SPSIM_DHALF_S4), f2(SPSIM_DHALF_S3));
  ps = fma2(z, ps, f2(SPSIM_DHALF_S2));
  ps = fma2(z, ps, f2(SPSIM_DHALF_S1));
  ps = fma2(z, ps, f2(SPSIM_DHALF_S0));
  float2 pc = fma2(z, f2(SPSIM_DHALF_C4), f2(SPSIM_DHALF_C3));
  pc = fma2(z, pc, f2(SPSIM_DHALF_C2));
  pc = fma2(z, pc, f2(SPSIM_DHALF_C1));
  pc = fma2(z, pc, f2(SPSIM_DHALF_C0));
  S = mul2(y, ps);
  C = pc;
}

// the NARROW pair (|y| <= 0.32 cycle) on two phases
__device__ __forceinline__ void sincos_narrow_poly2(float2 y, float2 &S, float2 &C) {
  const float2 z = mul2(y, y);
  float2 ps = fma2(z, f2(SPSIM_NARROW_S4), f2(SPSIM_NARROW_S3));
  ps = fma2(z, ps, f2(SPSIM_NARROW_S2));
  ps = fma2(z, ps, f2(SPSIM_NARROW_S1));
  ps = fma2(z, ps, f2(SPSIM_NARROW_S0));
  float2 pc = fma2(z, f2(SPSIM_NARROW_C5), f2(SPSIM_NARROW_C4));
  pc = fma2(z, pc, f2(SPSIM_NARROW_C3));
  pc = fma2(z, pc, f2(SPSIM_NARROW_C2));
  pc = fma2(z, pc, f2(SPSIM_NARROW_C1));
  pc = fma2(z, pc, f2(SPSIM_NARROW_C0));
  S = mul2(y, ps);
  C = pc;
}

// the WIDER pair (|y| <= 0.41 cycle) on two phases
__device__ __forceinline__ void sincos_wider_poly2(float2 y, float2 &S, float2 &C) {
  const float2 z = mul2(y, y);
  float2 ps = fma2(z, f2(SPSIM_WIDER_S5), f2(SPSIM_WIDER_S4));
  ps = fma2(z, ps, f2(SPSIM_WIDER_S3));
  ps = fma2(z, ps, f2(SPSIM_WIDER_S2));
  ps = fma2(z, ps, f2(SPSIM_WIDER_S1));
  ps = fma2(z, ps, f2(SPSIM_WIDER_S0));
  float2 pc = fma2(z, f2(SPSIM_WIDER_C5), f2(SPSIM_WIDER_C4));
  pc = fma2(z, pc, f2(SPSIM_WIDER_C3));
  pc = fma2(z, pc, f2(SPSIM_WIDER_C2));
  pc = fma2(z, pc, f2(SPSIM_WIDER_C1));
  pc = fma2(z, pc, f2(SPSIM_WIDER_C0));
  S = mul2(y, ps);
  C = pc;
}

// (-1)^k w for an integer k whose bit 0 sits in bit 0 of kbits: one integer
// multiply-add, w_bits + kbits * 2^31 (adding 2^31 flips the sign bit).  The
// multiplier comes in as a register (m31 = 2^31, a kernel argument) so the
// operation stays a single multiply-add on the FMA pipe instead of a shift and
// a logic op.
__device__ __forceinline__ float sign_by_parity(float w, uint32_t kbits, uint32_t m31) {
  uint32_t r;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(kbits), "r"(m31), "r"(__float_as_uint(w)));
  return __uint_as_float(r);
}

// The same sign as a shift and a logic op on the ALU pipe, for the
// polynomial-only neighbour-quad and neighbour-pair kernels, whose FMA pipe
// binds: on 50,000 atoms x 1024^2 0.3 % (quads) and 0.9 % (pairs) faster, on
// 5,000 atoms x 512^2 x 256 orientations with per-atom B factors (a sign per
// pixel) 3.8 % faster.  The split-pipe quads, the FP64-phase kernel and the
// adjoint keep the multiply-add (0.4 %, 1.5 % and 3 % slower with the shift).
__device__ __forceinline__ float sign_by_parity_alu(float w, uint32_t kbits) {
  return __uint_as_float(__float_as_uint(w) ^ (kbits << 31));
}

// ---------------------------------------------------------------------------
// Fixed-point phase word.  While |s q.(r - c)| < 2^19, the FP64 sum
//   t = s q.(r - c) + base,  base = 1.5 * 2^20 (+ 1/2)
// lies in [2^20, 2^21), where the ulp is 2^-32: the low 32 bits of t's
// mantissa hold frac(s q.r + base) * 2^32 (as rounded by the three FMAs,
// error <= 3 * 2^-33 of a cycle) and bit 0 of the high word holds the parity
// of floor(s q.r + base) (1.5 * 2^20 is even).  The phase and its reduction
// thus cost three DFMA instead of six, and the reduced phase reaches FP32
// through one integer conversion.
constexpr double PHASE_WORD_BASE = 1572864.0;       // 1.5 * 2^20
constexpr double PHASE_WORD_BASE_HALF = 1572864.5;  // 1.5 * 2^20 + 1/2

__device__ __forceinline__ double phase_word(double qx, double qy, double qz, double rx, double ry, double rz,
                                             double base) {
  double t = fma(qx, rx, base);
  t = fma(qy, ry, t);
  return fma(qz, rz, t);
}

// POLY (s = 2, base 1.5 * 2^20 + 1/2): with u = k/2 + y, k = rint(2u), the low
// word is (2y + 1/2) 2^32; flipping its bit 31 gives 2y 2^32 as a signed
// integer, and bit 0 of the high word is k mod 2.  The flip is a logic op:
// the logic pipe is nearly idle in these kernels, where an integer add or
// multiply-add would take FMA-pipe slots (measured slower on B200).
// MUFU (s = 1, base 1.5 * 2^20): the low word as a signed integer is
// (u - rint(u)) 2^32 (whole-cycle reduction; no sign).
template <int MODE>
__device__ __forceinline__ void reduce_phase_word(double t, float &yw, uint32_t &kbits) {
  const int lo = __double2loint(t);
  if (MODE == PREC_MODE_POLY) {
    yw = __int2float_rn(lo ^ (int)0x80000000);
    kbits = (uint32_t)__double2hiint(t);
  } else {
    yw = __int2float_rn(lo);
    kbits = 0;
  }
}

// reduce_phase_word's integer units -> cycles, and -> the kernels' sin/cos argument
template <int MODE>
__device__ __forceinline__ constexpr float word_to_cycles() {
  return MODE == PREC_MODE_POLY ? 0x1p-33f : 0x1p-32f;
}
template <int MODE>
__device__ __forceinline__ constexpr float word_to_phase() {
  return MODE == PREC_MODE_POLY ? 0x1p-33f : 6.28318530717958648f * 0x1p-32f;
}

// 2^x with the XU pipe's approximation (PTX ex2.approx.ftz.f32, relative
// error ~2^-22; results below 2^-126 flush to zero): the per-atom B-factor
// weight exp(-B s^2) of one term, where the library exp2f spends extra FMA-pipe
// instructions on full-range accuracy that a weight in (0, 1] does not need.
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// log2(x) by the XU pipe's approximation (PTX lg2.approx.ftz.f32; -inf at 0)
__device__ __forceinline__ float lg2_approx(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Packed Fast2Sum: the block sums b of two pixels into their float-float
// sums (hi, lo); s - hi and b - z as FMAs with -1, so every step stays packed.
__device__ __forceinline__ void ff_accumulate2(float2 &hi, float2 &lo, float2 b) {
  const float2 s = add2(hi, b);
  const float2 z = fma2(hi, f2(-1.0f), s);
  lo = add2(lo, fma2(z, f2(-1.0f), b));
  hi = s;
}

// Fast2Sum-style float-float accumulation of a block sum b into (hi, lo).
__device__ __forceinline__ void ff_accumulate(float &hi, float &lo, float b) {
  const float s = hi + b;
  const float z = s - hi;
  lo += b - z;
  hi = s;
}

}  // namespace spsim
