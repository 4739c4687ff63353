// Adjoint of I = |F|^2 through the structure factor: given g_p = dL/dI_p,
//   dL/dr_j   = 4 pi w_j     sum_p g_p f_e(p) E_pj q_p Im(conj(A_p) e^{-2 pi i u_pj})
//   dL/docc_j = 2 wbase_j    sum_p g_p f_e(p) E_pj     Re(conj(A_p) e^{-2 pi i u_pj})
//   dL/dB_j   = -2 w_j       sum_p g_p f_e(p) E_pj s_p^2 Re(...)
// with A_p = e^{+2 pi i q_p.c} F_p the centred amplitude, u_pj = q_p.(r_j - c),
// E_pj = exp(-B_j s_p^2) (1 without per-atom B) and s^2 = (|q| 1e-10)^2 / 4.
// Phases are recomputed with the forward's arithmetic (compensated FP32 or the
// FP64-phase form); nothing of size atoms x pixels is stored.  One CTA owns a
// block of atoms (registers; one element, or in the FP64-phase adjoint up to
// two element segments) and streams a range of pixel records through shared
// memory.
#include "adjoint_kernels.cuh"

namespace spsim {

// pixel record: 4 x float4
//   {qhx, qhy, qhz, qx} {qy, qz, qlx, qly} {qlz, hr, hi, s2} {s2n, 0, 0, 0}
constexpr int ADJ_PIX_TILE = 256;

// One pixel of the adjoint: q (rotated, FP64), (hr, hi) = g_p f_e(p) A_p with
// the centred amplitude A_p = e^{+2 pi i q.c} F_p, and s^2 = (|q| 1e-10)^2 / 4.
__device__ __forceinline__ void adj_pixel(const AdjParams &prm, int elem, long long gp, double q[3], double &hr,
                                          double &hi, double &s2) {
  const int pat = (int)(gp / prm.npix);
  const long long p = gp - (long long)pat * prm.npix;
  double a, b, c;
  if (prm.hkl) {
    a = prm.hkl[3 * p];
    b = prm.hkl[3 * p + 1];
    c = prm.hkl[3 * p + 2];
  } else {
    a = prm.q64[3 * p];
    b = prm.q64[3 * p + 1];
    c = prm.q64[3 * p + 2];
  }
  if (prm.rot) {
    const double *R = prm.rot + 9 * pat;
    q[0] = R[0] * a + R[1] * b + R[2] * c;
    q[1] = R[3] * a + R[4] * b + R[5] * c;
    q[2] = R[6] * a + R[7] * b + R[8] * c;
  } else {
    q[0] = a;
    q[1] = b;
    q[2] = c;
  }
  // centred amplitude A = e^{+2 pi i q.c} F
  double t = q[0] * prm.cx + q[1] * prm.cy + q[2] * prm.cz;
  t -= rint(t);
  double sn, cs;
  sincospi(2.0 * t, &sn, &cs);
  const float2 F = prm.F[gp];
  const double ar = F.x * cs - F.y * sn;
  const double ai = F.x * sn + F.y * cs;
  const double h = (double)prm.G[gp] * prm.ff[(long long)elem * prm.npix + p];
  hr = h * ar;
  hi = h * ai;
  s2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) * 1e-20 * 0.25;
}

template <int MODE>
__device__ __forceinline__ void adj_sincos(const float4 a0, const float4 a1, const float4 p0, const float4 p1,
                                           const float4 p2, float &S, float &C) {
  float u = p0.x * a0.x;
  u = fmaf(p0.y, a0.y, u);
  u = fmaf(p0.z, a0.z, u);
  float c = p0.w * a1.x;
  c = fmaf(p1.x, a1.y, c);
  c = fmaf(p1.y, a1.z, c);
  c = fmaf(p1.z, a0.x, c);
  c = fmaf(p1.w, a0.y, c);
  c = fmaf(p2.x, a0.z, c);
  if (MODE == 0) {
    const float t = fmaf(u, 4.0f, RINT_MAGIC);
    const float kf = t - RINT_MAGIC;
    const float y = fmaf(kf, -0.25f, u) + c;
    const int ki = __float_as_int(t);
    float s, co;
    sincos_quad_poly(y, s, co);
    const bool odd = (ki & 1) != 0;
    const float ca = odd ? s : co;
    const float sa = odd ? co : s;
    C = __uint_as_float(__float_as_uint(ca) ^ (((unsigned)(ki + 1) << 30) & 0x80000000u));
    S = __uint_as_float(__float_as_uint(sa) ^ (((unsigned)ki << 30) & 0x80000000u));
  } else {
    const float t = u + RINT_MAGIC;
    const float kf = t - RINT_MAGIC;
    const float y = (u - kf) + c;
    __sincosf(y * 6.28318530717958648f, &S, &C);
  }
}

template <int MODE, int NT, int A, bool PERB>
__global__ void __launch_bounds__(NT) adj_kernel(AdjParams prm) {
  __shared__ __align__(16) float4 pix[ADJ_PIX_TILE * 4];
  const int tid = threadIdx.x;
  const AdjItem item = prm.items[blockIdx.x];
  const AdjBlock blk = prm.blocks[item.block];

  float4 a0[A], a1[A];
  int aidx[A];
#pragma unroll
  for (int k = 0; k < A; ++k) {
    aidx[k] = blk.atom_begin + tid + k * NT;
    if (aidx[k] < blk.atom_end) {
      a0[k] = prm.atoms[2 * aidx[k]];
      a1[k] = prm.atoms[2 * aidx[k] + 1];
    } else {
      a0[k] = make_float4(0, 0, 0, 0);
      a1[k] = make_float4(0, 0, 0, 0);
    }
  }
  double gx[A], gy[A], gz[A], go[A], gb[A];
#pragma unroll
  for (int k = 0; k < A; ++k) gx[k] = gy[k] = gz[k] = go[k] = gb[k] = 0.0;

  for (long long base = item.pix_begin; base < item.pix_end; base += ADJ_PIX_TILE) {
    const int n = (int)min((long long)ADJ_PIX_TILE, item.pix_end - base);
    __syncthreads();
    for (int i = tid; i < ADJ_PIX_TILE; i += NT) {
      float4 r0 = make_float4(0, 0, 0, 0), r1 = r0, r2 = r0, r3 = r0;
      if (i < n) {
        const long long gp = base + i;
        double q[3], hr, hi, s2;
        adj_pixel(prm, blk.elem, gp, q, hr, hi, s2);
        const double hx = (double)rintf((float)q[0] * prm.inv_dq) * prm.dq;
        const double hy = (double)rintf((float)q[1] * prm.inv_dq) * prm.dq;
        const double hz = (double)rintf((float)q[2] * prm.inv_dq) * prm.dq;
        r0 = make_float4((float)hx, (float)hy, (float)hz, (float)q[0]);
        r1 = make_float4((float)q[1], (float)q[2], (float)(q[0] - hx), (float)(q[1] - hy));
        r2 = make_float4((float)(q[2] - hz), (float)hr, (float)hi, (float)s2);
        r3 = make_float4((float)(-s2 * 1.4426950408889634), 0, 0, 0);
      }
      pix[4 * i] = r0;
      pix[4 * i + 1] = r1;
      pix[4 * i + 2] = r2;
      pix[4 * i + 3] = r3;
    }
    __syncthreads();
    float fx[A], fy[A], fz[A], fo[A], fb[A];
#pragma unroll
    for (int k = 0; k < A; ++k) fx[k] = fy[k] = fz[k] = fo[k] = fb[k] = 0.0f;
    for (int i = 0; i < n; ++i) {
      const float4 p0 = pix[4 * i], p1 = pix[4 * i + 1], p2 = pix[4 * i + 2];
      float s2n = 0.0f;
      if (PERB) s2n = pix[4 * i + 3].x;
#pragma unroll
      for (int k = 0; k < A; ++k) {
        float S, C;
        adj_sincos<MODE>(a0[k], a1[k], p0, p1, p2, S, C);
        // H conj(A) e^{-2 pi i u} = (hr C - hi S) - i (hr S + hi C)
        float zr = p2.y * C - p2.z * S;
        float zi = -(p2.y * S + p2.z * C);
        if (PERB) {
          const float E = ex2_approx(a1[k].w * s2n);
          zr *= E;
          zi *= E;
        }
        fx[k] = fmaf(zi, p0.w, fx[k]);
        fy[k] = fmaf(zi, p1.x, fy[k]);
        fz[k] = fmaf(zi, p1.y, fz[k]);
        fo[k] += zr;
        fb[k] = fmaf(zr, p2.w, fb[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < A; ++k) {
      gx[k] += fx[k];
      gy[k] += fy[k];
      gz[k] += fz[k];
      go[k] += fo[k];
      gb[k] += fb[k];
    }
  }
#pragma unroll
  for (int k = 0; k < A; ++k) {
    if (aidx[k] >= blk.atom_end) continue;
    const int src = prm.perm[aidx[k]];
    if (src < 0) continue;
    const double w = a0[k].w, wb = prm.wbase[aidx[k]];
    const double kp = 4.0 * 3.14159265358979323846 * w;
    atomicAdd(&prm.dpos[3 * src], kp * gx[k]);
    atomicAdd(&prm.dpos[3 * src + 1], kp * gy[k]);
    atomicAdd(&prm.dpos[3 * src + 2], kp * gz[k]);
    if (prm.docc) atomicAdd(&prm.docc[src], 2.0 * wb * go[k]);
    if (prm.dB) atomicAdd(&prm.dB[src], -2.0 * w * gb[k]);
  }
}

// FP64-phase adjoint: the phase u = q.(r - c) and its half-cycle reduction in
// FP64 (as in the FP64-phase forward), sin/cos and the five gradient sums in
// packed f32x2 over pairs of atoms.  Each thread holds A consecutive atoms
// (A/2 pairs, one element) in registers; a CTA's block of atoms spans at most
// two element segments, and the CTA streams the pixel records of each of its
// elements through shared memory.  With the
// fixed-point phase word (FIXW), H = |H| e^{i phi} enters as a phase and a
// magnitude, so the polynomial's cos / sin are the products z themselves:
//   pq[2i]   = {2 qx, 2 qy}  pq[2i+1] = {2 qz, word constant + phi / pi}   (FP64)
//   pf[2i]   = {|H| qx, |H| qy, |H| qz, |H|}  pf[2i+1] = {|H| s2, s2n, 0, 0}   (FP32)
// and otherwise (FP64 rounding reduction, phases beyond 2^17 cycles)
//   pq[2i]   = {qx, qy}  pq[2i+1] = {qz, 0}
//   pf[2i]   = {qx, qy, qz, hr}  pf[2i+1] = {hi, s2, s2n, 0}
// with z = H conj(A) e^{-2 pi i u} formed per term.  The sign (-1)^k of the
// half-cycle reduction is applied to the two products with one integer
// multiply-add each.
template <int NT, int A, bool PERB, bool FIXW>
__global__ void __launch_bounds__(NT) adj_dphase_kernel(AdjParams prm, uint32_t m31) {
  static_assert(A % 2 == 0, "atoms per thread must be even");
  constexpr int NP = A / 2;
  // pixel records of the block's (at most two) elements
  __shared__ __align__(16) double2 pq_all[2][ADJ_PIX_TILE * 2];
  __shared__ __align__(16) float4 pf_all[2][ADJ_PIX_TILE * 2];
  const int tid = threadIdx.x;
  const AdjItem item = prm.items[blockIdx.x];
  const AdjBlock blk = prm.blocks[item.block];
  const double M52 = 6755399441055744.0;  // 1.5 * 2^52
  // this thread's A consecutive atoms lie in one element segment (segments are
  // padded to multiples of 8, blocks start and split on multiples of A)
  const int a_first = blk.atom_begin + A * tid;
  const int slot = (blk.elem2 >= 0 && a_first >= blk.split) ? 1 : 0;
  const int nslot = blk.elem2 >= 0 ? 2 : 1;
  const double2 *__restrict__ pq = pq_all[slot];
  const float4 *__restrict__ pf = pf_all[slot];

  double rx[A], ry[A], rz[A];
  float bfac[A];
  int aidx[A];
#pragma unroll
  for (int k = 0; k < A; ++k) {
    aidx[k] = a_first + k;
    rx[k] = ry[k] = rz[k] = 0.0;
    bfac[k] = 0.0f;
    if (aidx[k] < blk.atom_end) {
      const AtomD a = prm.atomsd[aidx[k]];
      rx[k] = a.x;
      ry[k] = a.y;
      rz[k] = a.z;
      bfac[k] = a.b;
    }
  }
  double gx[A], gy[A], gz[A], go[A], gb[A];
#pragma unroll
  for (int k = 0; k < A; ++k) gx[k] = gy[k] = gz[k] = go[k] = gb[k] = 0.0;

  for (long long base = item.pix_begin; base < item.pix_end; base += ADJ_PIX_TILE) {
    const int n = (int)min((long long)ADJ_PIX_TILE, item.pix_end - base);
    __syncthreads();
    for (int c = tid; c < ADJ_PIX_TILE * nslot; c += NT) {
      const int i = c % ADJ_PIX_TILE, sl = c / ADJ_PIX_TILE;
      double2 *__restrict__ pq = pq_all[sl];
      float4 *__restrict__ pf = pf_all[sl];
      double q[3] = {0.0, 0.0, 0.0}, hr = 0.0, hi = 0.0, s2 = 0.0;
      if (i < n) adj_pixel(prm, sl ? blk.elem2 : blk.elem, base + i, q, hr, hi, s2);
      if (FIXW) {
        // H = |H| e^{i phi}: H e^{2 pi i u} = |H| e^{2 pi i (u + phi / 2 pi)}, so the
        // pixel's phase goes into the phase word's constant (2 q and 2 u + phi / pi
        // + 1/2 + 1.5 * 2^20, the half-cycle reduction) and |H| into its factors
        const double mag = hypot(hr, hi);
        const double phi = mag > 0.0 ? atan2(hi, hr) : 0.0;
        pq[2 * i] = make_double2(2.0 * q[0], 2.0 * q[1]);
        pq[2 * i + 1] = make_double2(2.0 * q[2], PHASE_WORD_BASE_HALF + phi * 0.31830988618379067);
        pf[2 * i] = make_float4((float)(mag * q[0]), (float)(mag * q[1]), (float)(mag * q[2]), (float)mag);
        pf[2 * i + 1] = make_float4((float)(mag * s2), (float)(-s2 * 1.4426950408889634), 0.0f, 0.0f);
      } else {
        pq[2 * i] = make_double2(q[0], q[1]);
        pq[2 * i + 1] = make_double2(q[2], 0.0);
        pf[2 * i] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)hr);
        pf[2 * i + 1] = make_float4((float)hi, (float)s2, (float)(-s2 * 1.4426950408889634), 0.0f);
      }
    }
    __syncthreads();
    // sums of z_i = -Im part (so that dL/dr = -4 pi w sum z_i q) and z_r
    float2 fx[NP], fy[NP], fz[NP], fo[NP], fb[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) fx[j] = fy[j] = fz[j] = fo[j] = fb[j] = make_float2(0.f, 0.f);
    // four pixels per iteration: independent chains for the scheduler (each
    // thread's two atom pairs alone left it waiting on fixed-latency results)
#pragma unroll 4
    for (int i = 0; i < n; ++i) {
      const double2 qa = pq[2 * i], qb = pq[2 * i + 1];
      const float4 f0 = pf[2 * i], f1 = pf[2 * i + 1];
      if (FIXW) {
        // cos / sin of 2 pi (u + phi / 2 pi), signed by the half-cycle parity, are
        // z_r / |H| and -Im / |H|: the five sums take them with |H|-scaled factors
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          float y[2];
          uint32_t kb[2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int k = 2 * j + h;
            const double t = phase_word(qa.x, qa.y, qb.x, rx[k], ry[k], rz[k], qb.y);
            reduce_phase_word<PREC_MODE_POLY>(t, y[h], kb[h]);
          }
          float2 S, C;
          if (j & 1) {  // every other atom pair on MUFU sin/cos (the XU pipe)
            const float2 x = mul2(make_float2(y[0], y[1]), f2(6.28318530717958648f * word_to_cycles<PREC_MODE_POLY>()));
            __sincosf(x.x, &S.x, &C.x);
            __sincosf(x.y, &S.y, &C.y);
          } else {
            sincos_dhalf_poly2(mul2(make_float2(y[0], y[1]), f2(word_to_cycles<PREC_MODE_POLY>())), S, C);
          }
          float2 zr, zn;
          if (PERB) {
            // the sign once, on the B-factor weight E, which then scales both
            const float2 E = make_float2(sign_by_parity(ex2_approx(bfac[2 * j] * f1.y), kb[0], m31),
                                         sign_by_parity(ex2_approx(bfac[2 * j + 1] * f1.y), kb[1], m31));
            zr = mul2(C, E);
            zn = mul2(S, E);
          } else {
            zr = make_float2(sign_by_parity(C.x, kb[0], m31), sign_by_parity(C.y, kb[1], m31));
            zn = make_float2(sign_by_parity(S.x, kb[0], m31), sign_by_parity(S.y, kb[1], m31));
          }
          fx[j] = fma2(zn, f2(f0.x), fx[j]);
          fy[j] = fma2(zn, f2(f0.y), fy[j]);
          fz[j] = fma2(zn, f2(f0.z), fz[j]);
          fo[j] = fma2(zr, f2(f0.w), fo[j]);
          fb[j] = fma2(zr, f2(f1.x), fb[j]);
        }
        continue;
      }
      const float2 hr = f2(f0.w), nhi = f2(-f1.x), hi = f2(f1.x);
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        float y[2];
        uint32_t kb[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int k = 2 * j + h;
          {
            double u = qa.x * rx[k];
            u = fma(qa.y, ry[k], u);
            u = fma(qb.x, rz[k], u);
            const double t = fma(u, 2.0, M52);
            y[h] = __double2float_rn(fma(t - M52, -0.5, u));
            kb[h] = (uint32_t)__double2loint(t);
          }
        }
        float2 S, C;
        if (j & 1) {  // every other atom pair on MUFU sin/cos (the XU pipe)
          const float2 x = mul2(make_float2(y[0], y[1]), f2(6.28318530717958648f));
          __sincosf(x.x, &S.x, &C.x);
          __sincosf(x.y, &S.y, &C.y);
        } else {
          sincos_dhalf_poly2(make_float2(y[0], y[1]), S, C);
        }
        // H conj(A) e^{-2 pi i u} = (hr C - hi S) - i (hr S + hi C), times (-1)^k
        float2 zr = fma2(nhi, S, mul2(hr, C));
        float2 zn = fma2(hi, C, mul2(hr, S));  // = -Im
        zr = make_float2(sign_by_parity(zr.x, kb[0], m31), sign_by_parity(zr.y, kb[1], m31));
        zn = make_float2(sign_by_parity(zn.x, kb[0], m31), sign_by_parity(zn.y, kb[1], m31));
        if (PERB) {
          const float2 E = make_float2(ex2_approx(bfac[2 * j] * f1.z), ex2_approx(bfac[2 * j + 1] * f1.z));
          zr = mul2(zr, E);
          zn = mul2(zn, E);
        }
        fx[j] = fma2(zn, f2(f0.x), fx[j]);
        fy[j] = fma2(zn, f2(f0.y), fy[j]);
        fz[j] = fma2(zn, f2(f0.z), fz[j]);
        fo[j] = add2(fo[j], zr);
        fb[j] = fma2(zr, f2(f1.y), fb[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      gx[2 * j] -= fx[j].x;
      gx[2 * j + 1] -= fx[j].y;
      gy[2 * j] -= fy[j].x;
      gy[2 * j + 1] -= fy[j].y;
      gz[2 * j] -= fz[j].x;
      gz[2 * j + 1] -= fz[j].y;
      go[2 * j] += fo[j].x;
      go[2 * j + 1] += fo[j].y;
      gb[2 * j] += fb[j].x;
      gb[2 * j + 1] += fb[j].y;
    }
  }
#pragma unroll
  for (int k = 0; k < A; ++k) {
    if (aidx[k] >= blk.atom_end) continue;
    const int src = prm.perm[aidx[k]];
    if (src < 0) continue;
    const double w = prm.atomsd[aidx[k]].w, wb = prm.wbase[aidx[k]];
    const double kp = 4.0 * 3.14159265358979323846 * w;
    atomicAdd(&prm.dpos[3 * src], kp * gx[k]);
    atomicAdd(&prm.dpos[3 * src + 1], kp * gy[k]);
    atomicAdd(&prm.dpos[3 * src + 2], kp * gz[k]);
    if (prm.docc) atomicAdd(&prm.docc[src], 2.0 * wb * go[k]);
    if (prm.dB) atomicAdd(&prm.dB[src], -2.0 * w * gb[k]);
  }
}

// plain FP64 adjoint: same decomposition, FP64 phase and sincos
template <int NT>
__global__ void __launch_bounds__(NT) adj_f64_kernel(AdjParams prm) {
  const int tid = threadIdx.x;
  const AdjItem item = prm.items[blockIdx.x];
  const AdjBlock blk = prm.blocks[item.block];
  const int j = blk.atom_begin + tid;
  if (j >= blk.atom_end) return;
  const float4 a0 = prm.atoms[2 * j], a1 = prm.atoms[2 * j + 1];
  const double rx = (double)a0.x + a1.x, ry = (double)a0.y + a1.y, rz = (double)a0.z + a1.z;
  double gx = 0, gy = 0, gz = 0, go = 0, gb = 0;
  for (long long gp = item.pix_begin; gp < item.pix_end; ++gp) {
    const int pat = (int)(gp / prm.npix);
    const long long p = gp - (long long)pat * prm.npix;
    double a, b, c, q[3];
    if (prm.hkl) {
      a = prm.hkl[3 * p];
      b = prm.hkl[3 * p + 1];
      c = prm.hkl[3 * p + 2];
    } else {
      a = prm.q64[3 * p];
      b = prm.q64[3 * p + 1];
      c = prm.q64[3 * p + 2];
    }
    if (prm.rot) {
      const double *R = prm.rot + 9 * pat;
      q[0] = R[0] * a + R[1] * b + R[2] * c;
      q[1] = R[3] * a + R[4] * b + R[5] * c;
      q[2] = R[6] * a + R[7] * b + R[8] * c;
    } else {
      q[0] = a;
      q[1] = b;
      q[2] = c;
    }
    double t = q[0] * prm.cx + q[1] * prm.cy + q[2] * prm.cz;
    t -= rint(t);
    double sn, cs;
    sincospi(2.0 * t, &sn, &cs);
    const float2 F = prm.F[gp];
    const double ar = F.x * cs - F.y * sn, ai = F.x * sn + F.y * cs;
    const double h = (double)prm.G[gp] * prm.ff[(long long)blk.elem * prm.npix + p];
    const double s2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) * 1e-20 * 0.25;
    double u = q[0] * rx + q[1] * ry + q[2] * rz;
    u -= rint(u);
    double S, C;
    sincospi(2.0 * u, &S, &C);
    double zr = h * (ar * C - ai * S), zi = -h * (ar * S + ai * C);
    if (prm.per_atom_b) {
      const double E = exp(-(double)a1.w * s2);
      zr *= E;
      zi *= E;
    }
    gx += zi * q[0];
    gy += zi * q[1];
    gz += zi * q[2];
    go += zr;
    gb += zr * s2;
  }
  const int src = prm.perm[j];
  if (src < 0) return;
  const double w = a0.w, wb = prm.wbase[j];
  const double kp = 4.0 * 3.14159265358979323846 * w;
  atomicAdd(&prm.dpos[3 * src], kp * gx);
  atomicAdd(&prm.dpos[3 * src + 1], kp * gy);
  atomicAdd(&prm.dpos[3 * src + 2], kp * gz);
  if (prm.docc) atomicAdd(&prm.docc[src], 2.0 * wb * go);
  if (prm.dB) atomicAdd(&prm.dB[src], -2.0 * w * gb);
}

int adjoint_occupancy(int precision_mode, bool perb) {
  int n = 0;
  if (precision_mode == 2)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, adj_f64_kernel<ADJ_THREADS>, ADJ_THREADS, 0);
  else if (precision_mode == 3 || precision_mode == 4) {
    const bool fw = precision_mode == 4;
    if (perb)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &n, fw ? adj_dphase_kernel<ADJ_THREADS, ADJ_DPHASE_ATOMS_PER_THREAD, true, true>
                 : adj_dphase_kernel<ADJ_THREADS, ADJ_DPHASE_ATOMS_PER_THREAD, true, false>,
          ADJ_THREADS, 0);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &n, fw ? adj_dphase_kernel<ADJ_THREADS, ADJ_DPHASE_ATOMS_PER_THREAD, false, true>
                 : adj_dphase_kernel<ADJ_THREADS, ADJ_DPHASE_ATOMS_PER_THREAD, false, false>,
          ADJ_THREADS, 0);
  } else if (precision_mode == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &n, perb ? adj_kernel<0, ADJ_THREADS, ADJ_ATOMS_PER_THREAD, true> : adj_kernel<0, ADJ_THREADS, ADJ_ATOMS_PER_THREAD, false>,
        ADJ_THREADS, 0);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &n, perb ? adj_kernel<1, ADJ_THREADS, ADJ_ATOMS_PER_THREAD, true> : adj_kernel<1, ADJ_THREADS, ADJ_ATOMS_PER_THREAD, false>,
        ADJ_THREADS, 0);
  }
  return n;
}

cudaError_t launch_adjoint(int precision_mode, const AdjParams &prm, int n_items, cudaStream_t st) {
  if (n_items <= 0) return cudaSuccess;
  if (precision_mode == 2) {
    adj_f64_kernel<ADJ_THREADS><<<n_items, ADJ_THREADS, 0, st>>>(prm);
  } else if (precision_mode == 3) {
    if (prm.per_atom_b)
      adj_dphase_kernel<ADJ_THREADS, ADJ_DPHASE_ATOMS_PER_THREAD, true, false><<<n_items, ADJ_THREADS, 0, st>>>(
          prm, 0x80000000u);
    else
      adj_dphase_kernel<ADJ_THREADS, ADJ_DPHASE_ATOMS_PER_THREAD, false, false><<<n_items, ADJ_THREADS, 0, st>>>(
          prm, 0x80000000u);
  } else if (precision_mode == 4) {
    if (prm.per_atom_b)
      adj_dphase_kernel<ADJ_THREADS, ADJ_DPHASE_ATOMS_PER_THREAD, true, true><<<n_items, ADJ_THREADS, 0, st>>>(
          prm, 0x80000000u);
    else
      adj_dphase_kernel<ADJ_THREADS, ADJ_DPHASE_ATOMS_PER_THREAD, false, true><<<n_items, ADJ_THREADS, 0, st>>>(
          prm, 0x80000000u);
  } else if (precision_mode == 0) {
    if (prm.per_atom_b)
      adj_kernel<0, ADJ_THREADS, ADJ_ATOMS_PER_THREAD, true><<<n_items, ADJ_THREADS, 0, st>>>(prm);
    else
      adj_kernel<0, ADJ_THREADS, ADJ_ATOMS_PER_THREAD, false><<<n_items, ADJ_THREADS, 0, st>>>(prm);
  } else {
    if (prm.per_atom_b)
      adj_kernel<1, ADJ_THREADS, ADJ_ATOMS_PER_THREAD, true><<<n_items, ADJ_THREADS, 0, st>>>(prm);
    else
      adj_kernel<1, ADJ_THREADS, ADJ_ATOMS_PER_THREAD, false><<<n_items, ADJ_THREADS, 0, st>>>(prm);
  }
  return cudaGetLastError();
}

}  // namespace spsim
