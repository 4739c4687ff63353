// Structure-factor kernels for sm_100a.
//
//   ff_table_kernel      f_e(|q|) per pixel per element, FP64 (src/diffraction.c:183-193)
//   sf_f32_kernel        compensated-FP32 forward, persistent over cost-sorted work items;
//                        atom tiles staged in shared memory by 1-D bulk copies on an
//                        mbarrier ring and read as warp-broadcasts
//   sf_f64_kernel        plain FP64 per-pixel forward (the precision/speed baseline)
//   sf_finalize_kernel   centre phase, complex64 F and |F|^2
//   ewald_kernel         HKL list of a flat/spherical detector (src/diffraction.c:237-297)
//   atoms_update_kernel  refinement: device positions -> atom records
#include "sf_kernels.cuh"

#include <cstdio>
#include <cstring>

namespace spsim {

// Minimum resident CTAs per SM requested of the compiler for the structure-
// factor kernels.  The FMA-polynomial kernels run fastest with every register
// they can use (1: the 128 x 8 neighbour-pair kernel takes 188 registers
// without spilling, where the compiler's own choice was 128 with spills, and
// runs 6 % faster); the MUFU kernels, bound by the XU pipe, keep the
// compiler's own choice (0), which leaves more warps per SM (asking for 1
// gave them up to 252 registers and cost 5 %).
__host__ __device__ constexpr int sf_min_blocks(int mode) { return mode == PREC_MODE_POLY ? 1 : 0; }

// Bounded waits on the atom-tile ring.  A wait that runs out sets the error
// word, drains (bounded) the copies this CTA still has in flight and returns.
// g_copy_stall is the test hook behind spsim_b200_debug_stall_first_copy:
// while it is set, each CTA arms the barrier of its first tile without issuing
// that tile's copy (a barrier that nothing completes) and its waits give up
// after kStallWaitCycles, so the exit path runs in milliseconds and without a
// fault; read once per CTA at launch.
__device__ int g_copy_stall = 0;
constexpr long long kWaitCyclesDefault = 4000000000LL;  // ~2 s at 2 GHz
constexpr long long kStallWaitCycles = 20000000LL;      // ~10 ms

cudaError_t set_copy_stall(int on) {
  const int v = on ? 1 : 0;
  return cudaMemcpyToSymbol(g_copy_stall, &v, sizeof(int));
}

// ---------------------------------------------------------------------------
// form factors

__global__ void ff_table_kernel(const float *__restrict__ hkl, const double *__restrict__ q64, long long npix,
                                int n_elem, const float *__restrict__ coeffs, double B, int delta_atoms,
                                double *__restrict__ ff) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int e = blockIdx.y;
  if (p >= npix || e >= n_elem) return;
  double qx, qy, qz;
  if (hkl) {
    qx = hkl[3 * p];
    qy = hkl[3 * p + 1];
    qz = hkl[3 * p + 2];
  } else {
    qx = q64[3 * p];
    qy = q64[3 * p + 1];
    qz = q64[3 * p + 2];
  }
  double f = 1.0;
  if (!delta_atoms) {
    const double qlen = sqrt(qx * qx + qy * qy + qz * qz);
    const double d = qlen * 1e-10;
    const double s2 = d * d * 0.25;
    const float *c = coeffs + 9 * e;
    f = 0.0;
    for (int i = 0; i < 4; ++i) f += (double)c[i] * exp(-((double)c[i + 4] + B) * s2);
    f += (double)c[8] * exp(-B * s2);
  }
  ff[(long long)e * npix + p] = f;
}

// ---------------------------------------------------------------------------
// pixel set-up shared by the kernels: q (FP64) of pixel p, rotated

__device__ __forceinline__ void load_q(const SfPattern &pt, long long p, double q[3]) {
  double a, b, c;
  if (pt.hkl) {
    a = pt.hkl[3 * p];
    b = pt.hkl[3 * p + 1];
    c = pt.hkl[3 * p + 2];
  } else {
    a = pt.q64[3 * p];
    b = pt.q64[3 * p + 1];
    c = pt.q64[3 * p + 2];
  }
  if (pt.has_rot) {
    q[0] = pt.rot[0] * a + pt.rot[1] * b + pt.rot[2] * c;
    q[1] = pt.rot[3] * a + pt.rot[4] * b + pt.rot[5] * c;
    q[2] = pt.rot[6] * a + pt.rot[7] * b + pt.rot[8] * c;
  } else {
    q[0] = a;
    q[1] = b;
    q[2] = c;
  }
  q[0] *= pt.qscale;
  q[1] *= pt.qscale;
  q[2] *= pt.qscale;
}

// ---------------------------------------------------------------------------
// compensated FP32 forward

template <int MODE>
__device__ __forceinline__ void sf_term(const float4 a0, const float4 a1, float w, float qhx, float qhy, float qhz,
                                        float qx, float qy, float qz, float qlx, float qly, float qlz, float &bc,
                                        float &bs) {
  // u = Q_hi . R_hi : exact on the dq*dr grid
  float u = qhx * a0.x;
  u = fmaf(qhy, a0.y, u);
  u = fmaf(qhz, a0.z, u);
  // cross term Q . R_lo + Q_lo . R_hi (|c| <= 1/16 cycle, checked on the host)
  float c = qx * a1.x;
  c = fmaf(qy, a1.y, c);
  c = fmaf(qz, a1.z, c);
  c = fmaf(qlx, a0.x, c);
  c = fmaf(qly, a0.y, c);
  c = fmaf(qlz, a0.z, c);
  if (MODE == PREC_MODE_POLY) {
    // half-cycle reduction: u = k/2 + y0 exactly, |y0| <= 1/4; e^{2 pi i u} = (-1)^k e^{2 pi i y}
    const float t = fmaf(u, 2.0f, RINT_MAGIC);
    const float kf = t - RINT_MAGIC;
    const float y = fmaf(kf, -0.5f, u) + c;
    float s, co;
    sincos_half_poly(y, s, co);
    const float ws = __uint_as_float(__float_as_uint(w) ^ (__float_as_uint(t) << 31));
    bc = fmaf(ws, co, bc);  // sum w cos(2 pi u)
    bs = fmaf(ws, s, bs);   // sum w sin(2 pi u)
  } else {
    // whole-cycle reduction, MUFU sin/cos on |x| <= pi (1 + 1/8)
    const float t = u + RINT_MAGIC;
    const float kf = t - RINT_MAGIC;
    const float y = (u - kf) + c;
    float s, co;
    __sincosf(y * 6.28318530717958648f, &s, &co);
    bc = fmaf(w, co, bc);
    bs = fmaf(w, s, bs);
  }
}

template <int MODE, int NT, int P, bool PERB>
__global__ void __launch_bounds__(NT, sf_min_blocks(MODE)) sf_f32_kernel(const SfPattern *__restrict__ pats,
                                                    const WorkItem *__restrict__ items, int n_items,
                                                    int *__restrict__ queue, int *__restrict__ err) {
  __shared__ __align__(128) float4 ring[RING_STAGES][2 * TILE_ATOMS];
  __shared__ __align__(8) uint64_t full_bar[RING_STAGES];
  __shared__ int s_item;

  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < RING_STAGES; ++s) mbar_init(&full_bar[s], 1);
    fence_barrier_init();
  }
  __syncthreads();

  uint32_t g_issue = 0;  // tiles issued by this CTA (meaningful in thread 0)
  uint32_t g_cons = 0;   // tiles consumed by this CTA (uniform)
  const bool stall = g_copy_stall != 0;
  const long long kWaitCycles = stall ? kStallWaitCycles : kWaitCyclesDefault;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(queue, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WorkItem wi = items[it];
    const SfPattern &pt = pats[wi.pattern];
    const long long npix = pt.npix;
    const float dq = pt.dq, inv_dq = pt.inv_dq;
    const float4 *__restrict__ atoms = pt.atoms;
    const TileDesc *__restrict__ tiles = pt.tiles;

    // ---- per-thread pixels
    float qhx[P], qhy[P], qhz[P], qx[P], qy[P], qz[P], qlx[P], qly[P], qlz[P], s2n[P];
    long long pix[P];
#pragma unroll
    for (int i = 0; i < P; ++i) {
      pix[i] = (long long)wi.pixel_tile * (NT * P) + i * NT + tid;
      double q[3] = {0.0, 0.0, 0.0};
      if (pix[i] < npix) load_q(pt, pix[i], q);
      const double hx = (double)rintf((float)q[0] * inv_dq) * dq;
      const double hy = (double)rintf((float)q[1] * inv_dq) * dq;
      const double hz = (double)rintf((float)q[2] * inv_dq) * dq;
      qhx[i] = (float)hx;
      qhy[i] = (float)hy;
      qhz[i] = (float)hz;
      qx[i] = (float)q[0];
      qy[i] = (float)q[1];
      qz[i] = (float)q[2];
      qlx[i] = (float)(q[0] - hx);
      qly[i] = (float)(q[1] - hy);
      qlz[i] = (float)(q[2] - hz);
      // -(|q| 1e-10)^2 / 4 * log2(e): per-atom B factor exponent in base 2
      const double d2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) * 1e-20;
      s2n[i] = (float)(-0.25 * d2 * pt.s2scale * 1.4426950408889634);
    }
    double fre[P], fim[P];
    float shc[P], slc[P], shs[P], sls[P];
#pragma unroll
    for (int i = 0; i < P; ++i) {
      fre[i] = fim[i] = 0.0;
      shc[i] = slc[i] = shs[i] = sls[i] = 0.0f;
    }

    const int k0 = wi.k0, k1 = wi.k1;
    if (tid == 0) {
      for (int k = k0; k < k1 && k < k0 + RING_STAGES; ++k) {
        const TileDesc td = tiles[k];
        const uint32_t st = g_issue % RING_STAGES;
        const uint32_t bytes = (uint32_t)td.count * 32u;
        mbar_arrive_expect_tx(&full_bar[st], bytes);
        if (!(stall && g_issue == 0))  // the stall hook skips the CTA's first copy
          bulk_copy_g2s(&ring[st][0], atoms + 2 * (long long)td.atom_begin, bytes, &full_bar[st]);
        ++g_issue;
      }
    }

    for (int k = k0; k < k1; ++k) {
      const uint32_t st = g_cons % RING_STAGES;
      const uint32_t par = (g_cons / RING_STAGES) & 1u;
      const bool ok = mbar_wait_bounded(&full_bar[st], par, kWaitCycles);
      if (__syncthreads_or(!ok)) {
        // a copy never landed: report, wait (bounded) for copies still in flight, leave
        if (tid == 0) {
          atomicOr(err, 1);
          for (uint32_t g = g_cons; g < g_issue; ++g)
            mbar_wait_bounded(&full_bar[g % RING_STAGES], (g / RING_STAGES) & 1u, kWaitCycles);
        }
        return;
      }
      const TileDesc td = tiles[k];
      const float4 *__restrict__ ta = ring[st];
      for (int a = 0; a < td.count; a += ATOM_GROUP) {
        float bc[P], bs[P];
#pragma unroll
        for (int i = 0; i < P; ++i) bc[i] = bs[i] = 0.0f;
#pragma unroll
        for (int g = 0; g < ATOM_GROUP; ++g) {
          const float4 a0 = ta[2 * (a + g)];
          const float4 a1 = ta[2 * (a + g) + 1];
#pragma unroll
          for (int i = 0; i < P; ++i) {
            const float w = PERB ? a0.w * ex2_approx(a1.w * s2n[i]) : a0.w;
            sf_term<MODE>(a0, a1, w, qhx[i], qhy[i], qhz[i], qx[i], qy[i], qz[i], qlx[i], qly[i], qlz[i], bc[i],
                          bs[i]);
          }
        }
#pragma unroll
        for (int i = 0; i < P; ++i) {
          ff_accumulate(shc[i], slc[i], bc[i]);
          ff_accumulate(shs[i], sls[i], bs[i]);
        }
      }
      if (td.last || k == k1 - 1) {
        const double *__restrict__ ffe = pt.ff + (long long)td.elem * npix;
#pragma unroll
        for (int i = 0; i < P; ++i) {
          const double f = pix[i] < npix ? ffe[pix[i]] : 0.0;
          fre[i] += f * ((double)shc[i] + (double)slc[i]);
          fim[i] -= f * ((double)shs[i] + (double)sls[i]);
          shc[i] = slc[i] = shs[i] = sls[i] = 0.0f;
        }
      }
      __syncthreads();  // every thread is done with stage st
      if (tid == 0 && k + RING_STAGES < k1) {
        const TileDesc tn = tiles[k + RING_STAGES];
        const uint32_t bytes = (uint32_t)tn.count * 32u;
        mbar_arrive_expect_tx(&full_bar[st], bytes);
        bulk_copy_g2s(&ring[st][0], atoms + 2 * (long long)tn.atom_begin, bytes, &full_bar[st]);
        ++g_issue;
      }
      ++g_cons;
    }

#pragma unroll
    for (int i = 0; i < P; ++i) {
      if (pix[i] < npix) {
        atomicAdd(&pt.acc[pix[i]].x, fre[i]);
        atomicAdd(&pt.acc[pix[i]].y, fim[i]);
      }
    }
    __syncthreads();  // s_item is rewritten next round
  }
}

// ---------------------------------------------------------------------------
// compensated FP32 forward on pixel pairs: every FP32 operation of the term is
// a packed f32x2 instruction (two pixels, one issue slot).  Atom records are
// stored duplicated (4 float4 per atom, see SfPattern::atoms2) so each shared
// load yields ready operand pairs.  Element sums are flushed straight into the
// per-thread FP64 slots in shared memory, written once per work item.


template <int MODE, int NT, int P, bool PERB>
__global__ void __launch_bounds__(NT, sf_min_blocks(MODE)) sf_f32x2_kernel(const SfPattern *__restrict__ pats,
                                                      const WorkItem *__restrict__ items, int n_items,
                                                      int *__restrict__ queue, int *__restrict__ err) {
  static_assert(P % 2 == 0, "pixels per thread must be even");
  constexpr int NP = P / 2;
  __shared__ __align__(128) float4 ring[RING_STAGES][4 * TILE_ATOMS];
  __shared__ __align__(16) double2 sacc[P * NT];  // per-thread FP64 pixel sums of the current work item
  __shared__ __align__(8) uint64_t full_bar[RING_STAGES];
  __shared__ int s_item;

  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < RING_STAGES; ++s) mbar_init(&full_bar[s], 1);
    fence_barrier_init();
  }
  __syncthreads();

  uint32_t g_issue = 0, g_cons = 0;
  const bool stall = g_copy_stall != 0;
  const long long kWaitCycles = stall ? kStallWaitCycles : kWaitCyclesDefault;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(queue, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WorkItem wi = items[it];
    const SfPattern &pt = pats[wi.pattern];
    const long long npix = pt.npix;
    const float dq = pt.dq, inv_dq = pt.inv_dq;
    const float4 *__restrict__ atoms2 = pt.atoms2;
    const TileDesc *__restrict__ tiles = pt.tiles;

    float2 qhx[NP], qhy[NP], qhz[NP], qx[NP], qy[NP], qz[NP], qlx[NP], qly[NP], qlz[NP], s2n[NP];
    long long pix[P];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      float v[10][2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long long p = (long long)wi.pixel_tile * (NT * P) + (2 * j + h) * NT + tid;
        pix[2 * j + h] = p;
        double q[3] = {0.0, 0.0, 0.0};
        if (p < npix) load_q(pt, p, q);
        const double hx = (double)rintf((float)q[0] * inv_dq) * dq;
        const double hy = (double)rintf((float)q[1] * inv_dq) * dq;
        const double hz = (double)rintf((float)q[2] * inv_dq) * dq;
        v[0][h] = (float)hx;
        v[1][h] = (float)hy;
        v[2][h] = (float)hz;
        v[3][h] = (float)q[0];
        v[4][h] = (float)q[1];
        v[5][h] = (float)q[2];
        v[6][h] = (float)(q[0] - hx);
        v[7][h] = (float)(q[1] - hy);
        v[8][h] = (float)(q[2] - hz);
        v[9][h] = (float)(-0.25 * (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) * 1e-20 * pt.s2scale * 1.4426950408889634);
      }
      qhx[j] = make_float2(v[0][0], v[0][1]);
      qhy[j] = make_float2(v[1][0], v[1][1]);
      qhz[j] = make_float2(v[2][0], v[2][1]);
      qx[j] = make_float2(v[3][0], v[3][1]);
      qy[j] = make_float2(v[4][0], v[4][1]);
      qz[j] = make_float2(v[5][0], v[5][1]);
      qlx[j] = make_float2(v[6][0], v[6][1]);
      qly[j] = make_float2(v[7][0], v[7][1]);
      qlz[j] = make_float2(v[8][0], v[8][1]);
      s2n[j] = make_float2(v[9][0], v[9][1]);
    }
    float2 shc[NP], slc[NP], shs[NP], sls[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) shc[j] = slc[j] = shs[j] = sls[j] = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < P; ++i) sacc[i * NT + tid] = make_double2(0.0, 0.0);

    const int k0 = wi.k0, k1 = wi.k1;
    if (tid == 0) {
      for (int k = k0; k < k1 && k < k0 + RING_STAGES; ++k) {
        const TileDesc td = tiles[k];
        const uint32_t st = g_issue % RING_STAGES;
        const uint32_t bytes = (uint32_t)td.count * 64u;
        mbar_arrive_expect_tx(&full_bar[st], bytes);
        if (!(stall && g_issue == 0))  // the stall hook skips the CTA's first copy
          bulk_copy_g2s(&ring[st][0], atoms2 + 4 * (long long)td.atom_begin, bytes, &full_bar[st]);
        ++g_issue;
      }
    }

    for (int k = k0; k < k1; ++k) {
      const uint32_t st = g_cons % RING_STAGES;
      const uint32_t par = (g_cons / RING_STAGES) & 1u;
      const bool ok = mbar_wait_bounded(&full_bar[st], par, kWaitCycles);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicOr(err, 1);
          for (uint32_t g = g_cons; g < g_issue; ++g)
            mbar_wait_bounded(&full_bar[g % RING_STAGES], (g / RING_STAGES) & 1u, kWaitCycles);
        }
        return;
      }
      const TileDesc td = tiles[k];
      const float4 *__restrict__ ta = ring[st];
      for (int a = 0; a < td.count; a += ATOM_GROUP) {
        float2 bc[NP], bs[NP];
#pragma unroll
        for (int j = 0; j < NP; ++j) bc[j] = bs[j] = make_float2(0.f, 0.f);
#pragma unroll
        for (int g = 0; g < ATOM_GROUP; ++g) {
          const float4 d0 = ta[4 * (a + g)], d1 = ta[4 * (a + g) + 1];
          const float4 d2 = ta[4 * (a + g) + 2], d3 = ta[4 * (a + g) + 3];
          const float2 Hx = make_float2(d0.x, d0.y), Hy = make_float2(d0.z, d0.w);
          const float2 Hz = make_float2(d1.x, d1.y), W = make_float2(d1.z, d1.w);
          const float2 Lx = make_float2(d2.x, d2.y), Ly = make_float2(d2.z, d2.w);
          const float2 Lz = make_float2(d3.x, d3.y);
#pragma unroll
          for (int j = 0; j < NP; ++j) {
            float2 w = W;
            if (PERB) w = make_float2(W.x * ex2_approx(d3.z * s2n[j].x), W.y * ex2_approx(d3.w * s2n[j].y));
            float2 u = mul2(qhx[j], Hx);
            u = fma2(qhy[j], Hy, u);
            u = fma2(qhz[j], Hz, u);
            float2 c = mul2(qx[j], Lx);
            c = fma2(qy[j], Ly, c);
            c = fma2(qz[j], Lz, c);
            c = fma2(qlx[j], Hx, c);
            c = fma2(qly[j], Hy, c);
            c = fma2(qlz[j], Hz, c);
            if (MODE == PREC_MODE_POLY) {
              // half-cycle reduction, one sign per term: e^{2 pi i (k/2 + y)} = (-1)^k e^{2 pi i y}
              const float2 t = fma2(u, f2(2.0f), f2(RINT_MAGIC));
              const float2 kf = add2(t, f2(-RINT_MAGIC));
              const float2 y = add2(fma2(kf, f2(-0.5f), u), c);
              const float2 z = mul2(y, y);
              float2 ps = fma2(z, f2(SPSIM_HALF_S4), f2(SPSIM_HALF_S3));
              ps = fma2(z, ps, f2(SPSIM_HALF_S2));
              ps = fma2(z, ps, f2(SPSIM_HALF_S1));
              ps = fma2(z, ps, f2(SPSIM_HALF_S0));
              float2 pc = fma2(z, f2(SPSIM_HALF_C5), f2(SPSIM_HALF_C4));
              pc = fma2(z, pc, f2(SPSIM_HALF_C3));
              pc = fma2(z, pc, f2(SPSIM_HALF_C2));
              pc = fma2(z, pc, f2(SPSIM_HALF_C1));
              pc = fma2(z, pc, f2(SPSIM_HALF_C0));
              const float2 S = mul2(y, ps);
              const float2 ws = make_float2(__uint_as_float(__float_as_uint(w.x) ^ (__float_as_uint(t.x) << 31)),
                                            __uint_as_float(__float_as_uint(w.y) ^ (__float_as_uint(t.y) << 31)));
              bc[j] = fma2(ws, pc, bc[j]);
              bs[j] = fma2(ws, S, bs[j]);
            } else {
              const float2 t = add2(u, f2(RINT_MAGIC));
              const float2 kf = add2(t, f2(-RINT_MAGIC));
              const float2 y = add2(add2(u, make_float2(-kf.x, -kf.y)), c);
              const float2 x = mul2(y, f2(6.28318530717958648f));
              float2 sn, cs;
              __sincosf(x.x, &sn.x, &cs.x);
              __sincosf(x.y, &sn.y, &cs.y);
              bc[j] = fma2(w, cs, bc[j]);
              bs[j] = fma2(w, sn, bs[j]);
            }
          }
        }
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          // Fast2Sum of the group sums into the float-float element sums
          float2 s1 = add2(shc[j], bc[j]);
          slc[j] = add2(slc[j], add2(bc[j], make_float2(-(s1.x - shc[j].x), -(s1.y - shc[j].y))));
          shc[j] = s1;
          float2 s2 = add2(shs[j], bs[j]);
          sls[j] = add2(sls[j], add2(bs[j], make_float2(-(s2.x - shs[j].x), -(s2.y - shs[j].y))));
          shs[j] = s2;
        }
      }
      if (td.last || k == k1 - 1) {
        // element done: f_e times its float-float sums into this thread's FP64 slots
        const double *__restrict__ ffe = pt.ff + (long long)td.elem * npix;
#pragma unroll
        for (int j = 0; j < NP; ++j) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const long long p = pix[2 * j + h];
            if (p < npix) {
              const double f = ffe[p];
              const double re = h ? (double)shc[j].y + (double)slc[j].y : (double)shc[j].x + (double)slc[j].x;
              const double sm = h ? (double)shs[j].y + (double)sls[j].y : (double)shs[j].x + (double)sls[j].x;
              double2 v = sacc[(2 * j + h) * NT + tid];
              v.x = fma(f, re, v.x);
              v.y = fma(-f, sm, v.y);
              sacc[(2 * j + h) * NT + tid] = v;
            }
          }
          shc[j] = slc[j] = shs[j] = sls[j] = make_float2(0.f, 0.f);
        }
      }
      __syncthreads();
      if (tid == 0 && k + RING_STAGES < k1) {
        const TileDesc tn = tiles[k + RING_STAGES];
        const uint32_t bytes = (uint32_t)tn.count * 64u;
        mbar_arrive_expect_tx(&full_bar[st], bytes);
        bulk_copy_g2s(&ring[st][0], atoms2 + 4 * (long long)tn.atom_begin, bytes, &full_bar[st]);
        ++g_issue;
      }
      ++g_cons;
    }
    // work item done: one write per pixel, a plain store when the item covers
    // every atom tile of the molecule (no other item touches these pixels)
    const bool whole = k0 == 0 && k1 == pt.n_tiles;
#pragma unroll
    for (int i = 0; i < P; ++i) {
      if (pix[i] < npix) {
        const double2 v = sacc[i * NT + tid];
        if (whole) {
          pt.acc[pix[i]] = v;
        } else {
          atomicAdd(&pt.acc[pix[i]].x, v.x);
          atomicAdd(&pt.acc[pix[i]].y, v.y);
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// FP64-phase forward on pixel pairs.  B200 runs FP64 FMA at half the FP32 rate
// and largely beside the FP32 pipe, so the phase q.(r - c) and its half-cycle
// reduction are FP64 (3 + 3 DFMA per term, the reduction exact) and only the
// sin/cos polynomial and the accumulation stay FP32, as packed f32x2
// instructions.  The reduced phase |y| <= 1/4 carries no cross term, so the
// polynomial pair is the shorter DHALF one and the only phase-range limit is
// |q.r| < 2^50 cycles.  Atom records are AtomD (32 bytes), staged by the same
// bulk-copy ring as the compensated kernels.

template <int MODE, int NT, int P, bool PERB, bool FIXW>
__global__ void __launch_bounds__(NT, sf_min_blocks(MODE)) sf_dphase_kernel(const SfPattern *__restrict__ pats,
                                                       const WorkItem *__restrict__ items, int n_items,
                                                       int *__restrict__ queue, int *__restrict__ err, uint32_t m31) {
  static_assert(P % 2 == 0, "pixels per thread must be even");
  constexpr int NP = P / 2;
  __shared__ __align__(128) float4 ring[RING_STAGES][2 * TILE_ATOMS];
  __shared__ __align__(16) double2 sacc[P * NT];  // per-thread FP64 pixel sums of the current work item
  __shared__ __align__(8) uint64_t full_bar[RING_STAGES];
  __shared__ int s_item;

  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < RING_STAGES; ++s) mbar_init(&full_bar[s], 1);
    fence_barrier_init();
  }
  __syncthreads();

  uint32_t g_issue = 0, g_cons = 0;
  const bool stall = g_copy_stall != 0;
  const long long kWaitCycles = stall ? kStallWaitCycles : kWaitCyclesDefault;
  const double M52 = 6755399441055744.0;  // 1.5 * 2^52: adding it rounds to an integer
  // FIXW: pixel q pre-scaled by 2 (half-cycle reduction) and the phase summed onto kWordBase
  constexpr double kQScale = (FIXW && MODE == PREC_MODE_POLY) ? 2.0 : 1.0;
  constexpr double kWordBase = MODE == PREC_MODE_POLY ? PHASE_WORD_BASE_HALF : PHASE_WORD_BASE;
  // per-atom B factors with the half-cycle phase word: the weight folded into the exponent
  constexpr bool LOGW = PERB && FIXW && MODE == PREC_MODE_POLY;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(queue, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WorkItem wi = items[it];
    const SfPattern &pt = pats[wi.pattern];
    const long long npix = pt.npix;
    const AtomD *__restrict__ atomsd = pt.atomsd;
    const TileDesc *__restrict__ tiles = pt.tiles;

    double qx[P], qy[P], qz[P];
    float s2n[P];
    const long long pix0 = (long long)wi.pixel_tile * (NT * P) + tid;  // pixel i of this thread: pix0 + i * NT
#pragma unroll
    for (int i = 0; i < P; ++i) {
      const long long p = pix0 + i * NT;
      double q[3] = {0.0, 0.0, 0.0};
      if (p < npix) load_q(pt, p, q);
      qx[i] = kQScale * q[0];
      qy[i] = kQScale * q[1];
      qz[i] = kQScale * q[2];
      s2n[i] = (float)(-0.25 * (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) * 1e-20 * pt.s2scale * 1.4426950408889634);
    }
    float2 shc[NP], slc[NP], shs[NP], sls[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) shc[j] = slc[j] = shs[j] = sls[j] = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < P; ++i) sacc[i * NT + tid] = make_double2(0.0, 0.0);

    const int k0 = wi.k0, k1 = wi.k1;
    if (tid == 0) {
      for (int k = k0; k < k1 && k < k0 + RING_STAGES; ++k) {
        const TileDesc td = tiles[k];
        const uint32_t st = g_issue % RING_STAGES;
        const uint32_t bytes = (uint32_t)td.count * (uint32_t)sizeof(AtomD);
        mbar_arrive_expect_tx(&full_bar[st], bytes);
        if (!(stall && g_issue == 0))  // the stall hook skips the CTA's first copy
          bulk_copy_g2s(&ring[st][0], atomsd + td.atom_begin, bytes, &full_bar[st]);
        ++g_issue;
      }
    }

    for (int k = k0; k < k1; ++k) {
      const uint32_t st = g_cons % RING_STAGES;
      const uint32_t par = (g_cons / RING_STAGES) & 1u;
      const bool ok = mbar_wait_bounded(&full_bar[st], par, kWaitCycles);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicOr(err, 1);
          for (uint32_t g = g_cons; g < g_issue; ++g)
            mbar_wait_bounded(&full_bar[g % RING_STAGES], (g / RING_STAGES) & 1u, kWaitCycles);
        }
        return;
      }
      const TileDesc td = tiles[k];
      const float4 *__restrict__ ta = ring[st];
      // atoms in groups of 2 x ATOM_GROUP (the last group of a tile may be
      // ATOM_GROUP): FP32 sums within a group, Fast2Sum after it
      for (int a = 0; a < td.count; a += 2 * ATOM_GROUP) {
        float2 bc[NP], bs[NP];
#pragma unroll
        for (int j = 0; j < NP; ++j) bc[j] = bs[j] = make_float2(0.f, 0.f);
#pragma unroll
        for (int g = 0; g < 2 * ATOM_GROUP; ++g) {
          if (g == ATOM_GROUP && a + ATOM_GROUP >= td.count) break;
          const float4 d0 = ta[2 * (a + g)], d1 = ta[2 * (a + g) + 1];
          const double rx = __hiloint2double(__float_as_int(d0.y), __float_as_int(d0.x));
          const double ry = __hiloint2double(__float_as_int(d0.w), __float_as_int(d0.z));
          const double rz = __hiloint2double(__float_as_int(d1.y), __float_as_int(d1.x));
          const float W = d1.z;
          // LOGW: W exp2(b s2) as exp2(b s2 + log2|W|), the sign of W as one more
          // half cycle in the phase word (its parity bit flips the term's sign)
          const float lw = LOGW ? lg2_approx(fabsf(W)) : 0.0f;
          const double wbase = LOGW && W < 0.0f ? kWordBase + 1.0 : kWordBase;
#pragma unroll
          for (int j = 0; j < NP; ++j) {
            float y[2], w[2];
            uint32_t kb[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int i = 2 * j + h;
              if (FIXW) {
                const double t = phase_word(qx[i], qy[i], qz[i], rx, ry, rz, wbase);
                reduce_phase_word<MODE>(t, y[h], kb[h]);
              } else {
                double u = qx[i] * rx;
                u = fma(qy[i], ry, u);
                u = fma(qz[i], rz, u);
                if (MODE == PREC_MODE_POLY) {
                  const double t = fma(u, 2.0, M52);  // rint(2u) in the low bits
                  y[h] = __double2float_rn(fma(t - M52, -0.5, u));  // u - k/2, exact before the rounding
                  kb[h] = (uint32_t)__double2loint(t);
                } else {
                  const double t = u + M52;
                  y[h] = __double2float_rn(u - (t - M52));
                  kb[h] = 0;
                }
              }
              w[h] = LOGW ? ex2_approx(fmaf(d1.w, s2n[i], lw)) : PERB ? W * ex2_approx(d1.w * s2n[i]) : W;
            }
            const float2 yy = FIXW ? mul2(make_float2(y[0], y[1]), f2(word_to_phase<MODE>()))
                                   : make_float2(y[0], y[1]);
            if (MODE == PREC_MODE_POLY) {
              // e^{2 pi i (k/2 + y)} = (-1)^k e^{2 pi i y}, |y| <= 1/4
              float2 S, pc;
              sincos_dhalf_poly2(yy, S, pc);
              const float2 ws = make_float2(sign_by_parity(w[0], kb[0], m31), sign_by_parity(w[1], kb[1], m31));
              bc[j] = fma2(ws, pc, bc[j]);
              bs[j] = fma2(ws, S, bs[j]);
            } else {
              const float2 x = FIXW ? yy : mul2(yy, f2(6.28318530717958648f));
              float2 sn, cs;
              __sincosf(x.x, &sn.x, &cs.x);
              __sincosf(x.y, &sn.y, &cs.y);
              const float2 ww = make_float2(w[0], w[1]);
              bc[j] = fma2(ww, cs, bc[j]);
              bs[j] = fma2(ww, sn, bs[j]);
            }
          }
        }
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          // Fast2Sum of the group sums into the float-float element sums
          ff_accumulate2(shc[j], slc[j], bc[j]);
          ff_accumulate2(shs[j], sls[j], bs[j]);
        }
      }
      if (td.last || k == k1 - 1) {
        // element done: f_e times its float-float sums into this thread's FP64 slots
        const double *__restrict__ ffe = pt.ff + (long long)td.elem * npix;
#pragma unroll
        for (int j = 0; j < NP; ++j) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const long long p = pix0 + (2 * j + h) * NT;
            if (p < npix) {
              const double f = ffe[p];
              const double re = h ? (double)shc[j].y + (double)slc[j].y : (double)shc[j].x + (double)slc[j].x;
              const double sm = h ? (double)shs[j].y + (double)sls[j].y : (double)shs[j].x + (double)sls[j].x;
              double2 v = sacc[(2 * j + h) * NT + tid];
              v.x = fma(f, re, v.x);
              v.y = fma(-f, sm, v.y);
              sacc[(2 * j + h) * NT + tid] = v;
            }
          }
          shc[j] = slc[j] = shs[j] = sls[j] = make_float2(0.f, 0.f);
        }
      }
      __syncthreads();
      if (tid == 0 && k + RING_STAGES < k1) {
        const TileDesc tn = tiles[k + RING_STAGES];
        const uint32_t bytes = (uint32_t)tn.count * (uint32_t)sizeof(AtomD);
        mbar_arrive_expect_tx(&full_bar[st], bytes);
        bulk_copy_g2s(&ring[st][0], atomsd + tn.atom_begin, bytes, &full_bar[st]);
        ++g_issue;
      }
      ++g_cons;
    }
    // work item done: one write per pixel, a plain store when the item covers
    // every atom tile of the molecule (no other item touches these pixels)
    const bool whole = k0 == 0 && k1 == pt.n_tiles;
#pragma unroll
    for (int i = 0; i < P; ++i) {
      const long long p = pix0 + i * NT;
      if (p < npix) {
        const double2 v = sacc[i * NT + tid];
        if (whole) {
          pt.acc[p] = v;
        } else {
          atomicAdd(&pt.acc[p].x, v.x);
          atomicAdd(&pt.acc[p].y, v.y);
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// FP64-anchored pixel pairs.  Pixels 2m and 2m+1 of a q set are neighbours on
// a detector row, so their phases differ by a small delta = (q_b - q_a).r.
// The first pixel of each pair takes the FP64 phase and exact half-cycle
// reduction of sf_dphase_kernel (|y_a| <= 1/4, sign (-1)^k); the second is
// y_b = y_a + delta with delta in FP32 from the float step q_b - q_a and the
// atom's float position, and the same sign.  The host admits a q set only
// when |q_b - q_a| * |r|max <= 1/8 cycle for every pair, so |y_b| <= 3/8
// stays inside the WIDE polynomial's domain.  Per term this replaces 6 FP64
// operations on every other pixel by 4 FP32 ones (and one more polynomial
// step).  Threads hold P pixels as
// P/2 pairs; two pairs' anchors and two pairs' seconds share each packed
// f32x2 polynomial.

// NARROW: every pair's step is at most 0.07 cycle (host-checked), so the
// second pixel's |y| <= 0.32 takes the NARROW polynomial, one FMA shorter.
template <int MODE, int NT, int P, bool PERB, bool FIXW, bool NARROW = false>
__global__ void __launch_bounds__(NT, sf_min_blocks(MODE)) sf_dpair_kernel(const SfPattern *__restrict__ pats,
                                                      const WorkItem *__restrict__ items, int n_items,
                                                      int *__restrict__ queue, int *__restrict__ err, uint32_t m31) {
  static_assert(P % 4 == 0, "pixels per thread must be a multiple of 4 (two pairs per packed instruction)");
  constexpr int NPR = P / 2;   // pixel pairs per thread
  constexpr int NPK = P / 4;   // packed pair-of-pairs
  __shared__ __align__(128) float4 ring[RING_STAGES][2 * TILE_ATOMS];
  __shared__ __align__(16) double2 sacc[P * NT];  // per-thread FP64 pixel sums of the current work item
  __shared__ __align__(8) uint64_t full_bar[RING_STAGES];
  __shared__ int s_item;

  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < RING_STAGES; ++s) mbar_init(&full_bar[s], 1);
    fence_barrier_init();
  }
  __syncthreads();

  uint32_t g_issue = 0, g_cons = 0;
  const bool stall = g_copy_stall != 0;
  const long long kWaitCycles = stall ? kStallWaitCycles : kWaitCyclesDefault;
  const double M52 = 6755399441055744.0;  // 1.5 * 2^52
  constexpr double kQScale = (FIXW && MODE == PREC_MODE_POLY) ? 2.0 : 1.0;
  constexpr double kWordBase = MODE == PREC_MODE_POLY ? PHASE_WORD_BASE_HALF : PHASE_WORD_BASE;
  // per-atom B factors with the half-cycle phase word: the weight folded into the exponent
  constexpr bool LOGW = PERB && FIXW && MODE == PREC_MODE_POLY;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(queue, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WorkItem wi = items[it];
    const SfPattern &pt = pats[wi.pattern];
    const long long npix = pt.npix;
    const AtomD *__restrict__ atomsd = pt.atomsd;
    const TileDesc *__restrict__ tiles = pt.tiles;

    // pair m of this thread: pixels pa = pix0 + 2 m NT and pa + 1
    const long long pix0 = (long long)wi.pixel_tile * (NT * P) + 2 * tid;
    double qx[NPR], qy[NPR], qz[NPR];
    float dqx[NPR], dqy[NPR], dqz[NPR], s2a[NPR], s2b[NPR];
#pragma unroll
    for (int m = 0; m < NPR; ++m) {
      const long long pa = pix0 + 2LL * m * NT;
      double a[3] = {0.0, 0.0, 0.0}, b[3] = {0.0, 0.0, 0.0};
      if (pa < npix) load_q(pt, pa, a);
      if (pa + 1 < npix) load_q(pt, pa + 1, b);
      else b[0] = a[0], b[1] = a[1], b[2] = a[2];
      qx[m] = kQScale * a[0];
      qy[m] = kQScale * a[1];
      qz[m] = kQScale * a[2];
      dqx[m] = (float)(b[0] - a[0]);
      dqy[m] = (float)(b[1] - a[1]);
      dqz[m] = (float)(b[2] - a[2]);
      s2a[m] = (float)(-0.25 * (a[0] * a[0] + a[1] * a[1] + a[2] * a[2]) * 1e-20 * pt.s2scale * 1.4426950408889634);
      s2b[m] = (float)(-0.25 * (b[0] * b[0] + b[1] * b[1] + b[2] * b[2]) * 1e-20 * pt.s2scale * 1.4426950408889634);
    }
    // float-float element sums: [pair-of-pairs][first / second pixel]
    float2 shc[NPK][2], slc[NPK][2], shs[NPK][2], sls[NPK][2];
#pragma unroll
    for (int j = 0; j < NPK; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) shc[j][h] = slc[j][h] = shs[j][h] = sls[j][h] = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < P; ++i) sacc[i * NT + tid] = make_double2(0.0, 0.0);

    const int k0 = wi.k0, k1 = wi.k1;
    if (tid == 0) {
      for (int k = k0; k < k1 && k < k0 + RING_STAGES; ++k) {
        const TileDesc td = tiles[k];
        const uint32_t st = g_issue % RING_STAGES;
        const uint32_t bytes = (uint32_t)td.count * (uint32_t)sizeof(AtomD);
        mbar_arrive_expect_tx(&full_bar[st], bytes);
        if (!(stall && g_issue == 0))  // the stall hook skips the CTA's first copy
          bulk_copy_g2s(&ring[st][0], atomsd + td.atom_begin, bytes, &full_bar[st]);
        ++g_issue;
      }
    }

    for (int k = k0; k < k1; ++k) {
      const uint32_t st = g_cons % RING_STAGES;
      const uint32_t par = (g_cons / RING_STAGES) & 1u;
      const bool ok = mbar_wait_bounded(&full_bar[st], par, kWaitCycles);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicOr(err, 1);
          for (uint32_t g = g_cons; g < g_issue; ++g)
            mbar_wait_bounded(&full_bar[g % RING_STAGES], (g / RING_STAGES) & 1u, kWaitCycles);
        }
        return;
      }
      const TileDesc td = tiles[k];
      const float4 *__restrict__ ta = ring[st];
      // atoms in groups of 2 x ATOM_GROUP (the last group of a tile may be
      // ATOM_GROUP): FP32 sums within a group, Fast2Sum after it
      for (int a = 0; a < td.count; a += 2 * ATOM_GROUP) {
        float2 bc[NPK][2], bs[NPK][2];
#pragma unroll
        for (int j = 0; j < NPK; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h) bc[j][h] = bs[j][h] = make_float2(0.f, 0.f);
#pragma unroll
        for (int g = 0; g < 2 * ATOM_GROUP; ++g) {
          if (g == ATOM_GROUP && a + ATOM_GROUP >= td.count) break;
          const float4 d0 = ta[2 * (a + g)], d1 = ta[2 * (a + g) + 1];
          const double rx = __hiloint2double(__float_as_int(d0.y), __float_as_int(d0.x));
          const double ry = __hiloint2double(__float_as_int(d0.w), __float_as_int(d0.z));
          const double rz = __hiloint2double(__float_as_int(d1.y), __float_as_int(d1.x));
          const float W = d1.z;
          const float2 fx = f2(__double2float_rn(rx)), fy = f2(__double2float_rn(ry)), fz = f2(__double2float_rn(rz));
          // LOGW: W exp2(b s2) as exp2(b s2 + log2|W|), the sign of W as one more
          // half cycle in the phase word (its parity bit flips both pixels' sign)
          const float lw = LOGW ? lg2_approx(fabsf(W)) : 0.0f;
          const double wbase = LOGW && W < 0.0f ? kWordBase + 1.0 : kWordBase;
#pragma unroll
          for (int j = 0; j < NPK; ++j) {
            float ya[2];
            uint32_t kb[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int m = 2 * j + h;
              if (FIXW) {
                const double t = phase_word(qx[m], qy[m], qz[m], rx, ry, rz, wbase);
                reduce_phase_word<MODE>(t, ya[h], kb[h]);
              } else {
                double u = qx[m] * rx;
                u = fma(qy[m], ry, u);
                u = fma(qz[m], rz, u);
                if (MODE == PREC_MODE_POLY) {
                  const double t = fma(u, 2.0, M52);
                  ya[h] = __double2float_rn(fma(t - M52, -0.5, u));
                  kb[h] = (uint32_t)__double2loint(t);
                } else {
                  const double t = u + M52;
                  ya[h] = __double2float_rn(u - (t - M52));
                  kb[h] = 0;
                }
              }
            }
            // anchors' reduced phases in cycles
            const float2 Ya = FIXW ? mul2(make_float2(ya[0], ya[1]), f2(word_to_cycles<MODE>()))
                                   : make_float2(ya[0], ya[1]);
            // second pixels: y_b = y_a + (q_b - q_a).r in FP32
            float2 dl = mul2(make_float2(dqx[2 * j], dqx[2 * j + 1]), fx);
            dl = fma2(make_float2(dqy[2 * j], dqy[2 * j + 1]), fy, dl);
            dl = fma2(make_float2(dqz[2 * j], dqz[2 * j + 1]), fz, dl);
            const float2 Yb = add2(Ya, dl);
            float2 wa = f2(W), wb = f2(W);
            if (LOGW) {
              wa = make_float2(ex2_approx(fmaf(d1.w, s2a[2 * j], lw)), ex2_approx(fmaf(d1.w, s2a[2 * j + 1], lw)));
              wb = make_float2(ex2_approx(fmaf(d1.w, s2b[2 * j], lw)), ex2_approx(fmaf(d1.w, s2b[2 * j + 1], lw)));
            } else if (PERB) {
              wa = make_float2(W * ex2_approx(d1.w * s2a[2 * j]), W * ex2_approx(d1.w * s2a[2 * j + 1]));
              wb = make_float2(W * ex2_approx(d1.w * s2b[2 * j]), W * ex2_approx(d1.w * s2b[2 * j + 1]));
            }
            if (MODE == PREC_MODE_POLY) {
              float2 Sa, Ca;
              sincos_dhalf_poly2(Ya, Sa, Ca);
              const float2 zb = mul2(Yb, Yb);
              float2 ps, pc;
              if (NARROW) {
                ps = fma2(zb, f2(SPSIM_NARROW_S4), f2(SPSIM_NARROW_S3));
                ps = fma2(zb, ps, f2(SPSIM_NARROW_S2));
                ps = fma2(zb, ps, f2(SPSIM_NARROW_S1));
                ps = fma2(zb, ps, f2(SPSIM_NARROW_S0));
                pc = fma2(zb, f2(SPSIM_NARROW_C5), f2(SPSIM_NARROW_C4));
                pc = fma2(zb, pc, f2(SPSIM_NARROW_C3));
                pc = fma2(zb, pc, f2(SPSIM_NARROW_C2));
                pc = fma2(zb, pc, f2(SPSIM_NARROW_C1));
                pc = fma2(zb, pc, f2(SPSIM_NARROW_C0));
              } else {
                ps = fma2(zb, f2(SPSIM_WIDE_S5), f2(SPSIM_WIDE_S4));
                ps = fma2(zb, ps, f2(SPSIM_WIDE_S3));
                ps = fma2(zb, ps, f2(SPSIM_WIDE_S2));
                ps = fma2(zb, ps, f2(SPSIM_WIDE_S1));
                ps = fma2(zb, ps, f2(SPSIM_WIDE_S0));
                pc = fma2(zb, f2(SPSIM_WIDE_C5), f2(SPSIM_WIDE_C4));
                pc = fma2(zb, pc, f2(SPSIM_WIDE_C3));
                pc = fma2(zb, pc, f2(SPSIM_WIDE_C2));
                pc = fma2(zb, pc, f2(SPSIM_WIDE_C1));
                pc = fma2(zb, pc, f2(SPSIM_WIDE_C0));
              }
              const float2 Sb = mul2(Yb, ps);
              const float2 wsa = make_float2(sign_by_parity_alu(wa.x, kb[0]), sign_by_parity_alu(wa.y, kb[1]));
              const float2 wsb = PERB ? make_float2(sign_by_parity_alu(wb.x, kb[0]), sign_by_parity_alu(wb.y, kb[1]))
                                      : wsa;
              bc[j][0] = fma2(wsa, Ca, bc[j][0]);
              bs[j][0] = fma2(wsa, Sa, bs[j][0]);
              bc[j][1] = fma2(wsb, pc, bc[j][1]);
              bs[j][1] = fma2(wsb, Sb, bs[j][1]);
            } else {
              const float2 xa = mul2(Ya, f2(6.28318530717958648f)), xb = mul2(Yb, f2(6.28318530717958648f));
              float2 sa, ca, sb, cb;
              __sincosf(xa.x, &sa.x, &ca.x);
              __sincosf(xa.y, &sa.y, &ca.y);
              __sincosf(xb.x, &sb.x, &cb.x);
              __sincosf(xb.y, &sb.y, &cb.y);
              bc[j][0] = fma2(wa, ca, bc[j][0]);
              bs[j][0] = fma2(wa, sa, bs[j][0]);
              bc[j][1] = fma2(wb, cb, bc[j][1]);
              bs[j][1] = fma2(wb, sb, bs[j][1]);
            }
          }
        }
#pragma unroll
        for (int j = 0; j < NPK; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            ff_accumulate2(shc[j][h], slc[j][h], bc[j][h]);
            ff_accumulate2(shs[j][h], sls[j][h], bs[j][h]);
          }
      }
      if (td.last || k == k1 - 1) {
        const double *__restrict__ ffe = pt.ff + (long long)td.elem * npix;
#pragma unroll
        for (int j = 0; j < NPK; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h)      // first / second pixel of the pairs
#pragma unroll
            for (int e = 0; e < 2; ++e) {  // which pair of the packed two
              const int m = 2 * j + e;
              const long long p = pix0 + 2LL * m * NT + h;
              if (p < npix) {
                const double f = ffe[p];
                const double re = e ? (double)shc[j][h].y + (double)slc[j][h].y : (double)shc[j][h].x + (double)slc[j][h].x;
                const double sm = e ? (double)shs[j][h].y + (double)sls[j][h].y : (double)shs[j][h].x + (double)sls[j][h].x;
                double2 v = sacc[(2 * m + h) * NT + tid];
                v.x = fma(f, re, v.x);
                v.y = fma(-f, sm, v.y);
                sacc[(2 * m + h) * NT + tid] = v;
              }
            }
#pragma unroll
        for (int j = 0; j < NPK; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h) shc[j][h] = slc[j][h] = shs[j][h] = sls[j][h] = make_float2(0.f, 0.f);
      }
      __syncthreads();
      if (tid == 0 && k + RING_STAGES < k1) {
        const TileDesc tn = tiles[k + RING_STAGES];
        const uint32_t bytes = (uint32_t)tn.count * (uint32_t)sizeof(AtomD);
        mbar_arrive_expect_tx(&full_bar[st], bytes);
        bulk_copy_g2s(&ring[st][0], atomsd + tn.atom_begin, bytes, &full_bar[st]);
        ++g_issue;
      }
      ++g_cons;
    }
    const bool whole = k0 == 0 && k1 == pt.n_tiles;
#pragma unroll
    for (int m = 0; m < NPR; ++m)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long long p = pix0 + 2LL * m * NT + h;
        if (p < npix) {
          const double2 v = sacc[(2 * m + h) * NT + tid];
          if (whole) {
            pt.acc[p] = v;
          } else {
            atomicAdd(&pt.acc[p].x, v.x);
            atomicAdd(&pt.acc[p].y, v.y);
          }
        }
      }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// FP64-anchored pixel quads.  Pixels 4m .. 4m+3 of a q set are neighbours on a
// detector row.  Pixel 4m+1 (the anchor) takes the FP64 phase and exact
// half-cycle reduction of the pair form (|y_a| <= 1/4, sign (-1)^k); each of
// the other three is y = y_a + (q - q_a).r in FP32, the step's three products
// summed onto y_a in one FMA chain, with the anchor's sign.  The host admits a
// q set when, for every quad, the one-pixel steps (4m and 4m+2 from the anchor)
// stay within 1/8 cycle of the molecule's bound (0.07 for NARROW) and the
// two-pixel step (4m+3) within 0.16 cycle, so that |y| <= 0.41.
//
// SPSIM_PREC_F32 (HYB false): every pixel's sin/cos on FMA-pipe polynomials,
// DHALF for the anchor, NARROW (or WIDER, for steps up to 1/8) for the
// one-pixel steps, WIDER (|y| <= 0.41, 6 + 6 coefficients) for the two-pixel
// step.  SPSIM_PREC_F32_FAST (HYB true): the work split between two pipes,
// the anchor and pixel 4m on the polynomials, pixels 4m+2 and 4m+3 on the XU
// pipe (MUFU sin/cos of 2 pi y, |2 pi y| <= 2.6); with per-atom B factors,
// whose weight exp2 already issues one XU operation per term, only pixel
// 4m+3.  Per quad that leaves ~51 FMA-pipe lane slots (FP32, the anchor's 3
// DFMA and its sign's IMAD) against ~6.5 XU operations (4 MUFU, the anchor's
// conversion, the atom's three FP64 -> FP32 conversions per two quads), which
// the two pipes take in about equal time (2.07e12 against 1.78e12 terms/s on
// the 50,000-atom workload).  MUFU's error is a bias of ~2e-7 over wide
// ranges of its argument rather than zero-mean noise, so a pixel whose sin/cos
// all come from MUFU carries it into |F|^2: the floored maximum error of the
// 50,000-atom workload is 3.2e-6 (2.1e-6 with polynomials only) but reaches
// ~1.7e-5 on random neighbour quads at |q| ~ 1e10 1/m, beyond SPSIM_PREC_F32's
// 1e-5; hence the split belongs to the fast mode.
// Against the pair form: 3 DFMA per four terms instead of per two, and one
// FP32 operation fewer per stepped pixel.  A partial last quad (q sets whose
// length is not a multiple of 4) anchors on its first pixel when that is the
// only one.  Threads hold P pixels as P/4 quads; the corresponding pixels of
// two quads share each packed f32x2 instruction.

// Anchor of quad base qb and the pixel of slot s (0 = anchor, 1..3 = qb, qb+2,
// qb+3), or -1 where the slot holds no pixel of the q set.
__device__ __forceinline__ long long quad_anchor(long long qb, long long npix) { return qb + 1 < npix ? qb + 1 : qb; }
__device__ __forceinline__ long long quad_pixel(long long qb, int slot, long long npix) {
  const long long pa = quad_anchor(qb, npix);
  const long long p = slot == 0 ? pa : slot == 1 ? qb : qb + slot;
  return (p < npix && (slot == 0 || p != pa)) ? p : -1;
}

template <int NT, int P, bool PERB, bool FIXW, bool NARROW, bool HYB>
__global__ void __launch_bounds__(NT, sf_min_blocks(PREC_MODE_POLY)) sf_dquad_kernel(
    const SfPattern *__restrict__ pats, const WorkItem *__restrict__ items, int n_items, int *__restrict__ queue,
    int *__restrict__ err, uint32_t m31) {
  static_assert(P % 8 == 0, "pixels per thread must be a multiple of 8 (two quads per packed instruction)");
  constexpr int NQ = P / 4;    // quads per thread
  constexpr int NQP = P / 8;   // packed pairs of quads
  __shared__ __align__(128) float4 ring[RING_STAGES][2 * TILE_ATOMS];
  __shared__ __align__(16) double2 sacc[P * NT];  // per-thread FP64 pixel sums of the current work item
  __shared__ __align__(8) uint64_t full_bar[RING_STAGES];
  __shared__ int s_item;

  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < RING_STAGES; ++s) mbar_init(&full_bar[s], 1);
    fence_barrier_init();
  }
  __syncthreads();

  uint32_t g_issue = 0, g_cons = 0;
  const bool stall = g_copy_stall != 0;
  const long long kWaitCycles = stall ? kStallWaitCycles : kWaitCyclesDefault;
  const double M52 = 6755399441055744.0;  // 1.5 * 2^52
  constexpr double kQScale = FIXW ? 2.0 : 1.0;
  constexpr double kWordBase = PHASE_WORD_BASE_HALF;
  // per-atom B factors with the phase word: the weight folded into the exponent
  constexpr bool LOGW = PERB && FIXW;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(queue, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WorkItem wi = items[it];
    const SfPattern &pt = pats[wi.pattern];
    const long long npix = pt.npix;
    const AtomD *__restrict__ atomsd = pt.atomsd;
    const TileDesc *__restrict__ tiles = pt.tiles;

    // quad g of this thread: pixels qb .. qb + 3, qb = pix0 + 4 g NT
    const long long pix0 = (long long)wi.pixel_tile * (NT * P) + 4 * tid;
    double qx[NQ], qy[NQ], qz[NQ];
    float dqx[NQ][3], dqy[NQ][3], dqz[NQ][3], s2[NQ][4];
#pragma unroll
    for (int g = 0; g < NQ; ++g) {
      const long long qb = pix0 + 4LL * g * NT;
      double a[3] = {0.0, 0.0, 0.0};
      if (qb < npix) load_q(pt, quad_anchor(qb, npix), a);
      qx[g] = kQScale * a[0];
      qy[g] = kQScale * a[1];
      qz[g] = kQScale * a[2];
      s2[g][0] = (float)(-0.25 * (a[0] * a[0] + a[1] * a[1] + a[2] * a[2]) * 1e-20 * pt.s2scale * 1.4426950408889634);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const long long p = quad_pixel(qb, s + 1, npix);
        double b[3] = {a[0], a[1], a[2]};
        if (p >= 0) load_q(pt, p, b);
        dqx[g][s] = (float)(b[0] - a[0]);
        dqy[g][s] = (float)(b[1] - a[1]);
        dqz[g][s] = (float)(b[2] - a[2]);
        s2[g][s + 1] =
            (float)(-0.25 * (b[0] * b[0] + b[1] * b[1] + b[2] * b[2]) * 1e-20 * pt.s2scale * 1.4426950408889634);
      }
    }
    // float-float element sums: [pair of quads][slot]
    float2 shc[NQP][4], slc[NQP][4], shs[NQP][4], sls[NQP][4];
#pragma unroll
    for (int j = 0; j < NQP; ++j)
#pragma unroll
      for (int h = 0; h < 4; ++h) shc[j][h] = slc[j][h] = shs[j][h] = sls[j][h] = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < P; ++i) sacc[i * NT + tid] = make_double2(0.0, 0.0);

    const int k0 = wi.k0, k1 = wi.k1;
    if (tid == 0) {
      for (int k = k0; k < k1 && k < k0 + RING_STAGES; ++k) {
        const TileDesc td = tiles[k];
        const uint32_t st = g_issue % RING_STAGES;
        const uint32_t bytes = (uint32_t)td.count * (uint32_t)sizeof(AtomD);
        mbar_arrive_expect_tx(&full_bar[st], bytes);
        if (!(stall && g_issue == 0))  // the stall hook skips the CTA's first copy
          bulk_copy_g2s(&ring[st][0], atomsd + td.atom_begin, bytes, &full_bar[st]);
        ++g_issue;
      }
    }

    for (int k = k0; k < k1; ++k) {
      const uint32_t st = g_cons % RING_STAGES;
      const uint32_t par = (g_cons / RING_STAGES) & 1u;
      const bool ok = mbar_wait_bounded(&full_bar[st], par, kWaitCycles);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicOr(err, 1);
          for (uint32_t g = g_cons; g < g_issue; ++g)
            mbar_wait_bounded(&full_bar[g % RING_STAGES], (g / RING_STAGES) & 1u, kWaitCycles);
        }
        return;
      }
      const TileDesc td = tiles[k];
      const float4 *__restrict__ ta = ring[st];
      // atoms in groups of 2 x ATOM_GROUP (the last group of a tile may be
      // ATOM_GROUP): FP32 sums within a group, Fast2Sum after it
      for (int a = 0; a < td.count; a += 2 * ATOM_GROUP) {
        float2 bc[NQP][4], bs[NQP][4];
#pragma unroll
        for (int j = 0; j < NQP; ++j)
#pragma unroll
          for (int h = 0; h < 4; ++h) bc[j][h] = bs[j][h] = make_float2(0.f, 0.f);
#pragma unroll
        for (int g = 0; g < 2 * ATOM_GROUP; ++g) {
          if (g == ATOM_GROUP && a + ATOM_GROUP >= td.count) break;
          const float4 d0 = ta[2 * (a + g)], d1 = ta[2 * (a + g) + 1];
          const double rx = __hiloint2double(__float_as_int(d0.y), __float_as_int(d0.x));
          const double ry = __hiloint2double(__float_as_int(d0.w), __float_as_int(d0.z));
          const double rz = __hiloint2double(__float_as_int(d1.y), __float_as_int(d1.x));
          const float W = d1.z;
          const float2 fx = f2(__double2float_rn(rx)), fy = f2(__double2float_rn(ry)), fz = f2(__double2float_rn(rz));
          // LOGW: W exp2(b s2) as exp2(b s2 + log2|W|), the sign of W as one more
          // half cycle in the phase word (its parity bit flips every pixel's sign)
          const float lw = LOGW ? lg2_approx(fabsf(W)) : 0.0f;
          const double wbase = LOGW && W < 0.0f ? kWordBase + 1.0 : kWordBase;
#pragma unroll
          for (int j = 0; j < NQP; ++j) {
            float ya[2];
            uint32_t kb[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int m = 2 * j + h;
              if (FIXW) {
                const double t = phase_word(qx[m], qy[m], qz[m], rx, ry, rz, wbase);
                reduce_phase_word<PREC_MODE_POLY>(t, ya[h], kb[h]);
              } else {
                double u = qx[m] * rx;
                u = fma(qy[m], ry, u);
                u = fma(qz[m], rz, u);
                const double t = fma(u, 2.0, M52);
                ya[h] = __double2float_rn(fma(t - M52, -0.5, u));
                kb[h] = (uint32_t)__double2loint(t);
              }
            }
            // anchors' reduced phases in cycles, then the stepped pixels
            float2 Y[4];
            Y[0] = FIXW ? mul2(make_float2(ya[0], ya[1]), f2(word_to_cycles<PREC_MODE_POLY>()))
                        : make_float2(ya[0], ya[1]);
#pragma unroll
            for (int s = 0; s < 3; ++s) {
              float2 y = fma2(make_float2(dqx[2 * j][s], dqx[2 * j + 1][s]), fx, Y[0]);
              y = fma2(make_float2(dqy[2 * j][s], dqy[2 * j + 1][s]), fy, y);
              Y[s + 1] = fma2(make_float2(dqz[2 * j][s], dqz[2 * j + 1][s]), fz, y);
            }
            float2 ws[4];
            if (PERB) {
#pragma unroll
              for (int h = 0; h < 4; ++h) {
                const float w0 = LOGW ? ex2_approx(fmaf(d1.w, s2[2 * j][h], lw)) : W * ex2_approx(d1.w * s2[2 * j][h]);
                const float w1 =
                    LOGW ? ex2_approx(fmaf(d1.w, s2[2 * j + 1][h], lw)) : W * ex2_approx(d1.w * s2[2 * j + 1][h]);
                ws[h] = HYB ? make_float2(sign_by_parity(w0, kb[0], m31), sign_by_parity(w1, kb[1], m31))
                            : make_float2(sign_by_parity_alu(w0, kb[0]), sign_by_parity_alu(w1, kb[1]));
              }
            } else {
              ws[0] = HYB ? make_float2(sign_by_parity(W, kb[0], m31), sign_by_parity(W, kb[1], m31))
                          : make_float2(sign_by_parity_alu(W, kb[0]), sign_by_parity_alu(W, kb[1]));
              ws[1] = ws[2] = ws[3] = ws[0];
            }
            float2 S, C;
            sincos_dhalf_poly2(Y[0], S, C);
            bc[j][0] = fma2(ws[0], C, bc[j][0]);
            bs[j][0] = fma2(ws[0], S, bs[j][0]);
            // HYB: pixels 4m+2 and 4m+3 on MUFU; per-atom B factors already give
            // the XU pipe one ex2 per term, so there only pixel 4m+3
            constexpr int kFirstMufu = !HYB ? 4 : (PERB ? 3 : 2);
#pragma unroll
            for (int h = 1; h < kFirstMufu; ++h) {
              if (NARROW && h < 3)
                sincos_narrow_poly2(Y[h], S, C);
              else
                sincos_wider_poly2(Y[h], S, C);
              bc[j][h] = fma2(ws[h], C, bc[j][h]);
              bs[j][h] = fma2(ws[h], S, bs[j][h]);
            }
#pragma unroll
            for (int h = kFirstMufu; h < 4; ++h) {  // MUFU sin/cos on the XU pipe
              const float2 x = mul2(Y[h], f2(6.28318530717958648f));
              __sincosf(x.x, &S.x, &C.x);
              __sincosf(x.y, &S.y, &C.y);
              bc[j][h] = fma2(ws[h], C, bc[j][h]);
              bs[j][h] = fma2(ws[h], S, bs[j][h]);
            }
          }
        }
#pragma unroll
        for (int j = 0; j < NQP; ++j)
#pragma unroll
          for (int h = 0; h < 4; ++h) {
            ff_accumulate2(shc[j][h], slc[j][h], bc[j][h]);
            ff_accumulate2(shs[j][h], sls[j][h], bs[j][h]);
          }
      }
      if (td.last || k == k1 - 1) {
        const double *__restrict__ ffe = pt.ff + (long long)td.elem * npix;
#pragma unroll
        for (int j = 0; j < NQP; ++j)
#pragma unroll
          for (int h = 0; h < 4; ++h)      // slot: anchor, then the stepped pixels
#pragma unroll
            for (int e = 0; e < 2; ++e) {  // which quad of the packed two
              const int g = 2 * j + e;
              const long long p = quad_pixel(pix0 + 4LL * g * NT, h, npix);
              if (p >= 0) {
                const double f = ffe[p];
                const double re = e ? (double)shc[j][h].y + (double)slc[j][h].y : (double)shc[j][h].x + (double)slc[j][h].x;
                const double sm = e ? (double)shs[j][h].y + (double)sls[j][h].y : (double)shs[j][h].x + (double)sls[j][h].x;
                double2 v = sacc[(4 * g + h) * NT + tid];
                v.x = fma(f, re, v.x);
                v.y = fma(-f, sm, v.y);
                sacc[(4 * g + h) * NT + tid] = v;
              }
            }
#pragma unroll
        for (int j = 0; j < NQP; ++j)
#pragma unroll
          for (int h = 0; h < 4; ++h) shc[j][h] = slc[j][h] = shs[j][h] = sls[j][h] = make_float2(0.f, 0.f);
      }
      __syncthreads();
      if (tid == 0 && k + RING_STAGES < k1) {
        const TileDesc tn = tiles[k + RING_STAGES];
        const uint32_t bytes = (uint32_t)tn.count * (uint32_t)sizeof(AtomD);
        mbar_arrive_expect_tx(&full_bar[st], bytes);
        bulk_copy_g2s(&ring[st][0], atomsd + tn.atom_begin, bytes, &full_bar[st]);
        ++g_issue;
      }
      ++g_cons;
    }
    const bool whole = k0 == 0 && k1 == pt.n_tiles;
#pragma unroll
    for (int g = 0; g < NQ; ++g)
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const long long p = quad_pixel(pix0 + 4LL * g * NT, h, npix);
        if (p >= 0) {
          const double2 v = sacc[(4 * g + h) * NT + tid];
          if (whole) {
            pt.acc[p] = v;
          } else {
            atomicAdd(&pt.acc[p].x, v.x);
            atomicAdd(&pt.acc[p].y, v.y);
          }
        }
      }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// plain FP64 forward: one thread per pixel, atoms read as warp-uniform loads

__global__ void __launch_bounds__(256) sf_f64_kernel(const SfPattern *__restrict__ pats, int pattern) {
  const SfPattern &pt = pats[pattern];
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pt.npix) return;
  double q[3];
  load_q(pt, p, q);
  const double s2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) * 1e-20 * 0.25 * pt.s2scale;
  double fr = 0.0, fi = 0.0, ar = 0.0, ai = 0.0;
  for (int k = 0; k < pt.n_tiles; ++k) {
    const TileDesc td = pt.tiles[k];
    for (int j = td.atom_begin; j < td.atom_begin + td.count; ++j) {
      const float4 a0 = __ldg(&pt.atoms[2 * j]);
      const float4 a1 = __ldg(&pt.atoms[2 * j + 1]);
      const double rx = (double)a0.x + (double)a1.x;
      const double ry = (double)a0.y + (double)a1.y;
      const double rz = (double)a0.z + (double)a1.z;
      double t = q[0] * rx + q[1] * ry + q[2] * rz;
      t -= rint(t);
      double s, c;
      sincospi(2.0 * t, &s, &c);
      double w = a0.w;
      if (pt.per_atom_b) w *= exp(-(double)a1.w * s2);
      ar += w * c;
      ai -= w * s;
    }
    if (td.last) {
      const double f = pt.ff[(long long)td.elem * pt.npix + p];
      fr += f * ar;
      fi += f * ai;
      ar = ai = 0.0;
    }
  }
  pt.acc[p] = make_double2(fr, fi);
}

// ---------------------------------------------------------------------------
// finalize: F = e^{-2 pi i q.c} acc, I = |acc|^2

__global__ void sf_finalize_kernel(const SfPattern *__restrict__ pats, int pattern0) {
  const SfPattern &pt = pats[pattern0 + blockIdx.y];
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0 && pt.mol_err && *pt.mol_err) atomicOr(pt.plan_err, 1);
  if (p >= pt.npix) return;
  const double2 a = pt.acc[p];
  if (pt.I) pt.I[p] = (float)(a.x * a.x + a.y * a.y);
  if (pt.F) {
    double q[3];
    load_q(pt, p, q);
    double t = q[0] * pt.center[0] + q[1] * pt.center[1] + q[2] * pt.center[2];
    t -= rint(t);
    double s, c;
    sincospi(2.0 * t, &s, &c);
    pt.F[p] = make_float2((float)(a.x * c + a.y * s), (float)(a.y * c - a.x * s));
  }
}

// Polychromatic combination (src/diffraction.cu:415-476 semantics): the
// patterns pattern0 .. pattern0+S-1 hold the centred FP64 amplitudes of one
// detector at the phase-space scales lambda / lambda_j; F is their weighted
// sum, each with its own centre phase e^{-2 pi i s_j q.c}, and I = |F|^2.
__global__ void sf_spectrum_combine_kernel(const SfPattern *__restrict__ pats, int pattern0, int S,
                                           const double *__restrict__ weight, float2 *__restrict__ F,
                                           float *__restrict__ I, long long npix) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0 && pats[pattern0].mol_err && *pats[pattern0].mol_err) atomicOr(pats[pattern0].plan_err, 1);
  if (p >= npix) return;
  double re = 0.0, im = 0.0;
  for (int j = 0; j < S; ++j) {
    const SfPattern &pt = pats[pattern0 + j];
    const double2 a = pt.acc[p];
    double q[3];
    load_q(pt, p, q);
    double t = q[0] * pt.center[0] + q[1] * pt.center[1] + q[2] * pt.center[2];
    t -= rint(t);
    double s, c;
    sincospi(2.0 * t, &s, &c);
    re += weight[j] * (a.x * c + a.y * s);
    im += weight[j] * (a.y * c - a.x * s);
  }
  if (F) F[p] = make_float2((float)re, (float)im);
  if (I) I[p] = (float)(re * re + im * im);
}

// ---------------------------------------------------------------------------
// Ewald geometry: the reference's operation order, FP64 without contraction

__global__ void ewald_kernel(int nx, int ny, double width, double height, double distance, double cx, double cy,
                             double ewald, int spherical, double fpx, double fpy, double px_size, double py_size,
                             float *__restrict__ out32, double *__restrict__ out64) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nx * ny) return;
  const int x = (int)(i % nx), y = (int)(i / nx);
  const double px = __dsub_rn(__dmul_rn(__ddiv_rn(__dsub_rn((double)x, (nx - 1.0) / 2.0), (double)nx), width), cx);
  const double py = __dsub_rn(__dmul_rn(__ddiv_rn(__dsub_rn((double)y, (ny - 1.0) / 2.0), (double)ny), height), cy);
  const double pz = distance;
  double q0, q1, q2;
  if (!spherical) {
    const double p = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)), __dmul_rn(pz, pz)));
    q0 = __dmul_rn(__ddiv_rn(px, p), ewald);
    q1 = __dmul_rn(__ddiv_rn(py, p), ewald);
    q2 = __dmul_rn(__dsub_rn(__ddiv_rn(pz, p), 1.0), ewald);
  } else {
    q0 = __ddiv_rn(__dmul_rn(fpx, px), px_size);
    q1 = __ddiv_rn(__dmul_rn(fpy, py), py_size);
    q2 = 0.0;
  }
  if (out32) {
    out32[3 * i] = (float)q0;
    out32[3 * i + 1] = (float)q1;
    out32[3 * i + 2] = (float)q2;
  }
  if (out64) {
    out64[3 * i] = q0;
    out64[3 * i + 1] = q1;
    out64[3 * i + 2] = q2;
  }
}

// Reciprocal-space grid of a 3-D (volume) detector (src/diffraction.c:325-369):
// pixel centres scaled by 1 / (distance * wavelength), FP64 without
// contraction as the reference computes them, stored as float.
__global__ void volume_kernel(int nx, int ny, int nz, double width, double height, double depth, double cx, double cy,
                              double cz, double r2r, float *__restrict__ out32) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nx * ny * nz) return;
  const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
  const double px = __dsub_rn(__dmul_rn(__ddiv_rn(__dsub_rn((double)x, (nx - 1.0) / 2.0), (double)nx), width), cx);
  const double py = __dsub_rn(__dmul_rn(__ddiv_rn(__dsub_rn((double)y, (ny - 1.0) / 2.0), (double)ny), height), cy);
  const double pz = __dsub_rn(__dmul_rn(__ddiv_rn(__dsub_rn((double)z, (nz - 1.0) / 2.0), (double)nz), depth), cz);
  out32[3 * i] = (float)__dmul_rn(px, r2r);
  out32[3 * i + 1] = (float)__dmul_rn(py, r2r);
  out32[3 * i + 2] = (float)__dmul_rn(pz, r2r);
}

// Crystal lattice sum (src/crystal.c:39-71): F <- F * sum_{a,b,c} e^{-2 pi i q.(a A + b B + c C)}
// over na x nb x nc cells, I = |F|^2.  The lattice factor separates into three
// one-dimensional sums, each taken term by term in FP64 (no closed form, which
// loses accuracy next to Bragg peaks).
__device__ __forceinline__ double2 lattice_line(double u, int n) {
  double re = 0.0, im = 0.0;
  for (int a = 0; a < n; ++a) {
    double t = u * a;
    t -= rint(t);
    double s, c;
    sincospi(2.0 * t, &s, &c);
    re += c;
    im -= s;
  }
  return make_double2(re, im);
}

__global__ void crystal_kernel(long long npix, const float *__restrict__ hkl, double ax, double ay, double az,
                               double bx, double by, double bz, double cx, double cy, double cz, int na, int nb,
                               int nc, float2 *__restrict__ F, float *__restrict__ I) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npix) return;
  const double qx = hkl[3 * p], qy = hkl[3 * p + 1], qz = hkl[3 * p + 2];
  const double2 sa = lattice_line(qx * ax + qy * ay + qz * az, na);
  const double2 sb = lattice_line(qx * bx + qy * by + qz * bz, nb);
  const double2 sc = lattice_line(qx * cx + qy * cy + qz * cz, nc);
  const double2 ab = make_double2(sa.x * sb.x - sa.y * sb.y, sa.x * sb.y + sa.y * sb.x);
  const double2 s = make_double2(ab.x * sc.x - ab.y * sc.y, ab.x * sc.y + ab.y * sc.x);
  const float2 f = F[p];
  const double re = f.x * s.x - f.y * s.y, im = f.x * s.y + f.y * s.x;
  F[p] = make_float2((float)re, (float)im);
  if (I) I[p] = (float)(re * re + im * im);
}

// ---------------------------------------------------------------------------
// refinement: rewrite atom records from device positions (caller order)

__global__ void atoms_update_kernel(float4 *__restrict__ atoms, float4 *__restrict__ atoms2, AtomD *__restrict__ atomsd,
                                    const int *__restrict__ perm, int n_padded,
                                    const float *__restrict__ pos32, const double *__restrict__ pos64,
                                    const float *__restrict__ occ, const float *__restrict__ bfac,
                                    const float *__restrict__ wbase, double cx, double cy, double cz, float dr,
                                    float inv_dr, double rbound, int *__restrict__ range_err) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_padded) return;
  const int src = perm[j];
  if (src < 0) return;
  double r[3];
  if (pos64) {
    r[0] = pos64[3 * src] - cx;
    r[1] = pos64[3 * src + 1] - cy;
    r[2] = pos64[3 * src + 2] - cz;
  } else {
    r[0] = (double)pos32[3 * src] - cx;
    r[1] = (double)pos32[3 * src + 1] - cy;
    r[2] = (double)pos32[3 * src + 2] - cz;
  }
  if (r[0] * r[0] + r[1] * r[1] + r[2] * r[2] > rbound * rbound) atomicOr(range_err, 1);
  float4 a0 = atoms[2 * j], a1 = atoms[2 * j + 1];
  const double hx = (double)rintf((float)r[0] * inv_dr) * dr;
  const double hy = (double)rintf((float)r[1] * inv_dr) * dr;
  const double hz = (double)rintf((float)r[2] * inv_dr) * dr;
  a0.x = (float)hx;
  a0.y = (float)hy;
  a0.z = (float)hz;
  a1.x = (float)(r[0] - hx);
  a1.y = (float)(r[1] - hy);
  a1.z = (float)(r[2] - hz);
  if (occ) a0.w = occ[src] * wbase[j];
  if (bfac) a1.w = bfac[src];
  atoms[2 * j] = a0;
  atoms[2 * j + 1] = a1;
  atoms2[4 * j] = make_float4(a0.x, a0.x, a0.y, a0.y);
  atoms2[4 * j + 1] = make_float4(a0.z, a0.z, a0.w, a0.w);
  atoms2[4 * j + 2] = make_float4(a1.x, a1.x, a1.y, a1.y);
  atoms2[4 * j + 3] = make_float4(a1.z, a1.z, a1.w, a1.w);
  atomsd[j] = AtomD{r[0], r[1], r[2], a0.w, a1.w};
}

// Molecule creation on the device: the atom records of padded atom j from the
// caller's positions (atom perm[j]; perm < 0 is segment padding, all zero),
// with the host's arithmetic: r = pos - centre in FP64, the coarse part
// rint(r / dr) dr and the remainder, the weight occ * wbase in float.
template <typename PosT>
__global__ void atoms_build_kernel(float4 *__restrict__ atoms, float4 *__restrict__ atoms2, AtomD *__restrict__ atomsd,
                                   const int *__restrict__ perm, int n_padded, const PosT *__restrict__ pos,
                                   const float *__restrict__ occ, const float *__restrict__ bfac,
                                   const float *__restrict__ wbase, double cx, double cy, double cz, double dr,
                                   double inv_dr) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_padded) return;
  const int src = perm[j];
  if (src < 0) {
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    atoms[2 * j] = atoms[2 * j + 1] = z;
    atoms2[4 * j] = atoms2[4 * j + 1] = atoms2[4 * j + 2] = atoms2[4 * j + 3] = z;
    atomsd[j] = AtomD{0.0, 0.0, 0.0, 0.0f, 0.0f};
    return;
  }
  const double r0 = __dsub_rn((double)pos[3 * src], cx);
  const double r1 = __dsub_rn((double)pos[3 * src + 1], cy);
  const double r2 = __dsub_rn((double)pos[3 * src + 2], cz);
  const double hx = __dmul_rn(rint(__dmul_rn(r0, inv_dr)), dr);
  const double hy = __dmul_rn(rint(__dmul_rn(r1, inv_dr)), dr);
  const double hz = __dmul_rn(rint(__dmul_rn(r2, inv_dr)), dr);
  const float w = __fmul_rn(occ ? occ[src] : 1.0f, wbase[j]);
  const float b = bfac ? bfac[src] : 0.0f;
  const float4 a0 = make_float4((float)hx, (float)hy, (float)hz, w);
  const float4 a1 = make_float4((float)__dsub_rn(r0, hx), (float)__dsub_rn(r1, hy), (float)__dsub_rn(r2, hz), b);
  atoms[2 * j] = a0;
  atoms[2 * j + 1] = a1;
  atoms2[4 * j] = make_float4(a0.x, a0.x, a0.y, a0.y);
  atoms2[4 * j + 1] = make_float4(a0.z, a0.z, a0.w, a0.w);
  atoms2[4 * j + 2] = make_float4(a1.x, a1.x, a1.y, a1.y);
  atoms2[4 * j + 3] = make_float4(a1.z, a1.z, a1.w, a1.w);
  atomsd[j] = AtomD{r0, r1, r2, w, b};
}

template <typename PosT>
cudaError_t launch_atoms_build(float4 *atoms, float4 *atoms2, AtomD *atomsd, const int *perm, int n_padded,
                               const PosT *pos, const float *occ, const float *bfac, const float *wbase,
                               const double c[3], double dr, double inv_dr, cudaStream_t st) {
  if (n_padded <= 0) return cudaSuccess;
  atoms_build_kernel<PosT><<<(n_padded + 255) / 256, 256, 0, st>>>(atoms, atoms2, atomsd, perm, n_padded, pos, occ,
                                                                  bfac, wbase, c[0], c[1], c[2], dr, inv_dr);
  return cudaGetLastError();
}
template cudaError_t launch_atoms_build<float>(float4 *, float4 *, AtomD *, const int *, int, const float *,
                                               const float *, const float *, const float *, const double[3], double,
                                               double, cudaStream_t);
template cudaError_t launch_atoms_build<double>(float4 *, float4 *, AtomD *, const int *, int, const double *,
                                                const float *, const float *, const float *, const double[3], double,
                                                double, cudaStream_t);

// ---------------------------------------------------------------------------
// launch wrappers

cudaError_t launch_ff_table(const float *hkl, const double *q64, long long npix, int n_elem, const float *coeffs,
                            double B, int delta_atoms, double *ff, cudaStream_t st) {
  if (npix <= 0 || n_elem <= 0) return cudaSuccess;
  dim3 grid((unsigned)((npix + 255) / 256), (unsigned)n_elem);
  ff_table_kernel<<<grid, 256, 0, st>>>(hkl, q64, npix, n_elem, coeffs, B, delta_atoms, ff);
  return cudaGetLastError();
}

// Variants: (mode, threads, pixels per thread, form).  form 0 selects the
// scalar compensated kernel (sf_f32_kernel), 1 the pixel-pair compensated one
// (sf_f32x2_kernel), 2 the pixel-pair FP64-phase one (sf_dphase_kernel), 3 the
// FP64-anchored neighbour pairs (sf_dpair_kernel).
template <int MODE, int NT, int P, bool PERB, int PK, bool FW, bool NW = false>
static cudaError_t launch_f32_t(const SfPattern *pats, const WorkItem *items, int n_items, int *queue, int *err,
                                int grid, cudaStream_t st) {
  if constexpr (PK == 4)
    sf_dquad_kernel<NT, P, PERB, FW, NW, MODE == PREC_MODE_MUFU><<<grid, NT, 0, st>>>(pats, items, n_items, queue, err,
                                                                              0x80000000u);
  else if constexpr (PK == 3)
    sf_dpair_kernel<MODE, NT, P, PERB, FW, NW><<<grid, NT, 0, st>>>(pats, items, n_items, queue, err, 0x80000000u);
  else if constexpr (PK == 2)
    sf_dphase_kernel<MODE, NT, P, PERB, FW><<<grid, NT, 0, st>>>(pats, items, n_items, queue, err, 0x80000000u);
  else if constexpr (PK == 1)
    sf_f32x2_kernel<MODE, NT, P, PERB><<<grid, NT, 0, st>>>(pats, items, n_items, queue, err);
  else
    sf_f32_kernel<MODE, NT, P, PERB><<<grid, NT, 0, st>>>(pats, items, n_items, queue, err);
  return cudaGetLastError();
}

template <int MODE, int NT, int P, bool PERB, int PK, bool FW, bool NW = false>
static int occupancy_t() {
  int n = 0;
  if constexpr (PK == 4)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sf_dquad_kernel<NT, P, PERB, FW, NW, MODE == PREC_MODE_MUFU>, NT,
                                                  0);
  else if constexpr (PK == 3)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sf_dpair_kernel<MODE, NT, P, PERB, FW, NW>, NT, 0);
  else if constexpr (PK == 2)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sf_dphase_kernel<MODE, NT, P, PERB, FW>, NT, 0);
  else if constexpr (PK == 1)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sf_f32x2_kernel<MODE, NT, P, PERB>, NT, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sf_f32_kernel<MODE, NT, P, PERB>, NT, 0);
  return n;
}

#define SPSIM_F32_VARIANTS(X) \
  X(0, 128, 2, 0)             \
  X(0, 128, 4, 0)             \
  X(0, 256, 4, 0)             \
  X(1, 128, 2, 0)             \
  X(1, 128, 4, 0)             \
  X(1, 256, 4, 0)             \
  X(0, 128, 2, 1)             \
  X(0, 128, 4, 1)             \
  X(0, 256, 4, 1)             \
  X(0, 128, 6, 1)             \
  X(1, 128, 2, 1)             \
  X(1, 128, 4, 1)             \
  X(1, 256, 4, 1)             \
  X(1, 128, 6, 1)             \
  X(0, 128, 2, 2)             \
  X(0, 128, 4, 2)             \
  X(0, 256, 4, 2)             \
  X(0, 128, 6, 2)             \
  X(0, 128, 8, 2)             \
  X(1, 128, 2, 2)             \
  X(1, 128, 4, 2)             \
  X(1, 256, 4, 2)             \
  X(1, 128, 6, 2)             \
  X(1, 128, 8, 2)             \
  X(0, 128, 4, 3)             \
  X(0, 128, 8, 3)             \
  X(0, 128, 12, 3)            \
  X(0, 256, 4, 3)             \
  X(1, 128, 4, 3)             \
  X(1, 128, 8, 3)             \
  X(1, 128, 12, 3)            \
  X(1, 256, 4, 3)             \
  X(0, 128, 8, 4)             \
  X(0, 128, 16, 4)            \
  X(0, 256, 8, 4)             \
  X(1, 128, 8, 4)             \
  X(1, 128, 16, 4)            \
  X(1, 256, 8, 4)

// fixw selects the fixed-point phase word in the FP64-phase forms (2, 3, 4),
// narrow the NARROW polynomial of forms 3 and 4; the compensated forms ignore both.
cudaError_t launch_sf_f32(int mode, int nt, int p, int packed, bool perb, const SfPattern *pats,
                          const WorkItem *items, int n_items, int *queue, int *err, int grid, cudaStream_t st,
                          bool fixw, bool narrow) {
#define X(M, N, PP, PK)                                                                                   \
  if (mode == M && nt == N && p == PP && packed == PK) {                                                  \
    if (narrow && fixw && (PK == 4 || (PK == 3 && M == PREC_MODE_POLY)))                                  \
      return perb ? launch_f32_t<M, N, PP, true, PK, true, true>(pats, items, n_items, queue, err, grid, st) \
                  : launch_f32_t<M, N, PP, false, PK, true, true>(pats, items, n_items, queue, err, grid, st); \
    if (fixw && PK >= 2)                                                                                  \
      return perb ? launch_f32_t<M, N, PP, true, PK, true>(pats, items, n_items, queue, err, grid, st)    \
                  : launch_f32_t<M, N, PP, false, PK, true>(pats, items, n_items, queue, err, grid, st);  \
    return perb ? launch_f32_t<M, N, PP, true, PK, false>(pats, items, n_items, queue, err, grid, st)     \
                : launch_f32_t<M, N, PP, false, PK, false>(pats, items, n_items, queue, err, grid, st);   \
  }
  SPSIM_F32_VARIANTS(X)
#undef X
  return cudaErrorInvalidConfiguration;
}

int sf_f32_occupancy(int mode, int nt, int p, int packed, bool perb, bool fixw, bool narrow) {
#define X(M, N, PP, PK)                                                                          \
  if (mode == M && nt == N && p == PP && packed == PK) {                                         \
    if (narrow && fixw && (PK == 4 || (PK == 3 && M == PREC_MODE_POLY)))                         \
      return perb ? occupancy_t<M, N, PP, true, PK, true, true>()                                \
                  : occupancy_t<M, N, PP, false, PK, true, true>();                              \
    if (fixw && PK >= 2)                                                                         \
      return perb ? occupancy_t<M, N, PP, true, PK, true>() : occupancy_t<M, N, PP, false, PK, true>(); \
    return perb ? occupancy_t<M, N, PP, true, PK, false>() : occupancy_t<M, N, PP, false, PK, false>(); \
  }
  SPSIM_F32_VARIANTS(X)
#undef X
  return 0;
}

bool sf_f32_variant_exists(int mode, int nt, int p, int packed) {
#define X(M, N, PP, PK) \
  if (mode == M && nt == N && p == PP && packed == PK) return true;
  SPSIM_F32_VARIANTS(X)
#undef X
  return false;
}

cudaError_t launch_sf_f64(const SfPattern *pats, int pattern, long long npix, cudaStream_t st) {
  if (npix <= 0) return cudaSuccess;
  sf_f64_kernel<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(pats, pattern);
  return cudaGetLastError();
}

cudaError_t launch_spectrum_combine(const SfPattern *pats, int pattern0, int S, const double *weight, float *F,
                                    float *I, long long npix, cudaStream_t st) {
  if (npix <= 0) return cudaSuccess;
  sf_spectrum_combine_kernel<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(pats, pattern0, S, weight, (float2 *)F, I,
                                                                            npix);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const SfPattern *pats, int pattern0, int npat, long long max_npix, cudaStream_t st) {
  if (max_npix <= 0 || npat <= 0) return cudaSuccess;
  for (int p0 = 0; p0 < npat; p0 += 65535) {
    const int n = npat - p0 < 65535 ? npat - p0 : 65535;
    dim3 grid((unsigned)((max_npix + 255) / 256), (unsigned)n);
    sf_finalize_kernel<<<grid, 256, 0, st>>>(pats, pattern0 + p0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_ewald(int nx, int ny, double width, double height, double distance, double cx, double cy,
                         double wavelength, int spherical, float *out32, double *out64, cudaStream_t st) {
  const long long n = (long long)nx * ny;
  if (n <= 0) return cudaSuccess;
  const double ewald = 1.0 / wavelength;
  // the reference forms the pixel pitch as a float quotient (src/diffraction.c:259-260)
  const double px_size = (double)((float)width / nx);
  const double py_size = (double)((float)height / ny);
  const double fpx = 2 * sin(atan(px_size / distance) / 2) / wavelength;
  const double fpy = 2 * sin(atan(py_size / distance) / 2) / wavelength;
  ewald_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nx, ny, width, height, distance, cx, cy, ewald, spherical,
                                                           fpx, fpy, px_size, py_size, out32, out64);
  return cudaGetLastError();
}

cudaError_t launch_crystal(long long npix, const float *hkl, const double cell[9], int na, int nb, int nc, float *F,
                           float *I, cudaStream_t st) {
  if (npix <= 0) return cudaSuccess;
  crystal_kernel<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(npix, hkl, cell[0], cell[1], cell[2], cell[3], cell[4],
                                                                cell[5], cell[6], cell[7], cell[8], na, nb, nc,
                                                                (float2 *)F, I);
  return cudaGetLastError();
}

// Largest |q[2m+1] - q[2m]| over the pixel pairs of a q set (float or FP64
// list), as the bits of a non-negative double (which order like integers).
// Block-wide maximum of a non-negative double (256 threads), then one atomic
// per block on its bits: a million same-address atomics would serialise.
__device__ __forceinline__ void block_max_to(double v, unsigned long long *out) {
  __shared__ double wmax[8];
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = wmax[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, wmax[w]);
    atomicMax(out, (unsigned long long)__double_as_longlong(m));
  }
  __syncthreads();
}

// Neighbour steps of one quad of pixels 4m .. 4m+3 (the pair and quad
// forms' admission tests): st[0] = largest |q[2i+1] - q[2i]| of its two pairs,
// st[1] = largest |q - q_a| over its one-pixel neighbours of the anchor q_a
// (q[4m+1], or q[4m] where that is the quad's only pixel), st[2] = |q[4m+3] - q_a|.
__device__ __forceinline__ void quad_steps(const float *__restrict__ hkl, const double *__restrict__ q64,
                                           long long npix, long long m, double st[3]) {
  st[0] = st[1] = st[2] = 0.0;
  const long long qb = 4 * m;
  double q[4][3];
  const int n = (int)(npix - qb < 4 ? npix - qb : 4);
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) q[i][c] = hkl ? (double)hkl[3 * (qb + i) + c] : q64[3 * (qb + i) + c];
  auto dist = [&](int a, int b) {
    const double d0 = q[b][0] - q[a][0], d1 = q[b][1] - q[a][1], d2 = q[b][2] - q[a][2];
    return sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  };
  if (n >= 2) st[0] = dist(0, 1), st[1] = dist(1, 0);
  if (n >= 3) st[1] = fmax(st[1], dist(1, 2));
  if (n >= 4) st[0] = fmax(st[0], dist(2, 3)), st[2] = dist(1, 3);
}

__global__ void __launch_bounds__(256) qset_steps_kernel(const float *__restrict__ hkl, const double *__restrict__ q64,
                                                         long long npix, unsigned long long *__restrict__ out) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double st[3] = {0.0, 0.0, 0.0};
  if (4 * m < npix) quad_steps(hkl, q64, npix, m, st);
  block_max_to(st[0], out);
  block_max_to(st[1], out + 1);
  block_max_to(st[2], out + 2);
}

cudaError_t qset_steps(const float *hkl, const double *q64, long long npix, double steps[3]) {
  steps[0] = steps[1] = steps[2] = 0.0;
  if (npix < 2) return cudaSuccess;
  unsigned long long *d = nullptr, h[3] = {0, 0, 0};
  cudaError_t e = cudaMalloc(&d, sizeof(h));
  if (e != cudaSuccess) return e;
  if ((e = cudaMemset(d, 0, sizeof(h))) == cudaSuccess) {
    const long long quads = (npix + 3) / 4;
    qset_steps_kernel<<<(unsigned)((quads + 255) / 256), 256>>>(hkl, q64, npix, d);
    if ((e = cudaGetLastError()) == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (e == cudaSuccess) memcpy(steps, h, sizeof(h));
  return e;
}

// q <- R q on a float HKL list with the operations of the reference's
// apply_orientation_to_HKL_list loop (src/diffraction.c:300-323 through
// sp_matrix_vector_prod): per row acc = 0, then acc += R[r][c] * v[c] for
// c = 0, 1, 2, each product and sum rounded to float (no contraction), so the
// device list is bit-identical to the host loop's.
__global__ void rotate_hkl_kernel(long long n, float r0, float r1, float r2, float r3, float r4, float r5, float r6,
                                  float r7, float r8, float *__restrict__ hkl) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float v0 = hkl[3 * i], v1 = hkl[3 * i + 1], v2 = hkl[3 * i + 2];
  const float R[9] = {r0, r1, r2, r3, r4, r5, r6, r7, r8};
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    float acc = 0.0f;
    acc = __fadd_rn(acc, __fmul_rn(R[3 * r], v0));
    acc = __fadd_rn(acc, __fmul_rn(R[3 * r + 1], v1));
    acc = __fadd_rn(acc, __fmul_rn(R[3 * r + 2], v2));
    hkl[3 * i + r] = acc;
  }
}

cudaError_t launch_rotate_hkl(long long n, const float R[9], float *hkl, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  rotate_hkl_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, R[0], R[1], R[2], R[3], R[4], R[5], R[6], R[7],
                                                                R[8], hkl);
  return cudaGetLastError();
}

// Largest |q| of a float HKL list and its neighbour steps (qset_steps), as
// the bits of non-negative doubles (which order like integers) in out[0..3].
__global__ void __launch_bounds__(256) qset_stats_kernel(const float *__restrict__ hkl, long long npix,
                                                         unsigned long long *__restrict__ out) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double qq = 0.0, st[3] = {0.0, 0.0, 0.0};
  for (long long i = 4 * m; i < 4 * m + 4 && i < npix; ++i) {
    const double a = hkl[3 * i], b = hkl[3 * i + 1], c = hkl[3 * i + 2];
    qq = fmax(qq, a * a + b * b + c * c);
  }
  if (4 * m < npix) quad_steps(hkl, nullptr, npix, m, st);
  block_max_to(qq, out);
  block_max_to(st[0], out + 1);
  block_max_to(st[1], out + 2);
  block_max_to(st[2], out + 3);
}

cudaError_t qset_stats(const float *hkl, long long npix, unsigned long long *scratch4, double *qmax, double steps[3],
                       cudaStream_t st) {
  *qmax = steps[0] = steps[1] = steps[2] = 0.0;
  if (npix <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(scratch4, 0, 4 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  const long long quads = (npix + 3) / 4;
  qset_stats_kernel<<<(unsigned)((quads + 255) / 256), 256, 0, st>>>(hkl, npix, scratch4);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  unsigned long long h[4] = {0, 0, 0, 0};
  if ((e = cudaMemcpyAsync(h, scratch4, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  double v[4];
  memcpy(v, h, sizeof(v));
  *qmax = sqrt(v[0]);
  for (int k = 0; k < 3; ++k) steps[k] = v[k + 1];
  return cudaSuccess;
}

cudaError_t launch_volume(int nx, int ny, int nz, float width, float height, float depth, float distance, float cx,
                          float cy, float cz, float wavelength, float *out32, cudaStream_t st) {
  const long long n = (long long)nx * ny * nz;
  if (n <= 0) return cudaSuccess;
  // 1.0 / (distance * wavelength): a float product, then a double quotient (src/diffraction.c:334)
  const double r2r = 1.0 / (double)(distance * wavelength);
  volume_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nx, ny, nz, width, height, depth, cx, cy, cz, r2r, out32);
  return cudaGetLastError();
}

cudaError_t launch_atoms_update(float4 *atoms, float4 *atoms2, AtomD *atomsd, const int *perm, int n_padded, const float *pos32,
                                const double *pos64, const float *occ, const float *bfac, const float *wbase,
                                const double c[3], float dr, float inv_dr, double rbound, int *range_err,
                                cudaStream_t st) {
  if (n_padded <= 0) return cudaSuccess;
  atoms_update_kernel<<<(n_padded + 255) / 256, 256, 0, st>>>(atoms, atoms2, atomsd, perm, n_padded, pos32, pos64, occ, bfac, wbase,
                                                             c[0], c[1], c[2], dr, inv_dr, rbound, range_err);
  return cudaGetLastError();
}

}  // namespace spsim
