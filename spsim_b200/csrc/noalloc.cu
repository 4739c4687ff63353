// spsim_b200_structure_factor_host_noalloc: the host-memory structure factor
// without any allocation.  Same arguments and results as
// spsim_b200_structure_factor_host; every byte of device scratch it needs
// (atom records, tile table, pixel q, form factors, FP64 accumulator, F and I
// staging, work items) lives in one file-scope __device__ array of
// kNoAllocScratchBytes, and the host-side preparation lives in a file-scope
// host array, so the call makes no cudaMalloc / cudaFree and no heap
// allocation on its way through.
//
// The device array exists once per GPU that loads the library and is held until
// the process exits.  Host code cannot pass the array's name to a kernel (in host
// code it is only a stand-in symbol), so on the first call on each device the
// device address is looked up with cudaGetSymbolAddress while that device is
// current and cached; that first call on a device should come before any stream
// capture.  Every call reuses the same array and so inherits the last call's
// contents: the accumulator and the work-queue head are cleared on every call.
// Calls are serialised by a mutex and synchronise before returning; two calls
// that overlapped on the GPU would race on the array.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/spsim_b200.h"
#include "atomsf_data.h"
#include "sf_kernels.cuh"

using namespace spsim;

// defined in capi.cu
void spsim_internal_atomsf_row(int Z, float out[9]);

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;   // device scratch per GPU
constexpr size_t kNoAllocHostBytes = size_t(48) << 20;      // host staging
constexpr int kMaxDevices = 64;

std::mutex g_noalloc_mu;
void *g_scratch_addr[kMaxDevices] = {nullptr};
char g_noalloc_err[512];

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
alignas(256) static unsigned char g_noalloc_host[kNoAllocHostBytes];

static int noalloc_fail(int status, const char *msg) {
  snprintf(g_noalloc_err, sizeof(g_noalloc_err), "spsim_b200_structure_factor_host_noalloc: %s", msg);
  fprintf(stderr, "%s\n", g_noalloc_err);
  return status;
}

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

#define NA_CUDA(expr)                                                                   \
  do {                                                                                  \
    cudaError_t _e = (expr);                                                            \
    if (_e != cudaSuccess) {                                                            \
      snprintf(g_noalloc_err, sizeof(g_noalloc_err), "%s: %s", #expr, cudaGetErrorString(_e)); \
      return noalloc_fail(SPSIM_ERR_CUDA, g_noalloc_err);                               \
    }                                                                                   \
  } while (0)

extern "C" int spsim_b200_structure_factor_host_noalloc(int natoms, const int32_t *Z, const float *pos,
                                                        const float *occ, const float *bfac, float B,
                                                        int delta_atoms, const float *beam, int64_t npix,
                                                        const float *hkl, int precision, float *F_host,
                                                        float *I_host) {
  if (natoms < 0 || npix < 0) return noalloc_fail(SPSIM_ERR_INVALID_ARG, "negative size");
  if ((natoms > 0 && (!Z || !pos)) || (npix > 0 && !hkl))
    return noalloc_fail(SPSIM_ERR_INVALID_ARG, "NULL input array");
  if (precision < SPSIM_PREC_FP64 || precision > SPSIM_PREC_F32_FAST)
    return noalloc_fail(SPSIM_ERR_INVALID_ARG, "unknown precision");
  for (int j = 0; j < natoms; ++j)
    if (Z[j] < 0 || Z[j] >= SPSIM_B200_N_ELEMENTS) return noalloc_fail(SPSIM_ERR_INVALID_ARG, "atomic number out of range");

  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  int ndev = 0, dev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return noalloc_fail(SPSIM_ERR_NO_DEVICE, "no CUDA device");
  }
  NA_CUDA(cudaGetDevice(&dev));
  if (dev >= kMaxDevices) return noalloc_fail(SPSIM_ERR_UNSUPPORTED, "device index beyond the scratch table");
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    NA_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));  // the device's own address of the array
    g_scratch_addr[dev] = p;
  }
  unsigned char *dbase = (unsigned char *)g_scratch_addr[dev];

  // ---- host preparation into the static staging area
  int count[SPSIM_B200_N_ELEMENTS] = {0};
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  int n_kept = 0;
  for (int j = 0; j < natoms; ++j) {
    if (!Z[j]) continue;
    ++count[Z[j]];
    ++n_kept;
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], (double)pos[3 * j + k]);
      hi[k] = std::max(hi[k], (double)pos[3 * j + k]);
    }
  }
  double c[3] = {0, 0, 0};
  if (n_kept)
    for (int k = 0; k < 3; ++k) c[k] = 0.5 * (lo[k] + hi[k]);
  double rmax = 0;
  for (int j = 0; j < natoms; ++j) {
    if (!Z[j]) continue;
    double d2 = 0;
    for (int k = 0; k < 3; ++k) d2 += ((double)pos[3 * j + k] - c[k]) * ((double)pos[3 * j + k] - c[k]);
    rmax = std::max(rmax, std::sqrt(d2));
  }
  const double rbound = rmax + std::max(0.05 * rmax, 5e-10);
  int er = -80;
  if (rbound > 0) {
    er = (int)std::floor(std::log2(rbound)) + 1;
    while (std::ldexp(1.0, er) <= rbound) ++er;
    while (std::ldexp(1.0, er - 1) > rbound) --er;
  }
  const int kr = 11;
  const double dr = std::ldexp(1.0, er - kr), inv_dr = std::ldexp(1.0, kr - er);
  int elem_Z[SPSIM_B200_N_ELEMENTS], seg[SPSIM_B200_N_ELEMENTS + 1], slot[SPSIM_B200_N_ELEMENTS];
  int n_elem = 0, n_pad = 0;
  for (int z = 1; z < SPSIM_B200_N_ELEMENTS; ++z) {
    if (!count[z]) continue;
    elem_Z[n_elem] = z;
    slot[z] = n_elem;
    seg[n_elem++] = n_pad;
    n_pad += (count[z] + ATOM_GROUP - 1) / ATOM_GROUP * ATOM_GROUP;
  }
  seg[n_elem] = n_pad;
  int n_tiles = 0;
  for (int e = 0; e < n_elem; ++e) n_tiles += (seg[e + 1] - seg[e] + TILE_ATOMS - 1) / TILE_ATOMS;

  // work items for the FP32 kernels (pixel tile x atom-tile range, cost-sorted by construction)
  const int NT = 128, P = 4, PACKED = 1;
  const long long tile_pix = (long long)NT * P;
  const long long n_ptile = (npix + tile_pix - 1) / tile_pix;
  int num_sms = 148, occ_blocks = 1;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
  const bool perb = bfac != nullptr;
  const int mode = precision == SPSIM_PREC_F32_FAST ? PREC_MODE_MUFU : PREC_MODE_POLY;
  if (precision != SPSIM_PREC_FP64) occ_blocks = std::max(1, sf_f32_occupancy(mode, NT, P, PACKED, perb));
  const long long slots = (long long)num_sms * occ_blocks;
  int split = 1;
  if (n_ptile > 0 && n_tiles > 0 && n_ptile < 6 * slots)
    split = (int)std::min<long long>((6 * slots + n_ptile - 1) / n_ptile, n_tiles);
  split = std::max(1, std::min(split, std::max(1, n_tiles / 2)));
  const long long n_items = (precision != SPSIM_PREC_FP64 && n_tiles > 0) ? n_ptile * split : 0;

  // host staging layout
  size_t ho = 0;
  auto hput = [&](size_t bytes) {
    size_t o = ho;
    ho = align256(ho + bytes);
    return o;
  };
  const size_t h_atoms = hput(2 * (size_t)std::max(n_pad, 1) * sizeof(float4));
  const size_t h_atoms2 = hput(4 * (size_t)std::max(n_pad, 1) * sizeof(float4));
  const size_t h_tiles = hput((size_t)std::max(n_tiles, 1) * sizeof(TileDesc));
  const size_t h_coeffs = hput((size_t)std::max(n_elem, 1) * 9 * sizeof(float));
  const size_t h_pat = hput(sizeof(SfPattern));
  const size_t h_items = hput((size_t)std::max<long long>(n_items, 1) * sizeof(WorkItem));
  const size_t host_need = ho;
  // device scratch layout: the same blocks, then the per-pixel arrays
  size_t dof = host_need;
  auto dput = [&](size_t bytes) {
    size_t o = dof;
    dof = align256(dof + bytes);
    return o;
  };
  const size_t d_hkl = dput(3 * (size_t)std::max<int64_t>(npix, 1) * sizeof(float));
  const size_t d_acc = dput((size_t)std::max<int64_t>(npix, 1) * sizeof(double2));
  const size_t d_ff = dput((size_t)std::max(n_elem, 1) * (size_t)std::max<int64_t>(npix, 1) * sizeof(double));
  const size_t d_F = dput(2 * (size_t)std::max<int64_t>(npix, 1) * sizeof(float));
  const size_t d_I = dput((size_t)std::max<int64_t>(npix, 1) * sizeof(float));
  const size_t d_flags = dput(64);
  const size_t dev_need = dof;
  if (host_need > kNoAllocHostBytes || dev_need > kNoAllocScratchBytes) {
    snprintf(g_noalloc_err, sizeof(g_noalloc_err),
             "needs %zu bytes of device scratch (limit %zu) and %zu of host staging (limit %zu) for %d atoms "
             "and %lld pixels",
             dev_need, kNoAllocScratchBytes, host_need, kNoAllocHostBytes, natoms, (long long)npix);
    return noalloc_fail(SPSIM_ERR_INVALID_ARG, g_noalloc_err);
  }
  float4 *recs = (float4 *)(g_noalloc_host + h_atoms);
  float4 *recs2 = (float4 *)(g_noalloc_host + h_atoms2);
  TileDesc *tiles = (TileDesc *)(g_noalloc_host + h_tiles);
  float *coeffs = (float *)(g_noalloc_host + h_coeffs);
  SfPattern *pat = (SfPattern *)(g_noalloc_host + h_pat);
  WorkItem *items = (WorkItem *)(g_noalloc_host + h_items);
  memset(recs, 0, 2 * (size_t)std::max(n_pad, 1) * sizeof(float4));
  {
    int fill[SPSIM_B200_N_ELEMENTS] = {0};
    for (int j = 0; j < natoms; ++j) {
      if (!Z[j]) continue;
      const int e = slot[Z[j]];
      const int idx = seg[e] + fill[e]++;
      float w = 1.0f;
      if (!delta_atoms) {
        float illum = 1.0f;
        if (beam && beam[0] != 0.0f) {
          const double dx = (double)pos[3 * j] - (double)beam[1];
          const double dy = (double)pos[3 * j + 1] - (double)beam[2];
          const double sigma = (double)beam[0] / 2.355;
          illum = (float)std::exp(-(dx * dx + dy * dy) / (2 * sigma * sigma));
        }
        w = (float)std::sqrt((double)illum);
      }
      const float o = occ ? occ[j] : 1.0f;
      double r[3];
      for (int k = 0; k < 3; ++k) r[k] = (double)pos[3 * j + k] - c[k];
      const double hx = std::rint(r[0] * inv_dr) * dr, hy = std::rint(r[1] * inv_dr) * dr,
                   hz = std::rint(r[2] * inv_dr) * dr;
      recs[2 * idx] = make_float4((float)hx, (float)hy, (float)hz, o * w);
      recs[2 * idx + 1] = make_float4((float)(r[0] - hx), (float)(r[1] - hy), (float)(r[2] - hz), bfac ? bfac[j] : 0.0f);
    }
  }
  for (int j = 0; j < n_pad; ++j) {
    const float4 a0 = recs[2 * j], a1 = recs[2 * j + 1];
    recs2[4 * j] = make_float4(a0.x, a0.x, a0.y, a0.y);
    recs2[4 * j + 1] = make_float4(a0.z, a0.z, a0.w, a0.w);
    recs2[4 * j + 2] = make_float4(a1.x, a1.x, a1.y, a1.y);
    recs2[4 * j + 3] = make_float4(a1.z, a1.z, a1.w, a1.w);
  }
  {
    int t = 0;
    for (int e = 0; e < n_elem; ++e)
      for (int a = seg[e]; a < seg[e + 1]; a += TILE_ATOMS) {
        tiles[t].atom_begin = a;
        tiles[t].count = std::min(TILE_ATOMS, seg[e + 1] - a);
        tiles[t].elem = e;
        tiles[t].last = (a + TILE_ATOMS >= seg[e + 1]) ? 1 : 0;
        ++t;
      }
  }
  for (int e = 0; e < n_elem; ++e) spsim_internal_atomsf_row(elem_Z[e], coeffs + 9 * e);

  // phase grid of the pixel side and the compensated-kernel domain checks
  double qm2 = 0;
  for (long long i = 0; i < npix; ++i) {
    const double a = hkl[3 * i], b = hkl[3 * i + 1], cc = hkl[3 * i + 2];
    qm2 = std::max(qm2, a * a + b * b + cc * cc);
  }
  const double qmax = std::sqrt(qm2);
  int eq = -80;
  if (qmax > 0) {
    eq = (int)std::floor(std::log2(qmax)) + 1;
    while (std::ldexp(1.0, eq) <= qmax) ++eq;
    while (std::ldexp(1.0, eq - 1) > qmax) --eq;
  }
  const float dq = (float)std::ldexp(1.0, eq - (22 - kr)), inv_dq = (float)std::ldexp(1.0, (22 - kr) - eq);
  if (precision != SPSIM_PREC_FP64 && n_kept > 0 && npix > 0) {
    const double cmax = 0.8660254037844386 * (qmax * dr + (double)dq * (rbound + dr));
    const double lim = precision == SPSIM_PREC_F32 ? 1.0 / 16 : 0.25;
    if (qmax * rbound >= std::ldexp(1.0, 19) || cmax > lim)
      return noalloc_fail(SPSIM_ERR_RANGE, "phase range outside the FP32 kernel's domain; use SPSIM_PREC_FP64");
  }
  {
    long long w = 0;
    for (long long t = 0; t < n_ptile && precision != SPSIM_PREC_FP64 && n_tiles > 0; ++t)
      for (int s = 0; s < split; ++s) {
        items[w].pattern = 0;
        items[w].pixel_tile = (int)t;
        items[w].k0 = (int)((long long)n_tiles * s / split);
        items[w].k1 = (int)((long long)n_tiles * (s + 1) / split);
        ++w;
      }
  }
  memset(pat, 0, sizeof(SfPattern));
  pat->atoms = (const float4 *)(dbase + h_atoms);
  pat->atoms2 = (const float4 *)(dbase + h_atoms2);
  pat->tiles = (const TileDesc *)(dbase + h_tiles);
  pat->n_tiles = n_tiles;
  pat->n_elem = n_elem;
  pat->per_atom_b = perb ? 1 : 0;
  pat->has_rot = 0;
  for (int k = 0; k < 9; ++k) pat->rot[k] = (k % 4 == 0) ? 1.0 : 0.0;
  pat->qscale = 1.0;
  pat->s2scale = 1.0;
  pat->ff = (const double *)(dbase + d_ff);
  pat->npix = npix;
  pat->hkl = (const float *)(dbase + d_hkl);
  pat->q64 = nullptr;
  for (int k = 0; k < 3; ++k) pat->center[k] = c[k];
  pat->dq = dq;
  pat->inv_dq = inv_dq;
  pat->acc = (double2 *)(dbase + d_acc);
  pat->F = F_host ? (float2 *)(dbase + d_F) : nullptr;
  pat->I = I_host ? (float *)(dbase + d_I) : nullptr;

  // ---- device work on the legacy default stream, all inside the scratch array
  cudaStream_t st = nullptr;
  NA_CUDA(cudaMemcpyAsync(dbase, g_noalloc_host, host_need, cudaMemcpyHostToDevice, st));
  if (npix) NA_CUDA(cudaMemcpyAsync(dbase + d_hkl, hkl, 3 * (size_t)npix * sizeof(float), cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemsetAsync(dbase + d_acc, 0, (size_t)std::max<int64_t>(npix, 1) * sizeof(double2), st));
  NA_CUDA(cudaMemsetAsync(dbase + d_flags, 0, 64, st));  // work-queue head and error word
  NA_CUDA(launch_ff_table(pat->hkl, nullptr, npix, n_elem, (const float *)(dbase + h_coeffs), (double)B, delta_atoms,
                          (double *)(dbase + d_ff), st));
  const SfPattern *dpat = (const SfPattern *)(dbase + h_pat);
  int *dflags = (int *)(dbase + d_flags);
  if (precision == SPSIM_PREC_FP64) {
    NA_CUDA(launch_sf_f64(dpat, 0, npix, st));
  } else if (n_items > 0) {
    NA_CUDA(launch_sf_f32(mode, NT, P, PACKED, perb, dpat, (const WorkItem *)(dbase + h_items), (int)n_items,
                          dflags, dflags + 4, (int)std::min<long long>(n_items, slots), st));
  }
  NA_CUDA(launch_finalize(dpat, 0, 1, npix, st));
  if (F_host && npix) NA_CUDA(cudaMemcpyAsync(F_host, dbase + d_F, 2 * (size_t)npix * sizeof(float), cudaMemcpyDeviceToHost, st));
  if (I_host && npix) NA_CUDA(cudaMemcpyAsync(I_host, dbase + d_I, (size_t)npix * sizeof(float), cudaMemcpyDeviceToHost, st));
  int flags[8] = {0};
  NA_CUDA(cudaMemcpyAsync(flags, dflags, sizeof(flags), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaStreamSynchronize(st));
  if (flags[4]) return noalloc_fail(SPSIM_ERR_TIMEOUT, "an atom-tile copy did not complete in time");
  return SPSIM_OK;
}
