// spsim_b200_structure_factor_host_noalloc: the host-memory structure factor
// for callers that cannot allocate device memory while they run.  It takes the
// arguments of spsim_b200_structure_factor_host and runs the same kernels with
// the same arithmetic (atom records built on the device by atoms_build_kernel,
// the FP64-phase forms 2 and 3 of the FP32 forward chosen by the same rules as
// the untuned allocating call, the same phase-range limit of 2^48 cycles), but
// every byte of device scratch it needs (the caller's atoms and q, atom
// records, tile table, form factors, FP64 accumulator, F and I staging, work
// items) lives in one file-scope __device__ array of kNoAllocScratchBytes, and
// its host-side preparation in a file-scope host array: the call makes no
// cudaMalloc, cudaFree or heap allocation on its way through.
//
// The device array exists once per GPU that loads the library and is held
// until the process exits.  In host code the array's name is only a stand-in
// symbol, not a device address, so the first call on each device looks up
// that device's address with cudaGetSymbolAddress while the device is current
// and caches it; that first call on a device should come before any stream
// capture.  The cached address belongs to the device's primary context:
// cudaDeviceReset is not supported between calls (the address would be stale).
// Every call reuses the same array and so inherits the last call's contents:
// the accumulator, the work-queue head and the error word are cleared on
// every call.  Calls are serialised by a mutex and synchronise before
// returning; calls that overlapped on the GPU would race on the array.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/spsim_b200.h"
#include "atomsf_data.h"
#include "sf_kernels.cuh"

using namespace spsim;

// defined in capi.cu
void spsim_internal_atomsf_row(int Z, float out[9]);
int spsim_internal_fail(int status, const char *msg);

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;  // device scratch per GPU
constexpr size_t kNoAllocHostBytes = size_t(16) << 20;     // host staging
constexpr int kMaxDevices = 64;

std::mutex g_noalloc_mu;
void *g_scratch_addr[kMaxDevices] = {nullptr};

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
alignas(256) static unsigned char g_noalloc_host[kNoAllocHostBytes];

// The message is formatted once, into a local buffer, and handed to the
// library's thread-local error slot (spsim_b200_last_error).
static int noalloc_fail(int status, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
static int noalloc_fail(int status, const char *fmt, ...) {
  char msg[512];
  int n = snprintf(msg, sizeof(msg), "spsim_b200_structure_factor_host_noalloc: ");
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg + n, sizeof(msg) - n, fmt, ap);
  va_end(ap);
  return spsim_internal_fail(status, msg);
}

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

static int ceil_log2(double x) {  // smallest e with x < 2^e (-80 for x <= 0)
  if (!(x > 0)) return -80;
  int e = (int)std::floor(std::log2(x)) + 1;
  while (std::ldexp(1.0, e) <= x) ++e;
  while (e > -80 && std::ldexp(1.0, e - 1) > x) --e;
  return e;
}

#define NA_CUDA(expr)                                                                   \
  do {                                                                                  \
    cudaError_t _e = (expr);                                                            \
    if (_e != cudaSuccess) return noalloc_fail(SPSIM_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(_e)); \
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
    return noalloc_fail(SPSIM_ERR_INVALID_ARG, "unknown precision %d", precision);
  for (int j = 0; j < natoms; ++j)
    if (Z[j] < 0 || Z[j] >= SPSIM_B200_N_ELEMENTS)
      return noalloc_fail(SPSIM_ERR_INVALID_ARG, "atom %d: atomic number %d outside [0,%d)", j, Z[j],
                          SPSIM_B200_N_ELEMENTS);

  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  int ndev = 0, dev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return noalloc_fail(SPSIM_ERR_NO_DEVICE, "no CUDA device");
  }
  NA_CUDA(cudaGetDevice(&dev));
  if (dev >= kMaxDevices) return noalloc_fail(SPSIM_ERR_UNSUPPORTED, "device %d beyond the scratch table", dev);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    NA_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));  // this device's address of the array
    g_scratch_addr[dev] = p;
  }
  unsigned char *dbase = (unsigned char *)g_scratch_addr[dev];

  // ---- molecule: kept atoms, centre, bound, element segments (as spsim_b200_molecule_create)
  int count[SPSIM_B200_N_ELEMENTS] = {0};
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  int n_kept = 0;
  for (int j = 0; j < natoms; ++j) {
    if (!Z[j]) continue;  // src/diffraction.c:830-832
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
    for (int k = 0; k < 3; ++k) {
      const double d = (double)pos[3 * j + k] - c[k];
      d2 += d * d;
    }
    rmax = std::max(rmax, std::sqrt(d2));
  }
  const double rbound = rmax + std::max(0.05 * rmax, 5e-10);
  const int kr = 11;
  const int er = ceil_log2(rbound);
  const float dr = (float)std::ldexp(1.0, er - kr), inv_dr = (float)std::ldexp(1.0, kr - er);
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

  // ---- q set: largest |q| and the neighbour steps (as the q-set handles
  // measure them): of pixel pairs 2m, 2m+1, and from each quad's anchor 4m+1
  // (4m where that is the quad's only pixel) to its one-pixel neighbours 4m,
  // 4m+2 and to 4m+3
  double qm2 = 0, pair2 = 0, quad1 = 0, quad2 = 0;
  auto d2 = [&](long long i, long long j) {
    double s2 = 0;
    for (int k = 0; k < 3; ++k) {
      const double d = (double)hkl[3 * j + k] - (double)hkl[3 * i + k];
      s2 += d * d;
    }
    return s2;
  };
  for (long long i = 0; i < npix; ++i) {
    const double a = hkl[3 * i], b = hkl[3 * i + 1], cc = hkl[3 * i + 2];
    qm2 = std::max(qm2, a * a + b * b + cc * cc);
    if (i & 1) pair2 = std::max(pair2, d2(i - 1, i));
    const long long qb = i & ~3LL;
    if ((i & 3) == 0 && i + 1 < npix) quad1 = std::max(quad1, d2(i + 1, i));
    if ((i & 3) == 2) quad1 = std::max(quad1, d2(qb + 1, i));
    if ((i & 3) == 3) quad2 = std::max(quad2, d2(qb + 1, i));
  }
  const double qmax = std::sqrt(qm2);

  // ---- kernel form: the untuned allocating call's choice.  The
  // neighbour-quad form (4, 8 pixels per thread) where every one-pixel step
  // from a quad's anchor is within 1/8 cycle and every two-pixel step within
  // 0.16, else (FP32 only) the neighbour-pair form (3) where every pair's step
  // is within 1/8 cycle, else the FP64-phase form (2); forms 2 and 3 with 8
  // pixels per thread from 2^20 pixels, 4 below; the fixed-point phase word
  // below 2^17 cycles, FP64 rounding up to 2^48.
  const bool fp32 = precision != SPSIM_PREC_FP64;
  const int mode = precision == SPSIM_PREC_F32_FAST ? PREC_MODE_MUFU : PREC_MODE_POLY;
  const double s_pair = std::sqrt(pair2) * rbound, s_q1 = std::sqrt(quad1) * rbound, s_q2 = std::sqrt(quad2) * rbound;
  int form = 2;
  bool narrow = false;
  if (fp32 && s_q1 <= (1.0 / 8) * (1.0 - 1e-9) && s_q2 <= 0.16 * (1.0 - 1e-9)) {
    form = 4;
    narrow = s_q1 <= 0.07 * (1.0 - 1e-6);
  } else if (precision == SPSIM_PREC_F32 && s_pair <= (1.0 / 8) * (1.0 - 1e-9)) {
    form = 3;
    narrow = s_pair <= 0.07 * (1.0 - 1e-6);
  }
  const int NT = 128, P = (form == 4 || npix >= (1LL << 20)) ? 8 : 4;
  const bool perb = bfac != nullptr;
  const double qr = qmax * rbound;
  const bool fixw = qr < std::ldexp(1.0, 17);
  if (fp32 && n_kept > 0 && npix > 0 && qr >= std::ldexp(1.0, 48))
    return noalloc_fail(SPSIM_ERR_RANGE, "|q|max*|r|max = %.3g cycles exceeds 2^48", qr);

  // ---- work items: pixel tile x atom-tile range
  const long long tile_pix = (long long)NT * P;
  const long long n_ptile = (npix + tile_pix - 1) / tile_pix;
  int num_sms = 148;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
  const int occ_blocks = fp32 ? std::max(1, sf_f32_occupancy(mode, NT, P, form, perb, fixw, narrow)) : 1;
  const long long slots = (long long)num_sms * occ_blocks;
  int split = 1;
  if (n_ptile > 0 && n_tiles > 0 && n_ptile < 6 * slots)
    split = (int)std::min<long long>((6 * slots + n_ptile - 1) / n_ptile, n_tiles);
  split = std::max(1, std::min(split, std::max(1, n_tiles / 2)));
  const long long n_items = (fp32 && n_tiles > 0) ? n_ptile * split : 0;

  // ---- host staging layout (one upload); the device scratch starts with the same blocks
  size_t ho = 0;
  auto hput = [&](size_t bytes) {
    const size_t o = ho;
    ho = align256(ho + bytes);
    return o;
  };
  const size_t na = (size_t)std::max(n_pad, 1), nin = (size_t)std::max(natoms, 1);
  const size_t np = (size_t)std::max<int64_t>(npix, 1);
  const size_t h_perm = hput(na * sizeof(int));
  const size_t h_wbase = hput(na * sizeof(float));
  const size_t h_tiles = hput((size_t)std::max(n_tiles, 1) * sizeof(TileDesc));
  const size_t h_coeffs = hput((size_t)std::max(n_elem, 1) * 9 * sizeof(float));
  const size_t h_pat = hput(sizeof(SfPattern));
  const size_t h_items = hput((size_t)std::max<long long>(n_items, 1) * sizeof(WorkItem));
  const size_t host_need = ho;
  size_t dof = host_need;
  auto dput = [&](size_t bytes) {
    const size_t o = dof;
    dof = align256(dof + bytes);
    return o;
  };
  const size_t d_pos = dput(3 * nin * sizeof(float));
  const size_t d_occ = dput(nin * sizeof(float));
  const size_t d_bfac = dput(nin * sizeof(float));
  const size_t d_atoms = dput(2 * na * sizeof(float4));
  const size_t d_atoms2 = dput(4 * na * sizeof(float4));
  const size_t d_atomsd = dput(na * sizeof(AtomD));
  const size_t d_hkl = dput(3 * np * sizeof(float));
  const size_t d_acc = dput(np * sizeof(double2));
  const size_t d_ff = dput((size_t)std::max(n_elem, 1) * np * sizeof(double));
  const size_t d_F = dput(2 * np * sizeof(float));
  const size_t d_I = dput(np * sizeof(float));
  const size_t d_flags = dput(64);
  const size_t dev_need = dof;
  if (host_need > kNoAllocHostBytes || dev_need > kNoAllocScratchBytes)
    return noalloc_fail(SPSIM_ERR_INVALID_ARG,
                        "%d atoms and %lld pixels need %zu bytes of device scratch (limit %zu) and %zu bytes of "
                        "host staging (limit %zu)",
                        natoms, (long long)npix, dev_need, kNoAllocScratchBytes, host_need, kNoAllocHostBytes);

  int *perm = (int *)(g_noalloc_host + h_perm);
  float *wbase = (float *)(g_noalloc_host + h_wbase);
  TileDesc *tiles = (TileDesc *)(g_noalloc_host + h_tiles);
  float *coeffs = (float *)(g_noalloc_host + h_coeffs);
  SfPattern *pat = (SfPattern *)(g_noalloc_host + h_pat);
  WorkItem *items = (WorkItem *)(g_noalloc_host + h_items);
  for (size_t j = 0; j < na; ++j) {
    perm[j] = -1;
    wbase[j] = 0.0f;
  }
  {
    int fill[SPSIM_B200_N_ELEMENTS] = {0};
    for (int j = 0; j < natoms; ++j) {
      if (!Z[j]) continue;
      const int e = slot[Z[j]];
      const int idx = seg[e] + fill[e]++;
      perm[idx] = j;
      // weight sqrt(illumination) (src/diffraction.c:223-235, :834), float like the reference
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
      wbase[idx] = w;
    }
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
  {
    long long w = 0;
    for (long long t = 0; t < n_ptile && n_items > 0; ++t)
      for (int s = 0; s < split; ++s) {
        items[w].pattern = 0;
        items[w].pixel_tile = (int)t;
        items[w].k0 = (int)((long long)n_tiles * s / split);
        items[w].k1 = (int)((long long)n_tiles * (s + 1) / split);
        ++w;
      }
  }
  const int eq = ceil_log2(std::max(qmax, 1e-300));
  memset(pat, 0, sizeof(SfPattern));
  pat->atoms = (const float4 *)(dbase + d_atoms);
  pat->atoms2 = (const float4 *)(dbase + d_atoms2);
  pat->atomsd = (const AtomD *)(dbase + d_atomsd);
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
  pat->dq = (float)std::ldexp(1.0, eq - (22 - kr));
  pat->inv_dq = (float)std::ldexp(1.0, (22 - kr) - eq);
  pat->acc = (double2 *)(dbase + d_acc);
  pat->F = F_host ? (float2 *)(dbase + d_F) : nullptr;
  pat->I = I_host ? (float *)(dbase + d_I) : nullptr;

  // ---- device work on the legacy default stream, all inside the scratch array
  cudaStream_t st = nullptr;
  NA_CUDA(cudaMemcpyAsync(dbase, g_noalloc_host, host_need, cudaMemcpyHostToDevice, st));
  if (natoms) {
    NA_CUDA(cudaMemcpyAsync(dbase + d_pos, pos, 3 * (size_t)natoms * sizeof(float), cudaMemcpyHostToDevice, st));
    if (occ) NA_CUDA(cudaMemcpyAsync(dbase + d_occ, occ, (size_t)natoms * sizeof(float), cudaMemcpyHostToDevice, st));
    if (bfac)
      NA_CUDA(cudaMemcpyAsync(dbase + d_bfac, bfac, (size_t)natoms * sizeof(float), cudaMemcpyHostToDevice, st));
  }
  if (npix) NA_CUDA(cudaMemcpyAsync(dbase + d_hkl, hkl, 3 * (size_t)npix * sizeof(float), cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemsetAsync(dbase + d_acc, 0, np * sizeof(double2), st));
  NA_CUDA(cudaMemsetAsync(dbase + d_flags, 0, 64, st));  // work-queue head and error word
  NA_CUDA(launch_atoms_build<float>((float4 *)(dbase + d_atoms), (float4 *)(dbase + d_atoms2),
                                    (AtomD *)(dbase + d_atomsd), (const int *)(dbase + h_perm), n_pad,
                                    (const float *)(dbase + d_pos), occ ? (const float *)(dbase + d_occ) : nullptr,
                                    bfac ? (const float *)(dbase + d_bfac) : nullptr,
                                    (const float *)(dbase + h_wbase), c, (double)dr, (double)inv_dr, st));
  NA_CUDA(launch_ff_table(pat->hkl, nullptr, npix, n_elem, (const float *)(dbase + h_coeffs), (double)B, delta_atoms,
                          (double *)(dbase + d_ff), st));
  const SfPattern *dpat = (const SfPattern *)(dbase + h_pat);
  int *dflags = (int *)(dbase + d_flags);
  if (!fp32) {
    NA_CUDA(launch_sf_f64(dpat, 0, npix, st));
  } else if (n_items > 0) {
    NA_CUDA(launch_sf_f32(mode, NT, P, form, perb, dpat, (const WorkItem *)(dbase + h_items), (int)n_items, dflags,
                          dflags + 4, (int)std::min<long long>(n_items, slots), st, fixw, narrow));
  }
  NA_CUDA(launch_finalize(dpat, 0, 1, npix, st));
  if (F_host && npix)
    NA_CUDA(cudaMemcpyAsync(F_host, dbase + d_F, 2 * (size_t)npix * sizeof(float), cudaMemcpyDeviceToHost, st));
  if (I_host && npix)
    NA_CUDA(cudaMemcpyAsync(I_host, dbase + d_I, (size_t)npix * sizeof(float), cudaMemcpyDeviceToHost, st));
  int flags[8] = {0};
  NA_CUDA(cudaMemcpyAsync(flags, dflags, sizeof(flags), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaStreamSynchronize(st));
  if (flags[4]) return noalloc_fail(SPSIM_ERR_TIMEOUT, "an atom-tile copy did not complete in time");
  return SPSIM_OK;
}
