// C ABI of libspsim_b200.so: handles, planning, scheduling and launches.
// Declarations and contracts: include/spsim_b200.h.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/spsim_b200.h"
#include "atomsf_data.h"
#include "chain_kernels.cuh"
#include "adjoint_kernels.cuh"
#include "sf_kernels.cuh"
#include "nufft_kernels.cuh"


using namespace spsim;

// ---------------------------------------------------------------------------
// errors

static thread_local std::string g_last_error;

static int fail(int status, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

// Records a failure of the allocation-free entry point (noalloc.cu), so that
// spsim_b200_last_error() reports it like every other call's.
int spsim_internal_fail(int status, const char *msg) { return fail(status, "%s", msg); }

#define CUDA_TRY(expr)                                                                            \
  do {                                                                                            \
    cudaError_t _e = (expr);                                                                      \
    if (_e != cudaSuccess) return fail(SPSIM_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                                       __FILE__, __LINE__);                                       \
  } while (0)

extern "C" const char *spsim_b200_status_string(int s) {
  switch (s) {
    case SPSIM_OK: return "ok";
    case SPSIM_ERR_INVALID_ARG: return "invalid argument";
    case SPSIM_ERR_CUDA: return "CUDA error";
    case SPSIM_ERR_NO_DEVICE: return "no CUDA device";
    case SPSIM_ERR_OUT_OF_MEMORY: return "out of device memory";
    case SPSIM_ERR_RANGE: return "phase range outside the compensated FP32 kernel's domain";
    case SPSIM_ERR_TIMEOUT: return "a bounded device wait gave up";
    case SPSIM_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

extern "C" const char *spsim_b200_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *spsim_b200_version(void) { return "spsim_b200 0.1 (sm_100a)"; }

static std::mutex g_mu;  // serialises planning and workspace use

static int current_device(int *dev) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(SPSIM_ERR_NO_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
  }
  CUDA_TRY(cudaGetDevice(dev));
  return SPSIM_OK;
}

extern "C" int spsim_b200_device_count(int *count) {
  if (!count) return fail(SPSIM_ERR_INVALID_ARG, "count is NULL");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *count = n;
  return SPSIM_OK;
}

extern "C" int spsim_b200_init(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(SPSIM_ERR_NO_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
  }
  if (device < 0 || device >= n) return fail(SPSIM_ERR_INVALID_ARG, "device %d out of range [0,%d)", device, n);
  CUDA_TRY(cudaSetDevice(device));
  CUDA_TRY(cudaFree(nullptr));
  return SPSIM_OK;
}

// ---------------------------------------------------------------------------
// form-factor table, with the reference's ./atomsf.lib override
// (src/diffraction.c:118-177): read once, on first use, from the working
// directory; every row gets a1 = -1 and rows present in the file are replaced.

static float g_atomsf[SPSIM_B200_N_ELEMENTS][9];
static std::once_flag g_atomsf_once;

static void read_atomsf_table() {
  memcpy(g_atomsf, spsim_b200_atomsf_default, sizeof(g_atomsf));
  FILE *f = fopen("atomsf.lib", "r");
  if (!f) return;
  for (int i = 0; i < SPSIM_B200_N_ELEMENTS; ++i) g_atomsf[i][0] = -1;
  char line[1024];
  auto next = [&](char *buf) -> bool { return fgets(buf, sizeof(line), f) != nullptr; };
  line[0] = 0;
  // comment block: lines starting with "AD"
  while (next(line) && strncmp(line, "AD", 2) == 0) {
  }
  // `line` holds the first line of a record (its name line) or is empty
  while (line[0]) {
    char zl[1024] = {0}, al[1024] = {0}, bl[1024] = {0}, xl[1024] = {0};
    if (!next(zl)) break;
    int z = -1;
    if (sscanf(zl, "%d", &z) != 1 || z < 0 || z >= SPSIM_B200_N_ELEMENTS) break;
    next(al);
    next(bl);
    next(xl);
    if (g_atomsf[z][0] == -1) {
      float v;
      if (strlen(zl) > 23 && sscanf(zl + 23, "%f", &v) == 1) g_atomsf[z][8] = v;
      for (int k = 0; k < 4; ++k) {
        if (strlen(al) > (size_t)(16 * k) && sscanf(al + 16 * k, "%f", &v) == 1) g_atomsf[z][k] = v;
        if (strlen(bl) > (size_t)(16 * k) && sscanf(bl + 16 * k, "%f", &v) == 1) g_atomsf[z][4 + k] = v;
      }
    }
    line[0] = 0;
    next(line);
  }
  fclose(f);
}

// The table is read once per process, by whichever thread uses it first.
static void load_atomsf_table() { std::call_once(g_atomsf_once, read_atomsf_table); }

// Row Z of the coefficient table in use (the ./atomsf.lib override applied);
// internal, shared with the allocation-free entry point in noalloc.cu.
void spsim_internal_atomsf_row(int Z, float out[9]) {
  std::lock_guard<std::mutex> lk(g_mu);
  load_atomsf_table();
  memcpy(out, g_atomsf[Z], 9 * sizeof(float));
}

// ---------------------------------------------------------------------------
// molecules

static unsigned long long g_next_id = 1;

// A grow-only device buffer (no copies; swap hands a buffer to another owner).
struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { cudaFree(p); }
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) cap = bytes;
    return e;
  }
  void swap(DevBuf &o) {
    std::swap(p, o.p);
    std::swap(cap, o.cap);
  }
};

// Grow-only pinned host buffer (not freed at exit: the process's end returns it).
struct PinnedBuf {
  void *p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    release();
    cudaError_t e = cudaMallocHost(&p, bytes);
    if (e == cudaSuccess) cap = bytes;
    else p = nullptr;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};
static PinnedBuf g_upload_stage;  // molecule uploads, under g_mu

struct spsim_b200_molecule {
  unsigned long long id = 0;
  int device = 0;
  int natoms_in = 0;
  int n_kept = 0;
  int n_padded = 0;
  int n_elem = 0;
  int elem_Z[MAX_ELEM];
  std::vector<float> coeffs;  // n_elem x 9
  std::vector<int> perm;      // padded index -> caller index (-1 = padding)
  std::vector<TileDesc> tiles;
  double center[3] = {0, 0, 0};
  double rbound = 0;
  int er = 0, kr = 11;
  float dr = 1, inv_dr = 1;
  int per_atom_b = 0, delta_atoms = 0;
  // device views of the buffers below
  float4 *d_atoms = nullptr;
  float4 *d_atoms2 = nullptr;  // pixel-pair layout of the same records
  AtomD *d_atomsd = nullptr;   // FP64-phase records
  TileDesc *d_tiles = nullptr;
  int *d_perm = nullptr;
  float *d_wbase = nullptr;
  float *d_coeffs = nullptr;
  int *d_flags = nullptr;  // [0] range error
  // owned device memory; a new molecule may take over a dropped one's buffers
  DevBuf b_atoms, b_atoms2, b_atomsd, b_tiles, b_perm, b_wbase, b_coeffs, b_flags, b_inputs;
  void take_buffers(spsim_b200_molecule &o) {
    b_atoms.swap(o.b_atoms);
    b_atoms2.swap(o.b_atoms2);
    b_atomsd.swap(o.b_atomsd);
    b_tiles.swap(o.b_tiles);
    b_perm.swap(o.b_perm);
    b_wbase.swap(o.b_wbase);
    b_coeffs.swap(o.b_coeffs);
    b_flags.swap(o.b_flags);
    b_inputs.swap(o.b_inputs);
  }
};

static int ceil_log2_bound(double x) {
  // smallest e with x < 2^e
  if (!(x > 0)) return -80;
  int e = (int)std::floor(std::log2(x)) + 1;
  while (std::ldexp(1.0, e) <= x) ++e;
  while (e > -80 && std::ldexp(1.0, e - 1) > x) --e;
  return e;
}

// recycle: a molecule about to be destroyed, whose device buffers (not in use
// by queued work) the new one takes over instead of allocating its own.
template <typename PosT>
static int molecule_create_impl(int natoms, const int32_t *Z, const PosT *pos, const float *occ, const float *bfac,
                                int delta_atoms, const float *beam, spsim_b200_molecule **out,
                                spsim_b200_molecule *recycle = nullptr) {
  if (!out) return fail(SPSIM_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (natoms < 0) return fail(SPSIM_ERR_INVALID_ARG, "natoms < 0");
  if (natoms > 0 && (!Z || !pos)) return fail(SPSIM_ERR_INVALID_ARG, "Z or pos is NULL");
  for (int j = 0; j < natoms; ++j)
    if (Z[j] < 0 || Z[j] >= SPSIM_B200_N_ELEMENTS)
      return fail(SPSIM_ERR_INVALID_ARG, "atom %d: atomic number %d outside [0,%d)", j, Z[j], SPSIM_B200_N_ELEMENTS);
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  std::lock_guard<std::mutex> lk(g_mu);
  load_atomsf_table();
  std::unique_ptr<spsim_b200_molecule> m(new spsim_b200_molecule());
  m->id = __atomic_fetch_add(&g_next_id, 1, __ATOMIC_RELAXED);
  m->device = dev;
  m->natoms_in = natoms;
  m->per_atom_b = bfac != nullptr;
  m->delta_atoms = delta_atoms;

  // kept atoms, bounds (in the positions' own type: the extremes are exact)
  PosT lo[3] = {PosT(1e30), PosT(1e30), PosT(1e30)}, hi[3] = {PosT(-1e30), PosT(-1e30), PosT(-1e30)};
  int count[SPSIM_B200_N_ELEMENTS] = {0};
  for (int j = 0; j < natoms; ++j) {
    if (!Z[j]) continue;  // src/diffraction.c:830-832
    ++count[Z[j]];
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], pos[3 * j + k]);
      hi[k] = std::max(hi[k], pos[3 * j + k]);
    }
    ++m->n_kept;
  }
  if (m->n_kept > 0)
    for (int k = 0; k < 3; ++k) m->center[k] = 0.5 * ((double)lo[k] + (double)hi[k]);
  double d2max = 0;  // the square root of the largest squared distance (sqrt is monotonic)
  for (int j = 0; j < natoms; ++j) {
    if (!Z[j]) continue;
    double d2 = 0;
    for (int k = 0; k < 3; ++k) {
      const double d = (double)pos[3 * j + k] - m->center[k];
      d2 += d * d;
    }
    d2max = std::max(d2max, d2);
  }
  const double rmax = std::sqrt(d2max);
  // room for refinement moves: 5% or 0.5 nm, whichever is larger
  m->rbound = rmax + std::max(0.05 * rmax, 5e-10);
  m->er = ceil_log2_bound(m->rbound);
  m->dr = (float)std::ldexp(1.0, m->er - m->kr);
  m->inv_dr = (float)std::ldexp(1.0, m->kr - m->er);

  // element segments (ascending Z), padded to ATOM_GROUP
  std::vector<int> seg_begin;
  int n_pad = 0;
  for (int z = 1; z < SPSIM_B200_N_ELEMENTS; ++z) {
    if (!count[z]) continue;
    if (m->n_elem >= MAX_ELEM) return fail(SPSIM_ERR_INVALID_ARG, "too many elements");
    m->elem_Z[m->n_elem] = z;
    for (int k = 0; k < 9; ++k) m->coeffs.push_back(g_atomsf[z][k]);
    seg_begin.push_back(n_pad);
    n_pad += (count[z] + ATOM_GROUP - 1) / ATOM_GROUP * ATOM_GROUP;
    ++m->n_elem;
  }
  seg_begin.push_back(n_pad);
  m->n_padded = n_pad;
  m->perm.assign(n_pad, -1);
  std::vector<float> wbase(std::max(n_pad, 1), 0.0f);
  {
    std::vector<int> fill(m->n_elem, 0);
    int slot_of_z[SPSIM_B200_N_ELEMENTS];
    for (int e = 0; e < m->n_elem; ++e) slot_of_z[m->elem_Z[e]] = e;
    for (int j = 0; j < natoms; ++j) {
      if (!Z[j]) continue;
      const int e = slot_of_z[Z[j]];
      const int idx = seg_begin[e] + fill[e]++;
      m->perm[idx] = j;
      // weight: sqrt(illumination) (src/diffraction.c:223-235, :834), float like the reference
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
  // tile table
  for (int e = 0; e < m->n_elem; ++e) {
    for (int a = seg_begin[e]; a < seg_begin[e + 1]; a += TILE_ATOMS) {
      TileDesc t;
      t.atom_begin = a;
      t.count = std::min(TILE_ATOMS, seg_begin[e + 1] - a);
      t.elem = e;
      t.last = (a + TILE_ATOMS >= seg_begin[e + 1]) ? 1 : 0;
      m->tiles.push_back(t);
    }
  }
  // device buffers (taken over from `recycle` where they are large enough)
  if (recycle) m->take_buffers(*recycle);
  const size_t na = std::max(n_pad, 1);
  const size_t nin = (size_t)std::max(natoms, 1);
  const size_t in_pos = 3 * nin * sizeof(PosT), in_occ = nin * sizeof(float);
  const size_t in_bytes = in_pos + (occ ? in_occ : 0) + (bfac ? in_occ : 0);
  CUDA_TRY(m->b_atoms.ensure(2 * na * sizeof(float4)));
  CUDA_TRY(m->b_atoms2.ensure(4 * na * sizeof(float4)));
  CUDA_TRY(m->b_atomsd.ensure(na * sizeof(AtomD)));
  CUDA_TRY(m->b_tiles.ensure(std::max<size_t>(m->tiles.size(), 1) * sizeof(TileDesc)));
  CUDA_TRY(m->b_perm.ensure(na * sizeof(int)));
  CUDA_TRY(m->b_wbase.ensure(na * sizeof(float)));
  CUDA_TRY(m->b_coeffs.ensure(std::max<size_t>(m->coeffs.size(), 1) * sizeof(float)));
  CUDA_TRY(m->b_flags.ensure(4 * sizeof(int)));
  CUDA_TRY(m->b_inputs.ensure(std::max<size_t>(in_bytes, 16)));
  m->d_atoms = (float4 *)m->b_atoms.p;
  m->d_atoms2 = (float4 *)m->b_atoms2.p;
  m->d_atomsd = (AtomD *)m->b_atomsd.p;
  m->d_tiles = (TileDesc *)m->b_tiles.p;
  m->d_perm = (int *)m->b_perm.p;
  m->d_wbase = (float *)m->b_wbase.p;
  m->d_coeffs = (float *)m->b_coeffs.p;
  m->d_flags = (int *)m->b_flags.p;
  // upload the caller's arrays and the host-built tables; the records are
  // built on the device (atoms_build_kernel, the host's arithmetic)
  char *din = (char *)m->b_inputs.p;
  const PosT *d_pos = (const PosT *)din;
  const float *d_occ = occ ? (const float *)(din + in_pos) : nullptr;
  const float *d_bfac = bfac ? (const float *)(din + in_pos + (occ ? in_occ : 0)) : nullptr;
  // the uploads go through one pinned staging buffer (grow-only, under g_mu;
  // free again once the synchronisation below returns)
  struct Up {
    void *dst;
    const void *src;
    size_t bytes;
  };
  const Up ups[] = {{din, pos, natoms > 0 ? 3 * (size_t)natoms * sizeof(PosT) : 0},
                    {(void *)d_occ, occ, occ && natoms > 0 ? (size_t)natoms * sizeof(float) : 0},
                    {(void *)d_bfac, bfac, bfac && natoms > 0 ? (size_t)natoms * sizeof(float) : 0},
                    {m->d_tiles, m->tiles.data(), m->tiles.size() * sizeof(TileDesc)},
                    {m->d_perm, m->perm.data(), (size_t)n_pad * sizeof(int)},
                    {m->d_wbase, wbase.data(), na * sizeof(float)},
                    {m->d_coeffs, m->coeffs.data(), m->coeffs.size() * sizeof(float)}};
  size_t stage_bytes = 0;
  for (const Up &u : ups) stage_bytes += (u.bytes + 255) / 256 * 256;
  CUDA_TRY(g_upload_stage.ensure(stage_bytes));
  char *stage = (char *)g_upload_stage.p;
  for (const Up &u : ups) {
    if (!u.bytes) continue;
    memcpy(stage, u.src, u.bytes);
    CUDA_TRY(cudaMemcpyAsync(u.dst, stage, u.bytes, cudaMemcpyHostToDevice, nullptr));
    stage += (u.bytes + 255) / 256 * 256;
  }
  CUDA_TRY(cudaMemsetAsync(m->d_flags, 0, 4 * sizeof(int), nullptr));
  CUDA_TRY(launch_atoms_build<PosT>(m->d_atoms, m->d_atoms2, m->d_atomsd, m->d_perm, n_pad, d_pos, d_occ, d_bfac,
                                    m->d_wbase, m->center, (double)m->dr, (double)m->inv_dr, nullptr));
  // complete before return, so that work on any stream (non-blocking ones too) sees the records
  CUDA_TRY(cudaStreamSynchronize(nullptr));
  *out = m.release();
  return SPSIM_OK;
}

extern "C" int spsim_b200_molecule_create(int natoms, const int32_t *Z, const float *pos, const float *occ,
                                          const float *bfac, int delta_atoms, const float *beam,
                                          spsim_b200_molecule **out) {
  return molecule_create_impl<float>(natoms, Z, pos, occ, bfac, delta_atoms, beam, out);
}

extern "C" int spsim_b200_molecule_create_f64(int natoms, const int32_t *Z, const double *pos, const float *occ,
                                              const float *bfac, int delta_atoms, const float *beam,
                                              spsim_b200_molecule **out) {
  return molecule_create_impl<double>(natoms, Z, pos, occ, bfac, delta_atoms, beam, out);
}

extern "C" int spsim_b200_molecule_update_device(spsim_b200_molecule *m, const void *pos_dev, int pos_is_f64,
                                                 const float *occ_dev, const float *bfac_dev, void *stream) {
  if (!m || !pos_dev) return fail(SPSIM_ERR_INVALID_ARG, "molecule or positions NULL");
  if (bfac_dev && !m->per_atom_b)
    return fail(SPSIM_ERR_INVALID_ARG, "molecule was created without per-atom B factors");
  CUDA_TRY(cudaMemsetAsync(m->d_flags, 0, sizeof(int), (cudaStream_t)stream));  // the range word of this update
  CUDA_TRY(launch_atoms_update(m->d_atoms, m->d_atoms2, m->d_atomsd, m->d_perm, m->n_padded, pos_is_f64 ? nullptr : (const float *)pos_dev,
                               pos_is_f64 ? (const double *)pos_dev : nullptr, occ_dev, bfac_dev, m->d_wbase,
                               m->center, m->dr, m->inv_dr, m->rbound, m->d_flags, (cudaStream_t)stream));
  return SPSIM_OK;
}

extern "C" int spsim_b200_molecule_natoms(const spsim_b200_molecule *m, int *natoms) {
  if (!m || !natoms) return fail(SPSIM_ERR_INVALID_ARG, "NULL argument");
  *natoms = m->natoms_in;
  return SPSIM_OK;
}

extern "C" int spsim_b200_molecule_destroy(spsim_b200_molecule *m) {
  delete m;
  return SPSIM_OK;
}

// ---------------------------------------------------------------------------
// q sets

struct spsim_b200_qset {
  unsigned long long id = 0;
  int device = 0;
  long long npix = 0;
  size_t cap_bytes = 0;  // allocated bytes of d_hkl (reused q sets only)
  float *d_hkl = nullptr;
  double *d_q64 = nullptr;
  double qmax = 0;
  double pair_step = 0;  // largest |q[2m+1] - q[2m]| (the pixel-pair form's admission test)
  double quad_step1 = 0, quad_step2 = 0;  // largest one- and two-pixel steps from a quad's anchor (the quad form's)
  int row = 0;           // pixels per detector row (q sets made from a detector), 0 for a list
  ~spsim_b200_qset() {
    cudaFree(d_hkl);
    cudaFree(d_q64);
  }
};

static cudaError_t set_steps(spsim_b200_qset *q, const float *hkl, const double *q64) {
  double st[3];
  cudaError_t e = qset_steps(hkl, q64, q->npix, st);
  q->pair_step = st[0];
  q->quad_step1 = st[1];
  q->quad_step2 = st[2];
  return e;
}

extern "C" int spsim_b200_qset_from_list(int64_t npix, const float *hkl, int memory, spsim_b200_qset **out) {
  if (!out) return fail(SPSIM_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (npix < 0 || (npix > 0 && !hkl)) return fail(SPSIM_ERR_INVALID_ARG, "bad HKL list");
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  std::unique_ptr<spsim_b200_qset> q(new spsim_b200_qset());
  q->id = __atomic_fetch_add(&g_next_id, 1, __ATOMIC_RELAXED);
  q->device = dev;
  q->npix = npix;
  const size_t bytes = 3 * (size_t)std::max<int64_t>(npix, 1) * sizeof(float);
  CUDA_TRY(cudaMalloc(&q->d_hkl, bytes));
  std::vector<float> h;
  const float *hp = hkl;
  if (memory == SPSIM_MEM_DEVICE) {
    if (npix) CUDA_TRY(cudaMemcpy(q->d_hkl, hkl, 3 * npix * sizeof(float), cudaMemcpyDeviceToDevice));
    h.resize(3 * npix);
    if (npix) CUDA_TRY(cudaMemcpy(h.data(), hkl, 3 * npix * sizeof(float), cudaMemcpyDeviceToHost));
    hp = h.data();
  } else {
    if (npix) CUDA_TRY(cudaMemcpy(q->d_hkl, hkl, 3 * npix * sizeof(float), cudaMemcpyHostToDevice));
  }
  double qm2 = 0;
  for (long long i = 0; i < npix; ++i) {
    const double a = hp[3 * i], b = hp[3 * i + 1], c = hp[3 * i + 2];
    qm2 = std::max(qm2, a * a + b * b + c * c);
  }
  q->qmax = std::sqrt(qm2);
  CUDA_TRY(set_steps(q.get(), q->d_hkl, nullptr));
  *out = q.release();
  return SPSIM_OK;
}

static double detector_qmax(int nx, int ny, float width, float height, float distance, float cx, float cy,
                            float wavelength, int spherical) {
  double m = 0;
  const int xs[2] = {0, nx - 1}, ys[2] = {0, ny - 1};
  const double pxs = (double)(width / nx), pys = (double)(height / ny);
  const double fpx = 2 * std::sin(std::atan(pxs / distance) / 2) / wavelength;
  const double fpy = 2 * std::sin(std::atan(pys / distance) / 2) / wavelength;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      const double px = ((xs[a] - (nx - 1.0) / 2.0) / nx) * (double)width - cx;
      const double py = ((ys[b] - (ny - 1.0) / 2.0) / ny) * (double)height - cy;
      const double pz = distance;
      double q0, q1, q2;
      if (!spherical) {
        const double p = std::sqrt(px * px + py * py + pz * pz);
        const double ew = 1.0 / (double)wavelength;
        q0 = px / p * ew;
        q1 = py / p * ew;
        q2 = (pz / p - 1.0) * ew;
      } else {
        q0 = fpx * px / pxs;
        q1 = fpy * py / pys;
        q2 = 0;
      }
      m = std::max(m, std::sqrt(q0 * q0 + q1 * q1 + q2 * q2));
    }
  return m * (1 + 1e-12);
}

static int check_detector(int nx, int ny, float width, float height, float distance, float wavelength) {
  if (nx <= 0 || ny <= 0) return fail(SPSIM_ERR_INVALID_ARG, "detector has %d x %d pixels", nx, ny);
  if (!(width > 0) || !(height > 0) || !(distance > 0) || !(wavelength > 0))
    return fail(SPSIM_ERR_INVALID_ARG, "detector width/height/distance and wavelength must be > 0");
  return SPSIM_OK;
}

extern "C" int spsim_b200_qset_from_detector(int nx, int ny, float width, float height, float distance,
                                             float center_x, float center_y, float wavelength, int spherical,
                                             spsim_b200_qset **out) {
  if (!out) return fail(SPSIM_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  int st = check_detector(nx, ny, width, height, distance, wavelength);
  if (st) return st;
  int dev;
  st = current_device(&dev);
  if (st) return st;
  std::unique_ptr<spsim_b200_qset> q(new spsim_b200_qset());
  q->id = __atomic_fetch_add(&g_next_id, 1, __ATOMIC_RELAXED);
  q->device = dev;
  q->npix = (long long)nx * ny;
  q->row = nx;
  CUDA_TRY(cudaMalloc(&q->d_q64, 3 * q->npix * sizeof(double)));
  CUDA_TRY(launch_ewald(nx, ny, width, height, distance, center_x, center_y, wavelength, spherical, nullptr,
                        q->d_q64, 0));
  CUDA_TRY(cudaDeviceSynchronize());
  q->qmax = detector_qmax(nx, ny, width, height, distance, center_x, center_y, wavelength, spherical);
  CUDA_TRY(set_steps(q.get(), nullptr, q->d_q64));
  *out = q.release();
  return SPSIM_OK;
}

extern "C" int spsim_b200_qset_npix(const spsim_b200_qset *qs, int64_t *npix) {
  if (!qs || !npix) return fail(SPSIM_ERR_INVALID_ARG, "NULL argument");
  *npix = qs->npix;
  return SPSIM_OK;
}

__global__ static void q64_to_f32_kernel(const double *in, float *out, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)in[i];
}

extern "C" int spsim_b200_qset_copy_q(const spsim_b200_qset *qs, float *hkl_host) {
  if (!qs || !hkl_host) return fail(SPSIM_ERR_INVALID_ARG, "NULL argument");
  if (!qs->npix) return SPSIM_OK;
  if (qs->d_hkl) {
    CUDA_TRY(cudaMemcpy(hkl_host, qs->d_hkl, 3 * qs->npix * sizeof(float), cudaMemcpyDeviceToHost));
    return SPSIM_OK;
  }
  float *tmp = nullptr;
  CUDA_TRY(cudaMalloc(&tmp, 3 * qs->npix * sizeof(float)));
  const long long n = 3 * qs->npix;
  q64_to_f32_kernel<<<(unsigned)((n + 255) / 256), 256>>>(qs->d_q64, tmp, n);
  cudaError_t e = cudaMemcpy(hkl_host, tmp, n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(SPSIM_ERR_CUDA, "copy q: %s", cudaGetErrorString(e));
  return SPSIM_OK;
}

extern "C" int spsim_b200_qset_destroy(spsim_b200_qset *qs) {
  delete qs;
  return SPSIM_OK;
}

// ---------------------------------------------------------------------------
// forward planning


// A polychromatic forward: the plan's npat patterns are the wavelength
// samples of one detector (phase-space scales qscale[j]); their amplitudes are
// combined with weight[j] into one F / I instead of being finalized one by one.
struct Spectrum {
  int samples = 0;
  const double *qscale = nullptr;
  const double *weight = nullptr;
  float *F = nullptr;
  float *I = nullptr;
};

struct Plan {
  // key
  std::vector<const void *> key_ptrs;
  std::vector<double> key_vals;
  // device state
  DevBuf pats, items, acc, ff, flags;
  int n_items = 0, grid = 0, npat = 0;
  long long max_npix = 0;
  double terms = 0;
  int precision = 0, nt = 128, ppt = 4, packed = 1;
  bool perb = false;
  bool fixw = false;  // FP64-phase forms: fixed-point phase word (every pattern within 2^17 cycles)
  bool narrow = false;  // neighbour pairs: every step within 0.07 cycle (the NARROW second-pixel polynomial)
  std::vector<long long> npix_of;
  std::vector<SfPattern> host_pats;  // descriptors as last uploaded (rotations change per call)
  int spectrum = 0;                  // > 0: combine this many patterns into spec_F / spec_I
  DevBuf spec_w;
  float *spec_F = nullptr, *spec_I = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~Plan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

static std::vector<std::unique_ptr<Plan>> g_plans;  // most recent last
struct OneShot {  // per-thread scratch plan of uncached calls; lives until the process ends
  Plan *plan = nullptr;
  int device = -1;
};
static thread_local OneShot g_oneshot;
static const size_t kMaxPlans = 8;
static int g_force_nt = -1, g_force_p = -1, g_force_pk = 3;
struct Variant {
  int nt, p, packed;
  int p_fallback = 0;  // pixels per thread where form 4 or 3 is not admitted (0: p's nearest)
};
static std::map<long long, Variant> g_tuned;  // size class -> kernel variant
static bool g_timing = false;
static std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_timing_events;
static thread_local double g_last_terms = 0, g_last_ms = 0;
static thread_local int g_last_variant[3] = {0, 0, -1};  // threads, pixels per thread, form (-1: FP64 kernel)
static thread_local int g_last_phase_word = 0;            // forms 2/3: fixed-point phase word used
static thread_local int g_last_pair_narrow = 0;           // form 3: NARROW second-pixel polynomial used
static int g_num_sms = 0;

static int num_sms() {
  if (!g_num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

static long long size_class(double terms) { return (long long)std::floor(std::log2(std::max(terms, 1.0)) / 2); }

static Variant choose_variant(double terms, long long total_npix, int precision) {
  const int mode = precision == SPSIM_PREC_F32_FAST ? 1 : 0;
  if (g_force_nt > 0 && sf_f32_variant_exists(mode, g_force_nt, g_force_p, g_force_pk))
    return {g_force_nt, g_force_p, g_force_pk};
  auto it = g_tuned.find(size_class(terms) * 4 + precision);
  if (it != g_tuned.end()) return it->second;
  // untuned defaults, from sweeps on B200: the neighbour-pair FP64-phase form
  // for FP32, the FP64-phase form for FP32_FAST (MUFU sin/cos, where the
  // neighbour step saves nothing); 8 pixels per thread (two CTAs per SM) once
  // there are enough pixel tiles to fill every SM several times (fastest on
  // both the 50,000- and the 5,000-atom workloads)
  // the neighbour-quad form (8 pixels per thread), falling back (FP32) to the
  // pair form and then to form 2 where a q set is not admitted, there with 4
  // pixels per thread below 2^20 pixels; FP32_FAST falls back to form 2 (its
  // MUFU sin/cos gains nothing from pairs)
  return {128, 8, 4, total_npix >= (1LL << 20) ? 8 : 4};
}

// The variant of `form` nearest to (nt, p): p itself where compiled, else 8, else 4.
static Variant fit_variant(int precision, int nt, int p, int form) {
  const int mode = precision == SPSIM_PREC_F32_FAST ? 1 : 0;
  for (int pp : {p, 8, 4})
    if (sf_f32_variant_exists(mode, nt, pp, form)) return {nt, pp, form};
  return {128, 4, form};
}

static bool is_orthonormal(const double *R) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double d = 0;
      for (int k = 0; k < 3; ++k) d += R[3 * k + i] * R[3 * k + j];
      if (std::fabs(d - (i == j ? 1.0 : 0.0)) > 1e-6) return false;
    }
  return true;
}

static thread_local long long g_split_pixels_hint = 0;  // pixels of the whole shot while a shot part is planned

static int build_plan(Plan &pl, int npat, const spsim_b200_molecule *const *mols, const spsim_b200_qset *const *qsets,
                      const double *rot, float B, int precision, float *const *F_dev, float *const *I_dev,
                      cudaStream_t stream, const Spectrum *spec) {
  pl.npat = npat;
  pl.precision = precision;
  std::vector<SfPattern> pats(npat);
  // unique (molecule, q set) pairs share one form-factor table
  std::map<std::pair<const void *, const void *>, size_t> ff_off;
  size_t ff_total = 0, acc_total = 0;
  std::vector<size_t> acc_off(npat), ffo(npat);
  double terms = 0;
  long long total_npix = 0;
  bool perb = false;
  for (int i = 0; i < npat; ++i) {
    const spsim_b200_molecule *m = mols[i];
    const spsim_b200_qset *q = qsets[i];
    if (!m || !q) return fail(SPSIM_ERR_INVALID_ARG, "pattern %d: NULL molecule or q set", i);
    auto key = std::make_pair((const void *)m, (const void *)q);
    auto f = ff_off.find(key);
    if (f == ff_off.end()) {
      ff_off[key] = ff_total;
      ffo[i] = ff_total;
      ff_total += (size_t)m->n_elem * q->npix;
    } else {
      ffo[i] = f->second;
    }
    acc_off[i] = acc_total;
    acc_total += q->npix;
    terms += (double)q->npix * m->n_kept;
    total_npix += q->npix;
    perb = perb || m->per_atom_b;
  }
  pl.terms = terms;
  pl.perb = perb;
  CUDA_TRY(pl.acc.ensure(std::max<size_t>(acc_total, 1) * sizeof(double2)));
  CUDA_TRY(pl.ff.ensure(std::max<size_t>(ff_total, 1) * sizeof(double)));
  CUDA_TRY(pl.flags.ensure(64));
  CUDA_TRY(cudaMemsetAsync(pl.flags.p, 0, 64, stream));  // queue head and the sticky error word
  CUDA_TRY(pl.pats.ensure(std::max(npat, 1) * sizeof(SfPattern)));

  Variant var = {128, 4, 1};
  if (precision != SPSIM_PREC_FP64) var = choose_variant(terms, total_npix, precision);
  if (var.packed == 4) {
    // neighbour-quad form: every pattern needs its one-pixel steps within 1/8
    // cycle and its two-pixel steps within 0.16 cycle of the molecule's bound
    bool ok = precision != SPSIM_PREC_FP64;
    double max_step1 = 0.0;
    for (int i = 0; i < npat && ok; ++i) {
      double scale = spec ? std::fabs(spec->qscale[i]) : 1.0;
      if (rot && !is_orthonormal(rot + 9 * (size_t)i)) {
        double fro = 0;
        for (int k = 0; k < 9; ++k) fro += rot[9 * (size_t)i + k] * rot[9 * (size_t)i + k];
        scale *= std::sqrt(fro);
      }
      const double s1 = qsets[i]->quad_step1 * scale * mols[i]->rbound;
      const double s2 = qsets[i]->quad_step2 * scale * mols[i]->rbound;
      ok = s1 <= (1.0 / 8) * (1.0 - 1e-9) && s2 <= 0.16 * (1.0 - 1e-9);
      max_step1 = std::max(max_step1, s1);
    }
    pl.narrow = ok && max_step1 <= 0.07 * (1.0 - 1e-6);
    if (!ok) {
      const int pf = var.p_fallback;
      var = fit_variant(precision, var.nt, pf ? pf : var.p, precision == SPSIM_PREC_F32 ? 3 : 2);
      var.p_fallback = pf;
    }
  }
  if (var.packed == 3) {
    // neighbour-pair form: every pattern needs |q_b - q_a| |r|max <= 1/8 cycle
    bool ok = true;
    double max_step = 0.0;
    for (int i = 0; i < npat && ok; ++i) {
      double scale = spec ? std::fabs(spec->qscale[i]) : 1.0;
      if (rot && !is_orthonormal(rot + 9 * (size_t)i)) {
        double fro = 0;
        for (int k = 0; k < 9; ++k) fro += rot[9 * (size_t)i + k] * rot[9 * (size_t)i + k];
        scale *= std::sqrt(fro);
      }
      ok = qsets[i]->pair_step * scale * mols[i]->rbound <= (1.0 / 8) * (1.0 - 1e-9);
      max_step = std::max(max_step, qsets[i]->pair_step * scale * mols[i]->rbound);
    }
    pl.narrow = ok && max_step <= 0.07 * (1.0 - 1e-6);
    if (!ok) var = fit_variant(precision, var.nt, var.p_fallback ? var.p_fallback : var.p, 2);
  }
  const int nt = var.nt, ppt = var.p;
  pl.nt = var.nt;
  pl.ppt = var.p;
  pl.packed = var.packed;
  const long long tile_pix = (long long)nt * ppt;

  pl.max_npix = 0;
  pl.npix_of.resize(npat);
  for (int i = 0; i < npat; ++i) {
    const spsim_b200_molecule *m = mols[i];
    const spsim_b200_qset *q = qsets[i];
    SfPattern &pt = pats[i];
    memset(&pt, 0, sizeof(pt));
    pt.atoms = m->d_atoms;
    pt.atoms2 = m->d_atoms2;
    pt.atomsd = m->d_atomsd;
    pt.tiles = m->d_tiles;
    pt.n_tiles = (int)m->tiles.size();
    pt.n_elem = m->n_elem;
    pt.per_atom_b = m->per_atom_b;
    pt.ff = (double *)pl.ff.p + ffo[i];
    pt.npix = q->npix;
    pt.hkl = q->d_hkl;
    pt.q64 = q->d_q64;
    double qmax = q->qmax;
    if (rot) {
      const double *R = rot + 9 * (size_t)i;
      memcpy(pt.rot, R, 9 * sizeof(double));
      pt.has_rot = 1;
      if (!is_orthonormal(R)) {
        double fro = 0;
        for (int k = 0; k < 9; ++k) fro += R[k] * R[k];
        qmax *= std::sqrt(fro);
      }
    } else {
      pt.has_rot = 0;
      for (int k = 0; k < 9; ++k) pt.rot[k] = (k % 4 == 0) ? 1.0 : 0.0;
    }
    pt.qscale = spec ? spec->qscale[i] : 1.0;
    pt.s2scale = 1.0 / (pt.qscale * pt.qscale);
    qmax *= std::fabs(pt.qscale);
    memcpy(pt.center, m->center, sizeof(pt.center));
    pt.mol_err = m->d_flags;
    pt.plan_err = (int *)pl.flags.p + 5;
    const int eq = ceil_log2_bound(std::max(qmax, 1e-300));
    const int kq = 22 - m->kr;
    pt.dq = (float)std::ldexp(1.0, eq - kq);
    pt.inv_dq = (float)std::ldexp(1.0, kq - eq);
    pt.acc = (double2 *)pl.acc.p + acc_off[i];
    pt.F = F_dev ? (float2 *)F_dev[i] : nullptr;
    pt.I = I_dev ? I_dev[i] : nullptr;
    pl.max_npix = std::max(pl.max_npix, q->npix);
    pl.npix_of[i] = q->npix;
    if (precision != SPSIM_PREC_FP64 && pl.packed >= 2 && m->n_kept > 0 && q->npix > 0) {
      // FP64 phase: the half-cycle rounding needs |2 q.r| < 2^51
      const double qr = qmax * m->rbound;
      if (qr >= std::ldexp(1.0, 48))
        return fail(SPSIM_ERR_RANGE, "pattern %d: |q|max*|r|max = %.3g cycles exceeds 2^48", i, qr);
    } else if (precision != SPSIM_PREC_FP64 && m->n_kept > 0 && q->npix > 0) {
      // domain checks of the compensated phase
      const double qr = qmax * m->rbound;
      if (qr >= std::ldexp(1.0, 19))
        return fail(SPSIM_ERR_RANGE, "pattern %d: |q|max*|r|max = %.3g cycles exceeds 2^19; use SPSIM_PREC_FP64", i, qr);
      const double cmax = 0.8660254037844386 * (qmax * m->dr + (double)pt.dq * (m->rbound + m->dr));
      const double lim = precision == SPSIM_PREC_F32 ? 1.0 / 16 : 0.25;
      if (cmax > lim)
        return fail(SPSIM_ERR_RANGE,
                    "pattern %d: phase cross term %.4f cycles exceeds %.4f (|q|max %.3g 1/m, |r|max %.3g m); use "
                    "SPSIM_PREC_FP64",
                    i, cmax, lim, qmax, m->rbound);
    }
  }
  // the fixed-point phase word needs |q.(r - c)| < 2^18 cycles; 2^17 leaves a margin
  pl.fixw = precision != SPSIM_PREC_FP64 && pl.packed >= 2;
  for (int i = 0; i < npat && pl.fixw; ++i) {
    double qmax = qsets[i]->qmax * (spec ? std::fabs(spec->qscale[i]) : 1.0);
    if (rot && !is_orthonormal(rot + 9 * (size_t)i)) {
      double fro = 0;
      for (int k = 0; k < 9; ++k) fro += rot[9 * (size_t)i + k] * rot[9 * (size_t)i + k];
      qmax *= std::sqrt(fro);
    }
    if (mols[i]->n_kept > 0 && qsets[i]->npix > 0 && qmax * mols[i]->rbound >= std::ldexp(1.0, 17)) pl.fixw = false;
  }
  CUDA_TRY(cudaMemcpyAsync(pl.pats.p, pats.data(), npat * sizeof(SfPattern), cudaMemcpyHostToDevice, stream));
  pl.host_pats = pats;
  pl.spectrum = spec ? spec->samples : 0;
  pl.spec_F = spec ? spec->F : nullptr;
  pl.spec_I = spec ? spec->I : nullptr;
  if (spec) {
    CUDA_TRY(pl.spec_w.ensure(npat * sizeof(double)));
    CUDA_TRY(cudaMemcpyAsync(pl.spec_w.p, spec->weight, npat * sizeof(double), cudaMemcpyHostToDevice, stream));
  }

  if (precision != SPSIM_PREC_FP64) {
    // work items: pixel tile x atom-tile range, cost-sorted (largest first)
    const int occ =
        std::max(1, sf_f32_occupancy(precision == SPSIM_PREC_F32_FAST ? 1 : 0, nt, ppt, pl.packed, perb, pl.fixw,
                                     pl.narrow));
    const long long slots = (long long)num_sms() * occ;
    long long total_ptiles = 0;
    for (int i = 0; i < npat; ++i) total_ptiles += (qsets[i]->npix + tile_pix - 1) / tile_pix;
    // a row chunk of a pipelined shot splits its atoms as the whole shot
    // would: the next chunk, on the other stream, fills this one's tail
    if (g_split_pixels_hint > 0) total_ptiles = std::max(total_ptiles, (g_split_pixels_hint + tile_pix - 1) / tile_pix);
    // split atoms when pixel tiles alone cannot fill the GPU several times over
    const long long want = 6 * slots;
    std::vector<WorkItem> items;
    std::vector<double> cost;
    for (int i = 0; i < npat; ++i) {
      const long long nptile = (qsets[i]->npix + tile_pix - 1) / tile_pix;
      const int ntile = (int)mols[i]->tiles.size();
      if (ntile == 0 || qsets[i]->npix == 0) continue;
      int split = 1;
      if (total_ptiles < want) split = (int)std::min<long long>((want + total_ptiles - 1) / total_ptiles, ntile);
      split = std::max(1, std::min(split, std::max(1, ntile / 2)));
      for (long long t = 0; t < nptile; ++t) {
        const long long pix_here = std::min(tile_pix, qsets[i]->npix - t * tile_pix);
        for (int s = 0; s < split; ++s) {
          WorkItem w;
          w.pattern = i;
          w.pixel_tile = (int)t;
          w.k0 = (int)((long long)ntile * s / split);
          w.k1 = (int)((long long)ntile * (s + 1) / split);
          if (w.k1 <= w.k0) continue;
          items.push_back(w);
          int atoms_here = 0;
          for (int k = w.k0; k < w.k1; ++k) atoms_here += mols[i]->tiles[k].count;
          cost.push_back((double)pix_here * atoms_here);
        }
      }
    }
    std::vector<size_t> order(items.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
    std::vector<WorkItem> sorted(items.size());
    for (size_t k = 0; k < order.size(); ++k) sorted[k] = items[order[k]];
    pl.n_items = (int)sorted.size();
    pl.grid = (int)std::min<long long>(std::max(pl.n_items, 1), slots);
    CUDA_TRY(pl.items.ensure(std::max<size_t>(sorted.size(), 1) * sizeof(WorkItem)));
    if (!sorted.empty())
      CUDA_TRY(cudaMemcpyAsync(pl.items.p, sorted.data(), sorted.size() * sizeof(WorkItem), cudaMemcpyHostToDevice,
                               stream));
  }
  // form-factor tables (per unique molecule / q set pair; fixed for the plan's life)
  std::map<std::pair<const void *, const void *>, bool> done;
  for (int i = 0; i < npat; ++i) {
    auto key = std::make_pair((const void *)mols[i], (const void *)qsets[i]);
    if (done[key]) continue;
    done[key] = true;
    const spsim_b200_qset *q = qsets[i];
    CUDA_TRY(launch_ff_table(q->d_hkl, q->d_q64, q->npix, mols[i]->n_elem, mols[i]->d_coeffs, (double)B,
                             mols[i]->delta_atoms, (double *)pl.ff.p + ffo[i], stream));
  }
  return SPSIM_OK;
}

// ---------------------------------------------------------------------------
// enqueue, plan cache, forward entry points

static cudaError_t enqueue_plan(Plan &pl, cudaStream_t stream, cudaEvent_t ev0, cudaEvent_t ev1) {
  cudaError_t e;
  long long acc_total = 0;
  for (long long n : pl.npix_of) acc_total += n;
  if ((e = cudaMemsetAsync(pl.acc.p, 0, std::max<long long>(acc_total, 1) * sizeof(double2), stream))) return e;
  if ((e = cudaMemsetAsync(pl.flags.p, 0, sizeof(int), stream))) return e;  // work queue head
  if (ev0 && (e = cudaEventRecord(ev0, stream))) return e;
  if (pl.precision == SPSIM_PREC_FP64) {
    for (int i = 0; i < pl.npat; ++i)
      if ((e = launch_sf_f64((const SfPattern *)pl.pats.p, i, pl.npix_of[i], stream))) return e;
  } else if (pl.n_items > 0) {
    const int mode = pl.precision == SPSIM_PREC_F32_FAST ? PREC_MODE_MUFU : PREC_MODE_POLY;
    int *flags = (int *)pl.flags.p;
    if ((e = launch_sf_f32(mode, pl.nt, pl.ppt, pl.packed, pl.perb, (const SfPattern *)pl.pats.p, (const WorkItem *)pl.items.p,
                           pl.n_items, flags, flags + 4, pl.grid, stream, pl.fixw, pl.narrow)))
      return e;
  }
  if (ev1 && (e = cudaEventRecord(ev1, stream))) return e;
  if (pl.spectrum > 0)
    return launch_spectrum_combine((const SfPattern *)pl.pats.p, 0, pl.spectrum, (const double *)pl.spec_w.p, pl.spec_F,
                                   pl.spec_I, pl.npix_of.empty() ? 0 : pl.npix_of[0], stream);
  return launch_finalize((const SfPattern *)pl.pats.p, 0, pl.npat, pl.max_npix, stream);
}

static void plan_key(int npat, const spsim_b200_molecule *const *mols, const spsim_b200_qset *const *qsets,
                     const double *rot, float B, int precision, float *const *F_dev, float *const *I_dev,
                     const Spectrum *spec, std::vector<const void *> &kp, std::vector<double> &kv) {
  kv.push_back(npat);
  kv.push_back(spec ? spec->samples : 0);
  if (spec) {
    for (int i = 0; i < npat; ++i) {
      kv.push_back(spec->qscale[i]);
      kv.push_back(spec->weight[i]);
    }
    kp.push_back(spec->F);
    kp.push_back(spec->I);
  }
  kv.push_back(B);
  kv.push_back(precision);
  kv.push_back(g_force_nt);
  kv.push_back(g_force_p);
  kv.push_back(g_force_pk);
  for (int i = 0; i < npat; ++i) {
    kv.push_back((double)(mols[i] ? mols[i]->id : 0));
    kv.push_back((double)(qsets[i] ? qsets[i]->id : 0));
    kp.push_back(F_dev ? (const void *)F_dev[i] : nullptr);
    kp.push_back(I_dev ? (const void *)I_dev[i] : nullptr);
  }
  // Orthonormal rotations only change the descriptors, which are re-uploaded
  // per call; any other matrix changes the phase grid, so it keys the plan.
  bool ortho = true;
  if (rot)
    for (int i = 0; i < npat && ortho; ++i) ortho = is_orthonormal(rot + 9 * (size_t)i);
  kv.push_back(rot ? (ortho ? 1.0 : 2.0) : 0.0);
  if (rot && !ortho)
    for (long long k = 0; k < 9LL * npat; ++k) kv.push_back(rot[k]);
}

// Write this call's rotations into the plan's descriptors (device copy ordered on `stream`).
static cudaError_t refresh_rotations(Plan &pl, const double *rot, cudaStream_t stream) {
  if (!rot) return cudaSuccess;
  bool changed = false;
  for (int i = 0; i < pl.npat; ++i)
    if (memcmp(pl.host_pats[i].rot, rot + 9 * (size_t)i, 9 * sizeof(double)) != 0) {
      memcpy(pl.host_pats[i].rot, rot + 9 * (size_t)i, 9 * sizeof(double));
      changed = true;
    }
  if (!changed) return cudaSuccess;
  return cudaMemcpyAsync(pl.pats.p, pl.host_pats.data(), pl.npat * sizeof(SfPattern), cudaMemcpyHostToDevice, stream);
}

static int check_flags(Plan &pl) {
  int h[8] = {0};
  CUDA_TRY(cudaMemcpy(h, pl.flags.p, sizeof(h), cudaMemcpyDeviceToHost));
  if (h[4]) {
    int z = 0;
    cudaMemcpy((int *)pl.flags.p + 4, &z, sizeof(int), cudaMemcpyHostToDevice);
    return fail(SPSIM_ERR_TIMEOUT, "structure-factor kernel: an atom-tile copy did not complete in time");
  }
  if (h[5]) {
    int z = 0;
    cudaMemcpy((int *)pl.flags.p + 5, &z, sizeof(int), cudaMemcpyHostToDevice);
    return fail(SPSIM_ERR_RANGE, "atoms moved outside the molecule's creation-time bounds");
  }
  return SPSIM_OK;
}

// cache == false: a one-shot plan (host convenience path), synchronised before return
// cache == false and sync == false: the one-shot plan is enqueued and not
// waited for; spsim_internal_shot_check reads its error flags afterwards.
static int run_forward(int npat, const spsim_b200_molecule *const *mols, const spsim_b200_qset *const *qsets,
                       const double *rot, float B, int precision, float *const *F_dev, float *const *I_dev,
                       cudaStream_t stream, bool cache, const Spectrum *spec = nullptr, bool sync = true,
                       Plan *scratch = nullptr) {
  if (npat < 0) return fail(SPSIM_ERR_INVALID_ARG, "npatterns < 0");
  if (npat == 0) return SPSIM_OK;
  if (!mols || !qsets) return fail(SPSIM_ERR_INVALID_ARG, "NULL molecule or q-set array");
  if (precision < SPSIM_PREC_FP64 || precision > SPSIM_PREC_F32_FAST)
    return fail(SPSIM_ERR_INVALID_ARG, "unknown precision %d", precision);
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  for (int i = 0; i < npat; ++i) {
    if (!mols[i] || !qsets[i]) return fail(SPSIM_ERR_INVALID_ARG, "pattern %d: NULL handle", i);
    if (mols[i]->device != dev || qsets[i]->device != dev)
      return fail(SPSIM_ERR_INVALID_ARG, "pattern %d: handle belongs to another device", i);
  }
  std::lock_guard<std::mutex> lk(g_mu);
  std::vector<const void *> kp;
  std::vector<double> kv;
  plan_key(npat, mols, qsets, rot, B, precision, F_dev, I_dev, spec, kp, kv);
  Plan *pl = nullptr;
  if (cache) {
    for (size_t i = 0; i < g_plans.size(); ++i) {
      if (g_plans[i]->key_ptrs == kp && g_plans[i]->key_vals == kv) {
        std::unique_ptr<Plan> p = std::move(g_plans[i]);
        g_plans.erase(g_plans.begin() + i);
        g_plans.push_back(std::move(p));
        pl = g_plans.back().get();
        break;
      }
    }
  }
  if (!pl && cache) {
    std::unique_ptr<Plan> np(new Plan());
    np->key_ptrs = kp;
    np->key_vals = kv;
    st = build_plan(*np, npat, mols, qsets, rot, B, precision, F_dev, I_dev, stream, spec);
    if (st) return st;
    if (g_plans.size() >= kMaxPlans) {
      cudaDeviceSynchronize();  // the evicted plan's buffers may still be in use
      g_plans.erase(g_plans.begin());
    }
    g_plans.push_back(std::move(np));
    pl = g_plans.back().get();
  } else if (!pl) {
    // one-shot calls rebuild the descriptors of this thread's scratch plan (or
    // the caller's), whose device buffers only grow (no cudaMalloc / cudaFree
    // per call)
    OneShot &os = g_oneshot;
    if (scratch) {
      pl = scratch;
    } else {
      if (!os.plan || os.device != dev) {
        os.plan = new Plan();  // a plan left on another device is kept, not freed, while its context may be busy
        os.device = dev;
      }
      pl = os.plan;
    }
    pl->key_ptrs = kp;
    pl->key_vals = kv;
    st = build_plan(*pl, npat, mols, qsets, rot, B, precision, F_dev, I_dev, stream, spec);
    if (st) return st;
  }
  g_last_terms = pl->terms;
  g_last_variant[0] = pl->precision == SPSIM_PREC_FP64 ? 256 : pl->nt;
  g_last_variant[1] = pl->precision == SPSIM_PREC_FP64 ? 1 : pl->ppt;
  g_last_variant[2] = pl->precision == SPSIM_PREC_FP64 ? -1 : pl->packed;
  g_last_phase_word = pl->precision != SPSIM_PREC_FP64 && pl->fixw ? 1 : 0;
  g_last_pair_narrow =
      pl->precision != SPSIM_PREC_FP64 && (pl->packed == 4 || (pl->packed == 3 && pl->precision == SPSIM_PREC_F32)) &&
              pl->fixw && pl->narrow
          ? 1
          : 0;
  CUDA_TRY(refresh_rotations(*pl, rot, stream));
  if (g_timing || !cache || stream == nullptr) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (g_timing) {
      CUDA_TRY(cudaEventCreate(&e0));
      CUDA_TRY(cudaEventCreate(&e1));
      g_timing_events.push_back({e0, e1});
    }
    CUDA_TRY(enqueue_plan(*pl, stream, e0, e1));
  } else {
    if (!pl->exec) {
      CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t ce = enqueue_plan(*pl, stream, nullptr, nullptr);
      cudaGraph_t g = nullptr;
      cudaError_t ee = cudaStreamEndCapture(stream, &g);
      if (ce != cudaSuccess) return fail(SPSIM_ERR_CUDA, "capture: %s", cudaGetErrorString(ce));
      if (ee != cudaSuccess) return fail(SPSIM_ERR_CUDA, "end capture: %s", cudaGetErrorString(ee));
      pl->graph = g;
      CUDA_TRY(cudaGraphInstantiate(&pl->exec, g, 0));
    }
    CUDA_TRY(cudaGraphLaunch(pl->exec, stream));
  }
  if (!cache && sync) {
    CUDA_TRY(cudaStreamSynchronize(stream));
    return check_flags(*pl);
  }
  return SPSIM_OK;
}

extern "C" int spsim_b200_forward(const spsim_b200_molecule *m, const spsim_b200_qset *qs, const double *rot,
                                  float B, int precision, float *F_dev, float *I_dev, void *stream) {
  float *F[1] = {F_dev};
  float *I[1] = {I_dev};
  return run_forward(1, &m, &qs, rot, B, precision, F, I, (cudaStream_t)stream, true);
}

// Wavelength samples of a bandwidth-broadened beam, as spsim's spectrum kernel
// takes them (src/diffraction.cu:305-307, :415-476): an even sample count
// above one is raised by one; lambda_j = lambda (1 - bw/2) + j/(S-1) lambda bw;
// the phase uses q lambda / lambda_j (form factors stay at |q|); weights are
// exp(-z_j^2 / 2) with z_j = (lambda_j - lambda) / (lambda bw / 4), normalised
// to sum to one.  Returns the sample count used (1: monochromatic).
static int spectrum_samples(float wavelength, float bandwidth, int samples, std::vector<double> &qscale,
                            std::vector<double> &weight) {
  if (samples > 1 && (samples & 1) == 0) ++samples;
  qscale.clear();
  weight.clear();
  if (bandwidth == 0.0f || samples <= 1) {
    qscale.push_back(1.0);
    weight.push_back(1.0);
    return 1;
  }
  const double lam = wavelength, bw = bandwidth;
  const double sigma = (lam - lam * (1.0 - bw / 2.0)) / 2.0;
  double tot = 0.0;
  for (int j = 0; j < samples; ++j) {
    const double lj = lam * (1.0 - bw / 2.0) + ((double)j / (samples - 1)) * lam * bw;
    const double z = (lj - lam) / sigma;
    qscale.push_back(lam / lj);
    weight.push_back(std::exp(-z * z / 2.0));
    tot += weight.back();
  }
  for (double &w : weight) w /= tot;
  return samples;
}

static int forward_spectrum(const spsim_b200_molecule *m, const spsim_b200_qset *qs, const double *rot, float B,
                            int precision, float wavelength, float bandwidth, int samples, float *F_dev, float *I_dev,
                            cudaStream_t stream, bool cache, bool sync = true) {
  if (!m || !qs) return fail(SPSIM_ERR_INVALID_ARG, "NULL handle");
  if (samples < 1) return fail(SPSIM_ERR_INVALID_ARG, "wavelength samples must be >= 1 (got %d)", samples);
  if (bandwidth != 0.0f && !(wavelength > 0.0f))
    return fail(SPSIM_ERR_INVALID_ARG, "a bandwidth needs a wavelength > 0");
  std::vector<double> qscale, weight;
  const int S = spectrum_samples(wavelength, bandwidth, samples, qscale, weight);
  if (S == 1) {
    float *F[1] = {F_dev};
    float *I[1] = {I_dev};
    return run_forward(1, &m, &qs, rot, B, precision, F, I, stream, cache, nullptr, sync);
  }
  std::vector<const spsim_b200_molecule *> mols(S, m);
  std::vector<const spsim_b200_qset *> qsets(S, qs);
  std::vector<double> rots;
  if (rot)
    for (int j = 0; j < S; ++j) rots.insert(rots.end(), rot, rot + 9);
  std::vector<float *> none(S, nullptr);
  Spectrum spec;
  spec.samples = S;
  spec.qscale = qscale.data();
  spec.weight = weight.data();
  spec.F = F_dev;
  spec.I = I_dev;
  return run_forward(S, mols.data(), qsets.data(), rot ? rots.data() : nullptr, B, precision, none.data(), none.data(),
                     stream, cache, &spec, sync);
}

extern "C" int spsim_b200_forward_spectrum(const spsim_b200_molecule *m, const spsim_b200_qset *qs, const double *rot,
                                           float B, int precision, float wavelength, float bandwidth, int samples,
                                           float *F_dev, float *I_dev, void *stream) {
  return forward_spectrum(m, qs, rot, B, precision, wavelength, bandwidth, samples, F_dev, I_dev,
                          (cudaStream_t)stream, true);
}

extern "C" int spsim_b200_forward_batch(int npatterns, const spsim_b200_molecule *const *mols,
                                        const spsim_b200_qset *const *qsets, const double *rot, float B, int precision,
                                        float *const *F_dev, float *const *I_dev, void *stream) {
  return run_forward(npatterns, mols, qsets, rot, B, precision, F_dev, I_dev, (cudaStream_t)stream, true);
}

// Reusable state of the host-buffer entry point, one per thread: the last
// molecule (reused while the caller's atom arrays are byte-identical to the
// copies kept here), a q set whose device buffer grows and is rewritten per
// call, and device F / I buffers.  Nothing is freed per call; a device change
// starts a fresh session (the old one is dropped without freeing, as its
// context may still be in use).
struct HostSession {
  int device = -1;
  spsim_b200_molecule *mol = nullptr;
  std::vector<unsigned char> mol_inputs;  // natoms, Z, pos, occ, bfac, delta_atoms, beam, as passed
  spsim_b200_qset *qs = nullptr;
  DevBuf *F = nullptr, *I = nullptr;
  DevBuf *stats = nullptr;  // four words for the device q-set statistics
  // the pipelined simulate_shot: per row chunk a view of qs (its pixels, the
  // whole list's statistics) and a scratch plan; parts: chunks of this shot
  std::vector<spsim_b200_qset *> views;
  std::vector<Plan *> part_plans;
  int parts = 0;
  spsim_b200_qset *shot_q = nullptr;  // the shot's whole HKL list, borrowed (no copy)
};
static thread_local HostSession g_host;
static thread_local spsim_b200_molecule *g_shot_mol = nullptr;  // set by spsim_internal_shot_molecule

static void append_bytes(std::vector<unsigned char> &v, const void *p, size_t n) {
  const unsigned char *b = (const unsigned char *)p;
  v.insert(v.end(), b, b + n);
}

static int host_session_molecule(int natoms, const int32_t *Z, const float *pos, const float *occ, const float *bfac,
                                 int delta_atoms, const float *beam, spsim_b200_molecule **out) {
  std::vector<unsigned char> key;
  const size_t n = natoms > 0 ? (size_t)natoms : 0;
  key.reserve(3 * sizeof(int) + n * (sizeof(int32_t) + 3 * sizeof(float) + (occ ? 4 : 0) + (bfac ? 4 : 0)) +
              (beam ? 3 * sizeof(float) : 0));
  append_bytes(key, &natoms, sizeof(natoms));
  append_bytes(key, &delta_atoms, sizeof(delta_atoms));
  const int flags = (Z ? 1 : 0) | (pos ? 2 : 0) | (occ ? 4 : 0) | (bfac ? 8 : 0) | (beam ? 16 : 0);
  append_bytes(key, &flags, sizeof(flags));
  if (Z) append_bytes(key, Z, n * sizeof(int32_t));
  if (pos) append_bytes(key, pos, 3 * n * sizeof(float));
  if (occ) append_bytes(key, occ, n * sizeof(float));
  if (bfac) append_bytes(key, bfac, n * sizeof(float));
  if (beam) append_bytes(key, beam, 3 * sizeof(float));
  if (g_host.mol && key == g_host.mol_inputs) {
    *out = g_host.mol;
    return SPSIM_OK;
  }
  spsim_b200_molecule *m = nullptr;
  // the kept molecule's records may still be read by queued work: wait, then
  // hand its device buffers to the new molecule
  if (g_host.mol) CUDA_TRY(cudaDeviceSynchronize());
  int st = molecule_create_impl<float>(natoms, Z, pos, occ, bfac, delta_atoms, beam, &m, g_host.mol);
  if (g_host.mol) spsim_b200_molecule_destroy(g_host.mol);
  g_host.mol = nullptr;
  g_host.mol_inputs.clear();
  if (st) return st;
  g_host.mol = m;
  g_host.mol_inputs.swap(key);
  *out = m;
  return SPSIM_OK;
}

// Rewrite the session's q set with a host HKL list (new id: cached plans keyed
// on the old contents are never matched again).
static int host_session_qset(int64_t npix, const float *hkl, spsim_b200_qset **out) {
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  if (!g_host.qs) {
    g_host.qs = new spsim_b200_qset();
    g_host.qs->device = dev;
  }
  spsim_b200_qset *q = g_host.qs;
  const size_t need = 3 * (size_t)std::max<int64_t>(npix, 1) * sizeof(float);
  if (!q->d_hkl || q->cap_bytes < need) {
    cudaFree(q->d_hkl);
    q->d_hkl = nullptr;
    q->cap_bytes = 0;
    CUDA_TRY(cudaMalloc(&q->d_hkl, need));
    q->cap_bytes = need;
  }
  q->id = __atomic_fetch_add(&g_next_id, 1, __ATOMIC_RELAXED);
  q->npix = npix;
  q->row = 0;  // a list
  if (npix) CUDA_TRY(cudaMemcpy(q->d_hkl, hkl, 3 * npix * sizeof(float), cudaMemcpyHostToDevice));
  double qm2 = 0;
  for (long long i = 0; i < npix; ++i) {
    const double a = hkl[3 * i], b = hkl[3 * i + 1], c = hkl[3 * i + 2];
    qm2 = std::max(qm2, a * a + b * b + c * c);
  }
  q->qmax = std::sqrt(qm2);
  CUDA_TRY(set_steps(q, q->d_hkl, nullptr));
  *out = q;
  return SPSIM_OK;
}

// Frees this thread's host-call session and scratch plan (called by
// spsim_b200_release_scratch after a device synchronisation), the device's
// NUFFT grids and plans, and its cached adjoint plans.
static void nufft_release(int dev);
static void adjoint_release(int dev);

extern "C" void spsim_internal_release_host_session(void) {
  int dev = -1;
  cudaGetDevice(&dev);
  nufft_release(dev);
  adjoint_release(dev);
  if (g_host.device == dev) {
    if (g_host.mol) spsim_b200_molecule_destroy(g_host.mol);
    if (g_host.qs) spsim_b200_qset_destroy(g_host.qs);
    delete g_host.F;
    delete g_host.I;
    delete g_host.stats;
    // the shot's q sets borrow their lists: detach before deleting
    for (spsim_b200_qset *v : g_host.views) {
      v->d_hkl = nullptr;
      delete v;
    }
    if (g_host.shot_q) {
      g_host.shot_q->d_hkl = nullptr;
      delete g_host.shot_q;
    }
    for (Plan *p : g_host.part_plans) delete p;
  }
  g_host = HostSession();
  g_shot_mol = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_upload_stage.release();
  }
  if (g_oneshot.plan && g_oneshot.device == dev) delete g_oneshot.plan;
  g_oneshot = OneShot();
}

static int structure_factor_host(int natoms, const int32_t *Z, const float *pos, const float *occ, const float *bfac,
                                 float B, int delta_atoms, const float *beam, float wavelength, float bandwidth,
                                 int samples, int64_t npix, const float *hkl, int precision, float *F_host,
                                 float *I_host) {
  if (npix < 0 || (npix > 0 && !hkl)) return fail(SPSIM_ERR_INVALID_ARG, "bad HKL list");
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  if (g_host.device != dev) {
    g_host = HostSession();
    g_host.device = dev;
  }
  spsim_b200_molecule *m = nullptr;
  spsim_b200_qset *q = nullptr;
  st = host_session_molecule(natoms, Z, pos, occ, bfac, delta_atoms, beam, &m);
  if (st) return st;
  st = host_session_qset(npix, hkl, &q);
  if (st) return st;
  if (!g_host.F) g_host.F = new DevBuf();
  if (!g_host.I) g_host.I = new DevBuf();
  CUDA_TRY(g_host.F->ensure(2 * std::max<int64_t>(npix, 1) * sizeof(float)));
  CUDA_TRY(g_host.I->ensure(std::max<int64_t>(npix, 1) * sizeof(float)));
  float *F[1] = {F_host ? (float *)g_host.F->p : nullptr};
  float *I[1] = {I_host ? (float *)g_host.I->p : nullptr};
  const spsim_b200_molecule *mm = m;
  const spsim_b200_qset *qq = q;
  st = forward_spectrum(mm, qq, nullptr, B, precision, wavelength, bandwidth, samples, F[0], I[0], nullptr, false);
  if (st) return st;
  if (F_host && npix) CUDA_TRY(cudaMemcpy(F_host, F[0], 2 * npix * sizeof(float), cudaMemcpyDeviceToHost));
  if (I_host && npix) CUDA_TRY(cudaMemcpy(I_host, I[0], npix * sizeof(float), cudaMemcpyDeviceToHost));
  return SPSIM_OK;
}

// ---------------------------------------------------------------------------
// The reference-shaped simulate_shot path (host/legacy.c): the structure
// factor of host atom arrays on a float HKL list already in device memory,
// F and I left in device memory.  Internal to the library (not exported).

// The session q set takes a device float list: copied device to device, its
// largest |q| and neighbour step measured on the device.
static int host_session_qset_device(int64_t npix, const float *hkl_dev, cudaStream_t stream, spsim_b200_qset **out) {
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  if (!g_host.qs) {
    g_host.qs = new spsim_b200_qset();
    g_host.qs->device = dev;
  }
  spsim_b200_qset *q = g_host.qs;
  const size_t need = 3 * (size_t)std::max<int64_t>(npix, 1) * sizeof(float);
  if (!q->d_hkl || q->cap_bytes < need) {
    cudaFree(q->d_hkl);
    q->d_hkl = nullptr;
    q->cap_bytes = 0;
    CUDA_TRY(cudaMalloc(&q->d_hkl, need));
    q->cap_bytes = need;
  }
  q->id = __atomic_fetch_add(&g_next_id, 1, __ATOMIC_RELAXED);
  q->npix = npix;
  q->row = 0;  // a list (callers that know the detector's rows set it)
  if (npix)
    CUDA_TRY(cudaMemcpyAsync(q->d_hkl, hkl_dev, 3 * npix * sizeof(float), cudaMemcpyDeviceToDevice, stream));
  if (!g_host.stats) g_host.stats = new DevBuf();
  CUDA_TRY(g_host.stats->ensure(4 * sizeof(unsigned long long)));
  double steps[3];
  CUDA_TRY(qset_stats(q->d_hkl, npix, (unsigned long long *)g_host.stats->p, &q->qmax, steps, stream));
  q->pair_step = steps[0];
  q->quad_step1 = steps[1];
  q->quad_step2 = steps[2];
  *out = q;
  return SPSIM_OK;
}

// The session molecule for the caller's atom arrays, made ready before the
// shot's geometry is queued (a changed molecule synchronises the device before
// it takes over the old one's buffers, and then finds it idle); the structure
// factor call that follows uses it without comparing the arrays again.

extern "C" int spsim_internal_shot_molecule(int natoms, const int32_t *Z, const float *pos, int delta_atoms,
                                            const float *beam) {
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  if (g_host.device != dev) {
    g_host = HostSession();
    g_host.device = dev;
  }
  g_shot_mol = nullptr;
  g_host.parts = 0;
  spsim_b200_molecule *m = nullptr;
  st = host_session_molecule(natoms, Z, pos, nullptr, nullptr, delta_atoms, beam, &m);
  if (st) return st;
  g_shot_mol = m;
  return SPSIM_OK;
}

// Enqueued on the legacy default stream and not waited for: the caller
// synchronises, then calls spsim_internal_shot_check for kernel-side errors.
extern "C" int spsim_internal_shot_structure_factor(int natoms, const int32_t *Z, const float *pos, float B,
                                                    int delta_atoms, const float *beam, float wavelength,
                                                    float bandwidth, int samples, int64_t npix, const float *hkl_dev,
                                                    int precision, float *F_dev, float *I_dev) {
  if (npix < 0 || (npix > 0 && !hkl_dev)) return fail(SPSIM_ERR_INVALID_ARG, "bad HKL list");
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  if (g_host.device != dev) {
    g_host = HostSession();
    g_host.device = dev;
  }
  spsim_b200_molecule *m = g_shot_mol;
  g_shot_mol = nullptr;
  spsim_b200_qset *q = nullptr;
  if (!m || m != g_host.mol) {
    st = host_session_molecule(natoms, Z, pos, nullptr, nullptr, delta_atoms, beam, &m);
    if (st) return st;
  }
  st = host_session_qset_device(npix, hkl_dev, nullptr, &q);
  if (st) return st;
  return forward_spectrum(m, q, nullptr, B, precision, wavelength, bandwidth, samples, F_dev, I_dev, nullptr, false,
                          false);
}

// The pipelined simulate_shot (monochromatic direct sum): the session q set
// takes the whole HKL list once (its statistics decide the kernel form of
// every chunk), then each row chunk [p0, p1) runs on a view of it with its own
// scratch plan, on the caller's stream, not waited for.
extern "C" int spsim_internal_shot_parts_begin(int64_t npix, const float *hkl_dev) {
  if (npix < 0 || (npix > 0 && !hkl_dev)) return fail(SPSIM_ERR_INVALID_ARG, "bad HKL list");
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  if (g_host.device != dev || !g_shot_mol || g_shot_mol != g_host.mol)
    return fail(SPSIM_ERR_INVALID_ARG, "no shot molecule on this device");
  // the caller's list stays put for the shot: borrowed, not copied (a device
  // copy would queue behind the list's copy to the host on the copy engine)
  if (!g_host.shot_q) g_host.shot_q = new spsim_b200_qset();
  spsim_b200_qset *q = g_host.shot_q;
  q->device = dev;
  q->id = __atomic_fetch_add(&g_next_id, 1, __ATOMIC_RELAXED);
  q->npix = npix;
  q->d_hkl = const_cast<float *>(hkl_dev);
  q->d_q64 = nullptr;
  q->cap_bytes = 0;
  if (!g_host.stats) g_host.stats = new DevBuf();
  CUDA_TRY(g_host.stats->ensure(4 * sizeof(unsigned long long)));
  double steps[3];
  CUDA_TRY(qset_stats(q->d_hkl, npix, (unsigned long long *)g_host.stats->p, &q->qmax, steps, nullptr));
  q->pair_step = steps[0];
  q->quad_step1 = steps[1];
  q->quad_step2 = steps[2];
  g_host.parts = 0;
  return SPSIM_OK;
}

extern "C" int spsim_internal_shot_part(int64_t p0, int64_t p1, float B, int precision, float *F_dev, float *I_dev,
                                        void *stream) {
  spsim_b200_qset *q = g_host.shot_q;
  spsim_b200_molecule *m = g_host.mol;
  if (!q || !m || g_shot_mol != m) return fail(SPSIM_ERR_INVALID_ARG, "shot parts without a prepared shot");
  if (p0 < 0 || p1 > q->npix || p0 >= p1 || p0 % 4) return fail(SPSIM_ERR_INVALID_ARG, "bad shot part");
  const int k = g_host.parts;
  if ((int)g_host.views.size() <= k) {
    g_host.views.push_back(new spsim_b200_qset());
    g_host.part_plans.push_back(new Plan());
  }
  spsim_b200_qset *v = g_host.views[k];
  v->device = q->device;
  v->id = __atomic_fetch_add(&g_next_id, 1, __ATOMIC_RELAXED);
  v->npix = p1 - p0;
  v->d_hkl = q->d_hkl + 3 * p0;  // borrowed: views own no device memory
  v->d_q64 = nullptr;
  v->cap_bytes = 0;
  v->qmax = q->qmax;
  v->pair_step = q->pair_step;
  v->quad_step1 = q->quad_step1;
  v->quad_step2 = q->quad_step2;
  g_host.parts = k + 1;
  float *F[1] = {F_dev + 2 * p0};
  float *I[1] = {I_dev + p0};
  const spsim_b200_qset *qv = v;
  const spsim_b200_molecule *mc = m;
  g_split_pixels_hint = q->npix;
  const int st = run_forward(1, &mc, &qv, nullptr, B, precision, F, I, (cudaStream_t)stream, false, nullptr, false,
                             g_host.part_plans[k]);
  g_split_pixels_hint = 0;
  return st;
}

static int nufft_check_flags(int dev);

extern "C" int spsim_internal_shot_check(void) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lk(g_mu);
    int st = nufft_check_flags(dev);
    if (st) return st;
  }
  if (g_host.parts > 0) {
    const int n = g_host.parts;
    g_host.parts = 0;
    for (int k = 0; k < n; ++k) {
      const int st = check_flags(*g_host.part_plans[k]);
      if (st) return st;
    }
    return SPSIM_OK;
  }
  if (!g_oneshot.plan) return SPSIM_OK;
  return check_flags(*g_oneshot.plan);
}

extern "C" int spsim_internal_rotate_hkl(int64_t npix, const float R[9], float *hkl_dev) {
  CUDA_TRY(launch_rotate_hkl(npix, R, hkl_dev, nullptr));
  return SPSIM_OK;
}

extern "C" int spsim_b200_structure_factor_host(int natoms, const int32_t *Z, const float *pos, const float *occ,
                                                const float *bfac, float B, int delta_atoms, const float *beam,
                                                int64_t npix, const float *hkl, int precision, float *F_host,
                                                float *I_host) {
  return structure_factor_host(natoms, Z, pos, occ, bfac, B, delta_atoms, beam, 0.0f, 0.0f, 1, npix, hkl, precision,
                               F_host, I_host);
}

extern "C" int spsim_b200_structure_factor_host_spectrum(int natoms, const int32_t *Z, const float *pos,
                                                         const float *occ, const float *bfac, float B, int delta_atoms,
                                                         const float *beam, float wavelength, float bandwidth,
                                                         int samples, int64_t npix, const float *hkl, int precision,
                                                         float *F_host, float *I_host) {
  return structure_factor_host(natoms, Z, pos, occ, bfac, B, delta_atoms, beam, wavelength, bandwidth, samples, npix,
                               hkl, precision, F_host, I_host);
}

// ---------------------------------------------------------------------------
// Non-uniform FFT structure factor (nufft_kernels.cuh): the same F(q) as the
// direct sum, computed per element by spreading the atoms onto a real-space
// grid, one batched 3-D FFT and interpolation at every pixel's q, with FP64
// grids.  Its cost is O(atoms w^3 + grid log grid + pixels w^3) instead of
// O(atoms x pixels).  One context per device, under g_mu; calls on different
// streams are ordered by the context's completion event.

struct NufftCtx {
  DevBuf small, fa, fb, packed, dec, tw, seg, keys, flags, rots;
  FftAxis ax[3];  // the pruned FFT passes (twiddle tables in tw)
  std::vector<double> geom_key;   // inputs the q box was read for
  std::vector<double> size_key;   // q box, bound, elements, eps the grids were sized for
  unsigned long long seg_mol = 0;  // molecule whose segment table is on the device
  NufftGeom g;
  int n_coef = 0;
  int copies = 1;  // spreading-grid copies
  double psi_a[NUFFT_MAX_COEF];
  unsigned long long *h_keys = nullptr;  // pinned bounds read-back
  cudaEvent_t done = nullptr;
  bool has_done = false;
  // a pipelined shot's interpolation chunks read the grids after the call
  // that prepared them has returned: from then until its last chunk is
  // queued, other threads' NUFFT calls on the device wait
  bool shot_open = false;
  std::thread::id shot_owner;
};
static std::map<int, NufftCtx> g_nufft;
static std::condition_variable g_nufft_cv;  // signalled when a shot releases its device's grids

// under g_mu: no other thread's pipelined shot holds the device's grids
static bool nufft_free_for_this_thread(int dev) {
  const auto it = g_nufft.find(dev);
  return it == g_nufft.end() || !it->second.shot_open || it->second.shot_owner == std::this_thread::get_id();
}
static thread_local int g_last_nufft_w[2] = {0, 0};
static thread_local int g_last_nufft_n2[3] = {0, 0, 0};

static int fft_size(int n) {  // smallest even size >= n with prime factors 2, 3, 5, 7
  for (int m = std::max(n, 2);; ++m) {
    if (m & 1) continue;
    int r = m;
    for (int f : {2, 3, 5, 7})
      while (r % f == 0) r /= f;
    if (r == 1) return m;
  }
}

static double es_host(double u, double w, double beta) {
  const double t = 2.0 * u / w, a = 1.0 - t * t;
  return a >= 0.0 ? std::exp(beta * (std::sqrt(a) - 1.0)) : 0.0;
}

// Fourier transform of the ES kernel, int es(u) e^{-2 pi i xi u} du, by the
// trapezoid rule at spacing d (spectrally accurate: the kernel is smooth and
// vanishes to e^{-beta} at its ends)
static double es_hat_host(double xi, double w, double beta, double d) {
  const int n = (int)std::floor(0.5 * w / d);
  double s = 0.5 * es_host(0.0, w, beta);
  for (int i = 1; i <= n; ++i) s += es_host(i * d, w, beta) * std::cos(2.0 * M_PI * xi * i * d);
  return 2.0 * d * s;
}

// Interpolation kernel width (grid points) for a requested relative error of
// F: measured relative L2 errors against the direct sum are 1 to 4 x 10^-(w-1)
// with an FFT grid upsampled 2x; the spreading kernel, w + 3 points wide on a
// grid upsampled 1.5x, adds less (a wider one measured no better).
static int nufft_width(double eps) {
  const int w = (int)std::ceil(-std::log10(eps)) + 1;
  return std::min(std::max(w, NUFFT_MIN_W), NUFFT_MAX_W - 1);
}

// npat patterns of one molecule and q set, pattern i rotated by rot[9 i] (or
// none), outputs [npat][npix].  ball: size the grid for the ball |R q| <=
// |q|max instead of the box of the rotated list, so that it holds for every
// rotation (no read-back; the grid of a batch of orientations).  deferred:
// prepare the grid (spread and FFT passes) and return the interpolation's
// arguments there (F, I unset) instead of launching it; *deferred_empty is
// set when there is nothing to interpolate (no atoms or no pixels: the
// outputs are zeros).
static int nufft_forward(const spsim_b200_molecule *m, const spsim_b200_qset *qs, int npat, const double *rot,
                         bool ball, float B, double eps, float *F_dev, float *I_dev, cudaStream_t st,
                         NufftInterp *deferred = nullptr, bool *deferred_empty = nullptr) {
  if (!m || !qs) return fail(SPSIM_ERR_INVALID_ARG, "NULL handle");
  if (npat < 1 || npat > 65535) return fail(SPSIM_ERR_INVALID_ARG, "npatterns %d outside [1, 65535]", npat);
  if (!(eps >= 1e-14 && eps <= 1e-2)) return fail(SPSIM_ERR_INVALID_ARG, "eps %g outside [1e-14, 1e-2]", eps);
  if (m->per_atom_b)
    return fail(SPSIM_ERR_INVALID_ARG, "per-atom B factors are not supported by the NUFFT structure factor");
  int dev;
  int st0 = current_device(&dev);
  if (st0) return st0;
  if (m->device != dev || qs->device != dev) return fail(SPSIM_ERR_INVALID_ARG, "handle belongs to another device");
  const long long npix = qs->npix;
  if (deferred_empty) *deferred_empty = npix == 0 || m->n_kept == 0;
  if (npix == 0) return SPSIM_OK;
  if (m->n_kept == 0) {
    if (F_dev) CUDA_TRY(cudaMemsetAsync(F_dev, 0, 2 * npix * npat * sizeof(float), st));
    if (I_dev) CUDA_TRY(cudaMemsetAsync(I_dev, 0, npix * npat * sizeof(float), st));
    return SPSIM_OK;
  }
  double qball = qs->qmax;  // |R q| <= |q|max ||R||, ||R|| = 1 for rotations, <= Frobenius otherwise
  if (rot)
    for (int i = 0; i < npat; ++i)
      if (!is_orthonormal(rot + 9 * (size_t)i)) {
        double fro = 0;
        for (int k = 0; k < 9; ++k) fro += rot[9 * (size_t)i + k] * rot[9 * (size_t)i + k];
        qball = std::max(qball, qs->qmax * std::sqrt(fro));
      }
  std::unique_lock<std::mutex> lk(g_mu);
  g_nufft_cv.wait(lk, [dev] { return nufft_free_for_this_thread(dev); });
  NufftCtx &c = g_nufft[dev];
  if (!c.h_keys) CUDA_TRY(cudaMallocHost(&c.h_keys, 6 * sizeof(unsigned long long)));
  if (!c.done) CUDA_TRY(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming));
  if (c.has_done) CUDA_TRY(cudaStreamWaitEvent(st, c.done, 0));  // the buffers' previous user
  CUDA_TRY(c.flags.ensure(sizeof(int)));
  if (!c.has_done) CUDA_TRY(cudaMemsetAsync(c.flags.p, 0, sizeof(int), st));

  const int n_elem = m->n_elem;
  std::vector<double> key;
  if (ball) {
    key = {-1.0, qball, m->rbound, (double)n_elem, eps};
  } else {
    key = {(double)qs->id, (double)npix, m->rbound, (double)n_elem, eps, rot ? 1.0 : 0.0};
    if (rot) key.insert(key.end(), rot, rot + 9);
  }
  if (key != c.geom_key) {
    c.geom_key.clear();
    double lo[3], hi[3];
    if (ball) {
      if (!std::isfinite(qball)) return fail(SPSIM_ERR_INVALID_ARG, "NUFFT: non-finite q in the list");
      for (int d = 0; d < 3; ++d) {
        lo[d] = -qball;
        hi[d] = qball;
      }
    } else {
      // q box of R q over the list (one read-back), then the grids
      CUDA_TRY(c.keys.ensure(6 * sizeof(unsigned long long)));
      unsigned long long *dk = (unsigned long long *)c.keys.p;
      CUDA_TRY(nufft_bounds(qs->d_hkl, qs->d_q64, npix, rot, dk, st));
      CUDA_TRY(cudaMemcpyAsync(c.h_keys, dk, 6 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
      CUDA_TRY(cudaStreamSynchronize(st));
      for (int d = 0; d < 3; ++d) {
        lo[d] = nufft_key_to_double(c.h_keys[d]);
        hi[d] = nufft_key_to_double(c.h_keys[3 + d]);
        if (!(std::isfinite(lo[d]) && std::isfinite(hi[d])))
          return fail(SPSIM_ERR_INVALID_ARG, "NUFFT: non-finite q in the list");
      }
    }
    // the grids follow from the q box, the molecule's bound, the elements and
    // eps: an unchanged box (a new list of the same detector, say) keeps them
    // (the molecule's bound enters only through the spreading grid's size n1)
    std::vector<double> size_key = {lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], (double)n_elem, eps};
    {
      const int w1 = std::min(nufft_width(eps) + 3, NUFFT_MAX_W);
      for (int d = 0; d < 3; ++d) {
        const double S = std::max(0.5 * (hi[d] - lo[d]), 1e-3 / m->rbound);  // as below (a flat axis: from the bound)
        size_key.push_back(S);
        size_key.push_back(std::ceil(2.0 * m->rbound * (2.0 * 1.5 * S)) + w1 + 2);
      }
    }
    if (size_key != c.size_key) {
      c.size_key.clear();
      const int w = nufft_width(eps);
      const double sigma1 = 1.5, sigma2 = 2.0;  // spreading-grid and FFT-grid upsampling
      NufftGeom g;
      std::memset(&g, 0, sizeof(g));
      g.w1 = std::min(w + 3, NUFFT_MAX_W);
      g.w2 = w;
      g.beta1 = 0.97 * M_PI * g.w1 * (1.0 - 0.5 / sigma1);
      g.beta2 = 0.97 * M_PI * g.w2 * (1.0 - 0.5 / sigma2);
      const double X = m->rbound;
      size_t cells1 = 1, cells2 = 1;
      for (int d = 0; d < 3; ++d) {
        g.cq[d] = 0.5 * (lo[d] + hi[d]);
        const double S = std::max(0.5 * (hi[d] - lo[d]), 1e-3 / X);
        g.h[d] = 1.0 / (2.0 * sigma1 * S);
        g.inv_h[d] = 2.0 * sigma1 * S;
        const double n1 = std::ceil(2.0 * X * g.inv_h[d]) + g.w1 + 2;
        if (n1 > 4096) return fail(SPSIM_ERR_INVALID_ARG, "NUFFT: %.0f grid points along axis %d; use the direct sum", n1, d);
        g.n1[d] = (int)n1 + ((int)n1 & 1);
        g.n2[d] = fft_size((int)std::ceil(sigma2 * g.n1[d]));
        if (g.n2[d] > NUFFT_FFT_MAX)
          return fail(SPSIM_ERR_INVALID_ARG, "NUFFT: FFT of %d points along axis %d; use the direct sum", g.n2[d], d);
        g.L[d] = g.h[d] * g.n2[d];
        // the interpolation's stencils start at ceil(t - w/2), t = (q - cq) L,
        // for t in [(lo - cq) L, (hi - cq) L]: the output box, 2 points of margin
        const double tlo = (lo[d] - g.cq[d]) * g.L[d], thi = (hi[d] - g.cq[d]) * g.L[d];
        g.pmin[d] = (int)std::floor(tlo - 0.5 * w) - 2;
        g.m[d] = (int)std::ceil(thi - 0.5 * w) + w - 1 + 2 - g.pmin[d] + 1;
        cells1 *= (size_t)g.n1[d];
        cells2 *= (size_t)g.m[d];
      }
      // copies of the spreading grid while they stay small next to L2 (32 MB):
      // about 1,000 updates of one cell from 20,000 atoms on a 40 x 40 x 18 grid
      // otherwise serialise in the atomic units
      const size_t one1 = cells1 * n_elem * sizeof(double2);
      c.copies = (int)std::max<size_t>(1, std::min<size_t>(8, (32u << 20) / std::max<size_t>(one1, 1)));
      // x pass output [E][n1z][n1y][m_x], y pass output [E][n1z][m_y][m_x],
      // z pass output (the interpolation's FP32 grid) over the box
      const size_t bytes1 = one1 * c.copies;
      const size_t bytes_a = (size_t)n_elem * g.n1[2] * g.n1[1] * g.m[0] * sizeof(double2);
      const size_t bytes_b = (size_t)n_elem * g.n1[2] * g.m[1] * g.m[0] * sizeof(double2);
      const size_t bytes3 = cells2 * nufft_pack_groups(n_elem) * nufft_pack_halves(n_elem) * sizeof(float4);
      size_t free_b = 0, total_b = 0;
      CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
      const size_t have = free_b + c.small.cap + c.fa.cap + c.fb.cap + c.packed.cap;
      if (bytes1 + bytes_a + bytes_b + bytes3 > have / 10 * 9)
        return fail(SPSIM_ERR_INVALID_ARG, "NUFFT: grids of %.3g GB do not fit; use the direct sum",
                    (double)(bytes1 + bytes_a + bytes_b + bytes3) * 1e-9);
      // 1 / phi2hat per spreading-grid index, and psi1hat's trapezoid coefficients
      std::vector<double> dec;
      for (int d = 0; d < 3; ++d)
        for (int l = 0; l < g.n1[d]; ++l)
          dec.push_back(1.0 / es_hat_host((double)(l - g.n1[d] / 2) / g.n2[d], g.w2, g.beta2, 0.01));
      c.n_coef = (int)std::floor(0.5 * g.w1 / 0.25) + 1;
      for (int k = 0; k < c.n_coef; ++k) c.psi_a[k] = 0.25 * (k == 0 ? 1.0 : 2.0) * es_host(0.25 * k, g.w1, g.beta1);
      // twiddle tables of the three transforms, after dec in one upload
      std::vector<double2> tw((size_t)g.n2[0] + g.n2[1] + g.n2[2]);
      size_t tw_at[3];
      for (int d = 0, at = 0; d < 3; at += g.n2[d], ++d) {
        tw_at[d] = at;
        nufft_fft_twiddles(g.n2[d], tw.data() + at);
      }
      CUDA_TRY(c.small.ensure(bytes1));
      CUDA_TRY(c.fa.ensure(bytes_a));
      CUDA_TRY(c.fb.ensure(bytes_b));
      CUDA_TRY(c.packed.ensure(bytes3));
      CUDA_TRY(c.dec.ensure(dec.size() * sizeof(double)));
      CUDA_TRY(c.tw.ensure(tw.size() * sizeof(double2)));
      CUDA_TRY(cudaMemcpyAsync(c.dec.p, dec.data(), dec.size() * sizeof(double), cudaMemcpyHostToDevice, st));
      CUDA_TRY(cudaMemcpyAsync(c.tw.p, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
      for (int d = 0; d < 3; ++d)
        if (nufft_fft_axis(g.n2[d], g.n1[d], g.pmin[d], g.m[d], (const double2 *)c.tw.p + tw_at[d], &c.ax[d]))
          return fail(SPSIM_ERR_UNSUPPORTED, "NUFFT: no FFT pass for %d points", g.n2[d]);
      // the read-back and the uploads above are complete when this returns
      CUDA_TRY(cudaStreamSynchronize(st));
      c.g = g;
      c.size_key = size_key;
    }
    c.geom_key = key;
  }
  if (c.seg_mol != m->id) {
    // element segments of the padded atom records
    std::vector<int> seg(n_elem + 1, 0);
    for (const TileDesc &t : m->tiles) seg[t.elem + 1] = std::max(seg[t.elem + 1], t.atom_begin + t.count);
    CUDA_TRY(c.seg.ensure(seg.size() * sizeof(int)));
    CUDA_TRY(cudaMemcpy(c.seg.p, seg.data(), seg.size() * sizeof(int), cudaMemcpyHostToDevice));
    c.seg_mol = m->id;
  }
  NufftGeom g = c.g;
  for (int d = 0; d < 3; ++d) g.center[d] = m->center[d];
  size_t cells1 = (size_t)g.n1[0] * g.n1[1] * g.n1[2];
  CUDA_TRY(cudaMemsetAsync(c.small.p, 0, cells1 * n_elem * c.copies * sizeof(double2), st));
  CUDA_TRY(nufft_spread(m->d_atomsd, (const int *)c.seg.p, n_elem, m->n_padded, g, (double *)c.small.p, c.copies,
                        (int *)c.flags.p, st));
  CUDA_TRY(nufft_fft3((const double *)c.small.p, c.copies, (const double *)c.dec.p, g, n_elem, c.ax,
                      (double2 *)c.fa.p, (double2 *)c.fb.p, (float4 *)c.packed.p, st));
  const long long cells2 = (long long)g.m[0] * g.m[1] * g.m[2];
  NufftInterp a;
  std::memset(&a, 0, sizeof(a));
  a.g = g;
  a.hkl = qs->d_hkl;
  a.q64 = qs->d_q64;
  a.npix = npix;
  a.tile_nx = qs->row > 0 && npix % qs->row == 0 ? qs->row : 0;
  a.npat = npat;
  if (npat > 1 && rot) {
    CUDA_TRY(c.rots.ensure(9 * (size_t)npat * sizeof(double)));
    CUDA_TRY(cudaMemcpyAsync(c.rots.p, rot, 9 * (size_t)npat * sizeof(double), cudaMemcpyHostToDevice, st));
    a.rots = (const double *)c.rots.p;
  } else {
    a.has_rot = rot != nullptr;
    for (int k = 0; k < 9; ++k) a.rot[k] = rot ? rot[k] : 0.0;
  }
  a.packed = (const float4 *)c.packed.p;
  a.cell2 = cells2;
  a.halves = nufft_pack_halves(n_elem);
  a.n_groups = nufft_pack_groups(n_elem);
  a.n_elem = n_elem;
  a.coeffs = m->d_coeffs;
  a.B = (double)B;
  a.delta_atoms = m->delta_atoms;
  a.n_coef = c.n_coef;
  std::memcpy(a.psi_a, c.psi_a, sizeof(a.psi_a));
  a.F = (float2 *)F_dev;
  a.I = I_dev;
  if (deferred) {
    *deferred = a;
    c.shot_open = true;
    c.shot_owner = std::this_thread::get_id();
  } else {
    CUDA_TRY(nufft_interp(a, st));
  }
  CUDA_TRY(cudaEventRecord(c.done, st));
  c.has_done = true;
  g_last_nufft_w[0] = g.w1;
  g_last_nufft_w[1] = g.w2;
  for (int d = 0; d < 3; ++d) g_last_nufft_n2[d] = g.n2[d];
  return SPSIM_OK;
}

static void nufft_release(int dev) {
  std::unique_lock<std::mutex> lk(g_mu);
  g_nufft_cv.wait(lk, [dev] { return nufft_free_for_this_thread(dev); });
  auto it = g_nufft.find(dev);
  if (it == g_nufft.end()) return;
  NufftCtx &c = it->second;
  if (c.h_keys) cudaFreeHost(c.h_keys);
  if (c.done) cudaEventDestroy(c.done);
  g_nufft.erase(it);  // the grids' DevBufs free themselves
}

// Sticky error word of this device's NUFFT context (atoms outside the grid).
static int nufft_check_flags(int dev) {
  auto it = g_nufft.find(dev);
  if (it == g_nufft.end() || !it->second.flags.p) return SPSIM_OK;
  int h = 0;
  CUDA_TRY(cudaMemcpy(&h, it->second.flags.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    CUDA_TRY(cudaMemset(it->second.flags.p, 0, sizeof(int)));
    return fail(SPSIM_ERR_RANGE, "NUFFT: atoms outside the molecule's creation-time bounds");
  }
  return SPSIM_OK;
}

extern "C" int spsim_b200_forward_nufft(const spsim_b200_molecule *m, const spsim_b200_qset *qs, const double *rot,
                                        float B, double eps, float *F_dev, float *I_dev, void *stream) {
  return nufft_forward(m, qs, 1, rot, false, B, eps, F_dev, I_dev, (cudaStream_t)stream);
}

extern "C" int spsim_b200_forward_nufft_batch(const spsim_b200_molecule *m, const spsim_b200_qset *qs, int npatterns,
                                              const double *rot, float B, double eps, float *F_dev, float *I_dev,
                                              void *stream) {
  return nufft_forward(m, qs, npatterns, rot, true, B, eps, F_dev, I_dev, (cudaStream_t)stream);
}

extern "C" int spsim_b200_set_nufft_interp(int mode) {
  if (mode != 0 && mode != 1) return fail(SPSIM_ERR_INVALID_ARG, "NUFFT interpolation mode %d (0 or 1)", mode);
  std::lock_guard<std::mutex> lk(g_mu);
  nufft_set_interp_mode(mode);
  return SPSIM_OK;
}

extern "C" int spsim_b200_last_nufft_grid(int *w_spread, int *w_interp, int *n2) {
  if (w_spread) *w_spread = g_last_nufft_w[0];
  if (w_interp) *w_interp = g_last_nufft_w[1];
  if (n2)
    for (int d = 0; d < 3; ++d) n2[d] = g_last_nufft_n2[d];
  return SPSIM_OK;
}

// Host arrays in and out (the reference-shaped NFFT path): the session
// molecule and q set of the direct host calls, synchronised before return.
extern "C" int spsim_b200_structure_factor_host_nufft(int natoms, const int32_t *Z, const float *pos, float B,
                                                      int delta_atoms, int64_t npix, const float *hkl, double eps,
                                                      float *F_host, float *I_host) {
  if (npix < 0 || (npix > 0 && !hkl)) return fail(SPSIM_ERR_INVALID_ARG, "bad HKL list");
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  if (g_host.device != dev) {
    g_host = HostSession();
    g_host.device = dev;
  }
  spsim_b200_molecule *m = nullptr;
  spsim_b200_qset *q = nullptr;
  st = host_session_molecule(natoms, Z, pos, nullptr, nullptr, delta_atoms, nullptr, &m);
  if (st) return st;
  st = host_session_qset(npix, hkl, &q);
  if (st) return st;
  if (!g_host.F) g_host.F = new DevBuf();
  if (!g_host.I) g_host.I = new DevBuf();
  CUDA_TRY(g_host.F->ensure(2 * std::max<int64_t>(npix, 1) * sizeof(float)));
  CUDA_TRY(g_host.I->ensure(std::max<int64_t>(npix, 1) * sizeof(float)));
  float *F = F_host ? (float *)g_host.F->p : nullptr;
  float *I = I_host ? (float *)g_host.I->p : nullptr;
  st = nufft_forward(m, q, 1, nullptr, false, B, eps, F, I, nullptr);
  if (st) return st;
  CUDA_TRY(cudaStreamSynchronize(nullptr));
  {
    std::lock_guard<std::mutex> lk(g_mu);
    st = nufft_check_flags(dev);
  }
  if (st) return st;
  if (F_host && npix) CUDA_TRY(cudaMemcpy(F_host, F, 2 * npix * sizeof(float), cudaMemcpyDeviceToHost));
  if (I_host && npix) CUDA_TRY(cudaMemcpy(I_host, I, npix * sizeof(float), cudaMemcpyDeviceToHost));
  return SPSIM_OK;
}

// simulate_shot with use_nfft_for_sf: the session molecule (unit weights) on
// the device HKL list, enqueued on the legacy default stream like
// spsim_internal_shot_structure_factor.
extern "C" int spsim_internal_shot_structure_factor_nufft(int natoms, const int32_t *Z, const float *pos, float B,
                                                          int delta_atoms, int64_t npix, const float *hkl_dev,
                                                          int row, double eps, float *F_dev, float *I_dev) {
  if (npix < 0 || (npix > 0 && !hkl_dev)) return fail(SPSIM_ERR_INVALID_ARG, "bad HKL list");
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  if (g_host.device != dev) {
    g_host = HostSession();
    g_host.device = dev;
  }
  spsim_b200_molecule *m = g_shot_mol;
  g_shot_mol = nullptr;
  spsim_b200_qset *q = nullptr;
  if (!m || m != g_host.mol) {
    st = host_session_molecule(natoms, Z, pos, nullptr, nullptr, delta_atoms, nullptr, &m);
    if (st) return st;
  }
  st = host_session_qset_device(npix, hkl_dev, nullptr, &q);
  if (st) return st;
  // a detector's rows: the interpolation takes its pixel-tile path
  q->row = row > 0 && npix % row == 0 ? row : 0;
  return nufft_forward(m, q, 1, nullptr, false, B, eps, F_dev, I_dev, nullptr);
}

// The pipelined simulate_shot with the NUFFT structure factor: the grid is
// prepared once (spread, FFT passes), then each whole-row chunk [p0, p1) is
// interpolated on the legacy stream, in order, so that its detector chain and
// copies overlap the next chunk's interpolation.
static thread_local NufftInterp g_shot_interp;
static thread_local bool g_shot_interp_empty = true;
static thread_local int64_t g_shot_npix = 0;  // pixels of the prepared shot (also when it has no atoms)

extern "C" int spsim_internal_shot_nufft_begin(int natoms, const int32_t *Z, const float *pos, float B,
                                               int delta_atoms, int64_t npix, const float *hkl_dev, int row,
                                               double eps) {
  if (npix < 0 || (npix > 0 && !hkl_dev)) return fail(SPSIM_ERR_INVALID_ARG, "bad HKL list");
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  if (g_host.device != dev) {
    g_host = HostSession();
    g_host.device = dev;
  }
  spsim_b200_molecule *m = g_shot_mol;
  g_shot_mol = nullptr;
  spsim_b200_qset *q = nullptr;
  if (!m || m != g_host.mol) {
    st = host_session_molecule(natoms, Z, pos, nullptr, nullptr, delta_atoms, nullptr, &m);
    if (st) return st;
  }
  st = host_session_qset_device(npix, hkl_dev, nullptr, &q);
  if (st) return st;
  q->row = row > 0 && npix % row == 0 ? row : 0;
  g_shot_interp_empty = true;
  g_shot_npix = npix;
  return nufft_forward(m, q, 1, nullptr, false, B, eps, nullptr, nullptr, nullptr, &g_shot_interp,
                       &g_shot_interp_empty);
}

extern "C" int spsim_internal_shot_nufft_part(int64_t p0, int64_t p1, float *F_dev, float *I_dev) {
  NufftInterp a = g_shot_interp;
  if (p0 < 0 || p1 > g_shot_npix || p0 >= p1) return fail(SPSIM_ERR_INVALID_ARG, "bad NUFFT shot part");
  if (g_shot_interp_empty) {
    CUDA_TRY(cudaMemsetAsync(F_dev + 2 * p0, 0, 2 * (p1 - p0) * sizeof(float), nullptr));
    CUDA_TRY(cudaMemsetAsync(I_dev + p0, 0, (p1 - p0) * sizeof(float), nullptr));
    return SPSIM_OK;
  }
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_nufft.find(dev);
  if (it == g_nufft.end()) return fail(SPSIM_ERR_INVALID_ARG, "NUFFT shot part without a prepared grid");
  if (a.hkl) a.hkl += 3 * p0;
  if (a.q64) a.q64 += 3 * p0;
  a.npix = p1 - p0;
  if (a.tile_nx > 0 && (p0 % a.tile_nx || a.npix % a.tile_nx)) a.tile_nx = 0;
  a.F = (float2 *)F_dev + p0;
  a.I = I_dev + p0;
  const cudaError_t e = nufft_interp(a, nullptr);
  const cudaError_t er = cudaEventRecord(it->second.done, nullptr);
  if (p1 == g_shot_npix || e != cudaSuccess || er != cudaSuccess) {  // the last chunk: the grids are free again
    it->second.shot_open = false;
    g_nufft_cv.notify_all();
  }
  CUDA_TRY(e);
  CUDA_TRY(er);
  return SPSIM_OK;
}

// ---------------------------------------------------------------------------
// completion, timing, statistics, variants

extern "C" int spsim_b200_synchronize(void *stream) {
  CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto &p : g_plans) {
    int st = check_flags(*p);
    if (st) return st;
  }
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  return nufft_check_flags(dev);
}

extern "C" int spsim_b200_debug_stall_first_copy(int on) {
  int dev;
  int st = current_device(&dev);
  if (st) return st;
  std::lock_guard<std::mutex> lk(g_mu);
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(set_copy_stall(on));
  return SPSIM_OK;
}

extern "C" int spsim_b200_timing_enable(int enable) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_timing = enable != 0;
  return SPSIM_OK;
}

extern "C" int spsim_b200_timing_read(double *ms, int cap, int *n) {
  if (!n) return fail(SPSIM_ERR_INVALID_ARG, "n is NULL");
  std::lock_guard<std::mutex> lk(g_mu);
  int k = 0;
  for (auto &pr : g_timing_events) {
    float t = 0;
    CUDA_TRY(cudaEventSynchronize(pr.second));
    CUDA_TRY(cudaEventElapsedTime(&t, pr.first, pr.second));
    if (ms && k < cap) ms[k] = t;
    ++k;
    g_last_ms = t;
    cudaEventDestroy(pr.first);
    cudaEventDestroy(pr.second);
  }
  g_timing_events.clear();
  *n = std::min(k, cap);
  return SPSIM_OK;
}

extern "C" int spsim_b200_last_forward_stats(double *terms, double *kernel_ms) {
  if (terms) *terms = g_last_terms;
  if (kernel_ms) *kernel_ms = g_last_ms;
  return SPSIM_OK;
}

extern "C" int spsim_b200_last_variant(int *threads, int *pixels_per_thread, int *form) {
  if (threads) *threads = g_last_variant[0];
  if (pixels_per_thread) *pixels_per_thread = g_last_variant[1];
  if (form) *form = g_last_variant[2];
  return SPSIM_OK;
}

extern "C" int spsim_b200_last_phase_word(int *on) {
  if (on) *on = g_last_phase_word;
  return SPSIM_OK;
}

extern "C" int spsim_b200_last_pair_narrow(int *on) {
  if (on) *on = g_last_pair_narrow;
  return SPSIM_OK;
}

extern "C" int spsim_b200_set_variant(int threads, int pixels_per_thread, int packed) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (threads < 0) {
    g_force_nt = g_force_p = -1;
    g_force_pk = 3;
    return SPSIM_OK;
  }
  // form 4 exists for SPSIM_PREC_F32 only; FP32_FAST forwards ignore a forced
  // variant they have not compiled
  if (!sf_f32_variant_exists(0, threads, pixels_per_thread, packed) &&
      !sf_f32_variant_exists(1, threads, pixels_per_thread, packed))
    return fail(SPSIM_ERR_INVALID_ARG, "no compiled variant with %d threads x %d pixels (packed %d)", threads,
                pixels_per_thread, packed);
  g_force_nt = threads;
  g_force_p = pixels_per_thread;
  g_force_pk = packed;
  return SPSIM_OK;
}

// Times every compiled FP32 variant on one forward of the given patterns and
// keeps the fastest for workloads of that size class (total terms).
static int autotune_impl(int npat, const spsim_b200_molecule *const *mols, const spsim_b200_qset *const *qsets,
                         const double *rot, int precision, cudaStream_t stream, int *best_threads,
                         int *best_pixels_per_thread, int *best_packed) {
  if (npat < 1 || !mols || !qsets) return fail(SPSIM_ERR_INVALID_ARG, "no patterns to tune on");
  double terms = 0;
  long long total = 0;
  for (int i = 0; i < npat; ++i) {
    if (!mols[i] || !qsets[i]) return fail(SPSIM_ERR_INVALID_ARG, "pattern %d: NULL handle", i);
    terms += (double)qsets[i]->npix * mols[i]->n_kept;
    total += qsets[i]->npix;
  }
  if (precision == SPSIM_PREC_FP64) return fail(SPSIM_ERR_INVALID_ARG, "the FP64 kernel has a single variant");
  const int cand[][3] = {{128, 2, 0}, {128, 4, 0}, {256, 4, 0}, {128, 2, 1}, {128, 4, 1}, {256, 4, 1},
                         {128, 6, 1}, {128, 2, 2}, {128, 4, 2}, {256, 4, 2}, {128, 6, 2}, {128, 8, 2},
                         {128, 4, 3}, {128, 8, 3}, {128, 12, 3}, {256, 4, 3}, {128, 8, 4}, {128, 16, 4},
                         {256, 8, 4}};
  float *dI = nullptr;
  CUDA_TRY(cudaMalloc(&dI, std::max<long long>(total, 1) * sizeof(float)));
  std::vector<float *> I(npat), F(npat, nullptr);
  {
    long long off = 0;
    for (int i = 0; i < npat; ++i) {
      I[i] = dI + off;
      off += qsets[i]->npix;
    }
  }
  float best = 1e30f;
  int bt = 128, bp = 4, bk = 2;
  const int saved_nt = g_force_nt, saved_p = g_force_p, saved_pk = g_force_pk;
  const bool saved_timing = g_timing;
  int st = SPSIM_OK;
  for (auto &c : cand) {
    if (!sf_f32_variant_exists(precision == SPSIM_PREC_F32_FAST ? 1 : 0, c[0], c[1], c[2])) continue;
    g_force_nt = c[0];
    g_force_p = c[1];
    g_force_pk = c[2];
    // warm-up, then three timed launches
    st = run_forward(npat, mols, qsets, rot, 0.0f, precision, F.data(), I.data(), stream, false);
    if (st) break;
    float tot = 0;
    for (int r = 0; r < 3 && !st; ++r) {
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, stream);
      st = run_forward(npat, mols, qsets, rot, 0.0f, precision, F.data(), I.data(), stream, false);
      cudaEventRecord(b, stream);
      cudaEventSynchronize(b);
      float t = 0;
      cudaEventElapsedTime(&t, a, b);
      tot += t;
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
    if (st) break;
    if (tot < best) {
      best = tot;
      bt = c[0];
      bp = c[1];
      bk = c[2];
    }
  }
  g_force_nt = saved_nt;
  g_force_p = saved_p;
  g_force_pk = saved_pk;
  g_timing = saved_timing;
  cudaFree(dI);
  if (st) return st;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_tuned[size_class(terms) * 4 + precision] = {bt, bp, bk};
  }
  if (best_threads) *best_threads = bt;
  if (best_pixels_per_thread) *best_pixels_per_thread = bp;
  if (best_packed) *best_packed = bk;
  return SPSIM_OK;
}

extern "C" int spsim_b200_autotune(const spsim_b200_molecule *m, const spsim_b200_qset *qs, int precision,
                                   void *stream, int *best_threads, int *best_pixels_per_thread, int *best_packed) {
  if (!m || !qs) return fail(SPSIM_ERR_INVALID_ARG, "NULL handle");
  return autotune_impl(1, &m, &qs, nullptr, precision, (cudaStream_t)stream, best_threads, best_pixels_per_thread,
                       best_packed);
}

extern "C" int spsim_b200_clear_tuning(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_tuned.clear();
  return SPSIM_OK;
}

extern "C" int spsim_b200_autotune_batch(int npatterns, const spsim_b200_molecule *const *mols,
                                         const spsim_b200_qset *const *qsets, const double *rot, int precision,
                                         void *stream, int *best_threads, int *best_pixels_per_thread,
                                         int *best_form) {
  return autotune_impl(npatterns, mols, qsets, rot, precision, (cudaStream_t)stream, best_threads,
                       best_pixels_per_thread, best_form);
}

// ---------------------------------------------------------------------------
// geometry and detector chain

extern "C" int spsim_b200_crystal_lattice_sum(int64_t npix, const float *hkl_dev, const float *cell, int na, int nb,
                                              int nc, float *F_dev, float *I_dev, void *stream) {
  if (npix < 0 || (npix > 0 && (!hkl_dev || !F_dev)) || !cell)
    return fail(SPSIM_ERR_INVALID_ARG, "crystal lattice sum: bad arguments");
  if (na < 0 || nb < 0 || nc < 0) return fail(SPSIM_ERR_INVALID_ARG, "crystal size %d x %d x %d", na, nb, nc);
  double c[9];
  for (int k = 0; k < 9; ++k) c[k] = cell[k];
  CUDA_TRY(launch_crystal(npix, hkl_dev, c, na, nb, nc, F_dev, I_dev, (cudaStream_t)stream));
  return SPSIM_OK;
}

extern "C" int spsim_b200_hkl_for_3d_detector(int nx, int ny, int nz, float width, float height, float depth,
                                              float distance, float center_x, float center_y, float center_z,
                                              float wavelength, float *hkl_dev, void *stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return fail(SPSIM_ERR_INVALID_ARG, "detector has %d x %d x %d pixels", nx, ny, nz);
  if (!hkl_dev) return fail(SPSIM_ERR_INVALID_ARG, "hkl_dev is NULL");
  CUDA_TRY(launch_volume(nx, ny, nz, width, height, depth, distance, center_x, center_y, center_z, wavelength, hkl_dev,
                         (cudaStream_t)stream));
  return SPSIM_OK;
}

extern "C" int spsim_b200_hkl_for_detector(int nx, int ny, float width, float height, float distance,
                                           float center_x, float center_y, float wavelength, int spherical,
                                           float *hkl_dev, void *stream) {
  int st = check_detector(nx, ny, width, height, distance, wavelength);
  if (st) return st;
  if (!hkl_dev) return fail(SPSIM_ERR_INVALID_ARG, "output is NULL");
  CUDA_TRY(launch_ewald(nx, ny, width, height, distance, center_x, center_y, wavelength, spherical, hkl_dev, nullptr,
                        (cudaStream_t)stream));
  return SPSIM_OK;
}

static int chain_dev(const spsim_b200_chain_params *p, ChainDev *c) {
  if (!p) return fail(SPSIM_ERR_INVALID_ARG, "params is NULL");
  if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0) return fail(SPSIM_ERR_INVALID_ARG, "detector size must be > 0");
  if (p->binning_x <= 0 || p->binning_y <= 0 || p->binning_z <= 0)
    return fail(SPSIM_ERR_INVALID_ARG, "binning must be >= 1");
  memset(c, 0, sizeof(*c));
  c->nx = p->nx;
  c->ny = p->ny;
  c->nz = p->nz;
  c->bx = p->binning_x;
  c->by = p->binning_y;
  c->bz = p->binning_z;
  c->spherical = p->spherical;
  c->polarization = p->polarization;
  c->unbinned = (c->bx == 1 && c->by == 1 && c->bz == 1);
  c->clamp = p->clamp_to_maximum;
  c->width = p->width;
  c->height = p->height;
  c->distance = p->distance;
  c->cx = p->center_x;
  c->cy = p->center_y;
  c->pw = p->pixel_width;
  c->ph = p->pixel_height;
  c->beam_intensity = p->beam_intensity;
  c->qe = p->quantum_efficiency;
  // src/amplification.c:56-61 and :121-123
  const double h_c = 1.98644521e-25;
  const double photon_energy = h_c / (double)p->wavelength;
  c->epp = 1.0f;
  if (p->electron_hole_production_energy) c->epp = (float)(photon_energy / (double)p->electron_hole_production_energy);
  c->epp_noiseless = (float)(photon_energy / (double)p->electron_hole_production_energy);
  c->dark_t = p->dark_current * p->exposure_time;
  c->readout = p->readout_noise;
  c->adc = 1.0f;
  if (p->linear_full_well && p->maximum_value) c->adc = p->maximum_value / p->linear_full_well;
  c->maxv = p->maximum_value;
  c->seed = p->seed;
  c->pattern = p->pattern_index;
  c->i0 = 0;
  c->i1 = (long long)p->nx * p->ny * p->nz;
  c->b0 = 0;
  c->b1 = (long long)(p->nx / p->binning_x) * (p->ny / p->binning_y) * (p->nz / p->binning_z);
  return SPSIM_OK;
}

static DevBuf g_chain_ph, g_chain_el;

extern "C" int spsim_b200_detector_chain(const spsim_b200_chain_params *p, const float *I_dev,
                                         const spsim_b200_chain_outputs *out, void *stream) {
  ChainDev c;
  int st = chain_dev(p, &c);
  if (st) return st;
  if (!out) return fail(SPSIM_ERR_INVALID_ARG, "outputs is NULL");
  const bool needs_I = out->photons_per_pixel || out->photon_count || out->electrons_per_pixel || out->real_output ||
                       out->noiseless_output;
  if (needs_I && !I_dev) return fail(SPSIM_ERR_INVALID_ARG, "intensities are NULL");
  ChainOut o = {out->thomson_correction, out->solid_angle,  out->photons_per_pixel, out->photon_count,
                out->electrons_per_pixel, out->real_output, out->noiseless_output};
  float *sph = nullptr, *sel = nullptr;
  const size_t n = (size_t)p->nx * p->ny * p->nz;
  if (!c.unbinned) {
    std::lock_guard<std::mutex> lk(g_mu);
    CUDA_TRY(g_chain_ph.ensure(n * sizeof(float)));
    CUDA_TRY(g_chain_el.ensure(n * sizeof(float)));
    sph = (float *)g_chain_ph.p;
    sel = (float *)g_chain_el.p;
  }
  CUDA_TRY(launch_chain(c, I_dev, o, sph, sel, (cudaStream_t)stream));
  return SPSIM_OK;
}

// Rows [row0, row1) of a flat detector's fused chain (library-internal, the
// pipelined simulate_shot): the pixels' and bins' values are those of the
// whole-detector call, as every pixel keeps its index (Philox counter) and
// row0 (and row1, unless it is ny) is a multiple of the y binning.
extern "C" int spsim_internal_chain_rows(const spsim_b200_chain_params *p, const float *I_dev,
                                         const spsim_b200_chain_outputs *out, int64_t row0, int64_t row1,
                                         void *stream) {
  ChainDev c;
  int st = chain_dev(p, &c);
  if (st) return st;
  if (!out || !I_dev) return fail(SPSIM_ERR_INVALID_ARG, "outputs or intensities are NULL");
  if (p->nz != 1 || row0 < 0 || row1 > p->ny || row0 > row1 || row0 % p->binning_y ||
      (row1 != p->ny && row1 % p->binning_y))
    return fail(SPSIM_ERR_INVALID_ARG, "chain rows [%lld, %lld) of %d", (long long)row0, (long long)row1, p->ny);
  if (!c.unbinned && (!out->photons_per_pixel || !out->electrons_per_pixel))
    return fail(SPSIM_ERR_INVALID_ARG, "binned chain rows need the photon and electron arrays");
  const long long bnx = p->nx / p->binning_x;
  c.i0 = row0 * p->nx;
  c.i1 = row1 * p->nx;
  c.b0 = row0 / p->binning_y * bnx;
  c.b1 = std::min<long long>(row1 / p->binning_y, p->ny / p->binning_y) * bnx;
  ChainOut o = {out->thomson_correction, out->solid_angle,  out->photons_per_pixel, out->photon_count,
                out->electrons_per_pixel, out->real_output, out->noiseless_output};
  CUDA_TRY(launch_chain(c, I_dev, o, nullptr, nullptr, (cudaStream_t)stream));
  return SPSIM_OK;
}

extern "C" int spsim_b200_thomson(const spsim_b200_chain_params *p, float *out_dev, void *stream) {
  spsim_b200_chain_outputs o;
  memset(&o, 0, sizeof(o));
  o.thomson_correction = out_dev;
  return spsim_b200_detector_chain(p, nullptr, &o, stream);
}

extern "C" int spsim_b200_solid_angle(const spsim_b200_chain_params *p, float *out_dev, void *stream) {
  spsim_b200_chain_outputs o;
  memset(&o, 0, sizeof(o));
  o.solid_angle = out_dev;
  return spsim_b200_detector_chain(p, nullptr, &o, stream);
}

extern "C" int spsim_b200_poisson(int64_t n, const float *lambda_dev, uint64_t seed, uint32_t pattern_index,
                                  float *photon_count_dev, void *stream) {
  if (n < 0 || (n > 0 && (!lambda_dev || !photon_count_dev))) return fail(SPSIM_ERR_INVALID_ARG, "bad arrays");
  CUDA_TRY(launch_poisson(n, lambda_dev, seed, pattern_index, photon_count_dev, (cudaStream_t)stream));
  return SPSIM_OK;
}

extern "C" int spsim_b200_photons(int64_t n, const float *thomson_dev, const float *solid_angle_dev,
                                  const float *I_dev, float beam_intensity, float *photons_dev, void *stream) {
  if (n < 0 || (n > 0 && (!thomson_dev || !solid_angle_dev || !I_dev || !photons_dev)))
    return fail(SPSIM_ERR_INVALID_ARG, "bad arrays");
  CUDA_TRY(launch_photons(n, thomson_dev, solid_angle_dev, I_dev, beam_intensity, photons_dev, (cudaStream_t)stream));
  return SPSIM_OK;
}

extern "C" int spsim_b200_photon_counts(const spsim_b200_chain_params *p, const float *photons_dev,
                                        float *counts_dev, void *stream) {
  ChainDev c;
  int st = chain_dev(p, &c);
  if (st) return st;
  if (!photons_dev || !counts_dev) return fail(SPSIM_ERR_INVALID_ARG, "bad arrays");
  CUDA_TRY(launch_counts(c, photons_dev, counts_dev, (cudaStream_t)stream));
  return SPSIM_OK;
}

extern "C" int spsim_b200_electrons(const spsim_b200_chain_params *p, const float *counts_dev, float *electrons_dev,
                                    void *stream) {
  ChainDev c;
  int st = chain_dev(p, &c);
  if (st) return st;
  if (!counts_dev || !electrons_dev) return fail(SPSIM_ERR_INVALID_ARG, "bad arrays");
  CUDA_TRY(launch_electrons(c, counts_dev, electrons_dev, (cudaStream_t)stream));
  return SPSIM_OK;
}

extern "C" int spsim_b200_binned_outputs(const spsim_b200_chain_params *p, const float *electrons_dev,
                                         const float *photons_dev, float *real_output_dev,
                                         float *noiseless_output_dev, void *stream) {
  ChainDev c;
  int st = chain_dev(p, &c);
  if (st) return st;
  if ((real_output_dev && !electrons_dev) || (noiseless_output_dev && !photons_dev))
    return fail(SPSIM_ERR_INVALID_ARG, "an output needs its input array");
  CUDA_TRY(launch_binned(c, electrons_dev, photons_dev, real_output_dev, noiseless_output_dev, (cudaStream_t)stream));
  return SPSIM_OK;
}

// ---------------------------------------------------------------------------
// adjoint

// Adjoint plans: the form-factor table, the atom blocks and the work items of
// one (molecule, q set, pattern count, B, kernel mode) are built on the first
// call and reused; only the rotations are uploaded again, when they change.
struct AdjPlan {
  unsigned long long mol_id = 0, qs_id = 0;
  int npat = 0, mode = 0, device = 0;
  float B = 0;
  int n_items = 0;
  DevBuf ff, blocks, items, rot;
  std::vector<double> host_rot;  // the rotations as last uploaded
  // recorded after each call's launch: the next call, on whatever stream,
  // waits for it before it rewrites the rotations the last launch reads
  cudaEvent_t done = nullptr;
  ~AdjPlan() {
    if (done) cudaEventDestroy(done);
  }
};
static std::vector<std::unique_ptr<AdjPlan>> g_adj_plans;  // most recent last
static const size_t kMaxAdjPlans = 4;

static void adjoint_release(int dev) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (size_t i = g_adj_plans.size(); i-- > 0;)
    if (g_adj_plans[i]->device == dev) g_adj_plans.erase(g_adj_plans.begin() + i);
}

extern "C" int spsim_b200_adjoint(const spsim_b200_molecule *m, const spsim_b200_qset *qs, int npat,
                                  const double *rot, float B, int precision, const float *F_dev, const float *G_dev,
                                  double *dpos_dev, double *docc_dev, double *dB_dev, void *stream) {
  if (!m || !qs) return fail(SPSIM_ERR_INVALID_ARG, "NULL handle");
  if (npat <= 0) return fail(SPSIM_ERR_INVALID_ARG, "npat must be > 0");
  if (!F_dev || !G_dev || !dpos_dev) return fail(SPSIM_ERR_INVALID_ARG, "F, G and dpos are required");
  if (precision < SPSIM_PREC_FP64 || precision > SPSIM_PREC_F32_FAST)
    return fail(SPSIM_ERR_INVALID_ARG, "unknown precision %d", precision);
  if (dB_dev && !m->per_atom_b) return fail(SPSIM_ERR_INVALID_ARG, "dB needs a molecule with per-atom B factors");
  cudaStream_t st = (cudaStream_t)stream;
  const long long npix = qs->npix;
  const long long total = npix * npat;
  double qmax = qs->qmax;
  if (rot) {
    for (int i = 0; i < npat; ++i)
      if (!is_orthonormal(rot + 9 * (size_t)i)) {
        double fro = 0;
        for (int k = 0; k < 9; ++k) fro += rot[9 * (size_t)i + k] * rot[9 * (size_t)i + k];
        qmax = std::max(qmax, qs->qmax * std::sqrt(fro));
      }
  }
  const int eq = ceil_log2_bound(std::max(qmax, 1e-300));
  const int kq = 22 - m->kr;
  const float dq = (float)std::ldexp(1.0, eq - kq);
  // FP32 adjoints follow the forward's kernel form: the FP64-phase one unless
  // a compensated form is forced with spsim_b200_set_variant
  const bool dphase = precision == SPSIM_PREC_F32 && !(g_force_nt > 0 && g_force_pk < 2);
  if (dphase && qmax * m->rbound >= std::ldexp(1.0, 48))
    return fail(SPSIM_ERR_RANGE, "adjoint: |q|max*|r|max exceeds 2^48 cycles");
  if (precision != SPSIM_PREC_FP64 && !dphase && m->n_kept > 0) {
    const double cmax = 0.8660254037844386 * (qmax * m->dr + (double)dq * (m->rbound + m->dr));
    const double lim = precision == SPSIM_PREC_F32 ? 1.0 / 16 : 0.25;
    if (qmax * m->rbound >= std::ldexp(1.0, 19) || cmax > lim)
      return fail(SPSIM_ERR_RANGE, "adjoint: phase range outside the FP32 kernel's domain; use SPSIM_PREC_FP64");
  }
  CUDA_TRY(cudaMemsetAsync(dpos_dev, 0, 3 * (size_t)m->natoms_in * sizeof(double), st));
  if (docc_dev) CUDA_TRY(cudaMemsetAsync(docc_dev, 0, (size_t)m->natoms_in * sizeof(double), st));
  if (dB_dev) CUDA_TRY(cudaMemsetAsync(dB_dev, 0, (size_t)m->natoms_in * sizeof(double), st));
  if (m->n_kept == 0 || total == 0) return SPSIM_OK;

  // mode 4: the FP64-phase adjoint with the fixed-point phase word (phases within 2^17 cycles)
  const bool fixw = dphase && qmax * m->rbound < std::ldexp(1.0, 17);
  const int mode =
      precision == SPSIM_PREC_FP64 ? 2 : (precision == SPSIM_PREC_F32_FAST ? 1 : (dphase ? (fixw ? 4 : 3) : 0));
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_mu);
  AdjPlan *pl = nullptr;
  for (size_t i = 0; i < g_adj_plans.size(); ++i) {
    AdjPlan &c = *g_adj_plans[i];
    if (c.mol_id == m->id && c.qs_id == qs->id && c.npat == npat && c.B == B && c.mode == mode &&
        c.device == dev) {
      std::unique_ptr<AdjPlan> keep = std::move(g_adj_plans[i]);
      g_adj_plans.erase(g_adj_plans.begin() + i);
      g_adj_plans.push_back(std::move(keep));
      pl = g_adj_plans.back().get();
      break;
    }
  }
  if (!pl) {
    std::unique_ptr<AdjPlan> np(new AdjPlan());
    np->mol_id = m->id;
    np->qs_id = qs->id;
    np->npat = npat;
    np->B = B;
    np->mode = mode;
    np->device = dev;
    // atom blocks x pixel chunks.  The FP64-phase adjoint's blocks are
    // consecutive runs of the element-sorted atoms that may span two element
    // segments (each thread's atoms stay in one), so short segments do not leave
    // blocks mostly empty; the other adjoints take one element per block.
    const int block_atoms =
        precision == SPSIM_PREC_FP64 ? ADJ_THREADS : (dphase ? ADJ_DPHASE_BLOCK_ATOMS : ADJ_BLOCK_ATOMS);
    std::vector<AdjBlock> blocks;
    {
      struct Seg {
        int elem, begin, end;
      };
      std::vector<Seg> segs;
      int e = -1, seg0 = 0;
      for (size_t k = 0; k <= m->tiles.size(); ++k) {
        const bool end = k == m->tiles.size();
        if (end || m->tiles[k].elem != e) {
          if (e >= 0) segs.push_back({e, seg0, m->tiles[k - 1].atom_begin + m->tiles[k - 1].count});
          if (!end) {
            e = m->tiles[k].elem;
            seg0 = m->tiles[k].atom_begin;
          }
        }
      }
      if (dphase) {
        size_t s0 = 0;
        int a = segs.empty() ? 0 : segs[0].begin;
        while (s0 < segs.size()) {
          AdjBlock b = {a, std::min(a + block_atoms, segs[s0].end), segs[s0].elem, -1, 0, 0};
          b.split = b.atom_end;
          if (b.atom_end == segs[s0].end && b.atom_end - a < block_atoms && s0 + 1 < segs.size()) {
            // fill the rest of the block from the next segment (segments are contiguous)
            b.elem2 = segs[s0 + 1].elem;
            b.split = segs[s0 + 1].begin;
            b.atom_end = std::min(a + block_atoms, segs[s0 + 1].end);
          }
          blocks.push_back(b);
          a = b.atom_end;
          while (s0 < segs.size() && a >= segs[s0].end) ++s0;
        }
      } else {
        for (const Seg &sg : segs)
          for (int a = sg.begin; a < sg.end; a += block_atoms)
            blocks.push_back({a, std::min(a + block_atoms, sg.end), sg.elem, -1, std::min(a + block_atoms, sg.end), 0});
      }
    }
    // pixel chunks per block so that the equal-cost CTAs fill at most four whole
    // waves of the resident slots (a last wave of a few CTAs would leave the GPU
    // idle for one item's length: 1,190 CTAs on 592 slots ran as three waves)
    const long long slots = (long long)num_sms() * std::max(1, adjoint_occupancy(mode, m->per_atom_b != 0));
    long long nchunk = std::max<long long>(1, 4 * slots / (long long)blocks.size());
    long long chunk = (total + nchunk - 1) / nchunk;
    chunk = (chunk + 255) / 256 * 256;
    std::vector<AdjItem> items;
    for (size_t b = 0; b < blocks.size(); ++b)
      for (long long p0 = 0; p0 < total; p0 += chunk) items.push_back({(int)b, 0, p0, std::min(total, p0 + chunk)});
    np->n_items = (int)items.size();
    CUDA_TRY(np->ff.ensure(std::max<size_t>((size_t)m->n_elem * npix, 1) * sizeof(double)));
    CUDA_TRY(np->blocks.ensure(blocks.size() * sizeof(AdjBlock)));
    CUDA_TRY(np->items.ensure(items.size() * sizeof(AdjItem)));
    CUDA_TRY(np->rot.ensure(9 * (size_t)npat * sizeof(double)));
    CUDA_TRY(cudaMemcpyAsync(np->blocks.p, blocks.data(), blocks.size() * sizeof(AdjBlock), cudaMemcpyHostToDevice,
                             st));
    CUDA_TRY(cudaMemcpyAsync(np->items.p, items.data(), items.size() * sizeof(AdjItem), cudaMemcpyHostToDevice, st));
    CUDA_TRY(launch_ff_table(qs->d_hkl, qs->d_q64, npix, m->n_elem, m->d_coeffs, (double)B, m->delta_atoms,
                             (double *)np->ff.p, st));
    CUDA_TRY(cudaEventCreateWithFlags(&np->done, cudaEventDisableTiming));
    CUDA_TRY(cudaEventRecord(np->done, st));
    if (g_adj_plans.size() >= kMaxAdjPlans) {
      cudaDeviceSynchronize();  // the evicted plan's buffers may still be in use
      g_adj_plans.erase(g_adj_plans.begin());
    }
    g_adj_plans.push_back(std::move(np));
    pl = g_adj_plans.back().get();
  }
  CUDA_TRY(cudaStreamWaitEvent(st, pl->done, 0));
  // this call's rotations, uploaded when they differ from the last call's
  if (rot && (pl->host_rot.size() != 9 * (size_t)npat ||
              memcmp(pl->host_rot.data(), rot, 9 * (size_t)npat * sizeof(double)) != 0)) {
    pl->host_rot.assign(rot, rot + 9 * (size_t)npat);
    CUDA_TRY(cudaMemcpyAsync(pl->rot.p, pl->host_rot.data(), 9 * (size_t)npat * sizeof(double),
                             cudaMemcpyHostToDevice, st));
  }
  AdjParams prm;
  memset(&prm, 0, sizeof(prm));
  prm.atoms = m->d_atoms;
  prm.atomsd = m->d_atomsd;
  prm.perm = m->d_perm;
  prm.wbase = m->d_wbase;
  prm.blocks = (const AdjBlock *)pl->blocks.p;
  prm.items = (const AdjItem *)pl->items.p;
  prm.hkl = qs->d_hkl;
  prm.q64 = qs->d_q64;
  prm.rot = rot ? (const double *)pl->rot.p : nullptr;
  prm.ff = (const double *)pl->ff.p;
  prm.F = (const float2 *)F_dev;
  prm.G = G_dev;
  prm.npix = npix;
  prm.cx = m->center[0];
  prm.cy = m->center[1];
  prm.cz = m->center[2];
  prm.dq = dq;
  prm.inv_dq = (float)std::ldexp(1.0, kq - eq);
  prm.per_atom_b = m->per_atom_b;
  prm.dpos = dpos_dev;
  prm.docc = docc_dev;
  prm.dB = dB_dev;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (g_timing) {
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    CUDA_TRY(cudaEventRecord(e0, st));
  }
  CUDA_TRY(launch_adjoint(mode, prm, pl->n_items, st));
  CUDA_TRY(cudaEventRecord(pl->done, st));
  if (g_timing) {
    CUDA_TRY(cudaEventRecord(e1, st));
    g_timing_events.push_back({e0, e1});
  }
  return SPSIM_OK;
}
