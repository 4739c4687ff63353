/*
 * Reference-shaped entry points (include/spsim.h) on top of the native ABI.
 * Each function keeps the reference's signature, allocation and ownership
 * rules; the arithmetic runs on the GPU.  Failures print the reason and
 * abort(), as the reference's sp_error_fatal paths do: there is no CPU fallback.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <time.h>
#include <unistd.h>

#include <cuda_runtime.h>

#include "../../../include/spsim.h"
#include "../../../include/spsim_b200.h"

static int g_precision = SPSIM_PREC_F32;
static double g_nufft_eps = 1e-8;
static unsigned long long g_seed = 0x5eed5eedULL;
static uint32_t g_pattern_counter = 0;

void spsim_b200_set_legacy_precision(int precision) { g_precision = precision; }
int spsim_b200_get_legacy_precision(void) { return g_precision; }
void spsim_b200_set_legacy_nufft_eps(double eps) { g_nufft_eps = eps; }
double spsim_b200_get_legacy_nufft_eps(void) { return g_nufft_eps; }
void spsim_b200_set_noise_seed(unsigned long long seed) { g_seed = seed; }

static void die(const char *where, int st) {
  fprintf(stderr, "spsim_b200: %s failed: %s (%s)\n", where, spsim_b200_status_string(st), spsim_b200_last_error());
  abort();
}

static void cuda_die(const char *where, cudaError_t e) {
  fprintf(stderr, "spsim_b200: %s failed: %s\n", where, cudaGetErrorString(e));
  abort();
}

/* Output arrays the caller frees with free(), as the reference's are.  Large
 * ones are 2 MiB aligned and advised for transparent huge pages, so that
 * filling them (device-to-host copies) takes a few page faults instead of
 * one per 4 KiB page; free() releases them like any malloc'd block. */
static void *host_alloc(size_t bytes) {
  if (!bytes) bytes = 4;
  void *p = NULL;
  if (bytes >= ((size_t)2 << 20)) {
    const size_t huge = (size_t)2 << 20;
    if (posix_memalign(&p, huge, (bytes + huge - 1) / huge * huge) == 0) {
      madvise(p, (bytes + huge - 1) / huge * huge, MADV_HUGEPAGE);
      return p;
    }
    p = NULL;
  }
  p = malloc(bytes);
  if (!p) {
    fprintf(stderr, "spsim_b200: out of host memory (%zu bytes)\n", bytes);
    abort();
  }
  return p;
}

/* Device scratch of the reference-shaped calls: one grow-only buffer per
 * slot, kept between calls (no cudaMalloc / cudaFree per call) and released by
 * spsim_b200_release_scratch.  Each call site owns its slots, so nested calls
 * (calculate_photons_per_pixel computing the Thomson factor first) never share
 * one.  Like the reference's own static state, this makes the calls
 * non-reentrant. */
enum {
  SLOT_HKL,
  SLOT_THOMSON,
  SLOT_SOLID,
  SLOT_PH_T, SLOT_PH_O, SLOT_PH_I, SLOT_PH_P,
  SLOT_PO_P, SLOT_PO_C,
  SLOT_EL_C, SLOT_EL_E,
  SLOT_RO_E, SLOT_RO_R,
  SLOT_NL_P, SLOT_NL_N,
  SLOT_SHOT_I, SLOT_SHOT_F, SLOT_SHOT_0,
  N_SLOTS = SLOT_SHOT_0 + 7
};
static void *g_slot[N_SLOTS];
static size_t g_slot_bytes[N_SLOTS];
static int g_slot_device[N_SLOTS];

static void *dev_alloc(int slot, size_t bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (!bytes) bytes = 4;
  if (g_slot[slot] && g_slot_bytes[slot] >= bytes && g_slot_device[slot] == dev) return g_slot[slot];
  if (g_slot[slot] && g_slot_device[slot] == dev) cudaFree(g_slot[slot]);
  g_slot[slot] = NULL; /* a buffer left on another device is dropped, not freed */
  g_slot_bytes[slot] = 0;
  cudaError_t e = cudaMalloc(&g_slot[slot], bytes);
  if (e != cudaSuccess) cuda_die("cudaMalloc", e);
  g_slot_bytes[slot] = bytes;
  g_slot_device[slot] = dev;
  return g_slot[slot];
}

void spsim_internal_release_host_session(void);
/* library-internal (capi.cu): the simulate_shot structure factor on a device
 * HKL list, its error check, and the float rotation of a device HKL list */
int spsim_internal_shot_structure_factor(int natoms, const int32_t *Z, const float *pos, float B, int delta_atoms,
                                         const float *beam, float wavelength, float bandwidth, int samples,
                                         int64_t npix, const float *hkl_dev, int precision, float *F_dev,
                                         float *I_dev);
int spsim_internal_shot_structure_factor_nufft(int natoms, const int32_t *Z, const float *pos, float B,
                                               int delta_atoms, int64_t npix, const float *hkl_dev, int row,
                                               double eps, float *F_dev, float *I_dev);
int spsim_internal_shot_check(void);
int spsim_internal_shot_molecule(int natoms, const int32_t *Z, const float *pos, int delta_atoms, const float *beam);
int spsim_internal_shot_parts_begin(int64_t npix, const float *hkl_dev);
int spsim_internal_shot_nufft_begin(int natoms, const int32_t *Z, const float *pos, float B, int delta_atoms,
                                    int64_t npix, const float *hkl_dev, int row, double eps);
int spsim_internal_shot_nufft_part(int64_t p0, int64_t p1, float *F_dev, float *I_dev);
int spsim_internal_shot_part(int64_t p0, int64_t p1, float B, int precision, float *F_dev, float *I_dev,
                             void *stream);
int spsim_internal_chain_rows(const spsim_b200_chain_params *p, const float *I_dev,
                              const spsim_b200_chain_outputs *out, int64_t row0, int64_t row1, void *stream);
int spsim_internal_rotate_hkl(int64_t npix, const float R[9], float *hkl_dev);

/* Pinned staging buffer of simulate_shot's device-to-host copies (grow-only,
 * released by spsim_b200_release_scratch). */
static void *g_pinned = NULL;
static size_t g_pinned_bytes = 0;
static cudaStream_t g_copy_stream = NULL; /* non-blocking side stream of simulate_shot */
static int g_copy_stream_device = -1;
/* the pipelined simulate_shot's two compute streams (row chunks alternate) */
static cudaStream_t g_comp_stream[2] = {NULL, NULL};
static int g_comp_stream_device = -1;
static int g_shot_chunks = 0; /* row chunks of simulate_shot: 0 automatic, 1 none */

enum { MAX_SHOT_CHUNKS = 8 }; /* row chunks of simulate_shot, at most */
void spsim_b200_set_shot_chunks(int chunks) { g_shot_chunks = chunks < 0 ? 0 : chunks > MAX_SHOT_CHUNKS ? MAX_SHOT_CHUNKS : chunks; }
int spsim_b200_get_shot_chunks(void) { return g_shot_chunks; }

static void *pinned_alloc(size_t bytes) {
  if (g_pinned && g_pinned_bytes >= bytes) return g_pinned;
  if (g_pinned) cudaFreeHost(g_pinned);
  g_pinned = NULL;
  g_pinned_bytes = 0;
  cudaError_t e = cudaHostAlloc(&g_pinned, bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) cuda_die("cudaHostAlloc", e);
  g_pinned_bytes = bytes;
  return g_pinned;
}

void spsim_b200_release_scratch(void) {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceSynchronize();
  for (int k = 0; k < N_SLOTS; k++) {
    if (g_slot[k] && g_slot_device[k] == dev) cudaFree(g_slot[k]);
    g_slot[k] = NULL;
    g_slot_bytes[k] = 0;
  }
  if (g_pinned) cudaFreeHost(g_pinned);
  g_pinned = NULL;
  g_pinned_bytes = 0;
  if (g_copy_stream && g_copy_stream_device == dev) cudaStreamDestroy(g_copy_stream);
  g_copy_stream = NULL;
  g_copy_stream_device = -1;
  for (int k = 0; k < 2; k++) {
    if (g_comp_stream[k] && g_comp_stream_device == dev) cudaStreamDestroy(g_comp_stream[k]);
    g_comp_stream[k] = NULL;
  }
  g_comp_stream_device = -1;
  spsim_internal_release_host_session();
}

/* Host copies and first touches of large arrays: a batch of (dst, src, bytes)
 * jobs (src NULL: fill with zeros, the first touch of fresh pages) cut into
 * equal byte ranges over a few threads. */
typedef struct {
  char *dst;
  const char *src;
  size_t bytes;
} HostCopy;

typedef struct {
  const HostCopy *jobs;
  int njobs;
  size_t begin, end; /* byte range of the concatenated jobs */
} HostCopyRange;

static void *host_copy_worker(void *arg) {
  const HostCopyRange *r = (const HostCopyRange *)arg;
  size_t base = 0;
  for (int j = 0; j < r->njobs; j++) {
    const HostCopy *c = &r->jobs[j];
    const size_t lo = r->begin > base ? r->begin - base : 0;
    const size_t hi = r->end - base < c->bytes ? r->end - base : c->bytes;
    if (r->end > base && lo < hi && lo < c->bytes) {
      if (c->src)
        memcpy(c->dst + lo, c->src + lo, hi - lo);
      else
        memset(c->dst + lo, 0, hi - lo);
    }
    base += c->bytes;
    if (base >= r->end) break;
  }
  return NULL;
}

static void host_copy_batch(const HostCopy *jobs, int njobs) {
  enum { MAX_THREADS = 8 };
  size_t total = 0;
  for (int j = 0; j < njobs; j++) total += jobs[j].bytes;
  long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
  int nt = (int)(total >> 21); /* one thread per 2 MiB */
  if (nt > MAX_THREADS) nt = MAX_THREADS;
  if (nt > ncpu) nt = (int)ncpu;
  if (nt < 1) nt = 1;
  pthread_t th[MAX_THREADS];
  HostCopyRange rg[MAX_THREADS];
  int started[MAX_THREADS] = {0};
  const size_t chunk = (total / nt + 4095) & ~(size_t)4095;
  for (int t = 0; t < nt; t++) {
    rg[t].jobs = jobs;
    rg[t].njobs = njobs;
    rg[t].begin = (size_t)t * chunk < total ? (size_t)t * chunk : total;
    rg[t].end = (size_t)(t + 1) * chunk < total ? (size_t)(t + 1) * chunk : total;
    if (t == nt - 1) rg[t].end = total;
    started[t] = t > 0 && pthread_create(&th[t], NULL, host_copy_worker, &rg[t]) == 0;
  }
  host_copy_worker(&rg[0]);
  for (int t = 1; t < nt; t++) {
    if (started[t])
      pthread_join(th[t], NULL);
    else
      host_copy_worker(&rg[t]);
  }
}

static void h2d(void *d, const void *h, size_t bytes) {
  cudaError_t e = cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) cuda_die("cudaMemcpy H2D", e);
}

static void d2h(void *h, const void *d, size_t bytes) {
  cudaError_t e = cudaMemcpy(h, d, bytes, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) cuda_die("cudaMemcpy D2H", e);
}

static double now_us(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec * 1e6 + t.tv_nsec * 1e-3;
}

/* ------------------------------------------------------------ geometry */

/* src/diffraction.c:237-297, computed on the GPU in FP64, stored as float */
float *get_HKL_list_for_detector(CCD *det, Experiment *exp, int *HKL_list_size) {
  const long long n = (long long)det->nx * det->ny;
  float *out = (float *)host_alloc(sizeof(float) * 3 * (n > 0 ? n : 1));
  float *d = (float *)dev_alloc(SLOT_HKL, sizeof(float) * 3 * n);
  int st = spsim_b200_hkl_for_detector(det->nx, det->ny, det->width, det->height, det->distance, det->center_x,
                                       det->center_y, exp->wavelength, det->spherical, d, NULL);
  if (st) die("get_HKL_list_for_detector", st);
  d2h(out, d, sizeof(float) * 3 * n);
  *HKL_list_size = (int)n;
  return out;
}

/* src/diffraction.c:325-369, on the GPU in FP64, stored as float */
float *get_HKL_list_for_3d_detector(CCD *det, Experiment *exp, int *HKL_list_size) {
  const long long n = (long long)det->nx * det->ny * det->nz;
  float *out = (float *)host_alloc(sizeof(float) * 3 * (n > 0 ? n : 1));
  float *d = (float *)dev_alloc(SLOT_HKL, sizeof(float) * 3 * n);
  int st = spsim_b200_hkl_for_3d_detector(det->nx, det->ny, det->nz, det->width, det->height, det->depth,
                                          det->distance, det->center_x, det->center_y, det->center_z, exp->wavelength,
                                          d, NULL);
  if (st) die("get_HKL_list_for_3d_detector", st);
  d2h(out, d, sizeof(float) * 3 * n);
  *HKL_list_size = (int)n;
  return out;
}

/* src/spsim.c:98-108 */
float *get_HKL_list(Options *opts, int *HKL_list_size) {
  if (opts->detector->nz > 1) return get_HKL_list_for_3d_detector(opts->detector, opts->experiment, HKL_list_size);
  return get_HKL_list_for_detector(opts->detector, opts->experiment, HKL_list_size);
}

/* Rotation R = Rz(a1) Ry(a2) Rz(a3) (intrinsic z-y-z Euler angles) or a
 * Haar-uniform rotation from Shoemake's quaternion construction, drawn from
 * a splitmix64 stream keyed by the noise seed and a call counter. */
static uint64_t g_rot_state = 0;
static uint64_t splitmix64(void) {
  uint64_t z = (g_rot_state += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static double u01(void) { return ((splitmix64() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

static void rotation_matrix(Options *opts, double m[9]) {
  if (opts->random_orientation) {
    if (!g_rot_state) g_rot_state = g_seed ^ 0xA5A5A5A5DEADBEEFULL;
    double u1 = u01(), u2 = u01(), u3 = u01();
    double a = sqrt(1 - u1), b = sqrt(u1);
    double w = a * sin(2 * M_PI * u2), x = a * cos(2 * M_PI * u2);
    double y = b * sin(2 * M_PI * u3), z = b * cos(2 * M_PI * u3);
    double r[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                   2 * (x * y + z * w),     1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                   2 * (x * z - y * w),     2 * (y * z + x * w), 1 - 2 * (x * x + y * y)};
    memcpy(m, r, sizeof(r));
  } else {
    double a1 = opts->euler_orientation[0], a2 = opts->euler_orientation[1], a3 = opts->euler_orientation[2];
    double c1 = cos(a1), s1 = sin(a1), c2 = cos(a2), s2 = sin(a2), c3 = cos(a3), s3 = sin(a3);
    double r[9] = {c1 * c2 * c3 - s1 * s3, -c1 * c2 * s3 - s1 * c3, c1 * s2,
                   s1 * c2 * c3 + c1 * s3, -s1 * c2 * s3 + c1 * c3, s1 * s2,
                   -s2 * c3,               s2 * s3,                 c2};
    memcpy(m, r, sizeof(r));
  }
}

/* src/diffraction.c:300-323: q <- R q in float, like sp_matrix_vector_prod.
 * The returned rotation owns its data in the same allocation, so free() on it
 * (src/spsim.c:357-359) releases everything. */
static SpRotation *new_rotation(Options *opts) {
  double m[9];
  rotation_matrix(opts, m);
  SpRotation *rot = (SpRotation *)malloc(sizeof(SpRotation) + 9 * sizeof(float));
  rot->rows = 3;
  rot->cols = 3;
  rot->data = (float *)(rot + 1);
  for (int k = 0; k < 9; k++) rot->data[k] = (float)m[k];
  return rot;
}

SpRotation *apply_orientation_to_HKL_list(float **HKL_list, int *HKL_list_size, Options *opts) {
  SpRotation *rot = new_rotation(opts);
  float *q = *HKL_list;
  for (long long i = 0; i < *HKL_list_size; i++) {
    float v[3] = {q[3 * i], q[3 * i + 1], q[3 * i + 2]};
    for (int r = 0; r < 3; r++) {
      float acc = 0;
      for (int c = 0; c < 3; c++) acc += rot->data[3 * r + c] * v[c];
      q[3 * i + r] = acc;
    }
  }
  return rot;
}

/* ------------------------------------------------------------ structure factor */

/* spectrum != 0: the semantics of spsim's default CUDA path
 * (cuda_compute_pattern_on_list2, src/diffraction.cu:235-339): an even
 * wavelength_samples above one is raised by one in opts (as the reference
 * does), and a non-zero bandwidth samples the spectrum. */
static Diffraction_Pattern *pattern_on_list(Molecule *mol, float *HKL_list, int n, float B, Experiment *exp,
                                            Options *opts, int spectrum) {
  double t0 = now_us();
  Diffraction_Pattern *res = (Diffraction_Pattern *)calloc(1, sizeof(Diffraction_Pattern));
  res->F = (Complex *)host_alloc(sizeof(Complex) * (n > 0 ? n : 1));
  res->ints = (float *)host_alloc(sizeof(float) * (n > 0 ? n : 1));
  res->HKL_list = (float *)host_alloc(sizeof(float) * 3 * (n > 0 ? n : 1));
  if (n > 0) memcpy(res->HKL_list, HKL_list, sizeof(float) * 3 * n);
  res->HKL_list_size = n;
  res->N_pix = n;
  float beam[3] = {exp ? exp->beam_fwhm : 0.0f, exp ? exp->beam_center_x : 0.0f, exp ? exp->beam_center_y : 0.0f};
  int samples = 1;
  if (spectrum && opts) {
    if (opts->wavelength_samples > 1 && (opts->wavelength_samples & 1) == 0) opts->wavelength_samples++;
    samples = opts->wavelength_samples;
  }
  int st;
  if (spectrum && exp && exp->bandwidth != 0.0f && samples != 1) {
    if (samples < 1) {
      fprintf(stderr, "spsim_b200: wavelength_samples must be >= 1 with a bandwidth (got %d)\n", samples);
      abort();
    }
    st = spsim_b200_structure_factor_host_spectrum(mol->natoms, mol->atomic_number, mol->pos, NULL, NULL, B,
                                                   opts->delta_atoms, beam, exp->wavelength, exp->bandwidth, samples,
                                                   n, HKL_list, g_precision, (float *)res->F, res->ints);
  } else {
    st = spsim_b200_structure_factor_host(mol->natoms, mol->atomic_number, mol->pos, NULL, NULL, B,
                                          opts ? opts->delta_atoms : 0, beam, n, HKL_list, g_precision,
                                          (float *)res->F, res->ints);
  }
  if (st) die("compute_pattern_on_list", st);
  if (opts && opts->verbosity_level > 0) /* src/diffraction.c:849-851 */
    printf("%g atoms.pixel/s\n", 1.0e6 * n * mol->natoms / (now_us() - t0));
  return res;
}

/* src/diffraction.c:770 */
Diffraction_Pattern *compute_pattern_on_list(Molecule *mol, float *HKL_list, int HKL_list_size, float B,
                                             Experiment *exp, Options *opts) {
  return pattern_on_list(mol, HKL_list, HKL_list_size, B, exp, opts, 0);
}

/* src/diffraction.c:856 (the SSE path): same GPU evaluation */
Diffraction_Pattern *vector_compute_pattern_on_list(Molecule *mol, float *HKL_list, int HKL_list_size, float B,
                                                    Experiment *exp, Options *opts) {
  return pattern_on_list(mol, HKL_list, HKL_list_size, B, exp, opts, 0);
}

/* src/diffraction.cu:135 */
Diffraction_Pattern *cuda_compute_pattern_on_list(Molecule *mol, float *HKL_list, int HKL_list_size, float B,
                                                  Experiment *exp, Options *opts) {
  return pattern_on_list(mol, HKL_list, HKL_list_size, B, exp, opts, 0);
}

/* src/diffraction.cu:235: the default CUDA path, including the spectrum */
Diffraction_Pattern *cuda_compute_pattern_on_list2(Molecule *mol, float *HKL_list, int HKL_list_size, float B,
                                                   Experiment *exp, Options *opts) {
  return pattern_on_list(mol, HKL_list, HKL_list_size, B, exp, opts, 1);
}

/* src/diffraction.c:528-675: the NNFFT structure factor on a q list, with
 * unit atom weights (no illumination), the form factor of |q| with the B
 * factor and delta_atoms as the direct sum.  Here a type-3 NUFFT on the GPU
 * (spsim_b200_forward_nufft) at relative error g_nufft_eps; the reference ran
 * the NFFT library with a cut-off of m = 2.  The detector is not used (as in
 * the reference); HKL_list is copied into the result, which the reference
 * leaves uninitialised. */
Diffraction_Pattern *compute_pattern_on_list_by_nfft(Molecule *mol, float *HKL_list, int HKL_list_size, CCD *det,
                                                     float B, Options *opts) {
  (void)det;
  double t0 = now_us();
  const int n = HKL_list_size;
  Diffraction_Pattern *res = (Diffraction_Pattern *)calloc(1, sizeof(Diffraction_Pattern));
  res->F = (Complex *)host_alloc(sizeof(Complex) * (n > 0 ? n : 1));
  res->ints = (float *)host_alloc(sizeof(float) * (n > 0 ? n : 1));
  res->HKL_list = (float *)host_alloc(sizeof(float) * 3 * (n > 0 ? n : 1));
  if (n > 0) memcpy(res->HKL_list, HKL_list, sizeof(float) * 3 * n);
  res->HKL_list_size = n;
  res->N_pix = n;
  int st = spsim_b200_structure_factor_host_nufft(mol->natoms, mol->atomic_number, mol->pos, B,
                                                  opts ? opts->delta_atoms : 0, n, HKL_list, g_nufft_eps,
                                                  (float *)res->F, res->ints);
  if (st) die("compute_pattern_on_list_by_nfft", st);
  if (opts && opts->verbosity_level > 0)
    printf("%g atoms.pixel/s\n", 1.0e6 * n * mol->natoms / (now_us() - t0));
  return res;
}

/* src/spsim.c:110-144: use_nfft_for_sf takes the NUFFT structure factor
 * (compute_pattern_on_list_by_nfft, as the reference's dispatch); the FFT of
 * a gridded electron density (use_fft_for_sf) is another algorithm, not
 * provided.  Every direct-summation path runs on the GPU.  The dispatch
 * follows the reference's: use_cuda == 2 is the first CUDA path, any other
 * non-zero use_cuda the second (with the spectrum), use_cuda == 0 the CPU
 * paths (monochromatic). */
Diffraction_Pattern *compute_sf(Molecule *mol, float *HKL_list, int HKL_list_size, Options *opts) {
  if (opts->use_fft_for_sf) {
    fprintf(stderr, "spsim_b200: the FFT structure factor (use_fft_for_sf) is not supported\n");
    abort();
  }
  if (opts->use_nfft_for_sf) {
    Diffraction_Pattern *p =
        compute_pattern_on_list_by_nfft(mol, HKL_list, HKL_list_size, opts->detector, opts->b_factor, opts);
    p->rot = NULL;
    return p;
  }
  const int spectrum = opts->use_cuda != 0 && opts->use_cuda != 2;
  Diffraction_Pattern *p =
      pattern_on_list(mol, HKL_list, HKL_list_size, opts->b_factor, opts->experiment, opts, spectrum);
  p->rot = NULL;
  return p;
}

/* ------------------------------------------------------------ detector chain */

static spsim_b200_chain_params chain_params(const CCD *det, const Experiment *exp) {
  spsim_b200_chain_params p;
  memset(&p, 0, sizeof(p));
  p.nx = det->nx;
  p.ny = det->ny;
  p.nz = det->nz > 0 ? det->nz : 1;
  p.binning_x = det->binning_x;
  p.binning_y = det->binning_y;
  p.binning_z = det->binning_z;
  p.spherical = det->spherical;
  p.polarization = exp ? exp->polarization : 0;
  p.width = det->width;
  p.height = det->height;
  p.distance = det->distance;
  p.center_x = det->center_x;
  p.center_y = det->center_y;
  p.pixel_width = det->pixel_width;
  p.pixel_height = det->pixel_height;
  p.wavelength = exp ? exp->wavelength : 0.0f;
  p.beam_intensity = exp ? exp->beam_intensity : 0.0f;
  p.quantum_efficiency = det->quantum_efficiency;
  p.electron_hole_production_energy = det->electron_hole_production_energy;
  p.dark_current = det->dark_current;
  p.exposure_time = exp ? exp->exposure_time : 0.0f;
  p.readout_noise = det->readout_noise;
  p.linear_full_well = det->linear_full_well;
  p.maximum_value = det->maximum_value;
  p.clamp_to_maximum = 0;
  p.seed = g_seed;
  p.pattern_index = g_pattern_counter;
  return p;
}

static long long npix_of(const CCD *det) { return (long long)det->nx * det->ny * (det->nz > 0 ? det->nz : 1); }
static long long nbin_of(const CCD *det) {
  return (long long)(det->nx / det->binning_x) * (det->ny / det->binning_y) *
         ((det->nz > 0 ? det->nz : 1) / det->binning_z);
}

/* src/diffraction.c:1109 */
void calculate_thomson_correction(CCD *det, Experiment *exp) {
  const long long n = npix_of(det);
  spsim_b200_chain_params p = chain_params(det, exp);
  float *d = (float *)dev_alloc(SLOT_THOMSON, sizeof(float) * n);
  int st = spsim_b200_thomson(&p, d, NULL);
  if (st) die("calculate_thomson_correction", st);
  det->thomson_correction = (float *)host_alloc(sizeof(float) * (n > 0 ? n : 1));
  d2h(det->thomson_correction, d, sizeof(float) * n);
}

/* src/diffraction.c:1146 */
void calculate_pixel_solid_angle(CCD *det) {
  const long long n = npix_of(det);
  spsim_b200_chain_params p = chain_params(det, NULL);
  float *d = (float *)dev_alloc(SLOT_SOLID, sizeof(float) * n);
  int st = spsim_b200_solid_angle(&p, d, NULL);
  if (st) die("calculate_pixel_solid_angle", st);
  det->solid_angle = (float *)host_alloc(sizeof(float) * (n > 0 ? n : 1));
  d2h(det->solid_angle, d, sizeof(float) * n);
}

/* src/diffraction.c:1190 */
void calculate_photons_per_pixel(Diffraction_Pattern *pattern, Options *opts) {
  CCD *det = opts->detector;
  Experiment *exp = opts->experiment;
  if (!det->thomson_correction) calculate_thomson_correction(det, exp);
  if (!det->solid_angle) calculate_pixel_solid_angle(det);
  const long long n = npix_of(det);
  float *dT = (float *)dev_alloc(SLOT_PH_T, sizeof(float) * n), *dO = (float *)dev_alloc(SLOT_PH_O, sizeof(float) * n);
  float *dI = (float *)dev_alloc(SLOT_PH_I, sizeof(float) * n), *dP = (float *)dev_alloc(SLOT_PH_P, sizeof(float) * n);
  h2d(dT, det->thomson_correction, sizeof(float) * n);
  h2d(dO, det->solid_angle, sizeof(float) * n);
  h2d(dI, pattern->ints, sizeof(float) * n);
  int st = spsim_b200_photons(n, dT, dO, dI, exp->beam_intensity, dP, NULL);
  if (st) die("calculate_photons_per_pixel", st);
  det->photons_per_pixel = (float *)host_alloc(sizeof(float) * (n > 0 ? n : 1));
  d2h(det->photons_per_pixel, dP, sizeof(float) * n);
}

/* src/noise.c:32 */
void generate_poisson_noise(CCD *det) {
  if (!det->photons_per_pixel) {
    fprintf(stderr, "Please calculate photons per pixel first\n");
    return;
  }
  const long long n = npix_of(det);
  spsim_b200_chain_params p = chain_params(det, NULL);
  float *dP = (float *)dev_alloc(SLOT_PO_P, sizeof(float) * n), *dC = (float *)dev_alloc(SLOT_PO_C, sizeof(float) * n);
  h2d(dP, det->photons_per_pixel, sizeof(float) * n);
  int st = spsim_b200_photon_counts(&p, dP, dC, NULL);
  if (st) die("generate_poisson_noise", st);
  det->photon_count = (float *)host_alloc(sizeof(float) * (n > 0 ? n : 1));
  d2h(det->photon_count, dC, sizeof(float) * n);
}

/* src/amplification.c:54 */
void calculate_electrons_per_pixel(CCD *det, Experiment *experiment) {
  if (!det->photon_count) {
    fprintf(stderr, "Calculate photon_count first\n");
    return;
  }
  const long long n = npix_of(det);
  spsim_b200_chain_params p = chain_params(det, experiment);
  float *dC = (float *)dev_alloc(SLOT_EL_C, sizeof(float) * n), *dE = (float *)dev_alloc(SLOT_EL_E, sizeof(float) * n);
  h2d(dC, det->photon_count, sizeof(float) * n);
  int st = spsim_b200_electrons(&p, dC, dE, NULL);
  if (st) die("calculate_electrons_per_pixel", st);
  det->electrons_per_pixel = (float *)host_alloc(sizeof(float) * (n > 0 ? n : 1));
  d2h(det->electrons_per_pixel, dE, sizeof(float) * n);
}

/* src/amplification.c:77 */
void calculate_real_detector_output(CCD *det, Experiment *experiment) {
  if (!det->electrons_per_pixel) {
    fprintf(stderr, "Calculate electrons_per_pixel first\n");
    return;
  }
  const long long n = npix_of(det), nb = nbin_of(det);
  spsim_b200_chain_params p = chain_params(det, experiment);
  float *dE = (float *)dev_alloc(SLOT_RO_E, sizeof(float) * n), *dR = (float *)dev_alloc(SLOT_RO_R, sizeof(float) * nb);
  h2d(dE, det->electrons_per_pixel, sizeof(float) * n);
  int st = spsim_b200_binned_outputs(&p, dE, NULL, dR, NULL, NULL);
  if (st) die("calculate_real_detector_output", st);
  det->real_output = (float *)host_alloc(sizeof(float) * (nb > 0 ? nb : 1));
  d2h(det->real_output, dR, sizeof(float) * nb);
}

/* src/amplification.c:119 */
void calculate_noiseless_detector_output(CCD *det, Experiment *experiment) {
  if (!det->photons_per_pixel) {
    fprintf(stderr, "Calculate photons_per_pixel first\n");
    return;
  }
  const long long n = npix_of(det), nb = nbin_of(det);
  spsim_b200_chain_params p = chain_params(det, experiment);
  float *dP = (float *)dev_alloc(SLOT_NL_P, sizeof(float) * n), *dN = (float *)dev_alloc(SLOT_NL_N, sizeof(float) * nb);
  h2d(dP, det->photons_per_pixel, sizeof(float) * n);
  int st = spsim_b200_binned_outputs(&p, NULL, dP, NULL, dN, NULL);
  if (st) die("calculate_noiseless_detector_output", st);
  det->noiseless_output = (float *)host_alloc(sizeof(float) * (nb > 0 ? nb : 1));
  d2h(det->noiseless_output, dN, sizeof(float) * nb);
}

/* ------------------------------------------------------------ orchestration */

/* simulate_shot's HKL list to the pinned staging buffer on the copy stream,
 * after the work queued so far on the legacy stream; ev is recorded after it */
static void queue_hkl_copy(cudaEvent_t ev, char *s_hkl, const float *d_hkl, size_t bytes) {
  cudaEventRecord(ev, 0);
  cudaStreamWaitEvent(g_copy_stream, ev, 0);
  if (bytes) {
    cudaError_t e = cudaMemcpyAsync(s_hkl, d_hkl, bytes, cudaMemcpyDeviceToHost, g_copy_stream);
    if (e != cudaSuccess) cuda_die("cudaMemcpyAsync HKL", e);
  }
  cudaEventRecord(ev, g_copy_stream);
}

/* Row chunks of the pipelined simulate_shot for a flat detector's
 * monochromatic structure factor, direct or NUFFT (others: 1), as row
 * boundaries rb[0..K].
 * Automatic: 4 from 2^19 pixels on.  The last chunk, whose copies to the
 * host nothing hides, gets a quarter of the others' rows.  Chunk rows are a
 * multiple of the y binning and give a pixel count that is a multiple of 4
 * (the neighbour-quad kernel's alignment). */
static int shot_row_chunks(const CCD *det, long long n, int nfft, int poly, int vol, long long *rb) {
  rb[0] = 0;
  rb[1] = det->ny;
  if (vol || (poly && !nfft) || n <= 0) return 1;
  int k = g_shot_chunks > 0 ? g_shot_chunks : (n >= (1LL << 19) ? 4 : 1);
  if (k > MAX_SHOT_CHUNKS) k = MAX_SHOT_CHUNKS;
  if (k <= 1) return 1;
  const int q = det->nx % 4 == 0 ? 1 : det->nx % 2 == 0 ? 2 : 4;
  int unit = det->binning_y;
  while (unit % q) unit += det->binning_y; /* lcm(binning_y, q) */
  /* rows: k - 1 chunks of 4 parts and one of 1 part, in units */
  const long long units = (det->ny + unit - 1) / unit, parts = 4LL * (k - 1) + 1;
  long long last = units / parts;
  if (last < 1) last = 1;
  const long long rest = units - last;
  if (rest < k - 1) return 1;
  int chunks = 0;
  for (int c = 0; c < k - 1; c++) {
    const long long hi = rest * (c + 1) / (k - 1) * unit;
    if (hi > rb[chunks]) rb[++chunks] = hi < det->ny ? hi : det->ny;
  }
  if (rb[chunks] < det->ny) rb[++chunks] = det->ny;
  return chunks;
}

/* src/spsim.c:281-346 as one device pipeline with the reference's outputs:
 * the HKL list is computed and rotated on the device (bit-identical to
 * get_HKL_list and apply_orientation_to_HKL_list), the structure factor and
 * the fused detector chain run on it without host round trips, and every
 * output comes back through one pinned staging buffer.  While the structure
 * factor runs, the host allocates and first-touches the output arrays and
 * copies out the HKL list.  Outputs, ownership and values are those of the
 * step-by-step reference sequence. */
Diffraction_Pattern *simulate_shot(Molecule *mol, Options *opts) {
  CCD *det = opts->detector;
  Experiment *exp = opts->experiment;
  if (opts->sf_filename[0]) {
    fprintf(stderr, "spsim_b200: precalculated_sf patterns are not supported\n");
    abort();
  }
  if (det->gaussian_blurring != 0.0f) {
    fprintf(stderr, "spsim_b200: detector_gaussian_blurring is not supported\n");
    abort();
  }
  if (opts->use_fft_for_sf) {
    fprintf(stderr, "spsim_b200: the FFT structure factor (use_fft_for_sf) is not supported\n");
    abort();
  }
  if (opts->random_seed >= 0) spsim_b200_set_noise_seed((unsigned long long)opts->random_seed);
  const double t0 = now_us();
  const float beam[3] = {exp->beam_fwhm, exp->beam_center_x, exp->beam_center_y};
  /* the molecule first: a changed one waits for the device, which is idle now */
  /* the NNFFT path weighs every atom by 1 (no illumination) */
  int st = spsim_internal_shot_molecule(mol->natoms, mol->atomic_number, mol->pos, opts->delta_atoms,
                                        opts->use_nfft_for_sf ? NULL : beam);
  if (st) die("simulate_shot molecule", st);

  /* geometry (src/spsim.c:98-108, src/diffraction.c:300-323) */
  const int vol = det->nz > 1;
  const long long n = vol ? (long long)det->nx * det->ny * det->nz : (long long)det->nx * det->ny;
  float *d_hkl = (float *)dev_alloc(SLOT_HKL, sizeof(float) * 3 * (n > 0 ? n : 1));
  st = vol ? spsim_b200_hkl_for_3d_detector(det->nx, det->ny, det->nz, det->width, det->height, det->depth,
                                                 det->distance, det->center_x, det->center_y, det->center_z,
                                                 exp->wavelength, d_hkl, NULL)
               : spsim_b200_hkl_for_detector(det->nx, det->ny, det->width, det->height, det->distance,
                                             det->center_x, det->center_y, exp->wavelength, det->spherical, d_hkl,
                                             NULL);
  if (st) die("simulate_shot geometry", st);
  SpRotation *rot = new_rotation(opts);
  st = spsim_internal_rotate_hkl(n, rot->data, d_hkl);
  if (st) die("simulate_shot orientation", st);

  /* staging layout: HKL list, F, ints, the five per-pixel and two binned chain arrays */
  const long long np = npix_of(det), nb = nbin_of(det);
  if (np != n) {
    fprintf(stderr, "spsim_b200: simulate_shot: detector of %lld pixels but %lld q vectors\n", np, n);
    abort();
  }
  const size_t b_hkl = sizeof(float) * 3 * (size_t)n, b_F = sizeof(Complex) * (size_t)n, b_I = sizeof(float) * (size_t)n;
  const size_t b_nb = sizeof(float) * (size_t)(nb > 0 ? nb : 0);
  char *stage = (char *)pinned_alloc(b_hkl + b_F + b_I + 5 * b_I + 2 * b_nb + 64);
  char *s_hkl = stage, *s_F = s_hkl + b_hkl, *s_I = s_F + b_F, *s_chain = s_I + b_I;
  cudaEvent_t ev_hkl, ev_out;
  cudaError_t e = cudaEventCreateWithFlags(&ev_hkl, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming);
  if (e != cudaSuccess) cuda_die("cudaEventCreate", e);
  /* the HKL list goes down on a side stream, beside the structure factor;
   * it is queued once the structure factor's q-set statistics have come
   * back, which would otherwise wait behind it on the copy engine */
  int cur_dev = 0;
  cudaGetDevice(&cur_dev);
  if (!g_copy_stream || g_copy_stream_device != cur_dev) { /* a stream left on another device is kept */
    e = cudaStreamCreateWithFlags(&g_copy_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) cuda_die("cudaStreamCreate", e);
    g_copy_stream_device = cur_dev;
  }

  /* structure factor (compute_sf, src/spsim.c:110-144): the CUDA dispatch decides the spectrum */
  const int spectrum = opts->use_cuda != 0 && opts->use_cuda != 2;
  int samples = 1;
  if (spectrum) {
    if (opts->wavelength_samples > 1 && (opts->wavelength_samples & 1) == 0) opts->wavelength_samples++;
    samples = opts->wavelength_samples;
  }
  const int poly = spectrum && exp->bandwidth != 0.0f && samples != 1;
  if (poly && samples < 1) {
    fprintf(stderr, "spsim_b200: wavelength_samples must be >= 1 with a bandwidth (got %d)\n", samples);
    abort();
  }
  float *dF = (float *)dev_alloc(SLOT_SHOT_F, b_F > 0 ? b_F : 8);
  float *dI = (float *)dev_alloc(SLOT_SHOT_I, b_I > 0 ? b_I : 4);
  spsim_b200_chain_params p = chain_params(det, exp);
  float *bufs[7];
  for (int k = 0; k < 5; k++) bufs[k] = (float *)dev_alloc(SLOT_SHOT_0 + k, sizeof(float) * np);
  bufs[5] = (float *)dev_alloc(SLOT_SHOT_0 + 5, sizeof(float) * nb);
  bufs[6] = (float *)dev_alloc(SLOT_SHOT_0 + 6, sizeof(float) * nb);
  spsim_b200_chain_outputs o = {bufs[0], bufs[1], bufs[2], bufs[3], bufs[4], bufs[5], bufs[6]};
  long long rb[MAX_SHOT_CHUNKS + 1];
  const int K = shot_row_chunks(det, n, opts->use_nfft_for_sf, poly, vol, rb);
  const long long bnx = det->nx / det->binning_x;
  cudaEvent_t ev_fi = NULL, ev_copied[MAX_SHOT_CHUNKS];

  if (K == 1) {
    if (opts->use_nfft_for_sf)
      st = spsim_internal_shot_structure_factor_nufft(mol->natoms, mol->atomic_number, mol->pos, opts->b_factor,
                                                      opts->delta_atoms, n, d_hkl, det->nx, g_nufft_eps, dF, dI);
    else
      st = spsim_internal_shot_structure_factor(mol->natoms, mol->atomic_number, mol->pos, opts->b_factor,
                                                opts->delta_atoms, beam, poly ? exp->wavelength : 0.0f,
                                                poly ? exp->bandwidth : 0.0f, poly ? samples : 1, n, d_hkl,
                                                g_precision, dF, dI);
    if (st) die("simulate_shot structure factor", st);
    queue_hkl_copy(ev_hkl, s_hkl, d_hkl, b_hkl);

    /* F and |F|^2 go down ahead of the chain, so the host can copy them out
     * while the chain's arrays are still in flight */
    e = cudaEventCreateWithFlags(&ev_fi, cudaEventDisableTiming);
    if (e != cudaSuccess) cuda_die("cudaEventCreate", e);
    if (n > 0) {
      e = cudaMemcpyAsync(s_F, dF, b_F, cudaMemcpyDeviceToHost, 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(s_I, dI, b_I, cudaMemcpyDeviceToHost, 0);
      if (e != cudaSuccess) cuda_die("cudaMemcpyAsync F, I", e);
    }
    cudaEventRecord(ev_fi, 0);

    /* detector chain on the device intensities (src/spsim.c:300-336) */
    st = spsim_b200_detector_chain(&p, dI, &o, NULL);
    if (st) die("simulate_shot detector chain", st);
    if (n > 0) {
      for (int k = 0; k < 7 && e == cudaSuccess; k++) {
        const size_t b = k < 5 ? b_I : b_nb;
        if (b) e = cudaMemcpyAsync(s_chain + (k < 5 ? k * b_I : 5 * b_I + (k - 5) * b_nb), bufs[k], b,
                                   cudaMemcpyDeviceToHost, 0);
      }
      if (e != cudaSuccess) cuda_die("cudaMemcpyAsync outputs", e);
    }
    cudaEventRecord(ev_out, 0);
  } else {
    /* row chunks: chunk c's structure factor and chain run on one of two
     * compute streams (the NUFFT: its grid prepared once, the chunks'
     * interpolations in order on the legacy stream), its outputs go down on
     * the copy stream and into the caller's arrays while chunk c + 1 computes */
    const int nfft = opts->use_nfft_for_sf != 0;
    if (nfft)
      st = spsim_internal_shot_nufft_begin(mol->natoms, mol->atomic_number, mol->pos, opts->b_factor,
                                           opts->delta_atoms, n, d_hkl, det->nx, g_nufft_eps);
    else
      st = spsim_internal_shot_parts_begin(n, d_hkl);
    if (st) die("simulate_shot structure factor", st);
    queue_hkl_copy(ev_hkl, s_hkl, d_hkl, b_hkl);
    if (!g_comp_stream[0] || g_comp_stream_device != cur_dev) {
      for (int k = 0; k < 2; k++) {
        e = cudaStreamCreateWithFlags(&g_comp_stream[k], cudaStreamNonBlocking);
        if (e != cudaSuccess) cuda_die("cudaStreamCreate", e);
      }
      g_comp_stream_device = cur_dev;
    }
    cudaEvent_t ev_ready;
    e = cudaEventCreateWithFlags(&ev_ready, cudaEventDisableTiming);
    if (e != cudaSuccess) cuda_die("cudaEventCreate", e);
    cudaEventRecord(ev_ready, 0);
    for (int c = 0; c < K; c++) {
      const long long r0 = rb[c], r1 = rb[c + 1];
      const long long p0 = r0 * det->nx, p1 = r1 * det->nx;
      const long long b0 = r0 / det->binning_y * bnx;
      const long long b1 = (r1 / det->binning_y < det->ny / det->binning_y ? r1 / det->binning_y
                                                                            : det->ny / det->binning_y) * bnx;
      cudaStream_t s = nfft ? (cudaStream_t)0 : g_comp_stream[c & 1];
      if (s) cudaStreamWaitEvent(s, ev_ready, 0);
      st = nfft ? spsim_internal_shot_nufft_part(p0, p1, dF, dI)
                : spsim_internal_shot_part(p0, p1, opts->b_factor, g_precision, dF, dI, s);
      if (st) die("simulate_shot structure factor", st);
      st = spsim_internal_chain_rows(&p, dI, &o, r0, r1, s);
      if (st) die("simulate_shot detector chain", st);
      cudaEvent_t ev_part;
      e = cudaEventCreateWithFlags(&ev_part, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_copied[c], cudaEventDisableTiming);
      if (e != cudaSuccess) cuda_die("cudaEventCreate", e);
      cudaEventRecord(ev_part, s);
      cudaStreamWaitEvent(g_copy_stream, ev_part, 0);
      cudaEventDestroy(ev_part); /* released once the wait has run */
      e = cudaMemcpyAsync(s_F + sizeof(Complex) * p0, dF + 2 * p0, sizeof(Complex) * (p1 - p0),
                          cudaMemcpyDeviceToHost, g_copy_stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(s_I + sizeof(float) * p0, dI + p0, sizeof(float) * (p1 - p0), cudaMemcpyDeviceToHost,
                            g_copy_stream);
      for (int k = 0; k < 7 && e == cudaSuccess; k++) {
        const long long lo = k < 5 ? p0 : b0, hi = k < 5 ? p1 : b1;
        char *dst = s_chain + (k < 5 ? k * b_I : 5 * b_I + (k - 5) * b_nb) + sizeof(float) * lo;
        if (hi > lo)
          e = cudaMemcpyAsync(dst, bufs[k] + lo, sizeof(float) * (hi - lo), cudaMemcpyDeviceToHost, g_copy_stream);
      }
      if (e != cudaSuccess) cuda_die("cudaMemcpyAsync outputs", e);
      cudaEventRecord(ev_copied[c], g_copy_stream);
    }
    cudaEventDestroy(ev_ready);
  }

  /* meanwhile on the host: the reference-owned outputs, first touched now */
  Diffraction_Pattern *pattern = (Diffraction_Pattern *)calloc(1, sizeof(Diffraction_Pattern));
  pattern->F = (Complex *)host_alloc(b_F > 0 ? b_F : sizeof(Complex));
  pattern->ints = (float *)host_alloc(b_I > 0 ? b_I : sizeof(float));
  pattern->HKL_list = (float *)host_alloc(b_hkl > 0 ? b_hkl : 3 * sizeof(float));
  pattern->HKL_list_size = (int)n;
  pattern->N_pix = (int)n;
  pattern->rot = rot;
  float **dst[7] = {&det->thomson_correction, &det->solid_angle, &det->photons_per_pixel, &det->photon_count,
                    &det->electrons_per_pixel, &det->real_output, &det->noiseless_output};
  HostCopy out[9];
  out[0] = (HostCopy){(char *)pattern->F, s_F, b_F};
  out[1] = (HostCopy){(char *)pattern->ints, s_I, b_I};
  for (int k = 0; k < 7; k++) {
    const size_t b = k < 5 ? b_I : b_nb;
    *dst[k] = (float *)host_alloc(b > 0 ? b : sizeof(float));
    out[2 + k] = (HostCopy){(char *)*dst[k], s_chain + (k < 5 ? k * b_I : 5 * b_I + (k - 5) * b_nb), b};
  }
  HostCopy touch[10];
  for (int k = 0; k < 9; k++) touch[k] = (HostCopy){out[k].dst, NULL, out[k].bytes};
  touch[9] = (HostCopy){(char *)pattern->HKL_list, NULL, b_hkl};
  host_copy_batch(touch, 10);
  e = cudaEventSynchronize(ev_hkl);
  if (e != cudaSuccess) cuda_die("simulate_shot HKL copy", e);
  const HostCopy hk = {(char *)pattern->HKL_list, s_hkl, b_hkl};
  host_copy_batch(&hk, 1);
  if (K == 1) {
    e = cudaEventSynchronize(ev_fi);
    if (e != cudaSuccess) cuda_die("simulate_shot F, I", e);
    host_copy_batch(out, 2);
    e = cudaEventSynchronize(ev_out);
    if (e != cudaSuccess) cuda_die("simulate_shot outputs", e);
    cudaEventDestroy(ev_fi);
    st = spsim_internal_shot_check();
    if (st) die("simulate_shot structure factor", st);
    host_copy_batch(out + 2, 7);
  } else {
    for (int c = 0; c < K; c++) {
      const long long r0 = rb[c], r1 = rb[c + 1];
      const long long p0 = r0 * det->nx, p1 = r1 * det->nx;
      const long long b0 = r0 / det->binning_y * bnx;
      const long long b1 = (r1 / det->binning_y < det->ny / det->binning_y ? r1 / det->binning_y
                                                                            : det->ny / det->binning_y) * bnx;
      e = cudaEventSynchronize(ev_copied[c]);
      if (e != cudaSuccess) cuda_die("simulate_shot outputs", e);
      cudaEventDestroy(ev_copied[c]);
      HostCopy part[9];
      for (int k = 0; k < 9; k++) {
        const size_t el = k == 0 ? sizeof(Complex) : sizeof(float);
        const long long lo = k < 7 ? p0 : b0, hi = k < 7 ? p1 : b1;
        part[k] = (HostCopy){out[k].dst + el * lo, out[k].src + el * lo, hi > lo ? el * (size_t)(hi - lo) : 0};
      }
      host_copy_batch(part, 9);
    }
    st = spsim_internal_shot_check();
    if (st) die("simulate_shot structure factor", st);
  }
  cudaEventDestroy(ev_hkl);
  cudaEventDestroy(ev_out);
  if (opts->verbosity_level > 0) /* src/diffraction.c:849-851 */
    printf("%g atoms.pixel/s\n", 1.0e6 * n * mol->natoms / (now_us() - t0));
  g_pattern_counter++;
  return pattern;
}

/* src/spsim.c:348-371 */
void free_diffraction_pattern(Diffraction_Pattern *pattern) {
  free(pattern->F);
  free(pattern->ints);
  free(pattern->HKL_list);
  if (pattern->rot) free(pattern->rot);
  free(pattern);
}

void free_output_in_options(Options *opts) {
  CCD *d = opts->detector;
  free(d->photons_per_pixel);
  free(d->thomson_correction);
  free(d->solid_angle);
  free(d->photon_count);
  free(d->electrons_per_pixel);
  free(d->real_output);
  free(d->noiseless_output);
  d->photons_per_pixel = d->thomson_correction = d->solid_angle = d->photon_count = NULL;
  d->electrons_per_pixel = d->real_output = d->noiseless_output = NULL;
}

void free_stuff(Diffraction_Pattern *pattern, Options *opts) {
  free_diffraction_pattern(pattern);
  free_output_in_options(opts);
}

/* ------------------------------------------------------------ molecules */

/* src/molecule.c:394-417 */
Molecule *alloc_mol(void) {
  Molecule *mol = (Molecule *)malloc(sizeof(Molecule));
  mol->natoms = 0;
  mol->atomic_number = NULL;
  mol->pos = NULL;
  mol->delta_atoms = 0;
  return mol;
}

void add_atom_to_mol(Molecule *mol, int atomic_number, float x, float y, float z) {
  int i = mol->natoms++;
  mol->atomic_number = (int *)realloc(mol->atomic_number, sizeof(int) * mol->natoms);
  mol->pos = (float *)realloc(mol->pos, sizeof(float) * 3 * mol->natoms);
  mol->atomic_number[i] = atomic_number;
  mol->pos[3 * i] = x;
  mol->pos[3 * i + 1] = y;
  mol->pos[3 * i + 2] = z;
}

void free_mol(Molecule *mol) {
  free(mol->atomic_number);
  free(mol->pos);
  free(mol);
}

/* ------------------------------------------------------------ distribution */

/* src/mpi.c:30-48 without MPI: the whole range */
void get_my_loop_start_and_end(int size, int *start, int *end) {
  *start = 0;
  *end = size;
}

void syncronize_patterns(Diffraction_Pattern *pat) { (void)pat; }
void sum_patterns(Diffraction_Pattern *pat) { (void)pat; }
