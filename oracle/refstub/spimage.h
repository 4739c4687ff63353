/*
 * Test infrastructure only: a minimal stand-in for libspimage's public header,
 * written for this project so that spsim's own hot-path sources
 * (src/diffraction.c, src/amplification.c, src/mpi.c, src/noise.c,
 * src/config.c) compile unchanged into the CPU reference library under
 * oracle/_ref/.  libspimage itself is not available (spsim's CI clones its
 * master branch; .github/workflows/test.yml:40-50), so nothing here is its
 * code: it declares the names and signatures those sources use, implements
 * the few that the structure-factor / detector-chain path calls (complex
 * helpers, timers, 3x3 rotations, p_drand48) and makes every image/FFT
 * routine abort, since the hot path never reaches them.
 *
 * Parity unpinned for libspimage-owned behaviour (rotation conventions,
 * p_drand48 stream): the rebuild documents its own conventions instead.
 */
#ifndef SPSIM_ORACLE_SPIMAGE_STUB_H
#define SPSIM_ORACLE_SPIMAGE_STUB_H

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

/* the CUDA build of src/diffraction.cu: libspimage's CUDA helpers, as checks
 * that print and abort; cufftComplex comes from the toolkit header */
#ifdef __CUDACC__
#include <cuda_runtime.h>
#include <cufft.h>
#define cutilSafeCall(call)                                                            \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      fprintf(stderr, "reference CUDA call failed: %s\n", cudaGetErrorString(e_));     \
      abort();                                                                         \
    }                                                                                  \
  } while (0)
#define sp_cuda_check_errors() cutilSafeCall(cudaGetLastError())
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef float real;

typedef struct {
  real re;
  real im;
} Complex;

#define sp_real(a) ((a).re)
#define sp_imag(a) ((a).im)
#define sp_min(a, b) (((a) < (b)) ? (a) : (b))
#define sp_max(a, b) (((a) > (b)) ? (a) : (b))

static inline real sp_cabs(Complex a) { return (real)sqrt(a.re * a.re + a.im * a.im); }
static inline real sp_cabs2(Complex a) { return a.re * a.re + a.im * a.im; }
static inline real sp_carg(Complex a) { return (real)atan2(a.im, a.re); }
static inline Complex sp_cinit(real re, real im) { Complex c; c.re = re; c.im = im; return c; }
static inline Complex sp_cscale(Complex a, real s) { Complex c; c.re = a.re * s; c.im = a.im * s; return c; }

/* row-major dense matrix, the layout libspimage's sp_matrix uses */
typedef struct {
  unsigned int rows;
  unsigned int cols;
  real *data;
} sp_matrix;

typedef struct {
  unsigned int size;
  real *data;
} sp_vector;

typedef sp_matrix SpRotation;

typedef struct {
  real image_center[3];
  real pixel_size[3];
  real detector_distance;
  real wavelength;
  SpRotation *orientation;
} Detector;

typedef struct {
  int x, y, z;
  Complex *data;
} sp_c3matrix;

typedef struct {
  int x, y, z;
  int *data;
} sp_i3matrix;

typedef struct {
  sp_c3matrix *image;
  sp_i3matrix *mask;
  Detector *detector;
} Image;

int sp_timer_start(void);
long long sp_timer_stop(int timer); /* microseconds */

sp_vector *sp_vector_alloc(unsigned int n);
void sp_vector_free(sp_vector *v);
sp_vector *sp_matrix_vector_prod(const sp_matrix *m, const sp_vector *v);
SpRotation *sp_rot_euler(real a1, real a2, real a3);
SpRotation *sp_rot_uniform(void);

double p_drand48(void);
void sp_srand(int seed);
void sp_error_fatal(const char *msg, ...);

Image *sp_image_alloc(int x, int y, int z);
void sp_image_free(Image *img);
int sp_image_write(Image *img, const char *filename, int flags);
Image *sp_image_fft(Image *img);
Image *sp_image_shift(Image *img);
Complex sp_image_get(Image *img, int x, int y, int z);
void sp_image_set(Image *img, int x, int y, int z, Complex v);
void sp_i3matrix_set(sp_i3matrix *m, int x, int y, int z, int v);
#define sp_image_x(a) ((a)->image->x)
#define sp_image_y(a) ((a)->image->y)
#define sp_image_z(a) ((a)->image->z)
#define sp_image_size(a) ((a)->image->x * (a)->image->y * (a)->image->z)

#ifdef __cplusplus
}
#endif

#endif
