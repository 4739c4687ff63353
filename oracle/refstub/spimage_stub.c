/*
 * Test infrastructure only: definitions behind oracle/refstub/spimage.h.
 * Linked into oracle/_ref/libspsim_ref.so together with spsim's own sources.
 *
 * sp_rot_euler follows the convention this project documents for its own
 * geometry (intrinsic z-y-z: R = Rz(a1) Ry(a2) Rz(a3)); libspimage's own
 * convention is not available here, so orientation parity is unpinned.
 */
#include "spimage.h"

#include <stdarg.h>
#include <stdint.h>
#include <string.h>
#include <time.h>

#define MAX_TIMERS 64
static struct timespec g_timers[MAX_TIMERS];
static int g_next_timer = 0;

int sp_timer_start(void) {
  int t = g_next_timer;
  g_next_timer = (g_next_timer + 1) % MAX_TIMERS;
  clock_gettime(CLOCK_MONOTONIC, &g_timers[t]);
  return t;
}

long long sp_timer_stop(int timer) {
  struct timespec now;
  clock_gettime(CLOCK_MONOTONIC, &now);
  long long us = (long long)(now.tv_sec - g_timers[timer].tv_sec) * 1000000LL +
                 (now.tv_nsec - g_timers[timer].tv_nsec) / 1000;
  return us > 0 ? us : 1;
}

sp_vector *sp_vector_alloc(unsigned int n) {
  sp_vector *v = (sp_vector *)malloc(sizeof(sp_vector));
  v->size = n;
  v->data = (real *)calloc(n, sizeof(real));
  return v;
}

void sp_vector_free(sp_vector *v) {
  if (!v) return;
  free(v->data);
  free(v);
}

sp_vector *sp_matrix_vector_prod(const sp_matrix *m, const sp_vector *v) {
  sp_vector *u = sp_vector_alloc(m->rows);
  for (unsigned int i = 0; i < m->rows; i++) {
    real acc = 0;
    for (unsigned int j = 0; j < m->cols; j++) acc += m->data[i * m->cols + j] * v->data[j];
    u->data[i] = acc;
  }
  return u;
}

static SpRotation *rot_alloc(void) {
  SpRotation *r = (SpRotation *)malloc(sizeof(SpRotation));
  r->rows = 3;
  r->cols = 3;
  r->data = (real *)calloc(9, sizeof(real));
  return r;
}

SpRotation *sp_rot_euler(real a1, real a2, real a3) {
  double c1 = cos(a1), s1 = sin(a1), c2 = cos(a2), s2 = sin(a2), c3 = cos(a3), s3 = sin(a3);
  /* Rz(a1) * Ry(a2) * Rz(a3) */
  double m[9] = {c1 * c2 * c3 - s1 * s3, -c1 * c2 * s3 - s1 * c3, c1 * s2,
                 s1 * c2 * c3 + c1 * s3, -s1 * c2 * s3 + c1 * c3, s1 * s2,
                 -s2 * c3, s2 * s3, c2};
  SpRotation *r = rot_alloc();
  for (int i = 0; i < 9; i++) r->data[i] = (real)m[i];
  return r;
}

SpRotation *sp_rot_uniform(void) {
  /* Shoemake's uniform random quaternion from three uniform deviates */
  double u1 = p_drand48(), u2 = p_drand48(), u3 = p_drand48();
  double a = sqrt(1 - u1), b = sqrt(u1);
  double w = a * sin(2 * M_PI * u2), x = a * cos(2 * M_PI * u2);
  double y = b * sin(2 * M_PI * u3), z = b * cos(2 * M_PI * u3);
  double m[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                 2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                 2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)};
  SpRotation *r = rot_alloc();
  for (int i = 0; i < 9; i++) r->data[i] = (real)m[i];
  return r;
}

/* POSIX drand48 recurrence: X <- (0x5DEECE66D X + 0xB) mod 2^48 */
static uint64_t g_rand48 = 0x1234ABCD330EULL;

double p_drand48(void) {
  g_rand48 = (0x5DEECE66DULL * g_rand48 + 0xBULL) & ((1ULL << 48) - 1);
  return (double)g_rand48 / (double)(1ULL << 48);
}

void sp_srand(int seed) { g_rand48 = (((uint64_t)(uint32_t)seed) << 16) | 0x330EULL; }

void sp_error_fatal(const char *msg, ...) {
  va_list ap;
  va_start(ap, msg);
  fprintf(stderr, "spimage stub fatal: ");
  vfprintf(stderr, msg, ap);
  fprintf(stderr, "\n");
  va_end(ap);
  abort();
}

static void unavailable(const char *what) {
  fprintf(stderr, "spimage stub: %s is not available in the oracle build\n", what);
  abort();
}

Image *sp_image_alloc(int x, int y, int z) { (void)x; (void)y; (void)z; unavailable("sp_image_alloc"); return NULL; }
void sp_image_free(Image *img) { (void)img; unavailable("sp_image_free"); }
int sp_image_write(Image *img, const char *f, int fl) { (void)img; (void)f; (void)fl; unavailable("sp_image_write"); return 0; }
Image *sp_image_fft(Image *img) { (void)img; unavailable("sp_image_fft"); return NULL; }
Image *sp_image_shift(Image *img) { (void)img; unavailable("sp_image_shift"); return NULL; }
Complex sp_image_get(Image *img, int x, int y, int z) {
  (void)img; (void)x; (void)y; (void)z;
  unavailable("sp_image_get");
  return sp_cinit(0, 0);
}
void sp_image_set(Image *img, int x, int y, int z, Complex v) { (void)img; (void)x; (void)y; (void)z; (void)v; unavailable("sp_image_set"); }
void sp_i3matrix_set(sp_i3matrix *m, int x, int y, int z, int v) { (void)m; (void)x; (void)y; (void)z; (void)v; unavailable("sp_i3matrix_set"); }
