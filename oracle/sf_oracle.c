/*
 * ORACLE — test infrastructure only.  Nothing in the product links, loads or
 * calls this file: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, as the checker.
 *
 * An FP64 CPU restatement of spsim's structure-factor and detector-chain
 * arithmetic, written from the reference's behaviour (each function cites the
 * reference lines it follows, paths relative to the spsim tree).  Where the
 * reference computes in float, this restatement computes in double from the
 * same float inputs, so it is the accuracy yardstick; the reference's own
 * float results are checked against it in tests/test_oracle_golden.py.
 *
 * Pinned against: golden vectors produced by spsim's own sources compiled
 * unchanged (oracle/Makefile, target ref -> oracle/_ref/libspsim_ref.so), committed
 * under tests/golden/.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../spsim_b200/csrc/atomsf_data.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static float g_atomsf[SPSIM_B200_N_ELEMENTS][9];
static int g_atomsf_ready = 0;

static void ensure_table(void) {
  if (!g_atomsf_ready) {
    memcpy(g_atomsf, spsim_b200_atomsf_default, sizeof(g_atomsf));
    g_atomsf_ready = 1;
  }
}

/* Replace one row of the coefficient table (the reference lets ./atomsf.lib
 * override the compiled-in rows: src/diffraction.c:118-177). */
void oracle_set_atomsf_row(int Z, const float *coeffs9) {
  ensure_table();
  if (Z < 0 || Z >= SPSIM_B200_N_ELEMENTS) return;
  memcpy(g_atomsf[Z], coeffs9, 9 * sizeof(float));
}

void oracle_reset_atomsf(void) { g_atomsf_ready = 0; ensure_table(); }

/* Row Z of the coefficient table in use. */
void oracle_get_atomsf_row(int Z, float *coeffs9) {
  ensure_table();
  if (Z < 0 || Z >= SPSIM_B200_N_ELEMENTS) return;
  memcpy(coeffs9, g_atomsf[Z], 9 * sizeof(float));
}

/* src/diffraction.c:183-193: f(|q|) = sum_i a_i exp(-(b_i+B) d^2/4) + c exp(-B d^2/4),
 * d = |q| * 1e-10 (1/m -> 1/Angstrom).  Here in FP64 throughout. */
double oracle_scatt_factor(double q_len, int Z, double B) {
  ensure_table();
  double d = q_len * 1e-10;
  double d2q = d * d * 0.25;
  double res = 0.0;
  for (int i = 0; i < 4; i++) res += (double)g_atomsf[Z][i] * exp(-((double)g_atomsf[Z][i + 4] + B) * d2q);
  res += (double)g_atomsf[Z][8] * exp(-B * d2q);
  return res;
}

/* src/diffraction.c:223-235: Gaussian beam profile; 1 when fwhm == 0. */
static double illumination(double fwhm, double cx, double cy, double x, double y) {
  if (fwhm == 0.0) return 1.0;
  double dist2 = (x - cx) * (x - cx) + (y - cy) * (y - cy);
  double sigma = fwhm / 2.355;
  return exp(-dist2 / (2 * sigma * sigma));
}

/* src/diffraction.c:237-297: Ewald-sphere q (1/m) of every pixel of a flat
 * 2-D detector, row-major (y outer, x inner); FP64 out.  The spherical branch
 * keeps the reference's float quotient width/nx (:259-260). */
void oracle_hkl_detector(int nx, int ny, float width, float height, float distance, float center_x,
                         float center_y, float wavelength, int spherical, double *q) {
  double ewald = 1.0 / (double)wavelength;
  double pz = distance;
  double px_size = (double)(width / nx);
  double py_size = (double)(height / ny);
  double fpx = 2 * sin(atan(px_size / pz) / 2) / (double)wavelength;
  double fpy = 2 * sin(atan(py_size / pz) / 2) / (double)wavelength;
  long idx = 0;
  for (int y = 0; y < ny; y++) {
    for (int x = 0; x < nx; x++) {
      double px = ((x - (nx - 1.0) / 2.0) / nx) * (double)width - (double)center_x;
      double py = ((y - (ny - 1.0) / 2.0) / ny) * (double)height - (double)center_y;
      double p = sqrt(px * px + py * py + pz * pz);
      if (!spherical) {
        q[idx++] = px / p * ewald;
        q[idx++] = py / p * ewald;
        q[idx++] = (pz / p - 1.0) * ewald;
      } else {
        q[idx++] = fpx * px / px_size;
        q[idx++] = fpy * py / py_size;
        q[idx++] = 0.0;
      }
    }
  }
}

/* src/crystal.c:39-71 in FP64: F <- F * sum over the na x nb x nc cells r =
 * aA + bB + cC of exp(-2 pi i q.r) (cell rows A, B, C), I = |F|^2. */
void oracle_crystal(long npix, const double *q, const double *cell, int na, int nb, int nc, double *F_re,
                    double *F_im, double *I) {
  for (long p = 0; p < npix; p++) {
    double sr = 0.0, si = 0.0;
    for (int a = 0; a < na; a++)
      for (int b = 0; b < nb; b++)
        for (int c = 0; c < nc; c++) {
          const double r[3] = {cell[0] * a + cell[3] * b + cell[6] * c, cell[1] * a + cell[4] * b + cell[7] * c,
                               cell[2] * a + cell[5] * b + cell[8] * c};
          double t = q[3 * p] * r[0] + q[3 * p + 1] * r[1] + q[3 * p + 2] * r[2];
          t -= rint(t);
          sr += cos(2.0 * M_PI * t);
          si -= sin(2.0 * M_PI * t);
        }
    const double re = F_re[p] * sr - F_im[p] * si, im = F_re[p] * si + F_im[p] * sr;
    F_re[p] = re;
    F_im[p] = im;
    if (I) I[p] = re * re + im * im;
  }
}

/* src/diffraction.c:325-369: the reciprocal-space grid of a 3-D detector,
 * FP64, stored as float like the reference (z outer, x inner). */
void oracle_hkl_3d_detector(int nx, int ny, int nz, float width, float height, float depth, float distance,
                            float center_x, float center_y, float center_z, float wavelength, float *out) {
  const float dl = distance * wavelength;
  const double r2r = 1.0 / dl;
  long idx = 0;
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        const double px = ((x - (nx - 1.0) / 2.0) / nx) * width - center_x;
        const double py = ((y - (ny - 1.0) / 2.0) / ny) * height - center_y;
        const double pz = ((z - (nz - 1.0) / 2.0) / nz) * depth - center_z;
        out[idx++] = (float)(px * r2r);
        out[idx++] = (float)(py * r2r);
        out[idx++] = (float)(pz * r2r);
      }
}

/*
 * src/diffraction.c:770-853 (compute_pattern_on_list), FP64:
 *   F(q) = sum_j f_Zj(|q|, B_j) * occ_j * sqrt(illum_j) * exp(-2 pi i q.r_j),  I = |F|^2
 * Atoms with Z == 0 are skipped (:830-832); delta_atoms replaces f*sqrt(illum)
 * by 1 (:837-843).  Extensions beyond the reference: per-atom occupancy (occ,
 * NULL = 1) and per-atom B (bj, NULL = none), added to the global B.
 */
typedef struct {
  int natoms;
  const int *Z;
  const double *pos, *occ, *bj, *w;
  double B;
  int delta_atoms;
  long p0, p1;
  const double *q;
  double *F_re, *F_im, *I;
  double qscale; /* the phase uses qscale * q; form factors stay at |q| */
} sf_job_t;

static void *sf_worker(void *arg) {
  sf_job_t *jb = (sf_job_t *)arg;
  for (long i = jb->p0; i < jb->p1; i++) {
    double qx = jb->q[3 * i], qy = jb->q[3 * i + 1], qz = jb->q[3 * i + 2];
    double qlen = sqrt(qx * qx + qy * qy + qz * qz);
    double cache[SPSIM_B200_N_ELEMENTS];
    int have[SPSIM_B200_N_ELEMENTS];
    memset(have, 0, sizeof(have));
    double re = 0.0, im = 0.0;
    for (int j = 0; j < jb->natoms; j++) {
      int z = jb->Z[j];
      if (!z) continue;
      double f;
      if (jb->delta_atoms) {
        f = 1.0;
      } else if (jb->bj) {
        f = oracle_scatt_factor(qlen, z, jb->B + jb->bj[j]);  /* the global B adds to the atom's own */
      } else {
        if (!have[z]) {
          cache[z] = oracle_scatt_factor(qlen, z, jb->B);
          have[z] = 1;
        }
        f = cache[z];
      }
      const double *r = jb->pos + 3 * j;
      double t = jb->qscale * (qx * r[0] + qy * r[1] + qz * r[2]);
      t -= rint(t);
      double s, c;
      sincos(-2.0 * M_PI * t, &s, &c);
      re += f * jb->w[j] * c;
      im += f * jb->w[j] * s;
    }
    jb->F_re[i] = re;
    jb->F_im[i] = im;
    if (jb->I) jb->I[i] = re * re + im * im;
  }
  return NULL;
}

/* Run fn on nthreads prepared jobs, each a contiguous slab (the reference's
 * own MPI pixel-slab split, src/mpi.c:30-48). */
static void run_slabs(int nthreads, void *jobs, size_t job_size, void *(*fn)(void *)) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  for (int t = 0; t < nthreads; t++) {
    char *jb = (char *)jobs + (size_t)t * job_size;
    if (nthreads == 1) {
      fn(jb);
    } else {
      pthread_create(&th[t], NULL, fn, jb);
    }
  }
  if (nthreads > 1)
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
}

void oracle_structure_factor(int natoms, const int *Z, const double *pos, const double *occ,
                             const double *bj, double B, int delta_atoms, double beam_fwhm,
                             double beam_cx, double beam_cy, long npix, const double *q,
                             double *F_re, double *F_im, double *I, int nthreads) {
  ensure_table();
  double *w = (double *)malloc(sizeof(double) * (natoms > 0 ? natoms : 1));
  for (int j = 0; j < natoms; j++) {
    double o = occ ? occ[j] : 1.0;
    w[j] = delta_atoms ? 1.0 : o * sqrt(illumination(beam_fwhm, beam_cx, beam_cy, pos[3 * j], pos[3 * j + 1]));
  }
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  sf_job_t jobs[256];
  for (int t = 0; t < nthreads; t++) {
    sf_job_t j = {natoms, Z, pos, occ, bj, w, B, delta_atoms,
                  npix * t / nthreads, npix * (t + 1) / nthreads, q, F_re, F_im, I, 1.0};
    jobs[t] = j;
  }
  run_slabs(nthreads, jobs, sizeof(sf_job_t), sf_worker);
  free(w);
}

/*
 * src/diffraction.cu:415-476 (CUDA_spectrum_scattering_from_all_atoms) in FP64,
 * with the sample count rule of :305-307 (an even count above one is raised by
 * one).  lambda_j = lambda (1 - bw/2) + j/(S-1) lambda bw, the phase of sample
 * j uses q lambda/lambda_j, the form factor the unscaled |q| (:440-447), the
 * weight exp(-z^2/2) with z = (lambda_j - lambda) / ((lambda - lambda (1 -
 * bw/2)) / 2) (:431, :454-456); the amplitude is the weighted mean over the
 * samples (:465-466).  bandwidth == 0 or S == 1: the monochromatic sum.
 */
void oracle_structure_factor_spectrum(int natoms, const int *Z, const double *pos, const double *occ,
                                      const double *bj, double B, int delta_atoms, double beam_fwhm,
                                      double beam_cx, double beam_cy, double wavelength, double bandwidth,
                                      int samples, long npix, const double *q, double *F_re, double *F_im,
                                      double *I, int nthreads) {
  if (samples > 1 && (samples & 1) == 0) samples++;
  if (bandwidth == 0.0 || samples <= 1) {
    oracle_structure_factor(natoms, Z, pos, occ, bj, B, delta_atoms, beam_fwhm, beam_cx, beam_cy, npix, q, F_re,
                            F_im, I, nthreads);
    return;
  }
  ensure_table();
  double *w = (double *)malloc(sizeof(double) * (natoms > 0 ? natoms : 1));
  for (int j = 0; j < natoms; j++) {
    double o = occ ? occ[j] : 1.0;
    w[j] = delta_atoms ? 1.0 : o * sqrt(illumination(beam_fwhm, beam_cx, beam_cy, pos[3 * j], pos[3 * j + 1]));
  }
  double *re = (double *)malloc(sizeof(double) * (npix > 0 ? npix : 1));
  double *im = (double *)malloc(sizeof(double) * (npix > 0 ? npix : 1));
  for (long i = 0; i < npix; i++) F_re[i] = F_im[i] = 0.0;
  const double sigma = (wavelength - wavelength * (1.0 - bandwidth / 2.0)) / 2.0;
  double total = 0.0;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  for (int s = 0; s < samples; s++) {
    const double lj = wavelength * (1.0 - bandwidth / 2.0) + ((double)s / (samples - 1)) * wavelength * bandwidth;
    const double z = (lj - wavelength) / sigma;
    const double ws = exp(-z * z / 2.0);
    total += ws;
    sf_job_t jobs[256];
    for (int t = 0; t < nthreads; t++) {
      sf_job_t jb = {natoms, Z, pos, occ, bj, w, B, delta_atoms,
                     npix * t / nthreads, npix * (t + 1) / nthreads, q, re, im, NULL, wavelength / lj};
      jobs[t] = jb;
    }
    run_slabs(nthreads, jobs, sizeof(sf_job_t), sf_worker);
    for (long i = 0; i < npix; i++) {
      F_re[i] += ws * re[i];
      F_im[i] += ws * im[i];
    }
  }
  for (long i = 0; i < npix; i++) {
    F_re[i] /= total;
    F_im[i] /= total;
    if (I) I[i] = F_re[i] * F_re[i] + F_im[i] * F_im[i];
  }
  free(re);
  free(im);
  free(w);
}

/*
 * Vector-Jacobian product of I = |F|^2 through the structure factor above:
 * given g_p = dL/dI_p, returns dL/dr_j (1/m units, 3 per atom), dL/docc_j and
 * dL/dB_j (per Angstrom^2), all FP64.  Used to check the adjoint kernel.
 *   dI/dr   = 4 pi Re... : dL/dr_j  = sum_p 4 pi g_p a_pj q_p Im(conj(F_p) e^{i phi_pj})
 *   dL/docc_j = sum_p 2 g_p (a_pj/occ_j) Re(conj(F_p) e^{i phi_pj})
 *   dL/dB_j   = sum_p 2 g_p a_pj (-s_p^2) Re(conj(F_p) e^{i phi_pj}),  s^2 = (|q| 1e-10)^2/4
 * with a_pj = f_Zj(|q_p|, B_j) occ_j and phi_pj = -2 pi q_p.r_j (no illumination
 * weighting: the refinement path uses a plane-wave beam).
 */
typedef struct {
  int j0, j1;
  const int *Z;
  const double *pos, *occ, *bj, *q, *g, *Fr, *Fi;
  long npix;
  double *d_pos, *d_occ, *d_b;
} vjp_job_t;

static void *vjp_worker(void *arg) {
  vjp_job_t *jb = (vjp_job_t *)arg;
  for (int j = jb->j0; j < jb->j1; j++) {
    double gx = 0, gy = 0, gz = 0, go = 0, gb = 0;
    int z = jb->Z[j];
    if (z) {
      for (long p = 0; p < jb->npix; p++) {
        const double *qq = jb->q + 3 * p;
        double qlen = sqrt(qq[0] * qq[0] + qq[1] * qq[1] + qq[2] * qq[2]);
        double d = qlen * 1e-10;
        double s2 = d * d * 0.25;
        double f = oracle_scatt_factor(qlen, z, jb->bj ? jb->bj[j] : 0.0);
        double o = jb->occ ? jb->occ[j] : 1.0;
        const double *r = jb->pos + 3 * j;
        double t = qq[0] * r[0] + qq[1] * r[1] + qq[2] * r[2];
        t -= rint(t);
        double s, c;
        sincos(-2.0 * M_PI * t, &s, &c);
        /* conj(F) * e^{i phi} */
        double zr = jb->Fr[p] * c + jb->Fi[p] * s;
        double zi = jb->Fr[p] * s - jb->Fi[p] * c;
        double a = f * o;
        double k = 4.0 * M_PI * jb->g[p] * a * zi;
        gx += k * qq[0];
        gy += k * qq[1];
        gz += k * qq[2];
        go += 2.0 * jb->g[p] * f * zr;
        gb += 2.0 * jb->g[p] * a * (-s2) * zr;
      }
    }
    jb->d_pos[3 * j] = gx;
    jb->d_pos[3 * j + 1] = gy;
    jb->d_pos[3 * j + 2] = gz;
    if (jb->d_occ) jb->d_occ[j] = go;
    if (jb->d_b) jb->d_b[j] = gb;
  }
  return NULL;
}

void oracle_structure_factor_vjp(int natoms, const int *Z, const double *pos, const double *occ,
                                 const double *bj, long npix, const double *q, const double *g,
                                 double *d_pos, double *d_occ, double *d_b, int nthreads) {
  ensure_table();
  double *Fr = (double *)malloc(sizeof(double) * (npix > 0 ? npix : 1));
  double *Fi = (double *)malloc(sizeof(double) * (npix > 0 ? npix : 1));
  oracle_structure_factor(natoms, Z, pos, occ, bj, 0.0, 0, 0.0, 0.0, 0.0, npix, q, Fr, Fi, NULL, nthreads);
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  vjp_job_t jobs[256];
  for (int t = 0; t < nthreads; t++) {
    vjp_job_t jb = {(int)((long)natoms * t / nthreads), (int)((long)natoms * (t + 1) / nthreads), Z, pos, occ, bj,
                    q, g, Fr, Fi, npix, d_pos, d_occ, d_b};
    jobs[t] = jb;
  }
  run_slabs(nthreads, jobs, sizeof(vjp_job_t), vjp_worker);
  free(Fr);
  free(Fi);
}

/* src/diffraction.c:1109-1144: r0^2 times the polarisation factor. */
void oracle_thomson(int nx, int ny, int nz, float width, float height, float distance, float center_x,
                    float center_y, int polarization, double *out) {
  double r0 = 2.81794e-15;
  double DD = (double)distance * distance;
  long idx = 0;
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        double pf = 1.0;
        if (polarization != 0) {
          double px = ((x - (nx - 1.0) / 2.0) / nx) * (double)width - (double)center_x;
          double py = ((y - (ny - 1.0) / 2.0) / ny) * (double)height - (double)center_y;
          double r = sqrt(px * px + py * py + DD);
          double chi;
          if (polarization == 1) { /* vertical */
            chi = asin(py / r);
            pf = cos(chi) * cos(chi);
          } else if (polarization == 2) { /* horizontal */
            chi = asin(px / r);
            pf = cos(chi) * cos(chi);
          } else if (polarization == 3) { /* unpolarised */
            chi = asin(sqrt(px * px + py * py) / r);
            pf = (1.0 + cos(chi) * cos(chi)) / 2.0;
          }
        }
        out[idx++] = r0 * r0 * pf;
      }
}

/* src/diffraction.c:1146-1187: pixel solid angle; cos^3 of the incidence
 * angle for a flat 2-D detector, pw*ph/d^2 for 3-D or spherical. */
void oracle_solid_angle(int nx, int ny, int nz, float width, float height, float distance, float center_x,
                        float center_y, float pixel_width, float pixel_height, int spherical, double *out) {
  int is3d = nz > 1;
  double d2 = (double)distance * distance;
  long idx = 0;
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        if (is3d || spherical) {
          double r = distance;
          out[idx++] = (double)pixel_width * pixel_height / (r * r);
        } else {
          double px = ((x - (nx - 1.0) / 2.0) / nx) * (double)width - (double)center_x;
          double py = ((y - (ny - 1.0) / 2.0) / ny) * (double)height - (double)center_y;
          double inc = cos(atan(sqrt(px * px + py * py) / distance));
          out[idx++] = (double)pixel_width * pixel_height / d2 * inc * inc * inc;
        }
      }
}

/* src/amplification.c:119-155: noiseless binned output
 *   sum_bin photons * QE * (hc/lambda)/e_hole * ADC,  ADC = max/full_well when both set. */
void oracle_noiseless_output(int nx, int ny, int nz, int bx, int by, int bz, const double *photons, double qe,
                             double wavelength, double e_hole, double full_well, double max_value, double *out) {
  double hc = 1.98644521e-25;
  double epp = (hc / wavelength) / e_hole;
  double adc = (full_well != 0 && max_value != 0) ? max_value / full_well : 1.0;
  long i = 0;
  for (int z = 0; z < nz / bz; z++)
    for (int y = 0; y < ny / by; y++)
      for (int x = 0; x < nx / bx; x++) {
        double acc = 0;
        for (int zi = 0; zi < bz; zi++)
          for (int yi = 0; yi < by; yi++)
            for (int xi = 0; xi < bx; xi++)
              acc += photons[((long)(z * bz + zi) * ny + (y * by + yi)) * nx + (x * bx + xi)] * qe * epp * adc;
        out[i++] = acc;
      }
}

/* src/amplification.c:77-116: binned real output for given readout deviates
 * noise[b] ~ N(0, sigma):  max(0, sum_bin(e + dark*t) + noise) * ADC, plus the
 * optional upper clamp at max_value (an extension, off when clamp == 0). */
void oracle_real_output(int nx, int ny, int nz, int bx, int by, int bz, const double *electrons, double dark,
                        double exposure, const double *noise, double full_well, double max_value, int clamp,
                        double *out) {
  double adc = (full_well != 0 && max_value != 0) ? max_value / full_well : 1.0;
  long i = 0;
  for (int z = 0; z < nz / bz; z++)
    for (int y = 0; y < ny / by; y++)
      for (int x = 0; x < nx / bx; x++) {
        double acc = 0;
        for (int zi = 0; zi < bz; zi++)
          for (int yi = 0; yi < by; yi++)
            for (int xi = 0; xi < bx; xi++)
              acc += electrons[((long)(z * bz + zi) * ny + (y * by + yi)) * nx + (x * bx + xi)] + dark * exposure;
        acc += noise ? noise[i] : 0.0;
        if (acc < 0) acc = 0;
        acc *= adc;
        if (clamp && max_value != 0 && acc > max_value) acc = max_value;
        out[i++] = acc;
      }
}

/* ------------------------------------------------------------------------ */
/* Counter-based noise, restated for the checker.  Philox4x32-10 (Salmon,
 * Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11)
 * keyed by the 64-bit seed; counter = (pixel, pattern, stream, draw).      */

static void philox4x32_10(uint32_t ctr[4], uint32_t key0, uint32_t key1, uint32_t out[4]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key0, k1 = key1;
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)M0 * c0, p1 = (uint64_t)M1 * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += W0;
    k1 += W1;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void oracle_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t seed, uint32_t *out4) {
  uint32_t ctr[4] = {c0, c1, c2, c3};
  philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), out4);
}

/* 32 random bits -> float uniform in (0, 1): (x >> 8 + 0.5) * 2^-24 */
static float u01(uint32_t x) { return ((float)(x >> 8) + 0.5f) * 5.9604644775390625e-8f; }

typedef struct {
  uint32_t ctr[4];
  uint32_t key0, key1;
  uint32_t buf[4];
  int left;
} stream_t;

static void stream_init(stream_t *s, uint32_t pixel, uint32_t pattern, uint32_t sid, uint64_t seed) {
  s->ctr[0] = pixel; s->ctr[1] = pattern; s->ctr[2] = sid; s->ctr[3] = 0;
  s->key0 = (uint32_t)seed; s->key1 = (uint32_t)(seed >> 32);
  s->left = 0;
}

static float stream_uniform(stream_t *s) {
  if (s->left == 0) {
    philox4x32_10(s->ctr, s->key0, s->key1, s->buf);
    s->ctr[3]++;
    s->left = 4;
  }
  return u01(s->buf[4 - s->left--]);
}

/* Box-Muller on two uniforms, first of the pair. */
static float stream_normal(stream_t *s) {
  float a = stream_uniform(s), b = stream_uniform(s);
  return sqrtf(-2.0f * logf(a)) * cosf(6.2831853071795864f * b);
}

/* Poisson(lam) as the product samples it: inversion for lam < 10, Hormann's
 * PTRS transformed rejection (Insurance: Math. & Econ. 12 (1993) 39-45) for
 * 10 <= lam < 1000, and the reference's Gaussian approximation
 * (int)(lam + N(0, sqrt(lam))) at lam >= 1000 (src/noise.c:42-46). */
static float poisson_sample(stream_t *s, float lam) {
  if (!(lam > 0.0f)) return 0.0f;
  if (lam >= 1000.0f) {
    float v = lam + sqrtf(lam) * stream_normal(s);
    return (float)(int)v;
  }
  if (lam < 10.0f) {
    float u = stream_uniform(s);
    float p = expf(-lam), F = p;
    int k = 0;
    while (u > F && k < 200) {
      k++;
      p *= lam / (float)k;
      F += p;
    }
    return (float)k;
  }
  float slam = sqrtf(lam), loglam = logf(lam);
  float b = 0.931f + 2.53f * slam;
  float a = -0.059f + 0.02483f * b;
  float inv_alpha = 1.1239f + 1.1328f / (b - 3.4f);
  float vr = 0.9277f - 3.6224f / (b - 2.0f);
  for (int it = 0; it < 64; it++) {
    float U = stream_uniform(s) - 0.5f;
    float V = stream_uniform(s);
    float us = 0.5f - fabsf(U);
    float k = floorf((2.0f * a / us + b) * U + lam + 0.43f);
    if (us >= 0.07f && V <= vr) return k;
    if (k < 0.0f || (us < 0.013f && V > us)) continue;
    if (logf(V) + logf(inv_alpha) - logf(a / (us * us) + b) <= -lam + k * loglam - lgammaf(k + 1.0f)) return k;
  }
  return (float)(int)(lam + slam * stream_normal(s));
}

/* Photon counts for an array of expected values lam[i] (already times QE):
 * the checker's copy of the product's noise stream 0. */
void oracle_poisson(long n, const float *lam, uint32_t pattern, uint64_t seed, float *out) {
  for (long i = 0; i < n; i++) {
    stream_t s;
    stream_init(&s, (uint32_t)i, pattern, 0u, seed);
    out[i] = poisson_sample(&s, lam[i]);
  }
}

/* Readout deviates N(0, sigma) per binned pixel: noise stream 1. */
void oracle_readout_noise(long n, float sigma, uint32_t pattern, uint64_t seed, float *out) {
  for (long i = 0; i < n; i++) {
    stream_t s;
    stream_init(&s, (uint32_t)i, pattern, 1u, seed);
    out[i] = sigma * stream_normal(&s);
  }
}
