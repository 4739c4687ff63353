/*
 * The spsim command-line program (src/spsim.c:374-415) on this library: read
 * spsim.conf, echo the options to spsim.confout, build the molecule (PDB or
 * chemical formula), and for each of n_patterns shots run simulate_shot and
 * write the requested outputs.
 *
 * Outputs: spsim writes its arrays as CXI files through libspimage (HDF5),
 * neither of which this build has; each array goes instead to
 * <name>-NNNNN.npy (NumPy format 1.0, little-endian float32, shape (nz, ny, nx)
 * with singleton nz dropped; complex64 for the scattering factors) under the
 * same base name spsim uses (src/spsim.c:228-279).  scattering_factor-NNNNN.vtk
 * (output_sf_vtk) is written exactly as spsim does.  Real-space outputs and the
 * real-space histogram (FFT of the pattern) are not part of this path and are
 * reported as skipped.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../../include/spsim.h"
#include "../../../include/spsim_b200.h"

static void write_npy(const char *base, int index, const void *data, int complex_values, const CCD *det, int binned) {
  char name[1100];
  snprintf(name, sizeof(name), "%s-%05d.npy", base, index);
  const int nx = binned ? det->nx / det->binning_x : det->nx;
  const int ny = binned ? det->ny / det->binning_y : det->ny;
  const int nzr = det->nz > 0 ? det->nz : 1;
  const int nz = binned ? nzr / det->binning_z : nzr;
  char shape[96];
  if (nz > 1)
    snprintf(shape, sizeof(shape), "(%d, %d, %d)", nz, ny, nx);
  else
    snprintf(shape, sizeof(shape), "(%d, %d)", ny, nx);
  char header[256];
  int hl = snprintf(header, sizeof(header), "{'descr': '%s', 'fortran_order': False, 'shape': %s, }",
                    complex_values ? "<c8" : "<f4", shape);
  const int total = 10 + hl + 1;
  const int pad = (64 - total % 64) % 64;
  FILE *f = fopen(name, "wb");
  if (!f) {
    perror(name);
    abort();
  }
  const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
  fwrite(magic, 1, 8, f);
  const uint16_t len = (uint16_t)(hl + pad + 1);
  const unsigned char lb[2] = {(unsigned char)(len & 0xff), (unsigned char)(len >> 8)};
  fwrite(lb, 1, 2, f);
  fwrite(header, 1, hl, f);
  for (int i = 0; i < pad; i++) fputc(' ', f);
  fputc('\n', f);
  const size_t n = (size_t)nx * ny * nz;
  if (data) fwrite(data, complex_values ? 8 : 4, n, f);
  fclose(f);
}

/* src/spsim.c:228-279 */
static void output_files(Diffraction_Pattern *pattern, Options *opts, int index) {
  CCD *det = opts->detector;
  if (opts->output_scatt_int || opts->output_intensities) write_npy("scattering_int", index, pattern->ints, 0, det, 0);
  if (opts->output_sf_vtk) {
    char buffer[1024];
    snprintf(buffer, sizeof(buffer), "scattering_factor-%05d.vtk", index);
    write_3D_array_to_vtk(pattern->ints, det->nx, det->ny, det->nz, buffer);
  }
  if (opts->output_noiseless_photons) write_npy("noiseless_photon_out", index, det->photons_per_pixel, 0, det, 0);
  if (opts->output_scattering_factors) write_npy("scattering_factors", index, pattern->F, 1, det, 0);
  if (opts->output_solid_angles) write_npy("solid_angles", index, det->solid_angle, 0, det, 0);
  if (opts->output_photons) write_npy("photon_out", index, det->photon_count, 0, det, 0);
  if (opts->output_count) write_npy("counts_out", index, det->real_output, 0, det, 1);
  if (opts->output_noiseless_count) write_npy("noiseless_counts_out", index, det->noiseless_output, 0, det, 1);
  if (opts->output_real_space || opts->output_realspace_histogram)
    fprintf(stderr, "spsim_b200: real-space outputs are not produced (outside the structure-factor path)\n");
}

int main(int argc, char **argv) {
  (void)argc;
  (void)argv;
  Options *opts = set_defaults();
  read_options_file("spsim.conf", opts);
  if (opts->random_seed < 0) opts->random_seed = (int)time(NULL);
  spsim_b200_set_noise_seed((unsigned long long)opts->random_seed);
  spsim_b200_set_formula_seed((unsigned long long)opts->random_seed);
  write_options_file("spsim.confout", opts);
  opts->detector->n_patterns = opts->n_patterns;
  Molecule *mol = get_molecule(opts);
  for (int n = 0; n < opts->n_patterns; n++) {
    Diffraction_Pattern *pattern = simulate_shot(mol, opts);
    output_files(pattern, opts, n);
    free_stuff(pattern, opts);
  }
  free_mol(mol);
  return 0;
}
