/*
 * The spsim command-line program (src/spsim.c:374-415) on this library: read
 * spsim.conf, echo the options to spsim.confout, build the molecule (PDB or
 * chemical formula), and for each of n_patterns shots run simulate_shot and
 * write the requested outputs.
 *
 * Outputs: output_files (the library's, spsim's src/spsim.c:228-279) writes
 * each requested array as <name>-NNNNN.cxi, an HDF5 file in the CXI image
 * layout, under the base names spsim uses, and scattering_factor-NNNNN.vtk on
 * request.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../../include/spsim.h"
#include "../../../include/spsim_b200.h"

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
