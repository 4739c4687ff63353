/*
 * Molecule input and output of the reference (src/molecule.c, src/spsim.c:83-97)
 * and its VTK writers (src/io.c): PDB reading with BIOMT expansion, random
 * molecules from a chemical formula, PDB writing, centring on the electron
 * centre of mass.  Host-side C; the arithmetic follows the reference's float
 * operations in the same order (built with -ffp-contract=off), so positions
 * come out bit-identical.
 *
 * Deliberate differences, each a memory-safety fix of an input the reference
 * mishandles:
 *  - a record whose element cannot be identified is skipped; the reference
 *    instead overwrites the previous atom's atomic number with 0 (and writes
 *    before its array when it is the first atom);
 *  - columns missing from a short ATOM line read as blanks (the reference
 *    reads whatever an earlier, longer line left in its buffer);
 *  - BIOMT records with an operator or row number below 1 are ignored and the
 *    operator table grows to any operator number (the reference indexes
 *    before its arrays, or past them after a jump of more than one doubling).
 */
#include <ctype.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/spsim.h"
#include "../../../include/spsim_b200.h"

/* Element symbols, two characters each, left-justified (Z = index + 1). */
static const char k_symbols[] =
    "H HELIBEB C N O F NE"
    "NAMGALSIP S CLARK CA"
    "SCTIV CRMNFECONICUZN"
    "GAGEASSEBRKRRBSRY ZR"
    "NBMOTCRURHPDAGCDINSN"
    "SBTEI XECSBALACEPRND"
    "PMSMEUGDTBDYHOERTMYB"
    "LUHFTAW REOSIRPTAUHG"
    "TLPBBIPOATRNFRRAACTH"
    "PAU NPPUAMCMBKCFESFM"
    "MDNOLRRFHA";
#define N_SYMBOLS ((int)(sizeof(k_symbols) - 1) / 2)

static int find_symbol(char a, char b) {
  for (int z = 0; z < N_SYMBOLS; z++)
    if (a == k_symbols[2 * z] && b == k_symbols[2 * z + 1]) return z + 1;
  return 0;
}

/* src/molecule.c:305-341: a two-character element field -> Z (0: unknown). */
static int z_from_symbol(char s0, char s1) {
  if (isalpha((unsigned char)s0)) {
    s0 = (char)toupper((unsigned char)s0);
  } else if (isalpha((unsigned char)s1)) {
    s0 = (char)toupper((unsigned char)s1);
    s1 = ' ';
  } else {
    return 0;
  }
  s1 = isalpha((unsigned char)s1) ? (char)toupper((unsigned char)s1) : ' ';
  int z = find_symbol(s0, s1);
  if (z) return z;
  z = find_symbol(s0, ' '); /* fall back to the first letter alone */
  if (z) return z;
  fprintf(stderr, "Could not find element for atom named '%c%c'\n", s0, ' ');
  return 0;
}

/* Characters [from, to) of a line as a number, like atof on that field. */
static double field(const char *line, size_t len, size_t from, size_t to) {
  char tmp[32];
  size_t n = 0;
  for (size_t i = from; i < to && i < len && n < sizeof(tmp) - 1; i++) tmp[n++] = line[i];
  tmp[n] = 0;
  return atof(tmp);
}

static char column(const char *line, size_t len, size_t i) {
  return i < len && line[i] != '\n' && line[i] != '\r' && line[i] != 0 ? line[i] : ' ';
}

/* src/molecule.c:65-297 */
Molecule *get_Molecule_from_pdb(char *filename) {
  FILE *fp = fopen(filename, "r");
  if (!fp) {
    perror("Error reading PDB\n");
    abort();
  }
  Molecule *res = (Molecule *)malloc(sizeof(Molecule));
  int cap = 1024;
  res->natoms = 0;
  res->atomic_number = (int *)malloc(sizeof(int) * cap);
  res->pos = (float *)malloc(3 * sizeof(float) * cap);
  res->delta_atoms = 0;
  int cap_symm = 1, num_symm = 0;
  float *rot = (float *)calloc(9 * cap_symm, sizeof(float));
  float *trans = (float *)calloc(3 * cap_symm, sizeof(float));
  int electrons = 0;
  char line[1024];
  while (fgets(line, sizeof(line), fp)) {
    const size_t len = strlen(line);
    if (len <= 1) continue;
    if (strncmp(line, "ATOM", 4) == 0 || strncmp(line, "HETATM", 6) == 0) {
      if (res->natoms >= cap) {
        cap *= 2;
        res->atomic_number = (int *)realloc(res->atomic_number, sizeof(int) * cap);
        res->pos = (float *)realloc(res->pos, 3 * sizeof(float) * cap);
      }
      /* coordinates: columns 31-38, 39-46, 47-54 (Angstrom) */
      const float x = (float)field(line, len, 30, 38);
      const float y = (float)field(line, len, 38, 46);
      const float z = (float)field(line, len, 46, 54);
      /* element: columns 77-78, right-justified */
      char e0 = column(line, len, 76), e1 = column(line, len, 77);
      if (isspace((unsigned char)e0)) {
        e0 = e1;
        e1 = ' ';
      }
      const int Z = z_from_symbol(e0, e1);
      if (!Z) {
        fprintf(stderr, "WARNING: Null atom at line '%.16s'. Skipping\n", line);
        continue;
      }
      res->pos[3 * res->natoms + 0] = x * 1e-10;
      res->pos[3 * res->natoms + 1] = y * 1e-10;
      res->pos[3 * res->natoms + 2] = z * 1e-10;
      res->atomic_number[res->natoms] = Z;
      electrons += Z;
      res->natoms++;
    } else if (strncmp(line, "REMARK 350   BIOMT", 18) == 0) {
      const int row = (int)field(line, len, 18, 19) - 1;
      const int op = (int)field(line, len, 20, 24) - 1;
      if (row < 0 || row > 2 || op < 0) continue;
      if (op >= cap_symm) {
        int ncap = cap_symm;
        while (op >= ncap) ncap *= 2;
        rot = (float *)realloc(rot, 9 * sizeof(float) * ncap);
        trans = (float *)realloc(trans, 3 * sizeof(float) * ncap);
        memset(rot + 9 * cap_symm, 0, 9 * sizeof(float) * (ncap - cap_symm));
        memset(trans + 3 * cap_symm, 0, 3 * sizeof(float) * (ncap - cap_symm));
        cap_symm = ncap;
      }
      if (op >= num_symm) num_symm = op + 1;
      rot[9 * op + 3 * row + 0] = (float)field(line, len, 24, 33);
      rot[9 * op + 3 * row + 1] = (float)field(line, len, 34, 43);
      rot[9 * op + 3 * row + 2] = (float)field(line, len, 44, 53);
      trans[3 * op + row] = (float)(field(line, len, 59, 68) * 1e-10);
    }
  }
  fprintf(stderr, "Read %d atoms with %d electrons\n", res->natoms, electrons);
  fprintf(stderr, "Read %d symmetry transformations\n", num_symm);
  fclose(fp);

  const int n = res->natoms;
  const int total = num_symm ? n * num_symm : n;
  res->atomic_number = (int *)realloc(res->atomic_number, sizeof(int) * (total > 0 ? total : 1));
  res->pos = (float *)realloc(res->pos, 3 * sizeof(float) * (total > 0 ? total : 1));
  /* Each operator k writes copy k in place, reading atom i's coordinates from
   * the first copy; operator 0 is meant to be the identity.  The three
   * components are written one after the other, so operator 0 sees its own
   * updated x when it computes y (src/molecule.c:264-285). */
  float *p = res->pos;
  for (int k = 0; k < num_symm; k++)
    for (int i = 0; i < n; i++) {
      const float *R = rot + 9 * k, *t = trans + 3 * k;
      float *dst = p + 3 * ((size_t)k * n + i);
      res->atomic_number[(size_t)k * n + i] = res->atomic_number[i];
      dst[0] = p[3 * i + 0] * R[0] + p[3 * i + 1] * R[1] + p[3 * i + 2] * R[2] + t[0];
      dst[1] = p[3 * i + 0] * R[3] + p[3 * i + 1] * R[4] + p[3 * i + 2] * R[5] + t[1];
      dst[2] = p[3 * i + 0] * R[6] + p[3 * i + 1] * R[7] + p[3 * i + 2] * R[8] + t[2];
    }
  if (num_symm > 0) {
    res->natoms = total;
    fprintf(stderr, "%d atoms with %d electrons after symmetrization\n", res->natoms, electrons * num_symm);
  }
  free(rot);
  free(trans);
  return res;
}

/* src/molecule.c:359-379 */
void write_pdb_from_mol(char *filename, Molecule *mol) {
  FILE *f = fopen(filename, "w");
  if (!f) {
    perror("Cannot open file\n");
    abort();
  }
  for (int i = 0; i < mol->natoms; i++) {
    const int z = mol->atomic_number[i];
    const char *sym = (z >= 1 && z <= N_SYMBOLS) ? &k_symbols[2 * (z - 1)] : "  ";
    fprintf(f, "ATOM  %5d  %.2s      A   1    %8.3f%8.3f%8.3f\n", i % 99999, sym, mol->pos[3 * i] * 1e10,
            mol->pos[3 * i + 1] * 1e10, mol->pos[3 * i + 2] * 1e10);
  }
  fprintf(f, "END\n");
  fclose(f);
}

/* Uniform [0,1) doubles for the random-molecule builder: splitmix64 keyed by
 * the noise seed (the reference draws from libspimage's p_drand48, which is
 * not available; positions are therefore reproducible here but not equal to
 * the reference's). */
static uint64_t g_formula_state = 0;
static double formula_u01(void) {
  uint64_t z = (g_formula_state += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  return (z >> 11) * (1.0 / 9007199254740992.0);
}

void spsim_b200_set_formula_seed(unsigned long long seed) { g_formula_state = seed; }

/* src/molecule.c:33-63: the formula's atoms, in formula order, uniform in a
 * ball of diameter box_dimension centred on the origin (BOX_SPHERICAL, by
 * rejection from the enclosing cube) or in [0, box_dimension)^3
 * (BOX_PARALLEL). */
Molecule *get_Molecule_from_formula(Chem_Formula *form, Options *opts) {
  Molecule *res = (Molecule *)malloc(sizeof(Molecule));
  res->natoms = 0;
  res->delta_atoms = 0;
  int total = 0;
  for (int i = 0; i < form->n_elements; i++) total += form->quantity[i];
  res->atomic_number = (int *)malloc(sizeof(int) * (total > 0 ? total : 1));
  res->pos = (float *)malloc(3 * sizeof(float) * (total > 0 ? total : 1));
  const float d = opts->box_dimension;
  for (int i = 0; i < form->n_elements; i++)
    for (int k = 0; k < form->quantity[i]; k++) {
      const int j = res->natoms++;
      res->atomic_number[j] = form->atomic_number[i];
      float *r = res->pos + 3 * j;
      if (opts->box_type == BOX_SPHERICAL) {
        float dist;
        do {
          dist = 0;
          for (int c = 0; c < 3; c++) {
            r[c] = (float)((formula_u01() - 0.5) * d);
            dist += r[c] * r[c];
          }
          dist = sqrtf(dist);
        } while (dist > d / 2.0);
      } else if (opts->box_type == BOX_PARALLEL) {
        for (int c = 0; c < 3; c++) r[c] = (float)(formula_u01() * d);
      }
    }
  return res;
}

/* src/molecule.c:440-464: origin moved to the centre of the electron density
 * (positions weighted by Z), float arithmetic. */
void origin_to_center_of_mass(Molecule *mol) {
  float com[3] = {0.f, 0.f, 0.f};
  int N = 0;
  for (int i = 0; i < mol->natoms; i++) {
    N += mol->atomic_number[i];
    com[0] += mol->pos[3 * i + 0] * mol->atomic_number[i];
    com[1] += mol->pos[3 * i + 1] * mol->atomic_number[i];
    com[2] += mol->pos[3 * i + 2] * mol->atomic_number[i];
  }
  com[0] /= N;
  com[1] /= N;
  com[2] /= N;
  for (int i = 0; i < mol->natoms; i++) {
    mol->pos[3 * i + 0] -= com[0];
    mol->pos[3 * i + 1] -= com[1];
    mol->pos[3 * i + 2] -= com[2];
  }
}

/* src/spsim.c:83-97; a formula molecule is also written to molout.pdb */
Molecule *get_molecule(Options *opts) {
  Molecule *mol = NULL;
  if (opts->input_type == CHEM_FORMULA) {
    mol = get_Molecule_from_formula(opts->chem_formula, opts);
    write_pdb_from_mol("molout.pdb", mol);
  } else if (opts->input_type == PDB) {
    mol = get_Molecule_from_pdb(opts->pdb_filename);
  } else {
    fprintf(stderr, "input_type not specified!\n");
    exit(0);
  }
  return mol;
}

/* ------------------------------------------------------------ VTK output */

static void write_vtk(const float *F, int nx, int ny, int nz, const char *filename) {
  FILE *f = fopen(filename, "w");
  if (!f) {
    perror("Bad file in write_vtk!");
    abort();
  }
  const long n = (long)nx * ny * nz;
  fprintf(f, "# vtk DataFile Version 2.0\n");
  fprintf(f, "Generated by image_util write_vtk()\n");
  fprintf(f, "ASCII\n");
  fprintf(f, "DATASET STRUCTURED_POINTS\n");
  fprintf(f, "DIMENSIONS %d %d %d\n", nx, ny, nz);
  fprintf(f, "ORIGIN 0 0 0\n");
  fprintf(f, "SPACING 1 1 1\n");
  fprintf(f, "POINT_DATA %ld\n", n);
  fprintf(f, "SCALARS intensity float 1\n");
  fprintf(f, "LOOKUP_TABLE default\n");
  fprintf(f, "%6e", n > 0 ? F[0] : 0.0f);
  for (long i = 1; i < n; i++) fprintf(f, " %e", F[i]);
  fprintf(f, "\n");
  fclose(f);
}

/* src/io.c:29-57 */
void write_2D_array_to_vtk(float *F, int nx, int ny, char *filename) { write_vtk(F, nx, ny, 1, filename); }

/* src/io.c:60-89 */
void write_3D_array_to_vtk(float *F, int nx, int ny, int nz, char *filename) { write_vtk(F, nx, ny, nz, filename); }
