/*
 * spsim.conf handling: set_defaults, read_options_file, write_options_file
 * with the semantics of src/config.c:30-642.
 *
 * The reference parses spsim.conf with a vendored libconfig; this file has its
 * own small parser for the same syntax, as strict as that libconfig version:
 * settings "name = value;" or "name : value;" each ending in ';', groups { },
 * lists ( ), arrays [ ], strings with escapes and concatenation, decimal and
 * 0x integers, floats with a '.' and at least one fraction digit, booleans,
 * and #, // and block comments.  It keeps the lookup rules spsim depends on:
 *   - a float key given as an integer literal reads as 0.0 (and vice versa),
 *     the quirk documented in doc/UserManual.tex:91-93;
 *   - paths use ':' '.' or '/' as separators ("chemical_formula/atom6").
 * write_options_file reproduces libconfig's writer layout byte for byte:
 * "name = value;" per line, floats as %e, groups as "name : \n{\n  ...\n};".
 */
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/spsim.h"

/* ---------------------------------------------------------------- values */

enum { V_NONE = 0, V_GROUP, V_INT, V_FLOAT, V_STRING, V_BOOL, V_LIST };

typedef struct cfg_node {
  char *name;
  int type;
  long ival;
  double fval;
  char *sval;
  struct cfg_node **kids;
  int nkids;
} cfg_node;

static cfg_node *node_new(const char *name, int type) {
  cfg_node *n = (cfg_node *)calloc(1, sizeof(cfg_node));
  n->name = name ? strdup(name) : NULL;
  n->type = type;
  return n;
}

static void node_free(cfg_node *n) {
  if (!n) return;
  for (int i = 0; i < n->nkids; i++) node_free(n->kids[i]);
  free(n->kids);
  free(n->name);
  free(n->sval);
  free(n);
}

static void node_add(cfg_node *parent, cfg_node *kid) {
  parent->kids = (cfg_node **)realloc(parent->kids, sizeof(cfg_node *) * (parent->nkids + 1));
  parent->kids[parent->nkids++] = kid;
}

/* ---------------------------------------------------------------- lexer */

typedef struct {
  const char *s;
  size_t i, n;
  int line;
  char err[256];
} lexer;

static void skip_ws(lexer *L) {
  for (;;) {
    while (L->i < L->n && isspace((unsigned char)L->s[L->i])) {
      if (L->s[L->i] == '\n') L->line++;
      L->i++;
    }
    if (L->i >= L->n) return;
    if (L->s[L->i] == '#' || (L->s[L->i] == '/' && L->i + 1 < L->n && L->s[L->i + 1] == '/')) {
      while (L->i < L->n && L->s[L->i] != '\n') L->i++;
      continue;
    }
    if (L->s[L->i] == '/' && L->i + 1 < L->n && L->s[L->i + 1] == '*') {
      L->i += 2;
      while (L->i + 1 < L->n && !(L->s[L->i] == '*' && L->s[L->i + 1] == '/')) {
        if (L->s[L->i] == '\n') L->line++;
        L->i++;
      }
      L->i += 2;
      continue;
    }
    return;
  }
}

static int peek(lexer *L) {
  skip_ws(L);
  return L->i < L->n ? (unsigned char)L->s[L->i] : -1;
}

static int parse_name(lexer *L, char *buf, size_t cap) {
  skip_ws(L);
  size_t k = 0;
  if (L->i >= L->n || !(isalpha((unsigned char)L->s[L->i]) || L->s[L->i] == '*')) return 0;
  while (L->i < L->n && (isalnum((unsigned char)L->s[L->i]) || strchr("-_*", L->s[L->i]))) {
    if (k + 1 < cap) buf[k++] = L->s[L->i];
    L->i++;
  }
  buf[k] = 0;
  return 1;
}

static int parse_value(lexer *L, cfg_node *n);
static int parse_settings(lexer *L, cfg_node *group, int close);

static int parse_string(lexer *L, cfg_node *n) {
  size_t cap = 64, k = 0;
  char *out = (char *)malloc(cap);
  while (peek(L) == '"') {
    L->i++;
    while (L->i < L->n && L->s[L->i] != '"') {
      char c = L->s[L->i++];
      if (c == '\\' && L->i < L->n) {
        char e = L->s[L->i++];
        c = e == 'n' ? '\n' : e == 't' ? '\t' : e == 'r' ? '\r' : e == 'f' ? '\f' : e;
      }
      if (k + 2 > cap) out = (char *)realloc(out, cap *= 2);
      out[k++] = c;
    }
    if (L->i >= L->n) {
      free(out);
      snprintf(L->err, sizeof(L->err), "unterminated string");
      return 0;
    }
    L->i++; /* closing quote; adjacent strings concatenate */
  }
  out[k] = 0;
  n->type = V_STRING;
  n->sval = out;
  return 1;
}

/* Numbers as spsim's libconfig scans them: a float needs a '.' followed by at
 * least one digit ("1.5e-6", ".5"; not "5." or "1e5"), an integer is decimal
 * or 0x-hexadecimal; anything else is a syntax error. */
static int parse_number(lexer *L, cfg_node *n) {
  size_t st = L->i, k = L->i;
  if (k < L->n && (L->s[k] == '+' || L->s[k] == '-')) k++;
  if (k + 1 < L->n && L->s[k] == '0' && (L->s[k + 1] == 'x' || L->s[k + 1] == 'X')) {
    size_t h = k + 2;
    while (h < L->n && isxdigit((unsigned char)L->s[h])) h++;
    if (h == k + 2) goto bad;
    char tmp[64];
    size_t len = h - st < 63 ? h - st : 63;
    memcpy(tmp, L->s + st, len);
    tmp[len] = 0;
    n->type = V_INT;
    n->ival = (long)strtoul(tmp, NULL, 16);
    L->i = h;
    return 1;
  }
  size_t d0 = k;
  while (k < L->n && isdigit((unsigned char)L->s[k])) k++;
  size_t nint = k - d0;
  int is_float = 0;
  if (k < L->n && L->s[k] == '.') {
    size_t f0 = ++k;
    while (k < L->n && isdigit((unsigned char)L->s[k])) k++;
    if (k == f0) goto bad; /* "5." */
    is_float = 1;
    if (k < L->n && (L->s[k] == 'e' || L->s[k] == 'E')) {
      size_t e = k + 1;
      if (e < L->n && (L->s[e] == '+' || L->s[e] == '-')) e++;
      size_t e0 = e;
      while (e < L->n && isdigit((unsigned char)L->s[e])) e++;
      if (e == e0) goto bad;
      k = e;
    }
  } else if (nint == 0) {
    goto bad;
  }
  {
    char tmp[128];
    size_t len = k - st < 127 ? k - st : 127;
    memcpy(tmp, L->s + st, len);
    tmp[len] = 0;
    if (is_float) {
      n->type = V_FLOAT;
      n->fval = atof(tmp);
    } else {
      n->type = V_INT;
      n->ival = atoi(tmp);
    }
    L->i = k;
    return 1;
  }
bad:
  snprintf(L->err, sizeof(L->err), "syntax error");
  return 0;
}

static int parse_value(lexer *L, cfg_node *n) {
  int c = peek(L);
  if (c == '"') return parse_string(L, n);
  if (c == '{') {
    L->i++;
    n->type = V_GROUP;
    return parse_settings(L, n, '}');
  }
  if (c == '(' || c == '[') {
    int close = c == '(' ? ')' : ']';
    L->i++;
    n->type = V_LIST;
    if (peek(L) == close) {
      L->i++;
      return 1;
    }
    for (;;) {
      cfg_node *k = node_new(NULL, V_NONE);
      node_add(n, k);
      if (!parse_value(L, k)) return 0;
      int d = peek(L);
      if (d == ',') {
        L->i++;
        continue;
      }
      if (d == close) {
        L->i++;
        return 1;
      }
      snprintf(L->err, sizeof(L->err), "syntax error in list");
      return 0;
    }
  }
  if (c == '-' || c == '+' || c == '.' || (c >= '0' && c <= '9')) return parse_number(L, n);
  char word[64];
  if (parse_name(L, word, sizeof(word))) {
    for (char *p = word; *p; p++) *p = (char)tolower((unsigned char)*p);
    if (!strcmp(word, "true") || !strcmp(word, "false")) {
      n->type = V_BOOL;
      n->ival = word[0] == 't';
      return 1;
    }
  }
  snprintf(L->err, sizeof(L->err), "syntax error");
  return 0;
}

static int parse_settings(lexer *L, cfg_node *group, int close) {
  for (;;) {
    int c = peek(L);
    if (c == -1) {
      if (close) {
        snprintf(L->err, sizeof(L->err), "unexpected end of file");
        return 0;
      }
      return 1;
    }
    if (close && c == close) {
      L->i++;
      return 1;
    }
    char name[256];
    if (!parse_name(L, name, sizeof(name))) {
      snprintf(L->err, sizeof(L->err), "syntax error");
      return 0;
    }
    c = peek(L);
    if (c != '=' && c != ':') {
      snprintf(L->err, sizeof(L->err), "syntax error");
      return 0;
    }
    L->i++;
    cfg_node *k = node_new(name, V_NONE);
    node_add(group, k);
    if (!parse_value(L, k)) return 0;
    if (peek(L) != ';') { /* every setting, groups included, ends with ';' */
      snprintf(L->err, sizeof(L->err), "syntax error");
      return 0;
    }
    L->i++;
  }
}

static cfg_node *parse_file(const char *filename, int *err_line, char *err, size_t errcap) {
  FILE *f = fopen(filename, "rb");
  if (!f) {
    *err_line = 0;
    snprintf(err, errcap, "file I/O error");
    return NULL;
  }
  fseek(f, 0, SEEK_END);
  long len = ftell(f);
  fseek(f, 0, SEEK_SET);
  char *buf = (char *)malloc(len + 1);
  size_t got = fread(buf, 1, len, f);
  buf[got] = 0;
  fclose(f);
  lexer L = {buf, 0, got, 1, {0}};
  cfg_node *root = node_new(NULL, V_GROUP);
  int ok = parse_settings(&L, root, 0);
  free(buf);
  if (!ok) {
    *err_line = L.line;
    snprintf(err, errcap, "%s", L.err);
    node_free(root);
    return NULL;
  }
  return root;
}

/* ---------------------------------------------------------------- lookup */

static cfg_node *lookup(cfg_node *root, const char *path) {
  cfg_node *cur = root;
  const char *p = path;
  while (cur && *p) {
    while (*p && strchr(":./", *p)) p++;
    if (!*p) break;
    const char *q = p;
    while (*q && !strchr(":./", *q)) q++;
    size_t len = (size_t)(q - p);
    cfg_node *found = NULL;
    if (cur->type == V_GROUP)
      for (int i = 0; i < cur->nkids; i++)
        if (cur->kids[i]->name && strlen(cur->kids[i]->name) == len && !strncmp(cur->kids[i]->name, p, len)) {
          found = cur->kids[i];
          break;
        }
    cur = found;
    p = q;
  }
  return cur == root ? NULL : cur;
}

static double lookup_float(cfg_node *root, const char *path) {
  cfg_node *n = lookup(root, path);
  return (n && n->type == V_FLOAT) ? n->fval : 0.0;
}

static long lookup_int(cfg_node *root, const char *path) {
  cfg_node *n = lookup(root, path);
  return (n && n->type == V_INT) ? n->ival : 0;
}

static const char *lookup_string(cfg_node *root, const char *path) {
  cfg_node *n = lookup(root, path);
  return (n && n->type == V_STRING) ? n->sval : NULL;
}

/* ---------------------------------------------------------------- spsim */

/* src/config.c:30-87 */
Options *set_defaults(void) {
  Options *opt = (Options *)calloc(1, sizeof(Options));
  opt->chem_formula = (Chem_Formula *)calloc(1, sizeof(Chem_Formula));
  opt->experiment = (Experiment *)calloc(1, sizeof(Experiment));
  opt->experiment->polarization = POLARIZATION_IGNORE;
  opt->detector = (CCD *)calloc(1, sizeof(CCD));
  opt->detector->binning_x = 1;
  opt->detector->binning_y = 1;
  opt->detector->binning_z = 1;
  opt->box_type = BOX_SPHERICAL;
  opt->box_dimension = 1e-9f;
  opt->n_patterns = 1;
  opt->vectorize = 1;
  opt->use_cuda = 1;
  opt->crystal_size[0] = opt->crystal_size[1] = opt->crystal_size[2] = 1;
  opt->crystal_cell[3] = opt->crystal_cell[4] = opt->crystal_cell[5] = 90;
  opt->wavelength_samples = 5;
  opt->random_seed = -1;
  opt->output_noiseless_photons = 1;
  opt->output_photons = 1;
  opt->verbosity_level = 1;
  return opt;
}

#define GETF(key, dst) \
  if (lookup(root, key)) (dst) = (float)lookup_float(root, key)
#define GETI(key, dst) \
  if (lookup(root, key)) (dst) = (int)lookup_int(root, key)

/* src/config.c:89-427 */
void read_options_file(char *filename, Options *res) {
  int line = 0;
  char err[256];
  cfg_node *root = parse_file(filename, &line, err, sizeof(err));
  if (!root) {
    fprintf(stderr, "Error parsing %s on line %d:\n,%s\n", filename, line, err);
    exit(1);
  }
  const char *tmp;
  if ((tmp = lookup_string(root, "box_type"))) {
    if (!strcmp(tmp, "spherical")) res->box_type = BOX_SPHERICAL;
    else if (!strcmp(tmp, "parallelepipedic")) res->box_type = BOX_PARALLEL;
  }
  GETF("box_dimension", res->box_dimension);
  if ((tmp = lookup_string(root, "input_type"))) {
    if (!strcmp(tmp, "chemical_formula")) {
      res->input_type = CHEM_FORMULA;
      res->chem_formula->n_elements = 0;
      for (int i = 0; i < 100; i++) {
        char key[64];
        snprintf(key, sizeof(key), "chemical_formula/atom%d", i);
        long q = lookup_int(root, key);
        if (q) {
          Chem_Formula *cf = res->chem_formula;
          cf->n_elements++;
          cf->atomic_number = (int *)realloc(cf->atomic_number, sizeof(int) * cf->n_elements);
          cf->atomic_number[cf->n_elements - 1] = i;
          cf->quantity = (int *)realloc(cf->quantity, sizeof(int) * cf->n_elements);
          cf->quantity[cf->n_elements - 1] = (int)q;
        }
      }
    } else if (!strcmp(tmp, "pdb")) {
      res->input_type = PDB;
      if (lookup(root, "pdb_filename") && lookup_string(root, "pdb_filename")) {
        snprintf(res->pdb_filename, sizeof(res->pdb_filename), "%s", lookup_string(root, "pdb_filename"));
      } else {
        fprintf(stderr, "Error: You need to specify \"pdb_filename\" when you use input_type = \"pdb\"\n");
        exit(0);
      }
    }
  }
  CCD *d = res->detector;
  Experiment *e = res->experiment;
  GETF("detector_distance", d->distance);
  GETF("detector_center_x", d->center_x);
  GETF("detector_center_y", d->center_y);
  GETF("detector_center_z", d->center_z);
  GETF("detector_width", d->width);
  GETF("detector_height", d->height);
  GETF("detector_depth", d->depth);
  GETF("detector_pixel_width", d->pixel_width);
  GETF("detector_pixel_height", d->pixel_height);
  GETF("detector_pixel_depth", d->pixel_depth);
  GETF("detector_quantum_efficiency", d->quantum_efficiency);
  GETF("detector_electron_hole_production_energy", d->electron_hole_production_energy);
  GETF("detector_readout_noise", d->readout_noise);
  GETF("detector_dark_current", d->dark_current);
  GETF("detector_linear_full_well", d->linear_full_well);
  if (lookup(root, "detector_binning")) {
    d->binning_x = (int)lookup_int(root, "detector_binning");
    d->binning_y = (int)lookup_int(root, "detector_binning");
    d->binning_z = 1;
  }
  GETI("detector_binning_x", d->binning_x);
  GETI("detector_binning_y", d->binning_y);
  GETI("detector_binning_z", d->binning_z);
  GETF("detector_maximum_value", d->maximum_value);
  GETF("experiment_wavelength", e->wavelength);
  GETF("experiment_photon_energy", e->photon_energy);
  GETF("experiment_bandwidth", e->bandwidth);
  GETF("experiment_exposure_time", e->exposure_time);
  GETF("experiment_beam_intensity", e->beam_intensity);
  GETF("experiment_beam_center_x", e->beam_center_x);
  GETF("experiment_beam_center_y", e->beam_center_y);
  GETF("experiment_beam_fwhm", e->beam_fwhm);
  GETF("experiment_beam_energy", e->beam_energy);
  GETF("experiment_focal_diameter", e->focal_diameter);
  if ((tmp = lookup_string(root, "experiment_polarization"))) {
    if (!strcmp(tmp, "ignore")) e->polarization = POLARIZATION_IGNORE;
    else if (!strcmp(tmp, "horizontal")) e->polarization = POLARIZATION_HORIZONTAL;
    else if (!strcmp(tmp, "vertical")) e->polarization = POLARIZATION_VERTICAL;
    else if (!strcmp(tmp, "unpolarized")) e->polarization = POLARIZATION_UNPOLARIZED;
    else fprintf(stderr, "Warning: polarization is set to an undefined option!\n");
  }
  if ((tmp = lookup_string(root, "precalculated_sf"))) snprintf(res->sf_filename, sizeof(res->sf_filename), "%s", tmp);
  if ((tmp = lookup_string(root, "hkl_grid")))
    snprintf(res->hkl_grid_filename, sizeof(res->hkl_grid_filename), "%s", tmp);
  GETI("detector_spherical", d->spherical);
  GETF("detector_gaussian_blurring", d->gaussian_blurring);
  GETF("real_space_blurring", d->real_space_blurring);
  GETI("use_fft_for_sf", res->use_fft_for_sf);
  GETI("use_nfft_for_sf", res->use_nfft_for_sf);
  GETF("b_factor", res->b_factor);
  GETI("origin_to_com", res->origin_to_com);
  GETF("phi", res->euler_orientation[0]);
  GETF("theta", res->euler_orientation[1]);
  GETF("psi", res->euler_orientation[2]);
  GETI("random_orientation", res->random_orientation);
  GETI("number_of_patterns", res->n_patterns);
  GETI("vectorize", res->vectorize);
  GETI("delta_atoms", res->delta_atoms);
  GETI("fast_exit", res->fast_exit);
  GETI("crystal_size_a", res->crystal_size[0]);
  GETI("crystal_size_b", res->crystal_size[1]);
  GETI("crystal_size_c", res->crystal_size[2]);
  GETF("crystal_cell_a", res->crystal_cell[0]);
  GETF("crystal_cell_b", res->crystal_cell[1]);
  GETF("crystal_cell_c", res->crystal_cell[2]);
  GETF("crystal_cell_alpha", res->crystal_cell[3]);
  GETF("crystal_cell_beta", res->crystal_cell[4]);
  GETF("crystal_cell_gamma", res->crystal_cell[5]);
  GETI("use_cuda", res->use_cuda);
  GETI("wavelength_samples", res->wavelength_samples);
  GETI("random_seed", res->random_seed);
  GETI("output_noiseless_photons", res->output_noiseless_photons);
  GETI("output_photons", res->output_photons);
  GETI("output_noiseless_count", res->output_noiseless_count);
  GETI("output_count", res->output_count);
  GETI("output_scattering_factors", res->output_scattering_factors);
  GETI("output_solid_angles", res->output_solid_angles);
  GETI("output_real_space", res->output_real_space);
  /* derived values, src/config.c:386-423 */
  d->nx = (int)rint(d->width / d->pixel_width);
  d->ny = (int)rint(d->height / d->pixel_height);
  if (d->pixel_depth) {
    d->nz = (int)rint(d->depth / d->pixel_depth);
  } else {
    d->nz = 1;
    d->binning_z = 1;
  }
  if (d->nz > 1 && e->polarization != POLARIZATION_IGNORE) {
    fprintf(stderr,
            "Warning: For a 3D detector polarization effects (Thomson correction) have to be neglected "
            "(polarization = \"ignore\")!\n");
    e->polarization = POLARIZATION_IGNORE;
  }
  if (e->photon_energy) {
    float lambda = (float)(1.240e-6 / e->photon_energy);
    if (e->wavelength) {
      if ((lambda - e->wavelength) / (lambda + e->wavelength) > 0.01)
        fprintf(stderr, "Warning: experiment_wavelength does not agree with experiment_photon_energy!\n");
    } else {
      e->wavelength = lambda;
    }
  } else {
    if (e->wavelength) {
      float eV = (float)(1.240e-6 / e->wavelength);
      e->photon_energy = eV;
    } else {
      fprintf(stderr, "Warning: you need to specify the experiment_wavelength!\n");
    }
  }
  if (!e->beam_intensity) {
    if (e->focal_diameter && e->beam_energy) {
      float eV = (float)(1.240e-6 / e->wavelength);
      float nphotons = (float)(e->beam_energy * 6.24150974e18 / eV);
      float area = e->focal_diameter * e->focal_diameter;
      e->beam_intensity = nphotons / area;
    }
  }
  GETI("verbosity_level", res->verbosity_level);
  node_free(root);
}

/* ---------------------------------------------------------------- writer */

static void w_float(FILE *f, const char *k, double v) { fprintf(f, "%s = %e;\n", k, v); }
static void w_int(FILE *f, const char *k, long v) { fprintf(f, "%s = %ld;\n", k, v); }
static void w_str(FILE *f, const char *k, const char *v) {
  fprintf(f, "%s = \"", k);
  for (const char *p = v; *p; p++) {
    switch (*p) {
      case '"': fputs("\\\"", f); break;
      case '\\': fputs("\\\\", f); break;
      case '\n': fputs("\\n", f); break;
      case '\r': fputs("\\r", f); break;
      case '\f': fputs("\\f", f); break;
      case '\t': fputs("\\t", f); break;
      default: fputc(*p, f);
    }
  }
  fputs("\";\n", f);
}

/* src/config.c:433-642 */
void write_options_file(char *filename, Options *res) {
  FILE *f = fopen(filename, "w");
  if (!f) return;
  CCD *d = res->detector;
  Experiment *e = res->experiment;
  if (res->input_type == CHEM_FORMULA) {
    w_str(f, "input_type", "chemical_formula");
    fprintf(f, "chemical_formula : \n{\n");
    for (int i = 0; i < res->chem_formula->n_elements; i++)
      fprintf(f, "  atom%d = %d;\n", res->chem_formula->atomic_number[i], res->chem_formula->quantity[i]);
    fprintf(f, "};\n");
  } else if (res->input_type == PDB) {
    w_str(f, "input_type", "pdb");
    w_str(f, "pdb_filename", res->pdb_filename);
  } else if (!res->input_type) {
    w_str(f, "input_type", "none");
  }
  if (res->box_type == BOX_SPHERICAL) w_str(f, "box_type", "spherical");
  else if (res->box_type == BOX_PARALLEL) w_str(f, "box_type", "parallelepipedic");
  w_float(f, "detector_distance", d->distance);
  w_float(f, "detector_width", d->width);
  w_float(f, "detector_height", d->height);
  w_float(f, "detector_depth", d->depth);
  w_float(f, "detector_center_x", d->center_x);
  w_float(f, "detector_center_y", d->center_y);
  w_float(f, "detector_center_z", d->center_z);
  w_float(f, "detector_pixel_width", d->pixel_width);
  w_float(f, "detector_pixel_height", d->pixel_height);
  w_float(f, "detector_pixel_depth", d->pixel_depth);
  w_float(f, "detector_quantum_efficiency", d->quantum_efficiency);
  w_float(f, "detector_electron_hole_production_energy", d->electron_hole_production_energy);
  w_float(f, "detector_readout_noise", d->readout_noise);
  w_float(f, "detector_dark_current", d->dark_current);
  w_float(f, "detector_linear_full_well", d->linear_full_well);
  w_int(f, "detector_binning_x", d->binning_x);
  w_int(f, "detector_binning_y", d->binning_y);
  w_int(f, "detector_binning_z", d->binning_z);
  w_float(f, "detector_maximum_value", d->maximum_value);
  w_float(f, "experiment_wavelength", e->wavelength);
  w_float(f, "experiment_bandwidth", e->bandwidth);
  w_float(f, "experiment_exposure_time", e->exposure_time);
  w_float(f, "experiment_beam_intensity", e->beam_intensity);
  w_float(f, "experiment_beam_center_x", e->beam_center_x);
  w_float(f, "experiment_beam_center_y", e->beam_center_y);
  w_float(f, "experiment_beam_fwhm", e->beam_fwhm);
  w_float(f, "experiment_beam_energy", e->beam_energy);
  w_float(f, "experiment_photon_energy", e->photon_energy);
  w_float(f, "experiment_focal_diameter", e->focal_diameter);
  w_float(f, "box_dimension", res->box_dimension);
  w_int(f, "detector_spherical", d->spherical);
  w_float(f, "detector_gaussian_blurring", d->gaussian_blurring);
  /* the reference writes this key misspelt (src/config.c:547) */
  w_float(f, "real_sapce_blurring", d->real_space_blurring);
  w_int(f, "use_fft_for_sf", res->use_fft_for_sf);
  w_int(f, "use_nfft_for_sf", res->use_nfft_for_sf);
  w_float(f, "b_factor", res->b_factor);
  w_int(f, "origin_to_com", res->origin_to_com);
  w_float(f, "phi", res->euler_orientation[0]);
  w_float(f, "theta", res->euler_orientation[1]);
  w_float(f, "psi", res->euler_orientation[2]);
  w_int(f, "random_orientation", res->random_orientation);
  w_int(f, "number_of_patterns", res->n_patterns);
  w_int(f, "vectorize", res->vectorize);
  w_int(f, "delta_atoms", res->delta_atoms);
  w_int(f, "fast_exit", res->fast_exit);
  w_int(f, "crystal_size_a", res->crystal_size[0]);
  w_int(f, "crystal_size_b", res->crystal_size[1]);
  w_int(f, "crystal_size_c", res->crystal_size[2]);
  w_float(f, "crystal_cell_a", res->crystal_cell[0]);
  w_float(f, "crystal_cell_b", res->crystal_cell[1]);
  w_float(f, "crystal_cell_c", res->crystal_cell[2]);
  w_float(f, "crystal_cell_alpha", res->crystal_cell[3]);
  w_float(f, "crystal_cell_beta", res->crystal_cell[4]);
  w_float(f, "crystal_cell_gamma", res->crystal_cell[5]);
  if (e->polarization == POLARIZATION_IGNORE) w_str(f, "experiment_polarization", "ignore");
  else if (e->polarization == POLARIZATION_VERTICAL) w_str(f, "experiment_polarization", "vertical");
  else if (e->polarization == POLARIZATION_HORIZONTAL) w_str(f, "experiment_polarization", "horizontal");
  else if (e->polarization == POLARIZATION_UNPOLARIZED) w_str(f, "experiment_polarization", "unpolarized");
  w_int(f, "use_cuda", res->use_cuda);
  w_int(f, "wavelength_samples", res->wavelength_samples);
  w_int(f, "random_seed", res->random_seed);
  w_int(f, "output_photons", res->output_photons);
  w_int(f, "output_noiseless_photons", res->output_noiseless_photons);
  w_int(f, "output_count", res->output_count);
  w_int(f, "output_noiseless_count", res->output_noiseless_count);
  w_int(f, "output_solid_angles", res->output_solid_angles);
  w_int(f, "output_scattering_factors", res->output_scattering_factors);
  w_int(f, "output_real_space", res->output_real_space);
  w_int(f, "verbosity_level", res->verbosity_level);
  if (res->sf_filename[0]) w_str(f, "precalculated_sf", res->sf_filename);
  fclose(f);
}
