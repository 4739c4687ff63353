/*
 * CXI output of the spsim program (src/spsim.c:146-279): output_array,
 * output_carray and output_files write each requested array as
 * <basename>-NNNNN.cxi.  spsim writes them through libspimage's
 * sp_image_write, which needs libspimage and HDF5; neither is in this build,
 * so this file writes the HDF5 container itself, from the HDF5 file format
 * specification (version 0 superblock, version 1 object headers, groups as
 * symbol tables: a version 1 B-tree leaf, one symbol table node and a local
 * heap per group), with contiguous little-endian datasets.  The layout is the
 * CXI image layout:
 *
 *   /cxi_version                               int32 scalar, 150
 *   /entry_1/image_1/data                      float32 (or complex {r, i}) [nz,] ny, nx
 *   /entry_1/image_1/mask                      int32, same shape, 1 (spsim marks every pixel valid)
 *   /entry_1/image_1/detector_1/distance       float64, metres
 *   /entry_1/image_1/detector_1/x_pixel_size   float64, metres (pixel width x binning)
 *   /entry_1/image_1/detector_1/y_pixel_size   float64, metres
 *   /entry_1/image_1/source_1/wavelength       float64, metres
 *   /entry_1/image_1/orientation               float64 3 x 3, when the shot has a rotation
 *
 * (the image metadata make_image sets, src/spsim.c:154-173).  libspimage's
 * own CXI writer is not available here, so parity with its exact layout is
 * unpinned.  Binned arrays (counts_out, noiseless_counts_out) are written with
 * their binned shape; spsim's make_image sizes every image by the unbinned
 * detector and reads past the end of a binned array.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/spsim.h"

/* ---------------------------------------------------------------- byte buffer */

typedef struct {
  unsigned char *p;
  size_t n, cap;
} Buf;

static void buf_reserve(Buf *b, size_t n) {
  if (b->n + n <= b->cap) return;
  size_t cap = b->cap ? b->cap : 4096;
  while (cap < b->n + n) cap *= 2;
  unsigned char *q = (unsigned char *)realloc(b->p, cap);
  if (!q) {
    fprintf(stderr, "cxi: out of memory\n");
    abort();
  }
  memset(q + b->cap, 0, cap - b->cap);
  b->p = q;
  b->cap = cap;
}
static size_t buf_zeros(Buf *b, size_t n) {  // appends n zero bytes, returns their offset
  buf_reserve(b, n);
  const size_t at = b->n;
  b->n += n;
  return at;
}
static void put_le(Buf *b, size_t at, uint64_t v, int bytes) {
  for (int i = 0; i < bytes; i++) b->p[at + i] = (unsigned char)(v >> (8 * i));
}
static size_t pad8(size_t n) { return (n + 7) & ~(size_t)7; }

#define UNDEF_ADDR 0xffffffffffffffffULL
#define HEAP_FREE_NULL 1ULL  /* the local heap's "no free block" offset */
#define LEAF_K 4             /* group leaf node K: 2K entries per symbol table node */
#define INTERNAL_K 16        /* group internal node K: 2K children per B-tree node */

/* ---------------------------------------------------------------- object tree */

enum { T_F32, T_F64, T_I32, T_C64 };

typedef struct Node {
  const char *name;
  int is_group;
  /* group */
  struct Node *child[2 * LEAF_K];
  int nchild;
  /* dataset */
  int type, rank;
  uint64_t dims[4];
  const void *data;
  /* written address of the object header */
  uint64_t addr;
} Node;

static void add_child(Node *g, Node *c) {
  if (g->nchild >= 2 * LEAF_K) {
    fprintf(stderr, "cxi: group %s has more than %d members\n", g->name, 2 * LEAF_K);
    abort();
  }
  g->child[g->nchild++] = c;
}

static size_t type_size(int t) { return t == T_F64 || t == T_C64 ? 8 : 4; }

/* datatype message body (HDF5 datatype message, class version 1) */
static size_t datatype_bytes(int t) {
  if (t == T_I32) return 8 + 4;
  if (t == T_C64) return 8 + 2 * (8 + 4 + 4 + 4 + 4 + 16 + 20);
  return 8 + 12;
}
static void write_float_type(Buf *b, size_t at, int dbl) {
  b->p[at] = 0x11;                 /* version 1, class 1: floating point */
  b->p[at + 1] = 0x20;             /* little-endian, mantissa normalisation: implied msb */
  b->p[at + 2] = dbl ? 63 : 31;    /* sign bit position */
  b->p[at + 3] = 0;
  put_le(b, at + 4, dbl ? 8 : 4, 4);
  put_le(b, at + 8, 0, 2);                     /* bit offset */
  put_le(b, at + 10, dbl ? 64 : 32, 2);        /* bit precision */
  b->p[at + 12] = dbl ? 52 : 23;               /* exponent location */
  b->p[at + 13] = dbl ? 11 : 8;                /* exponent size */
  b->p[at + 14] = 0;                           /* mantissa location */
  b->p[at + 15] = dbl ? 52 : 23;               /* mantissa size */
  put_le(b, at + 16, dbl ? 1023 : 127, 4);     /* exponent bias */
}
static void write_datatype(Buf *b, size_t at, int t) {
  if (t == T_F32 || t == T_F64) {
    write_float_type(b, at, t == T_F64);
  } else if (t == T_I32) {
    b->p[at] = 0x10;   /* version 1, class 0: fixed point */
    b->p[at + 1] = 0x08; /* little-endian, signed */
    put_le(b, at + 4, 4, 4);
    put_le(b, at + 8, 0, 2);
    put_le(b, at + 10, 32, 2);
  } else {             /* complex as a compound of two float32 members, r and i */
    b->p[at] = 0x16;   /* version 1, class 6: compound */
    put_le(b, at + 1, 2, 2);  /* two members */
    put_le(b, at + 4, 8, 4);
    size_t m = at + 8;
    const char *names[2] = {"r", "i"};
    for (int k = 0; k < 2; k++) {
      memcpy(b->p + m, names[k], 1);  /* null-terminated, padded to 8 */
      put_le(b, m + 8, 4 * k, 4);     /* byte offset */
      b->p[m + 12] = 0;               /* dimensionality: scalar member */
      write_float_type(b, m + 40, 0);
      m += 60;
    }
  }
}

/* ---------------------------------------------------------------- writers */

/* one object-header message: returns the offset of its body */
static size_t message(Buf *b, size_t *cursor, int type, size_t body) {
  put_le(b, *cursor, (uint64_t)type, 2);
  put_le(b, *cursor + 2, (uint64_t)pad8(body), 2);
  const size_t at = *cursor + 8;
  *cursor = at + pad8(body);
  return at;
}

/* version 1 object header with `nmsg` messages of the given padded sizes */
static size_t object_header(Buf *b, int nmsg, size_t msg_bytes) {
  const size_t at = buf_zeros(b, 16 + msg_bytes);
  b->p[at] = 1;                          /* version */
  put_le(b, at + 2, (uint64_t)nmsg, 2);  /* number of messages */
  put_le(b, at + 4, 1, 4);               /* reference count */
  put_le(b, at + 8, (uint64_t)msg_bytes, 4);
  return at;
}

static void write_dataset(Buf *b, Node *d) {
  const size_t dspace = 8 + 8 * (size_t)d->rank;
  const size_t dtype = datatype_bytes(d->type);
  const size_t fill = 4, layout = 18;
  const size_t msgs = 4 * 8 + pad8(dspace) + pad8(dtype) + pad8(fill) + pad8(layout);
  const size_t oh = object_header(b, 4, msgs);
  d->addr = oh;
  uint64_t count = 1;
  for (int k = 0; k < d->rank; k++) count *= d->dims[k];
  const size_t nbytes = (size_t)count * type_size(d->type);
  const size_t data_at = buf_zeros(b, pad8(nbytes));
  if (nbytes) memcpy(b->p + data_at, d->data, nbytes);
  size_t cur = oh + 16;
  size_t m = message(b, &cur, 0x0001, dspace);  /* dataspace, version 1 */
  b->p[m] = 1;
  b->p[m + 1] = (unsigned char)d->rank;
  for (int k = 0; k < d->rank; k++) put_le(b, m + 8 + 8 * k, d->dims[k], 8);
  m = message(b, &cur, 0x0003, dtype);          /* datatype */
  write_datatype(b, m, d->type);
  m = message(b, &cur, 0x0005, fill);           /* fill value, version 2: late allocation, none defined */
  b->p[m] = 2;
  b->p[m + 1] = 2;
  b->p[m + 2] = 2;
  b->p[m + 3] = 0;
  m = message(b, &cur, 0x0008, layout);         /* data layout, version 3: contiguous */
  b->p[m] = 3;
  b->p[m + 1] = 1;
  put_le(b, m + 2, data_at, 8);
  put_le(b, m + 10, nbytes, 8);
}

static int name_cmp(const void *a, const void *b) {
  return strcmp((*(Node *const *)a)->name, (*(Node *const *)b)->name);
}

/* A group: object header (symbol table message), B-tree leaf, symbol table
 * node and local heap; members first, so their addresses are known.  Returns
 * the B-tree and heap addresses through bt / hp for the parent's entry. */
static void write_group(Buf *b, Node *g, uint64_t *bt, uint64_t *hp) {
  qsort(g->child, (size_t)g->nchild, sizeof(Node *), name_cmp);
  uint64_t cbt[2 * LEAF_K], chp[2 * LEAF_K];
  for (int k = 0; k < g->nchild; k++) {
    if (g->child[k]->is_group)
      write_group(b, g->child[k], &cbt[k], &chp[k]);
    else
      write_dataset(b, g->child[k]);
  }
  /* local heap: offset 0 holds the empty string, then the member names */
  size_t heap_data = 8, name_off[2 * LEAF_K];
  for (int k = 0; k < g->nchild; k++) {
    name_off[k] = heap_data;
    heap_data += pad8(strlen(g->child[k]->name) + 1);
  }
  const size_t heap = buf_zeros(b, 32 + heap_data);
  memcpy(b->p + heap, "HEAP", 4);
  put_le(b, heap + 8, heap_data, 8);
  put_le(b, heap + 16, HEAP_FREE_NULL, 8);
  put_le(b, heap + 24, heap + 32, 8);
  for (int k = 0; k < g->nchild; k++) memcpy(b->p + heap + 32 + name_off[k], g->child[k]->name, strlen(g->child[k]->name));
  /* symbol table node: 2K entries of 40 bytes */
  const size_t snod = buf_zeros(b, 8 + 2 * LEAF_K * 40);
  memcpy(b->p + snod, "SNOD", 4);
  b->p[snod + 4] = 1;
  put_le(b, snod + 6, (uint64_t)g->nchild, 2);
  for (int k = 0; k < g->nchild; k++) {
    const size_t e = snod + 8 + 40 * (size_t)k;
    put_le(b, e, name_off[k], 8);
    put_le(b, e + 8, g->child[k]->addr, 8);
    if (g->child[k]->is_group) {  /* cache type 1: the member group's B-tree and heap */
      put_le(b, e + 16, 1, 4);
      put_le(b, e + 24, cbt[k], 8);
      put_le(b, e + 32, chp[k], 8);
    }
  }
  /* B-tree leaf of node type 0 (group), one child: keys are heap offsets, the
   * left one the empty string, the right one the last (greatest) member name;
   * allocated for 2K children like every group B-tree node */
  const size_t tree = buf_zeros(b, 24 + (2 * INTERNAL_K + 1) * 8 + 2 * INTERNAL_K * 8);
  memcpy(b->p + tree, "TREE", 4);
  b->p[tree + 4] = 0;
  b->p[tree + 5] = 0;
  put_le(b, tree + 6, g->nchild ? 1 : 0, 2);
  put_le(b, tree + 8, UNDEF_ADDR, 8);
  put_le(b, tree + 16, UNDEF_ADDR, 8);
  if (g->nchild) {
    put_le(b, tree + 24, 0, 8);
    put_le(b, tree + 32, snod, 8);
    put_le(b, tree + 40, name_off[g->nchild - 1], 8);
  }
  /* the group's object header: one symbol table message */
  const size_t oh = object_header(b, 1, 8 + 16);
  size_t cur = oh + 16;
  const size_t m = message(b, &cur, 0x0011, 16);
  put_le(b, m, tree, 8);
  put_le(b, m + 8, heap, 8);
  g->addr = oh;
  *bt = tree;
  *hp = heap;
}

/* Writes the tree rooted at `root` as an HDF5 file at `path`. */
static void write_h5(const char *path, Node *root) {
  Buf b = {0};
  buf_zeros(&b, 96);  /* superblock, filled in below */
  uint64_t bt = 0, hp = 0;
  write_group(&b, root, &bt, &hp);
  static const unsigned char sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  memcpy(b.p, sig, 8);
  /* versions: superblock 0, free space 0, root symbol table entry 0, shared headers 0 */
  b.p[13] = 8; /* size of offsets */
  b.p[14] = 8; /* size of lengths */
  put_le(&b, 16, LEAF_K, 2);
  put_le(&b, 18, INTERNAL_K, 2);
  put_le(&b, 24, 0, 8);            /* base address */
  put_le(&b, 32, UNDEF_ADDR, 8);   /* free-space info */
  put_le(&b, 40, b.n, 8);          /* end of file */
  put_le(&b, 48, UNDEF_ADDR, 8);   /* driver information */
  put_le(&b, 56, 0, 8);            /* root entry: link name offset */
  put_le(&b, 64, root->addr, 8);   /* object header */
  put_le(&b, 72, 1, 4);            /* cache type 1 */
  put_le(&b, 80, bt, 8);
  put_le(&b, 88, hp, 8);
  FILE *f = fopen(path, "wb");
  if (!f || fwrite(b.p, 1, b.n, f) != b.n) {
    perror(path);
    abort();
  }
  fclose(f);
  free(b.p);
}

/* ---------------------------------------------------------------- spsim's outputs */

static void write_cxi(const char *basename, int index, const void *array, int complex_values, int binned,
                      const SpRotation *rot, const Options *opts) {
  if (!array) {  /* the array was never computed (spsim would read a NULL pointer here) */
    fprintf(stderr, "spsim_b200: %s not computed; %s-%05d.cxi not written\n", basename, basename, index);
    return;
  }
  const CCD *det = opts->detector;
  const int bx = binned && det->binning_x > 0 ? det->binning_x : 1;
  const int by = binned && det->binning_y > 0 ? det->binning_y : 1;
  const int bz = binned && det->binning_z > 0 ? det->binning_z : 1;
  const int nx = det->nx / bx, ny = det->ny / by, nz = (det->nz > 0 ? det->nz : 1) / bz;
  const size_t n = (size_t)nx * ny * nz;
  int32_t *mask = (int32_t *)malloc((n ? n : 1) * sizeof(int32_t));
  if (!mask) abort();
  for (size_t i = 0; i < n; i++) mask[i] = 1;
  const int32_t version = 150;
  const double distance = det->distance, wavelength = opts->experiment->wavelength;
  const double xs = (double)(det->pixel_width * (binned ? bx : det->binning_x));
  const double ys = (double)(det->pixel_height * (binned ? by : det->binning_y));
  double R[9];
  Node root = {"", 1}, entry = {"entry_1", 1}, image = {"image_1", 1}, detn = {"detector_1", 1},
       src = {"source_1", 1};
  Node cv = {"cxi_version", 0}, data = {"data", 0}, msk = {"mask", 0}, dist = {"distance", 0},
       xps = {"x_pixel_size", 0}, yps = {"y_pixel_size", 0}, wl = {"wavelength", 0}, ori = {"orientation", 0};
  cv.type = T_I32, cv.rank = 0, cv.data = &version;
  data.type = complex_values ? T_C64 : T_F32;
  msk.type = T_I32;
  data.rank = msk.rank = nz > 1 ? 3 : 2;
  for (Node *d = &data; d; d = d == &data ? &msk : NULL) {
    if (d->rank == 3) {
      d->dims[0] = (uint64_t)nz, d->dims[1] = (uint64_t)ny, d->dims[2] = (uint64_t)nx;
    } else {
      d->dims[0] = (uint64_t)ny, d->dims[1] = (uint64_t)nx;
    }
  }
  data.data = array;
  msk.data = mask;
  dist.type = xps.type = yps.type = wl.type = T_F64;
  dist.data = &distance, xps.data = &xs, yps.data = &ys, wl.data = &wavelength;
  add_child(&root, &cv);
  add_child(&root, &entry);
  add_child(&entry, &image);
  add_child(&image, &data);
  add_child(&image, &msk);
  add_child(&image, &detn);
  add_child(&image, &src);
  add_child(&detn, &dist);
  add_child(&detn, &xps);
  add_child(&detn, &yps);
  add_child(&src, &wl);
  if (rot && rot->data && rot->rows == 3 && rot->cols == 3) {
    for (int k = 0; k < 9; k++) R[k] = (double)rot->data[k];
    ori.type = T_F64, ori.rank = 2, ori.dims[0] = 3, ori.dims[1] = 3, ori.data = R;
    add_child(&image, &ori);
  }
  char path[1100];
  snprintf(path, sizeof(path), "%s-%05d.cxi", basename, index);
  write_h5(path, &root);
  free(mask);
}

/* src/spsim.c:146-152 */
void output_array(char *basename, int index, float *array, SpRotation *rot, Options *opts) {
  write_cxi(basename, index, array, 0, 0, rot, opts);
}

/* src/spsim.c:175-181 */
void output_carray(char *basename, int index, Complex *array, SpRotation *rot, Options *opts) {
  write_cxi(basename, index, array, 1, 0, rot, opts);
}

/* src/spsim.c:228-279: the requested arrays as CXI files (the binned detector
 * outputs with their binned shape), the scattering intensity as VTK on request;
 * the real-space outputs (an FFT of the pattern, outside this path) are
 * reported and skipped. */
void output_files(Diffraction_Pattern *pattern, Options *opts, int index) {
  CCD *det = opts->detector;
  if (opts->output_scatt_int || opts->output_intensities)
    write_cxi("scattering_int", index, pattern->ints, 0, 0, pattern->rot, opts);
  if (opts->output_sf_vtk) {
    char buffer[1024];
    snprintf(buffer, sizeof(buffer), "scattering_factor-%05d.vtk", index);
    write_3D_array_to_vtk(pattern->ints, det->nx, det->ny, det->nz > 0 ? det->nz : 1, buffer);
  }
  if (opts->output_noiseless_photons)
    write_cxi("noiseless_photon_out", index, det->photons_per_pixel, 0, 0, pattern->rot, opts);
  if (opts->output_scattering_factors) write_cxi("scattering_factors", index, pattern->F, 1, 0, pattern->rot, opts);
  if (opts->output_solid_angles) write_cxi("solid_angles", index, det->solid_angle, 0, 0, pattern->rot, opts);
  if (opts->output_photons) write_cxi("photon_out", index, det->photon_count, 0, 0, pattern->rot, opts);
  if (opts->output_count) write_cxi("counts_out", index, det->real_output, 0, 1, pattern->rot, opts);
  if (opts->output_noiseless_count)
    write_cxi("noiseless_counts_out", index, det->noiseless_output, 0, 1, pattern->rot, opts);
  if (opts->output_real_space || opts->output_realspace_histogram)
    fprintf(stderr, "spsim_b200: real-space outputs are not produced (outside the structure-factor path)\n");
}
