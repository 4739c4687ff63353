/*
 * spsim.h — the reference-shaped C entry points of libspsim_b200.so.
 *
 * Same names, signatures, ownership and error behaviour as spsim's own
 * (the file:line after each names the reference declaration it replaces);
 * the structure factor and the detector chain run on the GPU through the
 * native ABI in spsim_b200.h.  Ownership is the reference's: the callee
 * mallocs returned patterns and the CCD output arrays; free them with
 * free_diffraction_pattern / free_output_in_options.  Like the reference,
 * these functions have no status return: on a failure they print the reason
 * to stderr and abort() (no silent CPU fallback).
 */
#ifndef SPSIM_B200_SPSIM_H
#define SPSIM_B200_SPSIM_H

#include "spsim_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- configuration: include/config.h:184-187 ---- */
Options *set_defaults(void);                                     /* src/config.c:30 */
void read_options_file(char *filename, Options *opt);            /* src/config.c:89 */
void write_options_file(char *filename, Options *opt);           /* src/config.c:433 */

/* ---- geometry: include/diffraction.h:72-73, :104 ---- */
float *get_HKL_list_for_detector(CCD *det, Experiment *exp, int *HKL_list_size);  /* src/diffraction.c:237 */
float *get_HKL_list_for_3d_detector(CCD *det, Experiment *exp, int *HKL_list_size); /* src/diffraction.c:325 */
SpRotation *apply_orientation_to_HKL_list(float **HKL_list, int *HKL_list_size, Options *opts); /* :300 */
float *get_HKL_list(Options *opts, int *HKL_list_size);          /* include/spsim.h:44, src/spsim.c:98 */

/* ---- structure factor: include/diffraction.h:76-83 ---- */
Diffraction_Pattern *compute_pattern_on_list(Molecule *mol, float *HKL_list, int HKL_list_size, float B,
                                             Experiment *exp, Options *opts);        /* src/diffraction.c:770 */
Diffraction_Pattern *vector_compute_pattern_on_list(Molecule *mol, float *HKL_list, int HKL_list_size, float B,
                                                    Experiment *exp, Options *opts); /* src/diffraction.c:856 */
Diffraction_Pattern *cuda_compute_pattern_on_list(Molecule *mol, float *HKL_list, int HKL_list_size, float B,
                                                  Experiment *exp, Options *opts);   /* src/diffraction.cu:135 */
Diffraction_Pattern *cuda_compute_pattern_on_list2(Molecule *mol, float *HKL_list, int HKL_list_size, float B,
                                                   Experiment *exp, Options *opts);  /* src/diffraction.cu:235 */
Diffraction_Pattern *compute_pattern_on_list_by_nfft(Molecule *mol, float *HKL_list, int HKL_list_size, CCD *det,
                                                     float B, Options *opts);        /* src/diffraction.c:528 */
Diffraction_Pattern *compute_sf(Molecule *mol, float *HKL_list, int HKL_list_size, Options *opts); /* src/spsim.c:110 */

/* ---- detector chain: include/diffraction.h:85-89, include/noise.h:33, include/amplification.h:24-26 ---- */
void calculate_thomson_correction(CCD *det, Experiment *exp);            /* src/diffraction.c:1109 */
void calculate_pixel_solid_angle(CCD *det);                              /* src/diffraction.c:1146 */
void calculate_photons_per_pixel(Diffraction_Pattern *pattern, Options *opts); /* src/diffraction.c:1190 */
void generate_poisson_noise(CCD *det);                                   /* src/noise.c:32 */
void calculate_electrons_per_pixel(CCD *det, Experiment *experiment);    /* src/amplification.c:54 */
void calculate_real_detector_output(CCD *det, Experiment *experiment);   /* src/amplification.c:77 */
void calculate_noiseless_detector_output(CCD *det, Experiment *experiment); /* src/amplification.c:119 */

/* ---- orchestration: include/spsim.h:45-59 ---- */
Diffraction_Pattern *simulate_shot(Molecule *mol, Options *opts);        /* src/spsim.c:281 */
void free_stuff(Diffraction_Pattern *pattern, Options *opts);            /* src/spsim.c:348 */
void free_diffraction_pattern(Diffraction_Pattern *pattern);             /* src/spsim.c:353 */
void free_output_in_options(Options *opts);                              /* src/spsim.c:363 */

/* ---- output files: include/spsim.h:47-52 of spsim ----
 * <basename>-NNNNN.cxi, an HDF5 file in the CXI image layout written without
 * libspimage or the HDF5 library (see spsim_b200/csrc/host/cxi.c). */
void output_array(char *basename, int index, float *array, SpRotation *rot, Options *opts);     /* src/spsim.c:146 */
void output_carray(char *basename, int index, Complex *array, SpRotation *rot, Options *opts);  /* src/spsim.c:175 */
void output_files(Diffraction_Pattern *pattern, Options *opts, int index);                     /* src/spsim.c:228 */

/* ---- molecules: include/molecule.h:25-28 ---- */
Molecule *alloc_mol(void);                                               /* src/molecule.c:394 */
void add_atom_to_mol(Molecule *mol, int atomic_number, float x, float y, float z); /* src/molecule.c:402 */
void free_mol(Molecule *mol);                                            /* src/molecule.c:413 */

/* ---- molecule files: include/molecule.h:22-31, include/spsim.h (get_molecule) ----
 * PDB ATOM/HETATM records (coordinates in Angstrom -> metres, element from
 * columns 77-78) expanded by the REMARK 350 BIOMT operators; a chemical
 * formula as random positions in the options' box; PDB writing; centring on
 * the electron centre of mass.  Unidentifiable elements are skipped (the
 * reference overwrites the previous atom's Z instead). */
Molecule *get_Molecule_from_pdb(char *filename);                          /* src/molecule.c:65 */
Molecule *get_Molecule_from_formula(Chem_Formula *form, Options *opts);   /* src/molecule.c:33 */
void write_pdb_from_mol(char *filename, Molecule *mol);                   /* src/molecule.c:359 */
void origin_to_center_of_mass(Molecule *mol);                             /* src/molecule.c:440 */
Molecule *get_molecule(Options *opts);                                    /* src/spsim.c:83 */

/* ---- crystal lattice: include/crystal.h:30-33 ----
 * cell matrix rows A, B, C from crystal_cell (lengths in metres, angles in
 * degrees); the lattice sum over crystal_size cells runs on the GPU in FP64 */
void crystal_axis_to_cartesian(Options *opts, CrystalAxis axis, float *x, float *y, float *z); /* src/crystal.c:4 */
void crystal_cell_matrix(Options *opts, float *matrix);                  /* src/crystal.c:23 */
void calculate_pattern_from_crystal(float *I, Complex *F, float *HKL_list, int HKL_list_size,
                                    Options *opts);                      /* src/crystal.c:39 */

/* ---- VTK output: include/io.h ---- */
void write_2D_array_to_vtk(float *F, int nx, int ny, char *filename);     /* src/io.c:29 */
void write_3D_array_to_vtk(float *F, int nx, int ny, int nz, char *filename); /* src/io.c:60 */

/* ---- distribution: include/mpi_comm.h:30-32 (single-process semantics;
 *      multi-GPU sharding lives in the Python layer over torch.distributed) ---- */
void get_my_loop_start_and_end(int size, int *start, int *end);          /* src/mpi.c:30 */
void syncronize_patterns(Diffraction_Pattern *pat);                      /* src/mpi.c:50 */
void sum_patterns(Diffraction_Pattern *pat);                             /* src/mpi.c:62 */

/* ---- library controls (no counterpart in the reference) ----
 * Precision used by the reference-shaped structure-factor calls above
 * (SPSIM_PREC_* of spsim_b200.h; default SPSIM_PREC_F32), and the Philox key
 * of the noise stages (simulate_shot sets it from opts->random_seed). */
void spsim_b200_set_legacy_precision(int precision);
int spsim_b200_get_legacy_precision(void);
/* Relative error of the NUFFT structure factor behind
 * compute_pattern_on_list_by_nfft and use_nfft_for_sf (default 1e-8; see
 * spsim_b200_forward_nufft). */
void spsim_b200_set_legacy_nufft_eps(double eps);
double spsim_b200_get_legacy_nufft_eps(void);
void spsim_b200_set_noise_seed(unsigned long long seed);
/* Row chunks of simulate_shot on a flat detector with the direct
 * monochromatic or the NUFFT structure factor: chunk c's structure factor
 * (the NUFFT: its interpolation, the grid prepared once) and detector chain
 * run while chunk c - 1's outputs are copied to the host, so that only the
 * last chunk's copies follow the computation.  0 (default): 4 chunks from
 * 2^19 pixels on, none below; 1: none; at most 8.  Every output is that of
 * one whole-detector pass (each pixel keeps its noise stream; chunk rows are
 * a multiple of the y binning), up to the FP32 summation order of the
 * structure factor. */
void spsim_b200_set_shot_chunks(int chunks);
int spsim_b200_get_shot_chunks(void);

#ifdef __cplusplus
}
#endif

#endif
