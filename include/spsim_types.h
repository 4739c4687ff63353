/*
 * spsim_types.h — spsim's data model, layout-compatible with the reference
 * headers include/config.h:44-181 and include/diffraction.h:46-62, so a caller
 * compiled against spsim can link against libspsim_b200.so unchanged.
 * libspimage types that appear in those structs (Complex, SpRotation) are
 * given their libspimage layouts here, since libspimage is not a dependency.
 */
#ifndef SPSIM_B200_TYPES_H
#define SPSIM_B200_TYPES_H

#ifdef __cplusplus
extern "C" {
#endif

/* include/config.h:33-41 */
#define CHEM_FORMULA 1
#define PDB 2
#define BOX_SPHERICAL 1
#define BOX_PARALLEL 2
#define POLARIZATION_IGNORE 0
#define POLARIZATION_VERTICAL 1
#define POLARIZATION_HORIZONTAL 2
#define POLARIZATION_UNPOLARIZED 3

#ifndef SPSIM_B200_NO_LIBSPIMAGE_TYPES
/* libspimage: Complex with real == float; sp_matrix (rows, cols, row-major data) */
typedef struct {
  float re;
  float im;
} Complex;

typedef struct {
  unsigned int rows;
  unsigned int cols;
  float *data;
} SpRotation;
#endif

/* include/crystal.h:30 */
typedef enum { CrystalA, CrystalB, CrystalC } CrystalAxis;

/* include/config.h:44-48 */
typedef struct {
  int n_elements;
  int *atomic_number;
  int *quantity;
} Chem_Formula;

/* include/config.h:50-58: positions in metres, xyz per atom */
typedef struct {
  int natoms;
  int *atomic_number;
  float *pos;
  int delta_atoms;
} Molecule;

/* include/config.h:60-76 */
typedef struct {
  float wavelength;
  float bandwidth;
  float exposure_time;
  float beam_intensity;
  float beam_center_x;
  float beam_center_y;
  float beam_fwhm;
  float beam_energy;
  float photon_energy;
  float focal_diameter;
  int polarization;
} Experiment;

/* include/config.h:78-128 */
typedef struct {
  float *photons_per_pixel;
  float *thomson_correction;
  float *solid_angle;
  float *photon_count;
  float *electrons_per_pixel;
  float *real_output;
  float *noiseless_output;
  float distance;
  float width;
  float height;
  float depth;
  float pixel_width;
  float pixel_height;
  float pixel_depth;
  float quantum_efficiency;
  float electron_hole_production_energy;
  float readout_noise;
  float dark_current;
  float linear_full_well;
  int binning_x;
  int binning_y;
  int binning_z;
  int nx;
  int ny;
  int nz;
  float maximum_value;
  int spherical;
  float gaussian_blurring;
  float real_space_blurring;
  float center_x;
  float center_y;
  float center_z;
  int n_patterns;
} CCD;

/* include/config.h:131-181 */
typedef struct {
  int input_type;
  Chem_Formula *chem_formula;
  Experiment *experiment;
  CCD *detector;
  char pdb_filename[1024];
  char sf_filename[1024];
  char hkl_grid_filename[1024];
  int box_type;
  float box_dimension;
  int use_fft_for_sf;
  int use_nfft_for_sf;
  float b_factor;
  int origin_to_com;
  float euler_orientation[3];
  int random_orientation;
  int n_patterns;
  int vectorize;
  int delta_atoms;
  int fast_exit;
  int crystal_size[3];
  float crystal_cell[6];
  int use_cuda;
  int wavelength_samples;
  int random_seed;
  int output_sf_vtk;
  int output_scatt_int;
  int output_ewald_vtk;
  int output_intensities;
  int output_noiseless_photons;
  int output_photons;
  int output_electron_pixel_vtk;
  int output_noiseless_count;
  int output_count;
  int output_realspace_histogram;
  int output_scattering_factors;
  int output_solid_angles;
  int output_real_space;
  int verbosity_level;
} Options;

/* include/diffraction.h:46-62 */
typedef struct {
  float *ints;
  Complex *F;
  int N_pix;
  float max_s[3];
  float d_s[3];
  float *HKL_list;
  int HKL_list_size;
  SpRotation *rot;
} Diffraction_Pattern;

#ifdef __cplusplus
}
#endif

#endif
