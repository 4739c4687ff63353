/*
 * spsim_b200.h — native C ABI of the B200 structure-factor and detector-chain
 * library (libspsim_b200.so).
 *
 * Everything is plain C: opaque handles, pointers and sizes.  Every function
 * returns an int status (SPSIM_OK == 0); spsim_b200_last_error() gives the
 * message of the last failure on the calling thread.  The reference-shaped
 * entry points (compute_pattern_on_list, simulate_shot, read_options_file, ...)
 * live in spsim.h and are implemented on top of these.
 *
 * Units follow spsim: lengths in metres, scattering vectors q in 1/m (the
 * reference's HKL list, src/diffraction.c:237-297), B factors in Angstrom^2.
 * Sign convention: F(q) = sum_j f_j exp(-2 pi i q . r_j) (src/diffraction.c:836).
 */
#ifndef SPSIM_B200_H
#define SPSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SPSIM_OK 0
#define SPSIM_ERR_INVALID_ARG 1
#define SPSIM_ERR_CUDA 2
#define SPSIM_ERR_NO_DEVICE 3
#define SPSIM_ERR_OUT_OF_MEMORY 4
#define SPSIM_ERR_RANGE 5       /* phase range beyond the compensated FP32 kernel's domain */
#define SPSIM_ERR_TIMEOUT 6     /* a bounded device-side wait gave up (kernel returned early) */
#define SPSIM_ERR_UNSUPPORTED 7

/* ---- precision of the structure-factor sum ----------------------------- */
#define SPSIM_PREC_FP64 0        /* plain FP64 per-pixel kernel (FP64 phase, sincos, sum)      */
#define SPSIM_PREC_F32 1         /* FP64 (or compensated FP32) phase, FMA-pipe minimax sin/cos,*/
                                 /* float-float segment sums, FP64 cross-tile/element sum;     */
                                 /* <= 1e-5 relative |F|^2 error against FP64                  */
#define SPSIM_PREC_F32_FAST 2    /* the same phase and sums, MUFU sin/cos (on neighbour quads   */
                                 /* for half the pixels, the others on the polynomials)        */

/* ---- where caller buffers live ----------------------------------------- */
#define SPSIM_MEM_HOST 0
#define SPSIM_MEM_DEVICE 1

/* Detector-chain polarisation codes (include/config.h:36-39 of spsim). */
#define SPSIM_POL_IGNORE 0
#define SPSIM_POL_VERTICAL 1
#define SPSIM_POL_HORIZONTAL 2
#define SPSIM_POL_UNPOLARIZED 3

const char *spsim_b200_status_string(int status);
const char *spsim_b200_last_error(void);
/* Library version string. */
const char *spsim_b200_version(void);

/* Selects the CUDA device for the calling thread's later calls and checks it
 * is present (the reference's device probe, src/config.c:344-356, but as an
 * error instead of a silent CPU fallback). */
int spsim_b200_init(int device);
/* Number of visible CUDA devices (0 when none; never an error). */
int spsim_b200_device_count(int *count);

/* ---- molecules ----------------------------------------------------------
 * A molecule handle owns device-resident atom records: atoms with Z == 0 are
 * dropped (src/diffraction.c:830-832), the rest are sorted by element,
 * centred, and split into a coarse grid part and a remainder for the
 * compensated phase.  Weights are occ_j * sqrt(illumination_j)
 * (src/diffraction.c:223-235, :834), or 1 under delta_atoms.
 * pos: xyz per atom (metres), host memory.  occ / bfac may be NULL (1 / 0).
 * beam: {fwhm, centre_x, centre_y} in metres, or NULL for a plane wave.
 * bfac != NULL selects per-atom Debye-Waller factors exp(-B_j |q|^2/4), on top
 * of the global B of the forward call (the total is exp(-(B + B_j) |q|^2/4)). */
typedef struct spsim_b200_molecule spsim_b200_molecule;
int spsim_b200_molecule_create(int natoms, const int32_t *Z, const float *pos, const float *occ,
                               const float *bfac, int delta_atoms, const float *beam,
                               spsim_b200_molecule **out);
/* Same from FP64 positions (host). */
int spsim_b200_molecule_create_f64(int natoms, const int32_t *Z, const double *pos, const float *occ,
                                   const float *bfac, int delta_atoms, const float *beam,
                                   spsim_b200_molecule **out);
/* Refinement: rewrites positions / occupancies / B factors from DEVICE arrays
 * in the caller's original atom order, on `stream`, keeping the element
 * order and grid chosen at creation.  pos_dev is float (pos_is_f64 == 0) or
 * double; occ_dev / bfac_dev may be NULL (unchanged).  Positions that leave the
 * creation-time bounds (the radius about the centre plus 5 % or 0.5 nm) make
 * the next forward (direct or NUFFT) report SPSIM_ERR_RANGE through
 * spsim_b200_synchronize; each update clears the molecule's range word. */
int spsim_b200_molecule_update_device(spsim_b200_molecule *m, const void *pos_dev, int pos_is_f64,
                                      const float *occ_dev, const float *bfac_dev, void *stream);
int spsim_b200_molecule_natoms(const spsim_b200_molecule *m, int *natoms);
int spsim_b200_molecule_destroy(spsim_b200_molecule *m);

/* ---- pixel q sets -------------------------------------------------------
 * A q set owns the device-resident scattering vectors of one detector.
 * from_list: the reference's float HKL list (3 floats per pixel), in host or
 * device memory (src/diffraction.c:770, HKL_list argument).
 * from_detector: the Ewald-sphere geometry of src/diffraction.c:237-297
 * evaluated on the device in FP64 and kept in FP64 (flat or spherical). */
typedef struct spsim_b200_qset spsim_b200_qset;
int spsim_b200_qset_from_list(int64_t npix, const float *hkl, int memory, spsim_b200_qset **out);
int spsim_b200_qset_from_detector(int nx, int ny, float width, float height, float distance,
                                  float center_x, float center_y, float wavelength, int spherical,
                                  spsim_b200_qset **out);
int spsim_b200_qset_npix(const spsim_b200_qset *qs, int64_t *npix);
/* Copies the set's q vectors (3 per pixel, float) to host memory. */
int spsim_b200_qset_copy_q(const spsim_b200_qset *qs, float *hkl_host);
int spsim_b200_qset_destroy(spsim_b200_qset *qs);

/* ---- structure factor ---------------------------------------------------
 * One pattern: F (complex64, interleaved re/im, npix) and I = |F|^2 (float)
 * into DEVICE buffers on `stream` (a cudaStream_t, NULL = legacy default).
 * rot: optional 3x3 row-major FP64 rotation applied to every q (q' = R q,
 * src/diffraction.c:300-323), NULL = identity.  B: global B factor
 * (src/diffraction.c:183-193).  Either output may be NULL. */
int spsim_b200_forward(const spsim_b200_molecule *m, const spsim_b200_qset *qs, const double *rot,
                       float B, int precision, float *F_dev, float *I_dev, void *stream);

/* Many patterns in one persistent launch: pattern i uses mols[i], qsets[i],
 * rot[9*i] (NULL = identity for all) and writes F_dev[i] / I_dev[i] (device
 * pointers, entries may be NULL).  Work items (pixel tile x atom range) are
 * cost-sorted and drained by a persistent kernel; the whole launch sequence
 * is captured once per plan into a CUDA graph and replayed while the plan's
 * shapes and pointers stay the same. */
int spsim_b200_forward_batch(int npatterns, const spsim_b200_molecule *const *mols,
                             const spsim_b200_qset *const *qsets, const double *rot, float B,
                             int precision, float *const *F_dev, float *const *I_dev, void *stream);

/* Polychromatic forward, the semantics of spsim's spectrum kernel
 * (src/diffraction.cu:415-476, CUDA_spectrum_scattering_from_all_atoms, which
 * its default CUDA path runs when experiment_bandwidth != 0): with S samples
 * (an even S > 1 is raised by one, src/diffraction.cu:305-307),
 *   lambda_j = lambda (1 - bw/2) + j/(S-1) lambda bw,
 *   F(q) = sum_j w_j sum_atoms f_e(|q|) w_a exp(-2 pi i (lambda/lambda_j) q.r),
 * w_j proportional to exp(-z_j^2/2), z_j = (lambda_j - lambda)/(lambda bw/4),
 * summing to one; form factors stay at the unscaled |q| as in the reference.
 * All S samples run as one batched launch (a captured graph on non-default
 * streams), combined in FP64.  bandwidth == 0 or samples == 1 is the plain
 * forward.  samples < 1 is SPSIM_ERR_INVALID_ARG. */
int spsim_b200_forward_spectrum(const spsim_b200_molecule *m, const spsim_b200_qset *qs, const double *rot,
                                float B, int precision, float wavelength, float bandwidth, int samples,
                                float *F_dev, float *I_dev, void *stream);

/* Host-memory convenience: atoms and HKL list from host, F / I back to host
 * (copies inside).  The reference-shaped compute_pattern_on_list is built on it. */
int spsim_b200_structure_factor_host(int natoms, const int32_t *Z, const float *pos, const float *occ,
                                     const float *bfac, float B, int delta_atoms, const float *beam,
                                     int64_t npix, const float *hkl, int precision, float *F_host,
                                     float *I_host);

/* spsim_b200_structure_factor_host with a bandwidth-broadened beam
 * (spsim_b200_forward_spectrum's semantics); cuda_compute_pattern_on_list2
 * and compute_sf (use_cuda = 1) are built on it. */
int spsim_b200_structure_factor_host_spectrum(int natoms, const int32_t *Z, const float *pos, const float *occ,
                                              const float *bfac, float B, int delta_atoms, const float *beam,
                                              float wavelength, float bandwidth, int samples, int64_t npix,
                                              const float *hkl, int precision, float *F_host, float *I_host);

/* ---- non-uniform FFT structure factor --------------------------------------
 * The same F(q) = sum_e f_e(|q|) sum_{j in e} w_j exp(-2 pi i q.r_j) as
 * spsim_b200_forward, computed per element as a type-3 non-uniform FFT
 * (atoms spread onto a real-space grid, one batched 3-D FFT, interpolation at
 * every pixel's q; FP64 spreading and FFT, an FP32 copy of the FFT grid for
 * the interpolation) in O(atoms w^3 + grid log grid + pixels w^3)
 * instead of O(atoms x pixels).  Replaces the reference's NNFFT path
 * (compute_pattern_on_list_by_nfft, src/diffraction.c:528-675, dispatched by
 * compute_sf when use_nfft_for_sf is set, src/spsim.c:119-123), which runs
 * the NFFT library with a cut-off of m = 2.
 * eps: target relative L2 error of F against the exact sum, in
 * [1e-14, 1e-2] (measured errors come out within a few eps, and not below the
 * complex64 output's ~3e-8); it sets the interpolation kernel width
 * w = ceil(-log10 eps) + 1 grid points (up to 15) and the spreading width
 * w + 3 (up to 16).  The grids follow the bounding box of R q and the
 * molecule's radius r_b: about 6 S_d r_b + w + 5 spreading points per axis
 * (S_d: half-width of the q box along d) and twice that, rounded up to a size
 * with factors 2, 3, 5, 7, for the FFT.
 * Not supported: per-atom B factors (SPSIM_ERR_INVALID_ARG).  F_dev, I_dev
 * as spsim_b200_forward; enqueued on `stream` after a one-time read-back of
 * the q box per (q set, rotation); atoms that moved outside the creation-time
 * bounds are left out and reported as SPSIM_ERR_RANGE by
 * spsim_b200_synchronize.  No reference counterpart beyond the NNFFT path. */
int spsim_b200_forward_nufft(const spsim_b200_molecule *m, const spsim_b200_qset *qs, const double *rot, float B,
                             double eps, float *F_dev, float *I_dev, void *stream);
/* npatterns orientations of one molecule on one q set (pattern i at rot[9 i],
 * or all unrotated if rot is NULL), outputs [npatterns][npix] in F_dev / I_dev.
 * The grid is sized for the ball |R q| <= |q|max, which holds for every
 * rotation: the atoms are spread and transformed once, every pattern is one
 * interpolation pass, and nothing is read back to the host.  Otherwise as
 * spsim_b200_forward_nufft (which sizes its grid for the box of the one
 * rotated list); npatterns in [1, 65535]. */
int spsim_b200_forward_nufft_batch(const spsim_b200_molecule *m, const spsim_b200_qset *qs, int npatterns,
                                   const double *rot, float B, double eps, float *F_dev, float *I_dev,
                                   void *stream);
/* Kernel widths (spreading, interpolation) and FFT grid (x, y, z) of the last
 * NUFFT forward on this thread. */
int spsim_b200_last_nufft_grid(int *w_spread, int *w_interp, int *n2);
/* Interpolation path of the NUFFT forwards (process-wide): 0 (default) lets
 * q sets made from a detector walk each 16 x 8 pixel tile's grid region in
 * shared memory together; 1 reads every pixel's stencil on its own.  Both
 * give the same bits.  Other values: SPSIM_ERR_INVALID_ARG. */
int spsim_b200_set_nufft_interp(int mode);
/* The NUFFT structure factor of host arrays with unit atom weights (the
 * reference NNFFT's semantics: no illumination weights), host F (complex64)
 * and I out; synchronous. */
int spsim_b200_structure_factor_host_nufft(int natoms, const int32_t *Z, const float *pos, float B, int delta_atoms,
                                           int64_t npix, const float *hkl, double eps, float *F_host, float *I_host);

/* ---- allocation-free variant (no counterpart in the reference) ------------
 * The computation, arguments and results of spsim_b200_structure_factor_host
 * (the same kernels, chosen by the same rules as its untuned defaults, and the
 * same phase-range limit: SPSIM_ERR_RANGE beyond 2^48 cycles), for callers
 * that may not allocate device memory while they run: applications that hand
 * out all device memory from their own fixed budget or pool, and services
 * that cannot afford a cudaMalloc / cudaFree (which synchronise the whole
 * device) on every call.  It calls no cudaMalloc, cudaFree or other allocating
 * routine: its device scratch is one static 64 MiB array per GPU (held by
 * every GPU that loads the library, until the process exits) and its host
 * staging a static 16 MiB array.  A call needs about 160 bytes per atom plus
 * (40 + 8 x number of elements) bytes per pixel of scratch, e.g. 100,000 atoms
 * on a 256 x 256 detector; larger calls return SPSIM_ERR_INVALID_ARG, with the
 * sizes in spsim_b200_last_error().  The first call on a device looks up that
 * device's address of the array, so make it before any stream capture;
 * cudaDeviceReset between calls is not supported.  Calls share the array: they
 * are serialised and synchronised before returning; calls that overlapped on
 * the GPU would race. */
int spsim_b200_structure_factor_host_noalloc(int natoms, const int32_t *Z, const float *pos, const float *occ,
                                             const float *bfac, float B, int delta_atoms, const float *beam,
                                             int64_t npix, const float *hkl, int precision, float *F_host,
                                             float *I_host);

/* ---- adjoint -------------------------------------------------------------
 * Given G_p = dL/dI_p for every pixel of `npat` patterns (device, float,
 * npat*npix) and the forward's F (device, complex64, npat*npix), accumulates
 * dL/dpos (double, 3 per atom, caller's atom order), dL/docc and dL/dB (double
 * per atom; NULL to skip) on `stream`.  Phases are recomputed, nothing of size
 * atoms x pixels is stored.  The outputs are overwritten.  The form-factor
 * table, atom blocks and work items of a (molecule, q set, pattern count, B,
 * precision) are built on the first call and reused by the next ones, which
 * allocate nothing; calls that share such a plan run in call order, whatever
 * their streams. */
int spsim_b200_adjoint(const spsim_b200_molecule *m, const spsim_b200_qset *qs, int npat,
                       const double *rot, float B, int precision, const float *F_dev, const float *G_dev,
                       double *dpos_dev, double *docc_dev, double *dB_dev, void *stream);

/* ---- detector chain ------------------------------------------------------
 * The per-pixel chain of src/spsim.c:281-346 after the structure factor:
 * Thomson (src/diffraction.c:1109-1144), solid angle (:1146-1187), photons
 * (:1190-1204), Poisson counts (src/noise.c:32-51, counter-based Philox
 * instead of GSL), electrons (src/amplification.c:54-74), binned real output
 * with dark current, readout noise and ADC (:77-116), and the noiseless
 * output (:119-155).  All arrays are DEVICE pointers; any output may be NULL. */
typedef struct {
  int nx, ny, nz;                /* detector pixels */
  int binning_x, binning_y, binning_z;
  int spherical;
  int polarization;              /* SPSIM_POL_* */
  float width, height, distance; /* metres */
  float center_x, center_y;
  float pixel_width, pixel_height;
  float wavelength;              /* metres */
  float beam_intensity;          /* photons / m^2 */
  float quantum_efficiency;
  float electron_hole_production_energy; /* joules; 0 = one electron per photon */
  float dark_current;            /* electrons / (pixel s) */
  float exposure_time;           /* s */
  float readout_noise;           /* electrons rms per binned pixel */
  float linear_full_well;        /* electrons */
  float maximum_value;           /* ADC counts */
  int clamp_to_maximum;          /* extension: clamp the ADC output at maximum_value */
  uint64_t seed;                 /* Philox key */
  uint32_t pattern_index;        /* Philox counter word: independent streams per pattern */
} spsim_b200_chain_params;

typedef struct {
  float *thomson_correction;   /* [nx*ny*nz] */
  float *solid_angle;          /* [nx*ny*nz] */
  float *photons_per_pixel;    /* [nx*ny*nz] */
  float *photon_count;         /* [nx*ny*nz] */
  float *electrons_per_pixel;  /* [nx*ny*nz] */
  float *real_output;          /* [(nx/bx)*(ny/by)*(nz/bz)] */
  float *noiseless_output;     /* [(nx/bx)*(ny/by)*(nz/bz)] */
} spsim_b200_chain_outputs;

/* Runs the fused chain on intensities I_dev (|F|^2, device, nx*ny*nz floats). */
int spsim_b200_detector_chain(const spsim_b200_chain_params *p, const float *I_dev,
                              const spsim_b200_chain_outputs *out, void *stream);
/* Individual stages, for the reference-shaped per-stage entry points. */
int spsim_b200_thomson(const spsim_b200_chain_params *p, float *out_dev, void *stream);
int spsim_b200_solid_angle(const spsim_b200_chain_params *p, float *out_dev, void *stream);
/* photon_count_dev[i] = Poisson(lambda_dev[i]) (Gaussian approximation at >= 1000). */
int spsim_b200_poisson(int64_t n, const float *lambda_dev, uint64_t seed, uint32_t pattern_index,
                       float *photon_count_dev, void *stream);
/* photons_dev[i] = T[i] * Omega[i] * I[i] * beam_intensity, in that float order
 * (src/diffraction.c:1190-1204). */
int spsim_b200_photons(int64_t n, const float *thomson_dev, const float *solid_angle_dev, const float *I_dev,
                       float beam_intensity, float *photons_dev, void *stream);
/* Poisson photon counts of photons_dev[i] * QE (src/noise.c:32-51). */
int spsim_b200_photon_counts(const spsim_b200_chain_params *p, const float *photons_dev, float *counts_dev,
                             void *stream);
/* electrons_dev[i] = counts_dev[i] * electrons-per-photon (src/amplification.c:54-74). */
int spsim_b200_electrons(const spsim_b200_chain_params *p, const float *counts_dev, float *electrons_dev,
                         void *stream);
/* Binned real output from electrons and / or binned noiseless output from
 * photons (src/amplification.c:77-155); either input/output pair may be NULL. */
int spsim_b200_binned_outputs(const spsim_b200_chain_params *p, const float *electrons_dev,
                              const float *photons_dev, float *real_output_dev, float *noiseless_output_dev,
                              void *stream);

/* ---- Ewald geometry ----------------------------------------------------- */
/* The reference's HKL list (float, 3 per pixel, row-major) for a flat or
 * spherical 2-D detector, computed in FP64 on the device and stored as float
 * (src/diffraction.c:237-297).  out is a DEVICE pointer. */
int spsim_b200_hkl_for_detector(int nx, int ny, float width, float height, float distance,
                                float center_x, float center_y, float wavelength, int spherical,
                                float *hkl_dev, void *stream);

/* The reciprocal-space grid of a 3-D (volume) detector, spsim's
 * get_HKL_list_for_3d_detector (src/diffraction.c:325-369): pixel centres
 * ((i - (n-1)/2)/n) * extent - centre along x, y, z, times
 * 1 / (distance * wavelength), FP64, stored as float (z outer, x inner). */
int spsim_b200_hkl_for_3d_detector(int nx, int ny, int nz, float width, float height, float depth,
                                   float distance, float center_x, float center_y, float center_z,
                                   float wavelength, float *hkl_dev, void *stream);

/* Crystal lattice sum, spsim's calculate_pattern_from_crystal
 * (src/crystal.c:39-71), in place on device data: F <- F * sum over
 * na x nb x nc cells of exp(-2 pi i q.(a A + b B + c C)), I = |F|^2 (I_dev may
 * be NULL).  cell: the 3x3 cell matrix, rows A, B, C in metres (as
 * crystal_cell_matrix returns it); hkl_dev: float q per pixel.  The lattice
 * factor is the product of three one-dimensional sums, each in FP64. */
int spsim_b200_crystal_lattice_sum(int64_t npix, const float *hkl_dev, const float *cell, int na, int nb, int nc,
                                   float *F_dev, float *I_dev, void *stream);

/* ---- completion, errors and timing -------------------------------------
 * Device-side failures of asynchronous calls (a bounded wait that gave up,
 * refined positions outside the molecule's bounds) are recorded in device
 * flags; spsim_b200_synchronize waits for `stream` and reports them. */
int spsim_b200_synchronize(void *stream);

/* Test hook for the bounded device waits (no reference counterpart; spsim has
 * no device-side waits).  While `on` is set for the current device, every
 * structure-factor kernel (the direct FP32 forms, not the plain FP64 kernel)
 * arms the barrier of its first atom tile without issuing the tile's copy, so
 * that its first wait runs out after ~10 ms instead of ~2 s: the kernel sets
 * its error word, waits for its copies still in flight and returns, and the
 * forward reports SPSIM_ERR_TIMEOUT (the synchronous calls directly, the others
 * through spsim_b200_synchronize).  Nothing faults and the context stays
 * usable; with the hook off again the next forward runs normally.  Waits for
 * the device to go idle before it changes the setting. */
int spsim_b200_debug_stall_first_copy(int on);

/* Per-launch timing of the structure-factor kernel with CUDA events recorded
 * on the launching stream.  While enabled, forwards run as direct launches
 * (no graph replay) so every launch is bracketed. */
int spsim_b200_timing_enable(int enable);
/* Waits for the recorded events and returns up to `cap` kernel durations (ms)
 * recorded since the last read, oldest first; *n is the number returned. */
int spsim_b200_timing_read(double *ms, int cap, int *n);

/* Atom-pixel terms evaluated by the last forward on this thread and the
 * duration (ms) of its last timed kernel launch (0 when timing is off): the
 * reference's "atoms.pixel/s" self-report (src/diffraction.c:849-851). */
int spsim_b200_last_forward_stats(double *terms, double *kernel_ms);

/* The reference-shaped calls (include/spsim.h) and
 * spsim_b200_structure_factor_host keep device scratch between calls on the
 * calling thread (grow-only buffers, the last molecule while its atom arrays
 * stay byte-identical, a reusable plan), the NUFFT forwards keep their grids
 * and twiddle tables per device, and the adjoint keeps its last few plans (form
 * factors, atom blocks, work items, rotations); this frees all of them for the
 * current device.  No reference counterpart: spsim allocates and frees per
 * call. */
void spsim_b200_release_scratch(void);

/* Seed of the random positions get_Molecule_from_formula draws (the reference
 * draws them from libspimage's p_drand48 stream, which is not available here;
 * no counterpart). */
void spsim_b200_set_formula_seed(unsigned long long seed);

/* Autotuner: the kernel variant used for FP32 forwards: threads per CTA,
 * pixels per thread and form:
 *   0  compensated FP32 phase (hi/lo split), one pixel per lane
 *   1  compensated FP32 phase, pixel pairs in f32x2 instructions
 *   2  FP64 phase and half-cycle reduction, FP32 sin/cos and sums on pixel
 *      pairs (f32x2); free of the compensated forms' phase range limit
 *      (SPSIM_ERR_RANGE); the SPSIM_PREC_F32_FAST default
 *   3  form 2 on the first pixel of each neighbour pair (pixels 2m, 2m+1),
 *      the second pixel's phase as the first's plus (q_b - q_a).r in FP32;
 *      used where |q_b - q_a| |r|max <= 1/8 cycle for every pair of the q
 *      set (detector rows of even width)
 *   4  form 2 on the second pixel of each neighbour quad (pixels 4m..4m+3),
 *      the other three as its phase plus (q - q_a).r in FP32 (with
 *      SPSIM_PREC_F32_FAST the sin/cos of pixels 4m+2 and 4m+3 on MUFU, the
 *      rest on FMA-pipe polynomials); the default of both FP32 precisions,
 *      used where every one-pixel step from a quad's anchor stays within 1/8
 *      cycle of |r|max and every two-pixel step within 0.16 cycle (detector
 *      rows of width divisible by 4), else form 3 (SPSIM_PREC_F32), else
 *      form 2
 * Forms 2, 3 and 4 read the reduced phase from a fixed-point phase word (three
 * FP64 FMAs) while |q|max |r - centre|max < 2^17 cycles, and reduce by FP64
 * rounding (six FP64 operations, up to 2^48 cycles) beyond.
 * threads < 0 restores automatic choice; autotune times every compiled
 * variant on the given workload and keeps the fastest for workloads of that
 * size class. */
int spsim_b200_set_variant(int threads, int pixels_per_thread, int form);
/* The kernel variant the last forward on this thread ran: threads per CTA,
 * pixels per thread and form (-1 for the plain FP64 kernel). */
int spsim_b200_last_variant(int *threads, int *pixels_per_thread, int *form);
/* Whether the last forward on this thread (forms 2, 3 and 4) took the phase from
 * the fixed-point phase word (1) or reduced it by FP64 rounding (0); 0 for the
 * other forms and the plain FP64 kernel.  No reference counterpart. */
int spsim_b200_last_phase_word(int *on);
/* Whether the last forward on this thread ran the neighbour-pair form with
 * every pair's step within 0.07 cycle, or the neighbour-quad form with every
 * one-pixel step within 0.07 cycle, so that those pixels took the shorter
 * NARROW sin/cos polynomial (1), or not (0).  No reference counterpart. */
int spsim_b200_last_pair_narrow(int *on);
int spsim_b200_autotune(const spsim_b200_molecule *m, const spsim_b200_qset *qs, int precision, void *stream,
                        int *best_threads, int *best_pixels_per_thread, int *best_form);
/* The same over a batch (the arguments of spsim_b200_forward_batch, without
 * B and outputs): every variant is timed on the whole batched launch, and the
 * fastest is kept for batches of that size class (total atom.pixel terms).
 * No reference counterpart. */
int spsim_b200_autotune_batch(int npatterns, const spsim_b200_molecule *const *mols,
                              const spsim_b200_qset *const *qsets, const double *rot, int precision, void *stream,
                              int *best_threads, int *best_pixels_per_thread, int *best_form);
/* Forget every autotuned choice (later forwards use the untuned defaults
 * again).  No reference counterpart. */
int spsim_b200_clear_tuning(void);

#ifdef __cplusplus
}
#endif

#endif
