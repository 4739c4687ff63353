// Launch wrappers for the structure-factor kernels (internal C++ interface).
#pragma once

#include "sf_device.cuh"

namespace spsim {


cudaError_t launch_ff_table(const float *hkl, const double *q64, long long npix, int n_elem, const float *coeffs,
                            double B, int delta_atoms, double *ff, cudaStream_t st);
// fixw: the FP64-phase forms (2, 3) take the fixed-point phase word, valid
// while |q|max |r - c|max < 2^18 cycles (the host checks 2^17); narrow: the
// neighbour-pair form (3, FP32 polynomial, fixw) with every pair's step at
// most 0.07 cycle evaluates its second pixels with the NARROW polynomial
cudaError_t launch_sf_f32(int mode, int nt, int p, int packed, bool perb, const SfPattern *pats,
                          const WorkItem *items, int n_items, int *queue, int *err, int grid, cudaStream_t st,
                          bool fixw = false, bool narrow = false);
// The bounded-wait test hook (see g_copy_stall in sf_kernels.cu), current device.
cudaError_t set_copy_stall(int on);
int sf_f32_occupancy(int mode, int nt, int p, int packed, bool perb, bool fixw = false, bool narrow = false);
bool sf_f32_variant_exists(int mode, int nt, int p, int packed);
cudaError_t launch_sf_f64(const SfPattern *pats, int pattern, long long npix, cudaStream_t st);
cudaError_t launch_spectrum_combine(const SfPattern *pats, int pattern0, int S, const double *weight, float *F,
                                    float *I, long long npix, cudaStream_t st);
cudaError_t launch_volume(int nx, int ny, int nz, float width, float height, float depth, float distance, float cx,
                          float cy, float cz, float wavelength, float *out32, cudaStream_t st);
cudaError_t launch_crystal(long long npix, const float *hkl, const double cell[9], int na, int nb, int nc, float *F,
                           float *I, cudaStream_t st);
// q <- R q in float on a device HKL list, bit-identical to the reference's host loop.
cudaError_t launch_rotate_hkl(long long n, const float R[9], float *hkl, cudaStream_t st);
// Neighbour steps of a q set (synchronous, small): steps[0] the largest
// |q[2m+1] - q[2m]| (the pair form's admission), steps[1] the largest step from
// a quad's anchor q[4m+1] to q[4m] or q[4m+2], steps[2] the largest to q[4m+3]
// (the quad form's).
cudaError_t qset_steps(const float *hkl, const double *q64, long long npix, double steps[3]);
// Largest |q| and the neighbour steps of a device float HKL list (scratch4:
// four device words; waits for `st`).
cudaError_t qset_stats(const float *hkl, long long npix, unsigned long long *scratch4, double *qmax, double steps[3],
                       cudaStream_t st);
cudaError_t launch_finalize(const SfPattern *pats, int pattern0, int npat, long long max_npix, cudaStream_t st);
cudaError_t launch_ewald(int nx, int ny, double width, double height, double distance, double cx, double cy,
                         double wavelength, int spherical, float *out32, double *out64, cudaStream_t st);
// Atom records of a new molecule from the caller's positions (float or double),
// arithmetic identical to the host's record building.
template <typename PosT>
cudaError_t launch_atoms_build(float4 *atoms, float4 *atoms2, AtomD *atomsd, const int *perm, int n_padded,
                               const PosT *pos, const float *occ, const float *bfac, const float *wbase,
                               const double c[3], double dr, double inv_dr, cudaStream_t st);
cudaError_t launch_atoms_update(float4 *atoms, float4 *atoms2, AtomD *atomsd, const int *perm, int n_padded, const float *pos32,
                                const double *pos64, const float *occ, const float *bfac, const float *wbase,
                                const double c[3], float dr, float inv_dr, double rbound, int *range_err,
                                cudaStream_t st);

}  // namespace spsim
