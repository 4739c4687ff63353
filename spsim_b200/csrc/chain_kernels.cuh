// Detector-chain kernels (internal C++ interface).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace spsim {

// Scalars of the chain, with the reference's derived constants precomputed on
// the host in the reference's own precision.
struct ChainDev {
  int nx, ny, nz, bx, by, bz;
  int spherical, polarization;
  int unbinned;          // bx == by == bz == 1
  int clamp;
  double width, height, distance, cx, cy, pw, ph;
  float beam_intensity;
  float qe;
  float epp;             // electrons per photon for counts (1 when e_hole == 0), src/amplification.c:57-61
  float epp_noiseless;   // hc/lambda/e_hole as float, src/amplification.c:123
  float dark_t;          // dark_current * exposure_time (float product)
  float readout;
  float adc;             // maximum_value / linear_full_well when both set, else 1
  float maxv;
  uint64_t seed;
  uint32_t pattern;
  long long i0, i1;      // pixels [i0, i1) of the fused chain (row ranges of a pipelined shot)
  long long b0, b1;      // bins [b0, b1) of the binning pass
};

struct ChainOut {
  float *thomson, *solid_angle, *photons, *counts, *electrons, *real_out, *noiseless;
};

cudaError_t launch_chain(const ChainDev &c, const float *I, const ChainOut &o, float *scratch_ph, float *scratch_el,
                         cudaStream_t st);
cudaError_t launch_photons(long long n, const float *T, const float *Om, const float *I, float I0, float *out,
                           cudaStream_t st);
cudaError_t launch_counts(const ChainDev &c, const float *ph, float *out, cudaStream_t st);
cudaError_t launch_electrons(const ChainDev &c, const float *cnt, float *out, cudaStream_t st);
cudaError_t launch_binned(const ChainDev &c, const float *electrons, const float *photons, float *real_out,
                          float *noiseless, cudaStream_t st);
cudaError_t launch_poisson(long long n, const float *lam, uint64_t seed, uint32_t pattern, float *out,
                           cudaStream_t st);

}  // namespace spsim
