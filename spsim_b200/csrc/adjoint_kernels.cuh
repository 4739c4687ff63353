// Adjoint kernels (internal C++ interface).
#pragma once

#include "sf_device.cuh"

namespace spsim {

constexpr int ADJ_THREADS = 128;
constexpr int ADJ_ATOMS_PER_THREAD = 2;
constexpr int ADJ_BLOCK_ATOMS = ADJ_THREADS * ADJ_ATOMS_PER_THREAD;
constexpr int ADJ_DPHASE_ATOMS_PER_THREAD = 4;
constexpr int ADJ_DPHASE_BLOCK_ATOMS = ADJ_THREADS * ADJ_DPHASE_ATOMS_PER_THREAD;

// atoms [atom_begin, atom_end): of element `elem`, or, in the FP64-phase
// adjoint's blocks, of `elem` below `split` and of `elem2` from `split` on
// (elem2 < 0: one element)
struct AdjBlock {
  int atom_begin, atom_end, elem, elem2, split, pad;
};

struct AdjItem {    // one CTA: an atom block x a range of (pattern, pixel) indices
  int block, pad;
  long long pix_begin, pix_end;
};

struct AdjParams {
  const float4 *atoms;
  const AtomD *atomsd;
  const int *perm;
  const float *wbase;
  const AdjBlock *blocks;
  const AdjItem *items;
  const float *hkl;
  const double *q64;
  const double *rot;   // device, 9 per pattern, or nullptr
  const double *ff;    // [n_elem][npix]
  const float2 *F;     // npat * npix
  const float *G;      // npat * npix
  long long npix;
  double cx, cy, cz;
  float dq, inv_dq;
  int per_atom_b;
  double *dpos, *docc, *dB;
};

// precision_mode: 0 compensated FP32 polynomial, 1 compensated FP32 MUFU,
// 2 plain FP64, 3 FP64 phase with FP32 polynomial (packed over atom pairs),
// 4 the same with the fixed-point phase word (|q.(r - c)| < 2^17 cycles)
cudaError_t launch_adjoint(int precision_mode, const AdjParams &prm, int n_items, cudaStream_t st);
// resident CTAs per SM of the adjoint kernel launch_adjoint picks for this mode
int adjoint_occupancy(int precision_mode, bool perb);

}  // namespace spsim
