/*
 * Crystal lattice of the reference (src/crystal.c): the cell matrix from the
 * options' cell lengths and angles, and the lattice sum of a pattern.  The
 * cell arithmetic follows the reference's float expressions (same order,
 * built with -ffp-contract=off); the lattice sum runs on the GPU in FP64
 * (spsim_b200_crystal_lattice_sum).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <cuda_runtime.h>

#include "../../../include/spsim.h"
#include "../../../include/spsim_b200.h"

/* src/crystal.c:4-21 */
void crystal_axis_to_cartesian(Options *opts, CrystalAxis axis, float *x, float *y, float *z) {
  const float pi = 3.14159265;
  const float grad_to_rad = pi / 180.0;
  const float *c = opts->crystal_cell;
  if (axis == CrystalA) {
    *x = c[0];
    *y = 0;
    *z = 0;
  } else if (axis == CrystalB) {
    *x = cos(c[5] * grad_to_rad) * c[1];
    *y = sin(c[5] * grad_to_rad) * c[1];
    *z = 0;
  } else if (axis == CrystalC) {
    *x = c[2] * cos(c[4] * grad_to_rad);
    *y = c[2] * (cos(c[3] * grad_to_rad) - cos(c[4] * grad_to_rad) * cos(c[5] * grad_to_rad)) / sin(c[5] * grad_to_rad);
    *z = sqrt(c[2] * c[2] - (*x) * (*x) - (*y) * (*y));
  }
}

/* src/crystal.c:23-37: rows A, B, C */
void crystal_cell_matrix(Options *opts, float *matrix) {
  crystal_axis_to_cartesian(opts, CrystalA, &matrix[0], &matrix[1], &matrix[2]);
  crystal_axis_to_cartesian(opts, CrystalB, &matrix[3], &matrix[4], &matrix[5]);
  crystal_axis_to_cartesian(opts, CrystalC, &matrix[6], &matrix[7], &matrix[8]);
}

static void check(const char *where, int st) {
  if (st) {
    fprintf(stderr, "spsim_b200: %s failed: %s (%s)\n", where, spsim_b200_status_string(st), spsim_b200_last_error());
    abort();
  }
}

static void cuda_check(const char *where, cudaError_t e) {
  if (e != cudaSuccess) {
    fprintf(stderr, "spsim_b200: %s failed: %s\n", where, cudaGetErrorString(e));
    abort();
  }
}

/* src/crystal.c:39-71: F <- F * (lattice factor) over crystal_size cells,
 * I = |F|^2, host arrays.  The reference prints a progress line per cell;
 * here that line is printed only with verbosity_level > 0. */
void calculate_pattern_from_crystal(float *I, Complex *F, float *HKL_list, int HKL_list_size, Options *opts) {
  float cell[9];
  crystal_cell_matrix(opts, cell);
  const long long n = HKL_list_size > 0 ? HKL_list_size : 0;
  if (opts->verbosity_level > 0) {
    const int cells = opts->crystal_size[0] * opts->crystal_size[1] * opts->crystal_size[2];
    for (int k = 0; k < cells; k++) printf("%f%% done\n", 100.0 * k / cells);
  }
  if (!n) return;
  float *dq = NULL, *dF = NULL, *dI = NULL;
  cuda_check("cudaMalloc", cudaMalloc((void **)&dq, 3 * n * sizeof(float)));
  cuda_check("cudaMalloc", cudaMalloc((void **)&dF, 2 * n * sizeof(float)));
  cuda_check("cudaMalloc", cudaMalloc((void **)&dI, n * sizeof(float)));
  cuda_check("cudaMemcpy", cudaMemcpy(dq, HKL_list, 3 * n * sizeof(float), cudaMemcpyHostToDevice));
  cuda_check("cudaMemcpy", cudaMemcpy(dF, F, 2 * n * sizeof(float), cudaMemcpyHostToDevice));
  check("calculate_pattern_from_crystal",
        spsim_b200_crystal_lattice_sum(n, dq, cell, opts->crystal_size[0], opts->crystal_size[1],
                                       opts->crystal_size[2], dF, dI, NULL));
  cuda_check("cudaMemcpy", cudaMemcpy(F, dF, 2 * n * sizeof(float), cudaMemcpyDeviceToHost));
  cuda_check("cudaMemcpy", cudaMemcpy(I, dI, n * sizeof(float), cudaMemcpyDeviceToHost));
  cudaFree(dq);
  cudaFree(dF);
  cudaFree(dI);
}
