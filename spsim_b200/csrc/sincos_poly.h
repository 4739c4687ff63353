/* Generated by gen_sincos_poly.py (Remez minimax, float32 coefficients).
 * sin(2 pi y) ~ y * sum_k S_k (y^2)^k,  cos(2 pi y) ~ sum_k C_k (y^2)^k. */
#ifndef SPSIM_B200_SINCOS_POLY_H
#define SPSIM_B200_SINCOS_POLY_H
/* HALF: |y| <= 0.312500 cycles; float32 evaluation error vs float64:
 *   sin max 2.595e-07 rms 6.101e-08, cos max 1.184e-07 rms 2.720e-08 */
#define SPSIM_HALF_YMAX 3.125000000e-01f
#define SPSIM_HALF_SIN_DEG 6
#define SPSIM_HALF_COS_DEG 6
#define SPSIM_HALF_S0 6.283185482e+00f
#define SPSIM_HALF_S1 -4.134169769e+01f
#define SPSIM_HALF_S2 8.160501862e+01f
#define SPSIM_HALF_S3 -7.669766998e+01f
#define SPSIM_HALF_S4 4.191793442e+01f
#define SPSIM_HALF_S5 -1.392658710e+01f
#define SPSIM_HALF_C0 1.000000000e+00f
#define SPSIM_HALF_C1 -1.973920631e+01f
#define SPSIM_HALF_C2 6.493911743e+01f
#define SPSIM_HALF_C3 -8.544470978e+01f
#define SPSIM_HALF_C4 6.000373840e+01f
#define SPSIM_HALF_C5 -2.420245552e+01f
/* QUAD: |y| <= 0.187500 cycles; float32 evaluation error vs float64:
 *   sin max 1.219e-07 rms 2.794e-08, cos max 9.501e-08 rms 2.294e-08 */
#define SPSIM_QUAD_YMAX 1.875000000e-01f
#define SPSIM_QUAD_SIN_DEG 5
#define SPSIM_QUAD_COS_DEG 5
#define SPSIM_QUAD_S0 6.283185482e+00f
#define SPSIM_QUAD_S1 -4.134169769e+01f
#define SPSIM_QUAD_S2 8.160447693e+01f
#define SPSIM_QUAD_S3 -7.665564728e+01f
#define SPSIM_QUAD_S4 4.062243271e+01f
#define SPSIM_QUAD_C0 1.000000000e+00f
#define SPSIM_QUAD_C1 -1.973920441e+01f
#define SPSIM_QUAD_C2 6.493852234e+01f
#define SPSIM_QUAD_C3 -8.538704681e+01f
#define SPSIM_QUAD_C4 5.796249008e+01f
#endif

