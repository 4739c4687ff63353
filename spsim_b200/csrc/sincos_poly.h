/* Generated by gen_sincos_poly.py (Remez minimax, float32 coefficients).
 * sin(2 pi y) ~ y * sum_k S_k (y^2)^k,  cos(2 pi y) ~ sum_k C_k (y^2)^k. */
#ifndef SPSIM_B200_SINCOS_POLY_H
#define SPSIM_B200_SINCOS_POLY_H
/* HALF: |y| <= 0.312500 cycles; float32 evaluation error vs float64:
 *   sin max 1.987e-07 rms 4.760e-08, cos max 1.627e-07 rms 3.891e-08 */
#define SPSIM_HALF_YMAX 3.125000000e-01f
#define SPSIM_HALF_SIN_DEG 5
#define SPSIM_HALF_COS_DEG 6
#define SPSIM_HALF_S0 6.283185482e+00f
#define SPSIM_HALF_S1 -4.134158325e+01f
#define SPSIM_HALF_S2 8.159436798e+01f
#define SPSIM_HALF_S3 -7.639367676e+01f
#define SPSIM_HALF_S4 3.843774796e+01f
#define SPSIM_HALF_C0 1.000000000e+00f
#define SPSIM_HALF_C1 -1.973920631e+01f
#define SPSIM_HALF_C2 6.493915558e+01f
#define SPSIM_HALF_C3 -8.544567108e+01f
#define SPSIM_HALF_C4 6.001371002e+01f
#define SPSIM_HALF_C5 -2.423987198e+01f
/* QUAD: |y| <= 0.187500 cycles; float32 evaluation error vs float64:
 *   sin max 9.063e-08 rms 2.071e-08, cos max 8.102e-08 rms 2.020e-08 */
#define SPSIM_QUAD_YMAX 1.875000000e-01f
#define SPSIM_QUAD_SIN_DEG 5
#define SPSIM_QUAD_COS_DEG 5
#define SPSIM_QUAD_S0 6.283185482e+00f
#define SPSIM_QUAD_S1 -4.134176636e+01f
#define SPSIM_QUAD_S2 8.161145020e+01f
#define SPSIM_QUAD_S3 -7.691862488e+01f
#define SPSIM_QUAD_S4 4.393268204e+01f
#define SPSIM_QUAD_C0 1.000000000e+00f
#define SPSIM_QUAD_C1 -1.973920631e+01f
#define SPSIM_QUAD_C2 6.493863678e+01f
#define SPSIM_QUAD_C3 -8.539147186e+01f
#define SPSIM_QUAD_C4 5.801905441e+01f
/* DHALF: |y| <= 0.250000 cycles; float32 evaluation error vs float64:
 *   sin max 1.324e-07 rms 2.650e-08, cos max 1.567e-07 rms 4.422e-08 */
#define SPSIM_DHALF_YMAX 2.500000000e-01f
#define SPSIM_DHALF_SIN_DEG 5
#define SPSIM_DHALF_COS_DEG 5
#define SPSIM_DHALF_S0 6.283185482e+00f
#define SPSIM_DHALF_S1 -4.134171295e+01f
#define SPSIM_DHALF_S2 8.160400391e+01f
#define SPSIM_DHALF_S3 -7.660961151e+01f
#define SPSIM_DHALF_S4 3.994231033e+01f
#define SPSIM_DHALF_C0 1.000000000e+00f
#define SPSIM_DHALF_C1 -1.973918152e+01f
#define SPSIM_DHALF_C2 6.493521881e+01f
#define SPSIM_DHALF_C3 -8.525400543e+01f
#define SPSIM_DHALF_C4 5.634064865e+01f
/* WIDE: |y| <= 0.375000 cycles; float32 evaluation error vs float64:
 *   sin max 2.583e-07 rms 4.398e-08, cos max 1.903e-07 rms 3.701e-08 */
#define SPSIM_WIDE_YMAX 3.750000000e-01f
#define SPSIM_WIDE_SIN_DEG 6
#define SPSIM_WIDE_COS_DEG 6
#define SPSIM_WIDE_S0 6.283185482e+00f
#define SPSIM_WIDE_S1 -4.134171677e+01f
#define SPSIM_WIDE_S2 8.160549164e+01f
#define SPSIM_WIDE_S3 -7.670075226e+01f
#define SPSIM_WIDE_S4 4.190143585e+01f
#define SPSIM_WIDE_S5 -1.376170635e+01f
#define SPSIM_WIDE_C0 1.000000000e+00f
#define SPSIM_WIDE_C1 -1.973919868e+01f
#define SPSIM_WIDE_C2 6.493840790e+01f
#define SPSIM_WIDE_C3 -8.542442322e+01f
#define SPSIM_WIDE_C4 5.977695465e+01f
#define SPSIM_WIDE_C5 -2.333224869e+01f
#endif

