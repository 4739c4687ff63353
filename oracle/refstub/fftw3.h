/* Test infrastructure only: spsim's src/diffraction.c names fftw_complex in
 * two helpers that the hot path never calls; this is the one type it needs. */
#ifndef SPSIM_ORACLE_FFTW3_STUB_H
#define SPSIM_ORACLE_FFTW3_STUB_H
typedef double fftw_complex[2];
#endif
