/* Test infrastructure only: spsim's generated build-config header, left empty
 * (no GSL, no NFFT, no MPI, no CUDA) for the CPU reference build. */
