/* Stand-in for FFTW3's header, which is not installed here. The reference's
 * FFTBackend declaration (include/cosmo_nbody/mesh/fft_backend.hpp) only needs
 * the fftw_plan handle type; oracle/ref/fftw_shim.cpp never uses it. */
#ifndef HYOWON_FFTW3_STANDIN_H
#define HYOWON_FFTW3_STANDIN_H
typedef struct fftw_plan_s* fftw_plan;
#endif
