/*
 * fft3d.h -- CPU 3-D real<->half-complex FFT used ONLY as test infrastructure.
 *
 * This is the oracle's FFT: it stands in for FFTW3, which the reference links
 * (src/mesh/fft_backend.cpp:1088-1145) but which is absent here. Conventions
 * follow the reference FFTBackend (include/cosmo_nbody/mesh/fft_backend.hpp:1-3):
 *   - forward r2c is unnormalised;
 *   - inverse c2r is followed by a multiply by norm = 1.0/(N*N*N)
 *     (src/mesh/fft_backend.cpp:784,1118-1130);
 *   - half-complex layout iz + (N/2+1)*(iy + N*ix)
 *     (include/cosmo_nbody/mesh/mesh_geometry.hpp:90-96);
 *   - real layout (ix*N + iy)*N + iz (mesh_geometry.hpp:74-79).
 * Complex values are interleaved (re, im) doubles.
 *
 * Written from the mathematics (radix-2 Cooley-Tukey, two-for-one real
 * packing); any N >= 1 is accepted, non-powers of two use a direct DFT.
 */
#ifndef HYOWON_ORACLE_FFT3D_H
#define HYOWON_ORACLE_FFT3D_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* out[N*N*(N/2+1)*2] = unnormalised r2c of in[N*N*N]. */
void orc_fft3d_r2c(size_t N, const double* in, double* out);

/* out[N*N*N] = c2r of in (Hermitian half spectrum), NOT normalised. `in` is
 * left unchanged. Imaginary parts of self-conjugate modes are ignored as an
 * FFTW c2r does. */
void orc_fft3d_c2r(size_t N, const double* in, double* out);

/* As orc_fft3d_c2r but transforms in place in `in`, which is destroyed (the
 * FFTW c2r contract the reference relies on, fft_backend.cpp:1133-1145). */
void orc_fft3d_c2r_destroy(size_t N, double* in, double* out);

/* 1-D complex transform of length n, in place, sign = -1 forward / +1 inverse,
 * unnormalised. Exposed for the naive-DFT cross-check in tests. */
void orc_fft1d(size_t n, double* data, int sign);

#ifdef __cplusplus
}
#endif
#endif
