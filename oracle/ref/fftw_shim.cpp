// fftw_shim.cpp -- test infrastructure: an implementation of the reference's
// cosmo_nbody::mesh::FFTBackend (include/cosmo_nbody/mesh/fft_backend.hpp:20-72)
// over this repository's own CPU FFT (oracle/fft3d.c), because FFTW3 is not
// installed here. It keeps the reference's contract:
//   - forward r2c unnormalised (src/mesh/fft_backend.cpp:1088-1100);
//   - inverse c2r then `out *= norm_factor_` with
//     norm_factor_ = 1/(N*N*N) formed as in fft_backend.cpp:784-786;
//   - inverse may destroy its complex input (FFTW c2r semantics).
// Only the methods the hot path links are provided.
#include "cosmo_nbody/mesh/fft_backend.hpp"

#include <stdexcept>

extern "C" {
#include "../fft3d.h"
}

namespace cosmo_nbody::mesh {

FFTBackend::FFTBackend(const MeshGeometry& geom, config::ScratchMode,
                       const std::string&)
    : geom_(geom),
      N_(geom.grid_size()),
      real_size_(geom.real_size()),
      complex_size_(geom.complex_size()),
      norm_factor_(1.0 / (static_cast<core::Real>(geom.grid_size())
                          * static_cast<core::Real>(geom.grid_size())
                          * static_cast<core::Real>(geom.grid_size()))),
      forward_plan_(nullptr),
      inverse_plan_(nullptr),
      forward_unaligned_plan_(nullptr),
      inverse_unaligned_plan_(nullptr) {
    if (geom_.local_n0() != N_ || geom_.local_0_start() != 0) {
        throw std::invalid_argument(
            "FFT shim requires single-rank full-mesh geometry");
    }
}

FFTBackend::~FFTBackend() = default;

void FFTBackend::normalize_inverse_buffer(core::Real* out,
                                          std::size_t out_size) const {
    if (!out || out_size != real_size_) {
        throw std::invalid_argument("FFT shim inverse normalization: bad buffer");
    }
#pragma omp parallel for schedule(static) if (out_size >= 32768)
    for (std::size_t i = 0; i < out_size; ++i) out[i] *= norm_factor_;
}

void FFTBackend::forward(RealField& in, ComplexField& out) {
    if (in.size() != real_size_ || out.size() != complex_size_) {
        throw std::invalid_argument("FFT shim forward: invalid field size");
    }
    orc_fft3d_r2c(N_, in.data(), reinterpret_cast<double*>(out.data()));
}

void FFTBackend::forward_external_output(RealField& in,
                                         std::complex<core::Real>* out,
                                         std::size_t out_size) {
    if (in.size() != real_size_ || !out || out_size != complex_size_) {
        throw std::invalid_argument("FFT shim forward_external_output: bad buffer");
    }
    orc_fft3d_r2c(N_, in.data(), reinterpret_cast<double*>(out));
}

void FFTBackend::inverse(ComplexField& in_k, RealField& out_r) {
    if (in_k.size() != complex_size_ || out_r.size() != real_size_) {
        throw std::invalid_argument("FFT shim inverse: invalid field size");
    }
    orc_fft3d_c2r_destroy(N_, reinterpret_cast<double*>(in_k.data()), out_r.data());
    normalize_inverse_buffer(out_r.data(), out_r.size());
}

void FFTBackend::forward_external(core::Real* in, std::size_t in_size,
                                  ComplexField& out) {
    if (!in || in_size != real_size_ || out.size() != complex_size_) {
        throw std::invalid_argument("FFT shim forward_external: bad buffer");
    }
    orc_fft3d_r2c(N_, in, reinterpret_cast<double*>(out.data()));
}

void FFTBackend::inverse_external(ComplexField& in, core::Real* out,
                                  std::size_t out_size) {
    if (in.size() != complex_size_ || !out || out_size != real_size_) {
        throw std::invalid_argument("FFT shim inverse_external: bad buffer");
    }
    orc_fft3d_c2r_destroy(N_, reinterpret_cast<double*>(in.data()), out);
    normalize_inverse_buffer(out, out_size);
}

}  // namespace cosmo_nbody::mesh
