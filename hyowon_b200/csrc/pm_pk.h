// pm_pk.h -- binary64 matter power spectrum of device particle positions
// (internal interface of hyowon_pm_power_spectrum).
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

namespace hyowon {
namespace pk {

struct Request {
    int num_bins;
    double max_k_fraction_nyquist;
    bool subtract_shot_noise;
    bool interlaced;
};

struct Bin {
    double k_low, k_mean, k_high, p_raw, p_corrected, mean_deconvolution, shot_noise;
    uint64_t mode_count;
};

// Positions x, y, z (n, binary64, device) in a periodic box of side L on an
// N^3 estimator mesh. weights: device per-particle CIC weights m_i / max m, or
// null for equal masses (weight 1). weight_sum = sum w_i and
// mass_square_fraction = sum w_i^2 / (sum w_i)^2, formed by the caller.
// Fills out[num_bins]; returns a hyowon_status code with *err on failure.
// Allocates its meshes, the transform plan and scratch for the call.
int compute(double L, int N, uint32_t n, const double* x, const double* y, const double* z,
            const double* weights, double weight_sum, double mass_square_fraction,
            const Request& req, Bin* out, std::string* err, cudaStream_t s);

}  // namespace pk
}  // namespace hyowon
