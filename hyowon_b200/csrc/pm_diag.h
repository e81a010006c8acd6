// pm_diag.h -- binary64 global diagnostics of the particle state (internal).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "pm_common.cuh"

namespace hyowon {
namespace diag {

// Terms, in this order: sum m phi, sum 0.5 m |p|^2, sum m p (3), sum m a (3),
// sum m |a|, sum m p.a, sum m p . grad_S phi (one-sided CIC-weight gradient).
constexpr int kTerms = 11;
constexpr int kBlocks = 1024;   // fixed, so the summation order is too
constexpr int kThreads = 256;

// Device scratch of one diagnostics call: block partials (sum, compensation)
// followed by the kTerms results.
constexpr size_t partial_doubles() { return static_cast<size_t>(kBlocks) * kTerms * 2; }
constexpr size_t scratch_doubles() { return partial_doubles() + kTerms; }

struct InputsF64 {
    uint32_t n;
    const double *x, *y, *z, *px, *py, *pz, *ax, *ay, *az;
    const double* mass;     // per particle, or null for uniform_mass
    double uniform_mass;
    const double* phi;      // real-space potential N^3, or null (no potential term)
    Axis axis;
};

struct InputsF32 {
    uint32_t n;
    const uint32_t *ux, *uy, *uz;   // x = u L / 2^32
    const float *px, *py, *pz, *ax, *ay, *az;
    double uniform_mass;
    const float* phi;       // real-space potential N^3, or null
    int N;
    double inv_dx;          // 1 / cell size
};

// Enqueue the pass and the final combination; the kTerms results land at
// scratch + partial_doubles(). Return the number of kernels launched, or -1.
int launch_f64(const InputsF64& in, double* scratch, unsigned int* status, cudaStream_t s);
int launch_f32(const InputsF32& in, double* scratch, cudaStream_t s);

}  // namespace diag
}  // namespace hyowon
