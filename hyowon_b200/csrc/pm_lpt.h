// pm_lpt.h -- device 1LPT initial conditions (internal, see pm_lpt.cu).
#pragma once

#include <cuda_runtime.h>

namespace hyowon {

// Writes positions / momenta of the N^3 lattice particles (index (iN+j)N+k)
// into d_pos[3] / d_mom[3]. d_noise (N^3 doubles, device) may be overwritten.
// Returns 0, 6 (CUDA / cuFFT) or 7 (allocation); *err names the failure.
int lpt_ics_device(int N, double L, const double* d_noise, const double* d_xs,
                   const double* d_ys, const double* d_y2, int n_nodes, double pf,
                   double* const d_pos[3], double* const d_mom[3], unsigned int* d_status,
                   cudaStream_t s, const char** err);

// Vector-Jacobian product of the displacement map w.r.t. the noise: given the
// per-particle cotangents g_d (lattice order, N^3 each), writes
// d_grad = sum_d B_d^T g_d = -sum_d B_d g_d (B_d is antisymmetric).
int lpt_adjoint_device(int N, double L, double* const d_g[3], const double* d_xs,
                       const double* d_ys, const double* d_y2, int n_nodes, double* d_grad,
                       cudaStream_t s, const char** err);

}  // namespace hyowon
