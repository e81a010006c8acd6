// pm_ic.h -- generated initial conditions on the device (internal; the C ABI
// is include/hyowon_ic.h, implemented in pm_ic.cu and pm_handle.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "hyowon_ic.h"

namespace hyowon {
namespace ic {

// Resolved generation parameters (hyowon_ic_resolve).
struct Params {
    int N;            // particles per dimension
    int M;            // IC mesh per dimension (multiple of N)
    double L;
    uint64_t seed;
    int K;            // Cartesian support |m_i| <= K
    bool fixed;       // fixed amplitude (stream 1) instead of Gaussian (stream 0)
    bool negate;      // pair_b
    int order;        // 1 or 2
    double p1, x2, p2;
};

// Device status bits of the generator.
enum Status : unsigned int {
    IC_AMPLITUDE = 1u << 0,   // a used amplitude is not finite and positive
    IC_PSI1 = 1u << 1,        // non-finite 1LPT displacement / update
    IC_HESSIAN = 1u << 2,     // non-finite first-order Hessian
    IC_SOURCE = 1u << 3,      // non-finite 2LPT source
    IC_PSI2 = 1u << 4,        // non-finite 2LPT displacement / update
};

// Host. Returns a hyowon_status; *err names the failure.
int resolve(const hyowon_ic_params_t* in, Params* out, const char** err);
int mode_amplitudes(uint64_t M, double L, uint64_t n, const double* power, double* amp,
                    const char** err);
// Validates power[0 .. 3K^2] and uploads the amplitude table {sqrt(var),
// sqrt(var/2)} per s; *d_amp is a new device allocation on success.
int upload_amplitudes(const Params& p, uint64_t n_power, const double* power, double2** d_amp,
                      const char** err);
// Maps the status word to a hyowon_status and message (0 when clean).
int status_code(unsigned int st, const char** err);

// Device. RandomField::generate into d_modes (M * M * (M/2+1)): row-major
// when cc == 0, else the five-pass transform's chunked layout with cc kz
// columns per chunk (poisson::chunk_columns_f64).
int field_device(const Params& p, const double2* d_amp, double2* d_modes, unsigned int* d_status,
                 cudaStream_t s, const char** err, int cc = 0);
// Work arrays and plans of a 2LPT generation on a power-of-two IC mesh
// (about four IC-mesh fields), kept between generations of the same (N, M, L)
// by whoever owns the workspace.
struct Workspace;
Workspace* workspace_create();
void workspace_destroy(Workspace* w);

// The whole generate branch into d_pos[3] / d_mom[3] (N^3 each, particle order).
// With ws, the work arrays come from (and stay in) ws; else they are
// allocated and freed within the call.
int generate_device(const Params& p, const double2* d_amp, double* const d_pos[3],
                    double* const d_mom[3], unsigned int* d_status, cudaStream_t s,
                    const char** err, Workspace* ws = nullptr);

}  // namespace ic
}  // namespace hyowon
