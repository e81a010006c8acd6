// pm_kernels.h -- host-callable launchers of the PM kernels (internal).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pm_common.cuh"

namespace hyowon {

// One particle set in structure-of-arrays form.
struct ParticlesF64 {
    double* x;
    double* y;
    double* z;
    double* px;
    double* py;
    double* pz;
};

struct SortWork {
    uint32_t* key;      // bucket of each particle (n)
    uint32_t* rank;     // position of the particle inside its bucket (n)
    uint32_t* count;    // particles per bucket (n_buckets)
    uint32_t* offset;   // exclusive prefix of count (n_buckets + 1)
    uint32_t* scan_tmp; // scratch for the multi-level scan
    uint32_t n_buckets;
    int shift;          // bucket = cell_index >> shift
};

// ---- sort (pm_sort.cu) ----------------------------------------------------
size_t scan_tmp_elements(uint32_t n_buckets);
// Returns the number of kernels launched.
int launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n,
                          uint32_t* tmp, cudaStream_t s);
void launch_scatter_u32(uint32_t n, const uint32_t* key, const uint32_t* rank,
                        const uint32_t* offset, const uint32_t* src, uint32_t* dst,
                        const unsigned int* status, cudaStream_t s);
void launch_scatter_f64(uint32_t n, const uint32_t* key, const uint32_t* rank,
                        const uint32_t* offset, const double* src, double* dst,
                        const unsigned int* status, cudaStream_t s);
void launch_unpermute_f64(uint32_t n, const uint32_t* id, const double* src, double* dst,
                          cudaStream_t s);
void launch_scatter_multi(uint32_t n, const uint32_t* key, const uint32_t* rank,
                          const uint32_t* offset, int n_f64, const double* const* src,
                          double* const* dst, int n_u32, const uint32_t* const* src_u,
                          uint32_t* const* dst_u, const unsigned int* status,
                          cudaStream_t s);
void launch_scatter4_multi(uint32_t n, const uint32_t* key, const uint32_t* rank,
                           const uint32_t* offset, int count, const uint32_t* const* src,
                           uint32_t* const* dst, const unsigned int* status, cudaStream_t s);
void launch_iota_u32(uint32_t n, uint32_t* out, cudaStream_t s);
// order[offset[key[i]] + rank[i]] = i: the cell order of unmoved particles.
void launch_order(uint32_t n, const uint32_t* key, const uint32_t* rank, const uint32_t* offset,
                  uint32_t* order, const unsigned int* status, cudaStream_t s);

// ---- FP64 form (pm_fp64.cu) -----------------------------------------------
void launch_validate_inputs_f64(uint32_t n, const double* x, const double* y,
                                const double* z, const double* mass, unsigned int* status,
                                cudaStream_t s);
void launch_key_f64(uint32_t n, const ParticlesF64& p, Axis a, const SortWork& w,
                    unsigned int* status, cudaStream_t s);
void launch_kick_drift_key_f64(uint32_t n, const ParticlesF64& cur, const double* ax,
                               const double* ay, const double* az, double K1, double D,
                               Axis a, const ParticlesF64& cand, const SortWork& w,
                               bool with_key, unsigned long long* max_drift_bits,
                               unsigned int* status, cudaStream_t s);
void launch_deposit_f64(uint32_t n, const ParticlesF64& p, const double* mass,
                        double uniform_mass, Axis a, double* mesh, unsigned int* status,
                        cudaStream_t s);
// Deterministic owner-computes deposit (k_deposit_tiles): mesh written whole,
// no zeroing needed. Needs the bucket offsets of the deposited set in w, the
// cell order `order` (or null when the arrays are in cell order), the largest
// bucket count in *max_count (and its value on the host, which picks the
// kernel) and e_max = deposit_mass_exponent_f64(max mass).
int deposit_mass_exponent_f64(double max_mass);
// With `modes` non-null (a power-of-two mesh of 32 to 2048), the tiles are
// transformed along z and stored to that chunked half spectrum (twiddles `tw`)
// instead of `mesh`: the five-pass solve then continues with its column passes.
cudaError_t launch_deposit_tiles_f64(const ParticlesF64& p, const double* mass,
                                     double uniform_mass, const uint32_t* order,
                                     const SortWork& w, Axis a, const uint32_t* max_count,
                                     uint32_t max_count_host, int e_max, double* mesh,
                                     double2* modes, const double2* tw, unsigned int* status,
                                     cudaStream_t s);
void launch_max_count_f64(uint32_t n_buckets, const uint32_t* count, uint32_t* max_count,
                          cudaStream_t s);
void launch_green_f64(int N, double2* modes, const double* lap, const double* win,
                      double four_pi_G, double scale, int deconvolve, double input_mass,
                      double mass_tolerance, unsigned int* status, cudaStream_t s);
void launch_green_spectral_f64(int N, double L, double2* modes, const double* win,
                               double four_pi_G, double scale, double r_s,
                               double input_mass, double mass_tolerance,
                               unsigned int* status, cudaStream_t s);
void launch_spectral_axis_f64(int N, double L, int axis, const double2* phi_k,
                              double2* out_k, cudaStream_t s);
void launch_interp_add_f64(uint32_t n, const double* field, const ParticlesF64& p,
                           Axis a, double* out, unsigned int* status, cudaStream_t s);
void launch_gather_kick_f64(uint32_t n, const double* phi, const ParticlesF64& p,
                            double* ax, double* ay, double* az, int do_kick, double K2,
                            double* pxo, double* pyo, double* pzo, Axis a,
                            unsigned int* status, cudaStream_t s);
void launch_kick_only_f64(uint32_t n, const ParticlesF64& p, const double* ax,
                          const double* ay, const double* az, double K2, double* pxo,
                          double* pyo, double* pzo, unsigned int* status, cudaStream_t s);
void launch_cell_coords_f64(uint32_t n, const double* pos, Axis a, int64_t* base,
                            double* frac, unsigned int* status, cudaStream_t s);

}  // namespace hyowon
