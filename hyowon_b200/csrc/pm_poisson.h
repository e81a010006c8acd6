// pm_poisson.h -- the pure-PM potential solve on power-of-two meshes
// (internal interface): mass mesh -> r2c -> Green's multiply -> c2r, as five
// passes over HBM instead of separate transforms and a Green's kernel.
//
//   forward : z pass (real rows -> half-complex rows, r2c of each row) and
//             y pass (complex transform of every y column),
//   green   : x pass (forward x transform, Green's multiply in registers,
//             inverse x transform),
//   inverse : y pass (inverse) and z pass (c2r of each row).
//
// The half spectrum between the passes is kz-chunk-major (see pm_poisson.cu);
// results equal an unnormalised r2c / c2r pair with the Green's multiply
// between them.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace hyowon {
namespace poisson {

// Power of two in [32, 2048].
bool supported(int N);

// Complex elements the half-spectrum buffer must hold (N^2 (N/2+1) rounded up
// to whole kz chunks).
size_t modes_elements_f64(int N);
size_t modes_elements_f32(int N);

// TMA tensor maps of one half-spectrum buffer (built on the host once per
// buffer). create_plan returns nullptr and sets *err on failure.
struct Plan;
Plan* create_plan(int N, bool fp32, void* modes, const char** err);
void destroy_plan(Plan* p);
// Polls of each pipeline wait before a block of a column pass gives up with
// ST_PIPELINE (default 2^24; tests lower it to exercise the failure path).
void set_wait_limit(Plan* p, unsigned polls);

// exp(-2 pi i m / N) for m < N as (re, im) pairs, rounded from long double.
void twiddles(int N, double* re_im);

// Pure-PM Green's function of the binary64 form, evaluated exactly as the
// separate Green's kernel does (src/mesh/green_function.cpp:165-207): mode
// (0,0,0) carries the deposited mass, which is checked against input_mass and
// then zeroed.
struct GreenF64 {
    const double* lap;
    const double* win;
    double four_pi_G;
    double scale;
    int deconvolve;
    double input_mass;
    double mass_tol;
    unsigned int* status;
};

// Precision form: factor *c_green / (lap sum) [/ W^2], mode (0,0,0) zeroed.
struct GreenF32 {
    const float* lap;
    const float* win;
    int deconvolve;
    const float* c_green;
};

// Kz columns per chunk of the FP64 chunked half spectrum: element
// (kx, ky, kz) of an N^3 transform sits at
// (kz / CC) N^2 CC + (kx N + ky) CC + kz % CC.
int chunk_columns_f64(int N);

// One Hessian field of the 2LPT source of the IC generator
// (LPTDisplacement, src/ic/lpt_displacement.cpp:386-520): H_ab = c2r(d k_a k_b /
// k^2) from the fully transformed spectrum d (chunked, tensor maps in pd),
// normalised by t.norm and folded into the real accumulators t.acc / t.src
// (SourceTermF64::op), in three passes: the symbol and the inverse x
// transform into `work` (maps in pw), the inverse y transform, and the c2r
// along z whose epilogue does the folding.
struct HessianF64 {
    const double* k;   // k[i] = (2 pi m(i)) / L for array index i (m the signed mode)
    int a, b;
};
struct SourceTermF64 {
    int op;            // 0: acc = h; 1: src = acc h, acc += h; 2: src += acc h; 3: src -= h^2
    int last;          // check the source for finiteness
    double norm;       // 1 / N^3
    double* acc;
    double* src;
    unsigned int* status;
    unsigned int hessian_flag, source_flag;
};
int hessian_source_f64(const Plan* pd, const Plan* pw, int N, double2* work, const double2* tw,
                       const HessianF64& h, const SourceTermF64& t, unsigned int* status,
                       cudaStream_t s);

// Each returns the number of kernels launched, or -1 if a launch failed.
// status receives ST_PIPELINE if a pipelined pass gives up waiting.
int forward_f64(const Plan* p, int N, const double* mass, double2* modes, const double2* tw,
                unsigned int* status, cudaStream_t s);
// The forward pass after the z pass: for spectra whose rows the deposit already
// transformed along z (chunked::rows_r2c in pm_chunk.cuh).
int forward_columns_f64(const Plan* p, int N, double2* modes, const double2* tw,
                        unsigned int* status, cudaStream_t s);
int green_f64(const Plan* p, int N, double2* modes, const double2* tw, const GreenF64& g,
              cudaStream_t s);
int inverse_f64(const Plan* p, int N, double2* modes, double* phi, const double2* tw,
                unsigned int* status, cudaStream_t s);

int forward_f32(const Plan* p, int N, const float* mesh, float2* modes, const float2* tw,
                unsigned int* status, cudaStream_t s);
int forward_columns_f32(const Plan* p, int N, float2* modes, const float2* tw,
                        unsigned int* status, cudaStream_t s);
int green_f32(const Plan* p, int N, float2* modes, const float2* tw, const GreenF32& g,
              unsigned int* status, cudaStream_t s);
int inverse_f32(const Plan* p, int N, float2* modes, float* phi, const float2* tw,
                unsigned int* status, cudaStream_t s);

}  // namespace poisson
}  // namespace hyowon
