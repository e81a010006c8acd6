// pm_diag.cu -- binary64 global diagnostics of the device particle state.
//
// One pass over the particles forms, per particle i, the terms of
//   W  = sum_i m_i phi(x_i)            (CIC-interpolated potential of the last
//                                       force solve; PMForceDiagnostics reports
//                                       0.5 W, src/gravity/pm_solver.cpp:812-840)
//   K  = sum_i 0.5 m_i |p_i|^2          (divided by a^2 on the host,
//                                       src/validation/conservation_checks.cpp:589-625)
//   P  = sum_i m_i p_i,  F = sum_i m_i a_i,  S = sum_i m_i |a_i|
//                                      (force balance |F| / S,
//                                       include/cosmo_nbody/validation/force_balance_diagnostics.hpp:19-27)
//   C  = sum_i m_i p_i . a_i           (ConservationChecks::compute_momentum_force_contraction)
//   D  = sum_i m_i p_i . grad_S phi(x_i) (the directional derivative of the CIC
//                                       particle-position energy along the
//                                       momenta; PMPostForceEnergyDiagnostics,
//                                       src/gravity/pm_post_force_energy_diagnostics.cpp:17-100)
// in binary64 for both arithmetic forms (the precision form widens its FP32
// momenta, accelerations and potential and its fixed-point positions exactly).
//
// The per-particle potential term follows
// CICMassAssignment::interpolate_mass_weighted_sum_full_mesh
// (src/mesh/mass_assignment_gather.inc:283-391) operation for operation:
// value = sum over the 8 corners (x, y, z offsets in that nesting) of
// phi * ((wx * wy) * wz), then m * value. This unit is compiled with
// --fmad=false so those products are not contracted.
//
// The gradient of D is the derivative of the CIC weights, one-sided per cell
// (CICMassAssignment::interpolate_mass_weighted_directional_derivative,
// src/mesh/mass_assignment_directional.cpp:133-166): g_x = sum over (y, z)
// corners of (phi[x+1] - phi[x]) * w_y * w_z, likewise for y and z, times
// 1 / dx; then m (p . g). The reference forms g in long double; here it is
// binary64 (agreement to rounding of each term).
//
// The sums are deterministic run to run: a fixed grid of kBlocks blocks, each
// thread accumulating a grid-stride subsequence with Neumaier compensation,
// fixed shuffle / shared-memory trees inside a block, block partials written
// to their own slots, and one block combining the partials in a fixed tree.
// The summation order differs from the reference's blocked order, so results
// agree with it to rounding (~1e-15 relative), not bit for bit.
#include "pm_diag.h"

namespace hyowon {
namespace diag {

namespace {

struct Acc {
    double s, c;
};

__device__ __forceinline__ void add(Acc& a, double v) {
    const double t = a.s + v;
    if (fabs(a.s) >= fabs(v))
        a.c += (a.s - t) + v;
    else
        a.c += (v - t) + a.s;
    a.s = t;
}

__device__ __forceinline__ void merge(Acc& a, const Acc& b) {
    add(a, b.s);
    a.c += b.c;
}

// Block-wide fixed-order combination of kTerms accumulators; the result is
// valid in thread 0.
__device__ __forceinline__ void block_merge(Acc (&acc)[kTerms]) {
    __shared__ Acc part[kThreads / 32][kTerms];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < kTerms; ++t) {
        for (int o = 16; o > 0; o >>= 1) {
            Acc other;
            other.s = __shfl_down_sync(0xffffffffu, acc[t].s, o);
            other.c = __shfl_down_sync(0xffffffffu, acc[t].c, o);
            if (lane < o) merge(acc[t], other);
        }
        if (lane == 0) part[warp][t] = acc[t];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int t = 0; t < kTerms; ++t) {
            Acc a = part[0][t];
            for (int w = 1; w < kThreads / 32; ++w) merge(a, part[w][t]);
            acc[t] = a;
        }
    }
}

__device__ __forceinline__ void store_partial(const Acc (&acc)[kTerms], double* partial) {
    if (threadIdx.x == 0) {
#pragma unroll
        for (int t = 0; t < kTerms; ++t) {
            partial[(static_cast<size_t>(blockIdx.x) * kTerms + t) * 2] = acc[t].s;
            partial[(static_cast<size_t>(blockIdx.x) * kTerms + t) * 2 + 1] = acc[t].c;
        }
    }
}

// One-sided CIC-weight gradient of the 8 corner values v[x][y][z] (weights
// w*[0] = 1 - f, w*[1] = f), dotted with p, times 1/dx.
__device__ __forceinline__ double directional(const double (&v)[2][2][2], const double (&wx)[2],
                                              const double (&wy)[2], const double (&wz)[2],
                                              double inv_dx, double px, double py, double pz) {
    double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            gx += (v[1][a][b] - v[0][a][b]) * wy[a] * wz[b];
            gy += (v[a][1][b] - v[a][0][b]) * wx[a] * wz[b];
            gz += (v[a][b][1] - v[a][b][0]) * wx[a] * wy[b];
        }
    }
    return px * (gx * inv_dx) + py * (gy * inv_dx) + pz * (gz * inv_dx);
}

// Per-particle terms shared by both forms; `value` is the CIC sum of phi and
// `dir` the directional derivative along p.
__device__ __forceinline__ void particle_terms(Acc (&acc)[kTerms], double m, double value,
                                               double dir, double px, double py, double pz,
                                               double ax, double ay, double az) {
    add(acc[0], m * value);
    add(acc[1], 0.5 * m * (px * px + py * py + pz * pz));
    add(acc[2], m * px);
    add(acc[3], m * py);
    add(acc[4], m * pz);
    add(acc[5], m * ax);
    add(acc[6], m * ay);
    add(acc[7], m * az);
    add(acc[8], m * sqrt(ax * ax + ay * ay + az * az));
    add(acc[9], m * (px * ax + py * ay + pz * az));
    add(acc[10], m * dir);
}

__global__ void __launch_bounds__(kThreads)
k_diag_f64(InputsF64 in, double* __restrict__ partial, unsigned int* status) {
    Acc acc[kTerms];
#pragma unroll
    for (int t = 0; t < kTerms; ++t) acc[t] = Acc{0.0, 0.0};
    const int N = in.axis.N;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < in.n; i += kBlocks * kThreads) {
        const double m = in.mass ? in.mass[i] : in.uniform_mass;
        double value = 0.0, dir = 0.0;
        if (in.phi) {
            int b[3];
            double f[3];
            const double pos[3] = {in.x[i], in.y[i], in.z[i]};
            bool ok = true;
#pragma unroll
            for (int d = 0; d < 3; ++d) ok &= cic_coord_f64(pos[d], in.axis, b[d], f[d]);
            if (!ok) {
                raise_status(status, ST_CELL_ESCAPE);
                continue;
            }
            const double wx[2] = {1.0 - f[0], f[0]};
            const double wy[2] = {1.0 - f[1], f[1]};
            const double wz[2] = {1.0 - f[2], f[2]};
            bool lost = false;
            double v[2][2][2];
#pragma unroll
            for (int ox = 0; ox < 2; ++ox) {
                const size_t gx = static_cast<size_t>(wrap_index(b[0] + ox, N));
#pragma unroll
                for (int oy = 0; oy < 2; ++oy) {
                    const size_t gy = static_cast<size_t>(wrap_index(b[1] + oy, N));
#pragma unroll
                    for (int oz = 0; oz < 2; ++oz) {
                        const size_t gz = static_cast<size_t>(wrap_index(b[2] + oz, N));
                        const double fv = in.phi[(gx * N + gy) * N + gz];
                        v[ox][oy][oz] = fv;
                        const double xy = wx[ox] * wy[oy];
                        const double w = xy * wz[oz];
                        if (w == 0.0 && wx[ox] != 0.0 && wy[oy] != 0.0 && wz[oz] != 0.0 && fv != 0.0
                            && m != 0.0)
                            lost = true;
                        const double contribution = fv * w;
                        if (fv != 0.0 && w != 0.0 && contribution == 0.0 && m != 0.0) lost = true;
                        value += contribution;
                    }
                }
            }
            if (lost || (m != 0.0 && value != 0.0 && m * value == 0.0))
                raise_status(status, ST_UNDERFLOW);
            dir = directional(v, wx, wy, wz, 1.0 / in.axis.dx, in.px[i], in.py[i], in.pz[i]);
        }
        particle_terms(acc, m, value, dir, in.px[i], in.py[i], in.pz[i], in.ax[i], in.ay[i],
                       in.az[i]);
    }
    block_merge(acc);
    store_partial(acc, partial);
}

__global__ void __launch_bounds__(kThreads)
k_diag_f32(InputsF32 in, double* __restrict__ partial) {
    Acc acc[kTerms];
#pragma unroll
    for (int t = 0; t < kTerms; ++t) acc[t] = Acc{0.0, 0.0};
    const uint32_t N = static_cast<uint32_t>(in.N);
    const double m = in.uniform_mass;
    constexpr double kInv32 = 1.0 / 4294967296.0;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < in.n; i += kBlocks * kThreads) {
        double value = 0.0, dir = 0.0;
        const double px = static_cast<double>(in.px[i]), py = static_cast<double>(in.py[i]),
                     pz = static_cast<double>(in.pz[i]);
        if (in.phi) {
            // u * N = cell * 2^32 + fraction * 2^32 exactly in 64 bits
            const unsigned long long qx = static_cast<unsigned long long>(in.ux[i]) * N;
            const unsigned long long qy = static_cast<unsigned long long>(in.uy[i]) * N;
            const unsigned long long qz = static_cast<unsigned long long>(in.uz[i]) * N;
            const uint32_t b[3] = {static_cast<uint32_t>(qx >> 32), static_cast<uint32_t>(qy >> 32),
                                   static_cast<uint32_t>(qz >> 32)};
            const double f[3] = {static_cast<double>(static_cast<uint32_t>(qx)) * kInv32,
                                 static_cast<double>(static_cast<uint32_t>(qy)) * kInv32,
                                 static_cast<double>(static_cast<uint32_t>(qz)) * kInv32};
            const double wx[2] = {1.0 - f[0], f[0]};
            const double wy[2] = {1.0 - f[1], f[1]};
            const double wz[2] = {1.0 - f[2], f[2]};
            double v[2][2][2];
#pragma unroll
            for (int ox = 0; ox < 2; ++ox) {
                const size_t gx = b[0] + ox == N ? 0 : b[0] + ox;
#pragma unroll
                for (int oy = 0; oy < 2; ++oy) {
                    const size_t gy = b[1] + oy == N ? 0 : b[1] + oy;
#pragma unroll
                    for (int oz = 0; oz < 2; ++oz) {
                        const size_t gz = b[2] + oz == N ? 0 : b[2] + oz;
                        const double fv = static_cast<double>(in.phi[(gx * N + gy) * N + gz]);
                        v[ox][oy][oz] = fv;
                        value += fv * ((wx[ox] * wy[oy]) * wz[oz]);
                    }
                }
            }
            dir = directional(v, wx, wy, wz, in.inv_dx, px, py, pz);
        }
        particle_terms(acc, m, value, dir, px, py, pz, in.ax[i], in.ay[i], in.az[i]);
    }
    block_merge(acc);
    store_partial(acc, partial);
}

// One block: partial slots 0..kBlocks-1 combined in a fixed tree; the kTerms
// results (sum + compensation) go to out.
__global__ void __launch_bounds__(kThreads)
k_diag_finish(const double* __restrict__ partial, double* __restrict__ out) {
    Acc acc[kTerms];
#pragma unroll
    for (int t = 0; t < kTerms; ++t) acc[t] = Acc{0.0, 0.0};
    for (int b = threadIdx.x; b < kBlocks; b += kThreads) {
#pragma unroll
        for (int t = 0; t < kTerms; ++t) {
            const Acc p{partial[(static_cast<size_t>(b) * kTerms + t) * 2],
                        partial[(static_cast<size_t>(b) * kTerms + t) * 2 + 1]};
            merge(acc[t], p);
        }
    }
    block_merge(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int t = 0; t < kTerms; ++t) out[t] = acc[t].s + acc[t].c;
    }
}

}  // namespace

int launch_f64(const InputsF64& in, double* scratch, unsigned int* status, cudaStream_t s) {
    k_diag_f64<<<kBlocks, kThreads, 0, s>>>(in, scratch, status);
    k_diag_finish<<<1, kThreads, 0, s>>>(scratch, scratch + partial_doubles());
    return cudaPeekAtLastError() == cudaSuccess ? 2 : -1;
}

int launch_f32(const InputsF32& in, double* scratch, cudaStream_t s) {
    k_diag_f32<<<kBlocks, kThreads, 0, s>>>(in, scratch);
    k_diag_finish<<<1, kThreads, 0, s>>>(scratch, scratch + partial_doubles());
    return cudaPeekAtLastError() == cudaSuccess ? 2 : -1;
}

}  // namespace diag
}  // namespace hyowon
