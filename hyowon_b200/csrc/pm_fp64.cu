// pm_fp64.cu -- binary64 PM kernels: cell key, K1 kick + drift, CIC deposit,
// Green's function, centred-gradient gather fused with the K2 kick.
//
// Compiled with --fmad=false: every product and sum below rounds exactly as
// the reference's -ffp-contract=off build does, in the reference's operation
// order (cited per kernel). Summation across particles (the deposit) is exact
// fixed-point integer arithmetic rounded once per cell (k_deposit_tiles), so the
// mesh is the same bits run to run whatever order the atomics land in, as the
// reference's plane-ordered sum is; the two differ by the rounding of the
// reference's sequential binary64 sum.
#include <cuda_runtime.h>

#include <cmath>

#include "pm_chunk.cuh"
#include "pm_kernels.h"

namespace hyowon {

namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(uint64_t n, int threads = kThreads) {
    return static_cast<unsigned>((n + threads - 1) / threads);
}

// Row-major cell index; 64-bit because a mesh side above 1625 has more than
// 2^32 cells (the row ix N + iy still fits 32 bits).
__device__ __forceinline__ uint64_t cell_index(int ix, int iy, int iz, int N) {
    const uint32_t row = static_cast<uint32_t>(ix) * static_cast<uint32_t>(N) + static_cast<uint32_t>(iy);
    return static_cast<uint64_t>(row) * static_cast<uint32_t>(N) + static_cast<uint32_t>(iz);
}

// The same in index type IDX: the gather uses 32-bit indices whenever the
// mesh has at most 2^32 cells (fewer registers for its 32 stencil loads).
template <typename IDX>
__device__ __forceinline__ IDX cell_index_t(int ix, int iy, int iz, int N) {
    const uint32_t row = static_cast<uint32_t>(ix) * static_cast<uint32_t>(N) + static_cast<uint32_t>(iy);
    return static_cast<IDX>(row) * static_cast<uint32_t>(N) + static_cast<uint32_t>(iz);
}

inline bool cells_fit_u32(int N) {
    return static_cast<uint64_t>(N) * N * N <= 0xffffffffull;
}

__global__ void k_validate_inputs(uint32_t n, const double* __restrict__ x,
                                  const double* __restrict__ y,
                                  const double* __restrict__ z,
                                  const double* __restrict__ mass,
                                  unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool bad = !isfinite(x[i]) || !isfinite(y[i]) || !isfinite(z[i]);
    if (mass) bad |= !isfinite(mass[i]) || mass[i] < 0.0;
    if (bad) raise_status(status, ST_NONFINITE_INPUT);
}

// Cell key + bucket rank for the current positions.
__global__ void k_key(uint32_t n, const double* __restrict__ x, const double* __restrict__ y,
                      const double* __restrict__ z, Axis a, uint32_t* __restrict__ key,
                      uint32_t* __restrict__ rank, uint32_t* __restrict__ count, int shift,
                      unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int bx, by, bz;
    double fx, fy, fz;
    const bool ok = cic_coord_f64(x[i], a, bx, fx) & cic_coord_f64(y[i], a, by, fy)
        & cic_coord_f64(z[i], a, bz, fz);
    if (!ok) {
        raise_status(status, isfinite(x[i]) && isfinite(y[i]) && isfinite(z[i])
                                 ? ST_CELL_ESCAPE
                                 : ST_NONFINITE_INPUT);
        bx = by = bz = 0;
    }
    const uint32_t b = static_cast<uint32_t>(cell_index(bx, by, bz, a.N) >> shift);
    key[i] = b;
    rank[i] = bucket_rank(count, b);
}

// K1 kick + drift (particle_update.hpp:20-116, leapfrog_integrator.cpp:170-225)
// writing the candidate state, its sort key and the drift telemetry.
// Eight blocks per SM (32 registers): the bucket-rank atomics and the nine
// particle streams are latency-bound, and full occupancy hides them best
// (sort phase at c3 4.04-4.12 ms against 4.39 with the compiler's own choice).
#ifndef HYOWON_KICK64_MINB
#define HYOWON_KICK64_MINB 8
#endif
__global__ void __launch_bounds__(kThreads, HYOWON_KICK64_MINB)
k_kick_drift_key(uint32_t n, const double* __restrict__ x,
                                 const double* __restrict__ y, const double* __restrict__ z,
                                 const double* __restrict__ px, const double* __restrict__ py,
                                 const double* __restrict__ pz, const double* __restrict__ ax,
                                 const double* __restrict__ ay, const double* __restrict__ az,
                                 double K1, double D, Axis a, double* __restrict__ xo,
                                 double* __restrict__ yo, double* __restrict__ zo,
                                 double* __restrict__ pxo, double* __restrict__ pyo,
                                 double* __restrict__ pzo, uint32_t* __restrict__ key,
                                 uint32_t* __restrict__ rank, uint32_t* __restrict__ count,
                                 int shift, int with_key, unsigned long long* max_drift_bits,
                                 unsigned int* status) {
    double drift_max = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double drift_norm = 0.0;
        const double qx = px[i] + ax[i] * K1;
        const double qy = py[i] + ay[i] * K1;
        const double qz = pz[i] + az[i] * K1;
        const double dx = qx * D;
        const double dy = qy * D;
        const double dz = qz * D;
        // add_periodic_displacement: wrap(wrap(x) + minimum_image(d)).
        const double nx = wrap_f64(wrap_f64(x[i], a.L) + minimum_image_f64(dx, a.L), a.L);
        const double ny = wrap_f64(wrap_f64(y[i], a.L) + minimum_image_f64(dy, a.L), a.L);
        const double nz = wrap_f64(wrap_f64(z[i], a.L) + minimum_image_f64(dz, a.L), a.L);
        bool ok = isfinite(qx) && isfinite(qy) && isfinite(qz) && isfinite(dx)
            && isfinite(dy) && isfinite(dz) && isfinite(nx) && isfinite(ny) && isfinite(nz);
        int bx = 0, by = 0, bz = 0;
        if (ok) {
            double fx, fy, fz;
            if (!(cic_coord_f64(nx, a, bx, fx) & cic_coord_f64(ny, a, by, fy)
                  & cic_coord_f64(nz, a, bz, fz))) {
                raise_status(status, ST_CELL_ESCAPE);
                bx = by = bz = 0;
            }
            drift_norm = hypot(hypot(D * qx, D * qy), D * qz);
        } else {
            raise_status(status, ST_KICK_DRIFT);
        }
        xo[i] = nx;
        yo[i] = ny;
        zo[i] = nz;
        pxo[i] = qx;
        pyo[i] = qy;
        pzo[i] = qz;
        if (with_key) {
            const uint32_t b = static_cast<uint32_t>(cell_index(bx, by, bz, a.N) >> shift);
            key[i] = b;
            rank[i] = bucket_rank(count, b);
        }
        drift_max = drift_norm > drift_max ? drift_norm : drift_max;
    }
    // Non-negative doubles order like their bit patterns.
    block_max_to(static_cast<unsigned long long>(__double_as_longlong(drift_max)), max_drift_bits);
}

// CIC deposit (src/mesh/mass_assignment_deposit.inc:193-240): each particle adds
// mass*wx*wy*wz (that product order) to its 8 cells.
__global__ void k_deposit(uint32_t n, const double* __restrict__ x,
                          const double* __restrict__ y, const double* __restrict__ z,
                          const double* __restrict__ mass, double uniform_mass, Axis a,
                          double* __restrict__ mesh, unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (*status & ST_BLOCKS_PUBLISH)) return;
    int ix, iy, iz;
    double tx, ty, tz;
    if (!(cic_coord_f64(x[i], a, ix, tx) & cic_coord_f64(y[i], a, iy, ty)
          & cic_coord_f64(z[i], a, iz, tz))) {
        raise_status(status, ST_CELL_ESCAPE);
        return;
    }
    const double m = mass ? mass[i] : uniform_mass;
    const double wx[2] = {1.0 - tx, tx};
    const double wy[2] = {1.0 - ty, ty};
    const double wz[2] = {1.0 - tz, tz};
    const int N = a.N;
    const int gy[2] = {iy, iy + 1 == N ? 0 : iy + 1};
    const int gz[2] = {iz, iz + 1 == N ? 0 : iz + 1};
#pragma unroll
    for (int ox = 0; ox < 2; ++ox) {
        const int gx = ox == 0 ? ix : (ix + 1 == N ? 0 : ix + 1);
        const double mx = m * wx[ox];
#pragma unroll
        for (int oy = 0; oy < 2; ++oy) {
            const double mxy = mx * wy[oy];
#pragma unroll
            for (int oz = 0; oz < 2; ++oz) {
                atomicAdd(&mesh[cell_index(gx, gy[oy], gz[oz], N)], mxy * wz[oz]);
            }
        }
    }
}

// Deterministic binary64 deposit (CICMassAssignment::deposit,
// src/mesh/mass_assignment_deposit.inc:193-240, whose plane-owned sum is
// deterministic whatever the thread count, :302-333).
//
// Owner-computes tiles: one block per tile of TY mesh rows (x0, y0 .. y0+TY-1,
// all z). Each particle term t = m*wx*wy*wz (the reference's product order, in
// binary64) is converted exactly in scale to fixed point. A cell's contributors
// lie in 8 buckets, so W = 63 - floor(log2(8 max_bucket)) bounds their count by
// 2^(64-W). Two forms, chosen on the device from W (kOneWordMinW below):
//  * one word: q = rint(t 2^(W-1-e)) with m_max < 2^e, summed into one 64-bit
//    shared-memory word per cell (sums below 2^63), quantum 2^(e+1-W) <=
//    2^(e-54) per term;
//  * two words: q = rint(t 2^(62-e)) <= 2^62, split at bit W into hi = q >> W
//    and lo = q mod 2^W, both halves summed into two arrays; every lo sum stays
//    below 2^64, so the cell holds the exact integer sum hi 2^W + lo of its
//    terms, quantum 2^(e-62) per term.
// Integer sums do not depend on the order atomics land in. Each cell is written
// once: the sum correctly rounded to binary64 and scaled by a power of two.
//
// Contributors are the particles whose base cell lies in plane x0 (weight
// 1 - fx) or x0-1 (weight fx) and rows y0-1 .. y0+TY-1: at most four contiguous
// ranges of the cell-ordered particles, found through the bucket starts
// `offset` (`order`: cell-order slot -> particle slot, or null when the arrays
// are in cell order). A bucket can straddle a range edge, so each particle is
// kept only in the range of its own plane and row; the ranges are disjoint in
// (plane, row), so every contributor counts once.
constexpr int kTileThreads = 256;
#ifndef HYOWON_DEPOSIT64_TILE_CELLS
#define HYOWON_DEPOSIT64_TILE_CELLS 4096
#endif
// One-word accumulators: while the densest bucket is small enough that
// W >= kOneWordMinW, a single 64-bit word per cell holds the sum of terms
// quantised to q = rint(t 2^(W-1-e)): a quantum of 2^(e+1-W) <= 2^(e-54), below
// half the binary64 spacing of a full-weight term (t < 2^e). Cell sums stay
// below 2^63. Denser states use the exact two-word (hi/lo) sums. The host reads
// the densest bucket count before the deposit and launches the form that
// applies (the kernel checks the same condition on the device).
constexpr int kOneWordMinW = 55;
// Two words: a hi part is below 2^(62-W) <= c/2 for c = 8 max_bucket
// contributors, so hi sums stay below c^2 / 2 < 2^64 while c < 2^32, i.e.
// W >= 31 (a bucket of fewer than 2^29 particles); beyond that the deposit
// reports ST_CAPACITY.
constexpr int kTwoWordMinW = 31;
// Blocks per SM the deposit tiles' registers are sized for: five (48 registers,
// spilling a little to L1) measured faster than four (64) and three (8.7-8.8 ms
// against 8.9-9.0 and 10.4 at 512^3 / 1024^3).
#ifndef HYOWON_DEPOSIT64_MINB
#define HYOWON_DEPOSIT64_MINB 5
#endif
// Particles each thread loads ahead per pass of the tile loop.
#ifndef HYOWON_DEPOSIT64_BATCH
#define HYOWON_DEPOSIT64_BATCH 2
#endif
constexpr int kDepositBatch = HYOWON_DEPOSIT64_BATCH;

// Tile rows for 8-byte-per-cell accumulators of HYOWON_DEPOSIT64_TILE_CELLS
// cells, halved for the two-word form (same shared memory per tile).
__host__ __device__ constexpr int tile_rows_f64(int N, int words) {
    return HYOWON_DEPOSIT64_TILE_CELLS / words / N < 1 ? 1
         : (HYOWON_DEPOSIT64_TILE_CELLS / words / N > N ? N : HYOWON_DEPOSIT64_TILE_CELLS / words / N);
}

__device__ __forceinline__ int fixed_split_bits(const uint32_t* max_count) {
    const unsigned long long c = 8ull * (*max_count > 0u ? *max_count : 1u);
    return 63 - (63 - __clzll(c));   // 63 - floor(log2 c)
}

// hi 2^W + lo as a 128-bit integer, correctly rounded to binary64 (the bits
// below the leading 64 fold into a sticky bit).
__device__ __forceinline__ double fixed_to_double(unsigned long long hi, unsigned long long lo,
                                                  int W) {
    unsigned long long low = hi << W;
    unsigned long long high = hi >> (64 - W);
    low += lo;
    high += low < lo ? 1ull : 0ull;
    if (high == 0ull) return __ull2double_rn(low);
    const int lz = __clzll(high);
    unsigned long long top = lz ? (high << lz) | (low >> (64 - lz)) : high;
    const unsigned long long rest = lz ? (low << lz) : low;
    top |= rest != 0ull ? 1ull : 0ull;
    return ldexp(__ull2double_rn(top), 64 - lz);
}

//
// ZLOG > 0 (N = 2^ZLOG, a mesh of the five-pass solve): the tile's rows are
// transformed along z in shared memory (chunked::tile_r2c) and stored to the
// chunked half spectrum H instead of the real mesh.
template <int kDepositWords, int ZLOG>
__global__ void __launch_bounds__(kTileThreads, HYOWON_DEPOSIT64_MINB)
k_deposit_tiles(const double* __restrict__ x, const double* __restrict__ y,
                const double* __restrict__ z, const double* __restrict__ mass,
                double uniform_mass, const uint32_t* __restrict__ order,
                const uint32_t* __restrict__ offset, int shift, Axis a, int TY,
                const uint32_t* __restrict__ max_count, int e_max, double* __restrict__ mesh,
                unsigned int* status, double2* __restrict__ H, const double2* __restrict__ tw) {
    extern __shared__ __align__(16) unsigned long long acc[];
    __shared__ uint32_t seg_p0[4], seg_len[4];
    __shared__ int seg_plane[4], seg_row_lo[4], seg_row_hi[4], seg_own[4];
    __shared__ int seg_n;
    if (*status & ST_BLOCKS_PUBLISH) return;
    const int W = fixed_split_bits(max_count);
    if ((kDepositWords == 1) != (W >= kOneWordMinW)) return;
    if (kDepositWords == 2 && W < kTwoWordMinW) {
        // more than 2^32 contributors per cell could overflow a hi sum
        if (threadIdx.x == 0 && blockIdx.x == 0 && blockIdx.y == 0) raise_status(status, ST_CAPACITY);
        return;
    }
    const int N = a.N;
    const int tid = threadIdx.x;
    const int x0 = blockIdx.y;
    const int y0 = blockIdx.x * TY;
    const int ty = N - y0 < TY ? N - y0 : TY;
    const int halo = ty == N ? 0 : 1;
    const int tcells = ty * N;
    unsigned long long* acc_lo = acc;
    unsigned long long* acc_hi = acc + (kDepositWords == 2 ? static_cast<size_t>(TY) * N : 0);
    if (tid == 0) {
        int ns = 0;
        for (int own = 1; own >= 0; --own) {
            const int p = own ? x0 : (x0 == 0 ? N - 1 : x0 - 1);
            int lo[2], hi[2], nr = 0;
            if (halo && y0 == 0) {
                lo[nr] = N - 1; hi[nr++] = N - 1;
                lo[nr] = 0; hi[nr++] = ty - 1;
            } else {
                lo[nr] = y0 - halo; hi[nr++] = y0 + ty - 1;
            }
            for (int k = 0; k < nr; ++k) {
                const uint64_t c_lo = (static_cast<uint64_t>(p) * N + lo[k]) * N;
                const uint64_t c_hi = (static_cast<uint64_t>(p) * N + hi[k]) * N + (N - 1);
                const uint32_t b0 = offset[c_lo >> shift];
                const uint32_t b1 = offset[(c_hi >> shift) + 1];
                seg_p0[ns] = b0;
                seg_len[ns] = b1 - b0;
                seg_plane[ns] = p;
                seg_row_lo[ns] = lo[k];
                seg_row_hi[ns] = hi[k];
                seg_own[ns] = own;
                ++ns;
            }
        }
        seg_n = ns;
    }
    for (int e = tid; e < tcells; e += kTileThreads) {
        acc_lo[e] = 0ull;
        if (kDepositWords == 2) acc_hi[e] = 0ull;
    }
    __syncthreads();
    const unsigned long long lo_mask = (1ull << W) - 1ull;
    // 2^(62 - e_max) (one word: 2^(W-1-e_max)): a multiplication by it is
    // exact (the product is at most 2^62, and below 2^-1022 it rounds to the
    // integer 0 either way)
    const double to_fixed = ldexp(1.0, kDepositWords == 2 ? 62 - e_max : W - 1 - e_max);
    const int ns = seg_n;
    for (int g = 0; g < ns; ++g) {
        const uint32_t p0 = seg_p0[g];
        const uint32_t len = seg_len[g];
        const int plane = seg_plane[g];
        const int row_lo = seg_row_lo[g], row_hi = seg_row_hi[g];
        const bool own = seg_own[g] != 0;
        // kDepositBatch particles per thread and pass: their index and
        // position loads are all issued before the first is used
        for (uint32_t v0 = tid; v0 < len; v0 += kDepositBatch * kTileThreads) {
            uint32_t idx[kDepositBatch];
#pragma unroll
            for (int k = 0; k < kDepositBatch; ++k) {
                const uint32_t v = v0 + k * kTileThreads;
                idx[k] = v < len ? (order ? order[p0 + v] : p0 + v) : 0xffffffffu;
            }
            double px[kDepositBatch], py[kDepositBatch], pz[kDepositBatch];
#pragma unroll
            for (int k = 0; k < kDepositBatch; ++k) {
                if (idx[k] != 0xffffffffu) {
                    px[k] = x[idx[k]];
                    py[k] = y[idx[k]];
                    pz[k] = z[idx[k]];
                }
            }
#pragma unroll
            for (int k = 0; k < kDepositBatch; ++k) {
                if (idx[k] == 0xffffffffu) continue;
                const uint32_t i = idx[k];
                int ix, iy, iz;
                double tx, ty_, tz;
                if (!(cic_coord_f64(px[k], a, ix, tx) & cic_coord_f64(py[k], a, iy, ty_)
                      & cic_coord_f64(pz[k], a, iz, tz)))
                    continue;   // never in cell order: the key pass raised the status
                if (ix != plane || iy < row_lo || iy > row_hi) continue;
                const double m = mass ? mass[i] : uniform_mass;
                const double mx = m * (own ? 1.0 - tx : tx);
                const double wy[2] = {1.0 - ty_, ty_};
                const double wz[2] = {1.0 - tz, tz};
                const int gz[2] = {iz, iz + 1 == N ? 0 : iz + 1};
#pragma unroll
                for (int oy = 0; oy < 2; ++oy) {
                    const int row = iy + oy == N ? 0 : iy + oy;
                    const int ly = row - y0;
                    if (ly < 0 || ly >= ty) continue;
                    const double mxy = mx * wy[oy];
                    unsigned long long* rlo = acc_lo + ly * N;
                    unsigned long long* rhi = acc_hi + ly * N;
#pragma unroll
                    for (int oz = 0; oz < 2; ++oz) {
                        const unsigned long long q = static_cast<unsigned long long>(
                            __double2ll_rn(mxy * wz[oz] * to_fixed));
                        if (q == 0ull) continue;
                        if (kDepositWords == 1) {
                            atomicAdd(rlo + gz[oz], q);
                        } else {
                            atomicAdd(rlo + gz[oz], q & lo_mask);
                            const unsigned long long qh = q >> W;
                            if (qh) atomicAdd(rhi + gz[oz], qh);
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
    if constexpr (ZLOG > 0) {
        // N = 2^ZLOG and TY = tile_rows_f64(N, words) divides N, so ty == TY;
        // each cell pair is read once, by the transform's first stage
        using Lz = chunked::Layout<double, ZLOG>;
        constexpr int TYc = tile_rows_f64(Lz::N, kDepositWords);
        static_assert(TYc * (Lz::M / 8) <= kTileThreads,
                      "the tile's z transform needs a thread per 8 values of a row set");
        const double from_fixed = ldexp(1.0, kDepositWords == 1 ? e_max + 1 - W : e_max - 62);
        const ulonglong2* lo2 = reinterpret_cast<const ulonglong2*>(acc_lo);
        const ulonglong2* hi2 = reinterpret_cast<const ulonglong2*>(acc_hi);
        auto pair = [&](int r, int k) {
            const int e = r * (Lz::N / 2) + k;
            const ulonglong2 lo = lo2[e];
            if (kDepositWords == 1)
                return make_double2(__ull2double_rn(lo.x) * from_fixed, __ull2double_rn(lo.y) * from_fixed);
            const ulonglong2 hi = hi2[e];
            return make_double2(fixed_to_double(hi.x, lo.x, W) * from_fixed,
                                fixed_to_double(hi.y, lo.y, W) * from_fixed);
        };
        chunked::tile_r2c<double, ZLOG, TYc>(pair, reinterpret_cast<double2*>(acc), tw, H, x0, y0, tid,
                                             kTileThreads);
        return;
    }
    double* out = mesh + (static_cast<uint64_t>(x0) * N + y0) * N;
    if (kDepositWords == 1) {
        const double from_fixed = ldexp(1.0, e_max + 1 - W);
        for (int e = tid; e < tcells; e += kTileThreads)
            out[e] = __ull2double_rn(acc_lo[e]) * from_fixed;
    } else {
        const double from_fixed = ldexp(1.0, e_max - 62);
        for (int e = tid; e < tcells; e += kTileThreads)
            out[e] = fixed_to_double(acc_hi[e], acc_lo[e], W) * from_fixed;
    }
}

__global__ void k_max_count64(uint32_t nb, const uint32_t* __restrict__ count,
                              uint32_t* max_count) {
    uint32_t m = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
        m = max(m, count[i]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(max_count, m);
}

// Pure-PM Green's function (src/mesh/green_function.cpp:165-207) applied to the
// r2c of the mass mesh. `scale` folds in the density normalisation 1/dx^3 and
// the 1/N^3 of the inverse transform; the mean subtraction of
// DensityNormalization only changes the k=0 mode, which the kernel zeroes. The
// k=0 thread also checks CIC mass conservation against the reference bound
// (src/math/cic_mass_conservation.cpp:26-59): Re(delta_0) is the mesh mass.
__global__ void k_green(int N, double2* __restrict__ modes, const double* __restrict__ lap,
                        const double* __restrict__ win, double four_pi_G, double scale,
                        int deconvolve, double input_mass, double mass_tolerance,
                        unsigned int* status) {
    const int Hz = N / 2 + 1;
    const uint64_t total = static_cast<uint64_t>(N) * N * Hz;
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int iz = static_cast<int>(idx % Hz);
    const uint64_t t = idx / Hz;
    const int iy = static_cast<int>(t % N);
    const int ix = static_cast<int>(t / N);
    double2 v = modes[idx];
    if (idx == 0) {
        const double deposited = v.x;
        if (!(fabs(deposited - input_mass) <= mass_tolerance)) raise_status(status, ST_MASS);
        modes[0] = make_double2(0.0, 0.0);
        return;
    }
    const double Dk = lap[ix] + lap[iy] + lap[iz];
    double f = four_pi_G / Dk;
    if (deconvolve) {
        const double wt = win[ix] * win[iy] * win[iz];
        f /= (wt * wt);
    }
    f *= scale;
    v.x *= f;
    v.y *= f;
    modes[idx] = v;
}

// TreePM long-range Green's function (green_function.cpp:174-200):
// 4 pi G/(-k^2) * exp(-k^2 r_s^2) / W^2, with the same folded scale.
__global__ void k_green_spectral(int N, double L, double2* __restrict__ modes,
                                 const double* __restrict__ win, double four_pi_G,
                                 double scale, double r_s, double input_mass,
                                 double mass_tolerance, unsigned int* status) {
    const int Hz = N / 2 + 1;
    const uint64_t total = static_cast<uint64_t>(N) * N * Hz;
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int iz = static_cast<int>(idx % Hz);
    const uint64_t t = idx / Hz;
    const int iy = static_cast<int>(t % N);
    const int ix = static_cast<int>(t / N);
    double2 v = modes[idx];
    if (idx == 0) {
        if (!(fabs(v.x - input_mass) <= mass_tolerance)) raise_status(status, ST_MASS);
        modes[0] = make_double2(0.0, 0.0);
        return;
    }
    const double two_pi = 2.0 * 3.141592653589793;
    const int mx = ix <= N / 2 ? ix : ix - N;
    const int my = iy <= N / 2 ? iy : iy - N;
    const int mz = iz <= N / 2 ? iz : iz - N;
    const double kx = two_pi * static_cast<double>(mx) / L;
    const double ky = two_pi * static_cast<double>(my) / L;
    const double kz = two_pi * static_cast<double>(mz) / L;
    const double k2 = kx * kx + ky * ky + kz * kz;
    double f = four_pi_G / (-k2);
    f *= exp(-k2 * r_s * r_s);
    const double wt = win[ix] * win[iy] * win[iz];
    f /= (wt * wt);
    f *= scale;
    v.x *= f;
    v.y *= f;
    modes[idx] = v;
}

// out_k = -i k_axis phi_k with the Nyquist component zeroed
// (src/gravity/pm_solver.cpp:775-797).
__global__ void k_spectral_axis(int N, double L, int axis, const double2* __restrict__ phi,
                                double2* __restrict__ out) {
    const int Hz = N / 2 + 1;
    const uint64_t total = static_cast<uint64_t>(N) * N * Hz;
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int iz = static_cast<int>(idx % Hz);
    const uint64_t t = idx / Hz;
    const int iy = static_cast<int>(t % N);
    const int ix = static_cast<int>(t / N);
    const int i = axis == 0 ? ix : (axis == 1 ? iy : iz);
    double k = 0.0;
    if (!(N % 2 == 0 && i == N / 2)) {
        const int m = i <= N / 2 ? i : i - N;
        k = 2.0 * 3.141592653589793 * static_cast<double>(m) / L;
    }
    const double2 p = phi[idx];
    out[idx] = make_double2(p.y * k, -p.x * k);
}

// Plain CIC interpolation added to out (mass_assignment_gather.inc:402-450).
__global__ void k_interp_add(uint32_t n, const double* __restrict__ field,
                             const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, Axis a, double* __restrict__ out,
                             unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (*status & ST_BLOCKS_PUBLISH)) return;
    int ix, iy, iz;
    double tx, ty, tz;
    if (!(cic_coord_f64(x[i], a, ix, tx) & cic_coord_f64(y[i], a, iy, ty)
          & cic_coord_f64(z[i], a, iz, tz))) {
        raise_status(status, ST_CELL_ESCAPE);
        return;
    }
    const int N = a.N;
    const double wx[2] = {1.0 - tx, tx};
    const double wy[2] = {1.0 - ty, ty};
    const double wz[2] = {1.0 - tz, tz};
    double s = 0.0;
#pragma unroll
    for (int ox = 0; ox < 2; ++ox) {
        const int gx = ox == 0 ? ix : (ix + 1 == N ? 0 : ix + 1);
#pragma unroll
        for (int oy = 0; oy < 2; ++oy) {
            const int gy = oy == 0 ? iy : (iy + 1 == N ? 0 : iy + 1);
#pragma unroll
            for (int oz = 0; oz < 2; ++oz) {
                const int gz = oz == 0 ? iz : (iz + 1 == N ? 0 : iz + 1);
                const double w = wx[ox] * wy[oy] * wz[oz];
                s += __ldg(&field[cell_index(gx, gy, gz, N)]) * w;
            }
        }
    }
    const double r = out[i] + s;
    if (!isfinite(r)) raise_status(status, ST_FORCE);
    out[i] = r;
}

// -d / (2 dx) with the divisor fixed per launch: the product with the
// precomputed reciprocal y = RN(1/(2dx)), corrected by one exact-remainder FMA
// step (Markstein, IBM J. Res. Dev. 34(1), 1990): q = RN(d y), r = d - q (2dx)
// exactly, q' = RN(q + r y). q' is the correctly rounded quotient except in
// rare double-rounding cases, where it is within one ulp of it.
__device__ __forceinline__ double neg_quot(double d, double two_dx, double inv_two_dx) {
    const double q = d * inv_two_dx;
    const double r = fma(-q, two_dx, d);
    return -fma(r, inv_two_dx, q);
}

// One axis of the centred-gradient gather: adds w * (-(phi+ - phi-)/(2dx)) over
// the 8 CIC corners, in the reference's corner order, to *sum and accumulates
// the underflow flags. lo/hi are the stencil values one cell below / above
// the 2x2x2 block along the axis, in the block's other two indices.
template <int AXIS>
__device__ __forceinline__ void gather_axis(const double (&c)[2][2][2], const double (&lo)[2][2],
                                            const double (&hi)[2][2], const double (&wx)[2],
                                            const double (&wy)[2], const double (&wz)[2],
                                            double two_dx, double inv_two_dx, double& sum,
                                            bool& lost) {
#pragma unroll
    for (int ox = 0; ox < 2; ++ox) {
#pragma unroll
        for (int oy = 0; oy < 2; ++oy) {
#pragma unroll
            for (int oz = 0; oz < 2; ++oz) {
                const double w = wx[ox] * wy[oy] * wz[oz];
                const bool w_lost = wx[ox] != 0.0 && wy[oy] != 0.0 && wz[oz] != 0.0 && w == 0.0;
                double dv;
                if (AXIS == 0)
                    dv = (ox == 0 ? c[1][oy][oz] : hi[oy][oz]) - (ox == 0 ? lo[oy][oz] : c[0][oy][oz]);
                else if (AXIS == 1)
                    dv = (oy == 0 ? c[ox][1][oz] : hi[ox][oz]) - (oy == 0 ? lo[ox][oz] : c[ox][0][oz]);
                else
                    dv = (oz == 0 ? c[ox][oy][1] : hi[ox][oy]) - (oz == 0 ? lo[ox][oy] : c[ox][oy][0]);
                const double g = neg_quot(dv, two_dx, inv_two_dx);
                const bool w_nonzero = w != 0.0 || w_lost;
                lost |= w_nonzero && dv != 0.0 && g == 0.0;
                lost |= w_lost && g != 0.0;
                const double cg = w * g;
                lost |= w != 0.0 && g != 0.0 && cg == 0.0;
                sum += cg;
            }
        }
    }
}

// Binary exponent field of |v| (0 for zero and subnormals).
__device__ __forceinline__ int exp_field(double v) {
    return static_cast<int>((static_cast<unsigned long long>(__double_as_longlong(v)) >> 52) & 0x7ffu);
}

// Fast form of one gather axis: -(sum_corners w * dphi) / (2 dx), corners in
// the reference's order, one scaling at the end. Used when no product can
// reach the subnormal range: every non-zero weight factor >= 2^-250 (so
// w >= 2^-750), every non-zero potential difference >= 2^-200 and
// 1/(2dx) >= 2^-50, so |w dphi / (2dx)| >= 2^-1000 stays normal and the
// reference's lost-product checks cannot fire. Differs from the per-corner
// quotient sequence only in rounding (a few ulp of the axis sum). Returns
// false (nothing accumulated) when the exact sequence is needed instead.
template <int AXIS>
__device__ __forceinline__ bool gather_axis_fast(const double (&c)[2][2][2], const double (&lo)[2][2],
                                                 const double (&hi)[2][2], const double (&w)[2][2][2],
                                                 double inv_two_dx, double& sum) {
    double dv[2][2][2];
    bool ok = true;
#pragma unroll
    for (int ox = 0; ox < 2; ++ox)
#pragma unroll
        for (int oy = 0; oy < 2; ++oy)
#pragma unroll
            for (int oz = 0; oz < 2; ++oz) {
                double d;
                if (AXIS == 0)
                    d = (ox == 0 ? c[1][oy][oz] : hi[oy][oz]) - (ox == 0 ? lo[oy][oz] : c[0][oy][oz]);
                else if (AXIS == 1)
                    d = (oy == 0 ? c[ox][1][oz] : hi[ox][oz]) - (oy == 0 ? lo[ox][oz] : c[ox][0][oz]);
                else
                    d = (oz == 0 ? c[ox][oy][1] : hi[ox][oy]) - (oz == 0 ? lo[ox][oy] : c[ox][oy][0]);
                const int e = exp_field(d);
                ok &= d == 0.0 || e >= 1023 - 200;
                dv[ox][oy][oz] = d;
            }
    if (!ok) return false;
    double s = 0.0;
#pragma unroll
    for (int ox = 0; ox < 2; ++ox)
#pragma unroll
        for (int oy = 0; oy < 2; ++oy)
#pragma unroll
            for (int oz = 0; oz < 2; ++oz) s = fma(w[ox][oy][oz], dv[ox][oy][oz], s);
    sum = -(s * inv_two_dx);
    return true;
}

// interpolate_centered_gradient3_add_full_mesh
// (src/mesh/mass_assignment_gradient.cpp:117-206) into zeroed accelerations,
// fused with the K2 kick (leapfrog_integrator.cpp:240-278). The 32 distinct
// potential values of the 4x4x4 stencil footprint are loaded once: the 2x2x2
// block first, then the two outer faces of one axis at a time, so each axis
// sum is formed in the reference's corner order with few values live.
// Five blocks per SM (48 registers, the rest spilled to L1) hide the stencil
// loads' latency best: at c3 7.31 ms against 7.80 at four and 8.18 at three.
#ifndef HYOWON_GATHER64_MINB
#define HYOWON_GATHER64_MINB 5
#endif
template <typename IDX>
__global__ void __launch_bounds__(kThreads, HYOWON_GATHER64_MINB)
k_gather_kick(uint32_t n, const double* __restrict__ phi, const double* __restrict__ x,
              const double* __restrict__ y, const double* __restrict__ z,
              const double* __restrict__ px, const double* __restrict__ py,
              const double* __restrict__ pz, double* __restrict__ ax,
              double* __restrict__ ay, double* __restrict__ az, int do_kick, double K2,
              double* __restrict__ pxo, double* __restrict__ pyo,
              double* __restrict__ pzo, Axis a, double inv_two_dx, unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (*status & ST_BLOCKS_PUBLISH)) return;
    int ix, iy, iz;
    double tx, ty, tz;
    if (!(cic_coord_f64(x[i], a, ix, tx) & cic_coord_f64(y[i], a, iy, ty)
          & cic_coord_f64(z[i], a, iz, tz))) {
        raise_status(status, ST_CELL_ESCAPE);
        return;
    }
    const int N = a.N;
    const int xs[4] = {ix == 0 ? N - 1 : ix - 1, ix, ix + 1 == N ? 0 : ix + 1,
                       ix + 2 >= N ? ix + 2 - N : ix + 2};
    const int ys[4] = {iy == 0 ? N - 1 : iy - 1, iy, iy + 1 == N ? 0 : iy + 1,
                       iy + 2 >= N ? iy + 2 - N : iy + 2};
    const int zs[4] = {iz == 0 ? N - 1 : iz - 1, iz, iz + 1 == N ? 0 : iz + 1,
                       iz + 2 >= N ? iz + 2 - N : iz + 2};
#define PHI(a_, b_, c_) __ldg(&phi[cell_index_t<IDX>(xs[a_], ys[b_], zs[c_], N)])
    double c[2][2][2];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int v = 0; v < 2; ++v)
#pragma unroll
            for (int w = 0; w < 2; ++w) c[u][v][w] = PHI(u + 1, v + 1, w + 1);
    const double wx[2] = {1.0 - tx, tx};
    const double wy[2] = {1.0 - ty, ty};
    const double wz[2] = {1.0 - tz, tz};
    const double two_dx = 2.0 * a.dx;
    double gx_sum = 0.0, gy_sum = 0.0, gz_sum = 0.0;
    bool lost = false;
    // weights in the reference's product order, and whether every non-zero
    // factor is far from the subnormal range (see gather_axis_fast)
    double w[2][2][2];
    bool fast = exp_field(inv_two_dx) >= 1023 - 50 && exp_field(inv_two_dx) < 0x7ff;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        fast &= (wx[q] == 0.0 || exp_field(wx[q]) >= 1023 - 250)
            && (wy[q] == 0.0 || exp_field(wy[q]) >= 1023 - 250)
            && (wz[q] == 0.0 || exp_field(wz[q]) >= 1023 - 250);
    }
#pragma unroll
    for (int ox = 0; ox < 2; ++ox)
#pragma unroll
        for (int oy = 0; oy < 2; ++oy)
#pragma unroll
            for (int oz = 0; oz < 2; ++oz) w[ox][oy][oz] = wx[ox] * wy[oy] * wz[oz];
    double lo[2][2], hi[2][2];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            lo[u][v] = PHI(0, u + 1, v + 1);
            hi[u][v] = PHI(3, u + 1, v + 1);
        }
    if (!(fast && gather_axis_fast<0>(c, lo, hi, w, inv_two_dx, gx_sum)))
        gather_axis<0>(c, lo, hi, wx, wy, wz, two_dx, inv_two_dx, gx_sum, lost);
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            lo[u][v] = PHI(u + 1, 0, v + 1);
            hi[u][v] = PHI(u + 1, 3, v + 1);
        }
    if (!(fast && gather_axis_fast<1>(c, lo, hi, w, inv_two_dx, gy_sum)))
        gather_axis<1>(c, lo, hi, wx, wy, wz, two_dx, inv_two_dx, gy_sum, lost);
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            lo[u][v] = PHI(u + 1, v + 1, 0);
            hi[u][v] = PHI(u + 1, v + 1, 3);
        }
    if (!(fast && gather_axis_fast<2>(c, lo, hi, w, inv_two_dx, gz_sum)))
        gather_axis<2>(c, lo, hi, wx, wy, wz, two_dx, inv_two_dx, gz_sum, lost);
#undef PHI
    if (lost) raise_status(status, ST_UNDERFLOW);
    // The evolution path adds into zeroed accelerations (leapfrog_integrator.cpp:75-83).
    const double gax = 0.0 + gx_sum;
    const double gay = 0.0 + gy_sum;
    const double gaz = 0.0 + gz_sum;
    if (!(isfinite(gax) && isfinite(gay) && isfinite(gaz))) raise_status(status, ST_FORCE);
    ax[i] = gax;
    ay[i] = gay;
    az[i] = gaz;
    if (do_kick) {
        const double qx = px[i] + gax * K2;
        const double qy = py[i] + gay * K2;
        const double qz = pz[i] + gaz * K2;
        if (!(isfinite(qx) && isfinite(qy) && isfinite(qz))) raise_status(status, ST_KICK2);
        pxo[i] = qx;
        pyo[i] = qy;
        pzo[i] = qz;
    }
}

// K2 kick alone, for force paths that do not end in the fused gather.
__global__ void k_kick_only(uint32_t n, const double* __restrict__ px,
                            const double* __restrict__ py, const double* __restrict__ pz,
                            const double* __restrict__ ax, const double* __restrict__ ay,
                            const double* __restrict__ az, double K2,
                            double* __restrict__ pxo, double* __restrict__ pyo,
                            double* __restrict__ pzo, unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (*status & ST_BLOCKS_PUBLISH)) return;
    const double qx = px[i] + ax[i] * K2;
    const double qy = py[i] + ay[i] * K2;
    const double qz = pz[i] + az[i] * K2;
    if (!(isfinite(qx) && isfinite(qy) && isfinite(qz))) raise_status(status, ST_KICK2);
    pxo[i] = qx;
    pyo[i] = qy;
    pzo[i] = qz;
}

__global__ void k_cell_coords(uint32_t n, const double* __restrict__ pos, Axis a,
                              int64_t* __restrict__ base, double* __restrict__ frac,
                              unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int b = -1;
    double f = 0.0;
    if (!cic_coord_f64(pos[i], a, b, f)) {
        raise_status(status, ST_CELL_ESCAPE);
        b = -1;
    }
    base[i] = b;
    frac[i] = f;
}

}  // namespace

void launch_validate_inputs_f64(uint32_t n, const double* x, const double* y,
                                const double* z, const double* mass, unsigned int* status,
                                cudaStream_t s) {
    if (n == 0) return;
    k_validate_inputs<<<blocks_for(n), kThreads, 0, s>>>(n, x, y, z, mass, status);
}

void launch_key_f64(uint32_t n, const ParticlesF64& p, Axis a, const SortWork& w,
                    unsigned int* status, cudaStream_t s) {
    if (n == 0) return;
    k_key<<<blocks_for(n), kThreads, 0, s>>>(n, p.x, p.y, p.z, a, w.key, w.rank, w.count,
                                             w.shift, status);
}

void launch_kick_drift_key_f64(uint32_t n, const ParticlesF64& cur, const double* ax,
                               const double* ay, const double* az, double K1, double D,
                               Axis a, const ParticlesF64& cand, const SortWork& w,
                               bool with_key, unsigned long long* max_drift_bits,
                               unsigned int* status, cudaStream_t s) {
    if (n == 0) return;
    k_kick_drift_key<<<stream_blocks(n, kThreads), kThreads, 0, s>>>(
        n, cur.x, cur.y, cur.z, cur.px, cur.py, cur.pz, ax, ay, az, K1, D, a, cand.x, cand.y,
        cand.z, cand.px, cand.py, cand.pz, w.key, w.rank, w.count, w.shift, with_key ? 1 : 0,
        max_drift_bits, status);
}

void launch_deposit_f64(uint32_t n, const ParticlesF64& p, const double* mass,
                        double uniform_mass, Axis a, double* mesh, unsigned int* status,
                        cudaStream_t s) {
    if (n == 0) return;
    k_deposit<<<blocks_for(n), kThreads, 0, s>>>(n, p.x, p.y, p.z, mass, uniform_mass, a,
                                                 mesh, status);
}


int deposit_mass_exponent_f64(double max_mass) {
    int e = 0;
    if (max_mass > 0.0) std::frexp(max_mass, &e);   // max_mass < 2^e
    return e;
}

template <int WORDS, int ZLOG>
cudaError_t launch_tiles(const ParticlesF64& p, const double* mass, double uniform_mass,
                         const uint32_t* order, const SortWork& w, Axis a,
                         const uint32_t* max_count, int e_max, double* mesh, double2* modes,
                         const double2* tw, unsigned int* status, cudaStream_t s) {
    const int N = a.N;
    const int TY = tile_rows_f64(N, WORDS);
    size_t smem = 8 * WORDS * static_cast<size_t>(TY) * N;
    if constexpr (ZLOG > 0) {
        // the z transform runs in the accumulators' memory
        const size_t rows = sizeof(double2) * static_cast<size_t>(N / 2) * TY;
        if (rows > smem) smem = rows;
    }
    cudaError_t e = cudaFuncSetAttribute(k_deposit_tiles<WORDS, ZLOG>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const dim3 grid(static_cast<unsigned>((N + TY - 1) / TY), static_cast<unsigned>(N));
    k_deposit_tiles<WORDS, ZLOG><<<grid, kTileThreads, smem, s>>>(
        p.x, p.y, p.z, mass, uniform_mass, order, w.offset, w.shift, a, TY, max_count, e_max, mesh,
        status, modes, tw);
    return cudaPeekAtLastError();
}

template <int WORDS>
cudaError_t launch_tiles_n(const ParticlesF64& p, const double* mass, double uniform_mass,
                           const uint32_t* order, const SortWork& w, Axis a,
                           const uint32_t* max_count, int e_max, double* mesh, double2* modes,
                           const double2* tw, unsigned int* status, cudaStream_t s) {
#define HYOWON_TILES(LG) \
    launch_tiles<WORDS, LG>(p, mass, uniform_mass, order, w, a, max_count, e_max, mesh, modes, tw, status, s)
    if (!modes) return HYOWON_TILES(0);
    switch (a.N) {
    case 32: return HYOWON_TILES(5);
    case 64: return HYOWON_TILES(6);
    case 128: return HYOWON_TILES(7);
    case 256: return HYOWON_TILES(8);
    case 512: return HYOWON_TILES(9);
    case 1024: return HYOWON_TILES(10);
    case 2048: return HYOWON_TILES(11);
    default: return cudaErrorInvalidValue;
    }
#undef HYOWON_TILES
}

cudaError_t launch_deposit_tiles_f64(const ParticlesF64& p, const double* mass,
                                     double uniform_mass, const uint32_t* order,
                                     const SortWork& w, Axis a, const uint32_t* max_count,
                                     uint32_t max_count_host, int e_max, double* mesh,
                                     double2* modes, const double2* tw, unsigned int* status,
                                     cudaStream_t s) {
    // the same W the kernels derive from *max_count (they check it again)
    const unsigned long long c = 8ull * (max_count_host > 0u ? max_count_host : 1u);
    int lg = 0;
    while ((c >> (lg + 1)) != 0ull) ++lg;
    const int W = 63 - lg;
    if (W >= kOneWordMinW)
        return launch_tiles_n<1>(p, mass, uniform_mass, order, w, a, max_count, e_max, mesh, modes,
                                 tw, status, s);
    return launch_tiles_n<2>(p, mass, uniform_mass, order, w, a, max_count, e_max, mesh, modes, tw,
                             status, s);
}

void launch_max_count_f64(uint32_t n_buckets, const uint32_t* count, uint32_t* max_count,
                          cudaStream_t s) {
    k_max_count64<<<stream_blocks(n_buckets, kThreads), kThreads, 0, s>>>(n_buckets, count,
                                                                          max_count);
}



void launch_green_f64(int N, double2* modes, const double* lap, const double* win,
                      double four_pi_G, double scale, int deconvolve, double input_mass,
                      double mass_tolerance, unsigned int* status, cudaStream_t s) {
    const uint64_t total = static_cast<uint64_t>(N) * N * (N / 2 + 1);
    k_green<<<blocks_for(total), kThreads, 0, s>>>(N, modes, lap, win, four_pi_G, scale,
                                                   deconvolve, input_mass, mass_tolerance,
                                                   status);
}

void launch_green_spectral_f64(int N, double L, double2* modes, const double* win,
                               double four_pi_G, double scale, double r_s,
                               double input_mass, double mass_tolerance,
                               unsigned int* status, cudaStream_t s) {
    const uint64_t total = static_cast<uint64_t>(N) * N * (N / 2 + 1);
    k_green_spectral<<<blocks_for(total), kThreads, 0, s>>>(
        N, L, modes, win, four_pi_G, scale, r_s, input_mass, mass_tolerance, status);
}

void launch_spectral_axis_f64(int N, double L, int axis, const double2* phi_k,
                              double2* out_k, cudaStream_t s) {
    const uint64_t total = static_cast<uint64_t>(N) * N * (N / 2 + 1);
    k_spectral_axis<<<blocks_for(total), kThreads, 0, s>>>(N, L, axis, phi_k, out_k);
}

void launch_interp_add_f64(uint32_t n, const double* field, const ParticlesF64& p,
                           Axis a, double* out, unsigned int* status, cudaStream_t s) {
    if (n == 0) return;
    k_interp_add<<<blocks_for(n), kThreads, 0, s>>>(n, field, p.x, p.y, p.z, a, out, status);
}

void launch_gather_kick_f64(uint32_t n, const double* phi, const ParticlesF64& p,
                            double* ax, double* ay, double* az, int do_kick, double K2,
                            double* pxo, double* pyo, double* pzo, Axis a,
                            unsigned int* status, cudaStream_t s) {
    if (n == 0) return;
    if (cells_fit_u32(a.N))
        k_gather_kick<uint32_t><<<blocks_for(n), kThreads, 0, s>>>(
            n, phi, p.x, p.y, p.z, p.px, p.py, p.pz, ax, ay, az, do_kick, K2, pxo, pyo, pzo, a,
            1.0 / (2.0 * a.dx), status);
    else
        k_gather_kick<uint64_t><<<blocks_for(n), kThreads, 0, s>>>(
            n, phi, p.x, p.y, p.z, p.px, p.py, p.pz, ax, ay, az, do_kick, K2, pxo, pyo, pzo, a,
            1.0 / (2.0 * a.dx), status);
}

void launch_kick_only_f64(uint32_t n, const ParticlesF64& p, const double* ax,
                          const double* ay, const double* az, double K2, double* pxo,
                          double* pyo, double* pzo, unsigned int* status, cudaStream_t s) {
    if (n == 0) return;
    k_kick_only<<<blocks_for(n), kThreads, 0, s>>>(n, p.px, p.py, p.pz, ax, ay, az, K2, pxo,
                                                   pyo, pzo, status);
}

void launch_cell_coords_f64(uint32_t n, const double* pos, Axis a, int64_t* base,
                            double* frac, unsigned int* status, cudaStream_t s) {
    if (n == 0) return;
    k_cell_coords<<<blocks_for(n), kThreads, 0, s>>>(n, pos, a, base, frac, status);
}

}  // namespace hyowon
