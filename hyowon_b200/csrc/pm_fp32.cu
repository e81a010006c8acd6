// pm_fp32.cu -- precision form of the PM step (see pm_fp32.h).
//
// Per particle: u32 fixed-point position per axis (x = u L / 2^32), FP32
// momentum and acceleration. The cell of u on an N mesh is (u*N) >> 32 and the
// CIC fraction is the low word of u*N, so cell assignment needs no division and
// the periodic wrap of the drift is the natural wrap of 32-bit integers.
//
// Deposit: each particle adds the exact integer weights
// w = wx*wy*wz, wx in {2^B - f, f} with f the top B bits of the fraction, to
// int64 cells that start at -mean (the deposit is an offset from the mean cell
// mass). Integer addition is associative, so the mesh is bit-identical run to
// run whatever order the atomics land in, and the mesh sum equals
// n 2^(3B) - mean*N^3 exactly (checked every step). B <= 16 is chosen per step
// on the device from the densest sort bucket so that no cell can overflow.
//
// The int64 offsets are converted to FP32 for cuFFT R2C, the Green's function
// (with the density normalisation and the 1/N^3 folded into one constant) is
// applied in FP32, C2R gives the FP32 potential, and the centred-gradient gather
// + K2 kick run in FP32. Only the drift p*D and its rounding into the
// fixed-point position are FP64.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "hyowon_pm.h"
#include "pm_diag.h"
#include "pm_fp32.h"
#include "pm_chunk.cuh"
#include "pm_poisson.h"
#include "pm_kernels.h"

namespace hyowon::fp32 {

namespace {

constexpr int kThreads = 256;
constexpr double kTwo32 = 4294967296.0;

inline unsigned blocks_for(uint64_t n, int t = kThreads) {
    return static_cast<unsigned>((n + t - 1) / t);
}

struct FixedPlan {
    int B;                 // fraction bits per axis of the deposit weights
    int pad;
    long long mean_q;      // floor(n 2^(3B) / N^3)
    unsigned long long residual;  // n 2^(3B) - mean_q N^3 (the exact mesh sum)
    float c_green;         // 4 pi G m / dx^3 / N^3 * 2^(-3B)
    float pad2;
};

__device__ __forceinline__ uint32_t cell_of(uint32_t u, int N, uint32_t& frac) {
    const unsigned long long p = static_cast<unsigned long long>(u) * static_cast<unsigned>(N);
    frac = static_cast<uint32_t>(p);
    return static_cast<uint32_t>(p >> 32);
}

// Row-major cell index; 64-bit because a mesh side above 1625 has more than
// 2^32 cells (the row ix N + iy still fits 32 bits).
__device__ __forceinline__ uint64_t cell_index(uint32_t ix, uint32_t iy, uint32_t iz, int N) {
    return static_cast<uint64_t>(ix * static_cast<uint32_t>(N) + iy) * static_cast<uint32_t>(N) + iz;
}

// The same in index type IDX: the gather uses 32-bit indices whenever the
// mesh has at most 2^32 cells (fewer registers for its 32 stencil loads).
template <typename IDX>
__device__ __forceinline__ IDX cell_index_t(uint32_t ix, uint32_t iy, uint32_t iz, int N) {
    return static_cast<IDX>(ix * static_cast<uint32_t>(N) + iy) * static_cast<uint32_t>(N) + iz;
}

inline bool cells_fit_u32(int N) {
    return static_cast<uint64_t>(N) * N * N <= 0xffffffffull;
}

__device__ __forceinline__ uint32_t to_fixed(double x, double L, bool& ok) {
    const double w = wrap_f64(x, L);
    ok = isfinite(w) && w >= 0.0 && w < L;
    if (!ok) return 0u;
    double t = floor(w / L * kTwo32);
    if (t >= kTwo32) t = kTwo32 - 1.0;
    if (t < 0.0) t = 0.0;
    return static_cast<uint32_t>(t);
}

__global__ void k_to_fixed(uint32_t n, const double* __restrict__ x, const double* __restrict__ y,
                           const double* __restrict__ z, const double* __restrict__ px,
                           const double* __restrict__ py, const double* __restrict__ pz,
                           double L, uint32_t* __restrict__ ux, uint32_t* __restrict__ uy,
                           uint32_t* __restrict__ uz, float* __restrict__ fx,
                           float* __restrict__ fy, float* __restrict__ fz,
                           unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool a, b, c;
    ux[i] = to_fixed(x[i], L, a);
    uy[i] = to_fixed(y[i], L, b);
    uz[i] = to_fixed(z[i], L, c);
    const double qx = px ? px[i] : 0.0, qy = py ? py[i] : 0.0, qz = pz ? pz[i] : 0.0;
    if (!(a && b && c) || !isfinite(qx) || !isfinite(qy) || !isfinite(qz))
        raise_status(status, ST_NONFINITE_INPUT);
    fx[i] = static_cast<float>(qx);
    fy[i] = static_cast<float>(qy);
    fz[i] = static_cast<float>(qz);
}

__global__ void k_key(uint32_t n, const uint32_t* __restrict__ ux, const uint32_t* __restrict__ uy,
                      const uint32_t* __restrict__ uz, int N, int shift,
                      uint32_t* __restrict__ key, uint32_t* __restrict__ rank,
                      uint32_t* __restrict__ count, uint32_t* max_count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t f;
    const uint32_t b = static_cast<uint32_t>(
        cell_index(cell_of(ux[i], N, f), cell_of(uy[i], N, f), cell_of(uz[i], N, f), N) >> shift);
    key[i] = b;
    rank[i] = bucket_rank(count, b);
}

// K1 kick (FP32) + drift (FP64 increment rounded once into the fixed point).
// Eight blocks per SM (32 registers, no spill): sort phase at c3 2.84 ms
// against 3.13 at four blocks and 3.49 at six.
#ifndef HYOWON_KICK32_MINB
#define HYOWON_KICK32_MINB 8
#endif
__global__ void __launch_bounds__(kThreads, HYOWON_KICK32_MINB)
k_kick_drift_key(uint32_t n, const uint32_t* __restrict__ ux,
                                 const uint32_t* __restrict__ uy, const uint32_t* __restrict__ uz,
                                 const float* __restrict__ px, const float* __restrict__ py,
                                 const float* __restrict__ pz, const float* __restrict__ ax,
                                 const float* __restrict__ ay, const float* __restrict__ az,
                                 float K1, double D, double to_units, int N,
                                 uint32_t* __restrict__ uxo, uint32_t* __restrict__ uyo,
                                 uint32_t* __restrict__ uzo, float* __restrict__ pxo,
                                 float* __restrict__ pyo, float* __restrict__ pzo, int shift,
                                 int with_rank, uint32_t* __restrict__ key,
                                 uint32_t* __restrict__ rank, uint32_t* __restrict__ count,
                                 uint32_t* max_count, unsigned long long* max_drift_bits,
                                 unsigned int* status) {
    double drift_max = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double drift_norm = 0.0;
        const float qx = fmaf(ax[i], K1, px[i]);
        const float qy = fmaf(ay[i], K1, py[i]);
        const float qz = fmaf(az[i], K1, pz[i]);
        const double dx = static_cast<double>(qx) * D;
        const double dy = static_cast<double>(qy) * D;
        const double dz = static_cast<double>(qz) * D;
        const double sx = dx * to_units, sy = dy * to_units, sz = dz * to_units;
        const double lim = 4.0e18;
        const bool ok = isfinite(qx) && isfinite(qy) && isfinite(qz) && fabs(sx) < lim
            && fabs(sy) < lim && fabs(sz) < lim;
        uint32_t nx = ux[i], ny = uy[i], nz = uz[i];
        if (ok) {
            nx += static_cast<uint32_t>(static_cast<unsigned long long>(__double2ll_rn(sx)));
            ny += static_cast<uint32_t>(static_cast<unsigned long long>(__double2ll_rn(sy)));
            nz += static_cast<uint32_t>(static_cast<unsigned long long>(__double2ll_rn(sz)));
            drift_norm = hypot(hypot(dx, dy), dz);
        } else {
            raise_status(status, ST_KICK_DRIFT);
        }
        uxo[i] = nx;
        uyo[i] = ny;
        uzo[i] = nz;
        pxo[i] = qx;
        pyo[i] = qy;
        pzo[i] = qz;
        uint32_t f;
        const uint32_t b = static_cast<uint32_t>(
            cell_index(cell_of(nx, N, f), cell_of(ny, N, f), cell_of(nz, N, f), N) >> shift);
        if (with_rank) {
            key[i] = b;
            rank[i] = bucket_rank(count, b);
        } else {
            // occupancy only (bounds the deposit weights): one atomic per group
            // of lanes that share the bucket, as sorted neighbours mostly do
            const unsigned active = __activemask();
            const unsigned peers = __match_any_sync(active, b);
            if ((threadIdx.x & 31) == __ffs(peers) - 1)
                atomicAdd(&count[b], static_cast<uint32_t>(__popc(peers)));
        }
        drift_max = drift_norm > drift_max ? drift_norm : drift_max;
    }
    block_max_to(static_cast<unsigned long long>(__double_as_longlong(drift_max)), max_drift_bits);
}

__global__ void k_max_count(uint32_t nb, const uint32_t* __restrict__ count, uint32_t* max_count) {
    uint32_t m = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
        m = max(m, count[i]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(max_count, m);
}

// Chooses the deposit fraction bits B for this step: the largest B <= 16 with
// 8 * max_bucket * 2^(3B) <= 2^63 - 1, so no cell (fed by at most 8 buckets'
// particles) can overflow; then the mean offset and the Green constant.
__global__ void k_plan(uint32_t n, uint64_t cells, const uint32_t* max_count, double c0,
                       int centre, FixedPlan* plan) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const unsigned long long mc = *max_count > 0 ? *max_count : 1u;
    int B = 16;
    while (B > 4) {
        const unsigned __int128 worst =
            static_cast<unsigned __int128>(8ull * mc) << (3 * B);
        if (worst <= static_cast<unsigned __int128>(0x7fffffffffffffffull)) break;
        --B;
    }
    const unsigned __int128 total = static_cast<unsigned __int128>(n) << (3 * B);
    const unsigned long long mean = centre ? static_cast<unsigned long long>(total / cells) : 0ull;
    plan->B = B;
    plan->mean_q = static_cast<long long>(mean);
    plan->residual = static_cast<unsigned long long>(total - static_cast<unsigned __int128>(mean) * cells);
    plan->c_green = static_cast<float>(ldexp(c0, -3 * B));
}

__device__ __forceinline__ void store_cell(float* out, long long q) { *out = __ll2float_rn(q); }
__device__ __forceinline__ void store_cell(long long* out, long long q) { *out = q; }
// Two adjacent cells (8-byte aligned for float, 16-byte for int64).
__device__ __forceinline__ void store_cell2(float* out, long long a, long long b) {
    *reinterpret_cast<float2*>(out) = make_float2(__ll2float_rn(a), __ll2float_rn(b));
}
__device__ __forceinline__ void store_cell2(long long* out, long long a, long long b) {
    *reinterpret_cast<longlong2*>(out) = make_longlong2(a, b);
}

// Owner-computes fixed-point deposit: one block per tile of TY mesh rows
// (x0, y0 .. y0+TY-1, all z) accumulating int64 weights in shared memory
// (integer atomics: the result does not depend on their order), then writing
// each cell once as its offset from the mean, q - mean_q (FP32 for the
// transform, or int64 exactly), and folding the offsets into *qsum (mod 2^64)
// for the exact mass check.
//
// Contributors are the particles whose base cell lies in planes x0 or x0-1
// and rows y0-1 .. y0+TY-1. In cell order the rows of one plane are a single
// contiguous range (two when row y0-1 wraps to N-1), so the tile reads at most
// four contiguous segments of the cell-ordered particles, located through the
// bucket starts `offset` (`order`: sorted slot -> particle, or null when the
// arrays are in cell order). A bucket can straddle a segment edge, so each
// particle is kept only if its own base cell lies in the segment's plane and
// rows: segments are disjoint in (plane, row), hence every contributor is
// counted exactly once. Threads walk the concatenated segments
// kDepositBatch particles at a time.
constexpr int kDepositThreads = 256;
#ifndef HYOWON_DEPOSIT_BATCH
#define HYOWON_DEPOSIT_BATCH 4
#endif
constexpr int kDepositBatch = HYOWON_DEPOSIT_BATCH;

// Adds w to a shared-memory int64 accumulator. HYOWON_DEPOSIT_RED selects the
// reduction form (red.shared.add.u64: no value returned) over atomicAdd.
#ifndef HYOWON_DEPOSIT_RED
#define HYOWON_DEPOSIT_RED 0
#endif
__device__ __forceinline__ void shared_add_u64(unsigned long long* a, unsigned long long w) {
#if HYOWON_DEPOSIT_RED
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(a));
    asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(sa), "l"(w) : "memory");
#else
    atomicAdd(a, w);
#endif
}

// Rows of a deposit tile: 8-byte accumulators, at most HYOWON_DEPOSIT_TILE_CELLS
// cells (32 KiB at 4096: 6 blocks per SM, which hides the particle loads
// better than 64 KiB tiles despite more halo rows) per tile.
#ifndef HYOWON_DEPOSIT_TILE_CELLS
#define HYOWON_DEPOSIT_TILE_CELLS 4096
#endif
__host__ __device__ constexpr int deposit_rows(int N) {
    return HYOWON_DEPOSIT_TILE_CELLS / N < 1 ? 1
         : (HYOWON_DEPOSIT_TILE_CELLS / N > N ? N : HYOWON_DEPOSIT_TILE_CELLS / N);
}

#ifndef HYOWON_DEPOSIT_MINB
#define HYOWON_DEPOSIT_MINB 0
#endif
#if HYOWON_DEPOSIT_MINB > 0
#define HYOWON_DEPOSIT_BOUNDS __launch_bounds__(kDepositThreads, HYOWON_DEPOSIT_MINB)
#else
#define HYOWON_DEPOSIT_BOUNDS __launch_bounds__(kDepositThreads)
#endif
//
// ZLOG > 0 (N = 2^ZLOG, a power-of-two mesh of the five-pass solve): instead of
// the real cells the tile's rows are transformed along z in shared memory
// (chunked::tile_r2c) and stored to the chunked half spectrum H, the first
// pass of the potential solve done while the tile is on chip.
template <typename OUT, int ZLOG>
__global__ void HYOWON_DEPOSIT_BOUNDS
k_deposit_tiles(const uint32_t* __restrict__ ux, const uint32_t* __restrict__ uy,
                const uint32_t* __restrict__ uz, const uint32_t* __restrict__ order,
                const uint32_t* __restrict__ offset, int shift, int N, int TY,
                const FixedPlan* plan, OUT* __restrict__ out, unsigned long long* qsum,
                const unsigned int* status, float2* __restrict__ H,
                const float2* __restrict__ tw) {
    extern __shared__ __align__(16) unsigned long long qtile[];
    __shared__ uint32_t seg_p0[4], seg_len[4];
    __shared__ int seg_plane[4], seg_row_lo[4], seg_row_hi[4], seg_xr[4];
    __shared__ int seg_n;
    if (*status & ST_BLOCKS_PUBLISH) return;
    const int tid = threadIdx.x;
    const int x0 = blockIdx.y;
    const int y0 = blockIdx.x * TY;
    const int ty = N - y0 < TY ? N - y0 : TY;
    const int halo = ty == N ? 0 : 1;   // a tile spanning all rows has no halo
    if (tid == 0) {
        // segments: (plane x0 then x0-1) x (row ranges); a wrapped halo row
        // N-1 is its own segment
        int ns = 0;
        for (int xr = 0; xr < 2; ++xr) {
            const int p = xr == 0 ? x0 : (x0 == 0 ? N - 1 : x0 - 1);
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
                const uint32_t a = offset[c_lo >> shift];
                const uint32_t b = offset[(c_hi >> shift) + 1];
                seg_p0[ns] = a;
                seg_len[ns] = b - a;
                seg_plane[ns] = p;
                seg_row_lo[ns] = lo[k];
                seg_row_hi[ns] = hi[k];
                seg_xr[ns] = xr;
                ++ns;
            }
        }
        seg_n = ns;
    }
    const int tcells = ty * N;
    {
        ulonglong2* q2 = reinterpret_cast<ulonglong2*>(qtile);
        for (int e = tid; e < tcells / 2; e += kDepositThreads) q2[e] = make_ulonglong2(0ull, 0ull);
        if ((tcells & 1) && tid == 0) qtile[tcells - 1] = 0ull;
    }
    __syncthreads();
    const int B = plan->B;
    const uint32_t one = 1u << B;
    const int sh = 32 - B;
    const uint32_t uN = static_cast<uint32_t>(N);
    const int ns = seg_n;
    // one segment at a time: its bounds, plane and rows are block-uniform
    for (int g = 0; g < ns; ++g) {
        const uint32_t p0 = seg_p0[g];
        const uint32_t len = seg_len[g];
        const uint32_t plane = static_cast<uint32_t>(seg_plane[g]);
        const int row_lo = seg_row_lo[g], row_hi = seg_row_hi[g];
        const bool own_plane = seg_xr[g] == 0;
        for (uint32_t v0 = tid; v0 < len; v0 += kDepositBatch * kDepositThreads) {
            uint32_t idx[kDepositBatch];
#pragma unroll
            for (int k = 0; k < kDepositBatch; ++k) {
                const uint32_t v = v0 + k * kDepositThreads;
                idx[k] = v < len ? (order ? order[p0 + v] : p0 + v) : 0xffffffffu;
            }
            uint32_t u[kDepositBatch][3];
#pragma unroll
            for (int k = 0; k < kDepositBatch; ++k) {
                if (idx[k] != 0xffffffffu) {
                    u[k][0] = ux[idx[k]];
                    u[k][1] = uy[idx[k]];
                    u[k][2] = uz[idx[k]];
                }
            }
#pragma unroll
            for (int k = 0; k < kDepositBatch; ++k) {
                if (idx[k] == 0xffffffffu) continue;
                uint32_t fx, fy, fz;
                const uint32_t ix = cell_of(u[k][0], N, fx);
                const uint32_t iy = cell_of(u[k][1], N, fy);
                const uint32_t iz = cell_of(u[k][2], N, fz);
                // keep the particle only in the segment of its own base cell
                if (ix != plane || static_cast<int>(iy) < row_lo || static_cast<int>(iy) > row_hi)
                    continue;
                fx >>= sh;
                fy >>= sh;
                fz >>= sh;
                const uint32_t wx = own_plane ? one - fx : fx;
                const uint32_t wz0 = one - fz, wz1 = fz;
                const uint32_t gz1 = iz + 1 == uN ? 0u : iz + 1;
#pragma unroll
                for (int oy = 0; oy < 2; ++oy) {
                    const uint32_t ys = iy + oy == uN ? 0u : iy + oy;
                    const int ly = static_cast<int>(ys) - y0;
                    if (ly < 0 || ly >= ty) continue;
                    // (wx wy) wz: a 32x32 -> 64 product, then 64 x 32
                    const unsigned long long wxy =
                        static_cast<unsigned long long>(wx) * (oy ? fy : one - fy);
                    unsigned long long* row = qtile + static_cast<uint32_t>(ly) * uN;
                    const unsigned long long w0 = wxy * wz0;
                    const unsigned long long w1 = wxy * wz1;
                    if (w0) shared_add_u64(row + iz, w0);
                    if (w1) shared_add_u64(row + gz1, w1);
                }
            }
        }
    }
    __syncthreads();
    const long long mean = plan->mean_q;
    if constexpr (ZLOG > 0) {
        // N = 2^ZLOG and TY = deposit_rows(N) divides N, so ty == TY here;
        // each cell pair is read once, by the transform's first stage
        using Lz = chunked::Layout<float, ZLOG>;
        constexpr int TYc = deposit_rows(Lz::N);
        static_assert(TYc * (Lz::M / 8) <= kDepositThreads,
                      "the tile's z transform needs a thread per 8 values of a row set");
        const ulonglong2* q2 = reinterpret_cast<const ulonglong2*>(qtile);
        unsigned long long local = 0;
        auto pair = [&](int r, int k) {
            const ulonglong2 q = q2[r * (Lz::N / 2) + k];
            const long long a0 = static_cast<long long>(q.x) - mean;
            const long long a1 = static_cast<long long>(q.y) - mean;
            local += static_cast<unsigned long long>(a0) + static_cast<unsigned long long>(a1);
            return make_float2(__ll2float_rn(a0), __ll2float_rn(a1));
        };
        chunked::tile_r2c<float, ZLOG, TYc>(pair, reinterpret_cast<float2*>(qtile), tw, H, x0, y0, tid,
                                            kDepositThreads);
        if (qsum) block_sum_to(local, qsum);
        return;
    }
    OUT* o = out + (static_cast<uint64_t>(x0) * N + y0) * N;
    unsigned long long local = 0;
    if ((tcells & 1) == 0 && (N & 1) == 0) {
        // two cells per thread and iteration: the tile starts on an even cell
        const ulonglong2* q2 = reinterpret_cast<const ulonglong2*>(qtile);
        for (int e = tid; e < tcells / 2; e += kDepositThreads) {
            const ulonglong2 q = q2[e];
            const long long v0 = static_cast<long long>(q.x) - mean;
            const long long v1 = static_cast<long long>(q.y) - mean;
            store_cell2(&o[2 * e], v0, v1);
            local += static_cast<unsigned long long>(v0) + static_cast<unsigned long long>(v1);
        }
    } else {
        for (int e = tid; e < tcells; e += kDepositThreads) {
            const long long v = static_cast<long long>(qtile[e]) - mean;
            store_cell(&o[e], v);
            local += static_cast<unsigned long long>(v);
        }
    }
    if (qsum) block_sum_to(local, qsum);
}

// `expect_offset` is 0 except in tests of the failure path, which move the
// expected sum off the exact one.
__global__ void k_check_mass(const unsigned long long* qsum, const FixedPlan* plan,
                             unsigned long long expect_offset, unsigned int* status) {
    if (threadIdx.x == 0 && *qsum != plan->residual + expect_offset) raise_status(status, ST_MASS);
}

__global__ void k_green(int N, float2* __restrict__ modes, const float* __restrict__ lap,
                        const float* __restrict__ win, int deconvolve, const FixedPlan* plan) {
    const int Hz = N / 2 + 1;
    const uint64_t total = static_cast<uint64_t>(N) * N * Hz;
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    if (idx == 0) {
        modes[0] = make_float2(0.f, 0.f);
        return;
    }
    const int iz = static_cast<int>(idx % Hz);
    const uint64_t t = idx / Hz;
    const int iy = static_cast<int>(t % N);
    const int ix = static_cast<int>(t / N);
    float f = plan->c_green / (lap[ix] + lap[iy] + lap[iz]);
    if (deconvolve) {
        const float wt = win[ix] * win[iy] * win[iz];
        f /= wt * wt;
    }
    float2 v = modes[idx];
    v.x *= f;
    v.y *= f;
    modes[idx] = v;
}

__global__ void k_green_spectral(int N, double L, float2* __restrict__ modes,
                                 const float* __restrict__ win, float r_s, const FixedPlan* plan) {
    const int Hz = N / 2 + 1;
    const uint64_t total = static_cast<uint64_t>(N) * N * Hz;
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    if (idx == 0) {
        modes[0] = make_float2(0.f, 0.f);
        return;
    }
    const int iz = static_cast<int>(idx % Hz);
    const uint64_t t = idx / Hz;
    const int iy = static_cast<int>(t % N);
    const int ix = static_cast<int>(t / N);
    const float kf = static_cast<float>(2.0 * 3.141592653589793 / L);
    const float kx = kf * static_cast<float>(ix <= N / 2 ? ix : ix - N);
    const float ky = kf * static_cast<float>(iy <= N / 2 ? iy : iy - N);
    const float kz = kf * static_cast<float>(iz);
    const float k2 = kx * kx + ky * ky + kz * kz;
    const float wt = win[ix] * win[iy] * win[iz];
    const float f = -plan->c_green / k2 * expf(-k2 * r_s * r_s) / (wt * wt);
    float2 v = modes[idx];
    v.x *= f;
    v.y *= f;
    modes[idx] = v;
}

__global__ void k_spectral_axis(int N, double L, int axis, const float2* __restrict__ phi,
                                float2* __restrict__ out) {
    const int Hz = N / 2 + 1;
    const uint64_t total = static_cast<uint64_t>(N) * N * Hz;
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int iz = static_cast<int>(idx % Hz);
    const uint64_t t = idx / Hz;
    const int iy = static_cast<int>(t % N);
    const int ix = static_cast<int>(t / N);
    const int i = axis == 0 ? ix : (axis == 1 ? iy : iz);
    float k = 0.f;
    if (!(N % 2 == 0 && i == N / 2))
        k = static_cast<float>(2.0 * 3.141592653589793 / L) * static_cast<float>(i <= N / 2 ? i : i - N);
    const float2 p = phi[idx];
    out[idx] = make_float2(p.y * k, -p.x * k);
}

__global__ void k_interp_add(uint32_t n, const float* __restrict__ field,
                             const uint32_t* __restrict__ ux, const uint32_t* __restrict__ uy,
                             const uint32_t* __restrict__ uz, int N, float* __restrict__ out,
                             const unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (*status & ST_BLOCKS_PUBLISH)) return;
    uint32_t fx, fy, fz;
    const uint32_t ix = cell_of(ux[i], N, fx), iy = cell_of(uy[i], N, fy), iz = cell_of(uz[i], N, fz);
    const float tx = __uint2float_rn(fx) * 2.3283064365386963e-10f;
    const float ty = __uint2float_rn(fy) * 2.3283064365386963e-10f;
    const float tz = __uint2float_rn(fz) * 2.3283064365386963e-10f;
    const float wx[2] = {1.f - tx, tx}, wy[2] = {1.f - ty, ty}, wz[2] = {1.f - tz, tz};
    const uint32_t gx[2] = {ix, ix + 1 == static_cast<uint32_t>(N) ? 0u : ix + 1};
    const uint32_t gy[2] = {iy, iy + 1 == static_cast<uint32_t>(N) ? 0u : iy + 1};
    const uint32_t gz[2] = {iz, iz + 1 == static_cast<uint32_t>(N) ? 0u : iz + 1};
    float s = 0.f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int c = 0; c < 2; ++c)
                s += __ldg(&field[cell_index(gx[a], gy[b], gz[c], N)]) * (wx[a] * wy[b] * wz[c]);
    out[i] += s;
}

// Centred-gradient CIC gather (FP32) fused with the K2 kick.
#ifndef HYOWON_GATHER_MINB
#define HYOWON_GATHER_MINB 1
#endif
template <typename IDX>
__global__ void __launch_bounds__(kThreads, HYOWON_GATHER_MINB)
k_gather_kick(uint32_t n, const float* __restrict__ phi, const uint32_t* __restrict__ ux,
              const uint32_t* __restrict__ uy, const uint32_t* __restrict__ uz,
              const float* __restrict__ px, const float* __restrict__ py,
              const float* __restrict__ pz, float* __restrict__ ax, float* __restrict__ ay,
              float* __restrict__ az, int do_kick, float K2, float* __restrict__ pxo,
              float* __restrict__ pyo, float* __restrict__ pzo, int N, float inv_two_dx,
              unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (*status & ST_BLOCKS_PUBLISH)) return;
    // the momenta load while the stencil does (2.96 -> 2.60 ms at 512^3 / 1024^3;
    // the binary64 gather, at 48 registers with spills, was slower so)
    float p0[3] = {0.f, 0.f, 0.f};
    if (do_kick) {
        p0[0] = px[i];
        p0[1] = py[i];
        p0[2] = pz[i];
    }
    uint32_t fx, fy, fz;
    const int ix = static_cast<int>(cell_of(ux[i], N, fx));
    const int iy = static_cast<int>(cell_of(uy[i], N, fy));
    const int iz = static_cast<int>(cell_of(uz[i], N, fz));
    const int xs[4] = {ix == 0 ? N - 1 : ix - 1, ix, ix + 1 == N ? 0 : ix + 1,
                       ix + 2 >= N ? ix + 2 - N : ix + 2};
    const int ys[4] = {iy == 0 ? N - 1 : iy - 1, iy, iy + 1 == N ? 0 : iy + 1,
                       iy + 2 >= N ? iy + 2 - N : iy + 2};
    const int zs[4] = {iz == 0 ? N - 1 : iz - 1, iz, iz + 1 == N ? 0 : iz + 1,
                       iz + 2 >= N ? iz + 2 - N : iz + 2};
#define PHI(a_, b_, c_) __ldg(&phi[cell_index_t<IDX>(xs[a_], ys[b_], zs[c_], N)])
    float c[2][2][2], xm[2][2], xp[2][2], ym[2][2], yp[2][2], zm[2][2], zp[2][2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            xm[u][v] = PHI(0, u + 1, v + 1);
            xp[u][v] = PHI(3, u + 1, v + 1);
            ym[u][v] = PHI(u + 1, 0, v + 1);
            yp[u][v] = PHI(u + 1, 3, v + 1);
            zm[u][v] = PHI(u + 1, v + 1, 0);
            zp[u][v] = PHI(u + 1, v + 1, 3);
#pragma unroll
            for (int w = 0; w < 2; ++w) c[u][v][w] = PHI(u + 1, v + 1, w + 1);
        }
    }
#undef PHI
    const float tx = __uint2float_rn(fx) * 2.3283064365386963e-10f;
    const float ty = __uint2float_rn(fy) * 2.3283064365386963e-10f;
    const float tz = __uint2float_rn(fz) * 2.3283064365386963e-10f;
    const float wx[2] = {1.f - tx, tx}, wy[2] = {1.f - ty, ty}, wz[2] = {1.f - tz, tz};
    float gxs = 0.f, gys = 0.f, gzs = 0.f;
#pragma unroll
    for (int ox = 0; ox < 2; ++ox) {
#pragma unroll
        for (int oy = 0; oy < 2; ++oy) {
#pragma unroll
            for (int oz = 0; oz < 2; ++oz) {
                const float w = wx[ox] * wy[oy] * wz[oz];
                const float dxv = (ox == 0 ? c[1][oy][oz] : xp[oy][oz])
                    - (ox == 0 ? xm[oy][oz] : c[0][oy][oz]);
                const float dyv = (oy == 0 ? c[ox][1][oz] : yp[ox][oz])
                    - (oy == 0 ? ym[ox][oz] : c[ox][0][oz]);
                const float dzv = (oz == 0 ? c[ox][oy][1] : zp[ox][oy])
                    - (oz == 0 ? zm[ox][oy] : c[ox][oy][0]);
                gxs -= w * dxv;
                gys -= w * dyv;
                gzs -= w * dzv;
            }
        }
    }
    const float gx = gxs * inv_two_dx, gy = gys * inv_two_dx, gz = gzs * inv_two_dx;
    if (!(isfinite(gx) && isfinite(gy) && isfinite(gz))) raise_status(status, ST_FORCE);
    ax[i] = gx;
    ay[i] = gy;
    az[i] = gz;
    if (do_kick) {
        const float qx = fmaf(gx, K2, p0[0]);
        const float qy = fmaf(gy, K2, p0[1]);
        const float qz = fmaf(gz, K2, p0[2]);
        if (!(isfinite(qx) && isfinite(qy) && isfinite(qz))) raise_status(status, ST_KICK2);
        pxo[i] = qx;
        pyo[i] = qy;
        pzo[i] = qz;
    }
}

__global__ void k_kick_only(uint32_t n, const float* __restrict__ px, const float* __restrict__ py,
                            const float* __restrict__ pz, const float* __restrict__ ax,
                            const float* __restrict__ ay, const float* __restrict__ az, float K2,
                            float* __restrict__ pxo, float* __restrict__ pyo,
                            float* __restrict__ pzo, unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (*status & ST_BLOCKS_PUBLISH)) return;
    const float qx = fmaf(ax[i], K2, px[i]);
    const float qy = fmaf(ay[i], K2, py[i]);
    const float qz = fmaf(az[i], K2, pz[i]);
    if (!(isfinite(qx) && isfinite(qy) && isfinite(qz))) raise_status(status, ST_KICK2);
    pxo[i] = qx;
    pyo[i] = qy;
    pzo[i] = qz;
}

template <typename T>
__global__ void k_unpermute_widen(uint32_t n, const uint32_t* __restrict__ id,
                                  const T* __restrict__ src, double scale,
                                  double* __restrict__ dst) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[id[i]] = static_cast<double>(src[i]) * scale;
}

__global__ void k_widen_mesh(uint64_t cells, const float* __restrict__ r, double* __restrict__ d) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < cells;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        d[i] = static_cast<double>(r[i]);
}

__global__ void k_mass_mesh(uint64_t cells, const long long* __restrict__ q, const FixedPlan* plan,
                            double m, double* __restrict__ d) {
    const double s = ldexp(m, -3 * plan->B);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < cells;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        d[i] = static_cast<double>(q[i]) * s;
}

}  // namespace

struct State {
    double L = 0.0;
    int N = 0;
    int method = 0;
    int deconvolve = 0;
    double r_s = 0.0;
    double four_pi_G = 0.0;
    uint32_t n = 0, cap = 0;
    uint32_t* pos[2][3] = {};
    float* mom[2][3] = {};
    uint32_t* id[2] = {};
    float* acc[3] = {};
    int pc = 0, mc = 0, ic = 0;
    int ic_before = 0;
    double uniform_mass = 0.0;
    double input_mass = 0.0;
    SortWork sort{};
    uint32_t sort_cap = 0;
    uint32_t* d_max_count = nullptr;
    FixedPlan* d_plan = nullptr;
    unsigned long long* d_qsum = nullptr;
    uint32_t* order = nullptr;   // cell order of unmoved particles (steps between re-sorts)
    bool order_perm = false;     // the current positions' cell order is `order` (else identity)
    bool step_perm = false;      // same, for the positions of the step in flight
    bool order_state_invalid = true;  // offsets/order do not describe the current positions
    float* rmesh = nullptr;
    float2* modes = nullptr;
    size_t modes_elems = 0;   // 8-byte slots of `modes` (host staging between solves)
    unsigned int* d_flag = nullptr;  // input validation flag of upload
    cudaStream_t copy_stream = nullptr;  // download: device->host copies beside the kernels
    cudaEvent_t staged[2] = {}, copied[2] = {};
    float2* phi_k = nullptr;
    float* lap = nullptr;
    float* win = nullptr;
    float2* tw = nullptr;     // exp(-2 pi i m/N) (N): five-pass potential solve
    poisson::Plan* fft_plan = nullptr;  // its tensor maps of `modes`
    bool five_pass = false;   // pure PM on a power-of-two mesh: pm_poisson.cu
    cufftHandle r2c = 0, c2r = 0;
    bool plans = false;
    void* fft_work = nullptr;
    unsigned fill_blocks = 0;
    int sort_interval = 4;
    int since_sort = 0;
    int step_P = 0, step_M = 0;  // position / momentum sets of the step in flight
    bool step_sorted = false;
    uint64_t launches = 0;  // kernels launched (cuFFT's excluded)
    // TreePM short range: called between the long-range accumulation and the
    // K2 kick with the position set of the solve (null: long range alone).
    ShortRangeHook short_range = nullptr;
    void* short_ctx = nullptr;
    unsigned long long mass_check_offset = 0;  // tests of the mass-check failure path
    std::string err;
};

namespace {

int fail(State* st, int code, const std::string& m) {
    st->err = m;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(st, e_ == cudaErrorMemoryAllocation ? HYOWON_ENOMEM : HYOWON_ECUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));              \
    } while (0)

#define CKFFT(call)                                                                     \
    do {                                                                                \
        if ((call) != CUFFT_SUCCESS) return fail(st, HYOWON_ECUDA, std::string(#call)); \
    } while (0)

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    *p = nullptr;
    return cudaMalloc(reinterpret_cast<void**>(p), (count ? count : 1) * sizeof(T));
}

void free_particles(State* st) {
    for (int s = 0; s < 2; ++s) {
        for (int a = 0; a < 3; ++a) {
            cudaFree(st->pos[s][a]);
            cudaFree(st->mom[s][a]);
            st->pos[s][a] = nullptr;
            st->mom[s][a] = nullptr;
        }
        cudaFree(st->id[s]);
        st->id[s] = nullptr;
    }
    for (int a = 0; a < 3; ++a) {
        cudaFree(st->acc[a]);
        st->acc[a] = nullptr;
    }
    cudaFree(st->sort.key);
    cudaFree(st->sort.rank);
    cudaFree(st->order);
    st->order = nullptr;
    st->sort.key = st->sort.rank = nullptr;
    st->cap = 0;
}

int ensure(State* st, uint32_t n) {
    if (n > st->cap) {
        free_particles(st);
        for (int s = 0; s < 2; ++s) {
            for (int a = 0; a < 3; ++a) {
                CK(dalloc(&st->pos[s][a], n));
                CK(dalloc(&st->mom[s][a], n));
            }
            CK(dalloc(&st->id[s], n));
        }
        for (int a = 0; a < 3; ++a) CK(dalloc(&st->acc[a], n));
        CK(dalloc(&st->sort.key, n));
        CK(dalloc(&st->sort.rank, n));
        CK(dalloc(&st->order, n));
        st->cap = n;
    }
    const uint64_t cells = static_cast<uint64_t>(st->N) * st->N * st->N;
    int shift = 0;
    while (shift < 30 && (cells >> (shift + 1)) * 8 >= n && (cells >> (shift + 1)) > 0) ++shift;
    const uint32_t nb = static_cast<uint32_t>((cells + (1ull << shift) - 1) >> shift);
    st->sort.shift = shift;
    st->sort.n_buckets = nb;
    if (nb > st->sort_cap) {
        cudaFree(st->sort.count);
        cudaFree(st->sort.offset);
        cudaFree(st->sort.scan_tmp);
        CK(dalloc(&st->sort.count, nb + 1));
        CK(dalloc(&st->sort.offset, nb + 1));
        CK(dalloc(&st->sort.scan_tmp, scan_tmp_elements(nb + 1)));
        st->sort_cap = nb;
    }
    return HYOWON_OK;
}

void rec(cudaEvent_t* ev, int i, cudaStream_t s) {
    if (ev) cudaEventRecord(ev[i], s);
}

double green_c0(const State* st) {
    const double dx = st->L / st->N;
    const double n3 = static_cast<double>(st->N) * st->N * st->N;
    return st->four_pi_G * st->uniform_mass / (dx * dx * dx) / n3;
}

}  // namespace

int create(State** out, double L, int N, int method, int deconvolve, double r_s,
           const double* lap, const double* win, double four_pi_G, cudaStream_t s) {
    State* st = new State();
    *out = st;
    st->L = L;
    st->N = N;
    st->method = method;
    st->deconvolve = deconvolve;
    st->r_s = r_s;
    st->four_pi_G = four_pi_G;
    const size_t cells = static_cast<size_t>(N) * N * N;
    const size_t half = static_cast<size_t>(N) * N * (N / 2 + 1);
    CK(dalloc(&st->rmesh, cells));
    const size_t modes_n = method == HYOWON_PURE_PM && poisson::supported(N)
        ? std::max(half, poisson::modes_elements_f32(N)) : half;
    CK(dalloc(&st->modes, modes_n));
    st->modes_elems = modes_n;
    CK(dalloc(&st->d_flag, 1));
    CK(cudaStreamCreateWithFlags(&st->copy_stream, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
        CK(cudaEventCreateWithFlags(&st->staged[b], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&st->copied[b], cudaEventDisableTiming));
    }
    if (method == HYOWON_TREEPM_LONG_RANGE) CK(dalloc(&st->phi_k, half));
    CK(dalloc(&st->lap, N));
    CK(dalloc(&st->win, N));
    CK(dalloc(&st->d_max_count, 1));
    CK(dalloc(&st->d_plan, 1));
    CK(dalloc(&st->d_qsum, 1));
    std::vector<float> lf(N), wf(N);
    for (int i = 0; i < N; ++i) {
        lf[i] = static_cast<float>(lap[i]);
        wf[i] = static_cast<float>(win[i]);
    }
    CK(cudaMemcpy(st->lap, lf.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(st->win, wf.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    st->fill_blocks = static_cast<unsigned>(sms) * 8;
    if (method == HYOWON_PURE_PM && poisson::supported(N)) {
        std::vector<double> t(2 * static_cast<size_t>(N));
        poisson::twiddles(N, t.data());
        std::vector<float> tf(t.begin(), t.end());
        CK(dalloc(&st->tw, N));
        CK(cudaMemcpy(st->tw, tf.data(), sizeof(float2) * N, cudaMemcpyHostToDevice));
        const char* perr = "";
        st->fft_plan = poisson::create_plan(N, true, st->modes, &perr);
        if (!st->fft_plan) return fail(st, HYOWON_ECUDA, perr);
        st->five_pass = true;
        return HYOWON_OK;
    }
    CKFFT(cufftCreate(&st->r2c));
    CKFFT(cufftCreate(&st->c2r));
    st->plans = true;
    cufftSetAutoAllocation(st->r2c, 0);
    cufftSetAutoAllocation(st->c2r, 0);
    size_t w1 = 0, w2 = 0;
    CKFFT(cufftMakePlan3d(st->r2c, N, N, N, CUFFT_R2C, &w1));
    CKFFT(cufftMakePlan3d(st->c2r, N, N, N, CUFFT_C2R, &w2));
    CK(cudaMalloc(&st->fft_work, std::max<size_t>(1, std::max(w1, w2))));
    cufftSetWorkArea(st->r2c, st->fft_work);
    cufftSetWorkArea(st->c2r, st->fft_work);
    cufftSetStream(st->r2c, s);
    cufftSetStream(st->c2r, s);
    return HYOWON_OK;
}

void destroy(State* st) {
    if (!st) return;
    if (st->plans) {
        cufftDestroy(st->r2c);
        cufftDestroy(st->c2r);
    }
    cudaFree(st->fft_work);
    cudaFree(st->tw);
    poisson::destroy_plan(st->fft_plan);
    cudaFree(st->rmesh);
    cudaFree(st->modes);
    cudaFree(st->phi_k);
    cudaFree(st->lap);
    cudaFree(st->win);
    cudaFree(st->d_max_count);
    cudaFree(st->d_plan);
    cudaFree(st->d_qsum);
    cudaFree(st->d_flag);
    for (int b = 0; b < 2; ++b) {
        if (st->staged[b]) cudaEventDestroy(st->staged[b]);
        if (st->copied[b]) cudaEventDestroy(st->copied[b]);
    }
    if (st->copy_stream) cudaStreamDestroy(st->copy_stream);
    free_particles(st);
    cudaFree(st->sort.count);
    cudaFree(st->sort.offset);
    cudaFree(st->sort.scan_tmp);
    delete st;
}

const std::string& last_error(State* st) { return st->err; }

int upload_device(State* st, uint32_t n, double* const pos[3], double* const mom[3],
                  double uniform_mass, double total_mass, double, cudaStream_t s) {
    int rc = ensure(st, n);
    if (rc) return rc;
    st->n = n;
    st->uniform_mass = uniform_mass;
    st->input_mass = total_mass;
    st->pc = st->mc = st->ic = 0;
    CK(cudaMemsetAsync(st->d_flag, 0, sizeof(unsigned int), s));
    ++st->launches;
    k_to_fixed<<<blocks_for(n), kThreads, 0, s>>>(n, pos[0], pos[1], pos[2], mom[0], mom[1], mom[2],
                                                  st->L, st->pos[0][0], st->pos[0][1], st->pos[0][2],
                                                  st->mom[0][0], st->mom[0][1], st->mom[0][2], st->d_flag);
    ++st->launches;
    launch_iota_u32(n, st->id[0], s);
    unsigned int h = 0;
    cudaMemcpyAsync(&h, st->d_flag, sizeof(unsigned int), cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    st->order_state_invalid = true;
    if (e != cudaSuccess) return fail(st, HYOWON_ECUDA, cudaGetErrorString(e));
    if (h) return fail(st, HYOWON_EINVAL, "particle positions and momenta must be finite");
    return HYOWON_OK;
}

int upload(State* st, uint32_t n, const double* x, const double* y, const double* z,
           const double* px, const double* py, const double* pz, const double* masses,
           double uniform_mass, double total_mass, double, cudaStream_t s) {
    if (masses) return fail(st, HYOWON_EINVAL, "the FP32 fixed-point form requires a uniform particle mass");
    int rc = ensure(st, n);
    if (rc) return rc;
    st->n = n;
    st->uniform_mass = uniform_mass;
    st->input_mass = total_mass;
    st->pc = st->mc = st->ic = 0;
    // The binary64 host arrays are staged through the half-spectrum buffer,
    // which holds nothing live between force solves, in chunks of up to
    // modes_elems / 6 particles, and converted on the device chunk by chunk.
    const double* src[6] = {x, y, z, px, py, pz};
    const uint64_t per = st->modes_elems / 6;
    const uint32_t chunk = static_cast<uint32_t>(per < n ? (per > 0 ? per : 1) : n);
    double* stage = reinterpret_cast<double*>(st->modes);
    CK(cudaMemsetAsync(st->d_flag, 0, sizeof(unsigned int), s));
    for (uint32_t off = 0; off < n; off += chunk) {
        const uint32_t c = n - off < chunk ? n - off : chunk;
        const double* d[6] = {};
        for (int a = 0; a < 6; ++a) {
            if (!src[a]) continue;
            double* slot = stage + static_cast<size_t>(a) * c;
            CK(cudaMemcpyAsync(slot, src[a] + off, sizeof(double) * c, cudaMemcpyHostToDevice, s));
            d[a] = slot;
        }
        ++st->launches;
        k_to_fixed<<<blocks_for(c), kThreads, 0, s>>>(
            c, d[0], d[1], d[2], d[3], d[4], d[5], st->L, st->pos[0][0] + off, st->pos[0][1] + off,
            st->pos[0][2] + off, st->mom[0][0] + off, st->mom[0][1] + off, st->mom[0][2] + off,
            st->d_flag);
    }
    ++st->launches;
    launch_iota_u32(n, st->id[0], s);
    unsigned int h = 0;
    CK(cudaMemcpyAsync(&h, st->d_flag, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    st->order_state_invalid = true;
    if (h) return fail(st, HYOWON_EINVAL, "particle positions and momenta must be finite");
    return HYOWON_OK;
}

void validate(State*, cudaStream_t, unsigned int*) {}

int sort_current(State* st, cudaStream_t s, unsigned int* d_status) {
    const uint32_t n = st->n;
    CK(cudaMemsetAsync(st->sort.count, 0, sizeof(uint32_t) * (st->sort.n_buckets + 1), s));
    CK(cudaMemsetAsync(st->d_max_count, 0, sizeof(uint32_t), s));
    ++st->launches;
    k_key<<<blocks_for(n), kThreads, 0, s>>>(n, st->pos[st->pc][0], st->pos[st->pc][1],
                                             st->pos[st->pc][2], st->N, st->sort.shift, st->sort.key,
                                             st->sort.rank, st->sort.count, st->d_max_count);
    ++st->launches;
    k_max_count<<<st->fill_blocks, kThreads, 0, s>>>(st->sort.n_buckets, st->sort.count,
                                                     st->d_max_count);
    st->launches += launch_exclusive_scan(st->sort.count, st->sort.offset, st->sort.n_buckets + 1,
                          st->sort.scan_tmp, s);
    const uint32_t* src[7];
    uint32_t* dst[7];
    for (int a = 0; a < 3; ++a) {
        src[a] = st->pos[st->pc][a];
        dst[a] = st->pos[1 - st->pc][a];
        src[3 + a] = reinterpret_cast<const uint32_t*>(st->mom[st->mc][a]);
        dst[3 + a] = reinterpret_cast<uint32_t*>(st->mom[1 - st->mc][a]);
    }
    src[6] = st->id[st->ic];
    dst[6] = st->id[1 - st->ic];
    ++st->launches;
    launch_scatter4_multi(n, st->sort.key, st->sort.rank, st->sort.offset, 7, src, dst, nullptr, s);
    CK(cudaStreamSynchronize(s));
    (void)d_status;
    st->pc = 1 - st->pc;
    st->mc = 1 - st->mc;
    st->ic = 1 - st->ic;
    st->order_perm = false;
    st->order_state_invalid = false;
    return HYOWON_OK;
}

namespace {
int enqueue_force_sets(State* st, cudaStream_t s, unsigned int* d_status, bool kick, double K2,
                       cudaEvent_t* ev, int P, int M, const uint32_t* order);

// Owner-computes deposit of position set P into `out` (FP32 offsets for the
// transform, or exact int64), see k_deposit_tiles. With ZLOG > 0 the tiles go
// to the chunked half spectrum `H` transformed along z instead.
template <typename OUT, int ZLOG = 0>
int deposit_tiles(State* st, int P, const uint32_t* order, OUT* out, unsigned long long* qsum,
                  const unsigned int* d_status, cudaStream_t s, float2* H = nullptr) {
    const int N = st->N;
    const int TY = deposit_rows(N);
    size_t smem = 8 * static_cast<size_t>(TY) * N;
    if constexpr (ZLOG > 0) {
        // the z transform runs in the accumulators' memory
        const size_t rows = sizeof(float2) * static_cast<size_t>(N / 2) * TY;
        if (rows > smem) smem = rows;
    }
    CK(cudaFuncSetAttribute(k_deposit_tiles<OUT, ZLOG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(smem)));
    const dim3 grid((N + TY - 1) / TY, N);
    ++st->launches;
    k_deposit_tiles<OUT, ZLOG><<<grid, kDepositThreads, smem, s>>>(
        st->pos[P][0], st->pos[P][1], st->pos[P][2], order, st->sort.offset, st->sort.shift, N, TY,
        st->d_plan, out, qsum, d_status, H, st->tw);
    CK(cudaPeekAtLastError());
    return HYOWON_OK;
}

// The deposit of the five-pass solve: tiles transformed along z into st->modes.
int deposit_spectrum(State* st, int P, const uint32_t* order, unsigned long long* qsum,
                     const unsigned int* d_status, cudaStream_t s) {
    float* const none = nullptr;
    switch (st->N) {
    case 32: return deposit_tiles<float, 5>(st, P, order, none, qsum, d_status, s, st->modes);
    case 64: return deposit_tiles<float, 6>(st, P, order, none, qsum, d_status, s, st->modes);
    case 128: return deposit_tiles<float, 7>(st, P, order, none, qsum, d_status, s, st->modes);
    case 256: return deposit_tiles<float, 8>(st, P, order, none, qsum, d_status, s, st->modes);
    case 512: return deposit_tiles<float, 9>(st, P, order, none, qsum, d_status, s, st->modes);
    case 1024: return deposit_tiles<float, 10>(st, P, order, none, qsum, d_status, s, st->modes);
    case 2048: return deposit_tiles<float, 11>(st, P, order, none, qsum, d_status, s, st->modes);
    default: return fail(st, HYOWON_ELOGIC, "five-pass deposit on a mesh the solve does not support");
    }
}
}

int enqueue_force(State* st, cudaStream_t s, unsigned int* d_status, bool kick, double K2,
                  cudaEvent_t* ev) {
    if (st->order_state_invalid) {
        const int rc = sort_current(st, s, d_status);
        if (rc) return rc;
    }
    return enqueue_force_sets(st, s, d_status, kick, K2, ev, st->pc, st->mc,
                              st->order_perm ? st->order : nullptr);
}

namespace {
int enqueue_force_sets(State* st, cudaStream_t s, unsigned int* d_status, bool kick, double K2,
                       cudaEvent_t* ev, int P, int M, const uint32_t* order) {
    const uint32_t n = st->n;
    const int N = st->N;
    const uint64_t cells = static_cast<uint64_t>(N) * N * N;
    const uint64_t half = static_cast<uint64_t>(N) * N * (N / 2 + 1);
    rec(ev, 1, s);
    ++st->launches;
    k_plan<<<1, 32, 0, s>>>(n, cells, st->d_max_count, green_c0(st), 1, st->d_plan);
    CK(cudaMemsetAsync(st->d_qsum, 0, sizeof(unsigned long long), s));
    int rc = st->five_pass ? deposit_spectrum(st, P, order, st->d_qsum, d_status, s)
                           : deposit_tiles<float>(st, P, order, st->rmesh, st->d_qsum, d_status, s);
    if (rc) return rc;
    ++st->launches;
    k_check_mass<<<1, 32, 0, s>>>(st->d_qsum, st->d_plan, st->mass_check_offset, d_status);
    float* const pxo = st->mom[1 - M][0];
    float* const pyo = st->mom[1 - M][1];
    float* const pzo = st->mom[1 - M][2];
    const float K2f = static_cast<float>(K2);
    if (st->five_pass) {
        rec(ev, 2, s);
        int k = poisson::forward_columns_f32(st->fft_plan, N, st->modes, st->tw, d_status, s);
        if (k < 0) return fail(st, HYOWON_ECUDA, "potential solve: forward pass launch failed");
        st->launches += k;
        rec(ev, 3, s);
        const float* c_green = reinterpret_cast<const float*>(
            reinterpret_cast<const char*>(st->d_plan) + offsetof(FixedPlan, c_green));
        const poisson::GreenF32 g{st->lap, st->win, st->deconvolve, c_green};
        k = poisson::green_f32(st->fft_plan, N, st->modes, st->tw, g, d_status, s);
        if (k < 0) return fail(st, HYOWON_ECUDA, "potential solve: Green pass launch failed");
        st->launches += k;
        rec(ev, 4, s);
        k = poisson::inverse_f32(st->fft_plan, N, st->modes, st->rmesh, st->tw, d_status, s);
        if (k < 0) return fail(st, HYOWON_ECUDA, "potential solve: inverse pass launch failed");
        st->launches += k;
        rec(ev, 5, s);
        const float inv_two_dx = static_cast<float>(1.0 / (2.0 * st->L / N));
        ++st->launches;
        if (cells_fit_u32(N))
            k_gather_kick<uint32_t><<<blocks_for(n), kThreads, 0, s>>>(
                n, st->rmesh, st->pos[P][0], st->pos[P][1], st->pos[P][2],
                st->mom[M][0], st->mom[M][1], st->mom[M][2], st->acc[0], st->acc[1],
                st->acc[2], kick ? 1 : 0, K2f, pxo, pyo, pzo, N, inv_two_dx, d_status);
        else
            k_gather_kick<uint64_t><<<blocks_for(n), kThreads, 0, s>>>(
                n, st->rmesh, st->pos[P][0], st->pos[P][1], st->pos[P][2],
                st->mom[M][0], st->mom[M][1], st->mom[M][2], st->acc[0], st->acc[1],
                st->acc[2], kick ? 1 : 0, K2f, pxo, pyo, pzo, N, inv_two_dx, d_status);
        rec(ev, 6, s);
        return HYOWON_OK;
    }
    rec(ev, 2, s);
    CKFFT(cufftExecR2C(st->r2c, st->rmesh, reinterpret_cast<cufftComplex*>(st->modes)));
    rec(ev, 3, s);
    if (st->method == HYOWON_PURE_PM) {
        ++st->launches;
        k_green<<<blocks_for(half), kThreads, 0, s>>>(N, st->modes, st->lap, st->win, st->deconvolve,
                                                      st->d_plan);
        rec(ev, 4, s);
        CKFFT(cufftExecC2R(st->c2r, reinterpret_cast<cufftComplex*>(st->modes), st->rmesh));
        rec(ev, 5, s);
        const float inv_two_dx = static_cast<float>(1.0 / (2.0 * st->L / N));
        ++st->launches;
        if (cells_fit_u32(N))
            k_gather_kick<uint32_t><<<blocks_for(n), kThreads, 0, s>>>(
                n, st->rmesh, st->pos[P][0], st->pos[P][1], st->pos[P][2],
                st->mom[M][0], st->mom[M][1], st->mom[M][2], st->acc[0], st->acc[1],
                st->acc[2], kick ? 1 : 0, K2f, pxo, pyo, pzo, N, inv_two_dx, d_status);
        else
            k_gather_kick<uint64_t><<<blocks_for(n), kThreads, 0, s>>>(
                n, st->rmesh, st->pos[P][0], st->pos[P][1], st->pos[P][2],
                st->mom[M][0], st->mom[M][1], st->mom[M][2], st->acc[0], st->acc[1],
                st->acc[2], kick ? 1 : 0, K2f, pxo, pyo, pzo, N, inv_two_dx, d_status);
        rec(ev, 6, s);
        return HYOWON_OK;
    }
    ++st->launches;
    k_green_spectral<<<blocks_for(half), kThreads, 0, s>>>(N, st->L, st->modes, st->win,
                                                           static_cast<float>(st->r_s), st->d_plan);
    CK(cudaMemcpyAsync(st->phi_k, st->modes, sizeof(float2) * half, cudaMemcpyDeviceToDevice, s));
    rec(ev, 4, s);
    for (int a = 0; a < 3; ++a) {
        CK(cudaMemsetAsync(st->acc[a], 0, sizeof(float) * n, s));
        ++st->launches;
        k_spectral_axis<<<blocks_for(half), kThreads, 0, s>>>(N, st->L, a, st->phi_k, st->modes);
        CKFFT(cufftExecC2R(st->c2r, reinterpret_cast<cufftComplex*>(st->modes), st->rmesh));
        ++st->launches;
        k_interp_add<<<blocks_for(n), kThreads, 0, s>>>(n, st->rmesh, st->pos[P][0],
                                                        st->pos[P][1], st->pos[P][2], N,
                                                        st->acc[a], d_status);
    }
    if (st->short_range) {
        const int rc = st->short_range(st->short_ctx, s, P);
        if (rc) return rc;
    }
    rec(ev, 5, s);
    if (kick) {
        ++st->launches;
        k_kick_only<<<blocks_for(n), kThreads, 0, s>>>(n, st->mom[M][0], st->mom[M][1],
                                                       st->mom[M][2], st->acc[0], st->acc[1],
                                                       st->acc[2], K2f, pxo, pyo, pzo, d_status);
    }
    rec(ev, 6, s);
    return HYOWON_OK;
}
}  // namespace

int kdk_step(State* st, cudaStream_t s, unsigned int* d_status, unsigned long long* d_maxdrift,
             double K1, double D, double K2, cudaEvent_t* ev) {
    const uint32_t n = st->n;
    const bool sort_now = st->sort_interval <= 1 || st->since_sort + 1 >= st->sort_interval;
    CK(cudaMemsetAsync(d_status, 0, sizeof(unsigned int), s));
    CK(cudaMemsetAsync(d_maxdrift, 0, sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(st->sort.count, 0, sizeof(uint32_t) * (st->sort.n_buckets + 1), s));
    CK(cudaMemsetAsync(st->d_max_count, 0, sizeof(uint32_t), s));
    rec(ev, 0, s);
    const int pc = st->pc, mc = st->mc;
    ++st->launches;
    k_kick_drift_key<<<stream_blocks(n, kThreads), kThreads, 0, s>>>(
        n, st->pos[pc][0], st->pos[pc][1], st->pos[pc][2], st->mom[mc][0], st->mom[mc][1],
        st->mom[mc][2], st->acc[0], st->acc[1], st->acc[2], static_cast<float>(K1), D,
        kTwo32 / st->L, st->N, st->pos[1 - pc][0], st->pos[1 - pc][1], st->pos[1 - pc][2],
        st->mom[1 - mc][0], st->mom[1 - mc][1], st->mom[1 - mc][2], st->sort.shift,
        1, st->sort.key, st->sort.rank, st->sort.count, st->d_max_count, d_maxdrift, d_status);
    st->step_sorted = sort_now;
    st->ic_before = st->ic;
    int P = 1 - pc, M = 1 - mc;
    // cell order of the candidate positions: bucket offsets every step; the
    // particle arrays themselves are permuted only on re-sort steps
    st->launches += launch_exclusive_scan(st->sort.count, st->sort.offset, st->sort.n_buckets + 1,
                                          st->sort.scan_tmp, s);
    st->step_perm = !sort_now;
    if (!sort_now) {
        ++st->launches;
        launch_order(n, st->sort.key, st->sort.rank, st->sort.offset, st->order, d_status, s);
    }
    if (sort_now) {
        const uint32_t* src[7];
        uint32_t* dst[7];
        for (int a = 0; a < 3; ++a) {
            src[a] = st->pos[1 - pc][a];
            dst[a] = st->pos[pc][a];
            src[3 + a] = reinterpret_cast<const uint32_t*>(st->mom[1 - mc][a]);
            dst[3 + a] = reinterpret_cast<uint32_t*>(st->mom[mc][a]);
        }
        src[6] = st->id[st->ic];
        dst[6] = st->id[1 - st->ic];
        ++st->launches;
        launch_scatter4_multi(n, st->sort.key, st->sort.rank, st->sort.offset, 7, src, dst,
                              d_status, s);
        st->ic = 1 - st->ic;
        P = pc;
        M = mc;
    }
    ++st->launches;
    k_max_count<<<st->fill_blocks, kThreads, 0, s>>>(st->sort.n_buckets, st->sort.count,
                                                     st->d_max_count);
    st->step_P = P;
    st->step_M = M;
    return enqueue_force_sets(st, s, d_status, true, K2, ev, P, M,
                              st->step_perm ? st->order : nullptr);
}

uint64_t launches(const State* st) { return st->launches; }

void set_sort_interval(State* st, int steps) { st->sort_interval = steps < 1 ? 1 : steps; }

void commit_step(State* st, bool published, bool ok) {
    if (!published) {
        st->ic = st->ic_before;
        st->order_state_invalid = true;  // offsets describe the unpublished candidate
        return;
    }
    st->order_perm = st->step_perm;
    st->order_state_invalid = false;
    st->pc = st->step_P;
    st->mc = ok ? 1 - st->step_M : st->step_M;
    st->since_sort = st->step_sorted ? 0 : st->since_sort + 1;
}

int download(State* st, cudaStream_t s, double* x, double* y, double* z, double* px, double* py,
             double* pz, double* ax, double* ay, double* az) {
    const uint32_t n = st->n;
    // Widened components are scattered back to the original particle order in
    // staging arrays of n doubles: two in the half-spectrum buffer when it
    // holds 2n slots (it holds nothing live between force solves; the
    // potential mesh is left intact), so that the scatter of one component on
    // the handle's stream overlaps the device-to-host copy of the previous one
    // on the copy stream; else one (in the buffer, or a temporary allocation).
    double* stage[2] = {};
    int nstage = 1;
    bool owned = false;
    if (st->modes_elems >= 2ull * n) {
        stage[0] = reinterpret_cast<double*>(st->modes);
        stage[1] = stage[0] + n;
        nstage = 2;
    } else if (st->modes_elems >= n) {
        stage[0] = reinterpret_cast<double*>(st->modes);
    } else {
        CK(dalloc(&stage[0], n));
        owned = true;
    }
    double* outs[9] = {x, y, z, px, py, pz, ax, ay, az};
    const double pos_scale = st->L / kTwo32;
    int rc = HYOWON_OK;
    int j = 0;
    for (int a = 0; a < 9 && rc == HYOWON_OK; ++a) {
        if (!outs[a]) continue;
        const int b = j % nstage;
        if (j >= nstage && cudaStreamWaitEvent(s, st->copied[b], 0) != cudaSuccess) {
            rc = fail(st, HYOWON_ECUDA, "download: stream wait failed");
            break;
        }
        ++st->launches;
        if (a < 3)
            k_unpermute_widen<uint32_t><<<blocks_for(n), kThreads, 0, s>>>(n, st->id[st->ic],
                                                                         st->pos[st->pc][a], pos_scale, stage[b]);
        else if (a < 6)
            k_unpermute_widen<float><<<blocks_for(n), kThreads, 0, s>>>(n, st->id[st->ic],
                                                                      st->mom[st->mc][a - 3], 1.0, stage[b]);
        else
            k_unpermute_widen<float><<<blocks_for(n), kThreads, 0, s>>>(n, st->id[st->ic],
                                                                      st->acc[a - 6], 1.0, stage[b]);
        if (cudaEventRecord(st->staged[b], s) != cudaSuccess
            || cudaStreamWaitEvent(st->copy_stream, st->staged[b], 0) != cudaSuccess
            || cudaMemcpyAsync(outs[a], stage[b], sizeof(double) * n, cudaMemcpyDeviceToHost,
                               st->copy_stream) != cudaSuccess
            || cudaEventRecord(st->copied[b], st->copy_stream) != cudaSuccess)
            rc = fail(st, HYOWON_ECUDA, "download copy failed");
        ++j;
    }
    if (cudaStreamSynchronize(st->copy_stream) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        rc = rc ? rc : fail(st, HYOWON_ECUDA, "download copy failed");
    if (owned) cudaFree(stage[0]);
    return rc;
}

void snapshot_view(State* st, snapshot::Component pos[3], snapshot::Component mom[3],
                   const uint32_t** id, double** stage, uint64_t* stage_doubles) {
    for (int a = 0; a < 3; ++a) {
        pos[a] = {st->pos[st->pc][a], snapshot::kFixedU32, st->L / kTwo32};
        mom[a] = {st->mom[st->mc][a], snapshot::kF32, 1.0};
    }
    *id = st->id[st->ic];
    *stage = reinterpret_cast<double*>(st->modes);
    *stage_doubles = st->modes_elems;
}

__global__ void k_widen_positions(uint32_t n, const uint32_t* __restrict__ u, double scale,
                                  double* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<double>(u[i]) * scale;
}

int positions_f64(State* st, cudaStream_t s, double* x, double* y, double* z) {
    return positions_f64_of_set(st, s, st->pc, x, y, z);
}

int positions_f64_of_set(State* st, cudaStream_t s, int P, double* x, double* y, double* z) {
    double* outs[3] = {x, y, z};
    for (int a = 0; a < 3; ++a) {
        ++st->launches;
        k_widen_positions<<<blocks_for(st->n), kThreads, 0, s>>>(st->n, st->pos[P][a],
                                                                 st->L / kTwo32, outs[a]);
    }
    CK(cudaPeekAtLastError());
    return HYOWON_OK;
}

__global__ void k_add_acc(uint32_t n, const double* __restrict__ ax, const double* __restrict__ ay,
                          const double* __restrict__ az, float* __restrict__ gx,
                          float* __restrict__ gy, float* __restrict__ gz) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    gx[i] += static_cast<float>(ax[i]);
    gy[i] += static_cast<float>(ay[i]);
    gz[i] += static_cast<float>(az[i]);
}

int add_accelerations(State* st, cudaStream_t s, const double* ax, const double* ay,
                      const double* az) {
    ++st->launches;
    k_add_acc<<<blocks_for(st->n), kThreads, 0, s>>>(st->n, ax, ay, az, st->acc[0], st->acc[1],
                                                     st->acc[2]);
    CK(cudaPeekAtLastError());
    return HYOWON_OK;
}

void set_mass_check_offset(State* st, unsigned long long units) { st->mass_check_offset = units; }

void set_wait_limit(State* st, unsigned polls) { poisson::set_wait_limit(st->fft_plan, polls); }

void set_short_range_hook(State* st, ShortRangeHook fn, void* ctx) {
    st->short_range = fn;
    st->short_ctx = ctx;
}

const uint32_t* current_ids(State* st) { return st->id[st->ic]; }

int diagnostics(State* st, cudaStream_t s, bool with_potential, double* scratch, double* sums) {
    diag::InputsF32 in{};
    in.n = st->n;
    in.ux = st->pos[st->pc][0];
    in.uy = st->pos[st->pc][1];
    in.uz = st->pos[st->pc][2];
    in.px = st->mom[st->mc][0];
    in.py = st->mom[st->mc][1];
    in.pz = st->mom[st->mc][2];
    in.ax = st->acc[0];
    in.ay = st->acc[1];
    in.az = st->acc[2];
    in.uniform_mass = st->uniform_mass;
    in.phi = with_potential ? st->rmesh : nullptr;
    in.N = st->N;
    in.inv_dx = static_cast<double>(st->N) / st->L;
    const int k = diag::launch_f32(in, scratch, s);
    if (k < 0) return fail(st, HYOWON_ECUDA, "diagnostics launch failed");
    st->launches += k;
    CK(cudaMemcpyAsync(sums, scratch + diag::partial_doubles(), sizeof(double) * diag::kTerms,
                       cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return HYOWON_OK;
}

int download_potential(State* st, cudaStream_t s, double* phi) {
    const uint64_t cells = static_cast<uint64_t>(st->N) * st->N * st->N;
    double* d = nullptr;
    CK(dalloc(&d, cells));
    ++st->launches;
    k_widen_mesh<<<st->fill_blocks, kThreads, 0, s>>>(cells, st->rmesh, d);
    const cudaError_t e = cudaMemcpyAsync(phi, d, sizeof(double) * cells, cudaMemcpyDeviceToHost, s);
    const cudaError_t e2 = cudaStreamSynchronize(s);
    cudaFree(d);
    if (e != cudaSuccess || e2 != cudaSuccess) return fail(st, HYOWON_ECUDA, "potential copy failed");
    return HYOWON_OK;
}

int download_mass_mesh(State* st, cudaStream_t s, unsigned int* d_status, double* mesh) {
    const uint32_t n = st->n;
    const uint64_t cells = static_cast<uint64_t>(st->N) * st->N * st->N;
    if (st->order_state_invalid) {
        const int rc = sort_current(st, s, d_status);
        if (rc) return rc;
    }
    ++st->launches;
    k_plan<<<1, 32, 0, s>>>(n, cells, st->d_max_count, green_c0(st), 0, st->d_plan);
    CK(cudaMemsetAsync(d_status, 0, sizeof(unsigned int), s));
    long long* q = nullptr;
    CK(dalloc(&q, cells));
    int rc = deposit_tiles<long long>(st, st->pc, st->order_perm ? st->order : nullptr, q, nullptr,
                                      d_status, s);
    double* d = nullptr;
    if (rc == HYOWON_OK && dalloc(&d, cells) != cudaSuccess) rc = fail(st, HYOWON_ENOMEM, "mass mesh staging");
    if (rc == HYOWON_OK) {
        ++st->launches;
        k_mass_mesh<<<st->fill_blocks, kThreads, 0, s>>>(cells, q, st->d_plan, st->uniform_mass, d);
        const cudaError_t e = cudaMemcpyAsync(mesh, d, sizeof(double) * cells, cudaMemcpyDeviceToHost, s);
        const cudaError_t e2 = cudaStreamSynchronize(s);
        if (e != cudaSuccess || e2 != cudaSuccess) rc = fail(st, HYOWON_ECUDA, "mass mesh copy failed");
    }
    cudaFree(d);
    cudaFree(q);
    return rc;
}

}  // namespace hyowon::fp32
