// pm_chunk.cuh -- the kz-chunked half-spectrum layout of the potential solve on
// power-of-two meshes, and the row r2c that fills it. Shared by the transform
// passes (pm_poisson.cu) and by the deposits that transform their finished
// tiles along z before writing them (pm_fp32.cu, pm_fp64.cu), so both produce
// the same spectrum layout with the same arithmetic.
//
// Element (kx, ky, kz) of the half spectrum of an N^3 mesh sits at
// (kz / CC) N^2 CC + (kx N + ky) CC + kz % CC: chunks of CC complex values
// (64 bytes: CC = 8 FP32 / 4 FP64, half that at N = 2048), kz-chunk-major. The
// last chunk holds the Nyquist plane kz = N/2 and CC-1 unused columns.
#pragma once

#include <cstddef>

#include "pm_fft.cuh"

#ifndef HYOWON_FFT_CC32
#define HYOWON_FFT_CC32 8
#endif
#ifndef HYOWON_FFT_CC64
#define HYOWON_FFT_CC64 4
#endif

namespace hyowon {
namespace chunked {

using fft::cx_t;

template <typename T, int LOG2N> struct Columns;
template <int LOG2N> struct Columns<float, LOG2N> {
    static constexpr int CC = LOG2N >= 11 ? (HYOWON_FFT_CC32 > 4 ? 4 : HYOWON_FFT_CC32) : HYOWON_FFT_CC32;
};
template <int LOG2N> struct Columns<double, LOG2N> {
    static constexpr int CC = LOG2N >= 11 ? (HYOWON_FFT_CC64 > 2 ? 2 : HYOWON_FFT_CC64) : HYOWON_FFT_CC64;
};

template <typename T, int LOG2N> struct Layout {
    static constexpr int N = 1 << LOG2N;
    static constexpr int M = N / 2;          // complex length of a packed row
    static constexpr int Hz = M + 1;         // half-complex row length
    static constexpr int K = M / 2 + 1;      // (k, M-k) pairs of a row
    static constexpr int CC = Columns<T, LOG2N>::CC;
    static constexpr int KC = (Hz + CC - 1) / CC;                     // kz chunks
    static constexpr size_t chunk = static_cast<size_t>(N) * N * CC;  // elements per chunk
    __device__ static __forceinline__ size_t at(int kx, int ky, int kz) {
        return static_cast<size_t>(kz / CC) * chunk + (static_cast<size_t>(kx) * N + ky) * CC + (kz % CC);
    }
};

// Unpacks R transformed rows, sm[k * S + r] = Z_r[k] (the length-N/2 forward
// transform of row r's N reals read as N/2 complex values), into
// X[k] = E[k] + W_N^k O[k] with E/O the transforms of the even/odd samples,
// for k = 0..N/2, and stores them to the chunked spectrum H at rows
// (x, y0 .. y0+R-1). All `nthreads` threads take part. Consecutive threads
// take consecutive kz of a chunk row (ROW_FAST false: 64-byte runs of H per
// row) or consecutive rows of one kz (ROW_FAST true: for dense rows, S = R,
// whose shared-memory reads are then one contiguous block per warp).
template <typename T, int LOG2N, int R, int S, bool ROW_FAST = false>
__device__ __forceinline__ void rows_unpack(const cx_t<T>* sm, const cx_t<T>* __restrict__ tw,
                                            cx_t<T>* __restrict__ H, int x, int y0, int tid,
                                            int nthreads) {
    using L = Layout<T, LOG2N>;
    using C = cx_t<T>;
    const T half = static_cast<T>(0.5);
    constexpr int KP = (L::K + L::CC - 1) / L::CC;   // chunks covering k = 0..M/2
    for (int e = tid; e < KP * R * L::CC; e += nthreads) {
        const int ki = ROW_FAST ? (e / R) % L::CC : e % L::CC;
        const int r = ROW_FAST ? e % R : (e / L::CC) % R;
        const int k = (e / (L::CC * R)) * L::CC + ki;
        if (k >= L::K) continue;
        const C zk = sm[k * S + r];
        const C zm = sm[((L::M - k) & (L::M - 1)) * S + r];
        const C w = __ldg(&tw[k]);
        const C E = fft::mk(half * (zk.x + zm.x), half * (zk.y - zm.y));
        const T dx = zk.x - zm.x;
        const T dy = zk.y + zm.y;
        const C O = fft::mk(half * dy, -half * dx);        // (zk - conj(zm)) / 2i
        H[L::at(x, y0 + r, k)] = fft::cadd(E, fft::cmul(w, O));
        if (L::M - k != k) {
            const C E2 = fft::mk(E.x, -E.y);
            const C O2 = fft::mk(half * dy, half * dx);    // (zm - conj(zk)) / 2i
            const C w2 = fft::mk(-w.x, w.y);               // W_N^(M-k) = -conj(W_N^k)
            H[L::at(x, y0 + r, L::M - k)] = fft::cadd(E2, fft::cmul(w2, O2));
        }
    }
}

// r2c of R consecutive rows (x, y0 .. y0+R-1) whose N reals sit packed in
// shared memory as N/2 complex values, sm[k * S + r] = (row r [2k], row r
// [2k+1]): a length-N/2 forward transform, then rows_unpack. Every thread of
// the block calls it (the transform's barriers); threads [0, R N/(2 EPT))
// carry the transform, EPT elements each (8 or 16), all `nthreads` the
// stores. The caller has synchronised after filling sm.
template <typename T, int LOG2N, int R, int S, int EPT = 16>
__device__ __forceinline__ void rows_r2c(cx_t<T>* sm, const cx_t<T>* __restrict__ tw,
                                         cx_t<T>* __restrict__ H, int x, int y0, int tid,
                                         int nthreads) {
    using L = Layout<T, LOG2N>;
    constexpr int P = L::M / EPT;   // butterfly groups per row
    fft::smem_fft<LOG2N - 1, -1, R, S, EPT>(sm, tw, L::N, tid % R, tid / R, tid < R * P);
    rows_unpack<T, LOG2N, R, S>(sm, tw, H, x, y0, tid, nthreads);
}

// The r2c of a finished deposit tile of TY rows (x, y0 .. y0+TY-1): the
// first radix-8 stage reads its inputs straight from the tile's accumulators
// (pair(r, k) returns cells 2k and 2k+1 of row r as one complex value, each
// pair read once), every thread's reads end before the first write, and the
// transform then runs in place in the accumulators' shared memory `sm` (at
// least N/2 TY complex values): rows of TY dense columns, the first stage's
// output rows permuted so that no stage has bank conflicts, then rows_unpack.
// Every thread of the block calls it; threads [0, TY N/16) carry the transform.
template <typename T, int LOG2N, int TY, typename PAIR>
__device__ __forceinline__ void tile_r2c(PAIR pair, cx_t<T>* sm, const cx_t<T>* __restrict__ tw,
                                         cx_t<T>* __restrict__ H, int x, int y0, int tid,
                                         int nthreads) {
    using L = Layout<T, LOG2N>;
    using C = cx_t<T>;
    constexpr int E = 8;
    constexpr int LOG2M = LOG2N - 1;
    constexpr int M = L::M;
    constexpr int P = M / E;
    constexpr int S = TY;
    // row groups a 128-byte bank row holds: the first stage's lanes write rows
    // 8 j + r, spread over them by the permutation
    constexpr int Q = 128 / (TY * static_cast<int>(sizeof(C))) > 1
                          ? 128 / (TY * static_cast<int>(sizeof(C))) : 1;
    constexpr int MASK = Q - 1;
    constexpr int nE = LOG2M / 3;
    constexpr int rem = LOG2M % 3;
    static_assert(LOG2M >= 3, "rows of at least 16 cells");
    const bool active = tid < TY * P;
    const int c = tid % TY;
    const int j = tid / TY;
    C v[E];
    if (active) {
#pragma unroll
        for (int r = 0; r < E; ++r) v[r] = pair(c, j + r * (M / E));
    }
    __syncthreads();
    if (active) {
        fft::dft<E, -1>(v);
#pragma unroll
        for (int r = 0; r < E; ++r) sm[fft::row_at<true, 3, MASK>(j * E + r) * S + c] = v[r];
    }
    __syncthreads();
    int Ns = E;
    if constexpr (nE >= 2) {
        fft::smem_stage<LOG2M, E, -1, TY, S, E, true, false, MASK>(sm, Ns, tw, L::N, c, j, active);
        Ns *= E;
#pragma unroll 1
        for (int s = 2; s < nE; ++s) {
            fft::smem_stage<LOG2M, E, -1, TY, S, E>(sm, Ns, tw, L::N, c, j, active);
            Ns *= E;
        }
        if constexpr (rem != 0)
            fft::smem_stage<LOG2M, (1 << rem), -1, TY, S, E>(sm, Ns, tw, L::N, c, j, active);
    } else if constexpr (rem != 0) {
        fft::smem_stage<LOG2M, (1 << rem), -1, TY, S, E, true, false, MASK>(sm, Ns, tw, L::N, c, j,
                                                                           active);
    }
    rows_unpack<T, LOG2N, TY, S, true>(sm, tw, H, x, y0, tid, nthreads);
}

}  // namespace chunked
}  // namespace hyowon
