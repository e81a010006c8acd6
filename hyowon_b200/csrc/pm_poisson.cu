// pm_poisson.cu -- pure-PM potential solve on power-of-two meshes in five
// passes over HBM (see pm_poisson.h for the pass structure).
//
// The half spectrum is held kz-chunk-major: H[kc][kx][ky][kzc] with
// kz = kc * CC + kzc, CC = 8 FP32 / 4 FP64 complex values (64 bytes; half
// that at N = 2048), so
//  * a y-pass tile (kc, kx) is one contiguous N * 64-byte block,
//  * an x-pass tile (kc, ky) reads 64-byte runs inside one N^2 * 64-byte
//    chunk (a small page footprint instead of the whole 4-8 GB mesh),
//  * a z-pass block of CZ consecutive rows writes CZ * 64 contiguous bytes
//    per chunk.
// The last chunk holds the Nyquist plane kz = N/2 and CC-1 unused columns
// (memory and transform work +1/(N/(2 CC)+1)).
//
// Bytes moved per solve on an N^3 mesh with b-byte reals: z forward reads the
// N^3 mass values and writes H; the y forward, x (forward, Green's multiply,
// inverse) and y inverse passes read and write H in place; z inverse reads H
// and writes the N^3 potential.
#include "pm_poisson.h"

#include "pm_chunk.cuh"
#include "pm_common.cuh"
#include "pm_fft.cuh"
#include "pm_tma.cuh"

#include <cuda.h>

#include <cmath>
#include <new>

namespace hyowon {
namespace poisson {

// Tensor maps of the chunked half spectrum viewed as a 3-D array of 8-byte
// units: (units per row = CC complex, ky, kc * N + kx). `y` loads a y-pass
// tile in boxes of (units, box, 1), `x` an x-pass tile in boxes of
// (units, 1, box).
struct Plan {
    CUtensorMap y;
    CUtensorMap x;
    int N = 0;
    bool fp32 = false;
    unsigned wait_limit = 1u << 24;  // polls of a pipeline wait before a block gives up
};

namespace {

using fft::cx_t;
using fft::mk;

// Tuning: sequences per block of the z passes (rows) and of the y/x passes
// (columns), and the blocks per SM the register budget is sized for.
#ifndef HYOWON_FFT_CZ32
#define HYOWON_FFT_CZ32 16
#endif
#ifndef HYOWON_FFT_CZ64
#define HYOWON_FFT_CZ64 8
#endif
#ifndef HYOWON_FFT_MINB_Z
#define HYOWON_FFT_MINB_Z 2
#endif
#ifndef HYOWON_FFT_NBUF64
#define HYOWON_FFT_NBUF64 2
#endif
#ifndef HYOWON_FFT_NBUF
#define HYOWON_FFT_NBUF 2
#endif
#ifndef HYOWON_FFT_MINB_C32
#define HYOWON_FFT_MINB_C32 1
#endif
#ifndef HYOWON_FFT_MINB_C64
#define HYOWON_FFT_MINB_C64 1
#endif
// Column passes on meshes of 256 and more: each tile's CC columns are split
// into HYOWON_FFT_SPLIT blocks of CC / SPLIT columns (half-width TMA boxes of
// the same 64-byte rows), so that SPLIT independent blocks share an SM and one
// block's barrier waits overlap the other's arithmetic.
#ifndef HYOWON_FFT_SPLIT
#define HYOWON_FFT_SPLIT 1
#endif
// Elements each thread of a column pass holds (16: radix-16 stages, CC N / 16
// threads a tile; 8: radix-8 stages and twice the threads, measured slower on
// B200 at N = 1024: 3.66 against 3.32 ms for the FP32 x pass).
#ifndef HYOWON_FFT_EPT
#define HYOWON_FFT_EPT 16
#endif

template <typename T, int LOG2N> struct Shape;
template <int LOG2N> struct Shape<float, LOG2N> {
    static constexpr int CZ = LOG2N >= 11 ? (HYOWON_FFT_CZ32 > 8 ? 8 : HYOWON_FFT_CZ32) : HYOWON_FFT_CZ32;
};
template <int LOG2N> struct Shape<double, LOG2N> {
    static constexpr int CZ = LOG2N >= 11 ? (HYOWON_FFT_CZ64 > 4 ? 4 : HYOWON_FFT_CZ64) : HYOWON_FFT_CZ64;
};

template <typename T, int LOG2N> struct Geo : chunked::Layout<T, LOG2N> {
    using C = cx_t<T>;
    using L = chunked::Layout<T, LOG2N>;
    using L::N;
    using L::M;
    using L::Hz;
    using L::K;
    using L::CC;
    using L::KC;
    using L::chunk;
    static constexpr int CZ = Shape<T, LOG2N>::CZ;
    static constexpr int SZ = CZ + 1;
    static constexpr int TZ = CZ * M / 16;   // threads of a z-pass block
    static constexpr int PZ = CZ * M / TZ;   // row pairs each z-pass thread loads (16)
    static constexpr int QZ = (KC * CZ * CC + TZ - 1) / TZ;  // chunked values per z-pass thread
    static constexpr size_t smem_zf = sizeof(C) * M * SZ;
    static constexpr size_t smem_zi = sizeof(C) * Hz * SZ;
    static constexpr int box = N < 256 ? N : 256;                 // TMA box rows
    // column passes: a tile is N rows of CC columns, split into SP blocks of
    // CB columns; each block keeps nbuf_b of its parts in shared memory
    // (HYOWON_FFT_NBUF deep where shared memory allows)
    static constexpr int SP = (LOG2N >= 8 && CC % HYOWON_FFT_SPLIT == 0) ? HYOWON_FFT_SPLIT : 1;
    static constexpr int CB = CC / SP;
    static constexpr int EC = HYOWON_FFT_EPT == 8 ? 8 : 16;  // elements per thread
    static constexpr int TCB = CB * N / EC;                       // threads of a column block
    static constexpr unsigned tile_bytes_b = sizeof(C) * N * CB;  // one block's part of a tile
    static constexpr int nbuf_want = sizeof(T) == 4 ? HYOWON_FFT_NBUF : HYOWON_FFT_NBUF64;
    static constexpr int nbuf_b = (nbuf_want * tile_bytes_b <= 200u * 1024u) ? nbuf_want : 2;
    static constexpr size_t smem_cb = static_cast<size_t>(nbuf_b) * tile_bytes_b;
    static constexpr int units_b = CB * static_cast<int>(sizeof(C)) / 8;  // 8-byte units per part row
    static constexpr int units = CC * static_cast<int>(sizeof(C)) / 8;  // 8-byte units per row
    // column-pass blocks per SM the registers are sized for: FP32 blocks of
    // fewer than 512 threads (N <= 512) get several per SM, as many as make
    // 512 threads and their shared memory allows (at N = 512: 2, at most 128
    // registers, where the compiler would take 180 and fit one)
    static constexpr int smem_blocks = static_cast<int>((227u * 1024u) / smem_cb);
    static constexpr int minb_want = sizeof(T) == 4 ? (512 / TCB > HYOWON_FFT_MINB_C32 ? 512 / TCB : HYOWON_FFT_MINB_C32)
                                                    : HYOWON_FFT_MINB_C64;
    static constexpr int minb_c = SP * (minb_want < smem_blocks ? minb_want : (smem_blocks > 0 ? smem_blocks : 1));
};

// Buffers and blocks per SM of a column pass. The x pass (MODE 1: two
// transforms and the Green's multiply per tile) holds one tile buffer per
// block and runs two (N >= 1024) or three blocks per SM: more warps hide its
// latency better than the second buffer's prefetch (c3: binary64 7.37 -> 6.31
// ms, FP32 3.32 -> 3.11 ms; 512^3: 0.82 -> 0.75 and 0.378 -> 0.364 ms), while
// the y passes keep two buffers and one block, which measured faster for them.
// HYOWON_FFT_X64_NBUF / HYOWON_FFT_X32_NBUF = 2 give the x pass the y passes'
// configuration.
#ifndef HYOWON_FFT_X64_NBUF
#define HYOWON_FFT_X64_NBUF 1
#endif
#ifndef HYOWON_FFT_X32_NBUF
#define HYOWON_FFT_X32_NBUF 1
#endif
template <typename T, int LOG2N, int MODE> struct ColumnCfg {
    using G = Geo<T, LOG2N>;
    static constexpr bool single_buffer =
        MODE == 1 && (sizeof(T) == 8 ? HYOWON_FFT_X64_NBUF == 1 : HYOWON_FFT_X32_NBUF == 1);
    static constexpr int nbuf = single_buffer ? 1 : G::nbuf_b;
    static constexpr size_t smem = static_cast<size_t>(nbuf) * G::tile_bytes_b;
    static constexpr int smem_blocks = static_cast<int>((227u * 1024u) / smem);
    static constexpr int want = LOG2N >= 10 ? 2 : 3;
    static constexpr int minb =
        single_buffer ? G::SP * (want < smem_blocks ? want : smem_blocks) : G::minb_c;
};

template <typename S> struct Raw;   // raw row pair of the z forward input
template <> struct Raw<double> { using type = double2; };
template <> struct Raw<float> { using type = float2; };

__device__ __forceinline__ double2 to_complex(double2 v, unsigned long long&) { return v; }
__device__ __forceinline__ float2 to_complex(float2 v, unsigned long long&) { return v; }

// r2c of CZ rows per block: pack the N reals of a row as N/2 complex values,
// transform, and unpack X[k] = E[k] + W_N^k O[k] with E/O the transforms of
// the even/odd samples, for k = 0..N/2. Each thread issues all its row loads
// before the first shared-memory store.
template <typename T, typename SRC, int LOG2N>
__global__ void __launch_bounds__(Geo<T, LOG2N>::TZ, HYOWON_FFT_MINB_Z)
k_z_forward(const SRC* __restrict__ in, cx_t<T>* __restrict__ H, const cx_t<T>* __restrict__ tw,
            unsigned long long* qsum) {
    using G = Geo<T, LOG2N>;
    using C = cx_t<T>;
    using RawT = typename Raw<SRC>::type;
    constexpr int S = G::SZ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sm = reinterpret_cast<C*>(smem_raw);
    const int tid = threadIdx.x;
    const size_t row0 = static_cast<size_t>(blockIdx.x) * G::CZ;
    const RawT* src = reinterpret_cast<const RawT*>(in + row0 * G::N);
    RawT raw[G::PZ];
#pragma unroll
    for (int i = 0; i < G::PZ; ++i) raw[i] = __ldcs(&src[tid + i * G::TZ]);
    unsigned long long sum = 0;
#pragma unroll
    for (int i = 0; i < G::PZ; ++i) {
        const int e = tid + i * G::TZ;
        sm[(e % G::M) * S + e / G::M] = to_complex(raw[i], sum);
    }
    if (qsum) {
        if constexpr (G::TZ >= 32 && G::TZ % 32 == 0) {
            block_sum_to(sum, qsum);
        } else {
            if (sum) atomicAdd(qsum, sum);
        }
    }
    __syncthreads();
    chunked::rows_r2c<T, LOG2N, G::CZ, S>(sm, tw, H, static_cast<int>(row0 / G::N),
                                         static_cast<int>(row0 % G::N), tid, G::TZ);
}

// c2r of CZ rows per block: Z[k] = (X[k] + conj X[M-k]) + i W_N^-k (X[k] - conj X[M-k]),
// inverse length-M transform, real output pairs (Re, Im).
// Stores the two reals (row element 2jj, 2jj+1) of a z-inverse output pair.
struct StorePair {
    template <typename T, typename C>
    __device__ __forceinline__ void operator()(T* out, size_t idx, C v) const {
        __stcs(reinterpret_cast<C*>(out + idx), v);
    }
};

// The rows (x, y0 .. y0+CZ-1) of the c2r: loads their half-complex values from
// H (LOAD(p) reads one element), transforms in sm, hands each output pair to
// epi. Every thread of the TZ-thread block calls it; it ends with sm in use
// (the caller synchronises before refilling it).
template <typename T, int LOG2N, typename EPI, typename LOAD>
__device__ __forceinline__ void z_inverse_rows(const cx_t<T>* __restrict__ H, T* __restrict__ out,
                                               const cx_t<T>* __restrict__ tw, EPI epi, LOAD load,
                                               cx_t<T>* sm, int x, int y0, int tid) {
    using G = Geo<T, LOG2N>;
    using C = cx_t<T>;
    constexpr int S = G::SZ;
    const size_t row0 = static_cast<size_t>(x) * G::N + y0;
    C v[G::QZ];
#pragma unroll
    for (int i = 0; i < G::QZ; ++i) {
        const int e = tid + i * G::TZ;
        const int k = (e / (G::CC * G::CZ)) * G::CC + e % G::CC;
        if (e < G::KC * G::CZ * G::CC && k < G::Hz)
            v[i] = load(&H[G::at(x, y0 + (e / G::CC) % G::CZ, k)]);
    }
#pragma unroll
    for (int i = 0; i < G::QZ; ++i) {
        const int e = tid + i * G::TZ;
        const int k = (e / (G::CC * G::CZ)) * G::CC + e % G::CC;
        if (e < G::KC * G::CZ * G::CC && k < G::Hz) sm[k * S + (e / G::CC) % G::CZ] = v[i];
    }
    __syncthreads();
    for (int e = tid; e < G::CZ * G::K; e += G::TZ) {
        const int r = e / G::K;
        const int k = e % G::K;
        const C xk = sm[k * S + r];
        const C xm = sm[(G::M - k) * S + r];
        const C w = __ldg(&tw[k]);
        const C Ep = mk(xk.x + xm.x, xk.y - xm.y);
        const C Dp = mk(xk.x - xm.x, xk.y + xm.y);
        const C Op = fft::cmul(Dp, fft::conj(w));
        sm[k * S + r] = mk(Ep.x - Op.y, Ep.y + Op.x);
        if (k != 0 && G::M - k != k) {
            const C Op2 = fft::cmul(mk(-Dp.x, Dp.y), mk(-w.x, -w.y));
            sm[(G::M - k) * S + r] = mk(Ep.x - Op2.y, -Ep.y + Op2.x);
        }
    }
    __syncthreads();
    fft::smem_fft<LOG2N - 1, +1, G::CZ, G::SZ>(sm, tw, G::N, tid % G::CZ, tid / G::CZ);
    for (int e = tid; e < G::CZ * G::M; e += G::TZ) {
        const int r = e / G::M;
        const int jj = e % G::M;
        epi(out, (row0 + r) * G::N + 2 * jj, sm[jj * S + r]);
    }
}

struct LoadStreaming {
    template <typename C>
    __device__ __forceinline__ C operator()(const C* p) const { return __ldcs(p); }
};

template <typename T, int LOG2N, typename EPI>
__global__ void __launch_bounds__(Geo<T, LOG2N>::TZ, HYOWON_FFT_MINB_Z)
k_z_inverse(const cx_t<T>* __restrict__ H, T* __restrict__ out, const cx_t<T>* __restrict__ tw,
            EPI epi) {
    using G = Geo<T, LOG2N>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const size_t row0 = static_cast<size_t>(blockIdx.x) * G::CZ;
    z_inverse_rows<T, LOG2N>(H, out, tw, epi, LoadStreaming{}, reinterpret_cast<cx_t<T>*>(smem_raw),
                             static_cast<int>(row0 / G::N), static_cast<int>(row0 % G::N),
                             static_cast<int>(threadIdx.x));
}

struct NoGreen {
    template <typename C>
    __device__ __forceinline__ C operator()(int, int, int, C v) const { return v; }
};

// Green's multiply of the binary64 form, operation for operation as k_green.
struct DevGreenF64 {
    GreenF64 g;
    __device__ __forceinline__ double2 operator()(int ix, int iy, int iz, double2 v) const {
        if ((ix | iy | iz) == 0) {
            if (!(fabs(v.x - g.input_mass) <= g.mass_tol)) raise_status(g.status, ST_MASS);
            return make_double2(0.0, 0.0);
        }
        const double Dk = g.lap[ix] + g.lap[iy] + g.lap[iz];
        double f = g.four_pi_G / Dk;
        if (g.deconvolve) {
            const double wt = g.win[ix] * g.win[iy] * g.win[iz];
            f /= (wt * wt);
        }
        f *= g.scale;
        v.x *= f;
        v.y *= f;
        return v;
    }
};

struct DevGreenF32 {
    GreenF32 g;
    __device__ __forceinline__ float2 operator()(int ix, int iy, int iz, float2 v) const {
        if ((ix | iy | iz) == 0) return make_float2(0.f, 0.f);
        float f = *g.c_green / (g.lap[ix] + g.lap[iy] + g.lap[iz]);
        if (g.deconvolve) {
            const float wt = g.win[ix] * g.win[iy] * g.win[iz];
            f /= wt * wt;
        }
        v.x *= f;
        v.y *= f;
        return v;
    }
};

// 2LPT Hessian symbol k_a k_b / k^2 (mixed terms 0 on either axis's Nyquist
// plane; k = 0 gives 0), wavenumbers (2 pi m) / L from a table formed with
// the same two roundings: the arithmetic of the IC generator's Hessian
// kernel, rounded operation by operation.
struct DevHessianF64 {
    HessianF64 h;
    int N;
    __device__ __forceinline__ double2 operator()(int ix, int iy, int iz, double2 v) const {
        const double k[3] = {__ldg(&h.k[ix]), __ldg(&h.k[iy]), __ldg(&h.k[iz])};
        const double k2 = __dadd_rn(__dadd_rn(__dmul_rn(k[0], k[0]), __dmul_rn(k[1], k[1])),
                                    __dmul_rn(k[2], k[2]));
        if (k2 == 0.0) return make_double2(0.0, 0.0);
        const bool even = (N & 1) == 0;
        const int ia = h.a == 0 ? ix : (h.a == 1 ? iy : iz);
        const int ib = h.b == 0 ? ix : (h.b == 1 ? iy : iz);
        const double ka = h.a == 0 ? k[0] : (h.a == 1 ? k[1] : k[2]);
        const double kb = h.b == 0 ? k[0] : (h.b == 1 ? k[1] : k[2]);
        const bool mixed_nyquist = h.a != h.b && even && (ia == N / 2 || ib == N / 2);
        const double q = __ddiv_rn(mixed_nyquist ? 0.0 : __dmul_rn(ka, kb), k2);
        return make_double2(__dmul_rn(v.x, q), __dmul_rn(v.y, q));
    }
};

// z-inverse epilogue folding the normalised field h into the 2LPT source,
// the IC generator's source kernel applied to each output pair:
// op 0: acc = h; 1: src = acc h, acc += h; 2: src += acc h; 3: src -= h h.
struct SourceEpiF64 {
    SourceTermF64 t;
    __device__ __forceinline__ void operator()(double*, size_t idx, double2 v) const {
        const double h0 = __dmul_rn(v.x, t.norm), h1 = __dmul_rn(v.y, t.norm);
        if (!isfinite(h0) || !isfinite(h1)) atomicOr(t.status, t.hessian_flag);
        double2* acc = reinterpret_cast<double2*>(t.acc + idx);
        double2* src = reinterpret_cast<double2*>(t.src + idx);
        if (t.op == 0) {
            *acc = make_double2(h0, h1);
            return;
        }
        double2 out;
        if (t.op == 1) {
            const double2 a = *acc;
            out = make_double2(__dmul_rn(a.x, h0), __dmul_rn(a.y, h1));
            *acc = make_double2(__dadd_rn(a.x, h0), __dadd_rn(a.y, h1));
        } else if (t.op == 2) {
            const double2 a = *acc, sv = *src;
            out = make_double2(__dadd_rn(sv.x, __dmul_rn(a.x, h0)), __dadd_rn(sv.y, __dmul_rn(a.y, h1)));
        } else {
            const double2 sv = *src;
            out = make_double2(__dsub_rn(sv.x, __dmul_rn(h0, h0)), __dsub_rn(sv.y, __dmul_rn(h1, h1)));
        }
        if (t.last && (!isfinite(out.x) || !isfinite(out.y))) atomicOr(t.status, t.source_flag);
        *src = out;
    }
};

// Bounded polls of a pipeline barrier before a block gives up (each poll may
// suspend for a hardware-chosen interval; a healthy wait needs a few). The
// first wait of each tile uses the plan's limit (this value unless a test
// lowered it); draining the copies in flight after a failure always uses this.
constexpr unsigned kWaitLimit = 1u << 24;

// Complex transforms of the CC columns of each tile of the chunked half
// spectrum: tile t = (kc, s) with kc = t / N, s = t % N; y pass (AXIS 1):
// s = kx, the tile is the contiguous block H[kc][kx][.][.]; x pass (AXIS 0):
// s = ky, elements H[kc][.][ky][.] (128-byte-or-less runs N*CC apart).
// Persistent blocks; one thread keeps the next nbuf-1 tiles of the block
// streaming into the other shared-memory buffers with TMA loads while the
// block transforms the current one (dense rows, no padding: a half/quarter
// warp reads one 64-byte row). With GREEN (the x pass): forward transform,
// Green's multiply, inverse transform. Results are stored from registers.
// MODE 0: one transform (SIGN); 1: forward transform, Green's multiply,
// inverse transform (the x pass of the potential solve); 2: the symbol
// `green` applied to the untransformed tile, then one transform (SIGN).
template <typename T, int LOG2N, int AXIS, int SIGN, int MODE, typename GF>
__global__ void __launch_bounds__(Geo<T, LOG2N>::TCB, (ColumnCfg<T, LOG2N, MODE>::minb))
k_columns(const __grid_constant__ CUtensorMap map, cx_t<T>* __restrict__ H,
          const cx_t<T>* __restrict__ tw, GF green, unsigned int* status, unsigned wait_limit) {
    using G = Geo<T, LOG2N>;
    using C = cx_t<T>;
    constexpr int EC = G::EC;
    constexpr int P = G::N / EC;
    constexpr int CB = G::CB;     // columns of this block's part of a tile
    constexpr int S = CB;
    constexpr int NB = ColumnCfg<T, LOG2N, MODE>::nbuf;
    constexpr size_t axis_stride = AXIS == 1 ? static_cast<size_t>(G::CC)
                                             : static_cast<size_t>(G::N) * G::CC;
    constexpr size_t seq_stride = AXIS == 1 ? static_cast<size_t>(G::N) * G::CC
                                            : static_cast<size_t>(G::CC);
    extern __shared__ __align__(1024) unsigned char smem_tiles[];
    __shared__ __align__(8) uint64_t full[NB];
    const int tid = threadIdx.x;
    const int c = tid % CB;
    const int j = tid / CB;
    // work items: (tile, part) with tile = kc * N + seq and part the column block
    const unsigned tiles = static_cast<unsigned>(G::KC) * G::N * G::SP;
    auto tile_buf = [&](int b) { return reinterpret_cast<C*>(smem_tiles + b * G::tile_bytes_b); };
    auto issue = [&](unsigned item, int b) {
        const unsigned tile = item / G::SP;
        const int part = static_cast<int>(item % G::SP);
        const int kc = static_cast<int>(tile / G::N);
        const int sq = static_cast<int>(tile % G::N);
        C* dst = tile_buf(b);
        tma::mbar_arrive_expect_tx(&full[b], G::tile_bytes_b);
        const int c0 = part * G::units_b;   // 8-byte units: a multiple of 16 bytes
#pragma unroll
        for (int g = 0; g < G::N / G::box; ++g) {
            if (AXIS == 1)
                tma::load_3d(dst + g * G::box * CB, &map, c0, g * G::box, kc * G::N + sq, &full[b]);
            else
                tma::load_3d(dst + g * G::box * CB, &map, c0, sq, kc * G::N + g * G::box, &full[b]);
        }
    };
    if (tid == 0) {
#pragma unroll
        for (int b = 0; b < NB; ++b) tma::mbar_init(&full[b], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    unsigned t = blockIdx.x;
    if (tid == 0) {
        // prologue: the first nbuf-1 tiles of this block
#pragma unroll
        for (int b = 0; b < NB - 1; ++b) {
            const unsigned tb = t + static_cast<unsigned>(b) * gridDim.x;
            if (tb < tiles) issue(tb, b);
        }
    }
    for (unsigned i = 0; t < tiles; ++i, t += gridDim.x) {
        const int b = static_cast<int>(i % NB);
        const unsigned parity = (i / NB) & 1u;
        // refill the buffer the previous iteration finished with
        const unsigned nt = t + static_cast<unsigned>(NB - 1) * gridDim.x;
        if (tid == 0 && nt < tiles) {
            tma::fence_proxy_async();
            issue(nt, static_cast<int>((i + NB - 1) % NB));
        }
        const bool ok = tma::mbar_wait(&full[b], parity, wait_limit);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicOr(status, ST_PIPELINE);
                // let this block's copies in flight land before it exits
                for (int k = 0; k < NB; ++k) {
                    const unsigned ik = i + static_cast<unsigned>(k);
                    const unsigned tk = t + static_cast<unsigned>(k) * gridDim.x;
                    if (tk < tiles) tma::mbar_wait(&full[ik % NB], (ik / NB) & 1u, kWaitLimit);
                }
            }
            return;
        }
        C* sm = tile_buf(b);
        const unsigned tile = t / G::SP;
        const int col = static_cast<int>(t % G::SP) * CB + c;   // column within the chunk
        const int kc = static_cast<int>(tile / G::N);
        const int seq = static_cast<int>(tile % G::N);
        const int kz = kc * G::CC + col;
        C v[EC];
        if constexpr (MODE == 2) {
            // element j + q P of column c, untransformed
#pragma unroll
            for (int q = 0; q < EC; ++q) v[q] = sm[(j + q * P) * S + c];
            if (kz < G::Hz) {
#pragma unroll
                for (int q = 0; q < EC; ++q)
                    v[q] = AXIS == 0 ? green(j + q * P, seq, kz, v[q]) : green(seq, j + q * P, kz, v[q]);
            }
            __syncthreads();
            fft::first_stage_to_smem<LOG2N, SIGN, CB, S, EC>(v, sm, c, j);
            fft::rest_to_registers<LOG2N, SIGN, CB, S, EC>(sm, tw, G::N, c, j, v);
        } else {
            fft::smem_to_registers<LOG2N, SIGN, CB, S, EC>(sm, tw, G::N, c, j, v);
        }
        if constexpr (MODE == 1) {
            if (kz < G::Hz) {
#pragma unroll
                for (int q = 0; q < EC; ++q)
                    v[q] = AXIS == 0 ? green(j + q * P, seq, kz, v[q]) : green(seq, j + q * P, kz, v[q]);
            }
            __syncthreads();
            fft::first_stage_to_smem<LOG2N, -SIGN, CB, S, EC>(v, sm, c, j);
            fft::rest_to_registers<LOG2N, -SIGN, CB, S, EC>(sm, tw, G::N, c, j, v);
        }
        if (kz < G::Hz) {
            C* dst = H + static_cast<size_t>(kc) * G::chunk + static_cast<size_t>(seq) * seq_stride + col;
#pragma unroll
            for (int q = 0; q < EC; ++q) __stcs(&dst[static_cast<size_t>(j + q * P) * axis_stride], v[q]);
        }
        __syncthreads();
    }
}

template <typename K>
bool prepare(K kernel, size_t smem) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)) == cudaSuccess;
}

template <typename T, typename SRC, int LOG2N>
int z_forward(const SRC* in, cx_t<T>* H, const cx_t<T>* tw, unsigned long long* qsum,
              cudaStream_t s) {
    using G = Geo<T, LOG2N>;
    if (!prepare(k_z_forward<T, SRC, LOG2N>, G::smem_zf)) return -1;
    const unsigned blocks = static_cast<unsigned>(static_cast<size_t>(G::N) * G::N / G::CZ);
    k_z_forward<T, SRC, LOG2N><<<blocks, G::TZ, G::smem_zf, s>>>(in, H, tw, qsum);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

template <typename T, int LOG2N, typename EPI = StorePair>
int z_inverse(const cx_t<T>* H, T* out, const cx_t<T>* tw, cudaStream_t s, EPI epi = EPI{}) {
    using G = Geo<T, LOG2N>;
    if (!prepare(k_z_inverse<T, LOG2N, EPI>, G::smem_zi)) return -1;
    const unsigned blocks = static_cast<unsigned>(static_cast<size_t>(G::N) * G::N / G::CZ);
    k_z_inverse<T, LOG2N, EPI><<<blocks, G::TZ, G::smem_zi, s>>>(H, out, tw, epi);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

// AXIS 1: y transforms of every (kc, kx) block; AXIS 0: x transforms of
// every (kc, ky) column set.
template <typename T, int LOG2N, int AXIS, int SIGN, int MODE, typename GF>
int columns(const Plan* p, cx_t<T>* H, const cx_t<T>* tw, GF green, unsigned int* status,
            cudaStream_t s);

// The complex pass that also applies the Green's function (0: x, 1: y); the
// other axis is transformed forward after the z pass and inverse before it.
#ifndef HYOWON_FFT_GREEN_AXIS
#define HYOWON_FFT_GREEN_AXIS 0
#endif
constexpr int kGreenAxis = HYOWON_FFT_GREEN_AXIS;
constexpr int kPlainAxis = 1 - kGreenAxis;

template <typename T, typename SRC, int LOG2N>
int forward_t(const Plan* p, const SRC* in, cx_t<T>* H, const cx_t<T>* tw, unsigned long long* qsum,
              unsigned int* status, cudaStream_t s) {
    if (z_forward<T, SRC, LOG2N>(in, H, tw, qsum, s) < 0) return -1;
    if (columns<T, LOG2N, kPlainAxis, -1, 0>(p, H, tw, NoGreen{}, status, s) < 0) return -1;
    return 2;
}

template <typename T, int LOG2N>
int forward_columns_t(const Plan* p, cx_t<T>* H, const cx_t<T>* tw, unsigned int* status,
                      cudaStream_t s) {
    return columns<T, LOG2N, kPlainAxis, -1, 0>(p, H, tw, NoGreen{}, status, s);
}

template <typename T, int LOG2N, typename GF>
int green_t(const Plan* p, cx_t<T>* H, const cx_t<T>* tw, GF g, unsigned int* status,
            cudaStream_t s) {
    return columns<T, LOG2N, kGreenAxis, -1, 1>(p, H, tw, g, status, s);
}

template <typename T, int LOG2N>
int inverse_t(const Plan* p, cx_t<T>* H, T* out, const cx_t<T>* tw, unsigned int* status,
              cudaStream_t s) {
    if (columns<T, LOG2N, kPlainAxis, +1, 0>(p, H, tw, NoGreen{}, status, s) < 0) return -1;
    if (z_inverse<T, LOG2N>(H, out, tw, s) < 0) return -1;
    return 2;
}

template <typename T, int LOG2N, int AXIS, int SIGN, int MODE, typename GF>
int columns(const Plan* p, cx_t<T>* H, const cx_t<T>* tw, GF green, unsigned int* status,
            cudaStream_t s) {
    using G = Geo<T, LOG2N>;
    if (!p || p->N != G::N) return -1;
    auto kernel = k_columns<T, LOG2N, AXIS, SIGN, MODE, GF>;
    constexpr size_t smem = ColumnCfg<T, LOG2N, MODE>::smem;
    if (!prepare(kernel, smem)) return -1;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess
        || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess
        || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, G::TCB, smem) != cudaSuccess
        || per_sm < 1)
        return -1;
    const unsigned tiles = static_cast<unsigned>(G::KC) * G::N * G::SP;
    const unsigned full = static_cast<unsigned>(sms) * static_cast<unsigned>(per_sm);
    const unsigned grid = tiles < full ? tiles : full;
    kernel<<<grid, G::TCB, smem, s>>>(AXIS == 1 ? p->y : p->x, H, tw, green, status,
                                          p->wait_limit);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
    static EncodeTiled fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess
            || q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return static_cast<EncodeTiled>(nullptr);
        }
        return reinterpret_cast<EncodeTiled>(f);
    }();
    return fn;
}

template <typename T, int LOG2N>
bool encode_maps(Plan* p, void* modes) {
    using G = Geo<T, LOG2N>;
    EncodeTiled enc = encode_fn();
    if (!enc) return false;
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(G::units), static_cast<cuuint64_t>(G::N),
                                static_cast<cuuint64_t>(G::KC) * G::N};
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(G::units) * 8,
                                   static_cast<cuuint64_t>(G::units) * 8 * G::N};
    const cuuint32_t estr[3] = {1, 1, 1};
    const cuuint32_t box_y[3] = {static_cast<cuuint32_t>(G::units_b), static_cast<cuuint32_t>(G::box), 1};
    const cuuint32_t box_x[3] = {static_cast<cuuint32_t>(G::units_b), 1, static_cast<cuuint32_t>(G::box)};
    return enc(&p->y, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, modes, dims, strides, box_y, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS
        && enc(&p->x, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, modes, dims, strides, box_x, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int log2_of(int N) {
    int l = 0;
    while ((1 << l) < N) ++l;
    return l;
}

#define HYOWON_DISPATCH(N, CALL)              \
    switch (log2_of(N)) {                     \
    case 5: { constexpr int LG = 5; return CALL; }   \
    case 6: { constexpr int LG = 6; return CALL; }   \
    case 7: { constexpr int LG = 7; return CALL; }   \
    case 8: { constexpr int LG = 8; return CALL; }   \
    case 9: { constexpr int LG = 9; return CALL; }   \
    case 10: { constexpr int LG = 10; return CALL; } \
    case 11: { constexpr int LG = 11; return CALL; } \
    default: return -1;                       \
    }

}  // namespace

bool supported(int N) { return N >= 32 && N <= 2048 && (N & (N - 1)) == 0; }

namespace {
template <typename T, int LG> constexpr size_t chunked_elements() {
    return Geo<T, LG>::chunk * Geo<T, LG>::KC;
}
template <typename T> size_t chunked_elements(int N) {
    switch (log2_of(N)) {
    case 5: return chunked_elements<T, 5>();
    case 6: return chunked_elements<T, 6>();
    case 7: return chunked_elements<T, 7>();
    case 8: return chunked_elements<T, 8>();
    case 9: return chunked_elements<T, 9>();
    case 10: return chunked_elements<T, 10>();
    case 11: return chunked_elements<T, 11>();
    default: return 0;
    }
}
}  // namespace

size_t modes_elements_f64(int N) { return supported(N) ? chunked_elements<double>(N) : 0; }
size_t modes_elements_f32(int N) { return supported(N) ? chunked_elements<float>(N) : 0; }

void twiddles(int N, double* re_im) {
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < N; ++m) {
        const long double a = two_pi * static_cast<long double>(m) / static_cast<long double>(N);
        re_im[2 * m] = static_cast<double>(cosl(a));
        re_im[2 * m + 1] = static_cast<double>(-sinl(a));
    }
}

Plan* create_plan(int N, bool fp32, void* modes, const char** err) {
    if (!supported(N)) {
        *err = "mesh size not supported by the five-pass solve";
        return nullptr;
    }
    Plan* p = new (std::nothrow) Plan();
    if (!p) {
        *err = "out of host memory";
        return nullptr;
    }
    p->N = N;
    p->fp32 = fp32;
    bool ok = false;
    switch (log2_of(N)) {
    case 5: ok = fp32 ? encode_maps<float, 5>(p, modes) : encode_maps<double, 5>(p, modes); break;
    case 6: ok = fp32 ? encode_maps<float, 6>(p, modes) : encode_maps<double, 6>(p, modes); break;
    case 7: ok = fp32 ? encode_maps<float, 7>(p, modes) : encode_maps<double, 7>(p, modes); break;
    case 8: ok = fp32 ? encode_maps<float, 8>(p, modes) : encode_maps<double, 8>(p, modes); break;
    case 9: ok = fp32 ? encode_maps<float, 9>(p, modes) : encode_maps<double, 9>(p, modes); break;
    case 10: ok = fp32 ? encode_maps<float, 10>(p, modes) : encode_maps<double, 10>(p, modes); break;
    case 11: ok = fp32 ? encode_maps<float, 11>(p, modes) : encode_maps<double, 11>(p, modes); break;
    default: break;
    }
    if (!ok) {
        delete p;
        *err = "cuTensorMapEncodeTiled failed for the half-spectrum buffer";
        return nullptr;
    }
    return p;
}

void destroy_plan(Plan* p) { delete p; }

void set_wait_limit(Plan* p, unsigned polls) {
    if (p) p->wait_limit = polls;
}

int forward_f64(const Plan* p, int N, const double* mass, double2* modes, const double2* tw,
                unsigned int* status, cudaStream_t s) {
    if (!supported(N) || !p || p->fp32) return -1;
    HYOWON_DISPATCH(N, (forward_t<double, double, LG>(p, mass, modes, tw, nullptr, status, s)))
}

int forward_columns_f64(const Plan* p, int N, double2* modes, const double2* tw,
                        unsigned int* status, cudaStream_t s) {
    if (!supported(N) || !p || p->fp32) return -1;
    HYOWON_DISPATCH(N, (forward_columns_t<double, LG>(p, modes, tw, status, s)))
}

int green_f64(const Plan* p, int N, double2* modes, const double2* tw, const GreenF64& g,
              cudaStream_t s) {
    if (!supported(N) || !p || p->fp32) return -1;
    HYOWON_DISPATCH(N, (green_t<double, LG>(p, modes, tw, DevGreenF64{g}, g.status, s)))
}

int inverse_f64(const Plan* p, int N, double2* modes, double* phi, const double2* tw,
                unsigned int* status, cudaStream_t s) {
    if (!supported(N) || !p || p->fp32) return -1;
    HYOWON_DISPATCH(N, (inverse_t<double, LG>(p, modes, phi, tw, status, s)))
}

namespace {
template <int LOG2N>
int hessian_source_t(const Plan* pd, const Plan* pw, int N, double2* work, const double2* tw,
                     const HessianF64& h, const SourceTermF64& t, unsigned int* status,
                     cudaStream_t s) {
    // symbol then inverse x: tiles read from the spectrum of pd, stored to work
    if (columns<double, LOG2N, 0, +1, 2>(pd, work, tw, DevHessianF64{h, N}, status, s) < 0)
        return -1;
    if (columns<double, LOG2N, 1, +1, 0>(pw, work, tw, NoGreen{}, status, s) < 0) return -1;
    if (z_inverse<double, LOG2N, SourceEpiF64>(work, nullptr, tw, s, SourceEpiF64{t}) < 0)
        return -1;
    return 3;
}
}  // namespace

int hessian_source_f64(const Plan* pd, const Plan* pw, int N, double2* work, const double2* tw,
                       const HessianF64& h, const SourceTermF64& t, unsigned int* status,
                       cudaStream_t s) {
    if (!supported(N) || !pd || !pw || pd->fp32 || pw->fp32) return -1;
    HYOWON_DISPATCH(N, (hessian_source_t<LG>(pd, pw, N, work, tw, h, t, status, s)))
}

int chunk_columns_f64(int N) {
    switch (log2_of(N)) {
    case 5: return Geo<double, 5>::CC;
    case 6: return Geo<double, 6>::CC;
    case 7: return Geo<double, 7>::CC;
    case 8: return Geo<double, 8>::CC;
    case 9: return Geo<double, 9>::CC;
    case 10: return Geo<double, 10>::CC;
    case 11: return Geo<double, 11>::CC;
    default: return 0;
    }
}

int forward_f32(const Plan* p, int N, const float* mesh, float2* modes, const float2* tw,
                unsigned int* status, cudaStream_t s) {
    if (!supported(N) || !p || !p->fp32) return -1;
    HYOWON_DISPATCH(N, (forward_t<float, float, LG>(p, mesh, modes, tw, nullptr, status, s)))
}

int forward_columns_f32(const Plan* p, int N, float2* modes, const float2* tw,
                        unsigned int* status, cudaStream_t s) {
    if (!supported(N) || !p || !p->fp32) return -1;
    HYOWON_DISPATCH(N, (forward_columns_t<float, LG>(p, modes, tw, status, s)))
}

int green_f32(const Plan* p, int N, float2* modes, const float2* tw, const GreenF32& g,
              unsigned int* status, cudaStream_t s) {
    if (!supported(N) || !p || !p->fp32) return -1;
    HYOWON_DISPATCH(N, (green_t<float, LG>(p, modes, tw, DevGreenF32{g}, status, s)))
}

int inverse_f32(const Plan* p, int N, float2* modes, float* phi, const float2* tw,
                unsigned int* status, cudaStream_t s) {
    if (!supported(N) || !p || !p->fp32) return -1;
    HYOWON_DISPATCH(N, (inverse_t<float, LG>(p, modes, phi, tw, status, s)))
}

}  // namespace poisson
}  // namespace hyowon
