// pm_fft.cuh -- register/shared-memory FFT building blocks for the mesh
// transforms of the PM step.
//
// Transforms are unnormalised, forward exp(-2 pi i jk/L), inverse exp(+...),
// the conventions of the r2c / c2r pair the reference's FFT backend uses
// (src/mesh/fft_backend.cpp:1088-1145). Lengths are powers of two.
//
// A length-L transform runs as a Stockham autosort sequence of radix-R stages
// (radix 16, then one radix 2/4/8 stage for the remaining bits): stage s, with
// Ns = product of the earlier radices, takes for butterfly j the R inputs
// j + r L/R, multiplies input r by W_{Ns R}^{(j mod Ns) r}, does an R-point DFT
// in registers and writes output r to ((j div Ns) Ns R + j mod Ns) + r Ns.
// The first stage reads natural order, the last writes natural order. Several
// independent sequences share a thread block; shared memory holds them
// interleaved, element i of sequence c at [i * S + c] with S = C + 1 (the odd
// stride keeps both the strided and the sequence-fastest accesses free of
// bank conflicts) or S = C for tiles written densely by TMA. Thread t works
// on sequence t % C, butterfly group t / C.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hyowon {
namespace fft {

template <typename T> struct Cx;
template <> struct Cx<float> { using type = float2; };
template <> struct Cx<double> { using type = double2; };
template <typename T> using cx_t = typename Cx<T>::type;

__device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C conj(C a) { return mk(a.x, -a.y); }
template <typename C> __device__ __forceinline__ C scale(C a, decltype(a.x) s) { return mk(a.x * s, a.y * s); }

// cos and sin of 2 pi q / 32 for q in [0, 8], correctly rounded binary64.
__host__ __device__ constexpr double cos32_oct(int q) {
    return q == 0 ? 1.0
         : q == 1 ? 0x1.f6297cff75cb0p-1
         : q == 2 ? 0x1.d906bcf328d46p-1
         : q == 3 ? 0x1.a9b66290ea1a3p-1
         : q == 4 ? 0x1.6a09e667f3bcdp-1
         : q == 5 ? 0x1.1c73b39ae68c8p-1
         : q == 6 ? 0x1.87de2a6aea963p-2
         : q == 7 ? 0x1.8f8b83c69a60bp-3
         : 0.0;
}
__host__ __device__ constexpr double sin32_oct(int q) { return cos32_oct(8 - q); }

// v * exp(SIGN 2 pi i Q / 32), Q in [0, 16). Q is a constant wherever this is
// called from the unrolled butterflies, so the branches and the table fold.
template <int SIGN, typename C>
__device__ __forceinline__ C rot32(C v, int Q) {
    using T = decltype(v.x);
    if (Q == 0) return v;
    if (Q == 8) return SIGN > 0 ? mk(-v.y, v.x) : mk(v.y, -v.x);  // * (+-i)
    // for Q > 8: exp(i(pi/2 + a)) = i exp(i a)
    const int q = Q > 8 ? Q - 8 : Q;
    const T c = static_cast<T>(cos32_oct(q));
    const T s = static_cast<T>(SIGN) * static_cast<T>(sin32_oct(q));
    C r;
    if (q == 4) {
        r = mk((v.x - v.y * static_cast<T>(SIGN)) * c, (v.y + v.x * static_cast<T>(SIGN)) * c);
    } else {
        r = mk(v.x * c - v.y * s, v.x * s + v.y * c);
    }
    if (Q > 8) r = SIGN > 0 ? mk(-r.y, r.x) : mk(r.y, -r.x);
    return r;
}

template <int R> __host__ __device__ constexpr int ilog2() { return R <= 1 ? 0 : 1 + ilog2<R / 2>(); }

__host__ __device__ constexpr int bitrev(int k, int bits) {
    int r = 0;
    for (int i = 0; i < bits; ++i) r |= ((k >> i) & 1) << (bits - 1 - i);
    return r;
}

// Radix-2 decimation-in-frequency butterflies of span S over v[R].
template <int R, int S, int SIGN, typename C>
__device__ __forceinline__ void dif_pass(C (&v)[R]) {
#pragma unroll
    for (int b = 0; b < R; b += 2 * S) {
#pragma unroll
        for (int i = 0; i < S; ++i) {
            const C a = v[b + i];
            const C c = v[b + i + S];
            v[b + i] = cadd(a, c);
            // W_{2S}^i = exp(SIGN 2 pi i * (i * 16 / S) / 32)
            v[b + i + S] = rot32<SIGN>(csub(a, c), (i * 16) / S);
        }
    }
    if constexpr (S > 1) dif_pass<R, S / 2, SIGN>(v);
}

// In-register R-point DFT (R <= 32), natural order in and out.
template <int R, int SIGN, typename C>
__device__ __forceinline__ void dft(C (&v)[R]) {
    if constexpr (R > 1) {
        dif_pass<R, R / 2, SIGN>(v);
        C t[R];
#pragma unroll
        for (int k = 0; k < R; ++k) t[k] = v[bitrev(k, ilog2<R>())];
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = t[k];
    }
}

// Multiplies v[r] by W^{k r}, W = exp(SIGN 2 pi i / (Ns R)), from the table
// tw[m] = exp(-2 pi i m / NT) (NT a multiple of Ns R).
template <int R, int SIGN, typename C>
__device__ __forceinline__ void twiddle(C (&v)[R], int k, int Ns, const C* __restrict__ tw, int NT) {
    if (Ns == 1 || k == 0) return;
    const int step = k * (NT / (Ns * R));
#pragma unroll
    for (int r = 1; r < R; ++r) {
        C w = __ldg(&tw[(step * r) & (NT - 1)]);
        if (SIGN > 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
    }
}

// Stage geometry for a length L = 2^LOG2L transform with E (8 or 16)
// elements per thread: radix-E stages, then one stage of radix 2^(LOG2L mod
// log2 E) if that is not zero.
template <int LOG2L, int E = 16> struct Plan {
    static constexpr int L = 1 << LOG2L;
    static constexpr int LE = ilog2<E>();
    static constexpr int nE = LOG2L / LE;
    static constexpr int rem = LOG2L % LE;
    static constexpr int RF = rem ? (1 << rem) : E;    // radix of the last stage
    static constexpr int P = L / E;                     // butterfly groups per sequence
    static_assert(LOG2L >= LE, "transform shorter than the elements per thread");
};

// Row order of the first stage's output in the dense column tiles: row rho is
// kept at rho ^ ((rho >> LE) & 1) for a radix-2^LE first stage. That stage
// writes rows 2^LE j + r for the lanes' consecutive j, which all fall in the
// same half of a 128-byte bank row when a row is 64 bytes (CC columns);
// swapping row pairs in every other group of 2^LE rows spreads them over both
// halves (4- and 8-way bank conflicts become none), while the next stage's
// reads of consecutive rows stay consecutive. Every access to that stage's
// output applies it (PIN / POUT below); other layouts are untouched.
#ifndef HYOWON_FFT_ROWPERM
#define HYOWON_FFT_ROWPERM 1
#endif
// MASK widens the swap to the low log2(MASK + 1) bits (rows narrower than 64
// bytes need more row groups spread over a 128-byte bank row).
template <bool PERMUTED, int LE = 4, int MASK = 1>
__device__ __forceinline__ int row_at(int row) {
    return (PERMUTED && HYOWON_FFT_ROWPERM) ? (row ^ ((row >> LE) & MASK)) : row;
}

// One shared-memory stage of radix R (R <= E) on C interleaved sequences of
// length L, E elements per thread: each thread does E/R butterflies (groups
// j + P b, P = L/E). The caller has synchronised since the last writes to sm;
// the stage ends synchronised. Threads with `active` false only take part in
// the barriers.
template <int LOG2L, int R, int SIGN, int C, int S, int E = 16, bool PIN = false, bool POUT = false,
          int PMASK = 1, typename Cplx>
__device__ __forceinline__ void smem_stage(Cplx* sm, int Ns, const Cplx* __restrict__ tw, int NT,
                                           int c, int j, bool active = true) {
    constexpr int L = 1 << LOG2L;
    constexpr int P = L / E;
    constexpr int NB = E / R;
    Cplx v[NB][R];
    if (active) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int jb = j + P * b;
#pragma unroll
            for (int r = 0; r < R; ++r)
                v[b][r] = sm[row_at<PIN, ilog2<E>(), PMASK>(jb + r * (L / R)) * S + c];
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int jb = j + P * b;
            const int k = jb & (Ns - 1);
            twiddle<R, SIGN>(v[b], k, Ns, tw, NT);
            dft<R, SIGN>(v[b]);
            const int base = (jb - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) sm[row_at<POUT, ilog2<E>(), PMASK>(base + r * Ns) * S + c] = v[b][r];
        }
    }
    __syncthreads();
}

// Whole transform in shared memory (natural order in and out): radix-E
// stages, then one stage of the remaining radix, E (8 or 16) elements per
// thread, thread (c, j) for j < L/E.
template <int LOG2L, int SIGN, int C, int S, int E = 16, typename Cplx>
__device__ __forceinline__ void smem_fft(Cplx* sm, const Cplx* __restrict__ tw, int NT, int c, int j,
                                         bool active = true) {
    constexpr int LE = ilog2<E>();
    constexpr int nE = LOG2L / LE;
    constexpr int rem = LOG2L % LE;
    static_assert(LOG2L >= LE, "transform shorter than the elements per thread");
    int Ns = 1;
#pragma unroll 1
    for (int s = 0; s < nE; ++s) {
        smem_stage<LOG2L, E, SIGN, C, S, E>(sm, Ns, tw, NT, c, j, active);
        Ns *= E;
    }
    if constexpr (rem != 0) smem_stage<LOG2L, (1 << rem), SIGN, C, S, E>(sm, Ns, tw, NT, c, j, active);
}

// First stage (radix E, no twiddles) from E values already in registers,
// v[r] = element j + r P, written to shared memory in the permuted row order
// (row_at) that rest_to_registers reads.
template <int LOG2L, int SIGN, int C, int S, int E = 16, typename Cplx>
__device__ __forceinline__ void first_stage_to_smem(Cplx (&v)[E], Cplx* sm, int c, int j) {
    dft<E, SIGN>(v);
#pragma unroll
    for (int r = 0; r < E; ++r) sm[row_at<true, ilog2<E>()>(j * E + r) * S + c] = v[r];
}

// The last stage (stride Ns = L / RF), read from shared memory and returned in
// registers: out[q] = element j + q P of the transform (q < E).
template <int LOG2L, int SIGN, int C, int S, int E = 16, bool PIN = false, typename Cplx>
__device__ __forceinline__ void final_to_registers(const Cplx* sm, int Ns, const Cplx* __restrict__ tw,
                                                   int NT, int c, int j, Cplx (&out)[E]) {
    using PL = Plan<LOG2L, E>;
    constexpr int L = PL::L;
    constexpr int P = PL::P;
    constexpr int R = PL::RF;
    constexpr int NB = E / R;
    Cplx v[NB][R];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int jb = j + P * b;
#pragma unroll
        for (int r = 0; r < R; ++r) v[b][r] = sm[row_at<PIN, PL::LE>(jb + r * (L / R)) * S + c];
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int jb = j + P * b;
        twiddle<R, SIGN>(v[b], jb & (Ns - 1), Ns, tw, NT);
        dft<R, SIGN>(v[b]);
        // Ns = L / R here, so output r of butterfly jb is element jb + r L/R
        // = j + P (b + NB r).
#pragma unroll
        for (int r = 0; r < R; ++r) out[b + NB * r] = v[b][r];
    }
}

// Middle stages plus the last stage, after first_stage_to_smem.
template <int LOG2L, int SIGN, int C, int S, int E = 16, typename Cplx>
__device__ __forceinline__ void rest_to_registers(Cplx* sm, const Cplx* __restrict__ tw, int NT, int c,
                                                  int j, Cplx (&out)[E]) {
    using PL = Plan<LOG2L, E>;
    int Ns = E;
    // the first stage's shared-memory writes must land before anyone reads
    __syncthreads();
    // radix-E stages after the first, except a final radix-E one; the first
    // of them reads the first stage's permuted rows
    constexpr int mid = PL::rem ? PL::nE - 1 : PL::nE - 2;
    if constexpr (mid >= 1) {
        smem_stage<LOG2L, E, SIGN, C, S, E, true, false>(sm, Ns, tw, NT, c, j);
        Ns *= E;
#pragma unroll 1
        for (int s = 1; s < mid; ++s) {
            smem_stage<LOG2L, E, SIGN, C, S, E>(sm, Ns, tw, NT, c, j);
            Ns *= E;
        }
        final_to_registers<LOG2L, SIGN, C, S, E>(sm, Ns, tw, NT, c, j, out);
    } else {
        final_to_registers<LOG2L, SIGN, C, S, E, true>(sm, Ns, tw, NT, c, j, out);
    }
}

// Whole transform from natural order in shared memory (the caller has
// synchronised after filling it) to registers, out[q] = element j + q P.
template <int LOG2L, int SIGN, int C, int S, int E = 16, typename Cplx>
__device__ __forceinline__ void smem_to_registers(Cplx* sm, const Cplx* __restrict__ tw, int NT, int c,
                                                  int j, Cplx (&out)[E]) {
    using PL = Plan<LOG2L, E>;
    int Ns = 1;
    // every radix-E stage but a final radix-E one; the first writes its rows
    // permuted (row_at) and the stage after it reads them so
    constexpr int n = PL::rem ? PL::nE : PL::nE - 1;
    if constexpr (n == 0) {
        final_to_registers<LOG2L, SIGN, C, S, E>(sm, Ns, tw, NT, c, j, out);
    } else {
        smem_stage<LOG2L, E, SIGN, C, S, E, false, true>(sm, Ns, tw, NT, c, j);
        Ns = E;
        if constexpr (n >= 2) {
            smem_stage<LOG2L, E, SIGN, C, S, E, true, false>(sm, Ns, tw, NT, c, j);
            Ns = E * E;
#pragma unroll 1
            for (int s = 2; s < n; ++s) {
                smem_stage<LOG2L, E, SIGN, C, S, E>(sm, Ns, tw, NT, c, j);
                Ns *= E;
            }
            final_to_registers<LOG2L, SIGN, C, S, E>(sm, Ns, tw, NT, c, j, out);
        } else {
            final_to_registers<LOG2L, SIGN, C, S, E, true>(sm, Ns, tw, NT, c, j, out);
        }
    }
}

// Asynchronous global -> shared copies (cp.async) of BYTES = 8 or 16 bytes;
// when `valid` is false nothing is read and the destination is zero-filled.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, bool valid) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    const int src = valid ? BYTES : 0;
    if constexpr (BYTES == 16) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src)
                     : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sa), "l"(gmem),
                     "n"(BYTES), "r"(src)
                     : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

}  // namespace fft
}  // namespace hyowon
