// pm_ic.cu -- HYOWON's generated initial conditions on the device.
//
// Field (RandomField::generate, src/ic/random_field.cpp:70-330): one thread
// per half-spectrum mode. The mode's integer numbers (mx, my, mz) outside the
// Cartesian support |m_i| <= K (or m = 0) give 0. On the kz = 0 and Nyquist
// planes the half spectrum stores each conjugate pair once: the member whose
// conjugate index (M-i, M-j) is smaller (i first, then j) is drawn with the
// conjugate's counter and its imaginary part negated; self-conjugate modes are
// real. The draw is Philox4x32-10 (src/ic/philox_rng.cpp:43-62) on the
// counter (mx, my, mz, stream) and key (seed low, seed high), mapped to two
// 53-bit open uniforms and a Box-Muller pair (:27-36,85-96). The amplitudes
// sqrt(var_s), sqrt(var_s/2) of s = |m|^2 come from a host table formed as
// the reference forms them, so the only difference from the reference's field
// is the device log / sin / cos of Box-Muller (a few ulp).
//
// LPT (LPTDisplacement::apply_to_arrays, src/ic/lpt_displacement.cpp:150-520):
// per axis a, psi_k = (-Im d, Re d) k_a/k^2, inverse transform times 1/M^3,
// sampled at lattice node (i, j, k) M/N and applied as x = wrap(x + x_f psi),
// p = p + p_f psi. The displacement spectra are zero outside the support
// |m_i| <= K < N/2, so their lattice samples are the N^3 inverse transform of
// the same modes (k_displacement): 8x less transform work than the M^3
// inverse when M = 2N, same values up to rounding. 2LPT: the six Hessian
// fields H_ab = c2r(d k_a k_b / k^2) (mixed terms 0 on either Nyquist plane)
// are transformed one at a time and folded into
// S = Hxx Hyy + (Hxx + Hyy) Hzz - Hxy^2 - Hxz^2 - Hyz^2, which is the
// reference's -1/2 sum H_aa^2 - sum H_ab^2 + 1/2 (tr H)^2 (tr H = d) without
// its trace transform; D2Z of S, band limit |m_i| <= K, then
// psi2_k = (Im S, -Re S) k_a/k^2. Wavenumbers are (2 pi m)/L
// (include/cosmo_nbody/mesh/mesh_geometry.hpp:112-115).
//
// Compiled with --fmad=false: the spectral multipliers and the particle
// update are the reference's expressions, rounded as its -ffp-contract=off
// build rounds them; the transforms (cuFFT) and the source's summation order
// round differently, at the level of the last bits.
//
// HBM traffic per mode / cell is a few words in each kernel; the FP64
// transforms dominate: 1LPT = 3 Z2D of N^3; 2LPT = 6 inverse transforms and 1
// D2Z of M^3 and 6 Z2D of N^3. On power-of-two IC meshes the six Hessian
// transforms run through the potential solve's own passes (generate_fused):
// the symbol is applied inside the x pass and the source accumulation inside
// the z pass, so no separate multiply or accumulate sweep touches HBM.
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <cufft.h>
#include <new>

#include "pm_common.cuh"
#include "pm_ic.h"
#include "pm_poisson.h"

namespace hyowon {
namespace ic {

namespace {

constexpr double kTwoPi = 6.283185307179586;  // 2.0 * std::numbers::pi, exact doubling

// ---------------------------------------------------------------- Philox ----

struct Draw {
    double u1, u2;
};

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
    constexpr uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u;
    constexpr uint32_t kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(kM0, c.x), lo0 = kM0 * c.x;
        const uint32_t hi1 = __umulhi(kM1, c.z), lo1 = kM1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        if (r != 9) {
            k0 += kW0;
            k1 += kW1;
        }
    }
    return c;
}

__device__ __forceinline__ double open_uniform(uint32_t hi, uint32_t lo) {
    const uint64_t bits = (static_cast<uint64_t>(hi) << 21) | (static_cast<uint64_t>(lo) >> 11);
    if (bits == 0) return 0x1.0p-54;
    return static_cast<double>(bits) * 0x1.0p-53;
}

__device__ __forceinline__ Draw mode_uniforms(uint64_t seed, int32_t mx, int32_t my, int32_t mz,
                                              uint32_t stream) {
    const uint4 w = philox4x32_10(
        make_uint4(static_cast<uint32_t>(mx), static_cast<uint32_t>(my),
                   static_cast<uint32_t>(mz), stream),
        static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
    return {open_uniform(w.x, w.y), open_uniform(w.z, w.w)};
}

__device__ __forceinline__ int mode_number(int i, int n) { return i <= n / 2 ? i : i - n; }

__device__ __forceinline__ void half_index(uint64_t idx, int M, int& ix, int& iy, int& iz) {
    const int hz = M / 2 + 1;
    iz = static_cast<int>(idx % hz);
    const uint64_t t = idx / hz;
    iy = static_cast<int>(t % M);
    ix = static_cast<int>(t / M);
}

// ----------------------------------------------------------------- field ----

// Element (i, j, k) of an M^3 half spectrum: row-major ((i M + j)(M/2+1) + k)
// when cc == 0, else the chunked layout of the five-pass transform
// ((k / cc) M^2 cc + (i M + j) cc + k % cc).
__device__ __forceinline__ uint64_t spectrum_at(int i, int j, int k, int M, int cc) {
    if (cc == 0)
        return (static_cast<uint64_t>(i) * M + j) * static_cast<uint64_t>(M / 2 + 1) + k;
    return static_cast<uint64_t>(k / cc) * static_cast<uint64_t>(M) * M * cc +
           (static_cast<uint64_t>(i) * M + j) * cc + k % cc;
}

__global__ void k_field(int M, int K, uint64_t seed, int fixed, int negate,
                        const double2* __restrict__ amp, double2* __restrict__ out_modes, int cc,
                        unsigned int* status) {
    const uint64_t total = static_cast<uint64_t>(M) * M * (M / 2 + 1);
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    int i, j, k;
    half_index(idx, M, i, j, k);
    double2* const out = out_modes + spectrum_at(i, j, k, M, cc);
    const int mx = mode_number(i, M), my = mode_number(j, M), mz = k;
    if ((mx == 0 && my == 0 && mz == 0) || abs(mx) > K || abs(my) > K || mz > K) {
        *out = make_double2(0.0, 0.0);
        return;
    }
    bool conjugate = false, self_conjugate = false;
    int ci = i, cj = j;
    if (k == 0 || ((M & 1) == 0 && k == M / 2)) {
        const int ti = (M - i) % M, tj = (M - j) % M;
        self_conjugate = ti == i && tj == j;
        if (!self_conjugate && (ti < i || (ti == i && tj < j))) {
            ci = ti;
            cj = tj;
            conjugate = true;
        }
    }
    const int64_t s = static_cast<int64_t>(mx) * mx + static_cast<int64_t>(my) * my +
                      static_cast<int64_t>(mz) * mz;
    const double2 a = amp[s];
    if (!(a.x > 0.0) || !(a.y > 0.0) || !isfinite(a.x) || !isfinite(a.y)) {
        raise_status(status, IC_AMPLITUDE);
        *out = make_double2(0.0, 0.0);
        return;
    }
    const Draw d = mode_uniforms(seed, mode_number(ci, M), mode_number(cj, M), mz, fixed ? 1u : 0u);
    double re, im;
    if (fixed) {
        if (self_conjugate) {
            re = d.u1 < 0.5 ? -a.x : a.x;
            im = 0.0;
        } else {
            double sn, cs;
            sincos(kTwoPi * d.u1, &sn, &cs);
            im = a.x * sn;
            if (conjugate) im = -im;
            re = a.x * cs;
        }
    } else {
        const double radius = sqrt(-2.0 * log(d.u1));
        double sn, cs;
        sincos(kTwoPi * d.u2, &sn, &cs);
        const double n1 = radius * cs, n2 = radius * sn;
        if (self_conjugate) {
            re = a.x * n1;
            im = 0.0;
        } else {
            re = a.y * n1;
            im = a.y * n2;
            if (conjugate) im = -im;
        }
    }
    if (negate) {
        re = -re;
        im = -im;
    }
    *out = make_double2(re, im);
}

// ------------------------------------------------------- spectral stages ----

// Half-spectrum coordinates of element idx with the index type I (32-bit
// whenever the spectrum has fewer than 2^32 elements: cheaper division).
template <typename I>
__device__ __forceinline__ void half_coords(I idx, I M, I hz, int& i, int& j, int& k) {
    k = static_cast<int>(idx % hz);
    const I t = idx / hz;
    j = static_cast<int>(t % M);
    i = static_cast<int>(t / M);
}

__device__ __forceinline__ double wavenumber(int m, double L) {
    return kTwoPi * static_cast<double>(m) / L;
}

// Hessian (a, b) of the field: dst = src * (k_a k_b / k^2), the mixed terms 0
// on either axis's Nyquist plane (include/cosmo_nbody/mesh/fourier_hessian.hpp).
template <typename I>
__global__ void k_hessian(int M, double L, int a, int b, const double2* __restrict__ src,
                          double2* __restrict__ dst) {
    const I total = static_cast<I>(M) * static_cast<I>(M) * static_cast<I>(M / 2 + 1);
    const I idx = static_cast<I>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    int i, j, k;
    half_coords<I>(idx, static_cast<I>(M), static_cast<I>(M / 2 + 1), i, j, k);
    const double kx = wavenumber(mode_number(i, M), L);
    const double ky = wavenumber(mode_number(j, M), L);
    const double kz = wavenumber(mode_number(k, M), L);
    const double k2 = kx * kx + ky * ky + kz * kz;
    if (k2 == 0.0) {
        dst[idx] = make_double2(0.0, 0.0);
        return;
    }
    const bool even = (M & 1) == 0;
    const int ia = a == 0 ? i : (a == 1 ? j : k);
    const int ib = b == 0 ? i : (b == 1 ? j : k);
    const double ka = a == 0 ? kx : (a == 1 ? ky : kz);
    const double kb = b == 0 ? kx : (b == 1 ? ky : kz);
    const bool mixed_nyquist = a != b && even && (ia == M / 2 || ib == M / 2);
    const double num = mixed_nyquist ? 0.0 : ka * kb;
    const double q = num / k2;
    const double2 v = src[idx];
    dst[idx] = make_double2(v.x * q, v.y * q);
}

// Displacement spectrum of axis a on the particle lattice's own N^3 mesh.
// The IC mesh field src (M^3 half spectrum) is zero outside the Cartesian
// support |m_i| <= K < N/2, so every retained mode has one image on the
// lattice mesh and the N^3 inverse transform of the restricted spectrum is
// exactly the M^3 inverse sampled at the lattice nodes (i, j, k) M/N.
// first: psi_k = (-Im d, Re d) k_a/k^2; second (2LPT, source S band-limited to
// K): (Im S, -Re S) k_a/k^2. Nyquist planes of the IC mesh lie outside the
// support (K < N/2 <= M/2), where k_a would be 0.
template <typename I>
__global__ void k_displacement(int N, int M, double L, int a, int K, bool second,
                               const double2* __restrict__ src, int cc, double2* __restrict__ dst) {
    const I total = static_cast<I>(N) * static_cast<I>(N) * static_cast<I>(N / 2 + 1);
    const I idx = static_cast<I>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    int i, j, k;
    half_coords<I>(idx, static_cast<I>(N), static_cast<I>(N / 2 + 1), i, j, k);
    const int mx = mode_number(i, N), my = mode_number(j, N), mz = k;
    if (abs(mx) > K || abs(my) > K || mz > K || (mx == 0 && my == 0 && mz == 0)) {
        dst[idx] = make_double2(0.0, 0.0);
        return;
    }
    const uint64_t at = spectrum_at(mx < 0 ? mx + M : mx, my < 0 ? my + M : my, mz, M, cc);
    const double kx = wavenumber(mx, L), ky = wavenumber(my, L), kz = wavenumber(mz, L);
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double kd = a == 0 ? kx : (a == 1 ? ky : kz);
    const double f = kd / k2;
    const double2 v = src[at];
    dst[idx] = second ? make_double2(v.y * f, -v.x * f) : make_double2(-v.y * f, v.x * f);
}

// ------------------------------------------------------------ real stages ----

// Corner lattice (src/ic/initial_conditions.cpp:295-313).
__global__ void k_lattice(int N, double dx, double* __restrict__ x, double* __restrict__ y,
                          double* __restrict__ z, double* __restrict__ px,
                          double* __restrict__ py, double* __restrict__ pz) {
    const uint64_t total = static_cast<uint64_t>(N) * N * N;
    const uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= total) return;
    const int k = static_cast<int>(p % N);
    const int j = static_cast<int>((p / N) % N);
    const int i = static_cast<int>(p / (static_cast<uint64_t>(N) * N));
    x[p] = static_cast<double>(i) * dx;
    y[p] = static_cast<double>(j) * dx;
    z[p] = static_cast<double>(k) * dx;
    px[p] = 0.0;
    py[p] = 0.0;
    pz[p] = 0.0;
}

// apply_lpt_component_update (src/ic/lpt_displacement.cpp:101-128): particle p
// sits on lattice node p of the N^3 displacement field; a non-finite psi or
// candidate leaves it unchanged and raises `flag`.
__global__ void k_apply(uint64_t n, const double* __restrict__ field, double norm, double xf,
                        double pf, double L, double* __restrict__ pos, double* __restrict__ mom,
                        unsigned int flag, unsigned int* status) {
    const uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double psi = field[p] * norm;
    const double disp = xf * psi;
    const double dmom = pf * psi;
    const double xc = pos[p] + disp;
    const double mc = mom[p] + dmom;
    const double w = wrap_f64(xc, L);
    if (!isfinite(psi) || !isfinite(disp) || !isfinite(dmom) || !isfinite(xc) || !isfinite(mc) ||
        !isfinite(w)) {
        raise_status(status, flag);
        return;
    }
    pos[p] = w;
    mom[p] = mc;
}

// The 2LPT source as the second invariant of the Hessian minus the mixed
// squares, S = Hxx Hyy + (Hxx + Hyy) Hzz - Hxy^2 - Hxz^2 - Hyz^2: equal to the
// reference's -1/2 sum H_aa^2 - sum H_ab^2 + 1/2 (tr H)^2 with tr H = sum H_aa
// (its Hessian keeps k_a^2 on Nyquist planes), one transform fewer and no
// cancellation between the trace and diagonal squares. One normalised field
// h per launch: op 0 (xx): A = h; 1 (yy): S = A h, A += h; 2 (zz): S += A h;
// 3 (mixed): S -= h h; the last launch checks S.
__global__ void k_source(uint64_t n, const double* __restrict__ field, double norm, int op,
                         bool last, double* __restrict__ acc, double* __restrict__ src,
                         unsigned int* status) {
    const uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double h = field[c] * norm;
    if (!isfinite(h)) raise_status(status, IC_HESSIAN);
    double s;
    if (op == 0) {
        acc[c] = h;
        return;
    } else if (op == 1) {
        const double a = acc[c];
        s = a * h;
        acc[c] = a + h;
    } else if (op == 2) {
        s = src[c] + acc[c] * h;
    } else {
        s = src[c] - h * h;
    }
    if (last && !isfinite(s)) raise_status(status, IC_SOURCE);
    src[c] = s;
}

inline unsigned grid(uint64_t n) { return static_cast<unsigned>((n + 255) / 256); }

// cuFFT plans on the IC mesh with one shared work area.
struct Fft {
    cufftHandle c2r = 0, r2c = 0;
    bool has_c2r = false, has_r2c = false;
    void* ws = nullptr;
    ~Fft() { reset(); }
    void reset() {
        if (has_c2r) cufftDestroy(c2r);
        if (has_r2c) cufftDestroy(r2c);
        cudaFree(ws);
        has_c2r = has_r2c = false;
        ws = nullptr;
    }
    int make(int M, bool forward, cudaStream_t s, const char** err, bool inverse = true) {
        reset();
        size_t w1 = 0, w2 = 0;
        if (inverse) {
            if (cufftCreate(&c2r) != CUFFT_SUCCESS) return *err = "cufftCreate failed", HYOWON_ECUDA;
            has_c2r = true;
            cufftSetAutoAllocation(c2r, 0);
            if (cufftMakePlan3d(c2r, M, M, M, CUFFT_Z2D, &w1) != CUFFT_SUCCESS)
                return *err = "cuFFT Z2D plan for the IC mesh failed", HYOWON_ECUDA;
        }
        if (forward) {
            if (cufftCreate(&r2c) != CUFFT_SUCCESS) return *err = "cufftCreate failed", HYOWON_ECUDA;
            has_r2c = true;
            cufftSetAutoAllocation(r2c, 0);
            if (cufftMakePlan3d(r2c, M, M, M, CUFFT_D2Z, &w2) != CUFFT_SUCCESS)
                return *err = "cuFFT D2Z plan for the IC mesh failed", HYOWON_ECUDA;
        }
        size_t w = w1 > w2 ? w1 : w2;
        if (w < 256) w = 256;
        if (cudaMalloc(&ws, w) != cudaSuccess)
            return *err = "cuFFT work area for the IC mesh could not be allocated", HYOWON_ENOMEM;
        if (inverse) {
            cufftSetWorkArea(c2r, ws);
            cufftSetStream(c2r, s);
        }
        if (forward) {
            cufftSetWorkArea(r2c, ws);
            cufftSetStream(r2c, s);
        }
        return HYOWON_OK;
    }
};

template <typename T>
struct DeviceBuffer {
    T* p = nullptr;
    ~DeviceBuffer() { cudaFree(p); }
    bool alloc(size_t n) {
        cudaFree(p);
        p = nullptr;
        return cudaMalloc(&p, sizeof(T) * n) == cudaSuccess;
    }
};

// ------------------------------------------------- scaled positive product --

// Binary mantissa / exponent product in long double, one factor at a time, as
// math::ScaledPositiveProduct consumes and materialises
// (include/cosmo_nbody/math/scaled_positive_product.hpp:425-512).
struct Scaled {
    long double mant = 1.0L;
    long long expo = 0;
    void consume(double factor, bool divide) {
        int fe = 0;
        const long double fw = static_cast<long double>(std::frexp(factor, &fe));
        if (divide) {
            mant = mant / fw;
            expo -= fe;
        } else {
            mant = mant * fw;
            expo += fe;
        }
        int ne = 0;
        mant = std::frexp(mant, &ne);
        expo += ne;
    }
    // 0 on success, 1 underflow, 2 overflow.
    static int materialize(long double m, long long e, double* out) {
        if (e < INT_MIN || e > INT_MAX) return 2;
        const long double wide = std::scalbn(m, static_cast<int>(e));
        if (wide == 0.0L) return 1;
        if (!std::isfinite(wide) || wide < 0.0L || wide > static_cast<long double>(DBL_MAX)) return 2;
        const double r = static_cast<double>(wide);
        if (!std::isfinite(r) || r <= 0.0) return 1;
        *out = r;
        return 0;
    }
    // sqrt(this * num / den) without materialising the square.
    int sqrt_of_quotient(double num, double den, double* out) const {
        Scaled t = *this;
        t.consume(num, false);
        t.consume(den, true);
        long long q = t.expo / 2, rem = t.expo % 2;
        if (rem < 0) {
            rem += 2;
            --q;
        }
        const long double root = std::sqrt(std::scalbn(t.mant, static_cast<int>(rem)));
        if (!std::isfinite(root) || !(root > 0.0L)) return 2;
        return materialize(root, q, out);
    }
};

}  // namespace

// ------------------------------------------------------------------ host ----

int resolve(const hyowon_ic_params_t* in, Params* out, const char** err) {
    if (!in || !out) return *err = "null IC parameters", HYOWON_EINVAL;
    const uint64_t N = in->particles_per_dimension;
    if (N == 0) return *err = "particles_per_dimension must be positive", HYOWON_EINVAL;
    if (N > 1625) return *err = "Configured particle population N^3 exceeds the uint32 count range", HYOWON_EOVERFLOW;
    if (!std::isfinite(in->box_size) || !(in->box_size > 0.0))
        return *err = "Box size must be finite and positive", HYOWON_EINVAL;
    if (in->max_mode_per_axis >= 0 &&
        (in->max_mode_per_axis == 0 || static_cast<uint64_t>(in->max_mode_per_axis) > (N - 1) / 2))
        return *err = "ic.max_mode_per_axis must be positive and satisfy 2*K < particles_per_dimension",
               HYOWON_EINVAL;
    const uint64_t K = in->max_mode_per_axis >= 0 ? static_cast<uint64_t>(in->max_mode_per_axis)
                                                  : (N - 1) / 2;
    if (K == 0)
        return *err = "Generated IC particle lattice must admit at least one nonzero Fourier mode",
               HYOWON_EINVAL;
    if (in->lpt_order != 1 && in->lpt_order != 2)
        return *err = "ic.lpt_order must be 1 or 2", HYOWON_EINVAL;
    // projected_2lpt_source_mesh_is_alias_free (particle_lattice_bandlimit.hpp:56-61)
    auto alias_free = [](uint64_t m, uint64_t k) { return m != 0 && k <= (m - 1) / 3; };
    uint64_t M = in->mesh_per_dimension;
    if (M == 0) M = (in->lpt_order == 2 && !alias_free(N, K)) ? 2 * N : N;
    if (M > static_cast<uint64_t>(INT_MAX))
        return *err = "IC mesh dimension must fit the int-based FFT and mesh APIs", HYOWON_EOVERFLOW;
    if (M % N != 0)
        return *err = "Generated IC mesh must be an integer multiple of particles_per_dimension",
               HYOWON_EINVAL;
    if (in->lpt_order == 2 && !alias_free(M, K))
        return *err = "Generated projected 2LPT IC mesh must satisfy M > 3*K", HYOWON_EINVAL;
    if (in->amplitude_mode != HYOWON_IC_GAUSSIAN && in->amplitude_mode != HYOWON_IC_FIXED)
        return *err = "ic.amplitude_mode must be 'gaussian' or 'fixed'", HYOWON_EINVAL;
    if (in->phase_pairing < HYOWON_IC_INDEPENDENT || in->phase_pairing > HYOWON_IC_PAIR_B)
        return *err = "ic.phase_pairing must be 'independent', 'pair_a', or 'pair_b'", HYOWON_EINVAL;
    if (!std::isfinite(in->momentum_factor_1) ||
        (in->lpt_order == 2 &&
         (!std::isfinite(in->position_factor_2) || !std::isfinite(in->momentum_factor_2))))
        return *err = "Invalid start-scaled LPT normalization", HYOWON_ERUNTIME;
    out->N = static_cast<int>(N);
    out->M = static_cast<int>(M);
    out->L = in->box_size;
    out->seed = in->seed;
    out->K = static_cast<int>(K);
    out->fixed = in->amplitude_mode == HYOWON_IC_FIXED;
    out->negate = in->phase_pairing == HYOWON_IC_PAIR_B;
    out->order = in->lpt_order;
    out->p1 = in->momentum_factor_1;
    out->x2 = in->position_factor_2;
    out->p2 = in->momentum_factor_2;
    return HYOWON_OK;
}

int mode_amplitudes(uint64_t M, double L, uint64_t n, const double* power, double* amp,
                    const char** err) {
    if (M == 0 || !std::isfinite(L) || !(L > 0.0) || (n && (!power || !amp)))
        return *err = "mode amplitudes need M > 0, a finite positive box and the tables",
               HYOWON_EINVAL;
    Scaled norm;
    const double nr = static_cast<double>(M);
    for (int r = 0; r < 6; ++r) norm.consume(nr, false);
    for (int r = 0; r < 3; ++r) norm.consume(L, true);
    for (uint64_t s = 0; s < n; ++s) {
        amp[2 * s] = amp[2 * s + 1] = 0.0;
        if (s == 0) continue;
        const double p = power[s];
        if (!std::isfinite(p) || !(p > 0.0))
            return *err = "RandomField power spectrum returned invalid P(k)", HYOWON_ERUNTIME;
        Scaled t = norm;
        t.consume(p, false);
        double var = 0.0;
        const bool have = Scaled::materialize(t.mant, t.expo, &var) == 0;
        double a1 = 0.0, a2 = 0.0;
        int bad = 0;
        if (have) {
            a1 = std::sqrt(var);
            const double reduced = var / 2.0;
            if (reduced > 0.0) a2 = std::sqrt(reduced);
            else bad |= norm.sqrt_of_quotient(p, 2.0, &a2);
        } else {
            bad |= norm.sqrt_of_quotient(p, 1.0, &a1);
            bad |= norm.sqrt_of_quotient(p, 2.0, &a2);
        }
        if (bad || !std::isfinite(a1) || !std::isfinite(a2))
            return *err = "RandomField mode amplitude is not representable as finite core::Real",
                   HYOWON_EOVERFLOW;
        amp[2 * s] = a1;
        amp[2 * s + 1] = a2;
    }
    return HYOWON_OK;
}

int upload_amplitudes(const Params& p, uint64_t n_power, const double* power, double2** d_amp,
                      const char** err) {
    const uint64_t need = 3ull * p.K * p.K + 1;
    if (!power || n_power < need)
        return *err = "power must hold P(k_s) for s = 0 .. 3K^2", HYOWON_EINVAL;
    double* amp = static_cast<double*>(std::malloc(sizeof(double) * 2 * need));
    if (!amp) return *err = "host amplitude table could not be allocated", HYOWON_ENOMEM;
    int rc = mode_amplitudes(static_cast<uint64_t>(p.M), p.L, need, power, amp, err);
    if (rc == HYOWON_OK) {
        if (cudaMalloc(d_amp, sizeof(double2) * need) != cudaSuccess) {
            *err = "device amplitude table could not be allocated";
            rc = HYOWON_ENOMEM;
        } else if (cudaMemcpy(*d_amp, amp, sizeof(double2) * need, cudaMemcpyHostToDevice) !=
                   cudaSuccess) {
            cudaFree(*d_amp);
            *d_amp = nullptr;
            *err = "amplitude table upload failed";
            rc = HYOWON_ECUDA;
        }
    }
    std::free(amp);
    return rc;
}

int status_code(unsigned int st, const char** err) {
    if (!st) return HYOWON_OK;
    if (st & IC_AMPLITUDE) return *err = "RandomField power spectrum returned invalid P(k)", HYOWON_ERUNTIME;
    if (st & IC_PSI1) return *err = "1LPT particle update is non-finite or unrepresentable", HYOWON_ERUNTIME;
    if (st & IC_HESSIAN) return *err = "2LPT first-order Hessian is non-finite", HYOWON_ERUNTIME;
    if (st & IC_SOURCE) return *err = "2LPT quadratic source is non-finite", HYOWON_EOVERFLOW;
    return *err = "2LPT particle update is non-finite or unrepresentable", HYOWON_ERUNTIME;
}

// ---------------------------------------------------------------- device ----

int field_device(const Params& p, const double2* d_amp, double2* d_modes, unsigned int* d_status,
                 cudaStream_t s, const char** err, int cc) {
    const uint64_t half = static_cast<uint64_t>(p.M) * p.M * (p.M / 2 + 1);
    k_field<<<grid(half), 256, 0, s>>>(p.M, p.K, p.seed, p.fixed, p.negate, d_amp, d_modes, cc,
                                       d_status);
    if (cudaGetLastError() != cudaSuccess) return *err = "IC field launch failed", HYOWON_ECUDA;
    return HYOWON_OK;
}

namespace {
struct PlanOwner {
    poisson::Plan* p = nullptr;
    ~PlanOwner() { poisson::destroy_plan(p); }
    void reset() {
        poisson::destroy_plan(p);
        p = nullptr;
    }
};
}  // namespace

// Work arrays and plans of generate_fused for one (N, M, L).
struct Workspace {
    int N = 0, M = 0;
    double L = 0.0;
    bool ready = false;
    DeviceBuffer<double2> delta, work, psi_n, tw;
    DeviceBuffer<double> acc, source, field_n, ktab;
    PlanOwner pd, pw;
    Fft fft_m, fft_n;

    int prepare(const Params& p, cudaStream_t s, const char** err) {
        if (ready && N == p.N && M == p.M && L == p.L) {
            // the cuFFT plans follow the caller's stream
            cufftSetStream(fft_m.r2c, s);
            cufftSetStream(fft_n.c2r, s);
            return HYOWON_OK;
        }
        ready = false;
        N = p.N;
        M = p.M;
        L = p.L;
        const uint64_t cells = static_cast<uint64_t>(M) * M * M;
        const uint64_t n = static_cast<uint64_t>(N) * N * N;
        const uint64_t half_n = static_cast<uint64_t>(N) * N * (N / 2 + 1);
        const size_t chunked = poisson::modes_elements_f64(M);
        if (!delta.alloc(chunked) || !work.alloc(chunked) || !acc.alloc(cells) ||
            !source.alloc(cells) || !psi_n.alloc(half_n) || !field_n.alloc(n) || !tw.alloc(M) ||
            !ktab.alloc(M))
            return *err = "IC mesh work arrays could not be allocated", HYOWON_ENOMEM;
        // twiddles exp(-2 pi i m / M) and wavenumbers (2 pi m) / L (the device
        // expression: two IEEE roundings, as on the host)
        double* h = static_cast<double*>(std::malloc(sizeof(double) * 3 * M));
        if (!h) return *err = "host twiddle table could not be allocated", HYOWON_ENOMEM;
        poisson::twiddles(M, h);
        for (int i = 0; i < M; ++i) {
            const int m = i <= M / 2 ? i : i - M;
            h[2 * M + i] = kTwoPi * static_cast<double>(m) / p.L;
        }
        const bool ok =
            cudaMemcpy(tw.p, h, sizeof(double2) * M, cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(ktab.p, h + 2 * M, sizeof(double) * M, cudaMemcpyHostToDevice) == cudaSuccess;
        std::free(h);
        if (!ok) return *err = "twiddle upload failed", HYOWON_ECUDA;
        pd.reset();
        pw.reset();
        if (!(pd.p = poisson::create_plan(M, false, delta.p, err)) ||
            !(pw.p = poisson::create_plan(M, false, work.p, err)))
            return HYOWON_ECUDA;
        int rc = fft_m.make(M, true, s, err, false);   // D2Z of the source only
        if (!rc) rc = fft_n.make(N, false, s, err);
        if (rc) return rc;
        ready = true;
        return HYOWON_OK;
    }
};

Workspace* workspace_create() { return new (std::nothrow) Workspace(); }
void workspace_destroy(Workspace* w) { delete w; }

namespace {
// 2LPT on a power-of-two IC mesh with the five-pass transform machinery: the
// field in its chunked layout, each Hessian as three passes (symbol and
// inverse x, inverse y, c2r along z folding into the source), the D2Z of the
// source and the N^3 displacement transforms by cuFFT. The arithmetic is the
// generator's; the transforms round differently from cuFFT's. Four M^3
// fields (spectrum, work spectrum, two source accumulators) instead of five.
int generate_fused(const Params& p, const double2* d_amp, double* const d_pos[3],
                   double* const d_mom[3], unsigned int* d_status, cudaStream_t s,
                   const char** err, Workspace& w) {
    const int M = p.M, N = p.N;
    const uint64_t n = static_cast<uint64_t>(N) * N * N;
    const uint64_t half_n = static_cast<uint64_t>(N) * N * (N / 2 + 1);
    const int cc = poisson::chunk_columns_f64(M);
    const double norm = 1.0 / (static_cast<double>(M) * M * M);
    int rc = w.prepare(p, s, err);
    if (rc) return rc;
    const bool small_n = half_n < (1ull << 32);
    auto displacements = [&](const double2* src, int src_cc, bool second_order, double xf,
                             double pf, unsigned int flag) -> int {
        for (int a = 0; a < 3; ++a) {
            if (small_n)
                k_displacement<uint32_t><<<grid(half_n), 256, 0, s>>>(N, M, p.L, a, p.K,
                                                                      second_order, src, src_cc,
                                                                      w.psi_n.p);
            else
                k_displacement<uint64_t><<<grid(half_n), 256, 0, s>>>(N, M, p.L, a, p.K,
                                                                      second_order, src, src_cc,
                                                                      w.psi_n.p);
            if (cufftExecZ2D(w.fft_n.c2r, reinterpret_cast<cufftDoubleComplex*>(w.psi_n.p),
                             w.field_n.p) != CUFFT_SUCCESS)
                return *err = "IC c2r failed", HYOWON_ECUDA;
            k_apply<<<grid(n), 256, 0, s>>>(n, w.field_n.p, norm, xf, pf, p.L, d_pos[a],
                                            d_mom[a], flag, d_status);
        }
        return HYOWON_OK;
    };
    k_lattice<<<grid(n), 256, 0, s>>>(N, p.L / static_cast<double>(N), d_pos[0], d_pos[1],
                                      d_pos[2], d_mom[0], d_mom[1], d_mom[2]);
    if ((rc = field_device(p, d_amp, w.delta.p, d_status, s, err, cc))) return rc;
    if ((rc = displacements(w.delta.p, cc, false, 1.0, p.p1, IC_PSI1))) return rc;
    static const int pairs[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    for (int t = 0; t < 6; ++t) {
        const poisson::HessianF64 h{w.ktab.p, pairs[t][0], pairs[t][1]};
        const poisson::SourceTermF64 term{t < 3 ? t : 3, t == 5, norm, w.acc.p, w.source.p,
                                          d_status, IC_HESSIAN, IC_SOURCE};
        if (poisson::hessian_source_f64(w.pd.p, w.pw.p, M, w.work.p, w.tw.p, h, term, d_status,
                                        s) < 0)
            return *err = "IC Hessian pass launch failed", HYOWON_ECUDA;
    }
    // S -> S_k, row-major, in the work buffer
    if (cufftExecD2Z(w.fft_m.r2c, w.source.p, reinterpret_cast<cufftDoubleComplex*>(w.work.p)) !=
        CUFFT_SUCCESS)
        return *err = "IC r2c of the 2LPT source failed", HYOWON_ECUDA;
    if ((rc = displacements(w.work.p, 0, true, p.x2, p.p2, IC_PSI2))) return rc;
    if (cudaStreamSynchronize(s) != cudaSuccess) return *err = "IC kernels failed", HYOWON_ECUDA;
    return HYOWON_OK;
}
}  // namespace

// HYOWON_IC_FUSED: 2LPT on power-of-two IC meshes through generate_fused.
#ifndef HYOWON_IC_FUSED
#define HYOWON_IC_FUSED 1
#endif

int generate_device(const Params& p, const double2* d_amp, double* const d_pos[3],
                    double* const d_mom[3], unsigned int* d_status, cudaStream_t s,
                    const char** err, Workspace* ws) {
    if (HYOWON_IC_FUSED && p.order == 2 && poisson::supported(p.M)) {
        if (ws) return generate_fused(p, d_amp, d_pos, d_mom, d_status, s, err, *ws);
        Workspace local;
        return generate_fused(p, d_amp, d_pos, d_mom, d_status, s, err, local);
    }
    const int M = p.M, N = p.N;
    const uint64_t half = static_cast<uint64_t>(M) * M * (M / 2 + 1);
    const uint64_t cells = static_cast<uint64_t>(M) * M * M;
    const uint64_t n = static_cast<uint64_t>(N) * N * N;
    const uint64_t half_n = static_cast<uint64_t>(N) * N * (N / 2 + 1);
    const bool folded = M != N;
    const double norm = 1.0 / (static_cast<double>(M) * M * M);
    const bool small_m = half < (1ull << 32), small_n = half_n < (1ull << 32);
    // delta (M half spectrum) stays; work / field serve the Hessians (M) and,
    // when M == N, the displacements; psi_n / field_n hold the folded N^3
    // displacements otherwise. acc / source: the 2LPT source terms.
    DeviceBuffer<double2> delta, work, psi_n;
    DeviceBuffer<double> field, field_n, acc, source;
    const bool second = p.order == 2;
    if (!delta.alloc(half) || (second && (!work.alloc(half) || !field.alloc(cells))) ||
        (second && (!acc.alloc(cells) || !source.alloc(cells))) ||
        ((folded || !second) && (!psi_n.alloc(half_n) || !field_n.alloc(n))))
        return *err = "IC mesh work arrays could not be allocated", HYOWON_ENOMEM;
    // M == N with 2LPT: the displacements reuse the Hessian buffers
    double2* const disp_k = psi_n.p ? psi_n.p : work.p;
    double* const disp_r = field_n.p ? field_n.p : field.p;
    Fft fft_m, fft_n;
    int rc = 0;
    if (second && (rc = fft_m.make(M, true, s, err))) return rc;
    if ((folded || !second) && (rc = fft_n.make(N, false, s, err))) return rc;
    const cufftHandle c2r_n = (folded || !second) ? fft_n.c2r : fft_m.c2r;

    auto displacements = [&](const double2* src, int src_cc, bool second_order, double xf,
                             double pf, unsigned int flag) -> int {
        for (int a = 0; a < 3; ++a) {
            if (small_n)
                k_displacement<uint32_t><<<grid(half_n), 256, 0, s>>>(N, M, p.L, a, p.K,
                                                                      second_order, src, src_cc,
                                                                      disp_k);
            else
                k_displacement<uint64_t><<<grid(half_n), 256, 0, s>>>(N, M, p.L, a, p.K,
                                                                      second_order, src, src_cc,
                                                                      disp_k);
            if (cufftExecZ2D(c2r_n, reinterpret_cast<cufftDoubleComplex*>(disp_k), disp_r) !=
                CUFFT_SUCCESS)
                return *err = "IC c2r failed", HYOWON_ECUDA;
            k_apply<<<grid(n), 256, 0, s>>>(n, disp_r, norm, xf, pf, p.L, d_pos[a], d_mom[a],
                                            flag, d_status);
        }
        return HYOWON_OK;
    };

    k_lattice<<<grid(n), 256, 0, s>>>(N, p.L / static_cast<double>(N), d_pos[0], d_pos[1],
                                      d_pos[2], d_mom[0], d_mom[1], d_mom[2]);
    if ((rc = field_device(p, d_amp, delta.p, d_status, s, err))) return rc;
    if ((rc = displacements(delta.p, 0, false, 1.0, p.p1, IC_PSI1))) return rc;
    if (second) {
        static const int pairs[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
        for (int t = 0; t < 6; ++t) {
            if (small_m)
                k_hessian<uint32_t><<<grid(half), 256, 0, s>>>(M, p.L, pairs[t][0], pairs[t][1],
                                                               delta.p, work.p);
            else
                k_hessian<uint64_t><<<grid(half), 256, 0, s>>>(M, p.L, pairs[t][0], pairs[t][1],
                                                               delta.p, work.p);
            if (cufftExecZ2D(fft_m.c2r, reinterpret_cast<cufftDoubleComplex*>(work.p), field.p) !=
                CUFFT_SUCCESS)
                return *err = "IC c2r failed", HYOWON_ECUDA;
            k_source<<<grid(cells), 256, 0, s>>>(cells, field.p, norm, t < 3 ? t : 3, t == 5,
                                                 acc.p, source.p, d_status);
        }
        // S -> S_k in the delta buffer (delta is no longer needed)
        if (cufftExecD2Z(fft_m.r2c, source.p, reinterpret_cast<cufftDoubleComplex*>(delta.p)) !=
            CUFFT_SUCCESS)
            return *err = "IC r2c of the 2LPT source failed", HYOWON_ECUDA;
        if ((rc = displacements(delta.p, 0, true, p.x2, p.p2, IC_PSI2))) return rc;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return *err = "IC kernels failed", HYOWON_ECUDA;
    return HYOWON_OK;
}

}  // namespace ic
}  // namespace hyowon

// ------------------------------------------------------------------ C ABI ---

namespace {
thread_local char g_ic_err[256] = "";

int ic_fail(int rc, const char* msg) {
    std::strncpy(g_ic_err, msg ? msg : "IC generation failed", sizeof(g_ic_err) - 1);
    g_ic_err[sizeof(g_ic_err) - 1] = '\0';
    return rc;
}

// Device state of one standalone call.
struct Call {
    cudaStream_t s = nullptr;
    unsigned int* d_status = nullptr;
    double2* d_amp = nullptr;
    ~Call() {
        if (s) cudaStreamDestroy(s);
        cudaFree(d_status);
        cudaFree(d_amp);
    }
    int open(const hyowon::ic::Params& p, uint64_t n_power, const double* power,
             const char** err) {
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaMalloc(&d_status, sizeof(unsigned int)) != cudaSuccess ||
            cudaMemset(d_status, 0, sizeof(unsigned int)) != cudaSuccess)
            return *err = "CUDA stream / status allocation failed", HYOWON_ECUDA;
        return hyowon::ic::upload_amplitudes(p, n_power, power, &d_amp, err);
    }
    int finish(const char** err) {
        unsigned int st = 0;
        if (cudaStreamSynchronize(s) != cudaSuccess ||
            cudaMemcpy(&st, d_status, sizeof(st), cudaMemcpyDeviceToHost) != cudaSuccess)
            return *err = "IC kernels failed", HYOWON_ECUDA;
        return hyowon::ic::status_code(st, err);
    }
};
}  // namespace

extern "C" {

const char* hyowon_ic_last_error(void) { return g_ic_err; }

int hyowon_ic_resolve(const hyowon_ic_params_t* p, uint64_t* mesh, uint64_t* max_mode) {
    hyowon::ic::Params r;
    const char* err = nullptr;
    const int rc = hyowon::ic::resolve(p, &r, &err);
    if (rc) return ic_fail(rc, err);
    if (mesh) *mesh = static_cast<uint64_t>(r.M);
    if (max_mode) *max_mode = static_cast<uint64_t>(r.K);
    return HYOWON_OK;
}

int hyowon_ic_mode_amplitudes(uint64_t mesh, double box_size, uint64_t n, const double* power,
                              double* amp) {
    const char* err = nullptr;
    const int rc = hyowon::ic::mode_amplitudes(mesh, box_size, n, power, amp, &err);
    return rc ? ic_fail(rc, err) : HYOWON_OK;
}

int hyowon_ic_field(const hyowon_ic_params_t* p, uint64_t n_power, const double* power,
                    double* modes) {
    hyowon::ic::Params r;
    const char* err = nullptr;
    int rc = hyowon::ic::resolve(p, &r, &err);
    if (rc) return ic_fail(rc, err);
    if (!modes) return ic_fail(HYOWON_EINVAL, "modes must not be NULL");
    Call c;
    if ((rc = c.open(r, n_power, power, &err))) return ic_fail(rc, err);
    const uint64_t half = static_cast<uint64_t>(r.M) * r.M * (r.M / 2 + 1);
    double2* d_modes = nullptr;
    if (cudaMalloc(&d_modes, sizeof(double2) * half) != cudaSuccess)
        return ic_fail(HYOWON_ENOMEM, "IC field could not be allocated");
    rc = hyowon::ic::field_device(r, c.d_amp, d_modes, c.d_status, c.s, &err);
    if (!rc) rc = c.finish(&err);
    if (!rc && cudaMemcpy(modes, d_modes, sizeof(double2) * half, cudaMemcpyDeviceToHost) !=
                   cudaSuccess) {
        rc = HYOWON_ECUDA;
        err = "IC field download failed";
    }
    cudaFree(d_modes);
    return rc ? ic_fail(rc, err) : HYOWON_OK;
}

int hyowon_ic_generate(const hyowon_ic_params_t* p, uint64_t n_power, const double* power,
                       double* x, double* y, double* z, double* px, double* py, double* pz) {
    hyowon::ic::Params r;
    const char* err = nullptr;
    int rc = hyowon::ic::resolve(p, &r, &err);
    if (rc) return ic_fail(rc, err);
    double* host[6] = {x, y, z, px, py, pz};
    for (double* h : host)
        if (!h) return ic_fail(HYOWON_EINVAL, "particle arrays must not be NULL");
    Call c;
    if ((rc = c.open(r, n_power, power, &err))) return ic_fail(rc, err);
    const uint64_t n = static_cast<uint64_t>(r.N) * r.N * r.N;
    double* d = nullptr;
    if (cudaMalloc(&d, sizeof(double) * 6 * n) != cudaSuccess)
        return ic_fail(HYOWON_ENOMEM, "particle arrays could not be allocated on the device");
    double* const pos[3] = {d, d + n, d + 2 * n};
    double* const mom[3] = {d + 3 * n, d + 4 * n, d + 5 * n};
    rc = hyowon::ic::generate_device(r, c.d_amp, pos, mom, c.d_status, c.s, &err);
    if (!rc) rc = c.finish(&err);
    for (int a = 0; a < 6 && !rc; ++a)
        if (cudaMemcpy(host[a], d + a * n, sizeof(double) * n, cudaMemcpyDeviceToHost) !=
            cudaSuccess) {
            rc = HYOWON_ECUDA;
            err = "particle download failed";
        }
    cudaFree(d);
    return rc ? ic_fail(rc, err) : HYOWON_OK;
}

}  // extern "C"
