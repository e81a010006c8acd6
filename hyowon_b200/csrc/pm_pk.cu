// pm_pk.cu -- binary64 matter power spectrum of the device particle state:
// the estimator of analysis::MatterPowerSpectrum::compute_pk
// (src/analysis/matter_power_spectrum.cpp:50-226) over the density field of
// FourierDensityBuilder::build (src/analysis/fourier_density_field.cpp:110-376).
//
//   CIC deposit of weights w_i = m_i / max m (1 for equal masses) on an N^3
//   mesh -> contrast rho / (sum w / N^3) - 1 -> unnormalised r2c -> modes / N^3
//   [interlaced: the same from positions wrap(x - dx/2) combined as
//   0.5 (F + F_shift e^{-i (kx+ky+kz) dx/2})] -> per mode with 0 < |k| <= k_max:
//   raw power L^3 |delta|^2, CIC window W = prod_axes min(1, |sin a / a|)^2
//   (a = k dx / 2), corrected power (raw or L^3 |delta|^2 minus the aliased
//   shot noise L^3 sum w^2/(sum w)^2 prod_axes (1 - 2/3 sin^2 a)) / W^2,
//   half-spectrum multiplicity 1 (kz = 0, Nyquist plane) or 2 -> logarithmic
//   bins from 2 pi / L to k_max (PositiveLogBinGrid, last bin closed):
//   multiplicity-weighted means and mode counts.
//
// This unit is compiled with --fmad=false: the per-mode products, the complex
// interlacing product and the contrast follow the reference's operation order
// without contraction. Per-axis k, window and sin^2 values are tabulated on
// the host with the reference's formulas (the window in long double). The
// deposit adds with binary64 atomics, so results agree with the reference to
// rounding (~1e-15 relative), not bit for bit.
#include "pm_pk.h"

#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "hyowon_pm.h"
#include "pm_common.cuh"
#include "pm_kernels.h"

namespace hyowon {
namespace pk {

namespace {

constexpr int kThreads = 256;
constexpr int kFields = 4;   // k, raw power, corrected power, deconvolution factor

__global__ void k_contrast(uint64_t cells, double* __restrict__ rho, double mean) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < cells;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        rho[i] = rho[i] / mean - 1.0;
}

__global__ void k_shift_wrap(uint32_t n, const double* __restrict__ in, double shift, double L,
                             double* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = wrap_f64(in[i] - shift, L);
}

// Per-block bin sums over a grid-stride range of half-spectrum modes
// (row-major [ix][iy][iz], iz <= N/2), shared-memory accumulators, block
// partials to partial[block][bin][field] and pcount[block][bin].
__global__ void __launch_bounds__(kThreads)
k_bins(int N, double L3, double norm, const double2* __restrict__ modes,
       const double2* __restrict__ shifted, double shift, const double* __restrict__ kt,
       const double* __restrict__ wt, const double* __restrict__ s2t,
       const double* __restrict__ edges, int nb, double k_max, double shot, int subtract,
       double* __restrict__ partial, unsigned long long* __restrict__ pcount) {
    extern __shared__ double sb[];
    double* sums = sb;                                                    // nb * kFields
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(sb + nb * kFields);  // nb
    double* ed = sb + nb * kFields + nb;                                  // nb + 1
    for (int i = threadIdx.x; i < nb * kFields; i += blockDim.x) sums[i] = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) cnt[i] = 0ull;
    for (int i = threadIdx.x; i <= nb; i += blockDim.x) ed[i] = edges[i];
    __syncthreads();
    const int Hz = N / 2 + 1;
    const bool even = (N % 2) == 0;
    const uint64_t total = static_cast<uint64_t>(N) * N * Hz;
    for (uint64_t m = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; m < total;
         m += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const int iz = static_cast<int>(m % Hz);
        const int iy = static_cast<int>((m / Hz) % N);
        const int ix = static_cast<int>(m / (static_cast<uint64_t>(Hz) * N));
        const double kx = kt[ix], ky = kt[iy], kz = kt[iz];
        const double kmag = hypot(hypot(kx, ky), kz);
        if (!(kmag > 0.0) || kmag > k_max) continue;
        if (kmag < ed[0] || kmag > ed[nb]) continue;
        int bin;
        if (kmag == ed[nb]) {
            bin = nb - 1;
        } else {
            int lo = 0, hi = nb;   // first edge > kmag lies in (lo, hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (ed[mid] > kmag) hi = mid; else lo = mid;
            }
            bin = lo;
        }
        double2 a = modes[m];
        a.x *= norm;
        a.y *= norm;
        if (shifted) {
            double2 b = shifted[m];
            b.x *= norm;
            b.y *= norm;
            const double phase = -(kx + ky + kz) * shift;
            const double c = cos(phase), s = sin(phase);
            const double bcx = b.x * c - b.y * s;
            const double bcy = b.x * s + b.y * c;
            a.x = 0.5 * (a.x + bcx);
            a.y = 0.5 * (a.y + bcy);
        }
        const double norm2 = a.x * a.x + a.y * a.y;
        const double p_raw = L3 * norm2;
        const double window = wt[ix] * wt[iy] * wt[iz];
        const double deconv = 1.0 / (window * window);
        double p_corr = p_raw;
        if (subtract) {
            const double aliased = shot * (1.0 - 2.0 / 3.0 * s2t[ix]) * (1.0 - 2.0 / 3.0 * s2t[iy])
                * (1.0 - 2.0 / 3.0 * s2t[iz]);
            p_corr = L3 * norm2 - aliased;
        }
        p_corr *= deconv;
        const unsigned mult = (iz == 0 || (even && iz == N / 2)) ? 1u : 2u;
        const double md = static_cast<double>(mult);
        atomicAdd(&sums[bin * kFields + 0], kmag * md);
        atomicAdd(&sums[bin * kFields + 1], p_raw * md);
        atomicAdd(&sums[bin * kFields + 2], p_corr * md);
        atomicAdd(&sums[bin * kFields + 3], deconv * md);
        atomicAdd(&cnt[bin], static_cast<unsigned long long>(mult));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb * kFields; i += blockDim.x)
        partial[static_cast<size_t>(blockIdx.x) * nb * kFields + i] = sums[i];
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
        pcount[static_cast<size_t>(blockIdx.x) * nb + i] = cnt[i];
}

// Block partials combined in block order: one thread per (bin, field).
__global__ void k_bins_finish(int blocks, int nb, const double* __restrict__ partial,
                              const unsigned long long* __restrict__ pcount,
                              double* __restrict__ out, unsigned long long* __restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb * kFields) {
        double s = 0.0;
        for (int b = 0; b < blocks; ++b) s += partial[static_cast<size_t>(b) * nb * kFields + i];
        out[i] = s;
    }
    if (i < nb) {
        unsigned long long c = 0;
        for (int b = 0; b < blocks; ++b) c += pcount[static_cast<size_t>(b) * nb + i];
        count[i] = c;
    }
}

// detail::stable_positive_log_interpolate (include/cosmo_nbody/analysis/spectral_numeric.hpp:54-92).
double log_interpolate(double lower, double upper, double fraction) {
    if (fraction == 0.0 || lower == upper) return lower;
    if (fraction == 1.0) return upper;
    const double rel = (upper - lower) / lower;
    const double span = std::isfinite(rel) ? std::log1p(rel) : std::log(upper) - std::log(lower);
    if (span <= 1.0) return lower * std::exp(fraction * span);
    const long double v = std::log(static_cast<long double>(lower))
        + static_cast<long double>(fraction) * static_cast<long double>(span);
    return static_cast<double>(std::exp(v));
}

// detail::cic_window_axis_wide (include/cosmo_nbody/analysis/cic_spectral_window.hpp:13-36).
long double window_axis(double k, double dx) {
    const long double a = 0.5L * static_cast<long double>(k) * static_cast<long double>(dx);
    if (a == 0.0L) return 1.0L;
    const long double s = std::min(1.0L, std::fabs(std::sin(a) / a));
    return s * s;
}

struct Buffers {
    double* rho = nullptr;
    double2* modes = nullptr;
    double2* shifted = nullptr;
    double* pos = nullptr;      // interlacing: shifted positions (3 n)
    double* tables = nullptr;   // k, window, sin^2 (3 N) and edges (nb + 1)
    double* partial = nullptr;
    unsigned long long* pcount = nullptr;
    double* sums = nullptr;
    unsigned long long* count = nullptr;
    unsigned int* status = nullptr;
    cufftHandle plan = 0;
    bool has_plan = false;
    ~Buffers() {
        cudaFree(rho);
        cudaFree(modes);
        cudaFree(shifted);
        cudaFree(pos);
        cudaFree(tables);
        cudaFree(partial);
        cudaFree(pcount);
        cudaFree(sums);
        cudaFree(count);
        cudaFree(status);
        if (has_plan) cufftDestroy(plan);
    }
};

template <typename T>
bool dalloc(T** p, size_t count) {
    return cudaMalloc(reinterpret_cast<void**>(p), (count ? count : 1) * sizeof(T)) == cudaSuccess;
}

}  // namespace

int compute(double L, int N, uint32_t n, const double* x, const double* y, const double* z,
            const double* weights, double weight_sum, double mass_square_fraction,
            const Request& req, Bin* out, std::string* err, cudaStream_t s) {
    auto fail = [&](int code, const char* m) {
        *err = m;
        return code;
    };
    const int nb = req.num_bins;
    const double pi = 3.14159265358979323846;
    const double k_nyquist = pi * static_cast<double>(N) / L;
    const double k_max = req.max_k_fraction_nyquist * k_nyquist;
    const double k_fundamental = 2.0 * pi / L;
    if (!(k_max > k_fundamental))
        return fail(HYOWON_EINVAL, "MatterPowerSpectrum requested range contains no nonzero shell");
    const double dx = L / static_cast<double>(N);
    const uint64_t cells = static_cast<uint64_t>(N) * N * N;
    const uint64_t half = static_cast<uint64_t>(N) * N * (N / 2 + 1);

    // host tables: per-axis k, CIC window, sin^2(k dx / 2); bin edges
    std::vector<double> tab(3 * static_cast<size_t>(N) + nb + 1);
    for (int i = 0; i < N; ++i) {
        const long long mode = i <= N / 2 ? i : static_cast<long long>(i) - N;
        const double k = 2.0 * pi * static_cast<double>(mode) / L;
        const double sarg = 0.5 * k * dx;
        tab[i] = k;
        tab[N + i] = static_cast<double>(window_axis(k, dx));
        tab[2 * N + i] = std::sin(sarg) * std::sin(sarg);
    }
    for (int b = 0; b <= nb; ++b)
        tab[3 * N + b] = log_interpolate(k_fundamental, k_max,
                                         static_cast<double>(b) / static_cast<double>(nb));
    for (int b = 1; b <= nb; ++b)
        if (!(tab[3 * N + b] > tab[3 * N + b - 1]))
            return fail(HYOWON_EOVERFLOW, "Positive logarithmic bin edges are not strictly representable");

    Buffers buf;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 4;
    if (!dalloc(&buf.rho, cells) || !dalloc(&buf.modes, half) || !dalloc(&buf.tables, tab.size())
        || !dalloc(&buf.partial, static_cast<size_t>(blocks) * nb * kFields)
        || !dalloc(&buf.pcount, static_cast<size_t>(blocks) * nb)
        || !dalloc(&buf.sums, static_cast<size_t>(nb) * kFields) || !dalloc(&buf.count, nb)
        || !dalloc(&buf.status, 1)
        || (req.interlaced && (!dalloc(&buf.shifted, half) || !dalloc(&buf.pos, 3ull * n))))
        return fail(HYOWON_ENOMEM, "power spectrum: device allocation failed");
    if (cufftCreate(&buf.plan) != CUFFT_SUCCESS)
        return fail(HYOWON_ECUDA, "power spectrum: cuFFT plan creation failed");
    buf.has_plan = true;
    size_t work = 0;
    if (cufftMakePlan3d(buf.plan, N, N, N, CUFFT_D2Z, &work) != CUFFT_SUCCESS
        || cufftSetStream(buf.plan, s) != CUFFT_SUCCESS)
        return fail(HYOWON_ECUDA, "power spectrum: cuFFT plan creation failed");
    if (cudaMemcpyAsync(buf.tables, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice,
                        s) != cudaSuccess
        || cudaMemsetAsync(buf.status, 0, sizeof(unsigned int), s) != cudaSuccess)
        return fail(HYOWON_ECUDA, "power spectrum: table upload failed");

    Axis axis{};
    axis.L = L;
    axis.dx = dx;
    axis.upper = std::nextafter(static_cast<double>(N), 0.0);
    axis.N = N;
    const double mean = weight_sum / static_cast<double>(cells);
    auto build_one = [&](const double* px, const double* py, const double* pz, double2* dst) {
        if (cudaMemsetAsync(buf.rho, 0, sizeof(double) * cells, s) != cudaSuccess) return false;
        launch_deposit_f64(n, ParticlesF64{const_cast<double*>(px), const_cast<double*>(py),
                                           const_cast<double*>(pz), nullptr, nullptr, nullptr},
                           weights, 1.0, axis, buf.rho, buf.status, s);
        k_contrast<<<blocks, kThreads, 0, s>>>(cells, buf.rho, mean);
        return cufftExecD2Z(buf.plan, buf.rho, reinterpret_cast<cufftDoubleComplex*>(dst))
            == CUFFT_SUCCESS;
    };
    if (!build_one(x, y, z, buf.modes)) return fail(HYOWON_ECUDA, "power spectrum: transform failed");
    const double shift = 0.5 * dx;
    if (req.interlaced) {
        double* sx = buf.pos;
        double* sy = buf.pos + n;
        double* sz = buf.pos + 2ull * n;
        const unsigned pb = (n + kThreads - 1) / kThreads;
        k_shift_wrap<<<pb, kThreads, 0, s>>>(n, x, shift, L, sx);
        k_shift_wrap<<<pb, kThreads, 0, s>>>(n, y, shift, L, sy);
        k_shift_wrap<<<pb, kThreads, 0, s>>>(n, z, shift, L, sz);
        if (!build_one(sx, sy, sz, buf.shifted))
            return fail(HYOWON_ECUDA, "power spectrum: transform failed");
    }
    const double L3 = L * L * L;
    const double shot = L3 * mass_square_fraction;
    const size_t smem = sizeof(double) * (static_cast<size_t>(nb) * kFields + nb + nb + 1);
    k_bins<<<blocks, kThreads, smem, s>>>(N, L3, 1.0 / static_cast<double>(cells), buf.modes,
                                          req.interlaced ? buf.shifted : nullptr, shift, buf.tables,
                                          buf.tables + N, buf.tables + 2 * N, buf.tables + 3 * N,
                                          nb, k_max, shot, req.subtract_shot_noise ? 1 : 0,
                                          buf.partial, buf.pcount);
    k_bins_finish<<<(nb * kFields + 127) / 128, 128, 0, s>>>(blocks, nb, buf.partial, buf.pcount,
                                                            buf.sums, buf.count);
    std::vector<double> sums(static_cast<size_t>(nb) * kFields);
    std::vector<unsigned long long> count(nb);
    unsigned int st = 0;
    if (cudaMemcpyAsync(sums.data(), buf.sums, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost,
                        s) != cudaSuccess
        || cudaMemcpyAsync(count.data(), buf.count, sizeof(unsigned long long) * nb,
                           cudaMemcpyDeviceToHost, s) != cudaSuccess
        || cudaMemcpyAsync(&st, buf.status, sizeof(unsigned int), cudaMemcpyDeviceToHost, s)
               != cudaSuccess
        || cudaStreamSynchronize(s) != cudaSuccess)
        return fail(HYOWON_ECUDA, "power spectrum: kernel or copy failed");
    if (st & ST_CELL_ESCAPE) return fail(HYOWON_ELOGIC, "power spectrum: cell assignment escaped the mesh");
    if (st & ST_NONFINITE_INPUT) return fail(HYOWON_EINVAL, "power spectrum: non-finite particle input");
    for (int b = 0; b < nb; ++b) {
        Bin& o = out[b];
        o = Bin{};
        o.k_low = tab[3 * N + b];
        o.k_high = tab[3 * N + b + 1];
        o.shot_noise = shot;
        o.mode_count = count[b];
        if (count[b] == 0) continue;
        const double c = static_cast<double>(count[b]);
        o.k_mean = sums[b * kFields + 0] / c;
        o.p_raw = sums[b * kFields + 1] / c;
        o.p_corrected = sums[b * kFields + 2] / c;
        o.mean_deconvolution = sums[b * kFields + 3] / c;
        if (!std::isfinite(o.p_raw) || !std::isfinite(o.p_corrected))
            return fail(HYOWON_EOVERFLOW, "MatterPowerSpectrum power is not finite");
    }
    return HYOWON_OK;
}

}  // namespace pk
}  // namespace hyowon
