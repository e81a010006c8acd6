// pm_lpt.cu -- first-order LPT (Zel'dovich) initial conditions on the device.
//
// From a white-noise field w on the N_ic^3 particle lattice:
//   delta_k = r2c(w)_k * sqrt(P(|k|) N^3 / L^3)                (k != 0)
//     (the variance normalisation of src/ic/random_field.cpp:119-129 applied
//      to unit-variance noise; P already back-scaled to a_start)
//   psi_d,k = i k_d delta_k / k^2, k_d = 0 on the Nyquist plane of axis d
//     (src/ic/lpt_displacement.cpp:330-338)
//   psi_d   = c2r(psi_d,k) / N^3, sampled at the lattice node q
//   x_d = wrap(q_d + psi_d), p_d = (a^2 H f1) psi_d   (lpt_displacement.cpp:101-128)
// with q = (i, j, k) L / N_ic and particle index (i N + j) N + k
// (src/ic/initial_conditions.cpp:295-313). P(k) is a natural cubic spline in
// (ln k, ln P) (src/ic/linear_power_spectrum.cpp:649-664) whose nodes and second
// derivatives come from the host.
#include <cuda_runtime.h>
#include <cufft.h>

#include "pm_common.cuh"
#include "pm_lpt.h"

namespace hyowon {

namespace {

__device__ double spline_eval(double xq, const double* __restrict__ xs,
                              const double* __restrict__ ys, const double* __restrict__ y2,
                              int n) {
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (xs[mid] > xq) hi = mid;
        else lo = mid;
    }
    const double h = xs[hi] - xs[lo];
    const double A = (xs[hi] - xq) / h;
    const double B = (xq - xs[lo]) / h;
    return A * ys[lo] + B * ys[hi] + ((A * A * A - A) * y2[lo] + (B * B * B - B) * y2[hi]) * h * h / 6.0;
}

__device__ __forceinline__ void mode_of(uint64_t idx, int N, int& ix, int& iy, int& iz) {
    const int Hz = N / 2 + 1;
    iz = static_cast<int>(idx % Hz);
    const uint64_t t = idx / Hz;
    iy = static_cast<int>(t % N);
    ix = static_cast<int>(t / N);
}

__global__ void k_lpt_amplitude(int N, double L, double2* __restrict__ modes,
                                const double* __restrict__ xs, const double* __restrict__ ys,
                                const double* __restrict__ y2, int n_nodes, double norm,
                                unsigned int* status) {
    const uint64_t total = static_cast<uint64_t>(N) * N * (N / 2 + 1);
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    int ix, iy, iz;
    mode_of(idx, N, ix, iy, iz);
    const double kf = 2.0 * 3.141592653589793 / L;
    const int mx = ix <= N / 2 ? ix : ix - N;
    const int my = iy <= N / 2 ? iy : iy - N;
    const double kx = kf * mx, ky = kf * my, kz = kf * iz;
    const double k2 = kx * kx + ky * ky + kz * kz;
    if (k2 == 0.0) {
        modes[idx] = make_double2(0.0, 0.0);
        return;
    }
    const double lk = 0.5 * log(k2);
    if (lk < xs[0] || lk > xs[n_nodes - 1]) {
        raise_status(status, ST_NONFINITE_INPUT);  // outside the tabulated support
        modes[idx] = make_double2(0.0, 0.0);
        return;
    }
    const double P = exp(spline_eval(lk, xs, ys, y2, n_nodes));
    const double amp = sqrt(P * norm);
    double2 v = modes[idx];
    v.x *= amp;
    v.y *= amp;
    modes[idx] = v;
}

__global__ void k_lpt_psi(int N, double L, int axis, const double2* __restrict__ delta,
                          double2* __restrict__ out) {
    const uint64_t total = static_cast<uint64_t>(N) * N * (N / 2 + 1);
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    int ix, iy, iz;
    mode_of(idx, N, ix, iy, iz);
    const double kf = 2.0 * 3.141592653589793 / L;
    const int mx = ix <= N / 2 ? ix : ix - N;
    const int my = iy <= N / 2 ? iy : iy - N;
    const double kx = kf * mx, ky = kf * my, kz = kf * iz;
    const double k2 = kx * kx + ky * ky + kz * kz;
    if (k2 == 0.0) {
        out[idx] = make_double2(0.0, 0.0);
        return;
    }
    const int i = axis == 0 ? ix : (axis == 1 ? iy : iz);
    double kd = axis == 0 ? kx : (axis == 1 ? ky : kz);
    if (N % 2 == 0 && i == N / 2) kd = 0.0;
    const double f = kd / k2;
    const double2 d = delta[idx];
    out[idx] = make_double2(-d.y * f, d.x * f);
}

__global__ void k_lpt_apply(int N, double L, int axis, const double* __restrict__ psi,
                            double inv_n3, double pf, double* __restrict__ pos,
                            double* __restrict__ mom) {
    const uint64_t total = static_cast<uint64_t>(N) * N * N;
    const uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= total) return;
    const int k = static_cast<int>(p % N);
    const int j = static_cast<int>((p / N) % N);
    const int i = static_cast<int>(p / (static_cast<uint64_t>(N) * N));
    const int c = axis == 0 ? i : (axis == 1 ? j : k);
    const double q = static_cast<double>(c) * (L / static_cast<double>(N));
    const double s = psi[p] * inv_n3;
    pos[p] = wrap_f64(q + s, L);
    mom[p] = pf * s;
}

// Transpose of the displacement operator, accumulated over axes:
// acc_k (+)= i k_d T(k) / k^2 * g_k, the same symbol as k_lpt_psi.
__global__ void k_lpt_adjoint_accumulate(int N, double L, int axis, const double2* __restrict__ gk,
                                         const double* __restrict__ xs,
                                         const double* __restrict__ ys,
                                         const double* __restrict__ y2, int n_nodes, double norm,
                                         int first, double2* __restrict__ acc) {
    const uint64_t total = static_cast<uint64_t>(N) * N * (N / 2 + 1);
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    int ix, iy, iz;
    mode_of(idx, N, ix, iy, iz);
    const double kf = 2.0 * 3.141592653589793 / L;
    const int mx = ix <= N / 2 ? ix : ix - N;
    const int my = iy <= N / 2 ? iy : iy - N;
    const double kx = kf * mx, ky = kf * my, kz = kf * iz;
    const double k2 = kx * kx + ky * ky + kz * kz;
    double2 r = first ? make_double2(0.0, 0.0) : acc[idx];
    if (k2 > 0.0) {
        const double lk = 0.5 * log(k2);
        const int i = axis == 0 ? ix : (axis == 1 ? iy : iz);
        double kd = axis == 0 ? kx : (axis == 1 ? ky : kz);
        if (N % 2 == 0 && i == N / 2) kd = 0.0;
        if (lk >= xs[0] && lk <= xs[n_nodes - 1]) {
            const double amp = sqrt(exp(spline_eval(lk, xs, ys, y2, n_nodes)) * norm);
            const double f = kd / k2 * amp;
            const double2 g = gk[idx];
            r.x += -g.y * f;
            r.y += g.x * f;
        }
    }
    acc[idx] = r;
}

__global__ void k_scale(uint64_t n, const double* __restrict__ in, double s, double* __restrict__ out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i] * s;
}

}  // namespace

int lpt_adjoint_device(int N, double L, double* const d_g[3], const double* d_xs,
                       const double* d_ys, const double* d_y2, int n_nodes, double* d_grad,
                       cudaStream_t s, const char** err) {
    const size_t cells = static_cast<size_t>(N) * N * N;
    const size_t half = static_cast<size_t>(N) * N * (N / 2 + 1);
    double2* gk = nullptr;
    double2* acc = nullptr;
    double* real = nullptr;
    void* ws = nullptr;
    cufftHandle r2c = 0, c2r = 0;
    bool hr = false, hc = false;
    size_t w1 = 0, w2 = 0;
    int rc = 0;
    *err = nullptr;
    const unsigned bh = static_cast<unsigned>((half + 255) / 256);
    const unsigned bc = static_cast<unsigned>((cells + 255) / 256);
    const double norm = static_cast<double>(cells) / (L * L * L);
    if (cudaMalloc(&gk, sizeof(double2) * half) != cudaSuccess
        || cudaMalloc(&acc, sizeof(double2) * half) != cudaSuccess
        || cudaMalloc(&real, sizeof(double) * cells) != cudaSuccess) {
        *err = "LPT adjoint work arrays could not be allocated";
        rc = 7;
        goto done;
    }
    if (cufftCreate(&r2c) != CUFFT_SUCCESS || cufftCreate(&c2r) != CUFFT_SUCCESS) {
        *err = "cufftCreate failed";
        rc = 6;
        goto done;
    }
    hr = hc = true;
    cufftSetAutoAllocation(r2c, 0);
    cufftSetAutoAllocation(c2r, 0);
    if (cufftMakePlan3d(r2c, N, N, N, CUFFT_D2Z, &w1) != CUFFT_SUCCESS
        || cufftMakePlan3d(c2r, N, N, N, CUFFT_Z2D, &w2) != CUFFT_SUCCESS
        || cudaMalloc(&ws, w1 > w2 ? w1 : w2) != cudaSuccess) {
        *err = "cuFFT plan for the LPT adjoint failed";
        rc = 6;
        goto done;
    }
    cufftSetWorkArea(r2c, ws);
    cufftSetWorkArea(c2r, ws);
    cufftSetStream(r2c, s);
    cufftSetStream(c2r, s);
    for (int a = 0; a < 3; ++a) {
        // the D2Z input is copied so the caller's cotangent survives
        cudaMemcpyAsync(real, d_g[a], sizeof(double) * cells, cudaMemcpyDeviceToDevice, s);
        if (cufftExecD2Z(r2c, real, reinterpret_cast<cufftDoubleComplex*>(gk)) != CUFFT_SUCCESS) {
            *err = "LPT adjoint r2c failed";
            rc = 6;
            goto done;
        }
        k_lpt_adjoint_accumulate<<<bh, 256, 0, s>>>(N, L, a, gk, d_xs, d_ys, d_y2, n_nodes, norm,
                                                    a == 0, acc);
    }
    if (cufftExecZ2D(c2r, reinterpret_cast<cufftDoubleComplex*>(acc), real) != CUFFT_SUCCESS) {
        *err = "LPT adjoint c2r failed";
        rc = 6;
        goto done;
    }
    // grad = -(1/N^3) c2r(acc): the displacement operator is antisymmetric.
    k_scale<<<bc, 256, 0, s>>>(cells, real, -1.0 / static_cast<double>(cells), d_grad);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        *err = "LPT adjoint kernels failed";
        rc = 6;
    }
done:
    if (hr) cufftDestroy(r2c);
    if (hc) cufftDestroy(c2r);
    cudaFree(ws);
    cudaFree(gk);
    cudaFree(acc);
    cudaFree(real);
    return rc;
}

int lpt_ics_device(int N, double L, const double* d_noise, const double* d_xs,
                   const double* d_ys, const double* d_y2, int n_nodes, double pf,
                   double* const d_pos[3], double* const d_mom[3], unsigned int* d_status,
                   cudaStream_t s, const char** err) {
    const size_t cells = static_cast<size_t>(N) * N * N;
    const size_t half = static_cast<size_t>(N) * N * (N / 2 + 1);
    double2* delta = nullptr;
    double2* work = nullptr;
    double* real = nullptr;
    void* fft_ws = nullptr;
    cufftHandle r2c = 0, c2r = 0;
    bool have_r2c = false, have_c2r = false;
    int rc = 0;
    size_t ws1 = 0, ws2 = 0;
    *err = nullptr;
    if (cudaMalloc(&delta, sizeof(double2) * half) != cudaSuccess
        || cudaMalloc(&work, sizeof(double2) * half) != cudaSuccess
        || cudaMalloc(&real, sizeof(double) * cells) != cudaSuccess) {
        *err = "LPT work arrays could not be allocated";
        rc = 7;
        goto done;
    }
    if (cufftCreate(&r2c) != CUFFT_SUCCESS || cufftCreate(&c2r) != CUFFT_SUCCESS) {
        *err = "cufftCreate failed";
        rc = 6;
        goto done;
    }
    have_r2c = have_c2r = true;
    cufftSetAutoAllocation(r2c, 0);
    cufftSetAutoAllocation(c2r, 0);
    if (cufftMakePlan3d(r2c, N, N, N, CUFFT_D2Z, &ws1) != CUFFT_SUCCESS
        || cufftMakePlan3d(c2r, N, N, N, CUFFT_Z2D, &ws2) != CUFFT_SUCCESS) {
        *err = "cuFFT plan for the IC mesh failed";
        rc = 6;
        goto done;
    }
    if (cudaMalloc(&fft_ws, ws1 > ws2 ? ws1 : ws2) != cudaSuccess) {
        *err = "cuFFT workspace could not be allocated";
        rc = 7;
        goto done;
    }
    cufftSetWorkArea(r2c, fft_ws);
    cufftSetWorkArea(c2r, fft_ws);
    cufftSetStream(r2c, s);
    cufftSetStream(c2r, s);
    {
        const unsigned bh = static_cast<unsigned>((half + 255) / 256);
        const unsigned bc = static_cast<unsigned>((cells + 255) / 256);
        const double norm = static_cast<double>(cells) / (L * L * L);
        const double inv_n3 = 1.0 / (static_cast<double>(N) * N * N);
        if (cufftExecD2Z(r2c, const_cast<double*>(d_noise),
                         reinterpret_cast<cufftDoubleComplex*>(delta)) != CUFFT_SUCCESS) {
            *err = "IC r2c failed";
            rc = 6;
            goto done;
        }
        k_lpt_amplitude<<<bh, 256, 0, s>>>(N, L, delta, d_xs, d_ys, d_y2, n_nodes, norm, d_status);
        for (int a = 0; a < 3; ++a) {
            k_lpt_psi<<<bh, 256, 0, s>>>(N, L, a, delta, work);
            if (cufftExecZ2D(c2r, reinterpret_cast<cufftDoubleComplex*>(work), real) != CUFFT_SUCCESS) {
                *err = "IC c2r failed";
                rc = 6;
                goto done;
            }
            k_lpt_apply<<<bc, 256, 0, s>>>(N, L, a, real, inv_n3, pf, d_pos[a], d_mom[a]);
        }
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            *err = "LPT kernels failed";
            rc = 6;
        }
    }
done:
    if (have_r2c) cufftDestroy(r2c);
    if (have_c2r) cufftDestroy(c2r);
    cudaFree(fft_ws);
    cudaFree(delta);
    cudaFree(work);
    cudaFree(real);
    return rc;
}

}  // namespace hyowon
