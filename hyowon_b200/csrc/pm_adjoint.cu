// pm_adjoint.cu -- the differentiation form: gradient of a density-field loss
// with respect to the initial white noise, through 1LPT and the KDK PM step.
//
// Forward model (positions binary64 in both precisions; momenta, forces,
// meshes and FFTs in Real = double or float):
//   x0, p0 = 1LPT(w);  a_k = F(x_k)
//   p' = p_k + K1_k a_k;  x_{k+1} = wrap(x_k + D_k p');  p_{k+1} = p' + K2_k a_{k+1}
//   F(x) = gather_-grad( A deposit(x) ),  A = (1/dx^3) c2r(G(k) r2c(.))/N^3
//   L = 1/2 sum_c (delta_c - t_c)^2,  delta_c = M_c / Mbar - 1 on the PM mesh.
//
// Reverse pass ("reverse leapfrog"): KDK is time reversible, so the state of
// step k is reconstructed from step k+1 (x_k = x_{k+1} - D p', p' = p_{k+1} -
// K2 a_{k+1}, p_k = p' - K1 a_k) with one force solve per step; the stored
// (x, p) checkpoints every `ckpt_every` steps replace the reconstruction and
// bound its round-off drift. Cotangents (binary64):
//   lx += VJP_F(x_{k+1}; (K2_k + K1_{k+1}) lp)   (the two kicks that use
//         a_{k+1} share one VJP)
//   lp += D_k lx
// and a final VJP_F(x_0; K1_0 lp). The force VJP for a per-particle cotangent v:
//   u_d = CIC scatter of v_d            (transpose of the interpolation)
//   s   = sum_d D_d u_d                 (transpose of -grad: centred divergence)
//   psi = A s                           (A is real, even, hence symmetric)
//   d(v.F)/dx_j = sum_c dW_jc/dx_j (m psi_c + v_j . g_c),  g = -grad(phi(x))
// with the CIC weight derivative of the particle's own base cell (the one-sided
// convention of src/mesh/mass_assignment_directional.cpp:133-166). The
// 1LPT adjoint is dL/dw = -sum_d B_d (lx_d + pf lp_d) (pm_lpt.cu).
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "hyowon_adjoint.h"
#include "hyowon_pm.h"
#include "pm_common.cuh"
#include "pm_lpt.h"
#include "pm_adjoint.h"
#include "pm_poisson.h"

namespace hyowon::adj {

namespace {

constexpr int kT = 256;
inline unsigned nb(uint64_t n) { return static_cast<unsigned>((n + kT - 1) / kT); }

template <typename R>
struct FFTTypes;
template <>
struct FFTTypes<double> {
    using C = double2;
    static constexpr cufftType R2C = CUFFT_D2Z;
    static constexpr cufftType C2R = CUFFT_Z2D;
    static cufftResult fwd(cufftHandle p, double* in, double2* out) {
        return cufftExecD2Z(p, in, reinterpret_cast<cufftDoubleComplex*>(out));
    }
    static cufftResult inv(cufftHandle p, double2* in, double* out) {
        return cufftExecZ2D(p, reinterpret_cast<cufftDoubleComplex*>(in), out);
    }
};
template <>
struct FFTTypes<float> {
    using C = float2;
    static constexpr cufftType R2C = CUFFT_R2C;
    static constexpr cufftType C2R = CUFFT_C2R;
    static cufftResult fwd(cufftHandle p, float* in, float2* out) {
        return cufftExecR2C(p, in, reinterpret_cast<cufftComplex*>(out));
    }
    static cufftResult inv(cufftHandle p, float2* in, float* out) {
        return cufftExecC2R(p, reinterpret_cast<cufftComplex*>(in), out);
    }
};

struct Corner {
    int ix, iy, iz;
    double fx, fy, fz;
};

__device__ __forceinline__ bool corner_of(double x, double y, double z, const Axis& a, Corner& c) {
    return cic_coord_f64(x, a, c.ix, c.fx) & cic_coord_f64(y, a, c.iy, c.fy)
        & cic_coord_f64(z, a, c.iz, c.fz);
}

__device__ __forceinline__ size_t cidx(int x, int y, int z, int N) {
    return (static_cast<size_t>(x) * N + y) * N + z;
}

__device__ __forceinline__ int up(int i, int N) { return i + 1 == N ? 0 : i + 1; }
__device__ __forceinline__ int dn(int i, int N) { return i == 0 ? N - 1 : i - 1; }

template <typename R>
__global__ void k_deposit(uint32_t n, const double* __restrict__ x, const double* __restrict__ y,
                          const double* __restrict__ z, R m, Axis a, R* __restrict__ mesh,
                          unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Corner c;
    if (!corner_of(x[i], y[i], z[i], a, c)) {
        raise_status(status, ST_CELL_ESCAPE);
        return;
    }
    const int N = a.N;
    const R wx[2] = {R(1) - R(c.fx), R(c.fx)}, wy[2] = {R(1) - R(c.fy), R(c.fy)},
            wz[2] = {R(1) - R(c.fz), R(c.fz)};
    const int gx[2] = {c.ix, up(c.ix, N)}, gy[2] = {c.iy, up(c.iy, N)}, gz[2] = {c.iz, up(c.iz, N)};
    for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v)
            for (int w = 0; w < 2; ++w)
                atomicAdd(&mesh[cidx(gx[u], gy[v], gz[w], N)], m * wx[u] * wy[v] * wz[w]);
}

// Three-component CIC scatter (transpose of the interpolation). Particles
// stay in lattice order, so consecutive lanes usually hold z-neighbours in the
// same (x, y) cell column: when lane l+1's lower z cells are lane l's upper z
// cells, lane l hands its upper-z weights to lane l+1, which adds them to its
// own before the atomics (half the atomics for a matched pair; the sum is
// the same up to the order of additions, which atomics leave open anyway).
template <typename R>
__global__ void k_scatter3(uint32_t n, const double* __restrict__ x, const double* __restrict__ y,
                           const double* __restrict__ z, const R* __restrict__ v0,
                           const R* __restrict__ v1, const R* __restrict__ v2, Axis a,
                           R* __restrict__ u0, R* __restrict__ u1, R* __restrict__ u2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int N = a.N;
    Corner c{};
    const bool ok = i < n && corner_of(x[i], y[i], z[i], a, c);
    // contributions lo[u][v][d] (z cell iz) and hi[u][v][d] (z cell iz + 1)
    R lo[2][2][3], hi[2][2][3];
    int gx[2] = {0, 0}, gy[2] = {0, 0}, gz[2] = {0, 0};
    if (ok) {
        const R wx[2] = {R(1) - R(c.fx), R(c.fx)}, wy[2] = {R(1) - R(c.fy), R(c.fy)},
                wz[2] = {R(1) - R(c.fz), R(c.fz)};
        gx[0] = c.ix; gx[1] = up(c.ix, N);
        gy[0] = c.iy; gy[1] = up(c.iy, N);
        gz[0] = c.iz; gz[1] = up(c.iz, N);
        const R av[3] = {v0[i], v1[i], v2[i]};
        for (int u = 0; u < 2; ++u)
            for (int v = 0; v < 2; ++v)
                for (int d = 0; d < 3; ++d) {
                    lo[u][v][d] = wx[u] * wy[v] * wz[0] * av[d];
                    hi[u][v][d] = wx[u] * wy[v] * wz[1] * av[d];
                }
    } else {
        for (int u = 0; u < 2; ++u)
            for (int v = 0; v < 2; ++v)
                for (int d = 0; d < 3; ++d) lo[u][v][d] = hi[u][v][d] = R(0);
    }
    // the cell column and upper z cell of the lane below
    const int col = ok ? c.ix * N + c.iy : -1;
    const int col_below = __shfl_up_sync(0xffffffffu, col, 1);
    const int ztop_below = __shfl_up_sync(0xffffffffu, gz[1], 1);
    const bool take = lane > 0 && ok && col_below == col && ztop_below == gz[0];
    for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v)
            for (int d = 0; d < 3; ++d) {
                const R h = __shfl_up_sync(0xffffffffu, hi[u][v][d], 1);
                if (take) lo[u][v][d] += h;
            }
    // whether the lane above took this lane's upper weights
    const bool given = __shfl_down_sync(0xffffffffu, take ? 1 : 0, 1) != 0 && lane < 31;
    if (!ok) return;
    for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v) {
            const size_t k0 = cidx(gx[u], gy[v], gz[0], N);
            atomicAdd(&u0[k0], lo[u][v][0]);
            atomicAdd(&u1[k0], lo[u][v][1]);
            atomicAdd(&u2[k0], lo[u][v][2]);
            if (!given) {
                const size_t k1 = cidx(gx[u], gy[v], gz[1], N);
                atomicAdd(&u0[k1], hi[u][v][0]);
                atomicAdd(&u1[k1], hi[u][v][1]);
                atomicAdd(&u2[k1], hi[u][v][2]);
            }
        }
}

// s = sum_d (u_d[c+e_d] - u_d[c-e_d]) / (2 dx)
template <typename R>
__global__ void k_divergence(int N, const R* __restrict__ u0, const R* __restrict__ u1,
                             const R* __restrict__ u2, R inv_two_dx, R* __restrict__ s) {
    const uint64_t cells = static_cast<uint64_t>(N) * N * N;
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    const int z = static_cast<int>(i % N);
    const int y = static_cast<int>((i / N) % N);
    const int x = static_cast<int>(i / (static_cast<uint64_t>(N) * N));
    s[i] = ((u0[cidx(up(x, N), y, z, N)] - u0[cidx(dn(x, N), y, z, N)])
            + (u1[cidx(x, up(y, N), z, N)] - u1[cidx(x, dn(y, N), z, N)])
            + (u2[cidx(x, y, up(z, N), N)] - u2[cidx(x, y, dn(z, N), N)]))
        * inv_two_dx;
}

template <typename R, typename C>
__global__ void k_green(int N, C* __restrict__ modes, const R* __restrict__ lap, R c) {
    const int Hz = N / 2 + 1;
    const uint64_t total = static_cast<uint64_t>(N) * N * Hz;
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    if (idx == 0) {
        modes[0].x = R(0);
        modes[0].y = R(0);
        return;
    }
    const int iz = static_cast<int>(idx % Hz);
    const uint64_t t = idx / Hz;
    const int iy = static_cast<int>(t % N);
    const int ix = static_cast<int>(t / N);
    const R f = c / (lap[ix] + lap[iy] + lap[iz]);
    C v = modes[idx];
    v.x *= f;
    v.y *= f;
    modes[idx] = v;
}

// Loads the 4x4x4 stencil footprint of a particle's 8 corners and returns the
// centred-difference force g = -grad(phi) at each corner.
template <typename R>
__device__ __forceinline__ void corner_forces(const R* __restrict__ phi, const Corner& c, int N,
                                              R inv_two_dx, R g[2][2][2][3]) {
    const int xs[4] = {dn(c.ix, N), c.ix, up(c.ix, N), up(up(c.ix, N), N)};
    const int ys[4] = {dn(c.iy, N), c.iy, up(c.iy, N), up(up(c.iy, N), N)};
    const int zs[4] = {dn(c.iz, N), c.iz, up(c.iz, N), up(up(c.iz, N), N)};
    for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v)
            for (int w = 0; w < 2; ++w) {
                const int X = u + 1, Y = v + 1, Z = w + 1;
                g[u][v][w][0] = -(phi[cidx(xs[X + 1], ys[Y], zs[Z], N)] - phi[cidx(xs[X - 1], ys[Y], zs[Z], N)]) * inv_two_dx;
                g[u][v][w][1] = -(phi[cidx(xs[X], ys[Y + 1], zs[Z], N)] - phi[cidx(xs[X], ys[Y - 1], zs[Z], N)]) * inv_two_dx;
                g[u][v][w][2] = -(phi[cidx(xs[X], ys[Y], zs[Z + 1], N)] - phi[cidx(xs[X], ys[Y], zs[Z - 1], N)]) * inv_two_dx;
            }
}

// CIC-interpolated centred-gradient force at one position; false (nothing
// written) where the cell assignment fails.
template <typename R>
__device__ __forceinline__ bool force_at(double px, double py, double pz, const R* __restrict__ phi,
                                         const Axis& a, R inv_two_dx, R& s0, R& s1, R& s2) {
    Corner c;
    if (!corner_of(px, py, pz, a, c)) return false;
    R g[2][2][2][3];
    corner_forces(phi, c, a.N, inv_two_dx, g);
    const R wx[2] = {R(1) - R(c.fx), R(c.fx)}, wy[2] = {R(1) - R(c.fy), R(c.fy)},
            wz[2] = {R(1) - R(c.fz), R(c.fz)};
    s0 = s1 = s2 = 0;
    for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v)
            for (int w = 0; w < 2; ++w) {
                const R W = wx[u] * wy[v] * wz[w];
                s0 += W * g[u][v][w][0];
                s1 += W * g[u][v][w][1];
                s2 += W * g[u][v][w][2];
            }
    return true;
}

// One step of the reverse leapfrog between re-solves: x = wrap(x - D p_half),
// a = F(x) from the potential the forward pass kept for that state,
// p = p_half - K1 a (the inverse of kick K1 + drift D).
template <typename R>
__global__ void k_unstep(uint32_t n, double* __restrict__ x0, double* __restrict__ x1,
                         double* __restrict__ x2, R* __restrict__ p0, R* __restrict__ p1,
                         R* __restrict__ p2, double D, double L, const R* __restrict__ phi, Axis a,
                         R inv_two_dx, R K1, R* __restrict__ ax, R* __restrict__ ay,
                         R* __restrict__ az) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const R q0 = p0[i], q1 = p1[i], q2 = p2[i];
    const double nx = wrap_f64(x0[i] + D * static_cast<double>(q0), L);
    const double ny = wrap_f64(x1[i] + D * static_cast<double>(q1), L);
    const double nz = wrap_f64(x2[i] + D * static_cast<double>(q2), L);
    x0[i] = nx;
    x1[i] = ny;
    x2[i] = nz;
    R s0, s1, s2;
    if (!force_at(nx, ny, nz, phi, a, inv_two_dx, s0, s1, s2)) return;
    ax[i] = s0;
    ay[i] = s1;
    az[i] = s2;
    p0[i] = q0 + K1 * s0;
    p1[i] = q1 + K1 * s1;
    p2[i] = q2 + K1 * s2;
}

// lp += D lx (the drift's transpose) and p += K a (a kick), one pass.
template <typename R>
__global__ void k_axpy3_kick(uint32_t n, double D, const double* __restrict__ x0,
                             const double* __restrict__ x1, const double* __restrict__ x2,
                             double* __restrict__ y0, double* __restrict__ y1,
                             double* __restrict__ y2, R* __restrict__ p0, R* __restrict__ p1,
                             R* __restrict__ p2, const R* __restrict__ a0,
                             const R* __restrict__ a1, const R* __restrict__ a2, R K) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    y0[i] += D * x0[i];
    y1[i] += D * x1[i];
    y2[i] += D * x2[i];
    p0[i] += K * a0[i];
    p1[i] += K * a1[i];
    p2[i] += K * a2[i];
}

template <typename R>
__global__ void k_force(uint32_t n, const double* __restrict__ x, const double* __restrict__ y,
                        const double* __restrict__ z, const R* __restrict__ phi, Axis a,
                        R inv_two_dx, R* __restrict__ ax, R* __restrict__ ay, R* __restrict__ az) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Corner c;
    if (!corner_of(x[i], y[i], z[i], a, c)) return;
    R g[2][2][2][3];
    corner_forces(phi, c, a.N, inv_two_dx, g);
    const R wx[2] = {R(1) - R(c.fx), R(c.fx)}, wy[2] = {R(1) - R(c.fy), R(c.fy)},
            wz[2] = {R(1) - R(c.fz), R(c.fz)};
    R s0 = 0, s1 = 0, s2 = 0;
    for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v)
            for (int w = 0; w < 2; ++w) {
                const R W = wx[u] * wy[v] * wz[w];
                s0 += W * g[u][v][w][0];
                s1 += W * g[u][v][w][1];
                s2 += W * g[u][v][w][2];
            }
    ax[i] = s0;
    ay[i] = s1;
    az[i] = s2;
}

// out_j += sum_c dW_jc/dx_j (mpsi * psi_c + v_j . g_c)   (phi / v may be null)
template <typename R>
__global__ void k_vjp_gather(uint32_t n, const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, const R* __restrict__ psi, R mpsi,
                             const R* __restrict__ phi, const R* __restrict__ v0,
                             const R* __restrict__ v1, const R* __restrict__ v2, Axis a,
                             R inv_two_dx, double* __restrict__ o0, double* __restrict__ o1,
                             double* __restrict__ o2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Corner c;
    if (!corner_of(x[i], y[i], z[i], a, c)) return;
    const int N = a.N;
    R g[2][2][2][3];
    const bool with_v = phi != nullptr;
    if (with_v) corner_forces(phi, c, N, inv_two_dx, g);
    const R vv[3] = {with_v ? v0[i] : R(0), with_v ? v1[i] : R(0), with_v ? v2[i] : R(0)};
    const R inv_dx = R(2) * inv_two_dx;
    const R wx[2] = {R(1) - R(c.fx), R(c.fx)}, wy[2] = {R(1) - R(c.fy), R(c.fy)},
            wz[2] = {R(1) - R(c.fz), R(c.fz)};
    const R dw[2] = {-inv_dx, inv_dx};
    const int gx[2] = {c.ix, up(c.ix, N)}, gy[2] = {c.iy, up(c.iy, N)}, gz[2] = {c.iz, up(c.iz, N)};
    R s0 = 0, s1 = 0, s2 = 0;
    for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v)
            for (int w = 0; w < 2; ++w) {
                R h = psi ? mpsi * psi[cidx(gx[u], gy[v], gz[w], N)] : R(0);
                if (with_v) h += vv[0] * g[u][v][w][0] + vv[1] * g[u][v][w][1] + vv[2] * g[u][v][w][2];
                s0 += dw[u] * wy[v] * wz[w] * h;
                s1 += wx[u] * dw[v] * wz[w] * h;
                s2 += wx[u] * wy[v] * dw[w] * h;
            }
    o0[i] += static_cast<double>(s0);
    o1[i] += static_cast<double>(s1);
    o2[i] += static_cast<double>(s2);
}

template <typename R>
__global__ void k_kick(uint32_t n, R* __restrict__ p0, R* __restrict__ p1, R* __restrict__ p2,
                       const R* __restrict__ a0, const R* __restrict__ a1,
                       const R* __restrict__ a2, R K) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    p0[i] += K * a0[i];
    p1[i] += K * a1[i];
    p2[i] += K * a2[i];
}

template <typename R>
__global__ void k_drift(uint32_t n, double* __restrict__ x0, double* __restrict__ x1,
                        double* __restrict__ x2, const R* __restrict__ p0, const R* __restrict__ p1,
                        const R* __restrict__ p2, double D, double L) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x0[i] = wrap_f64(x0[i] + D * static_cast<double>(p0[i]), L);
    x1[i] = wrap_f64(x1[i] + D * static_cast<double>(p1[i]), L);
    x2[i] = wrap_f64(x2[i] + D * static_cast<double>(p2[i]), L);
}

// v = coef * lp (as Real) ; lp += D * lx
template <typename R>
__global__ void k_cotangent(uint32_t n, const double* __restrict__ l0, const double* __restrict__ l1,
                            const double* __restrict__ l2, double coef, R* __restrict__ v0,
                            R* __restrict__ v1, R* __restrict__ v2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    v0[i] = static_cast<R>(coef * l0[i]);
    v1[i] = static_cast<R>(coef * l1[i]);
    v2[i] = static_cast<R>(coef * l2[i]);
}

__global__ void k_axpy3(uint32_t n, double a, const double* __restrict__ x0,
                        const double* __restrict__ x1, const double* __restrict__ x2,
                        double* __restrict__ y0, double* __restrict__ y1, double* __restrict__ y2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    y0[i] += a * x0[i];
    y1[i] += a * x1[i];
    y2[i] += a * x2[i];
}

template <typename R>
__global__ void k_from_double(uint32_t n, const double* __restrict__ in, R* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<R>(in[i]);
}

// delta = M / Mbar - 1; residual field r = (delta - t) * m / Mbar; loss += 1/2 (delta-t)^2
template <typename R>
__global__ void k_loss(uint64_t cells, const R* __restrict__ mesh, const double* __restrict__ target,
                       double inv_mbar, double m_over_mbar, R* __restrict__ field,
                       double* __restrict__ delta_out, double* loss) {
    double local = 0.0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < cells;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double delta = static_cast<double>(mesh[i]) * inv_mbar - 1.0;
        if (delta_out) delta_out[i] = delta;
        const double r = target ? delta - target[i] : 0.0;
        local += 0.5 * r * r;
        if (field) field[i] = static_cast<R>(r * m_over_mbar);
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, local);
}

struct Fail {
    int code;
    std::string msg;
};

#define ACK(call)                                                              \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) throw Fail{e_ == cudaErrorMemoryAllocation ? 7 : 6, \
                                          std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)
#define AFFT(call)                                                            \
    do {                                                                      \
        if ((call) != CUFFT_SUCCESS) throw Fail{6, std::string(#call)};       \
    } while (0)

template <typename T>
T* dmalloc(size_t count, std::vector<void*>& owned) {
    void* p = nullptr;
    ACK(cudaMalloc(&p, (count ? count : 1) * sizeof(T)));
    owned.push_back(p);
    return static_cast<T*>(p);
}

template <typename R>
class Engine {
public:
    using C = typename FFTTypes<R>::C;

    Engine(const VjpConfig& cfg, cudaStream_t s) : cfg_(cfg), s_(s) {
        N_ = static_cast<int>(cfg.mesh_size);
        n_ = static_cast<uint32_t>(cfg.n_side * cfg.n_side * cfg.n_side);
        cells_ = static_cast<uint64_t>(N_) * N_ * N_;
        half_ = static_cast<uint64_t>(N_) * N_ * (N_ / 2 + 1);
        axis_.L = cfg.box_size;
        axis_.dx = cfg.box_size / static_cast<double>(N_);
        axis_.upper = std::nextafter(static_cast<double>(N_), 0.0);
        axis_.N = N_;
        inv_two_dx_ = static_cast<R>(1.0 / (2.0 * axis_.dx));
        const double pi = 3.14159265358979323846;
        const double G = 6.67430e-11 * (1e10 * 1.98847e30) / (3.085677581491367e22 * 1000.0 * 1000.0);
        const double dx = axis_.dx;
        // Mass mesh in mass units; A = (4 pi G / dx^3) / N^3 G(k) with the
        // 1/N^3 of the inverse transform folded in (mean removed at k = 0).
        c_green_ = static_cast<R>(4.0 * pi * G / (dx * dx * dx) / static_cast<double>(cells_));
        std::vector<R> lap(N_);
        for (int i = 0; i < N_; ++i) {
            const long long mode = i <= N_ / 2 ? i : static_cast<long long>(i) - N_;
            const double sn = std::sin(pi * static_cast<double>(mode) / N_);
            lap[i] = static_cast<R>(-4.0 / (dx * dx) * sn * sn);
        }
        lap_ = dmalloc<R>(N_, owned_);
        ACK(cudaMemcpy(lap_, lap.data(), sizeof(R) * N_, cudaMemcpyHostToDevice));
        four_pi_G_ = 4.0 * pi * G;
        scale_ = 1.0 / (dx * dx * dx) / static_cast<double>(cells_);
        five_ = poisson::supported(N_);
        if (five_) {
            // the production five-pass solve: own transforms with the Green's
            // multiply fused into the x pass (chunked half spectrum)
            const size_t elems = sizeof(R) == 8 ? poisson::modes_elements_f64(N_)
                                                : poisson::modes_elements_f32(N_);
            modes_ = dmalloc<C>(elems, owned_);
            const char* perr = nullptr;
            plan_ = poisson::create_plan(N_, sizeof(R) == 4, modes_, &perr);
            if (!plan_) throw Fail{HYOWON_ECUDA, perr ? perr : "five-pass plan"};
            std::vector<double> t(2 * static_cast<size_t>(N_));
            poisson::twiddles(N_, t.data());
            std::vector<C> tc(N_);
            for (int i = 0; i < N_; ++i) {
                tc[i].x = static_cast<R>(t[2 * i]);
                tc[i].y = static_cast<R>(t[2 * i + 1]);
            }
            tw_ = dmalloc<C>(N_, owned_);
            ACK(cudaMemcpy(tw_, tc.data(), sizeof(C) * N_, cudaMemcpyHostToDevice));
            c_green_dev_ = dmalloc<R>(1, owned_);
            ACK(cudaMemcpy(c_green_dev_, &c_green_, sizeof(R), cudaMemcpyHostToDevice));
        } else {
            AFFT(cufftCreate(&r2c_));
            AFFT(cufftCreate(&c2r_));
            plans_ = true;
            cufftSetAutoAllocation(r2c_, 0);
            cufftSetAutoAllocation(c2r_, 0);
            size_t w1 = 0, w2 = 0;
            AFFT(cufftMakePlan3d(r2c_, N_, N_, N_, FFTTypes<R>::R2C, &w1));
            AFFT(cufftMakePlan3d(c2r_, N_, N_, N_, FFTTypes<R>::C2R, &w2));
            void* ws = dmalloc<char>(w1 > w2 ? w1 : w2, owned_);
            cufftSetWorkArea(r2c_, ws);
            cufftSetWorkArea(c2r_, ws);
            cufftSetStream(r2c_, s_);
            cufftSetStream(c2r_, s_);
            modes_ = dmalloc<C>(half_, owned_);
        }
        mesh_ = dmalloc<R>(cells_, owned_);
        phi_own_ = dmalloc<R>(cells_, owned_);
        phi_ = phi_own_;
        status_ = dmalloc<unsigned int>(1, owned_);
        ACK(cudaMemsetAsync(status_, 0, sizeof(unsigned int), s_));
        for (int a = 0; a < 3; ++a) {
            x_[a] = dmalloc<double>(n_, owned_);
            p_[a] = dmalloc<R>(n_, owned_);
            acc_[a] = dmalloc<R>(n_, owned_);
        }
    }

    // A later call with the same geometry (box, mesh, lattice, form) reuses the
    // engine: its plans and work arrays; the rest of the configuration (P(k)
    // table, schedule, masses, checkpoints) is the call's own.
    bool same_geometry(const VjpConfig& c) const {
        return c.box_size == cfg_.box_size && c.mesh_size == cfg_.mesh_size
            && c.n_side == cfg_.n_side && c.precision == cfg_.precision;
    }
    void set_config(const VjpConfig& c) { cfg_ = c; }

    ~Engine() {
        poisson::destroy_plan(plan_);
        if (plans_) {
            cufftDestroy(r2c_);
            cufftDestroy(c2r_);
        }
        for (void* p : owned_) cudaFree(p);
    }

    // acc = F(x); phi_ = potential at x, written to `keep` when given (the
    // forward pass's copy of it), else to the engine's own mesh.
    void force(R* keep = nullptr) {
        phi_ = keep ? keep : phi_own_;
        ACK(cudaMemsetAsync(mesh_, 0, sizeof(R) * cells_, s_));
        k_deposit<R><<<nb(n_), kT, 0, s_>>>(n_, x_[0], x_[1], x_[2], static_cast<R>(cfg_.particle_mass),
                                            axis_, mesh_, status_);
        apply_green(mesh_, phi_);
        k_force<R><<<nb(n_), kT, 0, s_>>>(n_, x_[0], x_[1], x_[2], phi_, axis_, inv_two_dx_, acc_[0],
                                          acc_[1], acc_[2]);
        ++solves_;
    }

    // acc = F(x) from a potential the forward pass kept for this state.
    void force_from(R* kept) {
        phi_ = kept;
        k_force<R><<<nb(n_), kT, 0, s_>>>(n_, x_[0], x_[1], x_[2], phi_, axis_, inv_two_dx_, acc_[0],
                                          acc_[1], acc_[2]);
    }

    // out = A in: r2c, Green's function (k = 0 zeroed), c2r with 1/N^3. On
    // power-of-two meshes the production five-pass solve (Green's multiply
    // inside the x pass; A is self-adjoint, so the adjoint uses it as is);
    // elsewhere cuFFT with a separate multiply.
    void apply_green(R* in, R* out) {
        if (five_) {
            int k = 0;
            if constexpr (sizeof(R) == 8) {
                // no mass check here: the source is a mass mesh or a divergence
                const poisson::GreenF64 g{lap_, nullptr, four_pi_G_, scale_, 0, 0.0, INFINITY,
                                          status_};
                k = poisson::forward_f64(plan_, N_, in, modes_, tw_, status_, s_) < 0
                        || poisson::green_f64(plan_, N_, modes_, tw_, g, s_) < 0
                        || poisson::inverse_f64(plan_, N_, modes_, out, tw_, status_, s_) < 0;
            } else {
                const poisson::GreenF32 g{lap_, nullptr, 0, c_green_dev_};
                k = poisson::forward_f32(plan_, N_, in, modes_, tw_, status_, s_) < 0
                        || poisson::green_f32(plan_, N_, modes_, tw_, g, status_, s_) < 0
                        || poisson::inverse_f32(plan_, N_, modes_, out, tw_, status_, s_) < 0;
            }
            if (k) throw Fail{HYOWON_ECUDA, "potential solve launch failed"};
            return;
        }
        AFFT(FFTTypes<R>::fwd(r2c_, in, modes_));
        k_green<R, C><<<nb(half_), kT, 0, s_>>>(N_, modes_, lap_, c_green_);
        AFFT(FFTTypes<R>::inv(c2r_, modes_, out));
    }

    void kick(double K) {
        k_kick<R><<<nb(n_), kT, 0, s_>>>(n_, p_[0], p_[1], p_[2], acc_[0], acc_[1], acc_[2],
                                         static_cast<R>(K));
    }

    void drift(double D) {
        k_drift<R><<<nb(n_), kT, 0, s_>>>(n_, x_[0], x_[1], x_[2], p_[0], p_[1], p_[2], D, cfg_.box_size);
    }

    // lx += VJP_F(x; v), v = coef * lp
    void vjp(double coef, double* const lx[3], double* const lp[3], R* const v[3], R* const u[3], R* psi) {
        k_cotangent<R><<<nb(n_), kT, 0, s_>>>(n_, lp[0], lp[1], lp[2], coef, v[0], v[1], v[2]);
        for (int a = 0; a < 3; ++a) ACK(cudaMemsetAsync(u[a], 0, sizeof(R) * cells_, s_));
        k_scatter3<R><<<nb(n_), kT, 0, s_>>>(n_, x_[0], x_[1], x_[2], v[0], v[1], v[2], axis_, u[0],
                                             u[1], u[2]);
        k_divergence<R><<<nb(cells_), kT, 0, s_>>>(N_, u[0], u[1], u[2], inv_two_dx_, mesh_);
        apply_green(mesh_, psi);
        k_vjp_gather<R><<<nb(n_), kT, 0, s_>>>(n_, x_[0], x_[1], x_[2], psi,
                                               static_cast<R>(cfg_.particle_mass), phi_, v[0], v[1],
                                               v[2], axis_, inv_two_dx_, lx[0], lx[1], lx[2]);
        ++vjps_;
    }

    void run(const double* noise, const double* target, double* loss_out, double* grad_out,
             double* delta_out, double* timings) {
        const uint64_t S = cfg_.n_steps;
        const uint64_t k = cfg_.ckpt_every > 0 ? cfg_.ckpt_every : 1;
        std::vector<void*> tmp;
        cudaEvent_t e0, e1, e2;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventCreate(&e2);
        // ---- 1LPT ---------------------------------------------------------
        double* d_noise = dmalloc<double>(n_, tmp);
        double* tab = dmalloc<double>(3 * cfg_.n_nodes, tmp);
        double* pd[3];
        for (int a = 0; a < 3; ++a) pd[a] = dmalloc<double>(n_, tmp);
        ACK(cudaMemcpy(d_noise, noise, sizeof(double) * n_, cudaMemcpyHostToDevice));
        ACK(cudaMemcpy(tab, cfg_.ln_k, sizeof(double) * cfg_.n_nodes, cudaMemcpyHostToDevice));
        ACK(cudaMemcpy(tab + cfg_.n_nodes, cfg_.ln_p, sizeof(double) * cfg_.n_nodes, cudaMemcpyHostToDevice));
        ACK(cudaMemcpy(tab + 2 * cfg_.n_nodes, cfg_.ln_p_y2, sizeof(double) * cfg_.n_nodes, cudaMemcpyHostToDevice));
        const char* err = nullptr;
        const int lrc = lpt_ics_device(static_cast<int>(cfg_.n_side), cfg_.box_size, d_noise, tab,
                                       tab + cfg_.n_nodes, tab + 2 * cfg_.n_nodes,
                                       static_cast<int>(cfg_.n_nodes), cfg_.momentum_factor, x_, pd,
                                       status_, s_, &err);
        if (lrc) throw Fail{lrc, err ? err : "LPT failed"};
        for (int a = 0; a < 3; ++a) k_from_double<R><<<nb(n_), kT, 0, s_>>>(n_, pd[a], p_[a]);
        // ---- forward with checkpoints -------------------------------------
        const uint64_t n_ckpt = (S + k - 1) / k + 1;
        std::vector<double*> cx(3 * n_ckpt);
        std::vector<R*> cp(3 * n_ckpt);
        for (uint64_t c = 0; c < n_ckpt; ++c)
            for (int a = 0; a < 3; ++a) {
                cx[3 * c + a] = dmalloc<double>(n_, tmp);
                cp[3 * c + a] = dmalloc<R>(n_, tmp);
            }
        auto save = [&](uint64_t c) {
            for (int a = 0; a < 3; ++a) {
                ACK(cudaMemcpyAsync(cx[3 * c + a], x_[a], sizeof(double) * n_, cudaMemcpyDeviceToDevice, s_));
                ACK(cudaMemcpyAsync(cp[3 * c + a], p_[a], sizeof(R) * n_, cudaMemcpyDeviceToDevice, s_));
            }
        };
        auto restore = [&](uint64_t c) {
            for (int a = 0; a < 3; ++a) {
                ACK(cudaMemcpyAsync(x_[a], cx[3 * c + a], sizeof(double) * n_, cudaMemcpyDeviceToDevice, s_));
                ACK(cudaMemcpyAsync(p_[a], cp[3 * c + a], sizeof(R) * n_, cudaMemcpyDeviceToDevice, s_));
            }
        };
        // Reverse-pass work arrays are allocated before timing starts.
        double* lx[3];
        double* lp[3];
        R* v[3];
        R* u[3];
        R* psi = nullptr;
        const bool want_grad = grad_out && target;
        if (want_grad) {
            for (int a = 0; a < 3; ++a) {
                lx[a] = dmalloc<double>(n_, tmp);
                lp[a] = dmalloc<double>(n_, tmp);
                v[a] = dmalloc<R>(n_, tmp);
                u[a] = dmalloc<R>(cells_, tmp);
            }
            psi = dmalloc<R>(cells_, tmp);
        }
        // The potential of every forward state (S + 1 meshes) is kept when
        // device memory allows: the reverse pass then re-derives each state's
        // force by one gather instead of a deposit and a Green's-function
        // solve. Particle states stay checkpointed every k steps either way.
        std::vector<R*> kept;
        if (want_grad) {
            size_t free_b = 0, total_b = 0;
            const size_t need = (S + 1) * cells_ * sizeof(R);
            if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && need + (size_t(1) << 30) < free_b / 2) {
                R* block = dmalloc<R>((S + 1) * cells_, tmp);
                for (uint64_t j = 0; j <= S; ++j) kept.push_back(block + j * cells_);
            }
        }
        auto keep_of = [&](uint64_t j) { return kept.empty() ? nullptr : kept[j]; };
        double* d_loss = dmalloc<double>(1, tmp);
        double* d_delta = delta_out ? dmalloc<double>(cells_, tmp) : nullptr;
        double* d_target = nullptr;
        if (target) {
            d_target = dmalloc<double>(cells_, tmp);
            ACK(cudaMemcpy(d_target, target, sizeof(double) * cells_, cudaMemcpyHostToDevice));
        }
        R* field = dmalloc<R>(cells_, tmp);
        // Timed: the KDK forward from the 1LPT state, the loss, and the reverse
        // KDK pass (the 1LPT map and its adjoint, one FFT set each, are setup).
        cudaEventRecord(e0, s_);
        force(keep_of(0));
        save(0);
        for (uint64_t j = 0; j < S; ++j) {
            kick(cfg_.K1[j]);
            drift(cfg_.D[j]);
            force(keep_of(j + 1));
            kick(cfg_.K2[j]);
            if ((j + 1) % k == 0 && j + 1 < S) save((j + 1) / k);
        }
        // ---- loss on the final CIC density ----------------------------------
        const double mbar = cfg_.particle_mass * static_cast<double>(n_) / static_cast<double>(cells_);
        ACK(cudaMemsetAsync(d_loss, 0, sizeof(double), s_));
        ACK(cudaMemsetAsync(mesh_, 0, sizeof(R) * cells_, s_));
        k_deposit<R><<<nb(n_), kT, 0, s_>>>(n_, x_[0], x_[1], x_[2], static_cast<R>(cfg_.particle_mass),
                                            axis_, mesh_, status_);
        k_loss<R><<<1184, kT, 0, s_>>>(cells_, mesh_, d_target, 1.0 / mbar, cfg_.particle_mass / mbar,
                                       field, d_delta, d_loss);
        ACK(cudaMemcpyAsync(loss_out, d_loss, sizeof(double), cudaMemcpyDeviceToHost, s_));
        if (delta_out)
            ACK(cudaMemcpyAsync(delta_out, d_delta, sizeof(double) * cells_, cudaMemcpyDeviceToHost, s_));
        cudaEventRecord(e1, s_);
        if (want_grad) {
            // ---- reverse leapfrog ---------------------------------------------
            for (int a = 0; a < 3; ++a) {
                ACK(cudaMemsetAsync(lx[a], 0, sizeof(double) * n_, s_));
                ACK(cudaMemsetAsync(lp[a], 0, sizeof(double) * n_, s_));
            }
            // dL/dx_S: deposit transpose with the weight derivative.
            k_vjp_gather<R><<<nb(n_), kT, 0, s_>>>(n_, x_[0], x_[1], x_[2], field, R(1), nullptr,
                                                   nullptr, nullptr, nullptr, axis_, inv_two_dx_,
                                                   lx[0], lx[1], lx[2]);
            for (uint64_t jj = S; jj-- > 0;) {
                const double coef = cfg_.K2[jj] + (jj + 1 < S ? cfg_.K1[jj + 1] : 0.0);
                vjp(coef, lx, lp, v, u, psi);  // at x_{jj+1} with phi_{jj+1}
                // lp += D lx; reconstruct state jj: p' = p_{jj+1} - K2 a_{jj+1}
                k_axpy3_kick<R><<<nb(n_), kT, 0, s_>>>(n_, cfg_.D[jj], lx[0], lx[1], lx[2], lp[0],
                                                       lp[1], lp[2], p_[0], p_[1], p_[2], acc_[0],
                                                       acc_[1], acc_[2], static_cast<R>(-cfg_.K2[jj]));
                if (jj % k == 0) {
                    restore(jj / k);
                    if (kept.empty()) force(); else force_from(kept[jj]);
                } else if (kept.empty()) {
                    drift(-cfg_.D[jj]);
                    force();
                    kick(-cfg_.K1[jj]);
                } else {
                    phi_ = kept[jj];
                    k_unstep<R><<<nb(n_), kT, 0, s_>>>(n_, x_[0], x_[1], x_[2], p_[0], p_[1], p_[2],
                                                       -cfg_.D[jj], cfg_.box_size, phi_, axis_,
                                                       inv_two_dx_, static_cast<R>(-cfg_.K1[jj]),
                                                       acc_[0], acc_[1], acc_[2]);
                }
            }
            vjp(cfg_.K1[0], lx, lp, v, u, psi);  // at x_0
            cudaEventRecord(e2, s_);
            // ---- 1LPT adjoint: g_d = lx_d + pf lp_d -----------------------------
            k_axpy3<<<nb(n_), kT, 0, s_>>>(n_, cfg_.momentum_factor, lp[0], lp[1], lp[2], lx[0],
                                           lx[1], lx[2]);
            double* grad = dmalloc<double>(n_, tmp);
            const int arc = lpt_adjoint_device(static_cast<int>(cfg_.n_side), cfg_.box_size, lx, tab,
                                               tab + cfg_.n_nodes, tab + 2 * cfg_.n_nodes,
                                               static_cast<int>(cfg_.n_nodes), grad, s_, &err);
            if (arc) throw Fail{arc, err ? err : "LPT adjoint failed"};
            ACK(cudaMemcpyAsync(grad_out, grad, sizeof(double) * n_, cudaMemcpyDeviceToHost, s_));
        } else {
            cudaEventRecord(e2, s_);
        }
        ACK(cudaStreamSynchronize(s_));
        unsigned int st = 0;
        ACK(cudaMemcpy(&st, status_, sizeof(unsigned int), cudaMemcpyDeviceToHost));
        if (timings) {
            float t1 = 0.f, t2 = 0.f;
            cudaEventElapsedTime(&t1, e0, e1);
            cudaEventElapsedTime(&t2, e1, e2);
            timings[0] = t1;
            timings[1] = t2;
            timings[2] = static_cast<double>(solves_);
            timings[3] = static_cast<double>(vjps_);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(e2);
        for (void* p : tmp) cudaFree(p);
        if (st) throw Fail{HYOWON_ELOGIC, "a position left the mesh domain"};
    }

private:
    VjpConfig cfg_;
    cudaStream_t s_;
    int N_ = 0;
    uint32_t n_ = 0;
    uint64_t cells_ = 0, half_ = 0;
    Axis axis_{};
    R inv_two_dx_ = 0, c_green_ = 0;
    R* lap_ = nullptr;
    cufftHandle r2c_ = 0, c2r_ = 0;
    bool five_ = false;               // power-of-two mesh: five-pass solve
    poisson::Plan* plan_ = nullptr;
    C* tw_ = nullptr;
    R* c_green_dev_ = nullptr;
    double four_pi_G_ = 0.0, scale_ = 0.0;
    bool plans_ = false;
    R* mesh_ = nullptr;
    R* phi_own_ = nullptr;
    R* phi_ = nullptr;
    C* modes_ = nullptr;
    unsigned int* status_ = nullptr;
    double* x_[3] = {};
    R* p_[3] = {};
    R* acc_[3] = {};
    uint64_t solves_ = 0, vjps_ = 0;
    std::vector<void*> owned_;
};

thread_local std::string g_adj_err;

}  // namespace

// Engines kept by a PM handle between its VJP calls.
struct Cache {
    Engine<double>* e64 = nullptr;
    Engine<float>* e32 = nullptr;
    ~Cache() {
        delete e64;
        delete e32;
    }
};

void destroy_cache(Cache* c) { delete c; }

int run_cached(Cache** cache, const VjpConfig& cfg, cudaStream_t s, const double* noise,
               const double* target_delta, double* loss, double* grad_noise,
               double* final_delta, double* timings, std::string* err) {
    try {
        if (!*cache) *cache = new Cache();
        Cache* c = *cache;
        if (cfg.precision == HYOWON_FP64) {
            if (c->e64 && !c->e64->same_geometry(cfg)) {
                delete c->e64;
                c->e64 = nullptr;
            }
            if (!c->e64) c->e64 = new Engine<double>(cfg, s);
            c->e64->set_config(cfg);
            c->e64->run(noise, target_delta, loss, grad_noise, final_delta, timings);
        } else {
            if (c->e32 && !c->e32->same_geometry(cfg)) {
                delete c->e32;
                c->e32 = nullptr;
            }
            if (!c->e32) c->e32 = new Engine<float>(cfg, s);
            c->e32->set_config(cfg);
            c->e32->run(noise, target_delta, loss, grad_noise, final_delta, timings);
        }
    } catch (const Fail& f) {
        if (err) *err = f.msg;
        return f.code;
    } catch (const std::bad_alloc&) {
        if (err) *err = "out of host memory";
        return HYOWON_ENOMEM;
    }
    return HYOWON_OK;
}

}  // namespace hyowon::adj

extern "C" {

const char* hyowon_vjp_last_error(void) { return hyowon::adj::g_adj_err.c_str(); }

int hyowon_vjp_1lpt_pm(const hyowon_vjp_config* cfg, const double* noise,
                       const double* target_delta, double* loss, double* grad_noise,
                       double* final_delta, double* timings) {
    using namespace hyowon::adj;
    g_adj_err.clear();
    if (!cfg || !noise || !loss) {
        g_adj_err = "config, noise and loss must be non-null";
        return HYOWON_EINVAL;
    }
    if (cfg->n_side < 2 || cfg->mesh_size < 2 || cfg->n_steps < 1 || !cfg->K1 || !cfg->D || !cfg->K2
        || cfg->n_nodes < 2 || !cfg->ln_k || !cfg->ln_p || !cfg->ln_p_y2
        || !(cfg->particle_mass > 0.0) || !(cfg->box_size > 0.0)
        || (cfg->precision != HYOWON_FP64 && cfg->precision != HYOWON_FP32_FIXED)) {
        g_adj_err = "invalid VJP configuration";
        return HYOWON_EINVAL;
    }
    if (grad_noise && !target_delta) {
        g_adj_err = "the gradient needs a target density";
        return HYOWON_EINVAL;
    }
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        g_adj_err = "stream creation failed";
        return HYOWON_ECUDA;
    }
    int rc = HYOWON_OK;
    try {
        if (cfg->precision == HYOWON_FP64) {
            Engine<double> e(*cfg, s);
            e.run(noise, target_delta, loss, grad_noise, final_delta, timings);
        } else {
            Engine<float> e(*cfg, s);
            e.run(noise, target_delta, loss, grad_noise, final_delta, timings);
        }
    } catch (const Fail& f) {
        g_adj_err = f.msg;
        rc = f.code;
    }
    cudaStreamDestroy(s);
    return rc;
}

}  // extern "C"
