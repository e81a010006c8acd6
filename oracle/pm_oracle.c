/*
 * pm_oracle.c -- CPU restatement of HYOWON's PM force and KDK update.
 *
 * TEST INFRASTRUCTURE ONLY (see pm_oracle.h). Every function follows the
 * reference's operation order so that, compiled with -ffp-contract=off, the
 * cell assignment, the deposit, the Green's-function symbol, the gradient
 * gather and the KDK arithmetic reproduce the reference bit for bit; only the
 * FFT (oracle/fft3d.c instead of FFTW) rounds differently.
 */
#include "pm_oracle.h"
#include "fft3d.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#pragma STDC FP_CONTRACT OFF

#define ORC_OK 0
#define ORC_EINVAL 1
#define ORC_ELOGIC 2
#define ORC_EOVERFLOW 3
#define ORC_EUNDERFLOW 4

static const double ORC_PI = 3.14159265358979323846;

/* include/cosmo_nbody/cosmology/units.hpp:12-25 */
double orc_gravitational_constant(void) {
    const double G_SI = 6.67430e-11;
    const double Mpc_in_m = 3.085677581491367e22;
    const double Msun_in_kg = 1.98847e30;
    const double MassUnit_in_kg = 1e10 * Msun_in_kg;
    const double V = 1000.0;
    return G_SI * MassUnit_in_kg / (Mpc_in_m * V * V);
}

/* include/cosmo_nbody/math/periodic_box.hpp:27-41 */
double orc_wrap(double x, double L) {
    if (!isfinite(x) || !isfinite(L) || L <= 0.0) return NAN;
    if (x >= 0.0 && x < L) return x;
    double w = fmod(x, L);
    if (!isfinite(w)) return NAN;
    if (w < 0.0) w += L;
    if (w >= L) w = 0.0;
    return w == 0.0 ? 0.0 : w;
}

/* include/cosmo_nbody/math/periodic_box.hpp:44-61 */
double orc_minimum_image(double dx, double L) {
    if (!isfinite(dx) || !isfinite(L) || L <= 0.0) return NAN;
    const double half_L = 0.5 * L;
    if (!isfinite(half_L) || half_L <= 0.0) return NAN;
    if (dx >= -half_L && dx < half_L) return dx;
    double w = remainder(dx, L);
    if (!isfinite(w)) return NAN;
    if (w >= half_L) w -= L;
    else if (w < -half_L) w += L;
    return w == 0.0 ? 0.0 : w;
}

typedef struct {
    double L, dx, upper;
    uint64_t N;
} orc_axis;

/* CICCoordinateAxis ctor (src/mesh/cic_coordinate.hpp:45-93); dx as
 * MeshGeometry forms it (include/cosmo_nbody/mesh/mesh_geometry.hpp:44). */
static orc_axis axis_make(double L, uint64_t N) {
    orc_axis a;
    a.L = L;
    a.N = N;
    a.dx = L / (double)N;
    a.upper = nextafter((double)N, 0.0);
    return a;
}

/* CICCoordinateAxis::operator() (src/mesh/cic_coordinate.hpp:95-121). */
static int axis_coord(const orc_axis* a, double pos, int64_t* base, double* frac) {
    const double wrapped = orc_wrap(pos, a->L);
    if (!isfinite(wrapped) || wrapped < 0.0 || !(wrapped < a->L)) return ORC_ELOGIC;
    const double unbounded = wrapped / a->dx;
    if (!isfinite(unbounded)) return ORC_ELOGIC;
    double scaled = unbounded < 0.0 ? 0.0 : unbounded;
    if (scaled > a->upper) scaled = a->upper;
    const int64_t b = (int64_t)floor(scaled);
    if (b < 0 || (uint64_t)b >= a->N) return ORC_ELOGIC;
    const double f = scaled - (double)b;
    if (!(f >= 0.0 && f < 1.0)) return ORC_ELOGIC;
    *base = b;
    *frac = f;
    return ORC_OK;
}

static uint64_t wrap_index(int64_t i, uint64_t N) {
    const int64_t n = (int64_t)N;
    int64_t w = i % n;
    if (w < 0) w += n;
    return (uint64_t)w;
}

int orc_cic_coords(double L, uint64_t N, uint64_t n, const double* pos,
                   int64_t* base, double* frac) {
    if (N == 0 || !isfinite(L) || L <= 0.0) return ORC_EINVAL;
    const orc_axis a = axis_make(L, N);
    for (uint64_t i = 0; i < n; ++i) {
        const int rc = axis_coord(&a, pos[i], &base[i], &frac[i]);
        if (rc) return rc;
    }
    return ORC_OK;
}

static int require_finite_positions(uint64_t n, const double* x, const double* y,
                                    const double* z) {
    for (uint64_t i = 0; i < n; ++i) {
        if (!isfinite(x[i]) || !isfinite(y[i]) || !isfinite(z[i])) return ORC_EINVAL;
    }
    return ORC_OK;
}

int orc_x_plane_bins(double L, uint64_t N, uint64_t n, const double* x,
                     uint64_t* offsets, uint32_t* order) {
    if (N == 0) return ORC_EINVAL;
    const orc_axis a = axis_make(L, N);
    int64_t* bx = (int64_t*)malloc(sizeof(int64_t) * (n ? n : 1));
    for (uint64_t i = 0; i < n; ++i) {
        double f;
        const int rc = axis_coord(&a, x[i], &bx[i], &f);
        if (rc) { free(bx); return rc; }
    }
    memset(offsets, 0, sizeof(uint64_t) * (N + 1));
    for (uint64_t i = 0; i < n; ++i) offsets[bx[i] + 1] += 1;
    for (uint64_t p = 0; p < N; ++p) offsets[p + 1] += offsets[p];
    uint64_t* cursor = (uint64_t*)malloc(sizeof(uint64_t) * N);
    memcpy(cursor, offsets, sizeof(uint64_t) * N);
    for (uint64_t i = 0; i < n; ++i) order[cursor[bx[i]]++] = (uint32_t)i;
    free(cursor);
    free(bx);
    return ORC_OK;
}

static int check_masses(uint64_t n, const double* masses, double uniform_mass) {
    if (!masses) {
        if (!isfinite(uniform_mass) || uniform_mass < 0.0) return ORC_EINVAL;
        return ORC_OK;
    }
    for (uint64_t i = 0; i < n; ++i) {
        if (!isfinite(masses[i]) || masses[i] < 0.0) return ORC_EINVAL;
    }
    return ORC_OK;
}

int orc_deposit(double L, uint64_t N, uint64_t n, const double* x, const double* y,
                const double* z, const double* masses, double uniform_mass,
                double* mesh) {
    if (N == 0 || !isfinite(L) || L <= 0.0) return ORC_EINVAL;
    int rc = require_finite_positions(n, x, y, z);
    if (rc) return rc;
    rc = check_masses(n, masses, uniform_mass);
    if (rc) return rc;
    const uint64_t plane = N * N;
    memset(mesh, 0, sizeof(double) * plane * N);
    if (n == 0) return ORC_OK;

    uint64_t* offsets = (uint64_t*)malloc(sizeof(uint64_t) * (N + 1));
    uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * n);
    rc = orc_x_plane_bins(L, N, n, x, offsets, order);
    if (rc) { free(offsets); free(order); return rc; }
    const orc_axis a = axis_make(L, N);

    /* Destination plane gx receives lower-x weights from particles based in
     * gx, then upper-x weights from particles based in gx-1
     * (mass_assignment_deposit.inc:193-240). Planes are independent. */
#pragma omp parallel for schedule(dynamic, 1) reduction(| : rc)
    for (long long gxl = 0; gxl < (long long)N; ++gxl) {
        const uint64_t gx = (uint64_t)gxl;
        double* dst = mesh + gx * plane;
        for (int pass = 0; pass < 2; ++pass) {
            const uint64_t src = pass == 0 ? gx : wrap_index((int64_t)gx - 1, N);
            const int upper_x = pass == 1;
            for (uint64_t c = offsets[src]; c < offsets[src + 1]; ++c) {
                const uint32_t p = order[c];
                int64_t ixb, iy, iz;
                double tx, ty, tz;
                int e = axis_coord(&a, x[p], &ixb, &tx);
                e |= axis_coord(&a, y[p], &iy, &ty);
                e |= axis_coord(&a, z[p], &iz, &tz);
                if (e) { rc |= ORC_ELOGIC; continue; }
                const double xw = upper_x ? tx : (1.0 - tx);
                const double wy[2] = {1.0 - ty, ty};
                const double wz[2] = {1.0 - tz, tz};
                const double mass = masses ? masses[p] : uniform_mass;
                for (int yo = 0; yo < 2; ++yo) {
                    const uint64_t gy = wrap_index(iy + yo, N);
                    for (int zo = 0; zo < 2; ++zo) {
                        const uint64_t gz = wrap_index(iz + zo, N);
                        dst[gy * N + gz] += mass * xw * wy[yo] * wz[zo];
                    }
                }
            }
        }
    }
    free(offsets);
    free(order);
    return rc;
}

/* Exact input mass (src/gravity/pm_solver.cpp:87-118); uniform mass is the
 * correctly rounded product, explicit masses are summed in a wide format. */
static double input_mass(uint64_t n, const double* masses, double uniform_mass) {
    if (!masses) return uniform_mass * (double)n;
#if defined(__SIZEOF_FLOAT128__)
    __float128 s = 0;
    for (uint64_t i = 0; i < n; ++i) s += (__float128)masses[i];
    return (double)s;
#else
    long double s = 0;
    for (uint64_t i = 0; i < n; ++i) s += masses[i];
    return (double)s;
#endif
}

/* GreenFunction tables and kernel (src/mesh/green_function.cpp:59-87,137-207). */
static void green_tables(double L, uint64_t N, double* lap, double* win) {
    const double dx = L / (double)N;
    const double inv = 1.0 / dx;
    const double inv2 = inv * inv;
    const double n = (double)N;
    for (uint64_t i = 0; i < N; ++i) {
        const int64_t mode = i <= N / 2 ? (int64_t)i : (int64_t)i - (int64_t)N;
        const double kdh = ORC_PI * (double)mode / n;
        const double s = sin(kdh);
        lap[i] = -4.0 * inv2 * s * s;
        const long double arg = 3.141592653589793238462643383279502884L
            * (long double)mode / (long double)N;
        if (arg == 0.0L) {
            win[i] = 1.0;
        } else {
            long double raw = sinl(arg) / arg;
            long double mag = fabsl(raw);
            if (mag > 1.0L) mag = 1.0L;
            win[i] = (double)(mag * mag);
        }
    }
}

int orc_potential(double L, uint64_t N, int deconvolve, uint64_t n, const double* x,
                  const double* y, const double* z, const double* masses,
                  double uniform_mass, double* density_out, double* phi_out) {
    const uint64_t cells = N * N * N;
    double* field = (double*)malloc(sizeof(double) * cells);
    int rc = orc_deposit(L, N, n, x, y, z, masses, uniform_mass, field);
    if (rc) { free(field); return rc; }
    const double total = input_mass(n, masses, uniform_mass);
    if (!isfinite(total) || total <= 0.0) { free(field); return ORC_EINVAL; }

    /* DensityNormalization (include/cosmo_nbody/math/density_normalization.hpp:34-71)
     * as applied by PMSolver (src/gravity/pm_solver.cpp:710-759). */
    const double dx = L / (double)N;
    const double cells_real = (double)cells;
    const double mean = total / cells_real;
    const double inv_vol = 1.0 / (dx * dx * dx);
    const int direct = fma(mean, cells_real, -total) == 0.0;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)cells; ++i) {
        if (direct) {
            field[i] = (field[i] - mean) * inv_vol;
        } else {
            const double num = fma(field[i], cells_real, -total);
            field[i] = num * (inv_vol * (1.0 / cells_real));
        }
    }
    if (density_out) memcpy(density_out, field, sizeof(double) * cells);

    const uint64_t H = N / 2 + 1;
    double* modes = (double*)malloc(sizeof(double) * 2 * N * N * H);
    orc_fft3d_r2c(N, field, modes);

    double* lap = (double*)malloc(sizeof(double) * N);
    double* win = (double*)malloc(sizeof(double) * N);
    green_tables(L, N, lap, win);
    const double four_pi_G = 4.0 * ORC_PI * orc_gravitational_constant();
#pragma omp parallel for schedule(static)
    for (long long ixl = 0; ixl < (long long)N; ++ixl) {
        const uint64_t ix = (uint64_t)ixl;
        for (uint64_t iy = 0; iy < N; ++iy) {
            for (uint64_t iz = 0; iz < H; ++iz) {
                double f = 0.0;
                if (!(ix == 0 && iy == 0 && iz == 0)) {
                    const double Dk = lap[ix] + lap[iy] + lap[iz];
                    f = four_pi_G / Dk;
                    if (deconvolve) {
                        const double wt = win[ix] * win[iy] * win[iz];
                        f /= (wt * wt);
                    }
                }
                const uint64_t idx = iz + H * (iy + N * ix);
                modes[2 * idx] *= f;
                modes[2 * idx + 1] *= f;
            }
        }
    }
    orc_fft3d_c2r_destroy(N, modes, phi_out);
    const double norm = 1.0 / ((double)N * (double)N * (double)N);
    for (uint64_t i = 0; i < cells; ++i) phi_out[i] *= norm;
    free(lap);
    free(win);
    free(modes);
    free(field);
    return ORC_OK;
}

int orc_gradient_gather_add(double L, uint64_t N, const double* phi, uint64_t n,
                            const double* x, const double* y, const double* z,
                            double* ax, double* ay, double* az) {
    int rc = require_finite_positions(n, x, y, z);
    if (rc) return rc;
    for (uint64_t i = 0; i < N * N * N; ++i) {
        if (!isfinite(phi[i])) return ORC_EINVAL;
    }
    const orc_axis a = axis_make(L, N);
    const double two_dx = 2.0 * a.dx;
#define PHI(gx, gy, gz) phi[((gx) * N + (gy)) * N + (gz)]
#pragma omp parallel for schedule(static) reduction(| : rc)
    for (long long pl = 0; pl < (long long)n; ++pl) {
        const uint64_t p = (uint64_t)pl;
        int64_t ix, iy, iz;
        double fx, fy, fz;
        int e = axis_coord(&a, x[p], &ix, &fx);
        e |= axis_coord(&a, y[p], &iy, &fy);
        e |= axis_coord(&a, z[p], &iz, &fz);
        if (e) { rc |= ORC_ELOGIC; continue; }
        const double wx[2] = {1.0 - fx, fx};
        const double wy[2] = {1.0 - fy, fy};
        const double wz[2] = {1.0 - fz, fz};
        double gxs = 0.0, gys = 0.0, gzs = 0.0;
        for (int ox = 0; ox < 2; ++ox) {
            const uint64_t gx = wrap_index(ix + ox, N);
            const uint64_t gxp = wrap_index((int64_t)gx + 1, N);
            const uint64_t gxm = wrap_index((int64_t)gx - 1, N);
            for (int oy = 0; oy < 2; ++oy) {
                const uint64_t gy = wrap_index(iy + oy, N);
                const uint64_t gyp = wrap_index((int64_t)gy + 1, N);
                const uint64_t gym = wrap_index((int64_t)gy - 1, N);
                for (int oz = 0; oz < 2; ++oz) {
                    const uint64_t gz = wrap_index(iz + oz, N);
                    const uint64_t gzp = wrap_index((int64_t)gz + 1, N);
                    const uint64_t gzm = wrap_index((int64_t)gz - 1, N);
                    const double w = wx[ox] * wy[oy] * wz[oz];
                    const double dxv = PHI(gxp, gy, gz) - PHI(gxm, gy, gz);
                    const double dyv = PHI(gx, gyp, gz) - PHI(gx, gym, gz);
                    const double dzv = PHI(gx, gy, gzp) - PHI(gx, gy, gzm);
                    gxs += w * (-dxv / two_dx);
                    gys += w * (-dyv / two_dx);
                    gzs += w * (-dzv / two_dx);
                }
            }
        }
        ax[p] += gxs;
        ay[p] += gys;
        az[p] += gzs;
    }
#undef PHI
    for (uint64_t p = 0; p < n; ++p) {
        if (!isfinite(ax[p]) || !isfinite(ay[p]) || !isfinite(az[p])) return ORC_EOVERFLOW;
    }
    return rc;
}

int orc_pm_forces(double L, uint64_t N, int deconvolve, uint64_t n, const double* x,
                  const double* y, const double* z, const double* masses,
                  double uniform_mass, double* ax, double* ay, double* az) {
    const uint64_t cells = N * N * N;
    double* phi = (double*)malloc(sizeof(double) * cells);
    double* fx = (double*)calloc(n ? n : 1, sizeof(double));
    double* fy = (double*)calloc(n ? n : 1, sizeof(double));
    double* fz = (double*)calloc(n ? n : 1, sizeof(double));
    int rc = orc_potential(L, N, deconvolve, n, x, y, z, masses, uniform_mass, NULL, phi);
    if (!rc) rc = orc_gradient_gather_add(L, N, phi, n, x, y, z, fx, fy, fz);
    if (!rc) {
        /* validate_force_commit then commit (src/gravity/pm_solver.cpp:281-345) */
        for (uint64_t i = 0; i < n && !rc; ++i) {
            if (!isfinite(ax[i] + fx[i]) || !isfinite(ay[i] + fy[i])
                || !isfinite(az[i] + fz[i])) rc = ORC_EOVERFLOW;
        }
        if (!rc) {
            for (uint64_t i = 0; i < n; ++i) {
                ax[i] += fx[i];
                ay[i] += fy[i];
                az[i] += fz[i];
            }
        }
    }
    free(phi);
    free(fx);
    free(fy);
    free(fz);
    return rc;
}

/* time/particle_update.hpp:45-68 */
static double add_periodic_displacement(double pos, double disp, double L) {
    if (!isfinite(pos) || !isfinite(disp) || !isfinite(L) || L <= 0.0) return NAN;
    const double wp = orc_wrap(pos, L);
    const double rd = orc_minimum_image(disp, L);
    if (!isfinite(wp) || !isfinite(rd)) return NAN;
    return orc_wrap(wp + rd, L);
}

int orc_kdk_step(double L, uint64_t N, int deconvolve, uint64_t n, double* x,
                 double* y, double* z, double* px, double* py, double* pz,
                 double* ax, double* ay, double* az, const double* masses,
                 double uniform_mass, double K1, double D, double K2,
                 double* max_drift) {
    /* K1 + drift preflight (leapfrog_integrator.cpp:170-190 with
     * particle_update.hpp:20-116). */
    if (!isfinite(K1) || !isfinite(D) || !isfinite(K2)) return ORC_EOVERFLOW;
    for (uint64_t i = 0; i < n; ++i) {
        const double qx = px[i] + ax[i] * K1;
        const double qy = py[i] + ay[i] * K1;
        const double qz = pz[i] + az[i] * K1;
        if (!isfinite(x[i]) || !isfinite(y[i]) || !isfinite(z[i]) || !isfinite(qx)
            || !isfinite(qy) || !isfinite(qz) || !isfinite(qx * D)
            || !isfinite(qy * D) || !isfinite(qz * D)) return ORC_EOVERFLOW;
        if (!isfinite(add_periodic_displacement(x[i], qx * D, L))
            || !isfinite(add_periodic_displacement(y[i], qy * D, L))
            || !isfinite(add_periodic_displacement(z[i], qz * D, L))) return ORC_EOVERFLOW;
    }
    double mx = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
        const double qx = px[i] + ax[i] * K1;
        const double qy = py[i] + ay[i] * K1;
        const double qz = pz[i] + az[i] * K1;
        px[i] = qx;
        py[i] = qy;
        pz[i] = qz;
        x[i] = add_periodic_displacement(x[i], qx * D, L);
        y[i] = add_periodic_displacement(y[i], qy * D, L);
        z[i] = add_periodic_displacement(z[i], qz * D, L);
        const double d = hypot(hypot(D * qx, D * qy), D * qz);
        if (d > mx) mx = d;
    }
    if (max_drift) *max_drift = mx;
    /* Force at a_end into zeroed accelerations (leapfrog_integrator.cpp:42-132). */
    memset(ax, 0, sizeof(double) * n);
    memset(ay, 0, sizeof(double) * n);
    memset(az, 0, sizeof(double) * n);
    int rc = orc_pm_forces(L, N, deconvolve, n, x, y, z, masses, uniform_mass, ax, ay, az);
    if (rc) return rc;
    /* K2 preflight and publish (leapfrog_integrator.cpp:240-278). */
    for (uint64_t i = 0; i < n; ++i) {
        if (!isfinite(px[i] + ax[i] * K2) || !isfinite(py[i] + ay[i] * K2)
            || !isfinite(pz[i] + az[i] * K2)) return ORC_EOVERFLOW;
    }
    for (uint64_t i = 0; i < n; ++i) {
        px[i] = px[i] + ax[i] * K2;
        py[i] = py[i] + ay[i] * K2;
        pz[i] = pz[i] + az[i] * K2;
    }
    return ORC_OK;
}

/* G m [(r^2+eps^2)^(-3/2) - (1 - M_S(q))/r^3] in long double; the small-q
 * branch uses the series of (1 - M_S(q))/q^3 = (1/6 - q^2/40 + q^4/448 -
 * q^6/6912 + q^8/110592)/sqrt(pi). */
static long double short_factor_ld(long double r2, long double eps2, long double r_s,
                                   long double Gm) {
    const long double r = sqrtl(r2);
    const long double q = r / r_s;
    const long double isp = 0.564189583547756286948079451560772586L;
    long double longf;
    if (q < 0.02L) {
        const long double q2 = q * q;
        longf = isp * (1.0L / 6.0L + q2 * (-1.0L / 40.0L + q2 * (1.0L / 448.0L
                + q2 * (-1.0L / 6912.0L + q2 / 110592.0L)))) / (r_s * r_s * r_s);
    } else {
        const long double one_minus_ms = erfl(0.5L * q) - q * isp * expl(-0.25L * q * q);
        longf = one_minus_ms / (r2 * r);
    }
    const long double s = r2 + eps2;
    return Gm * (1.0L / (s * sqrtl(s)) - longf);
}

void orc_short_range_pair(double r_s, double eps, double mass, uint64_t n, const double* dx,
                          const double* dy, const double* dz, double* ax, double* ay, double* az) {
    const long double Gm = (long double)orc_gravitational_constant() * mass;
    for (uint64_t i = 0; i < n; ++i) {
        const long double r2 = (long double)dx[i] * dx[i] + (long double)dy[i] * dy[i]
            + (long double)dz[i] * dz[i];
        const long double f = short_factor_ld(r2, (long double)eps * eps, r_s, Gm);
        ax[i] = (double)(f * dx[i]);
        ay[i] = (double)(f * dy[i]);
        az[i] = (double)(f * dz[i]);
    }
}

int orc_short_range_direct(double L, uint64_t n, const double* x, const double* y,
                           const double* z, double mass, uint64_t n_targets,
                           const uint32_t* targets, double r_s, double r_cut, double eps,
                           double* ax, double* ay, double* az) {
    if (!(L > 0.0) || !(r_cut > 0.0) || !(r_cut < 0.5 * L)) return ORC_EINVAL;
    int nc = (int)floor(L / r_cut);
    if (nc < 3) nc = 1;
    const double cs = L / nc;
    const uint64_t ncells = (uint64_t)nc * nc * nc;
    uint64_t* start = (uint64_t*)calloc(ncells + 1, sizeof(uint64_t));
    uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    int* cell = (int*)malloc(sizeof(int) * (n ? n : 1));
    double* wx = (double*)malloc(sizeof(double) * (n ? n : 1));
    double* wy = (double*)malloc(sizeof(double) * (n ? n : 1));
    double* wz = (double*)malloc(sizeof(double) * (n ? n : 1));
    for (uint64_t i = 0; i < n; ++i) {
        wx[i] = orc_wrap(x[i], L);
        wy[i] = orc_wrap(y[i], L);
        wz[i] = orc_wrap(z[i], L);
        int cx = (int)(wx[i] / cs), cy = (int)(wy[i] / cs), cz = (int)(wz[i] / cs);
        if (cx >= nc) cx = nc - 1;
        if (cy >= nc) cy = nc - 1;
        if (cz >= nc) cz = nc - 1;
        cell[i] = (cx * nc + cy) * nc + cz;
        start[cell[i] + 1]++;
    }
    for (uint64_t c = 0; c < ncells; ++c) start[c + 1] += start[c];
    uint64_t* cur = (uint64_t*)malloc(sizeof(uint64_t) * ncells);
    memcpy(cur, start, sizeof(uint64_t) * ncells);
    for (uint64_t i = 0; i < n; ++i) order[cur[cell[i]]++] = (uint32_t)i;
    free(cur);
    const long double Gm = (long double)orc_gravitational_constant() * mass;
    const long double eps2 = (long double)eps * eps;
    const double rc2 = r_cut * r_cut;
    const int reach = nc >= 3 ? 1 : 0;
#pragma omp parallel for schedule(dynamic, 8)
    for (long long ti = 0; ti < (long long)n_targets; ++ti) {
        const uint32_t t = targets[ti];
        const double tx = wx[t], ty = wy[t], tz = wz[t];
        const int cx = cell[t] / (nc * nc), cy = (cell[t] / nc) % nc, cz = cell[t] % nc;
        long double sx = 0, sy = 0, sz = 0;
        for (int ox = -reach; ox <= reach; ++ox)
            for (int oy = -reach; oy <= reach; ++oy)
                for (int oz = -reach; oz <= reach; ++oz) {
                    const int qx = (cx + ox + nc) % nc, qy = (cy + oy + nc) % nc, qz = (cz + oz + nc) % nc;
                    const uint64_t c = ((uint64_t)qx * nc + qy) * nc + qz;
                    for (uint64_t k = start[c]; k < start[c + 1]; ++k) {
                        const uint32_t j = order[k];
                        if (j == t) continue;
                        const double dx = orc_minimum_image(wx[j] - tx, L);
                        const double dy = orc_minimum_image(wy[j] - ty, L);
                        const double dz = orc_minimum_image(wz[j] - tz, L);
                        const double r2 = dx * dx + dy * dy + dz * dz;
                        if (!(r2 < rc2) || r2 == 0.0) continue;
                        const long double f = short_factor_ld(r2, eps2, r_s, Gm);
                        sx += f * dx;
                        sy += f * dy;
                        sz += f * dz;
                    }
                }
        ax[ti] = (double)sx;
        ay[ti] = (double)sy;
        az[ti] = (double)sz;
    }
    free(start);
    free(order);
    free(cell);
    free(wx);
    free(wy);
    free(wz);
    return ORC_OK;
}
