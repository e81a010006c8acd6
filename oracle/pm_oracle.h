/*
 * pm_oracle.h -- CPU restatement of HYOWON's particle-mesh hot path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline use it, as the checker. It is pinned against the reference's own
 * compiled sources (oracle/_ref, built by oracle/ref/Makefile) through the
 * golden fixtures in tests/golden/.
 *
 * Status codes: 0 ok, 1 invalid argument (non-finite input, size mismatch),
 * 3 overflow (non-finite result), 4 underflow.
 */
#ifndef HYOWON_PM_ORACLE_H
#define HYOWON_PM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* G in (Mpc/h)(km/s)^2/(1e10 Msun/h) and 4*pi*G, evaluated in the
 * reference's operation order (include/cosmo_nbody/cosmology/units.hpp:12-25,
 * src/mesh/green_function.cpp:185-186). */
double orc_gravitational_constant(void);

/* math::wrap and math::minimum_image (include/cosmo_nbody/math/periodic_box.hpp:27-61). */
double orc_wrap(double x, double L);
double orc_minimum_image(double dx, double L);

/* CICCoordinateAxis::operator() (src/mesh/cic_coordinate.hpp:95-121) for n
 * positions; returns 2 (logic error) when a coordinate is not admissible. */
int orc_cic_coords(double L, uint64_t N, uint64_t n, const double* pos,
                   int64_t* base, double* frac);

/* build_x_plane_bins (src/mesh/mass_assignment_workspace.inc:264-374): stable
 * counting sort by base x-plane. offsets[N+1], order[n]. */
int orc_x_plane_bins(double L, uint64_t N, uint64_t n, const double* x,
                     uint64_t* offsets, uint32_t* order);

/* CICMassAssignment::deposit (src/mesh/mass_assignment_deposit.inc:15-334) in
 * the reference's plane-owned accumulation order (bit-exact). masses may be
 * NULL for uniform mass. mesh[N^3] is overwritten. */
int orc_deposit(double L, uint64_t N, uint64_t n, const double* x, const double* y,
                const double* z, const double* masses, double uniform_mass,
                double* mesh);

/* PM potential (src/gravity/pm_solver.cpp:710-816 with
 * src/mesh/green_function.cpp:15-241): deposit, density normalisation,
 * r2c, Green's function (pure PM discrete Laplacian, optional W^-2), c2r
 * with 1/N^3. density_out may be NULL. */
int orc_potential(double L, uint64_t N, int deconvolve, uint64_t n, const double* x,
                  const double* y, const double* z, const double* masses,
                  double uniform_mass, double* density_out, double* phi_out);

/* interpolate_centered_gradient3_add_full_mesh
 * (src/mesh/mass_assignment_gradient.cpp:46-226): ADDS -grad(phi) gathered
 * by CIC to ax/ay/az. */
int orc_gradient_gather_add(double L, uint64_t N, const double* phi, uint64_t n,
                            const double* x, const double* y, const double* z,
                            double* ax, double* ay, double* az);

/* PMSolver::compute_forces (src/gravity/pm_solver.cpp:494-567) for the pure-PM
 * method: ADDS the PM acceleration to ax/ay/az. */
int orc_pm_forces(double L, uint64_t N, int deconvolve, uint64_t n, const double* x,
                  const double* y, const double* z, const double* masses,
                  double uniform_mass, double* ax, double* ay, double* az);

/* One LeapfrogIntegrator::step (src/time/leapfrog_integrator.cpp:143-279) with
 * the PM force: on entry a* hold the force at a_begin; on exit the state is at
 * a_end and a* hold the force at a_end. K1, D, K2 are the drift/kick factors
 * of the step. max_drift receives max ||D p_half||. */
int orc_kdk_step(double L, uint64_t N, int deconvolve, uint64_t n, double* x,
                 double* y, double* z, double* px, double* py, double* pz,
                 double* ax, double* ay, double* az, const double* masses,
                 double uniform_mass, double K1, double D, double K2,
                 double* max_drift);

/* TreePM short-range force by direct summation (the checker of the tree walk):
 * for each target index t, the sum over all sources j != t with r < r_cut of
 * G m dx [(r^2+eps^2)^(-3/2) - (1 - M_S(r/r_s))/r^3], dx the minimum-image
 * displacement, M_S(q) = erfc(q/2) + q/sqrt(pi) exp(-q^2/4)
 * (include/cosmo_nbody/gravity/force_split.hpp:1-6), evaluated in long double
 * with a cell list of side >= r_cut. Writes ax/ay/az[n_targets]. */
int orc_short_range_direct(double L, uint64_t n, const double* x, const double* y,
                           const double* z, double mass, uint64_t n_targets,
                           const uint32_t* targets, double r_s, double r_cut, double eps,
                           double* ax, double* ay, double* az);

/* The pair law alone: acceleration from a source of mass m at displacement d. */
void orc_short_range_pair(double r_s, double eps, double mass, uint64_t n, const double* dx,
                          const double* dy, const double* dz, double* ax, double* ay, double* az);

#ifdef __cplusplus
}
#endif
#endif
