/*
 * hyowon_cosmology.h -- host-side binary64 scalars of the KDK step for flat
 * matter + Lambda: expansion rate, drift / kick factors, the logarithmic step
 * schedule and linear growth. These stay on the host (they are O(steps)
 * scalars); the device step consumes the K1, D, K2 they produce.
 *
 * All functions return 0 on success, 1 on invalid arguments, 3 when a result
 * is not finite.
 */
#ifndef HYOWON_COSMOLOGY_H
#define HYOWON_COSMOLOGY_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* CosmologyModel::H(a) in km/s/(Mpc/h), H0 = 100
 * (src/cosmology/cosmology_model.cpp:167-179). */
int hyowon_hubble(double omega_m, double omega_l, uint64_t n, const double* a, double* H);

/* DriftKickIntegrator::drift_factor / kick_factor
 * (src/cosmology/drift_kick_factors.cpp:91-141): D = int da/(a^3 H),
 * K = int da/(a^2 H), by composite Gauss-Legendre refined until the 8/16-point
 * gap and the refinement change are below one binary64 spacing. */
int hyowon_drift_factor(double omega_m, double omega_l, double a1, double a2, double* D);
int hyowon_kick_factor(double omega_m, double omega_l, double a1, double a2, double* K);

/* Correctly rounded sqrt(a*b) of positive binary64 values (the KDK midpoint,
 * src/time/time_stepper.cpp:66-86). */
int hyowon_geometric_mean(double a, double b, double* out);

/* TimeStepper boundaries (src/time/time_stepper.cpp:194-276) for a single final
 * stop, plus the factors of each step. out6[6*k..] = {a_begin, a_half, a_end,
 * D, K1, K2}. *n_steps receives the step count; HYOWON returns 1 if it
 * exceeds max_steps. */
int hyowon_schedule(double omega_m, double omega_l, double a_start, double a_final,
                    double delta_ln_a, uint64_t max_steps, double* out6, uint64_t* n_steps);

/* Linear growth D1(a) (normalised to 1 at a = 1) and f1 = dlnD1/dlna of flat
 * matter + Lambda (include/cosmo_nbody/cosmology/cosmology_model.hpp:47-48),
 * from the integral solution D1 ~ E(a) int_0^a da'/(a' E(a'))^3. */
int hyowon_growth(double omega_m, double omega_l, uint64_t n, const double* a, double* D1,
                  double* f1);

/* Second-order growth D2(a) (normalised by D1(1)^2, negative) and
 * f2 = dln|D2|/dlna of flat matter + Lambda together with D1, f1
 * (include/cosmo_nbody/cosmology/cosmology_model.hpp:50-53): RK4 in ln a of
 * the growth ODE from the matter era. 0 < a <= 1. The 2LPT factors of
 * hyowon_ic_params_t are D2/D1^2 and a^2 H f2 D2/D1^2. */
int hyowon_growth2(double omega_m, double omega_l, uint64_t n, const double* a, double* D1,
                   double* f1, double* D2, double* f2);

#ifdef __cplusplus
}
#endif
#endif
