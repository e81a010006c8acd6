/*
 * hyowon_ic.h -- C ABI of HYOWON's generated initial conditions on the
 * device: the Philox per-mode Gaussian Fourier field and first- or
 * second-order (projected) LPT displacements of the particle lattice.
 *
 * Replaces, for one process, the generate branch of
 * InitialConditions (src/ic/initial_conditions.cpp:295-378):
 *   corner lattice  x = (i, j, k) L / N, p = 0, particle (i N + j) N + k
 *   RandomField::generate          (src/ic/random_field.cpp:70-330)
 *   LPTDisplacement::apply_to_arrays (src/ic/lpt_displacement.cpp:150-520)
 * The host keeps what is O(1) or O(K^2): the power-spectrum file and its
 * spline (LinearPowerSpectrum), the growth factors (CosmologyModel) and the
 * configuration rules; the device does everything that is O(M^3).
 *
 * The spectrum crosses the boundary as P evaluated at the represented
 * wavenumbers k_s = double(sqrt((long double) s)) * (2 pi / L) for
 * s = |m|^2 = 0 .. 3K^2 (include/cosmo_nbody/ic/particle_lattice_bandlimit.hpp:27-37):
 * every retained mode's power is one of these, so power[s] is
 * pk.evaluate(k_s) exactly as the reference's generator forms it
 * (power[0] is ignored). Every entry s >= 1 must be finite and positive.
 *
 * All calls are synchronous and return a hyowon_status (include/hyowon_pm.h);
 * hyowon_ic_last_error() gives the message of the last failure on the
 * calling thread.
 */
#ifndef HYOWON_IC_H
#define HYOWON_IC_H

#include <stdint.h>

#include "hyowon_pm.h"

#ifdef __cplusplus
extern "C" {
#endif

enum hyowon_ic_amplitude { HYOWON_IC_GAUSSIAN = 0, HYOWON_IC_FIXED = 1 };
enum hyowon_ic_pairing { HYOWON_IC_INDEPENDENT = 0, HYOWON_IC_PAIR_A = 1, HYOWON_IC_PAIR_B = 2 };

/* The ic.* coordinates of SimulationParameters
 * (include/cosmo_nbody/config/simulation_parameters.hpp:59-82) plus the
 * start-epoch LPT factors apply_to_arrays derives from CosmologyModel
 * (src/ic/lpt_displacement.cpp:197-222). */
typedef struct hyowon_ic_params {
    uint64_t particles_per_dimension; /* N (box.N)                                  */
    uint64_t mesh_per_dimension;      /* M; 0 = automatic: N, or 2N for 2LPT when
                                         M = N is not alias free (M > 3K)          */
    double box_size;                  /* L                                          */
    uint64_t seed;
    int64_t max_mode_per_axis;        /* K; < 0 = (N - 1) / 2                       */
    int amplitude_mode;               /* hyowon_ic_amplitude                        */
    int phase_pairing;                /* hyowon_ic_pairing                          */
    int lpt_order;                    /* 1 or 2                                     */
    double momentum_factor_1;         /* a^2 H(a) f1(a)                             */
    double position_factor_2;         /* D2(a) / D1(a)^2          (2LPT only)       */
    double momentum_factor_2;         /* a^2 H(a) f2(a) D2 / D1^2 (2LPT only)       */
} hyowon_ic_params_t;

/* Validates p like SimulationParameters::validate_initial_conditions
 * (src/config/simulation_parameters.cpp:153-202,262-330) and returns the IC
 * mesh M and the Cartesian support K. No device work. */
int hyowon_ic_resolve(const hyowon_ic_params_t* p, uint64_t* mesh, uint64_t* max_mode);

/* Host only: amp[2s] = sqrt(var_s), amp[2s+1] = sqrt(var_s / 2) with
 * var_s = M^6 / L^3 * power[s] formed as the generator forms it
 * (math::ScaledPositiveProduct, random_field.cpp:119-129,218-247), for
 * s = 0 .. n - 1 (zeros at s = 0). */
int hyowon_ic_mode_amplitudes(uint64_t mesh, double box_size, uint64_t n, const double* power,
                              double* amp);

/* RandomField::generate on the device; modes (host) receives the half
 * spectrum, M * M * (M/2 + 1) complex values as interleaved doubles in
 * complex_index order ((i M + j)(M/2 + 1) + k). n_power >= 3K^2 + 1. */
int hyowon_ic_field(const hyowon_ic_params_t* p, uint64_t n_power, const double* power,
                    double* modes);

/* The whole generate branch on the device; the N^3 particles (host arrays,
 * particle order) receive positions in [0, L) and canonical momenta. */
int hyowon_ic_generate(const hyowon_ic_params_t* p, uint64_t n_power, const double* power,
                       double* x, double* y, double* z, double* px, double* py, double* pz);

/* The same, written straight into the solver's device-resident particle
 * state (replacing it); every particle gets uniform_mass
 * (SimulationParameters::particle_mass). For 2LPT on a power-of-two IC mesh
 * the handle keeps the generation's work arrays (four M^3 binary64 fields:
 * 34 GB at M = 1024) and plans until its next upload, step, force solve,
 * power spectrum or destroy, so that generating several realisations
 * (seeds) allocates once. Errors are read with hyowon_pm_last_error(h). */
int hyowon_pm_generate_ics(hyowon_pm_t h, const hyowon_ic_params_t* p, uint64_t n_power,
                           const double* power, double uniform_mass);

const char* hyowon_ic_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
