/*
 * hyowon_pm.h -- C ABI of the B200 particle-mesh gravity step and
 * kick-drift-kick update for HYOWON.
 *
 * One opaque handle owns everything on the device: the particle state
 * (positions, momenta, accelerations, ids, optional masses), the mass / potential
 * meshes, the cuFFT plans and their workspace, and one CUDA stream. Particle
 * state stays device-resident across steps; the host synchronises it only
 * through hyowon_pm_upload / hyowon_pm_download. Every call is synchronous at
 * return, must come from one host thread per handle, and returns a status code
 * (HYOWON_OK = 0). hyowon_pm_last_error() gives the message of the last failure.
 *
 * Reference interfaces each entry replaces are cited per function
 * (paths relative to the HYOWON source tree).
 */
#ifndef HYOWON_PM_H
#define HYOWON_PM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The C++ wrapper (hyowon_b200/csrc/gpu_pm_solver.hpp) maps
 * them onto the exception types the reference throws for the same condition
 * (src/gravity/pm_solver.cpp:509-525,281-326; src/time/leapfrog_integrator.cpp:183-261). */
enum hyowon_status {
    HYOWON_OK = 0,
    HYOWON_EINVAL = 1,      /* std::invalid_argument: sizes, non-finite inputs   */
    HYOWON_ELOGIC = 2,      /* std::logic_error: state / cell-assignment escape  */
    HYOWON_EOVERFLOW = 3,   /* std::overflow_error: non-finite force or update   */
    HYOWON_EUNDERFLOW = 4,  /* std::underflow_error                              */
    HYOWON_ERUNTIME = 5,    /* std::runtime_error: mass conservation, capacity   */
    HYOWON_ECUDA = 6,       /* CUDA / cuFFT failure                              */
    HYOWON_ENOMEM = 7       /* device allocation failed                          */
};

/* PM force discretisation (include/cosmo_nbody/mesh/pm_force_method.hpp:16-67). */
enum hyowon_method {
    HYOWON_PURE_PM = 0,          /* discrete Laplacian + centred-gradient gather */
    HYOWON_TREEPM_LONG_RANGE = 1 /* continuum -k^2, Gaussian split, spectral -ik */
};

/* Arithmetic form of the step. */
enum hyowon_precision {
    HYOWON_FP64 = 0,        /* binary64 throughout: the drop-in form             */
    HYOWON_FP32_FIXED = 1   /* u32 fixed-point positions, int64 fixed-point mass
                               deposit, FP32 FFT/Green/gather, FP64 drift        */
};

typedef struct hyowon_pm_s* hyowon_pm_t;

/* Replaces the PMSolver constructor (src/gravity/pm_solver.cpp:378-386,
 * include/cosmo_nbody/gravity/pm_solver.hpp:52-56) together with
 * MeshGeometry(L, N_g) (include/cosmo_nbody/mesh/mesh_geometry.hpp:18-62) and
 * PMForceMethod::pure_pm / treepm_long_range. split_scale is r_s for
 * HYOWON_TREEPM_LONG_RANGE and ignored otherwise. mesh_size is 2 .. 2048
 * (HYOWON_EINVAL outside); meshes above 1625 have more than 2^32 cells and
 * are indexed in 64 bits. */
int hyowon_pm_create(double box_size, uint64_t mesh_size, int method,
                     int deconvolve_cic, double split_scale, int precision,
                     hyowon_pm_t* out);

int hyowon_pm_destroy(hyowon_pm_t h);

/* Message of the last failing call on h (never NULL). */
const char* hyowon_pm_last_error(hyowon_pm_t h);

/* Loads the ParticleStore SoA (include/cosmo_nbody/core/particle_store.hpp:33-124)
 * into device memory: positions (any finite value; wrapped on device), canonical
 * momenta p = a^2 dx/dt, and either per-particle masses (masses != NULL) or one
 * uniform mass. Momenta may be NULL (zero). Accelerations become invalid until
 * the next force solve. n = 0 fails with HYOWON_ERUNTIME, as PMSolver's exact
 * input-mass identity does for a zero particle count
 * (src/gravity/pm_solver.cpp:664-679); n is at most 2^32 - 16. */
int hyowon_pm_upload(hyowon_pm_t h, uint64_t n, const double* x, const double* y,
                     const double* z, const double* px, const double* py,
                     const double* pz, const double* masses, double uniform_mass);

/* First-order LPT initial conditions generated on the device, replacing the
 * particle state: from white noise w[n_side^3] (host, unit variance per lattice
 * cell, row-major), delta_k = r2c(w) * sqrt(P(k) n_side^3 / L^3),
 * psi = c2r(i k delta_k / k^2) / n_side^3 (Nyquist derivative zeroed),
 * x = wrap(q + psi), p = momentum_factor * psi on the corner lattice
 * q = (i,j,k) L / n_side, particle index (i n_side + j) n_side + k
 * (src/ic/lpt_displacement.cpp:150-384, src/ic/initial_conditions.cpp:295-313,
 * src/ic/random_field.cpp:119-129). P(k) at the start epoch is a natural cubic
 * spline through (ln_k[i], ln_p[i]) with second derivatives ln_p_y2[i]
 * (src/ic/linear_power_spectrum.cpp:649-664); momentum_factor = a^2 H(a) f1(a).
 * All particles get uniform_mass. */
int hyowon_pm_lpt_ics(hyowon_pm_t h, uint64_t n_side, const double* noise,
                      uint64_t n_nodes, const double* ln_k, const double* ln_p,
                      const double* ln_p_y2, double momentum_factor,
                      double uniform_mass);

/* Copies the device state back in the caller's original particle order. Any
 * pointer may be NULL to skip that component. Positions are returned as
 * stored (the drift wraps them to [0,L)); accelerations are those of the last
 * force solve (HYOWON_ELOGIC if none). */
int hyowon_pm_download(hyowon_pm_t h, double* x, double* y, double* z, double* px,
                       double* py, double* pz, double* ax, double* ay, double* az);

/* Snapshot payload staging for the native HDF5 writer: the /PartType1
 * Coordinates and Velocities datasets (include/cosmo_nbody/io/output_schema.hpp:132-135)
 * as n x 3 row-major binary64 arrays in the caller's original particle order,
 * Velocities = p * (1 / a) (peculiar km/s; write_vector_dataset_batched,
 * src/io/snapshot_io_particle_helpers.inc:116-200). The payload is validated
 * as require_finite_particle_payload (:48-104) does, on the device, before
 * anything is written: HYOWON_EINVAL for a non-finite field or a coordinate
 * outside [0, L), HYOWON_EOVERFLOW when p / a is not finite. Either pointer
 * may be NULL. ParticleIDs stay the caller's (row i is upload index i). */
int hyowon_pm_snapshot_payload(hyowon_pm_t h, double a, double* coordinates,
                               double* velocities);

/* PMSolver::compute_forces (src/gravity/pm_solver.cpp:494-567) on the device
 * state: solves the force at the current positions, stores it as the valid
 * acceleration field, and ADDS it to the host arrays ax/ay/az when they are
 * non-NULL (in original particle order), after validating that every sum is
 * finite (validate_force_commit, src/gravity/pm_solver.cpp:281-326). */
int hyowon_pm_compute_forces(hyowon_pm_t h, double* ax, double* ay, double* az);

/* The stateless drop-in of PMSolver::compute_forces on HOST spans: uploads the
 * positions (and masses), solves, adds the force to ax/ay/az. Equivalent to
 * upload + compute_forces; the handle's previous particle state is replaced. */
int hyowon_pm_forces_host(hyowon_pm_t h, uint64_t n, const double* x, const double* y,
                          const double* z, const double* masses, double uniform_mass,
                          double* ax, double* ay, double* az);

/* One LeapfrogIntegrator::step (src/time/leapfrog_integrator.cpp:143-279) on
 * the device state: K1 kick + drift with periodic wrap, force at a_end, K2 kick.
 * K1, D, K2 are DriftKickIntegrator::kick_factor(a_begin,a_half),
 * drift_factor(a_begin,a_end), kick_factor(a_half,a_end)
 * (src/cosmology/drift_kick_factors.cpp:91-141), computed on the host. If the
 * acceleration field is not valid a force solve runs first
 * (ensure_force_at, :134-141). max_drift (may be NULL) receives
 * max_i ||D p_half,i||, last_step_max_drift_displacement (:214-225).
 * A non-finite K1/drift candidate publishes nothing (HYOWON_EOVERFLOW). */
int hyowon_pm_kdk_step(hyowon_pm_t h, double K1, double D, double K2,
                       double* max_drift);

/* n_steps consecutive KDK steps with per-step factors K1[i], D[i], K2[i]
 * (the SimulationRunner step loop, src/runtime/simulation_runner.cpp:1348-1351,
 * without host work between steps). max_drift may be NULL or hold n_steps. */
int hyowon_pm_run(hyowon_pm_t h, uint64_t n_steps, const double* K1, const double* D,
                  const double* K2, double* max_drift);

/* Particle count and mesh size of the handle. */
int hyowon_pm_info(hyowon_pm_t h, uint64_t* n_particles, uint64_t* mesh_size,
                   int* precision, int* method);

/* Copies the real-space potential of the last force solve (pure PM, FP64 or
 * FP32 widened to double, row-major (ix*N+iy)*N+iz, including the 1/N^3 of the
 * inverse transform) to host memory phi[N^3]. Diagnostic / parity access. */
int hyowon_pm_download_potential(hyowon_pm_t h, double* phi);

/* Copies the deposited CIC mass mesh of the last force solve (mass per cell,
 * before density normalisation; FP32_FIXED converts its fixed-point cells to
 * mass) to host memory mesh[N^3]. */
int hyowon_pm_download_mass_mesh(hyowon_pm_t h, double* mesh);

/* Per-axis cell assignment of the device positions: base[3*n] (int64, axis-major:
 * x block then y then z) and frac[3*n] in original particle order, computed by
 * the same device function the sort key uses (src/mesh/cic_coordinate.hpp:95-121). */
int hyowon_pm_cell_coords(hyowon_pm_t h, int64_t* base, double* frac);

/* Particles are permuted into cell order every `steps` KDK steps (default 4);
 * between re-sorts the drift is published by swapping candidate buffers. The
 * sort only serves memory locality: results do not depend on the interval
 * beyond floating-point summation order. */
int hyowon_pm_set_sort_interval(hyowon_pm_t h, int steps);

/* Device timing, measured with CUDA events on the handle's stream. When
 * enabled, times[0] is the device time of the whole last hyowon_pm_run /
 * kdk_step / compute_forces call; times[1..6] the phases summed over the force
 * solves of that call: kick/drift + sort, deposit (with fill / conversion),
 * forward FFT, Green, inverse FFT, gather (+K2), in milliseconds; times[7] the
 * kernels this library launched during the call (cuFFT's own excluded);
 * times[8] the number of force solves timed. times has 9 entries. */
int hyowon_pm_set_timing(hyowon_pm_t h, int enabled);
int hyowon_pm_last_timing(hyowon_pm_t h, double* times);

/* Global diagnostics of the device state at the last force solve, reduced in
 * binary64 in both arithmetic forms, deterministic run to run (fixed
 * reduction order with compensated partial sums).
 *   potential_energy_comoving  0.5 sum_i m_i phi(x_i), phi CIC-interpolated from
 *       the potential mesh of the last force solve: PMForceDiagnostics of
 *       PMSolver::compute_forces(..., collect_potential_energy = true)
 *       (include/cosmo_nbody/gravity/pm_solver.hpp:30-35,
 *       src/gravity/pm_solver.cpp:812-840, per-particle arithmetic of
 *       src/mesh/mass_assignment_gather.inc:283-391). Pure PM only; NaN for
 *       HYOWON_TREEPM_LONG_RANGE, whose solve keeps no real-space potential.
 *   kinetic_energy  sum_i 0.5 m_i |p_i|^2 / a^2
 *       (ConservationChecks::compute_kinetic_energy,
 *       src/validation/conservation_checks.cpp:589-625,1376-1480).
 *   momentum  sum_i m_i p_i.
 *   mass_weighted_force  sum_i m_i a_i;  force_norm_sum  sum_i m_i |a_i|;
 *   force_balance  |sum_i m_i a_i| / sum_i m_i |a_i|, the force-balance
 *       residual R_F (include/cosmo_nbody/validation/force_balance_diagnostics.hpp:19-27).
 *   momentum_force_contraction  sum_i m_i p_i . a_i
 *       (ConservationChecks::compute_momentum_force_contraction,
 *       include/cosmo_nbody/validation/conservation_checks.hpp).
 *   directional_potential_energy_comoving  sum_i m_i p_i . grad_S phi(x_i), the
 *       derivative of the CIC particle-position energy along the momenta with
 *       the one-sided CIC-weight gradient (PMPostForceEnergyDiagnostics of
 *       PMSolver::measure_post_force_energy_diagnostics_in_place,
 *       src/gravity/pm_post_force_energy_diagnostics.cpp:17-100,
 *       src/mesh/mass_assignment_directional.cpp:12-194); NaN for TreePM.
 * a is the scale factor of the state (finite, > 0). HYOWON_ELOGIC when no
 * force solve is valid for the current positions; HYOWON_EOVERFLOW for a
 * non-finite sum; HYOWON_EUNDERFLOW when a non-zero CIC product is lost
 * (the reference's std::underflow_error). */
typedef struct hyowon_pm_diagnostics {
    double potential_energy_comoving;
    double kinetic_energy;
    double momentum[3];
    double mass_weighted_force[3];
    double force_norm_sum;
    double force_balance;
    double momentum_force_contraction;
    double directional_potential_energy_comoving;
} hyowon_pm_diagnostics_t;
int hyowon_pm_diagnostics(hyowon_pm_t h, double a, hyowon_pm_diagnostics_t* out);

/* Matter power spectrum of the device particle state, the estimator of
 * analysis::MatterPowerSpectrum::compute_pk (src/analysis/matter_power_spectrum.cpp:50-226,
 * include/cosmo_nbody/analysis/matter_power_spectrum.hpp:16-60) over
 * FourierDensityBuilder::build (src/analysis/fourier_density_field.cpp:110-376):
 * CIC density contrast on its own mesh of side mesh_size (0: the handle's
 * mesh), r2c / N^3, optional interlacing, CIC-window deconvolution,
 * optional aliased shot-noise subtraction, num_bins logarithmic bins from
 * 2 pi / L to max_k_fraction_nyquist * pi N / L. Binary64 in both arithmetic
 * forms (the precision form's fixed-point positions are widened exactly).
 * bins[num_bins] receives PowerSpectrumBin's fields. 1 <= num_bins <= 256;
 * max_k_fraction_nyquist in (0, 1]; interlaced together with
 * subtract_shot_noise is rejected (HYOWON_EINVAL), as the reference does.
 * Allocates its meshes and transform plan for the call. */
typedef struct hyowon_pk_bin {
    double k_low;
    double k_mean;
    double k_high;
    double p_raw;
    double p_corrected;
    double mean_cic_power_deconvolution_factor;
    double shot_noise_reference;
    uint64_t mode_count;
} hyowon_pk_bin_t;
int hyowon_pm_power_spectrum(hyowon_pm_t h, uint64_t mesh_size, int num_bins,
                             double max_k_fraction_nyquist, int subtract_shot_noise,
                             int interlaced, hyowon_pk_bin_t* bins);

#ifdef __cplusplus
}
#endif
#endif
