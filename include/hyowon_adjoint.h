/*
 * hyowon_adjoint.h -- C ABI of the differentiation form: the gradient of a
 * scalar loss on the final density field with respect to the initial
 * white-noise field, through first-order LPT and n KDK PM steps.
 *
 * Forward model: noise w (n_side^3, lattice order) -> 1LPT (as
 * hyowon_pm_lpt_ics) -> n_steps KDK steps with the pure-PM force on a
 * mesh_size^3 mesh (as hyowon_pm_kdk_step, particles kept in lattice order)
 * -> CIC density contrast delta = M / Mbar - 1 on the same mesh ->
 * L = 1/2 sum_cells (delta - target)^2.
 * Reverse pass: reverse leapfrog (the KDK step run backwards reconstructs the
 * trajectory) with position / momentum checkpoints every ckpt_every steps;
 * when device memory allows, the forward pass also keeps the potential mesh
 * of every state (n_steps + 1 meshes), so the reverse pass re-derives each
 * state's force by a gather instead of a deposit and a Green's-function solve;
 * hand-written adjoints of the gather (CIC scatter of the force cotangent),
 * of the deposit (gather with the CIC weight derivative), of the centred
 * gradient (centred divergence), of the Green's function (self-adjoint) and of
 * the 1LPT map. The reference code has no adjoint: this is new functionality
 * built on its discretisation (src/gravity/pm_solver.cpp:569-852,
 * src/time/leapfrog_integrator.cpp:143-279, src/ic/lpt_displacement.cpp:150-384).
 */
#ifndef HYOWON_ADJOINT_H
#define HYOWON_ADJOINT_H

#include <stdint.h>

#include "hyowon_pm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hyowon_vjp_config {
    double box_size;          /* L, Mpc/h */
    uint64_t n_side;          /* particles per side = IC lattice size */
    uint64_t mesh_size;       /* PM / loss mesh size */
    int precision;            /* HYOWON_FP64 or HYOWON_FP32_FIXED (FP32 meshes,
                                 forces, momenta; binary64 positions) */
    uint64_t n_nodes;         /* P(k) spline at the start epoch (hyowon_pm_lpt_ics) */
    const double* ln_k;
    const double* ln_p;
    const double* ln_p_y2;
    double momentum_factor;   /* a^2 H f1 at the start epoch */
    double particle_mass;
    uint64_t n_steps;         /* KDK steps and their factors */
    const double* K1;
    const double* D;
    const double* K2;
    uint64_t ckpt_every;      /* checkpoint interval of the reverse pass */
} hyowon_vjp_config;

/* Runs the forward model; writes the loss (needs target_delta, else 0 and only
 * final_delta is produced), optionally the final density contrast
 * final_delta[mesh^3] and, when grad_noise != NULL, dL/dw into
 * grad_noise[n_side^3]. timings (may be NULL) receives {forward ms, reverse ms,
 * force solves, force VJPs}. Returns a hyowon_status code. */
int hyowon_vjp_1lpt_pm(const hyowon_vjp_config* cfg, const double* noise,
                       const double* target_delta, double* loss, double* grad_noise,
                       double* final_delta, double* timings);

const char* hyowon_vjp_last_error(void);

/* The same VJP on a PM handle (the drop-in's vjp(handle, ...)): the handle
 * supplies the box, the mesh and the arithmetic form (cfg->box_size,
 * mesh_size and precision are ignored), runs on the handle's stream and keeps
 * the adjoint's FFT plans and work arrays between calls with the same
 * geometry (freed by hyowon_pm_destroy). The handle's particle state is not
 * touched. The handle must use HYOWON_PURE_PM. Errors go to
 * hyowon_pm_last_error(h). */
int hyowon_pm_vjp(hyowon_pm_t h, const hyowon_vjp_config* cfg, const double* noise,
                  const double* target_delta, double* loss, double* grad_noise,
                  double* final_delta, double* timings);

#ifdef __cplusplus
}

namespace hyowon::adj {
using VjpConfig = hyowon_vjp_config;
}
#endif
#endif
