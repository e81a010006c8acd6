/*
 * hyowon_treepm.h -- C ABI of the TreePM short-range force on the device.
 *
 * Pair acceleration of a target from a source of mass m at minimum-image
 * displacement dx = x_source - x_target, r = |dx|, q = r / r_s
 * (include/cosmo_nbody/gravity/force_split.hpp:1-6,
 *  src/gravity/force_split_stable_ratio.cpp:150-196):
 *   a = G m dx [ (r^2 + eps^2)^(-3/2) - (1 - M_S(q)) / r^3 ],
 *   M_S(q) = erfc(q/2) + q/sqrt(pi) exp(-q^2/4),
 * summed over sources with r < r_cut. Distant groups within the cutoff are
 * replaced by monopoles of octree nodes accepted by the modified Barnes-Hut
 * criterion r > l/theta + |COM - centre|_1 when the node neither contains the
 * target nor straddles the cutoff sphere (src/gravity/tree_walk.cpp:75-126,
 * 203-464). The octree covers [0, L)^3 and subdivides until one source per leaf
 * (src/gravity/octree.cpp:169-440); here it is built from 63-bit Morton keys
 * (21 bits per axis, x most significant), so coincident sources at that
 * resolution share an exact-pair leaf.
 */
#ifndef HYOWON_TREEPM_H
#define HYOWON_TREEPM_H

#include <stdint.h>

#include "hyowon_pm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hyowon_treepm_params {
    double box_size;       /* L */
    double split_scale;    /* r_s */
    double cutoff;         /* r_cut < L/2 */
    double softening;      /* Plummer eps */
    double theta;          /* opening angle (> 0) */
    double particle_mass;  /* uniform source mass */
    int precision;         /* HYOWON_FP64 or HYOWON_FP32_FIXED (FP32 pair and
                              monopole arithmetic, binary64 positions / tree) */
} hyowon_treepm_params;

/* Short-range accelerations at n_targets target particles (indices into the
 * n sources; the target itself is excluded) from all n sources, written to
 * ax/ay/az[n_targets]. Positions are host arrays, wrapped to [0, L) on entry.
 * stats (may be NULL) receives {tree nodes, max depth, node visits per target,
 * exact pairs per target, build ms, walk ms}. Returns a hyowon_status code. */
int hyowon_treepm_short_forces(const hyowon_treepm_params* params, uint64_t n,
                               const double* x, const double* y, const double* z,
                               uint64_t n_targets, const uint32_t* targets, double* ax,
                               double* ay, double* az, double* stats);

const char* hyowon_treepm_last_error(void);

/* ---- TreePM on a PM handle ------------------------------------------------
 * The handle must be created with HYOWON_TREEPM_LONG_RANGE (its split_scale is
 * r_s). Sources are the handle's device-resident particles with their masses
 * (per-particle in the binary64 form, uniform in the precision form); the
 * short-range sum is the same as hyowon_treepm_short_forces's. */
/* Makes every force solve of the handle (compute_forces, kdk_step, run) the
 * TreePM force of TreePMSolver::compute_forces (src/gravity/treepm_solver.cpp:
 * 631-717): the PM long range (Gaussian split at r_s, spectral -ik) plus the
 * octree short range with opening angle theta, Plummer softening and cutoff
 * r_cut < L/2, summed per particle before the K2 kick. cutoff = 0 returns the
 * handle to the long range alone. HYOWON_EINVAL for a pure-PM handle or
 * invalid parameters. Invalidates the current accelerations. */
int hyowon_pm_set_treepm_short_range(hyowon_pm_t h, double theta, double softening,
                                     double cutoff);

/* The short-range accelerations of every particle of the handle's current
 * state (TreeWalk::compute_force per target, src/gravity/tree_walk.cpp:
 * 203-464, on Octree::build of all sources, src/gravity/octree.cpp:169-440),
 * written to host ax/ay/az[n] in the caller's original particle order (any may
 * be NULL). stats as hyowon_treepm_short_forces (may be NULL). Leaves the
 * handle's accelerations untouched. */
int hyowon_pm_treepm_short_forces(hyowon_pm_t h, double theta, double softening,
                                  double cutoff, double* ax, double* ay, double* az,
                                  double* stats);

#ifdef __cplusplus
}
#endif
#endif
