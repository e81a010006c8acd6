/*
 * hyowon_debug.h -- failure injection for tests of the error paths.
 *
 * No counterpart in the reference. These calls make the handle's own bounded
 * checks fail from the host, so that tests can see a failure reported as a
 * status code and the handle stay usable afterwards, without faulting, trapping
 * or hanging a GPU: a pipeline wait that is given zero polls returns an error
 * status (after draining its own copies in flight), and a mass-conservation
 * check that is given a wrong target reports a violation.
 */
#ifndef HYOWON_DEBUG_H
#define HYOWON_DEBUG_H

#include "hyowon_pm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Polls of each pipeline wait in the column passes of the five-pass potential
 * solve (power-of-two meshes) before a block gives up and the solve fails with
 * HYOWON_ERUNTIME ("pipeline wait timed out"). 0 makes every wait give up at
 * once; HYOWON_DEBUG_DEFAULT_WAIT restores the default. */
#define HYOWON_DEBUG_DEFAULT_WAIT 16777216u
int hyowon_pm_debug_set_wait_limit(hyowon_pm_t h, unsigned polls);

/* Moves the CIC mass-conservation target of the force solves: the binary64
 * form compares the deposited mass with input_mass + delta (the reference's
 * bound around the exact input mass, src/math/cic_mass_conservation.cpp:41-59),
 * the precision form its exact fixed-point mesh sum with the expected sum
 * plus delta units. 0 restores the exact target. */
int hyowon_pm_debug_offset_mass_target(hyowon_pm_t h, double delta);

#ifdef __cplusplus
}
#endif
#endif
