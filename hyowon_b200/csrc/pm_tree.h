// pm_tree.h -- TreePM short-range force on device-resident particles (internal).
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "hyowon_treepm.h"

namespace hyowon::tree {

// Device scratch of the tree build and walk kept between calls (the octree
// nodes, sort buffers and level arrays: a few hundred bytes a particle), so
// that repeated solves of one size allocate nothing.
struct Workspace;
Workspace* create_workspace();
void destroy_workspace(Workspace* ws);

// Octree of the n device sources (x, y, z in [0, L) after wrapping; masses or,
// when null, P.particle_mass) and the short-range walk of every source as a
// target; each source's acceleration is ADDED to ax/ay/az[source] (device).
// Work is ordered on s and finished at return. stats as hyowon_treepm_short_forces.
// ws (may be null: allocate for this call only) holds the scratch.
int device_short_forces(const hyowon_treepm_params& P, uint32_t n, const double* x,
                        const double* y, const double* z, const double* masses, double* ax,
                        double* ay, double* az, cudaStream_t s, double* stats, std::string* err,
                        Workspace* ws = nullptr);

}  // namespace hyowon::tree
