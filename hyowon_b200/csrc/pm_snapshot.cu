// pm_snapshot.cu -- /PartType1 snapshot payload staging on the device.
//
// The reference's snapshot writer stages each vector dataset as rows of
// three binary64 values in particle order: Coordinates (x, y, z) and
// Velocities (px, py, pz) * (1 / a), the peculiar velocity of the canonical
// momentum p = a^2 dx/dt (write_vector_dataset_batched,
// src/io/snapshot_io_particle_helpers.inc:116-200), after validating the
// payload (require_finite_particle_payload, :48-104: finite phase-space
// fields, coordinates in [0, L), finite velocities). Here one kernel per
// dataset reads the device state in its sorted slots and writes row id[j]
// (the slot's original particle index) of a device staging array, raising
// flags instead of throwing; the host copies a dataset only when no flag is
// set. Coordinates are the stored values (widened exactly from the
// fixed-point form); velocities are p * inv_a with inv_a = 1 / a formed on
// the host, the reference's arithmetic.
#include "pm_snapshot.h"

#include "pm_common.cuh"

namespace hyowon {
namespace snapshot {

namespace {

__device__ __forceinline__ double value(const Component& c, uint32_t j) {
    switch (c.kind) {
        case kF64: return static_cast<const double*>(c.p)[j];
        case kF32: return static_cast<double>(static_cast<const float*>(c.p)[j]);
        default: return static_cast<double>(static_cast<const uint32_t*>(c.p)[j]) * c.scale;
    }
}

__global__ void k_rows(uint32_t n, const uint32_t* __restrict__ id, Component c0, Component c1,
                       Component c2, int velocity, double inv_a, double L,
                       double* __restrict__ rows, unsigned int* flag) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double v[3] = {value(c0, j), value(c1, j), value(c2, j)};
    const uint64_t r = 3ull * id[j];
    unsigned int bad = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (!isfinite(v[d])) bad |= kNonFinite;
        double out = v[d];
        if (velocity) {
            out = v[d] * inv_a;
            if (isfinite(v[d]) && !isfinite(out)) bad |= kVelocityOverflow;
        } else if (!(v[d] >= 0.0 && v[d] < L)) {
            bad |= kOutsideBox;
        }
        rows[r + d] = out;
    }
    if (bad) atomicOr(flag, bad);
}

}  // namespace

int launch_rows(uint32_t n, const uint32_t* id, const Component (&c)[3], bool velocity,
                double inv_a, double L, double* rows, unsigned int* flag, cudaStream_t s) {
    if (n == 0) return 0;
    k_rows<<<(n + 255) / 256, 256, 0, s>>>(n, id, c[0], c[1], c[2], velocity ? 1 : 0, inv_a, L,
                                           rows, flag);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

}  // namespace snapshot
}  // namespace hyowon
