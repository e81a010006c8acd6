// pm_snapshot.h -- snapshot payload staging (internal; see pm_snapshot.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hyowon {
namespace snapshot {

enum Kind : int { kF64 = 0, kF32 = 1, kFixedU32 = 2 };

// One per-particle component in sorted slots: binary64, FP32, or u32 fixed
// point (value = u * scale).
struct Component {
    const void* p;
    int kind;
    double scale;
};

// Flag bits of a staging pass.
enum Flags : unsigned int {
    kNonFinite = 1u << 0,         // a non-finite position or momentum
    kOutsideBox = 1u << 1,        // a coordinate outside [0, L)
    kVelocityOverflow = 1u << 2,  // p * (1 / a) not finite
};

// rows[3 id[j] + d] = c[d](j) (coordinates) or c[d](j) * inv_a (velocity),
// for the n sorted slots j. Returns the kernels launched (1) or -1.
int launch_rows(uint32_t n, const uint32_t* id, const Component (&c)[3], bool velocity,
                double inv_a, double L, double* rows, unsigned int* flag, cudaStream_t s);

}  // namespace snapshot
}  // namespace hyowon
