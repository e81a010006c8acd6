/*
 * hyowon_noalloc.h -- an entry point that allocates no device memory.
 *
 * No counterpart in the reference: HYOWON's deposit
 * (CICMassAssignment::deposit, src/mesh/mass_assignment_deposit.inc:15-334)
 * runs on host memory it manages itself. This entry serves device-side callers
 * that own all of their device memory and must not have a library allocate:
 * a host that has handed the GPU's memory to its own pool or budget (a
 * framework caching allocator, a fixed memory policy), where a cudaMalloc
 * would fail or would synchronise the device and stall the caller's streams.
 */
#ifndef HYOWON_NOALLOC_H
#define HYOWON_NOALLOC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Largest mesh side the static scratch holds: 64^3 cells of 8 bytes (2 MiB),
 * plus a 256-byte header. */
#define HYOWON_NOALLOC_MAX_MESH 64

/* CIC mass deposit of n particles into mesh[mesh_size^3] (row-major
 * (ix*N+iy)*N+iz, mass per cell; overwritten), the same operation as the PM
 * handle's binary64 deposit (each particle adds m*wx*wy*wz to its 8 cells),
 * accumulated in 64-bit fixed point in a static device scratch array, so the
 * result does not depend on atomic ordering and agrees with the binary64
 * deposit to about n * 2^-61 relative to the total mass.
 *
 * x, y, z (n each), masses (n, or NULL for uniform_mass) and mesh are DEVICE
 * pointers of the current device (another GPU's memory is refused); stream is
 * a cudaStream_t of that device (NULL: the legacy default stream). The call
 * allocates nothing, enqueues its kernels on stream and waits for them; it
 * returns HYOWON_OK, HYOWON_EINVAL (mesh_size outside
 * [2, HYOWON_NOALLOC_MAX_MESH], n >= 2^32, host, peer or too-small buffers, a
 * non-finite or negative mass, n * max mass not finite, a capturing stream),
 * HYOWON_ELOGIC (a non-finite position, whatever the masses) or HYOWON_ECUDA.
 * On an error the mesh is not written. The first call on a device (and the
 * first after its driver context changes, e.g. after cudaDeviceReset) resolves
 * the scratch address with that device current. The call is synchronous and
 * reads a status word back, so it cannot be issued on a stream that is being
 * captured. Calls on one device are serialised: they share the scratch.
 */
int hyowon_cic_deposit_noalloc(double box_size, uint64_t mesh_size, uint64_t n,
                               const double* x, const double* y, const double* z,
                               const double* masses, double uniform_mass, double* mesh,
                               void* stream);

/* Message of the calling thread's last failing hyowon_cic_deposit_noalloc. */
const char* hyowon_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
