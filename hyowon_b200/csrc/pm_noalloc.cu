// pm_noalloc.cu -- CIC mass deposit that allocates nothing.
//
// hyowon_cic_deposit_noalloc deposits particles given as DEVICE arrays into a
// caller-owned DEVICE mass mesh, the same operation as the handle's binary64
// deposit (CICMassAssignment::deposit, src/mesh/mass_assignment_deposit.inc:
// 193-240: each particle adds m*wx*wy*wz, in that product order, to its 8
// cells). Its one piece of scratch -- an integer accumulation mesh plus a small
// header -- is the file-scope device array g_noalloc_scratch below, so the call
// never allocates device memory: no cudaMalloc / cudaFree, no allocating
// library routine. Accumulation is in 64-bit fixed point (2^S units, S chosen
// per call from n * max mass), which also makes the result independent of the
// order in which atomics land: two calls on the same input give the same bits.
//
// Set-up: the first call on each device (and again after the device's driver
// context changes, e.g. after cudaDeviceReset) resolves the scratch address
// with cudaGetSymbolAddress, with that device current; this can load the
// module and so may allocate inside the driver. The call is synchronous and
// reads a status word back, so it refuses a capturing stream (HYOWON_EINVAL).
//
// Zeroing: the header and the first N^3 accumulation cells must start at zero;
// every call zeroes them itself as its first kernel, so nothing is required of
// the caller and scratch contents after a call are unspecified.
//
// Overlap: the scratch is one per device and process. Two calls whose device
// work overlapped would race on it, so calls are serialised per device by a
// lock held until the call's work has finished (the call is synchronous).
// Work the caller itself enqueues that touches the output mesh meanwhile races
// as any other stream-ordered access would.
#include "hyowon_noalloc.h"
#include "hyowon_pm.h"
#include "pm_common.cuh"

#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <mutex>

namespace hyowon {
namespace {

constexpr int kMaxMesh = HYOWON_NOALLOC_MAX_MESH;
static_assert(kMaxMesh <= 1024, "cell indices are 32-bit");
constexpr uint64_t kMaxCells = static_cast<uint64_t>(kMaxMesh) * kMaxMesh * kMaxMesh;
// Header words before the cells: [0] status bits, [1] max particle mass (bits
// of a non-negative double), the rest padding so the cells start 256 B in.
constexpr uint64_t kHeaderWords = 32;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kHeaderWords + kMaxCells];

__device__ __forceinline__ uint32_t cell_of(int ix, int iy, int iz, int N) {
    return (static_cast<uint32_t>(ix) * static_cast<uint32_t>(N) + static_cast<uint32_t>(iy))
               * static_cast<uint32_t>(N) + static_cast<uint32_t>(iz);
}

__global__ void k_na_zero(unsigned long long* scratch, uint32_t cells) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kHeaderWords + cells) scratch[i] = 0ull;
}

// Validates masses (finite, >= 0) and records their maximum.
__global__ void k_na_max_mass(uint32_t n, const double* __restrict__ mass,
                              unsigned long long* scratch) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long bits = 0ull;
    if (i < n) {
        const double m = mass[i];
        if (!(isfinite(m) && m >= 0.0)) {
            atomicOr(&scratch[0], static_cast<unsigned long long>(ST_NONFINITE_INPUT));
        } else {
            bits = static_cast<unsigned long long>(__double_as_longlong(m + 0.0));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, bits, o);
        bits = other > bits ? other : bits;
    }
    if ((threadIdx.x & 31) == 0 && bits != 0ull) atomicMax(&scratch[1], bits);
}

// Fixed-point exponent S: n * max_mass * 2^S < 2^61, so the sum of all
// contributions (each particle's 8 weights sum to one) and every cell stay
// below 2^61 with room for the rounding of 8n contributions.
__device__ __forceinline__ int fixed_exponent(uint32_t n, double max_mass) {
    int e = 0;
    frexp(static_cast<double>(n) * max_mass, &e);
    return 61 - e;
}

__global__ void k_na_deposit(uint32_t n, const double* __restrict__ x,
                             const double* __restrict__ y, const double* __restrict__ z,
                             const double* __restrict__ mass, double uniform_mass, Axis a,
                             unsigned long long* scratch) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || scratch[0] != 0ull) return;
    // Cell assignment first: a non-finite position is an error whatever the masses.
    int ix, iy, iz;
    double tx, ty, tz;
    if (!(cic_coord_f64(x[i], a, ix, tx) & cic_coord_f64(y[i], a, iy, ty)
          & cic_coord_f64(z[i], a, iz, tz))) {
        atomicOr(&scratch[0], static_cast<unsigned long long>(ST_CELL_ESCAPE));
        return;
    }
    const double max_mass = mass ? __longlong_as_double(static_cast<long long>(scratch[1]))
                                 : uniform_mass;
    if (!(max_mass > 0.0)) return;  // all-zero masses: the mesh stays zero
    if (!isfinite(static_cast<double>(n) * max_mass)) {
        // the fixed-point exponent needs a finite total-mass bound
        atomicOr(&scratch[0], static_cast<unsigned long long>(ST_NONFINITE_INPUT));
        return;
    }
    const int S = fixed_exponent(n, max_mass);
    const double m = mass ? mass[i] : uniform_mass;
    const double wx[2] = {1.0 - tx, tx};
    const double wy[2] = {1.0 - ty, ty};
    const double wz[2] = {1.0 - tz, tz};
    const int N = a.N;
    const int gy[2] = {iy, iy + 1 == N ? 0 : iy + 1};
    const int gz[2] = {iz, iz + 1 == N ? 0 : iz + 1};
    unsigned long long* cells = scratch + kHeaderWords;
#pragma unroll
    for (int ox = 0; ox < 2; ++ox) {
        const int gx = ox == 0 ? ix : (ix + 1 == N ? 0 : ix + 1);
        const double mx = m * wx[ox];
#pragma unroll
        for (int oy = 0; oy < 2; ++oy) {
            const double mxy = mx * wy[oy];
#pragma unroll
            for (int oz = 0; oz < 2; ++oz) {
                // ldexp by a power of two is exact; rounding to the nearest
                // integer is the only quantisation.
                const long long q = llrint(ldexp(mxy * wz[oz], S));
                atomicAdd(&cells[cell_of(gx, gy[oy], gz[oz], N)],
                          static_cast<unsigned long long>(q));
            }
        }
    }
}

// Fixed point -> mass; writes nothing when an earlier kernel raised a status.
__global__ void k_na_to_mesh(uint32_t n, uint32_t cells_n, const double* __restrict__ mass,
                             double uniform_mass, const unsigned long long* scratch,
                             double* __restrict__ mesh) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells_n || scratch[0] != 0ull) return;
    const double max_mass = mass ? __longlong_as_double(static_cast<long long>(scratch[1]))
                                 : uniform_mass;
    if (!(max_mass > 0.0) || n == 0 || !isfinite(static_cast<double>(n) * max_mass)) {
        mesh[c] = 0.0;
        return;
    }
    const int S = fixed_exponent(n, max_mass);
    mesh[c] = ldexp(static_cast<double>(static_cast<long long>(scratch[kHeaderWords + c])), -S);
}

std::mutex g_lock[kMaxDevices];
// Scratch address per device, valid for the driver context it was resolved in
// (a cudaDeviceReset or another context on the device needs a new address).
unsigned long long* g_scratch_ptr[kMaxDevices] = {};
CUcontext g_scratch_ctx[kMaxDevices] = {};
thread_local char g_err[256] = "";

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

// cuMemGetAddressRange through the runtime's driver entry point (no link-time
// dependency on libcuda): the allocation that contains a device pointer.
using AddressRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
using CtxGetCurrentFn = CUresult (*)(CUcontext*);

template <typename F>
F driver_fn(const char* name) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint(name, &f, cudaEnableDefault, &q) != cudaSuccess
        || q != cudaDriverEntryPointSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return reinterpret_cast<F>(f);
}

AddressRangeFn address_range_fn() {
    static AddressRangeFn fn = driver_fn<AddressRangeFn>("cuMemGetAddressRange");
    return fn;
}

CtxGetCurrentFn ctx_get_current_fn() {
    static CtxGetCurrentFn fn = driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
    return fn;
}

// True when [p, p + bytes) is device memory of device `dev` (or managed
// memory) inside one allocation. Another GPU's memory is refused: the kernels
// would read and write it over the peer path, or fault without peer access.
bool device_extent_ok(const void* p, uint64_t bytes, int dev) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) return false;
    if (at.type == cudaMemoryTypeDevice && at.device != dev) return false;
    AddressRangeFn fn = address_range_fn();
    if (!fn) return false;
    CUdeviceptr base = 0;
    size_t size = 0;
    const CUdeviceptr d = reinterpret_cast<CUdeviceptr>(p);
    if (fn(&base, &size, d) != CUDA_SUCCESS) return false;
    return d >= base && bytes <= static_cast<uint64_t>(base + size - d);
}

}  // namespace
}  // namespace hyowon

using namespace hyowon;

extern "C" const char* hyowon_noalloc_last_error(void) { return g_err; }

extern "C" int hyowon_cic_deposit_noalloc(double box_size, uint64_t mesh_size, uint64_t n,
                                          const double* x, const double* y, const double* z,
                                          const double* masses, double uniform_mass,
                                          double* mesh, void* stream) {
    g_err[0] = '\0';
    if (!std::isfinite(box_size) || box_size <= 0.0)
        return fail(HYOWON_EINVAL, "box size must be finite and positive");
    if (mesh_size < 2 || mesh_size > static_cast<uint64_t>(kMaxMesh))
        return fail(HYOWON_EINVAL,
                    "mesh size %llu outside [2, %d]: the static scratch holds at most %d^3 cells",
                    static_cast<unsigned long long>(mesh_size), kMaxMesh, kMaxMesh);
    if (n >= (1ull << 32)) return fail(HYOWON_EINVAL, "particle count must be below 2^32");
    if (!masses && !(std::isfinite(uniform_mass) && uniform_mass >= 0.0
                     && std::isfinite(static_cast<double>(n) * uniform_mass)))
        return fail(HYOWON_EINVAL,
                    "uniform mass must be finite and non-negative, with n * mass finite");
    if (!mesh || (n > 0 && (!x || !y || !z)))
        return fail(HYOWON_EINVAL, "null position or mesh pointer");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return fail(HYOWON_ECUDA, "no usable current CUDA device");
    }
    const uint64_t pbytes = n * sizeof(double);
    const uint64_t mbytes = mesh_size * mesh_size * mesh_size * sizeof(double);
    if (!device_extent_ok(mesh, mbytes, dev))
        return fail(HYOWON_EINVAL,
                    "mesh must be device memory of the current device (%d), at least %llu bytes",
                    dev, static_cast<unsigned long long>(mbytes));
    if (n > 0 && (!device_extent_ok(x, pbytes, dev) || !device_extent_ok(y, pbytes, dev)
                  || !device_extent_ok(z, pbytes, dev)
                  || (masses && !device_extent_ok(masses, pbytes, dev))))
        return fail(HYOWON_EINVAL,
                    "positions and masses must be device memory of the current device (%d), "
                    "at least %llu bytes each",
                    dev, static_cast<unsigned long long>(pbytes));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        cudaGetLastError();
        return fail(HYOWON_EINVAL, "stream is not usable on the current device");
    }
    if (cap != cudaStreamCaptureStatusNone)
        return fail(HYOWON_EINVAL,
                    "the call waits for its own work and reads a status word back, so it "
                    "cannot be issued on a capturing stream");

    std::lock_guard<std::mutex> guard(g_lock[dev]);
    CUcontext ctx = nullptr;
    CtxGetCurrentFn get_ctx = ctx_get_current_fn();
    if (!get_ctx || get_ctx(&ctx) != CUDA_SUCCESS || !ctx)
        return fail(HYOWON_ECUDA, "no current CUDA context on device %d", dev);
    if (!g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(HYOWON_ECUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
        }
        g_scratch_ptr[dev] = static_cast<unsigned long long*>(p);
        g_scratch_ctx[dev] = ctx;
    }
    unsigned long long* scratch = g_scratch_ptr[dev];

    const int N = static_cast<int>(mesh_size);
    const uint32_t cells = static_cast<uint32_t>(mesh_size * mesh_size * mesh_size);
    const uint32_t nn = static_cast<uint32_t>(n);
    Axis a;
    a.L = box_size;
    a.dx = box_size / static_cast<double>(N);
    a.upper = std::nextafter(static_cast<double>(N), 0.0);
    a.N = N;
    constexpr uint64_t T = 256;
    // block counts in 64 bits: n may be as large as 2^32 - 1
    const unsigned zero_blocks = static_cast<unsigned>((kHeaderWords + cells + T - 1) / T);
    const unsigned particle_blocks = static_cast<unsigned>((n + T - 1) / T);
    const unsigned cell_blocks = static_cast<unsigned>((static_cast<uint64_t>(cells) + T - 1) / T);
    k_na_zero<<<zero_blocks, T, 0, s>>>(scratch, cells);
    if (nn > 0) {
        if (masses) k_na_max_mass<<<particle_blocks, T, 0, s>>>(nn, masses, scratch);
        k_na_deposit<<<particle_blocks, T, 0, s>>>(nn, x, y, z, masses, uniform_mass, a, scratch);
    }
    k_na_to_mesh<<<cell_blocks, T, 0, s>>>(nn, cells, masses, uniform_mass, scratch, mesh);
    unsigned long long status = 0ull;
    cudaError_t e = cudaMemcpyAsync(&status, scratch, sizeof(status), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(HYOWON_ECUDA, "deposit launch: %s", cudaGetErrorString(e));
    }
    if (status & ST_NONFINITE_INPUT)
        return fail(HYOWON_EINVAL,
                    "particle masses must be finite and non-negative, with n * max mass finite");
    if (status & ST_CELL_ESCAPE)
        return fail(HYOWON_ELOGIC, "non-finite position: CIC cell assignment left the mesh");
    return HYOWON_OK;
}
