// pm_common.cuh -- device-side definitions shared by the PM kernels.
//
// The FP64 functions here restate the reference's scalar arithmetic in the same
// operation order; translation units that include them for the FP64 form are
// compiled with --fmad=false so no product is contracted into an FMA, which is
// what makes cell assignment, CIC weights, the gradient stencil and the KDK
// update bit-identical to the reference (built with -ffp-contract=off,
// CMakeLists.txt:47-51).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hyowon {

// Device status word bits. Kernels OR these into one device word; the host
// maps them to the C status codes of hyowon_pm.h.
enum StatusBits : unsigned int {
    ST_NONFINITE_INPUT = 1u << 0,  // non-finite position / mass      -> EINVAL
    ST_CELL_ESCAPE = 1u << 1,      // cell assignment left the mesh   -> ELOGIC
    ST_KICK_DRIFT = 1u << 2,       // non-finite K1/drift candidate   -> EOVERFLOW
    ST_FORCE = 1u << 3,            // non-finite force                -> EOVERFLOW
    ST_KICK2 = 1u << 4,            // non-finite K2 candidate         -> EOVERFLOW
    ST_MASS = 1u << 5,             // CIC mass conservation violated  -> ERUNTIME
    ST_CAPACITY = 1u << 6,         // fixed-point cell capacity       -> ERUNTIME
    ST_UNDERFLOW = 1u << 7,        // lost non-zero product           -> EUNDERFLOW
    ST_PIPELINE = 1u << 8,         // a bounded device wait timed out -> ERUNTIME
};

// Kernels that publish state check this mask first and skip all writes when a
// preceding stage of the same step failed (transactional publication, as
// LeapfrogIntegrator's preflight/publish passes,
// src/time/leapfrog_integrator.cpp:170-225).
constexpr unsigned int ST_BLOCKS_PUBLISH =
    ST_NONFINITE_INPUT | ST_CELL_ESCAPE | ST_KICK_DRIFT;

struct Axis {
    double L;      // box size
    double dx;     // L / N, formed as MeshGeometry does (mesh_geometry.hpp:44)
    double upper;  // nextafter(N, 0)  (cic_coordinate.hpp:92)
    int N;
};

// math::wrap (include/cosmo_nbody/math/periodic_box.hpp:27-41). fmod is exact.
__device__ __forceinline__ double wrap_f64(double x, double L) {
    if (!isfinite(x)) return __longlong_as_double(0x7ff8000000000000ll);
    if (x >= 0.0 && x < L) return x;
    double w = fmod(x, L);
    if (w < 0.0) w += L;
    if (w >= L) w = 0.0;
    return w == 0.0 ? 0.0 : w;
}

// math::minimum_image (periodic_box.hpp:44-61). remainder is exact.
__device__ __forceinline__ double minimum_image_f64(double d, double L) {
    if (!isfinite(d)) return __longlong_as_double(0x7ff8000000000000ll);
    const double half = 0.5 * L;
    if (d >= -half && d < half) return d;
    double w = remainder(d, L);
    if (w >= half) w -= L;
    else if (w < -half) w += L;
    return w == 0.0 ? 0.0 : w;
}

// CICCoordinateAxis::operator() (src/mesh/cic_coordinate.hpp:95-121): wrap,
// divide, clamp to [0, nextafter(N,0)], floor, subtract. Returns false where
// the reference throws.
__device__ __forceinline__ bool cic_coord_f64(double pos, const Axis& a, int& base,
                                              double& frac) {
    const double w = wrap_f64(pos, a.L);
    if (!(w >= 0.0 && w < a.L)) return false;
    double s = w / a.dx;
    if (!isfinite(s)) return false;
    s = s < 0.0 ? 0.0 : (a.upper < s ? a.upper : s);
    const double fl = floor(s);
    const int b = static_cast<int>(fl);
    if (b < 0 || b >= a.N) return false;
    // frac = scaled - (double)base, as the reference forms it: for scaled = -0.0
    // this keeps the sign (-0.0 - +0.0), which `s - floor(s)` would not.
    const double f = s - static_cast<double>(b);
    if (!(f >= 0.0 && f < 1.0)) return false;
    base = b;
    frac = f;
    return true;
}

__device__ __forceinline__ int wrap_index(int i, int N) {
    i %= N;
    return i < 0 ? i + N : i;
}

// Rank of this particle inside its bucket with one atomic per group of lanes
// that share the bucket (sorted particles share buckets ~8-way).
__device__ __forceinline__ uint32_t bucket_rank(uint32_t* count, uint32_t b) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, b);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&count[b], static_cast<uint32_t>(__popc(peers)));
    base = __shfl_sync(peers, base, leader);
    return base + static_cast<uint32_t>(__popc(peers & ((1u << lane) - 1u)));
}

__device__ __forceinline__ void raise_status(unsigned int* status, unsigned int bits) {
    atomicOr(status, bits);
}

// Block-wide maximum of non-negative 64-bit values folded into *out with one
// atomic per block (not per warp: a single address serialises its atomics).
// Every thread of the block calls it; blockDim.x is a multiple of 32.
__device__ __forceinline__ void block_max_to(unsigned long long v, unsigned long long* out) {
    __shared__ unsigned long long part[32];
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (lane == 0) part[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < static_cast<int>(blockDim.x >> 5) ? part[lane] : 0ull;
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
            v = w > v ? w : v;
        }
        if (lane == 0 && v != 0ull) atomicMax(out, v);
    }
}

// Block-wide sum modulo 2^64 folded into *out with one atomic per block.
__device__ __forceinline__ void block_sum_to(unsigned long long v, unsigned long long* out) {
    __shared__ unsigned long long part[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (lane == 0) part[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < static_cast<int>(blockDim.x >> 5) ? part[lane] : 0ull;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && v != 0ull) atomicAdd(out, v);
    }
}

// Blocks of `threads` for a grid-stride pass over n items: enough to fill
// every SM with resident blocks, never more than the items need.
inline unsigned stream_blocks(uint64_t n, int threads) {
    static int sms = [] {
        int dev = 0, v = 148;
        if (cudaGetDevice(&dev) != cudaSuccess
            || cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            v = 148;
        return v;
    }();
    const uint64_t need = (n + threads - 1) / threads;
    const uint64_t fill = static_cast<uint64_t>(sms) * (2048 / threads);
    return static_cast<unsigned>(need < fill ? (need ? need : 1) : fill);
}

}  // namespace hyowon
