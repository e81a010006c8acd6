// pm_sort.cu -- counting sort of particles by cell bucket.
//
// The reference orders particles with a stable counting sort by base x-plane
// (build_x_plane_bins, src/mesh/mass_assignment_workspace.inc:264-374) so that
// its deposit can own whole planes. Here the key is the full row-major cell
// index of the reference's cell assignment (bit-identical, pm_common.cuh),
// shifted down into buckets of 2^shift consecutive cells, and the particle
// state itself is permuted: afterwards deposit and gather sweep the mesh in
// memory order, so the working set of mesh planes stays in L2 and particle
// reads are coalesced. The rank inside a bucket comes from the atomicAdd that
// built the histogram, so the sort is one histogram pass (fused into the kick /
// drift kernel), one exclusive scan and one scatter.
#include <cuda_runtime.h>

#include "pm_kernels.h"

namespace hyowon {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads)
k_scan_block(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t n,
             uint32_t* __restrict__ block_sums) {
    __shared__ uint32_t warp_tot[kScanThreads / 32];
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        v[j] = base + j < n ? in[base + j] : 0u;
        sum += v[j];
    }
    // Inclusive warp scan of the per-thread totals.
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_tot[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        warp_tot[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    uint32_t run = incl - sum + (warp > 0 ? warp_tot[warp - 1] : 0u);
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        if (base + j < n) out[base + j] = run;
        run += v[j];
    }
    if (threadIdx.x == kScanThreads - 1 && block_sums) block_sums[blockIdx.x] = run;
}

__global__ void k_scan_add(uint32_t* __restrict__ out, uint32_t n,
                           const uint32_t* __restrict__ block_offsets) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] += block_offsets[i / kScanTile];
}

// Permute up to 8 binary64 arrays and 2 u32 arrays in one pass.
struct ScatterArrays {
    const double* src[8];
    double* dst[8];
    const uint32_t* src_u[2];
    uint32_t* dst_u[2];
    int n_f64;
    int n_u32;
};

__global__ void k_scatter(uint32_t n, const uint32_t* __restrict__ key,
                          const uint32_t* __restrict__ rank,
                          const uint32_t* __restrict__ offset, ScatterArrays arr,
                          const unsigned int* status) {
    if (status && (*status & ST_BLOCKS_PUBLISH)) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t d = offset[key[i]] + rank[i];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        if (a < arr.n_f64) arr.dst[a][d] = arr.src[a][i];
    }
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        if (a < arr.n_u32) arr.dst_u[a][d] = arr.src_u[a][i];
    }
}

// Permute up to 8 arrays of 4-byte elements (u32 or float bit patterns).
struct Scatter4 {
    const uint32_t* src[8];
    uint32_t* dst[8];
    int count;
};

__global__ void k_scatter4(uint32_t n, const uint32_t* __restrict__ key,
                           const uint32_t* __restrict__ rank,
                           const uint32_t* __restrict__ offset, Scatter4 arr,
                           const unsigned int* status) {
    if (status && (*status & ST_BLOCKS_PUBLISH)) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t d = offset[key[i]] + rank[i];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        if (a < arr.count) arr.dst[a][d] = arr.src[a][i];
    }
}

__global__ void k_unpermute(uint32_t n, const uint32_t* __restrict__ id,
                            const double* __restrict__ src, double* __restrict__ dst) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[id[i]] = src[i];
}

// Cell order of the particles without moving them: order[offset[key]+rank] = i.
__global__ void k_order(uint32_t n, const uint32_t* __restrict__ key,
                        const uint32_t* __restrict__ rank, const uint32_t* __restrict__ offset,
                        uint32_t* __restrict__ order, const unsigned int* status) {
    if (status && (*status & ST_BLOCKS_PUBLISH)) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    order[offset[key[i]] + rank[i]] = i;
}

__global__ void k_iota(uint32_t n, uint32_t* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = i;
}

inline unsigned blocks_for(uint64_t n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

}  // namespace

size_t scan_tmp_elements(uint32_t n) {
    size_t total = 0;
    uint64_t m = n;
    while (m > 1) {
        const uint64_t b = (m + kScanTile - 1) / kScanTile;
        total += 2 * b + 64;
        m = b;
    }
    return total + 64;
}

int launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp,
                          cudaStream_t s) {
    if (n == 0) return 0;
    const uint32_t nb = static_cast<uint32_t>((static_cast<uint64_t>(n) + kScanTile - 1) / kScanTile);
    if (nb == 1) {
        k_scan_block<<<1, kScanThreads, 0, s>>>(in, out, n, nullptr);
        return 1;
    }
    uint32_t* sums = tmp;
    uint32_t* sums_scanned = tmp + nb + 32;
    k_scan_block<<<nb, kScanThreads, 0, s>>>(in, out, n, sums);
    const int inner = launch_exclusive_scan(sums, sums_scanned, nb, tmp + 2 * nb + 64, s);
    k_scan_add<<<blocks_for(n, 256), 256, 0, s>>>(out, n, sums_scanned);
    return inner + 2;
}

void launch_scatter_f64(uint32_t n, const uint32_t* key, const uint32_t* rank,
                        const uint32_t* offset, const double* src, double* dst,
                        const unsigned int* status, cudaStream_t s) {
    if (n == 0) return;
    ScatterArrays a{};
    a.src[0] = src;
    a.dst[0] = dst;
    a.n_f64 = 1;
    a.n_u32 = 0;
    k_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, key, rank, offset, a, status);
}

void launch_scatter_u32(uint32_t n, const uint32_t* key, const uint32_t* rank,
                        const uint32_t* offset, const uint32_t* src, uint32_t* dst,
                        const unsigned int* status, cudaStream_t s) {
    if (n == 0) return;
    ScatterArrays a{};
    a.src_u[0] = src;
    a.dst_u[0] = dst;
    a.n_f64 = 0;
    a.n_u32 = 1;
    k_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, key, rank, offset, a, status);
}

void launch_scatter_multi(uint32_t n, const uint32_t* key, const uint32_t* rank,
                          const uint32_t* offset, int n_f64, const double* const* src,
                          double* const* dst, int n_u32, const uint32_t* const* src_u,
                          uint32_t* const* dst_u, const unsigned int* status,
                          cudaStream_t s) {
    if (n == 0) return;
    ScatterArrays a{};
    for (int i = 0; i < n_f64; ++i) {
        a.src[i] = src[i];
        a.dst[i] = dst[i];
    }
    for (int i = 0; i < n_u32; ++i) {
        a.src_u[i] = src_u[i];
        a.dst_u[i] = dst_u[i];
    }
    a.n_f64 = n_f64;
    a.n_u32 = n_u32;
    k_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, key, rank, offset, a, status);
}

void launch_scatter4_multi(uint32_t n, const uint32_t* key, const uint32_t* rank,
                           const uint32_t* offset, int count, const uint32_t* const* src,
                           uint32_t* const* dst, const unsigned int* status, cudaStream_t s) {
    if (n == 0) return;
    Scatter4 a{};
    for (int i = 0; i < count; ++i) {
        a.src[i] = src[i];
        a.dst[i] = dst[i];
    }
    a.count = count;
    k_scatter4<<<blocks_for(n, 256), 256, 0, s>>>(n, key, rank, offset, a, status);
}

void launch_unpermute_f64(uint32_t n, const uint32_t* id, const double* src, double* dst,
                          cudaStream_t s) {
    if (n == 0) return;
    k_unpermute<<<blocks_for(n, 256), 256, 0, s>>>(n, id, src, dst);
}

void launch_order(uint32_t n, const uint32_t* key, const uint32_t* rank, const uint32_t* offset,
                  uint32_t* order, const unsigned int* status, cudaStream_t s) {
    if (n == 0) return;
    k_order<<<blocks_for(n, 256), 256, 0, s>>>(n, key, rank, offset, order, status);
}

void launch_iota_u32(uint32_t n, uint32_t* out, cudaStream_t s) {
    if (n == 0) return;
    k_iota<<<blocks_for(n, 256), 256, 0, s>>>(n, out);
}

}  // namespace hyowon
