// pm_tree.cu -- TreePM short-range force: Morton-key octree + warp-cooperative
// walk (include/hyowon_treepm.h).
//
// Build:
//   1. 63-bit Morton key per source (21 bits per axis, x most significant, so
//      the octant of a level-l node is bits 3(21-l)..3(21-l)+2 with x >= centre
//      as bit 2, the reference's octant order, src/gravity/octree.cpp:336-357);
//   2. stable LSD radix sort of (key, index), 8 passes of 8 bits;
//   3. level-wise node extraction: a node at level l is a maximal run of equal
//      key >> 3(21-l) whose parent run holds >= 2 sources; runs holding one
//      source (or level 21) are leaves, so every leaf holds one source unless
//      sources coincide at 2^-21 L;
//   4. node mass and COM from exact 64-bit prefix sums of 2^-40 L fixed-point
//      coordinates (no summation-order error).
// Walk: one warp per 32 targets (sorted by key, so a warp's targets are close).
// The warp traverses a shared depth-first stack; each lane classifies the node
// against its target -- pruned (cube outside the cutoff sphere), leaf (exact
// pairs), monopole (modified Barnes-Hut criterion, not containing the target,
// not straddling the cutoff) or open -- and the node's children are pushed if
// any lane needs them. A lane that pruned or accepted a node records its end
// index and ignores that node's descendants, which follow it contiguously in
// depth-first order. Stack depth and iterations are bounded; overflow is an
// error status, never an unbounded loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "hyowon_pm.h"
#include "hyowon_treepm.h"
#include "pm_common.cuh"
#include "pm_kernels.h"
#include "pm_tree.h"

namespace hyowon::tree {

namespace {

constexpr int kT = 256;
constexpr int kBits = 21;
constexpr int kStack = 192;        // per-warp stack entries (>= 7 * 21 + 8)
constexpr unsigned kMaxIter = 1u << 24;

inline unsigned nb(uint64_t n, int t = kT) { return static_cast<unsigned>((n + t - 1) / t); }

struct Node {
    double cx, cy, cz, half;       // geometric cube
    double mx, my, mz, mass;       // centre of mass, mass
    unsigned long long prefix;     // key >> 3(21-level)
    uint32_t start, end;           // sorted source range
    uint32_t first_child, n_child; // children in the node array
    uint32_t level, leaf;
    double open2;                  // (2 half / theta + |COM - centre|_1)^2, set after the build
};

__device__ __forceinline__ unsigned long long spread3(unsigned v) {
    unsigned long long x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x1f00000000ffffull;
    x = (x | (x << 16)) & 0x1f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

__device__ __forceinline__ unsigned quant(double w, double L) {
    double t = floor(w / L * 2097152.0);
    t = t < 0.0 ? 0.0 : (t > 2097151.0 ? 2097151.0 : t);
    return static_cast<unsigned>(t);
}

__global__ void k_keys(uint32_t n, const double* __restrict__ x, const double* __restrict__ y,
                       const double* __restrict__ z, double L, double* __restrict__ wx,
                       double* __restrict__ wy, double* __restrict__ wz,
                       unsigned long long* __restrict__ key, uint32_t* __restrict__ val,
                       unsigned int* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double a = wrap_f64(x[i], L), b = wrap_f64(y[i], L), c = wrap_f64(z[i], L);
    if (!(a >= 0.0 && a < L && b >= 0.0 && b < L && c >= 0.0 && c < L)) {
        raise_status(status, ST_NONFINITE_INPUT);
    }
    wx[i] = a;
    wy[i] = b;
    wz[i] = c;
    key[i] = (spread3(quant(a, L)) << 2) | (spread3(quant(b, L)) << 1) | spread3(quant(c, L));
    val[i] = i;
}

// ---- stable LSD radix sort, 8-bit digits --------------------------------
constexpr int kTile = 4096;  // keys per tile (256 threads x 16 rounds)

__global__ void k_tile_hist(uint32_t n, const unsigned long long* __restrict__ key, int shift,
                            uint32_t n_tiles, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kTile;
    for (int r = 0; r < kTile / kT; ++r) {
        const uint64_t i = base + r * kT + threadIdx.x;
        if (i < n) atomicAdd(&h[(key[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[static_cast<uint64_t>(threadIdx.x) * n_tiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void k_tile_scatter(uint32_t n, const unsigned long long* __restrict__ key,
                               const uint32_t* __restrict__ val, int shift, uint32_t n_tiles,
                               const uint32_t* __restrict__ offs,
                               unsigned long long* __restrict__ key_out,
                               uint32_t* __restrict__ val_out) {
    __shared__ uint32_t run[256];        // keys of each digit already placed by this tile
    __shared__ uint32_t wcount[8][256];  // per-warp digit counts of the current round
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    run[threadIdx.x] = offs[static_cast<uint64_t>(threadIdx.x) * n_tiles + blockIdx.x];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kTile;
    for (int r = 0; r < kTile / kT; ++r) {
        for (int w = 0; w < 8; ++w) wcount[w][threadIdx.x] = 0;
        __syncthreads();
        const uint64_t i = base + r * kT + threadIdx.x;
        const bool ok = i < n;
        const unsigned long long k = ok ? key[i] : 0ull;
        const unsigned d = ok ? static_cast<unsigned>((k >> shift) & 255u) : 256u;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned rank = __popc(peers & ((1u << lane) - 1u));
        if (ok && rank == 0) wcount[warp][d] = __popc(peers);
        __syncthreads();
        if (ok) {
            uint32_t before = run[d] + rank;
            for (int w = 0; w < warp; ++w) before += wcount[w][d];
            key_out[before] = k;
            val_out[before] = val[i];
        }
        __syncthreads();
        uint32_t tot = 0;
        for (int w = 0; w < 8; ++w) tot += wcount[w][threadIdx.x];
        run[threadIdx.x] += tot;
        __syncthreads();
    }
}

// ---- 64-bit exclusive scan (fixed-point COM prefix sums) ------------------
__global__ void k_scan64_block(const unsigned long long* __restrict__ in,
                               unsigned long long* __restrict__ out, uint64_t n,
                               unsigned long long* __restrict__ sums) {
    __shared__ unsigned long long wt[32];
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * 1024 + threadIdx.x;
    const unsigned long long v = i < n ? in[i] : 0ull;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) wt[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = wt[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        wt[lane] = w;
    }
    __syncthreads();
    const unsigned long long ex = inc - v + (warp ? wt[warp - 1] : 0ull);
    if (i < n) out[i] = ex;
    if (threadIdx.x == 1023 && sums) sums[blockIdx.x] = ex + v;
}

__global__ void k_scan64_add(unsigned long long* __restrict__ out, uint64_t n,
                             const unsigned long long* __restrict__ add) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] += add[i / 1024];
}

// ---- node extraction -------------------------------------------------------
__global__ void k_gather_sorted(uint32_t n, const uint32_t* __restrict__ val,
                                const double* __restrict__ wx, const double* __restrict__ wy,
                                const double* __restrict__ wz, double L, double* __restrict__ sx,
                                double* __restrict__ sy, double* __restrict__ sz,
                                unsigned long long* __restrict__ qx, unsigned long long* __restrict__ qy,
                                unsigned long long* __restrict__ qz, uint32_t* __restrict__ inv) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) {  // sentinel for the inclusive end of the prefix sums
        qx[n] = qy[n] = qz[n] = 0ull;
        return;
    }
    const uint32_t j = val[i];
    sx[i] = wx[j];
    sy[i] = wy[j];
    sz[i] = wz[j];
    const double s = 1099511627776.0 / L;  // 2^40 / L
    qx[i] = static_cast<unsigned long long>(llrint(wx[j] * s));
    qy[i] = static_cast<unsigned long long>(llrint(wy[j] * s));
    qz[i] = static_cast<unsigned long long>(llrint(wz[j] * s));
    inv[j] = i;
}

__global__ void k_flags(uint32_t n, const unsigned long long* __restrict__ key, int shift,
                        uint32_t* __restrict__ flag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flag[i] = (i == 0 || (key[i] >> shift) != (key[i - 1] >> shift)) ? 1u : 0u;
}

// run id of source i = (exclusive scan of flags)[i] + flag[i] - 1; run start.
__global__ void k_runs(uint32_t n, const uint32_t* __restrict__ flag,
                       const uint32_t* __restrict__ excl, uint32_t* __restrict__ runid,
                       uint32_t* __restrict__ run_start) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t r = excl[i] + flag[i] - 1u;
    runid[i] = r;
    if (flag[i]) run_start[r] = i;
}

// A level-l run is a node when its level-(l-1) run is an internal node.
__global__ void k_active(uint32_t n_runs, uint32_t n, const uint32_t* __restrict__ run_start,
                         const uint32_t* __restrict__ prev_runid,
                         const uint32_t* __restrict__ prev_internal, int level,
                         uint32_t* __restrict__ active) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > n_runs) return;
    if (r == n_runs) {
        active[r] = 0;
        return;
    }
    active[r] = level == 0 ? 1u : prev_internal[prev_runid[run_start[r]]];
}

__global__ void k_make_nodes(uint32_t n_runs, uint32_t n, int level, double L,
                             const uint32_t* __restrict__ run_start,
                             const uint32_t* __restrict__ active,
                             const uint32_t* __restrict__ node_excl, uint32_t node_base,
                             const unsigned long long* __restrict__ key,
                             const unsigned long long* __restrict__ qx,
                             const unsigned long long* __restrict__ qy,
                             const unsigned long long* __restrict__ qz, double m,
                             Node* __restrict__ nodes, uint32_t* __restrict__ internal,
                             uint32_t* __restrict__ node_of_run) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_runs) return;
    if (!active[r]) {
        internal[r] = 0;
        node_of_run[r] = 0xffffffffu;
        return;
    }
    const uint32_t s = run_start[r];
    const uint32_t e = r + 1 < n_runs ? run_start[r + 1] : n;
    const uint32_t idx = node_base + node_excl[r];
    node_of_run[r] = idx;
    Node nd;
    const int shift = 3 * (kBits - level);
    nd.prefix = shift >= 64 ? 0ull : (key[s] >> shift);
    // cube: integer coordinates of the level-l cell from the prefix bits
    unsigned cxi = 0, cyi = 0, czi = 0;
    for (int b = 0; b < level; ++b) {
        const unsigned long long t = nd.prefix >> (3 * (level - 1 - b));
        cxi = (cxi << 1) | static_cast<unsigned>((t >> 2) & 1ull);
        cyi = (cyi << 1) | static_cast<unsigned>((t >> 1) & 1ull);
        czi = (czi << 1) | static_cast<unsigned>(t & 1ull);
    }
    const double side = L / static_cast<double>(1ull << level);
    nd.half = 0.5 * side;
    nd.cx = (cxi + 0.5) * side;
    nd.cy = (cyi + 0.5) * side;
    nd.cz = (czi + 0.5) * side;
    const uint32_t cnt = e - s;
    const double inv = 1.0 / (static_cast<double>(cnt) * (1099511627776.0 / L));
    nd.mx = static_cast<double>(qx[e] - qx[s]) * inv;
    nd.my = static_cast<double>(qy[e] - qy[s]) * inv;
    nd.mz = static_cast<double>(qz[e] - qz[s]) * inv;
    nd.mass = m * cnt;
    nd.start = s;
    nd.end = e;
    nd.first_child = 0xffffffffu;
    nd.n_child = 0;
    nd.level = level;
    nd.leaf = (cnt == 1 || level == kBits) ? 1u : 0u;
    nodes[idx] = nd;
    internal[r] = nd.leaf ? 0u : 1u;
}

// Children of the level-(l-1) internal nodes are the level-l runs in their range.
__global__ void k_link(uint32_t n_prev_runs, const uint32_t* __restrict__ prev_node_of_run,
                       const uint32_t* __restrict__ prev_internal, Node* __restrict__ nodes,
                       const uint32_t* __restrict__ runid, const uint32_t* __restrict__ node_of_run) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_prev_runs || !prev_internal[r]) return;
    Node& p = nodes[prev_node_of_run[r]];
    const uint32_t a = runid[p.start], b = runid[p.end - 1];
    p.first_child = node_of_run[a];
    p.n_child = b - a + 1;
}

// ---- pair force -----------------------------------------------------------
// (r^2+eps^2)^(-3/2) - (1 - M_S(q)) / r^3 with M_S = erfc(q/2) + q/sqrt(pi) e^{-q^2/4}.
// For q < 0.05 the long-range part uses its series
//   (1 - M_S(q)) / r^3 = (1/sqrt(pi)) (1/6 - q^2/40 + q^4/448 - q^6/6912 + ...) / r_s^3
// (1 - M_S cancels there); otherwise (r^2+eps^2)^(-3/2) - 1/r^3 is formed as
// expm1(-1.5 log1p(eps^2/r^2)) / r^3 so no large terms cancel.
template <typename R>
__device__ __forceinline__ R short_factor_impl(R r2, R eps2, R inv_rs, R inv_rs3) {
    const R r = sqrt(r2);
    const R q = r * inv_rs;
    const R isp = R(0.5641895835477563);
    if (q < R(0.05)) {
        const R q2 = q * q;
        const R longf = isp * (R(1.0 / 6.0) + q2 * (R(-1.0 / 40.0)
                                                    + q2 * (R(1.0 / 448.0) - q2 * R(1.0 / 6912.0))))
            * inv_rs3;
        const R s = r2 + eps2;
        return R(1) / (s * sqrt(s)) - longf;
    }
    const R ms = erfc(R(0.5) * q) + q * isp * exp(R(-0.25) * q * q);
    const R ir = R(1) / r;
    return (expm1(R(-1.5) * log1p(eps2 / r2)) + ms) * ir * ir * ir;
}

__device__ __forceinline__ double min_image(double d, double L) {
    const double h = 0.5 * L;
    if (d >= h) d -= L;
    else if (d < -h) d += L;
    return d;
}

struct WalkParams {
    double L, r_cut, eps, theta, r_s, G, m;
};

// The monopole criterion's target-independent side, once per node: a node is
// accepted when its COM distance squared exceeds (2 half / theta + off)^2
// with off the L1 offset of the COM from the cube centre (the expression the
// walk would otherwise evaluate at every visit, in the same operations).
__global__ void k_open_radius(uint32_t n_nodes, double theta, Node* __restrict__ nodes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    Node& nd = nodes[i];
    const double off = fabs(nd.mx - nd.cx) + fabs(nd.my - nd.cy) + fabs(nd.mz - nd.cz);
    const double need = 2.0 * nd.half / theta + off;
    nd.open2 = need * need;
}

// Targets: sorted slots tslot[t] (null: target t is sorted slot t, every
// source). Output of target t goes to index out_idx[t] (null: t), written, or
// added to what is there when `add`. Source masses: sorted sm[] (null: P.m).
//
// Blocks per SM the registers are sized for. The binary64 walk waits mostly on
// the FP64 pipe's fixed latencies, which more warps hide: eight 128-thread
// blocks (64 registers, 52 bytes of spill) against the compiler's five (88
// registers) took the c5 walk from 1444 to 1283 ms. The FP32 walk measured
// 863 ms at the compiler's 71 registers (seven blocks), 874 at eight blocks and
// 879 at six, so it keeps its own choice.
#ifndef HYOWON_WALK_MINB64
#define HYOWON_WALK_MINB64 8
#endif
#ifndef HYOWON_WALK_MINB32
#define HYOWON_WALK_MINB32 1
#endif
template <typename R> struct WalkBlocks {
    static constexpr int minb = sizeof(R) == 8 ? HYOWON_WALK_MINB64 : HYOWON_WALK_MINB32;
};
template <typename R>
__global__ void __launch_bounds__(128, WalkBlocks<R>::minb)
k_walk(uint32_t n_targets, const uint32_t* __restrict__ tslot, const double* __restrict__ sx,
       const double* __restrict__ sy, const double* __restrict__ sz,
       const double* __restrict__ sm, const unsigned long long* __restrict__ skey,
       const Node* __restrict__ nodes, uint32_t n_nodes, WalkParams P,
       const uint32_t* __restrict__ out_idx, int add, double* __restrict__ ax,
       double* __restrict__ ay, double* __restrict__ az,
       unsigned long long* __restrict__ counters, unsigned int* status) {
    __shared__ uint32_t stack[4][kStack];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t t = (blockIdx.x * 4 + warp) * 32 + lane;
    const bool valid = t < n_targets;
    uint32_t slot = valid ? (tslot ? tslot[t] : t) : 0u;
    const double tx = sx[slot], ty = sy[slot], tz = sz[slot];
    const unsigned long long tkey = skey[slot];
    const R eps2 = static_cast<R>(P.eps * P.eps);
    const R inv_rs = static_cast<R>(1.0 / P.r_s);
    const R inv_rs3 = inv_rs * inv_rs * inv_rs;
    const double rc2 = P.r_cut * P.r_cut;
    R fx = 0, fy = 0, fz = 0;
    uint32_t skip_end = valid ? 0u : 0xffffffffu;
    unsigned long long visits = 0, pairs = 0;
    uint32_t* st = stack[warp];
    int sp = 0;
    if (lane == 0) st[0] = 0;
    sp = 1;
    __syncwarp();
    unsigned iter = 0;
    while (sp > 0) {
        if (++iter > kMaxIter) {
            if (lane == 0) raise_status(status, ST_CAPACITY);
            break;
        }
        const uint32_t ni = st[sp - 1];
        --sp;
        __syncwarp();
        const Node nd = nodes[ni];
        bool need_open = false;
        if (nd.start >= skip_end) {
            ++visits;
            // cube vs cutoff sphere (minimum image of the centre)
            const double dcx = min_image(nd.cx - tx, P.L), dcy = min_image(nd.cy - ty, P.L),
                         dcz = min_image(nd.cz - tz, P.L);
            const double h = nd.half;
            int rel;
            if (h >= 0.25 * P.L) {
                rel = 0;
            } else {
                const double ex = fmax(fabs(dcx) - h, 0.0), ey = fmax(fabs(dcy) - h, 0.0),
                             ez = fmax(fabs(dcz) - h, 0.0);
                const double fx2 = fabs(dcx) + h, fy2 = fabs(dcy) + h, fz2 = fabs(dcz) + h;
                if (ex * ex + ey * ey + ez * ez >= rc2) rel = -1;
                else if (fx2 * fx2 + fy2 * fy2 + fz2 * fz2 < rc2) rel = 1;
                else rel = 0;
            }
            if (rel < 0) {
                skip_end = nd.end;
            } else if (nd.leaf) {
                for (uint32_t i = nd.start; i < nd.end; ++i) {
                    if (i == slot) continue;
                    const double dx = min_image(sx[i] - tx, P.L), dy = min_image(sy[i] - ty, P.L),
                                 dz = min_image(sz[i] - tz, P.L);
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    if (!(r2 < rc2) || r2 == 0.0) continue;
                    const R f = short_factor_impl<R>(static_cast<R>(r2), eps2, inv_rs, inv_rs3)
                        * static_cast<R>(P.G * (sm ? sm[i] : P.m));
                    fx += f * static_cast<R>(dx);
                    fy += f * static_cast<R>(dy);
                    fz += f * static_cast<R>(dz);
                    ++pairs;
                }
                skip_end = nd.end;
            } else {
                const int shift = 3 * (kBits - static_cast<int>(nd.level));
                const bool contains = shift >= 64 ? true : ((tkey >> shift) == nd.prefix);
                bool accept = false;
                double dx = 0, dy = 0, dz = 0, r2 = 0;
                if (!contains && rel > 0) {
                    dx = min_image(nd.mx - tx, P.L);
                    dy = min_image(nd.my - ty, P.L);
                    dz = min_image(nd.mz - tz, P.L);
                    r2 = dx * dx + dy * dy + dz * dz;
                    accept = r2 > nd.open2;
                }
                if (accept) {
                    const R f = short_factor_impl<R>(static_cast<R>(r2), eps2, inv_rs, inv_rs3)
                        * static_cast<R>(P.G * nd.mass);
                    fx += f * static_cast<R>(dx);
                    fy += f * static_cast<R>(dy);
                    fz += f * static_cast<R>(dz);
                    ++pairs;
                    skip_end = nd.end;
                } else {
                    need_open = true;
                }
            }
        }
        const unsigned open = __ballot_sync(0xffffffffu, need_open);
        if (open) {
            if (nd.first_child >= n_nodes || nd.n_child > n_nodes - nd.first_child) {
                if (lane == 0) raise_status(status, ST_CELL_ESCAPE);
                break;
            }
            if (sp + static_cast<int>(nd.n_child) > kStack) {
                if (lane == 0) raise_status(status, ST_CAPACITY);
                break;
            }
            if (lane == 0) {
                for (uint32_t c = 0; c < nd.n_child; ++c)
                    st[sp + c] = nd.first_child + nd.n_child - 1 - c;
            }
            sp += static_cast<int>(nd.n_child);
            __syncwarp();
        }
    }
    if (valid) {
        const uint32_t o = out_idx ? out_idx[t] : t;
        if (add) {
            ax[o] += static_cast<double>(fx);
            ay[o] += static_cast<double>(fy);
            az[o] += static_cast<double>(fz);
        } else {
            ax[o] = static_cast<double>(fx);
            ay[o] = static_cast<double>(fy);
            az[o] = static_cast<double>(fz);
        }
    }
    // walk statistics: one atomic per warp (every lane of the warp leaves the
    // walk loop together)
    for (int o = 16; o > 0; o >>= 1) {
        visits += __shfl_down_sync(0xffffffffu, visits, o);
        pairs += __shfl_down_sync(0xffffffffu, pairs, o);
    }
    if (lane == 0) {
        atomicAdd(&counters[0], visits);
        atomicAdd(&counters[1], pairs);
    }
}

// Per-particle masses: node mass and centre of mass summed bottom-up, one
// level at a time from the deepest (leaves from their sources in sorted order,
// internal nodes from their children in child order: a fixed order, so the
// moments are the same bits run to run). A massless node keeps its cube centre.
__global__ void k_gather_masses(uint32_t n, const uint32_t* __restrict__ val,
                                const double* __restrict__ mass, double* __restrict__ sm) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) sm[i] = mass[val[i]];
}

__global__ void k_moments(uint32_t begin, uint32_t end, const double* __restrict__ sx,
                          const double* __restrict__ sy, const double* __restrict__ sz,
                          const double* __restrict__ sm, Node* __restrict__ nodes) {
    const uint32_t k = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= end) return;
    Node& nd = nodes[k];
    double M = 0.0, X = 0.0, Y = 0.0, Z = 0.0;
    if (nd.leaf) {
        for (uint32_t i = nd.start; i < nd.end; ++i) {
            const double m = sm[i];
            M += m;
            X += m * sx[i];
            Y += m * sy[i];
            Z += m * sz[i];
        }
    } else {
        for (uint32_t c = 0; c < nd.n_child; ++c) {
            const Node& ch = nodes[nd.first_child + c];
            M += ch.mass;
            X += ch.mass * ch.mx;
            Y += ch.mass * ch.my;
            Z += ch.mass * ch.mz;
        }
    }
    nd.mass = M;
    if (M > 0.0) {
        nd.mx = X / M;
        nd.my = Y / M;
        nd.mz = Z / M;
    } else {
        nd.mx = nd.cx;
        nd.my = nd.cy;
        nd.mz = nd.cz;
    }
}

struct Fail {
    int code;
    std::string msg;
};

#define TCK(call)                                                                           \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) throw Fail{e_ == cudaErrorMemoryAllocation ? HYOWON_ENOMEM  \
                                                                         : HYOWON_ECUDA,    \
                                          std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

}  // namespace

// Device scratch kept between calls: one block that the buffers of a call are
// carved from (256-byte aligned), so that repeated solves allocate nothing.
// A call that needs more than it holds takes the rest from cudaMalloc and
// records the total, and the next call regrows the block to that size.
struct Workspace {
    void* base = nullptr;
    size_t cap = 0;
    size_t want = 0;
};

Workspace* create_workspace() { return new (std::nothrow) Workspace(); }

void destroy_workspace(Workspace* ws) {
    if (!ws) return;
    if (ws->base) cudaFree(ws->base);
    delete ws;
}

namespace {

struct Mem {
    Workspace* ws;
    size_t off = 0;
    std::vector<void*> p;   // buffers beyond the workspace, freed with this
    explicit Mem(Workspace* w = nullptr) : ws(w) {
        if (ws && ws->want > ws->cap) {
            // the previous call finished its work before returning
            if (ws->base) cudaFree(ws->base);
            ws->base = nullptr;
            ws->cap = 0;
            TCK(cudaMalloc(&ws->base, ws->want));
            ws->cap = ws->want;
        }
    }
    template <typename T>
    T* get(size_t count) {
        const size_t bytes = (((count ? count : 1) * sizeof(T)) + 255) & ~static_cast<size_t>(255);
        if (ws) {
            const size_t at = off;
            off += bytes;
            if (off <= ws->cap) return reinterpret_cast<T*>(static_cast<char*>(ws->base) + at);
        }
        void* q = nullptr;
        TCK(cudaMalloc(&q, bytes));
        p.push_back(q);
        return static_cast<T*>(q);
    }
    ~Mem() {
        if (ws && off > ws->want) ws->want = off;
        for (void* q : p) cudaFree(q);
    }
};

void scan64(Mem& mem, const unsigned long long* in, unsigned long long* out, uint64_t n,
            cudaStream_t s) {
    const uint64_t blocks = (n + 1023) / 1024;
    if (blocks == 1) {
        k_scan64_block<<<1, 1024, 0, s>>>(in, out, n, nullptr);
        return;
    }
    unsigned long long* sums = mem.get<unsigned long long>(blocks);
    unsigned long long* sums_ex = mem.get<unsigned long long>(blocks);
    k_scan64_block<<<static_cast<unsigned>(blocks), 1024, 0, s>>>(in, out, n, sums);
    scan64(mem, sums, sums_ex, blocks, s);
    k_scan64_add<<<nb(n), kT, 0, s>>>(out, n, sums_ex);
}

uint32_t read_u32(const uint32_t* d, cudaStream_t s) {
    uint32_t v = 0;
    TCK(cudaMemcpyAsync(&v, d, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    TCK(cudaStreamSynchronize(s));
    return v;
}

thread_local std::string g_err;

}  // namespace

// Builds the octree of the n device sources (x, y, z; masses or, when null,
// P.particle_mass) and walks the targets on stream s: with host_targets the
// nt listed source indices, results written to ax/ay/az[target] in list order;
// without (nt = n), every source in key order, results added to
// ax/ay/az[source]. Output arrays are device memory. Device work is ordered on
// s; the call returns after it has finished.
int run(const hyowon_treepm_params& P, uint32_t n, const double* x, const double* y,
        const double* z, const double* masses, const uint32_t* host_targets, uint32_t nt,
        double* ax, double* ay, double* az, cudaStream_t s, double* stats,
        Workspace* ws = nullptr) {
    Mem mem(ws);
    struct Events {
        cudaEvent_t e[4] = {};
        Events() { for (auto& v : e) cudaEventCreate(&v); }
        ~Events() { for (auto& v : e) cudaEventDestroy(v); }
    } ev;
    unsigned int* status = mem.get<unsigned int>(1);
    TCK(cudaMemsetAsync(status, 0, sizeof(unsigned int), s));
    double* wx = mem.get<double>(n);
    double* wy = mem.get<double>(n);
    double* wz = mem.get<double>(n);
    unsigned long long* key[2] = {mem.get<unsigned long long>(n), mem.get<unsigned long long>(n)};
    uint32_t* val[2] = {mem.get<uint32_t>(n), mem.get<uint32_t>(n)};
    cudaEventRecord(ev.e[0], s);
    k_keys<<<nb(n), kT, 0, s>>>(n, x, y, z, P.box_size, wx, wy, wz, key[0], val[0], status);
    // radix sort
    const uint32_t n_tiles = static_cast<uint32_t>((n + kTile - 1) / kTile);
    uint32_t* hist = mem.get<uint32_t>(256ull * n_tiles + 1);
    uint32_t* offs = mem.get<uint32_t>(256ull * n_tiles + 1);
    uint32_t* scan_tmp = mem.get<uint32_t>(scan_tmp_elements(256u * n_tiles + 1));
    int cur = 0;
    for (int pass = 0; pass < 8; ++pass) {
        const int shift = 8 * pass;
        k_tile_hist<<<n_tiles, kT, 0, s>>>(n, key[cur], shift, n_tiles, hist);
        launch_exclusive_scan(hist, offs, 256u * n_tiles, scan_tmp, s);
        k_tile_scatter<<<n_tiles, kT, 0, s>>>(n, key[cur], val[cur], shift, n_tiles, offs,
                                               key[1 - cur], val[1 - cur]);
        cur = 1 - cur;
    }
    const unsigned long long* skey = key[cur];
    const uint32_t* sval = val[cur];
    double* sx = mem.get<double>(n);
    double* sy = mem.get<double>(n);
    double* sz = mem.get<double>(n);
    unsigned long long* q[3];
    unsigned long long* pq[3];
    for (int a = 0; a < 3; ++a) {
        q[a] = mem.get<unsigned long long>(n + 1);
        pq[a] = mem.get<unsigned long long>(n + 1);
    }
    uint32_t* inv = mem.get<uint32_t>(n);
    k_gather_sorted<<<nb(n + 1), kT, 0, s>>>(n, sval, wx, wy, wz, P.box_size, sx, sy, sz, q[0],
                                             q[1], q[2], inv);
    for (int a = 0; a < 3; ++a) scan64(mem, q[a], pq[a], n + 1, s);
    double* sm = nullptr;
    if (masses) {
        sm = mem.get<double>(n);
        k_gather_masses<<<nb(n), kT, 0, s>>>(n, sval, masses, sm);
    }
    // level-wise build
    const uint64_t cap = 6ull * n + 64;  // nodes; exceeding it is reported, not overrun
    Node* nodes = mem.get<Node>(cap);
    uint32_t* flag = mem.get<uint32_t>(n);
    uint32_t* excl = mem.get<uint32_t>(n + 1);
    uint32_t* ntmp = mem.get<uint32_t>(scan_tmp_elements(n + 2));
    uint32_t* runid[2] = {mem.get<uint32_t>(n), mem.get<uint32_t>(n)};
    uint32_t* run_start = mem.get<uint32_t>(n + 1);
    uint32_t* active = mem.get<uint32_t>(n + 1);
    uint32_t* node_excl = mem.get<uint32_t>(n + 2);
    uint32_t* internal[2] = {mem.get<uint32_t>(n + 1), mem.get<uint32_t>(n + 1)};
    uint32_t* node_of_run[2] = {mem.get<uint32_t>(n + 1), mem.get<uint32_t>(n + 1)};
    uint32_t node_base = 0, prev_runs = 0;
    int depth = 0;
    std::vector<uint32_t> level_begin;
    for (int level = 0; level <= kBits; ++level) {
        const int c = level & 1, p = 1 - c;
        const int shift = 3 * (kBits - level);
        k_flags<<<nb(n), kT, 0, s>>>(n, skey, shift >= 64 ? 63 : shift, flag);
        launch_exclusive_scan(flag, excl, n, ntmp, s);
        k_runs<<<nb(n), kT, 0, s>>>(n, flag, excl, runid[c], run_start);
        uint32_t last_excl = 0, last_flag = 0;
        TCK(cudaMemcpyAsync(&last_excl, excl + n - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        TCK(cudaMemcpyAsync(&last_flag, flag + n - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        TCK(cudaStreamSynchronize(s));
        const uint32_t n_runs = last_excl + last_flag;
        k_active<<<nb(n_runs + 1), kT, 0, s>>>(n_runs, n, run_start, runid[p], internal[p], level,
                                               active);
        launch_exclusive_scan(active, node_excl, n_runs + 1, ntmp, s);
        const uint32_t n_new = read_u32(node_excl + n_runs, s);
        if (n_new == 0) break;
        if (node_base + n_new > cap) throw Fail{HYOWON_ERUNTIME, "octree node capacity exceeded"};
        k_make_nodes<<<nb(n_runs), kT, 0, s>>>(n_runs, n, level, P.box_size, run_start, active,
                                               node_excl, node_base, skey, pq[0], pq[1], pq[2],
                                               P.particle_mass, nodes, internal[c], node_of_run[c]);
        if (level > 0)
            k_link<<<nb(prev_runs), kT, 0, s>>>(prev_runs, node_of_run[p], internal[p], nodes,
                                                runid[c], node_of_run[c]);
        level_begin.push_back(node_base);
        node_base += n_new;
        prev_runs = n_runs;
        depth = level;
    }
    level_begin.push_back(node_base);
    if (sm) {
        for (int l = static_cast<int>(level_begin.size()) - 2; l >= 0; --l) {
            const uint32_t b = level_begin[l], e = level_begin[l + 1];
            k_moments<<<nb(e - b), kT, 0, s>>>(b, e, sx, sy, sz, sm, nodes);
        }
    }
    if (node_base) k_open_radius<<<nb(node_base), kT, 0, s>>>(node_base, P.theta, nodes);
    cudaEventRecord(ev.e[1], s);
    const uint32_t* dslots = nullptr;
    const uint32_t* out_idx = nullptr;
    std::vector<uint32_t> order;
    if (host_targets) {
        // targets in key order for warp coherence; results land in key order
        std::vector<uint32_t> inv_h(n);
        TCK(cudaMemcpyAsync(inv_h.data(), inv, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
        TCK(cudaStreamSynchronize(s));
        order.resize(nt);
        for (uint32_t i = 0; i < nt; ++i) {
            if (host_targets[i] >= n) throw Fail{HYOWON_EINVAL, "target index out of range"};
            order[i] = i;
        }
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
            return inv_h[host_targets[a]] < inv_h[host_targets[b]];
        });
        std::vector<uint32_t> slots(nt), dest(nt);
        for (uint32_t i = 0; i < nt; ++i) {
            slots[i] = inv_h[host_targets[order[i]]];
            dest[i] = order[i];
        }
        uint32_t* d_slots = mem.get<uint32_t>(nt);
        uint32_t* d_dest = mem.get<uint32_t>(nt);
        TCK(cudaMemcpyAsync(d_slots, slots.data(), sizeof(uint32_t) * nt, cudaMemcpyHostToDevice, s));
        TCK(cudaMemcpyAsync(d_dest, dest.data(), sizeof(uint32_t) * nt, cudaMemcpyHostToDevice, s));
        TCK(cudaStreamSynchronize(s));
        dslots = d_slots;
        out_idx = d_dest;
    } else {
        out_idx = sval;   // sorted slot t holds source sval[t]
    }
    unsigned long long* counters = mem.get<unsigned long long>(2);
    TCK(cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), s));
    const double G = 6.67430e-11 * (1e10 * 1.98847e30) / (3.085677581491367e22 * 1000.0 * 1000.0);
    WalkParams W{P.box_size, P.cutoff, P.softening, P.theta, P.split_scale, G, P.particle_mass};
    cudaEventRecord(ev.e[2], s);
    const unsigned blocks = static_cast<unsigned>((nt + 127) / 128);
    const int add = host_targets ? 0 : 1;
    if (P.precision == HYOWON_FP64)
        k_walk<double><<<blocks, 128, 0, s>>>(nt, dslots, sx, sy, sz, sm, skey, nodes, node_base, W,
                                               out_idx, add, ax, ay, az, counters, status);
    else
        k_walk<float><<<blocks, 128, 0, s>>>(nt, dslots, sx, sy, sz, sm, skey, nodes, node_base, W,
                                              out_idx, add, ax, ay, az, counters, status);
    TCK(cudaPeekAtLastError());
    cudaEventRecord(ev.e[3], s);
    unsigned long long cnt[2] = {0, 0};
    unsigned int st = 0;
    TCK(cudaMemcpyAsync(cnt, counters, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    TCK(cudaMemcpyAsync(&st, status, sizeof(st), cudaMemcpyDeviceToHost, s));
    TCK(cudaStreamSynchronize(s));
    if (stats) {
        float tb = 0.f, tw = 0.f;
        cudaEventElapsedTime(&tb, ev.e[0], ev.e[1]);
        cudaEventElapsedTime(&tw, ev.e[2], ev.e[3]);
        stats[0] = node_base;
        stats[1] = depth;
        stats[2] = nt ? static_cast<double>(cnt[0]) / nt : 0.0;
        stats[3] = nt ? static_cast<double>(cnt[1]) / nt : 0.0;
        stats[4] = tb;
        stats[5] = tw;
    }
    if (st & ST_NONFINITE_INPUT) throw Fail{HYOWON_EINVAL, "source positions must be finite"};
    if (st & ST_CAPACITY) throw Fail{HYOWON_ERUNTIME, "tree walk exceeded its stack or iteration bound"};
    if (st & ST_CELL_ESCAPE) throw Fail{HYOWON_ELOGIC, "octree child link out of range"};
    return HYOWON_OK;
}

int short_forces(const hyowon_treepm_params& P, uint32_t n, const double* hx, const double* hy,
                 const double* hz, uint32_t nt, const uint32_t* htargets, double* hax,
                 double* hay, double* haz, double* stats) {
    cudaStream_t s = nullptr;
    TCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{s};
    Mem mem;
    double* x = mem.get<double>(n);
    double* y = mem.get<double>(n);
    double* z = mem.get<double>(n);
    TCK(cudaMemcpyAsync(x, hx, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    TCK(cudaMemcpyAsync(y, hy, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    TCK(cudaMemcpyAsync(z, hz, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    double* oax = mem.get<double>(nt);
    double* oay = mem.get<double>(nt);
    double* oaz = mem.get<double>(nt);
    run(P, n, x, y, z, nullptr, htargets, nt, oax, oay, oaz, s, stats);
    TCK(cudaMemcpyAsync(hax, oax, sizeof(double) * nt, cudaMemcpyDeviceToHost, s));
    TCK(cudaMemcpyAsync(hay, oay, sizeof(double) * nt, cudaMemcpyDeviceToHost, s));
    TCK(cudaMemcpyAsync(haz, oaz, sizeof(double) * nt, cudaMemcpyDeviceToHost, s));
    TCK(cudaStreamSynchronize(s));
    return HYOWON_OK;
}

int device_short_forces(const hyowon_treepm_params& P, uint32_t n, const double* x,
                        const double* y, const double* z, const double* masses, double* ax,
                        double* ay, double* az, cudaStream_t s, double* stats, std::string* err,
                        Workspace* ws) {
    try {
        return run(P, n, x, y, z, masses, nullptr, n, ax, ay, az, s, stats, ws);
    } catch (const Fail& f) {
        if (err) *err = f.msg;
        return f.code;
    }
}

}  // namespace hyowon::tree

extern "C" {

const char* hyowon_treepm_last_error(void) { return hyowon::tree::g_err.c_str(); }

int hyowon_treepm_short_forces(const hyowon_treepm_params* params, uint64_t n, const double* x,
                               const double* y, const double* z, uint64_t n_targets,
                               const uint32_t* targets, double* ax, double* ay, double* az,
                               double* stats) {
    using namespace hyowon::tree;
    g_err.clear();
    if (!params || !x || !y || !z || !targets || !ax || !ay || !az || n < 2 || n > 0xFFFFFFF0ull
        || n_targets == 0 || n_targets > n) {
        g_err = "invalid TreePM short-range arguments";
        return HYOWON_EINVAL;
    }
    const hyowon_treepm_params& P = *params;
    if (!(P.box_size > 0.0) || !(P.split_scale > 0.0) || !(P.cutoff > 0.0)
        || !(P.cutoff < 0.5 * P.box_size) || !(P.softening > 0.0) || !(P.theta > 0.0)
        || !(P.particle_mass > 0.0)
        || (P.precision != HYOWON_FP64 && P.precision != HYOWON_FP32_FIXED)) {
        g_err = "TreePM parameters must be finite positive with r_cut < L/2";
        return HYOWON_EINVAL;
    }
    try {
        return short_forces(P, static_cast<uint32_t>(n), x, y, z,
                            static_cast<uint32_t>(n_targets), targets, ax, ay, az, stats);
    } catch (const Fail& f) {
        g_err = f.msg;
        return f.code;
    }
}

}  // extern "C"
