// pm_handle.cu -- the C ABI of include/hyowon_pm.h: device state, cuFFT plans
// and the orchestration of one force solve / one KDK step on one stream.
//
// Step structure (binary64 form), for particle state P, accelerations A:
//   1. kick_drift_key: P' = K1-kick + drift of P into the spare buffer set,
//      cell-bucket key + histogram (rank) per particle;
//   2. exclusive scan of the bucket histogram;
//   3. scatter P' -> P in bucket order (skipped on a device error: nothing is
//      published, as LeapfrogIntegrator's preflight, leapfrog_integrator.cpp:170-190);
//   4. deterministic fixed-point tile deposit (particles located through the
//      bucket offsets and, between re-sorts, the cell-order index), D2Z,
//      Green (+ density normalisation, 1/N^3, mass check), Z2D;
//   5. gather_kick: A = -grad(phi) at P, p'' = p' + A*K2 into the spare
//      momentum buffer, published by a pointer swap after the status check.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "hyowon_pm.h"
#include "pm_diag.h"
#include "pm_fp32.h"
#include "pm_poisson.h"
#include "pm_kernels.h"
#include "pm_ic.h"
#include "pm_snapshot.h"
#include "pm_lpt.h"
#include "pm_pk.h"
#include "pm_tree.h"
#include "hyowon_treepm.h"
#include "hyowon_debug.h"
#include "hyowon_adjoint.h"
#include "pm_adjoint.h"

using namespace hyowon;

namespace {

constexpr double kPi = 3.14159265358979323846;

// include/cosmo_nbody/cosmology/units.hpp:12-25, evaluated in that order.
double gravitational_constant() {
    const double G_SI = 6.67430e-11;
    const double Mpc_in_m = 3.085677581491367e22;
    const double Msun_in_kg = 1.98847e30;
    const double MassUnit_in_kg = 1e10 * Msun_in_kg;
    const double V = 1000.0;
    return G_SI * MassUnit_in_kg / (Mpc_in_m * V * V);
}

struct Error {
    int code;
    std::string msg;
};

}  // namespace

struct hyowon_pm_s {
    hyowon::ic::Workspace* ic_ws = nullptr;  // generated-IC work arrays (hyowon_pm_generate_ics)
    double L = 0.0;
    int N = 0;
    int method = HYOWON_PURE_PM;
    int deconvolve = 0;
    double r_s = 0.0;
    int precision = HYOWON_FP64;
    Axis axis{};
    double four_pi_G = 0.0;
    double field_scale = 0.0;  // (1/dx^3) * (1/N^3)

    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // download: device->host copies beside the kernels
    cudaEvent_t staged[2] = {}, copied[2] = {};
    cufftHandle plan_r2c = 0;
    cufftHandle plan_c2r = 0;
    bool plans = false;
    void* fft_work = nullptr;

    double* mesh = nullptr;      // real N^3: mass, then potential
    double2* modes = nullptr;    // half spectrum
    double2* phi_k = nullptr;    // spectral method: kept copy of phi_k
    double* lap = nullptr;       // 1-D discrete Laplacian symbol (N)
    double* win = nullptr;       // 1-D CIC window W(k) (N)
    double2* tw = nullptr;       // exp(-2 pi i m/N) (N): five-pass potential solve
    poisson::Plan* fft_plan = nullptr;  // its tensor maps of `modes`
    bool five_pass = false;      // pure PM on a power-of-two mesh: pm_poisson.cu

    uint32_t n = 0;
    uint32_t cap = 0;
    double* pos[2][3] = {};
    double* mom[2][3] = {};
    uint32_t* id[2] = {};
    double* mass[2] = {};
    int pc = 0, mc = 0, ic = 0;
    double* acc[3] = {};
    bool acc_valid = false;
    bool sorted = false;
    bool has_state = false;
    double uniform_mass = 0.0;
    bool has_masses = false;
    double input_mass = 0.0;
    double mass_tol = 0.0;
    double mass_target_offset = 0.0;  // failure-path tests (hyowon_debug.h)

    SortWork sort{};
    uint32_t sort_cap_buckets = 0;
    uint32_t* order = nullptr;        // cell-order slot -> particle slot (n)
    uint32_t* d_max_count = nullptr;  // largest bucket count of the last keying
    double max_mass = 0.0;            // largest particle mass (fixed-point scale)
    // What the bucket offsets describe for the current position set:
    // 0 nothing, 1 the arrays themselves are in cell order, 2 `order` holds it.
    int order_state = 0;

    unsigned int* d_status = nullptr;
    unsigned long long* d_maxdrift = nullptr;
    double* d_diag = nullptr;                   // diagnostics scratch (pm_diag.h)
    unsigned int* h_status = nullptr;           // pinned
    uint32_t* h_max_count = nullptr;            // pinned
    unsigned long long* h_maxdrift = nullptr;   // pinned

    fp32::State* f32 = nullptr;  // precision form (pm_fp32.cu)

    hyowon::adj::Cache* adj = nullptr;  // adjoint engines of hyowon_pm_vjp

    // TreePM short range (hyowon_pm_set_treepm_short_range)
    bool treepm_short = false;
    hyowon_treepm_params tp{};
    double* tree_buf = nullptr;       // 6 n doubles: widened positions, short-range output
    uint32_t tree_cap = 0;
    tree::Workspace* tree_ws = nullptr;   // octree build and walk scratch, kept between solves

    bool timing = false;
    cudaEvent_t ev[8] = {};
    cudaEvent_t call_ev[2] = {};
    double last_times[9] = {};
    double phase_sum[6] = {};  // per-phase device ms summed over the steps of a call
    int phase_steps = 0;
    uint64_t launches = 0;  // kernels launched by this library (cuFFT excluded)
    int sort_interval = 4;  // re-sort the particles every this many steps
    int since_sort = 0;

    std::string err;
};

namespace {

int fail(hyowon_pm_t h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

int cuda_fail(hyowon_pm_t h, cudaError_t e, const char* where) {
    return fail(h, e == cudaErrorMemoryAllocation ? HYOWON_ENOMEM : HYOWON_ECUDA,
                std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

#define CKFFT(call)                                                             \
    do {                                                                        \
        cufftResult r_ = (call);                                                \
        if (r_ != CUFFT_SUCCESS)                                                \
            return fail(h, HYOWON_ECUDA, std::string(#call) + ": cufft error " \
                                             + std::to_string(static_cast<int>(r_))); \
    } while (0)

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
}

// Maps device status bits onto the reference's exception classes.
int status_to_code(hyowon_pm_t h, unsigned int st) {
    if (st == 0) return HYOWON_OK;
    if (st & ST_NONFINITE_INPUT)
        return fail(h, HYOWON_EINVAL, "particle positions and masses must be finite (masses non-negative)");
    if (st & ST_CELL_ESCAPE)
        return fail(h, HYOWON_ELOGIC, "CIC bounded coordinate escaped the mesh domain");
    if (st & ST_KICK_DRIFT)
        return fail(h, HYOWON_EOVERFLOW, "Leapfrog K1/drift update is not finite and representable");
    if (st & ST_MASS)
        return fail(h, HYOWON_ERUNTIME, "CIC deposited mass violates the binary64 forward-error bound");
    if (st & ST_CAPACITY)
        return fail(h, HYOWON_ERUNTIME, "fixed-point mass cell capacity exceeded");
    if (st & ST_FORCE)
        return fail(h, HYOWON_EOVERFLOW, "PM backend produced a non-finite force");
    if (st & ST_KICK2)
        return fail(h, HYOWON_EOVERFLOW, "Leapfrog K2 update is not finite and representable");
    if (st & ST_UNDERFLOW)
        return fail(h, HYOWON_EUNDERFLOW, "CIC centered-gradient gather lost a non-zero product");
    if (st & ST_PIPELINE)
        return fail(h, HYOWON_ERUNTIME, "potential solve: a device pipeline wait timed out");
    return fail(h, HYOWON_ERUNTIME, "unknown device status");
}

ParticlesF64 set_view(hyowon_pm_t h, int pset, int mset) {
    return ParticlesF64{h->pos[pset][0], h->pos[pset][1], h->pos[pset][2],
                        h->mom[mset][0], h->mom[mset][1], h->mom[mset][2]};
}

void free_particles(hyowon_pm_t h) {
    for (int s = 0; s < 2; ++s) {
        for (int a = 0; a < 3; ++a) {
            cudaFree(h->pos[s][a]);
            cudaFree(h->mom[s][a]);
            h->pos[s][a] = h->mom[s][a] = nullptr;
        }
        cudaFree(h->id[s]);
        cudaFree(h->mass[s]);
        h->id[s] = nullptr;
        h->mass[s] = nullptr;
    }
    for (int a = 0; a < 3; ++a) {
        cudaFree(h->acc[a]);
        h->acc[a] = nullptr;
    }
    cudaFree(h->sort.key);
    cudaFree(h->sort.rank);
    cudaFree(h->order);
    h->sort.key = h->sort.rank = nullptr;
    h->order = nullptr;
    h->cap = 0;
    h->order_state = 0;
}

int ensure_capacity(hyowon_pm_t h, uint32_t n, bool masses) {
    if (n <= h->cap && (!masses || h->mass[0])) return HYOWON_OK;
    free_particles(h);
    for (int s = 0; s < 2; ++s) {
        for (int a = 0; a < 3; ++a) {
            CK(dalloc(&h->pos[s][a], n));
            CK(dalloc(&h->mom[s][a], n));
        }
        CK(dalloc(&h->id[s], n));
        if (masses) CK(dalloc(&h->mass[s], n));
    }
    for (int a = 0; a < 3; ++a) CK(dalloc(&h->acc[a], n));
    CK(dalloc(&h->sort.key, n));
    CK(dalloc(&h->sort.rank, n));
    CK(dalloc(&h->order, n));
    h->cap = n;
    return HYOWON_OK;
}

// Buckets of 2^shift consecutive cells, about eight particles per bucket.
int ensure_sort_buckets(hyowon_pm_t h, uint32_t n) {
    const uint64_t cells = static_cast<uint64_t>(h->N) * h->N * h->N;
    int shift = 0;
    while (shift < 30 && (cells >> (shift + 1)) * 8 >= static_cast<uint64_t>(n) && (cells >> (shift + 1)) > 0)
        ++shift;
    const uint32_t nb = static_cast<uint32_t>((cells + (1ull << shift) - 1) >> shift);
    h->sort.shift = shift;
    h->sort.n_buckets = nb;
    if (nb > h->sort_cap_buckets) {
        cudaFree(h->sort.count);
        cudaFree(h->sort.offset);
        cudaFree(h->sort.scan_tmp);
        CK(dalloc(&h->sort.count, nb + 1));
        CK(dalloc(&h->sort.offset, nb + 1));
        CK(dalloc(&h->sort.scan_tmp, scan_tmp_elements(nb + 1)));
        h->sort_cap_buckets = nb;
    }
    return HYOWON_OK;
}

// Input mass and the CIC mass-conservation bound of
// src/math/cic_mass_conservation.cpp:26-59, with a small allowance for the
// rounding of the FFT's k=0 sum that stands in for the exact mesh-mass sum.
void set_input_mass(hyowon_pm_t h, double total, uint32_t n) {
    h->input_mass = total;
    const long double eps = std::numeric_limits<double>::epsilon();
    const long double nu = (32.0L * n + 1.0L) * eps;
    const long double gamma = nu / (1.0L - nu);
    h->mass_tol = static_cast<double>((gamma + 64.0L * eps) * total * (1.0L + 4.0L * gamma));
}

// The generated-IC work arrays are kept between hyowon_pm_generate_ics calls
// and given back before anything else that needs device memory runs.
void release_ic_workspace(hyowon_pm_t h) {
    if (h && h->ic_ws) {
        hyowon::ic::workspace_destroy(h->ic_ws);
    hyowon::adj::destroy_cache(h->adj);
        h->ic_ws = nullptr;
    }
}

int read_status(hyowon_pm_t h, unsigned int* st) {
    CK(cudaMemcpyAsync(h->h_status, h->d_status, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *st = *h->h_status;
    return HYOWON_OK;
}

// The densest bucket count of the last keying (it picks the deposit form);
// waits for the work before it.
int read_max_count(hyowon_pm_t h, uint32_t* out) {
    CK(cudaMemcpyAsync(h->h_max_count, h->d_max_count, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *out = *h->h_max_count;
    return HYOWON_OK;
}

// Permutes the current particle state into bucket order (used after upload).
int sort_current(hyowon_pm_t h) {
    const uint32_t n = h->n;
    CK(cudaMemsetAsync(h->sort.count, 0, sizeof(uint32_t) * (h->sort.n_buckets + 1), h->stream));
    ++h->launches;
    launch_key_f64(n, set_view(h, h->pc, h->mc), h->axis, h->sort, h->d_status, h->stream);
    h->launches += launch_exclusive_scan(h->sort.count, h->sort.offset, h->sort.n_buckets + 1, h->sort.scan_tmp,
                          h->stream);
    CK(cudaMemsetAsync(h->d_max_count, 0, sizeof(uint32_t), h->stream));
    ++h->launches;
    launch_max_count_f64(h->sort.n_buckets, h->sort.count, h->d_max_count, h->stream);
    const double* src[8];
    double* dst[8];
    int k = 0;
    for (int a = 0; a < 3; ++a) {
        src[k] = h->pos[h->pc][a];
        dst[k++] = h->pos[1 - h->pc][a];
    }
    for (int a = 0; a < 3; ++a) {
        src[k] = h->mom[h->mc][a];
        dst[k++] = h->mom[1 - h->mc][a];
    }
    if (h->has_masses) {
        src[k] = h->mass[h->ic];
        dst[k++] = h->mass[1 - h->ic];
    }
    const uint32_t* su[1] = {h->id[h->ic]};
    uint32_t* du[1] = {h->id[1 - h->ic]};
    ++h->launches;
    launch_scatter_multi(n, h->sort.key, h->sort.rank, h->sort.offset, k, src, dst, 1, su, du,
                         h->d_status, h->stream);
    unsigned int st = 0;
    int rc = read_status(h, &st);
    if (rc) return rc;
    if (st) return status_to_code(h, st);
    h->pc = 1 - h->pc;
    h->mc = 1 - h->mc;
    h->ic = 1 - h->ic;
    h->sorted = true;
    h->order_state = 1;
    return HYOWON_OK;
}

// Cell order of the current position set through the order index (its
// arrays stay where they are): keys, bucket offsets, order, largest bucket.
int index_current(hyowon_pm_t h) {
    const uint32_t n = h->n;
    CK(cudaMemsetAsync(h->sort.count, 0, sizeof(uint32_t) * (h->sort.n_buckets + 1), h->stream));
    ++h->launches;
    launch_key_f64(n, set_view(h, h->pc, h->mc), h->axis, h->sort, h->d_status, h->stream);
    h->launches += launch_exclusive_scan(h->sort.count, h->sort.offset, h->sort.n_buckets + 1,
                                         h->sort.scan_tmp, h->stream);
    ++h->launches;
    launch_order(n, h->sort.key, h->sort.rank, h->sort.offset, h->order, h->d_status, h->stream);
    CK(cudaMemsetAsync(h->d_max_count, 0, sizeof(uint32_t), h->stream));
    ++h->launches;
    launch_max_count_f64(h->sort.n_buckets, h->sort.count, h->d_max_count, h->stream);
    unsigned int st = 0;
    int rc = read_status(h, &st);
    if (rc) return rc;
    if (st) return status_to_code(h, st);
    h->order_state = 2;
    return HYOWON_OK;
}

// The order argument of the binary64 deposit for the current set.
const uint32_t* current_order(hyowon_pm_t h) { return h->order_state == 2 ? h->order : nullptr; }

void record(hyowon_pm_t h, int i) {
    if (h->timing) cudaEventRecord(h->ev[i], h->stream);
}

int add_short_range_f64(hyowon_pm_t h, int pset);

// Deposit -> FFT -> Green -> inverse FFT -> gather (+ K2 into the spare momenta).
// Leaves the status check to the caller.
int enqueue_force(hyowon_pm_t h, int pset, int mset, bool kick, double K2,
                  const uint32_t* order) {
    const uint32_t n = h->n;
    const int N = h->N;
    const size_t cells = static_cast<size_t>(N) * N * N;
    if (h->precision == HYOWON_FP32_FIXED) {
        return fp32::enqueue_force(h->f32, h->stream, h->d_status, kick, K2, h->timing ? h->ev : nullptr);
    }
    const ParticlesF64 p = set_view(h, pset, mset);
    (void)cells;
    uint32_t max_count = 0;
    int rc0 = read_max_count(h, &max_count);
    if (rc0) return rc0;
    record(h, 1);
    ++h->launches;
    // five-pass solve: the deposit writes its tiles transformed along z
    CK(launch_deposit_tiles_f64(p, h->has_masses ? h->mass[h->ic] : nullptr, h->uniform_mass,
                                order, h->sort, h->axis, h->d_max_count, max_count,
                                deposit_mass_exponent_f64(h->max_mass), h->mesh,
                                h->five_pass ? h->modes : nullptr, h->tw, h->d_status,
                                h->stream));
    record(h, 2);
    double* const pxo = h->mom[1 - mset][0];
    double* const pyo = h->mom[1 - mset][1];
    double* const pzo = h->mom[1 - mset][2];
    if (h->five_pass) {
        int k = poisson::forward_columns_f64(h->fft_plan, N, h->modes, h->tw, h->d_status, h->stream);
        if (k < 0) return fail(h, HYOWON_ECUDA, "potential solve: forward pass launch failed");
        h->launches += k;
        record(h, 3);
        const poisson::GreenF64 g{h->lap, h->win, h->four_pi_G, h->field_scale, h->deconvolve,
                                  h->input_mass + h->mass_target_offset, h->mass_tol, h->d_status};
        k = poisson::green_f64(h->fft_plan, N, h->modes, h->tw, g, h->stream);
        if (k < 0) return fail(h, HYOWON_ECUDA, "potential solve: Green pass launch failed");
        h->launches += k;
        record(h, 4);
        k = poisson::inverse_f64(h->fft_plan, N, h->modes, h->mesh, h->tw, h->d_status, h->stream);
        if (k < 0) return fail(h, HYOWON_ECUDA, "potential solve: inverse pass launch failed");
        h->launches += k;
        record(h, 5);
        ++h->launches;
        launch_gather_kick_f64(n, h->mesh, p, h->acc[0], h->acc[1], h->acc[2], kick ? 1 : 0, K2,
                               pxo, pyo, pzo, h->axis, h->d_status, h->stream);
        record(h, 6);
        return HYOWON_OK;
    }
    CKFFT(cufftExecD2Z(h->plan_r2c, h->mesh, reinterpret_cast<cufftDoubleComplex*>(h->modes)));
    record(h, 3);
    if (h->method == HYOWON_PURE_PM) {
        ++h->launches;
        launch_green_f64(N, h->modes, h->lap, h->win, h->four_pi_G, h->field_scale, h->deconvolve,
                         h->input_mass + h->mass_target_offset, h->mass_tol, h->d_status,
                         h->stream);
        record(h, 4);
        CKFFT(cufftExecZ2D(h->plan_c2r, reinterpret_cast<cufftDoubleComplex*>(h->modes), h->mesh));
        record(h, 5);
        ++h->launches;
        launch_gather_kick_f64(n, h->mesh, p, h->acc[0], h->acc[1], h->acc[2], kick ? 1 : 0, K2,
                               pxo, pyo, pzo, h->axis, h->d_status, h->stream);
        record(h, 6);
        return HYOWON_OK;
    }
    // TreePM long range: Green's function once, then per axis -ik, C2R and a
    // plain CIC gather added to the zeroed acceleration.
    ++h->launches;
    launch_green_spectral_f64(N, h->L, h->modes, h->win, h->four_pi_G, h->field_scale, h->r_s,
                              h->input_mass + h->mass_target_offset, h->mass_tol, h->d_status,
                              h->stream);
    CK(cudaMemcpyAsync(h->phi_k, h->modes, sizeof(double2) * static_cast<size_t>(N) * N * (N / 2 + 1),
                       cudaMemcpyDeviceToDevice, h->stream));
    record(h, 4);
    for (int a = 0; a < 3; ++a) {
        CK(cudaMemsetAsync(h->acc[a], 0, sizeof(double) * n, h->stream));
        ++h->launches;
        launch_spectral_axis_f64(N, h->L, a, h->phi_k, h->modes, h->stream);
        CKFFT(cufftExecZ2D(h->plan_c2r, reinterpret_cast<cufftDoubleComplex*>(h->modes), h->mesh));
        ++h->launches;
        launch_interp_add_f64(n, h->mesh, p, h->axis, h->acc[a], h->d_status, h->stream);
    }
    if (h->treepm_short) {
        int rc = add_short_range_f64(h, pset);
        if (rc) return rc;
    }
    record(h, 5);
    if (kick) {
        ++h->launches;
        launch_kick_only_f64(n, p, h->acc[0], h->acc[1], h->acc[2], K2, pxo, pyo, pzo, h->d_status,
                             h->stream);
    }
    record(h, 6);
    return HYOWON_OK;
}

void collect_timing(hyowon_pm_t h) {
    if (!h->timing) return;
    cudaEventSynchronize(h->ev[6]);
    float t = 0.f;
    for (int i = 0; i < 6; ++i) {
        cudaEventElapsedTime(&t, h->ev[i], h->ev[i + 1]);
        h->phase_sum[i] += t;
    }
    ++h->phase_steps;
}

// Whole-call device time and launch count (hyowon_pm_last_timing).
struct CallTimer {
    hyowon_pm_t h;
    uint64_t launches0;
    static uint64_t total(hyowon_pm_t hh) {
        return hh->launches + (hh->f32 ? fp32::launches(hh->f32) : 0);
    }
    explicit CallTimer(hyowon_pm_t hh) : h(hh), launches0(total(hh)) {
        for (double& v : h->phase_sum) v = 0.0;
        h->phase_steps = 0;
        if (h->timing) cudaEventRecord(h->call_ev[0], h->stream);
    }
    ~CallTimer() {
        if (!h->timing) return;
        cudaEventRecord(h->call_ev[1], h->stream);
        cudaEventSynchronize(h->call_ev[1]);
        float t = 0.f;
        cudaEventElapsedTime(&t, h->call_ev[0], h->call_ev[1]);
        h->last_times[0] = t;
        for (int i = 0; i < 6; ++i) h->last_times[i + 1] = h->phase_sum[i];
        h->last_times[7] = static_cast<double>(total(h) - launches0);
        h->last_times[8] = h->phase_steps;
    }
};

int ensure_tree_workspace(hyowon_pm_t h) {
    if (!h->tree_ws) {
        h->tree_ws = tree::create_workspace();
        if (!h->tree_ws) return fail(h, HYOWON_ENOMEM, "out of host memory");
    }
    return HYOWON_OK;
}

int ensure_tree_buffer(hyowon_pm_t h) {
    const int rc = ensure_tree_workspace(h);
    if (rc) return rc;
    if (h->tree_buf && h->tree_cap >= h->n) return HYOWON_OK;
    cudaFree(h->tree_buf);
    h->tree_buf = nullptr;
    h->tree_cap = 0;
    CK(dalloc(&h->tree_buf, 6 * static_cast<size_t>(h->n)));
    h->tree_cap = h->n;
    return HYOWON_OK;
}

// Short-range accelerations of position set pset added to the binary64
// accelerations (the TreePM force method), unless an earlier kernel of the
// step already failed.
int add_short_range_f64(hyowon_pm_t h, int pset) {
    unsigned int st = 0;
    int rc = read_status(h, &st);
    if (rc) return rc;
    if (st) return HYOWON_OK;   // the status decides the outcome; K2 is gated on it
    rc = ensure_tree_workspace(h);
    if (rc) return rc;
    std::string err;
    hyowon_treepm_params P = h->tp;
    P.particle_mass = h->uniform_mass > 0.0 ? h->uniform_mass : 1.0;  // masses win when present
    rc = tree::device_short_forces(P, h->n, h->pos[pset][0], h->pos[pset][1], h->pos[pset][2],
                                   h->has_masses ? h->mass[h->ic] : nullptr, h->acc[0], h->acc[1],
                                   h->acc[2], h->stream, nullptr, &err, h->tree_ws);
    return rc ? fail(h, rc, "TreePM short range: " + err) : HYOWON_OK;
}

// The precision form's hook: widen set P, walk, add to its FP32 accelerations.
int short_range_hook_f32(void* ctx, cudaStream_t s, int P) {
    hyowon_pm_t h = static_cast<hyowon_pm_t>(ctx);
    unsigned int st = 0;
    int rc = read_status(h, &st);
    if (rc) return rc;
    if (st) return HYOWON_OK;
    rc = ensure_tree_buffer(h);
    if (rc) return rc;
    const size_t n = h->n;
    double* px = h->tree_buf;
    double* out = h->tree_buf + 3 * n;
    rc = fp32::positions_f64_of_set(h->f32, s, P, px, px + n, px + 2 * n);
    if (rc) return status_or_cuda(h, rc);
    CK(cudaMemsetAsync(out, 0, sizeof(double) * 3 * n, s));
    std::string err;
    hyowon_treepm_params Pm = h->tp;
    Pm.particle_mass = h->uniform_mass;
    rc = tree::device_short_forces(Pm, h->n, px, px + n, px + 2 * n, nullptr, out, out + n,
                                   out + 2 * n, s, nullptr, &err, h->tree_ws);
    if (rc) return fail(h, rc, "TreePM short range: " + err);
    return status_or_cuda(h, fp32::add_accelerations(h->f32, s, out, out + n, out + 2 * n));
}

// Force solve at the current positions; accelerations become valid.
int solve_force(hyowon_pm_t h) {
    if (!h->sorted) {
        int rc = h->precision == HYOWON_FP32_FIXED ? fp32::sort_current(h->f32, h->stream, h->d_status)
                                                   : sort_current(h);
        if (rc) return h->precision == HYOWON_FP32_FIXED ? status_or_cuda(h, rc) : rc;
        h->sorted = true;
    }
    if (h->precision == HYOWON_FP64 && h->order_state == 0) {
        int rc = index_current(h);
        if (rc) return rc;
    }
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream));
    record(h, 0);
    int rc = enqueue_force(h, h->pc, h->mc, false, 0.0, current_order(h));
    if (rc) return rc;
    unsigned int st = 0;
    rc = read_status(h, &st);
    if (rc) return rc;
    collect_timing(h);
    if (st) {
        h->acc_valid = false;
        return status_to_code(h, st);
    }
    h->acc_valid = true;
    return HYOWON_OK;
}

}  // namespace

namespace hyowon {
// Used by the precision form to report CUDA failures through the handle.
int status_or_cuda(hyowon_pm_t h, int rc) {
    if (rc == HYOWON_OK) return rc;
    if (h->f32 && !fp32::last_error(h->f32).empty()) h->err = fp32::last_error(h->f32);
    return rc;
}
}  // namespace hyowon

namespace {

int kdk_step_impl(hyowon_pm_t h, double K1, double D, double K2, double* max_drift) {
    if (!h->has_state) return fail(h, HYOWON_ELOGIC, "no particles uploaded");
    if (!std::isfinite(K1) || !std::isfinite(D) || !std::isfinite(K2))
        return fail(h, HYOWON_EOVERFLOW, "Leapfrog K1/drift update is not finite and representable");
    if (!h->acc_valid) {
        int rc = solve_force(h);
        if (rc) return rc;
    }
    if (h->precision == HYOWON_FP32_FIXED) {
        int rc = fp32::kdk_step(h->f32, h->stream, h->d_status, h->d_maxdrift, K1, D, K2,
                                h->timing ? h->ev : nullptr);
        if (rc) return status_or_cuda(h, rc);
        unsigned int st = 0;
        rc = read_status(h, &st);
        if (rc) return rc;
        collect_timing(h);
        const bool published = (st & ST_BLOCKS_PUBLISH) == 0;
        fp32::commit_step(h->f32, published, st == 0);
        if (!published) h->sorted = false;  // the form re-sorts before its next solve
        if (st) {
            h->acc_valid = false;
            return status_to_code(h, st);
        }
        if (max_drift) {
            CK(cudaMemcpy(h->h_maxdrift, h->d_maxdrift, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
            double d;
            std::memcpy(&d, h->h_maxdrift, sizeof(double));
            *max_drift = d;
        }
        return HYOWON_OK;
    }
    const uint32_t n = h->n;
    const bool sort_now = h->sort_interval <= 1 || h->since_sort + 1 >= h->sort_interval;
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream));
    CK(cudaMemsetAsync(h->d_maxdrift, 0, sizeof(unsigned long long), h->stream));
    CK(cudaMemsetAsync(h->sort.count, 0, sizeof(uint32_t) * (h->sort.n_buckets + 1), h->stream));
    CK(cudaMemsetAsync(h->d_max_count, 0, sizeof(uint32_t), h->stream));
    record(h, 0);
    // 1. candidate = K1 kick + drift of the current state, into the spare set.
    const ParticlesF64 cur = set_view(h, h->pc, h->mc);
    const ParticlesF64 cand = set_view(h, 1 - h->pc, 1 - h->mc);
    ++h->launches;
    launch_kick_drift_key_f64(n, cur, h->acc[0], h->acc[1], h->acc[2], K1, D, h->axis, cand,
                              h->sort, true, h->d_maxdrift, h->d_status, h->stream);
    // Positions / momenta of the force solve: the candidate set itself, in cell
    // order through the order index, or, on sort steps, the current set the
    // candidate is scattered into in cell order.
    int P = 1 - h->pc, M = 1 - h->mc;
    const int ic_before = h->ic;
    h->launches += launch_exclusive_scan(h->sort.count, h->sort.offset, h->sort.n_buckets + 1,
                                         h->sort.scan_tmp, h->stream);
    ++h->launches;
    launch_max_count_f64(h->sort.n_buckets, h->sort.count, h->d_max_count, h->stream);
    const uint32_t* order = nullptr;
    if (!sort_now) {
        ++h->launches;
        launch_order(n, h->sort.key, h->sort.rank, h->sort.offset, h->order, h->d_status,
                     h->stream);
        order = h->order;
    }
    if (sort_now) {
        const double* src[8];
        double* dst[8];
        int k = 0;
        src[k] = cand.x; dst[k++] = cur.x;
        src[k] = cand.y; dst[k++] = cur.y;
        src[k] = cand.z; dst[k++] = cur.z;
        src[k] = cand.px; dst[k++] = cur.px;
        src[k] = cand.py; dst[k++] = cur.py;
        src[k] = cand.pz; dst[k++] = cur.pz;
        if (h->has_masses) {
            src[k] = h->mass[h->ic];
            dst[k++] = h->mass[1 - h->ic];
        }
        const uint32_t* su[1] = {h->id[h->ic]};
        uint32_t* du[1] = {h->id[1 - h->ic]};
        ++h->launches;
        launch_scatter_multi(n, h->sort.key, h->sort.rank, h->sort.offset, k, src, dst, 1, su, du,
                             h->d_status, h->stream);
        P = h->pc;
        M = h->mc;
        h->ic = 1 - h->ic;
    }
    // Kernels after the candidate skip all writes when it failed (status gate).
    int rc = enqueue_force(h, P, M, true, K2, order);
    if (rc) return rc;
    unsigned int st = 0;
    rc = read_status(h, &st);
    if (rc) return rc;
    collect_timing(h);
    if (st & ST_BLOCKS_PUBLISH) {
        // Nothing was published: state is that of the step's start; the bucket
        // offsets now describe the unpublished candidate.
        h->ic = ic_before;
        h->order_state = 0;
        return status_to_code(h, st);
    }
    h->pc = P;
    h->order_state = sort_now ? 1 : 2;
    h->since_sort = sort_now ? 0 : h->since_sort + 1;
    if (st) {
        // Positions drifted and momenta K1-kicked are published; the force or
        // the K2 kick failed, so momenta stay at p' and acceleration is invalid.
        h->mc = M;
        h->acc_valid = false;
        return status_to_code(h, st);
    }
    h->mc = 1 - M;  // publish p''
    h->acc_valid = true;
    if (max_drift) {
        CK(cudaMemcpy(h->h_maxdrift, h->d_maxdrift, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        double d;
        std::memcpy(&d, h->h_maxdrift, sizeof(double));
        *max_drift = d;
    }
    return HYOWON_OK;
}

}  // namespace

extern "C" {

int hyowon_pm_create(double box_size, uint64_t mesh_size, int method, int deconvolve_cic,
                     double split_scale, int precision, hyowon_pm_t* out) {
    if (!out) return HYOWON_EINVAL;
    *out = nullptr;
    if (!std::isfinite(box_size) || box_size <= 0.0 || mesh_size < 2 || mesh_size > 2048)
        return HYOWON_EINVAL;
    if (method != HYOWON_PURE_PM && method != HYOWON_TREEPM_LONG_RANGE) return HYOWON_EINVAL;
    if (precision != HYOWON_FP64 && precision != HYOWON_FP32_FIXED) return HYOWON_EINVAL;
    if (method == HYOWON_TREEPM_LONG_RANGE && (!std::isfinite(split_scale) || split_scale <= 0.0))
        return HYOWON_EINVAL;
    hyowon_pm_t h = new (std::nothrow) hyowon_pm_s();
    if (!h) return HYOWON_ENOMEM;
    h->L = box_size;
    h->N = static_cast<int>(mesh_size);
    h->method = method;
    h->deconvolve = method == HYOWON_TREEPM_LONG_RANGE ? 1 : (deconvolve_cic ? 1 : 0);
    h->r_s = split_scale;
    h->precision = precision;
    const int N = h->N;
    h->axis.L = box_size;
    h->axis.dx = box_size / static_cast<double>(N);
    h->axis.upper = std::nextafter(static_cast<double>(N), 0.0);
    h->axis.N = N;
    h->four_pi_G = 4.0 * kPi * gravitational_constant();
    const double dx = h->axis.dx;
    const double inv_vol = 1.0 / (dx * dx * dx);
    const double norm = 1.0 / (static_cast<double>(N) * static_cast<double>(N) * static_cast<double>(N));
    h->field_scale = inv_vol * norm;

    auto bail = [&](int code) {
        hyowon_pm_destroy(h);
        return code;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess
        || cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(HYOWON_ECUDA);
    for (int b = 0; b < 2; ++b) {
        if (cudaEventCreateWithFlags(&h->staged[b], cudaEventDisableTiming) != cudaSuccess
            || cudaEventCreateWithFlags(&h->copied[b], cudaEventDisableTiming) != cudaSuccess)
            return bail(HYOWON_ECUDA);
    }
    if (cudaMallocHost(reinterpret_cast<void**>(&h->h_status), sizeof(unsigned int)) != cudaSuccess
        || cudaMallocHost(reinterpret_cast<void**>(&h->h_maxdrift), sizeof(unsigned long long)) != cudaSuccess
        || cudaMallocHost(reinterpret_cast<void**>(&h->h_max_count), sizeof(uint32_t)) != cudaSuccess
        || dalloc(&h->d_status, 1) != cudaSuccess || dalloc(&h->d_maxdrift, 1) != cudaSuccess
        || dalloc(&h->d_max_count, 1) != cudaSuccess
        || dalloc(&h->d_diag, diag::scratch_doubles()) != cudaSuccess)
        return bail(HYOWON_ENOMEM);
    for (auto& e : h->ev) {
        if (cudaEventCreate(&e) != cudaSuccess) return bail(HYOWON_ECUDA);
    }
    for (auto& e : h->call_ev) {
        if (cudaEventCreate(&e) != cudaSuccess) return bail(HYOWON_ECUDA);
    }

    // Green's-function 1-D tables on the host with the reference's formulas
    // (src/mesh/green_function.cpp:59-87,137-163) so the device symbol is
    // bit-identical to the reference's.
    std::vector<double> lap(N), win(N);
    {
        const double inv = 1.0 / dx;
        const double inv2 = inv * inv;
        const double nn = static_cast<double>(N);
        for (int i = 0; i < N; ++i) {
            const long long mode = i <= N / 2 ? i : static_cast<long long>(i) - N;
            const double s = std::sin(kPi * static_cast<double>(mode) / nn);
            lap[i] = -4.0 * inv2 * s * s;
            const long double arg = 3.141592653589793238462643383279502884L
                * static_cast<long double>(mode) / static_cast<long double>(N);
            if (arg == 0.0L) {
                win[i] = 1.0;
            } else {
                long double mag = std::fabs(std::sin(arg) / arg);
                if (mag > 1.0L) mag = 1.0L;
                win[i] = static_cast<double>(mag * mag);
            }
        }
    }
    if (dalloc(&h->lap, N) != cudaSuccess || dalloc(&h->win, N) != cudaSuccess) return bail(HYOWON_ENOMEM);
    cudaMemcpy(h->lap, lap.data(), sizeof(double) * N, cudaMemcpyHostToDevice);
    cudaMemcpy(h->win, win.data(), sizeof(double) * N, cudaMemcpyHostToDevice);

    if (precision == HYOWON_FP32_FIXED) {
        int rc = fp32::create(&h->f32, h->L, N, method, h->deconvolve, split_scale, lap.data(),
                              win.data(), h->four_pi_G, h->stream);
        if (rc) {
            if (h->f32) h->err = fp32::last_error(h->f32);
            return bail(rc);
        }
        *out = h;
        return HYOWON_OK;
    }

    const size_t cells = static_cast<size_t>(N) * N * N;
    const size_t half = static_cast<size_t>(N) * N * (N / 2 + 1);
    const size_t modes_n = method == HYOWON_PURE_PM && poisson::supported(N)
        ? std::max(half, poisson::modes_elements_f64(N)) : half;
    if (dalloc(&h->mesh, cells) != cudaSuccess || dalloc(&h->modes, modes_n) != cudaSuccess)
        return bail(HYOWON_ENOMEM);
    if (method == HYOWON_TREEPM_LONG_RANGE && dalloc(&h->phi_k, half) != cudaSuccess)
        return bail(HYOWON_ENOMEM);
    if (method == HYOWON_PURE_PM && poisson::supported(N)) {
        std::vector<double> t(2 * static_cast<size_t>(N));
        poisson::twiddles(N, t.data());
        if (dalloc(&h->tw, N) != cudaSuccess) return bail(HYOWON_ENOMEM);
        if (cudaMemcpy(h->tw, t.data(), sizeof(double2) * N, cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(HYOWON_ECUDA);
        const char* perr = "";
        h->fft_plan = poisson::create_plan(N, false, h->modes, &perr);
        if (!h->fft_plan) {
            h->err = perr;
            return bail(HYOWON_ECUDA);
        }
        h->five_pass = true;
        *out = h;
        return HYOWON_OK;
    }
    size_t ws1 = 0, ws2 = 0;
    if (cufftCreate(&h->plan_r2c) != CUFFT_SUCCESS || cufftCreate(&h->plan_c2r) != CUFFT_SUCCESS)
        return bail(HYOWON_ECUDA);
    h->plans = true;
    cufftSetAutoAllocation(h->plan_r2c, 0);
    cufftSetAutoAllocation(h->plan_c2r, 0);
    if (cufftMakePlan3d(h->plan_r2c, N, N, N, CUFFT_D2Z, &ws1) != CUFFT_SUCCESS
        || cufftMakePlan3d(h->plan_c2r, N, N, N, CUFFT_Z2D, &ws2) != CUFFT_SUCCESS)
        return bail(HYOWON_ECUDA);
    if (cudaMalloc(&h->fft_work, std::max<size_t>(1, std::max(ws1, ws2))) != cudaSuccess)
        return bail(HYOWON_ENOMEM);
    cufftSetWorkArea(h->plan_r2c, h->fft_work);
    cufftSetWorkArea(h->plan_c2r, h->fft_work);
    cufftSetStream(h->plan_r2c, h->stream);
    cufftSetStream(h->plan_c2r, h->stream);
    *out = h;
    return HYOWON_OK;
}

int hyowon_pm_destroy(hyowon_pm_t h) {
    if (!h) return HYOWON_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    hyowon::ic::workspace_destroy(h->ic_ws);
    hyowon::adj::destroy_cache(h->adj);
    if (h->f32) fp32::destroy(h->f32);
    if (h->plans) {
        cufftDestroy(h->plan_r2c);
        cufftDestroy(h->plan_c2r);
    }
    cudaFree(h->fft_work);
    cudaFree(h->tw);
    poisson::destroy_plan(h->fft_plan);
    cudaFree(h->mesh);
    cudaFree(h->modes);
    cudaFree(h->phi_k);
    cudaFree(h->lap);
    cudaFree(h->win);
    free_particles(h);
    cudaFree(h->tree_buf);
    hyowon::tree::destroy_workspace(h->tree_ws);
    cudaFree(h->sort.count);
    cudaFree(h->sort.offset);
    cudaFree(h->sort.scan_tmp);
    cudaFree(h->d_status);
    cudaFree(h->d_maxdrift);
    cudaFree(h->d_max_count);
    cudaFree(h->d_diag);
    if (h->h_status) cudaFreeHost(h->h_status);
    if (h->h_max_count) cudaFreeHost(h->h_max_count);
    if (h->h_maxdrift) cudaFreeHost(h->h_maxdrift);
    for (auto& e : h->ev) {
        if (e) cudaEventDestroy(e);
    }
    for (auto& e : h->call_ev) {
        if (e) cudaEventDestroy(e);
    }
    for (int b = 0; b < 2; ++b) {
        if (h->staged[b]) cudaEventDestroy(h->staged[b]);
        if (h->copied[b]) cudaEventDestroy(h->copied[b]);
    }
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return HYOWON_OK;
}

const char* hyowon_pm_last_error(hyowon_pm_t h) {
    if (!h) return "null handle";
    return h->err.c_str();
}

int hyowon_pm_upload(hyowon_pm_t h, uint64_t n64, const double* x, const double* y, const double* z,
                     const double* px, const double* py, const double* pz, const double* masses,
                     double uniform_mass) {
    release_ic_workspace(h);
    if (!h) return HYOWON_EINVAL;
    // no particles: PMSolver's exact input-mass identity throws std::runtime_error
    // for a zero particle count (src/gravity/pm_solver.cpp:664-679)
    if (n64 == 0)
        return fail(h, HYOWON_ERUNTIME, "PMSolver exact input mass identity must be finite and positive");
    if (n64 > 0xFFFFFFF0ull) return fail(h, HYOWON_EINVAL, "particle count must be at most 2^32-16");
    if (!x || !y || !z) return fail(h, HYOWON_EINVAL, "position arrays must be non-null");
    if (!masses && (!std::isfinite(uniform_mass) || uniform_mass <= 0.0))
        return fail(h, HYOWON_EINVAL, "PMSolver uniform mass must be finite and positive");
    const uint32_t n = static_cast<uint32_t>(n64);
    h->has_state = false;
    h->acc_valid = false;
    h->sorted = false;
    h->order_state = 0;
    // Input mass (pm_solver.cpp:87-118): uniform = correctly rounded m*n;
    // explicit masses summed in a wide accumulator.
    double total = 0.0;
    double max_mass = masses ? 0.0 : uniform_mass;
    if (masses) {
        long double s = 0.0L, c = 0.0L;
        for (uint32_t i = 0; i < n; ++i) {
            const double m = masses[i];
            if (!std::isfinite(m) || m < 0.0)
                return fail(h, HYOWON_EINVAL, "PMSolver explicit masses must be finite and non-negative");
            max_mass = m > max_mass ? m : max_mass;
            const long double t = s + m;
            c += (std::fabs(s) >= std::fabs(static_cast<long double>(m))) ? (s - t) + m : (m - t) + s;
            s = t;
        }
        total = static_cast<double>(s + c);
    } else {
        total = uniform_mass * static_cast<double>(n);
    }
    if (!std::isfinite(total) || total <= 0.0)
        return fail(h, HYOWON_ERUNTIME, "PMSolver exact input mass identity must be finite and positive");
    set_input_mass(h, total, n);
    h->max_mass = max_mass;
    h->uniform_mass = masses ? 0.0 : uniform_mass;
    h->has_masses = masses != nullptr;
    h->n = n;
    if (h->precision == HYOWON_FP32_FIXED) {
        int rc = fp32::upload(h->f32, n, x, y, z, px, py, pz, masses, uniform_mass, total,
                              h->mass_tol, h->stream);
        if (rc) return status_or_cuda(h, rc);
        CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream));
        fp32::validate(h->f32, h->stream, h->d_status);
        unsigned int st = 0;
        rc = read_status(h, &st);
        if (rc) return rc;
        if (st) return status_to_code(h, st);
        h->has_state = true;
        return HYOWON_OK;
    }
    int rc = ensure_capacity(h, n, masses != nullptr);
    if (rc) return rc;
    rc = ensure_sort_buckets(h, n);
    if (rc) return rc;
    h->pc = h->mc = h->ic = 0;
    CK(cudaMemcpyAsync(h->pos[0][0], x, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->pos[0][1], y, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->pos[0][2], z, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    const double* moms[3] = {px, py, pz};
    for (int a = 0; a < 3; ++a) {
        if (moms[a]) {
            CK(cudaMemcpyAsync(h->mom[0][a], moms[a], sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
        } else {
            CK(cudaMemsetAsync(h->mom[0][a], 0, sizeof(double) * n, h->stream));
        }
    }
    if (masses) CK(cudaMemcpyAsync(h->mass[0], masses, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    ++h->launches;
    launch_iota_u32(n, h->id[0], h->stream);
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream));
    ++h->launches;
    launch_validate_inputs_f64(n, h->pos[0][0], h->pos[0][1], h->pos[0][2],
                               masses ? h->mass[0] : nullptr, h->d_status, h->stream);
    unsigned int st = 0;
    rc = read_status(h, &st);
    if (rc) return rc;
    if (st) return status_to_code(h, st);
    h->has_state = true;
    return HYOWON_OK;
}

int hyowon_pm_lpt_ics(hyowon_pm_t h, uint64_t n_side, const double* noise, uint64_t n_nodes,
                      const double* ln_k, const double* ln_p, const double* ln_p_y2,
                      double momentum_factor, double uniform_mass) {
    release_ic_workspace(h);
    if (!h) return HYOWON_EINVAL;
    if (n_side < 2 || n_side > 2048 || !noise || n_nodes < 2 || !ln_k || !ln_p || !ln_p_y2)
        return fail(h, HYOWON_EINVAL, "LPT requires n_side in [2,2048], noise and a spline table");
    if (!std::isfinite(uniform_mass) || uniform_mass <= 0.0 || !std::isfinite(momentum_factor))
        return fail(h, HYOWON_EINVAL, "LPT uniform mass and momentum factor must be finite (mass positive)");
    const uint64_t n64 = n_side * n_side * n_side;
    if (n64 > 0xFFFFFFF0ull) return fail(h, HYOWON_EINVAL, "particle count exceeds 2^32-16");
    const uint32_t n = static_cast<uint32_t>(n64);
    const int N = static_cast<int>(n_side);
    h->has_state = h->acc_valid = h->sorted = false;
    h->order_state = 0;
    double* d_noise = nullptr;
    double* tab = nullptr;
    CK(dalloc(&d_noise, n64));
    CK(dalloc(&tab, 3 * n_nodes));
    int rc = HYOWON_OK;
    double* tmp_pos[3] = {};
    double* tmp_mom[3] = {};
    const char* err = nullptr;
    if (cudaMemcpy(d_noise, noise, sizeof(double) * n64, cudaMemcpyHostToDevice) != cudaSuccess
        || cudaMemcpy(tab, ln_k, sizeof(double) * n_nodes, cudaMemcpyHostToDevice) != cudaSuccess
        || cudaMemcpy(tab + n_nodes, ln_p, sizeof(double) * n_nodes, cudaMemcpyHostToDevice) != cudaSuccess
        || cudaMemcpy(tab + 2 * n_nodes, ln_p_y2, sizeof(double) * n_nodes, cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = fail(h, HYOWON_ECUDA, "LPT input copy failed");
    }
    if (rc == HYOWON_OK && h->precision == HYOWON_FP64) {
        rc = ensure_capacity(h, n, false);
        if (rc == HYOWON_OK) rc = ensure_sort_buckets(h, n);
        for (int a = 0; a < 3; ++a) {
            tmp_pos[a] = h->pos[0][a];
            tmp_mom[a] = h->mom[0][a];
        }
    } else if (rc == HYOWON_OK) {
        for (int a = 0; a < 3 && rc == HYOWON_OK; ++a) {
            if (dalloc(&tmp_pos[a], n) != cudaSuccess || dalloc(&tmp_mom[a], n) != cudaSuccess)
                rc = fail(h, HYOWON_ENOMEM, "LPT staging allocation failed");
        }
    }
    if (rc == HYOWON_OK) {
        cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream);
        const int lrc = lpt_ics_device(N, h->L, d_noise, tab, tab + n_nodes, tab + 2 * n_nodes,
                                       static_cast<int>(n_nodes), momentum_factor, tmp_pos,
                                       tmp_mom, h->d_status, h->stream, &err);
        if (lrc) rc = fail(h, lrc, err ? err : "LPT failed");
    }
    unsigned int st = 0;
    if (rc == HYOWON_OK) rc = read_status(h, &st);
    if (rc == HYOWON_OK && st)
        rc = fail(h, HYOWON_EINVAL, "LPT spectrum table does not cover the mesh wavenumbers");
    h->n = n;
    h->uniform_mass = uniform_mass;
    h->has_masses = false;
    set_input_mass(h, uniform_mass * static_cast<double>(n), n);
    h->max_mass = uniform_mass;
    if (rc == HYOWON_OK) {
        if (h->precision == HYOWON_FP64) {
            h->pc = h->mc = h->ic = 0;
            ++h->launches;
            launch_iota_u32(n, h->id[0], h->stream);
            if (cudaStreamSynchronize(h->stream) != cudaSuccess) rc = fail(h, HYOWON_ECUDA, "iota failed");
        } else {
            rc = status_or_cuda(h, fp32::upload_device(h->f32, n, tmp_pos, tmp_mom, uniform_mass,
                                                       h->input_mass, h->mass_tol, h->stream));
        }
    }
    if (h->precision != HYOWON_FP64) {
        for (int a = 0; a < 3; ++a) {
            cudaFree(tmp_pos[a]);
            cudaFree(tmp_mom[a]);
        }
    }
    cudaFree(d_noise);
    cudaFree(tab);
    if (rc == HYOWON_OK) h->has_state = true;
    return rc;
}

int hyowon_pm_generate_ics(hyowon_pm_t h, const hyowon_ic_params_t* p, uint64_t n_power,
                           const double* power, double uniform_mass) {
    if (!h) return HYOWON_EINVAL;
    hyowon::ic::Params r;
    const char* err = nullptr;
    int rc = hyowon::ic::resolve(p, &r, &err);
    if (rc) return fail(h, rc, err);
    if (!std::isfinite(uniform_mass) || uniform_mass <= 0.0)
        return fail(h, HYOWON_EINVAL, "uniform mass must be finite and positive");
    const uint64_t n64 = static_cast<uint64_t>(r.N) * r.N * r.N;
    if (n64 > 0xFFFFFFF0ull) return fail(h, HYOWON_EINVAL, "particle count exceeds 2^32-16");
    const uint32_t n = static_cast<uint32_t>(n64);
    double2* d_amp = nullptr;
    if ((rc = hyowon::ic::upload_amplitudes(r, n_power, power, &d_amp, &err))) return fail(h, rc, err);
    h->has_state = h->acc_valid = h->sorted = false;
    h->order_state = 0;
    double* tmp_pos[3] = {};
    double* tmp_mom[3] = {};
    if (h->precision == HYOWON_FP64) {
        rc = ensure_capacity(h, n, false);
        if (rc == HYOWON_OK) rc = ensure_sort_buckets(h, n);
        for (int a = 0; a < 3; ++a) {
            tmp_pos[a] = h->pos[0][a];
            tmp_mom[a] = h->mom[0][a];
        }
    } else {
        for (int a = 0; a < 3 && rc == HYOWON_OK; ++a) {
            if (dalloc(&tmp_pos[a], n) != cudaSuccess || dalloc(&tmp_mom[a], n) != cudaSuccess)
                rc = fail(h, HYOWON_ENOMEM, "IC staging allocation failed");
        }
    }
    if (rc == HYOWON_OK) {
        cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream);
        if (!h->ic_ws) h->ic_ws = hyowon::ic::workspace_create();
        const int grc = hyowon::ic::generate_device(r, d_amp, tmp_pos, tmp_mom, h->d_status,
                                                    h->stream, &err, h->ic_ws);
        if (grc) rc = fail(h, grc, err);
    }
    unsigned int st = 0;
    if (rc == HYOWON_OK) rc = read_status(h, &st);
    if (rc == HYOWON_OK && st) {
        const int src = hyowon::ic::status_code(st, &err);
        cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream);
        rc = fail(h, src, err);
    }
    h->n = n;
    h->uniform_mass = uniform_mass;
    h->has_masses = false;
    set_input_mass(h, uniform_mass * static_cast<double>(n), n);
    h->max_mass = uniform_mass;
    if (rc == HYOWON_OK) {
        if (h->precision == HYOWON_FP64) {
            h->pc = h->mc = h->ic = 0;
            ++h->launches;
            launch_iota_u32(n, h->id[0], h->stream);
            if (cudaStreamSynchronize(h->stream) != cudaSuccess) rc = fail(h, HYOWON_ECUDA, "iota failed");
        } else {
            rc = status_or_cuda(h, fp32::upload_device(h->f32, n, tmp_pos, tmp_mom, uniform_mass,
                                                       h->input_mass, h->mass_tol, h->stream));
        }
    }
    if (h->precision != HYOWON_FP64) {
        for (int a = 0; a < 3; ++a) {
            cudaFree(tmp_pos[a]);
            cudaFree(tmp_mom[a]);
        }
    }
    cudaFree(d_amp);
    if (rc == HYOWON_OK) h->has_state = true;
    return rc;
}

int hyowon_pm_download(hyowon_pm_t h, double* x, double* y, double* z, double* px, double* py,
                       double* pz, double* ax, double* ay, double* az) {
    if (!h) return HYOWON_EINVAL;
    if (!h->has_state) return fail(h, HYOWON_ELOGIC, "no particles uploaded");
    if ((ax || ay || az) && !h->acc_valid)
        return fail(h, HYOWON_ELOGIC, "accelerations are not valid (no successful force solve)");
    if (h->precision == HYOWON_FP32_FIXED) {
        int rc = fp32::download(h->f32, h->stream, x, y, z, px, py, pz, ax, ay, az);
        return status_or_cuda(h, rc);
    }
    const uint32_t n = h->n;
    // The spare position buffers are dead between calls: two of them stage
    // the reordered components, so that the reorder of one component on the
    // handle's stream overlaps the device-to-host copy of the previous one on
    // the copy stream.
    double* stage[2] = {h->pos[1 - h->pc][0], h->pos[1 - h->pc][1]};
    double* outs[9] = {x, y, z, px, py, pz, ax, ay, az};
    const double* srcs[9] = {h->pos[h->pc][0], h->pos[h->pc][1], h->pos[h->pc][2],
                             h->mom[h->mc][0], h->mom[h->mc][1], h->mom[h->mc][2],
                             h->acc[0], h->acc[1], h->acc[2]};
    int j = 0;
    for (int a = 0; a < 9; ++a) {
        if (!outs[a]) continue;
        const int b = j & 1;
        if (j >= 2) CK(cudaStreamWaitEvent(h->stream, h->copied[b], 0));
        ++h->launches;
        launch_unpermute_f64(n, h->id[h->ic], srcs[a], stage[b], h->stream);
        CK(cudaEventRecord(h->staged[b], h->stream));
        CK(cudaStreamWaitEvent(h->copy_stream, h->staged[b], 0));
        CK(cudaMemcpyAsync(outs[a], stage[b], sizeof(double) * n, cudaMemcpyDeviceToHost,
                           h->copy_stream));
        CK(cudaEventRecord(h->copied[b], h->copy_stream));
        ++j;
    }
    CK(cudaStreamSynchronize(h->copy_stream));
    CK(cudaStreamSynchronize(h->stream));
    return HYOWON_OK;
}

int hyowon_pm_snapshot_payload(hyowon_pm_t h, double a, double* coordinates,
                               double* velocities) {
    if (!h) return HYOWON_EINVAL;
    if (!h->has_state) return fail(h, HYOWON_ELOGIC, "no particles uploaded");
    if (!std::isfinite(a) || a <= 0.0)
        return fail(h, HYOWON_EINVAL, "Snapshot scale factor must be finite and positive");
    const double inv_a = 1.0 / a;
    if (!std::isfinite(inv_a) || inv_a <= 0.0)
        return fail(h, HYOWON_EOVERFLOW, "Snapshot inverse scale factor is not finite and positive");
    const uint32_t n = h->n;
    snapshot::Component pos[3], mom[3];
    const uint32_t* id = nullptr;
    double* stage = nullptr;
    uint64_t stage_doubles = 0;
    if (h->precision == HYOWON_FP32_FIXED) {
        fp32::snapshot_view(h->f32, pos, mom, &id, &stage, &stage_doubles);
    } else {
        for (int d = 0; d < 3; ++d) {
            pos[d] = {h->pos[h->pc][d], snapshot::kF64, 1.0};
            mom[d] = {h->mom[h->mc][d], snapshot::kF64, 1.0};
        }
        id = h->id[h->ic];
        const size_t half = static_cast<size_t>(h->N) * h->N * (h->N / 2 + 1);
        stage = reinterpret_cast<double*>(h->modes);   // dead between force solves
        stage_doubles = 2ull * half;
    }
    double* outs[2] = {coordinates, velocities};
    const int sets = (coordinates ? 1 : 0) + (velocities ? 1 : 0);
    if (sets == 0) return HYOWON_OK;
    // every requested dataset is staged and validated before any is copied
    const uint64_t need = 3ull * n * sets;
    double* owned = nullptr;
    if (stage_doubles < need) {
        CK(dalloc(&owned, need));
        stage = owned;
    }
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream));
    int rc = HYOWON_OK;
    int k = 0;
    for (int set = 0; set < 2 && rc == HYOWON_OK; ++set) {
        if (!outs[set]) continue;
        ++h->launches;
        if (snapshot::launch_rows(n, id, set == 0 ? pos : mom, set == 1, inv_a, h->L,
                                  stage + 3ull * n * k, h->d_status, h->stream) < 0)
            rc = fail(h, HYOWON_ECUDA, "snapshot staging launch failed");
        ++k;
    }
    unsigned int st = 0;
    if (rc == HYOWON_OK) rc = read_status(h, &st);
    if (rc == HYOWON_OK && st) {
        if (st & snapshot::kNonFinite)
            rc = fail(h, HYOWON_EINVAL, "Snapshot particle phase-space fields must be finite");
        else if (st & snapshot::kOutsideBox)
            rc = fail(h, HYOWON_EINVAL,
                      "Snapshot coordinates must lie in the periodic half-open interval [0,L)");
        else
            rc = fail(h, HYOWON_EOVERFLOW, "Snapshot momentum-to-velocity conversion overflowed");
    }
    k = 0;
    for (int set = 0; set < 2 && rc == HYOWON_OK; ++set) {
        if (!outs[set]) continue;
        if (cudaMemcpyAsync(outs[set], stage + 3ull * n * k, sizeof(double) * 3ull * n,
                            cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
            rc = fail(h, HYOWON_ECUDA, "snapshot copy failed");
        ++k;
    }
    if (cudaStreamSynchronize(h->stream) != cudaSuccess && rc == HYOWON_OK)
        rc = fail(h, HYOWON_ECUDA, "snapshot copy failed");
    cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream);
    cudaFree(owned);
    return rc;
}

int hyowon_pm_compute_forces(hyowon_pm_t h, double* ax, double* ay, double* az) {
    release_ic_workspace(h);
    if (!h) return HYOWON_EINVAL;
    if (!h->has_state) return fail(h, HYOWON_ELOGIC, "no particles uploaded");
    int rc;
    {
        CallTimer timer(h);
        rc = solve_force(h);
    }
    if (rc) return rc;
    if (!ax && !ay && !az) return HYOWON_OK;
    const uint32_t n = h->n;
    double* outs[3] = {ax, ay, az};
    std::vector<double> forces[3];
    for (int a = 0; a < 3; ++a) {
        if (outs[a]) forces[a].resize(n);
    }
    rc = hyowon_pm_download(h, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                            ax ? forces[0].data() : nullptr, ay ? forces[1].data() : nullptr,
                            az ? forces[2].data() : nullptr);
    if (rc) return rc;
    // validate_force_commit (pm_solver.cpp:281-326) before any add.
    for (int a = 0; a < 3; ++a) {
        if (!outs[a]) continue;
        for (uint32_t i = 0; i < n; ++i) {
            if (!std::isfinite(outs[a][i]) || !std::isfinite(outs[a][i] + forces[a][i]))
                return fail(h, HYOWON_EOVERFLOW, "PMSolver force commit is not representable");
        }
    }
    for (int a = 0; a < 3; ++a) {
        if (!outs[a]) continue;
        for (uint32_t i = 0; i < n; ++i) outs[a][i] += forces[a][i];
    }
    return HYOWON_OK;
}

int hyowon_pm_forces_host(hyowon_pm_t h, uint64_t n, const double* x, const double* y,
                          const double* z, const double* masses, double uniform_mass, double* ax,
                          double* ay, double* az) {
    release_ic_workspace(h);
    int rc = hyowon_pm_upload(h, n, x, y, z, nullptr, nullptr, nullptr, masses, uniform_mass);
    if (rc) return rc;
    return hyowon_pm_compute_forces(h, ax, ay, az);
}

int hyowon_pm_kdk_step(hyowon_pm_t h, double K1, double D, double K2, double* max_drift) {
    release_ic_workspace(h);
    if (!h) return HYOWON_EINVAL;
    CallTimer timer(h);
    return kdk_step_impl(h, K1, D, K2, max_drift);
}

int hyowon_pm_run(hyowon_pm_t h, uint64_t n_steps, const double* K1, const double* D,
                  const double* K2, double* max_drift) {
    release_ic_workspace(h);
    if (!h) return HYOWON_EINVAL;
    if (n_steps > 0 && (!K1 || !D || !K2)) return fail(h, HYOWON_EINVAL, "factor arrays must be non-null");
    CallTimer timer(h);
    for (uint64_t s = 0; s < n_steps; ++s) {
        int rc = kdk_step_impl(h, K1[s], D[s], K2[s], max_drift ? &max_drift[s] : nullptr);
        if (rc) {
            h->err = "step " + std::to_string(s) + ": " + h->err;
            return rc;
        }
    }
    return HYOWON_OK;
}

int hyowon_pm_info(hyowon_pm_t h, uint64_t* n_particles, uint64_t* mesh_size, int* precision,
                   int* method) {
    if (!h) return HYOWON_EINVAL;
    if (n_particles) *n_particles = h->n;
    if (mesh_size) *mesh_size = static_cast<uint64_t>(h->N);
    if (precision) *precision = h->precision;
    if (method) *method = h->method;
    return HYOWON_OK;
}

int hyowon_pm_download_potential(hyowon_pm_t h, double* phi) {
    if (!h || !phi) return HYOWON_EINVAL;
    if (h->method != HYOWON_PURE_PM) return fail(h, HYOWON_ELOGIC, "potential is kept only for pure PM");
    if (!h->acc_valid) return fail(h, HYOWON_ELOGIC, "no valid force solve");
    if (h->precision == HYOWON_FP32_FIXED) return status_or_cuda(h, fp32::download_potential(h->f32, h->stream, phi));
    const size_t cells = static_cast<size_t>(h->N) * h->N * h->N;
    CK(cudaMemcpy(phi, h->mesh, sizeof(double) * cells, cudaMemcpyDeviceToHost));
    return HYOWON_OK;
}

int hyowon_pm_download_mass_mesh(hyowon_pm_t h, double* mesh) {
    release_ic_workspace(h);
    if (!h || !mesh) return HYOWON_EINVAL;
    if (!h->has_state) return fail(h, HYOWON_ELOGIC, "no particles uploaded");
    if (!h->sorted) {
        int rc = h->precision == HYOWON_FP32_FIXED ? status_or_cuda(h, fp32::sort_current(h->f32, h->stream, h->d_status))
                                                   : sort_current(h);
        if (rc) return rc;
        h->sorted = true;
    }
    if (h->precision == HYOWON_FP32_FIXED)
        return status_or_cuda(h, fp32::download_mass_mesh(h->f32, h->stream, h->d_status, mesh));
    const size_t cells = static_cast<size_t>(h->N) * h->N * h->N;
    if (h->order_state == 0) {
        int rc = index_current(h);
        if (rc) return rc;
    }
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream));
    uint32_t max_count = 0;
    int rc0 = read_max_count(h, &max_count);
    if (rc0) return rc0;
    ++h->launches;
    CK(launch_deposit_tiles_f64(set_view(h, h->pc, h->mc), h->has_masses ? h->mass[h->ic] : nullptr,
                                h->uniform_mass, current_order(h), h->sort, h->axis,
                                h->d_max_count, max_count, deposit_mass_exponent_f64(h->max_mass),
                                h->mesh, nullptr, nullptr, h->d_status, h->stream));
    unsigned int st = 0;
    int rc = read_status(h, &st);
    if (rc) return rc;
    if (st) return status_to_code(h, st);
    CK(cudaMemcpy(mesh, h->mesh, sizeof(double) * cells, cudaMemcpyDeviceToHost));
    h->acc_valid = false;  // the potential buffer was overwritten
    return HYOWON_OK;
}

int hyowon_pm_cell_coords(hyowon_pm_t h, int64_t* base, double* frac) {
    if (!h || !base || !frac) return HYOWON_EINVAL;
    if (!h->has_state) return fail(h, HYOWON_ELOGIC, "no particles uploaded");
    if (h->precision == HYOWON_FP32_FIXED) return fail(h, HYOWON_ELOGIC, "cell coordinates of the binary64 form only");
    const uint32_t n = h->n;
    int64_t* db = nullptr;
    double* df = nullptr;
    double* stage = nullptr;
    CK(dalloc(&db, static_cast<size_t>(n)));
    CK(dalloc(&df, static_cast<size_t>(n)));
    CK(dalloc(&stage, static_cast<size_t>(n)));
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream));
    int rc = HYOWON_OK;
    for (int a = 0; a < 3 && rc == HYOWON_OK; ++a) {
        ++h->launches;
        launch_unpermute_f64(n, h->id[h->ic], h->pos[h->pc][a], stage, h->stream);
        ++h->launches;
        launch_cell_coords_f64(n, stage, h->axis, db, df, h->d_status, h->stream);
        if (cudaMemcpyAsync(base + static_cast<size_t>(a) * n, db, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess
            || cudaMemcpyAsync(frac + static_cast<size_t>(a) * n, df, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess
            || cudaStreamSynchronize(h->stream) != cudaSuccess)
            rc = fail(h, HYOWON_ECUDA, "cell coordinate copy failed");
    }
    cudaFree(db);
    cudaFree(df);
    cudaFree(stage);
    return rc;
}

int hyowon_pm_set_treepm_short_range(hyowon_pm_t h, double theta, double softening,
                                     double cutoff) {
    if (!h) return HYOWON_EINVAL;
    if (h->method != HYOWON_TREEPM_LONG_RANGE)
        return fail(h, HYOWON_EINVAL, "TreePM short range needs a HYOWON_TREEPM_LONG_RANGE handle");
    if (cutoff == 0.0) {
        h->treepm_short = false;
        if (h->f32) fp32::set_short_range_hook(h->f32, nullptr, nullptr);
        h->acc_valid = false;
        return HYOWON_OK;
    }
    if (!(std::isfinite(theta) && theta > 0.0) || !(std::isfinite(softening) && softening > 0.0)
        || !(std::isfinite(cutoff) && cutoff > 0.0 && cutoff < 0.5 * h->L))
        return fail(h, HYOWON_EINVAL,
                    "TreePM parameters must be finite and positive with r_cut < L/2");
    h->tp = hyowon_treepm_params{};
    h->tp.box_size = h->L;
    h->tp.split_scale = h->r_s;
    h->tp.cutoff = cutoff;
    h->tp.softening = softening;
    h->tp.theta = theta;
    h->tp.particle_mass = 1.0;   // the handle's mass at solve time is used
    h->tp.precision = h->precision;
    h->treepm_short = true;
    if (h->f32) fp32::set_short_range_hook(h->f32, short_range_hook_f32, h);
    h->acc_valid = false;
    return HYOWON_OK;
}

int hyowon_pm_treepm_short_forces(hyowon_pm_t h, double theta, double softening, double cutoff,
                                  double* ax, double* ay, double* az, double* stats) {
    release_ic_workspace(h);
    if (!h) return HYOWON_EINVAL;
    if (!h->has_state) return fail(h, HYOWON_ELOGIC, "no particles uploaded");
    if (h->method != HYOWON_TREEPM_LONG_RANGE)
        return fail(h, HYOWON_EINVAL, "TreePM short range needs a HYOWON_TREEPM_LONG_RANGE handle");
    if (!(std::isfinite(theta) && theta > 0.0) || !(std::isfinite(softening) && softening > 0.0)
        || !(std::isfinite(cutoff) && cutoff > 0.0 && cutoff < 0.5 * h->L))
        return fail(h, HYOWON_EINVAL,
                    "TreePM parameters must be finite and positive with r_cut < L/2");
    int rc = ensure_tree_buffer(h);
    if (rc) return rc;
    hyowon_treepm_params P{};
    P.box_size = h->L;
    P.split_scale = h->r_s;
    P.cutoff = cutoff;
    P.softening = softening;
    P.theta = theta;
    P.particle_mass = h->uniform_mass > 0.0 ? h->uniform_mass : 1.0;
    P.precision = h->precision;
    const size_t n = h->n;
    double* pos = h->tree_buf;
    double* out = h->tree_buf + 3 * n;
    const double *x, *y, *z;
    const double* masses = nullptr;
    const uint32_t* id;
    if (h->precision == HYOWON_FP32_FIXED) {
        rc = fp32::positions_f64(h->f32, h->stream, pos, pos + n, pos + 2 * n);
        if (rc) return status_or_cuda(h, rc);
        x = pos;
        y = pos + n;
        z = pos + 2 * n;
        id = fp32::current_ids(h->f32);
    } else {
        x = h->pos[h->pc][0];
        y = h->pos[h->pc][1];
        z = h->pos[h->pc][2];
        masses = h->has_masses ? h->mass[h->ic] : nullptr;
        id = h->id[h->ic];
    }
    CK(cudaMemsetAsync(out, 0, sizeof(double) * 3 * n, h->stream));
    std::string err;
    rc = tree::device_short_forces(P, h->n, x, y, z, masses, out, out + n, out + 2 * n, h->stream,
                                   stats, &err, h->tree_ws);
    if (rc) return fail(h, rc, "TreePM short range: " + err);
    double* host[3] = {ax, ay, az};
    for (int a = 0; a < 3; ++a) {
        if (!host[a]) continue;
        ++h->launches;
        launch_unpermute_f64(h->n, id, out + a * n, pos + a * n, h->stream);
        CK(cudaMemcpyAsync(host[a], pos + a * n, sizeof(double) * n, cudaMemcpyDeviceToHost,
                           h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    return HYOWON_OK;
}

int hyowon_pm_debug_set_wait_limit(hyowon_pm_t h, unsigned polls) {
    if (!h) return HYOWON_EINVAL;
    if (h->fft_plan) poisson::set_wait_limit(h->fft_plan, polls);
    if (h->f32) fp32::set_wait_limit(h->f32, polls);
    return HYOWON_OK;
}

int hyowon_pm_debug_offset_mass_target(hyowon_pm_t h, double delta) {
    if (!h || !std::isfinite(delta)) return HYOWON_EINVAL;
    h->mass_target_offset = delta;
    if (h->f32) {
        const double u = std::fabs(delta);
        fp32::set_mass_check_offset(h->f32, u >= 1.0 ? static_cast<unsigned long long>(u) : (delta != 0.0 ? 1ull : 0ull));
    }
    h->acc_valid = false;
    return HYOWON_OK;
}

int hyowon_pm_vjp(hyowon_pm_t h, const hyowon_vjp_config* cfg, const double* noise,
                  const double* target_delta, double* loss, double* grad_noise,
                  double* final_delta, double* timings) {
    release_ic_workspace(h);
    if (!h) return HYOWON_EINVAL;
    if (!cfg || !noise || !loss) return fail(h, HYOWON_EINVAL, "config, noise and loss must be non-null");
    if (h->method != HYOWON_PURE_PM)
        return fail(h, HYOWON_EINVAL, "the VJP differentiates the pure-PM step");
    hyowon_vjp_config c = *cfg;
    c.box_size = h->L;
    c.mesh_size = static_cast<uint64_t>(h->N);
    c.precision = h->precision;
    if (c.n_side < 2 || c.n_steps < 1 || !c.K1 || !c.D || !c.K2 || c.n_nodes < 2 || !c.ln_k
        || !c.ln_p || !c.ln_p_y2 || !(c.particle_mass > 0.0))
        return fail(h, HYOWON_EINVAL, "invalid VJP configuration");
    if (grad_noise && !target_delta)
        return fail(h, HYOWON_EINVAL, "the gradient needs a target density");
    std::string err;
    const int rc = hyowon::adj::run_cached(&h->adj, c, h->stream, noise, target_delta, loss,
                                           grad_noise, final_delta, timings, &err);
    return rc ? fail(h, rc, "VJP: " + err) : HYOWON_OK;
}

int hyowon_pm_set_sort_interval(hyowon_pm_t h, int steps) {
    if (!h || steps < 1) return HYOWON_EINVAL;
    h->sort_interval = steps;
    if (h->f32) fp32::set_sort_interval(h->f32, steps);
    return HYOWON_OK;
}

int hyowon_pm_set_timing(hyowon_pm_t h, int enabled) {
    if (!h) return HYOWON_EINVAL;
    h->timing = enabled != 0;
    return HYOWON_OK;
}

int hyowon_pm_last_timing(hyowon_pm_t h, double* times) {
    if (!h || !times) return HYOWON_EINVAL;
    for (int i = 0; i < 9; ++i) times[i] = h->last_times[i];
    return HYOWON_OK;
}


int hyowon_pm_diagnostics(hyowon_pm_t h, double a, hyowon_pm_diagnostics_t* out) {
    if (!h || !out) return HYOWON_EINVAL;
    if (!std::isfinite(a) || a <= 0.0)
        return fail(h, HYOWON_EINVAL, "diagnostics scale factor must be finite and positive");
    if (!h->has_state) return fail(h, HYOWON_ELOGIC, "no particles uploaded");
    if (!h->acc_valid)
        return fail(h, HYOWON_ELOGIC, "diagnostics need a valid force solve at the current positions");
    const bool with_phi = h->method == HYOWON_PURE_PM;
    double r[diag::kTerms] = {};
    if (h->precision == HYOWON_FP32_FIXED) {
        int rc = fp32::diagnostics(h->f32, h->stream, with_phi, h->d_diag, r);
        if (rc) return status_or_cuda(h, rc);
    } else {
        diag::InputsF64 in{};
        in.n = h->n;
        in.x = h->pos[h->pc][0];
        in.y = h->pos[h->pc][1];
        in.z = h->pos[h->pc][2];
        in.px = h->mom[h->mc][0];
        in.py = h->mom[h->mc][1];
        in.pz = h->mom[h->mc][2];
        in.ax = h->acc[0];
        in.ay = h->acc[1];
        in.az = h->acc[2];
        in.mass = h->has_masses ? h->mass[h->ic] : nullptr;
        in.uniform_mass = h->uniform_mass;
        in.phi = with_phi ? h->mesh : nullptr;
        in.axis = h->axis;
        CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned int), h->stream));
        const int k = diag::launch_f64(in, h->d_diag, h->d_status, h->stream);
        if (k < 0) return fail(h, HYOWON_ECUDA, "diagnostics launch failed");
        h->launches += k;
        CK(cudaMemcpyAsync(r, h->d_diag + diag::partial_doubles(), sizeof(r), cudaMemcpyDeviceToHost,
                           h->stream));
        unsigned int st = 0;
        int rc = read_status(h, &st);
        if (rc) return rc;
        if (st) return status_to_code(h, st);
    }
    const double nan = std::numeric_limits<double>::quiet_NaN();
    out->potential_energy_comoving = with_phi ? 0.5 * r[0] : nan;
    out->kinetic_energy = r[1] / (a * a);
    for (int d = 0; d < 3; ++d) {
        out->momentum[d] = r[2 + d];
        out->mass_weighted_force[d] = r[5 + d];
    }
    out->force_norm_sum = r[8];
    const double net = std::sqrt(r[5] * r[5] + r[6] * r[6] + r[7] * r[7]);
    out->force_balance = r[8] > 0.0 ? net / r[8] : 0.0;
    out->momentum_force_contraction = r[9];
    out->directional_potential_energy_comoving = with_phi ? r[10] : nan;
    for (int t = 1; t < 10; ++t)
        if (!std::isfinite(r[t])) return fail(h, HYOWON_EOVERFLOW, "diagnostic sum is non-finite");
    if (with_phi && !std::isfinite(r[10]))
        return fail(h, HYOWON_EOVERFLOW, "PMSolver post-force energy diagnostic is non-finite");
    if (with_phi && !std::isfinite(out->potential_energy_comoving))
        return fail(h, HYOWON_EOVERFLOW, "PMSolver potential-energy diagnostic is non-finite");
    if (with_phi && r[0] != 0.0 && out->potential_energy_comoving == 0.0)
        return fail(h, HYOWON_EUNDERFLOW, "PMSolver potential-energy diagnostic underflowed");
    return HYOWON_OK;
}

int hyowon_pm_power_spectrum(hyowon_pm_t h, uint64_t mesh_size, int num_bins,
                             double max_k_fraction_nyquist, int subtract_shot_noise,
                             int interlaced, hyowon_pk_bin_t* bins) {
    release_ic_workspace(h);
    if (!h || !bins) return HYOWON_EINVAL;
    if (!h->has_state) return fail(h, HYOWON_ELOGIC, "no particles uploaded");
    const uint64_t N = mesh_size ? mesh_size : static_cast<uint64_t>(h->N);
    if (N < 2 || N > 4096) return fail(h, HYOWON_EINVAL, "MatterPowerSpectrum mesh_size must be in [2, 4096]");
    if (num_bins < 1 || num_bins > 256)
        return fail(h, HYOWON_EINVAL, "MatterPowerSpectrum num_bins must be in [1, 256]");
    if (!std::isfinite(max_k_fraction_nyquist) || max_k_fraction_nyquist <= 0.0
        || max_k_fraction_nyquist > 1.0)
        return fail(h, HYOWON_EINVAL, "MatterPowerSpectrum max_k_fraction_nyquist must be in (0,1]");
    if (interlaced && subtract_shot_noise)
        return fail(h, HYOWON_EINVAL,
                    "Interlaced shot-noise subtraction is disabled until the estimator uses an "
                    "interlacing-matched alias model");
    const uint32_t n = h->n;
    double* pos = nullptr;       // widened positions of the precision form
    double* weights = nullptr;   // m_i / max m, explicit masses only
    double weight_sum = static_cast<double>(n);
    double msf = 1.0 / static_cast<double>(n);
    int rc = HYOWON_OK;
    const double *x = nullptr, *y = nullptr, *z = nullptr;
    if (h->precision == HYOWON_FP32_FIXED) {
        if (dalloc(&pos, 3ull * n) != cudaSuccess) return fail(h, HYOWON_ENOMEM, "power spectrum: staging");
        rc = status_or_cuda(h, fp32::positions_f64(h->f32, h->stream, pos, pos + n, pos + 2ull * n));
        x = pos;
        y = pos + n;
        z = pos + 2ull * n;
    } else {
        x = h->pos[h->pc][0];
        y = h->pos[h->pc][1];
        z = h->pos[h->pc][2];
        if (h->has_masses) {
            // FourierDensityBuilder::build: weights in units of the largest
            // mass, compensated sums of w and w^2 (fourier_density_field.cpp:170-230)
            std::vector<double> m(n);
            if (cudaMemcpyAsync(m.data(), h->mass[h->ic], sizeof(double) * n, cudaMemcpyDeviceToHost,
                                h->stream) != cudaSuccess
                || cudaStreamSynchronize(h->stream) != cudaSuccess)
                return fail(h, HYOWON_ECUDA, "power spectrum: mass copy failed");
            double unit = 0.0;
            for (double v : m) unit = std::max(unit, v);
            if (!(unit > 0.0) || !std::isfinite(unit))
                return fail(h, HYOWON_EINVAL, "FourierDensityBuilder masses must be finite and positive");
            long double s1 = 0.0L, c1 = 0.0L, s2 = 0.0L, c2 = 0.0L;
            auto add = [](long double& s, long double& c, long double v) {
                const long double t = s + v;
                c += std::fabs(s) >= std::fabs(v) ? (s - t) + v : (v - t) + s;
                s = t;
            };
            for (double& v : m) {
                v = v / unit;
                add(s1, c1, static_cast<long double>(v));
                add(s2, c2, static_cast<long double>(v) * static_cast<long double>(v));
            }
            const long double ws = s1 + c1;
            weight_sum = static_cast<double>(ws);
            msf = std::min(1.0, static_cast<double>((s2 + c2) / (ws * ws)));
            if (dalloc(&weights, n) != cudaSuccess
                || cudaMemcpyAsync(weights, m.data(), sizeof(double) * n, cudaMemcpyHostToDevice,
                                   h->stream) != cudaSuccess
                || cudaStreamSynchronize(h->stream) != cudaSuccess) {
                cudaFree(weights);
                return fail(h, HYOWON_ENOMEM, "power spectrum: weight staging");
            }
        }
    }
    if (rc == HYOWON_OK) {
        const pk::Request req{num_bins, max_k_fraction_nyquist, subtract_shot_noise != 0,
                              interlaced != 0};
        std::vector<pk::Bin> out(num_bins);
        std::string err;
        rc = pk::compute(h->L, static_cast<int>(N), n, x, y, z, weights, weight_sum, msf, req,
                         out.data(), &err, h->stream);
        if (rc) {
            fail(h, rc, err);
        } else {
            for (int b = 0; b < num_bins; ++b) {
                bins[b].k_low = out[b].k_low;
                bins[b].k_mean = out[b].k_mean;
                bins[b].k_high = out[b].k_high;
                bins[b].p_raw = out[b].p_raw;
                bins[b].p_corrected = out[b].p_corrected;
                bins[b].mean_cic_power_deconvolution_factor = out[b].mean_deconvolution;
                bins[b].shot_noise_reference = out[b].shot_noise;
                bins[b].mode_count = out[b].mode_count;
            }
        }
    }
    cudaFree(pos);
    cudaFree(weights);
    return rc;
}

}  // extern "C"
