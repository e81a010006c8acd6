// pm_fp32.h -- the precision form of the PM step (internal interface).
//
// Positions are 32-bit periodic fixed-point lattice coordinates u, with
// x = u * L / 2^32; the cell of u on an N mesh is floor(u*N / 2^32) and its CIC
// fraction the low 32 bits of u*N. Mass is deposited as int64 fixed-point
// offsets from the mean cell mass (deterministic integer atomics), converted to
// FP32 for the R2C transform; the Green's multiply, C2R and gather run in FP32;
// momenta are FP32; the drift p*D is formed in FP64 and rounded once into the
// fixed-point position.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "pm_snapshot.h"

struct hyowon_pm_s;

namespace hyowon {

int status_or_cuda(hyowon_pm_s* h, int rc);

namespace fp32 {

struct State;

// TreePM short-range hook (see set_short_range_hook).
using ShortRangeHook = int (*)(void* ctx, cudaStream_t s, int position_set);

int create(State** out, double L, int N, int method, int deconvolve, double r_s,
           const double* lap, const double* win, double four_pi_G, cudaStream_t s);
void destroy(State* st);
const std::string& last_error(State* st);

int upload(State* st, uint32_t n, const double* x, const double* y, const double* z,
           const double* px, const double* py, const double* pz, const double* masses,
           double uniform_mass, double total_mass, double mass_tol, cudaStream_t s);
// Same as upload from device-resident binary64 arrays (LPT initial conditions).
int upload_device(State* st, uint32_t n, double* const pos[3], double* const mom[3],
                  double uniform_mass, double total_mass, double mass_tol, cudaStream_t s);
void validate(State* st, cudaStream_t s, unsigned int* d_status);
int sort_current(State* st, cudaStream_t s, unsigned int* d_status);
int enqueue_force(State* st, cudaStream_t s, unsigned int* d_status, bool kick, double K2,
                  cudaEvent_t* ev);
int kdk_step(State* st, cudaStream_t s, unsigned int* d_status,
             unsigned long long* d_maxdrift, double K1, double D, double K2,
             cudaEvent_t* ev);
void set_sort_interval(State* st, int steps);
uint64_t launches(const State* st);
// Host bookkeeping after a kdk_step: `published` when the drift was published,
// `ok` when the whole step succeeded.
void commit_step(State* st, bool published, bool ok);
int download(State* st, cudaStream_t s, double* x, double* y, double* z, double* px,
             double* py, double* pz, double* ax, double* ay, double* az);
int download_potential(State* st, cudaStream_t s, double* phi);
// Global binary64 sums of the current state (pm_diag.h order) into host
// sums[kTerms], using the device scratch `scratch` (diag::scratch_doubles()).
int diagnostics(State* st, cudaStream_t s, bool with_potential, double* scratch, double* sums);
// Positions widened to binary64 (x = u L / 2^32, exact) into device arrays of
// the particle count, in the current storage order.
int positions_f64(State* st, cudaStream_t s, double* x, double* y, double* z);
int download_mass_mesh(State* st, cudaStream_t s, unsigned int* d_status, double* mesh);
// Positions of set P (0/1) widened to binary64.
int positions_f64_of_set(State* st, cudaStream_t s, int P, double* x, double* y, double* z);
// acc[i] += (float) a[i] for the accelerations of the solve in flight.
int add_accelerations(State* st, cudaStream_t s, const double* ax, const double* ay,
                      const double* az);
// TreePM long-range solves call fn(ctx, s, P) after the three long-range
// gathers and before the K2 kick, P the position set of the solve; fn adds the
// short-range accelerations (add_accelerations). A non-zero return aborts the
// solve with that status. fn null: long range alone.
void set_short_range_hook(State* st, ShortRangeHook fn, void* ctx);
// Failure-path tests: the expected fixed-point mesh sum is moved by `units`
// (0 restores the exact check), and the column passes' pipeline waits give up
// after `polls` polls.
void set_mass_check_offset(State* st, unsigned long long units);
void set_wait_limit(State* st, unsigned polls);
// slot -> particle index of the current storage order.
const uint32_t* current_ids(State* st);
// The device state as snapshot components (positions as u32 fixed point,
// momenta FP32), the slot -> particle index, and the staging area available
// between force solves (the half-spectrum buffer, *stage_doubles doubles).
void snapshot_view(State* st, snapshot::Component pos[3], snapshot::Component mom[3],
                   const uint32_t** id, double** stage, uint64_t* stage_doubles);

}  // namespace fp32
}  // namespace hyowon
