// pm_adjoint.h -- the differentiation form on a PM handle (internal).
#pragma once

#include <string>

#include <cuda_runtime.h>

#include "hyowon_adjoint.h"

namespace hyowon::adj {

// Adjoint engines (plans and work arrays) a handle keeps between VJP calls.
struct Cache;
void destroy_cache(Cache* c);
// hyowon_vjp_1lpt_pm on stream s with the engine of *cache (created, or
// re-created when the geometry changed). Returns a hyowon_status code.
int run_cached(Cache** cache, const VjpConfig& cfg, cudaStream_t s, const double* noise,
               const double* target_delta, double* loss, double* grad_noise,
               double* final_delta, double* timings, std::string* err);

}  // namespace hyowon::adj
