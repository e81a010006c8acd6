// pm_fp32.cu -- precision form of the PM step (see pm_fp32.h).
#include "hyowon_pm.h"
#include "pm_fp32.h"

namespace hyowon::fp32 {

struct State {
    std::string err = "the FP32 fixed-point form is not available in this build";
};

int create(State** out, double, int, int, int, double, const double*, const double*, double,
           cudaStream_t) {
    *out = new State();
    return HYOWON_EINVAL;
}
void destroy(State* st) { delete st; }
const std::string& last_error(State* st) { return st->err; }
int upload(State*, uint32_t, const double*, const double*, const double*, const double*,
           const double*, const double*, const double*, double, double, double, cudaStream_t) {
    return HYOWON_EINVAL;
}
int upload_device(State*, uint32_t, double* const*, double* const*, double, double, double,
                  cudaStream_t) {
    return HYOWON_EINVAL;
}
void validate(State*, cudaStream_t, unsigned int*) {}
int sort_current(State*, cudaStream_t, unsigned int*) { return HYOWON_EINVAL; }
int enqueue_force(State*, cudaStream_t, unsigned int*, bool, double, cudaEvent_t*) {
    return HYOWON_EINVAL;
}
int kdk_step(State*, cudaStream_t, unsigned int*, unsigned long long*, double, double, double,
             cudaEvent_t*) {
    return HYOWON_EINVAL;
}
void commit_step(State*, bool, bool) {}
int download(State*, cudaStream_t, double*, double*, double*, double*, double*, double*, double*,
             double*, double*) {
    return HYOWON_EINVAL;
}
int download_potential(State*, cudaStream_t, double*) { return HYOWON_EINVAL; }
int download_mass_mesh(State*, cudaStream_t, unsigned int*, double*) { return HYOWON_EINVAL; }

}  // namespace hyowon::fp32
