// gpu_pm_solver.hpp -- header-only C++20 face of the C ABI in hyowon_pm.h,
// shaped like HYOWON's gravity::PMSolver and time::LeapfrogIntegrator so that a
// host written against those classes can switch to the device path.
//
// Status codes become the exception types the reference throws for the same
// condition (src/gravity/pm_solver.cpp:509-525 and :281-326,
// src/time/leapfrog_integrator.cpp:183-261):
//   HYOWON_EINVAL     -> std::invalid_argument
//   HYOWON_ELOGIC     -> std::logic_error
//   HYOWON_EOVERFLOW  -> std::overflow_error
//   HYOWON_EUNDERFLOW -> std::underflow_error
//   HYOWON_ERUNTIME   -> std::runtime_error
//   HYOWON_ECUDA      -> std::runtime_error ("CUDA: ...")
//   HYOWON_ENOMEM     -> std::bad_alloc
// Link with libhyowon_pm.so.
#pragma once

#include "hyowon_adjoint.h"
#include "hyowon_pm.h"
#include "hyowon_treepm.h"

#include <cstdint>
#include <new>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

namespace hyowon::b200 {

// gravity::PMForceDiagnostics (include/cosmo_nbody/gravity/pm_solver.hpp:30-35).
struct PMForceDiagnostics {
    double potential_energy_comoving = 0.0;
};

// gravity::PMPostForceEnergyDiagnostics (include/cosmo_nbody/gravity/pm_solver.hpp:37-46),
// the single-process fields.
struct PMPostForceEnergyDiagnostics {
    double potential_energy_comoving = 0.0;
    double directional_potential_energy_comoving = 0.0;
};

enum class Method { PurePM = HYOWON_PURE_PM, TreePMLongRange = HYOWON_TREEPM_LONG_RANGE };
enum class Precision { FP64 = HYOWON_FP64, FP32Fixed = HYOWON_FP32_FIXED };

inline void throw_on_status(int code, const char* what) {
    if (code == HYOWON_OK) return;
    const std::string msg = std::string("hyowon: ") + (what ? what : "");
    switch (code) {
    case HYOWON_EINVAL: throw std::invalid_argument(msg);
    case HYOWON_ELOGIC: throw std::logic_error(msg);
    case HYOWON_EOVERFLOW: throw std::overflow_error(msg);
    case HYOWON_EUNDERFLOW: throw std::underflow_error(msg);
    case HYOWON_ENOMEM: throw std::bad_alloc();
    case HYOWON_ECUDA: throw std::runtime_error("CUDA: " + msg);
    default: throw std::runtime_error(msg);
    }
}

// PMSolver(MeshGeometry{L, N}, PMForceMethod, ...) on one device. Owns the
// handle; movable, not copyable.
class GpuPMSolver {
public:
    GpuPMSolver(double box_size, std::uint64_t mesh_size, Method method = Method::PurePM,
                bool deconvolve_cic = false, double split_scale = 0.0,
                Precision precision = Precision::FP64) {
        const int rc = hyowon_pm_create(box_size, mesh_size, static_cast<int>(method),
                                        deconvolve_cic ? 1 : 0, split_scale,
                                        static_cast<int>(precision), &h_);
        throw_on_status(rc, rc == HYOWON_EINVAL ? "invalid PM solver configuration"
                                                : "PM solver creation failed");
    }
    GpuPMSolver(const GpuPMSolver&) = delete;
    GpuPMSolver& operator=(const GpuPMSolver&) = delete;
    GpuPMSolver(GpuPMSolver&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
    GpuPMSolver& operator=(GpuPMSolver&& o) noexcept {
        if (this != &o) {
            reset();
            h_ = o.h_;
            o.h_ = nullptr;
        }
        return *this;
    }
    ~GpuPMSolver() { reset(); }

    hyowon_pm_t handle() const noexcept { return h_; }

    // PMSolver::compute_forces (src/gravity/pm_solver.cpp:494-567) on host
    // spans: ADDS the PM acceleration to acc_*; masses empty means uniform_mass.
    // The device particle state is replaced by these positions.
    // With collect_potential_energy the reference's PMForceDiagnostics is
    // returned (0.5 sum_i m_i phi(x_i), src/gravity/pm_solver.cpp:812-840).
    std::optional<PMForceDiagnostics> compute_forces(
        std::span<const double> pos_x, std::span<const double> pos_y,
        std::span<const double> pos_z, std::span<const double> masses,
        std::optional<double> uniform_mass, std::span<double> acc_x, std::span<double> acc_y,
        std::span<double> acc_z, bool collect_potential_energy = false) {
        const std::size_t n = pos_x.size();
        if (pos_y.size() != n || pos_z.size() != n || acc_x.size() != n || acc_y.size() != n
            || acc_z.size() != n)
            throw std::invalid_argument("PMSolver: position/acceleration span sizes differ");
        if (masses.empty() == !uniform_mass.has_value() && n != 0)
            throw std::invalid_argument("PMSolver: give either masses or a uniform mass");
        if (!masses.empty() && masses.size() != n)
            throw std::invalid_argument("PMSolver: mass span size differs");
        check(hyowon_pm_forces_host(h_, n, pos_x.data(), pos_y.data(), pos_z.data(),
                                    masses.empty() ? nullptr : masses.data(),
                                    uniform_mass.value_or(0.0), acc_x.data(), acc_y.data(),
                                    acc_z.data()));
        if (!collect_potential_energy) return std::nullopt;
        return PMForceDiagnostics{diagnostics(1.0).potential_energy_comoving};
    }

    // Binary64 global sums of the state at the last force solve (kinetic and
    // potential energy, momentum, force balance; hyowon_pm_diagnostics).
    hyowon_pm_diagnostics_t diagnostics(double a) const {
        hyowon_pm_diagnostics_t d{};
        check(hyowon_pm_diagnostics(h_, a, &d));
        return d;
    }

    // PMSolver::measure_post_force_energy_diagnostics_in_place
    // (src/gravity/pm_post_force_energy_diagnostics.cpp:17-100) on the device
    // state: the potential of the last force solve at the current positions,
    // directional derivative along the current momenta. Pure PM only, as in
    // the reference (std::logic_error otherwise).
    PMPostForceEnergyDiagnostics measure_post_force_energy_diagnostics() const {
        const hyowon_pm_diagnostics_t d = diagnostics(1.0);
        if (d.directional_potential_energy_comoving != d.directional_potential_energy_comoving)
            throw std::logic_error(
                "PMSolver post-force energy diagnostic is defined only for pure PM");
        return {d.potential_energy_comoving, d.directional_potential_energy_comoving};
    }

    // /PartType1 Coordinates and Velocities rows (n x 3, original particle
    // order, velocities p / a) for the snapshot writer; either span may be
    // empty. hyowon_pm_snapshot_payload.
    void snapshot_payload(double a, std::span<double> coordinates, std::span<double> velocities) {
        check(hyowon_pm_snapshot_payload(h_, a, coordinates.empty() ? nullptr : coordinates.data(),
                                         velocities.empty() ? nullptr : velocities.data()));
    }

    // ParticleStore -> device. Momenta may be empty (zero).
    void upload(std::span<const double> x, std::span<const double> y, std::span<const double> z,
                std::span<const double> px, std::span<const double> py,
                std::span<const double> pz, std::span<const double> masses,
                std::optional<double> uniform_mass) {
        const std::size_t n = x.size();
        if (y.size() != n || z.size() != n || (!px.empty() && (px.size() != n || py.size() != n
                                                                || pz.size() != n)))
            throw std::invalid_argument("upload: span sizes differ");
        if (!masses.empty() && masses.size() != n)
            throw std::invalid_argument("upload: mass span size differs");
        check(hyowon_pm_upload(h_, n, x.data(), y.data(), z.data(),
                               px.empty() ? nullptr : px.data(),
                               py.empty() ? nullptr : py.data(),
                               pz.empty() ? nullptr : pz.data(),
                               masses.empty() ? nullptr : masses.data(),
                               uniform_mass.value_or(0.0)));
    }

    // Device -> host in the original particle order; empty spans are skipped.
    void download(std::span<double> x, std::span<double> y, std::span<double> z,
                  std::span<double> px = {}, std::span<double> py = {}, std::span<double> pz = {},
                  std::span<double> ax = {}, std::span<double> ay = {},
                  std::span<double> az = {}) {
        const std::uint64_t n = particle_count();
        for (auto s : {x, y, z, px, py, pz, ax, ay, az})
            if (!s.empty() && s.size() != n)
                throw std::invalid_argument("download: span size differs from particle count");
        auto p = [](std::span<double> s) { return s.empty() ? nullptr : s.data(); };
        check(hyowon_pm_download(h_, p(x), p(y), p(z), p(px), p(py), p(pz), p(ax), p(ay), p(az)));
    }

    // LeapfrogIntegrator::step (src/time/leapfrog_integrator.cpp:143-279) with
    // host-computed factors; returns max ||D p_half|| (the integrator's
    // last_step_max_drift_displacement).
    double kdk_step(double K1, double D, double K2) {
        double max_drift = 0.0;
        check(hyowon_pm_kdk_step(h_, K1, D, K2, &max_drift));
        return max_drift;
    }

    // Several steps without host work in between; returns per-step max drift.
    std::vector<double> run(std::span<const double> K1, std::span<const double> D,
                            std::span<const double> K2) {
        if (D.size() != K1.size() || K2.size() != K1.size())
            throw std::invalid_argument("run: factor span sizes differ");
        std::vector<double> drift(K1.size());
        check(hyowon_pm_run(h_, K1.size(), K1.data(), D.data(), K2.data(), drift.data()));
        return drift;
    }

    // TreePMSolver::compute_forces as the force of every later solve
    // (src/gravity/treepm_solver.cpp:631-717): the long range of a
    // Method::TreePMLongRange solver plus the octree short range; cutoff 0
    // returns to the long range alone. hyowon_pm_set_treepm_short_range.
    void set_treepm_short_range(double theta, double softening, double cutoff) {
        check(hyowon_pm_set_treepm_short_range(h_, theta, softening, cutoff));
    }

    // Short-range accelerations of the device state in particle order (spans of
    // the particle count, or empty to skip); stats as hyowon_treepm_short_forces.
    void treepm_short_forces(double theta, double softening, double cutoff,
                             std::span<double> ax, std::span<double> ay, std::span<double> az,
                             std::span<double> stats = {}) {
        if (!stats.empty() && stats.size() < 6)
            throw std::invalid_argument("treepm_short_forces: stats needs 6 entries");
        auto p = [](std::span<double> v) { return v.empty() ? nullptr : v.data(); };
        check(hyowon_pm_treepm_short_forces(h_, theta, softening, cutoff, p(ax), p(ay), p(az),
                                            p(stats)));
    }

    // Loss and d loss / d noise of the differentiable forward model on this
    // solver's box, mesh and form (hyowon_pm_vjp); returns the loss.
    double vjp(const hyowon_vjp_config& cfg, std::span<const double> noise,
               std::span<const double> target_delta, std::span<double> grad_noise) {
        double loss = 0.0;
        check(hyowon_pm_vjp(h_, &cfg, noise.data(),
                            target_delta.empty() ? nullptr : target_delta.data(), &loss,
                            grad_noise.empty() ? nullptr : grad_noise.data(), nullptr, nullptr));
        return loss;
    }

    std::uint64_t particle_count() const {
        std::uint64_t n = 0, mesh = 0;
        int prec = 0, meth = 0;
        check(hyowon_pm_info(h_, &n, &mesh, &prec, &meth));
        return n;
    }

private:
    hyowon_pm_t h_ = nullptr;

    void reset() noexcept {
        if (h_) hyowon_pm_destroy(h_);
        h_ = nullptr;
    }
    void check(int code) const { throw_on_status(code, hyowon_pm_last_error(h_)); }
};

}  // namespace hyowon::b200
