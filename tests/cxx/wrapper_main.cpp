// Drives hyowon::b200::GpuPMSolver the way a C++ host of the reference would.
//   wrapper_main invalid             -> prints the exception type of a bad config
//   wrapper_main forces IN OUT       -> IN: u64 n, u64 N, f64 L, f64 m, x[n], y[n], z[n]
//                                       OUT: ax[n], ay[n], az[n] (added to zero)
//   wrapper_main post IN OUT         -> IN: as forces, then px[n], py[n], pz[n]
//                                       OUT: {potential energy, directional derivative}
//                                       after upload + a zero KDK step, then the
//                                       snapshot rows coordinates[3n], velocities[3n] at a = 0.5
//   wrapper_main treepm IN OUT       -> IN: u64 n, u64 N, f64 L, f64 r_s, f64 theta, f64 eps,
//                                       f64 r_cut, masses[n], x[n], y[n], z[n], px[n], py[n],
//                                       pz[n]; a TreePM solver (long range + short range)
//                                       KDK step (K1, D, K2) = (1e-3, 1e-3, 1e-3)
//                                       OUT: x[n], y[n], z[n], ax[n], ay[n], az[n], then the
//                                       short-range part alone at the final state ax..az
#include "gpu_pm_solver.hpp"

#include <cstdio>
#include <fstream>
#include <iostream>
#include <typeinfo>
#include <vector>

using hyowon::b200::GpuPMSolver;

int main(int argc, char** argv) {
    if (argc >= 2 && std::string(argv[1]) == "invalid") {
        try {
            GpuPMSolver s(-1.0, 64);
        } catch (const std::invalid_argument&) {
            std::cout << "invalid_argument\n";
            return 0;
        } catch (const std::exception& e) {
            std::cout << "other: " << e.what() << "\n";
            return 1;
        }
        std::cout << "no exception\n";
        return 1;
    }
    if (argc == 4 && std::string(argv[1]) == "forces") {
        std::ifstream in(argv[2], std::ios::binary);
        std::uint64_t n = 0, N = 0;
        double L = 0.0, m = 0.0;
        in.read(reinterpret_cast<char*>(&n), 8);
        in.read(reinterpret_cast<char*>(&N), 8);
        in.read(reinterpret_cast<char*>(&L), 8);
        in.read(reinterpret_cast<char*>(&m), 8);
        std::vector<double> x(n), y(n), z(n), ax(n, 0.0), ay(n, 0.0), az(n, 0.0);
        in.read(reinterpret_cast<char*>(x.data()), 8 * n);
        in.read(reinterpret_cast<char*>(y.data()), 8 * n);
        in.read(reinterpret_cast<char*>(z.data()), 8 * n);
        if (!in) return 2;
        try {
            GpuPMSolver s(L, N);
            s.compute_forces(x, y, z, {}, m, ax, ay, az);
            // a second solve adds the same force again (PMSolver add semantics)
            s.compute_forces(x, y, z, {}, m, ax, ay, az);
        } catch (const std::exception& e) {
            std::cerr << typeid(e).name() << ": " << e.what() << "\n";
            return 3;
        }
        std::ofstream out(argv[3], std::ios::binary);
        out.write(reinterpret_cast<const char*>(ax.data()), 8 * n);
        out.write(reinterpret_cast<const char*>(ay.data()), 8 * n);
        out.write(reinterpret_cast<const char*>(az.data()), 8 * n);
        return out ? 0 : 4;
    }
    if (argc == 4 && std::string(argv[1]) == "post") {
        std::ifstream in(argv[2], std::ios::binary);
        std::uint64_t n = 0, N = 0;
        double L = 0.0, m = 0.0;
        in.read(reinterpret_cast<char*>(&n), 8);
        in.read(reinterpret_cast<char*>(&N), 8);
        in.read(reinterpret_cast<char*>(&L), 8);
        in.read(reinterpret_cast<char*>(&m), 8);
        std::vector<std::vector<double>> c(6, std::vector<double>(n));
        for (auto& v : c) in.read(reinterpret_cast<char*>(v.data()), 8 * n);
        if (!in) return 2;
        std::vector<double> coords(3 * n), vel(3 * n);
        double out2[2] = {};
        try {
            GpuPMSolver s(L, N);
            s.upload(c[0], c[1], c[2], c[3], c[4], c[5], {}, m);
            s.kdk_step(0.0, 0.0, 0.0);   // force at the uploaded positions, state unchanged
            const auto d = s.measure_post_force_energy_diagnostics();
            out2[0] = d.potential_energy_comoving;
            out2[1] = d.directional_potential_energy_comoving;
            s.snapshot_payload(0.5, coords, vel);
        } catch (const std::exception& e) {
            std::cerr << typeid(e).name() << ": " << e.what() << "\n";
            return 3;
        }
        std::ofstream out(argv[3], std::ios::binary);
        out.write(reinterpret_cast<const char*>(out2), 16);
        out.write(reinterpret_cast<const char*>(coords.data()), 8 * 3 * n);
        out.write(reinterpret_cast<const char*>(vel.data()), 8 * 3 * n);
        return out ? 0 : 4;
    }
    if (argc == 4 && std::string(argv[1]) == "treepm") {
        std::ifstream in(argv[2], std::ios::binary);
        std::uint64_t n = 0, N = 0;
        double prm[5] = {};
        in.read(reinterpret_cast<char*>(&n), 8);
        in.read(reinterpret_cast<char*>(&N), 8);
        in.read(reinterpret_cast<char*>(prm), 40);
        const double L = prm[0], r_s = prm[1], theta = prm[2], eps = prm[3], r_cut = prm[4];
        std::vector<std::vector<double>> c(7, std::vector<double>(n));
        for (auto& v : c) in.read(reinterpret_cast<char*>(v.data()), 8 * n);
        if (!in) return 2;
        std::vector<std::vector<double>> o(9, std::vector<double>(n));
        try {
            using hyowon::b200::Method;
            GpuPMSolver s(L, N, Method::TreePMLongRange, true, r_s);
            s.set_treepm_short_range(theta, eps, r_cut);
            s.upload(c[1], c[2], c[3], c[4], c[5], c[6], c[0], std::nullopt);
            s.kdk_step(1e-3, 1e-3, 1e-3);
            s.download(o[0], o[1], o[2], {}, {}, {}, o[3], o[4], o[5]);
            s.treepm_short_forces(theta, eps, r_cut, o[6], o[7], o[8]);
        } catch (const std::exception& e) {
            std::cerr << typeid(e).name() << ": " << e.what() << "\n";
            return 3;
        }
        std::ofstream out(argv[3], std::ios::binary);
        for (const auto& v : o) out.write(reinterpret_cast<const char*>(v.data()), 8 * n);
        return out ? 0 : 4;
    }
    std::cerr << "usage: wrapper_main invalid | forces IN OUT | post IN OUT | treepm IN OUT\n";
    return 64;
}
