"""CPU restatement of HYOWON's global PM diagnostics (TEST INFRASTRUCTURE ONLY).

The checker for hyowon_pm_diagnostics. Only tests/ import it.

* ``potential_energy_comoving`` -- PMForceDiagnostics of
  PMSolver::compute_forces(..., collect_potential_energy=true)
  (src/gravity/pm_solver.cpp:812-840): 0.5 * sum_i m_i * value_i with
  value_i = sum over the 8 CIC corners (x, y, z offset nesting) of
  phi[corner] * ((wx * wy) * wz)
  (CICMassAssignment::interpolate_mass_weighted_sum_full_mesh,
  src/mesh/mass_assignment_gather.inc:283-391; the weight product is
  cic_weight_3d, src/mesh/cic_coordinate.hpp:26-38).
* ``kinetic_energy`` -- sum_i 0.5 m_i |p_i|^2 / a^2
  (ConservationChecks::compute_kinetic_energy,
  src/validation/conservation_checks.cpp:589-625,1376-1480).
* ``force_balance`` -- |sum_i m_i a_i| / sum_i m_i |a_i|
  (include/cosmo_nbody/validation/force_balance_diagnostics.hpp:19-27).
* ``momentum_force_contraction`` -- sum_i m_i p_i . a_i
  (src/validation/conservation_force_energy.cpp:148-200).

Sums use math.fsum (correctly rounded), so they are at least as accurate as
the reference's blocked compensated sums; agreement with the reference is to
rounding of the final sum, not bit for bit.
"""
from __future__ import annotations

import math

import numpy as np


def cic_interpolated_sum(L, N, phi, base, frac):
    """Per-particle CIC value sum_corners phi * ((wx*wy)*wz); base/frac are the
    reference's per-axis cell assignment (3, n) arrays."""
    phi = np.asarray(phi, dtype=np.float64).reshape(N, N, N)
    value = np.zeros(base.shape[1])
    for ox in (0, 1):
        wx = frac[0] if ox else 1.0 - frac[0]
        gx = (base[0] + ox) % N
        for oy in (0, 1):
            wy = frac[1] if oy else 1.0 - frac[1]
            gy = (base[1] + oy) % N
            xy = wx * wy
            for oz in (0, 1):
                wz = frac[2] if oz else 1.0 - frac[2]
                gz = (base[2] + oz) % N
                value = value + phi[gx, gy, gz] * (xy * wz)
    return value


def potential_energy_comoving(L, N, phi, base, frac, masses):
    value = cic_interpolated_sum(L, N, phi, base, frac)
    m = np.broadcast_to(np.asarray(masses, dtype=np.float64), value.shape)
    return 0.5 * math.fsum(m * value)


def kinetic_energy(px, py, pz, masses, a):
    m = np.broadcast_to(np.asarray(masses, dtype=np.float64), np.shape(px))
    return math.fsum(0.5 * m * (px * px + py * py + pz * pz)) / (a * a)


def momentum(px, py, pz, masses):
    m = np.broadcast_to(np.asarray(masses, dtype=np.float64), np.shape(px))
    return np.array([math.fsum(m * v) for v in (px, py, pz)])


def mass_weighted_force(ax, ay, az, masses):
    m = np.broadcast_to(np.asarray(masses, dtype=np.float64), np.shape(ax))
    return np.array([math.fsum(m * v) for v in (ax, ay, az)])


def force_norm_sum(ax, ay, az, masses):
    m = np.broadcast_to(np.asarray(masses, dtype=np.float64), np.shape(ax))
    return math.fsum(m * np.sqrt(ax * ax + ay * ay + az * az))


def force_balance(ax, ay, az, masses):
    net = mass_weighted_force(ax, ay, az, masses)
    den = force_norm_sum(ax, ay, az, masses)
    return float(np.sqrt(np.sum(net * net)) / den) if den > 0 else 0.0


def momentum_force_contraction(px, py, pz, ax, ay, az, masses):
    m = np.broadcast_to(np.asarray(masses, dtype=np.float64), np.shape(px))
    return math.fsum(m * (px * ax + py * ay + pz * az))


def directional_potential_energy(L, N, phi, base, frac, masses, px, py, pz):
    """sum_i m_i p_i . grad_S phi(x_i) with the one-sided CIC-weight gradient
    (CICMassAssignment::interpolate_mass_weighted_directional_derivative,
    src/mesh/mass_assignment_directional.cpp:133-180): per axis the sum over
    the other two axes' corners of (phi[+1] - phi[0]) w w, in long double,
    times 1 / dx (long double); the per-particle term m (p . g) rounded to
    binary64 (PMSolver::measure_post_force_energy_diagnostics_in_place,
    src/gravity/pm_post_force_energy_diagnostics.cpp:67-100)."""
    ld = np.longdouble
    phi = np.asarray(phi, dtype=np.float64).reshape(N, N, N)
    g = [(base[d] % N, (base[d] + 1) % N) for d in range(3)]
    v = np.empty((2, 2, 2, base.shape[1]), dtype=ld)
    for ox in (0, 1):
        for oy in (0, 1):
            for oz in (0, 1):
                v[ox, oy, oz] = phi[g[0][ox], g[1][oy], g[2][oz]].astype(ld)
    w = [np.stack([(1.0 - frac[d]), frac[d]]).astype(ld) for d in range(3)]
    gx = np.zeros(base.shape[1], dtype=ld)
    gy = np.zeros_like(gx)
    gz = np.zeros_like(gx)
    for a in (0, 1):
        for b in (0, 1):
            gx = gx + (v[1, a, b] - v[0, a, b]) * w[1][a] * w[2][b]
    for a in (0, 1):
        for b in (0, 1):
            gy = gy + (v[a, 1, b] - v[a, 0, b]) * w[0][a] * w[2][b]
    for a in (0, 1):
        for b in (0, 1):
            gz = gz + (v[a, b, 1] - v[a, b, 0]) * w[0][a] * w[1][b]
    inv = ld(1.0) / ld(L / N)
    gx, gy, gz = gx * inv, gy * inv, gz * inv
    m = np.broadcast_to(np.asarray(masses, dtype=np.float64), gx.shape).astype(ld)
    d = (np.asarray(px, dtype=np.float64).astype(ld) * gx
         + np.asarray(py, dtype=np.float64).astype(ld) * gy
         + np.asarray(pz, dtype=np.float64).astype(ld) * gz)
    terms = (m * d).astype(np.float64)
    return math.fsum(terms), math.fsum(np.abs(terms))
