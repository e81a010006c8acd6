"""The diagnostics restatement (oracle/diag_oracle.py) pinned to the
reference's own values (tests/golden/c1_diag.npz, made by
tests/golden/make_golden.py from PMSolver with collect_potential_energy,
ConservationChecks and compute_force_balance_diagnostics).

Tolerances: energies and the momentum-force contraction within 1e-13
relative (the reference sums in fixed blocks with compensation, the oracle
with math.fsum); the force balance R_F ~ 1e-17 within 1e-15 absolute.
"""
import numpy as np
import pytest

from oracle import diag_oracle as dg


def _phi(oracle, L, N, x, y, z, masses=None, uniform_mass=1.0):
    _, phi = oracle.potential(L, N, x, y, z, masses=masses, uniform_mass=uniform_mass)
    b = np.empty((3, x.size), dtype=np.int64)
    f = np.empty((3, x.size))
    for d, v in enumerate((x, y, z)):
        b[d], f[d] = oracle.cic_coords(L, N, v)
    return phi, b, f


@pytest.mark.parametrize("tag", ["ic", "s32"])
def test_c1_diagnostics_match_reference(oracle, c1_kdk, c1_diag, tag):
    d, g = c1_kdk, c1_diag
    L, N, m = float(d["box"]), int(d["mesh"]), float(d["particle_mass"])
    x, y, z = d[tag + "_x"], d[tag + "_y"], d[tag + "_z"]
    px, py, pz = d[tag + "_px"], d[tag + "_py"], d[tag + "_pz"]
    if tag == "ic":
        ax, ay, az = d["f0_x"], d["f0_y"], d["f0_z"]
    else:
        ax, ay, az = d["s32_ax"], d["s32_ay"], d["s32_az"]
    a = float(g[tag + "_a"])
    phi, b, f = _phi(oracle, L, N, x, y, z, uniform_mass=m)
    e = dg.potential_energy_comoving(L, N, phi, b, f, m)
    assert abs(e / float(g[tag + "_potential_energy"]) - 1) < 1e-13
    K = dg.kinetic_energy(px, py, pz, m, a)
    assert abs(K / float(g[tag + "_kinetic_energy"]) - 1) < 1e-13
    C = dg.momentum_force_contraction(px, py, pz, ax, ay, az, m)
    assert abs(C / float(g[tag + "_momentum_force_contraction"]) - 1) < 1e-13
    assert abs(dg.force_balance(ax, ay, az, m) - float(g[tag + "_force_balance"])) < 1e-15


def test_small_pm_masses_potential_energy(oracle, small_pm, c1_diag):
    s = small_pm
    L, N = float(s["L"]), int(s["N"])
    phi, b, f = _phi(oracle, L, N, s["x"], s["y"], s["z"], masses=s["masses"])
    e = dg.potential_energy_comoving(L, N, phi, b, f, s["masses"])
    assert abs(e / float(c1_diag["small_masses_potential_energy"]) - 1) < 1e-13


@pytest.mark.parametrize("tag", ["ic", "s32"])
def test_directional_derivative_matches_reference(oracle, c1_kdk, c1_diag, tag):
    """PMSolver::measure_post_force_energy_diagnostics_in_place: the one-sided
    CIC-weight directional derivative along the momenta, within 1e-15 of
    sum |term| (long-double per-particle terms as the reference forms them)."""
    d, g = c1_kdk, c1_diag
    L, N, m = float(d["box"]), int(d["mesh"]), float(d["particle_mass"])
    x, y, z = d[tag + "_x"], d[tag + "_y"], d[tag + "_z"]
    phi, b, f = _phi(oracle, L, N, x, y, z, uniform_mass=m)
    v, scale = dg.directional_potential_energy(L, N, phi, b, f, m, d[tag + "_px"],
                                               d[tag + "_py"], d[tag + "_pz"])
    assert abs(v - float(g[tag + "_directional"])) <= 1e-15 * scale
    assert float(g[tag + "_post_potential_energy"]) == float(g[tag + "_potential_energy"])


def test_directional_derivative_masses(oracle, small_pm, c1_diag):
    s_ = small_pm
    L, N = float(s_["L"]), int(s_["N"])
    phi, b, f = _phi(oracle, L, N, s_["x"], s_["y"], s_["z"], masses=s_["masses"])
    v, scale = dg.directional_potential_energy(L, N, phi, b, f, s_["masses"], c1_diag["small_px"],
                                               c1_diag["small_py"], c1_diag["small_pz"])
    assert abs(v - float(c1_diag["small_masses_directional"])) <= 1e-15 * scale
