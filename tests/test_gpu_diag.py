"""GPU tests of hyowon_pm_diagnostics (binary64 global sums of the device
state) against the reference's values (tests/golden/c1_diag.npz) and the
diagnostics oracle (oracle/diag_oracle.py) evaluated on the device's own
downloaded state.

Tolerances:
* binary64 form at the c1 ICs vs the reference: potential energy 1e-12
  relative (device forces/potential agree with the reference to 1e-12 of the
  field maximum), kinetic energy and momentum-force contraction 1e-13
  relative, force balance R_F ~ 1e-17 within 1e-14 absolute;
* either form vs the oracle on the same downloaded state: 1e-12 relative
  (binary64 sums of identical per-particle terms in another order);
* after 32 c1 steps vs the reference: 1e-5 relative (positions differ by
  <= 1e-6 cell after 32 chaotic steps);
* directional derivative sum m p . grad_S phi (sign-mixed): within 1e-12 of
  the sum of its terms' magnitudes vs the reference and the oracle (1e-10 for
  the precision form vs the oracle on its own state);
* repeated calls: bit-identical (fixed reduction order).
"""
import math

import numpy as np
import pytest

import hyowon_b200 as hb
from hyowon_b200 import _native as nat
from oracle import diag_oracle as dg

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a / b - 1.0)


def oracle_of_state(oracle, L, N, st, phi, masses, a):
    b = np.empty((3, st["x"].size), dtype=np.int64)
    f = np.empty((3, st["x"].size))
    for d, k in enumerate("xyz"):
        b[d], f[d] = oracle.cic_coords(L, N, st[k])
    return {
        "potential_energy_comoving": dg.potential_energy_comoving(L, N, phi, b, f, masses),
        "kinetic_energy": dg.kinetic_energy(st["px"], st["py"], st["pz"], masses, a),
        "momentum": dg.momentum(st["px"], st["py"], st["pz"], masses),
        "mass_weighted_force": dg.mass_weighted_force(st["ax"], st["ay"], st["az"], masses),
        "force_norm_sum": dg.force_norm_sum(st["ax"], st["ay"], st["az"], masses),
        "force_balance": dg.force_balance(st["ax"], st["ay"], st["az"], masses),
        "momentum_force_contraction": dg.momentum_force_contraction(
            st["px"], st["py"], st["pz"], st["ax"], st["ay"], st["az"], masses),
        "directional": dg.directional_potential_energy(L, N, phi, b, f, masses, st["px"],
                                                       st["py"], st["pz"]),
    }


def check_against(d, o, tol):
    for k in ("potential_energy_comoving", "kinetic_energy", "force_norm_sum",
              "momentum_force_contraction"):
        assert rel(d[k], o[k]) < tol, (k, d[k], o[k])
    scale_p = float(np.max(np.abs(o["momentum"]))) + 1e-300
    assert np.max(np.abs(d["momentum"] - o["momentum"])) <= tol * max(scale_p, 1.0)
    # net force and R_F are sums that cancel to rounding: absolute bounds
    assert np.max(np.abs(d["mass_weighted_force"] - o["mass_weighted_force"])) \
        <= 1e-12 * o["force_norm_sum"]
    assert abs(d["force_balance"] - o["force_balance"]) < 1e-12
    # sign-mixed sum: bounded by the sum of the magnitudes of its terms
    dv, scale = o["directional"]
    assert abs(d["directional_potential_energy_comoving"] - dv) <= tol * scale


def test_fp64_c1_ics_match_reference(oracle, c1_kdk, c1_diag):
    d, g = c1_kdk, c1_diag
    L, N, m = float(d["box"]), int(d["mesh"]), float(d["particle_mass"])
    a0 = float(d["a_start"])
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False)) as s:
        s.upload(d["ic_x"], d["ic_y"], d["ic_z"], d["ic_px"], d["ic_py"], d["ic_pz"],
                 uniform_mass=m)
        s.solve_forces()
        r1 = s.diagnostics(a0)
        r2 = s.diagnostics(a0)
        st = s.download()
        phi = s.potential()
    assert rel(r1["potential_energy_comoving"], float(g["ic_potential_energy"])) < 1e-12
    assert rel(r1["kinetic_energy"], float(g["ic_kinetic_energy"])) < 1e-13
    assert rel(r1["momentum_force_contraction"],
               float(g["ic_momentum_force_contraction"])) < 1e-12
    assert abs(r1["force_balance"] - float(g["ic_force_balance"])) < 1e-14
    o = oracle_of_state(oracle, L, N, st, phi, m, a0)
    assert abs(r1["directional_potential_energy_comoving"] - float(g["ic_directional"])) \
        <= 1e-12 * o["directional"][1]
    for k in r1:
        assert np.array_equal(np.asarray(r1[k]), np.asarray(r2[k])), k
    check_against(r1, oracle_of_state(oracle, L, N, st, phi, m, a0), 1e-12)
    print(f"c1 ICs: W {r1['potential_energy_comoving']:.12e} (ref "
          f"{float(g['ic_potential_energy']):.12e}), K {r1['kinetic_energy']:.12e}, "
          f"R_F {r1['force_balance']:.2e}")


def test_fp64_c1_after_32_steps(oracle, c1_kdk, c1_diag):
    d, g = c1_kdk, c1_diag
    L, N, m = float(d["box"]), int(d["mesh"]), float(d["particle_mass"])
    a0, dl = float(d["a_start"]), float(d["delta_ln_a"])
    K1, D, K2 = hb.TimeStepper(a0, 1.0, dl).factors()
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False)) as s:
        s.upload(d["ic_x"], d["ic_y"], d["ic_z"], d["ic_px"], d["ic_py"], d["ic_pz"],
                 uniform_mass=m)
        s.run(K1, D, K2)
        r = s.diagnostics(1.0)
        st = s.download()
        phi = s.potential()
    check_against(r, oracle_of_state(oracle, L, N, st, phi, m, 1.0), 1e-12)
    for k, gk in (("potential_energy_comoving", "s32_potential_energy"),
                  ("kinetic_energy", "s32_kinetic_energy"),
                  ("momentum_force_contraction", "s32_momentum_force_contraction")):
        assert rel(r[k], float(g[gk])) < 1e-5, (k, r[k], float(g[gk]))


def test_fp64_explicit_masses_collect_potential_energy(oracle, small_pm, c1_diag):
    s_ = small_pm
    L, N = float(s_["L"]), int(s_["N"])
    n = s_["x"].size
    ax, ay, az = np.zeros(n), np.zeros(n), np.zeros(n)
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False)) as s:
        out = s.compute_forces(s_["x"], s_["y"], s_["z"], s_["masses"], None, ax, ay, az,
                               collect_potential_energy=True)
        none = s.compute_forces(s_["x"], s_["y"], s_["z"], s_["masses"], None, ax, ay, az)
        r = s.diagnostics(1.0)
    assert none is None
    assert rel(out["potential_energy_comoving"],
               float(c1_diag["small_masses_potential_energy"])) < 1e-12
    assert abs(r["force_balance"] - float(c1_diag["small_masses_force_balance"])) < 1e-14
    # directional derivative along given momenta: upload them with the state
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False)) as s:
        s.upload(s_["x"], s_["y"], s_["z"], c1_diag["small_px"], c1_diag["small_py"],
                 c1_diag["small_pz"], masses=s_["masses"])
        s.solve_forces()
        r = s.diagnostics(1.0)
    _, phi = oracle.potential(L, N, s_["x"], s_["y"], s_["z"], masses=s_["masses"])
    b = np.empty((3, n), dtype=np.int64)
    f = np.empty((3, n))
    for d, v in enumerate((s_["x"], s_["y"], s_["z"])):
        b[d], f[d] = oracle.cic_coords(L, N, v)
    _, scale = dg.directional_potential_energy(L, N, phi, b, f, s_["masses"], c1_diag["small_px"],
                                               c1_diag["small_py"], c1_diag["small_pz"])
    ref = float(c1_diag["small_masses_directional"])
    assert abs(r["directional_potential_energy_comoving"] - ref) <= 1e-12 * scale


def test_fp32_matches_oracle_on_its_state(oracle, c1_kdk):
    d = c1_kdk
    L, N, m = float(d["box"]), int(d["mesh"]), float(d["particle_mass"])
    a0, dl = float(d["a_start"]), float(d["delta_ln_a"])
    K1, D, K2 = hb.TimeStepper(a0, 1.0, dl).factors()
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), "fp32") as s:
        s.upload(d["ic_x"], d["ic_y"], d["ic_z"], d["ic_px"], d["ic_py"], d["ic_pz"],
                 uniform_mass=m)
        s.run(K1[:8], D[:8], K2[:8])
        a = float(hb.TimeStepper(a0, 1.0, dl).steps[7].a_end)
        r1 = s.diagnostics(a)
        r2 = s.diagnostics(a)
        st = s.download()
        phi = s.potential()
    for k in r1:
        assert np.array_equal(np.asarray(r1[k]), np.asarray(r2[k])), k
    check_against(r1, oracle_of_state(oracle, L, N, st, phi, m, a), 1e-10)


def test_errors_and_treepm():
    rng = np.random.default_rng(5)
    L, N, n = 20.0, 16, 2000
    x, y, z = (rng.uniform(0, L, n) for _ in range(3))
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False)) as s:
        s.upload(x, y, z, uniform_mass=1.0)
        with pytest.raises(nat.HyowonLogicError):
            s.diagnostics(1.0)
        s.solve_forces()
        with pytest.raises(ValueError):
            s.diagnostics(0.0)
        with pytest.raises(ValueError):
            s.diagnostics(float("nan"))
        assert math.isfinite(s.diagnostics(0.5)["potential_energy_comoving"])
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.treepm_long_range(1.25 * L / N)) as s:
        s.upload(x, y, z, uniform_mass=1.0)
        s.solve_forces()
        r = s.diagnostics(1.0)
        assert math.isnan(r["potential_energy_comoving"])
        assert math.isnan(r["directional_potential_energy_comoving"])
        assert math.isfinite(r["force_norm_sum"]) and r["force_norm_sum"] > 0
