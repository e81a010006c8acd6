"""GPU tests of the TreePM pieces.

* Long range (spectral -ik PM, continuum Green's function, Gaussian split,
  W^-2): binary64 vs the reference's own PMSolver in TreePM mode, max error
  <= 1e-12 of the largest force; precision form <= 1e-4 relative RMS.
* Short range (octree walk): with a tiny opening angle every node is opened,
  so the walk must reproduce direct summation to 1e-12 (binary64); at
  theta = 0.5 it must reproduce the reference's own Octree + TreeWalk (same
  tree, same acceptance decisions) to 1e-10 relative RMS in binary64 and 1e-4
  in FP32, and its approximation error vs direct summation must equal the
  reference tree's to 1e-6 of that error.
* The c5 workload (256^3 particles, clustered z = 0 state of a 64-step PM run,
  seed 5): 4096 seeded random targets vs direct summation within the cutoff
  plus the long-range PM part: short-range relative RMS <= 1e-2, total force
  relative RMS <= 5e-3 (the theta = 0.5 monopole error).
"""
import math

import numpy as np
import pytest

import hyowon_b200 as hb
from hyowon_b200 import ic
from hyowon_b200.treepm import short_range_forces

pytestmark = pytest.mark.gpu


def rel_rms(got, ref):
    g = np.stack(got)
    r = np.stack(ref)
    return float(np.sqrt(np.sum((g - r) ** 2) / np.sum(r ** 2)))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-4)])
def test_long_range_pm_matches_reference(small_pm, precision, tol):
    g = small_pm
    L, N = float(g["L"]), int(g["N"])
    if precision == "fp32":
        L, N = float(g["L"]), int(g["N"])
    method = hb.PMForceMethod.treepm_long_range(float(g["tl_r_s"]))
    with hb.PMSolver(hb.MeshGeometry(L, N), method, precision) as s:
        s.upload(g["x"], g["y"], g["z"], uniform_mass=float(g["uniform_mass"]))
        s.solve_forces()
        out = s.download()
    ref = (g["tl_x"], g["tl_y"], g["tl_z"])
    got = (out["ax"], out["ay"], out["az"])
    if precision == "fp64":
        scale = max(np.max(np.abs(r)) for r in ref)
        assert max(np.max(np.abs(a - b)) for a, b in zip(got, ref)) <= tol * scale
    else:
        assert rel_rms(got, ref) <= tol


def uniform(n_side, L, seed):
    rng = np.random.default_rng(seed)
    return tuple(rng.uniform(0, L, n_side ** 3) for _ in range(3))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_walk_with_tiny_opening_angle_is_direct_summation(oracle, precision):
    L, n_side = 24.0, 24
    x, y, z = uniform(n_side, L, 1)
    targets = np.random.default_rng(2).choice(x.size, 512, replace=False).astype(np.uint32)
    r_s, r_cut, eps, m = 1.0, 4.5, 1.0 / 30.0, 1.0
    ref = oracle.short_range_direct(L, x, y, z, m, targets, r_s, r_cut, eps)
    ax, ay, az, info = short_range_forces(L, x, y, z, m, targets, r_s, r_cut, eps,
                                          theta=1e-6, precision=precision)
    err = rel_rms((ax, ay, az), ref)
    print(f"theta->0 walk ({precision}) vs direct: rel RMS {err:.3e}, {info}")
    assert err <= (1e-12 if precision == "fp64" else 1e-5)


@pytest.mark.parametrize("case", ["u", "c"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-4)])
def test_walk_matches_reference_tree(c1_kdk, case, precision, tol):
    """Same octree, same acceptance decisions: the reference's own Octree +
    TreeWalk at theta = 0.5 on a uniform and on a clustered (c1 z = 0) input."""
    from conftest import load_golden
    g = load_golden("treepm_tree.npz")
    if case == "u":
        L, x, y, z, m = float(g["u_L"]), g["u_x"], g["u_y"], g["u_z"], float(g["u_mass"])
    else:
        c = c1_kdk
        L, x, y, z, m = float(c["box"]), c["s32_x"], c["s32_y"], c["s32_z"], float(c["particle_mass"])
    ref = (g[case + "_ax"], g[case + "_ay"], g[case + "_az"])
    ax, ay, az, info = short_range_forces(L, x, y, z, m, g[case + "_targets"],
                                          float(g[case + "_r_s"]), float(g[case + "_r_cut"]),
                                          float(g[case + "_eps"]), 0.5, precision)
    err = rel_rms((ax, ay, az), ref)
    print(f"tree ({case}, {precision}) vs reference tree: rel RMS {err:.3e}; {info}")
    assert err <= tol


def test_walk_theta_half_error_equals_reference_tree_error(oracle):
    from conftest import load_golden
    g = load_golden("treepm_tree.npz")
    L, x, y, z = float(g["u_L"]), g["u_x"], g["u_y"], g["u_z"]
    t = g["u_targets"]
    args = (float(g["u_r_s"]), float(g["u_r_cut"]), float(g["u_eps"]))
    direct = oracle.short_range_direct(L, x, y, z, 1.0, t, *args)
    ours = short_range_forces(L, x, y, z, 1.0, t, *args, 0.5, "fp64")[:3]
    e_ours = rel_rms(ours, direct)
    e_ref = rel_rms((g["u_ax"], g["u_ay"], g["u_az"]), direct)
    print(f"theta=0.5 error vs direct: ours {e_ours:.6e}, reference tree {e_ref:.6e}")
    assert abs(e_ours - e_ref) <= 1e-6 * e_ref + 1e-12


def c5_state(n_side=256, L=256.0, mesh=256, seed=5, steps=64):
    """Clustered z = 0 state of a PM run (the c5 input), binary64 form."""
    a0 = 1.0 / 50.0
    stepper = hb.TimeStepper(a0, 1.0, math.log(1.0 / a0) / steps)
    K1, D, K2 = stepper.factors()
    m = ic.particle_mass(L, n_side)
    with hb.PMSolver(hb.MeshGeometry(L, mesh), hb.PMForceMethod.pure_pm(False)) as s:
        ic.lpt_on_device(s, ic.white_noise(n_side, seed), n_side, a0, m)
        s.run(K1, D, K2)
        st = s.download(acc=False)
    return st, m


def test_c5_treepm_forces_vs_direct_plus_long_range(oracle):
    n_side, L, mesh = 256, 256.0, 256
    st, m = c5_state(n_side, L, mesh)
    dx = L / mesh
    r_s = 1.25 * dx
    r_cut = 4.5 * r_s
    eps = (L / n_side) / 30.0
    targets = np.sort(np.random.default_rng(5).choice(n_side ** 3, 4096, replace=False)).astype(np.uint32)
    # long range: spectral PM on the full state
    with hb.PMSolver(hb.MeshGeometry(L, mesh), hb.PMForceMethod.treepm_long_range(r_s)) as s:
        s.upload(st["x"], st["y"], st["z"], uniform_mass=m)
        s.solve_forces()
        lr = s.download()
    short_ref = oracle.short_range_direct(L, st["x"], st["y"], st["z"], m, targets, r_s, r_cut, eps)
    total_ref = [short_ref[k] + lr[a][targets] for k, a in enumerate(("ax", "ay", "az"))]
    for prec in ("fp64", "fp32"):
        ax, ay, az, info = short_range_forces(L, st["x"], st["y"], st["z"], m, targets, r_s,
                                              r_cut, eps, 0.5, prec)
        tot = [ax + lr["ax"][targets], ay + lr["ay"][targets], az + lr["az"][targets]]
        e_short = rel_rms((ax, ay, az), short_ref)
        e_total = rel_rms(tot, total_ref)
        print(f"c5 {prec}: short-range rel RMS {e_short:.3e}, total force rel RMS "
              f"{e_total:.3e}; {info}")
        assert e_short <= 1e-2
        assert e_total <= 5e-3
