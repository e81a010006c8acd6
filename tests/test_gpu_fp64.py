"""GPU parity tests of the binary64 (drop-in) form against the oracle and the
reference's golden vectors. All compute goes through the C ABI
(libhyowon_pm.so) on cuda:0.

Tolerances (binary64 form):
* cell assignment: bit-exact (same operation order, --fmad=false);
* deposit: each cell within 64 ulp-scale of the largest cell (atomic summation
  order is the only difference from the reference's plane-ordered sum);
* potential / forces: max |error| <= 1e-12 of the field maximum (cuFFT vs the
  oracle FFT differ at the 1e-15 level);
* one KDK step: positions within 1e-12 cell, momenta within 1e-10 relative;
* 32 KDK steps of c1: position RMS <= 1e-6 cell (chaotic growth of
  round-off differences), force relative RMS <= 1e-6.
"""
import numpy as np
import pytest

import hyowon_b200 as hb

pytestmark = pytest.mark.gpu


def solver(L, N, deconvolve=False, precision="fp64"):
    return hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(deconvolve), precision)


def rel_rms(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def test_cell_assignment_bit_exact(small_pm, oracle):
    g = small_pm
    L, N = float(g["L"]), int(g["N"])
    with solver(L, N) as s:
        s.upload(g["x"], g["y"], g["z"], uniform_mass=1.0)
        base, frac = s.cell_coords()
    assert np.array_equal(base[0], g["base_x"])
    assert np.array_equal(frac[0].view(np.int64), g["frac_x"].view(np.int64))
    by, fy = oracle.cic_coords(L, N, g["y"])
    bz, fz = oracle.cic_coords(L, N, g["z"])
    assert np.array_equal(base[1], by) and np.array_equal(base[2], bz)
    assert np.array_equal(frac[1], fy) and np.array_equal(frac[2], fz)


def test_cell_assignment_random_bit_exact(oracle):
    rng = np.random.default_rng(11)
    L, N, n = 1000.0, 1024, 200_000
    x = rng.uniform(-3 * L, 4 * L, n)
    x[:4] = [0.0, np.nextafter(L, 0), L, -1e-300]
    with solver(L, N) as s:
        s.upload(x, x[::-1].copy(), rng.uniform(0, L, n), uniform_mass=1.0)
        base, frac = s.cell_coords()
    b, f = oracle.cic_coords(L, N, x)
    assert np.array_equal(base[0], b)
    assert np.array_equal(frac[0], f)


@pytest.mark.parametrize("masses", [False, True])
def test_deposit_matches_reference(small_pm, masses):
    g = small_pm
    L, N = float(g["L"]), int(g["N"])
    with solver(L, N) as s:
        if masses:
            s.upload(g["x"], g["y"], g["z"], masses=g["masses"])
            ref = g["deposit_masses"]
        else:
            s.upload(g["x"], g["y"], g["z"], uniform_mass=float(g["uniform_mass"]))
            ref = g["deposit_uniform"]
        mesh = s.mass_mesh()
    assert np.max(np.abs(mesh - ref)) <= 64 * np.finfo(float).eps * np.max(ref)
    assert abs(mesh.sum() - ref.sum()) <= 1e-12 * ref.sum()


@pytest.mark.parametrize("deconvolve", [False, True])
def test_potential_and_forces_match_reference(small_pm, deconvolve):
    g = small_pm
    L, N, m = float(g["L"]), int(g["N"]), float(g["uniform_mass"])
    with solver(L, N, deconvolve) as s:
        s.upload(g["x"], g["y"], g["z"], uniform_mass=m)
        s.solve_forces()
        phi = s.potential()
        out = s.download()
    ref_phi = g["phi_deconvolved"] if deconvolve else g["phi"]
    assert np.max(np.abs(phi - ref_phi)) <= 1e-12 * np.max(np.abs(ref_phi))
    if not deconvolve:
        for k, r in (("ax", g["ax"]), ("ay", g["ay"]), ("az", g["az"])):
            assert np.max(np.abs(out[k] - r)) <= 1e-12 * np.max(np.abs(r)), k


def test_compute_forces_adds_like_pmsolver(small_pm):
    g = small_pm
    L, N = float(g["L"]), int(g["N"])
    n = g["x"].size
    ax = np.full(n, 1.5)
    ay = np.zeros(n)
    az = np.full(n, -2.0)
    with solver(L, N) as s:
        s.compute_forces(g["x"], g["y"], g["z"], g["masses"], None, ax, ay, az)
    for got, ref, base in ((ax, g["ax_m"], 1.5), (ay, g["ay_m"], 0.0), (az, g["az_m"], -2.0)):
        assert np.max(np.abs(got - base - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_c1_initial_force(c1_kdk):
    c = c1_kdk
    with solver(float(c["box"]), int(c["mesh"])) as s:
        s.upload(c["ic_x"], c["ic_y"], c["ic_z"], c["ic_px"], c["ic_py"], c["ic_pz"],
                 uniform_mass=float(c["particle_mass"]))
        s.solve_forces()
        out = s.download()
    for k, r in (("ax", c["f0_x"]), ("ay", c["f0_y"]), ("az", c["f0_z"])):
        assert rel_rms(out[k], r) <= 1e-13, k
    # pure PM conserves momentum: sum of forces ~ 0 relative to sum of |a|
    for k in ("ax", "ay", "az"):
        assert abs(out[k].sum()) <= 1e-10 * np.abs(out[k]).sum()


def test_c1_kdk_one_and_32_steps(c1_kdk, schedules):
    c = c1_kdk
    L, N = float(c["box"]), int(c["mesh"])
    dx = L / N
    sched = schedules["c1"]
    with solver(L, N) as s:
        s.upload(c["ic_x"], c["ic_y"], c["ic_z"], c["ic_px"], c["ic_py"], c["ic_pz"],
                 uniform_mass=float(c["particle_mass"]))
        md = s.kdk_step(sched[0, 4], sched[0, 3], sched[0, 5])
        one = s.download()
        assert md == pytest.approx(float(c["max_drift_1"][0]), rel=1e-12)
        for k in ("x", "y", "z"):
            d = (one[k] - c["s1_" + k] + L / 2) % L - L / 2
            assert np.max(np.abs(d)) <= 1e-12 * dx, k
        for k in ("px", "py", "pz", "ax", "ay", "az"):
            assert np.max(np.abs(one[k] - c["s1_" + k])) <= 1e-10 * np.max(np.abs(c["s1_" + k])), k
        K1, D, K2 = sched[1:, 4], sched[1:, 3], sched[1:, 5]
        s.run(K1, D, K2)
        fin = s.download()
    pos_rms = np.sqrt(np.mean([(((fin[k] - c["s32_" + k] + L / 2) % L - L / 2) ** 2).mean()
                               for k in "xyz"])) / dx
    assert pos_rms <= 1e-6, pos_rms
    f_err = rel_rms(np.concatenate([fin["ax"], fin["ay"], fin["az"]]),
                    np.concatenate([c["s32_ax"], c["s32_ay"], c["s32_az"]]))
    assert f_err <= 1e-6, f_err


def test_nonfinite_input_rejected():
    x = np.linspace(0, 9, 64)
    y = x.copy()
    z = x.copy()
    x[5] = np.inf
    with solver(10.0, 8) as s:
        with pytest.raises(ValueError):
            s.upload(x, y, z, uniform_mass=1.0)
        with pytest.raises(ValueError):
            s.upload(y, y, z, uniform_mass=0.0)
        with pytest.raises(ValueError):
            s.upload(y, y, z, masses=np.full(64, -1.0))


def test_kick_drift_failure_publishes_nothing(c1_kdk, schedules):
    c = c1_kdk
    with solver(float(c["box"]), int(c["mesh"])) as s:
        s.upload(c["ic_x"], c["ic_y"], c["ic_z"], c["ic_px"], c["ic_py"], c["ic_pz"],
                 uniform_mass=float(c["particle_mass"]))
        s.solve_forces()
        before = s.download()
        with pytest.raises(OverflowError):
            s.kdk_step(1e308, 1e308, 0.0)     # non-finite candidate
        after = s.download()
    for k in before:
        assert np.array_equal(before[k], after[k]), k


def test_device_lpt_matches_oracle():
    from hyowon_b200 import ic
    from oracle.lpt_oracle import lpt_ics
    n_side, L, a0 = 32, 100.0, 1 / 50
    noise = ic.white_noise(n_side, 1)
    ref = lpt_ics(noise, n_side, L, a0)
    with solver(L, 64) as s:
        ic.lpt_on_device(s, noise, n_side, a0, ic.particle_mass(L, n_side))
        got = s.download(acc=False)
    for k in "xyz":
        d = (got[k] - ref[k] + L / 2) % L - L / 2
        assert np.max(np.abs(d)) <= 1e-11, k
    for k in ("px", "py", "pz"):
        assert np.max(np.abs(got[k] - ref[k])) <= 1e-10 * np.max(np.abs(ref[k])), k


def test_run_equals_repeated_steps(c1_kdk, schedules):
    c = c1_kdk
    L, N = float(c["box"]), int(c["mesh"])
    sched = schedules["c1"][:4]
    outs = []
    for mode in ("run", "step"):
        with solver(L, N) as s:
            s.upload(c["ic_x"], c["ic_y"], c["ic_z"], c["ic_px"], c["ic_py"], c["ic_pz"],
                     uniform_mass=float(c["particle_mass"]))
            if mode == "run":
                s.run(sched[:, 4], sched[:, 3], sched[:, 5])
            else:
                for r in sched:
                    s.kdk_step(r[4], r[3], r[5])
            outs.append(s.download())
    for k in outs[0]:
        scale = np.max(np.abs(outs[1][k]))
        assert np.max(np.abs(outs[0][k] - outs[1][k])) <= 1e-12 * scale, k
