"""Parity at the metric's configurations against the reference itself.

The reference runs here are oracle/_ref: the reference's own PMSolver,
LeapfrogIntegrator, TimeStepper, LinearPowerSpectrum, LPTDisplacement and
MatterPowerSpectrum, compiled unmodified (the FP64 oracle of every claim
below). Its initial conditions come from oracle/workload.py and the
reference's own 1LPT (ref_lpt_white_noise), so nothing of this repository's
product runs on the reference's side.

c2 (128^3 particles, L = 256 Mpc/h, 256^3 mesh, 1LPT at z = 49, seed 1,
64 KDK steps uniform in ln a to z = 0), the reference's evolution against:

* the binary64 form from the same initial state: final positions within
  1e-6 cell RMS, accelerations at the reference's own z = 0 positions within
  1e-10 relative RMS (the reference's last force solve);
* the precision form: forces at the reference's z = 0 positions within 1e-4
  relative RMS, and its own 64-step evolution's P(k) (the reference's
  MatterPowerSpectrum on both z = 0 states, 256^3 estimator mesh, raw power)
  within 0.1% of the reference's in every bin below k_Nyquist / 2; its
  final-position RMS against the reference is printed (chaotic growth of the
  FP32 round-off), with a loose 0.05-cell bound.

c3 (512^3 particles, L = 1000 Mpc/h, 1024^3 mesh, 1LPT at z = 49, seed 7):
the reference's PMSolver::compute_forces on the initial state against the
binary64 form (1e-10 relative RMS) and the precision form (1e-4).
"""
import math

import numpy as np
import pytest

import hyowon_b200 as hb

pytestmark = pytest.mark.gpu

COMPS = ("x", "y", "z", "px", "py", "pz")


def rel_rms(a, b):
    num = sum(float(np.sum((a[k] - b[k]) ** 2)) for k in ("ax", "ay", "az"))
    den = sum(float(np.sum(b[k] ** 2)) for k in ("ax", "ay", "az"))
    return math.sqrt(num / den)


def pos_rms_cells(a, b, L, N):
    return math.sqrt(np.mean([float(np.mean(((a[k] - b[k] + L / 2) % L - L / 2) ** 2))
                              for k in "xyz"])) / (L / N)


@pytest.fixture(scope="module")
def reference():
    from oracle.bindings import Reference
    return Reference()


@pytest.fixture(scope="module")
def c2_reference_run(reference):
    from oracle import workload
    c = workload.CONFIGS["c2"]
    st = workload.reference_ics(reference, "c2")
    ics = {k: np.array(st[k]) for k in COMPS}
    run = {k: v.copy() for k, v in ics.items()}
    for k in ("ax", "ay", "az"):
        run[k] = np.zeros_like(run["x"])
    a0, dl = workload.schedule("c2")
    m = workload.particle_mass(c["box"], c["n_side"])
    _, secs = reference.kdk_run(c["box"], c["mesh"], run, a0, 1.0, dl, c["steps"], m)
    print(f"reference c2: {c['steps']} steps in {secs:.1f} s")
    return c, ics, run, m


def evolve(c, ics, m, form):
    a0 = 1.0 / (1.0 + c["z_start"])
    K1, D, K2 = hb.TimeStepper(a0, 1.0, math.log(1.0 / a0) / c["steps"]).factors()
    assert K1.size == c["steps"]
    with hb.PMSolver(hb.MeshGeometry(c["box"], c["mesh"]), hb.PMForceMethod.pure_pm(False),
                     form) as s:
        s.upload(*(ics[k] for k in COMPS), uniform_mass=m)
        s.run(K1, D, K2)
        return s.download()


def forces_at(c, state, m, form):
    with hb.PMSolver(hb.MeshGeometry(c["box"], c["mesh"]), hb.PMForceMethod.pure_pm(False),
                     form) as s:
        s.upload(state["x"], state["y"], state["z"], uniform_mass=m)
        s.solve_forces()
        return s.download()


def test_c2_binary64_form_matches_reference_evolution(c2_reference_run):
    c, ics, ref, m = c2_reference_run
    got = evolve(c, ics, m, "fp64")
    prms = pos_rms_cells(got, ref, c["box"], c["mesh"])
    pmax = max(float(np.max(np.abs(ref[k]))) for k in ("px", "py", "pz"))
    mom = max(float(np.max(np.abs(got[k] - ref[k]))) for k in ("px", "py", "pz")) / pmax
    same = forces_at(c, ref, m, "fp64")
    ferr = rel_rms(same, ref)
    print(f"c2 binary64 vs reference after 64 steps: position RMS {prms:.3e} cells, "
          f"max |dp| {mom:.3e} of max |p|; forces at the reference's z=0 state: "
          f"relative RMS {ferr:.3e}")
    assert prms <= 1e-6
    assert ferr <= 1e-10


def test_c2_precision_form_against_reference(c2_reference_run, reference):
    c, ics, ref, m = c2_reference_run
    L, N = c["box"], c["mesh"]
    same = forces_at(c, ref, m, "fp32")
    ferr = rel_rms(same, ref)
    got = evolve(c, ics, m, "fp32")
    prms = pos_rms_cells(got, ref, L, N)
    kw = dict(uniform_mass=m, num_bins=24, max_k_fraction_nyquist=0.5)
    pk_ref = reference.power_spectrum(L, N, ref["x"], ref["y"], ref["z"], **kw)
    pk_got = reference.power_spectrum(L, N, got["x"], got["y"], got["z"], **kw)
    sel = pk_ref["mode_count"] > 0
    ratio = pk_got["p_raw"][sel] / pk_ref["p_raw"][sel]
    dev = float(np.max(np.abs(ratio - 1.0)))
    print(f"c2 precision form vs reference: force relative RMS {ferr:.3e} at the reference's "
          f"z=0 state; after 64 steps position RMS {prms:.3e} cells, max |P/P_ref - 1| "
          f"below k_Nyq/2 {dev:.3e} ({int(sel.sum())} bins)")
    assert np.array_equal(pk_got["mode_count"], pk_ref["mode_count"])
    assert ferr <= 1e-4
    assert dev <= 1e-3
    assert prms <= 0.05


def test_c3_initial_forces_match_reference(reference):
    from hyowon_b200 import ic
    c = ic.CONFIGS["c3"]
    n_side, N, L = c["n_side"], c["mesh"], c["box"]
    a0, _ = ic.config_schedule("c3")
    m = ic.particle_mass(L, n_side)
    geom = hb.MeshGeometry(L, N)
    with hb.PMSolver(geom, hb.PMForceMethod.pure_pm(False), "fp64") as s:
        ic.lpt_on_device(s, ic.white_noise(n_side, c["seed"]), n_side, a0, m)
        s.solve_forces()
        f64 = s.download()
    f32 = forces_at(c, f64, m, "fp32")
    ref = dict(zip(("ax", "ay", "az"),
                   reference.pm_forces(L, N, f64["x"], f64["y"], f64["z"], uniform_mass=m)))
    e64, e32 = rel_rms(f64, ref), rel_rms(f32, ref)
    print(f"c3 initial forces vs reference PMSolver: binary64 relative RMS {e64:.3e}, "
          f"precision form {e32:.3e}")
    assert e64 <= 1e-10
    assert e32 <= 1e-4
