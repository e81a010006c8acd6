"""TreePM as a force method of the PM handle, against the reference's
TreePMSolver (src/gravity/treepm_solver.cpp:631-717) driving its
LeapfrogIntegrator (oracle/_ref, ref_treepm_kdk_run).

Case: 16^3 particles from the reference's own 1LPT of the configs' white noise
(L = 50 Mpc/h, z = 49, seed 1), 32^3 PM mesh, r_s = 1.25 mesh cells,
r_cut = 4.5 r_s, Plummer softening 1/30 of the mean interparticle spacing,
opening angle 0.5, 4 KDK steps of the c1 schedule (steps uniform in ln a from
z = 49).

* binary64 form with explicit per-particle masses (uniform in [0.5, 1.5] of
  the lattice mass): accelerations of the last solve within 1e-9 relative RMS
  and positions within 1e-8 cell RMS of the reference (the node moments and
  the pair sums differ from the reference's only in summation order);
* precision form with the uniform lattice mass: accelerations within 1e-4
  relative RMS, positions within 1e-3 cell RMS;
* the handle's short-range call (hyowon_pm_treepm_short_forces) on the initial
  state equals the standalone host-array call (hyowon_treepm_short_forces)
  within 1e-12 relative RMS (same octree, other source order).
"""
import math

import numpy as np
import pytest

import hyowon_b200 as hb
from hyowon_b200 import treepm

pytestmark = pytest.mark.gpu

L, NS, NM, STEPS = 50.0, 16, 32, 4
RS_CELLS, CUT_MULT, THETA = 1.25, 4.5, 0.5
EPS = L / NS / 30.0
COMPS = ("x", "y", "z", "px", "py", "pz")


def rel_rms(a, b):
    num = sum(float(np.sum((a[k] - b[k]) ** 2)) for k in ("ax", "ay", "az"))
    den = sum(float(np.sum(b[k] ** 2)) for k in ("ax", "ay", "az"))
    return math.sqrt(num / den)


def pos_rms_cells(a, b):
    return math.sqrt(np.mean([float(np.mean(((a[k] - b[k] + L / 2) % L - L / 2) ** 2))
                              for k in "xyz"])) / (L / NM)


@pytest.fixture(scope="module")
def setup():
    from oracle import workload
    from oracle.bindings import Reference
    ref = Reference()
    st = workload.reference_ics(ref, "c1", n_side=NS, box=L)
    ics = {k: np.array(st[k]) for k in COMPS}
    m_lat = workload.particle_mass(L, NS)
    masses = np.random.default_rng(9).uniform(0.5, 1.5, NS ** 3) * m_lat
    a0, dl = workload.schedule("c1")
    return ref, ics, masses, m_lat, a0, dl


def reference_run(setup, masses):
    ref, ics, _, m_lat, a0, dl = setup
    st = {k: v.copy() for k, v in ics.items()}
    ref.treepm_kdk_run(L, NS, NM, RS_CELLS, CUT_MULT, EPS, THETA, st, a0, 1.0, dl, STEPS,
                       masses=masses, uniform_mass=m_lat)
    return st


def our_run(setup, form, masses):
    _, ics, _, m_lat, a0, dl = setup
    r_s = RS_CELLS * L / NM
    K1, D, K2 = hb.TimeStepper(a0, 1.0, dl).factors()
    with hb.PMSolver(hb.MeshGeometry(L, NM), hb.PMForceMethod.treepm_long_range(r_s), form) as s:
        s.set_treepm_short_range(THETA, EPS, CUT_MULT * r_s)
        if masses is None:
            s.upload(*(ics[k] for k in COMPS), uniform_mass=m_lat)
        else:
            s.upload(*(ics[k] for k in COMPS), masses=masses)
        s.run(K1[:STEPS], D[:STEPS], K2[:STEPS])
        return s.download()


def test_binary64_treepm_steps_with_masses_match_reference(setup):
    masses = setup[2]
    ref = reference_run(setup, masses)
    got = our_run(setup, "fp64", masses)
    ferr, perr = rel_rms(got, ref), pos_rms_cells(got, ref)
    print(f"TreePM binary64, masses, {STEPS} steps: acceleration relative RMS {ferr:.3e}, "
          f"position RMS {perr:.3e} cells")
    assert ferr <= 1e-9
    assert perr <= 1e-8


def test_precision_form_treepm_steps_match_reference(setup):
    ref = reference_run(setup, None)
    got = our_run(setup, "fp32", None)
    ferr, perr = rel_rms(got, ref), pos_rms_cells(got, ref)
    print(f"TreePM precision form, {STEPS} steps: acceleration relative RMS {ferr:.3e}, "
          f"position RMS {perr:.3e} cells")
    assert ferr <= 1e-4
    assert perr <= 1e-3


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_handle_short_range_equals_standalone_call(setup, form):
    _, ics, _, m_lat, _, _ = setup
    r_s = RS_CELLS * L / NM
    with hb.PMSolver(hb.MeshGeometry(L, NM), hb.PMForceMethod.treepm_long_range(r_s), form) as s:
        s.upload(*(ics[k] for k in COMPS), uniform_mass=m_lat)
        ax, ay, az, info = s.treepm_short_forces(THETA, EPS, CUT_MULT * r_s)
        state = s.download(acc=False)
    targets = np.arange(NS ** 3, dtype=np.uint32)
    bx, by, bz, _ = treepm.short_range_forces(L, state["x"], state["y"], state["z"], m_lat,
                                              targets, r_s, CUT_MULT * r_s, EPS, THETA,
                                              precision=form)
    got = dict(ax=ax, ay=ay, az=az)
    want = dict(ax=bx, ay=by, az=bz)
    err = rel_rms(got, want)
    print(f"{form}: handle vs standalone short range {err:.3e}; {info}")
    assert err <= (1e-12 if form == "fp64" else 1e-6)
