"""Run-to-run determinism of the binary64 drop-in form.

The reference's deposit is plane-owned and sums in a fixed order whatever the
thread count (src/mesh/mass_assignment_deposit.inc:302-333), so its evolution
reproduces itself bit for bit. The binary64 form's deposit sums exact
fixed-point integers per cell and rounds each cell once, so its mesh, and
therefore the whole evolution, does not depend on the order in which atomics
land: two runs of the same steps give identical bits.

* c2 (128^3 particles, 256^3 mesh, 1LPT at z = 49, seed 1), all 64 KDK steps
  to z = 0, run twice in separate handles: positions, momenta and
  accelerations bit-identical;
* explicit per-particle masses (a clustered 32^3 set on a 48^3 cuFFT mesh and
  a 64^3 five-pass mesh), 8 steps twice: bit-identical; the deposited mass
  mesh of the first state against the oracle's binary64 deposit within
  64 ulp of the largest cell.
"""
import math

import numpy as np
import pytest

import hyowon_b200 as hb
from hyowon_b200 import ic

pytestmark = pytest.mark.gpu

COMPS = ("x", "y", "z", "px", "py", "pz", "ax", "ay", "az")


def test_c2_binary64_evolution_is_bit_reproducible():
    c = ic.CONFIGS["c2"]
    n_side, N, L = c["n_side"], c["mesh"], c["box"]
    a0, dl = ic.config_schedule("c2")
    K1, D, K2 = hb.TimeStepper(a0, 1.0, dl).factors()
    m = ic.particle_mass(L, n_side)
    noise = ic.white_noise(n_side, c["seed"])
    runs = []
    for _ in range(2):
        with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), "fp64") as s:
            ic.lpt_on_device(s, noise, n_side, a0, m)
            s.run(K1, D, K2)
            runs.append(s.download())
    for k in COMPS:
        assert np.array_equal(runs[0][k], runs[1][k]), k


@pytest.mark.parametrize("N", [48, 64])
def test_binary64_with_masses_is_bit_reproducible(N, oracle):
    rng = np.random.default_rng(N)
    L, n = 60.0, 32 ** 3
    centres = rng.uniform(0.0, L, (12, 3))
    pick = rng.integers(0, 12, n)
    pos = (centres[pick] + rng.normal(0.0, 1.5, (n, 3))) % L
    x, y, z = (np.ascontiguousarray(pos[:, d]) for d in range(3))
    masses = rng.uniform(0.2, 3.0, n)
    p = [rng.normal(0.0, 50.0, n) for _ in range(3)]
    K1 = np.full(8, 2e-4)
    D = np.full(8, 4e-3)
    K2 = np.full(8, 2e-4)
    runs = []
    mesh0 = None
    for r in range(2):
        with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), "fp64") as s:
            s.upload(x, y, z, *p, masses=masses)
            if r == 0:
                s.solve_forces()
                mesh0 = s.mass_mesh().reshape(-1)
            s.run(K1, D, K2)
            runs.append(s.download())
    for k in COMPS:
        assert np.array_equal(runs[0][k], runs[1][k]), k
    ref = oracle.deposit(L, N, x, y, z, masses=masses)
    tol = 64 * np.finfo(np.float64).eps * np.max(np.abs(ref))
    err = np.max(np.abs(mesh0 - ref))
    print(f"N={N}: deposit vs oracle max |diff| {err:.3e} (64 ulp of the largest cell {tol:.3e})")
    assert err <= tol
    assert math.isclose(mesh0.sum(), masses.sum(), rel_tol=1e-12)


def test_binary64_exact_two_word_deposit_on_a_dense_cluster(oracle):
    """All 32^3 particles within a quarter cell of one point of a 64^3
    five-pass mesh: the densest bucket holds thousands of particles, so the
    deposit takes its exact two-word (hi/lo) form, then transforms each tile
    along z. The potential matches the oracle's to 1e-12 of its largest value
    and two runs give identical accelerations."""
    rng = np.random.default_rng(11)
    L, N, n = 64.0, 64, 32 ** 3
    centre = np.array([17.3, 40.6, 5.2])
    pos = (centre + rng.uniform(-0.25, 0.25, (n, 3))) % L
    x, y, z = (np.ascontiguousarray(pos[:, d]) for d in range(3))
    masses = rng.uniform(0.5, 2.0, n)
    accs, phis = [], []
    for _ in range(2):
        with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), "fp64") as s:
            s.upload(x, y, z, masses=masses)
            s.solve_forces()
            phis.append(s.potential().reshape(-1))
            accs.append(s.download())
    for k in ("ax", "ay", "az"):
        assert np.array_equal(accs[0][k], accs[1][k]), k
    _, ref = oracle.potential(L, N, x, y, z, masses=masses)
    err = np.max(np.abs(phis[0] - ref)) / np.max(np.abs(ref))
    print(f"dense cluster: potential max error / max |phi| = {err:.3e}")
    assert err <= 1e-12


@pytest.mark.parametrize("N", [48, 64])
def test_run_equals_single_steps(N):
    """hyowon_pm_run and the same steps as hyowon_pm_kdk_step calls give
    identical bits: positions, momenta, accelerations and the per-step drift
    maxima over 12 steps (three re-sorts), on a five-pass (64) and a cuFFT (48)
    mesh. (It guards any work run() shares across steps, e.g. a gather that
    also makes the next step's candidate, against the single-step path.)"""
    rng = np.random.default_rng(7 + N)
    L, n = 40.0, 24 ** 3
    centres = rng.uniform(0.0, L, (6, 3))
    pick = rng.integers(0, 6, n)
    pos = (centres[pick] + rng.normal(0.0, 2.0, (n, 3))) % L
    x, y, z = (np.ascontiguousarray(pos[:, d]) for d in range(3))
    p = [rng.normal(0.0, 30.0, n) for _ in range(3)]
    steps = 12
    K1 = np.linspace(1.5e-4, 2.5e-4, steps)
    D = np.linspace(3e-3, 5e-3, steps)
    K2 = np.linspace(1.6e-4, 2.6e-4, steps)
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), "fp64") as s:
        s.upload(x, y, z, *p, uniform_mass=1.3)
        drift_run = s.run(K1, D, K2)
        fused = s.download()
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), "fp64") as s:
        s.upload(x, y, z, *p, uniform_mass=1.3)
        drift_steps = [s.kdk_step(K1[k], D[k], K2[k]) for k in range(steps)]
        single = s.download()
    for k in COMPS:
        assert np.array_equal(fused[k], single[k]), k
    assert np.array_equal(np.asarray(drift_run, dtype=np.float64),
                          np.asarray(drift_steps, dtype=np.float64))
