"""Error paths of the device checks, made to fail from the host
(include/hyowon_debug.h): no GPU fault, trap or hang is involved.

* A pipeline wait of the five-pass potential solve that is given zero polls
  gives up at once: each block drains its own copies in flight, sets
  ST_PIPELINE and returns; the solve fails with the runtime error the status
  maps to, nothing is published, and with the default limit restored the same
  handle solves again with the same forces as a fresh handle.
* A CIC mass-conservation target moved off the deposited mass makes the
  solve fail with the reference's runtime error (src/math/cic_mass_conservation.cpp:41-59);
  with the target restored the handle solves again.
Both forms, on a power-of-two mesh (the five-pass solve) of 64^3 cells.
"""
import numpy as np
import pytest

import hyowon_b200 as hb
from hyowon_b200 import _native as nat

pytestmark = pytest.mark.gpu

DEFAULT_WAIT = 16777216


def state(n=20000, L=50.0, seed=4):
    rng = np.random.default_rng(seed)
    return L, [rng.uniform(0.0, L, n) for _ in range(3)]


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_pipeline_wait_timeout_is_reported_and_recovered(form):
    L, pos = state()
    with hb.PMSolver(hb.MeshGeometry(L, 64), hb.PMForceMethod.pure_pm(False), form) as fresh:
        fresh.upload(*pos, uniform_mass=1.0)
        fresh.solve_forces()
        want = fresh.download()
    with hb.PMSolver(hb.MeshGeometry(L, 64), hb.PMForceMethod.pure_pm(False), form) as s:
        s.upload(*pos, uniform_mass=1.0)
        assert nat.lib().hyowon_pm_debug_set_wait_limit(s.handle, 0) == 0
        with pytest.raises(RuntimeError, match="pipeline wait timed out"):
            s.solve_forces()
        assert nat.lib().hyowon_pm_debug_set_wait_limit(s.handle, DEFAULT_WAIT) == 0
        s.solve_forces()
        got = s.download()
    for k in ("ax", "ay", "az"):
        assert np.array_equal(got[k], want[k]), k


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_mass_conservation_violation_is_reported_and_recovered(form):
    L, pos = state(seed=5)
    with hb.PMSolver(hb.MeshGeometry(L, 64), hb.PMForceMethod.pure_pm(False), form) as s:
        s.upload(*pos, uniform_mass=1.0)
        s.solve_forces()
        want = s.download()
        # binary64: 1e-6 of the total mass, far outside the forward-error bound;
        # precision form: one fixed-point unit off the exact integer sum
        assert nat.lib().hyowon_pm_debug_offset_mass_target(s.handle, 0.02 if form == "fp64" else 1.0) == 0
        with pytest.raises(RuntimeError, match="mass"):
            s.solve_forces()
        assert nat.lib().hyowon_pm_debug_offset_mass_target(s.handle, 0.0) == 0
        s.solve_forces()
        got = s.download()
    for k in ("ax", "ay", "az"):
        assert np.array_equal(got[k], want[k]), k
