"""GPU tests of hyowon_pm_snapshot_payload: the /PartType1 Coordinates and
Velocities rows the reference's snapshot writer stages
(src/io/snapshot_io_particle_helpers.inc:116-200), checked against the
device state read back by hyowon_pm_download and the reference's arithmetic
restated in numpy (rows in particle order, velocities = p * (1 / a)):
bit-identical in both forms; the payload validation of
require_finite_particle_payload (:48-104) raises before anything is written.
"""
import numpy as np
import pytest

import hyowon_b200 as hb

pytestmark = pytest.mark.gpu


def state(n, L, seed):
    rng = np.random.default_rng(seed)
    x, y, z = (rng.uniform(0, L, n) for _ in range(3))
    px, py, pz = (rng.normal(0, 50.0, n) for _ in range(3))
    return x, y, z, px, py, pz


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_rows_match_download(form):
    L, N, n = 64.0, 32, 20000
    x, y, z, px, py, pz = state(n, L, 3)
    a = 0.37
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), form) as s:
        s.upload(x, y, z, px, py, pz, uniform_mass=1.0)
        s.run(np.full(3, 1e-3), np.full(3, 2e-3), np.full(3, 1e-3))
        d = s.download(acc=False)
        c, v = s.snapshot_payload(a)
        c2, none = s.snapshot_payload(a, velocities=False)
    inv_a = 1.0 / a
    assert none is None
    assert np.array_equal(c, np.stack([d["x"], d["y"], d["z"]], axis=1))
    assert np.array_equal(c2, c)
    assert np.array_equal(v, np.stack([d["px"], d["py"], d["pz"]], axis=1) * inv_a)
    assert np.all((c >= 0.0) & (c < L))


def test_validation():
    L, N, n = 64.0, 16, 1000
    x, y, z, px, py, pz = state(n, L, 4)
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False)) as s:
        with pytest.raises(hb.HyowonLogicError):
            s.snapshot_payload(1.0)
        s.upload(x, y, z, px, py, pz, uniform_mass=1.0)
        with pytest.raises(ValueError):
            s.snapshot_payload(0.0)
        with pytest.raises(ValueError):
            s.snapshot_payload(float("nan"))
        with pytest.raises(OverflowError):
            s.snapshot_payload(1e-310)      # 1 / a overflows
        big = px.copy()
        big[7] = 1e308
        s.upload(x, y, z, big, py, pz, uniform_mass=1.0)
        with pytest.raises(OverflowError):
            s.snapshot_payload(0.5)         # 1e308 * 2 overflows
        c, v = s.snapshot_payload(1.0)      # 1e308 * 1 is finite
        assert c.shape == (n, 3) and v[7, 0] == 1e308
