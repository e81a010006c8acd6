"""GPU edge cases of the PM step in both forms, through the C ABI.

* empty particle set: PMSolver's exact input-mass identity throws
  std::runtime_error for a zero particle count
  (src/gravity/pm_solver.cpp:664-679); both forms raise RuntimeError, for
  compute_forces and for upload;
* ragged particle counts (1, 3, 255, 257, 1001) on a power-of-two mesh (the
  five-pass transforms) and on N = 48 (cuFFT): binary64 forces within 1e-12
  of the force scale of the oracle's, precision form within 2e-4 of it. The
  force scale is max(max |a|, the acceleration of a pair one cell apart):
  a lone particle feels no self-force (the CIC deposit, the even Green's
  function and the centred-difference gather cancel it), so its forces are
  round-off and are checked against the pair scale;
* mesh sides outside [2, 2048] are rejected with ValueError;
* mesh 2048 (2^33 cells, cell indices above 2^32): translation by whole
  cells from the low corner into planes past 2^32 / N^2 gives the same forces
  (binary64 1e-11, precision form 1e-5 of max |a|), and the precision form
  agrees with binary64 there (2e-4 of max |a|). Positions are multiples of
  2^-20 in a box of 2048 so that the translation is exact in both forms.
"""
import numpy as np
import pytest

import hyowon_b200 as hb

pytestmark = pytest.mark.gpu


def solver(L, N, precision="fp64"):
    return hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), precision)


def forces(L, N, x, y, z, precision, m=1.0):
    ax, ay, az = np.zeros(x.size), np.zeros(x.size), np.zeros(x.size)
    with solver(L, N, precision) as s:
        s.compute_forces(x, y, z, None, m, ax, ay, az)
    return np.stack([ax, ay, az])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_empty_particle_set_raises_runtime_error(precision):
    e = np.zeros(0)
    with solver(100.0, 32, precision) as s:
        with pytest.raises(RuntimeError, match="input mass identity"):
            s.compute_forces(e, e, e, None, 1.0, np.zeros(0), np.zeros(0), np.zeros(0))
        with pytest.raises(RuntimeError, match="input mass identity"):
            s.upload(e, e, e, uniform_mass=1.0)
        # the handle stays usable: a pair 25 apart on each axis pulls with equal
        # and opposite forces (about 0.01; a pair one cell apart feels 5.8, and
        # the precision form's error is a fraction of that scale)
        x = np.array([10.0, 35.0])
        ax, ay, az = np.zeros(2), np.zeros(2), np.zeros(2)
        s.compute_forces(x, x, x, None, 1.0, ax, ay, az)
        assert np.all(np.isfinite(ax)) and ax[0] > 0.009
        assert abs(ax[0] + ax[1]) <= (1e-12 if precision == "fp64" else 2e-4 * 5.8)


@pytest.mark.parametrize("N", [32, 48])
@pytest.mark.parametrize("n", [1, 3, 255, 257, 1001])
def test_ragged_counts_match_oracle(oracle, n, N):
    L = 100.0
    rng = np.random.default_rng(1000 + n + N)
    x, y, z = (rng.uniform(0.0, L, n) for _ in range(3))
    dx = L / N
    px = np.array([0.5 * L, 0.5 * L + dx])
    ph = np.full(2, 0.5 * L)
    pair = max(np.max(np.abs(a)) for a in oracle.pm_forces(L, N, px, ph, ph))
    ref = np.stack(oracle.pm_forces(L, N, x, y, z))
    scale = max(np.max(np.abs(ref)), pair)
    f64 = forces(L, N, x, y, z, "fp64")
    e64 = np.max(np.abs(f64 - ref)) / scale
    assert e64 <= 1e-12, e64
    f32 = forces(L, N, x, y, z, "fp32")
    e32 = np.max(np.abs(f32 - ref)) / scale
    assert e32 <= 2e-4, e32
    print(f"n={n} N={N}: binary64 {e64:.2e}, precision form {e32:.2e} of the force scale")


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("N", [1, 4096])
def test_mesh_side_limits(precision, N):
    with pytest.raises(ValueError):
        solver(100.0, N, precision)


def test_mesh_2048_translation_past_32bit_cell_indices():
    L, N, n = 2048.0, 2048, 128
    rng = np.random.default_rng(2048)
    q = 2.0 ** -20
    # a clump within 16 cells of (40, 40, 40), positions on the 2^-20 grid
    base = [40.0 + np.round(rng.uniform(0.0, 16.0, n) / q) * q for _ in range(3)]
    # 1900 planes further along x: cell indices from 1940 * 2048^2 > 2^32
    shifted = [base[0] + 1900.0, base[1], base[2]]
    assert 1940 * N * N > 2 ** 32
    out = {}
    for precision in ("fp32", "fp64"):
        with solver(L, N, precision) as s:
            for tag, (x, y, z) in (("low", base), ("high", shifted)):
                ax, ay, az = np.zeros(n), np.zeros(n), np.zeros(n)
                s.compute_forces(x, y, z, None, 1.0, ax, ay, az)
                out[(precision, tag)] = np.stack([ax, ay, az])
    amax = np.max(np.abs(out[("fp64", "low")]))
    assert amax > 0.0
    d64 = np.max(np.abs(out[("fp64", "high")] - out[("fp64", "low")])) / amax
    d32 = np.max(np.abs(out[("fp32", "high")] - out[("fp32", "low")])) / amax
    x32 = max(np.max(np.abs(out[("fp32", t)] - out[("fp64", t)])) for t in ("low", "high")) / amax
    print(f"mesh 2048: translation binary64 {d64:.2e}, precision form {d32:.2e}; "
          f"forms differ by {x32:.2e} of max |a|")
    assert d64 <= 1e-11, d64
    assert d32 <= 1e-5, d32
    assert x32 <= 2e-4, x32
