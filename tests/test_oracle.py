"""CPU tests of the oracle itself: pinned against the reference's golden
vectors (tests/golden, produced by the reference's own compiled sources) and
against a direct DFT. No GPU needed."""
import math

import numpy as np
import pytest

from oracle.bindings import OracleError


def test_fft_against_direct_dft():
    import ctypes
    from oracle.bindings import Oracle
    o = Oracle()
    rng = np.random.default_rng(0)
    for n in (1, 2, 6, 8, 16):
        a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        buf = np.stack([a.real, a.imag], axis=1).ravel().copy()
        o.lib.orc_fft1d(ctypes.c_size_t(n), buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                        ctypes.c_int(-1))
        got = buf[0::2] + 1j * buf[1::2]
        np.testing.assert_allclose(got, np.fft.fft(a), rtol=0, atol=1e-13 * max(1, n))


@pytest.mark.parametrize("N", [4, 6, 8, 16])
def test_fft3d_roundtrip_and_numpy(N):
    import ctypes
    from oracle.bindings import Oracle
    o = Oracle()
    rng = np.random.default_rng(N)
    r = rng.standard_normal(N ** 3)
    H = N // 2 + 1
    out = np.zeros(2 * N * N * H)
    P = ctypes.POINTER(ctypes.c_double)
    o.lib.orc_fft3d_r2c(ctypes.c_size_t(N), r.ctypes.data_as(P), out.ctypes.data_as(P))
    ref = np.fft.rfftn(r.reshape(N, N, N)).ravel()
    got = out[0::2] + 1j * out[1::2]
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * N ** 1.5)
    back = np.zeros(N ** 3)
    o.lib.orc_fft3d_c2r(ctypes.c_size_t(N), out.ctypes.data_as(P), back.ctypes.data_as(P))
    np.testing.assert_allclose(back / N ** 3, r, rtol=0, atol=1e-13)


def test_gravitational_constant(oracle):
    # units.hpp:12-25 evaluated in order; CODATA G_SI with 1e10 Msun/h, Mpc/h, km/s.
    assert oracle.G() == pytest.approx(43007.1, rel=1e-3) or oracle.G() > 0
    assert math.isclose(oracle.G(), 6.67430e-11 * 1.98847e40 / (3.085677581491367e22 * 1e6),
                        rel_tol=1e-15)


def test_wrap_and_minimum_image_semantics(oracle):
    L = 10.0
    # in-range values (including -0.0) are returned unchanged (periodic_box.hpp:31)
    assert math.copysign(1, oracle.lib.orc_wrap(-0.0, L)) < 0
    assert oracle.lib.orc_wrap(L, L) == 0.0
    assert oracle.lib.orc_wrap(-1e-300, L) < L
    assert oracle.lib.orc_wrap(25.5, L) == 5.5
    assert oracle.lib.orc_minimum_image(5.0, L) == -5.0     # +L/2 ties map to -L/2
    assert oracle.lib.orc_minimum_image(-5.0, L) == -5.0
    assert oracle.lib.orc_minimum_image(7.0, L) == -3.0
    assert math.isnan(oracle.lib.orc_wrap(float("nan"), L))


def test_cell_assignment_matches_reference_bits(oracle, small_pm):
    g = small_pm
    base, frac = oracle.cic_coords(float(g["L"]), int(g["N"]), g["x"])
    assert np.array_equal(base, g["base_x"])
    assert np.array_equal(frac.view(np.int64), g["frac_x"].view(np.int64))


def test_deposit_matches_reference_bits(oracle, small_pm):
    g = small_pm
    L, N = float(g["L"]), int(g["N"])
    m = oracle.deposit(L, N, g["x"], g["y"], g["z"], uniform_mass=float(g["uniform_mass"]))
    assert np.array_equal(m.view(np.int64), g["deposit_uniform"].view(np.int64))
    m = oracle.deposit(L, N, g["x"], g["y"], g["z"], masses=g["masses"])
    assert np.array_equal(m.view(np.int64), g["deposit_masses"].view(np.int64))


def test_x_plane_bins_cover_every_particle_once(oracle, small_pm):
    # Counting-sort coverage identity (mass_assignment_deposit.inc:153-158).
    g = small_pm
    offsets, order = oracle.x_plane_bins(float(g["L"]), int(g["N"]), g["x"])
    assert offsets[0] == 0 and offsets[-1] == g["x"].size
    assert np.array_equal(np.sort(order), np.arange(g["x"].size))
    # stable: ascending particle index inside each plane
    for p in range(int(g["N"])):
        seg = order[offsets[p]:offsets[p + 1]]
        assert np.all(np.diff(seg.astype(np.int64)) > 0)


def test_potential_and_forces_match_reference(oracle, small_pm):
    g = small_pm
    L, N = float(g["L"]), int(g["N"])
    # N = 12 is not a power of two: the density normalisation takes the
    # scale-safe branch, restated here to within one rounding.
    dens, phi = oracle.potential(L, N, g["x"], g["y"], g["z"], uniform_mass=float(g["uniform_mass"]))
    scale = np.max(np.abs(g["density"]))
    assert np.max(np.abs(dens - g["density"])) <= 4e-16 * scale
    assert np.max(np.abs(phi - g["phi"])) <= 4e-15 * np.max(np.abs(g["phi"]))
    ax, ay, az = oracle.pm_forces(L, N, g["x"], g["y"], g["z"], uniform_mass=float(g["uniform_mass"]))
    for got, ref in ((ax, g["ax"]), (ay, g["ay"]), (az, g["az"])):
        assert np.max(np.abs(got - ref)) <= 4e-15 * np.max(np.abs(ref))


def test_c1_force_and_32_step_evolution_bit_exact(oracle, c1_kdk, schedules):
    c = c1_kdk
    L, N, m = float(c["box"]), int(c["mesh"]), float(c["particle_mass"])
    st = {k: c["ic_" + k].copy() for k in ("x", "y", "z", "px", "py", "pz")}
    for k in ("ax", "ay", "az"):
        st[k] = np.zeros_like(st["x"])
    oracle.pm_forces(L, N, st["x"], st["y"], st["z"], uniform_mass=m,
                     ax=st["ax"], ay=st["ay"], az=st["az"])
    assert np.array_equal(st["ax"], c["f0_x"])
    assert np.array_equal(st["az"], c["f0_z"])
    drift = []
    for row in schedules["c1"]:
        drift.append(oracle.kdk_step(L, N, st, row[4], row[3], row[5], uniform_mass=m))
        if len(drift) == 1:
            assert all(np.array_equal(st[k], c["s1_" + k]) for k in st)
    for k in st:
        assert np.array_equal(st[k], c["s32_" + k]), k
    np.testing.assert_allclose(drift, c["max_drift_32"], rtol=1e-15)


def test_nonfinite_position_rejected(oracle, small_pm):
    g = small_pm
    x = g["x"].copy()
    x[3] = np.nan
    with pytest.raises(OracleError) as e:
        oracle.deposit(float(g["L"]), int(g["N"]), x, g["y"], g["z"], uniform_mass=1.0)
    assert e.value.code == 1


def test_short_range_pair_law_matches_reference(oracle):
    from conftest import load_golden
    g = load_golden("treepm_pair.npz")
    got = np.stack(oracle.short_range_pair(float(g["r_s"]), float(g["eps"]), float(g["mass"]),
                                           g["dx"], g["dy"], g["dz"]))
    ref = np.stack([g["ax"], g["ay"], g["az"]])
    scale = np.abs(ref).max(axis=0)
    assert np.max(np.abs(got - ref) / scale) <= 1e-14


def test_short_range_direct_is_pairwise_sum(oracle):
    rng = np.random.default_rng(3)
    L, n = 20.0, 300
    x, y, z = (rng.uniform(0, L, n) for _ in range(3))
    targets = np.arange(0, n, 7, dtype=np.uint32)
    r_s, r_cut, eps = 1.0, 4.5, 0.05
    ax, ay, az = oracle.short_range_direct(L, x, y, z, 2.0, targets, r_s, r_cut, eps)
    for k, t in enumerate(targets[:10]):
        d = np.stack([x - x[t], y - y[t], z - z[t]], axis=1)
        d = (d + L / 2) % L - L / 2
        r = np.linalg.norm(d, axis=1)
        sel = (r < r_cut) & (r > 0)
        px, py, pz = oracle.short_range_pair(r_s, eps, 2.0, d[sel, 0], d[sel, 1], d[sel, 2])
        np.testing.assert_allclose([ax[k], ay[k], az[k]], [px.sum(), py.sum(), pz.sum()],
                                   rtol=1e-12, atol=1e-12 * np.abs(px).sum())
