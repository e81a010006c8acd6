"""GPU tests of the device IC generator (include/hyowon_ic.h) against the
reference's generated ICs (tests/golden/ic.npz) and the restatement
(oracle/ic_oracle.py).

Tolerances (the device differs from the reference only in the Box-Muller
log / sincos of CUDA's libdevice, a few ulp, and in cuFFT's rounding):
* field: identical zero pattern; every non-zero component within 4e-15 of
  its own magnitude (about 36 ulp);
* particles: positions within 1e-12 L (minimum image), momenta within 1e-12
  of the largest |p|;
* pairing / linearity (full size): pair_b momenta of 1LPT are exactly the
  negated pair_a ones; (p_a - p_b) / 2 of 2LPT equals the 1LPT momenta to
  1e-13 of max |p|, and (p_a + p_b) / 2 is the second-order part;
* the handle path writes the same state as the standalone call (bit for bit
  in binary64).
"""
import math

import numpy as np
import pytest

import hyowon_b200 as hb
from hyowon_b200 import ic
from oracle import ic_oracle as io

pytestmark = pytest.mark.gpu

SPEC = {
    "n16_1lpt": (16, 1, 0, "gaussian", "independent", None, 11),
    "n16_2lpt": (16, 2, 0, "gaussian", "independent", None, 11),
    "n16_2lpt_fixed_pair_b": (16, 2, 0, "fixed", "pair_b", None, 12345678901),
    "n12_2lpt_pair_a_k4": (12, 2, 0, "gaussian", "pair_a", 4, 5),
    "n16_1lpt_m32_k5": (16, 1, 32, "gaussian", "independent", 5, 3),
}


def case(g, name):
    return {k.split("__", 1)[1]: g[k] for k in g.files if k.startswith(name + "__")}


def params_of(g, name):
    c = case(g, name)
    N, order, mesh, amp, pair, K, seed = SPEC[name]
    a0 = float(c["a_start"])
    p1 = a0 * a0 * float(c["H"]) * float(c["f1"])
    x2 = float(c["D2"]) / (float(c["D1"]) * float(c["D1"]))
    p2 = a0 * a0 * float(c["H"]) * float(c["f2"]) * x2
    p = ic.ICParams(N, float(g["box"]), seed, a0, lpt_order=order, mesh_per_dimension=mesh,
                    max_mode_per_axis=K, amplitude_mode=amp, phase_pairing=pair,
                    factors=(p1, x2, p2))
    return p, c


def check_field(dev, ref):
    assert np.array_equal(dev == 0, ref == 0)
    for part in (np.real, np.imag):
        d, r = part(dev), part(ref)
        nz = r != 0
        assert np.array_equal(d == 0, r == 0)
        rel = np.abs(d[nz] - r[nz]) / np.abs(r[nz])
        assert rel.max() <= 4e-15, rel.max()
    return float(np.max(np.abs(dev - ref) / np.maximum(np.abs(ref), 1e-300)))


def check_particles(st, ref, L):
    for k in "xyz":
        d = (st[k] - ref[k] + 0.5 * L) % L - 0.5 * L
        assert np.max(np.abs(d)) <= 1e-12 * L, (k, np.max(np.abs(d)))
        assert np.all((st[k] >= 0.0) & (st[k] < L))
    pmax = max(np.max(np.abs(ref[k])) for k in ("px", "py", "pz"))
    for k in ("px", "py", "pz"):
        assert np.max(np.abs(st[k] - ref[k])) <= 1e-12 * pmax, k


@pytest.mark.parametrize("name", list(SPEC))
def test_field_matches_reference(ic_golden, name):
    p, c = params_of(ic_golden, name)
    f = ic.RandomField.generate(p, c["power"])
    r = check_field(f, c["modes"])
    print(f"{name}: field max relative difference {r:.2e}")


@pytest.mark.parametrize("name", list(SPEC))
def test_particles_match_reference(ic_golden, name):
    p, c = params_of(ic_golden, name)
    st = ic.generate_ics(p, c["power"])
    check_particles(st, c, float(ic_golden["box"]))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_handle_path(ic_golden, precision):
    p, c = params_of(ic_golden, "n16_2lpt")
    L = float(ic_golden["box"])
    st = ic.generate_ics(p, c["power"])
    m = ic.particle_mass(L, 16)
    with hb.PMSolver(hb.MeshGeometry(L, 32), hb.PMForceMethod.pure_pm(False), precision) as s:
        s.generate_ics(p, c["power"], m)
        d = s.download(acc=False)
        s.solve_forces()
        assert s.info()[0] == 16 ** 3
    if precision == "fp64":
        for k in ("x", "y", "z", "px", "py", "pz"):
            assert np.array_equal(d[k], st[k]), k
    else:
        # u32 fixed-point positions: L / 2^32 quantisation
        for k in "xyz":
            dd = (d[k] - st[k] + 0.5 * L) % L - 0.5 * L
            assert np.max(np.abs(dd)) <= L * 2.0 ** -31, k
        for k in ("px", "py", "pz"):
            assert np.max(np.abs(d[k] - st[k])) <= 1e-6 * np.max(np.abs(st[k])), k


def test_against_oracle_n32_2lpt():
    """Device vs the restatement on a fresh case (N = 32, 2LPT, M = 64)."""
    a0 = 1.0 / 50.0
    p = ic.ICParams(32, 200.0, 424242, a0, lpt_order=2)
    M, K = p.resolve()
    assert (M, K) == (64, 15)
    power = ic.power_table(p, ic.start_spectrum(a0))
    amp = io.mode_amplitudes(M, 200.0, power)
    ref = io.gaussian_field(M, 424242, K, amp)
    check_field(ic.RandomField.generate(p, power), ref)
    p1, x2, p2 = p.factors
    o = io.lpt(ref, 32, 200.0, K, p1, 2, x2, p2)
    check_particles(ic.generate_ics(p, power), o, 200.0)


def test_errors():
    p = ic.ICParams(16, 100.0, 1, 0.02, factors=(1.0, -0.4, -1.0))
    _, K = p.resolve()
    power = np.ones(3 * K * K + 1)
    with pytest.raises(ValueError):
        ic.generate_ics(p, power[:-1])  # table too short
    bad = power.copy()
    bad[5] = 0.0
    with pytest.raises(RuntimeError):
        ic.generate_ics(p, bad)
    with pytest.raises(ValueError):
        with hb.PMSolver(hb.MeshGeometry(100.0, 16), hb.PMForceMethod.pure_pm(False)) as s:
            s.generate_ics(ic.ICParams(16, 100.0, 1, 0.02, lpt_order=3, factors=(1, 1, 1)),
                           power, 1.0)


def test_full_size_pairing_and_variance():
    """c3 lattice (512^3, 2LPT on the automatic 1024^3 IC mesh, L = 1000):
    size-independent properties of the device output."""
    a0 = 1.0 / 50.0
    L, N = 1000.0, 512
    sp = ic.start_spectrum(a0)
    out = {}
    for order, pair in ((2, "pair_a"), (2, "pair_b"), (1, "pair_a"), (1, "pair_b")):
        p = ic.ICParams(N, L, 7, a0, lpt_order=order, phase_pairing=pair)
        power = ic.power_table(p, sp)
        with hb.PMSolver(hb.MeshGeometry(L, 1024), hb.PMForceMethod.pure_pm(False)) as s:
            s.generate_ics(p, power, ic.particle_mass(L, N))
            d = s.download(acc=False)
        out[(order, pair)] = {k: d[k] for k in ("px", "py", "pz")}
    pmax = max(np.max(np.abs(out[(1, "pair_a")][k])) for k in ("px", "py", "pz"))
    for k in ("px", "py", "pz"):
        a1, b1 = out[(1, "pair_a")][k], out[(1, "pair_b")][k]
        assert np.array_equal(a1, -b1), k
        a2, b2 = out[(2, "pair_a")][k], out[(2, "pair_b")][k]
        first = 0.5 * (a2 - b2)
        second = 0.5 * (a2 + b2)
        assert np.max(np.abs(first - a1)) <= 1e-13 * pmax, k
        # the second-order part is small, not zero, and even in delta
        s_rms = float(np.sqrt(np.mean(second * second)))
        f_rms = float(np.sqrt(np.mean(a1 * a1)))
        assert 0.0 < s_rms < 0.5 * f_rms, (k, s_rms, f_rms)
        print(f"{k}: rms first-order {f_rms:.4e}, second-order {s_rms:.4e}")
    # field statistics: |delta_k|^2 / var_s has mean 1 over the support
    p = ic.ICParams(128, 250.0, 99, a0, lpt_order=1)
    M, K = p.resolve()
    power = ic.power_table(p, sp)
    f = ic.RandomField.generate(p, power)
    amp = ic.mode_amplitudes(M, 250.0, power)
    m = np.where(np.arange(M) <= M // 2, np.arange(M), np.arange(M) - M)
    s = m[:, None, None] ** 2 + m[None, :, None] ** 2 + np.arange(M // 2 + 1)[None, None, :] ** 2
    sel = (f != 0)
    ratio = np.abs(f[sel]) ** 2 / (amp[s[sel], 0] ** 2)
    n = ratio.size
    assert abs(ratio.mean() - 1.0) < 6.0 / math.sqrt(n), (ratio.mean(), n)


def test_handle_keeps_work_arrays_between_generations(ic_golden):
    """hyowon_pm_generate_ics keeps its work arrays in the handle: repeated
    generations, a change of lattice / IC mesh, and a generation after a KDK
    step (which gives the arrays back) all write the standalone call's state."""
    L = float(ic_golden["box"])
    p16, c16 = params_of(ic_golden, "n16_2lpt")
    pb, cb = params_of(ic_golden, "n16_2lpt_fixed_pair_b")
    p32 = ic.ICParams(32, L, 5, p16.a_start, lpt_order=2, factors=p16.factors)
    w32 = ic.power_table(p32, ic.start_spectrum(p16.a_start))
    ref16 = ic.generate_ics(p16, c16["power"])
    refb = ic.generate_ics(pb, cb["power"])
    ref32 = ic.generate_ics(p32, w32)
    comps = ("x", "y", "z", "px", "py", "pz")
    with hb.PMSolver(hb.MeshGeometry(L, 32), hb.PMForceMethod.pure_pm(False)) as s:
        for p, power, ref in ((p16, c16["power"], ref16), (p16, c16["power"], ref16),
                              (pb, cb["power"], refb), (p32, w32, ref32),
                              (p16, c16["power"], ref16)):
            s.generate_ics(p, power, 1.0)
            d = s.download(acc=False)
            for k in comps:
                assert np.array_equal(d[k], ref[k]), k
        s.kdk_step(1e-4, 1e-4, 1e-4)
        s.generate_ics(p16, c16["power"], 1.0)
        d = s.download(acc=False)
        for k in comps:
            assert np.array_equal(d[k], ref16[k]), k
