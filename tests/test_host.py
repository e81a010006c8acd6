"""CPU tests of the host side of the product: the C ABI library loads and
exports every symbol its headers declare, the host cosmology matches the
reference's schedule, and the synthetic IC generator behaves. No GPU calls."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"^\s*(?:int|const char\*|void)\s+(hyowon_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from hyowon_b200 import _native
    L = _native.lib()
    decl = declared_symbols()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(L, name), name
    # the Python binding covers the whole ABI
    assert set(decl) <= set(_native.exported_symbols())


def test_schedule_matches_reference(schedules):
    from hyowon_b200 import TimeStepper
    for name in ("c1", "c2", "c4"):
        a0, a1, dl = schedules[name + "_args"]
        ref = schedules[name]
        ts = TimeStepper(a0, a1, dl)
        assert ts.num_steps() == ref.shape[0] == {"c1": 32, "c2": 64, "c4": 16}[name]
        # boundaries and geometric midpoints are bit-exact
        assert np.array_equal(ts.table[:, :3], ref[:, :3])
        # drift / kick quadrature agrees to the binary64 spacing
        np.testing.assert_allclose(ts.table[:, 3:], ref[:, 3:], rtol=1e-15, atol=0)


def test_geometric_mean_correctly_rounded():
    from hyowon_b200 import _native
    from fractions import Fraction
    L = _native.lib()
    rng = np.random.default_rng(5)
    out = ctypes.c_double()
    for _ in range(2000):
        a, b = np.exp(rng.uniform(-30, 30, 2))
        assert L.hyowon_geometric_mean(a, b, ctypes.byref(out)) == 0
        g = out.value
        # correctly rounded: g^2 closest to a*b among neighbours
        exact = Fraction(a) * Fraction(b)
        lo, hi = np.nextafter(g, 0), np.nextafter(g, np.inf)
        mid_lo = (Fraction(lo) + Fraction(g)) / 2
        mid_hi = (Fraction(g) + Fraction(hi)) / 2
        assert mid_lo ** 2 <= exact <= mid_hi ** 2


def test_hubble_and_growth():
    from hyowon_b200 import CosmologyModel
    m = CosmologyModel(0.3, 0.7)
    assert m.H(1.0)[0] == pytest.approx(100.0, rel=1e-15)
    assert m.H(0.5)[0] == pytest.approx(100 * math.sqrt(0.3 * 8 + 0.7), rel=1e-15)
    D, f = m.growth(np.array([1.0, 0.02]))
    assert D[0] == pytest.approx(1.0, rel=1e-14)
    # matter era: D ~ a, f ~ 1
    assert D[1] == pytest.approx(0.02 / 0.7789, rel=1e-3)
    assert f[1] == pytest.approx(1.0, abs=5e-4)


def test_invalid_schedule_raises():
    from hyowon_b200 import TimeStepper
    with pytest.raises(ValueError):
        TimeStepper(0.5, 0.25, 0.1)
    with pytest.raises(ValueError):
        TimeStepper(0.5, 1.0, -0.1)


def test_ic_generator_matches_numpy_restatement():
    from hyowon_b200 import ic
    k, P = ic.bbks_table()
    assert k.size == 512 and k[0] == pytest.approx(1e-4) and k[-1] == pytest.approx(1e2)
    # sigma_8 normalisation
    lk = np.linspace(math.log(1e-5), math.log(1e2), 40001)
    kk = np.exp(lk)
    s = ic.LinearSpectrum(k, P)
    s2 = np.trapezoid(kk ** 3 * s(kk) * ic._tophat(8 * kk) ** 2 / (2 * math.pi ** 2), lk)
    assert math.sqrt(s2) == pytest.approx(0.8, rel=2e-3)
    from oracle.lpt_oracle import lpt_ics
    st = lpt_ics(ic.white_noise(16, 1), 16, 100.0, 1 / 50)
    assert all(np.all((st[a] >= 0) & (st[a] < 100.0)) for a in "xyz")
    # displacement field has zero mean (k=0 removed)
    q = np.arange(16) * 100 / 16
    qx = np.repeat(q, 256)
    dx = (st["x"] - qx + 50) % 100 - 50
    assert abs(dx.mean()) < 1e-12
    # p = a^2 H f1 psi
    from hyowon_b200 import CosmologyModel
    m = CosmologyModel()
    D, f = m.growth(1 / 50)
    np.testing.assert_allclose(st["px"], (1 / 50) ** 2 * m.H(1 / 50)[0] * f[0] * dx,
                               rtol=1e-9, atol=1e-9)


def test_particle_mass():
    from hyowon_b200 import ic
    # rho_crit0 = 3 H0^2 / (8 pi G) = 27.75 (1e10 Msun/h) / (Mpc/h)^3
    assert ic.RHO_CRIT0 == pytest.approx(27.754, rel=1e-3)
    assert ic.particle_mass(100.0, 32) == pytest.approx(27.754 * 0.3 * (100 / 32) ** 3, rel=1e-3)


def test_clock_sampler_keeps_readings_inside_the_timed_region(tmp_path, monkeypatch):
    """bench.py's clock sampler, driven by a stand-in nvidia-smi that prints a
    timestamped reading every 50 ms: it waits for the first reading, keeps only
    those stamped inside the region, and names active slowdown reasons."""
    import sys
    import time
    fake = tmp_path / "nvidia-smi"
    fake.write_text(
        "#!" + sys.executable + "\n"
        "import datetime, sys, time\n"
        "time.sleep(0.3)\n"
        "i = 0\n"
        "while True:\n"
        "    t = datetime.datetime.now().strftime('%Y/%m/%d %H:%M:%S.%f')[:-3]\n"
        "    slow = 'Active' if i == 3 else 'Not Active'\n"
        "    print(f'{t}, 0, 1965, 1965, 700.00, 0x0, Not Active, Not Active, {slow}, Not Active',"
        " flush=True)\n"
        "    i += 1\n"
        "    time.sleep(0.05)\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", str(tmp_path) + os.pathsep + os.environ["PATH"])
    import bench
    with bench.ClockSampler(0) as clk:
        time.sleep(0.5)
    s = clk.summary()
    # about 10 readings in 0.5 s; none of the 0.3 s start-up is in the region
    assert 5 <= s["samples"] <= 12, s
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_thermal_slowdown"], s
    with bench.ClockSampler(0) as clk:
        pass
    assert clk.summary()["samples"] <= 1
