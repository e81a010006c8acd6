"""CPU tests of the generated-IC restatement (oracle/ic_oracle.py) and of the
library's host side (include/hyowon_ic.h: resolve, mode amplitudes, growth),
pinned to the reference's own outputs in tests/golden/ic.npz.

Bars:
* Philox blocks, 53-bit uniforms, Box-Muller normals, the amplitude table
  and the whole Fourier field: bit-identical (the oracle uses the C library's
  log / sin / cos, as the reference build does);
* LPT particles: positions within 4 ulp of L (minimum image), momenta within
  1e-14 of the largest |p| -- numpy's FFT and the reference build's FFT round
  differently, nothing else does;
* host growth D1, D2 within 1e-13 and f1, f2 within 1e-11 relative of the
  reference's RK4 table; P(k_s) of the repository's spline within 1e-13.
"""
import math

import numpy as np
import pytest

from oracle import ic_oracle as io

CASES = ["n16_1lpt", "n16_2lpt", "n16_2lpt_fixed_pair_b", "n12_2lpt_pair_a_k4", "n16_1lpt_m32_k5"]
# name -> (N, order, mesh request, fixed, pairing, K, seed), as generated
SPEC = {
    "n16_1lpt": (16, 1, 0, False, 0, -1, 11),
    "n16_2lpt": (16, 2, 0, False, 0, -1, 11),
    "n16_2lpt_fixed_pair_b": (16, 2, 0, True, 2, -1, 12345678901),
    "n12_2lpt_pair_a_k4": (12, 2, 0, False, 1, 4, 5),
    "n16_1lpt_m32_k5": (16, 1, 32, False, 0, 5, 3),
}


def case(g, name):
    return {k.split("__", 1)[1]: g[k] for k in g.files if k.startswith(name + "__")}


def factors(c):
    a0 = float(c["a_start"])
    p1 = a0 * a0 * float(c["H"]) * float(c["f1"])
    x2 = float(c["D2"]) / (float(c["D1"]) * float(c["D1"]))
    p2 = a0 * a0 * float(c["H"]) * float(c["f2"]) * x2
    return p1, x2, p2


def test_philox_and_draws_bit_exact(ic_golden):
    g = ic_golden
    assert np.array_equal(io.philox4x32_10(g["philox_ctr"], g["philox_key"]), g["philox_out"])
    for seed, stream in ((0, 0), (11, 0), (12345678901, 1)):
        d = io.mode_draws(seed, stream, g["draw_modes"])
        assert np.array_equal(d, g[f"draws_{seed}_{stream}"]), (seed, stream)
    u = g["draws_11_0"][:, :2]
    assert np.all((u > 0.0) & (u < 1.0))


@pytest.mark.parametrize("name", CASES)
def test_field_bit_exact(ic_golden, name):
    c = case(ic_golden, name)
    N, order, mesh, fixed, pairing, K, seed = SPEC[name]
    M, Kr = int(c["M"]), int(c["K"])
    amp = io.mode_amplitudes(M, float(ic_golden["box"]), c["power"])
    assert np.array_equal(amp, c["amp"])
    f = io.gaussian_field(M, seed, Kr, c["amp"], fixed, pairing)
    assert np.array_equal(f, c["modes"])
    # structure: zero outside the Cartesian support and at k = 0
    m = np.where(np.arange(M) <= M // 2, np.arange(M), np.arange(M) - M)
    outside = (np.abs(m)[:, None, None] > Kr) | (np.abs(m)[None, :, None] > Kr) \
        | (np.arange(M // 2 + 1)[None, None, :] > Kr)
    assert np.all(c["modes"][outside] == 0) and c["modes"][0, 0, 0] == 0
    # Hermitian pairs on the kz = 0 plane
    p0 = c["modes"][:, :, 0]
    assert np.array_equal(p0, np.conj(p0[(-np.arange(M)) % M][:, (-np.arange(M)) % M]))


@pytest.mark.parametrize("name", CASES)
def test_lpt_matches_reference(ic_golden, name):
    c = case(ic_golden, name)
    N, order = SPEC[name][:2]
    L = float(ic_golden["box"])
    p1, x2, p2 = factors(c)
    o = io.lpt(c["modes"], N, L, int(c["K"]), p1, order, x2, p2)
    ulp = np.spacing(L)
    for k in "xyz":
        d = (o[k] - c[k] + 0.5 * L) % L - 0.5 * L
        assert np.max(np.abs(d)) <= 4 * ulp, (k, np.max(np.abs(d)))
        assert np.all((o[k] >= 0.0) & (o[k] < L))
    pmax = max(np.max(np.abs(c[k])) for k in ("px", "py", "pz"))
    for k in ("px", "py", "pz"):
        assert np.max(np.abs(o[k] - c[k])) <= 1e-14 * pmax, k


def test_library_amplitudes_bit_exact(ic_golden):
    from hyowon_b200 import ic
    for name in CASES:
        c = case(ic_golden, name)
        amp = ic.mode_amplitudes(int(c["M"]), float(ic_golden["box"]), c["power"])
        assert np.array_equal(amp, c["amp"]), name
    with pytest.raises(RuntimeError):
        ic.mode_amplitudes(16, 100.0, np.array([0.0, 1.0, -1.0]))
    with pytest.raises(RuntimeError):
        ic.mode_amplitudes(16, 100.0, np.array([0.0, float("nan")]))


def test_resolve_matches_reference_rules(ic_golden):
    from hyowon_b200 import ic
    for name in CASES:
        c = case(ic_golden, name)
        N, order, mesh, fixed, pairing, K, seed = SPEC[name]
        p = ic.ICParams(N, 100.0, seed, float(c["a_start"]), lpt_order=order,
                        mesh_per_dimension=mesh, max_mode_per_axis=None if K < 0 else K,
                        factors=factors(c))
        assert p.resolve() == (int(c["M"]), int(c["K"])), name
    bad = [dict(lpt_order=3), dict(max_mode_per_axis=8), dict(max_mode_per_axis=0),
           dict(mesh_per_dimension=24), dict(lpt_order=2, mesh_per_dimension=16)]
    for kw in bad:
        with pytest.raises(ValueError):
            ic.ICParams(16, 100.0, 1, 0.02, factors=(1.0, -0.4, -1.0), **kw).resolve()
    with pytest.raises(ValueError):
        ic.ICParams(2, 100.0, 1, 0.02, factors=(1.0, -0.4, -1.0)).resolve()  # K = 0
    with pytest.raises(RuntimeError):
        ic.ICParams(16, 100.0, 1, 0.02, factors=(float("nan"), 0.0, 0.0)).resolve()


def test_host_growth_and_spectrum_match_reference(ic_golden):
    from hyowon_b200 import ic
    c = case(ic_golden, "n16_2lpt")
    a0 = float(c["a_start"])
    D1, f1, D2, f2 = (float(v[0]) for v in ic.CosmologyModel().growth2(a0))
    assert abs(D1 / float(c["D1"]) - 1) < 1e-13
    assert abs(D2 / float(c["D2"]) - 1) < 1e-13
    assert abs(f1 / float(c["f1"]) - 1) < 1e-11
    assert abs(f2 / float(c["f2"]) - 1) < 1e-11
    p1, x2, p2 = ic.lpt_factors(a0)
    r1, r2, r3 = factors(c)
    assert abs(p1 / r1 - 1) < 1e-11 and abs(x2 / r2 - 1) < 1e-13 and abs(p2 / r3 - 1) < 1e-11
    sp = ic.start_spectrum(a0, ic.LinearSpectrum(ic_golden["pk_k"], ic_golden["pk_P"]))
    p = ic.ICParams(16, 100.0, 11, a0, lpt_order=2, factors=(r1, r2, r3))
    pw = ic.power_table(p, sp)
    assert pw[0] == 0.0
    assert np.max(np.abs(pw[1:] / c["power"][1:] - 1)) < 1e-13
    k = ic.represented_wavenumbers(100.0, int(c["K"]))
    assert np.array_equal(k, io.represented_wavenumbers(100.0, int(c["K"])))
    assert k[1] == 2.0 * math.pi / 100.0
