"""The white-noise 1LPT map pinned to the reference (tests/golden/lpt.npz).

The fixture holds the reference's own 1LPT state for the configs' white noise:
LinearPowerSpectrum of the BBKS table file, the FFTBackend r2c, the variance
scaling sqrt(P N^3 / L^3) and LPTDisplacement::apply_to_arrays
(src/ic/lpt_displacement.cpp:150-384) on the corner lattice.

CPU: the oracle's numpy restatement (oracle/lpt_oracle.py) against it, and the
reference-side workload inputs (oracle/workload.py) against the product's
(hyowon_b200.ic). GPU: the device map (hyowon_pm_lpt_ics) against it.

Tolerances: positions 1e-13 L (wrapped difference; FFT rounding only, the
reference's FFT and numpy's differ in summation order), momenta 1e-11 of
max |p| (D1, f1 and H come from each side's own cosmology integrator: D1 and
H agree to a few 1e-15, the growth rate f1 to 5e-13 at z = 49 and 3e-12 at
z = 19, and the momenta carry that difference)."""
import numpy as np
import pytest

from conftest import load_golden

CASES = ["c1", "s16_z19"]


def case(name):
    g = load_golden("lpt.npz")
    n_side, box, seed, z_start = g[f"{name}__args"]
    st = {k: g[f"{name}__{k}"] for k in ("x", "y", "z", "px", "py", "pz")}
    return int(n_side), float(box), int(seed), float(z_start), st


def compare(got, ref, box):
    err_x = max(np.max(np.abs((got[k] - ref[k] + box / 2) % box - box / 2)) for k in "xyz")
    pmax = max(np.max(np.abs(ref[k])) for k in ("px", "py", "pz"))
    err_p = max(np.max(np.abs(got[k] - ref[k])) for k in ("px", "py", "pz"))
    return err_x / box, err_p / pmax


@pytest.mark.parametrize("name", CASES)
def test_oracle_lpt_matches_reference(name):
    from hyowon_b200 import ic
    from oracle.lpt_oracle import lpt_ics
    n_side, box, seed, z_start, ref = case(name)
    got = lpt_ics(ic.white_noise(n_side, seed), n_side, box, 1.0 / (1.0 + z_start))
    ex, ep = compare(got, ref, box)
    print(f"{name}: oracle vs reference: positions {ex:.2e} L, momenta {ep:.2e} max|p|")
    assert ex <= 1e-13 and ep <= 1e-11


def test_reference_side_workload_inputs_equal_the_products():
    from hyowon_b200 import ic
    from oracle import workload
    k1, P1 = workload.bbks_table()
    k2, P2 = ic.bbks_table()
    assert np.array_equal(k1, k2) and np.array_equal(P1, P2)
    assert np.array_equal(workload.white_noise(16, 3), ic.white_noise(16, 3))
    for name, c in workload.CONFIGS.items():
        assert c == ic.CONFIGS[name], name
        assert workload.schedule(name) == ic.config_schedule(name)
        assert workload.particle_mass(c["box"], c["n_side"]) == ic.particle_mass(c["box"], c["n_side"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_device_lpt_matches_reference(name):
    import hyowon_b200 as hb
    from hyowon_b200 import ic
    n_side, box, seed, z_start, ref = case(name)
    a0 = 1.0 / (1.0 + z_start)
    with hb.PMSolver(hb.MeshGeometry(box, 2 * n_side), hb.PMForceMethod.pure_pm(False)) as s:
        ic.lpt_on_device(s, ic.white_noise(n_side, seed), n_side, a0,
                         ic.particle_mass(box, n_side))
        got = s.download(acc=False)
    ex, ep = compare(got, ref, box)
    print(f"{name}: device vs reference: positions {ex:.2e} L, momenta {ep:.2e} max|p|")
    assert ex <= 1e-13 and ep <= 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_device_lpt_precision_form_matches_reference(name):
    """The precision form stores positions as 32-bit fixed point (L 2^-32
    resolution) and momenta in FP32."""
    import hyowon_b200 as hb
    from hyowon_b200 import ic
    n_side, box, seed, z_start, ref = case(name)
    a0 = 1.0 / (1.0 + z_start)
    with hb.PMSolver(hb.MeshGeometry(box, 2 * n_side), hb.PMForceMethod.pure_pm(False),
                     precision="fp32") as s:
        ic.lpt_on_device(s, ic.white_noise(n_side, seed), n_side, a0,
                         ic.particle_mass(box, n_side))
        got = s.download(acc=False)
    ex, ep = compare(got, ref, box)
    print(f"{name}: precision form vs reference: positions {ex:.2e} L, momenta {ep:.2e} max|p|")
    assert ex <= 2.0 ** -32 + 1e-13 and ep <= 2e-7
