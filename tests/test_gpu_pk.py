"""GPU tests of hyowon_pm_power_spectrum (the MatterPowerSpectrum estimator on
the device) against the reference's own values (tests/golden/pk.npz) and the
restatement (oracle/pk_oracle.py) on the device's own state.

Tolerances: every float field of every bin within 1e-10 relative of the
reference (binary64 deposit atomics and cuFFT vs the reference's ordered sums
and FFT differ at ~1e-15 per mode); mode counts and bin edges exact. Bin
counts are chosen so that no |k| = 2 pi |n| / L lies on an edge to the last
ulp (with 10 bins from k_f to k_Nyq = 32 k_f every other edge is a power of
two times k_f, where the device's hypot and the host libm's may round a
mode's |k| to opposite sides of the edge).
"""
import numpy as np
import pytest

import hyowon_b200 as hb
from oracle import pk_oracle
from tests.golden.make_golden import PK_CASES, PK_FIELDS

pytestmark = pytest.mark.gpu

FLOAT_FIELDS = [f for f in PK_FIELDS if f != "mode_count"]


def compare(out, ref_of, tol):
    assert np.array_equal(out["mode_count"], ref_of("mode_count"))
    for f in FLOAT_FIELDS:
        ref = ref_of(f)
        err = np.max(np.abs(out[f] - ref) / np.maximum(np.abs(ref), 1e-300))
        assert err < tol, (f, err)


@pytest.mark.parametrize("case", PK_CASES, ids=[c[0] for c in PK_CASES])
def test_fp64_matches_reference(c1_kdk, pk_golden, case):
    name, tag, mesh, nb, shot, il, frac = case
    d = c1_kdk
    with hb.PMSolver(hb.MeshGeometry(float(d["box"]), int(d["mesh"])),
                     hb.PMForceMethod.pure_pm(False)) as s:
        s.upload(d[tag + "_x"], d[tag + "_y"], d[tag + "_z"], uniform_mass=float(d["particle_mass"]))
        out = s.power_spectrum(nb, frac, shot, il, mesh_size=mesh)
        again = s.power_spectrum(nb, frac, shot, il, mesh_size=mesh)
    compare(out, lambda f: pk_golden[f"{name}__{f}"], 1e-10)
    assert np.array_equal(out["mode_count"], again["mode_count"])


@pytest.mark.parametrize("name,shot,il", [("masses_shot", True, False),
                                          ("masses_interlaced", False, True)])
def test_fp64_explicit_masses(small_pm, pk_golden, name, shot, il):
    sp = small_pm
    with hb.PMSolver(hb.MeshGeometry(float(sp["L"]), int(sp["N"])),
                     hb.PMForceMethod.pure_pm(False)) as s:
        s.upload(sp["x"], sp["y"], sp["z"], masses=sp["masses"])
        out = s.power_spectrum(5, 0.8, shot, il)
    compare(out, lambda f: pk_golden[f"{name}__{f}"], 1e-10)


@pytest.mark.parametrize("shot,il", [(True, False), (False, True)])
def test_fp32_form_matches_oracle_on_its_state(oracle, c1_kdk, shot, il):
    d = c1_kdk
    L, N = float(d["box"]), int(d["mesh"])
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), "fp32") as s:
        s.upload(d["s32_x"], d["s32_y"], d["s32_z"], uniform_mass=float(d["particle_mass"]))
        st = s.download(acc=False)
        out = s.power_spectrum(12, 1.0, shot, il)
    ref = pk_oracle.power_spectrum(oracle, L, N, st["x"], st["y"], st["z"], num_bins=12,
                                   subtract_shot_noise=shot, interlaced=il)
    compare(out, lambda f: ref[f], 1e-10)


def test_rejects_what_the_reference_rejects(c1_kdk):
    d = c1_kdk
    with hb.PMSolver(hb.MeshGeometry(float(d["box"]), int(d["mesh"])),
                     hb.PMForceMethod.pure_pm(False)) as s:
        s.upload(d["ic_x"], d["ic_y"], d["ic_z"], uniform_mass=float(d["particle_mass"]))
        with pytest.raises(ValueError):
            s.power_spectrum(8, 1.0, subtract_shot_noise=True, interlaced=True)
        with pytest.raises(ValueError):
            s.power_spectrum(0, 1.0)
        with pytest.raises(ValueError):
            s.power_spectrum(8, 0.0)
        with pytest.raises(ValueError):
            s.power_spectrum(8, 1.5)
        with pytest.raises(ValueError):   # k_max below the fundamental: no shell
            s.power_spectrum(4, 1e-3)
