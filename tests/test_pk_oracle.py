"""The power-spectrum restatement (oracle/pk_oracle.py) pinned to the
reference's MatterPowerSpectrum::compute_pk (tests/golden/pk.npz, made by
tests/golden/make_golden.py). Tolerance: 1e-13 relative per bin field, mode
counts and bin edges exact to 1 ulp."""
import numpy as np
import pytest

from oracle import pk_oracle
from tests.golden.make_golden import PK_CASES, PK_FIELDS

FLOAT_FIELDS = [f for f in PK_FIELDS if f != "mode_count"]


def compare(out, g, name, tol):
    assert np.array_equal(out["mode_count"], g[f"{name}__mode_count"]), name
    for f in FLOAT_FIELDS:
        ref = g[f"{name}__{f}"]
        err = np.max(np.abs(out[f] - ref) / np.maximum(np.abs(ref), 1e-300))
        assert err < tol, (name, f, err)


@pytest.mark.parametrize("case", PK_CASES, ids=[c[0] for c in PK_CASES])
def test_c1_power_spectrum_matches_reference(oracle, c1_kdk, pk_golden, case):
    name, tag, mesh, nb, shot, il, frac = case
    d = c1_kdk
    out = pk_oracle.power_spectrum(oracle, float(d["box"]), mesh, d[tag + "_x"], d[tag + "_y"],
                                   d[tag + "_z"], num_bins=nb, subtract_shot_noise=shot,
                                   interlaced=il, max_k_fraction_nyquist=frac)
    compare(out, pk_golden, name, 1e-13)


@pytest.mark.parametrize("name,shot,il", [("masses_shot", True, False),
                                          ("masses_interlaced", False, True)])
def test_explicit_masses_match_reference(oracle, small_pm, pk_golden, name, shot, il):
    s = small_pm
    out = pk_oracle.power_spectrum(oracle, float(s["L"]), int(s["N"]), s["x"], s["y"], s["z"],
                                   masses=s["masses"], num_bins=5, subtract_shot_noise=shot,
                                   interlaced=il, max_k_fraction_nyquist=0.8)
    compare(out, pk_golden, name, 1e-13)
