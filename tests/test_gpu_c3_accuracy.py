"""The precision form's accuracy targets at the throughput workload c3
(512^3 particles, 1024^3 mesh, L = 1000 Mpc/h, 1LPT at z = 49, seed 7,
64 KDK steps to z = 0), against the binary64 form on the same device:

* force relative RMS <= 1e-4 over all particles: both forms' forces at the
  binary64 run's z = 0 positions;
* P(k) of the z = 0 states (the device estimator, raw power) within 0.1 %
  in every logarithmic bin below k_Nyquist / 2;
* final-position RMS <= 0.05 cell (chaotic growth of the FP32 round-off).
"""
import math

import numpy as np
import pytest

import hyowon_b200 as hb
from hyowon_b200 import ic

pytestmark = pytest.mark.gpu


def test_precision_form_c3_z0_targets():
    cfg = ic.CONFIGS["c3"]
    n_side, N, L = cfg["n_side"], cfg["mesh"], cfg["box"]
    a0, dl = ic.config_schedule("c3")
    K1, D, K2 = hb.TimeStepper(a0, 1.0, dl).factors()
    m = ic.particle_mass(L, n_side)
    noise = ic.white_noise(n_side, cfg["seed"])
    geom = hb.MeshGeometry(L, N)
    method = hb.PMForceMethod.pure_pm(False)
    kn = math.pi * N / L
    with hb.PMSolver(geom, method, "fp64") as s:
        ic.lpt_on_device(s, noise, n_side, a0, m)
        s.run(K1, D, K2)
        pk64 = s.power_spectrum(40, 1.0)
        f64 = s.download()
    with hb.PMSolver(geom, method, "fp32") as s:
        ic.lpt_on_device(s, noise, n_side, a0, m)
        s.run(K1, D, K2)
        pk32 = s.power_spectrum(40, 1.0)
        f32 = s.download(acc=False)
        s.upload(f64["x"], f64["y"], f64["z"], uniform_mass=m)
        s.solve_forces()
        same = s.download()
    num = sum(float(np.sum((same[k] - f64[k]) ** 2)) for k in ("ax", "ay", "az"))
    den = sum(float(np.sum(f64[k] ** 2)) for k in ("ax", "ay", "az"))
    err = math.sqrt(num / den)
    dx = L / N
    pos_rms = math.sqrt(np.mean([float(np.mean(((f32[k] - f64[k] + L / 2) % L - L / 2) ** 2))
                                 for k in "xyz"])) / dx
    sel = (pk64["mode_count"] > 0) & (pk64["k_high"] <= 0.5 * kn)
    ratio = pk32["p_raw"][sel] / pk64["p_raw"][sel]
    print(f"c3 z=0 FP32 vs FP64: force rel RMS {err:.3e}, position RMS {pos_rms:.3e} cells, "
          f"max |P32/P64-1| below k_Nyq/2 {np.max(np.abs(ratio - 1)):.3e} ({int(sel.sum())} bins)")
    assert np.array_equal(pk32["mode_count"], pk64["mode_count"])
    assert err <= 1e-4
    assert pos_rms <= 0.05
    assert np.max(np.abs(ratio - 1)) <= 1e-3
