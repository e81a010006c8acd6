"""GPU tests of the precision form (u32 fixed-point positions, int64
fixed-point offset-from-mean deposit, FP32 FFT / Green / gather, FP64 drift).

Stated tolerances against binary64 (the oracle, or the binary64 GPU form that
is itself pinned to the oracle):
* deposit: |m_fixed - m_f64| <= 8 m_p 2^-15 per cell (16-bit CIC fractions);
* force relative RMS <= 1e-4 (c1 initial conditions, and c2 at z = 0);
* c2 after 64 steps: position RMS <= 0.05 cell; P(k) within 0.1% of the
  binary64 run for k < k_Nyq / 2;
* bit-identical results run to run (integer deposit).
"""
import math

import numpy as np
import pytest

import hyowon_b200 as hb
from hyowon_b200 import ic

pytestmark = pytest.mark.gpu


def solver(L, N, precision):
    return hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), precision)


def rel_rms3(a, b):
    num = sum(np.sum((a[k] - b[k]) ** 2) for k in ("ax", "ay", "az"))
    den = sum(np.sum(b[k] ** 2) for k in ("ax", "ay", "az"))
    return math.sqrt(num / den)


def test_fixed_point_deposit_matches_oracle(c1_kdk, oracle):
    c = c1_kdk
    L, N, m = float(c["box"]), int(c["mesh"]), float(c["particle_mass"])
    with solver(L, N, "fp32") as s:
        s.upload(c["ic_x"], c["ic_y"], c["ic_z"], uniform_mass=m)
        mesh = s.mass_mesh()
    ref = oracle.deposit(L, N, c["ic_x"], c["ic_y"], c["ic_z"], uniform_mass=m)
    assert np.max(np.abs(mesh - ref)) <= 8 * m * 2.0 ** -15
    # integer deposit conserves mass exactly (n 2^48 units)
    assert abs(mesh.sum() - m * c["ic_x"].size) <= 1e-9 * m * c["ic_x"].size


def test_precision_form_force_error_c1(c1_kdk):
    c = c1_kdk
    L, N, m = float(c["box"]), int(c["mesh"]), float(c["particle_mass"])
    with solver(L, N, "fp32") as s:
        s.upload(c["ic_x"], c["ic_y"], c["ic_z"], c["ic_px"], c["ic_py"], c["ic_pz"],
                 uniform_mass=m)
        s.solve_forces()
        got = s.download()
    ref = {"ax": c["f0_x"], "ay": c["f0_y"], "az": c["f0_z"]}
    err = rel_rms3(got, ref)
    print(f"c1 FP32 force relative RMS vs reference: {err:.3e}")
    assert err <= 1e-4


def test_precision_form_is_deterministic(c1_kdk, schedules):
    c = c1_kdk
    L, N, m = float(c["box"]), int(c["mesh"]), float(c["particle_mass"])
    sched = schedules["c1"][:8]
    outs = []
    for _ in range(2):
        with solver(L, N, "fp32") as s:
            s.upload(c["ic_x"], c["ic_y"], c["ic_z"], c["ic_px"], c["ic_py"], c["ic_pz"],
                     uniform_mass=m)
            s.run(sched[:, 4], sched[:, 3], sched[:, 5])
            outs.append((s.download(), s.mass_mesh()))
    for k in outs[0][0]:
        assert np.array_equal(outs[0][0][k], outs[1][0][k]), k
    assert np.array_equal(outs[0][1], outs[1][1])


def test_precision_form_c1_evolution(c1_kdk, schedules):
    c = c1_kdk
    L, N, m = float(c["box"]), int(c["mesh"]), float(c["particle_mass"])
    sched = schedules["c1"]
    with solver(L, N, "fp32") as s:
        s.upload(c["ic_x"], c["ic_y"], c["ic_z"], c["ic_px"], c["ic_py"], c["ic_pz"],
                 uniform_mass=m)
        s.run(sched[:, 4], sched[:, 3], sched[:, 5])
        fin = s.download()
    dx = L / N
    pos_rms = math.sqrt(np.mean([(((fin[k] - c["s32_" + k] + L / 2) % L - L / 2) ** 2).mean()
                                 for k in "xyz"])) / dx
    ref = {"ax": c["s32_ax"], "ay": c["s32_ay"], "az": c["s32_az"]}
    err = rel_rms3(fin, ref)
    print(f"c1 FP32 after 32 steps: position RMS {pos_rms:.3e} cells, force rel RMS {err:.3e}")
    assert pos_rms <= 0.05
    assert err <= 1e-2


def cic_power(L, N, pos, oracle, n_bins=40):
    """P(k) of the CIC density (oracle deposit + numpy FFT), log bins to k_Nyq."""
    m = oracle.deposit(L, N, pos["x"], pos["y"], pos["z"], uniform_mass=1.0)
    delta = m / m.mean() - 1.0
    dk = np.fft.rfftn(delta.reshape(N, N, N))
    p = np.abs(dk) ** 2
    kx, ky, kz = ic.mode_k2(N, L)
    k = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    kf, kn = 2 * math.pi / L, math.pi * N / L
    edges = np.exp(np.linspace(math.log(kf), math.log(kn), n_bins + 1))
    idx = np.digitize(k.ravel(), edges) - 1
    ok = (idx >= 0) & (idx < n_bins)
    s = np.bincount(idx[ok], weights=p.ravel()[ok], minlength=n_bins)
    cnt = np.bincount(idx[ok], minlength=n_bins)
    kc = np.bincount(idx[ok], weights=k.ravel()[ok], minlength=n_bins)
    good = cnt > 0
    return kc[good] / cnt[good], s[good] / cnt[good]


def test_precision_form_c2_accuracy_targets(oracle):
    name = "c2"
    cfg = ic.CONFIGS[name]
    n_side, N, L = cfg["n_side"], cfg["mesh"], cfg["box"]
    a0, dl = ic.config_schedule(name)
    stepper = hb.TimeStepper(a0, 1.0, dl)
    K1, D, K2 = stepper.factors()
    m = ic.particle_mass(L, n_side)
    noise = ic.white_noise(n_side, cfg["seed"])
    res = {}
    for form in ("fp64", "fp32"):
        with solver(L, N, form) as s:
            ic.lpt_on_device(s, noise, n_side, a0, m)
            s.run(K1, D, K2)
            res[form] = s.download()
    f64, f32 = res["fp64"], res["fp32"]
    # force error of the precision form on the same z = 0 positions
    with solver(L, N, "fp32") as s:
        s.upload(f64["x"], f64["y"], f64["z"], uniform_mass=m)
        s.solve_forces()
        same = s.download()
    err = rel_rms3(same, f64)
    dx = L / N
    pos_rms = math.sqrt(np.mean([(((f32[k] - f64[k] + L / 2) % L - L / 2) ** 2).mean()
                                 for k in "xyz"])) / dx
    k, p64 = cic_power(L, N, f64, oracle)
    _, p32 = cic_power(L, N, f32, oracle)
    sel = k < 0.5 * math.pi * N / L
    ratio = p32[sel] / p64[sel]
    print(f"c2 z=0 FP32 vs FP64: force rel RMS {err:.3e}, position RMS {pos_rms:.3e} cells, "
          f"max |P32/P64-1| below k_Nyq/2 {np.max(np.abs(ratio - 1)):.3e}")
    assert err <= 1e-4
    assert pos_rms <= 0.05
    assert np.max(np.abs(ratio - 1)) <= 1e-3
