"""GPU tests of the differentiation form (hyowon_vjp_1lpt_pm).

Stated tolerances:
* forward loss of the binary64 form vs the oracle (1LPT + KDK + CIC deposit on
  the CPU): relative 1e-8;
* gradient vs central finite differences of the binary64 forward model
  (eps = 1e-3 in the noise, 64 random cells of the 128^3 configuration): the
  relative error ||g - g_fd|| / ||g_fd|| <= 1e-3, for the binary64 gradient
  and for the FP32 gradient (whose own FP32 losses are too noisy for central
  differences at this eps);
* FP32 gradient vs binary64 gradient: relative 1e-3;
* checkpoint interval: gradients with ckpt_every 1 / 4 / 16 agree to 1e-9;
* cost: (forward + adjoint) / forward <= 3 with the module's own forward
  (the best of three evaluations); bench.py --workload adjoint reports it
  against the production forward as well.
"""
import math

import numpy as np
import pytest

from hyowon_b200 import ic
from hyowon_b200.adjoint import DifferentiablePM

pytestmark = pytest.mark.gpu


def oracle_final_delta(oracle, dpm, noise):
    from oracle.lpt_oracle import lpt_ics
    a0 = 1.0 / 20.0
    st = lpt_ics(noise, dpm.n_side, dpm.box, a0)
    for k in ("ax", "ay", "az"):
        st[k] = np.zeros_like(st["x"])
    oracle.pm_forces(dpm.box, dpm.mesh, st["x"], st["y"], st["z"], uniform_mass=dpm.m,
                     ax=st["ax"], ay=st["ay"], az=st["az"])
    for K1, D, K2 in zip(dpm.K1, dpm.D, dpm.K2):
        oracle.kdk_step(dpm.box, dpm.mesh, st, K1, D, K2, uniform_mass=dpm.m)
    mesh = oracle.deposit(dpm.box, dpm.mesh, st["x"], st["y"], st["z"], uniform_mass=dpm.m)
    mbar = dpm.m * dpm.n_side ** 3 / dpm.mesh ** 3
    return mesh / mbar - 1.0


def test_forward_model_matches_oracle(oracle):
    dpm = DifferentiablePM(64.0, 32, 32, 1 / 20, 8, "fp64")
    noise = ic.white_noise(32, 3)
    target = ic.white_noise(32, 4) * 0.1
    got = dpm.final_delta(noise)
    ref = oracle_final_delta(oracle, dpm, noise)
    assert np.max(np.abs(got - ref)) <= 1e-8 * np.max(np.abs(ref))
    loss = dpm.loss(noise, target)
    ref_loss = 0.5 * np.sum((ref - target) ** 2)
    assert loss == pytest.approx(ref_loss, rel=1e-8)


def fd_check(dpm, noise, target, cells, eps=1e-3):
    loss, grad = dpm.loss_and_grad(noise, target)
    fd = np.empty(len(cells))
    for i, c in enumerate(cells):
        w = noise.copy()
        w[c] += eps
        lp = dpm.loss(w, target)
        w[c] -= 2 * eps
        lm = dpm.loss(w, target)
        fd[i] = (lp - lm) / (2 * eps)
    return grad, grad[cells], fd


def c4_problem(precision, ckpt=4):
    cfg = ic.CONFIGS["c4"]
    dpm = DifferentiablePM(cfg["box"], cfg["n_side"], cfg["mesh"], 1 / (1 + cfg["z_start"]),
                           cfg["steps"], precision, ckpt)
    noise = ic.white_noise(cfg["n_side"], cfg["seed"])
    target = dpm.final_delta(ic.white_noise(cfg["n_side"], 4))
    return dpm, noise, target


@pytest.fixture(scope="module")
def c4_fd():
    """Binary64 gradient and central differences on 64 random noise cells."""
    dpm, noise, target = c4_problem("fp64")
    cells = np.random.default_rng(12).choice(noise.size, 64, replace=False)
    grad, g, fd = fd_check(dpm, noise, target, cells)
    return noise, target, cells, grad, fd


def test_gradient_vs_finite_differences_c4_fp64(c4_fd):
    _, _, cells, grad, fd = c4_fd
    err = np.linalg.norm(grad[cells] - fd) / np.linalg.norm(fd)
    print(f"c4 FP64: |g - fd| / |fd| = {err:.3e} (64 cells)")
    assert err <= 1e-3
    assert np.all(np.isfinite(grad))


def test_gradient_fp32_vs_fp64_and_fd_c4(c4_fd):
    noise, target, cells, g64, fd = c4_fd
    d64, _, _ = c4_problem("fp64")
    d32, _, _ = c4_problem("fp32")
    l64 = d64.loss(noise, target)
    l32, g32 = d32.loss_and_grad(noise, target)
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    print(f"c4 FP32 vs FP64: loss rel {abs(l32 / l64 - 1):.3e}, gradient rel {rel:.3e}")
    assert abs(l32 / l64 - 1) <= 1e-3
    assert rel <= 1e-3
    err = np.linalg.norm(g32[cells] - fd) / np.linalg.norm(fd)
    print(f"c4 FP32 gradient vs binary64 FD: {err:.3e} (64 cells)")
    assert err <= 1e-3


def test_checkpoint_interval_does_not_change_gradient():
    grads = []
    for ckpt in (1, 4, 16):
        dpm, noise, target = c4_problem("fp64", ckpt)
        grads.append(dpm.loss_and_grad(noise, target)[1])
    for g in grads[1:]:
        assert np.linalg.norm(g - grads[0]) <= 1e-9 * np.linalg.norm(grads[0])


def test_adjoint_cost_ratio_c4():
    dpm, noise, target = c4_problem("fp64")
    dpm.loss_and_grad(noise, target)
    ratios = []
    for _ in range(3):
        dpm.loss_and_grad(noise, target)
        t = dpm.last_timings
        ratios.append((t["forward_ms"] + t["reverse_ms"]) / t["forward_ms"])
    ratio = min(ratios)
    print(f"c4 (forward + adjoint) / forward = {ratio:.2f} "
          f"(forward {t['forward_ms']:.1f} ms, reverse {t['reverse_ms']:.1f} ms)")
    assert ratio <= 3.0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_handle_vjp_equals_standalone_vjp(precision):
    """hyowon_pm_vjp on a PM handle (the drop-in's vjp(handle, ...)) gives the
    standalone call's loss and gradient, and a second call on the same handle
    (reusing its adjoint plans and work arrays) the same again. Tolerances,
    relative: binary64 1e-12; FP32 1e-6 (loss) and 1e-4 (gradient, measured
    3e-6): the adjoint's deposit and scatter sum with atomics, so the last bits
    move between calls and the FP32 reverse pass carries them into the
    gradient."""
    import hyowon_b200 as hb
    cfg = ic.CONFIGS["c4"]
    noise = ic.white_noise(32, 3)
    target = ic.white_noise(32, 4) * 0.1
    ref = DifferentiablePM(64.0, 32, 32, 1 / 20, 8, precision)
    l0, g0 = ref.loss_and_grad(noise, target)
    with hb.PMSolver(hb.MeshGeometry(64.0, 32), hb.PMForceMethod.pure_pm(False), precision) as s:
        dpm = DifferentiablePM(64.0, 32, 32, 1 / 20, 8, precision, solver=s)
        tol_l, tol_g = (1e-12, 1e-12) if precision == "fp64" else (1e-6, 1e-4)
        for _ in range(2):
            l1, g1 = dpm.loss_and_grad(noise, target)
            assert abs(l1 / l0 - 1) <= tol_l
            assert np.linalg.norm(g1 - g0) <= tol_g * np.linalg.norm(g0)
    assert cfg["n_side"] == 128  # the c4 sizes are exercised by the tests above
