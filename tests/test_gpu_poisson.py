"""The five-pass potential solve (the deposit's r2c along z of each finished
tile, pm_chunk.cuh; pm_poisson.cu: y transforms, x transform with the Green's
multiply, inverse y + z c2r) on power-of-two meshes, against the oracle's
potential (its own FFT, pinned to the reference), for every radix layout the
passes use (N = 32 .. 512 covers a final radix of 2, 4, 8 and 16, one to three
stages in the row and column transforms, and deposit tiles of 128 down to 8
rows); at N = 1024 against a plain torch binary64 spectral
solve (torch.fft.rfftn / irfftn of the downloaded mass mesh with the same
discrete-Laplacian Green's function).

Tolerances: binary64 max |error| <= 1e-12 of the largest potential value;
precision form relative RMS <= 2e-5 (FP32 transforms of the fixed-point
mass, 16-bit CIC fractions)."""
import numpy as np
import pytest

import hyowon_b200 as hb

pytestmark = pytest.mark.gpu


def particles(N, L, seed, clustered):
    rng = np.random.default_rng(seed)
    n = min(N ** 3 // 2, 4_000_000)
    if clustered:
        centres = rng.uniform(0, L, (16, 3))
        pick = centres[rng.integers(0, 16, n)]
        pos = (pick + rng.normal(scale=0.04 * L, size=(n, 3))) % L
    else:
        pos = rng.uniform(0, L, (n, 3))
    return pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy()


@pytest.mark.parametrize("N", [32, 64, 128, 256, 512])
@pytest.mark.parametrize("deconvolve", [False, True])
def test_potential_fp64_matches_oracle(oracle, N, deconvolve):
    L, m = 50.0, 0.37
    x, y, z = particles(N, L, N, clustered=True)
    _, ref = oracle.potential(L, N, x, y, z, uniform_mass=m, deconvolve=deconvolve)
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(deconvolve)) as s:
        s.upload(x, y, z, uniform_mass=m)
        s.solve_forces()
        phi = s.potential().reshape(-1)
    err = np.max(np.abs(phi - ref)) / np.max(np.abs(ref))
    print(f"N={N} deconvolve={deconvolve}: max error / max |phi| = {err:.3e}")
    assert err <= 1e-12


@pytest.mark.parametrize("N", [32, 64, 128, 256, 512])
def test_potential_fp32_matches_oracle(oracle, N):
    L, m = 50.0, 0.37
    x, y, z = particles(N, L, 2 * N, clustered=False)
    _, ref = oracle.potential(L, N, x, y, z, uniform_mass=m)
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), "fp32") as s:
        s.upload(x, y, z, uniform_mass=m)
        s.solve_forces()
        phi = s.potential().reshape(-1)
    err = float(np.sqrt(np.sum((phi - ref) ** 2) / np.sum(ref ** 2)))
    print(f"N={N} fp32: potential relative RMS {err:.3e}")
    assert err <= 2e-5


def torch_potential(mass, L, N, four_pi_G):
    """phi = irfftn(rfftn(rho - mean) * 4 pi G / sum_axes(-4/dx^2 sin^2(pi m/N))),
    rho = mass / dx^3, in torch binary64 on the GPU."""
    import torch
    dev = torch.device("cuda", 0)
    dx = L / N
    rho = torch.from_numpy(mass.reshape(N, N, N)).to(dev) / dx ** 3
    rho -= rho.mean()
    modes = torch.fft.rfftn(rho)
    del rho
    m = torch.arange(N, device=dev, dtype=torch.float64)
    lap = -4.0 / dx ** 2 * torch.sin(torch.pi * m / N) ** 2
    lz = lap[: N // 2 + 1]
    denom = lap.view(N, 1, 1) + lap.view(1, N, 1) + lz.view(1, 1, -1)
    denom[0, 0, 0] = 1.0
    modes *= four_pi_G / denom
    modes[0, 0, 0] = 0.0
    del denom
    phi = torch.fft.irfftn(modes, s=(N, N, N))
    return phi.cpu().numpy().reshape(-1)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-5)])
def test_potential_n1024_matches_torch(oracle, precision, tol):
    N, L, m = 1024, 1000.0, 62.0
    x, y, z = particles(N, L, 1024, clustered=True)
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), precision) as s:
        s.upload(x, y, z, uniform_mass=m)
        s.solve_forces()
        phi = s.potential().reshape(-1)
        mass = s.mass_mesh().reshape(-1)
    ref = torch_potential(mass, L, N, 4.0 * np.pi * oracle.G())
    if precision == "fp64":
        err = np.max(np.abs(phi - ref)) / np.max(np.abs(ref))
    else:
        err = float(np.sqrt(np.sum((phi - ref) ** 2) / np.sum(ref ** 2)))
    print(f"N=1024 {precision}: error vs torch {err:.3e}")
    assert err <= tol
