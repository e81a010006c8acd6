"""The benchmark configurations' synthetic inputs, for the reference's own
CPU runs (TEST INFRASTRUCTURE ONLY).

The reference arm of bench.py and the reference-side parity runs build their
initial conditions here and in oracle/_ref alone, so that no code of the
product package runs on the reference's side of a comparison:

* seeded N(0,1) white noise per lattice cell (numpy's default generator);
* the z = 0 spectrum P(k) = A k^n_s T_BBKS(k; Gamma)^2 normalised to sigma_8
  with a top-hat of R = 8 Mpc/h, at 512 log-spaced k in [1e-4, 1e2] h/Mpc,
  written as the P(k) file the reference's LinearPowerSpectrum reads;
* 1LPT through the reference's LinearPowerSpectrum, FFT and LPTDisplacement
  (Reference.lpt_white_noise).

tests/test_workload.py checks that the noise, the table and the configurations
are identical to those the product's bench leg uses (hyowon_b200.ic).
"""
from __future__ import annotations

import math
import os
import tempfile

import numpy as np

G_INTERNAL = 6.67430e-11 * (1e10 * 1.98847e30) / (3.085677581491367e22 * 1000.0 * 1000.0)
RHO_CRIT0 = 3.0 * 100.0 * 100.0 / (8.0 * math.pi * G_INTERNAL)

CONFIGS = {
    "c1": dict(n_side=32, box=100.0, mesh=64, z_start=49.0, steps=32, seed=1),
    "c2": dict(n_side=128, box=256.0, mesh=256, z_start=49.0, steps=64, seed=1),
    "c3": dict(n_side=512, box=1000.0, mesh=1024, z_start=49.0, steps=64, seed=7),
    "c4": dict(n_side=128, box=256.0, mesh=128, z_start=19.0, steps=16, seed=3),
    "c3h": dict(n_side=256, box=500.0, mesh=512, z_start=49.0, steps=64, seed=7),
}


def particle_mass(box_size: float, n_side: int, omega_m: float = 0.3) -> float:
    """rho_crit0 Omega_m (L/N)^3 (src/config/simulation_parameters.cpp:403-416)."""
    return RHO_CRIT0 * omega_m * (box_size / n_side) ** 3


def schedule(name: str):
    """(a_start, delta ln a) of a configuration: steps uniform in ln a to a = 1."""
    c = CONFIGS[name]
    a_start = 1.0 / (1.0 + c["z_start"])
    return a_start, math.log(1.0 / a_start) / c["steps"]


def white_noise(n_side: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).standard_normal(n_side ** 3)


def _bbks_transfer(k, gamma):
    q = np.asarray(k, dtype=np.float64) / gamma
    return (np.log1p(2.34 * q) / (2.34 * q)
            * (1.0 + 3.89 * q + (16.1 * q) ** 2 + (5.46 * q) ** 3 + (6.71 * q) ** 4) ** -0.25)


def _tophat(x):
    out = np.empty_like(x)
    small = x < 1e-3
    out[small] = 1.0 - x[small] ** 2 / 10.0
    xl = x[~small]
    out[~small] = 3.0 * (np.sin(xl) - xl * np.cos(xl)) / xl ** 3
    return out


def bbks_table(n=512, kmin=1e-4, kmax=1e2, sigma8=0.8, n_s=0.965, gamma=0.21, R=8.0):
    """(k, P(k)) at z = 0; sigma_8 by the trapezoid rule over ln k in [1e-6, 1e3]."""
    k = np.exp(np.linspace(math.log(kmin), math.log(kmax), n))
    lk = np.linspace(math.log(1e-6), math.log(1e3), 200001)
    kk = np.exp(lk)
    integrand = (kk ** 3 * kk ** n_s * _bbks_transfer(kk, gamma) ** 2 * _tophat(kk * R) ** 2
                 / (2.0 * math.pi ** 2))
    A = sigma8 ** 2 / np.trapezoid(integrand, lk)
    return k, A * k ** n_s * _bbks_transfer(k, gamma) ** 2


def reference_ics(ref, name: str, n_side: int = None, box: float = None, seed: int = None):
    """The configuration's 1LPT state built by the reference (oracle/_ref)."""
    from .bindings import write_power_spectrum_file
    c = CONFIGS[name]
    n_side = n_side or c["n_side"]
    box = box or c["box"]
    seed = c["seed"] if seed is None else seed
    k, P = bbks_table()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "pk.txt")
        write_power_spectrum_file(path, k, P, 0.0)
        return ref.lpt_white_noise(box, n_side, white_noise(n_side, seed), path, 0.0,
                                   c["z_start"])


def loaded_native_libraries():
    """Shared objects of this repository mapped into the current process."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libs = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 6 and parts[-1].endswith(".so") and parts[-1].startswith(root):
                    libs.add(os.path.relpath(parts[-1], root))
    except OSError:
        pass
    return sorted(libs)
