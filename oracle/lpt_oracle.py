"""CPU restatement of HYOWON's first-order LPT map (TEST INFRASTRUCTURE ONLY).

Follows src/ic/lpt_displacement.cpp:150-384 (psi_k = i k_d delta_k / k^2 with
the Nyquist derivative zeroed, c2r normalised by 1/N^3, x = wrap(q + psi),
p = a^2 H f1 psi), src/ic/initial_conditions.cpp:295-313 (corner lattice,
particle order) and the variance normalisation of src/ic/random_field.cpp:119-129
(delta_k = r2c(w) sqrt(P N^3 / L^3) for unit-variance noise w). numpy's FFT
has the reference's conventions (unnormalised forward, 1/N^3 inverse).
Used as the checker of the device map and to build golden ICs.
"""
from __future__ import annotations

import math

import numpy as np

from hyowon_b200.ic import LinearSpectrum, mode_k2
from hyowon_b200.pm import CosmologyModel


def lpt_ics(noise, n_side: int, box: float, a_start: float, spectrum: LinearSpectrum = None,
            model: CosmologyModel = None):
    """1LPT particle state {x, y, z, px, py, pz} from white noise (float64)."""
    spectrum = spectrum or LinearSpectrum()
    model = model or CosmologyModel()
    N = n_side
    D1, f1 = model.growth(a_start)
    H = model.H(a_start)[0]
    kx, ky, kz = mode_k2(N, box)
    k2 = kx * kx + ky * ky + kz * kz
    kmag = np.sqrt(k2)
    amp = np.sqrt(spectrum(kmag) * float(D1[0]) ** 2 * N ** 3 / box ** 3)
    delta_k = np.fft.rfftn(np.asarray(noise, dtype=np.float64).reshape(N, N, N)) * amp
    delta_k[0, 0, 0] = 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        inv_k2 = np.where(k2 > 0, 1.0 / np.where(k2 > 0, k2, 1.0), 0.0)
    comps = []
    for d, kd in enumerate((kx, ky, kz)):
        kd = np.broadcast_to(kd, k2.shape).copy()
        if N % 2 == 0:
            if d == 0:
                kd[N // 2, :, :] = 0.0
            elif d == 1:
                kd[:, N // 2, :] = 0.0
            else:
                kd[:, :, N // 2] = 0.0
        psi_k = 1j * kd * inv_k2 * delta_k
        comps.append(np.fft.irfftn(psi_k, s=(N, N, N), axes=(0, 1, 2)).ravel())
    q = np.arange(N, dtype=np.float64) * (box / N)
    qx, qy, qz = np.meshgrid(q, q, q, indexing="ij")
    pf = a_start * a_start * H * float(f1[0])
    out = {}
    for name, qd, psi in (("x", qx, comps[0]), ("y", qy, comps[1]), ("z", qz, comps[2])):
        out[name] = np.mod(qd.ravel() + psi, box)
        out[name][out[name] >= box] = 0.0
        out["p" + name] = pf * psi
    return out


