"""CPU restatement of HYOWON's matter power spectrum estimator
(TEST INFRASTRUCTURE ONLY; the checker for hyowon_pm_power_spectrum).

Follows analysis::MatterPowerSpectrum::compute_pk
(src/analysis/matter_power_spectrum.cpp:50-226) over
FourierDensityBuilder::build (src/analysis/fourier_density_field.cpp:110-376):

* CIC deposit of the particles in units of the largest mass (uniform mass:
  weight 1 per particle), mean weight per cell = sum(w) / N^3, density
  contrast rho / mean - 1, unnormalised r2c, modes times 1/N^3;
* interlaced: a second field from positions wrap(x - dx/2, L) combined as
  0.5 (F + F_shift e^{-i (kx+ky+kz) dx/2}); the k = 0 mode is zeroed;
* per mode with 0 < |k| <= k_max (k_max = fraction * pi N / L): raw power
  L^3 |delta_k|^2; CIC window W = prod_axes min(1, |sin(a)/a|)^2,
  a = k_axis dx / 2 (include/cosmo_nbody/analysis/cic_spectral_window.hpp); deconvolution 1/W^2;
  shot noise L^3 sum(w^2)/sum(w)^2, aliased by prod (1 - 2/3 sin^2(a));
  corrected power (raw, or L^3|delta|^2 - aliased shot noise) / W^2;
  half-spectrum multiplicity 1 for kz = 0 and the Nyquist plane, else 2;
* logarithmic bins from k_f = 2 pi / L to k_max
  (detail::PositiveLogBinGrid,
  include/cosmo_nbody/analysis/spectral_numeric.hpp:96-143), the last
  bin closed; per bin the multiplicity-weighted means of k, raw power,
  corrected power and the deconvolution factor, and the mode count.

The deposit is the oracle's C restatement (oracle/pm_oracle.c). Sums are
accumulated in long double like the reference's; the reference's
scale-safe exponent handling is not needed at these magnitudes.
"""
from __future__ import annotations

import math

import numpy as np


def _wrap(x, L):
    x = np.asarray(x, dtype=np.float64)
    inside = (x >= 0.0) & (x < L)
    w = np.fmod(x, L)
    w = np.where(w < 0.0, w + L, w)
    w = np.where(w >= L, 0.0, w)
    return np.where(inside, x, w)


def log_edges(k_min, k_max, num_bins):
    """PositiveLogBinGrid edges via stable_positive_log_interpolate."""
    edges = []
    rel = (k_max - k_min) / k_min
    span = math.log1p(rel) if math.isfinite(rel) else math.log(k_max) - math.log(k_min)
    for i in range(num_bins + 1):
        f = float(i) / float(num_bins)
        if f == 0.0:
            e = k_min
        elif f == 1.0:
            e = k_max
        elif span <= 1.0:
            e = k_min * math.exp(f * span)
        else:
            e = float(np.exp(np.longdouble(math.log(k_min)) + np.longdouble(f) * np.longdouble(span)))
        edges.append(e)
    return np.array(edges)


def _modes(oracle, L, N, x, y, z, weights):
    """FourierDensityBuilder::build's build_one: r2c of the contrast / N^3."""
    if weights is None:
        dens = oracle.deposit(L, N, x, y, z, uniform_mass=1.0)
        total = float(x.size)
    else:
        dens = oracle.deposit(L, N, x, y, z, masses=weights)
        total = float(np.sum(weights.astype(np.longdouble)))
    mean = total / float(N ** 3)
    contrast = (dens / mean - 1.0).reshape(N, N, N)
    return np.fft.rfftn(contrast) * (1.0 / float(N ** 3))


def power_spectrum(oracle, L, N, x, y, z, masses=None, num_bins=16, subtract_shot_noise=False,
                   interlaced=False, max_k_fraction_nyquist=1.0):
    x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
    if masses is None:
        weights = None
        msf = 1.0 / float(x.size)
    else:
        m = np.ascontiguousarray(masses, dtype=np.float64)
        weights = m / np.max(m)
        ws = np.sum(weights.astype(np.longdouble))
        msf = float(np.sum(weights.astype(np.longdouble) ** 2) / (ws * ws))
    modes = _modes(oracle, L, N, x, y, z, weights)
    dx = L / N
    k1 = 2.0 * np.pi * np.where(np.arange(N) <= N // 2, np.arange(N), np.arange(N) - N) / L
    kz1 = k1[: N // 2 + 1]
    if interlaced:
        s = 0.5 * dx
        shifted = _modes(oracle, L, N, _wrap(x - s, L), _wrap(y - s, L), _wrap(z - s, L), weights)
        phase = -(k1[:, None, None] + k1[None, :, None] + kz1[None, None, :]) * s
        modes = 0.5 * (modes + shifted * (np.cos(phase) + 1j * np.sin(phase)))
    modes[0, 0, 0] = 0.0
    k_nyq = np.pi * N / L
    k_max = max_k_fraction_nyquist * k_nyq
    edges = log_edges(2.0 * np.pi / L, k_max, num_bins)
    KX, KY, KZ = np.meshgrid(k1, k1, kz1, indexing="ij")
    kmag = np.hypot(np.hypot(KX, KY), KZ)
    sel = (kmag > 0.0) & (kmag <= k_max)
    L3 = L ** 3
    p_raw = L3 * (modes.real ** 2 + modes.imag ** 2)

    def window_axis(k):
        a = np.longdouble(0.5) * k.astype(np.longdouble) * np.longdouble(dx)
        with np.errstate(invalid="ignore", divide="ignore"):
            s = np.where(a == 0, np.longdouble(1.0), np.sin(a) / a)
        s = np.minimum(np.longdouble(1.0), np.abs(s))
        return s * s

    window = window_axis(KX) * window_axis(KY) * window_axis(KZ)
    deconv = (np.longdouble(1.0) / (window * window)).astype(np.float64)
    shot = L3 * msf
    sin2 = [np.sin(0.5 * K * dx) ** 2 for K in (KX, KY, KZ)]
    aliased = shot * (1.0 - 2.0 / 3.0 * sin2[0]) * (1.0 - 2.0 / 3.0 * sin2[1]) \
        * (1.0 - 2.0 / 3.0 * sin2[2])
    p_corr = (p_raw - aliased if subtract_shot_noise else p_raw) * deconv
    iz = np.arange(N // 2 + 1)[None, None, :]
    mult = np.where((iz == 0) | ((N % 2 == 0) & (iz == N // 2)), 1, 2) * np.ones_like(kmag)
    b = np.searchsorted(edges, kmag, side="right") - 1
    b = np.where(kmag == edges[-1], num_bins - 1, b)
    sel &= (b >= 0) & (b < num_bins)
    out = {k: np.zeros(num_bins) for k in ("k_mean", "p_raw", "p_corrected",
                                           "mean_cic_power_deconvolution_factor")}
    out["mode_count"] = np.zeros(num_bins, dtype=np.uint64)
    bs, ms = b[sel], mult[sel].astype(np.longdouble)
    for name, v in (("k_mean", kmag), ("p_raw", p_raw), ("p_corrected", p_corr),
                    ("mean_cic_power_deconvolution_factor", deconv)):
        acc = np.zeros(num_bins, dtype=np.longdouble)
        np.add.at(acc, bs, v[sel].astype(np.longdouble) * ms)
        out[name] = acc
    cnt = np.zeros(num_bins, dtype=np.int64)
    np.add.at(cnt, bs, mult[sel].astype(np.int64))
    for name in ("k_mean", "p_raw", "p_corrected", "mean_cic_power_deconvolution_factor"):
        with np.errstate(invalid="ignore", divide="ignore"):
            out[name] = np.where(cnt > 0, (out[name] / np.maximum(cnt, 1)).astype(np.float64), 0.0)
    out["mode_count"] = cnt.astype(np.uint64)
    out["k_low"] = edges[:-1].copy()
    out["k_high"] = edges[1:].copy()
    out["shot_noise_reference"] = np.full(num_bins, shot)
    return out
