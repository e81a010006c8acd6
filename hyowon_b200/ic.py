"""Synthetic initial conditions for the benchmark configurations.

Seeded unit-Gaussian white noise per lattice cell, shaped by a tabulated
linear spectrum P(k) = A k^n_s T_BBKS(k; Gamma)^2 normalised to sigma_8, then
mapped by first-order LPT (Zel'dovich) on the corner lattice q = i L / N:

* spectrum table: 512 log-spaced k in [1e-4, 1e2] h/Mpc, interpolated by a
  natural cubic spline in (ln k, ln P) -- the reference's LinearPowerSpectrum
  contract (src/ic/linear_power_spectrum.cpp:649-664), back-scaled by
  D1(a_start)^2;
* Fourier amplitude of each white-noise mode scaled by sqrt(P(k) N^3 / L^3),
  the variance normalisation of src/ic/random_field.cpp:119-129 applied to
  noise of unit variance per cell;
* 1LPT: psi_k = i k_d delta_k / k^2 with the Nyquist component of k_d zeroed,
  x = wrap(q + psi), p = a^2 H f1 psi (src/ic/lpt_displacement.cpp:101-128,
  201-233, 330-356); lattice and particle order (i N + j) N + k as in
  src/ic/initial_conditions.cpp:295-313.

The map itself runs on the device (hyowon_pm_lpt_ics); this module prepares
its inputs (noise, spectrum spline, growth factors).
"""
from __future__ import annotations

import math

import numpy as np

from .pm import CosmologyModel

G_INTERNAL = 6.67430e-11 * (1e10 * 1.98847e30) / (3.085677581491367e22 * 1000.0 * 1000.0)
RHO_CRIT0 = 3.0 * 100.0 * 100.0 / (8.0 * math.pi * G_INTERNAL)  # units.hpp:27


def particle_mass(box_size: float, n_side: int, omega_m: float = 0.3) -> float:
    """rho_crit0 * Omega_m * (L/N)^3 (src/config/simulation_parameters.cpp:403-416)."""
    return RHO_CRIT0 * omega_m * (box_size / n_side) ** 3


def bbks_transfer(k, gamma=0.21):
    q = np.asarray(k, dtype=np.float64) / gamma
    return (np.log1p(2.34 * q) / (2.34 * q)
            * (1.0 + 3.89 * q + (16.1 * q) ** 2 + (5.46 * q) ** 3 + (6.71 * q) ** 4) ** -0.25)


def _tophat(x):
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    small = x < 1e-3
    xs = x[small]
    out[small] = 1.0 - xs * xs / 10.0
    xl = x[~small]
    out[~small] = 3.0 * (np.sin(xl) - xl * np.cos(xl)) / xl ** 3
    return out


def bbks_table(n=512, kmin=1e-4, kmax=1e2, sigma8=0.8, n_s=0.965, gamma=0.21, R=8.0):
    """(k, P(k)) at z = 0, normalised to sigma_8 with a top-hat of radius R."""
    k = np.exp(np.linspace(math.log(kmin), math.log(kmax), n))
    lk = np.linspace(math.log(1e-6), math.log(1e3), 200001)
    kk = np.exp(lk)
    shape = kk ** n_s * bbks_transfer(kk, gamma) ** 2
    integrand = kk ** 3 * shape * _tophat(kk * R) ** 2 / (2.0 * math.pi ** 2)
    s2 = np.trapezoid(integrand, lk)
    A = sigma8 ** 2 / s2
    return k, A * k ** n_s * bbks_transfer(k, gamma) ** 2


class NaturalCubicSpline:
    """Natural cubic spline y(x) through (x_i, y_i)."""

    def __init__(self, x, y):
        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        n = x.size
        h = np.diff(x)
        a = np.zeros(n)
        b = np.ones(n)
        c = np.zeros(n)
        d = np.zeros(n)
        a[1:-1] = h[:-1] / 6.0
        b[1:-1] = (h[:-1] + h[1:]) / 3.0
        c[1:-1] = h[1:] / 6.0
        d[1:-1] = (y[2:] - y[1:-1]) / h[1:] - (y[1:-1] - y[:-2]) / h[:-1]
        # Thomas algorithm, natural ends y2[0] = y2[-1] = 0.
        cp = np.zeros(n)
        dp = np.zeros(n)
        cp[0] = c[0] / b[0]
        dp[0] = d[0] / b[0]
        for i in range(1, n):
            m = b[i] - a[i] * cp[i - 1]
            cp[i] = c[i] / m
            dp[i] = (d[i] - a[i] * dp[i - 1]) / m
        y2 = np.zeros(n)
        y2[-1] = dp[-1]
        for i in range(n - 2, -1, -1):
            y2[i] = dp[i] - cp[i] * y2[i + 1]
        self.x, self.y, self.y2 = x, y, y2

    def __call__(self, xq):
        xq = np.asarray(xq, dtype=np.float64)
        x, y, y2 = self.x, self.y, self.y2
        i = np.clip(np.searchsorted(x, xq) - 1, 0, x.size - 2)
        h = x[i + 1] - x[i]
        A = (x[i + 1] - xq) / h
        B = (xq - x[i]) / h
        return (A * y[i] + B * y[i + 1]
                + ((A ** 3 - A) * y2[i] + (B ** 3 - B) * y2[i + 1]) * h * h / 6.0)


class LinearSpectrum:
    """Tabulated z=0 spectrum evaluated by a log-log natural cubic spline."""

    def __init__(self, k=None, P=None):
        if k is None:
            k, P = bbks_table()
        self.k = np.asarray(k, dtype=np.float64)
        self.P = np.asarray(P, dtype=np.float64)
        self.spline = NaturalCubicSpline(np.log(self.k), np.log(self.P))

    def __call__(self, k):
        k = np.asarray(k, dtype=np.float64)
        out = np.zeros_like(k)
        pos = k > 0
        out[pos] = np.exp(self.spline(np.log(k[pos])))
        return out


def white_noise(n_side: int, seed: int) -> np.ndarray:
    """Seeded N(0,1) per lattice cell, row-major (i N + j) N + k."""
    return np.random.default_rng(seed).standard_normal(n_side ** 3)


def mode_k2(n: int, box: float):
    m = np.fft.fftfreq(n, d=1.0 / n)
    kf = 2.0 * math.pi / box
    kx = (kf * m)[:, None, None]
    ky = (kf * m)[None, :, None]
    kz = (kf * np.arange(n // 2 + 1))[None, None, :]
    return kx, ky, kz


def lpt_table(a_start: float, spectrum: "LinearSpectrum" = None, model: CosmologyModel = None):
    """Spline table of ln P(k, a_start) = ln P_0(k) + 2 ln D1(a_start) and the
    1LPT momentum factor a^2 H f1, for hyowon_pm_lpt_ics."""
    spectrum = spectrum or LinearSpectrum()
    model = model or CosmologyModel()
    D1, f1 = model.growth(a_start)
    H = model.H(a_start)[0]
    sp = spectrum.spline
    ln_p = sp.y + 2.0 * math.log(float(D1[0]))
    return (np.ascontiguousarray(sp.x), np.ascontiguousarray(ln_p),
            np.ascontiguousarray(sp.y2), a_start * a_start * H * float(f1[0]))


def lpt_on_device(solver, noise, n_side: int, a_start: float, particle_mass_value: float,
                  spectrum: "LinearSpectrum" = None, model: CosmologyModel = None):
    """Generates the 1LPT state on the device of `solver` (hyowon_pm_lpt_ics)."""
    from . import _native as nat
    ln_k, ln_p, y2, pf = lpt_table(a_start, spectrum, model)
    noise = np.ascontiguousarray(noise, dtype=np.float64)
    if noise.size != n_side ** 3:
        raise ValueError("noise must hold n_side^3 values")
    rc = nat.lib().hyowon_pm_lpt_ics(solver.handle, n_side, nat.dptr(noise), ln_k.size,
                                     nat.dptr(ln_k), nat.dptr(ln_p), nat.dptr(y2), pf,
                                     particle_mass_value)
    nat.raise_for(rc, solver.handle, "lpt_ics")


# The five benchmark configurations (flat LCDM Om=0.3, OL=0.7, h=0.7).
CONFIGS = {
    "c1": dict(n_side=32, box=100.0, mesh=64, z_start=49.0, steps=32, seed=1),
    "c2": dict(n_side=128, box=256.0, mesh=256, z_start=49.0, steps=64, seed=1),
    "c3": dict(n_side=512, box=1000.0, mesh=1024, z_start=49.0, steps=64, seed=7),
    "c4": dict(n_side=128, box=256.0, mesh=128, z_start=19.0, steps=16, seed=3),
    # c3 at half the side length: same cell size and particle density, 1/8 of
    # the volume (meshes still far larger than L2); the size profiling
    # captures of the step kernels use
    "c3h": dict(n_side=256, box=500.0, mesh=512, z_start=49.0, steps=64, seed=7),
}


def config_schedule(name: str):
    c = CONFIGS[name]
    a_start = 1.0 / (1.0 + c["z_start"])
    return a_start, math.log(1.0 / a_start) / c["steps"]


# --------------------------------------------------------------------------
# Generated initial conditions (include/hyowon_ic.h): HYOWON's own generator,
# the Philox per-mode Fourier field and 1LPT / projected 2LPT, on the device.
# --------------------------------------------------------------------------
_AMPLITUDE = {"gaussian": 0, "fixed": 1}
_PAIRING = {"independent": 0, "pair_a": 1, "pair_b": 2}


class ICParams:
    """The ic.* coordinates of SimulationParameters in generate mode
    (include/cosmo_nbody/config/simulation_parameters.hpp:59-82) plus the
    start-epoch LPT factors (src/ic/lpt_displacement.cpp:197-222)."""

    def __init__(self, particles_per_dimension: int, box_size: float, seed: int,
                 a_start: float, lpt_order: int = 1, mesh_per_dimension: int = 0,
                 max_mode_per_axis: int = None, amplitude_mode: str = "gaussian",
                 phase_pairing: str = "independent", model: CosmologyModel = None,
                 factors=None):
        if amplitude_mode not in _AMPLITUDE:
            raise ValueError("ic.amplitude_mode must be 'gaussian' or 'fixed'")
        if phase_pairing not in _PAIRING:
            raise ValueError("ic.phase_pairing must be 'independent', 'pair_a', or 'pair_b'")
        self.particles_per_dimension = int(particles_per_dimension)
        self.box_size = float(box_size)
        self.seed = int(seed)
        self.a_start = float(a_start)
        self.lpt_order = int(lpt_order)
        self.mesh_per_dimension = int(mesh_per_dimension)
        self.max_mode_per_axis = max_mode_per_axis
        self.amplitude_mode = amplitude_mode
        self.phase_pairing = phase_pairing
        self.factors = tuple(factors) if factors is not None else lpt_factors(a_start, model)

    def to_c(self):
        from . import _native as nat
        p1, x2, p2 = self.factors
        return nat.ICParams(self.particles_per_dimension, self.mesh_per_dimension, self.box_size,
                            self.seed, -1 if self.max_mode_per_axis is None
                            else int(self.max_mode_per_axis), _AMPLITUDE[self.amplitude_mode],
                            _PAIRING[self.phase_pairing], self.lpt_order, p1, x2, p2)

    def resolve(self):
        """(M, K): the IC mesh and Cartesian support (hyowon_ic_resolve)."""
        import ctypes
        from . import _native as nat
        c = self.to_c()
        M, K = ctypes.c_uint64(0), ctypes.c_uint64(0)
        _ic_check(nat.lib().hyowon_ic_resolve(ctypes.byref(c), ctypes.byref(M), ctypes.byref(K)),
                  "resolve")
        return int(M.value), int(K.value)


def _ic_check(rc, where):
    from . import _native as nat
    if rc != nat.OK:
        msg = nat.lib().hyowon_ic_last_error().decode(errors="replace")
        raise nat._EXC.get(rc, RuntimeError)(f"{where}: {msg}")


def lpt_factors(a_start: float, model: CosmologyModel = None):
    """(a^2 H f1, D2/D1^2, a^2 H f2 D2/D1^2) at a_start, formed as
    apply_to_arrays forms them (src/ic/lpt_displacement.cpp:197-222)."""
    model = model or CosmologyModel()
    D1, f1, D2, f2 = (float(v[0]) for v in model.growth2(a_start))
    H = float(model.H(a_start)[0])
    p1 = a_start * a_start * H * f1
    x2 = D2 / (D1 * D1)
    p2 = a_start * a_start * H * f2 * x2
    return p1, x2, p2


def represented_wavenumbers(box_size: float, max_mode: int):
    """k_s = double(sqrt((long double) s)) * (2 pi / L) for s = 0 .. 3K^2
    (include/cosmo_nbody/ic/particle_lattice_bandlimit.hpp:27-37)."""
    s = np.arange(3 * max_mode * max_mode + 1, dtype=np.longdouble)
    return np.sqrt(s).astype(np.float64) * (2.0 * math.pi / box_size)


def start_spectrum(a_start: float, spectrum: "LinearSpectrum" = None,
                   model: CosmologyModel = None, table_a: float = 1.0) -> "LinearSpectrum":
    """LinearPowerSpectrum(config): the table rescaled by (D1(a_start) /
    D1(table_a))^2 before the log-log spline (src/ic/linear_power_spectrum.cpp:451-488)."""
    spectrum = spectrum or LinearSpectrum()
    model = model or CosmologyModel()
    D1 = model.growth(np.array([a_start, table_a]))[0]
    scale = (float(D1[0]) / float(D1[1])) ** 2.0
    return LinearSpectrum(spectrum.k, spectrum.P * scale)


def power_table(params: ICParams, spectrum: "LinearSpectrum"):
    """P at the represented wavenumbers of every |m|^2 in the support (the
    `power` argument of include/hyowon_ic.h); spectrum at the start epoch."""
    _, K = params.resolve()
    k = represented_wavenumbers(params.box_size, K)
    out = np.zeros_like(k)
    out[1:] = spectrum(k[1:])
    return out


def mode_amplitudes(mesh: int, box_size: float, power):
    """{sqrt(var_s), sqrt(var_s/2)} per s (hyowon_ic_mode_amplitudes; host only)."""
    from . import _native as nat
    power = np.ascontiguousarray(power, dtype=np.float64)
    amp = np.zeros((power.size, 2))
    _ic_check(nat.lib().hyowon_ic_mode_amplitudes(mesh, box_size, power.size, nat.dptr(power),
                                                  nat.dptr(amp)), "mode_amplitudes")
    return amp


class RandomField:
    """RandomField::generate (src/ic/random_field.cpp:70-330) on the device."""

    @staticmethod
    def generate(params: ICParams, power) -> np.ndarray:
        import ctypes
        from . import _native as nat
        M, _ = params.resolve()
        power = np.ascontiguousarray(power, dtype=np.float64)
        out = np.zeros((M, M, M // 2 + 1), dtype=np.complex128)
        c = params.to_c()
        _ic_check(nat.lib().hyowon_ic_field(ctypes.byref(c), power.size, nat.dptr(power),
                                            out.ctypes.data_as(nat.P_double)), "RandomField")
        return out


def generate_ics(params: ICParams, power) -> dict:
    """The generate branch of InitialConditions on the device
    (hyowon_ic_generate): {x, y, z, px, py, pz} in particle order."""
    import ctypes
    from . import _native as nat
    n = params.particles_per_dimension ** 3
    st = {k: np.zeros(n) for k in ("x", "y", "z", "px", "py", "pz")}
    power = np.ascontiguousarray(power, dtype=np.float64)
    c = params.to_c()
    _ic_check(nat.lib().hyowon_ic_generate(ctypes.byref(c), power.size, nat.dptr(power),
                                           *[nat.dptr(st[k]) for k in
                                             ("x", "y", "z", "px", "py", "pz")]),
              "generate_ics")
    return st
