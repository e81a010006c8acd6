"""Python mirror of HYOWON's PM solver / leapfrog interface over the C ABI.

Names and argument meaning follow the reference C++ classes so that code (and
tests) written against the reference read the same:

* ``MeshGeometry(box_size, n_mesh)``  -- include/cosmo_nbody/mesh/mesh_geometry.hpp:18-62
* ``PMForceMethod.pure_pm(deconvolve_cic)`` / ``.treepm_long_range(split_scale)``
  -- include/cosmo_nbody/mesh/pm_force_method.hpp:16-67
* ``PMSolver(geom, method).compute_forces(pos_x, pos_y, pos_z, masses,
  uniform_mass, acc_x, acc_y, acc_z)`` ADDS the PM acceleration
  -- include/cosmo_nbody/gravity/pm_solver.hpp:52-68
* ``LeapfrogIntegrator`` -- include/cosmo_nbody/time/leapfrog_integrator.hpp:14-60,
  with the particle state resident on the device between steps.
* ``CosmologyModel``, ``DriftKickIntegrator``, ``TimeStepper`` -- host scalars.

Errors map onto the exception types the reference throws for the same
condition (ValueError ~ std::invalid_argument, OverflowError ~
std::overflow_error, HyowonLogicError ~ std::logic_error, ...).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _native as nat

FP64 = 0
FP32_FIXED = 1
_PRECISIONS = {"fp64": FP64, "fp32": FP32_FIXED, "fp32_fixed": FP32_FIXED}


@dataclass(frozen=True)
class MeshGeometry:
    box_size: float
    n_mesh: int

    def __post_init__(self):
        if not math.isfinite(self.box_size) or self.box_size <= 0.0:
            raise ValueError("MeshGeometry box size must be finite and positive")
        if self.n_mesh <= 0:
            raise ValueError("MeshGeometry grid size must be positive")

    @property
    def cell_size(self) -> float:
        return self.box_size / float(self.n_mesh)


@dataclass(frozen=True)
class PMForceMethod:
    kind: int  # 0 pure PM, 1 TreePM long range
    split_scale: float = 0.0
    deconvolve_cic: bool = False

    @staticmethod
    def pure_pm(deconvolve_cic: bool) -> "PMForceMethod":
        return PMForceMethod(0, 0.0, bool(deconvolve_cic))

    @staticmethod
    def treepm_long_range(split_scale: float) -> "PMForceMethod":
        if not math.isfinite(split_scale) or split_scale <= 0.0:
            raise ValueError("TreePM long-range PM method requires a finite positive split scale")
        return PMForceMethod(1, float(split_scale), True)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class PMSolver:
    """Device PM solver; one handle = one CUDA stream + device meshes + state."""

    def __init__(self, geom: MeshGeometry, method: PMForceMethod, precision: str = "fp64"):
        self.geom = geom
        self.method = method
        self.precision = _PRECISIONS[precision]
        h = ctypes.c_void_p()
        rc = nat.lib().hyowon_pm_create(geom.box_size, geom.n_mesh, method.kind,
                                        int(method.deconvolve_cic), method.split_scale,
                                        self.precision, ctypes.byref(h))
        if rc != nat.OK:
            raise nat._EXC.get(rc, RuntimeError)(
                f"hyowon_pm_create failed (status {rc}) for N={geom.n_mesh}")
        self._h = h

    # -- lifetime ----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            nat.lib().hyowon_pm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc, where):
        nat.raise_for(rc, self._h, where)

    # -- PMSolver::compute_forces ------------------------------------------
    def compute_forces(self, pos_x, pos_y, pos_z, masses, uniform_mass, acc_x, acc_y, acc_z,
                       collect_potential_energy=False):
        """Adds the PM acceleration at the given positions to acc_* (in place).

        With collect_potential_energy, returns the reference's PMForceDiagnostics
        as a dict {"potential_energy_comoving": 0.5 sum_i m_i phi(x_i)}
        (src/gravity/pm_solver.cpp:812-840); otherwise None."""
        n = len(pos_x)
        if not (len(pos_y) == len(pos_z) == len(acc_x) == len(acc_y) == len(acc_z) == n):
            raise ValueError("PMSolver position and acceleration component sizes must match")
        if uniform_mass is not None:
            if masses is not None and len(masses) != 0:
                raise ValueError("PMSolver uniform mass mode requires an empty explicit mass span")
            if not math.isfinite(uniform_mass) or uniform_mass <= 0.0:
                raise ValueError("PMSolver uniform mass must be finite and positive")
        elif masses is None or len(masses) != n:
            raise ValueError("PMSolver explicit mass count must match particle count")
        for a in (acc_x, acc_y, acc_z):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]):
                raise ValueError("acceleration outputs must be C-contiguous float64 arrays")
        x, y, z = _f64(pos_x), _f64(pos_y), _f64(pos_z)
        m = None if uniform_mass is not None else _f64(masses)
        rc = nat.lib().hyowon_pm_forces_host(self._h, n, nat.dptr(x), nat.dptr(y), nat.dptr(z),
                                             nat.dptr(m), float(uniform_mass or 0.0),
                                             nat.dptr(acc_x), nat.dptr(acc_y), nat.dptr(acc_z))
        self._check(rc, "PMSolver.compute_forces")
        if collect_potential_energy:
            return {"potential_energy_comoving": self.diagnostics(1.0)["potential_energy_comoving"]}
        return None

    # -- device-resident state --------------------------------------------
    def upload(self, x, y, z, px=None, py=None, pz=None, masses=None, uniform_mass=None):
        x, y, z = _f64(x), _f64(y), _f64(z)
        px = None if px is None else _f64(px)
        py = None if py is None else _f64(py)
        pz = None if pz is None else _f64(pz)
        m = None if masses is None else _f64(masses)
        rc = nat.lib().hyowon_pm_upload(self._h, x.size, nat.dptr(x), nat.dptr(y), nat.dptr(z),
                                        nat.dptr(px), nat.dptr(py), nat.dptr(pz), nat.dptr(m),
                                        float(uniform_mass or 0.0))
        self._check(rc, "upload")

    def info(self):
        n = ctypes.c_uint64()
        N = ctypes.c_uint64()
        p = ctypes.c_int()
        mth = ctypes.c_int()
        self._check(nat.lib().hyowon_pm_info(self._h, ctypes.byref(n), ctypes.byref(N),
                                             ctypes.byref(p), ctypes.byref(mth)), "info")
        return n.value, N.value, p.value, mth.value

    def download(self, acc=True, out=None):
        """Particle state in the original particle order. With `out` (a dict of
        C-contiguous float64 arrays of the particle count, e.g. pinned host
        buffers), only the components it names are copied, into those arrays."""
        n = self.info()[0]
        if out is None:
            out = {k: np.empty(n) for k in ("x", "y", "z", "px", "py", "pz")}
            if acc:
                out.update({k: np.empty(n) for k in ("ax", "ay", "az")})
        else:
            for k, a in out.items():
                if k not in ("x", "y", "z", "px", "py", "pz", "ax", "ay", "az"):
                    raise ValueError(f"unknown particle component {k!r}")
                if not (isinstance(a, np.ndarray) and a.dtype == np.float64
                        and a.flags["C_CONTIGUOUS"] and a.size == n):
                    raise ValueError("download outputs must be C-contiguous float64 arrays "
                                     "of the particle count")
        g = out.get
        rc = nat.lib().hyowon_pm_download(
            self._h, nat.dptr(g("x")), nat.dptr(g("y")), nat.dptr(g("z")), nat.dptr(g("px")),
            nat.dptr(g("py")), nat.dptr(g("pz")), nat.dptr(g("ax")), nat.dptr(g("ay")),
            nat.dptr(g("az")))
        self._check(rc, "download")
        return out

    def snapshot_payload(self, a: float, coordinates=True, velocities=True):
        """The /PartType1 Coordinates and Velocities datasets as (n, 3) arrays
        in the original particle order, velocities p / a
        (hyowon_pm_snapshot_payload); validated on the device first."""
        n = self.info()[0]
        c = np.empty((n, 3)) if coordinates else None
        v = np.empty((n, 3)) if velocities else None
        self._check(nat.lib().hyowon_pm_snapshot_payload(
            self._h, float(a), None if c is None else c.ctypes.data_as(nat.P_double),
            None if v is None else v.ctypes.data_as(nat.P_double)), "snapshot_payload")
        return c, v

    def solve_forces(self):
        """Force solve at the device positions (accelerations become valid)."""
        self._check(nat.lib().hyowon_pm_compute_forces(self._h, None, None, None), "solve_forces")

    def kdk_step(self, K1, D, K2) -> float:
        md = ctypes.c_double(0.0)
        self._check(nat.lib().hyowon_pm_kdk_step(self._h, K1, D, K2, ctypes.byref(md)),
                    "kdk_step")
        return md.value

    def run(self, K1, D, K2):
        K1, D, K2 = _f64(K1), _f64(D), _f64(K2)
        md = np.zeros(K1.size)
        self._check(nat.lib().hyowon_pm_run(self._h, K1.size, nat.dptr(K1), nat.dptr(D),
                                            nat.dptr(K2), nat.dptr(md)), "run")
        return md

    def generate_ics(self, params, power, uniform_mass: float):
        """Generated initial conditions straight into the device state
        (hyowon_pm_generate_ics): params is an ic.ICParams, power the table
        of ic.power_table."""
        c = params.to_c()
        power = _f64(power)
        self._check(nat.lib().hyowon_pm_generate_ics(self._h, ctypes.byref(c), power.size,
                                                     nat.dptr(power), float(uniform_mass)),
                    "generate_ics")

    def potential(self):
        N = self.geom.n_mesh
        phi = np.empty(N ** 3)
        self._check(nat.lib().hyowon_pm_download_potential(self._h, nat.dptr(phi)), "potential")
        return phi

    def mass_mesh(self):
        N = self.geom.n_mesh
        m = np.empty(N ** 3)
        self._check(nat.lib().hyowon_pm_download_mass_mesh(self._h, nat.dptr(m)), "mass_mesh")
        return m

    def cell_coords(self):
        n = self.info()[0]
        base = np.empty(3 * n, dtype=np.int64)
        frac = np.empty(3 * n)
        self._check(nat.lib().hyowon_pm_cell_coords(
            self._h, base.ctypes.data_as(nat.P_i64), nat.dptr(frac)), "cell_coords")
        return base.reshape(3, n), frac.reshape(3, n)

    def set_treepm_short_range(self, theta: float, softening: float, cutoff: float):
        """TreePM force method: every solve adds the octree short range (theta,
        Plummer softening, cutoff < L/2) to the long range; cutoff = 0 turns it
        off (hyowon_pm_set_treepm_short_range)."""
        self._check(nat.lib().hyowon_pm_set_treepm_short_range(self._h, theta, softening, cutoff),
                    "set_treepm_short_range")

    def treepm_short_forces(self, theta: float, softening: float, cutoff: float):
        """Short-range accelerations of every particle of the device state in
        original order: (ax, ay, az, stats) (hyowon_pm_treepm_short_forces)."""
        n = self.info()[0]
        out = [np.empty(n) for _ in range(3)]
        stats = np.zeros(6)
        self._check(nat.lib().hyowon_pm_treepm_short_forces(
            self._h, theta, softening, cutoff, *(nat.dptr(o) for o in out), nat.dptr(stats)),
            "treepm_short_forces")
        info = dict(zip(("nodes", "depth", "visits_per_target", "interactions_per_target",
                         "build_ms", "walk_ms"), stats.tolist()))
        return out[0], out[1], out[2], info

    def set_sort_interval(self, steps: int):
        self._check(nat.lib().hyowon_pm_set_sort_interval(self._h, int(steps)), "set_sort_interval")

    def diagnostics(self, a: float) -> dict:
        """Binary64 global sums of the state at the last force solve
        (hyowon_pm_diagnostics): potential_energy_comoving, kinetic_energy
        (sum 0.5 m p^2 / a^2), momentum, mass_weighted_force, force_norm_sum,
        force_balance (|sum m a| / sum m |a|), momentum_force_contraction,
        directional_potential_energy_comoving (sum m p . grad_S phi)."""
        d = nat.Diagnostics()
        self._check(nat.lib().hyowon_pm_diagnostics(self._h, float(a), ctypes.byref(d)),
                    "diagnostics")
        return {"potential_energy_comoving": d.potential_energy_comoving,
                "kinetic_energy": d.kinetic_energy,
                "momentum": np.array(d.momentum[:]),
                "mass_weighted_force": np.array(d.mass_weighted_force[:]),
                "force_norm_sum": d.force_norm_sum, "force_balance": d.force_balance,
                "momentum_force_contraction": d.momentum_force_contraction,
                "directional_potential_energy_comoving":
                    d.directional_potential_energy_comoving}

    def power_spectrum(self, num_bins: int, max_k_fraction_nyquist: float = 1.0,
                       subtract_shot_noise: bool = False, interlaced: bool = False,
                       mesh_size: int = 0) -> dict:
        """MatterPowerSpectrum::compute_pk of the device state
        (hyowon_pm_power_spectrum): per-bin arrays k_low, k_mean, k_high,
        p_raw, p_corrected, mean_cic_power_deconvolution_factor,
        shot_noise_reference, mode_count. mesh_size 0 uses the solver's mesh."""
        bins = (nat.PkBin * int(num_bins))()
        self._check(nat.lib().hyowon_pm_power_spectrum(
            self._h, int(mesh_size), int(num_bins), float(max_k_fraction_nyquist),
            int(bool(subtract_shot_noise)), int(bool(interlaced)), bins), "power_spectrum")
        keys = ("k_low", "k_mean", "k_high", "p_raw", "p_corrected",
                "mean_cic_power_deconvolution_factor", "shot_noise_reference")
        out = {k: np.array([getattr(b, k) for b in bins]) for k in keys}
        out["mode_count"] = np.array([b.mode_count for b in bins], dtype=np.uint64)
        return out

    def set_timing(self, on: bool):
        self._check(nat.lib().hyowon_pm_set_timing(self._h, int(on)), "set_timing")

    def last_timing(self):
        t = np.zeros(9)
        self._check(nat.lib().hyowon_pm_last_timing(self._h, nat.dptr(t)), "last_timing")
        return dict(zip(("total", "sort", "deposit", "fft_forward", "green", "fft_inverse",
                         "gather", "launches", "solves"), t.tolist()))


# --------------------------------------------------------------------------
# Host scalars (include/hyowon_cosmology.h)
# --------------------------------------------------------------------------
class CosmologyModel:
    """Flat matter + Lambda (src/cosmology/cosmology_model.cpp)."""

    def __init__(self, omega_m: float = 0.3, omega_lambda: float = 0.7):
        self.omega_m = float(omega_m)
        self.omega_lambda = float(omega_lambda)

    def H(self, a):
        a = np.atleast_1d(_f64(a))
        out = np.empty_like(a)
        rc = nat.lib().hyowon_hubble(self.omega_m, self.omega_lambda, a.size, nat.dptr(a),
                                     nat.dptr(out))
        nat.raise_for(rc, None, "CosmologyModel.H")
        return out

    def growth(self, a):
        a = np.atleast_1d(_f64(a))
        D1 = np.empty_like(a)
        f1 = np.empty_like(a)
        rc = nat.lib().hyowon_growth(self.omega_m, self.omega_lambda, a.size, nat.dptr(a),
                                     nat.dptr(D1), nat.dptr(f1))
        nat.raise_for(rc, None, "CosmologyModel.growth")
        return D1, f1

    def growth2(self, a):
        """(D1, f1, D2, f2) at a (0 < a <= 1); D2 < 0 normalised by D1(1)^2."""
        a = np.atleast_1d(_f64(a))
        out = [np.empty_like(a) for _ in range(4)]
        rc = nat.lib().hyowon_growth2(self.omega_m, self.omega_lambda, a.size, nat.dptr(a),
                                      *[nat.dptr(o) for o in out])
        nat.raise_for(rc, None, "CosmologyModel.growth2")
        return tuple(out)


class DriftKickIntegrator:
    """D = int da/(a^3 H), K = int da/(a^2 H) (src/cosmology/drift_kick_factors.cpp)."""

    def __init__(self, model: CosmologyModel):
        self.model = model

    def drift_factor(self, a1, a2) -> float:
        out = ctypes.c_double()
        rc = nat.lib().hyowon_drift_factor(self.model.omega_m, self.model.omega_lambda, a1, a2,
                                           ctypes.byref(out))
        nat.raise_for(rc, None, "drift_factor")
        return out.value

    def kick_factor(self, a1, a2) -> float:
        out = ctypes.c_double()
        rc = nat.lib().hyowon_kick_factor(self.model.omega_m, self.model.omega_lambda, a1, a2,
                                          ctypes.byref(out))
        nat.raise_for(rc, None, "kick_factor")
        return out.value


@dataclass(frozen=True)
class TimeStep:
    a_begin: float
    a_half: float
    a_end: float
    D: float
    K1: float
    K2: float


class TimeStepper:
    """Steps uniform in ln a with an exact final stop (src/time/time_stepper.cpp)."""

    def __init__(self, a_start, a_final, delta_ln_a, model: Optional[CosmologyModel] = None,
                 max_steps: int = 1 << 20):
        model = model or CosmologyModel()
        out = np.zeros(6 * max_steps)
        n = ctypes.c_uint64()
        rc = nat.lib().hyowon_schedule(model.omega_m, model.omega_lambda, a_start, a_final,
                                       delta_ln_a, max_steps, nat.dptr(out), ctypes.byref(n))
        nat.raise_for(rc, None, "TimeStepper")
        self.table = out[: 6 * n.value].reshape(n.value, 6).copy()
        self.steps = [TimeStep(*row) for row in self.table]

    def num_steps(self) -> int:
        return len(self.steps)

    def factors(self):
        """(K1, D, K2) arrays for LeapfrogIntegrator.run."""
        t = self.table
        return t[:, 4].copy(), t[:, 3].copy(), t[:, 5].copy()


class LeapfrogIntegrator:
    """KDK driver over a device-resident particle state
    (src/time/leapfrog_integrator.cpp:143-279)."""

    def __init__(self, solver: PMSolver, model: Optional[CosmologyModel] = None):
        self.solver = solver
        self.factors = DriftKickIntegrator(model or CosmologyModel())
        self.last_step_max_drift_displacement = None

    def step(self, step: TimeStep):
        self.last_step_max_drift_displacement = self.solver.kdk_step(step.K1, step.D, step.K2)

    def run(self, stepper: TimeStepper):
        K1, D, K2 = stepper.factors()
        md = self.solver.run(K1, D, K2)
        if md.size:
            self.last_step_max_drift_displacement = float(md[-1])
        return md
