"""ctypes bindings for the CPU checker libraries (TEST INFRASTRUCTURE ONLY).

* ``Oracle`` wraps ``oracle/liboracle.so`` -- this repository's C restatement of
  HYOWON's PM hot path (oracle/pm_oracle.c).
* ``Reference`` wraps ``oracle/_ref/libhyowon_ref.so`` -- the reference's own
  sources compiled unmodified (oracle/ref/Makefile) behind a small harness.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, as the checker. The product library never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhyowon_ref.so")

_c_double = ctypes.c_double
_c_u64 = ctypes.c_uint64
_c_int = ctypes.c_int


def _dp(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def reference_root(ref_root: str | None = None) -> str:
    """The reference source tree: the argument, else $HYOWON_REF_ROOT, else
    the REF_ROOT default of oracle/ref/Makefile (the recipe that reads it)."""
    if ref_root:
        return ref_root
    env = os.environ.get("HYOWON_REF_ROOT")
    if env:
        return env
    with open(os.path.join(HERE, "ref", "Makefile")) as f:
        for line in f:
            if line.startswith("REF_ROOT") and "?=" in line:
                return line.split("?=", 1)[1].strip()
    return ""


def build_reference(ref_root: str | None = None) -> bool:
    """Compile the reference's hot path into oracle/_ref when its tree exists."""
    root = reference_root(ref_root)
    if not root or not os.path.isdir(root):
        return os.path.exists(REF_SO)
    jobs = str(max(1, min(16, os.cpu_count() or 1)))
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", os.path.join(HERE, "ref"),
                    f"REF_ROOT={root}"], check=True)
    return True


class OracleError(RuntimeError):
    def __init__(self, code: int, where: str, message: str = ""):
        super().__init__(f"{where}: status {code} {message}".strip())
        self.code = code


class Oracle:
    """The C restatement (oracle/pm_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build_oracle()
        self.lib = ctypes.CDLL(path)
        self.lib.orc_gravitational_constant.restype = ctypes.c_double
        self.lib.orc_wrap.restype = ctypes.c_double
        self.lib.orc_wrap.argtypes = [_c_double, _c_double]
        self.lib.orc_minimum_image.restype = ctypes.c_double
        self.lib.orc_minimum_image.argtypes = [_c_double, _c_double]

    def _check(self, rc, where):
        if rc != 0:
            raise OracleError(rc, where)

    def G(self) -> float:
        return self.lib.orc_gravitational_constant()

    def cic_coords(self, L, N, pos):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        base = np.zeros(pos.size, dtype=np.int64)
        frac = np.zeros(pos.size, dtype=np.float64)
        rc = self.lib.orc_cic_coords(_c_double(L), _c_u64(N), _c_u64(pos.size), _dp(pos),
                                     _ip(base, ctypes.c_int64), _dp(frac))
        self._check(rc, "orc_cic_coords")
        return base, frac

    def x_plane_bins(self, L, N, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        offsets = np.zeros(N + 1, dtype=np.uint64)
        order = np.zeros(x.size, dtype=np.uint32)
        rc = self.lib.orc_x_plane_bins(_c_double(L), _c_u64(N), _c_u64(x.size), _dp(x),
                                       _ip(offsets, ctypes.c_uint64), _ip(order, ctypes.c_uint32))
        self._check(rc, "orc_x_plane_bins")
        return offsets, order

    def deposit(self, L, N, x, y, z, masses=None, uniform_mass=1.0):
        mesh = np.zeros(N * N * N, dtype=np.float64)
        rc = self.lib.orc_deposit(_c_double(L), _c_u64(N), _c_u64(x.size), _dp(x), _dp(y),
                                  _dp(z), _dp(masses), _c_double(uniform_mass), _dp(mesh))
        self._check(rc, "orc_deposit")
        return mesh

    def potential(self, L, N, x, y, z, masses=None, uniform_mass=1.0, deconvolve=False):
        dens = np.zeros(N * N * N, dtype=np.float64)
        phi = np.zeros(N * N * N, dtype=np.float64)
        rc = self.lib.orc_potential(_c_double(L), _c_u64(N), _c_int(int(deconvolve)),
                                    _c_u64(x.size), _dp(x), _dp(y), _dp(z), _dp(masses),
                                    _c_double(uniform_mass), _dp(dens), _dp(phi))
        self._check(rc, "orc_potential")
        return dens, phi

    def gradient_gather_add(self, L, N, phi, x, y, z, ax, ay, az):
        rc = self.lib.orc_gradient_gather_add(_c_double(L), _c_u64(N), _dp(phi), _c_u64(x.size),
                                              _dp(x), _dp(y), _dp(z), _dp(ax), _dp(ay), _dp(az))
        self._check(rc, "orc_gradient_gather_add")

    def pm_forces(self, L, N, x, y, z, masses=None, uniform_mass=1.0, deconvolve=False,
                  ax=None, ay=None, az=None):
        n = x.size
        ax = np.zeros(n) if ax is None else ax
        ay = np.zeros(n) if ay is None else ay
        az = np.zeros(n) if az is None else az
        rc = self.lib.orc_pm_forces(_c_double(L), _c_u64(N), _c_int(int(deconvolve)), _c_u64(n),
                                    _dp(x), _dp(y), _dp(z), _dp(masses), _c_double(uniform_mass),
                                    _dp(ax), _dp(ay), _dp(az))
        self._check(rc, "orc_pm_forces")
        return ax, ay, az

    def short_range_pair(self, r_s, eps, mass, dx, dy, dz):
        dx, dy, dz = (np.ascontiguousarray(a, dtype=np.float64) for a in (dx, dy, dz))
        out = [np.zeros(dx.size) for _ in range(3)]
        self.lib.orc_short_range_pair(_c_double(r_s), _c_double(eps), _c_double(mass),
                                      _c_u64(dx.size), _dp(dx), _dp(dy), _dp(dz),
                                      *(_dp(o) for o in out))
        return out

    def short_range_direct(self, L, x, y, z, mass, targets, r_s, r_cut, eps):
        targets = np.ascontiguousarray(targets, dtype=np.uint32)
        out = [np.zeros(targets.size) for _ in range(3)]
        rc = self.lib.orc_short_range_direct(
            _c_double(L), _c_u64(x.size), _dp(x), _dp(y), _dp(z), _c_double(mass),
            _c_u64(targets.size), _ip(targets, ctypes.c_uint32), _c_double(r_s),
            _c_double(r_cut), _c_double(eps), *(_dp(o) for o in out))
        self._check(rc, "orc_short_range_direct")
        return out

    def kdk_step(self, L, N, state, K1, D, K2, masses=None, uniform_mass=1.0,
                 deconvolve=False):
        """state: dict of float64 arrays x,y,z,px,py,pz,ax,ay,az (updated in place)."""
        md = ctypes.c_double(0.0)
        s = state
        rc = self.lib.orc_kdk_step(
            _c_double(L), _c_u64(N), _c_int(int(deconvolve)), _c_u64(s["x"].size),
            _dp(s["x"]), _dp(s["y"]), _dp(s["z"]), _dp(s["px"]), _dp(s["py"]), _dp(s["pz"]),
            _dp(s["ax"]), _dp(s["ay"]), _dp(s["az"]), _dp(masses), _c_double(uniform_mass),
            _c_double(K1), _c_double(D), _c_double(K2), ctypes.byref(md))
        self._check(rc, "orc_kdk_step")
        return md.value


class Reference:
    """The reference's own compiled sources (oracle/_ref/libhyowon_ref.so)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (oracle/ref/Makefile)")
        self.lib = ctypes.CDLL(path)
        self.lib.ref_last_error.restype = ctypes.c_char_p

    def _check(self, rc, where):
        if rc != 0:
            raise OracleError(rc, where, self.lib.ref_last_error().decode())

    def cic_coords(self, L, N, pos):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        base = np.zeros(pos.size, dtype=np.int64)
        frac = np.zeros(pos.size, dtype=np.float64)
        rc = self.lib.ref_cic_coords(_c_double(L), _c_u64(N), _c_u64(pos.size), _dp(pos),
                                     _ip(base, ctypes.c_int64), _dp(frac))
        self._check(rc, "ref_cic_coords")
        return base, frac

    def deposit(self, L, N, x, y, z, masses=None, uniform_mass=1.0):
        mesh = np.zeros(N * N * N, dtype=np.float64)
        rc = self.lib.ref_deposit(_c_double(L), _c_u64(N), _c_u64(x.size), _dp(x), _dp(y), _dp(z),
                                  _dp(masses), _c_double(uniform_mass), _dp(mesh))
        self._check(rc, "ref_deposit")
        return mesh

    def potential(self, L, N, x, y, z, masses=None, uniform_mass=1.0, deconvolve=False):
        dens = np.zeros(N * N * N)
        phi = np.zeros(N * N * N)
        rc = self.lib.ref_potential(_c_double(L), _c_u64(N), _c_int(int(deconvolve)),
                                    _c_u64(x.size), _dp(x), _dp(y), _dp(z), _dp(masses),
                                    _c_double(uniform_mass), _dp(dens), _dp(phi))
        self._check(rc, "ref_potential")
        return dens, phi

    def pm_forces(self, L, N, x, y, z, masses=None, uniform_mass=1.0, deconvolve=False,
                  method=0, r_s=0.0, ax=None, ay=None, az=None):
        n = x.size
        ax = np.zeros(n) if ax is None else ax
        ay = np.zeros(n) if ay is None else ay
        az = np.zeros(n) if az is None else az
        rc = self.lib.ref_pm_forces(_c_double(L), _c_u64(N), _c_int(method),
                                    _c_int(int(deconvolve)), _c_double(r_s), _c_u64(n),
                                    _dp(x), _dp(y), _dp(z), _dp(masses), _c_double(uniform_mass),
                                    _dp(ax), _dp(ay), _dp(az))
        self._check(rc, "ref_pm_forces")
        return ax, ay, az

    def pm_forces_energy(self, L, N, x, y, z, masses=None, uniform_mass=1.0, deconvolve=False):
        """PMSolver::compute_forces(..., collect_potential_energy=true): returns
        (ax, ay, az, potential_energy_comoving)."""
        n = len(x)
        x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
        ax, ay, az = np.zeros(n), np.zeros(n), np.zeros(n)
        e = ctypes.c_double(0.0)
        m = None if masses is None else np.ascontiguousarray(masses, dtype=np.float64)
        rc = self.lib.ref_pm_forces_energy(
            _c_double(L), _c_u64(N), _c_int(int(deconvolve)), _c_u64(n), _dp(x), _dp(y), _dp(z),
            _dp(m), _c_double(uniform_mass), _dp(ax), _dp(ay), _dp(az), ctypes.byref(e))
        self._check(rc, "ref_pm_forces_energy")
        return ax, ay, az, e.value

    def post_force_energy(self, L, N, x, y, z, px, py, pz, masses=None, uniform_mass=1.0,
                          deconvolve=False):
        """PMSolver::measure_post_force_energy_diagnostics_in_place after a force
        solve: (potential_energy_comoving, directional_potential_energy_comoving)."""
        n = len(x)
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z, px, py, pz)]
        m = None if masses is None else np.ascontiguousarray(masses, dtype=np.float64)
        out = np.zeros(2)
        rc = self.lib.ref_post_force_energy(
            _c_double(L), _c_u64(N), _c_int(int(deconvolve)), _c_u64(n), _dp(a[0]), _dp(a[1]),
            _dp(a[2]), _dp(m), _c_double(uniform_mass), _dp(a[3]), _dp(a[4]), _dp(a[5]), _dp(out))
        self._check(rc, "ref_post_force_energy")
        return float(out[0]), float(out[1])

    def power_spectrum(self, L, mesh, x, y, z, masses=None, uniform_mass=1.0, num_bins=16,
                       subtract_shot_noise=False, interlaced=False, max_k_fraction_nyquist=1.0):
        """MatterPowerSpectrum::compute_pk: dict of per-bin arrays."""
        x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
        m = None if masses is None else np.ascontiguousarray(masses, dtype=np.float64)
        out = np.zeros(7 * num_bins)
        counts = np.zeros(num_bins, dtype=np.uint64)
        rc = self.lib.ref_power_spectrum(
            _c_double(L), _c_u64(mesh), _c_u64(x.size), _dp(x), _dp(y), _dp(z), _dp(m),
            _c_double(uniform_mass), _c_int(num_bins), _c_int(int(subtract_shot_noise)),
            _c_int(int(interlaced)), _c_double(max_k_fraction_nyquist), _dp(out),
            _ip(counts, ctypes.c_uint64))
        self._check(rc, "ref_power_spectrum")
        o = out.reshape(num_bins, 7)
        keys = ("k_low", "k_mean", "k_high", "p_raw", "p_corrected",
                "mean_cic_power_deconvolution_factor", "shot_noise_reference")
        res = {k: o[:, i].copy() for i, k in enumerate(keys)}
        res["mode_count"] = counts
        return res

    def conservation(self, L, N, px, py, pz, ax, ay, az, mass, a):
        """ConservationChecks: (kinetic energy at a, sum m p . g)."""
        arr = [np.ascontiguousarray(v, dtype=np.float64) for v in (px, py, pz, ax, ay, az)]
        out = np.zeros(2)
        rc = self.lib.ref_conservation(_c_double(L), _c_u64(N), _c_u64(arr[0].size),
                                       *[_dp(v) for v in arr], _c_double(mass), _c_double(a),
                                       _dp(out))
        self._check(rc, "ref_conservation")
        return float(out[0]), float(out[1])

    def force_balance(self, ax, ay, az, masses=None, uniform_mass=1.0):
        """validation::compute_force_balance_diagnostics: |sum m a| / sum m |a|."""
        ax, ay, az = (np.ascontiguousarray(v, dtype=np.float64) for v in (ax, ay, az))
        m = None if masses is None else np.ascontiguousarray(masses, dtype=np.float64)
        r = ctypes.c_double(0.0)
        rc = self.lib.ref_force_balance(_c_u64(len(ax)), _dp(m), _c_double(uniform_mass),
                                        _dp(ax), _dp(ay), _dp(az), ctypes.byref(r))
        self._check(rc, "ref_force_balance")
        return r.value

    def short_range_pair(self, r_s, cutoff_multiplier, eps, mass, dx, dy, dz):
        dx, dy, dz = (np.ascontiguousarray(a, dtype=np.float64) for a in (dx, dy, dz))
        out = [np.zeros(dx.size) for _ in range(3)]
        rc = self.lib.ref_short_range_pair(_c_double(r_s), _c_double(cutoff_multiplier),
                                           _c_double(eps), _c_double(mass), _c_u64(dx.size),
                                           _dp(dx), _dp(dy), _dp(dz), *(_dp(o) for o in out))
        self._check(rc, "ref_short_range_pair")
        return out

    def tree_short_forces(self, L, n_side, n_mesh, split_scale_cells, cutoff_multiplier, eps,
                          theta, mass, x, y, z, targets):
        targets = np.ascontiguousarray(targets, dtype=np.uint32)
        out = [np.zeros(targets.size) for _ in range(3)]
        rc = self.lib.ref_tree_short_forces(
            _c_double(L), _c_u64(n_side), _c_u64(n_mesh), _c_double(split_scale_cells),
            _c_double(cutoff_multiplier), _c_double(eps), _c_double(theta), _c_double(mass),
            _c_u64(x.size), _dp(x), _dp(y), _dp(z), _c_u64(targets.size),
            _ip(targets, ctypes.c_uint32), *(_dp(o) for o in out))
        self._check(rc, "ref_tree_short_forces")
        return out

    def schedule(self, a_start, a_final, delta_ln_a, omega_m=0.3, omega_l=0.7, max_steps=100000):
        out = np.zeros(6 * max_steps)
        n = ctypes.c_uint64(0)
        rc = self.lib.ref_schedule(_c_double(omega_m), _c_double(omega_l), _c_double(a_start),
                                   _c_double(a_final), _c_double(delta_ln_a), _c_u64(max_steps),
                                   _dp(out), ctypes.byref(n))
        self._check(rc, "ref_schedule")
        return out[: 6 * n.value].reshape(n.value, 6)

    def hubble(self, a, omega_m=0.3, omega_l=0.7):
        a = np.ascontiguousarray(a, dtype=np.float64)
        H = np.zeros_like(a)
        rc = self.lib.ref_hubble(_c_double(omega_m), _c_double(omega_l), _c_u64(a.size), _dp(a), _dp(H))
        self._check(rc, "ref_hubble")
        return H

    def growth(self, a, omega_m=0.3, omega_l=0.7):
        a = np.ascontiguousarray(a, dtype=np.float64)
        D1 = np.zeros_like(a)
        f1 = np.zeros_like(a)
        rc = self.lib.ref_growth(_c_double(omega_m), _c_double(omega_l), _c_u64(a.size), _dp(a),
                                 _dp(D1), _dp(f1))
        self._check(rc, "ref_growth")
        return D1, f1

    def growth2(self, a, omega_m=0.3, omega_l=0.7):
        a = np.ascontiguousarray(a, dtype=np.float64)
        out = [np.zeros_like(a) for _ in range(4)]
        rc = self.lib.ref_growth2(_c_double(omega_m), _c_double(omega_l), _c_u64(a.size), _dp(a),
                                  *[_dp(o) for o in out])
        self._check(rc, "ref_growth2")
        return tuple(out)

    def kdk_run(self, L, N, state, a_start, a_final, delta_ln_a, steps, uniform_mass,
                deconvolve=False, omega_m=0.3, omega_l=0.7):
        """Runs `steps` KDK steps in place on state (x..pz); fills ax..az.
        Returns (per-step max drift, seconds of the step loop)."""
        s = state
        md = np.zeros(max(steps, 1))
        sec = ctypes.c_double(0.0)
        rc = self.lib.ref_kdk_run(
            _c_double(L), _c_u64(N), _c_int(int(deconvolve)), _c_double(omega_m),
            _c_double(omega_l), _c_double(a_start), _c_double(a_final), _c_double(delta_ln_a),
            _c_u64(steps), _c_u64(s["x"].size), _dp(s["x"]), _dp(s["y"]), _dp(s["z"]),
            _dp(s["px"]), _dp(s["py"]), _dp(s["pz"]), _c_double(uniform_mass), _dp(s["ax"]),
            _dp(s["ay"]), _dp(s["az"]), _dp(md), ctypes.byref(sec))
        self._check(rc, "ref_kdk_run")
        return md[:steps], sec.value

    def philox(self, counters, keys):
        """Philox4x32-10 blocks: counters (n, 4) u32, keys (n, 2) u32 -> (n, 4) u32."""
        c = np.ascontiguousarray(counters, dtype=np.uint32).reshape(-1, 4)
        k = np.ascontiguousarray(keys, dtype=np.uint32).reshape(-1, 2)
        out = np.zeros_like(c)
        rc = self.lib.ref_philox(_c_u64(c.shape[0]), _ip(c, ctypes.c_uint32),
                                 _ip(k, ctypes.c_uint32), _ip(out, ctypes.c_uint32))
        self._check(rc, "ref_philox")
        return out

    def mode_draws(self, seed, stream, modes):
        """(u1, u2, n1, n2) per integer mode counter (n, 3) under seed/stream."""
        m = np.ascontiguousarray(modes, dtype=np.int32).reshape(-1, 3)
        out = np.zeros((m.shape[0], 4))
        rc = self.lib.ref_mode_draws(_c_u64(seed), ctypes.c_uint32(stream), _c_u64(m.shape[0]),
                                     _ip(m, ctypes.c_int32), _dp(out))
        self._check(rc, "ref_mode_draws")
        return out

    def generate_ics(self, L, N, pk_path, z_pk, z_start, seed, lpt_order=1, mesh=0,
                     amplitude_fixed=False, pairing=0, max_mode=-1, particles=True):
        """RandomField::generate + LPTDisplacement::apply_to_arrays on the
        corner lattice. Returns a dict: M, K, D1, D2, f1, f2, H, a_start,
        modes (M, M, M//2+1) complex, power[s], amp (s, 2) and, when
        `particles`, x..pz."""
        meta = np.zeros(8)
        args = (_c_double(L), _c_u64(N), _c_u64(0), _c_u64(seed), _c_int(int(amplitude_fixed)),
                _c_int(pairing), _c_int(lpt_order), ctypes.c_int64(max_mode),
                _c_double(z_start), pk_path.encode(), _c_double(z_pk), _dp(meta))
        # first call: IC mesh and support only
        self.lib.ref_generate_ics.argtypes = None
        rc = self.lib.ref_generate_ics(*args[:2], _c_u64(mesh), *args[3:], None, None, None,
                                       None, None, None, None, None, None)
        self._check(rc, "ref_generate_ics")
        M, K = int(meta[0]), int(meta[1])
        modes = np.zeros((M, M, M // 2 + 1), dtype=np.complex128)
        power = np.zeros(3 * K * K + 1)
        amp = np.zeros((3 * K * K + 1, 2))
        n = N ** 3
        st = {k: np.zeros(n) for k in ("x", "y", "z", "px", "py", "pz")} if particles else None
        pp = [_dp(st[k]) for k in ("x", "y", "z", "px", "py", "pz")] if particles else [None] * 6
        rc = self.lib.ref_generate_ics(*args[:2], _c_u64(mesh), *args[3:],
                                       modes.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       _dp(power), _dp(amp), *pp)
        self._check(rc, "ref_generate_ics")
        out = dict(M=M, K=K, D1=meta[2], D2=meta[3], f1=meta[4], f2=meta[5], H=meta[6],
                   a_start=meta[7], modes=modes, power=power, amp=amp)
        if particles:
            out.update(st)
        return out

    def treepm_kdk_run(self, L, n_side, n_mesh, split_scale_cells, cutoff_multiplier, eps, theta,
                       state, a_start, a_final, delta_ln_a, steps, masses=None, uniform_mass=1.0):
        """TreePMSolver-driven KDK steps in place on state (x..pz); fills ax..az."""
        s = state
        for k in ("ax", "ay", "az"):
            s.setdefault(k, np.zeros_like(s["x"]))
        m = None if masses is None else np.ascontiguousarray(masses, dtype=np.float64)
        self.lib.ref_treepm_kdk_run.argtypes = None
        rc = self.lib.ref_treepm_kdk_run(
            _c_double(L), _c_u64(n_side), _c_u64(n_mesh), _c_double(split_scale_cells),
            _c_double(cutoff_multiplier), _c_double(eps), _c_double(theta), _c_double(a_start),
            _c_double(a_final), _c_double(delta_ln_a), _c_u64(steps),
            *(_dp(s[k]) for k in ("x", "y", "z", "px", "py", "pz")), _dp(m),
            _c_double(uniform_mass), _dp(s["ax"]), _dp(s["ay"]), _dp(s["az"]))
        self._check(rc, "ref_treepm_kdk_run")
        return s

    def lpt_white_noise(self, L, N, noise, pk_path, z_pk, z_start):
        """1LPT state from white noise through the reference's LinearPowerSpectrum,
        FFTBackend and LPTDisplacement (ref_lpt_white_noise). Returns a dict
        x..pz plus a_start, D1, f1, H."""
        noise = np.ascontiguousarray(noise, dtype=np.float64).reshape(-1)
        if noise.size != N ** 3:
            raise ValueError("noise must hold N^3 values")
        meta = np.zeros(4)
        st = {k: np.zeros(N ** 3) for k in ("x", "y", "z", "px", "py", "pz")}
        self.lib.ref_lpt_white_noise.argtypes = None
        rc = self.lib.ref_lpt_white_noise(_c_double(L), _c_u64(N), _dp(noise), pk_path.encode(),
                                          _c_double(z_pk), _c_double(z_start), _dp(meta),
                                          *(_dp(st[k]) for k in ("x", "y", "z", "px", "py", "pz")))
        self._check(rc, "ref_lpt_white_noise")
        st.update(a_start=meta[0], D1=meta[1], f1=meta[2], H=meta[3])
        return st


# The semantic header LinearPowerSpectrum requires
# (src/ic/linear_power_spectrum.cpp:31-46,184-229), for the flat LCDM
# cosmology of the harness (h 0.7, Om 0.3, Ob 0, OL 0.7, n_s 0.965, sigma8 0.8).
def write_power_spectrum_file(path, k, P, redshift):
    lines = ["# k_unit=h/Mpc", "# power_unit=(Mpc/h)^3", f"# redshift={redshift!r}",
             "# species=cold_plus_baryon", "# gauge=synchronous",
             "# fidelity=precision_boltzmann", "# normalization=sigma8_z0",
             "# normalization_value=0.8", "# nonlinear=false", "# massive_neutrino_sum_eV=0",
             "# h=0.7", "# omega_m=0.3", "# omega_b=0", "# omega_lambda=0.7", "# n_s=0.965"]
    lines += [f"{float(a)!r} {float(b)!r}" for a, b in zip(k, P)]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
