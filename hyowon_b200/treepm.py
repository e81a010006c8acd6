"""TreePM short-range force on the device (include/hyowon_treepm.h) and the
TreePM force split helpers (include/cosmo_nbody/gravity/force_split.hpp)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat


class _Params(ctypes.Structure):
    _fields_ = [("box_size", ctypes.c_double), ("split_scale", ctypes.c_double),
                ("cutoff", ctypes.c_double), ("softening", ctypes.c_double),
                ("theta", ctypes.c_double), ("particle_mass", ctypes.c_double),
                ("precision", ctypes.c_int)]


def short_range_forces(box, x, y, z, particle_mass, targets, split_scale, cutoff, softening,
                       theta=0.5, precision="fp64"):
    """Short-range accelerations at `targets` (indices) from all sources.
    Returns (ax, ay, az, stats)."""
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    targets = np.ascontiguousarray(targets, dtype=np.uint32)
    p = _Params(box, split_scale, cutoff, softening, theta, particle_mass,
                {"fp64": 0, "fp32": 1}[precision])
    out = [np.empty(targets.size) for _ in range(3)]
    stats = np.zeros(6)
    rc = nat.lib().hyowon_treepm_short_forces(
        ctypes.byref(p), x.size, nat.dptr(x), nat.dptr(y), nat.dptr(z), targets.size,
        targets.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), *(nat.dptr(o) for o in out),
        nat.dptr(stats))
    if rc != nat.OK:
        msg = nat.lib().hyowon_treepm_last_error().decode(errors="replace")
        raise nat._EXC.get(rc, RuntimeError)(f"hyowon_treepm_short_forces: {msg}")
    info = dict(zip(("nodes", "depth", "visits_per_target", "interactions_per_target",
                     "build_ms", "walk_ms"), stats.tolist()))
    return out[0], out[1], out[2], info
