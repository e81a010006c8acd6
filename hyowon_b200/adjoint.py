"""Differentiable PM: loss on the final CIC density and its gradient with
respect to the initial white noise (include/hyowon_adjoint.h)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat
from . import ic
from .pm import CosmologyModel, TimeStepper


class _Cfg(ctypes.Structure):
    _fields_ = [
        ("box_size", ctypes.c_double), ("n_side", ctypes.c_uint64),
        ("mesh_size", ctypes.c_uint64), ("precision", ctypes.c_int),
        ("n_nodes", ctypes.c_uint64), ("ln_k", nat.P_double), ("ln_p", nat.P_double),
        ("ln_p_y2", nat.P_double), ("momentum_factor", ctypes.c_double),
        ("particle_mass", ctypes.c_double), ("n_steps", ctypes.c_uint64),
        ("K1", nat.P_double), ("D", nat.P_double), ("K2", nat.P_double),
        ("ckpt_every", ctypes.c_uint64),
    ]


class DifferentiablePM:
    """noise -> 1LPT -> KDK steps -> CIC density; loss and d loss / d noise."""

    def __init__(self, box, n_side, mesh, a_start, n_steps, precision="fp64", ckpt_every=4,
                 model: CosmologyModel = None, solver=None):
        """With `solver` (a pure-PM PMSolver of this box, mesh and form) the
        VJP runs on that handle (hyowon_pm_vjp), which keeps the adjoint's
        plans and work arrays between calls."""
        self.solver = solver
        model = model or CosmologyModel()
        self.box, self.n_side, self.mesh = float(box), int(n_side), int(mesh)
        self.precision = {"fp64": 0, "fp32": 1}[precision]
        self.ckpt_every = int(ckpt_every)
        import math
        stepper = TimeStepper(a_start, 1.0, math.log(1.0 / a_start) / n_steps, model)
        self.K1, self.D, self.K2 = stepper.factors()
        self.ln_k, self.ln_p, self.y2, self.pf = ic.lpt_table(a_start, model=model)
        self.m = ic.particle_mass(self.box, self.n_side, model.omega_m)

    def _cfg(self):
        c = _Cfg()
        c.box_size, c.n_side, c.mesh_size, c.precision = self.box, self.n_side, self.mesh, self.precision
        c.n_nodes = self.ln_k.size
        c.ln_k, c.ln_p, c.ln_p_y2 = nat.dptr(self.ln_k), nat.dptr(self.ln_p), nat.dptr(self.y2)
        c.momentum_factor, c.particle_mass = self.pf, self.m
        c.n_steps = self.K1.size
        c.K1, c.D, c.K2 = nat.dptr(self.K1), nat.dptr(self.D), nat.dptr(self.K2)
        c.ckpt_every = self.ckpt_every
        return c

    def _call(self, noise, target, want_grad, want_delta):
        noise = np.ascontiguousarray(noise, dtype=np.float64)
        target = None if target is None else np.ascontiguousarray(target, dtype=np.float64)
        loss = ctypes.c_double(0.0)
        grad = np.empty(self.n_side ** 3) if want_grad else None
        delta = np.empty(self.mesh ** 3) if want_delta else None
        t = np.zeros(4)
        cfg = self._cfg()
        if self.solver is not None:
            rc = nat.lib().hyowon_pm_vjp(self.solver.handle, ctypes.byref(cfg), nat.dptr(noise),
                                         nat.dptr(target), ctypes.byref(loss), nat.dptr(grad),
                                         nat.dptr(delta), nat.dptr(t))
            nat.raise_for(rc, self.solver.handle, "hyowon_pm_vjp")
        else:
            rc = nat.lib().hyowon_vjp_1lpt_pm(ctypes.byref(cfg), nat.dptr(noise), nat.dptr(target),
                                              ctypes.byref(loss), nat.dptr(grad), nat.dptr(delta),
                                              nat.dptr(t))
            if rc != nat.OK:
                msg = nat.lib().hyowon_vjp_last_error().decode(errors="replace")
                raise nat._EXC.get(rc, RuntimeError)(f"hyowon_vjp_1lpt_pm: {msg}")
        self.last_timings = {"forward_ms": t[0], "reverse_ms": t[1], "force_solves": t[2],
                             "force_vjps": t[3]}
        return loss.value, grad, delta

    def final_delta(self, noise):
        return self._call(noise, None, False, True)[2]

    def loss(self, noise, target):
        return self._call(noise, target, False, False)[0]

    def loss_and_grad(self, noise, target):
        loss, grad, _ = self._call(noise, target, True, False)
        return loss, grad
