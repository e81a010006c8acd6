"""Generate the golden fixtures in tests/golden/ from the REFERENCE's own code.

Run in a checkout where the reference tree is available (it is compiled by
oracle/ref/Makefile into oracle/_ref/libhyowon_ref.so):

    python tests/golden/make_golden.py [--ref-root /path/to/HYOWON]

Every array here is produced by the reference's classes (CICCoordinateAxis,
CICMassAssignment, PMSolver, TimeStepper, DriftKickIntegrator,
LeapfrogIntegrator) driven through oracle/ref/ref_harness.cpp; the FFT under
them is oracle/fft3d.c because FFTW3 is not installed. The inputs are the
synthetic ICs (seeded white noise + BBKS spectrum + oracle/lpt_oracle.py 1LPT), stored in
the fixture so that the GPU box never regenerates them.

Fixtures:
  c1_schedule.npz     TimeStepper/DriftKick table for c1, c2, c4 (a_b, a_h, a_e, D, K1, K2)
  small_pm.npz        12^3-mesh deposit / density / potential / forces of 500
                      random particles incl. boundary positions (bit-level)
  c1_kdk.npz          c1 ICs, force at a_start, state after 1 and after 32 KDK
                      steps of the reference integrator
"""
from __future__ import annotations

import argparse
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.bindings import Reference, build_reference  # noqa: E402
from hyowon_b200 import ic  # noqa: E402
from oracle.lpt_oracle import lpt_ics  # noqa: E402


def edge_positions(rng, n, L):
    x = rng.uniform(0.0, L, n)
    special = np.array([0.0, -0.0, L, -L, np.nextafter(L, 0.0), np.nextafter(0.0, 1.0),
                        -1e-300, 3.5 * L, -2.25 * L, L / 2, np.nextafter(L / 2, 0.0),
                        L * (1 - 1e-16)])
    x[: special.size] = special
    return x


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default="/root/reference")
    args = ap.parse_args()
    build_reference(args.ref_root)
    ref = Reference()

    # -- schedules --------------------------------------------------------
    sched = {}
    for name in ("c1", "c2", "c4"):
        a0, dl = ic.config_schedule(name)
        sched[name] = ref.schedule(a0, 1.0, dl)
        sched[name + "_args"] = np.array([a0, 1.0, dl])
    np.savez_compressed(os.path.join(HERE, "c1_schedule.npz"), **sched)

    # -- small PM pipeline with boundary positions ---------------------------
    rng = np.random.default_rng(2024)
    L, N, n = 37.5, 12, 500
    x = edge_positions(rng, n, L)
    y = rng.uniform(-L, 2 * L, n)
    z = edge_positions(np.random.default_rng(7), n, L)[::-1].copy()
    masses = rng.uniform(0.5, 2.0, n)
    base_x, frac_x = ref.cic_coords(L, N, x)
    dep_u = ref.deposit(L, N, x, y, z, uniform_mass=0.75)
    dep_m = ref.deposit(L, N, x, y, z, masses=masses)
    dens, phi = ref.potential(L, N, x, y, z, uniform_mass=0.75)
    _, phi_dec = ref.potential(L, N, x, y, z, uniform_mass=0.75, deconvolve=True)
    ax, ay, az = ref.pm_forces(L, N, x, y, z, uniform_mass=0.75)
    bx, by, bz = ref.pm_forces(L, N, x, y, z, masses=masses)
    np.savez_compressed(
        os.path.join(HERE, "small_pm.npz"), L=L, N=N, x=x, y=y, z=z, masses=masses,
        base_x=base_x, frac_x=frac_x, deposit_uniform=dep_u, deposit_masses=dep_m,
        density=dens, phi=phi, phi_deconvolved=phi_dec, ax=ax, ay=ay, az=az,
        ax_m=bx, ay_m=by, az_m=bz, uniform_mass=0.75)

    # -- c1 evolution -------------------------------------------------------
    c = ic.CONFIGS["c1"]
    a0, dl = ic.config_schedule("c1")
    noise = ic.white_noise(c["n_side"], c["seed"])
    st = lpt_ics(noise, c["n_side"], c["box"], a0)
    m_p = ic.particle_mass(c["box"], c["n_side"])
    ics = {k: v.copy() for k, v in st.items()}
    f0 = ref.pm_forces(c["box"], c["mesh"], st["x"], st["y"], st["z"], uniform_mass=m_p)
    one = {k: v.copy() for k, v in st.items()}
    for k in ("ax", "ay", "az"):
        one[k] = np.zeros_like(st["x"])
    md1, _ = ref.kdk_run(c["box"], c["mesh"], one, a0, 1.0, dl, 1, m_p)
    full = {k: v.copy() for k, v in st.items()}
    for k in ("ax", "ay", "az"):
        full[k] = np.zeros_like(st["x"])
    mdf, secs = ref.kdk_run(c["box"], c["mesh"], full, a0, 1.0, dl, c["steps"], m_p)
    out = dict(box=c["box"], mesh=c["mesh"], particle_mass=m_p, a_start=a0, delta_ln_a=dl)
    out.update({"ic_" + k: v for k, v in ics.items()})
    out.update(f0_x=f0[0], f0_y=f0[1], f0_z=f0[2])
    out.update({"s1_" + k: v for k, v in one.items()})
    out.update({"s32_" + k: v for k, v in full.items()})
    out.update(max_drift_1=md1, max_drift_32=mdf)
    np.savez_compressed(os.path.join(HERE, "c1_kdk.npz"), **out)
    print(f"c1 reference evolution: {c['steps']} steps in {secs:.2f} s")


if __name__ == "__main__":
    main()
