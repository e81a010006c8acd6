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
  c1_diag.npz         global diagnostics of the reference at the c1 ICs and after
                      32 steps (PMForceDiagnostics potential energy, kinetic
                      energy, force balance, momentum-force contraction, the
                      post-force directional energy derivative) and the
                      potential energy / force balance / directional derivative
                      of small_pm with masses

  pk.npz              MatterPowerSpectrum::compute_pk of the c1 states (own mesh
                      64 and 32; raw, shot-noise-subtracted, interlaced) and of
                      small_pm with explicit masses

  ic.npz              generated initial conditions of the reference
                      (RandomField::generate + LPTDisplacement::apply_to_arrays
                      on the corner lattice, IC_CASES: 1LPT / 2LPT, gaussian /
                      fixed, pairings, explicit K and mesh), the P(k) table
                      they read, Philox4x32-10 blocks and per-mode draws

    python tests/golden/make_golden.py --only diag    # c1_diag.npz alone
    python tests/golden/make_golden.py --only pk      # pk.npz alone
  lpt.npz             the white-noise 1LPT map of the configurations through the
                      reference (LinearPowerSpectrum of the BBKS table file,
                      FFTBackend r2c, LPTDisplacement::apply_to_arrays on the
                      corner lattice; oracle/workload.py + ref_lpt_white_noise):
                      LPT_CASES (c1, and 16^3 at z = 19 in a 50 Mpc/h box)

    python tests/golden/make_golden.py --only ic      # ic.npz alone
    python tests/golden/make_golden.py --only lpt     # lpt.npz alone
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


def diag_fixture(ref):
    """c1_diag.npz from the reference's PMSolver (collect_potential_energy),
    ConservationChecks and compute_force_balance_diagnostics, evaluated on the
    c1 states and the small_pm inputs already stored in the fixtures."""
    d = np.load(os.path.join(HERE, "c1_kdk.npz"))
    L, N, m = float(d["box"]), int(d["mesh"]), float(d["particle_mass"])
    out = {}
    for tag, a in (("ic", float(d["a_start"])), ("s32", 1.0)):
        x, y, z = d[tag + "_x"], d[tag + "_y"], d[tag + "_z"]
        px, py, pz = d[tag + "_px"], d[tag + "_py"], d[tag + "_pz"]
        ax, ay, az, e = ref.pm_forces_energy(L, N, x, y, z, uniform_mass=m)
        K, C = ref.conservation(L, N, px, py, pz, ax, ay, az, m, a)
        out.update({tag + "_a": a, tag + "_potential_energy": e, tag + "_kinetic_energy": K,
                    tag + "_momentum_force_contraction": C,
                    tag + "_force_balance": ref.force_balance(ax, ay, az, uniform_mass=m)})
        pe, de = ref.post_force_energy(L, N, x, y, z, px, py, pz, uniform_mass=m)
        out.update({tag + "_post_potential_energy": pe, tag + "_directional": de})
    sp = np.load(os.path.join(HERE, "small_pm.npz"))
    Ls, Ns = float(sp["L"]), int(sp["N"])
    ax, ay, az, e = ref.pm_forces_energy(Ls, Ns, sp["x"], sp["y"], sp["z"], masses=sp["masses"])
    out.update(small_masses_potential_energy=e,
               small_masses_force_balance=ref.force_balance(ax, ay, az, masses=sp["masses"]))
    dr = np.random.default_rng(31)
    spx, spy, spz = (dr.normal(0.0, 2.0, sp["x"].size) for _ in range(3))
    _, de = ref.post_force_energy(Ls, Ns, sp["x"], sp["y"], sp["z"], spx, spy, spz,
                                  masses=sp["masses"])
    out.update(small_px=spx, small_py=spy, small_pz=spz, small_masses_directional=de)
    np.savez_compressed(os.path.join(HERE, "c1_diag.npz"), **out)


PK_CASES = [  # (name, state, mesh, bins, shot, interlaced, max_k_fraction_nyquist)
    ("ic_raw", "ic", 64, 12, False, False, 1.0),
    ("s32_raw", "s32", 64, 12, False, False, 1.0),
    ("s32_shot", "s32", 64, 12, True, False, 1.0),
    ("s32_interlaced", "s32", 64, 12, False, True, 1.0),
    ("s32_mesh32", "s32", 32, 8, True, False, 0.5),
]
PK_FIELDS = ("k_low", "k_mean", "k_high", "p_raw", "p_corrected",
             "mean_cic_power_deconvolution_factor", "shot_noise_reference", "mode_count")


def pk_fixture(ref):
    """pk.npz from the reference's MatterPowerSpectrum on the stored c1 states
    and the small_pm inputs with explicit masses."""
    d = np.load(os.path.join(HERE, "c1_kdk.npz"))
    L, m = float(d["box"]), float(d["particle_mass"])
    out = {}
    for name, tag, mesh, nb, shot, il, frac in PK_CASES:
        r = ref.power_spectrum(L, mesh, d[tag + "_x"], d[tag + "_y"], d[tag + "_z"],
                               uniform_mass=m, num_bins=nb, subtract_shot_noise=shot,
                               interlaced=il, max_k_fraction_nyquist=frac)
        out.update({f"{name}__{k}": r[k] for k in PK_FIELDS})
    sp = np.load(os.path.join(HERE, "small_pm.npz"))
    for name, shot, il in (("masses_shot", True, False), ("masses_interlaced", False, True)):
        r = ref.power_spectrum(float(sp["L"]), int(sp["N"]), sp["x"], sp["y"], sp["z"],
                               masses=sp["masses"], num_bins=5, subtract_shot_noise=shot,
                               interlaced=il, max_k_fraction_nyquist=0.8)
        out.update({f"{name}__{k}": r[k] for k in PK_FIELDS})
    np.savez_compressed(os.path.join(HERE, "pk.npz"), **out)


# name, N, lpt_order, mesh request (0 = automatic), fixed amplitude, pairing
# (0 independent, 1 pair_a, 2 pair_b), K (-1 = (N-1)/2), seed
IC_CASES = [
    ("n16_1lpt", 16, 1, 0, False, 0, -1, 11),
    ("n16_2lpt", 16, 2, 0, False, 0, -1, 11),
    ("n16_2lpt_fixed_pair_b", 16, 2, 0, True, 2, -1, 12345678901),
    ("n12_2lpt_pair_a_k4", 12, 2, 0, False, 1, 4, 5),
    ("n16_1lpt_m32_k5", 16, 1, 32, False, 0, 5, 3),
]
IC_BOX, IC_Z_START, IC_Z_PK = 100.0, 49.0, 0.0


def ic_fixture(ref):
    """ic.npz from the reference's RandomField / LPTDisplacement / Philox."""
    import tempfile
    from oracle.bindings import write_power_spectrum_file
    k, P = ic.bbks_table()
    out = dict(pk_k=k, pk_P=P, box=IC_BOX, z_start=IC_Z_START, z_pk=IC_Z_PK)
    rng = np.random.default_rng(77)
    ctr = rng.integers(0, 2 ** 32, (254, 4), dtype=np.uint64)
    key = rng.integers(0, 2 ** 32, (254, 2), dtype=np.uint64)
    ctr = np.concatenate([np.zeros((1, 4), np.uint64), np.full((1, 4), 2 ** 32 - 1, np.uint64), ctr])
    key = np.concatenate([np.zeros((1, 2), np.uint64), np.full((1, 2), 2 ** 32 - 1, np.uint64), key])
    out.update(philox_ctr=ctr.astype(np.uint32), philox_key=key.astype(np.uint32),
               philox_out=ref.philox(ctr, key))
    modes = rng.integers(-700, 701, (512, 3)).astype(np.int32)
    out["draw_modes"] = modes
    for seed, stream in ((0, 0), (11, 0), (12345678901, 1)):
        out[f"draws_{seed}_{stream}"] = ref.mode_draws(seed, stream, modes)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "pk.txt")
        write_power_spectrum_file(path, k, P, IC_Z_PK)
        for name, N, order, mesh, fixed, pairing, K, seed in IC_CASES:
            g = ref.generate_ics(IC_BOX, N, path, IC_Z_PK, IC_Z_START, seed, lpt_order=order,
                                 mesh=mesh, amplitude_fixed=fixed, pairing=pairing, max_mode=K)
            for f in ("M", "K", "D1", "D2", "f1", "f2", "H", "a_start", "modes", "power", "amp",
                      "x", "y", "z", "px", "py", "pz"):
                out[f"{name}__{f}"] = g[f]
    np.savez_compressed(os.path.join(HERE, "ic.npz"), **out)


# name, lattice side, box, seed, z_start
LPT_CASES = [
    ("c1", 32, 100.0, 1, 49.0),
    ("s16_z19", 16, 50.0, 3, 19.0),
]


def lpt_fixture(ref):
    """lpt.npz: the reference's 1LPT state from the configs' white noise."""
    import tempfile
    from oracle import workload
    from oracle.bindings import write_power_spectrum_file
    k, P = workload.bbks_table()
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "pk.txt")
        write_power_spectrum_file(path, k, P, 0.0)
        for name, n_side, box, seed, z_start in LPT_CASES:
            noise = workload.white_noise(n_side, seed)
            st = ref.lpt_white_noise(box, n_side, noise, path, 0.0, z_start)
            out.update({f"{name}__{f}": np.asarray(st[f]) for f in
                        ("x", "y", "z", "px", "py", "pz", "a_start", "D1", "f1", "H")})
            out[f"{name}__args"] = np.array([n_side, box, seed, z_start])
    np.savez_compressed(os.path.join(HERE, "lpt.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=None,
                    help="reference source tree (default: $HYOWON_REF_ROOT, else the "
                         "REF_ROOT default of oracle/ref/Makefile)")
    ap.add_argument("--only", choices=["diag", "pk", "ic", "lpt"], default=None)
    args = ap.parse_args()
    build_reference(args.ref_root)
    ref = Reference()
    if args.only == "diag":
        diag_fixture(ref)
        return
    if args.only == "pk":
        pk_fixture(ref)
        return
    if args.only == "ic":
        ic_fixture(ref)
        return
    if args.only == "lpt":
        lpt_fixture(ref)
        return

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
    # TreePM long range: continuum Green's function, Gaussian split, W^-2, -ik
    tx, ty, tz = ref.pm_forces(L, N, x, y, z, uniform_mass=0.75, method=1, r_s=1.25 * L / N)
    np.savez_compressed(
        os.path.join(HERE, "small_pm.npz"), L=L, N=N, x=x, y=y, z=z, masses=masses,
        base_x=base_x, frac_x=frac_x, deposit_uniform=dep_u, deposit_masses=dep_m,
        density=dens, phi=phi, phi_deconvolved=phi_dec, ax=ax, ay=ay, az=az,
        ax_m=bx, ay_m=by, az_m=bz, uniform_mass=0.75, tl_x=tx, tl_y=ty, tl_z=tz,
        tl_r_s=1.25 * L / N)

    # -- TreePM short-range pair law (ForceSplitKernel) --------------------------
    prng = np.random.default_rng(55)
    r_s, mult, eps = 1.25, 4.5, 1.0 / 30.0
    r = np.concatenate([np.exp(prng.uniform(np.log(1e-4), np.log(5.6), 400)),
                        [1e-6, 0.001, 0.05, 0.0625, 0.06249, 1.25, 5.624]])
    u = prng.normal(size=(r.size, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    d = u * r[:, None]
    pax, pay, paz = ref.short_range_pair(r_s, mult, eps, 2.5, d[:, 0], d[:, 1], d[:, 2])
    np.savez_compressed(os.path.join(HERE, "treepm_pair.npz"), r_s=r_s, cutoff_multiplier=mult,
                        eps=eps, mass=2.5, dx=d[:, 0], dy=d[:, 1], dz=d[:, 2], ax=pax, ay=pay,
                        az=paz)

    # -- TreePM short-range walk of the reference (Octree + TreeWalk) ------------
    trng = np.random.default_rng(3)
    Lt, nst = 32.0, 32
    ux, uy, uz = (trng.uniform(0, Lt, nst ** 3) for _ in range(3))
    ut = np.sort(np.random.default_rng(4).choice(nst ** 3, 256, replace=False)).astype(np.uint32)
    uf = ref.tree_short_forces(Lt, nst, 32, 1.25, 4.5, 1.0 / 30.0, 0.5, 1.0, ux, uy, uz, ut)
    tree_out = dict(u_L=Lt, u_x=ux, u_y=uy, u_z=uz, u_targets=ut, u_ax=uf[0], u_ay=uf[1],
                    u_az=uf[2], u_r_s=1.25, u_r_cut=5.625, u_eps=1.0 / 30.0, u_mass=1.0)

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

    # clustered input for the tree: the c1 state at z = 0
    dxc = c["box"] / c["mesh"]
    ct = np.sort(np.random.default_rng(6).choice(c["n_side"] ** 3, 256, replace=False)).astype(np.uint32)
    cf = ref.tree_short_forces(c["box"], c["n_side"], c["mesh"], 1.25, 4.5,
                               c["box"] / c["n_side"] / 30.0, 0.5, m_p, full["x"], full["y"],
                               full["z"], ct)
    tree_out.update(c_targets=ct, c_ax=cf[0], c_ay=cf[1], c_az=cf[2], c_r_s=1.25 * dxc,
                    c_r_cut=4.5 * 1.25 * dxc, c_eps=c["box"] / c["n_side"] / 30.0)
    np.savez_compressed(os.path.join(HERE, "treepm_tree.npz"), **tree_out)
    diag_fixture(ref)
    pk_fixture(ref)
    ic_fixture(ref)
    lpt_fixture(ref)
    print(f"c1 reference evolution: {c['steps']} steps in {secs:.2f} s")


if __name__ == "__main__":
    main()
