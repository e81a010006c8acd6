"""Multi-GPU design of the binary64 step over x-slabs (hyowon_b200/slab.py),
run as gloo ranks on the CPU against the single-domain oracle
(oracle/pm_oracle.c, pinned bit for bit to the reference's PMSolver and
LeapfrogIntegrator).

* slab layout: the reference's FFTW-MPI block partition, owners, halo planes;
* 1, 2 and 3 ranks (a 32^3 mesh splits 16+16 and 11+11+10): particles handed
  out to ranks arbitrarily, migrated to the owner of their CIC base plane,
  overflow-plane deposit, slab FFT with all-to-all transposes, halo planes,
  centred-gradient gather -- accelerations within 1e-12 relative RMS of the
  oracle's full-mesh solve, with explicit per-particle masses;
* 3 KDK steps (drift, migration across slab edges, force, kicks): positions
  within 1e-9 of a cell and momenta within 1e-10 of max |p| of the oracle's.
The difference from the oracle is the FFT's summation order only.
"""
import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from hyowon_b200.slab import SlabLayout, SlabPM, cic_coords

L, N, NS = 100.0, 32, 16
STEPS = [(2e-3, 0.05, 2e-3), (2e-3, 0.05, 2e-3), (2e-3, 0.05, 2e-3)]


def initial_state():
    rng = np.random.default_rng(42)
    q = (np.arange(NS) + 0.25) * (L / NS)
    gx, gy, gz = np.meshgrid(q, q, q, indexing="ij")
    n = NS ** 3
    st = {
        "x": (gx.ravel() + rng.normal(0, 1.5, n)) % L,
        "y": (gy.ravel() + rng.normal(0, 1.5, n)) % L,
        "z": (gz.ravel() + rng.normal(0, 1.5, n)) % L,
        "px": rng.normal(0, 30.0, n), "py": rng.normal(0, 30.0, n), "pz": rng.normal(0, 30.0, n),
        "mass": rng.uniform(0.5, 2.0, n) * 1e3,
    }
    # a few particles on slab and box edges
    st["x"][:6] = [0.0, L / 2, np.nextafter(L / 2, 0.0), np.nextafter(L, 0.0), L * 11 / 32, L / 32]
    return st


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        st0 = initial_state()
        n = st0["x"].size
        mine = np.arange(rank, n, world)   # an arbitrary hand-out, not by slab
        st = {k: torch.from_numpy(np.ascontiguousarray(v[mine])) for k, v in st0.items()}
        st["id"] = torch.from_numpy(mine.astype(np.int64))
        pm = SlabPM(L, N)
        st = pm.migrate(st)
        base, _ = cic_coords(st["x"], L, N)
        assert bool(((base >= pm.x0) & (base < pm.x0 + pm.nx)).all())
        acc = pm.forces(st)
        first = (st["id"].numpy(), [a.numpy() for a in acc])
        for K1, D, K2 in STEPS:
            st, acc = pm.kdk_step(st, acc, K1, D, K2)
        final = {k: v.numpy() for k, v in st.items()}
        gathered = [None] * world
        dist.all_gather_object(gathered, (first, final, [a.numpy() for a in acc]))
        if rank == 0:
            np.save(out_path, np.array(gathered, dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def run_ranks(world, tmp_path):
    out = str(tmp_path / f"slab_{world}.npy")
    mp.start_processes(worker, args=(world, free_port(), out), nprocs=world, start_method="spawn")
    return np.load(out, allow_pickle=True)


def test_slab_layout():
    lay = SlabLayout(32, 3)
    assert [lay.start(r) for r in range(3)] == [0, 11, 22]
    assert [lay.count(r) for r in range(3)] == [11, 11, 10]
    assert lay.owner(10) == 0 and lay.owner(11) == 1 and lay.owner(31) == 2
    assert lay.halo_planes(0) == [31, 11, 12] and lay.halo_planes(2) == [21, 0, 1]
    with pytest.raises(ValueError):
        SlabLayout(4, 5)


def test_cic_coords_bit_exact_with_oracle(oracle):
    rng = np.random.default_rng(3)
    pos = np.concatenate([rng.uniform(-L, 2 * L, 5000),
                          [0.0, -0.0, L, np.nextafter(L, 0.0), -1e-300, 2.5 * L]])
    base, frac = cic_coords(torch.from_numpy(pos), L, N)
    ob, of = oracle.cic_coords(L, N, pos)
    assert np.array_equal(base.numpy(), ob) and np.array_equal(frac.numpy(), of)


@pytest.mark.parametrize("world", [1, 2, 3])
def test_slab_step_matches_single_domain_oracle(world, tmp_path, oracle):
    res = run_ranks(world, tmp_path)
    st0 = initial_state()
    n = st0["x"].size
    # forces at the initial state
    ax, ay, az = oracle.pm_forces(L, N, st0["x"], st0["y"], st0["z"], masses=st0["mass"])
    got = np.zeros((3, n))
    for (ids, acc), _, _ in res:
        for d in range(3):
            got[d, ids] = acc[d]
    want = np.stack([ax, ay, az])
    err = math.sqrt(np.sum((got - want) ** 2) / np.sum(want ** 2))
    print(f"{world} rank(s): initial force relative RMS vs oracle {err:.3e}")
    assert err <= 1e-12
    # KDK steps
    ref = {k: st0[k].copy() for k in ("x", "y", "z", "px", "py", "pz")}
    ref.update(ax=ax.copy(), ay=ay.copy(), az=az.copy())
    for K1, D, K2 in STEPS:
        oracle.kdk_step(L, N, ref, K1, D, K2, masses=st0["mass"])
    fin = {k: np.zeros(n) for k in ("x", "y", "z", "px", "py", "pz")}
    counted = np.zeros(n, dtype=int)
    for _, final, _ in res:
        ids = final["id"]
        counted[ids] += 1
        for k in fin:
            fin[k][ids] = final[k]
    assert np.all(counted == 1)
    dpos = max(np.max(np.abs((fin[k] - ref[k] + L / 2) % L - L / 2)) for k in "xyz") / (L / N)
    pmax = max(np.max(np.abs(ref[k])) for k in ("px", "py", "pz"))
    dmom = max(np.max(np.abs(fin[k] - ref[k])) for k in ("px", "py", "pz")) / pmax
    print(f"{world} rank(s): after {len(STEPS)} KDK steps max |dx| {dpos:.3e} cells, "
          f"max |dp| {dmom:.3e} of max |p|")
    assert dpos <= 1e-9 and dmom <= 1e-10
