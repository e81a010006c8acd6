#!/usr/bin/env python
"""Benchmark of the HYOWON PM step (particle-mesh force + KDK update) on B200.

Workload (default): the 512^3-particle / 1024^3-mesh configuration, L = 1000
Mpc/h, flat LCDM (Om 0.3, OL 0.7), 1LPT at z = 49 from seeded white noise
(seed 7) shaped by a BBKS spectrum with sigma_8 = 0.8, steps uniform in ln a
(64 steps to z = 0). A "step" is one KDK step (one force evaluation). Synthetic
inputs: no public dataset is involved.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form fp64|fp32]
                    [--config c1|c2|c3|c3h] [--impl ours|reference]
    python bench.py --workload ic|adjoint|treepm [--steps K] [--warmup W]

The default line also carries `adjoint_cost` (the c4 adjoint workload below,
3 timed evaluations) and `treepm_step` (the c5 TreePM workload, 3 timed steps)
unless --no-side-workloads is given.

`--workload adjoint` times the differentiation form on its configuration
(128^3 particles, L = 256 Mpc/h, 128^3 mesh, 1LPT at z = 19 from white noise
seed 3, 16 KDK steps to z = 0, loss against the z = 0 CIC density of seed 4,
checkpoints every 4 steps): a "step" is one loss-and-gradient evaluation
(hyowon_vjp_1lpt_pm), and the line carries (forward + adjoint) / forward
against the production forward (hyowon_pm_lpt_ics + hyowon_pm_run + the CIC
mass mesh of the same model) in both arithmetic forms.

`--workload treepm` times the TreePM force on its configuration (256^3
particles, L = 256 Mpc/h, 256^3 mesh, r_s = 1.25 cells, r_cut = 4.5 r_s,
opening angle 0.5, softening 1/30 of the mean spacing, the clustered z = 0
state of a 64-step PM run of seed 5): a "step" is one KDK step with the TreePM
force (long range plus the octree short range of every particle).
`--treepm-side S` scales it to S^3 particles, L = S Mpc/h and an S^3 mesh (the
same density and cell size) for kernel profiles of a smaller case.

`--workload cufft` times cuFFT (through torch.fft) on the data of the c3
potential solve, for comparison with the five-pass transforms: 1-D transforms
along x and y of the chunked FP32 half spectrum (65 x 1024 x 1024 x 8
complex) and the 3-D r2c / c2r of the 1024^3 FP32 mesh.

`--workload ic` times HYOWON's generated initial conditions instead (the
Philox Fourier field and 2LPT of the 512^3 lattice on the automatic 1024^3 IC
mesh, L = 1000, z = 49): a "step" is one whole generation through
hyowon_pm_generate_ics into device-resident state (the handle's work arrays
kept from the first call, whose time is reported as first_call_ms); `e2e`
the same through hyowon_ic_generate into host arrays (allocating per call).

Prints one JSON line (rank 0). `value` = particle-steps/s over the K timed steps
with the state resident in HBM, timed with CUDA events on the library's stream
(max over ranks); `e2e` = the same metric through the public C ABI with host
buffers: upload of the IC state from pinned host memory, K calls of
hyowon_pm_kdk_step (host scalars in, max-drift read back), download of the final
state, all inside the timed region. Multi-GPU runs are independent replicas
(the PM step does not shard across GPUs in this build).
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--form", default="fp32", choices=["fp64", "fp32"])
    ap.add_argument("--sort-interval", type=int, default=None,
                    help="re-sort the particles every this many steps (library default 4)")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip timing the other arithmetic form")
    ap.add_argument("--config", default="c3", choices=["c1", "c2", "c3", "c3h"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="step",
                    choices=["step", "ic", "adjoint", "treepm", "cufft"])
    ap.add_argument("--no-side-workloads", action="store_true",
                    help="skip the adjoint (c4) and TreePM (c5) measurements the default step "
                         "line carries")
    ap.add_argument("--treepm-side", type=int, default=256,
                    help="particles per side of the TreePM workload; box (Mpc/h) and mesh scale "
                         "with it, so 128 is c5 at 1/8 of its particles and volume (for kernel "
                         "profiles)")
    args = ap.parse_args()
    if args.treepm_side < 32 or args.treepm_side & (args.treepm_side - 1):
        ap.error("--treepm-side must be a power of two of at least 32")
    return args


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region.

    The sampler is started, and its first reading awaited (up to 10 s), before
    the region opens; readings every 50 ms are kept only when their timestamp
    lies inside the region, so start-up and idle readings after it are left out.
    """

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    INTERVAL_MS = 50

    def __init__(self, device_index=0):
        self.dev = device_index
        self.proc = None
        self.path = None
        self.t_open = None
        self.t_close = None

    def _lines(self):
        try:
            with open(self.path) as f:
                return [ln for ln in f.read().splitlines() if ln.count(",") >= 9]
        except OSError:
            return []

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", str(self.INTERVAL_MS)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        if self.proc:
            deadline = time.time() + 10.0
            while time.time() < deadline and self.proc.poll() is None and not self._lines():
                time.sleep(0.02)
        self.t_open = time.time()
        return self

    def __exit__(self, *exc):
        self.t_close = time.time()
        if self.proc:
            # the reading in flight at the close lands within one interval
            time.sleep(2 * self.INTERVAL_MS / 1000.0)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    @staticmethod
    def _stamp(text):
        try:
            return datetime.datetime.strptime(text.strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def summary(self):
        rows = []
        for line in self._lines():
            parts = [p.strip() for p in line.split(",")]
            t = self._stamp(parts[0])
            if t is None or self.t_open is None or self.t_close is None:
                continue
            if self.t_open <= t <= self.t_close:
                rows.append(parts[1:])
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def replica_seed(base_seed: int, rank: int) -> int:
    """Noise seed of replica `rank`: each GPU evolves its own realisation."""
    return base_seed + rank


def max_over_ranks(value: float, device: str = "cuda") -> float:
    """The slowest rank's device time (all ranks call it; one all-reduce)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, n_per_rank: int, steps: int, max_ms: float) -> float:
    """Particle-steps/s of all replicas over the slowest rank's time."""
    return world * n_per_rank * steps / (max_ms * 1e-3)


def setup_dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def algorithmic_bytes(form, n_particles, n_mesh):
    """Algorithmic HBM bytes of one KDK step (particles sorted, gather reading
    the mesh once, Green's function fused between the transforms):
    B = Np (9 bx + 6 bp) + Ng^3 (b_dep + 5 b_fft).
    The precision form accumulates its int64 fixed-point cells in shared
    memory and writes each cell once as an FP32 offset, so b_dep = 4 there
    (no int64 mesh and no conversion pass reach HBM); binary64: b_dep = 8."""
    G = n_mesh ** 3
    if form == "fp64":
        return n_particles * (9 * 8 + 6 * 8) + G * (8 + 5 * 8)
    return n_particles * (9 * 4 + 6 * 4) + G * (4 + 5 * 4)


def phase_bytes(form, n, N, sort_fraction):
    """Algorithmic HBM bytes of one launch of each phase of ours (per step).

    kick/drift: read x, p, a; write candidate x, p (+ keys / ranks, and the
      scatter of x, p, id on sort steps or the cell-order index on the other
      steps, weighted by how often they occur);
    deposit: read positions once, write the half spectrum once (each finished
      shared-memory tile of cells is transformed along z before it is
      written, so the r2c along z is part of this launch; int64 / fixed-point
      accumulators never reach HBM);
    fft_forward / green / fft_inverse: the rest of the five-pass transform on a
      power-of-two mesh, each pass reading and writing its array once -- y pass
      (half spectrum in and out); x pass with the Green's multiply (in and
      out); y pass + z c2r (half spectrum in, mesh out);
    gather: read x, p and the potential once; write a and p.
    """
    G = N ** 3
    H = N * N * (N // 2 + 1)
    if form == "fp64":
        bx = bp = b = 8
    else:
        bx = bp = b = 4
    cplx = H * 2 * b
    dep = n * 3 * bx + cplx
    gather = n * (3 * bx + 3 * bp + 3 * bp + 3 * bp) + G * b
    kick = n * (3 * bx + 3 * bp + 3 * bp + 3 * bx + 3 * bp + 8)
    kick += sort_fraction * n * 2 * (3 * bx + 3 * bp + 4 + 8)
    kick += (1.0 - sort_fraction) * n * (4 + 4 + 4)   # cell order: key, rank in; order out
    return {"sort": kick, "deposit": dep, "fft_forward": 2 * cplx,
            "green": 2 * cplx, "fft_inverse": 2 * cplx + cplx + G * b, "gather": gather}


# DRAM bytes (read + write) per launch of the single-kernel phases on the c3
# workload, from an ncu --set full capture of the half-size c3 workload (c3h:
# 1/8 of the particles and mesh cells) times 8; each kernel's traffic scales
# with the particles and cells it processes.
TRAFFIC_C3 = {
    ("fp32", "deposit"): 8 * (285 + 492) * 1e6,
    ("fp32", "green"): 8 * (554 + 503) * 1e6,
    ("fp32", "gather"): 8 * (942 + 383) * 1e6,
    ("fp64", "deposit"): 8 * (487 + 1030) * 1e6,
    ("fp64", "green"): 8 * (1091 + 1034) * 1e6,
    ("fp64", "gather"): 8 * (1885 + 789) * 1e6,
}


def run_reference(args, world, rank):
    """The reference's own CPU implementation (oracle/_ref) on the host cores.

    Nothing of the product package runs here: the initial conditions come
    from oracle/workload.py and the reference's own LinearPowerSpectrum, FFT
    and LPTDisplacement; the timed region is the reference's TimeStepper +
    LeapfrogIntegrator + PMSolver loop."""
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    from oracle import workload
    from oracle.bindings import Reference
    cfg_name = args.config
    c = workload.CONFIGS[cfg_name]
    ref = Reference()
    a0, dl = workload.schedule(cfg_name)
    n_side = c["n_side"]
    st = workload.reference_ics(ref, cfg_name)
    for k in ("ax", "ay", "az"):
        st[k] = np.zeros_like(st["x"])
    m_p = workload.particle_mass(c["box"], n_side)
    # Bounded sample of the workload: the first steps of the schedule; the c3
    # workload (31 GB of host RAM in the reference) is sampled two steps at a time.
    steps = max(1, min(args.steps, 2 if cfg_name == "c3" else args.steps))
    _, secs = ref.kdk_run(c["box"], c["mesh"], st, a0, 1.0, dl, steps, m_p)
    value = n_side ** 3 * steps / secs
    libs = workload.loaded_native_libraries()
    if any("hyowon_b200" in lib for lib in libs):
        raise RuntimeError(f"the reference arm loaded the product library: {libs}")
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": value,
        "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": steps, "warmup": 0,
        "ms_per_step": 1e3 * secs / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": cfg_name, "particles": n_side ** 3, "mesh": c["mesh"],
                   "box": c["box"]},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores,
                         "kind": "reference",
                         "sample": f"{steps} KDK step(s) of {cfg_name} after the initial force; "
                                   f"reference Release build (-O3 -DNDEBUG, OpenMP on, "
                                   f"OMP_NUM_THREADS={os.environ.get('OMP_NUM_THREADS')}, "
                                   f"OMP_PROC_BIND={os.environ.get('OMP_PROC_BIND', 'unset')}), "
                                   f"FFT: oracle/fft3d.c in place of FFTW3 (not installed)"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "native_libraries": libs,
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(cfg_name):
    """Times the reference (oracle/_ref) on a bounded sample: KDK steps of the
    c2-sized problem when the full configuration would exceed ~30 s. Its
    initial conditions are the reference's own (oracle/workload.py)."""
    try:
        from oracle import workload
        from oracle.bindings import Reference
        ref = Reference()
    except Exception as e:  # pragma: no cover
        return {"value": None, "unit": "particle-steps/s", "cores": os.cpu_count(),
                "kind": "reference", "sample": f"unavailable: {e}"}
    name = "c2" if cfg_name in ("c3", "c3h") else cfg_name
    c = workload.CONFIGS[name]
    a0, dl = workload.schedule(name)
    st = workload.reference_ics(ref, name)
    for k in ("ax", "ay", "az"):
        st[k] = np.zeros_like(st["x"])
    steps = 8 if name == "c2" else 16
    _, secs = ref.kdk_run(c["box"], c["mesh"], st, a0, 1.0, dl, steps,
                          workload.particle_mass(c["box"], c["n_side"]))
    return {"value": c["n_side"] ** 3 * steps / secs, "unit": "particle-steps/s",
            "cores": os.cpu_count(), "kind": "reference",
            "sample": f"{steps} KDK steps of {name} ({c['n_side']}^3 particles, "
                      f"{c['mesh']}^3 mesh) on all host threads, reference Release build "
                      f"with OpenMP"}


IC_WORKLOAD = dict(n_side=512, box=1000.0, z_start=49.0, seed=7, lpt_order=2)
IC_SAMPLE = dict(n_side=128, box=250.0)  # the CPU sample: same cell size, 1/64 of the volume


def ic_params(n_side, box, seed, order=2):
    from hyowon_b200 import ic
    a0 = 1.0 / (1.0 + IC_WORKLOAD["z_start"])
    p = ic.ICParams(n_side, box, seed, a0, lpt_order=order)
    return p, ic.power_table(p, ic.start_spectrum(a0))


def ic_cpu_baseline():
    """The reference's RandomField + LPTDisplacement (oracle/_ref) on the host
    cores for the 64^3 lattice, 2LPT, 128^3 IC mesh (same cell size)."""
    try:
        from oracle import workload
        from oracle.bindings import Reference, write_power_spectrum_file
        ref = Reference()
    except Exception as e:  # pragma: no cover
        return {"value": None, "unit": "particles/s", "cores": os.cpu_count(),
                "kind": "reference", "sample": f"unavailable: {e}"}
    k, P = workload.bbks_table()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "pk.txt")
        write_power_spectrum_file(path, k, P, 0.0)
        n = IC_SAMPLE["n_side"]
        t0 = time.perf_counter()
        ref.generate_ics(IC_SAMPLE["box"], n, path, 0.0, IC_WORKLOAD["z_start"],
                         IC_WORKLOAD["seed"], lpt_order=2)
        secs = time.perf_counter() - t0
    return {"value": n ** 3 / secs, "unit": "particles/s", "cores": os.cpu_count(),
            "kind": "reference",
            "sample": f"one 2LPT generation of a {n}^3 lattice on the {2 * n}^3 IC mesh "
                      f"(L = {IC_SAMPLE['box']}), all host threads, {secs:.2f} s"}


def run_ic(args, rank):
    """Generated-IC workload (see the module docstring)."""
    if rank != 0:
        return
    import hyowon_b200 as hb
    from hyowon_b200 import ic
    w = IC_WORKLOAD
    p, power = ic_params(w["n_side"], w["box"], w["seed"], w["lpt_order"])
    M, K = p.resolve()
    n = w["n_side"] ** 3
    m_p = ic.particle_mass(w["box"], w["n_side"])
    solver = hb.PMSolver(hb.MeshGeometry(w["box"], 1024), hb.PMForceMethod.pure_pm(False))
    # the first generation allocates the handle's IC work arrays and plans
    t0 = time.perf_counter()
    solver.generate_ics(p, power, m_p)
    first_ms = 1e3 * (time.perf_counter() - t0)
    for _ in range(max(0, args.warmup - 1)):
        solver.generate_ics(p, power, m_p)
    with ClockSampler() as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            solver.generate_ics(p, power, m_p)
        secs = time.perf_counter() - t0
    solver.close()
    ms = 1e3 * secs / args.steps
    host = {k: np.empty(n) for k in ("x", "y", "z", "px", "py", "pz")}
    # e2e: the standalone call into host arrays (device -> host copy inside)
    ic.generate_ics(p, power)
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps // 2)):
        host = ic.generate_ics(p, power)
    e2e_s = (time.perf_counter() - t0) / max(1, args.steps // 2)
    # lattice + field, 3 x (displacement + apply), 2LPT: 6 x (Hessian + source)
    # and 3 x (displacement + apply); cuFFT's own kernels not counted
    launches = 2 + 3 * 2 + (6 * 2 + 3 * 2 if w["lpt_order"] == 2 else 0)
    line = {
        "metric": "IC particles/s", "value": n / (ms * 1e-3), "unit": "particles/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"generated ICs: {w['n_side']}^3 lattice, {w['lpt_order']}LPT on "
                               f"the {M}^3 IC mesh, K = {K}", "box": w["box"],
                   "z_start": w["z_start"], "seed": w["seed"],
                   "l2": "IC mesh fields (8.6 GB each) >> 126 MB L2",
                   "timing": "wall clock around the synchronous call; the handle keeps its "
                             "IC work arrays and plans between generations (first_call_ms: "
                             "the cold call that allocates them)"},
        "first_call_ms": first_ms,
        "cpu_baseline": None if args.no_cpu_baseline else ic_cpu_baseline(),
        "e2e": {"value": n / e2e_s, "unit": "particles/s", "h2d_bytes_per_step": 8 * power.size,
                "d2h_bytes_per_step": 6 * 8 * n},
        "gpu_launches": launches * args.steps,
        "clocks": clk.summary(),
        "check": {"x_range": [float(host["x"].min()), float(host["x"].max())]},
    }
    print(json.dumps(line), flush=True)


def run_adjoint(args, rank, emit=True):
    """Differentiation form on c4 (see the module docstring)."""
    if rank != 0:
        return None
    import hyowon_b200 as hb
    from hyowon_b200 import ic
    from hyowon_b200.adjoint import DifferentiablePM
    c = ic.CONFIGS["c4"]
    n_side, N, L = c["n_side"], c["mesh"], c["box"]
    a0, dl = ic.config_schedule("c4")
    noise = ic.white_noise(n_side, c["seed"])
    res = {}
    for form in ("fp64", "fp32"):
        dpm = DifferentiablePM(L, n_side, N, a0, c["steps"], form, ckpt_every=4)
        target = dpm.final_delta(ic.white_noise(n_side, 4))
        for _ in range(max(1, args.warmup)):
            dpm.loss_and_grad(noise, target)
        t0 = time.perf_counter()
        internal = []
        for _ in range(args.steps):
            dpm.loss_and_grad(noise, target)
            internal.append(dpm.last_timings)
        grad_s = (time.perf_counter() - t0) / args.steps
        # the production forward of the same model on a PM handle: 16 KDK steps
        # from the same 1LPT state, device time from the handle's own events
        K1, D, K2 = hb.TimeStepper(a0, 1.0, dl).factors()
        m = ic.particle_mass(L, n_side)
        runs, lpts = [], []
        with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), form) as s:
            s.set_timing(True)
            for it in range(max(1, args.warmup) + args.steps):
                t0 = time.perf_counter()
                ic.lpt_on_device(s, noise, n_side, a0, m)
                t1 = time.perf_counter()
                s.run(K1, D, K2)
                if it >= max(1, args.warmup):
                    lpts.append(1e3 * (t1 - t0))
                    runs.append(s.last_timing()["total"])
        fwd_ms = float(np.median(runs))
        fi = float(np.median([t["forward_ms"] for t in internal]))
        ri = float(np.median([t["reverse_ms"] for t in internal]))
        res[form] = {"production_forward_ms": fwd_ms,
                     "adjoint_forward_ms": fi, "adjoint_reverse_ms": ri,
                     "cost_ratio_vs_production_forward": (fi + ri) / fwd_ms,
                     "cost_ratio_vs_own_forward": (fi + ri) / fi,
                     "gradient_wall_ms": 1e3 * grad_s,
                     "production_lpt_wall_ms": float(np.median(lpts))}
    n = n_side ** 3
    line = {
        "metric": "(forward + adjoint) / forward cost", "value": res["fp64"]["cost_ratio_vs_production_forward"],
        "unit": "x", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["fp64"]["adjoint_forward_ms"] + res["fp64"]["adjoint_reverse_ms"],
        "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"c4 differentiable PM: {n_side}^3 particles, {N}^3 mesh, "
                               f"L = {L}, 1LPT at z = {c['z_start']}, {c['steps']} KDK steps, "
                               f"checkpoints every 4", "seed": c["seed"], "target_seed": 4,
                   "timing": "CUDA events on the device: the adjoint's 16 KDK steps + loss "
                             "(forward) and reverse pass, against the production handle's "
                             "hyowon_pm_run of the same 16 steps from the same 1LPT state; "
                             "the 1LPT map, uploads and allocations are outside both"},
        "forms": res,
        "gradient_particle_steps_per_s": n * c["steps"] / (
            (res["fp64"]["adjoint_forward_ms"] + res["fp64"]["adjoint_reverse_ms"]) * 1e-3),
        "e2e": {"value": res["fp64"]["cost_ratio_vs_production_forward"], "unit": "x",
                "h2d_bytes_per_step": 8 * (n + N ** 3), "d2h_bytes_per_step": 8 * n},
    }
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_treepm(args, rank, emit=True):
    """TreePM KDK steps on c5 (see the module docstring)."""
    if rank != 0:
        return None
    import hyowon_b200 as hb
    from hyowon_b200 import ic
    n_side = args.treepm_side
    L, N, seed = float(n_side), n_side, 5
    a0 = 1.0 / 50.0
    K1, D, K2 = hb.TimeStepper(a0, 1.0, math.log(1.0 / a0) / 64).factors()
    m = ic.particle_mass(L, n_side)
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False)) as s:
        ic.lpt_on_device(s, ic.white_noise(n_side, seed), n_side, a0, m)
        s.run(K1, D, K2)
        st = s.download(acc=False)
    r_s = 1.25 * L / N
    eps = (L / n_side) / 30.0
    n = n_side ** 3
    # late steps of a continued run: K1/D/K2 of a step of the same size at a = 1
    dl = math.log(1.0 / a0) / 64
    sched = hb.TimeStepper(1.0 / math.exp(dl * (args.warmup + args.steps)), 1.0, dl).factors()
    res = {}
    for form in ("fp64", "fp32"):
        with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.treepm_long_range(r_s), form) as s:
            s.upload(st["x"], st["y"], st["z"], st["px"], st["py"], st["pz"], uniform_mass=m)
            sx, sy, sz, info = s.treepm_short_forces(0.5, eps, 4.5 * r_s)
            s.set_treepm_short_range(0.5, eps, 4.5 * r_s)
            s.solve_forces()
            W = args.warmup
            s.run(sched[0][:W], sched[1][:W], sched[2][:W])
            s.set_timing(True)
            with ClockSampler() as clk:
                t0 = time.perf_counter()
                s.run(sched[0][W:W + args.steps], sched[1][W:W + args.steps],
                      sched[2][W:W + args.steps])
                wall = time.perf_counter() - t0
            tm = s.last_timing()
            res[form] = {"ms_per_step": tm["total"] / args.steps, "wall_ms_per_step": 1e3 * wall / args.steps,
                         "short_range_build_ms": info["build_ms"], "short_range_walk_ms": info["walk_ms"],
                         "tree_nodes": info["nodes"], "visits_per_target": info["visits_per_target"],
                         "interactions_per_target": info["interactions_per_target"],
                         "clocks": clk.summary()}
    v = n / (res["fp64"]["ms_per_step"] * 1e-3)
    line = {
        "metric": "particle-steps/s", "value": v, "unit": "particle-steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["fp64"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"{'c5' if n_side == 256 else 'c5-shaped'} TreePM KDK: {n_side}^3 particles, {N}^3 mesh, L = {L}, "
                               f"r_s = 1.25 cells, r_cut = 4.5 r_s, theta = 0.5, eps = L/{n_side}/30, "
                               "clustered z = 0 state of a 64-step PM run", "seed": seed,
                   "l2": "particle arrays and meshes >> 126 MB"},
        "forms": res,
        "other_form": {"form": "fp32", "value": n / (res["fp32"]["ms_per_step"] * 1e-3)},
        "e2e": None,
    }
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_cufft(args, rank):
    """cuFFT on the c3 potential solve's data (see the module docstring)."""
    if rank != 0:
        return
    import torch
    N, CC = 1024, 8
    KC = (N // 2 + 1 + CC - 1) // CC
    x = torch.randn(KC, N, N, CC, dtype=torch.complex64, device="cuda")

    def timed(f):
        for _ in range(max(1, args.warmup)):
            f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            f()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    res = {"fft_x_ms": timed(lambda: torch.fft.fft(x, dim=1)),
           "fft_y_ms": timed(lambda: torch.fft.fft(x, dim=2)),
           "fft_ifft_x_ms": timed(lambda: torch.fft.ifft(torch.fft.fft(x, dim=1), dim=1))}
    del x
    torch.cuda.empty_cache()
    r = torch.randn(N, N, N, dtype=torch.float32, device="cuda")
    res["rfftn_ms"] = timed(lambda: torch.fft.rfftn(r))
    h = torch.fft.rfftn(r)
    res["irfftn_ms"] = timed(lambda: torch.fft.irfftn(h, s=(N, N, N)))
    line = {"metric": "cuFFT time on the c3 solve's data", "value": res["rfftn_ms"] + res["irfftn_ms"],
            "unit": "ms", "higher_is_better": False, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "cuFFT via torch.fft: 1024^3 r2c + c2r, and 1-D transforms of "
                                   "the 65 x 1024 x 1024 x 8 chunked half spectrum"},
            "timings": res, "e2e": None}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = setup_dist()
    if args.workload == "ic":
        run_ic(args, rank)
        return
    if args.workload == "adjoint":
        run_adjoint(args, rank)
        return
    if args.workload == "treepm":
        run_treepm(args, rank)
        return
    if args.workload == "cufft":
        run_cufft(args, rank)
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import hyowon_b200 as hb
    from hyowon_b200 import ic

    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=600))
    os.environ.setdefault("CUDA_VISIBLE_DEVICES", os.environ.get("CUDA_VISIBLE_DEVICES", ""))

    c = ic.CONFIGS[args.config]
    n_side, N, L = c["n_side"], c["mesh"], c["box"]
    n = n_side ** 3
    a0, dl = ic.config_schedule(args.config)
    stepper = hb.TimeStepper(a0, 1.0, dl)
    K1, D, K2 = stepper.factors()
    total_steps = args.warmup + args.steps
    if total_steps > K1.size:
        reps = math.ceil(total_steps / K1.size)
        K1, D, K2 = np.tile(K1, reps), np.tile(D, reps), np.tile(K2, reps)
    m_p = ic.particle_mass(L, n_side)
    noise = ic.white_noise(n_side, replica_seed(c["seed"], rank))

    def measure(form):
        """Device-resident K-step throughput of one arithmetic form."""
        solver = hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), form)
        ic.lpt_on_device(solver, noise, n_side, a0, m_p)
        if args.sort_interval is not None:
            solver.set_sort_interval(args.sort_interval)
        ics = solver.download(acc=False) if not args.no_e2e else None
        solver.solve_forces()
        solver.set_timing(True)
        solver.run(K1[:args.warmup], D[:args.warmup], K2[:args.warmup])
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        with ClockSampler(local) as clocks:
            t0 = time.perf_counter()
            solver.run(K1[args.warmup:total_steps], D[args.warmup:total_steps],
                       K2[args.warmup:total_steps])
            wall = time.perf_counter() - t0
        timing = solver.last_timing()
        dev_ms = timing["total"]
        if world > 1:
            dev_ms = max_over_ranks(dev_ms)
        return solver, ics, timing, dev_ms, wall, clocks.summary()

    solver, ics, timing, dev_ms, wall, clock_summary = measure(args.form)
    ms_per_step = dev_ms / args.steps
    value = whole_job_rate(world, n, args.steps, dev_ms)
    solves = max(1.0, timing["solves"])
    phases = {k: timing[k] / solves for k in ("sort", "deposit", "fft_forward", "green",
                                              "fft_inverse", "gather")}
    launches = int(timing["launches"])

    # -- roofline: every phase of ours at its algorithmic bytes over its CUDA-event
    #    time; the headline kernel is the longest of the phases that are one
    #    kernel each (deposit, the x pass with the Green's multiply, gather) ---
    hbm, peak_kind = peaks()
    pb = phase_bytes(args.form, n, N, sort_fraction=0.25)
    table = {}
    for k, b in pb.items():
        if phases[k] > 0:
            ach = b / (phases[k] * 1e-3) / 1e9
            table[k] = {"avg_ms": phases[k], "algorithmic_bytes": b, "achieved_GBs": ach,
                        "frac": ach / hbm}
    single = [k for k in ("deposit", "green", "gather") if k in table]
    dom = max(single, key=lambda k: table[k]["avg_ms"])
    kernel_name = {"deposit": "deposit + r2c along z", "green": "x pass + Green's multiply",
                   "gather": "gather + K2"}[dom]
    traffic = TRAFFIC_C3.get((args.form, dom)) if args.config == "c3" else None
    bound_note = {
        "deposit": "the kernel is bound by shared memory (fixed-point atomics, tile zeroing and "
                   "the r2c along z of each finished tile; 78% of the shared pipe's cycles in the "
                   "ncu capture of the half-size workload), not HBM: its HBM bytes are the "
                   "positions read and the half spectrum written once",
        "green": "two transforms per tile (forward x, Green's multiply, inverse x), issue- and "
                 "occupancy-bound",
        "gather": "latency of the 32 stencil loads per particle",
    }[dom]
    roofline = {"bound": "hbm", "kernel": kernel_name, "phase": dom, "note": bound_note,
                "achieved": table[dom]["achieved_GBs"], "peak": hbm, "unit": "GB/s",
                "frac": table[dom]["frac"], "traffic": traffic,
                "traffic_source": "ncu capture of the half-size c3 workload x 8" if traffic else None,
                "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": table[dom]["algorithmic_bytes"],
                "phases": table}
    step_bytes = algorithmic_bytes(args.form, n, N)
    step_roofline = {"algorithmic_bytes_per_step": step_bytes,
                     "achieved_GBs": step_bytes / (ms_per_step * 1e-3) / 1e9,
                     "frac": step_bytes / (ms_per_step * 1e-3) / 1e9 / hbm}

    # -- end to end through the C ABI with host buffers -------------------------
    def measure_e2e(e2e_solver, ics):
        import torch
        comps = ("x", "y", "z", "px", "py", "pz")
        pinned = {k: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for k in comps}
        result = {k: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for k in comps}
        for k in comps:
            pinned[k][:] = ics[k]
            result[k][:] = 0.0   # touch the pages before the timed region
        t0 = time.perf_counter()
        e2e_solver.upload(pinned["x"], pinned["y"], pinned["z"], pinned["px"], pinned["py"],
                          pinned["pz"], uniform_mass=m_p)
        for s in range(args.steps):
            e2e_solver.kdk_step(K1[s], D[s], K2[s])
        e2e_solver.download(out=result)
        e2e_secs = time.perf_counter() - t0
        if world > 1:
            e2e_secs = max_over_ranks(e2e_secs * 1e3) * 1e-3
        h2d = 6 * 8 * n + 24 * args.steps
        d2h = 6 * 8 * n + 8 * args.steps
        return {"value": whole_job_rate(world, n, args.steps, e2e_secs * 1e3),
                "unit": "particle-steps/s",
                "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": d2h / args.steps,
                "note": "pinned host buffers: upload of the IC positions and momenta, K "
                        "hyowon_pm_kdk_step calls (K1, D, K2 in, max drift out), download of "
                        "the final positions and momenta"}

    e2e = None if args.no_e2e else measure_e2e(solver, ics)
    final = solver.download() if args.form == "fp64" else None
    solver.close()
    compare = None
    if not args.no_compare:
        other = "fp64" if args.form == "fp32" else "fp32"
        s2, ics2, t2, dev2, _, _ = measure(other)
        e2e2 = None if args.no_e2e else measure_e2e(s2, ics2)
        if other == "fp64":
            final = s2.download()
        s2.close()
        v2 = whole_job_rate(world, n, args.steps, dev2)
        compare = {"form": other, "value": v2, "ms_per_step": dev2 / args.steps,
                   "ratio_fp32_over_fp64": (value / v2) if args.form == "fp32" else (v2 / value),
                   "phases_ms_avg": {k: t2[k] / max(1.0, t2["solves"])
                                     for k in ("sort", "deposit", "fft_forward", "green",
                                               "fft_inverse", "gather")},
                   "e2e": e2e2}

    # -- the precision form's force error at the state the binary64 run reached
    force_error = None
    if final is not None:
        with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False), "fp32") as s3:
            s3.upload(final["x"], final["y"], final["z"], uniform_mass=m_p)
            s3.solve_forces()
            f32 = s3.download()
        num = sum(float(np.sum((f32[k] - final[k]) ** 2)) for k in ("ax", "ay", "az"))
        den = sum(float(np.sum(final[k] ** 2)) for k in ("ax", "ay", "az"))
        # the binary64 handle last ran the e2e leg (K steps from the ICs), else W + K
        reached = args.steps if not args.no_e2e else total_steps
        a_end = a0 * math.exp(dl * reached) if reached <= c["steps"] else None
        force_error = {"fp32_vs_fp64_force_rel_rms": math.sqrt(num / den),
                       "state": f"the binary64 run's state after {reached} steps from the ICs"
                                + (f" (a = {a_end:.4f})" if a_end else ""),
                       "particles": n}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(args.config)

    # the metric's other two figures, on their own configurations (1 GPU)
    side = {}
    if rank == 0 and world == 1 and not args.no_side_workloads:
        side_args = argparse.Namespace(steps=3, warmup=1, treepm_side=256)
        for name, fn in (("adjoint", run_adjoint), ("treepm", run_treepm)):
            try:
                side[name] = fn(side_args, 0, emit=False)
            except Exception as e:  # reported, not hidden: the step line stands
                side[name] = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f32+i64",
            "data": "synthetic",
            "config": {"workload": args.config, "form": args.form, "particles": n, "mesh": N,
                       "box": L, "z_start": c["z_start"], "seed": c["seed"],
                       "l2": "inputs larger than L2 (meshes and particle arrays >> 126 MB)",
                       "parallelism": f"replicas{world}",
                       "sort_interval": 4 if args.sort_interval is None else args.sort_interval},
            "phases_ms_avg": phases,
            "other_form": compare,
            "roofline": roofline,
            "step_roofline": step_roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "force_error": force_error,
            "adjoint_cost": side.get("adjoint"),
            "treepm_step": side.get("treepm"),
            "gpu_launches": launches,
            "clocks": clock_summary,
            "wall_s_timed_region": wall,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
