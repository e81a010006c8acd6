"""Distributed PM step over x-slabs: the multi-GPU design of the binary64 step.

HYOWON shards its PM solve across MPI ranks by x-slabs of the mesh
(src/gravity/distributed_pm_solver.cpp): a rank owns the planes
[x0, x0 + nx) and the particles whose CIC base plane lies in them; its deposit
spills into one plane past its slab, which is added into the right neighbour's
first plane (exchange_deposit_planes, :508-553); the transform is a slab FFT
whose transposes are an all-to-all (src/mesh/mpi_fft_backend.cpp); the
centred-gradient gather reads the potential of one plane on the left and two on
the right of the slab from the neighbours (potential halo,
include/cosmo_nbody/mesh/mpi_centered_gradient.hpp); after the drift, particles
that left the slab move to the rank that owns their new base plane
(src/domain/bounded_migration.cpp).

This module is that data plane over ``torch.distributed``: one process per GPU,
NCCL over NVLink / NVSwitch on GPUs (gloo on the CPU for tests). Every exchange
lands remote planes or particles in the receiving rank's own memory before
use (all-to-all and its variable-size form); no rank reads another's memory
directly. The per-rank arithmetic (cell assignment, deposit, 2-D/1-D
transforms, Green's function, gather, KDK) is written with torch tensor
operations on the slab, in the reference's formulas: it is the design and the
CPU-tested host logic of the multi-GPU step, not the tuned single-GPU kernels
of libhyowon_pm.so. Every collective is taken by every rank in the same order.

The exchanges, per force solve on P ranks with N^3 cells and n particles:
  migration   all-to-all of (counts, then 7-8 binary64 fields) of the movers;
  overflow    one N^2 plane per rank to the owner of plane x0 + nx;
  transpose   2 all-to-alls of the N^2 (N/2+1) half spectrum (forward, inverse);
  halo        three N^2 planes per rank (x0 - 1, x0 + nx, x0 + nx + 1).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch
import torch.distributed as dist

# include/cosmo_nbody/cosmology/units.hpp:12-25, evaluated in that order
_G = 6.67430e-11 * (1e10 * 1.98847e30) / (3.085677581491367e22 * 1000.0 * 1000.0)

FIELDS = ("x", "y", "z", "px", "py", "pz", "id", "mass")


@dataclass(frozen=True)
class SlabLayout:
    """x-slab partition of an N-plane mesh over P ranks, the block layout of
    the reference's FFTW-MPI slabs (block = ceil(N / P); trailing ranks may own
    fewer planes). Every rank must own at least one plane."""

    N: int
    world: int

    def __post_init__(self):
        if self.world < 1 or self.N < 2:
            raise ValueError("need at least one rank and a mesh of at least 2 planes")
        if self.count(self.world - 1) < 1:
            raise ValueError(f"{self.world} ranks leave a rank without planes on an {self.N}^3 mesh")

    @property
    def block(self) -> int:
        return -(-self.N // self.world)

    def start(self, rank: int) -> int:
        return min(rank * self.block, self.N)

    def count(self, rank: int) -> int:
        return max(0, min(self.N, (rank + 1) * self.block) - self.start(rank))

    def owner(self, plane):
        """Rank owning global plane(s) `plane` (int or integer tensor)."""
        return plane // self.block

    def halo_planes(self, rank: int):
        """Global planes rank needs from the others for its gather: one on the
        left, two on the right (periodic)."""
        x0, nx = self.start(rank), self.count(rank)
        return [(x0 - 1) % self.N, (x0 + nx) % self.N, (x0 + nx + 1) % self.N]


def cic_coords(pos: torch.Tensor, L: float, N: int):
    """CICCoordinateAxis (src/mesh/cic_coordinate.hpp:95-121) in binary64:
    wrap to [0, L) (fmod, exact), s = w / dx, clamp to [0, nextafter(N, 0)],
    base = floor(s), frac = s - base. Returns (base int64, frac)."""
    w = torch.where((pos >= 0) & (pos < L), pos, torch.fmod(pos, L))
    w = torch.where(w < 0, w + L, w)
    w = torch.where(w >= L, torch.zeros_like(w), w)
    if not bool(torch.isfinite(w).all()):
        raise ValueError("CIC bounded coordinate escaped the mesh domain")
    dx = L / N
    upper = math.nextafter(float(N), 0.0)
    s = torch.clamp(w / dx, 0.0, upper)
    base = torch.floor(s)
    return base.to(torch.int64), s - base


class SlabPM:
    """Pure-PM force and KDK step of the particles of this rank's slab.

    Particle state is a dict of 1-D tensors ``x, y, z, px, py, pz`` (binary64),
    ``id`` (int64, global particle index) and ``mass`` (binary64, per particle).
    """

    def __init__(self, box_size: float, mesh_size: int, group=None, deconvolve_cic=False):
        self.L = float(box_size)
        self.N = int(mesh_size)
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.layout = SlabLayout(self.N, self.world)
        self.x0 = self.layout.start(self.rank)
        self.nx = self.layout.count(self.rank)
        self.dx = self.L / self.N
        self.deconvolve = bool(deconvolve_cic)
        # 1-D Green's tables of src/mesh/green_function.cpp:59-80
        m = torch.arange(self.N, dtype=torch.float64)
        mode = torch.where(m <= self.N // 2, m, m - self.N)
        s = torch.sin(math.pi * mode / self.N)
        self.lap = -4.0 / (self.dx * self.dx) * s * s
        sinc = torch.where(mode == 0, torch.ones_like(mode),
                           torch.sin(math.pi * mode / self.N) / (math.pi * mode / self.N))
        self.win = sinc * sinc

    # -- collectives -------------------------------------------------------------
    def _all_to_all(self, send: torch.Tensor, send_counts, recv_counts) -> torch.Tensor:
        """Variable-size all-to-all along dim 0 of a real tensor."""
        out = torch.empty((sum(recv_counts),) + tuple(send.shape[1:]), dtype=send.dtype,
                          device=send.device)
        if self.world == 1:
            out.copy_(send)
            return out
        dist.all_to_all_single(out, send.contiguous(), list(recv_counts), list(send_counts),
                               group=self.group)
        return out

    def _exchange_counts(self, send_counts):
        t = torch.tensor(send_counts, dtype=torch.int64)
        if self.world == 1:
            return send_counts
        r = torch.empty_like(t)
        dist.all_to_all_single(r, t, group=self.group)
        return r.tolist()

    # -- particles ---------------------------------------------------------------
    def migrate(self, st: dict) -> dict:
        """Moves every particle to the rank owning its CIC base plane."""
        base, _ = cic_coords(st["x"], self.L, self.N)
        dest = self.layout.owner(base)
        order = torch.argsort(dest, stable=True)
        counts = torch.bincount(dest, minlength=self.world).tolist()
        recv = self._exchange_counts(counts)
        out = {}
        for k in FIELDS:
            v = st[k][order]
            if v.dtype == torch.int64:
                out[k] = self._all_to_all(v.view(torch.float64), counts, recv).view(torch.int64)
            else:
                out[k] = self._all_to_all(v, counts, recv)
        # a fixed local order (by global id) keeps results independent of arrival order
        keep = torch.argsort(out["id"], stable=True)
        return {k: v[keep] for k, v in out.items()}

    # -- mesh --------------------------------------------------------------------
    def deposit(self, st: dict) -> torch.Tensor:
        """CIC mass of the slab (nx, N, N): local deposit into nx + 1 planes,
        the overflow plane x0 + nx added into its owner's first plane."""
        N, nx = self.N, self.nx
        ix, fx = cic_coords(st["x"], self.L, N)
        iy, fy = cic_coords(st["y"], self.L, N)
        iz, fz = cic_coords(st["z"], self.L, N)
        lx = ix - self.x0
        if bool(((lx < 0) | (lx >= nx)).any()):
            raise RuntimeError("a particle outside this rank's slab reached the deposit")
        mesh = torch.zeros((nx + 1) * N * N, dtype=torch.float64, device=st["x"].device)
        m = st["mass"]
        for ox, wx in ((0, 1.0 - fx), (1, fx)):
            mx = m * wx
            gx = lx + ox
            for oy, wy in ((0, 1.0 - fy), (1, fy)):
                mxy = mx * wy
                gy = (iy + oy) % N
                for oz, wz in ((0, 1.0 - fz), (1, fz)):
                    gz = (iz + oz) % N
                    mesh.index_add_(0, (gx * N + gy) * N + gz, mxy * wz)
        mesh = mesh.view(nx + 1, N, N)
        # the overflow plane goes to the owner of global plane x0 + nx
        target = self.layout.owner((self.x0 + nx) % N)
        counts = [1 if q == target else 0 for q in range(self.world)]
        recv = [1 if self.layout.owner((self.layout.start(q) + self.layout.count(q)) % N) == self.rank
                else 0 for q in range(self.world)]
        got = self._all_to_all(mesh[nx:nx + 1].reshape(1, N * N), counts, recv)
        slab = mesh[:nx].clone()
        for plane in got:
            slab[0] += plane.view(N, N)
        return slab

    def potential(self, slab_mass: torch.Tensor, total_mass: float) -> torch.Tensor:
        """phi on the slab: rfft2 over (y, z) per plane, transpose to ky-slabs,
        fft along x, the discrete-Laplacian Green's function (optionally / W^2),
        inverse, transpose back, irfft2; the density (m - M/N^3)/dx^3 with the
        k = 0 mode zeroed (src/gravity/pm_solver.cpp:710-759,
        src/mesh/green_function.cpp:165-207). One 1/N^3 in the inverse."""
        N, nx, Hz = self.N, self.nx, self.N // 2 + 1
        rho = (slab_mass - total_mass / N ** 3) * (1.0 / self.dx ** 3)
        f = torch.fft.rfft2(rho, dim=(1, 2))                    # (nx, N, Hz)
        # transpose: rank q receives ky in its block range for all x
        ky_counts = [self.layout.count(q) for q in range(self.world)]
        parts = [f[:, self.layout.start(q):self.layout.start(q) + ky_counts[q], :]
                 for q in range(self.world)]
        send = torch.cat([torch.view_as_real(p.contiguous()).reshape(-1) for p in parts])
        send_counts = [nx * ky_counts[q] * Hz * 2 for q in range(self.world)]
        my_ky = ky_counts[self.rank]
        recv_counts = [self.layout.count(q) * my_ky * Hz * 2 for q in range(self.world)]
        got = self._all_to_all(send, send_counts, recv_counts)
        g = torch.view_as_complex(got.view(N, my_ky, Hz, 2))    # (N, my_ky, Hz), x ordered
        g = torch.fft.fft(g, dim=0)
        ky0 = self.layout.start(self.rank)
        Dk = (self.lap.view(N, 1, 1) + self.lap[ky0:ky0 + my_ky].view(1, my_ky, 1)
              + self.lap[:Hz].view(1, 1, Hz))
        green = 4.0 * math.pi * _G / torch.where(Dk == 0, torch.ones_like(Dk), Dk)
        if self.deconvolve:
            wt = (self.win.view(N, 1, 1) * self.win[ky0:ky0 + my_ky].view(1, my_ky, 1)
                  * self.win[:Hz].view(1, 1, Hz))
            green = green / (wt * wt)
        green = torch.where(Dk == 0, torch.zeros_like(green), green)
        g = torch.fft.ifft(g * green, dim=0)
        # transpose back: rank q receives its x planes for my ky range
        parts = [g[self.layout.start(q):self.layout.start(q) + self.layout.count(q)]
                 for q in range(self.world)]
        send = torch.cat([torch.view_as_real(p.contiguous()).reshape(-1) for p in parts])
        send_counts = [self.layout.count(q) * my_ky * Hz * 2 for q in range(self.world)]
        recv_counts = [nx * ky_counts[q] * Hz * 2 for q in range(self.world)]
        got = self._all_to_all(send, send_counts, recv_counts)
        blocks, off = [], 0
        for q in range(self.world):
            sz = nx * ky_counts[q] * Hz * 2
            blocks.append(torch.view_as_complex(got[off:off + sz].view(nx, ky_counts[q], Hz, 2)))
            off += sz
        h = torch.cat(blocks, dim=1)                            # (nx, N, Hz)
        return torch.fft.irfft2(h, s=(N, N), dim=(1, 2))

    def halo(self, phi: torch.Tensor) -> torch.Tensor:
        """phi extended by the halo planes: index 0 = plane x0 - 1, 1..nx = the
        slab, nx + 1 and nx + 2 = planes x0 + nx and x0 + nx + 1."""
        N, lay = self.N, self.layout
        send_planes, send_counts = [], []
        for q in range(self.world):
            mine = [g for g in lay.halo_planes(q) if lay.owner(g) == self.rank]
            send_planes += [phi[g - self.x0].reshape(-1) for g in mine]
            send_counts.append(len(mine) * N * N)
        recv_planes = lay.halo_planes(self.rank)
        recv_counts = [sum(1 for g in recv_planes if lay.owner(g) == q) * N * N
                       for q in range(self.world)]
        send = torch.cat(send_planes) if send_planes else phi.new_empty(0)
        got = self._all_to_all(send, send_counts, recv_counts)
        # received blocks arrive by source rank, each in this rank's halo order
        # (a plane listed twice, as on a 2-plane mesh, arrives twice)
        planes, off = [None] * len(recv_planes), 0
        for q in range(self.world):
            for i, g in enumerate(recv_planes):
                if lay.owner(g) == q:
                    planes[i] = got[off:off + N * N].view(N, N)
                    off += N * N
        ext = phi.new_empty((self.nx + 3, N, N))
        ext[1:self.nx + 1] = phi
        ext[0] = planes[0]
        ext[self.nx + 1] = planes[1]
        ext[self.nx + 2] = planes[2]
        return ext

    def gather(self, ext: torch.Tensor, st: dict):
        """Centred-gradient CIC gather (src/mesh/mass_assignment_gradient.cpp:
        46-226): a_d = sum_corners w (-(phi[c+e_d] - phi[c-e_d]) / (2 dx))."""
        N = self.N
        ix, fx = cic_coords(st["x"], self.L, N)
        iy, fy = cic_coords(st["y"], self.L, N)
        iz, fz = cic_coords(st["z"], self.L, N)
        lx = ix - self.x0 + 1          # index of the base plane in ext
        flat = ext.reshape(-1)

        def at(px, py, pz):
            return flat[(px * N + py % N) * N + pz % N]

        inv2dx = 1.0 / (2.0 * self.dx)
        acc = [torch.zeros_like(fx) for _ in range(3)]
        for ox, wx in ((0, 1.0 - fx), (1, fx)):
            cx = lx + ox
            for oy, wy in ((0, 1.0 - fy), (1, fy)):
                cy = iy + oy
                for oz, wz in ((0, 1.0 - fz), (1, fz)):
                    cz = iz + oz
                    w = wx * wy * wz
                    acc[0] += w * (-(at(cx + 1, cy, cz) - at(cx - 1, cy, cz)) * inv2dx)
                    acc[1] += w * (-(at(cx, cy + 1, cz) - at(cx, cy - 1, cz)) * inv2dx)
                    acc[2] += w * (-(at(cx, cy, cz + 1) - at(cx, cy, cz - 1)) * inv2dx)
        return acc

    def total_mass(self, st: dict) -> float:
        t = st["mass"].sum().reshape(1).clone()
        if self.world > 1:
            dist.all_reduce(t, group=self.group)
        return float(t.item())

    def forces(self, st: dict):
        """Accelerations of this rank's particles (st must be migrated)."""
        slab = self.deposit(st)
        phi = self.potential(slab, self.total_mass(st))
        return self.gather(self.halo(phi), st)

    def kdk_step(self, st: dict, acc, K1: float, D: float, K2: float):
        """K1 kick, drift with periodic wrap (add_periodic_displacement), migration,
        force, K2 kick (src/time/leapfrog_integrator.cpp:143-279,
        include/cosmo_nbody/time/particle_update.hpp:20-116). Returns (state, acc)."""
        L = self.L
        out = dict(st)
        for d, (p, x) in enumerate((("px", "x"), ("py", "y"), ("pz", "z"))):
            q = st[p] + acc[d] * K1
            disp = q * D
            half = 0.5 * L
            mi = torch.where((disp >= -half) & (disp < half), disp,
                             torch.remainder(disp + half, L) - half)
            w = torch.remainder(st[x], L)
            nxp = torch.remainder(w + mi, L)
            nxp = torch.where(nxp >= L, torch.zeros_like(nxp), nxp)
            out[p], out[x] = q, nxp
        out = self.migrate(out)
        a = self.forces(out)
        for d, p in enumerate(("px", "py", "pz")):
            out[p] = out[p] + a[d] * K2
        return out, a
