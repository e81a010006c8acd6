"""hyowon_cic_deposit_noalloc (include/hyowon_noalloc.h): the CIC deposit that
allocates nothing, called through the C ABI on device buffers, against the PM
handle's binary64 deposit (hyowon_pm_download_mass_mesh after a force solve)
on the same particles. Tolerance: 1e-10 of the largest cell mass (the fixed
point quantises each contribution to n * max_mass * 2^-61); two calls in a row
must agree with the handle and give identical bits.

Collected last so it also runs after every other GPU test in one process."""
import ctypes
import os

import numpy as np
import pytest

import hyowon_b200 as hb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "hyowon_b200", "libhyowon_pm.so")
MAX_MESH = 64


def noalloc_lib():
    lib = ctypes.CDLL(LIB)
    f = lib.hyowon_cic_deposit_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                  ctypes.c_void_p, ctypes.c_void_p]
    lib.hyowon_noalloc_last_error.restype = ctypes.c_char_p
    return lib


def test_rejects_mesh_beyond_static_scratch():
    """Size checks come before any CUDA call, so this runs without a GPU."""
    lib = noalloc_lib()
    dummy = ctypes.c_void_p(16)
    rc = lib.hyowon_cic_deposit_noalloc(100.0, MAX_MESH + 1, 10, dummy, dummy, dummy, None,
                                        1.0, dummy, None)
    assert rc == 1  # HYOWON_EINVAL
    msg = lib.hyowon_noalloc_last_error().decode()
    assert "static scratch" in msg and str(MAX_MESH) in msg
    assert lib.hyowon_cic_deposit_noalloc(100.0, 1, 10, dummy, dummy, dummy, None, 1.0,
                                          dummy, None) == 1


def handle_deposit(L, N, x, y, z, masses, uniform_mass):
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.pure_pm(False)) as s:
        if masses is None:
            s.upload(x, y, z, uniform_mass=uniform_mass)
        else:
            s.upload(x, y, z, masses=masses)
        s.solve_forces()
        return s.mass_mesh().reshape(-1)


@pytest.mark.gpu
@pytest.mark.parametrize("N,n,per_particle", [(64, 200_000, False), (32, 50_000, True)])
def test_noalloc_deposit_matches_handle_deposit(N, n, per_particle):
    import torch

    lib = noalloc_lib()
    rng = np.random.default_rng(17 + N)
    L = 100.0
    x, y, z = (rng.uniform(0.0, L, n) for _ in range(3))
    # cell-assignment edge cases: the box faces, a negative zero, a wrap
    x[:4] = [0.0, -0.0, np.nextafter(L, 0.0), L]
    y[:4] = [L, 0.0, -1e-300, 2.5 * L]
    masses = rng.uniform(0.5, 2.0, n) if per_particle else None
    m = 0.73
    ref = handle_deposit(L, N, x, y, z, masses, m)

    dev = torch.device("cuda", 0)
    dx, dy, dz = (torch.from_numpy(a).to(dev) for a in (x, y, z))
    dm = torch.from_numpy(masses).to(dev) if per_particle else None
    mesh = torch.empty(N ** 3, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    outs = []
    for _ in range(2):
        mesh.fill_(-1.0)
        rc = lib.hyowon_cic_deposit_noalloc(L, N, n, dx.data_ptr(), dy.data_ptr(),
                                            dz.data_ptr(), dm.data_ptr() if dm is not None else None,
                                            m, mesh.data_ptr(), stream)
        assert rc == 0, lib.hyowon_noalloc_last_error().decode()
        got = mesh.cpu().numpy()
        scale = np.max(np.abs(ref))
        err = np.max(np.abs(got - ref))
        print(f"N={N} n={n}: max |noalloc - handle| = {err:.3e} (max cell {scale:.3e})")
        assert err <= 1e-10 * scale
        outs.append(got)
    assert np.array_equal(outs[0], outs[1])
    total = masses.sum() if per_particle else n * m
    assert abs(outs[0].sum() - total) <= 1e-10 * total


@pytest.mark.gpu
def test_noalloc_deposit_errors_leave_mesh_untouched():
    import torch

    lib = noalloc_lib()
    dev = torch.device("cuda", 0)
    N, n, L = 16, 1000, 10.0
    rng = np.random.default_rng(3)
    pos = [rng.uniform(0.0, L, n) for _ in range(3)]
    pos[1][7] = np.nan
    dx, dy, dz = (torch.from_numpy(a).to(dev) for a in pos)
    mesh = torch.full((N ** 3,), 7.0, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.hyowon_cic_deposit_noalloc(L, N, n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(),
                                        None, 1.0, mesh.data_ptr(), stream)
    assert rc == 2  # HYOWON_ELOGIC, as the reference's cell assignment throws logic_error
    assert torch.all(mesh == 7.0).item()
    # host memory is refused before any launch
    host = np.zeros(N ** 3)
    rc = lib.hyowon_cic_deposit_noalloc(L, N, n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(),
                                        None, 1.0, host.ctypes.data, stream)
    assert rc == 1
    assert "device memory" in lib.hyowon_noalloc_last_error().decode()
    # pinned host memory is not device memory either
    pinned = torch.zeros(N ** 3, dtype=torch.float64).pin_memory()
    rc = lib.hyowon_cic_deposit_noalloc(L, N, n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(),
                                        None, 1.0, pinned.data_ptr(), stream)
    assert rc == 1
    assert torch.all(pinned == 0.0).item()


@pytest.mark.gpu
def test_noalloc_deposit_checks_positions_and_mass_range_whatever_the_masses():
    """A non-finite position fails even when every mass is zero (nothing would
    be deposited), and masses whose total n * max_mass overflows binary64 are
    refused instead of giving a meaningless fixed-point scale."""
    import torch

    lib = noalloc_lib()
    dev = torch.device("cuda", 0)
    N, n, L = 16, 1000, 10.0
    rng = np.random.default_rng(5)
    pos = [rng.uniform(0.0, L, n) for _ in range(3)]
    pos[2][11] = np.inf
    dx, dy, dz = (torch.from_numpy(a).to(dev) for a in pos)
    mesh = torch.full((N ** 3,), 7.0, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.hyowon_cic_deposit_noalloc(L, N, n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(),
                                        None, 0.0, mesh.data_ptr(), stream)
    assert rc == 2, lib.hyowon_noalloc_last_error().decode()
    zero = torch.zeros(n, dtype=torch.float64, device=dev)
    rc = lib.hyowon_cic_deposit_noalloc(L, N, n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(),
                                        zero.data_ptr(), 0.0, mesh.data_ptr(), stream)
    assert rc == 2, lib.hyowon_noalloc_last_error().decode()
    assert torch.all(mesh == 7.0).item()
    pos[2][11] = 1.0
    dz = torch.from_numpy(pos[2]).to(dev)
    huge = torch.full((n,), 1e306, dtype=torch.float64, device=dev)
    rc = lib.hyowon_cic_deposit_noalloc(L, N, n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(),
                                        huge.data_ptr(), 0.0, mesh.data_ptr(), stream)
    assert rc == 1, lib.hyowon_noalloc_last_error().decode()
    assert torch.all(mesh == 7.0).item()
    rc = lib.hyowon_cic_deposit_noalloc(L, N, n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(),
                                        None, 1e306, mesh.data_ptr(), stream)
    assert rc == 1
    # all-zero masses with finite positions give an empty mesh
    rc = lib.hyowon_cic_deposit_noalloc(L, N, n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(),
                                        zero.data_ptr(), 0.0, mesh.data_ptr(), stream)
    assert rc == 0, lib.hyowon_noalloc_last_error().decode()
    assert torch.all(mesh == 0.0).item()
