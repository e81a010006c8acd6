"""The header-only C++ face (hyowon_b200/csrc/gpu_pm_solver.hpp) as a C++ host
of the reference would use it: status codes become the reference's exception
types, and GpuPMSolver::compute_forces keeps PMSolver's add semantics
(src/gravity/pm_solver.cpp:494-567)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "hyowon_b200")


@pytest.fixture(scope="module")
def wrapper_exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    if not os.path.exists(os.path.join(LIBDIR, "libhyowon_pm.so")):
        pytest.fail("libhyowon_pm.so is not built")
    exe = str(tmp_path_factory.mktemp("cxx") / "wrapper_main")
    subprocess.run(["g++", "-std=c++20", "-O1", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(ROOT, "hyowon_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cxx", "wrapper_main.cpp"), "-L" + LIBDIR,
                    "-lhyowon_pm", "-Wl,-rpath," + LIBDIR, "-o", exe], check=True)
    return exe


def test_invalid_configuration_throws_invalid_argument(wrapper_exe):
    out = subprocess.run([wrapper_exe, "invalid"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "invalid_argument"


@pytest.mark.gpu
def test_compute_forces_through_cxx_matches_oracle(wrapper_exe, oracle, tmp_path):
    rng = np.random.default_rng(11)
    n, N, L, m = 20000, 32, 50.0, 0.7
    x, y, z = (rng.uniform(0, L, n) for _ in range(3))
    src = tmp_path / "in.bin"
    dst = tmp_path / "out.bin"
    with open(src, "wb") as f:
        f.write(np.array([n, N], dtype=np.uint64).tobytes())
        f.write(np.array([L, m], dtype=np.float64).tobytes())
        for a in (x, y, z):
            f.write(a.tobytes())
    out = subprocess.run([wrapper_exe, "forces", str(src), str(dst)], capture_output=True,
                         text=True)
    assert out.returncode == 0, out.stderr
    got = np.fromfile(dst, dtype=np.float64).reshape(3, n)
    ref = oracle.pm_forces(L, N, x, y, z, uniform_mass=m)
    scale = max(np.max(np.abs(r)) for r in ref)
    for g, r in zip(got, ref):
        # two solves were added to zeroed arrays
        assert np.max(np.abs(g - 2.0 * r)) <= 1e-12 * scale


@pytest.mark.gpu
def test_post_force_diagnostics_and_snapshot_through_cxx(wrapper_exe, oracle, tmp_path):
    """GpuPMSolver::measure_post_force_energy_diagnostics and snapshot_payload
    from C++: the oracle's values of the uploaded state."""
    from oracle import diag_oracle as dg
    rng = np.random.default_rng(12)
    n, N, L, m = 20000, 32, 50.0, 0.7
    x, y, z = (rng.uniform(0, L, n) for _ in range(3))
    px, py, pz = (rng.normal(0, 30.0, n) for _ in range(3))
    src = tmp_path / "in.bin"
    dst = tmp_path / "out.bin"
    with open(src, "wb") as f:
        f.write(np.array([n, N], dtype=np.uint64).tobytes())
        f.write(np.array([L, m], dtype=np.float64).tobytes())
        for a in (x, y, z, px, py, pz):
            f.write(a.tobytes())
    out = subprocess.run([wrapper_exe, "post", str(src), str(dst)], capture_output=True,
                         text=True)
    assert out.returncode == 0, out.stderr
    raw = np.fromfile(dst, dtype=np.float64)
    pe, de = raw[0], raw[1]
    coords = raw[2:2 + 3 * n].reshape(n, 3)
    vel = raw[2 + 3 * n:].reshape(n, 3)
    _, phi = oracle.potential(L, N, x, y, z, uniform_mass=m)
    b = np.empty((3, n), dtype=np.int64)
    f = np.empty((3, n))
    for d, v in enumerate((x, y, z)):
        b[d], f[d] = oracle.cic_coords(L, N, v)
    e_ref = dg.potential_energy_comoving(L, N, phi, b, f, m)
    d_ref, scale = dg.directional_potential_energy(L, N, phi, b, f, m, px, py, pz)
    assert abs(pe / e_ref - 1.0) < 1e-12
    assert abs(de - d_ref) <= 1e-12 * scale
    assert np.array_equal(coords, np.stack([x, y, z], axis=1))
    assert np.array_equal(vel, np.stack([px, py, pz], axis=1) * (1.0 / 0.5))


@pytest.mark.gpu
def test_treepm_step_through_cxx_equals_python_handle(wrapper_exe, tmp_path):
    """GpuPMSolver with Method::TreePMLongRange and set_treepm_short_range: a
    KDK step with explicit masses from C++ gives the same bits as the same
    calls through the Python view, and treepm_short_forces the short range."""
    import hyowon_b200 as hb
    rng = np.random.default_rng(21)
    n, N, L = 4096, 32, 50.0
    r_s = 1.25 * L / N
    theta, eps, r_cut = 0.5, L / 16 / 30, 4.5 * r_s
    masses = rng.uniform(0.5, 1.5, n) * 1e3
    c = [rng.uniform(0, L, n) for _ in range(3)] + [rng.normal(0, 20.0, n) for _ in range(3)]
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(src, "wb") as f:
        f.write(np.array([n, N], dtype=np.uint64).tobytes())
        f.write(np.array([L, r_s, theta, eps, r_cut], dtype=np.float64).tobytes())
        for a in [masses] + c:
            f.write(a.tobytes())
    out = subprocess.run([wrapper_exe, "treepm", str(src), str(dst)], capture_output=True,
                         text=True)
    assert out.returncode == 0, out.stderr
    got = np.fromfile(dst, dtype=np.float64).reshape(9, n)
    with hb.PMSolver(hb.MeshGeometry(L, N), hb.PMForceMethod.treepm_long_range(r_s)) as s:
        s.set_treepm_short_range(theta, eps, r_cut)
        s.upload(*c, masses=masses)
        s.kdk_step(1e-3, 1e-3, 1e-3)
        st = s.download()
        sx, sy, sz, _ = s.treepm_short_forces(theta, eps, r_cut)
    for k, name in enumerate(("x", "y", "z", "ax", "ay", "az")):
        assert np.array_equal(got[k], st[name]), name
    for k, v in zip((6, 7, 8), (sx, sy, sz)):
        assert np.array_equal(got[k], v)
