"""A C program calls libccsd_gpu.so the way eT's Fortran shim would (tests/c_harness/et_driver.c):
host arrays in eT's column-major layouts, int64 dimensions, the four Cholesky blocks, int status
codes.  The CPU test builds it against include/ccsd_gpu.h and the library; the GPU test runs it
and checks its energy, Omega and both transformations against the oracle."""

import os
import subprocess

import numpy as np
import pytest

from et_b200.synthetic import make_system
from oracle import ccsd as oc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_harness", "et_driver.c")
LIBDIR = os.path.join(ROOT, "et_b200")


def _build(tmp_path):
    from et_b200.ccsd import load_library
    load_library()                      # the library must exist (build() made it)
    exe = str(tmp_path / "et_driver")
    cmd = ["gcc", "-std=c99", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", LIBDIR, "-lccsd_gpu", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_harness_builds_against_the_header_and_library(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
def test_c_harness_matches_oracle(tmp_path):
    exe = _build(tmp_path)
    n_o, n_v, n_J = 3, 8, 20
    s = make_system(n_o, n_v, n_J, seed=12)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o, s.e_hf)
    rng = np.random.default_rng(5)
    amp = 0.05 * rng.standard_normal(ref.n_amp)
    c = rng.standard_normal(ref.n_amp)
    ref.set_amplitudes(amp)
    L = s.L_mo
    o, v = slice(0, n_o), slice(n_o, None)
    with open(tmp_path / "in.bin", "wb") as f:
        np.array([n_o, n_v, n_J], dtype=np.int64).tofile(f)
        for blk in (L[:, o, o], L[:, o, v], L[:, v, o], L[:, v, v]):
            np.asarray(blk).ravel(order="F").tofile(f)          # (J, p, q), J fastest
        np.asarray(s.h_mo).ravel(order="F").tofile(f)
        np.asarray(s.eps, dtype=np.float64).tofile(f)
        np.array([s.e_hf]).tofile(f)
        amp.tofile(f)
        c.tofile(f)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(tmp_path / "out.bin")
    n = ref.n_amp
    energy, omega, rho, sigma = out[0], out[1:1 + n], out[1 + n:1 + 2 * n], out[1 + 2 * n:]
    assert abs(energy - ref.energy()) < 1e-12
    om_ref = ref.omega()
    assert np.abs(omega - om_ref).max() <= 1e-12 * max(1.0, np.abs(om_ref).max())
    A = ref.jacobian_matrix()
    assert np.abs(rho - A @ c).max() <= 1e-11 * max(1.0, np.abs(A).max())
    assert np.abs(sigma - A.T @ c).max() <= 1e-11 * max(1.0, np.abs(A).max())
