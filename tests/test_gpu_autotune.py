"""Measured GEMM routes (DGEMM or tensor cores, K-split count): results with the tuner on stay within
the mixed-precision tolerance of the oracle, and routes saved to CCSD_GPU_TUNE_FILE are loaded by a
later process, which then repeats the first one's residual bit for bit."""

import os
import subprocess
import sys

import numpy as np
import pytest

from et_b200.synthetic import make_system
from oracle import ccsd as oc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from et_b200 import CCSD, MIXED
from et_b200.synthetic import make_system
s = make_system(8, 40, 100, seed=9)
with CCSD(8, 40, 100, precision=MIXED, autotune=1) as g:
    g.set_system(s.L_mo, s.h_mo, s.eps)
    g.set_initial_amplitudes_guess()
    np.save(sys.argv[2], g.construct_omega())
"""


@pytest.mark.parametrize("dims", [(8, 40, 100), (12, 60, 160)])
def test_autotuned_omega_close_to_oracle(dims):
    from et_b200 import CCSD, MIXED
    n_o, n_v, n_J = dims
    s = make_system(n_o, n_v, n_J, seed=9)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    ref.set_amplitudes(0.05 * np.random.default_rng(4).standard_normal(ref.n_amp))
    with CCSD(n_o, n_v, n_J, precision=MIXED, autotune=1) as gpu:
        gpu.set_system(s.L_mo, s.h_mo, s.eps)
        gpu.set_amplitudes(ref.get_amplitudes())
        om = gpu.construct_omega()
        om2 = gpu.construct_omega()
    om_ref = ref.omega()
    assert np.linalg.norm(om - om_ref) <= 1e-4 * np.linalg.norm(om_ref)
    # the second call takes the stored routes: same kernels, same rounding
    assert np.array_equal(om, om2)


def test_tune_file_routes_repeat_in_a_later_process(tmp_path):
    routes = tmp_path / "routes.txt"
    env = dict(os.environ, CCSD_GPU_TUNE_FILE=str(routes), CCSD_GPU_TRACE="1")
    out = []
    for name in ("first", "second"):
        r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT, str(tmp_path / f"{name}.npy")], env=env,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out.append(r.stderr)
    lines = [ln.split() for ln in routes.read_text().splitlines() if ln.strip()]
    assert lines and all(len(ln) == 2 and int(ln[1]) >= 0 for ln in lines)
    assert "ccsd_gpu tune" in out[0]        # the first process timed its shapes
    assert "ccsd_gpu tune" not in out[1]    # the second loaded every route
    a, b = np.load(tmp_path / "first.npy"), np.load(tmp_path / "second.npy")
    assert np.array_equal(a, b)
