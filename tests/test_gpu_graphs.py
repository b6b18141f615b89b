"""Residual evaluations replayed from captured CUDA graphs: bit for bit the eager result in both
precisions, reading new amplitudes in place, re-captured when the Cholesky vectors change, and used
by the ground-state solver and the batch executor."""

import numpy as np
import pytest

from et_b200.synthetic import make_system

pytestmark = pytest.mark.gpu


def _pair(prec, dims=(6, 30, 80), seed=3):
    from et_b200 import CCSD
    s = make_system(*dims, seed=seed)
    g, e = CCSD(*dims, precision=prec), CCSD(*dims, precision=prec)
    g.set_graphs(True)
    e.set_graphs(False)
    for c in (g, e):
        c.set_system(s.L_mo, s.h_mo, s.eps)
        c.set_initial_amplitudes_guess()
    return s, g, e


@pytest.mark.parametrize("prec_name", ["FP64", "MIXED"])
def test_replayed_residual_equals_eager(prec_name):
    import et_b200
    prec = getattr(et_b200, prec_name)
    s, g, e = _pair(prec)
    ref = e.construct_omega()
    outs = [g.construct_omega() for _ in range(3)]
    replays, _ = g.graph_stats()
    assert replays == 2          # the first evaluation runs eagerly, then capture + launch, then replay
    assert e.graph_stats()[0] == 0
    for o in outs:
        assert np.array_equal(o, ref)
    # new amplitudes are read in place by the same graph
    t = 0.02 * np.random.default_rng(1).standard_normal(g.n_amp)
    g.set_amplitudes(t)
    e.set_amplitudes(t)
    assert np.array_equal(g.construct_omega(), e.construct_omega())
    assert g.graph_stats()[0] == 3
    # new Cholesky vectors: the graph is captured again for the new caches
    L2 = s.L_mo * 1.01
    for c in (g, e):
        c.set_cholesky_mo(L2)
        c.set_amplitudes(t)
    for _ in range(2):
        assert np.array_equal(g.construct_omega(), e.construct_omega())
    assert g.graph_stats()[0] == 5
    g.close()
    e.close()


def test_device_output_pointer_may_change():
    import torch
    from et_b200 import MIXED
    s, g, e = _pair(MIXED)
    ref = e.construct_omega()
    bufs = [torch.empty(g.n_amp, dtype=torch.float64, device="cuda") for _ in range(3)]
    for b in bufs:
        g.construct_omega_device(b.data_ptr())
    g.synchronize()
    for b in bufs:
        assert np.array_equal(b.cpu().numpy(), ref)
    g.close()
    e.close()


@pytest.mark.parametrize("prec_name", ["FP64", "MIXED"])
def test_solver_with_graphs_matches_eager_solver(prec_name):
    import et_b200
    prec = getattr(et_b200, prec_name)
    s, g, e = _pair(prec, dims=(8, 40, 100), seed=5)
    res = []
    for c in (g, e):
        res.append(c.solve_ground_state(omega_threshold=1e-8, energy_threshold=1e-10))
    (eg, itg, hg, _), (ee, ite, he, _) = res
    assert itg == ite and eg == ee
    assert np.array_equal(hg, he)
    assert g.graph_stats()[0] > 0
    assert np.array_equal(g.get_amplitudes(), e.get_amplitudes())
    g.close()
    e.close()
