"""Multi-process replica path (one system per rank, no data-path collective) on CPU with gloo.

The benchmark's multi-GPU mode runs independent systems per rank and reduces only the timing
(max over ranks) and the per-rank results; this test runs that pattern with world_size 2 on the
CPU oracle so the host logic is covered without GPUs.
"""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from et_b200.synthetic import make_system
    from oracle import ccsd as oc
    sizes = [2, 3, 2, 3]
    energies = torch.zeros(len(sizes), dtype=torch.float64)
    for k in range(rank, len(sizes), world):          # replicas: systems striped over ranks
        o = sizes[k]
        s = make_system(o, 4 * o, 6 * o, seed=2026 + k)
        sy = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
        sy.mp2_start()
        e, _, conv = oc.solve_gs(sy, omega_threshold=1e-9, energy_threshold=1e-11)
        assert conv
        energies[k] = e
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)          # max-over-ranks timing reduction
    dist.all_reduce(energies, op=dist.ReduceOp.SUM)   # gather the per-system results
    if rank == 0:
        out.put((float(t.item()), energies.numpy().tolist()))
    dist.destroy_process_group()


def test_replicas_world_size_2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    tmax, energies = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert tmax == 2.0
    # every system was solved exactly once and matches a serial solve
    from et_b200.synthetic import make_system
    from oracle import ccsd as oc
    for k, o in enumerate([2, 3, 2, 3]):
        s = make_system(o, 4 * o, 6 * o, seed=2026 + k)
        sy = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
        sy.mp2_start()
        e, _, _ = oc.solve_gs(sy, omega_threshold=1e-9, energy_threshold=1e-11)
        assert abs(energies[k] - e) < 1e-12
