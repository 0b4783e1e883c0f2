"""Replica / ensemble distribution over ranks (morphoshell_b200.ensemble) with
the gloo backend on CPU, world size 2: every instance is stepped exactly once,
results equal a single-process run, and the ensemble time is the max over
ranks.  The per-instance stepper here is the CPU oracle (the GPU stepper runs
the same harness on the GPU box)."""
from __future__ import annotations

import os
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NAMES = ["disk100", "disk100", "disk50", "disk100"]


class OracleInstance:
    def __init__(self, i, workdir):
        import sys
        sys.path.insert(0, ROOT)
        from morphoshell_b200 import Model, meshgen
        from oracle import Oracle
        st, vtk = meshgen.write_workload(os.path.join(workdir, "inst%d" % i), NAMES[i], seed=10 + i)
        self.model = Model(st, vtk)
        s = self.model.scalars
        a, b = self.model.programmed()
        self.o = Oracle("orc", self.model, threads=1)
        self.o.set_programmed(3, a, b, s.dial_factors_to_hold_at_spacing)
        self.o.upload(self.model.dofs(1))
        self.num_tris = self.model.num_tris
        self.s = s

    def step(self, n):
        dials = 0.2 + 1e-4 * np.arange(n)
        rc, _ = self.o.step_n(n, dials, self.s.timestep, self.s.damping_factor_1)
        assert rc == 0

    def result(self):
        x, _ = self.o.download()
        return {"x": x}


def _worker(rank, world, port, workdir, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    from morphoshell_b200.ensemble import run_instances
    res, total = run_instances(lambda i: OracleInstance(i, workdir), len(NAMES), 40, dist=dist)
    if rank == 0:
        np.savez(out, x=np.concatenate([r.payload["x"] for r in res]), idx=[r.index for r in res],
                 ranks=[r.rank for r in res], total=total, secs=[r.seconds for r in res])
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_world2_matches_single_process():
    workdir = tempfile.mkdtemp()
    out = os.path.join(workdir, "res.npz")
    port = 29500 + (os.getpid() % 1000)
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, workdir, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    r = np.load(out)
    assert list(r["idx"]) == [0, 1, 2, 3]
    assert set(r["ranks"]) == {0, 1}
    from morphoshell_b200.ensemble import run_instances
    single, _ = run_instances(lambda i: OracleInstance(i, workdir), len(NAMES), 40)
    x1 = np.concatenate([s.payload["x"] for s in single])
    assert np.array_equal(r["x"], x1)
    # ensemble time is the slowest rank's total, at least any instance's time
    assert float(r["total"]) >= max(r["secs"]) - 1e-12


def test_assignment_balances_weights():
    from morphoshell_b200.ensemble import assign
    w = [100, 1, 1, 1, 50, 50]
    a0, a1 = assign(6, 2, 0, w), assign(6, 2, 1, w)
    assert sorted(a0 + a1) == list(range(6))
    l0, l1 = sum(w[i] for i in a0), sum(w[i] for i in a1)
    assert abs(l0 - l1) <= 100
