"""Independent instances across ranks (one process per GPU).

The loop has no data-path exchange between meshes: an ensemble of meshes
(different sizes, programmed fields, thicknesses) is split over the ranks of
a ``torch.distributed`` process group, every rank steps its own instances on
its own GPU, and rank 0 gathers the per-instance results.  The only
collectives are a barrier around the timed region, a MAX of the per-rank
device times (the slowest rank defines the ensemble's time) and the final
gather.  Ranks must all call these functions in the same order.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field


@dataclass
class InstanceResult:
    index: int
    rank: int
    num_tris: int
    steps: int
    seconds: float
    payload: dict = field(default_factory=dict)


def assign(num_instances: int, world: int, rank: int, weights=None):
    """Instances of this rank: greedy longest-processing-time assignment by
    weight (e.g. triangle count), deterministic on every rank."""
    if weights is None:
        return [i for i in range(num_instances) if i % world == rank]
    order = sorted(range(num_instances), key=lambda i: (-weights[i], i))
    load = [0.0] * world
    owner = [0] * num_instances
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += weights[i]
    return [i for i in range(num_instances) if owner[i] == rank]


def run_instances(make_instance, num_instances: int, steps: int, dist=None, weights=None, timer=None):
    """Step every instance of this rank ``steps`` times.

    ``make_instance(i)`` returns an object with ``num_tris``, ``step(n)``
    and ``result() -> dict``.  ``timer`` (optional) returns a (start, stop)
    pair of callables measuring device time in seconds; the default is the
    host clock.  Returns (results gathered on rank 0 or None elsewhere,
    ensemble seconds = max over ranks)."""
    world = dist.get_world_size() if dist else 1
    rank = dist.get_rank() if dist else 0
    mine = assign(num_instances, world, rank, weights)
    insts = [(i, make_instance(i)) for i in mine]
    if dist:
        dist.barrier()
    results = []
    total = 0.0
    for i, inst in insts:
        if timer:
            start, stop = timer()
            start()
            inst.step(steps)
            sec = stop()
        else:
            t0 = time.perf_counter()
            inst.step(steps)
            sec = time.perf_counter() - t0
        total += sec
        results.append(InstanceResult(i, rank, inst.num_tris, steps, sec, inst.result()))
    if dist:
        import torch
        dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
        t = torch.tensor([total], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(results, gathered, dst=0)
        if rank == 0:
            results = sorted((r for part in gathered for r in part), key=lambda r: r.index)
        else:
            results = None
    return results, total


def _member_arrays(args):
    from . import meshgen
    k, seed, spacing_range = args
    mesh, info, bbar, over, params = meshgen.ensemble_member(k, seed=seed, spacing_range=spacing_range)
    return mesh.nodes, mesh.tris, info, bbar, over, params


def build_members(indices, directory: str, seed: int = 7, spacing_range=(0.004, 0.02), threads: int = 8,
                  processes: int = 0, **settings):
    """Host set-up (Model.from_arrays) of the batched-ensemble members
    ``indices`` (meshgen.ensemble_member).  Meshes are generated in
    ``processes`` spawned worker processes (0: in the calling process) and
    set up in ``threads`` threads (the native set-up releases the GIL).
    Extra keyword arguments override settings of every member.  Returns
    (models, parameters)."""
    import multiprocessing as mp
    import os
    from concurrent.futures import ProcessPoolExecutor, ThreadPoolExecutor

    from . import Model, meshgen

    os.makedirs(directory, exist_ok=True)
    jobs = [(k, seed, spacing_range) for k in indices]
    if processes > 0:
        with ProcessPoolExecutor(max_workers=processes, mp_context=mp.get_context("spawn")) as ex:
            arrays = list(ex.map(_member_arrays, jobs))
    else:
        with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
            arrays = list(ex.map(_member_arrays, jobs))

    def one(item):
        k, (nodes, tris, info, bbar, over, params) = item
        st = os.path.join(directory, "member%05d_settings.txt" % k)
        meshgen.write_settings(st, protocol=3, **dict(over, **settings))
        model = Model.from_arrays(st, nodes, tris, info, bbar, quiet=True, noise=True)
        params = dict(params, num_tris=model.num_tris)
        return model, params

    with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        out = list(ex.map(one, zip(list(indices), arrays)))
    return [m for m, _ in out], [p for _, p in out]
