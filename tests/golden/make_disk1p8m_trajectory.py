"""Generate tests/golden/disk1p8m_traj.npz: the reference's own per-step
functions (oracle/_ref/libmorpho_ref.so, compiled from its source by
oracle/build.py) run for 10^4 fixed dialling steps on the 1.8M-triangle disk.

    python tests/golden/make_disk1p8m_trajectory.py [--threads K] [--steps 10000]

Workload: ``meshgen.write_workload(dir, "disk1p8m")`` -- unit disk, jittered
hex spacing 0.002 (908,139 nodes, 1,813,134 triangles), wavy azimuthal
director (theta + pi/2 + 0.3 sin 3 theta), lambda 1 -> 0.85, bbar = 0,
h = 0.01, nu = 0.5, the reference's initial noise (``Model(..., noise=True)``,
perturb_node_positions_with_noise.cpp:50-61).  Step k dials to
dial_factors_to_hold_at_spacing * k / timesteps_per_dial_phase, as the
reference's dialling phase does (main.cpp:478-488); the sequence per step is
main.cpp:308-488 (surface derivatives, protocol-3 dialling, deformation
forces, damping, constraints, force guard, symplectic Euler).

The whole final state (0.9M nodes) is too large to commit, so the file holds
a seeded sample of 65,536 nodes (positions and velocities after the last
step), the global maxima of the last step (max |F| and max |v| over all nodes
with their nodes, is_at_equilibrium.cpp:62-90), the largest |z| over all
nodes with its node, and a fingerprint of the mesh and initial state so the
test can check it rebuilt the same inputs.  The test runs on a GPU box where
this reference tree is absent; it reads only this file.
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile
import time
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "disk1p8m_traj.npz")
SAMPLE = 65536
SAMPLE_SEED = 20261204


def fingerprint(model) -> np.ndarray:
    """(N, T, crc32 of the patch ids, sum of the initial dofs, sum of their
    squares, sum of the triangle areas): identifies the mesh, its set-up and
    the initial noise."""
    tb = model.tables()
    x0 = model.dofs(1)
    crc = zlib.crc32(np.ascontiguousarray(tb["patch_ids"], dtype=np.int32).tobytes())
    return np.array([model.num_nodes, model.num_tris, crc, float(np.sum(x0)), float(np.sum(x0 * x0)),
                     float(np.sum(tb["ref_area"]))], dtype=np.float64)


def sample_nodes(num_nodes: int) -> np.ndarray:
    rng = np.random.default_rng(SAMPLE_SEED)
    return np.sort(rng.choice(num_nodes, size=min(SAMPLE, num_nodes), replace=False)).astype(np.int64)


def dial_schedule(scalars, steps: int) -> np.ndarray:
    k = np.arange(steps)
    return scalars.dial_factors_to_hold_at_spacing * (k / scalars.timesteps_per_dial_phase)


def main() -> None:
    from morphoshell_b200 import Model, meshgen
    from oracle import Oracle

    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--kind", default="ref", choices=["ref", "orc"])
    a = ap.parse_args()
    t0 = time.time()
    d = tempfile.mkdtemp(prefix="disk1p8m_traj_")
    st, vtk = meshgen.write_workload(d, "disk1p8m")
    m = Model(st, vtk, quiet=True)
    s = m.scalars
    info, bbar = m.programmed()
    print("set-up %.1f s: N=%d T=%d" % (time.time() - t0, m.num_nodes, m.num_tris), flush=True)
    o = Oracle(a.kind, m, threads=a.threads)
    o.set_programmed(3, info, bbar, s.dial_factors_to_hold_at_spacing)
    x0 = m.dofs(1)
    o.upload(x0)
    dials = dial_schedule(s, a.steps)
    t1 = time.time()
    done_total = 0
    chunk = 500
    while done_total < a.steps:
        n = min(chunk, a.steps - done_total)
        rc, done = o.step_n(n, dials[done_total:done_total + n], s.timestep, s.damping_factor_1)
        if rc != 0 or done != n:
            raise RuntimeError("oracle stopped at step %d (status %d)" % (done_total + done, rc))
        done_total += n
        el = time.time() - t1
        print("%d steps, %.0f s, %.3g tri-steps/s" % (done_total, el, m.num_tris * done_total / el), flush=True)
    x, v = o.download()
    eq, eqv = o.is_at_equilibrium()
    N = m.num_nodes
    idx = sample_nodes(N)
    z = x[2 * N:]
    zmax_node = int(np.argmax(np.abs(z)))
    np.savez_compressed(
        OUT, steps=a.steps, kind=a.kind, fingerprint=fingerprint(m), sample=idx,
        x=np.stack([x[idx], x[N + idx], x[2 * N + idx]]), v=np.stack([v[idx], v[N + idx], v[2 * N + idx]]),
        equil=np.array(eqv, dtype=np.float64), zmax=np.array([zmax_node, z[zmax_node]]),
        abs_max=np.array([np.abs(x).max(), np.abs(v).max()]), timestep=s.timestep, damping=s.damping_factor_1,
        dial_last=dials[-1], tps_reference=m.num_tris * a.steps / (time.time() - t1), threads=a.threads)
    print("wrote %s in %.0f s" % (OUT, time.time() - t0))


if __name__ == "__main__":
    main()
