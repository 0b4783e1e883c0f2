"""Generate the golden vectors of tests/golden/ by running the reference's own
per-step functions (compiled from its source by oracle/build.py into
oracle/_ref/libmorpho_ref.so) on small, seeded inputs.

    python tests/golden/make_golden.py

Each .npz holds its inputs (mesh, programmed fields, initial state) and the
reference's outputs, so the test that reads it needs neither the reference
tree nor the mesh generator to reproduce the inputs.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def deformed(model, seed):
    rng = np.random.default_rng(seed)
    N = model.num_nodes
    x = model.dofs(0).reshape(3, N).copy()
    x[2] += 0.05 * np.exp(-4.0 * (x[0] ** 2 + x[1] ** 2)) + 1e-3 * rng.standard_normal(N)
    x[0] *= 1.02
    x[1] += 0.01 * x[0] * x[1]
    return x.ravel(), 1e-3 * rng.standard_normal(3 * N)


def make(name: str, protocol: int, seed: int = 1, steps: int = 200) -> str:
    from morphoshell_b200 import Model, meshgen
    from oracle import Oracle

    mesh, info, bbar = meshgen.workload(name, seed=seed)
    if protocol == 1:
        info = meshgen.lce_abar_comps(info, 1.0)
        bbar = 0.2 * np.random.default_rng(seed + 100).standard_normal((mesh.num_tris, 3))
    d = tempfile.mkdtemp()
    st = os.path.join(d, "s.txt")
    meshgen.write_settings(st, protocol=protocol)
    m = Model.from_arrays(st, mesh.nodes, mesh.tris, info, bbar)
    s = m.scalars
    ref = Oracle("ref", m)
    x, v = deformed(m, seed)
    ref.set_programmed(protocol, info, bbar, s.dial_factors_to_hold_at_spacing)
    ref.upload(x, v)
    ref.do_dialling(0.5)
    abar, bbarv = ref.programmed()
    cq = ref.surface_derivs()
    forces_def, dE = ref.deformation_forces()
    ref.non_deformation_forces(s.damping_factor_1)
    ref.impose_constraints()
    forces = ref.forces()
    eq, eqv = ref.is_at_equilibrium()
    out = ref.output_quantities()
    # a short trajectory of full steps, dialling on
    x0 = m.dofs(1)
    ref.upload(x0)
    dials = s.dial_factors_to_hold_at_spacing * (np.arange(steps) / s.timesteps_per_dial_phase) + 0.3
    rc, done = ref.step_n(steps, dials, s.timestep, s.damping_factor_1)
    assert rc == 0
    xs, vs = ref.download()
    path = os.path.join(HERE, "%s_p%d.npz" % (name, protocol))
    np.savez_compressed(
        path, nodes=mesh.nodes, tris=mesh.tris, abar_info=info, bbar_info=bbar, protocol=protocol,
        state_x=x, state_v=v, dial=0.5, abar=abar, bbar=bbarv, cq=cq, dE=dE, forces_deformation=forces_def,
        forces=forces, equil=np.array([float(eq), *eqv]), curvatures=out["curvatures"],
        energy_densities=out["energy_densities"], strains=out["strains"], stresses=out["stresses"],
        angle_deficits=out["angle_deficits"], energies=out["energies"], traj_x0=x0, traj_dials=dials,
        traj_x=xs, traj_v=vs, timestep=s.timestep, damping=s.damping_factor_1)
    return path


if __name__ == "__main__":
    for p in (3, 1):
        print(make("disk100", p))
