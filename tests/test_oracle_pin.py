"""Pins the CPU oracle (oracle/morpho_oracle.cpp) to the reference -- CPU only.

1. Against the golden vectors of tests/golden/, produced by the reference's
   own per-step functions compiled from source (tests/golden/make_golden.py).
2. Live against the same compiled reference (oracle/_ref) where it was built.

Tolerances: 1e-12 relative (norm-wise) on per-step forces and dE/dcq on
well-conditioned deformed states; 1e-9 relative on positions after 10^4
steps.  The two implementations group the same double-precision sums
differently (the reference expands its energy derivatives, the oracle
differentiates the energy by dual numbers), so agreement is to rounding,
not bitwise.
"""
from __future__ import annotations

import glob
import os
import tempfile

import numpy as np
import pytest

from conftest import deformed_state, make_model, protocol_inputs, rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
# The per-function golden vectors (make_golden.py); disk1p8m_traj.npz is the
# GPU trajectory fixture of tests/test_gpu_disk1p8m_trajectory.py.
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*_p[0-9].npz")))


def _golden_model(g):
    from morphoshell_b200 import Model, meshgen
    d = tempfile.mkdtemp()
    st = os.path.join(d, "s.txt")
    meshgen.write_settings(st, protocol=int(g["protocol"]))
    return Model.from_arrays(st, g["nodes"], g["tris"], g["abar_info"], g["bbar_info"])


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_against_golden(path):
    from oracle import Oracle
    g = np.load(path)
    m = _golden_model(g)
    s = m.scalars
    o = Oracle("orc", m)
    o.set_programmed(int(g["protocol"]), g["abar_info"], g["bbar_info"], s.dial_factors_to_hold_at_spacing)
    o.upload(g["state_x"], g["state_v"])
    o.do_dialling(float(g["dial"]))
    a, b = o.programmed()
    assert rel_err(a, g["abar"]) < 1e-15
    assert np.abs(b - g["bbar"]).max() <= 1e-15 * max(1.0, np.abs(g["bbar"]).max())
    assert rel_err(o.surface_derivs(), g["cq"]) < 1e-13
    f, de = o.deformation_forces()
    assert rel_err(de, g["dE"]) < 1e-12
    assert rel_err(f, g["forces_deformation"]) < 1e-12
    o.non_deformation_forces(s.damping_factor_1)
    o.impose_constraints()
    assert rel_err(o.forces(), g["forces"]) < 1e-12
    eq, ev = o.is_at_equilibrium()
    assert float(eq) == g["equil"][0]
    assert rel_err(ev[:2], g["equil"][1:3]) < 1e-12
    assert np.array_equal(ev[2:], g["equil"][3:])
    out = o.output_quantities()
    for k in ("curvatures", "energy_densities", "strains", "angle_deficits", "energies"):
        assert rel_err(out[k], g[k]) < 1e-11, k
    st_o, st_g = out["stresses"], g["stresses"]
    assert rel_err(st_o[:, [0, 4]], st_g[:, [0, 4]]) < 1e-11
    for c in (slice(1, 4), slice(5, 8)):
        assert np.all(np.abs(np.abs(np.sum(st_o[:, c] * st_g[:, c], axis=1)) - 1.0) < 1e-9)
    o.upload(g["traj_x0"])
    rc, done = o.step_n(len(g["traj_dials"]), g["traj_dials"], float(g["timestep"]), float(g["damping"]))
    assert rc == 0
    x, v = o.download()
    assert rel_err(x, g["traj_x"]) < 1e-12
    assert rel_err(v, g["traj_v"]) < 1e-9


def _need_ref():
    import oracle
    if not oracle.available("ref"):
        pytest.skip("reference build absent (oracle/_ref)")


@pytest.mark.parametrize("name,seed", [("disk50", 0), ("disk50", 1), ("disk18k", 2)])
def test_oracle_against_reference_live(workdir, name, seed):
    _need_ref()
    from oracle import Oracle
    m = make_model(workdir, name)
    s = m.scalars
    a_info, b_info = m.programmed()
    o, r = Oracle("orc", m), Oracle("ref", m)
    x, v = deformed_state(m, seed=seed)
    for t in (o, r):
        t.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
        t.upload(x, v)
        t.do_dialling(0.25 + 0.25 * seed)
    assert rel_err(o.surface_derivs(), r.surface_derivs()) < 1e-13
    fo, do = o.deformation_forces()
    fr, dr = r.deformation_forces()
    assert rel_err(do, dr) < 1e-12
    assert rel_err(fo, fr) < 1e-12


def test_trajectory_1e4_steps_against_reference(workdir):
    """10^4 dialling steps from the noisy flat start (the start of the
    18k-disk workload's first dial phase, on the small disk): positions
    within 1e-9 relative."""
    _need_ref()
    from oracle import Oracle
    m = make_model(workdir, "disk100")
    s = m.scalars
    a_info, b_info = m.programmed()
    n = 10000
    dials = s.dial_factors_to_hold_at_spacing * (np.arange(n) / s.timesteps_per_dial_phase)
    res = []
    for kind in ("orc", "ref"):
        t = Oracle(kind, m)
        t.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
        t.upload(m.dofs(1))
        rc, done = t.step_n(n, dials, s.timestep, s.damping_factor_1)
        assert rc == 0 and done == n
        res.append(t.download())
    assert rel_err(res[0][0], res[1][0]) < 1e-9
    assert np.abs(res[0][0] - m.dofs(1)).max() > 0  # it moved


@pytest.mark.parametrize("proto", [1, 2, 3, 4, 5])
def test_dialling_protocols_and_ansatz_dialling_against_reference(workdir, proto):
    """Every dialling protocol of do_dialling.cpp (the reference's own file,
    compiled once per protocol with that protocol's block switched on), with
    and without dialling from an ansatz."""
    _need_ref()
    from oracle import Oracle
    m = make_model(workdir, "disk100")
    T = m.num_tris
    ai, bi, spacing = protocol_inputs(m, proto)
    rng = np.random.default_rng(1)
    a0 = np.column_stack([1 + 0.1 * rng.random(T), 0.05 * rng.random(T), 1 + 0.1 * rng.random(T)])
    b0 = 0.1 * rng.standard_normal((T, 3))
    for ansatz in (False, True):
        o, r = Oracle("orc", m), Oracle("ref", m)
        for t in (o, r):
            t.set_programmed(proto, ai, bi, spacing, ansatz)
            t.set_zero_dial_state(a0, b0)
        for dial in (0.0, 0.3, 0.37, 0.55, 1.0):
            o.do_dialling(dial)
            r.do_dialling(dial)
            ao, bo = o.programmed()
            ar, br = r.programmed()
            assert rel_err(ao, ar) < 1e-15, (proto, ansatz, dial)
            assert np.abs(bo - br).max() <= 1e-15 * max(1.0, np.abs(br).max())


def test_force_guard_against_reference(workdir):
    _need_ref()
    from oracle import Oracle
    m = make_model(workdir, "disk50")
    s = m.scalars
    a_info, b_info = m.programmed()
    x, v = deformed_state(m, seed=3)
    N = m.num_nodes
    x = x.copy()
    x[N + 11] += 1e5
    outs = []
    for kind in ("orc", "ref"):
        t = Oracle(kind, m)
        t.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
        t.upload(x, v)
        t.surface_derivs()
        t.do_dialling(0.1)
        t.deformation_forces()
        t.non_deformation_forces(s.damping_factor_1)
        t.impose_constraints()
        outs.append(t.advance_dynamics(s.timestep, s.damping_factor_1))
        xs, _ = t.download()
        assert np.array_equal(xs, x)  # nothing moved
    assert outs[0][0] == outs[1][0] == 3
    assert outs[0][1] == outs[1][1]
    assert abs(outs[0][2] - outs[1][2]) <= 1e-12 * abs(outs[1][2])
