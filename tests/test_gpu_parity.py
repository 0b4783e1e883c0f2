"""GPU path (C ABI of include/morphoshell_gpu.h) against the CPU oracle.

Tolerances are the stated ones for this path: per-step forces within 1e-12
relative (norm-wise, max|dF| / max|F|) on well-conditioned deformed states,
node positions within 1e-9 relative after 10^4 steps.  The oracle is the
project's restatement (oracle/morpho_oracle.cpp), itself pinned against the
reference compiled from source (tests/test_oracle_pin.py, tests/golden/).
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import check_forces_to_rounding, deformed_state, make_model, protocol_inputs, rel_err

FORCE_RTOL = 1e-12
POS_RTOL = 1e-9

pytestmark = pytest.mark.gpu


def _pair(workdir, name="disk100", protocol=3, dial=0.5, seed=0, precision=0):
    from morphoshell_b200 import GpuLoop
    from oracle import Oracle
    m = make_model(workdir, name)
    a_info, b_info = m.programmed()
    g = GpuLoop(m, precision=precision)
    o = Oracle("orc", m)
    x, v = deformed_state(m, seed=seed)
    for s in (g, o):
        s.set_programmed(protocol, a_info, b_info, m.scalars.dial_factors_to_hold_at_spacing)
        s.upload(x, v)
        s.do_dialling(dial)
    return m, g, o, x, v


@pytest.mark.parametrize("name", ["disk100", "disk50", "disk18k"])
def test_surface_derivs_and_forces(workdir, name):
    m, g, o, x, v = _pair(workdir, name)
    ga, gb = g.programmed()
    oa, ob = o.programmed()
    assert rel_err(ga, oa) < 1e-14
    assert rel_err(gb, ob) == 0.0 or np.abs(gb - ob).max() < 1e-300
    assert rel_err(g.surface_derivs(), o.surface_derivs()) < 1e-13
    gf, gde = g.deformation_forces()
    of, ode = o.deformation_forces()
    assert rel_err(gde, ode) < FORCE_RTOL
    assert rel_err(gf, of) < FORCE_RTOL


def test_damping_constraints_equilibrium(workdir):
    m, g, o, x, v = _pair(workdir, "disk50")
    s = m.scalars
    for t in (g, o):
        t.surface_derivs()
        t.deformation_forces()
        t.non_deformation_forces(s.damping_factor_1)
        t.impose_constraints()
    assert rel_err(g.forces(), o.forces()) < FORCE_RTOL
    ge = g.is_at_equilibrium()
    oeq, oe = o.is_at_equilibrium()
    assert abs(ge.max_force - oe[0]) <= 1e-12 * oe[0]
    assert ge.max_speed == oe[1]
    assert ge.max_force_node == int(oe[2]) and ge.max_speed_node == int(oe[3])
    assert bool(ge.at_equilibrium) == oeq


def test_advance_dynamics(workdir):
    m, g, o, x, v = _pair(workdir, "disk50")
    s = m.scalars
    for t in (g, o):
        t.surface_derivs()
        t.deformation_forces()
        t.non_deformation_forces(s.damping_factor_1)
        t.impose_constraints()
        t.advance_dynamics(s.timestep, s.damping_factor_1)
    gx, gv = g.download()
    ox, ov = o.download()
    assert rel_err(gx, ox) < 1e-15
    assert rel_err(gv, ov) < 1e-12


@pytest.mark.parametrize("protocol", [1, 2, 3, 4, 5])
def test_dialling_protocols(workdir, protocol):
    """do_dialling.cpp's protocols (4: lambda interpolated between eleven
    per-triangle checkpoints, do_dialling.cpp:128-153), from the reference
    state and from an ansatz, against the oracle."""
    from morphoshell_b200 import GpuLoop
    from oracle import Oracle
    m = make_model(workdir, "disk100")
    T = m.num_tris
    a_info, b_info, spacing = protocol_inputs(m, protocol)
    g, o = GpuLoop(m), Oracle("orc", m)
    rng = np.random.default_rng(7)
    a0 = np.column_stack([1 + 0.1 * rng.random(T), 0.05 * rng.random(T), 1 + 0.1 * rng.random(T)])
    b0 = 0.1 * rng.standard_normal((T, 3))
    for from_ansatz in (False, True):
        for t in (g, o):
            t.set_programmed(protocol, a_info, b_info, spacing, from_ansatz)
            t.set_zero_dial_state(a0, b0)
        for dial in (0.0, 0.3, 0.55, 0.97, 1.0):
            g.do_dialling(dial)
            o.do_dialling(dial)
            ga, gb = g.programmed()
            oa, ob = o.programmed()
            assert rel_err(ga, oa) < 1e-14, (protocol, from_ansatz, dial)
            assert np.abs(gb - ob).max() <= 1e-14 * max(1.0, np.abs(ob).max())


def test_a_b_normals(workdir):
    """calc_a_comps_and_b_comps_and_normals.cpp:27-62 (the metric a, the
    second fundamental form b and the unit normal of every triangle), as
    called at step 0 when dialling from an ansatz (main.cpp:320-329)."""
    m, g, o, x, v = _pair(workdir, "disk18k")
    g.surface_derivs()
    o.surface_derivs()
    ga, gb, gn = g.a_b_normals()
    oa, ob, on = o.a_b_normals()
    # a = R_a . R_b from derivatives formed as weighted sums of positions
    # (weights ~ 1 / spacing): rounding of 1e-14 relative, as for cq itself.
    assert rel_err(ga, oa) < 1e-13
    assert rel_err(gb, ob) < 1e-12
    assert rel_err(gn, on) < 1e-13
    assert np.allclose(np.linalg.norm(gn, axis=1), 1.0, atol=1e-14)


def test_fused_step_matches_per_function_path(workdir):
    """ms_step_n (the fused step) against the one-call-per-function
    sequence on the same device: same state after 50 steps."""
    from morphoshell_b200 import GpuLoop
    m = make_model(workdir, "disk50")
    s = m.scalars
    a_info, b_info = m.programmed()
    x, v = deformed_state(m, seed=2, amp=0.02)
    g1, g2 = GpuLoop(m), GpuLoop(m)
    dials = 0.2 + 1e-4 * np.arange(50)
    for g in (g1, g2):
        g.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
        g.upload(x, v)
    g1.step_n(50, dials, s.timestep, s.damping_factor_1)
    for i in range(50):
        g2.surface_derivs()
        g2.do_dialling(dials[i])
        g2.deformation_forces()
        g2.non_deformation_forces(s.damping_factor_1)
        g2.impose_constraints()
        g2.advance_dynamics(s.timestep, s.damping_factor_1)
    x1, v1 = g1.download()
    x2, v2 = g2.download()
    assert rel_err(x1, x2) < 1e-13
    assert rel_err(v1, v2) < 1e-10


_trajectories = {}


def _oracle_trajectory(workdir, name, n):
    """The oracle's state after n dialling steps from the noisy flat start
    (step k dials to dial_factors_to_hold_at_spacing * k /
    timesteps_per_dial_phase, main.cpp:478-488), with its final forces;
    computed once per mesh."""
    from oracle import Oracle
    if (name, n) not in _trajectories:
        m = make_model(workdir, name)
        s = m.scalars
        a_info, b_info = m.programmed()
        dials = s.dial_factors_to_hold_at_spacing * (np.arange(n) / s.timesteps_per_dial_phase)
        o = Oracle("orc", m, threads=os.cpu_count())
        o.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
        o.upload(m.dofs(1))
        rc, done = o.step_n(n, dials, s.timestep, s.damping_factor_1)
        assert rc == 0 and done == n
        _trajectories[(name, n)] = (o.download(), dials)
        o.close()
    return _trajectories[(name, n)]


@pytest.mark.parametrize("name,path", [("disk100", 2), ("disk100", 3), ("disk18k", 2), ("disk18k", 3)])
def test_fused_steps_vs_oracle_1e4(workdir, name, path):
    """10^4 fused dialling steps from the flat, noisy initial state against the
    oracle, on the two-kernel and on the node-tiled step: node positions
    within 1e-9 relative.  disk18k is the 18k-triangle disk with its own
    settings (azimuthal director, lambda 1 -> 0.9, 20 dial phases, h = 0.01,
    nu = 0.5).  Forces on the state reached are compared too: the GPU's
    deformation forces on the GPU's final state against the oracle's on the
    same state -- a state close to flat, where forces are rounding-dominated
    in every double-precision evaluation, so the bar is the reference's own
    distance from the oracle there (check_forces_to_rounding)."""
    from morphoshell_b200 import GpuLoop
    from oracle import Oracle
    m = make_model(workdir, name)
    s = m.scalars
    a_info, b_info = m.programmed()
    n = 10000
    (ox, ov), dials = _oracle_trajectory(workdir, name, n)
    g = GpuLoop(m)
    g.set_step_path(path)
    g.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
    g.upload(m.dofs(1))
    g.step_n(n, dials, s.timestep, s.damping_factor_1)
    gx, gv = g.download()
    assert np.isfinite(gx).all()
    assert rel_err(gx, ox) < POS_RTOL
    assert np.abs(gx - m.dofs(1)).max() > 0  # it moved
    # per-step forces on the state the dynamics reached
    g.upload(gx, gv)
    g.surface_derivs()
    g.do_dialling(dials[-1])
    gf, _ = g.deformation_forces()
    errs = check_forces_to_rounding(m, gx, gv, dials[-1], gf, FORCE_RTOL, threads=os.cpu_count())
    print("%s path %d: forces after 10^4 steps, GPU vs oracle %.2e, reference vs oracle %s, GPU vs reference %s"
          % (name, path, errs[0], errs[1], errs[2]))


def test_bitwise_determinism(workdir):
    from morphoshell_b200 import GpuLoop
    m = make_model(workdir, "disk18k")
    s = m.scalars
    a_info, b_info = m.programmed()
    x, v = deformed_state(m, seed=4, amp=0.01)
    outs = []
    for _ in range(2):
        g = GpuLoop(m)
        g.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
        g.upload(x, v)
        g.step_n(300, np.full(300, 0.3), s.timestep, s.damping_factor_1)
        outs.append(g.download())
        g.close()
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_force_guard_reports_first_offender(workdir):
    """A node placed far away produces an implausible force; the fused stepper
    stops before that step and reports the first offending dof, like
    advance_dynamics.cpp:58-73 (fault made on the host, not on the GPU)."""
    from morphoshell_b200 import GpuLoop, MsError
    from oracle import Oracle
    m = make_model(workdir, "disk50")
    s = m.scalars
    a_info, b_info = m.programmed()
    x, v = deformed_state(m, seed=5, amp=0.01)
    g = GpuLoop(m)
    g.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
    g.upload(x, v)
    g.step_n(5, np.full(5, 0.1), s.timestep, s.damping_factor_1)
    xs, vs = g.download()
    bad = xs.copy()
    N = m.num_nodes
    bad[2 * N + 17] += 1e6
    g.upload(bad, vs)
    with pytest.raises(MsError) as ei:
        g.step_n(20, np.full(20, 0.1), s.timestep, s.damping_factor_1)
    rep = ei.value.report
    assert rep.error_step == 0
    o = Oracle("orc", m)
    o.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
    o.upload(bad, vs)
    o.surface_derivs()
    o.do_dialling(0.1)
    o.deformation_forces()
    o.non_deformation_forces(s.damping_factor_1)
    o.impose_constraints()
    rc, dof, f = o.advance_dynamics(s.timestep, s.damping_factor_1)
    assert rc == 3 and rep.offending_dof == dof
    # A node 1e6 away makes terms of ~1e6 cancel down to ~1e3: rounding-level
    # agreement here is ~1e-11, not 1e-12.
    assert abs(rep.offending_force - f) <= 1e-9 * abs(f)
    # state is the one before the failing step
    gx, gv = g.download()
    assert np.array_equal(gx, bad)


def test_output_quantities(workdir):
    m, g, o, x, v = _pair(workdir, "disk100")
    go, oo = g.output_quantities(), o.output_quantities()
    assert rel_err(go["curvatures"], oo["curvatures"]) < 1e-11
    assert rel_err(go["energy_densities"], oo["energy_densities"]) < 1e-12
    assert rel_err(go["strains"], oo["strains"]) < 1e-12
    assert rel_err(go["angle_deficits"], oo["angle_deficits"]) < 1e-13
    assert rel_err(go["energies"], oo["energies"]) < 1e-13
    # eigenvalues exactly comparable, eigenvectors up to sign
    gs, os_ = go["stresses"], oo["stresses"]
    assert rel_err(gs[:, [0, 4]], os_[:, [0, 4]]) < 1e-11
    for c in (slice(1, 4), slice(5, 8)):
        dots = np.abs(np.sum(gs[:, c] * os_[:, c], axis=1))
        assert np.all(np.abs(dots - 1.0) < 1e-9)
