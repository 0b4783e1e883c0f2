"""The cluster-tiled step (ms_set_step_path 0) against the
two-kernel step and the oracle, and the mixed-precision path's error against
FP64 -- GPU."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import deformed_state, make_model, rel_err

pytestmark = pytest.mark.gpu


def _loops(m, paths, precision=0):
    from morphoshell_b200 import GpuLoop
    s = m.scalars
    a_info, b_info = m.programmed()
    out = []
    for p in paths:
        g = GpuLoop(m, precision=precision)
        g.set_step_path(p)
        g.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
        out.append(g)
    return out


@pytest.mark.parametrize("name", ["disk100", "disk18k"])
def test_cluster_equals_two_kernel_bitwise_when_waiting(workdir, name):
    """Waiting-phase steps (programmed tensors read from memory): identical
    arithmetic and summation order on both paths, so identical bits."""
    m = make_model(workdir, name)
    s = m.scalars
    x, v = deformed_state(m, seed=21, amp=0.02)
    g0, g1 = _loops(m, [0, 1])
    for g in (g0, g1):
        g.upload(x, v)
        g.do_dialling(0.4)
        g.step_n(200, None, s.timestep, s.damping_factor_2)
    x0, v0 = g0.download()
    x1, v1 = g1.download()
    assert np.array_equal(x0, x1) and np.array_equal(v0, v1)
    info = g0.plan_info()
    assert info["path"] == 0 and info["cluster_size"] >= 1
    assert g1.plan_info()["path"] == 1


def test_cluster_dialling_matches_two_kernel(workdir):
    """Protocol-3 dialling in-kernel: both paths evaluate the same per-triangle
    code and sum in the same order, so they agree bitwise."""
    m = make_model(workdir, "disk18k")
    s = m.scalars
    x, v = deformed_state(m, seed=22, amp=0.02)
    g0, g1 = _loops(m, [0, 1])
    dials = 0.3 + 1e-5 * np.arange(300)
    for g in (g0, g1):
        g.upload(x, v)
        g.step_n(300, dials, s.timestep, s.damping_factor_1)
    x0, v0 = g0.download()
    x1, v1 = g1.download()
    assert np.array_equal(x0, x1) and np.array_equal(v0, v1)
    a0, _ = g0.programmed()
    a1, _ = g1.programmed()
    assert rel_err(a0, a1) < 1e-15


def test_cluster_equilibrium_and_guard(workdir):
    from morphoshell_b200 import MsError
    m = make_model(workdir, "disk18k")
    s = m.scalars
    x, v = deformed_state(m, seed=23, amp=0.02)
    g0, g1 = _loops(m, [0, 1])
    reps = []
    for g in (g0, g1):
        g.upload(x, v)
        g.do_dialling(0.2)
        reps.append(g.step_n(130, None, s.timestep, s.damping_factor_2, check_last=True))
    e0, e1 = reps[0].equil, reps[1].equil
    assert e0.max_force == e1.max_force and e0.max_speed == e1.max_speed
    assert e0.max_force_node == e1.max_force_node and e0.max_speed_node == e1.max_speed_node
    # guard: one node thrown far away
    xs, vs = g0.download()
    bad = xs.copy()
    bad[2 * m.num_nodes + 4321] += 1e6
    offs = []
    for g in (g0, g1):
        g.upload(bad, vs)
        with pytest.raises(MsError) as ei:
            g.step_n(10, None, s.timestep, s.damping_factor_2)
        offs.append((ei.value.report.error_step, ei.value.report.offending_dof))
        gx, _ = g.download()
        assert np.array_equal(gx, bad)
    assert offs[0] == offs[1] and offs[0][0] == 0


def test_cluster_plan_halo_fraction(workdir):
    from morphoshell_b200 import GpuLoop
    m = make_model(workdir, "disk18k")
    info = GpuLoop(m).plan_info()
    assert info["clusters"] * info["cluster_size"] * info["tris_per_cta"] >= m.num_tris
    assert 0 < info["halo_nodes"] < 0.35 * m.num_nodes


def test_mixed_precision_force_error(workdir):
    """Mixed path (strain formed in FP64, the rest of the per-triangle
    arithmetic and the contributions in FP32, FP64 node state): the per-step
    force, recovered from one velocity update, against FP64 on a deformed
    state whose largest nodal force is about 4 characteristic forces.  A
    float strain a - abar would give about 4e-6 here."""
    from morphoshell_b200 import MS_PRECISION_MIXED
    m = make_model(workdir, "disk18k")
    s = m.scalars
    mass = np.tile(m.tables()["node_mass"], 3)
    x, v = deformed_state(m, seed=24, amp=0.02)
    forces = []
    for prec in (0, MS_PRECISION_MIXED):
        g, = _loops(m, [1], precision=prec)
        g.upload(x, v)
        g.step_n(1, np.array([0.5]), s.timestep, 0.0)
        _, v1 = g.download()
        forces.append((v1 - v) * mass / s.timestep)
    err = rel_err(forces[1], forces[0])
    assert err < 1.5e-6, err
    cf = s.char_force_scale
    assert np.abs(forces[1] - forces[0]).max() / cf < 6e-6


def test_mixed_precision_force_error_against_oracle(workdir):
    """The mixed path's per-step force (recovered from one velocity update)
    against the FP64 oracle's forces on the same state
    (calc_deformation_forces.cpp:185 + calc_non_deformation_forces.cpp +
    impose_constraints.cpp), norm-wise."""
    from morphoshell_b200 import MS_PRECISION_MIXED
    from oracle import Oracle
    m = make_model(workdir, "disk18k")
    s = m.scalars
    a_info, b_info = m.programmed()
    mass = np.tile(m.tables()["node_mass"], 3)
    x, v = deformed_state(m, seed=24, amp=0.02)
    g, = _loops(m, [1], precision=MS_PRECISION_MIXED)
    g.upload(x, v)
    g.step_n(1, np.array([0.5]), s.timestep, 0.0)
    _, v1 = g.download()
    mixed = (v1 - v) * mass / s.timestep
    o = Oracle("orc", m)
    o.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
    o.upload(x, v)
    o.surface_derivs()
    o.do_dialling(0.5)
    o.deformation_forces()
    o.non_deformation_forces(0.0)
    o.impose_constraints()
    err = rel_err(mixed, o.forces())
    print("mixed-precision force error against the FP64 oracle: %.3e (norm-wise)" % err)
    assert err < 1.5e-6, err


def test_mixed_precision_equilibrium_shape(workdir):
    """Both precisions run the whole dialling schedule to the final
    equilibrium; shapes agree to well within 1e-5 of the mesh size (1), and
    the elastic energy of the mixed path's equilibrium, evaluated by the
    FP64 oracle (calc_energies.cpp:44-63), is within 1e-4 of the FP64
    path's (itself pinned to the oracle step by step)."""
    from morphoshell_b200 import MS_PRECISION_MIXED
    from oracle import Oracle
    m = make_model(workdir, "disk100", dial_factors_to_hold_at_spacing=0.5, dial_phase_time_prefactor=0.02,
                   force_to_char_force_ratio_equil_threshold=1e-5, speed_to_char_speed_ratio_equil_threshold=1e-4)
    s = m.scalars
    a_info, b_info = m.programmed()
    shapes, energies = [], []
    for prec in (0, MS_PRECISION_MIXED):
        r, x = m.run(max_steps=3_000_000, precision=prec)
        assert r.final_dial_factor == 1.0 and r.equilibria_reached >= 2, (r.final_dial_factor, r.equilibria_reached)
        shapes.append(x)
        o = Oracle("orc", m)
        o.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
        o.upload(x)
        o.do_dialling(1.0)
        e = o.output_quantities()["energies"]
        energies.append(e[0] + e[1])
    shape_err = np.abs(shapes[1] - shapes[0]).max()
    energy_err = abs(energies[1] - energies[0]) / abs(energies[0])
    print("mixed-precision equilibrium: shape error %.3e of the mesh size, elastic energy error %.3e"
          % (shape_err, energy_err))
    assert shape_err < 1e-5
    assert energy_err < 1e-4


@pytest.mark.parametrize("precision", [0, 1])
def test_tile_path_equals_two_kernel_bitwise(workdir, precision):
    """The bulk-copy-fed per-triangle kernel (path 2) reads the same tables
    from shared memory and runs the same arithmetic: identical bits, in
    dialling and in waiting steps, for both precisions."""
    m = make_model(workdir, "disk18k")
    s = m.scalars
    x, v = deformed_state(m, seed=25, amp=0.02)
    g1, g2 = _loops(m, [1, 2], precision=precision)
    dials = 0.2 + 1e-5 * np.arange(300)
    for g in (g1, g2):
        g.upload(x, v)
        g.step_n(300, dials, s.timestep, s.damping_factor_1)
        g.step_n(200, None, s.timestep, s.damping_factor_2)
    x1, v1 = g1.download()
    x2, v2 = g2.download()
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    assert g2.plan_info()["path"] == 2
