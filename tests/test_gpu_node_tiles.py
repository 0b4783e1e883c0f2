"""The node-tiled one-kernel steps (ms_set_step_path 3, and 4 with
warp-specialised roles, on the plan built for it) against the two-kernel
step -- GPU.

Paths 3 and 4 compute each triangle with the same arithmetic as the
bulk-copy per-triangle kernel and sum every node's contributions in
ascending triangle order from zero, as the node kernel does, so all give
the same bits (calc_deformation_forces.cpp:185 is the sum they restate)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import deformed_state, make_model

pytestmark = pytest.mark.gpu


def new_loop(m, path, precision=0):
    """A handle whose plan serves `path`: the warp-specialised step (4) needs
    the plan built for it (MSB_NODE_TILE_PLAN=4 when the handle is made)."""
    from morphoshell_b200 import GpuLoop
    if path == 4:
        os.environ["MSB_NODE_TILE_PLAN"] = "4"
    try:
        g = GpuLoop(m, precision=precision)
    finally:
        os.environ.pop("MSB_NODE_TILE_PLAN", None)
    g.set_step_path(path)
    return g


def _loops(m, paths, precision=0, protocol=3, a_info=None, b_info=None):
    s = m.scalars
    if a_info is None:
        a_info, b_info = m.programmed()
    out = []
    for p in paths:
        g = new_loop(m, p, precision)
        g.set_programmed(protocol, a_info, b_info, s.dial_factors_to_hold_at_spacing)
        out.append(g)
    return out


def _run(gs, x, v, m, dial_steps=300, wait_steps=200, check=True):
    s = m.scalars
    dials = 0.2 + 1e-5 * np.arange(dial_steps)
    reps = []
    for g in gs:
        g.upload(x, v)
        g.step_n(dial_steps, dials, s.timestep, s.damping_factor_1)
        reps.append(g.step_n(wait_steps, None, s.timestep, s.damping_factor_2, check_last=check))
    return reps


@pytest.mark.parametrize("path", [3, 4])
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["disk18k", "disk100"])
def test_node_tiles_equal_two_kernel_bitwise(workdir, precision, name, path):
    """Dialling steps (protocol 3 in-kernel) and waiting steps (programmed
    tensors from memory): identical positions, velocities and equilibrium
    maxima, both precisions; disk100 is a single tile."""
    m = make_model(workdir, name)
    x, v = deformed_state(m, seed=31, amp=0.02)
    g2, g3 = _loops(m, [2, path], precision=precision)
    r2, r3 = _run((g2, g3), x, v, m)
    x2, v2 = g2.download()
    x3, v3 = g3.download()
    assert np.array_equal(x2, x3) and np.array_equal(v2, v3)
    e2, e3 = r2.equil, r3.equil
    assert (e2.max_force, e2.max_speed, e2.max_force_node, e2.max_speed_node) == \
        (e3.max_force, e3.max_speed, e3.max_force_node, e3.max_speed_node)
    assert g3.plan_info()["path"] == path


def test_node_tiles_other_protocol_bitwise(workdir):
    """A protocol whose dialling writes the programmed tensors to memory each
    step (the kernel reads abar/bbar by triangle id)."""
    from morphoshell_b200 import meshgen
    m = make_model(workdir, "disk50")
    info, _ = m.programmed()
    T = m.num_tris
    a_info = meshgen.lce_abar_comps(info, 1.0)
    b_info = 0.3 * np.random.default_rng(1).standard_normal((T, 3))
    x, v = deformed_state(m, seed=32, amp=0.02)
    g2, g3, g4 = _loops(m, [2, 3, 4], protocol=1, a_info=a_info, b_info=b_info)
    _run((g2, g3, g4), x, v, m, dial_steps=150, wait_steps=50)
    ref = g2.download()
    for g in (g3, g4):
        assert all(np.array_equal(a, b) for a, b in zip(ref, g.download()))


def test_node_tiles_nonuniform_material_and_field(workdir, tmp_path):
    """Per-triangle thickness and shear modulus, and per-triangle lambda_final
    and nu_ot (the kernel reads them by triangle id)."""
    from morphoshell_b200 import Model, meshgen
    mesh, info, bbar = meshgen.workload("disk30")
    rng = np.random.default_rng(3)
    T = mesh.num_tris
    info = info.copy()
    info[:, 1] = 0.85 + 0.05 * rng.random(T)
    info[:, 2] = 0.45 + 0.1 * rng.random(T)
    st = os.path.join(str(tmp_path), "nonuni.txt")
    meshgen.write_settings(st, protocol=3)
    m = Model.from_arrays(st, mesh.nodes, mesh.tris, info, bbar, thickness=0.01 * (1 + 0.2 * rng.random(T)),
                          shear_modulus=1 + 0.3 * rng.random(T))
    x, v = deformed_state(m, seed=33, amp=0.02)
    for prec in (0, 1):
        g2, g3, g4 = _loops(m, [2, 3, 4], precision=prec)
        _run((g2, g3, g4), x, v, m, dial_steps=120, wait_steps=40)
        ref = g2.download()
        for g in (g3, g4):
            assert all(np.array_equal(a, b) for a, b in zip(ref, g.download()))


def test_node_tiles_guard(workdir):
    """A node thrown far away trips the guard at the same step and dof; the
    pre-step state survives."""
    from morphoshell_b200 import MsError
    m = make_model(workdir, "disk18k")
    s = m.scalars
    x, v = deformed_state(m, seed=34, amp=0.02)
    bad = x.copy()
    bad[2 * m.num_nodes + 4321] += 1e6
    offs = []
    for g in _loops(m, [2, 3, 4]):
        g.upload(bad, v)
        with pytest.raises(MsError) as ei:
            g.step_n(10, None, s.timestep, s.damping_factor_2)
        offs.append((ei.value.report.error_step, ei.value.report.offending_dof, ei.value.report.offending_force))
        gx, _ = g.download()
        assert np.array_equal(gx, bad)
    assert offs[0] == offs[1] == offs[2] and offs[0][0] == 0


@pytest.mark.parametrize("path", [3, 4])
def test_node_tiles_kernel_timing(workdir, path):
    """ms_time_kernels reports the one kernel of paths 3 and 4 and no node
    kernel."""
    m = make_model(workdir, "disk18k")
    s = m.scalars
    (g,) = _loops(m, [path])
    x, v = deformed_state(m, seed=35, amp=0.02)
    g.upload(x, v)
    t_tri, t_node = g.time_kernels(5, 0.2, s.timestep, s.damping_factor_1)
    assert t_tri > 0 and t_node == 0


def test_node_tile_plan_balances_blocks(workdir):
    """The tile count is a multiple of the persistent blocks (or the tiles
    are at their smallest size), so no block walks more tiles than another
    by more than one."""
    from morphoshell_b200 import GpuLoop
    m = make_model(workdir, "disk18k")
    for prec in (0, 1):
        info = GpuLoop(m, precision=prec).plan_info()
        nt, tiles, blocks = info["nodes_per_tile"], info["node_tiles"], info["node_tile_blocks"]
        assert tiles == -(-m.num_nodes // nt) and 0 < blocks <= tiles
        assert nt == 256 or tiles % blocks == 0 or tiles % blocks > 0.9 * blocks


def test_prepared_graphs_give_the_same_steps(workdir):
    """ms_prepare_steps builds the graphs of a later ms_step_n call and runs
    nothing: the state is untouched, and the prepared call gives the bits of
    an unprepared one."""
    m = make_model(workdir, "disk18k")
    s = m.scalars
    x, v = deformed_state(m, seed=36, amp=0.02)
    dials = 0.2 + 1e-5 * np.arange(40)
    out = []
    for prepare in (True, False):
        (g,) = _loops(m, [3])
        g.upload(x, v)
        if prepare:
            g.prepare_steps(40, True, s.timestep, s.damping_factor_1)
            assert all(np.array_equal(a, b) for a, b in zip(g.download(), (x, v)))
        g.step_n(40, dials, s.timestep, s.damping_factor_1)
        out.append(g.download())
    assert all(np.array_equal(a, b) for a, b in zip(out[0], out[1]))
