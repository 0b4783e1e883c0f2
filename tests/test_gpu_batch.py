"""Batched ensembles (ms_batch_*, msh_run_batch) -- GPU.

Every instance follows its own copy of the main loop's state machine
(main.cpp:269-508); the batch must reproduce each mesh's own run.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import make_model

pytestmark = pytest.mark.gpu

# Short dial phases and loose thresholds so that whole runs take a few
# thousand steps.
FAST = dict(dial_factors_to_hold_at_spacing=0.5, dial_phase_time_prefactor=0.02,
            force_to_char_force_ratio_equil_threshold=1e-5, speed_to_char_speed_ratio_equil_threshold=1e-4)


def _members(tmp_path, idx, spacing_range=(0.05, 0.1), **settings):
    from morphoshell_b200 import ensemble
    over = dict(FAST)
    over.update(settings)
    return ensemble.build_members(idx, str(tmp_path), spacing_range=spacing_range, threads=4, **over)


def test_batch_run_matches_single_runs(workdir):
    """Three meshes with different sizes, fields and thicknesses: the batch
    driver reaches each mesh's final equilibrium at the same step as that
    mesh's own msh_run, in the same shape."""
    from morphoshell_b200 import run_batch
    models = [make_model(workdir, "disk100", **FAST), make_model(workdir, "disk80", **FAST),
              make_model(workdir, "disk120", **FAST)]
    solo = [m.run(max_steps=400_000) for m in models]
    batch = run_batch(models, max_steps=400_000)
    for (rs, xs), (rb, xb) in zip(solo, batch):
        assert rs.final_dial_factor == 1.0 and rb.final_dial_factor == 1.0
        assert rb.equilibria_reached == rs.equilibria_reached
        assert rb.steps == rs.steps, (rb.steps, rs.steps)
        assert np.abs(xb - xs).max() < 1e-7, np.abs(xb - xs).max()


def test_batch_member_isolation_bitwise(tmp_path):
    """An instance gives the same bits alone as inside a batch of others."""
    from morphoshell_b200 import Batch
    models, _ = _members(tmp_path, [0, 1, 2])
    together = Batch(models)
    alone = Batch([models[1]])
    together.run(600)
    alone.run(600)
    xa, va = alone.download(0)
    xt, vt = together.download(1)
    assert np.array_equal(xa, xt) and np.array_equal(va, vt)
    sa, st = alone.status(0), together.status(1)
    assert (sa.stepcount, sa.status, sa.dial_factor) == (st.stepcount, st.status, st.dial_factor)


def test_batch_guard_fails_one_instance_only(tmp_path):
    """A node thrown far away trips the force guard of its own instance,
    which keeps its pre-step state; the others run on unchanged."""
    from morphoshell_b200 import MS_INST_FAILED, Batch, GpuLoop, MsError
    models, _ = _members(tmp_path, [3, 4, 5])
    ref = Batch(models)
    ref.run(300)
    bad = models[1].dofs(1).copy()
    N = models[1].num_nodes
    bad[2 * N + 17] += 1e6
    b = Batch(models, dofs=[None, bad, None])
    b.run(300)
    st = b.status(1)
    assert st.status == MS_INST_FAILED and st.stepcount == 0
    # The same state through the single-mesh stepper trips on the same dof.
    m = models[1]
    s = m.scalars
    g = GpuLoop(m)
    a_info, b_info = m.programmed()
    g.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
    g.upload(bad)
    with pytest.raises(MsError) as ei:
        g.step_n(1, np.array([s.dial_factor_to_start_from]), s.timestep, s.damping_factor_1)
    assert ei.value.report.error_step == 0
    assert st.offending_dof == ei.value.report.offending_dof
    x1, _ = b.download(1)
    assert np.array_equal(x1, bad)
    for i in (0, 2):
        assert np.array_equal(b.download(i)[0], ref.download(i)[0])


def test_batch_schedules_agree_and_autotune_keeps_state(tmp_path):
    """Every built-in schedule gives the same bits; autotuning leaves the
    state where it was."""
    from morphoshell_b200 import Batch
    models, _ = _members(tmp_path, [6, 7])
    a = Batch(models)
    a.run(200)
    x_before = [a.download(i)[0] for i in range(2)]
    sched, ms = a.autotune(steps_per_trial=10)
    assert ms > 0 and sched["chunk_steps"] % 2 == 0
    for i in range(2):
        assert np.array_equal(a.download(i)[0], x_before[i])
        assert a.status(i).stepcount == 200
    a.run(200)
    b = Batch(models)
    b.set_schedule(64, 128, 32)
    b.run(400)
    for i in range(2):
        assert np.array_equal(a.download(i)[0], b.download(i)[0])


def test_autotune_searches_node_tile_plans_with_the_same_bits(tmp_path):
    """On a union big enough for several tile sizes, the autotuner rebuilds
    the node-tiled plan (tables gathered on the device) and times each; the
    steps after it give the bits of the default plan."""
    from morphoshell_b200 import Batch
    models, _ = _members(tmp_path, [3, 5], spacing_range=(0.004, 0.0041))
    a = Batch(models)
    a.run(64)
    sched, ms = a.autotune(steps_per_trial=8)
    assert ms > 0 and sched["nodes_per_tile"] >= 256 and sched["blocks_per_sm"] >= 1, sched
    trials = a.autotune_report()
    assert sum("node-tiled plan" in t for t in trials) >= 1, trials
    for i in range(2):
        assert a.status(i).stepcount == 64
    a.run(128)
    b = Batch(models)
    b.set_schedule(-1, 0, 64)
    assert b.schedule()["nodes_per_tile"] >= 256
    b.run(192)
    for i in range(2):
        xa, va = a.download(i)
        xb, vb = b.download(i)
        assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_batch_done_instance_freezes(tmp_path):
    """An instance that reaches equilibrium at dial factor 1 stops; its
    final state stays available while the run goes on for the rest."""
    from morphoshell_b200 import MS_INST_DONE, Batch
    models, _ = _members(tmp_path, [8, 9], spacing_range=(0.08, 0.1))
    b = Batch(models)
    steps = b.run(400_000)
    sts = [b.status(i) for i in range(2)]
    assert all(s.status == MS_INST_DONE for s in sts), [s.status for s in sts]
    assert steps >= max(s.stepcount for s in sts)
    x0 = b.download(0)[0]
    b.run(100)
    assert np.array_equal(b.download(0)[0], x0)


def test_batch_mixed_precision_shapes(tmp_path):
    """The mixed-precision batch reaches the same final equilibria as FP64
    to within 1e-5 of the mesh size."""
    from morphoshell_b200 import MS_INST_DONE, MS_PRECISION_MIXED, Batch
    models, _ = _members(tmp_path, [10, 11], spacing_range=(0.08, 0.1))
    out = []
    for prec in (0, MS_PRECISION_MIXED):
        b = Batch(models, precision=prec)
        b.run(400_000)
        assert all(b.status(i).status == MS_INST_DONE for i in range(2))
        out.append([b.download(i)[0] for i in range(2)])
    for i in range(2):
        assert np.abs(out[1][i] - out[0][i]).max() < 1e-5


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_node_tiles_bitwise(tmp_path, precision):
    """The node-tiled one-kernel schedule gives the bits of the two-kernel
    tile schedule, through dialling, checks, one instance reaching its final
    equilibrium and one failing on the guard."""
    from morphoshell_b200 import MS_INST_DONE, MS_INST_FAILED, Batch
    models, _ = _members(tmp_path, [12, 13, 14], spacing_range=(0.07, 0.1))
    bad = models[2].dofs(1).copy()
    bad[2 * models[2].num_nodes + 5] += 1e6
    out = []
    for sched in ((-1, 0), (0, 256)):
        b = Batch(models, precision=precision, dofs=[None, None, bad])
        b.set_schedule(sched[0], sched[1], 32)
        steps = b.run(400_000)
        sts = [b.status(i) for i in range(3)]
        out.append((steps, [(s.status, s.stepcount, s.equilibria) for s in sts],
                    [b.download(i) for i in range(3)]))
        assert sts[2].status == MS_INST_FAILED
        assert sts[0].status == MS_INST_DONE and sts[1].status == MS_INST_DONE
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    for i in range(3):
        assert np.array_equal(out[0][2][i][0], out[1][2][i][0]) and np.array_equal(out[0][2][i][1], out[1][2][i][1])


def test_batch_members_against_oracle(tmp_path):
    """Batch members against the CPU oracle, not only against the
    single-mesh driver: each instance's dialling trajectory (protocol 3,
    dialled in-kernel from the instance's own field, step k at
    dial_factors_to_hold_at_spacing * k / timesteps_per_dial_phase,
    main.cpp:478-488) after the same number of steps, positions within 1e-9
    relative.  Step 0 is dialled in-kernel too and lambda^(-2 nu_ot) comes
    from the device pow, the two places the batch can differ from the
    reference's do_dialling (do_dialling.cpp:112-123)."""
    from morphoshell_b200 import MS_INST_DIALLING, Batch
    from oracle import Oracle
    models, _ = _members(tmp_path, [15, 16, 17], spacing_range=(0.05, 0.08))
    n = min(3000, min(m.scalars.timesteps_per_dial_phase for m in models) - 1)
    b = Batch(models)
    assert b.run(n) == n
    for i, m in enumerate(models):
        st = b.status(i)
        assert st.status == MS_INST_DIALLING and st.stepcount == n
        s = m.scalars
        a_info, b_info = m.programmed()
        o = Oracle("orc", m)
        o.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
        o.upload(m.dofs(1))
        dials = s.dial_factors_to_hold_at_spacing * (np.arange(n) / s.timesteps_per_dial_phase)
        rc, done = o.step_n(n, dials, s.timestep, s.damping_factor_1)
        assert rc == 0 and done == n
        ox, ov = o.download()
        bx, bv = b.download(i)
        assert np.abs(bx - ox).max() <= 1e-9 * np.abs(ox).max(), i
        assert np.abs(bx - m.dofs(1)).max() > 0
