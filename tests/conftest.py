"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running parity check")


def _ensure_built():
    from morphoshell_b200 import LIB_PATH
    import oracle
    if not os.path.exists(LIB_PATH):
        from morphoshell_b200 import build
        build.build()
    if not os.path.exists(oracle.PORT_LIB):
        from oracle import build as obuild
        obuild.build_port()


_ensure_built()


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("workloads"))


_models = {}


def make_model(workdir, name, noise=True, **settings):
    """A host-side Model of a named synthetic workload (see meshgen.workload)."""
    from morphoshell_b200 import Model, meshgen
    key = (name, noise, tuple(sorted(settings.items())))
    if key not in _models:
        sub = os.path.join(workdir, "%s_%d" % (name, len(_models)))
        st, vtk = meshgen.write_workload(sub, name, **settings)
        _models[key] = Model(st, vtk, quiet=True, noise=noise)
    return _models[key]


def deformed_state(model, seed=0, amp=0.05, noise=1e-3, stretch=1.02):
    """A smooth, well-conditioned deformed state with velocities (SoA dofs)."""
    rng = np.random.default_rng(seed)
    N = model.num_nodes
    x = model.dofs(0).reshape(3, N).copy()
    r2 = x[0] ** 2 + x[1] ** 2
    x[2] += amp * np.exp(-4.0 * r2) + noise * rng.standard_normal(N)
    x[0] *= stretch
    x[1] += 0.01 * x[0] * x[1]
    v = 1e-3 * rng.standard_normal(3 * N)
    return x.ravel(), v


def rel_err(a, b):
    """Norm-wise relative difference max|a-b| / max|b|."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def protocol_inputs(model, protocol, seed=0):
    """(abar_info, bbar_info, dial_factors_to_hold_at_spacing) for a
    dialling protocol of do_dialling.cpp on a model's mesh: 1 and 2 final
    abar/bbar (T x 3 each); 3 the LCE director angle, lambda_final and nu_ot;
    4 eleven lambda checkpoints at dial factors 0, 0.1, ..., 1 then nu_ot and
    the director angle (T x 13, spacing 0.1, do_dialling.cpp:128-153); 5 the
    radial coordinate of the centroid (do_dialling.cpp:158-177)."""
    from morphoshell_b200 import meshgen
    info, _ = model.programmed()
    T = model.num_tris
    rng = np.random.default_rng(seed)
    if protocol in (1, 2):
        return meshgen.lce_abar_comps(info, 1.0), 0.3 * rng.standard_normal((T, 3)), 0.05
    if protocol == 3:
        return info, np.zeros((T, 1)), 0.05
    if protocol == 4:
        lam_final = 0.8 + 0.4 * rng.random(T)
        k = np.arange(11) / 10.0
        wobble = 0.02 * rng.standard_normal((T, 11))
        wobble[:, 0] = 0.0
        lam = 1.0 + np.outer(lam_final - 1.0, k) + wobble
        return np.column_stack([lam, np.full(T, 0.5), info[:, 0]]), np.zeros((T, 1)), 0.1
    x = model.dofs(0).reshape(3, -1)
    tri = model.tables()["patch_ids"][:, :3]
    cx, cy = x[0][tri].mean(1), x[1][tri].mean(1)
    return np.sqrt(cx * cx + cy * cy).reshape(-1, 1), np.zeros((T, 1)), 0.05


def deformation_forces_of(kind, model, x, v, dial, threads=None):
    """Deformation forces of a CPU oracle (``orc``: the restatement, ``ref``:
    the reference's own functions) on a state, protocol-3 dialling at `dial`."""
    from oracle import Oracle
    s = model.scalars
    a_info, b_info = model.programmed()
    o = Oracle(kind, model, threads=threads)
    o.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
    o.upload(x, v)
    o.surface_derivs()
    o.do_dialling(dial)
    f, _ = o.deformation_forces()
    o.close()
    return f


def check_forces_to_rounding(model, x, v, dial, gpu_forces, rtol=1e-12, threads=None):
    """GPU deformation forces on a state against the oracle's: within rtol
    (norm-wise), or -- on states where the forces are small next to the
    terms they cancel from (near the flat start a - abar is tiny, and two
    correct double-precision evaluations differ by about eps |a| / |a - abar|
    relative) -- no further from the oracle than the reference's own code is
    (compiled from its source), and within three times that of the
    reference.  Returns (gpu vs oracle, reference vs oracle, gpu vs
    reference); the last two are None without the reference build."""
    import oracle
    of = deformation_forces_of("orc", model, x, v, dial, threads)
    e_go = rel_err(gpu_forces, of)
    if not oracle.available("ref"):
        assert e_go < rtol, e_go
        return e_go, None, None
    rf = deformation_forces_of("ref", model, x, v, dial, threads)
    e_ro, e_gr = rel_err(rf, of), rel_err(gpu_forces, rf)
    floor = max(rtol, e_ro)
    assert e_go <= 2 * floor and e_gr <= 3 * floor, (e_go, e_ro, e_gr)
    return e_go, e_ro, e_gr

