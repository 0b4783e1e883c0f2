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
