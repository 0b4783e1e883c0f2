"""Set-up on the device (msh_load / msh_build flag bit 2, setup.cu) against
the host set-up (mesh_setup.cpp) -- GPU.

The patch search and fit (set_up_patch_fitting.cpp:48-305) and the
derivative weights (calc_deriv_mats.cpp:46-136) run one thread per triangle
with the host's operations in the host's order, so the patch nodes and the
24 weights of every triangle must come out bit for bit the same, including
on a regular lattice where many candidate distances tie (those triangles
are redone on the host).
"""
from __future__ import annotations

import os
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same_tables(a, b):
    ta, tb = a.tables(), b.tables()
    assert np.array_equal(ta["patch_ids"], tb["patch_ids"])
    # Bit patterns, so that a sign of zero counts too.
    assert np.array_equal(ta["deriv_coeffs"].view(np.uint64), tb["deriv_coeffs"].view(np.uint64))
    assert np.array_equal(ta["node_mass"], tb["node_mass"])


@pytest.mark.parametrize("name", ["disk18k", "disk1p8m"])
def test_device_setup_matches_host_setup(tmp_path, name):
    from morphoshell_b200 import Model, meshgen
    st, vtk = meshgen.write_workload(str(tmp_path), name)
    t0 = time.perf_counter()
    host = Model(st, vtk, noise=False)
    t1 = time.perf_counter()
    dev = Model(st, vtk, noise=False, device_setup=True)
    t2 = time.perf_counter()
    _same_tables(host, dev)
    print("%s set-up: host %.2f s, device %.2f s" % (name, t1 - t0, t2 - t1))


def test_device_setup_on_a_regular_lattice(tmp_path):
    """No jitter: equal candidate distances everywhere; the host decides
    those triangles' order, and the tables still agree bit for bit."""
    from morphoshell_b200 import Model, meshgen
    mesh = meshgen.disk_mesh(0.05, seed=0, jitter=0.0)
    info = meshgen.lce_abar_info(mesh, meshgen.azimuthal_director, 0.9)
    bbar = np.zeros((mesh.num_tris, 3))
    st = os.path.join(str(tmp_path), "lattice_settings.txt")
    meshgen.write_settings(st, protocol=3)
    kw = dict(positions=mesh.nodes, tris=mesh.tris, abar_info=info, bbar_info=bbar,
              thickness=np.full(mesh.num_tris, 0.01), noise=False)
    host = Model.from_arrays(st, **kw)
    dev = Model.from_arrays(st, device_setup=True, **kw)
    _same_tables(host, dev)
