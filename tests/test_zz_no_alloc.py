"""The allocation-free deformation-forces entry point
(ms_deformation_forces_noalloc), checked against ms_deformation_forces.

Some callers cannot call cudaMalloc: host frameworks that route all device
memory through their own pool, and real-time loops that must not allocate
once started.  They hand in device buffers they already own; the entry point
works in a fixed scratch array inside the library.  Because every call
reuses that array, the test makes two calls in a row on different states of
one mesh and then a third on a smaller mesh (stale counts and lists of the
larger mesh lie beyond its nodes in the scratch), and compares each with the
handle-based entry point, at the force tolerance of the other parity tests.

The file name makes pytest collect it last, so that a run stopping at the
first failure has already run every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import deformed_state, make_model, rel_err

FORCE_RTOL = 1e-12

pytestmark = pytest.mark.gpu


def _reference_forces(model, x, v, dial):
    from morphoshell_b200 import GpuLoop
    s = model.scalars
    a_info, b_info = model.programmed()
    g = GpuLoop(model)
    g.set_programmed(3, a_info, b_info, s.dial_factors_to_hold_at_spacing)
    g.upload(x, v)
    g.do_dialling(dial)
    g.surface_derivs()
    f, _ = g.deformation_forces()
    abar, bbar = g.programmed()
    g.close()
    return f, abar, bbar


def _noalloc(model, x, abar, bbar):
    import torch
    from morphoshell_b200 import MS_OK, lib
    tb = model.tables()
    p = model.params
    dev = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in {
        "patch": tb["patch_ids"].astype(np.int32), "coef": tb["deriv_coeffs"], "area": tb["ref_area"],
        "thick": tb["ref_thickness"], "shear": tb["ref_shear_modulus"], "abar": abar, "bbar": bbar,
        "dofs": x}.items()}
    forces = torch.empty(3 * model.num_nodes, dtype=torch.float64, device=dev)
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib().ms_deformation_forces_noalloc(
        model.num_nodes, model.num_tris, t["patch"].data_ptr(), t["coef"].data_ptr(), t["area"].data_ptr(),
        t["thick"].data_ptr(), t["shear"].data_ptr(), t["abar"].data_ptr(), t["bbar"].data_ptr(),
        p.def_poisson_ratio, p.bend_stiffening_scale_factor, t["dofs"].data_ptr(), forces.data_ptr(), stream, err,
        256)
    assert rc == MS_OK, err.value
    return forces.cpu().numpy()


def test_noalloc_matches_handle_path_on_two_calls(workdir):
    big = make_model(workdir, "disk18k")
    small = make_model(workdir, "disk50")
    for m, seed, dial in ((big, 11, 0.4), (big, 12, 0.8), (small, 13, 0.6)):
        x, v = deformed_state(m, seed=seed)
        ref, abar, bbar = _reference_forces(m, x, v, dial)
        got = _noalloc(m, x, abar, bbar)
        assert rel_err(got, ref) < FORCE_RTOL, (m.num_tris, seed, rel_err(got, ref))


def test_noalloc_rejects_meshes_beyond_its_scratch():
    from morphoshell_b200 import lib
    err = C.create_string_buffer(256)
    fake = C.c_void_p(16)
    rc = lib().ms_deformation_forces_noalloc(10, 70000, fake, fake, fake, fake, fake, fake, fake, 0.5, 1.0, fake,
                                             fake, None, err, 256)
    assert rc == 1
    assert b"exceeds the static scratch limit" in err.value
