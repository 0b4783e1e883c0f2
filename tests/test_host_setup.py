"""Host-side set-up (settings, VTK input, topology, patch fitting, derivative
weights, masses, characteristic scales) -- CPU only.

Where the reference tree was available at build time, the whole set-up is
compared with the reference's own set-up code compiled from source
(oracle/_ref, ``ref_setup_from_files``)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from conftest import make_model


def _ref_setup(settings, vtk, N, T):
    import oracle
    if not oracle.available("ref"):
        pytest.skip("reference build absent")
    L = C.CDLL(oracle.REF_LIB)
    d = C.POINTER(C.c_double)
    f = L.ref_setup_from_files
    f.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int32), d, d, d, d,
                  C.c_char_p, C.c_int]
    patch = np.zeros((T, 6), np.int32)
    mat2 = np.zeros((T, 18))
    mass = np.zeros(N)
    dofs = np.zeros(3 * N)
    scal = np.zeros(14)
    err = C.create_string_buffer(512)
    n, t = C.c_int(), C.c_int()
    rc = f(settings.encode(), vtk.encode(), C.byref(n), C.byref(t), patch.ctypes.data_as(C.POINTER(C.c_int32)),
           mat2.ctypes.data_as(d), mass.ctypes.data_as(d), dofs.ctypes.data_as(d), scal.ctypes.data_as(d), err, 512)
    assert rc == 0, err.value
    return patch, mat2, mass, dofs, scal


@pytest.mark.parametrize("name", ["disk100", "disk50", "disk18k"])
def test_setup_matches_reference_code(workdir, name):
    m = make_model(workdir, name)
    from morphoshell_b200 import meshgen
    sub = os.path.join(workdir, "ref_%s" % name)
    st, vtk = meshgen.write_workload(sub, name)
    patch, mat2, mass, dofs0, scal = _ref_setup(st, vtk, m.num_nodes, m.num_tris)
    tb = m.tables()
    s = m.scalars
    # identical patch choice, patch matrices to rounding
    assert np.array_equal(tb["patch_ids"], patch)
    assert np.abs(tb["deriv_coeffs"][:, 6:] - mat2).max() <= 1e-12 * np.abs(mat2).max()
    assert np.abs(tb["node_mass"] - mass).max() <= 1e-15 * mass.max()
    # initial noise: the same minimal-standard generator stream
    assert np.abs(m.dofs(1) - dofs0).max() <= 1e-15
    mine = [s.sample_char_length, s.approx_min_tri_size, s.min_ref_thickness, s.char_force_scale,
            s.char_speed_scale, s.char_long_time, s.damping_factor_1, s.timestep, s.timesteps_per_dial_phase,
            s.timesteps_between_equil_checks, s.total_ref_area, s.num_edges, s.num_boundary_nodes, s.damping_factor_2]
    np.testing.assert_allclose(mine, scal, rtol=1e-14, atol=0)


def test_topology_identities(workdir):
    m = make_model(workdir, "disk50")
    s = m.scalars
    assert 3 * s.num_tris == 2 * s.num_edges - s.num_boundary_edges
    assert 1 + s.num_edges - s.num_nodes - s.num_tris == 0  # a disk has no holes
    assert s.num_boundary_nodes == s.num_boundary_edges


def test_patch_fit_is_exact_on_quadratics(workdir):
    """The 6x3 patch matrices reproduce the second derivatives of any quadratic
    exactly, and the first-derivative weights reproduce any linear field."""
    m = make_model(workdir, "disk50")
    tb = m.tables()
    ref = m.dofs(0).reshape(3, -1)
    x, y = ref[0], ref[1]
    f = 0.7 * x * x - 1.3 * x * y + 2.1 * y * y + 0.4 * x - 0.2 * y + 3.0
    p = tb["patch_ids"]
    c = tb["deriv_coeffs"]
    fxx = np.einsum("tn,tn->t", c[:, 6::3], f[p])
    fxy = np.einsum("tn,tn->t", c[:, 7::3], f[p])
    fyy = np.einsum("tn,tn->t", c[:, 8::3], f[p])
    np.testing.assert_allclose(fxx, 1.4, atol=1e-7)
    np.testing.assert_allclose(fxy, -1.3, atol=1e-7)
    np.testing.assert_allclose(fyy, 4.2, atol=1e-7)
    g = 0.4 * x - 0.2 * y + 3.0
    gx = np.einsum("tv,tv->t", c[:, 0:3], g[p[:, :3]])
    gy = np.einsum("tv,tv->t", c[:, 3:6], g[p[:, :3]])
    np.testing.assert_allclose(gx, 0.4, atol=1e-10)
    np.testing.assert_allclose(gy, -0.2, atol=1e-10)


def _settings_text(**over):
    from morphoshell_b200 import meshgen
    lines = []
    for k, v in meshgen.SETTINGS_ORDER:
        lines.append("%s = %s;" % (k, meshgen._fmt(over.get(k, v))))
    return lines


def _load(tmp_path, lines, vtk_text=None, name="s.txt"):
    from morphoshell_b200 import Model, meshgen
    st = tmp_path / name
    st.write_text("\n".join(lines) + "\n")
    vtk = tmp_path / "m.vtk"
    if vtk_text is None:
        mesh, info, bbar = meshgen.workload("disk100")
        meshgen.write_vtk(str(vtk), "t", mesh.nodes, mesh.tris, info, bbar)
    else:
        vtk.write_text(vtk_text)
    return Model(str(st), str(vtk))


def test_settings_comments_whitespace_and_order(tmp_path):
    lines = _settings_text()
    lines = ["// a comment line"] + [l.replace(" = ", "  =\t") + "  // trailing" for l in lines]
    m = _load(tmp_path, lines + ["dialling_protocol = 3;"])
    assert m.scalars.dialling_protocol == 3
    with pytest.raises(RuntimeError, match="ref_thickness_if_uniform"):
        bad = _settings_text()
        bad[1], bad[2] = bad[2], bad[1]
        _load(tmp_path, bad)
    with pytest.raises(RuntimeError, match="semicolon"):
        bad = _settings_text()
        bad[3] = bad[3].rstrip(";")
        _load(tmp_path, bad)
    with pytest.raises(RuntimeError, match="neither true nor false"):
        bad = _settings_text()
        bad[3] = "dialling_from_ansatz_rather_than_ref_state = yes;"
        _load(tmp_path, bad)
    with pytest.raises(RuntimeError, match="ansatz"):
        _load(tmp_path, _settings_text(dialling_from_ansatz_rather_than_ref_state=True))
    with pytest.raises(RuntimeError, match="largest permitted value"):
        _load(tmp_path, _settings_text(dial_factors_to_hold_at_spacing=1.5))
    with pytest.raises(RuntimeError, match="glass slides"):
        _load(tmp_path, _settings_text(slide_stiffness_prefactor=1.0))


def test_vtk_reader_errors(tmp_path):
    from morphoshell_b200 import meshgen
    mesh, info, bbar = meshgen.workload("disk100")
    good = tmp_path / "g.vtk"
    meshgen.write_vtk(str(good), "t", mesh.nodes, mesh.tris, info, bbar)
    text = good.read_text()
    lines = _settings_text()
    # one triangle too few -> CELL_DATA sentinel not where expected
    i = text.index("POLYGONS")
    hdr_end = text.index("\n", i)
    first_tri_end = text.index("\n", hdr_end + 1)
    with pytest.raises(RuntimeError, match="CELL_DATA"):
        _load(tmp_path, lines, text[:hdr_end + 1] + text[first_tri_end + 1:])
    # ids not starting at zero
    with pytest.raises(RuntimeError):
        t2 = text.replace("POLYGONS", "POLYGONS")
        mesh2 = mesh.tris + 1
        nodes2 = np.vstack([mesh.nodes, [[5.0, 5.0, 0.0]]])
        p = tmp_path / "z.vtk"
        meshgen.write_vtk(str(p), "t", nodes2, mesh2, info, bbar)
        _load(tmp_path, lines, p.read_text())
    # trailing garbage -> end-of-file check
    with pytest.raises(RuntimeError, match="end of reference data file"):
        _load(tmp_path, lines, text + "extra\n")


def test_model_from_arrays_equals_file(workdir):
    from morphoshell_b200 import Model, meshgen
    m1 = make_model(workdir, "disk50")
    mesh, info, bbar = meshgen.workload("disk50")
    st = os.path.join(workdir, "arr_settings.txt")
    meshgen.write_settings(st, protocol=3)
    m2 = Model.from_arrays(st, mesh.nodes, mesh.tris, info, bbar, thickness=np.full(mesh.num_tris, 0.01))
    t1, t2 = m1.tables(), m2.tables()
    # The file stores positions with 16 significant digits; the arrays are exact.
    for k in t1:
        if t1[k].dtype.kind == "f":
            np.testing.assert_allclose(t1[k], t2[k], rtol=1e-11, atol=1e-11 * np.abs(t1[k]).max(), err_msg=k)
        else:
            assert np.array_equal(t1[k], t2[k]), k
    assert abs(m1.scalars.timestep - m2.scalars.timestep) <= 1e-13 * m1.scalars.timestep


def test_parallel_setup_matches_serial(tmp_path, monkeypatch):
    """The per-triangle set-up loops run in threads on larger meshes; the
    tables are identical to a one-thread run."""
    from morphoshell_b200 import Model, meshgen
    mesh, info, bbar = meshgen.workload("disk12")
    st = str(tmp_path / "s.txt")
    meshgen.write_settings(st, protocol=3)
    out = []
    for threads in ("1", "7"):
        monkeypatch.setenv("MORPHOSHELL_SETUP_THREADS", threads)
        m = Model.from_arrays(st, mesh.nodes, mesh.tris, info, bbar)
        assert m.num_tris > 4096
        out.append(m.tables())
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_ansatz_file_is_read(tmp_path):
    """An ansatz file in the output format (read_vtk_data.cpp:380-445): its
    dial factor and node positions become the start of the dynamics; a file
    with the wrong node count is refused with the reference's message."""
    from morphoshell_b200 import Model, meshgen
    mesh, info, bbar = meshgen.workload("disk100")
    st = tmp_path / "s.txt"
    st.write_text("\n".join(_settings_text()) + "\n")
    vtk = tmp_path / "m.vtk"
    meshgen.write_vtk(str(vtk), "t", mesh.nodes, mesh.tris, info, bbar)
    N = mesh.nodes.shape[0]
    rng = np.random.default_rng(3)
    pos = np.column_stack([mesh.nodes[:, 0], mesh.nodes[:, 1], 0.01 * rng.standard_normal(N)])

    def ansatz_text(n, dial):
        head = ["# vtk DataFile Version 4.2", "dial_factor = %.14e, stepcount = 1200" % dial, "ASCII",
                "DATASET POLYDATA", "POINTS %d double" % n]
        return "\n".join(head + ["%.17g %.17g %.17g" % tuple(p) for p in pos[:n]]) + "\n"

    an = tmp_path / "ansatz.vtk"
    an.write_text(ansatz_text(N, 0.375))
    m = Model(str(st), str(vtk), str(an), noise=False)
    x = m.dofs(1).reshape(3, -1).T
    assert np.array_equal(x, pos)
    assert m.scalars.dial_factor_to_start_from == 0.375
    an.write_text(ansatz_text(N - 1, 0.375))
    with pytest.raises(RuntimeError, match="number of nodes in ansatz data file"):
        Model(str(st), str(vtk), str(an), noise=False)


def test_vtk_reader_line_forms(tmp_path):
    """Blocks are read line by line in parallel only when every line holds
    its values; other layouts get the stream reader's behaviour: extra
    values at a line's end are ignored, CRLF line ends read the same, and a
    line short of a value pulls it from the next line, so the file runs out
    of step and fails at the next section header."""
    from morphoshell_b200 import meshgen
    mesh, info, bbar = meshgen.workload("disk100")
    good = tmp_path / "g.vtk"
    meshgen.write_vtk(str(good), "t", mesh.nodes, mesh.tris, info, bbar)
    text = good.read_text()
    lines = _settings_text()
    ref = _load(tmp_path, lines, text).tables()

    def same(m):
        t = m.tables()
        return all(np.array_equal(t[k], ref[k]) for k in ref)

    i = text.index("POINTS")
    first = text.index("\n", i) + 1
    second = text.index("\n", first)
    assert same(_load(tmp_path, lines, text[:second] + " 7 8 9" + text[second:]))
    assert same(_load(tmp_path, lines, text.replace("\n", "\r\n")))
    short = text[:first] + " ".join(text[first:second].split()[:2]) + text[second:]
    with pytest.raises(RuntimeError, match="POLYGONS"):
        _load(tmp_path, lines, short)


def test_set_up_from_file_same_with_one_thread_and_many(tmp_path, monkeypatch):
    """The file's blocks, the mesh bookkeeping and the patch fit run in
    parallel ranges; the model does not depend on how many threads."""
    from morphoshell_b200 import Model, meshgen
    st, vtk = meshgen.write_workload(str(tmp_path), "disk18k")
    models = []
    for threads in ("1", "6"):
        monkeypatch.setenv("MORPHOSHELL_SETUP_THREADS", threads)
        models.append(Model(st, vtk, noise=False))
    a, b = (m.tables() for m in models)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(models[0].dofs(0), models[1].dofs(0))
    assert models[0].scalars.timestep == models[1].scalars.timestep
