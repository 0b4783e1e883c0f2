"""The whole driver against the reference's own executable.

The reference's executable (oracle/_ref/morphoshell_ref_p3: every file of
source_files/ compiled unmodified, main.cpp included, with do_dialling.cpp's
protocol-3 block switched on) and this project's command-line driver
(morphoshell_b200/lib/morphoshell_gpu: host set-up, msh_run's state machine,
the GPU loop) run the same settings file and mesh: the 0.05-spacing disk,
four short dial phases, regular output on, looser equilibrium thresholds so
that the run reaches equilibria in seconds.  The reference never leaves its
loop by itself (main.cpp:493-495), so it is stopped on the host once it has
logged its N-th output; the driver then runs to the same step.

Checked (main.cpp:282-304, 396-438, 478-507; write_output.cpp:60-170):
* the same steps carry output files and the same steps reach equilibrium;
* every output file has the same header line (dial factor and step), the
  same section layout and the same triangles;
* points within 1e-9 of the disk's size, per-triangle fields within a
  norm-wise 1e-9 (stress eigenvectors up to sign) and angle deficits within
  1e-9 of their largest value;
* aux_output.txt has the same rows.
"""
from __future__ import annotations

import os
import re
import subprocess
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_OUT = 5
SETTINGS = dict(dial_phase_time_prefactor=0.02, dial_factors_to_hold_at_spacing=0.25, outputs_per_char_long_time=20.0,
                force_to_char_force_ratio_equil_threshold=1e-4, speed_to_char_speed_ratio_equil_threshold=1e-3)
POINT_TOL = 1e-9
FIELD_TOL = 1e-9


def _parse_vtk(path):
    """(layout lines, {section: float array}) of an output file: every line
    that is not all numbers is layout; the numbers that follow it form that
    section."""
    layout, data, cur = [], {}, None
    num = re.compile(r"^[-+0-9.eE ]+$")
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n")
            if num.match(line) and cur is not None:
                data[cur].append([float(v) for v in line.split()])
            else:
                layout.append(line)
                cur = "%d: %s" % (len(layout) - 1, line)
                data[cur] = []
    return layout, {k: np.array(v) for k, v in data.items() if v}


def _logged(path, pattern):
    if not os.path.exists(path):
        return []
    with open(path) as f:
        return [int(m.group(1)) for m in re.finditer(pattern, f.read())]


WROTE = r"Wrote VTK output at [^\n]*stepcount = (\d+),"
EQUIL = r"Equilibrium reached\. Writing VTK output at [^\n]*stepcount = (\d+),"


def test_driver_matches_reference_executable(tmp_path):
    import oracle
    from morphoshell_b200 import meshgen
    from morphoshell_b200.build import EXE
    if not os.path.exists(oracle.REF_EXE_P3):
        pytest.skip("reference executable absent (built only where the reference tree is present)")
    ref_dir, gpu_dir = tmp_path / "ref", tmp_path / "gpu"
    for d in (ref_dir, gpu_dir):
        meshgen.write_workload(str(d), "disk50", **SETTINGS)
    # The reference, stopped once it has logged its N-th output.
    env = dict(os.environ, OMP_NUM_THREADS=str(min(8, os.cpu_count() or 1)))
    ref_out = ref_dir / "output_using_disk50_settings.txt"
    proc = subprocess.Popen([oracle.REF_EXE_P3, "disk50_settings.txt", "disk50.vtk"], cwd=ref_dir, env=env,
                            stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    t0 = time.time()
    try:
        while len(_logged(ref_out / "log.txt", WROTE)) < N_OUT:
            assert proc.poll() is None, "reference executable exited early"
            assert time.time() - t0 < 600, "reference executable too slow"
            time.sleep(0.2)
    finally:
        proc.kill()
        proc.wait()
    ref_steps = _logged(ref_out / "log.txt", WROTE)[:N_OUT]
    last = ref_steps[-1]
    ref_equil = [s for s in _logged(ref_out / "log.txt", EQUIL) if s <= last]
    assert ref_equil, "the reference reached no equilibrium in the compared stretch"
    # The driver, to the same step.
    gpu_out = gpu_dir / "out"
    r = subprocess.run([EXE, "disk50_settings.txt", "disk50.vtk", "--out", str(gpu_out), "--max-steps",
                        str(last + 1), "--keep-going"], cwd=gpu_dir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    gpu_steps = sorted(int(m.group(1)) for m in (re.match(r"stepcount_(\d+)_output\.vtk", f)
                                                  for f in os.listdir(gpu_out)) if m)
    assert gpu_steps == ref_steps
    assert [s for s in _logged(gpu_out / "log.txt", EQUIL) if s <= last] == ref_equil
    for step in ref_steps:
        name = "stepcount_%d_output.vtk" % step
        lr, dr = _parse_vtk(ref_out / name)
        lg, dg = _parse_vtk(gpu_out / name)
        assert lg == lr, name  # header line (dial factor, step), sections, sizes
        assert sorted(dg) == sorted(dr), name
        pts, tris = "4: " + lr[4], "5: " + lr[5]
        assert lr[4].startswith("POINTS") and lr[5].startswith("POLYGONS")
        assert np.array_equal(dg[tris], dr[tris]), name
        scale = np.abs(dr[pts]).max()
        assert np.abs(dg[pts] - dr[pts]).max() <= POINT_TOL * scale, name
        for key in dr:
            if key in (pts, tris):
                continue
            a, b = dg[key], dr[key]
            if "eigvec" in key:
                dots = np.abs(np.sum(a * b, axis=1))
                bad = np.abs(dots - 1.0) > 1e-6
                assert bad.mean() < 1e-3, (name, key)  # near-degenerate eigenpairs may rotate
                continue
            assert np.abs(a - b).max() <= FIELD_TOL * max(np.abs(b).max(), 1e-300), (name, key)
    with open(ref_out / "aux_output.txt") as f:
        aux_r = [l.split() for l in f.read().splitlines()[:N_OUT + 1]]
    with open(gpu_out / "aux_output.txt") as f:
        aux_g = [l.split() for l in f.read().splitlines()[:N_OUT + 1]]
    assert aux_g == aux_r
