"""Generate tests/golden/disk18k_equilibria.npz: the reference's own executable
(oracle/_ref/morphoshell_ref_p3: every file of source_files/ compiled
unmodified by oracle/build.py, with do_dialling.cpp's protocol-3 block
switched on) run on the 18k-triangle disk to its first equilibrium at dial
factor 1.

    python tests/golden/make_disk18k_equilibria.py [--reuse RUN_DIR]

Workload: ``meshgen.write_workload(dir, "disk18k", **SETTINGS)`` -- unit disk,
jittered hex spacing 0.02 (9,201 nodes, 18,086 triangles), azimuthal
director, lambda 1 -> 0.9, h = 0.01, nu = 0.5, the reference's equilibrium
criterion (force and speed thresholds 1e-6 and 1e-5 of the characteristic
scales, is_at_equilibrium.cpp:92-98), four dial phases (spacing 0.25) of
0.02 of the long time each (the default schedule of 20 phases of 0.25 long
times runs about 10^7 steps, three hours of the reference on 8 threads).
Regular output is off, so the reference writes a file at each equilibrium
only (main.cpp:412-436).  The reference never leaves its loop
(main.cpp:493-495); it is stopped once it has logged the equilibrium at dial
factor 1 (about half an hour on 8 threads).

The file holds the step and dial factor of every equilibrium up to that one,
the node positions written at each, and every field of the last output file
(write_output.cpp:77-170).  ``--reuse RUN_DIR`` reads an existing
output_using_disk18k_settings.txt directory of such a run instead of running
the reference again.
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "disk18k_equilibria.npz")
SETTINGS = dict(dial_phase_time_prefactor=0.02, dial_factors_to_hold_at_spacing=0.25)
EQUIL = re.compile(r"Equilibrium reached\. Writing VTK output at [^\n]*stepcount = (\d+), "
                   r"simulation time = [^,]*, dial_factor = ([-+0-9.eE]+)")


def equilibria(log_path):
    if not os.path.exists(log_path):
        return []
    with open(log_path) as f:
        return [(int(m.group(1)), float(m.group(2))) for m in EQUIL.finditer(f.read())]


def parse_vtk(path):
    """(layout lines, {section key: array}) of an output file; a section is
    the numbers that follow a layout line, keyed 'index: line'."""
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


def run_reference(threads):
    import oracle
    from morphoshell_b200 import meshgen
    d = tempfile.mkdtemp(prefix="disk18k_eq_")
    meshgen.write_workload(d, "disk18k", **SETTINGS)
    out = os.path.join(d, "output_using_disk18k_settings.txt")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    proc = subprocess.Popen([oracle.REF_EXE_P3, "disk18k_settings.txt", "disk18k.vtk"], cwd=d, env=env,
                            stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    t0 = time.time()
    try:
        while not any(dial >= 1.0 for _, dial in equilibria(os.path.join(out, "log.txt"))):
            if proc.poll() is not None:
                raise RuntimeError("the reference executable exited early")
            time.sleep(2.0)
            print("%.0f s: %s" % (time.time() - t0, equilibria(os.path.join(out, "log.txt"))), flush=True)
    finally:
        proc.kill()
        proc.wait()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--reuse", default=None, help="an existing output_using_disk18k_settings.txt directory")
    a = ap.parse_args()
    out = a.reuse or run_reference(a.threads)
    eq = equilibria(os.path.join(out, "log.txt"))
    last = next(i for i, (_, dial) in enumerate(eq) if dial >= 1.0)
    eq = eq[:last + 1]
    points = []
    for step, _ in eq:
        layout, data = parse_vtk(os.path.join(out, "stepcount_%d_output.vtk" % step))
        points.append(data["4: " + layout[4]])
    # The last file's fields besides the points (kept above) and the
    # triangles (the input mesh's).
    keys = sorted(k for k in data if not k.startswith(("4: ", "5: ")))
    fields = {"field_%02d" % i: data[k] for i, k in enumerate(keys)}
    np.savez_compressed(OUT, steps=np.array([s for s, _ in eq]), dials=np.array([d for _, d in eq]),
                        points=np.stack(points), layout=np.array(layout), field_keys=np.array(keys), **fields)
    print("wrote %s: equilibria at steps %s" % (OUT, [s for s, _ in eq]))


if __name__ == "__main__":
    main()
