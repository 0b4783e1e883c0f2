"""Throughput of the force-and-dynamics loop: triangle-steps per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
                    [--workload disk1p8m] [--impl ours|reference]

Workload (default ``disk1p8m``): unit disk, jittered hexagonal lattice of
spacing 0.002 (908,139 nodes, 1,813,134 triangles), LCE dialling protocol 3
with an azimuthal director perturbed by 0.3 sin(3 theta) and lambda dialled
1 -> 0.85, bbar = 0, h = 0.01, nu = 0.5, unit modulus and density; seeded
synthetic inputs (there is no public dataset for this path).  A step is one
timestep of the dialling phase: surface derivatives, in-line dialling,
deformation forces, damping, constraints, force guard and symplectic Euler
update -- one kernel per step on the node-tiled paths (the warp-specialised
one is the default at this size).  Per-step traffic is ~0.7 GB, far above the 126 MB L2, so no flush is
needed between steps.

``value``: K * T * N / (max over ranks of the device time of K steps), FP64.
``mixed``: the same K steps on the mixed-precision path (FP32 per-triangle
arithmetic), with its ratio to FP64 and its force error against FP64.
``time_to_equilibrium``: learned warm start against the plain start on a
small disk (time_to_equilibrium()).
``e2e``: the same metric with the state on the host, through the C ABI, every
step: pinned host dofs + velocities copied in (ms_upload_dofs), one fused step
(ms_step_n), dofs + velocities copied back (ms_download_dofs).
Multi-GPU: one independent replica per GPU (the benchmark mesh fits one GPU);
``scaling`` is weak.

``--impl reference`` times the reference's own C++ (compiled from its source
files against oracle/eigen_shim; the port oracle if that build is absent) on
the host cores, with all threads, on the same mesh and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic bytes per triangle-step of the timed variant (FP64, protocol-3
# dialling evaluated in-kernel, bbar = 0): per triangle 6 int32 patch ids
# (24 B), 24 derivative weights (192 B), 3 abar_info columns (24 B) and the
# reference area (8 B); per node read+write of position and velocity
# (96 B) and the mass (8 B), i.e. 104 B per node = 52 B per triangle at
# N = T/2.  Mixed precision reads the 24 weights as float (the director
# trigonometry and the area stay double: they set abar, which the strain
# a - abar is formed against in double).
BYTES_PER_TRI = {"fp64": 24 + 192 + 24 + 8 + 52, "mixed": 24 + 96 + 24 + 8 + 52}
METRIC = "tri-steps/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_workload(name: str, seed: int = 1):
    from morphoshell_b200 import Model, meshgen
    mesh, info, bbar = meshgen.workload(name, seed=seed)
    d = tempfile.mkdtemp(prefix="ms_bench_")
    st = os.path.join(d, "settings.txt")
    meshgen.write_settings(st, protocol=3)
    model = Model.from_arrays(st, mesh.nodes, mesh.tris, info, bbar)
    return model, info, bbar


def dial_sequence(model, n: int) -> np.ndarray:
    s = model.scalars
    k = np.arange(n, dtype=np.float64)
    return 0.0 + s.dial_factors_to_hold_at_spacing * (k / float(s.timesteps_per_dial_phase))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(workload: str, precision: str, path: str):
    """DRAM bytes per step from the committed ncu summary, if one exists
    (lines ``workload precision path bytes``)."""
    p = os.path.join(ROOT, "profiles", "step_traffic.txt")
    try:
        with open(p) as f:
            for line in f:
                parts = line.split("#")[0].split()
                if len(parts) >= 4 and parts[:3] == [workload, precision, path]:
                    return float(parts[3])
    except OSError:
        pass
    return None


def cpu_baseline(model, info, bbar, budget_s: float = 20.0):
    """The reference's own CPU path on a bounded sample of this workload."""
    import oracle
    kind = "ref" if oracle.available("ref") else "orc"
    cores = os.cpu_count() or 1
    o = oracle.Oracle(kind, model, threads=cores)
    s = model.scalars
    o.set_programmed(3, info, bbar, s.dial_factors_to_hold_at_spacing)
    o.upload(model.dofs(1))
    dials = dial_sequence(model, 1000)
    t0 = time.perf_counter()
    o.step_n(1, dials[:1], s.timestep, s.damping_factor_1)
    one = time.perf_counter() - t0
    n = int(max(2, min(200, budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    o.step_n(n, dials[1:1 + n], s.timestep, s.damping_factor_1)
    el = time.perf_counter() - t0
    o.close()
    # One thread, a few steps (the reference's serial speed, for scale).
    o1 = oracle.Oracle(kind, model, threads=1)
    o1.set_programmed(3, info, bbar, s.dial_factors_to_hold_at_spacing)
    o1.upload(model.dofs(1))
    t0 = time.perf_counter()
    o1.step_n(1, dials[:1], s.timestep, s.damping_factor_1)
    one1 = time.perf_counter() - t0
    n1 = int(max(1, min(20, 0.25 * budget_s / max(one1, 1e-6))))
    t0 = time.perf_counter()
    o1.step_n(n1, dials[1:1 + n1], s.timestep, s.damping_factor_1)
    el1 = time.perf_counter() - t0
    o1.close()
    return {"value": model.num_tris * n / el, "unit": METRIC, "cores": cores,
            "kind": "reference" if kind == "ref" else "port",
            "sample": "%d steps of the full %d-triangle mesh (protocol-3 dialling) after 1 warm-up step, %d threads"
                      % (n, model.num_tris, cores),
            "note": SHIM_NOTE if kind == "ref" else "the oracle port (reference build absent)",
            "single_thread_value": model.num_tris * n1 / el1,
            "single_thread_sample": "%d steps, 1 thread" % n1}


# The reference's own code runs against this project's stand-in for Eigen 3
# (oracle/eigen_shim: Eigen is not installed and cannot be fetched here), so
# its sparse products and vector temporaries are the stand-in's.
SHIM_NOTE = ("reference sources compiled unmodified against oracle/eigen_shim, this project's stand-in for the "
             "Eigen 3 subset they use (Eigen is absent here); its sparse x dense product allocates a fresh result "
             "vector per call, and real Eigen's threaded product may run faster or slower")


def reference_workload(name: str, seed: int = 1):
    """The workload written to a settings file and a mesh file and set up by
    the reference's own code (oracle.RefSetup), with the programmed fields;
    the mesh generator is pure Python, so the process maps no library of
    this project."""
    import oracle
    from morphoshell_b200 import meshgen
    mesh, info, bbar = meshgen.workload(name, seed=seed)
    d = tempfile.mkdtemp(prefix="ms_ref_")
    st = os.path.join(d, "settings.txt")
    vtk = os.path.join(d, "%s.vtk" % name)
    meshgen.write_settings(st, protocol=3)
    meshgen.write_vtk(vtk, "%s seed %d" % (name, seed), mesh.nodes, mesh.tris, info, bbar,
                      ref_thicknesses=np.full(mesh.num_tris, 0.01))
    return oracle.RefSetup(st, vtk, mesh.num_nodes, mesh.num_tris), info, bbar


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    kind = "ref" if oracle.available("ref") else "orc"
    t0 = time.perf_counter()
    if kind == "ref":
        model, info, bbar = reference_workload(args.workload)
    else:
        model, info, bbar = make_workload(args.workload)
    setup_s = time.perf_counter() - t0
    cores = os.cpu_count() or 1
    o = oracle.Oracle(kind, model, threads=cores)
    s = model.scalars
    o.set_programmed(3, info, bbar, s.dial_factors_to_hold_at_spacing)
    o.upload(model.dofs(1))
    dials = dial_sequence(model, args.warmup + args.steps + 1)
    # W warm-up steps (each a full CPU step of the whole mesh), then as many
    # of the K steps as fit in ~60 s of host time.
    w = args.warmup
    t0 = time.perf_counter()
    o.step_n(w, dials[:w], s.timestep, s.damping_factor_1)
    one = (time.perf_counter() - t0) / max(w, 1)
    n = int(max(1, min(args.steps, 60.0 / max(one, 1e-9))))
    t0 = time.perf_counter()
    o.step_n(n, dials[w:w + n], s.timestep, s.damping_factor_1)
    el = time.perf_counter() - t0
    value = model.num_tris * n / el
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
        "steps": n, "warmup": w, "ms_per_step": 1e3 * el / n,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(args, model),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores,
                         "kind": "reference" if kind == "ref" else "port",
                         "sample": "%d of the requested %d steps of the full mesh, %d threads"
                                   % (n, args.steps, cores),
                         "note": SHIM_NOTE if kind == "ref" else "the oracle port (reference build absent)",
                         "setup": "the reference's own set-up code (read_settings, read_vtk_data, calc_mesh_info, "
                                  "set_up_patch_fitting, calc_dof_masses, noise)" if kind == "ref" else
                                  "this project's host set-up"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "setup_s": {"mesh_and_host": setup_s,
                    "note": "mesh generation, files written, then the reference's own set-up from them"},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(args, model):
    if args.workload == "disk1p8m":
        shape = "jittered hex spacing 0.002, wavy azimuthal director, lambda 1 -> 0.85"
    elif args.workload == "disk18k":
        shape = "jittered hex spacing 0.02, azimuthal director, lambda 1 -> 0.9"
    else:
        shape = "jittered hex spacing %g, azimuthal director, lambda 1 -> 0.9" % (int(args.workload[4:]) / 1000.0)
    return {"workload": "%s: unit disk, %s, %d nodes, %d triangles, LCE protocol-3 dialling, bbar = 0, h = 0.01, "
                        "nu = 0.5" % (args.workload, shape, model.num_nodes, model.num_tris),
            "precision": args.precision, "num_tris": model.num_tris, "num_nodes": model.num_nodes,
            "l2": ("inputs larger than L2 (%.2f GB of tables and node state per step vs 126 MB L2); no flush"
                   % (BYTES_PER_TRI["fp64"] * model.num_tris / 1e9)
                   if BYTES_PER_TRI["fp64"] * model.num_tris > 126e6 else
                   "working set smaller than L2 (a test-size workload); no flush"),
            "parallelism": "replicas x%d" % args.gpus}


KERNEL_NAMES = {"cluster": ("k_cluster_step", "k_halo_update"), "two-kernel": ("k_tri_aos", "k_node_update"),
                "tiles": ("k_tri_tiles", "k_node_update"), "node-tiles": ("k_node_tiles", None),
                "node-pipe": ("k_node_pipe", None)}
PATH_IDS = {"cluster": 0, "two-kernel": 1, "tiles": 2, "node-tiles": 3, "node-pipe": 4}


def timed_steps(model, info, bbar, precision, path, args, dials, local, dist, clock=None, setup=None):
    """One handle at `precision`: W warm-up steps, then K fused steps timed
    with CUDA events on the library's stream (barrier + synchronize on both
    sides, max over ranks), then the per-launch kernel times for the
    roofline.  Returns (handle, ms of the K steps, kernel ms, path name)."""
    import contextlib

    import torch
    from morphoshell_b200 import MS_PRECISION_FP64, MS_PRECISION_MIXED, GpuLoop
    s = model.scalars
    prec = MS_PRECISION_MIXED if precision == "mixed" else MS_PRECISION_FP64
    t0 = time.perf_counter()
    g = GpuLoop(model, precision=prec, device=local)
    if setup is not None:
        setup["device_s"] = time.perf_counter() - t0
    if path != "auto":
        g.set_step_path(PATH_IDS[path])
    path = {v: k for k, v in PATH_IDS.items()}[g.plan_info()["path"]]
    g.set_programmed(3, info, bbar, s.dial_factors_to_hold_at_spacing)
    g.upload(model.dofs(1))
    dt, damp = s.timestep, s.damping_factor_1
    g.step_n(args.warmup, dials[:args.warmup], dt, damp)
    # The CUDA graphs of the K-step call are built during the warm-up, as a
    # long-running loop builds them once.
    g.prepare_steps(args.steps, True, dt, damp)
    stream = torch.cuda.ExternalStream(g.stream(), device=torch.device("cuda", local))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with (clock or contextlib.nullcontext()):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        g.step_n(args.steps, dials[args.warmup:args.warmup + args.steps], dt, damp)
        e1.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    # Per-kernel device time for the roofline (CUDA events on the library's
    # stream, from a copy of the state so the run above stays as it ended).
    x, v = g.download()
    t_tri, t_node = g.time_kernels(50, dial=float(dials[args.warmup]), dt=dt, damping=damp)
    g.upload(x, v)
    tri_name, node_name = KERNEL_NAMES[path]
    kernel_ms = {tri_name: t_tri} if node_name is None else {tri_name: t_tri, node_name: t_node}
    return g, ms_max, kernel_ms, path


def roofline(model, precision, path, workload, kernel_ms, step_ms):
    """HBM roofline of the step.  A one-kernel step (one launch of the path's
    kernel per step, plus one k_chunk_end per captured graph of 128 steps)
    takes the mean launch duration from the timed region itself (its
    device time / K, so the chunk-end launches count against it); a
    two-kernel step takes the per-launch times of ms_time_kernels."""
    T = model.num_tris
    bpt = BYTES_PER_TRI[precision]
    one_kernel = KERNEL_NAMES[path][1] is None
    launch_ms = step_ms if one_kernel else sum(kernel_ms.values())
    achieved = bpt * T / (launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": profiled_traffic(workload, precision, path), "peak_kind": peak_kind,
            "kernel": "one step = " + " + ".join(kernel_ms), "algorithmic_bytes_per_tri": bpt,
            "launch_ms": launch_ms,
            "launch_ms_source": "timed region (device time / steps)" if one_kernel
            else "ms_time_kernels (CUDA events around each launch)",
            "kernel_ms_isolated": kernel_ms}


def launches(path, steps):
    per_step = 1 if KERNEL_NAMES[path][1] is None else 2
    return per_step * steps + (steps + 127) // 128  # + one chunk-end kernel per captured graph of 128 steps


def force_difference(model, g_a, g_b, x, v, dial):
    """max |F_a - F_b| / max |F_b| of the forces the fused step of each handle
    applies on the same state and dial factor (each in its own precision),
    recovered from one velocity update without damping: F = (v1 - v) m / dt."""
    dt = model.scalars.timestep
    mass = np.tile(model.tables()["node_mass"], 3)
    out = []
    for g in (g_a, g_b):
        g.upload(x, v)
        g.step_n(1, np.array([dial]), dt, 0.0)
        _, v1 = g.download()
        out.append((v1 - v) * mass / dt)
    return float(np.abs(out[0] - out[1]).max() / np.abs(out[1]).max())


def run_ours(args):
    import torch
    from morphoshell_b200 import lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    t0 = time.perf_counter()
    model, info, bbar = make_workload(args.workload)
    host_setup_s = time.perf_counter() - t0
    s = model.scalars
    T = model.num_tris
    dials = dial_sequence(model, args.warmup + args.steps + 64)
    dt, damp = s.timestep, s.damping_factor_1
    clk = ClockSampler(local)
    setup = {}
    g, ms_max, kernel_ms, path = timed_steps(model, info, bbar, args.precision, args.path, args, dials, local, dist,
                                             clock=clk, setup=setup)
    value = T * args.steps * world / (ms_max / 1e3)

    # End to end through the C ABI with the state on the host every step.
    N = model.num_nodes
    hx = torch.empty(3 * N, dtype=torch.float64, pin_memory=True).numpy()
    hv = torch.empty(3 * N, dtype=torch.float64, pin_memory=True).numpy()
    hx[:], hv[:] = g.download()
    e2e_steps = min(args.steps, 200)
    dl = dials[args.warmup:args.warmup + e2e_steps]
    stream = torch.cuda.ExternalStream(g.stream(), device=torch.device("cuda", local))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    L = lib()
    import ctypes as C
    pd = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    from morphoshell_b200 import ms_step_report
    rep = ms_step_report()
    for i in range(e2e_steps):
        L.ms_upload_dofs(g._h, pd(hx), pd(hv))
        one = np.ascontiguousarray(dl[i:i + 1])
        L.ms_step_n(g._h, 1, pd(one), 1, dt, damp, 0, 0, C.byref(rep))
        L.ms_download_dofs(g._h, pd(hx), pd(hv))
    e3.record(stream)
    torch.cuda.synchronize()
    t2 = torch.tensor([e2.elapsed_time(e3)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
    e2e_value = T * e2e_steps * world / (float(t2.item()) / 1e3)
    n_launch = launches(path, args.steps)

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32/f64 mixed", "data": "synthetic",
        "config": workload_config(args, model),
        "step_path": path,
        "gpu_launches": n_launch,
        "roofline": roofline(model, args.precision, path, args.workload, kernel_ms, ms_max / args.steps),
        "plan": g.plan_info(),
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 2 * 24 * N + 8,
                "d2h_bytes_per_step": 2 * 24 * N + 16, "steps": e2e_steps},
        "clocks": clk.summary(),
        "setup_s": {"mesh_and_host": host_setup_s, "device": setup.get("device_s"),
                    "note": "mesh generation + host set-up (Model.from_arrays), then ms_create (tables, plans, "
                            "uploads)"},
    }

    # The other half of the metric: the mixed-precision path on the same mesh,
    # steps and dial factors, with its force error against FP64 on the state
    # the FP64 run ended in.
    if args.precision == "fp64" and not args.no_mixed:
        clk_m = ClockSampler(local)
        gm, ms_m, kernel_m, path_m = timed_steps(model, info, bbar, "mixed", args.path, args, dials, local, dist,
                                                 clock=clk_m)
        xm, _ = gm.download()
        x64, v64 = g.download()
        dial_last = float(dials[args.warmup + args.steps - 1])
        ferr = force_difference(model, gm, g, x64, v64, dial_last)
        value_m = T * args.steps * world / (ms_m / 1e3)
        line["mixed"] = {
            "value": value_m, "unit": METRIC, "ms_per_step": ms_m / args.steps, "ratio_vs_fp64": value_m / value,
            "step_path": path_m, "roofline": roofline(model, "mixed", path_m, args.workload, kernel_m,
                                                               ms_m / args.steps),
            "max_force_err_vs_fp64": ferr,
            "max_position_diff_vs_fp64": float(np.abs(xm - x64).max() / np.abs(x64).max()),
            "force_err_state": "the FP64 run's final state, dial factor of its last step; forces from one "
                               "undamped velocity update of each path",
            "clocks": clk_m.summary()}
        line["gpu_launches"] = n_launch + launches(path_m, args.steps)
        gm.close()
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(model, info, bbar)
    g.close()
    if rank == 0 and world == 1 and not args.no_warmstart:
        line["time_to_equilibrium"] = time_to_equilibrium(local)
    if rank == 0 and world == 1 and not args.no_ensemble:
        # The batched-ensemble workload (256 disks of assorted sizes stepped
        # together) on the same GPU and precision, after the single-mesh runs
        # have released their memory.
        r = ensemble_measurement(256, args.precision, args.warmup, 200, local, None, 1, 0)
        r["unit"] = METRIC
        line["ensemble"] = r
        line["gpu_launches"] += r["gpu_launches"]
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def time_to_equilibrium(device: int, seed: int = 11) -> dict:
    """The metric's last part, at a reduced scale: time to the first
    equilibrium at dial factor 1 from the plain start and from the learned
    warm start (morphoshell_b200.warmstart).  The plain method's own
    equilibria of 64 seeded programmed fields (director theta + sum_k a_k
    sin(k theta + phi_k), lambda ~ U(0.8, 1.2)) on a 0.06-spacing disk train
    the tensor-core network; 16 held-out fields then run from both starts in
    one batch each.  Four short dial phases and thresholds 1e-5 / 1e-4 keep
    it to about a minute (the full-scale studies are 4096 fields on the 18k
    disk and 64 on the 1.8M disk)."""
    import tempfile as _tf

    from morphoshell_b200 import Mlp, Model, meshgen, warmstart
    t0 = time.time()
    d = _tf.mkdtemp(prefix="ms_tte_")
    st, vtk = meshgen.write_workload(d, "disk60", dial_factors_to_hold_at_spacing=0.25,
                                     dial_phase_time_prefactor=0.02, force_to_char_force_ratio_equil_threshold=1e-5,
                                     speed_to_char_speed_ratio_equil_threshold=1e-4)
    m = Model(st, vtk, quiet=True)
    train = warmstart.fields(64, seed=seed)
    held = warmstart.fields(16, seed=seed + 1)
    finals, _, status, _ = warmstart.solve(m, train)
    keep = [i for i, s_ in enumerate(status) if s_ == 3]
    net = Mlp(warmstart.N_FEATURES, width=128, hidden_layers=3, out_dim=3, seed=1, device=device)
    losses = warmstart.train_network(net, m, [train[i] for i in keep], [finals[i] for i in keep], epochs=300,
                                     batch=4096, lr=2e-3, rounds=3)
    r = warmstart.evaluate(net, m, held)
    net.close()
    return {"workload": "disk60: %d triangles, %d training fields, %d held out, 4 dial phases of 0.02 long times, "
                        "thresholds 1e-5 / 1e-4" % (m.num_tris, len(keep), len(held)),
            "plain_steps_mean": r["plain_steps_mean"], "learned_steps_mean": r["learned_steps_mean"],
            "step_speedup": r["step_speedup"], "plain_wall_s": r["plain_wall_s"], "learned_wall_s": r["learned_wall_s"],
            "wall_speedup": r["wall_speedup"], "fell_back": r["fell_back"],
            "same_shape_fraction": r["same_shape_fraction"],
            "energy_ratio_learned_to_plain": r["learned_energy_median"] / r["plain_energy_median"],
            "loss_first_last": [float(losses[0]), float(losses[-1])], "total_s": time.time() - t0,
            "note": "reduced-scale stand-in for the 4096-field 18k-disk and 64-field 1.8M-disk studies; same_shape_fraction is the share of held-out "
                    "fields whose learned-start equilibrium is the plain-start one"}


def ensemble_measurement(n: int, precision: str, warmup: int, steps: int, local: int, dist, world: int,
                         rank: int) -> dict:
    """N independent disks in one batch (ms_batch_*) on this rank's GPU,
    spacing log-uniform in [0.004, 0.02], lambda_final ~ U(0.8, 1.2), defect
    charge from {+1, -1, +1/2} (director angle = charge * theta), thickness
    ~ U(0.005, 0.02), seed 7.  Every instance runs its own dialling /
    equilibrium state machine on the device; the timed steps are
    ms_batch_run over the whole ensemble after the schedule autotuner
    (ms_batch_autotune) has chosen the step's kernels.  With N GPUs the
    members are split over the ranks by weight (strong scaling, no
    collective on the data path).  Returns the figures of one line."""
    import torch
    from morphoshell_b200 import MS_PRECISION_FP64, MS_PRECISION_MIXED, Batch, ensemble, meshgen

    # The members are split over the ranks by their triangle counts (about
    # 1 / spacing^2), so the whole ensemble is the workload at every N.
    weights = [1.0 / meshgen.ensemble_params(k, seed=7)["spacing"] ** 2 for k in range(n)]
    mine = ensemble.assign(n, world, rank, weights)
    t0 = time.time()
    cores = os.cpu_count() or 8
    models, params = ensemble.build_members(mine, tempfile.mkdtemp(prefix="ms_ens_"), seed=7,
                                            threads=cores, processes=min(cores, 32))
    setup_s = time.time() - t0
    log("ensemble of %d built in %.1f s" % (n, setup_s))
    prec = MS_PRECISION_MIXED if precision == "mixed" else MS_PRECISION_FP64
    b = Batch(models, precision=prec, device=local)
    info = b.info()
    T = info["num_tris"]
    sched, tune_ms = b.autotune(steps_per_trial=8)
    trials = b.autotune_report()
    b.run(warmup)
    stream = torch.cuda.ExternalStream(b.stream(), device=torch.device("cuda", local))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        done = b.run(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    tt = torch.tensor([float(T) * done], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(tt, op=dist.ReduceOp.SUM)
    ms_max = float(t.item())
    value = float(tt.item()) / (ms_max / 1e3)
    bpt = BYTES_PER_TRI[precision]
    achieved = bpt * T / (ms_max / done / 1e3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    sizes = [p["num_tris"] for p in params]
    if sched["tri_block"] < 0:
        kernels, per_step = "k_batch_pre + k_batch_node_tiles + k_batch_post (node-tiled schedule)", 3
    elif sched["tri_block"] == 0:
        kernels, per_step = "k_batch_pre + k_batch_tri_tiles + k_batch_node + k_batch_post (tiled schedule)", 4
    else:
        kernels, per_step = "k_batch_pre + k_batch_tri + k_batch_node + k_batch_post (per-thread schedule)", 4
    b.close()
    return {
        "value": value, "steps": done, "ms_per_step": ms_max / done,
        "workload": "ensemble%d: %d unit disks in one batch per GPU, spacing log-uniform [0.004, 0.02] "
                    "(%d..%d triangles, %d in all), lambda_final ~ U(0.8, 1.2), charge in "
                    "{+1, -1, +1/2}, h ~ U(0.005, 0.02), per-instance dialling state machines"
                    % (n, len(mine), min(sizes), max(sizes), T),
        "num_tris": T, "num_nodes": info["num_nodes"], "instances": n, "schedule": sched,
        "autotune_ms_per_step": tune_ms, "autotune_trials": trials, "host_setup_s": setup_s,
        "gpu_launches": per_step * done,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind, "kernel": kernels + ", whole step",
                     "algorithmic_bytes_per_tri": bpt},
        "clocks": clk.summary(),
    }


def run_ensemble(args):
    """``--workload ensembleN`` (default N = 256): the batch of N disks that
    ensemble_measurement describes, as its own line."""
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=1800),
                                device_id=torch.device("cuda", local))
    n = int(args.workload[len("ensemble"):] or 256)
    r = ensemble_measurement(n, args.precision, args.warmup, args.steps, local, dist, world, rank)
    line = {
        "metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": world, "steps": r["steps"],
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32/f64 mixed", "data": "synthetic",
        "config": {"workload": r["workload"], "precision": args.precision, "num_tris": r["num_tris"],
                   "num_nodes": r["num_nodes"], "instances": n, "schedule": r["schedule"],
                   "autotune_ms_per_step": r["autotune_ms_per_step"], "autotune_trials": r["autotune_trials"],
                   "host_setup_s": r["host_setup_s"],
                   "parallelism": "members split over %d GPUs" % world,
                   "l2": "inputs far larger than L2; no flush"},
        "gpu_launches": r["gpu_launches"],
        "roofline": r["roofline"],
        "clocks": r["clocks"],
    }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_mlp(args):
    """``--workload mlp``: training throughput of the warm-start network on
    the tensor cores (ms_mlp_train: tcgen05 BF16 GEMMs, FP32 accumulation,
    Adam), 22 -> 256 x 4 (SiLU) -> 3, batches of 32768 rows of 2^20 seeded
    synthetic rows (the node features' shape; no dataset exists).  A step is
    one epoch; value = FLOP/s of the forward and backward GEMMs."""
    import torch
    from morphoshell_b200 import Mlp, warmstart

    rows = 1 << 20
    rng = np.random.default_rng(0)
    x = rng.standard_normal((rows, warmstart.N_FEATURES)).astype(np.float32)
    t = np.stack([np.sin(x[:, 0]) * np.cos(x[:, 1]), 0.5 * x[:, 2] * x[:, 3], np.tanh(x[:, 4])], 1)
    net = Mlp(warmstart.N_FEATURES, width=256, hidden_layers=4, out_dim=3, seed=1)
    net.set_data(x, t.astype(np.float32))
    net.train(args.warmup, batch=32768, lr=1e-3, seed=0)
    stream = torch.cuda.ExternalStream(net.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        losses = net.train(args.steps, batch=32768, lr=1e-3, seed=1)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    flops = 3.0 * warmstart.network_flops_per_row(warmstart.N_FEATURES, 256, 4) * rows * args.steps
    tflops = flops / (ms / 1e3) / 1e12
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, peak_kind = float(json.load(f)["bf16_tflops_sustained"]), "measured (sustained)"
    except (OSError, KeyError, ValueError):
        peak, peak_kind = 1400.0, "fallback"
    line = {"metric": "TFLOP/s (network training)", "value": tflops, "unit": "TFLOP/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (fp32 accumulate)", "data": "synthetic",
            "config": {"workload": "mlp: warm-start network 22 -> 256 x 4 -> 3, %d rows per epoch, batch 32768" % rows,
                       "rows_per_s": rows * args.steps / (ms / 1e3), "loss_last": float(losses[-1])},
            "roofline": {"bound": "tensor", "achieved": tflops, "peak": peak, "unit": "TFLOP/s",
                         "frac": tflops / peak, "traffic": None, "peak_kind": peak_kind,
                         "kernel": "k_gemm (tcgen05, the whole training step incl. transposes, Adam, host loss reads)"},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--workload", default="disk1p8m")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision half of the line")
    ap.add_argument("--no-warmstart", action="store_true", help="skip the time-to-equilibrium part of the line")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 256-disk batched-ensemble part of the line")
    ap.add_argument("--path", choices=["auto", "cluster", "two-kernel", "tiles", "node-tiles", "node-pipe"],
                    default="auto",
                    help="fused-step implementation (ms_set_step_path); auto: the library's default")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload.startswith("ensemble"):
        return run_ensemble(args)
    if args.workload == "mlp":
        return run_mlp(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
