"""Learned warm start: a coordinate network that predicts a mesh's
equilibrium shape from its programmed field, used instead of the flat start
(or move_nodes_to_ansatz_positions, main.cpp:226-230) as the state the
damped dynamics begin from.

* Fields: director angle = theta + sum_{k<=4} a_k sin(k theta + phi_k),
  a_k ~ N(0, 0.2^2), phi_k ~ U(0, 2 pi), lambda_final ~ U(0.8, 1.2),
  nu_ot = 0.5 (dialling protocol 3, do_dialling.cpp:112-123).
* Training data: equilibria at dial factor 1 that the plain method itself
  reaches (the batched engine, ms_batch_*), one row per node: the node's
  features -> its displacement from the flat reference position.  A shape
  and its mirror image z -> -z are both equilibria of an in-plane metric
  with b-bar = 0, so targets are mirrored to a common orientation (mean
  displacement z >= 0).
* Network: ms_mlp_* (tensor-core BF16 SiLU MLP, FP32 accumulation, Adam).
* Warm start: predicted positions uploaded into a batch instance that waits
  for equilibrium at dial factor 1 (ms_batch_set_start).  The plain damped
  dynamics always run from there to full equilibrium and judge the start:
  a prediction that is not finite, or whose run trips the force guard or
  does not reach equilibrium, falls back to the plain start (optionally
  also one with more elastic energy at dial factor 1 than the flat start;
  a flat start is a stressed saddle whose energy is low next to a
  prediction with small-scale errors, so that test rejects useful starts).
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass

import numpy as np

from . import MS_INST_DONE, MS_INST_FAILED, MS_PRECISION_FP64, Batch, GpuLoop, Mlp

N_FEATURES = 22


@dataclass
class Field:
    a: np.ndarray      # (4,)
    phi: np.ndarray    # (4,)
    lam: float

    def angle(self, theta):
        k = np.arange(1, 5)
        return theta + (self.a[None, :] * np.sin(k[None, :] * np.asarray(theta)[:, None] + self.phi[None, :])).sum(1)


def random_field(rng) -> Field:
    return Field(a=rng.normal(0.0, 0.2, 4), phi=rng.uniform(0.0, 2.0 * math.pi, 4), lam=float(rng.uniform(0.8, 1.2)))


def fields(n: int, seed: int):
    rng = np.random.default_rng(seed)
    return [random_field(rng) for _ in range(n)]


def abar_info(model_tris_centroids: np.ndarray, f: Field) -> np.ndarray:
    """(T, 3) protocol-3 columns (angle, lambda_final, nu_ot) at triangle centroids."""
    c = model_tris_centroids
    theta = np.arctan2(c[:, 1], c[:, 0])
    ang = f.angle(theta)
    return np.ascontiguousarray(np.column_stack([ang, np.full_like(ang, f.lam), np.full_like(ang, 0.5)]))


def node_features(xy: np.ndarray, f: Field) -> np.ndarray:
    """Per-node inputs, all continuous at the disk's centre (where theta is
    undefined and the director has its defect): x, y, r, the harmonic
    polynomials r^k cos k theta, r^k sin k theta (k = 1..4), the director
    angle alpha as r cos 2 alpha, r sin 2 alpha (the programmed metric
    depends on 2 alpha), lambda_final, and the field's coefficients
    a_k cos phi_k, a_k sin phi_k (k = 1..4)."""
    x, y = xy[:, 0], xy[:, 1]
    r = np.hypot(x, y)
    theta = np.arctan2(y, x)
    alpha = f.angle(theta)
    cols = [x, y, r]
    for k in range(1, 5):
        rk = r ** k
        cols += [rk * np.cos(k * theta), rk * np.sin(k * theta)]
    cols += [r * np.cos(2 * alpha), r * np.sin(2 * alpha), np.full_like(x, f.lam)]
    for k in range(4):
        cols += [np.full_like(x, f.a[k] * math.cos(f.phi[k])), np.full_like(x, f.a[k] * math.sin(f.phi[k]))]
    return np.column_stack(cols).astype(np.float32)


def centroids(model) -> np.ndarray:
    from . import lib
    import ctypes as C
    T = model.num_tris
    tv = np.empty((T, 3), dtype=np.int32)
    lib().msh_get_tri_vertices(model._h, tv.ctypes.data_as(C.POINTER(C.c_int32)))
    ref = model.dofs(0).reshape(3, -1).T
    return ref[tv].mean(1)


def solve(model, flds, precision=MS_PRECISION_FP64, starts=None, max_steps=2_000_000, autotune=True):
    """Runs every field to its first equilibrium at dial factor 1 in one
    batch.  starts[i] (3N SoA positions or None) makes instance i a warm
    start waiting at dial factor 1.  Returns (final positions per field,
    steps per field, statuses, wall seconds of the batch run)."""
    cen = centroids(model)
    infos = [abar_info(cen, f) for f in flds]
    b = Batch([model] * len(flds), precision=precision, abar_infos=infos)
    if starts is not None:
        for i, x in enumerate(starts):
            if x is not None:
                b.upload(i, x)
                b.set_start(i, 1.0, True)
    if autotune:
        b.autotune(steps_per_trial=8)
    t0 = time.time()
    b.run(max_steps)
    wall = time.time() - t0
    out, steps, stat = [], [], []
    for i in range(len(flds)):
        st = b.status(i)
        out.append(b.download(i)[0])
        steps.append(st.stepcount)
        stat.append(st.status)
    b.close()
    return out, np.array(steps), np.array(stat), wall


def align(P: np.ndarray, Q: np.ndarray) -> np.ndarray:
    """P (N, 3) moved by the proper rigid motion that best matches it to Q
    in the least-squares sense (Kabsch).  Equilibria are defined up to
    rigid motions, and the damped dynamics of an unconstrained sheet drift
    and turn it."""
    pc, qc = P.mean(0), Q.mean(0)
    H = (P - pc).T @ (Q - qc)
    U, _, Vt = np.linalg.svd(H)
    d = np.sign(np.linalg.det(Vt.T @ U.T))
    D = np.diag([1.0, 1.0, d])
    R = Vt.T @ D @ U.T
    return (P - pc) @ R.T + qc


def shape_distance(a: np.ndarray, b: np.ndarray) -> float:
    """Largest node distance between two shapes (3N SoA) after the best
    rigid motion, allowing b's mirror image z -> -z."""
    A, B = a.reshape(3, -1).T, b.reshape(3, -1).T
    Bm = B * np.array([1.0, 1.0, -1.0])
    return float(min(np.abs(align(B, A) - A).max(), np.abs(align(Bm, A) - A).max()))


def canonical(disp: np.ndarray) -> np.ndarray:
    """(N, 3) displacement mirrored so that its mean z is >= 0."""
    d = disp.copy()
    if d[:, 2].mean() < 0:
        d[:, 2] = -d[:, 2]
    return d


def dataset(model, flds, finals):
    ref = model.dofs(0).reshape(3, -1).T
    xy = ref[:, :2]
    X, Y = [], []
    for f, x in zip(flds, finals):
        X.append(node_features(xy, f))
        Y.append(canonical(align(x.reshape(3, -1).T, ref) - ref).astype(np.float32))
    return np.concatenate(X), np.concatenate(Y)


def train_network(net: Mlp, model, flds, finals, epochs: int, batch: int = 8192, lr: float = 1e-3,
                  rounds: int = 3, seed: int = 1):
    """Trains on the equilibria of ``flds``.  Each equilibrium counts up to
    its mirror image: the first round uses the orientation with mean z >= 0,
    later rounds the orientation closer to the network's current prediction
    (so near-symmetric shapes, whose mean z is ~0, get a consistent
    orientation).  Returns the per-epoch losses."""
    ref = model.dofs(0).reshape(3, -1).T
    xy = ref[:, :2]
    N = ref.shape[0]
    X = np.concatenate([node_features(xy, f) for f in flds])
    disp = [align(x.reshape(3, -1).T, ref) - ref for x in finals]
    Y = np.concatenate([canonical(d) for d in disp]).astype(np.float32)
    losses = []
    per_round = max(1, epochs // max(rounds, 1))
    done = 0
    for r in range(max(rounds, 1)):
        n_ep = per_round if r < rounds - 1 else epochs - done
        if r > 0:
            pred = net.forward(X)
            for i, d in enumerate(disp):
                p = pred[i * N:(i + 1) * N]
                m = d.copy()
                m[:, 2] = -m[:, 2]
                Y[i * N:(i + 1) * N] = d if ((p - d) ** 2).sum() <= ((p - m) ** 2).sum() else m
        net.set_data(X, Y)
        losses += list(net.train(n_ep, batch=batch, lr=lr, seed=seed + r))
        done += n_ep
    return np.array(losses)


def predict_positions(net: Mlp, model, f: Field) -> np.ndarray:
    ref = model.dofs(0).reshape(3, -1).T
    d = net.forward(node_features(ref[:, :2], f))
    return np.ascontiguousarray((ref + d).T.ravel())


def elastic_energy(model, f: Field, x: np.ndarray) -> float:
    """Stretch + bend energy at dial factor 1 (calc_energies.cpp:44-63)."""
    g = GpuLoop(model)
    info = abar_info(centroids(model), f)
    _, b_info = model.programmed()
    g.set_programmed(3, info, b_info, model.scalars.dial_factors_to_hold_at_spacing)
    g.upload(x)
    g.do_dialling(1.0)
    e = g.output_quantities()["energies"]
    g.close()
    return float(e[0] + e[1])


def warm_starts(net: Mlp, model, flds, energy_check: bool = False):
    """Predicted start per field, or None (plain start) when the prediction
    is not finite (or, with energy_check, has more elastic energy at dial
    factor 1 than the flat start)."""
    flat = model.dofs(1)
    out, fell_back = [], 0
    for f in flds:
        x = predict_positions(net, model, f)
        ok = bool(np.all(np.isfinite(x)))
        if ok and energy_check:
            ok = elastic_energy(model, f, x) <= elastic_energy(model, f, flat)
        out.append(x if ok else None)
        fell_back += 0 if ok else 1
    return out, fell_back


def evaluate(net: Mlp, model, flds, precision=MS_PRECISION_FP64, max_steps=2_000_000, energy_check: bool = False):
    """Time to the first equilibrium at dial factor 1 from the plain start
    and from the learned start, and the distance between the two shapes.
    The plain dynamics run from every learned start; a start whose run
    trips the force guard or does not reach equilibrium within max_steps
    falls back to the plain start, and its time is the learned attempt plus
    the plain run."""
    plain, s_plain, st_plain, w_plain = solve(model, flds, precision, None, max_steps)
    starts, fell_back = warm_starts(net, model, flds, energy_check)
    budget = min(max_steps, int(2 * s_plain.max()) + 1000)
    learned, s_learn, st_learn, w_learn = solve(model, flds, precision, starts, budget)
    s_total = s_learn.astype(np.float64).copy()
    for i, st in enumerate(st_learn):
        if st != MS_INST_DONE:
            fell_back += 1
            learned[i] = plain[i]
            s_total[i] = s_learn[i] + s_plain[i]
        elif starts[i] is None:
            s_total[i] = s_plain[i]
    dist = [shape_distance(a, b) for a, b in zip(plain, learned)]
    start_dist = [shape_distance(x, p) for x, p in zip(starts, plain) if x is not None]
    e_plain = [elastic_energy(model, f, x) for f, x in zip(flds, plain)]
    e_learn = [elastic_energy(model, f, x) for f, x in zip(flds, learned)]
    return {
        "fields": len(flds), "fell_back": fell_back,
        "plain_steps_mean": float(s_plain.mean()), "learned_steps_mean": float(s_total.mean()),
        "step_speedup": float(s_plain.mean() / max(s_total.mean(), 1.0)),
        "step_speedup_median": float(np.median(s_plain / np.maximum(s_total, 1.0))),
        "plain_wall_s": w_plain, "learned_wall_s": w_learn, "wall_speedup": w_plain / max(w_learn, 1e-9),
        "plain_done": int((st_plain == MS_INST_DONE).sum()), "learned_done": int((st_learn == MS_INST_DONE).sum()),
        "failed": int((st_plain == MS_INST_FAILED).sum() + (st_learn == MS_INST_FAILED).sum()),
        "shape_distance_max": float(np.max(dist)), "shape_distance_median": float(np.median(dist)),
        "start_distance_median": float(np.median(start_dist)) if start_dist else None,
        "same_shape_fraction": float(np.mean(np.array(dist) < 0.05)),
        "plain_energy_median": float(np.median(e_plain)), "learned_energy_median": float(np.median(e_learn)),
        "learned_lower_energy_fraction": float(np.mean(np.array(e_learn) <= np.array(e_plain))),
    }


def network_flops_per_row(in_dim: int, width: int, hidden: int, out_dim: int = 3) -> float:
    """Multiply-adds x 2 of one forward pass per row (padded widths)."""
    in_pad = (in_dim + 15) // 16 * 16
    macs = in_pad * width + (hidden - 1) * width * width + width * 16
    return 2.0 * macs


def main(argv=None):
    """The warm-start experiment: plain-method equilibria of random fields
    train the network; on held-out fields, time to the first equilibrium at
    dial factor 1 from the plain start and from the learned start."""
    import argparse
    import json
    import os
    import tempfile

    from . import MS_PRECISION_MIXED, Model, meshgen

    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", default="disk18k")
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--held-out", type=int, default=256)
    ap.add_argument("--chunk", type=int, default=1024, help="fields per batch while generating data")
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--width", type=int, default=256)
    ap.add_argument("--hidden", type=int, default=4)
    ap.add_argument("--spacing", type=float, default=0.25, help="dial_factors_to_hold_at_spacing")
    ap.add_argument("--phase-prefactor", type=float, default=0.02, help="dial_phase_time_prefactor")
    ap.add_argument("--force-thr", type=float, default=1e-6)
    ap.add_argument("--speed-thr", type=float, default=1e-5)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--max-steps", type=int, default=3_000_000)
    ap.add_argument("--out", default="warmstart.json")
    a = ap.parse_args(argv)
    prec = MS_PRECISION_MIXED if a.precision == "mixed" else MS_PRECISION_FP64
    d = tempfile.mkdtemp(prefix="ms_ws_")
    st, vtk = meshgen.write_workload(d, a.mesh, dial_factors_to_hold_at_spacing=a.spacing,
                                     dial_phase_time_prefactor=a.phase_prefactor,
                                     force_to_char_force_ratio_equil_threshold=a.force_thr,
                                     speed_to_char_speed_ratio_equil_threshold=a.speed_thr)
    model = Model(st, vtk, quiet=True)
    report = {"mesh": a.mesh, "num_tris": model.num_tris, "num_nodes": model.num_nodes, "settings": vars(a)}
    train_f = fields(a.train, seed=100)
    held_f = fields(a.held_out, seed=200)

    import sys as _sys

    def note(msg):
        print("[warmstart %.0fs] %s" % (time.time() - t_start, msg), file=_sys.stderr, flush=True)

    t_start = time.time()
    note("model %s: %d nodes, %d triangles" % (a.mesh, model.num_nodes, model.num_tris))
    t0 = time.time()
    finals, steps, kept = [], [], []
    report["train_not_done"] = 0
    for c0 in range(0, len(train_f), a.chunk):
        part = train_f[c0:c0 + a.chunk]
        fx, sx, stx, _ = solve(model, part, prec, None, a.max_steps)
        for f, x, n_steps, status in zip(part, fx, sx, stx):
            if status == MS_INST_DONE:
                kept.append(f)
                finals.append(x)
                steps.append(n_steps)
            else:
                report["train_not_done"] += 1
        note("solved %d training fields (steps mean %.0f)" % (min(len(train_f), c0 + a.chunk), np.mean(sx)))
    report["datagen_s"] = time.time() - t0
    report["train_steps_mean"] = float(np.mean(steps))
    net = Mlp(N_FEATURES, width=a.width, hidden_layers=a.hidden, out_dim=3, seed=7)
    t0 = time.time()
    losses = train_network(net, model, kept, finals, a.epochs, batch=a.batch, lr=a.lr)
    train_s = time.time() - t0
    rows = len(kept) * model.num_nodes
    flops = 3.0 * network_flops_per_row(N_FEATURES, a.width, a.hidden) * rows * a.epochs
    report.update({"rows": int(rows), "train_s": train_s, "train_tflops": flops / train_s / 1e12,
                   "loss_first": float(losses[0]), "loss_last": float(losses[-1])})
    note("trained: loss %.3e -> %.3e in %.1fs" % (losses[0], losses[-1], train_s))
    report["eval"] = evaluate(net, model, held_f, prec, a.max_steps)
    note("evaluated")
    with open(a.out, "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps(report))
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
