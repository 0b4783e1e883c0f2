"""Synthetic disk meshes and programmed fields in MorphoShell's input VTK format.

The reference ships no meshes; its own meshing scripts (DistMesh + matplotlib)
cannot run here.  This module builds the seeded synthetic inputs the workloads
are defined on:

* a unit disk: a hexagonal lattice of spacing ``s`` with node jitter
  U(+-0.1 s), interior nodes kept at r <= 1 - s/2 and a ring of equally spaced
  boundary nodes at r = 1, Delaunay-triangulated (``scipy.spatial.Delaunay``);
* nodes and triangles relabelled along a Morton (Z-order) space-filling curve,
  playing the role of the reference's reverse-Cuthill-McKee relabelling
  (meshing_scripts/mesh_processing_module.py:53-140): spatially close
  elements get close labels;
* ``abar_info`` columns for the LCE dialling protocol (director angle,
  final lambda, opto-thermal Poisson ratio), as read by
  source_files/do_dialling.cpp:112-123 (protocol 3);
* the legacy-VTK POLYDATA layout written by
  meshing_scripts/mesh_processing_module.py:523-595 (``write_VTK``) and read
  by source_files/read_vtk_data.cpp:65-371.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class DiskMesh:
    nodes: np.ndarray      # (N, 3) float64 reference positions (z = 0)
    tris: np.ndarray       # (T, 3) int32 vertex ids, counter-clockwise
    boundary: np.ndarray   # (N,) bool, node lies on r = 1

    @property
    def num_nodes(self) -> int:
        return int(self.nodes.shape[0])

    @property
    def num_tris(self) -> int:
        return int(self.tris.shape[0])

    def centroids(self) -> np.ndarray:
        return self.nodes[self.tris].mean(axis=1)


def _morton_keys(xy: np.ndarray, bits: int = 20) -> np.ndarray:
    """Interleave the bits of quantised (x, y) into a 2*bits Z-order key."""
    lo = xy.min(axis=0)
    span = float(max((xy.max(axis=0) - lo).max(), 1e-300))
    q = np.floor((xy - lo) / span * ((1 << bits) - 1)).astype(np.uint64)

    def spread(v: np.ndarray) -> np.ndarray:
        v = v & np.uint64(0x00000000FFFFFFFF)
        v = (v | (v << np.uint64(16))) & np.uint64(0x0000FFFF0000FFFF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF00FF00FF)
        v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F0F0F0F0F)
        v = (v | (v << np.uint64(2))) & np.uint64(0x3333333333333333)
        v = (v | (v << np.uint64(1))) & np.uint64(0x5555555555555555)
        return v

    return spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1))


def sfc_relabel(nodes: np.ndarray, tris: np.ndarray, boundary: np.ndarray):
    """Relabel nodes by the Z-order of their positions and triangles by the
    Z-order of their centroids (stable, so ties keep their old order)."""
    node_order = np.argsort(_morton_keys(nodes[:, :2]), kind="stable")
    new_label = np.empty_like(node_order)
    new_label[node_order] = np.arange(node_order.size)
    nodes = nodes[node_order]
    boundary = boundary[node_order]
    tris = new_label[tris]
    cent = nodes[tris].mean(axis=1)
    tri_order = np.argsort(_morton_keys(cent[:, :2]), kind="stable")
    return nodes, tris[tri_order].astype(np.int32), boundary


def disk_mesh(spacing: float, seed: int = 0, jitter: float = 0.1,
              radius: float = 1.0, reorder: bool = True) -> DiskMesh:
    """Jittered-hexagonal Delaunay mesh of a disk of the given radius."""
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    s = float(spacing)
    dy = s * math.sqrt(3.0) / 2.0
    nrow = int(math.ceil(radius / dy)) + 1
    ncol = int(math.ceil(radius / s)) + 2
    j = np.arange(-nrow, nrow + 1)
    i = np.arange(-ncol, ncol + 1)
    jj, ii = np.meshgrid(j, i, indexing="ij")
    x = ii * s + (jj % 2) * (s / 2.0)
    y = jj * dy
    pts = np.column_stack([x.ravel(), y.ravel()])
    r = np.hypot(pts[:, 0], pts[:, 1])
    pts = pts[r <= radius - 0.5 * s]
    pts = pts + rng.uniform(-jitter * s, jitter * s, size=pts.shape)
    # Re-clip after jitter so that no interior node crowds the boundary ring.
    pts = pts[np.hypot(pts[:, 0], pts[:, 1]) <= radius - 0.4 * s]

    nb = max(12, int(round(2.0 * math.pi * radius / s)))
    phi0 = rng.uniform(0.0, 2.0 * math.pi / nb)
    phi = phi0 + 2.0 * math.pi * np.arange(nb) / nb
    phi = phi + rng.uniform(-jitter, jitter, size=nb) * (2.0 * math.pi / nb)
    bpts = radius * np.column_stack([np.cos(phi), np.sin(phi)])

    allpts = np.vstack([pts, bpts])
    boundary = np.zeros(allpts.shape[0], dtype=bool)
    boundary[pts.shape[0]:] = True
    tri = Delaunay(allpts).simplices.astype(np.int64)

    # Orient counter-clockwise and drop degenerate triangles (zero area).
    p = allpts[tri]
    area2 = ((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1])
             - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))
    flip = area2 < 0
    tri[flip] = tri[flip][:, [0, 2, 1]]
    tri = tri[np.abs(area2) > 1e-12 * s * s]

    # Drop nodes no triangle touches (cannot happen for a Delaunay of these
    # points, but keeps the topology identities of calc_mesh_info honest).
    used = np.zeros(allpts.shape[0], dtype=bool)
    used[tri.ravel()] = True
    remap = -np.ones(allpts.shape[0], dtype=np.int64)
    remap[used] = np.arange(int(used.sum()))
    allpts = allpts[used]
    boundary = boundary[used]
    tri = remap[tri]

    nodes = np.column_stack([allpts, np.zeros(allpts.shape[0])])
    if reorder:
        nodes, tri, boundary = sfc_relabel(nodes, tri, boundary)
    return DiskMesh(nodes=np.ascontiguousarray(nodes, dtype=np.float64),
                    tris=np.ascontiguousarray(tri, dtype=np.int32),
                    boundary=boundary)


def lce_abar_info(mesh: DiskMesh, director_angle, lam_final, nu_ot=0.5) -> np.ndarray:
    """(T, 3) rows of (director angle, final lambda, opto-thermal Poisson ratio)
    at triangle centroids; ``director_angle`` maps (theta, r) arrays to angles,
    ``lam_final`` is a scalar or a (T,) array."""
    c = mesh.centroids()
    theta = np.arctan2(c[:, 1], c[:, 0])
    rr = np.hypot(c[:, 0], c[:, 1])
    ang = np.asarray(director_angle(theta, rr), dtype=np.float64)
    lam = np.broadcast_to(np.asarray(lam_final, dtype=np.float64), ang.shape)
    nu = np.broadcast_to(np.asarray(nu_ot, dtype=np.float64), ang.shape)
    return np.ascontiguousarray(np.column_stack([ang, lam, nu]))


def lce_abar_comps(abar_info: np.ndarray, dial_factor: float) -> np.ndarray:
    """Metric components (xx, xy, yy) of protocol 3 at a dial factor; numpy
    restatement of source_files/do_dialling.cpp:112-123 used by the fixture
    generators (protocol-1 inputs are final metrics, not LCE columns)."""
    ang, lamf, nu = abar_info[:, 0], abar_info[:, 1], abar_info[:, 2]
    lam = (1.0 - dial_factor) * 1.0 + dial_factor * lamf
    c, s = np.cos(ang), np.sin(ang)
    p = lam ** (-2.0 * nu)
    return np.column_stack([lam * lam * c * c + p * s * s,
                            (lam * lam - p) * c * s,
                            p * c * c + lam * lam * s * s])


def write_vtk(path: str, header: str, nodes: np.ndarray, tris: np.ndarray,
              abar_info: np.ndarray, bbar_info: np.ndarray,
              ref_thicknesses=None, ref_shear_moduli=None, tri_tags=None,
              constraint_indicators=None, node_tags=None) -> None:
    """Write the reference's input file (legacy VTK POLYDATA subset)."""
    n = nodes.shape[0]
    t = tris.shape[0]
    if nodes.shape[1] == 2:
        nodes = np.column_stack([nodes, np.zeros(n)])
    ones_t = np.ones(t)
    ref_thicknesses = ones_t if ref_thicknesses is None else np.asarray(ref_thicknesses)
    ref_shear_moduli = ones_t if ref_shear_moduli is None else np.asarray(ref_shear_moduli)
    tri_tags = np.zeros(t, dtype=int) if tri_tags is None else np.asarray(tri_tags, dtype=int)
    constraint_indicators = (np.zeros(n, dtype=int) if constraint_indicators is None
                             else np.asarray(constraint_indicators, dtype=int))
    node_tags = np.zeros(n, dtype=int) if node_tags is None else np.asarray(node_tags, dtype=int)
    abar_info = np.atleast_2d(np.asarray(abar_info, dtype=np.float64))
    bbar_info = np.atleast_2d(np.asarray(bbar_info, dtype=np.float64))
    fp = "%.15e"
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 2.0\n%s\nASCII\nDATASET POLYDATA\n" % header)
        f.write("POINTS %d double\n" % n)
        np.savetxt(f, nodes, fmt=fp, delimiter=" ")
        f.write("POLYGONS %d %d\n" % (t, 4 * t))
        np.savetxt(f, np.column_stack([3 * np.ones(t, dtype=int), tris]), fmt="%d", delimiter=" ")
        f.write("CELL_DATA %d\nFIELD tri_quantities 5\n" % t)
        f.write("abar_info %d %d double\n" % (abar_info.shape[1], t))
        np.savetxt(f, abar_info, fmt=fp, delimiter=" ")
        f.write("bbar_info %d %d double\n" % (bbar_info.shape[1], t))
        np.savetxt(f, bbar_info, fmt=fp, delimiter=" ")
        f.write("ref_thicknesses 1 %d double\n" % t)
        np.savetxt(f, ref_thicknesses.reshape(-1, 1), fmt=fp)
        f.write("ref_shear_moduli 1 %d double\n" % t)
        np.savetxt(f, ref_shear_moduli.reshape(-1, 1), fmt=fp)
        f.write("tri_tags 1 %d int\n" % t)
        np.savetxt(f, tri_tags.reshape(-1, 1), fmt="%d")
        f.write("POINT_DATA %d\nFIELD node_quantities 2\n" % n)
        f.write("constraint_indicators 1 %d int\n" % n)
        np.savetxt(f, constraint_indicators.reshape(-1, 1), fmt="%d")
        f.write("node_tags 1 %d int\n" % n)
        np.savetxt(f, node_tags.reshape(-1, 1), fmt="%d")


# ---------------------------------------------------------------------------
# The named workloads.

def azimuthal_director(theta, r):
    """+1 defect with the director along circles (azimuthal)."""
    return theta + 0.5 * math.pi


def wavy_azimuthal_director(theta, r):
    """Azimuthal director perturbed by 0.3 sin(3 theta)."""
    return theta + 0.5 * math.pi + 0.3 * np.sin(3.0 * theta)


def workload(name: str, seed: int = 1):
    """(mesh, abar_info, bbar_info, settings overrides) of a named workload.

    ``disk18k``: spacing 0.02, azimuthal director, lambda 1 -> 0.9 (about
    9.1k nodes, 18k triangles).  ``disk1p8m``: spacing 0.002, wavy azimuthal
    director, lambda 1 -> 0.85 (about 0.9M nodes, 1.8M triangles).  ``diskN``
    with N a spacing in thousandths (e.g. ``disk50``) gives smaller meshes of
    the first kind for tests."""
    if name == "disk18k":
        mesh = disk_mesh(0.02, seed=seed)
        info = lce_abar_info(mesh, azimuthal_director, 0.9)
    elif name == "disk1p8m":
        mesh = disk_mesh(0.002, seed=seed)
        info = lce_abar_info(mesh, wavy_azimuthal_director, 0.85)
    elif name.startswith("disk") and name[4:].isdigit():
        mesh = disk_mesh(int(name[4:]) / 1000.0, seed=seed)
        info = lce_abar_info(mesh, azimuthal_director, 0.9)
    else:
        raise ValueError("unknown workload %r" % name)
    bbar = np.zeros((mesh.num_tris, 3))
    return mesh, info, bbar


# Settings in the reference's order (source_files/read_settings.cpp:90-188),
# defaults from its shipped example; ``dialling_protocol`` is this project's
# optional trailing setting.
SETTINGS_ORDER = [
    ("outputs_per_char_long_time", -1.0),
    ("ref_thickness_if_uniform", 0.01),
    ("timestep_prefactor", 0.6),
    ("dialling_from_ansatz_rather_than_ref_state", False),
    ("dial_factors_to_hold_at_spacing", 0.05),
    ("dial_phase_time_prefactor", 0.25),
    ("time_between_equil_checks_prefactor", 0.01),
    ("damping_prefactor_1", 35.0),
    ("damping_prefactor_2", 35.0),
    ("num_steps_to_use_gradient_descent_dynamics_for_before_switching_to_newtonian_dynamics", 0),
    ("force_to_char_force_ratio_equil_threshold", 1e-6),
    ("speed_to_char_speed_ratio_equil_threshold", 1e-5),
    ("def_poisson_ratio", 0.5),
    ("ref_shear_modulus_if_uniform", 1.0),
    ("ref_density", 1.0),
    ("bend_stiffening_scale_factor", 1e17),
    ("patch_mat_dimless_conditioning_thresh", 10.0),
    ("slide_stiffness_prefactor", 0.0),
    ("slide_friction_coefficent", 0.0),
    ("slide_speed_prefactor", 0.0),
    ("using_initial_glass_slide_z_coords_from_settings_file", False),
    ("initial_upper_slide_z_coord", 12345.0),
    ("initial_lower_slide_z_coord", 12345.0),
]


def _fmt(v) -> str:
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int):
        return str(v)
    return repr(float(v))


def write_settings(path: str, protocol: int | None = 3, **overrides) -> None:
    """Write a settings file; ``protocol=None`` omits the trailing
    ``dialling_protocol`` line (the reference's own format)."""
    known = dict(SETTINGS_ORDER)
    for k in overrides:
        if k not in known:
            raise KeyError(k)
    with open(path, "w") as f:
        f.write("// MorphoShell settings (generated)\n")
        for k, v in SETTINGS_ORDER:
            f.write("%s = %s;\n" % (k, _fmt(overrides.get(k, v))))
        if protocol is not None:
            f.write("dialling_protocol = %d;\n" % protocol)


def ensemble_member(k: int, seed: int = 7, spacing_range=(0.004, 0.02)):
    """Member k of the batched-ensemble workload: mesh spacing log-uniform
    over ``spacing_range``, lambda_final ~ U(0.8, 1.2), defect charge drawn
    from {+1, -1, +1/2} with director angle = charge * theta, thickness
    ~ U(0.005, 0.02), b-bar = 0.  Deterministic in (seed, k).  Returns
    (mesh, abar_info, bbar_info, settings overrides, parameters)."""
    params = ensemble_params(k, seed, spacing_range)
    mesh = disk_mesh(params["spacing"], seed=params["mesh_seed"])
    charge = params["charge"]
    info = lce_abar_info(mesh, lambda th, r: charge * th, params["lam_final"])
    bbar = np.zeros((mesh.num_tris, 3))
    return mesh, info, bbar, {"ref_thickness_if_uniform": params["thickness"]}, params


def ensemble_params(k: int, seed: int = 7, spacing_range=(0.004, 0.02)) -> dict:
    """The random draws of ensemble_member k, without building its mesh."""
    rng = np.random.default_rng([seed, k])
    lo, hi = spacing_range
    spacing = float(np.exp(rng.uniform(math.log(lo), math.log(hi))))
    lam = float(rng.uniform(0.8, 1.2))
    charge = (1.0, -1.0, 0.5)[int(rng.integers(3))]
    h = float(rng.uniform(0.005, 0.02))
    return {"spacing": spacing, "lam_final": lam, "charge": charge, "thickness": h,
            "mesh_seed": int(rng.integers(1 << 31))}


def write_workload(directory: str, name: str, seed: int = 1, protocol: int = 3, **settings):
    """Write ``<name>.vtk`` and ``<name>_settings.txt`` into directory and
    return their paths."""
    import os
    os.makedirs(directory, exist_ok=True)
    mesh, info, bbar = workload(name, seed=seed)
    vtk = os.path.join(directory, "%s.vtk" % name)
    st = os.path.join(directory, "%s_settings.txt" % name)
    write_vtk(vtk, "%s seed %d" % (name, seed), mesh.nodes, mesh.tris, info, bbar,
              ref_thicknesses=np.full(mesh.num_tris, settings.get("ref_thickness_if_uniform", 0.01)))
    write_settings(st, protocol=protocol, **settings)
    return st, vtk
