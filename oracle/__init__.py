"""CPU oracles of the force-and-dynamics loop -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
bench.py as the checker; never by the product (morphoshell_b200).

* ``Oracle("orc", model)``: this project's C++ restatement
  (oracle/morpho_oracle.cpp, oracle/lib/libmorpho_oracle.so);
* ``Oracle("ref", model)``: the reference's own source files compiled
  unmodified against oracle/eigen_shim (oracle/_ref/libmorpho_ref.so,
  present only where oracle/build.py could see the reference tree).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "lib", "libmorpho_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libmorpho_ref.so")
REF_EXE = os.path.join(HERE, "_ref", "morphoshell_ref")
REF_EXE_P3 = os.path.join(HERE, "_ref", "morphoshell_ref_p3")

_libs: dict = {}


def available(kind: str) -> bool:
    return os.path.exists(PORT_LIB if kind == "orc" else REF_LIB)


def _load(kind: str):
    if kind in _libs:
        return _libs[kind]
    path = PORT_LIB if kind == "orc" else REF_LIB
    if not os.path.exists(path):
        raise RuntimeError("oracle library %s is missing (python oracle/build.py)" % path)
    L = C.CDLL(path)
    d = C.POINTER(C.c_double)
    i32 = C.POINTER(C.c_int32)
    u8 = C.POINTER(C.c_uint8)
    f = lambda n: getattr(L, "%s_%s" % (kind, n))
    f("create").argtypes = [C.c_int, C.c_int, d, i32, d, d, d, d, d, d, u8, u8, d]
    f("create").restype = C.c_void_p
    f("destroy").argtypes = [C.c_void_p]
    f("set_programmed").argtypes = [C.c_void_p, C.c_int, d, C.c_int, d, C.c_int, C.c_double, C.c_int]
    f("set_zero_dial_state").argtypes = [C.c_void_p, d, d]
    f("set_state").argtypes = [C.c_void_p, d, d]
    f("get_state").argtypes = [C.c_void_p, d, d]
    f("get_forces").argtypes = [C.c_void_p, d]
    f("do_dialling").argtypes = [C.c_void_p, C.c_double]
    f("get_programmed").argtypes = [C.c_void_p, d, d]
    f("surface_derivs").argtypes = [C.c_void_p, d]
    f("a_b_normals").argtypes = [C.c_void_p, d, d, d]
    f("deformation_forces").argtypes = [C.c_void_p, d, d]
    f("non_deformation_forces").argtypes = [C.c_void_p, C.c_double, C.c_int]
    f("impose_constraints").argtypes = [C.c_void_p]
    f("is_at_equilibrium").argtypes = [C.c_void_p, d]
    f("advance_dynamics").argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.POINTER(C.c_int64), d]
    f("step_n").argtypes = [C.c_void_p, C.c_int, d, C.c_double, C.c_double, C.c_int, C.POINTER(C.c_int)]
    f("output_quantities").argtypes = [C.c_void_p, d, d, d, d, d, d]
    f("set_threads").argtypes = [C.c_int]
    _libs[kind] = L
    return L


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def read_settings_file(path: str) -> dict:
    """``name = value;`` lines of a settings file (read_settings.cpp:47-264's
    format) as a dict of floats (booleans as 0/1)."""
    out = {}
    with open(path) as f:
        for line in f:
            line = line.split("//")[0].strip()
            if "=" not in line or not line.endswith(";"):
                continue
            k, v = (x.strip() for x in line[:-1].split("=", 1))
            out[k] = {"true": 1.0, "false": 0.0}.get(v, None)
            if out[k] is None:
                out[k] = float(v)
    return out


class _NS:
    def __init__(self, **kw):
        self.__dict__.update(kw)


class RefSetup:
    """A workload set up by the reference's own code alone
    (``ref_setup_full``: read_settings, read_vtk_data, calc_mesh_info,
    set_up_patch_fitting, calc_dof_masses, the scales, timestep and dialling
    schedule, perturb_node_positions_with_noise; main.cpp:91-209), in the
    shape ``Oracle`` takes (num_nodes, num_tris, tables(), dofs(), scalars,
    params), so that a reference run maps no library of this project."""

    def __init__(self, settings_path: str, vtk_path: str, num_nodes: int, num_tris: int):
        if not available("ref"):
            raise RuntimeError("reference build absent (python oracle/build.py --reference DIR)")
        L = _load("ref")
        d = C.POINTER(C.c_double)
        u8 = C.POINTER(C.c_uint8)
        f = L.ref_setup_full
        f.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int32), d, d, d,
                      d, d, d, d, d, u8, u8, C.c_char_p, C.c_int]
        N, T = num_nodes, num_tris
        self.num_nodes, self.num_tris = N, T
        patch = np.zeros((T, 6), np.int32)
        mat2 = np.zeros((T, 18))
        mass, dofs0, scal = np.zeros(N), np.zeros(3 * N), np.zeros(14)
        ref_pos = np.zeros((N, 3))
        area, thick, shear = np.zeros(T), np.zeros(T), np.zeros(T)
        fixed, boundary = np.zeros(N, np.uint8), np.zeros(N, np.uint8)
        err = C.create_string_buffer(512)
        n, t = C.c_int(), C.c_int()
        rc = f(settings_path.encode(), vtk_path.encode(), C.byref(n), C.byref(t),
               patch.ctypes.data_as(C.POINTER(C.c_int32)), _dp(mat2), _dp(mass), _dp(dofs0), _dp(scal),
               _dp(ref_pos), _dp(area), _dp(thick), _dp(shear), fixed.ctypes.data_as(u8),
               boundary.ctypes.data_as(u8), err, 512)
        if rc != 0:
            raise RuntimeError("reference set-up failed: %s" % err.value.decode(errors="replace"))
        if (n.value, t.value) != (N, T):
            raise RuntimeError("reference set-up read %d nodes / %d triangles, expected %d / %d"
                               % (n.value, t.value, N, T))
        coeffs = np.zeros((T, 24))
        coeffs[:, 6:] = mat2  # the reference builds its first-derivative weights itself (calc_deriv_mats)
        self._tables = {"patch_ids": patch, "deriv_coeffs": coeffs, "node_mass": mass, "ref_area": area,
                        "ref_thickness": thick, "ref_shear_modulus": shear, "is_constrained": fixed,
                        "is_boundary": boundary}
        self._flat = ref_pos.T.reshape(-1).copy()
        self._dofs0 = dofs0
        st = read_settings_file(settings_path)
        self.scalars = _NS(min_ref_thickness=scal[2], char_force_scale=scal[3], char_speed_scale=scal[4],
                           damping_factor_1=scal[6], timestep=scal[7], timesteps_per_dial_phase=int(scal[8]),
                           timesteps_between_equil_checks=int(scal[9]), damping_factor_2=scal[13],
                           dial_factors_to_hold_at_spacing=st["dial_factors_to_hold_at_spacing"])
        self.params = _NS(def_poisson_ratio=st["def_poisson_ratio"],
                          bend_stiffening_scale_factor=st["bend_stiffening_scale_factor"],
                          ref_density=st["ref_density"], min_ref_thickness=scal[2], char_force_scale=scal[3],
                          char_speed_scale=scal[4],
                          force_to_char_force_ratio_equil_threshold=st["force_to_char_force_ratio_equil_threshold"],
                          speed_to_char_speed_ratio_equil_threshold=st["speed_to_char_speed_ratio_equil_threshold"])

    def tables(self) -> dict:
        return self._tables

    def dofs(self, which: int = 1) -> np.ndarray:
        """SoA dofs: 0 the flat reference state, 1 after the initial noise."""
        return (self._flat if which == 0 else self._dofs0).copy()


class Oracle:
    """One CPU oracle instance over a ``morphoshell_b200.Model``'s tables."""

    def __init__(self, kind: str, model, threads: int | None = None):
        self.kind = kind
        self.L = _load(kind)
        tb = model.tables()
        self.N, self.T = model.num_nodes, model.num_tris
        ref = model.dofs(0).reshape(3, self.N).T.copy()
        s = model.scalars
        p = model.params
        self._keep = [np.ascontiguousarray(ref), tb]
        mat2 = np.ascontiguousarray(tb["deriv_coeffs"][:, 6:])
        self._keep.append(mat2)
        scal = np.array([p.def_poisson_ratio, p.bend_stiffening_scale_factor, p.ref_density, p.min_ref_thickness,
                         p.char_force_scale, p.char_speed_scale, p.force_to_char_force_ratio_equil_threshold,
                         p.speed_to_char_speed_ratio_equil_threshold, 0.0])
        self._keep.append(scal)
        u8 = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint8))
        if threads:
            self.fn("set_threads")(threads)
        self.h = self.fn("create")(
            self.N, self.T, _dp(self._keep[0]), tb["patch_ids"].ctypes.data_as(C.POINTER(C.c_int32)), _dp(mat2),
            _dp(tb["deriv_coeffs"]), _dp(tb["node_mass"]), _dp(tb["ref_area"]), _dp(tb["ref_thickness"]),
            _dp(tb["ref_shear_modulus"]), u8(tb["is_constrained"]), u8(tb["is_boundary"]), _dp(scal))
        self.scalars = s

    def fn(self, name):
        return getattr(self.L, "%s_%s" % (self.kind, name))

    def close(self):
        if getattr(self, "h", None):
            self.fn("destroy")(self.h)
            self.h = None

    __del__ = close

    def set_programmed(self, protocol, abar_info, bbar_info, spacing, from_ansatz=False):
        a = np.ascontiguousarray(abar_info, dtype=np.float64)
        b = np.ascontiguousarray(bbar_info, dtype=np.float64)
        rc = self.fn("set_programmed")(self.h, protocol, _dp(a), a.shape[1], _dp(b), b.shape[1], spacing,
                                       int(from_ansatz))
        if rc != 0:
            raise RuntimeError("%s_set_programmed: status %d" % (self.kind, rc))

    def set_zero_dial_state(self, a0=None, b0=None):
        a0 = None if a0 is None else np.ascontiguousarray(a0, dtype=np.float64)
        b0 = None if b0 is None else np.ascontiguousarray(b0, dtype=np.float64)
        self.fn("set_zero_dial_state")(self.h, _dp(a0), _dp(b0))

    def upload(self, dofs, vel=None):
        x = np.ascontiguousarray(dofs, dtype=np.float64)
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        self.fn("set_state")(self.h, _dp(x), _dp(v))

    def download(self):
        x, v = np.empty(3 * self.N), np.empty(3 * self.N)
        self.fn("get_state")(self.h, _dp(x), _dp(v))
        return x, v

    def forces(self):
        f = np.empty(3 * self.N)
        self.fn("get_forces")(self.h, _dp(f))
        return f

    def do_dialling(self, dial):
        self.fn("do_dialling")(self.h, dial)

    def programmed(self):
        a, b = np.empty((self.T, 3)), np.empty((self.T, 3))
        self.fn("get_programmed")(self.h, _dp(a), _dp(b))
        return a, b

    def surface_derivs(self):
        cq = np.empty(15 * self.T)
        self.fn("surface_derivs")(self.h, _dp(cq))
        return cq

    def a_b_normals(self):
        a, b, n = (np.empty((self.T, 3)) for _ in range(3))
        self.fn("a_b_normals")(self.h, _dp(a), _dp(b), _dp(n))
        return a, b, n

    def deformation_forces(self):
        f, de = np.empty(3 * self.N), np.empty(15 * self.T)
        self.fn("deformation_forces")(self.h, _dp(f), _dp(de))
        return f, de

    def non_deformation_forces(self, damping, gd=False):
        self.fn("non_deformation_forces")(self.h, damping, int(gd))

    def impose_constraints(self):
        self.fn("impose_constraints")(self.h)

    def is_at_equilibrium(self):
        out = np.empty(4)
        eq = self.fn("is_at_equilibrium")(self.h, _dp(out))
        return bool(eq), out

    def advance_dynamics(self, dt, damping, gd=False):
        dof = C.c_int64(-1)
        f = np.zeros(1)
        rc = self.fn("advance_dynamics")(self.h, dt, damping, int(gd), C.byref(dof), _dp(f))
        return rc, dof.value, float(f[0])

    def step_n(self, n, dials=None, dt=0.0, damping=0.0, gd=False):
        dl = None if dials is None else np.ascontiguousarray(dials, dtype=np.float64)
        done = C.c_int(0)
        rc = self.fn("step_n")(self.h, n, _dp(dl), dt, damping, int(gd), C.byref(done))
        return rc, done.value

    def output_quantities(self):
        T, N = self.T, self.N
        curv, ed = np.empty((T, 2)), np.empty((T, 2))
        strain, stress, dfc, en = np.empty(T), np.empty((T, 8)), np.empty(N), np.empty(3)
        self.fn("output_quantities")(self.h, _dp(curv), _dp(ed), _dp(strain), _dp(stress), _dp(dfc), _dp(en))
        return {"curvatures": curv, "energy_densities": ed, "strains": strain, "stresses": stress,
                "angle_deficits": dfc, "energies": en}
