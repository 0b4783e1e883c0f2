"""B200-native force-and-dynamics loop of MorphoShell.

Python access to the native library ``lib/libmorphoshell.so`` (host set-up
plus sm_100a kernels) through its C ABI (``include/morphoshell_gpu.h`` and
``include/morphoshell_host.h``).  There is no Python or CPU implementation of
the per-step physics here: if the library is missing or no GPU is present,
the GPU calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libmorphoshell.so")

MS_OK = 0
MS_ERR_IMPLAUSIBLE_FORCE = 3
MS_PRECISION_FP64 = 0
MS_PRECISION_MIXED = 1

GPU_SYMBOLS = [
    "ms_create", "ms_destroy", "ms_last_error", "ms_status_string", "ms_upload_dofs", "ms_download_dofs",
    "ms_download_forces", "ms_set_programmed", "ms_set_zero_dial_state", "ms_do_dialling",
    "ms_download_programmed", "ms_surface_derivs", "ms_a_b_normals", "ms_deformation_forces",
    "ms_non_deformation_forces", "ms_impose_constraints", "ms_is_at_equilibrium", "ms_advance_dynamics",
    "ms_step_n", "ms_prepare_steps", "ms_output_quantities", "ms_device_info", "ms_stream", "ms_time_kernels",
    "ms_deformation_forces_noalloc", "ms_set_step_path", "ms_plan_info", "ms_node_tile_layout", "ms_node_tile_plan",
    "ms_batch_create", "ms_batch_destroy", "ms_batch_last_error", "ms_batch_run", "ms_batch_status",
    "ms_batch_download_dofs", "ms_batch_upload_dofs", "ms_batch_set_schedule", "ms_batch_get_schedule",
    "ms_batch_autotune", "ms_batch_autotune_report", "ms_batch_info", "ms_batch_stream", "ms_batch_set_start",
    "ms_mlp_create", "ms_mlp_destroy", "ms_mlp_last_error", "ms_mlp_num_params", "ms_mlp_get_params",
    "ms_mlp_set_params", "ms_mlp_forward", "ms_mlp_loss_grad", "ms_mlp_set_data", "ms_mlp_train", "ms_mlp_stream",
]
HOST_SYMBOLS = [
    "msh_load", "msh_build", "msh_free", "msh_last_error", "msh_get_scalars", "msh_get_desc", "msh_get_dofs",
    "msh_get_programmed", "msh_get_tri_vertices", "msh_get_boundary", "msh_run", "msh_run_batch",
]


class MsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class ms_mesh_desc(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("num_tris", C.c_int32), ("patch_ids", C.POINTER(C.c_int32)),
                ("deriv_coeffs", C.POINTER(C.c_double)), ("ref_area", C.POINTER(C.c_double)),
                ("ref_thickness", C.POINTER(C.c_double)), ("ref_shear_modulus", C.POINTER(C.c_double)),
                ("node_mass", C.POINTER(C.c_double)), ("is_constrained", C.POINTER(C.c_uint8)),
                ("is_boundary", C.POINTER(C.c_uint8))]


class ms_params(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "def_poisson_ratio", "bend_stiffening_scale_factor", "ref_density", "min_ref_thickness",
        "char_force_scale", "char_speed_scale", "force_to_char_force_ratio_equil_threshold",
        "speed_to_char_speed_ratio_equil_threshold")]


class ms_equil_result(C.Structure):
    _fields_ = [("max_force", C.c_double), ("max_speed", C.c_double), ("max_force_node", C.c_int64),
                ("max_speed_node", C.c_int64), ("at_equilibrium", C.c_int32)]


class ms_step_report(C.Structure):
    _fields_ = [("steps_done", C.c_int32), ("error_step", C.c_int32), ("offending_dof", C.c_int64),
                ("offending_force", C.c_double), ("equil", ms_equil_result)]


class msh_scalars(C.Structure):
    _fields_ = ([(n, C.c_int32) for n in ("num_nodes", "num_tris", "num_edges", "num_boundary_nodes",
                                          "num_boundary_edges", "dialling_protocol", "dialling_from_ansatz",
                                          "using_gradient_descent_dynamics", "num_gd_steps", "output_regularly")]
                + [(n, C.c_int64) for n in ("steps_between_outputs", "timesteps_per_dial_phase",
                                            "timesteps_between_equil_checks")]
                + [(n, C.c_double) for n in (
                    "sample_char_length", "approx_min_tri_size", "min_ref_thickness", "min_ref_shear_modulus",
                    "char_long_time", "dial_phase_time", "timestep", "damping_factor_1", "damping_factor_2",
                    "char_force_scale", "char_speed_scale", "char_stretch_energy_density_scale", "total_ref_area",
                    "dial_factors_to_hold_at_spacing", "dial_factor_to_start_from", "def_poisson_ratio",
                    "bend_stiffening_scale_factor", "ref_density", "force_thresh", "speed_thresh")])


class msh_run_options(C.Structure):
    _fields_ = [("max_steps", C.c_int64), ("stop_at_final_equilibrium", C.c_int32), ("write_outputs", C.c_int32),
                ("precision", C.c_int32), ("device", C.c_int32), ("quiet", C.c_int32), ("output_dir", C.c_char_p)]


class msh_run_result(C.Structure):
    _fields_ = [("status", C.c_int32), ("steps", C.c_int64), ("final_dial_factor", C.c_double),
                ("sim_time", C.c_double), ("equilibria_reached", C.c_int32), ("final_status", C.c_int32),
                ("wall_seconds", C.c_double), ("last_max_force_ratio", C.c_double),
                ("last_max_speed_ratio", C.c_double)]


class ms_node_tile_info(C.Structure):
    _fields_ = [("tiles", C.c_int), ("chunks", C.c_int), ("tri_tile_pairs", C.c_longlong),
                ("node_section_max", C.c_longlong), ("record_stride", C.c_longlong),
                ("bytes_per_step", C.c_longlong), ("shared_bytes", C.c_longlong),
                ("sliced_entries", C.c_longlong), ("pipe_shared_bytes", C.c_longlong)]


class ms_batch_instance(C.Structure):
    _fields_ = [("mesh", ms_mesh_desc), ("params", ms_params), ("abar_info", C.POINTER(C.c_double)),
                ("timestep", C.c_double), ("damping_factor_1", C.c_double), ("damping_factor_2", C.c_double),
                ("timesteps_per_dial_phase", C.c_int64), ("timesteps_between_equil_checks", C.c_int64),
                ("dial_factors_to_hold_at_spacing", C.c_double), ("dial_factor_to_start_from", C.c_double),
                ("stop_at_final_equilibrium", C.c_int32), ("dofs", C.POINTER(C.c_double)),
                ("velocities", C.POINTER(C.c_double))]


class ms_batch_inst_status(C.Structure):
    _fields_ = [("status", C.c_int32), ("equilibria", C.c_int32), ("stepcount", C.c_int64),
                ("dial_factor", C.c_double), ("last_equil_dial", C.c_double), ("sim_time", C.c_double),
                ("max_force_ratio", C.c_double), ("max_speed_ratio", C.c_double), ("max_force_node", C.c_int64),
                ("max_speed_node", C.c_int64), ("offending_dof", C.c_int64)]


class ms_batch_schedule(C.Structure):
    _fields_ = [("tri_block", C.c_int32), ("node_block", C.c_int32), ("chunk_steps", C.c_int32),
                ("nodes_per_tile", C.c_int32), ("blocks_per_sm", C.c_int32)]


MS_INST_DIALLING, MS_INST_WAITING, MS_INST_EQUIL, MS_INST_DONE, MS_INST_FAILED = range(5)

_lib = None


def lib() -> C.CDLL:
    """The loaded native library (built in-tree by ``morphoshell_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("native library %s is missing; run `python -m morphoshell_b200.build`" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        d = C.POINTER(C.c_double)
        L.ms_create.argtypes = [P(ms_mesh_desc), P(ms_params), C.c_int, C.c_int, P(C.c_void_p)]
        L.ms_destroy.argtypes = [C.c_void_p]
        L.ms_last_error.argtypes = [C.c_void_p]
        L.ms_last_error.restype = C.c_char_p
        L.ms_status_string.argtypes = [C.c_int]
        L.ms_status_string.restype = C.c_char_p
        L.ms_upload_dofs.argtypes = [C.c_void_p, d, d]
        L.ms_download_dofs.argtypes = [C.c_void_p, d, d]
        L.ms_download_forces.argtypes = [C.c_void_p, d]
        L.ms_set_programmed.argtypes = [C.c_void_p, C.c_int, d, C.c_int, d, C.c_int, C.c_double, C.c_int]
        L.ms_set_zero_dial_state.argtypes = [C.c_void_p, d, d]
        L.ms_do_dialling.argtypes = [C.c_void_p, C.c_double]
        L.ms_download_programmed.argtypes = [C.c_void_p, d, d]
        L.ms_surface_derivs.argtypes = [C.c_void_p, d]
        L.ms_a_b_normals.argtypes = [C.c_void_p, d, d, d]
        L.ms_deformation_forces.argtypes = [C.c_void_p, d, d]
        L.ms_non_deformation_forces.argtypes = [C.c_void_p, C.c_double, C.c_int]
        L.ms_impose_constraints.argtypes = [C.c_void_p]
        L.ms_is_at_equilibrium.argtypes = [C.c_void_p, P(ms_equil_result)]
        L.ms_advance_dynamics.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, P(C.c_int64), d]
        L.ms_step_n.argtypes = [C.c_void_p, C.c_int, d, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                P(ms_step_report)]
        L.ms_prepare_steps.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int]
        L.ms_output_quantities.argtypes = [C.c_void_p, d, d, d, d, d, d]
        L.ms_device_info.argtypes = [C.c_char_p, C.c_size_t]
        L.ms_deformation_forces_noalloc.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                                    C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p,
                                                    C.c_size_t]
        L.ms_set_step_path.argtypes = [C.c_void_p, C.c_int]
        ip = C.POINTER(C.c_int)
        L.ms_plan_info.argtypes = [C.c_void_p, ip, ip, ip, ip, ip]
        L.ms_node_tile_plan.argtypes = [C.c_void_p, ip, ip, ip, ip]
        L.ms_node_tile_layout.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, P(ms_node_tile_info)]
        L.ms_stream.argtypes = [C.c_void_p]
        L.ms_stream.restype = C.c_void_p
        L.ms_time_kernels.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, d, d]
        L.ms_batch_create.argtypes = [P(ms_batch_instance), C.c_int32, C.c_int32, C.c_int32, P(C.c_void_p)]
        L.ms_batch_destroy.argtypes = [C.c_void_p]
        L.ms_batch_destroy.restype = None
        L.ms_batch_last_error.argtypes = [C.c_void_p]
        L.ms_batch_last_error.restype = C.c_char_p
        L.ms_batch_run.argtypes = [C.c_void_p, C.c_int64, P(C.c_int64)]
        L.ms_batch_status.argtypes = [C.c_void_p, C.c_int32, P(ms_batch_inst_status)]
        L.ms_batch_download_dofs.argtypes = [C.c_void_p, C.c_int32, d, d]
        L.ms_batch_upload_dofs.argtypes = [C.c_void_p, C.c_int32, d, d]
        L.ms_batch_set_schedule.argtypes = [C.c_void_p, P(ms_batch_schedule)]
        L.ms_batch_set_start.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_int32]
        L.ms_batch_get_schedule.argtypes = [C.c_void_p, P(ms_batch_schedule)]
        L.ms_batch_autotune.argtypes = [C.c_void_p, C.c_int32, P(ms_batch_schedule), d]
        L.ms_batch_autotune_report.argtypes = [C.c_void_p, C.c_char_p, C.c_int32]
        L.ms_batch_autotune_report.restype = C.c_int32
        i64p = C.POINTER(C.c_int64)
        L.ms_batch_info.argtypes = [C.c_void_p, i64p, i64p, P(C.c_int32)]
        L.ms_batch_stream.argtypes = [C.c_void_p]
        L.ms_batch_stream.restype = C.c_void_p
        fp = C.POINTER(C.c_float)
        L.ms_mlp_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_int32,
                                    P(C.c_void_p)]
        L.ms_mlp_destroy.argtypes = [C.c_void_p]
        L.ms_mlp_destroy.restype = None
        L.ms_mlp_last_error.argtypes = [C.c_void_p]
        L.ms_mlp_last_error.restype = C.c_char_p
        L.ms_mlp_num_params.argtypes = [C.c_void_p, i64p]
        L.ms_mlp_get_params.argtypes = [C.c_void_p, fp]
        L.ms_mlp_set_params.argtypes = [C.c_void_p, fp]
        L.ms_mlp_forward.argtypes = [C.c_void_p, fp, C.c_int64, fp]
        L.ms_mlp_loss_grad.argtypes = [C.c_void_p, fp, fp, C.c_int64, d, fp]
        L.ms_mlp_set_data.argtypes = [C.c_void_p, fp, fp, C.c_int64]
        L.ms_mlp_train.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_uint64, fp]
        L.ms_mlp_stream.argtypes = [C.c_void_p]
        L.ms_mlp_stream.restype = C.c_void_p
        L.msh_run_batch.argtypes = [P(C.c_void_p), C.c_int32, P(msh_run_options), P(msh_run_result),
                                    P(C.POINTER(C.c_double))]
        L.msh_load.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, P(C.c_void_p)]
        L.msh_build.argtypes = [C.c_char_p, C.c_int32, C.c_int32, d, P(C.c_int32), d, C.c_int32, d, C.c_int32,
                                d, d, P(C.c_uint8), C.c_int, P(C.c_void_p)]
        L.msh_free.argtypes = [C.c_void_p]
        L.msh_free.restype = None
        L.msh_last_error.restype = C.c_char_p
        L.msh_get_scalars.argtypes = [C.c_void_p, P(msh_scalars)]
        L.msh_get_desc.argtypes = [C.c_void_p, P(ms_mesh_desc), P(ms_params)]
        L.msh_get_dofs.argtypes = [C.c_void_p, C.c_int, d]
        L.msh_get_programmed.argtypes = [C.c_void_p, d, P(C.c_int32), d, P(C.c_int32)]
        L.msh_get_tri_vertices.argtypes = [C.c_void_p, P(C.c_int32)]
        L.msh_get_boundary.argtypes = [C.c_void_p, P(C.c_uint8)]
        L.msh_run.argtypes = [C.c_void_p, P(msh_run_options), P(msh_run_result), d]
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Model:
    """Host set-up of one run (msh_load): settings + mesh (+ ansatz)."""

    def __init__(self, settings_path: str, vtk_path: str | None, ansatz_path: str | None = None,
                 quiet: bool = True, noise: bool = True, device_setup: bool = False, _handle=None):
        """device_setup: patch search, patch fit and derivative weights on the
        current CUDA device (the host set-up's results, bit for bit)."""
        L = lib()
        if _handle is None:
            h = C.c_void_p()
            flags = (1 if quiet else 0) | (0 if noise else 2) | (4 if device_setup else 0)
            rc = L.msh_load(settings_path.encode(), vtk_path.encode(),
                            ansatz_path.encode() if ansatz_path else None, flags, C.byref(h))
            if rc != 0:
                raise RuntimeError(L.msh_last_error().decode())
        else:
            h = _handle
        self._h = h
        s = msh_scalars()
        L.msh_get_scalars(h, C.byref(s))
        self.scalars = s
        self.desc = ms_mesh_desc()
        self.params = ms_params()
        L.msh_get_desc(h, C.byref(self.desc), C.byref(self.params))

    @classmethod
    def from_arrays(cls, settings_path: str, positions, tris, abar_info, bbar_info, thickness=None,
                    shear_modulus=None, constrained=None, quiet: bool = True, noise: bool = True,
                    device_setup: bool = False) -> "Model":
        """Set-up from in-memory mesh arrays (msh_build) instead of a VTK file;
        device_setup as for the constructor."""
        L = lib()
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        if pos.shape[1] == 2:
            pos = np.ascontiguousarray(np.column_stack([pos, np.zeros(len(pos))]))
        tri = np.ascontiguousarray(tris, dtype=np.int32)
        a = np.ascontiguousarray(abar_info, dtype=np.float64)
        b = np.ascontiguousarray(bbar_info, dtype=np.float64)
        th = None if thickness is None else np.ascontiguousarray(thickness, dtype=np.float64)
        sm = None if shear_modulus is None else np.ascontiguousarray(shear_modulus, dtype=np.float64)
        cn = None if constrained is None else np.ascontiguousarray(constrained, dtype=np.uint8)
        h = C.c_void_p()
        flags = (1 if quiet else 0) | (0 if noise else 2) | (4 if device_setup else 0)
        rc = L.msh_build(settings_path.encode(), pos.shape[0], tri.shape[0], _dp(pos),
                         tri.ctypes.data_as(C.POINTER(C.c_int32)), _dp(a), a.shape[1], _dp(b), b.shape[1], _dp(th),
                         _dp(sm), None if cn is None else cn.ctypes.data_as(C.POINTER(C.c_uint8)), flags, C.byref(h))
        if rc != 0:
            raise RuntimeError(L.msh_last_error().decode())
        return cls(settings_path, None, _handle=h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().msh_free(self._h)
            self._h = None

    @property
    def num_nodes(self) -> int:
        return self.scalars.num_nodes

    @property
    def num_tris(self) -> int:
        return self.scalars.num_tris

    def dofs(self, which: int = 1) -> np.ndarray:
        out = np.empty(3 * self.num_nodes)
        lib().msh_get_dofs(self._h, which, _dp(out))
        return out

    def programmed(self):
        ka, kb = C.c_int32(), C.c_int32()
        lib().msh_get_programmed(self._h, None, C.byref(ka), None, C.byref(kb))
        a = np.empty((self.num_tris, ka.value))
        b = np.empty((self.num_tris, kb.value))
        lib().msh_get_programmed(self._h, _dp(a), None, _dp(b), None)
        return a, b

    def tables(self) -> dict:
        """numpy copies of the mesh tables handed to ms_create."""
        d, T, N = self.desc, self.num_tris, self.num_nodes
        np_ = np.ctypeslib.as_array
        return {
            "patch_ids": np_(d.patch_ids, (T * 6,)).reshape(T, 6).copy(),
            "deriv_coeffs": np_(d.deriv_coeffs, (T * 24,)).reshape(T, 24).copy(),
            "ref_area": np_(d.ref_area, (T,)).copy(),
            "ref_thickness": np_(d.ref_thickness, (T,)).copy(),
            "ref_shear_modulus": np_(d.ref_shear_modulus, (T,)).copy(),
            "node_mass": np_(d.node_mass, (N,)).copy(),
            "is_constrained": np_(d.is_constrained, (N,)).copy(),
            "is_boundary": np_(d.is_boundary, (N,)).copy(),
        }

    def run(self, max_steps: int = 0, precision: int = MS_PRECISION_FP64, output_dir: str | None = None,
            stop_at_final_equilibrium: bool = True, quiet: bool = True, device: int = -1):
        o = msh_run_options(max_steps, int(stop_at_final_equilibrium), 1 if output_dir else 0, precision, device,
                            int(quiet), output_dir.encode() if output_dir else None)
        r = msh_run_result()
        out = np.empty(3 * self.num_nodes)
        rc = lib().msh_run(self._h, C.byref(o), C.byref(r), _dp(out))
        if rc != 0 and r.status != MS_ERR_IMPLAUSIBLE_FORCE:
            raise RuntimeError(lib().msh_last_error().decode())
        return r, out


class GpuLoop:
    """One device handle (ms_create) over a Model's tables."""

    def __init__(self, model: Model, precision: int = MS_PRECISION_FP64, device: int = -1):
        L = lib()
        h = C.c_void_p()
        rc = L.ms_create(C.byref(model.desc), C.byref(model.params), device, precision, C.byref(h))
        if rc != MS_OK:
            raise MsError(rc, "ms_create: %s" % L.ms_status_string(rc).decode())
        self._h = h
        self.N = model.num_nodes
        self.T = model.num_tris
        self.model = model

    def close(self):
        if getattr(self, "_h", None):
            lib().ms_destroy(self._h)
            self._h = None

    __del__ = close

    def _chk(self, rc, what):
        if rc != MS_OK:
            raise MsError(rc, "%s: %s (%s)" % (what, lib().ms_status_string(rc).decode(),
                                                lib().ms_last_error(self._h).decode()))

    def upload(self, dofs, vel=None):
        self._chk(lib().ms_upload_dofs(self._h, _dp(_f64(dofs)), _dp(None if vel is None else _f64(vel))), "upload")

    def download(self):
        x = np.empty(3 * self.N)
        v = np.empty(3 * self.N)
        self._chk(lib().ms_download_dofs(self._h, _dp(x), _dp(v)), "download")
        return x, v

    def forces(self):
        f = np.empty(3 * self.N)
        self._chk(lib().ms_download_forces(self._h, _dp(f)), "forces")
        return f

    def set_programmed(self, protocol, abar_info, bbar_info, spacing, from_ansatz=False):
        a, b = _f64(abar_info), _f64(bbar_info)
        self._a, self._b = a, b
        self._chk(lib().ms_set_programmed(self._h, protocol, _dp(a), a.shape[1], _dp(b), b.shape[1], spacing,
                                          int(from_ansatz)), "set_programmed")

    def set_zero_dial_state(self, a0=None, b0=None):
        self._chk(lib().ms_set_zero_dial_state(self._h, _dp(None if a0 is None else _f64(a0)),
                                               _dp(None if b0 is None else _f64(b0))), "set_zero_dial_state")

    def do_dialling(self, dial):
        self._chk(lib().ms_do_dialling(self._h, dial), "do_dialling")

    def programmed(self):
        a = np.empty((self.T, 3))
        b = np.empty((self.T, 3))
        self._chk(lib().ms_download_programmed(self._h, _dp(a), _dp(b)), "download_programmed")
        return a, b

    def surface_derivs(self):
        cq = np.empty(15 * self.T)
        self._chk(lib().ms_surface_derivs(self._h, _dp(cq)), "surface_derivs")
        return cq

    def a_b_normals(self):
        a, b, n = (np.empty((self.T, 3)) for _ in range(3))
        self._chk(lib().ms_a_b_normals(self._h, _dp(a), _dp(b), _dp(n)), "a_b_normals")
        return a, b, n

    def deformation_forces(self):
        f = np.empty(3 * self.N)
        de = np.empty(15 * self.T)
        self._chk(lib().ms_deformation_forces(self._h, _dp(f), _dp(de)), "deformation_forces")
        return f, de

    def non_deformation_forces(self, damping, gd=False):
        self._chk(lib().ms_non_deformation_forces(self._h, damping, int(gd)), "non_deformation_forces")

    def impose_constraints(self):
        self._chk(lib().ms_impose_constraints(self._h), "impose_constraints")

    def is_at_equilibrium(self):
        r = ms_equil_result()
        self._chk(lib().ms_is_at_equilibrium(self._h, C.byref(r)), "is_at_equilibrium")
        return r

    def advance_dynamics(self, dt, damping, gd=False):
        dof = C.c_int64(-1)
        f = C.c_double(0.0)
        rc = lib().ms_advance_dynamics(self._h, dt, damping, int(gd), C.byref(dof), C.byref(f))
        if rc == MS_ERR_IMPLAUSIBLE_FORCE:
            raise MsError(rc, "implausibly_high_force (dof %d, force %g)" % (dof.value, f.value))
        self._chk(rc, "advance_dynamics")

    def step_n(self, n, dials=None, dt=0.0, damping=0.0, gd=False, check_last=False):
        rep = ms_step_report()
        dl = None if dials is None else _f64(dials)
        rc = lib().ms_step_n(self._h, n, _dp(dl), 0 if dl is None else 1, dt, damping, int(gd), int(check_last),
                             C.byref(rep))
        if rc == MS_ERR_IMPLAUSIBLE_FORCE:
            err = MsError(rc, "implausibly_high_force at step %d (dof %d)" % (rep.error_step, rep.offending_dof))
            err.report = rep
            raise err
        self._chk(rc, "step_n")
        return rep

    def prepare_steps(self, n, dialling=True, dt=0.0, damping=0.0, gd=False, check_last=False):
        """Build the CUDA graphs step_n(n, ...) with these arguments will use,
        without running any step."""
        self._chk(lib().ms_prepare_steps(self._h, n, int(dialling), dt, damping, int(gd), int(check_last)),
                  "prepare_steps")

    def set_step_path(self, path: int):
        """0: cluster-tiled step, 1: two-kernel step, 2: two-kernel step with
        the per-triangle tables fed by bulk asynchronous copies, 3: node-tiled
        one-kernel step (forces summed in shared memory per tile of nodes),
        4: the node-tiled step with warp-specialised roles (two warpgroups
        compute triangles while a third sums and updates nodes; the default
        on meshes with a node tile for every SM)."""
        self._chk(lib().ms_set_step_path(self._h, path), "set_step_path")

    def plan_info(self) -> dict:
        v = [C.c_int() for _ in range(5)]
        self._chk(lib().ms_plan_info(self._h, *[C.byref(x) for x in v]), "plan_info")
        out = dict(zip(["cluster_size", "tris_per_cta", "clusters", "halo_nodes", "path"], [x.value for x in v]))
        w = [C.c_int() for _ in range(4)]
        self._chk(lib().ms_node_tile_plan(self._h, *[C.byref(x) for x in w]), "node_tile_plan")
        out.update(zip(["nodes_per_tile", "node_tiles", "node_tile_chunks", "node_tile_blocks"], [x.value for x in w]))
        return out

    def stream(self) -> int:
        """cudaStream_t of this handle, as an integer."""
        return lib().ms_stream(self._h) or 0

    def time_kernels(self, reps, dial=None, dt=0.0, damping=0.0):
        """Mean device ms per launch of (per-triangle kernel, per-node kernel)."""
        a, b = np.zeros(1), np.zeros(1)
        self._chk(lib().ms_time_kernels(self._h, reps, 0 if dial is None else 1, 0.0 if dial is None else dial, dt,
                                        damping, _dp(a), _dp(b)), "time_kernels")
        return float(a[0]), float(b[0])

    def output_quantities(self):
        T, N = self.T, self.N
        curv, ed = np.empty((T, 2)), np.empty((T, 2))
        strain, stress, dfc, en = np.empty(T), np.empty((T, 8)), np.empty(N), np.empty(3)
        self._chk(lib().ms_output_quantities(self._h, _dp(curv), _dp(ed), _dp(strain), _dp(stress), _dp(dfc),
                                             _dp(en)), "output_quantities")
        return {"curvatures": curv, "energy_densities": ed, "strains": strain, "stresses": stress,
                "angle_deficits": dfc, "energies": en}


class Batch:
    """Many Models stepped together on one device (ms_batch_*): each runs its
    own dialling / waiting / equilibrium state machine; see
    include/morphoshell_gpu.h."""

    def __init__(self, models, precision: int = MS_PRECISION_FP64, device: int = -1, dofs=None,
                 stop_at_final_equilibrium: bool = True, abar_infos=None):
        """``models`` may repeat one Model (a shared mesh); ``abar_infos[i]``
        (T x 3, optional) then gives instance i its own protocol-3 field."""
        L = lib()
        n = len(models)
        arr = (ms_batch_instance * n)()
        self._keep = []
        for i, m in enumerate(models):
            s = m.scalars
            if abar_infos is not None and abar_infos[i] is not None:
                a_info = np.asarray(abar_infos[i], dtype=np.float64)
            else:
                a_info, _ = m.programmed()
            if a_info.shape[1] < 3:
                raise ValueError("instance %d: protocol-3 abar_info needs 3 columns" % i)
            info = np.ascontiguousarray(a_info[:, :3], dtype=np.float64)
            x0 = _f64(m.dofs(1) if dofs is None or dofs[i] is None else dofs[i])
            self._keep += [info, x0]
            it = arr[i]
            it.mesh = m.desc
            it.params = m.params
            it.abar_info = _dp(info)
            it.timestep = s.timestep
            it.damping_factor_1 = s.damping_factor_1
            it.damping_factor_2 = s.damping_factor_2
            it.timesteps_per_dial_phase = s.timesteps_per_dial_phase
            it.timesteps_between_equil_checks = s.timesteps_between_equil_checks
            it.dial_factors_to_hold_at_spacing = s.dial_factors_to_hold_at_spacing
            it.dial_factor_to_start_from = s.dial_factor_to_start_from
            it.stop_at_final_equilibrium = int(stop_at_final_equilibrium)
            it.dofs = _dp(x0)
            it.velocities = None
        h = C.c_void_p()
        rc = L.ms_batch_create(arr, n, device, precision, C.byref(h))
        if rc != MS_OK:
            raise MsError(rc, "ms_batch_create: %s" % L.ms_status_string(rc).decode())
        self._h = h
        self.models = list(models)
        self.n = n

    def close(self):
        if getattr(self, "_h", None):
            lib().ms_batch_destroy(self._h)
            self._h = None

    __del__ = close

    def _chk(self, rc, what):
        if rc != MS_OK:
            raise MsError(rc, "%s: %s (%s)" % (what, lib().ms_status_string(rc).decode(),
                                                lib().ms_batch_last_error(self._h).decode()))

    def run(self, max_steps: int) -> int:
        done = C.c_int64()
        self._chk(lib().ms_batch_run(self._h, max_steps, C.byref(done)), "ms_batch_run")
        return done.value

    def status(self, i: int) -> ms_batch_inst_status:
        st = ms_batch_inst_status()
        self._chk(lib().ms_batch_status(self._h, i, C.byref(st)), "ms_batch_status")
        return st

    def download(self, i: int):
        N = self.models[i].num_nodes
        x, v = np.empty(3 * N), np.empty(3 * N)
        self._chk(lib().ms_batch_download_dofs(self._h, i, _dp(x), _dp(v)), "ms_batch_download_dofs")
        return x, v

    def upload(self, i: int, dofs, vel=None):
        self._chk(lib().ms_batch_upload_dofs(self._h, i, _dp(_f64(dofs)), _dp(None if vel is None else _f64(vel))),
                  "ms_batch_upload_dofs")

    def set_start(self, i: int, dial_factor: float, waiting: bool):
        self._chk(lib().ms_batch_set_start(self._h, i, dial_factor, int(waiting)), "ms_batch_set_start")

    def schedule(self) -> dict:
        s = ms_batch_schedule()
        self._chk(lib().ms_batch_get_schedule(self._h, C.byref(s)), "ms_batch_get_schedule")
        return {k: getattr(s, k) for k, _ in s._fields_}

    def set_schedule(self, tri_block: int, node_block: int, chunk_steps: int):
        """tri_block -1: node-tiled one-kernel step (node_block ignored); 0:
        bulk-copy tile kernel; 64/128/256: per-triangle kernel block size."""
        s = ms_batch_schedule(tri_block, node_block, chunk_steps, 0, 0)
        self._chk(lib().ms_batch_set_schedule(self._h, C.byref(s)), "ms_batch_set_schedule")

    def autotune(self, steps_per_trial: int = 20):
        s = ms_batch_schedule()
        ms = np.zeros(1)
        self._chk(lib().ms_batch_autotune(self._h, steps_per_trial, C.byref(s), _dp(ms)), "ms_batch_autotune")
        return {k: getattr(s, k) for k, _ in s._fields_}, float(ms[0])

    def autotune_report(self) -> list[str]:
        """The last autotune's trials (schedule or node-tiled plan: ms per step)."""
        n = lib().ms_batch_autotune_report(self._h, None, 0)
        buf = C.create_string_buffer(max(n, 0) + 1)
        lib().ms_batch_autotune_report(self._h, buf, len(buf))
        return [ln for ln in buf.value.decode().splitlines() if ln]

    def info(self):
        N, T, n = C.c_int64(), C.c_int64(), C.c_int32()
        lib().ms_batch_info(self._h, C.byref(N), C.byref(T), C.byref(n))
        return {"num_nodes": N.value, "num_tris": T.value, "instances": n.value}

    def stream(self) -> int:
        return lib().ms_batch_stream(self._h)


def _fp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    """The warm-start coordinate network (ms_mlp_*): SiLU MLP on the tensor
    cores, BF16 operands, FP32 accumulation and master weights, Adam."""

    def __init__(self, in_dim: int, width: int = 256, hidden_layers: int = 4, out_dim: int = 3, seed: int = 0,
                 device: int = -1):
        h = C.c_void_p()
        rc = lib().ms_mlp_create(in_dim, width, hidden_layers, out_dim, seed, device, C.byref(h))
        if rc != MS_OK:
            raise MsError(rc, "ms_mlp_create: %s" % lib().ms_status_string(rc).decode())
        self._h = h
        self.in_dim, self.width, self.hidden_layers, self.out_dim = in_dim, width, hidden_layers, out_dim
        self.in_pad = (in_dim + 15) // 16 * 16

    def close(self):
        if getattr(self, "_h", None):
            lib().ms_mlp_destroy(self._h)
            self._h = None

    __del__ = close

    def _chk(self, rc, what):
        if rc != MS_OK:
            raise MsError(rc, "%s: %s (%s)" % (what, lib().ms_status_string(rc).decode(),
                                                lib().ms_mlp_last_error(self._h).decode()))

    def num_params(self) -> int:
        n = C.c_int64()
        self._chk(lib().ms_mlp_num_params(self._h, C.byref(n)), "ms_mlp_num_params")
        return n.value

    def params(self) -> np.ndarray:
        p = np.empty(self.num_params(), dtype=np.float32)
        self._chk(lib().ms_mlp_get_params(self._h, _fp(p)), "ms_mlp_get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.num_params()
        self._chk(lib().ms_mlp_set_params(self._h, _fp(p)), "ms_mlp_set_params")

    def layers(self):
        """[(W [N][K], b [Np]) views into a params() vector's layout]: (offset, N, K, Np) per layer."""
        out, off = [], 0
        nl = self.hidden_layers + 1
        for l in range(nl):
            K = self.in_pad if l == 0 else self.width
            N = self.out_dim if l == nl - 1 else self.width
            Np = 16 if l == nl - 1 else self.width
            out.append((off, N, K, Np))
            off += N * K + Np
        return out

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty((x.shape[0], self.out_dim), dtype=np.float32)
        self._chk(lib().ms_mlp_forward(self._h, _fp(x), x.shape[0], _fp(y)), "ms_mlp_forward")
        return y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.empty(self.num_params(), dtype=np.float32)
        loss = np.zeros(1)
        self._chk(lib().ms_mlp_loss_grad(self._h, _fp(x), _fp(t), x.shape[0], _dp(loss), _fp(g)),
                  "ms_mlp_loss_grad")
        return float(loss[0]), g

    def set_data(self, x, t):
        self._x = np.ascontiguousarray(x, dtype=np.float32)
        self._t = np.ascontiguousarray(t, dtype=np.float32)
        self._chk(lib().ms_mlp_set_data(self._h, _fp(self._x), _fp(self._t), self._x.shape[0]), "ms_mlp_set_data")

    def train(self, epochs: int, batch: int = 8192, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        losses = np.zeros(epochs, dtype=np.float32)
        self._chk(lib().ms_mlp_train(self._h, epochs, batch, lr, seed, _fp(losses)), "ms_mlp_train")
        return losses

    def stream(self) -> int:
        return lib().ms_mlp_stream(self._h)


def run_batch(models, max_steps: int = 0, precision: int = MS_PRECISION_FP64, device: int = -1,
              stop_at_final_equilibrium: bool = True):
    """msh_run_batch: the host driver over a batch; returns per-model
    (msh_run_result, final dofs)."""
    n = len(models)
    hs = (C.c_void_p * n)(*[m._h for m in models])
    o = msh_run_options(max_steps, int(stop_at_final_equilibrium), 0, precision, device, 1, None)
    res = (msh_run_result * n)()
    outs = [np.empty(3 * m.num_nodes) for m in models]
    ptrs = (C.POINTER(C.c_double) * n)(*[_dp(x) for x in outs])
    rc = lib().msh_run_batch(hs, n, C.byref(o), res, ptrs)
    if rc != 0:
        raise RuntimeError(lib().msh_last_error().decode())
    return [(res[i], outs[i]) for i in range(n)]


def node_tile_layout(patch_ids, num_nodes: int, nodes_per_tile: int = 1024,
                     precision: int = MS_PRECISION_FP64) -> dict:
    """Layout of the node-tiled steps (step paths 3 and 4) for a mesh's patch
    table ([T][6] node ids), computed on the host with the checks ms_create
    runs: tiles, chunks, triangles computed per step, record sizes, the
    sliced staging size and the shared memory per block of each kernel."""
    p = np.ascontiguousarray(patch_ids, dtype=np.int32)
    info = ms_node_tile_info()
    rc = lib().ms_node_tile_layout(int(num_nodes), p.shape[0], p.ctypes.data, int(nodes_per_tile), int(precision),
                                   C.byref(info))
    if rc != 0:
        raise MsError(rc, "ms_node_tile_layout failed")
    return {k: getattr(info, k) for k, _ in ms_node_tile_info._fields_}


def device_info() -> str:
    buf = C.create_string_buffer(256)
    lib().ms_device_info(buf, 256)
    return buf.value.decode()
