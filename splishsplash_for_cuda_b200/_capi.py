"""ctypes binding of the C ABI in include/dfsph_c.h (libdfsph_b200.so, built in-tree).

Loading fails loudly when the library is missing: there is no CPU fallback for the time step.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libdfsph_b200.so"
CHECKED_LIB_PATH = Path(__file__).resolve().parent / "libdfsph_b200_checked.so"  # range-checked variant

DFSPH_OK = 0
DFSPH_E_INVALID = -1
DFSPH_E_CUDA = -2
DFSPH_E_STATE = -3
DFSPH_E_NOMEM = -4
DFSPH_E_DEVICE = -5

ST_NEIGHBOR_OVERFLOW = 0x1
ST_NONFINITE = 0x2
ST_ESCAPED = 0x4
ST_PRESSURE_NOT_CONVERGED = 0x8
ST_DIVERGENCE_NOT_CONVERGED = 0x10
ST_SORT_TIMEOUT = 0x20
ST_BOUNDARY_OVERFLOW = 0x40
ST_FLUID_CAPACITY = 0x80
ST_MMA_TIMEOUT = 0x100
ST_INDEX = 0x200

SURFACE_PLANE, SURFACE_CUBOID, SURFACE_CYLINDER, SURFACE_MESH, SURFACE_SPHERE, SURFACE_STAR = 0, 1, 2, 3, 4, 5
MAX_SURFACE_MESHES = 8


class Surface(C.Structure):
    """dfsph_surface (include/dfsph_c.h)."""
    _fields_ = [
        ("type", C.c_int32),
        ("reversed", C.c_int32),
        ("origin", C.c_float * 3),
        ("normal", C.c_float * 3),
        ("center", C.c_float * 3),
        ("half_lengths", C.c_float * 3),
        ("radius", C.c_float),
        ("radius_internal", C.c_float),
        ("points", C.c_uint32),
        ("direction", C.c_float * 3),
    ]

FIELDS = {
    "position": (0, 3),
    "velocity": (1, 3),
    "mass": (2, 1),
    "density": (3, 1),
    "factor": (4, 1),
    "density_adv": (5, 1),
    "kappa": (6, 1),
    "kappa_v": (7, 1),
    "acceleration": (8, 1 * 3),
    "id": (9, 1),
    "boundary_psi": (10, 1),
    "boundary_position": (11, 3),
    "neighbor_counts": (12, 2),
    "boundary_velocity": (13, 3),
    "boundary_force": (14, 3),
    "features": (15, 5),
}
DTYPE_F32, DTYPE_F64, DTYPE_U32 = 0, 1, 2
ORDER_ID, ORDER_SORTED = 0, 1


class DfsphScene(C.Structure):
    _fields_ = [
        ("particle_radius", C.c_double),
        ("density0", C.c_double),
        ("viscosity", C.c_double),
        ("gravitation", C.c_double * 3),
        ("time_step", C.c_double),
        ("max_iterations", C.c_int32),
        ("max_error", C.c_double),
        ("max_iterations_v", C.c_int32),
        ("max_error_v", C.c_double),
        ("enable_divergence_solver", C.c_int32),
        ("cfl_method", C.c_int32),
        ("cfl_factor", C.c_double),
        ("cfl_max_time_step", C.c_double),
        ("cfl_min_time_step", C.c_double),
        ("fluid_capacity", C.c_uint32),
        ("boundary_capacity", C.c_uint32),
        ("neighbor_capacity", C.c_uint32),
        ("precision", C.c_int32),
        ("device", C.c_int32),
        ("use_graphs", C.c_int32),
        ("grid_min", C.c_double * 3),
        ("grid_max", C.c_double * 3),
    ]


class DfsphStepStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("iterations_v", C.c_int32),
        ("density_error", C.c_double),
        ("divergence_error", C.c_double),
        ("h", C.c_double),
        ("h_future", C.c_double),
        ("status", C.c_uint32),
        ("num_fluid", C.c_uint32),
        ("ms_total", C.c_double),
        ("warm_start", C.c_uint32),
        ("trained", C.c_uint32),
    ]


# Every symbol the header declares, with its ctypes signature.
_P = C.c_void_p
_F = C.POINTER(C.c_float)
_U = C.POINTER(C.c_uint32)
SIGNATURES = {
    "dfsph_scene_defaults": (C.c_int, [C.POINTER(DfsphScene)]),
    "dfsph_create": (C.c_int, [C.POINTER(DfsphScene), C.POINTER(_P)]),
    "dfsph_destroy": (C.c_int, [_P]),
    "dfsph_last_error": (C.c_char_p, [_P]),
    "dfsph_set_boundary": (C.c_int, [_P, _F, _F, C.c_uint32]),
    "dfsph_move_boundary": (C.c_int, [_P, _F, _F]),
    "dfsph_move_boundary_rigid": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P, _P, _P]),
    "dfsph_upload_fluid": (C.c_int, [_P, _F, _F, _F, C.c_uint32]),
    "dfsph_update_fluid": (C.c_int, [_P, _F, _F]),
    "dfsph_download": (C.c_int, [_P, C.c_int, C.c_int, _P, C.c_size_t, C.c_int]),
    "dfsph_get_neighbors": (C.c_int, [_P, _U, _U, C.c_uint32]),
    "dfsph_step": (C.c_int, [_P, C.POINTER(DfsphStepStats)]),
    "dfsph_neighbors_search": (C.c_int, [_P, C.c_int]),
    "dfsph_divergence_solve": (C.c_int, [_P, C.c_uint32, C.c_double, C.POINTER(C.c_int32)]),
    "dfsph_external_forces": (C.c_int, [_P]),
    "dfsph_update_time_step": (C.c_int, [_P, C.c_double]),
    "dfsph_cfl": (C.c_int, [_P, C.c_double, C.c_double, C.c_double]),
    "dfsph_update_vel": (C.c_int, [_P]),
    "dfsph_pressure_solve": (C.c_int, [_P, C.c_uint32, C.c_double, C.POINTER(C.c_int32)]),
    "dfsph_update_pos": (C.c_int, [_P]),
    "dfsph_on_step_end": (C.c_int, [_P]),
    "dfsph_set_param": (C.c_int, [_P, C.c_char_p, C.c_double]),
    "dfsph_get_param": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_double)]),
    "dfsph_status": (C.c_int, [_P, _U, C.c_int]),
    "dfsph_num_fluid": (C.c_int, [_P, _U]),
    "dfsph_synchronize": (C.c_int, [_P]),
    "dfsph_launch_count": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "dfsph_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "dfsph_time_kernel": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "dfsph_save_snapshot": (C.c_int, [_P, C.c_char_p, C.c_int]),
    "dfsph_load_snapshot": (C.c_int, [_P, C.c_char_p, C.c_int, C.c_int]),
    "dfsph_checkpoint_save": (C.c_int, [_P, C.c_char_p]),
    "dfsph_export_bgeo": (C.c_int, [_P, C.c_char_p]),
    "dfsph_read_dynamic_data": (C.c_int, [_P, _P, _P]),
    "dfsph_body_wrench": (C.c_int, [_P, C.c_uint32, _P, _P, _P, _P]),
    "dfsph_check_particles_positions": (C.c_int, [_P, C.c_int, C.POINTER(C.c_uint32)]),
    "dfsph_open_boundary_init": (C.c_int, [_P, C.POINTER(Surface), C.POINTER(Surface), C.POINTER(Surface), _P,
                                           C.c_uint32, C.POINTER(C.c_uint32)]),
    "dfsph_open_boundary_apply": (C.c_int, [_P, C.c_double, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_uint32),
                                            C.POINTER(C.c_uint32)]),
    "dfsph_open_boundary_shift": (C.c_int, [_P, _P]),
    "dfsph_set_surface_mesh": (C.c_int, [_P, C.c_uint32, _P, C.c_uint32, _P, C.c_uint32]),
    "dfsph_dynamic_window_stabilize": (C.c_int, [_P, C.c_uint32, C.c_double, C.c_double, C.c_int]),
    "dfsph_fluid_level": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "dfsph_fluid_level_control": (C.c_int, [_P, C.c_double, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "dfsph_read_obj": (C.c_int, [C.c_char_p, _P, C.c_uint32, C.POINTER(C.c_uint32), _P, C.c_uint32,
                                 C.POINTER(C.c_uint32)]),
    "dfsph_dynamic_window_init": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_uint32, _P, C.c_uint32]),
    "dfsph_dynamic_window_shift": (C.c_int, [_P, _P, C.c_double, C.c_double, C.POINTER(C.c_uint32),
                                             C.POINTER(C.c_uint32)]),
    "dfsph_dynamic_window_displacement": (C.c_int, [_P, _P]),
    "dfsph_open_boundary_samples": (C.c_int, [_P, _P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "dfsph_bgeo_write": (C.c_int, [C.c_char_p, _P, _P, C.c_uint64, C.c_float]),
    "dfsph_bgeo_read": (C.c_int, [C.c_char_p, _P, _P, C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_int)]),
    "dfsph_checkpoint_load": (C.c_int, [_P, C.c_char_p]),
    "dfsph_mlp_get_params": (C.c_int, [_P, _F, C.c_size_t]),
    "dfsph_mlp_set_params": (C.c_int, [_P, _F, C.c_size_t]),
    "dfsph_mlp_get_scales": (C.c_int, [_P, _F, _F]),
    "dfsph_mlp_set_scales": (C.c_int, [_P, _F, _F]),
    "dfsph_mlp_forward": (C.c_int, [_P, _F, C.c_uint32, _F]),
    "dfsph_mlp_gradient": (C.c_int, [_P, _F, _F, C.c_uint32, _F, C.POINTER(C.c_double)]),
    "dfsph_mlp_train": (C.c_int, [_P, _F, _F, C.c_uint32, C.c_int32, C.c_double, C.POINTER(C.c_double)]),
    "dfsph_mlp_reset": (C.c_int, [_P, C.c_uint32]),
    "dfsph_sort_cell_keys_noalloc": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_int, _P]),
    "dfsph_scene_load": (C.c_int, [C.c_char_p, C.POINTER(DfsphScene), C.POINTER(C.c_void_p)]),
    "dfsph_scene_file_counts": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_int)]),
    "dfsph_scene_file_fluid": (C.c_int, [_P, _P, _P]),
    "dfsph_scene_file_boundary": (C.c_int, [_P, _P]),
    "dfsph_scene_file_free": (None, [_P]),
    "dfsph_create_from_scene_file": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
}

MLP_INPUTS, MLP_OUTPUTS, MLP_PARAMS = 8, 2, 4866
SNAP_FLUID, SNAP_BOUNDARY = 1, 2

NOALLOC_MAX_KEYS = 1 << 18

KERNELS = ["neighbor_build", "density_alpha", "divergence_jacobi", "divergence_residual", "viscosity",
           "pressure_warm_jacobi", "pressure_residual", "pressure_jacobi", "update_pos", "sort_reorder"]

_lib = None


class DfsphError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"DFSPH error {code}: {message}")
        self.code = code


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Loads libdfsph_b200.so and binds every entry point. Raises if the library is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build it with `python -m splishsplash_for_cuda_b200.build` "
            "(the DFSPH time step has no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(lib: C.CDLL, ctx, code: int) -> None:
    if code != DFSPH_OK:
        msg = lib.dfsph_last_error(ctx)
        raise DfsphError(code, msg.decode() if msg else "")
