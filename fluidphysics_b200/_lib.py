"""ctypes binding of libupbd.so (the C ABI declared in include/upbd.h).

The library is loaded from this package directory. There is no fallback:
if the CUDA library is missing, `load()` raises, and every caller fails
loudly instead of running some other implementation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

UPBD_OK = 0
ERRORS = {
    -1: "UPBD_ERR_INVALID", -2: "UPBD_ERR_OOM", -3: "UPBD_ERR_CUDA", -4: "UPBD_ERR_TIMEOUT",
    -5: "UPBD_ERR_NAN", -6: "UPBD_ERR_BUSY", -7: "UPBD_ERR_NO_DEVICE", -8: "UPBD_ERR_CAPACITY", -9: "UPBD_ERR_INTERNAL",
}
F_ACTIVE = 1
F_GRABBED = 2
FEAT_TETS = 1
FEAT_SOLID_CONTACTS = 2
HEALTH_NAN = 1
HEALTH_TIMEOUT = 2

PASS = dict(INTEGRATE=1, GRID=2, DENSITY=3, DISP=4, APPLY_FLUID=5, SOLID=7, BONDS=8, CONTACTS=9,
            APPLY_ALL=10, BOUNDS=11, VELOCITY=12, SOLID_VISC=13, XSPH=14, XSPH_APPLY=15)


class SceneDesc(C.Structure):
    _fields_ = [
        ("solid_dim", C.c_int32), ("solid_dim2", C.c_int32), ("max_fluid", C.c_int32),
        ("table_size", C.c_int32), ("substeps", C.c_int32), ("solid_iters", C.c_int32),
        ("features", C.c_uint32), ("device", C.c_int32),
        ("spacing", C.c_double), ("solid_mass", C.c_double), ("fluid_mass", C.c_double),
        ("cube_center", C.c_double * 3), ("cube2_center", C.c_double * 3),
        ("reserved", C.c_uint32 * 8),
    ]


PARAM_FIELDS = [
    "h", "gravity", "solid_radius", "fluid_radius", "cell_size", "fluid_h", "rest_density",
    "stiffness", "near_stiffness", "viscosity", "compliance", "omega", "plastic_threshold",
    "plastic_rate", "tear_gap", "max_speed", "wall_x", "wall_z", "wall_h", "wall_t", "cull_r",
    "damp_solid", "damp_fluid", "friction_solid", "friction_fluid", "grab_k", "sleep_speed",
    "solid_viscosity", "break_strain", "contact_scale",
]


class Params(C.Structure):
    _fields_ = [(f, C.c_double) for f in PARAM_FIELDS] + [
        ("tear_mode", C.c_int32), ("plastic_clamp", C.c_int32), ("reserved", C.c_uint32 * 6),
    ]


class Info(C.Structure):
    _fields_ = [
        ("solid_n", C.c_int32), ("n1", C.c_int32), ("dim1", C.c_int32), ("dim2", C.c_int32),
        ("max_fluid", C.c_int32), ("total", C.c_int32), ("num_cons", C.c_int32),
        ("num_tets", C.c_int32), ("table_size", C.c_int32), ("substeps", C.c_int32),
        ("solid_iters", C.c_int32), ("fluid_next", C.c_int32), ("features", C.c_uint32),
        ("frames", C.c_int32), ("device_bytes", C.c_uint64), ("param_bytes", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class DevicePtrs(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in ("pos", "prev", "vel", "density", "flags", "cons", "stream")]


class BatchDesc(C.Structure):
    """upbd_batch_desc (include/upbd_batch.h)."""
    _fields_ = [
        ("device", C.c_int32), ("solid_iters", C.c_int32), ("features", C.c_uint32),
        ("max_scenes", C.c_int32), ("block_threads", C.c_int32), ("ctas_per_sm", C.c_int32),
        ("hbm_budget", C.c_uint64), ("reserved", C.c_int32 * 8),
    ]


class BatchInfo(C.Structure):
    """upbd_batch_info (include/upbd_batch.h)."""
    _fields_ = [
        ("scenes", C.c_int32), ("max_scenes", C.c_int32), ("particles", C.c_int64), ("solids", C.c_int64),
        ("bytes_in_use", C.c_uint64), ("bytes_reserved", C.c_uint64), ("hbm_budget", C.c_uint64),
        ("frames", C.c_uint64), ("launches", C.c_uint64), ("block_threads", C.c_int32),
        ("ctas_per_sm", C.c_int32), ("num_sms", C.c_int32), ("reserved0", C.c_int32),
        ("reserved", C.c_int32 * 8),
    ]


class ServerDesc(C.Structure):
    """upbd_server_desc (include/upbd_server.h)."""
    _fields_ = [("batch", BatchDesc), ("dt", C.c_double), ("substeps", C.c_int32), ("builders", C.c_int32),
                ("keep_results", C.c_int32), ("reserved", C.c_int32 * 9)]


class Request(C.Structure):
    """upbd_request (include/upbd_server.h)."""
    _fields_ = [("desc", SceneDesc), ("params", Params), ("frames", C.c_int32), ("n_fluid", C.c_int32),
                ("fluid_mass", C.c_double), ("arrival_s", C.c_double),
                ("fluid_pos3", C.POINTER(C.c_float)), ("fluid_vel3", C.POINTER(C.c_float)),
                ("reserved", C.c_int32 * 8)]


class RequestResult(C.Structure):
    """upbd_request_result (include/upbd_server.h)."""
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("frames_done", C.c_int32), ("slots", C.c_int32),
                ("arrival_s", C.c_double), ("admit_s", C.c_double), ("done_s", C.c_double),
                ("frame_ms_max", C.c_double), ("reserved", C.c_int32 * 8)]


class ServerStats(C.Structure):
    """upbd_server_stats (include/upbd_server.h)."""
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64),
                ("rejected", C.c_int64), ("scene_frames", C.c_int64), ("batch_frames", C.c_int64),
                ("particle_substeps", C.c_double), ("wall_s", C.c_double), ("device_s", C.c_double),
                ("frame_ms_p50", C.c_double), ("frame_ms_p90", C.c_double), ("frame_ms_p99", C.c_double),
                ("frame_ms_max", C.c_double), ("frame_ms_mean", C.c_double), ("wait_ms_p50", C.c_double),
                ("wait_ms_p99", C.c_double), ("batch_ms_p50", C.c_double), ("batch_ms_p99", C.c_double),
                ("mean_scenes", C.c_double), ("peak_scenes", C.c_int32), ("reserved0", C.c_int32),
                ("peak_bytes", C.c_uint64), ("reserved", C.c_double * 8)]


# (name, restype, argtypes)
_P = C.c_void_p
_D3 = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_U = C.POINTER(C.c_uint32)
_SIGS = [
    ("upbd_default_desc", C.c_int, [C.POINTER(SceneDesc)]),
    ("upbd_default_params", C.c_int, [C.POINTER(Params)]),
    ("upbd_create", C.c_int, [C.POINTER(SceneDesc), C.POINTER(Params), C.POINTER(_P)]),
    ("upbd_destroy", C.c_int, [_P]),
    ("upbd_get_info", C.c_int, [_P, C.POINTER(Info)]),
    ("upbd_set_params", C.c_int, [_P, C.POINTER(Params)]),
    ("upbd_get_params", C.c_int, [_P, C.POINTER(Params)]),
    ("upbd_set_stream", C.c_int, [_P, _P]),
    ("upbd_get_device_ptrs", C.c_int, [_P, C.POINTER(DevicePtrs)]),
    ("upbd_last_error", C.c_char_p, [_P]),
    ("upbd_step", C.c_int, [_P, C.c_double, C.c_int32]),
    ("upbd_frame", C.c_int, [_P]),
    ("upbd_sync", C.c_int, [_P]),
    ("upbd_health", C.c_int, [_P, _U]),
    ("upbd_clear_health", C.c_int, [_P]),
    ("upbd_set_graphs", C.c_int, [_P, C.c_int32]),
    ("upbd_reset_solid", C.c_int, [_P]),
    ("upbd_drain", C.c_int, [_P]),
    ("upbd_active_count", C.c_int, [_P, _U]),
    ("upbd_emit", C.c_int, [_P, C.c_int32, _F, _F, _F, _F, C.c_float, C.c_float]),
    ("upbd_emit_particles", C.c_int, [_P, C.c_int32, _F, _F, C.c_double]),
    ("upbd_slice", C.c_int, [_P, _D3, _D3, _D3]),
    ("upbd_slice_now", C.c_int, [_P, _D3, _D3, _D3, _U]),
    ("upbd_pick", C.c_int, [_P, _D3, _D3, C.c_double, C.POINTER(C.c_int32), _D3]),
    ("upbd_grab_select", C.c_int, [_P, _F, C.c_float, C.c_uint32]),
    ("upbd_grab_indices", C.c_int, [_P, _U, C.c_int32, _F, _F]),
    ("upbd_grab_move", C.c_int, [_P, _F]),
    ("upbd_release", C.c_int, [_P]),
    ("upbd_read_state", C.c_int, [_P, _F, _F, _F, _F, _U]),
    ("upbd_read_state_async", C.c_int, [_P, _F, _U]),
    ("upbd_read_wait", C.c_int, [_P]),
    ("upbd_write_state", C.c_int, [_P, _F, _F, _F, _F, _U]),
    ("upbd_read_constraints", C.c_int, [_P, _U]),
    ("upbd_write_constraints", C.c_int, [_P, _U]),
    ("upbd_read_adjacency", C.c_int, [_P, _U]),
    ("upbd_read_grid", C.c_int, [_P, _U, _U, _U, _U]),
    ("upbd_rebuild_grid", C.c_int, [_P]),
    ("upbd_substep_partial", C.c_int, [_P, C.c_double, C.c_int32]),
    ("upbd_read_tets", C.c_int, [_P, _U]),
    ("upbd_write_tets", C.c_int, [_P, _U]),
    ("upbd_set_fluid_next", C.c_int, [_P, C.c_int32]),
    ("upbd_groups", C.c_int, [_P, C.POINTER(C.c_int32)]),
    ("upbd_groups_device", C.c_int, [_P, C.c_void_p]),
    ("upbd_grid_build", C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_double, _P, _P, _P, _P]),
    ("upbd_grid_build_noalloc", C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_double, _P, _P, _P, _P]),
    ("upbd_launch_count", C.c_uint64, [_P]),
    ("upbd_profile_frame", C.c_int, [_P, C.c_double, C.c_int32, C.POINTER(C.c_double), _U]),
    ("upbd_profile_graph_floor", C.c_int, [_P, C.c_double, C.c_int32, C.c_int32, C.POINTER(C.c_double), _U]),
    ("upbd_kernel_name", C.c_char_p, [C.c_int32]),
    # scene batch (include/upbd_batch.h)
    ("upbd_batch_default_desc", C.c_int, [C.POINTER(BatchDesc)]),
    ("upbd_batch_create", C.c_int, [C.POINTER(BatchDesc), C.POINTER(_P)]),
    ("upbd_batch_destroy", C.c_int, [_P]),
    ("upbd_batch_last_error", C.c_char_p, [_P]),
    ("upbd_batch_get_info", C.c_int, [_P, C.POINTER(BatchInfo)]),
    ("upbd_batch_scene_bytes", C.c_int, [C.POINTER(SceneDesc), C.POINTER(C.c_uint64)]),
    ("upbd_batch_add_scene", C.c_int, [_P, C.POINTER(SceneDesc), C.POINTER(Params), C.c_int32, _F, _F,
                                       C.c_double, C.POINTER(C.c_int32)]),
    ("upbd_batch_remove_scene", C.c_int, [_P, C.c_int32]),
    ("upbd_batch_set_params", C.c_int, [_P, C.c_int32, C.POINTER(Params)]),
    ("upbd_batch_step", C.c_int, [_P, C.c_double, C.c_int32]),
    ("upbd_batch_sync", C.c_int, [_P]),
    ("upbd_batch_set_stream", C.c_int, [_P, _P]),
    ("upbd_batch_set_tuning", C.c_int, [_P, C.c_int32, C.c_int32]),
    ("upbd_batch_read_state", C.c_int, [_P, C.c_int32, _F, _F, _F, _F, _U]),
    ("upbd_batch_write_state", C.c_int, [_P, C.c_int32, _F, _F, _F, _F, _U]),
    ("upbd_batch_read_constraints", C.c_int, [_P, C.c_int32, _U]),
    ("upbd_batch_write_constraints", C.c_int, [_P, C.c_int32, _U]),
    ("upbd_batch_scene_info", C.c_int, [_P, C.c_int32, C.POINTER(Info)]),
    ("upbd_batch_active_count", C.c_int, [_P, C.c_int32, _U]),
    ("upbd_batch_profile_frame", C.c_int, [_P, C.c_double, C.c_int32, C.POINTER(C.c_double), _U]),
    # frame server (include/upbd_server.h)
    ("upbd_server_default_desc", C.c_int, [C.POINTER(ServerDesc)]),
    ("upbd_server_create", C.c_int, [C.POINTER(ServerDesc), C.POINTER(_P)]),
    ("upbd_server_destroy", C.c_int, [_P]),
    ("upbd_server_last_error", C.c_char_p, [_P]),
    ("upbd_server_submit", C.c_int, [_P, C.POINTER(Request), C.POINTER(C.c_int64)]),
    ("upbd_server_run", C.c_int, [_P, C.c_double]),
    ("upbd_server_get_stats", C.c_int, [_P, C.POINTER(ServerStats)]),
    ("upbd_server_result", C.c_int, [_P, C.c_int64, C.POINTER(RequestResult), _F, _U]),
]
KERNEL_KINDS = 32

EXPORTED = [s[0] for s in _SIGS]

_libs: dict[str, C.CDLL] = {}


class UpbdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


LIB_NAMES = {"product": "libupbd.so", "parity": "libupbd_parity.so", "fp64": "libupbd_fp64.so",
             "checked": "libupbd_checked.so"}


def lib_path(variant: str = "product") -> Path:
    return HERE / LIB_NAMES[variant]


def load(variant: str = "product") -> C.CDLL:
    """Load libupbd.so ("product"), libupbd_parity.so ("parity") or one of
    the test-only builds: libupbd_fp64.so ("fp64": the same pass bodies on
    double, the single-scene entry points only) and libupbd_checked.so
    ("checked": the product with device-side index guards)."""
    if variant in _libs:
        return _libs[variant]
    path = lib_path(variant)
    if not path.exists():
        raise RuntimeError(
            f"{path.name} is not built; run `python -m fluidphysics_b200.build` "
            "(there is no non-CUDA fallback)")
    lib = C.CDLL(str(path))
    for name, res, args in _SIGS:
        if variant == "fp64" and name.startswith(("upbd_batch_", "upbd_server_")):
            continue  # the FP64 build holds the single-scene library only
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _libs[variant] = lib
    return lib


def check(lib: C.CDLL, handle, rc: int) -> None:
    if rc != UPBD_OK:
        msg = lib.upbd_last_error(handle)
        raise UpbdError(rc, msg.decode() if msg else "")


def check_batch(lib: C.CDLL, handle, rc: int) -> None:
    if rc != UPBD_OK:
        msg = lib.upbd_batch_last_error(handle)
        raise UpbdError(rc, msg.decode() if msg else "")


def fptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


def uptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_U)


def d3(v) -> C.Array:
    return (C.c_double * 3)(*[float(x) for x in v])


def f3(v) -> C.Array:
    return (C.c_float * 3)(*[float(x) for x in v])
