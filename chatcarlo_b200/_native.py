"""ctypes binding of include/chatcarlo_b200.h.

The library is loaded from chatcarlo_b200/lib/libccb200.so.  There is no
fallback: a missing or unloadable library raises NativeLibraryError.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import os

LIB_PATH = Path(os.environ.get("CHATCARLO_B200_LIB") or
                Path(__file__).resolve().parent / "lib" / "libccb200.so")
# the same engine built with FP64 tracking (the precision reference)
FP64_LIB_PATH = Path(os.environ.get("CHATCARLO_B200_FP64_LIB") or
                     Path(__file__).resolve().parent / "lib" / "libccb200_fp64.so")

CC_OK = 0
CC_E_INVALID = -1
CC_E_ENERGY_RANGE = -2
CC_E_RAYLEIGH_Q_RANGE = -3
CC_E_UNKNOWN_MATERIAL = -4
CC_E_BAD_SHAPE = -5
CC_E_DEVICE = -6
CC_E_TIMEOUT = -7
CC_E_BOUNDS = -8
CC_E_NOMEM = -9

CC_SHAPE_BOX, CC_SHAPE_SPHERE, CC_SHAPE_CYLINDER, CC_SHAPE_ELLIPSOID = 0, 1, 2, 3
CC_GRID_STATS = 1
CC_FIELD_RECT, CC_FIELD_CONE, CC_FIELD_PARALLEL = 0, 1, 2
CC_INTERACT_PHOTO, CC_INTERACT_COMPTON, CC_INTERACT_RAYLEIGH = 0, 1, 2

# every symbol the header declares
EXPORTED = [
    "cc_version", "cc_last_error", "cc_ctx_create", "cc_ctx_destroy", "cc_ctx_set_launch",
    "cc_ctx_set_step_limit", "cc_ctx_set_tally_fp32", "cc_ctx_set_tally_queue", "cc_tables_create", "cc_tables_destroy", "cc_scene_create",
    "cc_scene_destroy", "cc_source_create", "cc_source_destroy", "cc_grid_create",
    "cc_grid_destroy", "cc_grid_reset", "cc_grid_download", "cc_grid_end_batch", "cc_grid_maps", "cc_grid_upload",
    "cc_transport_photons", "cc_transport_photons_device", "cc_run", "cc_sample_source",
    "cc_transport_photons_device_noalloc", "cc_batch_create", "cc_batch_run", "cc_batch_destroy",
    "cc_sample_interactions", "cc_philox4x32_10", "cc_grid_device_buffers", "cc_grid_set_counts",
    "cc_measure_fp64_reductions",
]


class NativeLibraryError(RuntimeError):
    pass


class CCError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Primitive(C.Structure):
    _fields_ = [("type", C.c_int32), ("material", C.c_int32), ("axis", C.c_int32), ("pad", C.c_int32),
                ("center", C.c_double * 3), ("size", C.c_double * 3), ("radius", C.c_double),
                ("height", C.c_double)]


class MaterialDesc(C.Structure):
    _fields_ = [("density", C.c_double), ("n_nodes", C.c_int32), ("n_elements", C.c_int32),
                ("log_e", C.POINTER(C.c_double)), ("log_parts", C.POINTER(C.c_double)),
                ("log_elem", C.POINTER(C.c_double)), ("element_slot", C.POINTER(C.c_int32)),
                ("log_tally", C.POINTER(C.c_double))]


class ElementDesc(C.Structure):
    _fields_ = [("z", C.c_int32), ("n_lines", C.c_int32),
                ("s_over_z", C.POINTER(C.c_double)), ("ray_x", C.POINTER(C.c_double)),
                ("ray_a", C.POINTER(C.c_double)), ("k_edge_kev", C.c_double),
                ("k_shell_prob", C.c_double), ("omega_k", C.c_double),
                ("line_e", C.c_double * 8), ("line_p", C.c_double * 8),
                ("emits", C.c_int32), ("pad", C.c_int32)]


class TableDesc(C.Structure):
    _fields_ = [("n_materials", C.c_int32), ("n_elements", C.c_int32),
                ("materials", C.POINTER(MaterialDesc)), ("elements", C.POINTER(ElementDesc))]


class HeelDesc(C.Structure):
    _fields_ = [("h_u", C.c_double), ("h_v", C.c_double), ("span_cm", C.c_double), ("n_bins", C.c_int32),
                ("pad", C.c_int32), ("centers", C.POINTER(C.c_double)), ("rel_fluence", C.POINTER(C.c_double)),
                ("bin_sizes", C.POINTER(C.c_int32)), ("energies_kev", C.POINTER(C.c_double)),
                ("weights", C.POINTER(C.c_double))]


class SourceDesc(C.Structure):
    _fields_ = [("field", C.c_int32), ("rotation", C.c_int32), ("rot_axis", C.c_int32),
                ("n_angles", C.c_int32), ("position", C.c_double * 3), ("direction", C.c_double * 3),
                ("u", C.c_double * 3), ("v", C.c_double * 3), ("sid_cm", C.c_double),
                ("size_u", C.c_double), ("size_v", C.c_double), ("cos_half_angle", C.c_double),
                ("isocenter", C.c_double * 3), ("scan_length_cm", C.c_double),
                ("n_energies", C.c_int32), ("pad", C.c_int32),
                ("energies_kev", C.POINTER(C.c_double)), ("weights", C.POINTER(C.c_double)),
                ("heel", C.POINTER(HeelDesc))]


class RunOut(C.Structure):
    _fields_ = [("n_histories", C.c_int64), ("n_absorbed", C.c_int64), ("n_escaped", C.c_int64),
                ("scatter_sum", C.c_int64), ("n_fluorescence", C.c_int64), ("n_batches", C.c_int64),
                ("gpu_launches", C.c_int64), ("elapsed_ms", C.c_double), ("n_steps", C.c_int64),
                ("n_voxel_visits", C.c_int64), ("transport_ms", C.c_double),
                ("transport_launches", C.c_int64)]


P = C.c_void_p
PD = C.POINTER(C.c_double)
_libs: dict = {}


def _bind(lib):
    sig = {
        "cc_version": (C.c_int, []),
        "cc_last_error": (C.c_char_p, []),
        "cc_ctx_create": (C.c_int, [C.c_int, C.POINTER(P)]),
        "cc_ctx_destroy": (C.c_int, [P]),
        "cc_ctx_set_launch": (C.c_int, [P, C.c_int, C.c_int]),
        "cc_ctx_set_step_limit": (C.c_int, [P, C.c_int64]),
        "cc_ctx_set_tally_fp32": (C.c_int, [P, C.c_int32]),
        "cc_ctx_set_tally_queue": (C.c_int, [P, C.c_int32, C.c_int64]),
        "cc_tables_create": (C.c_int, [P, C.POINTER(TableDesc), C.POINTER(P)]),
        "cc_tables_destroy": (C.c_int, [P]),
        "cc_scene_create": (C.c_int, [P, C.POINTER(Primitive), C.c_int32, C.c_int32, PD, PD, C.POINTER(P)]),
        "cc_scene_destroy": (C.c_int, [P]),
        "cc_source_create": (C.c_int, [P, C.POINTER(SourceDesc), C.POINTER(P)]),
        "cc_source_destroy": (C.c_int, [P]),
        "cc_grid_create": (C.c_int, [P, PD, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_int32, C.POINTER(P)]),
        "cc_grid_destroy": (C.c_int, [P]),
        "cc_grid_reset": (C.c_int, [P]),
        "cc_grid_download": (C.c_int, [P, PD, PD, PD, PD, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "cc_grid_end_batch": (C.c_int, [P, C.c_int64]),
        "cc_grid_upload": (C.c_int, [P, PD, PD, PD, PD, C.POINTER(C.c_int32), C.c_int64, C.c_int64]),
        "cc_grid_maps": (C.c_int, [P, C.POINTER(Primitive), C.c_int32, PD, C.c_double, C.c_double, C.c_double, C.c_int32, P, P, P, P]),
        "cc_transport_photons": (C.c_int, [P, P, P, P, C.c_int64, PD, PD, PD, C.c_uint64, C.c_uint64, C.c_int32,
                                           C.POINTER(C.c_int64), C.POINTER(C.c_uint8), C.POINTER(C.c_uint8), PD,
                                           C.POINTER(C.c_int64)]),
        "cc_transport_photons_device": (C.c_int, [P, P, P, P, C.c_int64, P, P, P, C.c_uint64, C.c_uint64, C.c_int32,
                                                  P, P, P, PD, C.POINTER(C.c_int64)]),
        "cc_run": (C.c_int, [P, P, P, P, P, C.c_int64, C.c_int64, C.c_uint64, C.c_int64, C.c_int32, PD, PD,
                             C.POINTER(RunOut)]),
        "cc_sample_source": (C.c_int, [P, P, C.c_int64, C.c_uint64, C.c_int64, PD, PD, PD]),
        "cc_batch_create": (C.c_int, [P, P, C.c_int32, C.POINTER(P), C.POINTER(P), C.POINTER(P),
                                      C.POINTER(C.c_int64), C.c_int32, C.c_int32, C.POINTER(P)]),
        "cc_batch_run": (C.c_int, [P, C.c_uint64, C.c_int32, C.POINTER(C.c_int64), C.POINTER(RunOut)]),
        "cc_batch_destroy": (C.c_int, [P]),
        "cc_transport_photons_device_noalloc": (C.c_int, [P, P, C.c_int64, P, P, P, C.c_uint64, C.c_uint64,
                                                          C.c_int32, P, P, P, PD, C.POINTER(C.c_int64), P]),
        "cc_sample_interactions": (C.c_int, [P, P, C.c_int32, C.c_int64, C.POINTER(C.c_int32), PD, C.c_uint64,
                                             C.c_int32, PD, PD, C.POINTER(C.c_int32)]),
        "cc_philox4x32_10": (C.c_int, [P, C.c_int64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                       C.POINTER(C.c_uint32)]),
        "cc_grid_device_buffers": (C.c_int, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(C.c_int64),
                                             C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "cc_grid_set_counts": (C.c_int, [P, C.c_int64, C.c_int64]),
        "cc_measure_fp64_reductions": (C.c_int, [C.c_int, P, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                                 C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.c_int32, PD]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


def lib(path: Path | None = None):
    """The loaded engine library (each path loaded once); the FP32-tracking
    build unless another path is given."""
    path = Path(path) if path is not None else LIB_PATH
    handle = _libs.get(path)
    if handle is None:
        if not path.exists():
            raise NativeLibraryError(
                f"{path} is missing; build it with `python -m chatcarlo_b200.build`")
        try:
            handle = C.CDLL(str(path))
        except OSError as e:
            raise NativeLibraryError(f"cannot load {path}: {e}") from e
        _bind(handle)
        _libs[path] = handle
    return handle


_PY_ERRORS = {CC_E_ENERGY_RANGE: ValueError, CC_E_RAYLEIGH_Q_RANGE: ValueError,
              CC_E_UNKNOWN_MATERIAL: ValueError, CC_E_BAD_SHAPE: ValueError, CC_E_INVALID: ValueError}


def check(rc: int, handle=None) -> None:
    if rc != CC_OK:
        msg = (handle or lib()).cc_last_error().decode(errors="replace")
        exc = _PY_ERRORS.get(rc)
        if exc is not None:
            raise exc(f"[{rc}] {msg}")
        raise CCError(rc, msg)


def dptr(a):
    """ctypes double* of a C-contiguous float64 numpy array."""
    return a.ctypes.data_as(PD)
