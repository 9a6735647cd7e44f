"""ctypes binding of include/mts.h (libmts_b200.so, built in-tree).

The library is loaded from ``matched-time-splitting-3d_b200/lib``; when it is
missing or older than its sources it is rebuilt with nvcc.  There is no CPU
fallback: every compute call needs the CUDA library and a device.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MTS_OK = 0
STATUS_NAMES = {
    1: "MTS_ERR_ARG",
    2: "MTS_ERR_SETUP",
    3: "MTS_ERR_ZERO_PIVOT",
    4: "MTS_ERR_NONFINITE",
    5: "MTS_ERR_CUDA",
    6: "MTS_ERR_NO_DEVICE",
    7: "MTS_ERR_OOM",
}
METHODS = {"adi": 0, "lod-ie": 1, "lod-cn": 2, "ts": 3}
SURFACES = {"ellipsoid": 0, "torus": 1}

# Every entry point include/mts.h declares.
EXPORTS = [
    "mts_create",
    "mts_create_from_crossings",
    "mts_setup_host",
    "mts_setup_device",
    "mts_destroy",
    "mts_initialize",
    "mts_set_solution",
    "mts_get_solution",
    "mts_solve_2nd",
    "mts_advance",
    "mts_advance_host",
    "mts_batch_advance",
    "mts_batch_advance_steps",
    "mts_norms",
    "mts_norms_noalloc",
    "mts_fp_errors",
    "mts_jump_errors",
    "mts_get_time",
    "mts_set_time",
    "mts_synchronize",
    "mts_get_counts",
    "mts_export_tags",
    "mts_export_crossings",
    "mts_get_launch_count",
    "mts_get_device_bytes",
    "mts_get_stream",
    "mts_set_profiling",
    "mts_profile_read",
    "mts_sweep_shape_count",
    "mts_set_sweep_shape",
    "mts_autotune",
    "mts_set_precision",
    "mts_get_precision",
    "mts_last_error",
    "mts_version",
]


class MtsError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {message}")


class mts_grid(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("pad", ctypes.c_int32),
        ("xl", ctypes.c_double),
        ("xr", ctypes.c_double),
        ("yl", ctypes.c_double),
        ("yr", ctypes.c_double),
        ("zl", ctypes.c_double),
        ("zr", ctypes.c_double),
    ]


class mts_surface(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("pad", ctypes.c_int32), ("params", ctypes.c_double * 7)]


class mts_params(ctypes.Structure):
    _fields_ = [
        ("beta_in", ctypes.c_double),
        ("beta_out", ctypes.c_double),
        ("eq", ctypes.c_int32),
        ("method", ctypes.c_int32),
        ("mib", ctypes.c_int32),
        ("setup", ctypes.c_int32),
        ("dt", ctypes.c_double),
        ("t0", ctypes.c_double),
    ]


# Same layout as mts_crossing (296 bytes).
CROSSING_DTYPE = np.dtype(
    [
        ("dir", "<i4"),
        ("indx1", "<i4"),
        ("indx2", "<i4"),
        ("id", "<i4"),
        ("left_loc", "<i4"),
        ("nwei", "<i4"),
        ("coord", "<f8", 3),
        ("gamma", "<f8"),
        ("normal", "<f8", 3),
        ("p", "<f8", 9),
        ("weil", "<f8", 9),
        ("weir", "<f8", 9),
    ]
)
assert CROSSING_DTYPE.itemsize == 296

_lib = None
_lock = threading.Lock()


def lib_path() -> str:
    return os.path.join(PKG_DIR, "lib", "libmts_b200.so")


def load(build_if_missing: bool = True):
    """Loads libmts_b200.so, building it first when needed."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        import importlib.util

        spec = importlib.util.spec_from_file_location("_mts_build", os.path.join(PKG_DIR, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        if build_if_missing and not mod.up_to_date():
            mod.build()
        path = lib_path()
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing; run matched-time-splitting-3d_b200/build.py")
        L = ctypes.CDLL(path)
        P = ctypes.POINTER
        H = ctypes.c_void_p
        vp = ctypes.c_void_p
        sig = {
            "mts_create": [P(mts_grid), P(mts_surface), P(mts_params), P(H)],
            "mts_create_from_crossings": [P(mts_grid), vp, vp, ctypes.c_int32, P(mts_params), P(H)],
            "mts_setup_host": [P(mts_grid), P(mts_surface), P(mts_params), vp, vp, ctypes.c_int32,
                               P(ctypes.c_int32), vp],
            "mts_setup_device": [P(mts_grid), P(mts_surface), P(mts_params), vp, vp, ctypes.c_int32,
                                 P(ctypes.c_int32), vp],
            "mts_destroy": [H],
            "mts_initialize": [H],
            "mts_set_solution": [H, vp],
            "mts_get_solution": [H, vp],
            "mts_solve_2nd": [H, ctypes.c_double, ctypes.c_double, ctypes.c_double],
            "mts_advance": [H, ctypes.c_int32],
            "mts_advance_host": [H, vp, vp, ctypes.c_int32],
            "mts_batch_advance": [vp, ctypes.c_int32, ctypes.c_int32],
            "mts_batch_advance_steps": [vp, vp, ctypes.c_int32],
            "mts_norms": [H, P(ctypes.c_double), P(ctypes.c_double), vp],
            "mts_norms_noalloc": [H, vp, ctypes.c_double, P(ctypes.c_double), P(ctypes.c_double), vp],
            "mts_fp_errors": [H, P(ctypes.c_double), P(ctypes.c_double)],
            "mts_jump_errors": [H, P(ctypes.c_double), P(ctypes.c_double)],
            "mts_get_time": [H, P(ctypes.c_double)],
            "mts_set_time": [H, ctypes.c_double],
            "mts_synchronize": [H],
            "mts_get_counts": [H, vp],
            "mts_export_tags": [H, vp],
            "mts_export_crossings": [H, vp, ctypes.c_int32, P(ctypes.c_int32)],
            "mts_get_launch_count": [H, P(ctypes.c_int64)],
            "mts_get_device_bytes": [H, P(ctypes.c_int64)],
            "mts_get_stream": [H, P(ctypes.c_void_p)],
            "mts_set_profiling": [H, ctypes.c_int32],
            "mts_profile_read": [H, vp, vp],
            "mts_set_sweep_shape": [H, ctypes.c_int32, ctypes.c_int32],
            "mts_autotune": [H, ctypes.c_int32, vp],
            "mts_set_precision": [H, ctypes.c_int32],
            "mts_get_precision": [H, P(ctypes.c_int32)],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.mts_last_error.argtypes = []
        L.mts_last_error.restype = ctypes.c_char_p
        L.mts_version.argtypes = []
        L.mts_version.restype = ctypes.c_int32
        L.mts_sweep_shape_count.argtypes = []
        L.mts_sweep_shape_count.restype = ctypes.c_int32
        _lib = L
        return L


def check(status: int, where: str) -> None:
    if status != MTS_OK:
        msg = load().mts_last_error().decode(errors="replace")
        raise MtsError(status, where, msg)


def make_grid(n, domain) -> mts_grid:
    return mts_grid(int(n[0]), int(n[1]), int(n[2]), 0, *map(float, domain))


def make_surface(kind: str, params) -> mts_surface:
    s = mts_surface()
    s.kind = SURFACES[kind]
    p = list(map(float, params))
    if kind == "ellipsoid" and len(p) == 4:
        p += [0.0, 0.0, 0.0]
    for i, v in enumerate(p[:7]):
        s.params[i] = v
    return s


SETUPS = {"host": 0, "device": 1}


def make_params(beta_in, beta_out, eq, method, mib, dt, t0=0.0, setup="host") -> mts_params:
    m = METHODS[method] if isinstance(method, str) else int(method)
    return mts_params(float(beta_in), float(beta_out), int(eq), m, int(mib), SETUPS[setup], float(dt), float(t0))
