"""Matched-TS time stepping on B200: Python front end of libmts_b200.so.

``Solver`` owns one problem resident on the current CUDA device (one
``mts_handle``).  ``setup_host`` runs only the host setup (mesh tags, crossing
list, MIB weights) and needs no device.  ``mts_b200.reference_api`` mirrors
the reference's class interfaces (Mesh, Intersections, Douglas_ADI, LOD, TS).

Fields are float64 numpy arrays of nx*ny*nz values, x fastest (the order of
the reference's Mesh::To1d, src/mesh/mesh.cc:93-99).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from ._lib import (CROSSING_DTYPE, EXPORTS, METHODS, MtsError, check, lib_path, load, make_grid, make_params,
                   make_surface)

__all__ = [
    "Spec",
    "Solver",
    "setup_host",
    "setup_device",
    "batch_advance",
    "batch_advance_steps",
    "MtsError",
    "CROSSING_DTYPE",
    "METHODS",
    "EXPORTS",
    "load",
    "lib_path",
]


@dataclass
class Spec:
    """One parabolic interface problem."""

    n: tuple = (33, 33, 33)
    domain: tuple = (-1.0, 1.0, -1.0, 1.0, -1.0, 1.0)
    surface: str = "ellipsoid"  # ellipsoid (a b c r [cx cy cz]) or torus (R r)
    surface_params: tuple = (1.0, 1.0, 1.0, 0.49, 0.0, 0.0, 0.0)
    beta_in: float = 1.0
    beta_out: float = 10.0
    eq: int = 8
    method: str = "adi"
    mib: int = 1
    dt: float = 1.0 / 32
    t0: float = 0.0
    setup: str = "host"  # where mts_create builds tags, crossings and MIB weights: host or device

    @property
    def nodes(self) -> int:
        return int(self.n[0]) * int(self.n[1]) * int(self.n[2])

    def c_structs(self):
        return (make_grid(self.n, self.domain), make_surface(self.surface, self.surface_params),
                make_params(self.beta_in, self.beta_out, self.eq, self.method, self.mib, self.dt, self.t0,
                            self.setup))


def _setup(spec: Spec, name: str):
    L = load()
    fn = getattr(L, name)
    g, s, p = spec.c_structs()
    count = ctypes.c_int32(0)
    check(fn(ctypes.byref(g), ctypes.byref(s), ctypes.byref(p), None, None, 0, ctypes.byref(count), None), name)
    tags = np.empty(spec.nodes, dtype=np.int8)
    cr = np.zeros(count.value, dtype=CROSSING_DTYPE)
    counts = np.zeros(2, dtype=np.int64)
    check(fn(ctypes.byref(g), ctypes.byref(s), ctypes.byref(p), tags.ctypes.data, cr.ctypes.data if cr.size else None,
             cr.size, ctypes.byref(count), counts.ctypes.data), name)
    return tags, cr, {"corner_pairs": int(counts[0]), "singular_warnings": int(counts[1])}


def setup_host(spec: Spec):
    """Host setup only: returns (tags int8[N], crossings CROSSING_DTYPE[n],
    {"corner_pairs", "singular_warnings"})."""
    return _setup(spec, "mts_setup_host")


def setup_device(spec: Spec):
    """The same setup on the CUDA device (mts_setup_device), same results:
    tags identical, crossing records identical except in the last bits where
    the reference's pow(v, 2) is not the correctly rounded square."""
    return _setup(spec, "mts_setup_device")


def batch_advance(solvers, nsteps: int) -> None:
    """nsteps steps of every solver in one batch (mts_batch_advance): each
    kernel of a step is one launch for all plain-form problems of a method,
    a CTA working on one problem's part.  Results equal those of advancing
    each solver on its own."""
    solvers = list(solvers)
    if not solvers:
        return
    L = load()
    arr = (ctypes.c_void_p * len(solvers))(*[s.handle.value for s in solvers])
    check(L.mts_batch_advance(arr, len(solvers), int(nsteps)), "mts_batch_advance")


def batch_advance_steps(solvers, counts) -> None:
    """counts[i] steps of solvers[i], all in one batch
    (mts_batch_advance_steps)."""
    solvers = list(solvers)
    if not solvers:
        return
    L = load()
    arr = (ctypes.c_void_p * len(solvers))(*[s.handle.value for s in solvers])
    cnt = (ctypes.c_int32 * len(solvers))(*[int(c) for c in counts])
    check(L.mts_batch_advance_steps(arr, cnt, len(solvers)), "mts_batch_advance_steps")


class Solver:
    """A problem resident on the GPU.

    Solver(spec) runs the setup on the host and uploads it;
    Solver(spec, tags=..., crossings=...) uses a caller-supplied mesh and
    crossing list instead (the drop-in path for the reference's own
    Mesh/Intersections objects)."""

    def __init__(self, spec: Spec, tags: np.ndarray | None = None, crossings: np.ndarray | None = None):
        self.spec = spec
        self._L = load()
        self._h = ctypes.c_void_p()
        g, s, p = spec.c_structs()
        if tags is None:
            check(self._L.mts_create(ctypes.byref(g), ctypes.byref(s), ctypes.byref(p), ctypes.byref(self._h)),
                  "mts_create")
        else:
            t = np.ascontiguousarray(tags, dtype=np.int8)
            cr = np.ascontiguousarray(crossings if crossings is not None else np.zeros(0, CROSSING_DTYPE),
                                      dtype=CROSSING_DTYPE)
            check(self._L.mts_create_from_crossings(ctypes.byref(g), t.ctypes.data, cr.ctypes.data if cr.size else None,
                                                    cr.size, ctypes.byref(p), ctypes.byref(self._h)),
                  "mts_create_from_crossings")

    # -- lifecycle -----------------------------------------------------------
    def close(self) -> None:
        if self._h and self._h.value:
            check(self._L.mts_destroy(self._h), "mts_destroy")
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state ---------------------------------------------------------------
    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @property
    def time(self) -> float:
        t = ctypes.c_double()
        check(self._L.mts_get_time(self._h, ctypes.byref(t)), "mts_get_time")
        return t.value

    @time.setter
    def time(self, t: float) -> None:
        check(self._L.mts_set_time(self._h, float(t)), "mts_set_time")

    def initialize(self) -> None:
        check(self._L.mts_initialize(self._h), "mts_initialize")

    def set_solution(self, u: np.ndarray) -> None:
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.size != self.spec.nodes:
            raise ValueError("field size mismatch")
        check(self._L.mts_set_solution(self._h, u.ctypes.data), "mts_set_solution")

    def solution(self) -> np.ndarray:
        u = np.empty(self.spec.nodes, dtype=np.float64)
        check(self._L.mts_get_solution(self._h, u.ctypes.data), "mts_get_solution")
        return u

    # -- stepping ------------------------------------------------------------
    def advance(self, nsteps: int = 1) -> None:
        check(self._L.mts_advance(self._h, int(nsteps)), "mts_advance")

    def solve_2nd(self, t_prev: float, t_half: float, t_next: float) -> None:
        check(self._L.mts_solve_2nd(self._h, float(t_prev), float(t_half), float(t_next)), "mts_solve_2nd")

    def advance_host(self, u_in: np.ndarray, u_out: np.ndarray, nsteps: int = 1) -> None:
        """u_in/u_out: C-contiguous float64 host arrays (pinned for full speed)."""
        check(self._L.mts_advance_host(self._h, u_in.ctypes.data, u_out.ctypes.data, int(nsteps)), "mts_advance_host")

    def advance_host_ptr(self, in_ptr: int, out_ptr: int, nsteps: int = 1) -> None:
        check(self._L.mts_advance_host(self._h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr), int(nsteps)),
              "mts_advance_host")

    def synchronize(self) -> None:
        check(self._L.mts_synchronize(self._h), "mts_synchronize")

    def norms(self):
        """(L-infinity, L2, argmax (ix, iy, iz)) against the exact solution."""
        lmax, l2 = ctypes.c_double(), ctypes.c_double()
        am = np.zeros(3, dtype=np.int32)
        check(self._L.mts_norms(self._h, ctypes.byref(lmax), ctypes.byref(l2), am.ctypes.data), "mts_norms")
        return lmax.value, l2.value, tuple(int(v) for v in am)

    def norms_noalloc(self, u_dev_ptr: int | None = None, t: float = 0.0):
        """The same norms with no allocation (mts_norms_noalloc): of the
        device field at address u_dev_ptr evaluated at time t, or of the
        solver's own solution when u_dev_ptr is None.  Grids of at most
        4194304 nodes."""
        lmax, l2 = ctypes.c_double(), ctypes.c_double()
        am = np.zeros(3, dtype=np.int32)
        ptr = ctypes.c_void_p(u_dev_ptr) if u_dev_ptr else None
        check(self._L.mts_norms_noalloc(self._h, ptr, float(t), ctypes.byref(lmax), ctypes.byref(l2),
                                        am.ctypes.data), "mts_norms_noalloc")
        return lmax.value, l2.value, tuple(int(v) for v in am)

    # -- introspection -------------------------------------------------------
    def counts(self) -> dict:
        c = np.zeros(8, dtype=np.int64)
        check(self._L.mts_get_counts(self._h, c.ctypes.data), "mts_get_counts")
        return {"crossings": c[0:3].tolist(), "blocks": c[3:6].tolist(), "corner_pairs": int(c[6]),
                "singular_warnings": int(c[7])}

    def tags(self) -> np.ndarray:
        t = np.empty(self.spec.nodes, dtype=np.int8)
        check(self._L.mts_export_tags(self._h, t.ctypes.data), "mts_export_tags")
        return t

    def crossings(self) -> np.ndarray:
        n = ctypes.c_int32(0)
        check(self._L.mts_export_crossings(self._h, None, 0, ctypes.byref(n)), "mts_export_crossings")
        cr = np.zeros(n.value, dtype=CROSSING_DTYPE)
        check(self._L.mts_export_crossings(self._h, cr.ctypes.data if cr.size else None, cr.size, ctypes.byref(n)),
              "mts_export_crossings")
        return cr

    def launch_count(self) -> int:
        v = ctypes.c_int64()
        check(self._L.mts_get_launch_count(self._h, ctypes.byref(v)), "mts_get_launch_count")
        return int(v.value)

    def device_bytes(self) -> int:
        """Device memory this solver holds (mts_get_device_bytes)."""
        v = ctypes.c_int64()
        check(self._L.mts_get_device_bytes(self._h, ctypes.byref(v)), "mts_get_device_bytes")
        return int(v.value)

    def set_profiling(self, on: bool) -> None:
        check(self._L.mts_set_profiling(self._h, 1 if on else 0), "mts_set_profiling")

    def profile_read(self):
        """(ms[8], launches[8]) per kernel slot since the last read."""
        ms = np.zeros(8, dtype=np.float64)
        n = np.zeros(8, dtype=np.int64)
        check(self._L.mts_profile_read(self._h, ms.ctypes.data, n.ctypes.data), "mts_profile_read")
        return ms, n

    def set_sweep_shape(self, sweep: int, shape: int) -> None:
        check(self._L.mts_set_sweep_shape(self._h, int(sweep), int(shape)), "mts_set_sweep_shape")

    PRECISIONS = {"plain": 0, "mixed": 1, "fast": 2}

    def set_precision(self, precision: str) -> None:
        """"plain" (FP64, bit-identical to the reference), "mixed" (FP32
        line solves on the step's increment, FP64 residual and state;
        Douglas-ADI only) or "fast" (FP64 throughout, warp-segmented line
        solves of the increment, equal to the plain form up to rounding;
        Douglas-ADI only)."""
        check(self._L.mts_set_precision(self._h, self.PRECISIONS[precision]), "mts_set_precision")

    @property
    def precision(self) -> str:
        v = ctypes.c_int32()
        check(self._L.mts_get_precision(self._h, ctypes.byref(v)), "mts_get_precision")
        return {v_: k for k, v_ in self.PRECISIONS.items()}[v.value]

    def autotune(self, steps: int = 2):
        """Times every compiled sweep shape on this problem and keeps the
        fastest per sweep; the solution and time are left unchanged."""
        out = np.zeros(3, dtype=np.int32)
        check(self._L.mts_autotune(self._h, int(steps), out.ctypes.data), "mts_autotune")
        return tuple(int(v) for v in out)

    def fp_errors(self):
        """The fictitious points' error report at the current time
        (mts_fp_errors: Refresh_Fp + Error_Fp on the device): (L-infinity,
        root mean square) of their relative errors."""
        a, b = ctypes.c_double(), ctypes.c_double()
        check(self._L.mts_fp_errors(self._h, ctypes.byref(a), ctypes.byref(b)), "mts_fp_errors")
        return a.value, b.value

    def jump_errors(self):
        """The jumps' error report at the current time (mts_jump_errors:
        Refresh_Jump's check + Error_Jump on the device): (L-infinity, root
        mean square) of the relative errors of the jump data the solvers are
        given against the exact flux jumps."""
        a, b = ctypes.c_double(), ctypes.c_double()
        check(self._L.mts_jump_errors(self._h, ctypes.byref(a), ctypes.byref(b)), "mts_jump_errors")
        return a.value, b.value

    def stream(self) -> int:
        v = ctypes.c_void_p()
        check(self._L.mts_get_stream(self._h, ctypes.byref(v)), "mts_get_stream")
        return int(v.value or 0)
