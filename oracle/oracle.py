"""Test infrastructure only: Python access to the checker.

* ``run_reference`` runs the reference's own time-stepping code (the binaries
  oracle/Makefile builds from the reference sources into oracle/_ref/) and
  returns its solution, node tags and crossing list.
* ``port_*`` call the plain-C restatement in oracle/mts_oracle.c.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REF_BIN = os.path.join(REF_DIR, "mts_ref")
REF_BIN_NOAUX = os.path.join(REF_DIR, "mts_ref_noaux")
# mts_ref_noaux with mts::GpuStepper (include/mts_reference_adapter.hpp)
# linked in: --gpu runs the reference's time loop on libmts_b200.so
REF_BIN_DROPIN = os.path.join(REF_DIR, "mts_dropin")
PORT_LIB = os.path.join(REF_DIR, "libmts_oracle.so")

METHODS = {"adi": 0, "lod-ie": 1, "lod-cn": 2, "ts": 3}

# One record per crossing; field meanings of Intersection_Data
# (src/constant.h:141-156).  Layout shared with oracle/ref_harness.cc.
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


@dataclass
class Problem:
    """One parabolic interface problem in the reference's terms."""

    n: tuple = (33, 33, 33)
    domain: tuple = (-1.0, 1.0, -1.0, 1.0, -1.0, 1.0)
    surface: str = "ellipsoid"  # "ellipsoid" (a b c r cx cy cz) or "torus" (R r)
    surface_params: tuple = (1.0, 1.0, 1.0, 0.49, 0.0, 0.0, 0.0)
    beta_in: float = 1.0
    beta_out: float = 10.0
    eq: int = 8
    method: str = "adi"
    mib: int = 1
    dt: float = 1.0 / 32
    t0: float = 0.0
    steps: int = 1

    def ref_args(self) -> list[str]:
        a = ["--n", *map(str, self.n), "--domain", *map(repr, self.domain)]
        a += ["--surface", self.surface, *map(repr, self.surface_params)]
        a += ["--beta", repr(self.beta_in), repr(self.beta_out), "--eq", str(self.eq)]
        a += ["--method", self.method, "--mib", str(self.mib), "--dt", repr(self.dt)]
        a += ["--t0", repr(self.t0), "--steps", str(self.steps)]
        return a


@dataclass
class RefResult:
    info: dict
    u: np.ndarray
    u0: np.ndarray
    tags: np.ndarray
    crossings: np.ndarray = field(repr=False)


def reference_available(noaux: bool = False, dropin: bool = False) -> bool:
    return os.path.exists(REF_BIN_DROPIN if dropin else REF_BIN_NOAUX if noaux else REF_BIN)


def run_reference(prob: Problem, noaux: bool = False, timeout: float = 3600, dropin_gpu: bool = False,
                  binary: str | None = None, report: str | None = None) -> RefResult:
    """Run the reference binary on ``prob``; raises RuntimeError when the
    reference aborts (it exits 0 on setup failures, so the JSON line is the
    success signal, as src/mesh/mesh.cc:64-65 and intersection.cc:2827 show).

    dropin_gpu: run the reference's setup and time loop with mts::GpuStepper
    stepping on the GPU in place of Douglas_ADI / LOD / TS (mts_dropin --gpu);
    the setup is the noaux one.  binary: run this build instead.  report: a
    path for the stepper's own Error() report after the last step."""
    binary = binary or (REF_BIN_DROPIN if dropin_gpu else REF_BIN_NOAUX if noaux else REF_BIN)
    with tempfile.TemporaryDirectory() as td:
        fu, fu0 = os.path.join(td, "u.bin"), os.path.join(td, "u0.bin")
        ft, fm = os.path.join(td, "tags.bin"), os.path.join(td, "mib.bin")
        cmd = [binary, *prob.ref_args(), "--dump-u", fu, "--dump-u0", fu0, "--dump-tags", ft, "--dump-mib", fm]
        if dropin_gpu:
            cmd.append("--gpu")
        if report:
            cmd += ["--report", report]
        cp = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        lines = [ln for ln in cp.stdout.splitlines() if ln.startswith("{")]
        if cp.returncode != 0 or not lines:
            raise RuntimeError(f"reference run failed (rc={cp.returncode}): {cp.stdout[-400:]} {cp.stderr[-400:]}")
        info = json.loads(lines[-1])
        u = np.fromfile(fu, dtype="<f8")
        u0 = np.fromfile(fu0, dtype="<f8")
        tags = np.fromfile(ft, dtype=np.int8)
        cr = np.fromfile(fm, dtype=CROSSING_DTYPE)
    return RefResult(info, u, u0, tags, cr)


class _OracleProblem(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("xl", ctypes.c_double),
        ("xr", ctypes.c_double),
        ("yl", ctypes.c_double),
        ("yr", ctypes.c_double),
        ("zl", ctypes.c_double),
        ("zr", ctypes.c_double),
        ("beta_in", ctypes.c_double),
        ("beta_out", ctypes.c_double),
        ("eq", ctypes.c_int32),
        ("pad", ctypes.c_int32),
        ("dt", ctypes.c_double),
    ]


_lib = None


def _port():
    global _lib
    if _lib is None:
        if not os.path.exists(PORT_LIB):
            subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
        lib = ctypes.CDLL(PORT_LIB)
        P = ctypes.POINTER
        lib.mts_oracle_init.argtypes = [P(_OracleProblem), ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
        lib.mts_oracle_run.argtypes = [
            P(_OracleProblem),
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_int32,
            ctypes.c_int32,
            ctypes.c_double,
            ctypes.c_int32,
            ctypes.c_void_p,
        ]
        lib.mts_oracle_norms.argtypes = [
            P(_OracleProblem),
            ctypes.c_void_p,
            ctypes.c_double,
            ctypes.c_void_p,
            P(ctypes.c_double),
            P(ctypes.c_double),
            ctypes.c_void_p,
        ]
        _lib = lib
    return _lib


def _cprob(prob: Problem) -> _OracleProblem:
    d = prob.domain
    return _OracleProblem(*prob.n, *d, prob.beta_in, prob.beta_out, prob.eq, 0, prob.dt)


def port_init(prob: Problem, tags: np.ndarray, t: float | None = None) -> np.ndarray:
    tags = np.ascontiguousarray(tags, dtype=np.int8)
    u = np.empty(tags.size, dtype=np.float64)
    cp = _cprob(prob)
    _port().mts_oracle_init(ctypes.byref(cp), tags.ctypes.data, prob.t0 if t is None else t, u.ctypes.data)
    return u


def port_run(prob: Problem, tags: np.ndarray, crossings: np.ndarray, u0: np.ndarray, steps: int | None = None,
             t0: float | None = None) -> np.ndarray:
    tags = np.ascontiguousarray(tags, dtype=np.int8)
    cr = np.ascontiguousarray(crossings, dtype=CROSSING_DTYPE)
    u = np.array(u0, dtype=np.float64, copy=True)
    cp = _cprob(prob)
    rc = _port().mts_oracle_run(
        ctypes.byref(cp), tags.ctypes.data, cr.ctypes.data if cr.size else None, cr.size,
        METHODS[prob.method], prob.t0 if t0 is None else t0, prob.steps if steps is None else steps, u.ctypes.data,
    )
    if rc != 0:
        raise RuntimeError(f"oracle step failed with status {rc}")
    return u


def port_norms(prob: Problem, tags: np.ndarray, t: float, u: np.ndarray):
    tags = np.ascontiguousarray(tags, dtype=np.int8)
    u = np.ascontiguousarray(u, dtype=np.float64)
    lmax, l2 = ctypes.c_double(), ctypes.c_double()
    am = np.zeros(3, dtype=np.int32)
    cp = _cprob(prob)
    _port().mts_oracle_norms(ctypes.byref(cp), tags.ctypes.data, t, u.ctypes.data, ctypes.byref(lmax),
                             ctypes.byref(l2), am.ctypes.data)
    return lmax.value, l2.value, tuple(int(v) for v in am)
