"""Seeded synthetic problem families of the batched and served workloads, and
the device-memory estimate that admission control uses.

Batched family: per-axis node counts uniform over {17, 25, 33, 49, 65}
(anisotropic grids on [-1,1]^3), ellipsoid interfaces with semi-axes
U(0.3, 0.7) and centres U(-0.2, 0.2)^3, beta_in = 1 and beta_out
log-uniform in [1e-3, 1e3], method uniform over ADI / LOD-IE / LOD-CN / TS,
MIB-L1 or L2, dt = the smallest axis spacing.  The generator is numpy's
PCG64 (numpy.random.default_rng(seed)).  A draw whose interface passes
through a grid node (which the reference rejects at setup) is redrawn.

Served family: the same draws, with 5 % of the grids at 129^3 and 1 % at
257^3, and t_end uniform over 20..200 steps.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import MtsError, Spec, setup_host

METHODS = ("adi", "lod-ie", "lod-cn", "ts")
BATCH_SIZES = (17, 25, 33, 49, 65)


def draw_problem(rng: np.random.Generator, sizes=BATCH_SIZES, n=None, validate=None) -> Spec:
    """One problem of the batched family (n forces the grid).  validate is
    the setup that accepts or rejects a draw (setup_host by default;
    setup_device accepts and rejects the same draws: the family's ellipsoid
    level set has no pow(v, 2))."""
    validate = validate or setup_host
    while True:
        grid = tuple(int(v) for v in rng.choice(sizes, 3)) if n is None else tuple(n)
        axes = rng.uniform(0.3, 0.7, 3)
        centre = rng.uniform(-0.2, 0.2, 3)
        spec = Spec(n=grid, surface="ellipsoid", surface_params=(*map(float, axes), 1.0, *map(float, centre)),
                    beta_in=1.0, beta_out=float(10.0 ** rng.uniform(-3.0, 3.0)), method=METHODS[int(rng.integers(4))],
                    mib=int(rng.integers(1, 3)), dt=min(2.0 / (k - 1) for k in grid))
        try:
            validate(spec)
            return spec
        except MtsError:
            continue  # interface through a grid node: the reference rejects it too


def batched_problems(count: int = 512, seed: int = 0, sizes=BATCH_SIZES) -> list[Spec]:
    rng = np.random.default_rng(seed)
    return [draw_problem(rng, sizes) for _ in range(count)]


@dataclass
class Request:
    id: int
    spec: Spec
    steps: int
    arrival: float  # seconds after the start of the stream


_STREAMS: dict = {}


def served_requests(count: int, rate: float, seed: int = 0, validate=None) -> list[Request]:
    """A Poisson stream of `count` requests at `rate` per second.  The
    problems and step counts do not depend on the rate (the gaps are one
    series of standard exponential draws scaled by 1/rate), so they are drawn
    once per (count, seed) and kept."""
    key = (count, seed)
    if key not in _STREAMS:
        rng = np.random.default_rng(seed)
        draws = []
        for _ in range(count):
            e = float(rng.standard_exponential())
            u = rng.uniform()
            n = (257, 257, 257) if u < 0.01 else (129, 129, 129) if u < 0.06 else None
            spec = draw_problem(rng, BATCH_SIZES, n, validate)
            draws.append((e, spec, int(rng.integers(20, 201))))
        _STREAMS[key] = draws
    t = 0.0
    out = []
    scale = 1.0 / rate
    for i, (e, spec, steps) in enumerate(_STREAMS[key]):
        t += scale * e
        out.append(Request(i, spec, steps, t))
    return out


def size_class(spec: Spec) -> str:
    """The served stream's strata: the batched family's grids, 129^3, 257^3."""
    m = max(spec.n)
    return "257" if m >= 257 else "129" if m >= 129 else "small"


def device_bytes_bound(spec: Spec, ncrossings: int, sms: int = 148, precision: str = "plain") -> int:
    """An upper bound on the device memory mts_create allocates for `spec`
    with `ncrossings` crossings (the layout of the library's allocations: two
    FP64 fields, FP64 and FP32 per-node factors for every direction, the FP32
    increment, both d' scratches, the tables and the MIB data), plus, for the
    mixed form, the segmented solves' per-node coefficients (three FP32
    values per node and direction, built when the form is switched on)."""
    nx, ny, nz = spec.n
    N = nx * ny * nz
    nmax = max(spec.n)
    lines = [ny * nz, nx * nz, nx * ny]
    maxlines = max(lines)
    pad = 16 * nx * ny
    t64 = min(sms * 512, maxlines + 512)
    t32 = min(sms * 448, maxlines + 448)
    b = 0
    b += 2 * 8 * (N + pad)                       # u0, u1
    b += 8 * (nmax + 16) * t64                   # d' scratch, FP64
    b += 3 * 2 * 8 * (N + pad)                   # per-node bet, gam (FP64)
    b += 3 * 2 * 4 * (N + pad)                   # per-node 1/bet, gam (FP32)
    b += 4 * (N + pad) + 4 * (nmax + 16) * t32   # FP32 increment and d' scratch
    b += N + sum(lines) * 5 + 4 * 3              # tags, line sides, CSR offsets
    b += 3 * 2 * 2 * 12 * nmax + 3 * 3 * 8 * nmax  # prefix tables, axis tables
    b += ncrossings * (432 + 3 * 12 + 88 + 16 + 3 * 8)  # blocks, block RHS, constants, jumps, MIB nodes
    b += 4096 * 3 * 8 + 64                        # norm partials
    if precision == "mixed" and spec.method == "adi" and nmax <= 544:
        b += 3 * 3 * 4 * N                        # cib, cp, cq per direction
    return int(b * 1.02) + (1 << 20)
