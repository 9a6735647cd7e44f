"""Batched stepping (mts_batch_advance): the plain problems of a method
advance together, one launch per kernel of a step for all of them; large and
mixed-precision problems step on their own streams alongside.  Each
problem's result must be bit-identical to
stepping it alone, whatever the mix of methods, MIB variants, grid shapes,
beta ratios and precision forms in the batch (the problems are drawn as the
batched workload draws them: anisotropic grids, shifted ellipsoids, beta_out
log-uniform)."""
import numpy as np
import pytest

import mts_b200 as M

pytestmark = pytest.mark.gpu
METHODS = ["adi", "lod-ie", "lod-cn", "ts"]


def draw(rng, sizes=(17, 25, 33)):
    """One problem of the batched workload, redrawn while the interface
    touches a grid node (the reference rejects such geometries)."""
    while True:
        n = tuple(int(v) for v in rng.choice(sizes, 3))
        axes = rng.uniform(0.3, 0.7, 3)
        centre = rng.uniform(-0.2, 0.2, 3)
        spec = M.Spec(n=n, surface="ellipsoid", surface_params=(*axes, 1.0, *centre), beta_in=1.0,
                      beta_out=float(10.0 ** rng.uniform(-3, 3)), method=METHODS[rng.integers(4)],
                      mib=int(rng.integers(1, 3)), dt=min(2.0 / (k - 1) for k in n))
        try:
            M.setup_host(spec)
            return spec
        except M.MtsError:
            continue


def solve_alone(spec, precision, steps):
    with M.Solver(spec) as s:
        s.set_precision(precision)
        s.initialize()
        s.advance(steps)
        s.synchronize()
        return s.solution(), s.time


def test_batch_equals_individual_runs():
    rng = np.random.default_rng(7)
    specs = [draw(rng) for _ in range(12)]
    # one mixed-precision Douglas-ADI problem in the mix
    adi = next(i for i, s in enumerate(specs) if s.method == "adi")
    precision = ["mixed" if i == adi else "plain" for i in range(len(specs))]
    solvers = [M.Solver(sp) for sp in specs]
    try:
        for s, p in zip(solvers, precision):
            s.set_precision(p)
            s.initialize()
        M.batch_advance(solvers, 5)
        M.batch_advance(solvers, 4)
        for sp, s, p in zip(specs, solvers, precision):
            u, t = solve_alone(sp, p, 9)
            assert s.time == t
            assert np.array_equal(s.solution(), u), (sp, p)
    finally:
        for s in solvers:
            s.close()


def test_batch_rejects_duplicates():
    rng = np.random.default_rng(3)
    sp = draw(rng)
    with M.Solver(sp) as s:
        with pytest.raises(M.MtsError, match="twice"):
            M.batch_advance([s, s], 1)


def test_batch_with_per_problem_step_counts():
    """Problems with different numbers of steps in one batch: each stops at
    its own count (the server's chunks)."""
    rng = np.random.default_rng(21)
    specs = [draw(rng) for _ in range(8)]
    counts = [int(c) for c in rng.integers(0, 7, len(specs))]
    solvers = [M.Solver(sp) for sp in specs]
    try:
        for s in solvers:
            s.initialize()
        M.batch_advance_steps(solvers, counts)
        for sp, s, c in zip(specs, solvers, counts):
            u, t = solve_alone(sp, "plain", c)
            assert s.time == t
            assert np.array_equal(s.solution(), u), (sp, c)
    finally:
        for s in solvers:
            s.close()


def test_batch_with_large_problems_on_their_own_streams():
    """Problems whose lines fill the GPU (here 200^3 = 39,204 lines a
    direction, plain ADI and TS) step on their own streams with their own
    shapes, beside the batched small ones and a 129^3 one: every result is
    still that of stepping the problem alone."""
    rng = np.random.default_rng(5)
    specs = [draw(rng) for _ in range(3)]
    specs.append(M.Spec(n=(129, 129, 129), surface="torus", surface_params=(0.5, 0.2), beta_in=1.0,
                        beta_out=1000.0, method="lod-cn", mib=1, dt=2.0 / 128))
    for method in ("adi", "ts"):
        specs.append(M.Spec(n=(200, 200, 200), surface="torus", surface_params=(0.5, 0.2), beta_in=1.0,
                            beta_out=1000.0, method=method, mib=2, dt=2.0 / 199))
    counts = [3, 0, 5, 2, 4, 3]
    solvers = [M.Solver(sp) for sp in specs]
    try:
        for s in solvers:
            s.initialize()
        M.batch_advance_steps(solvers, counts)
        for sp, s, c in zip(specs, solvers, counts):
            u, t = solve_alone(sp, "plain", c)
            assert s.time == t
            assert np.array_equal(s.solution(), u), (sp, c)
    finally:
        for s in solvers:
            s.close()


def test_mixed_problems_batch_in_their_own_group():
    """Mixed-precision Douglas-ADI problems with lines of at most 160 rows
    advance together in one batched launch sequence of the mixed step (the
    FP32 segmented solves, a warp per line, inside multi-problem launches):
    bit-identical to stepping each alone, beside plain problems of every
    method, with uneven step counts; their L-infinity error stays within
    1.05x of the plain form's."""
    rng = np.random.default_rng(21)
    specs = []
    while len([s for s in specs if s.method == "adi"]) < 6:
        specs.append(draw(rng, sizes=(17, 25, 33, 49, 65)))
    precision = ["mixed" if s.method == "adi" else "plain" for s in specs]
    counts = [4 + (i % 5) for i in range(len(specs))]
    solvers = [M.Solver(sp) for sp in specs]
    try:
        for s, p in zip(solvers, precision):
            s.set_precision(p)
            s.initialize()
        M.batch_advance_steps(solvers, counts)
        for sp, s, p, k in zip(specs, solvers, precision, counts):
            u, t = solve_alone(sp, p, k)
            assert s.time == t
            assert np.array_equal(s.solution(), u), (sp, p)
            if p == "mixed":
                with M.Solver(sp) as ref:
                    ref.initialize()
                    ref.advance(k)
                    ref.synchronize()
                    lp = ref.norms()[0]
                assert s.norms()[0] <= 1.05 * lp + 1e-12, (sp, s.norms()[0], lp)
    finally:
        for s in solvers:
            s.close()
