"""GPU parity: the CUDA path (through the C ABI) against the reference's
golden outputs and against the oracle.

Tolerance: 1e-10 relative max-norm (max |u_gpu - u_ref| / max |u_ref|), the
plain FP64 form's contract.  The kernels round every operation exactly as the
reference build does, so the observed difference is expected to be 0; the
tests also assert that, to catch any drift early."""
import numpy as np
import pytest

import mts_b200 as M
import oracle as O
from conftest import load_golden, problem_from_dict, rel_maxdiff, spec_from_problem

pytestmark = pytest.mark.gpu
TOL = 1e-10


def run_gpu(spec, steps, tags=None, crossings=None, u0=None):
    with M.Solver(spec, tags=tags, crossings=crossings) as s:
        if u0 is None:
            s.initialize()
        else:
            s.set_solution(u0)
        s.advance(steps)
        s.synchronize()
        return s.solution(), s.norms(), s.time


@pytest.mark.parametrize("path", ["own_setup", "reference_crossings"])
def test_gpu_matches_golden(golden, path):
    worst = 0.0
    for name, entry in golden.items():
        prob = problem_from_dict(entry["problem"])
        u_ref, u0, tags, cr = load_golden(name)
        spec = spec_from_problem(prob)
        if path == "own_setup":
            u, (lmax, l2, am), t = run_gpu(spec, prob.steps)
        else:
            u, (lmax, l2, am), t = run_gpu(spec, prob.steps, tags=tags, crossings=cr, u0=u0)
        d = rel_maxdiff(u, u_ref)
        worst = max(worst, d)
        assert d <= TOL, f"{name}: relative max-norm difference {d:.3e}"
        assert np.array_equal(u, u_ref), f"{name}: not bit-identical (rel {d:.3e})"
        assert t == entry["info"]["t"]
        assert lmax == entry["info"]["lmax"], name
        assert abs(l2 - entry["info"]["l2"]) <= 1e-12 * max(1.0, entry["info"]["l2"]), name
        assert list(am) == entry["info"]["argmax"], name
    print(f"worst relative difference over {len(golden)} golden cases: {worst:.3e}")


def test_gpu_initialize_matches_reference(golden):
    for name, entry in golden.items():
        prob = problem_from_dict(entry["problem"])
        _, u0, _, _ = load_golden(name)
        with M.Solver(spec_from_problem(prob)) as s:
            s.initialize()
            assert np.array_equal(s.solution(), u0), name


RANDOM_CASES = []
_rng = np.random.default_rng(0)
for _i in range(8):
    _n = tuple(int(v) for v in _rng.choice([17, 25, 33, 49, 65], size=3))
    _ax = tuple(float(v) for v in _rng.uniform(0.3, 0.7, size=3))
    _c = tuple(float(v) for v in _rng.uniform(-0.2, 0.2, size=3))
    _bo = float(10 ** _rng.uniform(-3, 3))
    _method = ["adi", "lod-ie", "lod-cn", "ts"][_i % 4]
    RANDOM_CASES.append(dict(n=_n, surface_params=(*_ax, 1.0, *_c), beta_out=_bo, method=_method, mib=1 + (_i // 4)))


@pytest.mark.parametrize("case", RANDOM_CASES, ids=[f"{c['method']}-l{c['mib']}-{c['n']}" for c in RANDOM_CASES])
def test_gpu_matches_oracle_random_family(case):
    """Problems drawn like the batched family (anisotropic grids, shifted
    ellipsoids, beta_out log-uniform in [1e-3, 1e3]): GPU vs oracle."""
    n = case["n"]
    h = 2.0 / (min(n) - 1)
    spec = M.Spec(n=n, surface_params=case["surface_params"], beta_in=1.0, beta_out=case["beta_out"],
                  method=case["method"], mib=case["mib"], dt=h)
    try:
        tags, cr, _ = M.setup_host(spec)
    except M.MtsError:
        pytest.skip("geometry rejected by the reference setup rules")
    prob = O.Problem(n=n, surface_params=case["surface_params"], beta_in=1.0, beta_out=case["beta_out"],
                     method=case["method"], mib=case["mib"], dt=h, steps=5)
    u0 = O.port_init(prob, tags)
    u_or = O.port_run(prob, tags, cr, u0)
    u, _, _ = run_gpu(spec, 5)
    assert rel_maxdiff(u, u_or) <= TOL
    assert np.array_equal(u, u_or)


@pytest.mark.parametrize("method", ["adi", "lod-ie", "lod-cn", "ts"])
@pytest.mark.parametrize("surface", ["ellipsoid", "torus"])
def test_gpu_matches_oracle_65(method, surface):
    """The drop-in configuration at 65^3 (beta 1:1000, dt = h) with MIB-L2,
    a few steps, GPU vs oracle."""
    sp = (0.7001, 0.4999, 0.4001, 1.0) if surface == "ellipsoid" else (0.5, 0.2)
    spec = M.Spec(n=(65, 65, 65), surface=surface, surface_params=sp, beta_in=1.0, beta_out=1000.0, method=method,
                  mib=2, dt=2.0 / 64)
    tags, cr, _ = M.setup_host(spec)
    prob = O.Problem(n=(65, 65, 65), surface=surface, surface_params=sp, beta_in=1.0, beta_out=1000.0,
                     method=method, mib=2, dt=2.0 / 64, steps=3)
    u_or = O.port_run(prob, tags, cr, O.port_init(prob, tags))
    u, (lmax, l2, am), t = run_gpu(spec, 3)
    assert rel_maxdiff(u, u_or) <= TOL
    assert np.array_equal(u, u_or)
    lo, l2o, amo = O.port_norms(prob, tags, t, u_or)
    assert lmax == lo and tuple(am) == amo
    assert abs(l2 - l2o) <= 1e-12 * l2o


@pytest.mark.parametrize("method", ["adi", "lod-ie", "lod-cn", "ts"])
def test_every_sweep_shape_gives_the_oracle_bits(method):
    """Every compiled sweep shape (chunk rows, ring depth, threads per CTA)
    takes different fast and slow paths through a line; all must give the
    oracle's bits.  Line lengths 67/61/70 are not multiples of the chunk rows,
    so every line ends inside a partial chunk."""
    n = (67, 61, 70)
    spec = M.Spec(n=n, surface="torus", surface_params=(0.5, 0.2), beta_in=1.0, beta_out=1000.0, method=method,
                  mib=2, dt=2.0 / 64)
    tags, cr, _ = M.setup_host(spec)
    prob = O.Problem(n=n, surface="torus", surface_params=(0.5, 0.2), beta_in=1.0, beta_out=1000.0, method=method,
                     mib=2, dt=2.0 / 64, steps=2)
    u_or = O.port_run(prob, tags, cr, O.port_init(prob, tags))
    tried = 0
    with M.Solver(spec) as s:
        for shape in range(M.load().mts_sweep_shape_count()):
            try:
                for k in range(3):
                    s.set_sweep_shape(k, shape)
            except M.MtsError:
                continue  # needs more shared memory than these lines allow
            s.time = 0.0
            s.initialize()
            s.advance(2)
            s.synchronize()
            u = s.solution()
            assert np.array_equal(u, u_or), f"shape {shape}: rel {rel_maxdiff(u, u_or):.3e}"
            tried += 1
    assert tried >= 6


@pytest.mark.parametrize("method", ["adi", "lod-ie", "lod-cn", "ts"])
@pytest.mark.parametrize("mib", [1, 2])
@pytest.mark.parametrize("surface", ["ellipsoid", "torus"])
def test_gpu_matches_oracle_129(method, mib, surface):
    """The 129^3 grid of the drop-in configuration (beta 1:1000, dt = h),
    every method and MIB variant, 2 steps, GPU vs oracle bit for bit."""
    n = (129, 129, 129)
    sp = (0.7001, 0.4999, 0.4001, 1.0) if surface == "ellipsoid" else (0.5, 0.2)
    spec = M.Spec(n=n, surface=surface, surface_params=sp, beta_in=1.0, beta_out=1000.0, method=method, mib=mib,
                  dt=2.0 / 128)
    tags, cr, _ = M.setup_host(spec)
    prob = O.Problem(n=n, surface=surface, surface_params=sp, beta_in=1.0, beta_out=1000.0, method=method, mib=mib,
                     dt=2.0 / 128, steps=2)
    u_or = O.port_run(prob, tags, cr, O.port_init(prob, tags))
    u, _, _ = run_gpu(spec, 2)
    assert rel_maxdiff(u, u_or) <= TOL
    assert np.array_equal(u, u_or)


@pytest.mark.parametrize("method", ["adi", "lod-ie", "lod-cn", "ts"])
def test_gpu_matches_oracle_257(method):
    """The bench's 257^3 grid (torus, MIB-L2, beta 1:1000, dt = h), 2 steps of
    every method, GPU vs oracle bit for bit."""
    n = (257, 257, 257)
    spec = M.Spec(n=n, surface="torus", surface_params=(0.5, 0.2), beta_in=1.0, beta_out=1000.0, method=method,
                  mib=2, dt=2.0 / 256)
    tags, cr, _ = M.setup_host(spec)
    prob = O.Problem(n=n, surface="torus", surface_params=(0.5, 0.2), beta_in=1.0, beta_out=1000.0, method=method,
                     mib=2, dt=2.0 / 256, steps=2)
    u_or = O.port_run(prob, tags, cr, O.port_init(prob, tags))
    u, (lmax, l2, am), t = run_gpu(spec, 2)
    assert rel_maxdiff(u, u_or) <= TOL
    assert np.array_equal(u, u_or)
    lo, l2o, amo = O.port_norms(prob, tags, t, u_or)
    assert lmax == lo and tuple(am) == amo


def test_eq0_constant_solution_is_kept_at_257():
    """A size-independent property at the full size: with Eq_0 (constant
    solutions 80 inside, 100 outside, zero source, jumps [u] = 20) the scheme
    keeps the exact solution to rounding, as the reference does (its Eq_0
    error is 4e-12 at 33^3)."""
    spec = M.Spec(n=(257, 257, 257), surface="torus", surface_params=(0.5, 0.2), beta_in=1.0, beta_out=1000.0,
                  eq=0, method="adi", mib=2, dt=2.0 / 256)
    u, (lmax, l2, _), _ = run_gpu(spec, 3)
    assert lmax <= 1e-9 * 100.0, lmax


@pytest.mark.parametrize("method", ["adi", "lod-ie", "lod-cn", "ts"])
def test_gpu_without_crossings(method):
    """An interface that crosses no grid line (a sphere between the nodes):
    no MIB rows, no per-node factors, no jump data; GPU vs oracle, alone and
    in a batch."""
    spec = M.Spec(n=(17, 17, 17), surface="ellipsoid", surface_params=(1.0, 1.0, 1.0, 0.1, 0.0625, 0.0625, 0.0625),
                  beta_in=1.0, beta_out=10.0, method=method, mib=2, dt=0.125)
    tags, cr, _ = M.setup_host(spec)
    assert len(cr) == 0
    prob = O.Problem(n=spec.n, surface="ellipsoid", surface_params=spec.surface_params, beta_in=1.0, beta_out=10.0,
                     method=method, mib=2, dt=0.125, steps=3)
    u_or = O.port_run(prob, tags, cr, O.port_init(prob, tags))
    u, _, _ = run_gpu(spec, 3)
    assert np.array_equal(u, u_or)
    with M.Solver(spec) as s:
        s.initialize()
        M.batch_advance([s], 3)
        assert np.array_equal(s.solution(), u_or)
