"""The fast FP64 form of the Douglas-ADI step (MTS_PRECISION_FAST) against the
reference's golden outputs, the oracle, and the bit-exact plain form.

The fast form computes in FP64 throughout but in another order (the step is
solved for its increment, the residual is formed inside the x sweep with
fused multiply-adds, and each line is solved by one warp in segments joined
by shuffle scans), so it matches the reference up to rounding only.
Tolerance, the plain form's contract: 1e-10 relative max-norm
(max |u_fast - u_ref| / max |u_ref|).  The L-infinity and L2 errors against
the exact solution must agree with the reference's to 1e-8 relative (plus
1e-11 absolute, for the Eq_0 case whose errors are rounding alone)."""
import numpy as np
import pytest

import mts_b200 as M
import oracle as O
from conftest import load_golden, problem_from_dict, rel_maxdiff, spec_from_problem

pytestmark = pytest.mark.gpu
TOL = 1e-10
NORM_TOL = 1e-8
ELLIPSOID = (0.7001, 0.4999, 0.4001, 1.0)
SPHERE = (1.0, 1.0, 1.0, 0.49)
TORUS = (0.5, 0.2)


def run(spec, steps, precision="fast", tags=None, crossings=None, u0=None):
    with M.Solver(spec, tags=tags, crossings=crossings) as s:
        s.set_precision(precision)
        assert s.precision == precision
        if u0 is None:
            s.initialize()
        else:
            s.set_solution(u0)
        s.advance(steps)
        s.synchronize()
        return s.solution(), s.norms(), s.time


def close_norms(a, b):
    # (plus 1e-11 absolute: the Eq_0 known answer has errors of ~1e-13 that
    # are rounding alone)
    return abs(a - b) <= NORM_TOL * abs(b) + 1e-11


@pytest.mark.parametrize("path", ["own_setup", "reference_crossings"])
def test_fast_matches_golden(golden, path):
    """Every Douglas-ADI golden case: spheres, the shifted anisotropic
    ellipsoid with corner pairs, the torus, Eq_0, and the config-0 run to
    t = 1 (32 steps)."""
    cases = [n for n, e in golden.items() if e["problem"]["method"] == "adi"]
    assert len(cases) >= 6
    for name in cases:
        entry = golden[name]
        prob = problem_from_dict(entry["problem"])
        u_ref, u0, tags, cr = load_golden(name)
        spec = spec_from_problem(prob)
        if path == "own_setup":
            u, (lmax, l2, _), t = run(spec, prob.steps)
        else:
            u, (lmax, l2, _), t = run(spec, prob.steps, tags=tags, crossings=cr, u0=u0)
        d = rel_maxdiff(u, u_ref)
        assert d <= TOL, f"{name}: relative max-norm difference {d:.3e}"
        assert t == entry["info"]["t"]
        assert close_norms(lmax, entry["info"]["lmax"]), (name, lmax, entry["info"]["lmax"])
        assert close_norms(l2, entry["info"]["l2"]), (name, l2, entry["info"]["l2"])


RANDOM_CASES = []
_rng = np.random.default_rng(7)
for _i in range(6):
    _n = tuple(int(v) for v in _rng.choice([17, 25, 33, 49, 65], size=3))
    _ax = tuple(float(v) for v in _rng.uniform(0.3, 0.7, size=3))
    _c = tuple(float(v) for v in _rng.uniform(-0.2, 0.2, size=3))
    _bo = float(10 ** _rng.uniform(-3, 3))
    RANDOM_CASES.append(dict(n=_n, surface_params=(*_ax, 1.0, *_c), beta_out=_bo, mib=1 + _i % 2))


@pytest.mark.parametrize("case", RANDOM_CASES, ids=[f"l{c['mib']}-{c['n']}" for c in RANDOM_CASES])
def test_fast_matches_oracle_random_family(case):
    """Anisotropic grids of the batched family (segment lengths 1, 3 per
    lane, partial tiles), shifted ellipsoids, beta_out in [1e-3, 1e3]."""
    n = case["n"]
    h = 2.0 / (min(n) - 1)
    spec = M.Spec(n=n, surface_params=case["surface_params"], beta_in=1.0, beta_out=case["beta_out"], method="adi",
                  mib=case["mib"], dt=h)
    try:
        tags, cr, _ = M.setup_host(spec)
    except M.MtsError:
        pytest.skip("geometry rejected by the reference setup rules")
    prob = O.Problem(n=n, surface_params=case["surface_params"], beta_in=1.0, beta_out=case["beta_out"],
                     method="adi", mib=case["mib"], dt=h, steps=6)
    u_or = O.port_run(prob, tags, cr, O.port_init(prob, tags))
    u, _, _ = run(spec, 6)
    assert rel_maxdiff(u, u_or) <= TOL


@pytest.mark.parametrize("mib", [1, 2])
@pytest.mark.parametrize("surface,params", [("ellipsoid", SPHERE), ("ellipsoid", ELLIPSOID), ("torus", TORUS)],
                         ids=["sphere", "ellipsoid", "torus"])
def test_fast_matches_oracle_65_to_t1(surface, params, mib):
    """The drop-in configuration at 65^3 (beta 1:1000, dt = h) to t_end = 1
    (32 steps), fast form against the oracle, with the error norms."""
    spec = M.Spec(n=(65, 65, 65), surface=surface, surface_params=params, beta_in=1.0, beta_out=1000.0,
                  method="adi", mib=mib, dt=2.0 / 64)
    tags, cr, _ = M.setup_host(spec)
    prob = O.Problem(n=(65, 65, 65), surface=surface, surface_params=params, beta_in=1.0, beta_out=1000.0,
                     method="adi", mib=mib, dt=2.0 / 64, steps=32)
    u_or = O.port_run(prob, tags, cr, O.port_init(prob, tags))
    lo, l2o, _ = O.port_norms(prob, tags, 1.0, u_or)
    u, (lmax, l2, _), t = run(spec, 32)
    assert t == 1.0
    d = rel_maxdiff(u, u_or)
    assert d <= TOL, f"relative max-norm difference {d:.3e}"
    assert close_norms(lmax, lo) and close_norms(l2, l2o), (lmax, lo, l2, l2o)


@pytest.mark.parametrize("n", [(17, 17, 17), (33, 65, 129), (37, 29, 45), (129, 129, 129)])
def test_fast_matches_plain_edges(n):
    """Line lengths that leave the last lanes short or empty, a different
    segment length per direction, odd sizes and partial tiles; against the
    plain form (bit-identical to the reference)."""
    spec = M.Spec(n=n, surface="torus", surface_params=TORUS, beta_in=1.0, beta_out=1000.0, method="adi", mib=2,
                  dt=2.0 / (max(n) - 1))
    u_p, _, _ = run(spec, 4, "plain")
    u_f, _, _ = run(spec, 4, "fast")
    assert rel_maxdiff(u_f, u_p) <= TOL


@pytest.mark.parametrize("n", [(400, 33, 35), (33, 520, 35), (35, 33, 300), (300, 300, 40)])
def test_fast_long_lines(n):
    """Lines of 289-544 rows (13 and 17 rows per lane) in x (the x pass with
    4 lines per CTA), in y, and in z with the update."""
    spec = M.Spec(n=n, surface="ellipsoid", surface_params=(0.61, 0.52, 0.43, 1.0, 0.05, -0.03, 0.02),
                  beta_in=1.0, beta_out=100.0, method="adi", mib=2, dt=2.0 / (max(n) - 1))
    u_p, _, _ = run(spec, 3, "plain")
    u_f, _, _ = run(spec, 3, "fast")
    assert rel_maxdiff(u_f, u_p) <= TOL


@pytest.mark.parametrize("mib", [1, 2])
def test_fast_257_torus(mib):
    """The bench workload (257^3, torus, beta 1:1000, dt = h), 3 steps,
    against the plain form and against the oracle."""
    spec = M.Spec(n=(257, 257, 257), surface="torus", surface_params=TORUS, beta_in=1.0, beta_out=1000.0,
                  method="adi", mib=mib, dt=2.0 / 256)
    u_p, (lp, l2p, _), _ = run(spec, 3, "plain")
    u_f, (lf, l2f, _), _ = run(spec, 3, "fast")
    assert rel_maxdiff(u_f, u_p) <= TOL
    assert close_norms(lf, lp) and close_norms(l2f, l2p)
    tags, cr, _ = M.setup_host(spec)
    prob = O.Problem(n=(257, 257, 257), surface="torus", surface_params=TORUS, beta_in=1.0, beta_out=1000.0,
                     method="adi", mib=mib, dt=2.0 / 256, steps=3)
    u_or = O.port_run(prob, tags, cr, O.port_init(prob, tags))
    assert rel_maxdiff(u_f, u_or) <= TOL


def test_fast_sphere_257():
    spec = M.Spec(n=(257, 257, 257), surface="ellipsoid", surface_params=SPHERE, beta_in=1.0, beta_out=1000.0,
                  method="adi", mib=2, dt=2.0 / 256)
    u_p, _, _ = run(spec, 3, "plain")
    u_f, _, _ = run(spec, 3, "fast")
    assert rel_maxdiff(u_f, u_p) <= TOL


def test_fast_rejects_what_it_cannot_take():
    spec = M.Spec(n=(33, 33, 33), surface="torus", surface_params=TORUS, beta_in=1.0, beta_out=10.0,
                  method="lod-cn", mib=2, dt=1.0 / 16)
    with M.Solver(spec) as s:
        with pytest.raises(M.MtsError, match="Douglas-ADI only"):
            s.set_precision("fast")
        assert s.precision == "plain"
    spec = M.Spec(n=(600, 17, 17), surface="ellipsoid", surface_params=(0.61, 0.52, 0.43, 1.0, 0.05, -0.03, 0.02),
                  beta_in=1.0, beta_out=10.0, method="adi", mib=2, dt=2.0 / 16)
    with M.Solver(spec) as s:
        with pytest.raises(M.MtsError, match="544"):
            s.set_precision("fast")


def test_fast_switches_back_and_forth():
    """Plain and fast steps interleave on one handle: the state is the same
    field, only the kernels differ."""
    spec = M.Spec(n=(49, 41, 57), surface="ellipsoid", surface_params=(0.61, 0.52, 0.43, 1.0, 0.05, -0.03, 0.02),
                  beta_in=1.0, beta_out=1000.0, method="adi", mib=2, dt=2.0 / 56)
    assert M.setup_host(spec)[2]["singular_warnings"] == 0
    u_p, _, _ = run(spec, 4, "plain")
    with M.Solver(spec) as s:
        s.initialize()
        for k in range(4):
            s.set_precision("fast" if k % 2 else "plain")
            s.advance(1)
        s.synchronize()
        u = s.solution()
    assert rel_maxdiff(u, u_p) <= TOL


def test_fast_on_a_problem_sensitive_to_rounding():
    """A torus on a coarse anisotropic grid (49 x 41 x 57) where four of the
    MIB weight systems are near-singular (the setup's singular-matrix
    warnings, intersection.cc:1034-1057).  There the reference's own result
    moves by about 1e-5 under any change of rounding (its code compiled with
    fused multiply-adds differs from itself by 9e-6 after 4 steps), so the
    1e-10 contract can only be met bit for bit, by the plain form; the fast
    form stays within that sensitivity."""
    spec = M.Spec(n=(49, 41, 57), surface="torus", surface_params=TORUS, beta_in=1.0, beta_out=1000.0,
                  method="adi", mib=2, dt=2.0 / 56)
    assert M.setup_host(spec)[2]["singular_warnings"] > 0
    u_p, _, _ = run(spec, 4, "plain")
    u_f, _, _ = run(spec, 4, "fast")
    assert rel_maxdiff(u_f, u_p) <= 1e-4


@pytest.mark.parametrize("mib", [1, 2])
@pytest.mark.parametrize("surface,params", [("ellipsoid", SPHERE), ("ellipsoid", ELLIPSOID), ("torus", TORUS)],
                         ids=["sphere", "ellipsoid", "torus"])
def test_fast_matches_oracle_129(surface, params, mib):
    """129^3 (beta 1:1000, dt = h), 2 steps, every interface and MIB variant."""
    spec = M.Spec(n=(129, 129, 129), surface=surface, surface_params=params, beta_in=1.0, beta_out=1000.0,
                  method="adi", mib=mib, dt=2.0 / 128)
    tags, cr, _ = M.setup_host(spec)
    prob = O.Problem(n=(129, 129, 129), surface=surface, surface_params=params, beta_in=1.0, beta_out=1000.0,
                     method="adi", mib=mib, dt=2.0 / 128, steps=2)
    u_or = O.port_run(prob, tags, cr, O.port_init(prob, tags))
    u, (lmax, l2, _), t = run(spec, 2)
    assert rel_maxdiff(u, u_or) <= TOL
    lo, l2o, _ = O.port_norms(prob, tags, t, u_or)
    assert close_norms(lmax, lo) and close_norms(l2, l2o)


@pytest.mark.parametrize("params", [SPHERE, ELLIPSOID], ids=["sphere", "ellipsoid"])
def test_fast_257_l1(params):
    spec = M.Spec(n=(257, 257, 257), surface="ellipsoid", surface_params=params, beta_in=1.0, beta_out=1000.0,
                  method="adi", mib=1, dt=2.0 / 256)
    u_p, _, _ = run(spec, 2, "plain")
    u_f, _, _ = run(spec, 2, "fast")
    assert rel_maxdiff(u_f, u_p) <= TOL
