"""The served form on the GPU: requests arriving over time are admitted into
the running batch (continuous batching); each result must be the one the
request gets alone, bit for bit, and the memory bound that admission uses
must hold for the handles actually created."""
import numpy as np
import pytest

import mts_b200 as M
from mts_b200 import serve
from mts_b200.workloads import Request, device_bytes_bound, draw_problem

pytestmark = pytest.mark.gpu


def test_served_results_equal_solving_alone():
    rng = np.random.default_rng(11)
    reqs, t = [], 0.0
    for i in range(16):
        t += float(rng.exponential(1.0 / 400.0))
        reqs.append(Request(i, draw_problem(rng, (17, 25, 33)), int(rng.integers(3, 13)), t))
    srv = serve.Server(hbm_budget=2e9, chunk_steps=2, host_threads=4, keep_solutions=True)
    out = srv.run(reqs)
    assert srv.peak_active >= 2  # the work of several requests overlapped
    for q, r in zip(reqs, out):
        alone = serve.solve_alone(q, keep_solution=True)
        assert r.t == alone.t and r.steps == q.steps
        assert np.array_equal(r.solution, alone.solution), q.spec
        assert r.lmax == alone.lmax
        assert r.latency > 0


@pytest.mark.parametrize("n", [(17, 25, 33), (65, 49, 65), (129, 129, 129)])
def test_device_bytes_bound_holds(n):
    rng = np.random.default_rng(5)
    spec = draw_problem(rng, n=n)
    tags, cr, _ = M.setup_host(spec)
    bound = device_bytes_bound(spec, len(cr))
    with M.Solver(spec, tags=tags, crossings=cr) as s:
        used = s.device_bytes()
    assert used <= bound <= 1.5 * used + (4 << 20), (used, bound)


@pytest.mark.parametrize("n", [(33, 49, 65), (129, 129, 129)])
def test_device_bytes_bound_holds_mixed(n):
    """The bound with the mixed form's per-node coefficients, which the
    library allocates when the form is switched on."""
    from dataclasses import replace

    spec = replace(draw_problem(np.random.default_rng(6), n=n), method="adi")
    tags, cr, _ = M.setup_host(spec)
    bound = device_bytes_bound(spec, len(cr), precision="mixed")
    with M.Solver(spec, tags=tags, crossings=cr) as s:
        s.set_precision("mixed")
        used = s.device_bytes()
    assert used <= bound <= 1.5 * used + (4 << 20), (used, bound)
