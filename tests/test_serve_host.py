"""Host logic of the server (mts_b200.serve) without a GPU: admission against
the memory budget, continuous batching of arrivals into the running batch,
retirement, and the FIFO model of the sequential baseline.  The device calls
are replaced by fakes that count steps."""
import time

import numpy as np
import pytest

import mts_b200 as M
from mts_b200 import serve
from mts_b200.workloads import Request


class FakeSolver:
    live = 0
    peak = 0

    def __init__(self, spec, tags=None, crossings=None):
        self.spec, self.time, self.closed = spec, spec.t0, False
        FakeSolver.live += 1
        FakeSolver.peak = max(FakeSolver.peak, FakeSolver.live)

    def initialize(self):
        pass

    def synchronize(self):
        pass

    def device_bytes(self):
        return 1000

    def norms(self):
        return (self.time, 0.0, (0, 0, 0))

    def solution(self):
        return np.full(3, self.time)

    def close(self):
        if not self.closed:
            FakeSolver.live -= 1
            self.closed = True


def fake_batch(solvers, ks):
    time.sleep(0.001)
    for s, k in zip(solvers, ks):
        s.time += k * s.spec.dt


@pytest.fixture
def fakes(monkeypatch):
    monkeypatch.setattr(serve, "Solver", FakeSolver)
    monkeypatch.setattr(serve, "batch_advance_steps", fake_batch)
    monkeypatch.setattr(serve, "setup_host", lambda spec: (None, np.zeros(4), None))
    monkeypatch.setattr(serve, "device_bytes_bound", lambda spec, nc, **kw: 100)
    FakeSolver.live = FakeSolver.peak = 0


def reqs(n, gap, steps=lambda i: 5 + 3 * (i % 4)):
    spec = M.Spec(n=(17, 17, 17), dt=0.125)
    return [Request(i, spec, steps(i), gap * i) for i in range(n)]


def test_every_request_completes_with_its_own_steps(fakes):
    out = serve.Server(hbm_budget=1e9, chunk_steps=4, host_threads=4).run(reqs(20, 0.002))
    assert [r.id for r in out] == list(range(20))
    for r in out:
        assert r.steps == 5 + 3 * (r.id % 4)
        assert r.t == pytest.approx(r.steps * 0.125)
        assert r.done >= r.admitted >= r.arrival
    assert FakeSolver.live == 0


def test_budget_bounds_the_problems_on_the_device(fakes):
    srv = serve.Server(hbm_budget=350, chunk_steps=2, host_threads=4)
    out = srv.run(reqs(12, 0.0))
    assert len(out) == 12
    assert srv.peak_bytes <= 350
    assert FakeSolver.peak <= 3


def test_arrivals_join_the_running_batch(fakes):
    # long first requests; later arrivals are admitted while they run
    srv = serve.Server(hbm_budget=1e9, chunk_steps=1, host_threads=2)
    out = srv.run(reqs(6, 0.005, steps=lambda i: 400 if i == 0 else 3))
    assert srv.peak_active >= 2
    first = out[0]
    assert all(r.done < first.done for r in out[1:])


def test_request_over_budget_is_an_error(fakes):
    with pytest.raises(RuntimeError, match="over the budget"):
        serve.Server(hbm_budget=50, host_threads=1).run(reqs(1, 0.0))


def test_fifo_latencies():
    a = np.array([0.0, 0.5, 0.6, 5.0])
    s = np.array([1.0, 1.0, 1.0, 1.0])
    assert np.allclose(serve.fifo_latencies(a, s), [1.0, 1.5, 2.4, 1.0])


def test_active_cap_bounds_problems_in_flight(fakes):
    """max_active bounds the problems on the device at once; every request
    still completes."""
    srv = serve.Server(hbm_budget=1e9, chunk_steps=2, host_threads=4, max_active=3)
    out = srv.run(reqs(30, 0.0))
    assert [r.id for r in out] == list(range(30))
    assert 1 <= srv.peak_active <= 3
