"""The host setup of large grids runs over threads (ranges of lines, planes
of tags) and joins the results in line order: the output must equal one
thread's byte for byte, and a geometry the reference rejects must fail with
the same status either way.  MTS_SETUP_THREADS sets the thread count."""
import numpy as np
import pytest

import mts_b200 as M


def setup(spec, threads, monkeypatch):
    monkeypatch.setenv("MTS_SETUP_THREADS", str(threads))
    return M.setup_host(spec)


@pytest.mark.parametrize("surface,params,mib", [
    ("torus", (0.5, 0.2), 2),
    ("ellipsoid", (0.61, 0.52, 0.43, 1.0, 0.05, -0.03, 0.02), 1),
])
def test_threaded_setup_equals_one_thread(surface, params, mib, monkeypatch):
    spec = M.Spec(n=(71, 53, 97), surface=surface, surface_params=params, beta_in=1.0, beta_out=1000.0,
                  method="adi", mib=mib, dt=0.02)
    t1, c1, r1 = setup(spec, 1, monkeypatch)
    for threads in (3, 8):
        tn, cn, rn = setup(spec, threads, monkeypatch)
        assert np.array_equal(t1, tn)
        assert c1.tobytes() == cn.tobytes()
        assert r1 == rn
    assert len(c1) > 0


def test_threaded_setup_rejects_as_one_thread(monkeypatch):
    # a sphere of radius 0.5 on [-1, 1] with 33 nodes puts the interface on
    # grid nodes: the reference's "Interface on grid" rejection
    spec = M.Spec(n=(33, 33, 33), surface="ellipsoid", surface_params=(1.0, 1.0, 1.0, 0.5), beta_in=1.0,
                  beta_out=10.0, method="adi", mib=1, dt=1.0 / 16)
    errs = []
    for threads in (1, 4):
        with pytest.raises(M.MtsError) as e:
            setup(spec, threads, monkeypatch)
        errs.append(e.value.status)
    assert errs[0] == errs[1]
