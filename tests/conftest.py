import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "matched-time-splitting-3d_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running case")


def golden_index():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def load_golden(name):
    import oracle as O

    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cr = z["crossings"].view(O.CROSSING_DTYPE)
    return z["u"], z["u0"], z["tags"], cr


def problem_from_dict(d):
    import oracle as O

    d = dict(d)
    d["n"] = tuple(d["n"])
    d["domain"] = tuple(d["domain"])
    d["surface_params"] = tuple(d["surface_params"])
    return O.Problem(**d)


def spec_from_problem(p):
    import mts_b200 as M

    return M.Spec(n=p.n, domain=p.domain, surface=p.surface, surface_params=p.surface_params, beta_in=p.beta_in,
                  beta_out=p.beta_out, eq=p.eq, method=p.method, mib=p.mib, dt=p.dt, t0=p.t0)


def rel_maxdiff(a, b):
    """max |a-b| / max |b| (the parity norm: relative max-norm)."""
    scale = float(np.max(np.abs(b))) or 1.0
    return float(np.max(np.abs(a - b))) / scale


@pytest.fixture(scope="session")
def golden():
    return golden_index()
