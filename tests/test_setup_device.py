"""The device setup (mts_setup_device, and mts_create with setup = device)
against the host setup that is pinned to the reference
(tests/test_setup_parity.py).

The tags must be identical.  The crossing records must agree in every
integer field and, field by field, within 1e-12 relative (plus 1e-12
absolute): the device squares with v * v where the reference calls glibc's
pow(v, 2), which is not always the correctly rounded square, so a root,
normal or weight can differ in its last bits; most records are
bit-identical, and the test reports how many.  Failing geometries must fail
with the host's status.  A problem stepped from a device setup must match
the oracle (host setup) to the 1e-10 relative max-norm of the contract."""
import numpy as np
import pytest

import mts_b200 as M
import oracle as O
from conftest import golden_index, problem_from_dict, rel_maxdiff, spec_from_problem

pytestmark = pytest.mark.gpu
FLOAT_FIELDS = ["coord", "gamma", "normal", "p", "weil", "weir"]
INT_FIELDS = ["dir", "indx1", "indx2", "id", "left_loc", "nwei"]


def compare(spec):
    """Returns (records, bit-identical records) or raises on a mismatch."""
    try:
        th, ch, ih = M.setup_host(spec)
    except M.MtsError as e:
        with pytest.raises(M.MtsError) as ed:
            M.setup_device(spec)
        assert ed.value.status == e.status, (spec, e, ed.value)
        return 0, 0
    td, cd, idv = M.setup_device(spec)
    assert np.array_equal(td, th)
    assert len(cd) == len(ch), (len(cd), len(ch))
    assert idv == ih
    for f in INT_FIELDS:
        assert np.array_equal(cd[f], ch[f]), f
    same = np.ones(len(ch), dtype=bool)
    for f in FLOAT_FIELDS:
        a, b = cd[f].reshape(len(ch), -1), ch[f].reshape(len(ch), -1)
        assert np.all(np.abs(a - b) <= 1e-12 * np.maximum(1.0, np.abs(b))), (f, float(np.abs(a - b).max()))
        same &= np.all(a.view(np.int64) == b.view(np.int64), axis=1)
    return len(ch), int(same.sum())


def test_device_setup_matches_host_on_golden_problems():
    total = ident = 0
    for name, entry in golden_index().items():
        prob = problem_from_dict(entry["problem"])
        n, s = compare(spec_from_problem(prob))
        total += n
        ident += s
    print(f"golden problems: {ident}/{total} crossing records bit-identical")
    assert total > 0


FAMILY = []
_rng = np.random.default_rng(11)
for _i in range(40):
    _n = tuple(int(v) for v in _rng.choice([17, 25, 33, 49, 65], size=3))
    _ax = tuple(float(v) for v in _rng.uniform(0.3, 0.7, size=3))
    _c = tuple(float(v) for v in _rng.uniform(-0.2, 0.2, size=3))
    FAMILY.append(dict(n=_n, surface_params=(*_ax, 1.0, *_c), beta_out=float(10 ** _rng.uniform(-3, 3)),
                       mib=1 + _i % 2))


def test_device_setup_matches_host_on_a_random_family():
    """40 anisotropic problems of the batched family, L1 and L2; those the
    reference's rules reject must be rejected with the same status."""
    total = ident = rejected = 0
    for c in FAMILY:
        spec = M.Spec(n=c["n"], surface_params=c["surface_params"], beta_in=1.0, beta_out=c["beta_out"], method="adi",
                      mib=c["mib"], dt=2.0 / (min(c["n"]) - 1))
        n, s = compare(spec)
        rejected += n == 0
        total += n
        ident += s
    print(f"random family: {ident}/{total} records bit-identical, {rejected} problems rejected by both")
    assert total > 0


@pytest.mark.parametrize("mib", [1, 2])
@pytest.mark.parametrize("surface,params", [("torus", (0.5, 0.2)), ("ellipsoid", (1.0, 1.0, 1.0, 0.49)),
                                            ("ellipsoid", (0.7001, 0.4999, 0.4001, 1.0))],
                         ids=["torus", "sphere", "ellipsoid"])
def test_device_setup_matches_host_at_257(surface, params, mib):
    spec = M.Spec(n=(257, 257, 257), surface=surface, surface_params=params, beta_in=1.0, beta_out=1000.0,
                  method="adi", mib=mib, dt=2.0 / 256)
    n, s = compare(spec)
    print(f"257^3 {surface} L{mib}: {s}/{n} records bit-identical")
    assert n > 0


def test_device_setup_rejects_a_node_on_the_interface():
    # r = 0.5 on [-1, 1]^3 at 33^3: node (0.5, 0, 0) lies on the sphere
    spec = M.Spec(n=(33, 33, 33), surface="ellipsoid", surface_params=(1.0, 1.0, 1.0, 0.5), beta_in=1.0,
                  beta_out=10.0, method="adi", mib=2, dt=1.0 / 16)
    with pytest.raises(M.MtsError) as eh:
        M.setup_host(spec)
    with pytest.raises(M.MtsError) as ed:
        M.setup_device(spec)
    assert ed.value.status == eh.value.status == 2


@pytest.mark.parametrize("method", ["adi", "ts"])
@pytest.mark.parametrize("mib", [1, 2])
def test_solver_on_device_setup_matches_oracle(method, mib):
    """65^3 torus (corner pairs) to t = 1 from a device setup, against the
    oracle run on the host setup."""
    kw = dict(n=(65, 65, 65), surface="torus", surface_params=(0.5, 0.2), beta_in=1.0, beta_out=1000.0,
              method=method, mib=mib, dt=2.0 / 64)
    spec = M.Spec(**kw, setup="device")
    tags, cr, _ = M.setup_host(M.Spec(**kw))
    prob = O.Problem(**kw, steps=32)
    u_or = O.port_run(prob, tags, cr, O.port_init(prob, tags))
    with M.Solver(spec) as s:
        s.initialize()
        s.advance(32)
        s.synchronize()
        u = s.solution()
    assert rel_maxdiff(u, u_or) <= 1e-10
