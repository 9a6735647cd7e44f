"""The product's host setup (mesh tags, crossings, MIB-L1/L2 weights) against
the reference's Mesh/Intersections: bit for bit, from the golden fixtures and
from fresh reference runs when the reference build is present.  No GPU."""
import numpy as np
import pytest

import mts_b200 as M
import oracle as O
from conftest import load_golden, problem_from_dict, spec_from_problem


def test_setup_matches_golden_bitwise(golden):
    for name, entry in golden.items():
        prob = problem_from_dict(entry["problem"])
        _, _, tags_ref, cr_ref = load_golden(name)
        tags, cr, _ = M.setup_host(spec_from_problem(prob))
        assert np.array_equal(tags, tags_ref), name
        assert len(cr) == len(cr_ref), name
        assert cr.tobytes() == cr_ref.tobytes(), name


needs_ref = pytest.mark.skipif(not O.reference_available(noaux=True), reason="reference build (oracle/_ref) absent")

SETUP_CASES = [
    # the measured geometries (substitutes for on-grid originals), beta 1:1000
    dict(n=(65, 65, 65), surface="ellipsoid", surface_params=(1.0, 1.0, 1.0, 0.49), mib=2),
    dict(n=(65, 65, 65), surface="ellipsoid", surface_params=(0.7001, 0.4999, 0.4001, 1.0), mib=1),
    dict(n=(65, 65, 65), surface="torus", surface_params=(0.5, 0.2), mib=2),
    # random-family ellipsoids with centres on anisotropic grids
    dict(n=(17, 49, 25), surface="ellipsoid", surface_params=(0.31, 0.68, 0.52, 1.0, 0.17, -0.12, 0.04), mib=2),
    dict(n=(49, 17, 33), surface="ellipsoid", surface_params=(0.66, 0.35, 0.41, 1.0, -0.19, 0.02, -0.15), mib=1),
]


@needs_ref
@pytest.mark.parametrize("case", SETUP_CASES)
def test_setup_matches_fresh_reference(case):
    prob = O.Problem(n=case["n"], surface=case["surface"], surface_params=tuple(case["surface_params"]),
                     beta_in=1.0, beta_out=1000.0, mib=case["mib"], dt=0.05, steps=0)
    r = O.run_reference(prob, noaux=True)
    tags, cr, counts = M.setup_host(spec_from_problem(prob))
    assert np.array_equal(tags, r.tags)
    assert cr.tobytes() == r.crossings.tobytes()
    assert counts["corner_pairs"] == int((r.crossings["id"] < 0).sum()) // 2


def test_setup_rejects_interface_on_grid():
    """r = 0.5 puts node (0.5, 0, 0) on the sphere: the reference aborts
    ("Interface on grid", src/mesh/mesh.cc:63-65); the setup returns
    MTS_ERR_SETUP."""
    spec = M.Spec(n=(33, 33, 33), surface_params=(1.0, 1.0, 1.0, 0.5))
    with pytest.raises(M.MtsError) as e:
        M.setup_host(spec)
    assert e.value.status == 2


@pytest.mark.parametrize("bad", [dict(mib=3), dict(eq=5), dict(method=7), dict(dt=-1.0), dict(n=(2, 33, 33)),
                                 dict(beta_out=0.0)])
def test_setup_rejects_bad_arguments(bad):
    kw = dict(n=(17, 17, 17))
    kw.update(bad)
    spec = M.Spec(**kw)
    with pytest.raises((M.MtsError, KeyError)):
        M.setup_host(spec)
