"""Pins the oracle (oracle/mts_oracle.c, the C restatement of the time step)
to the reference: against the committed golden fixtures (produced by the
reference binary, tests/golden/make_golden.py) everywhere, and against fresh
reference runs where the reference build (oracle/_ref) is present."""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden, problem_from_dict

TOL = 1e-10  # relative max-norm; the restatement is expected to be bit-identical


def test_oracle_matches_golden_bitwise(golden):
    for name, entry in golden.items():
        prob = problem_from_dict(entry["problem"])
        u_ref, u0, tags, cr = load_golden(name)
        u = O.port_run(prob, tags, cr, u0)
        assert np.array_equal(u, u_ref), f"{name}: oracle differs from the reference (max {np.max(np.abs(u - u_ref))})"


def test_oracle_init_and_norms_match_reference(golden):
    for name, entry in golden.items():
        prob = problem_from_dict(entry["problem"])
        u_ref, u0, tags, cr = load_golden(name)
        assert np.array_equal(O.port_init(prob, tags), u0), name
        t = entry["info"]["t"]
        lmax, l2, am = O.port_norms(prob, tags, t, u_ref)
        assert lmax == entry["info"]["lmax"], name
        assert l2 == entry["info"]["l2"], name
        assert list(am) == entry["info"]["argmax"], name


def test_known_answer_eq0_exact(golden):
    """Eq_0 (80 inside, 100 outside, f = 0) is reproduced to round-off by every
    method: L-infinity below 1e-11 after 4 steps."""
    for name, entry in golden.items():
        if not name.startswith("eq0_"):
            continue
        assert entry["info"]["lmax"] < 1e-11, name


def test_config0_error_table():
    """ADI + MIB-L1 on the r=0.49 sphere, beta 1/10, dt = h/2, t = 1: the
    reference's as-shipped errors (L-infinity 2.978e-1, L2 1.944e-2 at 33^3)."""
    from conftest import golden_index

    info = golden_index()["config0_sphere33_adi_l1"]["info"]
    assert abs(info["lmax"] - 0.29780300359917933) < 1e-15
    assert abs(info["l2"] - 0.019439634319839867) < 1e-15


needs_ref = pytest.mark.skipif(not O.reference_available(noaux=True), reason="reference build (oracle/_ref) absent")


@needs_ref
@pytest.mark.parametrize("method", ["adi", "lod-ie", "lod-cn", "ts"])
@pytest.mark.parametrize("mib", [1, 2])
def test_oracle_matches_fresh_reference(method, mib):
    cases = [
        O.Problem(n=(19, 23, 17), surface_params=(0.55, 0.62, 0.45, 1.0, -0.03, 0.08, 0.02), beta_in=1.0,
                  beta_out=300.0, method=method, mib=mib, dt=1 / 12, steps=3),
        O.Problem(n=(33, 33, 33), surface="torus", surface_params=(0.5, 0.2), beta_in=2.0, beta_out=0.005,
                  method=method, mib=mib, dt=1 / 20, steps=2),
    ]
    for prob in cases:
        r = O.run_reference(prob, noaux=True)
        u = O.port_run(prob, r.tags, r.crossings, r.u0)
        assert np.array_equal(u, r.u)


@needs_ref
def test_aux_bypass_is_solution_neutral():
    """mts_ref_noaux (auxiliary eta/tau search compiled out) returns the
    unmodified reference's solution bit for bit where the latter runs."""
    for method in ("adi", "ts"):
        for mib in (1, 2):
            prob = O.Problem(n=(33, 33, 33), beta_out=10.0, method=method, mib=mib, dt=1 / 32, steps=3)
            a = O.run_reference(prob, noaux=False)
            b = O.run_reference(prob, noaux=True)
            assert np.array_equal(a.u, b.u)
            assert a.crossings.tobytes() == b.crossings.tobytes()


@needs_ref
@pytest.mark.parametrize("method", ["adi", "lod-ie", "lod-cn", "ts"])
def test_oracle_without_crossings_matches_reference(method):
    """A sphere between the grid nodes crosses no grid line: the oracle runs
    with an empty crossing list and returns the reference's solution."""
    prob = O.Problem(n=(17, 17, 17), surface_params=(1.0, 1.0, 1.0, 0.1, 0.0625, 0.0625, 0.0625), beta_in=1.0,
                     beta_out=10.0, method=method, mib=2, dt=0.125, steps=3)
    r = O.run_reference(prob, noaux=True)
    assert len(r.crossings) == 0
    u = O.port_run(prob, r.tags, r.crossings, r.u0)
    assert np.array_equal(u, r.u)
