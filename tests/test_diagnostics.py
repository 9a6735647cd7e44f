"""The fictitious points' error report on the device (mts_fp_errors:
Refresh_Fp + Error_Fp, src/spatial/intersection.cc:1841-2281, 4667-4771)
against the reference's own values (tests/golden/fp_errors.json, made by
tests/golden/make_fp_golden.py from the reference build).

The per-crossing errors are computed with the reference's operations in its
order and added up in its loop order, so L-infinity and the root mean square
must be the reference's bits, inf and NaN included (odd grids put nodes at
x = 0 or z = 0, where the measured inside solution vanishes and the
reference divides by it).  The text of Error_Fp (4 digits) must match too."""
import dataclasses
import json
import math
import os

import pytest

import mts_b200 as M
from conftest import GOLDEN, problem_from_dict, spec_from_problem

pytestmark = pytest.mark.gpu

with open(os.path.join(GOLDEN, "fp_errors.json")) as _f:
    CASES = json.load(_f)


def same(a, b):
    return (math.isnan(a) and math.isnan(b)) or a == b


def report_text(lmax, l2):
    """Error_Fp's text: setprecision(3) scientific."""
    def fmt(v):
        return "nan" if math.isnan(v) else f"{v:.3e}"
    return (f"------------------------ Error of FPs ------------------------\n"
            f"Lmax = {fmt(lmax)}\nL2   = {fmt(l2)}")


@pytest.mark.parametrize("setup", ["host", "device"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_fp_errors_match_reference(name, setup):
    c = CASES[name]
    prob = problem_from_dict(c["problem"])
    spec = dataclasses.replace(spec_from_problem(prob), setup=setup)
    with M.Solver(spec) as s:
        s.initialize()
        s.advance(prob.steps)
        s.synchronize()
        assert s.time == c["t"]
        lmax, l2 = s.fp_errors()
        # the report does not depend on the solution: again after more steps
        # and back at the same time gives the same bits
        s.advance(1)
        s.time = c["t"]
        again = s.fp_errors()
    want = float(c["lmax"]), float(c["l2"])
    assert same(lmax, want[0]) and same(l2, want[1]), (name, lmax, l2, want)
    assert same(again[0], lmax) and same(again[1], l2)
    ref_text = "\n".join(ln.replace("-nan", "nan") for ln in c["text"].splitlines() if ln.strip())
    assert report_text(lmax, l2) == ref_text, (report_text(lmax, l2), ref_text)
