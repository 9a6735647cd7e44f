"""The error reports on the device against the reference's own values
(tests/golden/fp_errors.json, made by tests/golden/make_fp_golden.py from the
reference build):

- the fictitious points' report (mts_fp_errors: Refresh_Fp + Error_Fp,
  src/spatial/intersection.cc:1841-2281, 4667-4771);
- the jumps' report (mts_jump_errors: Refresh_Jump's jump.err + Error_Jump,
  :2294-2490, 4594-4662).

The per-crossing errors are computed with the reference's operations in its
order and added up in its loop order, so L-infinity and the root mean square
must be the reference's bits, inf and NaN included (odd grids put nodes at
x = 0 or z = 0, where the measured inside solution vanishes and the
reference divides by it; Eq_0's flux jumps are 0, and its jump errors 0/0).
The reports' text (4 digits) must match too.  A CPU restatement of the jump
check from the host setup's crossing records pins the golden jump values."""
import dataclasses
import json
import math
import os

import numpy as np
import pytest

import mts_b200 as M
from conftest import GOLDEN, problem_from_dict, spec_from_problem

with open(os.path.join(GOLDEN, "fp_errors.json")) as _f:
    CASES = json.load(_f)


def same(a, b):
    return (math.isnan(a) and math.isnan(b)) or a == b


def report_text(lmax, l2, title="FPs"):
    """Error_Fp's / Error_Jump's text: setprecision(3) scientific."""
    def fmt(v):
        return "nan" if math.isnan(v) else f"{v:.3e}"
    return (f"------------------------ Error of {title} ------------------------\n"
            f"Lmax = {fmt(lmax)}\nL2   = {fmt(l2)}")


def golden_text(text):
    return "\n".join(ln.replace("-nan", "nan") for ln in text.splitlines() if ln.strip())


@pytest.mark.gpu
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
    ref_text = golden_text(c["text"])
    assert report_text(lmax, l2) == ref_text, (report_text(lmax, l2), ref_text)


@pytest.mark.gpu
@pytest.mark.parametrize("setup", ["host", "device"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_jump_errors_match_reference(name, setup):
    c = CASES[name]
    prob = problem_from_dict(c["problem"])
    spec = dataclasses.replace(spec_from_problem(prob), setup=setup)
    with M.Solver(spec) as s:
        s.initialize()
        s.advance(prob.steps)
        s.synchronize()
        assert s.time == c["t"]
        lmax, l2 = s.jump_errors()
        # the fictitious-point report in between shares the tables and the
        # error buffer: the jump report stays the same
        s.fp_errors()
        again = s.jump_errors()
    want = float(c["jump"]["lmax"]), float(c["jump"]["l2"])
    assert same(lmax, want[0]) and same(l2, want[1]), (name, lmax, l2, want)
    assert same(again[0], lmax) and same(again[1], l2)
    ref_text = golden_text(c["jump"]["text"])
    assert report_text(lmax, l2, "Jumps") == ref_text, (report_text(lmax, l2, "Jumps"), ref_text)


def jump_report_restated(c):
    """Refresh_Jump's jump.err (intersection.cc:2294-2490) and Error_Jump's
    sums (:4594-4662) restated from the host setup's crossing records:
    u_dir = (P^-1)[d][0] [beta u_xi] against [beta u_d] of the exact
    solution (inside sin 2x cos 2y sin 2z e^-t, outside (x^2+y^2+z^2) e^-t;
    Eq_0: flux jumps 0).  numpy's inverse stands in for the reference's LU,
    so the values agree to rounding, not bit for bit."""
    prob = problem_from_dict(c["problem"])
    _, cr, _ = M.setup_host(spec_from_problem(prob))
    E = math.exp(-c["t"])
    bi, bo = prob.beta_in, prob.beta_out
    order = sorted(range(len(cr)), key=lambda i: (-int(cr["dir"][i]), int(cr["indx1"][i]), int(cr["indx2"][i]),
                                                  int(cr["left_loc"][i])))
    jmax, total = 0.0, 0.0
    for i in order:
        x, y, z = (float(v) for v in cr["coord"][i])
        d = int(cr["dir"][i])
        if prob.eq == 0:
            jb = [0.0, 0.0, 0.0]
        else:
            D = [2 * math.cos(2 * x) * math.cos(2 * y) * math.sin(2 * z),
                 -2 * math.sin(2 * x) * math.sin(2 * y) * math.sin(2 * z),
                 2 * math.sin(2 * x) * math.cos(2 * y) * math.cos(2 * z)]
            jb = [bo * (2 * v * E) - bi * (D[k] * E) for k, v in enumerate((x, y, z))]
        p = np.asarray(cr["p"][i], dtype=np.float64).reshape(3, 3)
        bxi = float(p[0] @ np.asarray(jb))
        udir = float(np.linalg.inv(p)[d][0]) * bxi
        with np.errstate(invalid="ignore", divide="ignore"):
            e = float(np.float64(abs(udir - jb[d])) / np.float64(jb[d]))
        total += e * e
        if abs(e) > jmax:
            jmax = abs(e)
    return jmax, math.sqrt(total / len(order)), len(order)


@pytest.mark.parametrize("name", sorted(CASES))
def test_jump_report_restatement_pins_golden(name):
    c = CASES[name]
    jmax, l2, count = jump_report_restated(c)
    g = c["jump"]
    assert count == g["count"]
    for got, want in ((jmax, float(g["lmax"])), (l2, float(g["l2"]))):
        if math.isnan(want):
            assert math.isnan(got)
        else:
            assert got == pytest.approx(want, rel=1e-9, abs=0.0), (name, got, want)
