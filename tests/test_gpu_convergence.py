"""The GPU path reproduces the reference's error and its observed convergence
under grid refinement on the config-0 problem: Douglas-ADI + MIB-L1, sphere
r = 0.49 on [-1, 1]^3, beta 1 inside / 10 outside, the e^{-t} exact solution
(eq 8), dt = h/2 to t = 1.

The reference as shipped does not converge at second order here: its L-inf
error stays at about 0.3 from 33^3 on (order ~0) and its L2 order falls from
1.6 to 0.3.  The table is the reference build's own output (17^3-129^3); the
GPU path is bit-identical to it, so each entry must agree to the digits the
table gives."""
import math

import pytest

import mts_b200 as M

pytestmark = pytest.mark.gpu

# (n, L-inf, L2) of the reference build, 3 and 3 significant digits
REFERENCE = [(17, 2.227e-1, 5.94e-2), (33, 2.978e-1, 1.94e-2), (65, 3.206e-1, 1.09e-2), (129, 3.197e-1, 8.88e-3)]


def run(n):
    spec = M.Spec(n=(n, n, n), surface="ellipsoid", surface_params=(1.0, 1.0, 1.0, 0.49), beta_in=1.0,
                  beta_out=10.0, method="adi", mib=1, dt=1.0 / (n - 1))
    with M.Solver(spec) as s:
        s.initialize()
        s.advance(n - 1)
        s.synchronize()
        assert s.time == pytest.approx(1.0, abs=1e-12)
        lmax, l2, _ = s.norms()
    return lmax, l2


def test_error_table_and_orders_under_refinement():
    got = [run(n) for n, _, _ in REFERENCE]
    for (n, lref, l2ref), (lmax, l2) in zip(REFERENCE, got):
        assert abs(lmax - lref) <= 0.5e-3 * lref, (n, lmax, lref)
        assert abs(l2 - l2ref) <= 0.5e-2 * l2ref, (n, l2, l2ref)
    # observed orders between successive grids (h halves)
    lo = [math.log2(got[k][0] / got[k + 1][0]) for k in range(3)]
    l2o = [math.log2(got[k][1] / got[k + 1][1]) for k in range(3)]
    assert all(abs(o) < 0.5 for o in lo[1:]), lo      # L-inf: no convergence from 33^3 on
    assert l2o[0] > 1.4 and 0.6 < l2o[1] < 1.0 and 0.1 < l2o[2] < 0.5, l2o
