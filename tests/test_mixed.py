"""The mixed-precision form of the Douglas-ADI step against the plain FP64
form (itself bit-identical to the reference).

The mixed form solves each step for its increment in FP32, with the residual
and the state in FP64, so it differs from the plain form by the FP32 rounding
of the increments.  Tolerances, written here:
  * relative max-norm difference from the plain solution <= 2e-5 after 8
    steps (a few ulp of FP32 per step on an O(dt) increment);
  * L-infinity error against the exact solution within 1.05x of the plain
    form's (the accuracy contract of the mixed form)."""
import numpy as np
import pytest

import mts_b200 as M
from conftest import rel_maxdiff

pytestmark = pytest.mark.gpu
REL_TOL = 2e-5
LINF_RATIO = 1.05


def run(spec, precision, steps):
    with M.Solver(spec) as s:
        s.set_precision(precision)
        assert s.precision == precision
        s.initialize()
        s.advance(steps)
        s.synchronize()
        return s.solution(), s.norms()


@pytest.mark.parametrize("surface,mib", [("torus", 2), ("torus", 1), ("ellipsoid", 2), ("ellipsoid", 1)])
def test_mixed_matches_plain(surface, mib):
    sp = (0.5, 0.2) if surface == "torus" else (0.7001, 0.4999, 0.4001, 1.0)
    spec = M.Spec(n=(65, 65, 65), surface=surface, surface_params=sp, beta_in=1.0, beta_out=1000.0, method="adi",
                  mib=mib, dt=2.0 / 64)
    u_p, (l_p, l2_p, _) = run(spec, "plain", 8)
    u_m, (l_m, l2_m, _) = run(spec, "mixed", 8)
    d = rel_maxdiff(u_m, u_p)
    assert d <= REL_TOL, f"relative max-norm difference {d:.3e}"
    assert l_m <= LINF_RATIO * l_p and l_p <= LINF_RATIO * l_m, (l_m, l_p)
    assert abs(l2_m - l2_p) <= 0.05 * l2_p


@pytest.mark.parametrize("beta_out", [1e-3, 1.0, 1e3])
def test_mixed_beta_ratios_anisotropic(beta_out):
    """The precision config's beta ratios, on an anisotropic grid with line
    lengths that are not multiples of the sweep chunk."""
    spec = M.Spec(n=(67, 61, 70), surface="torus", surface_params=(0.5, 0.2), beta_in=1.0, beta_out=beta_out,
                  method="adi", mib=2, dt=2.0 / 64)
    u_p, (l_p, _, _) = run(spec, "plain", 6)
    u_m, (l_m, _, _) = run(spec, "mixed", 6)
    assert rel_maxdiff(u_m, u_p) <= REL_TOL
    assert l_m <= LINF_RATIO * l_p


def test_mixed_long_lines_take_the_ring_sweeps():
    """Lines too long for the segmented tiles' shared memory (600 rows in x)
    take the ring sweeps, the others (17 rows) the tiles, in one step."""
    spec = M.Spec(n=(600, 17, 17), surface="ellipsoid", surface_params=(0.61, 0.52, 0.43, 1.0, 0.05, -0.03, 0.02),
                  beta_in=1.0, beta_out=10.0, method="adi", mib=2, dt=2.0 / 16)
    u_p, (l_p, _, _) = run(spec, "plain", 4)
    u_m, (l_m, _, _) = run(spec, "mixed", 4)
    assert rel_maxdiff(u_m, u_p) <= REL_TOL
    assert l_m <= LINF_RATIO * l_p


@pytest.mark.parametrize("n", [(17, 17, 17), (33, 65, 129), (257, 257, 257)])
def test_mixed_segment_edges(n):
    """Line lengths that leave the last segments short or empty (17 rows over
    8 segments of 3), mixed lengths per direction, and the bench grid."""
    spec = M.Spec(n=n, surface="torus", surface_params=(0.5, 0.2), beta_in=1.0, beta_out=1000.0, method="adi",
                  mib=2, dt=2.0 / (max(n) - 1))
    u_p, (l_p, _, _) = run(spec, "plain", 3)
    u_m, (l_m, _, _) = run(spec, "mixed", 3)
    assert rel_maxdiff(u_m, u_p) <= REL_TOL
    assert l_m <= LINF_RATIO * l_p


@pytest.mark.parametrize("n", [(400, 33, 35), (33, 520, 35), (35, 33, 300)])
def test_mixed_long_lines_within_the_segments(n):
    """Lines of 289-544 rows (13 and 17 rows per lane) in x, in y, and in z
    with the accumulation; dt = the finest spacing."""
    spec = M.Spec(n=n, surface="ellipsoid", surface_params=(0.61, 0.52, 0.43, 1.0, 0.05, -0.03, 0.02),
                  beta_in=1.0, beta_out=100.0, method="adi", mib=2, dt=2.0 / (max(n) - 1))
    u_p, (l_p, _, _) = run(spec, "plain", 4)
    u_m, (l_m, _, _) = run(spec, "mixed", 4)
    assert rel_maxdiff(u_m, u_p) <= REL_TOL
    assert l_m <= LINF_RATIO * l_p


def test_mixed_stiff_long_lines():
    """400-row x lines with dt set by the coarse axes (dt beta_out / h_x^2 =
    2.5e5): the forward multipliers sit within 1/sqrt(kappa) of 1, so FP32
    rounding accumulates along a line (as in any FP32 recurrence) to about
    n eps_32.  Tolerance 4 n eps_32 of the plain form, and the accuracy
    contract against the exact solution."""
    n = (400, 33, 35)
    spec = M.Spec(n=n, surface="ellipsoid", surface_params=(0.61, 0.52, 0.43, 1.0, 0.05, -0.03, 0.02),
                  beta_in=1.0, beta_out=100.0, method="adi", mib=2, dt=2.0 / (min(n) - 1))
    u_p, (l_p, _, _) = run(spec, "plain", 4)
    u_m, (l_m, _, _) = run(spec, "mixed", 4)
    assert rel_maxdiff(u_m, u_p) <= 4 * n[0] * 2.0 ** -24
    assert l_m <= LINF_RATIO * l_p and l_p <= LINF_RATIO * l_m


def test_mixed_rejects_other_methods():
    spec = M.Spec(n=(33, 33, 33), surface="torus", surface_params=(0.5, 0.2), beta_in=1.0, beta_out=10.0,
                  method="lod-cn", mib=2, dt=1.0 / 16)
    with M.Solver(spec) as s:
        with pytest.raises(M.MtsError, match="Douglas-ADI only"):
            s.set_precision("mixed")
        assert s.precision == "plain"
