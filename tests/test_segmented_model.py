"""The algebra of the mixed form's segmented line solve, checked on the CPU in
FP64 against a sequential Thomas solve (the GPU kernels themselves are
checked against the plain form in tests/test_mixed.py).

The kernel (csrc/mixed.cu, solve_line32) cuts a line of n rows into 32 lane
segments of MX rows, MX odd and 32 MX >= n, so the last lanes may be partly
or wholly past the line end.  Each lane runs the forward recurrence
d_j = ib_j r_j + p_j d_{j-1} from a zero carry while multiplying up P_j, an
inclusive scan composes the lanes' end maps c -> P c + d, and the carry into
lane l is the composition over lanes < l applied to 0; the backward
recurrence x_j = d_j + q_j x_{j+1} runs the same way with a suffix scan.
This restates those steps with numpy and checks them against Thomas."""
import numpy as np
import pytest


def thomas(a, b, c, r):
    """Sequential Thomas solve of rows a_j x_{j-1} + b_j x_j + c_j x_{j+1} = r_j."""
    n = len(b)
    gam = np.zeros(n)
    d = np.zeros(n)
    bet = b[0]
    d[0] = r[0] / bet
    for j in range(1, n):
        gam[j] = c[j - 1] / bet
        bet = b[j] - a[j] * gam[j]
        d[j] = (r[j] - a[j] * d[j - 1]) / bet
    x = d.copy()
    for j in range(n - 2, -1, -1):
        x[j] -= gam[j + 1] * x[j + 1]
    return x


def coefficients(a, b, c):
    """ib_j = 1/bet_j, p_j = -a_j/bet_j, q_j = -gam_{j+1} (0 on the last row)."""
    n = len(b)
    bet = np.zeros(n)
    gam = np.zeros(n)
    bet[0] = b[0]
    for j in range(1, n):
        gam[j] = c[j - 1] / bet[j - 1]
        bet[j] = b[j] - a[j] * gam[j]
    ib = 1.0 / bet
    p = -a / bet
    q = np.zeros(n)
    q[:-1] = -gam[1:]
    return ib, p, q


def segmented(ib, p, q, r, mx):
    """The lane-segment solve of one line, 32 lanes of mx rows."""
    n = len(r)
    lanes = 32
    d = np.zeros(lanes * mx)
    pm = np.ones(lanes * mx)
    A = np.ones(lanes)
    B = np.zeros(lanes)
    for l in range(lanes):
        dl, pl = 0.0, 1.0
        for k in range(mx):
            j = l * mx + k
            if j < n:
                dl = p[j] * dl + r[j] * ib[j]
                pl = pl * p[j]
                d[j], pm[j] = dl, pl
        A[l], B[l] = pl, dl
    # inclusive scan (Kogge-Stone, as the shuffles do it)
    off = 1
    while off < lanes:
        A2, B2 = A.copy(), B.copy()
        for l in range(off, lanes):
            B2[l] = A[l] * B[l - off] + B[l]
            A2[l] = A[l] * A[l - off]
        A, B = A2, B2
        off *= 2
    C = np.concatenate([[0.0], B[:-1]])
    xs = np.zeros(lanes * mx)
    for l in range(lanes):
        xl, ql = 0.0, 1.0
        for k in range(mx - 1, -1, -1):
            j = l * mx + k
            if j < n:
                xl = q[j] * xl + (pm[j] * C[l] + d[j])
                ql = ql * q[j]
                d[j], pm[j] = xl, ql
        A[l], B[l] = ql, xl
    off = 1
    while off < lanes:
        A2, B2 = A.copy(), B.copy()
        for l in range(lanes - off):
            B2[l] = A[l] * B[l + off] + B[l]
            A2[l] = A[l] * A[l + off]
        A, B = A2, B2
        off *= 2
    X = np.concatenate([B[1:], [0.0]])
    for l in range(lanes):
        for k in range(mx):
            j = l * mx + k
            if j < n:
                xs[j] = pm[j] * X[l] + d[j]
    return xs[:n]


def line_system(rng, n, kappa):
    """A line of the implicit operator: identity face rows, regular rows
    -kappa, 1 + 2 kappa, -kappa with a jump of the coefficient inside (two
    sides), and a few perturbed rows (the MIB blocks' rows)."""
    a = np.zeros(n)
    b = np.ones(n)
    c = np.zeros(n)
    split = int(rng.integers(n // 4, 3 * n // 4))
    for j in range(1, n - 1):
        k = kappa if j < split else kappa * 10.0
        a[j], b[j], c[j] = -k, 1.0 + 2.0 * k, -k
    for j in rng.choice(np.arange(2, n - 2), size=min(4, n - 4), replace=False):
        a[j] *= rng.uniform(0.5, 1.5)
        c[j] *= rng.uniform(0.5, 1.5)
    r = rng.standard_normal(n)
    return a, b, c, r


@pytest.mark.parametrize("n,mx", [(17, 3), (65, 3), (96, 3), (129, 5), (257, 9), (288, 9), (385, 13), (544, 17)])
@pytest.mark.parametrize("kappa", [0.5, 50.0, 5e4])
def test_segmented_solve_equals_thomas(n, mx, kappa):
    rng = np.random.default_rng(n * 7 + int(kappa))
    a, b, c, r = line_system(rng, n, kappa)
    ib, p, q = coefficients(a, b, c)
    x = segmented(ib, p, q, r, mx)
    ref = thomas(a, b, c, r)
    assert np.max(np.abs(x - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))
