"""The drop-in stepper (include/mts_reference_adapter.hpp) refuses plugins the
device does not evaluate, before any device work: a variable-coefficient
Beta (the reference's Beta_1, src/diffusion/beta_1.cc) at construction, and
an Equation other than the one it was built for (the reference's Eq_3,
src/equation/eq_3.cc) at Initialization and at every Solve_2nd.  Run through
the reference's own time loop (oracle/_ref/mts_dropin --gpu), on the CPU:
with supported plugins the run gets past the checks and, without a GPU,
stops at the device with the library's "no CUDA device" error."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "mts_dropin")
ARGS = ["--n", "17", "17", "17", "--surface", "ellipsoid", "1", "1", "1", "0.49", "--beta", "1", "10", "--mib", "1",
        "--dt", "0.0625", "--steps", "2", "--gpu"]

pytestmark = pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in demonstration not built (needs the "
                                                                   "reference checkout)")


def run(*extra):
    cp = subprocess.run([DROPIN, *ARGS, *extra], capture_output=True, text=True, timeout=120)
    return cp.returncode, cp.stderr


@pytest.mark.parametrize("method", ["adi", "lod-ie", "ts"])
def test_variable_beta_is_refused(method):
    rc, err = run("--beta-plugin", "1", "--eq", "8", "--method", method)
    assert rc == 3
    assert "beta must be piecewise constant" in err


@pytest.mark.parametrize("method", ["adi", "lod-cn", "ts"])
def test_other_equation_is_refused(method):
    rc, err = run("--eq", "3", "--method", method)
    assert rc == 3
    assert "Equation is not the exact solution" in err


@pytest.mark.parametrize("eq,method", [("8", "adi"), ("0", "lod-cn"), ("8", "ts")])
def test_supported_plugins_pass_the_checks(eq, method):
    rc, err = run("--eq", eq, "--method", method)
    assert rc == 0 or "no CUDA device" in err, err
    assert "Equation is not" not in err and "piecewise constant" not in err
