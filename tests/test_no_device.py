"""No CPU fallback: every entry point that computes needs the CUDA device,
and without one it fails with MTS_ERR_NO_DEVICE instead of computing on
the host.  Runs where no device is visible (the CPU suite); on a GPU box it
hides the devices from a child process."""
import json
import math
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "matched-time-splitting-3d_b200")

CHILD = r"""
import sys
sys.path.insert(0, %r)
import mts_b200 as M
spec = M.Spec(n=(17, 17, 17), surface="ellipsoid", surface_params=(1.0, 1.0, 1.0, 0.49), beta_in=1.0,
              beta_out=10.0, method="adi", mib=2, dt=1.0 / 8)
out = {}
for name, call in [("setup_device", lambda: M.setup_device(spec)),
                   ("create_host_setup", lambda: M.Solver(spec)),
                   ("create_device_setup", lambda: M.Solver(M.Spec(**{**spec.__dict__, "setup": "device"})))]:
    try:
        call()
        out[name] = "computed"
    except M.MtsError as e:
        out[name] = e.status
# the host half alone needs no device
tags, cr, info = M.setup_host(spec)
out["setup_host"] = len(cr)
print(out)
""" % PKG


def test_compute_entry_points_refuse_without_a_device():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cp = subprocess.run([sys.executable, "-c", CHILD], capture_output=True, text=True, timeout=300, env=env)
    assert cp.returncode == 0, cp.stderr[-2000:]
    out = eval(cp.stdout.strip().splitlines()[-1])
    assert out["setup_device"] == 6  # MTS_ERR_NO_DEVICE
    assert out["create_host_setup"] == 6
    assert out["create_device_setup"] == 6
    assert out["setup_host"] > 0


def test_fp_error_fixtures_are_consistent():
    """tests/golden/fp_errors.json: each case's root mean square is
    sqrt(sum / count) of its own sum, and its text is Error_Fp's."""
    with open(os.path.join(ROOT, "tests", "golden", "fp_errors.json")) as f:
        cases = json.load(f)
    assert len(cases) >= 10
    for name, c in cases.items():
        lmax, l2, s, n = float(c["lmax"]), float(c["l2"]), float(c["sum"]), int(c["count"])
        assert n > 0 and n % 2 == 0, name
        want = math.sqrt(s / n)
        assert (math.isnan(l2) and math.isnan(want)) or l2 == want, name
        assert c["text"].startswith("------------------------ Error of FPs"), name
        if math.isfinite(lmax):
            assert f"Lmax = {lmax:.3e}" in c["text"], name
