"""The drop-in: the reference's own setup and time loop, with
mts::GpuStepper (include/mts_reference_adapter.hpp) constructed and called
where the loop constructs and calls Douglas_ADI, LOD or TS.

oracle/_ref/mts_dropin is the noaux reference build with the harness compiled
-DMTS_DROPIN and linked against libmts_b200.so; `--gpu` selects the adapter.
Its initial field, final field and error norms must equal the reference
stepper's bit for bit."""
import subprocess

import numpy as np
import pytest

import oracle as O

needs_dropin = pytest.mark.skipif(not O.reference_available(dropin=True),
                                  reason="drop-in build (oracle/_ref/mts_dropin) absent")

CASES = [
    # (id, Problem)
    ("ts_l2_ellipsoid_17", O.Problem(n=(17, 17, 17), surface="ellipsoid",
                                     surface_params=(0.61, 0.52, 0.43, 1.0, 0.05, -0.03, 0.02),
                                     beta_in=1.0, beta_out=1000.0, method="ts", mib=2, dt=0.125, steps=3)),
    ("adi_l1_torus_25", O.Problem(n=(25, 25, 25), surface="torus", surface_params=(0.5, 0.2), beta_in=1.0,
                                  beta_out=10.0, method="adi", mib=1, dt=2.0 / 24, steps=4)),
    ("lodcn_l2_sphere_33", O.Problem(n=(33, 33, 33), beta_in=1.0, beta_out=10.0, method="lod-cn", mib=2,
                                     dt=1.0 / 32, steps=4)),
    ("lodie_l1_eq0_anisotropic", O.Problem(n=(21, 19, 23), surface="ellipsoid",
                                           surface_params=(0.55, 0.6, 0.45, 1.0, -0.04, 0.03, 0.01), beta_in=1.0,
                                           beta_out=0.01, eq=0, method="lod-ie", mib=1, dt=0.1, steps=3)),
    # the reference's shipped configuration: ADI + MIB-L1, r = 0.49 sphere,
    # beta 1/10, dt = h/2, to t = 1
    ("config0_adi_l1_sphere_33", O.Problem(n=(33, 33, 33), beta_in=1.0, beta_out=10.0, method="adi", mib=1,
                                           dt=1.0 / 32, steps=32)),
]


@needs_dropin
def test_dropin_without_gpu_flag_is_the_reference():
    """Without --gpu the drop-in binary runs the reference stepper (the loop
    code is shared), bit for bit the noaux reference."""
    prob = CASES[0][1]
    a = O.run_reference(prob, noaux=True)
    b = O.run_reference(prob, binary=O.REF_BIN_DROPIN)
    assert np.array_equal(a.u0, b.u0) and np.array_equal(a.u, b.u)
    assert a.info["lmax"] == b.info["lmax"] and a.info["l2"] == b.info["l2"]


@needs_dropin
def test_dropin_fails_loudly_without_a_device():
    """--gpu never falls back to the CPU: with no CUDA device visible the
    adapter throws and the process exits non-zero without a result line."""
    cmd = [O.REF_BIN_DROPIN, *CASES[0][1].ref_args(), "--gpu"]
    cp = subprocess.run(cmd, capture_output=True, text=True, timeout=120, env={"CUDA_VISIBLE_DEVICES": ""})
    assert cp.returncode != 0
    assert not [ln for ln in cp.stdout.splitlines() if ln.startswith("{")]
    assert "mts:" in cp.stderr


@pytest.mark.gpu
@needs_dropin
@pytest.mark.parametrize("name,prob", CASES, ids=[c[0] for c in CASES])
def test_dropin_gpu_equals_reference_bitwise(name, prob, tmp_path):
    """Fields and norms bit for bit, and the stepper's Error() report (norms
    from the device) the same text as the reference stepper's."""
    ref = O.run_reference(prob, noaux=True, report=str(tmp_path / "ref.txt"))
    gpu = O.run_reference(prob, dropin_gpu=True, report=str(tmp_path / "gpu.txt"))
    assert np.array_equal(gpu.u0, ref.u0), name
    diff = np.max(np.abs(gpu.u - ref.u))
    assert np.array_equal(gpu.u, ref.u), f"{name}: max |gpu - reference| = {diff}"
    for k in ("t", "lmax", "l2", "argmax", "ncross"):
        assert gpu.info[k] == ref.info[k], (name, k, gpu.info[k], ref.info[k])
    ref_rep = (tmp_path / "ref.txt").read_text()
    assert ref_rep.startswith("[Xmax,Ymax,Zmax] = [")
    assert (tmp_path / "gpu.txt").read_text() == ref_rep


@pytest.mark.gpu
@needs_dropin
@pytest.mark.parametrize("mib", [1, 2])
def test_dropin_error_reports(mib, tmp_path):
    """The stepper's Error_Fp and Error_Jump (the device's Refresh_Fp +
    Error_Fp, Refresh_Jump's check + Error_Jump) write the same reports as
    the reference's Intersections::Error_Fp and Error_Jump in the same run."""
    prob = O.Problem(n=(26, 30, 28), surface="ellipsoid", surface_params=(0.61, 0.52, 0.43, 1.0, 0.05, -0.03, 0.02),
                     beta_in=1.0, beta_out=100.0, method="adi", mib=mib, dt=1.0 / 16, steps=3)
    f = tmp_path / "fp.txt"
    fj = tmp_path / "jump.txt"
    cp = subprocess.run([O.REF_BIN_DROPIN, *prob.ref_args(), "--gpu", "--fp-errors", str(f), "--jump-errors",
                         str(fj)], capture_output=True, text=True, timeout=300)
    assert cp.returncode == 0, cp.stderr
    for path, title in ((f, "Error of FPs"), (fj, "Error of Jumps")):
        ref_text = "\n".join(path.read_text().splitlines()[1:])
        gpu_text = (tmp_path / (path.name + ".gpu")).read_text()
        assert title in ref_text and "inf" not in ref_text and "nan" not in ref_text
        assert gpu_text.strip() == ref_text.strip()


@pytest.mark.gpu
@needs_dropin
@pytest.mark.parametrize("method", ["adi", "lod-ie", "ts"])
def test_dropin_write_txt_files_match(method, tmp_path):
    """The reference's own near-interface dump (Write_txt, helper.h:442-575:
    the closest outside node of every crossing, its value and its error)
    written from the drop-in's field is byte for byte the file written from
    the reference stepper's.  Write_txt knows the reference's Eq_0..Eq_7
    only, so the run uses Eq_0."""
    prob = O.Problem(n=(21, 19, 23), surface="ellipsoid", surface_params=(0.55, 0.6, 0.45, 1.0, -0.04, 0.03, 0.01),
                     beta_in=1.0, beta_out=0.01, eq=0, method=method, mib=2, dt=0.1, steps=3)
    out = {}
    for arm, extra in (("ref", []), ("gpu", ["--gpu"])):
        d = tmp_path / arm
        d.mkdir()
        cp = subprocess.run([O.REF_BIN_DROPIN, *prob.ref_args(), "--write-txt", *extra], capture_output=True,
                            text=True, timeout=300, cwd=str(d))
        assert cp.returncode == 0, cp.stderr
        out[arm] = [(d / f).read_bytes() for f in ("Numerical Solutions.txt", "Numerical Error.txt")]
    assert out["ref"][0].count(b"\n") > 100
    assert out["gpu"] == out["ref"]
