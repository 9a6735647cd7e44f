"""Generates tests/golden/fp_errors.json: the reference's fictitious-point
error report (Refresh_Fp then Error_Fp, src/spatial/intersection.cc:1841-2281,
4667-4771) and its jump error report (Refresh_Jump then Error_Jump,
:2294-2490, 4594-4662; under the key "jump") at the end of short runs, from
the reference's own code (oracle/_ref/mts_ref_noaux --fp-errors
--jump-errors, built by oracle/Makefile; the noaux build leaves Refresh_Fp,
the jump errors and the solution unchanged).  Needs the reference
tree; the GPU box only reads the committed JSON.

    make -C oracle REF=<reference checkout> && python tests/golden/make_fp_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402

SPHERE = (1.0, 1.0, 1.0, 0.49, 0.0, 0.0, 0.0)
ELLIPSOID = (0.7001, 0.4999, 0.4001, 1.0, 0.0, 0.0, 0.0)
TORUS = (0.5, 0.2)


def cases():
    out = []
    # even node counts: no node at x = 0 or z = 0, where the inside solution
    # of the measured problem vanishes and the relative errors divide by 0
    for mib in (1, 2):
        out.append((f"sphere32_l{mib}", O.Problem(n=(32, 32, 32), surface_params=SPHERE, beta_in=1.0, beta_out=10.0,
                                                  method="adi", mib=mib, dt=1 / 16, steps=3)))
        out.append((f"ellip32_l{mib}", O.Problem(n=(32, 32, 32), surface_params=ELLIPSOID, beta_in=1.0,
                                                 beta_out=1000.0, method="adi", mib=mib, dt=1 / 16, steps=2)))
        out.append((f"torus48_l{mib}", O.Problem(n=(48, 48, 48), surface="torus", surface_params=TORUS, beta_in=1.0,
                                                 beta_out=1000.0, method="ts", mib=mib, dt=1 / 24, steps=2)))
        out.append((f"ellip_aniso_l{mib}", O.Problem(n=(22, 26, 30), surface_params=(0.6, 0.5, 0.4, 1.0, 0.1, -0.05,
                                                                                      0.07),
                                                     beta_in=1.0, beta_out=0.01, method="lod-cn", mib=mib, dt=1 / 14,
                                                     steps=3)))
        # Eq_0: constant solutions, finite errors at every node
        out.append((f"eq0_sphere33_l{mib}", O.Problem(n=(33, 33, 33), surface_params=SPHERE, eq=0, beta_in=1.0,
                                                      beta_out=10.0, method="adi", mib=mib, dt=1 / 16, steps=2)))
    # odd node counts with the measured solution: the reference reports
    # Lmax = inf and L2 = nan
    out.append(("sphere33_l2_inf", O.Problem(n=(33, 33, 33), surface_params=SPHERE, beta_in=1.0, beta_out=10.0,
                                             method="adi", mib=2, dt=1 / 16, steps=2)))
    return out


def main():
    out = {}
    for name, prob in cases():
        with tempfile.TemporaryDirectory() as td:
            f = os.path.join(td, "fp.txt")
            fj = os.path.join(td, "jump.txt")
            cp = subprocess.run([O.REF_BIN_NOAUX, *prob.ref_args(), "--fp-errors", f, "--jump-errors", fj],
                                capture_output=True, text=True, timeout=600)
            if cp.returncode != 0:
                raise RuntimeError(cp.stderr[-400:])
            info = json.loads([ln for ln in cp.stdout.splitlines() if ln.startswith("{")][-1])
            lines = open(f).read().splitlines()
            jlines = open(fj).read().splitlines()
        lmax, l2, s, no = lines[0].split()
        jmax, jl2, js, jno = jlines[0].split()
        d = dict(prob.__dict__)
        d["n"] = list(prob.n)
        d["domain"] = list(prob.domain)
        d["surface_params"] = list(prob.surface_params)
        out[name] = {"problem": d, "t": info["t"], "lmax": lmax, "l2": l2, "sum": s, "count": int(no),
                     "text": "\n".join(lines[1:]),
                     "jump": {"lmax": jmax, "l2": jl2, "sum": js, "count": int(jno), "text": "\n".join(jlines[1:])}}
        print(name, lmax, l2, no, "jumps:", jmax, jl2, jno)
    with open(os.path.join(HERE, "fp_errors.json"), "w") as fo:
        json.dump(out, fo, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
