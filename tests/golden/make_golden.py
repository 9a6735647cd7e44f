"""Generates the golden fixtures in tests/golden/ by running the reference's
own time-stepping code (oracle/_ref/mts_ref, built from the reference sources
by oracle/Makefile).  Needs the reference tree; the GPU box only reads the
committed .npz files.

    make -C oracle REF=<reference checkout> && python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402

SPHERE = (1.0, 1.0, 1.0, 0.49, 0.0, 0.0, 0.0)
ELLIPSOID = (0.7001, 0.4999, 0.4001, 1.0, 0.0, 0.0, 0.0)
TORUS = (0.5, 0.2)


def cases():
    out = []
    # every method x MIB variant, 17^3 sphere (no corners) and 25^3 shifted
    # anisotropic ellipsoid on an anisotropic grid (corner pairs present)
    for method in ("adi", "lod-ie", "lod-cn", "ts"):
        for mib in (1, 2):
            out.append((f"sphere17_{method}_l{mib}",
                        O.Problem(n=(17, 17, 17), surface_params=SPHERE, beta_in=1.0, beta_out=10.0, method=method,
                                  mib=mib, dt=1 / 16, steps=4), False))
            out.append((f"ellip_aniso_{method}_l{mib}",
                        O.Problem(n=(21, 25, 29), surface_params=(0.6, 0.5, 0.4, 1.0, 0.1, -0.05, 0.07), beta_in=1.0,
                                  beta_out=0.01, method=method, mib=mib, dt=1 / 14, steps=3), True))
    # the measured problem family at 33^3: beta 1:1000, torus and ellipsoid
    out.append(("torus33_adi_l2", O.Problem(n=(33, 33, 33), surface="torus", surface_params=TORUS, beta_in=1.0,
                                            beta_out=1000.0, method="adi", mib=2, dt=1 / 16, steps=4), True))
    out.append(("ellip33_ts_l2", O.Problem(n=(33, 33, 33), surface_params=ELLIPSOID, beta_in=1.0, beta_out=1000.0,
                                           method="ts", mib=2, dt=1 / 16, steps=3), True))
    out.append(("sphere33_lodcn_l1", O.Problem(n=(33, 33, 33), surface_params=SPHERE, beta_in=1.0, beta_out=1000.0,
                                               method="lod-cn", mib=1, dt=1 / 16, steps=3), False))
    # config-0 of the measured problem: ADI + MIB-L1, dt = h/2, t in [0, 1]
    out.append(("config0_sphere33_adi_l1", O.Problem(n=(33, 33, 33), surface_params=SPHERE, beta_in=1.0,
                                                     beta_out=10.0, method="adi", mib=1, dt=1 / 32, steps=32), False))
    # known answer: Eq_0 (80 inside, 100 outside) stays exact
    for method in ("adi", "lod-ie", "lod-cn", "ts"):
        out.append((f"eq0_{method}_l2", O.Problem(n=(17, 17, 17), surface_params=SPHERE, eq=0, beta_in=1.0,
                                                  beta_out=10.0, method=method, mib=2, dt=1 / 16, steps=4), False))
    return out


def main():
    index = {}
    for name, prob, noaux in cases():
        r = O.run_reference(prob, noaux=noaux)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), u=r.u, u0=r.u0, tags=r.tags,
                            crossings=r.crossings.view(np.uint8))
        d = dict(prob.__dict__)
        d["n"] = list(prob.n)
        d["domain"] = list(prob.domain)
        d["surface_params"] = list(prob.surface_params)
        index[name] = {"problem": d, "reference_binary": "mts_ref_noaux" if noaux else "mts_ref", "info": r.info}
        print(name, r.info["lmax"], r.info["ncross"])
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
