"""mts_norms_noalloc, the error norms that allocate nothing (their reduction
scratch is a static device array), against mts_norms through the C ABI.

The file name sorts last, so in a full run it executes after every other
test; it must pass both that way and alone.  Each case calls the entry point
twice in a row, which also checks that a call leaves the static scratch's
ticket counter ready for the next."""
import numpy as np
import pytest

import mts_b200 as M

pytestmark = pytest.mark.gpu


def spec(n, surface="torus", method="adi"):
    params = (0.5, 0.2) if surface == "torus" else (1.0, 1.0, 1.0, 0.3)
    return M.Spec(n=(n, n, n), surface=surface, surface_params=params, beta_in=1.0, beta_out=1000.0,
                  method=method, mib=2, dt=2.0 / (n - 1))


@pytest.mark.parametrize("surface,method", [("torus", "adi"), ("ellipsoid", "ts")])
def test_noalloc_matches_norms_on_two_calls_in_a_row(surface, method):
    import torch

    with M.Solver(spec(65, surface, method)) as s:
        s.initialize()
        s.advance(2)
        s.synchronize()
        for call in range(2):
            ref = s.norms()
            assert ref[0] > 0.0
            # the solver's own solution
            got = s.norms_noalloc()
            assert got == ref, (call, got, ref)
            # a caller-owned device field with the same values, at the same time
            u = torch.from_numpy(s.solution()).to("cuda")
            torch.cuda.synchronize()
            got_dev = s.norms_noalloc(u.data_ptr(), s.time)
            assert got_dev == ref, (call, got_dev, ref)
            # and a different field: a perturbation well above the current
            # error becomes the maximum, at its node
            delta = 10.0 * (1.0 + ref[0])
            v = u.clone()
            v[12345] += delta
            torch.cuda.synchronize()
            lmax, l2, am = s.norms_noalloc(v.data_ptr(), s.time)
            assert lmax >= delta - ref[0] and l2 > ref[1]
            ix, iy, iz = am
            assert ix + 65 * (iy + 65 * iz) == 12345
            s.advance(1)
            s.synchronize()


def test_noalloc_rejects_grids_beyond_its_scratch():
    # 163^3 = 4330747 nodes need 2115 reduction blocks, the scratch holds 2048
    with M.Solver(spec(163, "ellipsoid")) as s:
        s.initialize()
        ref = s.norms()
        with pytest.raises(RuntimeError, match="static scratch holds 2048"):
            s.norms_noalloc()
        assert s.norms() == ref


def test_noalloc_two_handles_in_turn():
    """Two handles on one device, each with its own stream, call the entry
    point one after the other (serialised, as the shared scratch requires);
    each result equals that handle's own mts_norms."""
    with M.Solver(spec(65, "torus", "adi")) as a, M.Solver(spec(49, "ellipsoid", "ts")) as b:
        assert a.stream() != b.stream()
        for s in (a, b):
            s.initialize()
            s.advance(2)
            s.synchronize()
        refs = {id(a): a.norms(), id(b): b.norms()}
        assert refs[id(a)] != refs[id(b)]
        for _ in range(3):
            for s in (a, b, b, a):
                assert s.norms_noalloc() == refs[id(s)]
        a.advance(1)
        b.advance(1)
        a.synchronize()
        b.synchronize()
        ra, rb = a.norms(), b.norms()
        assert a.norms_noalloc() == ra and b.norms_noalloc() == rb
