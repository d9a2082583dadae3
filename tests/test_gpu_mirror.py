"""Host mirrors downloaded batch by batch (page-locked blocks filled on a
copy stream while later batches compute) hold exactly the device factors:
the same problem approximated with the mirror flag, and without it and
downloaded afterwards, gives bit-identical U, V and dense blocks, for one
problem split over several batches and for a batched call of several
problems; freeing the matrices returns the blocks to the pool and a second
round of calls reuses them."""
import ctypes
from ctypes import POINTER, byref

import numpy as np
import pytest

import oracle
import starsh_b200 as sb
from harness import RefProblem, approximate_b200, as_ref_blrm

CASES = [
    dict(kind="spatial", n=4096, nb=512, kernel_name="sqexp", maxrank=120,
         tol=1e-7),
    dict(kind="coulomb", n=2048, nb=256, ndim=3, place=1, maxrank=120,
         tol=1e-6),
]


def _problem(ref, case):
    kw = {k: v for k, v in case.items()
          if k not in ("kind", "n", "nb", "maxrank", "tol")}
    return RefProblem(ref, case["kind"], case["n"], case["nb"], **kw)


def _same(M1, M2):
    c1 = oracle.blrm_contents(as_ref_blrm(M1))
    c2 = oracle.blrm_contents(as_ref_blrm(M2))
    np.testing.assert_array_equal(c1["ranks"], c2["ranks"])
    assert len(c1["U"]) == len(c2["U"]) and len(c1["D"]) == len(c2["D"])
    for a, b in zip(c1["U"], c2["U"]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(c1["V"], c2["V"]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(c1["D"], c2["D"]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("engine", [sb.ENGINE_FP64, sb.ENGINE_MIXED])
def test_mirror_during_batches_equals_download(ref, lib, engine, monkeypatch):
    # a small workspace splits each problem over several batches
    monkeypatch.setenv("STARSH_B200_WORKSPACE_MB", "64")
    for _ in range(2):                      # the second round reuses blocks
        for case in CASES:
            pr = _problem(ref, case)
            M1 = approximate_b200(lib, pr.b200_format(), case["maxrank"],
                                  case["tol"], engine=engine, flags=1)
            if case["kind"] == "spatial":
                assert sb.stats(lib).batches > 1
            pr2 = _problem(ref, case)
            M2 = approximate_b200(lib, pr2.b200_format(), case["maxrank"],
                                  case["tol"], engine=engine, flags=0)
            assert lib.starsh_b200_blrm_download(M2) == 0
            _same(M1, M2)
            assert ref.dfe(as_ref_blrm(M1)) <= case["tol"]
            lib.starsh_blrm_free(M1)
            lib.starsh_blrm_free(M2)


@pytest.mark.gpu
def test_batched_call_mirrors_each_problem(ref, lib):
    lib.starsh_set_oversample(b"10")
    probs = [_problem(ref, c) for c in CASES]
    n = len(CASES)
    Fs = (POINTER(sb.Blrf) * n)(*[p.b200_format() for p in probs])
    Ms = (POINTER(sb.Blrm) * n)()
    ranks = (ctypes.c_int * n)(*[c["maxrank"] for c in CASES])
    tols = (ctypes.c_double * n)(*[c["tol"] for c in CASES])
    assert lib.starsh_b200_approximate_batch(n, Ms, Fs, ranks, tols, None,
                                             sb.ENGINE_MIXED, 1) == 0
    for i, case in enumerate(CASES):
        pr = _problem(ref, case)
        M = approximate_b200(lib, pr.b200_format(), case["maxrank"],
                             case["tol"], engine=sb.ENGINE_MIXED, flags=0)
        assert lib.starsh_b200_blrm_download(M) == 0
        _same(Ms[i], M)
        lib.starsh_blrm_free(M)
        lib.starsh_blrm_free(Ms[i])
