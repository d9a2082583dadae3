"""Tile-size autotuner (starsh_b200_autotune_tile): it picks one of the
candidates from measured marginal costs, reports a finite cost for every
candidate not above N and infinity for the others, caches its choice per
problem class, and the chosen tile size compresses the problem within tol
(checked with the reference's own dfe)."""
import ctypes
import math
from ctypes import POINTER, byref, c_double, c_int

import pytest

import oracle
import starsh_b200 as sb
from harness import RefProblem, approximate_b200, as_ref_blrm


@pytest.mark.gpu
def test_autotune_picks_and_caches(ref, lib):
    lib.starsh_b200_autotune_clear()
    n, tol = 3600, 1e-5
    pr = RefProblem(ref, "spatial", n, 400, kernel_name="exp", beta=0.1)
    P = ctypes.cast(pr.P, POINTER(sb.Problem))
    cands = (c_int * 4)(256, 512, 1024, 4096)
    ranks = (c_int * 4)(128, 200, 256, 256)
    best = c_int(0)
    costs = (c_double * 4)()
    lib.starsh_set_oversample(b"10")
    assert lib.starsh_b200_autotune_tile(P, 4, cands, ranks, tol,
                                         sb.ENGINE_MIXED, byref(best),
                                         costs) == 0, lib.starsh_b200_last_error()
    assert best.value in (256, 512, 1024)
    assert all(math.isfinite(costs[c]) and costs[c] > 0 for c in range(3))
    assert math.isinf(costs[3])                    # 4096 > N
    assert costs[[256, 512, 1024].index(best.value)] == min(costs[:3])
    # a second problem of the same class reuses the measurement
    pr2 = RefProblem(ref, "spatial", n, 400, kernel_name="exp", beta=0.1, seed=3)
    best2 = c_int(0)
    costs2 = (c_double * 4)()
    assert lib.starsh_b200_autotune_tile(ctypes.cast(pr2.P, POINTER(sb.Problem)),
                                         4, cands, ranks, tol, sb.ENGINE_MIXED,
                                         byref(best2), costs2) == 0
    assert best2.value == best.value and list(costs2) == list(costs)
    # the chosen tile size, through the drop-in path, is within tol
    pb = RefProblem(ref, "spatial", n, best.value, kernel_name="exp", beta=0.1)
    M = approximate_b200(lib, pb.b200_format(),
                         ranks[[256, 512, 1024].index(best.value)], tol,
                         engine=sb.ENGINE_MIXED)
    assert ref.dfe(as_ref_blrm(M)) <= tol
    lib.starsh_blrm_free(M)
    lib.starsh_b200_autotune_clear()


def test_autotune_rejects_bad_arguments(lib):
    best = c_int(0)
    cands = (c_int * 1)(256)
    ranks = (c_int * 1)(64)
    assert lib.starsh_b200_autotune_tile(None, 1, cands, ranks, 1e-5, 1,
                                         byref(best), None) == sb.WRONG_PARAMETER
