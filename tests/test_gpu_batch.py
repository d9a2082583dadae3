"""Multi-problem batches and the serving loop: a problem's result is the same
alone and inside a batch of other problems (different kernels, tile sizes,
maxrank and tol), bit for bit; the server admits requests by its HBM budget
and groups requests that wait together."""
import ctypes
from ctypes import POINTER, byref, c_double, c_int, c_longlong, c_void_p

import numpy as np
import pytest

import oracle
import starsh_b200 as sb
from harness import RefProblem, approximate_b200, as_ref_blrm

CASES = [
    dict(kind="spatial", n=2048, nb=512, kernel_name="exp", maxrank=100,
         tol=1e-5),
    dict(kind="coulomb", n=2048, nb=256, ndim=3, place=1, maxrank=120,
         tol=1e-6),
    # ragged clusters (1500 = 3 x 400 + 300)
    dict(kind="sin", n=1500, nb=400, ndim=3, place=1, maxrank=150, tol=1e-4),
    dict(kind="spatial", n=3000, nb=1000, kernel_name="sqexp", maxrank=200,
         tol=1e-7),
]


def _problem(ref, case):
    kw = {k: v for k, v in case.items()
          if k not in ("kind", "n", "nb", "maxrank", "tol")}
    return RefProblem(ref, case["kind"], case["n"], case["nb"], **kw)


def _near_set(M):
    F = as_ref_blrm(M).contents.format.contents
    return sorted((F.block_near[2 * b], F.block_near[2 * b + 1])
                  for b in range(F.nblocks_near))


def _assert_same(M1, M2):
    c1 = oracle.blrm_contents(as_ref_blrm(M1))
    c2 = oracle.blrm_contents(as_ref_blrm(M2))
    np.testing.assert_array_equal(c1["ranks"], c2["ranks"])
    for a, b in zip(c1["U"], c2["U"]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(c1["V"], c2["V"]):
        np.testing.assert_array_equal(a, b)
    assert _near_set(M1) == _near_set(M2)


@pytest.mark.gpu
@pytest.mark.parametrize("engine", [sb.ENGINE_FP64, sb.ENGINE_MIXED])
def test_batch_equals_alone(ref, lib, engine):
    lib.starsh_set_oversample(b"10")
    alone, keep = [], []
    for case in CASES:
        pr = _problem(ref, case)
        keep.append(pr)
        M = approximate_b200(lib, pr.b200_format(), case["maxrank"],
                             case["tol"], engine=engine)
        err = ref.dfe(as_ref_blrm(M))
        assert 0 <= err <= case["tol"], (case, err)
        alone.append(M)
    prs = [_problem(ref, case) for case in CASES]
    n = len(CASES)
    Ms = (POINTER(sb.Blrm) * n)()
    Fs = (POINTER(sb.Blrf) * n)(*[pr.b200_format() for pr in prs])
    ranks = (c_int * n)(*[c["maxrank"] for c in CASES])
    tols = (c_double * n)(*[c["tol"] for c in CASES])
    info = lib.starsh_b200_approximate_batch(n, Ms, Fs, ranks, tols, None,
                                             engine, sb.FLAG_HOST_MIRROR)
    assert info == 0, lib.starsh_b200_last_error()
    st = sb.stats(lib)
    assert st.tiles == sum((-(-c["n"] // c["nb"])) ** 2 for c in CASES)
    for p in range(n):
        _assert_same(alone[p], Ms[p])
        lib.starsh_blrm_free(alone[p])
        lib.starsh_blrm_free(Ms[p])


def _server(lib, budget, engine=sb.ENGINE_MIXED, max_group=0):
    srv = c_void_p()
    assert lib.starsh_b200_server_new(byref(srv), budget, engine,
                                      max_group) == 0
    return srv


def _server_stats(lib, srv):
    st = sb.ServerStats()
    assert lib.starsh_b200_server_get_stats(srv, byref(st)) == 0
    return st


@pytest.mark.gpu
def test_server_alone_vs_mix(ref, lib):
    lib.starsh_set_oversample(b"10")
    srv = _server(lib, 8e9)
    target = CASES[1]
    nrhs = 4
    rng = np.random.default_rng(7)
    A = np.asfortranarray(rng.standard_normal((target["n"], nrhs)))

    def submit(pr, case, B, keep):
        t = c_longlong()
        a_ptr = A.ctypes.data if B is not None else None
        b_ptr = B.ctypes.data if B is not None else None
        assert lib.starsh_b200_server_submit(
            srv, pr.b200_format(), case["maxrank"], case["tol"],
            nrhs if B is not None else 0, a_ptr, target["n"], b_ptr,
            target["n"], keep, byref(t)) == 0
        return t.value

    def wait(t):
        M = POINTER(sb.Blrm)()
        lat = c_double()
        assert lib.starsh_b200_server_wait(srv, t, byref(M), byref(lat)) == 0
        assert lat.value > 0.0
        return M

    # alone
    pr1 = _problem(ref, target)
    B1 = np.zeros((target["n"], nrhs), order="F")
    M1 = wait(submit(pr1, target, B1, 1))
    assert _server_stats(lib, srv).groups == 1
    # in a mix: admission held until every request is queued, so all four
    # share one group
    assert lib.starsh_b200_server_pause(srv, 1) == 0
    others = [_problem(ref, c) for c in (CASES[0], CASES[2], CASES[3])]
    pr2 = _problem(ref, target)
    B2 = np.zeros((target["n"], nrhs), order="F")
    tickets = [submit(others[0], CASES[0], None, 0),
               submit(pr2, target, B2, 1),
               submit(others[1], CASES[2], None, 0),
               submit(others[2], CASES[3], None, 0)]
    assert lib.starsh_b200_server_pause(srv, 0) == 0
    Ms = [wait(t) for t in tickets]
    st = _server_stats(lib, srv)
    assert st.groups == 2 and st.completed == 5 and st.failed == 0
    M2 = Ms[1]
    assert lib.starsh_b200_blrm_download(M1) == 0
    assert lib.starsh_b200_blrm_download(M2) == 0
    _assert_same(M1, M2)
    np.testing.assert_array_equal(B1, B2)
    # and the product is the one of the reference's dmml on those factors
    Bref = ref.dmml(as_ref_blrm(M1), A)
    assert np.max(np.abs(B1 - Bref)) <= 1e-12 * np.max(np.abs(Bref))
    assert _server_stats(lib, srv).resident_bytes > 0
    assert lib.starsh_b200_server_release(srv, M1) == 0
    assert lib.starsh_b200_server_release(srv, M2) == 0
    assert _server_stats(lib, srv).resident_bytes == 0
    assert lib.starsh_b200_server_free(srv) == 0


@pytest.mark.gpu
def test_server_admits_by_budget(ref, lib):
    lib.starsh_set_oversample(b"10")
    case = dict(kind="spatial", n=2048, nb=512, kernel_name="exp",
                maxrank=100, tol=1e-5)
    # admission estimate of one request: 16 tiles of 512 x 512 with factors
    # at rank 100, plus 4 doubles per row and column index
    est = 16 * 8 * (512 + 512) * 100 + 8 * 4 * 4096
    srv = _server(lib, 1.5 * est)
    assert lib.starsh_b200_server_pause(srv, 1) == 0
    prs = [_problem(ref, case) for _ in range(3)]
    big = _problem(ref, dict(case, n=4096))
    tickets = []
    for pr in prs + [big]:
        t = c_longlong()
        assert lib.starsh_b200_server_submit(
            srv, pr.b200_format(), case["maxrank"], case["tol"], 0, None, 0,
            None, 0, 0, byref(t)) == 0
        tickets.append(t.value)
    assert lib.starsh_b200_server_pause(srv, 0) == 0
    status = [lib.starsh_b200_server_wait(srv, t, None, None) for t in tickets]
    assert status[:3] == [0, 0, 0]
    assert status[3] == sb.MALLOC_ERROR     # never fits the budget
    st = _server_stats(lib, srv)
    assert st.groups == 3                   # one request per group
    assert st.completed == 3 and st.failed == 1
    assert lib.starsh_b200_server_free(srv) == 0
