"""The no-allocation entry point starsh_b200_dense_rsvd_noalloc, for callers
that cannot call cudaMalloc (stream capture, allocator-owned device memory,
threads that must not wait on the allocator): its factors match the drop-in
engine's on the same one-tile problem, on two calls in a row (the scratch
array keeps the first call's contents), and oversized tiles are refused.

Collected last (file name) so a failure here leaves every other test run."""
import ctypes
from ctypes import POINTER, byref

import numpy as np
import pytest

import oracle
import starsh_b200 as sb
from harness import RefProblem, approximate_b200, as_ref_blrm

TOL = 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("N,MAXRANK,OVERSAMPLE", [(200, 64, 16), (256, 80, 16)])
def test_noalloc_matches_engine_twice(ref, lib, N, MAXRANK, OVERSAMPLE):
    # the second case uses the largest tile and sketch width the fixed
    # scratch accepts (256 x 256, 96 columns)
    import torch
    # one 200 x 200 tile: a smooth 2-D kernel whose rank is below maxrank
    pr = RefProblem(ref, "spatial", N, N, kernel_name="sqexp", beta=0.3)
    M = approximate_b200(lib, pr.b200_format(), MAXRANK, TOL,
                         oversample=OVERSAMPLE)
    c = oracle.blrm_contents(as_ref_blrm(M))
    assert c["ranks"].shape == (1,) and 0 < c["ranks"][0] <= MAXRANK
    r_ref, U_ref, V_ref = int(c["ranks"][0]), c["U"][0], c["V"][0]
    lib.starsh_blrm_free(M)

    # the same tile as the engine generated it: this library's device
    # generator, reached through its host kernel entry point
    gen = sb.KERNEL(sb.kernel_symbol(lib, "starsh_ssdata_block_sqrexp_kernel_2d"))
    idx = np.arange(N, dtype=np.int64)
    host = np.zeros((N, N))
    gen(N, N, idx.ctypes.data_as(POINTER(sb.STARSH_int)),
        idx.ctypes.data_as(POINTER(sb.STARSH_int)), pr.data, pr.data,
        host.ctypes.data, N)
    D = torch.tensor(host.T, dtype=torch.float64, device="cuda")
    D = D.t().contiguous().t()                       # column-major, ld = N
    stream = torch.cuda.current_stream()
    for call in range(2):
        U = torch.full((MAXRANK, N), float("nan"), dtype=torch.float64,
                       device="cuda")                # column-major N x maxrank
        V = torch.full((MAXRANK, N), float("nan"), dtype=torch.float64,
                       device="cuda")
        rank = torch.full((1,), -7, dtype=torch.int32, device="cuda")
        info = lib.starsh_b200_dense_rsvd_noalloc(
            D.data_ptr(), N, N, N, MAXRANK, OVERSAMPLE, TOL, U.data_ptr(),
            V.data_ptr(), rank.data_ptr(), stream.cuda_stream)
        assert info == 0, lib.starsh_b200_last_error()
        torch.cuda.synchronize()
        r = int(rank.item())
        assert r == r_ref, (call, r, r_ref)
        Uh = U[:r].cpu().numpy().T
        Vh = V[:r].cpu().numpy().T
        for got, want in ((Uh, U_ref), (Vh, V_ref), (Uh @ Vh.T, U_ref @ V_ref.T)):
            assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want)), call


@pytest.mark.gpu
def test_noalloc_rejects_oversized_tiles(lib):
    import torch
    D = torch.zeros(300 * 300, dtype=torch.float64, device="cuda")
    out = torch.zeros(300 * 300, dtype=torch.float64, device="cuda")
    rank = torch.zeros(1, dtype=torch.int32, device="cuda")
    # rows above 256
    assert lib.starsh_b200_dense_rsvd_noalloc(
        D.data_ptr(), 300, 200, 300, 50, 10, 1e-6, out.data_ptr(),
        out.data_ptr(), rank.data_ptr(), None) == sb.WRONG_PARAMETER
    assert b"exceeds the fixed scratch" in lib.starsh_b200_last_error()
    # sketch width above 96
    assert lib.starsh_b200_dense_rsvd_noalloc(
        D.data_ptr(), 256, 256, 256, 90, 10, 1e-6, out.data_ptr(),
        out.data_ptr(), rank.data_ptr(), None) == sb.WRONG_PARAMETER


@pytest.mark.gpu
def test_noalloc_rank_above_maxrank_leaves_factors_unwritten(ref, lib):
    # a rough kernel (exponential, short correlation length) on one 128 x 128
    # tile needs far more than maxrank = 4 columns at tol 1e-6: the call
    # reports rank -1 and writes neither factor, so the caller keeps the
    # tile dense
    import torch
    N, MAXRANK = 128, 4
    pr = RefProblem(ref, "spatial", N, N, kernel_name="exp", beta=0.02)
    gen = sb.KERNEL(sb.kernel_symbol(lib, "starsh_ssdata_block_exp_kernel_2d"))
    idx = np.arange(N, dtype=np.int64)
    host = np.zeros((N, N))
    gen(N, N, idx.ctypes.data_as(POINTER(sb.STARSH_int)),
        idx.ctypes.data_as(POINTER(sb.STARSH_int)), pr.data, pr.data,
        host.ctypes.data, N)
    D = torch.tensor(host.T, dtype=torch.float64, device="cuda")
    D = D.t().contiguous().t()
    U = torch.full((MAXRANK, N), float("nan"), dtype=torch.float64, device="cuda")
    V = torch.full((MAXRANK, N), float("nan"), dtype=torch.float64, device="cuda")
    rank = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    info = lib.starsh_b200_dense_rsvd_noalloc(
        D.data_ptr(), N, N, N, MAXRANK, 10, TOL, U.data_ptr(), V.data_ptr(),
        rank.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert info == 0, lib.starsh_b200_last_error()
    torch.cuda.synchronize()
    assert int(rank.item()) == -1
    assert torch.isnan(U).all() and torch.isnan(V).all()
