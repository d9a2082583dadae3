"""TLR-by-dense product and error on the device against the reference's
starsh_blrm__dmml / starsh_blrm__dfe and the numpy restatement, on the same
factors (so the comparison is to FP64 rounding, 1e-12 relative)."""
import ctypes
from ctypes import POINTER, c_double

import numpy as np
import pytest

import oracle
import starsh_b200 as sb
from harness import RefProblem, approximate_b200, as_ref_blrm


def dmml_b200(lib, M, A, alpha=1.0, beta=0.0, B=None):
    A = np.asfortranarray(A, np.float64)
    n, nrhs = A.shape
    B = np.zeros_like(A) if B is None else np.asfortranarray(B, np.float64).copy(order="F")
    info = lib.starsh_blrm__dmml_b200(M, nrhs, alpha,
                                      A.ctypes.data_as(POINTER(c_double)), n,
                                      beta, B.ctypes.data_as(POINTER(c_double)), n)
    assert info == 0
    return B


def close(a, b, rtol=1e-12):
    return np.max(np.abs(a - b)) <= rtol * np.max(np.abs(b))


@pytest.fixture(scope="module")
def c1(ref, lib):
    pr = RefProblem(ref, "spatial", 3600, 400, kernel_name="exp", beta=0.1)
    M = approximate_b200(lib, pr.b200_format(), 100, 1e-5)
    yield pr, M
    lib.starsh_blrm_free(M)


@pytest.mark.gpu
@pytest.mark.parametrize("nrhs,alpha,beta", [(1, 1.0, 0.0), (7, -0.5, 2.0),
                                             (64, 1.0, 1.0)])
def test_dmml_matches_reference_on_same_factors(ref, lib, c1, nrhs, alpha, beta):
    pr, M = c1
    rng = np.random.default_rng(nrhs)
    A = rng.standard_normal((3600, nrhs))
    B0 = rng.standard_normal((3600, nrhs))
    got = dmml_b200(lib, M, A, alpha, beta, B0)
    want = ref.dmml(as_ref_blrm(M), A, alpha, beta, B0)
    assert close(got, want)
    c = oracle.blrm_contents(as_ref_blrm(M))
    assert close(got, oracle.dmml(c, pr.block, A, alpha, beta, B0))


@pytest.mark.gpu
def test_dmml_onfly_and_symmetric(ref, lib):
    A = np.random.default_rng(3).standard_normal((2000, 5))
    for symm, onfly in [(b"N", 1), (b"S", 0), (b"S", 1)]:
        pr = RefProblem(ref, "spatial", 2000, 250, kernel_name="exp",
                        beta=0.1, symm=symm)
        M = approximate_b200(lib, pr.b200_format(), 60, 1e-6, onfly=onfly)
        c = oracle.blrm_contents(as_ref_blrm(M))
        got = dmml_b200(lib, M, A)
        assert close(got, oracle.dmml(c, pr.block, A)), (symm, onfly)
        if onfly == 0:
            assert close(got, ref.dmml(as_ref_blrm(M), A))
        lib.starsh_blrm_free(M)


@pytest.mark.gpu
def test_dmml_and_dfe_of_reference_engine_result(ref, lib):
    # a matrix compressed by the reference engine: factors are uploaded
    pr = RefProblem(ref, "coulomb", 1536, 256, ndim=3, place=1)
    Mref = ref.approximate(pr.F, 80, 1e-5)
    A = np.random.default_rng(5).standard_normal((1536, 3))
    Mb = ctypes.cast(Mref, POINTER(sb.Blrm))
    assert close(dmml_b200(lib, Mb, A), ref.dmml(Mref, A))
    assert abs(lib.starsh_blrm__dfe_b200(Mb) - ref.dfe(Mref)) <= 1e-9 * ref.dfe(Mref)
    lib.starsh_b200_blrm_release(Mb)
    ref.lib.starsh_blrm_free(Mref)


@pytest.mark.gpu
def test_dmml_device_pointers(ref, lib, c1):
    import torch
    pr, M = c1
    A = torch.randn(3600, 16, dtype=torch.float64, device="cuda").t().contiguous().t()
    B = torch.zeros(3600, 16, dtype=torch.float64, device="cuda").t().contiguous().t()
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.starsh_b200_blrm_dmml_device(M, 16, 1.0, A.data_ptr(), 3600, 0.0,
                                            B.data_ptr(), 3600, stream) == 0
    torch.cuda.synchronize()
    want = ref.dmml(as_ref_blrm(M), A.cpu().numpy())
    assert close(B.cpu().numpy(), want)


@pytest.mark.gpu
def test_dmml_argument_errors(lib, c1):
    _, M = c1
    A = np.zeros((3600, 2))
    B = np.zeros((3600, 2))
    D = POINTER(c_double)
    assert lib.starsh_blrm__dmml_b200(M, 2, 1.0, A.ctypes.data_as(D), 100, 0.0,
                                      B.ctypes.data_as(D), 3600) == sb.WRONG_PARAMETER
    assert lib.starsh_blrm__dmml_b200(M, -1, 1.0, A.ctypes.data_as(D), 3600, 0.0,
                                      B.ctypes.data_as(D), 3600) == sb.WRONG_PARAMETER
