"""Conjugate gradients on the device-resident TLR matrix against the
reference's starsh_itersolvers__dcg_omp on the same factors (an SPD
covariance: exponential kernel with a nugget)."""
import ctypes
from ctypes import byref, c_int

import numpy as np
import pytest

import starsh_b200 as sb
from harness import RefProblem, approximate_b200, as_ref_blrm


@pytest.mark.gpu
@pytest.mark.parametrize("nrhs", [1, 3])
def test_cg_matches_reference(ref, lib, nrhs):
    import torch
    pr = RefProblem(ref, "spatial", 2025, 225, kernel_name="exp", beta=0.1,
                    noise=0.5)
    M = approximate_b200(lib, pr.b200_format(), 100, 1e-9)
    n = 2025
    rng = np.random.default_rng(nrhs)
    B = np.asfortranarray(rng.standard_normal((n, nrhs)))
    X0 = np.zeros((n, nrhs), order="F")
    tol = 1e-10
    it_ref, Xref = ref.cg(as_ref_blrm(M), B, X0, tol)
    assert it_ref >= 0
    # host entry point (the reference's signature)
    X = X0.copy(order="F")
    it = lib.starsh_itersolvers__dcg_b200(M, nrhs, B.ctypes.data, n,
                                          X.ctypes.data, n, tol, None)
    assert it >= 0, lib.starsh_b200_last_error()
    assert abs(it - it_ref) <= 2
    # the solution solves the same TLR system to tol (residual through the
    # reference's dmml on these factors) and agrees with the reference's
    R = B - ref.dmml(as_ref_blrm(M), X)
    for j in range(nrhs):
        assert np.linalg.norm(R[:, j]) <= 1.5 * tol * np.linalg.norm(B[:, j])
    assert np.max(np.abs(X - Xref)) <= 1e-8 * np.max(np.abs(Xref))
    # device entry point: same iterations and solution
    dB = torch.tensor(B.T.copy(), device="cuda")   # row j = column j
    dX = torch.zeros_like(dB)
    its = c_int()
    assert lib.starsh_b200_dcg_device(M, nrhs, dB.data_ptr(), n, dX.data_ptr(),
                                      n, tol, 0, None, byref(its)) == 0
    torch.cuda.synchronize()
    assert its.value == it
    np.testing.assert_array_equal(dX.cpu().numpy().T, X)
    lib.starsh_blrm_free(M)
