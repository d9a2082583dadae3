"""A device-resident B200 result through the matrix stream: writing brings
the factors to the host, reading gives a host matrix whose factors the
device entry points upload again; products and error on the copy are the
original's bit for bit."""
import ctypes
from ctypes import POINTER, byref, c_double, c_size_t

import numpy as np
import pytest

import oracle
import starsh_b200 as sb
from harness import RefProblem, approximate_b200, as_ref_blrm


def _dmml(lib, M, A):
    A = np.asfortranarray(A, np.float64)
    B = np.zeros_like(A, order="F")
    assert lib.starsh_blrm__dmml_b200(M, A.shape[1], 1.0,
                                      A.ctypes.data_as(POINTER(c_double)),
                                      A.shape[0], 0.0,
                                      B.ctypes.data_as(POINTER(c_double)),
                                      A.shape[0]) == 0
    return B


@pytest.mark.gpu
@pytest.mark.parametrize("engine", [0, 1])
def test_device_result_round_trip(ref, lib, tmp_path, engine):
    pr = RefProblem(ref, "spatial", 4096, 512, kernel_name="sqexp", beta=0.1,
                    noise=1e-2)
    M = approximate_b200(lib, pr.b200_format(), 128, 1e-7, engine=engine,
                         flags=0)   # factors stay on the device
    path = str(tmp_path / "m.tlr").encode()
    assert lib.starsh_b200_blrm_write_to_file(M, path) == 0
    L = POINTER(sb.Blrm)()
    assert lib.starsh_b200_blrm_read_from_file(byref(L), pr.P, path) == 0
    a = oracle.blrm_contents(as_ref_blrm(M))
    b = oracle.blrm_contents(as_ref_blrm(L))
    assert np.array_equal(a["ranks"], b["ranks"])
    assert np.array_equal(a["near"], b["near"])
    for x, y in zip(a["U"] + a["V"] + a["D"], b["U"] + b["V"] + b["D"]):
        assert np.array_equal(x, y)
    A = np.random.default_rng(2).standard_normal((4096, 8))
    assert np.array_equal(_dmml(lib, M, A), _dmml(lib, L, A))
    assert lib.starsh_blrm__dfe_b200(M) == lib.starsh_blrm__dfe_b200(L)
    # the stream of the device result and of its host copy are the same
    n1, n2 = c_size_t(), c_size_t()
    assert lib.starsh_b200_blrm_serialize(M, None, 0, byref(n1)) == 0
    assert lib.starsh_b200_blrm_serialize(L, None, 0, byref(n2)) == 0
    assert n1.value == n2.value == len(open(path, "rb").read())
    lib.starsh_b200_blrm_free_read(L)
    lib.starsh_blrm_free(M)
