"""Generated kernel blocks: the library's device generator (reached through
its host kernel entry points, which evaluate on the GPU) against the
reference's own kernel functions on the same point sets and index lists,
entry-wise within 1e-13 relative; Matérn against the mpmath goldens."""
import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_void_p

import numpy as np
import pytest

import oracle
import starsh_b200 as sb

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
KTYPE = ctypes.CFUNCTYPE(None, c_int, c_int, POINTER(sb.STARSH_int),
                         POINTER(sb.STARSH_int), c_void_p, c_void_p, c_void_p,
                         c_int)


def call_kernel(addr, data, irow, icol, col_data=None):
    fn = KTYPE(addr)
    irow = np.ascontiguousarray(irow, np.int64)
    icol = np.ascontiguousarray(icol, np.int64)
    m, n = len(irow), len(icol)
    out = np.full((n, m + 3), np.nan)      # ld = m + 3
    fn(m, n, irow.ctypes.data_as(POINTER(sb.STARSH_int)),
       icol.ctypes.data_as(POINTER(sb.STARSH_int)), data, col_data or data,
       out.ctypes.data, m + 3)
    assert np.isnan(out[:, m:]).all()        # padding untouched
    return out[:, :m].T.copy()


def rel_close(a, b, rtol=1e-13):
    scale = np.maximum(np.abs(b), 1e-300)
    return np.max(np.abs(a - b) / scale) <= rtol


def index_sets(n, rng):
    rows = rng.integers(0, n, 37)
    cols = rng.integers(0, n, 53)
    cols[:5] = rows[:5]                      # coinciding points (r = 0)
    return rows, cols


@pytest.mark.gpu
@pytest.mark.parametrize("ktype,name", [(1, "exp"), (2, "sqrexp"),
                                        (11, "exp"), (12, "sqrexp")])
@pytest.mark.parametrize("ndim", [1, 2, 3, 4, 5])
def test_spatial_blocks(ref, lib, ktype, name, ndim):
    rng = np.random.default_rng(ndim * 100 + ktype)
    data, kern, info = ref.spatial(700, ndim, ktype, 0.13, 0.5, 0.25, 1,
                                   sigma=1.7, seed=ndim)
    assert info == 0
    suffix = f"{ndim}d" if ndim <= 4 else "nd"
    if ktype > 10:
        suffix += "_simd"
    mine = sb.kernel_symbol(lib, f"starsh_ssdata_block_{name}_kernel_{suffix}")
    rows, cols = index_sets(700, rng)
    want = ref.block(kern, data, rows, cols)
    got = call_kernel(mine, data, rows, cols)
    assert rel_close(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("ndim", [2, 3])
def test_coulomb_blocks(ref, lib, ndim):
    rng = np.random.default_rng(7)
    data = ref.particles_data(900, ndim, 1, seed=3)
    name = f"starsh_esdata_block_coulomb_potential_kernel_{ndim}d"
    rows, cols = index_sets(900, rng)
    want = ref.block(ref.kernel_ptr(name), data, rows, cols)
    got = call_kernel(sb.kernel_symbol(lib, name), data, rows, cols)
    assert rel_close(got, want)
    assert (got[want == 0] == 0).all()


@pytest.mark.gpu
@pytest.mark.parametrize("fam", ["sin", "cos"])
def test_helmholtz_blocks(ref, lib, fam):
    rng = np.random.default_rng(11)
    data = ref.eddata(800, 3, 1, 20.0, 1.0, seed=5)
    name = f"starsh_eddata_block_{fam}_kernel_3d"
    rows, cols = index_sets(800, rng)
    want = ref.block(ref.kernel_ptr(name), data, rows, cols)
    got = call_kernel(sb.kernel_symbol(lib, name), data, rows, cols)
    assert rel_close(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4, 7, 8, 9])
def test_rbf_virus_blocks(ref, lib, kind):
    rng = np.random.default_rng(kind)
    n = 500
    mesh = np.ascontiguousarray(rng.random((n, 3)) * 0.3)   # point-major
    md = oracle_md = sb.MDData(sb.Particles(n, 3, mesh.ctypes.data_as(POINTER(c_double))),
                               0.5, kind, 1, 1, 0.1, -1.0, n, 0)
    ptr = ctypes.cast(ctypes.byref(md), c_void_p)
    rows, cols = index_sets(n, rng)
    want = ref.block(ref.kernel_ptr("starsh_generate_3d_virus"), ptr, rows, cols)
    got = call_kernel(sb.kernel_symbol(lib, "starsh_generate_3d_virus"), ptr,
                      rows, cols)
    assert rel_close(got, want)
    del oracle_md


@pytest.mark.gpu
def test_matern_blocks_against_mpmath(lib):
    g = np.load(os.path.join(GOLDEN, "matern.npz"))
    for case in range(int(g["ncases"])):
        pts = g[f"pts{case}"]
        nu, beta, sigma, noise = g[f"par{case}"]
        family = int(g[f"fam{case}"])
        ndim, n = pts.shape
        flat = np.ascontiguousarray(pts.ravel())
        ss = sb.SSData(sb.Particles(n, ndim, flat.ctypes.data_as(POINTER(c_double))),
                       beta, nu, noise, sigma, 0.0, 0.0, 0.0)
        ptr = ctypes.cast(ctypes.byref(ss), c_void_p)
        name = "matern" if family == 3 else "matern2"
        fn = sb.kernel_symbol(lib, f"starsh_ssdata_block_{name}_kernel_{ndim}d")
        got = call_kernel(fn, ptr, g[f"rows{case}"], g[f"cols{case}"])
        want = g[f"want{case}"]
        assert rel_close(got, want, 1e-13), case
