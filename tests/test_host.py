"""Host side of libstarsh_b200 (no GPU calls): the library loads and exports
every function the headers declare, point sets and Z-order match the
reference bit for bit, the TLR format lists match, kernel pointers of both
libraries are recognised, backend selection follows the environment."""
import ctypes
import os
import re
from ctypes import POINTER, byref, c_double, c_int, c_void_p

import numpy as np
import pytest

import oracle
import starsh_b200 as sb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        text = open(os.path.join(ROOT, "include", f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        # function prototypes: identifier followed by '(' at top level
        for m in re.finditer(r"\b(starsh_\w+|array_\w+)\s*\(", text):
            names.add(m.group(1))
        # kernel symbol groups declared through macros
        for fam in ("exp", "sqrexp", "matern", "matern2"):
            for d in ("1d", "2d", "3d", "4d", "nd"):
                for s in ("", "_simd"):
                    names.add(f"starsh_ssdata_block_{fam}_kernel_{d}{s}")
        for fam in ("sin", "cos"):
            for d in ("1d", "2d", "3d", "4d", "nd"):
                for s in ("", "_simd"):
                    names.add(f"starsh_eddata_block_{fam}_kernel_{d}{s}")
    names.discard("starsh_blrm_approximate")   # a variable, checked below
    return names


def test_exports_every_declared_symbol(lib):
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing
    ctypes.c_void_p.in_dll(lib, "starsh_blrm_approximate")
    ctypes.c_int.in_dll(lib, "starsh_params")


def _particles(lib, n, ndim, place, seed):
    oracle.srand(seed)
    p = POINTER(sb.Particles)()
    assert lib.starsh_particles_generate(byref(p), n, ndim, place) == 0
    a = np.ctypeslib.as_array(p.contents.point, shape=(n * ndim,)).reshape(ndim, n).copy()
    lib.starsh_particles_free(p)
    return a


@pytest.mark.parametrize("n,ndim,place", [(3600, 2, 6), (4096, 3, 1),
                                          (100, 2, 3), (1000, 3, 6), (33, 1, 6),
                                          (50, 4, 1)])
def test_points_bit_exact_vs_reference(lib, ref, n, ndim, place):
    assert np.array_equal(_particles(lib, n, ndim, place, 3),
                          ref.points(n, ndim, place, seed=3))


def test_zsort_of_given_points(lib, orc):
    rng = np.random.default_rng(1)
    pts = rng.random(3 * 999)
    mine = pts.copy()
    p = sb.Particles(999, 3, mine.ctypes.data_as(POINTER(c_double)))
    # zsort replaces the point buffer: give it a malloc'd copy
    libc = ctypes.CDLL("libc.so.6")
    libc.malloc.restype = c_void_p
    buf = libc.malloc(8 * 3 * 999)
    ctypes.memmove(buf, mine.ctypes.data, 8 * 3 * 999)
    p.point = ctypes.cast(buf, POINTER(c_double))
    assert lib.starsh_particles_zsort_inplace(byref(p)) == 0
    got = np.ctypeslib.as_array(p.point, shape=(3 * 999,)).copy()
    want = pts.copy()
    orc.lib.oracle_zsort(999, 3, want.ctypes.data_as(POINTER(c_double)))
    assert np.array_equal(got, want)


def test_tlr_format_matches_reference(lib, ref):
    for n, nb, symm in [(3600, 400, b"N"), (3000, 400, b"N"), (2000, 250, b"S")]:
        data, kern, _ = ref.spatial(n, 2, 1, 0.1, seed=0)
        P = ref.problem(data, kern, n, symm=symm)
        C, F = ref.tlr(P, data, n, nb, symm=symm)
        # same through this library, on the same data and kernel pointer
        shape = (sb.STARSH_int * 2)(n, n)
        Pm = POINTER(sb.Problem)()
        assert lib.starsh_problem_new(byref(Pm), 2, shape, symm, b"d", data,
                                      data, kern, b"x") == 0
        Cm = POINTER(sb.Cluster)()
        assert lib.starsh_cluster_new_plain(byref(Cm), data, n, nb) == 0
        Fm = POINTER(sb.Blrf)()
        assert lib.starsh_blrf_new_tlr(byref(Fm), Pm, symm, Cm, Cm) == 0
        a, b = F.contents, Fm.contents
        assert (a.nbrows, a.nbcols, a.nblocks_far, a.nblocks_near) == \
               (b.nbrows, b.nbcols, b.nblocks_far, b.nblocks_near)
        nf = a.nblocks_far
        for fld, cnt in [("block_far", 2 * nf), ("brow_far_start", a.nbrows + 1),
                         ("brow_far", nf), ("bcol_far_start", a.nbcols + 1),
                         ("bcol_far", nf)]:
            x = np.ctypeslib.as_array(getattr(a, fld), shape=(cnt,))
            y = np.ctypeslib.as_array(getattr(b, fld), shape=(cnt,))
            assert np.array_equal(x, y), fld
        R, Rm = C.contents, Cm.contents
        assert np.array_equal(np.ctypeslib.as_array(R.size, shape=(R.nblocks,)),
                              np.ctypeslib.as_array(Rm.size, shape=(Rm.nblocks,)))


def test_kernel_registry_recognises_both_libraries(lib, ref):
    hint = c_int()
    cases = {"starsh_ssdata_block_exp_kernel_2d": (1, 2),
             "starsh_ssdata_block_sqrexp_kernel_nd_simd": (2, 0),
             "starsh_ssdata_block_matern2_kernel_3d": (4, 3),
             "starsh_esdata_block_coulomb_potential_kernel_3d": (5, 3),
             "starsh_eddata_block_sin_kernel_3d_simd": (6, 3),
             "starsh_eddata_block_cos_kernel_1d": (7, 1),
             "starsh_generate_3d_virus": (8, 3)}
    for name, (fam, nd) in cases.items():
        addrs = [sb.kernel_symbol(lib, name)]
        if hasattr(ref.lib, name):       # Matérn needs GSL in the reference
            addrs.append(ref.symbol(name))
        for addr in addrs:
            assert lib.starsh_b200_kernel_family(addr, byref(hint)) == fam, name
            assert hint.value == nd, name
    libc = ctypes.CDLL("libc.so.6")
    assert lib.starsh_b200_kernel_family(
        ctypes.cast(libc.abs, c_void_p).value, byref(hint)) == 0
    # explicit registration (e.g. a Coulomb kernel with a unit diagonal)
    assert lib.starsh_b200_kernel_register(ctypes.cast(libc.labs, c_void_p).value,
                                           5, 1.0) == 0
    assert lib.starsh_b200_kernel_family(ctypes.cast(libc.labs, c_void_p).value,
                                         byref(hint)) == 5


def test_backend_selection(lib):
    approx = lambda: ctypes.c_void_p.in_dll(lib, "starsh_blrm_approximate").value
    assert lib.starsh_set_lrengine(b"RSVD") == 0
    assert lib.starsh_set_backend(b"B200") == 0
    assert approx() == ctypes.cast(lib.starsh_blrm__drsdd_b200, c_void_p).value
    assert lib.starsh_set_lrengine(b"RSVD_MP") == 0
    assert approx() == ctypes.cast(lib.starsh_blrm__drsdd_b200_mp, c_void_p).value
    # CPU backends are not part of this library; an invalid name is refused
    assert lib.starsh_set_backend(b"OPENMP") == sb.WRONG_PARAMETER
    assert lib.starsh_set_backend(b"NOPE") == sb.WRONG_PARAMETER
    assert lib.starsh_set_oversample(b"0") == sb.WRONG_PARAMETER
    assert lib.starsh_set_oversample(b"16") == 0
    assert lib.starsh_set_lrengine(b"RSVD") == 0
    assert lib.starsh_init() == 0
