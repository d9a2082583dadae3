"""Particle files and serialised matrices (CPU).

Particle files: the B200 library and the compiled reference
(src/applications/particles.c:789-1088) write byte-identical ASCII and
binary files, read each other's files to the same points, and return the
same error codes on missing, malformed and short files.

Matrix streams: a matrix produced by the reference engine
(starsh_blrm__drsdd) survives serialise -> deserialise bit for bit (block
lists, ranks, factors, dense near blocks), the reference's own dmml and dfe
give identical results on the copy, file and memory streams agree, and
damaged streams are refused."""
import ctypes
import os
from ctypes import POINTER, byref, c_char_p, c_int, c_size_t, c_void_p

import numpy as np
import pytest

import oracle
import starsh_b200 as sb
from harness import RefProblem

ASCII, BINARY = 1, 2
SUCCESS, FILE_NOT_EXIST, FILE_WRONG_INPUT, WRONG_PARAMETER = 0, 2, 3, 4


@pytest.fixture(scope="module")
def ref_io(ref):
    L = ref.lib
    for name, args in [
        ("starsh_particles_read_from_file", [POINTER(POINTER(oracle.Particles)),
                                             c_char_p, c_int]),
        ("starsh_particles_write_to_file", [c_void_p, c_char_p, c_int]),
    ]:
        fn = getattr(L, name)
        fn.restype = c_int
        fn.argtypes = args
    return L


def _points(lib, n, ndim, seed):
    oracle.srand(seed)
    p = POINTER(sb.Particles)()
    assert lib.starsh_particles_generate(byref(p), n, ndim, 1) == 0
    return p


def _as_array(p):
    c = p.contents
    return np.ctypeslib.as_array(c.point, shape=(c.count * c.ndim,)).reshape(
        c.ndim, c.count).copy()


@pytest.mark.parametrize("ftype", [ASCII, BINARY])
@pytest.mark.parametrize("n,ndim", [(1000, 3), (17, 1), (64, 4)])
def test_particle_files_match_reference(lib, ref_io, tmp_path, ftype, n, ndim):
    p = _points(lib, n, ndim, 5)
    ours, theirs = str(tmp_path / "ours"), str(tmp_path / "theirs")
    assert lib.starsh_particles_write_to_file(p, ours.encode(), ftype) == 0
    assert ref_io.starsh_particles_write_to_file(
        ctypes.cast(p, c_void_p), theirs.encode(), ftype) == 0
    assert open(ours, "rb").read() == open(theirs, "rb").read()
    q = POINTER(sb.Particles)()
    assert lib.starsh_particles_read_from_file(byref(q), theirs.encode(),
                                               ftype) == 0
    r = POINTER(oracle.Particles)()
    assert ref_io.starsh_particles_read_from_file(byref(r), ours.encode(),
                                                  ftype) == 0
    a, b = _as_array(q), _as_array(ctypes.cast(r, POINTER(sb.Particles)))
    assert a.shape == (ndim, n) and np.array_equal(a, b)
    orig = _as_array(p)
    if ftype == BINARY:
        assert np.array_equal(a, orig)
    else:   # six decimals, as the reference prints them
        assert np.abs(a - orig).max() <= 5e-7
    lib.starsh_particles_free(q)
    lib.starsh_particles_free(p)


def _write(path, data):
    with open(path, "wb") as f:
        f.write(data)


@pytest.mark.parametrize("content,ftype", [
    (b"cnt=3, ndim=2\n1,2\n", ASCII),                  # bad header
    (b"count=3, ndim=2\n1.0, 2.0\n3.0, 4.0\n", ASCII),  # one point short
    (b"count=2, ndim=2\n1.0, 2.0\n3.0 4.0\n", ASCII),   # missing comma
    (np.array([5], np.uint64).tobytes() + np.array([2], np.int32).tobytes()
     + np.zeros(3).tobytes(), BINARY),                 # 3 of 10 doubles
    (b"\x01\x02", BINARY),                             # no header
])
def test_particle_file_errors_match_reference(lib, ref_io, tmp_path, content,
                                              ftype):
    path = str(tmp_path / "bad")
    _write(path, content)
    q = POINTER(sb.Particles)()
    r = POINTER(oracle.Particles)()
    mine = lib.starsh_particles_read_from_file(byref(q), path.encode(), ftype)
    theirs = ref_io.starsh_particles_read_from_file(byref(r), path.encode(),
                                                    ftype)
    assert mine == theirs == FILE_WRONG_INPUT


def test_particle_file_missing_and_bad_type(lib, ref_io, tmp_path):
    path = str(tmp_path / "absent").encode()
    q = POINTER(sb.Particles)()
    r = POINTER(oracle.Particles)()
    for ftype in (ASCII, BINARY):
        assert lib.starsh_particles_read_from_file(byref(q), path, ftype) == \
            ref_io.starsh_particles_read_from_file(byref(r), path, ftype) == \
            FILE_NOT_EXIST
    assert lib.starsh_particles_read_from_file(byref(q), path, 7) == \
        ref_io.starsh_particles_read_from_file(byref(r), path, 7) == \
        WRONG_PARAMETER
    p = _points(lib, 10, 2, 1)
    assert lib.starsh_particles_write_to_file(
        p, str(tmp_path / "no" / "dir").encode(), ASCII) == FILE_NOT_EXIST
    lib.starsh_particles_free(p)


# ------------------------------------------------------------ matrices

def _serialize(lib, M):
    n = c_size_t()
    Mb = ctypes.cast(M, POINTER(sb.Blrm))
    assert lib.starsh_b200_blrm_serialize(Mb, None, 0, byref(n)) == 0
    buf = ctypes.create_string_buffer(n.value)
    m = c_size_t()
    assert lib.starsh_b200_blrm_serialize(Mb, buf, n.value, byref(m)) == 0
    assert m.value == n.value
    return buf.raw


def _deserialize(lib, P, data):
    M = POINTER(sb.Blrm)()
    info = lib.starsh_b200_blrm_deserialize(byref(M), P, data, len(data))
    return info, M


def _same(a, b):
    for key in ("far", "near", "ranks", "rstart", "rsize", "cstart", "csize"):
        assert np.array_equal(a[key], b[key]), key
    assert a["symm"] == b["symm"] and a["onfly"] == b["onfly"]
    for key in ("U", "V", "D"):
        assert len(a[key]) == len(b[key])
        for x, y in zip(a[key], b[key]):
            assert x.shape == y.shape and np.array_equal(x, y), key


@pytest.fixture(scope="module")
def ref_result(ref):
    """exp kernel, 2-D, 1600 points in 4 x 4 tiles of 400: the reference's
    sequential engine at maxrank 100 demotes the diagonal tiles, so the
    result holds far and near blocks."""
    pr = RefProblem(ref, "spatial", 1600, 400, kernel_name="exp", beta=0.1)
    M = ref.approximate(pr.F, 100, 1e-7, sequential=True)
    yield pr, M
    ref.lib.starsh_blrm_free(M)


def test_blrm_stream_round_trip_of_reference_result(lib, ref, ref_result,
                                                    tmp_path):
    pr, M = ref_result
    orig = oracle.blrm_contents(M)
    assert len(orig["near"]) > 0 and len(orig["far"]) > 0
    data = _serialize(lib, M)
    info, L = _deserialize(lib, pr.P, data)
    assert info == SUCCESS
    copy = oracle.blrm_contents(ctypes.cast(L, POINTER(oracle.Blrm)))
    _same(orig, copy)
    # the reference's own products and error on the copy
    A = np.random.default_rng(0).standard_normal((1600, 3))
    Lr = ctypes.cast(L, POINTER(oracle.Blrm))
    assert np.array_equal(ref.dmml(M, A), ref.dmml(Lr, A))
    assert ref.lib.starsh_blrm__dfe(M) == ref.lib.starsh_blrm__dfe(Lr)
    # the file stream is the memory stream
    path = str(tmp_path / "m.tlr").encode()
    assert lib.starsh_b200_blrm_write_to_file(
        ctypes.cast(M, POINTER(sb.Blrm)), path) == 0
    assert open(path, "rb").read() == data
    F2 = POINTER(sb.Blrm)()
    assert lib.starsh_b200_blrm_read_from_file(byref(F2), pr.P, path) == 0
    _same(orig, oracle.blrm_contents(ctypes.cast(F2, POINTER(oracle.Blrm))))
    # a stream of the copy is the same stream
    assert _serialize(lib, L) == data
    lib.starsh_b200_blrm_free_read(F2)
    lib.starsh_b200_blrm_free_read(L)


def test_blrm_stream_symmetric_onfly(lib, ref):
    pr = RefProblem(ref, "spatial", 1200, 300, kernel_name="sqexp", beta=0.2,
                    noise=1e-4, symm=b"S")
    M = ref.approximate(pr.F, 60, 1e-6, onfly=1, sequential=True)
    data = _serialize(lib, M)
    info, L = _deserialize(lib, pr.P, data)
    assert info == SUCCESS
    Lc = L.contents
    assert Lc.onfly == 1 and Lc.format.contents.symm == b"S"
    assert ctypes.addressof(Lc.format.contents.row_cluster.contents) == \
        ctypes.addressof(Lc.format.contents.col_cluster.contents)
    _same(oracle.blrm_contents(M),
          oracle.blrm_contents(ctypes.cast(L, POINTER(oracle.Blrm))))
    A = np.random.default_rng(1).standard_normal((1200, 2))
    assert np.array_equal(ref.dmml(M, A),
                          ref.dmml(ctypes.cast(L, POINTER(oracle.Blrm)), A))
    lib.starsh_b200_blrm_free_read(L)
    ref.lib.starsh_blrm_free(M)


def test_blrm_stream_rejects_damage(lib, ref, ref_result):
    pr, M = ref_result
    data = _serialize(lib, M)
    for cut in (0, 8, 40, len(data) // 2, len(data) - 8, len(data) - 1):
        assert _deserialize(lib, pr.P, data[:cut])[0] == FILE_WRONG_INPUT, cut
    def flipped(pos, bit=0x10):
        bad = bytearray(data)
        bad[pos] ^= bit
        return _deserialize(lib, pr.P, bytes(bad))[0]
    # magic, version, an unknown flag, block counts, clusterings, factors,
    # checksum
    for pos in (0, 9, 12, 33, 60, len(data) // 3, len(data) - 20,
                len(data) - 3):
        assert flipped(pos) == FILE_WRONG_INPUT, pos
    # a stored shape or symmetry that is not the problem's
    for pos, bit in ((12, 1), (16, 0x10), (24, 0x10)):
        assert flipped(pos, bit) == WRONG_PARAMETER, pos
    # another problem's shape
    other = RefProblem(ref, "spatial", 1200, 400, kernel_name="exp", beta=0.1)
    assert _deserialize(lib, other.P, data)[0] == WRONG_PARAMETER
    # a buffer too small: the size needed comes back
    need = c_size_t()
    buf = ctypes.create_string_buffer(100)
    assert lib.starsh_b200_blrm_serialize(ctypes.cast(M, POINTER(sb.Blrm)),
                                          buf, 100, byref(need)) == WRONG_PARAMETER
    assert need.value == len(data)
    M2 = POINTER(sb.Blrm)()
    assert lib.starsh_b200_blrm_read_from_file(
        byref(M2), pr.P, b"/nonexistent/m.tlr") == FILE_NOT_EXIST
