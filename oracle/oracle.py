"""Oracle for the STARS-H TLR path -- TEST INFRASTRUCTURE.

Nothing in the product imports this module; the tests, the smoke check and
the CPU-baseline leg of bench.py use it as the checker.  It provides

* `Ref`: ctypes harness around the unmodified reference library compiled
  by oracle/Makefile (oracle/_ref/libstarsh_ref.so): point sets, problems,
  TLR formats, starsh_blrm__drsdd_omp, starsh_blrm__dfe(_omp),
  starsh_blrm__dmml;
* `Oracle`: the C restatement oracle/starsh_oracle.c
  (oracle/_ref/liboracle.so);
* numpy restatements of the per-tile RSVD (sequential/dense/drsdd.c:16-93),
  the rank cut (dense/dsvfr.c:16-47), dfe (sequential/blrm/dfe.c:16-134) and
  dmml (sequential/blrm/dmml.c:16-145), for small cases;
* Matérn entries from scipy (pinned to the mpmath goldens).
"""
import ctypes
import os
import subprocess
from ctypes import (POINTER, byref, c_char, c_char_p, c_double, c_int,
                    c_longlong, c_void_p)

import numpy as np

# The reference calls OpenBLAS from inside OpenMP loops; OpenBLAS must stay
# single-threaded there (the reference CI sets MKL_NUM_THREADS=1 likewise).
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libstarsh_ref.so")
ORACLE_SO = os.path.join(HERE, "_ref", "liboracle.so")
REF_SRC = "/root/reference"

_libc = ctypes.CDLL("libc.so.6")


def build():
    """Compiles the oracle (and the reference, when its sources exist)."""
    targets = ["_ref/liboracle.so"]
    if os.path.isdir(REF_SRC):
        targets.append("_ref/libstarsh_ref.so")
    subprocess.run(["make", "-C", HERE, "-s"] + targets, check=True)


def srand(seed):
    _libc.srand(seed)


# Structure layouts (same as stars-h_b200/starsh_b200, kept separate so
# that the oracle has no dependency on the product package).
from ctypes import Structure, c_size_t, c_ssize_t  # noqa: E402

STARSH_int = c_ssize_t


class Array(Structure):
    _fields_ = [("ndim", c_int), ("shape", POINTER(c_int)),
                ("stride", POINTER(c_ssize_t)), ("order", c_char),
                ("size", c_size_t), ("dtype", c_char),
                ("dtype_size", c_size_t), ("nbytes", c_size_t),
                ("data_nbytes", c_size_t), ("data", c_void_p)]


class Particles(Structure):
    _fields_ = [("count", STARSH_int), ("ndim", c_int),
                ("point", POINTER(c_double))]


class Cluster(Structure):
    _fields_ = [("data", c_void_p), ("ndata", STARSH_int),
                ("pivot", POINTER(STARSH_int)), ("nblocks", STARSH_int),
                ("nlevels", STARSH_int), ("level", POINTER(STARSH_int)),
                ("start", POINTER(STARSH_int)), ("size", POINTER(STARSH_int)),
                ("parent", c_void_p), ("child_start", c_void_p),
                ("child", c_void_p), ("type", c_int)]


class Blrf(Structure):
    _fields_ = [("problem", c_void_p), ("symm", c_char),
                ("row_cluster", POINTER(Cluster)),
                ("col_cluster", POINTER(Cluster)),
                ("nbrows", STARSH_int), ("nbcols", STARSH_int),
                ("nblocks_far", STARSH_int),
                ("block_far", POINTER(STARSH_int)),
                ("brow_far_start", POINTER(STARSH_int)),
                ("brow_far", POINTER(STARSH_int)),
                ("bcol_far_start", POINTER(STARSH_int)),
                ("bcol_far", POINTER(STARSH_int)),
                ("nblocks_far_local", STARSH_int),
                ("block_far_local", c_void_p),
                ("nblocks_near", STARSH_int),
                ("block_near", POINTER(STARSH_int)),
                ("brow_near_start", POINTER(STARSH_int)),
                ("brow_near", POINTER(STARSH_int)),
                ("bcol_near_start", POINTER(STARSH_int)),
                ("bcol_near", POINTER(STARSH_int)),
                ("nblocks_near_local", STARSH_int),
                ("block_near_local", c_void_p), ("type", c_int)]


class Blrm(Structure):
    _fields_ = [("format", POINTER(Blrf)), ("far_rank", POINTER(c_int)),
                ("far_U", POINTER(POINTER(Array))),
                ("far_V", POINTER(POINTER(Array))), ("onfly", c_int),
                ("near_D", POINTER(POINTER(Array))), ("alloc_U", c_void_p),
                ("alloc_V", c_void_p), ("alloc_D", c_void_p),
                ("alloc_type", c_char), ("nbytes", c_size_t),
                ("data_nbytes", c_size_t)]


def _arr(ptr, n, dtype=np.float64):
    if n == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def blrm_contents(Mp):
    """Python copy of a STARSH_blrm (any library): ranks, far/near block
    lists, U/V/D as numpy arrays."""
    M = Mp.contents
    F = M.format.contents
    nf, nn = F.nblocks_far, F.nblocks_near
    far = _arr(F.block_far, 2 * nf, np.int64).reshape(nf, 2) if nf else np.zeros((0, 2), np.int64)
    near = _arr(F.block_near, 2 * nn, np.int64).reshape(nn, 2) if nn else np.zeros((0, 2), np.int64)
    ranks = _arr(M.far_rank, nf, np.int64) if nf else np.zeros(0, np.int64)
    U, V, D = [], [], []
    for b in range(nf):
        u = M.far_U[b].contents
        v = M.far_V[b].contents
        m, r = u.shape[0], u.shape[1]
        n = v.shape[0]
        up = ctypes.cast(u.data, POINTER(c_double))
        vp = ctypes.cast(v.data, POINTER(c_double))
        U.append(_arr(up, m * r).reshape(r, m).T if r else np.zeros((m, 0)))
        V.append(_arr(vp, n * r).reshape(r, n).T if r else np.zeros((n, 0)))
    if M.onfly == 0:
        for b in range(nn):
            d = M.near_D[b].contents
            m, n = d.shape[0], d.shape[1]
            dp = ctypes.cast(d.data, POINTER(c_double))
            D.append(_arr(dp, m * n).reshape(n, m).T)
    R = F.row_cluster.contents
    C = F.col_cluster.contents
    return dict(far=far, near=near, ranks=ranks, U=U, V=V, D=D,
                rstart=_arr(R.start, R.nblocks, np.int64),
                rsize=_arr(R.size, R.nblocks, np.int64),
                cstart=_arr(C.start, C.nblocks, np.int64),
                csize=_arr(C.size, C.nblocks, np.int64),
                symm=F.symm.decode(), onfly=M.onfly)


class Ref:
    """The compiled reference library (unmodified STARS-H sources)."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = L = ctypes.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        P = POINTER
        for name, res, args in [
            ("starsh_set_oversample", c_int, [c_char_p]),
            ("starsh_set_backend", c_int, [c_char_p]),
            ("starsh_set_lrengine", c_int, [c_char_p]),
            ("starsh_ssdata_generate", c_int, [P(c_void_p), STARSH_int, c_int,
                                               c_double, c_double, c_double,
                                               c_int, c_double]),
            ("starsh_ssdata_get_kernel", c_int, [P(c_void_p), c_void_p, c_int]),
            ("starsh_particles_generate", c_int, [P(P(Particles)), STARSH_int,
                                                  c_int, c_int]),
            ("starsh_esdata_get_kernel", c_int, [P(c_void_p), c_void_p, c_int]),
            ("starsh_eddata_get_kernel", c_int, [P(c_void_p), c_void_p, c_int]),
            ("starsh_problem_new", c_int, [P(c_void_p), c_int, P(STARSH_int),
                                           c_char, c_char, c_void_p, c_void_p,
                                           c_void_p, c_char_p]),
            ("starsh_cluster_new_plain", c_int, [P(P(Cluster)), c_void_p,
                                                 STARSH_int, STARSH_int]),
            ("starsh_blrf_new_tlr", c_int, [P(P(Blrf)), c_void_p, c_char,
                                            P(Cluster), P(Cluster)]),
            ("starsh_blrf_free", None, [P(Blrf)]),
            ("starsh_blrm__drsdd_omp", c_int, [P(P(Blrm)), P(Blrf), c_int,
                                               c_double, c_int]),
            ("starsh_blrm__drsdd", c_int, [P(P(Blrm)), P(Blrf), c_int,
                                           c_double, c_int]),
            ("starsh_blrm__dfe_omp", c_double, [P(Blrm)]),
            ("starsh_blrm__dfe", c_double, [P(Blrm)]),
            ("starsh_blrm__dmml", c_int, [P(Blrm), c_int, c_double,
                                          P(c_double), c_int, c_double,
                                          P(c_double), c_int]),
            ("starsh_blrm_free", None, [P(Blrm)]),
            ("starsh_itersolvers__dcg_omp", c_int, [P(Blrm), c_int,
                                                    P(c_double), c_int,
                                                    P(c_double), c_int,
                                                    c_double, P(c_double)]),
        ]:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        self._keep = []

    def symbol(self, name):
        return ctypes.cast(getattr(self.lib, name), c_void_p).value

    # ---------------------------------------------------------- data
    def points(self, n, ndim, place, seed=0):
        """Reference point generator (seeded with srand)."""
        srand(seed)
        p = POINTER(Particles)()
        assert self.lib.starsh_particles_generate(byref(p), n, ndim, place) == 0
        pts = _arr(p.contents.point, n * ndim).reshape(ndim, n)
        return pts

    def spatial(self, n, ndim, kernel_type, beta, nu=0.5, noise=0.0,
                place=6, sigma=1.0, seed=0):
        srand(seed)
        data = c_void_p()
        assert self.lib.starsh_ssdata_generate(byref(data), n, ndim, beta, nu,
                                               noise, place, sigma) == 0
        kern = c_void_p()
        info = self.lib.starsh_ssdata_get_kernel(byref(kern), data, kernel_type)
        return data, kern, info

    def particles_data(self, n, ndim, place, seed=0):
        """Reference STARSH_particles (= STARSH_esdata)."""
        srand(seed)
        p = POINTER(Particles)()
        assert self.lib.starsh_particles_generate(byref(p), n, ndim, place) == 0
        return ctypes.cast(p, c_void_p)

    def eddata(self, n, ndim, place, k, diag, seed=0):
        """STARSH_eddata built around reference-generated particles (the
        reference's starsh_eddata_init does not return its structure)."""
        part = self.particles_data(n, ndim, place, seed)
        p = ctypes.cast(part, POINTER(Particles)).contents

        class ED(Structure):
            _fields_ = [("particles", Particles), ("k", c_double),
                        ("diag", c_double)]
        ed = ED(p, k, diag)
        self._keep.append(ed)
        return ctypes.cast(byref(ed), c_void_p)

    def kernel_ptr(self, name):
        return c_void_p(self.symbol(name))

    def problem(self, data, kernel, n, symm=b"N", col_data=None):
        P = c_void_p()
        shape = (STARSH_int * 2)(n, n)
        assert self.lib.starsh_problem_new(byref(P), 2, shape, symm, b"d",
                                           data, col_data or data, kernel,
                                           b"oracle") == 0
        self._keep.append(shape)
        return P

    def tlr(self, P, data, n, nb, symm=b"N"):
        C = POINTER(Cluster)()
        assert self.lib.starsh_cluster_new_plain(byref(C), data, n, nb) == 0
        F = POINTER(Blrf)()
        assert self.lib.starsh_blrf_new_tlr(byref(F), P, symm, C, C) == 0
        return C, F

    def approximate(self, F, maxrank, tol, onfly=0, oversample=10,
                    sequential=False):
        self.lib.starsh_set_oversample(str(oversample).encode())
        M = POINTER(Blrm)()
        fn = self.lib.starsh_blrm__drsdd if sequential else self.lib.starsh_blrm__drsdd_omp
        info = fn(byref(M), F, maxrank, tol, onfly)
        assert info == 0, info
        return M

    def dfe(self, M):
        return self.lib.starsh_blrm__dfe_omp(M)

    def dmml(self, M, A, alpha=1.0, beta=0.0, B=None):
        A = np.asfortranarray(A, dtype=np.float64)
        n, nrhs = A.shape
        if B is None:
            B = np.zeros_like(A)
        B = np.asfortranarray(B, dtype=np.float64).copy(order="F")
        info = self.lib.starsh_blrm__dmml(
            M, nrhs, alpha, A.ctypes.data_as(POINTER(c_double)), n, beta,
            B.ctypes.data_as(POINTER(c_double)), n)
        assert info == 0
        return B

    def cg(self, M, B, X0, tol):
        """src/itersolvers/cg.c:24-95 (starsh_itersolvers__dcg_omp):
        returns (iterations, X)."""
        B = np.asfortranarray(B, dtype=np.float64)
        n, nrhs = B.shape
        X = np.asfortranarray(X0, dtype=np.float64).copy(order="F")
        work = np.zeros(3 * n * nrhs + 3 * nrhs)
        it = self.lib.starsh_itersolvers__dcg_omp(
            M, nrhs, B.ctypes.data_as(POINTER(c_double)), n,
            X.ctypes.data_as(POINTER(c_double)), n, tol,
            work.ctypes.data_as(POINTER(c_double)))
        return it, X

    def block(self, kernel, data, irow, icol, col_data=None):
        fn = ctypes.CFUNCTYPE(None, c_int, c_int, POINTER(STARSH_int),
                              POINTER(STARSH_int), c_void_p, c_void_p,
                              c_void_p, c_int)(kernel.value if hasattr(kernel, "value") else kernel)
        irow = np.ascontiguousarray(irow, np.int64)
        icol = np.ascontiguousarray(icol, np.int64)
        m, n = len(irow), len(icol)
        out = np.zeros((n, m))
        fn(m, n, irow.ctypes.data_as(POINTER(STARSH_int)),
           icol.ctypes.data_as(POINTER(STARSH_int)), data, col_data or data,
           out.ctypes.data, m)
        return out.T


class Oracle:
    """The C restatement (oracle/starsh_oracle.c)."""

    P_COUNT = 11

    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = L = ctypes.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        D = POINTER(c_double)
        LL = POINTER(c_longlong)
        L.oracle_zsort.argtypes = [c_longlong, c_int, D]
        L.oracle_points_rand.argtypes = [c_longlong, c_int, D]
        L.oracle_points_grid.argtypes = [c_longlong, c_int, c_int, D]
        L.oracle_block.argtypes = [c_int, c_int, D, c_longlong, D, c_longlong,
                                   LL, LL, c_int, c_int, D, D, c_int]
        L.oracle_block.restype = None
        L.oracle_dsvfr.argtypes = [c_int, D, c_double]
        L.oracle_dsvfr.restype = c_int

    def points(self, n, ndim, place, seed=0):
        pts = np.zeros(n * ndim)
        srand(seed)
        ptr = pts.ctypes.data_as(POINTER(c_double))
        if place == 1:
            self.lib.oracle_points_rand(n, ndim, ptr)
        elif place in (3, 6):
            self.lib.oracle_points_grid(n, ndim, 1 if place == 6 else 0, ptr)
        else:
            raise ValueError(place)
        return pts.reshape(ndim, n)

    def block(self, family, pts_r, pts_c, irow, icol, sigma=1.0, beta=0.1,
              nu=0.5, noise=0.0, wave_k=1.0, diag=1.0, rad=1.0, reg=0.0,
              isreg=0, rbf_kind=0, zero_diag=0, aos=False):
        par = np.array([sigma, beta, nu, noise, wave_k, diag, rad, reg, isreg,
                        rbf_kind, zero_diag], np.float64)
        pr = np.ascontiguousarray(pts_r, np.float64).ravel()
        pc = np.ascontiguousarray(pts_c, np.float64).ravel()
        ndim = 3 if aos else pts_r.shape[0]
        cr = len(pr) // ndim
        cc = len(pc) // ndim
        irow = np.ascontiguousarray(irow, np.int64)
        icol = np.ascontiguousarray(icol, np.int64)
        m, n = len(irow), len(icol)
        out = np.zeros((n, m))
        D = POINTER(c_double)
        self.lib.oracle_block(family, ndim, pr.ctypes.data_as(D), cr,
                              pc.ctypes.data_as(D), cc,
                              irow.ctypes.data_as(POINTER(c_longlong)),
                              icol.ctypes.data_as(POINTER(c_longlong)), m, n,
                              par.ctypes.data_as(D), out.ctypes.data_as(D), m)
        return out.T.copy()

    def dsvfr(self, S, tol):
        S = np.ascontiguousarray(S, np.float64)
        return self.lib.oracle_dsvfr(len(S), S.ctypes.data_as(POINTER(c_double)),
                                     tol)


# ------------------------------------------------- numpy restatements


def dsvfr(S, tol):
    """src/backends/sequential/dense/dsvfr.c:16-47."""
    S = np.asarray(S, np.float64)
    total = float(np.sum(S * S))
    if total == 0:
        return 0
    budget, tail, r = total * tol * tol, S[-1] ** 2, len(S)
    while r > 1 and budget >= tail:
        r -= 1
        tail += S[r - 1] ** 2
    return r


def rsvd_tile(D, omega, tol, maxrank):
    """src/backends/sequential/dense/drsdd.c:16-93 with a given Omega:
    returns (rank or -1, U, V)."""
    Y = D @ omega
    Q, _ = np.linalg.qr(Y)
    B = Q.T @ D
    Us, S, Vt = np.linalg.svd(B, full_matrices=False)
    r = dsvfr(S, tol)
    if r > maxrank:
        return -1, None, None
    return r, Q @ Us[:, :r], (S[:r, None] * Vt[:r]).T


def dfe(contents, block_fn):
    """src/backends/sequential/blrm/dfe.c:16-134 on blrm_contents() output;
    block_fn(i, j) returns the exact dense block (i, j)."""
    norm2 = diff2 = 0.0
    symm = contents["symm"] == "S"
    for b, (i, j) in enumerate(contents["far"]):
        D = block_fn(i, j)
        w = 2.0 if symm and i != j else 1.0
        norm2 += w * np.sum(D * D)
        E = D - contents["U"][b] @ contents["V"][b].T
        diff2 += w * np.sum(E * E)
    for b, (i, j) in enumerate(contents["near"]):
        D = contents["D"][b] if contents["onfly"] == 0 else block_fn(i, j)
        w = 2.0 if symm and i != j else 1.0
        norm2 += w * np.sum(D * D)
    return np.sqrt(diff2) / np.sqrt(norm2)


def dmml(contents, block_fn, A, alpha=1.0, beta=0.0, B=None):
    """src/backends/sequential/blrm/dmml.c:16-145 on blrm_contents()."""
    A = np.asarray(A, np.float64)
    B = np.zeros_like(A) if B is None else beta * np.asarray(B, np.float64)
    rs, cs = contents["rstart"], contents["cstart"]
    rz, cz = contents["rsize"], contents["csize"]
    symm = contents["symm"] == "S"
    for b, (i, j) in enumerate(contents["far"]):
        U, V = contents["U"][b], contents["V"][b]
        B[rs[i]:rs[i] + rz[i]] += alpha * U @ (V.T @ A[cs[j]:cs[j] + cz[j]])
        if symm and i != j:
            B[cs[j]:cs[j] + cz[j]] += alpha * V @ (U.T @ A[rs[i]:rs[i] + rz[i]])
    for b, (i, j) in enumerate(contents["near"]):
        D = contents["D"][b] if contents["onfly"] == 0 else block_fn(i, j)
        B[rs[i]:rs[i] + rz[i]] += alpha * D @ A[cs[j]:cs[j] + cz[j]]
        if symm and i != j:
            B[cs[j]:cs[j] + cz[j]] += alpha * D.T @ A[rs[i]:rs[i] + rz[i]]
    return B


def matern(r, sigma, beta, nu, noise=0.0, sqrt2nu=True):
    """Matérn covariance as written in src/applications/spatial/
    kernel_matern.c:111-117 (sqrt2nu) and kernel_matern2.c:110-116, with
    K_nu and Gamma from scipy (checked against the mpmath goldens)."""
    from scipy.special import gamma, kv
    r = np.asarray(r, np.float64)
    x = r * (np.sqrt(2 * nu) / beta) if sqrt2nu else r / beta
    with np.errstate(divide="ignore", invalid="ignore"):
        v = sigma * 2.0 ** (1 - nu) / gamma(nu) * x ** nu * kv(nu, x)
    return np.where(x == 0, sigma + noise, v)
