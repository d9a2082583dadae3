"""Approximation parity: the B200 engine against the reference's
starsh_blrm__drsdd_omp on the same STARSH_blrf, checked by the reference's
own starsh_blrm__dfe and by the set of false far-field blocks and ranks.

The reference's RSVD draws its sketch from LAPACK dlarnv and this library
from Philox, so factors are not bit-comparable; parity is on the error
(<= tol), on which blocks fail the rank test (the reference's, plus blocks
whose energy outside the sketch exceeds their tolerance, which the
reference's factors miss too) and on the ranks (within a few units)."""
import ctypes

import numpy as np
import pytest

import oracle
import starsh_b200 as sb
from harness import RefProblem, approximate_b200, as_ref_blrm


def _compare(ref, lib, kind, n, nb, maxrank, tol, oversample=10, rank_slack=3,
             engine=sb.ENGINE_FP64, **kw):
    pr = RefProblem(ref, kind, n, nb, **kw)
    Mref = ref.approximate(pr.F, maxrank, tol, oversample=oversample)
    err_ref = ref.dfe(Mref)
    cref = oracle.blrm_contents(Mref)
    pb = RefProblem(ref, kind, n, nb, **kw)
    M = approximate_b200(lib, pb.b200_format(), maxrank, tol,
                         oversample=oversample, engine=engine)
    Mr = as_ref_blrm(M)
    err = ref.dfe(Mr)
    c = oracle.blrm_contents(Mr)
    # False far-field blocks: every block the reference demotes is demoted
    # here too.  This library also demotes a block whose energy outside the
    # sketch exceeds tol^2 ||D||_F^2 (the reference's rank rule does not see
    # that energy); the reference's own factors of such a block must miss
    # the block's tolerance as well.
    near, near_ref = set(map(tuple, c["near"])), set(map(tuple, cref["near"]))
    assert near_ref <= near
    far_ref = {tuple(ij): b for b, ij in enumerate(cref["far"])}
    for ij in near - near_ref:
        b = far_ref[ij]
        D = pr.block(*ij)
        R = D - cref["U"][b] @ cref["V"][b].T
        assert np.linalg.norm(R) > 0.5 * tol * np.linalg.norm(D), ij
    far = {tuple(ij): b for b, ij in enumerate(c["far"])}
    assert set(far) == set(far_ref) - (near - near_ref)
    # Ranks within a few units; a rank further above the reference's only
    # where the reference's factors leave the block near or above its
    # tolerance (energy outside the reference's sketch).
    for ij, b in far.items():
        r, rr = c["ranks"][b], cref["ranks"][far_ref[ij]]
        assert r >= rr - rank_slack, (ij, r, rr)
        if r > rr + rank_slack:
            D = pr.block(*ij)
            R = D - cref["U"][far_ref[ij]] @ cref["V"][far_ref[ij]].T
            assert np.linalg.norm(R) > 0.5 * tol * np.linalg.norm(D), (ij, r, rr)
    assert err <= tol, (err, err_ref)
    gpu_err = lib.starsh_blrm__dfe_b200(M)
    assert abs(gpu_err - err) <= 1e-6 * err + 1e-15
    st = sb.stats(lib)
    lib.starsh_blrm_free(M)
    ref.lib.starsh_blrm_free(Mref)
    return err, err_ref, c, cref, st


@pytest.mark.gpu
def test_c1_exp2d_matches_reference(ref, lib):
    # 2-D exponential, N=3600 jittered grid, nb=400, maxrank 100, os 10,
    # tol 1e-5: the reference's own CPU-runnable configuration.
    err, err_ref, c, cref, st = _compare(ref, lib, "spatial", 3600, 400, 100,
                                         1e-5, kernel_name="exp", beta=0.1)
    assert err <= 1e-5
    assert len(c["near"]) == 9          # the 9 diagonal tiles are dense
    assert st.tiles == 81 and st.false_far == 9


@pytest.mark.gpu
def test_sqexp_tol1e7_residual_pass(ref, lib):
    # tol 1e-7 needs the second (residual) basis pass
    err, err_ref, *_ = _compare(ref, lib, "spatial", 4096, 512, 128, 1e-7,
                                oversample=16, kernel_name="sqexp", beta=0.1)
    assert err <= 1e-7


@pytest.mark.gpu
def test_ragged_last_tile(ref, lib):
    # N not a multiple of the block size: last block row/column is short
    _compare(ref, lib, "spatial", 3000, 400, 100, 1e-5, kernel_name="exp",
             beta=0.1)


@pytest.mark.gpu
def test_coulomb3d_and_sin3d(ref, lib):
    _compare(ref, lib, "coulomb", 2048, 256, 100, 1e-5, ndim=3, place=1)
    _compare(ref, lib, "sin", 2048, 256, 100, 1e-5, ndim=3, place=1,
             wave_k=20.0, diag=1.0)


@pytest.mark.gpu
def test_symmetric_format(ref, lib):
    _compare(ref, lib, "spatial", 2000, 250, 60, 1e-6, kernel_name="sqexp",
             beta=0.2, symm=b"S")


@pytest.mark.gpu
def test_onfly_and_rank_zero_tiles(ref, lib):
    # far sqexp tiles with beta=0.02 underflow to exactly zero -> rank 0
    pr = RefProblem(ref, "spatial", 2500, 250, kernel_name="sqexp", beta=0.02)
    M = approximate_b200(lib, pr.b200_format(), 50, 1e-6, onfly=1)
    c = oracle.blrm_contents(as_ref_blrm(M))
    assert (c["ranks"] == 0).any()
    assert ref.dfe(as_ref_blrm(M)) <= 1e-6
    lib.starsh_blrm_free(M)


@pytest.mark.gpu
def test_device_only_then_download(ref, lib):
    pr = RefProblem(ref, "spatial", 3600, 400, kernel_name="exp", beta=0.1)
    M = approximate_b200(lib, pr.b200_format(), 100, 1e-5, flags=0)
    assert M.contents.far_U[0].contents.data is None
    assert lib.starsh_b200_blrm_download(M) == 0
    assert ref.dfe(as_ref_blrm(M)) <= 1e-5
    lib.starsh_blrm_free(M)


@pytest.mark.gpu
def test_unknown_kernel_is_an_error(ref, lib):
    # a kernel pointer the library cannot map to a device generator
    libc = ctypes.CDLL("libc.so.6")
    pr = RefProblem(ref, "custom", 400, 100,
                    data=ref.particles_data(400, 2, 6),
                    kernel=ctypes.c_void_p(ctypes.cast(libc.abs, ctypes.c_void_p).value))
    M = ctypes.POINTER(sb.Blrm)()
    info = lib.starsh_b200_approximate(ctypes.byref(M), pr.b200_format(), 10,
                                       1e-5, 0, 0, 1)
    assert info == sb.WRONG_PARAMETER


# ------------------------------------------------------------------ mixed
# The mixed engine samples the sketch adaptively (blocks of 64 columns until
# the FP64 residual estimate is below (tol/10)^2 ||D||_F^2, at most
# maxrank + oversample columns); parity is checked exactly as above.

@pytest.mark.gpu
@pytest.mark.parametrize("case", [
    dict(kind="spatial", n=3600, nb=400, maxrank=100, tol=1e-5,
         kernel_name="exp", beta=0.1),
    dict(kind="spatial", n=4096, nb=512, maxrank=128, tol=1e-7, oversample=16,
         kernel_name="sqexp", beta=0.1),
    dict(kind="coulomb", n=2048, nb=256, maxrank=100, tol=1e-5, ndim=3, place=1),
    dict(kind="sin", n=2048, nb=256, maxrank=100, tol=1e-5, ndim=3, place=1,
         wave_k=20.0, diag=1.0),
    dict(kind="spatial", n=3000, nb=400, maxrank=100, tol=1e-5,
         kernel_name="exp", beta=0.1, symm=b"S"),
])
def test_mixed_engine_matches_reference(ref, lib, case):
    case = dict(case)
    kind, n, nb = case.pop("kind"), case.pop("n"), case.pop("nb")
    maxrank, tol = case.pop("maxrank"), case.pop("tol")
    err, err_ref, c, cref, st = _compare(ref, lib, kind, n, nb, maxrank, tol,
                                         engine=sb.ENGINE_MIXED, **case)
    assert err <= tol
    # never more sketch columns than the fixed-width reference sketch
    k = min(maxrank + case.get("oversample", 10), nb)
    assert st.sketch_flops <= 2.0 * nb * nb * k * st.tiles


@pytest.mark.gpu
@pytest.mark.parametrize("engine", [sb.ENGINE_FP64, sb.ENGINE_MIXED])
def test_high_rank_tiles_large_jacobi_classes(ref, lib, engine):
    # 512-point 3-D Coulomb tiles with maxrank 200: the diagonal and
    # neighbouring blocks keep k1 ~ 200 basis columns, whose small SVD runs
    # in the large Jacobi classes (shared memory up to 220 KB, then global
    # memory), the far blocks in the small ones
    err, err_ref, c, cref, st = _compare(ref, lib, "coulomb", 2048, 512, 200,
                                         1e-5, ndim=3, place=1, engine=engine)
    assert err <= 1e-5
    assert st.max_rank > 100


# ----------------------------------------------------------------- Matérn
# The reference evaluates Matérn only through GSL, which is absent, so its
# own Matérn kernels cannot run.  The reference's RSVD driver
# (starsh_blrm__drsdd_omp) and dfe take any kernel pointer, though: here
# they run on blocks from this library's host-callable Matérn entry point,
# whose entries are pinned to mpmath at 1e-13 (test_gpu_generate.py).  The
# B200 result is also checked against a numpy dfe over the scipy restatement
# of the reference formula (oracle.matern, itself pinned to mpmath), which
# shares no code with this library.

def _matern_kwargs(ref, lib, n, nu, beta, family="matern"):
    # reference points (jittered grid, Z-sorted) and parameters; the kernel
    # pointer is this library's Matérn
    data, _, info = ref.spatial(n, 2, 1, beta, nu)
    assert info == 0
    kern = ctypes.c_void_p(sb.kernel_symbol(
        lib, f"starsh_ssdata_block_{family}_kernel_2d"))
    return dict(data=data, kernel=kern)


def _numpy_dfe_matern(pts, c, nu, beta, sqrt2nu=True):
    def block(i, j):
        r0, rs = c["rstart"][i], c["rsize"][i]
        c0, cs = c["cstart"][j], c["csize"][j]
        P, Q = pts[:, r0:r0 + rs], pts[:, c0:c0 + cs]
        d = np.zeros((rs, cs))
        for k in range(pts.shape[0]):
            t = P[k][:, None] - Q[k][None, :]
            d = d + t * t
        return oracle.matern(np.sqrt(d), 1.0, beta, nu, sqrt2nu=sqrt2nu)
    return oracle.dfe(c, block)


@pytest.mark.gpu
@pytest.mark.parametrize("engine", [sb.ENGINE_FP64, sb.ENGINE_MIXED])
@pytest.mark.parametrize("nu,beta,tol", [(0.7, 0.05, 1e-7), (0.7, 0.05, 1e-5),
                                         (1.5, 0.05, 1e-7)])
def test_matern_matches_reference_engine(ref, lib, engine, nu, beta, tol):
    # the C2 Matérn kernel (nu = 0.7: Temme series and quadrature for K_nu;
    # nu = 1.5: the closed form) on a 64 x 64 jittered grid, 512-point tiles
    n, nb, maxrank = 4096, 512, 200
    kw = _matern_kwargs(ref, lib, n, nu, beta)
    pr = RefProblem(ref, "custom", n, nb, **kw)
    pts = pr.points()
    err, err_ref, c, cref, st = _compare(ref, lib, "custom", n, nb, maxrank,
                                         tol, oversample=16, engine=engine,
                                         **kw)
    assert err <= tol
    # an error measured without this library's generator
    err_np = _numpy_dfe_matern(pts, c, nu, beta)
    assert err_np <= tol, (err_np, err)
    assert abs(err_np - err) <= 1e-3 * err + 1e-14, (err_np, err)


@pytest.mark.gpu
def test_matern2_mixed_engine(ref, lib):
    # the second Matérn form (no sqrt(2 nu) in the scale), nu = 0.7
    n, nb, tol = 3600, 400, 1e-6
    kw = _matern_kwargs(ref, lib, n, 0.7, 0.05, family="matern2")
    pr = RefProblem(ref, "custom", n, nb, **kw)
    pts = pr.points()
    err, err_ref, c, cref, st = _compare(ref, lib, "custom", n, nb, 150, tol,
                                         oversample=16,
                                         engine=sb.ENGINE_MIXED, **kw)
    err_np = _numpy_dfe_matern(pts, c, 0.7, 0.05, sqrt2nu=False)
    assert err_np <= tol and abs(err_np - err) <= 1e-3 * err + 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("engine", [sb.ENGINE_FP64, sb.ENGINE_MIXED])
def test_block_jacobi_classes_257_to_512_rows(ref, lib, engine, tmp_path,
                                              monkeypatch):
    # 1024-point 3-D Coulomb tiles with maxrank 600 (sketch width 610):
    # the far blocks keep 257-512 basis columns, so their small SVD runs in
    # the block one-sided Jacobi classes for 257-288, 289-320 and 321-512
    # rows (pairs of column blocks in shared memory), checked against the
    # reference's dgesdd-based engine on the same format
    log = tmp_path / "tiles.log"
    monkeypatch.setenv("STARSH_B200_TILE_LOG", str(log))
    err, err_ref, c, cref, st = _compare(ref, lib, "coulomb", 4096, 1024, 600,
                                         1e-5, ndim=3, place=1, engine=engine)
    assert err <= 1e-5
    # m n cols k1 k2 sweeps rank status per tile
    rows = np.loadtxt(log, dtype=np.int64, ndmin=2)
    k1 = rows[rows[:, 4] > 0, 3]
    assert ((k1 > 256) & (k1 <= 288)).any()
    assert ((k1 > 288) & (k1 <= 320)).any()
    assert ((k1 > 320) & (k1 <= 512)).any()
    assert st.max_rank > 200


@pytest.mark.gpu
def test_streamed_jacobi_class_above_512_rows(ref, lib, tmp_path, monkeypatch):
    # 3-D sin(kr)/r with k = 40 at tol 1e-8, 1024-point tiles, maxrank 1000:
    # the far blocks keep more than 512 basis columns (ranks 560-590), whose
    # small SVD runs in the streamed one-sided Jacobi form
    log = tmp_path / "tiles.log"
    monkeypatch.setenv("STARSH_B200_TILE_LOG", str(log))
    err, err_ref, c, cref, st = _compare(ref, lib, "sin", 4096, 1024, 1000,
                                         1e-8, ndim=3, place=1, wave_k=40.0,
                                         diag=1.0, engine=sb.ENGINE_MIXED)
    assert err <= 1e-8
    rows = np.loadtxt(log, dtype=np.int64, ndmin=2)
    assert (rows[rows[:, 4] > 0, 3] > 512).any()
    assert st.max_rank > 512
