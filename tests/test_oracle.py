"""The oracle pinned: its C restatement and numpy restatements against the
compiled reference and the committed golden vectors (CPU only)."""
import hashlib
import os

import numpy as np
import pytest

import oracle
from harness import RefProblem

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLDEN, "reference.npz"))


@pytest.mark.parametrize("name,n,ndim,place", [
    ("q1_2d_3600", 3600, 2, 6), ("rand_3d_4096", 4096, 3, 1),
    ("uniform_2d_100", 100, 2, 3), ("q1_3d_1000", 1000, 3, 6)])
def test_points_bit_exact(orc, gold, name, n, ndim, place):
    p = orc.points(n, ndim, place, seed=0)
    assert sha(p) == str(gold[f"pts_{name}_sha"])
    assert np.array_equal(p[:, :16], gold[f"pts_{name}_head"])


def test_points_match_live_reference(orc, ref):
    for n, ndim, place in [(777, 2, 6), (1000, 3, 1), (64, 4, 3)]:
        assert np.array_equal(orc.points(n, ndim, place, seed=5),
                              ref.points(n, ndim, place, seed=5))


def test_kernel_blocks_against_golden(orc, ref, gold):
    rows, cols = gold["blk_rows"], gold["blk_cols"]
    cases = [("blk_exp2d", 1, dict(beta=0.1, noise=0.25), (600, 2, 6, 1)),
             ("blk_sqexp3d", 2, dict(beta=0.2), (600, 3, 1, 2)),
             ("blk_coulomb3d", 5, dict(), (600, 3, 1, 3)),
             ("blk_sin3d", 6, dict(wave_k=20.0, diag=1.0), (600, 3, 1, 4))]
    for key, fam, par, (n, ndim, place, seed) in cases:
        pts = ref.points(n, ndim, place, seed=seed)
        got = orc.block(fam, pts, pts, rows, cols, **par)
        want = gold[key]
        assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300)) <= 1e-15, key


def test_dsvfr_kats(orc, gold):
    for idx, tol, want in gold["dsvfr_kats"]:
        S = gold[f"dsvfr_S{int(idx) // 5}"]
        assert orc.dsvfr(S, tol) == int(want)
        assert oracle.dsvfr(S, tol) == int(want)


def test_matern_restatement_against_mpmath():
    g = np.load(os.path.join(GOLDEN, "matern.npz"))
    for c in range(int(g["ncases"])):
        pts = g[f"pts{c}"]
        rows, cols = g[f"rows{c}"], g[f"cols{c}"]
        nu, beta, sigma, noise = g[f"par{c}"]
        d = np.zeros((len(rows), len(cols)))
        for k in range(pts.shape[0]):
            t = pts[k][rows][:, None] - pts[k][cols][None, :]
            d = d + t * t
        got = oracle.matern(np.sqrt(d), sigma, beta, nu, noise,
                            sqrt2nu=int(g[f"fam{c}"]) == 3)
        want = g[f"want{c}"]
        assert np.max(np.abs(got - want) / np.abs(want)) < 1e-12


def test_c1_reference_is_reproducible(ref, gold):
    pr = RefProblem(ref, "spatial", 3600, 400, kernel_name="exp", beta=0.1)
    M = ref.approximate(pr.F, 100, 1e-5, oversample=10)
    c = oracle.blrm_contents(M)
    assert np.array_equal(c["ranks"], gold["c1_ranks"])
    assert np.array_equal(c["near"], gold["c1_near"])
    assert abs(ref.dfe(M) - float(gold["c1_dfe"])) <= 1e-12 * float(gold["c1_dfe"])
    # numpy restatements of dfe and dmml agree with the reference
    assert abs(oracle.dfe(c, pr.block) - float(gold["c1_dfe"])) <= 1e-9 * float(gold["c1_dfe"])
    B = oracle.dmml(c, pr.block, gold["c1_rhs"])
    assert np.allclose(B, gold["c1_dmml"], rtol=1e-12, atol=1e-12 * np.abs(B).max())
    assert np.allclose(ref.dmml(M, gold["c1_rhs"]), gold["c1_dmml"], rtol=1e-13,
                       atol=1e-13 * np.abs(B).max())
    ref.lib.starsh_blrm_free(M)


def test_rsvd_restatement_matches_reference_rank_rule(ref):
    # per-tile RSVD restated in numpy: same rank decision as dsvfr on the
    # SVD of the projected block, error within tol on a low-rank tile
    pr = RefProblem(ref, "spatial", 3600, 400, kernel_name="exp", beta=0.1)
    D = pr.block(0, 2)
    om = np.random.default_rng(0).standard_normal((400, 110))
    r, U, V = oracle.rsvd_tile(D, om, 1e-5, 100)
    assert 0 < r <= 100
    assert np.linalg.norm(D - U @ V.T) <= 1.2e-5 * np.linalg.norm(D)
