"""Generates the golden fixtures in this directory (run in a container where
the reference sources exist; the fixtures travel, the reference does not).

    python tests/golden/make_golden.py

* reference.npz -- outputs of the compiled reference library
  (oracle/_ref/libstarsh_ref.so, built by oracle/Makefile from the reference
  sources): point sets of its generators, kernel blocks of its kernel
  functions, starsh_dense_dsvfr on crafted spectra, and the C1 configuration
  (2-D exp, N=3600, nb=400, maxrank 100, oversample 10, tol 1e-5) through
  starsh_blrm__drsdd_omp, starsh_blrm__dfe_omp and starsh_blrm__dmml.
* matern.npz -- Matérn and Matérn2 entries evaluated with mpmath at 40
  digits (besselk, gamma) on FP64 distances computed as the reference does;
  the reference needs GSL for these kernels and GSL is not available.
"""
import ctypes
import hashlib
import os
import sys
from ctypes import POINTER, c_double, c_int

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def fp64_dist(pts, rows, cols):
    """Squared distance summed dimension by dimension as the reference
    kernels do (tmp = a - b; dist += tmp*tmp)."""
    d = np.zeros((len(rows), len(cols)))
    for k in range(pts.shape[0]):
        t = pts[k][rows][:, None] - pts[k][cols][None, :]
        d = d + t * t
    return d


def make_reference(ref):
    out = {}
    # point generators (seeded like testing/spatial.c:53)
    for name, n, ndim, place in [("q1_2d_3600", 3600, 2, 6),
                                 ("rand_3d_4096", 4096, 3, 1),
                                 ("uniform_2d_100", 100, 2, 3),
                                 ("q1_3d_1000", 1000, 3, 6)]:
        p = ref.points(n, ndim, place, seed=0)
        out[f"pts_{name}_sha"] = np.array(sha(p))
        out[f"pts_{name}_head"] = p[:, :16].copy()
    # kernel blocks
    rng = np.random.default_rng(2024)
    rows = rng.integers(0, 600, 20)
    cols = rng.integers(0, 600, 30)
    cols[:4] = rows[:4]
    out["blk_rows"], out["blk_cols"] = rows, cols
    data, kern, _ = ref.spatial(600, 2, 1, 0.1, 0.5, 0.25, 6, seed=1)
    out["blk_exp2d"] = ref.block(kern, data, rows, cols)
    data, kern, _ = ref.spatial(600, 3, 2, 0.2, 0.5, 0.0, 1, seed=2)
    out["blk_sqexp3d"] = ref.block(kern, data, rows, cols)
    data = ref.particles_data(600, 3, 1, seed=3)
    out["blk_coulomb3d"] = ref.block(
        ref.kernel_ptr("starsh_esdata_block_coulomb_potential_kernel_3d"),
        data, rows, cols)
    data = ref.eddata(600, 3, 1, 20.0, 1.0, seed=4)
    out["blk_sin3d"] = ref.block(
        ref.kernel_ptr("starsh_eddata_block_sin_kernel_3d"), data, rows, cols)
    # dsvfr on crafted spectra
    dsvfr = ref.lib.starsh_dense_dsvfr
    dsvfr.restype = c_int
    dsvfr.argtypes = [c_int, POINTER(c_double), c_double]
    spectra = [np.logspace(0, -12, 40), np.ones(7), np.zeros(5),
               np.array([1.0]), np.array([3.0, 4.0, 1e-9, 1e-10]),
               np.exp(-np.arange(60) / 3.0)]
    kats = []
    for s in spectra:
        s = np.ascontiguousarray(s, np.float64)
        for tol in (1e-1, 1e-3, 1e-5, 1e-7, 0.0):
            kats.append((len(kats), tol, dsvfr(len(s), s.ctypes.data_as(
                POINTER(c_double)), tol)))
        out[f"dsvfr_S{len(kats)//5 - 1}"] = s
    out["dsvfr_kats"] = np.array(kats, dtype=np.float64)
    # C1 through the reference OpenMP engine
    from harness import RefProblem
    pr = RefProblem(ref, "spatial", 3600, 400, kernel_name="exp", beta=0.1)
    M = ref.approximate(pr.F, 100, 1e-5, oversample=10)
    c = oracle.blrm_contents(M)
    out["c1_ranks"] = c["ranks"]
    out["c1_far"] = c["far"]
    out["c1_near"] = c["near"]
    out["c1_dfe"] = np.array(ref.dfe(M))
    A = np.random.default_rng(7).standard_normal((3600, 3))
    out["c1_rhs"] = A
    out["c1_dmml"] = ref.dmml(M, A)
    return out


def make_matern(ref):
    import mpmath as mp
    mp.mp.dps = 40
    out = {}
    cases = [(2, 0.7, 0.05, 1.0, 0.0, 3), (2, 1.5, 0.1, 1.3, 0.1, 3),
             (2, 0.5, 0.1, 1.0, 0.0, 3), (3, 2.5, 0.2, 0.7, 0.0, 3),
             (2, 0.7, 0.1, 1.0, 0.0, 4), (1, 0.3, 0.05, 1.0, 0.0, 4)]
    rng = np.random.default_rng(99)
    for ci, (ndim, nu, beta, sigma, noise, fam) in enumerate(cases):
        pts = ref.points(256, ndim, 6, seed=ci)
        rows = rng.integers(0, 256, 24)
        cols = rng.integers(0, 256, 31)
        cols[:3] = rows[:3]
        d2 = fp64_dist(pts, rows, cols)
        r = np.sqrt(d2)
        x = r * (np.sqrt(2 * nu) / beta) if fam == 3 else r / beta
        coef = mp.mpf(sigma) * mp.power(2, 1 - mp.mpf(nu)) / mp.gamma(nu)
        want = np.empty_like(x)
        for idx, xv in np.ndenumerate(x):
            if xv == 0:
                want[idx] = sigma + noise
            else:
                xm = mp.mpf(float(xv))
                want[idx] = float(coef * mp.power(xm, nu) * mp.besselk(nu, xm))
        out[f"pts{ci}"] = pts
        out[f"rows{ci}"] = rows
        out[f"cols{ci}"] = cols
        out[f"par{ci}"] = np.array([nu, beta, sigma, noise])
        out[f"fam{ci}"] = np.array(fam)
        out[f"want{ci}"] = want
    out["ncases"] = np.array(len(cases))
    return out


if __name__ == "__main__":
    oracle.build()
    ref = oracle.Ref()
    np.savez_compressed(os.path.join(HERE, "reference.npz"), **make_reference(ref))
    np.savez_compressed(os.path.join(HERE, "matern.npz"), **make_matern(ref))
    print("written", os.listdir(HERE))
