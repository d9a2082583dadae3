"""Problem construction shared by the tests: the same problem built through
the reference library (the oracle side) and handed to the B200 entry points
(the drop-in side)."""
import ctypes
from ctypes import POINTER, byref, c_double, c_int, c_void_p

import numpy as np

import oracle


class RefProblem:
    """A TLR problem whose structures come from the reference library."""

    def __init__(self, ref, kind, n, nb, ndim=2, place=6, seed=0, beta=0.1,
                 nu=0.5, noise=0.0, wave_k=20.0, diag=1.0, symm=b"N",
                 kernel_name=None, data=None, kernel=None):
        self.ref, self.n, self.nb = ref, n, nb
        if kind == "spatial":
            ktype = {"exp": 1, "sqexp": 2, "matern": 3, "matern2": 4}[kernel_name]
            data, kern, info = ref.spatial(n, ndim, ktype, beta, nu, noise,
                                           place, seed=seed)
            assert info == 0
        elif kind == "coulomb":
            data = ref.particles_data(n, ndim, place, seed)
            kern = ref.kernel_ptr(kernel_name or
                                  f"starsh_esdata_block_coulomb_potential_kernel_{ndim}d")
        elif kind in ("sin", "cos"):
            data = ref.eddata(n, ndim, place, wave_k, diag, seed)
            kern = ref.kernel_ptr(f"starsh_eddata_block_{kind}_kernel_{ndim}d")
        elif kind == "custom":
            kern = kernel
        else:
            raise ValueError(kind)
        self.data, self.kernel = data, kern
        self.P = ref.problem(data, kern, n, symm=symm)
        self.C, self.F = ref.tlr(self.P, data, n, nb, symm=symm)
        self.symm = symm

    def points(self):
        p = ctypes.cast(self.data, POINTER(oracle.Particles)).contents
        return np.ctypeslib.as_array(p.point, shape=(p.ndim * p.count,)).reshape(
            p.ndim, p.count).copy()

    def block(self, i, j):
        R = self.C.contents
        r0, rs = R.start[i], R.size[i]
        c0, cs = R.start[j], R.size[j]
        return self.ref.block(self.kernel, self.data, np.arange(r0, r0 + rs),
                              np.arange(c0, c0 + cs))

    def b200_format(self):
        import starsh_b200 as sb
        return ctypes.cast(self.F, POINTER(sb.Blrf))


def approximate_b200(lib, fmt, maxrank, tol, onfly=0, engine=0, flags=1,
                     oversample=10):
    import starsh_b200 as sb
    lib.starsh_set_oversample(str(oversample).encode())
    M = POINTER(sb.Blrm)()
    info = lib.starsh_b200_approximate(byref(M), fmt, maxrank, tol, onfly,
                                       engine, flags)
    assert info == 0, (info, lib.starsh_b200_last_error())
    return M


def as_ref_blrm(M):
    return ctypes.cast(M, POINTER(oracle.Blrm))
