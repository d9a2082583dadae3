"""ctypes bindings of libstarsh_b200.so.

The structure layouts below are those of include/starsh*.h (the STARS-H
0.3.1 binary interface).  `load()` opens the library that
stars-h_b200/build.py produces; there is no pure-Python implementation of
any computation here, only argument marshalling.
"""
import ctypes
import os
from ctypes import (POINTER, Structure, c_char, c_char_p, c_double, c_int,
                    c_longlong, c_size_t, c_ssize_t, c_void_p)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "libstarsh_b200.so")

STARSH_int = c_ssize_t
KERNEL = ctypes.CFUNCTYPE(None, c_int, c_int, POINTER(STARSH_int),
                          POINTER(STARSH_int), c_void_p, c_void_p, c_void_p,
                          c_int)

# enum values (include/starsh-constants.h and the application headers)
SUCCESS, MALLOC_ERROR, WRONG_PARAMETER, UNKNOWN_ERROR = 0, 1, 4, -1
SPATIAL, ELECTROSTATICS, ELECTRODYNAMICS = 3, 5, 6
EXP, SQREXP, MATERN, MATERN2 = 1, 2, 3, 4
COULOMB = 1
SIN, COS = 1, 2
PLACE_RAND, PLACE_UNIFORM, PLACE_QUASIUNIFORM1 = 1, 3, 6
SPATIAL_NDIM, SPATIAL_BETA, SPATIAL_NU, SPATIAL_NOISE, SPATIAL_PLACE, \
    SPATIAL_SIGMA = 1, 2, 3, 4, 5, 6
ES_NDIM, ES_PLACE = 1, 2
ED_NDIM, ED_K, ED_DIAG, ED_PLACE = 1, 2, 3, 4
ENGINE_FP64, ENGINE_MIXED = 0, 1
FLAG_HOST_MIRROR = 1
FAMILY = dict(exp=1, sqrexp=2, matern=3, matern2=4, coulomb=5, sin=6, cos=7,
              rbf=8)


class Array(Structure):
    _fields_ = [("ndim", c_int), ("shape", POINTER(c_int)),
                ("stride", POINTER(c_ssize_t)), ("order", c_char),
                ("size", c_size_t), ("dtype", c_char),
                ("dtype_size", c_size_t), ("nbytes", c_size_t),
                ("data_nbytes", c_size_t), ("data", c_void_p)]


class Problem(Structure):
    _fields_ = [("ndim", c_int), ("shape", POINTER(STARSH_int)),
                ("symm", c_char), ("dtype", c_char),
                ("dtype_size", c_size_t), ("entry_size", c_size_t),
                ("row_data", c_void_p), ("col_data", c_void_p),
                ("kernel", c_void_p), ("name", c_char_p)]


class Cluster(Structure):
    _fields_ = [("data", c_void_p), ("ndata", STARSH_int),
                ("pivot", POINTER(STARSH_int)), ("nblocks", STARSH_int),
                ("nlevels", STARSH_int), ("level", POINTER(STARSH_int)),
                ("start", POINTER(STARSH_int)), ("size", POINTER(STARSH_int)),
                ("parent", POINTER(STARSH_int)),
                ("child_start", POINTER(STARSH_int)),
                ("child", POINTER(STARSH_int)), ("type", c_int)]


class Blrf(Structure):
    _fields_ = [("problem", POINTER(Problem)), ("symm", c_char),
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
                ("block_far_local", POINTER(STARSH_int)),
                ("nblocks_near", STARSH_int),
                ("block_near", POINTER(STARSH_int)),
                ("brow_near_start", POINTER(STARSH_int)),
                ("brow_near", POINTER(STARSH_int)),
                ("bcol_near_start", POINTER(STARSH_int)),
                ("bcol_near", POINTER(STARSH_int)),
                ("nblocks_near_local", STARSH_int),
                ("block_near_local", POINTER(STARSH_int)), ("type", c_int)]


class Blrm(Structure):
    _fields_ = [("format", POINTER(Blrf)), ("far_rank", POINTER(c_int)),
                ("far_U", POINTER(POINTER(Array))),
                ("far_V", POINTER(POINTER(Array))), ("onfly", c_int),
                ("near_D", POINTER(POINTER(Array))), ("alloc_U", c_void_p),
                ("alloc_V", c_void_p), ("alloc_D", c_void_p),
                ("alloc_type", c_char), ("nbytes", c_size_t),
                ("data_nbytes", c_size_t)]


class Particles(Structure):
    _fields_ = [("count", STARSH_int), ("ndim", c_int),
                ("point", POINTER(c_double))]


class SSData(Structure):
    _fields_ = [("particles", Particles), ("beta", c_double),
                ("nu", c_double), ("noise", c_double), ("sigma", c_double),
                ("nu2", c_double), ("sigma2", c_double), ("corr", c_double)]


class EDData(Structure):
    _fields_ = [("particles", Particles), ("k", c_double),
                ("diag", c_double)]


class MDData(Structure):
    _fields_ = [("particles", Particles), ("reg", c_double),
                ("kernel", c_int), ("numobj", c_int), ("isreg", c_int),
                ("rad", c_double), ("denst", c_double),
                ("mesh_points", c_int), ("mordering", c_int)]


class Stats(Structure):
    _fields_ = [("total_ms", c_double), ("device_ms", c_double),
                ("sketch_ms", c_double), ("project_ms", c_double),
                ("sketch_flops", c_double), ("project_flops", c_double),
                ("tiles", c_longlong), ("false_far", c_longlong),
                ("entries", c_longlong), ("kernel_launches", c_longlong),
                ("rank_sum", c_longlong), ("max_rank", c_int),
                ("h2d_bytes", c_longlong), ("d2h_bytes", c_longlong),
                ("batches", c_longlong), ("sketch_launches", c_longlong),
                ("gen_ms", c_double), ("basis_ms", c_double),
                ("svd_ms", c_double), ("output_ms", c_double),
                ("sketch_bytes", c_double), ("sketch_int8", c_int),
                ("fused_ms", c_double), ("fused_launches", c_longlong),
                ("fused_bytes", c_double), ("resketch_tiles", c_longlong),
                ("mirror_wait_ms", c_double), ("finish_ms", c_double)]


class ServerStats(Structure):
    _fields_ = [("submitted", c_longlong), ("completed", c_longlong),
                ("failed", c_longlong), ("groups", c_longlong),
                ("entries", c_longlong), ("busy_ms", c_double),
                ("resident_bytes", c_double),
                ("peak_resident_bytes", c_double),
                ("queue_ms", c_double), ("approx_ms", c_double),
                ("products_ms", c_double)]


def _proto(lib):
    P = POINTER
    sig = {
        "starsh_init": (c_int, []),
        "starsh_set_backend": (c_int, [c_char_p]),
        "starsh_set_lrengine": (c_int, [c_char_p]),
        "starsh_set_oversample": (c_int, [c_char_p]),
        "starsh_problem_new": (c_int, [P(P(Problem)), c_int, P(STARSH_int),
                                       c_char, c_char, c_void_p, c_void_p,
                                       c_void_p, c_char_p]),
        "starsh_problem_free": (None, [P(Problem)]),
        "starsh_cluster_new_plain": (c_int, [P(P(Cluster)), c_void_p,
                                             STARSH_int, STARSH_int]),
        "starsh_cluster_free": (None, [P(Cluster)]),
        "starsh_blrf_new_tlr": (c_int, [P(P(Blrf)), P(Problem), c_char,
                                        P(Cluster), P(Cluster)]),
        "starsh_blrf_new_from_coo": (c_int, [P(P(Blrf)), P(Problem), c_char,
                                             P(Cluster), P(Cluster),
                                             STARSH_int, P(STARSH_int),
                                             STARSH_int, P(STARSH_int),
                                             c_int]),
        "starsh_blrf_free": (None, [P(Blrf)]),
        "starsh_blrm_free": (None, [P(Blrm)]),
        "starsh_blrm__drsdd_b200": (c_int, [P(P(Blrm)), P(Blrf), c_int,
                                            c_double, c_int]),
        "starsh_blrm__drsdd_b200_mp": (c_int, [P(P(Blrm)), P(Blrf), c_int,
                                               c_double, c_int]),
        "starsh_b200_approximate": (c_int, [P(P(Blrm)), P(Blrf), c_int,
                                            c_double, c_int, c_int, c_int]),
        "starsh_b200_approximate_batch": (c_int, [c_int, P(P(Blrm)),
                                                  P(P(Blrf)), P(c_int),
                                                  P(c_double), P(c_int),
                                                  c_int, c_int]),
        "starsh_b200_server_new": (c_int, [P(c_void_p), c_double, c_int,
                                           c_int]),
        "starsh_b200_server_submit": (c_int, [c_void_p, P(Blrf), c_int,
                                              c_double, c_int, c_void_p, c_int,
                                              c_void_p, c_int, c_int,
                                              P(c_longlong)]),
        "starsh_b200_server_wait": (c_int, [c_void_p, c_longlong, P(P(Blrm)),
                                            P(c_double)]),
        "starsh_b200_server_release": (c_int, [c_void_p, P(Blrm)]),
        "starsh_b200_server_pause": (c_int, [c_void_p, c_int]),
        "starsh_b200_server_get_stats": (c_int, [c_void_p, P(ServerStats)]),
        "starsh_b200_server_free": (c_int, [c_void_p]),
        "starsh_itersolvers__dcg_b200": (c_int, [P(Blrm), c_int, c_void_p,
                                                 c_int, c_void_p, c_int,
                                                 c_double, c_void_p]),
        "starsh_b200_dcg_device": (c_int, [P(Blrm), c_int, c_void_p, c_int,
                                           c_void_p, c_int, c_double, c_int,
                                           c_void_p, P(c_int)]),
        "starsh_b200_blrm_download": (c_int, [P(Blrm)]),
        "starsh_b200_blrm_write_to_file": (c_int, [P(Blrm), c_char_p]),
        "starsh_b200_blrm_write_to_file_pointer": (c_int, [P(Blrm), c_void_p]),
        "starsh_b200_blrm_serialize": (c_int, [P(Blrm), c_void_p, c_size_t,
                                               P(c_size_t)]),
        "starsh_b200_blrm_read_from_file": (c_int, [P(P(Blrm)), c_void_p,
                                                    c_char_p]),
        "starsh_b200_blrm_read_from_file_pointer": (c_int, [P(P(Blrm)),
                                                            c_void_p,
                                                            c_void_p]),
        "starsh_b200_blrm_deserialize": (c_int, [P(P(Blrm)), c_void_p,
                                                 c_void_p, c_size_t]),
        "starsh_b200_blrm_free_read": (None, [P(Blrm)]),
        "starsh_b200_blrm_release": (None, [P(Blrm)]),
        "starsh_b200_blrm_dmml_device": (c_int, [P(Blrm), c_int, c_double,
                                                 c_void_p, c_int, c_double,
                                                 c_void_p, c_int, c_void_p]),
        "starsh_blrm__dmml_b200": (c_int, [P(Blrm), c_int, c_double,
                                           P(c_double), c_int, c_double,
                                           P(c_double), c_int]),
        "starsh_blrm__dmml": (c_int, [P(Blrm), c_int, c_double, P(c_double),
                                      c_int, c_double, P(c_double), c_int]),
        "starsh_blrm__dfe_b200": (c_double, [P(Blrm)]),
        "starsh_b200_blrm_dfe_sums": (c_int, [P(Blrm), P(c_double),
                                              P(c_double)]),
        "starsh_blrm__dfe": (c_double, [P(Blrm)]),
        "starsh_b200_kernel_register": (c_int, [c_void_p, c_int, c_double]),
        "starsh_b200_kernel_family": (c_int, [c_void_p, P(c_int)]),
        "starsh_b200_autotune_tile": (c_int, [P(Problem), c_int, P(c_int),
                                              P(c_int), c_double, c_int,
                                              P(c_int), P(c_double)]),
        "starsh_b200_autotune_clear": (None, []),
        "starsh_b200_get_stats": (c_int, [P(Stats)]),
        "starsh_b200_set_device": (c_int, [c_int]),
        "starsh_b200_dense_rsvd_noalloc": (c_int, [c_void_p, c_int, c_int,
                                                   c_int, c_int, c_int,
                                                   c_double, c_void_p,
                                                   c_void_p, c_void_p,
                                                   c_void_p]),
        "starsh_b200_stream": (c_void_p, []),
        "starsh_b200_last_error": (c_char_p, []),
        "starsh_ssdata_init": (c_int, [P(P(SSData)), STARSH_int, c_int,
                                       P(c_double), c_double, c_double,
                                       c_double, c_double]),
        "starsh_ssdata_generate": (c_int, [P(P(SSData)), STARSH_int, c_int,
                                           c_double, c_double, c_double,
                                           c_int, c_double]),
        "starsh_ssdata_get_kernel": (c_int, [P(c_void_p), P(SSData), c_int]),
        "starsh_ssdata_free": (None, [P(SSData)]),
        "starsh_esdata_init": (c_int, [P(P(Particles)), STARSH_int, c_int,
                                       P(c_double)]),
        "starsh_esdata_get_kernel": (c_int, [P(c_void_p), P(Particles),
                                             c_int]),
        "starsh_eddata_init": (c_int, [P(P(EDData)), STARSH_int, c_int,
                                       P(c_double), c_double, c_double]),
        "starsh_eddata_get_kernel": (c_int, [P(c_void_p), P(EDData), c_int]),
        "starsh_mddata_init": (c_int, [P(P(MDData)), STARSH_int, P(c_double),
                                       c_int, c_int, c_int, c_double,
                                       c_double, c_double]),
        "starsh_particles_generate": (c_int, [P(P(Particles)), STARSH_int,
                                              c_int, c_int]),
        "starsh_particles_init": (c_int, [P(P(Particles)), STARSH_int, c_int,
                                          P(c_double)]),
        "starsh_particles_zsort_inplace": (c_int, [P(Particles)]),
        "starsh_particles_free": (None, [P(Particles)]),
        "starsh_particles_read_from_file": (c_int, [P(P(Particles)), c_char_p,
                                                    c_int]),
        "starsh_particles_read_from_file_pointer": (c_int, [P(P(Particles)),
                                                            c_void_p, c_int]),
        "starsh_particles_write_to_file": (c_int, [P(Particles), c_char_p,
                                                   c_int]),
        "starsh_particles_write_to_file_pointer": (c_int, [P(Particles),
                                                           c_void_p, c_int]),
        "starsh_blrm_get_block": (c_int, [P(Blrm), STARSH_int, STARSH_int,
                                          P(c_int), P(c_int), P(c_void_p),
                                          P(c_void_p), P(c_void_p)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def load(path=None):
    """Opens libstarsh_b200.so (RTLD_LOCAL) and declares its prototypes.

    Raises OSError when the library has not been built: there is no
    fallback implementation."""
    global _lib
    if _lib is None or path is not None:
        lib = ctypes.CDLL(path or LIB_PATH, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        _lib = _proto(lib)
    return _lib


def stats(lib=None):
    s = Stats()
    (lib or load()).starsh_b200_get_stats(ctypes.byref(s))
    return s


def kernel_symbol(lib, name):
    """Address of an exported kernel function (e.g.
    'starsh_ssdata_block_exp_kernel_2d')."""
    return ctypes.cast(getattr(lib, name), c_void_p).value
