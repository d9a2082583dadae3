/* Enumerated constants of the STARS-H C API, as implemented by the B200
 * library (libstarsh_b200.so).
 *
 * The numeric values of every pre-existing enumerator are part of the
 * binary interface shared with STARS-H 0.3.1 (include/starsh-constants.h:17-127
 * in the reference): callers compiled against either header must agree on
 * them, so they are kept unchanged.  Two values are new:
 *   STARSH_BACKEND_B200      -- the device backend of this library;
 *   STARSH_LRENGINE_RSVD_MP  -- its mixed-precision randomized-SVD engine.
 */
#ifndef STARSH_B200_CONSTANTS_H
#define STARSH_B200_CONSTANTS_H

enum STARSH_BACKEND
{
    STARSH_BACKEND_NOTSELECTED = -2,
    STARSH_BACKEND_NOTSUPPORTED = -1,
    STARSH_BACKEND_SEQUENTIAL = 0,
    STARSH_BACKEND_OPENMP = 1,
    STARSH_BACKEND_MPI = 2,
    STARSH_BACKEND_MPI_OPENMP = 3,
    STARSH_BACKEND_STARPU = 4,
    STARSH_BACKEND_MPI_STARPU = 5,
    STARSH_BACKEND_STARPU_KBLAS = 6,
    STARSH_BACKEND_STARPU_CUDA = 7,
    STARSH_BACKEND_MPI_STARPU_KBLAS = 8,
    /* One B200 GPU: tiles generated and compressed on the device. */
    STARSH_BACKEND_B200 = 9,
};

enum STARSH_LRENGINE
{
    STARSH_LRENGINE_NOTSELECTED = -2,
    STARSH_LRENGINE_NOTSUPPORTED = -1,
    STARSH_LRENGINE_SVD = 0,
    STARSH_LRENGINE_DCSVD = 1,
    STARSH_LRENGINE_RRQR = 2,
    /* On the B200 backend: randomized SVD with every step in FP64. */
    STARSH_LRENGINE_RSVD = 3,
    STARSH_LRENGINE_CROSS = 4,
    /* On the B200 backend: randomized SVD with an adaptive sketch width
     * (Gaussian columns in blocks until a posterior residual estimate
     * falls below tol); projection, small SVD and the tolerance test are
     * FP64 as in RSVD. */
    STARSH_LRENGINE_RSVD_MP = 5,
};

enum STARSH_ERRNO
{
    STARSH_SUCCESS = 0,
    STARSH_MALLOC_ERROR = 1,
    STARSH_FILE_NOT_EXIST = 2,
    STARSH_FILE_WRONG_INPUT = 3,
    STARSH_WRONG_PARAMETER = 4,
    STARSH_FPRINTF_ERROR = 5,
    STARSH_FWRITE_ERROR = 6,
    STARSH_UNKNOWN_ERROR = -1
};

enum STARSH_PROBLEM_TYPE
{
    STARSH_MINIMAL = 1,
    STARSH_RANDTLR = 2,
    STARSH_SPATIAL = 3,
    STARSH_CAUCHY = 4,
    STARSH_ELECTROSTATICS = 5,
    STARSH_ELECTRODYNAMICS = 6,
};

enum STARSH_BLRF_TYPE
{
    STARSH_TLR = 1,
};

enum STARSH_CLUSTER_TYPE
{
    STARSH_PLAIN = 1,
};

enum STARSH_FILE_TYPE
{
    STARSH_ASCII = 1,
    STARSH_BINARY = 2
};

#endif
