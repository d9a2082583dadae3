/* Internal interface between the host C files and the CUDA part of
 * libstarsh_b200.so.  Not installed; not part of the public API. */
#ifndef STARSH_B200_HOST_INTERNAL_H
#define STARSH_B200_HOST_INTERNAL_H

#include <stdio.h>
#include "starsh.h"

#ifdef __cplusplus
extern "C" {
#endif

#define B200_ERROR(...) \
    do { \
        fprintf(stderr, "STARSH ERROR: %s(): ", __func__); \
        fprintf(stderr, __VA_ARGS__); \
        fprintf(stderr, "\n"); \
    } while(0)

/* Device description of a kernel: family and its parameters, resolved on
 * the host from the kernel pointer and row_data. */
typedef struct b200_kspec
{
    int family;        /* STARSH_B200_FAMILY_*                          */
    int ndim;          /* coordinates per point                         */
    int aos;           /* 1: point-major coordinates (RBF meshes)       */
    int rbf_kind;      /* RBF basis selector (STARSH_mddata.kernel)     */
    int isreg;         /* RBF: add reg on coinciding indices            */
    int zero_mode;     /* Coulomb: 0 -> r=0 entries are 0, 1 -> `diag`  */
    double sigma, beta, nu, noise;   /* spatial statistics              */
    double matern_coef;              /* sigma*2^(1-nu)/Gamma(nu)        */
    double matern_scale;             /* sqrt(2 nu)/beta or 1/beta       */
    double wave_k, diag;             /* electrodynamics; Coulomb diag   */
    double rad, reg;                 /* RBF                             */
} b200_kspec;

/* Resolves `kernel` for the given row/col data; STARSH_WRONG_PARAMETER if
 * the kernel is not recognised (there is no host fallback). */
int b200_resolve_kernel(STARSH_kernel *kernel, void *row_data,
        b200_kspec *spec, const double **row_points, STARSH_int *row_count,
        const double **col_points, STARSH_int *col_count, void *col_data);

/* Evaluates a block on the GPU and copies it to host `result` (the host
 * STARSH_kernel entry points of this library call this). */
void b200_eval_block_host(STARSH_kernel *kernel, int nrows, int ncols,
        STARSH_int *irow, STARSH_int *icol, void *row_data, void *col_data,
        double *result, int ld);

/* Oversampling of the randomized engines (starsh_params.oversample). */
int b200_oversample(void);

#ifdef __cplusplus
}
#endif
#endif
