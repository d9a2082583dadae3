/* Public C API of the B200 TLR approximation library (libstarsh_b200.so).
 *
 * This is the subset of the STARS-H 0.3.1 API that lies on the tile
 * low-rank approximation path: environment/backend selection, the
 * matrix-free problem, plain clustering, the TLR block format, the
 * block-low-rank matrix container, approximation, TLR-by-dense product and
 * the Frobenius error measure.  Type layouts and function signatures are the
 * binary interface of the reference (include/starsh.h:37-686), so that
 *   - code written against STARS-H compiles and links against this library
 *     unchanged and switches to the GPU by STARSH_BACKEND=B200, and
 *   - structures built by the reference library itself can be passed to the
 *     B200 entry points declared in starsh-b200.h.
 * The B200-specific entry points are declared in starsh-b200.h.
 */
#ifndef STARSH_B200_STARSH_H
#define STARSH_B200_STARSH_H

#include <sys/types.h>
#include <stdarg.h>
#include <stddef.h>
#include "starsh-constants.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- params */

/* Backend, low-rank engine and oversampling chosen by starsh_init()
 * (reference: include/starsh.h:39-48, src/control/init.c:26-175). */
struct starsh_params
{
    enum STARSH_BACKEND backend;
    enum STARSH_LRENGINE lrengine;
    int oversample;
};
extern struct starsh_params starsh_params;

/* Reads STARSH_BACKEND, STARSH_LRENGINE and STARSH_OVERSAMPLE.  An invalid
 * or unsupported value falls back to the default (B200, RSVD, 10).
 * Reference: src/control/init.c:26-67. */
int starsh_init(void);
/* Each takes the bare value ("B200", "RSVD_MP", "16"); NULL selects the
 * default.  Reference: src/control/init.c:69-175. */
int starsh_set_backend(const char *string);
int starsh_set_lrengine(const char *string);
int starsh_set_oversample(const char *string);

/* --------------------------------------------------------------- typedefs */

typedef ssize_t STARSH_int;

/* Fills the nrows x ncols column-major block (leading dimension ld) on the
 * intersection of rows irow[] and columns icol[].  Reference:
 * include/starsh.h:68-70. */
typedef void STARSH_kernel(int nrows, int ncols, STARSH_int *irow,
        STARSH_int *icol, void *row_data, void *col_data, void *result,
        int ld);

typedef struct array Array;
typedef struct starsh_problem STARSH_problem;
typedef struct starsh_cluster STARSH_cluster;
typedef struct starsh_blrf STARSH_blrf;
typedef struct starsh_blrm STARSH_blrm;

int starsh_application(void **data, STARSH_kernel **kernel, STARSH_int count,
        char dtype, int problem_type, int kernel_type, ...);

/* ------------------------------------------------------------------ array */

/* N-dimensional array view (reference: include/starsh.h:120-151). */
struct array
{
    int ndim;
    int *shape;
    ssize_t *stride;
    char order;
    size_t size;
    char dtype;
    size_t dtype_size;
    size_t nbytes;
    size_t data_nbytes;
    void *data;
};

int array_from_buffer(Array **A, int ndim, int *shape, char dtype, char order,
        void *buffer);
int array_new(Array **A, int ndim, int *shape, char dtype, char order);
void array_free(Array *A);

/* ---------------------------------------------------------------- problem */

/* Matrix-free kernel matrix (reference: include/starsh.h:186-237). */
struct starsh_problem
{
    int ndim;
    STARSH_int *shape;
    char symm;
    char dtype;
    size_t dtype_size;
    size_t entry_size;
    void *row_data;
    void *col_data;
    STARSH_kernel *kernel;
    char *name;
};
int starsh_problem_new(STARSH_problem **problem, int ndim, STARSH_int *shape,
        char symm, char dtype, void *row_data, void *col_data,
        STARSH_kernel *kernel, char *name);
void starsh_problem_free(STARSH_problem *problem);
void starsh_problem_info(STARSH_problem *problem);

/* ---------------------------------------------------------------- cluster */

/* Clusterisation of rows or columns (reference: include/starsh.h:263-319).*/
struct starsh_cluster
{
    void *data;
    STARSH_int ndata;
    STARSH_int *pivot;
    STARSH_int nblocks;
    STARSH_int nlevels;
    STARSH_int *level;
    STARSH_int *start;
    STARSH_int *size;
    STARSH_int *parent;
    STARSH_int *child_start;
    STARSH_int *child;
    enum STARSH_CLUSTER_TYPE type;
};
int starsh_cluster_new(STARSH_cluster **cluster, void *data, STARSH_int ndata,
        STARSH_int *pivot, STARSH_int nblocks, STARSH_int nlevels,
        STARSH_int *level, STARSH_int *start, STARSH_int *size,
        STARSH_int *parent, STARSH_int *child_start, STARSH_int *child,
        enum STARSH_CLUSTER_TYPE type);
void starsh_cluster_free(STARSH_cluster *cluster);
void starsh_cluster_info(STARSH_cluster *cluster);
int starsh_cluster_new_plain(STARSH_cluster **cluster, void *data,
        STARSH_int ndata, STARSH_int block_size);

/* ------------------------------------------------------------------- blrf */

/* Non-nested division into admissible far-field (low-rank) and near-field
 * (dense) blocks, kept as COO, CSR and CSC lists
 * (reference: include/starsh.h:345-457). */
struct starsh_blrf
{
    STARSH_problem *problem;
    char symm;
    STARSH_cluster *row_cluster;
    STARSH_cluster *col_cluster;
    STARSH_int nbrows;
    STARSH_int nbcols;
    STARSH_int nblocks_far;
    STARSH_int *block_far;
    STARSH_int *brow_far_start;
    STARSH_int *brow_far;
    STARSH_int *bcol_far_start;
    STARSH_int *bcol_far;
    STARSH_int nblocks_far_local;
    STARSH_int *block_far_local;
    STARSH_int nblocks_near;
    STARSH_int *block_near;
    STARSH_int *brow_near_start;
    STARSH_int *brow_near;
    STARSH_int *bcol_near_start;
    STARSH_int *bcol_near;
    STARSH_int nblocks_near_local;
    STARSH_int *block_near_local;
    enum STARSH_BLRF_TYPE type;
};
int starsh_blrf_new_from_coo(STARSH_blrf **format, STARSH_problem *problem,
        char symm, STARSH_cluster *row_cluster, STARSH_cluster *col_cluster,
        STARSH_int nblocks_far, STARSH_int *block_far,
        STARSH_int nblocks_near, STARSH_int *block_near,
        enum STARSH_BLRF_TYPE type);
int starsh_blrf_new_tlr(STARSH_blrf **format, STARSH_problem *problem,
        char symm, STARSH_cluster *row_cluster, STARSH_cluster *col_cluster);
void starsh_blrf_free(STARSH_blrf *format);
void starsh_blrf_info(STARSH_blrf *format);
int starsh_blrf_get_block(STARSH_blrf *format, STARSH_int i, STARSH_int j,
        int *shape, void **D);

/* ------------------------------------------------------------------- blrm */

/* Block-low-rank matrix: U_i V_i^T per far-field block, dense near-field
 * blocks (reference: include/starsh.h:497-537).  alloc_type '1' means three
 * big host buffers alloc_U/alloc_V/alloc_D; '2' per-block buffers. */
struct starsh_blrm
{
    STARSH_blrf *format;
    int *far_rank;
    Array **far_U;
    Array **far_V;
    int onfly;
    Array **near_D;
    void *alloc_U;
    void *alloc_V;
    void *alloc_D;
    char alloc_type;
    size_t nbytes;
    size_t data_nbytes;
};
int starsh_blrm_new(STARSH_blrm **matrix, STARSH_blrf *format, int *far_rank,
        Array **far_U, Array **far_V, int onfly, Array **near_D, void *alloc_U,
        void *alloc_V, void *alloc_D, char alloc_type);
/* Frees host buffers and, for matrices produced by the B200 backend, the
 * device-resident factors. */
void starsh_blrm_free(STARSH_blrm *matrix);
void starsh_blrm_info(STARSH_blrm *matrix);
int starsh_blrm_get_block(STARSH_blrm *matrix, STARSH_int i, STARSH_int j,
        int *shape, int *rank, void **U, void **V, void **D);

/* ----------------------------------------------------------- approximation */

/* Approximates every far-field block to relative Frobenius error tol with
 * rank <= maxrank; blocks that need more become dense near-field blocks and
 * *format is rewritten in place (reference: include/starsh.h:563-567,
 * src/backends/openmp/blrm/drsdd.c:146-212). */
typedef int STARSH_blrm_approximate(STARSH_blrm **matrix, STARSH_blrf *format,
        int maxrank, double tol, int onfly);
/* Selected by starsh_init()/starsh_set_backend()/starsh_set_lrengine(). */
extern STARSH_blrm_approximate *starsh_blrm_approximate;

/* B = alpha*M*A + beta*B for nrhs columns, rows in cluster order
 * (reference: include/starsh.h:602-603, src/backends/sequential/blrm/
 * dmml.c:16-145).  Matrices from the B200 backend run on the device. */
int starsh_blrm__dmml(STARSH_blrm *matrix, int nrhs, double alpha, double *A,
        int lda, double beta, double *B, int ldb);
/* Relative Frobenius error ||A - M||_F / ||A||_F, every block regenerated
 * in FP64 (reference: include/starsh.h:622, src/backends/sequential/blrm/
 * dfe.c:16-134).  Matrices from the B200 backend run on the device. */
double starsh_blrm__dfe(STARSH_blrm *matrix);

#ifdef __cplusplus
}
#endif

#endif
