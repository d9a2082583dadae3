/* Host control plane of the B200 library: backend selection, arrays,
 * problem, plain clustering, TLR block format and the block-low-rank matrix
 * container.
 *
 * Behaviour follows STARS-H 0.3.1 so that existing callers see the same
 * structures: src/control/init.c (environment and dispatch),
 * src/control/array.c:16-120 (array views), src/control/problem.c:16-102,
 * src/control/cluster.c:16-146, src/control/blrf.c:90-371 (COO -> CSR/CSC
 * lists; TLR block order) and src/control/blrm.c:17-187.  The backend table
 * has one working row, B200; the CPU backends of the reference are not part
 * of this library and are reported as unsupported.
 */
#define _GNU_SOURCE
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "starsh.h"
#include "starsh-b200.h"
#include "b200_host.h"

/* ------------------------------------------------------- environment */

struct starsh_params starsh_params =
{
    STARSH_BACKEND_NOTSELECTED, STARSH_LRENGINE_NOTSELECTED, -1
};

STARSH_blrm_approximate *starsh_blrm_approximate = NULL;

/* Names accepted in STARSH_BACKEND, in the reference's order (its
 * backend[] table) followed by the new B200 entry. */
static const char *const backend_name[] =
{
    "SEQUENTIAL", "OPENMP", "MPI", "MPI_OPENMP", "STARPU", "MPI_STARPU",
    "STARPU_KBLAS", "STARPU_CUDA", "MPI_STARPU_KBLAS", "B200"
};
static const char *const lrengine_name[] =
{
    "SVD", "DCSVD", "RRQR", "RSVD", "CROSS", "RSVD_MP"
};
#define N_BACKEND ((int)(sizeof(backend_name)/sizeof(backend_name[0])))
#define N_LRENGINE ((int)(sizeof(lrengine_name)/sizeof(lrengine_name[0])))

/* The approximation routine for the current (backend, engine) pair.  Only
 * the B200 row is populated; SVD/DCSVD/RRQR/CROSS map to the FP64
 * randomized engine, as the reference maps CROSS to RSVD. */
static void update_dispatch(void)
{
    starsh_blrm_approximate = NULL;
    if(starsh_params.backend != STARSH_BACKEND_B200)
        return;
    if(starsh_params.lrengine == STARSH_LRENGINE_RSVD_MP)
        starsh_blrm_approximate = starsh_blrm__drsdd_b200_mp;
    else if(starsh_params.lrengine >= 0)
        starsh_blrm_approximate = starsh_blrm__drsdd_b200;
}

int starsh_set_backend(const char *string)
{
    int selected = -1;
    if(string == NULL)
        selected = STARSH_BACKEND_B200;
    else
        for(int i = 0; i < N_BACKEND; i++)
            if(strcmp(string, backend_name[i]) == 0)
                selected = i;
    if(selected < 0)
    {
        fprintf(stderr, "Environment variable STARSH_BACKEND=%s is invalid\n",
                string);
        return STARSH_WRONG_PARAMETER;
    }
    if(selected != STARSH_BACKEND_B200)
    {
        fprintf(stderr, "Specified backend %s is not supported\n", string);
        return STARSH_WRONG_PARAMETER;
    }
    starsh_params.backend = (enum STARSH_BACKEND)selected;
    fprintf(stderr, "Selected backend is %s\n", backend_name[selected]);
    update_dispatch();
    return STARSH_SUCCESS;
}

int starsh_set_lrengine(const char *string)
{
    int selected = -1;
    if(string == NULL)
        selected = STARSH_LRENGINE_RSVD;
    else
        for(int i = 0; i < N_LRENGINE; i++)
            if(strcmp(string, lrengine_name[i]) == 0)
                selected = i;
    if(selected < 0)
    {
        fprintf(stderr, "Environment variable STARSH_LRENGINE=%s is "
                "invalid\n", string);
        return STARSH_WRONG_PARAMETER;
    }
    starsh_params.lrengine = (enum STARSH_LRENGINE)selected;
    fprintf(stderr, "Selected low-rank engine is %s\n",
            lrengine_name[selected]);
    update_dispatch();
    return STARSH_SUCCESS;
}

int starsh_set_oversample(const char *string)
{
    int value = string == NULL ? 10 : atoi(string);
    if(value <= 0)
    {
        fprintf(stderr, "Environment variable STARSH_OVERSAMPLE=%s is "
                "invalid\n", string);
        return STARSH_WRONG_PARAMETER;
    }
    fprintf(stderr, "Selected oversample size %d\n", value);
    starsh_params.oversample = value;
    return STARSH_SUCCESS;
}

int starsh_init(void)
{
    /* The engine is chosen first so that the dispatch update of
     * starsh_set_backend() never reads an unset engine (the reference does,
     * src/control/init.c:52 with init.h:97-100). */
    if(starsh_set_lrengine(getenv("STARSH_LRENGINE")) != STARSH_SUCCESS)
        starsh_set_lrengine(NULL);
    if(starsh_set_backend(getenv("STARSH_BACKEND")) != STARSH_SUCCESS)
        starsh_set_backend(NULL);
    if(starsh_set_oversample(getenv("STARSH_OVERSAMPLE")) != STARSH_SUCCESS)
        starsh_set_oversample(NULL);
    return STARSH_SUCCESS;
}

int b200_oversample(void)
{
    return starsh_params.oversample > 0 ? starsh_params.oversample : 10;
}

/* ------------------------------------------------------------- arrays */

static size_t dtype_bytes(char dtype)
{
    switch(dtype)
    {
        case 's': return 4;
        case 'd': return 8;
        case 'c': return 8;
        case 'z': return 16;
        default: return 0;
    }
}

int array_from_buffer(Array **A, int ndim, int *shape, char dtype, char order,
        void *buffer)
{
    if(A == NULL || ndim < 0 || (order != 'F' && order != 'C') ||
            dtype_bytes(dtype) == 0)
    {
        B200_ERROR("Invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    Array *a = malloc(sizeof(*a));
    if(a == NULL)
        return STARSH_MALLOC_ERROR;
    a->ndim = ndim;
    a->order = order;
    a->dtype = dtype;
    a->dtype_size = dtype_bytes(dtype);
    a->data = buffer;
    if(ndim == 0)
    {
        a->shape = NULL;
        a->stride = NULL;
        a->size = 0;
        a->nbytes = 0;
        a->data_nbytes = sizeof(*a);
        *A = a;
        return STARSH_SUCCESS;
    }
    a->shape = malloc(sizeof(*a->shape)*ndim);
    a->stride = malloc(sizeof(*a->stride)*ndim);
    if(a->shape == NULL || a->stride == NULL)
    {
        free(a->shape);
        free(a->stride);
        free(a);
        return STARSH_MALLOC_ERROR;
    }
    size_t size = 1;
    for(int i = 0; i < ndim; i++)
    {
        a->shape[i] = shape[i];
        size *= (size_t)shape[i];
    }
    /* Fortran order: stride[0] = 1, growing with the dimension index;
     * C order: the reverse. */
    ssize_t s = 1;
    if(order == 'F')
        for(int i = 0; i < ndim; i++)
        {
            a->stride[i] = s;
            s *= shape[i];
        }
    else
        for(int i = ndim-1; i >= 0; i--)
        {
            a->stride[i] = s;
            s *= shape[i];
        }
    a->size = size;
    a->data_nbytes = size*a->dtype_size;
    a->nbytes = sizeof(*a)+ndim*(sizeof(*a->shape)+sizeof(*a->stride))+
        a->data_nbytes;
    *A = a;
    return STARSH_SUCCESS;
}

int array_new(Array **A, int ndim, int *shape, char dtype, char order)
{
    size_t size = 1;
    for(int i = 0; i < ndim; i++)
        size *= (size_t)shape[i];
    void *data = malloc(size*dtype_bytes(dtype)+1);
    if(data == NULL)
        return STARSH_MALLOC_ERROR;
    int info = array_from_buffer(A, ndim, shape, dtype, order, data);
    if(info != STARSH_SUCCESS)
        free(data);
    return info;
}

void array_free(Array *A)
{
    if(A == NULL)
        return;
    free(A->data);
    free(A->shape);
    free(A->stride);
    free(A);
}

/* ------------------------------------------------------------ problem */

int starsh_problem_new(STARSH_problem **problem, int ndim, STARSH_int *shape,
        char symm, char dtype, void *row_data, void *col_data,
        STARSH_kernel *kernel, char *name)
{
    if(problem == NULL || ndim < 2 || shape == NULL ||
            (symm != 'S' && symm != 'N') || kernel == NULL ||
            dtype_bytes(dtype) == 0)
    {
        B200_ERROR("Invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    for(int i = 0; i < ndim; i++)
        if(shape[i] <= 0)
        {
            B200_ERROR("Invalid value of `shape`");
            return STARSH_WRONG_PARAMETER;
        }
    STARSH_problem *P = calloc(1, sizeof(*P));
    if(P == NULL)
        return STARSH_MALLOC_ERROR;
    P->shape = malloc(sizeof(*P->shape)*ndim);
    if(P->shape == NULL)
    {
        free(P);
        return STARSH_MALLOC_ERROR;
    }
    memcpy(P->shape, shape, sizeof(*P->shape)*ndim);
    P->ndim = ndim;
    P->symm = symm;
    P->dtype = dtype;
    P->dtype_size = dtype_bytes(dtype);
    P->entry_size = P->dtype_size;
    for(int i = 1; i < ndim-1; i++)
        P->entry_size *= shape[i];
    P->row_data = row_data;
    P->col_data = col_data;
    P->kernel = kernel;
    P->name = name == NULL ? NULL : strdup(name);
    *problem = P;
    return STARSH_SUCCESS;
}

void starsh_problem_free(STARSH_problem *problem)
{
    if(problem == NULL)
        return;
    free(problem->shape);
    free(problem->name);
    free(problem);
}

void starsh_problem_info(STARSH_problem *problem)
{
    if(problem == NULL)
        return;
    printf("<STARS_Problem at %p, name \"%s\", shape (%zd", (void *)problem,
            problem->name ? problem->name : "", problem->shape[0]);
    for(int i = 1; i < problem->ndim; i++)
        printf(",%zd", problem->shape[i]);
    printf("), '%c' dtype, '%c' symmetric>\n", problem->dtype,
            problem->symm);
}

/* ------------------------------------------------------------ cluster */

int starsh_cluster_new(STARSH_cluster **cluster, void *data, STARSH_int ndata,
        STARSH_int *pivot, STARSH_int nblocks, STARSH_int nlevels,
        STARSH_int *level, STARSH_int *start, STARSH_int *size,
        STARSH_int *parent, STARSH_int *child_start, STARSH_int *child,
        enum STARSH_CLUSTER_TYPE type)
{
    if(cluster == NULL || pivot == NULL || start == NULL || size == NULL ||
            nblocks <= 0)
    {
        B200_ERROR("Invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    STARSH_cluster *C = malloc(sizeof(*C));
    if(C == NULL)
        return STARSH_MALLOC_ERROR;
    C->data = data;
    C->ndata = ndata;
    C->pivot = pivot;
    C->nblocks = nblocks;
    C->nlevels = nlevels;
    C->level = level;
    C->start = start;
    C->size = size;
    C->parent = parent;
    C->child_start = child_start;
    C->child = child;
    C->type = type;
    *cluster = C;
    return STARSH_SUCCESS;
}

void starsh_cluster_free(STARSH_cluster *cluster)
{
    if(cluster == NULL)
        return;
    free(cluster->pivot);
    free(cluster->level);
    free(cluster->start);
    free(cluster->size);
    free(cluster->parent);
    free(cluster->child_start);
    free(cluster->child);
    free(cluster);
}

void starsh_cluster_info(STARSH_cluster *cluster)
{
    if(cluster == NULL)
        return;
    printf("<STARS_Cluster at %p, %s, %zd blocks>\n", (void *)cluster,
            cluster->nlevels == 0 ? "tiled" : "hierarchical",
            cluster->nblocks);
}

/* Consecutive blocks of block_size elements, identity pivot; the last block
 * holds the remainder (reference src/control/cluster.c:106-146). */
int starsh_cluster_new_plain(STARSH_cluster **cluster, void *data,
        STARSH_int ndata, STARSH_int block_size)
{
    if(cluster == NULL || ndata <= 0 || block_size <= 0)
    {
        B200_ERROR("Invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    STARSH_int nblocks = (ndata+block_size-1)/block_size;
    STARSH_int *start = malloc(sizeof(*start)*nblocks);
    STARSH_int *size = malloc(sizeof(*size)*nblocks);
    STARSH_int *pivot = malloc(sizeof(*pivot)*ndata);
    if(start == NULL || size == NULL || pivot == NULL)
    {
        free(start);
        free(size);
        free(pivot);
        return STARSH_MALLOC_ERROR;
    }
    for(STARSH_int b = 0; b < nblocks; b++)
    {
        start[b] = b*block_size;
        size[b] = ndata-start[b] < block_size ? ndata-start[b] : block_size;
    }
    for(STARSH_int i = 0; i < ndata; i++)
        pivot[i] = i;
    return starsh_cluster_new(cluster, data, ndata, pivot, nblocks, 0, NULL,
            start, size, NULL, NULL, NULL, STARSH_PLAIN);
}

/* --------------------------------------------------------------- blrf */

/* Builds the CSR-like index (`first`, `list`) of a COO block list along one
 * coordinate (0: block rows, 1: block columns).  Within a row (column) the
 * blocks keep their COO order, as in the reference's counting sort. */
static int coo_index(STARSH_int nlines, STARSH_int nblocks,
        const STARSH_int *coo, int coord, STARSH_int **first,
        STARSH_int **list)
{
    *first = NULL;
    *list = NULL;
    if(nblocks <= 0)
        return STARSH_SUCCESS;
    STARSH_int *f = calloc(nlines+1, sizeof(*f));
    STARSH_int *l = malloc(sizeof(*l)*nblocks);
    STARSH_int *fill = calloc(nlines, sizeof(*fill));
    if(f == NULL || l == NULL || fill == NULL)
    {
        free(f);
        free(l);
        free(fill);
        return STARSH_MALLOC_ERROR;
    }
    for(STARSH_int b = 0; b < nblocks; b++)
        f[coo[2*b+coord]+1]++;
    for(STARSH_int i = 0; i < nlines; i++)
        f[i+1] += f[i];
    for(STARSH_int b = 0; b < nblocks; b++)
    {
        STARSH_int line = coo[2*b+coord];
        l[f[line]+fill[line]++] = b;
    }
    free(fill);
    *first = f;
    *list = l;
    return STARSH_SUCCESS;
}

int starsh_blrf_new_from_coo(STARSH_blrf **format, STARSH_problem *problem,
        char symm, STARSH_cluster *row_cluster, STARSH_cluster *col_cluster,
        STARSH_int nblocks_far, STARSH_int *block_far,
        STARSH_int nblocks_near, STARSH_int *block_near,
        enum STARSH_BLRF_TYPE type)
{
    if(format == NULL || problem == NULL || (symm != 'S' && symm != 'N') ||
            row_cluster == NULL || col_cluster == NULL ||
            (nblocks_far > 0 && block_far == NULL) ||
            (nblocks_near > 0 && block_near == NULL))
    {
        B200_ERROR("Invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    STARSH_blrf *F = calloc(1, sizeof(*F));
    if(F == NULL)
        return STARSH_MALLOC_ERROR;
    F->problem = problem;
    F->symm = symm;
    F->row_cluster = row_cluster;
    F->col_cluster = symm == 'S' ? row_cluster : col_cluster;
    F->nbrows = row_cluster->nblocks;
    F->nbcols = F->col_cluster->nblocks;
    F->nblocks_far = nblocks_far;
    F->block_far = nblocks_far > 0 ? block_far : NULL;
    F->nblocks_near = nblocks_near;
    F->block_near = nblocks_near > 0 ? block_near : NULL;
    F->type = type;
    int info = coo_index(F->nbrows, nblocks_far, block_far, 0,
            &F->brow_far_start, &F->brow_far);
    if(info == STARSH_SUCCESS)
        info = coo_index(F->nbrows, nblocks_near, block_near, 0,
                &F->brow_near_start, &F->brow_near);
    if(info == STARSH_SUCCESS && symm == 'N')
    {
        info = coo_index(F->nbcols, nblocks_far, block_far, 1,
                &F->bcol_far_start, &F->bcol_far);
        if(info == STARSH_SUCCESS)
            info = coo_index(F->nbcols, nblocks_near, block_near, 1,
                    &F->bcol_near_start, &F->bcol_near);
    }
    else if(symm == 'S')
    {
        F->bcol_far_start = F->brow_far_start;
        F->bcol_far = F->brow_far;
        F->bcol_near_start = F->brow_near_start;
        F->bcol_near = F->brow_near;
    }
    if(info != STARSH_SUCCESS)
    {
        F->block_far = NULL;
        F->block_near = NULL;
        starsh_blrf_free(F);
        return info;
    }
    *format = F;
    return STARSH_SUCCESS;
}

/* Every (block row, block column) pair is far-field: all pairs in row-major
 * order for 'N', the lower triangle j <= i for 'S' (reference
 * src/control/blrf.c:291-371). */
int starsh_blrf_new_tlr(STARSH_blrf **format, STARSH_problem *problem,
        char symm, STARSH_cluster *row_cluster, STARSH_cluster *col_cluster)
{
    if(format == NULL || problem == NULL || row_cluster == NULL ||
            col_cluster == NULL || (symm != 'S' && symm != 'N') ||
            (symm == 'S' && problem->symm == 'N') ||
            (symm == 'S' && row_cluster != col_cluster))
    {
        B200_ERROR("Invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    STARSH_int nbr = row_cluster->nblocks, nbc = col_cluster->nblocks;
    STARSH_int nfar = symm == 'N' ? nbr*nbc : nbr*(nbr+1)/2;
    STARSH_int *coo = malloc(sizeof(*coo)*2*nfar);
    if(coo == NULL)
        return STARSH_MALLOC_ERROR;
    STARSH_int b = 0;
    for(STARSH_int i = 0; i < nbr; i++)
        for(STARSH_int j = 0; j < (symm == 'N' ? nbc : i+1); j++)
        {
            coo[2*b] = i;
            coo[2*b+1] = j;
            b++;
        }
    int info = starsh_blrf_new_from_coo(format, problem, symm, row_cluster,
            col_cluster, nfar, coo, 0, NULL, STARSH_TLR);
    if(info != STARSH_SUCCESS)
        free(coo);
    return info;
}

/* Frees the block lists that exist for non-empty far/near sets.  The
 * *_local fields are never set on the TLR path (the reference leaves them
 * uninitialised), so they are not touched: a format built by the reference
 * library may be freed here after an in-place swap. */
void starsh_blrf_free(STARSH_blrf *format)
{
    STARSH_blrf *F = format;
    if(F == NULL)
        return;
    if(F->nblocks_far > 0)
    {
        free(F->block_far);
        free(F->brow_far_start);
        free(F->brow_far);
    }
    if(F->nblocks_near > 0)
    {
        free(F->block_near);
        free(F->brow_near_start);
        free(F->brow_near);
    }
    if(F->symm == 'N')
    {
        if(F->nblocks_far > 0)
        {
            free(F->bcol_far_start);
            free(F->bcol_far);
        }
        if(F->nblocks_near > 0)
        {
            free(F->bcol_near_start);
            free(F->bcol_near);
        }
    }
    free(F);
}

void starsh_blrf_info(STARSH_blrf *format)
{
    if(format == NULL)
        return;
    printf("<STARS_BLRF at %p, '%c' symmetric, %zd block rows, %zd "
            "block columns, %zd far-field blocks, %zd near-field blocks>\n",
            (void *)format, format->symm, format->nbrows, format->nbcols,
            format->nblocks_far, format->nblocks_near);
}

int starsh_blrf_get_block(STARSH_blrf *format, STARSH_int i, STARSH_int j,
        int *shape, void **D)
{
    if(format == NULL || shape == NULL || D == NULL || i < 0 ||
            i >= format->nbrows || j < 0 || j >= format->nbcols)
    {
        B200_ERROR("Invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    STARSH_problem *P = format->problem;
    STARSH_cluster *R = format->row_cluster, *C = format->col_cluster;
    int m = (int)R->size[i], n = (int)C->size[j];
    double *buf = malloc(sizeof(double)*(size_t)m*n);
    if(buf == NULL)
        return STARSH_MALLOC_ERROR;
    P->kernel(m, n, R->pivot+R->start[i], C->pivot+C->start[j],
            P->row_data, P->col_data, buf, m);
    shape[0] = m;
    shape[1] = n;
    *D = buf;
    return STARSH_SUCCESS;
}

/* --------------------------------------------------------------- blrm */

int starsh_blrm_new(STARSH_blrm **matrix, STARSH_blrf *format, int *far_rank,
        Array **far_U, Array **far_V, int onfly, Array **near_D, void *alloc_U,
        void *alloc_V, void *alloc_D, char alloc_type)
{
    STARSH_blrf *F = format;
    if(matrix == NULL || F == NULL || (onfly != 0 && onfly != 1) ||
            (alloc_type != '1' && alloc_type != '2') ||
            (F->nblocks_far > 0 && (far_rank == NULL || far_U == NULL ||
                                    far_V == NULL)) ||
            (F->nblocks_near > 0 && onfly == 0 && near_D == NULL))
    {
        B200_ERROR("Invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    STARSH_blrm *M = malloc(sizeof(*M));
    if(M == NULL)
        return STARSH_MALLOC_ERROR;
    M->format = F;
    M->far_rank = far_rank;
    M->far_U = far_U;
    M->far_V = far_V;
    M->onfly = onfly;
    M->near_D = near_D;
    M->alloc_U = alloc_U;
    M->alloc_V = alloc_V;
    M->alloc_D = alloc_D;
    M->alloc_type = alloc_type;
    size_t size = sizeof(*M), data_size = 0;
    size += F->nblocks_far*(sizeof(*far_rank)+sizeof(*far_U)+
            sizeof(*far_V));
    for(STARSH_int b = 0; b < F->nblocks_far; b++)
    {
        size += far_U[b]->nbytes+far_V[b]->nbytes;
        data_size += far_U[b]->data_nbytes+far_V[b]->data_nbytes;
    }
    if(onfly == 0)
    {
        size += F->nblocks_near*sizeof(*near_D);
        for(STARSH_int b = 0; b < F->nblocks_near; b++)
        {
            size += near_D[b]->nbytes;
            data_size += near_D[b]->data_nbytes;
        }
    }
    M->nbytes = size;
    M->data_nbytes = data_size;
    *matrix = M;
    return STARSH_SUCCESS;
}

void starsh_blrm_free(STARSH_blrm *matrix)
{
    STARSH_blrm *M = matrix;
    if(M == NULL)
        return;
    starsh_b200_blrm_release(M);
    starsh_b200_blrm_host_release(M);
    STARSH_blrf *F = M->format;
    if(F->nblocks_far > 0)
    {
        for(STARSH_int b = 0; b < F->nblocks_far; b++)
        {
            if(M->alloc_type == '1')
            {
                M->far_U[b]->data = NULL;
                M->far_V[b]->data = NULL;
            }
            array_free(M->far_U[b]);
            array_free(M->far_V[b]);
        }
        if(M->alloc_type == '1')
        {
            free(M->alloc_U);
            free(M->alloc_V);
        }
        free(M->far_rank);
        free(M->far_U);
        free(M->far_V);
    }
    if(F->nblocks_near > 0 && M->onfly == 0)
    {
        for(STARSH_int b = 0; b < F->nblocks_near; b++)
        {
            if(M->alloc_type == '1')
                M->near_D[b]->data = NULL;
            array_free(M->near_D[b]);
        }
        if(M->alloc_type == '1')
            free(M->alloc_D);
        free(M->near_D);
    }
    free(M);
}

void starsh_blrm_info(STARSH_blrm *matrix)
{
    if(matrix == NULL)
        return;
    printf("<STARSH_blrm at %p, %d onfly, allocation type '%c', %f MB memory "
            "footprint>\n", (void *)matrix, matrix->onfly,
            matrix->alloc_type, matrix->nbytes/1024./1024.);
}

/* Low-rank factors of an admissible far-field block, its dense copy for a
 * stored near-field block, or a freshly generated dense block otherwise
 * (reference src/control/blrm.c:200-322).  Device-resident matrices are
 * downloaded first. */
int starsh_blrm_get_block(STARSH_blrm *matrix, STARSH_int i, STARSH_int j,
        int *shape, int *rank, void **U, void **V, void **D)
{
    STARSH_blrm *M = matrix;
    if(M == NULL || shape == NULL || rank == NULL || U == NULL ||
            V == NULL || D == NULL)
    {
        B200_ERROR("Invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    STARSH_blrf *F = M->format;
    if(i < 0 || i >= F->nbrows || j < 0 || j >= F->nbcols ||
            F->problem->ndim != 2)
    {
        B200_ERROR("Invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    int info = starsh_b200_blrm_download(M);
    if(info != STARSH_SUCCESS)
        return info;
    STARSH_cluster *R = F->row_cluster, *C = F->col_cluster;
    int m = (int)R->size[i], n = (int)C->size[j];
    shape[0] = m;
    shape[1] = n;
    *rank = m < n ? m : n;
    *U = NULL;
    *V = NULL;
    *D = NULL;
    for(STARSH_int k = F->brow_far_start ? F->brow_far_start[i] : 0;
            F->brow_far_start && k < F->brow_far_start[i+1]; k++)
    {
        STARSH_int b = F->brow_far[k];
        if(F->block_far[2*b+1] == j)
        {
            *rank = M->far_rank[b];
            *U = M->far_U[b]->data;
            *V = M->far_V[b]->data;
            return STARSH_SUCCESS;
        }
    }
    for(STARSH_int k = F->brow_near_start ? F->brow_near_start[i] : 0;
            F->brow_near_start && k < F->brow_near_start[i+1]; k++)
    {
        STARSH_int b = F->brow_near[k];
        if(F->block_near[2*b+1] == j && M->onfly == 0)
        {
            *D = M->near_D[b]->data;
            return STARSH_SUCCESS;
        }
    }
    return starsh_blrf_get_block(F, i, j, shape, D);
}
