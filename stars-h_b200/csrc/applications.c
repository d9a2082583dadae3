/* Applications on the TLR path: point sets, the spatial-statistics,
 * electrostatics, electrodynamics and RBF problem data, starsh_application(),
 * kernel selection, the host-callable kernel entry points and the
 * kernel-pointer -> device-generator registry.
 *
 * Point generation reproduces the reference bit for bit given the same libc
 * rand() stream (callers seed it with srand(), as testing/spatial.c:53
 * does): src/applications/particles.c:177-201 (RAND), :260-333 (UNIFORM),
 * :341-411 (QUASIUNIFORM1: grid cell origin + 0.1 cell + 0.8 cell * U) and
 * the Z-order sort :1090-1221.  The Z-order sort partitions MSB first,
 * highest dimension first, zero bits forward and one bits filled from the
 * back, which reverses the order of the one-bit group at every level; that
 * order is part of the point permutation every caller sees, so it is kept.
 *
 * The reference's *_init constructors of esdata/eddata/particles allocate
 * the structure but never store it in *data; here they do.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "starsh.h"
#include "starsh-b200.h"
#include "starsh-particles.h"
#include "starsh-spatial.h"
#include "starsh-electrostatics.h"
#include "starsh-electrodynamics.h"
#include "starsh-rbf.h"
#include "b200_host.h"

/* ------------------------------------------------------------ particles */

int starsh_particles_new(STARSH_particles **data, STARSH_int count, int ndim)
{
    if(data == NULL || ndim <= 0 || count <= 0)
        return STARSH_WRONG_PARAMETER;
    STARSH_particles *p = malloc(sizeof(*p));
    if(p == NULL)
        return STARSH_MALLOC_ERROR;
    p->point = malloc(sizeof(double)*(size_t)count*ndim);
    if(p->point == NULL)
    {
        free(p);
        return STARSH_MALLOC_ERROR;
    }
    p->count = count;
    p->ndim = ndim;
    *data = p;
    return STARSH_SUCCESS;
}

int starsh_particles_init(STARSH_particles **data, STARSH_int count, int ndim,
        double *point)
{
    if(data == NULL || ndim <= 0 || count <= 0 || point == NULL)
        return STARSH_WRONG_PARAMETER;
    STARSH_particles *p = malloc(sizeof(*p));
    if(p == NULL)
        return STARSH_MALLOC_ERROR;
    p->count = count;
    p->ndim = ndim;
    p->point = point;
    *data = p;
    return STARSH_SUCCESS;
}

void starsh_particles_free(STARSH_particles *data)
{
    if(data == NULL)
        return;
    free(data->point);
    free(data);
}

/* Partition of order[lo..hi] by bit `bit` of dimension `dim`, recursing
 * to the next (dimension, bit) pair on both halves. */
static void zorder_split(const uint32_t *key, STARSH_int count, int ndim,
        STARSH_int *order, STARSH_int *scratch, int dim, int bit,
        STARSH_int lo, STARSH_int hi)
{
    const uint32_t *k = key+(size_t)dim*count;
    const uint32_t mask = (uint32_t)1 << bit;
    STARSH_int front = lo, back = hi;
    for(STARSH_int i = lo; i <= hi; i++)
    {
        if(k[order[i]] & mask)
            scratch[back--] = order[i];
        else
            scratch[front++] = order[i];
    }
    memcpy(order+lo, scratch+lo, sizeof(*order)*(size_t)(hi-lo+1));
    int next_dim = dim-1, next_bit = bit;
    if(dim == 0)
    {
        if(bit == 0)
            return;
        next_dim = ndim-1;
        next_bit = bit-1;
    }
    if(front-lo > 1)
        zorder_split(key, count, ndim, order, scratch, next_dim, next_bit,
                lo, front-1);
    if(hi-back > 1)
        zorder_split(key, count, ndim, order, scratch, next_dim, next_bit,
                back+1, hi);
}

int starsh_particles_zsort_inplace(STARSH_particles *data)
{
    if(data == NULL || data->count <= 0 || data->ndim <= 0)
        return STARSH_WRONG_PARAMETER;
    STARSH_int n = data->count;
    int ndim = data->ndim;
    double *pt = data->point;
    uint32_t *key = malloc(sizeof(*key)*(size_t)n*ndim);
    STARSH_int *order = malloc(sizeof(*order)*(size_t)n);
    STARSH_int *scratch = malloc(sizeof(*scratch)*(size_t)n);
    double *sorted = malloc(sizeof(*sorted)*(size_t)n*ndim);
    if(!key || !order || !scratch || !sorted)
    {
        free(key);
        free(order);
        free(scratch);
        free(sorted);
        return STARSH_MALLOC_ERROR;
    }
    /* Coordinates scaled to [0, 2^32-1] per dimension by its own range. */
    for(int d = 0; d < ndim; d++)
    {
        const double *x = pt+(size_t)d*n;
        double lo = x[0], hi = x[0];
        for(STARSH_int i = 1; i < n; i++)
        {
            if(x[i] < lo)
                lo = x[i];
            else if(x[i] > hi)
                hi = x[i];
        }
        double range = hi-lo;
        for(STARSH_int i = 0; i < n; i++)
            key[(size_t)d*n+i] = (uint32_t)((x[i]-lo)/range*UINT32_MAX);
    }
    for(STARSH_int i = 0; i < n; i++)
        order[i] = i;
    if(n > 1)
        zorder_split(key, n, ndim, order, scratch, ndim-1, 31, 0, n-1);
    for(STARSH_int i = 0; i < n; i++)
        for(int d = 0; d < ndim; d++)
            sorted[(size_t)d*n+i] = pt[(size_t)d*n+order[i]];
    data->point = sorted;
    free(pt);
    free(key);
    free(order);
    free(scratch);
    return STARSH_SUCCESS;
}

int starsh_particles_generate_rand(STARSH_particles **data, STARSH_int count,
        int ndim)
{
    int info = starsh_particles_new(data, count, ndim);
    if(info != STARSH_SUCCESS)
        return info;
    double *pt = (*data)->point;
    for(size_t i = 0; i < (size_t)count*ndim; i++)
        pt[i] = (double)rand()/RAND_MAX;
    return starsh_particles_zsort_inplace(*data);
}

/* Smallest grid side with side^ndim >= count, as the reference computes it
 * (ceil of the floating-point root). */
static STARSH_int grid_side(STARSH_int count, int ndim)
{
    return (STARSH_int)ceil(pow((double)count, 1.0/ndim));
}

/* Fills point[] with the first `count` nodes of the side^ndim grid in
 * lexicographic order (last dimension fastest); `jitter` adds the
 * QUASIUNIFORM1 offset 0.1 cell + 0.8 cell * rand()/RAND_MAX. */
static int grid_points(STARSH_particles **data, STARSH_int count, int ndim,
        int jitter)
{
    STARSH_int side = grid_side(count, ndim);
    double total = 1;
    for(int d = 0; d < ndim; d++)
        total *= (double)side;
    if(total < (double)count)
        return STARSH_UNKNOWN_ERROR;
    int info = starsh_particles_new(data, count, ndim);
    if(info != STARSH_SUCCESS)
        return info;
    double *pt = (*data)->point;
    STARSH_int *idx = calloc(ndim, sizeof(*idx));
    if(idx == NULL)
    {
        starsh_particles_free(*data);
        return STARSH_MALLOC_ERROR;
    }
    const double mult = 0.8/side/RAND_MAX, add = 0.1/side;
    for(STARSH_int i = 0; i < count; i++)
    {
        for(int d = 0; d < ndim; d++)
        {
            double cell = (double)idx[d]/side;
            pt[i+(size_t)d*count] = jitter ? cell+add+mult*rand() : cell;
        }
        int d = ndim-1;
        idx[d]++;
        while(idx[d] == side)
        {
            idx[d] = 0;
            if(d == 0)
                break;
            d--;
            idx[d]++;
        }
    }
    free(idx);
    return starsh_particles_zsort_inplace(*data);
}

int starsh_particles_generate_uniform(STARSH_particles **data,
        STARSH_int count, int ndim)
{
    return grid_points(data, count, ndim, 0);
}

int starsh_particles_generate_quasiuniform1(STARSH_particles **data,
        STARSH_int count, int ndim)
{
    return grid_points(data, count, ndim, 1);
}

int starsh_particles_generate(STARSH_particles **data, STARSH_int count,
        int ndim, enum STARSH_PARTICLES_PLACEMENT ptype)
{
    switch(ptype)
    {
        case STARSH_PARTICLES_RAND:
            return starsh_particles_generate_rand(data, count, ndim);
        case STARSH_PARTICLES_UNIFORM:
            return starsh_particles_generate_uniform(data, count, ndim);
        case STARSH_PARTICLES_QUASIUNIFORM1:
            return starsh_particles_generate_quasiuniform1(data, count, ndim);
        default:
            B200_ERROR("Placement %d is not provided by this library",
                    (int)ptype);
            return STARSH_WRONG_PARAMETER;
    }
}

/* ------------------------------------------------------ spatial data */

int starsh_ssdata_new(STARSH_ssdata **data, STARSH_int count, int ndim)
{
    if(data == NULL || ndim <= 0 || count <= 0)
        return STARSH_WRONG_PARAMETER;
    STARSH_ssdata *s = calloc(1, sizeof(*s));
    if(s == NULL)
        return STARSH_MALLOC_ERROR;
    s->particles.point = malloc(sizeof(double)*(size_t)count*ndim);
    if(s->particles.point == NULL)
    {
        free(s);
        return STARSH_MALLOC_ERROR;
    }
    s->particles.count = count;
    s->particles.ndim = ndim;
    *data = s;
    return STARSH_SUCCESS;
}

static int check_spatial(double beta, double nu, double noise, double sigma)
{
    if(beta <= 0 || nu < 0 || noise < 0 || sigma < 0)
    {
        B200_ERROR("Invalid spatial parameters");
        return STARSH_WRONG_PARAMETER;
    }
    return STARSH_SUCCESS;
}

int starsh_ssdata_init(STARSH_ssdata **data, STARSH_int count, int ndim,
        double *point, double beta, double nu, double noise, double sigma)
{
    if(data == NULL || ndim <= 0 || point == NULL)
        return STARSH_WRONG_PARAMETER;
    int info = check_spatial(beta, nu, noise, sigma);
    if(info != STARSH_SUCCESS)
        return info;
    STARSH_ssdata *s = calloc(1, sizeof(*s));
    if(s == NULL)
        return STARSH_MALLOC_ERROR;
    s->particles.count = count;
    s->particles.ndim = ndim;
    s->particles.point = point;
    s->beta = beta;
    s->nu = nu;
    s->noise = noise;
    s->sigma = sigma;
    *data = s;
    return STARSH_SUCCESS;
}

int starsh_ssdata_generate(STARSH_ssdata **data, STARSH_int count, int ndim,
        double beta, double nu, double noise,
        enum STARSH_PARTICLES_PLACEMENT place, double sigma)
{
    if(data == NULL)
        return STARSH_WRONG_PARAMETER;
    int info = check_spatial(beta, nu, noise, sigma);
    if(info != STARSH_SUCCESS)
        return info;
    STARSH_particles *p;
    info = starsh_particles_generate(&p, count, ndim, place);
    if(info != STARSH_SUCCESS)
        return info;
    STARSH_ssdata *s = calloc(1, sizeof(*s));
    if(s == NULL)
    {
        starsh_particles_free(p);
        return STARSH_MALLOC_ERROR;
    }
    s->particles = *p;
    free(p);
    s->beta = beta;
    s->nu = nu;
    s->noise = noise;
    s->sigma = sigma;
    *data = s;
    return STARSH_SUCCESS;
}

/* Defaults as in the reference (src/applications/spatial.c:376-385):
 * ndim 2, beta 0.1, nu 0.5, noise 0, UNIFORM placement, sigma 1.  The
 * bivariate parameters (SIGMA2, NU2, CORR) are accepted but the bivariate
 * kernels are not part of this library. */
int starsh_ssdata_generate_va(STARSH_ssdata **data, STARSH_int count,
        va_list args)
{
    int ndim = 2, arg;
    double beta = 0.1, nu = 0.5, noise = 0, sigma = 1.0;
    double nu2 = 0.5, sigma2 = -1.0, corr = 0.0;
    enum STARSH_PARTICLES_PLACEMENT place = STARSH_PARTICLES_UNIFORM;
    while((arg = va_arg(args, int)) != 0)
    {
        switch(arg)
        {
            case STARSH_SPATIAL_NDIM: ndim = va_arg(args, int); break;
            case STARSH_SPATIAL_BETA: beta = va_arg(args, double); break;
            case STARSH_SPATIAL_NU: nu = va_arg(args, double); break;
            case STARSH_SPATIAL_NOISE: noise = va_arg(args, double); break;
            case STARSH_SPATIAL_PLACE:
                place = (enum STARSH_PARTICLES_PLACEMENT)va_arg(args, int);
                break;
            case STARSH_SPATIAL_SIGMA: sigma = va_arg(args, double); break;
            case STARSH_SPATIAL_SIGMA2: sigma2 = va_arg(args, double); break;
            case STARSH_SPATIAL_NU2: nu2 = va_arg(args, double); break;
            case STARSH_SPATIAL_CORR: corr = va_arg(args, double); break;
            default:
                B200_ERROR("Wrong parameter type");
                return STARSH_WRONG_PARAMETER;
        }
    }
    if(sigma2 >= 0)
    {
        B200_ERROR("Bivariate (parsimonious) spatial data is not provided "
                "by this library");
        return STARSH_WRONG_PARAMETER;
    }
    (void)nu2;
    (void)corr;
    return starsh_ssdata_generate(data, count, ndim, beta, nu, noise, place,
            sigma);
}

int starsh_ssdata_generate_el(STARSH_ssdata **data, STARSH_int count, ...)
{
    va_list args;
    va_start(args, count);
    int info = starsh_ssdata_generate_va(data, count, args);
    va_end(args);
    return info;
}

void starsh_ssdata_free(STARSH_ssdata *data)
{
    if(data == NULL)
        return;
    free(data->particles.point);
    free(data);
}

/* Kernel function for a spatial family and dimension; families and the
 * d-specific names as in src/applications/spatial.c:557-893. */
#define SPATIAL_TABLE(fam) \
    { starsh_ssdata_block_##fam##_kernel_1d, \
      starsh_ssdata_block_##fam##_kernel_2d, \
      starsh_ssdata_block_##fam##_kernel_3d, \
      starsh_ssdata_block_##fam##_kernel_4d, \
      starsh_ssdata_block_##fam##_kernel_nd }, \
    { starsh_ssdata_block_##fam##_kernel_1d_simd, \
      starsh_ssdata_block_##fam##_kernel_2d_simd, \
      starsh_ssdata_block_##fam##_kernel_3d_simd, \
      starsh_ssdata_block_##fam##_kernel_4d_simd, \
      starsh_ssdata_block_##fam##_kernel_nd_simd }

static STARSH_kernel *const spatial_kernels[8][5] =
{
    SPATIAL_TABLE(exp), SPATIAL_TABLE(sqrexp), SPATIAL_TABLE(matern),
    SPATIAL_TABLE(matern2)
};

static int dim_slot(int ndim)
{
    return ndim >= 1 && ndim <= 4 ? ndim-1 : 4;
}

int starsh_ssdata_get_kernel(STARSH_kernel **kernel, STARSH_ssdata *data,
        enum STARSH_SPATIAL_KERNEL type)
{
    if(kernel == NULL || data == NULL)
        return STARSH_WRONG_PARAMETER;
    int row;
    switch(type)
    {
        case STARSH_SPATIAL_EXP: row = 0; break;
        case STARSH_SPATIAL_EXP_SIMD: row = 1; break;
        case STARSH_SPATIAL_SQREXP: row = 2; break;
        case STARSH_SPATIAL_SQREXP_SIMD: row = 3; break;
        case STARSH_SPATIAL_MATERN: row = 4; break;
        case STARSH_SPATIAL_MATERN_SIMD: row = 5; break;
        case STARSH_SPATIAL_MATERN2: row = 6; break;
        case STARSH_SPATIAL_MATERN2_SIMD: row = 7; break;
        default:
            B200_ERROR("Wrong type of kernel");
            return STARSH_WRONG_PARAMETER;
    }
    *kernel = spatial_kernels[row][dim_slot(data->particles.ndim)];
    return STARSH_SUCCESS;
}

/* ------------------------------------------------ electrostatics data */

int starsh_esdata_init(STARSH_esdata **data, STARSH_int count, int ndim,
        double *point)
{
    return starsh_particles_init(data, count, ndim, point);
}

int starsh_esdata_generate(STARSH_esdata **data, STARSH_int count, int ndim,
        enum STARSH_PARTICLES_PLACEMENT place)
{
    return starsh_particles_generate(data, count, ndim, place);
}

int starsh_esdata_generate_va(STARSH_esdata **data, STARSH_int count,
        va_list args)
{
    int ndim = 2, arg;
    enum STARSH_PARTICLES_PLACEMENT place = STARSH_PARTICLES_UNIFORM;
    while((arg = va_arg(args, int)) != 0)
    {
        switch(arg)
        {
            case STARSH_ELECTROSTATICS_NDIM: ndim = va_arg(args, int); break;
            case STARSH_ELECTROSTATICS_PLACE:
                place = (enum STARSH_PARTICLES_PLACEMENT)va_arg(args, int);
                break;
            default:
                B200_ERROR("Wrong parameter type");
                return STARSH_WRONG_PARAMETER;
        }
    }
    return starsh_esdata_generate(data, count, ndim, place);
}

int starsh_esdata_generate_el(STARSH_esdata **data, STARSH_int count, ...)
{
    va_list args;
    va_start(args, count);
    int info = starsh_esdata_generate_va(data, count, args);
    va_end(args);
    return info;
}

void starsh_esdata_free(STARSH_esdata *data)
{
    starsh_particles_free(data);
}

static STARSH_kernel *const coulomb_kernels[2][5] =
{
    { starsh_esdata_block_coulomb_potential_kernel_1d,
      starsh_esdata_block_coulomb_potential_kernel_2d,
      starsh_esdata_block_coulomb_potential_kernel_3d,
      starsh_esdata_block_coulomb_potential_kernel_4d,
      starsh_esdata_block_coulomb_potential_kernel_nd },
    { starsh_esdata_block_coulomb_potential_kernel_1d_simd,
      starsh_esdata_block_coulomb_potential_kernel_2d_simd,
      starsh_esdata_block_coulomb_potential_kernel_3d_simd,
      starsh_esdata_block_coulomb_potential_kernel_4d_simd,
      starsh_esdata_block_coulomb_potential_kernel_nd_simd }
};

int starsh_esdata_get_kernel(STARSH_kernel **kernel, STARSH_esdata *data,
        enum STARSH_ELECTROSTATICS_KERNEL type)
{
    if(kernel == NULL || data == NULL)
        return STARSH_WRONG_PARAMETER;
    if(type != STARSH_ELECTROSTATICS_COULOMB_POTENTIAL &&
            type != STARSH_ELECTROSTATICS_COULOMB_POTENTIAL_SIMD)
    {
        B200_ERROR("Wrong type of kernel");
        return STARSH_WRONG_PARAMETER;
    }
    *kernel = coulomb_kernels[type == STARSH_ELECTROSTATICS_COULOMB_POTENTIAL
        ? 0 : 1][dim_slot(data->ndim)];
    return STARSH_SUCCESS;
}

/* ---------------------------------------------- electrodynamics data */

int starsh_eddata_init(STARSH_eddata **data, STARSH_int count, int ndim,
        double *point, double k, double diag)
{
    if(data == NULL || ndim <= 0 || point == NULL)
        return STARSH_WRONG_PARAMETER;
    STARSH_eddata *e = calloc(1, sizeof(*e));
    if(e == NULL)
        return STARSH_MALLOC_ERROR;
    e->particles.count = count;
    e->particles.ndim = ndim;
    e->particles.point = point;
    e->k = k;
    e->diag = diag;
    *data = e;
    return STARSH_SUCCESS;
}

int starsh_eddata_generate(STARSH_eddata **data, STARSH_int count, int ndim,
        double k, double diag, enum STARSH_PARTICLES_PLACEMENT place)
{
    if(data == NULL)
        return STARSH_WRONG_PARAMETER;
    STARSH_particles *p;
    int info = starsh_particles_generate(&p, count, ndim, place);
    if(info != STARSH_SUCCESS)
        return info;
    STARSH_eddata *e = calloc(1, sizeof(*e));
    if(e == NULL)
    {
        starsh_particles_free(p);
        return STARSH_MALLOC_ERROR;
    }
    e->particles = *p;
    free(p);
    e->k = k;
    e->diag = diag;
    *data = e;
    return STARSH_SUCCESS;
}

/* Defaults as in src/applications/electrodynamics.c:160-176: ndim 2, k 1,
 * diag 1, UNIFORM placement. */
int starsh_eddata_generate_va(STARSH_eddata **data, STARSH_int count,
        va_list args)
{
    int ndim = 2, arg;
    double k = 1.0, diag = 1.0;
    enum STARSH_PARTICLES_PLACEMENT place = STARSH_PARTICLES_UNIFORM;
    while((arg = va_arg(args, int)) != 0)
    {
        switch(arg)
        {
            case STARSH_ELECTRODYNAMICS_NDIM: ndim = va_arg(args, int); break;
            case STARSH_ELECTRODYNAMICS_K: k = va_arg(args, double); break;
            case STARSH_ELECTRODYNAMICS_DIAG: diag = va_arg(args, double);
                break;
            case STARSH_ELECTRODYNAMICS_PLACE:
                place = (enum STARSH_PARTICLES_PLACEMENT)va_arg(args, int);
                break;
            default:
                B200_ERROR("Wrong parameter type");
                return STARSH_WRONG_PARAMETER;
        }
    }
    return starsh_eddata_generate(data, count, ndim, k, diag, place);
}

int starsh_eddata_generate_el(STARSH_eddata **data, STARSH_int count, ...)
{
    va_list args;
    va_start(args, count);
    int info = starsh_eddata_generate_va(data, count, args);
    va_end(args);
    return info;
}

void starsh_eddata_free(STARSH_eddata *data)
{
    if(data == NULL)
        return;
    free(data->particles.point);
    free(data);
}

#define ED_TABLE(fam) \
    { starsh_eddata_block_##fam##_kernel_1d, \
      starsh_eddata_block_##fam##_kernel_2d, \
      starsh_eddata_block_##fam##_kernel_3d, \
      starsh_eddata_block_##fam##_kernel_4d, \
      starsh_eddata_block_##fam##_kernel_nd }, \
    { starsh_eddata_block_##fam##_kernel_1d_simd, \
      starsh_eddata_block_##fam##_kernel_2d_simd, \
      starsh_eddata_block_##fam##_kernel_3d_simd, \
      starsh_eddata_block_##fam##_kernel_4d_simd, \
      starsh_eddata_block_##fam##_kernel_nd_simd }

static STARSH_kernel *const ed_kernels[4][5] =
{
    ED_TABLE(sin), ED_TABLE(cos)
};

int starsh_eddata_get_kernel(STARSH_kernel **kernel, STARSH_eddata *data,
        enum STARSH_ELECTRODYNAMICS_KERNEL type)
{
    if(kernel == NULL || data == NULL)
        return STARSH_WRONG_PARAMETER;
    int row;
    switch(type)
    {
        case STARSH_ELECTRODYNAMICS_SIN: row = 0; break;
        case STARSH_ELECTRODYNAMICS_SIN_SIMD: row = 1; break;
        case STARSH_ELECTRODYNAMICS_COS: row = 2; break;
        case STARSH_ELECTRODYNAMICS_COS_SIMD: row = 3; break;
        default:
            B200_ERROR("Wrong type of kernel");
            return STARSH_WRONG_PARAMETER;
    }
    *kernel = ed_kernels[row][dim_slot(data->particles.ndim)];
    return STARSH_SUCCESS;
}

/* --------------------------------------------------------- RBF data */

int starsh_mddata_init(STARSH_mddata **data, STARSH_int count, double *mesh,
        int kernel, int numobj, int isreg, double reg, double rad,
        double denst)
{
    if(data == NULL || count <= 0 || mesh == NULL)
        return STARSH_WRONG_PARAMETER;
    STARSH_mddata *m = calloc(1, sizeof(*m));
    if(m == NULL)
        return STARSH_MALLOC_ERROR;
    m->particles.count = count;
    m->particles.ndim = 3;
    m->particles.point = mesh;
    m->kernel = kernel;
    m->numobj = numobj;
    m->isreg = isreg;
    m->reg = reg;
    m->rad = rad;
    m->denst = denst;
    m->mesh_points = (int)count;
    *data = m;
    return STARSH_SUCCESS;
}

void starsh_mddata_free(STARSH_mddata *data)
{
    if(data == NULL)
        return;
    free(data->particles.point);
    free(data);
}

/* ------------------------------------------------------- application */

int starsh_application(void **data, STARSH_kernel **kernel, STARSH_int count,
        char dtype, int problem_type, int kernel_type, ...)
{
    (void)dtype;
    va_list args;
    va_start(args, kernel_type);
    int info;
    switch(problem_type)
    {
        case STARSH_SPATIAL:
            info = starsh_ssdata_generate_va((STARSH_ssdata **)data, count,
                    args);
            if(info == STARSH_SUCCESS)
                info = starsh_ssdata_get_kernel(kernel, *data,
                        (enum STARSH_SPATIAL_KERNEL)kernel_type);
            break;
        case STARSH_ELECTROSTATICS:
            info = starsh_esdata_generate_va((STARSH_esdata **)data, count,
                    args);
            if(info == STARSH_SUCCESS)
                info = starsh_esdata_get_kernel(kernel, *data,
                        (enum STARSH_ELECTROSTATICS_KERNEL)kernel_type);
            break;
        case STARSH_ELECTRODYNAMICS:
            info = starsh_eddata_generate_va((STARSH_eddata **)data, count,
                    args);
            if(info == STARSH_SUCCESS)
                info = starsh_eddata_get_kernel(kernel, *data,
                        (enum STARSH_ELECTRODYNAMICS_KERNEL)kernel_type);
            break;
        default:
            B200_ERROR("Problem type %d is not on the TLR path of this "
                    "library", problem_type);
            info = STARSH_WRONG_PARAMETER;
    }
    va_end(args);
    return info;
}

/* ------------------------------------------- host kernel entry points */

/* Every kernel symbol evaluates its block on the GPU.  The functions are
 * distinct (each passes its own address) so that the registry can map any
 * of them, or the reference library's function of the same name, to the
 * device generator. */
#define HOST_ENTRY(name) \
    void name(int nrows, int ncols, STARSH_int *irow, STARSH_int *icol, \
            void *row_data, void *col_data, void *result, int ld) \
    { \
        b200_eval_block_host(name, nrows, ncols, irow, icol, row_data, \
                col_data, (double *)result, ld); \
    }
#define HOST_ENTRIES_ND(prefix) \
    HOST_ENTRY(prefix##_1d) HOST_ENTRY(prefix##_2d) HOST_ENTRY(prefix##_3d) \
    HOST_ENTRY(prefix##_4d) HOST_ENTRY(prefix##_nd) \
    HOST_ENTRY(prefix##_1d_simd) HOST_ENTRY(prefix##_2d_simd) \
    HOST_ENTRY(prefix##_3d_simd) HOST_ENTRY(prefix##_4d_simd) \
    HOST_ENTRY(prefix##_nd_simd)

HOST_ENTRIES_ND(starsh_ssdata_block_exp_kernel)
HOST_ENTRIES_ND(starsh_ssdata_block_sqrexp_kernel)
HOST_ENTRIES_ND(starsh_ssdata_block_matern_kernel)
HOST_ENTRIES_ND(starsh_ssdata_block_matern2_kernel)
HOST_ENTRIES_ND(starsh_esdata_block_coulomb_potential_kernel)
HOST_ENTRIES_ND(starsh_eddata_block_sin_kernel)
HOST_ENTRIES_ND(starsh_eddata_block_cos_kernel)
HOST_ENTRY(starsh_generate_3d_virus)
HOST_ENTRY(starsh_generate_3d_cube)

/* ----------------------------------------------------------- registry */

/* Kernel families by symbol name.  A name ends in _1d.._4d or _nd,
 * optionally followed by _simd (the SIMD variants compute the same
 * values). */
static const struct { const char *prefix; int family; } name_table[] =
{
    { "starsh_ssdata_block_exp_kernel_", STARSH_B200_FAMILY_EXP },
    { "starsh_ssdata_block_sqrexp_kernel_", STARSH_B200_FAMILY_SQREXP },
    { "starsh_ssdata_block_matern_kernel_", STARSH_B200_FAMILY_MATERN },
    { "starsh_ssdata_block_matern2_kernel_", STARSH_B200_FAMILY_MATERN2 },
    { "starsh_esdata_block_coulomb_potential_kernel_",
        STARSH_B200_FAMILY_COULOMB },
    { "starsh_eddata_block_sin_kernel_", STARSH_B200_FAMILY_SIN },
    { "starsh_eddata_block_cos_kernel_", STARSH_B200_FAMILY_COS },
};

#define MAX_REGISTERED 64
static struct { STARSH_kernel *fn; int family; double param; }
    registered[MAX_REGISTERED];
static int n_registered = 0;
static pthread_mutex_t registry_lock = PTHREAD_MUTEX_INITIALIZER;

int starsh_b200_kernel_register(STARSH_kernel *kernel, int family,
        double param)
{
    if(kernel == NULL || family < STARSH_B200_FAMILY_EXP ||
            family > STARSH_B200_FAMILY_RBF)
        return STARSH_WRONG_PARAMETER;
    int info = STARSH_SUCCESS;
    pthread_mutex_lock(&registry_lock);
    int slot = -1;
    for(int i = 0; i < n_registered; i++)
        if(registered[i].fn == kernel)
            slot = i;
    if(slot < 0 && n_registered < MAX_REGISTERED)
        slot = n_registered++;
    if(slot < 0)
        info = STARSH_WRONG_PARAMETER;
    else
    {
        registered[slot].fn = kernel;
        registered[slot].family = family;
        registered[slot].param = param;
    }
    pthread_mutex_unlock(&registry_lock);
    return info;
}

/* Family and dimension hint of a kernel known by name; 0 if unknown. */
static int family_by_name(const char *name, int *ndim_hint)
{
    if(name == NULL)
        return 0;
    if(strcmp(name, "starsh_generate_3d_virus") == 0 ||
            strcmp(name, "starsh_generate_3d_cube") == 0)
    {
        *ndim_hint = 3;
        return STARSH_B200_FAMILY_RBF;
    }
    for(size_t t = 0; t < sizeof(name_table)/sizeof(name_table[0]); t++)
    {
        size_t len = strlen(name_table[t].prefix);
        if(strncmp(name, name_table[t].prefix, len) != 0)
            continue;
        const char *suffix = name+len;
        if(suffix[0] == 'n' && suffix[1] == 'd')
            *ndim_hint = 0;
        else if(suffix[0] >= '1' && suffix[0] <= '4' && suffix[1] == 'd')
            *ndim_hint = suffix[0]-'0';
        else
            return 0;
        if(suffix[2] != '\0' && strcmp(suffix+2, "_simd") != 0)
            return 0;
        return name_table[t].family;
    }
    return 0;
}

static int lookup(STARSH_kernel *kernel, int *ndim_hint, double *param)
{
    *ndim_hint = 0;
    *param = 0.0;
    pthread_mutex_lock(&registry_lock);
    for(int i = 0; i < n_registered; i++)
        if(registered[i].fn == kernel)
        {
            int fam = registered[i].family;
            *param = registered[i].param;
            pthread_mutex_unlock(&registry_lock);
            if(fam == STARSH_B200_FAMILY_RBF)
                *ndim_hint = 3;
            return fam;
        }
    pthread_mutex_unlock(&registry_lock);
    Dl_info info;
    if(dladdr((void *)kernel, &info) == 0 || info.dli_saddr !=
            (void *)kernel)
        return 0;
    return family_by_name(info.dli_sname, ndim_hint);
}

int starsh_b200_kernel_family(STARSH_kernel *kernel, int *ndim_hint)
{
    int hint;
    double param;
    int fam = lookup(kernel, &hint, &param);
    if(ndim_hint != NULL)
        *ndim_hint = hint;
    return fam;
}

static double rbf_radius(const STARSH_mddata *m)
{
    /* Radius override of src/applications/mesh_deformation/virus.c:50-54;
     * its exponent (1/3) is integer division, i.e. 0. */
    double rad = m->rad;
    if(m->numobj > 1 && m->rad < 0 && m->denst < 0)
        rad = 0.25*m->numobj*sqrt(3.0);
    else if(m->numobj > 1 && m->rad < 0 && m->denst > 0)
        rad = sqrt(3.0)*(1.0+0.18);
    return rad;
}

int b200_resolve_kernel(STARSH_kernel *kernel, void *row_data,
        b200_kspec *spec, const double **row_points, STARSH_int *row_count,
        const double **col_points, STARSH_int *col_count, void *col_data)
{
    int hint;
    double param;
    int fam = lookup(kernel, &hint, &param);
    if(fam == 0 || row_data == NULL || col_data == NULL)
    {
        B200_ERROR("Kernel %p is not a recognised STARS-H kernel; register "
                "it with starsh_b200_kernel_register()", (void *)kernel);
        return STARSH_WRONG_PARAMETER;
    }
    memset(spec, 0, sizeof(*spec));
    spec->family = fam;
    /* Every supported data structure starts with STARSH_particles. */
    const STARSH_particles *rp = row_data, *cp = col_data;
    spec->ndim = rp->ndim;
    if(cp->ndim != rp->ndim || rp->ndim <= 0 || (hint && hint != rp->ndim))
    {
        B200_ERROR("Dimension of the points does not match the kernel");
        return STARSH_WRONG_PARAMETER;
    }
    *row_points = rp->point;
    *row_count = rp->count;
    *col_points = cp->point;
    *col_count = cp->count;
    switch(fam)
    {
        case STARSH_B200_FAMILY_EXP:
        case STARSH_B200_FAMILY_SQREXP:
        case STARSH_B200_FAMILY_MATERN:
        case STARSH_B200_FAMILY_MATERN2:
        {
            const STARSH_ssdata *s = row_data;
            spec->sigma = s->sigma;
            spec->beta = s->beta;
            spec->nu = s->nu;
            spec->noise = s->noise;
            if(fam == STARSH_B200_FAMILY_MATERN ||
                    fam == STARSH_B200_FAMILY_MATERN2)
            {
                if(s->nu <= 0)
                {
                    B200_ERROR("Matern kernels need nu > 0");
                    return STARSH_WRONG_PARAMETER;
                }
                /* Same operation order as kernel_matern.c:111-117:
                 * sigma*pow(2, 1-nu)/Gamma(nu), then *x^nu*K_nu(x). */
                spec->matern_coef = s->sigma*pow(2.0, 1.0-s->nu)/
                    tgamma(s->nu);
                spec->matern_scale = fam == STARSH_B200_FAMILY_MATERN ?
                    sqrt(2*s->nu)/s->beta : 0.0;
            }
            break;
        }
        case STARSH_B200_FAMILY_COULOMB:
            /* Reference value at r = 0 is 0; a registered kernel may ask
             * for another diagonal value. */
            spec->diag = param;
            spec->zero_mode = param != 0.0;
            break;
        case STARSH_B200_FAMILY_SIN:
        case STARSH_B200_FAMILY_COS:
        {
            const STARSH_eddata *e = row_data;
            spec->wave_k = e->k;
            spec->diag = e->diag;
            break;
        }
        case STARSH_B200_FAMILY_RBF:
        {
            const STARSH_mddata *m = row_data;
            if(rp->ndim != 3)
            {
                B200_ERROR("RBF kernels need 3-D meshes");
                return STARSH_WRONG_PARAMETER;
            }
            spec->aos = 1;
            spec->rbf_kind = m->kernel;
            spec->isreg = m->isreg;
            spec->reg = m->reg;
            spec->rad = rbf_radius(m);
            break;
        }
    }
    return STARSH_SUCCESS;
}
