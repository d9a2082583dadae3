/* CPU restatement of the STARS-H TLR-path primitives -- TEST INFRASTRUCTURE.
 *
 * This file is the checker for libstarsh_b200, never part of it: only the
 * tests, the smoke check and the CPU-baseline leg of bench.py load the
 * library built from it (oracle/_ref/liboracle.so).  Each function restates
 * the reference routine named beside it in plain scalar C so that the
 * restatement itself can be pinned against the compiled reference
 * (oracle/_ref/libstarsh_ref.so) by tests/test_oracle.py.
 *
 * Matérn entries need K_nu, which the reference takes from GSL (absent
 * here); their checker is the mpmath golden file tests/golden/matern.npz,
 * not this file.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------- point sets */

/* src/applications/particles.c:1166-1221 (radix_sort_recursive): split
 * order[lo..hi] on one bit of one dimension, zeros forward, ones filled
 * from the back (reversing their order), recurse on dimension-1, wrapping
 * to the next lower bit after dimension 0. */
static void split(const uint32_t *key, long long n, int ndim, long long *ord,
                  long long *tmp, int dim, int bit, long long lo, long long hi)
{
    long long a = lo, b = hi;
    for (long long i = lo; i <= hi; i++)
    {
        if ((key[(size_t)dim*n+ord[i]] >> bit) & 1u)
            tmp[b--] = ord[i];
        else
            tmp[a++] = ord[i];
    }
    for (long long i = lo; i <= hi; i++)
        ord[i] = tmp[i];
    int nd = dim > 0 ? dim-1 : ndim-1;
    int nb = dim > 0 ? bit : bit-1;
    if (dim == 0 && bit == 0)
        return;
    if (a-lo > 1)
        split(key, n, ndim, ord, tmp, nd, nb, lo, a-1);
    if (hi-b > 1)
        split(key, n, ndim, ord, tmp, nd, nb, b+1, hi);
}

/* src/applications/particles.c:1090-1164 (starsh_particles_zsort_inplace)*/
int oracle_zsort(long long n, int ndim, double *pt)
{
    uint32_t *key = malloc(sizeof(*key)*(size_t)n*ndim);
    long long *ord = malloc(sizeof(*ord)*(size_t)n);
    long long *tmp = malloc(sizeof(*tmp)*(size_t)n);
    double *out = malloc(sizeof(*out)*(size_t)n*ndim);
    if (!key || !ord || !tmp || !out)
        return 1;
    for (int d = 0; d < ndim; d++)
    {
        double *x = pt+(size_t)d*n, mn = x[0], mx = x[0];
        for (long long i = 1; i < n; i++)
        {
            if (mn > x[i]) mn = x[i];
            else if (mx < x[i]) mx = x[i];
        }
        for (long long i = 0; i < n; i++)
            key[(size_t)d*n+i] = (x[i]-mn)/(mx-mn)*UINT32_MAX;
    }
    for (long long i = 0; i < n; i++)
        ord[i] = i;
    if (n > 1)
        split(key, n, ndim, ord, tmp, ndim-1, 31, 0, n-1);
    for (long long i = 0; i < n; i++)
        for (int d = 0; d < ndim; d++)
            out[(size_t)d*n+i] = pt[(size_t)d*n+ord[i]];
    memcpy(pt, out, sizeof(*out)*(size_t)n*ndim);
    free(key); free(ord); free(tmp); free(out);
    return 0;
}

/* src/applications/particles.c:177-201 (RAND, before the sort). */
void oracle_points_rand(long long n, int ndim, double *pt)
{
    for (size_t i = 0; i < (size_t)n*ndim; i++)
        pt[i] = (double)rand()/RAND_MAX;
    oracle_zsort(n, ndim, pt);
}

/* src/applications/particles.c:260-333 (UNIFORM) and :341-411
 * (QUASIUNIFORM1): grid nodes i/side in lexicographic order, last
 * dimension fastest; QUASIUNIFORM1 adds 0.1/side + 0.8/side/RAND_MAX*rand()
 * to every coordinate. */
int oracle_points_grid(long long n, int ndim, int jitter, double *pt)
{
    long long side = (long long)ceil(pow((double)n, 1.0/ndim));
    long long *idx = calloc(ndim, sizeof(*idx));
    if (!idx)
        return 1;
    double mult = 0.8/side/RAND_MAX, add = 0.1/side;
    for (long long i = 0; i < n; i++)
    {
        for (int d = 0; d < ndim; d++)
        {
            double c = (double)idx[d]/side;
            pt[i+(size_t)d*n] = jitter ? c+add+mult*rand() : c;
        }
        int d = ndim-1;
        idx[d]++;
        while (idx[d] == side && d > 0)
        {
            idx[d] = 0;
            idx[--d]++;
        }
    }
    free(idx);
    return oracle_zsort(n, ndim, pt);
}

/* ------------------------------------------------------------ kernels */

/* Parameters of oracle_block, by index. */
enum { P_SIGMA, P_BETA, P_NU, P_NOISE, P_WAVEK, P_DIAG, P_RAD, P_REG,
       P_ISREG, P_RBFKIND, P_ZERO_DIAG, P_COUNT };

/* One block of a kernel matrix with rows irow[] and columns icol[].
 * family: 1 exp (kernel_exp.c:93-109), 2 sqexp (kernel_sqrexp.c:94-110),
 * 5 Coulomb (kernel_coulomb_potential.c:83-97; r = 0 gives par[P_DIAG] when
 * par[P_ZERO_DIAG] != 0, else 0), 6 sin (kernel_sin.c:88-104),
 * 7 cos (kernel_cos.c:88-104), 8 RBF on point-major 3-D meshes
 * (mesh_deformation/virus.c:56-91 with kernels_rbf.c:29-121). */
void oracle_block(int family, int ndim, const double *pr, long long cr,
                  const double *pc, long long cc, const long long *irow,
                  const long long *icol, int m, int n, const double *par,
                  double *out, int ld)
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++)
        {
            long long a = irow[i], b = icol[j];
            double dist = 0.0, v;
            if (family == 8)
            {
                for (int d = 0; d < 3; d++)
                    dist += pow(pr[3*a+d]-pc[3*b+d], 2);
                double x = pow(dist, 0.5)/par[P_RAD];
                switch ((int)par[P_RBFKIND])
                {
                    case 0: v = exp(-pow(x, 2)); break;
                    case 1: v = exp(-x); break;
                    case 2: v = 1/(1+pow(x, 2)); break;
                    case 3: v = 1/sqrt(1+pow(x, 2)); break;
                    case 4: case 5: v = exp(-x)+(1+x); break;
                    case 6: v = pow(x, 2)*log(x); break;
                    case 7: v = x > 1 ? 0 : pow(1-x, 5); break;
                    case 8: v = 1+pow(x, 2); break;
                    default: v = x > 1 ? 0 : pow(1-x, 4)*(4*x+1);
                }
                if ((int)a == (int)b && par[P_ISREG] != 0)
                    v += par[P_REG];
                out[(size_t)j*ld+i] = v;
                continue;
            }
            for (int d = 0; d < ndim; d++)
            {
                double t = pr[(size_t)d*cr+a]-pc[(size_t)d*cc+b];
                dist += t*t;
            }
            switch (family)
            {
                case 1:
                    dist = sqrt(dist)/(-par[P_BETA]);
                    v = dist == 0 ? par[P_SIGMA]+par[P_NOISE]
                                  : par[P_SIGMA]*exp(dist);
                    break;
                case 2:
                    dist = dist/(-2*par[P_BETA]*par[P_BETA]);
                    v = dist == 0 ? par[P_SIGMA]+par[P_NOISE]
                                  : par[P_SIGMA]*exp(dist);
                    break;
                case 5:
                    v = dist == 0 ? (par[P_ZERO_DIAG] != 0 ? par[P_DIAG] : 0)
                                  : 1.0/sqrt(dist);
                    break;
                case 6:
                case 7:
                    if (dist == 0)
                        v = par[P_DIAG];
                    else
                    {
                        dist = sqrt(dist);
                        v = (family == 6 ? sin(par[P_WAVEK]*dist)
                                         : cos(par[P_WAVEK]*dist))/dist;
                    }
                    break;
                default:
                    v = NAN;
            }
            out[(size_t)j*ld+i] = v;
        }
}

/* ------------------------------------------------------------ rank cut */

/* src/backends/sequential/dense/dsvfr.c:16-47: smallest rank r >= 1 whose
 * discarded tail sum_{i >= r} S_i^2 is <= tol^2 sum S_i^2 (0 if S = 0). */
int oracle_dsvfr(int size, const double *S, double tol)
{
    double total = 0;
    for (int i = 0; i < size; i++)
        total += S[i]*S[i];
    if (total == 0)
        return 0;
    double budget = total*tol*tol, tail = S[size-1]*S[size-1];
    int r = size;
    while (r > 1 && budget >= tail)
    {
        r--;
        tail += S[r-1]*S[r-1];
    }
    return r;
}

/* ------------------------------------------------ regularised Coulomb */

/* The Coulomb kernel with a unit diagonal, as a STARSH_kernel that a
 * reference-built problem can carry: the reference entry point fills the
 * block (kernel_coulomb_potential.c emits 0 at r = 0) and this wrapper sets
 * the r = 0 entries to 1.  `ref_kernel` must be set to the reference's
 * starsh_esdata_block_coulomb_potential_kernel_* before use. */
typedef void kernel_fn(int, int, long long *, long long *, void *, void *,
                       void *, int);
kernel_fn *oracle_coulomb_ref_kernel = NULL;

void oracle_coulomb_unit_diag(int m, int n, long long *irow, long long *icol,
                              void *rd, void *cd, void *result, int ld)
{
    double *out = result;
    oracle_coulomb_ref_kernel(m, n, irow, icol, rd, cd, result, ld);
    /* the point sets start with (count, ndim, point) */
    struct { long long count; int ndim; double *point; } *p = rd, *q = cd;
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++)
        {
            double dist = 0;
            for (int d = 0; d < p->ndim; d++)
            {
                double t = p->point[(size_t)d*p->count+irow[i]]-
                    q->point[(size_t)d*q->count+icol[j]];
                dist += t*t;
            }
            if (dist == 0)
                out[(size_t)j*ld+i] = 1.0;
        }
}
