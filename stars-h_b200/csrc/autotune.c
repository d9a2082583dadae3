/* Tile-size autotuner of the B200 engines: picks, per problem class, the
 * block size of the TLR format (the cluster size of
 * starsh_cluster_new_plain, reference src/control/cluster.c:106-146) that
 * compresses fastest on this GPU.
 *
 * For each candidate the tuner builds the plain clustering and TLR format
 * of the caller's problem, draws blocks of it at random (a fixed-seed
 * generator, with replacement), and times starsh_b200_approximate() on S
 * and on 2S of them (the first S again): the difference is the marginal
 * cost of S blocks, free of the fixed cost of a call (launches, set-up),
 * which a shared batched call pays once for all its problems.  The cost
 * per matrix entry decides.  Results are cached per class: kernel family,
 * the dimension its name fixes, N in half-octaves, tol in decades, engine
 * and the candidate list; the first problem of a class pays for the
 * measurement, the others reuse it. */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "starsh.h"
#include "starsh-b200.h"

#define TUNE_MAX_CAND 8
#define TUNE_CACHE 512
#define TUNE_SAMPLE 24

struct tune_key {
    int family, ndim, nbucket, tbucket, engine, ncand;
    int nb[TUNE_MAX_CAND], maxrank[TUNE_MAX_CAND];
};

struct tune_entry {
    struct tune_key key;
    int best;
    double cost[TUNE_MAX_CAND];
};

static struct tune_entry g_cache[TUNE_CACHE];
static int g_ncache = 0;
static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;

/* splitmix64: the block sampler's generator */
static uint64_t next_u64(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* Host milliseconds and matrix entries of one device-only approximation of
 * the first nblk blocks of `blocks` (pairs). */
static int time_blocks(STARSH_problem *P, STARSH_cluster *C,
                       const STARSH_int *blocks, STARSH_int nblk, int maxrank,
                       double tol, int engine, double *ms, double *entries)
{
    STARSH_int *far = malloc(sizeof(STARSH_int) * 2 * nblk);
    if (far == NULL) return STARSH_MALLOC_ERROR;
    memcpy(far, blocks, sizeof(STARSH_int) * 2 * nblk);
    STARSH_blrf *F = NULL;
    int info = starsh_blrf_new_from_coo(&F, P, 'N', C, C, nblk, far, 0, NULL,
                                        STARSH_TLR);
    if (info) {
        free(far);
        return info;
    }
    STARSH_blrm *M = NULL;
    info = starsh_b200_approximate(&M, F, maxrank, tol, 0, engine, 0);
    if (info == STARSH_SUCCESS) {
        starsh_b200_stats st;
        starsh_b200_get_stats(&st);
        *ms = st.total_ms;
        *entries = (double)st.entries;
        starsh_blrm_free(M);
    }
    starsh_blrf_free(F);
    return info;
}

/* Marginal cost (ns per entry) of compressing blocks of the tile size nb. */
static int measure(STARSH_problem *P, int nb, int maxrank, double tol,
                   int engine, double *cost)
{
    const STARSH_int n = P->shape[0];
    STARSH_cluster *C = NULL;
    int info = starsh_cluster_new_plain(&C, P->row_data, n, nb);
    if (info) return info;
    const STARSH_int nt = C->nblocks;
    STARSH_int blocks[4 * TUNE_SAMPLE];
    uint64_t seed = 0x5354415253480002ull;
    for (int q = 0; q < 2 * TUNE_SAMPLE; ++q) {
        const STARSH_int b = (STARSH_int)(next_u64(&seed) % (uint64_t)(nt * nt));
        blocks[2 * q] = b / nt;
        blocks[2 * q + 1] = b % nt;
    }
    double t1 = 0, e1 = 0, t1b = 0, e1b = 0, t2 = 0, e2 = 0;
    /* S blocks twice (the first call of a shape may set up the engine's
     * sketch matrices), then 2S blocks */
    info = time_blocks(P, C, blocks, TUNE_SAMPLE, maxrank, tol, engine, &t1, &e1);
    if (!info)
        info = time_blocks(P, C, blocks, TUNE_SAMPLE, maxrank, tol, engine, &t1b, &e1b);
    if (!info)
        info = time_blocks(P, C, blocks, 2 * TUNE_SAMPLE, maxrank, tol, engine,
                           &t2, &e2);
    starsh_cluster_free(C);
    if (info) return info;
    const double ts = t1 < t1b ? t1 : t1b;
    double dt = t2 - ts, de = e2 - e1;
    /* timing noise larger than the marginal cost: fall back to the mean */
    if (!(dt > 0.0) || !(de > 0.0)) {
        dt = t2;
        de = e2;
    }
    *cost = de > 0.0 ? dt * 1e6 / de : INFINITY;
    return STARSH_SUCCESS;
}

int starsh_b200_autotune_tile(STARSH_problem *problem, int ncand,
                              const int *cand_nb, const int *cand_maxrank,
                              double tol, int engine, int *best_nb,
                              double *costs)
{
    if (problem == NULL || ncand <= 0 || ncand > TUNE_MAX_CAND ||
        cand_nb == NULL || cand_maxrank == NULL || best_nb == NULL ||
        !(tol > 0.0) || problem->ndim != 2)
        return STARSH_WRONG_PARAMETER;
    const STARSH_int n = problem->shape[0];
    struct tune_key key;
    memset(&key, 0, sizeof(key));
    key.family = starsh_b200_kernel_family(problem->kernel, &key.ndim);
    if (key.family == 0) return STARSH_WRONG_PARAMETER;
    key.nbucket = (int)floor(2.0 * log2((double)n));
    key.tbucket = (int)floor(log10(tol));
    key.engine = engine;
    key.ncand = ncand;
    for (int c = 0; c < ncand; ++c) {
        if (cand_nb[c] <= 0 || cand_maxrank[c] < 0) return STARSH_WRONG_PARAMETER;
        key.nb[c] = cand_nb[c];
        key.maxrank[c] = cand_maxrank[c];
    }
    pthread_mutex_lock(&g_lock);
    for (int q = 0; q < g_ncache; ++q)
        if (memcmp(&g_cache[q].key, &key, sizeof(key)) == 0) {
            *best_nb = g_cache[q].key.nb[g_cache[q].best];
            if (costs)
                memcpy(costs, g_cache[q].cost, sizeof(double) * ncand);
            pthread_mutex_unlock(&g_lock);
            return STARSH_SUCCESS;
        }
    pthread_mutex_unlock(&g_lock);
    struct tune_entry e;
    e.key = key;
    e.best = -1;
    for (int c = 0; c < ncand; ++c) {
        e.cost[c] = INFINITY;
        if (cand_nb[c] > n) continue;
        int info = measure(problem, cand_nb[c], cand_maxrank[c], tol, engine,
                           &e.cost[c]);
        if (info) return info;
        if (e.best < 0 || e.cost[c] < e.cost[e.best]) e.best = c;
    }
    if (e.best < 0) return STARSH_WRONG_PARAMETER;
    pthread_mutex_lock(&g_lock);
    if (g_ncache < TUNE_CACHE) g_cache[g_ncache++] = e;
    pthread_mutex_unlock(&g_lock);
    *best_nb = cand_nb[e.best];
    if (costs) memcpy(costs, e.cost, sizeof(double) * ncand);
    return STARSH_SUCCESS;
}

void starsh_b200_autotune_clear(void)
{
    pthread_mutex_lock(&g_lock);
    g_ncache = 0;
    pthread_mutex_unlock(&g_lock);
}
