/* Files and byte streams: particle sets in the reference's ASCII and binary
 * formats, and a block-low-rank matrix (STARSH_blrm) as a self-checking
 * byte stream.
 *
 * Particle files follow src/applications/particles.c:789-1088 of the
 * reference, so that files move both ways between the two libraries:
 *   ASCII   "count=<count>, ndim=<ndim>\n", then one line per point, its
 *           coordinates printed with "%lf" and separated by ", ";
 *   binary  count (size_t), ndim (int), then the count*ndim doubles of
 *           `point` as they lie in memory (coordinate-major).
 * Error codes are the reference's: STARSH_FILE_NOT_EXIST when the file
 * cannot be opened, STARSH_FILE_WRONG_INPUT for a malformed or short file,
 * STARSH_FPRINTF_ERROR / STARSH_FWRITE_ERROR when writing fails.
 *
 * The reference has no serialised form of a STARSH_blrm.  The stream
 * written here (version 1, little-endian, every integer 64-bit unless
 * stated) is
 *   "STARSHTL"                        8-byte magic
 *   u32 version, u32 flags            1 symmetric format ('S'), 2 onfly,
 *                                     4 columns use the row clustering
 *   nrows, ncols, nbrows, nbcols, nblocks_far, nblocks_near, format type
 *   row clustering: pivot[nrows], start[nbrows], size[nbrows]
 *   column clustering (unless flag 4): pivot[ncols], start[nbcols],
 *                                     size[nbcols]
 *   block_far[2 nblocks_far], block_near[2 nblocks_near]
 *   rank[nblocks_far] (int64)
 *   U then V of every far block (doubles, column-major, leading dimension
 *   the block's rows / columns), in block order
 *   the dense near blocks (unless onfly), in block order
 *   u64 checksum of every preceding byte
 * A stream is bound back to a STARSH_problem of the same shape and
 * symmetry when read; its factors land on the host, and the device entry
 * points (dmml, dfe, CG) upload them on first use as for any host-resident
 * matrix. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "starsh.h"
#include "starsh-b200.h"
#include "starsh-particles.h"
#include "b200_host.h"

/* ------------------------------------------------------------ particles */

int starsh_particles_read_from_file_pointer_ascii(STARSH_particles **data,
        FILE *fp)
{
    if(data == NULL || fp == NULL)
        return STARSH_WRONG_PARAMETER;
    size_t count;
    int ndim;
    if(fscanf(fp, "count=%zu, ndim=%d", &count, &ndim) != 2 || ndim <= 0 ||
            count == 0 || count > (SIZE_MAX/sizeof(double))/(size_t)ndim)
        return STARSH_FILE_WRONG_INPUT;
    double *point = malloc(sizeof(*point)*count*(size_t)ndim);
    STARSH_particles *p = malloc(sizeof(*p));
    if(point == NULL || p == NULL)
    {
        free(point);
        free(p);
        return STARSH_MALLOC_ERROR;
    }
    /* Point i is one record: its first coordinate after optional white
     * space, then each further coordinate right after a comma. */
    for(size_t i = 0; i < count; i++)
        for(int d = 0; d < ndim; d++)
            if(fscanf(fp, d == 0 ? "%lf" : ",%lf", point+(size_t)d*count+i)
                    != 1)
            {
                free(point);
                free(p);
                return STARSH_FILE_WRONG_INPUT;
            }
    p->count = (STARSH_int)count;
    p->ndim = ndim;
    p->point = point;
    *data = p;
    return STARSH_SUCCESS;
}

int starsh_particles_read_from_file_pointer_binary(STARSH_particles **data,
        FILE *fp)
{
    if(data == NULL || fp == NULL)
        return STARSH_WRONG_PARAMETER;
    size_t count;
    int ndim;
    if(fread(&count, sizeof(count), 1, fp) != 1 ||
            fread(&ndim, sizeof(ndim), 1, fp) != 1 || ndim <= 0 ||
            count == 0 || count > (SIZE_MAX/sizeof(double))/(size_t)ndim)
        return STARSH_FILE_WRONG_INPUT;
    const size_t nmemb = count*(size_t)ndim;
    /* A seekable file shorter than its header claims is refused before
     * the allocation. */
    long here = ftell(fp);
    if(here >= 0 && fseek(fp, 0, SEEK_END) == 0)
    {
        long end = ftell(fp);
        fseek(fp, here, SEEK_SET);
        if(end >= here && (size_t)(end-here)/sizeof(double) < nmemb)
            return STARSH_FILE_WRONG_INPUT;
    }
    double *point = malloc(sizeof(*point)*nmemb);
    STARSH_particles *p = malloc(sizeof(*p));
    if(point == NULL || p == NULL)
    {
        free(point);
        free(p);
        return STARSH_MALLOC_ERROR;
    }
    if(fread(point, sizeof(*point), nmemb, fp) != nmemb)
    {
        free(point);
        free(p);
        return STARSH_FILE_WRONG_INPUT;
    }
    p->count = (STARSH_int)count;
    p->ndim = ndim;
    p->point = point;
    *data = p;
    return STARSH_SUCCESS;
}

int starsh_particles_read_from_file_pointer(STARSH_particles **data,
        FILE *fp, const enum STARSH_FILE_TYPE ftype)
{
    if(ftype == STARSH_ASCII)
        return starsh_particles_read_from_file_pointer_ascii(data, fp);
    if(ftype == STARSH_BINARY)
        return starsh_particles_read_from_file_pointer_binary(data, fp);
    return STARSH_WRONG_PARAMETER;
}

int starsh_particles_read_from_file(STARSH_particles **data,
        const char *fname, const enum STARSH_FILE_TYPE ftype)
{
    if(ftype != STARSH_ASCII && ftype != STARSH_BINARY)
        return STARSH_WRONG_PARAMETER;
    if(fname == NULL)
        return STARSH_WRONG_PARAMETER;
    FILE *fp = fopen(fname, ftype == STARSH_ASCII ? "r" : "rb");
    if(fp == NULL)
        return STARSH_FILE_NOT_EXIST;
    int info = starsh_particles_read_from_file_pointer(data, fp, ftype);
    fclose(fp);
    return info;
}

int starsh_particles_write_to_file_pointer_ascii(const STARSH_particles *data,
        FILE *fp)
{
    if(data == NULL || fp == NULL || data->point == NULL)
        return STARSH_WRONG_PARAMETER;
    const size_t count = (size_t)data->count;
    const int ndim = data->ndim;
    if(fprintf(fp, "count=%zu, ndim=%d\n", count, ndim) < 0)
        return STARSH_FPRINTF_ERROR;
    for(size_t i = 0; i < count; i++)
    {
        for(int d = 0; d < ndim; d++)
            if(fprintf(fp, d == 0 ? "%lf" : ", %lf",
                        data->point[(size_t)d*count+i]) < 0)
                return STARSH_FPRINTF_ERROR;
        if(fputc('\n', fp) == EOF)
            return STARSH_FPRINTF_ERROR;
    }
    return STARSH_SUCCESS;
}

int starsh_particles_write_to_file_pointer_binary(const STARSH_particles *data,
        FILE *fp)
{
    if(data == NULL || fp == NULL || data->point == NULL)
        return STARSH_WRONG_PARAMETER;
    const size_t count = (size_t)data->count;
    const int ndim = data->ndim;
    const size_t nmemb = count*(size_t)ndim;
    if(fwrite(&count, sizeof(count), 1, fp) != 1 ||
            fwrite(&ndim, sizeof(ndim), 1, fp) != 1 ||
            fwrite(data->point, sizeof(double), nmemb, fp) != nmemb)
        return STARSH_FWRITE_ERROR;
    return STARSH_SUCCESS;
}

int starsh_particles_write_to_file_pointer(const STARSH_particles *data,
        FILE *fp, const enum STARSH_FILE_TYPE ftype)
{
    if(ftype == STARSH_ASCII)
        return starsh_particles_write_to_file_pointer_ascii(data, fp);
    if(ftype == STARSH_BINARY)
        return starsh_particles_write_to_file_pointer_binary(data, fp);
    return STARSH_WRONG_PARAMETER;
}

int starsh_particles_write_to_file(const STARSH_particles *data,
        const char *fname, const enum STARSH_FILE_TYPE ftype)
{
    if(ftype != STARSH_ASCII && ftype != STARSH_BINARY)
        return STARSH_WRONG_PARAMETER;
    if(fname == NULL)
        return STARSH_WRONG_PARAMETER;
    FILE *fp = fopen(fname, ftype == STARSH_ASCII ? "w" : "wb");
    if(fp == NULL)
        return STARSH_FILE_NOT_EXIST;
    int info = starsh_particles_write_to_file_pointer(data, fp, ftype);
    if(fclose(fp) != 0 && info == STARSH_SUCCESS)
        info = ftype == STARSH_ASCII ? STARSH_FPRINTF_ERROR :
            STARSH_FWRITE_ERROR;
    return info;
}

/* ------------------------------------------------------ STARSH_blrm stream */

/* Streaming 64-bit checksum: the body and finaliser of MurmurHash3 x64
 * (Austin Appleby, public domain) applied to the stream's little-endian
 * 64-bit words, the final partial word and the length folded in last. */
typedef struct
{
    uint64_t h;
    uint64_t tail;
    unsigned ntail;
    uint64_t total;
} tl_hash;

static uint64_t tl_mix(uint64_t h, uint64_t w)
{
    w *= 0x87c37b91114253d5ull;
    w = (w << 31) | (w >> 33);
    w *= 0x4cf5ad432745937full;
    h ^= w;
    h = (h << 27) | (h >> 37);
    return h*5+0x52dce729;
}

static void tl_hash_bytes(tl_hash *t, const void *ptr, size_t n)
{
    const unsigned char *p = ptr;
    t->total += n;
    while(n > 0 && t->ntail != 0)
    {
        t->tail |= (uint64_t)*p++ << (8*t->ntail);
        n--;
        if(++t->ntail == 8)
        {
            t->h = tl_mix(t->h, t->tail);
            t->tail = 0;
            t->ntail = 0;
        }
    }
    for(; n >= 8; n -= 8, p += 8)
    {
        uint64_t w;
        memcpy(&w, p, 8);
        t->h = tl_mix(t->h, w);
    }
    for(; n > 0; n--)
        t->tail |= (uint64_t)*p++ << (8*t->ntail++);
}

static uint64_t tl_hash_final(const tl_hash *t)
{
    uint64_t h = tl_mix(t->h, t->tail) ^ t->total;
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    return h;
}

static const char tl_magic[8] = {'S', 'T', 'A', 'R', 'S', 'H', 'T', 'L'};
enum { TL_VERSION = 1, TL_SYMM = 1, TL_ONFLY = 2, TL_SHARED_CLUSTER = 4 };

/* Where a stream goes: a FILE, a memory buffer, or nowhere (counting).  A
 * buffer that is too small stops the copying but not the counting, so that
 * the size needed is known at the end. */
typedef struct
{
    FILE *fp;
    unsigned char *buf;
    size_t cap, pos;
    int err, overflow;
    tl_hash hash;
} tl_sink;

static void tl_put(tl_sink *s, const void *p, size_t n)
{
    if(s->err || n == 0)
        return;
    tl_hash_bytes(&s->hash, p, n);
    if(s->fp != NULL)
    {
        if(fwrite(p, 1, n, s->fp) != n)
            s->err = STARSH_FWRITE_ERROR;
    }
    else if(s->buf != NULL && !s->overflow)
    {
        if(s->cap-s->pos < n)
            s->overflow = 1;
        else
            memcpy(s->buf+s->pos, p, n);
    }
    s->pos += n;
}

static void tl_put_i64(tl_sink *s, int64_t v)
{
    tl_put(s, &v, sizeof(v));
}

/* Clustering of one side: pivot, then start and size of every block. */
static void tl_put_cluster(tl_sink *s, const STARSH_cluster *C)
{
    for(STARSH_int i = 0; i < C->ndata; i++)
        tl_put_i64(s, C->pivot != NULL ? C->pivot[i] : i);
    for(STARSH_int b = 0; b < C->nblocks; b++)
        tl_put_i64(s, C->start[b]);
    for(STARSH_int b = 0; b < C->nblocks; b++)
        tl_put_i64(s, C->size[b]);
}

static int tl_write(STARSH_blrm *M, tl_sink *s)
{
    if(M == NULL || M->format == NULL || M->format->problem == NULL)
        return STARSH_WRONG_PARAMETER;
    STARSH_blrf *F = M->format;
    STARSH_problem *P = F->problem;
    STARSH_cluster *R = F->row_cluster, *C = F->col_cluster;
    if(P->ndim != 2 || P->dtype != 'd' || R == NULL || C == NULL ||
            R->ndata != P->shape[0] || C->ndata != P->shape[1])
        return STARSH_WRONG_PARAMETER;
    for(STARSH_int b = 0; b < F->nblocks_far; b++)
        if(M->far_rank[b] < 0)
            return STARSH_WRONG_PARAMETER;
    /* Factors of a device-resident result are brought to the host first
     * (nothing happens for a host matrix). */
    int info = starsh_b200_blrm_download(M);
    if(info != STARSH_SUCCESS)
        return info;
    uint32_t head[2] = {TL_VERSION, 0};
    if(F->symm == 'S')
        head[1] |= TL_SYMM;
    if(M->onfly)
        head[1] |= TL_ONFLY;
    if(R == C)
        head[1] |= TL_SHARED_CLUSTER;
    tl_put(s, tl_magic, sizeof(tl_magic));
    tl_put(s, head, sizeof(head));
    tl_put_i64(s, P->shape[0]);
    tl_put_i64(s, P->shape[1]);
    tl_put_i64(s, R->nblocks);
    tl_put_i64(s, C->nblocks);
    tl_put_i64(s, F->nblocks_far);
    tl_put_i64(s, F->nblocks_near);
    tl_put_i64(s, F->type);
    tl_put_cluster(s, R);
    if(R != C)
        tl_put_cluster(s, C);
    for(STARSH_int b = 0; b < 2*F->nblocks_far; b++)
        tl_put_i64(s, F->block_far[b]);
    for(STARSH_int b = 0; b < 2*F->nblocks_near; b++)
        tl_put_i64(s, F->block_near[b]);
    for(STARSH_int b = 0; b < F->nblocks_far; b++)
        tl_put_i64(s, M->far_rank[b]);
    for(STARSH_int b = 0; b < F->nblocks_far; b++)
    {
        const size_t r = (size_t)M->far_rank[b];
        const size_t m = (size_t)R->size[F->block_far[2*b]];
        const size_t n = (size_t)C->size[F->block_far[2*b+1]];
        if(r == 0)
            continue;
        tl_put(s, M->far_U[b]->data, m*r*sizeof(double));
        tl_put(s, M->far_V[b]->data, n*r*sizeof(double));
    }
    if(!M->onfly)
        for(STARSH_int b = 0; b < F->nblocks_near; b++)
        {
            const size_t m = (size_t)R->size[F->block_near[2*b]];
            const size_t n = (size_t)C->size[F->block_near[2*b+1]];
            tl_put(s, M->near_D[b]->data, m*n*sizeof(double));
        }
    uint64_t sum = tl_hash_final(&s->hash);
    tl_hash snapshot = s->hash;
    tl_put(s, &sum, sizeof(sum));
    s->hash = snapshot;
    return s->err;
}

int starsh_b200_blrm_write_to_file_pointer(STARSH_blrm *matrix, FILE *fp)
{
    if(fp == NULL)
        return STARSH_WRONG_PARAMETER;
    tl_sink s = {0};
    s.fp = fp;
    return tl_write(matrix, &s);
}

int starsh_b200_blrm_write_to_file(STARSH_blrm *matrix, const char *fname)
{
    if(matrix == NULL || fname == NULL)
        return STARSH_WRONG_PARAMETER;
    FILE *fp = fopen(fname, "wb");
    if(fp == NULL)
        return STARSH_FILE_NOT_EXIST;
    int info = starsh_b200_blrm_write_to_file_pointer(matrix, fp);
    if(fclose(fp) != 0 && info == STARSH_SUCCESS)
        info = STARSH_FWRITE_ERROR;
    return info;
}

int starsh_b200_blrm_serialize(STARSH_blrm *matrix, void *buffer,
        size_t capacity, size_t *nbytes)
{
    if(nbytes == NULL)
        return STARSH_WRONG_PARAMETER;
    tl_sink s = {0};
    s.buf = buffer;
    s.cap = buffer != NULL ? capacity : 0;
    int info = tl_write(matrix, &s);
    *nbytes = s.pos;
    if(info == STARSH_SUCCESS && s.overflow)
        info = STARSH_WRONG_PARAMETER;
    return info;
}

/* Where a stream comes from: a FILE or a memory buffer. */
typedef struct
{
    FILE *fp;
    const unsigned char *buf;
    size_t size, pos;
    int err;
    tl_hash hash;
} tl_source;

static int tl_get(tl_source *s, void *p, size_t n)
{
    if(s->err)
        return s->err;
    if(n == 0)
        return STARSH_SUCCESS;
    if(s->fp != NULL)
    {
        if(fread(p, 1, n, s->fp) != n)
            s->err = STARSH_FILE_WRONG_INPUT;
    }
    else if(s->size-s->pos < n)
        s->err = STARSH_FILE_WRONG_INPUT;
    else
        memcpy(p, s->buf+s->pos, n);
    if(!s->err)
    {
        tl_hash_bytes(&s->hash, p, n);
        s->pos += n;
    }
    return s->err;
}

/* Bytes left in the source, or SIZE_MAX when that cannot be known (a pipe). */
static size_t tl_remaining(tl_source *s)
{
    if(s->fp == NULL)
        return s->size-s->pos;
    long here = ftell(s->fp);
    if(here < 0 || fseek(s->fp, 0, SEEK_END) != 0)
        return SIZE_MAX;
    long end = ftell(s->fp);
    fseek(s->fp, here, SEEK_SET);
    return end >= here ? (size_t)(end-here) : 0;
}

/* Reads n int64 values after checking that the source can hold them. */
static int64_t *tl_get_i64s(tl_source *s, int64_t n)
{
    if(n < 0 || (uint64_t)n > tl_remaining(s)/8)
    {
        s->err = STARSH_FILE_WRONG_INPUT;
        return NULL;
    }
    int64_t *v = malloc(sizeof(*v)*(n > 0 ? (size_t)n : 1));
    if(v == NULL)
    {
        s->err = STARSH_MALLOC_ERROR;
        return NULL;
    }
    if(tl_get(s, v, sizeof(*v)*(size_t)n) != STARSH_SUCCESS)
    {
        free(v);
        return NULL;
    }
    return v;
}

/* A plain clustering of ndata items into nblocks consecutive blocks that
 * cover every item once, with pivots inside [0, ndata). */
static int tl_cluster_valid(int64_t ndata, int64_t nblocks,
        const int64_t *pivot, const int64_t *start, const int64_t *size)
{
    int64_t next = 0;
    for(int64_t b = 0; b < nblocks; b++)
    {
        if(start[b] != next || size[b] <= 0 || size[b] > ndata-next ||
                size[b] > INT32_MAX)
            return 0;
        next += size[b];
    }
    if(next != ndata)
        return 0;
    for(int64_t i = 0; i < ndata; i++)
        if(pivot[i] < 0 || pivot[i] >= ndata)
            return 0;
    return 1;
}

static int tl_read(STARSH_blrm **matrix, STARSH_problem *P, tl_source *s)
{
    if(matrix == NULL || P == NULL || P->ndim != 2 || P->dtype != 'd')
        return STARSH_WRONG_PARAMETER;
    char magic[8];
    uint32_t head[2];
    int64_t h[7];
    if(tl_get(s, magic, sizeof(magic)) || memcmp(magic, tl_magic, 8) != 0 ||
            tl_get(s, head, sizeof(head)) || head[0] != TL_VERSION ||
            tl_get(s, h, sizeof(h)))
        return STARSH_FILE_WRONG_INPUT;
    const int symm = (head[1] & TL_SYMM) != 0;
    const int onfly = (head[1] & TL_ONFLY) != 0;
    const int shared = (head[1] & TL_SHARED_CLUSTER) != 0;
    const int64_t nrows = h[0], ncols = h[1], nbrows = h[2], nbcols = h[3];
    const int64_t nfar = h[4], nnear = h[5];
    if(nrows != P->shape[0] || ncols != P->shape[1] ||
            (symm && (P->symm != 'S' || !shared)))
        return STARSH_WRONG_PARAMETER;
    if((head[1] & ~7u) != 0 || nbrows <= 0 || nbrows > nrows ||
            nbcols <= 0 || nbcols > ncols || (shared && (nrows != ncols ||
            nbrows != nbcols)) || nfar < 0 || nnear < 0 ||
            nfar > nbrows*nbcols || nnear > nbrows*nbcols ||
            h[6] < 0 || h[6] > INT32_MAX)
        return STARSH_FILE_WRONG_INPUT;
    int info = STARSH_SUCCESS;
    int64_t *rpiv = NULL, *rstart = NULL, *rsize = NULL;
    int64_t *cpiv = NULL, *cstart = NULL, *csize = NULL;
    int64_t *far = NULL, *near = NULL, *rank64 = NULL;
    int *rank = NULL;
    double *aU = NULL, *aV = NULL, *aD = NULL;
    Array **U = NULL, **V = NULL, **D = NULL;
    STARSH_cluster *R = NULL, *C = NULL;
    STARSH_blrf *F = NULL;
    rpiv = tl_get_i64s(s, nrows);
    rstart = tl_get_i64s(s, nbrows);
    rsize = tl_get_i64s(s, nbrows);
    if(!shared)
    {
        cpiv = tl_get_i64s(s, ncols);
        cstart = tl_get_i64s(s, nbcols);
        csize = tl_get_i64s(s, nbcols);
    }
    far = tl_get_i64s(s, 2*nfar);
    near = tl_get_i64s(s, 2*nnear);
    rank64 = tl_get_i64s(s, nfar);
    if(s->err)
    {
        info = s->err;
        goto fail;
    }
    const int64_t *cs = shared ? rsize : csize;
    if(!tl_cluster_valid(nrows, nbrows, rpiv, rstart, rsize) ||
            (!shared && !tl_cluster_valid(ncols, nbcols, cpiv, cstart, csize)))
    {
        info = STARSH_FILE_WRONG_INPUT;
        goto fail;
    }
    /* Block coordinates in range, ranks within the block, and the bytes
     * of the factors that follow. */
    uint64_t nu = 0, nv = 0, nd = 0;
    for(int64_t b = 0; b < nfar; b++)
    {
        const int64_t i = far[2*b], j = far[2*b+1];
        if(i < 0 || i >= nbrows || j < 0 || j >= nbcols || rank64[b] < 0 ||
                rank64[b] > rsize[i] || rank64[b] > cs[j])
        {
            info = STARSH_FILE_WRONG_INPUT;
            goto fail;
        }
        nu += (uint64_t)rsize[i]*(uint64_t)rank64[b];
        nv += (uint64_t)cs[j]*(uint64_t)rank64[b];
    }
    for(int64_t b = 0; b < nnear; b++)
    {
        const int64_t i = near[2*b], j = near[2*b+1];
        if(i < 0 || i >= nbrows || j < 0 || j >= nbcols)
        {
            info = STARSH_FILE_WRONG_INPUT;
            goto fail;
        }
        if(!onfly)
            nd += (uint64_t)rsize[i]*(uint64_t)cs[j];
    }
    if(nu+nv+nd+1 > tl_remaining(s)/8)
    {
        info = STARSH_FILE_WRONG_INPUT;
        goto fail;
    }
    aU = malloc(sizeof(double)*(nu > 0 ? nu : 1));
    aV = malloc(sizeof(double)*(nv > 0 ? nv : 1));
    aD = onfly ? NULL : malloc(sizeof(double)*(nd > 0 ? nd : 1));
    rank = malloc(sizeof(int)*(nfar > 0 ? nfar : 1));
    U = calloc(nfar > 0 ? nfar : 1, sizeof(*U));
    V = calloc(nfar > 0 ? nfar : 1, sizeof(*V));
    D = onfly ? NULL : calloc(nnear > 0 ? nnear : 1, sizeof(*D));
    if(aU == NULL || aV == NULL || rank == NULL || U == NULL || V == NULL ||
            (!onfly && (aD == NULL || D == NULL)))
    {
        info = STARSH_MALLOC_ERROR;
        goto fail;
    }
    size_t ou = 0, ov = 0, od = 0;
    for(int64_t b = 0; b < nfar && !info; b++)
    {
        const int r = (int)rank64[b];
        int su[2] = {(int)rsize[far[2*b]], r};
        int sv[2] = {(int)cs[far[2*b+1]], r};
        rank[b] = r;
        info = array_from_buffer(U+b, 2, su, 'd', 'F', aU+ou);
        if(!info)
            info = array_from_buffer(V+b, 2, sv, 'd', 'F', aV+ov);
        if(!info)
            info = tl_get(s, aU+ou, sizeof(double)*(size_t)su[0]*r);
        if(!info)
            info = tl_get(s, aV+ov, sizeof(double)*(size_t)sv[0]*r);
        ou += (size_t)su[0]*r;
        ov += (size_t)sv[0]*r;
    }
    for(int64_t b = 0; b < nnear && !onfly && !info; b++)
    {
        int sd[2] = {(int)rsize[near[2*b]], (int)cs[near[2*b+1]]};
        info = array_from_buffer(D+b, 2, sd, 'd', 'F', aD+od);
        if(!info)
            info = tl_get(s, aD+od, sizeof(double)*(size_t)sd[0]*sd[1]);
        od += (size_t)sd[0]*sd[1];
    }
    if(info)
        goto fail;
    const uint64_t want = tl_hash_final(&s->hash);
    uint64_t got;
    if(tl_get(s, &got, sizeof(got)) || got != want)
    {
        info = STARSH_FILE_WRONG_INPUT;
        goto fail;
    }
    /* STARSH_int is 64-bit, so the index arrays are taken over as read. */
    info = starsh_cluster_new(&R, P->row_data, nrows, (STARSH_int *)rpiv,
            nbrows, 0, NULL, (STARSH_int *)rstart, (STARSH_int *)rsize, NULL,
            NULL, NULL, STARSH_PLAIN);
    if(info)
        goto fail;
    rpiv = rstart = rsize = NULL;
    if(shared)
        C = R;
    else
    {
        info = starsh_cluster_new(&C, P->col_data, ncols, (STARSH_int *)cpiv,
                nbcols, 0, NULL, (STARSH_int *)cstart, (STARSH_int *)csize,
                NULL, NULL, NULL, STARSH_PLAIN);
        if(info)
            goto fail;
        cpiv = cstart = csize = NULL;
    }
    info = starsh_blrf_new_from_coo(&F, P, symm ? 'S' : 'N', R, C, nfar,
            (STARSH_int *)far, nnear, (STARSH_int *)near,
            (enum STARSH_BLRF_TYPE)h[6]);
    if(info)
        goto fail;
    if(nfar == 0)
        free(far);
    if(nnear == 0)
        free(near);
    far = near = NULL;
    info = starsh_blrm_new(matrix, F, nfar > 0 ? rank : NULL,
            nfar > 0 ? U : NULL, nfar > 0 ? V : NULL, onfly,
            onfly || nnear == 0 ? NULL : D, aU, aV, aD, '1');
    if(info)
        goto fail;
    if(nfar == 0)
    {
        free(rank);
        free(U);
        free(V);
        free(aU);
        free(aV);
        (*matrix)->alloc_U = (*matrix)->alloc_V = NULL;
    }
    if(!onfly && nnear == 0)
    {
        free(D);
        free(aD);
        (*matrix)->alloc_D = NULL;
    }
    free(rank64);
    return STARSH_SUCCESS;
fail:
    if(F != NULL)
    {
        /* the block lists still belong to this function */
        if(F->nblocks_far > 0)
            F->block_far = NULL;
        if(F->nblocks_near > 0)
            F->block_near = NULL;
        starsh_blrf_free(F);
    }
    if(C != NULL && C != R)
        starsh_cluster_free(C);
    starsh_cluster_free(R);
    if(U != NULL)
        for(int64_t b = 0; b < nfar; b++)
            if(U[b] != NULL)
            {
                U[b]->data = NULL;
                array_free(U[b]);
            }
    if(V != NULL)
        for(int64_t b = 0; b < nfar; b++)
            if(V[b] != NULL)
            {
                V[b]->data = NULL;
                array_free(V[b]);
            }
    if(D != NULL)
        for(int64_t b = 0; b < nnear; b++)
            if(D[b] != NULL)
            {
                D[b]->data = NULL;
                array_free(D[b]);
            }
    free(U);
    free(V);
    free(D);
    free(aU);
    free(aV);
    free(aD);
    free(rank);
    free(rank64);
    free(far);
    free(near);
    free(rpiv);
    free(rstart);
    free(rsize);
    free(cpiv);
    free(cstart);
    free(csize);
    return info;
}

int starsh_b200_blrm_read_from_file_pointer(STARSH_blrm **matrix,
        STARSH_problem *problem, FILE *fp)
{
    if(fp == NULL)
        return STARSH_WRONG_PARAMETER;
    tl_source s = {0};
    s.fp = fp;
    return tl_read(matrix, problem, &s);
}

int starsh_b200_blrm_read_from_file(STARSH_blrm **matrix,
        STARSH_problem *problem, const char *fname)
{
    if(matrix == NULL || problem == NULL || fname == NULL)
        return STARSH_WRONG_PARAMETER;
    FILE *fp = fopen(fname, "rb");
    if(fp == NULL)
        return STARSH_FILE_NOT_EXIST;
    int info = starsh_b200_blrm_read_from_file_pointer(matrix, problem, fp);
    fclose(fp);
    return info;
}

int starsh_b200_blrm_deserialize(STARSH_blrm **matrix,
        STARSH_problem *problem, const void *buffer, size_t nbytes)
{
    if(buffer == NULL)
        return STARSH_WRONG_PARAMETER;
    tl_source s = {0};
    s.buf = buffer;
    s.size = nbytes;
    return tl_read(matrix, problem, &s);
}

void starsh_b200_blrm_free_read(STARSH_blrm *matrix)
{
    if(matrix == NULL)
        return;
    STARSH_blrf *F = matrix->format;
    STARSH_cluster *R = F->row_cluster, *C = F->col_cluster;
    starsh_blrm_free(matrix);
    starsh_blrf_free(F);
    if(C != R)
        starsh_cluster_free(C);
    starsh_cluster_free(R);
}
