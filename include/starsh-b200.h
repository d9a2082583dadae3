/* B200 backend of the STARS-H TLR approximation path: entry points added by
 * libstarsh_b200.so beside the STARS-H API in starsh.h.
 *
 * The first group has exactly the signatures of the reference's function
 * pointer types, so a STARS-H build registers them in its dispatch table
 * (src/control/init.c dlr[][], include/control/init.h:111-190) under
 * STARSH_BACKEND_B200; the B200 library's own starsh_init() does so
 * already.  They accept STARSH_blrf/STARSH_problem structures built either
 * by this library or by the reference library, because the layouts are the
 * same.  Kernel functions are recognised by symbol name (dladdr), so the
 * reference's own kernel pointers select the matching device generator;
 * an unknown kernel pointer is an error (STARSH_WRONG_PARAMETER), there is
 * no CPU fallback.
 */
#ifndef STARSH_B200_H
#define STARSH_B200_H

#include <stdio.h>
#include "starsh.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------- drop-in entry points */

/* Randomized-SVD TLR approximation, every step FP64 on the GPU.
 * Signature of STARSH_blrm_approximate; replaces starsh_blrm__drsdd_omp
 * (reference src/backends/openmp/blrm/drsdd.c:16-307) and its dense engine
 * starsh_dense_dlrrsdd (src/backends/sequential/dense/drsdd.c:16-93).
 * The returned matrix has host factors (alloc_type '1', compact: far_U[i]
 * is nrows x rank) and keeps a device copy for starsh_blrm__dmml_b200. */
int starsh_blrm__drsdd_b200(STARSH_blrm **matrix, STARSH_blrf *format,
        int maxrank, double tol, int onfly);

/* Same contract with an adaptive sketch width: sketch columns are drawn in
 * blocks (64, then 32), each block is projected off the basis built so far
 * and only directions above (tol/10)^2 of the block's energy are kept; a
 * tile stops once a block leaves 10 columns below that threshold (a
 * posterior residual estimate) or its k = min(maxrank + oversample, m, n)
 * columns are used.  The sketch products run on the tcgen05 tensor cores
 * as exact integer products of five-byte slices of D with an int8 sketch
 * matrix (FP64-accurate to 2^-40 of each row's largest entry).
 * Projection, small SVD and the rank decision are as in
 * starsh_blrm__drsdd_b200, all in FP64.  Selected by STARSH_LRENGINE=
 * RSVD_MP on the B200 backend. */
int starsh_blrm__drsdd_b200_mp(STARSH_blrm **matrix, STARSH_blrf *format,
        int maxrank, double tol, int onfly);

/* B = alpha*M*A + beta*B with host A/B (N x nrhs, cluster order).
 * Signature and semantics of starsh_blrm__dmml (reference include/
 * starsh.h:602-603, src/backends/sequential/blrm/dmml.c:16-145); M may come
 * from the B200 engine (device factors are reused) or from any other
 * engine (factors are uploaded).  Returns STARSH_SUCCESS or an error. */
int starsh_blrm__dmml_b200(STARSH_blrm *matrix, int nrhs, double alpha,
        double *A, int lda, double beta, double *B, int ldb);

/* Relative Frobenius error of M, every block regenerated in FP64 on the GPU
 * (reference src/backends/sequential/blrm/dfe.c:16-134).  -1 on error. */
double starsh_blrm__dfe_b200(STARSH_blrm *matrix);

/* The two sums behind dfe: *diff2 = sum over far blocks of
 * ||D_b - U_b V_b^T||_F^2 and *norm2 = sum over all blocks of ||D_b||_F^2
 * (sqrt(2) weights of symmetric formats applied), so that a matrix split
 * over processes has dfe = sqrt(sum diff2 / sum norm2) after one sum
 * all-reduce of two doubles -- what the reference's MPI backend reduces
 * (src/backends/mpi/blrm/dfe.c:140-149). */
int starsh_b200_blrm_dfe_sums(STARSH_blrm *matrix, double *diff2,
        double *norm2);

/* ---------------------------------------------- device-resident results */

/* Engine selectors for starsh_b200_approximate(). */
enum STARSH_B200_ENGINE
{
    STARSH_B200_FP64 = 0,   /* starsh_blrm__drsdd_b200 */
    STARSH_B200_MIXED = 1,  /* starsh_blrm__drsdd_b200_mp */
};

/* Flags for starsh_b200_approximate(). */
enum STARSH_B200_FLAGS
{
    /* Copy factors and dense blocks to host memory before returning
     * (the drop-in entry points always set it).  Each batch's factors are
     * copied while later batches compute, into page-locked host blocks
     * that the matrix owns; starsh_blrm_free returns them to the
     * library's pool (STARSH_B200_PINNED_CACHE_MB of idle blocks kept). */
    STARSH_B200_HOST_MIRROR = 1,
};

/* Approximation with an explicit engine and flags.  Without
 * STARSH_B200_HOST_MIRROR the returned matrix has ranks and shapes on the
 * host but far_U[i]->data, far_V[i]->data and near_D[i]->data are NULL
 * until starsh_b200_blrm_download() fills them; the factors stay on the
 * device for starsh_b200_blrm_dmml_device().  maxrank, tol, onfly and the
 * in-place update of *format on rank failure are as in
 * starsh_blrm__drsdd_b200. */
int starsh_b200_approximate(STARSH_blrm **matrix, STARSH_blrf *format,
        int maxrank, double tol, int onfly, int engine, int flags);

/* Approximates nprob independent problems in shared batches: the tiles of
 * all problems (any kernels, tile sizes, maxrank and tol) go through the
 * same launches, so many small problems fill the GPU like one large one.
 * matrices[p] receives the approximation of formats[p] under maxrank[p],
 * tol[p] and onfly[p] (onfly may be NULL: all 0); each result equals what
 * starsh_b200_approximate() returns for that problem alone.  The formats
 * must be distinct.  On error no matrix is returned. */
int starsh_b200_approximate_batch(int nprob, STARSH_blrm **matrices,
        STARSH_blrf **formats, const int *maxrank, const double *tol,
        const int *onfly, int engine, int flags);

/* Fills the host mirror of a device-resident matrix (no-op if present). */
int starsh_b200_blrm_download(STARSH_blrm *matrix);

/* Releases the device copy of M.  starsh_blrm_free() of this library does
 * it as well; call this one when M is freed by the reference library. */
void starsh_b200_blrm_release(STARSH_blrm *matrix);

/* Returns the page-locked host blocks of M's host mirror (when its factors
 * were downloaded batch by batch, STARSH_B200_HOST_MIRROR) to the
 * library's pool; M's far_U/far_V/near_D data must not be used after it.
 * starsh_blrm_free() of this library does it as well; call this one, with
 * starsh_b200_blrm_release(), when M is freed by the reference library.
 * No-op for other matrices. */
void starsh_b200_blrm_host_release(const STARSH_blrm *matrix);

/* dmml with device pointers dA (lda) and dB (ldb) on `stream`
 * (a cudaStream_t, NULL for the default stream).  Asynchronous. */
int starsh_b200_blrm_dmml_device(STARSH_blrm *matrix, int nrhs,
        double alpha, const double *dA, int lda, double beta, double *dB,
        int ldb, void *stream);

/* ---------------------------------------------------- iterative solver */

/* Conjugate gradients on M with host B and X (N x nrhs, cluster order):
 * signature and iteration of starsh_itersolvers__dcg_omp (reference
 * include/starsh.h:671-672, src/itersolvers/cg.c:24-95), every product a
 * device dmml on the resident factors; `work` is not used.  Returns the
 * iteration at which the last column converged, or -1 if it did not
 * within N iterations (or on error: starsh_b200_last_error()). */
int starsh_itersolvers__dcg_b200(STARSH_blrm *matrix, int nrhs, double *B,
        int ldb, double *X, int ldx, double tol, double *work);

/* The same on device B and X (X holds the initial guess and receives the
 * solution) on `stream` (NULL: the library stream), at most maxiter
 * iterations (<= 0: N); *iterations as above.  Returns STARSH_SUCCESS or
 * an error. */
int starsh_b200_dcg_device(STARSH_blrm *matrix, int nrhs, const double *dB,
        int ldb, double *dX, int ldx, double tol, int maxiter, void *stream,
        int *iterations);

/* ------------------------------------------- serialised matrices */

/* A STARSH_blrm as a byte stream (the reference has no serialised form):
 * clusterings, block lists, ranks, factors and dense near blocks, ending
 * in a 64-bit checksum.  Writing brings device-resident factors to the
 * host first.  Reading binds the stream to `problem` (same shape and
 * symmetry, else STARSH_WRONG_PARAMETER) and builds new clusterings, a new
 * format and a host-resident matrix, all freed by
 * starsh_b200_blrm_free_read(); a malformed, truncated or corrupted stream
 * gives STARSH_FILE_WRONG_INPUT, a file that cannot be opened
 * STARSH_FILE_NOT_EXIST.  starsh_b200_blrm_serialize() with buffer NULL
 * only stores the stream's size in *nbytes; with a buffer smaller than the
 * stream it returns STARSH_WRONG_PARAMETER (*nbytes = the size needed). */
int starsh_b200_blrm_write_to_file(STARSH_blrm *matrix, const char *fname);
int starsh_b200_blrm_write_to_file_pointer(STARSH_blrm *matrix, FILE *fp);
int starsh_b200_blrm_serialize(STARSH_blrm *matrix, void *buffer,
        size_t capacity, size_t *nbytes);
int starsh_b200_blrm_read_from_file(STARSH_blrm **matrix,
        STARSH_problem *problem, const char *fname);
int starsh_b200_blrm_read_from_file_pointer(STARSH_blrm **matrix,
        STARSH_problem *problem, FILE *fp);
int starsh_b200_blrm_deserialize(STARSH_blrm **matrix,
        STARSH_problem *problem, const void *buffer, size_t nbytes);
void starsh_b200_blrm_free_read(STARSH_blrm *matrix);

/* ------------------------------------------------- kernel registration */

/* Device kernel families. */
enum STARSH_B200_FAMILY
{
    STARSH_B200_FAMILY_EXP = 1,
    STARSH_B200_FAMILY_SQREXP = 2,
    STARSH_B200_FAMILY_MATERN = 3,
    STARSH_B200_FAMILY_MATERN2 = 4,
    STARSH_B200_FAMILY_COULOMB = 5,
    STARSH_B200_FAMILY_SIN = 6,
    STARSH_B200_FAMILY_COS = 7,
    STARSH_B200_FAMILY_RBF = 8,
};

/* Associates a host kernel pointer with a device family.  For
 * STARSH_B200_FAMILY_COULOMB, `param` is the value of the r = 0 entries
 * (the reference emits 0; regularised problems use 1).  `param` is ignored
 * for the other families, whose parameters come from row_data.  Returns
 * STARSH_SUCCESS, or STARSH_WRONG_PARAMETER when the table is full. */
int starsh_b200_kernel_register(STARSH_kernel *kernel, int family,
        double param);

/* Family recognised for `kernel` (0 if none).  For a recognised kernel
 * *ndim_hint is the dimension fixed by its name (0 for "_nd"). */
int starsh_b200_kernel_family(STARSH_kernel *kernel, int *ndim_hint);

/* ------------------------------------------------------------ autotuner */

/* Tile-size autotuner.  No counterpart in the reference (which takes the
 * block size from the caller, src/control/cluster.c:106-146).  For each
 * candidate block size cand_nb[c] (with maxrank cand_maxrank[c]) it times
 * starsh_b200_approximate() with `engine` on a fixed-seed random sample of
 * the problem's TLR blocks -- 24 and then 48 of them, the difference being
 * the marginal cost free of per-call overheads -- and returns the fastest
 * in *best_nb (costs, if not NULL, receives ncand costs in nanoseconds per
 * matrix entry; INFINITY for candidates above N).  Results are cached per
 * problem class (kernel family and its dimension, N in half-octaves, tol in
 * decades, engine, candidate list): later problems of a class are not
 * measured again.  1 <= ncand <= 8.  Runs device work; thread-safe. */
int starsh_b200_autotune_tile(STARSH_problem *problem, int ncand,
        const int *cand_nb, const int *cand_maxrank, double tol, int engine,
        int *best_nb, double *costs);

/* Forgets the autotuner's cached choices. */
void starsh_b200_autotune_clear(void);

/* ------------------------------------------------ no-allocation variant */

/* Randomized-SVD compression of one dense tile already on the device,
 * without allocating any device memory.  No counterpart in the reference:
 * it is for callers that cannot call cudaMalloc (a host framework whose
 * caching allocator owns all device memory, a plugin handed device buffers
 * but no right to allocate, or threads that must not wait for the
 * allocator's implicit synchronisation).  Same algorithm
 * and Gaussian sketch as starsh_blrm__drsdd_b200 applied to that tile, with
 * the reference's rank rule (the tail of the projected tile's spectrum: the
 * batched engine also counts the energy its sketch missed, from the exact
 * block norms of its generator); its scratch is a fixed __device__ array of about 2.1 MB that every
 * GPU loading the library keeps until the process exits.
 *   dD      nrows x ncols tile, column-major, leading dimension ldd;
 *   dU      receives nrows x rank, leading dimension nrows;
 *   dV      receives ncols x rank, leading dimension ncols (U V^T ~ D);
 *           both need room for maxrank columns;
 *   d_rank  device int: the rank, or -1 when it exceeds maxrank (dU and
 *           dV are then left unwritten: store the tile dense);
 *   stream  cudaStream_t (NULL: default stream); the call is asynchronous.
 * Limits: nrows, ncols <= 256 and min(maxrank + oversample, nrows, ncols)
 * <= 96; beyond them STARSH_WRONG_PARAMETER.  The first call on a device
 * looks up the scratch address (cudaGetSymbolAddress) and should come
 * before any stream capture.  All calls share the scratch: calls that
 * overlap on the GPU race. */
int starsh_b200_dense_rsvd_noalloc(const double *dD, int nrows, int ncols,
        int ldd, int maxrank, int oversample, double tol, double *dU,
        double *dV, int *d_rank, void *stream);

/* ------------------------------------------------------------ serving */

/* A serving loop: approximation requests are admitted by an HBM budget and
 * run in shared batches, then each request's TLR-by-dense product runs on
 * the resident factors.  Continuous batching: worker threads (3 by
 * default, STARSH_B200_SERVER_WORKERS up to 8), each with its own CUDA
 * streams and buffers, take the next group whenever they are free, so
 * requests that arrive while groups are on the GPU are admitted by a free
 * worker as memory allows and the groups' kernels overlap on the device.
 * A group takes requests in FIFO order up to 5e8 matrix entries of work
 * (STARSH_B200_SERVER_GROUP_ENTRIES; its first request always goes in).
 * All calls are thread-safe. */
typedef struct starsh_b200_server starsh_b200_server;

typedef struct starsh_b200_server_stats
{
    long long submitted, completed, failed;
    long long groups;             /* batched approximation calls           */
    long long entries;            /* sum of m*n over approximated blocks   */
    double busy_ms;               /* worker time inside groups (summed
                                     over the workers)                     */
    double resident_bytes;        /* results kept and not yet released     */
    double peak_resident_bytes;
    double queue_ms;              /* sum over requests: submit to the start
                                     of their group                        */
    double approx_ms;             /* sum over groups: batched approximation */
    double products_ms;           /* sum over groups: the requests' products */
} starsh_b200_server_stats;

/* hbm_budget_bytes bounds the device memory of admitted and kept results
 * (admission uses an upper bound: factors at maxrank, dense near blocks);
 * engine is STARSH_B200_FP64 or STARSH_B200_MIXED; max_group caps the
 * requests of one group (<= 0: no cap). */
int starsh_b200_server_new(starsh_b200_server **server,
        double hbm_budget_bytes, int engine, int max_group);

/* Queues the approximation of `format` (updated in place on demotion, as
 * by starsh_blrm_approximate) followed, if nrhs > 0, by B = M A with host
 * A (N x nrhs, lda) and B (N x nrhs, ldb).  format, A and B must stay valid
 * until the request completes.  With keep = 0 the matrix is freed after
 * the product; with keep = 1 it stays resident (counted in the budget)
 * until starsh_b200_server_release().  *ticket identifies the request. */
int starsh_b200_server_submit(starsh_b200_server *server,
        STARSH_blrf *format, int maxrank, double tol, int nrhs,
        const double *A, int lda, double *B, int ldb, int keep,
        long long *ticket);

/* Blocks until the request completes; returns its status
 * (STARSH_MALLOC_ERROR if it can never fit the budget), the kept matrix
 * (device-resident, NULL if keep = 0) and the latency from submit to
 * completion in milliseconds.  Each ticket is waited for once. */
int starsh_b200_server_wait(starsh_b200_server *server, long long ticket,
        STARSH_blrm **matrix, double *latency_ms);

/* Frees a kept matrix and returns its memory to the budget. */
int starsh_b200_server_release(starsh_b200_server *server,
        STARSH_blrm *matrix);

/* paused = 1 holds admission (queued requests wait, running groups
 * finish); paused = 0 resumes. */
int starsh_b200_server_pause(starsh_b200_server *server, int paused);

int starsh_b200_server_get_stats(starsh_b200_server *server,
        starsh_b200_server_stats *stats);

/* Finishes the queued requests and stops the worker. */
int starsh_b200_server_free(starsh_b200_server *server);

/* ------------------------------------------------------------ device */

/* Selects the CUDA device the library uses; must be called before any
 * other B200 call of the process (default: device 0, or the device current
 * at the first call).  Returns STARSH_SUCCESS or STARSH_WRONG_PARAMETER. */
int starsh_b200_set_device(int device);

/* The cudaStream_t every library kernel is launched on (for timing with
 * events and for ordering user work). */
void *starsh_b200_stream(void);

/* ------------------------------------------------------- diagnostics */

/* Timings and counters of the last approximation on this host thread. */
typedef struct starsh_b200_stats
{
    double total_ms;          /* whole call, host clock                 */
    double device_ms;         /* device time of the compression phases  */
    double sketch_ms;         /* device time in the sketch kernels      */
    double project_ms;        /* device time in the projection kernels  */
    double sketch_flops;      /* algorithmic flops of the sketch        */
    double project_flops;     /* flops the projection GEMMs performed   */
    long long tiles;          /* far-field tiles compressed             */
    long long false_far;      /* tiles that exceeded maxrank            */
    long long entries;        /* sum of m*n over all admissible blocks  */
    long long kernel_launches;/* device kernels launched by the call    */
    long long rank_sum;       /* sum of accepted ranks                  */
    int max_rank;             /* largest accepted rank                  */
    long long h2d_bytes;      /* host to device bytes                   */
    long long d2h_bytes;      /* device to host bytes                   */
    long long batches;        /* tile batches (launches of each GEMM step) */
    long long sketch_launches;/* sketch GEMM launches (timed by sketch_ms) */
    double gen_ms;            /* device time generating far tiles       */
    double basis_ms;          /* sketch and orthogonalisation, in all   */
    double svd_ms;            /* Gram of B, its factor, Jacobi, rank cut */
    double output_ms;         /* U = Q W and V written to the arena     */
    double sketch_bytes;      /* algorithmic HBM bytes of the sketch:
                                 D read once per round, Y written      */
    int sketch_int8;          /* 1: sketch on the tcgen05 int8 path     */
    double fused_ms;          /* device time of the fused generation and
                                 first-round sketch (incl. re-sketches)  */
    long long fused_launches; /* batches whose round 0 ran fused        */
    double fused_bytes;       /* algorithmic HBM bytes of the fused
                                 kernel: D and the round-0 Y written     */
    long long resketch_tiles; /* tiles re-sketched from the stored D    */
    double mirror_wait_ms;    /* host mirror: host time waiting, after the
                                 last batch, for the batch downloads     */
    double finish_ms;         /* host time from the last batch to return
                                 (demotion, near blocks, host structure,
                                 mirror mapping and near-block copy)    */
} starsh_b200_stats;
int starsh_b200_get_stats(starsh_b200_stats *stats);

/* Last CUDA or watchdog error as text ("" if none). */
const char *starsh_b200_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
