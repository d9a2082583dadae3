// Host driver of the B200 TLR approximation: starsh_b200_approximate() and
// the drop-in entry points, the device-resident matrix records, host
// mirrors, and the host-callable block generator.
//
// Control flow follows starsh_blrm__drsdd_omp (reference
// src/backends/openmp/blrm/drsdd.c:16-307): compress every far-field block;
// blocks whose rank exceeds maxrank become near-field blocks and the format
// is rebuilt and swapped into *format in place (:146-212); near-field
// blocks are generated densely unless onfly (:214-256); ranks and factors
// are compacted (:259-282).  The per-block loop runs as batches of tiles
// through the device pipeline of rsvd_kernels.cu.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <atomic>
#include <mutex>
#include <thread>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <unordered_map>
#include <vector>

#include "device_ctx.cuh"
#include "engine.cuh"
#include "records.cuh"
#include "b200_host.h"
#include "starsh-b200.h"

namespace b200 {

// --------------------------------------------------------------- context

bool DeviceBuffer::reserve(size_t need, cudaStream_t s)
{
    if (need <= bytes) return true;
    if (ptr) cudaFreeAsync(ptr, s);
    ptr = nullptr;
    bytes = 0;
    if (cudaMallocAsync(&ptr, need, s) != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        return false;
    }
    bytes = need;
    stream = s;
    return true;
}

void DeviceBuffer::release()
{
    if (ptr) cudaFreeAsync(ptr, stream);
    ptr = nullptr;
    bytes = 0;
}

static Context g_ctx;
static std::once_flag g_ctx_once;
static bool g_ctx_ok = false;
static int g_requested_device = -1;
static thread_local std::string t_error;
static thread_local starsh_b200_stats t_stats;
static std::atomic<long long> g_launches{0};

// A context a thread has made its own (a serving worker's), or null.
static thread_local Context *t_ctx = nullptr;

Context *context()
{
    if (t_ctx != nullptr) {
        int cur = -1;
        if (cudaGetDevice(&cur) != cudaSuccess || cur != t_ctx->device)
            cudaSetDevice(t_ctx->device);
        return t_ctx;
    }
    std::call_once(g_ctx_once, [] {
        int dev = 0;
        if (g_requested_device >= 0 &&
            cudaSetDevice(g_requested_device) != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaSetDevice failed");
            return;
        }
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            set_error("no CUDA device available");
            return;
        }
        g_ctx.device = dev;
        if (cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking)
                != cudaSuccess ||
            cudaStreamCreateWithFlags(&g_ctx.side, cudaStreamNonBlocking)
                != cudaSuccess ||
            cudaStreamCreateWithFlags(&g_ctx.copy, cudaStreamNonBlocking)
                != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaStreamCreate failed");
            return;
        }
        // keep freed pool memory cached in the process; a block freed on
        // one stream is reused on another only once its free has
        // completed, never by making the allocating stream wait for the
        // freeing one (which would chain the serving workers' streams)
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold,
                                    &keep);
            int no = 0;
            cudaMemPoolSetAttribute(pool,
                                    cudaMemPoolReuseAllowInternalDependencies,
                                    &no);
        }
        cudaGetLastError();
        g_ctx_ok = true;
    });
    if (!g_ctx_ok) return nullptr;
    // every host thread that calls in works on the library's device
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != g_ctx.device)
        cudaSetDevice(g_ctx.device);
    return &g_ctx;
}

// Private contexts of finished workers (streams and grown buffers), kept
// for the next ones: a new server's workers start warm.
static std::mutex g_idle_mu;
static std::vector<Context *> g_idle_ctx;
constexpr size_t kIdleContexts = 8;

Context *context_new_private()
{
    {
        std::lock_guard<std::mutex> g(g_idle_mu);
        if (!g_idle_ctx.empty()) {
            Context *c = g_idle_ctx.back();
            g_idle_ctx.pop_back();
            cudaSetDevice(c->device);
            return c;
        }
    }
    Context *base = nullptr;
    {
        Context *saved = t_ctx;
        t_ctx = nullptr;
        base = context();        // the library's device, initialised once
        t_ctx = saved;
    }
    if (base == nullptr) return nullptr;
    Context *c = new Context();
    c->device = base->device;
    // a serving worker's batches stay at most this large (several workers
    // share the device; batches of this size already fill it), so its
    // workspace is reserved once, at the start
    size_t cap_mb = 8192;
    if (const char *e = getenv("STARSH_B200_SERVER_WORKSPACE_MB"))
        cap_mb = (size_t)std::max(64LL, atoll(e));
    c->workspace_cap = cap_mb << 20;
    cudaSetDevice(c->device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return nullptr;
    }
    return c;
}

void context_free_private(Context *c)
{
    if (c == nullptr) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    cudaStreamSynchronize(c->side);
    cudaStreamSynchronize(c->copy);
    {
        std::lock_guard<std::mutex> g(g_idle_mu);
        if (g_idle_ctx.size() < kIdleContexts) {
            g_idle_ctx.push_back(c);
            return;
        }
    }
    c->workspace.release();
    c->tiles.release();
    c->descs.release();
    c->omega.release();
    c->flag.release();
    c->act.release();
    c->kernels.release();
    c->omega8.release();
    if (c->mapped) cudaFreeHost(c->mapped);
    for (int i = 0; i < 2; ++i) {
        if (c->stage[i]) cudaFreeHost(c->stage[i]);
        if (c->stage_ev[i]) cudaEventDestroy(c->stage_ev[i]);
        if (c->tiles_pin[i]) host_pinned_free(c->tiles_pin[i]);
    }
    cudaStreamDestroy(c->stream);
    cudaStreamDestroy(c->side);
    cudaStreamDestroy(c->copy);
    delete c;
}

void set_thread_context(Context *c) { t_ctx = c; }

void *pool_alloc(size_t bytes, cudaStream_t s)
{
    void *p = nullptr;
    if (cudaMallocAsync(&p, bytes ? bytes : 8, s) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void pool_free(void *p)
{
    // ordered on the calling thread's stream (its own work on p, if any,
    // precedes the free; matrices are freed after a device synchronisation)
    if (p) cudaFreeAsync(p, t_ctx != nullptr ? t_ctx->stream : g_ctx.stream);
}

// ------------------------------------------------- pinned host memory

static std::mutex g_pin_mu;
static std::multimap<size_t, void *> g_pin_idle;        // size -> block
static std::unordered_map<void *, size_t> g_pin_owned;  // every block
static size_t g_pin_idle_bytes = 0;

static size_t pinned_cache_cap()
{
    static const size_t cap = [] {
        size_t mb = 32768;   // idle pinned memory kept for reuse
        if (const char *e = getenv("STARSH_B200_PINNED_CACHE_MB"))
            mb = (size_t)std::max(0, atoi(e));
        return mb << 20;
    }();
    return cap;
}

void *host_pinned_alloc(size_t bytes)
{
    bytes = std::max<size_t>(bytes, 1);
    {
        // an idle block at most a quarter larger than asked
        std::lock_guard<std::mutex> g(g_pin_mu);
        auto it = g_pin_idle.lower_bound(bytes);
        if (it != g_pin_idle.end() && it->first <= bytes + bytes / 4) {
            void *p = it->second;
            g_pin_idle_bytes -= it->first;
            g_pin_idle.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> g(g_pin_mu);
    g_pin_owned[p] = bytes;
    return p;
}

bool host_pinned_free(void *p)
{
    std::vector<void *> drop;
    {
        std::lock_guard<std::mutex> g(g_pin_mu);
        auto it = g_pin_owned.find(p);
        if (it == g_pin_owned.end()) return false;
        g_pin_idle.emplace(it->second, p);
        g_pin_idle_bytes += it->second;
        // above the cap: the largest idle blocks go back to the system
        while (g_pin_idle_bytes > pinned_cache_cap() && !g_pin_idle.empty()) {
            auto last = std::prev(g_pin_idle.end());
            g_pin_idle_bytes -= last->first;
            g_pin_owned.erase(last->second);
            drop.push_back(last->second);
            g_pin_idle.erase(last);
        }
    }
    for (void *q : drop) cudaFreeHost(q);
    return true;
}

void set_error(const std::string &msg)
{
    t_error = msg;
    fprintf(stderr, "STARSH B200 ERROR: %s\n", msg.c_str());
}

int cuda_fail(cudaError_t err, const char *what)
{
    set_error(std::string(what) + ": " + cudaGetErrorString(err));
    return err == cudaErrorMemoryAllocation ? STARSH_MALLOC_ERROR
                                            : STARSH_UNKNOWN_ERROR;
}

starsh_b200_stats &thread_stats() { return t_stats; }
void count_launch(long long n) { g_launches += n; }
long long launch_count() { return g_launches.load(); }

// --------------------------------------------------------- device points

void fill_kernel(DevKernel &K, const b200_kspec &sp)
{
    K.family = sp.family;
    K.ndim = sp.ndim;
    K.aos = sp.aos;
    K.rbf_kind = sp.rbf_kind;
    K.isreg = sp.isreg;
    K.zero_mode = sp.zero_mode;
    K.sigma = sp.sigma;
    K.beta = sp.beta;
    K.nu = sp.nu;
    K.noise = sp.noise;
    K.matern_coef = sp.matern_coef;
    K.matern_scale = sp.matern_scale;
    K.wave_k = sp.wave_k;
    K.diag = sp.diag;
    K.rad = sp.rad;
    K.reg = sp.reg;
    K.inv_neg_beta = sp.beta != 0.0 ? -1.0 / sp.beta : 0.0;
    K.inv_neg_2beta2 = sp.beta != 0.0 ? 1.0 / ((-2.0 * sp.beta) * sp.beta) : 0.0;
    K.matern_half = 0;
    if (sp.family == FAM_MATERN || sp.family == FAM_MATERN2) {
        if (sp.family == FAM_MATERN2)
            K.matern_scale = sp.beta != 0.0 ? 1.0 / sp.beta : 0.0;
        if (sp.nu == 0.5) K.matern_half = 1;
        else if (sp.nu == 1.5) K.matern_half = 2;
        else if (sp.nu == 2.5) K.matern_half = 3;
    }
}

// Polynomial pieces of G(x) = x^nu e^x K_nu(x) (one CTA per piece q:
// octave E = q / kMaternTabSub + kMaternTabEmin, eighth j = q %
// kMaternTabSub, x = 2^E (1 + (2 j + 1 + u) / 16), u in [-1, 1)).  G at
// the kMaternTabDeg + 1 Chebyshev points of the first kind u_i = cos(pi
// (i + 1/2) / (deg + 1)) gives the interpolant's Chebyshev coefficients
// c_k = 2 / (deg + 1) sum_i G(x_i) cos(pi k (i + 1/2) / (deg + 1)), c_0
// halved (the discrete cosine transform of Chebyshev interpolation); one
// thread turns them into monomial coefficients in u through the
// recurrence T_{k+1} = 2 u T_k - T_{k-1} (integer coefficients, exact in
// double; the terms decay like 34^-k, so the sum loses no digits).  Node
// values come from the trapezoidal integral for x >= 2 and from Temme's
// series below.
__global__ void k_matern_table(double nu, double *tab)
{
    constexpr int N1 = kMaternTabDeg + 1;
    __shared__ double g[N1], cc[N1];
    const int q = blockIdx.x, i = threadIdx.x;
    const int E = q / kMaternTabSub + kMaternTabEmin, jp = q % kMaternTabSub;
    if (i < N1) {
        const double u = cospi((i + 0.5) / N1);
        const double x = ldexp(1.0 + (2 * jp + 1 + u) / (2.0 * kMaternTabSub), E);
        g[i] = x >= 2.0
            ? exp(nu * log(x)) * bessel_k_large_scaled(nu, x, 2.0)
            : exp(nu * log(x) + x) * bessel_knu(nu, x);
    }
    __syncthreads();
    if (i < N1) {
        double c = 0.0;
        for (int k = 0; k < N1; ++k) c += g[k] * cospi(i * (k + 0.5) / N1);
        c *= 2.0 / N1;
        cc[i] = i == 0 ? 0.5 * c : c;
    }
    __syncthreads();
    if (i == 0) {
        double a[N1], t0[N1], t1[N1];
        #pragma unroll
        for (int k = 0; k < N1; ++k) { a[k] = 0.0; t0[k] = 0.0; t1[k] = 0.0; }
        t0[0] = 1.0;                 // T_0
        t1[1] = 1.0;                 // T_1
        a[0] = cc[0];
        a[1] = cc[1];
        #pragma unroll
        for (int k = 2; k < N1; ++k) {
            #pragma unroll
            for (int e = N1 - 1; e >= 0; --e) {
                const double t2 = (e > 0 ? 2.0 * t1[e - 1] : 0.0) - t0[e];
                t0[e] = t1[e];
                t1[e] = t2;
                a[e] += cc[k] * t2;
            }
        }
        #pragma unroll
        for (int k = 0; k < kMaternTabStride; ++k)
            tab[(size_t)q * kMaternTabStride + k] = k < N1 ? a[k] : 0.0;
    }
}

// Device tables a kernel family needs (the Matérn large-argument table),
// owned by dp.
static int prepare_kernel_tables(DevicePoints &dp, cudaStream_t s)
{
    DevKernel &K = dp.K;
    K.matern_tab = nullptr;
    if ((K.family == FAM_MATERN || K.family == FAM_MATERN2) &&
        K.matern_half == 0 && K.nu > 0.0) {
        const size_t n = (size_t)kMaternTabPieces * kMaternTabStride;
        double *tab = (double *)pool_alloc(n * sizeof(double), s);
        if (tab == nullptr)
            return cuda_fail(cudaErrorMemoryAllocation, "Matern table");
        dp.owned.push_back(tab);
        k_matern_table<<<kMaternTabPieces, 32, 0, s>>>(K.nu, tab);
        count_launch();
        B200_CUDA(cudaGetLastError(), "k_matern_table");
        K.matern_tab = tab;
    }
    return STARSH_SUCCESS;
}

// Uploads the point sets of a problem and the cluster pivots.
int upload_problem(DevicePoints &dp, STARSH_problem *P,
                          STARSH_cluster *R, STARSH_cluster *C,
                          cudaStream_t s)
{
    b200_kspec spec;
    const double *rp, *cp;
    STARSH_int rc, cc;
    int info = b200_resolve_kernel(P->kernel, P->row_data, &spec, &rp, &rc,
                                   &cp, &cc, P->col_data);
    if (info != STARSH_SUCCESS) return info;
    fill_kernel(dp.K, spec);
    if ((info = prepare_kernel_tables(dp, s))) return info;
    dp.h_row = rp;
    dp.h_col = cp;
    dp.h_row_count = rc;
    dp.h_col_count = cc;
    const void *d = nullptr;
    const size_t per = (size_t)spec.ndim * sizeof(double);
    if ((info = dp.upload(rp, rc * per, &d, s))) return info;
    dp.K.row_pt = (const double *)d;
    dp.K.row_count = rc;
    if (cp == rp && cc == rc) {
        dp.K.col_pt = dp.K.row_pt;
    } else {
        if ((info = dp.upload(cp, cc * per, &d, s))) return info;
        dp.K.col_pt = (const double *)d;
    }
    dp.K.col_count = cc;
    if ((info = dp.upload(R->pivot, R->ndata * sizeof(STARSH_int), &d, s)))
        return info;
    dp.K.row_piv = (const long long *)d;
    if (C == R) {
        dp.K.col_piv = dp.K.row_piv;
    } else {
        if ((info = dp.upload(C->pivot, C->ndata * sizeof(STARSH_int), &d, s)))
            return info;
        dp.K.col_piv = (const long long *)d;
    }
    return STARSH_SUCCESS;
}

// ---------------------------------------------------- dense block writer

__global__ void k_gen_blocks(DevKernel K, const BlockJob *__restrict__ jobs)
{
    const BlockJob jb = jobs[blockIdx.z];
    const int i = blockIdx.x * 64 + (threadIdx.x & 63);
    const int j0 = blockIdx.y * 64 + (threadIdx.x >> 6);
    if (i >= jb.m) return;
    for (int c = 0; c < 16; ++c) {
        const int j = j0 + 4 * c;
        if (j < jb.n)
            jb.out[(size_t)j * jb.m + i] = block_entry(K, jb.row0, jb.col0, i, j);
    }
}

int gen_blocks(const DevKernel &K, const std::vector<BlockJob> &jobs,
                      cudaStream_t s)
{
    if (jobs.empty()) return STARSH_SUCCESS;
    int mmax = 0, nmax = 0;
    for (const auto &j : jobs) {
        mmax = std::max(mmax, j.m);
        nmax = std::max(nmax, j.n);
    }
    BlockJob *dj = nullptr;
    B200_CUDA(cudaMallocAsync((void **)&dj, jobs.size() * sizeof(BlockJob), s),
              "cudaMallocAsync(jobs)");
    cudaMemcpyAsync(dj, jobs.data(), jobs.size() * sizeof(BlockJob),
                    cudaMemcpyHostToDevice, s);
    for (size_t b0 = 0; b0 < jobs.size(); b0 += 65535) {
        const unsigned nb = (unsigned)std::min<size_t>(65535, jobs.size() - b0);
        dim3 grid((mmax + 63) / 64, (nmax + 63) / 64, nb);
        k_gen_blocks<<<grid, 256, 0, s>>>(K, dj + b0);
        count_launch();
    }
    cudaFreeAsync(dj, s);
    B200_CUDA(cudaGetLastError(), "k_gen_blocks");
    return STARSH_SUCCESS;
}

// ------------------------------------------------------ device records

static std::mutex g_rec_lock;
static std::unordered_map<const STARSH_blrm *, Record *> g_records;

void add_record(const STARSH_blrm *M, Record *rec)
{
    std::lock_guard<std::mutex> g(g_rec_lock);
    g_records[M] = rec;
}

Record *find_record(const STARSH_blrm *M)
{
    std::lock_guard<std::mutex> g(g_rec_lock);
    auto it = g_records.find(M);
    return it == g_records.end() ? nullptr : it->second;
}

// -------------------------------------------------------------- engine

static const unsigned long long kOmegaSeed = 0x5354415253480001ull;

struct EngineParams {
    int oversample;
    int engine;
    int block;      // adaptive sketch: columns of the first round
    int block_next; // ... and of every later round
    int verify;     // unselected sample columns that finish a tile
    bool mirror;    // host mirrors wanted: download each batch when done
};

// One problem of a batched approximation call.
struct ProblemJob {
    STARSH_blrf *F;
    int maxrank;
    double tol;
    int onfly;
    Record *rec;              // owns the problem's points and factors
    std::vector<int> rank;    // per far block of F (filled by compress)
};

// Bounding boxes of the clusters of C over the given coordinates (SoA
// x[d * count + i], or AoS x[ndim * i + d]): lo/hi per cluster and
// dimension.
static void cluster_boxes(const double *pts, long long count, int ndim,
                          int aos, const STARSH_cluster *C,
                          std::vector<double> &lo, std::vector<double> &hi)
{
    const STARSH_int nc = C->nblocks;
    lo.assign((size_t)nc * ndim, 0.0);
    hi.assign((size_t)nc * ndim, 0.0);
    if (pts == nullptr) return;
    for (STARSH_int c = 0; c < nc; ++c)
        for (int d = 0; d < ndim; ++d) {
            double a = DBL_MAX, b = -DBL_MAX;
            for (STARSH_int q = C->start[c]; q < C->start[c] + C->size[c]; ++q) {
                const long long i = C->pivot[q];
                const double x = aos ? pts[(size_t)ndim * i + d]
                                     : pts[(size_t)d * count + i];
                a = std::min(a, x);
                b = std::max(b, x);
            }
            lo[(size_t)c * ndim + d] = a;
            hi[(size_t)c * ndim + d] = b;
        }
}

// The context's mapped host area: the round count at offset 0, a batch's
// tile records (at most kMaxBatchTiles) from offset 256.  Allocated once
// per context at its first approximation.
constexpr long long kMaxBatchTiles = 4096;
constexpr size_t kMappedRecords = 256;

static int mapped_area(Context &ctx)
{
    if (ctx.mapped != nullptr) return STARSH_SUCCESS;
    const size_t bytes = kMappedRecords + (size_t)kMaxBatchTiles * sizeof(TileWork);
    void *h = nullptr, *d = nullptr;
    B200_CUDA(cudaHostAlloc(&h, bytes, cudaHostAllocMapped), "cudaHostAlloc(mapped)");
    const cudaError_t e = cudaHostGetDevicePointer(&d, h, 0);
    if (e != cudaSuccess) {
        cudaFreeHost(h);
        return cuda_fail(e, "cudaHostGetDevicePointer");
    }
    ctx.mapped = h;
    ctx.mapped_dev = d;
    return STARSH_SUCCESS;
}

// Stores `words` 8-byte words of device memory into mapped host memory
// (visible to the host once the stream has passed the kernel).
__global__ void k_store_to_host(const unsigned long long *__restrict__ src,
                                unsigned long long *dst, size_t words)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words;
         i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

__global__ void k_count_to_host(const int *__restrict__ src, int *dst)
{
    *dst = *src;
}

// Runs the device pipeline over the far blocks of every problem of `jobs`
// in shared batches: tiles of different problems (kernels, sizes, tol,
// maxrank) share every launch.  Fills each job's ranks and the per-block
// device pointers of U and V in its record.  A tile's result does not
// depend on the other tiles of its batch: every kernel works per tile, and
// Omega(j, c) depends on (j, c) only.
static int compress_multi(Context &ctx, std::vector<ProblemJob> &jobs,
                          const EngineParams &ep)
{
    // every return waits for the batch downloads still in flight (their
    // device sources are freed with the records on failure)
    struct CopyDrain {
        cudaStream_t c;
        ~CopyDrain()
        {
            const auto t0 = std::chrono::steady_clock::now();
            cudaStreamSynchronize(c);
            thread_stats().mirror_wait_ms += std::chrono::duration<double, std::milli>(
                std::chrono::steady_clock::now() - t0).count();
        }
    } drain{ctx.copy};
    cudaStream_t s = ctx.stream;
    if (const int e = mapped_area(ctx)) return e;
    starsh_b200_stats &st = thread_stats();
    std::vector<TileWork> all;
    std::vector<std::pair<int, STARSH_int>> owner;   // (job, far block)
    std::vector<double> sep;                          // cluster separation
    int m_max = 0, n_max = 0, k_max = 0;
    bool may_repeat = false;
    std::vector<DevKernel> kernels;
    for (size_t p = 0; p < jobs.size(); ++p) {
        ProblemJob &jb = jobs[p];
        STARSH_blrf *F = jb.F;
        STARSH_cluster *R = F->row_cluster, *C = F->col_cluster;
        const STARSH_int nfar = F->nblocks_far;
        jb.rank.assign(nfar, 0);
        jb.rec->dU.assign(nfar, nullptr);
        jb.rec->dV.assign(nfar, nullptr);
        kernels.push_back(jb.rec->points->K);
        // cluster boxes, for ordering tiles by separation
        const DevicePoints &dp = *jb.rec->points;
        const int nd = dp.K.ndim;
        std::vector<double> rlo, rhi, clo, chi;
        cluster_boxes(dp.h_row, dp.h_row_count, nd, dp.K.aos, R, rlo, rhi);
        cluster_boxes(dp.h_col, dp.h_col_count, nd, dp.K.aos, C, clo, chi);
        // a repeat pass can only be needed when (tol/10)^2 lies below the
        // squared-noise floor of a Gram
        if (nfar > 0 && 0.01 * jb.tol * jb.tol < 1e-15) may_repeat = true;
        for (STARSH_int b = 0; b < nfar; ++b) {
            const STARSH_int i = F->block_far[2 * b], j = F->block_far[2 * b + 1];
            TileWork t;
            memset(&t, 0, sizeof(t));
            t.row0 = R->start[i];
            t.col0 = C->start[j];
            t.m = (int)R->size[i];
            t.n = (int)C->size[j];
            t.k = std::min(jb.maxrank + ep.oversample, std::min(t.m, t.n));
            t.prob = (int)p;
            t.maxrank = jb.maxrank;
            t.tol = jb.tol;
            m_max = std::max(m_max, t.m);
            n_max = std::max(n_max, t.n);
            k_max = std::max(k_max, t.k);
            st.entries += (long long)t.m * t.n;
            // separation of the two clusters relative to the larger
            // diameter: small for near-diagonal (high-rank) blocks
            double gap2 = 0.0, di = 0.0, dj = 0.0;
            for (int d = 0; d < nd; ++d) {
                const double a0 = rlo[(size_t)i * nd + d], a1 = rhi[(size_t)i * nd + d];
                const double b0 = clo[(size_t)j * nd + d], b1 = chi[(size_t)j * nd + d];
                const double g = std::max(0.0, std::max(a0 - b1, b0 - a1));
                gap2 += g * g;
                di += (a1 - a0) * (a1 - a0);
                dj += (b1 - b0) * (b1 - b0);
            }
            const double diam = std::sqrt(std::max(di, dj));
            sep.push_back(diam > 0.0 ? std::sqrt(gap2) / diam : 0.0);
            all.push_back(t);
            owner.emplace_back((int)p, b);
        }
    }
    const long long ntot = (long long)all.size();
    if (ntot == 0) return STARSH_SUCCESS;
    if (k_max > 1024) {
        set_error("maxrank + oversample above 1024 is not supported");
        return STARSH_WRONG_PARAMETER;
    }
    if (!ctx.kernels.reserve(kernels.size() * sizeof(DevKernel), s))
        return cuda_fail(cudaErrorMemoryAllocation, "kernel table");
    B200_CUDA(cudaMemcpyAsync(ctx.kernels.ptr, kernels.data(),
                              kernels.size() * sizeof(DevKernel),
                              cudaMemcpyHostToDevice, s), "kernel table");
    const DevKernel *d_kernels = (const DevKernel *)ctx.kernels.ptr;
    // the kernel family every problem of the call shares, or 0 (the
    // generator then reads each tile's family)
    int one_family = kernels.empty() ? 0 : kernels[0].family;
    for (const DevKernel &K : kernels)
        if (K.family != one_family) one_family = 0;
    // Gaussian sketch, shared by every tile (as the reference reuses the
    // same iseed for every block): n_max x k_max, ld n_max.
    if (ctx.omega_rows != n_max || ctx.omega_cols != k_max) {
        if (!ctx.omega.reserve((size_t)n_max * k_max * sizeof(double), s))
            return cuda_fail(cudaErrorMemoryAllocation, "omega");
        launch_gaussian((double *)ctx.omega.ptr, n_max, k_max, n_max,
                        kOmegaSeed, s);
        count_launch();
        ctx.omega_rows = n_max;
        ctx.omega_cols = k_max;
    }
    const double *omega = (const double *)ctx.omega.ptr;
    // the adaptive engine's int8 sketch matrix (tensor-core sketch)
    bool use_i8 = ep.engine == STARSH_B200_MIXED &&
                  sketch_i8_fits(std::max(ep.block, ep.block_next), n_max);
    if (const char *e = getenv("STARSH_B200_SKETCH"))
        if (strcmp(e, "dmma") == 0) use_i8 = false;
    const int ld_om8 = (n_max + 63) / 64 * 64;
    if (use_i8 && (ctx.omega8_rows != n_max || ctx.omega8_cols != k_max ||
                   ctx.omega8_ld != ld_om8)) {
        if (!ctx.omega8.reserve((size_t)ld_om8 * k_max, s))
            return cuda_fail(cudaErrorMemoryAllocation, "omega8");
        launch_gaussian_i8((int8_t *)ctx.omega8.ptr, n_max, k_max, ld_om8,
                           kOmegaSeed, s);
        count_launch();
        ctx.omega8_rows = n_max;
        ctx.omega8_cols = k_max;
        ctx.omega8_ld = ld_om8;
    }
    const int8_t *om8 = (const int8_t *)ctx.omega8.ptr;
    const int k_max_all = k_max;   // Omega8's width (batches shadow k_max)
    // the first round of the adaptive engine may fuse generation and sketch
    // (opt-in: STARSH_B200_FUSED=1; measured slower than the separate
    // generator and sketch on the square-exponential and Coulomb batches)
    bool fuse_gen = false;
    if (const char *e = getenv("STARSH_B200_FUSED"))
        fuse_gen = use_i8 && strcmp(e, "1") == 0;
    // E[w^2] of the sketch entries: round(32 g) has variance 1024 + 1/12
    for (TileWork &t : all) t.omega_var = use_i8 ? 1024.0 + 1.0 / 12.0 : 1.0;
    st.sketch_int8 = use_i8 ? 1 : 0;

    // Processing order: larger tiles first (a batch's workspace layout is
    // sized by its first tile), then by sketch width, then by cluster
    // separation (near-diagonal, high-rank blocks together, so that their
    // long small-SVD runs share batches), then the problems' block order.
    // Results do not depend on the order.
    {
        std::vector<long long> ord(ntot);
        for (long long q = 0; q < ntot; ++q) ord[q] = q;
        std::stable_sort(ord.begin(), ord.end(), [&](long long a, long long b) {
            const long long sa = (long long)all[a].m * all[a].n;
            const long long sb = (long long)all[b].m * all[b].n;
            if (sa != sb) return sa > sb;
            if (all[a].k != all[b].k) return all[a].k > all[b].k;
            return sep[a] < sep[b];
        });
        std::vector<TileWork> a2(ntot);
        std::vector<std::pair<int, STARSH_int>> o2(ntot);
        for (long long q = 0; q < ntot; ++q) {
            a2[q] = all[ord[q]];
            o2[q] = owner[ord[q]];
        }
        all.swap(a2);
        owner.swap(o2);
    }
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    size_t budget = std::min<size_t>(free_b / 2, (size_t)24 << 30);
    if (const char *e = getenv("STARSH_B200_WORKSPACE_MB"))
        budget = std::min<size_t>(budget, (size_t)atoll(e) << 20);
    budget = std::min(budget, ctx.workspace_cap);
    // Batch plan: each batch takes as many tiles as fit the budget with
    // the layout of its largest dimensions (at most 4096).
    struct BatchPlan { long long b0; int nt; int m, n, k; size_t stride; };
    std::vector<BatchPlan> plan;
    size_t ws_need = 0;
    long long max_slots = 1;
    // the adaptive engine's projection on the tensor cores (needs the
    // int8 path's row maxima and TMA descriptors)
    // (opt-in: STARSH_B200_PROJ=i8 until it beats the FP64 projection)
    bool proj_i8 = false;
    if (const char *e = getenv("STARSH_B200_PROJ"))
        proj_i8 = use_i8 && ep.engine == STARSH_B200_MIXED && strcmp(e, "i8") == 0;
    for (long long b0 = 0; b0 < ntot;) {
        Workspace probe{};
        int bm = all[b0].m, bn = all[b0].n, bk = all[b0].k;
        size_t stride = workspace_layout(probe, bm, bn, bk, true, proj_i8);
        long long cap = (long long)(budget / (stride * sizeof(double)));
        cap = std::max<long long>(1, std::min<long long>({cap, ntot - b0, kMaxBatchTiles}));
        for (long long q = b0; q < b0 + cap; ++q) {
            bm = std::max(bm, all[q].m);
            bn = std::max(bn, all[q].n);
            bk = std::max(bk, all[q].k);
        }
        // even leading dimension (16-byte column strides for the TMA)
        bm = (bm + 7) / 8 * 8;
        stride = workspace_layout(probe, bm, bn, bk, true, proj_i8);
        long long fit = (long long)(budget / (stride * sizeof(double)));
        const int nt = (int)std::max<long long>(1, std::min(cap, fit));
        plan.push_back({b0, nt, bm, bn, bk, stride});
        ws_need = std::max(ws_need, (size_t)nt * stride * sizeof(double));
        max_slots = std::max<long long>(max_slots, nt);
        b0 += nt;
    }
    if (!ctx.workspace.reserve(ws_need, s))
        return cuda_fail(cudaErrorMemoryAllocation, "workspace");
    if (!ctx.tiles.reserve((size_t)max_slots * sizeof(TileWork), s) ||
        !ctx.descs.reserve((size_t)max_slots * sizeof(GemmDesc), s) ||
        !ctx.flag.reserve(256, s) ||
        !ctx.act.reserve((size_t)max_slots * sizeof(int), s))
        return cuda_fail(cudaErrorMemoryAllocation, "batch arrays");
    const size_t pin_need = (size_t)max_slots * sizeof(TileWork);
    if (ctx.tiles_pin_bytes < pin_need) {
        B200_CUDA(cudaStreamSynchronize(s), "tile staging");
        for (void *&q : ctx.tiles_pin) {
            if (q) host_pinned_free(q);
            q = host_pinned_alloc(pin_need);
        }
        ctx.tiles_pin_bytes = ctx.tiles_pin[0] && ctx.tiles_pin[1] ? pin_need : 0;
    }
    // Uploads a batch's tile records through page-locked staging when there
    // is some (a copy from pageable memory would first wait for the whole
    // stream); `which` alternates between the two buffers.  The buffer is
    // free again once the stream has passed the previous upload from it:
    // every batch ends with a stream synchronisation.
    auto upload_tiles = [&](long long b0, int nt, int which) {
        const size_t bytes = (size_t)nt * sizeof(TileWork);
        if (ctx.tiles_pin_bytes >= bytes) {
            memcpy(ctx.tiles_pin[which], &all[b0], bytes);
            return cudaMemcpyAsync(ctx.tiles.ptr, ctx.tiles_pin[which], bytes,
                                   cudaMemcpyHostToDevice, s);
        }
        return cudaMemcpyAsync(ctx.tiles.ptr, &all[b0], bytes,
                               cudaMemcpyHostToDevice, s);
    };
    Workspace ws{};
    TileWork *dt = (TileWork *)ctx.tiles.ptr;
    GemmDesc *dd = (GemmDesc *)ctx.descs.ptr;

    // ev[0..1] sketch GEMM, ev[2..3] projection GEMM, ev[4] generation
    // start, ev[5] basis start, ev[6] SVD end, ev[7..8] output
    cudaEvent_t ev[9];
    for (auto &e : ev) cudaEventCreate(&e);
    bool output_pending = false;
    auto phase_ms = [&](int a, int b) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[a], ev[b]);
        return (double)ms;
    };
    OutArena none{nullptr, nullptr};
    int info = STARSH_SUCCESS;

    // round_count >= 0: the steps of an adaptive round whose sampling
    // tiles (round_count of them, known from the round flag) have compact
    // descriptors; -1: one descriptor per tile of the batch
    int round_count = -1;
    auto gemm = [&](GemmStep step, bool ta, bool tb, int nt, int mm, int nn,
                    OutArena out) -> int {
        const bool compact = round_count >= 0;
        make_gemm_descs(step, dt, nt, ws, omega, n_max, out, dd, s, compact);
        count_launch(2);
        // the transposed products of the adaptive rounds (outputs of a few
        // basis or sample columns, K = the tile height) and the Gram B B^T
        // of the small SVD (K = the tile width) split K inside the CTA
        // where a tile has few rows or columns
        const bool split_k = step == STEP_A_RES_Z || step == STEP_A_GRAM ||
                             step == STEP_A_RES_Z2 || step == STEP_A_GRAM2 ||
                             step == STEP_A_ORTH_Z || step == STEP_A_GRAM_R ||
                             step == STEP_GRAM_B;
        return gemm_f64_batched(ta, tb, dd, compact ? round_count : nt, mm, nn,
                                s, split_k) == cudaSuccess
                   ? STARSH_SUCCESS
                   : cuda_fail(cudaGetLastError(), "gemm_f64_batched");
    };

    for (size_t pi = 0; pi < plan.size() && info == STARSH_SUCCESS; ++pi) {
        const long long b0 = plan[pi].b0;
        const int nt = plan[pi].nt;
        const int m_max = plan[pi].m, k_max = plan[pi].k;
        workspace_layout(ws, plan[pi].m, plan[pi].n, plan[pi].k, true, proj_i8);
        ws.base = (double *)ctx.workspace.ptr;
        ws.stride = plan[pi].stride;
        for (int t = 0; t < nt; ++t) all[b0 + t].slot = t;
        // Round 0 of the adaptive engine with the generation fused into the
        // tensor-core sketch (every tile samples in round 0); tiles whose
        // bound-based row scales missed are sketched again from the stored
        // D, tiles the fused kernel cannot stage (wider than 1024 columns,
        // more than 4 dimensions) are generated and sketched separately.
        // Every choice is made per tile: a tile's result does not depend on
        // its batch.
        const int bmax0 = std::min(ep.block, k_max);
        const bool fused = ep.engine == STARSH_B200_MIXED && fuse_gen &&
            gen_sketch_i8_fits((bmax0 + 15) / 16 * 16);
        bool any_separate = false;
        if (fused)
            for (int t = 0; t < nt; ++t) {
                TileWork &w = all[b0 + t];
                if (!gen_sketch_i8_tile_ok(w.n, kernels[w.prob].ndim)) {
                    w.status |= TILE_GEN_SEPARATE;
                    any_separate = true;
                }
            }
        upload_tiles(b0, nt, 0);
        cudaEventRecord(ev[4], s);
        if (fused) {
            launch_round_setup(dt, nt, ep.block, (int *)ctx.flag.ptr,
                               (int *)ctx.act.ptr, s);
            if (any_separate) {
                launch_gen_tiles(d_kernels, dt, nt, ws, s, TILE_GEN_SEPARATE,
                                 one_family);
                count_launch();
            }
            if (!launch_gen_sketch_i8(d_kernels, dt, nt, ws, om8, ld_om8,
                                      k_max_all, bmax0, s) ||
                !launch_sketch_i8(dt, nt, ws, om8, ld_om8, k_max_all, bmax0, s,
                                  TILE_RESKETCH | TILE_GEN_SEPARATE)) {
                set_error("no TMA tensor map for the fused sketch");
                info = STARSH_UNKNOWN_ERROR;
                break;
            }
            count_launch(3);
            const cudaError_t ce = cudaGetLastError();
            if (ce != cudaSuccess) { info = cuda_fail(ce, "k_gen_sketch_i8"); break; }
        } else {
            launch_gen_tiles(d_kernels, dt, nt, ws, s, 0, one_family);
            count_launch();
        }
        cudaEventRecord(ev[5], s);
        // exact ||D||_F^2 of every block (generator partial sums)
        launch_block_norms(dt, dt, nt, ws, s);
        count_launch();
        if (ep.engine == STARSH_B200_FP64) {
        cudaEventRecord(ev[0], s);
        if ((info = gemm(STEP_SKETCH, false, false, nt, m_max, k_max, none))) break;
        cudaEventRecord(ev[1], s);
        // basis: pass A
        if ((info = gemm(STEP_GRAM_Y, true, false, nt, k_max, k_max, none))) break;
        launch_pivchol(0, dt, dt, nt, ws, s);
        launch_gather_cols(0, dt, nt, ws, s);
        count_launch(2);
        if ((info = gemm(STEP_Q1, false, false, nt, m_max, k_max, none))) break;
        if ((info = gemm(STEP_GRAM_Q1, true, false, nt, k_max, k_max, none))) break;
        launch_chol_inv(0, dt, nt, ws, s);
        count_launch();
        if ((info = gemm(STEP_Q, false, false, nt, m_max, k_max, none))) break;
        // basis: pass B (tiles that do not need it have empty GEMMs)
        if ((info = gemm(STEP_RES_Z, true, false, nt, k_max, k_max, none))) break;
        if ((info = gemm(STEP_RES_Y, false, false, nt, m_max, k_max, none))) break;
        if ((info = gemm(STEP_GRAM_YR, true, false, nt, k_max, k_max, none))) break;
        launch_pivchol(1, dt, dt, nt, ws, s);
        launch_gather_cols(1, dt, nt, ws, s);
        count_launch(2);
        if ((info = gemm(STEP_Q1B, false, false, nt, m_max, k_max, none))) break;
        if ((info = gemm(STEP_RES_Z2, true, false, nt, k_max, k_max, none))) break;
        if ((info = gemm(STEP_RES_Q1B, false, false, nt, m_max, k_max, none))) break;
        if ((info = gemm(STEP_GRAM_Q1B, true, false, nt, k_max, k_max, none))) break;
        launch_chol_inv(1, dt, nt, ws, s);
        count_launch();
        if ((info = gemm(STEP_QB, false, false, nt, m_max, k_max, none))) break;
        launch_merge_basis(dt, nt, s);
        count_launch();
        float ms = 0.f;
        cudaEventSynchronize(ev[1]);
        cudaEventElapsedTime(&ms, ev[0], ev[1]);
        st.sketch_ms += ms;
        st.sketch_launches += 1;
        } else {
        // Adaptive sketch: sample Omega in blocks; each round projects the
        // new sample off the basis, keeps the residual directions above
        // (tol/10)^2 ||D||_F^2 and stops a tile once `verify` columns of a
        // round stayed below that threshold (the residual estimate of
        // N. Halko, P.-G. Martinsson, J. A. Tropp, SIAM Review 53 (2011)
        // sec. 4.3), when a round adds none, or after k columns.
        int *d_active = (int *)ctx.flag.ptr;
        bool any_width = false;
        for (int t = 0; t < nt && !any_width; ++t) any_width = all[b0 + t].k > 0;
        // the per-tile kernels of a round: over its sampling tiles alone
        // when their count is known (round_count), else the whole batch
        const int *act = (const int *)ctx.act.ptr;
        auto rcount = [&]() { return round_count >= 0 ? round_count : nt; };
        auto ract = [&]() { return round_count >= 0 ? act : nullptr; };
        auto append = [&](int bmax) -> int {
            // orthonormalise the selected residual columns (kb of them)
            // against the basis and append them: CholQR of R_J, one more
            // projection, CholQR again (CGS2)
            int e;
            launch_gather_cols(1, dt, rcount(), ws, s, ract());
            count_launch();
            if ((e = gemm(STEP_A_Q1B, false, false, nt, m_max, bmax, none))) return e;
            if ((e = gemm(STEP_A_ORTH_Z, true, false, nt, k_max, bmax, none))) return e;
            if ((e = gemm(STEP_A_ORTH_R, false, false, nt, m_max, bmax, none))) return e;
            if ((e = gemm(STEP_A_GRAM_R, true, false, nt, bmax, bmax, none))) return e;
            launch_chol_inv(1, dt, rcount(), ws, s, ract());
            count_launch();
            if ((e = gemm(STEP_A_QB, false, false, nt, m_max, bmax, none))) return e;
            launch_merge_basis(dt, nt, s);
            count_launch();
            return STARSH_SUCCESS;
        };
        for (int round = 0; info == STARSH_SUCCESS; ++round) {
            const int block = round == 0 ? ep.block : ep.block_next;
            const int bmax = std::min(block, k_max);
            const bool pre_sketched = fused && round == 0;
            round_count = -1;
            if (!pre_sketched) {
            launch_round_setup(dt, nt, block, d_active, (int *)ctx.act.ptr, s);
            count_launch();
            // round 0 samples every tile with a sketch width (known on
            // the host): the round is enqueued behind the generation
            // without waiting for the flag; later rounds read how many
            // tiles sample and run their GEMMs over those alone
            if (round > 0 || !any_width) {
                k_count_to_host<<<1, 1, 0, s>>>(d_active, (int *)ctx.mapped_dev);
                count_launch();
                B200_CUDA(cudaGetLastError(), "k_count_to_host");
                B200_CUDA(cudaStreamSynchronize(s), "round flag");
                const int active = *(volatile int *)ctx.mapped;
                if (!active) break;
                round_count = active;
            }
            }
            cudaEventRecord(ev[0], s);
            if (pre_sketched) {
                // Y of round 0 came with the generation
            } else if (use_i8) {
                // every batch has an even leading dimension (plan), so the
                // tensor map exists unless the driver lacks the entry point
                if (!launch_sketch_i8(dt, nt, ws, om8, ld_om8, k_max_all, bmax, s)) {
                    set_error("no TMA tensor map for the sketch");
                    info = STARSH_UNKNOWN_ERROR;
                    break;
                }
                count_launch();
                const cudaError_t ce = cudaGetLastError();
                if (ce != cudaSuccess) { info = cuda_fail(ce, "k_sketch_i8"); break; }
            } else if ((info = gemm(STEP_A_SKETCH, false, false, nt, m_max, bmax, none))) {
                break;
            }
            cudaEventRecord(ev[1], s);
            if (round > 0) {
                if ((info = gemm(STEP_A_RES_Z, true, false, nt, k_max, bmax, none))) break;
                if ((info = gemm(STEP_A_RES_Y, false, false, nt, m_max, bmax, none))) break;
            }
            if ((info = gemm(STEP_A_GRAM, true, false, nt, bmax, bmax, none))) break;
            launch_round_pivchol(dt, rcount(), ws, 0, s, ract());
            count_launch();
            if ((info = append(bmax))) break;
            if (may_repeat) {
                // same sample, projected off the grown basis once more
                if ((info = gemm(STEP_A_RES_Z2, true, false, nt, k_max, bmax, none))) break;
                if ((info = gemm(STEP_A_RES_Y2, false, false, nt, m_max, bmax, none))) break;
                if ((info = gemm(STEP_A_GRAM2, true, false, nt, bmax, bmax, none))) break;
                launch_round_pivchol(dt, rcount(), ws, 1, s, ract());
                count_launch();
                if ((info = append(bmax))) break;
            }
            launch_round_end(dt, nt, ep.verify, s);
            count_launch();
            if (!pre_sketched) {
                float ms = 0.f;
                cudaEventSynchronize(ev[1]);
                cudaEventElapsedTime(&ms, ev[0], ev[1]);
                st.sketch_ms += ms;
                st.sketch_launches += 1;
            }
        }
        round_count = -1;
        if (info) break;
        }
        // projection (tiles with at most 64 basis columns on the tensor
        // cores, the others FP64) and small SVD
        cudaEventRecord(ev[2], s);
        if (proj_i8) {
            launch_proj_prep(dt, nt, ws, s);
            if (!launch_proj_i8(dt, nt, ws, s)) {
                set_error("no TMA tensor map for the projection");
                info = STARSH_UNKNOWN_ERROR;
                break;
            }
            count_launch(2);
        }
        if ((info = gemm(STEP_PROJECT, true, false, nt, k_max, plan[pi].n, none))) break;
        cudaEventRecord(ev[3], s);
        if ((info = gemm(STEP_GRAM_B, false, true, nt, k_max, k_max, none))) break;
        count_launch(launch_pivchol(2, dt, dt, nt, ws, s));
        count_launch(launch_jacobi(dt, nt, ws, s, ctx.side));
        if ((info = gemm(STEP_ROTATE, true, false, nt, k_max, plan[pi].n, none))) break;
        launch_rank_cut(dt, nt, ws, s);
        count_launch();
        cudaEventRecord(ev[6], s);
        {
            static_assert(sizeof(TileWork) % 8 == 0, "TileWork in 8-byte words");
            const size_t words = (size_t)nt * sizeof(TileWork) / 8;
            k_store_to_host<<<(unsigned)std::min<size_t>(296, (words + 255) / 256), 256, 0, s>>>(
                (const unsigned long long *)dt,
                (unsigned long long *)((char *)ctx.mapped_dev + kMappedRecords), words);
            count_launch();
            B200_CUDA(cudaGetLastError(), "k_store_to_host");
        }
        B200_CUDA(cudaStreamSynchronize(s), "compression pipeline");
        memcpy(&all[b0], (const char *)ctx.mapped + kMappedRecords,
               (size_t)nt * sizeof(TileWork));
        st.project_ms += phase_ms(2, 3);
        st.gen_ms += phase_ms(4, 5);
        if (fused) {
            st.fused_ms += phase_ms(4, 5);
            st.fused_launches += 1;
        }
        st.basis_ms += phase_ms(5, 2);
        st.svd_ms += phase_ms(3, 6);
        if (output_pending) st.output_ms += phase_ms(7, 8);
        output_pending = false;
        // Output placement of this batch: one device chunk, the U then V
        // factors of each problem contiguous (so every problem's host
        // mirror is a concatenation of its parts), shared by the records
        // of the problems with tiles here.
        std::vector<size_t> nu(jobs.size(), 0), nv(jobs.size(), 0);
        for (int t = 0; t < nt; ++t) {
            TileWork &w = all[b0 + t];
            st.sketch_flops += 2.0 * w.m * w.n *
                (ep.engine == STARSH_B200_FP64 ? w.k : w.cols_done);
            {
                // D is read once per round the tile takes part in, Y written
                // (the fused round 0 writes D and its Y instead of reading D)
                const int cols = ep.engine == STARSH_B200_FP64 ? w.k : w.cols_done;
                int rounds = ep.engine == STARSH_B200_FP64 ? 1
                    : 1 + (std::max(0, cols - ep.block) + ep.block_next - 1) / ep.block_next;
                int ycols = cols;
                if (fused) {
                    const int c0 = std::min(cols, bmax0);
                    st.fused_bytes += 8.0 * ((double)w.m * w.n + (double)w.m * c0);
                    rounds -= 1;
                    ycols -= c0;
                    if (w.status & TILE_RESKETCH) st.resketch_tiles += 1;
                }
                st.sketch_bytes += 8.0 * ((double)w.m * w.n * rounds + (double)w.m * ycols);
            }
            st.project_flops += 2.0 * w.m * w.n * w.k1;
            if (w.status & TILE_MMA_TIMEOUT) {
                set_error("tensor-core sketch timed out on a tile");
                info = STARSH_UNKNOWN_ERROR;
            }
            jobs[w.prob].rank[owner[b0 + t].second] = w.rank;
            if (w.rank > 0) {
                nu[w.prob] += (size_t)w.m * w.rank;
                nv[w.prob] += (size_t)w.n * w.rank;
            }
        }
        if (info) break;
        std::vector<size_t> u0(jobs.size()), v0(jobs.size());
        size_t total = 0;
        for (size_t p = 0; p < jobs.size(); ++p) {
            u0[p] = total;
            v0[p] = total + nu[p];
            total += nu[p] + nv[p];
        }
        std::shared_ptr<void> chunk;
        if (total > 0) {
            void *raw = pool_alloc(total * sizeof(double), s);
            if (raw == nullptr) {
                info = cuda_fail(cudaErrorMemoryAllocation, "factor chunk");
                break;
            }
            chunk = std::shared_ptr<void>(raw, [](void *q) { pool_free(q); });
        }
        double *base = (double *)chunk.get();
        std::vector<size_t> cu(u0), cv(v0);
        for (int t = 0; t < nt; ++t) {
            TileWork &w = all[b0 + t];
            if (w.rank <= 0) continue;
            w.off_u = (long long)cu[w.prob];
            w.off_v = (long long)cv[w.prob];
            cu[w.prob] += (size_t)w.m * w.rank;
            cv[w.prob] += (size_t)w.n * w.rank;
            Record *rec = jobs[w.prob].rec;
            rec->dU[owner[b0 + t].second] = base + w.off_u;
            rec->dV[owner[b0 + t].second] = base + w.off_v;
        }
        std::vector<size_t> part_of(jobs.size(), 0);
        for (size_t p = 0; p < jobs.size(); ++p) {
            if (nu[p] + nv[p] == 0) continue;
            Record *rec = jobs[p].rec;
            rec->shared.push_back(chunk);
            part_of[p] = rec->parts.size();
            rec->parts.push_back({base + u0[p], nu[p], base + v0[p], nv[p]});
            rec->u_total += nu[p];
            rec->v_total += nv[p];
        }
        if (total > 0) {
            OutArena out{base, base};
            upload_tiles(b0, nt, 1);
            cudaEventRecord(ev[7], s);
            launch_select_w(dt, nt, ws, s);
            count_launch();
            if ((info = gemm(STEP_OUT_U, false, false, nt, m_max, k_max, out))) break;
            launch_write_v(dt, nt, ws, out, s);
            count_launch();
            cudaEventRecord(ev[8], s);
            output_pending = true;
            if (ep.mirror) {
                // each problem's factors of this batch go to page-locked
                // host memory on the copy stream while later batches run
                B200_CUDA(cudaStreamWaitEvent(ctx.copy, ev[8], 0), "mirror wait");
                for (size_t p = 0; p < jobs.size(); ++p) {
                    if (nu[p] + nv[p] == 0) continue;
                    double *h = (double *)host_pinned_alloc(
                        (nu[p] + nv[p]) * sizeof(double));
                    if (h == nullptr) continue;   // mirrored later, staged
                    B200_CUDA(cudaMemcpyAsync(h, base + u0[p],
                                              (nu[p] + nv[p]) * sizeof(double),
                                              cudaMemcpyDeviceToHost, ctx.copy),
                              "mirror copy");
                    Record::Part &pt = jobs[p].rec->parts[part_of[p]];
                    pt.hU = h;
                    pt.hV = h + nu[p];
                }
            }
        }
        if (const char *path = getenv("STARSH_B200_TILE_LOG")) {
            // diagnostics: one line per tile of the shape, basis and factor
            // sizes, Jacobi sweeps and rank
            if (FILE *f = fopen(path, b0 == 0 ? "w" : "a")) {
                for (int t = 0; t < nt; ++t) {
                    const TileWork &w = all[b0 + t];
                    fprintf(f, "%d %d %d %d %d %d %d %d\n", w.m, w.n, w.cols_done,
                            w.k1, w.k2, w.sweeps, w.rank, w.status);
                }
                fclose(f);
            }
        }
        st.tiles += nt;
        st.batches += 1;
    }
    if (info == STARSH_SUCCESS) {
        B200_CUDA(cudaStreamSynchronize(s), "factor output");
        if (output_pending) st.output_ms += phase_ms(7, 8);
    }
    for (auto &e : ev) cudaEventDestroy(e);
    return info;
}

// Device bytes held by a matrix of this library: factors, dense near-field
// blocks and the problem's points (0 if M has no device record).
size_t matrix_device_bytes(const STARSH_blrm *M)
{
    Record *rec = find_record(M);
    if (rec == nullptr) return 0;
    return (rec->u_total + rec->v_total + rec->d_total) * sizeof(double) +
           (rec->points ? rec->points->h2d : 0);
}

// Host Array view helper (shape m x n, column-major).
static int make_view(Array **A, int m, int n, double *data)
{
    int shape[2] = {m, n};
    return array_from_buffer(A, 2, shape, 'd', 'F', data);
}

// Copies device memory into pageable (malloc'd) host memory through two
// pinned staging buffers: the DMA of one chunk overlaps the host-side copy
// of the previous one, and that copy -- which also takes the first-touch
// page faults of the destination -- is split over several threads.  A
// plain cudaMemcpy into fresh malloc'd memory is limited by those faults.
constexpr size_t kStageBytes = 64u << 20;

static void parallel_memcpy(char *dst, const char *src, size_t n)
{
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t per = (n + hw - 1) / hw;
    std::vector<std::thread> th;
    for (unsigned t = 1; t < hw && t * per < n; ++t)
        th.emplace_back([=] { memcpy(dst + t * per, src + t * per,
                                     std::min(per, n - t * per)); });
    memcpy(dst, src, std::min(per, n));
    for (auto &x : th) x.join();
}

struct D2HCopy {
    char *dst;
    const char *src;
    size_t n;
};

static int staged_d2h(Context &ctx, const std::vector<D2HCopy> &jobs,
                      cudaStream_t s)
{
    if (!ctx.stage[0]) {
        for (int i = 0; i < 2; ++i)
            B200_CUDA(cudaMallocHost(&ctx.stage[i], kStageBytes),
                      "cudaMallocHost(staging)");
        for (int i = 0; i < 2; ++i)
            B200_CUDA(cudaEventCreateWithFlags(&ctx.stage_ev[i],
                                               cudaEventDisableTiming),
                      "cudaEventCreate(staging)");
    }
    // flatten into chunks of at most kStageBytes
    struct Chunk { char *dst; const char *src; size_t n; };
    std::vector<Chunk> chunks;
    for (const D2HCopy &j : jobs)
        for (size_t o = 0; o < j.n; o += kStageBytes)
            chunks.push_back({j.dst + o, j.src + o, std::min(kStageBytes, j.n - o)});
    for (size_t c = 0; c < chunks.size(); ++c) {
        const int b = (int)(c & 1);
        B200_CUDA(cudaMemcpyAsync(ctx.stage[b], chunks[c].src, chunks[c].n,
                                  cudaMemcpyDeviceToHost, s), "staged D2H");
        B200_CUDA(cudaEventRecord(ctx.stage_ev[b], s), "staged D2H event");
        if (c >= 1) {
            const int pb = (int)((c - 1) & 1);
            B200_CUDA(cudaEventSynchronize(ctx.stage_ev[pb]), "staged D2H wait");
            parallel_memcpy(chunks[c - 1].dst, (const char *)ctx.stage[pb],
                            chunks[c - 1].n);
        }
    }
    if (!chunks.empty()) {
        const size_t c = chunks.size() - 1;
        const int b = (int)(c & 1);
        B200_CUDA(cudaEventSynchronize(ctx.stage_ev[b]), "staged D2H wait");
        parallel_memcpy(chunks[c].dst, (const char *)ctx.stage[b], chunks[c].n);
    }
    return STARSH_SUCCESS;
}

// Host mirrors held in page-locked blocks of the pinned pool, by matrix.
static std::mutex g_mirror_mu;
static std::unordered_map<const STARSH_blrm *, std::vector<void *>> g_mirrors;

// The host mirror from the parts downloaded batch by batch (the copies
// have completed): far_U/far_V point into the parts' page-locked blocks,
// the near blocks are copied into one more.
static int map_early_mirror(STARSH_blrm *M, Record &rec, cudaStream_t s)
{
    STARSH_blrf *F = M->format;
    starsh_b200_stats &st = thread_stats();
    struct Span { const double *dev; size_t n; double *host; };
    std::vector<Span> su, sv;
    for (const Record::Part &pt : rec.parts) {
        su.push_back({pt.U, pt.nu, pt.hU});
        sv.push_back({pt.V, pt.nv, pt.hV});
    }
    auto by_dev = [](const Span &a, const Span &b) { return a.dev < b.dev; };
    std::sort(su.begin(), su.end(), by_dev);
    std::sort(sv.begin(), sv.end(), by_dev);
    auto host_of = [](const std::vector<Span> &sp, const double *d) -> double * {
        auto it = std::upper_bound(sp.begin(), sp.end(), Span{d, 0, nullptr},
                                   [](const Span &a, const Span &b) {
                                       return a.dev < b.dev;
                                   });
        if (it == sp.begin()) return nullptr;
        --it;
        if (d < it->dev || d >= it->dev + it->n) return nullptr;
        return it->host + (d - it->dev);
    };
    for (STARSH_int b = 0; b < F->nblocks_far; ++b) {
        // blocks without factors point at the first block, as in the
        // single-allocation mirror
        M->far_U[b]->data = rec.parts[0].hU;
        M->far_V[b]->data = rec.parts[0].hV;
        if (M->far_rank[b] <= 0) continue;
        double *hu = host_of(su, rec.dU[b]), *hv = host_of(sv, rec.dV[b]);
        if (hu == nullptr || hv == nullptr) {
            set_error("host mirror: factor outside its chunks");
            return STARSH_UNKNOWN_ERROR;
        }
        M->far_U[b]->data = hu;
        M->far_V[b]->data = hv;
    }
    std::vector<void *> owned;
    double *hD = nullptr;
    bool d_pinned = false;
    if (M->onfly == 0 && F->nblocks_near > 0) {
        const size_t bytes = std::max<size_t>(rec.d_total, 1) * sizeof(double);
        hD = (double *)host_pinned_alloc(bytes);
        d_pinned = hD != nullptr;
        if (!d_pinned) hD = (double *)malloc(bytes);
        if (hD == nullptr) return STARSH_MALLOC_ERROR;
        if (rec.d_total) {
            // near blocks live in one contiguous device allocation
            cudaError_t e = d_pinned
                ? cudaMemcpyAsync(hD, rec.dD[0], rec.d_total * sizeof(double),
                                  cudaMemcpyDeviceToHost, s)
                : cudaSuccess;
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            int info = e == cudaSuccess ? STARSH_SUCCESS : cuda_fail(e, "near mirror");
            if (!info && !d_pinned)
                info = staged_d2h(*context(),
                                  {{(char *)hD, (const char *)rec.dD[0],
                                    rec.d_total * sizeof(double)}}, s);
            if (info) {
                if (d_pinned) host_pinned_free(hD);
                else free(hD);
                return info;
            }
        }
        size_t od = 0;
        for (STARSH_int b = 0; b < F->nblocks_near; ++b) {
            M->near_D[b]->data = hD + od;
            od += M->near_D[b]->size;
        }
        if (d_pinned) owned.push_back(hD);
    }
    // the matrix owns the blocks from here on (the device record may be
    // released before it)
    for (Record::Part &pt : rec.parts) {
        owned.push_back(pt.hU);
        pt.hU = pt.hV = nullptr;
    }
    {
        std::lock_guard<std::mutex> g(g_mirror_mu);
        g_mirrors[M] = std::move(owned);
    }
    st.d2h_bytes += (long long)(rec.u_total + rec.v_total + rec.d_total) * 8;
    M->alloc_U = nullptr;
    M->alloc_V = nullptr;
    M->alloc_D = d_pinned ? nullptr : hD;
    rec.host_filled = true;
    return STARSH_SUCCESS;
}

static int fill_host_mirror(STARSH_blrm *M, Record &rec, cudaStream_t s)
{
    if (rec.host_filled) return STARSH_SUCCESS;
    bool early = !rec.parts.empty();
    for (const Record::Part &pt : rec.parts) early = early && pt.hU != nullptr;
    if (early) return map_early_mirror(M, rec, s);
    STARSH_blrf *F = M->format;
    starsh_b200_stats &st = thread_stats();
    double *hU = (double *)malloc(std::max<size_t>(rec.u_total, 1) * sizeof(double));
    double *hV = (double *)malloc(std::max<size_t>(rec.v_total, 1) * sizeof(double));
    double *hD = nullptr;
    if (!hU || !hV) {
        free(hU);
        free(hV);
        return STARSH_MALLOC_ERROR;
    }
    // One copy per factor chunk; views follow the same order.
    std::vector<D2HCopy> jobs;
    size_t ou = 0, ov = 0;
    for (const Record::Part &pt : rec.parts) {
        jobs.push_back({(char *)(hU + ou), (const char *)pt.U, pt.nu * sizeof(double)});
        jobs.push_back({(char *)(hV + ov), (const char *)pt.V, pt.nv * sizeof(double)});
        ou += pt.nu;
        ov += pt.nv;
    }
    // Each block's host position: the host offset of the part holding its
    // device factors plus its offset inside that part (tiles of a problem
    // may have been processed in any order).
    struct Span { const double *dev; size_t n, host; };
    std::vector<Span> su, sv;
    ou = ov = 0;
    for (const Record::Part &pt : rec.parts) {
        su.push_back({pt.U, pt.nu, ou});
        sv.push_back({pt.V, pt.nv, ov});
        ou += pt.nu;
        ov += pt.nv;
    }
    auto by_dev = [](const Span &a, const Span &b) { return a.dev < b.dev; };
    std::sort(su.begin(), su.end(), by_dev);
    std::sort(sv.begin(), sv.end(), by_dev);
    auto host_of = [](const std::vector<Span> &sp, const double *d) -> size_t {
        auto it = std::upper_bound(sp.begin(), sp.end(), Span{d, 0, 0},
                                   [](const Span &a, const Span &b) {
                                       return a.dev < b.dev;
                                   });
        if (it == sp.begin()) return SIZE_MAX;
        --it;
        if (d < it->dev || d >= it->dev + it->n) return SIZE_MAX;
        return it->host + (size_t)(d - it->dev);
    };
    for (STARSH_int b = 0; b < F->nblocks_far; ++b) {
        M->far_U[b]->data = hU;
        M->far_V[b]->data = hV;
        if (M->far_rank[b] <= 0) continue;
        const size_t pu = host_of(su, rec.dU[b]), pv = host_of(sv, rec.dV[b]);
        if (pu == SIZE_MAX || pv == SIZE_MAX) {
            free(hU);
            free(hV);
            set_error("host mirror: factor outside its chunks");
            return STARSH_UNKNOWN_ERROR;
        }
        M->far_U[b]->data = hU + pu;
        M->far_V[b]->data = hV + pv;
    }
    if (M->onfly == 0 && F->nblocks_near > 0) {
        hD = (double *)malloc(std::max<size_t>(rec.d_total, 1) * sizeof(double));
        if (!hD) {
            free(hU);
            free(hV);
            return STARSH_MALLOC_ERROR;
        }
        // near blocks live in one contiguous device allocation
        if (rec.d_total)
            jobs.push_back({(char *)hD, (const char *)rec.dD[0],
                            rec.d_total * sizeof(double)});
        size_t od = 0;
        for (STARSH_int b = 0; b < F->nblocks_near; ++b) {
            M->near_D[b]->data = hD + od;
            od += M->near_D[b]->size;
        }
    }
    cudaError_t e = cudaStreamSynchronize(s);
    int info = e == cudaSuccess ? staged_d2h(*context(), jobs, s)
                                : cuda_fail(e, "host mirror copy");
    if (info) {
        free(hU);
        free(hV);
        free(hD);
        return info;
    }
    st.d2h_bytes += (long long)(rec.u_total + rec.v_total + rec.d_total) * 8;
    M->alloc_U = hU;
    M->alloc_V = hV;
    M->alloc_D = hD;
    rec.host_filled = true;
    return STARSH_SUCCESS;
}

// Turns the compressed far blocks of one problem into its STARSH_blrm:
// demotes false far-field blocks, generates the near-field blocks and builds
// the host structure (with its host mirror if requested).  On success the
// job's record belongs to the record table.
static int finish_problem(ProblemJob &jb, int flags, cudaStream_t s,
                          STARSH_blrm **matrix)
{
    starsh_b200_stats &st = thread_stats();
    STARSH_blrf *F = jb.F;
    STARSH_problem *P = F->problem;
    STARSH_cluster *R = F->row_cluster, *C = F->col_cluster;
    Record *rec = jb.rec;
    const std::vector<int> &rank = jb.rank;
    const int onfly = jb.onfly;
    int info = STARSH_SUCCESS;
    // False far-field blocks (rank -1) become near-field; the format is
    // rebuilt and swapped into *F, the old lists freed.
    const STARSH_int nfar = F->nblocks_far, nnear = F->nblocks_near;
    std::vector<STARSH_int> keep, demote;
    for (STARSH_int b = 0; b < nfar; ++b)
        (rank[b] < 0 ? demote : keep).push_back(b);
    st.false_far += (long long)demote.size();
    std::vector<double *> dU, dV;
    std::vector<int> far_rank;
    for (STARSH_int b : keep) {
        dU.push_back(rec->dU[b]);
        dV.push_back(rec->dV[b]);
        far_rank.push_back(rank[b]);
        st.rank_sum += rank[b];
        st.max_rank = std::max(st.max_rank, rank[b]);
    }
    if (!demote.empty()) {
        const STARSH_int new_near = nnear + (STARSH_int)demote.size();
        const STARSH_int new_far = (STARSH_int)keep.size();
        STARSH_int *bn = (STARSH_int *)malloc(sizeof(STARSH_int) * 2 * new_near);
        STARSH_int *bf = new_far > 0
            ? (STARSH_int *)malloc(sizeof(STARSH_int) * 2 * new_far) : nullptr;
        if (!bn || (new_far > 0 && !bf)) {
            free(bn);
            free(bf);
            return STARSH_MALLOC_ERROR;
        }
        for (STARSH_int b = 0; b < 2 * nnear; ++b) bn[b] = F->block_near[b];
        for (size_t q = 0; q < demote.size(); ++q) {
            bn[2 * (nnear + q)] = F->block_far[2 * demote[q]];
            bn[2 * (nnear + q) + 1] = F->block_far[2 * demote[q] + 1];
        }
        for (size_t q = 0; q < keep.size(); ++q) {
            bf[2 * q] = F->block_far[2 * keep[q]];
            bf[2 * q + 1] = F->block_far[2 * keep[q] + 1];
        }
        STARSH_blrf *F2 = nullptr;
        info = starsh_blrf_new_from_coo(&F2, P, F->symm, R, C, new_far, bf,
                                        new_near, bn, F->type);
        if (info) {
            free(bn);
            free(bf);
            return info;
        }
        STARSH_blrf tmp = *F;
        *F = *F2;
        *F2 = tmp;
        starsh_blrf_free(F2);
    }
    rec->dU = dU;
    rec->dV = dV;

    // Near-field blocks: dense on the device unless onfly.
    const STARSH_int near = F->nblocks_near;
    rec->dD.assign(near, nullptr);
    if (onfly == 0 && near > 0) {
        size_t total = 0;
        for (STARSH_int b = 0; b < near; ++b)
            total += (size_t)R->size[F->block_near[2 * b]] *
                     C->size[F->block_near[2 * b + 1]];
        double *dD = (double *)pool_alloc(total * sizeof(double), s);
        if (dD == nullptr)
            return cuda_fail(cudaErrorMemoryAllocation, "near blocks");
        rec->chunks.push_back(dD);
        rec->d_total = total;
        std::vector<BlockJob> jobs;
        size_t off = 0;
        for (STARSH_int b = 0; b < near; ++b) {
            const STARSH_int i = F->block_near[2 * b], j = F->block_near[2 * b + 1];
            BlockJob bj{R->start[i], C->start[j], (int)R->size[i],
                        (int)C->size[j], dD + off};
            rec->dD[b] = dD + off;
            jobs.push_back(bj);
            off += (size_t)bj.m * bj.n;
            st.entries += (long long)bj.m * bj.n;
        }
        if ((info = gen_blocks(rec->points->K, jobs, s))) {
            return info;
        }
    } else {
        for (STARSH_int b = 0; b < near; ++b)
            st.entries += (long long)R->size[F->block_near[2 * b]] *
                          C->size[F->block_near[2 * b + 1]];
    }

    // Host STARSH_blrm with views (data filled by the host mirror).
    const STARSH_int nf = F->nblocks_far;
    int *fr = nf > 0 ? (int *)malloc(sizeof(int) * nf) : nullptr;
    Array **fU = nf > 0 ? (Array **)calloc(nf, sizeof(Array *)) : nullptr;
    Array **fV = nf > 0 ? (Array **)calloc(nf, sizeof(Array *)) : nullptr;
    Array **nD = (onfly == 0 && near > 0)
                     ? (Array **)calloc(near, sizeof(Array *)) : nullptr;
    for (STARSH_int b = 0; b < nf; ++b) {
        fr[b] = far_rank[b];
        const int m = (int)R->size[F->block_far[2 * b]];
        const int n = (int)C->size[F->block_far[2 * b + 1]];
        make_view(&fU[b], m, fr[b], nullptr);
        make_view(&fV[b], n, fr[b], nullptr);
    }
    for (STARSH_int b = 0; nD && b < near; ++b) {
        const int m = (int)R->size[F->block_near[2 * b]];
        const int n = (int)C->size[F->block_near[2 * b + 1]];
        make_view(&nD[b], m, n, nullptr);
    }
    STARSH_blrm *M = nullptr;
    info = starsh_blrm_new(&M, F, fr, fU, fV, onfly, nD, nullptr, nullptr,
                           nullptr, '1');
    if (info) return info;
    add_record(M, rec);
    jb.rec = nullptr;   // owned by the record table now
    if (flags & STARSH_B200_HOST_MIRROR) {
        info = fill_host_mirror(M, *rec, s);
    } else {
        const cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) info = cuda_fail(e, "near blocks");
    }
    if (info) {
        starsh_blrm_free(M);   // releases the record as well
        return info;
    }
    *matrix = M;
    return STARSH_SUCCESS;
}

static void read_engine_env(EngineParams &ep)
{
    ep.block = 64;
    ep.block_next = 32;
    ep.verify = 10;
    if (const char *e = getenv("STARSH_B200_SKETCH_BLOCK"))
        ep.block = std::max(8, std::min(1024, atoi(e)));
    if (const char *e = getenv("STARSH_B200_SKETCH_STEP"))
        ep.block_next = std::max(8, std::min(1024, atoi(e)));
    if (const char *e = getenv("STARSH_B200_SKETCH_VERIFY"))
        ep.verify = std::max(1, std::min(1024, atoi(e)));
}

// Approximates `np` problems in shared batches (every launch carries tiles
// of all of them).  matrices[p] receives the result of formats[p]; each
// format is updated in place on demotion as by the single-problem call.
static int approximate_batch(int np, STARSH_blrm **matrices,
                             STARSH_blrf **formats, const int *maxranks,
                             const double *tols, const int *onflys,
                             int engine, int flags)
{
    auto t_start = std::chrono::steady_clock::now();
    starsh_b200_stats &st = thread_stats();
    memset(&st, 0, sizeof(st));
    const long long launches0 = launch_count();
    if (np <= 0 || matrices == nullptr || formats == nullptr ||
        maxranks == nullptr || tols == nullptr) {
        set_error("invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    for (int p = 0; p < np; ++p) {
        const int onfly = onflys ? onflys[p] : 0;
        if (formats[p] == nullptr ||
            maxranks[p] < 0 || !(tols[p] >= 0.0) ||
            (onfly != 0 && onfly != 1)) {
            set_error("invalid argument");
            return STARSH_WRONG_PARAMETER;
        }
        for (int q = 0; q < p; ++q)
            if (formats[q] == formats[p]) {
                set_error("the same format appears twice in one batch");
                return STARSH_WRONG_PARAMETER;
            }
        STARSH_blrf *F = formats[p];
        STARSH_problem *P = F->problem;
        if (P == nullptr || F->row_cluster == nullptr ||
            F->col_cluster == nullptr || P->ndim != 2 || P->dtype != 'd') {
            set_error("only scalar double-precision problems are supported");
            return STARSH_WRONG_PARAMETER;
        }
    }
    if (engine != STARSH_B200_FP64 && engine != STARSH_B200_MIXED) {
        set_error("unknown engine");
        return STARSH_WRONG_PARAMETER;
    }
    Context *ctx = context();
    if (!ctx) return STARSH_UNKNOWN_ERROR;
    std::lock_guard<std::mutex> guard(ctx->lock);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;

    std::vector<ProblemJob> jobs(np);
    auto cleanup = [&]() {
        for (ProblemJob &jb : jobs) {
            delete jb.rec;
            jb.rec = nullptr;
        }
    };
    for (int p = 0; p < np; ++p) {
        ProblemJob &jb = jobs[p];
        jb.F = formats[p];
        jb.maxrank = maxranks[p];
        jb.tol = tols[p];
        jb.onfly = onflys ? onflys[p] : 0;
        jb.rec = new Record();
        jb.rec->points = new DevicePoints();
        int info = upload_problem(*jb.rec->points, jb.F->problem,
                                  jb.F->row_cluster, jb.F->col_cluster, s);
        if (info) {
            cleanup();
            return info;
        }
        st.h2d_bytes += jb.rec->points->h2d;
    }
    EngineParams ep{};
    ep.oversample = b200_oversample();
    ep.engine = engine;
    ep.mirror = (flags & STARSH_B200_HOST_MIRROR) != 0;
    read_engine_env(ep);
    int info = compress_multi(*ctx, jobs, ep);
    const auto t_finish = std::chrono::steady_clock::now();
    int done = 0;
    for (; done < np && info == STARSH_SUCCESS; ++done)
        info = finish_problem(jobs[done], flags, s, &matrices[done]);
    st.finish_ms = std::chrono::duration<double, std::milli>(
                       std::chrono::steady_clock::now() - t_finish).count();
    if (info) {
        // the problems finished before the failure are released too
        for (int q = 0; q + 1 < done; ++q) {
            starsh_blrm_free(matrices[q]);
            matrices[q] = nullptr;
        }
        cleanup();
        return info;
    }
    st.kernel_launches = launch_count() - launches0;
    st.device_ms = st.sketch_ms + st.project_ms;
    st.total_ms = std::chrono::duration<double, std::milli>(
                      std::chrono::steady_clock::now() - t_start).count();
    return STARSH_SUCCESS;
}

static int approximate(STARSH_blrm **matrix, STARSH_blrf *F, int maxrank,
                       double tol, int onfly, int engine, int flags)
{
    if (matrix == nullptr || F == nullptr) {
        set_error("invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    return approximate_batch(1, matrix, &F, &maxrank, &tol, &onfly, engine,
                             flags);
}

}  // namespace b200

using namespace b200;

// ------------------------------------------------------------ C entries

extern "C" int starsh_b200_approximate(STARSH_blrm **matrix,
                                       STARSH_blrf *format, int maxrank,
                                       double tol, int onfly, int engine,
                                       int flags)
{
    return approximate(matrix, format, maxrank, tol, onfly, engine, flags);
}

extern "C" int starsh_b200_approximate_batch(int nprob, STARSH_blrm **matrices,
                                             STARSH_blrf **formats,
                                             const int *maxrank,
                                             const double *tol,
                                             const int *onfly, int engine,
                                             int flags)
{
    return approximate_batch(nprob, matrices, formats, maxrank, tol, onfly,
                             engine, flags);
}

extern "C" int starsh_blrm__drsdd_b200(STARSH_blrm **matrix,
                                       STARSH_blrf *format, int maxrank,
                                       double tol, int onfly)
{
    return approximate(matrix, format, maxrank, tol, onfly, STARSH_B200_FP64,
                       STARSH_B200_HOST_MIRROR);
}

extern "C" int starsh_blrm__drsdd_b200_mp(STARSH_blrm **matrix,
                                          STARSH_blrf *format, int maxrank,
                                          double tol, int onfly)
{
    return approximate(matrix, format, maxrank, tol, onfly, STARSH_B200_MIXED,
                       STARSH_B200_HOST_MIRROR);
}

extern "C" int starsh_b200_blrm_download(STARSH_blrm *matrix)
{
    if (matrix == nullptr) return STARSH_WRONG_PARAMETER;
    Record *rec = find_record(matrix);
    if (rec == nullptr || rec->host_filled) return STARSH_SUCCESS;
    Context *ctx = context();
    if (!ctx) return STARSH_UNKNOWN_ERROR;
    std::lock_guard<std::mutex> guard(ctx->lock);
    return fill_host_mirror(matrix, *rec, ctx->stream);
}

extern "C" void starsh_b200_blrm_release(STARSH_blrm *matrix)
{
    Record *rec = nullptr;
    {
        std::lock_guard<std::mutex> g(g_rec_lock);
        auto it = g_records.find(matrix);
        if (it == g_records.end()) return;
        rec = it->second;
        g_records.erase(it);
    }
    // the factors may still be read by work on any stream (a device dmml
    // on the caller's stream): wait for the device, then free
    Context *ctx = context();
    if (ctx) cudaDeviceSynchronize();
    delete rec;
}

extern "C" void starsh_b200_blrm_host_release(const STARSH_blrm *matrix)
{
    std::vector<void *> owned;
    {
        std::lock_guard<std::mutex> g(g_mirror_mu);
        auto it = g_mirrors.find(matrix);
        if (it == g_mirrors.end()) return;
        owned = std::move(it->second);
        g_mirrors.erase(it);
    }
    for (void *p : owned) host_pinned_free(p);
}

extern "C" int starsh_b200_set_device(int device)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 ||
        device >= count) {
        cudaGetLastError();
        return STARSH_WRONG_PARAMETER;
    }
    if (g_ctx_ok && g_ctx.device != device) return STARSH_WRONG_PARAMETER;
    g_requested_device = device;
    return STARSH_SUCCESS;
}

extern "C" void *starsh_b200_stream(void)
{
    Context *ctx = context();
    return ctx ? (void *)ctx->stream : nullptr;
}

extern "C" int starsh_b200_get_stats(starsh_b200_stats *stats)
{
    if (stats == nullptr) return STARSH_WRONG_PARAMETER;
    *stats = thread_stats();
    return STARSH_SUCCESS;
}

extern "C" const char *starsh_b200_last_error(void)
{
    return t_error.c_str();
}

// Host-callable kernel entry points: the block is generated on the GPU from
// caller-given row and column index lists and copied back.
extern "C" void b200_eval_block_host(STARSH_kernel *kernel, int nrows,
                                     int ncols, STARSH_int *irow,
                                     STARSH_int *icol, void *row_data,
                                     void *col_data, double *result, int ld)
{
    if (nrows <= 0 || ncols <= 0) return;
    Context *ctx = context();
    if (!ctx) {
        fprintf(stderr, "STARSH B200: kernel called without a GPU\n");
        abort();
    }
    std::lock_guard<std::mutex> guard(ctx->lock);
    cudaStream_t s = ctx->stream;
    b200_kspec spec;
    const double *rp, *cp;
    STARSH_int rc, cc;
    if (b200_resolve_kernel(kernel, row_data, &spec, &rp, &rc, &cp, &cc,
                            col_data) != STARSH_SUCCESS) {
        fprintf(stderr, "STARSH B200: unrecognised kernel\n");
        abort();
    }
    DevicePoints dp;
    fill_kernel(dp.K, spec);
    int info = prepare_kernel_tables(dp, s);
    const void *d = nullptr;
    const size_t per = (size_t)spec.ndim * sizeof(double);
    if (!info) info = dp.upload(rp, rc * per, &d, s);
    dp.K.row_pt = (const double *)d;
    dp.K.row_count = rc;
    if (!info) info = dp.upload(cp, cc * per, &d, s);
    dp.K.col_pt = (const double *)d;
    dp.K.col_count = cc;
    if (!info) info = dp.upload(irow, nrows * sizeof(STARSH_int), &d, s);
    dp.K.row_piv = (const long long *)d;
    if (!info) info = dp.upload(icol, ncols * sizeof(STARSH_int), &d, s);
    dp.K.col_piv = (const long long *)d;
    double *out = nullptr;
    if (!info) {
        out = (double *)pool_alloc((size_t)nrows * ncols * sizeof(double), s);
        if (out == nullptr) info = STARSH_MALLOC_ERROR;
    }
    if (!info) {
        std::vector<BlockJob> jobs{BlockJob{0, 0, nrows, ncols, out}};
        info = gen_blocks(dp.K, jobs, s);
    }
    if (!info &&
        (cudaMemcpy2DAsync(result, (size_t)ld * sizeof(double), out,
                           (size_t)nrows * sizeof(double),
                           (size_t)nrows * sizeof(double), ncols,
                           cudaMemcpyDeviceToHost, s) != cudaSuccess ||
         cudaStreamSynchronize(s) != cudaSuccess))
        info = STARSH_UNKNOWN_ERROR;
    if (out) pool_free(out);
    if (info) {
        fprintf(stderr, "STARSH B200: block generation failed: %s\n",
                t_error.c_str());
        abort();
    }
}
