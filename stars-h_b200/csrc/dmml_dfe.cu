// TLR-by-dense product and Frobenius error on the device.
//
// dmml: B = alpha M A + beta B (reference src/backends/sequential/blrm/
// dmml.c:16-145).  Per far block T = V^T A[cols] (one batched GEMM), then
// every block row accumulates sum_b U_b T_b + sum_near D_b A[cols] in one
// segmented GEMM whose K loop walks the blocks of that row, so no two CTAs
// write the same rows and the sum order is fixed (deterministic).  For
// symm == 'S' the transposed contribution of every off-diagonal block is
// added to the mirrored block row, as the reference does (:78-87, :111-117).
//
// dfe: ||A - M||_F / ||A||_F with every block regenerated in FP64
// (reference src/backends/sequential/blrm/dfe.c:16-134); off-diagonal
// blocks of a symmetric format count twice.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "device_ctx.cuh"
#include "engine.cuh"
#include "records.cuh"
#include "starsh-b200.h"

namespace b200 {

// ------------------------------------------------------ segmented GEMM

struct SegOut {
    double *C;
    int ldc, M, N;
    int seg0, seg1;
};

struct Seg {
    const double *A;   // M x K (or K x M if transA), column-major
    const double *B;   // K x N
    int lda, ldb, K, transA;
};

__device__ __forceinline__ void dmma_884(double &c0, double &c1, double a,
                                         double b)
{
    asm volatile(
        "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 "
        "{%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}

// C += alpha * sum over segments of op(A_s) B_s.  CTA tile 64 x 64, same
// fragment mapping as the batched GEMM (8 warps, 32 x 16 per warp).  The
// K steps of 16 of all the CTA's segments form one sequence; operand tiles
// are double-buffered in shared memory and the next step (possibly of the
// next segment) is loaded into registers while the current one is
// multiplied.  Each output element accumulates in the same order as a
// plain loop over segments and steps.
__global__ void __launch_bounds__(256)
k_gemm_seg(const SegOut *__restrict__ outs, const Seg *__restrict__ segs,
           double alpha, int tiles_n)
{
    const SegOut o = outs[blockIdx.y];
    const int m0 = (blockIdx.x / tiles_n) * 64, n0 = (blockIdx.x % tiles_n) * 64;
    if (m0 >= o.M || n0 >= o.N || o.seg0 >= o.seg1) return;
    __shared__ double As[2][64 * 20];
    __shared__ double Bs[2][64 * 20];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
    double acc[4][2][2] = {};
    double ra[4], rb[4];
    auto load = [&](const Seg &sg, int k0) {
        #pragma unroll
        for (int r = 0; r < 4; ++r) {
            int row, kk;
            if (!sg.transA) { row = t & 63; kk = (t >> 6) + 4 * r; }
            else { kk = t & 15; row = (t >> 4) + 16 * r; }
            const int gm = m0 + row, gk = k0 + kk;
            double v = 0.0;
            if (gm < o.M && gk < sg.K)
                v = sg.transA ? sg.A[(size_t)gm * sg.lda + gk]
                              : sg.A[(size_t)gk * sg.lda + gm];
            ra[r] = v;
        }
        #pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int kk = t & 15, col = (t >> 4) + 16 * r;
            const int gn = n0 + col, gk = k0 + kk;
            rb[r] = (gn < o.N && gk < sg.K) ? sg.B[(size_t)gn * sg.ldb + gk] : 0.0;
        }
    };
    auto store = [&](const Seg &sg, int buf) {
        #pragma unroll
        for (int r = 0; r < 4; ++r) {
            int row, kk;
            if (!sg.transA) { row = t & 63; kk = (t >> 6) + 4 * r; }
            else { kk = t & 15; row = (t >> 4) + 16 * r; }
            As[buf][row * 20 + kk] = ra[r];
        }
        #pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int kk = t & 15, col = (t >> 4) + 16 * r;
            Bs[buf][col * 20 + kk] = rb[r];
        }
    };
    // the first step of a non-empty segment at or after s
    auto first_from = [&](int s, Seg &sg) {
        for (; s < o.seg1; ++s) {
            sg = segs[s];
            if (sg.K > 0) break;
        }
        return s;
    };
    Seg cur{};
    int sidx = first_from(o.seg0, cur), k0 = 0, buf = 0;
    if (sidx < o.seg1) {
        load(cur, 0);
        store(cur, 0);
    }
    __syncthreads();
    while (sidx < o.seg1) {
        // the next step: k0 + 16 of this segment, or the next segment's 0
        Seg nxt = cur;
        int nsidx = sidx, nk0 = k0 + 16;
        if (nk0 >= cur.K) {
            nsidx = first_from(sidx + 1, nxt);
            nk0 = 0;
        }
        const bool more = nsidx < o.seg1;
        if (more) load(nxt, nk0);
        #pragma unroll
        for (int kk = 0; kk < 16; kk += 4) {
            double af[4], bf[2];
            #pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = As[buf][(wm + 8 * i + g) * 20 + kk + tig];
            #pragma unroll
            for (int j = 0; j < 2; ++j) bf[j] = Bs[buf][(wn + 8 * j + g) * 20 + kk + tig];
            #pragma unroll
            for (int i = 0; i < 4; ++i)
                #pragma unroll
                for (int j = 0; j < 2; ++j)
                    dmma_884(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
        if (more) store(nxt, buf ^ 1);
        __syncthreads();
        buf ^= 1;
        sidx = nsidx;
        k0 = nk0;
        cur = nxt;
    }
    #pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + wm + 8 * i + g;
        if (gm >= o.M) continue;
        #pragma unroll
        for (int j = 0; j < 2; ++j)
            #pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gn = n0 + wn + 8 * j + 2 * tig + h;
                if (gn < o.N) o.C[(size_t)gn * o.ldc + gm] += alpha * acc[i][j][h];
            }
    }
}

__global__ void k_scale_cols(double *B, int ldb, int rows, int cols,
                             double beta)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)rows * cols) return;
    const int i = (int)(idx % rows), j = (int)(idx / rows);
    double *p = B + (size_t)j * ldb + i;
    *p = beta == 0.0 ? 0.0 : beta * *p;
}

// -------------------------------------------------- record for any blrm

// Matrices from another engine (or whose device copy was released) get
// their factors uploaded once and a record attached.
static int ensure_record(STARSH_blrm *M, Context &ctx, Record **out)
{
    Record *rec = find_record(M);
    if (rec) {
        *out = rec;
        return STARSH_SUCCESS;
    }
    STARSH_blrf *F = M->format;
    cudaStream_t s = ctx.stream;
    rec = new Record();
    rec->points = new DevicePoints();
    int info = upload_problem(*rec->points, F->problem, F->row_cluster,
                              F->col_cluster, s);
    if (info) {
        delete rec;
        return info;
    }
    size_t nu = 0, nv = 0, nd = 0;
    for (STARSH_int b = 0; b < F->nblocks_far; ++b) {
        nu += M->far_U[b]->size;
        nv += M->far_V[b]->size;
    }
    if (M->onfly == 0)
        for (STARSH_int b = 0; b < F->nblocks_near; ++b) nd += M->near_D[b]->size;
    double *chunk = nullptr;
    if (nu + nv + nd > 0) {
        chunk = (double *)pool_alloc((nu + nv + nd) * sizeof(double), s);
        if (chunk == nullptr) {
            delete rec;
            return cuda_fail(cudaErrorMemoryAllocation, "uploaded factors");
        }
        rec->chunks.push_back(chunk);
    }
    size_t ou = 0, ov = nu, od = nu + nv;
    rec->dU.resize(F->nblocks_far);
    rec->dV.resize(F->nblocks_far);
    for (STARSH_int b = 0; b < F->nblocks_far; ++b) {
        rec->dU[b] = chunk + ou;
        rec->dV[b] = chunk + ov;
        cudaMemcpyAsync(chunk + ou, M->far_U[b]->data,
                        M->far_U[b]->size * sizeof(double),
                        cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(chunk + ov, M->far_V[b]->data,
                        M->far_V[b]->size * sizeof(double),
                        cudaMemcpyHostToDevice, s);
        ou += M->far_U[b]->size;
        ov += M->far_V[b]->size;
    }
    rec->dD.assign(F->nblocks_near, nullptr);
    if (M->onfly == 0)
        for (STARSH_int b = 0; b < F->nblocks_near; ++b) {
            rec->dD[b] = chunk + od;
            cudaMemcpyAsync(chunk + od, M->near_D[b]->data,
                            M->near_D[b]->size * sizeof(double),
                            cudaMemcpyHostToDevice, s);
            od += M->near_D[b]->size;
        }
    rec->u_total = nu;
    rec->v_total = nv;
    rec->d_total = nd;
    rec->host_filled = true;
    add_record(M, rec);
    *out = rec;
    return STARSH_SUCCESS;
}

// ---------------------------------------------------------------- dmml

int dmml_device(STARSH_blrm *M, int nrhs, double alpha,
                const double *dA, int lda, double beta, double *dB,
                int ldb, cudaStream_t user_stream, Context &ctx)
{
    if (M == nullptr || nrhs < 0 || dA == nullptr || dB == nullptr)
        return STARSH_WRONG_PARAMETER;
    STARSH_blrf *F = M->format;
    STARSH_problem *P = F->problem;
    STARSH_cluster *R = F->row_cluster, *C = F->col_cluster;
    const STARSH_int nrows = P->shape[0];
    if (lda < P->shape[P->ndim - 1] || ldb < nrows)
        return STARSH_WRONG_PARAMETER;
    if (nrhs == 0) return STARSH_SUCCESS;
    Record *rec = nullptr;
    int info = ensure_record(M, ctx, &rec);
    if (info) return info;
    cudaStream_t s = ctx.stream;
    // Order the user's stream before ours and ours before the user's.
    cudaEvent_t ev;
    cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (user_stream != s) {
        cudaEventRecord(ev, user_stream);
        cudaStreamWaitEvent(s, ev, 0);
    }
    {
        const long long tot = (long long)nrows * nrhs;
        k_scale_cols<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(
            dB, ldb, (int)nrows, nrhs, beta);
        count_launch();
    }
    const bool symm = F->symm == 'S';
    // products: (output block row, U, V, m, n, r, input offset)
    struct Prod { STARSH_int brow; const double *U, *V; int m, n, r; STARSH_int in0; };
    std::vector<Prod> prods;
    for (STARSH_int b = 0; b < F->nblocks_far; ++b) {
        const int r = M->far_rank[b];
        if (r <= 0) continue;
        const STARSH_int i = F->block_far[2 * b], j = F->block_far[2 * b + 1];
        const int m = (int)R->size[i], n = (int)C->size[j];
        prods.push_back({i, rec->dU[b], rec->dV[b], m, n, r, C->start[j]});
        if (symm && i != j)
            prods.push_back({j, rec->dV[b], rec->dU[b], n, m, r, R->start[i]});
    }
    // near blocks: dense D (stored or regenerated when onfly)
    double *onfly_buf = nullptr;
    std::vector<const double *> nearD(F->nblocks_near, nullptr);
    if (F->nblocks_near > 0) {
        if (M->onfly) {
            size_t tot = 0;
            for (STARSH_int b = 0; b < F->nblocks_near; ++b)
                tot += (size_t)R->size[F->block_near[2 * b]] *
                       C->size[F->block_near[2 * b + 1]];
            cudaError_t e = cudaMallocAsync((void **)&onfly_buf,
                                            tot * sizeof(double), s);
            if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync(onfly)");
            std::vector<BlockJob> jobs;
            size_t off = 0;
            for (STARSH_int b = 0; b < F->nblocks_near; ++b) {
                const STARSH_int i = F->block_near[2 * b], j = F->block_near[2 * b + 1];
                BlockJob jb{R->start[i], C->start[j], (int)R->size[i],
                            (int)C->size[j], onfly_buf + off};
                nearD[b] = onfly_buf + off;
                off += (size_t)jb.m * jb.n;
                jobs.push_back(jb);
            }
            if ((info = gen_blocks(rec->points->K, jobs, s))) return info;
        } else {
            for (STARSH_int b = 0; b < F->nblocks_near; ++b) nearD[b] = rec->dD[b];
        }
    }
    // T buffer: per product r x nrhs (ld r)
    std::vector<size_t> toff(prods.size());
    size_t ttot = 0;
    for (size_t p = 0; p < prods.size(); ++p) {
        toff[p] = ttot;
        ttot += (size_t)prods[p].r * nrhs;
    }
    double *T = nullptr;
    if (ttot) {
        cudaError_t e = cudaMallocAsync((void **)&T, ttot * sizeof(double), s);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync(T)");
    }
    // Phase 1: T_p = V_p^T A[in0:in0+n, :]
    std::vector<GemmDesc> d1;
    int max_r = 0;
    for (size_t p = 0; p < prods.size(); ++p) {
        const Prod &q = prods[p];
        GemmDesc d;
        d.A = q.V; d.lda = q.n;
        d.B = dA + q.in0; d.ldb = lda;
        d.C = T + toff[p]; d.ldc = q.r;
        d.M = q.r; d.N = nrhs; d.K = q.n;
        d.alpha = 1.0; d.beta = 0.0;
        d1.push_back(d);
        max_r = std::max(max_r, q.r);
    }
    // Phase 2: per block row, segments over its products and near blocks.
    std::vector<std::vector<Seg>> rowsegs(F->nbrows);
    for (size_t p = 0; p < prods.size(); ++p) {
        const Prod &q = prods[p];
        rowsegs[q.brow].push_back(Seg{q.U, T + toff[p], q.m, q.r, q.r, 0});
    }
    for (STARSH_int b = 0; b < F->nblocks_near; ++b) {
        const STARSH_int i = F->block_near[2 * b], j = F->block_near[2 * b + 1];
        const int m = (int)R->size[i], n = (int)C->size[j];
        rowsegs[i].push_back(Seg{nearD[b], dA + C->start[j], m, lda, n, 0});
        if (symm && i != j)
            rowsegs[j].push_back(Seg{nearD[b], dA + R->start[i], m, lda, m, 1});
    }
    std::vector<SegOut> outs;
    std::vector<Seg> segs;
    int max_m = 0;
    for (STARSH_int i = 0; i < F->nbrows; ++i) {
        if (rowsegs[i].empty()) continue;
        SegOut o;
        o.C = dB + R->start[i];
        o.ldc = ldb;
        o.M = (int)R->size[i];
        o.N = nrhs;
        o.seg0 = (int)segs.size();
        segs.insert(segs.end(), rowsegs[i].begin(), rowsegs[i].end());
        o.seg1 = (int)segs.size();
        outs.push_back(o);
        max_m = std::max(max_m, o.M);
    }
    // Upload descriptor arrays in one allocation.
    const size_t b1 = d1.size() * sizeof(GemmDesc);
    const size_t b2 = outs.size() * sizeof(SegOut);
    const size_t b3 = segs.size() * sizeof(Seg);
    char *dbuf = nullptr;
    if (b1 + b2 + b3) {
        cudaError_t e = cudaMallocAsync((void **)&dbuf, b1 + b2 + b3 + 64, s);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync(desc)");
        std::vector<char> hbuf(b1 + b2 + b3);
        memcpy(hbuf.data(), d1.data(), b1);
        memcpy(hbuf.data() + b1, outs.data(), b2);
        memcpy(hbuf.data() + b1 + b2, segs.data(), b3);
        cudaMemcpyAsync(dbuf, hbuf.data(), hbuf.size(), cudaMemcpyHostToDevice, s);
    }
    if (!d1.empty()) {
        gemm_f64_batched(true, false, (const GemmDesc *)dbuf, (int)d1.size(),
                         max_r, nrhs, s);
        count_launch();
    }
    if (!outs.empty()) {
        const int tiles_n = (nrhs + 63) / 64;
        const int tiles_m = (max_m + 63) / 64;
        for (size_t o0 = 0; o0 < outs.size(); o0 += 65535) {
            const unsigned no = (unsigned)std::min<size_t>(65535, outs.size() - o0);
            dim3 grid(tiles_m * tiles_n, no);
            k_gemm_seg<<<grid, 256, 0, s>>>(
                (const SegOut *)(dbuf + b1) + o0, (const Seg *)(dbuf + b1 + b2),
                alpha, tiles_n);
            count_launch();
        }
    }
    if (dbuf) cudaFreeAsync(dbuf, s);
    if (T) cudaFreeAsync(T, s);
    if (onfly_buf) cudaFreeAsync(onfly_buf, s);
    cudaError_t e = cudaGetLastError();
    if (user_stream != s) {
        cudaEventRecord(ev, s);
        cudaStreamWaitEvent(user_stream, ev, 0);
    }
    cudaEventDestroy(ev);
    if (e != cudaSuccess) return cuda_fail(e, "dmml kernels");
    return STARSH_SUCCESS;
}

// ----------------------------------------------------------------- dfe

struct DfeJob {
    long long row0, col0;
    int m, n, r;
    const double *U, *V, *D;   // D: stored dense block or null
};

// Each CTA stores its 64 x 64 piece's ||D||^2 and ||D - U V^T||^2 in its own
// slot of `part` (slot = (job, tile row, tile column)); k_dfe_sum adds a
// job's slots in a fixed order, so the error is the same on every run.
__global__ void __launch_bounds__(256)
k_dfe(DevKernel K, const DfeJob *__restrict__ jobs, double *__restrict__ part)
{
    const DfeJob jb = jobs[blockIdx.z];
    const int i0 = blockIdx.x * 64, j0 = blockIdx.y * 64;
    double *slot = part + 2 * (((size_t)blockIdx.z * gridDim.y + blockIdx.y) *
                               gridDim.x + blockIdx.x);
    if (i0 >= jb.m || j0 >= jb.n) {
        if (threadIdx.x == 0) slot[0] = slot[1] = 0.0;
        return;
    }
    __shared__ double Us[64][33];
    __shared__ double Vs[64][33];
    __shared__ double red[2][8];
    const int t = threadIdx.x;
    const int ii = t & 63, jj = t >> 6;
    double acc[16] = {};
    for (int p0 = 0; p0 < jb.r; p0 += 32) {
        for (int q = t; q < 64 * 32; q += 256) {
            const int row = q & 63, p = q >> 6;
            const bool okp = p0 + p < jb.r;
            Us[row][p] = (okp && i0 + row < jb.m)
                             ? jb.U[(size_t)(p0 + p) * jb.m + i0 + row] : 0.0;
            Vs[row][p] = (okp && j0 + row < jb.n)
                             ? jb.V[(size_t)(p0 + p) * jb.n + j0 + row] : 0.0;
        }
        __syncthreads();
        #pragma unroll 4
        for (int p = 0; p < 32; ++p) {
            const double u = Us[ii][p];
            #pragma unroll
            for (int c = 0; c < 16; ++c) acc[c] += u * Vs[jj + 4 * c][p];
        }
        __syncthreads();
    }
    double nrm = 0.0, dif = 0.0;
    const int i = i0 + ii;
    if (i < jb.m) {
        for (int c = 0; c < 16; ++c) {
            const int j = j0 + jj + 4 * c;
            if (j >= jb.n) continue;
            const double d = jb.D ? jb.D[(size_t)j * jb.m + i]
                                  : block_entry(K, jb.row0, jb.col0, i, j);
            const double e = d - acc[c];
            nrm += d * d;
            dif += e * e;
        }
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nrm += __shfl_down_sync(0xffffffffu, nrm, o);
        dif += __shfl_down_sync(0xffffffffu, dif, o);
    }
    if ((t & 31) == 0) {
        red[0][t >> 5] = nrm;
        red[1][t >> 5] = dif;
    }
    __syncthreads();
    if (t == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < 8; ++w) {
            a += red[0][w];
            b += red[1][w];
        }
        slot[0] = a;
        slot[1] = b;
    }
}

// out[2 job + {0, 1}] = the sums of the job's nslot slots, in slot order.
__global__ void k_dfe_sum(const double *__restrict__ part, int nslot,
                          long long njobs, double *__restrict__ out)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const double *p = part + 2 * (size_t)j * nslot;
    double a = 0.0, b = 0.0;
    for (int q = 0; q < nslot; ++q) {
        a += p[2 * q];
        b += p[2 * q + 1];
    }
    out[2 * j] = a;
    out[2 * j + 1] = b;
}

// The weighted sums sum ||D_b - U_b V_b^T||_F^2 (far blocks) and
// sum ||D_b||_F^2 (all blocks) of M; returns STARSH_SUCCESS or an error.
static int dfe_sums_device(STARSH_blrm *M, Context &ctx, double *diff2,
                           double *norm2)
{
    *diff2 = *norm2 = 0.0;
    Record *rec = nullptr;
    if (ensure_record(M, ctx, &rec)) return STARSH_UNKNOWN_ERROR;
    STARSH_blrf *F = M->format;
    STARSH_cluster *R = F->row_cluster, *C = F->col_cluster;
    cudaStream_t s = ctx.stream;
    const STARSH_int nf = F->nblocks_far, nn = F->nblocks_near;
    const size_t njobs = nf + nn;
    if (njobs == 0) return STARSH_SUCCESS;
    std::vector<DfeJob> jobs(njobs);
    int mmax = 0, nmax = 0;
    for (STARSH_int b = 0; b < nf; ++b) {
        const STARSH_int i = F->block_far[2 * b], j = F->block_far[2 * b + 1];
        jobs[b] = DfeJob{R->start[i], C->start[j], (int)R->size[i],
                         (int)C->size[j], M->far_rank[b], rec->dU[b],
                         rec->dV[b], nullptr};
    }
    for (STARSH_int b = 0; b < nn; ++b) {
        const STARSH_int i = F->block_near[2 * b], j = F->block_near[2 * b + 1];
        jobs[nf + b] = DfeJob{R->start[i], C->start[j], (int)R->size[i],
                              (int)C->size[j], 0, nullptr, nullptr,
                              M->onfly ? nullptr : rec->dD[b]};
    }
    for (const auto &j : jobs) {
        mmax = std::max(mmax, j.m);
        nmax = std::max(nmax, j.n);
    }
    const int gx = (mmax + 63) / 64, gy = (nmax + 63) / 64;
    const size_t nslot = (size_t)gx * gy;
    double *sums = (double *)pool_alloc(2 * njobs * sizeof(double), s);
    double *part = (double *)pool_alloc(2 * njobs * nslot * sizeof(double), s);
    DfeJob *dj = (DfeJob *)pool_alloc(njobs * sizeof(DfeJob), s);
    if (!sums || !part || !dj) {
        pool_free(sums);
        pool_free(part);
        pool_free(dj);
        return cuda_fail(cudaErrorMemoryAllocation, "dfe buffers");
    }
    cudaMemcpyAsync(dj, jobs.data(), njobs * sizeof(DfeJob),
                    cudaMemcpyHostToDevice, s);
    for (size_t b0 = 0; b0 < njobs; b0 += 65535) {
        const unsigned nb = (unsigned)std::min<size_t>(65535, njobs - b0);
        dim3 grid(gx, gy, nb);
        k_dfe<<<grid, 256, 0, s>>>(rec->points->K, dj + b0,
                                   part + 2 * b0 * nslot);
        count_launch();
    }
    k_dfe_sum<<<(unsigned)((njobs + 255) / 256), 256, 0, s>>>(
        part, (int)nslot, (long long)njobs, sums);
    count_launch();
    std::vector<double> h(2 * njobs);
    cudaMemcpyAsync(h.data(), sums, 2 * njobs * sizeof(double),
                    cudaMemcpyDeviceToHost, s);
    pool_free(sums);
    pool_free(part);
    pool_free(dj);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "dfe kernels");
    double diff = 0.0, norm = 0.0;
    const bool symm = F->symm == 'S';
    for (STARSH_int b = 0; b < nf; ++b) {
        const double w = (symm && F->block_far[2 * b] != F->block_far[2 * b + 1]) ? 2.0 : 1.0;
        norm += w * h[2 * b];
        diff += w * h[2 * b + 1];
    }
    for (STARSH_int b = 0; b < nn; ++b) {
        const double w = (symm && F->block_near[2 * b] != F->block_near[2 * b + 1]) ? 2.0 : 1.0;
        norm += w * h[2 * (nf + b)];
    }
    *diff2 = diff;
    *norm2 = norm;
    return STARSH_SUCCESS;
}

static double dfe_device(STARSH_blrm *M, Context &ctx)
{
    double diff = 0.0, norm = 0.0;
    if (dfe_sums_device(M, ctx, &diff, &norm) != STARSH_SUCCESS) return -1.0;
    return norm > 0.0 ? sqrt(diff) / sqrt(norm) : 0.0;
}

}  // namespace b200

using namespace b200;

extern "C" int starsh_b200_blrm_dmml_device(STARSH_blrm *matrix, int nrhs,
                                            double alpha, const double *dA,
                                            int lda, double beta, double *dB,
                                            int ldb, void *stream)
{
    Context *ctx = context();
    if (!ctx) return STARSH_UNKNOWN_ERROR;
    std::lock_guard<std::mutex> guard(ctx->lock);
    return dmml_device(matrix, nrhs, alpha, dA, lda, beta, dB, ldb,
                       stream ? (cudaStream_t)stream : ctx->stream, *ctx);
}

extern "C" int starsh_blrm__dmml_b200(STARSH_blrm *matrix, int nrhs,
                                      double alpha, double *A, int lda,
                                      double beta, double *B, int ldb)
{
    if (matrix == nullptr || A == nullptr || B == nullptr || nrhs < 0)
        return STARSH_WRONG_PARAMETER;
    Context *ctx = context();
    if (!ctx) return STARSH_UNKNOWN_ERROR;
    std::lock_guard<std::mutex> guard(ctx->lock);
    STARSH_problem *P = matrix->format->problem;
    const size_t nr = P->shape[0], nc = P->shape[P->ndim - 1];
    if (lda < (int)nc || ldb < (int)nr) return STARSH_WRONG_PARAMETER;
    cudaStream_t s = ctx->stream;
    double *dA = nullptr, *dB = nullptr;
    if (cudaMallocAsync((void **)&dA, nc * nrhs * sizeof(double) + 8, s) ||
        cudaMallocAsync((void **)&dB, nr * nrhs * sizeof(double) + 8, s))
        return cuda_fail(cudaGetLastError(), "cudaMallocAsync(dmml)");
    cudaMemcpy2DAsync(dA, nc * sizeof(double), A, (size_t)lda * sizeof(double),
                      nc * sizeof(double), nrhs, cudaMemcpyHostToDevice, s);
    if (beta != 0.0)
        cudaMemcpy2DAsync(dB, nr * sizeof(double), B,
                          (size_t)ldb * sizeof(double), nr * sizeof(double),
                          nrhs, cudaMemcpyHostToDevice, s);
    int info = dmml_device(matrix, nrhs, alpha, dA, (int)nc, beta, dB,
                           (int)nr, s, *ctx);
    if (!info)
        cudaMemcpy2DAsync(B, (size_t)ldb * sizeof(double), dB,
                          nr * sizeof(double), nr * sizeof(double), nrhs,
                          cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(dA, s);
    cudaFreeAsync(dB, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (!info && e != cudaSuccess) info = cuda_fail(e, "dmml");
    return info;
}

extern "C" int starsh_blrm__dmml(STARSH_blrm *matrix, int nrhs, double alpha,
                                 double *A, int lda, double beta, double *B,
                                 int ldb)
{
    return starsh_blrm__dmml_b200(matrix, nrhs, alpha, A, lda, beta, B, ldb);
}

extern "C" double starsh_blrm__dfe_b200(STARSH_blrm *matrix)
{
    if (matrix == nullptr) return -1.0;
    Context *ctx = context();
    if (!ctx) return -1.0;
    std::lock_guard<std::mutex> guard(ctx->lock);
    return dfe_device(matrix, *ctx);
}

extern "C" double starsh_blrm__dfe(STARSH_blrm *matrix)
{
    return starsh_blrm__dfe_b200(matrix);
}

extern "C" int starsh_b200_blrm_dfe_sums(STARSH_blrm *matrix, double *diff2,
                                         double *norm2)
{
    if (matrix == nullptr || diff2 == nullptr || norm2 == nullptr)
        return STARSH_WRONG_PARAMETER;
    Context *ctx = context();
    if (!ctx) return STARSH_UNKNOWN_ERROR;
    std::lock_guard<std::mutex> guard(ctx->lock);
    return dfe_sums_device(matrix, *ctx, diff2, norm2);
}
