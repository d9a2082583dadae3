// TLR-by-dense product and Frobenius error on the device.
//
// dmml: B = alpha M A + beta B (reference src/backends/sequential/blrm/
// dmml.c:16-145: per far block T = V^T A[cols], B[rows] += U T, near
// blocks dense).  Here every T of one input block column comes from one
// GEMM over the concatenated right factors, and every block row
// accumulates sum_b U_b T_b + sum_near D_b A[cols] in one GEMM whose K runs
// over the row's concatenated left factors and near blocks, so no two CTAs
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
#include <mutex>
#include <vector>

#include "device_ctx.cuh"
#include "engine.cuh"
#include "records.cuh"
#include "starsh-b200.h"

namespace b200 {

__device__ __forceinline__ void dmma_884(double &c0, double &c1, double a,
                                         double b)
{
    asm volatile(
        "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 "
        "{%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}

// ------------------------------------------------------ product kernels
//
// B = alpha M A as two long GEMMs instead of one small GEMM per block.
// Phase 1, per input block column j: the rows of T are the columns of all
// right factors V_p that multiply A_j (far block p, or its mirror in a
// symmetric format), T(rho, :) = V_p(:, c)^T A_j -- M runs over the
// concatenated factor columns, K over the block column's rows.  Phase 2,
// per output block row i: B_i += [U_p1 U_p2 ...] [T_p1; T_p2; ...] +
// sum_near op(D_b) A_j -- K runs over the concatenated left-factor columns
// of the row, then over the near blocks' columns.  T is written by phase 1
// straight into the row-ordered layout phase 2 reads: block row i's rows
// of T form one column-major (S_i x nrhs) matrix, S_i = sum of the row's
// ranks.  Each output element is written by one CTA, its sum in a fixed
// order (deterministic).
//
// CTA tile 128 x BN (BN = 16 FN), 8 warps as 4 (m) x 2 (n), warp tile
// 32 x 8 FN of FP64 mma.sync m8n8k4; K steps of 16 through a three-stage
// cp.async pipeline.  Shared-memory layouts are chosen so that the
// fragment reads and the copies are free of bank conflicts: B as [n][k]
// (row stride 20 doubles); A as [m][k] (stride 20) in phase 1, whose
// operand is contiguous along k in global memory, and as [k][m] (stride
// 132) in phase 2, whose operand is contiguous along m.

struct RowT {          // where phase 1 writes row rho of T
    long long base;    // first T row of the output block row (P_i)
    int kappa;         // row within the block row's T_i
    int ld;            // rows of T_i (S_i)
};

struct Job1 {          // phase 1: up to 128 rows of T that share A_j
    int rho0, rows;
    int K;             // rows of A_j
    long long in0;     // first row of A_j in A
};

struct NearPiece {
    int block;         // near block (its D pointer is given per call)
    int trans;         // 1: the mirrored block of a symmetric format
    int K;             // columns of op(D)
    int ld;            // leading dimension of D
    long long in0;     // first row of the input block in A
};

struct Job2 {          // phase 2: up to 128 rows of one output block row
    long long out0;    // first output row
    int m0, rows;      // rows m0 .. m0 + rows - 1 of the block row
    long long kap0;    // P_i (first concatenated column of the row)
    int kfar;          // S_i
    int near0, near1;  // the row's near pieces
};

constexpr int kPBM = 128, kPBK = 16, kPStages = 3;
constexpr int kPAStage = 2560;   // >= 128 * 20 (phase 1), 16 * 132 (phase 2)

template <int FN>
constexpr int prod_stage_doubles() { return kPAStage + 20 * 16 * FN; }

__device__ __forceinline__ void cp_async8(double *dst, const double *src,
                                          bool ok)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d),
                 "l"(src), "r"(ok ? 8 : 0));
}

__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;\n" ::);
}

__device__ __forceinline__ void cp_async_wait_stages()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kPStages - 2));
}

// acc += A_stage B_stage for one K step (A_KMAJOR: A stored as [k][m]).
template <int FN, bool A_KMAJOR>
__device__ __forceinline__ void prod_step(const double *As, const double *Bs,
                                          double (&acc)[4][FN][2], int wm,
                                          int wn, int g, int tig)
{
    #pragma unroll
    for (int kk = 0; kk < kPBK; kk += 4) {
        double af[4], bf[FN];
        #pragma unroll
        for (int i = 0; i < 4; ++i)
            af[i] = A_KMAJOR ? As[(kk + tig) * 132 + wm + 8 * i + g]
                             : As[(wm + 8 * i + g) * 20 + kk + tig];
        #pragma unroll
        for (int j = 0; j < FN; ++j) bf[j] = Bs[(wn + 8 * j + g) * 20 + kk + tig];
        #pragma unroll
        for (int i = 0; i < 4; ++i)
            #pragma unroll
            for (int j = 0; j < FN; ++j)
                dmma_884(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
}

// Phase 1: T rows of one job (rows rho0 .. rho0 + rows - 1), columns
// n0 .. n0 + BN - 1 of the right-hand sides.
template <int FN>
__global__ void __launch_bounds__(256, 2)
k_prod_t(const Job1 *__restrict__ jobs, const double *const *__restrict__ vcol,
         const RowT *__restrict__ rowt, const double *__restrict__ A, int lda,
         double *__restrict__ T, int nrhs)
{
    constexpr int BN = 16 * FN;
    constexpr int STAGE = prod_stage_doubles<FN>();
    extern __shared__ double sm[];
    __shared__ const double *rowp[kPBM];
    const Job1 jb = jobs[blockIdx.x];
    const int n0 = blockIdx.y * BN;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = (warp & 3) * 32, wn = (warp >> 2) * 8 * FN;
    for (int r = t; r < kPBM; r += 256)
        rowp[r] = r < jb.rows ? vcol[jb.rho0 + r] : nullptr;
    __syncthreads();
    const int lk = t & 15, lr = t >> 4;
    const double *Aj = A + jb.in0;
    const int steps = (jb.K + kPBK - 1) / kPBK;
    auto issue = [&](int step, int st) {
        double *As = sm + st * STAGE, *Bs = As + kPAStage;
        const int k = step * kPBK + lk;
        const bool kin = k < jb.K;
        #pragma unroll
        for (int q = 0; q < 8; ++q) {
            const double *p = rowp[lr + 16 * q];
            const bool ok = kin && p != nullptr;
            cp_async8(As + (lr + 16 * q) * 20 + lk, ok ? p + k : A, ok);
        }
        #pragma unroll
        for (int q = 0; q < FN; ++q) {
            const int col = n0 + lr + 16 * q;
            const bool ok = kin && col < nrhs;
            cp_async8(Bs + (lr + 16 * q) * 20 + lk,
                      ok ? Aj + k + (size_t)col * lda : A, ok);
        }
    };
    double acc[4][FN][2] = {};
    #pragma unroll
    for (int s = 0; s < kPStages - 1; ++s) {
        if (s < steps) issue(s, s);
        cp_async_commit();
    }
    for (int s = 0; s < steps; ++s) {
        cp_async_wait_stages();
        __syncthreads();
        if (s + kPStages - 1 < steps)
            issue(s + kPStages - 1, (s + kPStages - 1) % kPStages);
        cp_async_commit();
        const double *As = sm + (s % kPStages) * STAGE;
        prod_step<FN, false>(As, As + kPAStage, acc, wm, wn, g, tig);
    }
    #pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = wm + 8 * i + g;
        if (r >= jb.rows) continue;
        const RowT rt = rowt[jb.rho0 + r];
        double *out = T + (size_t)nrhs * rt.base + rt.kappa;
        #pragma unroll
        for (int j = 0; j < FN; ++j)
            #pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int col = n0 + wn + 8 * j + 2 * tig + h;
                if (col < nrhs) out[(size_t)col * rt.ld] = acc[i][j][h];
            }
    }
}

// Phase 2: rows m0 .. m0 + rows - 1 of one output block row.
template <int FN>
__global__ void __launch_bounds__(256, 2)
k_prod_b(const Job2 *__restrict__ jobs, const double *const *__restrict__ ucol,
         const double *__restrict__ T, int nrhs,
         const NearPiece *__restrict__ near, const double *const *__restrict__ nearD,
         const double *__restrict__ A, int lda, double *__restrict__ B, int ldb,
         double alpha)
{
    constexpr int BN = 16 * FN;
    constexpr int STAGE = prod_stage_doubles<FN>();
    extern __shared__ double sm[];
    const Job2 jb = jobs[blockIdx.x];
    const int n0 = blockIdx.y * BN;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = (warp & 3) * 32, wn = (warp >> 2) * 8 * FN;
    // A copies: rows am, am + 64 and columns ak + 4 q (q < 4) of the step;
    // B copies: column lk of the step, right-hand sides lr + 16 q
    const int am = t & 63, ak = t >> 6;
    const int lk = t & 15, lr = t >> 4;
    const double *Tf = T + (size_t)nrhs * jb.kap0;
    int total = (jb.kfar + kPBK - 1) / kPBK;
    for (int q = jb.near0; q < jb.near1; ++q) total += (near[q].K + kPBK - 1) / kPBK;
    // issue position: piece (-1: the factors, else a near piece) and k0
    int piece = jb.kfar > 0 ? -1 : jb.near0, k0 = 0;
    const double *up[4];            // factor columns of the next far step
    auto fetch_ptrs = [&]() {
        #pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int kap = k0 + ak + 4 * q;
            up[q] = piece < 0 && kap < jb.kfar ? ucol[jb.kap0 + kap] : nullptr;
        }
    };
    auto advance = [&]() {
        k0 += kPBK;
        const int K = piece < 0 ? jb.kfar : near[piece].K;
        if (k0 >= K) {
            piece = piece < 0 ? jb.near0 : piece + 1;
            k0 = 0;
        }
        fetch_ptrs();
    };
    auto issue = [&](int st) {
        double *As = sm + st * STAGE, *Bs = As + kPAStage;
        if (piece < 0) {
            #pragma unroll
            for (int q = 0; q < 4; ++q)
                #pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int m = am + 64 * h;
                    const bool ok = up[q] != nullptr && m < jb.rows;
                    cp_async8(As + (ak + 4 * q) * 132 + m,
                              ok ? up[q] + jb.m0 + m : A, ok);
                }
            #pragma unroll
            for (int q = 0; q < FN; ++q) {
                const int col = n0 + lr + 16 * q, kap = k0 + lk;
                const bool ok = kap < jb.kfar && col < nrhs;
                cp_async8(Bs + (lr + 16 * q) * 20 + lk,
                          ok ? Tf + kap + (size_t)col * jb.kfar : A, ok);
            }
        } else {
            const NearPiece np = near[piece];
            const double *D = nearD[np.block];
            #pragma unroll
            for (int q = 0; q < 4; ++q)
                #pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int m = am + 64 * h, kap = k0 + ak + 4 * q;
                    const bool ok = kap < np.K && m < jb.rows;
                    const size_t off = np.trans
                        ? (size_t)kap + (size_t)(jb.m0 + m) * np.ld
                        : (size_t)(jb.m0 + m) + (size_t)kap * np.ld;
                    cp_async8(As + (ak + 4 * q) * 132 + m, ok ? D + off : A, ok);
                }
            #pragma unroll
            for (int q = 0; q < FN; ++q) {
                const int col = n0 + lr + 16 * q, kap = k0 + lk;
                const bool ok = kap < np.K && col < nrhs;
                cp_async8(Bs + (lr + 16 * q) * 20 + lk,
                          ok ? A + np.in0 + kap + (size_t)col * lda : A, ok);
            }
        }
    };
    fetch_ptrs();
    double acc[4][FN][2] = {};
    #pragma unroll
    for (int s = 0; s < kPStages - 1; ++s) {
        if (s < total) {
            issue(s);
            advance();
        }
        cp_async_commit();
    }
    for (int s = 0; s < total; ++s) {
        cp_async_wait_stages();
        __syncthreads();
        if (s + kPStages - 1 < total) {
            issue((s + kPStages - 1) % kPStages);
            advance();
        }
        cp_async_commit();
        const double *As = sm + (s % kPStages) * STAGE;
        prod_step<FN, true>(As, As + kPAStage, acc, wm, wn, g, tig);
    }
    #pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = wm + 8 * i + g;
        if (m >= jb.rows) continue;
        double *out = B + jb.out0 + m;
        #pragma unroll
        for (int j = 0; j < FN; ++j)
            #pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int col = n0 + wn + 8 * j + 2 * tig + h;
                if (col < nrhs) out[(size_t)col * ldb] += alpha * acc[i][j][h];
            }
    }
}

template <int FN>
static void launch_products(const Job1 *j1, int n1, const double *const *vcol,
                            const RowT *rowt, const Job2 *j2, int n2,
                            const double *const *ucol, const NearPiece *near,
                            const double *const *nearD, const double *A, int lda,
                            double *T, double *B, int ldb, int nrhs, double alpha,
                            cudaStream_t s)
{
    constexpr size_t smem = (size_t)kPStages * prod_stage_doubles<FN>() * sizeof(double);
    static std::once_flag attr;
    std::call_once(attr, [] {
        cudaFuncSetAttribute(k_prod_t<FN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        cudaFuncSetAttribute(k_prod_b<FN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    });
    const unsigned ny = (unsigned)((nrhs + 16 * FN - 1) / (16 * FN));
    if (n1 > 0) {
        k_prod_t<FN><<<dim3((unsigned)n1, ny), 256, smem, s>>>(j1, vcol, rowt, A,
                                                              lda, T, nrhs);
        count_launch();
    }
    if (n2 > 0) {
        k_prod_b<FN><<<dim3((unsigned)n2, ny), 256, smem, s>>>(
            j2, ucol, T, nrhs, near, nearD, A, lda, B, ldb, alpha);
        count_launch();
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

// The product plan of a matrix (device arrays, built on its first product
// and kept with its record): phase-1 jobs with their factor-column
// pointers and T destinations, phase-2 jobs with the concatenated
// left-factor columns of every block row and the near pieces.
struct ProductPlan {
    void *dev = nullptr;
    const double **vcol = nullptr;
    RowT *rowt = nullptr;
    const double **ucol = nullptr;
    Job1 *j1 = nullptr;
    Job2 *j2 = nullptr;
    NearPiece *near = nullptr;
    int n1 = 0, n2 = 0, nnear = 0;
    long long trows = 0;       // rows of T over all block rows
    cudaEvent_t ready = nullptr;   // the upload has completed
    ~ProductPlan()
    {
        if (ready) cudaEventDestroy(ready);
        if (dev) pool_free(dev);
    }
};

template <class T>
static size_t put(std::vector<char> &buf, const std::vector<T> &v)
{
    const size_t off = (buf.size() + 255) / 256 * 256;
    buf.resize(off + v.size() * sizeof(T));
    if (!v.empty()) memcpy(buf.data() + off, v.data(), v.size() * sizeof(T));
    return off;
}

static int build_plan(STARSH_blrm *M, const Record &rec, cudaStream_t s,
                      ProductPlan **out)
{
    STARSH_blrf *F = M->format;
    STARSH_cluster *R = F->row_cluster, *C = F->col_cluster;
    const bool symm = F->symm == 'S';
    // products: output block row, input block (of the column clustering,
    // or of the row clustering for a mirrored block), factors, sizes
    struct Prod { STARSH_int orow, icol; const double *U, *V; int m, n, r; long long in0; };
    std::vector<Prod> prods;
    for (STARSH_int b = 0; b < F->nblocks_far; ++b) {
        const int r = M->far_rank[b];
        if (r <= 0) continue;
        const STARSH_int i = F->block_far[2 * b], j = F->block_far[2 * b + 1];
        const int m = (int)R->size[i], n = (int)C->size[j];
        prods.push_back({i, j, rec.dU[b], rec.dV[b], m, n, r, (long long)C->start[j]});
        if (symm && i != j)
            prods.push_back({j, i, rec.dV[b], rec.dU[b], n, m, r, (long long)R->start[i]});
    }
    const STARSH_int nbr = F->nbrows, nbc = std::max(F->nbrows, F->nbcols);
    // phase 2 layout: per output row its products in list order
    std::vector<long long> P(nbr + 1, 0);
    std::vector<int> S(nbr, 0);
    std::vector<int> kap(prods.size());
    for (size_t p = 0; p < prods.size(); ++p) {
        kap[p] = S[prods[p].orow];
        S[prods[p].orow] += prods[p].r;
    }
    for (STARSH_int i = 0; i < nbr; ++i) P[i + 1] = P[i] + S[i];
    const long long trows = P[nbr];
    std::vector<const double *> ucol(trows);
    for (size_t p = 0; p < prods.size(); ++p) {
        const Prod &q = prods[p];
        for (int c = 0; c < q.r; ++c)
            ucol[P[q.orow] + kap[p] + c] = q.U + (size_t)c * q.m;
    }
    // phase 1: products grouped by input block, list order within a group
    std::vector<std::vector<int>> bycol(nbc);
    for (size_t p = 0; p < prods.size(); ++p) bycol[prods[p].icol].push_back((int)p);
    std::vector<const double *> vcol;
    std::vector<RowT> rowt;
    std::vector<Job1> j1;
    vcol.reserve(trows);
    rowt.reserve(trows);
    for (STARSH_int j = 0; j < nbc; ++j) {
        if (bycol[j].empty()) continue;
        const int rho0 = (int)vcol.size();
        for (int p : bycol[j]) {
            const Prod &q = prods[p];
            for (int c = 0; c < q.r; ++c) {
                vcol.push_back(q.V + (size_t)c * q.n);
                rowt.push_back(RowT{P[q.orow], kap[p] + c, S[q.orow]});
            }
        }
        const int cnt = (int)vcol.size() - rho0;
        const Prod &q0 = prods[bycol[j][0]];
        for (int r0 = 0; r0 < cnt; r0 += kPBM)
            j1.push_back(Job1{rho0 + r0, std::min(kPBM, cnt - r0), q0.n, q0.in0});
    }
    // near pieces per output row, in near-block order
    std::vector<std::vector<NearPiece>> rownear(nbr);
    for (STARSH_int b = 0; b < F->nblocks_near; ++b) {
        const STARSH_int i = F->block_near[2 * b], j = F->block_near[2 * b + 1];
        const int m = (int)R->size[i], n = (int)C->size[j];
        rownear[i].push_back(NearPiece{(int)b, 0, n, m, (long long)C->start[j]});
        if (symm && i != j)
            rownear[j].push_back(NearPiece{(int)b, 1, m, m, (long long)R->start[i]});
    }
    std::vector<NearPiece> near;
    std::vector<Job2> j2;
    for (STARSH_int i = 0; i < nbr; ++i) {
        if (S[i] == 0 && rownear[i].empty()) continue;
        const int near0 = (int)near.size();
        near.insert(near.end(), rownear[i].begin(), rownear[i].end());
        const int mi = (int)R->size[i];
        for (int m0 = 0; m0 < mi; m0 += kPBM)
            j2.push_back(Job2{(long long)R->start[i] + m0, m0, std::min(kPBM, mi - m0),
                              P[i], S[i], near0, (int)near.size()});
    }
    // one device allocation for every array
    std::vector<char> buf;
    const size_t o_vcol = put(buf, vcol), o_rowt = put(buf, rowt),
                 o_ucol = put(buf, ucol), o_j1 = put(buf, j1), o_j2 = put(buf, j2),
                 o_near = put(buf, near);
    auto *plan = new ProductPlan();
    if (!buf.empty()) {
        char *d = (char *)pool_alloc(buf.size(), s);
        if (d == nullptr) {
            delete plan;
            return cuda_fail(cudaErrorMemoryAllocation, "product plan");
        }
        plan->dev = d;
        const cudaError_t e = cudaMemcpyAsync(d, buf.data(), buf.size(),
                                              cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
            delete plan;
            return cuda_fail(e, "product plan upload");
        }
        plan->vcol = (const double **)(d + o_vcol);
        plan->rowt = (RowT *)(d + o_rowt);
        plan->ucol = (const double **)(d + o_ucol);
        plan->j1 = (Job1 *)(d + o_j1);
        plan->j2 = (Job2 *)(d + o_j2);
        plan->near = (NearPiece *)(d + o_near);
        // products on any stream wait for the upload
        if (cudaEventCreateWithFlags(&plan->ready, cudaEventDisableTiming) !=
                cudaSuccess ||
            cudaEventRecord(plan->ready, s) != cudaSuccess) {
            delete plan;
            return cuda_fail(cudaGetLastError(), "product plan event");
        }
    }
    plan->n1 = (int)j1.size();
    plan->n2 = (int)j2.size();
    plan->nnear = (int)near.size();
    plan->trows = trows;
    *out = plan;
    return STARSH_SUCCESS;
}

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
    ProductPlan *plan = nullptr;
    {
        std::lock_guard<std::mutex> g(rec->plan_lock);
        if (!rec->plan) {
            ProductPlan *built = nullptr;
            if ((info = build_plan(M, *rec, s, &built))) {
                cudaEventDestroy(ev);
                return info;
            }
            rec->plan = std::shared_ptr<void>(built, [](void *q) {
                delete (ProductPlan *)q;
            });
        }
        plan = (ProductPlan *)rec->plan.get();
    }
    if (plan->ready) cudaStreamWaitEvent(s, plan->ready, 0);
    {
        const long long tot = (long long)nrows * nrhs;
        k_scale_cols<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(
            dB, ldb, (int)nrows, nrhs, beta);
        count_launch();
    }
    // near blocks: dense D (stored, or regenerated when onfly)
    double *onfly_buf = nullptr;
    std::vector<const double *> nearD(F->nblocks_near, nullptr);
    if (F->nblocks_near > 0) {
        if (M->onfly) {
            size_t tot = 0;
            for (STARSH_int b = 0; b < F->nblocks_near; ++b)
                tot += (size_t)R->size[F->block_near[2 * b]] *
                       C->size[F->block_near[2 * b + 1]];
            onfly_buf = (double *)pool_alloc(tot * sizeof(double), s);
            if (onfly_buf == nullptr) {
                cudaEventDestroy(ev);
                return cuda_fail(cudaErrorMemoryAllocation, "onfly blocks");
            }
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
            if ((info = gen_blocks(rec->points->K, jobs, s))) {
                pool_free(onfly_buf);
                cudaEventDestroy(ev);
                return info;
            }
        } else {
            for (STARSH_int b = 0; b < F->nblocks_near; ++b) nearD[b] = rec->dD[b];
        }
    }
    // per call: T (rows of every block row x nrhs) and the near pointers
    const size_t tbytes = (size_t)plan->trows * nrhs * sizeof(double);
    const size_t nbytes = nearD.size() * sizeof(double *);
    char *scratch = nullptr;
    if (tbytes + nbytes > 0) {
        scratch = (char *)pool_alloc((tbytes + 255) / 256 * 256 + nbytes, s);
        if (scratch == nullptr) {
            if (onfly_buf) pool_free(onfly_buf);
            cudaEventDestroy(ev);
            return cuda_fail(cudaErrorMemoryAllocation, "product scratch");
        }
    }
    double *T = (double *)scratch;
    const double **dnear = (const double **)(scratch + (tbytes + 255) / 256 * 256);
    if (nbytes)
        cudaMemcpyAsync(dnear, nearD.data(), nbytes, cudaMemcpyHostToDevice, s);
    if (nrhs > 32)
        launch_products<4>(plan->j1, plan->n1, plan->vcol, plan->rowt, plan->j2,
                           plan->n2, plan->ucol, plan->near, dnear, dA, lda, T, dB,
                           ldb, nrhs, alpha, s);
    else if (nrhs > 16)
        launch_products<2>(plan->j1, plan->n1, plan->vcol, plan->rowt, plan->j2,
                           plan->n2, plan->ucol, plan->near, dnear, dA, lda, T, dB,
                           ldb, nrhs, alpha, s);
    else
        launch_products<1>(plan->j1, plan->n1, plan->vcol, plan->rowt, plan->j2,
                           plan->n2, plan->ucol, plan->near, dnear, dA, lda, T, dB,
                           ldb, nrhs, alpha, s);
    if (scratch) pool_free(scratch);
    if (onfly_buf) pool_free(onfly_buf);
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
