// Conjugate gradients on a TLR matrix whose factors stay on the device:
// the iteration of starsh_itersolvers__dcg_omp (reference
// src/itersolvers/cg.c:24-95) with every product a device dmml and every
// vector operation a device kernel.  Per right-hand side j:
//     r = b - M x, p = r, rs = ||r||, check = tol rs;
//     repeat: q = M p; alpha = rs^2 / (p . q); x += alpha p; r -= alpha q;
//             rs' = ||r||; if rs' < check the column is finished;
//             else p = r + (rs'^2 / rs^2) p, rs = rs'.
// The result is the number of the iteration at which the last column
// finished (as the reference returns it) or -1 after n iterations.  Dot
// products and norms are block reductions in a fixed order (one CTA per
// column), so the iteration is deterministic.
#include <cmath>
#include <mutex>
#include <vector>

#include "device_ctx.cuh"
#include "records.cuh"
#include "starsh-b200.h"

namespace b200 {

constexpr int kCgThreads = 256;

// Per-column scalars of the iteration.
struct CgCol {
    double rsold;    // ||r||^2 of the previous iteration
    double check;    // tol ||r_0|| (negative once finished)
    double alpha;
    double dot;      // p . q
    int active;
};

__device__ __forceinline__ double block_sum_d(double v, double *red)
{
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += red[q];
    __syncthreads();
    return s;   // valid in thread 0
}

// r_j = b_j + r_j (r holds -M x), p_j = r_j, the column's initial scalars.
__global__ void k_cg_init(const double *__restrict__ B, int ldb,
                          double *__restrict__ R, double *__restrict__ P,
                          int n, double tol, CgCol *cols)
{
    __shared__ double red[32];
    const int j = blockIdx.x;
    double *r = R + (size_t)j * n, *p = P + (size_t)j * n;
    const double *b = B + (size_t)j * ldb;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = r[i] + b[i];
        r[i] = v;
        p[i] = v;
        s += v * v;
    }
    s = block_sum_d(s, red);
    if (threadIdx.x == 0) {
        const double nrm = sqrt(s);
        cols[j].check = nrm * tol;
        cols[j].rsold = s;
        cols[j].active = 1;
    }
}

// p_j . q_j for the active columns.
__global__ void k_cg_dot(const double *__restrict__ P,
                         const double *__restrict__ Q, int n, CgCol *cols)
{
    __shared__ double red[32];
    const int j = blockIdx.x;
    if (!cols[j].active) return;
    const double *p = P + (size_t)j * n, *q = Q + (size_t)j * n;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += p[i] * q[i];
    s = block_sum_d(s, red);
    if (threadIdx.x == 0) {
        cols[j].dot = s;
        cols[j].alpha = cols[j].rsold / s;
    }
}

// x += alpha p, r -= alpha q; then ||r||, the convergence test and, for
// columns still running, p = r + beta p.  One CTA per column.
__global__ void k_cg_step(double *__restrict__ X, int ldx,
                          double *__restrict__ R, double *__restrict__ P,
                          const double *__restrict__ Q, int n, CgCol *cols,
                          int *finished)
{
    __shared__ double red[32];
    __shared__ double beta;
    __shared__ int go_on;
    const int j = blockIdx.x;
    if (!cols[j].active) return;
    const double alpha = cols[j].alpha;
    double *x = X + (size_t)j * ldx, *r = R + (size_t)j * n;
    double *p = P + (size_t)j * n;
    const double *q = Q + (size_t)j * n;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        x[i] += alpha * p[i];
        const double v = r[i] - alpha * q[i];
        r[i] = v;
        s += v * v;
    }
    s = block_sum_d(s, red);
    if (threadIdx.x == 0) {
        const double nrm = sqrt(s);
        if (nrm < cols[j].check) {
            cols[j].active = 0;
            cols[j].check = -1.0;
            atomicAdd(finished, 1);
            go_on = 0;
        } else {
            beta = s / cols[j].rsold;
            cols[j].rsold = s;
            go_on = 1;
        }
    }
    __syncthreads();
    if (!go_on) return;
    for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = r[i] + beta * p[i];
}

// Device CG; returns the iteration count as the reference does, -1 when
// not converged within n iterations, or -2 - (STARSH error) on failure.
static int cg_device(STARSH_blrm *M, int nrhs, const double *dB, int ldb,
                     double *dX, int ldx, double tol, int maxiter,
                     cudaStream_t s, Context &ctx, int *info)
{
    *info = STARSH_SUCCESS;
    const int n = (int)M->format->problem->shape[0];
    double *work = (double *)pool_alloc((size_t)3 * n * nrhs * sizeof(double), s);
    CgCol *cols = (CgCol *)pool_alloc(nrhs * sizeof(CgCol), s);
    int *fin = (int *)pool_alloc(sizeof(int), s);
    if (!work || !cols || !fin) {
        pool_free(work);
        pool_free(cols);
        pool_free(fin);
        *info = STARSH_MALLOC_ERROR;
        return -1;
    }
    double *R = work, *P = R + (size_t)n * nrhs, *Q = P + (size_t)n * nrhs;
    cudaMemsetAsync(fin, 0, sizeof(int), s);
    int result = -1;
    // r = -M x, then r += b
    int e = dmml_device(M, nrhs, -1.0, dX, ldx, 0.0, R, n, s, ctx);
    if (!e) {
        k_cg_init<<<nrhs, kCgThreads, 0, s>>>(dB, ldb, R, P, n, tol, cols);
        count_launch();
    }
    for (int it = 0; !e && it < maxiter; ++it) {
        if ((e = dmml_device(M, nrhs, 1.0, P, n, 0.0, Q, n, s, ctx))) break;
        k_cg_dot<<<nrhs, kCgThreads, 0, s>>>(P, Q, n, cols);
        k_cg_step<<<nrhs, kCgThreads, 0, s>>>(dX, ldx, R, P, Q, n, cols, fin);
        count_launch(2);
        int done = 0;
        if (cudaMemcpyAsync(&done, fin, sizeof(int), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            e = cuda_fail(cudaGetLastError(), "cg iteration");
            break;
        }
        if (done == nrhs) {
            result = it;
            break;
        }
    }
    if (e) *info = e;
    const cudaError_t ce = cudaGetLastError();
    if (!e && ce != cudaSuccess) *info = cuda_fail(ce, "cg kernels");
    pool_free(work);
    pool_free(cols);
    pool_free(fin);
    return result;
}

}  // namespace b200

using namespace b200;

extern "C" int starsh_b200_dcg_device(STARSH_blrm *matrix, int nrhs,
                                      const double *dB, int ldb, double *dX,
                                      int ldx, double tol, int maxiter,
                                      void *stream, int *iterations)
{
    if (matrix == nullptr || nrhs <= 0 || dB == nullptr || dX == nullptr ||
        iterations == nullptr || !(tol >= 0.0))
        return STARSH_WRONG_PARAMETER;
    const int n = (int)matrix->format->problem->shape[0];
    if (ldb < n || ldx < n) return STARSH_WRONG_PARAMETER;
    Context *ctx = context();
    if (!ctx) return STARSH_UNKNOWN_ERROR;
    std::lock_guard<std::mutex> guard(ctx->lock);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    int info;
    *iterations = cg_device(matrix, nrhs, dB, ldb, dX, ldx, tol,
                            maxiter > 0 ? maxiter : n, s, *ctx, &info);
    return info;
}

// Signature of starsh_itersolvers__dcg_omp (reference include/starsh.h:671-672)
// with host B and X; `work` is not used (the iteration's vectors live on
// the device).  Returns the iteration count, or -1 if not converged (or on
// an error, which starsh_b200_last_error() describes).
extern "C" int starsh_itersolvers__dcg_b200(STARSH_blrm *matrix, int nrhs,
                                            double *B, int ldb, double *X,
                                            int ldx, double tol, double *work)
{
    (void)work;
    if (matrix == nullptr || nrhs <= 0 || B == nullptr || X == nullptr)
        return -1;
    const int n = (int)matrix->format->problem->shape[0];
    if (ldb < n || ldx < n) return -1;
    Context *ctx = context();
    if (!ctx) return -1;
    std::lock_guard<std::mutex> guard(ctx->lock);
    cudaStream_t s = ctx->stream;
    double *dB = (double *)pool_alloc((size_t)2 * n * nrhs * sizeof(double), s);
    if (dB == nullptr) {
        cuda_fail(cudaErrorMemoryAllocation, "cg vectors");
        return -1;
    }
    double *dX = dB + (size_t)n * nrhs;
    cudaMemcpy2DAsync(dB, n * sizeof(double), B, (size_t)ldb * sizeof(double),
                      n * sizeof(double), nrhs, cudaMemcpyHostToDevice, s);
    cudaMemcpy2DAsync(dX, n * sizeof(double), X, (size_t)ldx * sizeof(double),
                      n * sizeof(double), nrhs, cudaMemcpyHostToDevice, s);
    int info;
    const int it = cg_device(matrix, nrhs, dB, n, dX, n, tol, n, s, *ctx, &info);
    if (info == STARSH_SUCCESS)
        cudaMemcpy2DAsync(X, (size_t)ldx * sizeof(double), dX, n * sizeof(double),
                          n * sizeof(double), nrhs, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    pool_free(dB);
    return info == STARSH_SUCCESS ? it : -1;
}
