// Batched FP64 GEMM on the double-precision tensor-core path
// (mma.sync m8n8k4 .f64).  Every batch entry has its own operands and
// shape, read from a device descriptor array, so one launch covers all
// tiles of a batch even when their ranks differ:
//     C = alpha * op(A) * op(B) + beta * C,   op(A): M x K, op(B): K x N,
// all matrices column-major.  TA/TB select op = transpose at compile time.
#pragma once
#include <cuda_runtime.h>

namespace b200 {

struct GemmDesc {
    const double *A;
    const double *B;
    double *C;
    int M, N, K;
    int lda, ldb, ldc;
    double alpha, beta;
};

constexpr int kGemmBM = 64;
constexpr int kGemmBN = 64;
constexpr int kGemmBK = 16;
constexpr int kGemmThreads = 256;
// Shared-memory row stride (doubles) of the [row][k] tiles: 20 puts the
// 4x4 (row, k) footprint of a half-warp fragment load on 16 distinct bank
// pairs.
constexpr int kGemmLds = kGemmBK + 4;

// Launches one GEMM per descriptor; entries whose M, N or K is 0 are
// skipped (beta is still applied when K == 0).  max_m/max_n bound the
// shapes of all entries.  split_k (A^T B and A B^T): every entry runs on 64 x 64
// CTA tiles whatever the bounds, and a tile with few rows or columns of
// its own splits K over the spare warps; an entry's result then depends on
// its own shape alone, never on the bounds of the batch it is in.
// Returns the CUDA error of the launch.
cudaError_t gemm_f64_batched(bool ta, bool tb, const GemmDesc *d_desc,
                             int batch, int max_m, int max_n,
                             cudaStream_t stream, bool split_k = false);

}  // namespace b200
