// Shared definitions of the batched randomized-SVD engine: per-tile state,
// workspace layout and the launchers of the per-tile kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "gemm_f64.cuh"
#include "kernel_entry.cuh"

namespace b200 {

// Status bits of a tile.
enum : int {
    TILE_OK = 0,
    TILE_CHOL_TRUNC = 1,   // a re-orthogonalisation dropped dependent columns
    TILE_JACOBI_SLOW = 2,  // Jacobi sweeps hit their cap
    TILE_TAIL_LEFT = 4,    // energy outside the factors alone exceeds tol
    TILE_MMA_TIMEOUT = 8,  // a tensor-core wait of the sketch gave up
    TILE_RESKETCH = 16,    // the fused generator's row scales missed the
                           // exact row maxima: sketch again from stored D
    TILE_GEN_SEPARATE = 32,// too wide (or too many dimensions) for the
                           // fused kernel: separate generator and sketch
    TILE_PROJ_I8 = 64,     // projection on the tensor cores
};

// One far-field tile of a batch.
struct TileWork {
    long long row0, col0;   // offsets into the row/column cluster pivots
    int m, n, k;            // block shape and sketch width
    int slot;               // workspace slot
    int k1;                 // orthonormal basis columns after deflation
    int kb;                 // columns added by the residual pass
    int k2;                 // Gram factor columns for the small SVD
    int rank;               // accepted rank, or -1 (false far-field)
    int status;
    int need_pass_b;        // residual pass required by tol
    double tr_g;            // trace of the sketch Gram Y^T Y
    double tr_h;            // ||B||_F^2 = trace of B B^T
    double tail_h;          // energy left out of the Gram factor of B B^T
    // adaptive sketch (mixed engine)
    double dnorm2;          // ||D||_F^2 of the block, exact (FP64)
    int cols_done;          // sketch columns consumed so far
    int bcur;               // columns of the current round (0: inactive)
    int round_slot;         // its place among the round's sampling tiles,
                            // or -1 (compacted GEMM descriptors)
    int done;               // sampling finished (converged or capped)
    int kround;             // directions the current round's sample added
    int k1_round;           // basis columns when the current round began
    int sweeps;             // Jacobi sweeps the small SVD took
    int trunc_round;        // a CholQR of this round dropped columns
    double omega_var;       // variance of the sketch matrix's entries
    int prob;               // problem of the batch the tile belongs to
    int maxrank;            // the problem's maxrank and tol
    double tol;
    long long off_u, off_v; // output offsets (doubles)
};

// Per-slot workspace.  All matrices are column-major with the leading
// dimensions below; ints live in double-sized cells.
struct Workspace {
    double *base;
    size_t stride;          // doubles per slot
    int m_max, n_max, k_max;
    size_t oD, oY, oQ1, oQ, oS, oL, oT, oB, oC, oE, oSig, oPiv, oOrd, oNrm, oR, oRmx;
    // tensor-core projection (adaptive engine): byte slices of the scaled
    // basis, row and column exponents (0 when the layout has none)
    size_t oQd, oQe, oQf;

    __host__ __device__ double *D(int s) const { return base + s * stride + oD; }
    __host__ __device__ double *Y(int s) const { return base + s * stride + oY; }
    __host__ __device__ double *Q1(int s) const { return base + s * stride + oQ1; }
    __host__ __device__ double *Q(int s) const { return base + s * stride + oQ; }
    __host__ __device__ double *S(int s) const { return base + s * stride + oS; }
    __host__ __device__ double *L(int s) const { return base + s * stride + oL; }
    __host__ __device__ double *T(int s) const { return base + s * stride + oT; }
    __host__ __device__ double *B(int s) const { return base + s * stride + oB; }
    __host__ __device__ double *C(int s) const { return base + s * stride + oC; }
    __host__ __device__ double *E(int s) const { return base + s * stride + oE; }
    __host__ __device__ double *Sig(int s) const { return base + s * stride + oSig; }
    // per row, per 64-column block: the largest |D_ij| (ld (n_max+63)/64)
    __host__ __device__ double *Rmx(int s) const { return base + s * stride + oRmx; }
    __host__ __device__ int *Piv(int s) const { return (int *)(base + s * stride + oPiv); }
    __host__ __device__ int *Ord(int s) const { return (int *)(base + s * stride + oOrd); }
    // per-CTA partial sums of squares of the generated block
    __host__ __device__ double *Nrm(int s) const { return base + s * stride + oNrm; }
    // m x k temporary of the adaptive rounds (ld = m_max)
    __host__ __device__ double *R(int s) const { return base + s * stride + oR; }
    __host__ __device__ uint8_t *Qd(int s) const { return (uint8_t *)(base + s * stride + oQd); }
    __host__ __device__ int *Qe(int s) const { return (int *)(base + s * stride + oQe); }
    __host__ __device__ int *Qf(int s) const { return (int *)(base + s * stride + oQf); }
    // bytes per row of a Qd slice (rows: basis columns)
    __host__ __device__ int ldQd() const { return (m_max + 31) / 32 * 32; }
    // leading dimensions
    __host__ __device__ int ldD() const { return m_max; }
    __host__ __device__ int ldM() const { return m_max; }   // Y, Q1, Q
    __host__ __device__ int ldK() const { return k_max; }   // S, L, T, B, C
};

// Layout for the given maxima; returns doubles per slot.  proj_digits
// adds the fields of the tensor-core projection.
size_t workspace_layout(Workspace &w, int m_max, int n_max, int k_max,
                        bool store_d, bool proj_digits = false);

// GEMM steps of the pipeline, each turned into descriptors on the device.
enum GemmStep : int {
    STEP_SKETCH = 0,     // Y  = D Omega                  (m x k)
    STEP_GRAM_Y,         // S  = Y^T Y                    (k x k)
    STEP_Q1,             // Q1 = Yg T                     (m x k1)
    STEP_GRAM_Q1,        // S  = Q1^T Q1                  (k1 x k1)
    STEP_Q,              // Q  = Q1 T                     (m x k1)
    STEP_RES_Z,          // S  = Q^T Y                    (k1 x k)   pass B
    STEP_RES_Y,          // Y -= Q S                      (m x k)    pass B
    STEP_GRAM_YR,        // S  = Y^T Y of the residual    (k x k)    pass B
    STEP_Q1B,            // Q1 = Yg T                     (m x kb)   pass B
    STEP_RES_Z2,         // S  = Q^T Q1                   (k1 x kb)  pass B
    STEP_RES_Q1B,        // Q1 -= Q S                     (m x kb)   pass B
    STEP_GRAM_Q1B,       // S  = Q1^T Q1                  (kb x kb)  pass B
    STEP_QB,             // Q[:, k1:] = Q1 T              (m x kb)   pass B
    STEP_PROJECT,        // B  = Q^T D                    (k1 x n)
    STEP_GRAM_B,         // S  = B B^T                    (k1 x k1)
    STEP_ROTATE,         // C  = W^T B   (W in T)         (k2 x n)
    STEP_OUT_U,          // U  = Q Wsel  (Wsel in L)      (m x r)
    STEP_A_SKETCH,       // Y  = D Omega[:, c:c+b]        (m x b)    adaptive
    STEP_A_RES_Z,        // S  = Q^T Y                    (k1 x b)   adaptive
    STEP_A_RES_Y,        // Y -= Q S                      (m x b)    adaptive
    STEP_A_GRAM,         // S  = Y^T Y                    (b x b)    adaptive
    STEP_A_RES_Z2,       // second projection of the same sample (repeat
    STEP_A_RES_Y2,       //   pass, tiles flagged need_pass_b)
    STEP_A_GRAM2,
    STEP_A_Q1B,          // R  = Q1 T   (gathered residual columns)
    STEP_A_ORTH_Z,       // S  = Q^T R
    STEP_A_ORTH_R,       // R -= Q S
    STEP_A_GRAM_R,       // S  = R^T R
    STEP_A_QB,           // Q[:, k1:k1+kb] = R T
};

struct OutArena {
    double *U;
    double *V;
};

// Builds the descriptors of `step` for every tile of the batch.
void make_gemm_descs(GemmStep step, const TileWork *d_tiles, int ntiles,
                     Workspace ws, const double *d_omega, int ld_omega,
                     OutArena out, GemmDesc *d_desc, cudaStream_t stream,
                     bool compact = false);

// Per-tile kernels (one CTA per tile).
// Thresholds come from each tile's tol and maxrank; the generator reads
// the tile's kernel from d_kernels[tile.prob].
// need != 0: only tiles whose status has a bit of `need`.
// family != 0: every tile has that kernel family (a kernel compiled for
// it alone, where one exists).
void launch_gen_tiles(const DevKernel *d_kernels, const TileWork *d_tiles,
                      int ntiles, Workspace ws, cudaStream_t stream,
                      int need = 0, int family = 0);
// launch_pivchol and launch_jacobi return the number of kernels launched.
int launch_pivchol(int phase, const TileWork *d_tiles, TileWork *d_tiles_rw,
                   int ntiles, Workspace ws, cudaStream_t s);
// `act` (optional): the launch covers the `ntiles` tiles listed there (a
// round's sampling tiles) instead of the first `ntiles` of the batch.
void launch_gather_cols(int phase, const TileWork *d_tiles, int ntiles,
                        Workspace ws, cudaStream_t stream,
                        const int *act = nullptr);
void launch_chol_inv(int phase, TileWork *d_tiles, int ntiles, Workspace ws,
                     cudaStream_t stream, const int *act = nullptr);
int launch_jacobi(TileWork *d_tiles, int ntiles, Workspace ws,
                  cudaStream_t stream, cudaStream_t side);
void launch_rank_cut(TileWork *d_tiles, int ntiles, Workspace ws,
                     cudaStream_t stream);
void launch_merge_basis(TileWork *d_tiles, int ntiles, cudaStream_t stream);
// Adaptive sketch: squared Frobenius norms of the generated blocks, round
// set-up (returns through d_active whether any tile still samples) and the
// per-round pivoted Cholesky of the residual block's Gram.
void launch_block_norms(const TileWork *d_tiles, TileWork *d_rw, int ntiles,
                        Workspace ws, cudaStream_t stream);
void launch_round_setup(TileWork *d_tiles, int ntiles, int block,
                        int *d_active, int *d_act, cudaStream_t stream);
void launch_round_end(TileWork *d_tiles, int ntiles, int verify,
                      cudaStream_t stream);
void launch_round_pivchol(TileWork *d_tiles, int ntiles, Workspace ws,
                          int repeat, cudaStream_t stream,
                          const int *act = nullptr);
void launch_select_w(const TileWork *d_tiles, int ntiles, Workspace ws,
                     cudaStream_t stream);
// Tensor-core projection B = Q^T D (proj_i8.cu) of the tiles with at most
// 64 basis columns and 4096 rows: the preparation flags them
// TILE_PROJ_I8 (the FP64 projection step skips them).  launch_proj_i8
// returns false (nothing launched) when the layout has no digit fields or
// the TMA descriptors cannot be made.
void launch_proj_prep(TileWork *d_tiles, int ntiles, Workspace ws,
                      cudaStream_t stream);
bool launch_proj_i8(TileWork *d_tiles, int ntiles, Workspace ws,
                    cudaStream_t stream);
void launch_write_v(const TileWork *d_tiles, int ntiles, Workspace ws,
                    OutArena out, cudaStream_t stream);
// Adaptive sketch on the tensor cores (int8 digits of D, see
// sketch_i8.cu): Y(:, 0:bcur) = D Omega8(:, cols_done + (0:ncols)) for
// every tile with an active round.  sketch_i8_fits() tells whether a batch
// shape is supported (ncols <= 64, n_max <= 8192, shared memory).
bool sketch_i8_fits(int ncols, int n_max);
// Returns false (nothing launched) when the batch's layout cannot be
// described to the TMA unit (odd leading dimension).
bool launch_sketch_i8(const TileWork *d_tiles, int ntiles, Workspace ws,
                      const int8_t *om8, int ld_om8, int om8_cols, int ncols,
                      cudaStream_t stream, int need = 0);
// First sampling round with the generation fused in (gen_sketch_i8.cu):
// D, its exact norms and row maxima, and Y(:, 0:bcur) = D Omega8(:, 0:nc)
// with bound-based row scales; tiles whose bound missed are flagged
// TILE_RESKETCH.  Tiles flagged TILE_GEN_SEPARATE are skipped.
// gen_sketch_i8_fits(): the round's width is supported (ncols <= 64);
// gen_sketch_i8_tile_ok(): a tile can be generated by it (n <= 1024,
// ndim <= 4).
bool gen_sketch_i8_fits(int nc);
bool gen_sketch_i8_tile_ok(int n, int ndim);
bool launch_gen_sketch_i8(const DevKernel *d_kernels, TileWork *d_tiles,
                          int ntiles, Workspace ws, const int8_t *om8,
                          int ld_om8, int om8_cols, int ncols,
                          cudaStream_t stream);
// Omega8(j, c) = clip(round(32 g), -127, 127), g the Gaussian of
// launch_gaussian's (j, c); rows past `rows` up to ld are zero.
void launch_gaussian_i8(int8_t *d_om8, int rows, int cols, int ld,
                        unsigned long long seed, cudaStream_t stream);

// Omega(j, c) for j < rows, c < cols into column-major storage with leading
// dimension ld; entry (j, c) depends only on (j, c) and the seed, not on
// the storage shape.
void launch_gaussian(double *d_omega, int rows, int cols, int ld,
                     unsigned long long seed, cudaStream_t stream);

}  // namespace b200
