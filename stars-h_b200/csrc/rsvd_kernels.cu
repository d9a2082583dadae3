// Device kernels of the batched randomized-SVD engine (FP64 path).
//
// Per tile (D: m x n block, Omega: n x k Gaussian, k = min(maxrank +
// oversample, m, n)) the engine computes the same factorisation as the
// reference's starsh_dense_dlrrsdd (src/backends/sequential/dense/
// drsdd.c:16-93): Y = D Omega, an orthonormal basis Q of range(Y),
// B = Q^T D, the SVD of B, the rank cut of starsh_dense_dsvfr
// (src/backends/sequential/dense/dsvfr.c:16-47) and U = Q Us_r,
// V = (S_r Vs_r)^T.  The orthogonalisation and the small SVD are done with
// Gram matrices so that every O(m n k) and O(m k^2) step is a GEMM:
//   * basis: pivoted Cholesky of Y^T Y drops directions below the FP64
//     squared-noise floor or below (tol/10)^2 of the sketch energy, CholQR2
//     on the kept columns; when tol^2 is below the squared-noise floor a
//     second pass orthogonalises the explicit residual Y - Q Q^T Y, which
//     recovers the directions the squared Gram could not resolve;
//   * small SVD: B B^T = L L^T (pivoted Cholesky), one-sided Jacobi on L
//     gives the left singular vectors W of B; the energies of the rotated
//     rows C = W^T B are summed in FP64 directly from C, so the tail that
//     decides the rank is exact to FP64 rounding even where the Gram's
//     eigenvalues are not.
#include <cfloat>
#include <climits>
#include <cooperative_groups.h>
#include "engine.cuh"

namespace b200 {

// ------------------------------------------------------------ layout

size_t workspace_layout(Workspace &w, int m_max, int n_max, int k_max,
                        bool store_d, bool proj_digits)
{
    size_t o = 0;
    auto take = [&](size_t n) {
        const size_t r = o;
        o += (n + 31) & ~(size_t)31;   // 256-byte aligned fields
        return r;
    };
    w.m_max = m_max;
    w.n_max = n_max;
    w.k_max = k_max;
    w.oD = store_d ? take((size_t)m_max * n_max) : 0;
    w.oY = take((size_t)m_max * k_max);
    w.oQ1 = take((size_t)m_max * k_max);
    w.oQ = take((size_t)m_max * k_max);
    w.oS = take((size_t)k_max * k_max);
    w.oL = take((size_t)k_max * k_max);
    w.oT = take((size_t)k_max * k_max);
    w.oB = take((size_t)k_max * n_max);
    w.oC = take((size_t)k_max * n_max);
    w.oE = take(k_max);
    w.oSig = take(k_max);
    w.oPiv = take((k_max + 1) / 2);
    w.oOrd = take((k_max + 1) / 2);
    w.oNrm = take((size_t)((m_max + 63) / 64) * ((n_max + 63) / 64));
    w.oR = take((size_t)m_max * k_max);
    w.oRmx = take((size_t)m_max * ((n_max + 63) / 64));
    w.oQd = w.oQe = w.oQf = 0;
    if (proj_digits) {
        // 7 byte slices x 64 basis columns x ldQd bytes; m ints; 64 ints
        w.oQd = take((size_t)7 * 64 * ((m_max + 31) / 32 * 32) / 8);
        w.oQe = take(((size_t)m_max + 1) / 2);
        w.oQf = take(32);
    }
    w.stride = o;
    return o;
}

// -------------------------------------------------------- generation

// D(slot) = block of the tile, column-major with ld = m_max.  A CTA owns
// 64 rows and kGenCb column blocks of 64: the coordinates of its rows and
// columns are gathered through the cluster pivots into shared memory once
// (point-major layouts and dimensions above kStageDim read global memory
// directly), then each thread evaluates 16 entries of one row in each
// 64 x 64 block, so stores run down the columns and are coalesced.  Per
// 64 x 64 block the CTA writes the sum of squares of its entries to
// Nrm(slot) and each row's largest |D_ij| to Rmx(slot), reduced in a fixed
// order (deterministic per-tile norms for the adaptive sketch).  Several
// blocks per CTA spread the gathers and barriers of the staging over more
// entries.
constexpr int kStageDim = 4;
#ifndef GEN_CB
#define GEN_CB 4              // 64-column blocks of one generator CTA
#endif
constexpr int kGenCb = GEN_CB;
#ifndef GEN_MIN_BLOCKS
#define GEN_MIN_BLOCKS 3      // CTAs per SM the generator is compiled for
#endif
#ifndef GEN_MIN_BLOCKS_FIX
#define GEN_MIN_BLOCKS_FIX 4  // the same for a launch of one kernel family
#endif
#ifndef GEN_MIN_BLOCKS_MATERN
#define GEN_MIN_BLOCKS_MATERN 4   // ... of the Matérn family (its rare
#endif                            // series path spills; measured faster)
#ifndef GEN_UNROLL
#define GEN_UNROLL 8          // entries of a thread evaluated together
#endif
constexpr int kGenUnroll = GEN_UNROLL;
#ifndef GEN_UNROLL_MATERN
#define GEN_UNROLL_MATERN 2   // the same for the Matérn families
#endif

// The entries of one thread in a 64 x 64 block: rows ii, columns jj0,
// jj0 + 4, ... below jn, written to Dcol[jj * ld] (Dcol points at row ii of
// the block's first column); returns their sum of squares.
template <int FAM, int NDIM, int LDC>
__device__ __forceinline__ double gen_entries(
    const DevKernel &K, bool staged, const double (*rc)[64],
    const double (*cc)[LDC], const long long *ri, const long long *ci, int ii,
    int jj0, int jn, double *Dcol, int ld, double &amax)
{
    // NDIM > 0: coordinates staged in shared memory, dimension known at
    // compile time (the row's coordinates held in registers); NDIM == 0:
    // staged, any dimension up to kStageDim; NDIM < 0: read through the
    // pivots from global memory
    double xr[NDIM > 0 ? NDIM : 1];
    if constexpr (NDIM > 0) {
        #pragma unroll
        for (int d = 0; d < NDIM; ++d) xr[d] = rc[d][ii];
    }
    double ss = 0.0;
    amax = 0.0;
    // the Matern entry (table piece per entry) keeps a shorter unroll:
    // more of its bodies cost more registers than they save
    constexpr int kUnroll =
        FAM == FAM_MATERN || FAM == FAM_MATERN2 ? GEN_UNROLL_MATERN : kGenUnroll;
    #pragma unroll kUnroll
    for (int jj = jj0; jj < jn; jj += 4) {
        double dist = 0.0;
        if constexpr (NDIM > 0) {
            #pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                const double q = __dsub_rn(xr[d], cc[d][jj]);
                dist = __dadd_rn(dist, __dmul_rn(q, q));
            }
        } else if constexpr (NDIM == 0) {
            for (int d = 0; d < K.ndim; ++d) {
                const double q = __dsub_rn(rc[d][ii], cc[d][jj]);
                dist = __dadd_rn(dist, __dmul_rn(q, q));
            }
        } else {
            dist = sq_dist(K, ri[ii], ci[jj]);
        }
        const double v = entry_fam<FAM>(K, dist, ri[ii], ci[jj]);
        Dcol[(size_t)jj * ld] = v;
        ss += v * v;
        amax = fmax(amax, fabs(v));
    }
    return ss;
}

// Dispatch on the staging dimension for one family.
template <int FAM, int LDC>
__device__ __forceinline__ double gen_entries_dim(
    const DevKernel &K, bool staged, const double (*rc)[64],
    const double (*cc)[LDC], const long long *ri, const long long *ci, int ii,
    int jj0, int jn, double *Dcol, int ld, double &amax)
{
    if (!staged)
        return gen_entries<FAM, -1, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
    if (K.ndim == 2)
        return gen_entries<FAM, 2, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
    if (K.ndim == 3)
        return gen_entries<FAM, 3, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
    return gen_entries<FAM, 0, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
}

// The 16 entries of each thread in one 64 x 64 block of a generator CTA
// (columns jb0 .. jb0 + 63 of the tile), family dispatched once.
template <int LDC>
__device__ __forceinline__ double gen_block(
    const DevKernel &K, bool staged, const double (*rc)[64],
    const double (*cc)[LDC], const long long *ri, const long long *ci, int ii,
    int jj0, int jn, double *Dcol, int ld, double &amax)
{
    switch (K.family) {
    case FAM_EXP:
        return gen_entries_dim<FAM_EXP, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
    case FAM_SQREXP:
        return gen_entries_dim<FAM_SQREXP, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
    case FAM_MATERN:
        return gen_entries_dim<FAM_MATERN, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
    case FAM_MATERN2:
        return gen_entries_dim<FAM_MATERN2, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
    case FAM_COULOMB:
        return gen_entries_dim<FAM_COULOMB, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
    case FAM_SIN:
        return gen_entries_dim<FAM_SIN, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
    case FAM_COS:
        return gen_entries_dim<FAM_COS, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
    default:
        return gen_entries_dim<FAM_RBF, LDC>(K, staged, rc, cc, ri, ci, ii, jj0, jn, Dcol, ld, amax);
    }
}

// FIX != 0: every tile of the launch has kernel family FIX (the family's
// entry code alone, compiled for MINB CTAs per SM); FIX == 0: the family
// is read per CTA.
template <int FIX, int MINB>
__global__ void __launch_bounds__(256, MINB)
k_gen_tiles(const DevKernel *__restrict__ kernels,
            const TileWork *__restrict__ tiles, Workspace ws, int need)
{
    constexpr int W = 64 * kGenCb;   // columns of the CTA
    const TileWork tw = tiles[blockIdx.z];
    if (blockIdx.x * 64 >= tw.m || blockIdx.y * W >= tw.n) return;
    if (need != 0 && (tw.status & need) == 0) return;
    __shared__ double rc[kStageDim][64], cc[kStageDim][W];
    __shared__ long long ri[64], ci[W];
    __shared__ double red[kGenCb][8];
    __shared__ double rmx[kGenCb][4][64];
    __shared__ DevKernel Ks;
    const int t = threadIdx.x;
    if (t == 0) Ks = kernels[tw.prob];
    __syncthreads();
    const DevKernel &K = Ks;
    const int i0 = blockIdx.x * 64, j0 = blockIdx.y * W;
    const int ncol = min(W, tw.n - j0);      // columns of this CTA
    const bool staged = !K.aos && K.ndim <= kStageDim;
    if (t < 64) {
        const int i = min(i0 + t, tw.m - 1);
        ri[t] = K.row_piv[tw.row0 + i];
    }
    for (int e = t; e < W; e += 256) {
        const int j = min(j0 + e, tw.n - 1);
        ci[e] = K.col_piv[tw.col0 + j];
    }
    __syncthreads();
    if (staged) {
        for (int q = t; q < 64 * K.ndim; q += 256) {
            const int d = q / 64, e = q % 64;
            rc[d][e] = K.row_pt[d * K.row_count + ri[e]];
        }
        for (int q = t; q < W * K.ndim; q += 256) {
            const int d = q / W, e = q % W;
            cc[d][e] = K.col_pt[d * K.col_count + ci[e]];
        }
    }
    __syncthreads();
    const int ii = t & 63, i = i0 + ii;
    double *D = ws.D(tw.slot);
    const int ld = ws.ldD();
    #pragma unroll 1
    for (int b = 0; b < kGenCb; ++b) {
        const int jb = b * 64;                // first column of the block
        if (jb >= ncol) break;
        double ss = 0.0, amax = 0.0;
        if (i < tw.m)
            ss = FIX == 0
                ? gen_block<W>(K, staged, rc, (const double (*)[W])&cc[0][jb],
                               ri, ci + jb, ii, t >> 6, min(64, ncol - jb),
                               D + (size_t)(j0 + jb) * ld + i, ld, amax)
                : gen_entries_dim<FIX == 0 ? FAM_EXP : FIX, W>(
                      K, staged, rc, (const double (*)[W])&cc[0][jb], ri,
                      ci + jb, ii, t >> 6, min(64, ncol - jb),
                      D + (size_t)(j0 + jb) * ld + i, ld, amax);
        // largest |D_ij| of each row of the block (the int8 sketch's row
        // scales): the four threads of a row combine through shared memory
        rmx[b][t >> 6][ii] = amax;
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) ss += __shfl_down_sync(0xffffffffu, ss, o);
        if ((t & 31) == 0) red[b][t >> 5] = ss;
    }
    __syncthreads();
    const int nbc = (ws.n_max + 63) / 64;     // 64-column blocks of a tile row
    const int nblk = (ncol + 63) / 64;
    for (int q = t; q < 64 * nblk; q += 256) {
        const int b = q / 64, r = q % 64;
        if (i0 + r < tw.m)
            ws.Rmx(tw.slot)[(size_t)(i0 + r) * nbc + blockIdx.y * kGenCb + b] =
                fmax(fmax(rmx[b][0][r], rmx[b][1][r]), fmax(rmx[b][2][r], rmx[b][3][r]));
    }
    if (t < nblk) {
        double a = 0.0;
        for (int w = 0; w < 8; ++w) a += red[t][w];
        ws.Nrm(tw.slot)[blockIdx.x * nbc + blockIdx.y * kGenCb + t] = a;
    }
}

void launch_gen_tiles(const DevKernel *d_kernels, const TileWork *d_tiles,
                      int ntiles, Workspace ws, cudaStream_t stream, int need,
                      int family)
{
    dim3 grid((ws.m_max + 63) / 64, (ws.n_max + 64 * kGenCb - 1) / (64 * kGenCb), ntiles);
    switch (family) {
    case FAM_EXP:
        k_gen_tiles<FAM_EXP, GEN_MIN_BLOCKS_FIX><<<grid, 256, 0, stream>>>(d_kernels, d_tiles, ws, need);
        break;
    case FAM_SQREXP:
        k_gen_tiles<FAM_SQREXP, GEN_MIN_BLOCKS_FIX><<<grid, 256, 0, stream>>>(d_kernels, d_tiles, ws, need);
        break;
    case FAM_MATERN:
        k_gen_tiles<FAM_MATERN, GEN_MIN_BLOCKS_MATERN><<<grid, 256, 0, stream>>>(d_kernels, d_tiles, ws, need);
        break;
    case FAM_COULOMB:
        k_gen_tiles<FAM_COULOMB, GEN_MIN_BLOCKS_FIX><<<grid, 256, 0, stream>>>(d_kernels, d_tiles, ws, need);
        break;
    case FAM_SIN:
        k_gen_tiles<FAM_SIN, GEN_MIN_BLOCKS_FIX><<<grid, 256, 0, stream>>>(d_kernels, d_tiles, ws, need);
        break;
    default:
        k_gen_tiles<0, GEN_MIN_BLOCKS><<<grid, 256, 0, stream>>>(d_kernels, d_tiles, ws, need);
    }
}

// ---------------------------------------------------- Gaussian sketch

// Philox4x32-10 counter-based generator (J. K. Salmon, M. A. Moraes,
// R. O. Dror, D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11); multipliers and Weyl increments are the published constants.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
    #pragma unroll
    for (int r = 0; r < 10; ++r) {
        const unsigned lo0 = 0xD2511F53u * c.x;
        const unsigned hi0 = __umulhi(0xD2511F53u, c.x);
        const unsigned lo1 = 0xCD9E8D57u * c.z;
        const unsigned hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// Omega entries N(0,1): one Philox block -> two 53-bit uniforms in (0,1]
// -> one Box-Muller pair (G. E. P. Box, M. E. Muller, Ann. Math. Stat. 29
// (1958) 610-611).
// Entries (2q, c) and (2q + 1, c) come from the Philox block with counter
// (q, c, 0, 0).
__global__ void k_gaussian(double *out, int rows, int cols, int ld,
                           unsigned long long seed)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int col = blockIdx.y;
    if (2 * q >= rows || col >= cols) return;
    const uint4 c = make_uint4((unsigned)q, (unsigned)col, 0u, 0u);
    const uint4 r = philox4x32_10(c, make_uint2((unsigned)seed,
                                                (unsigned)(seed >> 32)));
    const unsigned long long b1 = ((unsigned long long)r.x << 32) | r.y;
    const unsigned long long b2 = ((unsigned long long)r.z << 32) | r.w;
    const double u1 = ((b1 >> 11) + 1) * 0x1.0p-53;   // (0, 1]
    const double u2 = (b2 >> 11) * 0x1.0p-53;         // [0, 1)
    const double rad = sqrt(-2.0 * log(u1));
    double s, co;
    sincospi(2.0 * u2, &s, &co);
    double *o = out + (size_t)col * ld;
    o[2 * q] = rad * co;
    if (2 * q + 1 < rows) o[2 * q + 1] = rad * s;
}

void launch_gaussian(double *d_omega, int rows, int cols, int ld,
                     unsigned long long seed, cudaStream_t stream)
{
    if (rows <= 0 || cols <= 0) return;
    const int pairs = (rows + 1) / 2;
    dim3 grid((pairs + 255) / 256, cols);
    k_gaussian<<<grid, 256, 0, stream>>>(d_omega, rows, cols, ld, seed);
}

// Omega8(j, c) = clip(round(32 g(j, c)), -127, 127) with g the Gaussian of
// k_gaussian for the same (j, c); rows rows .. ld - 1 are zero.
__global__ void k_gaussian_i8(int8_t *out, int rows, int cols, int ld,
                              unsigned long long seed)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int col = blockIdx.y;
    if (2 * q >= ld || col >= cols) return;
    const uint4 c = make_uint4((unsigned)q, (unsigned)col, 0u, 0u);
    const uint4 r = philox4x32_10(c, make_uint2((unsigned)seed,
                                                (unsigned)(seed >> 32)));
    const unsigned long long b1 = ((unsigned long long)r.x << 32) | r.y;
    const unsigned long long b2 = ((unsigned long long)r.z << 32) | r.w;
    const double u1 = ((b1 >> 11) + 1) * 0x1.0p-53;
    const double u2 = (b2 >> 11) * 0x1.0p-53;
    const double rad = sqrt(-2.0 * log(u1));
    double s, co;
    sincospi(2.0 * u2, &s, &co);
    int8_t *o = out + (size_t)col * ld;
    auto q8 = [](double g) {
        return (int8_t)fmax(-127.0, fmin(127.0, rint(32.0 * g)));
    };
    o[2 * q] = 2 * q < rows ? q8(rad * co) : (int8_t)0;
    if (2 * q + 1 < ld) o[2 * q + 1] = 2 * q + 1 < rows ? q8(rad * s) : (int8_t)0;
}

void launch_gaussian_i8(int8_t *d_om8, int rows, int cols, int ld,
                        unsigned long long seed, cudaStream_t stream)
{
    if (cols <= 0 || ld <= 0) return;
    const int pairs = (ld + 1) / 2;
    dim3 grid((pairs + 255) / 256, cols);
    k_gaussian_i8<<<grid, 256, 0, stream>>>(d_om8, rows, cols, ld, seed);
}

// ------------------------------------------------- GEMM descriptors

// With `compact`, only the tiles sampling in the current round write a
// descriptor, at their round slot: the GEMM then runs over that many
// descriptors instead of the whole batch (every adaptive-round step is
// empty for the other tiles).
__global__ void k_make_desc(GemmStep step, const TileWork *__restrict__ tiles,
                            int ntiles, Workspace ws,
                            const double *__restrict__ omega, int ld_omega,
                            OutArena out, GemmDesc *__restrict__ desc,
                            int compact)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const TileWork tw = tiles[t];
    if (compact && tw.round_slot < 0) return;
    const int s = tw.slot;
    GemmDesc d;
    d.alpha = 1.0;
    d.beta = 0.0;
    d.M = d.N = d.K = 0;
    d.A = d.B = nullptr;
    d.C = nullptr;
    d.lda = d.ldb = d.ldc = 1;
    const int ldm = ws.ldM(), ldk = ws.ldK();
    switch (step) {
    case STEP_SKETCH:
        d.A = ws.D(s); d.lda = ws.ldD();
        d.B = omega; d.ldb = ld_omega;
        d.C = ws.Y(s); d.ldc = ldm;
        d.M = tw.m; d.N = tw.k; d.K = tw.n;
        break;
    case STEP_GRAM_YR:  // TN, residual of pass B
        if (!tw.need_pass_b) break;
        d.A = ws.Y(s); d.lda = ldm;
        d.B = ws.Y(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.k; d.N = tw.k; d.K = tw.m;
        break;
    case STEP_GRAM_Y:   // TN
        d.A = ws.Y(s); d.lda = ldm;
        d.B = ws.Y(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.k; d.N = tw.k; d.K = tw.m;
        break;
    case STEP_Q1:       // NN: Q1buf = Qbuf(gathered) * T
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.T(s); d.ldb = ldk;
        d.C = ws.Q1(s); d.ldc = ldm;
        d.M = tw.m; d.N = tw.k1; d.K = tw.k1;
        break;
    case STEP_GRAM_Q1:  // TN
        d.A = ws.Q1(s); d.lda = ldm;
        d.B = ws.Q1(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.k1; d.N = tw.k1; d.K = tw.m;
        break;
    case STEP_Q:        // NN: Qbuf = Q1buf * T
        d.A = ws.Q1(s); d.lda = ldm;
        d.B = ws.T(s); d.ldb = ldk;
        d.C = ws.Q(s); d.ldc = ldm;
        d.M = tw.m; d.N = tw.k1; d.K = tw.k1;
        break;
    case STEP_RES_Z:    // TN: S = Q^T Y
        if (!tw.need_pass_b) break;
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.Y(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.k1; d.N = tw.k; d.K = tw.m;
        break;
    case STEP_RES_Y:    // NN: Y -= Q S
        if (!tw.need_pass_b) break;
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.S(s); d.ldb = ldk;
        d.C = ws.Y(s); d.ldc = ldm;
        d.alpha = -1.0; d.beta = 1.0;
        d.M = tw.m; d.N = tw.k; d.K = tw.k1;
        break;
    case STEP_Q1B:      // NN: Ybuf = Q1buf(gathered residual) * T
        if (tw.kb <= 0) break;
        d.A = ws.Q1(s); d.lda = ldm;
        d.B = ws.T(s); d.ldb = ldk;
        d.C = ws.Y(s); d.ldc = ldm;
        d.M = tw.m; d.N = tw.kb; d.K = tw.kb;
        break;
    case STEP_RES_Z2:   // TN: S = Q^T Ybuf
        if (tw.kb <= 0) break;
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.Y(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.k1; d.N = tw.kb; d.K = tw.m;
        break;
    case STEP_RES_Q1B:  // NN: Ybuf -= Q S
        if (tw.kb <= 0) break;
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.S(s); d.ldb = ldk;
        d.C = ws.Y(s); d.ldc = ldm;
        d.alpha = -1.0; d.beta = 1.0;
        d.M = tw.m; d.N = tw.kb; d.K = tw.k1;
        break;
    case STEP_GRAM_Q1B: // TN
        if (tw.kb <= 0) break;
        d.A = ws.Y(s); d.lda = ldm;
        d.B = ws.Y(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.kb; d.N = tw.kb; d.K = tw.m;
        break;
    case STEP_QB:       // NN: Q[:, k1:k1+kb] = Ybuf T
        if (tw.kb <= 0) break;
        d.A = ws.Y(s); d.lda = ldm;
        d.B = ws.T(s); d.ldb = ldk;
        d.C = ws.Q(s) + (size_t)tw.k1 * ldm; d.ldc = ldm;
        d.M = tw.m; d.N = tw.kb; d.K = tw.kb;
        break;
    case STEP_PROJECT:  // TN: B = Q^T D
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.D(s); d.ldb = ws.ldD();
        d.C = ws.B(s); d.ldc = ldk;
        d.M = tw.k1; d.N = tw.n; d.K = tw.m;
        if (tw.status & TILE_PROJ_I8) d.M = 0;   // on the tensor cores
        break;
    case STEP_GRAM_B:   // NT: S = B B^T
        d.A = ws.B(s); d.lda = ldk;
        d.B = ws.B(s); d.ldb = ldk;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.k1; d.N = tw.k1; d.K = tw.n;
        break;
    case STEP_ROTATE:   // TN: C = W^T B, W in T
        d.A = ws.T(s); d.lda = ldk;
        d.B = ws.B(s); d.ldb = ldk;
        d.C = ws.C(s); d.ldc = ldk;
        d.M = tw.k2; d.N = tw.n; d.K = tw.k1;
        break;
    case STEP_A_SKETCH: // NN: Y = D Omega[:, c:c+b]
        if (tw.bcur <= 0) break;
        d.A = ws.D(s); d.lda = ws.ldD();
        d.B = omega + (size_t)tw.cols_done * ld_omega; d.ldb = ld_omega;
        d.C = ws.Y(s); d.ldc = ldm;
        d.M = tw.m; d.N = tw.bcur; d.K = tw.n;
        break;
    case STEP_A_RES_Z:  // TN: S = Q^T Y
        if (tw.bcur <= 0 || tw.k1 <= 0) break;
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.Y(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.k1; d.N = tw.bcur; d.K = tw.m;
        break;
    case STEP_A_RES_Y:  // NN: Y -= Q S
        if (tw.bcur <= 0 || tw.k1 <= 0) break;
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.S(s); d.ldb = ldk;
        d.C = ws.Y(s); d.ldc = ldm;
        d.alpha = -1.0; d.beta = 1.0;
        d.M = tw.m; d.N = tw.bcur; d.K = tw.k1;
        break;
    case STEP_A_GRAM:   // TN: S = Y^T Y
        if (tw.bcur <= 0) break;
        d.A = ws.Y(s); d.lda = ldm;
        d.B = ws.Y(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.bcur; d.N = tw.bcur; d.K = tw.m;
        break;
    case STEP_A_RES_Z2: // TN: S = Q^T Y, repeat pass on the same sample
        if (!tw.need_pass_b || tw.bcur <= 0) break;
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.Y(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.k1; d.N = tw.bcur; d.K = tw.m;
        break;
    case STEP_A_RES_Y2: // NN: Y -= Q S
        if (!tw.need_pass_b || tw.bcur <= 0) break;
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.S(s); d.ldb = ldk;
        d.C = ws.Y(s); d.ldc = ldm;
        d.alpha = -1.0; d.beta = 1.0;
        d.M = tw.m; d.N = tw.bcur; d.K = tw.k1;
        break;
    case STEP_A_GRAM2:  // TN: S = Y^T Y
        if (!tw.need_pass_b || tw.bcur <= 0) break;
        d.A = ws.Y(s); d.lda = ldm;
        d.B = ws.Y(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.bcur; d.N = tw.bcur; d.K = tw.m;
        break;
    case STEP_A_Q1B:    // NN: R = Q1buf(gathered residual columns) T
        if (tw.kb <= 0) break;
        d.A = ws.Q1(s); d.lda = ldm;
        d.B = ws.T(s); d.ldb = ldk;
        d.C = ws.R(s); d.ldc = ldm;
        d.M = tw.m; d.N = tw.kb; d.K = tw.kb;
        break;
    case STEP_A_ORTH_Z: // TN: S = Q^T R
        if (tw.kb <= 0 || tw.k1 <= 0) break;
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.R(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.k1; d.N = tw.kb; d.K = tw.m;
        break;
    case STEP_A_ORTH_R: // NN: R -= Q S
        if (tw.kb <= 0 || tw.k1 <= 0) break;
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.S(s); d.ldb = ldk;
        d.C = ws.R(s); d.ldc = ldm;
        d.alpha = -1.0; d.beta = 1.0;
        d.M = tw.m; d.N = tw.kb; d.K = tw.k1;
        break;
    case STEP_A_GRAM_R: // TN: S = R^T R
        if (tw.kb <= 0) break;
        d.A = ws.R(s); d.lda = ldm;
        d.B = ws.R(s); d.ldb = ldm;
        d.C = ws.S(s); d.ldc = ldk;
        d.M = tw.kb; d.N = tw.kb; d.K = tw.m;
        break;
    case STEP_A_QB:     // NN: Q[:, k1:k1+kb] = R T
        if (tw.kb <= 0) break;
        d.A = ws.R(s); d.lda = ldm;
        d.B = ws.T(s); d.ldb = ldk;
        d.C = ws.Q(s) + (size_t)tw.k1 * ldm; d.ldc = ldm;
        d.M = tw.m; d.N = tw.kb; d.K = tw.kb;
        break;
    case STEP_OUT_U:    // NN: U = Q Wsel, Wsel in L
        if (tw.rank <= 0) break;
        d.A = ws.Q(s); d.lda = ldm;
        d.B = ws.L(s); d.ldb = ldk;
        d.C = out.U + tw.off_u; d.ldc = tw.m;
        d.M = tw.m; d.N = tw.rank; d.K = tw.k1;
        break;
    }
    desc[compact ? tw.round_slot : t] = d;
}

void make_gemm_descs(GemmStep step, const TileWork *d_tiles, int ntiles,
                     Workspace ws, const double *d_omega, int ld_omega,
                     OutArena out, GemmDesc *d_desc, cudaStream_t stream,
                     bool compact)
{
    k_make_desc<<<(ntiles + 127) / 128, 128, 0, stream>>>(
        step, d_tiles, ntiles, ws, d_omega, ld_omega, out, d_desc,
        compact ? 1 : 0);
}

// ------------------------------------------------- block reductions

struct MaxLoc {
    double v;
    int i;
};

// Block-wide argmax (largest value, then smallest index).  `red` holds one
// entry per warp.  All threads get the result.
__device__ MaxLoc block_argmax(MaxLoc x, MaxLoc *red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        MaxLoc y;
        y.v = __shfl_down_sync(0xffffffffu, x.v, o);
        y.i = __shfl_down_sync(0xffffffffu, x.i, o);
        if (y.v > x.v || (y.v == x.v && y.i < x.i)) x = y;
    }
    __syncthreads();
    if (lane == 0) red[warp] = x;
    __syncthreads();
    if (warp == 0) {
        x = lane < (int)(blockDim.x >> 5) ? red[lane] : MaxLoc{-DBL_MAX, 1 << 30};
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            MaxLoc y;
            y.v = __shfl_down_sync(0xffffffffu, x.v, o);
            y.i = __shfl_down_sync(0xffffffffu, x.i, o);
            if (y.v > x.v || (y.v == x.v && y.i < x.i)) x = y;
        }
        if (lane == 0) red[0] = x;
    }
    __syncthreads();
    MaxLoc r = red[0];
    __syncthreads();
    return r;
}

// block_argmax of x and, in the same pass, the block sum of y (returned in
// *sum; `reds` holds one double per warp).
__device__ MaxLoc block_argmax_sum(MaxLoc x, double y, MaxLoc *red,
                                   double *reds, double *sum)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        MaxLoc z;
        z.v = __shfl_down_sync(0xffffffffu, x.v, o);
        z.i = __shfl_down_sync(0xffffffffu, x.i, o);
        if (z.v > x.v || (z.v == x.v && z.i < x.i)) x = z;
        y += __shfl_down_sync(0xffffffffu, y, o);
    }
    __syncthreads();
    if (lane == 0) {
        red[warp] = x;
        reds[warp] = y;
    }
    __syncthreads();
    if (warp == 0) {
        const bool in = lane < (int)(blockDim.x >> 5);
        x = in ? red[lane] : MaxLoc{-DBL_MAX, 1 << 30};
        y = in ? reds[lane] : 0.0;
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            MaxLoc z;
            z.v = __shfl_down_sync(0xffffffffu, x.v, o);
            z.i = __shfl_down_sync(0xffffffffu, x.i, o);
            if (z.v > x.v || (z.v == x.v && z.i < x.i)) x = z;
            y += __shfl_down_sync(0xffffffffu, y, o);
        }
        if (lane == 0) {
            red[0] = x;
            reds[0] = y;
        }
    }
    __syncthreads();
    const MaxLoc r = red[0];
    *sum = reds[0];
    __syncthreads();
    return r;
}

__device__ double block_sum(double x, double *red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    __syncthreads();
    if (lane == 0) red[warp] = x;
    __syncthreads();
    if (warp == 0) {
        x = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[0] = x;
    }
    __syncthreads();
    const double r = red[0];
    __syncthreads();
    return r;
}

// ------------------------------------------------ pivoted Cholesky

// Phases: A/B basis passes of the fixed-width sketch, H small SVD, R a
// round of the adaptive sketch, R2 its repeat pass on the same sample.
enum : int { PH_A = 0, PH_B = 1, PH_H = 2, PH_R = 3, PH_R2 = 4 };

constexpr int kSmallThreads = 256;
#ifndef PIVCHOL_H_LANES
#define PIVCHOL_H_LANES 4
#endif
constexpr int kPivcholLanes = PIVCHOL_H_LANES;   // lanes per row, large phase-H factors
constexpr int kPivcholSplit = 128;               // "large": more rows than this
constexpr int kMaxK = 1024;   // largest sketch width handled by one CTA

// Left-looking pivoted Cholesky of the Gram in S(slot) (dimension nn):
// P^T G P ~ L L^T, L stored in L(slot) with rows in the original order
// (column j holds the multipliers of pivot j).  Stops when the largest
// remaining diagonal entry is <= thr.  For the basis phases (A, B) the
// pivot block R11 = L[piv, :]^T is inverted into T(slot).
//
// LPR lanes share a row's update (the left-looking product with the
// previous columns, read from L2): more loads in flight for the large
// factors of phase H, whose few tiles per batch bound the launch.  Tiles
// with nn outside [nn_lo, nn_hi] are left to another launch.
template <int LPR>
__global__ void __launch_bounds__(kSmallThreads * LPR)
k_pivchol(TileWork *__restrict__ tiles, Workspace ws, int phase, int nn_lo,
          int nn_hi, const int *__restrict__ act)
{
    TileWork &tw = tiles[act ? act[blockIdx.x] : blockIdx.x];
    const int s = tw.slot;
    const double tol = tw.tol;
    __shared__ double dg[kMaxK];
    __shared__ double lp[kMaxK];
    __shared__ unsigned char used[kMaxK];
    __shared__ MaxLoc red[32];
    __shared__ double redd[32];

    int nn;
    if (phase == PH_H) nn = tw.k1;
    else if (phase == PH_R) nn = tw.bcur;
    else if (phase == PH_R2) nn = tw.need_pass_b ? tw.bcur : 0;
    else nn = tw.k;
    if (nn < nn_lo || nn > nn_hi) return;   // another launch's tile
    if ((phase == PH_B && !tw.need_pass_b) ||
        ((phase == PH_R || phase == PH_R2) && nn <= 0)) {
        if (threadIdx.x == 0) {
            tw.kb = 0;
            if (phase == PH_R) tw.kround = 0;
            if (phase == PH_R2) tw.need_pass_b = 0;
        }
        return;
    }
    const double *G = ws.S(s);
    const int ld = ws.ldK();
    double *L = ws.L(s);
    int *piv = ws.Piv(s);

    double loc = 0.0;
    for (int i = threadIdx.x; i < nn; i += blockDim.x) {
        dg[i] = G[(size_t)i * ld + i];
        used[i] = 0;
        loc += dg[i];
    }
    const double trace = block_sum(loc, redd);
    MaxLoc mx{-DBL_MAX, 1 << 30};
    for (int i = threadIdx.x; i < nn; i += blockDim.x)
        if (dg[i] > mx.v) mx = MaxLoc{dg[i], i};
    const double dmax = block_argmax(mx, red).v;

    double thr;
    int cap = nn;
    double stop_trace = -1.0;   // PH_H: stop once the remaining trace is below
    if (phase == PH_A) {
        const double tol_floor = 0.01 * tol * tol * trace / nn;
        const double noise = 1e-15 * dmax;
        thr = fmax(noise, tol_floor);
        if (threadIdx.x == 0) {
            tw.tr_g = trace;
            tw.need_pass_b = noise > tol_floor && trace > 0.0;
        }
    } else if (phase == PH_B) {
        thr = fmax(1e-15 * dmax, 0.01 * tol * tol * tw.tr_g / tw.k);
        cap = tw.k - tw.k1;
    } else if (phase == PH_R || phase == PH_R2) {
        // residual columns r_i = (I - Q Q^T) D w_i have E||r_i||^2 =
        // ||(I - Q Q^T) D||_F^2: keep directions above (tol/10)^2 ||D||_F^2.
        // When the squared-noise floor of this Gram hides part of that
        // range, the same sample is projected and searched once more.
        // (E||r_i||^2 carries the variance of Omega's entries: 1 for the
        // Gaussian, about 32^2 for the int8 sketch matrix)
        const double noise = 1e-15 * dmax;
        const double var = tw.omega_var > 0.0 ? tw.omega_var : 1.0;
        const double floor_ = 0.01 * tol * tol * tw.dnorm2 * var;
        thr = fmax(noise, floor_);
        cap = min(nn, tw.k - tw.k1);
        // a repeat pass only where (tol/10)^2 lies below the squared-noise
        // floor at all (the same decision alone or in any batch)
        if (threadIdx.x == 0)
            tw.need_pass_b = phase == PH_R && noise > floor_ &&
                             0.01 * tol * tol < 1e-15;
    } else {
        thr = 1e-18 * dmax;
        if (threadIdx.x == 0) tw.tr_h = trace;
        // The energy the factor leaves out joins the rank rule's tail
        // (tail_h), so the factor may stop at 1% of the tile's error
        // budget: it, and the Jacobi SVD on it, are then no wider than the
        // tolerance needs (the rank grows by at most the directions that 1%
        // hides).
        const double energy = tw.dnorm2 > 0.0 ? fmax(tw.dnorm2, trace) : trace;
        stop_trace = 0.01 * tol * tol * energy;
        // A block whose energy outside the sketched basis, ||D||^2 -
        // ||B||^2 (less the rounding allowance of k_rank_cut), alone
        // exceeds the budget is stored dense whatever its small SVD says:
        // the rank cut reaches rank -1 from k2 = 0 by the same test, so the
        // factor and the Jacobi SVD are skipped.
        const double dn = tw.dnorm2;
        if (dn > 0.0 &&
            fmax(0.0, dn - trace - 2e-15 * dn) > tol * tol * fmax(dn, trace)) {
            if (threadIdx.x == 0) {
                tw.k2 = 0;
                tw.tail_h = trace;
                tw.status |= TILE_TAIL_LEFT;
            }
            return;
        }
    }
    if (!(dmax > 0.0)) thr = DBL_MAX;   // zero or invalid Gram: rank 0

    int j = 0;
    for (; j < cap; ++j) {
        MaxLoc cand{-DBL_MAX, 1 << 30};
        double rest = 0.0;          // remaining trace, for PH_H's stop
        for (int i = threadIdx.x; i < nn; i += blockDim.x)
            if (!used[i]) {
                if (dg[i] > cand.v) cand = MaxLoc{dg[i], i};
                rest += fmax(0.0, dg[i]);
            }
        MaxLoc best;
        if (stop_trace >= 0.0) {
            double total;
            best = block_argmax_sum(cand, rest, red, redd, &total);
            if (total <= stop_trace) break;
        } else {
            best = block_argmax(cand, red);
        }
        if (!(best.v > thr)) break;
        const int p = best.i;
        const double sp = sqrt(best.v);
        for (int l = threadIdx.x; l < j; l += blockDim.x)
            lp[l] = L[(size_t)l * ld + p];
        __syncthreads();
        if (threadIdx.x == 0) {
            piv[j] = p;
            used[p] = 1;
        }
        if constexpr (LPR == 1) {
        for (int i = threadIdx.x; i < nn; i += blockDim.x) {
            double v;
            if (i == p) {
                v = sp;
            } else if (used[i]) {
                v = 0.0;
            } else {
                // G(p, i) - sum_l L(i, l) L(p, l), in four independent
                // partial sums (the chain over l is the step's latency)
                double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
                int l = 0;
                for (; l + 3 < j; l += 4) {
                    a0 = fma(L[(size_t)l * ld + i], lp[l], a0);
                    a1 = fma(L[(size_t)(l + 1) * ld + i], lp[l + 1], a1);
                    a2 = fma(L[(size_t)(l + 2) * ld + i], lp[l + 2], a2);
                    a3 = fma(L[(size_t)(l + 3) * ld + i], lp[l + 3], a3);
                }
                for (; l < j; ++l) a0 = fma(L[(size_t)l * ld + i], lp[l], a0);
                const double acc = G[(size_t)p * ld + i] - ((a0 + a1) + (a2 + a3));
                v = acc / sp;
                dg[i] -= v * v;
            }
            L[(size_t)j * ld + i] = v;
        }
        } else {
        // lane q of a row's group sums l = q, q + LPR, ... (two chains);
        // the block-uniform row loop keeps every lane in the shuffles
        const int q = threadIdx.x % LPR;
        for (int i0 = 0; i0 < nn; i0 += blockDim.x / LPR) {
            const int i = i0 + threadIdx.x / LPR;
            const bool live = i < nn && i != p && !used[i];
            double a0 = 0.0, a1 = 0.0;
            if (live) {
                int l = q;
                for (; l + LPR < j; l += 2 * LPR) {
                    a0 = fma(L[(size_t)l * ld + i], lp[l], a0);
                    a1 = fma(L[(size_t)(l + LPR) * ld + i], lp[l + LPR], a1);
                }
                for (; l < j; l += LPR) a0 = fma(L[(size_t)l * ld + i], lp[l], a0);
            }
            double part = a0 + a1;
            #pragma unroll
            for (int o = LPR / 2; o > 0; o >>= 1)
                part += __shfl_xor_sync(0xffffffffu, part, o);
            if (i < nn && q == 0) {
                double v;
                if (i == p) {
                    v = sp;
                } else if (used[i]) {
                    v = 0.0;
                } else {
                    v = (G[(size_t)p * ld + i] - part) / sp;
                    dg[i] -= v * v;
                }
                L[(size_t)j * ld + i] = v;
            }
        }
        }
        __syncthreads();
    }
    const int cnt = j;
    if (threadIdx.x == 0) {
        if (phase == PH_A) tw.k1 = cnt;
        else if (phase == PH_B || phase == PH_R || phase == PH_R2) tw.kb = cnt;
        else tw.k2 = cnt;
        if (phase == PH_R) {
            tw.kround = cnt;
            if (cnt == 0) tw.need_pass_b = 0;
        }
    }
    if (phase == PH_H) {
        // energy of B outside the span of the factor's columns
        double rest = 0.0;
        for (int i = threadIdx.x; i < nn; i += blockDim.x)
            if (!used[i]) rest += fmax(0.0, dg[i]);
        rest = block_sum(rest, redd);
        if (threadIdx.x == 0) tw.tail_h = cnt > 0 ? rest : trace;
        return;
    }
    // T = R11^{-1}, R11(a, b) = L(piv[b], a) for a <= b (upper triangular).
    double *T = ws.T(s);
    for (int c = threadIdx.x; c < cnt; c += blockDim.x) {
        double *x = T + (size_t)c * ld;
        for (int a = c + 1; a < cnt; ++a) x[a] = 0.0;
        x[c] = 1.0 / L[(size_t)c * ld + piv[c]];
        for (int a = c - 1; a >= 0; --a) {
            double acc = 0.0;
            for (int b = a + 1; b <= c; ++b) acc += L[(size_t)a * ld + piv[b]] * x[b];
            x[a] = -acc / L[(size_t)a * ld + piv[a]];
        }
    }
}

void launch_round_pivchol(TileWork *d_tiles, int ntiles, Workspace ws,
                          int repeat, cudaStream_t stream, const int *act)
{
    k_pivchol<1><<<ntiles, kSmallThreads, 0, stream>>>(
        d_tiles, ws, repeat ? PH_R2 : PH_R, 0, INT_MAX, act);
}

// ||D||_F^2 of every block from the generator's per-CTA partial sums, in a
// fixed order.
__global__ void k_block_norms(TileWork *__restrict__ tiles, Workspace ws)
{
    TileWork &tw = tiles[blockIdx.x];
    const int gx = (tw.m + 63) / 64, gy = (tw.n + 63) / 64;
    const int ldn = (ws.n_max + 63) / 64;
    __shared__ double red[8];
    double a = 0.0;
    for (int q = threadIdx.x; q < gx * gy; q += blockDim.x)
        a += ws.Nrm(tw.slot)[(q / gy) * ldn + q % gy];
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        tw.dnorm2 = s;
    }
}

void launch_block_norms(const TileWork *, TileWork *d_rw, int ntiles,
                        Workspace ws, cudaStream_t stream)
{
    k_block_norms<<<ntiles, 256, 0, stream>>>(d_rw, ws);
}

// Start of a sampling round: tiles not done sample min(block, k - cols)
// more columns; *active counts them (each takes the next round slot, in
// any order: a slot only places the tile's GEMM descriptors).
__global__ void k_round_setup(TileWork *__restrict__ tiles, int ntiles,
                              int block, int *active, int *act)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    TileWork &tw = tiles[t];
    if (tw.done || tw.cols_done >= tw.k) {
        tw.bcur = 0;
        tw.done = 1;
        tw.round_slot = -1;
        return;
    }
    tw.bcur = min(block, tw.k - tw.cols_done);
    tw.k1_round = tw.k1;
    tw.trunc_round = 0;
    tw.round_slot = atomicAdd(active, 1);
    act[tw.round_slot] = t;
}

void launch_round_setup(TileWork *d_tiles, int ntiles, int block,
                        int *d_active, int *d_act, cudaStream_t stream)
{
    cudaMemsetAsync(d_active, 0, sizeof(int), stream);
    k_round_setup<<<(ntiles + 127) / 128, 128, 0, stream>>>(d_tiles, ntiles,
                                                            block, d_active,
                                                            d_act);
}

// End of a round: the new orthonormal columns join the basis.  The tile is
// finished when the round's sample left at least `verify` columns whose
// residuals against the grown basis all fell below the threshold (so the
// residual estimate rests on that many independent Gaussian samples), when
// it found no direction at all, or when the k columns are exhausted.
__global__ void k_round_end(TileWork *__restrict__ tiles, int ntiles,
                            int verify)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    TileWork &tw = tiles[t];
    if (tw.bcur <= 0) return;
    tw.cols_done += tw.bcur;
    const int added = tw.k1 + tw.kb - tw.k1_round;
    if (tw.kround == 0 || tw.cols_done >= tw.k ||
        (tw.bcur - added >= verify && !tw.trunc_round))
        tw.done = 1;
    tw.k1 += tw.kb;       // (kb is 0 here: each pass merged its columns)
    tw.kb = 0;
    tw.bcur = 0;
}

void launch_round_end(TileWork *d_tiles, int ntiles, int verify,
                      cudaStream_t stream)
{
    k_round_end<<<(ntiles + 127) / 128, 128, 0, stream>>>(d_tiles, ntiles,
                                                          verify);
}

int launch_pivchol(int phase, const TileWork *, TileWork *d_tiles_rw,
                    int ntiles, Workspace ws, cudaStream_t s)
{
    if (phase == PH_H && kPivcholLanes > 1) {
        // small factors one lane per row, large ones kPivcholLanes
        k_pivchol<1><<<ntiles, kSmallThreads, 0, s>>>(d_tiles_rw, ws, phase, 0,
                                                      kPivcholSplit, nullptr);
        k_pivchol<kPivcholLanes><<<ntiles, kSmallThreads * kPivcholLanes, 0, s>>>(
            d_tiles_rw, ws, phase, kPivcholSplit + 1, INT_MAX, nullptr);
        return 2;
    } else {
        k_pivchol<1><<<ntiles, kSmallThreads, 0, s>>>(d_tiles_rw, ws, phase, 0,
                                                      INT_MAX, nullptr);
        return 1;
    }
}

// Gathers the pivot columns of Y into the Q buffer (phase A) or the Q1
// buffer (phase B).
__global__ void k_gather_cols(const TileWork *__restrict__ tiles,
                              Workspace ws, int phase,
                              const int *__restrict__ act)
{
    const TileWork tw = tiles[act ? act[blockIdx.x] : blockIdx.x];
    const int s = tw.slot;
    const int cnt = phase == PH_A ? tw.k1 : tw.kb;
    if (cnt <= 0) return;
    const int *piv = ws.Piv(s);
    const double *Y = ws.Y(s);
    double *dst = phase == PH_A ? ws.Q(s) : ws.Q1(s);
    const int ld = ws.ldM();
    for (int c = blockIdx.y; c < cnt; c += gridDim.y) {
        const double *src = Y + (size_t)piv[c] * ld;
        for (int i = threadIdx.x; i < tw.m; i += blockDim.x)
            dst[(size_t)c * ld + i] = src[i];
    }
}

void launch_gather_cols(int phase, const TileWork *d_tiles, int ntiles,
                        Workspace ws, cudaStream_t stream, const int *act)
{
    dim3 grid(ntiles, 16);
    k_gather_cols<<<grid, 256, 0, stream>>>(d_tiles, ws, phase, act);
}

// Cholesky G = R^T R of the re-orthogonalisation Gram in S(slot)
// (dimension k1 for phase A, kb for phase B), R into L(slot), then
// T(slot) = R^{-1}.  For phase B the new columns are appended to the basis
// afterwards by the caller's merge step.
__global__ void __launch_bounds__(kSmallThreads)
k_chol_inv(TileWork *__restrict__ tiles, Workspace ws, int phase,
           const int *__restrict__ act)
{
    TileWork &tw = tiles[act ? act[blockIdx.x] : blockIdx.x];
    const int s = tw.slot;
    const int nn = phase == PH_A ? tw.k1 : tw.kb;
    if (nn <= 0) return;
    const double *G = ws.S(s);
    double *R = ws.L(s);
    double *T = ws.T(s);
    const int ld = ws.ldK();
    __shared__ double diag;
    __shared__ int stop;
    if (threadIdx.x == 0) stop = 0;
    __syncthreads();
    int nn_ok = nn;
    for (int j = 0; j < nn; ++j) {
        if (threadIdx.x == 0) {
            const double gjj = G[(size_t)j * ld + j];
            double acc = gjj;
            for (int l = 0; l < j; ++l) {
                const double r = R[(size_t)j * ld + l];
                acc -= r * r;
            }
            // a column numerically inside the span of the previous ones:
            // the factor keeps the columns before it (they come in
            // decreasing pivot order) and the round may not finish the
            // tile on its verification columns
            if (!(acc > 1e-14 * gjj)) stop = 1;
            diag = sqrt(fmax(acc, 0.0));
            R[(size_t)j * ld + j] = diag;
        }
        __syncthreads();
        if (stop) { nn_ok = j; break; }
        const double rjj = diag;
        for (int c = j + 1 + threadIdx.x; c < nn; c += blockDim.x) {
            double acc = G[(size_t)c * ld + j];
            for (int l = 0; l < j; ++l)
                acc -= R[(size_t)j * ld + l] * R[(size_t)c * ld + l];
            R[(size_t)c * ld + j] = acc / rjj;
        }
        __syncthreads();
    }
    for (int c = threadIdx.x; c < nn_ok; c += blockDim.x) {
        double *x = T + (size_t)c * ld;
        for (int a = c + 1; a < nn_ok; ++a) x[a] = 0.0;
        x[c] = 1.0 / R[(size_t)c * ld + c];
        for (int a = c - 1; a >= 0; --a) {
            double acc = 0.0;
            for (int b = a + 1; b <= c; ++b) acc += R[(size_t)b * ld + a] * x[b];
            x[a] = -acc / R[(size_t)a * ld + a];
        }
    }
    if (threadIdx.x == 0 && nn_ok < nn) {
        if (phase == PH_A) tw.k1 = nn_ok;
        else tw.kb = nn_ok;
        tw.trunc_round = 1;
        tw.status |= TILE_CHOL_TRUNC;
    }
}

void launch_chol_inv(int phase, TileWork *d_tiles, int ntiles, Workspace ws,
                     cudaStream_t stream, const int *act)
{
    k_chol_inv<<<ntiles, kSmallThreads, 0, stream>>>(d_tiles, ws, phase, act);
}

// -------------------------------------------------- one-sided Jacobi

// One-sided Jacobi (Hestenes) on the columns of A = L(slot) (k1 x k2):
// column pairs are rotated until mutually orthogonal; then the columns of
// A V are the eigenvectors of L L^T scaled by the singular values.  L comes
// from a pivoted Cholesky of B B^T (the transpose of a column-pivoted QR
// factor of B^T), the preconditioning under which one-sided Jacobi needs
// few sweeps (Z. Drmac, K. Veselic, SIAM J. Matrix Anal. Appl. 29 (2008)).
// Pairs follow the round-robin tournament ordering: k2/2 disjoint pairs per
// step, all rotated at once, a block barrier between steps.
//
// The cost is the chain of dependent steps (k2 - 1 per sweep), each issue
// bound on its SM for large tiles, so a pair is rotated by a group of G
// lanes holding E rows each in registers (G E >= k1): the group sizes its
// dot-product reduction to the column length, and a warp rotates 32 / G
// pairs at once, sharing the instructions of the rotation angle among
// them.  The kernel is instantiated per size
// class; tiles of one class share a launch, every other tile's CTA returns
// at once.  Columns live in shared memory when they fit, otherwise in
// global memory (L2-resident for the tiles of one launch).  W (normalised
// columns) goes to T(slot), squared norms to Sig(slot).
constexpr size_t kJacobiSmemMax = 220 * 1024;

// Size classes, by rows (k1), with G E just above the row count so that few
// lanes rotate padding; factors in shared memory when they fit, else the
// block kernel (k_jacobi_block).  The last class streams rows through
// registers for k1 > 512.
__host__ __device__ inline int jacobi_class(int rows, int cols)
{
    const size_t bytes = (size_t)(rows | 1) * cols * sizeof(double);
    const bool fits = bytes <= kJacobiSmemMax;
    if (rows <= 32) return 0;                     // G 4,  E 8,  64 threads
    if (rows <= 64) return 1;                     // G 4,  E 16, 128 threads
    if (rows <= 128) return 2;                    // G 8,  E 16, 512 threads
    if (rows <= 192) return fits ? 3 : 4;         // G 16, E 12, 512 threads
    if (rows <= 256) return fits ? 5 : 6;         // G 16, E 16, 512 threads
    if (rows <= 288) return 7;                    // G 16, E 18, blocks
    if (rows <= 320) return 8;                    // G 16, E 20, blocks
    if (rows <= 512) return 9;                    // G 32, E 16, blocks
    return 10;                                    // streamed, global
}

// Most columns a factor of the class can have (columns <= rows).
__host__ __device__ constexpr int jacobi_class_cols(int cls)
{
    return cls == 0 ? 32 : cls == 1 ? 64 : cls == 2 ? 128 : cls <= 4 ? 192
         : cls <= 6 ? 256 : cls == 7 ? 288 : cls == 8 ? 320 : cls == 9 ? 512
         : kMaxK;
}

// Convergence bookkeeping shared by the Jacobi kernels.  Every column
// pair is checked once per sweep at a fixed step of the schedule (T steps
// per sweep); lastrot[c] is the step at which column c was last rotated.
// A pair whose previous check (T steps ago) found it orthogonal and whose
// columns have not been rotated since is orthogonal still: it is skipped,
// so late sweeps, and the final sweep that confirms convergence, only
// look at the pairs that changed.  A sweep that rotates nothing ends the
// iteration exactly as when every pair is checked.
__device__ __forceinline__ bool jacobi_unchanged(const int *lastrot, int a,
                                                 int b, int since)
{
    return lastrot[a] < since && lastrot[b] < since;
}

// Rotation of the column pair (ca, cb) by the G lanes of one group (gl =
// lane within the group).  Every lane of the warp calls this (inactive
// groups with valid = false) because the reductions shuffle across the
// whole warp.  Returns true if the pair was rotated.
template <int G, int E>
__device__ __forceinline__ bool jacobi_rotate(double *ca, double *cb, int rows,
                                              int gl, bool valid, double eps2)
{
    double xa[E], xb[E];
    double al = 0.0, be = 0.0, ga = 0.0;
    #pragma unroll
    for (int q = 0; q < E; ++q) {
        const int i = gl + G * q;
        const bool in = valid && i < rows;
        xa[q] = in ? ca[i] : 0.0;
        xb[q] = in ? cb[i] : 0.0;
    }
    #pragma unroll
    for (int q = 0; q < E; ++q) {
        al = fma(xa[q], xa[q], al);
        be = fma(xb[q], xb[q], be);
        ga = fma(xa[q], xb[q], ga);
    }
    #pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
        al += __shfl_xor_sync(0xffffffffu, al, o);
        be += __shfl_xor_sync(0xffffffffu, be, o);
        ga += __shfl_xor_sync(0xffffffffu, ga, o);
    }
    // |gamma| > eps sqrt(alpha beta), compared in squares
    if (!(ga * ga > eps2 * al * be) || !(al > 0.0) || !(be > 0.0))
        return false;
    // t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)), zeta = (beta - alpha) /
    // (2 gamma), rewritten with one division: t = sign(d) g / (|d| + h),
    // d = beta - alpha, g = 2 gamma, h = sqrt(d^2 + g^2).
    const double d = be - al, g = 2.0 * ga;
    const double h = sqrt(fma(d, d, g * g));
    const double t = (d >= 0.0 ? g : -g) / (fabs(d) + h);
    const double c = rsqrt(fma(t, t, 1.0));
    const double sn = c * t;
    #pragma unroll
    for (int q = 0; q < E; ++q) {
        const int i = gl + G * q;
        if (i < rows) {
            ca[i] = c * xa[q] - sn * xb[q];
            cb[i] = sn * xa[q] + c * xb[q];
        }
    }
    return true;
}

// The same for long columns: rows streamed in chunks of 32 per lane (one
// warp per pair), loaded twice (dot products, then rotation).
__device__ bool jacobi_rotate_stream(double *ca, double *cb, int rows,
                                     int lane, bool valid, double eps2)
{
    double al = 0.0, be = 0.0, ga = 0.0;
    if (valid) {
        for (int i = lane; i < rows; i += 32) {
            const double x = ca[i], y = cb[i];
            al = fma(x, x, al);
            be = fma(y, y, be);
            ga = fma(x, y, ga);
        }
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        al += __shfl_xor_sync(0xffffffffu, al, o);
        be += __shfl_xor_sync(0xffffffffu, be, o);
        ga += __shfl_xor_sync(0xffffffffu, ga, o);
    }
    if (!(ga * ga > eps2 * al * be) || !(al > 0.0) || !(be > 0.0))
        return false;
    const double d = be - al, g = 2.0 * ga;
    const double h = sqrt(fma(d, d, g * g));
    const double t = (d >= 0.0 ? g : -g) / (fabs(d) + h);
    const double c = rsqrt(fma(t, t, 1.0));
    const double sn = c * t;
    for (int i = lane; i < rows; i += 32) {
        const double x = ca[i], y = cb[i];
        ca[i] = c * x - sn * y;
        cb[i] = sn * x + c * y;
    }
    return true;
}

template <int CLASS, int G, int E, int THREADS, bool SMEM>
__global__ void __launch_bounds__(THREADS, THREADS <= 128 ? 512 / THREADS : 1)
k_jacobi(TileWork *__restrict__ tiles, Workspace ws)
{
    extern __shared__ double sm[];
    __shared__ int rotated[2];
    __shared__ int lastrot[jacobi_class_cols(CLASS)];
    TileWork &tw = tiles[blockIdx.x];
    const int s = tw.slot;
    const int rows = tw.k1, cols = tw.k2;
    if (cols <= 0 || jacobi_class(rows, cols) != CLASS) return;   // uniform
    for (int c = threadIdx.x; c < cols; c += THREADS) lastrot[c] = -1;
    // Relative orthogonality the rotations stop at: the rank cut needs the
    // left singular vectors orthonormal to well below tol (their overlap
    // enters the tail energies squared and the projector linearly): 1 % of
    // tol, at most 1e-7.
    const double eps = fmax(1e-15, fmin(1e-7, 0.01 * tw.tol));
    const double eps2 = eps * eps;
    const int ldg = ws.ldK();
    const int lds = rows | 1;   // odd stride: fewer bank conflicts
    double *A = SMEM ? sm : ws.L(s);
    const int lda = SMEM ? lds : ldg;
    if (SMEM) {
        const double *Lg = ws.L(s);
        for (int e = threadIdx.x; e < rows * cols; e += THREADS) {
            const int c = e / rows, i = e - c * rows;
            A[(size_t)c * lda + i] = Lg[(size_t)c * ldg + i];
        }
    }
    if (threadIdx.x == 0) rotated[0] = rotated[1] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kGroupsPerWarp = 32 / G;
    constexpr int kWarps = THREADS / 32;
    const int gw = lane / G, gl = lane % G;
    const int nc = cols + (cols & 1);      // players, with a bye if odd
    const int npairs = nc / 2;
    const int T = nc - 1;                  // steps per sweep
    int sweep = 0;
    for (; sweep < 40; ++sweep) {
        bool any = false;
        for (int step = 0; step < nc - 1; ++step) {
            const int now = sweep * T + step;
            for (int base = warp * kGroupsPerWarp; base < npairs;
                 base += kWarps * kGroupsPerWarp) {
                const int p = base + gw;
                int a = 0, b = 0;
                if (p < npairs) {
                    // a = 1 + (p - 1 + step) mod (nc - 1) for p > 0,
                    // b = 1 + (nc - 2 - p + step) mod (nc - 1); both
                    // arguments lie in [0, 2 (nc - 1))
                    int x = p - 1 + step, y = nc - 2 - p + step;
                    if (x >= nc - 1) x -= nc - 1;
                    if (y >= nc - 1) y -= nc - 1;
                    a = p == 0 ? 0 : 1 + x;
                    b = 1 + y;
                }
                const bool valid = p < npairs && a < cols && b < cols &&
                                   !jacobi_unchanged(lastrot, a, b, now - T);
                if (!__any_sync(0xffffffffu, valid)) continue;   // warp-uniform
                double *ca = A + (size_t)a * lda, *cb = A + (size_t)b * lda;
                bool rot;
                if constexpr (E > 0)
                    rot = jacobi_rotate<G, E>(ca, cb, rows, gl, valid, eps2);
                else
                    rot = jacobi_rotate_stream(ca, cb, rows, lane, valid, eps2);
                if (rot && gl == 0) lastrot[a] = lastrot[b] = now;
                any |= rot;
            }
            __syncthreads();
        }
        // double-buffered flag: cleared one sweep ahead, read after a barrier
        if (any) rotated[sweep & 1] = 1;
        if (threadIdx.x == 0) rotated[(sweep + 1) & 1] = 0;
        __syncthreads();
        if (!rotated[sweep & 1]) break;
    }
    // Normalise into W = T(slot); squared norms into Sig.
    double *W = ws.T(s);
    double *sig = ws.Sig(s);
    for (int c = warp; c < cols; c += kWarps) {
        const double *ca = A + (size_t)c * lda;
        double nrm = 0.0;
        for (int i = lane; i < rows; i += 32) nrm = fma(ca[i], ca[i], nrm);
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
        const double inv = nrm > 0.0 ? 1.0 / sqrt(nrm) : 0.0;
        for (int i = lane; i < rows; i += 32) W[(size_t)c * ldg + i] = ca[i] * inv;
        if (lane == 0) sig[c] = nrm;
    }
    if (threadIdx.x == 0) {
        tw.sweeps = sweep;
        if (sweep >= 40) tw.status |= TILE_JACOBI_SLOW;
    }
}

// Block one-sided Jacobi for the classes whose factor does not fit in
// shared memory (k1 <= 512).  The k2 columns form blocks of B = 512 / G;
// the blocks meet in a round-robin tournament, and each meeting brings the
// block pair (2B columns, 164 KB at most) into shared memory, rotates the
// B^2 column pairs across the two blocks there (B steps of B disjoint
// pairs, one group of G lanes per pair, E rows per lane) and writes it
// back; the pairs inside each block are rotated in the tournament's first
// round.  A sweep (one tournament) thus rotates every pair once, as the
// cyclic order does, but every rotation reads shared memory instead of L2
// and global traffic is a few copies of the factor per sweep.  Sweeps
// repeat until one rotates nothing.
//
// The meetings of one round touch disjoint blocks, so a tile is taken by a
// cluster of CTAs (jacobi_cluster) that share each round's meetings and meet
// at a cluster barrier between rounds (which also publishes the round's
// columns in global memory): a tile's latency, which is what bounds the
// batches that hold few such tiles, drops by up to that factor.  Times
// (for the convergence bookkeeping) count the steps of a round once,
// whichever CTA runs a meeting: round 0 takes steps [0, 2B - 1) (B - 1
// within blocks, B across), round r > 0 the B steps from B - 1 + r B; a
// column is only rotated by the one meeting of a round that holds it.
// lastrot lives in the slot's Sig buffer during the iteration (the
// normalisation overwrites it at the end), each meeting works on its own
// copy of its columns' entries.  Data another CTA of the cluster wrote is
// read past L1 (__ldcg).
constexpr int kJacobiClusterMax = 8;

// CTAs per tile: 4 for the classes above 256 rows and for every block
// class of a batch that holds such factors (kmax > 256: its large tiles
// bound the batch), 2 otherwise (measured: on batches whose factors stay
// below 257 rows, 4 CTAs per tile take SMs from the shared-memory classes
// beside them and lose, on batches with larger factors they win);
// STARSH_B200_JACOBI_CLUSTER (1 .. 8) sets one size for all.
static int jacobi_cluster(int cls, int kmax)
{
    static const int forced = [] {
        int v = 0;
        if (const char *e = getenv("STARSH_B200_JACOBI_CLUSTER"))
            v = std::max(1, std::min(kJacobiClusterMax, atoi(e)));
        return v;
    }();
    return forced ? forced : (cls >= 7 || kmax > 256) ? 4 : 2;
}

template <int CLASS, int G, int E>
__global__ void __launch_bounds__(512, 1)
k_jacobi_block(TileWork *__restrict__ tiles, Workspace ws)
{
    constexpr int THREADS = 512;
    constexpr int B = THREADS / G;          // columns per block, pairs per step
    constexpr int P2 = 2 * B;               // columns in shared memory
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int crank = (int)cl.block_rank(), csize = (int)cl.num_blocks();
    extern __shared__ double sm[];
    __shared__ int rotated[2];              // in the cluster's first CTA
    __shared__ int lr[P2];                  // lastrot of the meeting's slots
    TileWork &tw = tiles[blockIdx.x / csize];
    const int s = tw.slot;
    const int rows = tw.k1, cols = tw.k2;
    if (cols <= 0 || jacobi_class(rows, cols) != CLASS) return;   // cluster-uniform
    const double eps = fmax(1e-15, fmin(1e-7, 0.01 * tw.tol));
    const double eps2 = eps * eps;
    const int ldg = ws.ldK();
    double *Lg = ws.L(s);
    int *lastrot = (int *)ws.Sig(s);
    int *rot0 = cl.map_shared_rank(rotated, 0);
    const int lds = rows | 1;
    const int nb = (cols + B - 1) / B;
    const int nbp = nb + (nb & 1);          // blocks, with a bye if odd
    const int gw = threadIdx.x / G, gl = threadIdx.x % G;
    for (int c = crank * THREADS + threadIdx.x; c < cols; c += csize * THREADS)
        lastrot[c] = -1;
    if (crank == 0 && threadIdx.x == 0) rotated[0] = rotated[1] = 0;
    cl.sync();
    auto column = [&](int q, int bi, int bj) {   // global column of slot q
        return q < B ? bi * B + q : bj * B + q - B;
    };
    const int T = (B - 1) + (nbp - 1) * B;      // steps per sweep
    int sweep = 0;
    for (; sweep < 40; ++sweep) {
        bool any = false;
        for (int rnd = 0; rnd < nbp - 1; ++rnd) {
            const int t0 = sweep * T + (rnd == 0 ? 0 : B - 1 + rnd * B);
            for (int pr = crank; pr < nbp / 2; pr += csize) {
                // block pair pr of round rnd (circle method, as for columns)
                int x = pr - 1 + rnd, y = nbp - 2 - pr + rnd;
                if (x >= nbp - 1) x -= nbp - 1;
                if (y >= nbp - 1) y -= nbp - 1;
                const int bi = pr == 0 ? 0 : 1 + x, bj = 1 + y;
                // Each block's own pairs are rotated once per sweep, in the
                // first round (where every block meets exactly one other,
                // or the bye); every meeting rotates the B^2 pairs across
                // its two blocks.
                const bool bye = bi >= nb || bj >= nb;
                if (bye && rnd > 0) continue;                   // uniform
                const int b0 = bye ? (bi < nb ? bi : bj) : bi;  // slots 0 .. B-1
                const int b1 = bye ? nb : bj;                   // slots B .. 2B-1
                const int nslots = bye ? B : P2;
                // A meeting none of whose columns has been rotated since
                // its previous occurrence (T steps ago, when all its pairs
                // were found orthogonal) is skipped with its copies.
                int hot = 0;
                for (int q = threadIdx.x; q < P2; q += THREADS) {
                    const int c = q < nslots ? column(q, b0, b1) : cols;
                    lr[q] = c < cols ? __ldcg(lastrot + c) : -1;
                    if (c < cols && lr[q] >= t0 - T) hot = 1;
                }
                if (!__syncthreads_or(hot)) continue;
                for (int e = threadIdx.x; e < nslots * rows; e += THREADS) {
                    const int q = e / rows, i = e - q * rows;
                    const int c = column(q, b0, b1);
                    sm[(size_t)q * lds + i] = c < cols ? __ldcg(Lg + (size_t)c * ldg + i) : 0.0;
                }
                __syncthreads();
                int now = t0;
                if (rnd == 0) {
                    // round-robin over the B columns of each block, B / 2
                    // pairs per block and step (groups B / 2 .. B - 1 take
                    // block b1, idle at the bye)
                    const int q = gw % (B / 2), off = gw < B / 2 ? 0 : B;
                    for (int step = 0; step < B - 1; ++step, ++now) {
                        int u = q - 1 + step, v = B - 2 - q + step;
                        if (u >= B - 1) u -= B - 1;
                        if (v >= B - 1) v -= B - 1;
                        const int a = off + (q == 0 ? 0 : 1 + u), b = off + 1 + v;
                        const bool valid = (off == 0 || !bye) &&
                                           column(a, b0, b1) < cols &&
                                           column(b, b0, b1) < cols &&
                                           !jacobi_unchanged(lr, a, b, now - T);
                        if (__any_sync(0xffffffffu, valid)) {
                            const bool rot = jacobi_rotate<G, E>(
                                sm + (size_t)a * lds, sm + (size_t)b * lds, rows,
                                gl, valid, eps2);
                            if (rot && gl == 0) lr[a] = lr[b] = now;
                            any |= rot;
                        }
                        __syncthreads();
                    }
                }
                if (!bye) {
                    // the cross pairs: slot gw with slot B + (gw + step) mod B
                    for (int step = 0; step < B; ++step, ++now) {
                        const int a = gw, b = B + (gw + step) % B;
                        const bool valid = column(a, b0, b1) < cols &&
                                           column(b, b0, b1) < cols &&
                                           !jacobi_unchanged(lr, a, b, now - T);
                        if (__any_sync(0xffffffffu, valid)) {
                            const bool rot = jacobi_rotate<G, E>(
                                sm + (size_t)a * lds, sm + (size_t)b * lds, rows,
                                gl, valid, eps2);
                            if (rot && gl == 0) lr[a] = lr[b] = now;
                            any |= rot;
                        }
                        __syncthreads();
                    }
                }
                for (int e = threadIdx.x; e < nslots * rows; e += THREADS) {
                    const int q = e / rows, i = e - q * rows;
                    const int c = column(q, b0, b1);
                    if (c < cols) Lg[(size_t)c * ldg + i] = sm[(size_t)q * lds + i];
                }
                for (int q = threadIdx.x; q < nslots; q += THREADS) {
                    const int c = column(q, b0, b1);
                    if (c < cols) lastrot[c] = lr[q];
                }
                __syncthreads();
            }
            // the round's columns and times, visible to the whole cluster
            cl.sync();
        }
        if (any) rot0[sweep & 1] = 1;
        if (crank == 0 && threadIdx.x == 0) rotated[(sweep + 1) & 1] = 0;
        cl.sync();
        if (!rot0[sweep & 1]) break;
    }
    // every CTA has read the first CTA's flag before any of them exits
    cl.sync();
    // Normalise into W = T(slot); squared norms into Sig (over lastrot).
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *W = ws.T(s);
    double *sig = ws.Sig(s);
    for (int c = crank * (THREADS / 32) + warp; c < cols;
         c += csize * (THREADS / 32)) {
        const double *ca = Lg + (size_t)c * ldg;
        double nrm = 0.0;
        for (int i = lane; i < rows; i += 32) {
            const double x = __ldcg(ca + i);
            nrm = fma(x, x, nrm);
        }
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
        const double inv = nrm > 0.0 ? 1.0 / sqrt(nrm) : 0.0;
        for (int i = lane; i < rows; i += 32) W[(size_t)c * ldg + i] = __ldcg(ca + i) * inv;
        if (lane == 0) sig[c] = nrm;
    }
    if (crank == 0 && threadIdx.x == 0) {
        tw.sweeps = sweep;
        if (sweep >= 40) tw.status |= TILE_JACOBI_SLOW;
    }
}

template <int CLASS, int G, int E>
static void jacobi_block_launch(TileWork *d_tiles, int ntiles, Workspace ws,
                                int max_rows, cudaStream_t stream)
{
    const int kmax = ws.k_max;
    auto *fn = k_jacobi_block<CLASS, G, E>;
    const size_t smem = (size_t)2 * (512 / G) * (max_rows | 1) * sizeof(double);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    cudaLaunchConfig_t cfg = {};
    const int cs = jacobi_cluster(CLASS, kmax);
    cfg.gridDim = dim3((unsigned)(ntiles * cs));
    cfg.blockDim = dim3(512);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, fn, d_tiles, ws);
}

template <int CLASS, int G, int E, int THREADS, bool SMEM>
static void jacobi_class_launch(TileWork *d_tiles, int ntiles, Workspace ws,
                                size_t smem, cudaStream_t stream)
{
    auto *fn = k_jacobi<CLASS, G, E, THREADS, SMEM>;
    if (SMEM && smem > 48 * 1024)
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    fn<<<ntiles, THREADS, SMEM ? smem : 0, stream>>>(d_tiles, ws);
}

int launch_jacobi(TileWork *d_tiles, int ntiles, Workspace ws,
                  cudaStream_t stream, cudaStream_t side)
{
    // Classes a batch can reach, from the largest factor it may hold
    // (k1, k2 <= k_max).  Shared memory is sized for the class's largest
    // tile that fits.
    const int kmax = ws.k_max;
    auto smem_for = [&](int rows) {
        const int r = std::min(rows, kmax);
        const size_t full = (size_t)(r | 1) * std::min(r, kmax) * sizeof(double);
        return std::min(full, kJacobiSmemMax);
    };
    // The block classes (one CTA per SM, long-running) run on `side`, the
    // others on `stream`, overlapping them.
    cudaStream_t big = side ? side : stream;
    cudaEvent_t fork = nullptr, join = nullptr;
    if (side && kmax > 64) {
        cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
        cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
        cudaEventRecord(fork, stream);
        cudaStreamWaitEvent(side, fork, 0);
    }
    // the block classes (factor in global memory) on `side`; the classes
    // whose factor sits in shared memory on `stream`, filling the SMs the
    // last wave of the block classes leaves idle
    if (kmax > 128)
        jacobi_block_launch<4, 16, 12>(d_tiles, ntiles, ws,
                                       std::min(kmax, 192), big);
    if (kmax > 192)
        jacobi_block_launch<6, 16, 16>(d_tiles, ntiles, ws,
                                       std::min(kmax, 256), big);
    if (kmax > 256)
        jacobi_block_launch<7, 16, 18>(d_tiles, ntiles, ws,
                                       std::min(kmax, 288), big);
    if (kmax > 288)
        jacobi_block_launch<8, 16, 20>(d_tiles, ntiles, ws,
                                       std::min(kmax, 320), big);
    if (kmax > 320)
        jacobi_block_launch<9, 32, 16>(d_tiles, ntiles, ws,
                                       std::min(kmax, 512), big);
    if (kmax > 512)
        jacobi_class_launch<10, 32, 0, 1024, false>(d_tiles, ntiles, ws, 0,
                                                    big);
    if (kmax > 192)
        jacobi_class_launch<5, 16, 16, 512, true>(d_tiles, ntiles, ws,
                                                  smem_for(256), stream);
    if (kmax > 128)
        jacobi_class_launch<3, 16, 12, 512, true>(d_tiles, ntiles, ws,
                                                  smem_for(192), stream);
    if (kmax > 64)
        jacobi_class_launch<2, 8, 16, 512, true>(d_tiles, ntiles, ws,
                                                 smem_for(128), stream);
    jacobi_class_launch<0, 4, 8, 64, true>(d_tiles, ntiles, ws,
                                           smem_for(32), stream);
    if (kmax > 32)
        jacobi_class_launch<1, 4, 16, 128, true>(d_tiles, ntiles, ws,
                                                 smem_for(64), stream);
    if (fork) {
        cudaEventRecord(join, side);
        cudaStreamWaitEvent(stream, join, 0);
        cudaEventDestroy(fork);
        cudaEventDestroy(join);
    }
    return 1 + (kmax > 32) + (kmax > 64) + 2 * (kmax > 128) + 2 * (kmax > 192) +
           (kmax > 256) + (kmax > 288) + (kmax > 320) + (kmax > 512);
}

// Appends the residual-pass columns to the basis: k1 += kb.
__global__ void k_merge_basis(TileWork *__restrict__ tiles, int ntiles)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ntiles && tiles[t].kb > 0) {
        tiles[t].k1 += tiles[t].kb;
        tiles[t].kb = 0;
    }
}

void launch_merge_basis(TileWork *d_tiles, int ntiles, cudaStream_t stream)
{
    k_merge_basis<<<(ntiles + 127) / 128, 128, 0, stream>>>(d_tiles, ntiles);
}

// --------------------------------------------------------- rank cut

// Energies e_c = ||C(c, :)||^2 of the rotated rows, order by decreasing
// energy, then the smallest r >= 1 with
//   sum_{c >= r} e_c + tail_h + outside  <=  tol^2 ||D||_F^2,
// i.e. starsh_dense_dsvfr applied to the exact energies plus the energy the
// Gram factor (tail_h) and the sketch (outside) left out (0 if D = 0).
// rank = r if r <= maxrank, else -1.
__global__ void __launch_bounds__(kSmallThreads)
k_rank_cut(TileWork *__restrict__ tiles, Workspace ws)
{
    TileWork &tw = tiles[blockIdx.x];
    const int s = tw.slot;
    const int k2 = tw.k2;
    const double tol = tw.tol;
    const int maxrank = tw.maxrank;
    __shared__ double e[kMaxK];
    __shared__ int ord[kMaxK];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double *C = ws.C(s);
    const int ld = ws.ldK();
    for (int c = warp; c < k2; c += blockDim.x >> 5) {
        double acc = 0.0;
        for (int j = lane; j < tw.n; j += 32) {
            const double v = C[(size_t)j * ld + c];
            acc += v * v;
        }
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) e[c] = acc;
    }
    __syncthreads();
    // Position of c = number of entries ranked before it.
    for (int c = threadIdx.x; c < k2; c += blockDim.x) {
        int pos = 0;
        const double ec = e[c];
        for (int o = 0; o < k2; ++o)
            pos += (e[o] > ec) || (e[o] == ec && o < c);
        ord[pos] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int *gord = ws.Ord(s);
        double *ge = ws.E(s);
        double total = 0.0;
        for (int c = 0; c < k2; ++c) {
            gord[c] = ord[c];
            ge[c] = e[ord[c]];
            total += e[c];
        }
        // With the block's exact ||D||_F^2 (dnorm2, from the generator) the
        // energy outside the sketched basis, ||D||^2 - ||B||^2, is known
        // too: it joins the tail, less an allowance for the rounding of the
        // two sums, and the budget is tol^2 ||D||^2.  A block whose
        // outside energy alone exceeds the budget cannot meet tol with its
        // sketch: it is stored dense (rank -1), like a block above maxrank.
        // Without dnorm2 (dense tiles given by the caller) the rule is the
        // reference's: the tail of the projected block's spectrum against
        // tol^2 ||B||^2.
        const double dn = tw.dnorm2;
        const double outside = dn > 0.0
            ? fmax(0.0, dn - tw.tr_h - 2e-15 * dn) : 0.0;
        const double energy = dn > 0.0 ? fmax(dn, tw.tr_h) : tw.tr_h;
        int r;
        if (!(energy > 0.0) || k2 == 0) {
            r = outside <= tol * tol * energy ? 0 : -1;
        } else {
            const double budget = tol * tol * energy;
            // energy outside span(W): what the Gram factor left out
            const double missing = fmax(0.0, tw.tail_h) + outside;
            // tail(r) for r = k2 down to 1; keep the smallest r that fits
            double tail = missing;
            r = -1;
            if (tail <= budget) r = k2;
            for (int c = k2 - 1; c >= 1; --c) {
                tail += ge[c];
                if (tail <= budget) r = c;
                else break;
            }
            if (r < 0) tw.status |= TILE_TAIL_LEFT;
        }
        tw.rank = r <= maxrank ? r : -1;
    }
}

void launch_rank_cut(TileWork *d_tiles, int ntiles, Workspace ws,
                     cudaStream_t stream)
{
    k_rank_cut<<<ntiles, kSmallThreads, 0, stream>>>(d_tiles, ws);
}

// Wsel(:, c) = W(:, ord[c]) for c < rank, into L(slot).
__global__ void k_select_w(const TileWork *__restrict__ tiles, Workspace ws)
{
    const TileWork tw = tiles[blockIdx.x];
    if (tw.rank <= 0) return;
    const int s = tw.slot, ld = ws.ldK();
    const int *ord = ws.Ord(s);
    const double *W = ws.T(s);
    double *dst = ws.L(s);
    for (int c = 0; c < tw.rank; ++c)
        for (int i = threadIdx.x; i < tw.k1; i += blockDim.x)
            dst[(size_t)c * ld + i] = W[(size_t)ord[c] * ld + i];
}

void launch_select_w(const TileWork *d_tiles, int ntiles, Workspace ws,
                     cudaStream_t stream)
{
    k_select_w<<<ntiles, 256, 0, stream>>>(d_tiles, ws);
}

// V(j, c) = C(ord[c], j): V is n x rank, leading dimension n.  A CTA
// transposes `cols` (8, 16 or 32) columns j of C at a time through shared
// memory: it reads the k2 rows of those columns (contiguous in C) and
// writes the rank selected rows as `cols` consecutive entries of each
// column of V, so both sides are coalesced.
__global__ void __launch_bounds__(256)
k_write_v(const TileWork *__restrict__ tiles, Workspace ws, OutArena out,
          int cols)
{
    extern __shared__ double wv_sm[];   // [cols][k2 + 1]
    const TileWork tw = tiles[blockIdx.x];
    if (tw.rank <= 0) return;
    const int s = tw.slot, ld = ws.ldK();
    const int *ord = ws.Ord(s);
    const double *C = ws.C(s);
    double *V = out.V + tw.off_v;
    const int kr = tw.k2, ls = kr + 1;   // rows of C; ord[c] < k2
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int j0 = blockIdx.y * cols; j0 < tw.n; j0 += gridDim.y * cols) {
        const int nj = min(cols, tw.n - j0);
        // warp w reads columns j0 + w, j0 + w + 8, ...: k2 contiguous rows
        for (int jj = warp; jj < nj; jj += 8)
            for (int i = lane; i < kr; i += 32)
                wv_sm[jj * ls + i] = C[(size_t)(j0 + jj) * ld + i];
        __syncthreads();
        for (int c = warp; c < tw.rank; c += 8) {
            const int row = ord[c];
            if (lane < nj) V[(size_t)c * tw.n + j0 + lane] = wv_sm[lane * ls + row];
        }
        __syncthreads();
    }
}

void launch_write_v(const TileWork *d_tiles, int ntiles, Workspace ws,
                    OutArena out, cudaStream_t stream)
{
    // 32 columns per pass while the tile fits 96 KB, fewer for wide bases
    int cols = 32;
    while (cols > 8 && (size_t)cols * (ws.k_max + 1) * sizeof(double) > 96 * 1024)
        cols /= 2;
    const size_t smem = (size_t)cols * (ws.k_max + 1) * sizeof(double);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_write_v, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    dim3 grid(ntiles, 8);
    k_write_v<<<grid, 256, smem, stream>>>(d_tiles, ws, out, cols);
}

}  // namespace b200
