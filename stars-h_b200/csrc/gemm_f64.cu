// Batched FP64 GEMM (see gemm_f64.cuh).
//
// CTA tile 64 x 64, 32 x 128 or 128 x 32, K step 16, 8 warps of 32 x 16
// output each (4 x 2 fragments of the m8n8k4 DMMA).  Operand tiles are staged
// in shared memory double-buffered, the next K tile is fetched into
// registers while the current one is multiplied.  Global loads are
// coalesced along whichever dimension is contiguous for the given transpose
// flag, and the staging layout follows it: [row][k] with row stride 20 where
// k is contiguous, [k][row] with stride rows + 4 where rows are, so that
// both the stores and the fragment reads are free of bank conflicts.  Warps
// skip the DMMAs of output regions outside the tile's own M x N and of k4
// steps past its K (those would add exact zeros).
#include <cstdint>
#include <mutex>
#include "gemm_f64.cuh"

namespace b200 {

__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a,
                                           double b)
{
    asm volatile(
        "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 "
        "{%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}

// The A B products (basis updates with K <= 64 and beta updates) keep
// three CTAs per SM: their short K makes them latency-bound.
template <bool TA, bool TB, int BM, int BN>
__global__ void __launch_bounds__(kGemmThreads, (!TA && !TB) ? 3 : 0)
k_gemm_f64(const GemmDesc *__restrict__ descs, int tiles_n)
{
    // 8 warps of 32 x 16 output each, BM / 32 along M and BN / 16 along N
    constexpr int WARPS_M = BM / 32;
    static_assert(WARPS_M * (BN / 16) == kGemmThreads / 32, "warp grid");
    constexpr int RA = BM * kGemmBK / kGemmThreads;   // A loads per thread
    constexpr int RB = BN * kGemmBK / kGemmThreads;   // B loads per thread
    const GemmDesc d = descs[blockIdx.y];
    const int tm = blockIdx.x / tiles_n;
    const int tn = blockIdx.x % tiles_n;
    const int m0 = tm * BM, n0 = tn * BN;
    if (m0 >= d.M || n0 >= d.N) return;

    // [2][BM * kGemmLds] then [2][BN * kGemmLds], dynamic (above 48 KB
    // for the 32 x 128 and 128 x 32 shapes)
    extern __shared__ double gemm_smem[];
    double (*As)[BM * kGemmLds] = reinterpret_cast<double (*)[BM * kGemmLds]>(gemm_smem);
    double (*Bs)[BN * kGemmLds] =
        reinterpret_cast<double (*)[BN * kGemmLds]>(gemm_smem + 2 * BM * kGemmLds);

    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = (warp % WARPS_M) * 32;   // warp row offset in the CTA tile
    const int wn = (warp / WARPS_M) * 16;   // warp column offset

    double acc[4][2][2];
    #pragma unroll
    for (int i = 0; i < 4; ++i)
        #pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    double ra[RA], rb[RB];
    // Element e = t + 256 r of a tile, laid out along whichever dimension
    // is contiguous in global memory (coalesced loads):
    //   A: !TA rows fastest, TA k fastest;  B: !TB k fastest, TB cols fastest.
    auto a_coord = [&](int r, int &row, int &kk) {
        const int e = t + kGemmThreads * r;
        if (!TA) { row = e % BM; kk = e / BM; }
        else     { kk = e % kGemmBK; row = e / kGemmBK; }
    };
    auto b_coord = [&](int r, int &col, int &kk) {
        const int e = t + kGemmThreads * r;
        if (!TB) { kk = e % kGemmBK; col = e / kGemmBK; }
        else     { col = e % BN; kk = e / BN; }
    };
    auto load_tiles = [&](int k0) {
        #pragma unroll
        for (int r = 0; r < RA; ++r) {
            int row, kk;
            a_coord(r, row, kk);
            const int gm = m0 + row, gk = k0 + kk;
            double v = 0.0;
            if (gm < d.M && gk < d.K)
                v = TA ? d.A[(size_t)gm * d.lda + gk]
                       : d.A[(size_t)gk * d.lda + gm];
            ra[r] = v;
        }
        #pragma unroll
        for (int r = 0; r < RB; ++r) {
            int col, kk;
            b_coord(r, col, kk);
            const int gn = n0 + col, gk = k0 + kk;
            double v = 0.0;
            if (gn < d.N && gk < d.K)
                v = TB ? d.B[(size_t)gk * d.ldb + gn]
                       : d.B[(size_t)gn * d.ldb + gk];
            rb[r] = v;
        }
    };
    // shared-memory index of (row, k) of A and (col, k) of B
    constexpr int LDA_K = BM + 4, LDB_K = BN + 4;   // [k][row] strides
    auto a_at = [](int row, int kk) {
        return TA ? row * kGemmLds + kk : kk * LDA_K + row;
    };
    auto b_at = [](int col, int kk) {
        return TB ? kk * LDB_K + col : col * kGemmLds + kk;
    };
    auto store_tiles = [&](int buf) {
        #pragma unroll
        for (int r = 0; r < RA; ++r) {
            int row, kk;
            a_coord(r, row, kk);
            As[buf][a_at(row, kk)] = ra[r];
        }
        #pragma unroll
        for (int r = 0; r < RB; ++r) {
            int col, kk;
            b_coord(r, col, kk);
            Bs[buf][b_at(col, kk)] = rb[r];
        }
    };

    const int ktiles = (d.K + kGemmBK - 1) / kGemmBK;
    if (ktiles > 0) {
        load_tiles(0);
        store_tiles(0);
        __syncthreads();
    }
    // this warp's 32 x 16 output region holds part of the tile's M x N
    const bool live = m0 + wm < d.M && n0 + wn < d.N;
    for (int kt = 0; kt < ktiles; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < ktiles) load_tiles((kt + 1) * kGemmBK);
        // k4 steps of this warp in the K step (warp-uniform; A B products
        // only, the other forms keep every step)
        const int kend = (TA || TB) ? kGemmBK
                         : live ? min(kGemmBK, d.K - kt * kGemmBK) : 0;
        #pragma unroll
        for (int kk = 0; kk < kGemmBK; kk += 4) {
            if (kk >= kend) break;
            double af[4], bf[2];
            #pragma unroll
            for (int i = 0; i < 4; ++i)
                af[i] = As[buf][a_at(wm + i * 8 + g, kk + tig)];
            #pragma unroll
            for (int j = 0; j < 2; ++j)
                bf[j] = Bs[buf][b_at(wn + j * 8 + g, kk + tig)];
            #pragma unroll
            for (int i = 0; i < 4; ++i)
                #pragma unroll
                for (int j = 0; j < 2; ++j)
                    dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
        if (kt + 1 < ktiles) {
            store_tiles(buf ^ 1);
        }
        __syncthreads();
    }

    // Accumulator (i, j, h) holds C(wm + 8i + g, wn + 8j + 2 tig + h).
    // With beta != 0 the old C values are all read before the first store
    // (the stores may alias later loads, so loads interleaved with them
    // would each wait a full memory round trip).
    double cold[4][2][2];
    const bool upd = d.beta != 0.0;
    if (upd) {
        #pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int gm = m0 + wm + i * 8 + g;
            #pragma unroll
            for (int j = 0; j < 2; ++j) {
                #pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int gn = n0 + wn + j * 8 + 2 * tig + h;
                    cold[i][j][h] = gm < d.M && gn < d.N
                                        ? d.C[(size_t)gn * d.ldc + gm] : 0.0;
                }
            }
        }
    }
    #pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + wm + i * 8 + g;
        if (gm >= d.M) continue;
        #pragma unroll
        for (int j = 0; j < 2; ++j) {
            #pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gn = n0 + wn + j * 8 + 2 * tig + h;
                if (gn >= d.N) continue;
                double *c = d.C + (size_t)gn * d.ldc + gm;
                double v = d.alpha * acc[i][j][h];
                if (upd) v += d.beta * cold[i][j][h];
                *c = v;
            }
        }
    }
}

// A^T B with 64 x 64 or 32 x 128 CTA tiles and a three-stage cp.async
// pipeline: the transposed products (Grams and projections onto the basis
// in the rounds; the projection B = Q^T D and rotation C = W^T B of the
// small SVD, 32 x 128) have outputs of a few tiles and K = the tile
// height, so one CTA walks a long K; the register-staged kernel above keeps
// one K step in flight and waits on memory latency every step.  Operand
// tiles land in shared memory directly (16-byte cp.async, k contiguous in
// both operands), two steps ahead of the multiply (60 or 75 KB of shared
// memory).  Where a tile fills every warp's output region, the per-element
// accumulation order is that of k_gemm_f64 (K steps of 16 in order, the
// DMMA's k-order inside a step), so results are identical to it; in a
// launch that asks for it (split_k), a 64 x 64 tile with at most 32 rows or
// 48 columns of its own splits K over the spare warps (fixed slice order,
// deterministic).
#ifndef GEMM_TN_STAGES
#define GEMM_TN_STAGES 3      // four measured slower on the projection
#endif
constexpr int kTnStages = GEMM_TN_STAGES;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool pred)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    const int n = pred ? 16 : 0;   // zero-fill when outside the operand
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;"
                 :: "r"(sa), "l"(gmem), "r"(n));
}

template <int BM, int BN>
__global__ void __launch_bounds__(kGemmThreads)
k_gemm_f64_tn_pipe(const GemmDesc *__restrict__ descs, int tiles_n, int split_k)
{
    constexpr int WARPS_M = BM / 32;
    static_assert(WARPS_M * (BN / 16) == kGemmThreads / 32, "warp grid");
    // 16-byte pieces of the two operand tiles (BM and BN rows of 16 k)
    constexpr int PA = BM * kGemmBK / 2, PIECES = (BM + BN) * kGemmBK / 2;
    const GemmDesc d = descs[blockIdx.y];
    const int tm = blockIdx.x / tiles_n, tn = blockIdx.x % tiles_n;
    const int m0 = tm * BM, n0 = tn * BN;
    if (m0 >= d.M || n0 >= d.N) return;
    extern __shared__ double gemm_smem[];
    // [stage][64 rows][kGemmLds] for A^T, then the same for B^T
    double *As = gemm_smem;
    double *Bs = gemm_smem + kTnStages * BM * kGemmLds;
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tig = lane & 3;
    // Output regions of 32 x 16, one per warp when the tile's own rows and
    // columns fill the CTA tile.  A 64 x 64 tile with fewer (the products
    // onto a narrow basis, Grams of a few columns) gives the spare warps a
    // share of K instead: nreg regions (rounded up to rp, a power of two),
    // warp w works on region w % rp over the k4 steps q = w / rp modulo
    // nsl = 8 / rp, and the nsl partial sums are added in slice order
    // through shared memory.  Every scheduler keeps the same share of the
    // DMMA work.
    int rh = WARPS_M, rp = 8, nsl = 1;
    if constexpr (BM == 64 && BN == 64) if (split_k) {
        rh = d.M - m0 > 32 ? 2 : 1;
        const int cq = min(4, (d.N - n0 + 15) / 16);
        const int nreg = rh * cq;
        rp = nreg <= 1 ? 1 : nreg <= 2 ? 2 : nreg <= 4 ? 4 : 8;
        nsl = 8 / rp;
    }
    const int reg = warp % rp, slice = warp / rp;
    const int wm = (reg % rh) * 32, wn = (reg / rh) * 16;
    const bool live = wm < BM && wn < BN && m0 + wm < d.M && n0 + wn < d.N;
    double acc[4][2][2];
    #pragma unroll
    for (int i = 0; i < 4; ++i)
        #pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    // the A tile (BM rows x 16 k) is pieces 0 .. PA - 1, the B tile (BN
    // rows) the rest; thread t copies pieces t, t + 256, ... (row = piece
    // / 8 within its tile, k pair = piece % 8)
    const bool evenA = (d.lda & 1) == 0 && ((uintptr_t)d.A & 15) == 0;
    const bool evenB = (d.ldb & 1) == 0 && ((uintptr_t)d.B & 15) == 0;
    auto issue = [&](int kt) {
        const int st = kt % kTnStages, k0 = kt * kGemmBK;
        #pragma unroll
        for (int r = 0; r < PIECES / kGemmThreads; ++r) {
            const int piece = t + kGemmThreads * r;
            if (piece < PA) {
                const int row = piece >> 3, kk = (piece & 7) * 2;
                const int gm = m0 + row, gk = k0 + kk;
                double *dst = As + (st * BM + row) * kGemmLds + kk;
                if (evenA && gm < d.M && gk + 1 < d.K) {
                    cp_async16(dst, d.A + (size_t)gm * d.lda + gk, true);
                } else {
                    dst[0] = (gm < d.M && gk < d.K) ? d.A[(size_t)gm * d.lda + gk] : 0.0;
                    dst[1] = (gm < d.M && gk + 1 < d.K) ? d.A[(size_t)gm * d.lda + gk + 1] : 0.0;
                }
            } else {
                const int q = piece - PA;
                const int row = q >> 3, kk = (q & 7) * 2;
                const int gn = n0 + row, gk = k0 + kk;
                double *dst = Bs + (st * BN + row) * kGemmLds + kk;
                if (evenB && gn < d.N && gk + 1 < d.K) {
                    cp_async16(dst, d.B + (size_t)gn * d.ldb + gk, true);
                } else {
                    dst[0] = (gn < d.N && gk < d.K) ? d.B[(size_t)gn * d.ldb + gk] : 0.0;
                    dst[1] = (gn < d.N && gk + 1 < d.K) ? d.B[(size_t)gn * d.ldb + gk + 1] : 0.0;
                }
            }
        }
        asm volatile("cp.async.commit_group;");
    };
    const int ktiles = (d.K + kGemmBK - 1) / kGemmBK;
    #pragma unroll
    for (int p = 0; p < kTnStages - 1; ++p) {
        if (p < ktiles) issue(p);
        else asm volatile("cp.async.commit_group;");
    }
    for (int kt = 0; kt < ktiles; ++kt) {
        // the group of step kt has landed (at most kTnStages - 2 newer ones
        // still in flight)
        asm volatile("cp.async.wait_group %0;" :: "n"(kTnStages - 2));
        __syncthreads();
        if (kt + kTnStages - 1 < ktiles) issue(kt + kTnStages - 1);
        else asm volatile("cp.async.commit_group;");
        const int st = kt % kTnStages;
        const double *Ab = As + st * BM * kGemmLds;
        const double *Bb = Bs + st * BN * kGemmLds;
        #pragma unroll
        for (int k4 = 0; k4 < kGemmBK / 4; ++k4) {
            // this warp's k4 steps (warp-uniform)
            if (!live || ((kt * (kGemmBK / 4) + k4 - slice) & (nsl - 1)) != 0) continue;
            const int kk = k4 * 4;
            double af[4], bf[2];
            #pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = Ab[(wm + i * 8 + g) * kGemmLds + kk + tig];
            #pragma unroll
            for (int j = 0; j < 2; ++j) bf[j] = Bb[(wn + j * 8 + g) * kGemmLds + kk + tig];
            #pragma unroll
            for (int i = 0; i < 4; ++i)
                #pragma unroll
                for (int j = 0; j < 2; ++j)
                    dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
    }
    asm volatile("cp.async.wait_group 0;");
    if (nsl > 1) {
        // partial sums of the slices, [warp][16 accumulators][32 lanes]
        // over the stage buffers, added by slice 0 in slice order
        __syncthreads();
        double *part = gemm_smem + warp * 512;
        #pragma unroll
        for (int i = 0; i < 4; ++i)
            #pragma unroll
            for (int j = 0; j < 2; ++j)
                #pragma unroll
                for (int h = 0; h < 2; ++h) part[((i * 2 + j) * 2 + h) * 32 + lane] = acc[i][j][h];
        __syncthreads();
        if (slice != 0) return;
        for (int q = 1; q < nsl; ++q) {
            const double *pq = gemm_smem + (warp + q * rp) * 512;
            #pragma unroll
            for (int i = 0; i < 4; ++i)
                #pragma unroll
                for (int j = 0; j < 2; ++j)
                    #pragma unroll
                    for (int h = 0; h < 2; ++h) acc[i][j][h] += pq[((i * 2 + j) * 2 + h) * 32 + lane];
        }
    }
    if (!live) return;
    #pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + wm + i * 8 + g;
        if (gm >= d.M) continue;
        #pragma unroll
        for (int j = 0; j < 2; ++j) {
            #pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gn = n0 + wn + j * 8 + 2 * tig + h;
                if (gn >= d.N) continue;
                double *c = d.C + (size_t)gn * d.ldc + gm;
                double v = d.alpha * acc[i][j][h];
                if (d.beta != 0.0) v += d.beta * *c;
                *c = v;
            }
        }
    }
}

// A B^T with 64 x 64 CTA tiles (the Gram B B^T of the small SVD, K = the
// tile width) through the same three-stage cp.async pipeline as the
// transposed products.  Here rows are contiguous in both operands and k is
// strided, so the tiles are staged as [k][row] (row stride 68 doubles:
// fragment reads free of bank conflicts); a 16-byte piece is two
// consecutive rows at one k.  Without split_k the per-element accumulation
// order is that of k_gemm_f64 (K steps of 16 in order), so results are
// identical to it; with it, K is split over the warps of empty output
// regions as in the transposed kernel.
constexpr int kNtLds = 64 + 4;

__global__ void __launch_bounds__(kGemmThreads)
k_gemm_f64_nt_pipe(const GemmDesc *__restrict__ descs, int tiles_n, int split_k)
{
    constexpr int BM = 64, BN = 64;
    const GemmDesc d = descs[blockIdx.y];
    const int tm = blockIdx.x / tiles_n, tn = blockIdx.x % tiles_n;
    const int m0 = tm * BM, n0 = tn * BN;
    if (m0 >= d.M || n0 >= d.N) return;
    extern __shared__ double gemm_smem[];
    // [stage][16 k][kNtLds] for A, then the same for B
    double *As = gemm_smem;
    double *Bs = gemm_smem + kTnStages * kGemmBK * kNtLds;
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tig = lane & 3;
    // output regions, K slices and 8-row fragments as in the transposed
    // kernel above
    int rh = 2, rp = 8, nsl = 1;
    if (split_k) {
        rh = d.M - m0 > 32 ? 2 : 1;
        const int cq = min(4, (d.N - n0 + 15) / 16);
        const int nreg = rh * cq;
        rp = nreg <= 1 ? 1 : nreg <= 2 ? 2 : nreg <= 4 ? 4 : 8;
        nsl = 8 / rp;
    }
    const int reg = warp % rp, slice = warp / rp;
    const int wm = (reg % rh) * 32, wn = (reg / rh) * 16;
    const bool live = wm < BM && wn < BN && m0 + wm < d.M && n0 + wn < d.N;
    double acc[4][2][2];
    #pragma unroll
    for (int i = 0; i < 4; ++i)
        #pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const bool evenA = (d.lda & 1) == 0 && ((uintptr_t)d.A & 15) == 0;
    const bool evenB = (d.ldb & 1) == 0 && ((uintptr_t)d.B & 15) == 0;
    // pieces 0 .. 511: A (row pair = piece % 32, k = piece / 32), 512 ..
    // 1023: B the same way; thread t copies t, t + 256, t + 512, t + 768
    auto issue = [&](int kt) {
        const int st = kt % kTnStages, k0 = kt * kGemmBK;
        #pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int piece = t + kGemmThreads * r;
            const bool isA = piece < 512;
            const int q = isA ? piece : piece - 512;
            const int row = (q & 31) * 2, kk = q >> 5;
            const int gk = k0 + kk;
            const double *src = isA ? d.A : d.B;
            const int ld = isA ? d.lda : d.ldb;
            const int lim = isA ? d.M : d.N;
            const int g0 = (isA ? m0 : n0) + row;
            double *dst = (isA ? As : Bs) + (st * kGemmBK + kk) * kNtLds + row;
            if ((isA ? evenA : evenB) && g0 + 1 < lim && gk < d.K) {
                cp_async16(dst, src + (size_t)gk * ld + g0, true);
            } else {
                dst[0] = (g0 < lim && gk < d.K) ? src[(size_t)gk * ld + g0] : 0.0;
                dst[1] = (g0 + 1 < lim && gk < d.K) ? src[(size_t)gk * ld + g0 + 1] : 0.0;
            }
        }
        asm volatile("cp.async.commit_group;");
    };
    const int ktiles = (d.K + kGemmBK - 1) / kGemmBK;
    #pragma unroll
    for (int p = 0; p < kTnStages - 1; ++p) {
        if (p < ktiles) issue(p);
        else asm volatile("cp.async.commit_group;");
    }
    for (int kt = 0; kt < ktiles; ++kt) {
        asm volatile("cp.async.wait_group %0;" :: "n"(kTnStages - 2));
        __syncthreads();
        if (kt + kTnStages - 1 < ktiles) issue(kt + kTnStages - 1);
        else asm volatile("cp.async.commit_group;");
        const int st = kt % kTnStages;
        const double *Ab = As + st * kGemmBK * kNtLds;
        const double *Bb = Bs + st * kGemmBK * kNtLds;
        #pragma unroll
        for (int k4 = 0; k4 < kGemmBK / 4; ++k4) {
            if (!live || ((kt * (kGemmBK / 4) + k4 - slice) & (nsl - 1)) != 0) continue;
            const int kk = k4 * 4;
            double af[4], bf[2];
            #pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = Ab[(kk + tig) * kNtLds + wm + i * 8 + g];
            #pragma unroll
            for (int j = 0; j < 2; ++j) bf[j] = Bb[(kk + tig) * kNtLds + wn + j * 8 + g];
            #pragma unroll
            for (int i = 0; i < 4; ++i)
                #pragma unroll
                for (int j = 0; j < 2; ++j)
                    dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
    }
    asm volatile("cp.async.wait_group 0;");
    if (nsl > 1) {
        __syncthreads();
        double *part = gemm_smem + warp * 512;
        #pragma unroll
        for (int i = 0; i < 4; ++i)
            #pragma unroll
            for (int j = 0; j < 2; ++j)
                #pragma unroll
                for (int h = 0; h < 2; ++h) part[((i * 2 + j) * 2 + h) * 32 + lane] = acc[i][j][h];
        __syncthreads();
        if (slice != 0) return;
        for (int q = 1; q < nsl; ++q) {
            const double *pq = gemm_smem + (warp + q * rp) * 512;
            #pragma unroll
            for (int i = 0; i < 4; ++i)
                #pragma unroll
                for (int j = 0; j < 2; ++j)
                    #pragma unroll
                    for (int h = 0; h < 2; ++h) acc[i][j][h] += pq[((i * 2 + j) * 2 + h) * 32 + lane];
        }
    }
    if (!live) return;
    #pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + wm + i * 8 + g;
        if (gm >= d.M) continue;
        #pragma unroll
        for (int j = 0; j < 2; ++j) {
            #pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gn = n0 + wn + j * 8 + 2 * tig + h;
                if (gn >= d.N) continue;
                double *c = d.C + (size_t)gn * d.ldc + gm;
                double v = d.alpha * acc[i][j][h];
                if (d.beta != 0.0) v += d.beta * *c;
                *c = v;
            }
        }
    }
}

template <int BM, int BN>
static void launch_shape(bool ta, bool tb, const GemmDesc *dd, int nb,
                         int tiles_m, int tiles_n, cudaStream_t stream)
{
    dim3 grid(tiles_m * tiles_n, nb);
    const size_t smem = 2 * (size_t)(BM + BN) * kGemmLds * sizeof(double);
    auto go = [&](auto fn) {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        fn<<<grid, kGemmThreads, smem, stream>>>(dd, tiles_n);
    };
    if (!ta && !tb) go(k_gemm_f64<false, false, BM, BN>);
    else if (ta && !tb) go(k_gemm_f64<true, false, BM, BN>);
    else if (!ta && tb) go(k_gemm_f64<false, true, BM, BN>);
    else go(k_gemm_f64<true, true, BM, BN>);
}

cudaError_t gemm_f64_batched(bool ta, bool tb, const GemmDesc *d_desc,
                             int batch, int max_m, int max_n,
                             cudaStream_t stream, bool split_k)
{
    if (batch <= 0 || max_m <= 0 || max_n <= 0) return cudaSuccess;
    split_k = split_k && ta != tb;
    // CTA shape: 64 x 64, or 32 x 128 when the output is wide and (as for
    // the projection B = Q^T D and the rotation C = W^T B) its rows are a
    // basis much narrower than the batch maximum, or 128 x 32 for narrow
    // outputs (sketch blocks of 32 columns); 64 x 64 always with split_k
    int bm = 64, bn = 64;
    if (split_k) { }
    else if (ta && !tb && max_n >= 256) { bm = 32; bn = 128; }
    else if (max_n <= 32 && max_m >= 128) { bm = 128; bn = 32; }
    const int tiles_m = (max_m + bm - 1) / bm;
    const int tiles_n = (max_n + bn - 1) / bn;
    // transposed products (64 x 64 and 32 x 128 tiles): the pipelined kernel
    const bool pipe = ta && !tb && (bm == 64 || bm == 32);
    for (int b0 = 0; b0 < batch; b0 += 65535) {
        const int nb = batch - b0 < 65535 ? batch - b0 : 65535;
        const GemmDesc *dd = d_desc + b0;
        if (pipe) {
            dim3 grid(tiles_m * tiles_n, nb);
            constexpr size_t smem64 = (size_t)kTnStages * 128 * kGemmLds * sizeof(double);
            constexpr size_t smem32 = (size_t)kTnStages * 160 * kGemmLds * sizeof(double);
            static std::once_flag attr;
            std::call_once(attr, [] {
                cudaFuncSetAttribute(k_gemm_f64_tn_pipe<64, 64>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem64);
                cudaFuncSetAttribute(k_gemm_f64_tn_pipe<32, 128>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem32);
            });
            if (bm == 64)
                k_gemm_f64_tn_pipe<64, 64><<<grid, kGemmThreads, smem64, stream>>>(dd, tiles_n, split_k ? 1 : 0);
            else
                k_gemm_f64_tn_pipe<32, 128><<<grid, kGemmThreads, smem32, stream>>>(dd, tiles_n, 0);
        } else if (!ta && tb && bm == 64) {
            dim3 grid(tiles_m * tiles_n, nb);
            constexpr size_t smem = (size_t)kTnStages * 2 * kGemmBK * kNtLds * sizeof(double);
            static std::once_flag attr_nt;
            std::call_once(attr_nt, [] {
                cudaFuncSetAttribute(k_gemm_f64_nt_pipe,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem);
            });
            k_gemm_f64_nt_pipe<<<grid, kGemmThreads, smem, stream>>>(dd, tiles_n, split_k ? 1 : 0);
        } else if (bm == 32) launch_shape<32, 128>(ta, tb, dd, nb, tiles_m, tiles_n, stream);
        else if (bm == 128) launch_shape<128, 32>(ta, tb, dd, nb, tiles_m, tiles_n, stream);
        else launch_shape<64, 64>(ta, tb, dd, nb, tiles_m, tiles_n, stream);
    }
    return cudaGetLastError();
}

}  // namespace b200
