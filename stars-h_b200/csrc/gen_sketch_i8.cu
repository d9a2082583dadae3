// First sampling round of the adaptive engine with the tile generation
// fused in: every entry of a far-field tile is evaluated in registers,
// stored once to the workspace (the projection and later rounds read it)
// and turned, still in registers, into the int8 digits that the tcgen05
// tensor cores multiply by the sketch matrix (the integer Ozaki scheme of
// sketch_i8.cu).  This replaces, for round 0, the generator's D write
// followed by the sketch kernel's D read (reference: the kernel call and
// the first GEMM of src/backends/openmp/blrm/drsdd.c:128-134 with
// src/backends/sequential/dense/drsdd.c:61-62).
//
// Row scales.  The digits of row i are those of x = D_ij 2^-e_i, e_i an
// exponent with |D_ij| < 2^e_i for every j of the tile.  The exact row
// maximum is only known once the row has been generated, so e_i comes from
// an upper bound: the kernel function evaluated at the distance rho_i from
// point i to the nearest of the bounding boxes of the tile's 32-column
// chunks (for the families whose |f| decreases with r; 1/r, sin(kr)/r and
// cos(kr)/r use 1/r and k).  x is rounded to a 48-bit integer (six bytes,
// the top one signed), so a bound up to 2^7 above the true maximum still
// leaves 40 bits.  The generator also computes the exact row maxima; a
// tile where any row's bound fell below its maximum, or more than 2^7
// above it, or where no bound exists, is flagged TILE_RESKETCH and its
// sketch is redone from the stored D by k_sketch_i8 with exact row scales.
//
// Persistent, warp-specialized, one 704-thread CTA per SM over the work
// items (tile, 128-row block):
//   * warp 16 (staging): once, the launch's Omega8 columns (all rows) by
//     TMA into shared memory; per item, the column and row coordinates and
//     point indices of the tile gathered through the cluster pivots, and
//     the bounding box of every 32-column chunk, double-buffered so the
//     next item is staged while the current one is generated;
//   * warps 0-15 (generators): per 32-column chunk, each thread 8 entries
//     of one row: evaluate, store D (coalesced down the columns), sum of
//     squares and row maximum, six digit bytes into a digit buffer;
//   * warp 17 (MMA): six tcgen05.mma.kind::i8 per chunk (M 128, N nc,
//     K 32) into six TMEM accumulators;
//   * warps 18-21 (epilogue): recombine the accumulators exactly (int64)
//     and write Y = 2^(e_i - 47) T.
// Every wait is bounded; after a timeout the CTA marks the tile
// TILE_MMA_TIMEOUT, lets its copies and MMAs in flight finish, and frees
// TMEM.  The generators keep their control flow uniform after a failure
// (they skip the work, not the named barriers).
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include "engine.cuh"
#include "tc_common.cuh"

namespace b200 {

constexpr int kGsSlices = 6;              // 48-bit digits
constexpr int kGsRows = 128;              // rows per item (MMA M)
constexpr int kGsChunk = 32;              // columns per chunk (MMA K)
constexpr int kGsMaxNc = 64;              // sketch columns
constexpr int kGsMaxCols = 1024;          // tile columns staged per item
constexpr int kGsMaxChunks = kGsMaxCols / kGsChunk;
constexpr int kGsMaxDim = 4;
constexpr int kGsAbufs = 2;
#ifndef GS_GEN_WARPS
#define GS_GEN_WARPS 16
#endif
// Generator warps: each thread generates kGsGpt groups of 8 columns of one
// row per chunk (kGsQd threads share a row).
constexpr int kGsGenWarps = GS_GEN_WARPS;
constexpr int kGsGenThreads = 32 * kGsGenWarps;
constexpr int kGsQd = kGsGenThreads / 128;
constexpr int kGsGpt = 4 / kGsQd;
static_assert(kGsQd * kGsGpt == 4, "8-column groups per chunk");
constexpr int kGsStageWarp = kGsGenWarps;
constexpr int kGsMmaWarp = kGsGenWarps + 1;
constexpr int kGsEpiWarp0 = kGsGenWarps + 2;   // four epilogue warps
constexpr int kGsThreads = (kGsGenWarps + 6) * 32;
constexpr int kGsLostBits = 7;            // tolerated looseness of a bound
constexpr int kGsAbufBytes = kGsSlices * kGsRows * kGsChunk;     // 24 KB

// Dynamic shared memory layout (bytes from a 1024-aligned base).
constexpr size_t kGsOffA = 0;
constexpr size_t kGsOffOm = kGsOffA + (size_t)kGsAbufs * kGsAbufBytes;
constexpr size_t kGsOffColc = kGsOffOm + (size_t)kGsMaxCols * kGsMaxNc;
constexpr size_t kGsOffRowc = kGsOffColc + (size_t)2 * kGsMaxDim * kGsMaxCols * 8;
constexpr size_t kGsOffColi = kGsOffRowc + (size_t)2 * kGsMaxDim * kGsRows * 8;
constexpr size_t kGsOffRowi = kGsOffColi + (size_t)2 * kGsMaxCols * 4;
constexpr size_t kGsOffBox = kGsOffRowi + (size_t)2 * kGsRows * 4;
constexpr size_t kGsOffRmax = kGsOffBox + (size_t)2 * kGsMaxChunks * 2 * kGsMaxDim * 8;
constexpr size_t kGsOffRss = kGsOffRmax + (size_t)2 * 4 * kGsRows * 8;
constexpr size_t kGsSmemBytes = kGsOffRss + (size_t)2 * 16 * 8 + 1024;

// The tile fields the kernel reads.
struct GsItem {
    long long row0, col0;
    int m, n, bcur, slot, prob, status;
};

__device__ __forceinline__ GsItem gs_item(const TileWork *tiles, int tile)
{
    const TileWork *w = tiles + tile;
    return GsItem{w->row0, w->col0, w->m, w->n, w->bcur, w->slot, w->prob,
                  w->status};
}

// Digits of 8 entries, given as y = x 2^47 + 1.5 2^52 (x in (-1, 1), one
// rounding): y lies in [2^52, 2^53) and its mantissa field is 2^51 + q,
// q = round(x 2^47), so the low word of y's bit pattern is q mod 2^32 and
// the high word is 0x43380000 + floor(q / 2^32), a 16-bit signed value in
// its low half (0x43380000 has no bits there).  Bytes 0-3 of the low word
// are the unsigned digits 0-3, byte 0 of the high word digit 4 (unsigned)
// and byte 1 the signed top digit 5:
//   q = sum_{s<5} 256^s u_s + 2^40 t_5.
// (Where a row's bound was too small the digits are meaningless; such a
// tile is flagged and sketched again from the stored D.)
__device__ __forceinline__ void digits6(const double (&y)[8],
                                        uint32_t (&w)[kGsSlices][2])
{
    uint32_t lo[8], hi[8];
    #pragma unroll
    for (int c = 0; c < 8; ++c) {
        lo[c] = (uint32_t)__double2loint(y[c]);
        hi[c] = (uint32_t)__double2hiint(y[c]);
    }
    #pragma unroll
    for (int g = 0; g < 2; ++g) {
        #pragma unroll
        for (int s = 0; s < 4; ++s) {
            const uint32_t sel = (uint32_t)s | ((uint32_t)(s + 4) << 4);
            const uint32_t a = __byte_perm(lo[4 * g], lo[4 * g + 1], sel);
            const uint32_t b = __byte_perm(lo[4 * g + 2], lo[4 * g + 3], sel);
            w[s][g] = __byte_perm(a, b, 0x5410);
        }
        #pragma unroll
        for (int s = 0; s < 2; ++s) {
            const uint32_t sel = (uint32_t)s | ((uint32_t)(s + 4) << 4);
            const uint32_t a = __byte_perm(hi[4 * g], hi[4 * g + 1], sel);
            const uint32_t b = __byte_perm(hi[4 * g + 2], hi[4 * g + 3], sel);
            w[4 + s][g] = __byte_perm(a, b, 0x5410);
        }
    }
}

// Upper bound on |f(r)| for every r >= rho (rho2 = rho^2) for the family
// of K; false when the family has none (the tile is then re-sketched).
template <int FAM>
__device__ __forceinline__ bool fam_bound(const DevKernel &K, double rho2,
                                          double &bound)
{
    if constexpr (FAM == FAM_EXP || FAM == FAM_SQREXP || FAM == FAM_MATERN ||
                  FAM == FAM_MATERN2) {
        // positive and decreasing in r (sigma + noise at r = 0)
        bound = fabs(entry_fam<FAM>(K, rho2, 0, 1));
        return true;
    } else if constexpr (FAM == FAM_COULOMB) {
        if (!(rho2 > 0.0)) return false;
        bound = 1.0 / sqrt(rho2);
        return true;
    } else if constexpr (FAM == FAM_SIN) {
        // |sin(kr) / r| <= min(|k|, 1 / r); r = 0 gives diag
        const double k = fabs(K.wave_k);
        bound = fmax(fabs(K.diag), rho2 > 0.0 ? fmin(k, 1.0 / sqrt(rho2)) : k);
        return true;
    } else if constexpr (FAM == FAM_COS) {
        if (!(rho2 > 0.0)) return false;
        bound = fmax(fabs(K.diag), 1.0 / sqrt(rho2));
        return true;
    } else {
        // the decreasing radial bases (Gaussian, exponential, inverse
        // quadratic and multiquadric, the two compactly supported ones)
        const int k = K.rbf_kind;
        if (k == 4 || k == 5 || k == 6 || k == 8) return false;
        bound = fabs(entry_fam<FAM_RBF>(K, rho2, 0, 1));
        return true;
    }
}

__device__ __forceinline__ bool row_bound(const DevKernel &K, double rho2,
                                          double &bound)
{
    switch (K.family) {
    case FAM_EXP: return fam_bound<FAM_EXP>(K, rho2, bound);
    case FAM_SQREXP: return fam_bound<FAM_SQREXP>(K, rho2, bound);
    case FAM_MATERN: return fam_bound<FAM_MATERN>(K, rho2, bound);
    case FAM_MATERN2: return fam_bound<FAM_MATERN2>(K, rho2, bound);
    case FAM_COULOMB: return fam_bound<FAM_COULOMB>(K, rho2, bound);
    case FAM_SIN: return fam_bound<FAM_SIN>(K, rho2, bound);
    case FAM_COS: return fam_bound<FAM_COS>(K, rho2, bound);
    default: return fam_bound<FAM_RBF>(K, rho2, bound);
    }
}

// Shared state of a launch (pointers into dynamic shared memory and the
// barriers).
struct GsShared {
    uint8_t *A;           // [kGsAbufs][6][128 x 32] digit buffers
    uint8_t *Om;          // Omega8 columns 0..nc-1, [j / 16][c][16]
    double *colc;         // [2][kGsMaxDim][kGsMaxCols]
    double *rowc;         // [2][kGsMaxDim][128]
    int *coli;            // [2][kGsMaxCols]
    int *rowi;            // [2][128]
    double *box;          // [2][kGsMaxChunks][2][kGsMaxDim]
    double *rmax;         // [2][4][128]
    double *rss;          // [2][16]
};

// Generation of one item's chunks by one generator thread (row r of the
// item, the 8-column groups qd kGsGpt .. qd kGsGpt + kGsGpt - 1 of every
// chunk).  Accumulates the sum of squares and the largest |D_ij| of its
// entries.
template <int FAM, int NDIM>
__device__ __forceinline__ void gs_generate(
    const DevKernel &K, const GsShared &S, int b, const GsItem &w, int r,
    int qd, int sh, double *D, int ld, uint64_t *afull, uint64_t *afree,
    uint64_t *expready, uint64_t *expfree, int it, int *rowexp,
    long long &gc, volatile int *failed, bool &dead, double &ss, double &amax)
{
    constexpr int ND = NDIM > 0 ? NDIM : kGsMaxDim;
    const int nch = (w.n + kGsChunk - 1) / kGsChunk;
    const double *cc = S.colc + (size_t)b * kGsMaxDim * kGsMaxCols;
    const int *ci = S.coli + (size_t)b * kGsMaxCols;
    const double *rc = S.rowc + (size_t)b * kGsMaxDim * kGsRows;
    const int ndim = NDIM > 0 ? NDIM : K.ndim;
    double xr[ND];
    #pragma unroll
    for (int d = 0; d < ND; ++d) xr[d] = d < ndim ? rc[d * kGsRows + r] : 0.0;
    const int ridx = S.rowi[b * kGsRows + r];
    const bool rowvalid = D != nullptr;
    // x 2^(47 - e) in two exact power-of-two factors when 47 - e lies
    // beyond the double range
    const double s1 = sh > 1000 ? ldexp(1.0, sh - 1000) : 1.0;
    const double s2 = ldexp(1.0, sh > 1000 ? 1000 : sh);
    const double magic = 0x1.8p52;
    for (int kc = 0; kc < nch; ++kc, ++gc) {
        const int buf = (int)(gc & 1);
        // every decision here is warp-uniform (the chunk ends in a
        // __syncwarp); `dead` is the same in all lanes of a warp
        if (!dead) {
            bool ok = gc < kGsAbufs ||
                      mbar_wait_or(&afree[buf], (uint32_t)((gc >> 1) - 1) & 1, failed);
            // qd is the same in all lanes of a warp
            if (ok && kc == 0 && qd == 0 && it >= 2)
                ok = mbar_wait_or(expfree, (uint32_t)((it >> 1) - 1) & 1, failed);
            if (!__all_sync(0xffffffffu, ok ? 1 : 0)) {
                dead = true;
                *failed = 1;
            } else if (kc == 0 && qd == 0) {
                // the epilogue has read this buffer's scales of item it - 2
                rowexp[r] = sh;
                mbar_arrive(expready);
            }
        }
        if (dead) continue;
        uint8_t *A = S.A + (size_t)buf * kGsAbufBytes;
        #pragma unroll
        for (int h = 0; h < kGsGpt; ++h) {
            const int g = qd * kGsGpt + h;
            const int jb = kc * kGsChunk + 8 * g;
            const bool full = rowvalid && jb + 8 <= w.n;
            double y[8];
            #pragma unroll
            for (int cp = 0; cp < 4; ++cp) {
                // two consecutive columns' coordinates per 16-byte
                // (broadcast) shared-memory load
                double2 xc[ND];
                #pragma unroll
                for (int d = 0; d < ND; ++d)
                    if (NDIM > 0 || d < ndim)
                        xc[d] = *reinterpret_cast<const double2 *>(
                            cc + d * kGsMaxCols + jb + 2 * cp);
                #pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int c = 2 * cp + e;
                    const int j = jb + c;
                    double v = 0.0;
                    if (full || (rowvalid && j < w.n)) {
                        double dist = 0.0;
                        #pragma unroll
                        for (int d = 0; d < ND; ++d) {
                            if (NDIM > 0 || d < ndim) {
                                const double q = __dsub_rn(xr[d], e ? xc[d].y : xc[d].x);
                                dist = __dadd_rn(dist, __dmul_rn(q, q));
                            }
                        }
                        v = entry_fam<FAM>(K, dist, ridx, FAM == FAM_RBF ? ci[j] : 0);
                        __stcs(D + (size_t)j * ld, v);
                        ss = fma(v, v, ss);
                        amax = fmax(amax, fabs(v));
                    }
                    if (sh > 1000) v *= s1;
                    y[c] = fma(v, s2, magic);
                }
            }
            uint32_t dg[kGsSlices][2];
            digits6(y, dg);
            #pragma unroll
            for (int s = 0; s < kGsSlices; ++s)
                *reinterpret_cast<uint2 *>(A + s * (kGsRows * kGsChunk) +
                                           (g >> 1) * 2048 + (r >> 3) * 128 +
                                           (r & 7) * 16 + (g & 1) * 8) =
                    make_uint2(dg[s][0], dg[s][1]);
        }
        // the digits are visible to the tensor cores (each thread's fence),
        // then one arrival per warp
        asm volatile("fence.proxy.async.shared::cta;");
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(&afull[buf]);
    }
}

template <int FAM>
__device__ __forceinline__ void gs_generate_dim(
    const DevKernel &K, const GsShared &S, int b, const GsItem &w, int r,
    int qd, int sh, double *D, int ld, uint64_t *afull, uint64_t *afree,
    uint64_t *expready, uint64_t *expfree, int it, int *rowexp,
    long long &gc, volatile int *failed, bool &dead, double &ss, double &amax)
{
    if (K.ndim == 2)
        gs_generate<FAM, 2>(K, S, b, w, r, qd, sh, D, ld, afull, afree, expready,
                            expfree, it, rowexp, gc, failed, dead, ss, amax);
    else if (K.ndim == 3)
        gs_generate<FAM, 3>(K, S, b, w, r, qd, sh, D, ld, afull, afree, expready,
                            expfree, it, rowexp, gc, failed, dead, ss, amax);
    else
        gs_generate<FAM, 0>(K, S, b, w, r, qd, sh, D, ld, afull, afree, expready,
                            expfree, it, rowexp, gc, failed, dead, ss, amax);
}

__global__ void __launch_bounds__(kGsThreads, 1)
k_gen_sketch_i8(const __grid_constant__ CUtensorMap omap,
                const DevKernel *__restrict__ kernels,
                TileWork *__restrict__ tiles, int ntiles, Workspace ws,
                int nc, int npad)
{
    extern __shared__ __align__(1024) uint8_t gs_smem_raw[];
    __shared__ __align__(8) uint64_t afull[kGsAbufs];   // digits written
    __shared__ __align__(8) uint64_t afree[kGsAbufs];   // digits consumed
    __shared__ __align__(8) uint64_t cfull[2];          // item staged
    __shared__ __align__(8) uint64_t cfree[2];          // staging read
    __shared__ __align__(8) uint64_t omfull;            // Omega8 landed
    __shared__ __align__(8) uint64_t accfull;           // item's MMAs done
    __shared__ __align__(8) uint64_t accempty;          // TMEM read out
    __shared__ __align__(8) uint64_t expready[2];       // row scales posted
    __shared__ __align__(8) uint64_t expfree[2];        // ... and read
    __shared__ int rowexp[2][kGsRows];
    __shared__ DevKernel Ks[2];
    __shared__ uint32_t tmem_base;
    __shared__ volatile int failed;

    uint8_t *base = gs_smem_raw +
        ((1024u - (smem_u32(gs_smem_raw) & 1023u)) & 1023u);
    GsShared S;
    S.A = base + kGsOffA;
    S.Om = base + kGsOffOm;
    S.colc = reinterpret_cast<double *>(base + kGsOffColc);
    S.rowc = reinterpret_cast<double *>(base + kGsOffRowc);
    S.coli = reinterpret_cast<int *>(base + kGsOffColi);
    S.rowi = reinterpret_cast<int *>(base + kGsOffRowi);
    S.box = reinterpret_cast<double *>(base + kGsOffBox);
    S.rmax = reinterpret_cast<double *>(base + kGsOffRmax);
    S.rss = reinterpret_cast<double *>(base + kGsOffRss);

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int rpt = (ws.m_max + kGsRows - 1) / kGsRows;
    const long long nitems = (long long)ntiles * rpt;
    const uint32_t ncols_alloc = nc * kGsSlices <= 128 ? 128
                               : nc * kGsSlices <= 256 ? 256 : 512;

    if (t == 0) {
        failed = 0;
        for (int q = 0; q < kGsAbufs; ++q) {
            mbar_init(&afull[q], kGsGenWarps);
            mbar_init(&afree[q], 1);
        }
        for (int q = 0; q < 2; ++q) {
            mbar_init(&cfull[q], 1);
            mbar_init(&cfree[q], kGsGenThreads / 32);
            mbar_init(&expready[q], kGsRows);
            mbar_init(&expfree[q], kGsRows);
        }
        mbar_init(&omfull, 1);
        mbar_init(&accfull, 1);
        mbar_init(&accempty, kGsRows);
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    if (warp == kGsMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_base)), "r"(ncols_alloc));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    // items of this CTA whose row block exists, of tiles generated here
    // (the same sequence in every role)
    auto item_valid = [&](long long item, GsItem &w) {
        w = gs_item(tiles, (int)(item / rpt));
        return (int)(item % rpt) * kGsRows < w.m &&
               (w.status & TILE_GEN_SEPARATE) == 0;
    };

    int fail_tile = -1;
    if (warp < kGsGenThreads / 32) {
        // ---------------------------------------------------- generators
        const int r = t & (kGsRows - 1), qd = t >> 7;
        const int ncb = (ws.n_max + 63) / 64;
        long long gc = 0;
        int it = 0;
        bool dead = false;
        for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
            GsItem w;
            if (!item_valid(item, w)) continue;
            const int tile = (int)(item / rpt);
            const int b = it & 1;
            const int row0 = (int)(item % rpt) * kGsRows;
            const int i = row0 + r;
            if (!dead) {
                const bool ok = mbar_wait_or(&cfull[b], (uint32_t)(it >> 1) & 1, &failed);
                if (!__all_sync(0xffffffffu, ok ? 1 : 0)) {
                    dead = true;
                    fail_tile = tile;
                    failed = 1;
                }
            }
            double ss = 0.0, amax = 0.0;
            int sh = 47;
            bool have_bound = true;
            if (!dead) {
                const DevKernel &K = Ks[b];
                // bound on the row's entries: the kernel at the distance to
                // the nearest chunk box
                const int nch = (w.n + kGsChunk - 1) / kGsChunk;
                const double *rc = S.rowc + (size_t)b * kGsMaxDim * kGsRows;
                const double *bx = S.box + (size_t)b * kGsMaxChunks * 2 * kGsMaxDim;
                double rho2 = DBL_MAX;
                for (int kc = 0; kc < nch; ++kc) {
                    double g2 = 0.0;
                    for (int d = 0; d < K.ndim; ++d) {
                        const double x = rc[d * kGsRows + r];
                        const double lo = bx[(kc * 2) * kGsMaxDim + d];
                        const double hi = bx[(kc * 2 + 1) * kGsMaxDim + d];
                        const double g = fmax(0.0, fmax(lo - x, x - hi));
                        g2 += g * g;
                    }
                    rho2 = fmin(rho2, g2);
                }
                double bound = 0.0;
                have_bound = row_bound(K, rho2, bound) && bound <= DBL_MAX;
                int e = 0;
                if (have_bound && bound > 0.0) frexp(bound, &e);
                sh = 47 - e;
                double *D = i < w.m ? ws.D(w.slot) + i : nullptr;
                const int ld = ws.ldD();
                switch (K.family) {
                case FAM_EXP:
                    gs_generate_dim<FAM_EXP>(K, S, b, w, r, qd, sh, D, ld, afull, afree, &expready[b], &expfree[b], it, rowexp[b], gc, &failed, dead, ss, amax);
                    break;
                case FAM_SQREXP:
                    gs_generate_dim<FAM_SQREXP>(K, S, b, w, r, qd, sh, D, ld, afull, afree, &expready[b], &expfree[b], it, rowexp[b], gc, &failed, dead, ss, amax);
                    break;
                case FAM_MATERN:
                    gs_generate_dim<FAM_MATERN>(K, S, b, w, r, qd, sh, D, ld, afull, afree, &expready[b], &expfree[b], it, rowexp[b], gc, &failed, dead, ss, amax);
                    break;
                case FAM_MATERN2:
                    gs_generate_dim<FAM_MATERN2>(K, S, b, w, r, qd, sh, D, ld, afull, afree, &expready[b], &expfree[b], it, rowexp[b], gc, &failed, dead, ss, amax);
                    break;
                case FAM_COULOMB:
                    gs_generate_dim<FAM_COULOMB>(K, S, b, w, r, qd, sh, D, ld, afull, afree, &expready[b], &expfree[b], it, rowexp[b], gc, &failed, dead, ss, amax);
                    break;
                case FAM_SIN:
                    gs_generate_dim<FAM_SIN>(K, S, b, w, r, qd, sh, D, ld, afull, afree, &expready[b], &expfree[b], it, rowexp[b], gc, &failed, dead, ss, amax);
                    break;
                case FAM_COS:
                    gs_generate_dim<FAM_COS>(K, S, b, w, r, qd, sh, D, ld, afull, afree, &expready[b], &expfree[b], it, rowexp[b], gc, &failed, dead, ss, amax);
                    break;
                default:
                    gs_generate_dim<FAM_RBF>(K, S, b, w, r, qd, sh, D, ld, afull, afree, &expready[b], &expfree[b], it, rowexp[b], gc, &failed, dead, ss, amax);
                }
                if (dead && fail_tile < 0) fail_tile = tile;
            } else {
                gc += (w.n + kGsChunk - 1) / kGsChunk;
            }
            // the staged coordinates of buffer b are no longer read
            __syncwarp();
            if (lane == 0 && !dead) mbar_arrive(&cfree[b]);
            // item end: exact row maxima (row scales of later rounds and
            // the bound check), per-64-row sums of squares (exact norms),
            // summed in a fixed order
            double *rm = S.rmax + (size_t)b * 4 * kGsRows;
            double *rs = S.rss + (size_t)b * 16;
            rm[qd * kGsRows + r] = amax;
            double sw = ss;
            #pragma unroll
            for (int o = 16; o > 0; o >>= 1) sw += __shfl_down_sync(0xffffffffu, sw, o);
            if (lane == 0) rs[warp] = sw;
            named_sync(1, kGsGenThreads);
            if (!dead) {
                if (qd == 0 && i < w.m) {
                    double mx = rm[r];
                    #pragma unroll
                    for (int q = 1; q < kGsQd; ++q) mx = fmax(mx, rm[q * kGsRows + r]);
                    double *rx = ws.Rmx(w.slot) + (size_t)i * ncb;
                    rx[0] = mx;
                    for (int cb = 1; cb < (w.n + 63) / 64; ++cb) rx[cb] = 0.0;
                    bool bad = !have_bound || !(mx <= DBL_MAX);
                    if (!bad && mx > 0.0) {
                        int et = 0;
                        frexp(mx, &et);
                        const int eu = 47 - sh;
                        bad = et > eu || eu - et > kGsLostBits;
                    }
                    if (bad) atomicOr(&tiles[tile].status, TILE_RESKETCH);
                }
                if (t < 2 && row0 + 64 * t < w.m) {
                    // rows 64 t .. 64 t + 63: warps 4 qd + 2 t and 4 qd + 2 t + 1
                    double a = 0.0;
                    for (int q = 0; q < kGsQd; ++q)
                        a += rs[4 * q + 2 * t] + rs[4 * q + 2 * t + 1];
                    const int ldn = (ws.n_max + 63) / 64;
                    double *nr = ws.Nrm(w.slot) + (size_t)(row0 / 64 + t) * ldn;
                    nr[0] = a;
                    for (int cb = 1; cb < (w.n + 63) / 64; ++cb) nr[cb] = 0.0;
                }
            }
            ++it;
        }
    } else if (warp == kGsStageWarp) {
        // ------------------------------------------------------- staging
        bool om_issued = false;
        if (lane == 0) {
            const uint32_t bytes = (uint32_t)npad * (uint32_t)nc;
            mbar_expect_tx(&omfull, bytes);
            for (int kh = 0; kh < npad / 16; ++kh)
                tma_load_2d(S.Om + (size_t)kh * nc * 16, &omap, kh * 16, 0, &omfull);
            om_issued = true;
        }
        int it = 0;
        for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
            // one decision for the whole warp (its shuffles need every lane)
            if (__shfl_sync(0xffffffffu, failed ? 1 : 0, 0)) break;
            GsItem w;
            if (!item_valid(item, w)) continue;
            const int tile = (int)(item / rpt);
            const int b = it & 1;
            bool ok = true;
            if (it >= 2) {
                if (lane == 0)
                    ok = mbar_wait_sleep(&cfree[b], (uint32_t)((it >> 1) - 1) & 1, &failed, 256);
                ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
            }
            if (!ok) {
                if (lane == 0) fail_tile = tile;
                failed = 1;
                break;
            }
            const int row0 = (int)(item % rpt) * kGsRows;
            if (lane == 0) Ks[b] = kernels[w.prob];
            const DevKernel &K = kernels[w.prob];
            const int ndim = K.ndim, aos = K.aos;
            const double *rp = K.row_pt, *cp = K.col_pt;
            const long long rcount = K.row_count, ccount = K.col_count;
            double *colc = S.colc + (size_t)b * kGsMaxDim * kGsMaxCols;
            double *rowc = S.rowc + (size_t)b * kGsMaxDim * kGsRows;
            int *coli = S.coli + (size_t)b * kGsMaxCols;
            int *rowi = S.rowi + (size_t)b * kGsRows;
            // point indices through the pivots (independent loads)
            #pragma unroll 8
            for (int q = 0; q < kGsMaxChunks; ++q) {
                const int j = q * 32 + lane;
                if (j < w.n) coli[j] = (int)K.col_piv[w.col0 + j];
            }
            #pragma unroll
            for (int q = 0; q < kGsRows / 32; ++q) {
                const int rr = q * 32 + lane, i = row0 + rr;
                rowi[rr] = i < w.m ? (int)K.row_piv[w.row0 + i] : 0;
            }
            __syncwarp();
            // coordinates (structure of arrays in shared memory)
            #pragma unroll 4
            for (int q = 0; q < kGsMaxChunks; ++q) {
                const int j = q * 32 + lane;
                if (j < w.n) {
                    const long long p = coli[j];
                    for (int d = 0; d < ndim; ++d)
                        colc[d * kGsMaxCols + j] = aos ? cp[(size_t)ndim * p + d]
                                                       : cp[(size_t)d * ccount + p];
                }
            }
            #pragma unroll
            for (int q = 0; q < kGsRows / 32; ++q) {
                const int rr = q * 32 + lane;
                const long long p = rowi[rr];
                for (int d = 0; d < ndim; ++d)
                    rowc[d * kGsRows + rr] = row0 + rr < w.m
                        ? (aos ? rp[(size_t)ndim * p + d] : rp[(size_t)d * rcount + p])
                        : 0.0;
            }
            __syncwarp();
            // bounding box of each 32-column chunk
            double *bx = S.box + (size_t)b * kGsMaxChunks * 2 * kGsMaxDim;
            const int nch = (w.n + kGsChunk - 1) / kGsChunk;
            for (int kc = 0; kc < nch; ++kc) {
                const int j = kc * kGsChunk + lane;
                for (int d = 0; d < ndim; ++d) {
                    double lo = j < w.n ? colc[d * kGsMaxCols + j] : DBL_MAX;
                    double hi = j < w.n ? colc[d * kGsMaxCols + j] : -DBL_MAX;
                    #pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
                    }
                    if (lane == 0) {
                        bx[(kc * 2) * kGsMaxDim + d] = lo;
                        bx[(kc * 2 + 1) * kGsMaxDim + d] = hi;
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&cfull[b]);
            ++it;
        }
        // the Omega8 copy lands before the CTA exits
        if (lane == 0 && om_issued) {
            int dummy = 0;
            mbar_wait_or(&omfull, 0, &dummy);
        }
    } else if (warp == kGsMmaWarp) {
        // ----------------------------------------------------------- MMA
        long long last = -1;
        if (lane == 0) {
            const uint32_t idu = idesc_i8_mn(kGsRows, nc, false);
            const uint32_t ids = idesc_i8_mn(kGsRows, nc, true);
            bool ok = mbar_wait_sleep(&omfull, 0, &failed, 128);
            long long gc = 0;
            int it = 0;
            for (long long item = blockIdx.x; ok && item < nitems && !failed;
                 item += gridDim.x) {
                GsItem w;
                if (!item_valid(item, w)) continue;
                const int tile = (int)(item / rpt);
                const int nch = (w.n + kGsChunk - 1) / kGsChunk;
                ok = it == 0 || mbar_wait_sleep(&accempty, (uint32_t)(it - 1) & 1, &failed, 64);
                for (int kc = 0; ok && kc < nch; ++kc, ++gc) {
                    const int buf = (int)(gc & 1);
                    if (!mbar_wait_sleep(&afull[buf], (uint32_t)(gc >> 1) & 1, &failed, 64)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint8_t *A = S.A + (size_t)buf * kGsAbufBytes;
                    const uint64_t db = umma_desc(
                        smem_u32(S.Om + (size_t)kc * 2 * nc * 16), nc * 16, 128);
                    #pragma unroll
                    for (int s = 0; s < kGsSlices; ++s) {
                        const uint64_t da = umma_desc(
                            smem_u32(A + s * (kGsRows * kGsChunk)), 2048, 128);
                        mma_i8(tmem + s * nc, da, db, s == kGsSlices - 1 ? ids : idu,
                               kc > 0);
                    }
                    mma_commit(&afree[buf]);
                    if (kc == nch - 1) mma_commit(&accfull);
                    last = gc;
                }
                if (!ok) {
                    fail_tile = tile;
                    failed = 1;
                    break;
                }
                ++it;
            }
            if (!ok && fail_tile < 0) failed = 1;
            // after a failure: the MMAs issued finish before TMEM is freed
            if (failed && last >= 0) {
                int dummy = 0;
                mbar_wait_or(&afree[last & 1], (uint32_t)(last >> 1) & 1, &dummy);
            }
        }
    } else {
        // ------------------------------------------------------ epilogue
        static_assert(kGsEpiWarp0 + 4 == kGsThreads / 32, "epilogue warps");
        const int lq = warp & 3;
        const int rr = 32 * lq + lane;
        int it = 0;
        for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
            GsItem w;
            if (!item_valid(item, w)) continue;
            const int tile = (int)(item / rpt);
            const int b = it & 1;
            bool ok = mbar_wait_sleep(&expready[b], (uint32_t)(it >> 1) & 1, &failed, 512) &&
                      mbar_wait_sleep(&accfull, (uint32_t)it & 1, &failed, 512);
            // the TMEM loads below are warp-collective: every lane goes on
            // or every lane stops
            if (!__all_sync(0xffffffffu, ok ? 1 : 0)) {
                if (lane == 0) fail_tile = tile;
                failed = 1;
                break;
            }
            const int sh = rowexp[b][rr];
            mbar_arrive(&expfree[b]);
            tc_fence_after();
            const int i = (int)(item % rpt) * kGsRows + rr;
            double *Y = ws.Y(w.slot);
            const int ldY = ws.ldM();
            for (int g = 0; g < nc / 8; ++g) {
                uint32_t v[kGsSlices][8];
                #pragma unroll
                for (int s = 0; s < kGsSlices; ++s)
                    tmem_ld8(tmem + ((uint32_t)(32 * lq) << 16) + s * nc + 8 * g, v[s]);
                asm volatile("tcgen05.wait::ld.sync.aligned;");
                if (i < w.m) {
                    #pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const int col = 8 * g + c;
                        // T = 2^32 (256 P5 + P4) + sum_{s<4} 256^s P_s, both
                        // parts exact in double, one rounding in the fma
                        const long long hi = (long long)(int)v[5][c] * 256 +
                                             (long long)(int)v[4][c];
                        long long lo = (long long)(int)v[3][c];
                        #pragma unroll
                        for (int s = 2; s >= 0; --s) lo = lo * 256 + (long long)(int)v[s][c];
                        const double T = fma((double)hi, 0x1p32, (double)lo);
                        if (col < w.bcur)
                            Y[(size_t)col * ldY + i] = ldexp(T, -sh);
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&accempty);
            ++it;
        }
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (fail_tile >= 0) atomicOr(&tiles[fail_tile].status, TILE_MMA_TIMEOUT);
    if (warp == kGsMmaWarp)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(ncols_alloc));
}

bool gen_sketch_i8_fits(int nc)
{
    return nc > 0 && nc <= kGsMaxNc && kGsSmemBytes <= 227 * 1024;
}

bool gen_sketch_i8_tile_ok(int n, int ndim)
{
    return n > 0 && n <= kGsMaxCols && ndim > 0 && ndim <= kGsMaxDim;
}

bool launch_gen_sketch_i8(const DevKernel *d_kernels, TileWork *d_tiles,
                          int ntiles, Workspace ws, const int8_t *om8,
                          int ld_om8, int om8_cols, int ncols,
                          cudaStream_t stream)
{
    const int nc = (ncols + 15) / 16 * 16;
    const int npad = (ws.n_max + kGsChunk - 1) / kGsChunk * kGsChunk;
    if (npad > ld_om8) return false;
    CUtensorMap omap;
    if (!i8_colmajor_map(&omap, om8, ld_om8, om8_cols, nc)) return false;
    static int sms = 0;
    if (sms == 0) {
        int dev = 0, count = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_gen_sketch_i8,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kGsSmemBytes);
        sms = count > 0 ? count : 148;
    }
    const long long items = (long long)ntiles * ((ws.m_max + kGsRows - 1) / kGsRows);
    const int grid = (int)std::min<long long>(sms, items);
    if (grid <= 0) return true;
    k_gen_sketch_i8<<<grid, kGsThreads, kGsSmemBytes, stream>>>(
        omap, d_kernels, d_tiles, ntiles, ws, nc, npad);
    return true;
}

}  // namespace b200
