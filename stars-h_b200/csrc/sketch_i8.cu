// Sketch Y = D * Omega of the adaptive engine on the tcgen05 tensor cores,
// FP64-accurate through integer slices (the Ozaki scheme: K. Ozaki,
// T. Ogita, S. Oishi, S. M. Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59 (2012), in its integer form).
//
// Omega is an int8 matrix (a rounded Gaussian, 32 N(0,1) clipped to
// [-127, 127]); any such matrix is a valid sketch.  Row i of a tile is
// scaled by 2^-e_i, e_i the exponent of the row's largest |D_ij| (from the
// generator's per-row maxima), so x = D_ij 2^-e_i lies in (-1, 1); x is
// rounded to the 40-bit integer q = round(x 2^39), written in two's
// complement as four unsigned bytes u_0..u_3 and a signed top byte t:
//     D_ij = 2^(e_i - 39) (sum_{s<4} 256^s u_s[i, j] + 2^32 t[i, j]) + err,
//     |err| <= 2^-40 2^e_i.
// Each digit matrix times Omega is an exact 8-bit x int8 -> int32 product
// (|sum| <= 255 * 127 * n < 2^31 for n <= 8192) on tcgen05.mma kind::i8
// (unsigned A for u_s, signed A for t), accumulated in TMEM, one
// accumulator per digit.  The epilogue recombines the digits in int64
// (exact) and converts once:
//     Y_ic = 2^(e_i - 39) T_ic,  T_ic = sum_{s<4} 256^s P_s + 2^32 P_t.
// The only error is the rounding of q: 2^-40 of the row maximum per entry,
// far below the tolerance-driven thresholds of the adaptive basis (the
// rank decision itself uses the FP64 projection and the exact block norm).
//
// Persistent and warp-specialized: one CTA of 704 threads per SM walks the
// work items (tile, 128-row block) of the launch.  Each item's rows are read
// from HBM once, in K chunks of 32 columns:
//   * warp 16 (producer) brings chunk after chunk into a five-stage ring by
//     TMA tile copies, the 128 x 32 FP64 box of D and the 32 x nc bytes of
//     Omega of the same columns, continuing across items;
//   * warps 0-15 (converters) turn a landed chunk into the five digit
//     matrices (each thread 8 columns of one row) in the no-swizzle K-major
//     core-matrix layout of one of two digit buffers;
//   * warp 17 (MMA) issues the chunk's five MMAs (M 128, N nc, K 32) and
//     commits them to the barriers that free the stage and the digit buffer
//     (and, after an item's last chunk, to the accumulator barrier);
//   * warps 18-21 (epilogue) read an item's accumulators from TMEM, write
//     Y and release TMEM to the next item, while the copies and the
//     conversion of that item's first chunks go on.
// Hand-over is by mbarriers only; every wait gives up after about two
// seconds or as soon as another thread has given up, and the CTA then
// marks its tile TILE_MMA_TIMEOUT, waits for its own copies and MMAs in
// flight and releases TMEM.
#include <algorithm>
#include <cstdint>
#include <cuda.h>
#include "engine.cuh"
#include "tc_common.cuh"

namespace b200 {

constexpr int kSlices = 5;             // bytes (digits) per entry
constexpr int kSkRows = 128;           // rows per item (MMA M)
constexpr int kSkChunk = 32;           // K columns per chunk (one MMA K)
constexpr int kSkMaxN = 64;            // sketch columns per launch
constexpr int kStages = 5;             // D / Omega chunks in flight
constexpr int kAbufs = 2;              // digit buffers
constexpr int kConvThreads = 512;      // warps 0-15
constexpr int kProducerWarp = 16;
constexpr int kMmaWarp = 17;
constexpr int kEpiWarp0 = 18;          // warps 18-21
constexpr int kSkThreads = 22 * 32;
constexpr int kAbufBytes = kSlices * kSkRows * kSkChunk;                // 20 KB
constexpr int kDStageBytes = kSkRows * kSkChunk * (int)sizeof(double);  // 32 KB
constexpr int kOmSlotBytes = kSkChunk * kSkMaxN;                        // 2 KB

// Instruction descriptor: int32 accumulator, int8 A (unsigned digits, or
// the signed top digit), signed int8 B (Omega), both K-major, M = 128,
// N = n.
__host__ __device__ constexpr uint32_t idesc_i8(int n, bool a_signed)
{
    return idesc_i8_mn(kSkRows, n, a_signed);
}

// Digits of 8 entries x in (-1, 1), given as y = x 2^39 + 1.5 2^52 (one
// rounding; y lies in [2^52, 2^53), so its mantissa field is the integer
// 2^51 + q, q = round(x 2^39)): the low word of y's bit pattern is q mod
// 2^32 and the high word less 0x43380000 is floor(q / 2^32) in [-128, 128]
// (q = 2^39 is clamped to 2^39 - 1).  Byte s < 4 of the low words of
// columns 4g .. 4g + 3 goes to w[s][g], the signed top bytes to w[4][g].
__device__ __forceinline__ void digits8(const double (&y)[8],
                                        uint32_t (&w)[kSlices][2])
{
    uint32_t lo[8], hi[8];
    #pragma unroll
    for (int c = 0; c < 8; ++c) {
        lo[c] = (uint32_t)__double2loint(y[c]);
        int top = __double2hiint(y[c]) - 0x43380000;
        if (top > 127) { top = 127; lo[c] = 0xFFFFFFFFu; }
        hi[c] = (uint32_t)top;
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
        const uint32_t a = __byte_perm(hi[4 * g], hi[4 * g + 1], 0x40);
        const uint32_t b = __byte_perm(hi[4 * g + 2], hi[4 * g + 3], 0x40);
        w[4][g] = __byte_perm(a, b, 0x5410);
    }
}

// TMA tile copy of the 128 x 32 FP64 box at (row0, col0, slot) of the
// workspace's D tensor; completes on mbar.
__device__ __forceinline__ void tma_load_d(void *dst, const CUtensorMap *map,
                                           int row0, int col0, int slot,
                                           uint64_t *mbar)
{
    tma_load_3d(dst, map, row0, col0, slot, mbar);
}

// TMA tile copy of the 16 (rows k) x nc (columns c) byte box of Omega8 at
// (k0, c0): nc rows of 16 bytes, i.e. nc / 8 core matrices of one K half.
__device__ __forceinline__ void tma_load_om(void *dst, const CUtensorMap *map,
                                            int k0, int c0, uint64_t *mbar)
{
    tma_load_2d(dst, map, k0, c0, mbar);
}

// Exponent e of the largest |D_ij| of row i over the tile's n columns
// (|D_ij| < 2^e), from the generator's per-64-column maxima; 0 for an
// all-zero row or a row past the tile's m.
__device__ __forceinline__ int row_exponent(const Workspace &ws, int m,
                                            int n, int slot, int i)
{
    int e = 0;
    if (i < m) {
        const int ncb = (ws.n_max + 63) / 64;
        const double *rm = ws.Rmx(slot) + (size_t)i * ncb;
        double mx = 0.0;
        for (int cb = 0; cb < (n + 63) / 64; ++cb) mx = fmax(mx, rm[cb]);
        if (mx > 0.0) frexp(mx, &e);
    }
    return e;
}

// The tile fields the kernel reads, loaded once per item.
struct SkItem {
    int m, n, bcur, slot, cols_done, status;
};

__device__ __forceinline__ SkItem sk_item(const TileWork *tiles, int tile)
{
    const TileWork *w = tiles + tile;
    return SkItem{w->m, w->n, w->bcur, w->slot, w->cols_done, w->status};
}

// A tile takes part when its round is active and, if `need` is non-zero,
// its status has one of the bits of `need` (tiles the fused generator
// flagged for a re-sketch from the stored D).
__device__ __forceinline__ bool sk_active(const SkItem &w, int need)
{
    return w.bcur > 0 && (need == 0 || (w.status & need) != 0);
}

// Y(:, 0:bcur) of every tile with an active round = D * Omega8(:, cols_done
// + (0:nc)); work items (tile, 128-row block) in tile-major order, items
// blockIdx.x + q gridDim.x for this CTA.
__global__ void __launch_bounds__(kSkThreads, 1)
k_sketch_i8(const __grid_constant__ CUtensorMap dmap,
            const __grid_constant__ CUtensorMap omap,
            const TileWork *__restrict__ tiles, int ntiles, Workspace ws,
            int nc, int need)
{
    extern __shared__ __align__(1024) uint8_t sk_smem_raw[];
    __shared__ __align__(8) uint64_t full[kStages];    // chunk landed
    __shared__ __align__(8) uint64_t empty[kStages];   // chunk's MMAs done
    __shared__ __align__(8) uint64_t afull[kAbufs];    // digits written
    __shared__ __align__(8) uint64_t afree[kAbufs];    // digits consumed
    __shared__ __align__(8) uint64_t accfull;          // item's MMAs done
    __shared__ __align__(8) uint64_t accempty;         // TMEM read out
    __shared__ uint32_t tmem_base;
    __shared__ volatile int failed;
    __shared__ __align__(8) uint64_t expready[2];      // row exponents posted
    __shared__ int rowexp[2][kSkRows];                 // ... for items it, it + 1

    // 1024-byte aligned base (the launch adds 1 KB of slack)
    uint8_t *base = sk_smem_raw + ((1024u - (smem_u32(sk_smem_raw) & 1023u)) & 1023u);
    uint8_t *Abuf = base;                                                  // [2][5][4 KB]
    double *Dst = reinterpret_cast<double *>(base + kAbufs * kAbufBytes);  // [5][32][128]
    uint8_t *Om = base + kAbufs * kAbufBytes + kStages * kDStageBytes;     // [5][2 KB]

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int rpt = (ws.m_max + kSkRows - 1) / kSkRows;
    const long long nitems = (long long)ntiles * rpt;
    const uint32_t ncols_alloc = nc * kSlices <= 128 ? 128
                               : nc * kSlices <= 256 ? 256 : 512;

    if (t == 0) {
        failed = 0;
        for (int q = 0; q < kStages; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], 1);
        }
        for (int b = 0; b < kAbufs; ++b) {
            mbar_init(&afull[b], kConvThreads / 32);
            mbar_init(&afree[b], 1);
        }
        mbar_init(&accfull, 1);
        mbar_init(&accempty, kSkRows);
        mbar_init(&expready[0], kSkRows);
        mbar_init(&expready[1], kSkRows);
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_base)), "r"(ncols_alloc));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    int fail_tile = -1;          // a tile whose item this thread gave up on
    long long gc = 0;            // chunks seen by this role (all items)
    int it = 0;                  // items processed by this CTA

    if (warp < kConvThreads / 32) {
        // ---------------------------------------------------- converters
        const int r = t & (kSkRows - 1), qd = t >> 7;
        const double magic = 0x1.8p52;
        SkItem wn = sk_item(tiles, (int)(blockIdx.x / rpt));
        for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
            const int tile = (int)(item / rpt);
            const SkItem w = wn;
            if (item + gridDim.x < nitems)   // the next item's fields, early
                wn = sk_item(tiles, (int)((item + gridDim.x) / rpt));
            const int row0 = (int)(item % rpt) * kSkRows;
            if (!sk_active(w, need) || row0 >= w.m) continue;
            const int nchunks = (w.n + kSkChunk - 1) / kSkChunk;
            const int i = row0 + r;
            // the item's row exponents, posted ahead by the epilogue warps
            // (every decision below is warp-uniform: the loop has a
            // __syncwarp)
            const bool eok = mbar_wait_or(&expready[it & 1], (uint32_t)(it >> 1) & 1, &failed);
            if (!__all_sync(0xffffffffu, eok ? 1 : 0)) {
                fail_tile = tile;
                failed = 1;
                break;
            }
            // x = D 2^(39 - e) (two exact power-of-two factors when 39 - e
            // is beyond the double range), y = x + 1.5 2^52 in one fma
            const int sh = 39 - rowexp[it & 1][r];
            const double s1 = sh > 1000 ? ldexp(1.0, sh - 1000) : 1.0;
            const double s2 = ldexp(1.0, sh > 1000 ? 1000 : sh);
            for (int kc = 0; kc < nchunks; ++kc, ++gc) {
                const int sg = (int)(gc % kStages), b = (int)(gc & 1);
                bool ok = mbar_wait_or(&full[sg], (uint32_t)(gc / kStages) & 1, &failed);
                ok = ok && (gc < kAbufs ||
                            mbar_wait_or(&afree[b], (uint32_t)((gc >> 1) - 1) & 1, &failed));
                if (!__all_sync(0xffffffffu, ok ? 1 : 0)) {
                    fail_tile = tile;
                    failed = 1;
                    break;
                }
                const double *st = Dst + (size_t)sg * (kSkRows * kSkChunk);
                double y[8];
                #pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int j = kc * kSkChunk + 8 * qd + c;
                    double v = (i < w.m && j < w.n) ? st[(8 * qd + c) * kSkRows + r] : 0.0;
                    if (sh > 1000) v *= s1;
                    y[c] = fma(v, s2, magic);
                }
                uint32_t dg[kSlices][2];
                digits8(y, dg);
                uint8_t *A = Abuf + b * kAbufBytes;
                #pragma unroll
                for (int s = 0; s < kSlices; ++s)
                    *reinterpret_cast<uint2 *>(A + s * (kSkRows * kSkChunk) +
                                               (qd >> 1) * 2048 + (r >> 3) * 128 +
                                               (r & 7) * 16 + (qd & 1) * 8) =
                        make_uint2(dg[s][0], dg[s][1]);
                // each thread's digits visible to the tensor cores, then
                // one arrival per warp
                asm volatile("fence.proxy.async.shared::cta;");
                __syncwarp();
                if ((t & 31) == 0) mbar_arrive(&afull[b]);
            }
            if (failed) break;
            ++it;
        }
    } else if (warp == kProducerWarp) {
        // ------------------------------------------------------ producer
        long long issued = 0;
        if (lane == 0) {
            const uint32_t bytes = kDStageBytes + 2 * 16 * nc;
            SkItem wn = sk_item(tiles, (int)(blockIdx.x / rpt));
            for (long long item = blockIdx.x; item < nitems && !failed;
                 item += gridDim.x) {
                const int tile = (int)(item / rpt);
                const SkItem w = wn;
                if (item + gridDim.x < nitems)
                    wn = sk_item(tiles, (int)((item + gridDim.x) / rpt));
                const int row0 = (int)(item % rpt) * kSkRows;
                if (!sk_active(w, need) || row0 >= w.m) continue;
                const int nchunks = (w.n + kSkChunk - 1) / kSkChunk;
                for (int kc = 0; kc < nchunks; ++kc, ++gc) {
                    const int sg = (int)(gc % kStages);
                    if (gc >= kStages &&
                        !mbar_wait_or(&empty[sg], (uint32_t)(gc / kStages - 1) & 1, &failed)) {
                        fail_tile = tile;
                        failed = 1;
                        break;
                    }
                    mbar_expect_tx(&full[sg], bytes);
                    tma_load_d(Dst + (size_t)sg * (kSkRows * kSkChunk), &dmap, row0,
                               kc * kSkChunk, w.slot, &full[sg]);
                    uint8_t *o = Om + sg * kOmSlotBytes;
                    tma_load_om(o, &omap, kc * kSkChunk, w.cols_done, &full[sg]);
                    tma_load_om(o + nc * 16, &omap, kc * kSkChunk + 16, w.cols_done,
                                &full[sg]);
                    issued = gc + 1;
                }
            }
            // after a failure: the copies still in flight land before the
            // CTA exits (bounded waits)
            if (failed) {
                int dummy = 0;
                for (long long q = issued > kStages ? issued - kStages : 0; q < issued; ++q)
                    mbar_wait_or(&full[q % kStages], (uint32_t)(q / kStages) & 1, &dummy);
            }
        }
    } else if (warp == kMmaWarp) {
        // ----------------------------------------------------------- MMA
        long long last = -1;
        if (lane == 0) {
            const uint32_t idu = idesc_i8(nc, false), ids = idesc_i8(nc, true);
            SkItem wn = sk_item(tiles, (int)(blockIdx.x / rpt));
            for (long long item = blockIdx.x; item < nitems && !failed;
                 item += gridDim.x) {
                const int tile = (int)(item / rpt);
                const SkItem w = wn;
                if (item + gridDim.x < nitems)
                    wn = sk_item(tiles, (int)((item + gridDim.x) / rpt));
                const int row0 = (int)(item % rpt) * kSkRows;
                if (!sk_active(w, need) || row0 >= w.m) continue;
                const int nchunks = (w.n + kSkChunk - 1) / kSkChunk;
                // the previous item's accumulators have been read out
                bool ok = it == 0 || mbar_wait_or(&accempty, (uint32_t)(it - 1) & 1, &failed);
                for (int kc = 0; ok && kc < nchunks; ++kc, ++gc) {
                    const int sg = (int)(gc % kStages), b = (int)(gc & 1);
                    if (!mbar_wait_or(&afull[b], (uint32_t)(gc >> 1) & 1, &failed)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    const uint8_t *A = Abuf + b * kAbufBytes;
                    const uint64_t db = umma_desc(smem_u32(Om + sg * kOmSlotBytes),
                                                  nc * 16, 128);
                    #pragma unroll
                    for (int s = 0; s < kSlices; ++s) {
                        const uint64_t da = umma_desc(
                            smem_u32(A + s * (kSkRows * kSkChunk)), 2048, 128);
                        mma_i8(tmem + s * nc, da, db, s == kSlices - 1 ? ids : idu,
                               kc > 0);
                    }
                    mma_commit(&empty[sg]);
                    mma_commit(&afree[b]);
                    if (kc == nchunks - 1) mma_commit(&accfull);
                    last = gc;
                }
                if (!ok) {
                    fail_tile = tile;
                    failed = 1;
                    break;
                }
                ++it;
            }
            // after a failure: the MMAs issued finish before TMEM is freed
            if (failed && last >= 0) {
                int dummy = 0;
                mbar_wait_or(&afree[last & 1], (uint32_t)(last >> 1) & 1, &dummy);
            }
        }
    } else {
        // ------------------------------------------------------ epilogue
        // warps kEpiWarp0 .. + 3: warp w may read TMEM lanes 32 (w % 4) ..
        // 32 (w % 4) + 31, the item's rows of the same numbers
        static_assert(kEpiWarp0 + 4 == kSkThreads / 32, "epilogue warps");
        const int lq = warp & 3;
        const int rr = 32 * lq + lane;
        // The converters' row exponents: those of the first item, then,
        // while an item's MMAs run, those of the next one.  Buffer
        // (it + 1) & 1 last served item it - 1, whose conversion is over
        // once its accumulators were full.
        auto valid = [&](const SkItem &w, long long item) {
            return sk_active(w, need) && (int)(item % rpt) * kSkRows < w.m;
        };
        auto next_valid = [&](long long item, SkItem &w) {
            for (; item < nitems; item += gridDim.x) {
                w = sk_item(tiles, (int)(item / rpt));
                if (valid(w, item)) break;
            }
            return item;
        };
        auto post = [&](long long item, const SkItem &w, int b) {
            rowexp[b][rr] = row_exponent(ws, w.m, w.n, w.slot,
                                         (int)(item % rpt) * kSkRows + rr);
            mbar_arrive(&expready[b]);
        };
        SkItem w{};
        long long item = next_valid(blockIdx.x, w);
        if (item < nitems) post(item, w, 0);
        while (item < nitems) {
            const int tile = (int)(item / rpt);
            SkItem wn{};
            const long long nx = next_valid(item + gridDim.x, wn);
            if (nx < nitems) post(nx, wn, (it + 1) & 1);
            const int row0 = (int)(item % rpt) * kSkRows;
            const int i = row0 + rr;
            const int e = rowexp[it & 1][rr];
            // the TMEM loads below are warp-collective: every lane goes on
            // or every lane stops
            const bool ok = mbar_wait_or(&accfull, (uint32_t)it & 1, &failed);
            if (!__all_sync(0xffffffffu, ok ? 1 : 0)) {
                if (lane == 0) fail_tile = tile;
                failed = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            double *Y = ws.Y(w.slot);
            const int ldY = ws.ldM();
            for (int g = 0; g < nc / 8; ++g) {
                uint32_t v[kSlices][8];
                #pragma unroll
                for (int s = 0; s < kSlices; ++s)
                    tmem_ld8(tmem + ((uint32_t)(32 * lq) << 16) + s * nc + 8 * g, v[s]);
                asm volatile("tcgen05.wait::ld.sync.aligned;");
                if (i < w.m) {
                    #pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const int col = 8 * g + c;
                        long long T = (long long)(int)v[kSlices - 1][c];
                        #pragma unroll
                        for (int s = kSlices - 2; s >= 0; --s)
                            T = T * 256 + (long long)(int)v[s][c];
                        if (col < w.bcur)
                            Y[(size_t)col * ldY + i] = ldexp((double)T, e - 39);
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            mbar_arrive(&accempty);
            ++it;
            item = nx;
            w = wn;
        }
    }

    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (fail_tile >= 0)
        atomicOr(&const_cast<TileWork *>(tiles)[fail_tile].status, TILE_MMA_TIMEOUT);
    if (warp == kMmaWarp)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(ncols_alloc));
}

static size_t sketch_i8_smem()
{
    return (size_t)kAbufs * kAbufBytes + (size_t)kStages * kDStageBytes +
           (size_t)kStages * kOmSlotBytes + 1024;
}

bool sketch_i8_fits(int nc, int n_max)
{
    return nc > 0 && nc <= kSkMaxN && n_max <= 8192 &&
           sketch_i8_smem() <= 227 * 1024;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (encode == nullptr) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn,
                                    cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || fn == nullptr) {
            cudaGetLastError();
            return nullptr;
        }
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    return encode;
}

// Tensor map of the batch's D blocks as one 3-D FP64 tensor (rows, columns,
// slots) with a 128 x 32 x 1 box; needs an even leading dimension (16-byte
// strides).
static bool d_tensor_map(CUtensorMap *map, const Workspace &ws, int nslots)
{
    auto encode = tensor_map_encoder();
    if (encode == nullptr || ws.ldD() % 2 != 0) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)ws.m_max, (cuuint64_t)ws.n_max,
                                (cuuint64_t)nslots};
    const cuuint64_t strides[2] = {(cuuint64_t)ws.ldD() * sizeof(double),
                                   (cuuint64_t)ws.stride * sizeof(double)};
    const cuuint32_t box[3] = {kSkRows, kSkChunk, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, ws.D(0), dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map of Omega8 (ld_om8 rows k, om8_cols columns c, column-major
// bytes) with a 16 x nc box: columns past om8_cols read as zero.
bool i8_colmajor_map(CUtensorMap *map, const int8_t *om8, int ld_om8,
                     int om8_cols, int nc)
{
    auto encode = tensor_map_encoder();
    if (encode == nullptr || ld_om8 % 16 != 0 || ((uintptr_t)om8 & 15u) != 0)
        return false;
    const cuuint64_t dims[2] = {(cuuint64_t)ld_om8, (cuuint64_t)om8_cols};
    const cuuint64_t strides[1] = {(cuuint64_t)ld_om8};
    const cuuint32_t box[2] = {16, (cuuint32_t)nc};
    const cuuint32_t estr[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void *)om8, dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool launch_sketch_i8(const TileWork *d_tiles, int ntiles, Workspace ws,
                      const int8_t *om8, int ld_om8, int om8_cols, int ncols,
                      cudaStream_t stream, int need)
{
    const int nc = (ncols + 15) / 16 * 16;
    CUtensorMap dmap, omap;
    if (!d_tensor_map(&dmap, ws, ntiles) ||
        !i8_colmajor_map(&omap, om8, ld_om8, om8_cols, nc))
        return false;
    static int sms = 0;
    if (sms == 0) {
        int dev = 0, count = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_sketch_i8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sketch_i8_smem());
        sms = count > 0 ? count : 148;
    }
    const long long items = (long long)ntiles * ((ws.m_max + kSkRows - 1) / kSkRows);
    const int grid = (int)std::min<long long>(sms, items);
    if (grid <= 0) return true;
    k_sketch_i8<<<grid, kSkThreads, sketch_i8_smem(), stream>>>(
        dmap, omap, d_tiles, ntiles, ws, nc, need);
    return true;
}

}  // namespace b200
