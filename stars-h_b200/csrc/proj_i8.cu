// Projection B = Q^T D of the adaptive engine on the tcgen05 tensor cores,
// FP64-accurate through integer slices (the integer Ozaki scheme of
// sketch_i8.cu); replaces the FP64 GEMM of the reference's
// src/backends/sequential/dense/drsdd.c:69-70 for tiles with at most 32
// basis columns.
//
// Scaling.  The contraction runs over the tile rows i.  Row i of D is
// scaled by 2^-e_i (e_i the exponent of its exact largest |D_ij|, from the
// generator), x_ij = D_ij 2^-e_i in (-1, 1), and the factor moves to Q:
// Q'_ic = Q_ic 2^e_i, so that B_cj = sum_i Q'_ic x_ij.  x is rounded to a
// 56-bit integer (seven bytes: six unsigned, the top one signed) and Q'
// column c, scaled by 2^-f_c (f_c the exponent of its largest entry), to
// a 54-bit integer in balanced base-256 digits (seven signed bytes):
//     x_ij = 2^-55 sum_{s<7} 256^s a_s(i, j),
//     Q'_ic = 2^(f_c - 54) sum_{t<7} 256^t b_t(i, c).
// Each a_s b_t is an exact int8 x int8 -> int32 product (tcgen05.mma
// kind::i8); the products of equal weight w = s + t share one TMEM
// accumulator block and only w >= 5 is kept (the dropped terms are below
// 2^-57 of the largest product).  With the basis slices stacked in shared
// memory between zero blocks, one MMA per D slice (N = 256) feeds all
// eight weight blocks: seven MMAs per 32-row chunk.  The epilogue combines
// the eight accumulators in two exact int64 words and converts once:
//     B_cj = 2^(f_c - 69) (2^32 H + L),  H = sum_{w>=9} 256^(w-9) P_w,
//                                        L = sum_{w<=8} 256^(w-5) P_w.
// The representation error is 2^-56 of each row's largest entry of D and
// 2^-55 of each Q' column's largest entry: the level of the FP64 product
// it replaces.  Accumulators stay below 2^31 for m <= 4096 (seven products
// of weight w per K step, each below 2^15 in magnitude); the kernel takes
// tiles of up to 2048 rows.
//
// k_proj_prep (one CTA per tile) computes e_i, f_c and the seven digit
// slices of Q' (32 columns, zero beyond k1) into the slot's workspace and
// flags the tile TILE_PROJ_I8; the FP64 projection skips flagged tiles.
//
// k_proj_i8 is persistent and warp-specialized like the sketch kernels:
// per 32-row chunk of an item (tile, 128-column block), one producer lane
// streams the 32 x 128 FP64 block of D (two 128B-swizzled TMA boxes) into
// a three-stage ring that the converters free as soon as they hold the
// values, another the chunk's 7 KB of basis slices (two bulk copies) into
// the stacks of a two-stage ring that the MMAs free; 16 converter warps
// write the seven digit slices of x (each thread 8 rows of one column);
// one warp issues the chunk's seven MMAs; four epilogue warps read the
// accumulators and write B.  Every wait is bounded; after a timeout the
// tile is marked TILE_MMA_TIMEOUT and the call fails.
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include "engine.cuh"
#include "tc_common.cuh"

namespace b200 {

constexpr int kPjSlices = 7;
constexpr int kPjCols = 128;          // columns of D per item (MMA M)
constexpr int kPjChunk = 32;          // rows of D per chunk (MMA K)
constexpr int kPjN = 32;              // basis columns per weight block
constexpr int kPjMinW = 5;            // weights kept: 5 .. 12
constexpr int kPjAcc = 2 * (kPjSlices - 1) - kPjMinW + 1;   // 8
// The basis slices sit in shared memory as one stack of kPjBlocks blocks
// of kPjN rows (per 16-byte K half, a "plane"): blocks 7 .. 13 hold slices
// t = 0 .. 6, the others are zero.  The eight consecutive blocks starting
// at block 12 - s are the B operand of D slice s: block w - 5 of that
// window is slice w - s (zero outside 0 .. 6), so one MMA (N = 8 kPjN =
// 256) adds a_s b_(w-s) into the accumulator of every weight w = 5 .. 12.
constexpr int kPjBlocks = 20;
constexpr int kPjPlane = kPjBlocks * kPjN * 16;                      // 10 KB
constexpr int kPjQData = kPjSlices * kPjN * 16;                      // 3.5 KB
constexpr int kPjDStages = 3;         // D chunks in flight
constexpr int kPjQStages = 2;         // Q' chunks in flight
constexpr int kPjConvThreads = 512;
constexpr int kPjProducerWarp = 16;
constexpr int kPjMmaWarp = 17;
constexpr int kPjEpiWarp0 = 18;
constexpr int kPjThreads = 22 * 32;
constexpr int kPjMaxRows = 2048;
constexpr int kPjAbufBytes = kPjSlices * kPjCols * kPjChunk;          // 28 KB
constexpr int kPjDBytes = kPjChunk * kPjCols * (int)sizeof(double);  // 32 KB
constexpr int kPjQBytes = 2 * kPjQData;          // one chunk in global, 7 KB
constexpr int kPjQStage = 2 * kPjPlane;          // one chunk's stack, 20 KB
constexpr size_t kPjSmemBytes = (size_t)kPjDStages * kPjDBytes +
                                (size_t)kPjQStages * kPjQStage +
                                (size_t)2 * kPjAbufBytes + 1024;

static_assert(kPjAcc * kPjN <= 256, "TMEM columns");

__host__ __device__ constexpr uint32_t idesc_i8_ab(int m, int n, bool a_signed,
                                                   bool b_signed)
{
    return (2u << 4) | ((a_signed ? 1u : 0u) << 7) | ((b_signed ? 1u : 0u) << 10) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// Bytes of the 56-bit two's-complement integer q = round(X), |X| < 2^55
// (X exact): q = 2^32 hi + lo with hi = round(X 2^-32), lo = round(X - 2^32
// hi) in [-2^31, 2^31], both by the 1.5 2^52 rounding constant; the low
// word of lo is bytes 0-3, the borrow of a negative lo moves into hi, whose
// bytes 0-1 are digits 4-5 and whose (signed) byte 2 is digit 6.
__device__ __forceinline__ void bytes56(double X, uint32_t &lo32, uint32_t &hi24)
{
    const double magic = 0x1.8p52;
    const double y1 = fma(X, 0x1p-32, magic);
    const double hid = y1 - magic;
    const int hi = __double2loint(y1);
    const double lo = fma(hid, -0x1p32, X);
    const double y2 = lo + magic;
    lo32 = (uint32_t)__double2loint(y2);
    hi24 = (uint32_t)(hi + (__double2hiint(y2) - 0x43380000));
}

// Exponent e of a largest |D_ij| of row i (|D_ij| < 2^e; 0 for a zero
// row), from the generator's per-64-column maxima.
__device__ __forceinline__ int proj_row_exp(const Workspace &ws, int n,
                                            int slot, int i)
{
    const int ncb = (ws.n_max + 63) / 64;
    const double *rm = ws.Rmx(slot) + (size_t)i * ncb;
    double mx = 0.0;
    for (int cb = 0; cb < (n + 63) / 64; ++cb) mx = fmax(mx, rm[cb]);
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);
    return e;
}

// Per tile: row exponents e_i (Qe, ints), column exponents f_c (Qf) and
// the byte slices of Q' = Q diag(2^e) 2^-f (Qd, chunk-major: per 32-row
// chunk, 7 slices x 2 K halves x 64 rows c x 16 bytes).
__global__ void __launch_bounds__(256)
k_proj_prep(TileWork *__restrict__ tiles, Workspace ws)
{
    TileWork &tw = tiles[blockIdx.x];
    const int m = tw.m, k1 = tw.k1, s = tw.slot;
    if (k1 <= 0 || k1 > kPjN || m > kPjMaxRows || !(tw.dnorm2 > 0.0)) return;
    __shared__ int fmaxe[kPjN];
    int *re = ws.Qe(s);
    const int ldq = ws.ldQd();
    for (int c = threadIdx.x; c < kPjN; c += blockDim.x) fmaxe[c] = INT32_MIN;
    for (int i = threadIdx.x; i < m; i += blockDim.x)
        re[i] = proj_row_exp(ws, tw.n, s, i);
    __syncthreads();
    const double *Q = ws.Q(s);
    const int ldm = ws.ldM();
    for (int e = threadIdx.x; e < k1 * m; e += blockDim.x) {
        const int c = e / m, i = e - c * m;
        const double q = Q[(size_t)c * ldm + i];
        if (q != 0.0) {
            int eq;
            frexp(q, &eq);
            atomicMax(&fmaxe[c], eq + re[i]);
        }
    }
    __syncthreads();
    int *fe = ws.Qf(s);
    for (int c = threadIdx.x; c < kPjN; c += blockDim.x)
        fe[c] = c < k1 && fmaxe[c] != INT32_MIN ? fmaxe[c] : 0;
    __syncthreads();
    // slices in balanced base-256 digits (every byte signed, so one MMA
    // can take all seven), chunk-major: per 32-row chunk, K half h, slice
    // t, basis column c < 32, 16 bytes of rows i; byte (t, c, i) at
    // i / 32 * kPjQBytes + (i % 32 / 16) * kPjQData + t * 512 + c * 16 +
    // i % 16.  A thread writes one 16-byte row (c, 16 i) of every slice;
    // columns c >= k1 and rows i >= m are zero.
    uint8_t *qd = ws.Qd(s);
    const int halves = ldq / 16;
    for (int e = threadIdx.x; e < kPjN * halves; e += blockDim.x) {
        const int c = e % kPjN, hh = e / kPjN, i0 = hh * 16;
        uint32_t w[kPjSlices][4];
        #pragma unroll
        for (int t = 0; t < kPjSlices; ++t)
            w[t][0] = w[t][1] = w[t][2] = w[t][3] = 0u;
        const int fc = c < k1 && fmaxe[c] != INT32_MIN ? fmaxe[c] : 0;
        #pragma unroll
        for (int u = 0; u < 16; ++u) {
            const int i = i0 + u;
            if (c < k1 && i < m) {
                const double q = Q[(size_t)c * ldm + i];
                // X = Q_ic 2^(e_i - f_c + 54), |X| < 2^54, in exact steps
                const int sh = re[i] - fc + 54;
                double X = q;
                if (sh > 1000) X = ldexp(ldexp(X, 1000), sh - 1000);
                else if (sh < -1000) X = ldexp(ldexp(X, -1000), sh + 1000);
                else X = ldexp(X, sh);
                uint32_t lo, hi;
                bytes56(X, lo, hi);
                long long v = ((long long)(int)hi << 32) | (long long)lo;
                #pragma unroll
                for (int t = 0; t < kPjSlices; ++t) {
                    const int d = (int)(int8_t)(v & 0xFF);   // in [-128, 127]
                    v = (v - d) >> 8;
                    w[t][u >> 2] |= ((uint32_t)d & 0xFFu) << (8 * (u & 3));
                }
            }
        }
        #pragma unroll
        for (int t = 0; t < kPjSlices; ++t)
            *reinterpret_cast<uint4 *>(qd + (size_t)(hh >> 1) * kPjQBytes +
                                       (hh & 1) * kPjQData + t * (kPjN * 16) + c * 16) =
                make_uint4(w[t][0], w[t][1], w[t][2], w[t][3]);
    }
    if (threadIdx.x == 0) tw.status |= TILE_PROJ_I8;
}

struct PjItem {
    int m, n, k1, slot, status;
};

__device__ __forceinline__ PjItem pj_item(const TileWork *tiles, int tile)
{
    const TileWork *w = tiles + tile;
    return PjItem{w->m, w->n, w->k1, w->slot, w->status};
}

// B(c, j) for the tiles flagged TILE_PROJ_I8; items (tile, 128-column
// block) in tile-major order.
__global__ void __launch_bounds__(kPjThreads, 1)
k_proj_i8(const __grid_constant__ CUtensorMap dmap,
          TileWork *__restrict__ tiles, int ntiles, Workspace ws)
{
    extern __shared__ __align__(1024) uint8_t pj_smem_raw[];
    __shared__ __align__(8) uint64_t dfull[kPjDStages];   // D chunk landed
    __shared__ __align__(8) uint64_t dempty[kPjDStages];  // ... read
    __shared__ __align__(8) uint64_t qfull[kPjQStages];   // Q' chunk landed
    __shared__ __align__(8) uint64_t qempty[kPjQStages];  // ... consumed
    __shared__ __align__(8) uint64_t afull[2];
    __shared__ __align__(8) uint64_t afree[2];
    __shared__ __align__(8) uint64_t accfull;
    __shared__ __align__(8) uint64_t accempty;
    __shared__ __align__(8) uint64_t rowready[2];   // row exponents staged
    __shared__ __align__(8) uint64_t rowfree[2];
    __shared__ int16_t rowe[2][kPjMaxRows];
    __shared__ uint32_t tmem_base;
    __shared__ volatile int failed;

    uint8_t *base = pj_smem_raw + ((1024u - (smem_u32(pj_smem_raw) & 1023u)) & 1023u);
    uint8_t *Dst = base;                                            // [3][32 KB]
    uint8_t *Qst = base + (size_t)kPjDStages * kPjDBytes;           // [2][20 KB]
    uint8_t *Abuf = Qst + (size_t)kPjQStages * kPjQStage;           // [2][28 KB]

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int cpt = (ws.n_max + kPjCols - 1) / kPjCols;    // items per tile
    const long long nitems = (long long)ntiles * cpt;

    if (t == 0) {
        failed = 0;
        for (int q = 0; q < kPjDStages; ++q) {
            mbar_init(&dfull[q], 1);
            mbar_init(&dempty[q], kPjConvThreads / 32);
        }
        for (int q = 0; q < kPjQStages; ++q) {
            mbar_init(&qfull[q], 1);
            mbar_init(&qempty[q], 1);
        }
        for (int q = 0; q < 2; ++q) {
            mbar_init(&afull[q], kPjConvThreads / 32);
            mbar_init(&afree[q], 1);
            mbar_init(&rowready[q], kPjConvThreads / 32);
            mbar_init(&rowfree[q], kPjConvThreads / 32);
        }
        mbar_init(&accfull, 1);
        mbar_init(&accempty, kPjCols);
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    // the zero blocks of the basis stacks (the copies fill blocks 7 .. 13)
    for (int q = t; q < kPjQStages * kPjQStage / 16; q += kPjThreads)
        reinterpret_cast<uint4 *>(Qst)[q] = make_uint4(0u, 0u, 0u, 0u);
    asm volatile("fence.proxy.async.shared::cta;");
    if (warp == kPjMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_base)), "r"(256));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    auto item_valid = [&](long long item, PjItem &w) {
        w = pj_item(tiles, (int)(item / cpt));
        return (w.status & TILE_PROJ_I8) != 0 && (int)(item % cpt) * kPjCols < w.n;
    };

    int fail_tile = -1;
    if (warp < kPjConvThreads / 32) {
        // ----------------------------------------------------- converters
        // thread: column j of the item and the rows 8 qd .. 8 qd + 7 of
        // each chunk, with the lanes of a warp on 16 columns x 2 row
        // groups, so that the warp's digit stores are 256 contiguous bytes
        // (the UMMA core matrices: 8 columns x 16 bytes of K).  Every
        // decision is warp-uniform (the loop has __syncwarp).
        const int j = 16 * (warp & 7) + (lane >> 1);
        const int qd = 2 * (warp >> 3) + (lane & 1);
        long long gc = 0;
        int it = 0;
        bool dead = false;
        for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
            PjItem w;
            if (!item_valid(item, w)) continue;
            const int tile = (int)(item / cpt);
            const int rb = it & 1;
            const int nch = (w.m + kPjChunk - 1) / kPjChunk;
            // row exponents of the tile into buffer rb (the buffer of item
            // it - 2 is free once every converter warp has left that item)
            if (!dead && it >= 2) {
                bool ok = true;
                if (lane == 0) ok = mbar_wait_or(&rowfree[rb], (uint32_t)((it >> 1) - 1) & 1, &failed);
                if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) { dead = true; failed = 1; fail_tile = tile; }
            }
            if (!dead) {
                const int *re = ws.Qe(w.slot);
                for (int i = t; i < w.m; i += kPjConvThreads) rowe[rb][i] = (int16_t)re[i];
                __syncwarp();
                if (lane == 0) mbar_arrive(&rowready[rb]);
                bool ok = true;
                if (lane == 0) ok = mbar_wait_or(&rowready[rb], (uint32_t)(it >> 1) & 1, &failed);
                if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) { dead = true; failed = 1; fail_tile = tile; }
            }
            const int jj = (int)(item % cpt) * kPjCols + j;
            for (int kc = 0; kc < nch; ++kc, ++gc) {
                const int sd = (int)(gc % kPjDStages), b = (int)(gc & 1);
                if (!dead) {
                    bool ok = mbar_wait_or(&dfull[sd], (uint32_t)(gc / kPjDStages) & 1, &failed);
                    ok = ok && (gc < 2 ||
                                mbar_wait_or(&afree[b], (uint32_t)((gc >> 1) - 1) & 1, &failed));
                    if (!__all_sync(0xffffffffu, ok ? 1 : 0)) {
                        dead = true;
                        failed = 1;
                        fail_tile = tile;
                    }
                }
                if (dead) continue;
                // rows i0 .. i0 + 7 of column jj: box qd >> 1 (16 rows), its
                // 16-byte chunks (qd & 1) 4 + q, 128B-swizzled by row j & 7
                const uint8_t *box = Dst + (size_t)sd * kPjDBytes + (qd >> 1) * (kPjCols * 128);
                double2 v2[4];
                #pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int c16 = ((qd & 1) * 4 + q) ^ (j & 7);
                    v2[q] = *reinterpret_cast<const double2 *>(box + j * 128 + c16 * 16);
                }
                // the stage is free for the next copy once every warp has
                // its values
                __syncwarp();
                if (lane == 0) mbar_arrive(&dempty[sd]);
                const int i0 = kc * kPjChunk + 8 * qd;
                uint32_t lo[8], hi[8];
                #pragma unroll
                for (int q = 0; q < 4; ++q) {
                    #pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int i = i0 + 2 * q + e;
                        const double v = e ? v2[q].y : v2[q].x;
                        uint32_t l = 0u, h = 0u;
                        if (jj < w.n && i < w.m) {
                            // X = v 2^sh (exact): one multiply by 2^sh built
                            // from its exponent field, two beyond 2^1000
                            const int sh = 55 - rowe[rb][i];
                            double X;
                            if (sh <= 1000)
                                X = v * __hiloint2double((1023 + sh) << 20, 0);
                            else
                                X = (v * 0x1p1000) *
                                    __hiloint2double((1023 + sh - 1000) << 20, 0);
                            bytes56(X, l, h);
                        }
                        lo[2 * q + e] = l;
                        hi[2 * q + e] = h;
                    }
                }
                uint8_t *A = Abuf + b * kPjAbufBytes;
                const int off = (qd >> 1) * 2048 + (j >> 3) * 128 + (j & 7) * 16 + (qd & 1) * 8;
                #pragma unroll
                for (int s = 0; s < kPjSlices; ++s) {
                    const uint32_t *src = s < 4 ? lo : hi;
                    const int sb = s < 4 ? s : s - 4;
                    const uint32_t sel = (uint32_t)sb | ((uint32_t)(sb + 4) << 4);
                    const uint32_t a0 = __byte_perm(src[0], src[1], sel);
                    const uint32_t b0 = __byte_perm(src[2], src[3], sel);
                    const uint32_t a1 = __byte_perm(src[4], src[5], sel);
                    const uint32_t b1 = __byte_perm(src[6], src[7], sel);
                    *reinterpret_cast<uint2 *>(A + s * (kPjCols * kPjChunk) + off) =
                        make_uint2(__byte_perm(a0, b0, 0x5410), __byte_perm(a1, b1, 0x5410));
                }
                // each thread's digits visible to the tensor cores, then
                // one arrival per warp
                asm volatile("fence.proxy.async.shared::cta;");
                __syncwarp();
                if (lane == 0) mbar_arrive(&afull[b]);
            }
            // the row exponents of buffer rb are no longer read
            __syncwarp();
            if (lane == 0 && !dead) mbar_arrive(&rowfree[rb]);
            ++it;
        }
    } else if (warp == kPjProducerWarp) {
        // ------------------------------------------------------ producers
        // lane 0 streams D through its four-stage ring, lane 1 the Q'
        // slices through theirs; the two run independently
        if (lane < 2) {
            const bool is_d = lane == 0;
            const int nst = is_d ? kPjDStages : kPjQStages;
            uint64_t *fullb = is_d ? dfull : qfull;
            uint64_t *emptyb = is_d ? dempty : qempty;
            long long gc = 0, issued = 0;
            for (long long item = blockIdx.x; item < nitems && !failed; item += gridDim.x) {
                PjItem w;
                if (!item_valid(item, w)) continue;
                const int tile = (int)(item / cpt);
                const int j0 = (int)(item % cpt) * kPjCols;
                const int nch = (w.m + kPjChunk - 1) / kPjChunk;
                for (int kc = 0; kc < nch; ++kc, ++gc) {
                    const int sg = (int)(gc % nst);
                    if (gc >= nst &&
                        !mbar_wait_sleep(&emptyb[sg], (uint32_t)(gc / nst - 1) & 1, &failed, 32)) {
                        fail_tile = tile;
                        failed = 1;
                        break;
                    }
                    if (is_d) {
                        // D rows kc 32 .. + 31 of columns j0 .. j0 + 127: two
                        // boxes of 16 rows (128 bytes) x 128 columns
                        uint8_t *st = Dst + (size_t)sg * kPjDBytes;
                        mbar_expect_tx(&fullb[sg], kPjDBytes);
                        tma_load_3d(st, &dmap, kc * kPjChunk, j0, w.slot, &fullb[sg]);
                        tma_load_3d(st + kPjCols * 128, &dmap, kc * kPjChunk + 16, j0,
                                    w.slot, &fullb[sg]);
                    } else {
                        // the chunk's basis slices, per K half one 3.5 KB
                        // copy into blocks 7 .. 13 of that half's plane
                        mbar_expect_tx(&fullb[sg], kPjQBytes);
                        const uint8_t *src = ws.Qd(w.slot) + (size_t)kc * kPjQBytes;
                        uint8_t *dst = Qst + (size_t)sg * kPjQStage + 7 * kPjN * 16;
                        bulk_load(dst, src, kPjQData, &fullb[sg]);
                        bulk_load(dst + kPjPlane, src + kPjQData, kPjQData, &fullb[sg]);
                    }
                    issued = gc + 1;
                }
                if (failed) break;
            }
            if (failed) {
                int dummy = 0;
                for (long long q = issued > nst ? issued - nst : 0; q < issued; ++q)
                    mbar_wait_or(&fullb[q % nst], (uint32_t)(q / nst) & 1, &dummy);
            }
        }
    } else if (warp == kPjMmaWarp) {
        // ----------------------------------------------------------- MMA
        long long last = -1;
        if (lane == 0) {
            long long gc = 0;
            int it = 0;
            bool ok = true;
            for (long long item = blockIdx.x; ok && item < nitems && !failed;
                 item += gridDim.x) {
                PjItem w;
                if (!item_valid(item, w)) continue;
                const int tile = (int)(item / cpt);
                const int nch = (w.m + kPjChunk - 1) / kPjChunk;
                ok = it == 0 || mbar_wait_sleep(&accempty, (uint32_t)(it - 1) & 1, &failed, 32);
                for (int kc = 0; ok && kc < nch; ++kc, ++gc) {
                    const int sq = (int)(gc % kPjQStages), b = (int)(gc & 1);
                    if (!mbar_wait_or(&afull[b], (uint32_t)(gc >> 1) & 1, &failed) ||
                        !mbar_wait_or(&qfull[sq], (uint32_t)(gc / kPjQStages) & 1, &failed)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint8_t *A = Abuf + b * kPjAbufBytes;
                    const uint8_t *qs = Qst + (size_t)sq * kPjQStage;
                    #pragma unroll
                    for (int sl = 0; sl < kPjSlices; ++sl) {
                        const uint64_t da = umma_desc(smem_u32(A + sl * (kPjCols * kPjChunk)),
                                                      2048, 128);
                        // window of blocks 12 - sl .. 19 - sl: block w - 5
                        // holds slice w - sl
                        const uint64_t db = umma_desc(
                            smem_u32(qs + (12 - sl) * kPjN * 16), kPjPlane, 128);
                        mma_i8(tmem, da, db,
                               idesc_i8_ab(kPjCols, kPjAcc * kPjN, sl == kPjSlices - 1, true),
                               kc == 0 && sl == 0 ? 0 : 1);
                    }
                    mma_commit(&qempty[sq]);
                    mma_commit(&afree[b]);
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
            if (failed && last >= 0) {
                int dummy = 0;
                mbar_wait_or(&afree[last & 1], (uint32_t)(last >> 1) & 1, &dummy);
            }
        }
    } else {
        // ------------------------------------------------------ epilogue
        static_assert(kPjEpiWarp0 + 4 == kPjThreads / 32, "epilogue warps");
        const int lq = warp & 3;
        const int rr = 32 * lq + lane;
        int it = 0;
        for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
            PjItem w;
            if (!item_valid(item, w)) continue;
            const int tile = (int)(item / cpt);
            const bool ok = mbar_wait_sleep(&accfull, (uint32_t)it & 1, &failed, 256);
            if (!__all_sync(0xffffffffu, ok ? 1 : 0)) {
                if (lane == 0) fail_tile = tile;
                failed = 1;
                break;
            }
            tc_fence_after();
            const int jj = (int)(item % cpt) * kPjCols + rr;
            const int *fe = ws.Qf(w.slot);
            double *Bm = ws.B(w.slot);
            const int ldk = ws.ldK();
            for (int g = 0; g < (w.k1 + 7) / 8; ++g) {
                uint32_t v[kPjAcc][8];
                #pragma unroll
                for (int a = 0; a < kPjAcc; ++a)
                    tmem_ld8(tmem + ((uint32_t)(32 * lq) << 16) + a * kPjN + 8 * g, v[a]);
                asm volatile("tcgen05.wait::ld.sync.aligned;");
                if (jj < w.n) {
                    #pragma unroll
                    for (int c8 = 0; c8 < 8; ++c8) {
                        const int c = 8 * g + c8;
                        if (c >= w.k1) break;
                        long long H = 0, L = 0;
                        #pragma unroll
                        for (int a = kPjAcc - 1; a >= 4; --a) H = H * 256 + (long long)(int)v[a][c8];
                        #pragma unroll
                        for (int a = 3; a >= 0; --a) L = L * 256 + (long long)(int)v[a][c8];
                        const double T = fma((double)H, 0x1p32, (double)L);
                        Bm[(size_t)jj * ldk + c] = ldexp(T, fe[c] - 69);
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
    if (warp == kPjMmaWarp)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(256));
}

void launch_proj_prep(TileWork *d_tiles, int ntiles, Workspace ws,
                      cudaStream_t stream)
{
    k_proj_prep<<<ntiles, 256, 0, stream>>>(d_tiles, ws);
}

bool launch_proj_i8(TileWork *d_tiles, int ntiles, Workspace ws,
                    cudaStream_t stream)
{
    auto encode = tensor_map_encoder();
    if (encode == nullptr || ws.ldD() % 2 != 0 || ws.oQd == 0) return false;
    CUtensorMap dmap;
    {
        const cuuint64_t dims[3] = {(cuuint64_t)ws.m_max, (cuuint64_t)ws.n_max,
                                    (cuuint64_t)ntiles};
        const cuuint64_t strides[2] = {(cuuint64_t)ws.ldD() * sizeof(double),
                                       (cuuint64_t)ws.stride * sizeof(double)};
        const cuuint32_t box[3] = {16, (cuuint32_t)kPjCols, 1};
        const cuuint32_t estr[3] = {1, 1, 1};
        if (encode(&dmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, ws.D(0), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    static int sms = 0;
    if (sms == 0) {
        int dev = 0, count = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_proj_i8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kPjSmemBytes);
        sms = count > 0 ? count : 148;
    }
    const long long items = (long long)ntiles * ((ws.n_max + kPjCols - 1) / kPjCols);
    const int grid = (int)std::min<long long>(sms, items);
    if (grid > 0)
        k_proj_i8<<<grid, kPjThreads, kPjSmemBytes, stream>>>(dmap, d_tiles, ntiles,
                                                               ws);
    return true;
}

}  // namespace b200
