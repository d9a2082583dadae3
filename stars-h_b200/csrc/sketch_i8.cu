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
// rounded to q = round(x 2^39) and written with an offset as the 40-bit
// unsigned integer q' = q + 2^39, whose five bytes u_0..u_4 are the digits:
//     D_ij = 2^(e_i - 39) (sum_s 256^s u_s[i, j] - 2^39) + err,
//     |err| <= 2^-40 2^e_i.
// Each digit matrix times Omega is an exact uint8 x int8 -> int32 product
// (|sum| <= 255 * 127 * n < 2^31 for n <= 8192) on tcgen05.mma kind::i8,
// accumulated in TMEM, one accumulator per digit.  The epilogue removes the
// offset exactly (2^39 = 128 * 2^32: the top digit's product less 128 times
// the column sums of Omega), recombines the digits in int64 (exact, |T| <
// 2^61) and converts once:
//     Y_ic = 2^(e_i - 39) T_ic,  T_ic = sum_s 256^s P_s - 2^39 sum_j Omega_jc.
// The only error is the rounding of q: 2^-40 of the row maximum per entry,
// far below the tolerance-driven thresholds of the adaptive basis (the
// rank decision itself uses the FP64 projection and the exact block norm).
//
// One CTA per (tile, 128-row block), 512 threads.  The tile's rows are
// read from HBM once, in K chunks of 32 columns, each brought into a
// three-stage shared-memory buffer by one TMA tile copy (the copies of the
// next two chunks overlap the work on this one); every thread converts 8
// columns of one row into digits and stores them in the no-swizzle K-major
// core-matrix layout; one thread issues the 5 MMAs (M 128, N nc, K 32) of
// the chunk and commits them to the chunk buffer's mbarrier, so the
// conversion of the next chunk overlaps the MMAs (two digit buffers); the
// chunks are handed over through mbarriers, without block-wide barriers.
// Omega's nc columns for the tile (nc x n bytes) stay in shared memory.
#include <cstdint>
#include <cuda.h>
#include <cudaTypedefs.h>
#include "engine.cuh"

namespace b200 {

constexpr int kSlices = 5;             // bytes (digits) per entry
constexpr int kSkRows = 128;           // rows per CTA (MMA M)
constexpr int kSkChunk = 32;           // K columns per chunk (one MMA K)
constexpr int kSkThreads = 512;
constexpr int kSkMaxN = 64;            // sketch columns per launch
constexpr int kStages = 3;             // D chunks in flight (TMA stages)

// Shared-memory descriptor of a K-major operand without swizzle:
// core matrices of 8 rows x 16 bytes (128 contiguous bytes), lbo = byte
// distance between the two 16-byte K halves of one MMA, sbo = byte
// distance between consecutive 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo,
                                              uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;            // descriptor version (sm_100)
    return d;                          // base offset 0, no swizzle
}

// Instruction descriptor: int32 accumulator, unsigned int8 A (digits),
// signed int8 B (Omega), both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_i8(int n)
{
    return (2u << 4) | (0u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(kSkRows >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da,
                                       uint64_t db, uint32_t idesc,
                                       int accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                 :: "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(mbar)));
}

__device__ __forceinline__ bool mbar_try(uint64_t *mbar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred P1;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(mbar)), "r"(parity) : "memory");
    return ok != 0;
}

// Waits for the completion of the phase of the given parity; gives up
// after about two seconds and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity)
{
    const long long t0 = clock64();
    while (!mbar_try(mbar, parity))
        if (clock64() - t0 > (1ll << 32)) return false;
    return true;
}

// The same, also giving up as soon as *abort is set by another thread.
__device__ __forceinline__ bool mbar_wait_or(uint64_t *mbar, uint32_t parity,
                                             volatile int *abort)
{
    const long long t0 = clock64();
    while (!mbar_try(mbar, parity)) {
        if (*abort) return false;
        if (clock64() - t0 > (1ll << 32)) return false;
    }
    return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *mbar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];"
                 :: "r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]),
                   "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
}

// Digits of 8 entries x in (-1, 1): q' = round(x 2^39) + 2^39 < 2^40 by
// the magic-number rounding (adding 1.5 2^52 leaves the integer in the low
// mantissa bits), then byte s of the four q' of columns 4c .. 4c + 3 goes
// to word w[s][c].
__device__ __forceinline__ void digits8(const double (&y)[8],
                                        uint32_t (&w)[kSlices][2])
{
    // y = x 2^39 + 2^39 + 1.5 2^52 (one rounding): the low word of y's bit
    // pattern is the low word of q', the high word less 0x43380000 its top
    // byte (q' = 2^40 after rounding is clamped to 2^40 - 1)
    uint32_t lo[8], hi[8];
    #pragma unroll
    for (int c = 0; c < 8; ++c) {
        lo[c] = (uint32_t)__double2loint(y[c]);
        hi[c] = (uint32_t)__double2hiint(y[c]) - 0x43380000u;
        if (hi[c] > 255u) { hi[c] = 255u; lo[c] = 0xFFFFFFFFu; }
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

// One TMA tile copy (this CTA only) of the 128 x 32 FP64 box at (row0,
// col0, slot) of the workspace's D tensor into shared memory, completing
// on mbar with its byte count.
__device__ __forceinline__ void tma_load_d(void *dst, const CUtensorMap *map,
                                           int row0, int col0, int slot,
                                           uint64_t *mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_u32(mbar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1, {%2, %3, %4}], [%5];"
                 :: "r"(smem_u32(dst)), "l"(map), "r"(row0), "r"(col0), "r"(slot),
                    "r"(smem_u32(mbar))
                 : "memory");
}

// Y(:, 0:bcur) of every tile with an active round = D * Omega8(:, cols_done
// + (0:nc)), rows in 128-row blocks (blockIdx.x), tiles in blockIdx.y.
__global__ void __launch_bounds__(kSkThreads, 1)
k_sketch_i8(const __grid_constant__ CUtensorMap dmap,
            const TileWork *__restrict__ tiles, Workspace ws,
            const int8_t *__restrict__ om8, int ld_om8, int om8_cols, int nc)
{
    extern __shared__ __align__(1024) uint8_t sk_smem_raw[];
    __shared__ __align__(8) uint64_t mbar[2];     // MMAs done with A buffer
    __shared__ __align__(8) uint64_t stbar[kStages];  // D chunk landed in stage
    __shared__ __align__(8) uint64_t abar[2];     // all digits of a chunk written
    __shared__ uint32_t tmem_base;
    __shared__ volatile int failed;
    __shared__ int colsum[kSkMaxN];

    const TileWork tw = tiles[blockIdx.y];
    const int row0 = blockIdx.x * kSkRows;
    if (tw.bcur <= 0 || row0 >= tw.m) return;            // uniform
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int r = t & (kSkRows - 1), qd = t >> 7;        // row, column quarter
    const int n = tw.n, m = tw.m;
    const int npad = (n + kSkChunk - 1) / kSkChunk * kSkChunk;
    const int nchunks = npad / kSkChunk;
    constexpr int kAbuf = kSlices * kSkRows * kSkChunk;  // bytes per buffer
    constexpr int kStage = kSkRows * kSkChunk;           // doubles per stage
    // 1024-byte aligned base (the launch adds 1 KB of slack)
    uint8_t *sk_smem = sk_smem_raw + ((1024u - (smem_u32(sk_smem_raw) & 1023u)) & 1023u);
    uint8_t *Abuf = sk_smem;                             // [2][kSlices][4 KB]
    uint8_t *Bsm = sk_smem + 2 * kAbuf;                  // nc x npad
    // raw FP64 chunks (column-major, 128 rows), kStages stages: the copies
    // of chunks kc + 1 .. kc + kStages - 1 run while chunk kc is converted
    const int npad_max = (ws.n_max + kSkChunk - 1) / kSkChunk * kSkChunk;
    double *stage = reinterpret_cast<double *>(Bsm + (size_t)nc * npad_max);
    const uint32_t ncols_alloc = nc * kSlices <= 128 ? 128
                               : nc * kSlices <= 256 ? 256 : 512;
    constexpr uint32_t kStageBytes = kStage * sizeof(double);

    if (t == 0) {
        failed = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&mbar[0])), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&mbar[1])), "r"(1));
        for (int q = 0; q < kStages; ++q)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&stbar[q])), "r"(1));
        for (int q = 0; q < 2; ++q)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&abar[q])), "r"(kSkThreads));
        asm volatile("fence.mbarrier_init.release.cluster;");
        // the first kStages chunks of D are requested before anything else
        // (Omega, row scales, TMEM): their copies overlap that set-up
        for (int q = 0; q < kStages && q < nchunks; ++q)
            tma_load_d(stage + q * kStage, &dmap, row0, q * kSkChunk, tw.slot,
                       &stbar[q], kStageBytes);
    }
    if (t < kSkMaxN) colsum[t] = 0;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_base)), "r"(ncols_alloc));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    // Omega8 columns cols_done .. cols_done + nc of this tile, K-major core
    // matrices: byte (c, k) at (k / 16) (nc 16) + (c / 8) 128 + (c % 8) 16
    // + k % 16.  Columns past Omega8's width are zero.  colsum[c] sums the
    // column as stored (padding rows included: their digits carry the
    // offset too).
    {
        const int c0 = tw.cols_done;
        const int units = nc * (npad / 16);
        for (int u = t; u < units; u += kSkThreads) {
            const int c = u % nc, k16 = u / nc;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (c0 + c < om8_cols)
                v = *reinterpret_cast<const uint4 *>(
                    om8 + (size_t)(c0 + c) * ld_om8 + (size_t)k16 * 16);
            *reinterpret_cast<uint4 *>(Bsm + (size_t)k16 * (nc * 16) +
                                       (c >> 3) * 128 + (c & 7) * 16) = v;
            int sum = 0;
            const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
            #pragma unroll
            for (int q = 0; q < 4; ++q)
                sum += __dp4a((int)wv[q], 0x01010101, 0);
            atomicAdd(&colsum[c], sum);
        }
    }
    // row scale 2^-e, e the exponent of the row's largest |D_ij|
    int e = 0;
    const int i = row0 + r;
    if (i < m) {
        const int ncb = (ws.n_max + 63) / 64;
        const double *rm = ws.Rmx(tw.slot) + (size_t)i * ncb;
        double mx = 0.0;
        for (int cb = 0; cb < (n + 63) / 64; ++cb) mx = fmax(mx, rm[cb]);
        if (mx > 0.0) frexp(mx, &e);
    }
    // y = D 2^(39 - e) + 2^39 + 1.5 2^52 in one fma (see digits8)
    const double scale39 = ldexp(1.0, 39 - e);
    const double magic = 0x1.8p52 + 0x1p39;
    asm volatile("fence.proxy.async.shared::cta;");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    const double *D = ws.D(tw.slot);
    const int ldD = ws.ldD();
    const uint32_t idesc = idesc_i8(nc);
    // chunk kc of D (128 rows x 32 columns) lands in stage kc % kStages by
    // one TMA copy; rows past m_max / columns past n_max read as zero, rows in
    // [m, m_max) and columns in [n, n_max) are masked below.
    // No block-wide barrier per chunk: every thread waits for its chunk's
    // data (stbar) and for the MMAs that read its digit buffer two chunks
    // ago (mbar), writes its digits and arrives on abar; thread 0 alone
    // waits for all 512 arrivals, issues the chunk's MMAs and the TMA copy
    // of chunk kc + kStages into the stage chunk kc has just left (every
    // converter has read its values before arriving), so kStages chunks
    // are in flight.  Each wait gives up after a bound or as soon as
    // another thread has given up (failed).
    // thread 0's view: the last chunk whose MMAs it committed, how many
    // chunks it has requested and how many of those it has seen land
    int last_commit = -1;
    int issued = min(kStages, nchunks), landed = 0;
    for (int kc = 0; kc < nchunks; ++kc) {
        const int b = kc & 1;
        const int sg = kc % kStages;
        bool ok = mbar_wait_or(&stbar[sg], (kc / kStages) & 1, &failed);
        if (ok && t == 0) landed = kc + 1;
        ok = ok && (kc < 2 || mbar_wait_or(&mbar[b], ((kc >> 1) - 1) & 1, &failed));
        if (ok) {
            // this thread: row r, columns 8 qd .. 8 qd + 7 of the chunk
            const double *st = stage + sg * kStage;
            double x[8];
            #pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int j = kc * kSkChunk + 8 * qd + c;
                const double v = (i < m && j < n) ? st[(8 * qd + c) * kSkRows + r] : 0.0;
                x[c] = fma(v, scale39, magic);
            }
            uint32_t w[kSlices][2];
            digits8(x, w);
            uint8_t *A = Abuf + b * kAbuf;
            #pragma unroll
            for (int s = 0; s < kSlices; ++s)
                *reinterpret_cast<uint2 *>(A + s * (kSkRows * kSkChunk) +
                                           (qd >> 1) * 2048 + (r >> 3) * 128 +
                                           (r & 7) * 16 + (qd & 1) * 8) =
                    make_uint2(w[s][0], w[s][1]);
            asm volatile("fence.proxy.async.shared::cta;");
        }
        mbar_arrive(&abar[b]);
        if (!ok) { failed = 1; break; }
        if (t == 0) {
            if (!mbar_wait_or(&abar[b], (kc >> 1) & 1, &failed)) {
                failed = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            uint8_t *A = Abuf + b * kAbuf;
            #pragma unroll
            for (int s = 0; s < kSlices; ++s) {
                const uint64_t da = umma_desc(
                    smem_u32(A + s * (kSkRows * kSkChunk)), 2048, 128);
                const uint64_t db = umma_desc(
                    smem_u32(Bsm + (size_t)(kc * 2) * (nc * 16)), nc * 16, 128);
                mma_i8(tmem + s * nc, da, db, idesc, kc > 0);
            }
            mma_commit(&mbar[b]);
            last_commit = kc;
            const int pf = kc + kStages;
            if (pf < nchunks) {
                asm volatile("fence.proxy.async.shared::cta;");
                tma_load_d(stage + (pf % kStages) * kStage, &dmap, row0,
                           pf * kSkChunk, tw.slot, &stbar[pf % kStages],
                           kStageBytes);
                issued = pf + 1;
            }
        }
        if (failed) break;
    }
    // the last commit covers every earlier MMA; after a failure thread 0
    // waits for the MMAs it issued before TMEM is released
    if (!failed) {
        const int last = nchunks - 1;
        if (!mbar_wait_or(&mbar[last & 1], (last >> 1) & 1, &failed)) failed = 1;
    } else if (t == 0) {
        // after a failure: the MMAs issued and the D copies still in
        // flight into shared memory finish (bounded waits) before the CTA
        // releases TMEM and exits
        int dummy = 0;
        if (last_commit >= 0)
            mbar_wait_or(&mbar[last_commit & 1], (last_commit >> 1) & 1, &dummy);
        for (int q = landed; q < issued; ++q)
            mbar_wait_or(&stbar[q % kStages], (q / kStages) & 1, &dummy);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    // warp w reads TMEM lanes 32 (w % 4) .. + 31 (rows) and the columns of
    // group w / 4 (16 columns each)
    const int lq = warp & 3, grp = warp >> 2;
    if (!failed && grp < nc / 16) {
        double *Y = ws.Y(tw.slot);
        const int ldY = ws.ldM();
        const int rr = row0 + 32 * lq + lane;
        // r = t & 127 = 32 (w % 4) + lane: this thread's own row, so its
        // exponent e is the row's
        const int er = e;
        uint32_t v[kSlices][16];
        #pragma unroll
        for (int s = 0; s < kSlices; ++s)
            tmem_ld16(tmem + ((uint32_t)(32 * lq) << 16) + s * nc + 16 * grp, v[s]);
        asm volatile("tcgen05.wait::ld.sync.aligned;");
        if (rr < m) {
            const double sc = ldexp(1.0, er - 39);
            #pragma unroll
            for (int c = 0; c < 16; ++c) {
                const int col = 16 * grp + c;
                long long T = (long long)(int)v[4][c] - 128ll * colsum[col];
                #pragma unroll
                for (int s = 3; s >= 0; --s) T = T * 256 + (long long)(int)v[s][c];
                if (col < tw.bcur) Y[(size_t)col * ldY + rr] = (double)T * sc;
            }
        }
    }
    if (failed && t == 0) {
        TileWork *tr = const_cast<TileWork *>(tiles) + blockIdx.y;
        atomicOr(&tr->status, TILE_MMA_TIMEOUT);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(ncols_alloc));
}

size_t sketch_i8_smem(int nc, int n_max)
{
    const int npad = (n_max + kSkChunk - 1) / kSkChunk * kSkChunk;
    return 2 * (size_t)kSlices * kSkRows * kSkChunk + (size_t)nc * npad +
           kStages * (size_t)kSkRows * kSkChunk * sizeof(double) + 1024;
}

bool sketch_i8_fits(int nc, int n_max)
{
    return nc > 0 && nc <= kSkMaxN && n_max <= 8192 &&
           sketch_i8_smem((nc + 15) / 16 * 16, n_max) <= 227 * 1024;
}

// Tensor map of the batch's D blocks as one 3-D FP64 tensor (rows, columns,
// slots) with a 128 x 32 x 1 box; needs an even leading dimension (16-byte
// strides).  Encoded through the driver entry point of the runtime.
static bool d_tensor_map(CUtensorMap *map, const Workspace &ws, int nslots)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (encode == nullptr) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn,
                                    cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || fn == nullptr) {
            cudaGetLastError();
            return false;
        }
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    if (ws.ldD() % 2 != 0) return false;
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

bool launch_sketch_i8(const TileWork *d_tiles, int ntiles, Workspace ws,
                      const int8_t *om8, int ld_om8, int om8_cols, int ncols,
                      cudaStream_t stream)
{
    CUtensorMap map;
    if (!d_tensor_map(&map, ws, ntiles)) return false;
    const int nc = (ncols + 15) / 16 * 16;
    const size_t smem = sketch_i8_smem(nc, ws.n_max);
    cudaFuncSetAttribute(k_sketch_i8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    dim3 grid((ws.m_max + kSkRows - 1) / kSkRows, ntiles);
    k_sketch_i8<<<grid, kSkThreads, smem, stream>>>(map, d_tiles, ws, om8,
                                                    ld_om8, om8_cols, nc);
    return true;
}

}  // namespace b200
