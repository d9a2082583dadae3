// Batched FP64 GEMM (see gemm_f64.cuh).
//
// CTA tile 64 x 64, K step 16, 8 warps in a 2 (M) x 4 (N) grid, warp tile
// 32 x 16 = 4 x 2 fragments of the m8n8k4 DMMA.  Operand tiles are staged
// in shared memory as [row][k] (A) and [col][k] (B) with row stride 20,
// double-buffered, the next K tile is fetched into registers while the
// current one is multiplied.  Global loads are coalesced along whichever
// dimension is contiguous for the given transpose flag.
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

template <bool TA, bool TB>
__global__ void __launch_bounds__(kGemmThreads)
k_gemm_f64(const GemmDesc *__restrict__ descs, int tiles_n)
{
    const GemmDesc d = descs[blockIdx.y];
    const int tm = blockIdx.x / tiles_n;
    const int tn = blockIdx.x % tiles_n;
    const int m0 = tm * kGemmBM, n0 = tn * kGemmBN;
    if (m0 >= d.M || n0 >= d.N) return;

    __shared__ double As[2][kGemmBM * kGemmLds];
    __shared__ double Bs[2][kGemmBN * kGemmLds];

    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = (warp & 1) * 32;   // warp row offset in the CTA tile
    const int wn = (warp >> 1) * 16;  // warp column offset

    double acc[4][2][2];
    #pragma unroll
    for (int i = 0; i < 4; ++i)
        #pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    double ra[4], rb[4];
    // Element coordinates this thread loads, per register slot r:
    //   A: (row am + ..., k ak + ...), B: (col bn + ..., k bk + ...).
    auto load_tiles = [&](int k0) {
        #pragma unroll
        for (int r = 0; r < 4; ++r) {
            int row, kk;
            if (!TA) { row = t & 63; kk = (t >> 6) + 4 * r; }
            else     { kk = t & 15; row = (t >> 4) + 16 * r; }
            const int gm = m0 + row, gk = k0 + kk;
            double v = 0.0;
            if (gm < d.M && gk < d.K)
                v = TA ? d.A[(size_t)gm * d.lda + gk]
                       : d.A[(size_t)gk * d.lda + gm];
            ra[r] = v;
        }
        #pragma unroll
        for (int r = 0; r < 4; ++r) {
            int col, kk;
            if (!TB) { kk = t & 15; col = (t >> 4) + 16 * r; }
            else     { col = t & 63; kk = (t >> 6) + 4 * r; }
            const int gn = n0 + col, gk = k0 + kk;
            double v = 0.0;
            if (gn < d.N && gk < d.K)
                v = TB ? d.B[(size_t)gk * d.ldb + gn]
                       : d.B[(size_t)gn * d.ldb + gk];
            rb[r] = v;
        }
    };
    auto store_tiles = [&](int buf) {
        #pragma unroll
        for (int r = 0; r < 4; ++r) {
            int row, kk;
            if (!TA) { row = t & 63; kk = (t >> 6) + 4 * r; }
            else     { kk = t & 15; row = (t >> 4) + 16 * r; }
            As[buf][row * kGemmLds + kk] = ra[r];
        }
        #pragma unroll
        for (int r = 0; r < 4; ++r) {
            int col, kk;
            if (!TB) { kk = t & 15; col = (t >> 4) + 16 * r; }
            else     { col = t & 63; kk = (t >> 6) + 4 * r; }
            Bs[buf][col * kGemmLds + kk] = rb[r];
        }
    };

    const int ktiles = (d.K + kGemmBK - 1) / kGemmBK;
    if (ktiles > 0) {
        load_tiles(0);
        store_tiles(0);
        __syncthreads();
    }
    for (int kt = 0; kt < ktiles; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < ktiles) load_tiles((kt + 1) * kGemmBK);
        #pragma unroll
        for (int kk = 0; kk < kGemmBK; kk += 4) {
            double af[4], bf[2];
            #pragma unroll
            for (int i = 0; i < 4; ++i)
                af[i] = As[buf][(wm + i * 8 + g) * kGemmLds + kk + tig];
            #pragma unroll
            for (int j = 0; j < 2; ++j)
                bf[j] = Bs[buf][(wn + j * 8 + g) * kGemmLds + kk + tig];
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

cudaError_t gemm_f64_batched(bool ta, bool tb, const GemmDesc *d_desc,
                             int batch, int max_m, int max_n,
                             cudaStream_t stream)
{
    if (batch <= 0 || max_m <= 0 || max_n <= 0) return cudaSuccess;
    const int tiles_m = (max_m + kGemmBM - 1) / kGemmBM;
    const int tiles_n = (max_n + kGemmBN - 1) / kGemmBN;
    for (int b0 = 0; b0 < batch; b0 += 65535) {
        const int nb = batch - b0 < 65535 ? batch - b0 : 65535;
        dim3 grid(tiles_m * tiles_n, nb);
        const GemmDesc *dd = d_desc + b0;
        if (!ta && !tb)
            k_gemm_f64<false, false><<<grid, kGemmThreads, 0, stream>>>(dd, tiles_n);
        else if (ta && !tb)
            k_gemm_f64<true, false><<<grid, kGemmThreads, 0, stream>>>(dd, tiles_n);
        else if (!ta && tb)
            k_gemm_f64<false, true><<<grid, kGemmThreads, 0, stream>>>(dd, tiles_n);
        else
            k_gemm_f64<true, true><<<grid, kGemmThreads, 0, stream>>>(dd, tiles_n);
    }
    return cudaGetLastError();
}

}  // namespace b200
