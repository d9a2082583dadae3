// starsh_b200_dense_rsvd_noalloc: randomized-SVD compression of one dense
// device tile with no device memory allocation.
//
// Some callers cannot call cudaMalloc at all: a host framework whose
// caching allocator owns all device memory (a second allocator would
// fragment it or exceed its budget), plugins that are handed device
// buffers but no right to allocate, and host threads that must not block
// on the allocator's implicit device synchronisation.  For them this entry
// point runs the same per-tile pipeline as the batched engine (engine.cu /
// rsvd_kernels.cu) on one tile whose scratch lives in a file-scope
// __device__ array of fixed size; the caller passes the tile and the output
// buffers.  Every step is a kernel launch or a device-to-device copy on the
// caller's stream: the tile record is written by a one-thread kernel from
// by-value arguments, so no host memory is read after the call returns.
//
// Limits: nrows, ncols <= 256 and min(maxrank + oversample, nrows, ncols)
// <= 96; larger sizes are rejected with STARSH_WRONG_PARAMETER.  The scratch
// array (about 2.1 MB) exists on every GPU that loads the library and stays
// allocated until the process exits.  All calls share it and it keeps the
// previous call's contents: the pipeline overwrites every field it reads,
// and two calls that overlap on the GPU (different streams, or different
// host threads) race on it.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "device_ctx.cuh"
#include "engine.cuh"
#include "starsh-b200.h"

namespace b200 {

constexpr int kNoAllocMaxDim = 256;
constexpr int kNoAllocMaxK = 96;

// Mirror of workspace_layout(): doubles per slot for the given maxima
// (every field rounded up to 32 doubles).
constexpr size_t round32(size_t n) { return (n + 31) & ~(size_t)31; }
constexpr size_t slot_doubles(size_t m, size_t n, size_t k)
{
    return round32(m * n) + 3 * round32(m * k) + 3 * round32(k * k) +
           2 * round32(k * n) + 2 * round32(k) + 2 * round32((k + 1) / 2) +
           round32(((m + 63) / 64) * ((n + 63) / 64)) + round32(m * k) +
           round32(m * ((n + 63) / 64));
}
constexpr size_t kSlotDoubles =
    slot_doubles(kNoAllocMaxDim, kNoAllocMaxDim, kNoAllocMaxK);
constexpr size_t kOmegaDoubles = round32((size_t)kNoAllocMaxDim * kNoAllocMaxK);
constexpr size_t kTileDoubles = round32((sizeof(TileWork) + 7) / 8);
constexpr size_t kDescDoubles = round32((sizeof(GemmDesc) + 7) / 8);
constexpr size_t kScratchDoubles =
    kSlotDoubles + kOmegaDoubles + kTileDoubles + kDescDoubles;

// The scratch.  Host code must not use this symbol as an address: on the
// host it is only a stand-in; the device address comes from
// cudaGetSymbolAddress (scratch_on_current_device below).
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Same seed as the batched engine, so a single-tile problem sees the same
// Gaussian sketch through both entry points.
static const unsigned long long kNoAllocOmegaSeed = 0x5354415253480001ull;

// The one tile's record: every field zero (the previous call's state is
// gone), then the shape, sketch width and the caller's maxrank and tol.
__global__ void k_noalloc_tile(TileWork *t, int m, int n, int k, int maxrank,
                               double tol)
{
    TileWork w;
    memset(&w, 0, sizeof(w));
    w.m = m;
    w.n = n;
    w.k = k;
    w.slot = 0;
    w.maxrank = maxrank;
    w.tol = tol;
    *t = w;
}

constexpr int kMaxDevices = 64;
static double *g_scratch_ptr[kMaxDevices];
static std::mutex g_scratch_lock;

// Device address of the scratch on the current device, looked up once per
// device (with that device current) on the first call.
static int scratch_on_current_device(double **out)
{
    int dev = 0;
    B200_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device index out of range for the no-allocation entry");
        return STARSH_WRONG_PARAMETER;
    }
    std::lock_guard<std::mutex> g(g_scratch_lock);
    if (g_scratch_ptr[dev] == nullptr) {
        void *p = nullptr;
        B200_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch),
                  "cudaGetSymbolAddress(no-alloc scratch)");
        g_scratch_ptr[dev] = (double *)p;
    }
    *out = g_scratch_ptr[dev];
    return STARSH_SUCCESS;
}

}  // namespace b200

using namespace b200;

extern "C" int starsh_b200_dense_rsvd_noalloc(const double *dD, int nrows,
                                              int ncols, int ldd, int maxrank,
                                              int oversample, double tol,
                                              double *dU, double *dV,
                                              int *d_rank, void *stream)
{
    if (dD == nullptr || dU == nullptr || dV == nullptr || d_rank == nullptr ||
        nrows <= 0 || ncols <= 0 || ldd < nrows || maxrank < 0 ||
        oversample <= 0 || !(tol >= 0.0)) {
        set_error("starsh_b200_dense_rsvd_noalloc: invalid argument");
        return STARSH_WRONG_PARAMETER;
    }
    const int k = std::min(maxrank + oversample, std::min(nrows, ncols));
    if (nrows > kNoAllocMaxDim || ncols > kNoAllocMaxDim || k > kNoAllocMaxK) {
        char msg[200];
        snprintf(msg, sizeof(msg),
                 "starsh_b200_dense_rsvd_noalloc: tile %dx%d with sketch width "
                 "%d exceeds the fixed scratch (rows, cols <= %d, width <= %d)",
                 nrows, ncols, k, kNoAllocMaxDim, kNoAllocMaxK);
        set_error(msg);
        return STARSH_WRONG_PARAMETER;
    }
    double *scratch = nullptr;
    int info = scratch_on_current_device(&scratch);
    if (info) return info;
    cudaStream_t s = (cudaStream_t)stream;

    Workspace ws{};
    const size_t stride = workspace_layout(ws, nrows, ncols, k, true);
    if (stride > kSlotDoubles) {
        set_error("starsh_b200_dense_rsvd_noalloc: scratch layout overflow");
        return STARSH_UNKNOWN_ERROR;
    }
    ws.base = scratch;
    ws.stride = stride;
    double *omega = scratch + kSlotDoubles;
    TileWork *dt = (TileWork *)(omega + kOmegaDoubles);
    GemmDesc *dd = (GemmDesc *)((double *)dt + kTileDoubles);

    k_noalloc_tile<<<1, 1, 0, s>>>(dt, nrows, ncols, k, maxrank, tol);
    B200_CUDA(cudaMemcpy2DAsync(ws.D(0), (size_t)ws.ldD() * sizeof(double), dD,
                                (size_t)ldd * sizeof(double),
                                (size_t)nrows * sizeof(double), ncols,
                                cudaMemcpyDeviceToDevice, s),
              "no-alloc tile copy");
    launch_gaussian(omega, ncols, k, ncols, kNoAllocOmegaSeed, s);

    const OutArena none{nullptr, nullptr};
    const OutArena out{dU, dV};
    auto gemm = [&](GemmStep step, bool ta, bool tb, int mm, int nn,
                    OutArena o) -> int {
        make_gemm_descs(step, dt, 1, ws, omega, ncols, o, dd, s);
        return gemm_f64_batched(ta, tb, dd, 1, mm, nn, s) == cudaSuccess
                   ? STARSH_SUCCESS
                   : cuda_fail(cudaGetLastError(), "no-alloc gemm");
    };
    const int m = nrows, n = ncols;
    if ((info = gemm(STEP_SKETCH, false, false, m, k, none))) return info;
    if ((info = gemm(STEP_GRAM_Y, true, false, k, k, none))) return info;
    launch_pivchol(0, dt, dt, 1, ws, s);
    launch_gather_cols(0, dt, 1, ws, s);
    if ((info = gemm(STEP_Q1, false, false, m, k, none))) return info;
    if ((info = gemm(STEP_GRAM_Q1, true, false, k, k, none))) return info;
    launch_chol_inv(0, dt, 1, ws, s);
    if ((info = gemm(STEP_Q, false, false, m, k, none))) return info;
    if ((info = gemm(STEP_RES_Z, true, false, k, k, none))) return info;
    if ((info = gemm(STEP_RES_Y, false, false, m, k, none))) return info;
    if ((info = gemm(STEP_GRAM_YR, true, false, k, k, none))) return info;
    launch_pivchol(1, dt, dt, 1, ws, s);
    launch_gather_cols(1, dt, 1, ws, s);
    if ((info = gemm(STEP_Q1B, false, false, m, k, none))) return info;
    if ((info = gemm(STEP_RES_Z2, true, false, k, k, none))) return info;
    if ((info = gemm(STEP_RES_Q1B, false, false, m, k, none))) return info;
    if ((info = gemm(STEP_GRAM_Q1B, true, false, k, k, none))) return info;
    launch_chol_inv(1, dt, 1, ws, s);
    if ((info = gemm(STEP_QB, false, false, m, k, none))) return info;
    launch_merge_basis(dt, 1, s);
    if ((info = gemm(STEP_PROJECT, true, false, k, n, none))) return info;
    if ((info = gemm(STEP_GRAM_B, false, true, k, k, none))) return info;
    launch_pivchol(2, dt, dt, 1, ws, s);
    launch_jacobi(dt, 1, ws, s, nullptr);
    if ((info = gemm(STEP_ROTATE, true, false, k, n, none))) return info;
    launch_rank_cut(dt, 1, ws, s);
    // One tile: its factors start at offset 0 of the caller's buffers, so
    // the output kernels run without a host round trip (rank <= 0 skips).
    launch_select_w(dt, 1, ws, s);
    if ((info = gemm(STEP_OUT_U, false, false, m, k, out))) return info;
    launch_write_v(dt, 1, ws, out, s);
    B200_CUDA(cudaMemcpyAsync(d_rank, &dt->rank, sizeof(int),
                              cudaMemcpyDeviceToDevice, s),
              "no-alloc rank");
    B200_CUDA(cudaGetLastError(), "no-alloc launches");
    return STARSH_SUCCESS;
}
