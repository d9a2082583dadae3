// Internal declarations shared by the engine and the TLR-product/error
// kernels: device copies of a problem's points, dense block jobs, and the
// device-resident record kept per STARSH_blrm.
#pragma once
#include <cuda_runtime.h>
#include <memory>
#include <mutex>
#include <vector>
#include "device_ctx.cuh"
#include "kernel_entry.cuh"
#include "b200_host.h"

namespace b200 {

// Device copies of the coordinates and pivots a kernel reads.
struct DevicePoints {
    DevKernel K{};
    std::vector<void *> owned;
    size_t h2d = 0;
    // host coordinates the device copy was made from (for tile ordering)
    const double *h_row = nullptr, *h_col = nullptr;
    long long h_row_count = 0, h_col_count = 0;
    ~DevicePoints()
    {
        for (void *p : owned) pool_free(p);
    }
    int upload(const void *host, size_t bytes, const void **dev,
               cudaStream_t s)
    {
        void *d = pool_alloc(bytes, s);
        if (d == nullptr)
            return cuda_fail(cudaErrorMemoryAllocation, "points");
        owned.push_back(d);
        if (bytes)
            B200_CUDA(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, s),
                      "cudaMemcpyAsync(points)");
        h2d += bytes;
        *dev = d;
        return STARSH_SUCCESS;
    }
};

struct BlockJob {
    long long row0, col0;
    int m, n;
    double *out;   // column-major, ld = m
};

// Device-resident factors of one STARSH_blrm.
struct Record {
    std::vector<void *> chunks;        // device allocations
    // factor chunks shared with other problems of the same batched call
    std::vector<std::shared_ptr<void>> shared;
    std::vector<double *> dU, dV;      // per far block (device)
    std::vector<double *> dD;          // per near block (device, or null)
    // Factor chunks in far-block order: the host mirror of U (V) is the
    // concatenation of the chunks' U (V) parts.
    // hU (hV): the part's host copy when it was downloaded as soon as its
    // batch finished (page-locked; U then V in one block), else null.
    struct Part {
        const double *U; size_t nu; const double *V; size_t nv;
        double *hU = nullptr, *hV = nullptr;
    };
    std::vector<Part> parts;
    size_t u_total = 0, v_total = 0, d_total = 0;
    bool host_filled = false;
    DevicePoints *points = nullptr;    // kept for onfly near blocks
    // the TLR-product plan (dmml_dfe.cu), built on the first product
    std::mutex plan_lock;
    std::shared_ptr<void> plan;
    ~Record()
    {
        for (Part &pt : parts)
            if (pt.hU) host_pinned_free(pt.hU);
        for (void *p : chunks) pool_free(p);
        delete points;
    }
};

void fill_kernel(DevKernel &K, const b200_kspec &sp);
int upload_problem(DevicePoints &dp, STARSH_problem *P, STARSH_cluster *R,
                   STARSH_cluster *C, cudaStream_t s);
// Generates dense blocks (column-major, ld = m) on stream s.
int gen_blocks(const DevKernel &K, const std::vector<BlockJob> &jobs,
               cudaStream_t s);
Record *find_record(const STARSH_blrm *M);
// B = alpha M A + beta B on the device (dmml_dfe.cu); the caller holds
// ctx.lock.
int dmml_device(STARSH_blrm *M, int nrhs, double alpha, const double *dA,
                int lda, double beta, double *dB, int ldb,
                cudaStream_t stream, Context &ctx);
// Registers a record for M (replacing none); used for matrices whose
// factors were uploaded from the host.
void add_record(const STARSH_blrm *M, Record *rec);

}  // namespace b200
