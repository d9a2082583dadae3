// Process-wide device context of libstarsh_b200: the CUDA stream all work
// runs on, grow-only device buffers that are reused across calls, the last
// error string and the statistics of the last approximation.
#pragma once
#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include "starsh-b200.h"

namespace b200 {

struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;   // the stream it was allocated on
    // Ensures capacity, stream-ordered on s (from the device's cached
    // pool: growing never synchronises the device); contents are not
    // preserved.  Returns false on OOM.
    bool reserve(size_t need, cudaStream_t s);
    void release();
};

struct Context {
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;   // second stream for overlapping launches
    cudaStream_t copy = nullptr;   // device-to-host copies of finished batches
    DeviceBuffer workspace;    // per-slot scratch of the engine
    DeviceBuffer tiles;        // TileWork array of a batch
    DeviceBuffer descs;        // GemmDesc array of a batch
    DeviceBuffer omega;        // Gaussian sketch matrix
    DeviceBuffer flag;         // round flag of the adaptive sketch
    DeviceBuffer act;          // a round's sampling tiles, by round slot
    void *stage[2] = {nullptr, nullptr};     // pinned D2H staging buffers
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    DeviceBuffer kernels;      // DevKernel table of a batch's problems
    DeviceBuffer omega8;       // int8 sketch matrix of the adaptive engine
    int omega8_rows = 0, omega8_cols = 0, omega8_ld = 0;
    int omega_rows = 0, omega_cols = 0;   // shape Omega was generated for
    size_t workspace_cap = (size_t)-1;    // most workspace one batch may use
    // page-locked staging of a batch's tile records (two, used in turn, so
    // that their uploads do not wait for the stream)
    void *tiles_pin[2] = {nullptr, nullptr};
    size_t tiles_pin_bytes = 0;
    // page-locked host memory mapped into the device, for the small reads
    // the host waits on (a round's sampling count, a batch's tile
    // records): a kernel stores them there, so they do not queue on a copy
    // engine behind the batch downloads of `copy`
    void *mapped = nullptr;
    void *mapped_dev = nullptr;
    std::mutex lock;           // one approximation / dmml at a time
};

// Initialises (once) and returns the context; nullptr if no usable GPU.
// A thread that installed its own context (set_thread_context) gets that
// one instead: its own streams and reusable buffers, so that several host
// threads (the serving workers) keep work on the GPU at the same time.
Context *context();
Context *context_new_private();
void context_free_private(Context *c);
void set_thread_context(Context *c);

// Stream-ordered device allocation from the device's memory pool, whose
// freed memory stays cached for the next call (repeated approximations do
// not go back to the driver, which can stall the stream for a long time).
// pool_alloc returns nullptr on failure; pool_free releases on the
// library stream.
void *pool_alloc(size_t bytes, cudaStream_t s);
void pool_free(void *p);

// Page-locked host memory for host mirrors, kept after use (up to a cap)
// so that repeated approximations copy straight into memory that is
// already pinned.  host_pinned_free returns false for a pointer the pool
// did not hand out.
void *host_pinned_alloc(size_t bytes);
bool host_pinned_free(void *p);

// Records a CUDA error (with the call site) as the library's last error and
// returns the matching STARSH error code.
int cuda_fail(cudaError_t err, const char *what);
void set_error(const std::string &msg);

// Statistics of the last approximation on this thread.
starsh_b200_stats &thread_stats();

// Counts launches of the library's own kernels (for reporting).
void count_launch(long long n = 1);
long long launch_count();

}  // namespace b200

#define B200_CUDA(call, what)                                   \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return b200::cuda_fail(e_, what); \
    } while (0)
