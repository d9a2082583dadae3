// Serving loop: approximation requests admitted by an HBM budget and run in
// shared batches (continuous batching), each followed by its TLR-by-dense
// products on the resident factors.
//
// Worker threads (three by default, STARSH_B200_SERVER_WORKERS) own the
// GPU work, each on its own engine context (streams and reusable buffers),
// so that several groups are on the GPU at the same time and their
// launches interleave.  A group's work is capped (5e8 matrix entries,
// STARSH_B200_SERVER_GROUP_ENTRIES; its first request always goes in).  Requests wait in FIFO order; a worker that becomes free
// admits, from the head of the queue, every request whose estimated device
// footprint still fits in the budget next to the results that are resident
// and the groups other workers are running, and runs them as one
// starsh_b200_approximate_batch() call: their tiles share every launch.
// Requests that arrive while groups are on the GPU are admitted by the next
// free worker, as memory allows.  After its group, each request's products
// B = M A run on the device (same worker, same stream) and the request
// completes (latency = submit to completion, host clock).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "device_ctx.cuh"
#include "records.cuh"
#include "starsh-b200.h"

namespace b200 {

size_t matrix_device_bytes(const STARSH_blrm *M);   // engine.cu

struct Request {
    long long ticket;
    STARSH_blrf *F;
    int maxrank;
    double tol;
    int nrhs;
    const double *A;
    int lda;
    double *B;
    int ldb;
    int keep;
    double estimate;          // admission estimate, bytes
    double entries;           // matrix entries (the request's work)
    std::chrono::steady_clock::time_point t_submit;
    // results
    bool done = false;
    int status = STARSH_SUCCESS;
    STARSH_blrm *M = nullptr;
    double latency_ms = 0.0;
};

}  // namespace b200

using namespace b200;

struct starsh_b200_server {
    double budget;
    int engine;
    int max_group;
    double group_entries;             // work cap of one group (entries)
    std::mutex mu;
    std::condition_variable cv_work;   // worker: new requests or releases
    std::condition_variable cv_done;   // waiters: completions
    std::deque<Request *> pending;
    std::unordered_map<long long, Request *> requests;
    std::unordered_map<const STARSH_blrm *, double> resident_of;
    double resident = 0.0;
    long long next_ticket = 1;
    double inflight = 0.0;            // estimates of groups being run
    bool stop = false;
    bool paused = false;
    starsh_b200_server_stats stats{};
    std::vector<std::thread> workers;
};

namespace b200 {

// Upper bound of a request's resident device memory: factors at maxrank
// (or full size when the tile cannot be compressed below maxrank), dense
// near-field blocks and the problem's points.
static double estimate_bytes(STARSH_blrf *F, int maxrank)
{
    const STARSH_cluster *R = F->row_cluster, *C = F->col_cluster;
    double bytes = 0.0;
    for (STARSH_int b = 0; b < F->nblocks_far; ++b) {
        const double m = (double)R->size[F->block_far[2 * b]];
        const double n = (double)C->size[F->block_far[2 * b + 1]];
        bytes += 8.0 * std::min((m + n) * std::min<double>(maxrank, std::min(m, n)),
                                m * n);
    }
    for (STARSH_int b = 0; b < F->nblocks_near; ++b)
        bytes += 8.0 * (double)R->size[F->block_near[2 * b]] *
                 (double)C->size[F->block_near[2 * b + 1]];
    bytes += 8.0 * 4.0 * (double)(R->ndata + C->ndata);
    return bytes;
}

static void complete(starsh_b200_server *sv, Request *r, int status,
                     STARSH_blrm *M)
{
    r->status = status;
    r->M = M;
    r->latency_ms = std::chrono::duration<double, std::milli>(
                        std::chrono::steady_clock::now() - r->t_submit).count();
    r->done = true;
    if (status == STARSH_SUCCESS) sv->stats.completed += 1;
    else sv->stats.failed += 1;
}

static void worker_loop(starsh_b200_server *sv)
{
    // this worker's engine context (the shared one if it cannot be made)
    Context *own = context_new_private();
    set_thread_context(own);
    // the worker's batch workspace, once, before it serves (growing it
    // while serving would map new memory in the middle of requests)
    if (own != nullptr && own->workspace_cap != (size_t)-1) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const size_t want = std::min(own->workspace_cap, free_b / 4);
        if (own->workspace.reserve(want, own->stream))
            cudaStreamSynchronize(own->stream);
    }
    for (;;) {
        std::vector<Request *> group;
        double group_estimate = 0.0;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            for (;;) {
                if (sv->stop && sv->pending.empty()) {
                    lk.unlock();
                    set_thread_context(nullptr);
                    context_free_private(own);
                    return;
                }
                // refuse requests larger than the whole budget
                while (!sv->pending.empty() &&
                       sv->pending.front()->estimate > sv->budget) {
                    Request *r = sv->pending.front();
                    sv->pending.pop_front();
                    complete(sv, r, STARSH_MALLOC_ERROR, nullptr);
                    sv->cv_done.notify_all();
                }
                // FIFO admission by memory, and by work: a group takes the
                // head request and then requests while the group's entries
                // stay within the cap, so one group's latency stays short
                // while other workers take the next ones
                double room = sv->budget - sv->resident - sv->inflight;
                double work = 0.0;
                while (!sv->paused && !sv->pending.empty() &&
                       (int)group.size() < sv->max_group &&
                       sv->pending.front()->estimate <= room &&
                       (group.empty() ||
                        work + sv->pending.front()->entries <= sv->group_entries)) {
                    room -= sv->pending.front()->estimate;
                    work += sv->pending.front()->entries;
                    group_estimate += sv->pending.front()->estimate;
                    group.push_back(sv->pending.front());
                    sv->pending.pop_front();
                }
                if (!group.empty()) {
                    sv->inflight += group_estimate;
                    const auto now = std::chrono::steady_clock::now();
                    for (const Request *r : group)
                        sv->stats.queue_ms += std::chrono::duration<double, std::milli>(
                                                  now - r->t_submit).count();
                    break;
                }
                // nothing admissible: wait for a request or a release
                sv->cv_work.wait(lk);
            }
            sv->stats.groups += 1;
        }
        auto t0 = std::chrono::steady_clock::now();
        const int np = (int)group.size();
        std::vector<STARSH_blrm *> mats(np, nullptr);
        std::vector<STARSH_blrf *> fmts(np);
        std::vector<int> mr(np);
        std::vector<double> tl(np);
        for (int i = 0; i < np; ++i) {
            fmts[i] = group[i]->F;
            mr[i] = group[i]->maxrank;
            tl[i] = group[i]->tol;
        }
        int info = starsh_b200_approximate_batch(np, mats.data(), fmts.data(),
                                                 mr.data(), tl.data(), nullptr,
                                                 sv->engine, 0);
        starsh_b200_stats st{};
        starsh_b200_get_stats(&st);
        auto t1 = std::chrono::steady_clock::now();
        std::vector<int> status(np, info);
        for (int i = 0; i < np && info == STARSH_SUCCESS; ++i) {
            Request *r = group[i];
            if (r->nrhs > 0)
                status[i] = starsh_blrm__dmml_b200(mats[i], r->nrhs, 1.0,
                                                   (double *)r->A, r->lda, 0.0,
                                                   r->B, r->ldb);
        }
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            sv->inflight -= group_estimate;
            if (info == STARSH_SUCCESS) sv->stats.entries += st.entries;
            for (int i = 0; i < np; ++i) {
                Request *r = group[i];
                STARSH_blrm *M = mats[i];
                if (M != nullptr && (status[i] != STARSH_SUCCESS || !r->keep)) {
                    starsh_blrm_free(M);
                    M = nullptr;
                }
                if (M != nullptr) {
                    const double b = (double)matrix_device_bytes(M);
                    sv->resident_of[M] = b;
                    sv->resident += b;
                    if (sv->resident > sv->stats.peak_resident_bytes)
                        sv->stats.peak_resident_bytes = sv->resident;
                }
                complete(sv, r, status[i], M);
            }
            sv->stats.resident_bytes = sv->resident;
            const auto t2 = std::chrono::steady_clock::now();
            sv->stats.busy_ms += std::chrono::duration<double, std::milli>(t2 - t0).count();
            sv->stats.approx_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
            sv->stats.products_ms += std::chrono::duration<double, std::milli>(t2 - t1).count();
        }
        sv->cv_done.notify_all();
        // memory came back: another worker may admit now
        sv->cv_work.notify_all();
    }
}

}  // namespace b200

extern "C" int starsh_b200_server_new(starsh_b200_server **server,
                                      double hbm_budget_bytes, int engine,
                                      int max_group)
{
    if (server == nullptr || !(hbm_budget_bytes > 0.0) ||
        (engine != STARSH_B200_FP64 && engine != STARSH_B200_MIXED))
        return STARSH_WRONG_PARAMETER;
    auto *sv = new starsh_b200_server();
    sv->budget = hbm_budget_bytes;
    sv->engine = engine;
    sv->max_group = max_group > 0 ? max_group : 1 << 30;
    sv->group_entries = 5e8;
    if (const char *e = getenv("STARSH_B200_SERVER_GROUP_ENTRIES"))
        sv->group_entries = std::max(1.0, atof(e));
    int nw = 3;
    if (const char *e = getenv("STARSH_B200_SERVER_WORKERS"))
        nw = std::max(1, std::min(8, atoi(e)));
    for (int w = 0; w < nw; ++w) sv->workers.emplace_back(worker_loop, sv);
    *server = sv;
    return STARSH_SUCCESS;
}

extern "C" int starsh_b200_server_submit(starsh_b200_server *server,
                                         STARSH_blrf *format, int maxrank,
                                         double tol, int nrhs, const double *A,
                                         int lda, double *B, int ldb, int keep,
                                         long long *ticket)
{
    if (server == nullptr || format == nullptr || ticket == nullptr ||
        maxrank < 0 || !(tol >= 0.0) || nrhs < 0 ||
        (nrhs > 0 && (A == nullptr || B == nullptr)))
        return STARSH_WRONG_PARAMETER;
    auto *r = new Request();
    r->F = format;
    r->maxrank = maxrank;
    r->tol = tol;
    r->nrhs = nrhs;
    r->A = A;
    r->lda = lda;
    r->B = B;
    r->ldb = ldb;
    r->keep = keep;
    r->estimate = estimate_bytes(format, maxrank);
    r->entries = (double)format->row_cluster->ndata * (double)format->col_cluster->ndata;
    r->t_submit = std::chrono::steady_clock::now();
    {
        std::lock_guard<std::mutex> lk(server->mu);
        if (server->stop) {
            delete r;
            return STARSH_WRONG_PARAMETER;
        }
        r->ticket = server->next_ticket++;
        server->requests[r->ticket] = r;
        server->pending.push_back(r);
        server->stats.submitted += 1;
        *ticket = r->ticket;
    }
    server->cv_work.notify_one();
    return STARSH_SUCCESS;
}

extern "C" int starsh_b200_server_wait(starsh_b200_server *server,
                                       long long ticket, STARSH_blrm **matrix,
                                       double *latency_ms)
{
    if (server == nullptr) return STARSH_WRONG_PARAMETER;
    std::unique_lock<std::mutex> lk(server->mu);
    auto it = server->requests.find(ticket);
    if (it == server->requests.end()) return STARSH_WRONG_PARAMETER;
    Request *r = it->second;
    server->cv_done.wait(lk, [&] { return r->done; });
    server->requests.erase(it);
    const int status = r->status;
    if (matrix) *matrix = r->M;
    if (latency_ms) *latency_ms = r->latency_ms;
    delete r;
    return status;
}

extern "C" int starsh_b200_server_release(starsh_b200_server *server,
                                          STARSH_blrm *matrix)
{
    if (server == nullptr || matrix == nullptr) return STARSH_WRONG_PARAMETER;
    {
        std::lock_guard<std::mutex> lk(server->mu);
        auto it = server->resident_of.find(matrix);
        if (it == server->resident_of.end()) return STARSH_WRONG_PARAMETER;
        server->resident -= it->second;
        server->stats.resident_bytes = server->resident;
        server->resident_of.erase(it);
    }
    starsh_blrm_free(matrix);
    server->cv_work.notify_one();
    return STARSH_SUCCESS;
}

extern "C" int starsh_b200_server_pause(starsh_b200_server *server,
                                         int paused)
{
    if (server == nullptr) return STARSH_WRONG_PARAMETER;
    {
        std::lock_guard<std::mutex> lk(server->mu);
        server->paused = paused != 0;
    }
    server->cv_work.notify_one();
    return STARSH_SUCCESS;
}

extern "C" int starsh_b200_server_get_stats(starsh_b200_server *server,
                                            starsh_b200_server_stats *stats)
{
    if (server == nullptr || stats == nullptr) return STARSH_WRONG_PARAMETER;
    std::lock_guard<std::mutex> lk(server->mu);
    *stats = server->stats;
    return STARSH_SUCCESS;
}

extern "C" int starsh_b200_server_free(starsh_b200_server *server)
{
    if (server == nullptr) return STARSH_WRONG_PARAMETER;
    {
        std::lock_guard<std::mutex> lk(server->mu);
        server->stop = true;
        server->paused = false;
    }
    server->cv_work.notify_all();
    for (std::thread &w : server->workers) w.join();
    // requests nobody waited for
    for (auto &kv : server->requests) {
        if (kv.second->M) starsh_blrm_free(kv.second->M);
        delete kv.second;
    }
    delete server;
    return STARSH_SUCCESS;
}
