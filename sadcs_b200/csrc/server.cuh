// server.cuh - a serving loop for suffix array / BWT requests on one GPU (no counterpart in the
// reference, which builds one text per call). Included by sadcs_gpu.cu after its driver.
//
// Requests arrive at any time (sadcs_gpu_server_submit) and complete asynchronously. Continuous
// batching: a worker that becomes free takes, in arrival order, either one large request or as
// many queued small requests as fit one batch, and builds them in ONE batched construction, so
// requests that arrived while others were on the GPU join the next launch. Admission is by device
// footprint: a worker starts only when its construction's planned peak fits the budget next to
// the constructions already admitted. Each worker has its own stream and takes its slab from a
// stream-ordered memory pool, so constructions of different workers overlap on the device (the
// radix look-back backs off while it waits, so that waiting tiles do not slow the constructions
// beside them: 3 workers give 1.2x the throughput of 1 on the served mix). With two workers or
// more, worker 0 is a small-request lane (server_policy.h): large requests never hold every worker,
// and its stream has the highest priority, so its kernels do not wait behind a large construction's.
// A request's outputs are exactly those of a construction of its text alone.
#pragma once

#include <atomic>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "server_policy.h"

namespace {

struct ServerRequest {
    uint64_t id = 0;
    const uint8_t* text = nullptr;
    uint64_t n = 0;
    uint32_t* sa = nullptr;
    uint8_t* bwt = nullptr;
    int64_t primary = 0;
    int status = SADCS_OK;
    std::string error;
    double submitted = 0, started = 0, finished = 0;
    uint32_t batchSize = 0;
    bool done = false;
};

// SADCS_SERVER_TRACE=1 in the environment: one line per construction on stderr.
bool serverTraceEnabled() {
    static const bool enabled = [] {
        const char* v = std::getenv("SADCS_SERVER_TRACE");
        return v && v[0] && v[0] != '0';
    }();
    return enabled;
}

double nowSeconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct sadcs_gpu_server {
    int device = 0;
    uint64_t budget = 0;
    uint64_t inUse = 0;
    uint64_t smallLimit = 0;   // requests up to this many bytes may share a batch
    uint64_t batchBytes = 0;   // bytes of text per batch
    uint32_t batchTexts = 0;   // texts per batch
    int workers = 0;           // worker threads (set before they start)
    uint64_t nextId = 1;
    bool stopping = false;
    cudaMemPool_t pool = nullptr;
    std::mutex mu;
    std::condition_variable work, finished;
    std::deque<ServerRequest*> queue;
    std::unordered_map<uint64_t, ServerRequest*> requests;
    std::vector<std::thread> threads;
    uint64_t launches = 0, constructions = 0;
    std::atomic<int64_t> failAllocations{0};  // constructions left whose slab allocation is made to fail
};

namespace {

// True (and one fewer left) while sadcs_gpu_server_fail_allocations has failures pending.
bool takeInjectedFailure(sadcs_gpu_server* srv) {
    int64_t pending = srv->failAllocations.load();
    while (pending > 0) {
        if (srv->failAllocations.compare_exchange_weak(pending, pending - 1)) return true;
    }
    return false;
}

// Footprint of a construction: its planned peak on the device (a one-text batch from the carry
// threshold on with room for carried words).
size_t footprintOf(const Batch& b) {
    return planLayout(extentOf(b), true, true, planCarry(b.outputs, b.count)).peak;
}

void serveBatch(sadcs_gpu_server* srv, sadcs_gpu_context& ctx, std::vector<ServerRequest*>& group, const Batch& b,
                size_t footprint) {
    sadcs_gpu_stats stats{};
    int status = SADCS_OK;
    std::string message;
    const double started = nowSeconds();
    double constructed = started;
    for (ServerRequest* r : group) r->started = started;
    cudaError_t error = takeInjectedFailure(srv) ? cudaErrorMemoryAllocation
                                                 : cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ctx.slab),
                                                                           footprint, srv->pool, ctx.stream);
    if (error != cudaSuccess) {
        status = failed("allocating from the pool", error);
        message = tLastError;
        ctx.slab = nullptr;
    }
    if (status == SADCS_OK) {
        ctx.slabBytes = footprint;
        ctx.capacity = b.outputs;
        ctx.maxTexts = b.count;
        // room for carried words if the footprint was planned with it
        ctx.carryRoom = b.count <= 1 && planLayout(extentOf(b), true, true, true).peak <= footprint;
        Io io;
        io.wantSa = true;
        io.wantBwt = true;
        std::vector<const uint8_t*> pieces;
        std::vector<uint32_t*> saPieces;
        std::vector<uint8_t*> bwtPieces;
        if (group.size() == 1) {
            io.hostText = group[0]->text;
            // Page-locked outputs are written by the merge itself (see sadcs_gpu_build_batch).
            io.outSa = static_cast<uint32_t*>(mappedHost(group[0]->sa));
            io.outBwt = static_cast<uint8_t*>(mappedHost(group[0]->bwt));
        } else {
            // Each request's text goes straight from the caller's buffer into the device staging
            // region (asynchronous from page-locked memory; the driver stages pageable memory).
            for (ServerRequest* r : group) pieces.push_back(r->text);
            io.hostPieces = pieces.data();
            // When every request's outputs are page-locked, the merge writes each into its own.
            bool mapped = true;
            for (ServerRequest* r : group) {
                uint32_t* s = static_cast<uint32_t*>(mappedHost(r->sa));
                uint8_t* w = static_cast<uint8_t*>(mappedHost(r->bwt));
                mapped = mapped && s && w;
                saPieces.push_back(s);
                bwtPieces.push_back(w);
            }
            if (mapped) {
                io.saPieces = saPieces.data();
                io.bwtPieces = bwtPieces.data();
            }
        }
        status = construct(&ctx, b, io, ctx.stream, stats);
        constructed = nowSeconds();
        if (status == SADCS_OK) {
            uint64_t offset = 0;
            for (ServerRequest* r : group) {
                if ((!io.outSa && !io.saPieces &&
                     (error = cudaMemcpyAsync(r->sa, io.deviceSa + offset, 4 * r->n, cudaMemcpyDeviceToHost,
                                              ctx.stream)) != cudaSuccess) ||
                    (!io.outBwt && !io.bwtPieces &&
                     (error = cudaMemcpyAsync(r->bwt, io.deviceBwt + offset, r->n, cudaMemcpyDeviceToHost,
                                              ctx.stream)) != cudaSuccess)) {
                    status = failed("download", error);
                    break;
                }
                offset += r->n;
            }
            if (status == SADCS_OK) {
                std::vector<int64_t> primaries(b.count);
                status = readPrimaries(&ctx, io, b.count, primaries.data());
                for (size_t k = 0; status == SADCS_OK && k < group.size(); k++) group[k]->primary = primaries[k];
            }
        }
        if (status != SADCS_OK) message = tLastError;
        cudaFreeAsync(ctx.slab, ctx.stream);
        ctx.slab = nullptr;
        cudaStreamSynchronize(ctx.stream);
    }
    const double done = nowSeconds();
    if (serverTraceEnabled()) {
        fprintf(stderr, "sadcs server: %zu texts, %.1f MiB: %.3f s (device %.3f, upload %.3f, after %.3f)\n",
                group.size(), b.outputs / 1048576.0, done - started, stats.device_seconds, stats.upload_seconds,
                done - constructed);
    }
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->inUse -= footprint;
    srv->launches += static_cast<uint64_t>(stats.kernel_launches);
    srv->constructions++;
    for (ServerRequest* r : group) {
        r->status = status;
        r->error = message;
        r->finished = done;
        r->batchSize = static_cast<uint32_t>(group.size());
        r->done = true;
    }
    srv->finished.notify_all();
    srv->work.notify_all();
}

void serverWorker(sadcs_gpu_server* srv, int worker) {
    cudaSetDevice(srv->device);
    const bool smallLane = serverIsSmallLane(worker, srv->workers);
    sadcs_gpu_context ctx;
    ctx.device = srv->device;
    ctx.hostWordCount = 64 + metaWords(srv->batchTexts, 0) + 2 * static_cast<size_t>(srv->batchTexts) + 64 + 256;
    // The small lane's stream has the device's highest priority: its kernels' blocks are dispatched
    // first as SMs free up, instead of queueing behind a large construction's grids.
    int leastPriority = 0, greatestPriority = 0;
    if (!smallLane || cudaDeviceGetStreamPriorityRange(&leastPriority, &greatestPriority) != cudaSuccess) {
        greatestPriority = 0;
    }
    bool ready = cudaStreamCreateWithPriority(&ctx.stream, cudaStreamNonBlocking, greatestPriority) == cudaSuccess &&
                 cudaMallocHost(&ctx.hostWords, 4 * ctx.hostWordCount) == cudaSuccess;
    for (cudaEvent_t& e : ctx.events) ready = ready && cudaEventCreate(&e) == cudaSuccess;
    for (;;) {
        std::vector<ServerRequest*> group;
        Batch b;
        size_t footprint = 0;
        {
            std::unique_lock<std::mutex> lock(srv->mu);
            for (;;) {
                if (srv->stopping && srv->queue.empty()) break;
                // The group's first request: the head, or for the small lane the first small one.
                const size_t first = serverGroupStart(
                    srv->queue.size(), [srv](size_t k) { return srv->queue[k]->n; }, srv->smallLimit, smallLane);
                if (first < srv->queue.size()) {
                    // Take that request alone (large) or it and the queued small requests after it
                    // that fit one batch (server_policy.h).
                    const size_t take = serverGroupSize(
                        srv->queue.size() - first, [srv, first](size_t k) { return srv->queue[first + k]->n; },
                        srv->smallLimit, srv->batchBytes, srv->batchTexts);
                    std::vector<uint64_t> lengths(take);
                    for (size_t k = 0; k < take; k++) lengths[k] = srv->queue[first + k]->n;
                    Batch candidate;
                    planBatch(lengths.data(), static_cast<uint32_t>(lengths.size()), candidate);
                    const size_t need = footprintOf(candidate);
                    if (serverAdmits(need, srv->inUse, srv->budget)) {
                        for (size_t k = 0; k < take; k++) group.push_back(srv->queue[first + k]);
                        srv->queue.erase(srv->queue.begin() + first, srv->queue.begin() + first + take);
                        b = std::move(candidate);
                        footprint = need;
                        srv->inUse += need;
                        break;
                    }
                }
                srv->work.wait(lock);
            }
            if (group.empty()) break;
        }
        if (!ready) {
            std::lock_guard<std::mutex> lock(srv->mu);
            srv->inUse -= footprint;
            for (ServerRequest* r : group) {
                r->status = SADCS_FAILED;
                r->error = "server worker could not be set up";
                r->done = true;
            }
            srv->finished.notify_all();
            continue;
        }
        serveBatch(srv, ctx, group, b, footprint);
    }
    for (cudaEvent_t& e : ctx.events) {
        if (e) cudaEventDestroy(e);
    }
    if (ctx.stream) cudaStreamDestroy(ctx.stream);
    if (ctx.hostWords) cudaFreeHost(ctx.hostWords);
    ctx.hostWords = nullptr;
    ctx.stream = nullptr;
}

}  // namespace

extern "C" {

int sadcs_gpu_server_create(int64_t memory_budget, int32_t workers, int64_t small_limit, int64_t batch_bytes,
                            int32_t batch_texts, sadcs_gpu_server** out) {
    tLastError[0] = '\0';
    if (!out) {
        setError("server pointer is null");
        return SADCS_FAILED;
    }
    *out = nullptr;
    sadcs_gpu_device device;
    if (const int status = queryDevice(&device); status != SADCS_OK) return status;
    if (workers < 1 || workers > 64 || batch_texts < 1 || static_cast<uint32_t>(batch_texts) > kMaxTexts ||
        small_limit < 0 || batch_bytes < small_limit || batch_bytes > kMaxText) {
        setError("server parameters out of range");
        return SADCS_FAILED;
    }
    const int64_t budget = memory_budget > 0 ? memory_budget : device.free_bytes - kMemoryReserve;
    if (budget <= 0 || budget + kMemoryReserve > device.free_bytes) {
        setError("memory budget of %lld MiB does not fit %lld MiB free (reserve %lld MiB)",
                 static_cast<long long>(budget >> 20), static_cast<long long>(device.free_bytes >> 20),
                 static_cast<long long>(kMemoryReserve >> 20));
        return SADCS_NOT_ENOUGH_MEMORY;
    }
    sadcs_gpu_server* srv = new (std::nothrow) sadcs_gpu_server;
    if (!srv) {
        setError("out of host memory");
        return SADCS_FAILED;
    }
    cudaGetDevice(&srv->device);
    srv->budget = static_cast<uint64_t>(budget);
    srv->smallLimit = static_cast<uint64_t>(small_limit);
    srv->batchBytes = static_cast<uint64_t>(batch_bytes);
    srv->batchTexts = static_cast<uint32_t>(batch_texts);
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = srv->device;
    uint64_t keep = srv->budget;  // keep freed memory in the pool up to the budget
    cudaError_t error;
    if ((error = cudaMemPoolCreate(&srv->pool, &props)) != cudaSuccess ||
        (error = cudaMemPoolSetAttribute(srv->pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
        const int status = failed("memory pool", error);
        if (srv->pool) cudaMemPoolDestroy(srv->pool);
        delete srv;
        return status;
    }
    srv->workers = workers;
    for (int32_t w = 0; w < workers; w++) srv->threads.emplace_back(serverWorker, srv, w);
    *out = srv;
    return SADCS_OK;
}

int sadcs_gpu_server_submit(sadcs_gpu_server* srv, const uint8_t* text, int64_t n, uint32_t* sa, uint8_t* bwt,
                            uint64_t* ticket) {
    tLastError[0] = '\0';
    if (!srv || !ticket || n < 0 || n > kMaxText || (n > 0 && (!text || !sa || !bwt))) {
        setError("invalid request");
        return SADCS_FAILED;
    }
    ServerRequest* r = new (std::nothrow) ServerRequest;
    if (!r) {
        setError("out of host memory");
        return SADCS_FAILED;
    }
    r->text = text;
    r->n = static_cast<uint64_t>(n);
    r->sa = sa;
    r->bwt = bwt;
    r->submitted = nowSeconds();
    std::lock_guard<std::mutex> lock(srv->mu);
    r->id = srv->nextId++;
    srv->requests[r->id] = r;
    if (n == 0) {
        r->started = r->finished = r->submitted;
        r->done = true;
    } else {
        srv->queue.push_back(r);
        srv->work.notify_one();
    }
    *ticket = r->id;
    return SADCS_OK;
}

// Waits for a request (timeout_seconds < 0: no limit). Returns its status, or SADCS_FAILED with
// "timed out" (the request stays pending). latency[0..2] = queued, on the device, total seconds.
int sadcs_gpu_server_wait(sadcs_gpu_server* srv, uint64_t ticket, double timeout_seconds, int64_t* primary,
                          double* latency, int32_t* batch_size) {
    tLastError[0] = '\0';
    if (!srv) {
        setError("server is null");
        return SADCS_FAILED;
    }
    std::unique_lock<std::mutex> lock(srv->mu);
    auto it = srv->requests.find(ticket);
    if (it == srv->requests.end()) {
        setError("unknown ticket %llu", static_cast<unsigned long long>(ticket));
        return SADCS_FAILED;
    }
    ServerRequest* r = it->second;
    auto ready = [r] { return r->done; };
    if (timeout_seconds < 0) {
        srv->finished.wait(lock, ready);
    } else if (!srv->finished.wait_for(lock, std::chrono::duration<double>(timeout_seconds), ready)) {
        setError("timed out");
        return SADCS_FAILED;
    }
    const int status = r->status;
    if (status != SADCS_OK) setError("%s", r->error.c_str());
    if (primary) *primary = r->primary;
    if (latency) {
        latency[0] = r->started - r->submitted;
        latency[1] = r->finished - r->started;
        latency[2] = r->finished - r->submitted;
    }
    if (batch_size) *batch_size = static_cast<int32_t>(r->batchSize);
    srv->requests.erase(it);
    delete r;
    return status;
}

// Takes a request that no worker has taken yet out of the queue; its wait then returns
// SADCS_FAILED with "cancelled". A request being built, done or unknown is left as it is.
int sadcs_gpu_server_cancel(sadcs_gpu_server* srv, uint64_t ticket) {
    tLastError[0] = '\0';
    if (!srv) {
        setError("server is null");
        return SADCS_FAILED;
    }
    std::lock_guard<std::mutex> lock(srv->mu);
    auto it = srv->requests.find(ticket);
    if (it == srv->requests.end()) {
        setError("unknown ticket %llu", static_cast<unsigned long long>(ticket));
        return SADCS_FAILED;
    }
    ServerRequest* r = it->second;
    auto queued = std::find(srv->queue.begin(), srv->queue.end(), r);
    if (queued == srv->queue.end()) {
        setError(r->done ? "request already done" : "request already being built");
        return SADCS_FAILED;
    }
    srv->queue.erase(queued);
    r->status = SADCS_FAILED;
    r->error = "cancelled";
    r->started = r->finished = nowSeconds();
    r->done = true;
    srv->finished.notify_all();
    srv->work.notify_all();  // the queue's head, and so what can be admitted, may have changed
    return SADCS_OK;
}

// The next `count` constructions fail their slab allocation as the pool would when out of memory.
void sadcs_gpu_server_fail_allocations(sadcs_gpu_server* srv, int64_t count) {
    if (srv) srv->failAllocations.store(count > 0 ? count : 0);
}

// Constructions run and kernels launched so far.
void sadcs_gpu_server_counters(sadcs_gpu_server* srv, int64_t* constructions, int64_t* launches) {
    if (!srv) return;
    std::lock_guard<std::mutex> lock(srv->mu);
    if (constructions) *constructions = static_cast<int64_t>(srv->constructions);
    if (launches) *launches = static_cast<int64_t>(srv->launches);
}

// Finishes every queued request, then stops the workers and frees the pool. Requests not yet
// waited for are discarded.
void sadcs_gpu_server_destroy(sadcs_gpu_server* srv) {
    if (!srv) return;
    {
        std::lock_guard<std::mutex> lock(srv->mu);
        srv->stopping = true;
        srv->work.notify_all();
    }
    for (std::thread& t : srv->threads) t.join();
    for (auto& entry : srv->requests) delete entry.second;
    if (srv->pool) cudaMemPoolDestroy(srv->pool);
    delete srv;
}

}  // extern "C"
