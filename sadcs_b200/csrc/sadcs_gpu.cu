// sadcs_gpu.cu - host driver and C ABI of libsadcs_gpu.so (declared in include/sadcs_gpu.h).
//
// One construction: upload (or device copy) of the text into a zero-padded buffer, sample ranking,
// class lists, merge into the SA and/or BWT, download. Every buffer comes from one device slab that
// a context reserves once (cudaMalloc of the planned peak); a construction carves it by a layout
// computed from n alone, so the plan and the allocation cannot disagree and nothing is allocated
// per call. Ranking scratch and the class/merge buffers overlap: the former is dead before the
// latter are written. Work runs on the context's own non-blocking stream, or the caller's stream for
// the device-resident entry point. Mirrors the reference's host driver, src/cuda/gpusa.cu.
#include "../../include/sadcs_gpu.h"

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>

#include "bwt.cuh"
#include "classes.cuh"
#include "common.cuh"
#include "merge.cuh"
#include "primitives.cuh"
#include "rank.cuh"

namespace {

using namespace sadcs;

thread_local char tLastError[512] = "";

void setError(const char* format, ...) {
    va_list args;
    va_start(args, format);
    vsnprintf(tLastError, sizeof tLastError, format, args);
    va_end(args);
}

int failed(const char* what, cudaError_t error) {
    setError("%s: %s", what, cudaGetErrorString(error));
    cudaGetLastError();  // clear a sticky launch error where possible
    return error == cudaErrorMemoryAllocation ? SADCS_NOT_ENOUGH_MEMORY : SADCS_FAILED;
}

double secondsSince(std::chrono::steady_clock::time_point start) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
}

constexpr int64_t kMemoryReserve = int64_t(256) << 20;          // gpusa.h:82
constexpr int64_t kMaxInt32Text = int64_t(INT32_MAX) - 1024;    // src/cpu/dcsort.h:21
constexpr int64_t kMaxText = (int64_t(1) << 32) - 256;

size_t align256(size_t bytes) {
    return (bytes + 255) & ~size_t(255);
}

// Byte offsets of every buffer of a construction of n bytes, and the peaks.
struct Layout {
    uint64_t n = 0, m = 0;
    size_t text = 0, ranks = 0;
    // ranking region
    size_t lst0 = 0, lst1 = 0, key0 = 0, key1 = 0, grp = 0, aux1 = 0, aux2 = 0, rankScratch = 0, counter = 0;
    // class + merge region (overlaps the ranking region)
    size_t lists = 0, classScratch = 0, splitters = 0, rows = 0, sa = 0, bwt = 0, mergeCounter = 0;
    size_t rankingEnd = 0, classEnd = 0, mergeEnd = 0, peak = 0;
    MergePlan merge;
};

Layout planLayout(uint64_t n, bool internalSa, bool internalBwt) {
    Layout L;
    L.n = n;
    L.m = sampleSize(n);
    const uint64_t m = L.m;
    size_t at = 0;
    auto take = [&at](size_t bytes) {
        const size_t offset = at;
        at += align256(bytes);
        return offset;
    };
    L.text = take(n + kTextPad);
    L.ranks = take(4 * (m + kRankPad));
    const size_t persistent = at;

    L.lst0 = take(4 * m);
    L.lst1 = take(4 * m);
    L.key0 = take(8 * m);
    L.key1 = take(8 * m);
    L.grp = take(4 * m);
    L.aux1 = take(4 * m);
    L.aux2 = take(4 * m);
    L.rankScratch = take(4 * std::max(radixScratchWords(m), scanScratchWords(m)));
    L.counter = take(256);
    L.rankingEnd = at;

    at = persistent;
    const ClassLayout classes = classLayout(n);
    uint64_t largest = 0;
    for (int d = 0; d < kClasses; d++) largest = std::max<uint64_t>(largest, classes.start[d + 1] - classes.start[d]);
    L.lists = take(4 * n);
    L.classScratch = take(4 * radixScratchWords(largest + 1));
    L.classEnd = at;
    at = L.classScratch;  // the merge reuses the class scratch
    L.merge = planMerge(classes.start);
    L.splitters = take(4 * L.merge.splitterWords);
    L.rows = take(sizeof(MergeRow) * (L.merge.rows + 1));
    L.mergeCounter = take(256);
    L.sa = internalSa ? take(4 * n) : 0;
    L.bwt = internalBwt ? take(n) : 0;
    L.mergeEnd = at;
    L.peak = std::max({L.rankingEnd, L.classEnd, L.mergeEnd});
    return L;
}

}  // namespace

struct sadcs_gpu_context {
    int device = 0;
    uint64_t capacity = 0;
    size_t slabBytes = 0;
    uint8_t* slab = nullptr;
    cudaStream_t stream = nullptr;
    uint32_t* hostWords = nullptr;  // page-locked
    cudaEvent_t events[6] = {};
};

namespace {

void destroyContext(sadcs_gpu_context* c) {
    if (!c) return;
    int previous = 0;
    cudaGetDevice(&previous);
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (cudaEvent_t& e : c->events) {
        if (e) cudaEventDestroy(e);
    }
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->slab) cudaFree(c->slab);
    if (c->hostWords) cudaFreeHost(c->hostWords);
    cudaSetDevice(previous);
    delete c;
}

int queryDevice(sadcs_gpu_device* device) {
    int count = 0;
    cudaError_t error = cudaGetDeviceCount(&count);
    if (error != cudaSuccess || count == 0) {
        if (error != cudaSuccess) {
            setError("cudaGetDeviceCount: %s", cudaGetErrorString(error));
            cudaGetLastError();
        } else {
            setError("no CUDA device");
        }
        return SADCS_UNAVAILABLE;
    }
    int current = 0;
    cudaDeviceProp properties;
    if ((error = cudaGetDevice(&current)) != cudaSuccess ||
        (error = cudaGetDeviceProperties(&properties, current)) != cudaSuccess) {
        setError("cudaGetDeviceProperties: %s", cudaGetErrorString(error));
        return SADCS_UNAVAILABLE;
    }
    size_t freeBytes = 0, totalBytes = 0;
    if ((error = cudaMemGetInfo(&freeBytes, &totalBytes)) != cudaSuccess) {
        setError("cudaMemGetInfo: %s", cudaGetErrorString(error));
        return SADCS_UNAVAILABLE;
    }
    if (device) {
        snprintf(device->name, sizeof device->name, "%s", properties.name);
        device->compute_major = properties.major;
        device->compute_minor = properties.minor;
        device->total_bytes = static_cast<int64_t>(totalBytes);
        device->free_bytes = static_cast<int64_t>(freeBytes);
    }
    return SADCS_OK;
}

int createContext(int64_t capacity, sadcs_gpu_context** out) {
    *out = nullptr;
    sadcs_gpu_device device;
    if (const int status = queryDevice(&device); status != SADCS_OK) return status;
    if (capacity < 0 || capacity > kMaxText) {
        setError("capacity %lld out of range (0 to %lld bytes)", static_cast<long long>(capacity),
                 static_cast<long long>(kMaxText));
        return SADCS_FAILED;
    }
    const Layout L = planLayout(static_cast<uint64_t>(capacity), true, true);
    const int64_t peak = static_cast<int64_t>(L.peak);
    if (peak + kMemoryReserve > device.free_bytes) {
        setError("needs %lld MiB of device memory plus %lld MiB reserve, %lld MiB free",
                 static_cast<long long>(peak >> 20), static_cast<long long>(kMemoryReserve >> 20),
                 static_cast<long long>(device.free_bytes >> 20));
        return SADCS_NOT_ENOUGH_MEMORY;
    }
    sadcs_gpu_context* c = new (std::nothrow) sadcs_gpu_context;
    if (!c) {
        setError("out of host memory");
        return SADCS_FAILED;
    }
    cudaGetDevice(&c->device);
    c->capacity = static_cast<uint64_t>(capacity);
    c->slabBytes = L.peak;
    cudaError_t error;
    if ((error = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (error = cudaMallocHost(&c->hostWords, 256)) != cudaSuccess ||
        (error = cudaMalloc(&c->slab, std::max<size_t>(c->slabBytes, 256))) != cudaSuccess) {
        const int status = failed("creating the context", error);
        destroyContext(c);
        return status;
    }
    for (cudaEvent_t& e : c->events) {
        if ((error = cudaEventCreate(&e)) != cudaSuccess) {
            const int status = failed("cudaEventCreate", error);
            destroyContext(c);
            return status;
        }
    }
    *out = c;
    return SADCS_OK;
}

bool isPinned(const void* host) {
    cudaPointerAttributes attributes;
    if (cudaPointerGetAttributes(&attributes, host) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attributes.type == cudaMemoryTypeHost;
}

float elapsedMs(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

// One construction on the context's slab. Either hostText or deviceText is given. Outputs: device
// pointers (outSa/outBwt, caller-owned) or, when null and wanted, the slab's internal buffers,
// returned through internalSa/internalBwt for the caller to download.
int construct(sadcs_gpu_context* c, const uint8_t* hostText, const uint8_t* deviceText, uint64_t n, bool wantSa,
              bool wantBwt, uint32_t* outSa, uint8_t* outBwt, cudaStream_t stream, sadcs_gpu_stats& s,
              uint32_t*& internalSa, uint8_t*& internalBwt, uint32_t& row0) {
    if (n > c->capacity) {
        setError("input of %llu bytes exceeds the context's capacity of %llu bytes", static_cast<unsigned long long>(n),
                 static_cast<unsigned long long>(c->capacity));
        return SADCS_NOT_ENOUGH_MEMORY;
    }
    const Layout L = planLayout(n, wantSa && !outSa, wantBwt && !outBwt);
    if (L.peak > c->slabBytes) {
        setError("internal: layout of %llu bytes exceeds the slab of %llu", static_cast<unsigned long long>(L.peak),
                 static_cast<unsigned long long>(c->slabBytes));
        return SADCS_FAILED;
    }
    uint8_t* slab = c->slab;
    uint8_t* text = slab + L.text;
    uint32_t* ranks = reinterpret_cast<uint32_t*>(slab + L.ranks);
    cudaError_t error;
    auto start = std::chrono::steady_clock::now();

    if ((error = cudaMemsetAsync(text + n, 0, kTextPad, stream)) != cudaSuccess) return failed("upload", error);
    if (hostText) {
        s.pinned = isPinned(hostText) ? 1 : 0;
        if ((error = cudaMemcpyAsync(text, hostText, n, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
            (error = cudaStreamSynchronize(stream)) != cudaSuccess) {
            return failed("upload", error);
        }
        s.upload_seconds = secondsSince(start);
    } else if ((error = cudaMemcpyAsync(text, deviceText, n, cudaMemcpyDeviceToDevice, stream)) != cudaSuccess) {
        return failed("copying the text", error);
    }
    start = std::chrono::steady_clock::now();
    cudaEventRecord(c->events[0], stream);

    // Sample ranking.
    if ((error = cudaMemsetAsync(ranks, 0, 4 * (L.m + kRankPad), stream)) != cudaSuccess) return failed("ranking", error);
    RankBuffers rb;
    rb.lst[0] = reinterpret_cast<uint32_t*>(slab + L.lst0);
    rb.lst[1] = reinterpret_cast<uint32_t*>(slab + L.lst1);
    rb.key[0] = reinterpret_cast<uint64_t*>(slab + L.key0);
    rb.key[1] = reinterpret_cast<uint64_t*>(slab + L.key1);
    rb.grp = reinterpret_cast<uint32_t*>(slab + L.grp);
    rb.aux1 = reinterpret_cast<uint32_t*>(slab + L.aux1);
    rb.aux2 = reinterpret_cast<uint32_t*>(slab + L.aux2);
    rb.scratch = reinterpret_cast<uint32_t*>(slab + L.rankScratch);
    rb.counter = reinterpret_cast<uint32_t*>(slab + L.counter);
    RankStats rankStats;
    if ((error = rankSample(text, static_cast<uint32_t>(n), ranks, rb, c->hostWords, stream, rankStats)) != cudaSuccess) {
        return failed("sample ranking", error);
    }
    s.character_passes = rankStats.characterPasses;
    s.doubling_rounds = rankStats.doublingRounds;
    cudaEventRecord(c->events[1], stream);
    if ((error = cudaStreamSynchronize(stream)) != cudaSuccess) return failed("sample ranking", error);
    s.ranking_seconds = secondsSince(start);
    s.ranking_bytes = static_cast<int64_t>(L.rankingEnd);
    start = std::chrono::steady_clock::now();

    // Class lists.
    uint32_t* lists = reinterpret_cast<uint32_t*>(slab + L.lists);
    if ((error = sortClasses(text, static_cast<uint32_t>(n), ranks, lists,
                             reinterpret_cast<uint32_t*>(slab + L.classScratch), stream)) != cudaSuccess) {
        return failed("class sorts", error);
    }
    cudaEventRecord(c->events[2], stream);
    if ((error = cudaStreamSynchronize(stream)) != cudaSuccess) return failed("class sorts", error);
    s.class_sort_seconds = secondsSince(start);
    s.class_sort_bytes = static_cast<int64_t>(L.classEnd);
    start = std::chrono::steady_clock::now();

    // Merge.
    uint32_t* sa = outSa ? outSa : (wantSa ? reinterpret_cast<uint32_t*>(slab + L.sa) : nullptr);
    uint8_t* bwt = outBwt ? outBwt : (wantBwt ? slab + L.bwt : nullptr);
    if ((error = mergeClasses(text, ranks, static_cast<uint32_t>(n), lists, L.merge,
                              reinterpret_cast<uint32_t*>(slab + L.splitters),
                              reinterpret_cast<MergeRow*>(slab + L.rows), sa, bwt,
                              reinterpret_cast<uint32_t*>(slab + L.mergeCounter), c->hostWords, stream, &row0)) !=
        cudaSuccess) {
        return failed("merge", error);
    }
    cudaEventRecord(c->events[3], stream);
    if ((error = cudaStreamSynchronize(stream)) != cudaSuccess) return failed("merge", error);
    s.merge_seconds = secondsSince(start);
    s.merge_bytes = static_cast<int64_t>(L.mergeEnd);
    s.device_bytes = static_cast<int64_t>(L.peak);
    s.device_seconds = elapsedMs(c->events[0], c->events[3]) / 1000.0;
    internalSa = outSa ? nullptr : sa;
    internalBwt = outBwt ? nullptr : bwt;
    return SADCS_OK;
}

// Runs body(context) with the given context, or a temporary one for n bytes (its creation is setup).
template <class Body>
int withContext(sadcs_gpu_context* context, uint64_t n, sadcs_gpu_stats& s, Body body) {
    if (context) {
        int previous = 0;
        cudaGetDevice(&previous);
        if (previous != context->device) cudaSetDevice(context->device);
        const int status = body(context);
        if (previous != context->device) cudaSetDevice(previous);
        return status;
    }
    const auto start = std::chrono::steady_clock::now();
    sadcs_gpu_context* temporary = nullptr;
    if (const int status = createContext(static_cast<int64_t>(n), &temporary); status != SADCS_OK) return status;
    s.setup_seconds = secondsSince(start);
    const int status = body(temporary);
    const double setup = s.setup_seconds;
    destroyContext(temporary);
    s.setup_seconds = setup;
    return status;
}

int download(sadcs_gpu_context* c, void* host, const void* device, size_t bytes, sadcs_gpu_stats& s) {
    const auto start = std::chrono::steady_clock::now();
    cudaError_t error;
    if ((error = cudaMemcpyAsync(host, device, bytes, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess ||
        (error = cudaStreamSynchronize(c->stream)) != cudaSuccess) {
        return failed("download", error);
    }
    s.download_seconds += secondsSince(start);
    return SADCS_OK;
}

}  // namespace

extern "C" {

int64_t sadcs_gpu_memory_reserve(void) {
    return kMemoryReserve;
}

int64_t sadcs_gpu_sample_size(int64_t n) {
    return n <= 0 ? 0 : static_cast<int64_t>(sampleSize(static_cast<uint64_t>(n)));
}

int sadcs_gpu_query_device(sadcs_gpu_device* device) {
    tLastError[0] = '\0';
    return queryDevice(device);
}

int64_t sadcs_gpu_required_bytes(int64_t n) {
    if (n < 0 || n > kMaxText) return -1;
    return n == 0 ? 0 : static_cast<int64_t>(planLayout(static_cast<uint64_t>(n), true, true).peak);
}

int sadcs_gpu_create_context(int64_t capacity, sadcs_gpu_context** context) {
    tLastError[0] = '\0';
    if (!context) {
        setError("context pointer is null");
        return SADCS_FAILED;
    }
    return createContext(std::max<int64_t>(capacity, 0), context);
}

void sadcs_gpu_destroy_context(sadcs_gpu_context* context) {
    destroyContext(context);
}

int64_t sadcs_gpu_context_capacity(const sadcs_gpu_context* context) {
    return context ? static_cast<int64_t>(context->capacity) : 0;
}

int sadcs_gpu_build(sadcs_gpu_context* context, const uint8_t* text, int64_t n, uint32_t* sa, uint8_t* bwt,
                    int64_t* primary, sadcs_gpu_stats* stats) {
    tLastError[0] = '\0';
    sadcs_gpu_stats local{};
    sadcs_gpu_stats& s = stats ? *stats : local;
    s = sadcs_gpu_stats{};
    if (primary) *primary = n > 0 ? -1 : 0;
    if (!sa && !bwt) {
        setError("neither a suffix array nor a BWT was asked for");
        return SADCS_FAILED;
    }
    if (n > kMaxText) {
        setError("text of %lld bytes exceeds the limit of %lld", static_cast<long long>(n), static_cast<long long>(kMaxText));
        return SADCS_FAILED;
    }
    if (n <= 0) return context ? SADCS_OK : queryDevice(nullptr);
    if (!text) {
        setError("text is null");
        return SADCS_FAILED;
    }
    return withContext(context, static_cast<uint64_t>(n), s, [&](sadcs_gpu_context* c) -> int {
        uint32_t* deviceSa = nullptr;
        uint8_t* deviceBwt = nullptr;
        uint32_t row0 = 0;
        int status = construct(c, text, nullptr, static_cast<uint64_t>(n), sa != nullptr, bwt != nullptr, nullptr,
                               nullptr, c->stream, s, deviceSa, deviceBwt, row0);
        if (status != SADCS_OK) return status;
        if (sa && (status = download(c, sa, deviceSa, 4 * static_cast<size_t>(n), s)) != SADCS_OK) return status;
        if (bwt && (status = download(c, bwt, deviceBwt, static_cast<size_t>(n), s)) != SADCS_OK) return status;
        if (primary) *primary = bwt ? static_cast<int64_t>(row0) + 1 : -1;
        return SADCS_OK;
    });
}

int sadcs_gpu_suffix_array(sadcs_gpu_context* context, const uint8_t* text, int64_t n, int32_t* sa,
                           sadcs_gpu_stats* stats) {
    if (n > kMaxInt32Text) {
        tLastError[0] = '\0';
        setError("text of %lld bytes is too large for an int32 suffix array (at most %lld); use sadcs_gpu_build",
                 static_cast<long long>(n), static_cast<long long>(kMaxInt32Text));
        if (stats) *stats = sadcs_gpu_stats{};
        return SADCS_FAILED;
    }
    if (n <= 0) {
        tLastError[0] = '\0';
        if (stats) *stats = sadcs_gpu_stats{};
        return context ? SADCS_OK : queryDevice(nullptr);
    }
    if (!sa) {
        tLastError[0] = '\0';
        setError("sa is null");
        return SADCS_FAILED;
    }
    return sadcs_gpu_build(context, text, n, reinterpret_cast<uint32_t*>(sa), nullptr, nullptr, stats);
}

int sadcs_gpu_bwt(sadcs_gpu_context* context, const uint8_t* text, int64_t n, uint8_t* bwt, int32_t* primary,
                  sadcs_gpu_stats* stats) {
    tLastError[0] = '\0';
    if (stats) *stats = sadcs_gpu_stats{};
    if (primary) *primary = n > 0 ? -1 : 0;
    if (n > kMaxInt32Text) {
        setError("text of %lld bytes is too large for an int32 primary index (at most %lld); use sadcs_gpu_build",
                 static_cast<long long>(n), static_cast<long long>(kMaxInt32Text));
        return SADCS_FAILED;
    }
    if (n <= 1) {
        // gpusa.cu:616-626: the sentinel's row is T[0]; suffix 0's row is left out.
        const int status = context ? SADCS_OK : queryDevice(nullptr);
        if (status == SADCS_OK && n == 1) {
            bwt[0] = text[0];
            if (primary) *primary = 1;
        }
        return status;
    }
    int64_t p = -1;
    const int status = sadcs_gpu_build(context, text, n, nullptr, bwt, &p, stats);
    if (status == SADCS_OK && primary) *primary = static_cast<int32_t>(p);
    return status;
}

int sadcs_gpu_build_device(sadcs_gpu_context* context, const uint8_t* d_text, int64_t n, uint32_t* d_sa,
                           uint8_t* d_bwt, int64_t* primary, void* stream, sadcs_gpu_stats* stats) {
    tLastError[0] = '\0';
    sadcs_gpu_stats local{};
    sadcs_gpu_stats& s = stats ? *stats : local;
    s = sadcs_gpu_stats{};
    if (primary) *primary = n > 0 ? -1 : 0;
    if (!d_sa && !d_bwt) {
        setError("neither a suffix array nor a BWT was asked for");
        return SADCS_FAILED;
    }
    if (n > kMaxText) {
        setError("text of %lld bytes exceeds the limit of %lld", static_cast<long long>(n), static_cast<long long>(kMaxText));
        return SADCS_FAILED;
    }
    if (n <= 0) return context ? SADCS_OK : queryDevice(nullptr);
    return withContext(context, static_cast<uint64_t>(n), s, [&](sadcs_gpu_context* c) -> int {
        uint32_t* unusedSa = nullptr;
        uint8_t* unusedBwt = nullptr;
        uint32_t row0 = 0;
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
        const int status = construct(c, nullptr, d_text, static_cast<uint64_t>(n), d_sa != nullptr, d_bwt != nullptr,
                                     d_sa, d_bwt, st, s, unusedSa, unusedBwt, row0);
        if (status == SADCS_OK && primary) *primary = d_bwt ? static_cast<int64_t>(row0) + 1 : -1;
        return status;
    });
}

int sadcs_gpu_bwt_from_sa(const uint8_t* d_text, int64_t n, const uint32_t* d_sa, uint8_t* d_bwt, int64_t* primary,
                          void* stream) {
    tLastError[0] = '\0';
    if (primary) *primary = n > 0 ? -1 : 0;
    if (n <= 0) return SADCS_OK;
    if (n > kMaxText) {
        setError("text of %lld bytes exceeds the limit of %lld", static_cast<long long>(n), static_cast<long long>(kMaxText));
        return SADCS_FAILED;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint32_t* word = nullptr;
    uint32_t* host = nullptr;
    cudaError_t error;
    if ((error = cudaMallocAsync(&word, sizeof(uint32_t), st)) != cudaSuccess) return failed("cudaMallocAsync", error);
    if ((error = cudaMallocHost(&host, sizeof(uint32_t))) != cudaSuccess) {
        cudaFreeAsync(word, st);
        return failed("cudaMallocHost", error);
    }
    uint32_t row0 = 0;
    error = bwtFromSa(d_text, static_cast<uint32_t>(n), d_sa, d_bwt, word, host, st, &row0);
    cudaFreeAsync(word, st);
    cudaStreamSynchronize(st);
    cudaFreeHost(host);
    if (error != cudaSuccess) return failed("SA-to-BWT gather", error);
    if (primary) *primary = static_cast<int64_t>(row0) + 1;
    return SADCS_OK;
}

int sadcs_gpu_rank_sample(const uint8_t* text, int64_t n, uint32_t* ranks, sadcs_gpu_stats* stats) {
    tLastError[0] = '\0';
    sadcs_gpu_stats local{};
    sadcs_gpu_stats& s = stats ? *stats : local;
    s = sadcs_gpu_stats{};
    if (n <= 0) return queryDevice(nullptr);
    if (n > kMaxText) {
        setError("text of %lld bytes exceeds the limit of %lld", static_cast<long long>(n), static_cast<long long>(kMaxText));
        return SADCS_FAILED;
    }
    return withContext(nullptr, static_cast<uint64_t>(n), s, [&](sadcs_gpu_context* c) -> int {
        const Layout L = planLayout(static_cast<uint64_t>(n), false, false);
        uint8_t* textBuffer = c->slab + L.text;
        uint32_t* rankBuffer = reinterpret_cast<uint32_t*>(c->slab + L.ranks);
        cudaError_t error;
        auto start = std::chrono::steady_clock::now();
        if ((error = cudaMemsetAsync(textBuffer + n, 0, kTextPad, c->stream)) != cudaSuccess ||
            (error = cudaMemcpyAsync(textBuffer, text, static_cast<size_t>(n), cudaMemcpyHostToDevice, c->stream)) !=
                cudaSuccess ||
            (error = cudaMemsetAsync(rankBuffer, 0, 4 * (L.m + kRankPad), c->stream)) != cudaSuccess ||
            (error = cudaStreamSynchronize(c->stream)) != cudaSuccess) {
            return failed("upload", error);
        }
        s.upload_seconds = secondsSince(start);
        start = std::chrono::steady_clock::now();
        RankBuffers rb;
        rb.lst[0] = reinterpret_cast<uint32_t*>(c->slab + L.lst0);
        rb.lst[1] = reinterpret_cast<uint32_t*>(c->slab + L.lst1);
        rb.key[0] = reinterpret_cast<uint64_t*>(c->slab + L.key0);
        rb.key[1] = reinterpret_cast<uint64_t*>(c->slab + L.key1);
        rb.grp = reinterpret_cast<uint32_t*>(c->slab + L.grp);
        rb.aux1 = reinterpret_cast<uint32_t*>(c->slab + L.aux1);
        rb.aux2 = reinterpret_cast<uint32_t*>(c->slab + L.aux2);
        rb.scratch = reinterpret_cast<uint32_t*>(c->slab + L.rankScratch);
        rb.counter = reinterpret_cast<uint32_t*>(c->slab + L.counter);
        RankStats rankStats;
        if ((error = rankSample(textBuffer, static_cast<uint32_t>(n), rankBuffer, rb, c->hostWords, c->stream,
                                rankStats)) != cudaSuccess) {
            return failed("sample ranking", error);
        }
        s.character_passes = rankStats.characterPasses;
        s.doubling_rounds = rankStats.doublingRounds;
        s.ranking_seconds = secondsSince(start);
        s.device_seconds = s.ranking_seconds;
        s.ranking_bytes = static_cast<int64_t>(L.rankingEnd);
        s.device_bytes = s.ranking_bytes;
        return download(c, ranks, rankBuffer, 4 * L.m, s);
    });
}

void* sadcs_gpu_allocate_pinned(size_t bytes) {
    void* pointer = nullptr;
    if (cudaMallocHost(&pointer, std::max<size_t>(bytes, 1)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return pointer;
}

void sadcs_gpu_free_pinned(void* pointer) {
    if (pointer) cudaFreeHost(pointer);
}

const char* sadcs_gpu_last_error(void) {
    return tLastError;
}

}  // extern "C"
