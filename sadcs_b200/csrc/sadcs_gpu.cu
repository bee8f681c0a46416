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
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "alphabet.cuh"
#include "bwt.cuh"
#include "check.cuh"
#include "classes.cuh"
#include "common.cuh"
#include "lcp.cuh"
#include "merge.cuh"
#include "merge_final.cuh"
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
// Texts from this size on carry words through the class passes (in a one-text context, codes of at
// most 2 bits): below it the packed text stays in the L2 and the final merge's record gathers hit
// there (tuning).
#ifndef SADCS_CARRY_MIN_BYTES
#define SADCS_CARRY_MIN_BYTES (256ull << 20)
#endif
constexpr uint64_t kCarryMinBytes = SADCS_CARRY_MIN_BYTES;

// The carry threshold: kCarryMinBytes, or the environment's SADCS_CARRY_MIN_BYTES (tests and tuning:
// 0 makes every eligible construction carry words), read at each construction.
uint64_t carryMinBytes() {
    const char* v = std::getenv("SADCS_CARRY_MIN_BYTES");
    return v && *v ? std::strtoull(v, nullptr, 0) : kCarryMinBytes;
}
constexpr uint32_t kMaxTexts = 1u << 20;

// NVTX ranges of a construction's phases (upload, ranking, classes, merge) on the calling thread,
// for profiler timelines and `ncu --nvtx --nvtx-include "sadcs merge/"`; without a tool attached
// each call returns at once. The range open when the construction returns, on any path, is closed.
class PhaseRange {
public:
    explicit PhaseRange(const char* name) { nvtxRangePushA(name); }
    void next(const char* name) {
        nvtxRangePop();
        nvtxRangePushA(name);
    }
    ~PhaseRange() { nvtxRangePop(); }
    PhaseRange(const PhaseRange&) = delete;
    PhaseRange& operator=(const PhaseRange&) = delete;
};

size_t align256(size_t bytes) {
    return (bytes + 255) & ~size_t(255);
}

// Host plan of one construction: a batch of texts (one text is a batch of one). Text j is placed
// at start[j], a multiple of 32, and ends at end[j]; empty texts are left out by the caller.
struct Batch {
    uint32_t count = 0;
    std::vector<uint64_t> lengths;
    std::vector<uint32_t> start, end, sampleBase, outBase;  // outBase: count + 1 entries
    uint64_t span = 0;     // bytes of the concatenation, gaps included (a multiple of 32)
    uint64_t slots = 0;    // rank entries: sample positions of the whole span
    uint64_t live = 0;     // sample positions inside texts
    uint64_t outputs = 0;  // total length: SA entries and BWT bytes
    uint64_t longest = 0;
    ClassPlan classes;
    std::vector<uint32_t> classTables;
    MergePlan merge;
};

bool planBatch(const uint64_t* lengths, uint32_t count, Batch& b) {
    b.count = count;
    b.lengths.assign(lengths, lengths + count);
    b.start.resize(count);
    b.end.resize(count);
    b.sampleBase.resize(count);
    b.outBase.resize(count + 1);
    uint64_t at = 0, live = 0, outputs = 0;
    for (uint32_t j = 0; j < count; j++) {
        b.start[j] = static_cast<uint32_t>(at);
        b.end[j] = static_cast<uint32_t>(at + lengths[j]);
        b.sampleBase[j] = static_cast<uint32_t>(live);
        b.outBase[j] = static_cast<uint32_t>(outputs);
        live += sampleSize(lengths[j]);
        outputs += lengths[j];
        b.longest = std::max<uint64_t>(b.longest, lengths[j]);
        at += (lengths[j] + kV - 1) / kV * kV;
        if (at > static_cast<uint64_t>(kMaxText)) return false;
    }
    b.outBase[count] = static_cast<uint32_t>(outputs);
    b.span = at;
    b.slots = (at / kV) * kK;
    b.live = live;
    b.outputs = outputs;
    b.classTables.assign(ClassTables::words(count), 0);
    planClasses(lengths, count, b.classTables.data(), b.classes);
    b.merge = planMerge(b.classes.start, kMergeRMin);  // the most rows any tile shape needs (memory plan)
    return true;
}

// Words of the per-construction tables: start, end, sampleBase, outBase, rowZero, the class
// tables and (several texts) the text of every 32-byte block.
size_t metaWords(uint32_t count, uint64_t span) {
    return 5 * static_cast<size_t>(count) + 1 + ClassTables::words(count) + (count > 1 ? span / kV + 1 : 0) + 16 +
           4 * static_cast<size_t>(count) + 2;  // + the per-text output pointer tables (8-byte aligned)
}

// Byte offsets of every buffer of a construction, and the peaks.
struct Layout {
    size_t packed = 0, alphabet = 0, ranks = 0, meta = 0;
    size_t text = 0, staging = 0;  // raw bytes: dead once packed, so they share the ranking region
    // ranking region (the packed upload of a batch is staged at its start)
    size_t lst0 = 0, lst1 = 0, key0 = 0, key1 = 0, grp = 0, aux1 = 0, aux2 = 0, rankScratch = 0, scanScratch = 0;
    size_t segScratch = 0;
    size_t counter = 0;
    // class + merge region (overlaps the ranking region)
    size_t lists = 0, classScratch = 0, chain0 = 0, chain1 = 0, splitters = 0, rows = 0, sa = 0, bwt = 0,
           mergeCounter = 0;
    size_t carried = 0;  // one word per list slot, through the class passes and the merge (0: none)
    size_t rankingEnd = 0, classEnd = 0, mergeEnd = 0, peak = 0;
};

// Sizes a layout depends on; for a context they are upper bounds over every batch it admits.
struct Extent {
    uint64_t span, slots, live, outputs, largestClass, splitterWords, rows;
    uint32_t count;
};

Extent extentOf(const Batch& b) {
    return {b.span, b.slots, b.live, b.outputs, b.classes.largest, b.merge.splitterWords, b.merge.rows, b.count};
}

// Bounds for any batch of at most `texts` texts and `total` bytes.
Extent extentBound(uint64_t total, uint32_t texts) {
    Extent e{};
    e.count = std::max<uint32_t>(texts, 1);
    e.span = (total + static_cast<uint64_t>(kV - 1) * e.count + kV - 1) / kV * kV;
    e.slots = (e.span / kV) * kK;
    e.live = std::min<uint64_t>(total, (total / kV) * kK + static_cast<uint64_t>(kK) * e.count);
    e.outputs = total;
    e.largestClass = e.live;
    uint64_t words = 0, rows = 0, level = total;
    while (level > mergeCap(kMergeRMin)) {
        const uint64_t next = level / kMergeG + kClasses;
        words += next + 64;
        rows += (next + kMergeRMin - 1) / kMergeRMin + 1;
        level = next;
    }
    e.splitterWords = words;
    e.rows = rows;
    return e;
}

// carry: room for the carried words (contexts of one text: their constructions carry words when the
// codes take at most 2 bits).
Layout planLayout(const Extent& x, bool internalSa, bool internalBwt, bool carry) {
    Layout L;
    size_t at = 0;
    auto take = [&at](size_t bytes) {
        const size_t offset = at;
        at += align256(bytes);
        return offset;
    };
    L.packed = take(8 * packedWords(x.span, 8));
    L.alphabet = take(4 * 256);
    L.ranks = take(4 * (x.slots + kRankPad));
    L.meta = take(4 * metaWords(x.count, x.span));
    const size_t persistent = at;
    L.text = take(x.span + kTextPad);
    L.staging = x.count > 1 ? take(x.outputs) : 0;
    const size_t rawEnd = at;
    at = persistent;

    const uint64_t m = x.live;
    L.lst0 = take(4 * m);
    L.lst1 = take(4 * m);
    L.key0 = take(8 * m);
    L.key1 = take(8 * m);
    L.grp = take(4 * (m + 64));  // grp and aux2 trade places every pass
    L.aux1 = take(4 * m);
    L.aux2 = take(4 * (m + 64));
    L.rankScratch = take(4 * radixScratchWords(m));
    L.segScratch = take(4 * segScratchWords(m));
    L.scanScratch = take(4 * scanScratchWords(m));
    L.counter = take(256);
    L.rankingEnd = std::max(at, rawEnd);

    at = persistent;
    L.lists = take(4 * x.outputs);
    L.classScratch = take(4 * classScratchWords(x.span, x.count));
    L.chain0 = take(8 * classChainWords(x.live));
    L.chain1 = take(8 * classChainWords(x.live));
    L.classEnd = at;
    at = L.classScratch;  // the merge reuses the class scratch
    L.splitters = take(4 * x.splitterWords);
    L.rows = take(sizeof(MergeRow) * (x.rows + 1));
    L.mergeCounter = take(256);
    L.sa = internalSa ? take(4 * x.outputs) : 0;
    L.bwt = internalBwt ? take(x.outputs) : 0;
    L.mergeEnd = at;
    if (carry) {  // after both the class and the merge region: live through both
        at = std::max(L.classEnd, L.mergeEnd);
        L.carried = take(8 * x.outputs);
        L.classEnd = L.mergeEnd = at;
    }
    L.peak = std::max({L.rankingEnd, L.classEnd, L.mergeEnd});
    return L;
}

// The text whose packed range [packedOffset[j], packedOffset[j + 1]) holds packed byte s (binary
// search; packedOffset has count + 1 entries).
__device__ __forceinline__ uint32_t packedTextOf(const uint32_t* __restrict__ packedOffset, uint32_t count, uint64_t s) {
    uint32_t lo = 0, hi = count;  // last j with packedOffset[j] <= s
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(packedOffset + mid) <= s) lo = mid; else hi = mid;
    }
    return lo;
}

// Copies the packed texts (text j at packedOffset[j]) to their 32-aligned places. Each thread moves
// 16 packed bytes (one aligned load) to their text's place, finding the text once per piece (again
// when the piece crosses into the next text). Gaps are zeroed by placeGaps.
__global__ void placeTexts(const uint8_t* __restrict__ packed, const uint32_t* __restrict__ start,
                           const uint32_t* __restrict__ packedOffset, uint32_t count, uint64_t outputs,
                           uint8_t* __restrict__ text) {
    const uint64_t s0 = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) * 16;
    if (s0 >= outputs) return;
    const uint4 v = *reinterpret_cast<const uint4*>(packed + s0);
    const uint32_t words[4] = {v.x, v.y, v.z, v.w};
    uint32_t j = packedTextOf(packedOffset, count, s0);
    uint32_t next = __ldg(packedOffset + j + 1);
#pragma unroll
    for (int b = 0; b < 16; b++) {
        const uint64_t s = s0 + b;
        if (s >= outputs) break;
        while (s >= next) {  // crossed into the next text (empty texts are not in a batch)
            j++;
            next = __ldg(packedOffset + j + 1);
        }
        text[__ldg(start + j) + (s - __ldg(packedOffset + j))] = static_cast<uint8_t>(words[b >> 2] >> (8 * (b & 3)));
    }
}

// Zeroes the gap after every text (up to the next 32-aligned start) and the padding after the last.
__global__ void placeGaps(const uint32_t* __restrict__ start, const uint32_t* __restrict__ end, uint32_t count,
                          uint32_t span, uint8_t* __restrict__ text) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const uint32_t next = j + 1 < count ? start[j + 1] : span + kTextPad;
    for (uint32_t i = end[j]; i < next; i++) text[i] = 0;
}

// blockText[k] = the text whose range contains or precedes the 32-byte block k (k = 0 .. span / 32).
__global__ void fillBlockText(const uint32_t* __restrict__ start, uint32_t count, uint32_t blocks,
                              uint32_t* __restrict__ blockText) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > blocks) return;
    const uint32_t p = k * kV;
    uint32_t lo = 0, hi = count;  // last j with start[j] <= p
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(start + mid) <= p) lo = mid; else hi = mid;
    }
    blockText[k] = lo;
}

}  // namespace

struct sadcs_gpu_context {
    int device = 0;
    uint64_t capacity = 0;
    uint32_t maxTexts = 1;
    size_t slabBytes = 0;
    bool carryRoom = false;  // the slab has room for carried words (one text)
    uint8_t* slab = nullptr;
    cudaStream_t stream = nullptr;
    uint32_t* hostWords = nullptr;  // page-locked: counters and the per-construction tables
    size_t hostWordCount = 0;
    cudaEvent_t events[6] = {};
    cudaStream_t copyStream = nullptr;  // the outputs' copies to page-locked host buffers during the merge
    cudaEvent_t chunkEvents[kMaxDownloadChunks + 1] = {};
};

namespace {

void destroyContext(sadcs_gpu_context* c) {
    if (!c) return;
    int previous = 0;
    cudaGetDevice(&previous);
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copyStream) cudaStreamSynchronize(c->copyStream);
    for (cudaEvent_t& e : c->events) {
        if (e) cudaEventDestroy(e);
    }
    for (cudaEvent_t& e : c->chunkEvents) {
        if (e) cudaEventDestroy(e);
    }
    if (c->copyStream) cudaStreamDestroy(c->copyStream);
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

// Whether a context for (capacity, texts) has room for carried words: one text, and a capacity that
// reaches the carry threshold (smaller contexts never carry, so they do not pay for the room).
bool planCarry(uint64_t capacity, uint32_t texts) { return texts <= 1 && capacity >= carryMinBytes(); }

size_t contextBytes(int64_t capacity, uint32_t texts, bool carry) {
    return planLayout(extentBound(static_cast<uint64_t>(capacity), texts), true, true, carry).peak;
}

size_t contextBytes(int64_t capacity, uint32_t texts) {
    return contextBytes(capacity, texts, planCarry(static_cast<uint64_t>(capacity), texts));
}

// carryRoom false: no room for carried words whatever the size (callers that never construct).
int createContext(int64_t capacity, uint32_t texts, sadcs_gpu_context** out, bool carryRoom = true) {
    *out = nullptr;
    sadcs_gpu_device device;
    if (const int status = queryDevice(&device); status != SADCS_OK) return status;
    if (capacity < 0 || capacity > kMaxText || texts == 0 || texts > kMaxTexts) {
        setError("capacity %lld bytes / %u texts out of range (0 to %lld bytes, 1 to %u texts)",
                 static_cast<long long>(capacity), texts, static_cast<long long>(kMaxText), kMaxTexts);
        return SADCS_FAILED;
    }
    const bool carry = carryRoom && planCarry(static_cast<uint64_t>(capacity), texts);
    const size_t bytes = contextBytes(capacity, texts, carry);
    if (static_cast<int64_t>(bytes) + kMemoryReserve > device.free_bytes) {
        setError("needs %lld MiB of device memory plus %lld MiB reserve, %lld MiB free",
                 static_cast<long long>(bytes >> 20), static_cast<long long>(kMemoryReserve >> 20),
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
    c->maxTexts = texts;
    c->carryRoom = carry;
    c->slabBytes = bytes;
    // counters, then the host copy of the tables (without the block map, built on the device)
    c->hostWordCount = 64 + metaWords(texts, 0) + 2 * static_cast<size_t>(texts) + 64 + 256;
    cudaError_t error;
    if ((error = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (error = cudaMallocHost(&c->hostWords, 4 * c->hostWordCount)) != cudaSuccess ||
        (error = cudaMalloc(&c->slab, std::max<size_t>(c->slabBytes, 256))) != cudaSuccess) {
        const int status = failed("creating the context", error);
        destroyContext(c);
        return status;
    }
    if ((error = cudaStreamCreateWithFlags(&c->copyStream, cudaStreamNonBlocking)) != cudaSuccess) {
        const int status = failed("creating the context", error);
        destroyContext(c);
        return status;
    }
    for (cudaEvent_t& e : c->chunkEvents) {
        if ((error = cudaEventCreateWithFlags(&e, cudaEventDisableTiming)) != cudaSuccess) {
            const int status = failed("cudaEventCreate", error);
            destroyContext(c);
            return status;
        }
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

// The device address of a page-locked host buffer (allocated or registered with CUDA and mapped
// into the device's address space), or null for pageable memory and null pointers.
void* mappedHost(void* host) {
    if (!host) return nullptr;
    cudaPointerAttributes attributes;
    if (cudaPointerGetAttributes(&attributes, host) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return attributes.type == cudaMemoryTypeHost ? attributes.devicePointer : nullptr;
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

// The alphabet of the placed texts, its key shape and the packed code stream (alphabet.cuh).
// counts: 256 device words; hostCounts: 256 page-locked words. Fills texts' stream fields.
cudaError_t prepareAlphabet(const uint8_t* text, uint64_t total, uint64_t span, uint32_t* counts, uint32_t* hostCounts,
                            uint64_t* packed, TextSet& texts, cudaStream_t stream) {
    SADCS_TRY(cudaMemsetAsync(counts, 0, 256 * 4, stream));
    const uint32_t blocks = std::min<uint32_t>(ceilDiv(total + 3ull, 256 * 4 * 8), 148 * 8);
    SADCS_TRY(launch(alphabetHistogram, std::max(blocks, 1u), 256, 0, stream, text, static_cast<uint32_t>(total), texts,
                     counts));
    SADCS_TRY(cudaMemcpyAsync(hostCounts, counts, 256 * 4, cudaMemcpyDeviceToHost, stream));
    SADCS_TRY(cudaStreamSynchronize(stream));
    // Code k stands for the k-th byte present (in byte order); codes past sigma decode to 0.
    CodeTable table{};
    uint8_t decodeTable[256] = {};
    uint32_t sigma = 0;
    for (int c = 0; c < 256; c++) {
        table.code[c] = static_cast<uint8_t>(sigma);
        if (hostCounts[c]) decodeTable[sigma++] = static_cast<uint8_t>(c);
    }
    uint8_t* decodeHost = reinterpret_cast<uint8_t*>(hostCounts);  // the counts are read by now
    memcpy(decodeHost, decodeTable, sizeof decodeTable);
    uint8_t* decode = reinterpret_cast<uint8_t*>(counts);
    SADCS_TRY(cudaMemcpyAsync(decode, decodeHost, 256, cudaMemcpyHostToDevice, stream));
    const KeyShape shape = keyShape(std::max(sigma, 1u));
    const uint64_t words = packedWords(span, shape.bits);
    const uint64_t groups = ceilDiv(words, packGroupChars(shape.bits) * shape.bits / 64);
    SADCS_TRY(launch(packCodes, ceilDiv(groups, 256), 256, 0, stream, text, static_cast<uint32_t>(total), table,
                     shape.bits, words, packed));
    SADCS_TRY(cudaStreamSynchronize(stream));  // the decode table's host words are reused by the caller
    texts.packed = packed;
    texts.decode = decode;
    texts.bits = shape.bits;
    texts.keyChars = shape.chars;
    texts.tagBits = shape.tagBits;
    return cudaSuccess;
}

// Where a construction's inputs come from and its outputs go.
struct Io {
    const uint8_t* hostText = nullptr;    // packed host texts, or
    const uint8_t* deviceText = nullptr;  // packed device texts, or
    const uint8_t* const* hostPieces = nullptr;  // one host buffer per text (a batch of several)
    uint32_t* const* saPieces = nullptr;  // device-accessible outputs, one per text (a batch of several),
    uint8_t* const* bwtPieces = nullptr;  // in place of outSa / outBwt
    bool wantSa = false, wantBwt = false;
    uint32_t* outSa = nullptr;            // device outputs (caller-owned), or null for the slab's
    uint8_t* outBwt = nullptr;
    uint32_t* hostSa = nullptr;           // page-locked host outputs, copied down from the slab's while
    uint8_t* hostBwt = nullptr;           // the last merge level runs (context copy stream)
    // results
    uint32_t* deviceSa = nullptr;         // where the SA / BWT ended up
    uint8_t* deviceBwt = nullptr;
    uint32_t* rowZero = nullptr;          // device, per text
};

// One construction of a batch on the context's slab.
int construct(sadcs_gpu_context* c, const Batch& b, Io& io, cudaStream_t stream, sadcs_gpu_stats& s) {
    if (b.outputs > c->capacity || b.count > c->maxTexts) {
        setError("input of %llu bytes in %u texts exceeds the context's capacity of %llu bytes / %u texts",
                 static_cast<unsigned long long>(b.outputs), b.count, static_cast<unsigned long long>(c->capacity),
                 c->maxTexts);
        return SADCS_NOT_ENOUGH_MEMORY;
    }
    const Layout L = planLayout(extentOf(b), io.wantSa && !io.outSa && !io.saPieces,
                                io.wantBwt && !io.outBwt && !io.bwtPieces, c->carryRoom && b.count == 1);
    if (L.peak > c->slabBytes) {
        setError("internal: layout of %llu bytes exceeds the slab of %llu", static_cast<unsigned long long>(L.peak),
                 static_cast<unsigned long long>(c->slabBytes));
        return SADCS_FAILED;
    }
    const uint64_t launchesBefore = tLaunches;
    uint8_t* slab = c->slab;
    uint8_t* text = slab + L.text;
    uint32_t* ranks = reinterpret_cast<uint32_t*>(slab + L.ranks);
    uint32_t* meta = reinterpret_cast<uint32_t*>(slab + L.meta);
    const uint32_t J = b.count;
    uint32_t* dStart = meta;
    uint32_t* dEnd = dStart + J;
    uint32_t* dSampleBase = dEnd + J;
    uint32_t* dOutBase = dSampleBase + J;
    uint32_t* dRowZero = dOutBase + J + 1;
    uint32_t* dClassTables = dRowZero + J;
    uint32_t* dBlockText = dClassTables + ClassTables::words(J);
    uint32_t* tablesEnd = dBlockText + (J > 1 ? b.span / kV + 1 : 0);
    uint64_t* dPieces = reinterpret_cast<uint64_t*>(tablesEnd + ((tablesEnd - meta) & 1));  // [sa J][bwt J]
    ClassTables classTables;
    classTables.carve(dClassTables, J);
    cudaError_t error;

    // The tables, staged in page-locked memory and copied in one piece.
    uint32_t* h = c->hostWords + 64;
    std::copy(b.start.begin(), b.start.end(), h);
    std::copy(b.end.begin(), b.end.end(), h + J);
    std::copy(b.sampleBase.begin(), b.sampleBase.end(), h + 2 * J);
    std::copy(b.outBase.begin(), b.outBase.end(), h + 3 * J);
    std::fill(h + 4 * J + 1, h + 5 * J + 1, 0u);
    std::copy(b.classTables.begin(), b.classTables.end(), h + 5 * J + 1);
    if ((error = cudaMemcpyAsync(meta, h, 4 * (5 * static_cast<size_t>(J) + 1 + b.classTables.size()),
                                 cudaMemcpyHostToDevice, stream)) != cudaSuccess) {
        return failed("tables", error);
    }
    if (io.saPieces || io.bwtPieces) {
        uint32_t* after = h + 5 * J + 1 + b.classTables.size();
        uint64_t* hp = reinterpret_cast<uint64_t*>(after + ((after - c->hostWords) & 1));
        for (uint32_t j = 0; j < J; j++) {
            hp[j] = io.saPieces ? reinterpret_cast<uint64_t>(io.saPieces[j]) : 0;
            hp[J + j] = io.bwtPieces ? reinterpret_cast<uint64_t>(io.bwtPieces[j]) : 0;
        }
        if ((error = cudaMemcpyAsync(dPieces, hp, 16 * static_cast<size_t>(J), cudaMemcpyHostToDevice, stream)) !=
            cudaSuccess) {
            return failed("tables", error);
        }
    }

    TextSet texts{};
    texts.count = J;
    texts.start = dStart;
    texts.end = dEnd;
    texts.oneEnd = J == 1 ? b.end[0] : 0;
    texts.blockText = J > 1 ? dBlockText : nullptr;

    // Upload: one text straight into place; several through the ranking region, then placed.
    PhaseRange phase("sadcs upload");
    auto start = std::chrono::steady_clock::now();
    const uint8_t* source = io.hostText ? io.hostText : io.deviceText;
    if (J == 1) {
        if ((error = cudaMemsetAsync(text + b.end[0], 0, b.span + kTextPad - b.end[0], stream)) != cudaSuccess ||
            (error = cudaMemcpyAsync(text, source, b.outputs, io.hostText ? cudaMemcpyHostToDevice
                                                                           : cudaMemcpyDeviceToDevice, stream)) !=
                cudaSuccess) {
            return failed("upload", error);
        }
    } else {
        uint8_t* staging = slab + L.staging;
        uint32_t* packedOffset = reinterpret_cast<uint32_t*>(slab + L.packed);  // free until the codes are packed
        if (io.hostPieces) {
            for (uint32_t j = 0; j < J; j++) {
                if ((error = cudaMemcpyAsync(staging + b.outBase[j], io.hostPieces[j], b.lengths[j],
                                             cudaMemcpyHostToDevice, stream)) != cudaSuccess) {
                    return failed("upload", error);
                }
            }
        } else if ((error = cudaMemcpyAsync(staging, source, b.outputs,
                                            io.hostText ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                            stream)) != cudaSuccess) {
            return failed("upload", error);
        }
        if ((error = cudaMemcpyAsync(packedOffset, dOutBase, 4 * (static_cast<size_t>(J) + 1), cudaMemcpyDeviceToDevice,
                                     stream)) != cudaSuccess) {
            return failed("upload", error);
        }
        const uint32_t blocks = static_cast<uint32_t>(b.span / kV);
        if ((error = launch(placeTexts, ceilDiv(ceilDiv(b.outputs, 16), 256), 256, 0, stream, staging, dStart, packedOffset,
                            J, b.outputs, text)) != cudaSuccess ||
            (error = launch(placeGaps, ceilDiv(J, 256), 256, 0, stream, dStart, dEnd, J, static_cast<uint32_t>(b.span),
                            text)) != cudaSuccess ||
            (error = launch(fillBlockText, ceilDiv(blocks + 1ull, 256), 256, 0, stream, dStart, J, blocks, dBlockText)) !=
                cudaSuccess) {
            return failed("placing the texts", error);
        }
    }
    if (io.hostText || io.hostPieces) {
        s.pinned = isPinned(io.hostText ? io.hostText : io.hostPieces[0]) ? 1 : 0;
        if ((error = cudaStreamSynchronize(stream)) != cudaSuccess) return failed("upload", error);
        s.upload_seconds = secondsSince(start);
    }
    start = std::chrono::steady_clock::now();
    cudaEventRecord(c->events[0], stream);

    // The alphabet and the packed code stream.
    phase.next("sadcs ranking");
    const uint64_t scanned = J == 1 ? b.end[0] : b.end[J - 1];
    if ((error = prepareAlphabet(text, scanned, b.span, reinterpret_cast<uint32_t*>(slab + L.alphabet),
                                 c->hostWords + c->hostWordCount - 256, reinterpret_cast<uint64_t*>(slab + L.packed),
                                 texts, stream)) != cudaSuccess) {
        return failed("alphabet", error);
    }

    // Sample ranking.
    if (J == 1 && (error = cudaMemsetAsync(ranks, 0, 4 * (b.slots + kRankPad), stream)) != cudaSuccess) {
        return failed("ranking", error);
    }
    if (J > 1 && (error = cudaMemsetAsync(ranks + b.slots, 0, 4 * kRankPad, stream)) != cudaSuccess) {
        return failed("ranking", error);
    }
    RankBuffers rb;
    rb.lst[0] = reinterpret_cast<uint32_t*>(slab + L.lst0);
    rb.lst[1] = reinterpret_cast<uint32_t*>(slab + L.lst1);
    rb.key[0] = reinterpret_cast<uint64_t*>(slab + L.key0);
    rb.key[1] = reinterpret_cast<uint64_t*>(slab + L.key1);
    rb.grp = reinterpret_cast<uint32_t*>(slab + L.grp);
    rb.aux1 = reinterpret_cast<uint32_t*>(slab + L.aux1);
    rb.aux2 = reinterpret_cast<uint32_t*>(slab + L.aux2);
    rb.scratch = reinterpret_cast<uint32_t*>(slab + L.rankScratch);
    rb.scanScratch = reinterpret_cast<uint32_t*>(slab + L.scanScratch);
    rb.segScratch = reinterpret_cast<uint32_t*>(slab + L.segScratch);
    rb.counter = reinterpret_cast<uint32_t*>(slab + L.counter);
    rb.keyEntries = static_cast<uint32_t>(std::min(L.key1 - L.key0, L.grp - L.key1) / 8);
    RankStats rankStats;
    if ((error = rankSample(text, texts, static_cast<uint32_t>(b.slots), static_cast<uint32_t>(b.live), dSampleBase,
                            static_cast<uint32_t>(b.longest), ranks, rb, c->hostWords, stream, rankStats)) !=
        cudaSuccess) {
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
    phase.next("sadcs classes");
    uint32_t* lists = reinterpret_cast<uint32_t*>(slab + L.lists);
    uint32_t* classScratch = reinterpret_cast<uint32_t*>(slab + L.classScratch);
    uint64_t* const chains[2] = {reinterpret_cast<uint64_t*>(slab + L.chain0), reinterpret_cast<uint64_t*>(slab + L.chain1)};
    // Carried words: on texts large enough that the final merge's record gathers leave the L2.
    uint64_t* carried = L.carried && carriesWords(texts) && b.outputs >= carryMinBytes()
                            ? reinterpret_cast<uint64_t*>(slab + L.carried)
                            : nullptr;
    if ((error = sortClasses(J == 1 ? b.end[0] : b.end[J - 1], texts, ranks, static_cast<uint32_t>(b.slots), b.classes,
                             classTables, lists, classScratch, chains, carried, stream)) != cudaSuccess) {
        return failed("class sorts", error);
    }
    cudaEventRecord(c->events[2], stream);
    if ((error = cudaMemcpyAsync(c->hostWords + 2, classErrorWord(classScratch, J), sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (error = cudaStreamSynchronize(stream)) != cudaSuccess) {
        return failed("class sorts", error);
    }
    if (c->hostWords[2]) return failed("class sorts", cudaErrorLaunchTimeout);
    s.class_sort_seconds = secondsSince(start);
    s.class_sort_bytes = static_cast<int64_t>(L.classEnd);
    start = std::chrono::steady_clock::now();

    // Merge.
    phase.next("sadcs merge");
    uint32_t* const* saPieces = io.saPieces ? reinterpret_cast<uint32_t* const*>(dPieces) : nullptr;
    uint8_t* const* bwtPieces = io.bwtPieces ? reinterpret_cast<uint8_t* const*>(dPieces + J) : nullptr;
    uint32_t* sa = saPieces ? nullptr
                            : (io.outSa ? io.outSa : (io.wantSa ? reinterpret_cast<uint32_t*>(slab + L.sa) : nullptr));
    uint8_t* bwt = bwtPieces ? nullptr : (io.outBwt ? io.outBwt : (io.wantBwt ? slab + L.bwt : nullptr));
    // The merge's tile shape follows the code width, known now (the memory plan bounds every shape).
    const MergePlan mergePlan = planMerge(b.classes.start, mergeR(finalWords(texts.bits)));
    OverlappedDownload download;
    const bool overlapped = (io.hostSa || io.hostBwt) && c->copyStream;
    if (overlapped) {
        download.sa = io.hostSa;
        download.bwt = io.hostBwt;
        download.deviceSa = sa;
        download.deviceBwt = bwt;
        download.stream = c->copyStream;
        download.events = c->chunkEvents;
        download.hostRows = c->hostWords + 64;  // the tables' staging words, free since their upload
        download.outputs = b.outputs;
    }
    if ((error = mergeClasses(text, ranks, texts, lists, mergePlan, classTables.rowBase, dOutBase, dRowZero,
                              reinterpret_cast<uint32_t*>(slab + L.splitters),
                              reinterpret_cast<MergeRow*>(slab + L.rows), sa, bwt,
                              reinterpret_cast<uint32_t*>(slab + L.mergeCounter), c->hostWords, stream,
                              c->events[4], c->events[5], saPieces, bwtPieces, carried,
                              overlapped ? &download : nullptr)) != cudaSuccess) {
        if (overlapped) cudaStreamSynchronize(c->copyStream);
        return failed("merge", error);
    }
    if (overlapped && (error = cudaStreamSynchronize(c->copyStream)) != cudaSuccess) return failed("download", error);
    cudaEventRecord(c->events[3], stream);
    if ((error = cudaStreamSynchronize(stream)) != cudaSuccess) return failed("merge", error);
    s.merge_seconds = secondsSince(start);
    s.merge_bytes = static_cast<int64_t>(L.mergeEnd);
    s.device_bytes = static_cast<int64_t>(L.peak);
    s.device_seconds = elapsedMs(c->events[0], c->events[3]) / 1000.0;
    s.ranking_device_ms = elapsedMs(c->events[0], c->events[1]);
    s.class_sort_device_ms = elapsedMs(c->events[1], c->events[2]);
    s.merge_device_ms = elapsedMs(c->events[2], c->events[3]);
    s.merge_kernel_ms = elapsedMs(c->events[4], c->events[5]);
    s.kernel_launches = static_cast<int64_t>(tLaunches - launchesBefore);
    io.deviceSa = sa;
    io.deviceBwt = bwt;
    io.rowZero = dRowZero;
    return SADCS_OK;
}

// Runs body(context) with the given context, or a temporary one for `total` bytes in `texts` texts
// (its creation is setup).
template <class Body>
int withContext(sadcs_gpu_context* context, uint64_t total, uint32_t texts, sadcs_gpu_stats& s, Body body,
                bool carryRoom = true) {
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
    if (const int status = createContext(static_cast<int64_t>(total), texts, &temporary, carryRoom);
        status != SADCS_OK) {
        return status;
    }
    s.setup_seconds = secondsSince(start);
    const int status = body(temporary);
    const double setup = s.setup_seconds;
    destroyContext(temporary);
    s.setup_seconds = setup;
    return status;
}

// How page-locked host outputs are filled: copied down in pieces while the last merge level runs
// (the default), written by the last merge level itself through their device mapping, or copied
// down after the construction. The environment's SADCS_HOST_OUTPUTS ("overlapped", "mapped",
// "after") overrides the default, read at each call (tests and tuning).
enum class HostOutputs { Overlapped, Mapped, After };
HostOutputs hostOutputMode() {
    const char* v = std::getenv("SADCS_HOST_OUTPUTS");
    if (v && std::strcmp(v, "mapped") == 0) return HostOutputs::Mapped;
    if (v && std::strcmp(v, "after") == 0) return HostOutputs::After;
    return HostOutputs::Overlapped;
}

int download(sadcs_gpu_context* c, void* host, const void* device, size_t bytes, sadcs_gpu_stats& s) {
    if (bytes == 0) return SADCS_OK;
    const auto start = std::chrono::steady_clock::now();
    cudaError_t error;
    if ((error = cudaMemcpyAsync(host, device, bytes, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess ||
        (error = cudaStreamSynchronize(c->stream)) != cudaSuccess) {
        return failed("download", error);
    }
    s.download_seconds += secondsSince(start);
    return SADCS_OK;
}

// The rows of the texts' first suffixes, read back: primary = row + 1 per text.
int readPrimaries(sadcs_gpu_context* c, const Io& io, uint32_t count, int64_t* primaries) {
    uint32_t* h = c->hostWords + 64;
    cudaError_t error;
    if ((error = cudaMemcpyAsync(h, io.rowZero, 4 * static_cast<size_t>(count), cudaMemcpyDeviceToHost, c->stream)) !=
            cudaSuccess ||
        (error = cudaStreamSynchronize(c->stream)) != cudaSuccess) {
        return failed("download", error);
    }
    for (uint32_t j = 0; j < count; j++) primaries[j] = static_cast<int64_t>(h[j]) + 1;
    return SADCS_OK;
}

// A batch of the non-empty texts among lengths[0, count): their indices in `kept`.
int batchOf(const int64_t* lengths, int64_t count, Batch& b, std::vector<uint32_t>& kept) {
    if (count < 0 || count > static_cast<int64_t>(kMaxTexts)) {
        setError("%lld texts out of range (at most %u)", static_cast<long long>(count), kMaxTexts);
        return SADCS_FAILED;
    }
    std::vector<uint64_t> nonEmpty;
    for (int64_t j = 0; j < count; j++) {
        if (lengths[j] < 0) {
            setError("text %lld has a negative length", static_cast<long long>(j));
            return SADCS_FAILED;
        }
        if (lengths[j] > 0) {
            nonEmpty.push_back(static_cast<uint64_t>(lengths[j]));
            kept.push_back(static_cast<uint32_t>(j));
        }
    }
    if (!planBatch(nonEmpty.data(), static_cast<uint32_t>(nonEmpty.size()), b)) {
        setError("texts exceed %lld bytes together", static_cast<long long>(kMaxText));
        return SADCS_FAILED;
    }
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
    return n == 0 ? 0 : static_cast<int64_t>(contextBytes(n, 1));
}

int64_t sadcs_gpu_required_bytes_batch(int64_t total, int64_t texts) {
    if (total < 0 || total > kMaxText || texts < 1 || texts > static_cast<int64_t>(kMaxTexts)) return -1;
    return static_cast<int64_t>(contextBytes(total, static_cast<uint32_t>(texts)));
}

int sadcs_gpu_create_context(int64_t capacity, sadcs_gpu_context** context) {
    tLastError[0] = '\0';
    if (!context) {
        setError("context pointer is null");
        return SADCS_FAILED;
    }
    return createContext(std::max<int64_t>(capacity, 0), 1, context);
}

int sadcs_gpu_create_batch_context(int64_t capacity, int64_t max_texts, sadcs_gpu_context** context) {
    tLastError[0] = '\0';
    if (!context) {
        setError("context pointer is null");
        return SADCS_FAILED;
    }
    if (max_texts < 1 || max_texts > static_cast<int64_t>(kMaxTexts)) {
        setError("max_texts %lld out of range (1 to %u)", static_cast<long long>(max_texts), kMaxTexts);
        return SADCS_FAILED;
    }
    return createContext(std::max<int64_t>(capacity, 0), static_cast<uint32_t>(max_texts), context);
}

void sadcs_gpu_destroy_context(sadcs_gpu_context* context) {
    destroyContext(context);
}

int64_t sadcs_gpu_context_capacity(const sadcs_gpu_context* context) {
    return context ? static_cast<int64_t>(context->capacity) : 0;
}

int sadcs_gpu_build_batch(sadcs_gpu_context* context, const uint8_t* texts, const int64_t* lengths, int64_t count,
                          uint32_t* sa, uint8_t* bwt, int64_t* primaries, sadcs_gpu_stats* stats) {
    tLastError[0] = '\0';
    sadcs_gpu_stats local{};
    sadcs_gpu_stats& s = stats ? *stats : local;
    s = sadcs_gpu_stats{};
    if (!sa && !bwt) {
        setError("neither a suffix array nor a BWT was asked for");
        return SADCS_FAILED;
    }
    if (count > 0 && !lengths) {
        setError("lengths is null");
        return SADCS_FAILED;
    }
    for (int64_t j = 0; primaries && j < count; j++) primaries[j] = 0;
    Batch b;
    std::vector<uint32_t> kept;
    if (const int status = batchOf(lengths, count, b, kept); status != SADCS_OK) return status;
    if (b.count == 0) return context ? SADCS_OK : queryDevice(nullptr);
    if (!texts) {
        setError("texts is null");
        return SADCS_FAILED;
    }
    return withContext(context, b.outputs, b.count, s, [&](sadcs_gpu_context* c) -> int {
        Io io;
        io.hostText = texts;
        io.wantSa = sa != nullptr;
        io.wantBwt = bwt != nullptr;
        // Page-locked outputs are copied down piece by piece while the last merge level runs (or
        // written by the merge itself over the host link, or copied after it: hostOutputMode).
        const HostOutputs mode = hostOutputMode();
        uint32_t* mappedSa = static_cast<uint32_t*>(mappedHost(sa));
        uint8_t* mappedBwt = static_cast<uint8_t*>(mappedHost(bwt));
        if (mode == HostOutputs::Mapped) {
            io.outSa = mappedSa;
            io.outBwt = mappedBwt;
        } else if (mode == HostOutputs::Overlapped && c->copyStream) {
            io.hostSa = mappedSa ? sa : nullptr;
            io.hostBwt = mappedBwt ? bwt : nullptr;
        }
        int status = construct(c, b, io, c->stream, s);
        if (status != SADCS_OK) return status;
        if (sa && !io.outSa && !io.hostSa && (status = download(c, sa, io.deviceSa, 4 * b.outputs, s)) != SADCS_OK) {
            return status;
        }
        if (bwt && !io.outBwt && !io.hostBwt && (status = download(c, bwt, io.deviceBwt, b.outputs, s)) != SADCS_OK) {
            return status;
        }
        if (bwt && primaries) {
            std::vector<int64_t> p(b.count);
            if ((status = readPrimaries(c, io, b.count, p.data())) != SADCS_OK) return status;
            for (uint32_t k = 0; k < b.count; k++) primaries[kept[k]] = p[k];
        }
        return SADCS_OK;
    });
}

int sadcs_gpu_build_batch_device(sadcs_gpu_context* context, const uint8_t* d_texts, const int64_t* lengths,
                                 int64_t count, uint32_t* d_sa, uint8_t* d_bwt, int64_t* primaries, void* stream,
                                 sadcs_gpu_stats* stats) {
    tLastError[0] = '\0';
    sadcs_gpu_stats local{};
    sadcs_gpu_stats& s = stats ? *stats : local;
    s = sadcs_gpu_stats{};
    if (!d_sa && !d_bwt) {
        setError("neither a suffix array nor a BWT was asked for");
        return SADCS_FAILED;
    }
    if (count > 0 && !lengths) {
        setError("lengths is null");
        return SADCS_FAILED;
    }
    for (int64_t j = 0; primaries && j < count; j++) primaries[j] = 0;
    Batch b;
    std::vector<uint32_t> kept;
    if (const int status = batchOf(lengths, count, b, kept); status != SADCS_OK) return status;
    if (b.count == 0) return context ? SADCS_OK : queryDevice(nullptr);
    return withContext(context, b.outputs, b.count, s, [&](sadcs_gpu_context* c) -> int {
        Io io;
        io.deviceText = d_texts;
        io.wantSa = d_sa != nullptr;
        io.wantBwt = d_bwt != nullptr;
        io.outSa = d_sa;
        io.outBwt = d_bwt;
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
        const int status = construct(c, b, io, st, s);
        if (status != SADCS_OK) return status;
        if (d_bwt && primaries) {
            uint32_t* h = c->hostWords + 64;
            cudaError_t error;
            if ((error = cudaMemcpyAsync(h, io.rowZero, 4 * static_cast<size_t>(b.count), cudaMemcpyDeviceToHost, st)) !=
                    cudaSuccess ||
                (error = cudaStreamSynchronize(st)) != cudaSuccess) {
                return failed("download", error);
            }
            for (uint32_t k = 0; k < b.count; k++) primaries[kept[k]] = static_cast<int64_t>(h[k]) + 1;
        }
        return SADCS_OK;
    });
}

int sadcs_gpu_build(sadcs_gpu_context* context, const uint8_t* text, int64_t n, uint32_t* sa, uint8_t* bwt,
                    int64_t* primary, sadcs_gpu_stats* stats) {
    if (n > kMaxText) {
        tLastError[0] = '\0';
        setError("text of %lld bytes exceeds the limit of %lld", static_cast<long long>(n), static_cast<long long>(kMaxText));
        if (stats) *stats = sadcs_gpu_stats{};
        return SADCS_FAILED;
    }
    const int64_t length = std::max<int64_t>(n, 0);
    int64_t p = 0;
    const int status = sadcs_gpu_build_batch(context, text, &length, 1, sa, bwt, &p, stats);
    if (primary) *primary = status == SADCS_OK ? (bwt ? p : -1) : (n > 0 ? -1 : 0);
    if (primary && n <= 0) *primary = 0;
    return status;
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
    if (n > kMaxText) {
        tLastError[0] = '\0';
        setError("text of %lld bytes exceeds the limit of %lld", static_cast<long long>(n), static_cast<long long>(kMaxText));
        if (stats) *stats = sadcs_gpu_stats{};
        return SADCS_FAILED;
    }
    const int64_t length = std::max<int64_t>(n, 0);
    int64_t p = 0;
    const int status = sadcs_gpu_build_batch_device(context, d_text, &length, 1, d_sa, d_bwt, &p, stream, stats);
    if (primary) *primary = n <= 0 ? 0 : (status == SADCS_OK && d_bwt ? p : -1);
    return status;
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

int sadcs_gpu_check_suffix_array(const uint8_t* d_text, int64_t n, const uint32_t* d_sa, int64_t* bad_index,
                                 const char** reason, void* stream) {
    tLastError[0] = '\0';
    if (bad_index) *bad_index = -1;
    if (reason) *reason = nullptr;
    if (n <= 0) return SADCS_OK;
    if (n > kMaxText) {
        setError("text of %lld bytes exceeds the limit of %lld", static_cast<long long>(n), static_cast<long long>(kMaxText));
        return SADCS_FAILED;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t count = static_cast<uint32_t>(n);
    uint32_t* isa = nullptr;
    unsigned long long* words = nullptr;
    unsigned long long* host = nullptr;
    cudaError_t error;
    if ((error = cudaMallocAsync(&isa, 4 * static_cast<size_t>(n), st)) != cudaSuccess) return failed("cudaMallocAsync", error);
    if ((error = cudaMallocAsync(&words, 3 * sizeof(unsigned long long), st)) != cudaSuccess ||
        (error = cudaMallocHost(&host, 3 * sizeof(unsigned long long))) != cudaSuccess) {
        cudaFreeAsync(isa, st);
        if (words) cudaFreeAsync(words, st);
        return failed("allocating check buffers", error);
    }
    const uint32_t blocks = (count + 255) / 256;
    error = cudaMemsetAsync(words, 0xFF, 3 * sizeof(unsigned long long), st);
    if (error == cudaSuccess) error = cudaMemsetAsync(isa, 0, 4 * static_cast<size_t>(count), st);
    if (error == cudaSuccess) error = launch(checkScatter, blocks, 256, 0, st, d_sa, count, isa, words);
    if (error == cudaSuccess) error = cudaMemcpyAsync(host, words, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (error == cudaSuccess) error = cudaStreamSynchronize(st);
    const char* why = nullptr;
    int64_t index = -1;
    if (error == cudaSuccess && host[0] != kNoFailure) {
        why = "entry out of range";
        index = static_cast<int64_t>(host[0]);
    }
    if (error == cudaSuccess && !why) {
        error = launch(checkDuplicates, blocks, 256, 0, st, d_sa, count, isa, words + 1);
        if (error == cudaSuccess) error = launch(checkOrder, blocks, 256, 0, st, d_text, d_sa, count, isa, words + 2);
        if (error == cudaSuccess)
            error = cudaMemcpyAsync(host + 1, words + 1, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
        if (error == cudaSuccess) error = cudaStreamSynchronize(st);
        if (error == cudaSuccess && host[1] != kNoFailure) {
            why = "duplicate entry";
            index = static_cast<int64_t>(host[1]);
        } else if (error == cudaSuccess && host[2] != kNoFailure) {
            why = "SA[index] and SA[index + 1] out of order";
            index = static_cast<int64_t>(host[2]);
        }
    }
    cudaFreeAsync(isa, st);
    cudaFreeAsync(words, st);
    cudaStreamSynchronize(st);
    cudaFreeHost(host);
    if (error != cudaSuccess) return failed("suffix array check", error);
    if (bad_index) *bad_index = index;
    if (reason) *reason = why;
    return SADCS_OK;
}

// ---- the suffix array check without allocation ------------------------------------------------

namespace {

// Scratch of sadcs_gpu_check_suffix_array_static, in module memory: three 64-bit result words at
// word 0 (set to all ones by every call), the inverse suffix array from word 64 (its first n words
// set to zero by every call: the scatter keeps the largest index per entry). Shared by every call
// on a device, so overlapping calls race.
constexpr int64_t kStaticCheckMax = SADCS_GPU_STATIC_CHECK_MAX;
constexpr size_t kStaticCheckIsaWord = 64;
static __device__ __align__(256) uint32_t gStaticCheckScratch[kStaticCheckIsaWord + kStaticCheckMax];

constexpr int kStaticCheckDevices = 64;
std::mutex gStaticCheckLock;
uint32_t* gStaticCheckAddress[kStaticCheckDevices] = {};

// The scratch's device address on the current device, looked up on the first call per device.
cudaError_t staticCheckScratch(uint32_t** out) {
    int device = 0;
    cudaError_t error = cudaGetDevice(&device);
    if (error != cudaSuccess) return error;
    if (device < 0 || device >= kStaticCheckDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> hold(gStaticCheckLock);
    if (!gStaticCheckAddress[device]) {
        void* address = nullptr;
        if ((error = cudaGetSymbolAddress(&address, gStaticCheckScratch)) != cudaSuccess) return error;
        gStaticCheckAddress[device] = static_cast<uint32_t*>(address);
    }
    *out = gStaticCheckAddress[device];
    return cudaSuccess;
}

}  // namespace

int sadcs_gpu_check_suffix_array_static(const uint8_t* d_text, int64_t n, const uint32_t* d_sa, int64_t* bad_index,
                                        const char** reason, void* stream) {
    tLastError[0] = '\0';
    if (bad_index) *bad_index = -1;
    if (reason) *reason = nullptr;
    if (n <= 0) return SADCS_OK;
    if (n > kStaticCheckMax) {
        setError("text of %lld bytes exceeds the %lld entries of the static scratch of "
                 "sadcs_gpu_check_suffix_array_static (sadcs_gpu_check_suffix_array has no such limit)",
                 static_cast<long long>(n), static_cast<long long>(kStaticCheckMax));
        return SADCS_FAILED;
    }
    uint32_t* scratch = nullptr;
    cudaError_t error = staticCheckScratch(&scratch);
    if (error != cudaSuccess) return failed("cudaGetSymbolAddress of the static check scratch", error);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t count = static_cast<uint32_t>(n);
    unsigned long long* words = reinterpret_cast<unsigned long long*>(scratch);
    uint32_t* isa = scratch + kStaticCheckIsaWord;
    unsigned long long host[3] = {kNoFailure, kNoFailure, kNoFailure};  // pageable: nothing is allocated
    const uint32_t blocks = (count + 255) / 256;
    error = cudaMemsetAsync(words, 0xFF, 3 * sizeof(unsigned long long), st);
    if (error == cudaSuccess) error = cudaMemsetAsync(isa, 0, 4 * static_cast<size_t>(count), st);
    if (error == cudaSuccess) error = launch(checkScatter, blocks, 256, 0, st, d_sa, count, isa, words);
    if (error == cudaSuccess) error = cudaMemcpyAsync(host, words, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (error == cudaSuccess) error = cudaStreamSynchronize(st);
    const char* why = nullptr;
    int64_t index = -1;
    if (error == cudaSuccess && host[0] != kNoFailure) {
        why = "entry out of range";
        index = static_cast<int64_t>(host[0]);
    }
    if (error == cudaSuccess && !why) {
        error = launch(checkDuplicates, blocks, 256, 0, st, d_sa, count, isa, words + 1);
        if (error == cudaSuccess) error = launch(checkOrder, blocks, 256, 0, st, d_text, d_sa, count, isa, words + 2);
        if (error == cudaSuccess)
            error = cudaMemcpyAsync(host + 1, words + 1, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
        if (error == cudaSuccess) error = cudaStreamSynchronize(st);
        if (error == cudaSuccess && host[1] != kNoFailure) {
            why = "duplicate entry";
            index = static_cast<int64_t>(host[1]);
        } else if (error == cudaSuccess && host[2] != kNoFailure) {
            why = "SA[index] and SA[index + 1] out of order";
            index = static_cast<int64_t>(host[2]);
        }
    }
    if (error != cudaSuccess) return failed("suffix array check (static scratch)", error);
    if (bad_index) *bad_index = index;
    if (reason) *reason = why;
    return SADCS_OK;
}

namespace {

// Inverse BWT into d_out with temporary device memory; valid = false for a broken BWT.
int inverseWithScratch(const uint8_t* d_bwt, int64_t n, int64_t primary, uint8_t* d_out, cudaStream_t st, bool& valid) {
    uint32_t* scratch = nullptr;
    uint32_t* host = nullptr;
    cudaError_t error;
    if ((error = cudaMallocAsync(&scratch, 4 * inverseScratchWords(static_cast<uint64_t>(n)), st)) != cudaSuccess) {
        return failed("cudaMallocAsync", error);
    }
    if ((error = cudaMallocHost(&host, 16)) != cudaSuccess) {
        cudaFreeAsync(scratch, st);
        return failed("cudaMallocHost", error);
    }
    error = inverseBwt(d_bwt, static_cast<uint32_t>(n), static_cast<uint32_t>(primary), d_out, scratch, host, st, valid);
    cudaFreeAsync(scratch, st);
    cudaStreamSynchronize(st);
    cudaFreeHost(host);
    return error == cudaSuccess ? SADCS_OK : failed("inverse BWT", error);
}

}  // namespace

int sadcs_gpu_inverse_bwt(const uint8_t* d_bwt, int64_t n, int64_t primary, uint8_t* d_text, void* stream) {
    tLastError[0] = '\0';
    if (n <= 0) return SADCS_OK;
    if (n > kMaxText || primary < 1 || primary > n) {
        setError("invalid BWT: n %lld, primary %lld", static_cast<long long>(n), static_cast<long long>(primary));
        return SADCS_FAILED;
    }
    bool valid = true;
    const int status = inverseWithScratch(d_bwt, n, primary, d_text, static_cast<cudaStream_t>(stream), valid);
    if (status == SADCS_OK && !valid) {
        setError("not a valid BWT: LF misses the primary row");
        return SADCS_FAILED;
    }
    return status;
}

int sadcs_gpu_check_bwt(const uint8_t* d_text, int64_t n, const uint8_t* d_bwt, int64_t primary, int64_t* bad_index,
                        void* stream) {
    tLastError[0] = '\0';
    if (bad_index) *bad_index = -1;
    if (n <= 0) {
        if (bad_index && primary != 0) *bad_index = 0;
        return SADCS_OK;
    }
    if (n > kMaxText) {
        setError("text of %lld bytes exceeds the limit of %lld", static_cast<long long>(n), static_cast<long long>(kMaxText));
        return SADCS_FAILED;
    }
    if (primary < 1 || primary > n) {
        if (bad_index) *bad_index = 0;
        return SADCS_OK;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint8_t* inverse = nullptr;
    unsigned long long* word = nullptr;
    unsigned long long host = 0;
    cudaError_t error;
    if ((error = cudaMallocAsync(&inverse, static_cast<size_t>(n), st)) != cudaSuccess ||
        (error = cudaMallocAsync(&word, 8, st)) != cudaSuccess) {
        if (inverse) cudaFreeAsync(inverse, st);
        return failed("cudaMallocAsync", error);
    }
    bool valid = true;
    int status = inverseWithScratch(d_bwt, n, primary, inverse, st, valid);
    if (status == SADCS_OK && valid) {
        if ((error = cudaMemsetAsync(word, 0xFF, 8, st)) != cudaSuccess ||
            (error = launch(lfCompare, ceilDiv(n, 256), 256, 0, st, d_text, inverse, static_cast<uint32_t>(n), word)) !=
                cudaSuccess ||
            (error = cudaMemcpyAsync(&host, word, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (error = cudaStreamSynchronize(st)) != cudaSuccess) {
            status = failed("BWT check", error);
        } else if (bad_index && host != kNoFailure) {
            *bad_index = static_cast<int64_t>(host);
        }
    } else if (status == SADCS_OK && bad_index) {
        *bad_index = 0;
    }
    cudaFreeAsync(inverse, st);
    cudaFreeAsync(word, st);
    cudaStreamSynchronize(st);
    return status;
}

}  // extern "C"

namespace {

// Device copies of a host check's inputs, on a stream of the check's own; the destructor frees
// them and the stream once the check's work on it is done.
struct HostCheckInputs {
    cudaStream_t stream = nullptr;
    void* first = nullptr;
    void* second = nullptr;

    cudaError_t upload(const void* a, size_t aBytes, const void* b, size_t bBytes) {
        cudaError_t error;
        if ((error = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)) != cudaSuccess) {
            stream = nullptr;
            return error;
        }
        if ((error = cudaMallocAsync(&first, aBytes, stream)) != cudaSuccess) return error;
        if ((error = cudaMallocAsync(&second, bBytes, stream)) != cudaSuccess) return error;
        if ((error = cudaMemcpyAsync(first, a, aBytes, cudaMemcpyHostToDevice, stream)) != cudaSuccess) return error;
        return cudaMemcpyAsync(second, b, bBytes, cudaMemcpyHostToDevice, stream);
    }
    ~HostCheckInputs() {
        if (!stream) return;
        if (first) cudaFreeAsync(first, stream);
        if (second) cudaFreeAsync(second, stream);
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
    }
};

}  // namespace

extern "C" {

int sadcs_gpu_check_suffix_array_host(const uint8_t* text, int64_t n, const uint32_t* sa, int64_t* bad_index,
                                      const char** reason) {
    tLastError[0] = '\0';
    if (bad_index) *bad_index = -1;
    if (reason) *reason = nullptr;
    if (n <= 0) return SADCS_OK;
    if (n > kMaxText) {
        setError("text of %lld bytes exceeds the limit of %lld", static_cast<long long>(n), static_cast<long long>(kMaxText));
        return SADCS_FAILED;
    }
    if (!text || !sa) {
        setError("text or suffix array is null");
        return SADCS_FAILED;
    }
    HostCheckInputs in;
    if (const cudaError_t error = in.upload(text, static_cast<size_t>(n), sa, 4 * static_cast<size_t>(n));
        error != cudaSuccess) {
        return failed("uploading the check's inputs", error);
    }
    return sadcs_gpu_check_suffix_array(static_cast<const uint8_t*>(in.first), n,
                                        static_cast<const uint32_t*>(in.second), bad_index, reason, in.stream);
}

int sadcs_gpu_check_bwt_host(const uint8_t* text, int64_t n, const uint8_t* bwt, int64_t primary, int64_t* bad_index) {
    tLastError[0] = '\0';
    if (bad_index) *bad_index = -1;
    if (n <= 0 || primary < 1 || primary > n) {  // decided without the device, as the device check does
        return sadcs_gpu_check_bwt(nullptr, n, nullptr, primary, bad_index, nullptr);
    }
    if (n > kMaxText) {
        setError("text of %lld bytes exceeds the limit of %lld", static_cast<long long>(n), static_cast<long long>(kMaxText));
        return SADCS_FAILED;
    }
    if (!text || !bwt) {
        setError("text or BWT is null");
        return SADCS_FAILED;
    }
    HostCheckInputs in;
    if (const cudaError_t error = in.upload(text, static_cast<size_t>(n), bwt, static_cast<size_t>(n));
        error != cudaSuccess) {
        return failed("uploading the check's inputs", error);
    }
    return sadcs_gpu_check_bwt(static_cast<const uint8_t*>(in.first), n, static_cast<const uint8_t*>(in.second),
                               primary, bad_index, in.stream);
}

int sadcs_gpu_test_lookback_timeout(int64_t limit_cycles, uint32_t* error_word) {
    tLastError[0] = '\0';
    if (error_word) *error_word = 0;
    if (limit_cycles <= 0 || limit_cycles > kLookbackLimitCycles) {
        setError("limit of %lld cycles out of range (1 to %lld)", static_cast<long long>(limit_cycles),
                 static_cast<long long>(kLookbackLimitCycles));
        return SADCS_FAILED;
    }
    // One radix pass of two tiles' elements in which a single block takes tile 1: tile 0 is never
    // taken, so its status words stay zero and the block's look-back waits on them until the limit.
    constexpr uint32_t count = 2 * kSortTile;
    cudaStream_t st = nullptr;
    cudaError_t error = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (error != cudaSuccess) return failed("cudaStreamCreate", error);
    uint64_t* keys = nullptr;
    uint32_t* vals = nullptr;
    uint32_t* scratch = nullptr;
    const size_t keyBytes = 2 * 8 * static_cast<size_t>(count), valBytes = 2 * 4 * static_cast<size_t>(count);
    const size_t scratchBytes = 4 * radixScratchWords(count);
    uint32_t word = 0;
    if ((error = cudaMallocAsync(&keys, keyBytes, st)) == cudaSuccess &&
        (error = cudaMallocAsync(&vals, valBytes, st)) == cudaSuccess &&
        (error = cudaMallocAsync(&scratch, scratchBytes, st)) == cudaSuccess &&
        (error = cudaMemsetAsync(keys, 0, keyBytes, st)) == cudaSuccess &&
        (error = cudaMemsetAsync(vals, 0, valBytes, st)) == cudaSuccess &&
        (error = cudaMemsetAsync(scratch, 0, scratchBytes, st)) == cudaSuccess) {
        const RadixScratch radix(scratch, count);
        SortLoader<uint64_t> ld{keys, vals, 0};
        SortStorer<uint64_t> out{keys + count, vals + count, count};
        error = radixOnesweepPass<uint64_t>(ld, out, OneSegment{count}, count, 1, radix.digitBase, radix, st,
                                            static_cast<long long>(limit_cycles), 1);
        if (error == cudaSuccess) {
            error = cudaMemcpyAsync(&word, radix.control + 1, sizeof word, cudaMemcpyDeviceToHost, st);
        }
        if (error == cudaSuccess) error = cudaStreamSynchronize(st);
    }
    if (keys) cudaFreeAsync(keys, st);
    if (vals) cudaFreeAsync(vals, st);
    if (scratch) cudaFreeAsync(scratch, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (error != cudaSuccess) return failed("look-back time-out test", error);
    if (error_word) *error_word = word;
    if (word) {
        setError("radix look-back gave up after %lld cycles (error word %u): nothing was stored",
                 static_cast<long long>(limit_cycles), word);
        return SADCS_FAILED;
    }
    return SADCS_OK;
}

int sadcs_gpu_lcp(const uint8_t* d_text, int64_t n, const uint32_t* d_sa, uint32_t* d_lcp, void* stream) {
    tLastError[0] = '\0';
    if (n <= 0) return SADCS_OK;
    if (n > kMaxText) {
        setError("text of %lld bytes exceeds the limit of %lld", static_cast<long long>(n), static_cast<long long>(kMaxText));
        return SADCS_FAILED;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PhaseRange phase("sadcs lcp");
    uint32_t* scratch = nullptr;
    cudaError_t error = cudaMallocAsync(&scratch, 4 * lcp::scratchWords(static_cast<uint64_t>(n)), st);
    if (error != cudaSuccess) return failed("cudaMallocAsync", error);
    error = lcp::lcpArray(d_text, static_cast<uint32_t>(n), d_sa, d_lcp, scratch, st);
    cudaFreeAsync(scratch, st);
    const cudaError_t done = cudaStreamSynchronize(st);
    if (error == cudaSuccess) error = done;
    return error == cudaSuccess ? SADCS_OK : failed("LCP array", error);
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
    const uint64_t length = static_cast<uint64_t>(n);
    Batch b;
    planBatch(&length, 1, b);
    return withContext(nullptr, length, 1, s, [&](sadcs_gpu_context* c) -> int {
        const Layout L = planLayout(extentOf(b), false, false, false);
        uint8_t* textBuffer = c->slab + L.text;
        uint32_t* rankBuffer = reinterpret_cast<uint32_t*>(c->slab + L.ranks);
        cudaError_t error;
        auto start = std::chrono::steady_clock::now();
        if ((error = cudaMemsetAsync(textBuffer + n, 0, b.span + kTextPad - length, c->stream)) != cudaSuccess ||
            (error = cudaMemcpyAsync(textBuffer, text, length, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
            (error = cudaMemsetAsync(rankBuffer, 0, 4 * (b.slots + kRankPad), c->stream)) != cudaSuccess ||
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
        rb.scanScratch = reinterpret_cast<uint32_t*>(c->slab + L.scanScratch);
        rb.segScratch = reinterpret_cast<uint32_t*>(c->slab + L.segScratch);
        rb.counter = reinterpret_cast<uint32_t*>(c->slab + L.counter);
        rb.keyEntries = static_cast<uint32_t>(std::min(L.key1 - L.key0, L.grp - L.key1) / 8);
        TextSet texts{};
        texts.count = 1;
        texts.oneEnd = static_cast<uint32_t>(length);
        if ((error = prepareAlphabet(textBuffer, length, b.span, reinterpret_cast<uint32_t*>(c->slab + L.alphabet),
                                     c->hostWords + c->hostWordCount - 256,
                                     reinterpret_cast<uint64_t*>(c->slab + L.packed), texts, c->stream)) !=
            cudaSuccess) {
            return failed("alphabet", error);
        }
        RankStats rankStats;
        if ((error = rankSample(textBuffer, texts, static_cast<uint32_t>(b.slots), static_cast<uint32_t>(b.live),
                                nullptr, static_cast<uint32_t>(length), rankBuffer, rb, c->hostWords, c->stream,
                                rankStats)) != cudaSuccess) {
            return failed("sample ranking", error);
        }
        s.character_passes = rankStats.characterPasses;
        s.doubling_rounds = rankStats.doublingRounds;
        s.ranking_seconds = secondsSince(start);
        s.device_seconds = s.ranking_seconds;
        s.ranking_bytes = static_cast<int64_t>(L.rankingEnd);
        s.device_bytes = s.ranking_bytes;
        return download(c, ranks, rankBuffer, 4 * b.live, s);
    }, /*carryRoom=*/false);  // ranking only: no class passes
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

#include "server.cuh"
