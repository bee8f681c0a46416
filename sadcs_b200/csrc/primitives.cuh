// primitives.cuh - device-wide scans and stable LSD radix passes, written for sm_100a.
//
// Scan: reduce-then-scan over tiles of 4096 u32 (256 threads x 16), recursive on the tile
// aggregates. Loads and stores are striped across the block (coalesced 128-byte lines); the scan
// inside a tile runs through shared memory with warp shuffles.
//
// Radix pass: one stable counting pass on an 8-bit digit. Upsweep counts digits per tile (warp
// ballots aggregate equal digits before a shared-memory add, so skewed digits do not serialise);
// the per-tile counts, digit-major, are scanned into global offsets; downsweep ranks each tile's
// elements stably (warp match on the digit + per-warp counters), stages them by digit in shared
// memory and writes each digit's run contiguously. Elements reach the kernels through a Loader
// (which may filter them out) and leave through a Storer, so the same kernels serve the sample
// sorts and the filtered class passes.
#pragma once

#include <algorithm>
#include <type_traits>

#include "common.cuh"

namespace sadcs {

// ---- scan ------------------------------------------------------------------------------------

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

struct OpSum {
    static __device__ __forceinline__ uint32_t apply(uint32_t a, uint32_t b) { return a + b; }
    static constexpr uint32_t identity = 0;
};
struct OpMax {
    static __device__ __forceinline__ uint32_t apply(uint32_t a, uint32_t b) { return a > b ? a : b; }
    static constexpr uint32_t identity = 0;
};

// Inclusive scan of v across the block; total gets the block aggregate. 256 threads.
template <class Op>
__device__ __forceinline__ uint32_t blockInclusiveScan(uint32_t v, uint32_t* warpTotals, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= static_cast<uint32_t>(d)) v = Op::apply(u, v);
    }
    if (lane == 31) warpTotals[warp] = v;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (blockDim.x >> 5) ? warpTotals[lane] : Op::identity;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= static_cast<uint32_t>(d)) w = Op::apply(u, w);
        }
        if (lane < (blockDim.x >> 5)) warpTotals[lane] = w;
    }
    __syncthreads();
    total = warpTotals[(blockDim.x >> 5) - 1];
    const uint32_t result = warp ? Op::apply(warpTotals[warp - 1], v) : v;
    __syncthreads();
    return result;
}

template <class Op>
__global__ void __launch_bounds__(kScanThreads) scanReduceKernel(const uint32_t* __restrict__ in, uint32_t count,
                                                                 uint32_t* __restrict__ partials) {
    __shared__ uint32_t warpTotals[32];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile;
    uint32_t acc = Op::identity;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint64_t i = base + j * kScanThreads + threadIdx.x;
        if (i < count) acc = Op::apply(acc, in[i]);
    }
    uint32_t total;
    blockInclusiveScan<Op>(acc, warpTotals, total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// Scans each tile with carry = carries[blockIdx.x] (exclusive-scanned aggregates) or the identity.
// The shared tile is padded by one word per 32 so the per-thread runs of 16 avoid bank conflicts.
__device__ __forceinline__ uint32_t scanPad(uint32_t i) { return i + (i >> 5); }

template <class Op, bool kInclusive>
__global__ void __launch_bounds__(kScanThreads) scanDownKernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                               uint32_t count, const uint32_t* __restrict__ carries,
                                                               uint32_t* __restrict__ totalOut) {
    __shared__ uint32_t tile[kScanTile + kScanTile / 32];
    __shared__ uint32_t warpTotals[32];
    __shared__ uint32_t threadInclusive[kScanThreads];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint32_t k = j * kScanThreads + threadIdx.x;
        const uint64_t i = base + k;
        tile[scanPad(k)] = i < count ? in[i] : Op::identity;
    }
    __syncthreads();
    uint32_t local[kScanItems];
    uint32_t acc = Op::identity;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        local[j] = tile[scanPad(threadIdx.x * kScanItems + j)];
        acc = Op::apply(acc, local[j]);
    }
    uint32_t blockTotal;
    const uint32_t inclusive = blockInclusiveScan<Op>(acc, warpTotals, blockTotal);
    const uint32_t carry = carries ? carries[blockIdx.x] : Op::identity;
    threadInclusive[threadIdx.x] = inclusive;
    __syncthreads();
    uint32_t start = threadIdx.x ? Op::apply(carry, threadInclusive[threadIdx.x - 1]) : carry;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint32_t next = Op::apply(start, local[j]);
        tile[scanPad(threadIdx.x * kScanItems + j)] = kInclusive ? next : start;
        start = next;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint32_t k = j * kScanThreads + threadIdx.x;
        const uint64_t i = base + k;
        if (i < count) out[i] = tile[scanPad(k)];
    }
    if (totalOut && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *totalOut = Op::apply(carry, blockTotal);
}

// Words of scratch a scan of count elements needs.
inline size_t scanScratchWords(uint64_t count) {
    size_t words = 0;
    uint64_t c = count;
    while (c > kScanTile) {
        c = (c + kScanTile - 1) / kScanTile;
        words += c + 64;
    }
    return words + 64;
}

// out may equal in. totalOut (device, optional) gets the reduction of all elements.
template <class Op, bool kInclusive>
cudaError_t deviceScan(const uint32_t* in, uint32_t* out, uint32_t count, uint32_t* scratch, uint32_t* totalOut,
                       cudaStream_t stream) {
    if (count == 0) {
        if (totalOut) SADCS_TRY(cudaMemsetAsync(totalOut, 0, sizeof(uint32_t), stream));
        return cudaSuccess;
    }
    const uint32_t blocks = ceilDiv(count, kScanTile);
    if (blocks == 1) {
        SADCS_TRY(launch(scanDownKernel<Op, kInclusive>, 1, kScanThreads, 0, stream, in, out, count, nullptr, totalOut));
        return cudaGetLastError();
    }
    uint32_t* partials = scratch;
    SADCS_TRY(launch(scanReduceKernel<Op>, blocks, kScanThreads, 0, stream, in, count, partials));
    SADCS_TRY((deviceScan<Op, false>(partials, partials, blocks, scratch + blocks + 64, nullptr, stream)));
    SADCS_TRY(launch(scanDownKernel<Op, kInclusive>, blocks, kScanThreads, 0, stream, in, out, count, partials, totalOut));
    return cudaGetLastError();
}

// ---- partition of 64-bit pairs into slices -------------------------------------------------------
//
// The two-level scatters (the class-0 list, the rank writes of large ranking passes) first move
// (index, value) pairs, index in the high word, into the slice of the target array their index
// belongs to: slice k of the pair array is [k << shift, (k + 1) << shift) and receives the pairs
// whose index lies in the target's slice k (at most 2^shift, one per index). A block stages its
// tile of pairs slice by slice in shared memory, reserves each slice's run with one atomic, and
// writes the runs with consecutive threads on consecutive words, so the pair array is written in
// whole sectors rather than by scattered 8-byte stores.
constexpr int kSliceThreads = 256;
constexpr int kSliceItems = 16;
constexpr uint32_t kSliceTile = kSliceThreads * kSliceItems;
constexpr uint32_t kMaxSlices = 256;
constexpr int kSlicesPerLane = kMaxSlices / 32;
static_assert(kMaxSlices <= kSliceThreads, "one thread per slice reserves the runs");
constexpr uint64_t kNoPair = ~uint64_t(0);

struct SliceStage {
    uint32_t count[kMaxSlices];
    uint32_t offset[kMaxSlices];
    uint32_t base[kMaxSlices];
    uint64_t pairs[kSliceTile];
};

// A companion word per pair (writeSliceMajor's second form) goes to the same place of a second
// array, staged after the pairs in the same buffer; the slice of every staged slot is kept for it.
struct SliceCompanion {
    uint8_t slice[kSliceTile];
};

// No companion words.
struct NoCompanion {
    __device__ __forceinline__ uint64_t operator()(uint64_t) const { return 0; }
};

// All threads of the block, each with its kSliceItems pairs (kNoPair where it has none, and for
// any pair whose slice is not below kMaxSlices). fill[k] (zeroed by the caller before the launch)
// counts the pairs placed in slice k; capacity bounds the pair array. With a companion (cs and dstW
// non-null), wordOf(v[j]) is written to dstW at the place v[j] goes to in dst (computed after the
// pairs are out, so that the words are not held in registers meanwhile).
template <class WordOf = NoCompanion>
__device__ __forceinline__ void writeSliceMajor(SliceStage& st, const uint64_t (&v)[kSliceItems], uint32_t shift,
                                                uint32_t* __restrict__ fill, uint64_t* __restrict__ dst,
                                                uint64_t capacity, SliceCompanion* cs = nullptr,
                                                WordOf wordOf = WordOf(), uint64_t* __restrict__ dstW = nullptr) {
    for (uint32_t i = threadIdx.x; i < kMaxSlices; i += kSliceThreads) st.count[i] = 0;
    __syncthreads();
    uint32_t local[kSliceItems];
#pragma unroll
    for (int j = 0; j < kSliceItems; j++) {
        local[j] = v[j] == kNoPair ? 0 : atomicAdd(&st.count[static_cast<uint32_t>(v[j] >> 32) >> shift], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // exclusive scan of the counts, kSlicesPerLane slices per lane
        const uint32_t lane = threadIdx.x;
        uint32_t c[kSlicesPerLane], sum = 0;
#pragma unroll
        for (int q = 0; q < kSlicesPerLane; q++) {
            c[q] = st.count[kSlicesPerLane * lane + q];
            sum += c[q];
        }
        uint32_t inclusive = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t up = __shfl_up_sync(0xffffffffu, inclusive, d);
            if (lane >= static_cast<uint32_t>(d)) inclusive += up;
        }
        uint32_t at = inclusive - sum;
#pragma unroll
        for (int q = 0; q < kSlicesPerLane; q++) {
            st.offset[kSlicesPerLane * lane + q] = at;
            at += c[q];
        }
    }
    if (threadIdx.x < kMaxSlices && st.count[threadIdx.x]) {
        st.base[threadIdx.x] = atomicAdd(fill + threadIdx.x, st.count[threadIdx.x]);
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSliceItems; j++) {
        if (v[j] != kNoPair) st.pairs[st.offset[static_cast<uint32_t>(v[j] >> 32) >> shift] + local[j]] = v[j];
    }
    __syncthreads();
    const uint32_t total = st.offset[kMaxSlices - 1] + st.count[kMaxSlices - 1];
    for (uint32_t i = threadIdx.x; i < total; i += kSliceThreads) {
        const uint64_t pair = st.pairs[i];
        const uint32_t k = static_cast<uint32_t>(pair >> 32) >> shift;
        const uint32_t rel = st.base[k] + (i - st.offset[k]);
        const uint64_t at = (static_cast<uint64_t>(k) << shift) + rel;
        if ((static_cast<uint64_t>(rel) >> shift) == 0 && at < capacity) dst[at] = pair;  // always, by construction
        if (cs) cs->slice[i] = static_cast<uint8_t>(k);
    }
    if (cs) {
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kSliceItems; j++) {
            if (v[j] != kNoPair) st.pairs[st.offset[static_cast<uint32_t>(v[j] >> 32) >> shift] + local[j]] = wordOf(v[j]);
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < total; i += kSliceThreads) {
            const uint32_t k = cs->slice[i];
            const uint32_t rel = st.base[k] + (i - st.offset[k]);
            const uint64_t at = (static_cast<uint64_t>(k) << shift) + rel;
            if ((static_cast<uint64_t>(rel) >> shift) == 0 && at < capacity) dstW[at] = st.pairs[i];
        }
    }
}

// ---- radix pass (onesweep) ------------------------------------------------------------------
//
// One stable counting pass on an 8-bit digit per kernel, reading and writing each element once
// (Adinets & Merrill's onesweep decomposition): a block takes the next tile in arrival order,
// ranks its elements stably (warp match on the digit + per-warp counters), publishes its per-digit
// counts, and looks back over the tiles before it for their running totals (decoupled look-back).
// The global digit offsets come from one histogram pass made beforehand (for all digits of a sort
// at once). Tiles are numbered in the order blocks start, so a tile's predecessors are resident or
// done and the look-back ends; it is still bounded by the SM cycle counter: past the limit a block
// sets the error word and stores nothing. Counts stay below 2^30 (flags in the top 2 bits).

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr uint32_t kSortTile = kSortThreads * kSortItems;
constexpr uint32_t kNoDigit = 0x100;
constexpr uint32_t kStatusAggregate = 1u << 30;
constexpr uint32_t kStatusPrefix = 2u << 30;
constexpr uint32_t kStatusValue = (1u << 30) - 1;
constexpr uint32_t kMaxSortCount = kStatusValue;
// The look-back gives up after this many SM cycles of waiting (2 s at the B200's 1965 MHz, longer at
// lower clocks): far above any real wait. (A kernel parameter, so that a test can make it give up
// quickly on a predecessor that never publishes.) The SM's own cycle counter is monotonic for the thread
// that reads it; a global-timer reading can jump when its two halves are read across a carry.
constexpr long long kLookbackLimitCycles = 4000000000ll;

// Shared memory of radixOnesweep for a key of keyBytes bytes: one staging buffer that holds the
// tile's keys, then its values, then (carry mode 0) its 64-bit carried words; the digit of every
// staged slot, (carry) a tag byte per slot, and the counting tables. The shared memory a block does
// not take is L1.
constexpr size_t radixSharedBytes(size_t keyBytes, bool carry = false, int carryMode = 0) {
    const size_t stage = carry && carryMode == 0 ? 8 : (keyBytes > 4 ? keyBytes : 4);
    return kSortTile * stage + kSortTile * (carry ? 2 : 1) + (kSortWarps * 256 + 256 + 256 + 32) * 4 + 64;
}

// Segments of a pass: element ranges sorted independently, each from its own digit bases, with
// tiles that never span two segments. The one-segment case is the plain sort.
struct OneSegment {
    uint32_t count;
    __device__ __forceinline__ void locate(uint32_t tile, uint32_t& segment, uint32_t& firstTile, uint32_t& begin,
                                           uint32_t& size) const {
        segment = 0;
        firstTile = 0;
        begin = 0;
        size = count;
    }
};

// Segment s holds elements [elementStart[s], elementStart[s + 1]) and tiles
// [tileStart[s], tileStart[s + 1]); its digit bases are row s of the digit-base table.
struct ManySegments {
    const uint32_t* __restrict__ tileStart;     // [segments + 1]
    const uint32_t* __restrict__ elementStart;  // [segments + 1]
    uint32_t segments;
    __device__ __forceinline__ void locate(uint32_t tile, uint32_t& segment, uint32_t& firstTile, uint32_t& begin,
                                           uint32_t& size) const {
        uint32_t lo = 0, hi = segments;  // last s with tileStart[s] <= tile
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(tileStart + mid) <= tile) lo = mid; else hi = mid;
        }
        segment = lo;
        firstTile = __ldg(tileStart + lo);
        begin = __ldg(elementStart + lo);
        size = __ldg(elementStart + lo + 1) - begin;
    }
};

// Loaders give, for (segment, element index in the pass, index within the segment), whether the
// element takes part, its key and digit (load), and later its value (value, called again for the
// same elements only, so that values are not held in registers through ranking and look-back).
// Storers write keys (when kKeys) and values at output positions.
// Tiles resident per SM the register budget is set for: a loader may ask for its own number
// (kTilesPerSm), otherwise SADCS_SORT_TILES (tuning).
#ifndef SADCS_SORT_TILES
#define SADCS_SORT_TILES 3
#endif
template <class Loader, class = void>
struct SortTilesPerSm {
    static constexpr int value = SADCS_SORT_TILES;
};
template <class Loader>
struct SortTilesPerSm<Loader, std::void_t<decltype(Loader::kTilesPerSm)>> {
    static constexpr int value = Loader::kTilesPerSm;
};

// A loader may carry a 64-bit word with every element (kCarry): it gives a tag byte from the key
// (carryTag), staged while the key is in registers, a source word read by the element's index
// (carrySource), and the element's carried word from the two (carryWord); the storer writes it
// (storeCarry). The sources are read after the look-back, all in flight at once. SADCS_CARRY_MODE:
// 1 stores each word from its thread (a warp's stores fall into one run per digit: few digits in
// the carrying passes); 0 stages the words by slot for whole-run stores (tuning). Measured on the
// 3 GiB genome-like text (class phase): mode 1 82.8 ms, mode 0 91.3; the sources read before the
// look-back, with the values, 93.8 (3 tiles per SM: the registers spill at 4); the sources copied
// asynchronously into a slot-ordered shared buffer before the look-back 95.6 (3 tiles per SM: its
// 32 KB); mode 1 with the values also stored from the threads, unstaged, 75.7 against 74.2 (with
// the later class-0 changes).
#ifndef SADCS_CARRY_MODE
#define SADCS_CARRY_MODE 1
#endif
template <class Loader, class = void>
struct LoaderCarries {
    static constexpr bool value = false;
};
template <class Loader>
struct LoaderCarries<Loader, std::void_t<decltype(Loader::kCarry)>> {
    static constexpr bool value = Loader::kCarry;
};

template <class Key, class Loader, class Storer, class Segments = OneSegment>
__global__ void __launch_bounds__(kSortThreads, SortTilesPerSm<Loader>::value) radixOnesweep(Loader ld, Storer st, Segments segs,
                                                                 const uint32_t* __restrict__ digitBase,
                                                                 uint32_t* __restrict__ status,
                                                                 uint32_t* __restrict__ tileCounter,
                                                                 uint32_t* __restrict__ error,
                                                                 long long lookbackLimit) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr bool kCarry = LoaderCarries<Loader>::value;
    constexpr bool kStageCarry = kCarry && SADCS_CARRY_MODE == 0;
    constexpr size_t kStageBytes = kSortTile * (kStageCarry ? 8 : (sizeof(Key) > 4 ? sizeof(Key) : 4));
    Key* sKeys = reinterpret_cast<Key*>(smem);
    uint32_t* sVals = reinterpret_cast<uint32_t*>(smem);  // the same buffer, after the keys are out
    uint64_t* sCarry = reinterpret_cast<uint64_t*>(smem);  // and after the values
    uint8_t* sDig = smem + kStageBytes;
    uint8_t* sTag = sDig + kSortTile;  // carry only
    uint32_t* warpCount = reinterpret_cast<uint32_t*>(sDig + kSortTile * (kCarry ? 2 : 1));
    uint32_t* digitStart = warpCount + kSortWarps * 256;
    uint32_t* digitGlobal = digitStart + 256;
    uint32_t* warpTotals = digitGlobal + 256;
    __shared__ uint32_t sTile;
    __shared__ int sFailed;

    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        sTile = atomicAdd(tileCounter, 1u);
        sFailed = 0;
    }
    for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) warpCount[i] = 0;
    __syncthreads();
    const uint32_t tile = sTile;
    uint32_t segment, firstTile, segBegin, segSize;
    segs.locate(tile, segment, firstTile, segBegin, segSize);
    const uint32_t localTile = tile - firstTile;
    const uint32_t count = segSize;

    const uint64_t warpBase = static_cast<uint64_t>(localTile) * kSortTile + warp * (kSortItems * 32);
    uint32_t* myCount = warpCount + warp * 256;
    const uint32_t lt = (1u << lane) - 1;
    Key keys[kSortItems];
    uint32_t rankDigit[kSortItems];  // (rank within warp << 9) | digit

    // Every load of the thread first (all in flight at once), then the ranking: a warp-synchronous
    // match between two loads would make each load wait for the one before.
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        const uint64_t i = warpBase + j * 32 + lane;
        uint32_t d = kNoDigit;
        if (!(i < count && ld.load(segment, segBegin + static_cast<uint32_t>(i), static_cast<uint32_t>(i), keys[j], d))) {
            d = kNoDigit;
        }
        rankDigit[j] = d;
    }
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        const uint32_t d = rankDigit[j];
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = 0;
        if (d != kNoDigit) before = myCount[d];
        __syncwarp();
        if (d != kNoDigit && (peers & lt) == 0) myCount[d] = before + __popc(peers);
        __syncwarp();
        rankDigit[j] = ((before + __popc(peers & lt)) << 9) | d;
    }
    __syncthreads();

    // Thread d: the tile's count of digit d, and each warp's exclusive prefix within the tile.
    const uint32_t d = threadIdx.x;  // kSortThreads == 256
    uint32_t digitTotal = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
        const uint32_t c = warpCount[w * 256 + d];
        warpCount[w * 256 + d] = digitTotal;
        digitTotal += c;
    }
    // Publish the tile's aggregate as early as possible: successors wait on it.
    volatile uint32_t* vs = status;
    vs[static_cast<size_t>(tile) * 256 + d] = (tile == firstTile ? kStatusPrefix : kStatusAggregate) | digitTotal;
    uint32_t tileTotal;
    const uint32_t inclusive = blockInclusiveScan<OpSum>(digitTotal, warpTotals, tileTotal);
    digitStart[d] = inclusive - digitTotal;
    __syncthreads();

    // Stage the keys (and every slot's digit) by digit before the look-back, so that the keys leave
    // the registers, and start the value loads, which complete while the look-back waits.
    uint32_t vals[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        const uint32_t dj = rankDigit[j] & 0x1FF;
        vals[j] = 0;
        if (dj != kNoDigit) {
            const uint32_t slot = digitStart[dj] + warpCount[warp * 256 + dj] + (rankDigit[j] >> 9);
            if constexpr (Storer::kKeys) sKeys[slot] = keys[j];
            sDig[slot] = static_cast<uint8_t>(dj);
            if constexpr (kCarry) sTag[slot] = ld.carryTag(keys[j]);
            rankDigit[j] = slot;  // from here on: the item's staged slot
            const uint64_t i = warpBase + j * 32 + lane;
            vals[j] = ld.value(segment, segBegin + static_cast<uint32_t>(i), static_cast<uint32_t>(i));
        } else {
            rankDigit[j] = 0xFFFFFFFFu;
        }
    }

    // Look back for the running total of every earlier tile, kWindow tiles per step (independent
    // loads), backing off while a predecessor has not published.
    uint32_t exclusive = 0;
    if (tile != firstTile) {
        uint32_t t = tile;
        long long waitStart = -1;
        bool failed = false;
        while (t > firstTile) {
            constexpr uint32_t kWindow = 16;
            const uint32_t avail = min(kWindow, t - firstTile);
            uint32_t w[kWindow];
#pragma unroll
            for (uint32_t k = 0; k < kWindow; k++) w[k] = k < avail ? vs[static_cast<size_t>(t - 1 - k) * 256 + d] : 0;
            uint32_t used = 0;
            bool prefix = false, blocked = false;
#pragma unroll
            for (uint32_t k = 0; k < kWindow; k++) {
                if (k >= avail || prefix || blocked) continue;
                if ((w[k] & ~kStatusValue) == 0) {
                    blocked = true;  // not published yet: resume from this tile
                    continue;
                }
                exclusive += w[k] & kStatusValue;
                used++;
                if (w[k] & kStatusPrefix) prefix = true;
            }
            if (prefix) break;
            t -= used;
            if (blocked) {
                const long long now = clock64();
                if (waitStart < 0 || now < waitStart) {
                    waitStart = now;
                } else if (now - waitStart > lookbackLimit) {
                    failed = true;
                    break;
                }
                __nanosleep(64);  // back off: spinning threads take issue slots and L2 bandwidth from other work
            }
        }
        if (failed) {
            sFailed = 1;
        } else {
            vs[static_cast<size_t>(tile) * 256 + d] = kStatusPrefix | (exclusive + digitTotal);
        }
    }
    digitGlobal[d] = digitBase[static_cast<size_t>(segment) * 256 + d] + exclusive;
    __syncthreads();
    if (sFailed) {
        if (threadIdx.x == 0) atomicExch(error, 1u);
        return;
    }

    if constexpr (Storer::kKeys) {
        for (uint32_t i = threadIdx.x; i < tileTotal; i += kSortThreads) {
            const uint32_t dj = sDig[i];
            st.storeKey(segment, digitGlobal[dj] + i - digitStart[dj], sKeys[i]);
        }
        __syncthreads();
    }
    // Values into the same buffer, then out.
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        if (rankDigit[j] != 0xFFFFFFFFu) sVals[rankDigit[j]] = vals[j];
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < tileTotal; i += kSortThreads) {
        const uint32_t dj = sDig[i];
        st.storeValue(segment, digitGlobal[dj] + i - digitStart[dj], sVals[i]);
    }
    if constexpr (kCarry) {
        // The carried words: sources read in element order (every read in flight), then each word
        // staged by slot and written in runs (mode 0) or written from its thread (mode 1).
        uint64_t sources[kSortItems];
#pragma unroll
        for (int j = 0; j < kSortItems; j++) {
            const uint64_t i = warpBase + j * 32 + lane;
            sources[j] = 0;
            if (rankDigit[j] != 0xFFFFFFFFu) {
                sources[j] = ld.carrySource(segment, segBegin + static_cast<uint32_t>(i), static_cast<uint32_t>(i));
            }
        }
        if constexpr (kStageCarry) {
            __syncthreads();  // the values are out of the staging buffer
#pragma unroll
            for (int j = 0; j < kSortItems; j++) {
                const uint32_t slot = rankDigit[j];
                if (slot != 0xFFFFFFFFu) {
                    const uint64_t i = warpBase + j * 32 + lane;
                    sCarry[slot] = ld.carryWord(static_cast<uint32_t>(i), sTag[slot], sources[j]);
                }
            }
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < tileTotal; i += kSortThreads) {
                const uint32_t dj = sDig[i];
                st.storeCarry(segment, digitGlobal[dj] + i - digitStart[dj], sCarry[i]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < kSortItems; j++) {
                const uint32_t slot = rankDigit[j];
                if (slot != 0xFFFFFFFFu) {
                    const uint64_t i = warpBase + j * 32 + lane;
                    const uint32_t dj = sDig[slot];
                    st.storeCarry(segment, digitGlobal[dj] + slot - digitStart[dj],
                                  ld.carryWord(static_cast<uint32_t>(i), sTag[slot], sources[j]));
                }
            }
        }
    }
}

// Digit histograms of a sort, all passes at once: hist[p * 256 + digit] (zeroed by the caller).
// Each thread counts runs of equal digits in registers (one run per digit position) and adds a run
// to the block's shared histogram only when its digit changes: a digit that is constant or nearly
// so (the length tag of the ranking keys, the top byte of a skewed alphabet) costs almost no atomics,
// and a random one one uncontended atomic per key. Warp-uniform trip counts are not needed (no
// warp-synchronous instruction).
// Keys read from an array (radixHistogramFrom's source).
template <class Key>
struct KeyArray {
    const Key* __restrict__ keys;
    __device__ __forceinline__ Key operator()(uint64_t i) const { return keys[i]; }
};

template <class Source>
__global__ void __launch_bounds__(256) radixHistogramFrom(Source source, uint32_t count, int beginBit, int passes,
                                                          uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[8][256];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&h[0][0])[i] = 0;
    __syncthreads();
    uint32_t run[8], digit[8];
#pragma unroll
    for (int p = 0; p < 8; p++) {
        run[p] = 0;
        digit[p] = 0;
    }
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
        const auto k = source(i);
#pragma unroll
        for (int p = 0; p < 8; p++) {
            if (p < passes) {
                const uint32_t dg = static_cast<uint32_t>(k >> (beginBit + 8 * p)) & 0xFF;
                if (dg != digit[p]) {
                    if (run[p]) atomicAdd(&h[p][digit[p]], run[p]);
                    digit[p] = dg;
                    run[p] = 0;
                }
                run[p]++;
            }
        }
    }
#pragma unroll
    for (int p = 0; p < 8; p++) {
        if (p < passes && run[p]) atomicAdd(&h[p][digit[p]], run[p]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
        const uint32_t v = (&h[0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
}

// Exclusive scan of each 256-entry row of hist, in place. One block per row.
__global__ void __launch_bounds__(256) radixDigitBase(uint32_t* __restrict__ hist) {
    __shared__ uint32_t warpTotals[32];
    uint32_t* row = hist + blockIdx.x * 256;
    const uint32_t v = row[threadIdx.x];
    uint32_t total;
    const uint32_t inclusive = blockInclusiveScan<OpSum>(v, warpTotals, total);
    row[threadIdx.x] = inclusive - v;
}

// Keys and values of a sort pass.
// Loaders get (segment, element index in the pass, index within the segment); storers get the
// segment and the output position.
template <class Key>
struct SortLoader {
    const Key* __restrict__ keys;
    const uint32_t* __restrict__ vals;
    int shift;
    __device__ __forceinline__ bool load(uint32_t, uint32_t i, uint32_t, Key& k, uint32_t& d) const {
        k = keys[i];
        d = static_cast<uint32_t>(k >> shift) & 0xFF;
        return true;
    }
    __device__ __forceinline__ uint32_t value(uint32_t, uint32_t i, uint32_t) const { return vals[i]; }
};

template <class Key>
struct SortStorer {
    static constexpr bool kKeys = true;
    Key* __restrict__ keys;
    uint32_t* __restrict__ vals;
    uint32_t limit;
    __device__ __forceinline__ void storeKey(uint32_t, uint32_t pos, Key k) const {
        if (pos < limit) keys[pos] = k;  // always, unless an earlier pass's look-back timed out
    }
    __device__ __forceinline__ void storeValue(uint32_t, uint32_t pos, uint32_t v) const {
        if (pos < limit) vals[pos] = v;
    }
};

// Words of scratch a radix sort (or one filtered pass) over count elements needs:
// 8 x 256 digit bases, the tile status words, the tile counter and the error word.
inline size_t radixScratchWords(uint64_t count) {
    const uint64_t tiles = (count + kSortTile - 1) / kSortTile;
    return 8 * 256 + static_cast<size_t>(tiles) * 256 + 64;
}

// The error word of a RadixScratch built on scratchWords.
inline uint32_t* radixErrorWord(uint32_t* scratchWords) {
    return scratchWords + 8 * 256 + 1;
}

struct RadixScratch {
    uint32_t* digitBase;  // [8][256]
    uint32_t* status;     // [tiles][256]
    uint32_t* control;    // [0] tile counter, [1] error word
    explicit RadixScratch(uint32_t* s, uint64_t count) {
        digitBase = s;
        control = s + 8 * 256;
        status = control + 64;
        (void)count;
    }
    // Control words and status words at given places (no digit-base table).
    static RadixScratch at(uint32_t* control, uint32_t* status) {
        RadixScratch r(control, 0);
        r.digitBase = nullptr;
        r.control = control;
        r.status = status;
        return r;
    }
};

// One pass over `tiles` tiles (ceilDiv(count, kSortTile) for one segment; the segment table's total
// otherwise). count bounds the elements of the pass (all segments together). skipTiles > 0 is for the
// test of the look-back's time-out only: tile numbers start there, so the first block's
// predecessors never publish (their elements are still read: count covers them).
template <class Key, class Loader, class Storer, class Segments = OneSegment>
cudaError_t radixOnesweepPass(const Loader& ld, const Storer& st, const Segments& segs, uint32_t count,
                              uint32_t tiles, const uint32_t* digitBase, const RadixScratch& scratch,
                              cudaStream_t stream, long long lookbackLimit = kLookbackLimitCycles,
                              uint32_t skipTiles = 0) {
    if (count == 0 || tiles == 0) return cudaSuccess;
    // A look-back word holds counts below 2^30: one segment at most that long (callers of the
    // segmented passes keep every segment below it).
    if (std::is_same<Segments, OneSegment>::value && count > kMaxSortCount) return cudaErrorInvalidValue;
    // status words and the tile counter start at zero (at skipTiles); the error word is kept.
    SADCS_TRY(cudaMemsetAsync(scratch.status, 0, static_cast<size_t>(tiles + skipTiles) * 256 * 4, stream));
    SADCS_TRY(cudaMemsetAsync(scratch.control, 0, 4, stream));
    if (skipTiles) SADCS_TRY(cudaMemsetAsync(scratch.control, static_cast<int>(skipTiles), 1, stream));
    constexpr size_t shared = radixSharedBytes(sizeof(Key), LoaderCarries<Loader>::value, SADCS_CARRY_MODE);
    // The opt-in above 48 KiB of dynamic shared memory is per function and per device.
    static std::atomic<uint64_t> configured{0};
    SADCS_TRY(configureOnce(configured, [] {
        return cudaFuncSetAttribute(radixOnesweep<Key, Loader, Storer, Segments>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shared));
    }));
    return launch(radixOnesweep<Key, Loader, Storer, Segments>, tiles, kSortThreads, shared, stream, ld, st, segs,
                  digitBase, scratch.status, scratch.control, scratch.control + 1, lookbackLimit);
}

// Stable LSD sort of (keys, vals) over bits [beginBit, endBit), ping-ponging with the alternates.
// On return keys/vals point at the sorted data (swapped with the alternates if the pass count is odd).
// The error word (scratch control[1]) is left nonzero if a look-back timed out.
template <class Key>
cudaError_t radixSortPairs(Key*& keys, Key*& keysAlt, uint32_t*& vals, uint32_t*& valsAlt, uint32_t count,
                           int beginBit, int endBit, uint32_t* scratchWords, cudaStream_t stream) {
    if (count <= 1 || endBit <= beginBit) return cudaSuccess;
    const RadixScratch scratch(scratchWords, count);
    const int passes = (endBit - beginBit + 7) / 8;
    SADCS_TRY(cudaMemsetAsync(scratch.digitBase, 0, static_cast<size_t>(passes) * 256 * 4, stream));
    const uint32_t histBlocks = std::min<uint32_t>(ceilDiv(count, 256 * 16), 148 * 8);
    SADCS_TRY(launch(radixHistogramFrom<KeyArray<Key>>, histBlocks, 256, 0, stream, KeyArray<Key>{keys}, count,
                     beginBit, passes, scratch.digitBase));
    SADCS_TRY(launch(radixDigitBase, passes, 256, 0, stream, scratch.digitBase));
    for (int p = 0; p < passes; p++) {
        SortLoader<Key> ld{keys, vals, beginBit + 8 * p};
        SortStorer<Key> st{keysAlt, valsAlt, count};
        SADCS_TRY((radixOnesweepPass<Key>(ld, st, OneSegment{count}, count, ceilDiv(count, kSortTile),
                                          scratch.digitBase + p * 256, scratch, stream)));
        Key* k = keys;
        keys = keysAlt;
        keysAlt = k;
        uint32_t* v = vals;
        vals = valsAlt;
        valsAlt = v;
    }
    return cudaSuccess;
}

}  // namespace sadcs
