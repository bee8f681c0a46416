// segsort.cuh - sorting the ranking list by subkey inside each group (segment), in place.
//
// After the first ranking pass the list holds whole groups, each a contiguous segment, and a pass
// only has to order every segment by its subkey (no global sort by (group, subkey) is needed).
// Most segments are small (on genome-like text every segment left after the first pass has at most
// 4 members; on natural-language text 80-95% of the remaining suffixes are in segments of up to a
// few thousand), so:
//   - segments of up to kSegTiny elements are sorted by one thread each in registers;
//   - segments of up to kSegSmall elements are sorted entirely in shared memory: a block takes the
//     segments that start in one kSegChunk-wide range of list positions (at most kSegCap elements)
//     and radix-sorts them by (segment, subkey) with 8-bit digits, the keys travelling in registers
//     and through one shared buffer per pass;
//   - larger segments are sorted by onesweep passes over their own ranges only (segmented tiles,
//     per-segment digit bases), in place between the two list buffers.
// Order among equal subkeys is not kept (nothing downstream depends on it).
#pragma once

#include <utility>

#include "primitives.cuh"

namespace sadcs {

#ifndef SADCS_SEGSORT_BLOCKS
#define SADCS_SEGSORT_BLOCKS 4  // resident blocks per SM the register budget is set for (tuning)
#endif

#ifndef SADCS_SEGSORT_SMALL
#define SADCS_SEGSORT_SMALL 1024  // largest segment sorted in shared memory (tuning; 1024 with 4 blocks per SM: 1.4 ms less ranking at 256 MiB than 2048 with 2)
#endif

constexpr uint32_t kSegSmall = SADCS_SEGSORT_SMALL;  // largest segment sorted in one block
constexpr uint32_t kSegTiny = 8;  // largest segment one thread sorts in registers
constexpr uint32_t kSegChunk = SADCS_SEGSORT_SMALL;  // a block owns the segments starting in such a range
constexpr uint32_t kSegCap = kSegChunk + kSegSmall;  // elements a block can hold
constexpr int kSegThreads = 256;
constexpr int kSegWarps = kSegThreads / 32;
constexpr int kSegItems = kSegCap / kSegThreads;     // 8 at the default
constexpr uint32_t kSegMaxLocal = kSegChunk;         // segments starting in a chunk (each has >= 1 element)

// The segments' big-path tables (host-sized): begin, size and first tile of each big segment.
struct ListSegments {
    const uint32_t* __restrict__ tileStart;  // [segments + 1]
    const uint32_t* __restrict__ begin;      // [segments]
    const uint32_t* __restrict__ size;       // [segments]
    uint32_t segments;
    __device__ __forceinline__ void locate(uint32_t tile, uint32_t& segment, uint32_t& firstTile, uint32_t& b,
                                           uint32_t& n) const {
        uint32_t lo = 0, hi = segments;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(tileStart + mid) <= tile) lo = mid; else hi = mid;
        }
        segment = lo;
        firstTile = __ldg(tileStart + lo);
        b = __ldg(begin + lo);
        n = __ldg(size + lo);
    }
};

// flags[i] = 1 where a segment (run of equal group ids) starts.
__global__ void segMarkHeads(const uint32_t* __restrict__ grp, uint32_t u, uint32_t* __restrict__ flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < u) flags[i] = i == 0 || grp[i] != grp[i - 1];
}

// heads[index[i]] = i for every segment start (index = exclusive scan of the flags); heads[S] = u.
__global__ void segCollectHeads(const uint32_t* __restrict__ grp, const uint32_t* __restrict__ index, uint32_t u,
                                uint32_t segments, uint32_t* __restrict__ heads) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < u && (i == 0 || grp[i] != grp[i - 1])) heads[index[i]] = i;
    if (i == 0) heads[segments] = u;
}

// Per segment k: bigFlag[k] = size > kSegSmall, tiles[k] = its tiles if big (both scanned later).
__global__ void segClassify(const uint32_t* __restrict__ heads, uint32_t segments, uint32_t* __restrict__ bigFlag,
                            uint32_t* __restrict__ tiles) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= segments) return;
    const uint32_t size = heads[k + 1] - heads[k];
    const bool big = size > kSegSmall;
    bigFlag[k] = big;
    tiles[k] = big ? (size + kSortTile - 1) / kSortTile : 0;
}

// The big segments' tables, from the scanned flags and tile counts.
__global__ void segCollectBig(const uint32_t* __restrict__ heads, uint32_t segments,
                              const uint32_t* __restrict__ bigIndex, const uint32_t* __restrict__ tileBase,
                              uint32_t bigCount, uint32_t totalTiles, uint32_t* __restrict__ begin,
                              uint32_t* __restrict__ size, uint32_t* __restrict__ tileStart) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < segments) {
        const uint32_t s = heads[k + 1] - heads[k];
        if (s > kSegSmall) {
            const uint32_t j = bigIndex[k];
            begin[j] = heads[k];
            size[j] = s;
            tileStart[j] = tileBase[k];
        }
    }
    if (k == 0) tileStart[bigCount] = totalTiles;
}

// hist[s * 256 + digit] of digit pass `pass` (bits [8 * pass, 8 * pass + 8)) of every big segment s
// (zeroed by the caller). One histogram per pass, made just before the pass, so that the table is
// big x 256 words, not passes times that. Runs of equal digits are counted in registers and added
// to the shared histogram when the digit changes, as in radixHistogram.
__global__ void __launch_bounds__(256) segHistogram(const uint64_t* __restrict__ keys, ListSegments segs, int pass,
                                                    uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    uint32_t segment, firstTile, begin, size;
    segs.locate(blockIdx.x, segment, firstTile, begin, size);
    const uint32_t local = blockIdx.x - firstTile;
    const uint32_t tileEnd = min((local + 1) * kSortTile, size);
    uint32_t run = 0, digit = 0;
    for (uint32_t k = local * kSortTile + threadIdx.x; k < tileEnd; k += blockDim.x) {
        const uint32_t d = static_cast<uint32_t>(keys[begin + k] >> (8 * pass)) & 0xFF;
        if (d != digit) {
            if (run) atomicAdd(&h[digit], run);
            digit = d;
            run = 0;
        }
        run++;
    }
    if (run) atomicAdd(&h[digit], run);
    __syncthreads();
    if (h[threadIdx.x]) atomicAdd(hist + static_cast<size_t>(segment) * 256 + threadIdx.x, h[threadIdx.x]);
}

// Row s of hist becomes begin[s] + its exclusive prefix. One block per big segment.
__global__ void __launch_bounds__(256) segDigitBase(uint32_t* __restrict__ hist, const uint32_t* __restrict__ begin) {
    __shared__ uint32_t warpTotals[32];
    uint32_t* row = hist + static_cast<size_t>(blockIdx.x) * 256;
    const uint32_t v = row[threadIdx.x];
    uint32_t total;
    const uint32_t inclusive = blockInclusiveScan<OpSum>(v, warpTotals, total);
    row[threadIdx.x] = begin[blockIdx.x] + inclusive - v;
}

// Segments of 2 to kSegTiny elements, one thread each: keys and values into registers, sorted
// by compare-exchange at fixed register indices (an insertion sort unrolled for kSegTiny), written
// back in place. On genome-like text most groups left after the first pass are a repeat and its
// copies (2-4 members), which the block-wide radix sort would take 4 to 8 passes over.
__global__ void __launch_bounds__(256) segSortTiny(const uint32_t* __restrict__ heads, uint32_t segments,
                                                   uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= segments) return;
    const uint32_t begin = heads[k], size = heads[k + 1] - begin;
    if (size < 2 || size > kSegTiny) return;
    uint64_t key[kSegTiny];
    uint32_t val[kSegTiny];
#pragma unroll
    for (uint32_t i = 0; i < kSegTiny; i++) {
        if (i < size) {
            key[i] = keys[begin + i];
            val[i] = vals[begin + i];
        }
    }
#pragma unroll
    for (uint32_t i = 1; i < kSegTiny; i++) {
        if (i < size) {
#pragma unroll
            for (uint32_t j = i; j > 0; j--) {
                if (key[j - 1] > key[j]) {
                    const uint64_t tk = key[j - 1];
                    key[j - 1] = key[j];
                    key[j] = tk;
                    const uint32_t tv = val[j - 1];
                    val[j - 1] = val[j];
                    val[j] = tv;
                }
            }
        }
    }
#pragma unroll
    for (uint32_t i = 0; i < kSegTiny; i++) {
        if (i < size) {
            keys[begin + i] = key[i];
            vals[begin + i] = val[i];
        }
    }
}

// Copies the big segments' ranges from one buffer pair to the other.
__global__ void segCopyBack(ListSegments segs, const uint64_t* __restrict__ kFrom, const uint32_t* __restrict__ vFrom,
                            uint64_t* __restrict__ kTo, uint32_t* __restrict__ vTo) {
    uint32_t segment, firstTile, begin, size;
    segs.locate(blockIdx.x, segment, firstTile, begin, size);
    const uint32_t local = blockIdx.x - firstTile;
    const uint32_t end = min((local + 1) * kSortTile, size);
    for (uint32_t k = local * kSortTile + threadIdx.x; k < end; k += blockDim.x) {
        kTo[begin + k] = kFrom[begin + k];
        vTo[begin + k] = vFrom[begin + k];
    }
}

// The small segments starting in [blockIdx.x * kSegChunk, + kSegChunk): sorted by subkey in
// shared memory and written to out (which may be in). keyBits: significant key bits.
__global__ void __launch_bounds__(kSegThreads, SADCS_SEGSORT_BLOCKS) segSortSmall(const uint32_t* __restrict__ heads, uint32_t segments,
                                                            const uint64_t* keyIn, const uint32_t* valIn,
                                                            uint64_t* keyOut, uint32_t* valOut, int keyBits) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* sKey = reinterpret_cast<uint64_t*>(smem);                 // kSegCap
    uint32_t* sVal = reinterpret_cast<uint32_t*>(sKey + kSegCap);       // kSegCap
    uint16_t* sSeg = reinterpret_cast<uint16_t*>(sVal + kSegCap);       // kSegCap
    uint32_t* segStart = reinterpret_cast<uint32_t*>(sSeg + kSegCap);   // kSegMaxLocal + 1 (global start)
    uint32_t* segLocal = segStart + kSegMaxLocal + 1;                   // kSegMaxLocal + 1 (local start)
    uint32_t* warpCount = segLocal + kSegMaxLocal + 1;                  // kSegWarps * 256
    uint32_t* digitStart = warpCount + kSegWarps * 256;                 // 256
    __shared__ uint32_t warpTotals[32];
    __shared__ uint32_t sFirst, sCount, sTotal;

    if (threadIdx.x == 0) {
        const uint32_t lo = blockIdx.x * kSegChunk, hi = lo + kSegChunk;
        uint32_t a = 0, b = segments;  // first segment starting at or after lo
        while (a < b) {
            const uint32_t mid = (a + b) >> 1;
            if (heads[mid] < lo) a = mid + 1; else b = mid;
        }
        uint32_t c = a, d = segments;  // first segment starting at or after hi
        while (c < d) {
            const uint32_t mid = (c + d) >> 1;
            if (heads[mid] < hi) c = mid + 1; else d = mid;
        }
        sFirst = a;
        sCount = c - a;
    }
    __syncthreads();
    const uint32_t first = sFirst, count = sCount;
    // Local starts of the small segments (big ones get size 0 here).
    uint32_t running = 0;
    for (uint32_t base = 0; base < count; base += kSegThreads) {
        const uint32_t s = base + threadIdx.x;
        uint32_t size = 0;
        if (s < count) {
            const uint32_t start = heads[first + s], end = heads[first + s + 1];
            size = end - start <= kSegSmall && end - start > kSegTiny ? end - start : 0;  // tiny ones: segSortTiny
            segStart[s] = start;
        }
        uint32_t total;
        const uint32_t inclusive = blockInclusiveScan<OpSum>(size, warpTotals, total);
        if (s < count) segLocal[s] = running + inclusive - size;
        running += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        segLocal[count] = running;
        sTotal = running;
    }
    __syncthreads();
    const uint32_t total = sTotal;
    if (total == 0) return;

    // Load: item j of warp w is element w * (kSegItems * 32) + j * 32 + lane, in segment order.
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t key[kSegItems];
    uint32_t val[kSegItems];
    uint32_t seg[kSegItems];
#pragma unroll
    for (int j = 0; j < kSegItems; j++) {
        const uint32_t t = warp * (kSegItems * 32) + j * 32 + lane;
        seg[j] = 0xFFFF;
        if (t < total) {
            uint32_t a = 0, b = count;  // last s with segLocal[s] <= t among the nonempty ones
            while (b - a > 1) {
                const uint32_t mid = (a + b) >> 1;
                if (segLocal[mid] <= t) a = mid; else b = mid;
            }
            while (segLocal[a + 1] <= t) a++;  // skip empty (big) segments sharing the start
            const uint32_t g = segStart[a] + (t - segLocal[a]);
            key[j] = keyIn[g];
            val[j] = valIn[g];
            seg[j] = a;
        }
    }
    int segBits = 0;
    while ((1u << segBits) < count) segBits++;
    const int keyPasses = (keyBits + 7) / 8, segPasses = (segBits + 7) / 8;
    const uint32_t lt = (1u << lane) - 1;
    for (int pass = 0; pass < keyPasses + segPasses; pass++) {
        for (int i = threadIdx.x; i < kSegWarps * 256; i += kSegThreads) warpCount[i] = 0;
        __syncthreads();
        uint32_t* myCount = warpCount + warp * 256;
        uint32_t rankDigit[kSegItems];
#pragma unroll
        for (int j = 0; j < kSegItems; j++) {
            uint32_t d = kNoDigit;
            if (seg[j] != 0xFFFF) {
                d = pass < keyPasses ? static_cast<uint32_t>(key[j] >> (8 * pass)) & 0xFF
                                     : (seg[j] >> (8 * (pass - keyPasses))) & 0xFF;
            }
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            uint32_t before = 0;
            if (d != kNoDigit) before = myCount[d];
            __syncwarp();
            if (d != kNoDigit && (peers & lt) == 0) myCount[d] = before + __popc(peers);
            __syncwarp();
            rankDigit[j] = ((before + __popc(peers & lt)) << 9) | d;
        }
        __syncthreads();
        const uint32_t dd = threadIdx.x;
        uint32_t digitTotal = 0;
#pragma unroll
        for (int w = 0; w < kSegWarps; w++) {
            const uint32_t c = warpCount[w * 256 + dd];
            warpCount[w * 256 + dd] = digitTotal;
            digitTotal += c;
        }
        uint32_t all;
        const uint32_t inclusive = blockInclusiveScan<OpSum>(digitTotal, warpTotals, all);
        digitStart[dd] = inclusive - digitTotal;
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kSegItems; j++) {
            const uint32_t d = rankDigit[j] & 0x1FF;
            if (d != kNoDigit) {
                const uint32_t pos = digitStart[d] + warpCount[warp * 256 + d] + (rankDigit[j] >> 9);
                sKey[pos] = key[j];
                sVal[pos] = val[j];
                sSeg[pos] = static_cast<uint16_t>(seg[j]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kSegItems; j++) {
            const uint32_t t = warp * (kSegItems * 32) + j * 32 + lane;
            if (t < total) {
                key[j] = sKey[t];
                val[j] = sVal[t];
                seg[j] = sSeg[t];
            } else {
                seg[j] = 0xFFFF;
            }
        }
        __syncthreads();
    }
    // Sorted by (segment, key): segment s occupies [segLocal[s], segLocal[s + 1]) again.
#pragma unroll
    for (int j = 0; j < kSegItems; j++) {
        const uint32_t t = warp * (kSegItems * 32) + j * 32 + lane;
        if (t < total) {
            const uint32_t s = seg[j];
            const uint32_t g = segStart[s] + (t - segLocal[s]);
            keyOut[g] = key[j];
            valOut[g] = val[j];
        }
    }
}

constexpr size_t segSortSharedBytes() {
    return kSegCap * (8 + 4 + 2) + 2 * (kSegMaxLocal + 1) * 4 + (kSegWarps * 256 + 256) * 4 + 64;
}

// Scratch words of segmentedSort for a list of u elements (besides the list buffers and aux arrays).
inline size_t segScratchWords(uint64_t u) {
    const uint64_t big = u / (kSegSmall + 1) + 2;
    const uint64_t tiles = u / kSortTile + big + 2;
    return static_cast<size_t>(big * 256 + 3 * (big + 1) + tiles * 256 + 256);
}

struct SegBuffers {
    uint32_t* radixControl;  // [0] tile counter, [1] the error word the caller checks
    uint32_t* flags;    // u words (aux)
    uint32_t* heads;    // u + 1 words (aux)
    uint32_t* perSeg;   // 2 * u words (free key buffer): big flags and tile counts per segment
    uint32_t* scratch;  // segScratchWords(u)
    uint32_t* counter;  // device words [0..3]
    uint32_t* scanScratch;
};

// Sorts the list (keys, vals: u elements in segments of equal grp) by key inside each segment.
// Big segments use the alternates as the other buffer of their passes; the result is left in
// keys/vals (pointers unchanged). hostWords: page-locked words for counts.
inline cudaError_t segmentedSort(const uint32_t* grp, uint32_t u, uint64_t* keys, uint32_t* vals, uint64_t* keysAlt,
                                 uint32_t* valsAlt, int keyBits, SegBuffers b, uint32_t* hostWords,
                                 cudaStream_t stream) {
    if (u <= 1) return cudaSuccess;
    SADCS_TRY(launch(segMarkHeads, ceilDiv(u, 256), 256, 0, stream, grp, u, b.flags));
    SADCS_TRY((deviceScan<OpSum, false>(b.flags, b.flags, u, b.scanScratch, b.counter, stream)));
    SADCS_TRY(cudaMemcpyAsync(hostWords, b.counter, 4, cudaMemcpyDeviceToHost, stream));
    SADCS_TRY(cudaStreamSynchronize(stream));
    const uint32_t segments = hostWords[0];
    SADCS_TRY(launch(segCollectHeads, ceilDiv(u, 256), 256, 0, stream, grp, b.flags, u, segments, b.heads));
    uint32_t* bigFlag = b.perSeg;
    uint32_t* tiles = b.perSeg + u;
    SADCS_TRY(launch(segClassify, ceilDiv(segments, 256), 256, 0, stream, b.heads, segments, bigFlag, tiles));
    SADCS_TRY((deviceScan<OpSum, false>(bigFlag, bigFlag, segments, b.scanScratch, b.counter + 1, stream)));
    SADCS_TRY((deviceScan<OpSum, false>(tiles, tiles, segments, b.scanScratch, b.counter + 2, stream)));
    SADCS_TRY(cudaMemcpyAsync(hostWords + 1, b.counter + 1, 8, cudaMemcpyDeviceToHost, stream));
    SADCS_TRY(cudaStreamSynchronize(stream));
    const uint32_t big = hostWords[1], bigTiles = hostWords[2];

    // Small segments, in place.
    static std::atomic<uint64_t> configured{0};
    SADCS_TRY(configureOnce(configured, [] {
        return cudaFuncSetAttribute(segSortSmall, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(segSortSharedBytes()));
    }));
    SADCS_TRY(launch(segSortTiny, ceilDiv(segments, 256), 256, 0, stream, b.heads, segments, keys, vals));
    SADCS_TRY(launch(segSortSmall, ceilDiv(u, kSegChunk), kSegThreads, segSortSharedBytes(), stream, b.heads,
                     segments, keys, vals, keys, vals, keyBits));
    if (big == 0) return cudaSuccess;

    // Big segments: onesweep passes over their own ranges, ping-ponging with the alternates.
    uint32_t* begin = b.scratch;
    uint32_t* size = begin + big + 1;
    uint32_t* tileStart = size + big + 1;
    uint32_t* hist = tileStart + big + 1;
    const int passes = (keyBits + 7) / 8;
    uint32_t* statusWords = hist + static_cast<size_t>(big) * 256;
    const RadixScratch radix = RadixScratch::at(b.radixControl, statusWords);
    SADCS_TRY(launch(segCollectBig, ceilDiv(segments, 256), 256, 0, stream, b.heads, segments, bigFlag, tiles, big,
                     bigTiles, begin, size, tileStart));
    ListSegments segs{tileStart, begin, size, big};
    uint64_t* kIn = keys;
    uint64_t* kOut = keysAlt;
    uint32_t* vIn = vals;
    uint32_t* vOut = valsAlt;
    for (int p = 0; p < passes; p++) {
        SADCS_TRY(cudaMemsetAsync(hist, 0, static_cast<size_t>(big) * 256 * 4, stream));
        SADCS_TRY(launch(segHistogram, bigTiles, 256, 0, stream, kIn, segs, p, hist));
        SADCS_TRY(launch(segDigitBase, big, 256, 0, stream, hist, begin));
        SortLoader<uint64_t> ld{kIn, vIn, 8 * p};
        SortStorer<uint64_t> st{kOut, vOut, u};
        SADCS_TRY((radixOnesweepPass<uint64_t, SortLoader<uint64_t>, SortStorer<uint64_t>, ListSegments>(
            ld, st, segs, u, bigTiles, hist, radix, stream)));
        std::swap(kIn, kOut);
        std::swap(vIn, vOut);
    }
    if (kIn != keys) {
        // An odd number of passes left the big segments in the alternates: copy their ranges back.
        SADCS_TRY(launch(segCopyBack, bigTiles, 256, 0, stream, segs, kIn, vIn, keys, vals));
    }
    return cudaSuccess;
}

}  // namespace sadcs
