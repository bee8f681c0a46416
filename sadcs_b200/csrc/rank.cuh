// rank.cuh - ranks of the difference-cover sample suffixes (the reference's step 2,
// src/cuda/samplerank.cuh; the result is the same rank array, gpusa.h:62-73).
//
// State: a list of the unresolved sample suffixes (compact sample indices t, position
// (t/7)*32 + D[t%7]) kept in group order, with each element's group id beside it: the number of
// sample suffixes known to be smaller than every member of its group, which is the final rank once
// the group is a singleton. The rank array (indexed by t) holds the final ranks of the resolved
// samples and, from the pass before the first doubling round on, the ids of all listed ones.
//
// One pass: key every listed suffix by a subkey, sort the list by (group id, subkey), split groups
// where the subkey changes (a new group's id is its old id plus its offset inside the old group,
// from the last old and new group heads before each element), write the ids, and compact away the
// singletons (three fused kernels per pass, below).
//   character passes: the keyChars codes at p + depth (alphabet.cuh: 29 for DNA, 10 for 6-bit text,
//     7 for bytes) in the top bits and min(remaining, keyChars) in the low tag bits (code 0 at or
//     past the end), so a suffix that ends inside the window is separated from every longer one
//     sharing its characters; depth grows by keyChars until it reaches 32
//   doubling rounds: 1 + the group id at p + h (0 past the end), h the largest multiple of 32 not
//     above the shared depth, so p + h is again a sample position; depth grows by h each round.
// Every subkey of a pass is read before any id of that pass is written.
#pragma once

#include <cstdio>
#include <cstdlib>

#include "alphabet.cuh"
#include "common.cuh"
#include "primitives.cuh"
#include "segsort.cuh"

namespace sadcs {

struct RankBuffers {
    uint32_t* lst[2];   // compact sample indices
    uint64_t* key[2];
    uint32_t* grp;
    uint32_t* aux1;
    uint32_t* aux2;
    uint32_t* scratch;      // radix scratch words (radixScratchWords(m))
    uint32_t* scanScratch;  // scan scratch words (scanScratchWords(m))
    uint32_t* segScratch;   // segmented-sort scratch (segScratchWords(m))
    uint32_t* counter;      // device words: [0] list count, [4..7] segmented sort
    uint32_t keyEntries;    // 64-bit entries of each key buffer (the pair arrays of a bucketed rank write)
};


// SADCS_TRACE=1 in the environment: one line per ranking pass on stderr.
inline bool traceEnabled() {
    static const bool enabled = [] {
        const char* v = std::getenv("SADCS_TRACE");
        return v && v[0] && v[0] != '0';
    }();
    return enabled;
}

// The keyChars characters at q in the top bits and min(remaining, keyChars) in the low tagBits
// bits; characters past the end read as code 0. Key width keyChars * bits + tagBits <= 64.
__device__ __forceinline__ uint64_t charKey(const TextSet& texts, uint32_t end, uint32_t q) {
    const uint32_t c = texts.keyChars, b = texts.bits;
    const uint32_t remaining = end - q;
    uint64_t v = streamBits(texts.packed, static_cast<uint64_t>(q) * b) >> (64 - c * b);
    uint32_t tag = c;
    if (remaining < c) {
        v &= ~((uint64_t(1) << ((c - remaining) * b)) - 1);
        tag = remaining;
    }
    return (v << texts.tagBits) | tag;
}

// The first sort of one text: sample i's key is its first characters (charKey at its own
// position) and its value is i, both made where they are needed: by the digit histograms and by the
// first radix pass's loader. No key or value array is written or read before that pass.
struct FirstKeys {
    TextSet texts;
    __device__ __forceinline__ uint64_t operator()(uint64_t i) const {
        return charKey(texts, texts.oneEnd, samplePosition(static_cast<uint32_t>(i)));
    }
};

struct FirstKeyLoader {
    FirstKeys keys;
    __device__ __forceinline__ bool load(uint32_t, uint32_t i, uint32_t, uint64_t& k, uint32_t& d) const {
        k = keys(i);
        d = static_cast<uint32_t>(k) & 0xFF;
        return true;
    }
    __device__ __forceinline__ uint32_t value(uint32_t, uint32_t i, uint32_t) const { return i; }
};

// Stable LSD sort of samples [0, count) of one text by their first keyChars characters (the
// ranking's first pass): as radixSortPairs, with the first pass's keys and values made by
// FirstKeyLoader. On return keys/vals point at the sorted keys and sample indices.
inline cudaError_t rankFirstSort(const TextSet& texts, uint32_t count, int keyBits, uint64_t*& keys,
                                 uint64_t*& keysAlt, uint32_t*& vals, uint32_t*& valsAlt, uint32_t* scratchWords,
                                 cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    const RadixScratch scratch(scratchWords, count);
    const int passes = (keyBits + 7) / 8;
    SADCS_TRY(cudaMemsetAsync(scratch.digitBase, 0, static_cast<size_t>(passes) * 256 * 4, stream));
    const uint32_t histBlocks = std::min<uint32_t>(ceilDiv(count, 256 * 16), 148 * 8);
    SADCS_TRY(launch(radixHistogramFrom<FirstKeys>, histBlocks, 256, 0, stream, FirstKeys{texts}, count, 0, passes,
                     scratch.digitBase));
    SADCS_TRY(launch(radixDigitBase, passes, 256, 0, stream, scratch.digitBase));
    for (int p = 0; p < passes; p++) {
        const SortStorer<uint64_t> st{keysAlt, valsAlt, count};
        if (p == 0) {
            SADCS_TRY((radixOnesweepPass<uint64_t>(FirstKeyLoader{FirstKeys{texts}}, st, OneSegment{count}, count,
                                                   ceilDiv(count, kSortTile), scratch.digitBase, scratch, stream)));
        } else {
            const SortLoader<uint64_t> ld{keys, vals, 8 * p};
            SADCS_TRY((radixOnesweepPass<uint64_t>(ld, st, OneSegment{count}, count, ceilDiv(count, kSortTile),
                                                   scratch.digitBase + p * 256, scratch, stream)));
        }
        std::swap(keys, keysAlt);
        std::swap(vals, valsAlt);
    }
    return cudaSuccess;
}

// doubling == 0: character key at depth; otherwise 1 + rank at p + h. Keys stop at the end of
// the suffix's own text.
__global__ void rankMakeKeys(const uint8_t* __restrict__ text, const uint32_t* __restrict__ ranks, TextSet texts,
                             const uint32_t* __restrict__ lst, uint64_t* __restrict__ key, uint32_t u,
                             uint32_t offset, int doubling) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= u) return;
    const uint32_t p = samplePosition(lst[i]);
    const uint32_t end = texts.endOf(p);
    const uint64_t q = static_cast<uint64_t>(p) + offset;
    if (doubling) {
        key[i] = q < end ? static_cast<uint64_t>(ranks[pack(static_cast<uint32_t>(q))]) + 1 : 0;
    } else {
        key[i] = q < end ? charKey(texts, end, static_cast<uint32_t>(q)) : 0;
    }
}

// Several texts: the list holds every live sample (a sample position inside its text) in text
// order, and each starts in its text's group: ranks[t] = live samples of the texts before.
__global__ void rankInitTexts(TextSet texts, const uint32_t* __restrict__ sampleBase, uint32_t slots,
                              uint32_t* __restrict__ lst, uint32_t* __restrict__ ranks) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= slots) return;
    const uint32_t p = samplePosition(t);
    const uint32_t j = texts.textOf(p);
    const uint32_t start = texts.startOf(j);
    if (p >= start && p < texts.endOfText(j)) {
        const uint32_t base = sampleBase[j];
        lst[base + (t - (start / kV) * kK)] = t;
        ranks[t] = base;
    } else {
        ranks[t] = 0;
    }
}

__global__ void rankGatherGroups(const uint32_t* __restrict__ ranks, const uint32_t* __restrict__ lst,
                                 uint32_t* __restrict__ grp, uint32_t u, uint32_t m) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < u) grp[i] = lst[i] < m ? ranks[lst[i]] : 0;
}

// ---- the refinement after a pass's sort, fused ------------------------------------------------
//
// With the list sorted by (group, key): an element starts an old group where its group id changes,
// a new group where its group id or its key changes; its new id is its old id plus (index of its
// new group's head - index of its old group's head), because ids are ranks of group heads; it stays
// listed unless its new group is a singleton. Three kernels over tiles of 4096 elements: per-tile
// aggregates (last old head, last new head, kept count), their scan, then each tile again with the
// carries: kept elements compacted into the other list buffer with their ids (the next pass's
// groups, in list order), and ids written to the rank array for the elements whose id is final
// (singletons) or, when writeAll is set (before and during the doubling rounds, whose keys read the
// ranks of other samples), for every element. The rank array is indexed by sample position, so
// each write lands at a random place: the character passes write each sample's rank once.

constexpr int kRefineThreads = 256;
constexpr int kRefineItems = 16;
constexpr uint32_t kRefineTile = kRefineThreads * kRefineItems;

// Bit k of old / next: element base + k starts an old / a new group (next has bit 16 for base + 16);
// keep: element base + k stays listed. Elements at or past u have no bits. g: their group ids.
__device__ __forceinline__ void refineFlags(const uint32_t* __restrict__ grp, const uint64_t* __restrict__ key,
                                            uint32_t u, uint32_t base, uint32_t g[kRefineItems], uint32_t& old,
                                            uint32_t& next, uint32_t& keep) {
    uint32_t prevG = base > 0 && base - 1 < u ? grp[base - 1] : 0xFFFFFFFFu;
    uint64_t prevK = base > 0 && base - 1 < u ? key[base - 1] : 0;
    // The thread's 16 elements by 16-byte loads (base is a multiple of 16 and the buffers are
    // 256-byte aligned), and the one after them.
    uint32_t gv[kRefineItems + 1];
    uint64_t kv[kRefineItems + 1];
    if (base + kRefineItems < u) {
#pragma unroll
        for (int q = 0; q < kRefineItems / 4; q++) {
            const uint4 v = *reinterpret_cast<const uint4*>(grp + base + 4 * q);
            gv[4 * q] = v.x;
            gv[4 * q + 1] = v.y;
            gv[4 * q + 2] = v.z;
            gv[4 * q + 3] = v.w;
        }
#pragma unroll
        for (int q = 0; q < kRefineItems / 2; q++) {
            const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(key + base + 2 * q);
            kv[2 * q] = v.x;
            kv[2 * q + 1] = v.y;
        }
        gv[kRefineItems] = grp[base + kRefineItems];
        kv[kRefineItems] = key[base + kRefineItems];
    } else {
#pragma unroll
        for (int k = 0; k <= kRefineItems; k++) {
            gv[k] = base + k < u ? grp[base + k] : 0;
            kv[k] = base + k < u ? key[base + k] : 0;
        }
    }
    old = 0;
    next = 0;
#pragma unroll
    for (int k = 0; k <= kRefineItems; k++) {
        const uint32_t e = base + k;
        if (e >= u) break;
        const uint32_t ge = gv[k];
        const uint64_t ke = kv[k];
        const bool startOld = e == 0 || ge != prevG;
        if (k < kRefineItems) {
            g[k] = ge;
            if (startOld) old |= 1u << k;
        }
        if (startOld || ke != prevK) next |= 1u << k;
        prevG = ge;
        prevK = ke;
    }
    keep = 0;
#pragma unroll
    for (int k = 0; k < kRefineItems; k++) {
        const uint32_t e = base + k;
        if (e >= u) break;
        const bool single = ((next >> k) & 1) && (e + 1 == u || ((next >> (k + 1)) & 1));
        if (!single) keep |= 1u << k;
    }
}

// agg[tile], agg[tiles + tile], agg[2 * tiles + tile] = last old head, last new head, kept count.
__global__ void __launch_bounds__(kRefineThreads) rankRefineReduce(const uint32_t* __restrict__ grp,
                                                                   const uint64_t* __restrict__ key, uint32_t u,
                                                                   uint32_t tiles, uint32_t* __restrict__ agg) {
    __shared__ uint32_t warpOld[kRefineThreads / 32], warpNew[kRefineThreads / 32], warpKept[kRefineThreads / 32];
    const uint32_t base = blockIdx.x * kRefineTile + threadIdx.x * kRefineItems;
    uint32_t g[kRefineItems], old, next, keep;
    refineFlags(grp, key, u, base, g, old, next, keep);
    const uint32_t mine = next & 0xFFFFu;
    uint32_t lastOld = old ? base + 31 - __clz(old) : 0;
    uint32_t lastNew = mine ? base + 31 - __clz(mine) : 0;
    uint32_t kept = __popc(keep);
    lastOld = __reduce_max_sync(0xffffffffu, lastOld);
    lastNew = __reduce_max_sync(0xffffffffu, lastNew);
    kept = __reduce_add_sync(0xffffffffu, kept);
    const uint32_t warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        warpOld[warp] = lastOld;
        warpNew[warp] = lastNew;
        warpKept[warp] = kept;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t o = 0, w = 0, c = 0;
        for (int i = 0; i < kRefineThreads / 32; i++) {
            o = max(o, warpOld[i]);
            w = max(w, warpNew[i]);
            c += warpKept[i];
        }
        agg[blockIdx.x] = o;
        agg[tiles + blockIdx.x] = w;
        agg[2 * tiles + blockIdx.x] = c;
    }
}

// The aggregates become exclusive prefixes (max, max, sum) over the tiles; total = all kept.
__global__ void __launch_bounds__(256) rankRefineScan(uint32_t* __restrict__ agg, uint32_t tiles,
                                                      uint32_t* __restrict__ total) {
    __shared__ uint32_t warpTotals[32];
    uint32_t carryOld = 0, carryNew = 0, carryKept = 0;
    for (uint32_t base = 0; base < tiles; base += blockDim.x) {
        const uint32_t t = base + threadIdx.x;
        const uint32_t o = t < tiles ? agg[t] : 0;
        const uint32_t w = t < tiles ? agg[tiles + t] : 0;
        const uint32_t c = t < tiles ? agg[2 * tiles + t] : 0;
        uint32_t chunkOld, chunkNew, chunkKept;
        const uint32_t io = blockInclusiveScan<OpMax>(o, warpTotals, chunkOld);
        const uint32_t iw = blockInclusiveScan<OpMax>(w, warpTotals, chunkNew);
        const uint32_t ic = blockInclusiveScan<OpSum>(c, warpTotals, chunkKept);
        // exclusive prefixes: the inclusive one of the thread before (a shuffle within the warp, the
        // warp before through a second scan would cost more than recomputing from inclusive - own)
        if (t < tiles) {
            agg[2 * tiles + t] = carryKept + ic - c;
        }
        __syncthreads();
        // max is not invertible: publish inclusive values, read the neighbour's
        __shared__ uint32_t incOld[256], incNew[256];
        incOld[threadIdx.x] = io;
        incNew[threadIdx.x] = iw;
        __syncthreads();
        if (t < tiles) {
            agg[t] = max(carryOld, threadIdx.x ? incOld[threadIdx.x - 1] : 0u);
            agg[tiles + t] = max(carryNew, threadIdx.x ? incNew[threadIdx.x - 1] : 0u);
        }
        carryOld = max(carryOld, chunkOld);
        carryNew = max(carryNew, chunkNew);
        carryKept += chunkKept;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carryKept;
}

// Each tile again with its carries: ids into the rank array, kept elements compacted into out.
__global__ void __launch_bounds__(kRefineThreads) rankRefineApply(const uint32_t* __restrict__ grp,
                                                                  const uint64_t* __restrict__ key,
                                                                  const uint32_t* __restrict__ lst, uint32_t u,
                                                                  uint32_t slots, uint32_t tiles,
                                                                  const uint32_t* __restrict__ agg,
                                                                  uint32_t* __restrict__ ranks,
                                                                  uint32_t* __restrict__ out,
                                                                  uint32_t* __restrict__ grpOut, uint32_t writeAll,
                                                                  uint64_t* __restrict__ pairs) {
    __shared__ uint32_t warpTotals[32];
    __shared__ uint32_t incOld[kRefineThreads], incNew[kRefineThreads];
    const uint32_t base = blockIdx.x * kRefineTile + threadIdx.x * kRefineItems;
    uint32_t g[kRefineItems], old, next, keep;
    refineFlags(grp, key, u, base, g, old, next, keep);
    const uint32_t mine = next & 0xFFFFu;
    const uint32_t lastOld = old ? base + 31 - __clz(old) : 0;
    const uint32_t lastNew = mine ? base + 31 - __clz(mine) : 0;
    const uint32_t kept = __popc(keep);
    uint32_t totalOld, totalNew, totalKept;
    const uint32_t io = blockInclusiveScan<OpMax>(lastOld, warpTotals, totalOld);
    const uint32_t iw = blockInclusiveScan<OpMax>(lastNew, warpTotals, totalNew);
    const uint32_t ic = blockInclusiveScan<OpSum>(kept, warpTotals, totalKept);
    incOld[threadIdx.x] = io;
    incNew[threadIdx.x] = iw;
    __syncthreads();
    uint32_t runOld = max(agg[blockIdx.x], threadIdx.x ? incOld[threadIdx.x - 1] : 0u);
    uint32_t runNew = max(agg[tiles + blockIdx.x], threadIdx.x ? incNew[threadIdx.x - 1] : 0u);
    uint32_t at = agg[2 * tiles + blockIdx.x] + ic - kept;
    uint32_t items[kRefineItems];
    if (base + kRefineItems <= u) {
#pragma unroll
        for (int q = 0; q < kRefineItems / 4; q++) {
            const uint4 v = *reinterpret_cast<const uint4*>(lst + base + 4 * q);
            items[4 * q] = v.x;
            items[4 * q + 1] = v.y;
            items[4 * q + 2] = v.z;
            items[4 * q + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kRefineItems; k++) items[k] = base + k < u ? lst[base + k] : 0;
    }
#pragma unroll
    for (int k = 0; k < kRefineItems; k++) {
        const uint32_t e = base + k;
        if (e >= u) break;
        if ((old >> k) & 1) runOld = e;
        if ((next >> k) & 1) runNew = e;
        const uint32_t item = items[k];
        const uint32_t id = g[k] + (runNew - runOld);
        const bool kept = (keep >> k) & 1;
        if (!kept || writeAll) {
            if (pairs) {
                // the pass's rank writes in list order: every element's, or the singletons' (an
                // element's place among them is its index less the kept elements before it)
                pairs[writeAll ? e : e - at] = item < slots ? (static_cast<uint64_t>(item) << 32) | id : ~uint64_t(0);
            } else if (item < slots) {
                ranks[item] = id;
            }
        }
        if (kept) {
            grpOut[at] = id;
            out[at++] = item;
        }
    }
}

// ---- the rank writes of a large pass, in two steps --------------------------------------------
//
// The rank array is indexed by sample, so a pass's writes land at random places of it (each a
// DRAM read and write of a sector once the array exceeds L2). A large pass instead writes its
// (sample, rank) pairs in list order (rankRefineApply), rankPartitionPairs moves them into the
// slice of the rank array they belong to (slice k: samples [k << shift, (k + 1) << shift); a pass
// writes each sample at most once, so slice k of the pair array has room for all of its pairs),
// and rankScatterPairs writes the slices one after another, each within an L2-sized part of the
// rank array.
#ifndef SADCS_RANK_SLICE_SHIFT
#define SADCS_RANK_SLICE_SHIFT 22  // 4M samples = 16 MB of the rank array per slice (tuning: 0.6 ms less ranking than 8M at 3 GiB)
#endif
constexpr uint32_t kRankSliceShift = SADCS_RANK_SLICE_SHIFT;
constexpr uint32_t kMaxRankSlices = kMaxSlices;
constexpr int kPairThreads = 256;
constexpr int kPairItems = 8;
constexpr uint32_t kPairTile = kPairThreads * kPairItems;  // divides 2^kRankSliceShift
// Passes writing fewer ranks than this write them directly.
constexpr uint32_t kBucketedRankWrites = 8u << 20;

inline uint32_t rankSliceShift(uint64_t slots) {
    uint32_t shift = kRankSliceShift;
    while ((slots >> shift) >= kMaxRankSlices) shift++;
    return shift;
}

// pairs[0, count) -> dst, slice-major (writeSliceMajor); count = u (every element wrote) or u less
// the kept total. fill[k] (zeroed by the caller) counts the pairs placed in slice k.
__global__ void __launch_bounds__(kSliceThreads) rankPartitionPairs(const uint64_t* __restrict__ pairs, uint32_t u,
                                                                    const uint32_t* __restrict__ keptTotal,
                                                                    uint32_t writeAll, uint32_t shift,
                                                                    uint32_t capacity, uint32_t* __restrict__ fill,
                                                                    uint64_t* __restrict__ dst) {
    __shared__ SliceStage stage;
    const uint32_t total = writeAll ? u : u - min(*keptTotal, u);
    uint64_t v[kSliceItems];
    const uint64_t first = static_cast<uint64_t>(blockIdx.x) * kSliceTile + threadIdx.x;
#pragma unroll
    for (int j = 0; j < kSliceItems; j++) {
        const uint64_t i = first + static_cast<uint64_t>(j) * kSliceThreads;
        v[j] = i < total ? __ldcs(pairs + i) : kNoPair;
        // no pair, or a guarded out-of-range sample
        if ((static_cast<uint32_t>(v[j] >> 32) >> shift) >= kMaxRankSlices) v[j] = kNoPair;
    }
    writeSliceMajor(stage, v, shift, fill, dst, capacity);
}

// Block b writes the pairs of dst[b * kPairTile, (b + 1) * kPairTile) that its slice holds.
__global__ void __launch_bounds__(kPairThreads) rankScatterPairs(const uint64_t* __restrict__ dst, uint32_t shift,
                                                                 uint32_t capacity, uint32_t slots,
                                                                 const uint32_t* __restrict__ fill,
                                                                 uint32_t* __restrict__ ranks) {
    const uint64_t start = static_cast<uint64_t>(blockIdx.x) * kPairTile;
    const uint32_t k = static_cast<uint32_t>(start >> shift);
    const uint64_t end = min((static_cast<uint64_t>(k) << shift) + __ldg(fill + k), static_cast<uint64_t>(capacity));
    for (uint64_t i = start + threadIdx.x; i < min(end, start + kPairTile); i += kPairThreads) {
        const uint64_t v = __ldcs(dst + i);
        const uint32_t t = static_cast<uint32_t>(v >> 32);
        if (t < slots) ranks[t] = static_cast<uint32_t>(v);
    }
}

inline uint32_t blocks256(uint64_t count) {
    return static_cast<uint32_t>((count + 255) / 256);
}

inline int bitWidth(uint64_t x) {
    int b = 0;
    while (x) {
        b++;
        x >>= 1;
    }
    return b;
}

// Characters of the first character pass of one text, a global sort of every sample: the fewest
// whole 8-bit radix passes whose key, tag included, holds enough characters for 2^(chars * bits)
// to exceed 16 times the samples (on a text without repeats, about 1 sample in 16 then shares its
// key with another; a repetitive text leaves its repeats to the later, segmented passes whatever
// the width), and as many characters as those passes hold, at most keyChars. A narrower key is
// taken only if it keeps at least kMinFirstPassChars characters: on the 3 GiB genome-like text
// (2-bit codes) 21 characters in 6 passes took the ranking from 129.6 to 118.1 ms, and 17 in 5 (a
// margin of 16 rather than 64 times the samples) to 89.2 ms against 91.9 with the other changes
// since, while on the 256 MiB natural-language-like text (6-bit codes) 6 characters in 5 passes
// left more suffixes in word-sized repeats for the later passes (17.5 to 19.2 ms).
constexpr uint32_t kMinFirstPassChars = 16;
#ifndef SADCS_FIRST_PASS_MARGIN_BITS
#define SADCS_FIRST_PASS_MARGIN_BITS 4  // 2^(chars * bits) >= 2^4 x samples (tuning)
#endif
inline uint32_t firstPassChars(const TextSet& texts, uint64_t samples) {
    auto width = [](uint32_t x) {
        uint32_t w = 0;
        while (x) {
            w++;
            x >>= 1;
        }
        return w;
    };
    const uint32_t b = texts.bits;
    const uint32_t wantBits = static_cast<uint32_t>(bitWidth(samples)) + SADCS_FIRST_PASS_MARGIN_BITS;
    for (uint32_t passes = 1; passes <= 8; passes++) {
        uint32_t c = std::min<uint32_t>(texts.keyChars, (8 * passes) / b);
        while (c > 0 && c * b + width(c) > 8 * passes) c--;
        if (c == texts.keyChars || c * b >= wantBits) return c >= kMinFirstPassChars ? c : texts.keyChars;
    }
    return texts.keyChars;
}

struct RankStats {
    int characterPasses = 0;
    int doublingRounds = 0;
};

// Ranks the live sample suffixes of the texts. slots = rank entries (sample positions of the whole
// concatenation); live = live samples; sampleBase (device, per text) is used with several texts.
// Ranks of live samples end up in [0, live), text by text; ranks are zeroed by the caller for one
// text (and kRankPad entries past slots always). hostCounter: two page-locked words.
inline cudaError_t rankSample(const uint8_t* text, const TextSet& texts, uint32_t slots, uint32_t live,
                              const uint32_t* sampleBase, uint32_t longest, uint32_t* ranks, RankBuffers b,
                              uint32_t* hostCounter, cudaStream_t stream, RankStats& stats) {
    if (live == 0) return cudaSuccess;
    uint32_t* cur = b.lst[0];
    uint32_t* alt = b.lst[1];
    if (texts.count > 1) {  // one text: the first sort makes the list itself (rankFirstSort)
        SADCS_TRY(launch(rankInitTexts, blocks256(slots), 256, 0, stream, texts, sampleBase, slots, cur, ranks));
    }
    uint32_t* error = radixErrorWord(b.scratch);
    SADCS_TRY(cudaMemsetAsync(error, 0, sizeof(uint32_t), stream));
    uint32_t u = live;
    uint64_t depth = 0;
    bool first = texts.count <= 1;  // one text: everything starts in one group, no group sort
    const int rankBits = bitWidth(static_cast<uint64_t>(live) + 1);
    // The first pass of one text may key fewer characters (fewer radix passes over every sample).
    TextSet firstTexts = texts;
    if (first) {
        firstTexts.keyChars = firstPassChars(texts, live);
        firstTexts.tagBits = static_cast<uint32_t>(bitWidth(firstTexts.keyChars));
    }
    while (u > 0) {
        const bool doubling = depth >= kV;
        const uint32_t offset = doubling ? static_cast<uint32_t>((depth / kV) * kV) : static_cast<uint32_t>(depth);
        if (depth > static_cast<uint64_t>(longest) + 2 * kV) return cudaErrorUnknown;  // groups share < n chars

        uint32_t* lst = cur;
        uint32_t* lstAlt = alt;
        uint64_t* key = b.key[0];
        uint64_t* keyAlt = b.key[1];
        const TextSet& passTexts = first ? firstTexts : texts;
        if (!first) {
            SADCS_TRY(launch(rankMakeKeys, blocks256(u), 256, 0, stream, text, ranks, passTexts, lst, key, u, offset,
                             doubling ? 1 : 0));
        }
        const int keyBits = doubling ? rankBits
                                     : static_cast<int>(passTexts.keyChars * passTexts.bits + passTexts.tagBits);
        if (first) {
            // Everything in one group: one global sort by subkey, its keys made as it goes.
            SADCS_TRY(rankFirstSort(passTexts, u, keyBits, key, keyAlt, lst, lstAlt, b.scratch, stream));
            SADCS_TRY(cudaMemsetAsync(b.grp, 0, static_cast<size_t>(u) * 4, stream));
        } else {
            // The list holds whole groups in id order: sort inside each group only. Group ids come
            // with the list from the pass before; the first pass of several texts reads the texts'
            // first ranks.
            if (depth == 0) {
                SADCS_TRY(launch(rankGatherGroups, blocks256(u), 256, 0, stream, ranks, lst, b.grp, u, slots));
            }
            SegBuffers sb{error - 1, b.aux1, b.aux2, reinterpret_cast<uint32_t*>(keyAlt), b.segScratch,
                          b.counter + 4, b.scanScratch};
            SADCS_TRY(segmentedSort(b.grp, u, key, lst, keyAlt, lstAlt, keyBits, sb, hostCounter + 8, stream));
        }
        // The next pass reads ranks of other samples when it is a doubling round.
        const bool writeAll = doubling || depth + passTexts.keyChars >= kV;
        const uint32_t refineTiles = ceilDiv(u, kRefineTile);
        SADCS_TRY(launch(rankRefineReduce, refineTiles, kRefineThreads, 0, stream, b.grp, key, u, refineTiles, b.aux1));
        SADCS_TRY(launch(rankRefineScan, 1, 256, 0, stream, b.aux1, refineTiles, b.counter));
        // A large pass writes its ranks through pairs in the free key buffer (bucketed, below).
        const bool bucketed = u >= kBucketedRankWrites && slots <= b.keyEntries;
        SADCS_TRY(launch(rankRefineApply, refineTiles, kRefineThreads, 0, stream, b.grp, key, lst, u, slots, refineTiles,
                         b.aux1, ranks, lstAlt, b.aux2, writeAll ? 1u : 0u, bucketed ? keyAlt : nullptr));
        if (bucketed) {
            // the sorted keys are dead now: they become the slice-major pair array
            const uint32_t shift = rankSliceShift(slots);
            uint32_t* fill = b.scratch;  // the first sort's digit bases, dead after it
            SADCS_TRY(cudaMemsetAsync(fill, 0, kMaxRankSlices * sizeof(uint32_t), stream));
            SADCS_TRY(launch(rankPartitionPairs, ceilDiv(u, kSliceTile), kSliceThreads, 0, stream, keyAlt, u,
                             b.counter, writeAll ? 1u : 0u, shift, b.keyEntries, fill, key));
            SADCS_TRY(launch(rankScatterPairs, ceilDiv(slots, kPairTile), kPairThreads, 0, stream, key, shift,
                             b.keyEntries, slots, fill, ranks));
        }
        std::swap(b.grp, b.aux2);  // the kept elements' ids are the next pass's groups
        SADCS_TRY(cudaMemcpyAsync(hostCounter, b.counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        SADCS_TRY(cudaMemcpyAsync(hostCounter + 1, error, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        SADCS_TRY(cudaStreamSynchronize(stream));
        if (hostCounter[1]) return cudaErrorLaunchTimeout;  // a radix look-back gave up
        if (traceEnabled()) {
            fprintf(stderr, "sadcs: ranking %s depth %llu: %u -> %u unresolved\n", doubling ? "doubling" : "characters",
                    static_cast<unsigned long long>(depth), u, *hostCounter);
        }
        u = *hostCounter;
        cur = lstAlt;
        alt = lst;
        if (doubling) {
            stats.doublingRounds++;
            depth += offset;
        } else {
            stats.characterPasses++;
            depth += passTexts.keyChars;
        }
        first = false;
    }
    return cudaSuccess;
}

}  // namespace sadcs
