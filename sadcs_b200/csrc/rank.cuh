// rank.cuh - ranks of the difference-cover sample suffixes (the reference's step 2,
// src/cuda/samplerank.cuh; the result is the same rank array, gpusa.h:62-73).
//
// State: a list of the unresolved sample suffixes (compact sample indices t, position
// (t/7)*32 + D[t%7]) kept in group order, and for every sample its group id in the rank array:
// the number of sample suffixes known to be smaller than every member of its group, which is the
// final rank once the group is a singleton.
//
// One pass: key every listed suffix by a subkey, sort the list stably by (group id, subkey), split
// groups where the subkey changes (a new group's id is its old id plus its offset inside the old
// group, propagated by max-scans), write the ids, and compact away the singletons.
//   character passes: the 7 characters at p + depth in the top 56 bits and min(remaining, 7) in the
//     low byte (0 at or past the end), so a suffix that ends inside the window is separated from
//     every longer one sharing its characters; depth 0, 7, 14, 21, 28 (35 >= 32 characters shared)
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

__global__ void rankInitList(uint32_t* __restrict__ lst, uint32_t m) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) lst[i] = i;
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

// aux1[i] = grp[i] - i at the first element of an old group (>= 0: every listed element before it
// belongs to a smaller group), else 0; its max-scan is grp - (start of the old group) everywhere.
__global__ void rankOldHeads(const uint32_t* __restrict__ grp, uint32_t* __restrict__ aux1, uint32_t u) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= u) return;
    const bool head = i == 0 || grp[i] != grp[i - 1];
    aux1[i] = head ? grp[i] - i : 0;
}

__device__ __forceinline__ bool newHead(const uint32_t* grp, const uint64_t* key, uint32_t i) {
    return i == 0 || grp[i] != grp[i - 1] || key[i] != key[i - 1];
}

// aux2[i] = i + delta at the first element of a new group, else 0; its max-scan is every id.
__global__ void rankNewHeads(const uint32_t* __restrict__ grp, const uint64_t* __restrict__ key,
                             const uint32_t* __restrict__ delta, uint32_t* __restrict__ aux2, uint32_t u) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= u) return;
    aux2[i] = newHead(grp, key, i) ? i + delta[i] : 0;
}

// Writes the ids; flags[i] = 1 for elements still in a group of two or more.
__global__ void rankStore(const uint32_t* __restrict__ grp, const uint64_t* __restrict__ key,
                          const uint32_t* __restrict__ ids, const uint32_t* __restrict__ lst,
                          uint32_t* __restrict__ ranks, uint32_t* __restrict__ flags, uint32_t u, uint32_t m) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= u) return;
    if (lst[i] < m) ranks[lst[i]] = ids[i];
    const bool single = newHead(grp, key, i) && (i + 1 == u || newHead(grp, key, i + 1));
    flags[i] = single ? 0 : 1;
}

__global__ void rankCompact(const uint32_t* __restrict__ lst, const uint32_t* __restrict__ flags,
                            const uint32_t* __restrict__ slots, uint32_t* __restrict__ out, uint32_t u) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < u && flags[i]) out[slots[i]] = lst[i];
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

struct RankStats {
    int characterPasses = 0;
    int doublingRounds = 0;
};

__global__ void rankGatherGroupKeys(const uint32_t* __restrict__ ranks, const uint32_t* __restrict__ lst,
                                    uint64_t* __restrict__ key, uint32_t u, uint32_t m) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < u) key[i] = lst[i] < m ? ranks[lst[i]] : 0;
}

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
    if (texts.count <= 1) {
        SADCS_TRY(launch(rankInitList, blocks256(live), 256, 0, stream, cur, live));
    } else {
        SADCS_TRY(launch(rankInitTexts, blocks256(slots), 256, 0, stream, texts, sampleBase, slots, cur, ranks));
    }
    uint32_t* error = radixErrorWord(b.scratch);
    SADCS_TRY(cudaMemsetAsync(error, 0, sizeof(uint32_t), stream));
    uint32_t u = live;
    uint64_t depth = 0;
    bool first = texts.count <= 1;  // one text: everything starts in one group, no group sort
    const int rankBits = bitWidth(static_cast<uint64_t>(live) + 1);
    const int charBits = static_cast<int>(texts.keyChars * texts.bits + texts.tagBits);
    while (u > 0) {
        const bool doubling = depth >= kV;
        const uint32_t offset = doubling ? static_cast<uint32_t>((depth / kV) * kV) : static_cast<uint32_t>(depth);
        if (depth > static_cast<uint64_t>(longest) + 2 * kV) return cudaErrorUnknown;  // groups share < n chars

        uint32_t* lst = cur;
        uint32_t* lstAlt = alt;
        uint64_t* key = b.key[0];
        uint64_t* keyAlt = b.key[1];
        SADCS_TRY(launch(rankMakeKeys, blocks256(u), 256, 0, stream, text, ranks, texts, lst, key, u, offset,
                         doubling ? 1 : 0));
        const int keyBits = doubling ? rankBits : charBits;
        if (first) {
            // Everything in one group: one global sort by subkey.
            SADCS_TRY(radixSortPairs<uint64_t>(key, keyAlt, lst, lstAlt, u, 0, keyBits, b.scratch, stream));
            SADCS_TRY(launch(rankGatherGroups, blocks256(u), 256, 0, stream, ranks, lst, b.grp, u, slots));
        } else {
            // The list holds whole groups in id order: sort inside each group only.
            SADCS_TRY(launch(rankGatherGroups, blocks256(u), 256, 0, stream, ranks, lst, b.grp, u, slots));
            SegBuffers sb{error - 1, b.aux1, b.aux2, reinterpret_cast<uint32_t*>(keyAlt), b.segScratch,
                          b.counter + 4, b.scanScratch};
            SADCS_TRY(segmentedSort(b.grp, u, key, lst, keyAlt, lstAlt, keyBits, sb, hostCounter + 8, stream));
        }
        SADCS_TRY(launch(rankOldHeads, blocks256(u), 256, 0, stream, b.grp, b.aux1, u));
        SADCS_TRY((deviceScan<OpMax, true>(b.aux1, b.aux1, u, b.scanScratch, nullptr, stream)));
        SADCS_TRY(launch(rankNewHeads, blocks256(u), 256, 0, stream, b.grp, key, b.aux1, b.aux2, u));
        SADCS_TRY((deviceScan<OpMax, true>(b.aux2, b.aux2, u, b.scanScratch, nullptr, stream)));
        SADCS_TRY(launch(rankStore, blocks256(u), 256, 0, stream, b.grp, key, b.aux2, lst, ranks, b.aux1, u, slots));
        SADCS_TRY((deviceScan<OpSum, false>(b.aux1, b.aux2, u, b.scanScratch, b.counter, stream)));
        SADCS_TRY(launch(rankCompact, blocks256(u), 256, 0, stream, lst, b.aux1, b.aux2, lstAlt, u));
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
            depth += texts.keyChars;
        }
        first = false;
    }
    return cudaSuccess;
}

}  // namespace sadcs
