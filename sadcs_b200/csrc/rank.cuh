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

#include "common.cuh"
#include "primitives.cuh"

namespace sadcs {

struct RankBuffers {
    uint32_t* lst[2];   // compact sample indices
    uint64_t* key[2];
    uint32_t* grp;
    uint32_t* aux1;
    uint32_t* aux2;
    uint32_t* scratch;      // radix scratch words (radixScratchWords(m))
    uint32_t* scanScratch;  // scan scratch words (scanScratchWords(m))
    uint32_t* counter;      // one device word
};

constexpr uint32_t kCharsPerPass = 7;

__device__ __forceinline__ uint64_t charKey(const uint8_t* __restrict__ text, uint32_t n, uint32_t q) {
    if (q >= n) return 0;
    const uint32_t remaining = n - q;
    const uint64_t chars = load8(text, q) & ~uint64_t(0xFF);
    if (remaining >= kCharsPerPass) return chars | kCharsPerPass;
    return (chars & (~uint64_t(0) << (64 - 8 * remaining))) | remaining;
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
        key[i] = q < end ? charKey(text, end, static_cast<uint32_t>(q)) : 0;
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
        SADCS_TRY(radixSortPairs<uint64_t>(key, keyAlt, lst, lstAlt, u, 0, doubling ? rankBits : 64, b.scratch, stream));
        if (!first) {
            // Stably by the old group id (the list keeps whole groups in id order), then recompute
            // the subkeys in the new order; the subkey buffer is free for the group keys meanwhile.
            SADCS_TRY(launch(rankGatherGroupKeys, blocks256(u), 256, 0, stream, ranks, lst, key, u, slots));
            SADCS_TRY(radixSortPairs<uint64_t>(key, keyAlt, lst, lstAlt, u, 0, rankBits, b.scratch, stream));
            SADCS_TRY(launch(rankMakeKeys, blocks256(u), 256, 0, stream, text, ranks, texts, lst, key, u, offset,
                             doubling ? 1 : 0));
        }
        SADCS_TRY(launch(rankGatherGroups, blocks256(u), 256, 0, stream, ranks, lst, b.grp, u, slots));
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
        u = *hostCounter;
        cur = lstAlt;
        alt = lst;
        if (doubling) {
            stats.doublingRounds++;
            depth += offset;
        } else {
            stats.characterPasses++;
            depth += kCharsPerPass;
        }
        first = false;
    }
    return cudaSuccess;
}

}  // namespace sadcs
