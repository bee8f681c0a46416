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
    uint32_t* scratch;  // sort/scan scratch words
    uint32_t* counter;  // one device word
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

// doubling == 0: character key at depth; otherwise 1 + rank at p + h.
__global__ void rankMakeKeys(const uint8_t* __restrict__ text, const uint32_t* __restrict__ ranks, uint32_t n,
                             const uint32_t* __restrict__ lst, uint64_t* __restrict__ key, uint32_t u,
                             uint32_t offset, int doubling) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= u) return;
    const uint32_t p = samplePosition(lst[i]);
    if (doubling) {
        const uint64_t q = static_cast<uint64_t>(p) + offset;
        key[i] = q < n ? static_cast<uint64_t>(ranks[pack(static_cast<uint32_t>(q))]) + 1 : 0;
    } else {
        const uint64_t q = static_cast<uint64_t>(p) + offset;
        key[i] = q < n ? charKey(text, n, static_cast<uint32_t>(q)) : 0;
    }
}

__global__ void rankGatherGroups(const uint32_t* __restrict__ ranks, const uint32_t* __restrict__ lst,
                                 uint32_t* __restrict__ grp, uint32_t u) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < u) grp[i] = ranks[lst[i]];
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
                          uint32_t* __restrict__ ranks, uint32_t* __restrict__ flags, uint32_t u) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= u) return;
    ranks[lst[i]] = ids[i];
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
                                    uint64_t* __restrict__ key, uint32_t u) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < u) key[i] = ranks[lst[i]];
}

// Ranks the m = sampleSize(n) sample suffixes of text into ranks[0, m) (ranks zeroed by the caller,
// including kRankPad entries past m). hostCounter: page-locked word for the per-pass count.
inline cudaError_t rankSample(const uint8_t* text, uint32_t n, uint32_t* ranks, RankBuffers b, uint32_t* hostCounter,
                              cudaStream_t stream, RankStats& stats) {
    const uint32_t m = static_cast<uint32_t>(sampleSize(n));
    if (m == 0) return cudaSuccess;
    uint32_t* cur = b.lst[0];
    uint32_t* alt = b.lst[1];
    rankInitList<<<blocks256(m), 256, 0, stream>>>(cur, m);
    SADCS_TRY(cudaGetLastError());
    uint32_t u = m;
    uint64_t depth = 0;
    bool first = true;
    const int rankBits = bitWidth(static_cast<uint64_t>(m) + 1);
    while (u > 0) {
        const bool doubling = depth >= kV;
        const uint32_t offset = doubling ? static_cast<uint32_t>((depth / kV) * kV) : static_cast<uint32_t>(depth);
        if (depth > static_cast<uint64_t>(n) + 2 * kV) return cudaErrorUnknown;  // invariant: groups share < n chars

        uint32_t* lst = cur;
        uint32_t* lstAlt = alt;
        uint64_t* key = b.key[0];
        uint64_t* keyAlt = b.key[1];
        rankMakeKeys<<<blocks256(u), 256, 0, stream>>>(text, ranks, n, lst, key, u, offset, doubling ? 1 : 0);
        SADCS_TRY(cudaGetLastError());
        SADCS_TRY(radixSortPairs<uint64_t>(key, keyAlt, lst, lstAlt, u, 0, doubling ? rankBits : 64, b.scratch, stream));
        if (!first) {
            // Stably by the old group id (the list keeps whole groups in id order), then recompute
            // the subkeys in the new order; the subkey buffer is free for the group keys meanwhile.
            rankGatherGroupKeys<<<blocks256(u), 256, 0, stream>>>(ranks, lst, key, u);
            SADCS_TRY(cudaGetLastError());
            SADCS_TRY(radixSortPairs<uint64_t>(key, keyAlt, lst, lstAlt, u, 0, rankBits, b.scratch, stream));
            rankMakeKeys<<<blocks256(u), 256, 0, stream>>>(text, ranks, n, lst, key, u, offset, doubling ? 1 : 0);
            SADCS_TRY(cudaGetLastError());
        }
        rankGatherGroups<<<blocks256(u), 256, 0, stream>>>(ranks, lst, b.grp, u);
        rankOldHeads<<<blocks256(u), 256, 0, stream>>>(b.grp, b.aux1, u);
        SADCS_TRY(cudaGetLastError());
        SADCS_TRY((deviceScan<OpMax, true>(b.aux1, b.aux1, u, b.scratch, nullptr, stream)));
        rankNewHeads<<<blocks256(u), 256, 0, stream>>>(b.grp, key, b.aux1, b.aux2, u);
        SADCS_TRY(cudaGetLastError());
        SADCS_TRY((deviceScan<OpMax, true>(b.aux2, b.aux2, u, b.scratch, nullptr, stream)));
        rankStore<<<blocks256(u), 256, 0, stream>>>(b.grp, key, b.aux2, lst, ranks, b.aux1, u);
        SADCS_TRY(cudaGetLastError());
        SADCS_TRY((deviceScan<OpSum, false>(b.aux1, b.aux2, u, b.scratch, b.counter, stream)));
        rankCompact<<<blocks256(u), 256, 0, stream>>>(lst, b.aux1, b.aux2, lstAlt, u);
        SADCS_TRY(cudaGetLastError());
        SADCS_TRY(cudaMemcpyAsync(hostCounter, b.counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        SADCS_TRY(cudaStreamSynchronize(stream));
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
