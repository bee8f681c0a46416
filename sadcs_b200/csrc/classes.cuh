// classes.cuh - the sorted list of every class (the reference's step 3, src/cuda/classsort.cuh:1-20).
//
// Class d holds the positions whose next sample position is d characters ahead; class 0 is the
// sample, ordered by its ranks. For i in class d >= 1, i + 1 is in class d - 1, so suffix i is
// ordered by (T[i], suffix i + 1): class d is class d - 1 walked in order with the text's end (the
// empty suffix, smallest) in front, keeping the predecessors that fall in class d, stably sorted
// by their first character. The text's last position comes from the prepended end and so leads its
// character bucket, as the one-character suffix must.
//
// Several texts: each global class list is the texts' class lists one after another (text order),
// and each text is a segment of the pass: a segmented onesweep pass sorts all texts at once, every
// text from its own digit bases. The walk, the filter and the stable counting sort are that one
// pass, keyed by the character each element carries (ClassLoader); the digit bases come from one
// streaming read of the text.
#pragma once

#include <algorithm>

#include "alphabet.cuh"
#include "common.cuh"
#include "primitives.cuh"

namespace sadcs {

// Device tables of the class phase for J texts (one text: J = 1), all in one block of words:
//   rowBase[kClasses][J]                 first slot of (class, text) in the global lists
//   elementStart[kClasses][J + 1]        segments of pass d: text j's class d - 1 plus its end
//   tileStart[kClasses][J + 1]           the tiles of those segments
struct ClassTables {
    uint32_t texts = 0;
    uint32_t* rowBase = nullptr;
    uint32_t* elementStart = nullptr;
    uint32_t* tileStart = nullptr;
    static size_t words(uint32_t texts) { return static_cast<size_t>(kClasses) * (3 * texts + 2) + 16; }
    void carve(uint32_t* base, uint32_t j) {
        texts = j;
        rowBase = base;
        elementStart = rowBase + static_cast<size_t>(kClasses) * j;
        tileStart = elementStart + static_cast<size_t>(kClasses) * (j + 1);
    }
};

// Host side of the class phase: sizes, offsets and tile counts from the text lengths.
struct ClassPlan {
    uint32_t start[kClasses + 1] = {};  // global class list offsets
    uint32_t largest = 0;               // largest class over all texts together
    uint32_t tiles[kClasses] = {};      // tiles of pass d (segmented)
    uint32_t inputs[kClasses] = {};     // elements of pass d (class d - 1 plus one end per text)
};

// Fills the host copy of the tables (a host block laid out like ClassTables) and the plan.
inline void planClasses(const uint64_t* lengths, uint32_t texts, uint32_t* tables, ClassPlan& plan) {
    ClassTables t;
    t.carve(tables, texts);
    uint64_t total[kClasses] = {};
    for (uint32_t j = 0; j < texts; j++) {
        for (int d = 0; d < kClasses; d++) total[d] += classSize(lengths[j], d);
    }
    plan.start[0] = 0;
    for (int d = 0; d < kClasses; d++) {
        plan.start[d + 1] = plan.start[d] + static_cast<uint32_t>(total[d]);
        plan.largest = std::max<uint32_t>(plan.largest, static_cast<uint32_t>(total[d]));
    }
    for (int d = 0; d < kClasses; d++) {
        uint64_t offset = plan.start[d];
        uint64_t elements = 0, tiles = 0;
        for (uint32_t j = 0; j < texts; j++) {
            t.rowBase[static_cast<size_t>(d) * texts + j] = static_cast<uint32_t>(offset);
            offset += classSize(lengths[j], d);
            const uint64_t input = d >= 1 ? classSize(lengths[j], d - 1) + 1 : 0;
            t.elementStart[static_cast<size_t>(d) * (texts + 1) + j] = static_cast<uint32_t>(elements);
            t.tileStart[static_cast<size_t>(d) * (texts + 1) + j] = static_cast<uint32_t>(tiles);
            elements += input;
            tiles += (input + kSortTile - 1) / kSortTile;
        }
        t.elementStart[static_cast<size_t>(d) * (texts + 1) + texts] = static_cast<uint32_t>(elements);
        t.tileStart[static_cast<size_t>(d) * (texts + 1) + texts] = static_cast<uint32_t>(tiles);
        plan.tiles[d] = static_cast<uint32_t>(tiles);
        plan.inputs[d] = static_cast<uint32_t>(elements);
    }
}

inline size_t classScratchWords(uint64_t totalLength, uint32_t texts) {
    // per-(class, text) histograms, then a radix scratch with room for every segmented tile
    const uint64_t tiles = totalLength / kSortTile + static_cast<uint64_t>(texts) * 2 + 2;
    return static_cast<size_t>(kClasses) * texts * 256 + 8 * 256 + 64 + static_cast<size_t>(tiles) * 256 + 64;
}

// 64-bit words of one chain buffer: the largest of classes 1 to kClasses - 2 (the last class stores
// no chains), bounded here by every class's own bound.
inline size_t classChainWords(uint64_t live) {
    return static_cast<size_t>(live) + 64;
}

inline uint32_t* classRadixScratch(uint32_t* scratch, uint32_t texts) {
    return scratch + static_cast<size_t>(kClasses) * texts * 256;
}

inline uint32_t* classErrorWord(uint32_t* scratch, uint32_t texts) {
    return radixErrorWord(classRadixScratch(scratch, texts));
}

// The carried word of position x (one text): 64 bits of the code stream from character x - 1 (code 0
// before position 0), so the character before x and at least the first 31 characters from x for
// codes of at most 2 bits. The class passes hand it on (carried(x - 1) is the code of T[x - 2] on
// top of carried(x) shifted down by one character), so that the final merge reads it in list order
// instead of gathering it from the text.
__device__ __forceinline__ uint64_t carriedWord(const uint64_t* __restrict__ packed, uint32_t x, uint32_t bits) {
    return x ? streamBits(packed, static_cast<uint64_t>(x - 1) * bits) : streamBits(packed, 0) >> bits;
}

// Class 0: the live sample positions in rank order, list[rank] = position. The ranks of the live
// samples are a permutation of [0, live), so the slice of ranks [k << shift, (k + 1) << shift)
// holds exactly 2^shift samples (the last slice the rest). Two steps, so that no write lands at a
// random place of the whole list: classPartitionSample streams the rank array once and writes each
// live sample's (rank, position) pair into its rank's slice of a pair array (in any order inside
// the slice; one run per slice and block); classScatterPairs then walks the pairs slice by slice,
// and each slice's writes stay within the list's L2-sized slice.
constexpr uint32_t kSampleSliceShift = 23;  // 8M ranks = 32 MB of the list per slice
#ifndef SADCS_CARRY_SLICE_SHIFT
#define SADCS_CARRY_SLICE_SHIFT 22  // with carried words: 4M ranks = 16 + 32 MB per slice (tuning)
#endif
constexpr uint32_t kCarrySampleSliceShift = SADCS_CARRY_SLICE_SHIFT;
constexpr uint32_t kMaxSampleSlices = kMaxSlices;

// The slice width (as a shift) for `live` samples: at least 8M ranks (4M with carried words), at
// most kMaxSampleSlices slices.
inline uint32_t sampleSliceShift(uint64_t live, bool carry) {
    uint32_t shift = carry ? kCarrySampleSliceShift : kSampleSliceShift;
    while ((live >> shift) >= kMaxSampleSlices) shift++;
    return shift;
}

// fill[k] (zeroed by the caller) counts the pairs placed in slice k so far. kCarry: words[x] = the
// carried word of the sample in pairs[x] (a block's samples are consecutive in the text, so their
// words are one short stretch of the code stream).
template <bool kCarry>
__global__ void __launch_bounds__(kSliceThreads) classPartitionSample(const uint32_t* __restrict__ ranks,
                                                                     uint32_t slots, uint32_t live, uint32_t shift,
                                                                     TextSet texts, uint32_t* __restrict__ fill,
                                                                     uint64_t* __restrict__ pairs,
                                                                     uint64_t* __restrict__ words) {
    __shared__ SliceStage stage;
    uint64_t v[kSliceItems];
    const uint64_t first = static_cast<uint64_t>(blockIdx.x) * kSliceTile + threadIdx.x;
#pragma unroll
    for (int j = 0; j < kSliceItems; j++) {
        const uint64_t t = first + static_cast<uint64_t>(j) * kSliceThreads;
        v[j] = kNoPair;
        if (t < slots) {
            const uint32_t rank = __ldcs(ranks + t);  // streamed: read once
            const uint32_t q = samplePosition(static_cast<uint32_t>(t));
            // a live sample (not past the end or between texts)
            if (q < texts.endOf(q) && rank < live) v[j] = (static_cast<uint64_t>(rank) << 32) | q;
        }
    }
    if constexpr (kCarry) {
        __shared__ SliceCompanion companion;
        const uint64_t* packed = texts.packed;
        const uint32_t bits = texts.bits;
        writeSliceMajor(stage, v, shift, fill, pairs, live, &companion,
                        [packed, bits](uint64_t pair) { return carriedWord(packed, static_cast<uint32_t>(pair), bits); },
                        words);
    } else {
        writeSliceMajor(stage, v, shift, fill, pairs, live);
    }
}

// list[rank] = position of every pair; with carried (one text), also carried[rank] = words[i], the
// pair's carried word.
__global__ void classScatterPairs(const uint64_t* __restrict__ pairs, uint32_t live, uint32_t* __restrict__ list,
                                  uint64_t* __restrict__ carried, const uint64_t* __restrict__ words) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= live) return;
    const uint64_t v = __ldcs(pairs + i);
    const uint32_t r = static_cast<uint32_t>(v >> 32);
    if (r < live) {
        list[r] = static_cast<uint32_t>(v);
        if (carried) carried[r] = __ldcs(words + i);
    }
}

// The class passes consume one character of an element's chain each: pass d keys class d - 1's
// element p by the code of T[p - 1] and hands p - 1 the rest. Six passes follow class 0, so a
// chain holds the codes of the kChainChars characters before p, b bits each: bits [i*b, (i+1)*b)
// hold the code of T[p - 1 - i] (0 before position 0). The chain travels as the sort key in the
// narrowest word that holds 6b bits: 16 bits for 2-bit codes (DNA), 32 for up to 5, 64 otherwise.
// Passes that carry words (one text, codes of at most 2 bits) keep one character more, T[p - 2] of
// the last pass's elements, the character before that pass's outputs.
constexpr int kChainChars = kClasses - 1;
constexpr int kCarryChainChars = kClasses;

template <class Chain, int kChars = kChainChars>
__device__ __forceinline__ Chain codesBefore(const TextSet& texts, uint32_t p) {
    const uint32_t b = texts.bits;
    const uint32_t first = p >= kChars ? p - kChars : 0;
    const uint64_t window = streamBits(texts.packed, static_cast<uint64_t>(first) * b);  // >= 8 codes
    const uint64_t mask = (uint64_t(1) << b) - 1;
    uint64_t chain = 0;
#pragma unroll
    for (int i = 0; i < kChars; i++) {
        const int at = static_cast<int>(p - first) - 1 - i;  // T[p - 1 - i] is character `at` of the window
        if (at >= 0) chain |= ((window >> (64 - (at + 1) * b)) & mask) << (b * i);
    }
    return static_cast<Chain>(chain);
}

// Element k of text j's class d - 1 with the text's end prepended; keeps p - 1 if it is in class d
// and in the text, keyed by the code of T[p - 1]. The sort key is the element's chain (above).
// Pass 1 reads the chains of the sample positions from the code stream (one window each); later
// passes read the chains the pass before stored in list order, so only pass 1 reads the text at
// random positions. A text's end reads its own chain every pass.
#ifndef SADCS_CLASS_TILES
#define SADCS_CLASS_TILES 4  // onesweep tiles per SM of the class passes (tuning)
#endif

template <class Chain, bool kCarryWords = false>
struct ClassLoader {
    // 4 tiles per SM (64 registers, some spilled) against 3 (80 registers): the class phase of the
    // 3 GiB genome-like text took 64.0 ms against 67.9, of the 256 MiB natural text 4.86 against 5.11
    // (64-bit chains).
    static constexpr int kTilesPerSm = SADCS_CLASS_TILES;
    static constexpr bool kCarry = kCarryWords;
    static constexpr int kChars = kCarryWords ? kCarryChainChars : kChainChars;
    const uint32_t* __restrict__ lists;       // global lists
    const uint32_t* __restrict__ prevOffset;  // rowBase row of class d - 1: text j's slice offset
    const Chain* __restrict__ chains;         // chains of class d - 1 by index from prevStart (d >= 2)
    const uint64_t* __restrict__ carried;     // kCarryWords: carried words by global slot
    uint32_t prevStart;                       // first slot of class d - 1 in the global lists
    TextSet texts;
    uint32_t d;
    __device__ __forceinline__ uint32_t element(uint32_t j, uint32_t k) const {
        return k == 0 ? texts.endOfText(j) : lists[__ldg(prevOffset + j) + k - 1];
    }
    __device__ __forceinline__ bool load(uint32_t j, uint32_t, uint32_t k, Chain& key, uint32_t& dig) const {
        const uint32_t start = texts.startOf(j), end = texts.endOfText(j);
        const uint32_t p = element(j, k);
        // A stored chain is read for every element, kept or not (the reads are sequential), so that
        // it is in flight together with the position instead of waiting for the filter.
        const bool stored = k > 0 && d > 1;
        const Chain chain = stored ? chains[__ldg(prevOffset + j) - prevStart + k - 1] : Chain(0);
        if (p <= start || p > end || classOfResidue((p - 1) % kV) != d) return false;
        key = stored ? chain : codesBefore<Chain, kChars>(texts, p);
        dig = static_cast<uint32_t>(key) & ((1u << texts.bits) - 1);  // codes order like the bytes they stand for
        return true;
    }
    __device__ __forceinline__ uint32_t value(uint32_t j, uint32_t, uint32_t k) const { return element(j, k) - 1; }
    // The code of T[p - 2], the character before the output p - 1.
    __device__ __forceinline__ uint8_t carryTag(Chain key) const {
        return static_cast<uint8_t>((static_cast<uint32_t>(key) >> texts.bits) & ((1u << texts.bits) - 1));
    }
    // carried(p) for the element p (the text's end: carried(end - 1) itself, from the code stream),
    // then carried(p - 1) from it and the code of T[p - 2].
    __device__ __forceinline__ uint64_t carrySource(uint32_t j, uint32_t, uint32_t k) const {
        if (k == 0) return carriedWord(texts.packed, texts.endOfText(j) - 1, texts.bits);
        return carried[__ldg(prevOffset + j) + k - 1];
    }
    __device__ __forceinline__ uint64_t carryWord(uint32_t k, uint32_t tag, uint64_t source) const {
        return k == 0 ? source : (static_cast<uint64_t>(tag) << (64 - texts.bits)) | (source >> texts.bits);
    }
};

// Writes class d's positions, and (unless chains is null: the last class) the chains of its
// elements: an element p - 1 has p's chain less its first character.
template <class Chain>
struct ClassStorer {
    static constexpr bool kKeys = true;
    uint32_t* __restrict__ lists;
    Chain* __restrict__ chains;  // by index from lo
    uint64_t* __restrict__ carried;  // carried words by global slot (loaders that carry them)
    uint32_t lo, hi;             // class d's slots in the global lists
    uint32_t bits;
    __device__ __forceinline__ void storeKey(uint32_t, uint32_t pos, Chain chain) const {
        if (chains && pos >= lo && pos < hi) chains[pos - lo] = static_cast<Chain>(chain >> bits);
    }
    __device__ __forceinline__ void storeValue(uint32_t, uint32_t pos, uint32_t v) const {
        if (pos >= lo && pos < hi) lists[pos] = v;  // always, unless a look-back timed out
    }
    __device__ __forceinline__ void storeCarry(uint32_t, uint32_t pos, uint64_t w) const {
        if (pos >= lo && pos < hi) carried[pos] = w;
    }
};

// hist[(d * J + j) * 256 + c] = positions q of text j in class d with code c (zeroed by the caller).
// Eight characters per thread from one 64-bit read of the code stream. Consecutive positions are in
// different classes, so the shared counters of one text rarely collide and plain atomics serve.
__global__ void __launch_bounds__(256) classHistogram(uint32_t total, TextSet texts, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[kClasses * 256];
    const bool one = texts.count <= 1;
    for (int i = threadIdx.x; i < kClasses * 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const uint32_t b = texts.bits;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x * 8;
    for (uint64_t base = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) * 8; base < total;
         base += stride) {
        const uint64_t chunk = streamBits(texts.packed, base * b);
        const uint32_t j = texts.textOf(static_cast<uint32_t>(base));
        const uint32_t end = texts.endOfText(j);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint64_t q = base + k;
            const uint32_t c = static_cast<uint32_t>(chunk >> (64 - (k + 1) * b)) & ((1u << b) - 1);
            const uint32_t cls = q < end ? classOfResidue(static_cast<uint32_t>(q % kV)) : 0;
            if (cls) {
                if (one) {
                    atomicAdd(&h[cls * 256 + c], 1u);
                } else {
                    atomicAdd(hist + (cls * texts.count + j) * 256 + c, 1u);
                }
            }
        }
    }
    if (one) {
        __syncthreads();
        for (int i = threadIdx.x; i < kClasses * 256; i += blockDim.x) {
            if (h[i]) atomicAdd(hist + i, h[i]);
        }
    }
}

// Each 256-entry row r of hist becomes rowBase[r] + its exclusive prefix. One block per row.
__global__ void __launch_bounds__(256) classDigitBase(uint32_t* __restrict__ hist, const uint32_t* __restrict__ rowBase) {
    __shared__ uint32_t warpTotals[32];
    uint32_t* row = hist + static_cast<size_t>(blockIdx.x) * 256;
    const uint32_t v = row[threadIdx.x];
    uint32_t total;
    const uint32_t inclusive = blockInclusiveScan<OpSum>(v, warpTotals, total);
    row[threadIdx.x] = rowBase[blockIdx.x] + inclusive - v;
}

// Passes 1 to kClasses - 1: class d from class d - 1, chains of type Chain in the two chain buffers;
// kCarry: the carried words too (carried: by global slot).
template <class Chain, bool kCarry = false>
inline cudaError_t classPasses(const TextSet& texts, const ClassPlan& plan, const ClassTables& tables, uint32_t* lists,
                               const uint32_t* hist, const RadixScratch& radix, uint64_t* const chains[2],
                               uint64_t* carried, cudaStream_t stream) {
    const uint32_t J = tables.texts;
    for (int d = 1; d < kClasses; d++) {
        if (plan.start[d + 1] == plan.start[d]) continue;
        ClassLoader<Chain, kCarry> ld{lists, tables.rowBase + static_cast<size_t>(d - 1) * J,
                                      reinterpret_cast<const Chain*>(chains[d & 1]), carried, plan.start[d - 1],
                                      texts, static_cast<uint32_t>(d)};
        ClassStorer<Chain> st{lists, d + 1 < kClasses ? reinterpret_cast<Chain*>(chains[(d + 1) & 1]) : nullptr,
                              carried, plan.start[d], plan.start[d + 1], texts.bits};
        ManySegments segs{tables.tileStart + static_cast<size_t>(d) * (J + 1),
                          tables.elementStart + static_cast<size_t>(d) * (J + 1), J};
        SADCS_TRY((radixOnesweepPass<Chain, ClassLoader<Chain, kCarry>, ClassStorer<Chain>, ManySegments>(
            ld, st, segs, plan.inputs[d], plan.tiles[d], hist + static_cast<size_t>(d) * J * 256, radix, stream)));
    }
    return cudaSuccess;
}

// Whether a construction carries words through the class passes: one text with codes of at most 2
// bits (the final merge's records are then one word).
inline bool carriesWords(const TextSet& texts) { return texts.count == 1 && texts.bits <= 2; }

// Fills lists (laid out by plan.start, text-major inside each class) from the sample ranks.
// tables: the ClassTables block on the device; scratch: classScratchWords(total, J) words.
// total: bytes of the concatenation (text buffer) scanned by the histogram.
// chains: two buffers of classChainWords(plan) 64-bit words each. carried: null, or (carriesWords)
// one word per list slot, filled with every element's carried word.
inline cudaError_t sortClasses(uint32_t total, const TextSet& texts, const uint32_t* ranks, uint32_t slots,
                               const ClassPlan& plan, const ClassTables& tables, uint32_t* lists, uint32_t* scratch,
                               uint64_t* const chains[2], uint64_t* carried, cudaStream_t stream) {
    if (carried && !carriesWords(texts)) return cudaErrorInvalidValue;
    const uint32_t J = tables.texts;
    const uint32_t live = plan.start[1];
    uint32_t* hist = scratch;  // [kClasses][J][256]
    const RadixScratch radix(classRadixScratch(scratch, J), 0);
    // Class 0 through the pair array (chain buffer 0, free until pass 1) and the slice counters
    // (the radix scratch's digit-base words, unused by the class passes).
    uint32_t* fill = radix.digitBase;
    SADCS_TRY(cudaMemsetAsync(fill, 0, kMaxSampleSlices * sizeof(uint32_t), stream));
    // (with carried words: the pairs' words in chain buffer 1, also free until pass 1)
    if (carried) {
        SADCS_TRY(launch(classPartitionSample<true>, ceilDiv(slots, kSliceTile), kSliceThreads, 0, stream, ranks, slots,
                         live, sampleSliceShift(live, true), texts, fill, chains[0], chains[1]));
    } else {
        SADCS_TRY(launch(classPartitionSample<false>, ceilDiv(slots, kSliceTile), kSliceThreads, 0, stream, ranks,
                         slots, live, sampleSliceShift(live, false), texts, fill, chains[0], nullptr));
    }
    SADCS_TRY(launch(classScatterPairs, ceilDiv(live, 256), 256, 0, stream, chains[0], live, lists, carried,
                     chains[1]));
    SADCS_TRY(cudaMemsetAsync(hist, 0, static_cast<size_t>(kClasses) * J * 256 * 4, stream));
    SADCS_TRY(cudaMemsetAsync(radix.control, 0, 8, stream));
    const uint32_t blocks = std::min<uint32_t>(ceilDiv(total + 7ull, 256 * 8 * 8), 148 * 8);
    SADCS_TRY(launch(classHistogram, std::max(blocks, 1u), 256, 0, stream, total, texts, hist));
    SADCS_TRY(launch(classDigitBase, kClasses * J, 256, 0, stream, hist, tables.rowBase));
    static_assert(2 * kCarryChainChars <= 16, "carrying chains of 2-bit codes fit 16 bits");
    if (carried) return classPasses<uint16_t, true>(texts, plan, tables, lists, hist, radix, chains, carried, stream);
    if (texts.bits * kChainChars <= 16) {
        return classPasses<uint16_t>(texts, plan, tables, lists, hist, radix, chains, nullptr, stream);
    }
    if (texts.bits * kChainChars <= 32) {
        return classPasses<uint32_t>(texts, plan, tables, lists, hist, radix, chains, nullptr, stream);
    }
    return classPasses<uint64_t>(texts, plan, tables, lists, hist, radix, chains, nullptr, stream);
}

}  // namespace sadcs
