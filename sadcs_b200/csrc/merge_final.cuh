// merge_final.cuh - the merge levels: every tile of the 7 lists of a level merged in shared memory;
// the last level writes the suffix array and the BWT, an upper level the rows of the level below.
//
// A tile's window set (at most kMergeCap records, merge.cuh) is held as arrays of fields, not as
// records, so the 32 threads of a warp reading one field of 32 records hit 32 different banks (the
// sample ranks stay in global memory: only comparisons whose first 31 characters agree read them):
//   words[W][cap]  the code stream from the suffix's first character, W = ceil(31 * bits / 64)
//                  64-bit words: every comparison reads k < 32 characters (k = the cover's tie
//                  offset), so no comparison reads global memory
//   pos[cap]       p; end[cap] the end of p's text (several texts only)
//   prev[cap]      the code of the character before p (the BWT byte)
//   idxA, idxB     u16 orders of the records
// The 7 windows are merged by a 3-level tree: (0,1) (2,3) (4,5) 6, then (01,23) (45,6), then
// (0123,456). Each level splits its output into equal chunks, one per thread; a thread finds its
// chunk's start on the merge path of its merge by binary search and walks it, writing record
// indices. The final order gives every record's rank within the window set, hence its place in the
// output (base + rank) for the records between the tile's two splitters.
#pragma once

#include "merge.cuh"

namespace sadcs {

// Shared-memory share of the unified L1/shared array preferred for the final level, in percent of
// the maximum (-1: the driver's choice). The record gathers go through L1 and the kernel runs 40%
// slower with 28 KB of L1 than with 60 KB: 85% gives 196 KB of shared memory (3 tiles of natural
// text per SM) and 60 KB of L1; the driver's own choice would take all 228 KB when the tiles fit.
#ifndef SADCS_MERGE_CARVEOUT
#define SADCS_MERGE_CARVEOUT 85
#endif

// Outputs per thread and tree level, at least: each thread's merge-path search is amortised over
// its chunk (tuning).
#ifndef SADCS_MERGE_MIN_CHUNK
#define SADCS_MERGE_MIN_CHUNK 1
#endif

// 64-bit words of the code stream a final-level record keeps: 31 characters of `bits` bits.
__host__ __device__ constexpr int finalWords(uint32_t bits) {
    return static_cast<int>((31 * bits + 63) / 64);
}

template <int W, bool kMulti>
struct FinalTile {
    static constexpr uint32_t kMergeCap = mergeCap(mergeR(W));
    static constexpr size_t kPerRecord = 8 * W + 4 + (kMulti ? 4 : 0) + 2 + 2 + 1;
    static constexpr size_t sharedBytes() { return kMergeCap * kPerRecord + 64; }
    uint64_t* words;
    uint32_t* pos;
    uint32_t* end;
    uint16_t* idxA;
    uint16_t* idxB;
    uint8_t* prev;
    const uint32_t* ranks;  // the sample ranks in global memory: read only when 31 characters agree
    __device__ __forceinline__ void carve(unsigned char* smem, const uint32_t* sampleRanks) {
        words = reinterpret_cast<uint64_t*>(smem);
        pos = reinterpret_cast<uint32_t*>(words + W * kMergeCap);
        end = pos + kMergeCap;
        ranks = sampleRanks;
        idxA = reinterpret_cast<uint16_t*>(end + (kMulti ? kMergeCap : 0));
        idxB = idxA + kMergeCap;
        prev = reinterpret_cast<uint8_t*>(idxB + kMergeCap);
    }
};

// The fields of a record a comparison reads first, kept in registers while the merge walk holds
// the record: its first code word, and with several texts its position and text end (the words
// are masked to the shorter suffix). With one text the position is read only when the first 31
// characters tie.
struct FinalHead {
    uint32_t idx, pos, end;  // pos, end: several texts only
    uint64_t w0;
};

template <int W, bool kMulti>
__device__ __forceinline__ FinalHead loadHead(const FinalTile<W, kMulti>& s, uint32_t x) {
    FinalHead h;
    h.idx = x;
    h.w0 = s.words[x];
    h.pos = kMulti ? s.pos[x] : 0;
    h.end = kMulti ? s.end[x] : 0;
    return h;
}

// Suffix a < suffix b, by the difference-cover comparison (merge.cuh: lessRecord), cheapest test
// first. The records hold at least the first 31 characters of each suffix. If those differ, the
// first difference orders the suffixes whatever the cover's tie offset k: compared characters past
// a single text's end are code 0, the smallest, so the shorter suffix is the smaller there too, as
// it must be; with several texts the stream continues into the next text, so the words are masked
// to the shorter suffix. Only when all compared characters agree (hence the first k, k < 32) do the
// sample ranks at a + k and b + k decide, or the lengths when one suffix ends within k.
template <int W, bool kMulti>
__device__ __forceinline__ bool headLess(const FinalTile<W, kMulti>& s, const FinalHead& a, const FinalHead& b,
                                         uint32_t n, uint32_t bits) {
    if constexpr (kMulti) {
        if (a.end != b.end) return a.end < b.end;  // different texts: text order
        n = a.end;
        const uint32_t i = a.pos, j = b.pos;
        const uint32_t lim = min(n - i, n - j) * bits;  // bits of the shorter suffix
        uint64_t x = a.w0, y = b.w0;
        if (lim < 64) {
            const uint64_t mk = lim ? ~uint64_t(0) << (64 - lim) : 0;
            x &= mk;
            y &= mk;
        }
        if (x != y) return x < y;
#pragma unroll
        for (int w = 1; w < W; w++) {
            if (lim <= 64u * w) break;
            x = s.words[w * s.kMergeCap + a.idx];
            y = s.words[w * s.kMergeCap + b.idx];
            if (lim < 64u * (w + 1)) {
                const uint64_t mk = ~uint64_t(0) << (64u * (w + 1) - lim);
                x &= mk;
                y &= mk;
            }
            if (x != y) return x < y;
        }
    } else {
        if (a.w0 != b.w0) return a.w0 < b.w0;
#pragma unroll
        for (int w = 1; w < W; w++) {
            const uint64_t x = s.words[w * s.kMergeCap + a.idx], y = s.words[w * s.kMergeCap + b.idx];
            if (x != y) return x < y;
        }
    }
    const uint32_t i = kMulti ? a.pos : s.pos[a.idx], j = kMulti ? b.pos : s.pos[b.idx];
    const uint32_t k = tieOffset(coverRotation(i), coverRotation(j));
    if (k > min(n - i, n - j) || i + k == n || j + k == n) return i > j;  // one is a prefix of the other
    // rare (2-3% of the comparisons on natural and DNA-like text): the ranks come from global memory
    return __ldg(s.ranks + pack(i + k)) < __ldg(s.ranks + pack(j + k));
}

// Record index at position x of a level's source order: src[x], or x itself for the first level,
// whose source is the windows in list order (kIdentity: src is not read).
template <bool kIdentity>
__device__ __forceinline__ uint32_t sourceAt(const uint16_t* src, uint32_t x) {
    if constexpr (kIdentity) {
        return x;
    } else {
        return src[x];
    }
}

// One tree level: the merges m (A = [mb[3m], mb[3m + 1]), B = [mb[3m + 1], mb[3m + 2]) of src,
// written to dst from mb[3m]), which together cover [0, size); mb is in shared memory. Thread t
// writes outputs [t * chunk, (t + 1) * chunk).
template <int W, bool kMulti, bool kIdentity>
__device__ __forceinline__ void finalLevel(const FinalTile<W, kMulti>& s, const uint16_t* src, uint16_t* dst,
                                           const uint32_t* mb, int merges, uint32_t size, uint32_t n,
                                           uint32_t bits) {
    constexpr uint32_t kThreads = mergeThreads(W);
    const uint32_t chunk = max((size + kThreads - 1) / kThreads, static_cast<uint32_t>(SADCS_MERGE_MIN_CHUNK));
    uint32_t at = threadIdx.x * chunk;
    const uint32_t stopAll = min(at + chunk, size);
    int m = 0;
    while (at < stopAll) {
        while (m + 1 < merges && at >= mb[3 * m + 2]) m++;
        const uint32_t a0 = mb[3 * m], a1 = mb[3 * m + 1], b1 = mb[3 * m + 2];
        const uint32_t lenA = a1 - a0, lenB = b1 - a1;
        uint32_t d = at - a0;
        const uint32_t stop = min(stopAll, b1) - a0;
        uint32_t lo = d > lenB ? d - lenB : 0, hi = min(d, lenA);
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (headLess(s, loadHead(s, sourceAt<kIdentity>(src, a0 + mid)),
                         loadHead(s, sourceAt<kIdentity>(src, a1 + d - 1 - mid)), n, bits)) {
                lo = mid + 1;
            } else {
                hi = mid;
            }
        }
        uint32_t i = lo, j = d - lo;
        // Both heads in registers; a step takes one side and loads that side's next record (the
        // merge's first record when the side is used up: in range, and never compared again), so
        // the lanes of a warp do not diverge on which side they took.
        FinalHead ha = loadHead(s, sourceAt<kIdentity>(src, i < lenA ? a0 + i : a0));
        FinalHead hb = loadHead(s, sourceAt<kIdentity>(src, j < lenB ? a1 + j : a0));
        for (; d < stop; d++) {
            const bool takeA = j == lenB || (i < lenA && headLess(s, ha, hb, n, bits));
            dst[a0 + d] = static_cast<uint16_t>(takeA ? ha.idx : hb.idx);
            i += takeA ? 1u : 0u;
            j += takeA ? 0u : 1u;
            const uint32_t x = takeA ? (i < lenA ? a0 + i : a0) : (j < lenB ? a1 + j : a0);
            const FinalHead h = loadHead(s, sourceAt<kIdentity>(src, x));
            if (takeA) {
                ha = h;
            } else {
                hb = h;
            }
        }
        at = a0 + stop;
    }
}

// Tiles resident per SM the register budget is set for: as many as the SM's 2048 threads hold for
// one-word records (their shared memory allows more), 4 for wider records, which fill shared
// memory at 4 (tuning).
#ifndef SADCS_MERGE_TILES_W1
#define SADCS_MERGE_TILES_W1 (2048 / SADCS_MERGE_THREADS_W1)
#endif
template <int W>
constexpr int mergeTilesPerSm() {
    return W == 1 ? SADCS_MERGE_TILES_W1 : 4;
}

// The merge tree over a gathered tile, and its outputs: the SA and BWT (kFinal) or the rows.
template <int W, bool kMulti, bool kFinal>
__device__ __forceinline__ void mergeTileTail(const MergeArgs& a, const FinalTile<W, kMulti>& s, const MergeTileInfo& t,
                                              const uint32_t* bounds, uint32_t size, uint32_t n, uint32_t bits,
                                              uint32_t& sLo, uint32_t& sHi) {
    constexpr int kMergeThreads = mergeThreads(W);
    constexpr uint32_t kMergeR = mergeR(W);
    // The merge tree.
    finalLevel<W, kMulti, true>(s, nullptr, s.idxB, bounds, 4, size, n, bits);
    __syncthreads();
    finalLevel<W, kMulti, false>(s, s.idxB, s.idxA, bounds + 12, 2, size, n, bits);
    __syncthreads();
    finalLevel<W, kMulti, false>(s, s.idxA, s.idxB, bounds + 18, 1, size, n, bits);
    __syncthreads();
    const uint16_t* order = s.idxB;

    // Ranks of the tile's splitters in the window set bound the outputs this tile owns.
    for (uint32_t r = threadIdx.x; r < size; r += kMergeThreads) {
        const uint32_t x = order[r];
        if (x == t.loIdx) sLo = r;
        if (x == t.hiIdx) sHi = r;
    }
    __syncthreads();
    const uint32_t lo = sLo, hi = sHi;
    if constexpr (kFinal) {
        for (uint32_t r = lo + threadIdx.x; r < hi; r += kMergeThreads) {
            const uint32_t x = order[r];
            const uint32_t q = s.pos[x];
            const uint32_t gIdx = t.base + r;
            if (gIdx >= a.level.start[kClasses]) {  // cannot happen for a correct tiling; never write out of range
                atomicExch(a.error, 2u);
                continue;
            }
            const uint32_t tj = kMulti ? a.texts.textOf(q) : 0;
            const uint32_t first = kMulti ? a.texts.startOf(tj) : 0;
            const uint32_t base = kMulti ? __ldg(a.outBase + tj) : 0;
            if (kMulti && a.saTexts) {
                a.saTexts[tj][gIdx - base] = q - first;
            } else if (a.sa) {
                a.sa[gIdx] = q - first;
            }
            if ((a.bwt || (kMulti && a.bwtTexts)) && q != first) {
                const uint32_t row = gIdx - base, zero = __ldg(a.rowZero + tj);
                const uint32_t local = row < zero ? row + 1 : row;
                const uint8_t c = __ldg(a.texts.decode + s.prev[x]);
                if (kMulti && a.bwtTexts) {
                    a.bwtTexts[tj][local] = c;
                } else {
                    a.bwt[base + local] = c;
                }
            }
        }
    } else {
        // rank[x] of every record in the merged order (idxA is free again), then the rows: for a
        // sampled element, the elements of each other list before it are those of its window with a
        // smaller rank (a binary search: each window is in list order, hence in rank order).
        uint16_t* rank = s.idxA;
        for (uint32_t r = threadIdx.x; r < size; r += kMergeThreads) rank[order[r]] = static_cast<uint16_t>(r);
        __syncthreads();
        for (uint32_t r = lo + threadIdx.x; r < hi; r += kMergeThreads) {
            const uint32_t g = t.base + r;
            if (g % kMergeR != 0) continue;
            if (g >= a.level.start[kClasses]) {  // cannot happen for a correct tiling; never write out of range
                atomicExch(a.error, 2u);
                continue;
            }
            const uint32_t x = order[r];
            const int l = listOfElement(t.seg, x);
            MergeRow row;
            row.list = static_cast<uint32_t>(l);
#pragma unroll
            for (int b = 0; b < kClasses; b++) {
                if (b == l) {
                    row.c[b] = t.win[l] + (x - t.seg[l]);
                    continue;
                }
                uint32_t from = t.seg[b], to = t.seg[b + 1];  // first record of list b ranked at or after r
                while (from < to) {
                    const uint32_t mid = (from + to) >> 1;
                    if (rank[mid] < r) from = mid + 1; else to = mid;
                }
                row.c[b] = t.win[b] + (from - t.seg[b]);
            }
            a.rowsOut[g / kMergeR] = row;
        }
    }
}

// kFinal: the last level, writing the SA and the BWT; otherwise an upper level, writing the rows
// (every R-th element of the merged order with its per-list counts) that bound the tiles below.
template <int W, bool kMulti, bool kFinal>
__global__ void __launch_bounds__(mergeThreads(W), mergeTilesPerSm<W>()) mergeTree(MergeArgs a) {
    constexpr int kMergeThreads = mergeThreads(W);
    constexpr uint32_t kMergeR = mergeR(W);
    constexpr uint32_t kMergeCap = FinalTile<W, kMulti>::kMergeCap;
    extern __shared__ __align__(16) unsigned char smem[];
    FinalTile<W, kMulti> s;
    s.carve(smem, a.ranks);
    __shared__ MergeTileInfo t;
    __shared__ uint32_t sLo, sHi;
    __shared__ uint32_t bounds[3 * 7];  // the tree's merges: 4 + 2 + 1 triples of window offsets
    if (threadIdx.x < 32) {
        planTileWindows(a, kMergeCap, t);
        __syncwarp();
        // (0,1) (2,3) (4,5) (6,-), then (01,23) (45,6), then (0123,456): indices into t.seg, 3 bits
        // each (a register constant: a table indexed by the lane would live in local memory)
        constexpr uint8_t kTree[21] = {0, 1, 2, 2, 3, 4, 4, 5, 6, 6, 7, 7, 0, 2, 4, 4, 6, 7, 0, 4, 7};
        constexpr uint64_t kTreePacked = [] {
            uint64_t v = 0;
            for (int i = 0; i < 21; i++) v |= static_cast<uint64_t>(kTree[i]) << (3 * i);
            return v;
        }();
        if (threadIdx.x < 21) bounds[threadIdx.x] = t.seg[(kTreePacked >> (3 * threadIdx.x)) & 7];
        if (threadIdx.x == 0) {
            sLo = 0;
            sHi = t.size;
            if (t.bad && a.error) atomicExch(a.error, 1u);
        }
    }
    __syncthreads();
    if (t.bad) return;
    const uint32_t size = t.size;
    const uint32_t* st = a.level.start;
    const uint32_t bits = a.texts.bits;
    const uint32_t n = kMulti ? 0u : a.texts.oneEnd;

    constexpr int kItems = (kMergeCap + kMergeThreads - 1) / kMergeThreads;
    if constexpr (kFinal && W == 1 && !kMulti) {
        if (a.carried) {
            // Carried words (one text): each record's code word and previous character come with its
            // position, read in list order beside it (half of a thread's items in flight at a time:
            // all of them would not fit the register budget).
            constexpr int kHalf = (kItems + 1) / 2;
#pragma unroll
            for (int h = 0; h < kItems; h += kHalf) {
                uint32_t p[kHalf];
                uint64_t c[kHalf];
#pragma unroll
                for (int j = 0; j < kHalf; j++) {
                    const uint32_t e = threadIdx.x + (h + j) * kMergeThreads;
                    p[j] = 0;
                    c[j] = 0;
                    if (h + j < kItems && e < size) {
                        const int l = listOfElement(t.seg, e);
                        const uint32_t slot = st[l] + t.win[l] + (e - t.seg[l]);
                        p[j] = a.level.lists[slot];
                        c[j] = a.carried[slot];
                    }
                }
#pragma unroll
                for (int j = 0; j < kHalf; j++) {
                    const uint32_t e = threadIdx.x + (h + j) * kMergeThreads;
                    if (h + j < kItems && e < size) {
                        uint32_t q = p[j];
                        if (q >= n) {  // cannot happen for valid class lists; never read out of range
                            atomicExch(a.error, 3u);
                            q = 0;
                        }
                        s.pos[e] = q;
                        s.words[e] = c[j] << bits;
                        s.prev[e] = static_cast<uint8_t>(c[j] >> (64 - bits));
                    }
                }
            }
            __syncthreads();
            mergeTileTail<W, kMulti, kFinal>(a, s, t, bounds, size, n, bits, sLo, sHi);
            return;
        }
    }

    // Gather: positions from the lists (coalesced), then each record's code words and ranks by
    // asynchronous copies, all in flight at once; the word after them and the word before them
    // (when the previous character starts there) by plain loads, also in flight.
    uint32_t p[kItems];
    uint64_t extra[kItems], before[kItems];
    // Positions first, every list load in flight at once (an asynchronous copy between two loads
    // would order them), then the records' copies.
#pragma unroll
    for (int j = 0; j < kItems; j++) {
        const uint32_t e = threadIdx.x + j * kMergeThreads;
        p[j] = 0;
        if (e < size) {
            const int l = listOfElement(t.seg, e);
            p[j] = a.level.lists[st[l] + t.win[l] + (e - t.seg[l])];
        }
    }
    // The end of each position's text (several texts: one load chain per item, all in flight).
    uint32_t ends[kMulti ? kItems : 1];
    if constexpr (kMulti) {
#pragma unroll
        for (int j = 0; j < kItems; j++) ends[j] = threadIdx.x + j * kMergeThreads < size ? a.texts.endOf(p[j]) : 0;
    }
#pragma unroll
    for (int j = 0; j < kItems; j++) {
        const uint32_t e = threadIdx.x + j * kMergeThreads;
        if (e < size) {
            uint32_t q = p[j];
            const uint32_t qEnd = kMulti ? ends[j] : a.texts.oneEnd;
            if (q >= qEnd) {  // cannot happen for valid class lists; never read out of range
                atomicExch(a.error, 3u);
                q = 0;
            }
            p[j] = q;
            s.pos[e] = q;
            if constexpr (kMulti) s.end[e] = q < qEnd ? qEnd : a.texts.endOf(0);
            const uint64_t* src = a.texts.packed + ((static_cast<uint64_t>(q) * bits) >> 6);
#pragma unroll
            for (int w = 0; w < W; w++) cpAsync8(&s.words[w * kMergeCap + e], src + w);
        }
    }
#pragma unroll
    for (int j = 0; j < kItems; j++) {
        const uint32_t e = threadIdx.x + j * kMergeThreads;
        extra[j] = 0;
        before[j] = 0;
        if (e < size) {
            const uint64_t bit = static_cast<uint64_t>(p[j]) * bits;
            const uint64_t w0 = bit >> 6;
            extra[j] = __ldg(a.texts.packed + w0 + W);
            if (kFinal && (bit & 63) < bits && w0 > 0) before[j] = __ldg(a.texts.packed + w0 - 1);
        }
    }
    cpAsyncWaitAll();
#pragma unroll
    for (int j = 0; j < kItems; j++) {
        const uint32_t e = threadIdx.x + j * kMergeThreads;
        if (e < size) {
            const uint32_t o = static_cast<uint32_t>((static_cast<uint64_t>(p[j]) * bits) & 63);
            uint64_t r[W + 1];
#pragma unroll
            for (int w = 0; w < W; w++) r[w] = s.words[w * kMergeCap + e];
            r[W] = extra[j];
            // the character before p ends at bit o of word 0: bits [64 + o - b, 64 + o) of before:r[0]
            if constexpr (kFinal) {
                const uint64_t window = o ? (before[j] << o) | (r[0] >> (64 - o)) : before[j];
                s.prev[e] = static_cast<uint8_t>(window & ((1u << bits) - 1));
            }
            if (o) {
#pragma unroll
                for (int w = 0; w < W; w++) s.words[w * kMergeCap + e] = (r[w] << o) | (r[w + 1] >> (64 - o));
            }
        }
    }
    __syncthreads();
    mergeTileTail<W, kMulti, kFinal>(a, s, t, bounds, size, n, bits, sLo, sHi);
}

// Launches a level (kFinal: the last) for the texts' code width (W words per record) and text count.
template <int W, bool kMulti, bool kFinal>
inline cudaError_t launchTreeFor(const MergeArgs& args, uint32_t tiles, cudaStream_t stream) {
    constexpr size_t shared = FinalTile<W, kMulti>::sharedBytes();
    static std::atomic<uint64_t> configured{0};
    SADCS_TRY(configureOnce(configured, [] {
        SADCS_TRY(cudaFuncSetAttribute(mergeTree<W, kMulti, kFinal>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(shared)));
#if SADCS_MERGE_CARVEOUT >= 0
        SADCS_TRY(cudaFuncSetAttribute(mergeTree<W, kMulti, kFinal>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       SADCS_MERGE_CARVEOUT));
#endif
        return cudaSuccess;
    }));
    return launch(mergeTree<W, kMulti, kFinal>, tiles, mergeThreads(W), shared, stream, args);
}

template <bool kMulti, bool kFinal>
inline cudaError_t launchTreeWidth(const MergeArgs& args, uint32_t tiles, cudaStream_t stream) {
    switch (finalWords(args.texts.bits)) {
        case 1: return launchTreeFor<1, kMulti, kFinal>(args, tiles, stream);
        case 2: return launchTreeFor<2, kMulti, kFinal>(args, tiles, stream);
        case 3: return launchTreeFor<3, kMulti, kFinal>(args, tiles, stream);
        default: return launchTreeFor<4, kMulti, kFinal>(args, tiles, stream);
    }
}

// One merge level: kFinal writes the SA and BWT, otherwise the rows of the level below.
template <bool kFinal>
inline cudaError_t launchTree(const MergeArgs& args, uint32_t tiles, cudaStream_t stream) {
    return args.texts.count > 1 ? launchTreeWidth<true, kFinal>(args, tiles, stream)
                                : launchTreeWidth<false, kFinal>(args, tiles, stream);
}

}  // namespace sadcs
