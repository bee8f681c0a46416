// merge.cuh - one multiway merge of the 7 sorted class lists into the suffix array and the BWT
// (the reference's step 4, src/cuda/merge.cuh; comparison as lessGlobal, merge.cuh:53-71).
//
// Two suffixes i, j compare in O(1): k = tie[i%32][j%32] < 32 has i + k and j + k both sampled, so
// compare T[i, i+k) with T[j, j+k) and then the sample ranks at i + k and j + k; a suffix that ends
// first is the smaller.
//
// Tiling (this build's own scheme). Level 0 is the 7 lists; level L+1 keeps every G-th element of
// each list of level L (its "splitters"), until a level fits in one tile. Merging level L+1 yields,
// for every R-th element s of its merged order, a row: s's list and, for every list b, c_b = the
// number of level-(L+1) elements of list b smaller than s. A tile of level L covers the output from
// one such splitter s_lo to the next, s_hi. For list b it loads the window
//   [ (c_b(s_lo) - 1) * G + 1 ,  c_b(s_hi) * G )      (exact at s_lo's and s_hi's own lists)
// which contains every element of b in [s_lo, s_hi), while every element of b before the window is
// smaller than s_lo. Since sum_b c_b(s) is s's merged position, a window set holds at most
// G*R + 6*(G-1) + 1 elements whatever the data: one fixed shared-memory capacity, no overflow path.
// Inside the tile the windows are merged by a tree of merge paths (merge_final.cuh); an element's
// output position is the windows' total start plus its rank in the merged window set, and the tile
// writes the elements between s_lo and s_hi (the last level: SA and BWT; upper levels: rows).
#pragma once

#include <algorithm>
#include <cstring>

#include "alphabet.cuh"
#include "common.cuh"

namespace sadcs {

constexpr uint32_t kMergeG = 32;

// Tile shape, by the number W of 64-bit code words a record keeps (the code width): rows every R
// splitters, so a tile holds at most G * R + 6 * (G - 1) + 1 records, and its threads. R sets the
// tile's shared memory and so the tiles per SM. One-word records (2-bit codes: 17 bytes) leave
// shared memory to spare and take larger tiles: on the 3 GiB genome-like text the final level took
// 170.3 ms at R = 64 with 384 threads (5 tiles per SM), 174.5 at R = 80 with 512 threads (4),
// 176.6 at R = 40 with 256 threads (8) and 188.6 at R = 40 with 384 (4); wider records (33 bytes for
// 6-bit codes) fill it: the 256 MiB natural-language-like text took 14.0 ms at R = 40, 14.6 at 56
// and 17.1 at 64 (tuning).
#ifndef SADCS_MERGE_R
#define SADCS_MERGE_R 40
#endif
#ifndef SADCS_MERGE_THREADS
#define SADCS_MERGE_THREADS 384
#endif
#ifndef SADCS_MERGE_R_W1
#define SADCS_MERGE_R_W1 64
#endif
#ifndef SADCS_MERGE_THREADS_W1
#define SADCS_MERGE_THREADS_W1 384
#endif
__host__ __device__ constexpr uint32_t mergeCap(uint32_t r) {
    return kMergeG * r + 6 * (kMergeG - 1) + 1;
}
__host__ __device__ constexpr uint32_t mergeR(int words) {
    return words == 1 ? SADCS_MERGE_R_W1 : SADCS_MERGE_R;
}
__host__ __device__ constexpr int mergeThreads(int words) {
    return words == 1 ? SADCS_MERGE_THREADS_W1 : SADCS_MERGE_THREADS;
}
// The smallest R of any shape: the most rows a plan can have (memory plans bound with it).
constexpr uint32_t kMergeRMin = SADCS_MERGE_R < SADCS_MERGE_R_W1 ? SADCS_MERGE_R : SADCS_MERGE_R_W1;
static_assert(mergeCap(SADCS_MERGE_R) <= 65535 && mergeCap(SADCS_MERGE_R_W1) <= 65535, "u16 record indices");
constexpr uint32_t kNoList = 0xFFFFFFFFu;
constexpr int kMaxLevels = 10;

struct __align__(16) MergeRow {
    uint32_t list;
    uint32_t c[kClasses];
};
static_assert(sizeof(MergeRow) == 32, "a row is 8 words");

// A suffix for single comparisons in registers (the searches of mergeSuffixZeroRows): w0, w1 = 128
// bits of the code stream from pos; end: the end of pos's text (texts are ordered by it); text: its
// index. Comparisons reaching past w1 read the code stream.
struct MergeRecord {
    uint64_t w0, w1;
    uint32_t rank[kK];
    uint32_t pos;
    uint32_t end;
    uint32_t text;
};

struct MergeLevel {
    const uint32_t* lists;
    uint32_t start[kClasses + 1];
};

struct MergeArgs {
    const uint8_t* text;
    const uint32_t* ranks;
    TextSet texts;
    MergeLevel level;
    const uint32_t* outBase;  // per text: first output slot (SA entry / BWT byte)
    uint32_t* rowZero;        // per text: the output row of the text's first suffix
    const MergeRow* rowsIn;  // null: one tile over the whole level
    MergeRow* rowsOut;       // levels >= 1
    uint32_t* sa;            // level 0, optional: text-local positions
    uint8_t* bwt;            // level 0, optional: the final BWT bytes of every text
    uint32_t* const* saTexts;  // level 0, optional, in place of sa: one output array per text
    uint8_t* const* bwtTexts;  // level 0, optional, in place of bwt: one output array per text
    uint32_t* error;         // set nonzero if a window set exceeds the capacity (never, by construction)
    const uint64_t* carried;  // level 0, optional: every list slot's carried word (one text, 1-word records)
    uint32_t tileOffset;      // tiles of this launch start here (a level launched in pieces)
};

// The top `bits` bits set (bits <= 64).
__device__ __forceinline__ uint64_t topMask(uint32_t bits) {
    return bits >= 64 ? ~uint64_t(0) : (bits == 0 ? uint64_t(0) : ~uint64_t(0) << (64 - bits));
}

__device__ __forceinline__ void loadRecord(const uint8_t* __restrict__ text, const uint32_t* __restrict__ ranks,
                                           const TextSet& texts, uint32_t p, MergeRecord& r) {
    const uint64_t bit = static_cast<uint64_t>(p) * texts.bits;
    r.w0 = streamBits(texts.packed, bit);
    r.w1 = streamBits(texts.packed, bit + 64);
    const uint32_t base = pack(p);
#pragma unroll
    for (int s = 0; s < kK; s++) r.rank[s] = __ldg(ranks + base + s);
    r.pos = p;
    r.text = texts.textOf(p);
    r.end = texts.endOfText(r.text);
}

// Cover tables the comparison reads, in shared memory: the threads of a warp index them at
// different places, which constant memory would serialise.
struct MergeTables {
    uint8_t tie[kV][kV];
    uint8_t slot[kV][kV];
};

__device__ __forceinline__ bool lessRecord(const MergeRecord& a, const MergeRecord& b, const TextSet& texts,
                                           const MergeTables& tb) {
    if (a.end != b.end) return a.end < b.end;  // different texts: text order
    const uint32_t n = a.end;
    const uint32_t i = a.pos, j = b.pos;
    const uint32_t k = tb.tie[i % kV][j % kV];
    const uint32_t common = min(k, min(n - i, n - j));
    const uint32_t bits = common * texts.bits;
    uint64_t x = a.w0, y = b.w0;
    if (bits < 64) {
        const uint64_t mk = topMask(bits);
        x &= mk;
        y &= mk;
    }
    if (x != y) return x < y;
    if (bits > 64) {
        x = a.w1;
        y = b.w1;
        if (bits < 128) {
            const uint64_t mk = topMask(bits - 64);
            x &= mk;
            y &= mk;
        }
        if (x != y) return x < y;
        for (uint32_t o = 128; o < bits; o += 64) {
            x = streamBits(texts.packed, static_cast<uint64_t>(i) * texts.bits + o);
            y = streamBits(texts.packed, static_cast<uint64_t>(j) * texts.bits + o);
            if (bits - o < 64) {
                const uint64_t mk = topMask(bits - o);
                x &= mk;
                y &= mk;
            }
            if (x != y) return x < y;
        }
    }
    if (common < k || i + k == n || j + k == n) return i > j;  // one is a prefix of the other
    return a.rank[tb.slot[i % kV][k]] < b.rank[tb.slot[j % kV][k]];
}

struct MergeTileInfo {
    uint32_t seg[kClasses + 1];
    uint32_t win[kClasses];
    uint32_t base, loIdx, hiIdx, size;
    int bad;
};


__device__ __forceinline__ int listOfElement(const uint32_t* seg, uint32_t e) {
    int l = 0;
    while (e >= seg[l + 1]) l++;
    return l;
}

// Warp 0 of a tile (all 32 lanes): its window in every list (t.win, t.seg; lane b plans list b),
// the number of elements before the windows (t.base), the window indices of the tile's two
// splitters (t.loIdx, t.hiIdx; kNoList for the ends of the level) and whether the window set fits
// (t.bad otherwise, never by construction).
__device__ __forceinline__ void planTileWindows(const MergeArgs& a, uint32_t cap, MergeTileInfo& t) {
    const uint32_t* st = a.level.start;
    const uint32_t b = threadIdx.x & 31;
    uint32_t w = 0, e = 0;
    uint32_t loList = kNoList, hiList = kNoList;
    if (!a.rowsIn) {
        if (b < kClasses) e = st[b + 1] - st[b];
    } else {
        const MergeRow* lo = a.rowsIn + a.tileOffset + blockIdx.x;
        const MergeRow* hi = lo + 1;
        loList = lo->list;
        hiList = hi->list;
        if (b < kClasses) {
            const uint32_t len = st[b + 1] - st[b];
            const uint32_t cLo = lo->c[b], cHi = hi->c[b];
            if (loList == kNoList) {
                w = 0;
            } else if (b == loList) {
                w = cLo * kMergeG;
            } else {
                w = cLo == 0 ? 0 : (cLo - 1) * kMergeG + 1;
            }
            if (hiList == kNoList) {
                e = len;
            } else if (b == hiList) {
                e = cHi * kMergeG + 1;
            } else {
                e = min(len, cHi * kMergeG);
            }
            w = min(w, len);
            e = max(min(e, len), w);
        }
    }
    // seg[b + 1] = the window lengths of lists 0..b (inclusive scan over the lanes)
    uint32_t seg = e - w;
#pragma unroll
    for (int d = 1; d < 8; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, seg, d);
        if (b >= static_cast<uint32_t>(d)) seg += v;
    }
    const uint32_t base = __reduce_add_sync(0xffffffffu, w);
    const uint32_t size = __shfl_sync(0xffffffffu, seg, kClasses - 1);
    const uint32_t loStart = loList == kNoList || loList == 0 ? 0u : __shfl_sync(0xffffffffu, seg, (loList - 1) & 31);
    const uint32_t hiEnd = hiList == kNoList ? 0u : __shfl_sync(0xffffffffu, seg, hiList & 31);
    if (b < kClasses) {
        t.win[b] = w;
        t.seg[b + 1] = seg;
    }
    if (b == 0) {
        t.seg[0] = 0;
        t.base = base;
        t.size = size;
        t.loIdx = loList == kNoList ? kNoList : loStart;
        t.hiIdx = hiList == kNoList ? kNoList : hiEnd - 1;
        t.bad = size > cap;
    }
}

// S_{L+1}: every G-th element of each list of level L.
__global__ void mergeGatherSplitters(const uint32_t* __restrict__ lists, MergeLevel from, MergeLevel to,
                                     uint32_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= to.start[kClasses]) return;
    int b = 0;
    while (i >= to.start[b + 1]) b++;
    out[i] = lists[from.start[b] + (i - to.start[b]) * kMergeG];
}

__global__ void mergeWriteSentinel(MergeRow* row, MergeLevel level) {
    if (threadIdx.x == 0) {
        MergeRow r;
        r.list = kNoList;
        for (int b = 0; b < kClasses; b++) r.c[b] = level.start[b + 1] - level.start[b];
        *row = r;
    }
}

// rowZero[j] += the elements of list threadIdx.x in text j smaller than text j's first suffix: its
// output row within the text. One block per text. rowBase: the class tables' first slot of every
// (class, text); classEnd: plan.start[1..7].
__global__ void mergeSuffixZeroRows(MergeArgs a, const uint32_t* __restrict__ rowBase, MergeLevel classes,
                                    uint32_t* rowZero) {
    __shared__ MergeTables tb;
    for (int i = threadIdx.x; i < kV * kV; i += blockDim.x) {
        (&tb.tie[0][0])[i] = (&cCover.tie[0][0])[i];
        (&tb.slot[0][0])[i] = (&cCover.slot[0][0])[i];
    }
    __syncthreads();
    const int b = threadIdx.x;
    const uint32_t j = blockIdx.x, J = a.texts.count;
    if (b >= kClasses) return;
    MergeRecord zero;
    loadRecord(a.text, a.ranks, a.texts, a.texts.startOf(j), zero);
    const uint32_t first = rowBase[static_cast<size_t>(b) * J + j];
    const uint32_t last = j + 1 < J ? rowBase[static_cast<size_t>(b) * J + j + 1] : classes.start[b + 1];
    const uint32_t* list = a.level.lists + first;
    uint32_t lo = 0, hi = last - first;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        MergeRecord r;
        loadRecord(a.text, a.ranks, a.texts, list[mid], r);
        if (lessRecord(r, zero, a.texts, tb)) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    atomicAdd(rowZero + j, lo);
}

// bwt[outBase[j]] = the last character of text j (the sentinel's row).
__global__ void mergeBwtHeads(const uint8_t* __restrict__ text, TextSet texts, const uint32_t* __restrict__ outBase,
                              uint8_t* bwt, uint8_t* const* bwtTexts) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= texts.count) return;
    const uint8_t c = charByte(texts, texts.endOfText(j) - 1);
    if (bwtTexts) {
        bwtTexts[j][0] = c;
    } else {
        bwt[outBase[j]] = c;
    }
}

// Sizes of every level, planned on the host from n alone.
struct MergePlan {
    int top = 0;                                   // levels 0..top; level top fits one tile
    uint32_t start[kMaxLevels][kClasses + 1] = {};
    size_t listWord[kMaxLevels] = {};              // word offset of level L >= 1 in the splitter buffer
    size_t rowIndex[kMaxLevels] = {};              // row offset of the rows serving level L's tiles
    uint32_t tiles[kMaxLevels] = {};
    size_t splitterWords = 0;
    size_t rows = 0;
};

// r: the tile shape's row spacing (mergeR of the texts' code width).
inline MergePlan planMerge(const uint32_t* classStart, uint32_t r) {
    MergePlan p;
    for (int b = 0; b <= kClasses; b++) p.start[0][b] = classStart[b];
    int L = 0;
    while (p.start[L][kClasses] > mergeCap(r) && L + 1 < kMaxLevels) {
        p.listWord[L + 1] = p.splitterWords;
        for (int b = 0; b < kClasses; b++) {
            const uint32_t len = p.start[L][b + 1] - p.start[L][b];
            p.start[L + 1][b + 1] = p.start[L + 1][b] + (len + kMergeG - 1) / kMergeG;
        }
        p.splitterWords += p.start[L + 1][kClasses] + 64;
        L++;
    }
    p.top = L;
    for (int l = 0; l < L; l++) {
        p.tiles[l] = (p.start[l + 1][kClasses] + r - 1) / r;
        p.rowIndex[l] = p.rows;
        p.rows += p.tiles[l] + 1;
    }
    p.tiles[L] = 1;
    return p;
}

// The merge levels (merge_final.cuh).
template <bool kFinal>
inline cudaError_t launchTree(const MergeArgs& args, uint32_t tiles, cudaStream_t stream);

// The download of the outputs to page-locked host buffers while the last level runs: the level is
// launched in `chunks` pieces of tiles, and once piece k is done, the outputs below the first
// output of its successor's first tile are final and are copied on `stream`. That first output is
// bounded below by the tile's window base, which the host computes from the tile's row (read back
// once the upper levels are done): no output below the base belongs to a later tile. A BWT byte at
// x comes from row x or x - 1, so the same bound holds for the BWT.
constexpr int kMaxDownloadChunks = 8;
struct OverlappedDownload {
    uint32_t* sa = nullptr;        // page-locked host outputs (either may be null)
    uint8_t* bwt = nullptr;
    const uint32_t* deviceSa = nullptr;  // where the last level writes them
    const uint8_t* deviceBwt = nullptr;
    cudaStream_t stream = nullptr;  // the copies' stream
    cudaEvent_t* events = nullptr;  // kMaxDownloadChunks + 1 events
    uint32_t* hostRows = nullptr;   // page-locked, 8 * kMaxDownloadChunks words
    uint64_t outputs = 0;
};

// The first output any tile from row `r` on can own: the sum of its window starts (planTileWindows).
inline uint64_t tileOutputBound(const MergeRow& r, const uint32_t* start) {
    if (r.list == kNoList) return 0;
    uint64_t sum = 0;
    for (int b = 0; b < kClasses; b++) {
        const uint32_t len = start[b + 1] - start[b];
        const uint32_t c = r.c[b];
        uint64_t w = static_cast<uint32_t>(b) == r.list ? static_cast<uint64_t>(c) * kMergeG
                                                         : (c == 0 ? 0 : static_cast<uint64_t>(c - 1) * kMergeG + 1);
        sum += w < len ? w : len;
    }
    return sum;
}

inline cudaError_t copyDown(const OverlappedDownload& d, uint64_t from, uint64_t to) {
    if (to <= from) return cudaSuccess;
    if (d.sa) {
        SADCS_TRY(cudaMemcpyAsync(d.sa + from, d.deviceSa + from, 4 * (to - from), cudaMemcpyDeviceToHost, d.stream));
    }
    if (d.bwt) {
        SADCS_TRY(cudaMemcpyAsync(d.bwt + from, d.deviceBwt + from, to - from, cudaMemcpyDeviceToHost, d.stream));
    }
    return cudaSuccess;
}

// Merges the class lists of the texts into sa and/or bwt (either may be null). splitters and rows
// are scratch sized by planMerge; counter is one device word (scratch); rowZero and outBase are per
// text (rowZero is filled here when a BWT is asked for); rowBase: the class tables' row bases.
inline cudaError_t mergeClasses(const uint8_t* text, const uint32_t* ranks, const TextSet& texts, const uint32_t* lists,
                                const MergePlan& plan, const uint32_t* rowBase, const uint32_t* outBase,
                                uint32_t* rowZero, uint32_t* splitters, MergeRow* rows, uint32_t* sa, uint8_t* bwt,
                                uint32_t* counter, uint32_t* hostWord, cudaStream_t stream,
                                cudaEvent_t finalStart = nullptr, cudaEvent_t finalStop = nullptr,
                                uint32_t* const* saTexts = nullptr, uint8_t* const* bwtTexts = nullptr,
                                const uint64_t* carried = nullptr, const OverlappedDownload* download = nullptr) {
    MergeLevel level[kMaxLevels];
    for (int L = 0; L <= plan.top; L++) {
        level[L].lists = L == 0 ? lists : splitters + plan.listWord[L];
        for (int b = 0; b <= kClasses; b++) level[L].start[b] = plan.start[L][b];
    }
    for (int L = 1; L <= plan.top; L++) {
        const uint32_t count = plan.start[L][kClasses];
        SADCS_TRY(launch(mergeGatherSplitters, (count + 255) / 256, 256, 0, stream, level[L - 1].lists, level[L - 1],
                         level[L], const_cast<uint32_t*>(level[L].lists)));
    }
    SADCS_TRY(cudaMemsetAsync(counter, 0, sizeof(uint32_t), stream));  // error word
    MergeArgs base{};
    base.text = text;
    base.ranks = ranks;
    base.texts = texts;
    base.outBase = outBase;
    base.rowZero = rowZero;
    base.error = counter;
    base.saTexts = saTexts;
    base.bwtTexts = bwtTexts;
    if (bwt || bwtTexts) {
        MergeArgs z = base;
        z.level = level[0];
        SADCS_TRY(cudaMemsetAsync(rowZero, 0, sizeof(uint32_t) * texts.count, stream));
        SADCS_TRY(launch(mergeSuffixZeroRows, texts.count, 32, 0, stream, z, rowBase, level[0], rowZero));
        SADCS_TRY(launch(mergeBwtHeads, (texts.count + 255) / 256, 256, 0, stream, text, texts, outBase, bwt, bwtTexts));
    }
    for (int L = plan.top; L >= 0; L--) {
        MergeArgs args = base;
        args.level = level[L];
        args.rowsIn = L == plan.top ? nullptr : rows + plan.rowIndex[L];
        const uint32_t tiles = L == plan.top ? 1 : plan.tiles[L];
        if (L == 0) {
            args.sa = sa;
            args.bwt = bwt;
            args.carried = carried;
            if (download && (download->sa || download->bwt)) {
                // In pieces, each piece's final outputs copied down while the next ones run.
                const int chunks = static_cast<int>(std::min<uint32_t>(kMaxDownloadChunks, args.rowsIn ? tiles : 1));
                uint32_t first[kMaxDownloadChunks + 1];
                for (int k = 0; k <= chunks; k++) {
                    first[k] = static_cast<uint32_t>(static_cast<uint64_t>(tiles) * k / chunks);
                }
                for (int k = 1; k < chunks; k++) {
                    SADCS_TRY(cudaMemcpyAsync(download->hostRows + 8 * (k - 1), args.rowsIn + first[k], sizeof(MergeRow),
                                              cudaMemcpyDeviceToHost, stream));
                }
                SADCS_TRY(cudaEventRecord(download->events[kMaxDownloadChunks], stream));
                if (finalStart) SADCS_TRY(cudaEventRecord(finalStart, stream));
                for (int k = 0; k < chunks; k++) {
                    args.tileOffset = first[k];
                    SADCS_TRY(launchTree<true>(args, first[k + 1] - first[k], stream));
                    SADCS_TRY(cudaEventRecord(download->events[k], stream));
                }
                if (finalStop) SADCS_TRY(cudaEventRecord(finalStop, stream));
                SADCS_TRY(cudaEventSynchronize(download->events[kMaxDownloadChunks]));  // the rows are here
                uint64_t done = 0;
                for (int k = 0; k < chunks; k++) {
                    uint64_t end = download->outputs;
                    if (k + 1 < chunks) {
                        MergeRow r;
                        std::memcpy(&r, download->hostRows + 8 * k, sizeof r);
                        end = std::min<uint64_t>(std::max<uint64_t>(tileOutputBound(r, plan.start[0]), done),
                                                 download->outputs);
                    }
                    SADCS_TRY(cudaStreamWaitEvent(download->stream, download->events[k], 0));
                    SADCS_TRY(copyDown(*download, done, end));
                    done = end;
                }
            } else {
                if (finalStart) SADCS_TRY(cudaEventRecord(finalStart, stream));
                SADCS_TRY(launchTree<true>(args, tiles, stream));
                if (finalStop) SADCS_TRY(cudaEventRecord(finalStop, stream));
            }
        } else {
            args.rowsOut = rows + plan.rowIndex[L - 1];
            SADCS_TRY(launch(mergeWriteSentinel, 1, 32, 0, stream, rows + plan.rowIndex[L - 1] + plan.tiles[L - 1],
                             level[L]));
            SADCS_TRY(launchTree<false>(args, tiles, stream));
        }
    }
    SADCS_TRY(cudaMemcpyAsync(hostWord, counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SADCS_TRY(cudaStreamSynchronize(stream));
    return *hostWord ? cudaErrorUnknown : cudaSuccess;
}

}  // namespace sadcs
