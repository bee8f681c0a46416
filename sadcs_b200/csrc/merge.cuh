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
// Inside the tile, each of the 21 pairs of windows is merged along a merge path cut into chunks
// (one diagonal search each, then one comparison per step); the walk records, for each element,
// how many elements of the other window precede it (each such count is written by exactly one
// thread, so no atomics). An element's output position is the windows' total start plus its index
// in its own window plus those counts; the tile writes the elements between s_lo and s_hi.
//
// Records (48 bytes, shared memory): the 16 text bytes at p, the 7 sample ranks of [p, p + 32)
// (all a comparison can need), and p. Comparisons reaching past 16 characters read the text.
#pragma once

#include "common.cuh"

namespace sadcs {

constexpr uint32_t kMergeG = 32;
constexpr uint32_t kMergeR = 32;
constexpr uint32_t kMergeCap = kMergeG * kMergeR + 6 * (kMergeG - 1) + 1;
constexpr int kMergeThreads = 256;
constexpr int kPairs = kClasses * (kClasses - 1) / 2;
constexpr uint32_t kNoList = 0xFFFFFFFFu;
constexpr int kMaxLevels = 10;

struct __align__(16) MergeRow {
    uint32_t list;
    uint32_t c[kClasses];
};

struct __align__(16) MergeRecord {
    uint64_t w0, w1;
    uint32_t rank[kK];
    uint32_t pos;
};
static_assert(sizeof(MergeRecord) == 48, "record size");

struct MergeLevel {
    const uint32_t* lists;
    uint32_t start[kClasses + 1];
};

struct MergeArgs {
    const uint8_t* text;
    const uint32_t* ranks;
    uint32_t n;
    MergeLevel level;
    const MergeRow* rowsIn;  // null: one tile over the whole level
    MergeRow* rowsOut;       // levels >= 1
    uint32_t* sa;            // level 0, optional
    uint8_t* bwt;            // level 0, optional: the final n-byte BWT
    uint32_t row0;           // output row of suffix 0
    uint32_t* error;         // set nonzero if a window set exceeds the capacity (never, by construction)
};

__device__ __forceinline__ uint64_t prefixMask(uint32_t c) {
    return c >= 8 ? ~uint64_t(0) : (c == 0 ? uint64_t(0) : ~uint64_t(0) << (64 - 8 * c));
}

__device__ __forceinline__ void loadRecord(const uint8_t* __restrict__ text, const uint32_t* __restrict__ ranks,
                                           uint32_t p, MergeRecord& r) {
    load16(text, p, r.w0, r.w1);
    const uint32_t base = pack(p);
#pragma unroll
    for (int s = 0; s < kK; s++) r.rank[s] = __ldg(ranks + base + s);
    r.pos = p;
}

__device__ __forceinline__ bool lessRecord(const MergeRecord& a, const MergeRecord& b,
                                           const uint8_t* __restrict__ text, uint32_t n) {
    const uint32_t i = a.pos, j = b.pos;
    const uint32_t k = cCover.tie[i % kV][j % kV];
    const uint32_t common = min(k, min(n - i, n - j));
    uint64_t x = a.w0, y = b.w0;
    if (common < 8) {
        const uint64_t mk = prefixMask(common);
        x &= mk;
        y &= mk;
    }
    if (x != y) return x < y;
    if (common > 8) {
        x = a.w1;
        y = b.w1;
        if (common < 16) {
            const uint64_t mk = prefixMask(common - 8);
            x &= mk;
            y &= mk;
        }
        if (x != y) return x < y;
        for (uint32_t o = 16; o < common; o += 8) {
            x = load8(text, i + o);
            y = load8(text, j + o);
            if (common - o < 8) {
                const uint64_t mk = prefixMask(common - o);
                x &= mk;
                y &= mk;
            }
            if (x != y) return x < y;
        }
    }
    if (common < k || i + k == n || j + k == n) return i > j;  // one is a prefix of the other
    return a.rank[cCover.slot[i % kV][k]] < b.rank[cCover.slot[j % kV][k]];
}

struct MergeTileInfo {
    uint32_t seg[kClasses + 1];
    uint32_t win[kClasses];
    uint32_t base, loIdx, hiIdx, lrLo, lrHi, size, chunk;
    uint32_t pairStart[kPairs + 1];
    uint8_t pairA[kPairs], pairB[kPairs];
    int bad;
};

constexpr size_t mergeSharedBytes() {
    return kMergeCap * sizeof(MergeRecord) + kMergeCap * 8 * sizeof(uint16_t) + kMergeCap * sizeof(uint32_t);
}

__device__ __forceinline__ int listOfElement(const uint32_t* seg, uint32_t e) {
    int l = 0;
    while (e >= seg[l + 1]) l++;
    return l;
}

template <bool kFinal>
__global__ void __launch_bounds__(kMergeThreads) mergeTiles(MergeArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    MergeRecord* rec = reinterpret_cast<MergeRecord*>(smem);
    uint16_t* cnt = reinterpret_cast<uint16_t*>(rec + kMergeCap);
    uint32_t* lr = reinterpret_cast<uint32_t*>(cnt + kMergeCap * 8);
    __shared__ MergeTileInfo t;

    if (threadIdx.x == 0) {
        const uint32_t* st = a.level.start;
        uint32_t w[kClasses], e[kClasses];
        uint32_t loList = kNoList, hiList = kNoList;
        if (!a.rowsIn) {
            for (int b = 0; b < kClasses; b++) {
                w[b] = 0;
                e[b] = st[b + 1] - st[b];
            }
        } else {
            const MergeRow lo = a.rowsIn[blockIdx.x];
            const MergeRow hi = a.rowsIn[blockIdx.x + 1];
            loList = lo.list;
            hiList = hi.list;
            for (int b = 0; b < kClasses; b++) {
                const uint32_t len = st[b + 1] - st[b];
                if (lo.list == kNoList) {
                    w[b] = 0;
                } else if (static_cast<uint32_t>(b) == lo.list) {
                    w[b] = lo.c[b] * kMergeG;
                } else {
                    w[b] = lo.c[b] == 0 ? 0 : (lo.c[b] - 1) * kMergeG + 1;
                }
                if (hi.list == kNoList) {
                    e[b] = len;
                } else if (static_cast<uint32_t>(b) == hi.list) {
                    e[b] = hi.c[b] * kMergeG + 1;
                } else {
                    e[b] = min(len, hi.c[b] * kMergeG);
                }
                w[b] = min(w[b], len);
                e[b] = max(min(e[b], len), w[b]);
            }
        }
        uint32_t base = 0;
        t.seg[0] = 0;
        for (int b = 0; b < kClasses; b++) {
            t.win[b] = w[b];
            t.seg[b + 1] = t.seg[b] + (e[b] - w[b]);
            base += w[b];
        }
        t.base = base;
        t.size = t.seg[kClasses];
        t.loIdx = loList == kNoList ? kNoList : t.seg[loList];
        t.hiIdx = hiList == kNoList ? kNoList : t.seg[hiList + 1] - 1;
        t.bad = t.size > kMergeCap;
        const uint32_t steps = (kClasses - 1) * t.size;
        const uint32_t lanes = kMergeThreads - kPairs;
        const uint32_t c = max(1u, (steps + lanes - 1) / lanes);
        uint32_t total = 0;
        int q = 0;
        for (int x = 0; x < kClasses; x++) {
            for (int y = x + 1; y < kClasses; y++, q++) {
                const uint32_t lenA = t.seg[x + 1] - t.seg[x], lenB = t.seg[y + 1] - t.seg[y];
                t.pairStart[q] = total;
                t.pairA[q] = static_cast<uint8_t>(x);
                t.pairB[q] = static_cast<uint8_t>(y);
                if (lenA && lenB) total += (lenA + lenB + c - 1) / c;
            }
        }
        t.pairStart[kPairs] = total;
        t.chunk = c;
        if (t.bad && a.error) atomicExch(a.error, 1u);
    }
    __syncthreads();
    if (t.bad) return;

    const uint32_t size = t.size;
    const uint32_t* st = a.level.start;
    for (uint32_t e = threadIdx.x; e < size; e += kMergeThreads) {
        const int l = listOfElement(t.seg, e);
        const uint32_t p = a.level.lists[st[l] + t.win[l] + (e - t.seg[l])];
        loadRecord(a.text, a.ranks, p, rec[e]);
    }
    uint32_t* cnt32 = reinterpret_cast<uint32_t*>(cnt);
    for (uint32_t i = threadIdx.x; i < size * 4; i += kMergeThreads) cnt32[i] = 0;
    __syncthreads();

    const uint32_t items = t.pairStart[kPairs], c = t.chunk;
    for (uint32_t item = threadIdx.x; item < items; item += kMergeThreads) {
        int q = 0;
        while (item >= t.pairStart[q + 1]) q++;
        const uint32_t la = t.pairA[q], lb = t.pairB[q];
        const uint32_t sa = t.seg[la], lenA = t.seg[la + 1] - sa;
        const uint32_t sb = t.seg[lb], lenB = t.seg[lb + 1] - sb;
        uint32_t d = (item - t.pairStart[q]) * c;
        const uint32_t end = min(d + c, lenA + lenB);
        uint32_t lo = d > lenB ? d - lenB : 0, hi = min(d, lenA);
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (lessRecord(rec[sa + mid], rec[sb + d - 1 - mid], a.text, a.n)) {
                lo = mid + 1;
            } else {
                hi = mid;
            }
        }
        uint32_t i = lo, j = d - lo;
        for (; d < end; d++) {
            if (j == lenB || (i < lenA && lessRecord(rec[sa + i], rec[sb + j], a.text, a.n))) {
                cnt[(sa + i) * 8 + lb] = static_cast<uint16_t>(j);
                i++;
            } else {
                cnt[(sb + j) * 8 + la] = static_cast<uint16_t>(i);
                j++;
            }
        }
    }
    __syncthreads();

    for (uint32_t e = threadIdx.x; e < size; e += kMergeThreads) {
        const int l = listOfElement(t.seg, e);
        uint32_t r = e - t.seg[l];
#pragma unroll
        for (int b = 0; b < kClasses; b++) r += b == l ? 0u : cnt[e * 8 + b];
        lr[e] = r;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        t.lrLo = t.loIdx == kNoList ? 0 : lr[t.loIdx];
        t.lrHi = t.hiIdx == kNoList ? size : lr[t.hiIdx];
    }
    __syncthreads();

    for (uint32_t e = threadIdx.x; e < size; e += kMergeThreads) {
        const uint32_t r = lr[e];
        if (r < t.lrLo || r >= t.lrHi) continue;
        const uint32_t g = t.base + r;
        if (g >= a.level.start[kClasses]) {  // cannot happen for a correct tiling; never write out of range
            atomicExch(a.error, 2u);
            continue;
        }
        if constexpr (kFinal) {
            const uint32_t p = rec[e].pos;
            if (a.sa) a.sa[g] = p;
            if (a.bwt && p != 0) a.bwt[g < a.row0 ? g + 1 : g] = a.text[p - 1];
        } else {
            if (g % kMergeR == 0) {
                const int l = listOfElement(t.seg, e);
                MergeRow row;
                row.list = static_cast<uint32_t>(l);
#pragma unroll
                for (int b = 0; b < kClasses; b++) {
                    row.c[b] = b == l ? t.win[l] + (e - t.seg[l]) : t.win[b] + cnt[e * 8 + b];
                }
                a.rowsOut[g / kMergeR] = row;
            }
        }
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

// out += number of elements of list threadIdx.x smaller than suffix 0: its output row.
__global__ void mergeSuffixZeroRow(MergeArgs a, uint32_t* out) {
    const int b = threadIdx.x;
    if (b >= kClasses) return;
    MergeRecord zero;
    loadRecord(a.text, a.ranks, 0, zero);
    const uint32_t* list = a.level.lists + a.level.start[b];
    uint32_t lo = 0, hi = a.level.start[b + 1] - a.level.start[b];
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        MergeRecord r;
        loadRecord(a.text, a.ranks, list[mid], r);
        if (lessRecord(r, zero, a.text, a.n)) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    atomicAdd(out, lo);
}

__global__ void mergeBwtHead(const uint8_t* __restrict__ text, uint32_t n, uint8_t* bwt) {
    if (threadIdx.x == 0 && n > 0) bwt[0] = text[n - 1];
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

inline MergePlan planMerge(const uint32_t* classStart) {
    MergePlan p;
    for (int b = 0; b <= kClasses; b++) p.start[0][b] = classStart[b];
    int L = 0;
    while (p.start[L][kClasses] > kMergeCap && L + 1 < kMaxLevels) {
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
        p.tiles[l] = (p.start[l + 1][kClasses] + kMergeR - 1) / kMergeR;
        p.rowIndex[l] = p.rows;
        p.rows += p.tiles[l] + 1;
    }
    p.tiles[L] = 1;
    return p;
}

// Merges the class lists of text into sa and/or bwt (either may be null). splitters and rows are
// scratch sized by planMerge; counter is one device word (scratch).
inline cudaError_t mergeClasses(const uint8_t* text, const uint32_t* ranks, uint32_t n, const uint32_t* lists,
                                const MergePlan& plan, uint32_t* splitters, MergeRow* rows, uint32_t* sa,
                                uint8_t* bwt, uint32_t* counter, uint32_t* hostWord, cudaStream_t stream,
                                uint32_t* row0Out) {
    static uint64_t configured[2] = {0, 0};
    int device = 0;
    SADCS_TRY(cudaGetDevice(&device));
    if (!(configured[0] >> (device & 63) & 1)) {
        SADCS_TRY(cudaFuncSetAttribute(mergeTiles<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(mergeSharedBytes())));
        SADCS_TRY(cudaFuncSetAttribute(mergeTiles<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(mergeSharedBytes())));
        configured[0] |= uint64_t(1) << (device & 63);
    }
    MergeLevel level[kMaxLevels];
    for (int L = 0; L <= plan.top; L++) {
        level[L].lists = L == 0 ? lists : splitters + plan.listWord[L];
        for (int b = 0; b <= kClasses; b++) level[L].start[b] = plan.start[L][b];
    }
    for (int L = 1; L <= plan.top; L++) {
        const uint32_t count = plan.start[L][kClasses];
        mergeGatherSplitters<<<(count + 255) / 256, 256, 0, stream>>>(level[L - 1].lists, level[L - 1], level[L],
                                                                      const_cast<uint32_t*>(level[L].lists));
        SADCS_TRY(cudaGetLastError());
    }
    SADCS_TRY(cudaMemsetAsync(counter, 0, 2 * sizeof(uint32_t), stream));  // [0] suffix 0's row, [1] error
    MergeArgs base{};
    base.text = text;
    base.ranks = ranks;
    base.n = n;
    base.error = counter + 1;
    uint32_t row0 = 0;
    if (bwt && n > 0) {
        MergeArgs z = base;
        z.level = level[0];
        mergeSuffixZeroRow<<<1, 32, 0, stream>>>(z, counter);
        SADCS_TRY(cudaGetLastError());
        SADCS_TRY(cudaMemcpyAsync(hostWord, counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        SADCS_TRY(cudaStreamSynchronize(stream));
        row0 = *hostWord;
        mergeBwtHead<<<1, 32, 0, stream>>>(text, n, bwt);
        SADCS_TRY(cudaGetLastError());
    }
    if (row0Out) *row0Out = row0;
    for (int L = plan.top; L >= 0; L--) {
        MergeArgs args = base;
        args.level = level[L];
        args.rowsIn = L == plan.top ? nullptr : rows + plan.rowIndex[L];
        const uint32_t tiles = L == plan.top ? 1 : plan.tiles[L];
        if (L == 0) {
            args.sa = sa;
            args.bwt = bwt;
            args.row0 = row0;
            mergeTiles<true><<<tiles, kMergeThreads, mergeSharedBytes(), stream>>>(args);
        } else {
            args.rowsOut = rows + plan.rowIndex[L - 1];
            mergeWriteSentinel<<<1, 32, 0, stream>>>(rows + plan.rowIndex[L - 1] + plan.tiles[L - 1], level[L]);
            mergeTiles<false><<<tiles, kMergeThreads, mergeSharedBytes(), stream>>>(args);
        }
        SADCS_TRY(cudaGetLastError());
    }
    SADCS_TRY(cudaMemcpyAsync(hostWord, counter + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SADCS_TRY(cudaStreamSynchronize(stream));
    return *hostWord ? cudaErrorUnknown : cudaSuccess;
}

}  // namespace sadcs
