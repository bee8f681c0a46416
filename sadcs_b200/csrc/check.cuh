// check.cuh - suffix array and BWT checks on the device (the reference's checker,
// src/common/checker.cpp:53-109 and :196-245, restated as data-parallel kernels).
//
// Suffix array (Burkhardt-Karkkainen): SA is a permutation (every entry in range, inverse SA
// written by scatter, each slot owned by exactly one entry), and every neighbour pair is in order
// by (T[SA[i]], ISA[SA[i] + 1]) with the empty suffix's rank -1.
//
// BWT: the LF mapping of the BWT (a stable counting pass on its bytes, the sentinel's row first)
// must be one cycle that, followed from the sentinel's row, spells the text backwards. The walk is
// sequential in the reference; here every row's text position is found by pointer jumping along
// LF (log2 n rounds), and then each row's byte is compared with the text byte before its position.
#pragma once

#include <algorithm>

#include "common.cuh"
#include "primitives.cuh"

namespace sadcs {

constexpr uint64_t kNoFailure = ~uint64_t(0);

// isa[p] = the largest i with sa[i] = p (isa zeroed by the caller), so that of equal entries the
// last one owns the slot whatever the order of the writes, as in a sequential scatter: the first
// duplicate reported is then the smallest index of any repeated entry, on every run.
__global__ void checkScatter(const uint32_t* __restrict__ sa, uint32_t n, uint32_t* __restrict__ isa,
                             unsigned long long* __restrict__ firstBad) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = sa[i];
    if (p >= n) {
        atomicMin(firstBad, static_cast<unsigned long long>(i));
    } else {
        atomicMax(isa + p, static_cast<uint32_t>(i));
    }
}

__global__ void checkDuplicates(const uint32_t* __restrict__ sa, uint32_t n, const uint32_t* __restrict__ isa,
                                unsigned long long* __restrict__ firstBad) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (isa[sa[i]] != i) atomicMin(firstBad, static_cast<unsigned long long>(i));
}

__global__ void checkOrder(const uint8_t* __restrict__ text, const uint32_t* __restrict__ sa, uint32_t n,
                           const uint32_t* __restrict__ isa, unsigned long long* __restrict__ firstBad) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i + 1 >= n) return;
    const uint32_t l = sa[i], r = sa[i + 1];
    bool ok = text[l] < text[r];
    if (text[l] == text[r]) {
        const int64_t ln = l + 1 < n ? static_cast<int64_t>(isa[l + 1]) : -1;
        const int64_t rn = r + 1 < n ? static_cast<int64_t>(isa[r + 1]) : -1;
        ok = ln < rn;
    }
    if (!ok) atomicMin(firstBad, static_cast<unsigned long long>(i));
}

}  // namespace sadcs

namespace sadcs {

// ---- BWT inversion by pointer jumping ----------------------------------------------------------
//
// Rows of the BWT matrix with the sentinel: n + 1; row r < primary holds bwt[r], row primary the
// sentinel, row r > primary bwt[r - 1]. LF maps the row of bwt[u] to the row of the suffix that
// starts one character earlier: 1 (the sentinel's suffix) + the smaller characters + the earlier
// occurrences of the same one, i.e. one plus u's position in a stable sort of the BWT bytes.
// Following LF from row 0 spells the text backwards and ends at the primary row after n steps
// (checker.cpp:196-245). Here every row's distance to the primary row along LF is found by pointer
// jumping (each round doubles the jump), and the row at distance d holds T[d - 1].

// lf[u] = 1 + sorted position of u, from the stable sort by byte (values = u in sorted order).
__global__ void lfScatter(const uint32_t* __restrict__ sortedU, uint32_t n, uint32_t* __restrict__ lf) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) lf[sortedU[s]] = s + 1;
}

// next[r] = LF of row r (the primary row points to itself), dist[r] = 1 (0 at the primary row).
__global__ void lfInitRows(const uint32_t* __restrict__ lf, uint32_t n, uint32_t primary, uint32_t* __restrict__ next,
                           uint32_t* __restrict__ dist) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > n) return;
    if (r == primary) {
        next[r] = r;
        dist[r] = 0;
    } else {
        const uint32_t u = r < primary ? r : r - 1;
        const uint32_t to = lf[u];
        next[r] = to <= n ? to : primary;
        dist[r] = 1;
    }
}

// One jump: dist += dist[next], next = next[next] (double-buffered). changed = 1 if any row has not
// reached the primary row.
__global__ void lfJump(const uint32_t* __restrict__ next, const uint32_t* __restrict__ dist, uint32_t n,
                       uint32_t primary, uint32_t* __restrict__ nextOut, uint32_t* __restrict__ distOut,
                       uint32_t* __restrict__ changed) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > n) return;
    const uint32_t to = next[r];
    const uint32_t d = dist[r] + dist[to];
    nextOut[r] = next[to];
    distOut[r] = d > n + 1 ? n + 1 : d;  // a cycle that misses the primary row stays bounded
    if (next[to] != primary) *changed = 1;
}

// text[dist[r] - 1] = the byte of row r, for every row but the primary. Rows whose distance is out
// of range (a broken BWT) are counted in bad.
__global__ void lfSpell(const uint8_t* __restrict__ bwt, const uint32_t* __restrict__ dist, uint32_t n,
                        uint32_t primary, uint8_t* __restrict__ text, unsigned long long* __restrict__ bad) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > n || r == primary) return;
    const uint32_t d = dist[r];
    if (d == 0 || d > n) {
        atomicMin(bad, 0ull);
        return;
    }
    text[d - 1] = bwt[r < primary ? r : r - 1];
}

// First text position where the inverse differs from the text.
__global__ void lfCompare(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b, uint32_t n,
                          unsigned long long* __restrict__ firstBad) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n && a[i] != b[i]) atomicMin(firstBad, static_cast<unsigned long long>(i));
}

struct ByteLoader {
    const uint8_t* __restrict__ bytes;
    __device__ __forceinline__ bool load(uint32_t, uint32_t i, uint32_t, uint8_t& k, uint32_t& d) const {
        k = bytes[i];
        d = k;
        return true;
    }
    __device__ __forceinline__ uint32_t value(uint32_t, uint32_t i, uint32_t) const { return i; }
};

struct ValueStorer {
    static constexpr bool kKeys = false;
    uint32_t* __restrict__ out;
    uint32_t limit;
    __device__ __forceinline__ void storeKey(uint32_t, uint32_t, uint8_t) const {}
    __device__ __forceinline__ void storeValue(uint32_t, uint32_t pos, uint32_t v) const {
        if (pos < limit) out[pos] = v;
    }
};

// Byte histogram (256 words, zeroed by the caller) of bytes[0, n).
__global__ void __launch_bounds__(256) byteHistogram(const uint8_t* __restrict__ bytes, uint32_t n,
                                                     uint32_t* __restrict__ counts) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t lt = (1u << (threadIdx.x & 31)) - 1;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t base = static_cast<uint64_t>(blockIdx.x) * blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        const uint32_t c = i < n ? bytes[i] : kNoDigit;
        const uint32_t peers = __match_any_sync(0xffffffffu, c);
        if (c != kNoDigit && (peers & lt) == 0) atomicAdd(&h[c], static_cast<uint32_t>(__popc(peers)));
    }
    __syncthreads();
    if (h[threadIdx.x]) atomicAdd(counts + threadIdx.x, h[threadIdx.x]);
}

// The stable pass by byte runs over chunks of kInverseChunk positions, each a segment with its own
// digit bases (the digit's start plus its count in the chunks before), so that no segment reaches the
// 2^30 counts a look-back word holds; one chunk below that size.
constexpr uint32_t kInverseChunk = 1u << 29;
constexpr uint32_t kInverseMaxChunks = 8;  // n < 2^32

// elementStart[s] / tileStart[s] of the chunks (s = 0..chunks). One thread per entry.
__global__ void inverseChunkTables(uint32_t n, uint32_t chunks, uint32_t* __restrict__ elementStart,
                                   uint32_t* __restrict__ tileStart) {
    const uint32_t s = threadIdx.x;
    if (s > chunks) return;
    const uint64_t e = min(static_cast<uint64_t>(s) * kInverseChunk, static_cast<uint64_t>(n));
    elementStart[s] = static_cast<uint32_t>(e);
    tileStart[s] = static_cast<uint32_t>((e + kSortTile - 1) / kSortTile);
}

// hist[s][d] (byte counts of chunk s) becomes the first output slot of byte d in chunk s: every
// smaller byte, then byte d in the chunks before. One block of 256 threads.
__global__ void __launch_bounds__(256) inverseChunkBases(uint32_t* __restrict__ hist, uint32_t chunks) {
    __shared__ uint32_t warpTotals[32];
    const uint32_t d = threadIdx.x;
    uint32_t total = 0;
    for (uint32_t s = 0; s < chunks; s++) total += hist[s * 256 + d];
    uint32_t all;
    const uint32_t inclusive = blockInclusiveScan<OpSum>(total, warpTotals, all);
    uint32_t base = inclusive - total;
    for (uint32_t s = 0; s < chunks; s++) {
        const uint32_t c = hist[s * 256 + d];
        hist[s * 256 + d] = base;
        base += c;
    }
}

// Inverts bwt (n bytes, primary) into text (n bytes) on the device. scratch: inverseScratchWords(n)
// words; hostWord: one page-locked word. *valid = false if the BWT is not a valid one (rows that
// never reach the primary row).
inline size_t inverseScratchWords(uint64_t n) {
    return 6 * static_cast<size_t>(n + 1) + 512 + radixScratchWords(n) + kInverseMaxChunks * 256 + 64;
}

inline cudaError_t inverseBwt(const uint8_t* bwt, uint32_t n, uint32_t primary, uint8_t* text, uint32_t* scratch,
                              uint32_t* hostWord, cudaStream_t stream, bool& valid) {
    valid = true;
    if (n == 0) return cudaSuccess;
    const size_t rows = static_cast<size_t>(n) + 1;  // offsets in 64 bits: 2 * rows passes 2^32 for n >= 2^31
    uint32_t* sorted = scratch;                   // rows
    uint32_t* lf = sorted + rows;                 // rows
    uint32_t* next[2] = {lf + rows, lf + 2 * rows};
    uint32_t* dist[2] = {next[1] + rows, next[1] + 2 * rows};
    uint32_t* words = dist[1] + rows;             // [256] changed, [258..259] first bad row
    uint32_t* radixWords = words + 512;
    uint32_t* hist = radixWords + radixScratchWords(n);  // [chunks][256], then the chunk tables
    uint32_t* elementStart = hist + kInverseMaxChunks * 256;  // 16 words, then tileStart (16)
    uint32_t* tileStart = elementStart + 16;
    const uint32_t chunks = ceilDiv(n, kInverseChunk);
    const RadixScratch radix(radixWords, n);
    SADCS_TRY(cudaMemsetAsync(words, 0, 512 * 4, stream));
    SADCS_TRY(cudaMemsetAsync(radix.control, 0, 8, stream));
    SADCS_TRY(cudaMemsetAsync(hist, 0, static_cast<size_t>(chunks) * 256 * 4, stream));
    for (uint32_t c = 0; c < chunks; c++) {
        const uint32_t count = std::min<uint32_t>(kInverseChunk, n - c * kInverseChunk);
        const uint32_t histBlocks = std::min<uint32_t>(ceilDiv(count, 256 * 16), 148 * 8);
        SADCS_TRY(launch(byteHistogram, histBlocks, 256, 0, stream, bwt + static_cast<size_t>(c) * kInverseChunk,
                         count, hist + static_cast<size_t>(c) * 256));
    }
    SADCS_TRY(launch(inverseChunkBases, 1, 256, 0, stream, hist, chunks));
    SADCS_TRY(launch(inverseChunkTables, 1, 32, 0, stream, n, chunks, elementStart, tileStart));
    SADCS_TRY((radixOnesweepPass<uint8_t, ByteLoader, ValueStorer, ManySegments>(
        ByteLoader{bwt}, ValueStorer{sorted, n}, ManySegments{tileStart, elementStart, chunks}, n, ceilDiv(n, kSortTile),
        hist, radix, stream)));
    SADCS_TRY(launch(lfScatter, ceilDiv(n, 256), 256, 0, stream, sorted, n, lf));
    SADCS_TRY(launch(lfInitRows, ceilDiv(n + 1ull, 256), 256, 0, stream, lf, n, primary, next[0], dist[0]));
    int cur = 0;
    for (int round = 0; round < 40; round++) {
        SADCS_TRY(cudaMemsetAsync(words + 256, 0, 4, stream));
        SADCS_TRY(launch(lfJump, ceilDiv(n + 1ull, 256), 256, 0, stream, next[cur], dist[cur], n, primary,
                         next[cur ^ 1], dist[cur ^ 1], words + 256));
        cur ^= 1;
        SADCS_TRY(cudaMemcpyAsync(hostWord, words + 256, 4, cudaMemcpyDeviceToHost, stream));
        SADCS_TRY(cudaStreamSynchronize(stream));
        if (!*hostWord) break;
    }
    unsigned long long* bad = reinterpret_cast<unsigned long long*>(words + 258);
    SADCS_TRY(cudaMemsetAsync(bad, 0xFF, 8, stream));
    SADCS_TRY(launch(lfSpell, ceilDiv(n + 1ull, 256), 256, 0, stream, bwt, dist[cur], n, primary, text, bad));
    SADCS_TRY(cudaMemcpyAsync(hostWord, bad, 4, cudaMemcpyDeviceToHost, stream));
    SADCS_TRY(cudaMemcpyAsync(hostWord + 1, radix.control + 1, 4, cudaMemcpyDeviceToHost, stream));
    SADCS_TRY(cudaStreamSynchronize(stream));
    if (hostWord[1]) return cudaErrorLaunchTimeout;
    valid = hostWord[0] == 0xFFFFFFFFu;
    return cudaSuccess;
}

}  // namespace sadcs
